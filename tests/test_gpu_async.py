"""Tickets and asynchronous reads (GpuParticles::read_positions as an async
read): a read queued behind steps returns the positions at its place in the
stream, whatever is queued after it; tickets complete in order; a scene
removed right after its read still reads back intact."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import (MpmPipeline, NexusError, PinnedArray, batched_state_from_scenes, state_from_scene)

pytestmark = pytest.mark.gpu


def test_tickets_complete_in_order(gpu_lib):
    sc = scenes.elastic_cube(n_side=12)
    st = state_from_scene(sc)
    pipe = MpmPipeline()
    tickets = []
    for _ in range(6):
        pipe.step(st)
        tickets.append(st.fence())
    assert tickets == sorted(tickets) and len(set(tickets)) == 6
    st.ticket_wait(tickets[3])
    assert all(st.ticket_done(t) for t in tickets[:4])
    st.synchronize()
    assert all(st.ticket_done(t) for t in tickets)
    with pytest.raises(NexusError):
        st.ticket_done(0)
    with pytest.raises(NexusError):
        st.ticket_done(tickets[-1] + 1)  # not issued yet


@pytest.mark.parametrize("pinned", [True, False])
def test_async_read_is_ordered_on_the_stream(gpu_lib, pinned):
    sc = scenes.elastic_cube(n_side=16)
    st = state_from_scene(sc)
    pipe = MpmPipeline()
    for _ in range(10):
        pipe.step(st)
    want = st.read_positions()
    n = len(want)
    buf = PinnedArray((n, 3)) if pinned else None
    out = buf.array if pinned else np.zeros((n, 3), np.float32)
    t = st.read_positions_range_async(0, n, out)
    for _ in range(5):  # queued after the read: must not show in it
        pipe.step(st)
    st.ticket_wait(t)
    np.testing.assert_array_equal(out, want)
    part = np.zeros((100, 3), np.float32)
    t2 = st.read_positions_range_async(200, 100, part)
    st.ticket_wait(t2)
    np.testing.assert_array_equal(part, st.read_positions()[200:300])


def test_scene_removed_behind_its_read(gpu_lib):
    scs = [scenes.elastic_cube(n_side=6 + i, seed=41 + i) for i in range(3)]
    st, slots = batched_state_from_scenes(scs)[:2]
    pipe = MpmPipeline()
    for _ in range(8):
        pipe.step(st)
    want = [st.read_scene_positions(s) for s in slots]
    bufs = [PinnedArray((sc.n, 3)) for sc in scs]
    tickets = [st.read_scene_positions_async(s, b.array) for s, b in zip(slots, bufs)]
    st.remove_scenes(slots[:2])  # queued behind the reads, no wait
    for _ in range(3):
        pipe.step(st)
    st.ticket_wait(tickets[-1])
    for w, b in zip(want, bufs):
        np.testing.assert_array_equal(b.array, w)
    assert len(st) == scs[2].n


def test_scene_add_checks_the_key_region(gpu_lib):
    """A scene whose particles leave its key region (or are NaN) is refused;
    a large scene takes the threaded check, a small one the serial one."""
    from nexus_b200.models import ParticleModel
    from nexus_b200.mpm import NXM_E_INVALID, MpmState
    from nexus_b200.particles import ParticleBatch
    st = MpmState(grid_size=1 << 13, particles_capacity=1 << 20)
    st.set_cell_width(1.0 / 64.0, 1 << 13)
    st.set_simulation_params((0.0, 0.0, -9.81), 1.0e-4)
    st.enable_scenes(64)  # key region of a scene: coordinates in [-0.4375, 3.375)
    rng = np.random.default_rng(3)
    model = ParticleModel.elastic_neo_hookean(1.0e5, 0.3)
    big = ParticleBatch.from_positions(rng.uniform(0.2, 0.8, (200000, 3)), np.float32(1 / 256), 1000.0, model)
    st.add_scene(big)
    for n in (1000, 200000):
        for bad in (9.5, -3.0, np.nan):
            b = big.take(np.arange(n))
            b.pos[n // 2, 1] = bad
            with pytest.raises(NexusError) as e:
                st.add_scene(b)
            assert e.value.code == NXM_E_INVALID
    edge = big.take(np.arange(1000))
    edge.pos[0] = (3.37, -0.43, 0.0)  # inside, near both ends
    st.add_scene(edge)
    assert len(st) == 201000
