"""Host calls whose device allocation fails (injected on the host by
nxm_debug_fail_allocation, as a full GPU would fail them; no GPU fault).

Adding a scene to a batched state that must grow fails in either of its two
allocations: the grown particle arrays, or the upload scratch after the growth.
Each time the call returns NXM_E_OOM and the state goes on as if the call had
not been made: its scenes step bit for bit as in a state that never saw the
call (deterministic mode), and a later add succeeds."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import (NXM_E_OOM, MpmPipeline, NexusError, batched_state_from_scenes,
                            debug_fail_allocation)

pytestmark = pytest.mark.gpu


def _mix():
    return [scenes.coupled_scene(s, dx=1.0 / 64.0, n_min=1500, n_max=3000, floor_vertices=21) for s in range(3)]


@pytest.mark.parametrize("which", [0, 1])  # 0: the grown particle arrays, 1: the upload scratch
def test_failed_allocation_leaves_the_batched_state_as_it_was(gpu_lib, which):
    mix = _mix()
    pipe = MpmPipeline()
    st, slots = batched_state_from_scenes(mix[:2], deterministic=True)  # capacity: exactly these two
    ref, rslots = batched_state_from_scenes(mix[:2], deterministic=True)
    for s in (st, ref):
        for _ in range(5):
            pipe.step(s)
    st.synchronize()
    third = mix[2]
    debug_fail_allocation(which)
    try:
        with pytest.raises(NexusError) as e:
            st.add_scene(third.particles, third.colliders, third.tri_vertices)
    finally:
        debug_fail_allocation(-1)
    assert e.value.code == NXM_E_OOM
    assert len(st) == len(ref)
    for s in (st, ref):
        for _ in range(10):
            pipe.step(s)
    st.synchronize()
    ref.synchronize()
    for a, b in zip(slots, rslots):
        assert np.array_equal(st.read_scene_positions(a), ref.read_scene_positions(b))
    # the state still grows and runs
    new = st.add_scene(third.particles, third.colliders, third.tri_vertices)
    for _ in range(3):
        pipe.step(st)
    st.synchronize()
    assert np.isfinite(st.read_scene_positions(new)).all()
