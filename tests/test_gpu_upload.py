"""Uploads through the pinned staging ring: many appends of varied sizes from
pageable arrays (and from pinned ones, copied directly), with parameter and
collider changes in between and no synchronisation until the read-back, so
the ring wraps and grows while earlier copies are still queued; every record
arrives intact and in order."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.models import ParticleModel
from nexus_b200.particles import ParticleBatch
from nexus_b200.mpm import MpmState

pytestmark = pytest.mark.gpu


def _batch(rng, n, model):
    b = ParticleBatch.from_positions(rng.uniform(0.2, 0.8, (n, 3)).astype(np.float32), np.float32(1 / 256), 1000.0,
                                     model)
    b.vel = rng.normal(0, 1, (n, 3)).astype(np.float32)
    b.def_grad = (np.eye(3, dtype=np.float32).reshape(1, 9) + rng.normal(0, 0.01, (n, 9))).astype(np.float32)
    b.phase = rng.uniform(0, 1, n).astype(np.float32)
    b.group_id = rng.integers(0, 7, n).astype(np.uint32)
    return b


def test_many_uploads_arrive_intact(gpu_lib):
    import torch
    rng = np.random.default_rng(11)
    models = [ParticleModel.elastic_neo_hookean(1e5, 0.3), ParticleModel.sand(3.5e5, 0.3), ParticleModel.water(1e5)]
    sc = scenes.elastic_cube(n_side=4)
    st = MpmState(grid_size=1 << 14, particles_capacity=1 << 22)
    st.set_cell_width(1 / 256, 1 << 14)
    batches = []
    for i in range(40):
        n = int(rng.integers(1000, 120000))
        b = _batch(rng, n, models[i % 3])
        if i % 7 == 3:  # pinned arrays: copied directly
            def pinned(a):
                t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
                v = t.numpy().view(a.dtype).reshape(a.shape)
                v[...] = a
                pinned.keep.append(t)
                return v
            pinned.keep = []
            b = ParticleBatch(**{k: pinned(getattr(b, k)) for k in ParticleBatch.__dataclass_fields__})
        st.append(b)
        batches.append(b)
        st.set_simulation_params((0.0, 0.0, -9.81), 1e-4 * (1 + i % 3))
        if i % 5 == 0:
            st.set_colliders(sc.colliders)
    want = ParticleBatch.concat(batches)
    np.testing.assert_array_equal(st.read_positions(), want.pos)
    np.testing.assert_array_equal(st.read_velocities(), want.vel)
    np.testing.assert_array_equal(st.read_def_grad(), want.def_grad)
    np.testing.assert_array_equal(st.read_mass(), want.mass)
    np.testing.assert_array_equal(st.read_models(), want.model)
    r = st.prep_readback(3)  # phase colours come from the uploaded phases
    np.testing.assert_allclose(r["color"][:, 1], np.float32(0.4) * want.phase, rtol=1e-6)
