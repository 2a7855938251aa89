"""Parity at the benchmark's full size: the 2,000,000-particle sand + water
scene (dx = 1/256) stepped 100 times in the fast mode (block-ordered storage,
atomic P2G, the fast model forms) against the FP32 oracle on the same seeded
input, within the 1e-3 relative L2 contract for positions, with the same
particles disabled.  The oracle takes about a minute on the host cores."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene
from tests.parity import rel_l2

pytestmark = pytest.mark.gpu


def test_sand_water_full_size_100_steps(gpu_lib, oracle_built):
    from oracle.oracle import OracleScene
    sc = scenes.sand_water()
    assert sc.n == 2_000_000
    pipe = MpmPipeline()
    st = state_from_scene(sc)
    steps = 100
    for _ in range(steps):
        pipe.step(st)
    st.synchronize()
    g = st.read_particles()
    o = OracleScene(sc)
    o.step(steps)
    want = o.particles()
    err = rel_l2(g["pos"], want["pos"])
    verr = rel_l2(g["vel"], want["vel"])
    print(f"sand+water full size, {steps} steps: positions rel L2 {err:.3e}, velocities {verr:.3e}")
    assert np.array_equal(g["enabled"], want["enabled"])
    assert err < 1e-3
