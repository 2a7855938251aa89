"""Parity at the benchmark's full size: the 2,000,000-particle sand + water
scene (dx = 1/256) stepped 100 times in the fast mode (block-ordered storage,
atomic P2G, the fast model forms) against the FP32 oracle on the same seeded
input.  Positions (as displacements), velocities, C and F are checked on what
the run changed (change_rel_l2 within FAST_BOUNDS), with the same particles
disabled; FP64-oracle errors are printed beside them; the unchanged input must
fail the same check.  The oracle takes about a minute on the host cores."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene
from tests.parity import FAST_BOUNDS, assert_run_matches, rel_l2, start_state

pytestmark = pytest.mark.gpu


def test_sand_water_full_size_100_steps(gpu_lib, oracle_built):
    from oracle.oracle import OracleScene
    sc = scenes.sand_water()
    assert sc.n == 2_000_000
    start = start_state(sc)
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
    o64 = OracleScene(sc, "f64")
    o64.step(steps)
    want64 = o64.particles()
    want64["pos"] = o64.positions_f64()
    print(f"sand+water full size, {steps} steps: plain position rel L2 {rel_l2(g['pos'], want['pos']):.3e}")
    assert_run_matches(f"sand+water full size, {steps} steps", g, want, want64, start, FAST_BOUNDS)
