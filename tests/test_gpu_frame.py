"""Adaptive substeps (NexusPipeline::simulate's MPM part with the substep
count from the CFL bound): the count follows the bound, the clamps hold, and a
frame equals write_substep_params(n) plus n steps, bit for bit."""
import math

import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene

pytestmark = pytest.mark.gpu

FRAME_DT = 1.0 / 60.0


def _state(sc):
    st = state_from_scene(sc, deterministic=True)
    st.set_simulation_params(sc.gravity, FRAME_DT)
    return st


def test_frame_substeps_follow_the_bound(gpu_lib):
    sc = scenes.elastic_cube(n_side=12)
    pipe = MpmPipeline()
    st = _state(sc)
    bound, bits = st.estimate_timestep_bound()
    want = math.ceil(FRAME_DT / (bits / 1.0e12))
    assert want > 1
    n = pipe.simulate_frame(st)
    assert n == want
    ref = _state(sc)
    ref.write_substep_params(n)
    for _ in range(n):
        pipe.step(ref)
    np.testing.assert_array_equal(st.read_positions(), ref.read_positions())
    np.testing.assert_array_equal(st.read_velocities(), ref.read_velocities())
    # the next frame adapts again from the state it left
    _, bits2 = st.estimate_timestep_bound()
    assert pipe.simulate_frame(st) == math.ceil(FRAME_DT / (bits2 / 1.0e12))
    st.synchronize()


def test_frame_substep_clamps(gpu_lib):
    sc = scenes.elastic_cube(n_side=8)
    pipe = MpmPipeline()
    assert pipe.simulate_frame(_state(sc), 1, 5) == 5
    assert pipe.simulate_frame(_state(sc), 200, 300) == 200
    fixed = _state(sc)  # min = max: the reference's fixed substep count
    assert pipe.simulate_frame(fixed, 20, 20) == 20
