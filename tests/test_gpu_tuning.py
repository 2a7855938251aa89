"""The autotuner (nxm_state_autotune) on the GPU: launch shapes change only
how the step is scheduled, never what it computes.  Every tuned knob set to
its extreme values still matches the oracle (the sort bit for bit, the run
within the fast bounds), the tuner's decision lands in the process-wide
table, and a fresh state of the same kind applies it without trials."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, NexusError, state_from_scene, tuning_table
from tests.parity import FAST_BOUNDS, assert_run_matches, compare_sort, start_state

pytestmark = pytest.mark.gpu

EXTREMES = [
    dict(sort_batch=2, sort_ctas_per_sm=1, p2g_ctas_per_sm=1, g2p_ctas_per_sm=1, grid_ctas_per_sm=1,
         range_min_fill=1),
    dict(sort_batch=8, sort_ctas_per_sm=16, p2g_ctas_per_sm=2, g2p_ctas_per_sm=3, grid_ctas_per_sm=16,
         range_min_fill=1 << 30),  # every G2P launch takes the one-block-per-unit loop
]


@pytest.mark.parametrize("knobs", EXTREMES)
def test_launch_shapes_do_not_change_results(gpu_lib, oracle_built, knobs):
    from oracle.oracle import OracleScene
    sc = scenes.mixed_materials(n_side=8)
    pipe = MpmPipeline()
    st = state_from_scene(sc)
    st.set_tuning(**knobs)
    got = st.tuning()
    assert all(got[k] == v for k, v in knobs.items())
    pipe.debug_sort(st)
    st.synchronize()
    o = OracleScene(sc)
    o.sort()
    errs = compare_sort(st.headers(), st.sorted_ids(), o.headers(), o.sorted_ids(), exact_order=False)
    assert not errs, "\n".join(errs[:10])
    st2 = state_from_scene(sc)
    st2.set_tuning(**knobs)
    for _ in range(40):
        pipe.step(st2)
    st2.synchronize()
    o32, o64 = OracleScene(sc, "f32"), OracleScene(sc, "f64")
    o32.step(40)
    o64.step(40)
    w64 = o64.particles()
    w64["pos"] = o64.positions_f64()
    assert_run_matches(f"tuning {knobs}", st2.read_particles(), o32.particles(), w64, start_state(sc), FAST_BOUNDS)


def test_invalid_tuning_is_refused(gpu_lib):
    st = state_from_scene(scenes.elastic_cube(n_side=4))
    with pytest.raises(NexusError):
        st.set_tuning(sort_batch=3)
    with pytest.raises(NexusError):
        st.set_tuning(g2p_ctas_per_sm=5)


def test_autotune_fills_the_table_and_applies_it(gpu_lib):
    sc = scenes.sand_water(scale=0.2, steps=10)
    st = state_from_scene(sc)
    d = st.autotune(trial_steps=3)
    assert d["density"] > 0 and d["ms_after"] > 0 and d["ms_after"] <= d["ms_before"] * 1.0001
    assert st.tuning()["sort_batch"] == d["sort_batch"]
    table = tuning_table()
    assert any(e["density"] == d["density"] and e["scenes"] == d["scenes"] for e in table)
    fresh = state_from_scene(sc)
    a = fresh.autotune(trial_steps=0)
    assert {k: a[k] for k in ("sort_batch", "range_min_fill", "g2p_ctas_per_sm")} == \
        {k: d[k] for k in ("sort_batch", "range_min_fill", "g2p_ctas_per_sm")}
    pipe = MpmPipeline()
    for _ in range(3):
        pipe.step(fresh)
    fresh.synchronize()
    assert np.isfinite(fresh.read_positions()).all()
