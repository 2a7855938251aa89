"""The accuracy checker of the parity tests can fail (CPU only, on the oracle).

The fast-mode contract bounds errors measured on what the run changed
(tests/parity.py change_rel_l2).  Checked here: an exact result scores 0; the
unmoved input scores 1 in every field that moved more than its noise floor and
fails every such bound; a run that stops
one step short of the oracle's fails the position bound; FP32 rounding (the
FP32 oracle against the FP64 one) passes."""
import numpy as np
import pytest

from nexus_b200 import scenes
from tests.parity import (FAST_BOUNDS, STATE_KEYS, change_rel_l2, check_state, moved_fields,
                          start_state, state_errors)


def _run(sc, steps, precision="f32"):
    from oracle.oracle import OracleScene
    o = OracleScene(sc, precision)
    o.step(steps)
    return o.particles()


@pytest.mark.parametrize("name", ["cube", "sandwater"])
def test_checker_rejects_unmoved_and_short_runs(oracle_built, name):
    sc = scenes.elastic_cube(n_side=12, steps=30) if name == "cube" else scenes.sand_water(scale=0.06, steps=30)
    start = start_state(sc)
    want = _run(sc, 30)
    err, bad = check_state(want, want, start, FAST_BOUNDS)
    assert not bad and all(v == 0.0 for v in err.values())
    # a step that returns its inputs unchanged scores exactly 1 in every field
    # that moved more than its noise floor, and fails those
    moved = moved_fields(want, start)
    assert "pos" in moved and "vel" in moved
    err0, bad0 = check_state({k: start[k] for k in STATE_KEYS}, want, start, FAST_BOUNDS)
    assert all(err0[k] == pytest.approx(1.0) for k in moved), err0
    assert set(moved) <= {b.split(":")[0] for b in bad0}
    # ... although its plain relative L2 of positions is far below 1e-3
    plain = np.linalg.norm(start["pos"].astype(np.float64) - want["pos"]) / np.linalg.norm(want["pos"])
    assert plain < 1e-3
    # one step short of the oracle's run
    short = _run(sc, 29)
    _, bad_short = check_state(short, want, start, FAST_BOUNDS)
    assert any(b.startswith("pos") for b in bad_short), bad_short
    # rounding alone (the FP64 oracle against the FP32 one) stays inside the fast bounds
    w64 = _run(sc, 30, "f64")
    err64, bad64 = check_state(w64, want, start, FAST_BOUNDS)
    print(name, "moved", moved, "f64 vs f32:", err64)
    assert not bad64, bad64


def test_change_rel_l2_edge_cases():
    a = np.ones((4, 3), np.float32)
    assert change_rel_l2(a, a, a) == 0.0
    assert change_rel_l2(a + 1, a, a) == float("inf")
    assert change_rel_l2(a, a + 2, a) == pytest.approx(1.0)
    assert change_rel_l2(a + 1, a + 2, a) == pytest.approx(0.5)
    # below the noise floor the error is measured against the floor
    b = np.ones((4, 3), np.float64)
    assert change_rel_l2(b + 1e-7, b, b, floor=1e-6) == pytest.approx(0.1, rel=1e-6)
