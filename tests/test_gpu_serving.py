"""Serving form (continuous batching): every request's result is the same
as its scene stepped alone for its step budget, whatever else was in the mix
and whenever it was admitted.  Deterministic mode, so "the same" is bit for
bit; a tight HBM budget makes later requests wait for earlier ones."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene
from nexus_b200.serving import MpmServer, Request, footprint, latency_summary

pytestmark = pytest.mark.gpu


def _requests():
    scs = [scenes.elastic_cube(n_side=6 + i, seed=31 + i) for i in range(4)] + [scenes.mixed_materials(n_side=5)]
    steps = [20, 45, 30, 60, 25]
    return [Request(i, sc, st, arrival=0.01 * i) for i, (sc, st) in enumerate(zip(scs, steps))]


def _alone(req):
    pipe = MpmPipeline()
    st = state_from_scene(req.scene, deterministic=True)
    for _ in range(req.steps):
        pipe.step(st)
    return st.read_positions()


@pytest.mark.parametrize("tight", [False, True])
def test_served_results_match_alone(gpu_lib, tight):
    reqs = _requests()
    budget = 2.2 * max(footprint(r.scene) for r in reqs) if tight else 150e9
    srv = MpmServer(hbm_budget=budget, particles_capacity=1 << 16, grid_capacity=1 << 13, deterministic=True)
    results, rejected = srv.run(reqs)
    assert not rejected and sorted(results) == [r.rid for r in reqs]
    for r in reqs:
        got = results[r.rid].positions
        assert np.array_equal(got, _alone(r)), r.rid
    summ = latency_summary(results)
    assert summ["completed"] == len(reqs) and summ["p99_s"] >= summ["p50_s"] > 0
    if tight:  # at most two scenes fit at once: someone waited for a slot
        assert any(results[r.rid].admitted > r.arrival + 1e-3 for r in reqs)
