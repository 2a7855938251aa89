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


def test_served_results_match_alone_fast_mode(gpu_lib, oracle_built):
    """Fast mode (atomic P2G: summation order differs between the mix and the
    scene alone): each served result matches the scene stepped alone and the
    FP32 oracle, measured on what the run changed (change_rel_l2 of positions),
    within the fast bound raised to the scene's FP32 precision floor."""
    from oracle.oracle import OracleScene
    from tests.parity import FAST_BOUNDS, change_rel_l2, noise_bounds, start_state, state_errors
    reqs = _requests()
    srv = MpmServer(hbm_budget=150e9, particles_capacity=1 << 16, grid_capacity=1 << 13, deterministic=False)
    results, rejected = srv.run(reqs)
    assert not rejected and not srv.failed and sorted(results) == [r.rid for r in reqs]
    for r in reqs:
        pipe = MpmPipeline()
        st = state_from_scene(r.scene)
        for _ in range(r.steps):
            pipe.step(st)
        alone = st.read_positions()
        start = start_state(r.scene)
        o32, o64 = OracleScene(r.scene, "f32"), OracleScene(r.scene, "f64")
        o32.step(r.steps)
        o64.step(r.steps)
        w32, w64 = o32.particles(), o64.particles()
        w64["pos"] = o64.positions_f64()
        bound = noise_bounds(FAST_BOUNDS, w32, w64, start)["pos"]
        got = results[r.rid].positions
        e_alone = change_rel_l2(got, alone, start["pos"], start["_floor"]["pos"])
        e_orc = change_rel_l2(got, w32["pos"], start["pos"], start["_floor"]["pos"])
        print(f"request {r.rid}: served vs alone {e_alone:.3e}, vs oracle {e_orc:.3e}, bound {bound:.1e}")
        assert e_alone <= bound and e_orc <= bound
        # the unmoved input fails the same check
        assert change_rel_l2(start["pos"], alone, start["pos"], start["_floor"]["pos"]) > bound


def test_grid_overflow_evicts_and_reports_the_scene(gpu_lib):
    """A request whose scene needs more grid blocks than the state holds
    (its admission estimate was too small) makes its step report the block
    capacity bit: the server evicts the scenes of that step, reports them in
    `failed`, and serves the next requests as if nothing had happened."""
    import copy
    sc = scenes.elastic_cube(n_side=8, seed=40)
    spread = copy.deepcopy(sc)
    k = np.arange(6, dtype=np.float32)
    pos = (np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3) * 8.0 + 6.5) * np.float32(sc.dx)
    spread.particles = spread.particles.__class__.concat([
        spread.particles.from_positions(pos.astype(np.float32), np.float32(sc.dx / 4), 1000.0,
                                        spread.particles.model[:1].repeat(len(pos), 0))])
    spread.grid_capacity = 8  # the estimate admits it; its 216 particles need 1728 blocks
    good = [Request(1 + i, scenes.elastic_cube(n_side=6, seed=41 + i), 20, 0.5 + 0.01 * i) for i in range(2)]
    reqs = [Request(0, spread, 20, 0.0)] + good
    srv = MpmServer(hbm_budget=150e9, particles_capacity=1 << 16, grid_capacity=1 << 9, deterministic=True)
    results, rejected = srv.run(reqs)
    assert not rejected
    assert list(srv.failed) == [0] and srv.failed[0].status & 2
    assert sorted(results) == [1, 2]
    for r in good:
        assert np.array_equal(results[r.rid].positions, _alone(r)), r.rid
