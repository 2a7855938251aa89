"""CPIC coupling on the GPU against the oracle: the deterministic build
follows the oracle's arithmetic (DET_BOUNDS on what the run changed, the same
affinity bits); the fast build (scatter P2G with the compatible /
incompatible split, fast-arithmetic G2P) changes summation order and fuses
multiply-adds (FAST_BOUNDS).  Errors are change_rel_l2 of positions, v, C and F (the error
over the oracle's own change from the start), FP64-oracle errors printed
beside them, and the unmoved input must fail the same check."""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene
from tests.parity import DET_BOUNDS, FAST_BOUNDS, assert_run_matches, start_state

pytestmark = pytest.mark.gpu


def _oracle64(sc, steps):
    from oracle.oracle import OracleScene
    o = OracleScene(sc, "f64")
    o.set_use_cpic(True)
    o.step(steps)
    out = o.particles()
    out["pos"] = o.positions_f64()
    return out


@pytest.mark.parametrize("deterministic", [True, False])
def test_cpic_matches_oracle(gpu_lib, oracle_built, deterministic):
    from oracle.oracle import OracleScene
    sc = scenes.cpic_drop()
    start = start_state(sc)
    pipe = MpmPipeline()
    st = state_from_scene(sc, deterministic=deterministic, use_cpic=True)
    for _ in range(sc.steps):
        pipe.step(st)
    st.synchronize()
    o = OracleScene(sc)
    o.set_use_cpic(True)
    o.step(sc.steps)
    g, want = st.read_particles(), o.particles()
    gc, wc = st.read_cdf(), o.cdf()
    assert_run_matches(f"cpic, deterministic={deterministic}", g, want, _oracle64(sc, sc.steps), start,
                       DET_BOUNDS if deterministic else FAST_BOUNDS)
    agree = (gc["affinity"] == wc["affinity"]).mean()
    print(f"cpic, deterministic={deterministic}: affinity agreement {agree:.4f}")
    assert (wc["affinity"] != 0).sum() > 100
    assert agree > (0.99 if deterministic else 0.95)


@pytest.mark.parametrize("deterministic", [True, False])
def test_cpic_trimesh_matches_oracle(gpu_lib, oracle_built, deterministic):
    """Trimesh colliders under CPIC: the library samples the same rigid
    particles as the oracle (bit for bit), and stepping the floor mesh plus
    the moving, spinning box mesh matches the oracle as the analytic case."""
    from oracle.oracle import OracleScene
    sc = scenes.cpic_trimesh()
    start = start_state(sc)
    pipe = MpmPipeline()
    st = state_from_scene(sc, deterministic=deterministic, use_cpic=True)
    o = OracleScene(sc)
    o.set_use_cpic(True)
    rg, ro = st.read_rigid_particles(), o.rigid_particles()
    assert len(ro["local"]) > 10000
    assert np.array_equal(rg["local"].view(np.uint32), ro["local"].view(np.uint32))
    assert np.array_equal(rg["collider"], ro["collider"]) and np.array_equal(rg["triangle"], ro["triangle"])
    for _ in range(sc.steps):
        pipe.step(st)
    st.synchronize()
    o.step(sc.steps)
    g, want = st.read_particles(), o.particles()
    gc, wc = st.read_cdf(), o.cdf()
    assert_run_matches(f"cpic trimesh, deterministic={deterministic}", g, want, _oracle64(sc, sc.steps), start,
                       DET_BOUNDS if deterministic else FAST_BOUNDS)
    agree = (gc["affinity"] == wc["affinity"]).mean()
    print(f"cpic trimesh, deterministic={deterministic}: affinity agreement {agree:.4f}")
    for bit in (5, 6):  # the floor mesh and the box mesh
        assert ((wc["affinity"] >> bit) & 1).sum() > 100
    assert agree > (0.99 if deterministic else 0.95)
    np.testing.assert_allclose(st.collider_pose(6), o.collider_pose(6), rtol=0, atol=1e-5)


def test_cpic_trimesh_resamples_with_the_cell_width(gpu_lib):
    """Rigid particles exist only with CPIC on, and follow the cell width."""
    sc = scenes.cpic_trimesh()
    st = state_from_scene(sc)
    assert st.num_rigid_particles() == 0
    st.set_use_cpic(True)
    n = st.num_rigid_particles()
    assert n > 10000
    st.set_cell_width(sc.dx * 2.0, sc.grid_capacity)
    assert 0 < st.num_rigid_particles() < n / 2
    st.set_use_cpic(False)
    assert st.num_rigid_particles() == 0


def test_cpic_trimesh_in_batched_scenes_matches_alone(gpu_lib, oracle_built):
    """Trimesh CPIC in batched-scene mode: each scene's rigid samples carry
    its key offset and its colliders' scene-local affinity bits, so in
    deterministic mode every scene of the batch steps bit for bit as it does
    alone, and in the fast mode (scatter P2G with the incompatible split)
    each stays within the fast bounds of its own oracle run."""
    from oracle.oracle import OracleScene
    from nexus_b200.mpm import batched_state_from_scenes
    scs = [scenes.cpic_trimesh(), scenes.cpic_drop()]
    steps = 60
    pipe = MpmPipeline()
    alone = []
    for sc in scs:
        st = state_from_scene(sc, deterministic=True, use_cpic=True)
        for _ in range(steps):
            pipe.step(st)
        alone.append(st.read_positions())
    bst, slots = batched_state_from_scenes(scs, deterministic=True)
    bst.set_use_cpic(True)
    assert bst.num_rigid_particles() > 10000
    for _ in range(steps):
        pipe.step(bst)
    bst.synchronize()
    for sc, sl, want in zip(scs, slots, alone):
        got = bst.read_scene_positions(sl)
        assert np.array_equal(got, want), (sc.name, np.abs(got - want).max())
    fst, fslots = batched_state_from_scenes(scs, deterministic=False)
    fst.set_use_cpic(True)
    for _ in range(steps):
        pipe.step(fst)
    fst.synchronize()
    for sc, sl in zip(scs, fslots):
        o = OracleScene(sc)
        o.set_use_cpic(True)
        o.step(steps)
        assert_run_matches(f"batched cpic {sc.name}, fast", fst.read_scene_particles(sl), o.particles(),
                           _oracle64(sc, steps), start_state(sc), FAST_BOUNDS)
