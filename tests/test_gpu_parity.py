"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integers (active blocks, per-bucket particle sets, neighbour relation) must
be bit-exact.  Floats are measured on what the run changed (tests/parity.py
change_rel_l2: the error divided by the oracle's own change from the start,
so a result that never moved scores 1): positions (the displacement), v, C
and F against the FP32 oracle within FAST_BOUNDS (fast mode: atomic scatter
P2G) or DET_BOUNDS (deterministic mode: canonical sort, gather-form P2G,
--fmad=false); the same errors against the FP64 oracle are printed beside
them, and every such check also runs on the unmoved input and must fail there.
"""
import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.mpm import MpmPipeline, state_from_scene, MpmState, NXM_E_CAPACITY, NexusError
from tests.parity import (DET_BOUNDS, FAST_BOUNDS, assert_run_matches, compare_sort, nodes_in_oracle_order,
                          rel_l2, start_state)

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-3   # relative L2 of positions after the run (fast mode)
DET_TOL = 1e-6    # relative L2 (deterministic mode)


@pytest.fixture(scope="module")
def pipe(gpu_lib, oracle_built):
    return MpmPipeline()


def _scene(name):
    if name == "cube":
        return scenes.elastic_cube(n_side=16, steps=100)
    if name == "mixed":
        return scenes.mixed_materials(n_side=8)
    if name == "sandwater":
        return scenes.sand_water(scale=0.12, steps=40)
    raise KeyError(name)


@pytest.mark.parametrize("name", ["cube", "mixed", "sandwater"])
@pytest.mark.parametrize("deterministic", [False, True])
def test_sort_matches_oracle(pipe, name, deterministic):
    from oracle.oracle import OracleScene
    sc = _scene(name)
    st = state_from_scene(sc, deterministic=deterministic)
    pipe.debug_sort(st)
    st.synchronize()
    o = OracleScene(sc)
    o.sort()
    errs = compare_sort(st.headers(), st.sorted_ids(), o.headers(), o.sorted_ids(), exact_order=deterministic)
    assert not errs, "\n".join(errs[:10])
    assert st.num_blocks() == o.num_blocks


@pytest.mark.parametrize("name", ["cube", "mixed"])
def test_p2g_deterministic_is_bit_exact(pipe, name):
    from oracle.oracle import OracleScene
    sc = _scene(name)
    rng = np.random.default_rng(5)
    sc.particles.aff[:] = (rng.standard_normal(sc.particles.aff.shape) * 3).astype(np.float32)
    st = state_from_scene(sc, deterministic=True)
    pipe.debug_sort(st, with_p2g=True)
    o = OracleScene(sc)
    o.sort()
    o.p2g()
    g = nodes_in_oracle_order(st.headers(), st.nodes(), o.headers())
    want = o.nodes()[:, :, :4]
    assert np.array_equal(g.view(np.uint32), want.view(np.uint32)), \
        f"max |diff| = {np.abs(g - want).max():.3e}"


@pytest.mark.parametrize("name", ["cube", "mixed"])
def test_p2g_fast_matches_within_rounding(pipe, name):
    from oracle.oracle import OracleScene
    sc = _scene(name)
    rng = np.random.default_rng(6)
    sc.particles.aff[:] = (rng.standard_normal(sc.particles.aff.shape) * 3).astype(np.float32)
    st = state_from_scene(sc, deterministic=False)
    pipe.debug_sort(st, with_p2g=True)
    o = OracleScene(sc, "f64")
    o.sort()
    o.p2g()
    g = nodes_in_oracle_order(st.headers(), st.nodes(), o.headers())
    want = o.nodes()[:, :, :4]
    assert rel_l2(g[..., 3], want[..., 3]) < 1e-6
    assert rel_l2(g[..., :3], want[..., :3]) < 1e-5


def _run_states(sc, deterministic, steps):
    from oracle.oracle import OracleScene
    pipe = MpmPipeline()
    st = state_from_scene(sc, deterministic=deterministic)
    for _ in range(steps):
        pipe.step(st)
    st.synchronize()
    o32, o64 = OracleScene(sc, "f32"), OracleScene(sc, "f64")
    o32.step(steps)
    o64.step(steps)
    return st, o32, o64


def _run_both(sc, deterministic, steps):
    st, o32, o64 = _run_states(sc, deterministic, steps)
    o64p = o64.particles()
    o64p["pos"] = o64.positions_f64()
    return st.read_particles(), o32.particles(), o64p




@pytest.mark.parametrize("deterministic", [False, True])
def test_elastic_cube_100_steps(pipe, deterministic):
    sc = scenes.elastic_cube(n_side=32, steps=100)
    start = start_state(sc)
    g, o, o64 = _run_both(sc, deterministic, 100)
    assert g["enabled"].all() and o["enabled"].all()
    assert_run_matches(f"elastic cube, deterministic={deterministic}", g, o, o64, start,
                       DET_BOUNDS if deterministic else FAST_BOUNDS)
    # the plain position error of the earlier contract, for reference
    assert rel_l2(g["pos"], o["pos"]) < (DET_TOL if deterministic else FAST_TOL)


@pytest.mark.parametrize("deterministic", [False, True])
def test_affine_velocity_field_is_transferred_exactly(pipe, deterministic):
    """APIC property on the CUDA path: an affine velocity field carried by
    the particles (C = A) comes back from P2G + G2P, v_p = A x_p + c, C = A."""
    from nexus_b200.models import ParticleModel
    from nexus_b200.particles import ParticleBatch, collider_array
    rng = np.random.default_rng(9)
    dx = 1.0 / 64.0
    pos = scenes.lattice_block((0.4, 0.4, 0.4), (12, 12, 12), dx, 5)
    b = ParticleBatch.from_positions(pos, np.float32(dx / 4), 1000.0, ParticleModel.elastic_neo_hookean(1e-3, 0.3))
    A = 0.5 * rng.standard_normal((3, 3))
    c = 0.3 * rng.standard_normal(3)
    x = pos.astype(np.float64)
    b.vel = (x @ A.T + c).astype(np.float32)
    b.aff = (b.mass.astype(np.float64)[:, None] * A.T.reshape(1, 9)).astype(np.float32)
    sc = scenes.Scene("affine", dx, 1.0e-4, (0.0, 0.0, 0.0), b, collider_array([]), 1, 4096)
    st = state_from_scene(sc, deterministic=deterministic)
    pipe.step(st)
    st.synchronize()
    g = st.read_particles()
    np.testing.assert_allclose(g["vel"], x @ A.T + c, rtol=0, atol=1e-5)
    aff = g["aff"].astype(np.float64).reshape(-1, 3, 3).transpose(0, 2, 1) / g["mass"][:, None, None]
    # C comes from sums of w v (x_i - x_p) scaled by 4 / dx^2: in fast mode the
    # atomic summation order changes run to run, which moves C by up to ~1e-4
    # (|A| ~ 0.5); a wrong transfer would be off by O(|A|)
    np.testing.assert_allclose(aff, np.broadcast_to(A, aff.shape), rtol=0, atol=1e-4 if deterministic else 3e-4)


@pytest.mark.parametrize("deterministic", [False, True])
def test_linear_momentum_is_conserved(pipe, deterministic):
    """No gravity, no colliders: the total momentum survives 20 steps of a
    stiff body with random velocities on the CUDA path."""
    from tests.test_oracle import _momentum_scene
    sc = _momentum_scene()
    p0 = (sc.particles.mass[:, None].astype(np.float64) * sc.particles.vel).sum(0)
    st = state_from_scene(sc, deterministic=deterministic)
    for _ in range(20):
        pipe.step(st)
    st.synchronize()
    g = st.read_particles()
    p1 = (g["mass"][:, None].astype(np.float64) * g["vel"]).sum(0)
    scale = (sc.particles.mass[:, None] * np.abs(sc.particles.vel)).sum()
    assert np.abs(p1 - p0).max() < 1e-5 * scale


@pytest.mark.parametrize("deterministic", [False, True])
def test_angular_momentum_is_conserved(pipe, deterministic):
    """APIC angular momentum (the affine part included) over 20 steps of a
    stiff body with random velocities on the CUDA path."""
    from tests.test_oracle import _momentum_scene, apic_angular_momentum
    sc = _momentum_scene()
    p = sc.particles
    l0, scale = apic_angular_momentum(p.pos, p.vel, p.aff, p.mass, sc.dx)
    st = state_from_scene(sc, deterministic=deterministic)
    for _ in range(20):
        pipe.step(st)
    st.synchronize()
    g = st.read_particles()
    l1, _ = apic_angular_momentum(g["pos"], g["vel"], g["aff"], g["mass"], sc.dx)
    assert np.abs(l1 - l0).max() < 1e-5 * scale


def test_sparse_blocks_fast_matches_oracle(pipe):
    """Particles scattered about two per block: each 256-position run of the
    fast G2P spans far more blocks than the four it stages at once, so it
    takes many passes; mixed with a dense cube (runs of one or two blocks)."""
    from nexus_b200.models import BoundaryCondition, ParticleModel
    from nexus_b200.particles import ParticleBatch, box_walls, collider_array
    rng = np.random.default_rng(12)
    dx = 1.0 / 64.0
    model = ParticleModel.elastic_neo_hookean(1.0e5, 0.3)
    sparse = ParticleBatch.from_positions(rng.uniform(0.15, 0.85, (3000, 3)), np.float32(dx / 4), 1000.0, model)
    sparse.vel = rng.normal(0.0, 0.5, (3000, 3)).astype(np.float32)
    dense = scenes.elastic_cube(n_side=16).particles
    batch = ParticleBatch.concat([sparse, dense])
    cols = collider_array(box_walls(0.0, 1.0, BoundaryCondition.slip(), BoundaryCondition.slip()))
    sc = scenes.Scene("sparse_blocks", dx, 1.0e-4, (0.0, 0.0, -9.81), batch, cols, 30, 16384)
    start = start_state(sc)
    g, o, o64 = _run_both(sc, False, 30)
    assert_run_matches("sparse blocks, fast", g, o, o64, start, FAST_BOUNDS)


@pytest.mark.parametrize("deterministic", [False, True])
def test_every_material_50_steps(pipe, deterministic):
    sc = scenes.mixed_materials(n_side=10)
    start = start_state(sc)
    g, o, o64 = _run_both(sc, deterministic, 50)
    # Deterministic mode follows the oracle's arithmetic except the 3x3 SVD of
    # the plastic models (float one-sided Jacobi here, double in the oracle)
    # and CUDA's logf / expf / sinf: the Drucker-Prager and snow particles'
    # return maps see F differing by float rounding, which their yield
    # decisions amplify to ~1e-4 of the run's velocity change.
    det = dict(DET_BOUNDS, vel=5e-4, aff=5e-3, def_grad=1e-3)
    assert_run_matches(f"mixed materials, deterministic={deterministic}", g, o, o64, start,
                       det if deterministic else FAST_BOUNDS)
    # plastic state words (Drucker-Prager, snow) follow the same trajectory.  The
    # accumulated hardening sums one return-mapping increment per step, each
    # computed from log singular values of a near-identity F: an f32 SVD (GPU)
    # and the oracle's f64 SVD differ by ~1e-7 in sigma, i.e. ~1e-4 relative in
    # a 1e-3 deviatoric strain, hence the 1e-3 bound even in deterministic mode.
    sand = (g["model"][:, 0] == 2) | (g["model"][:, 0] == 3)
    hard_g = g["model"][sand, 2].view(np.float32)
    hard_o = o["model"][sand, 2].view(np.float32)
    assert rel_l2(hard_g, hard_o) < (1e-3 if deterministic else 1e-2)


def test_sand_water_scaled_40_steps(pipe):
    sc = scenes.sand_water(scale=0.12, steps=40)
    start = start_state(sc)
    g, o, o64 = _run_both(sc, False, 40)
    assert_run_matches("sand+water (scaled), fast", g, o, o64, start, FAST_BOUNDS)


@pytest.mark.parametrize("deterministic", [False, True])
def test_trimesh_floor_100_steps(pipe, deterministic):
    """A cube dropped on a 800-triangle height field: BVH projection on the
    GPU against the oracle's brute-force closest-triangle search.  Equal
    distances to two triangles (points over a shared edge) may be resolved by
    a different triangle than the oracle's index-order scan, which moves the
    projected point by rounding only, hence 1e-5 in deterministic mode."""
    sc = scenes.trimesh_floor()
    start = start_state(sc)
    g, o, o64 = _run_both(sc, deterministic, sc.steps)
    bounds = dict(DET_BOUNDS, pos=1e-4, vel=1e-3, aff=1e-2, def_grad=1e-3) if deterministic else FAST_BOUNDS
    assert_run_matches(f"trimesh floor, deterministic={deterministic}", g, o, o64, start, bounds)
    # the mesh (heights >= 0.05) holds the cube up: without it the slip floor is at z = 0
    assert g["pos"][:, 2].min() > 0.05 - sc.dx


@pytest.mark.parametrize("name", ["cube", "mixed", "sandwater"])
def test_timestep_bound_matches_oracle(pipe, name):
    """CFL bound: the same fixed-point value as the f32 oracle on the uploaded
    state (random velocities and affine, so both terms matter), and within
    rounding after steps in either mode (fast mode: on reordered storage)."""
    from oracle.oracle import OracleScene
    sc = _scene(name)
    rng = np.random.default_rng(12)
    sc.particles.vel[:] = (rng.standard_normal(sc.particles.vel.shape) * 2.0).astype(np.float32)
    sc.particles.aff[:] = (rng.standard_normal(sc.particles.aff.shape) * 1e-3).astype(np.float32)
    o = OracleScene(sc)
    for deterministic in (False, True):
        st = state_from_scene(sc, deterministic=deterministic)
        dt, bits = st.estimate_timestep_bound()
        assert bits == o.timestep_bound_bits()
        assert dt == pytest.approx(bits / 1e12, rel=1e-6)
        for _ in range(10):
            pipe.step(st)
        _, bits10 = st.estimate_timestep_bound()
        o10 = OracleScene(sc)
        o10.step(10)
        assert bits10 == pytest.approx(o10.timestep_bound_bits(), rel=1e-5 if deterministic else 1e-3)


def test_upload_readback_roundtrip(pipe):
    sc = scenes.mixed_materials(n_side=4)
    rng = np.random.default_rng(9)
    p = sc.particles
    p.aff[:] = rng.standard_normal(p.aff.shape).astype(np.float32)
    p.def_grad[:] += (0.01 * rng.standard_normal(p.def_grad.shape)).astype(np.float32)
    st = state_from_scene(sc)
    got = st.read_particles()
    assert np.array_equal(got["pos"], p.pos) and np.array_equal(got["vel"], p.vel)
    assert np.array_equal(got["aff"], p.aff) and np.array_equal(got["def_grad"], p.def_grad)
    assert np.array_equal(got["mass"], p.mass) and np.array_equal(got["model"], p.model)
    assert got["enabled"].all()


def test_swap_and_shift_remove(pipe):
    sc = scenes.elastic_cube(n_side=4)
    st = state_from_scene(sc)
    pos = sc.particles.pos.copy()
    remaps = st.swap_remove([3, 10, 63, 10])
    # descending, deduplicated: 63 is the tail (dropped), 10 <- 62, 3 <- 61
    assert remaps == [(62, 10), (61, 3)]
    got = st.read_positions()
    assert len(st) == 61
    assert np.array_equal(got[10], pos[62]) and np.array_equal(got[3], pos[61])
    st.shift_remove(0, 5)
    assert len(st) == 56 and np.array_equal(st.read_positions()[0], got[5])
    pipe.step(st)
    st.synchronize()


def test_grid_capacity_overflow_is_reported(pipe):
    sc = scenes.elastic_cube(n_side=16)
    st = state_from_scene(sc, grid_capacity=8)
    pipe.step(st)
    with pytest.raises(NexusError) as e:
        st.synchronize()
    assert e.value.code == NXM_E_CAPACITY
    assert st.status(clear=True) & 2
    # no particle is lost or swapped: the ones without a block are carried over
    # unchanged, the others moved by less than one cell (velocity clamp dx/dt)
    got = st.read_positions()
    assert np.isfinite(got).all()
    assert np.abs(got - sc.particles.pos).max() <= sc.dx


def test_pipelined_status_arrives_one_call_late(pipe):
    """The status word a pipelined read enqueues (stored into mapped host
    memory by a kernel) is returned by the next call, in stream order."""
    sc = scenes.elastic_cube(n_side=16)
    ok = state_from_scene(sc)
    for _ in range(5):
        pipe.step(ok)
        assert ok.status_pipelined() == 0
    assert ok.status_pipelined() == 0
    bad = state_from_scene(sc, grid_capacity=8)
    assert bad.status_pipelined() == 0  # first call: nothing enqueued before it
    pipe.step(bad)
    assert bad.status_pipelined() == 0  # the word enqueued before the step
    assert bad.status_pipelined() & 2  # the step's overflow
    assert bad.status(clear=True) & 2
    assert bad.status_pipelined() & 2  # enqueued before the clear
    assert bad.status_pipelined() == 0  # enqueued after it


def test_sort_on_reordered_storage_matches_oracle(pipe):
    """After fast steps the records sit in block order; the sort of that storage
    reports particle ids and matches the oracle's sort of the same positions."""
    import copy
    from oracle.oracle import OracleScene
    sc = scenes.mixed_materials(n_side=8)
    st = state_from_scene(sc)
    for _ in range(5):
        pipe.step(st)
    pos = st.read_positions()
    pipe.debug_sort(st)
    st.synchronize()
    sc2 = copy.deepcopy(sc)
    sc2.particles.pos[:] = pos
    o = OracleScene(sc2)
    o.sort()
    errs = compare_sort(st.headers(), st.sorted_ids(), o.headers(), o.sorted_ids(), exact_order=False)
    assert not errs, "\n".join(errs[:10])


def test_edits_on_reordered_storage(pipe):
    """swap_remove / shift_remove / append address particles by id also after
    fast steps have left the records in block order."""
    sc = scenes.mixed_materials(n_side=6)
    st = state_from_scene(sc)
    for _ in range(4):
        pipe.step(st)
    before = st.read_particles()
    n = len(st)
    remaps = st.swap_remove([5, n - 1, 17])
    assert remaps == [(n - 2, 17), (n - 3, 5)]
    after = st.read_particles()
    idx = np.arange(n - 3)
    idx[17], idx[5] = n - 2, n - 3
    for k in ("pos", "vel", "aff", "def_grad", "mass", "model", "enabled"):
        assert np.array_equal(after[k], before[k][idx]), k
    st.shift_remove(10, 20)
    shifted = st.read_particles()
    keep = np.r_[0:10, 20:n - 3]
    for k in ("pos", "def_grad", "model"):
        assert np.array_equal(shifted[k], after[k][keep]), k
    extra = scenes.elastic_cube(n_side=4).particles
    m = len(st)
    st.append(extra)
    grown = st.read_particles()
    assert np.array_equal(grown["pos"][:m], shifted["pos"]) and np.array_equal(grown["pos"][m:], extra.pos)
    for _ in range(3):
        pipe.step(st)
    final = st.read_particles()
    assert np.isfinite(final["pos"]).all()
    assert np.abs(final["pos"][m:] - extra.pos).max() < 0.1


def test_graph_replay_counts_kernels(pipe):
    sc = scenes.elastic_cube(n_side=8)
    st = state_from_scene(sc)
    before = st.kernel_launches()
    for _ in range(3):
        pipe.step(st)
    st.synchronize()
    assert st.kernel_launches() - before >= 3 * 10


def test_particle_chunks(pipe):
    """NexusState chunk management (src/state.rs:665-774): add / extend /
    remove / remove_particles_from_chunk keep every particle's owner chunk and
    record through the swap-removals, also after fast steps (reordered storage)."""
    a = scenes.elastic_cube(n_side=6).particles
    b = scenes.mixed_materials(n_side=5).particles
    sc = scenes.elastic_cube(n_side=4)
    sc.particles.pos[:, 0] += np.float32(0.2)  # distinct from the n_side=6 cube's lattice (same seed)
    st = MpmState(grid_size=4096, particles_capacity=64)
    st.set_cell_width(sc.dx, 4096)
    st.set_simulation_params(sc.gravity, sc.dt)
    st.set_colliders(sc.colliders)
    ca = st.add_chunk(a)
    cb = st.add_chunk(b)
    st.extend_chunk(ca, sc.particles)
    assert st.chunk_len(ca) == a.n + sc.n and st.chunk_len(cb) == b.n
    owner = st.chunk_of_particles()
    assert (owner[:a.n] == ca).all() and (owner[a.n:a.n + b.n] == cb).all() and (owner[a.n + b.n:] == ca).all()
    for _ in range(3):
        pipe.step(st)
    before = st.read_positions()
    removed = st.remove_particles_from_chunk(cb, 40)
    assert removed == 40 and st.chunk_len(cb) == b.n - 40
    after = st.read_positions()
    owner2 = st.chunk_of_particles()
    assert (owner2 == cb).sum() == b.n - 40 and (owner2 == ca).sum() == a.n + sc.n
    # every surviving record is one of the records before, at most once, with its owner
    key = {tuple(p): o for p, o in zip(before.tolist(), owner.tolist())}
    assert len(key) == len(before)
    assert all(key[tuple(p)] == o for p, o in zip(after.tolist(), owner2.tolist()))
    st.remove_chunk(ca)
    assert len(st) == b.n - 40 and (st.chunk_of_particles() == cb).all()
    with pytest.raises(NexusError):
        st.chunk_len(ca)
    pipe.step(st)
    st.synchronize()
    assert np.isfinite(st.read_positions()).all()


def _batch_scenes():
    a = scenes.elastic_cube(n_side=12, seed=21)
    b = scenes.mixed_materials(n_side=6)
    c = scenes.trimesh_floor(n_side=10)
    return [a, b, c]


def test_batched_scenes_step_as_alone(pipe):
    """Several scenes in one state (one launch sequence per step): in
    deterministic mode every scene's particles are bit-identical to the same
    scene stepped alone, also after another scene is removed mid-run; in fast
    mode each stays within the fast tolerance of its own oracle run."""
    from nexus_b200.mpm import batched_state_from_scenes
    from oracle.oracle import OracleScene
    scs = _batch_scenes()
    alone = []
    for sc in scs:
        st = state_from_scene(sc, deterministic=True)
        for _ in range(30):
            pipe.step(st)
        alone.append(st.read_positions())
    bst, slots = batched_state_from_scenes(scs, deterministic=True)
    for _ in range(30):
        pipe.step(bst)
    for sc, sl, want in zip(scs, slots, alone):
        got = bst.read_scene_positions(sl)
        assert np.array_equal(got, want), (sc.name, np.abs(got - want).max())
    # remove the middle scene; the others continue exactly as alone
    bst.remove_scenes([slots[1]])
    for i in (0, 2):
        st = state_from_scene(scs[i], deterministic=True)
        for _ in range(40):
            pipe.step(st)
        alone[i] = st.read_positions()
    for _ in range(10):
        pipe.step(bst)
    for i in (0, 2):
        assert np.array_equal(bst.read_scene_positions(slots[i]), alone[i]), scs[i].name
    # fast mode (reordered storage, scatter P2G)
    fst, fslots = batched_state_from_scenes(scs, deterministic=False)
    for _ in range(30):
        pipe.step(fst)
    fst.synchronize()
    for sc, sl in zip(scs, fslots):
        o = OracleScene(sc)
        o.step(30)
        o64 = OracleScene(sc, "f64")
        o64.step(30)
        start = start_state(sc)
        g = fst.read_scene_particles(sl)
        want64 = o64.particles()
        want64["pos"] = o64.positions_f64()
        assert_run_matches(f"batched scene {sc.name}, fast", g, o.particles(), want64, start, FAST_BOUNDS)


def test_batched_scene_limits(pipe):
    from nexus_b200.mpm import batched_state_from_scenes, NXM_E_INVALID
    scs = _batch_scenes()[:1]
    st, _ = batched_state_from_scenes(scs)
    assert st.scene_capacity() == 31 * 15 * 31
    far = scenes.elastic_cube(n_side=4)
    far.particles.pos[:, 0] += np.float32(10.0)  # beyond the scene's key region
    with pytest.raises(NexusError) as e:
        st.add_scene(far.particles)
    assert e.value.code == NXM_E_INVALID
    with pytest.raises(NexusError):
        st.set_colliders(scs[0].colliders)  # colliders come per scene


def test_batched_coupled_scenes_step_as_alone(pipe):
    """Scenes with kinematic bodies (driven every step through the bulk velocity
    call) and trimesh floors: in a batch, bit-identical (deterministic mode) to
    each scene stepped alone with the same driving."""
    from nexus_b200.mpm import batched_state_from_scenes, batched_collider_offsets, drive_kinematics
    mix = [scenes.coupled_scene(s, dx=1.0 / 64.0, n_min=1500, n_max=3000, floor_vertices=21) for s in range(3)]
    dt = mix[0].dt
    alone = []
    for sc in mix:
        st = state_from_scene(sc, deterministic=True)
        for k in range(25):
            drive_kinematics(st, [sc], [0], k * dt)
            pipe.step(st)
        alone.append(st.read_positions())
    bst, slots = batched_state_from_scenes(mix, deterministic=True)
    offs = batched_collider_offsets(mix, slots)
    for k in range(25):
        drive_kinematics(bst, mix, offs, k * dt)
        pipe.step(bst)
    for sc, sl, want in zip(mix, slots, alone):
        assert np.array_equal(bst.read_scene_positions(sl), want), sc.name
    # the bodies moved as driven: pose integrated from the written velocities
    pose = bst.collider_pose(offs[0] + int(mix[0].kinematics[0, 0]))
    assert np.abs(pose[4:] - mix[0].colliders[int(mix[0].kinematics[0, 0])]["translation"]).max() > 0


def _bodies_in_the_box():
    """A coupled scene (trimesh floor, box walls, sand) whose eight bodies
    (cuboids, balls, capsules) are rotated, placed on and inside the sand
    box and move into it, spinning, so that many grid nodes lie within reach
    of several shapes."""
    sc = scenes.coupled_scene(0, dx=1.0 / 64.0, n_min=1500, n_max=3000, floor_vertices=21)
    lo, hi = sc.particles.pos.min(0), sc.particles.pos.max(0)
    rng = np.random.default_rng(7)
    for j, row in enumerate(sc.kinematics):
        i = int(row[0])
        q = rng.normal(size=4)
        sc.colliders[i]["rotation"] = (q / np.linalg.norm(q)).astype(np.float32)
        t = lo + (hi - lo) * rng.uniform(-0.1, 1.1, 3)
        sc.colliders[i]["translation"] = t.astype(np.float32)
        sc.colliders[i]["linvel"] = (0.5 * (0.5 * (lo + hi) - t) / np.linalg.norm(0.5 * (lo + hi) - t)).astype(np.float32)
        sc.colliders[i]["angvel"] = rng.uniform(-3.0, 3.0, 3).astype(np.float32)
    sc.kinematics = sc.kinematics[:0]  # constant velocities, no driving
    return sc


@pytest.mark.parametrize("deterministic", [False, True])
def test_rotated_bodies_in_the_sand_match_oracle(pipe, deterministic):
    """Grid-node collisions with rotated analytic shapes and a trimesh, every
    node near some shape: the per-block reach test that leaves out far
    colliders must leave the projections exactly as the oracle's full scan
    (deterministic bounds as for the trimesh floor: BVH ties)."""
    sc = _bodies_in_the_box()
    start = start_state(sc)
    st, o32, o64 = _run_states(sc, deterministic, 60)
    o64p = o64.particles()
    o64p["pos"] = o64.positions_f64()
    bounds = dict(DET_BOUNDS, pos=1e-4, vel=1e-3, aff=1e-2, def_grad=1e-3) if deterministic else FAST_BOUNDS
    assert_run_matches(f"rotated bodies, deterministic={deterministic}", st.read_particles(), o32.particles(), o64p,
                       start, bounds)
    # the bodies' poses, integrated once a step by the G2P launch, follow the
    # oracle's integration: quaternion and translation within float rounding
    for i in range(6, 14):
        got, want = st.collider_pose(i), o32.collider_pose(i)
        want0 = np.concatenate([sc.colliders[i]["rotation"], sc.colliders[i]["translation"]])
        assert np.abs(want[4:] - want0[4:]).max() > 5e-4, "the body moved"
        np.testing.assert_allclose(got, want, atol=1e-5, err_msg=f"collider {i}")


def test_hash_full_is_reported(pipe):
    """More distinct primary block keys than the hash has slots (a grid of 8
    blocks has a 1024-slot hash; 1331 particles 4 cells apart each sit in a
    block of their own): the step reports STATUS_HASH_FULL, synchronize raises
    NXM_E_HASH_FULL, and no particle is lost (those without a block are
    carried over unchanged)."""
    from nexus_b200.mpm import NXM_E_HASH_FULL
    from nexus_b200.models import ParticleModel
    from nexus_b200.particles import ParticleBatch, collider_array
    dx = 1.0 / 64.0
    k = np.arange(11, dtype=np.float32)
    pos = ((np.stack(np.meshgrid(k, k, k, indexing="ij"), -1).reshape(-1, 3) * 4.0 + 6.5) * np.float32(dx))
    b = ParticleBatch.from_positions(pos.astype(np.float32), np.float32(dx / 4), 1000.0,
                                     ParticleModel.elastic_neo_hookean(1e5, 0.3))
    sc = scenes.Scene("spread", dx, 1.0e-4, (0.0, 0.0, -9.81), b, collider_array([]), 1, 8)
    st = state_from_scene(sc)
    pipe.step(st)
    with pytest.raises(NexusError) as e:
        st.synchronize()
    assert e.value.code == NXM_E_HASH_FULL
    bits = st.status(clear=True)
    assert bits & 1 and bits & 2
    got = st.read_positions()
    assert np.isfinite(got).all() and np.abs(got - pos).max() <= dx


def test_sort_capacity_is_reported(pipe):
    """Deterministic mode orders each (block, z-slab) bucket in shared memory,
    4096 particles at most: a pile of 5000 particles inside one slab reports
    STATUS_SORT_CAPACITY (synchronize raises NXM_E_CAPACITY) instead of
    overrunning; the step still completes."""
    from nexus_b200.models import ParticleModel
    from nexus_b200.particles import ParticleBatch, collider_array
    dx = 1.0 / 64.0
    rng = np.random.default_rng(3)
    # x, y in cells [32.6, 35.4] dx, z in [32.55, 32.95] dx: associated cells
    # 32..34 in x and y and 32 in z, all in block (8, 8, 8), z-slab 0
    u = rng.uniform(0.0, 1.0, (5000, 3)).astype(np.float32)
    pos = (np.float32(32.0) + u * np.array([2.8, 2.8, 0.4], np.float32) +
           np.array([0.6, 0.6, 0.55], np.float32)) * np.float32(dx)
    b = ParticleBatch.from_positions(pos.astype(np.float32), np.float32(dx / 4), 1000.0,
                                     ParticleModel.elastic_neo_hookean(1e3, 0.3))
    sc = scenes.Scene("pile", dx, 1.0e-5, (0.0, 0.0, 0.0), b, collider_array([]), 1, 64)
    st = state_from_scene(sc, deterministic=True)
    pipe.step(st)
    with pytest.raises(NexusError) as e:
        st.synchronize()
    assert e.value.code == NXM_E_CAPACITY
    assert st.status(clear=True) & 8


def test_bulk_copy_wait_runs_out_into_a_status(pipe):
    """Waits on bulk copies are bounded: a barrier that no copy completes
    (nothing is issued) runs out of its rounds, the kernel records
    NXM_STATUS_COPY_TIMEOUT and returns, synchronize reports NXM_E_CUDA, and
    after the status is cleared the state steps on normally."""
    from nexus_b200.mpm import NXM_E_CUDA, _check
    sc = scenes.elastic_cube(n_side=8)
    st = state_from_scene(sc)
    _check(st.lib.nxm_debug_copy_wait_timeout(st.h, 1000), "debug_copy_wait_timeout")
    with pytest.raises(NexusError) as e:
        st.synchronize()
    assert e.value.code == NXM_E_CUDA
    assert st.status(clear=True) & 16
    for _ in range(3):
        pipe.step(st)
    st.synchronize()
    assert np.isfinite(st.read_positions()).all()
