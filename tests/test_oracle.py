"""Known-answer and property tests of the CPU oracle (no GPU).

The reference ships no MPM tests or fixtures, so these pin the oracle to the
mathematics of the cited shader code instead: closed forms, conservation
laws and brute-force recomputations.  The one pin against the reference's own
code is the prefix-sum CPU semantics (src_rbd/utils/prefix_sum.rs:112-136).
"""
import math

import numpy as np
import pytest

from nexus_b200 import scenes
from nexus_b200.models import ParticleModel, lame_lambda_mu
from nexus_b200.particles import ParticleBatch, Collider, collider_array
from nexus_b200.models import BoundaryCondition


def test_prefix_sum_matches_reference_cpu_semantics(oracle_built):
    o = oracle_built
    v = np.array([3, 0, 5, 1, 7, 2], np.uint32)
    # inclusive wrapping sum, shifted right, leading 0
    assert o.prefix_sum(v).tolist() == [0, 3, 3, 8, 9, 16]
    big = np.array([0xFFFFFFFF, 2, 1], np.uint32)
    assert o.prefix_sum(big).tolist() == [0, 0xFFFFFFFF, 1]


def test_pack_key_and_hash(oracle_built):
    o = oracle_built
    # grid.rs:101-106: 11/10/11 bits with offsets 1023/511/1023
    assert o.pack_key(0, 0, 0) == 0x3FF | (0x1FF << 11) | (0x3FF << 21)
    assert o.pack_key(-1023, -511, -1023) == 0
    k = o.pack_key(5, -3, 7)
    assert (k & 0x7FF) - 0x3FF == 5 and ((k >> 11) & 0x3FF) - 0x1FF == -3 and ((k >> 21) & 0x7FF) - 0x3FF == 7
    # Murmur3 fmix-style mix of grid.rs:430-436
    kk = 12345
    ref = (kk * 0xCC9E2D51) & 0xFFFFFFFF
    ref = ((ref << 15) | (ref >> 17)) & 0xFFFFFFFF
    ref = (ref * 0x1B873593) & 0xFFFFFFFF
    assert o.hash_key(kk) == ref


def test_quadratic_kernel_partition_of_unity(oracle_built):
    o = oracle_built
    for x in np.linspace(0.5, 1.5, 41):
        w = o.kernel_eval_all(float(x), "f64")
        assert abs(w.sum() - 1.0) < 1e-12
        # first moment: sum_i w_i (i - x) = 0 with nodes at 0, 1, 2
        assert abs(sum(w[i] * (i - x) for i in range(3))) < 1e-12
        # eval_all agrees with the branchless single-node eval
        for i in range(3):
            assert abs(w[i] - o.kernel_eval(i - x, "f64")) < 1e-12
    assert o.kernel_eval(1.5, "f64") == 0.0 and o.kernel_eval(-1.5, "f64") == 0.0
    assert o.kernel_eval(0.0, "f64") == 0.75


def test_block_of_point(oracle_built):
    o = oracle_built
    dx = 1.0 / 64.0
    # x = 10.4 dx -> round 10 -> assoc 9 -> block 2, cell 1; y = 0.6 dx -> assoc 0;
    # z = -3.2 dx -> round -3 -> assoc -4 -> block -1, cell 0
    b, a = o.block_of_point(dx, [10.4 * dx, 0.6 * dx, -3.2 * dx])
    assert b.tolist() == [2, 0, -1] and a.tolist() == [1, 0, 0]
    # round half away from zero: 2.5 -> 3
    b, a = o.block_of_point(1.0, [2.5, -2.5, 4.49])
    assert b.tolist() == [0, -1, 0] and a.tolist() == [2, 0, 3]


def _rot(axis, ang):
    axis = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * K @ K


def _cm(m):  # row-major 3x3 -> column-major 9
    return np.asarray(m, np.float32).T.reshape(9)


def _from_cm(v):
    return np.asarray(v, np.float64).reshape(3, 3).T


def test_neo_hookean_rest_and_rotation(oracle_built):
    o = oracle_built
    m = ParticleModel.elastic_neo_hookean(1e5, 0.3).gpu_words()
    tau, _, _ = o.model_update(m, _cm(np.eye(3)), np.zeros(9), "f64")
    assert np.abs(tau).max() < 1e-6
    # a rotation stores no energy; F enters as f32, so det F = 1 +- 1e-7 and
    # tau is zero up to (lambda + mu) * 1e-7
    tau, _, _ = o.model_update(m, _cm(_rot([1, 2, 3], 0.7)), np.zeros(9), "f64")
    assert np.abs(tau).max() < 1e-6 * 1e5
    # uniform stretch: tau = mu (s^2 - 1) I + lambda ln(s^3) I
    lam, mu = lame_lambda_mu(1e5, 0.3)
    s = 1.01
    tau, _, _ = o.model_update(m, _cm(np.eye(3) * s), np.zeros(9), "f64")
    expect = float(mu) * (s * s - 1) + float(lam) * math.log(s ** 3)
    assert np.allclose(_from_cm(tau), np.eye(3) * expect, rtol=1e-5, atol=1e-3)


def test_linear_corotated_rest_and_rotation(oracle_built):
    o = oracle_built
    m = ParticleModel.elastic(2e4, 0.25).gpu_words()
    for F in (np.eye(3), _rot([0, 0, 1], 1.2), _rot([1, -1, 0.5], -0.4)):
        tau, _, _ = o.model_update(m, _cm(F), np.zeros(9), "f64")
        assert np.abs(tau).max() < 2e-6 * 2e4


def test_elastic_stresses_closed_form(oracle_built):
    """Corotated (linear.rs): tau = 2 mu (F - R) F^T + lambda (J - 1) J I,
    for F = Q diag(s): 2 mu Q diag((s - 1) s) Q^T + lambda (J - 1) J I.
    Neo-Hookean (neo_hookean_elasticity.rs): tau = mu (F F^T - I) + lambda ln(J) I."""
    o = oracle_built
    lam, mu = (float(v) for v in lame_lambda_mu(3e4, 0.3))
    lin = ParticleModel.elastic(3e4, 0.3).gpu_words()
    nh = ParticleModel.elastic_neo_hookean(3e4, 0.3).gpu_words()
    rng = np.random.default_rng(8)
    for _ in range(5):
        Q = _rot(rng.standard_normal(3), rng.uniform(-1.0, 1.0))
        sv = rng.uniform(0.9, 1.1, 3)
        F = (Q @ np.diag(sv)).astype(np.float32).astype(np.float64)
        j = float(np.linalg.det(F))
        tau, _, _ = o.model_update(lin, _cm(F), np.zeros(9), "f64")
        want = 2 * mu * Q @ np.diag((sv - 1) * sv) @ Q.T + lam * (j - 1) * j * np.eye(3)
        assert np.allclose(_from_cm(tau), want, rtol=1e-4, atol=2e-2)
        G = F + 0.05 * rng.standard_normal((3, 3))  # a general F (shear too)
        G = G.astype(np.float32).astype(np.float64)
        tau, _, _ = o.model_update(nh, _cm(G), np.zeros(9), "f64")
        want = mu * (G @ G.T - np.eye(3)) + lam * math.log(np.linalg.det(G)) * np.eye(3)
        assert np.allclose(_from_cm(tau), want, rtol=1e-5, atol=1e-3)


def test_svd_reconstructs(oracle_built):
    o = oracle_built
    rng = np.random.default_rng(3)
    for _ in range(50):
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        u, s, vt = o.svd(_cm(F), "f64")
        U, Vt = _from_cm(u), _from_cm(vt)
        assert np.allclose(U @ np.diag(s) @ Vt, F, atol=1e-5)
        assert np.allclose(U.T @ U, np.eye(3), atol=1e-5)
        assert np.all(np.diff(s) <= 1e-7) and np.all(s >= 0)


def test_drucker_prager_tensile_and_inside_cone(oracle_built):
    o = oracle_built
    m = ParticleModel.sand(3.5e5, 0.3).gpu_words()
    # pure tension (positive volumetric strain, no cohesion): projected to exp(0/3) = I
    _, F, w = o.model_update(m, _cm(np.eye(3) * 1.05), np.zeros(9), "f64")
    assert np.allclose(_from_cm(F), np.eye(3), atol=1e-6)
    # compression with a small deviatoric part sits inside the cone: F unchanged
    # (gamma <= 0 -> invalid projection) and the plastic state untouched
    Fc = np.diag([0.98, 0.981, 0.979])
    _, F, w2 = o.model_update(m, _cm(Fc), np.zeros(9), "f64")
    assert np.allclose(_from_cm(F), Fc, atol=1e-6)
    assert np.array_equal(w2, m)
    # exactly hydrostatic strain (zero deviatoric part) is the degenerate case of
    # drucker_prager.rs:139: projected to the tip, exp(cohesion/3) I = I
    _, F, _ = o.model_update(m, _cm(np.eye(3) * 0.98), np.zeros(9), "f64")
    assert np.allclose(_from_cm(F), np.eye(3), atol=1e-6)
    # large shear is pulled back onto the cone: det and trace change, state advances
    Fs = np.array([[1.0, 0.2, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]) @ np.diag([0.99, 0.99, 0.99])
    _, F, w3 = o.model_update(m, _cm(Fs), np.zeros(9), "f64")
    assert not np.allclose(_from_cm(F), Fs, atol=1e-4)
    assert w3.view(np.float32)[2] > 1.0  # plastic hardening grew
    # cohesive sand: tensile projection goes to exp(cohesion/3) I
    mc = ParticleModel.cohesive_sand(3.5e5, 0.3, 0.003).gpu_words()
    _, F, _ = o.model_update(mc, _cm(np.eye(3) * 1.05), np.zeros(9), "f64")
    assert np.allclose(_from_cm(F), np.eye(3) * math.exp(0.001), atol=1e-6)


def test_snow_band_clamp_and_hardening(oracle_built):
    """snow.rs:452-488 in closed form: singular values inside [1 - theta_c,
    1 + theta_s] leave F and the plastic determinant alone (stress = the
    corotated stress of the same Lame parameters); outside, F is clamped,
    the plastic determinant takes the ratio (clamped to [0.1, 4]) and the
    Lame parameters scale by exp(h (1 - J_p))."""
    o = oracle_built
    E, nu = 1.4e5, 0.2
    m = ParticleModel.snow(E, nu).gpu_words()
    lin = ParticleModel.elastic(E, nu).gpu_words()
    tc, ts, h = float(np.float32(2.5e-2)), float(np.float32(7.5e-3)), 10.0
    Fin = _rot([1, 2, 0.5], 0.3) @ np.diag([1.004, 0.99, 0.98])
    tau, F, w = o.model_update(m, _cm(Fin), np.zeros(9), "f64")
    tl, _, _ = o.model_update(lin, _cm(Fin), np.zeros(9), "f64")
    assert np.allclose(_from_cm(F), Fin, atol=1e-6)
    assert abs(float(w.view(np.float32)[1]) - 1.0) < 1e-6
    assert np.allclose(tau, tl, rtol=1e-5, atol=1e-3)
    for s_, c in ((1.02, 1.0 + ts), (0.96, 1.0 - tc)):
        tau, F, w = o.model_update(m, _cm(np.eye(3) * s_), np.zeros(9), "f64")
        assert np.allclose(_from_cm(F), np.eye(3) * c, atol=1e-6)
        pdet = (float(np.float32(s_)) / c) ** 3
        assert abs(float(w.view(np.float32)[1]) - pdet) < 1e-5
        tl, _, _ = o.model_update(lin, _cm(np.eye(3) * c), np.zeros(9), "f64")
        assert np.allclose(tau, tl * math.exp(h * (1.0 - pdet)), rtol=1e-4, atol=1e-2)
    _, _, w = o.model_update(m, _cm(np.eye(3) * 2.0), np.zeros(9), "f64")
    assert w.view(np.float32)[1] == np.float32(4.0)


def test_fluid_pressure_and_volume_only(oracle_built):
    o = oracle_built
    m = ParticleModel.water(1e5).gpu_words()
    tau, _, _ = o.model_update(m, _cm(np.eye(3)), np.zeros(9), "f64")
    assert np.abs(tau).max() < 1e-6  # p(1) = 0, no strain rate
    j = 0.97 ** 3
    tau, _, _ = o.model_update(m, _cm(np.eye(3) * 0.97), np.zeros(9), "f64")
    p = 1e5 * (j ** -7 - 1)
    assert np.allclose(_from_cm(tau), -p * j * np.eye(3), rtol=1e-5)


def test_fluid_viscous_stress(oracle_built):
    """fluid.rs: tau = 2 eta J dev(S) - p(J) J I with S = (L + L^T) / 2."""
    o = oracle_built
    eta, k, gamma = 0.5, 1e5, 7.0
    m = ParticleModel.fluid(k, gamma, eta).gpu_words()
    L = np.random.default_rng(4).standard_normal((3, 3))
    S = 0.5 * (L + L.T)
    dev = S - np.trace(S) / 3.0 * np.eye(3)
    for c in (1.0, 0.98):
        tau, _, _ = o.model_update(m, _cm(np.eye(3) * c), _cm(L), "f64")
        j = float(np.float32(c)) ** 3
        p = k * (j ** -gamma - 1.0)
        assert np.allclose(_from_cm(tau), 2 * eta * j * dev - p * j * np.eye(3), rtol=1e-5, atol=1e-4)


def test_boundary_condition_projection(oracle_built):
    o = oracle_built
    n = np.array([0, 0, 1], np.float32)
    v = np.array([1.0, -2.0, -3.0], np.float32)
    assert np.allclose(o.bc_project(0, 0.0, v, n), 0)
    assert np.allclose(o.bc_project(1, 0.0, v, n), [1, -2, 0])
    # separate with friction 0.5: tangent |(1,-2)| reduced by 0.5*3
    t = math.sqrt(5.0)
    assert np.allclose(o.bc_project(2, 0.5, v, n), np.array([1, -2, 0]) / t * (t - 1.5), atol=1e-6)
    assert np.allclose(o.bc_project(2, 0.5, np.array([1, 1, 2], np.float32), n), [1, 1, 2])
    assert np.allclose(o.bc_project(3, 0.0, v, n), v)


def _scene_with(colliders, n=8):
    pos = np.full((n, 3), 0.5, np.float32)
    b = ParticleBatch.from_positions(pos, 0.01, 1000.0, ParticleModel.elastic(1e3, 0.2))
    return scenes.Scene("probe", 1.0 / 64, 1e-4, (0, 0, 0), b, collider_array(colliders), 1, 64)


def test_shape_projections(oracle_built):
    from oracle.oracle import OracleScene
    cols = [Collider.cuboid((0.2, 0.1, 0.3), (0.5, 0.5, 0.5), BoundaryCondition.slip()),
            Collider.ball(0.25, (0.1, 0.2, 0.3), BoundaryCondition.slip()),
            Collider.capsule((0.0, 0.0, -0.2), (0.0, 0.0, 0.2), 0.1, (0.7, 0.7, 0.7), BoundaryCondition.slip())]
    sc = OracleScene(_scene_with(cols))
    # cuboid: outside point clamps to the box; inside point goes to the nearest face
    p, inside = sc.project_point(0, [0.9, 0.5, 0.5])
    assert inside == 0 and np.allclose(p, [0.7, 0.5, 0.5], atol=1e-6)
    p, inside = sc.project_point(0, [0.5, 0.58, 0.5])
    assert inside == 1 and np.allclose(p, [0.5, 0.6, 0.5], atol=1e-6)
    # ball
    p, inside = sc.project_point(1, [0.1, 0.2, 0.9])
    assert inside == 0 and np.allclose(p, [0.1, 0.2, 0.55], atol=1e-6)
    p, inside = sc.project_point(1, [0.1, 0.3, 0.3])
    assert inside == 1 and np.allclose(p, [0.1, 0.45, 0.3], atol=1e-6)
    # capsule: beside the segment and beyond a cap
    p, inside = sc.project_point(2, [0.9, 0.7, 0.7])
    assert inside == 0 and np.allclose(p, [0.8, 0.7, 0.7], atol=1e-6)
    p, inside = sc.project_point(2, [0.7, 0.7, 1.2])
    assert inside == 0 and np.allclose(p, [0.7, 0.7, 1.0], atol=1e-6)


def test_activation_set_is_every_particles_block_neighbourhood(oracle_built):
    from oracle.oracle import OracleScene
    sc = scenes.mixed_materials(n_side=6)
    o = OracleScene(sc)
    o.sort()
    h = o.headers()
    got = {tuple(r[:3]) for r in h}
    dx = sc.dx
    pos = sc.particles.pos.astype(np.float32)
    assoc = np.round(pos / np.float32(dx)) - 1
    blk = np.floor(assoc / 4).astype(np.int64)
    want = set()
    for b in {tuple(r) for r in blk}:
        for s in range(8):
            want.add((b[0] + (s >> 2 & 1), b[1] + (s >> 1 & 1), b[2] + (s & 1)))
    assert got == want
    # every particle is the primary of exactly one block, and appears as extra
    # exactly where its stencil spills (bucket invariants)
    sorted_ids = o.sorted_ids()
    prim = np.concatenate([sorted_ids[r[3]:r[3] + r[4]] for r in h])
    assert np.array_equal(np.sort(prim), np.arange(sc.n))
    total_extras = int(h[:, 5].sum() - h[:, 4].sum())
    a_local = (assoc - blk * 4).astype(np.int64)
    spill = (a_local >= 2)
    expect = sum(int(np.prod([1 + int(s) for s in row])) - 1 for row in spill)
    assert total_extras == expect
    # within a block's primaries, the ids are grouped by ascending z-slab
    for r in h:
        seg = sorted_ids[r[3]:r[3] + r[4]]
        slabs = a_local[seg, 2]
        assert np.all(np.diff(slabs) >= 0)


def test_p2g_conserves_mass_and_momentum_fp64(oracle_built):
    from oracle.oracle import OracleScene
    sc = scenes.mixed_materials(n_side=5)
    rng = np.random.default_rng(0)
    sc.particles.aff[:] = rng.standard_normal(sc.particles.aff.shape).astype(np.float32)
    o = OracleScene(sc, "f64")
    o.sort()
    o.p2g()
    nodes = o.nodes().reshape(-1, 8).astype(np.float64)
    m = sc.particles.mass.astype(np.float64)
    # (node values come back rounded to f32, hence the 1e-6 relative bound)
    assert abs(nodes[:, 3].sum() - m.sum()) < 1e-6 * m.sum()
    # APIC: the affine term has zero net momentum (first moment of the kernel vanishes)
    mom = (sc.particles.vel.astype(np.float64) * m[:, None]).sum(0)
    assert np.allclose(nodes[:, :3].sum(0), mom, rtol=1e-6, atol=1e-9)


def test_free_fall_and_uniform_translation(oracle_built):
    from oracle.oracle import OracleScene
    sc = scenes.elastic_cube(n_side=8, steps=10)
    sc.colliders = sc.colliders[:0]
    sc.particles.vel[:] = np.array([0.3, -0.2, 0.0], np.float32)
    o = OracleScene(sc, "f64")
    o.step(10)
    p = o.particles()
    t = 10 * sc.dt
    assert np.allclose(p["vel"], [0.3, -0.2, -9.81 * t], atol=1e-6)
    assert p["enabled"].all()
    x0 = sc.particles.pos.astype(np.float64)
    disp = p["pos"].astype(np.float64) - x0
    # uniform translation: every particle moves by the same amount (rigid motion)
    assert np.abs(disp - disp.mean(0)).max() < 1e-6


def test_affine_velocity_field_is_transferred_exactly(oracle_built):
    """APIC (p2g.rs / g2p.rs): particles carrying an affine velocity field
    v(x) = A x + c with C = A give it back after P2G + G2P, v_p = A x_p + c and
    C = A, since quadratic B-splines reproduce linear functions.  No gravity,
    no colliders, a vanishing stiffness (the stored affine is m A minus the
    stress term)."""
    from oracle.oracle import OracleScene
    from nexus_b200.particles import ParticleBatch, collider_array
    from nexus_b200.scenes import Scene, lattice_block
    rng = np.random.default_rng(9)
    dx = 1.0 / 64.0
    pos = lattice_block((0.4, 0.4, 0.4), (12, 12, 12), dx, 5)
    b = ParticleBatch.from_positions(pos, np.float32(dx / 4), 1000.0, ParticleModel.elastic_neo_hookean(1e-3, 0.3))
    A = 0.5 * rng.standard_normal((3, 3))
    c = 0.3 * rng.standard_normal(3)
    x = pos.astype(np.float64)
    b.vel = (x @ A.T + c).astype(np.float32)
    b.aff = (b.mass.astype(np.float64)[:, None] * A.T.reshape(1, 9)).astype(np.float32)  # column-major m A
    sc = Scene("affine", dx, 1.0e-4, (0.0, 0.0, 0.0), b, collider_array([]), 1, 4096)
    o = OracleScene(sc, "f64")
    o.step(1)
    got = o.particles()
    np.testing.assert_allclose(got["vel"], x @ A.T + c, rtol=0, atol=2e-6)
    aff = got["aff"].astype(np.float64).reshape(-1, 3, 3).transpose(0, 2, 1) / got["mass"][:, None, None]
    np.testing.assert_allclose(aff, np.broadcast_to(A, aff.shape), rtol=0, atol=1e-5)
    np.testing.assert_allclose(got["pos"], x + got["vel"].astype(np.float64) * 1.0e-4, rtol=0, atol=1e-7)


def _momentum_scene():
    from nexus_b200.particles import ParticleBatch, collider_array
    from nexus_b200.scenes import Scene, lattice_block
    dx = 1.0 / 64.0
    pos = lattice_block((0.4, 0.4, 0.4), (12, 12, 12), dx, 6)
    b = ParticleBatch.from_positions(pos, np.float32(dx / 4), 1000.0, ParticleModel.elastic_neo_hookean(1e5, 0.3))
    b.vel = (0.5 * np.random.default_rng(10).standard_normal(pos.shape)).astype(np.float32)
    return Scene("momentum", dx, 1.0e-4, (0.0, 0.0, 0.0), b, collider_array([]), 20, 4096)


def test_linear_momentum_is_conserved(oracle_built):
    """No gravity, no colliders: P2G, the grid update and G2P keep the total
    momentum (the APIC term sums to zero over a stencil, internal forces
    cancel), while the random velocities deform the body."""
    from oracle.oracle import OracleScene
    sc = _momentum_scene()
    p0 = (sc.particles.mass[:, None].astype(np.float64) * sc.particles.vel).sum(0)
    o = OracleScene(sc, "f64")
    o.step(20)
    got = o.particles()
    p1 = (got["mass"][:, None].astype(np.float64) * got["vel"]).sum(0)
    scale = (sc.particles.mass[:, None] * np.abs(sc.particles.vel)).sum()
    assert np.abs(p1 - p0).max() < 1e-6 * scale
    assert np.abs(got["vel"] - sc.particles.vel).max() > 1e-3  # the velocities did change


def apic_angular_momentum(pos, vel, aff, mass, dx):
    """Total angular momentum of APIC particles: sum of m x x v plus the
    affine part D eps : M with D = dx^2 / 4 (quadratic B-splines) and M the
    stored affine matrix (m C minus a symmetric stress term, which the
    contraction with eps drops).  Returns it and the scale sum m |x| |v|."""
    x, v, m = pos.astype(np.float64), vel.astype(np.float64), mass.astype(np.float64)
    M = aff.astype(np.float64).reshape(-1, 3, 3).transpose(0, 2, 1)
    spin = np.stack([M[:, 2, 1] - M[:, 1, 2], M[:, 0, 2] - M[:, 2, 0], M[:, 1, 0] - M[:, 0, 1]], 1)
    total = (m[:, None] * np.cross(x, v)).sum(0) + dx * dx / 4.0 * spin.sum(0)
    scale = (m * np.linalg.norm(x, axis=1) * np.linalg.norm(v, axis=1)).sum()
    return total, scale


def test_angular_momentum_is_conserved(oracle_built):
    """APIC conserves angular momentum (its affine part included) through
    the transfers, the symmetric stress and the advection."""
    from oracle.oracle import OracleScene
    sc = _momentum_scene()
    p = sc.particles
    l0, scale = apic_angular_momentum(p.pos, p.vel, p.aff, p.mass, sc.dx)
    o = OracleScene(sc, "f64")
    o.step(20)
    g = o.particles()
    l1, _ = apic_angular_momentum(g["pos"], g["vel"], g["aff"], g["mass"], sc.dx)
    assert np.abs(l1 - l0).max() < 1e-7 * scale
    spin1 = apic_angular_momentum(g["pos"], g["vel"], np.zeros_like(g["aff"]), g["mass"], sc.dx)[0]
    assert np.abs(spin1 - l0).max() > 1e-5 * scale  # without the affine part it would not hold


def test_fp32_and_fp64_oracles_agree_on_elastic_cube(oracle_built):
    from oracle.oracle import OracleScene
    sc = scenes.elastic_cube(n_side=12, steps=20)
    a, b = OracleScene(sc, "f32"), OracleScene(sc, "f64")
    a.step(20)
    b.step(20)
    pa, pb = a.particles()["pos"], b.positions_f64()
    assert np.linalg.norm(pa - pb) / np.linalg.norm(pb) < 1e-6


def test_timestep_bound_closed_form(oracle_built):
    """CFL bound (solver/timestep_bound.rs:59-115): at rest with F = I and
    C = 0 it is cfl * dx / sqrt((K + 4/3 G) / rho0) (utils.rs:157-175) for an
    elastic solid and cfl * dx / sqrt(gamma K / rho0) for the Tait fluid; the
    velocity term takes over once |v| exceeds the sound speed."""
    from oracle.oracle import OracleScene
    dx = 1.0 / 64.0
    pos = scenes.lattice_block((0.4, 0.4, 0.4), (2, 2, 2), dx, 3)
    for model, rho, speed in (
            (ParticleModel.elastic_neo_hookean(1.0e5, 0.3), 1000.0, None),
            (ParticleModel.water(1.0e5), 1000.0, math.sqrt(7.0 * 1.0e5 / 1000.0))):
        batch = ParticleBatch.from_positions(pos, np.float32(dx / 4), rho, model)
        sc = scenes.Scene("bound", dx, 1e-4, (0.0, 0.0, 0.0), batch, collider_array([]), 1, 64)
        if speed is None:
            lam, mu = lame_lambda_mu(1.0e5, 0.3)
            speed = math.sqrt((lam + 2.0 * mu / 3.0 + 4.0 / 3.0 * mu) / rho)
        want = 0.5 * dx / speed
        got = OracleScene(sc).timestep_bound_bits() / 1e12
        assert got == pytest.approx(want, rel=1e-5)
        batch.vel[:] = (0.0, 0.0, 3.0 * speed)
        got = OracleScene(sc).timestep_bound_bits() / 1e12
        assert got == pytest.approx(min(0.5 * dx / (3.0 * speed), dx / (3.0 * speed)), rel=1e-5)


def test_inv4_matches_numpy(oracle_built):
    from oracle.oracle import inv4
    rng = np.random.default_rng(3)
    for _ in range(5):
        m = rng.standard_normal((4, 4))
        inv, det = inv4(m)
        assert np.allclose(inv, np.linalg.inv(m), atol=1e-10)
        assert det == pytest.approx(np.linalg.det(m), rel=1e-10)


def test_cpic_keeps_particles_at_the_colliders(oracle_built):
    """CPIC (analytic colliders): particles near the floor and the moving ball
    take affinities, come closer to the surfaces than the grid-projection band
    of the non-CPIC path (1.5 dx), stay outside the ball to a fraction of a
    cell, and none is lost to an inverted F, where the non-CPIC run loses some."""
    from oracle.oracle import OracleScene
    sc = scenes.cpic_drop()
    runs = {}
    for cpic in (False, True):
        o = OracleScene(sc)
        o.set_use_cpic(cpic)
        o.step(100)
        runs[cpic] = (o.particles(), o.cdf())
    p, c = runs[True]
    ball = np.array([12.8 + 2.0 * 0.1, 12.8, 0.0])
    assert p["enabled"].all() and not runs[False][0]["enabled"].all()
    assert (c["affinity"] != 0).sum() > 100
    assert p["pos"][:, 2].min() < 0.5 * 1.5 * sc.dx < runs[False][0]["pos"][:, 2].min()
    assert np.linalg.norm(p["pos"] - ball, axis=1).min() > 2.0 - 0.5 * sc.dx


def _mesh_scene(tri, meshes, dx, particle_pos=None):
    """A scene whose colliders are the trimeshes `meshes` ((first, count) each)
    over the triangles `tri` (k, 3, 3), with a few particles."""
    from nexus_b200.scenes import Scene, lattice_block
    pos = particle_pos if particle_pos is not None else lattice_block((50.0, 50.0, 50.0), (2, 2, 2), dx, 1)
    b = ParticleBatch.from_positions(pos, np.float32(dx) / np.float32(4.0), 1000.0,
                                     ParticleModel.elastic_neo_hookean(1.0e5, 0.3))
    cols = collider_array([Collider.trimesh(f, c, (0.0, 0.0, 0.0), BoundaryCondition.slip()) for f, c in meshes])
    return Scene("mesh", dx, 1.0e-3, (0.0, 0.0, 0.0), b, cols, 1, 1024,
                 tri_vertices=np.asarray(tri, np.float32).reshape(-1, 3))


def _rigid(sc):
    from oracle.oracle import OracleScene
    o = OracleScene(sc)
    o.set_use_cpic(True)
    return o.rigid_particles()


def test_trimesh_sampling_covers_the_triangle(oracle_built):
    """sample_trimesh.rs: every sample lies on the triangle (here in the plane
    z = 0.25) and every cell of the x-y grid of the sampling step that lies
    inside the triangle holds at least one sample."""
    step = 0.1
    tri = [[[0.0, 0.0, 0.25], [2.0, 0.0, 0.25], [0.0, 1.5, 0.25]]]
    r = _rigid(_mesh_scene(tri, [(0, 1)], step))
    p = r["local"]
    assert len(p) > 200 and (r["collider"] == 0).all() and (r["triangle"] == 0).all()
    assert (p[:, 2] == np.float32(0.25)).all()
    assert (p[:, 0] >= -1e-6).all() and (p[:, 1] >= -1e-6).all()
    assert (p[:, 0] / 2.0 + p[:, 1] / 1.5 <= 1.0 + 1e-5).all()
    cells = {(int(math.floor(x / step)), int(math.floor(y / step))) for x, y in p[:, :2]}
    for i in range(20):
        for j in range(15):
            if (i + 1) * step / 2.0 + (j + 1) * step / 1.5 <= 1.0 - 1e-6:  # cell fully inside
                assert (i, j) in cells, (i, j)


def test_trimesh_sampling_samples_a_shared_edge_once(oracle_built):
    """sample_trimesh.rs:73-81: an edge shared by two triangles of one mesh is
    sampled once; as two separate meshes it is sampled twice."""
    tri = [[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0]],
           [[0.0, 0.0, 0.0], [1.0, 1.0, 0.0], [0.0, 1.0, 0.0]]]
    one = _rigid(_mesh_scene(tri, [(0, 2)], 0.1))["local"]
    two = _rigid(_mesh_scene(tri, [(0, 1), (1, 1)], 0.1))["local"]
    on_diag = lambda p: int((np.abs(p[:, 0] - p[:, 1]) < 1e-6).sum())
    assert on_diag(two) > 0 and on_diag(two) == 2 * on_diag(one)
    assert len(two) - len(one) == on_diag(one)


def test_cpic_trimesh_plane_distance_field(oracle_built):
    """p2g_cdf + g2p_cdf on a flat two-triangle floor z = 1: the particle
    distance field of the particles within reach is the plane's signed
    distance z - 1 with normal +z (exact in the FP64 oracle: the MLS fit
    reproduces a linear field), and the FP32 oracle agrees to 1e-4."""
    from oracle.oracle import OracleScene
    from nexus_b200.scenes import lattice_block
    L, dx = 32.0, 0.5
    tri = [[[0, 0, 1], [L, 0, 1], [L, L, 1]], [[0, 0, 1], [L, L, 1], [0, L, 1]]]
    pos = lattice_block((10.0, 10.0, 1.3), (8, 8, 6), dx, 5)
    sc = _mesh_scene(tri, [(0, 2)], dx, pos)
    for prec, tol in (("f64", 1e-12), ("f32", 1e-4)):
        o = OracleScene(sc, precision=prec)
        o.set_use_cpic(True)
        o.step(1)
        c = o.cdf()
        m = c["affinity"] != 0
        assert m.sum() > 50 and (c["affinity"][m] == 1).all()
        assert np.abs(c["signed_distance"][m] - (pos[m, 2] - 1.0)).max() <= tol
        assert np.abs(c["normal"][m] - np.array([0.0, 0.0, 1.0])).max() <= tol


def test_readback_record_closed_form(oracle_built):
    """prep_readback.rs compute_deformation / compute_color on hand-set
    particles: deformation diag(2 r) clamp(F, -4, 4) as Mat4::from_mat3,
    the velocity, phase and default colors, group ids wrapping the palette,
    and a disabled particle drawn red."""
    from oracle.oracle import OracleScene
    from nexus_b200.scenes import Scene
    rng = np.random.default_rng(5)
    n = 8
    b = ParticleBatch.from_positions(rng.uniform(0.3, 0.7, (n, 3)), np.float32(0.01), 1000.0,
                                     ParticleModel.elastic_neo_hookean(1.0e5, 0.3))
    b.def_grad = rng.uniform(-6.0, 6.0, (n, 9)).astype(np.float32)
    b.vel = rng.uniform(-3.0, 3.0, (n, 3)).astype(np.float32)
    b.init_radius = rng.uniform(0.005, 0.02, n).astype(np.float32)
    b.phase = rng.uniform(0.0, 1.0, n).astype(np.float32)
    b.group_id = np.arange(n, dtype=np.uint32) * 3
    b.enabled[5] = 0
    sc = Scene("readback", 0.02, 1.0e-4, (0.0, 0.0, 0.0), b, collider_array([]), 1, 64)
    o = OracleScene(sc)
    pal = rng.uniform(0.0, 1.0, (5, 4)).astype(np.float32)
    F = b.def_grad.reshape(n, 3, 3)  # [particle, column, row]
    for mode in (0, 2, 3):
        r = o.prep_readback(mode, pal)
        base = pal[b.group_id % 5]
        want = {0: base,
                2: np.concatenate([np.abs(b.vel) * np.float32(1e-4) * np.float32(100.0) + np.float32(0.2),
                                   base[:, 3:]], 1),
                3: np.stack([np.zeros(n, np.float32), np.float32(0.4) * b.phase,
                             np.float32(0.4) * (np.float32(1.0) - b.phase), base[:, 3]], 1)}[mode].copy()
        want[5] = (1.0, 0.0, 0.0, 1.0)
        np.testing.assert_allclose(r["color"], want, rtol=1e-6, atol=1e-7)
        d = r["deformation"]  # [particle, column, row]
        np.testing.assert_allclose(d[:, :3, :3], 2.0 * b.init_radius[:, None, None] * np.clip(F, -4.0, 4.0),
                                   rtol=1e-6)
        assert (d[:, :3, 3] == 0).all() and (d[:, 3] == np.array([0, 0, 0, 1], np.float32)).all()
        np.testing.assert_array_equal(r["position"], b.pos)
    default = o.prep_readback(0)["color"]
    np.testing.assert_allclose(default[0], [124 / 255, 144 / 255, 1.0, 1.0], rtol=1e-6)
