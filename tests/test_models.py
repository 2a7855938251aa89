"""Host-side model packing (src_mpm/solver/particle_model.rs:52-325) and particle
construction (src_mpm/solver/particle.rs:100-122): bit-level checks."""
import math

import numpy as np

from nexus_b200.models import ParticleModel, lame_lambda_mu, MODEL_SAND_LINEAR, MODEL_FLUID, MODEL_SNOW
from nexus_b200.particles import ParticleBatch


def f(word):
    return float(np.array([word], np.uint32).view(np.float32)[0])


def test_lame_parameters_in_f32():
    lam, mu = lame_lambda_mu(1e5, 0.3)
    assert lam.dtype == np.float32 and mu.dtype == np.float32
    assert abs(float(lam) / (1e5 * 0.3 / (1.3 * 0.4)) - 1) < 1e-6
    assert abs(float(mu) / (1e5 / 2.6) - 1) < 1e-6


def test_sand_layout_matches_reference_struct_order():
    w = ParticleModel.sand(3.5e5, 0.3).gpu_words()
    assert w[0] == MODEL_SAND_LINEAR
    words = [f(x) for x in w[1:]]
    # plastic state (1, 1, 0), DruckerPragerPlasticity (ha, hb, hc, hd, lambda, mu, cohesion),
    # linear elastic backbone (lambda, mu, cfl 0.5), zero padding
    assert words[:3] == [1.0, 1.0, 0.0]
    assert abs(words[3] - math.radians(35)) < 1e-7 and abs(words[4] - math.radians(9)) < 1e-7
    assert words[5] == np.float32(0.2) and abs(words[6] - math.radians(10)) < 1e-7
    lam, mu = lame_lambda_mu(3.5e5, 0.3)
    assert words[7] == lam and words[8] == mu and words[9] == 0.0
    assert words[10] == lam and words[11] == mu and words[12] == 0.5
    assert all(x == 0.0 for x in words[13:])
    # a friction angle other than the reference's 35 degrees changes only ha
    w30 = ParticleModel.sand_with_friction_angle(3.5e5, 0.3, 30.0).gpu_words()
    assert abs(f(w30[4]) - math.radians(30)) < 1e-7
    assert np.array_equal(np.delete(w30, 4), np.delete(w, 4))


def test_fluid_and_snow_layouts():
    w = ParticleModel.water(1e5).gpu_words()
    assert w[0] == MODEL_FLUID
    assert [f(x) for x in w[1:6]] == [1e5, 7.0, np.float32(0.001), 0.5, 0.25]
    s = ParticleModel.snow(1.4e5, 0.2).gpu_words()
    assert s[0] == MODEL_SNOW
    assert [f(x) for x in s[1:5]] == [1.0, np.float32(2.5e-2), np.float32(7.5e-3), 10.0]


def test_particle_new_volume_and_mass():
    dx = np.float32(1 / 64)
    b = ParticleBatch.from_positions(np.zeros((3, 3)), dx / np.float32(4), 1000.0, ParticleModel.water(1e5))
    v0 = (dx / 2) ** 3
    assert np.allclose(b.init_volume, v0, rtol=1e-6)
    assert np.allclose(b.mass, v0 * 1000.0, rtol=1e-6)
    assert b.def_grad[0].tolist() == [1, 0, 0, 0, 1, 0, 0, 0, 1]
    assert b.enabled.tolist() == [1, 1, 1] and b.phase.tolist() == [1, 1, 1]
