"""Particle material models, packed exactly as the reference uploads them.

A model is a tag plus 24 u32 words (``GpuParticleModel``,
``src_mpm_shaders/models/default.rs:41-44``); the host packing follows
``src_mpm/solver/particle_model.rs:282-325`` and the constructors follow
``src_mpm/solver/particle_model.rs:52-251``, ``src_mpm/models/mod.rs:75-108``
and ``src_mpm/models/drucker_prager.rs:12-56``.  Every coefficient is computed
in float32, operation by operation, as the reference's ``f32`` code does, so
the packed words are bit-identical to what the reference would upload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

f32 = np.float32

MODEL_DATA_WORDS = 24

MODEL_ELASTIC_LINEAR = 0
MODEL_ELASTIC_NEO_HOOKEAN = 1
MODEL_SAND_LINEAR = 2
MODEL_SAND_NEO_HOOKEAN = 3
MODEL_FLUID = 4
MODEL_SNOW = 5

DEFAULT_YOUNG_MODULUS = f32(1000.0)
DEFAULT_POISSON_RATIO = f32(0.2)
DEFAULT_FLUID_TENSILE_STIFFNESS = f32(0.25)
DEFAULT_SNOW_CRITICAL_COMPRESSION = f32(2.5e-2)
DEFAULT_SNOW_CRITICAL_STRETCH = f32(7.5e-3)
DEFAULT_SNOW_HARDENING = f32(10.0)


def _to_radians(deg) -> np.float32:
    # Rust f32::to_radians: self * (PI / 180.0), constant folded in f32.
    return f32(deg) * (f32(math.pi) / f32(180.0))


def lame_lambda_mu(young_modulus, poisson_ratio):
    """src_mpm/models/mod.rs:76-86."""
    e, nu = f32(young_modulus), f32(poisson_ratio)
    lam = e * nu / ((f32(1.0) + nu) * (f32(1.0) - f32(2.0) * nu))
    mu = e / (f32(2.0) * (f32(1.0) + nu))
    return f32(lam), f32(mu)


def _bits(*vals) -> list[int]:
    return [int(np.array(v, dtype=np.float32).view(np.uint32)) for v in vals]


@dataclass(frozen=True)
class ParticleModel:
    """A constitutive model: ``tag`` and the 24 data words (u32 bit patterns)."""

    tag: int
    words: tuple = field(default_factory=tuple)

    def gpu_words(self) -> np.ndarray:
        out = np.zeros(1 + MODEL_DATA_WORDS, dtype=np.uint32)
        out[0] = self.tag
        out[1:1 + len(self.words)] = self.words
        return out

    # -- constructors (src_mpm/solver/particle_model.rs:52-251) -------------
    @staticmethod
    def elastic(young_modulus=DEFAULT_YOUNG_MODULUS, poisson_ratio=DEFAULT_POISSON_RATIO) -> "ParticleModel":
        lam, mu = lame_lambda_mu(young_modulus, poisson_ratio)
        return ParticleModel(MODEL_ELASTIC_LINEAR, tuple(_bits(lam, mu, 0.5)))

    @staticmethod
    def elastic_neo_hookean(young_modulus, poisson_ratio) -> "ParticleModel":
        lam, mu = lame_lambda_mu(young_modulus, poisson_ratio)
        return ParticleModel(MODEL_ELASTIC_NEO_HOOKEAN, tuple(_bits(lam, mu, 0.5)))

    @staticmethod
    def _drucker_prager(lam, mu, cohesion=0.0, friction_angle_deg=35.0):
        # src_mpm/models/drucker_prager.rs:46-56 (ha, hb, hc, hd, lambda, mu, cohesion)
        return [_to_radians(friction_angle_deg), _to_radians(9.0), f32(0.2), _to_radians(10.0),
                f32(lam), f32(mu), f32(cohesion)]

    @staticmethod
    def _sand(tag, young_modulus, poisson_ratio, cohesion=0.0, friction_angle_deg=35.0):
        if f32(young_modulus) > 0:
            plam, pmu = lame_lambda_mu(young_modulus, poisson_ratio)
        else:
            plam, pmu = f32(-1.0), f32(-1.0)
        elam, emu = lame_lambda_mu(young_modulus, poisson_ratio)
        state = [f32(1.0), f32(1.0), f32(0.0)]
        plastic = ParticleModel._drucker_prager(plam, pmu, cohesion, friction_angle_deg)
        elastic = [elam, emu, f32(0.5)]
        return ParticleModel(tag, tuple(_bits(*(state + plastic + elastic))))

    @staticmethod
    def sand(young_modulus, poisson_ratio) -> "ParticleModel":
        return ParticleModel._sand(MODEL_SAND_LINEAR, young_modulus, poisson_ratio)

    @staticmethod
    def sand_neo_hookean(young_modulus, poisson_ratio) -> "ParticleModel":
        return ParticleModel._sand(MODEL_SAND_NEO_HOOKEAN, young_modulus, poisson_ratio)

    @staticmethod
    def cohesive_sand(young_modulus, poisson_ratio, cohesion) -> "ParticleModel":
        return ParticleModel._sand(MODEL_SAND_LINEAR, young_modulus, poisson_ratio, cohesion)

    @staticmethod
    def sand_with_friction_angle(young_modulus, poisson_ratio, friction_angle_deg) -> "ParticleModel":
        """Drucker-Prager sand with a linear backbone and a chosen base friction
        angle ``ha`` (the reference's ``sand()`` fixes it at 35 degrees; a
        caller building ``DruckerPragerPlasticity`` directly can pick any)."""
        return ParticleModel._sand(MODEL_SAND_LINEAR, young_modulus, poisson_ratio, 0.0, friction_angle_deg)

    @staticmethod
    def fluid(bulk_modulus, gamma, viscosity) -> "ParticleModel":
        return ParticleModel(MODEL_FLUID, tuple(_bits(bulk_modulus, gamma, viscosity, 0.5,
                                                      DEFAULT_FLUID_TENSILE_STIFFNESS)))

    @staticmethod
    def water(bulk_modulus) -> "ParticleModel":
        return ParticleModel.fluid(bulk_modulus, 7.0, 0.001)

    @staticmethod
    def snow(young_modulus, poisson_ratio) -> "ParticleModel":
        return ParticleModel.snow_with_params(young_modulus, poisson_ratio, DEFAULT_SNOW_CRITICAL_COMPRESSION,
                                              DEFAULT_SNOW_CRITICAL_STRETCH, DEFAULT_SNOW_HARDENING)

    @staticmethod
    def snow_with_params(young_modulus, poisson_ratio, critical_compression, critical_stretch,
                         hardening) -> "ParticleModel":
        lam, mu = lame_lambda_mu(young_modulus, poisson_ratio)
        return ParticleModel(MODEL_SNOW, tuple(_bits(1.0, critical_compression, critical_stretch, hardening,
                                                     lam, mu, 0.5)))


# Boundary conditions: src_mpm_shaders/solver/boundary_condition.rs:94-129.
BOUNDARY_CONDITION_STICK = 0
BOUNDARY_CONDITION_SLIP = 1
BOUNDARY_CONDITION_SEPARATE = 2
BOUNDARY_CONDITION_NON_REFLECTING = 3


@dataclass(frozen=True)
class BoundaryCondition:
    ty: int
    friction: float = 0.0

    @staticmethod
    def stick() -> "BoundaryCondition":
        return BoundaryCondition(BOUNDARY_CONDITION_STICK, 0.0)

    @staticmethod
    def slip() -> "BoundaryCondition":
        return BoundaryCondition(BOUNDARY_CONDITION_SLIP, 0.0)

    @staticmethod
    def separate(friction) -> "BoundaryCondition":
        return BoundaryCondition(BOUNDARY_CONDITION_SEPARATE, float(friction))

    @staticmethod
    def non_reflecting() -> "BoundaryCondition":
        return BoundaryCondition(BOUNDARY_CONDITION_NON_REFLECTING, 0.0)
