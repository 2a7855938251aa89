"""Particle batches (structure of arrays) and collider descriptors.

``ParticleBatch`` carries the per-particle fields of the reference's
``Particle`` / ``ParticleDynamics`` (``src_mpm/solver/particle.rs:26-122``) as
numpy arrays, in the layout the C ABI's bulk upload takes (matrices are
column-major, 9 floats).  ``collider_array`` packs collider descriptors into
the 128-byte ``nxm_collider`` records of ``include/nexus_mpm.h``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .models import ParticleModel, BoundaryCondition

f32 = np.float32

IDENTITY9 = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], dtype=np.float32)


@dataclass
class ParticleBatch:
    pos: np.ndarray            # (n, 3) f32
    vel: np.ndarray            # (n, 3) f32
    aff: np.ndarray            # (n, 9) f32, column-major
    def_grad: np.ndarray       # (n, 9) f32, column-major
    vel_grad_det: np.ndarray   # (n,) f32
    mass: np.ndarray           # (n,) f32
    init_volume: np.ndarray    # (n,) f32
    init_radius: np.ndarray    # (n,) f32
    damping: np.ndarray        # (n,) f32
    phase: np.ndarray          # (n,) f32
    boundary_friction: np.ndarray  # (n,) f32
    group_id: np.ndarray       # (n,) u32
    enabled: np.ndarray        # (n,) u32
    fixed: np.ndarray          # (n,) u32
    model: np.ndarray          # (n, 25) u32: tag + 24 words

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @staticmethod
    def from_positions(pos, radius, density, model) -> "ParticleBatch":
        """``Particle::new(position, radius, density, model)`` for every row of
        ``pos``; ``radius``/``density`` may be scalars or per-particle arrays and
        ``model`` a ParticleModel or an (n, 25) u32 array."""
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        n = pos.shape[0]
        radius = np.broadcast_to(np.asarray(radius, dtype=np.float32), (n,)).copy()
        density = np.broadcast_to(np.asarray(density, dtype=np.float32), (n,)).copy()
        # ParticleDynamics::new: init_volume = (2r)^3, mass = init_volume * density
        d = radius * f32(2.0)
        init_volume = (d * d * d).astype(np.float32)
        mass = (init_volume * density).astype(np.float32)
        if isinstance(model, ParticleModel):
            words = np.broadcast_to(model.gpu_words(), (n, 25)).copy()
        else:
            words = np.ascontiguousarray(model, dtype=np.uint32).reshape(n, 25)
        return ParticleBatch(
            pos=pos.copy(),
            vel=np.zeros((n, 3), np.float32),
            aff=np.zeros((n, 9), np.float32),
            def_grad=np.broadcast_to(IDENTITY9, (n, 9)).copy(),
            vel_grad_det=np.zeros(n, np.float32),
            mass=mass,
            init_volume=init_volume,
            init_radius=radius,
            damping=np.zeros(n, np.float32),
            phase=np.ones(n, np.float32),
            boundary_friction=np.ones(n, np.float32),
            group_id=np.zeros(n, np.uint32),
            enabled=np.ones(n, np.uint32),
            fixed=np.zeros(n, np.uint32),
            model=words,
        )

    @staticmethod
    def concat(batches) -> "ParticleBatch":
        fields = ParticleBatch.__dataclass_fields__.keys()
        return ParticleBatch(**{k: np.concatenate([getattr(b, k) for b in batches], axis=0) for k in fields})

    def copy(self) -> "ParticleBatch":
        fields = ParticleBatch.__dataclass_fields__.keys()
        return ParticleBatch(**{k: getattr(self, k).copy() for k in fields})

    def take(self, idx) -> "ParticleBatch":
        fields = ParticleBatch.__dataclass_fields__.keys()
        return ParticleBatch(**{k: getattr(self, k)[idx].copy() for k in fields})


# ---------------------------------------------------------------------------
# Colliders: Shape (src_rbd_shaders/shapes/shape.rs:29-73), Pose3, Velocity
# (src_rbd_shaders/dynamics/body.rs:216-250), BoundaryCondition.
# ---------------------------------------------------------------------------

SHAPE_TYPE_BALL = 0
SHAPE_TYPE_CUBOID = 1
SHAPE_TYPE_CAPSULE = 2
SHAPE_TYPE_TRIMESH = 6

COLLIDER_DTYPE = np.dtype([
    ("shape_a", np.float32, 4), ("shape_b", np.float32, 4), ("shape_c", np.float32, 4),
    ("rotation", np.float32, 4), ("translation", np.float32, 3),
    ("linvel", np.float32, 3), ("angvel", np.float32, 3), ("local_com", np.float32, 3),
    ("bc_type", np.uint32), ("bc_friction", np.float32),
    ("tri_first", np.uint32), ("tri_count", np.uint32),
])
assert COLLIDER_DTYPE.itemsize == 128


# nxm_particle (include/nexus_mpm.h), the reference's `Particle` fields.
PARTICLE_DTYPE = np.dtype([
    ("position", np.float32, 3), ("velocity", np.float32, 3), ("def_grad", np.float32, 9),
    ("affine", np.float32, 9), ("force_dt", np.float32, 3), ("vel_grad_det", np.float32),
    ("init_volume", np.float32), ("init_radius", np.float32), ("mass", np.float32), ("damping", np.float32),
    ("phase", np.float32), ("boundary_friction", np.float32), ("group_id", np.uint32), ("enabled", np.uint32),
    ("fixed", np.uint32), ("model", np.uint32, 25),
])
assert PARTICLE_DTYPE.itemsize == 248


def particle_records(batch: "ParticleBatch") -> np.ndarray:
    """The batch as an array of nxm_particle records."""
    out = np.zeros(batch.n, dtype=PARTICLE_DTYPE)
    out["position"] = batch.pos
    out["velocity"] = batch.vel
    out["def_grad"] = batch.def_grad.reshape(batch.n, 9)
    out["affine"] = batch.aff.reshape(batch.n, 9)
    out["vel_grad_det"] = batch.vel_grad_det
    out["init_volume"] = batch.init_volume
    out["init_radius"] = batch.init_radius
    out["mass"] = batch.mass
    out["damping"] = batch.damping
    out["phase"] = batch.phase
    out["boundary_friction"] = batch.boundary_friction
    out["group_id"] = batch.group_id
    out["enabled"] = batch.enabled
    out["fixed"] = batch.fixed
    out["model"] = batch.model
    return out


def _tag(ty: int) -> np.float32:
    return np.array([ty], dtype=np.uint32).view(np.float32)[0]


@dataclass
class Collider:
    """One coupled collider: shape, pose, rigid velocity and boundary condition."""

    shape_type: int
    a: tuple = (0.0, 0.0, 0.0)
    b: tuple = (0.0, 0.0, 0.0, 0.0)
    translation: tuple = (0.0, 0.0, 0.0)
    rotation: tuple = (0.0, 0.0, 0.0, 1.0)  # quaternion x, y, z, w
    linvel: tuple = (0.0, 0.0, 0.0)
    angvel: tuple = (0.0, 0.0, 0.0)
    local_com: tuple = (0.0, 0.0, 0.0)
    bc: BoundaryCondition = BoundaryCondition.slip()
    tri_first: int = 0
    tri_count: int = 0

    @staticmethod
    def cuboid(half_extents, translation, bc, rotation=(0.0, 0.0, 0.0, 1.0)) -> "Collider":
        return Collider(SHAPE_TYPE_CUBOID, a=tuple(half_extents), translation=tuple(translation), rotation=rotation,
                        bc=bc)

    @staticmethod
    def ball(radius, translation, bc) -> "Collider":
        return Collider(SHAPE_TYPE_BALL, a=(radius, 0.0, 0.0), translation=tuple(translation), bc=bc)

    @staticmethod
    def capsule(a, b, radius, translation, bc, rotation=(0.0, 0.0, 0.0, 1.0)) -> "Collider":
        com = tuple((np.asarray(a, np.float64) + np.asarray(b, np.float64)) * 0.5)
        return Collider(SHAPE_TYPE_CAPSULE, a=tuple(a), b=tuple(b) + (radius,), translation=tuple(translation),
                        rotation=rotation, bc=bc, local_com=com)

    @staticmethod
    def trimesh(tri_first, tri_count, translation, bc, rotation=(0.0, 0.0, 0.0, 1.0)) -> "Collider":
        return Collider(SHAPE_TYPE_TRIMESH, translation=tuple(translation), rotation=rotation, bc=bc,
                        tri_first=tri_first, tri_count=tri_count)


def collider_array(colliders) -> np.ndarray:
    out = np.zeros(len(colliders), dtype=COLLIDER_DTYPE)
    for i, c in enumerate(colliders):
        out[i]["shape_a"][:3] = c.a[:3]
        out[i]["shape_a"][3] = _tag(c.shape_type)
        b = list(c.b) + [0.0] * (4 - len(c.b))
        out[i]["shape_b"][:] = b[:4]
        out[i]["rotation"][:] = c.rotation
        out[i]["translation"][:] = c.translation
        out[i]["linvel"][:] = c.linvel
        out[i]["angvel"][:] = c.angvel
        out[i]["local_com"][:] = c.local_com
        out[i]["bc_type"] = c.bc.ty
        out[i]["bc_friction"] = c.bc.friction
        out[i]["tri_first"] = c.tri_first
        out[i]["tri_count"] = c.tri_count
    return out


def box_walls(lo=0.0, hi=1.0, floor_bc=None, wall_bc=None, thickness=0.1) -> list:
    """Six cuboid walls whose inner faces bound [lo, hi]^3 (floor at z = lo)."""
    floor_bc = floor_bc or BoundaryCondition.slip()
    wall_bc = wall_bc or BoundaryCondition.slip()
    h = thickness
    c = 0.5 * (lo + hi)
    span = 0.5 * (hi - lo) + 2 * h
    return [
        Collider.cuboid((span, span, h), (c, c, lo - h), floor_bc),
        Collider.cuboid((span, span, h), (c, c, hi + h), wall_bc),
        Collider.cuboid((h, span, span), (lo - h, c, c), wall_bc),
        Collider.cuboid((h, span, span), (hi + h, c, c), wall_bc),
        Collider.cuboid((span, h, span), (c, lo - h, c), wall_bc),
        Collider.cuboid((span, h, span), (c, hi + h, c), wall_bc),
    ]
