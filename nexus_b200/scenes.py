"""Seeded synthetic MPM scenes (the benchmark and test workloads).

Random numbers come from SplitMix64 (Steele, Lea & Flood 2014) evaluated on a
counter, so a scene is a pure function of its seed and sizes; the same arrays
go to the CPU oracle and to the GPU.

Workloads (all 3D, unit domain, FP32 state):
  * ``elastic_cube``: dx = 1/64, a 32^3 lattice (2 particles per cell and
    axis, 32,768 particles) at 0.4 + (i + 1/2) dx/2 with +-dx/4 jitter,
    neo-Hookean E = 1e5, nu = 0.3, rho = 1000, gravity -9.81 z, slip walls on
    the six faces, dt = 1e-4.
  * ``sand_water``: dx = 1/256, a Drucker-Prager sand column (friction 30
    deg, E = 3.5e5, nu = 0.3, rho = 2700, 100 x 100 x 150 particles =
    1.5 M) and a weakly compressible water block (bulk modulus 1e5, rho =
    1000, 100 x 100 x 50 = 0.5 M), 8 particles per cell with +-dx/4 jitter,
    sticky floor, slip side walls and ceiling, dt = 5e-5.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import math

import numpy as np

from .models import ParticleModel, BoundaryCondition
from .particles import Collider, ParticleBatch, box_walls, collider_array

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """``count`` SplitMix64 outputs for stream ``seed`` starting at ``offset``."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """Uniform doubles in [0, 1) with 53 random bits."""
    return (splitmix64(seed, count, offset) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


@dataclass
class Scene:
    name: str
    dx: float
    dt: float
    gravity: tuple
    particles: ParticleBatch
    colliders: np.ndarray
    steps: int
    grid_capacity: int
    tri_vertices: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    # kinematic bodies: rows (collider index, p0 xyz, v0 xyz, a xyz, omega, phi) of
    # p(t) = p0 + v0 t + a sin(omega t + phi)
    kinematics: np.ndarray = field(default_factory=lambda: np.zeros((0, 12), np.float64))

    @property
    def n(self) -> int:
        return self.particles.n


def lattice_block(origin, counts, dx, seed, stream_offset=0) -> np.ndarray:
    """Particles at origin + (i + 1/2) dx/2 for i in [0, counts) per axis, each
    jittered by U(-dx/4, dx/4) per axis; x varies fastest."""
    nx, ny, nz = counts
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    pos = np.asarray(origin, np.float64)[None, :] + (base + 0.5) * (dx * 0.5)
    u = uniform(seed, pos.size, stream_offset).reshape(pos.shape)
    pos += (u * 2.0 - 1.0) * (0.25 * dx)
    return pos.astype(np.float32)


def grid_capacity_for(n_particles: int, ppc: float = 8.0, slack: float = 4.0) -> int:
    """Blocks (and hash slots) to reserve: active blocks are roughly the
    primary blocks (n / (64 ppc)) plus their +1 neighbours; ``slack`` covers
    both and thin or spread-out scenes."""
    blocks = max(64, int(n_particles / (64.0 * ppc) * slack) + 64)
    cap = 1
    while cap < blocks:
        cap <<= 1
    return cap


def elastic_cube(n_side: int = 32, seed: int = 1, steps: int = 100) -> Scene:
    dx = 1.0 / 64.0
    pos = lattice_block((0.4, 0.4, 0.4), (n_side, n_side, n_side), dx, seed)
    model = ParticleModel.elastic_neo_hookean(1.0e5, 0.3)
    batch = ParticleBatch.from_positions(pos, np.float32(dx) / np.float32(4.0), 1000.0, model)
    cols = collider_array(box_walls(0.0, 1.0, BoundaryCondition.slip(), BoundaryCondition.slip()))
    return Scene("elastic_cube", dx, 1.0e-4, (0.0, 0.0, -9.81), batch, cols, steps,
                 grid_capacity_for(batch.n))


def sand_water(scale: float = 1.0, seed: int = 2, steps: int = 500) -> Scene:
    """The 2 M-particle sand + water scene; ``scale`` < 1 shrinks each
    particle count per axis (for CPU-sized tests) at the same dx."""
    dx = 1.0 / 256.0
    s = lambda v: max(2, int(round(v * scale)))
    sand_counts = (s(100), s(100), s(150))
    water_counts = (s(100), s(100), s(50))
    z0 = 4 * dx
    sand_pos = lattice_block((0.20, 0.40, z0), sand_counts, dx, seed, 0)
    water_pos = lattice_block((0.45, 0.40, z0), water_counts, dx, seed, sand_pos.size)
    sand = ParticleBatch.from_positions(sand_pos, np.float32(dx) / np.float32(4.0), 2700.0,
                                        ParticleModel.sand_with_friction_angle(3.5e5, 0.3, 30.0))
    water = ParticleBatch.from_positions(water_pos, np.float32(dx) / np.float32(4.0), 1000.0,
                                         ParticleModel.water(1.0e5))
    batch = ParticleBatch.concat([sand, water])
    cols = collider_array(box_walls(0.0, 1.0, BoundaryCondition.stick(), BoundaryCondition.slip()))
    return Scene("sand_water", dx, 5.0e-5, (0.0, 0.0, -9.81), batch, cols, steps, grid_capacity_for(batch.n))


def mixed_materials(n_side: int = 12, seed: int = 7, dx: float = 1.0 / 64.0) -> Scene:
    """Small test scene with every model on a stack of blocks: linear and
    neo-Hookean elastic, sand (both backbones), fluid and snow, with random
    initial velocities so every branch of the update is exercised."""
    models = [ParticleModel.elastic(2.0e4, 0.25), ParticleModel.elastic_neo_hookean(5.0e4, 0.3),
              ParticleModel.sand(3.5e5, 0.3), ParticleModel.sand_neo_hookean(2.0e5, 0.3),
              ParticleModel.water(5.0e4), ParticleModel.snow(1.4e5, 0.2)]
    batches = []
    off = 0
    for m, model in enumerate(models):
        ox = 0.15 + 0.12 * (m % 3)
        oz = 0.2 + 0.15 * (m // 3)
        pos = lattice_block((ox, 0.4, oz), (n_side, n_side, n_side), dx, seed, off)
        off += pos.size
        b = ParticleBatch.from_positions(pos, np.float32(dx) / np.float32(4.0), 1000.0, model)
        u = uniform(seed + 101, pos.size, off).reshape(-1, 3)
        b.vel[:] = ((u * 2.0 - 1.0) * 0.5).astype(np.float32)
        batches.append(b)
    batch = ParticleBatch.concat(batches)
    cols = collider_array(box_walls(0.0, 1.0, BoundaryCondition.stick(), BoundaryCondition.separate(0.5)))
    return Scene("mixed_materials", dx, 1.0e-4, (0.0, 0.0, -9.81), batch, cols, 50, grid_capacity_for(batch.n))


def height_field(n_vertices: int, seed: int, lo: float = 0.0, hi: float = 1.0, base: float = 0.05,
                 amplitude: float = 0.02) -> np.ndarray:
    """Triangles (ntri, 3, 3) of a square height field over [lo, hi]^2: an
    n_vertices x n_vertices grid with heights base + U(0, amplitude), two
    triangles per quad, counter-clockwise seen from +z (normals point up)."""
    h = base + amplitude * uniform(seed, n_vertices * n_vertices)
    xs = np.linspace(lo, hi, n_vertices)
    v = np.stack(np.meshgrid(xs, xs, indexing="ij"), -1)  # [i, j] -> (x_i, y_j)
    v = np.concatenate([v, h.reshape(n_vertices, n_vertices, 1)], -1).astype(np.float32)
    a, b = v[:-1, :-1], v[1:, :-1]
    c, d = v[1:, 1:], v[:-1, 1:]
    t0 = np.stack([a, b, c], -2).reshape(-1, 3, 3)
    t1 = np.stack([a, c, d], -2).reshape(-1, 3, 3)
    return np.concatenate([t0, t1], 0)


def trimesh_floor(n_side: int = 16, n_vertices: int = 21, seed: int = 11, steps: int = 100) -> Scene:
    """A neo-Hookean cube (dx = 1/64) dropped onto a random height-field
    trimesh floor (heights 0.05 + U(0, 0.02), as the coupling workload's
    floor), inside five slip walls and a slip cuboid floor below the mesh."""
    dx = 1.0 / 64.0
    pos = lattice_block((0.35, 0.35, 0.085), (n_side, n_side, n_side), dx, seed)
    model = ParticleModel.elastic_neo_hookean(1.0e5, 0.3)
    batch = ParticleBatch.from_positions(pos, np.float32(dx) / np.float32(4.0), 1000.0, model)
    batch.vel[:, 2] = -1.0
    tri = height_field(n_vertices, seed + 1)
    walls = box_walls(0.0, 1.0, BoundaryCondition.slip(), BoundaryCondition.slip())
    mesh = Collider.trimesh(0, len(tri), (0.0, 0.0, 0.0), BoundaryCondition.separate(0.3))
    cols = collider_array(walls + [mesh])
    return Scene("trimesh_floor", dx, 1.0e-4, (0.0, 0.0, -9.81), batch, cols, steps, grid_capacity_for(batch.n),
                 tri_vertices=tri.reshape(-1, 3))


def random_box_scene(seed: int, dx: float, n_min: int, n_max: int, materials=("neo_hookean", "sand"),
                     steps: int = 200, name: str = "box") -> Scene:
    """One scene of the batched and serving workloads: a random axis-aligned
    box of N ~ logU(n_min, n_max) particles, uniform random inside it, of one
    material drawn uniformly from ``materials``: neo-Hookean solid (E ~
    logU(1e4, 1e6), nu = 0.3, rho = 1000), Drucker-Prager sand (30 degrees,
    E = 3.5e5, nu = 0.3, rho = 2700) or water (bulk modulus 1e5, rho = 1000).
    Box sides start U(0.1, 0.4), are rescaled to the volume N (dx/2)^3 (8
    particles per cell) and clamped to [0.1, 0.4]; the box sits at a random
    place inside [4dx, 1 - 4dx]^3.  V0 = box volume / N, m = rho V0.  Six
    slip walls bound [0, 1]^3; dt = 5e-5, gravity -z."""
    u = uniform(seed, 16)
    n = int(round(math.exp(math.log(n_min) + u[0] * (math.log(n_max) - math.log(n_min)))))
    sides = 0.1 + 0.3 * u[1:4]
    target = n * (dx / 2.0) ** 3
    sides = np.clip(sides * (target / np.prod(sides)) ** (1.0 / 3.0), 0.1, 0.4)
    lo = 4 * dx + u[4:7] * (1.0 - 8 * dx - sides)
    pos = (lo + sides * uniform(seed, 3 * n, 16).reshape(n, 3)).astype(np.float32)
    v0 = float(np.prod(sides)) / n
    radius = np.float32(0.5 * v0 ** (1.0 / 3.0))
    mat = materials[min(int(u[7] * len(materials)), len(materials) - 1)]
    if mat == "neo_hookean":
        e = math.exp(math.log(1.0e4) + u[8] * (math.log(1.0e6) - math.log(1.0e4)))
        batch = ParticleBatch.from_positions(pos, radius, 1000.0, ParticleModel.elastic_neo_hookean(e, 0.3))
    elif mat == "sand":
        batch = ParticleBatch.from_positions(pos, radius, 2700.0,
                                             ParticleModel.sand_with_friction_angle(3.5e5, 0.3, 30.0))
    else:
        batch = ParticleBatch.from_positions(pos, radius, 1000.0, ParticleModel.water(1.0e5))
    cols = collider_array(box_walls(0.0, 1.0, BoundaryCondition.slip(), BoundaryCondition.slip()))
    # blocks the box spans (plus a layer each side for neighbours and motion), twice over for slack
    blocks = int(np.prod(np.ceil(sides / (4 * dx)) + 3))
    cap = 1
    while cap < 2 * blocks + 64:
        cap <<= 1
    return Scene(name, dx, 5.0e-5, (0.0, 0.0, -9.81), batch, cols, steps, max(cap, grid_capacity_for(batch.n)))


def batched_mix(count: int = 256, seed: int = 1000, dx: float = 1.0 / 128.0, steps: int = 200,
                n_min: int = 4096, n_max: int = 131072) -> list:
    """The batched workload: ``count`` independent scenes (seed + s for scene
    s) from random_box_scene, neo-Hookean or sand half and half, 4k-128k
    particles each, dx = 1/128, 200 steps."""
    return [random_box_scene(seed + s, dx, n_min, n_max, ("neo_hookean", "sand"), steps, f"batched_{s}")
            for s in range(count)]


def serving_scene(i: int, seed: int = 3000) -> Scene:
    """Request i of the serving workload: 2k-512k particles, elastic, sand or
    water, dx = 1/128 or 1/256 (uniform)."""
    u = uniform(seed + 7919 * (i + 1), 1)
    dx = 1.0 / 128.0 if u[0] < 0.5 else 1.0 / 256.0
    return random_box_scene(seed + i, dx, 2048, 524288, ("neo_hookean", "sand", "water"), name=f"serve_{i}")


def cpic_drop(n_side: int = 12, seed: int = 17, steps: int = 100) -> Scene:
    """Colliders close to the particles from the first step, at the scale of
    the reference's CPIC scenes (cell width 0.5, a 32-unit domain: the
    particle distance-field fit keeps only nodes with a 4x4 moment
    determinant above 1e-8, which meter-sized cells pass): a neo-Hookean
    cube and a sand block falling at 10 m/s onto the slip floor, the cube
    also onto a ball moving along x at 2 m/s (the cube starts 0.4 above it,
    the sand 0.9 above the floor), inside five slip walls."""
    L, dx = 32.0, 0.5
    cube = ParticleBatch.from_positions(lattice_block((0.30 * L, 0.30 * L, 2.4), (n_side, n_side, n_side), dx, seed),
                                        np.float32(dx) / np.float32(4.0), 1000.0,
                                        ParticleModel.elastic_neo_hookean(1.0e5, 0.3))
    sand = ParticleBatch.from_positions(lattice_block((0.62 * L, 0.30 * L, 0.9), (n_side, n_side, n_side // 2), dx,
                                                      seed, 3 * n_side ** 3),
                                        np.float32(dx) / np.float32(4.0), 2700.0,
                                        ParticleModel.sand_with_friction_angle(3.5e5, 0.3, 30.0))
    batch = ParticleBatch.concat([cube, sand])
    batch.vel[:, 2] = -10.0
    ball = Collider.ball(2.0, (0.40 * L, 0.40 * L, 0.0), BoundaryCondition.separate(0.2))
    ball.linvel = (2.0, 0.0, 0.0)
    cols = collider_array(box_walls(0.0, L, BoundaryCondition.slip(), BoundaryCondition.slip(), thickness=2.0) + [ball])
    return Scene("cpic_drop", dx, 1.0e-3, (0.0, 0.0, -9.81), batch, cols, steps, grid_capacity_for(batch.n))


def box_mesh(half: float) -> np.ndarray:
    """Triangles (12, 3, 3) of the closed box [-half, half]^3, counter-clockwise
    seen from outside."""
    h = float(half)
    corner = lambda i: (h if i & 1 else -h, h if i & 2 else -h, h if i & 4 else -h)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tri = []
    for a, b, c, d in quads:
        tri += [[corner(a), corner(b), corner(c)], [corner(a), corner(c), corner(d)]]
    return np.asarray(tri, np.float32)


def cpic_trimesh(n_side: int = 10, seed: int = 23, steps: int = 100) -> Scene:
    """CPIC with trimesh colliders at the scale of the reference's CPIC scenes
    (cell width 0.5, a 32-unit domain): a height-field floor mesh (17 x 17
    vertices over the domain, heights 1 + U(0, 0.5)) under a neo-Hookean
    cube and a sand block falling at 10 m/s from 0.6 above its highest
    point, and a closed box mesh (half-size 1.5) beside the sand moving
    along -x at 5 m/s while spinning about z at 2 rad/s; five slip cuboid
    walls (analytic colliders) around the domain."""
    L, dx = 32.0, 0.5
    floor = height_field(17, seed + 1, 0.0, L, base=1.0, amplitude=0.5)
    box = box_mesh(1.5)
    tri = np.concatenate([floor, box], 0)
    cube = ParticleBatch.from_positions(lattice_block((0.30 * L, 0.30 * L, 2.1), (n_side, n_side, n_side), dx, seed),
                                        np.float32(dx) / np.float32(4.0), 1000.0,
                                        ParticleModel.elastic_neo_hookean(1.0e5, 0.3))
    sand = ParticleBatch.from_positions(lattice_block((0.60 * L, 0.55 * L, 2.1), (n_side, n_side, n_side // 2), dx,
                                                      seed, 3 * n_side ** 3),
                                        np.float32(dx) / np.float32(4.0), 2700.0,
                                        ParticleModel.sand_with_friction_angle(3.5e5, 0.3, 30.0))
    batch = ParticleBatch.concat([cube, sand])
    batch.vel[:, 2] = -10.0
    sand_hi_x = 0.60 * L + n_side * dx / 2
    mesh_floor = Collider.trimesh(0, len(floor), (0.0, 0.0, 0.0), BoundaryCondition.separate(0.3))
    mesh_box = Collider.trimesh(len(floor), len(box), (sand_hi_x + 1.8, 0.55 * L + 1.25, 2.9),
                                BoundaryCondition.slip())
    mesh_box.linvel = (-5.0, 0.0, 0.0)
    mesh_box.angvel = (0.0, 0.0, 2.0)
    walls = box_walls(0.0, L, BoundaryCondition.slip(), BoundaryCondition.slip(), thickness=2.0)[:-1]
    cols = collider_array(walls + [mesh_floor, mesh_box])
    return Scene("cpic_trimesh", dx, 1.0e-3, (0.0, 0.0, -9.81), batch, cols, steps, 4096,
                 tri_vertices=tri.reshape(-1, 3))


def kinematic_velocities(scene: Scene, t: float) -> tuple[np.ndarray, np.ndarray]:
    """(collider indices, (k, 6) linear + angular velocity) of the scene's
    kinematic bodies at time t: dp/dt = v0 + a omega cos(omega t + phi)."""
    k = scene.kinematics
    if k.size == 0:
        return np.zeros(0, np.int64), np.zeros((0, 6), np.float32)
    om, ph = k[:, 10:11], k[:, 11:12]
    v = k[:, 4:7] + k[:, 7:10] * om * np.cos(om * t + ph)
    out = np.zeros((len(k), 6), np.float32)
    out[:, :3] = v
    return k[:, 0].astype(np.int64), out


def coupled_scene(s: int, seed: int = 2000, dx: float = 1.0 / 128.0, n_min: int = 32768, n_max: int = 262144,
                  floor_vertices: int = 101, steps: int = 300) -> Scene:
    """Scene s of the coupled workload: a random box of N ~ logU(n_min, n_max)
    Drucker-Prager sand particles (as the batched workload, placed above the
    floor), eight kinematic bodies (cuboid, ball or capsule, size U(0.05,
    0.2)) moving along p(t) = p0 + v0 t + a sin(omega t + phi) with seeded
    parameters, a height-field trimesh floor (floor_vertices^2 vertices,
    heights 0.05 + U(0, 0.02)), and six slip walls bounding [0, 1]^3."""
    sd = seed + s
    box = random_box_scene(sd, dx, n_min, n_max, ("sand",), steps, f"coupled_{s}")
    pos = box.particles.pos
    lift = max(0.0, 0.09 - float(pos[:, 2].min()))  # the box starts above the floor mesh
    top = float(pos[:, 2].max()) + lift
    pos[:, 2] += np.float32(lift - max(0.0, top - (1.0 - 4 * dx)))
    u = uniform(sd + 7777, 8 * 16)
    cols = box_walls(0.0, 1.0, BoundaryCondition.slip(), BoundaryCondition.slip())
    kin = []
    for b in range(8):
        r = u[16 * b:16 * (b + 1)]
        size = 0.05 + 0.15 * r[0]
        p0 = np.array([0.2 + 0.6 * r[1], 0.2 + 0.6 * r[2], 0.2 + 0.4 * r[3]])
        v0 = -0.2 + 0.4 * r[4:7]
        a = 0.1 * r[7:10]
        om, ph = 1.0 + 9.0 * r[10], 2.0 * math.pi * r[11]
        start = tuple(p0 + a * math.sin(ph))
        bc = BoundaryCondition.separate(0.3)
        kind = int(r[12] * 3)
        if kind == 0:
            c = Collider.cuboid((size / 2, size / 2, size / 2), start, bc)
        elif kind == 1:
            c = Collider.ball(size / 2, start, bc)
        else:
            c = Collider.capsule((0.0, 0.0, -size / 2), (0.0, 0.0, size / 2), size / 4, start, bc)
        kin.append([len(cols), *p0, *v0, *a, om, ph])
        cols.append(c)
    tri = height_field(floor_vertices, sd + 1)
    cols.append(Collider.trimesh(0, len(tri), (0.0, 0.0, 0.0), BoundaryCondition.separate(0.3)))
    box.colliders = collider_array(cols)
    box.tri_vertices = tri.reshape(-1, 3)
    box.kinematics = np.asarray(kin, np.float64)
    return box


def coupled_mix(count: int = 64, seed: int = 2000, steps: int = 300, **kw) -> list:
    """The coupled batched workload: coupled_scene(s) for s in [0, count)."""
    return [coupled_scene(s, seed, steps=steps, **kw) for s in range(count)]

