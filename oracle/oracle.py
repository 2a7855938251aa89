"""ctypes front-end of the CPU oracle (test infrastructure only).

The oracle restates the reference's MLS-MPM step on the CPU (see
``mpm_oracle.c`` for the reference file:line each function follows; parity
is unpinned because the reference has no MPM tests or fixtures).  Only the
tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` use
this module, as the checker; the CUDA library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIBS: dict = {}

_f = C.POINTER(C.c_float)
_d = C.POINTER(C.c_double)
_u = C.POINTER(C.c_uint32)
_i = C.POINTER(C.c_int32)


def build() -> None:
    """Compile the FP32 and FP64 oracle libraries with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _host_key() -> str:
    """A short fingerprint of this host's CPU (model and feature flags), so
    that a -march=native build is only ever loaded where it was built."""
    import hashlib
    model = flags = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if not model and line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                elif not flags and line.startswith("flags"):
                    flags = line.split(":", 1)[1].strip()
                if model and flags:
                    break
    except OSError:
        pass
    return hashlib.sha256((model + "|" + flags).encode()).hexdigest()[:12]


def native_path() -> str | None:
    """The FP32 oracle built with -march=native for this host (built on first
    use, a few seconds of gcc), or None when it cannot be built here."""
    d = os.path.join(_HERE, f"_build_native_{_host_key()}")
    path = os.path.join(d, "liboracle_f32.so")
    if not os.path.exists(path):
        r = subprocess.run(["make", "-s", "-C", _HERE, "native", f"NATIVE={d}"], capture_output=True)
        if r.returncode != 0 or not os.path.exists(path):
            return None
    return path


def lib(precision: str = "f32", native: bool = False):
    """The oracle library; `native`: the FP32 build for this host's CPU when
    it can be built (same rounding flags, so the same results), else the
    portable build."""
    key = req = precision + ("_native" if native else "")
    if key in _LIBS:
        return _LIBS[key]
    path = native_path() if native and precision == "f32" else None
    if path is None:
        key = precision
        if key in _LIBS:
            return _LIBS[key]
        path = os.path.join(_BUILD, f"liboracle_{precision}.so")
        if not os.path.exists(path):
            build()
    L = C.CDLL(path)
    L.oracle_path = path
    L.orc_create.restype = C.c_void_p
    L.orc_create.argtypes = [C.c_uint32, C.c_double, C.c_uint32]
    L.orc_destroy.argtypes = [C.c_void_p]
    L.orc_set_particles.argtypes = [C.c_void_p, _f, _f, _f, _f, _f, _f, _f, _f, _u, _u, _u]
    L.orc_get_particles.argtypes = [C.c_void_p, _f, _f, _f, _f, _f, _f, _u, _u]
    L.orc_get_positions_f64.argtypes = [C.c_void_p, _d]
    L.orc_set_params.argtypes = [C.c_void_p, _f, C.c_float]
    L.orc_set_use_cpic.argtypes = [C.c_void_p, C.c_int]
    L.orc_set_colliders.argtypes = [C.c_void_p, C.c_uint32, _f, C.c_uint32, _f]
    L.orc_set_collider_velocity.argtypes = [C.c_void_p, C.c_uint32, _f, _f]
    L.orc_get_collider_pose.argtypes = [C.c_void_p, C.c_uint32, _f]
    for name in ("orc_sort", "orc_step"):
        getattr(L, name).argtypes = [C.c_void_p]
        getattr(L, name).restype = C.c_int
    L.orc_run.argtypes = [C.c_void_p, C.c_uint32]
    L.orc_run.restype = C.c_int
    L.orc_set_boundary_friction.argtypes = [C.c_void_p, _f]
    L.orc_get_cdf.argtypes = [C.c_void_p, _f]
    L.orc_inv4.argtypes = [_d, _d]
    L.orc_inv4.restype = C.c_double
    for name in ("orc_p2g", "orc_grid_update", "orc_g2p", "orc_particle_update", "orc_grid_update_cdf",
                 "orc_g2p_cdf"):
        getattr(L, name).argtypes = [C.c_void_p]
    L.orc_get_rigid.argtypes = [C.c_void_p, _f]
    L.orc_set_render_props.argtypes = [C.c_void_p, _f, _f, _u]
    L.orc_prep_readback.argtypes = [C.c_void_p, C.c_uint32, _f, C.c_uint32, _f]
    L.orc_prep_readback_rigid.argtypes = [C.c_void_p, _f, _f, C.c_uint32, _f]
    for name in ("orc_num_blocks", "orc_status", "orc_capacity", "orc_sorted_len", "orc_timestep_bound_bits",
                 "orc_num_rigid"):
        getattr(L, name).argtypes = [C.c_void_p]
        getattr(L, name).restype = C.c_uint32
    L.orc_get_headers.argtypes = [C.c_void_p, _i]
    L.orc_get_sorted.argtypes = [C.c_void_p, _u]
    L.orc_get_nodes.argtypes = [C.c_void_p, _f]
    L.orc_pack_key.argtypes = [C.c_int32, C.c_int32, C.c_int32]
    L.orc_pack_key.restype = C.c_uint32
    L.orc_hash.argtypes = [C.c_uint32]
    L.orc_hash.restype = C.c_uint32
    L.orc_kernel_eval.argtypes = [C.c_double]
    L.orc_kernel_eval.restype = C.c_double
    L.orc_kernel_eval_all.argtypes = [C.c_double, _d]
    L.orc_block_of_point.argtypes = [C.c_double, _f, _i, _u]
    L.orc_model_update.argtypes = [C.c_uint32, _u, _f, _f, _f]
    L.orc_svd.argtypes = [_f, _f, _f, _f]
    L.orc_project_point.argtypes = [C.c_void_p, C.c_uint32, _f, _f]
    L.orc_project_point.restype = C.c_int
    L.orc_bc_project.argtypes = [C.c_uint32, C.c_float, _f, _f, _f]
    L.orc_prefix_sum.argtypes = [_u, C.c_uint32]
    _LIBS[key] = _LIBS[req] = L
    return L


HEADER_FIELDS = 23  # vid[3], first, num, num_extras, cursors[10], nbh[7]


class OracleScene:
    """One scene held by the oracle (``precision`` = "f32" or "f64"; ``native``:
    the FP32 build for this host's CPU, where it can be built)."""

    def __init__(self, scene, precision: str = "f32", grid_capacity: int | None = None, native: bool = False):
        self.L = lib(precision, native)
        self.precision = precision
        p = scene.particles
        self.n = p.n
        cap = grid_capacity or scene.grid_capacity
        self.h = self.L.orc_create(p.n, scene.dx, cap)
        self.set_particles(p)
        g = np.asarray(scene.gravity, np.float32)
        self.L.orc_set_params(self.h, _ptr(g, _f), C.c_float(scene.dt))
        self.set_colliders(scene.colliders, getattr(scene, "tri_vertices", None))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    def set_particles(self, p):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in
                (p.pos, p.vel, p.aff, p.def_grad, p.vel_grad_det, p.mass, p.init_volume, p.damping)]
        ints = [np.ascontiguousarray(a, dtype=np.uint32) for a in (p.enabled, p.fixed, p.model)]
        self.L.orc_set_particles(self.h, *[_ptr(a, _f) for a in arrs], *[_ptr(a, _u) for a in ints])
        bf = np.ascontiguousarray(p.boundary_friction, dtype=np.float32)
        self.L.orc_set_boundary_friction(self.h, _ptr(bf, _f))
        r, ph = (np.ascontiguousarray(a, dtype=np.float32) for a in (p.init_radius, p.phase))
        g = np.ascontiguousarray(p.group_id, dtype=np.uint32)
        self.L.orc_set_render_props(self.h, _ptr(r, _f), _ptr(ph, _f), _ptr(g, _u))

    @staticmethod
    def _records(out: np.ndarray) -> dict:
        return dict(color=out[:, 0:4], deformation=out[:, 4:20].reshape(-1, 4, 4), position=out[:, 20:23])

    def prep_readback(self, mode: int, palette=None) -> dict:
        """ReadbackData of every particle (prep_readback.rs): color (n, 4),
        deformation (n, 4, 4) as columns, position (n, 3)."""
        pal = None if palette is None else np.ascontiguousarray(palette, np.float32).reshape(-1, 4)
        out = np.zeros((self.n, 24), np.float32)
        self.L.orc_prep_readback(self.h, mode, None if pal is None else _ptr(pal, _f),
                                 0 if pal is None else len(pal), _ptr(out, _f))
        return self._records(out)

    def prep_readback_rigid(self, colors=None, palette=None) -> dict:
        """ReadbackData of every rigid particle (prep_readback.rs:420-469)."""
        n = self.L.orc_num_rigid(self.h)
        cols = None if colors is None else np.ascontiguousarray(colors, np.float32).reshape(-1, 4)
        pal = None if palette is None else np.ascontiguousarray(palette, np.float32).reshape(-1, 4)
        out = np.zeros((max(n, 1), 24), np.float32)
        self.L.orc_prep_readback_rigid(self.h, None if cols is None else _ptr(cols, _f),
                                       None if pal is None else _ptr(pal, _f), 0 if pal is None else len(pal),
                                       _ptr(out, _f))
        return self._records(out[:n])

    def cdf(self) -> dict:
        """Particle Cdf (CPIC): normal, signed distance, rigid velocity, affinity bits."""
        out = np.zeros((self.n, 8), np.float32)
        self.L.orc_get_cdf(self.h, _ptr(out, _f))
        return dict(normal=out[:, :3], signed_distance=out[:, 3], rigid_vel=out[:, 4:7],
                    affinity=out[:, 7].copy().view(np.uint32))

    def grid_update_cdf(self):
        self.L.orc_grid_update_cdf(self.h)

    def collider_pose(self, index: int) -> np.ndarray:
        """Quaternion x, y, z, w then translation of collider `index`."""
        out = np.zeros(7, np.float32)
        self.L.orc_get_collider_pose(self.h, index, _ptr(out, _f))
        return out

    def rigid_particles(self) -> dict:
        """CPIC rigid particles (trimesh surface samples, sampling step = cell
        width): local position, collider index, triangle index inside the
        collider's triangle range."""
        n = self.L.orc_num_rigid(self.h)
        out = np.zeros((n, 5), np.float32)
        if n:
            self.L.orc_get_rigid(self.h, _ptr(out, _f))
        return dict(local=out[:, :3], collider=out[:, 3].copy().view(np.uint32),
                    triangle=out[:, 4].copy().view(np.uint32))

    def g2p_cdf(self):
        self.L.orc_g2p_cdf(self.h)

    def set_colliders(self, colliders, tri_vertices=None):
        cols = np.ascontiguousarray(colliders)
        desc = cols.view(np.float32).reshape(-1)
        tri = np.zeros((0, 3), np.float32) if tri_vertices is None else np.ascontiguousarray(tri_vertices, np.float32)
        ntri = tri.shape[0] // 3
        self.L.orc_set_colliders(self.h, len(cols), _ptr(desc, _f), ntri, _ptr(tri.reshape(-1), _f))

    def set_use_cpic(self, on: bool):
        self.L.orc_set_use_cpic(self.h, int(on))

    def step(self, steps: int = 1) -> int:
        return self.L.orc_run(self.h, steps)

    def sort(self) -> int:
        return self.L.orc_sort(self.h)

    def p2g(self):
        self.L.orc_p2g(self.h)

    def grid_update(self):
        self.L.orc_grid_update(self.h)

    def g2p(self):
        self.L.orc_g2p(self.h)

    def particle_update(self):
        self.L.orc_particle_update(self.h)

    @property
    def num_blocks(self) -> int:
        return self.L.orc_num_blocks(self.h)

    def timestep_bound_bits(self) -> int:
        """CFL bound (solver/timestep_bound.rs:59-115) as (dt * 1e12) as u32."""
        return int(self.L.orc_timestep_bound_bits(self.h))

    @property
    def status(self) -> int:
        return self.L.orc_status(self.h)

    def headers(self) -> np.ndarray:
        out = np.zeros((self.num_blocks, HEADER_FIELDS), np.int32)
        self.L.orc_get_headers(self.h, _ptr(out, _i))
        return out

    def sorted_ids(self) -> np.ndarray:
        out = np.zeros(self.L.orc_sorted_len(self.h), np.uint32)
        self.L.orc_get_sorted(self.h, _ptr(out, _u))
        return out

    def nodes(self) -> np.ndarray:
        out = np.zeros((self.num_blocks, 64, 8), np.float32)
        self.L.orc_get_nodes(self.h, _ptr(out, _f))
        return out

    def particles(self) -> dict:
        n = self.n
        out = dict(pos=np.zeros((n, 3), np.float32), vel=np.zeros((n, 3), np.float32),
                   aff=np.zeros((n, 9), np.float32), def_grad=np.zeros((n, 9), np.float32),
                   vel_grad_det=np.zeros(n, np.float32), mass=np.zeros(n, np.float32),
                   enabled=np.zeros(n, np.uint32), model=np.zeros((n, 25), np.uint32))
        self.L.orc_get_particles(self.h, _ptr(out["pos"], _f), _ptr(out["vel"], _f), _ptr(out["aff"], _f),
                                 _ptr(out["def_grad"], _f), _ptr(out["vel_grad_det"], _f), _ptr(out["mass"], _f),
                                 _ptr(out["enabled"], _u), _ptr(out["model"], _u))
        return out

    def positions_f64(self) -> np.ndarray:
        out = np.zeros((self.n, 3), np.float64)
        self.L.orc_get_positions_f64(self.h, _ptr(out, _d))
        return out

    def project_point(self, collider: int, pt):
        p = np.asarray(pt, np.float32)
        out = np.zeros(3, np.float32)
        inside = self.L.orc_project_point(self.h, collider, _ptr(p, _f), _ptr(out, _f))
        return out, inside


# -- free functions -----------------------------------------------------------

def pack_key(x, y, z, precision="f32") -> int:
    return lib(precision).orc_pack_key(x, y, z)


def hash_key(k, precision="f32") -> int:
    return lib(precision).orc_hash(k)


def kernel_eval(x, precision="f32") -> float:
    return lib(precision).orc_kernel_eval(x)


def kernel_eval_all(x, precision="f32") -> np.ndarray:
    out = np.zeros(3, np.float64)
    lib(precision).orc_kernel_eval_all(x, _ptr(out, _d))
    return out


def block_of_point(dx, pt, precision="f32"):
    p = np.asarray(pt, np.float32)
    b = np.zeros(3, np.int32)
    a = np.zeros(3, np.uint32)
    lib(precision).orc_block_of_point(dx, _ptr(p, _f), _ptr(b, _i), _ptr(a, _u))
    return b, a


def model_update(model_words, F, vel_grad, precision="f32"):
    """One constitutive update: returns (tau, new F, new model words)."""
    w = np.ascontiguousarray(np.asarray(model_words, np.uint32)[1:25].copy())
    Fm = np.ascontiguousarray(np.asarray(F, np.float32).reshape(9).copy())
    vg = np.ascontiguousarray(np.asarray(vel_grad, np.float32).reshape(9))
    tau = np.zeros(9, np.float32)
    lib(precision).orc_model_update(int(model_words[0]), _ptr(w, _u), _ptr(Fm, _f), _ptr(vg, _f), _ptr(tau, _f))
    words = np.concatenate([[model_words[0]], w]).astype(np.uint32)
    return tau, Fm, words


def svd(F, precision="f32"):
    Fm = np.ascontiguousarray(np.asarray(F, np.float32).reshape(9))
    u, s, vt = np.zeros(9, np.float32), np.zeros(3, np.float32), np.zeros(9, np.float32)
    lib(precision).orc_svd(_ptr(Fm, _f), _ptr(u, _f), _ptr(s, _f), _ptr(vt, _f))
    return u, s, vt


def bc_project(ty, friction, vel, n, precision="f32") -> np.ndarray:
    v = np.asarray(vel, np.float32)
    nn = np.asarray(n, np.float32)
    out = np.zeros(3, np.float32)
    lib(precision).orc_bc_project(ty, friction, _ptr(v, _f), _ptr(nn, _f), _ptr(out, _f))
    return out


def inv4(m, precision="f64"):
    """(inverse, determinant) of a 4x4 matrix by the oracle's 2x2-minor expansion."""
    a = np.ascontiguousarray(m, np.float64).reshape(16)
    out = np.zeros(16, np.float64)
    det = lib(precision).orc_inv4(_ptr(a, _d), _ptr(out, _d))
    return out.reshape(4, 4), det


def prefix_sum(values) -> np.ndarray:
    v = np.ascontiguousarray(np.asarray(values, np.uint32).copy())
    lib("f32").orc_prefix_sum(_ptr(v, _u), len(v))
    return v
