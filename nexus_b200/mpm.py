"""Python front-end over the C ABI (include/nexus_mpm.h), mirroring nexus_mpm.

``MpmPipeline`` / ``MpmState`` follow ``src_mpm/pipeline.rs`` (``MpmPipeline::new``,
``step``; ``MpmState::empty``, ``set_simulation_params``, ``write_substep_params``,
``set_cell_width``, ``set_coupling``, ``use_cpic``) and ``GpuParticles``
(``src_mpm/solver/particle.rs``: ``append``, ``swap_remove``, ``shift_remove``,
``read_positions``).  All work happens in libnexus_mpm.so on an sm_100 GPU;
loading fails loudly if the library or the GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .particles import ParticleBatch, COLLIDER_DTYPE, particle_records

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnexus_mpm.so")

NXM_OK = 0
NXM_E_INVALID = -1
NXM_E_CUDA = -2
NXM_E_CAPACITY = -3
NXM_E_HASH_FULL = -4
NXM_E_NO_DEVICE = -5
NXM_E_UNSUPPORTED = -6
NXM_E_OOM = -7

# RenderConfig modes of the render data (solver/prep_readback.rs:16-21)
RENDER_DEFAULT, RENDER_VOLUME, RENDER_VELOCITY, RENDER_PHASE = 0, 1, 2, 3
RENDER_CDF_NORMALS, RENDER_CDF_DISTANCES, RENDER_CDF_SIGNS = 4, 5, 6

HEADER_FIELDS = 23

# Every function the header declares, with its ctypes signature.
_vp = C.c_void_p
_f = C.POINTER(C.c_float)
_u = C.POINTER(C.c_uint32)
_i = C.POINTER(C.c_int32)
_pp = C.POINTER(C.c_void_p)


class SimulationParamsC(C.Structure):
    _fields_ = [("gravity", C.c_float * 3), ("dt", C.c_float)]


class CapacitiesC(C.Structure):
    _fields_ = [("grid_size", C.c_uint32), ("particles_capacity", C.c_uint32)]


class ParticlesSoAC(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in (
        "position", "velocity", "def_grad", "affine", "vel_grad_det", "init_volume", "init_radius", "mass",
        "damping", "phase", "boundary_friction", "group_id", "enabled", "fixed", "model")]


class TuningC(C.Structure):
    _fields_ = [("p2g_ctas_per_sm", C.c_uint32), ("g2p_ctas_per_sm", C.c_uint32), ("sort_ctas_per_sm", C.c_uint32),
                ("grid_ctas_per_sm", C.c_uint32), ("sort_batch", C.c_uint32), ("range_min_fill", C.c_uint32),
                ("density", C.c_uint32), ("scenes", C.c_uint32), ("ms_before", C.c_float), ("ms_after", C.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TimestampsC(C.Structure):
    _fields_ = [("sort_ms", C.c_float), ("p2g_ms", C.c_float), ("grid_update_ms", C.c_float),
                ("g2p_ms", C.c_float), ("total_ms", C.c_float)]


SIGNATURES = {
    "nxm_pipeline_create": (C.c_int, [_pp]),
    "nxm_pipeline_destroy": (None, [_vp]),
    "nxm_step": (C.c_int, [_vp, _vp, C.POINTER(TimestampsC)]),
    "nxm_state_create": (C.c_int, [C.POINTER(CapacitiesC), _pp]),
    "nxm_state_destroy": (None, [_vp]),
    "nxm_state_set_simulation_params": (C.c_int, [_vp, C.POINTER(SimulationParamsC)]),
    "nxm_state_write_substep_params": (C.c_int, [_vp, C.c_uint32]),
    "nxm_state_set_cell_width": (C.c_int, [_vp, C.c_float, C.c_uint32]),
    "nxm_state_set_colliders": (C.c_int, [_vp, _vp, C.c_uint32, _f, C.c_uint32]),
    "nxm_state_set_collider_velocity": (C.c_int, [_vp, C.c_uint32, _f, _f]),
    "nxm_state_read_collider_pose": (C.c_int, [_vp, C.c_uint32, _f]),
    "nxm_state_set_use_cpic": (C.c_int, [_vp, C.c_int]),
    "nxm_state_set_deterministic": (C.c_int, [_vp, C.c_int]),
    "nxm_particles_append": (C.c_int, [_vp, _vp, C.c_uint32]),
    "nxm_particles_append_soa": (C.c_int, [_vp, C.POINTER(ParticlesSoAC), C.c_uint32]),
    "nxm_particles_swap_remove": (C.c_int, [_vp, _u, C.c_uint32, _u, _u]),
    "nxm_particles_shift_remove": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "nxm_particles_len": (C.c_uint32, [_vp]),
    "nxm_read_positions": (C.c_int, [_vp, _f]),
    "nxm_read_velocities": (C.c_int, [_vp, _f]),
    "nxm_read_affine": (C.c_int, [_vp, _f]),
    "nxm_read_def_grad": (C.c_int, [_vp, _f]),
    "nxm_read_vel_grad_det": (C.c_int, [_vp, _f]),
    "nxm_read_mass": (C.c_int, [_vp, _f]),
    "nxm_read_enabled": (C.c_int, [_vp, _u]),
    "nxm_read_models": (C.c_int, [_vp, _u]),
    "nxm_grid_num_blocks": (C.c_int, [_vp, _u]),
    "nxm_grid_read_headers": (C.c_int, [_vp, _i, C.c_uint32]),
    "nxm_grid_sorted_len": (C.c_int, [_vp, _u]),
    "nxm_grid_read_sorted_ids": (C.c_int, [_vp, _u, C.c_uint32]),
    "nxm_grid_read_nodes": (C.c_int, [_vp, _f, C.c_uint32]),
    "nxm_debug_sort": (C.c_int, [_vp, _vp, C.c_int]),
    "nxm_debug_copy_wait_timeout": (C.c_int, [_vp, C.c_uint32]),
    "nxm_debug_fail_allocation": (C.c_int, [C.c_int64]),
    "nxm_state_estimate_timestep_bound": (C.c_int, [_vp, _f, _u]),
    "nxm_read_cdf": (C.c_int, [_vp, _f]),
    "nxm_simulate_frame": (C.c_int, [_vp, _vp, C.c_uint32, C.c_uint32, _u]),
    "nxm_state_status_pipelined": (C.c_int, [_vp, _u]),
    "nxm_state_status_poll": (C.c_int, [_vp, _u, C.POINTER(C.c_int)]),
    "nxm_state_read_status_async": (C.c_int, [_vp, _u, C.POINTER(C.c_uint64)]),
    "nxm_state_fence": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "nxm_state_ticket_done": (C.c_int, [_vp, C.c_uint64, C.POINTER(C.c_int)]),
    "nxm_state_ticket_wait": (C.c_int, [_vp, C.c_uint64]),
    "nxm_read_positions_range_async": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _f, C.POINTER(C.c_uint64)]),
    "nxm_host_alloc": (C.c_int, [C.c_size_t, _pp]),
    "nxm_host_free": (None, [_vp]),
    "nxm_state_num_rigid_particles": (C.c_int, [_vp, _u]),
    "nxm_read_rigid_particles": (C.c_int, [_vp, _f]),
    "nxm_prep_readback": (C.c_int, [_vp, C.c_uint32, _f, C.c_uint32, _f]),
    "nxm_prep_render": (C.c_int, [_vp, C.c_uint32, _f, C.c_uint32, _vp, _vp, _vp]),
    "nxm_prep_readback_rigid": (C.c_int, [_vp, _f, _f, C.c_uint32, _f]),
    "nxm_state_set_collider_velocities": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _f]),
    "nxm_state_enable_scenes": (C.c_int, [_vp, C.c_uint32]),
    "nxm_scene_capacity": (C.c_uint32, [_vp]),
    "nxm_scene_add": (C.c_int, [_vp, C.POINTER(ParticlesSoAC), C.c_uint32, _vp, C.c_uint32, _f, C.c_uint32, _u]),
    "nxm_scene_remove": (C.c_int, [_vp, _u, C.c_uint32]),
    "nxm_scene_range": (C.c_int, [_vp, C.c_uint32, _u, _u]),
    "nxm_scene_set_collider_velocity": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _f, _f]),
    "nxm_read_positions_range": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _f]),
    "nxm_chunk_add": (C.c_int, [_vp, _vp, C.c_uint32, _u]),
    "nxm_chunk_extend": (C.c_int, [_vp, C.c_uint32, _vp, C.c_uint32]),
    "nxm_chunk_remove": (C.c_int, [_vp, C.c_uint32]),
    "nxm_chunk_remove_particles": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _u]),
    "nxm_chunk_len": (C.c_int, [_vp, C.c_uint32, _u]),
    "nxm_chunk_of_particles": (C.c_int, [_vp, _u]),
    "nxm_synchronize": (C.c_int, [_vp]),
    "nxm_state_status": (C.c_int, [_vp, _u, C.c_int]),
    "nxm_error_string": (C.c_char_p, [C.c_int]),
    "nxm_state_kernel_launches": (C.c_uint64, [_vp]),
    "nxm_state_cuda_stream": (C.c_void_p, [_vp]),
    "nxm_sort_blocks_noalloc": (C.c_int, [_vp, C.c_uint32, C.c_float, _vp, _vp, _vp, C.c_uint32, _u, _vp]),
    "nxm_state_autotune": (C.c_int, [_vp, C.c_uint32, C.POINTER(TuningC)]),
    "nxm_state_get_tuning": (C.c_int, [_vp, C.POINTER(TuningC)]),
    "nxm_state_set_tuning": (C.c_int, [_vp, C.POINTER(TuningC)]),
    "nxm_tuning_table": (C.c_uint32, [C.POINTER(TuningC), C.c_uint32]),
}

_LIB = None


class NexusError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        msg = load().nxm_error_string(code).decode() if _LIB is not None else str(code)
        super().__init__(f"{what}: {msg} ({code})")


def load(path: str | None = None):
    """Loads libnexus_mpm.so (no fallback: a missing library is an error).
    NXM_LIB in the environment selects another build of the same library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = path or os.environ.get("NXM_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run python -m nexus_b200.build")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _check(rc: int, what: str):
    if rc != NXM_OK:
        raise NexusError(rc, what)


def _p(a, t=_f):
    return a.ctypes.data_as(t)


class PinnedArray:
    """Page-locked host memory (nxm_host_alloc) seen as a numpy array
    (``.array``); freed with the object, so keep it while a copy may still
    write into it."""

    def __init__(self, shape, dtype=np.float32):
        self.lib = load()
        count = int(np.prod(shape))
        nbytes = max(count * np.dtype(dtype).itemsize, 1)
        ptr = C.c_void_p()
        _check(self.lib.nxm_host_alloc(nbytes, C.byref(ptr)), "host_alloc")
        self.ptr = ptr
        buf = (C.c_char * nbytes).from_address(ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=count).reshape(shape)

    def close(self):
        if getattr(self, "ptr", None) is not None and self.ptr.value:
            self.array = None
            self.lib.nxm_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


class MpmPipeline:
    """``MpmPipeline::new`` (src_mpm/pipeline.rs:366-382)."""

    def __init__(self):
        self.lib = load()
        h = C.c_void_p()
        _check(self.lib.nxm_pipeline_create(C.byref(h)), "nxm_pipeline_create")
        self.h = h

    def simulate_frame(self, state: "MpmState", min_substeps: int = 1, max_substeps: int = 1000) -> int:
        """``NexusPipeline::simulate`` (MPM part) with the substep count from the
        CFL bound: returns the number of substeps run."""
        n = np.zeros(1, np.uint32)
        _check(self.lib.nxm_simulate_frame(self.h, state.h, min_substeps, max_substeps, _p(n, _u)), "simulate_frame")
        return int(n[0])

    def step(self, state: "MpmState", timestamps: bool = False):
        """``MpmPipeline::step`` (src_mpm/pipeline.rs:385-526).  Enqueued; with
        ``timestamps`` it waits and returns the per-phase device times (ms)."""
        if timestamps:
            ts = TimestampsC()
            _check(self.lib.nxm_step(self.h, state.h, C.byref(ts)), "nxm_step")
            return {k: getattr(ts, k) for k, _ in TimestampsC._fields_}
        _check(self.lib.nxm_step(self.h, state.h, None), "nxm_step")
        return None

    def debug_sort(self, state: "MpmState", with_p2g: bool = False):
        _check(self.lib.nxm_debug_sort(self.h, state.h, int(with_p2g)), "nxm_debug_sort")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.nxm_pipeline_destroy(self.h)
            self.h = None


class MpmState:
    """``MpmState::empty`` (src_mpm/pipeline.rs:107-165) plus its setters."""

    def __init__(self, grid_size: int = 32768, particles_capacity: int = 65536):
        self.lib = load()
        caps = CapacitiesC(grid_size, particles_capacity)
        h = C.c_void_p()
        _check(self.lib.nxm_state_create(C.byref(caps), C.byref(h)), "nxm_state_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.nxm_state_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- parameters -----------------------------------------------------------
    def set_simulation_params(self, gravity, dt):
        p = SimulationParamsC((C.c_float * 3)(*gravity), dt)
        _check(self.lib.nxm_state_set_simulation_params(self.h, C.byref(p)), "set_simulation_params")

    def write_substep_params(self, num_substeps: int):
        _check(self.lib.nxm_state_write_substep_params(self.h, num_substeps), "write_substep_params")

    def set_cell_width(self, cell_width: float, grid_capacity: int):
        _check(self.lib.nxm_state_set_cell_width(self.h, cell_width, grid_capacity), "set_cell_width")

    def set_colliders(self, colliders: np.ndarray, tri_vertices=None):
        cols = np.ascontiguousarray(colliders, dtype=COLLIDER_DTYPE)
        tri = (np.zeros((0,), np.float32) if tri_vertices is None
               else np.ascontiguousarray(tri_vertices, np.float32).reshape(-1))
        _check(self.lib.nxm_state_set_colliders(self.h, cols.ctypes.data_as(C.c_void_p), len(cols), _p(tri),
                                                tri.size // 9), "set_colliders")

    def set_collider_velocity(self, index: int, linvel, angvel):
        lv = np.asarray(linvel, np.float32)
        av = np.asarray(angvel, np.float32)
        _check(self.lib.nxm_state_set_collider_velocity(self.h, index, _p(lv), _p(av)), "set_collider_velocity")

    def collider_pose(self, index: int) -> np.ndarray:
        out = np.zeros(7, np.float32)
        _check(self.lib.nxm_state_read_collider_pose(self.h, index, _p(out)), "read_collider_pose")
        return out

    def set_collider_velocities(self, first: int, vel6):
        """Linear + angular velocity (n, 6) of colliders first.. first + n, stream-ordered."""
        v = np.ascontiguousarray(vel6, np.float32).reshape(-1, 6)
        _check(self.lib.nxm_state_set_collider_velocities(self.h, first, len(v), _p(v, _f)),
               "set_collider_velocities")

    def set_use_cpic(self, enabled: bool):
        _check(self.lib.nxm_state_set_use_cpic(self.h, int(enabled)), "set_use_cpic")

    def set_deterministic(self, enabled: bool):
        _check(self.lib.nxm_state_set_deterministic(self.h, int(enabled)), "set_deterministic")

    # -- particles --------------------------------------------------------------
    @staticmethod
    def _soa(batch: ParticleBatch, keep: dict):
        def arr(name, dtype):
            a = np.ascontiguousarray(getattr(batch, name), dtype=dtype)
            keep[name] = a
            return a.ctypes.data_as(C.c_void_p)

        return ParticlesSoAC(
            arr("pos", np.float32), arr("vel", np.float32), arr("def_grad", np.float32), arr("aff", np.float32),
            arr("vel_grad_det", np.float32), arr("init_volume", np.float32), arr("init_radius", np.float32),
            arr("mass", np.float32), arr("damping", np.float32), arr("phase", np.float32),
            arr("boundary_friction", np.float32), arr("group_id", np.uint32), arr("enabled", np.uint32),
            arr("fixed", np.uint32), arr("model", np.uint32))

    def append(self, batch: ParticleBatch):
        """``GpuParticles::append`` (src_mpm/solver/particle.rs:533-565), bulk SoA form."""
        keep = {}
        soa = self._soa(batch, keep)
        _check(self.lib.nxm_particles_append_soa(self.h, C.byref(soa), batch.n), "append")

    # -- batched scenes ------------------------------------------------------------------
    def enable_scenes(self, scene_blocks: int):
        _check(self.lib.nxm_state_enable_scenes(self.h, scene_blocks), "enable_scenes")

    def scene_capacity(self) -> int:
        return int(self.lib.nxm_scene_capacity(self.h))

    def add_scene(self, batch: ParticleBatch, colliders=None, tri_vertices=None) -> int:
        keep = {}
        soa = self._soa(batch, keep)
        cols = np.ascontiguousarray(colliders if colliders is not None else np.zeros(0, COLLIDER_DTYPE),
                                    dtype=COLLIDER_DTYPE)
        tri = (np.zeros((0,), np.float32) if tri_vertices is None
               else np.ascontiguousarray(tri_vertices, np.float32).reshape(-1))
        sid = C.c_uint32()
        _check(self.lib.nxm_scene_add(self.h, C.byref(soa), batch.n,
                                      cols.ctypes.data_as(C.c_void_p), len(cols), _p(tri), tri.size // 9,
                                      C.byref(sid)), "scene_add")
        return sid.value

    def remove_scenes(self, scenes):
        ids = np.ascontiguousarray(list(scenes), np.uint32)
        _check(self.lib.nxm_scene_remove(self.h, _p(ids, _u), len(ids)), "scene_remove")

    def scene_range(self, scene: int) -> tuple[int, int]:
        a, b = C.c_uint32(), C.c_uint32()
        _check(self.lib.nxm_scene_range(self.h, scene, C.byref(a), C.byref(b)), "scene_range")
        return a.value, b.value

    def set_scene_collider_velocity(self, scene: int, index: int, linvel, angvel):
        lv = np.asarray(linvel, np.float32)
        av = np.asarray(angvel, np.float32)
        _check(self.lib.nxm_scene_set_collider_velocity(self.h, scene, index, _p(lv), _p(av)),
               "scene_set_collider_velocity")

    def read_positions_range(self, first: int, count: int) -> np.ndarray:
        out = np.zeros((max(count, 1), 3), np.float32)
        _check(self.lib.nxm_read_positions_range(self.h, first, count, _p(out, _f)), "read_positions_range")
        return out[:count]

    def read_scene_positions(self, scene: int) -> np.ndarray:
        return self.read_positions_range(*self.scene_range(scene))

    def read_scene_particles(self, scene: int) -> dict:
        """Every field of ``read_particles`` for the particles of one scene."""
        first, count = self.scene_range(scene)
        return {k: v[first:first + count] for k, v in self.read_particles().items()}

    # -- asynchronous reads and tickets --------------------------------------------
    def fence(self) -> int:
        """A ticket for the work queued on the state's stream so far."""
        t = C.c_uint64()
        _check(self.lib.nxm_state_fence(self.h, C.byref(t)), "state_fence")
        return t.value

    def ticket_done(self, ticket: int) -> bool:
        d = C.c_int()
        _check(self.lib.nxm_state_ticket_done(self.h, ticket, C.byref(d)), "state_ticket_done")
        return bool(d.value)

    def ticket_wait(self, ticket: int):
        _check(self.lib.nxm_state_ticket_wait(self.h, ticket), "state_ticket_wait")

    def read_positions_range_async(self, first: int, count: int, out: np.ndarray) -> int:
        """``GpuParticles::read_positions`` as an async read: positions of ids
        [first, first + count) into ``out`` ((count, 3) float32, best pinned:
        ``PinnedArray``); returns the ticket after which ``out`` holds them."""
        assert out.dtype == np.float32 and out.shape == (count, 3) and out.flags.c_contiguous
        t = C.c_uint64()
        _check(self.lib.nxm_read_positions_range_async(self.h, first, count, _p(out, _f), C.byref(t)),
               "read_positions_range_async")
        return t.value

    def read_status_async(self, out: np.ndarray) -> int:
        """The status word at this point of the stream into ``out`` (one uint32,
        best pinned); returns the ticket after which it holds it."""
        assert out.dtype == np.uint32 and out.size == 1 and out.flags.c_contiguous
        t = C.c_uint64()
        _check(self.lib.nxm_state_read_status_async(self.h, _p(out, _u), C.byref(t)), "read_status_async")
        return t.value

    def read_scene_positions_async(self, scene: int, out: np.ndarray) -> int:
        return self.read_positions_range_async(*self.scene_range(scene), out)

    # -- particle chunks (NexusState, src/state.rs:665-774) ------------------------
    def add_chunk(self, batch: ParticleBatch) -> int:
        rec = particle_records(batch)
        c = C.c_uint32()
        _check(self.lib.nxm_chunk_add(self.h, rec.ctypes.data_as(C.c_void_p), batch.n, C.byref(c)), "chunk_add")
        return c.value

    def extend_chunk(self, chunk: int, batch: ParticleBatch):
        rec = particle_records(batch)
        _check(self.lib.nxm_chunk_extend(self.h, chunk, rec.ctypes.data_as(C.c_void_p), batch.n), "chunk_extend")

    def remove_chunk(self, chunk: int):
        _check(self.lib.nxm_chunk_remove(self.h, chunk), "chunk_remove")

    def remove_particles_from_chunk(self, chunk: int, count: int) -> int:
        r = C.c_uint32()
        _check(self.lib.nxm_chunk_remove_particles(self.h, chunk, count, C.byref(r)), "chunk_remove_particles")
        return r.value

    def chunk_len(self, chunk: int) -> int:
        r = C.c_uint32()
        _check(self.lib.nxm_chunk_len(self.h, chunk, C.byref(r)), "chunk_len")
        return r.value

    def chunk_of_particles(self) -> np.ndarray:
        out = np.zeros(max(len(self), 1), np.uint32)
        _check(self.lib.nxm_chunk_of_particles(self.h, _p(out, _u)), "chunk_of_particles")
        return out[:len(self)]

    def swap_remove(self, slots):
        s = np.ascontiguousarray(slots, np.uint32)
        remaps = np.zeros((max(len(s), 1), 2), np.uint32)
        nr = C.c_uint32()
        _check(self.lib.nxm_particles_swap_remove(self.h, _p(s, _u), len(s), _p(remaps, _u), C.byref(nr)),
               "swap_remove")
        return [tuple(r) for r in remaps[:nr.value]]

    def shift_remove(self, start: int, end: int):
        _check(self.lib.nxm_particles_shift_remove(self.h, start, end), "shift_remove")

    def __len__(self):
        return int(self.lib.nxm_particles_len(self.h))

    # -- readback -----------------------------------------------------------------
    def _read(self, fn, shape, dtype=np.float32, t=_f):
        out = np.zeros(shape, dtype)
        _check(getattr(self.lib, fn)(self.h, _p(out, t)), fn)
        return out

    def read_positions(self) -> np.ndarray:
        return self._read("nxm_read_positions", (len(self), 3))

    def read_positions_into(self, out: np.ndarray):
        """Positions into a caller-provided (n, 3) float32 host array (e.g. pinned)."""
        assert out.dtype == np.float32 and out.shape == (len(self), 3) and out.flags.c_contiguous
        _check(self.lib.nxm_read_positions(self.h, _p(out)), "nxm_read_positions")

    def read_velocities(self) -> np.ndarray:
        return self._read("nxm_read_velocities", (len(self), 3))

    def read_affine(self) -> np.ndarray:
        return self._read("nxm_read_affine", (len(self), 9))

    def read_def_grad(self) -> np.ndarray:
        return self._read("nxm_read_def_grad", (len(self), 9))

    def read_vel_grad_det(self) -> np.ndarray:
        return self._read("nxm_read_vel_grad_det", (len(self),))

    def read_mass(self) -> np.ndarray:
        return self._read("nxm_read_mass", (len(self),))

    def read_enabled(self) -> np.ndarray:
        return self._read("nxm_read_enabled", (len(self),), np.uint32, _u)

    def read_models(self) -> np.ndarray:
        return self._read("nxm_read_models", (len(self), 25), np.uint32, _u)

    def read_cdf(self) -> dict:
        """CPIC particle fields: normal, signed distance, rigid velocity, affinity bits."""
        out = np.zeros((max(len(self), 1), 8), np.float32)
        _check(self.lib.nxm_read_cdf(self.h, _p(out, _f)), "read_cdf")
        out = out[:len(self)]
        return dict(normal=out[:, :3], signed_distance=out[:, 3], rigid_vel=out[:, 4:7],
                    affinity=out[:, 7].copy().view(np.uint32))

    def num_rigid_particles(self) -> int:
        """``GpuRigidParticles::len``: CPIC surface samples of the trimesh colliders."""
        n = np.zeros(1, np.uint32)
        _check(self.lib.nxm_state_num_rigid_particles(self.h, _p(n, _u)), "num_rigid_particles")
        return int(n[0])

    def read_rigid_particles(self) -> dict:
        """CPIC rigid particles in sampling order: local position, collider,
        triangle index inside the collider's triangle range."""
        n = self.num_rigid_particles()
        out = np.zeros((max(n, 1), 5), np.float32)
        _check(self.lib.nxm_read_rigid_particles(self.h, _p(out, _f)), "read_rigid_particles")
        out = out[:n]
        return dict(local=out[:, :3], collider=out[:, 3].copy().view(np.uint32),
                    triangle=out[:, 4].copy().view(np.uint32))

    @staticmethod
    def _render_records(out: np.ndarray) -> dict:
        return dict(color=out[:, 0:4], deformation=out[:, 4:20].reshape(-1, 4, 4), position=out[:, 20:23])

    @staticmethod
    def _palette(palette):
        if palette is None:
            return None, 0
        pal = np.ascontiguousarray(palette, np.float32).reshape(-1, 4)
        return pal, len(pal)

    def prep_readback(self, mode: int = 0, palette=None) -> dict:
        """``WgPrepReadback::launch`` (headless): per particle in id order its
        render color for `mode` (RENDER_*), deformation (n, 4, 4) as columns
        of Mat4::from_mat3(diag(2 r) clamp(F, -4, 4)) and position."""
        pal, ng = self._palette(palette)
        out = np.zeros((max(len(self), 1), 24), np.float32)
        _check(self.lib.nxm_prep_readback(self.h, mode, None if pal is None else _p(pal, _f), ng, _p(out, _f)),
               "prep_readback")
        return self._render_records(out[:len(self)])

    def prep_render(self, mode: int, positions: int, deformations: int, colors: int, palette=None):
        """``WgPrepReadback::launch_render``: the render data written into
        caller-owned device buffers (device pointers as ints: n x 3, n x 9,
        n x 4 floats), asynchronously on the state's stream."""
        pal, ng = self._palette(palette)
        _check(self.lib.nxm_prep_render(self.h, mode, None if pal is None else _p(pal, _f), ng,
                                        C.c_void_p(positions), C.c_void_p(deformations), C.c_void_p(colors)),
               "prep_render")

    def prep_readback_rigid(self, colors=None, palette=None) -> dict:
        """``gpu_prep_readback_rigid``: per CPIC rigid particle its base color,
        deformation diag(0.4 dx) and world position."""
        n = self.num_rigid_particles()
        pal, ng = self._palette(palette)
        cols = None if colors is None else np.ascontiguousarray(colors, np.float32).reshape(-1, 4)
        out = np.zeros((max(n, 1), 24), np.float32)
        _check(self.lib.nxm_prep_readback_rigid(self.h, None if cols is None else _p(cols, _f),
                                                None if pal is None else _p(pal, _f), ng, _p(out, _f)),
               "prep_readback_rigid")
        return self._render_records(out[:n])

    def estimate_timestep_bound(self) -> tuple[float, int]:
        """``WgTimestepBounds::compute_bounds``: (max dt in seconds, fixed-point bits)."""
        dt = np.zeros(1, np.float32)
        bits = np.zeros(1, np.uint32)
        _check(self.lib.nxm_state_estimate_timestep_bound(self.h, _p(dt, _f), _p(bits, _u)), "estimate_timestep_bound")
        return float(dt[0]), int(bits[0])

    def read_particles(self) -> dict:
        return dict(pos=self.read_positions(), vel=self.read_velocities(), aff=self.read_affine(),
                    def_grad=self.read_def_grad(), vel_grad_det=self.read_vel_grad_det(), mass=self.read_mass(),
                    enabled=self.read_enabled(), model=self.read_models())

    # -- grid ------------------------------------------------------------------------
    def num_blocks(self) -> int:
        v = C.c_uint32()
        _check(self.lib.nxm_grid_num_blocks(self.h, C.byref(v)), "grid_num_blocks")
        return v.value

    def headers(self) -> np.ndarray:
        nb = self.num_blocks()
        out = np.zeros((nb, HEADER_FIELDS), np.int32)
        _check(self.lib.nxm_grid_read_headers(self.h, _p(out, _i), nb), "grid_read_headers")
        return out

    def sorted_ids(self) -> np.ndarray:
        v = C.c_uint32()
        _check(self.lib.nxm_grid_sorted_len(self.h, C.byref(v)), "grid_sorted_len")
        out = np.zeros(v.value, np.uint32)
        _check(self.lib.nxm_grid_read_sorted_ids(self.h, _p(out, _u), v.value), "grid_read_sorted_ids")
        return out

    def nodes(self) -> np.ndarray:
        nb = self.num_blocks()
        out = np.zeros((nb, 64, 4), np.float32)
        _check(self.lib.nxm_grid_read_nodes(self.h, _p(out), nb), "grid_read_nodes")
        return out

    # -- status ------------------------------------------------------------------------
    def synchronize(self):
        _check(self.lib.nxm_synchronize(self.h), "synchronize")

    def status(self, clear: bool = False) -> int:
        v = C.c_uint32()
        _check(self.lib.nxm_state_status(self.h, C.byref(v), int(clear)), "state_status")
        return v.value

    def status_pipelined(self) -> int:
        """Status word of the previous call's point in the stream, without
        draining the stream (the read for this point is enqueued)."""
        v = C.c_uint32()
        _check(self.lib.nxm_state_status_pipelined(self.h, C.byref(v)), "state_status_pipelined")
        return v.value

    def status_poll(self):
        """Non-blocking: the status word posted by an earlier call once its
        store has run on the GPU, else None (nothing waits)."""
        v, ready = C.c_uint32(), C.c_int()
        _check(self.lib.nxm_state_status_poll(self.h, C.byref(v), C.byref(ready)), "state_status_poll")
        return v.value if ready.value else None

    def autotune(self, trial_steps: int = 5) -> dict:
        """Picks the step's launch shapes by timing this state's own steps
        (the state advances by every step taken); trial_steps = 0 only applies
        the decision table's entry for this kind of state."""
        t = TuningC()
        _check(self.lib.nxm_state_autotune(self.h, trial_steps, C.byref(t)), "state_autotune")
        return t.as_dict()

    def tuning(self) -> dict:
        t = TuningC()
        _check(self.lib.nxm_state_get_tuning(self.h, C.byref(t)), "state_get_tuning")
        return t.as_dict()

    def set_tuning(self, **kw):
        t = TuningC()
        _check(self.lib.nxm_state_get_tuning(self.h, C.byref(t)), "state_get_tuning")
        for k, v in kw.items():
            setattr(t, k, v)
        _check(self.lib.nxm_state_set_tuning(self.h, C.byref(t)), "state_set_tuning")

    def kernel_launches(self) -> int:
        return int(self.lib.nxm_state_kernel_launches(self.h))

    def cuda_stream(self) -> int:
        """The cudaStream_t (as an integer) all of this state's work runs on."""
        return int(self.lib.nxm_state_cuda_stream(self.h) or 0)


def debug_fail_allocation(after: int):
    """Test hook (nxm_debug_fail_allocation): the after-th device allocation of
    the library from now on fails once with NXM_E_OOM; -1 disarms."""
    _check(load().nxm_debug_fail_allocation(int(after)), "debug_fail_allocation")


def tuning_table() -> list:
    """The autotuner's decision table of this process (one dict per key)."""
    lib = load()
    n = lib.nxm_tuning_table(None, 0)
    arr = (TuningC * max(n, 1))()
    lib.nxm_tuning_table(arr, n)
    return [arr[i].as_dict() for i in range(n)]


def state_from_scene(scene, deterministic: bool = False, grid_capacity: int | None = None,
                     use_cpic: bool = False) -> MpmState:
    """Builds a device state for a ``nexus_b200.scenes.Scene``."""
    st = MpmState(grid_size=grid_capacity or scene.grid_capacity, particles_capacity=scene.n)
    st.set_cell_width(scene.dx, grid_capacity or scene.grid_capacity)
    st.set_simulation_params(scene.gravity, scene.dt)
    st.set_colliders(scene.colliders, scene.tri_vertices if scene.tri_vertices.size else None)
    st.set_deterministic(deterministic)
    if use_cpic:
        st.set_use_cpic(True)
    st.append(scene.particles)
    return st


def batched_state_from_scenes(scenes_, deterministic: bool = False, scene_blocks: int = 64,
                              grid_capacity: int | None = None):
    """One device state advancing several ``Scene``s together (same dx, dt and
    gravity).  Returns the state and the scene slot of each input scene."""
    s0 = scenes_[0]
    for sc in scenes_:
        if (sc.dx, sc.dt, tuple(sc.gravity)) != (s0.dx, s0.dt, tuple(s0.gravity)):
            raise ValueError("batched scenes share dx, dt and gravity")
    n = sum(sc.n for sc in scenes_)
    cap = grid_capacity or sum(sc.grid_capacity for sc in scenes_)
    st = MpmState(grid_size=cap, particles_capacity=n)
    st.set_cell_width(s0.dx, cap)
    st.set_simulation_params(s0.gravity, s0.dt)
    st.set_deterministic(deterministic)
    st.enable_scenes(scene_blocks)
    slots = [st.add_scene(sc.particles, sc.colliders, sc.tri_vertices if sc.tri_vertices.size else None)
             for sc in scenes_]
    return st, slots


def batched_collider_offsets(scenes_, slots) -> list:
    """Index of each scene's first collider in a batched state's collider table
    (the live scenes' colliders in scene-slot order), for kinematic driving."""
    off, acc = {}, 0
    for i in sorted(range(len(slots)), key=lambda k: slots[k]):
        off[i] = acc
        acc += len(scenes_[i].colliders)
    return [off[i] for i in range(len(scenes_))]


def drive_kinematics(state: MpmState, scenes_, offsets, t: float):
    """Writes every kinematic body's velocity at time t (one stream-ordered call)."""
    from .scenes import kinematic_velocities
    total = max([o + len(sc.colliders) for o, sc in zip(offsets, scenes_)] + [0])
    vel = np.zeros((total, 6), np.float32)
    for o, sc in zip(offsets, scenes_):
        idx, v = kinematic_velocities(sc, t)
        vel[o + idx] = v
    if total:
        state.set_collider_velocities(0, vel)

