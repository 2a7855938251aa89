#!/usr/bin/env python
"""Throughput of the MLS-MPM step: particle-steps/s on one B200 per rank.

Workload (default ``sand_water``): the plain 3D single large scene, dx =
1/256, 1.5 M Drucker-Prager sand + 0.5 M weakly compressible water particles,
8 particles per cell, FP32 state, dt = 5e-5, sticky floor and slip walls
(seeded synthetic particles; nothing is read from disk).  A step is one full
MpmPipeline::step over all particles (sort, P2G, grid update with collider
projection, G2P + constitutive update), replayed as one CUDA graph.

Multi-GPU: a single scene does not shard, so ``--gpus N`` runs N independent
replicas (one per rank, seed + rank), weak scaling, no collective on the
data path; value = particle-steps of all ranks / max time over ranks.

``--impl reference`` times the reference algorithm's CPU restatement (the
oracle, OpenMP on all host cores) on the same scene; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "particle-steps/s on 1 B200 (plain single large scene)"
UNIT = "particle-steps/s"

# Algorithmic bytes per particle-step: each particle's persistent state read
# once and written once (x, v, C, F read and written; mass, V0, material id
# read; Drucker-Prager state, 3 floats, read and written for sand).
B_ALG_ELASTIC = 204
B_ALG_SAND = 228


def b_alg_per_particle(model_tags: np.ndarray) -> float:
    sand = np.isin(model_tags, (2, 3))
    return float(np.where(sand, B_ALG_SAND, B_ALG_ELASTIC).mean())


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, period_ms: int = 50):
        self.gpu = gpu_index
        self.period = period_ms
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 f"-lms={self.period}"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, which):
        if which == 0:
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(self.period / 1000.0 * 2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [l for (t, l) in self.lines if self.t0 is not None and self.t0 <= t <= (self.t1 or t)]
        if not rows:
            rows = [l for (_, l) in self.lines]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            f = [x.strip() for x in r.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene(workload: str, seed_offset: int = 0):
    from nexus_b200 import scenes
    if workload == "sand_water":
        return scenes.sand_water(seed=2 + seed_offset)
    if workload == "elastic_cube":
        return scenes.elastic_cube(seed=1 + seed_offset)
    raise SystemExit(f"unknown workload {workload}")


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def all_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_oracle_rate(scene, steps: int, warmup: int):
    """Particle-steps/s of the FP32 oracle (OpenMP, all host cores)."""
    from oracle.oracle import OracleScene
    o = OracleScene(scene, "f32")
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return scene.n * steps / dt, dt


def run_reference(args, world, rank):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    scene = make_scene(args.workload)
    cores = int(os.environ["OMP_NUM_THREADS"])
    rate, secs = cpu_oracle_rate(scene, args.ref_steps, args.ref_warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.ref_steps, "warmup": args.ref_warmup, "ms_per_step": secs / args.ref_steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles": scene.n, "dx": scene.dx, "dt": scene.dt},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.ref_steps} full steps of the {scene.n}-particle scene after "
                                   f"{args.ref_warmup} warm-up steps (C restatement of the reference step, "
                                   f"FP32, OpenMP)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own GPU (wgpu) and CPU (Rust) paths cannot run on this box: no Rust toolchain, "
                "no graphics stack",
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    from nexus_b200 import build as nb
    from nexus_b200.mpm import MpmPipeline, MpmState, state_from_scene, load

    nb.build()
    load()
    torch.cuda.set_device(local)
    scene = make_scene(args.workload, seed_offset=rank)
    n = scene.n
    pipe = MpmPipeline()
    st = state_from_scene(scene)
    stream = torch.cuda.ExternalStream(st.cuda_stream())

    for _ in range(args.warmup):
        pipe.step(st)
    st.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.2)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = st.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    clocks.mark(0)
    ev0.record(stream)
    for _ in range(args.steps):
        pipe.step(st)
    ev1.record(stream)
    ev1.synchronize()
    clocks.mark(1)
    torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    launches = st.kernel_launches() - launches0
    clk = clocks.stop()
    st.synchronize()  # raises on any device status error
    max_ms = all_max(ms, world)
    value = n * world * args.steps / (max_ms / 1e3)

    # per-phase breakdown on one extra (untimed) step
    phases = pipe.step(st, timestamps=True)
    st.synchronize()

    # roofline of one step (the captured graph): algorithmic bytes / step time
    tags = scene.particles.model[:, 0]
    bytes_per_step = b_alg_per_particle(tags) * n
    step_s = ms / args.steps / 1e3
    peak, peak_kind = load_peaks()
    achieved = bytes_per_step / step_s / 1e9

    # end to end through the C ABI from pinned host buffers
    e2e = measure_e2e(scene, args, torch) if args.e2e else None

    if rank != 0:
        return
    cpu = None
    if world == 1 and args.cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
        rate, secs = cpu_oracle_rate(scene, args.ref_steps, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
               "sample": f"{args.ref_steps} full steps of the same {n}-particle scene after 1 warm-up step "
                         f"({secs:.1f} s; C restatement of the reference step, FP32, OpenMP)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "particles_per_gpu": n, "dx": scene.dx, "dt": scene.dt,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": "inputs larger than L2 (particle state %.0f MB per GPU)" % (n * 144 / 1e6)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": args.traffic, "peak_kind": peak_kind,
                     "launch": "one step = one CUDA-graph launch of all step kernels",
                     "algorithmic_bytes_per_launch": bytes_per_step},
        "phases_ms": phases,
        "clocks": clk,
        "e2e": e2e,
        "gpu_launches": launches,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def measure_e2e(scene, args, torch):
    """Same metric through the C ABI with host buffers: upload the scene from
    pinned host memory, then per step write the (kinematic) collider
    velocity, step, and read back the device status word; finally read the
    positions back.  Host wall clock around everything."""
    from nexus_b200.mpm import MpmPipeline, MpmState

    from nexus_b200.particles import ParticleBatch

    def pinned_like(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype).reshape(a.shape)
        v[...] = a
        keep.append(t)
        return v

    keep = []
    p = scene.particles
    batch = ParticleBatch(**{k: pinned_like(getattr(p, k)) for k in ParticleBatch.__dataclass_fields__})
    out = pinned_like(np.zeros((p.n, 3), np.float32))
    zeros = np.zeros(3, np.float32)
    pipe = MpmPipeline()
    steps = args.e2e_steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = MpmState(grid_size=scene.grid_capacity, particles_capacity=p.n)
    st.set_cell_width(scene.dx, scene.grid_capacity)
    st.set_simulation_params(scene.gravity, scene.dt)
    st.set_colliders(scene.colliders)
    st.append(batch)
    for _ in range(steps):
        st.set_collider_velocity(0, zeros, zeros)
        pipe.step(st)
        st.status()
    st.read_positions_into(out)
    st.synchronize()
    dt = time.perf_counter() - t0
    upload = sum(a.nbytes for a in batch.__dict__.values())
    return {"value": p.n * steps / dt, "unit": UNIT, "steps": steps,
            "h2d_bytes_per_step": int(upload / steps + 32), "d2h_bytes_per_step": int(p.n * 12 / steps + 32),
            "how": "host wall clock: state create + SoA upload from pinned memory + per step (collider velocity "
                   "H2D, step, status D2H) + final positions D2H"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sand_water", choices=["sand_water", "elastic_cube"])
    ap.add_argument("--ref-steps", type=int, default=10)
    ap.add_argument("--ref-warmup", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=500)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per step from an ncu capture (see profiles/)")
    args = ap.parse_args()
    if args.impl == "reference":
        # CPU baseline arm: rank 0 alone runs it; other ranks exit without work.
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
