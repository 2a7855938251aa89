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

The batched form is measured beside it (``batched`` in the JSON line): the
256-scene mix (4k-128k particles per
scene, neo-Hookean or sand, dx = 1/128) advanced in one state, one launch
sequence per step for all scenes, against the same scenes stepped one by one
(each alone in its own state), the plain per-scene loop.  With ``--gpus N``
the scenes are sharded over the ranks (no collective on the data path).
"""
from __future__ import annotations

import argparse
import gc
import hashlib
import json
import os
import re
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
# Per phase (the roofline of each kernel group of one step), bytes per particle:
#   sort: the 4-byte block key read and the 4-byte sorted index written;
#   p2g:  x, mass, v, C read (12 + 4 + 12 + 36);
#   grid: node momentum + mass read and velocity + mass written, 32 bytes a
#         node, at the scene's nodes per particle (counted from the grid);
#   g2p:  x, v, F, V0, material read, x, v, C, F written (+ 24 for the
#         Drucker-Prager state words of sand).
PHASE_BYTES = {"sort": 8.0, "p2g": 64.0}
G2P_BYTES_ELASTIC = 24 + 36 + 8 + 96
G2P_BYTES_SAND = G2P_BYTES_ELASTIC + 24

# The DRAM traffic of one step (dram__bytes_read.sum + dram__bytes_write.sum
# over every kernel of the step) comes from an ncu capture summarised in a
# profiles/ file, which records the hash of the kernel sources it was taken
# on; the bench reports it only while the sources are unchanged.
TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "step_traffic_sand_water_2M.md")
KERNEL_SOURCES = os.path.join(ROOT, "nexus_b200", "csrc")


def b_alg_per_particle(model_tags: np.ndarray) -> float:
    sand = np.isin(model_tags, (2, 3))
    return float(np.where(sand, B_ALG_SAND, B_ALG_ELASTIC).mean())


def kernel_sources_hash() -> str:
    """sha256 (first 16 hex digits) of the CUDA library's sources."""
    h = hashlib.sha256()
    for name in sorted(os.listdir(KERNEL_SOURCES)):
        path = os.path.join(KERNEL_SOURCES, name)
        if os.path.isfile(path) and name.endswith((".cu", ".cuh", ".h")):
            h.update(name.encode())
            with open(path, "rb") as f:
                h.update(f.read())
    return h.hexdigest()[:16]


def load_traffic(workload: str):
    """(bytes per step or None, details): the captured traffic of this build's
    step, None when the capture predates the current kernel sources."""
    current = kernel_sources_hash()
    info = {"sources": current, "profile": os.path.basename(TRAFFIC_PROFILE)}
    if workload != "sand_water" or not os.path.exists(TRAFFIC_PROFILE):
        info["note"] = "no capture for this workload"
        return None, info
    text = open(TRAFFIC_PROFILE).read()
    m = re.search(r"traffic_bytes_per_step:\s*([0-9.eE+]+)\s+sources:\s*([0-9a-f]{16})", text)
    if not m:
        info["note"] = "no traffic line in the profile"
        return None, info
    captured, src = float(m.group(1)), m.group(2)
    info["captured_sources"] = src
    if src != current:
        info["stale"] = True
        info["last_capture_bytes"] = captured
        return None, info
    info["stale"] = False
    return captured, info


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


def make_scene(workload: str, seed_offset: int = 0, scale: float = 1.0):
    from nexus_b200 import scenes
    if workload == "sand_water":
        return scenes.sand_water(scale=scale, seed=2 + seed_offset)
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
    from nexus_b200.sharding import all_max as amax
    return amax(x, world)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_oracle_rate(scene, steps: int, warmup: int):
    """Particle-steps/s of the FP32 oracle (OpenMP, all host cores), and the
    oracle after its warmup + steps steps."""
    from oracle.oracle import OracleScene
    o = OracleScene(scene, "f32", native=True)
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return scene.n * steps / dt, dt, o


def oracle_build(o) -> str:
    """Which oracle library an OracleScene runs: the host-native build or the portable one."""
    return "-march=native on this host" if "_build_native_" in o.L.oracle_path else "portable -march=x86-64-v3"


def measure_accuracy(scene, o32, steps: int) -> dict:
    """The GPU path's x, v, C and F after `steps` steps of the scene from its
    start, in fast and in deterministic mode, against the FP32 oracle of the
    cpu_baseline leg (which ran the same steps) and an FP64 rerun: per field,
    the relative L2 of the error over the oracle's own change from the start
    (change_rel_l2 of tests/parity.py; a result that never moved scores 1)."""
    from oracle.oracle import OracleScene
    from nexus_b200.mpm import MpmPipeline, state_from_scene
    from tests.parity import start_state, state_errors
    start = start_state(scene)
    o64 = OracleScene(scene, "f64")
    o64.step(steps)
    w64 = o64.particles()
    w64["pos"] = o64.positions_f64()
    w32 = o32.particles()
    out = {"steps": steps, "metric": "||got - want|| / ||want - start|| per field (x, v, C, F)",
           "oracle_f32_vs_f64": state_errors(w32, w64, start)}
    pipe = MpmPipeline()
    for det in (False, True):
        st = state_from_scene(scene, deterministic=det)
        for _ in range(steps):
            pipe.step(st)
        st.synchronize()
        got = st.read_particles()
        out["deterministic" if det else "fast"] = {"vs_f32": state_errors(got, w32, start),
                                                   "vs_f64": state_errors(got, w64, start)}
        del st
    return out


def workload_config(scene, world: int) -> dict:
    """The `config` of both arms' lines (the same dict, so that they compare)."""
    return {"workload": scene.name, "particles_per_gpu": scene.n, "dx": scene.dx, "dt": scene.dt,
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "inputs larger than L2 (particle state %.0f MB per GPU)" % (scene.n * 144 / 1e6)}


# The reference arm times whole oracle steps of the full scene; it runs at
# most this many seconds of steps (about half a second each on 16 cores for
# the 2 M-particle scene), fewer than K when K would take longer.
REFERENCE_BUDGET_S = 150.0


def run_reference(args, world, rank):
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    from oracle.oracle import OracleScene
    scene = make_scene(args.workload, scale=args.scale)
    cores = int(os.environ["OMP_NUM_THREADS"])
    o = OracleScene(scene, "f32", native=True)
    warm = min(args.warmup, 2)
    t0 = time.perf_counter()
    if warm:
        o.step(warm)
    per_step = (time.perf_counter() - t0) / warm if warm else None
    steps = args.steps
    if per_step:
        steps = max(1, min(steps, int(REFERENCE_BUDGET_S / per_step)))
    t0 = time.perf_counter()
    o.step(steps)
    secs = time.perf_counter() - t0
    rate = scene.n * steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": secs / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(scene, args.gpus),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{steps} full steps of the {scene.n}-particle scene after {warm} warm-up "
                                   f"steps (of --steps {args.steps} / --warmup {args.warmup}: at most "
                                   f"{REFERENCE_BUDGET_S:.0f} s of steps; C restatement of the reference step, "
                                   f"FP32, OpenMP, {oracle_build(o)})"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own GPU (wgpu) and CPU (Rust) paths cannot run on this box: no Rust toolchain, "
                "no graphics stack",
    }
    print(json.dumps(line), flush=True)


def phase_rooflines(phases: dict, scene, st, peak: float) -> dict:
    """Achieved GB/s and fraction of the measured peak of each phase of one
    timestamped step, from the algorithmic bytes of that phase."""
    n = scene.n
    tags = scene.particles.model[:, 0]
    sand = np.isin(tags, (2, 3))
    nodes = st.num_blocks() * 64
    bytes_ = {"sort": PHASE_BYTES["sort"] * n, "p2g": PHASE_BYTES["p2g"] * n, "grid_update": 32.0 * nodes,
              "g2p": float(np.where(sand, G2P_BYTES_SAND, G2P_BYTES_ELASTIC).sum())}
    out = {}
    for k, b in bytes_.items():
        ms = phases.get(f"{k}_ms")
        if not ms:
            continue
        gbs = b / (ms / 1e3) / 1e9
        out[k] = {"ms": ms, "algorithmic_bytes": b, "achieved_gbs": gbs, "frac": gbs / peak}
    return out


def measure_cube(torch, steps: int = 100):
    """The 32,768-particle elastic cube, 100 steps, one graph per step."""
    from nexus_b200 import scenes
    from nexus_b200.mpm import MpmPipeline, state_from_scene
    sc = scenes.elastic_cube()
    st = state_from_scene(sc)
    pipe = MpmPipeline()
    stream = torch.cuda.ExternalStream(st.cuda_stream())
    for _ in range(5):
        pipe.step(st)
    st.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        pipe.step(st)
    b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b)
    st.synchronize()
    return {"workload": "elastic_cube", "particles": sc.n, "steps": steps, "value": sc.n * steps / (ms / 1e3),
            "unit": UNIT, "ms_per_step": ms / steps, "dx": sc.dx, "dt": sc.dt}


def run_ours(args, world, rank, local):
    import torch
    from nexus_b200 import build as nb
    from nexus_b200.mpm import MpmPipeline, MpmState, state_from_scene, load, tuning_table

    nb.build()
    load()
    torch.cuda.set_device(local)
    scene = make_scene(args.workload, seed_offset=rank, scale=args.scale)
    n = scene.n
    pipe = MpmPipeline()
    st = state_from_scene(scene)
    stream = torch.cuda.ExternalStream(st.cuda_stream())

    for _ in range(args.warmup):
        pipe.step(st)
    st.synchronize()
    # launch shapes picked by the autotuner on this state's own steps (the
    # state advances through the trials), then the timed steps
    tuning = st.autotune(trial_steps=args.tune_steps) if args.tune_steps > 0 else st.tuning()
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

    # per-phase breakdown: medians over five extra (untimed) timestamped steps
    ph = [pipe.step(st, timestamps=True) for _ in range(5)]
    phases = {k: float(np.median([p[k] for p in ph])) for k in ph[0]}
    st.synchronize()

    # roofline of one step (the captured graph): algorithmic bytes / step time
    tags = scene.particles.model[:, 0]
    bytes_per_step = b_alg_per_particle(tags) * n
    step_s = ms / args.steps / 1e3
    peak, peak_kind = load_peaks()
    achieved = bytes_per_step / step_s / 1e9
    traffic, traffic_info = load_traffic(args.workload if args.scale == 1.0 else "scaled")
    phase_roof = phase_rooflines(phases, scene, st, peak)

    # end to end through the C ABI from pinned host buffers (every rank its own
    # replica; the whole job's rate over the slowest rank's wall time), after
    # the device state above is released and one untimed pass of the same calls
    del st
    gc.collect()
    if args.e2e:
        measure_e2e(scene, args, torch, steps=3)
    e2e = measure_e2e(scene, args, torch) if args.e2e else None
    e2e_pageable = measure_e2e(scene, args, torch, pinned=False) if (args.e2e and world == 1) else None
    if e2e is not None and world > 1:
        wall = all_max(n * e2e["steps"] / e2e["value"], world)
        e2e["value"] = n * world * e2e["steps"] / wall
        e2e["h2d_bytes_per_step"] *= world
        e2e["d2h_bytes_per_step"] *= world
    batched = measure_batched(args, world, rank, torch) if args.batched_steps > 0 else None
    serving = measure_serving(args, torch, world, rank) if args.serving_requests > 0 else None
    coupled = measure_coupled(args, torch) if (args.coupled_steps > 0 and world == 1) else None
    coupled_cpic = measure_coupled(args, torch, cpic=True) if (args.coupled_steps > 0 and world == 1) else None
    cube = measure_cube(torch) if (args.cube and world == 1) else None

    if rank != 0:
        return
    cpu = accuracy = None
    if world == 1 and args.cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
        rate, secs, o32 = cpu_oracle_rate(scene, args.ref_steps, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
               "sample": f"{args.ref_steps} full steps of the same {n}-particle scene after 1 warm-up step "
                         f"({secs:.1f} s; C restatement of the reference step, FP32, OpenMP, {oracle_build(o32)})"}
        # the oracle as the checker: the same steps on the GPU against it
        accuracy = measure_accuracy(scene, o32, args.ref_steps + 1)
        del o32
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(scene, world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_info, "peak_kind": peak_kind,
                     "launch": "one step = one CUDA-graph launch of all step kernels",
                     "algorithmic_bytes_per_launch": bytes_per_step},
        "phases_ms": phases,
        "phase_roofline": phase_roof,
        "tuning": tuning,
        "clocks": clk,
        "e2e": e2e,
        "e2e_pageable": e2e_pageable,
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "accuracy": accuracy,
        "elastic_cube": cube,
        "batched": batched,
        "serving": serving,
        "coupled": coupled,
        "coupled_cpic": coupled_cpic,
        "tuning_table": tuning_table(),
    }
    print(json.dumps(line), flush=True)


def measure_batched(args, world, rank, torch):
    """The batched mix on this rank's shard: one state, timed steps, then the
    same scenes stepped one by one (plain loop) for the comparison."""
    from nexus_b200 import scenes as S
    from nexus_b200.mpm import MpmPipeline, batched_state_from_scenes, state_from_scene
    from nexus_b200.sharding import shard_scenes, all_sum
    mix = S.batched_mix(count=args.batched_scenes)
    mine = [mix[i] for i in shard_scenes([sc.n for sc in mix], world)[rank]]
    n = sum(sc.n for sc in mine)
    pipe = MpmPipeline()
    st, _ = batched_state_from_scenes(mine)
    stream = torch.cuda.ExternalStream(st.cuda_stream())
    for _ in range(max(3, args.warmup)):
        pipe.step(st)
    st.synchronize()
    tuning = st.autotune(trial_steps=args.tune_steps) if args.tune_steps > 0 else st.tuning()
    for _ in range(3):
        pipe.step(st)
    st.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.batched_steps):
        pipe.step(st)
    ev1.record(stream)
    ev1.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    st.synchronize()
    del st
    max_ms = all_max(ms, world)
    total = all_sum(float(n), world)
    value = total * args.batched_steps / (max_ms / 1e3)
    # plain loop: each scene alone, its own graph, one after the other
    plain_ms = 0.0
    for sc in mine:
        one = state_from_scene(sc)
        s1 = torch.cuda.ExternalStream(one.cuda_stream())
        for _ in range(3):
            pipe.step(one)
        one.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s1)
        for _ in range(args.plain_steps):
            pipe.step(one)
        b.record(s1)
        b.synchronize()
        plain_ms += a.elapsed_time(b) / args.plain_steps
        one.synchronize()
        del one
    plain_ms = all_max(plain_ms, world)
    plain = total / (plain_ms / 1e3)
    return {"workload": f"batched_mix_{len(mix)}", "scenes": len(mix), "particles": int(total),
            "value": value, "unit": UNIT, "steps": args.batched_steps, "ms_per_step": max_ms / args.batched_steps,
            "plain_scene_by_scene": {"value": plain, "unit": UNIT, "ms_per_step": plain_ms,
                                     "how": f"each scene alone in its own state and graph, {args.plain_steps} "
                                            f"timed steps after 3 warm-up, summed over scenes"},
            "speedup_vs_plain": value / plain, "dx": mix[0].dx, "dt": mix[0].dt, "tuning": tuning,
            "parallelism": f"scene-sharded{world}" if world > 1 else "single"}


def measure_coupled(args, torch, cpic: bool = False):
    """The coupled batched mix (64 sand scenes, each with eight
    kinematic bodies on seeded trajectories driven every step and a
    20,000-triangle height-field floor) in one state, against the same scenes
    stepped one by one with the same driving.  With `cpic`, every scene runs
    CPIC coupling (what a NexusState scene with colliders runs): node and
    particle distance fields, the floor meshes through their rigid particles,
    the compatible / incompatible P2G and G2P."""
    from nexus_b200 import scenes as S
    from nexus_b200.mpm import (MpmPipeline, batched_state_from_scenes, batched_collider_offsets,
                                drive_kinematics, state_from_scene)
    mix = S.coupled_mix(count=args.coupled_scenes)
    n = sum(sc.n for sc in mix)
    pipe = MpmPipeline()
    st, slots = batched_state_from_scenes(mix)
    if cpic:
        st.set_use_cpic(True)
    rigid = st.num_rigid_particles()
    offs = batched_collider_offsets(mix, slots)
    dt = mix[0].dt
    stream = torch.cuda.ExternalStream(st.cuda_stream())
    step = 0
    for _ in range(3):
        drive_kinematics(st, mix, offs, step * dt)
        pipe.step(st)
        step += 1
    st.synchronize()
    tuning = st.autotune(trial_steps=args.tune_steps) if args.tune_steps > 0 else st.tuning()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.coupled_steps):
        drive_kinematics(st, mix, offs, step * dt)
        pipe.step(st)
        step += 1
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    st.synchronize()
    del st
    plain_ms = 0.0
    for sc in mix:
        one = state_from_scene(sc, use_cpic=cpic)
        s1 = torch.cuda.ExternalStream(one.cuda_stream())
        for k in range(3):
            drive_kinematics(one, [sc], [0], k * dt)
            pipe.step(one)
        one.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s1)
        for k in range(args.plain_steps):
            drive_kinematics(one, [sc], [0], (3 + k) * dt)
            pipe.step(one)
        b.record(s1)
        b.synchronize()
        plain_ms += a.elapsed_time(b) / args.plain_steps
        one.synchronize()
        del one
    value = n * args.coupled_steps / (ms / 1e3)
    plain = n / (plain_ms / 1e3)
    return {"workload": f"coupled_mix_{len(mix)}" + ("_cpic" if cpic else ""), "scenes": len(mix), "particles": n,
            "coupling": "CPIC" if cpic else "one-way collider projection", "rigid_particles": rigid,
            "colliders_per_scene": int(len(mix[0].colliders)), "triangles_per_scene": int(len(mix[0].tri_vertices) // 3),
            "value": value, "unit": UNIT, "steps": args.coupled_steps, "ms_per_step": ms / args.coupled_steps,
            "plain_scene_by_scene": {"value": plain, "unit": UNIT, "ms_per_step": plain_ms},
            "speedup_vs_plain": value / plain, "dx": mix[0].dx, "dt": dt, "tuning": tuning,
            "how": "timed steps include writing every kinematic body's velocity (one stream-ordered call per step)"}


def measure_serving(args, torch, world: int = 1, rank: int = 0):
    """Continuous batching of a Poisson request stream (mean 200 scenes/s):
    aggregate particle-steps/s and p50/p99 arrival-to-completion latency,
    beside a FIFO loop that runs each request alone (plain step) in arrival
    order, whose latencies come from each scene's measured plain step time.
    With N ranks, each serves its LPT share of the same stream (no exchange on
    the data path); latencies are gathered and the rate is the whole stream's
    work over the slowest rank's wall time."""
    from nexus_b200 import scenes as S
    from nexus_b200.mpm import MpmPipeline, state_from_scene
    from nexus_b200.serving import MpmServer, poisson_requests, latency_summary, serve_sharded, shard_requests
    reqs = poisson_requests(args.serving_requests, 200.0, 3000, S.serving_scene, (50, 2000))
    mine = shard_requests(reqs, world, rank) if world > 1 else reqs
    srv = MpmServer(hbm_budget=150e9, particles_capacity=1 << 26, grid_capacity=1 << 22)
    srv.prepare([r.scene for r in mine])  # device states allocated before the first arrival
    barrier(world)
    t0 = time.perf_counter()
    results, rejected, failed = serve_sharded(srv, reqs, world, rank)
    wall = all_max(time.perf_counter() - t0, world)
    summ = latency_summary(results)
    del srv
    # FIFO plain loop: each request's plain step time (its scene alone in its
    # own state), then a virtual clock in arrival order.  The step time is
    # measured for every `every`-th request and interpolated by particle count
    # for the others, within their class (cell width, material).
    pipe = MpmPipeline()
    order = sorted(mine, key=lambda q: q.arrival)
    every = max(1, len(order) // args.fifo_samples)

    def klass(r):
        return (r.scene.dx, int(r.scene.particles.model[0, 0]))

    measured = {}
    for i, r in enumerate(order):
        if i % every:
            continue
        one = state_from_scene(r.scene)
        s1 = torch.cuda.ExternalStream(one.cuda_stream())
        for _ in range(3):
            pipe.step(one)
        one.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s1)
        for _ in range(args.plain_steps):
            pipe.step(one)
        b.record(s1)
        b.synchronize()
        measured[r.rid] = a.elapsed_time(b) / args.plain_steps / 1e3
        one.synchronize()
        del one
    samples = {}
    for r in order:
        if r.rid in measured:
            samples.setdefault(klass(r), []).append((r.scene.n, measured[r.rid]))
    t_done, lat = 0.0, []
    for r in order:
        if r.rid in measured:
            step_s = measured[r.rid]
        else:
            pts = sorted(samples.get(klass(r)) or [p for v in samples.values() for p in v])
            step_s = float(np.interp(r.scene.n, [p[0] for p in pts], [p[1] for p in pts]))
        t_done = max(t_done, r.arrival) + step_s * r.steps
        lat.append(t_done - r.arrival)
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, lat)
        lat = [x for p in parts for x in p]
    t_done = all_max(t_done, world)
    work = sum(r.scene.n * r.steps for r in reqs)
    return {"workload": "serving_poisson_200_per_s", "requests": len(reqs), "rejected": len(rejected),
            "failed": len(failed), "particles_per_request": "logU(2048, 524288)", "steps_per_request": "U{50..2000}",
            "value": work / wall, "unit": UNIT, "wall_s": wall, "p50_s": summ["p50_s"], "p99_s": summ["p99_s"],
            "parallelism": f"request-sharded{world}" if world > 1 else "single",
            "plain_fifo": {"value": work / t_done, "unit": UNIT, "p50_s": float(np.percentile(lat, 50)),
                           "p99_s": float(np.percentile(lat, 99)),
                           "how": "each request alone in its own state, in arrival order, for its step budget; "
                                  f"the plain step time measured (over {args.plain_steps} steps after 3 warm-up) "
                                  f"for every {every}-th request ({len(measured)} of {len(order)}), the others "
                                  "interpolated by particle count within their cell width and material"},
            "note": f"{len(reqs)} requests of the 4000-request stream (same arrival rate and distributions)"}


def measure_e2e(scene, args, torch, pinned: bool = True, steps: int = 0):
    """Same metric through the C ABI with host buffers: upload the scene from
    host memory (pinned buffers; or, `pinned` False, the plain numpy arrays an
    ordinary caller holds), then per step write the (kinematic) collider
    velocity, step, and read back the device status word; finally read the
    positions back.  Host wall clock around everything."""
    from nexus_b200.mpm import MpmPipeline, MpmState

    from nexus_b200.particles import ParticleBatch

    def pinned_like(a):
        if not pinned:
            return np.array(a, copy=True)
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
    steps = steps or args.e2e_steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = MpmState(grid_size=scene.grid_capacity, particles_capacity=p.n)
    st.set_cell_width(scene.dx, scene.grid_capacity)
    st.set_simulation_params(scene.gravity, scene.dt)
    st.set_colliders(scene.colliders)
    t1 = time.perf_counter()
    st.append(batch)
    t2 = time.perf_counter()
    for _ in range(steps):
        st.set_collider_velocity(0, zeros, zeros)
        pipe.step(st)
        st.status_pipelined()  # the previous step's status word; this step's is in flight
    st.status_pipelined()  # the last step's
    t3 = time.perf_counter()
    st.read_positions_into(out)
    st.synchronize()
    t4 = time.perf_counter()
    dt = t4 - t0
    # the SoA arrays copied to the device (the per-particle models stay on the
    # host: only their material runs travel)
    upload = sum(a.nbytes for k, a in batch.__dict__.items() if k != "model")
    return {"value": p.n * steps / dt, "unit": UNIT, "steps": steps,
            # per step: a 24-byte collider velocity write (kernel arguments), a 4-byte status word read
            "h2d_bytes_per_step": int(upload / steps + 24), "d2h_bytes_per_step": int(p.n * 12 / steps + 4),
            "how": "host wall clock: state create + SoA upload from %s (packed into records on the "
                   "device) + per step (collider velocity write, step, pipelined status D2H read one step late) + "
                   "final positions D2H; after one untimed 3-step pass of the same calls" %
                   ("pinned memory" if pinned else "pageable numpy arrays"),
            "phases_ms": {"create": (t1 - t0) * 1e3, "upload": (t2 - t1) * 1e3, "steps": (t3 - t2) * 1e3,
                          "readback": (t4 - t3) * 1e3}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sand_water", choices=["sand_water", "elastic_cube"])
    ap.add_argument("--scale", type=float, default=1.0,
                    help="sand_water only: fraction of its particles (smaller cases for profiling)")
    ap.add_argument("--ref-steps", type=int, default=10, help="oracle steps of the cpu_baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=500)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--batched-steps", type=int, default=200,
                    help="timed steps of the batched mix (0: skip it)")
    ap.add_argument("--batched-scenes", type=int, default=256)
    ap.add_argument("--plain-steps", type=int, default=10)
    ap.add_argument("--serving-requests", type=int, default=4000, help="0: skip the serving measurement")
    ap.add_argument("--fifo-samples", type=int, default=400,
                    help="requests whose plain step time the serving leg's FIFO baseline measures")
    ap.add_argument("--coupled-steps", type=int, default=300, help="timed steps of the coupled mix (0: skip it)")
    ap.add_argument("--coupled-scenes", type=int, default=64)
    ap.add_argument("--no-cube", dest="cube", action="store_false", help="skip the 32k elastic cube leg")
    ap.add_argument("--tune-steps", type=int, default=5,
                    help="timed steps per candidate of the autotuner before the timed region (0: default shapes)")
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
