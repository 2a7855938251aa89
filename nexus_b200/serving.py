"""Serving form: continuous batching of independent MPM scenes on one GPU.

Requests (a scene and a step budget) arrive over time.  A request is
admitted as soon as it has arrived and its estimated HBM footprint fits the
budget beside the scenes already running.  Every admitted scene then
advances in the same batched state as all the others of its cell width, dt
and gravity: one launch sequence per step for all of them (nxm_step on a
state with batched scenes).  When a scene has taken its step budget, its
particles are read back; finished scenes leave the state in batches (a
removal compacts the whole particle storage), sooner when an arrival needs
their room.  Scenes that arrive while others run start on the next step.

The host never drains the GPU: a finished scene's positions are read
asynchronously into pinned memory (queued behind the steps in flight), as is
the removal of a batch of finished scenes, and a result is collected when its
read's ticket completes; each batched state keeps at most a few steps queued
ahead.

Each scene steps exactly as it would alone (scene-local coordinates, its own
block-key region and colliders), so a result does not depend on what else was
in the mix or on when it was admitted.

Failures: the device status word of each batched state (grid blocks or hash
slots exhausted, a particle without a block) is sticky until cleared.  It is
polled without waiting (nxm_state_status_poll: a word posted after some
earlier step, once its store has run), and it is also read right after every
result read (nxm_state_read_status_async), so that a result is only handed
out when no step before it reported a bit.  When a state reports one, every
scene that may have taken part in the failing step (those active on the state
and those whose final read is still in flight) is evicted and reported in
``MpmServer.failed`` with the status bits (finished scenes still in the state
leave with them; their results were handed out before); the bits are cleared, the state's
grid admission estimate is doubled so that the same mix is not admitted
again, and serving continues with the other requests.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .mpm import MpmPipeline, MpmState, PinnedArray
from .scenes import Scene

# Estimated device bytes per particle of a batched state: two copies of the
# 144-byte particle record, sort scratch (block key 8, header 4, sorted ids
# reserved 32), ids 8, scene index 4.
BYTES_PER_PARTICLE = 2 * 144 + 8 + 4 + 32 + 8 + 4
# Per grid block: 64 nodes of 16 bytes, header arrays, hash slots.
BYTES_PER_BLOCK = 64 * 16 + 16 + 4 * 3 + 4 * 10 + 4 * 7 + 4 + 2 * 8


@dataclass
class Request:
    rid: int
    scene: Scene
    steps: int
    arrival: float  # seconds after the start of the run


@dataclass
class Failure:
    rid: int
    status: int  # NXM_STATUS_* bits the state reported
    steps_done: int  # steps the scene had taken when it was evicted (its budget if it had finished)


@dataclass
class Result:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    completed: float
    positions: np.ndarray = field(repr=False)

    @property
    def latency(self) -> float:
        return self.completed - self.arrival


def footprint(scene: Scene) -> int:
    """Estimated device bytes of a scene inside a batched state."""
    return scene.n * BYTES_PER_PARTICLE + scene.grid_capacity * BYTES_PER_BLOCK


class _Group:
    """One batched state: the scenes sharing a cell width, dt and gravity."""

    def __init__(self, key, particles_capacity: int, grid_capacity: int, scene_blocks: int, deterministic: bool):
        dx, dt, gravity = key
        self.state = MpmState(grid_size=grid_capacity, particles_capacity=particles_capacity)
        self.state.set_cell_width(dx, grid_capacity)
        self.state.set_simulation_params(gravity, dt)
        self.state.set_deterministic(deterministic)
        self.state.enable_scenes(scene_blocks)
        self.active = {}  # slot -> [request, remaining steps, admitted time]
        self.retired = []  # (slot, request): finished, read queued, awaiting removal with others
        self.particles = 0
        self.grid = 0
        self.grid_factor = 1.0  # admission estimate of a scene's grid blocks, doubled after an overflow
        self.steps = deque()  # tickets of the steps queued on this state


class MpmServer:
    """Request loop over batched states (one per cell width / dt / gravity)."""

    def __init__(self, hbm_budget: float = 150e9, particles_capacity: int = 1 << 24,
                 grid_capacity: int = 1 << 20, deterministic: bool = False, scene_blocks=None,
                 retire_fraction: float = 0.02):
        self.pipe = MpmPipeline()
        self.budget = hbm_budget
        self.particles_capacity = particles_capacity
        self.grid_capacity = grid_capacity
        self.deterministic = deterministic
        self.scene_blocks = scene_blocks  # None: 64 blocks per scene axis at dx >= 1/128, else 128
        # Finished scenes leave their state in batches: a removal compacts the
        # state's whole particle storage, whatever it removes, while a finished
        # scene left in place only steps along (its result was read at its last
        # step).  They leave once they hold this fraction of the state's
        # particles, when their room lets the next arrival in, or when the
        # state has nothing else to run.
        self.retire_fraction = float(retire_fraction)
        self.groups = {}
        self.failed = {}  # request id -> Failure
        self.in_use = 0
        self.steps_taken = 0
        self.particle_steps = 0
        self._pinned = {}  # capacity (particles) -> free pinned result buffers
        self._words = None  # pinned status words, one per result read in flight
        self._free_words = []

    def _buffer(self, n: int) -> PinnedArray:
        cap = 1 << max(int(n) - 1, 0).bit_length()
        free = self._pinned.get(cap)
        return free.pop() if free else PinnedArray((cap, 3))

    def _release(self, buf: PinnedArray):
        self._pinned.setdefault(buf.array.shape[0], []).append(buf)

    def _word(self) -> int:
        if not self._free_words:
            old = self._words
            n = 2 * (len(old.array) if old is not None else 1024)
            self._words = PinnedArray((n,), np.uint32)
            self._free_words = list(range(len(old.array) if old is not None else 0, n))
            self._retired_words = getattr(self, "_retired_words", []) + ([old] if old is not None else [])
        return self._free_words.pop()
    def _group(self, sc: Scene) -> _Group:
        key = (float(sc.dx), float(sc.dt), tuple(float(g) for g in sc.gravity))
        g = self.groups.get(key)
        if g is None:
            sb = self.scene_blocks or (64 if sc.dx >= 1.0 / 128.0 else 128)
            g = self.groups[key] = _Group(key, self.particles_capacity, self.grid_capacity, sb, self.deterministic)
        return g

    def prepare(self, scenes_):
        """Creates the batched states the given scenes would use (device
        allocation happens here rather than at a request's admission)."""
        for sc in scenes_:
            self._group(sc)

    def _fits(self, sc: Scene, g: _Group, without_retired: bool = False) -> bool:
        in_use, particles, grid = self.in_use, g.particles, g.grid
        if without_retired:  # as it would be once the finished scenes left
            in_use -= sum(footprint(r.scene) for _, r in g.retired)
            particles -= sum(r.scene.n for _, r in g.retired)
            grid -= sum(r.scene.grid_capacity * g.grid_factor for _, r in g.retired)
        return (in_use + footprint(sc) <= self.budget and particles + sc.n <= self.particles_capacity
                and grid + sc.grid_capacity * g.grid_factor <= self.grid_capacity)

    def _usage(self, g: _Group):
        live = [rec[0] for rec in g.active.values()] + [r for _, r in g.retired]
        g.particles = sum(r.scene.n for r in live)
        g.grid = sum(r.scene.grid_capacity * g.grid_factor for r in live)
        self.in_use = sum(footprint(rec[0].scene) for gg in self.groups.values() for rec in gg.active.values())
        self.in_use += sum(footprint(r.scene) for gg in self.groups.values() for _, r in gg.retired)

    def _remove_retired(self, g: _Group):
        """Removes the finished scenes still in `g` (queued behind their reads)."""
        if g.retired:
            g.state.remove_scenes([slot for slot, _ in g.retired])
            g.retired.clear()
            self._usage(g)

    def _fail(self, g: _Group, bits: int, reads: deque):
        """Evicts every scene of `g` that may have taken part in the failing
        step (see the module docstring) and reports it in self.failed."""
        for slot, (r, left, _) in g.active.items():
            self.failed[r.rid] = Failure(r.rid, bits, r.steps - left)
        slots = list(g.active) + [slot for slot, _ in g.retired]  # finished ones leave too
        if slots:
            g.state.remove_scenes(slots)
        g.active.clear()
        g.retired.clear()
        keep = deque()
        for item in reads:
            if item[0] is g:
                self.failed[item[2].rid] = Failure(item[2].rid, bits, item[2].steps)
                self._release(item[4])
                self._free_words.append(item[5])
            else:
                keep.append(item)
        reads.clear()
        reads.extend(keep)
        g.state.status(clear=True)  # waits for the stream: any earlier post has run
        g.state.status_poll()  # that post's word predates the clear: dropped
        g.grid_factor *= 2.0
        self._usage(g)

    def run(self, requests, clock=time.perf_counter, idle_sleep: float = 1e-4, depth: int = 32):
        """Serves ``requests`` (any order; by arrival) and returns the results by
        request id, plus requests that can never fit (rejected); requests
        evicted after a device status error are in ``self.failed``.
        ``depth``: steps each batched state may have queued ahead of the GPU."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        results, rejected = {}, []
        self.last_results = results
        reads = deque()  # (group, ticket, request, admitted time, pinned buffer), in issue order per state
        t0 = clock()
        while pending or reads or any(g.active for g in self.groups.values()):
            now = clock() - t0
            # admission, first come first served
            while pending and pending[0].arrival <= now:
                r = pending[0]
                g = self._group(r.scene)
                if (footprint(r.scene) > self.budget or r.scene.n > self.particles_capacity
                        or r.scene.grid_capacity * g.grid_factor > self.grid_capacity):
                    rejected.append(pending.pop(0))  # can never fit, even alone
                    continue
                if not self._fits(r.scene, g):
                    if not (g.retired and self._fits(r.scene, g, without_retired=True)):
                        break
                    self._remove_retired(g)  # the room held by finished scenes lets it in
                pending.pop(0)
                slot = g.state.add_scene(r.scene.particles, r.scene.colliders,
                                         r.scene.tri_vertices if r.scene.tri_vertices.size else None)
                g.active[slot] = [r, r.steps, clock() - t0]
                g.particles += r.scene.n
                g.grid += r.scene.grid_capacity * g.grid_factor
                self.in_use += footprint(r.scene)
            # results whose reads (and the status word read after them) have landed
            for _ in range(len(reads)):
                if not reads:
                    break
                g, ticket, r, admitted, buf, w = reads[0]
                reads.rotate(-1)
                if g.state.ticket_done(ticket):
                    reads.pop()
                    bits = int(self._words.array[w])
                    self._free_words.append(w)
                    if bits:  # a step before this read reported a status bit
                        self.failed[r.rid] = Failure(r.rid, bits, r.steps)
                        self._release(buf)
                        self._fail(g, bits, reads)
                        continue
                    results[r.rid] = Result(r.rid, r.scene.n, r.steps, r.arrival, admitted, clock() - t0,
                                            buf.array[:r.scene.n].copy())
                    self._release(buf)
            busy = [g for g in self.groups.values() if g.active]
            if not busy:
                if reads or pending:
                    wait = idle_sleep if reads else max(0.0, pending[0].arrival - (clock() - t0))
                    time.sleep(min(idle_sleep, wait))
                continue
            for g in busy:
                if len(g.steps) >= depth:  # keep at most `depth` steps queued on this state
                    g.state.ticket_wait(g.steps.popleft())
                self.pipe.step(g.state)
                g.steps.append(g.state.fence())
                self.steps_taken += 1
                self.particle_steps += g.particles
                bits = g.state.status_poll()  # an earlier point of this state's stream, or None
                if bits:
                    self._fail(g, bits, reads)
            busy = [g for g in busy if g.active]
            for g in busy:
                done = []
                for slot, rec in g.active.items():
                    rec[1] -= 1
                    if rec[1] == 0:
                        done.append(slot)
                for slot in done:
                    r, _, admitted = g.active.pop(slot)
                    buf = self._buffer(r.scene.n)
                    g.state.read_scene_positions_async(slot, buf.array[:r.scene.n])
                    w = self._word()
                    ticket = g.state.read_status_async(self._words.array[w:w + 1])
                    reads.append((g, ticket, r, admitted, buf, w))
                    g.retired.append((slot, r))
                if g.retired and (not g.active or sum(r.scene.n for _, r in g.retired)
                                  >= self.retire_fraction * g.particles):
                    self._remove_retired(g)  # queued behind the reads above
        for g in self.groups.values():
            self._remove_retired(g)
        return results, rejected


def poisson_requests(count: int, rate: float, seed: int, make_scene, steps_range) -> list:
    """``count`` requests with exponential inter-arrival times (mean 1/rate),
    scene i = make_scene(i), steps uniform in steps_range (inclusive)."""
    from .scenes import uniform
    u = uniform(seed, 2 * count)
    t, out = 0.0, []
    lo, hi = steps_range
    for i in range(count):
        t += -np.log(max(1.0 - u[2 * i], 1e-300)) / rate
        steps = lo + int(u[2 * i + 1] * (hi - lo + 1))
        out.append(Request(i, make_scene(i), min(steps, hi), t))
    return out


def latency_summary(results) -> dict:
    lat = np.array([r.latency for r in results.values()]) if results else np.zeros(0)
    return {"completed": int(lat.size), "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else None}


def shard_requests(requests, world: int, rank: int) -> list:
    """This rank's share of a request stream for serving on `world` GPUs: the
    longest-processing-time partition (nexus_b200.sharding) of the requests'
    particle-steps.  Scenes are independent, so ranks exchange nothing on the
    data path; every rank computes the same partition from the same stream."""
    from .sharding import shard_scenes
    work = [r.scene.n * r.steps for r in requests]
    return [requests[i] for i in shard_scenes(work, world)[rank]]


def serve_sharded(server: "MpmServer", requests, world: int, rank: int, **run_kw):
    """Runs this rank's shard of `requests` on `server`; returns (results,
    rejected, failed) of the whole job, gathered on every rank (each result
    without its positions, which stay on the rank that computed them)."""
    mine = shard_requests(requests, world, rank) if world > 1 else list(requests)
    results, rejected = server.run(mine, **run_kw)
    if world == 1:
        return results, rejected, dict(server.failed)
    import torch.distributed as dist
    light = {rid: Result(r.rid, r.n, r.steps, r.arrival, r.admitted, r.completed, np.zeros((0, 3), np.float32))
             for rid, r in results.items()}
    parts = [None] * world
    dist.all_gather_object(parts, (light, [r.rid for r in rejected], dict(server.failed)))
    all_results, all_rejected, all_failed = {}, [], {}
    for res, rej, fail in parts:
        all_results.update(res)
        all_rejected.extend(rej)
        all_failed.update(fail)
    return all_results, all_rejected, all_failed
