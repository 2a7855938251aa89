"""Host logic of the serving loop (nexus_b200/serving.py) on the CPU, with a
fake batched state: asynchronous reads complete only after a few polls, and
the fake counts the steps queued ahead of its simulated GPU.  Every request
must come back stepped exactly its budget, from a read that had completed,
with at most `depth` steps queued on a state at any time."""
import numpy as np
import pytest

from nexus_b200 import serving
from nexus_b200.models import ParticleModel
from nexus_b200.particles import ParticleBatch, box_walls, collider_array
from nexus_b200.scenes import Scene


class FakeArray:
    def __init__(self, shape, dtype=np.float32):
        self.array = np.zeros(shape, dtype)

    def close(self):
        pass


class FakeState:
    """Scenes as position arrays; a step adds 1 to every live scene's
    positions once the simulated GPU runs it.  Tickets complete in order, a
    few polls after they were taken."""

    def __init__(self, grid_size, particles_capacity):
        self.scenes = {}
        self.queue = []  # work in stream order: ("step",), ("read", slot, out), ("rm", slots), ("fence", ticket)
        self.ticket = 0
        self.done = 0
        self.max_queued_steps = 0
        self.bits = 0  # sticky device status word
        self.posted = 0  # the word a pipelined read returns next (one call late)
        self.fail_over = None  # particles live at a step above which the step sets bit 2 (grid blocks)

    # -- setup calls of _Group
    def set_cell_width(self, dx, cap): pass
    def set_simulation_params(self, g, dt): pass
    def set_deterministic(self, d): pass
    def enable_scenes(self, sb): pass

    def _run_one(self):
        op = self.queue.pop(0)
        if op[0] == "step":
            if self.fail_over is not None and sum(len(p) for p in self.scenes.values()) > self.fail_over:
                self.bits |= 2
            for pos in self.scenes.values():
                pos += 1.0
        elif op[0] == "read":
            _, slot, out = op[:3]
            out[...] = self.scenes[slot]
        elif op[0] == "rm":
            for slot in op[1]:
                del self.scenes[slot]
        elif op[0] == "fence":
            self.done = op[1]
        elif op[0] == "status":
            op[1][0] = self.bits

    def _drain_to(self, ticket):
        while self.done < ticket:
            self._run_one()

    def add_scene(self, batch, colliders, tri):
        self._drain_to(self.ticket)  # admission sees the state as queued so far
        slot = next(i for i in range(10 ** 6) if i not in self.scenes)
        self.scenes[slot] = batch.pos.astype(np.float64).copy()
        return slot

    def remove_scenes(self, slots):
        self.queue.append(("rm", list(slots)))

    def read_scene_positions_async(self, slot, out):
        self.queue.append(("read", slot, out))
        return self.fence()

    def read_status_async(self, out):
        self.queue.append(("status", out))
        return self.fence()

    def fence(self):
        self.ticket += 1
        self.queue.append(("fence", self.ticket))
        steps = sum(1 for op in self.queue if op[0] == "step")
        self.max_queued_steps = max(self.max_queued_steps, steps)
        return self.ticket

    def ticket_done(self, t):
        if self.queue:  # the GPU makes some progress between polls
            self._run_one()
        return t <= self.done

    def ticket_wait(self, t):
        self._drain_to(t)

    def status_poll(self):
        out, self.posted = self.posted, self.bits
        return out

    def status(self, clear=False):
        self._drain_to(self.ticket)
        out = self.bits
        if clear:
            self.bits = 0
        return out


class FakePipeline:
    def step(self, st):
        st.queue.append(("step",))


def _scene(i, n):
    pos = np.full((n, 3), 0.25 + 0.01 * i, np.float32)
    b = ParticleBatch.from_positions(pos, np.float32(1 / 256), 1000.0, ParticleModel.water(1e5))
    return Scene(f"s{i}", 1 / 64, 1e-4, (0.0, 0.0, -9.81), b, collider_array(box_walls()), 10, 64)


@pytest.mark.parametrize("depth", [1, 4, 32])
def test_served_requests_step_their_budget(monkeypatch, depth):
    monkeypatch.setattr(serving, "MpmState", FakeState)
    monkeypatch.setattr(serving, "MpmPipeline", FakePipeline)
    monkeypatch.setattr(serving, "PinnedArray", FakeArray)
    rng = np.random.default_rng(depth)
    reqs = [serving.Request(i, _scene(i, int(rng.integers(1, 50))), int(rng.integers(1, 40)), 0.0)
            for i in range(12)]
    srv = serving.MpmServer(hbm_budget=1e12, particles_capacity=1 << 20, grid_capacity=1 << 12)
    results, rejected = srv.run(reqs, clock=iter(np.arange(0.0, 1e6, 1e-3)).__next__, idle_sleep=0.0, depth=depth)
    assert not rejected and sorted(results) == list(range(12))
    for r in reqs:
        got = results[r.rid].positions
        assert got.shape == (r.scene.n, 3)
        np.testing.assert_array_equal(got, r.scene.particles.pos + np.float32(r.steps))
    (g,) = srv.groups.values()
    assert g.state.max_queued_steps <= depth
    while g.state.queue:  # the last removals are queued behind the reads
        g.state._run_one()
    assert not g.state.scenes  # every finished scene was removed


@pytest.mark.parametrize("poll", [True, False])
def test_status_error_evicts_and_reports_the_scenes_of_the_failing_step(monkeypatch, poll):
    """A state whose step reports a status bit (here: more live particles than
    its grid holds) has every scene that may have taken part evicted and
    reported in `failed` with the bits; the bits are cleared, the state's grid
    estimate doubled, and the other requests are served as usual."""
    monkeypatch.setattr(serving, "MpmState", FakeState)
    monkeypatch.setattr(serving, "MpmPipeline", FakePipeline)
    monkeypatch.setattr(serving, "PinnedArray", FakeArray)
    if not poll:  # the poll never returns in time: the status word read after each result catches it
        monkeypatch.setattr(FakeState, "status_poll", lambda self: None)
    reqs = [serving.Request(i, _scene(i, 20), 30, 0.0) for i in range(3)]  # all three at once: 60 particles
    reqs += [serving.Request(3 + i, _scene(3 + i, 20), 10, 100.0) for i in range(3)]  # later, one at a time fits
    srv = serving.MpmServer(hbm_budget=1e12, particles_capacity=1 << 20, grid_capacity=192)
    states = []
    orig = srv._group

    def group(sc):
        g = orig(sc)
        if g.state not in states:
            g.state.fail_over = 50
            states.append(g.state)
        return g
    srv._group = group
    results, rejected = srv.run(reqs, clock=iter(np.arange(0.0, 1e6, 1e-2)).__next__, idle_sleep=0.0, depth=4)
    assert not rejected
    assert sorted(srv.failed) == [0, 1, 2]
    assert all(f.status & 2 and 0 < f.steps_done <= 30 for f in srv.failed.values())
    (g,) = srv.groups.values()
    assert g.grid_factor == 2.0 and g.state.bits == 0
    # the later requests: the doubled estimate admits at most two at once (2 x 64 x 2 > 192), so they fit
    assert sorted(results) == [3, 4, 5]
    for r in reqs[3:]:
        np.testing.assert_array_equal(results[r.rid].positions, r.scene.particles.pos + np.float32(r.steps))


def _serve_rank(rank, world, port, out):
    import datetime
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        serving.MpmState, serving.MpmPipeline, serving.PinnedArray = FakeState, FakePipeline, FakeArray
        rng = np.random.default_rng(5)
        reqs = [serving.Request(i, _scene(i, int(rng.integers(1, 40))), int(rng.integers(1, 30)), 0.01 * i)
                for i in range(20)]
        mine = serving.shard_requests(reqs, world, rank)
        srv = serving.MpmServer(hbm_budget=1e12, particles_capacity=1 << 20, grid_capacity=1 << 12)
        results, rejected, failed = serving.serve_sharded(
            srv, reqs, world, rank, clock=iter(np.arange(0.0, 1e6, 1e-3)).__next__, idle_sleep=0.0, depth=4)
        ok = all(np.array_equal(srv_r.positions, reqs[rid].scene.particles.pos + np.float32(reqs[rid].steps))
                 for rid, srv_r in srv_results(srv, mine, results).items())
        out.put((rank, [r.rid for r in mine], sorted(results), rejected, sorted(failed), ok,
                 sum(r.scene.n * r.steps for r in mine)))
    finally:
        dist.destroy_process_group()


def srv_results(srv, mine, gathered):
    """This rank's own results (with positions) among the gathered ones."""
    return {r.rid: srv.last_results[r.rid] for r in mine if r.rid in srv.last_results}


def test_two_gloo_ranks_serve_disjoint_shards_of_one_stream():
    """Serving on two ranks: each serves its LPT share of the same request
    stream (no exchange on the data path); the gathered results cover every
    request exactly once, each stepped its budget, and the shares balance."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_serve_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, mine0, all0, rej0, f0, ok0, w0), (_, mine1, all1, rej1, f1, ok1, w1) = res
    assert not set(mine0) & set(mine1) and sorted(mine0 + mine1) == list(range(20))
    assert all0 == all1 == list(range(20)) and not rej0 and not rej1 and not f0 and not f1
    assert ok0 and ok1
    assert abs(w0 - w1) <= max(w0, w1) // 2


@pytest.mark.parametrize("fraction", [0.0, 0.02, 1.0])
def test_finished_scenes_leave_in_batches(monkeypatch, fraction):
    """Finished scenes stay in their state (stepping along) until they hold
    `retire_fraction` of its particles, their room admits the next arrival,
    or nothing else runs: results stay exact, a tight particle capacity still
    admits every request, and every scene is gone at the end."""
    monkeypatch.setattr(serving, "MpmState", FakeState)
    monkeypatch.setattr(serving, "MpmPipeline", FakePipeline)
    monkeypatch.setattr(serving, "PinnedArray", FakeArray)
    rng = np.random.default_rng(5)
    reqs = [serving.Request(i, _scene(i, int(rng.integers(10, 40))), int(rng.integers(1, 30)), 0.0)
            for i in range(16)]
    srv = serving.MpmServer(hbm_budget=1e12, particles_capacity=100, grid_capacity=1 << 12,
                            retire_fraction=fraction)
    removals = []
    orig = FakeState.remove_scenes
    monkeypatch.setattr(FakeState, "remove_scenes", lambda self, slots: (removals.append(len(slots)),
                                                                          orig(self, slots))[1])
    results, rejected = srv.run(reqs, clock=iter(np.arange(0.0, 1e6, 1e-3)).__next__, idle_sleep=0.0, depth=4)
    assert not rejected and sorted(results) == list(range(16))
    for r in reqs:
        np.testing.assert_array_equal(results[r.rid].positions, r.scene.particles.pos + np.float32(r.steps))
    (g,) = srv.groups.values()
    while g.state.queue:
        g.state._run_one()
    assert not g.state.scenes and not g.retired
    assert sum(removals) == 16
    if fraction == 1.0:  # only admissions and the end let finished scenes go
        assert len(removals) < 16
