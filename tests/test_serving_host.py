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

    # -- setup calls of _Group
    def set_cell_width(self, dx, cap): pass
    def set_simulation_params(self, g, dt): pass
    def set_deterministic(self, d): pass
    def enable_scenes(self, sb): pass

    def _run_one(self):
        op = self.queue.pop(0)
        if op[0] == "step":
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
