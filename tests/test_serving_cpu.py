"""Scheduler logic of the serving loop, on the CPU with a fake engine backend."""
import numpy as np

from spectral_analyzer_b200.rooms import Room
from spectral_analyzer_b200.serving import (BatchServer, Request, SequentialServer, mixed_room_requests,
                                            poisson_arrivals, room_bytes, summarize)


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeSolver:
    def __init__(self, room):
        self.room = room
        self.step = 0


class FakeBatch:
    """Advances every member `chunk` steps per call, capped at its limit; each
    batched step costs `cost` seconds of the fake clock."""

    def __init__(self, clock, cost=1e-4):
        self.clock, self.cost = clock, cost
        self.members, self.limits = [], []
        self.sets = []

    def set_segment(self, planes):
        pass

    def set_tile(self, tile_k):
        pass

    def set(self, solvers, limits):
        self.members, self.limits = list(solvers), list(limits)
        self.sets.append(len(solvers))

    def step(self, n, use_graph=True):
        for m, lim in zip(self.members, self.limits):
            m.step = min(lim, m.step + n)
        self.clock.t += self.cost * n

    def sync(self):
        return (np.array([m.step for m in self.members], np.int32),
                np.zeros(len(self.members), np.int32))


class FakeBackend:
    def __init__(self, clock, budget=1 << 40):
        self.clock, self.budget = clock, budget
        self.made = []
        self.peak = 0
        self.live = 0
        self.live_bytes = 0
        self.peak_bytes = 0

    def free_memory(self):
        return self.budget

    def make(self, room):
        self.made.append(room)
        self.live += 1
        self.peak = max(self.peak, self.live)
        self.live_bytes += room_bytes(room)
        self.peak_bytes = max(self.peak_bytes, self.live_bytes)
        return FakeSolver(room)

    def batch(self):
        return FakeBatch(self.clock)

    def run_plain(self, solver, n):
        solver.step = n
        self.clock.t += 1e-4 * n

    def traces(self, solver):
        return np.arange(solver.step, dtype=np.float32)[:, None]

    def release(self, solver):
        self.live -= 1
        self.live_bytes -= room_bytes(solver.room)


def small_requests(n=12, seed=1):
    reqs = mixed_room_requests(n, seed=seed, steps=(50, 400), axes=(32, 48, 64))
    for r, t in zip(reqs, poisson_arrivals(n, rate=200.0, seed=seed)):
        r.arrival = float(t)
    return reqs


def test_mixed_room_generator_shapes():
    reqs = mixed_room_requests(256, seed=3)
    assert len(reqs) == 256
    for r in reqs:
        rm = r.room
        assert {rm.nx, rm.ny, rm.nz} <= set(range(32, 257, 16))
        assert 500 <= rm.n_steps <= 8000 and 1 <= len(rm.receivers) <= 4
        assert all(0.02 <= a <= 0.3 for a in rm.absorption)
        for p in [rm.src] + rm.receivers:
            assert all(0 <= c < d for c, d in zip(p, (rm.nx, rm.ny, rm.nz)))
    assert {r.room.source_kind for r in reqs} == {"gaussian", "ricker"}
    # seeded: the same list again
    again = mixed_room_requests(256, seed=3)
    assert [r.room.describe() for r in reqs] == [r.room.describe() for r in again]


def test_batch_server_completes_every_request_in_order_of_need():
    clock = FakeClock()
    be = FakeBackend(clock)
    reqs = small_requests()
    srv = BatchServer(max_slots=4, chunk=16, backend=be, clock=clock, sleep=clock.sleep)
    res = srv.run(reqs)
    assert [r.rid for r in res] == sorted(r.rid for r in reqs)
    for r, q in zip(res, sorted(reqs, key=lambda q: q.rid)):
        assert r.traces.shape[0] == q.room.n_steps           # every step was recorded
        assert r.finish >= r.start >= r.arrival - 1e-12
    assert be.peak <= 4                                      # slot limit held
    # continuous batching: some request joined while another was running
    assert max(e["active"] for e in srv.log) > 1


def test_batch_server_respects_memory_budget():
    clock = FakeClock()
    reqs = small_requests()
    one = max(room_bytes(r.room) for r in reqs)
    be = FakeBackend(clock, budget=2 * one)
    srv = BatchServer(max_slots=16, chunk=16, backend=be, clock=clock, sleep=clock.sleep)
    srv.run(reqs)
    assert be.peak_bytes <= 2 * one
    assert be.peak >= 2


def test_sequential_server_and_summary():
    clock = FakeClock()
    be = FakeBackend(clock)
    reqs = small_requests()
    res = SequentialServer(backend=be, clock=clock, sleep=clock.sleep).run(reqs)
    s = summarize(res, work=1.0)
    assert s["requests"] == len(reqs)
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0
    starts = sorted(r.start for r in res)
    finishes = sorted(r.finish for r in res)
    assert all(b >= a for a, b in zip(finishes[:-1], starts[1:]))   # one at a time
