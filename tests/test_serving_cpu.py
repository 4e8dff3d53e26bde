"""Scheduler logic of the serving loop, on the CPU with a fake engine backend."""
import numpy as np

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
    def __init__(self, room, diverge_at=None):
        self.room = room
        self.step = 0
        self.diverge_at = diverge_at      # a step whose pressure goes non-finite
        self.unstable = False


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
            if m.unstable:
                continue
            target = min(lim, m.step + n)
            if m.diverge_at is not None:
                check = (m.diverge_at // 256 + 1) * 256     # the first 256-step check after it
                if check <= target:
                    m.step, m.unstable = check, True
                    continue
            m.step = target
        self.clock.t += self.cost * n

    def sync(self):
        return (np.array([m.step for m in self.members], np.int32),
                np.array([-3 if m.unstable else 0 for m in self.members], np.int32))


class FakeBackend:
    def __init__(self, clock, budget=1 << 40, diverge=None, alloc_fail=()):
        self.clock, self.budget = clock, budget
        self.diverge = diverge or {}          # id(room) -> step that goes non-finite
        self.alloc_fail = {id(r) for r in alloc_fail}
        self.made = []
        self.peak = 0
        self.live = 0
        self.live_bytes = 0
        self.peak_bytes = 0

    def free_memory(self):
        return self.budget

    def make(self, room):
        if id(room) in self.alloc_fail:
            raise MemoryError("fake: out of device memory")
        self.made.append(room)
        self.live += 1
        self.peak = max(self.peak, self.live)
        self.live_bytes += room_bytes(room)
        self.peak_bytes = max(self.peak_bytes, self.live_bytes)
        return FakeSolver(room, self.diverge.get(id(room)))

    def batch(self):
        return FakeBatch(self.clock)

    def run_plain(self, solver, n):
        solver.step = n
        self.clock.t += 1e-4 * n

    def traces(self, solver):
        return np.arange(getattr(solver, "start", 0), solver.step, dtype=np.float32)[:, None]

    def snapshot(self, solver):
        return {"step": solver.step}

    def restore(self, solver, snap):
        solver.step = solver.start = snap["step"]

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


def test_unstable_request_leaves_alone():
    """A room whose pressure diverges stops at its check step and leaves with
    an error and the traces it recorded; every other room completes."""
    clock = FakeClock()
    reqs = mixed_room_requests(10, seed=2, steps=(600, 900), axes=(32, 48))
    bad = reqs[3]
    be = FakeBackend(clock, diverge={id(bad.room): 300})
    res = BatchServer(max_slots=4, chunk=64, backend=be, clock=clock, sleep=clock.sleep).run(reqs)
    assert [r.rid for r in res] == sorted(r.rid for r in reqs)
    for r in res:
        q = next(x for x in reqs if x.rid == r.rid)
        if q is bad:
            assert r.error is not None and "UNSTABLE" in r.error and "512" in r.error
            assert r.traces.shape[0] == 512
        else:
            assert r.ok and r.traces.shape[0] == q.room.n_steps
    assert be.live == 0                                   # every solver released
    s = summarize(res, work=1.0)
    assert s["requests"] == 9 and s["failed"] == 1


def test_sequential_server_isolates_a_diverging_request():
    clock = FakeClock()
    reqs = small_requests(6)

    class Diverging(FakeBackend):
        def run_plain(self, solver, n):
            if solver.room is reqs[2].room:
                raise RuntimeError("AcousticFDTD: pressure diverged (FDTD_ERR_UNSTABLE)")
            super().run_plain(solver, n)

    res = SequentialServer(backend=Diverging(clock), clock=clock, sleep=clock.sleep).run(reqs)
    errs = {r.rid: r.error for r in res}
    assert errs[reqs[2].rid] is not None
    assert sum(e is None for e in errs.values()) == 5


def test_cancel_queued_and_running_requests():
    clock = FakeClock()
    reqs = mixed_room_requests(8, seed=4, steps=(2000, 3000), axes=(32,))
    for i, r in enumerate(reqs):
        r.arrival = 0.01 * i
    srv = BatchServer(max_slots=2, chunk=64, backend=FakeBackend(clock), clock=clock, sleep=clock.sleep)
    running, queued = reqs[0].rid, reqs[7].rid
    srv.cancel(queued)                       # dropped before it is admitted

    class Batch(FakeBatch):                  # cancels reqs[0] after its first chunk
        def step(self, n, use_graph=True):
            super().step(n, use_graph)
            srv.cancel(running)

    srv.backend.batch = lambda: Batch(clock)
    res = {r.rid: r for r in srv.run(reqs)}
    assert res[queued].error == "cancelled" and res[queued].traces.shape[0] == 0
    assert res[running].error == "cancelled" and 0 < res[running].traces.shape[0] < reqs[0].room.n_steps
    assert all(res[q.rid].ok for q in reqs[1:7])


def test_deadline_evicts_and_rejects():
    clock = FakeClock()
    reqs = mixed_room_requests(6, seed=5, steps=(1000, 1000), axes=(32,))
    for r in reqs:
        r.arrival = 0.0
    reqs[0].deadline = 0.03          # runs, but needs 1000 x 1e-4 s = 0.1 s
    reqs[5].deadline = 0.01          # still queued behind the two slots when it expires
    srv = BatchServer(max_slots=2, chunk=50, backend=FakeBackend(clock), clock=clock, sleep=clock.sleep)
    res = {r.rid: r for r in srv.run(reqs)}
    assert res[reqs[0].rid].error == "deadline exceeded"
    assert 0 < res[reqs[0].rid].traces.shape[0] < 1000
    assert res[reqs[5].rid].error == "deadline exceeded" and res[reqs[5].rid].traces.shape[0] == 0
    assert all(res[q.rid].ok for q in reqs[1:5])


def test_allocation_failure_and_oversized_request_are_rejected():
    clock = FakeClock()
    reqs = mixed_room_requests(6, seed=6, steps=(100, 200), axes=(32,))
    big = Request(99, mixed_room_requests(1, seed=7, steps=(100, 100), axes=(128,))[0].room)
    budget = 3 * max(room_bytes(r.room) for r in reqs)
    assert room_bytes(big.room) > budget
    be = FakeBackend(clock, budget=budget, alloc_fail=[reqs[1].room])
    res = {r.rid: r for r in BatchServer(max_slots=4, chunk=32, backend=be, clock=clock,
                                        sleep=clock.sleep).run(reqs + [big])}
    assert res[99].error == "exceeds the memory budget"
    assert res[reqs[1].rid].error.startswith("allocation failed")
    assert sum(r.ok for r in res.values()) == 5
    assert be.peak_bytes <= budget


def test_preempt_and_resume_continue_where_they_stopped():
    """A running request pre-empted at a chunk boundary leaves the GPU (slot and
    memory freed) with its state; resumed, it continues from its step and its
    result joins both parts, as if it had run without a pause."""
    clock = FakeClock()
    be = FakeBackend(clock)
    reqs = small_requests(6)
    for r in reqs:
        r.arrival = 0.0
        r.room.n_steps = 400
    srv = BatchServer(max_slots=8, chunk=64, backend=be, clock=clock, sleep=clock.sleep)
    target = reqs[2].rid
    srv.preempt(target)
    first = srv.run(reqs)
    assert target not in [r.rid for r in first] and target in srv.paused
    assert srv.log[0]["preempted"] == 1
    req, snap, part, _ = srv.paused[target]
    assert snap["step"] == 64 and part.shape == (64, 1)
    live_before = be.live
    srv.resume(target)
    second = srv.run([])
    assert [r.rid for r in second] == [target] and not srv.paused
    res = second[0]
    assert res.ok and np.array_equal(res.traces[:, 0], np.arange(400, dtype=np.float32))
    assert be.live == live_before                        # every solver released
    assert all(r.ok and r.traces.shape[0] == 400 for r in first)


def test_paused_request_stays_paused_without_resume():
    clock = FakeClock()
    be = FakeBackend(clock)
    reqs = small_requests(3)
    for r in reqs:
        r.arrival = 0.0
    srv = BatchServer(max_slots=4, chunk=32, backend=be, clock=clock, sleep=clock.sleep)
    srv.preempt(reqs[0].rid)
    out = srv.run(reqs)
    assert sorted(r.rid for r in out) == sorted(r.rid for r in reqs[1:])
    assert list(srv.paused) == [reqs[0].rid]
    assert srv.run([]) == []                             # nothing to do until resume
