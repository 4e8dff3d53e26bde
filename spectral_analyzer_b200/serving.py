"""Serving rooms: continuous batching of independent FDTD requests on one GPU.

A request is a room (grid, absorption, point source, receivers, step count);
its result is the receivers' traces.  ``BatchServer`` admits requests as they
arrive, whenever a slot and device memory are free, and advances all admitted
rooms together with the engine's batched step (one persistent kernel over the
work items of every room per time step, plus a small epilogue), replaying a
CUDA graph of ``chunk`` steps between scheduling points.  Rooms finish
independently and leave the batch at the next chunk boundary; newly arrived
rooms join there.  ``SequentialServer`` is the baseline: one request at a time
through the plain single-room path.

Both compute each room with the same arithmetic, so a room's traces are
bit-identical alone and in any mix of other rooms.

Failures stay with the request that caused them.  A room whose 256-step check
fails (FDTD_ERR_UNSTABLE, e.g. a NaN in its source signal) stops on the device
at that step and leaves with ``error`` set and the traces it recorded; a
request that does not fit the memory budget even alone, or whose solver cannot
be allocated, is rejected; ``cancel(rid)`` and a request's ``deadline`` evict
it at the next chunk boundary.  The other rooms carry on unchanged.  Only an
engine-level failure (a CUDA error or a timed-out load wait in the batched
kernel) ends the run.
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .rooms import Room

GRID_AXES = tuple(range(32, 257, 16))


@dataclass
class Request:
    rid: int
    room: Room
    arrival: float = 0.0                # seconds after the start of the run
    deadline: Optional[float] = None    # latency budget in seconds (None: none)


@dataclass
class Result:
    rid: int
    traces: np.ndarray          # (steps, n_rec) float32; the steps done when error is set
    arrival: float
    start: float
    finish: float
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.finish - self.arrival

    @property
    def ok(self) -> bool:
        return self.error is None


def room_bytes(room: Room) -> int:
    """Device memory of one room: 8 fields (P x2, V x2 sets) plus its trace."""
    sz = (room.nz + 7) // 8 * 8
    return 8 * room.nx * room.ny * sz * 4 + room.n_steps * len(room.receivers) * 4 + (1 << 16)


def mixed_room_requests(n: int = 256, seed: int = 3, steps=(500, 8000), axes=GRID_AXES,
                     rec=(1, 4), a_range=(0.02, 0.3), n_pml: int = 10) -> List[Request]:
    """Rooms with axes drawn from ``axes``, steps U{steps}, 1-4 receivers, per-face
    absorption U[a_range], Gaussian or Ricker source, interior source/receivers."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        nx, ny, nz = (int(rng.choice(axes)) for _ in range(3))
        n_steps = int(rng.integers(steps[0], steps[1] + 1))
        n_rec = int(rng.integers(rec[0], rec[1] + 1))
        a6 = tuple(float(v) for v in rng.uniform(a_range[0], a_range[1], 6).astype(np.float32))
        kind = "gaussian" if rng.random() < 0.5 else "ricker"

        def interior(d):
            lo, hi = n_pml + 2, d - n_pml - 2
            return int(rng.integers(lo, hi)) if lo < hi else d // 2

        src = (interior(nx), interior(ny), interior(nz))
        recs = [(interior(nx), interior(ny), interior(nz)) for _ in range(n_rec)]
        room = Room(nx, ny, nz, n_steps, src, recs, a6, kind, n_pml=n_pml, name=f"req{q}")
        out.append(Request(q, room))
    return out


def poisson_arrivals(n: int, rate: float, seed: int = 5) -> np.ndarray:
    """Arrival times (s) of a Poisson process with the given rate (requests/s)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def percentile(xs: Sequence[float], p: float) -> float:
    return float(np.percentile(np.asarray(xs, dtype=np.float64), p)) if len(xs) else float("nan")


def summarize(results: Sequence[Result], work: float) -> dict:
    """Throughput and latency over the completed requests (failed ones counted apart)."""
    done = [r for r in results if r.ok]
    lat = [r.latency for r in done]
    t_first = min(r.arrival for r in results)
    t_last = max(r.finish for r in results)
    span = t_last - t_first
    return {"requests": len(done), "failed": len(results) - len(done), "makespan_s": span,
            "requests_per_s": len(done) / span,
            "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)) if lat else float("nan"),
            "gcell_updates_per_s": work / span / 1e9}


def request_work(reqs: Sequence[Request]) -> float:
    return float(sum(r.room.cells * r.room.n_steps for r in reqs))


# ---------------------------------------------------------------- engine glue
def make_solver(room: Room, device=None):
    """A single-room solver configured for a request (source and receivers set)."""
    from .fdtd import AcousticFDTD
    f = AcousticFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho,
                     cell_type=room.cell_type(), plate_iz=-1, plate_active=room.plate_active(),
                     n_pml=room.n_pml, device=device)
    f.set_face_absorption(room.absorption)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    f.set_point_source(room.src_flat, room.signal())
    f.set_receivers(idx, w, room.n_steps)
    return f


class EngineBatch:
    """ctypes wrapper of the engine's batch object (fdtd_b200_batch_*)."""

    def __init__(self, device: int = 0):
        from . import _native
        self._lib = _native.load()
        self._native = _native
        h = self._lib.fdtd_b200_batch_create(device)
        if not h:
            raise RuntimeError("fdtd_b200_batch_create failed: " + _native.last_error())
        self._h = C.c_void_p(h)
        self.members: list = []

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.fdtd_b200_batch_destroy(self._h)
            self._h = None

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: rc={rc} {self._native.last_error()}")

    def set_segment(self, planes: int):
        self._check(self._lib.fdtd_b200_batch_set_segment(self._h, int(planes)), "batch_set_segment")

    def set_tile(self, tile_k: int):
        """Work-item tile width: 128 (8 rows) or 64 (16 rows); next set() on."""
        self._check(self._lib.fdtd_b200_batch_set_tile(self._h, int(tile_k)), "batch_set_tile")

    def set(self, solvers, limits):
        n = len(solvers)
        arr = (C.c_void_p * max(n, 1))(*[s._h.value for s in solvers])
        lim = np.ascontiguousarray(limits, dtype=np.int32)
        self._check(self._lib.fdtd_b200_batch_set(self._h, C.cast(arr, C.POINTER(C.c_void_p)),
                                                  lim.ctypes.data_as(C.POINTER(C.c_int)), n), "batch_set")
        self.members = list(solvers)

    def step(self, n_steps: int, use_graph: bool = True):
        self._check(self._lib.fdtd_b200_batch_step(self._h, int(n_steps), 1 if use_graph else 0), "batch_step")

    def sync(self):
        n = max(len(self.members), 1)
        steps = np.zeros(n, np.int32)
        status = np.zeros(n, np.int32)
        self._check(self._lib.fdtd_b200_batch_sync(self._h, steps.ctypes.data_as(C.POINTER(C.c_int)),
                                                   status.ctypes.data_as(C.POINTER(C.c_int))), "batch_sync")
        return steps[: len(self.members)], status[: len(self.members)]

    @property
    def launch_count(self) -> int:
        return self._lib.fdtd_b200_batch_launch_count(self._h)


# ---------------------------------------------------------------- schedulers
PREEMPTED = "pre-empted"      # a running request taken off the GPU by preempt()


class BatchServer:
    """Continuous batching: admit on arrival when a slot and memory are free.

    ``backend`` supplies ``make(room) -> solver``, ``batch() -> batch`` (with
    set/step/sync) and ``traces(solver)``; the default uses the CUDA engine.
    """

    def __init__(self, max_slots: int = 64, mem_budget: Optional[int] = None, chunk: int = 64,
                 use_graph: bool = True, seg_planes: int = 0, tile_k: int = 128, backend=None,
                 clock: Callable[[], float] = time.perf_counter, sleep=time.sleep):
        self.max_slots = max_slots
        self.mem_budget = mem_budget
        self.chunk = chunk
        self.use_graph = use_graph
        self.seg_planes = seg_planes
        self.tile_k = tile_k
        self.backend = backend or _EngineBackend()
        self.clock = clock
        self.sleep = sleep
        self.log: List[dict] = []
        self._cancelled: set = set()
        self._preempt: set = set()
        self._resume: set = set()
        self.paused: Dict[int, tuple] = {}   # rid -> (request, snapshot, traces so far, first start)

    def cancel(self, rid: int) -> None:
        """Ask for request ``rid`` to be dropped (queued) or evicted (running)
        at the next scheduling point; safe to call from another thread."""
        self._cancelled.add(rid)

    def preempt(self, rid: int) -> None:
        """Ask for running request ``rid`` to leave the GPU at the next
        scheduling point: its state (fields, step count, check phase) and the
        traces recorded so far go to host memory and its slot and device
        memory are freed.  It waits until ``resume(rid)``; then it is admitted
        again before the queued requests and continues exactly where it
        stopped (the traces of both parts are joined).  Safe to call from
        another thread."""
        self._preempt.add(rid)

    def resume(self, rid: int) -> None:
        """Let a pre-empted request ``rid`` back in (at the next scheduling point)."""
        self._resume.add(rid)

    def run(self, requests: Sequence[Request]) -> List[Result]:
        be = self.backend
        budget = self.mem_budget if self.mem_budget is not None else be.free_memory()
        queue = deque(sorted(requests, key=lambda r: r.arrival))
        batch = be.batch()
        if self.seg_planes:
            batch.set_segment(self.seg_planes)
        if self.tile_k != 128:
            batch.set_tile(self.tile_k)
        active: List[tuple] = []          # (request, solver, start_time)
        self._parts: Dict[int, np.ndarray] = {}   # traces recorded before a pre-emption
        used = 0
        results: List[Result] = []
        t0 = self.clock()
        dirty = False

        def reject(req, now, why):
            empty = np.zeros((0, len(req.room.receivers)), np.float32)
            results.append(Result(req.rid, empty, req.arrival, now, now, error=why))

        def late(req, now):
            return req.deadline is not None and now > req.arrival + req.deadline

        resumed: deque = deque()          # (request, snapshot, traces so far, first start)
        while queue or active or resumed or (self.paused and self._resume & set(self.paused)):
            now = self.clock() - t0
            for rid in list(self._resume):
                if rid in self.paused:
                    resumed.append(self.paused.pop(rid))
                    self._resume.discard(rid)
            # pre-empted requests come back first, when a slot and memory are free
            while resumed and room_bytes(resumed[0][0].room) > budget:
                reject(resumed.popleft()[0], now, "exceeds the memory budget")
            while resumed and len(active) < self.max_slots and used + room_bytes(resumed[0][0].room) <= budget:
                req, snap, part, start = resumed.popleft()
                try:
                    solver = be.make(req.room)
                    be.restore(solver, snap)
                except (RuntimeError, MemoryError) as e:
                    reject(req, now, f"allocation failed on resume: {e}")
                    continue
                self._parts[req.rid] = part
                active.append((req, solver, start))
                used += room_bytes(req.room)
                dirty = True
            # queued requests that were cancelled, ran out of time, or can never fit
            if queue:
                keep_q = deque()
                for req in queue:
                    if req.rid in self._cancelled:
                        reject(req, now, "cancelled")
                    elif late(req, now):
                        reject(req, now, "deadline exceeded")
                    elif room_bytes(req.room) > budget:
                        reject(req, now, "exceeds the memory budget")
                    else:
                        keep_q.append(req)
                queue = keep_q
            while (queue and queue[0].arrival <= now and len(active) < self.max_slots
                   and used + room_bytes(queue[0].room) <= budget):
                req = queue.popleft()
                try:
                    solver = be.make(req.room)
                except (RuntimeError, MemoryError) as e:
                    reject(req, now, f"allocation failed: {e}")
                    continue
                active.append((req, solver, now))
                used += room_bytes(req.room)
                dirty = True
            if not active:
                if queue:
                    self.sleep(min(max(queue[0].arrival - now, 0.0), 0.05))
                elif not resumed:
                    break                 # only pre-empted requests left, none resumed
                continue
            if dirty:
                batch.set([s for _, s, _ in active], [r.room.n_steps for r, _, _ in active])
                dirty = False
            batch.step(self.chunk, self.use_graph)
            steps, status = batch.sync()
            now = self.clock() - t0
            leave: Dict[int, Optional[str]] = {}
            for q, (r, _, _) in enumerate(active):
                if status[q] != 0:
                    leave[q] = f"pressure diverged (FDTD_ERR_UNSTABLE) by step {int(steps[q])}"
                elif steps[q] >= r.room.n_steps:
                    leave[q] = None
                elif r.rid in self._cancelled:
                    leave[q] = "cancelled"
                elif late(r, now):
                    leave[q] = "deadline exceeded"
                elif r.rid in self._preempt:
                    leave[q] = PREEMPTED
            self.log.append({"t": now, "active": len(active),
                             "finished": sum(1 for e in leave.values() if e is None),
                             "preempted": sum(1 for e in leave.values() if e is PREEMPTED),
                             "failed": sum(1 for e in leave.values() if e is not None and e is not PREEMPTED),
                             "queued": len(queue)})
            if leave:
                keep = [a for q, a in enumerate(active) if q not in leave]
                batch.set([s for _, s, _ in keep], [r.room.n_steps for r, _, _ in keep])
                for q, err in leave.items():
                    req, solver, start = active[q]
                    tr = be.traces(solver)
                    part = self._parts.pop(req.rid, None)
                    if part is not None:
                        tr = np.concatenate([part, tr], axis=0)
                    if err is PREEMPTED:
                        self._preempt.discard(req.rid)
                        self.paused[req.rid] = (req, be.snapshot(solver), tr, start)
                    else:
                        results.append(Result(req.rid, tr, req.arrival, start, now, error=err))
                    used -= room_bytes(req.room)
                    be.release(solver)
                active = keep
                dirty = False
        return sorted(results, key=lambda r: r.rid)


class SequentialServer:
    """Baseline: one request at a time through the plain single-room path."""

    def __init__(self, backend=None, clock: Callable[[], float] = time.perf_counter, sleep=time.sleep):
        self.backend = backend or _EngineBackend()
        self.clock = clock
        self.sleep = sleep

    def run(self, requests: Sequence[Request]) -> List[Result]:
        be = self.backend
        results = []
        t0 = self.clock()
        for req in sorted(requests, key=lambda r: r.arrival):
            now = self.clock() - t0
            if req.arrival > now:
                self.sleep(req.arrival - now)
            start = self.clock() - t0
            solver = be.make(req.room)
            err = None
            try:
                be.run_plain(solver, req.room.n_steps)
            except RuntimeError as e:          # FDTD_ERR_UNSTABLE: this request only
                err = f"pressure diverged: {e}"
            traces = be.traces(solver)
            results.append(Result(req.rid, traces, req.arrival, start, self.clock() - t0, error=err))
            be.release(solver)
        return sorted(results, key=lambda r: r.rid)


class _EngineBackend:
    def __init__(self, device: Optional[int] = None):
        import torch
        self.device = torch.cuda.current_device() if device is None else device

    def free_memory(self) -> int:
        import torch
        free, _ = torch.cuda.mem_get_info(self.device)
        return int(free * 0.85)

    def make(self, room: Room):
        return make_solver(room, device=self.device)

    def batch(self):
        return EngineBatch(self.device)

    def run_plain(self, solver, n_steps: int):
        solver.step(n_steps)

    def traces(self, solver) -> np.ndarray:
        return solver.get_traces()

    def snapshot(self, solver) -> dict:
        return solver.snapshot()

    def restore(self, solver, snap: dict):
        solver.restore(snap)

    def release(self, solver):
        solver.close()


def calibrate_sequential(requests: Sequence[Request], backend=None) -> float:
    """Mean plain-path service time (s) of the given requests run back to back."""
    be = backend or _EngineBackend()
    t0 = time.perf_counter()
    for req in requests:
        s = be.make(req.room)
        be.run_plain(s, req.room.n_steps)
        be.traces(s)
        be.release(s)
    return (time.perf_counter() - t0) / max(len(requests), 1)
