"""One room split along i over several ranks (one GPU each): slab decomposition.

Rank r owns the planes ``partition(Nx, world)[r]`` and keeps three ghost
planes on each side.  One step on every rank, fused schedule (the default):

    deposit(n)          source sample n into the local copy of the source cell
                        (owned or ghost: the copies stay identical)
    step()              the single-pass TMA kernel on the own planes; it
                        recomputes the Vx faces just outside the slab from
                        ghost P and ghost old Vx
    exchange(P, Vx)     3 planes of the new P and 2 of the new Vx to each
                        neighbour, one batch of point-to-point messages
    record()            receivers whose first tap lies in the own planes

or the two-pass schedule: deposit, velocity, exchange(Vx), pressure,
exchange(P), record.

and every 256 steps the stability sample of the reference
(csrc/kernels/acoustic_fdtd.cpp:1245-1268) over the own cells, reduced (min of
the failing flat index) over ranks.  Each slab computes exactly what the
whole-room kernels compute for its planes, so traces and fields equal the
single-GPU engine's bit for bit.

Backends: ``EngineSlab`` (the CUDA slab kernels, fields as torch CUDA
tensors).  Exchanges: ``DistExchange`` (torch.distributed point-to-point:
NCCL over NVLink between GPUs, or gloo between CPU processes) and
``LocalExchange`` (several slabs in one process, plane copies).  With peer
stores the fused step itself writes the neighbours' ghost planes (their next
buffers) through pointers to their fields, so no exchange runs at all:
``PeerStores`` for slabs in one process, ``PeerDistExchange`` across
processes (fields shared through CUDA IPC; between steps only a barrier —
a stream-ordered NCCL all-reduce of one word, or a host barrier).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

from .precision import pressure_taps
from .rooms import Room

GHOST = 3
# planes received from the left neighbour (= sent to the right one) and from
# the right neighbour (= sent to the left one), per exchanged field
WIDTHS = {"P": (3, 3), "Vx": (2, 2)}
CHECK_PERIOD, CHECK_STRIDE = 256, 1013


def partition(nx: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous plane ranges, sizes differing by at most one, each >= 3 planes."""
    if world < 1 or nx < 3 * world:
        raise ValueError(f"cannot split {nx} planes over {world} ranks (3 planes per rank at least)")
    base, rem = divmod(nx, world)
    out, i = [], 0
    for r in range(world):
        n = base + (1 if r < rem else 0)
        out.append((i, i + n))
        i += n
    return out


def receiver_owner(room: Room, ranges: Sequence[Tuple[int, int]]) -> List[int]:
    """Rank owning each receiver: the one whose planes hold its first tap."""
    idx, _ = pressure_taps(room.nx, room.ny, room.nz, room.receiver_xyz())
    planes = idx.reshape(-1, 8)[:, 0] // (room.ny * room.nz)
    return [next(r for r, (a, b) in enumerate(ranges) if a <= p < b) for p in planes]


class EngineSlab:
    """CUDA backend: one fdtd_b200_slab handle over torch-allocated fields.
    fused=True steps with the single-pass kernel, else with the two passes."""

    def __init__(self, room: Room, i0: int, i1: int, rec_ids: Sequence[int], device=None,
                 fused: bool = True):
        import torch
        from . import _native
        self._native, self._lib = _native, _native.load()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        L, sz = C.c_int(0), C.c_int(0)
        rc = self._lib.fdtd_b200_slab_layout(room.nx, room.ny, room.nz, i0, i1, C.byref(L), C.byref(sz))
        if rc != 0:
            raise ValueError(f"slab [{i0}, {i1}) of {room.nx} planes: rc={rc}")
        self.room, self.i0, self.i1, self.own = room, i0, i1, i1 - i0
        self.L, self.sz = L.value, sz.value
        self.fused = bool(fused)
        self.fields = [torch.zeros((self.L, room.ny, self.sz), dtype=torch.float32, device=self.device)
                       for _ in range(8)]
        ptrs = (C.c_void_p * 8)(*[t.data_ptr() for t in self.fields])
        a6 = np.ascontiguousarray(room.absorption, np.float32)
        h = self._lib.fdtd_b200_slab_create(room.nx, room.ny, room.nz, i0, i1, room.dx, room.c, room.rho,
                                            room.n_pml, a6.ctypes.data_as(_native.P_f32),
                                            C.cast(ptrs, C.POINTER(C.c_void_p)), self.device.index)
        if not h:
            raise RuntimeError("fdtd_b200_slab_create failed: " + _native.last_error())
        self._h = C.c_void_p(h)
        self._check(self._lib.fdtd_b200_slab_set_stream(
            self._h, C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)), "slab_set_stream")
        sig = np.ascontiguousarray(room.signal(), np.float32)
        self._check(self._lib.fdtd_b200_slab_set_source(self._h, room.src_flat,
                                                        sig.ctypes.data_as(_native.P_f32), sig.size),
                    "slab_set_source")
        idx, w = pressure_taps(room.nx, room.ny, room.nz, room.receiver_xyz())
        self.rec_ids = list(rec_ids)
        sel = np.concatenate([np.arange(8 * r, 8 * r + 8) for r in self.rec_ids]) if self.rec_ids else \
            np.zeros(0, np.int64)
        self._idx = np.ascontiguousarray(idx[sel], np.int32)
        self._w = np.ascontiguousarray(w[sel], np.float32)
        self._check(self._lib.fdtd_b200_slab_set_receivers(
            self._h, len(self.rec_ids), self._idx.ctypes.data_as(_native.P_i32),
            self._w.ctypes.data_as(_native.P_f32), room.n_steps), "slab_set_receivers")

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: rc={rc} {self._native.last_error()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fdtd_b200_slab_destroy(self._h)
            self._h = None

    __del__ = close

    def field(self, name: str):
        if name == "P":
            return self.fields[self._lib.fdtd_b200_slab_current(self._h)]
        return self.fields[2 + 3 * self._lib.fdtd_b200_slab_vset(self._h) + {"Vx": 0, "Vy": 1, "Vz": 2}[name]]

    def deposit(self, n: int):
        self._check(self._lib.fdtd_b200_slab_deposit(self._h, int(n)), "slab_deposit")

    def step(self):
        self._check(self._lib.fdtd_b200_slab_step(self._h), "slab_step")

    def add_pressure(self, cell: int, amp: float):
        """Deposit a host value into this slab's copy of a cell (if it has one)."""
        self._check(self._lib.fdtd_b200_slab_add_pressure(self._h, int(cell), float(amp)), "slab_add_pressure")

    def read_last(self, out: np.ndarray):
        """The last recorded step's samples of this slab's receivers, into out."""
        self._check(self._lib.fdtd_b200_slab_read_last(self._h, out.ctypes.data_as(self._native.P_f32),
                                                       out.size), "slab_read_last")

    def step_part(self, part: int):
        """Part 1: the own planes the neighbours keep as ghosts; part 2: the
        rest, then the buffer flip (together: one step)."""
        self._check(self._lib.fdtd_b200_slab_step_part(self._h, int(part)), "slab_step_part")

    def set_peer(self, side: int, fields, i0: int, i1: int):
        """Let the fused step write the neighbour's ghost planes: fields = its
        eight tensors (or None to clear), [i0, i1) = its planes."""
        if fields is None:
            self._check(self._lib.fdtd_b200_slab_set_peer(self._h, int(side), None, 0, 0), "slab_set_peer")
            return
        ptrs = (C.c_void_p * 8)(*[t.data_ptr() for t in fields])
        self._check(self._lib.fdtd_b200_slab_set_peer(self._h, int(side), C.cast(ptrs, C.POINTER(C.c_void_p)),
                                                      int(i0), int(i1)), "slab_set_peer")

    def velocity(self):
        self._check(self._lib.fdtd_b200_slab_velocity(self._h), "slab_velocity")

    def pressure(self):
        self._check(self._lib.fdtd_b200_slab_pressure(self._h), "slab_pressure")

    def record(self):
        self._check(self._lib.fdtd_b200_slab_record(self._h), "slab_record")

    def check(self, phase: int) -> int:
        bad = C.c_longlong(0)
        self._check(self._lib.fdtd_b200_slab_check(self._h, int(phase), C.byref(bad)), "slab_check")
        return bad.value

    def traces(self) -> np.ndarray:
        n_rec = len(self.rec_ids)
        out = np.empty(max(self.room.n_steps * n_rec, 1), np.float32)
        rows = C.c_int(0)
        self._check(self._lib.fdtd_b200_slab_get_traces(self._h, out.ctypes.data_as(self._native.P_f32),
                                                        out.size, C.byref(rows)), "slab_get_traces")
        return out[: rows.value * n_rec].reshape(rows.value, n_rec)

    def own_pressure(self) -> np.ndarray:
        """Current P of the own planes, (own, Ny, Nz)."""
        p = self.field("P")[GHOST:GHOST + self.own, :, : self.room.nz]
        return p.cpu().numpy()

    @property
    def launch_count(self) -> int:
        return self._lib.fdtd_b200_slab_launch_count(self._h)


class LocalExchange:
    """Ghost exchange between slabs held by one process (ordered by i)."""

    def __init__(self, slabs):
        self.slabs = slabs

    def exchange(self, *names: str):
        for name in names:
            wl, wr = WIDTHS[name]
            for a, b in zip(self.slabs[:-1], self.slabs[1:]):
                fa, fb = a.field(name), b.field(name)
                fb[GHOST - wl:GHOST].copy_(fa[a.own + GHOST - wl:a.own + GHOST])
                fa[a.own + GHOST:a.own + GHOST + wr].copy_(fb[GHOST:GHOST + wr])

    def reduce_min(self, value: int) -> int:
        return value

    def gather(self, obj) -> list:
        return [obj]


class PeerStores(LocalExchange):
    """Slabs in one process whose fused steps write each other's ghost planes:
    nothing to exchange (the kernels run in order on one stream)."""

    def __init__(self, slabs):
        super().__init__(slabs)
        for a, b in zip(self.slabs[:-1], self.slabs[1:]):
            a.set_peer(1, b.fields, b.i0, b.i1)
            b.set_peer(0, a.fields, a.i0, a.i1)

    def exchange(self, *names: str):
        pass


class DistExchange:
    """Ghost exchange with the neighbouring ranks over torch.distributed."""

    def __init__(self, slab, rank: int, world: int, group=None):
        self.slab, self.rank, self.world, self.group = slab, rank, world, group

    def exchange(self, *names: str):
        import torch.distributed as dist
        own = self.slab.own
        ops = []
        for name in names:
            t = self.slab.field(name)
            wl, wr = WIDTHS[name]
            if self.rank > 0:
                ops += [dist.P2POp(dist.isend, t[GHOST:GHOST + wr], self.rank - 1, self.group),
                        dist.P2POp(dist.irecv, t[GHOST - wl:GHOST], self.rank - 1, self.group)]
            if self.rank < self.world - 1:
                ops += [dist.P2POp(dist.isend, t[own + GHOST - wl:own + GHOST], self.rank + 1, self.group),
                        dist.P2POp(dist.irecv, t[own + GHOST:own + GHOST + wr], self.rank + 1, self.group)]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def reduce_min(self, value: int) -> int:
        import torch
        import torch.distributed as dist
        dev = self.slab.field("P").device
        t = torch.tensor([value if value >= 0 else np.iinfo(np.int64).max], dtype=torch.int64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        v = int(t.item())
        return -1 if v == np.iinfo(np.int64).max else v

    def gather(self, obj) -> list:
        import torch.distributed as dist
        out = [None] * self.world
        dist.all_gather_object(out, obj, group=self.group)
        return out


class SlabRunner:
    """Steps the slabs of one room in lockstep with their ghost exchanges.

    overlap (fused schedule with an exchange): each step computes the planes
    the neighbours keep as ghosts first, then sends them on a side stream
    while the interior planes are computed on the slabs' stream; the next
    step's kernels wait for the exchange."""

    def __init__(self, slabs, exchange, overlap: bool = False):
        self.slabs = list(slabs)
        self.ex = exchange
        self.fused = all(getattr(s, "fused", False) for s in self.slabs)
        self.overlap = bool(overlap) and self.fused and not isinstance(exchange, PeerStores)
        self.step_count = 0
        self.phase = 0
        if self.overlap:
            import torch
            dev = self.slabs[0].device
            self._main = torch.cuda.current_stream(dev)
            self._side = torch.cuda.Stream(dev)

    def _fused_overlapped(self):
        import torch
        for s in self.slabs:
            s.step_part(1)
        ready = torch.cuda.Event()
        ready.record(self._main)
        for s in self.slabs:
            s.step_part(2)                  # interior on the main stream; flips the buffers
        with torch.cuda.stream(self._side):
            self._side.wait_event(ready)
            self.ex.exchange("P", "Vx")     # the new ghost planes, beside the interior
        self._main.wait_stream(self._side)

    def step(self, n_steps: int = 1, host_sample=None):
        """n_steps steps; host_sample(n) -> the source amplitude of step n given
        by the host (deposited as a launch argument) instead of the slabs'
        device copy of the signal."""
        for _ in range(int(n_steps)):
            for s in self.slabs:
                if host_sample is None:
                    s.deposit(self.step_count)
                else:
                    s.add_pressure(s.room.src_flat, host_sample(self.step_count))
            if self.fused and self.overlap:
                self._fused_overlapped()
            elif self.fused:
                for s in self.slabs:
                    s.step()
                self.ex.exchange("P", "Vx")
            else:
                for s in self.slabs:
                    s.velocity()
                self.ex.exchange("Vx")
                for s in self.slabs:
                    s.pressure()
                self.ex.exchange("P")
            for s in self.slabs:
                s.record()
            self.step_count += 1
            if self.step_count % CHECK_PERIOD == 0:
                bads = [s.check(self.phase) for s in self.slabs]
                bad = min([b for b in bads if b >= 0], default=-1)
                bad = self.ex.reduce_min(bad)
                self.phase = (self.phase + 1) % CHECK_STRIDE
                if bad >= 0:
                    raise RuntimeError("AcousticFDTD: pressure diverged (FDTD_ERR_UNSTABLE)")

    def traces(self, n_rec: int) -> np.ndarray:
        """All receivers' traces (steps, n_rec), assembled on every rank."""
        parts = []
        for s in self.slabs:
            parts.append((list(s.rec_ids), s.traces()))
        gathered = [p for obj in self.ex.gather(parts) for p in obj]
        rows = max((t.shape[0] for _, t in gathered), default=0)
        out = np.zeros((rows, n_rec), np.float32)
        for ids, t in gathered:
            for q, r in enumerate(ids):
                out[:, r] = t[:, q]
        return out

    def pressure_field(self) -> np.ndarray:
        """The whole room's current P (Nx, Ny, Nz), assembled on every rank."""
        parts = [(s.i0, s.own_pressure()) for s in self.slabs]
        gathered = sorted((p for obj in self.ex.gather(parts) for p in obj), key=lambda x: x[0])
        return np.concatenate([p for _, p in gathered], axis=0)


class PeerDistExchange(DistExchange):
    """This rank's fused step writes its neighbours' ghost planes directly
    (their fields mapped here through CUDA IPC); a step then ends with a
    barrier instead of an exchange: a stream-ordered NCCL all-reduce of one
    word (every rank's step has finished, so its stores have landed), or,
    without NCCL, a stream synchronisation and a host barrier."""

    def __init__(self, slab, rank: int, world: int, group=None):
        import torch
        import torch.distributed as dist
        from torch.multiprocessing.reductions import reduce_tensor
        super().__init__(slab, rank, world, group)
        mine = (rank, slab.i0, slab.i1, [reduce_tensor(t) for t in slab.fields])
        infos = self.gather(mine)
        self._peers = []                     # keeps the IPC mappings alive
        for side, other in ((0, rank - 1), (1, rank + 1)):
            if 0 <= other < world:
                r, i0, i1, handles = infos[other]
                tensors = [fn(*args) for fn, args in handles]
                self._peers.append(tensors)
                slab.set_peer(side, tensors, i0, i1)
        self._nccl = dist.get_backend(group) == "nccl"
        self._token = torch.zeros(1, dtype=torch.int32, device=slab.device)

    def exchange(self, *names: str):
        import torch
        import torch.distributed as dist
        if self._nccl:
            dist.all_reduce(self._token, group=self.group)
        else:
            torch.cuda.current_stream(self.slab.device).synchronize()
            dist.barrier(group=self.group)


def local_room(room: Room, n_slabs: int, device=None, fused: bool = True, peer_stores: bool = False,
               overlap: bool = False) -> SlabRunner:
    """All slabs of a room in this process on one GPU (tests, single-GPU runs);
    peer_stores: the fused steps write each other's ghost planes directly;
    overlap: plane copies on a side stream beside the interior planes."""
    ranges = partition(room.nx, n_slabs)
    owners = receiver_owner(room, ranges)
    slabs = [EngineSlab(room, a, b, [q for q, o in enumerate(owners) if o == r], device, fused)
             for r, (a, b) in enumerate(ranges)]
    if peer_stores:
        if not fused:
            raise ValueError("peer stores come with the fused step")
        return SlabRunner(slabs, PeerStores(slabs))
    return SlabRunner(slabs, LocalExchange(slabs), overlap=overlap)


def distributed_room(room: Room, rank: int, world: int, group=None, device=None,
                     fused: bool = True, peer_memory: bool = False, overlap: bool = False) -> SlabRunner:
    """This rank's slab of a room split over `world` ranks (torch.distributed
    initialised); peer_memory: the fused step writes the neighbours' ghost
    planes through CUDA IPC mappings of their fields and steps end with a
    barrier (the ranks' GPUs must reach each other's memory); overlap: the
    exchange runs on a side stream beside the interior planes."""
    ranges = partition(room.nx, world)
    owners = receiver_owner(room, ranges)
    a, b = ranges[rank]
    slab = EngineSlab(room, a, b, [q for q, o in enumerate(owners) if o == rank], device, fused)
    if peer_memory:
        if not fused:
            raise ValueError("peer stores come with the fused step")
        return SlabRunner([slab], PeerDistExchange(slab, rank, world, group))
    return SlabRunner([slab], DistExchange(slab, rank, world, group), overlap=overlap)
