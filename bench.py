#!/usr/bin/env python
"""Throughput benchmark of the dense acoustic FDTD step on B200.

Workload: the 512x384x256 room (50.3M cells; Ricker 1 kHz point source at a
seeded interior cell, 8 seeded receivers, per-face absorption ~ U[0.02, 0.3],
reference time step).  One bench step = one FDTD time step over the whole grid
(velocity + pressure update, source deposit, 8 receiver samples).

Lines printed (rank 0, one JSON object):
  value     Gcell-updates/s with fields resident in HBM (async stepping,
            CUDA events on the solver's stream, max over ranks);
  e2e       the same metric through the reference-facing C ABI with host
            buffers, per step: fdtd_b200_add_pressure (source sample from the
            host), fdtd_step(st, 1), fdtd_sample_pressure_precomputed (host
            sampler arrays in, 8 receiver values out);
  roofline  the fused step kernel: 32 algorithmic bytes per cell-update over
            its mean launch duration (CUDA events around every launch on the
            launching stream) against the measured HBM copy bandwidth;
  cpu_baseline  the reference's own CPU solver (oracle/_ref, its std::thread
            pool over all host cores) on a time-bounded sample of the same room.

--impl reference times the reference's CPU solver alone (rank 0; other ranks
exit 0).  Multi-GPU: `python bench.py --gpus N` launches its N ranks itself
(torch.distributed.run, one GPU each), or runs under an external torchrun;
with N > 1 ranks the room is split along i into N slabs (strong scaling: one
ghost exchange of 3 P planes and 2 Vx faces per side and step over NCCL,
overlapped with the interior planes); value = the room's cells x steps over
the slowest rank's device time.  --scale-mode replicas runs N independent
copies of the room instead (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL_UPDATE = 32          # read + write of p, vx, vy, vz in float32
METRIC = "Gcell-updates/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "fused_step_room512x384x256.md")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--kernel", choices=["auto", "fused", "two_pass"], default="auto")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bound on the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=90.0,
                    help="bound on the timed part of --impl reference")
    ap.add_argument("--grid", default=None,
                    help="NX,NY,NZ: a smaller seeded room of the same kind (profiling only)")
    ap.add_argument("--serve", action="store_true",
                    help="serving benchmark: continuous batching vs sequential plain launches")
    ap.add_argument("--precision", action="store_true",
                    help="storage-precision study (FP32/BF16/FP16, compensated) vs an FP64 GPU run")
    ap.add_argument("--precision-steps", type=int, default=10000)
    ap.add_argument("--precision-audit", type=int, default=500)
    ap.add_argument("--precision-time-steps", type=int, default=300,
                    help="steps timed per 16-bit mode and step kernel (0: no timing)")
    ap.add_argument("--adjoint", action="store_true",
                    help="gradient w.r.t. per-cell absorption: adjoint timing and checks")
    ap.add_argument("--adjoint-steps", type=int, default=4000)
    ap.add_argument("--adjoint-checkpoint", type=int, default=200)
    ap.add_argument("--adjoint-fd-cells", type=int, default=16,
                    help="layer cells checked by central finite differences (0: none)")
    ap.add_argument("--decompose", action="store_true",
                    help="split the room into slabs along i (torchrun ranks, or --slabs on one GPU)")
    ap.add_argument("--slabs", type=int, default=2)
    ap.add_argument("--scale-mode", choices=["split", "replicas"], default="split",
                    help="N>1: split the room into N slabs along i (strong scaling, one ghost exchange "
                         "per step overlapped with the interior) or run N independent replicas (weak)")
    ap.add_argument("--walled", action="store_true",
                    help="a walled body scene (solid cells, cut-cell fractions, Kirchhoff plate) on both step "
                         "kernels; --grid sets its size (default 512,384,256)")
    ap.add_argument("--walled-steps", type=int, default=200)
    ap.add_argument("--amr", action="store_true",
                    help="the AMR pressure backend on a box grid of --amr-cells^3 cells (gradient order 2, "
                         "anechoic border): cell-updates/s and bytes moved per cell-step")
    ap.add_argument("--amr-cells", type=int, default=160)
    ap.add_argument("--amr-order", type=int, default=2)
    ap.add_argument("--plumbing-check", action="store_true",
                    help="no GPU: ranks on gloo with a host stand-in for the step, to check the "
                         "rank launch, the max-over-ranks timing and the JSON line")
    ap.add_argument("--peer", action="store_true",
                    help="with --decompose: the step writes the neighbours' ghost planes itself")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-load", type=float, default=1.5,
                    help="offered load as a multiple of the sequential plain capacity")
    ap.add_argument("--serve-slots", type=int, default=64)
    ap.add_argument("--serve-chunk", type=int, default=64)
    ap.add_argument("--serve-max-steps", type=int, default=8000)
    args = ap.parse_args()
    global GRID
    GRID = tuple(int(v) for v in args.grid.split(",")) if args.grid else None
    return args


GRID = None


def workload():
    from spectral_analyzer_b200.rooms import large_room, seeded_room
    if GRID:
        r = seeded_room(*GRID, 10000, seed=2, n_rec=8, source_kind="ricker")
        r.name = "room{}x{}x{}_ricker".format(*GRID)
        return r
    return large_room(n_steps=10000)


def config_dict(room, n, kernel):
    return {"workload": room.name + "_8rec", "grid": [room.nx, room.ny, room.nz],
            "cells": room.cells, "receivers": len(room.receivers), "source": "ricker_1kHz",
            "absorption": [round(a, 6) for a in room.absorption], "n_pml": room.n_pml,
            "dt_s": room.dt, "courant": 0.77 / 3 ** 0.5, "step_kernel": kernel,
            "parallelism": f"replicas{n}" if n > 1 else "single",
            "l2_flush": "none: working set 1.6 GB (P x2, V x2 sets) exceeds the 126 MB L2"}


def measured_peak():
    try:
        with open(PEAKS_FILE) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_per_launch():
    """DRAM bytes per fused-step launch from the committed ncu summary, if present."""
    try:
        with open(TRAFFIC_FILE) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch_full_room:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = os.path.join("/tmp", f"fdtd_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[4:]))
                except ValueError:
                    continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [r for r in rows if r[2] > 250.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in loaded for q, v in enumerate(r[3][1:5]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(loaded),
                "power_w_max": max(r[2] for r in rows)}


def cpu_baseline(room, seconds: float):
    """The reference's own solver on the same room, time-bounded; Gcell-updates/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    if orc.reference_available():
        f = orc.RefFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, n_pml=room.n_pml,
                        fast=True)
        f.set_face_absorption(room.absorption)
        kind, cores = "reference", orc.RefFDTD.pool_threads()
        lib = os.path.basename(f.library_path)
    else:
        f = orc.OracleFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, n_pml=room.n_pml)
        f.set_face_absorption(room.absorption)
        kind, cores, lib = "port", 1, "liboracle_fdtd.so"
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    sig = room.signal()
    f.add_pressure(room.src_flat, float(sig[0]))
    f.step(1)                                   # untimed first step (page-in)
    n = 0
    t0 = time.perf_counter()
    while True:
        sc = f.step_count
        f.add_pressure(room.src_flat, float(sig[sc]))
        f.step(1)
        f.sample_pressure_precomputed(idx, w)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 400:
            break
    del f
    val = room.cells * n / el / 1e9
    return {"value": val, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"{n} steps of the 512x384x256 room after 1 warm-up step ({el:.1f} s wall, "
                      f"{lib}, source deposit + step + 8-receiver sample per step)"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    room = workload()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    if orc.reference_available():
        f = orc.RefFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, n_pml=room.n_pml,
                        fast=True)
        kind, cores, lib = "reference", orc.RefFDTD.pool_threads(), None
        lib = os.path.basename(f.library_path)
    else:
        f = orc.OracleFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho, n_pml=room.n_pml)
        kind, cores, lib = "port", 1, "liboracle_fdtd.so"
    f.set_face_absorption(room.absorption)
    idx, w = f.precompute_pressure_samplers(room.receiver_xyz())
    sig = room.signal()

    def one():
        f.add_pressure(room.src_flat, float(sig[f.step_count]))
        f.step(1)
        f.sample_pressure_precomputed(idx, w)

    # the requested warm-up steps (time-bounded at 60 s; the count run is reported)
    warm = 0
    tw = time.perf_counter()
    while warm < args.warmup and (warm < 3 or time.perf_counter() - tw < 60.0):
        one()
        warm += 1
    n = 0
    t0 = time.perf_counter()
    while n < args.steps:
        one()
        n += 1
        if time.perf_counter() - t0 >= args.ref_seconds:
            break
    el = time.perf_counter() - t0
    val = room.cells * n / el / 1e9
    sample = (f"{n} of {args.steps} requested steps of the 512x384x256 room (time-bounded at "
              f"{args.ref_seconds:.0f} s) after {warm} warm-up steps, {lib}")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": METRIC, "n_gpus": args.gpus,
            "steps": n, "warmup": warm, "ms_per_step": el / n * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config_dict(room, 1, "reference_cpu"),
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def engine_arm(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from spectral_analyzer_b200 import AcousticFDTD, _native

    room = workload()
    f = AcousticFDTD(room.nx, room.ny, room.nz, room.dx, room.c, room.rho,
                     cell_type=room.cell_type(), plate_iz=-1, plate_active=room.plate_active(),
                     n_pml=room.n_pml)
    f.set_face_absorption(room.absorption)
    f.set_kernel(args.kernel)
    kernel = f.kernel
    idx8, wgt8 = f.precompute_pressure_samplers(room.receiver_xyz())
    sig = room.signal()
    K, W = args.steps, args.warmup
    f.set_point_source(room.src_flat, sig)
    f.set_receivers(idx8, wgt8, capacity=K + W)
    stream = f.torch_stream()          # the stream every solver kernel is launched on

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident throughput ----
    f.step_async(W)
    assert f.synchronize() == 0
    gpu_id = str(torch.cuda.get_device_properties(local).uuid)
    gpu_id = gpu_id if gpu_id.startswith("GPU-") else "GPU-" + gpu_id
    f.profile(True)
    launches0 = f.launch_count
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_id) as clk:
        e0.record(stream)
        rc = f.step_async(K)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = f.launch_count - launches0
    assert rc == 0 and f.synchronize() == 0, "instability during the timed run"
    ms = e0.elapsed_time(e1)
    prof_ms, prof_n, _ = f.profile_read()
    f.profile(False)
    t_max = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_max = float(t_max.item())
    traces = f.get_traces()
    assert traces.shape == (K + W, len(room.receivers))
    assert np.isfinite(traces).all()

    value = room.cells * K * world / (ms_max / 1e3) / 1e9
    kern_ms = prof_ms / max(prof_n, 1)
    achieved = BYTES_PER_CELL_UPDATE * room.cells / (kern_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = ncu_traffic_per_launch()

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        lib = _native.load()
        h = f._h
        f.set_point_source(room.src_flat, None)
        f.set_receivers(np.zeros(0, np.int32), np.zeros(0, np.float32), 0)
        idx_c = np.ascontiguousarray(idx8, np.int32)
        w_c = np.ascontiguousarray(wgt8, np.float32)
        out = np.zeros(len(room.receivers), np.float32)
        p_idx, p_w, p_out = (idx_c.ctypes.data_as(_native.P_i32), w_c.ctypes.data_as(_native.P_f32),
                             out.ctypes.data_as(_native.P_f32))
        n_rec = len(room.receivers)
        src = room.src_flat

        def e2e_step(n):
            lib.fdtd_b200_add_pressure(h, src, float(sig[n % len(sig)]))
            rc_ = lib.fdtd_step(h, 1)
            rc2 = lib.fdtd_sample_pressure_precomputed(h, n_rec, p_idx, p_w, p_out)
            return rc_ | rc2

        for n in range(W):
            e2e_step(n)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bad = 0
        for n in range(K):
            bad |= e2e_step(n)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        t2 = torch.tensor([el], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        el = float(t2.item())
        assert bad == 0
        e2e = {"value": room.cells * K * world / el / 1e9, "unit": METRIC,
               # per step: the source sample in (a launch argument) and the receivers out;
               # the sampler taps cross once, the engine skips re-sending unchanged taps
               "h2d_bytes_per_step": 4, "d2h_bytes_per_step": n_rec * 4,
               "h2d_once_bytes": n_rec * 8 * (8 + 4),
               "ms_per_step": el / K * 1e3,
               "path": "fdtd_b200_add_pressure + fdtd_step(st,1) + fdtd_sample_pressure_precomputed"}

    f.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(room, args.cpu_seconds)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
                "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict(room, world, kernel),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "peak_kind": f"{peak_kind} hbm_gbs",
                             "kernel": "k_fused_step" if kernel == "fused" else "k_velocity_general+k_pressure_general",
                             "kernel_ms_mean": kern_ms, "kernel_launches_timed": prof_n,
                             "algorithmic_bytes_per_launch": BYTES_PER_CELL_UPDATE * room.cells},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def gpu_uuid(local: int) -> str:
    import torch
    g = str(torch.cuda.get_device_properties(local).uuid)
    return g if g.startswith("GPU-") else "GPU-" + g


def serve_arm(args):
    """Serving 256 mixed rooms: Poisson arrivals at serve-load x the sequential capacity."""
    import torch
    from spectral_analyzer_b200 import autotune
    from spectral_analyzer_b200.serving import (BatchServer, SequentialServer, calibrate_sequential,
                                                mixed_room_requests, poisson_arrivals, request_work,
                                                summarize)
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    reqs = mixed_room_requests(args.serve_requests, seed=3, steps=(500, args.serve_max_steps))
    tune = autotune.tune_segment()
    sample = reqs[:: max(1, len(reqs) // 16)]
    service = calibrate_sequential(sample)
    rate = args.serve_load / service
    for r, t in zip(reqs, poisson_arrivals(len(reqs), rate, seed=5)):
        r.arrival = float(t)
    work = request_work(reqs)
    with ClockSampler(gpu_uuid(torch.cuda.current_device())) as clk:
        seq = SequentialServer().run(reqs)
        srv = BatchServer(max_slots=args.serve_slots, chunk=args.serve_chunk, seg_planes=tune["segment"],
                          tile_k=tune["tile"])
        bat = srv.run(reqs)
    same = all(np.array_equal(a.traces.view(np.uint32), b.traces.view(np.uint32)) for a, b in zip(seq, bat))
    s_seq, s_bat = summarize(seq, work), summarize(bat, work)
    line = {"metric": "serve requests/s", "value": s_bat["requests_per_s"], "unit": "requests/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "poisson_stream_rooms_32-256_cells_per_axis", "requests": len(reqs), "axes": "32..256 step 16",
                       "steps": [500, args.serve_max_steps], "receivers": "1..4",
                       "arrivals": "poisson", "offered_load_x_sequential": args.serve_load,
                       "arrival_rate_per_s": rate, "sequential_mean_service_s": service,
                       "slots": args.serve_slots, "chunk_steps": args.serve_chunk,
                       "segment_planes": tune["segment"], "tile_k": tune["tile"]},
            "batched": s_bat, "sequential": s_seq,
            "speedup_requests_per_s": s_bat["requests_per_s"] / s_seq["requests_per_s"],
            "traces_bit_identical": same, "max_rel_l2_vs_sequential": 0.0 if same else None,
            "autotune": tune, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0 if same else 1


def precision_timing(room, steps: int, warmup: int = 20) -> dict:
    """Device time per step of each 16-bit storage mode on both step kernels
    (CUDA events on the handle's stream, no audits), with the single pass's
    roofline on the mode's algorithmic bytes: one read and one write of the
    four fields, 2 B per value plain and 4 B compensated."""
    import torch
    from spectral_analyzer_b200.precision import BYTES_PER_VALUE, PrecisionRoom
    peak, peak_kind = measured_peak()
    out = {}
    for mode in ("bf16", "fp16", "bf16c", "fp16c"):
        row = {"bytes_per_update": 8 * BYTES_PER_VALUE[mode]}
        for kern in ("fused", "two_pass"):
            pr = PrecisionRoom(room, mode, kernel=kern, trace_capacity=steps + warmup + 4, audit_capacity=1)
            pr.step(warmup)
            torch.cuda.synchronize()
            s = pr.torch_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = pr.launch_count
            e0.record(s)
            pr.step(steps)
            e1.record(s)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            g = room.cells / ms / 1e6
            row[kern] = {"ms_per_step": ms, "gcell_updates_per_s": g, "launches": pr.launch_count - l0}
            pr.close()
        g = row["fused"]["gcell_updates_per_s"]
        achieved = g * row["bytes_per_update"]
        row["roofline_fused"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs"}
        out[mode] = row
    return out


def precision_arm(args):
    """Storage precision on the 512x384x256 room: traces and energy audit of each
    storage mode against the FP64 GPU oracle run of the same room, and the
    device time per step of the 16-bit modes on the single-pass and two-pass
    step kernels."""
    import torch
    from spectral_analyzer_b200.precision import study
    from spectral_analyzer_b200.rooms import large_room, seeded_room
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if GRID:
        room = seeded_room(*GRID, args.precision_steps, seed=2, n_rec=8, source_kind="ricker")
    else:
        room = large_room(n_steps=args.precision_steps)
    res = study(room, audit_every=args.precision_audit)
    rows = {r["mode"]: r for r in res["modes"]}
    line = {"metric": "receiver-trace rel L2 vs FP64 oracle", "value": rows["fp32"]["trace_rel_l2"],
            "unit": "rel L2 (fp32 storage)", "n_gpus": 1, "higher_is_better": False,
            "dtype": "f32 arithmetic; fp32/bf16/fp16 storage", "data": "synthetic",
            "config": {"workload": f"room{room.nx}x{room.ny}x{room.nz}_ricker_storage_precision",
                       "steps": room.n_steps, "receivers": len(room.receivers),
                       "audit_every": args.precision_audit,
                       "kernel": "16-bit modes: single-pass TMA step (fdtd_fused16.cu), two-pass on "
                                 "audit steps; FP32/FP64: two-pass (fdtd_precision.cu)"},
            "fp64_oracle": {k: v for k, v in res["fp64"].items() if k != "energy"},
            "energy_fp64": res["fp64"]["energy"],
            "modes": rows}
    if args.precision_time_steps > 0:
        line["step_time_16bit"] = precision_timing(room, args.precision_time_steps)
    print(json.dumps(line), flush=True)
    return 0


def adjoint_arm(args):
    """Gradient of the 4-receiver trace loss w.r.t. per-cell boundary absorption on
    the 128^3 room (4000 steps, checkpoints every 200): adjoint timing and central
    finite differences on 16 seeded layer cells (double forward runs).  The
    comparison with torch.autograd is a test (tests/test_adjoint_gpu.py)."""
    import torch
    from spectral_analyzer_b200.adjoint import AdjointRoom, differentiation_problem
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = GRID[0] if GRID else 128
    prob = differentiation_problem(n, n_steps=args.adjoint_steps, seed=5)
    room = AdjointRoom(prob, checkpoint_every=args.adjoint_checkpoint)
    room.set_absorption(prob.a_target)
    tgt = room.forward(keep_checkpoints=False)
    room.set_absorption(prob.a)
    room.forward()                                  # warm-up of the checkpointed forward
    g = room.backward(np.zeros((prob.n_steps, room.n_rec)))
    l0 = room.launch_count
    t0 = time.perf_counter()
    y = room.forward()
    t1 = time.perf_counter()
    g = room.backward(2.0 * (y - tgt))
    t2 = time.perf_counter()
    launches = room.launch_count - l0
    loss = float(np.sum((y - tgt) ** 2))
    t_f, t_b = t1 - t0, t2 - t1
    # central finite differences on 16 seeded layer cells, double forward runs
    dbl = AdjointRoom(prob, double=True, checkpoint_every=args.adjoint_checkpoint)
    a64 = prob.a.astype(np.float64)
    rng = np.random.default_rng(16)
    layer = np.argwhere(prob.a > 0)
    n_fd = min(args.adjoint_fd_cells, len(layer))
    cells = [tuple(int(v) for v in c) for c in layer[rng.choice(len(layer), n_fd, replace=False)]]
    fd_rows = []
    h = 1e-4
    t3 = time.perf_counter()
    for c in cells:
        ap, am = a64.copy(), a64.copy()
        ap[c] += h
        am[c] -= h
        fd = (dbl.loss(ap, tgt) - dbl.loss(am, tgt)) / (2 * h)
        fd_rows.append({"cell": list(c), "adjoint": float(g[c]), "fd": fd,
                        "rel_err": abs(float(g[c]) - fd) / abs(fd) if fd else None})
    t_fd = time.perf_counter() - t3
    fd_a = np.array([r["adjoint"] for r in fd_rows] or [0.0])
    fd_v = np.array([r["fd"] for r in fd_rows] or [1.0])
    dbl.close()
    line = {"metric": "adjoint gradient Gcell-steps/s (forward + backward)",
            "value": prob.cells * prob.n_steps / (t_f + t_b) / 1e9, "unit": "Gcell-steps/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f32 (gradient accumulated in f64)",
            "data": "synthetic",
            "config": {"workload": f"room{n}^3_boundary_absorption_gradient", "steps": prob.n_steps,
                       "receivers": len(prob.receivers), "checkpoint_every": args.adjoint_checkpoint,
                       "absorption": "GRF corr 8 cells, clipped [0.05, 0.5], 10-cell layer",
                       "targets": "float forward of the 10%-perturbed field"},
            "loss": loss, "forward_s": t_f, "backward_s": t_b, "backward_over_forward": t_b / t_f,
            "gpu_launches": launches,
            "finite_differences": {"cells": n_fd, "h": h, "forward": "double", "seconds": t_fd,
                                   "max_abs_err_over_max_abs_fd": float(np.max(np.abs(fd_a - fd_v)) / np.max(np.abs(fd_v))),
                                   "median_rel_err": float(np.median(np.abs(fd_a - fd_v) / np.abs(fd_v))),
                                   "rows": fd_rows},
            "torch_autograd": "checked in tests/test_adjoint_gpu.py (the plain-PyTorch model is a test checker)"}
    print(json.dumps(line), flush=True)
    return 0


def slab_arm(args):
    """One room split along i: torchrun ranks exchange ghost planes over NCCL
    (strong scaling of the same room); a single process steps --slabs slabs
    on one GPU with plane-copy exchanges (checks the decomposition's cost)."""
    import torch
    import torch.distributed as dist
    from spectral_analyzer_b200.slab import distributed_room, local_room
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    room = workload()
    room.n_steps = args.steps + args.warmup
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        run = distributed_room(room, rank, world, peer_memory=args.peer)
    else:
        run = local_room(room, args.slabs, peer_stores=args.peer)
    run.step(args.warmup)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = sum(s.launch_count for s in run.slabs)
    e0.record()
    run.step(args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    launches = sum(s.launch_count for s in run.slabs) - l0
    tr = run.traces(len(room.receivers))
    ms_max = float(ms.item())
    if rank == 0:
        line = {"metric": METRIC, "value": room.cells * args.steps / (ms_max / 1e3) / 1e9,
                "unit": "Gcell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong",
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": room.name, "cells": room.cells,
                           "parallelism": f"slab{world if world > 1 else args.slabs}",
                           "exchange": ("fused peer stores + " + ("NCCL one-word all-reduce barrier" if world > 1
                                                                   else "stream order")) if args.peer else
                                       ("NCCL send/recv" if world > 1 else "in-process plane copies"),
                           "kernel": ("fused single-pass kernel on slabs, one exchange per step" if run.fused
                                      else "two-pass slab kernels, two exchanges per step")},
                "gpu_launches": launches, "traces_finite": bool(np.isfinite(tr).all())}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def box_amr_grid(n: int, dx: float = 0.01, n_pml: int = 8):
    """A box of n^3 cells in the AMR solver's explicit cell/face form (cells in
    i-major order, faces x then y then z), the outer n_pml layers marked as
    PML cells (type 3); the layout a uniform region of an AMR grid has."""
    idx = np.arange(n ** 3, dtype=np.int64).reshape(n, n, n)
    ax = np.arange(n)
    I, J, K = np.meshgrid(ax, ax, ax, indexing="ij")
    centers = np.stack([(I + 0.5) * dx, (J + 0.5) * dx, (K + 0.5) * dx], axis=-1).reshape(-1, 3)
    edge = np.minimum.reduce([I, J, K, n - 1 - I, n - 1 - J, n - 1 - K]).ravel()
    types = np.where(edge < n_pml, 3, 0).astype(np.uint8)
    neg = np.concatenate([idx[:-1].ravel(), idx[:, :-1].ravel(), idx[:, :, :-1].ravel()]).astype(np.int32)
    pos = np.concatenate([idx[1:].ravel(), idx[:, 1:].ravel(), idx[:, :, 1:].ravel()]).astype(np.int32)
    nf = neg.size
    return {"cell_centers": centers, "cell_volumes": np.full(n ** 3, dx ** 3), "open_volume_frac": np.ones(n ** 3),
            "cell_types": types, "face_cell_neg": neg, "face_cell_pos": pos, "face_area": np.full(nf, dx * dx),
            "face_open_frac": np.ones(nf), "face_distance": np.full(nf, dx), "min_dx": dx,
            "bounds_min": np.zeros(3), "bounds_max": np.full(3, n * dx), "n_pml": n_pml}


def amr_arm(args):
    """AMR pressure backend throughput on a box grid (uniform region of an AMR
    grid): cell-updates/s over the step kernels (velocity + pressure; no plate),
    with the bytes one step moves per cell in this layout."""
    import torch
    from spectral_analyzer_b200.amr import AcousticAMR
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    g = box_amr_grid(args.amr_cells)
    s = AcousticAMR(g["cell_centers"], g["cell_volumes"], g["open_volume_frac"], g["cell_types"],
                    g["face_cell_neg"], g["face_cell_pos"], g["face_area"], g["face_open_frac"],
                    g["face_distance"], 343.0, 1.21, g["min_dx"], args.amr_order)
    assert s.set_border_condition(0, 3.0, 0.0, 0.0, g["n_pml"], g["bounds_min"], g["bounds_max"]) == 0
    s.inject_pressure_nearest(g["cell_centers"][len(g["cell_centers"]) // 2], 1.0)
    s.step_async(args.warmup)
    assert s.synchronize() == 0
    s.profile(True)
    l0 = s.launch_count
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.step_async(args.steps)
    rc = s.synchronize()
    wall = time.perf_counter() - t0
    ms, n = s.profile_read()
    assert rc == 0 and n == args.steps
    nc, nf = s.n_cells, s.n_faces
    entries = 2 * nf
    # algorithmic bytes per step, every array element touched once per kernel:
    # velocity: v in/out, V_damp, the gradient's operands (neg, pos, 1/d; or the
    #           8-slot stencil's cells and weights) per face, p once per cell;
    # pressure: p in/out, P_damp, P_src, 1/(V open), wall flag, CSR start per
    #           cell, CSR face and weight per entry, v once per face
    grad = (4 + 4 + 4) if args.amr_order == 2 else 8 * (4 + 4)
    face_b = nf * (4 + 4 + 4 + grad) + nf * 4
    cell_b = nc * 4 + nc * (4 + 4 + 4 + 4 + 4 + 1 + 4) + entries * (4 + 4)
    step_ms = ms / n
    peak, peak_kind = measured_peak()
    gbs = (face_b + cell_b) / (step_ms / 1e3) / 1e9
    line = {"metric": "AMR cell-updates/s", "value": nc / (step_ms / 1e3) / 1e9, "unit": "Gcell-updates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "wall_ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"amr_box{args.amr_cells}^3_order{args.amr_order}", "cells": nc, "faces": nf,
                       "border": "anechoic, 8 PML cells", "kernels": "k_amr_velocity + k_amr_pressure"},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "peak_kind": f"{peak_kind} hbm_gbs", "bytes_per_step": face_b + cell_b,
                         "bytes_per_cell_step": (face_b + cell_b) / nc},
            "gpu_launches": s.launch_count - l0}
    s.close()
    if not args.no_cpu_baseline:
        # the reference's own AMR stepper (oracle/_ref/libamr_ref.so, its thread pool) on the same grid
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from amr_oracle import AMRRef
        g["n_cells"], g["n_faces"], g["c"], g["rho_air"] = nc, nf, 343.0, 1.21
        r = AMRRef(g, gradient_order=args.amr_order, border=(0, 3.0, 0.0, 0.0))
        r.step_rc(1)
        n_cpu, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < args.cpu_seconds and n_cpu < 2000:
            assert r.step_rc(1) == 0
            n_cpu += 1
        el = time.perf_counter() - t0
        r.close()
        line["cpu_baseline"] = {"value": nc * n_cpu / el / 1e9, "unit": "Gcell-updates/s",
                                "cores": os.cpu_count(), "kind": "reference",
                                "sample": f"{n_cpu} steps of the same grid ({el:.1f} s wall, libamr_ref.so, "
                                          "its thread pool over all host cores)"}
    print(json.dumps(line), flush=True)
    return 0


def launch_ranks(n: int, argv) -> int:
    """Re-run this script as n ranks (torch.distributed.run, one GPU each) when
    it was started without a launcher; returns the launcher's exit code."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *argv]
    try:
        return subprocess.call(cmd, timeout=3600)
    except subprocess.TimeoutExpired:
        return 124


def walled_arm(args):
    """A body scene (back and rib walls, a plate with a soundhole, cut-cell face
    fractions, bridge sources) stepped by the two-pass kernels and by the walled
    single pass.  Per kernel: the step kernels' CUDA-event time per step (the
    profile window: velocity + pressure, or the single pass + plate faces +
    recomputed plate-face neighbours) and the wall time of fdtd_step(st, n),
    which also runs the plate update and its guard read-back every step."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from scenes import body_scene
    from spectral_analyzer_b200 import AcousticFDTD
    dims = GRID or (512, 384, 256)
    sc = body_scene(*dims, seed=4, n_pml=10)
    cells = dims[0] * dims[1] * dims[2]
    peak, peak_kind = measured_peak()
    rows = {}
    with ClockSampler(gpu_uuid(int(os.environ.get("LOCAL_RANK", "0")))) as clk:
        for kernel in ("two_pass", "fused"):
            f = AcousticFDTD(**sc.kwargs())
            f.set_kernel(kernel)
            f.set_face_fractions(*sc.fracs)
            f.set_bridge_sources(sc.bridge_idx, sc.bridge_wgt)
            f.step(10)
            torch.cuda.synchronize()
            f.profile(True)
            t0 = time.perf_counter()
            f.step(args.walled_steps)
            torch.cuda.synchronize()
            wall = (time.perf_counter() - t0) / args.walled_steps
            ms, n, nk = f.profile_read()
            kern_ms = ms / n
            rows[kernel] = {"kernel_ms_per_step": kern_ms, "wall_ms_per_step": wall * 1e3,
                            "gcell_updates_per_s_kernels": cells / kern_ms / 1e6,
                            "gcell_updates_per_s_wall": cells / wall / 1e9, "launches": f.launch_count}
            f.close()
    bpu = 45   # P, Vx, Vy, Vz read and written (32 B), three face fractions (12 B), solid mask (1 B)
    achieved = rows["fused"]["gcell_updates_per_s_kernels"] * bpu
    line = {"metric": "Gcell-updates/s (walled scene, step kernels)", "value": rows["fused"]["gcell_updates_per_s_kernels"],
            "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.walled_steps, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"body_scene{dims[0]}x{dims[1]}x{dims[2]}_walls_fractions_plate",
                       "cells": cells, "plate_nodes": int(sc.kwargs()["plate_active"].sum())},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                         "kernel": "walled single pass (k_fused_step walls + plate faces + k_pressure_groups)",
                         "algorithmic_bytes_per_update": bpu},
            "kernels": rows, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def split_line(args, world, ms_max, e2e, launches, clocks, own_cells, cells, kind):
    """The JSON line of an N-rank split-room run (rank 0 prints it)."""
    step_ms = ms_max / args.steps
    achieved = BYTES_PER_CELL_UPDATE * own_cells / (step_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    return {"metric": METRIC, "value": cells * args.steps / (ms_max / 1e3) / 1e9, "unit": METRIC,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": kind,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": f"{peak_kind} hbm_gbs",
                         "kernel": "one rank's whole step (both parts of the fused slab step, the ghost "
                                   "exchange overlapped with the interior, receivers)",
                         "algorithmic_bytes_per_step_per_rank": BYTES_PER_CELL_UPDATE * own_cells},
            "cpu_baseline": None, "e2e": e2e, "gpu_launches": launches, "clocks": clocks}


def split_arm(args):
    """N>1 ranks (torchrun, NCCL): the 512x384x256 room split along i into N
    slabs (strong scaling).  Each step: the planes the neighbours keep as ghosts,
    then the interior while 3 P planes and 2 Vx faces per side travel to the
    neighbours over NCCL on a side stream, then the receivers.  value = the
    room's cells x steps over the slowest rank's device time; e2e = the same with
    the source sample given by the host every step (a launch argument) and each
    rank's receiver samples read back every step."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ["WORLD_SIZE"])
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from spectral_analyzer_b200.slab import distributed_room
    room = workload()
    K, W = args.steps, args.warmup
    room.n_steps = W + 2 * K + 1
    run = distributed_room(room, rank, world, overlap=True)
    slab = run.slabs[0]
    run.step(W)
    dist.barrier()
    torch.cuda.synchronize()
    l0 = slab.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_uuid(local)) as clk:
        e0.record()
        run.step(K)
        e1.record()
        torch.cuda.synchronize()
    launches = slab.launch_count - l0
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    # end to end: host source sample in, this rank's receiver samples out, every step
    sig = room.signal()
    out = np.zeros(len(slab.rec_ids), np.float32)
    dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        run.step(1, host_sample=lambda q: float(sig[q % len(sig)]))
        if out.size:
            slab.read_last(out)
    torch.cuda.synchronize()
    t2 = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    el = float(t2.item())
    n_rec_all = torch.tensor([out.size], dtype=torch.int64, device="cuda")
    dist.all_reduce(n_rec_all)
    e2e = {"value": room.cells * K / el / 1e9, "unit": METRIC, "h2d_bytes_per_step": 4 * world,
           "d2h_bytes_per_step": 4 * int(n_rec_all.item()), "ms_per_step": el / K * 1e3,
           "path": "per rank: fdtd_b200_slab_add_pressure (host sample) + slab step + exchange + "
                   "record + fdtd_b200_slab_read_last"}
    finite = bool(np.isfinite(run.traces(len(room.receivers))).all())
    if rank == 0:
        kind = dict(config_dict(room, world, "fused"), parallelism=f"slab{world}",
                    exchange="NCCL send/recv of 3 P planes + 2 Vx faces per side, side stream, "
                             "overlapped with the interior planes")
        line = split_line(args, world, ms_max, e2e, launches, clk.summary(), slab.own * room.ny * room.nz,
                          room.cells, kind)
        line["traces_finite"] = finite
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def plumbing_check(args):
    """No GPU: the launch, the gloo rendezvous, the max-over-ranks timing and the
    JSON line of a split run, with a host stand-in for the step (checks the
    bench's multi-rank plumbing on a CPU box; prints no measurement)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    from spectral_analyzer_b200.slab import partition
    room = workload()
    a, b = partition(room.nx, world)[rank]
    t0 = time.perf_counter()
    x = np.zeros(((b - a), 8, 8), np.float32)
    for _ in range(args.steps):
        x += 1.0
        dist.barrier()
    t = torch.tensor([1e3 * (time.perf_counter() - t0)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        kind = dict(config_dict(room, world, "plumbing-check"), parallelism=f"slab{world}")
        line = split_line(args, world, float(t.item()), None, 0, None, (b - a) * room.ny * room.nz,
                          room.cells, kind)
        line["plumbing_check"] = True
        print(json.dumps(line), flush=True)
    dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "engine" and args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus, sys.argv[1:])
    if args.plumbing_check:
        return plumbing_check(args)
    if args.impl == "reference":
        return reference_arm(args)
    if args.serve:
        return serve_arm(args)
    if args.precision:
        return precision_arm(args)
    if args.adjoint:
        return adjoint_arm(args)
    if args.decompose:
        return slab_arm(args)
    if args.amr:
        return amr_arm(args)
    if args.walled:
        return walled_arm(args)
    if world > 1 and args.scale_mode == "split":
        return split_arm(args)
    return engine_arm(args)


if __name__ == "__main__":
    sys.exit(main())
