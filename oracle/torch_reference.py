"""Plain PyTorch restatement of the per-cell-absorption room, differentiated by
torch.autograd: the reference the adjoint kernels are checked against.
Test infrastructure only (imported by tests/ as a checker, never by the
engine).

Same model as fdtd_adjoint.cu (the reference's update,
csrc/kernels/acoustic_fdtd.cpp:1099-1148 and :894-952/:1176-1234, with
alpha*dt given per cell): source added before each step, velocity update
with 4th-order gradient on interior faces and 2nd-order on the first and
last face, pressure update with the zero-extended 4th-order divergence,
damping 1/(1+a) on cells and 1-(a_L+a_R)/2 on faces, 8-tap receivers after
each step.  Steps are grouped into checkpointed segments
(torch.utils.checkpoint) so that long runs fit in memory.
"""
from __future__ import annotations

import numpy as np

C1, C2 = 9.0 / 8.0, -1.0 / 24.0


def _grad(p, axis):
    n = p.shape[axis]
    sl = lambda a, b: p.narrow(axis, a, b - a)
    g2 = sl(1, n) - sl(0, n - 1)                                   # faces 0..n-2
    if n < 4:
        return g2
    g4 = C1 * (sl(2, n - 1) - sl(1, n - 2)) + C2 * (sl(3, n) - sl(0, n - 3))   # faces 1..n-3
    import torch
    return torch.cat([g2.narrow(axis, 0, 1), g4, g2.narrow(axis, n - 2, 1)], dim=axis)


def _pad(v, axis):
    import torch.nn.functional as F
    pad = [0, 0] * 3
    pad[2 * (2 - axis)] = 2       # F.pad lists the last dimension first
    pad[2 * (2 - axis) + 1] = 3
    return F.pad(v, pad)


def _div(vx, vy, vz, shape):
    d1 = 0
    d2 = 0
    for axis, v in enumerate((vx, vy, vz)):
        n = shape[axis]
        vp = _pad(v, axis)                 # vp[t + 2] = v[t], zero outside the faces
        sl = lambda a: vp.narrow(axis, a, n)
        d1 = d1 + (sl(2) - sl(1))
        d2 = d2 + (sl(3) - sl(0))
    return C1 * d1 + C2 * d2


def _face_damp(a, axis):
    n = a.shape[axis]
    return 1.0 - 0.5 * (a.narrow(axis, 0, n - 1) + a.narrow(axis, 1, n - 1))


def traces(a, prob, idx8, w8, dtype=None, segment: int = 200):
    """Receiver traces (n_steps, n_rec) of the room with absorption a (tensor)."""
    import torch
    from torch.utils.checkpoint import checkpoint
    dtype = dtype or a.dtype
    dev = a.device
    a = a.to(dtype)
    nx, ny, nz = prob.shape
    dt = 0.77 * prob.dx / (prob.c * 1.732050808)
    vc = dt / (prob.rho * prob.dx)
    bulk = prob.rho * prob.c * prob.c * dt * (1.0 / prob.dx)
    q = 1.0 / (1.0 + a)
    dmp = [_face_damp(a, ax) for ax in range(3)]
    sig = torch.as_tensor(np.asarray(prob.signal(), np.float64), dtype=dtype, device=dev)
    src = prob.flat(prob.src)
    idx = torch.as_tensor(np.asarray(idx8, np.int64), device=dev)
    w = torch.as_tensor(np.asarray(w8, np.float64), dtype=dtype, device=dev)
    n_rec = idx.numel() // 8
    onehot = torch.zeros(nx * ny * nz, dtype=dtype, device=dev)
    onehot[src] = 1.0
    onehot = onehot.reshape(nx, ny, nz)

    def run(n0, n1, p, vx, vy, vz, *damp):
        q_, dx_, dy_, dz_ = damp
        rows = []
        for n in range(n0, n1):
            if n < sig.numel():
                p = p + sig[n] * onehot
            vx = (vx - vc * _grad(p, 0)) * dx_
            vy = (vy - vc * _grad(p, 1)) * dy_
            vz = (vz - vc * _grad(p, 2)) * dz_
            p = (p - bulk * _div(vx, vy, vz, (nx, ny, nz))) * q_
            rows.append((p.reshape(-1)[idx] * w).reshape(n_rec, 8).sum(1))
        return (p, vx, vy, vz, torch.stack(rows))

    p = torch.zeros((nx, ny, nz), dtype=dtype, device=dev)
    vx = torch.zeros((nx - 1, ny, nz), dtype=dtype, device=dev)
    vy = torch.zeros((nx, ny - 1, nz), dtype=dtype, device=dev)
    vz = torch.zeros((nx, ny, nz - 1), dtype=dtype, device=dev)
    out = []
    for n0 in range(0, prob.n_steps, segment):
        n1 = min(n0 + segment, prob.n_steps)
        p, vx, vy, vz, rows = checkpoint(run, n0, n1, p, vx, vy, vz, q, *dmp, use_reentrant=False)
        out.append(rows)
    return torch.cat(out)


def loss_and_grad(a_np, prob, idx8, w8, targets, device="cuda", dtype=None, segment: int = 200):
    """(L, dL/da) by torch.autograd, in float64 unless dtype says otherwise."""
    import torch
    dtype = dtype or torch.float64
    a = torch.as_tensor(np.asarray(a_np), dtype=dtype, device=device).requires_grad_(True)
    y = traces(a, prob, idx8, w8, dtype, segment)
    t = torch.as_tensor(np.asarray(targets), dtype=dtype, device=device)
    loss = ((y - t) ** 2).sum()
    loss.backward()
    return float(loss.detach()), a.grad.detach().cpu().numpy()
