"""A NumPy slab of the open-room step, for testing the slab decomposition's
exchange schedule on CPU ranks (gloo).  Same interface and arithmetic as the
CUDA slab (every float32 operation separately rounded, the reference's
operand order: csrc/kernels/acoustic_fdtd.cpp:1099-1148, :894-952,
:1176-1234, :216-222, :469-476, :536-561), so its results are compared with
the oracle bit for bit.  Test infrastructure only."""
import numpy as np
import torch

from spectral_analyzer_b200.precision import pressure_taps
from spectral_analyzer_b200.slab import GHOST

f32 = np.float32


def _sigma(d, n_pml, dt, scale):
    if n_pml <= 0 or d <= 0:
        return f32(0)
    frac = f32(d) / f32(n_pml)
    smax = f32(scale) * (f32(3.45) / (dt * f32(n_pml)))
    return smax * frac * frac * frac


def _axis(i, n, n_pml, dt, lo, hi):
    if i < n_pml:
        return _sigma(n_pml - i, n_pml, dt, lo)
    if i >= n - n_pml:
        return _sigma(i - (n - n_pml) + 1, n_pml, dt, hi)
    return f32(0)


class NumpySlab:
    def __init__(self, room, i0, i1, rec_ids, fused=False):
        self.room, self.i0, self.i1, self.own = room, i0, i1, i1 - i0
        self.fused = fused
        self.L = self.own + 2 * GHOST
        self.x0 = i0 - GHOST
        ny, nz = room.ny, room.nz
        self.P = [np.zeros((self.L, ny, nz), f32) for _ in range(2)]
        self.V = [np.zeros((self.L, ny, nz), f32) for _ in range(3)]
        self.cur = 0
        self.dt = f32(0.77) * f32(room.dx) / (f32(room.c) * f32(1.732050808))
        self.vc = self.dt / (f32(room.rho) * f32(room.dx))
        self.bulk = f32(room.rho) * f32(room.c) * f32(room.c) * self.dt * (f32(1) / f32(room.dx))
        a6 = [f32(v) for v in room.absorption]
        np_ = room.n_pml
        self.ax = np.array([_axis(self.x0 + l, room.nx, np_, self.dt, a6[0], a6[1])
                            if 0 <= self.x0 + l < room.nx else f32(0) for l in range(self.L)], f32)
        self.ay = np.array([_axis(j, ny, np_, self.dt, a6[2], a6[3]) for j in range(ny)], f32)
        self.az = np.array([_axis(k, nz, np_, self.dt, a6[4], a6[5]) for k in range(nz)], f32)
        pd = lambda a: f32(1) / (f32(1) + a * self.dt)
        self.px, self.py, self.pz = pd(self.ax), pd(self.ay), pd(self.az)
        self.sig = np.asarray(room.signal(), f32)
        s = room.src
        self.src = (s[0] - self.x0, s[1], s[2]) if 0 <= s[0] - self.x0 < self.L else None
        idx, w = pressure_taps(room.nx, room.ny, room.nz, room.receiver_xyz())
        self.rec_ids = list(rec_ids)
        self.taps = [(idx[8 * r:8 * r + 8], w[8 * r:8 * r + 8]) for r in self.rec_ids]
        self.rows = []
        self.c1, self.c2 = f32(9) / f32(8), f32(-1) / f32(24)

    def field(self, name):
        if name == "P":
            return torch.from_numpy(self.P[self.cur])
        return torch.from_numpy(self.V[{"Vx": 0, "Vy": 1, "Vz": 2}[name]])

    def deposit(self, n):
        if self.src is not None and n < self.sig.size and self.sig[n] != 0:
            p = self.P[self.cur]
            p[self.src] = p[self.src] + self.sig[n]

    def _alpha(self, l_sl, j_sl, k_sl):
        return np.maximum(np.maximum(self.ax[l_sl][:, None, None], self.ay[j_sl][None, :, None]),
                          self.az[k_sl][None, None, :])

    def _grad(self, p, axis, lo, hi, n, g0):
        """Gradient on faces lo..hi-1 along axis; g0 = global index of position 0."""
        sl = lambda a, b: np.take(p, np.arange(a, b), axis=axis)
        f = np.arange(lo, hi) + g0
        g2 = sl(lo + 1, hi + 1) - sl(lo, hi)
        inner = (f > 0) & (f < n - 2)
        a = np.clip(np.arange(lo - 1, hi - 1), 0, p.shape[axis] - 1)
        b = np.clip(np.arange(lo + 2, hi + 2), 0, p.shape[axis] - 1)
        g4 = self.c1 * (sl(lo + 1, hi + 1) - sl(lo, hi)) + self.c2 * (np.take(p, b, axis) - np.take(p, a, axis))
        shape = [1, 1, 1]
        shape[axis] = -1
        return np.where(inner.reshape(shape), g4, g2)

    def velocity(self, x_lo=None, x_hi=None):
        """New V of the own planes; x faces on local planes [x_lo, x_hi) (own by default)."""
        room, p = self.room, self.P[self.cur]
        ny, nz, own, x0 = room.ny, room.nz, self.own, self.x0
        lo, hi = GHOST, GHOST + own
        x_lo = lo if x_lo is None else x_lo
        x_hi = hi if x_hi is None else x_hi
        ac = self._alpha(slice(lo, hi), slice(0, ny), slice(0, nz))
        dt, vc = self.dt, self.vc
        damp = lambda aL, aR: f32(1) - (f32(0.5) * (aL + aR)) * dt
        vx, vy, vz = self.V
        # x faces that exist globally
        ig = np.arange(x_lo, x_hi) + x0
        gx = self._grad(p, 0, x_lo, x_hi, room.nx, x0)
        acx = self._alpha(slice(x_lo, x_hi), slice(0, ny), slice(0, nz))
        ar = self._alpha(slice(x_lo + 1, x_hi + 1), slice(0, ny), slice(0, nz))
        new = (vx[x_lo:x_hi] - vc * gx) * damp(acx, ar)
        ok = ((ig >= 0) & (ig < room.nx - 1))[:, None, None]
        vx[x_lo:x_hi] = np.where(ok, new, vx[x_lo:x_hi])
        # y faces j < ny-1
        gy = self._grad(p[lo:hi], 1, 0, ny - 1, ny, 0)
        ar = self._alpha(slice(lo, hi), slice(1, ny), slice(0, nz))
        vy[lo:hi, : ny - 1] = (vy[lo:hi, : ny - 1] - vc * gy) * damp(ac[:, : ny - 1], ar)
        gz = self._grad(p[lo:hi], 2, 0, nz - 1, nz, 0)
        ar = self._alpha(slice(lo, hi), slice(0, ny), slice(1, nz))
        vz[lo:hi, :, : nz - 1] = (vz[lo:hi, :, : nz - 1] - vc * gz) * damp(ac[:, :, : nz - 1], ar)

    def step(self):
        """The fused kernel's step: x faces two left and one right of the own
        planes recomputed from ghost P and ghost old Vx, then the pressure."""
        self.velocity(GHOST - 2, GHOST + self.own + 1)
        self.pressure()

    def pressure(self):
        room, p = self.room, self.P[self.cur]
        ny, nz, own, x0 = room.ny, room.nz, self.own, self.x0
        lo, hi = GHOST, GHOST + own
        vx, vy, vz = self.V
        ig = (np.arange(lo, hi) + x0)[:, None, None]
        z = np.zeros((own, ny, nz), f32)
        xp = np.where(ig < room.nx - 1, vx[lo:hi], z)
        xm = np.where(ig > 0, vx[lo - 1:hi - 1], z)
        xpp = np.where(ig < room.nx - 2, vx[lo + 1:hi + 1], z)
        xmm = np.where(ig > 1, vx[lo - 2:hi - 2], z)

        def axis_terms(v, axis, n):
            t = np.arange(n)
            pad = [(0, 0)] * 3
            pad[axis] = (2, 3)
            vp = np.pad(v[lo:hi], pad)          # vp[t + 2] = v[t] on faces 0..n-2, zero elsewhere
            mask = [1, 1, 1]
            mask[axis] = -1
            keep = (t < n - 1).reshape(mask)
            vp_t = np.take(vp, np.arange(2, n + 2), axis)
            vp_t = np.where(keep, vp_t, f32(0))
            vp_m = np.where((t > 0).reshape(mask), np.take(vp, np.arange(1, n + 1), axis), f32(0))
            vp_pp = np.where((t < n - 2).reshape(mask), np.take(vp, np.arange(3, n + 3), axis), f32(0))
            vp_mm = np.where((t > 1).reshape(mask), np.take(vp, np.arange(0, n), axis), f32(0))
            return vp_t, vp_m, vp_pp, vp_mm

        yp, ym, ypp, ymm = axis_terms(vy, 1, ny)
        zp, zm, zpp, zmm = axis_terms(vz, 2, nz)
        d1 = ((xp - xm) + (yp - ym)) + (zp - zm)
        d2 = ((xpp - xmm) + (ypp - ymm)) + (zpp - zmm)
        dv = self.c1 * d1 + self.c2 * d2
        pd = np.minimum(np.minimum(self.px[lo:hi][:, None, None], self.py[None, :, None]), self.pz[None, None, :])
        pn = self.P[self.cur ^ 1]
        pn[lo:hi] = (p[lo:hi] - self.bulk * dv) * pd
        self.cur ^= 1

    def record(self):
        p = self.P[self.cur]
        ny, nz = self.room.ny, self.room.nz
        row = []
        for idx, w in self.taps:
            vals = []
            for q in idx:
                k, j, ig = q % nz, (q // nz) % ny, q // (ny * nz)
                vals.append(p[ig - self.x0, j, k])
            s = w[0] * vals[0]
            for t in range(1, 8):
                s = f32(s + w[t] * vals[t])
            row.append(s)
        self.rows.append(np.array(row, f32))

    def check(self, phase):
        ny, nz = self.room.ny, self.room.nz
        per = ny * nz
        q_lo, q_hi = self.i0 * per, self.i1 * per
        q = phase
        if q < q_lo:
            q += -(-(q_lo - q) // 1013) * 1013
        p = self.P[self.cur]
        while q < q_hi:
            v = p[q // per - self.x0, (q // nz) % ny, q % nz]
            if not np.isfinite(v) or abs(v) > 2e3:
                return q
            q += 1013
        return -1

    def traces(self):
        n = len(self.rec_ids)
        return np.array(self.rows, f32).reshape(len(self.rows), n)

    def own_pressure(self):
        return self.P[self.cur][GHOST:GHOST + self.own].copy()
