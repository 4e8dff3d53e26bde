/*
 * fdtd_adjoint.cu — gradient of a receiver-trace loss with respect to a
 * per-cell absorption field, by the discrete adjoint of the open-room step.
 *
 * Forward (the reference's update with its PML profile replaced by a per-cell
 * field a_c = alpha_c * dt, as csrc/kernels/acoustic_fdtd.cpp:64 and :387-389
 * store alpha per cell; damping as :469-476 and :536-561):
 *   p~^n       = p^n + s[n] e_src                                (source)
 *   v^{n+1/2}  = (v^{n-1/2} - vc G p~^n) (.) d,  d_f = 1 - (a_L + a_R)/2
 *   p^{n+1}    = (p~^n - bulk D v^{n+1/2}) (.) q,  q_c = 1 / (1 + a_c)
 *   y^n        = R p^{n+1}                                       (receivers)
 * with G the gradient (4th order on interior faces, 2nd order on the first
 * and last face, acoustic_fdtd.cpp:1099-1148) and D the divergence (4th order
 * with zero velocity outside the faces, :894-952).
 *
 * Reverse step n, given Lp = dL/dp~^{n+1} and Lv = dL/dv^{n+1/2} (partial,
 * through step n+1's velocity update) and r^n = dL/dy^n:
 *   lam  = Lp + R^T r^n                        (inside k_adj_cells1)
 *   U    = lam (.) q ;  g_c -= q_c^2 lam_c z_c, z = p~^n - bulk D v^{n+1/2}   (k_adj_cells1)
 *   mu   = Lv - bulk D^T U ;  W = mu (.) d ;  E_f = mu_f y_f,
 *          y = v^{n-1/2} - vc G p~^n ;  Lv <- W                            (k_adj_faces)
 *   Lp  <- U - vc G^T W ;  g_c -= 1/2 sum_{faces f of c} E_f               (k_adj_cells2)
 * Gradients accumulate in double.  The forward is recomputed segment by
 * segment from checkpoints (p~^n and v^{n-1/2} every K steps) into K+1
 * device slots, so the reverse sweep reads every state it needs from HBM.
 * Launches per step: forward 3 (velocity, pressure, an epilogue that records
 * the receivers and then adds the next step's source sample), recompute 2
 * (the pressure kernel adds the next sample), reverse 3.
 * Each sweep (forward, forward with checkpoints, backward) is captured once
 * as a CUDA graph and replayed while its length and buffers stay the same:
 * a gradient evaluation is then two graph launches.
 *
 * All kernels are templated on the working type R (float: the product path;
 * double: for finite-difference checks).  Every operation is separately
 * rounded (no contraction), so the float forward equals the reference's
 * arithmetic on the same absorption field bit for bit.
 */
#include "acoustic_fdtd_b200.h"
#include "fdtd_internal.h"

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

namespace fdtd {
namespace adj {

__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rrcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rrcp(double a) { return __drcp_rn(a); }

template <class R>
struct ACoef {
    R vc, bulk, c1, c2;
};

template <class R>
__device__ __forceinline__ R face_d(R aL, R aR) { return rsub(R(1), rmul(R(0.5), radd(aL, aR))); }
template <class R>
__device__ __forceinline__ R cell_q(R a) { return rrcp(radd(R(1), a)); }

// Gradient on face f = cell c's "+" face along an axis of n cells, at stride s.
template <class R>
__device__ __forceinline__ R grad_face(const R* p, long long id, long long s, int f, int n, const ACoef<R>& cf)
{
    const R pr = p[id + s], pc = p[id];
    if (f > 0 && f < n - 2)
        return radd(rmul(cf.c1, rsub(pr, pc)), rmul(cf.c2, rsub(p[id + 2 * s], p[id - s])));
    return rsub(pr, pc);
}

// Divergence at cell c (index t along each axis), zero velocity outside faces.
template <class R>
__device__ __forceinline__ R div_cell(const Grid& g, const R* vx, const R* vy, const R* vz, long long id,
                                      int i, int j, int k, const ACoef<R>& cf)
{
    const long long P = g.plane, S = g.sz;
    const R z0 = R(0);
    const R xp = (i < g.nx - 1) ? vx[id] : z0, xm = (i > 0) ? vx[id - P] : z0;
    const R xpp = (i < g.nx - 2) ? vx[id + P] : z0, xmm = (i > 1) ? vx[id - 2 * P] : z0;
    const R yp = (j < g.ny - 1) ? vy[id] : z0, ym = (j > 0) ? vy[id - S] : z0;
    const R ypp = (j < g.ny - 2) ? vy[id + S] : z0, ymm = (j > 1) ? vy[id - 2 * S] : z0;
    const R zp = (k < g.nz - 1) ? vz[id] : z0, zm = (k > 0) ? vz[id - 1] : z0;
    const R zpp = (k < g.nz - 2) ? vz[id + 1] : z0, zmm = (k > 1) ? vz[id - 2] : z0;
    const R d1 = radd(radd(rsub(xp, xm), rsub(yp, ym)), rsub(zp, zm));
    const R d2 = radd(radd(rsub(xpp, xmm), rsub(ypp, ymm)), rsub(zpp, zmm));
    return radd(rmul(cf.c1, d1), rmul(cf.c2, d2));
}

// Transposed divergence on face f of an axis with n cells, u at stride s.
template <class R>
__device__ __forceinline__ R divT_face(const R* u, long long id, long long s, int f, int n, const ACoef<R>& cf)
{
    R t = rmul(cf.c1, rsub(u[id], u[id + s]));
    const R um = (f >= 1) ? u[id - s] : R(0);
    const R upp = (f <= n - 3) ? u[id + 2 * s] : R(0);
    return radd(t, rmul(cf.c2, rsub(um, upp)));
}

// Transposed gradient at cell t of an axis with n cells (faces 0..n-2), w at stride s.
template <class R>
__device__ __forceinline__ R gradT_cell(const R* w, long long id, long long s, int t, int n, const ACoef<R>& cf)
{
    R acc = R(0);
    const int nf = n - 1;   // faces 0..n-2
    auto inner = [&](int f) { return f > 0 && f < n - 2; };
    if (t - 1 >= 0 && t - 1 < nf) acc = radd(acc, rmul(inner(t - 1) ? cf.c1 : R(1), w[id - s]));
    if (t < nf) acc = rsub(acc, rmul(inner(t) ? cf.c1 : R(1), w[id]));
    if (t - 2 >= 0 && inner(t - 2)) acc = radd(acc, rmul(cf.c2, w[id - 2 * s]));
    if (t + 1 < nf && inner(t + 1)) acc = rsub(acc, rmul(cf.c2, w[id + s]));
    return acc;
}

#define ADJ_INDEX                                                        \
    const int k = blockIdx.x * blockDim.x + threadIdx.x;                 \
    const int j = blockIdx.y * blockDim.y + threadIdx.y;                 \
    const int i = blockIdx.z;                                            \
    if (k >= g.nz || j >= g.ny) return;                                  \
    const long long id = ((long long)i * g.ny + j) * g.sz + k;

// Four consecutive values at an index that is a multiple of 4 (rows start on
// 8-element boundaries, so the access is aligned).
template <class R>
__device__ __forceinline__ void ld4r(const R* p, long long i, R (&v)[4])
{
    if constexpr (sizeof(R) == 4) {
        const float4 x = *reinterpret_cast<const float4*>(p + i);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
        const double2 x = *reinterpret_cast<const double2*>(p + i);
        const double2 y = *reinterpret_cast<const double2*>(p + i + 2);
        v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
    }
}
template <class R>
__device__ __forceinline__ void st4r(R* p, long long i, const R (&v)[4])
{
    if constexpr (sizeof(R) == 4) {
        *reinterpret_cast<float4*>(p + i) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        *reinterpret_cast<double2*>(p + i) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(p + i + 2) = make_double2(v[2], v[3]);
    }
}

// Threads own four consecutive cells k0 .. k0+3 of a row; every per-cell
// expression below is the scalar one of the helpers above, in the same order.
#define ADJ4_INDEX                                                       \
    const int k0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);          \
    const int j = blockIdx.y * blockDim.y + threadIdx.y;                 \
    const int i = blockIdx.z;                                            \
    if (k0 >= g.nz || j >= g.ny) return;                                 \
    const long long id = ((long long)i * g.ny + j) * g.sz + k0;

// Gradient on the faces of the four cells along x or y (stride s, face index f,
// n cells on that axis): grad_face for each cell.
template <class R>
__device__ __forceinline__ void grad4(const R* p, long long id, long long s, int f, int n, const ACoef<R>& cf,
                                      const R (&pc)[4], R (&gr)[4])
{
    R pr[4], pm[4], p2[4];
    ld4r(p, id + s, pr);
    if (f > 0 && f < n - 2) {
        ld4r(p, id - s, pm);
        ld4r(p, id + 2 * s, p2);
#pragma unroll
        for (int q = 0; q < 4; ++q) gr[q] = radd(rmul(cf.c1, rsub(pr[q], pc[q])), rmul(cf.c2, rsub(p2[q], pm[q])));
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) gr[q] = rsub(pr[q], pc[q]);
    }
}

// P (or any cell field) at k0-1 .. k0+5: e[t] = f[k0 - 1 + t], zero outside the row.
template <class R>
__device__ __forceinline__ void zrow(const R* f, long long id, int k0, int nz, const R (&c)[4], R (&e)[7])
{
    e[0] = k0 > 0 ? f[id - 1] : R(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) e[q + 1] = c[q];
    e[5] = k0 + 4 < nz ? f[id + 4] : R(0);
    e[6] = k0 + 5 < nz ? f[id + 5] : R(0);
}

// z-face gradient of cell k = k0+q from e (zrow of P): grad_face along z.
template <class R>
__device__ __forceinline__ R gradz(const R (&e)[7], int q, int k, int nz, const ACoef<R>& cf)
{
    if (k > 0 && k < nz - 2) return radd(rmul(cf.c1, rsub(e[q + 2], e[q + 1])), rmul(cf.c2, rsub(e[q + 3], e[q])));
    return rsub(e[q + 2], e[q + 1]);
}

// Divergence of the four cells (div_cell for each).
template <class R>
__device__ __forceinline__ void div4(const Grid& g, const R* vx, const R* vy, const R* vz, long long id, int i,
                                     int j, int k0, const ACoef<R>& cf, R (&dv)[4])
{
    const long long P = g.plane, S = g.sz;
    R xp[4] = {}, xm[4] = {}, xpp[4] = {}, xmm[4] = {}, yp[4] = {}, ym[4] = {}, ypp[4] = {}, ymm[4] = {};
    if (i < g.nx - 1) ld4r(vx, id, xp);
    if (i > 0) ld4r(vx, id - P, xm);
    if (i < g.nx - 2) ld4r(vx, id + P, xpp);
    if (i > 1) ld4r(vx, id - 2 * P, xmm);
    if (j < g.ny - 1) ld4r(vy, id, yp);
    if (j > 0) ld4r(vy, id - S, ym);
    if (j < g.ny - 2) ld4r(vy, id + S, ypp);
    if (j > 1) ld4r(vy, id - 2 * S, ymm);
    R zc[4], ez[7];   // ez[t] = Vz[k0 - 2 + t]
    ld4r(vz, id, zc);
    ez[0] = k0 >= 2 ? vz[id - 2] : R(0);
    ez[1] = k0 >= 1 ? vz[id - 1] : R(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) ez[q + 2] = zc[q];
    ez[6] = k0 + 4 < g.nz ? vz[id + 4] : R(0);
    const R z0 = R(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = k0 + q;
        const R zp = (k < g.nz - 1) ? ez[q + 2] : z0, zm = (k > 0) ? ez[q + 1] : z0;
        const R zpp = (k < g.nz - 2) ? ez[q + 3] : z0, zmm = (k > 1) ? ez[q] : z0;
        const R d1 = radd(radd(rsub(xp[q], xm[q]), rsub(yp[q], ym[q])), rsub(zp, zm));
        const R d2 = radd(radd(rsub(xpp[q], xmm[q]), rsub(ypp[q], ymm[q])), rsub(zpp, zmm));
        dv[q] = radd(rmul(cf.c1, d1), rmul(cf.c2, d2));
    }
}

template <class R>
__global__ void __launch_bounds__(256) k_fwd_vel(Grid g, ACoef<R> cf, const R* __restrict__ a,
                                                 const R* __restrict__ p, const R* vin0, const R* vin1,
                                                 const R* vin2, R* vout0, R* vout1, R* vout2)
{
    ADJ4_INDEX
    R ac[4], pc[4];
    ld4r(a, id, ac);
    ld4r(p, id, pc);
    if (i < g.nx - 1) {
        R gr[4], ar[4], v[4];
        grad4(p, id, g.plane, i, g.nx, cf, pc, gr);
        ld4r(a, id + g.plane, ar);
        ld4r(vin0, id, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (k0 + q < g.nz) v[q] = rmul(rsub(v[q], rmul(cf.vc, gr[q])), face_d(ac[q], ar[q]));
        st4r(vout0, id, v);
    }
    if (j < g.ny - 1) {
        R gr[4], ar[4], v[4];
        grad4(p, id, (long long)g.sz, j, g.ny, cf, pc, gr);
        ld4r(a, id + g.sz, ar);
        ld4r(vin1, id, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (k0 + q < g.nz) v[q] = rmul(rsub(v[q], rmul(cf.vc, gr[q])), face_d(ac[q], ar[q]));
        st4r(vout1, id, v);
    }
    {
        R e[7], v[4];
        zrow(p, id, k0, g.nz, pc, e);
        const R a4 = k0 + 4 < g.nz ? a[id + 4] : R(0);
        ld4r(vin2, id, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            if (k < g.nz - 1)
                v[q] = rmul(rsub(v[q], rmul(cf.vc, gradz(e, q, k, g.nz, cf))), face_d(ac[q], q < 3 ? ac[q + 1] : a4));
        }
        st4r(vout2, id, v);
    }
}

// dep >= 0: the next step's source sample sig[dep_n] is added to the new
// pressure of cell dep, as k_deposit would before that step.
template <class R>
__global__ void __launch_bounds__(256) k_fwd_pres(Grid g, ACoef<R> cf, const R* __restrict__ a,
                                                  const R* __restrict__ p, const R* __restrict__ vx,
                                                  const R* __restrict__ vy, const R* __restrict__ vz,
                                                  R* __restrict__ pn, long long dep, const R* __restrict__ sig,
                                                  int dep_n)
{
    ADJ4_INDEX
    R dv[4], pc[4], ac[4], out[4];
    div4(g, vx, vy, vz, id, i, j, k0, cf, dv);
    ld4r(p, id, pc);
    ld4r(a, id, ac);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        out[q] = (k0 + q < g.nz) ? rmul(rsub(pc[q], rmul(cf.bulk, dv[q])), cell_q(ac[q])) : R(0);
    if (dep >= id && dep < id + 4) {
        const R sv = sig[dep_n];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (dep == id + q && sv != R(0)) out[q] = radd(out[q], sv);
    }
    st4r(pn, id, out);
}

// Source deposit into the (open) source cell before step n.
template <class R>
__global__ void k_deposit(R* p, long long src, const R* sig, int n)
{
    const R s = sig[n];
    if (s != R(0)) p[src] = radd(p[src], s);
}

// After forward step n: the receivers of P^{n+1} (row; 8 taps summed
// w0*p0 + w1*p1 + ... as acoustic_fdtd.cpp:1663-1676), then the next step's
// source sample into P^{n+1} (dep_n >= 0); one block.
template <class R>
__global__ void k_fwd_epilogue(R* p, int n_rec, const long long* idx, const R* w, R* row, long long src,
                               const R* sig, int dep_n)
{
    if (row)
        for (int r = threadIdx.x; r < n_rec; r += blockDim.x) {
            R s = rmul(w[8 * r], p[idx[8 * r]]);
            for (int t = 1; t < 8; ++t) s = radd(s, rmul(w[8 * r + t], p[idx[8 * r + t]]));
            row[r] = s;
        }
    __syncthreads();
    if (threadIdx.x == 0 && dep_n >= 0 && src >= 0) {
        const R sv = sig[dep_n];
        if (sv != R(0)) p[src] = radd(p[src], sv);
    }
}

__device__ __forceinline__ void ld4d(const double* p, long long i, double (&v)[4]) { ld4r<double>(p, i, v); }
__device__ __forceinline__ void st4d(double* p, long long i, const double (&v)[4]) { st4r<double>(p, i, v); }

// The receivers' adjoint sources, by cell: the distinct tap cells in
// ascending order, and for each its taps (8 r + t) in the order R^T adds them.
template <class R>
struct TapSources {
    int n = 0;                       // distinct tap cells (0: none)
    const long long* cell = nullptr;
    const int* start = nullptr;      // [n + 1]
    const int* tap = nullptr;        // 8 r + t, ascending within a cell
    const R* w = nullptr;            // tap weights [8 n_rec]
    const R* rrow = nullptr;         // this step's receiver residuals [n_rec]
};

template <class R>
__global__ void __launch_bounds__(256) k_adj_cells1(Grid g, ACoef<R> cf, const R* __restrict__ a,
                                                    const R* __restrict__ lam, const R* __restrict__ pt,
                                                    const R* __restrict__ vx, const R* __restrict__ vy,
                                                    const R* __restrict__ vz, R* __restrict__ u,
                                                    double* __restrict__ grad, TapSources<R> ts)
{
    ADJ4_INDEX
    R ac[4], l[4], ptc[4], dv[4], uo[4];
    double gr[4];
    ld4r(a, id, ac);
    ld4r(lam, id, l);
    if (ts.n > 0) {   // lam = Lp + R^T r^n on the tap cells among these four
        int lo = 0, hi = ts.n;   // first tap cell >= id
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ts.cell[mid] < id) lo = mid + 1;
            else hi = mid;
        }
        for (int c = lo; c < ts.n && ts.cell[c] < id + 4; ++c) {
            const int q = (int)(ts.cell[c] - id);
            for (int e = ts.start[c]; e < ts.start[c + 1]; ++e) {
                const int tp = ts.tap[e];
#pragma unroll
                for (int qq = 0; qq < 4; ++qq)
                    if (qq == q) l[qq] = radd(l[qq], rmul(ts.w[tp], ts.rrow[tp >> 3]));
            }
        }
    }
    ld4r(pt, id, ptc);
    div4(g, vx, vy, vz, id, i, j, k0, cf, dv);
    ld4d(grad, id, gr);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uo[q] = R(0);
        if (k0 + q >= g.nz) continue;
        const R qq = cell_q(ac[q]);
        uo[q] = rmul(l[q], qq);
        const R z = rsub(ptc[q], rmul(cf.bulk, dv[q]));
        gr[q] -= (double)qq * (double)qq * (double)l[q] * (double)z;
    }
    st4r(u, id, uo);
    st4d(grad, id, gr);
}

// Transposed divergence on the x or y faces of the four cells (divT_face each).
template <class R>
__device__ __forceinline__ void divT4(const R* u, long long id, long long s, int f, int n, const ACoef<R>& cf,
                                      R (&out)[4])
{
    R uc[4], ur[4], um[4] = {}, upp[4] = {};
    ld4r(u, id, uc);
    ld4r(u, id + s, ur);
    if (f >= 1) ld4r(u, id - s, um);
    if (f <= n - 3) ld4r(u, id + 2 * s, upp);
#pragma unroll
    for (int q = 0; q < 4; ++q) out[q] = radd(rmul(cf.c1, rsub(uc[q], ur[q])), rmul(cf.c2, rsub(um[q], upp[q])));
}

template <class R>
__global__ void __launch_bounds__(256) k_adj_faces(Grid g, ACoef<R> cf, const R* __restrict__ a,
                                                   const R* __restrict__ u, const R* __restrict__ pt,
                                                   const R* __restrict__ vo0, const R* __restrict__ vo1,
                                                   const R* __restrict__ vo2, R* lv0, R* lv1, R* lv2,
                                                   R* __restrict__ e0, R* __restrict__ e1, R* __restrict__ e2)
{
    ADJ4_INDEX
    R ac[4], ptc[4];
    ld4r(a, id, ac);
    ld4r(pt, id, ptc);
    // x and y faces
#pragma unroll
    for (int ax = 0; ax < 2; ++ax) {
        const bool exists = ax == 0 ? i < g.nx - 1 : j < g.ny - 1;
        if (!exists) continue;
        const long long s = ax == 0 ? g.plane : (long long)g.sz;
        const int f = ax == 0 ? i : j, n = ax == 0 ? g.nx : g.ny;
        R* lv = ax == 0 ? lv0 : lv1;
        R* ef = ax == 0 ? e0 : e1;
        const R* vo = ax == 0 ? vo0 : vo1;
        R dt[4], gr[4], ar[4], l[4], v[4], eo[4];
        divT4(u, id, s, f, n, cf, dt);
        grad4(pt, id, s, f, n, cf, ptc, gr);
        ld4r(a, id + s, ar);
        ld4r(lv, id, l);
        ld4r(vo, id, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            eo[q] = R(0);
            if (k0 + q >= g.nz) continue;
            const R mu = rsub(l[q], rmul(cf.bulk, dt[q]));
            const R y = rsub(v[q], rmul(cf.vc, gr[q]));
            l[q] = rmul(mu, face_d(ac[q], ar[q]));
            eo[q] = rmul(mu, y);
        }
        st4r(lv, id, l);
        st4r(ef, id, eo);
    }
    // z faces: U and P at k0-1 .. k0+5, a at k0 .. k0+4
    {
        R uc[4], eu[7], ep[7], l[4], v[4], eo[4];
        ld4r(u, id, uc);
        zrow(u, id, k0, g.nz, uc, eu);
        zrow(pt, id, k0, g.nz, ptc, ep);
        const R a4 = k0 + 4 < g.nz ? a[id + 4] : R(0);
        ld4r(lv2, id, l);
        ld4r(vo2, id, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            eo[q] = R(0);
            if (k >= g.nz - 1) continue;
            // divT_face along z: c1 (u[k] - u[k+1]) + c2 (u[k-1] - u[k+2]), zero outside
            const R um = k >= 1 ? eu[q] : R(0), upp = k <= g.nz - 3 ? eu[q + 3] : R(0);
            const R dt = radd(rmul(cf.c1, rsub(eu[q + 1], eu[q + 2])), rmul(cf.c2, rsub(um, upp)));
            const R mu = rsub(l[q], rmul(cf.bulk, dt));
            const R y = rsub(v[q], rmul(cf.vc, gradz(ep, q, k, g.nz, cf)));
            l[q] = rmul(mu, face_d(ac[q], q < 3 ? ac[q + 1] : a4));
            eo[q] = rmul(mu, y);
        }
        st4r(lv2, id, l);
        st4r(e2, id, eo);
    }
}

// Transposed gradient of the four cells along x or y (cell index t uniform).
template <class R>
__device__ __forceinline__ void gradT4(const R* w, long long id, long long s, int t, int n, const ACoef<R>& cf,
                                       R (&out)[4])
{
    const int nf = n - 1;
    auto inner = [&](int f) { return f > 0 && f < n - 2; };
#pragma unroll
    for (int q = 0; q < 4; ++q) out[q] = R(0);
    R v[4];
    if (t - 1 >= 0 && t - 1 < nf) {
        ld4r(w, id - s, v);
        const R c = inner(t - 1) ? cf.c1 : R(1);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = radd(out[q], rmul(c, v[q]));
    }
    if (t < nf) {
        ld4r(w, id, v);
        const R c = inner(t) ? cf.c1 : R(1);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = rsub(out[q], rmul(c, v[q]));
    }
    if (t - 2 >= 0 && inner(t - 2)) {
        ld4r(w, id - 2 * s, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = radd(out[q], rmul(cf.c2, v[q]));
    }
    if (t + 1 < nf && inner(t + 1)) {
        ld4r(w, id + s, v);
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = rsub(out[q], rmul(cf.c2, v[q]));
    }
}

template <class R>
__global__ void __launch_bounds__(256) k_adj_cells2(Grid g, ACoef<R> cf, const R* __restrict__ u,
                                                    const R* __restrict__ w0, const R* __restrict__ w1,
                                                    const R* __restrict__ w2, const R* __restrict__ e0,
                                                    const R* __restrict__ e1, const R* __restrict__ e2,
                                                    R* __restrict__ lp, double* __restrict__ grad)
{
    ADJ4_INDEX
    const long long P = g.plane, S = g.sz;
    R gx[4], gy[4], uc[4], wc[4], ew[7], lo[4];
    gradT4(w0, id, P, i, g.nx, cf, gx);
    gradT4(w1, id, S, j, g.ny, cf, gy);
    ld4r(u, id, uc);
    // W_z at k0-2 .. k0+4: ew[t] = Wz[k0 - 2 + t]
    ld4r(w2, id, wc);
    ew[0] = k0 >= 2 ? w2[id - 2] : R(0);
    ew[1] = k0 >= 1 ? w2[id - 1] : R(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) ew[q + 2] = wc[q];
    ew[6] = k0 + 4 < g.nz ? w2[id + 4] : R(0);
    // E: x and y faces of the four cells, and the z faces k0-1 .. k0+3
    R ex[4] = {}, exm[4] = {}, ey[4] = {}, eym[4] = {}, ezc[4], ez[5];
    if (i < g.nx - 1) ld4r(e0, id, ex);
    if (i > 0) ld4r(e0, id - P, exm);
    if (j < g.ny - 1) ld4r(e1, id, ey);
    if (j > 0) ld4r(e1, id - S, eym);
    ld4r(e2, id, ezc);
    ez[0] = k0 >= 1 ? e2[id - 1] : R(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) ez[q + 1] = ezc[q];
    double gr[4];
    ld4d(grad, id, gr);
    const int nzf = g.nz - 1;
    auto innerz = [&](int f) { return f > 0 && f < g.nz - 2; };
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = k0 + q;
        lo[q] = R(0);
        if (k >= g.nz) continue;
        // gradT_cell along z, term order of the scalar helper
        R gz = R(0);
        if (k - 1 >= 0 && k - 1 < nzf) gz = radd(gz, rmul(innerz(k - 1) ? cf.c1 : R(1), ew[q + 1]));
        if (k < nzf) gz = rsub(gz, rmul(innerz(k) ? cf.c1 : R(1), ew[q + 2]));
        if (k - 2 >= 0 && innerz(k - 2)) gz = radd(gz, rmul(cf.c2, ew[q]));
        if (k + 1 < nzf && innerz(k + 1)) gz = rsub(gz, rmul(cf.c2, ew[q + 3]));
        R gt = radd(radd(gx[q], gy[q]), gz);
        lo[q] = rsub(uc[q], rmul(cf.vc, gt));
        double e = 0.0;
        if (i < g.nx - 1) e += (double)ex[q];
        if (i > 0) e += (double)exm[q];
        if (j < g.ny - 1) e += (double)ey[q];
        if (j > 0) e += (double)eym[q];
        if (k < g.nz - 1) e += (double)ez[q + 1];
        if (k > 0) e += (double)ez[q];
        gr[q] -= 0.5 * e;
    }
    st4r(lp, id, lo);
    st4d(grad, id, gr);
}

// a (reference order, float or double) -> padded R array
template <class R, class T>
__global__ void k_load_a(Grid g, const T* __restrict__ src, R* __restrict__ dst)
{
    ADJ_INDEX
    dst[id] = (R)src[((long long)i * g.ny + j) * g.nz + k];
}

// padded double grad -> reference order (double)
__global__ void k_store_grad(Grid g, const double* __restrict__ src, double* __restrict__ dst)
{
    ADJ_INDEX
    dst[((long long)i * g.ny + j) * g.nz + k] = src[id];
}

}  // namespace adj
}  // namespace fdtd

using namespace fdtd;
using namespace fdtd::adj;

struct FdtdB200Adj {
    int dbl = 0, device = 0, K = 200;
    cudaStream_t stream = nullptr;
    Grid g{};
    int N = 0;
    double dt = 0;
    ACoef<float> c32{};
    ACoef<double> c64{};
    size_t eb = 4;                 // bytes per value of R
    void* a = nullptr;             // padded R
    // loss-mode state and checkpoints
    void *P0 = nullptr, *P1 = nullptr, *V0[3] = {}, *V1[3] = {};
    std::vector<void*> ckP, ckV;   // ckV holds 3 per checkpoint
    // segment slots: K+1 P and K+1 x 3 V
    std::vector<void*> sP, sV;
    // adjoint state
    void *Lp = nullptr, *U = nullptr, *Lv[3] = {}, *E[3] = {};
    double* grad = nullptr;
    double* grad_ref = nullptr;    // reference-order staging
    // source/receivers
    long long src = -1;
    void* sig = nullptr;           // R[n_sig]
    int n_sig = 0;
    int n_rec = 0;
    long long* ridx = nullptr;
    void* rw = nullptr;            // R[8 n_rec]
    void* traces = nullptr;        // R[n_steps x n_rec]
    void* resid = nullptr;         // R[n_steps x n_rec]
    int n_tap_cells = 0;           // distinct receiver tap cells, sorted (TapSources)
    long long* tap_cell = nullptr;
    int* tap_start = nullptr;
    int* tap_ord = nullptr;
    int trace_cap = 0;
    int fwd_steps = -1;            // steps of the last checkpointed forward
    std::vector<void*> allocs;
    long long launches = 0;
    // CUDA graphs of whole sweeps, replayed while the buffers they name live:
    // forward without / with checkpoints (keyed by steps), backward (keyed by steps)
    struct Sweep {
        cudaGraphExec_t exec = nullptr;
        int steps = -1;
        long long launches = 0;
    } fwd[2], bwd;
};

namespace {

#define ACK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { record_cuda_error(e_, #x); return FDTD_ERR_CUDA; } } while (0)

int dalloc(FdtdB200Adj* h, void** p, size_t bytes)
{
    ACK(cudaMalloc(p, bytes));
    h->allocs.push_back(*p);
    ACK(cudaMemsetAsync(*p, 0, bytes, h->stream));
    return FDTD_OK;
}

void dfree(FdtdB200Adj* h, void*& p)
{
    if (!p) return;
    cudaFree(p);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), p), h->allocs.end());
    p = nullptr;
}

size_t field_bytes(const FdtdB200Adj* h) { return (size_t)h->g.cells * h->eb; }

dim3 cell_grid(const Grid& g) { return dim3((g.nz + 31) / 32, (g.ny + 7) / 8, g.nx); }
dim3 vec_grid(const Grid& g) { return dim3((g.sz / 4 + 31) / 32, (g.ny + 7) / 8, g.nx); }   // four cells per thread
const dim3 kBlock(32, 8, 1);

template <class R>
const ACoef<R>& coef(const FdtdB200Adj* h);
template <>
const ACoef<float>& coef<float>(const FdtdB200Adj* h) { return h->c32; }
template <>
const ACoef<double>& coef<double>(const FdtdB200Adj* h) { return h->c64; }

// One forward step from (p, vin) to (pn, vout); p already holds this step's
// source sample.  With next_deposit the next step's sample is added to pn:
// by the pressure kernel when no receivers are recorded (a recompute), else
// by the epilogue after it has recorded the receivers of pn.
template <class R>
void fwd_step(FdtdB200Adj* h, int n, void* p, void* const* vin, void* const* vout, void* pn, bool next_deposit,
              bool record)
{
    const Grid& g = h->g;
    const ACoef<R>& cf = coef<R>(h);
    const bool dep = next_deposit && h->src >= 0 && n + 1 < h->n_sig;
    const bool rec = record && h->n_rec > 0 && n < h->trace_cap;
    k_fwd_vel<R><<<vec_grid(g), kBlock, 0, h->stream>>>(g, cf, (const R*)h->a, (const R*)p, (const R*)vin[0],
                                                         (const R*)vin[1], (const R*)vin[2], (R*)vout[0],
                                                         (R*)vout[1], (R*)vout[2]);
    const bool dep_in_pres = dep && !rec;
    k_fwd_pres<R><<<vec_grid(g), kBlock, 0, h->stream>>>(g, cf, (const R*)h->a, (const R*)p, (const R*)vout[0],
                                                          (const R*)vout[1], (const R*)vout[2], (R*)pn,
                                                          dep_in_pres ? h->src : -1LL, (const R*)h->sig, n + 1);
    h->launches += 2;
    if (rec) {
        k_fwd_epilogue<R><<<1, 128, 0, h->stream>>>((R*)pn, h->n_rec, h->ridx, (const R*)h->rw,
                                                    (R*)h->traces + (size_t)n * h->n_rec, h->src,
                                                    (const R*)h->sig, dep ? n + 1 : -1);
        ++h->launches;
    }
}

int ensure_checkpoints(FdtdB200Adj* h, int n_steps)
{
    const size_t fb = field_bytes(h);
    const int n_ck = (n_steps + h->K - 1) / h->K;
    while ((int)h->ckP.size() < n_ck) {
        void* p = nullptr;
        int rc = dalloc(h, &p, fb);
        if (rc) return rc;
        h->ckP.push_back(p);
        for (int c = 0; c < 3; ++c) {
            void* v = nullptr;
            rc = dalloc(h, &v, fb);
            if (rc) return rc;
            h->ckV.push_back(v);
        }
    }
    return FDTD_OK;
}

// The forward sweep (enqueued only; checkpoints must already exist).
template <class R>
int forward_impl(FdtdB200Adj* h, int n_steps, int keep)
{
    const size_t fb = field_bytes(h);
    ACK(cudaMemsetAsync(h->P0, 0, fb, h->stream));
    for (int c = 0; c < 3; ++c) ACK(cudaMemsetAsync(h->V0[c], 0, fb, h->stream));
    void* P[2] = {h->P0, h->P1};
    void* V[2][3] = {{h->V0[0], h->V0[1], h->V0[2]}, {h->V1[0], h->V1[1], h->V1[2]}};
    int cur = 0;
    if (h->src >= 0 && h->n_sig > 0) {   // step 0's source sample; later ones come with the step before
        k_deposit<R><<<1, 1, 0, h->stream>>>((R*)P[cur], h->src, (const R*)h->sig, 0);
        ++h->launches;
    }
    for (int n = 0; n < n_steps; ++n) {
        if (keep && n % h->K == 0) {   // p~^n: P^n with its source sample
            const int q = n / h->K;
            ACK(cudaMemcpyAsync(h->ckP[q], P[cur], fb, cudaMemcpyDeviceToDevice, h->stream));
            for (int c = 0; c < 3; ++c)
                ACK(cudaMemcpyAsync(h->ckV[3 * q + c], V[cur][c], fb, cudaMemcpyDeviceToDevice, h->stream));
        }
        fwd_step<R>(h, n, P[cur], V[cur], V[cur ^ 1], P[cur ^ 1], n + 1 < n_steps, true);
        cur ^= 1;
    }
    ACK(cudaGetLastError());
    return FDTD_OK;
}

void drop_sweep(FdtdB200Adj::Sweep& g)
{
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = FdtdB200Adj::Sweep();
}

void drop_sweeps(FdtdB200Adj* h)
{
    drop_sweep(h->fwd[0]);
    drop_sweep(h->fwd[1]);
    drop_sweep(h->bwd);
}

// Replays the cached graph of a sweep, capturing it first when it is missing
// or was made for another length.  enqueue(h) issues the sweep on h->stream.
template <class F>
int run_sweep(FdtdB200Adj* h, FdtdB200Adj::Sweep& g, int steps, F enqueue)
{
    if (!g.exec || g.steps != steps) {
        drop_sweep(g);
        const long long l0 = h->launches;
        ACK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue(h);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        ACK(e);
        const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        ACK(ei);
        g.steps = steps;
        g.launches = h->launches - l0;
        h->launches = l0;
    }
    ACK(cudaGraphLaunch(g.exec, h->stream));
    h->launches += g.launches;
    return FDTD_OK;
}

int ensure_slots(FdtdB200Adj* h)
{
    const size_t fb = field_bytes(h);
    while ((int)h->sP.size() < h->K + 1) {
        void* p = nullptr;
        int rc = dalloc(h, &p, fb);
        if (rc) return rc;
        h->sP.push_back(p);
        for (int c = 0; c < 3; ++c) {
            void* v = nullptr;
            rc = dalloc(h, &v, fb);
            if (rc) return rc;
            h->sV.push_back(v);
        }
    }
    if (!h->Lp) {
        int rc = dalloc(h, &h->Lp, fb);
        if (!rc) rc = dalloc(h, &h->U, fb);
        for (int c = 0; c < 3 && !rc; ++c) rc = dalloc(h, &h->Lv[c], fb);
        for (int c = 0; c < 3 && !rc; ++c) rc = dalloc(h, &h->E[c], fb);
        if (!rc) {
            void* gp = nullptr;
            rc = dalloc(h, &gp, (size_t)h->g.cells * sizeof(double));
            h->grad = (double*)gp;
        }
        if (!rc) {
            void* gr = nullptr;
            rc = dalloc(h, &gr, (size_t)h->N * sizeof(double));
            h->grad_ref = (double*)gr;
        }
        if (rc) return rc;
    }
    return FDTD_OK;
}

template <class R>
int backward_impl(FdtdB200Adj* h)
{
    const Grid& g = h->g;
    const ACoef<R>& cf = coef<R>(h);
    const size_t fb = field_bytes(h);
    const int n_steps = h->fwd_steps;
    ACK(cudaMemsetAsync(h->Lp, 0, fb, h->stream));
    for (int c = 0; c < 3; ++c) {
        ACK(cudaMemsetAsync(h->Lv[c], 0, fb, h->stream));
        ACK(cudaMemsetAsync(h->E[c], 0, fb, h->stream));
    }
    ACK(cudaMemsetAsync(h->grad, 0, (size_t)g.cells * sizeof(double), h->stream));
    const int n_seg = (n_steps + h->K - 1) / h->K;
    for (int s = n_seg - 1; s >= 0; --s) {
        const int n0 = s * h->K, n1 = std::min(n0 + h->K, n_steps), len = n1 - n0;
        ACK(cudaMemcpyAsync(h->sP[0], h->ckP[s], fb, cudaMemcpyDeviceToDevice, h->stream));
        for (int c = 0; c < 3; ++c)
            ACK(cudaMemcpyAsync(h->sV[c], h->ckV[3 * s + c], fb, cudaMemcpyDeviceToDevice, h->stream));
        // recompute: slot t holds p~^{n0+t} (after its deposit; the checkpoint
        // already holds it) and v^{n0+t-1/2}; traces are already recorded
        for (int t = 0; t < len; ++t)
            fwd_step<R>(h, n0 + t, h->sP[t], &h->sV[3 * t], &h->sV[3 * (t + 1)], h->sP[t + 1], t + 1 < len,
                        false);
        for (int t = len - 1; t >= 0; --t) {
            const int n = n0 + t;
            void* const* vo = &h->sV[3 * t];       // v^{n-1/2}
            void* const* vn = &h->sV[3 * (t + 1)]; // v^{n+1/2}
            TapSources<R> ts;   // R^T r^n, added to Lp inside k_adj_cells1
            if (h->n_rec > 0) {
                ts.n = h->n_tap_cells;
                ts.cell = h->tap_cell;
                ts.start = h->tap_start;
                ts.tap = h->tap_ord;
                ts.w = (const R*)h->rw;
                ts.rrow = (const R*)h->resid + (size_t)n * h->n_rec;
            }
            k_adj_cells1<R><<<vec_grid(g), kBlock, 0, h->stream>>>(
                g, cf, (const R*)h->a, (const R*)h->Lp, (const R*)h->sP[t], (const R*)vn[0], (const R*)vn[1],
                (const R*)vn[2], (R*)h->U, h->grad, ts);
            k_adj_faces<R><<<vec_grid(g), kBlock, 0, h->stream>>>(
                g, cf, (const R*)h->a, (const R*)h->U, (const R*)h->sP[t], (const R*)vo[0], (const R*)vo[1],
                (const R*)vo[2], (R*)h->Lv[0], (R*)h->Lv[1], (R*)h->Lv[2], (R*)h->E[0], (R*)h->E[1],
                (R*)h->E[2]);
            k_adj_cells2<R><<<vec_grid(g), kBlock, 0, h->stream>>>(
                g, cf, (const R*)h->U, (const R*)h->Lv[0], (const R*)h->Lv[1], (const R*)h->Lv[2],
                (const R*)h->E[0], (const R*)h->E[1], (const R*)h->E[2], (R*)h->Lp, h->grad);
            h->launches += 3;
        }
        ACK(cudaGetLastError());
    }
    return FDTD_OK;
}

template <class R>
void set_coef(ACoef<R>& cf, R dx, R c, R rho, R dt)
{
    cf.vc = dt / (rho * dx);
    const R inv_dx = R(1) / dx;
    cf.bulk = rho * c * c * dt * inv_dx;
    cf.c1 = R(9) / R(8);
    cf.c2 = R(-1) / R(24);
}

long long pad_index(const Grid& g, int flat)
{
    const int k = flat % g.nz, t = flat / g.nz, j = t % g.ny, i = t / g.ny;
    return ((long long)i * g.ny + j) * g.sz + k;
}

}  // namespace

extern "C" {

FdtdB200Adj* fdtd_b200_adj_create(int Nx, int Ny, int Nz, double dx, double c, double rho_air,
                                  int use_double, int checkpoint_every, int device)
{
    if (Nx < 1 || Ny < 1 || Nz < 1 || dx <= 0 || c <= 0 || checkpoint_every < 1) return nullptr;
    if ((long long)Nx * Ny * Nz > INT_MAX) return nullptr;
    FdtdB200Adj* h = new FdtdB200Adj();
    h->dbl = use_double ? 1 : 0;
    h->eb = h->dbl ? 8 : 4;
    h->K = checkpoint_every;
    if (device < 0) cudaGetDevice(&device);
    h->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return nullptr;
    }
    Grid& g = h->g;
    g.nx = Nx; g.ny = Ny; g.nz = Nz;
    g.sz = (Nz + kRowAlign - 1) / kRowAlign * kRowAlign;
    g.plane = (long long)Ny * g.sz;
    g.cells = (long long)Nx * g.plane;
    h->N = Nx * Ny * Nz;
    // the reference's time step (acoustic_fdtd.cpp:345-349) in each working type
    const float dt32 = 0.77f * (float)dx / ((float)c * 1.732050808f);
    const double dt64 = 0.77 * dx / (c * 1.732050808);
    set_coef<float>(h->c32, (float)dx, (float)c, (float)rho_air, dt32);
    set_coef<double>(h->c64, dx, c, rho_air, dt64);
    h->dt = h->dbl ? dt64 : (double)dt32;
    const size_t fb = field_bytes(h);
    int rc = dalloc(h, &h->a, fb);
    if (!rc) rc = dalloc(h, &h->P0, fb);
    if (!rc) rc = dalloc(h, &h->P1, fb);
    for (int q = 0; q < 3 && !rc; ++q) rc = dalloc(h, &h->V0[q], fb);
    for (int q = 0; q < 3 && !rc; ++q) rc = dalloc(h, &h->V1[q], fb);
    if (!rc && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = FDTD_ERR_CUDA;
    if (rc) {
        fdtd_b200_adj_destroy(h);
        return nullptr;
    }
    return h;
}

void fdtd_b200_adj_destroy(FdtdB200Adj* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_sweeps(h);
    for (void* p : h->allocs) cudaFree(p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

double fdtd_b200_adj_dt(const FdtdB200Adj* h) { return h ? h->dt : 0.0; }

long long fdtd_b200_adj_launch_count(const FdtdB200Adj* h) { return h ? h->launches : 0; }

int fdtd_b200_adj_set_absorption(FdtdB200Adj* h, const void* a_cell, int len, int value_bytes)
{
    if (!h || !a_cell) return FDTD_ERR_NULL;
    if (len != h->N) return FDTD_ERR_DIM;
    if (value_bytes != 4 && value_bytes != 8) return FDTD_ERR_ARG;
    ACK(cudaSetDevice(h->device));
    void* stage = nullptr;
    ACK(cudaMallocAsync(&stage, (size_t)len * value_bytes, h->stream));
    cudaError_t e = cudaMemcpyAsync(stage, a_cell, (size_t)len * value_bytes, cudaMemcpyDefault, h->stream);
    if (e == cudaSuccess) {
        const Grid& g = h->g;
        if (h->dbl && value_bytes == 8)
            k_load_a<double, double><<<cell_grid(g), kBlock, 0, h->stream>>>(g, (const double*)stage, (double*)h->a);
        else if (h->dbl)
            k_load_a<double, float><<<cell_grid(g), kBlock, 0, h->stream>>>(g, (const float*)stage, (double*)h->a);
        else if (value_bytes == 8)
            k_load_a<float, double><<<cell_grid(g), kBlock, 0, h->stream>>>(g, (const double*)stage, (float*)h->a);
        else
            k_load_a<float, float><<<cell_grid(g), kBlock, 0, h->stream>>>(g, (const float*)stage, (float*)h->a);
        e = cudaGetLastError();
    }
    cudaFreeAsync(stage, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        record_cuda_error(e, "fdtd_b200_adj_set_absorption");
        return FDTD_ERR_CUDA;
    }
    h->fwd_steps = -1;
    return FDTD_OK;
}

int fdtd_b200_adj_set_source(FdtdB200Adj* h, int cell, const double* signal, int n)
{
    if (!h) return FDTD_ERR_NULL;
    if (cell < 0 || cell >= h->N || n < 0 || (n > 0 && !signal)) return FDTD_ERR_ARG;
    ACK(cudaSetDevice(h->device));
    ACK(cudaStreamSynchronize(h->stream));
    drop_sweeps(h);
    dfree(h, h->sig);
    h->src = pad_index(h->g, cell);
    h->n_sig = n;
    if (n > 0) {
        int rc = dalloc(h, &h->sig, (size_t)n * h->eb);
        if (rc) return rc;
        std::vector<unsigned char> buf((size_t)n * h->eb);
        for (int q = 0; q < n; ++q) {
            if (h->dbl) memcpy(&buf[(size_t)q * 8], &signal[q], 8);
            else { const float f = (float)signal[q]; memcpy(&buf[(size_t)q * 4], &f, 4); }
        }
        ACK(cudaMemcpyAsync(h->sig, buf.data(), buf.size(), cudaMemcpyHostToDevice, h->stream));
        ACK(cudaStreamSynchronize(h->stream));
    }
    h->fwd_steps = -1;
    return FDTD_OK;
}

int fdtd_b200_adj_set_receivers(FdtdB200Adj* h, int n_rec, const int* idx8, const double* wgt8, int max_steps)
{
    if (!h || (n_rec > 0 && (!idx8 || !wgt8))) return FDTD_ERR_NULL;
    if (n_rec < 0 || max_steps < 0) return FDTD_ERR_ARG;
    std::vector<long long> pi((size_t)n_rec * 8);
    for (size_t q = 0; q < pi.size(); ++q) {
        if (idx8[q] < 0 || idx8[q] >= h->N) return FDTD_ERR_ARG;
        pi[q] = pad_index(h->g, idx8[q]);
    }
    ACK(cudaSetDevice(h->device));
    ACK(cudaStreamSynchronize(h->stream));
    drop_sweeps(h);
    void* ri = h->ridx;
    dfree(h, ri);
    h->ridx = nullptr;
    dfree(h, h->rw);
    dfree(h, h->traces);
    dfree(h, h->resid);
    {
        void* t1 = h->tap_cell;
        void* t2 = h->tap_start;
        void* t3 = h->tap_ord;
        dfree(h, t1);
        dfree(h, t2);
        dfree(h, t3);
    }
    h->tap_cell = nullptr;
    h->tap_start = nullptr;
    h->tap_ord = nullptr;
    h->n_tap_cells = 0;
    h->n_rec = n_rec;
    h->trace_cap = max_steps;
    if (n_rec > 0) {
        void* p = nullptr;
        int rc = dalloc(h, &p, pi.size() * sizeof(long long));
        if (rc) return rc;
        h->ridx = (long long*)p;
        rc = dalloc(h, &h->rw, pi.size() * h->eb);
        if (!rc) rc = dalloc(h, &h->traces, (size_t)std::max(max_steps, 1) * n_rec * h->eb);
        if (!rc) rc = dalloc(h, &h->resid, (size_t)std::max(max_steps, 1) * n_rec * h->eb);
        if (rc) return rc;
        std::vector<unsigned char> wb(pi.size() * h->eb);
        for (size_t q = 0; q < pi.size(); ++q) {
            if (h->dbl) memcpy(&wb[q * 8], &wgt8[q], 8);
            else { const float f = (float)wgt8[q]; memcpy(&wb[q * 4], &f, 4); }
        }
        ACK(cudaMemcpyAsync(h->ridx, pi.data(), pi.size() * sizeof(long long), cudaMemcpyHostToDevice, h->stream));
        ACK(cudaMemcpyAsync(h->rw, wb.data(), wb.size(), cudaMemcpyHostToDevice, h->stream));
        // taps grouped by cell, each cell's taps in ascending 8 r + t (the order
        // in which R^T r adds them one after another)
        std::vector<int> ord(pi.size());
        for (size_t q = 0; q < ord.size(); ++q) ord[q] = (int)q;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return pi[x] < pi[y]; });
        std::vector<long long> cells;
        std::vector<int> start;
        for (size_t e = 0; e < ord.size(); ++e)
            if (e == 0 || pi[ord[e]] != pi[ord[e - 1]]) {
                cells.push_back(pi[ord[e]]);
                start.push_back((int)e);
            }
        start.push_back((int)ord.size());
        void* tc = nullptr;
        void* tsb = nullptr;
        void* to = nullptr;
        rc = dalloc(h, &tc, cells.size() * sizeof(long long));
        if (!rc) rc = dalloc(h, &tsb, start.size() * sizeof(int));
        if (!rc) rc = dalloc(h, &to, ord.size() * sizeof(int));
        if (rc) return rc;
        h->tap_cell = (long long*)tc;
        h->tap_start = (int*)tsb;
        h->tap_ord = (int*)to;
        h->n_tap_cells = (int)cells.size();
        ACK(cudaMemcpyAsync(h->tap_cell, cells.data(), cells.size() * sizeof(long long), cudaMemcpyHostToDevice,
                            h->stream));
        ACK(cudaMemcpyAsync(h->tap_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice,
                            h->stream));
        ACK(cudaMemcpyAsync(h->tap_ord, ord.data(), ord.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        ACK(cudaStreamSynchronize(h->stream));
    }
    h->fwd_steps = -1;
    return FDTD_OK;
}

int fdtd_b200_adj_forward(FdtdB200Adj* h, int n_steps, int keep_checkpoints, double* traces_out)
{
    if (!h) return FDTD_ERR_NULL;
    if (n_steps < 1 || n_steps > h->trace_cap) return FDTD_ERR_DIM;
    ACK(cudaSetDevice(h->device));
    const int keep = keep_checkpoints ? 1 : 0;
    int rc = keep ? ensure_checkpoints(h, n_steps) : FDTD_OK;
    if (rc) return rc;
    rc = run_sweep(h, h->fwd[keep], n_steps, [&](FdtdB200Adj* s) {
        return s->dbl ? forward_impl<double>(s, n_steps, keep) : forward_impl<float>(s, n_steps, keep);
    });
    if (rc) return rc;
    h->fwd_steps = keep ? n_steps : -1;
    if (traces_out && h->n_rec > 0) {
        const size_t n = (size_t)n_steps * h->n_rec;
        std::vector<unsigned char> buf(n * h->eb);
        ACK(cudaMemcpyAsync(buf.data(), h->traces, buf.size(), cudaMemcpyDeviceToHost, h->stream));
        ACK(cudaStreamSynchronize(h->stream));
        for (size_t q = 0; q < n; ++q) {
            if (h->dbl) memcpy(&traces_out[q], &buf[q * 8], 8);
            else { float f; memcpy(&f, &buf[q * 4], 4); traces_out[q] = f; }
        }
    } else {
        ACK(cudaStreamSynchronize(h->stream));
    }
    return FDTD_OK;
}

int fdtd_b200_adj_backward(FdtdB200Adj* h, const double* dloss_dtrace, double* grad_out)
{
    if (!h || !grad_out || (h->n_rec > 0 && !dloss_dtrace)) return FDTD_ERR_NULL;
    if (h->fwd_steps < 1) return FDTD_ERR_ARG;    // needs a checkpointed forward of the current inputs
    ACK(cudaSetDevice(h->device));
    int rc = ensure_slots(h);
    if (rc) return rc;
    const size_t n = (size_t)h->fwd_steps * h->n_rec;
    if (n > 0) {
        std::vector<unsigned char> buf(n * h->eb);
        for (size_t q = 0; q < n; ++q) {
            if (h->dbl) memcpy(&buf[q * 8], &dloss_dtrace[q], 8);
            else { const float f = (float)dloss_dtrace[q]; memcpy(&buf[q * 4], &f, 4); }
        }
        ACK(cudaMemcpyAsync(h->resid, buf.data(), buf.size(), cudaMemcpyHostToDevice, h->stream));
        ACK(cudaStreamSynchronize(h->stream));
    }
    rc = run_sweep(h, h->bwd, h->fwd_steps, [](FdtdB200Adj* s) {
        return s->dbl ? backward_impl<double>(s) : backward_impl<float>(s);
    });
    if (rc) return rc;
    k_store_grad<<<cell_grid(h->g), kBlock, 0, h->stream>>>(h->g, h->grad, h->grad_ref);
    ACK(cudaGetLastError());
    ACK(cudaMemcpyAsync(grad_out, h->grad_ref, (size_t)h->N * sizeof(double), cudaMemcpyDefault, h->stream));
    ACK(cudaStreamSynchronize(h->stream));
    return FDTD_OK;
}

}  // extern "C"
