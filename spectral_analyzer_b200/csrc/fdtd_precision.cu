/*
 * fdtd_precision.cu — the open-room step with selectable field storage, for
 * the storage-precision study, and its FP64 GPU oracle.
 *
 * Storage modes (P, Vx, Vy, Vz all stored the same way):
 *   FP32    float                      arithmetic float   (as the engine)
 *   FP64    double                     arithmetic double  (the GPU oracle)
 *   BF16    bfloat16                   arithmetic float
 *   FP16    half, scaled               arithmetic float
 *   BF16C   bfloat16 value + bfloat16 residual        (compensated)
 *   FP16C   half value + half residual, scaled        (compensated)
 * A compensated field keeps, beside the 16-bit value h = rn16(x), the 16-bit
 * rounding of the remainder r = rn16(x - h); a load returns h + r in float, so
 * each stored value carries about twice the 16-bit mantissa (the FP16 residual
 * is stored times 2^11, which keeps it out of half's subnormal range).  FP16 fields are
 * stored multiplied by a power of two (default 2^10 for P, 2^19 for V) so that
 * sub-millipascal pressures and micrometre-per-second velocities stay in the
 * normal range of half (the caller picks the powers of two from the source
 * amplitude; non-powers of two would add a rounding of their own).
 *
 * The step is the two-pass update of fdtd_general.cu (open rooms: no walls,
 * fractions or plate) with every operation separately rounded in the
 * reference's order (csrc/kernels/acoustic_fdtd.cpp:1099-1148, :894-952,
 * :1176-1234); FP32 mode therefore reproduces the engine bit for bit, and
 * FP64 mode reproduces the double instantiation of the CPU oracle.
 * Receivers accumulate their 8 taps in double.  Every audit_every steps the
 * velocity pass also accumulates, in double, the discrete energy
 *   E^n = dx^3/2 * ( sum_p (p^n)^2 / (rho c^2) + rho * sum_f v^{n-1/2} v^{n+1/2} ),
 * one block reduction and one atomic per block per sum.
 */
#include "acoustic_fdtd_b200.h"
#include "fdtd_internal.h"
#include "fdtd_prec_internal.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

namespace fdtd {
namespace prec {

__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x * blockDim.y + 31) / 32;
    double s = 0.0;
    if (wid == 0) {
        s = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    return s;   // valid in thread (0,0)
}

#define PREC_INDEX                                                        \
    const int k0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);           \
    const int j = blockIdx.y * blockDim.y + threadIdx.y;                  \
    const int i = blockIdx.z;                                             \
    const bool live = k0 < g.nz && j < g.ny;                              \
    const long long id = ((long long)i * g.ny + j) * g.sz + k0;

// Velocity pass over four cells per thread (k0 .. k0+3); with audit !=
// nullptr it also sums p^2 and v_old*v_new (double).  Faces that do not exist
// (and row padding) keep their stored zero.
template <int M>
__global__ void __launch_bounds__(256) k_vel(Grid g, PCoef<typename Traits<M>::A> cf, Field p,
                                             Field vx, Field vy, Field vz, double* audit)
{
    using A = typename Traits<M>::A;
    PREC_INDEX
    double e_p = 0.0, e_v = 0.0;
    if (live) {
        A pc[4], az4[4], ac[4];
        ld4<M>(p, id, pc);
        const A ay = cf.ay[j], axi = cf.ax[i];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            az4[q] = k < g.nz ? cf.az[k] : A(0);
            ac[q] = amax(amax(axi, ay), az4[q]);
            if (audit && k < g.nz) e_p += (double)pc[q] * (double)pc[q];
        }
        // x faces
        if (i < g.nx - 1) {
            const bool fourth = i > 0 && i < g.nx - 2;
            A pr[4], pm[4], p2[4], vo[4], vn[4];
            ld4<M>(p, id + g.plane, pr);
            if (fourth) {
                ld4<M>(p, id - g.plane, pm);
                ld4<M>(p, id + 2 * g.plane, p2);
            }
            ld4<M>(vx, id, vo);
            const A axr = cf.ax[i + 1];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                vn[q] = vo[q];
                if (k0 + q < g.nz) {
                    const A grad = fourth ? radd(rmul(cf.c1, rsub(pr[q], pc[q])), rmul(cf.c2, rsub(p2[q], pm[q])))
                                          : rsub(pr[q], pc[q]);
                    vn[q] = rmul(rsub(vo[q], rmul(cf.vc, grad)), fdamp(ac[q], amax(amax(axr, ay), az4[q]), cf.dt));
                    if (audit) e_v += (double)vo[q] * (double)vn[q];
                }
            }
            st4<M>(vx, id, vn);
        }
        // y faces
        if (j < g.ny - 1) {
            const bool fourth = j > 0 && j < g.ny - 2;
            A pr[4], pm[4], p2[4], vo[4], vn[4];
            ld4<M>(p, id + g.sz, pr);
            if (fourth) {
                ld4<M>(p, id - g.sz, pm);
                ld4<M>(p, id + 2 * g.sz, p2);
            }
            ld4<M>(vy, id, vo);
            const A ayr = cf.ay[j + 1];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                vn[q] = vo[q];
                if (k0 + q < g.nz) {
                    const A grad = fourth ? radd(rmul(cf.c1, rsub(pr[q], pc[q])), rmul(cf.c2, rsub(p2[q], pm[q])))
                                          : rsub(pr[q], pc[q]);
                    vn[q] = rmul(rsub(vo[q], rmul(cf.vc, grad)), fdamp(ac[q], amax(amax(axi, ayr), az4[q]), cf.dt));
                    if (audit) e_v += (double)vo[q] * (double)vn[q];
                }
            }
            st4<M>(vy, id, vn);
        }
        // z faces: P at k0-1 .. k0+5 (ext[t] = P[k0 - 1 + t])
        {
            A ext[7], vo[4], vn[4];
            ext[0] = k0 > 0 ? ld<M>(p, id - 1) : A(0);
#pragma unroll
            for (int q = 0; q < 4; ++q) ext[q + 1] = pc[q];
            ext[5] = k0 + 4 < g.nz ? ld<M>(p, id + 4) : A(0);
            ext[6] = k0 + 5 < g.nz ? ld<M>(p, id + 5) : A(0);
            ld4<M>(vz, id, vo);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int k = k0 + q;
                vn[q] = vo[q];
                if (k < g.nz - 1) {
                    const A grad = (k > 0 && k < g.nz - 2)
                                       ? radd(rmul(cf.c1, rsub(ext[q + 2], ext[q + 1])), rmul(cf.c2, rsub(ext[q + 3], ext[q])))
                                       : rsub(ext[q + 2], ext[q + 1]);
                    vn[q] = rmul(rsub(vo[q], rmul(cf.vc, grad)), fdamp(ac[q], amax(amax(axi, ay), cf.az[k + 1]), cf.dt));
                    if (audit) e_v += (double)vo[q] * (double)vn[q];
                }
            }
            st4<M>(vz, id, vn);
        }
    }
    if (audit) {   // uniform per launch
        const double sp = block_sum(e_p);
        __syncthreads();
        const double sv = block_sum(e_v);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            atomicAdd(audit, sp);
            atomicAdd(audit + 1, sv);
        }
    }
}

// Pressure pass over four cells per thread.
template <int M>
__global__ void __launch_bounds__(256) k_pres(Grid g, PCoef<typename Traits<M>::A> cf, Field p, Field pn,
                                              Field vx, Field vy, Field vz)
{
    using A = typename Traits<M>::A;
    PREC_INDEX
    if (!live) return;
    const long long P = g.plane, S = g.sz;
    A xp[4] = {}, xm[4] = {}, xpp[4] = {}, xmm[4] = {}, yp[4] = {}, ym[4] = {}, ypp[4] = {}, ymm[4] = {};
    if (i < g.nx - 1) ld4<M>(vx, id, xp);
    if (i > 0) ld4<M>(vx, id - P, xm);
    if (i < g.nx - 2) ld4<M>(vx, id + P, xpp);
    if (i > 1) ld4<M>(vx, id - 2 * P, xmm);
    if (j < g.ny - 1) ld4<M>(vy, id, yp);
    if (j > 0) ld4<M>(vy, id - S, ym);
    if (j < g.ny - 2) ld4<M>(vy, id + S, ypp);
    if (j > 1) ld4<M>(vy, id - 2 * S, ymm);
    // Vz at k0-2 .. k0+4: ext[t] = Vz[k0 - 2 + t]
    A ext[7], vzc[4], pc[4], out[4];
    ld4<M>(vz, id, vzc);
    ext[0] = k0 >= 2 ? ld<M>(vz, id - 2) : A(0);
    ext[1] = k0 >= 1 ? ld<M>(vz, id - 1) : A(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) ext[q + 2] = vzc[q];
    ext[6] = k0 + 4 < g.nz ? ld<M>(vz, id + 4) : A(0);
    ld4<M>(p, id, pc);
    const A z0 = A(0);
    const A pxy = amin(cf.px[i], cf.py[j]);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = k0 + q;
        out[q] = z0;
        if (k < g.nz) {
            const A zp = (k < g.nz - 1) ? ext[q + 2] : z0;
            const A zm = (k > 0) ? ext[q + 1] : z0;
            const A zpp = (k < g.nz - 2) ? ext[q + 3] : z0;
            const A zmm = (k > 1) ? ext[q] : z0;
            const A d1 = radd(radd(rsub(xp[q], xm[q]), rsub(yp[q], ym[q])), rsub(zp, zm));
            const A d2 = radd(radd(rsub(xpp[q], xmm[q]), rsub(ypp[q], ymm[q])), rsub(zpp, zmm));
            const A dv = radd(rmul(cf.c1, d1), rmul(cf.c2, d2));
            out[q] = rmul(rsub(pc[q], rmul(cf.bulk, dv)), amin(pxy, cf.pz[k]));
        }
    }
    st4<M>(pn, id, out);
}

// Source deposit into an open cell (the rooms here have no solid cells) and
// receiver record (8 taps, double accumulation), one block.
template <int M>
__global__ void k_src_rec(Field p, long long src, const double* sig, int step, int n_sig,
                          int n_rec, const long long* ridx, const double* rw, double* trace,
                          int record)
{
    using A = typename Traits<M>::A;
    if (record) {
        for (int r = threadIdx.x; r < n_rec; r += blockDim.x) {
            double s = 0.0;
            for (int t = 0; t < 8; ++t)
                s = __dadd_rn(s, __dmul_rn(rw[8 * r + t], (double)ld<M>(p, ridx[8 * r + t])));
            trace[r] = s;
        }
    } else if (threadIdx.x == 0 && src >= 0 && step < n_sig) {
        const A amp = (A)sig[step];
        if (amp != A(0)) st<M>(p, src, radd(ld<M>(p, src), amp));
    }
}

}  // namespace prec
}  // namespace fdtd

using namespace fdtd;
using namespace fdtd::prec;

struct FdtdB200Prec {
    int mode = 0, device = 0;
    cudaStream_t stream = nullptr;
    Grid g{};
    int N = 0;
    double dt = 0;
    double rho = 0, c = 0, dx = 0;
    // coefficients in both arithmetic types; tables on the device
    PCoef<float> cf32{};
    PCoef<double> cf64{};
    void* d_tab = nullptr;
    Field f[5] = {};            // P0, P1, Vx, Vy, Vz
    int cur = 0;                // P current = f[cur]
    // The single-pass 16-bit step writes the other velocity set (v2) and
    // flips vset; the two-pass step updates the current set in place.
    int kernel = 0;             // 1: single-pass step (16-bit modes), 0: two-pass
    int xi_lo = 0, xi_hi = 0;   // planes with alpha_x = 0 (the single pass's interior body)
    Field v2[3] = {};
    int vset = 0;
    F16Cache* maps = nullptr;
    unsigned* d_status = nullptr;
    std::vector<double> h_sig; // host copy of the source signal (the launch argument)
    bool rec_pending = false;   // the current P's receivers are not recorded yet
    long long launches = 0;     // kernels launched by prec_step
    std::vector<void*> allocs;
    long long src = -1;
    double* d_sig = nullptr;
    int n_sig = 0;
    int n_rec = 0;
    long long* d_ridx = nullptr;
    double* d_rw = nullptr;
    double* d_trace = nullptr;
    int cap = 0, n_rec_steps = 0;
    double* d_audit = nullptr;  // [cap_audit][2]
    std::vector<int> audit_steps;
    int cap_audit = 0;
    int step = 0;
};

namespace {

Field* vfields(FdtdB200Prec* p) { return p->vset ? p->v2 : p->f + 2; }

size_t elem_bytes(int mode) { return mode == kFP64 ? 8 : mode == kFP32 ? 4 : 2; }
bool compensated(int mode) { return mode == kBF16C || mode == kFP16C; }

template <class A>
A sig_scaled(int d, int n_pml, A dt, A scale)
{   // pml_sigma with sigma_max scaled (acoustic_fdtd.cpp:216-222), in A
    if (n_pml <= 0 || d <= 0) return A(0);
    A frac = (A)d / (A)n_pml;
    A sigma_max = scale * (A(3.45) / (dt * (A)n_pml));
    return sigma_max * frac * frac * frac;
}

template <class A>
A axis_alpha_t(int i, int n, int n_pml, A dt, A a_lo, A a_hi)
{
    if (i < n_pml) return sig_scaled<A>(n_pml - i, n_pml, dt, a_lo);
    if (i >= n - n_pml) return sig_scaled<A>(i - (n - n_pml) + 1, n_pml, dt, a_hi);
    return A(0);
}

template <class A>
void build(FdtdB200Prec* p, A dx, A c, A rho, A c77, A sqrt3, int n_pml, const float* a6,
           std::vector<A>& tab, PCoef<A>& cf)
{
    const Grid& g = p->g;
    const A dt = c77 * dx / (c * sqrt3);
    cf.dt = dt;
    cf.vc = dt / (rho * dx);
    const A inv_dx = A(1) / dx;
    cf.bulk = rho * c * c * dt * inv_dx;
    cf.c1 = A(9) / A(8);
    cf.c2 = A(-1) / A(24);
    tab.assign((size_t)2 * (g.nx + g.ny + g.nz), A(0));
    A* ax = tab.data();
    A* ay = ax + g.nx;
    A* az = ay + g.ny;
    A* pp = az + g.nz;
    for (int i = 0; i < g.nx; ++i) ax[i] = axis_alpha_t<A>(i, g.nx, n_pml, dt, (A)a6[0], (A)a6[1]);
    for (int j = 0; j < g.ny; ++j) ay[j] = axis_alpha_t<A>(j, g.ny, n_pml, dt, (A)a6[2], (A)a6[3]);
    for (int k = 0; k < g.nz; ++k) az[k] = axis_alpha_t<A>(k, g.nz, n_pml, dt, (A)a6[4], (A)a6[5]);
    for (int q = 0; q < g.nx + g.ny + g.nz; ++q) {
        A denom = A(1) + ax[q] * dt;
        pp[q] = A(1) / denom;
    }
}

template <class A>
void point_tables(PCoef<A>& cf, void* d_tab, const Grid& g)
{
    A* base = static_cast<A*>(d_tab);
    cf.ax = base;
    cf.ay = cf.ax + g.nx;
    cf.az = cf.ay + g.ny;
    cf.px = cf.az + g.nz;
    cf.py = cf.px + g.nx;
    cf.pz = cf.py + g.ny;
}

int fail(cudaError_t e, const char* what)
{
    record_cuda_error(e, what);
    return FDTD_ERR_CUDA;
}

#define PCK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(e_, #x); } while (0)

template <int M>
void record_now(FdtdB200Prec* p)
{
    if (p->n_rec > 0 && p->n_rec_steps < p->cap) {
        k_src_rec<M><<<1, 128, 0, p->stream>>>(p->f[p->cur], -1, nullptr, 0, 0, p->n_rec, p->d_ridx, p->d_rw,
                                               p->d_trace + (size_t)p->n_rec_steps * p->n_rec, 1);
        ++p->n_rec_steps;
        ++p->launches;
    }
}

// the second velocity set of the single-pass step, zeroed (faces it never
// writes — the last face of each axis and the row padding — stay zero)
int ensure_v2(FdtdB200Prec* p)
{
    if (p->v2[0].hi) return FDTD_OK;
    const size_t fb = (size_t)p->g.cells * elem_bytes(p->mode);
    for (int q = 0; q < 3; ++q) {
        Field& f = p->v2[q];
        f = p->f[2 + q];
        f.hi = f.lo = nullptr;
        PCK(cudaMalloc(&f.hi, fb));
        p->allocs.push_back(f.hi);
        PCK(cudaMemset(f.hi, 0, fb));
        if (compensated(p->mode)) {
            PCK(cudaMalloc(&f.lo, fb));
            p->allocs.push_back(f.lo);
            PCK(cudaMemset(f.lo, 0, fb));
        }
    }
    return FDTD_OK;
}

// one single-pass step (16-bit modes): P^n, V set -> P^{n+1}, other V set;
// records the previous step's receivers from P^n when they are pending
template <int M>
int fused16_step(FdtdB200Prec* p)
{
    const int rc = ensure_v2(p);
    if (rc != FDTD_OK) return rc;
    const Grid& g = p->g;
    Field* vin = vfields(p);
    Field* vout = p->vset ? p->f + 2 : p->v2;
    const Field& P = p->f[p->cur];
    const Field& PN = p->f[p->cur ^ 1];
    F16Args a{};
    a.g = g;
    a.cf = p->cf32;
    a.p_hi = P.hi; a.p_lo = P.lo;
    a.pn_hi = PN.hi; a.pn_lo = PN.lo;
    for (int q = 0; q < 3; ++q) {
        a.vout_hi[q] = vout[q].hi;
        a.vout_lo[q] = vout[q].lo;
    }
    a.sp = Sc{P.scale, P.inv_scale, P.lo_scale, P.inv_lo_scale};
    a.sv = Sc{vin[0].scale, vin[0].inv_scale, vin[0].lo_scale, vin[0].inv_lo_scale};
    a.dep_amp = 0.0f;
    a.dep_i = -1000;
    if (p->src >= 0 && p->step < p->n_sig) {
        a.dep_amp = (float)p->h_sig[p->step];
        a.dep_i = (int)(p->src / g.plane);
        a.dep_j = (int)((p->src % g.plane) / g.sz);
        a.dep_k = (int)(p->src % g.sz);
    }
    if (p->rec_pending && p->n_rec > 0 && p->n_rec_steps < p->cap) {
        a.n_rec = p->n_rec;
        a.rec_idx = p->d_ridx;
        a.rec_w = p->d_rw;
        a.rec_out = p->d_trace + (size_t)p->n_rec_steps * p->n_rec;
        ++p->n_rec_steps;
    }
    a.status = p->d_status;
    a.wait_us = kWaitUs;
    a.xi_lo = p->xi_lo;
    a.xi_hi = p->xi_hi;
    const void* bases[8] = {P.hi, P.lo, vin[0].hi, vin[0].lo, vin[1].hi, vin[1].lo, vin[2].hi, vin[2].lo};
    PCK(launch_fused16(p->mode, a, p->maps, bases, p->stream));
    ++p->launches;
    p->cur ^= 1;
    p->vset ^= 1;
    ++p->step;
    p->rec_pending = true;
    return FDTD_OK;
}

template <int M>
int step_impl(FdtdB200Prec* p, int n, int audit_every)
{
    using A = typename Traits<M>::A;
    const PCoef<A>& cf = *reinterpret_cast<const PCoef<A>*>(M == kFP64 ? (const void*)&p->cf64 : (const void*)&p->cf32);
    const Grid& g = p->g;
    dim3 block(32, 8, 1), grid((g.sz / 4 + 31) / 32, (g.ny + 7) / 8, g.nx);
    for (int s = 0; s < n; ++s) {
        const bool audit = audit_every > 0 && p->step % audit_every == 0;
        if constexpr (M == kBF16 || M == kFP16 || M == kBF16C || M == kFP16C) {
            if (p->kernel == 1 && !audit) {
                const int rc = fused16_step<M>(p);
                if (rc != FDTD_OK) return rc;
                continue;
            }
        }
        if (p->rec_pending) {
            record_now<M>(p);
            p->rec_pending = false;
        }
        Field& P = p->f[p->cur];
        Field& PN = p->f[p->cur ^ 1];
        Field* V = vfields(p);
        k_src_rec<M><<<1, 32, 0, p->stream>>>(P, p->src, p->d_sig, p->step, p->n_sig, 0, nullptr, nullptr,
                                              nullptr, 0);
        double* aud = nullptr;
        if (audit) {
            if ((int)p->audit_steps.size() >= p->cap_audit) return FDTD_ERR_DIM;
            aud = p->d_audit + 2 * p->audit_steps.size();
            PCK(cudaMemsetAsync(aud, 0, 2 * sizeof(double), p->stream));
            p->audit_steps.push_back(p->step);
        }
        k_vel<M><<<grid, block, 0, p->stream>>>(g, cf, P, V[0], V[1], V[2], aud);
        k_pres<M><<<grid, block, 0, p->stream>>>(g, cf, P, PN, V[0], V[1], V[2]);
        p->launches += 3;
        p->cur ^= 1;
        ++p->step;
        record_now<M>(p);
    }
    if (p->rec_pending) {
        record_now<M>(p);
        p->rec_pending = false;
    }
    PCK(cudaGetLastError());
    return FDTD_OK;
}

// a load wait of the single-pass step that ran out (status word set)
int check_status(FdtdB200Prec* p)
{
    unsigned st[kStatusWords];
    PCK(cudaMemcpy(st, p->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st[kStatusTimeout] != 0xFFFFFFFFu) {
        record_cuda_error(cudaErrorLaunchTimeout, "fdtd_b200_prec_step: load wait timed out");
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

}  // namespace

extern "C" {

FdtdB200Prec* fdtd_b200_prec_create(int Nx, int Ny, int Nz, double dx, double c, double rho_air,
                                    int n_pml, const float* a6, int mode, float p_scale,
                                    float v_scale, int device)
{
    if (Nx <= 0 || Ny <= 0 || Nz <= 0 || dx <= 0 || c <= 0 || mode < 0 || mode > 5) return nullptr;
    if (p_scale <= 0.0f) p_scale = 1024.0f;
    if (v_scale <= 0.0f) v_scale = 524288.0f;
    if ((long long)Nx * Ny * Nz > INT_MAX) return nullptr;
    FdtdB200Prec* p = new FdtdB200Prec();
    p->mode = mode;
    if (device < 0) cudaGetDevice(&device);
    p->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete p;
        return nullptr;
    }
    const float ones[6] = {1, 1, 1, 1, 1, 1};
    if (!a6) a6 = ones;
    p->g.nx = Nx; p->g.ny = Ny; p->g.nz = Nz;
    p->g.sz = (Nz + kRowAlign - 1) / kRowAlign * kRowAlign;
    p->g.plane = (long long)Ny * p->g.sz;
    p->g.cells = (long long)Nx * p->g.plane;
    p->N = Nx * Ny * Nz;
    p->dx = dx; p->c = c; p->rho = rho_air;
    // float coefficients exactly as the engine computes them, double ones for FP64
    std::vector<float> t32;
    std::vector<double> t64;
    build<float>(p, (float)dx, (float)c, (float)rho_air, 0.77f, 1.732050808f, n_pml, a6, t32, p->cf32);
    build<double>(p, dx, c, rho_air, 0.77, 1.732050808, n_pml, a6, t64, p->cf64);
    x_interior_run(t32.data(), Nx, &p->xi_lo, &p->xi_hi);
    p->dt = mode == kFP64 ? p->cf64.dt : (double)p->cf32.dt;
    const size_t tb = mode == kFP64 ? t64.size() * 8 : t32.size() * 4;
    bool ok = cudaMalloc(&p->d_tab, tb) == cudaSuccess &&
              cudaMemcpy(p->d_tab, mode == kFP64 ? (const void*)t64.data() : (const void*)t32.data(), tb,
                         cudaMemcpyHostToDevice) == cudaSuccess;
    if (mode == kFP64) point_tables<double>(p->cf64, p->d_tab, p->g);
    else point_tables<float>(p->cf32, p->d_tab, p->g);
    const size_t fb = (size_t)p->g.cells * elem_bytes(mode);
    const bool fp16 = (mode == kFP16 || mode == kFP16C);
    for (int q = 0; q < 5 && ok; ++q) {
        Field& f = p->f[q];
        // BF16 forms are stored unscaled (the single-pass kernel relies on it)
        f.scale = fp16 ? (q < 2 ? p_scale : v_scale) : 1.0f;
        f.inv_scale = 1.0f / f.scale;
        f.lo_scale = mode == kFP16C ? 2048.0f : 1.0f;   // keeps half residuals out of subnormals
        f.inv_lo_scale = 1.0f / f.lo_scale;
        ok = cudaMalloc(&f.hi, fb) == cudaSuccess && cudaMemset(f.hi, 0, fb) == cudaSuccess;
        if (ok) p->allocs.push_back(f.hi);
        if (ok && compensated(mode)) {
            ok = cudaMalloc(&f.lo, fb) == cudaSuccess && cudaMemset(f.lo, 0, fb) == cudaSuccess;
            if (ok) p->allocs.push_back(f.lo);
        }
    }
    ok = ok && cudaMalloc(&p->d_status, sizeof(unsigned) * kStatusWords) == cudaSuccess &&
         cudaMemset(p->d_status, 0xFF, sizeof(unsigned) * kStatusWords) == cudaSuccess;
    if (!ok) {
        fdtd_b200_prec_destroy(p);
        return nullptr;
    }
    p->maps = f16_cache_create();
    p->kernel = f16_supported(mode, p->g) ? 1 : 0;
    return p;
}

void fdtd_b200_prec_destroy(FdtdB200Prec* p)
{
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    for (void* a : p->allocs) cudaFree(a);
    cudaFree(p->d_tab);
    cudaFree(p->d_sig);
    cudaFree(p->d_ridx);
    cudaFree(p->d_rw);
    cudaFree(p->d_trace);
    cudaFree(p->d_audit);
    cudaFree(p->d_status);
    f16_cache_destroy(p->maps);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

double fdtd_b200_prec_dt(const FdtdB200Prec* p) { return p ? p->dt : 0.0; }

int fdtd_b200_prec_set_source(FdtdB200Prec* p, int cell, const double* signal, int n)
{
    if (!p) return FDTD_ERR_NULL;
    if (cell < 0 || cell >= p->N || n < 0 || (n > 0 && !signal)) return FDTD_ERR_ARG;
    cudaSetDevice(p->device);
    cudaFree(p->d_sig);
    p->d_sig = nullptr;
    p->n_sig = 0;
    p->h_sig.clear();
    const int nz = p->g.nz, ny = p->g.ny;
    p->src = ((long long)(cell / nz / ny) * ny + (cell / nz) % ny) * p->g.sz + cell % nz;
    if (n > 0) {
        PCK(cudaMalloc(&p->d_sig, sizeof(double) * n));
        PCK(cudaMemcpy(p->d_sig, signal, sizeof(double) * n, cudaMemcpyHostToDevice));
        p->n_sig = n;
        p->h_sig.assign(signal, signal + n);
    }
    return FDTD_OK;
}

int fdtd_b200_prec_set_receivers(FdtdB200Prec* p, int n_rec, const int* idx8, const double* wgt8,
                                 int capacity, int audit_capacity)
{
    if (!p || (n_rec > 0 && (!idx8 || !wgt8))) return FDTD_ERR_NULL;
    cudaSetDevice(p->device);
    std::vector<long long> pi((size_t)n_rec * 8);
    for (size_t q = 0; q < pi.size(); ++q) {
        const int f = idx8[q];
        if (f < 0 || f >= p->N) return FDTD_ERR_ARG;
        const int nz = p->g.nz, ny = p->g.ny;
        pi[q] = ((long long)(f / nz / ny) * ny + (f / nz) % ny) * p->g.sz + f % nz;
    }
    cudaFree(p->d_ridx); cudaFree(p->d_rw); cudaFree(p->d_trace); cudaFree(p->d_audit);
    p->d_ridx = nullptr; p->d_rw = nullptr; p->d_trace = nullptr; p->d_audit = nullptr;
    p->n_rec = n_rec;
    p->cap = capacity;
    p->n_rec_steps = 0;
    p->audit_steps.clear();
    p->cap_audit = audit_capacity;
    if (n_rec > 0) {
        PCK(cudaMalloc(&p->d_ridx, sizeof(long long) * pi.size()));
        PCK(cudaMalloc(&p->d_rw, sizeof(double) * pi.size()));
        PCK(cudaMalloc(&p->d_trace, sizeof(double) * n_rec * (size_t)std::max(capacity, 1)));
        PCK(cudaMemcpy(p->d_ridx, pi.data(), sizeof(long long) * pi.size(), cudaMemcpyHostToDevice));
        PCK(cudaMemcpy(p->d_rw, wgt8, sizeof(double) * pi.size(), cudaMemcpyHostToDevice));
    }
    if (audit_capacity > 0) PCK(cudaMalloc(&p->d_audit, sizeof(double) * 2 * audit_capacity));
    return FDTD_OK;
}

int fdtd_b200_prec_step(FdtdB200Prec* p, int n_steps, int audit_every)
{
    if (!p) return FDTD_ERR_NULL;
    if (n_steps <= 0) return FDTD_OK;
    cudaSetDevice(p->device);
    switch (p->mode) {
        case kFP32: return step_impl<kFP32>(p, n_steps, audit_every);
        case kFP64: return step_impl<kFP64>(p, n_steps, audit_every);
        case kBF16: return step_impl<kBF16>(p, n_steps, audit_every);
        case kFP16: return step_impl<kFP16>(p, n_steps, audit_every);
        case kBF16C: return step_impl<kBF16C>(p, n_steps, audit_every);
        default: return step_impl<kFP16C>(p, n_steps, audit_every);
    }
}

int fdtd_b200_prec_set_kernel(FdtdB200Prec* p, int kernel)
{
    if (!p) return FDTD_ERR_NULL;
    if (kernel != 0 && kernel != 1) return FDTD_ERR_ARG;
    if (kernel == 1 && !f16_supported(p->mode, p->g)) return FDTD_ERR_ARG;
    p->kernel = kernel;
    return FDTD_OK;
}

int fdtd_b200_prec_get_kernel(const FdtdB200Prec* p) { return p ? p->kernel : -1; }

long long fdtd_b200_prec_launch_count(const FdtdB200Prec* p) { return p ? p->launches : 0; }

void* fdtd_b200_prec_stream(const FdtdB200Prec* p) { return p ? (void*)p->stream : nullptr; }

int fdtd_b200_prec_get_traces(FdtdB200Prec* p, double* out, int out_len, int* n_recorded)
{
    if (!p || !out) return FDTD_ERR_NULL;
    const long long need = (long long)p->n_rec_steps * p->n_rec;
    if (out_len < need) return FDTD_ERR_DIM;
    PCK(cudaStreamSynchronize(p->stream));
    if (check_status(p) != FDTD_OK) return FDTD_ERR_CUDA;
    if (need > 0) PCK(cudaMemcpy(out, p->d_trace, sizeof(double) * need, cudaMemcpyDeviceToHost));
    if (n_recorded) *n_recorded = p->n_rec_steps;
    return FDTD_OK;
}

// Energy audits: out3 = [n][3] (step, sum p^2 / (rho c^2) term, E) with
// E = dx^3/2 * (sum p^2/(rho c^2) + rho * sum v_old v_new).
int fdtd_b200_prec_get_energy(FdtdB200Prec* p, double* out3, int out_rows, int* n_out)
{
    if (!p || !out3) return FDTD_ERR_NULL;
    const int n = (int)p->audit_steps.size();
    if (out_rows < n) return FDTD_ERR_DIM;
    PCK(cudaStreamSynchronize(p->stream));
    std::vector<double> raw((size_t)2 * n);
    if (n > 0) PCK(cudaMemcpy(raw.data(), p->d_audit, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost));
    const double dx3 = p->dx * p->dx * p->dx, rc2 = p->rho * p->c * p->c;
    for (int q = 0; q < n; ++q) {
        out3[3 * q] = p->audit_steps[q];
        out3[3 * q + 1] = raw[2 * q] / rc2;
        out3[3 * q + 2] = 0.5 * dx3 * (raw[2 * q] / rc2 + p->rho * raw[2 * q + 1]);
    }
    if (n_out) *n_out = n;
    return FDTD_OK;
}

// Current pressure field, reference layout, as double.
int fdtd_b200_prec_get_pressure(FdtdB200Prec* p, double* out, int out_len)
{
    if (!p || !out) return FDTD_ERR_NULL;
    if (out_len != p->N) return FDTD_ERR_DIM;
    PCK(cudaStreamSynchronize(p->stream));
    if (check_status(p) != FDTD_OK) return FDTD_ERR_CUDA;
    const Field& f = p->f[p->cur];
    const size_t eb = elem_bytes(p->mode);
    std::vector<unsigned char> hi((size_t)p->g.cells * eb), lo;
    PCK(cudaMemcpy(hi.data(), f.hi, hi.size(), cudaMemcpyDeviceToHost));
    if (compensated(p->mode)) {
        lo.resize(hi.size());
        PCK(cudaMemcpy(lo.data(), f.lo, lo.size(), cudaMemcpyDeviceToHost));
    }
    auto h2f = [&](const unsigned char* b) -> float {
        uint16_t u;
        memcpy(&u, b, 2);
        if (p->mode == kBF16 || p->mode == kBF16C) {
            uint32_t w = (uint32_t)u << 16;
            float x;
            memcpy(&x, &w, 4);
            return x;
        }
        __half_raw r;
        r.x = u;
        return __half2float(__half(r));
    };
    const Grid& g = p->g;
    for (int i = 0; i < g.nx; ++i)
        for (int j = 0; j < g.ny; ++j)
            for (int k = 0; k < g.nz; ++k) {
                const size_t id = ((size_t)i * g.ny + j) * g.sz + k;
                double v;
                if (p->mode == kFP64) memcpy(&v, &hi[id * 8], 8);
                else if (p->mode == kFP32) { float x; memcpy(&x, &hi[id * 4], 4); v = x; }
                else {
                    float x = h2f(&hi[id * 2]);
                    if (!lo.empty()) x = x + h2f(&lo[id * 2]) * f.inv_lo_scale;
                    v = (double)(x * f.inv_scale);
                }
                out[k + g.nz * (j + (size_t)g.ny * i)] = v;
            }
    return FDTD_OK;
}

}  // extern "C"
