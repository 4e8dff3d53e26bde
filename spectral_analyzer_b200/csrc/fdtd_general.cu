/*
 * fdtd_general.cu — two-pass step kernels for arbitrary scenes, plus the
 * small kernels around the step (plate, deposits, samplers, stability check).
 *
 * The two-pass step handles everything the reference's pressure_step does
 * (csrc/kernels/acoustic_fdtd.cpp:1081-1241): rigid walls, cut-cell face
 * fractions, closed faces and the moving-plate faces.  It costs one extra
 * read of P and V compared with the fused single pass (fdtd_fused.cu), which
 * open rooms use.  Memory bound: velocity pass 28 B/cell, pressure pass
 * 20 B/cell (+ fractions and solid mask when present).
 */
#include "fdtd_internal.h"

#include <math.h>

namespace fdtd {

namespace {

__device__ __forceinline__ float cell_alpha(const Tables& tb, int i, float ay, float az)
{
    return fmaxf(fmaxf(__ldg(tb.ax + i), ay), az);
}

// Velocity update on the three staggered face sets (acoustic_fdtd.cpp:1099-1148),
// then closed faces (fraction == 0) are zeroed (:1152-1154).  One thread per
// (i, j, k) handles Vx(i+1/2,j,k), Vy(i,j+1/2,k) and Vz(i,j,k+1/2) where they exist.
__global__ void __launch_bounds__(256) k_velocity_general(
    Grid g, Coef cf, Tables tb, const float* __restrict__ p, float* __restrict__ vx,
    float* __restrict__ vy, float* __restrict__ vz, const float* __restrict__ fx,
    const float* __restrict__ fy, const float* __restrict__ fz)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.nz || j >= g.ny) return;
    const long long id = ((long long)i * g.ny + j) * g.sz + k;
    const float ay = __ldg(tb.ay + j), az = __ldg(tb.az + k);
    const float ac = cell_alpha(tb, i, ay, az);
    const float pc = p[id];

    if (i < g.nx - 1) {
        const float pr = p[id + g.plane];
        float grad;
        if (i > 0 && i < g.nx - 2)
            grad = fadd(fmul(cf.c1, fsub(pr, pc)),
                        fmul(cf.c2, fsub(p[id + 2 * g.plane], p[id - g.plane])));
        else
            grad = fsub(pr, pc);
        const float ar = cell_alpha(tb, i + 1, ay, az);
        float v = fmul(fsub(vx[id], fmul(cf.vc, grad)), face_damp(ac, ar, cf.dt));
        if (fx && fx[id] == 0.0f) v = 0.0f;
        vx[id] = v;
    }
    if (j < g.ny - 1) {
        const float pr = p[id + g.sz];
        float grad;
        if (j > 0 && j < g.ny - 2)
            grad = fadd(fmul(cf.c1, fsub(pr, pc)),
                        fmul(cf.c2, fsub(p[id + 2 * g.sz], p[id - g.sz])));
        else
            grad = fsub(pr, pc);
        const float ar = cell_alpha(tb, i, __ldg(tb.ay + j + 1), az);
        float v = fmul(fsub(vy[id], fmul(cf.vc, grad)), face_damp(ac, ar, cf.dt));
        if (fy && fy[id] == 0.0f) v = 0.0f;
        vy[id] = v;
    }
    if (k < g.nz - 1) {
        const float pr = p[id + 1];
        float grad;
        if (k > 0 && k < g.nz - 2)
            grad = fadd(fmul(cf.c1, fsub(pr, pc)), fmul(cf.c2, fsub(p[id + 2], p[id - 1])));
        else
            grad = fsub(pr, pc);
        const float ar = cell_alpha(tb, i, ay, __ldg(tb.az + k + 1));
        float v = fmul(fsub(vz[id], fmul(cf.vc, grad)), face_damp(ac, ar, cf.dt));
        if (fz && fz[id] == 0.0f) v = 0.0f;
        vz[id] = v;
    }
}

// Pressure update from the 4th-order divergence (acoustic_fdtd.cpp:894-952,
// :1176-1234).  Faces outside the grid read as zero; with fractions each face
// is scaled by its open fraction; solid cells are skipped (they stay zero).
__global__ void __launch_bounds__(256) k_pressure_general(
    Grid g, Coef cf, Tables tb, const float* __restrict__ p, float* __restrict__ pn,
    const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz,
    const float* __restrict__ fx, const float* __restrict__ fy, const float* __restrict__ fz,
    const uint8_t* __restrict__ solid)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.nz || j >= g.ny) return;
    const long long id = ((long long)i * g.ny + j) * g.sz + k;
    if (solid && solid[id]) return;

#define FX(q) (fx ? fmul(vx[q], fx[q]) : vx[q])
#define FY(q) (fy ? fmul(vy[q], fy[q]) : vy[q])
#define FZ(q) (fz ? fmul(vz[q], fz[q]) : vz[q])
    const long long P = g.plane, S = g.sz;
    const float xp = (i < g.nx - 1) ? FX(id) : 0.0f;
    const float xm = (i > 0) ? FX(id - P) : 0.0f;
    const float xpp = (i < g.nx - 2) ? FX(id + P) : 0.0f;
    const float xmm = (i > 1) ? FX(id - 2 * P) : 0.0f;
    const float yp = (j < g.ny - 1) ? FY(id) : 0.0f;
    const float ym = (j > 0) ? FY(id - S) : 0.0f;
    const float ypp = (j < g.ny - 2) ? FY(id + S) : 0.0f;
    const float ymm = (j > 1) ? FY(id - 2 * S) : 0.0f;
    const float zp = (k < g.nz - 1) ? FZ(id) : 0.0f;
    const float zm = (k > 0) ? FZ(id - 1) : 0.0f;
    const float zpp = (k < g.nz - 2) ? FZ(id + 1) : 0.0f;
    const float zmm = (k > 1) ? FZ(id - 2) : 0.0f;
#undef FX
#undef FY
#undef FZ
    const float d1 = fadd(fadd(fsub(xp, xm), fsub(yp, ym)), fsub(zp, zm));
    const float d2 = fadd(fadd(fsub(xpp, xmm), fsub(ypp, ymm)), fsub(zpp, zmm));
    const float dv = fadd(fmul(cf.c1, d1), fmul(cf.c2, d2));
    const float pd = fminf(fminf(__ldg(tb.px + i), __ldg(tb.py + j)), __ldg(tb.pz + k));
    pn[id] = fmul(fsub(p[id], fmul(cf.bulk, dv)), pd);
}

// Kirchhoff plate step (acoustic_fdtd.cpp:984-1053), one thread per active node.
// A node whose new displacement is non-finite or above 0.02 m records its
// ordinal in status[kStatusPlate] (the host reports the lowest one).
__global__ void k_plate_step(int n_act, const int* __restrict__ act, const int* __restrict__ nb13,
                             const long long* __restrict__ above,
                             const long long* __restrict__ below, const float* __restrict__ w,
                             const float* __restrict__ wp, float* __restrict__ wt,
                             const float* __restrict__ ext, const float* __restrict__ p,
                             PlateCoef pc, unsigned* __restrict__ status)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_act) return;
    const float W13[13] = {20.f, -8.f, -8.f, -8.f, -8.f, 2.f, 2.f, 2.f, 2.f, 1.f, 1.f, 1.f, 1.f};
    const int pidx = act[q];
    const int* nb = nb13 + 13 * q;
    float bh = 0.0f, bhp = 0.0f;
    for (int t = 0; t < 13; ++t) bh = fadd(bh, fmul(W13[t], w[nb[t]]));
    const float pa = above[q] >= 0 ? p[above[q]] : 0.0f;
    const float pb = below[q] >= 0 ? p[below[q]] : 0.0f;
    const float fb = ext[pidx];
    for (int t = 0; t < 13; ++t) bhp = fadd(bhp, fmul(W13[t], wp[nb[t]]));
    const float vel = fsub(w[pidx], wp[pidx]);
    float wn = fadd(w[pidx], fmul(pc.vd, vel));
    wn = fadd(wn, fmul(pc.a, fadd(fsub(pb, pa), fb)));
    wn = fsub(wn, fmul(pc.bh, bh));
    wn = fsub(wn, fmul(pc.bk, fsub(bh, bhp)));
    if (!isfinite(wn) || fabsf(wn) > 0.02f) atomicMin(status + kStatusPlate, (unsigned)q);
    wt[pidx] = wn;
}

// Plate velocity imposed on the Vz faces beside each active node (acoustic_fdtd.cpp:1158-1163).
__global__ void k_plate_inject(int n_act, const int* __restrict__ act,
                               const long long* __restrict__ vzb, const long long* __restrict__ vza,
                               const float* __restrict__ w, const float* __restrict__ wp,
                               float inv_dt, float* __restrict__ vz)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_act) return;
    const int pidx = act[q];
    const float v = fmul(fsub(w[pidx], wp[pidx]), inv_dt);
    if (vzb[q] >= 0) vz[vzb[q]] = v;
    if (vza[q] >= 0) vz[vza[q]] = v;
}

// One deposit of the open-cell rule (acoustic_fdtd.cpp:840-872).  The amplitude
// is signal[step] when a signal is given, else `amp`; zero amplitude is a no-op.
__global__ void k_deposit(Deposit d, const float* __restrict__ signal, int step, float amp,
                          float* __restrict__ p)
{
    deposit_apply(d, signal ? signal[step] : amp, p);
}

// out[r] = sum_t w[r*taps+t] * f[idx[r*taps+t]] in tap order; from_zero starts
// the running sum at 0.0f (the direct samplers, acoustic_fdtd.cpp:1380-1389),
// otherwise at the first product (the precomputed samplers, :1673-1674).
__global__ void k_wsum(const float* __restrict__ f, const long long* __restrict__ idx,
                       const float* __restrict__ w, int n_out, int taps, int from_zero,
                       float* __restrict__ out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_out) return;
    const long long* id = idx + (long long)taps * r;
    const float* ww = w + (long long)taps * r;
    float s;
    int t0;
    if (from_zero) { s = 0.0f; t0 = 0; }
    else { s = fmul(ww[0], f[id[0]]); t0 = 1; }
    for (int t = t0; t < taps; ++t) s = fadd(s, fmul(ww[t], f[id[t]]));
    out[r] = s;
}

// Stability check (acoustic_fdtd.cpp:1245-1268): cells phase, phase+1013, ...
// (reference flat order) that are non-finite or beyond +-2e3 Pa record their
// flat index; the latch keeps the first failing step for async stepping.
__global__ void k_check(Grid g, const float* __restrict__ p, long long n_cells, int phase,
                        unsigned* __restrict__ status, int step)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long q = phase + t * kCheckStride;
    if (q >= n_cells) return;
    const int k = (int)(q % g.nz);
    const long long ij = q / g.nz;
    const int j = (int)(ij % g.ny);
    const long long i = ij / g.ny;
    const float v = p[(i * g.ny + j) * g.sz + k];
    if (!isfinite(v) || v > 2e3f || v < -2e3f) {
        atomicMin(status + kStatusCell, (unsigned)q);
        atomicCAS(status + kStatusLatch, 0xFFFFFFFFu, (unsigned)step);
    }
}

}  // namespace

cudaError_t launch_velocity_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* vx, float* vy, float* vz,
                                    const float* fx, const float* fy, const float* fz,
                                    cudaStream_t s)
{
    dim3 block(32, 8, 1);
    dim3 grid((g.nz + 31) / 32, (g.ny + 7) / 8, g.nx);
    k_velocity_general<<<grid, block, 0, s>>>(g, cf, tb, p, vx, vy, vz, fx, fy, fz);
    return cudaGetLastError();
}

cudaError_t launch_pressure_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* pn, const float* vx, const float* vy,
                                    const float* vz, const float* fx, const float* fy,
                                    const float* fz, const uint8_t* solid, cudaStream_t s)
{
    dim3 block(32, 8, 1);
    dim3 grid((g.nz + 31) / 32, (g.ny + 7) / 8, g.nx);
    k_pressure_general<<<grid, block, 0, s>>>(g, cf, tb, p, pn, vx, vy, vz, fx, fy, fz, solid);
    return cudaGetLastError();
}

cudaError_t launch_plate_step(int n_act, const int* act, const int* nb13, const long long* above,
                              const long long* below, const float* w, const float* wp, float* wt,
                              const float* ext, const float* p, const PlateCoef& pc,
                              unsigned* status, cudaStream_t s)
{
    if (n_act <= 0) return cudaSuccess;
    k_plate_step<<<(n_act + 127) / 128, 128, 0, s>>>(n_act, act, nb13, above, below, w, wp, wt,
                                                     ext, p, pc, status);
    return cudaGetLastError();
}

cudaError_t launch_plate_inject(int n_act, const int* act, const long long* vzb,
                                const long long* vza, const float* w, const float* wp,
                                float inv_dt, float* vz, cudaStream_t s)
{
    if (n_act <= 0) return cudaSuccess;
    k_plate_inject<<<(n_act + 127) / 128, 128, 0, s>>>(n_act, act, vzb, vza, w, wp, inv_dt, vz);
    return cudaGetLastError();
}

cudaError_t launch_deposit(const Deposit& d, const float* signal, int step, float amp, float* p,
                           cudaStream_t s)
{
    k_deposit<<<1, 1, 0, s>>>(d, signal, step, amp, p);
    return cudaGetLastError();
}

cudaError_t launch_wsum(const float* f, const long long* idx, const float* w, int n_out, int taps,
                        int from_zero, float* out, cudaStream_t s)
{
    if (n_out <= 0) return cudaSuccess;
    k_wsum<<<(n_out + 127) / 128, 128, 0, s>>>(f, idx, w, n_out, taps, from_zero, out);
    return cudaGetLastError();
}

cudaError_t launch_check(const Grid& g, const float* p, long long n_cells, int phase,
                         unsigned* status, int step, cudaStream_t s)
{
    if (phase >= n_cells) return cudaSuccess;
    const long long n = (n_cells - phase + kCheckStride - 1) / kCheckStride;
    const int blocks = (int)((n + 255) / 256);
    k_check<<<blocks, 256, 0, s>>>(g, p, n_cells, phase, status, step);
    return cudaGetLastError();
}

}  // namespace fdtd
