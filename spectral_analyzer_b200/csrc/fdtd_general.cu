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

__device__ __forceinline__ float4 ld4(const float* p, long long i) { return *reinterpret_cast<const float4*>(p + i); }
__device__ __forceinline__ void st4(float* p, long long i, const float (&v)[4])
{
    *reinterpret_cast<float4*>(p + i) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void unpack(const float4& x, float (&v)[4]) { v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w; }

// Threads own four consecutive cells k0 .. k0+3 of a row (k0 a multiple of 4;
// rows start on 8-float boundaries, so every float4 access is aligned).  The
// (row, group) pairs of a plane are numbered consecutively over 1-D blocks,
// so no lane idles when Nz/4 is not a multiple of the warp width (Nz = 74:
// 19 groups per row), and consecutive lanes read consecutive 16-byte groups.
#define GEN_INDEX                                                          \
    const int nq_ = (g.nz + 3) >> 2;                                       \
    const int t_ = blockIdx.x * blockDim.x + threadIdx.x;                  \
    if (t_ >= g.ny * nq_) return;                                          \
    const int j = t_ / nq_;                                                \
    const int k0 = 4 * (t_ - j * nq_);                                     \
    const int i = blockIdx.y;                                              \
    const long long id = ((long long)i * g.ny + j) * g.sz + k0;

// Velocity update on the three staggered face sets (acoustic_fdtd.cpp:1099-1148),
// then closed faces (fraction == 0) are zeroed (:1152-1154).  A thread handles
// Vx(i+1/2,j,k), Vy(i,j+1/2,k) and Vz(i,j,k+1/2) of its four cells where they
// exist; faces that do not exist (and the row padding) keep their stored zero.
__global__ void __launch_bounds__(256) k_velocity_general(
    Grid g, Coef cf, Tables tb, const float* __restrict__ p, float* __restrict__ vx,
    float* __restrict__ vy, float* __restrict__ vz, const float* __restrict__ fx,
    const float* __restrict__ fy, const float* __restrict__ fz, const unsigned* __restrict__ gate,
    PlateFaces pf)
{
    if (gate && gate[kStatusPlate] != 0xFFFFFFFFu) return;   // this step's plate update failed
    if (pf.m > 0 && blockIdx.x == 0 && blockIdx.y == 0)      // the consumed plate forces
        for (int q = threadIdx.x; q < pf.m; q += blockDim.x) pf.ext[pf.pack[q].x] = 0.0f;
    GEN_INDEX
    const float ay = __ldg(tb.ay + j), axi = __ldg(tb.ax + i);
    float pc[4], az4[4], ac[4];
    unpack(ld4(p, id), pc);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        az4[q] = (k0 + q < g.nz) ? __ldg(tb.az + k0 + q) : 0.0f;
        ac[q] = fmaxf(fmaxf(axi, ay), az4[q]);
    }
    if (i < g.nx - 1) {
        const bool fourth = i > 0 && i < g.nx - 2;
        float pr[4], pm[4] = {}, p2[4] = {}, v[4], fr[4] = {1.f, 1.f, 1.f, 1.f};
        unpack(ld4(p, id + g.plane), pr);
        if (fourth) {
            unpack(ld4(p, id - g.plane), pm);
            unpack(ld4(p, id + 2 * g.plane), p2);
        }
        unpack(ld4(vx, id), v);
        if (fx) unpack(ld4(fx, id), fr);
        const float axr = __ldg(tb.ax + i + 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (k0 + q >= g.nz) continue;
            const float grad = fourth ? fadd(fmul(cf.c1, fsub(pr[q], pc[q])), fmul(cf.c2, fsub(p2[q], pm[q])))
                                      : fsub(pr[q], pc[q]);
            float nv = fmul(fsub(v[q], fmul(cf.vc, grad)), face_damp(ac[q], fmaxf(fmaxf(axr, ay), az4[q]), cf.dt));
            if (fx && fr[q] == 0.0f) nv = 0.0f;
            v[q] = nv;
        }
        st4(vx, id, v);
    }
    if (j < g.ny - 1) {
        const bool fourth = j > 0 && j < g.ny - 2;
        float pr[4], pm[4] = {}, p2[4] = {}, v[4], fr[4] = {1.f, 1.f, 1.f, 1.f};
        unpack(ld4(p, id + g.sz), pr);
        if (fourth) {
            unpack(ld4(p, id - g.sz), pm);
            unpack(ld4(p, id + 2 * g.sz), p2);
        }
        unpack(ld4(vy, id), v);
        if (fy) unpack(ld4(fy, id), fr);
        const float ayr = __ldg(tb.ay + j + 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (k0 + q >= g.nz) continue;
            const float grad = fourth ? fadd(fmul(cf.c1, fsub(pr[q], pc[q])), fmul(cf.c2, fsub(p2[q], pm[q])))
                                      : fsub(pr[q], pc[q]);
            float nv = fmul(fsub(v[q], fmul(cf.vc, grad)), face_damp(ac[q], fmaxf(fmaxf(axi, ayr), az4[q]), cf.dt));
            if (fy && fr[q] == 0.0f) nv = 0.0f;
            v[q] = nv;
        }
        st4(vy, id, v);
    }
    {
        // P at k0-1 .. k0+5: e[t] = P[k0 - 1 + t]
        float e[7], v[4], fr[4] = {1.f, 1.f, 1.f, 1.f};
        e[0] = k0 > 0 ? p[id - 1] : 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) e[q + 1] = pc[q];
        e[5] = k0 + 4 < g.nz ? p[id + 4] : 0.0f;
        e[6] = k0 + 5 < g.nz ? p[id + 5] : 0.0f;
        unpack(ld4(vz, id), v);
        if (fz) unpack(ld4(fz, id), fr);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            if (k >= g.nz - 1) continue;
            const float grad = (k > 0 && k < g.nz - 2)
                                   ? fadd(fmul(cf.c1, fsub(e[q + 2], e[q + 1])), fmul(cf.c2, fsub(e[q + 3], e[q])))
                                   : fsub(e[q + 2], e[q + 1]);
            float nv = fmul(fsub(v[q], fmul(cf.vc, grad)),
                            face_damp(ac[q], fmaxf(fmaxf(axi, ay), __ldg(tb.az + k + 1)), cf.dt));
            if (fz && fr[q] == 0.0f) nv = 0.0f;
            v[q] = nv;
        }
        if (pf.code && k0 <= pf.iz && pf.iz - 1 <= k0 + 3) {   // the plate's faces
            const int node = j + g.ny * i;
            const unsigned c = pf.code[node];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int k = k0 + q;
                if ((k == pf.iz - 1 && (c & 1u)) || (k == pf.iz && (c & 2u)))
                    v[q] = fmul(fsub(pf.w[node], pf.wp[node]), pf.inv_dt);
            }
        }
        st4(vz, id, v);
    }
}

// The pressure update of cells k0 .. k0+3 of row (i, j), id = their padded index.
__device__ __forceinline__ void pressure_cells4(const Grid& g, const Coef& cf, const Tables& tb,
                                                const float* __restrict__ p, float* __restrict__ pn,
                                                const float* __restrict__ vx, const float* __restrict__ vy,
                                                const float* __restrict__ vz, const float* __restrict__ fx,
                                                const float* __restrict__ fy, const float* __restrict__ fz,
                                                const uint8_t* __restrict__ solid, int i, int j, int k0,
                                                long long id)
{
    const long long P = g.plane, S = g.sz;
    // face values times their fractions, four cells at a time (zero when absent)
    auto face4 = [&](const float* v, const float* f, long long q, bool exists, float (&out)[4]) {
        if (!exists) {
            out[0] = out[1] = out[2] = out[3] = 0.0f;
            return;
        }
        unpack(ld4(v, q), out);
        if (f) {
            float fr[4];
            unpack(ld4(f, q), fr);
#pragma unroll
            for (int t = 0; t < 4; ++t) out[t] = fmul(out[t], fr[t]);
        }
    };
    float xp[4], xm[4], xpp[4], xmm[4], yp[4], ym[4], ypp[4], ymm[4];
    face4(vx, fx, id, i < g.nx - 1, xp);
    face4(vx, fx, id - P, i > 0, xm);
    face4(vx, fx, id + P, i < g.nx - 2, xpp);
    face4(vx, fx, id - 2 * P, i > 1, xmm);
    face4(vy, fy, id, j < g.ny - 1, yp);
    face4(vy, fy, id - S, j > 0, ym);
    face4(vy, fy, id + S, j < g.ny - 2, ypp);
    face4(vy, fy, id - 2 * S, j > 1, ymm);
    // Vz (times fraction) at k0-2 .. k0+4: e[t] = FZ[k0 - 2 + t]
    auto fzv = [&](long long q) { return fz ? fmul(vz[q], fz[q]) : vz[q]; };
    float e[7], c4[4], pc[4], out[4];
    face4(vz, fz, id, true, c4);
    e[0] = k0 >= 2 ? fzv(id - 2) : 0.0f;
    e[1] = k0 >= 1 ? fzv(id - 1) : 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) e[q + 2] = c4[q];
    e[6] = k0 + 4 < g.nz ? fzv(id + 4) : 0.0f;
    unpack(ld4(p, id), pc);
    uint32_t sol = 0;
    if (solid) sol = *reinterpret_cast<const uint32_t*>(solid + id);
    const float pxy = fminf(__ldg(tb.px + i), __ldg(tb.py + j));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = k0 + q;
        out[q] = 0.0f;
        if (k >= g.nz || ((sol >> (8 * q)) & 0xFFu)) continue;
        const float zp = (k < g.nz - 1) ? e[q + 2] : 0.0f;
        const float zm = (k > 0) ? e[q + 1] : 0.0f;
        const float zpp = (k < g.nz - 2) ? e[q + 3] : 0.0f;
        const float zmm = (k > 1) ? e[q] : 0.0f;
        const float d1 = fadd(fadd(fsub(xp[q], xm[q]), fsub(yp[q], ym[q])), fsub(zp, zm));
        const float d2 = fadd(fadd(fsub(xpp[q], xmm[q]), fsub(ypp[q], ymm[q])), fsub(zpp, zmm));
        const float dv = fadd(fmul(cf.c1, d1), fmul(cf.c2, d2));
        out[q] = fmul(fsub(pc[q], fmul(cf.bulk, dv)), fminf(pxy, __ldg(tb.pz + k)));
    }
    st4(pn, id, out);
}

// Pressure update from the 4th-order divergence (acoustic_fdtd.cpp:894-952,
// :1176-1234).  Faces outside the grid read as zero; with fractions each face
// is scaled by its open fraction; solid cells are skipped (they stay zero in
// both pressure buffers, so the thread writes zero there).
__global__ void __launch_bounds__(256) k_pressure_general(
    Grid g, Coef cf, Tables tb, const float* __restrict__ p, float* __restrict__ pn,
    const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz,
    const float* __restrict__ fx, const float* __restrict__ fy, const float* __restrict__ fz,
    const uint8_t* __restrict__ solid, const unsigned* __restrict__ gate)
{
    GEN_INDEX
    if (gate && gate[kStatusPlate] != 0xFFFFFFFFu) return;   // this step's plate update failed
    pressure_cells4(g, cf, tb, p, pn, vx, vy, vz, fx, fy, fz, solid, i, j, k0, id);
}

// The same update on a list of four-cell groups (padded index of each group's
// first cell): after the single-pass walled step, the cells whose divergence
// reads a plate face, recomputed once the plate has set those faces.
__global__ void __launch_bounds__(256) k_pressure_groups(
    Grid g, Coef cf, Tables tb, const float* __restrict__ p, float* __restrict__ pn,
    const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz,
    const float* __restrict__ fx, const float* __restrict__ fy, const float* __restrict__ fz,
    const uint8_t* __restrict__ solid, const long long* __restrict__ groups, int n_groups)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_groups) return;
    const long long id = groups[t];
    const int i = (int)(id / g.plane);
    const long long r = id - (long long)i * g.plane;
    const int j = (int)(r / g.sz), k0 = (int)(r - (long long)j * g.sz);
    pressure_cells4(g, cf, tb, p, pn, vx, vy, vz, fx, fy, fz, solid, i, j, k0, id);
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
                               float inv_dt, float* __restrict__ vz, const unsigned* __restrict__ gate)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_act) return;
    if (gate && gate[kStatusPlate] != 0xFFFFFFFFu) return;   // this step's plate update failed
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
                        unsigned* __restrict__ status, int step, const unsigned* __restrict__ gate)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long q = phase + t * kCheckStride;
    if (q >= n_cells) return;
    if (gate && gate[kStatusPlate] != 0xFFFFFFFFu) return;   // this step's plate update failed

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


// Zeroes n floats unless this step's plate update failed (the consumed plate
// forces of a step whose success is only known after it ran).
__global__ void k_zero_gated(float* __restrict__ x, int n, const unsigned* __restrict__ gate)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n || gate[kStatusPlate] != 0xFFFFFFFFu) return;
    x[q] = 0.0f;
}

// The pending plate forces, sent as (node, value) pairs: written into the
// device force buffer (all other entries are zero there).
__global__ void k_ext_scatter(float* __restrict__ ext, const int2* __restrict__ pack, int m)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < m) ext[pack[q].x] = __int_as_float(pack[q].y);
}

// One plane of a field across the given axis, rows of the remaining two axes
// in (i, j, k) order: axis 0 -> (Ny, Nz), 1 -> (Nx, Nz), 2 -> (Nx, Ny).
__global__ void k_slice(const float* __restrict__ f, Grid g, int axis, int idx, float* __restrict__ out,
                        int na, int nb)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)na * nb) return;
    const long long a = q / nb, b = q % nb;
    const long long off = axis == 0 ? ((long long)idx * g.ny + a) * g.sz + b
                        : axis == 1 ? (a * g.ny + idx) * g.sz + b
                                    : (a * g.ny + b) * g.sz + idx;
    out[q] = f[off];
}
}  // namespace

cudaError_t launch_velocity_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* vx, float* vy, float* vz,
                                    const float* fx, const float* fy, const float* fz,
                                    cudaStream_t s, const unsigned* gate, const PlateFaces* pf)
{
    dim3 block(256, 1, 1);
    dim3 grid((g.ny * ((g.nz + 3) / 4) + 255) / 256, g.nx, 1);
    k_velocity_general<<<grid, block, 0, s>>>(g, cf, tb, p, vx, vy, vz, fx, fy, fz, gate,
                                              pf ? *pf : PlateFaces());
    return cudaGetLastError();
}

cudaError_t launch_pressure_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* pn, const float* vx, const float* vy,
                                    const float* vz, const float* fx, const float* fy,
                                    const float* fz, const uint8_t* solid, cudaStream_t s,
                                    const unsigned* gate)
{
    dim3 block(256, 1, 1);
    dim3 grid((g.ny * ((g.nz + 3) / 4) + 255) / 256, g.nx, 1);
    k_pressure_general<<<grid, block, 0, s>>>(g, cf, tb, p, pn, vx, vy, vz, fx, fy, fz, solid, gate);
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

cudaError_t launch_pressure_groups(const Grid& g, const Coef& cf, const Tables& tb, const float* p, float* pn,
                                   const float* vx, const float* vy, const float* vz, const float* fx,
                                   const float* fy, const float* fz, const uint8_t* solid,
                                   const long long* groups, int n_groups, cudaStream_t s)
{
    if (n_groups <= 0) return cudaSuccess;
    k_pressure_groups<<<(n_groups + 255) / 256, 256, 0, s>>>(g, cf, tb, p, pn, vx, vy, vz, fx, fy, fz, solid,
                                                             groups, n_groups);
    return cudaGetLastError();
}

cudaError_t launch_plate_inject(int n_act, const int* act, const long long* vzb,
                                const long long* vza, const float* w, const float* wp,
                                float inv_dt, float* vz, cudaStream_t s, const unsigned* gate)
{
    if (n_act <= 0) return cudaSuccess;
    k_plate_inject<<<(n_act + 127) / 128, 128, 0, s>>>(n_act, act, vzb, vza, w, wp, inv_dt, vz, gate);
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
                         unsigned* status, int step, cudaStream_t s, const unsigned* gate)
{
    if (phase >= n_cells) return cudaSuccess;
    const long long n = (n_cells - phase + kCheckStride - 1) / kCheckStride;
    const int blocks = (int)((n + 255) / 256);
    k_check<<<blocks, 256, 0, s>>>(g, p, n_cells, phase, status, step, gate);
    return cudaGetLastError();
}

cudaError_t launch_zero_gated(float* x, int n, const unsigned* gate, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_zero_gated<<<(n + 255) / 256, 256, 0, s>>>(x, n, gate);
    return cudaGetLastError();
}

cudaError_t launch_ext_scatter(float* ext, const int2* pack, int m, cudaStream_t s)
{
    if (m <= 0) return cudaSuccess;
    k_ext_scatter<<<(m + 255) / 256, 256, 0, s>>>(ext, pack, m);
    return cudaGetLastError();
}

cudaError_t launch_slice(const float* f, const Grid& g, int axis, int idx, float* out, int na, int nb,
                         cudaStream_t s)
{
    const long long n = (long long)na * nb;
    if (n <= 0) return cudaSuccess;
    k_slice<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f, g, axis, idx, out, na, nb);
    return cudaGetLastError();
}

}  // namespace fdtd
