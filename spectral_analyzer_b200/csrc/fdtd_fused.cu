/*
 * fdtd_fused.cu — single-pass velocity+pressure step for open rooms.
 *
 * One launch advances V^{n-1/2} -> V^{n+1/2} and P^n -> P^{n+1} over the whole
 * grid, reading each field once and writing each once: 16 B read + 16 B
 * written per cell-update, the HBM floor of the scheme (the two-pass step
 * moves 48 B).
 *
 * Decomposition (2.5D): a CTA owns a TJ x 128 tile of (j, k) columns — one warp
 * per row j, four consecutive k per lane (float4) — and marches along i over a
 * segment [i_beg, i_end).  Iteration u of the march
 *   - computes the new Vx on face f = u-2 of the own columns from P^n planes
 *     f-1 .. f+2 and keeps the last four faces in a register queue;
 *   - computes, for plane i = u-3, the new Vy of rows j0-2 .. j0+TJ and the new
 *     Vz of faces k0-2 .. k0+128: the faces outside the tile are recomputed
 *     here from V^{n-1/2}, never read back from a neighbour, so the step writes
 *     the other velocity set;
 *   - finishes P^{n+1} of plane i from the 4th-order divergence.
 * Loads go through a ring of shared-memory stages filled with cp.async
 * (16-byte chunks, zero-filled outside the grid) D planes ahead of use; each
 * thread's chunk offsets are computed once, before the march.  Halo rows and
 * columns are shared with neighbouring CTAs that march at the same pace, so
 * they are served mostly from L2.
 *
 * Absorption: inside the x-interior (alpha_x = 0 on the planes involved, all
 * but the 2*n_pml PML planes) a face's damping depends on (j, k) only and is a
 * per-thread constant computed once; PML planes take the general path.  Both
 * paths evaluate the same expression, so results do not depend on the path.
 *
 * Arithmetic is the reference's (csrc/kernels/acoustic_fdtd.cpp:1099-1148 for
 * the velocity, :894-952 and :1176-1234 for the pressure) with every operation
 * separately rounded (fadd/fsub/fmul): bit-identical to the two-pass kernels
 * and to the reference.
 */
#include "fdtd_internal.h"

namespace fdtd {

namespace {

template <int TJ_, int D_>
struct Cfg {
    static constexpr int TJ = TJ_;              // rows per CTA = warps
    static constexpr int TK = 128;              // 32 lanes x float4
    static constexpr int D = D_;                // prefetch distance (iterations)
    static constexpr int NT = 32 * TJ;
    static constexpr int PR = TJ + 6;           // P stage rows j0-3 .. j0+TJ+2
    static constexpr int PC = TK + 8;           // P stage cols k0-4 .. k0+TK+3
    static constexpr int PCH = PC / 4;          // 16-byte chunks per P row (34)
    static constexpr int RING = D + 4;          // planes u-3 .. u in use + D in flight
    static constexpr int VYR = TJ + 3;          // Vy rows j0-2 .. j0+TJ
    static constexpr int P_STAGE = PR * PC;
    static constexpr int VX_STAGE = TJ * TK;
    static constexpr int VY_STAGE = VYR * TK;
    static constexpr int VZ_STAGE = TJ * PC;    // Vz cols k0-4 .. k0+TK+3
    static constexpr int V_STAGE = VX_STAGE + VY_STAGE + VZ_STAGE;
    static constexpr int VSTAGES = D + 1;
    static constexpr int AY_N = TJ + 4;         // alpha_y rows j0-2 .. j0+TJ+1
    static constexpr int AY_PAD = (AY_N + 3) / 4 * 4;
    static constexpr int SMEM_FLOATS =
        RING * P_STAGE + VSTAGES * V_STAGE + VY_STAGE + VZ_STAGE + AY_PAD + PC;
    static constexpr size_t SMEM_BYTES = sizeof(float) * SMEM_FLOATS;
    // chunk counts of one iteration's loads and their per-thread share
    static constexpr int P_CH = PR * PCH;
    static constexpr int VX_CH = TJ * (TK / 4);
    static constexpr int VY_CH = VYR * (TK / 4);
    static constexpr int VZ_CH = TJ * PCH;
    static constexpr int P_PER = (P_CH + NT - 1) / NT;
    static constexpr int VY_PER = (VY_CH + NT - 1) / NT;
    static constexpr int VZ_PER = (VZ_CH + NT - 1) / NT;
    static_assert(VX_CH == NT, "one Vx chunk per thread");
    static_assert(VYR <= 2 * TJ, "at most two Vy rows per warp");
};

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;   // 0: the 16 bytes are zero-filled, nothing is read
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void sts4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ void stg4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float& at(float4& v, int q) { return reinterpret_cast<float*>(&v)[q]; }
__device__ __forceinline__ float at(const float4& v, int q) { return reinterpret_cast<const float*>(&v)[q]; }

// staggered gradient: 4th order in the interior of the face range, else 2nd
__device__ __forceinline__ float grad4(const Coef& cf, float pm, float p0, float p1, float p2, bool fourth)
{
    return fourth ? fadd(fmul(cf.c1, fsub(p1, p0)), fmul(cf.c2, fsub(p2, pm))) : fsub(p1, p0);
}

// V^{n+1/2} = (V^{n-1/2} - vc*grad) * damp
__device__ __forceinline__ float vupd(const Coef& cf, float vold, float grad, float damp)
{
    return fmul(fsub(vold, fmul(cf.vc, grad)), damp);
}

template <class C>
__global__ void __launch_bounds__(C::NT) k_fused_step(FusedArgs a, int seg_len, int tiles_k)
{
    extern __shared__ __align__(16) float smem[];
    float* const ring = smem;                                  // RING * P_STAGE
    float* const vst = ring + C::RING * C::P_STAGE;            // VSTAGES * V_STAGE
    float* const vyn = vst + C::VSTAGES * C::V_STAGE;          // VY_STAGE
    float* const vzn = vyn + C::VY_STAGE;                      // VZ_STAGE
    float* const ay_s = vzn + C::VZ_STAGE;                     // AY_PAD
    float* const az_s = ay_s + C::AY_PAD;                      // PC

    const Grid g = a.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, sz = g.sz;
    const long long PL = g.plane;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int tk = blockIdx.x % tiles_k, tj = blockIdx.x / tiles_k;
    const int j0 = tj * C::TJ, k0 = tk * C::TK;
    const int i_beg = blockIdx.y * seg_len;
    if (i_beg >= nx) return;
    const int i_end = min(i_beg + seg_len, nx);
    const Coef cf = a.cf;

    for (int e = tid; e < C::AY_PAD; e += C::NT) {
        const int j = j0 - 2 + e;
        ay_s[e] = (e < C::AY_N && j >= 0 && j < ny) ? __ldg(a.tb.ay + j) : 0.0f;
    }
    for (int e = tid; e < C::PC; e += C::NT) {
        const int k = k0 - 4 + e;
        az_s[e] = (k >= 0 && k < nz) ? __ldg(a.tb.az + k) : 0.0f;
    }

    // ---- per-thread load descriptors: in-plane element offset of each chunk, -1 = zero fill
    int p_off[C::P_PER], vy_off[C::VY_PER], vz_off[C::VZ_PER];
#pragma unroll
    for (int m = 0; m < C::P_PER; ++m) {
        const int e = tid + m * C::NT;
        const int r = e / C::PCH, c4 = e % C::PCH;
        const int j = j0 - 3 + r, kc = k0 - 4 + 4 * c4;
        p_off[m] = (e < C::P_CH && j >= 0 && j < ny && kc >= 0 && kc < sz) ? j * sz + kc : -1;
    }
    const int vx_off = (j0 + w < ny && k0 + 4 * lane < sz) ? (j0 + w) * sz + k0 + 4 * lane : -1;
#pragma unroll
    for (int m = 0; m < C::VY_PER; ++m) {
        const int e = tid + m * C::NT;
        const int r = e >> 5, c4 = e & 31;
        const int j = j0 - 2 + r, kc = k0 + 4 * c4;
        vy_off[m] = (e < C::VY_CH && j >= 0 && j <= ny - 2 && kc < sz) ? j * sz + kc : -1;
    }
#pragma unroll
    for (int m = 0; m < C::VZ_PER; ++m) {
        const int e = tid + m * C::NT;
        const int r = e / C::PCH, c4 = e % C::PCH;
        const int j = j0 + r, kc = k0 - 4 + 4 * c4;
        vz_off[m] = (e < C::VZ_CH && j < ny && kc >= 0 && kc < sz) ? j * sz + kc : -1;
    }

    // Loads feeding iteration u: P plane u, Vx face u-2, Vy/Vz of plane u-3.
    auto issue = [&](int u, float* pst, float* vs) {
        const bool pv = (u >= 0 && u < nx);
        const float* pb = a.p + (pv ? u : 0) * PL;
#pragma unroll
        for (int m = 0; m < C::P_PER; ++m) {
            const int e = tid + m * C::NT;
            if (e < C::P_CH) {
                const bool v = pv && p_off[m] >= 0;
                cp_async16(pst + 4 * e, v ? pb + p_off[m] : a.p, v);
            }
        }
        const int f = u - 2;
        if (u >= i_beg && f >= 0 && f <= nx - 2) {
            const bool v = vx_off >= 0;
            cp_async16(vs + 4 * tid, v ? a.vin[0] + f * PL + vx_off : a.vin[0], v);
        }
        const int io = u - 3;
        if (io >= i_beg && io < i_end) {
            const float* yb = a.vin[1] + io * PL;
            const float* zb = a.vin[2] + io * PL;
#pragma unroll
            for (int m = 0; m < C::VY_PER; ++m) {
                const int e = tid + m * C::NT;
                if (e < C::VY_CH) {
                    const bool v = vy_off[m] >= 0;
                    cp_async16(vs + C::VX_STAGE + 4 * e, v ? yb + vy_off[m] : a.vin[1], v);
                }
            }
#pragma unroll
            for (int m = 0; m < C::VZ_PER; ++m) {
                const int e = tid + m * C::NT;
                if (e < C::VZ_CH) {
                    const bool v = vz_off[m] >= 0;
                    cp_async16(vs + C::VX_STAGE + C::VY_STAGE + 4 * e, v ? zb + vz_off[m] : a.vin[2], v);
                }
            }
        }
        cp_async_commit();
    };

    const int u0 = i_beg - 3, u1 = i_end + 2;
    // ring slots, rotated by pointer (slot of plane u-3 .. u, then the D in flight)
    float* pslot[C::RING];
#pragma unroll
    for (int q = 0; q < C::RING; ++q) pslot[q] = ring + q * C::P_STAGE;
    float* vslot[C::VSTAGES];
#pragma unroll
    for (int q = 0; q < C::VSTAGES; ++q) vslot[q] = vst + q * C::V_STAGE;
    // At iteration u: pslot[0..3] hold planes u-3 .. u, pslot[4 .. 3+D-1] planes
    // u+1 .. u+D-1 in flight, pslot[3+D] is free; vslot[0] holds iteration u's V
    // data, vslot[1 .. D-1] the next iterations' in flight, vslot[D] is free.
#pragma unroll
    for (int q = 0; q < C::D; ++q) issue(u0 + q, pslot[3 + q], vslot[q]);
    __syncthreads();   // alpha tables

    // ---- per-thread constants of the own row and columns
    const int jr = j0 + w;
    const int kb = k0 + 4 * lane;                 // first own k
    const bool row_ok = jr < ny;
    const bool st_ok = row_ok && kb < sz;         // float4 store stays inside the row
    float4 myz, mpz, dxi, dzi;
    {
        const float pyj = row_ok ? __ldg(a.tb.py + jr) : 1.0f;
        const float ayj = ay_s[w + 2];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = kb + q;
            const float azk = az_s[4 * lane + 4 + q];
            at(myz, q) = fmaxf(ayj, azk);
            at(mpz, q) = fminf(pyj, k < nz ? __ldg(a.tb.pz + k) : 1.0f);
            at(dxi, q) = face_damp(at(myz, q), at(myz, q), cf.dt);
            at(dzi, q) = face_damp(fmaxf(ayj, azk), fmaxf(ayj, az_s[4 * lane + 5 + q]), cf.dt);
        }
    }
    // Vy items of this thread: row w (all warps) and row TJ+w (warps 0..2)
    constexpr int NY_IT = 2;
    float4 dyi[NY_IT];
#pragma unroll
    for (int m = 0; m < NY_IT; ++m) {
        const int r = m == 0 ? w : C::TJ + w;
        if (r < C::VYR) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float azk = az_s[4 * lane + 4 + q];
                at(dyi[m], q) = face_damp(fmaxf(ay_s[r], azk), fmaxf(ay_s[r + 1], azk), cf.dt);
            }
        }
    }
    float4 qx0 = make_float4(0.f, 0.f, 0.f, 0.f), qx1 = qx0, qx2 = qx0, qx3 = qx0;

    for (int u = u0; u <= u1; ++u) {
        cp_async_wait<C::D - 1>();
        __syncthreads();
        const float* vs = vslot[0];

        // ---- new Vx on face f = u-2 of the own columns (planes f-1 .. f+2) ----
        if (u >= i_beg) {
            const int f = u - 2;
            float4 vnew = make_float4(0.f, 0.f, 0.f, 0.f);
            if (f >= 0 && f <= nx - 2 && row_ok) {
                const bool fourth = (f > 0 && f < nx - 2);
                const float axf = __ldg(a.tb.ax + f), axf1 = __ldg(a.tb.ax + f + 1);
                const bool xint = (axf == 0.0f && axf1 == 0.0f);
                const int co = (w + 3) * C::PC + 4 * lane + 4;
                const float4 pm = lds4(pslot[0] + co), p0 = lds4(pslot[1] + co);
                const float4 p1 = lds4(pslot[2] + co), p2 = lds4(pslot[3] + co);
                const float4 vo = lds4(vs + 4 * tid);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float gr = grad4(cf, at(pm, q), at(p0, q), at(p1, q), at(p2, q), fourth);
                    const float dmp = xint ? at(dxi, q)
                        : face_damp(fmaxf(axf, at(myz, q)), fmaxf(axf1, at(myz, q)), cf.dt);
                    at(vnew, q) = (kb + q < nz) ? vupd(cf, at(vo, q), gr, dmp) : 0.0f;
                }
                if (f >= i_beg && f < i_end && st_ok) stg4(a.vout[0] + f * PL + (long long)jr * sz + kb, vnew);
            }
            qx0 = qx1; qx1 = qx2; qx2 = qx3; qx3 = vnew;
        }

        // ---- plane i = u-3: new Vy / Vz (with halos), then P^{n+1} ----
        const int i = u - 3;
        if (i >= i_beg) {
            const float axi = __ldg(a.tb.ax + i);
            const bool xint = (axi == 0.0f);
            const float* pst = pslot[0];
            const float* vys = vs + C::VX_STAGE;
            const float* vzs = vys + C::VY_STAGE;
            const long long ib = i * PL;

            // Vy rows: row w, and row TJ+w for the first three warps
#pragma unroll
            for (int m = 0; m < NY_IT; ++m) {
                const int r = m == 0 ? w : C::TJ + w;
                if (r < C::VYR) {
                    const int jf = j0 - 2 + r;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (jf >= 0 && jf <= ny - 2) {
                        const bool fourth = (jf > 0 && jf < ny - 2);
                        const float* pc = pst + 4 * lane + 4;
                        const float4 pm = lds4(pc + r * C::PC), p0 = lds4(pc + (r + 1) * C::PC);
                        const float4 p1 = lds4(pc + (r + 2) * C::PC), p2 = lds4(pc + (r + 3) * C::PC);
                        const float4 vo = lds4(vys + r * C::TK + 4 * lane);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float gr = grad4(cf, at(pm, q), at(p0, q), at(p1, q), at(p2, q), fourth);
                            float dmp;
                            if (xint) {
                                dmp = at(dyi[m], q);
                            } else {
                                const float azk = az_s[4 * lane + 4 + q];
                                dmp = face_damp(fmaxf(fmaxf(axi, ay_s[r]), azk),
                                                fmaxf(fmaxf(axi, ay_s[r + 1]), azk), cf.dt);
                            }
                            at(v, q) = (kb + q < nz) ? vupd(cf, at(vo, q), gr, dmp) : 0.0f;
                        }
                        if (r >= 2 && r < C::TJ + 2 && kb < sz)
                            stg4(a.vout[1] + ib + (long long)jf * sz + kb, v);
                    }
                    sts4(vyn + r * C::TK + 4 * lane, v);
                }
            }

            // Vz: own faces kb .. kb+3 of row jr, plus halo faces k0-2, k0-1 (lane 0)
            // and k0+TK (lane 31)
            {
                const float* prow = pst + (w + 3) * C::PC;
                const float* vzr = vzs + w * C::PC;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (row_ok) {
                    const int c = 4 * lane + 4;            // col of kb
                    const float4 pa = lds4(prow + c), pb = lds4(prow + c + 4);
                    const float pl = prow[c - 1];
                    const float4 vo = lds4(vzr + c);
                    const float pv[7] = {pl, pa.x, pa.y, pa.z, pa.w, pb.x, pb.y};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int kf = kb + q;
                        if (kf <= nz - 2) {
                            const bool fourth = (kf > 0 && kf < nz - 2);
                            const float gr = grad4(cf, pv[q], pv[q + 1], pv[q + 2], pv[q + 3], fourth);
                            float dmp;
                            if (xint) {
                                dmp = at(dzi, q);
                            } else {
                                const float ay = ay_s[w + 2];
                                dmp = face_damp(fmaxf(fmaxf(axi, ay), az_s[c + q]),
                                                fmaxf(fmaxf(axi, ay), az_s[c + q + 1]), cf.dt);
                            }
                            at(v, q) = vupd(cf, at(vo, q), gr, dmp);
                        }
                    }
                    if (st_ok) stg4(a.vout[2] + ib + (long long)jr * sz + kb, v);
                    // halo faces: lane 0 -> cols 2, 3; lane 31 -> col TK+4
                    if (lane == 0 || lane == 31) {
                        const float ay = ay_s[w + 2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int ch = lane == 0 ? 2 + h : C::TK + 4;
                            if (lane == 31 && h == 1) break;
                            const int kf = k0 - 4 + ch;
                            float vh = 0.0f;
                            if (kf >= 0 && kf <= nz - 2) {
                                const bool fourth = (kf > 0 && kf < nz - 2);
                                const float gr = grad4(cf, prow[ch - 1], prow[ch], prow[ch + 1], prow[ch + 2], fourth);
                                const float dmp = face_damp(fmaxf(fmaxf(axi, ay), az_s[ch]),
                                                            fmaxf(fmaxf(axi, ay), az_s[ch + 1]), cf.dt);
                                vh = vupd(cf, vzr[ch], gr, dmp);
                            }
                            vzn[w * C::PC + ch] = vh;
                        }
                    }
                }
                sts4(vzn + w * C::PC + 4 * lane + 4, v);
            }
            __syncthreads();

            // P^{n+1} of the own cells
            if (row_ok) {
                const float* yr = vyn + 4 * lane;
                const float4 ymm = lds4(yr + w * C::TK), ym = lds4(yr + (w + 1) * C::TK);
                const float4 yp = lds4(yr + (w + 2) * C::TK), ypp = lds4(yr + (w + 3) * C::TK);
                const float* zr = vzn + w * C::PC + 4 * lane;
                const float4 za = lds4(zr), zb = lds4(zr + 4), zc = lds4(zr + 8);
                const float zv[9] = {za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z};
                const float4 pc = lds4(pst + (w + 3) * C::PC + 4 * lane + 4);
                const float pxi = xint ? 1.0f : __ldg(a.tb.px + i);
                float4 out;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    // zv[q + 2] = face k, +1 = k-1, +3 = k+1, +0 = k-2
                    const float d1 = fadd(fadd(fsub(at(qx2, q), at(qx1, q)), fsub(at(yp, q), at(ym, q))),
                                          fsub(zv[q + 2], zv[q + 1]));
                    const float d2 = fadd(fadd(fsub(at(qx3, q), at(qx0, q)), fsub(at(ypp, q), at(ymm, q))),
                                          fsub(zv[q + 3], zv[q]));
                    const float dv = fadd(fmul(cf.c1, d1), fmul(cf.c2, d2));
                    const float pd = xint ? at(mpz, q) : fminf(pxi, at(mpz, q));
                    at(out, q) = (kb + q < nz) ? fmul(fsub(at(pc, q), fmul(cf.bulk, dv)), pd) : 0.0f;
                }
                if (kb < sz) stg4(a.pn + ib + (long long)jr * sz + kb, out);
            }
        }

        // rotate: after it pslot[q] holds plane u+1-3+q and vslot[q] iteration u+1+q.
        // The slots receiving iteration u+D's loads (pslot[3+D-1], vslot[D-1]) were
        // freed one iteration ago: their last reads (plane u-4, iteration u-1)
        // happened before this iteration's first barrier.
        float* pfree = pslot[0];
#pragma unroll
        for (int q = 0; q + 1 < C::RING; ++q) pslot[q] = pslot[q + 1];
        pslot[C::RING - 1] = pfree;
        float* vfree = vslot[0];
#pragma unroll
        for (int q = 0; q + 1 < C::VSTAGES; ++q) vslot[q] = vslot[q + 1];
        vslot[C::VSTAGES - 1] = vfree;
        if (u + C::D <= u1) issue(u + C::D, pslot[3 + C::D - 1], vslot[C::D - 1]);
        else cp_async_commit();
    }
    cp_async_wait<0>();
}

using FusedCfg = Cfg<8, 2>;

constexpr int kMaxDevices = 64;
int g_slots_per_sm[kMaxDevices];
int g_sms[kMaxDevices];
bool g_configured[kMaxDevices];

}  // namespace

bool fused_supported(const Grid& g)
{
    return g.nx >= 1 && g.ny >= 1 && g.nz >= 1 && (g.sz % 8) == 0;
}

int fused_kernel_launches_per_step() { return 1; }

cudaError_t launch_fused_step(const FusedArgs& a, cudaStream_t s)
{
    using C = FusedCfg;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_configured[dev]) {
        e = cudaFuncSetAttribute(k_fused_step<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        int slots = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&slots, k_fused_step<C>, C::NT, C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        g_slots_per_sm[dev] = slots > 0 ? slots : 1;
        g_configured[dev] = true;
    }
    const Grid& g = a.g;
    const int tiles_j = (g.ny + C::TJ - 1) / C::TJ;
    const int tiles_k = (g.nz + C::TK - 1) / C::TK;
    const long long tiles = (long long)tiles_j * tiles_k;
    // segments along i: as many as one wave of resident CTAs holds (every CTA
    // marches the same number of planes, so a single full wave has no tail)
    const long long slots = (long long)g_slots_per_sm[dev] * g_sms[dev];
    long long segs = slots / tiles;
    if (segs < 1) segs = 1;
    if (segs > g.nx) segs = g.nx;
    const int seg_len = (int)((g.nx + segs - 1) / segs);
    segs = (g.nx + seg_len - 1) / seg_len;
    dim3 grid((unsigned)tiles, (unsigned)segs, 1);
    k_fused_step<C><<<grid, C::NT, C::SMEM_BYTES, s>>>(a, seg_len, tiles_k);
    return cudaGetLastError();
}

}  // namespace fdtd
