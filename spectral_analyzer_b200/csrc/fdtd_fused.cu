/*
 * fdtd_fused.cu — single-pass velocity+pressure step for open rooms.
 *
 * One launch advances V^{n-1/2} -> V^{n+1/2} and P^n -> P^{n+1} over the whole
 * grid, reading each field once and writing each once: 16 B read + 16 B
 * written per cell-update, the HBM floor of the scheme.  (The two-pass step
 * reads P and V twice: 48 B.)
 *
 * Decomposition (2.5D): a CTA owns a TJ x TK tile of (j, k) columns and
 * marches along i over a segment [i_beg, i_end).  Per plane it needs
 *   - P^n of the plane with a 3-cell halo in j and k (y/z gradients of the halo
 *     faces),
 *   - the new Vx of faces i-2 .. i+1 (x divergence) — kept per thread in a
 *     4-deep register queue, so P^n planes i-1 .. i+2 of the thread's own
 *     columns feed the x gradient,
 *   - the new Vy of rows j0-2 .. j0+TJ and Vz of columns k0-2 .. k0+TK: the
 *     faces outside the tile are recomputed here from V^{n-1/2}, not read back
 *     from a neighbour, so the step writes into the other velocity set.
 * Loads go through a ring of shared-memory stages filled with cp.async
 * (16-byte chunks, zero-filled outside the grid) D planes ahead of use.
 * Halo rows and columns are shared with neighbouring CTAs that march at the
 * same pace, so they are served mostly from L2.
 *
 * Arithmetic is the reference's (csrc/kernels/acoustic_fdtd.cpp:1099-1148 for
 * the velocity, :894-952 and :1176-1234 for the pressure) with every operation
 * separately rounded (fadd/fsub/fmul), so the result is bit-identical to the
 * two-pass kernels and to the reference.
 */
#include "fdtd_internal.h"

namespace fdtd {

namespace {

template <int TJ_, int TK_, int D_>
struct Cfg {
    static constexpr int TJ = TJ_;
    static constexpr int TK = TK_;
    static constexpr int D = D_;               // prefetch distance (planes)
    static constexpr int NT = 32 * TJ;         // one warp per tile row
    static constexpr int CPT = TK / 32;        // cells per thread per plane
    static constexpr int PR = TJ + 6;          // P stage rows:  j0-3 .. j0+TJ+2
    static constexpr int PC = TK + 8;          // P stage cols:  k0-4 .. k0+TK+3
    static constexpr int RING = D + 4;         // P planes u-3 .. u in use + D in flight
    static constexpr int VYR = TJ + 3;         // Vy rows:       j0-2 .. j0+TJ
    static constexpr int VZC = TK + 8;         // Vz cols:       k0-4 .. k0+TK+3
    static constexpr int P_STAGE = PR * PC;
    static constexpr int VX_STAGE = TJ * TK;
    static constexpr int VY_STAGE = VYR * TK;
    static constexpr int VZ_STAGE = TJ * VZC;
    static constexpr int V_STAGE = VX_STAGE + VY_STAGE + VZ_STAGE;
    static constexpr int VSTAGES = D + 1;
    static constexpr int AY_N = TJ + 4;        // alpha_y rows j0-2 .. j0+TJ+1
    static constexpr int AY_PAD = (AY_N + 3) / 4 * 4;
    static constexpr int SMEM_FLOATS =
        RING * P_STAGE + VSTAGES * V_STAGE + VY_STAGE + VZ_STAGE + AY_PAD + PC;
    static constexpr size_t SMEM_BYTES = sizeof(float) * SMEM_FLOATS;
    static_assert(TK % 32 == 0, "TK must be a multiple of the warp size");
    static_assert(PC % 4 == 0 && TK % 4 == 0, "16-byte chunks");
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

__device__ __forceinline__ int wrap(int u, int m) { int r = u % m; return r < 0 ? r + m : r; }

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
    const float* __restrict__ p = a.p;
    const float* __restrict__ vxi = a.vin[0];
    const float* __restrict__ vyi = a.vin[1];
    const float* __restrict__ vzi = a.vin[2];
    float* __restrict__ pn = a.pn;
    float* __restrict__ vxo = a.vout[0];
    float* __restrict__ vyo = a.vout[1];
    float* __restrict__ vzo = a.vout[2];
    const Coef cf = a.cf;

    for (int e = tid; e < C::AY_PAD; e += C::NT) {
        const int j = j0 - 2 + e;
        ay_s[e] = (e < C::AY_N && j >= 0 && j < ny) ? __ldg(a.tb.ay + j) : 0.0f;
    }
    for (int e = tid; e < C::PC; e += C::NT) {
        const int k = k0 - 4 + e;
        az_s[e] = (k >= 0 && k < nz) ? __ldg(a.tb.az + k) : 0.0f;
    }

    // Loads feeding iteration u: P plane u, Vx faces u-2, Vy/Vz of plane u-3.
    auto issue = [&](int u) {
        float* pst = ring + wrap(u, C::RING) * C::P_STAGE;
        const bool pv = (u >= 0 && u < nx);
        for (int e = tid; e < C::PR * (C::PC / 4); e += C::NT) {
            const int r = e / (C::PC / 4), c4 = e % (C::PC / 4);
            const int j = j0 - 3 + r, kc = k0 - 4 + 4 * c4;
            const bool v = pv && j >= 0 && j < ny && kc >= 0 && kc < sz;
            cp_async16(pst + r * C::PC + 4 * c4, v ? p + (u * PL + (long long)j * sz + kc) : p, v);
        }
        float* vs = vst + wrap(u, C::VSTAGES) * C::V_STAGE;
        const int f = u - 2;
        if (u >= i_beg && f >= 0 && f <= nx - 2) {
            for (int e = tid; e < C::TJ * (C::TK / 4); e += C::NT) {
                const int r = e / (C::TK / 4), c4 = e % (C::TK / 4);
                const int j = j0 + r, kc = k0 + 4 * c4;
                const bool v = j < ny && kc < sz;
                cp_async16(vs + r * C::TK + 4 * c4, v ? vxi + (f * PL + (long long)j * sz + kc) : vxi, v);
            }
        }
        const int io = u - 3;
        if (io >= i_beg && io < i_end) {
            float* vys = vs + C::VX_STAGE;
            for (int e = tid; e < C::VYR * (C::TK / 4); e += C::NT) {
                const int r = e / (C::TK / 4), c4 = e % (C::TK / 4);
                const int j = j0 - 2 + r, kc = k0 + 4 * c4;
                const bool v = j >= 0 && j <= ny - 2 && kc < sz;
                cp_async16(vys + r * C::TK + 4 * c4, v ? vyi + (io * PL + (long long)j * sz + kc) : vyi, v);
            }
            float* vzs = vys + C::VY_STAGE;
            for (int e = tid; e < C::TJ * (C::VZC / 4); e += C::NT) {
                const int r = e / (C::VZC / 4), c4 = e % (C::VZC / 4);
                const int j = j0 + r, kc = k0 - 4 + 4 * c4;
                const bool v = j < ny && kc >= 0 && kc < sz;
                cp_async16(vzs + r * C::VZC + 4 * c4, v ? vzi + (io * PL + (long long)j * sz + kc) : vzi, v);
            }
        }
        cp_async_commit();
    };

    const int u0 = i_beg - 3, u1 = i_end + 2;
    for (int q = 0; q < C::D; ++q) issue(u0 + q);
    __syncthreads();   // alpha tables

    // per-thread constants of the own columns (constant along the march)
    const int jr = j0 + w;
    float myz[C::CPT], mpz[C::CPT], qx[C::CPT][4];
    const float py_j = (jr < ny) ? __ldg(a.tb.py + jr) : 1.0f;
#pragma unroll
    for (int c = 0; c < C::CPT; ++c) {
        const int kl = lane + 32 * c, k = k0 + kl;
        myz[c] = fmaxf(ay_s[w + 2], az_s[kl + 4]);
        mpz[c] = fminf(py_j, (k < nz) ? __ldg(a.tb.pz + k) : 1.0f);
        qx[c][0] = qx[c][1] = qx[c][2] = qx[c][3] = 0.0f;
    }

    for (int u = u0; u <= u1; ++u) {
        cp_async_wait<C::D - 1>();
        __syncthreads();
        const float* vs = vst + wrap(u, C::VSTAGES) * C::V_STAGE;

        // ---- new Vx on faces f = u-2 of the own columns ----
        if (u >= i_beg) {
            const int f = u - 2;
            const bool fv = (f >= 0 && f <= nx - 2);
            const bool fourth = (f > 0 && f < nx - 2);
            const float axf = fv ? __ldg(a.tb.ax + f) : 0.0f;
            const float axf1 = fv ? __ldg(a.tb.ax + f + 1) : 0.0f;
            const float* pm1 = ring + wrap(u - 3, C::RING) * C::P_STAGE + (w + 3) * C::PC + 4;
            const float* p0 = ring + wrap(u - 2, C::RING) * C::P_STAGE + (w + 3) * C::PC + 4;
            const float* p1 = ring + wrap(u - 1, C::RING) * C::P_STAGE + (w + 3) * C::PC + 4;
            const float* p2 = ring + wrap(u, C::RING) * C::P_STAGE + (w + 3) * C::PC + 4;
            const bool own = fv && f >= i_beg && f < i_end;
#pragma unroll
            for (int c = 0; c < C::CPT; ++c) {
                const int kl = lane + 32 * c, k = k0 + kl;
                float vnew = 0.0f;
                if (fv && jr < ny && k < nz) {
                    const float pc = p0[kl], pr = p1[kl];
                    const float grad = fourth
                        ? fadd(fmul(cf.c1, fsub(pr, pc)), fmul(cf.c2, fsub(p2[kl], pm1[kl])))
                        : fsub(pr, pc);
                    const float damp = face_damp(fmaxf(axf, myz[c]), fmaxf(axf1, myz[c]), cf.dt);
                    vnew = fmul(fsub(vs[w * C::TK + kl], fmul(cf.vc, grad)), damp);
                    if (own) vxo[f * PL + (long long)jr * sz + k] = vnew;
                }
                qx[c][0] = qx[c][1];
                qx[c][1] = qx[c][2];
                qx[c][2] = qx[c][3];
                qx[c][3] = vnew;
            }
        }

        // ---- plane i = u-3: new Vy / Vz (with halos), then P^{n+1} ----
        const int i = u - 3;
        if (i >= i_beg) {
            const float axi = __ldg(a.tb.ax + i);
            const float* pst = ring + wrap(i, C::RING) * C::P_STAGE;
            const float* vys = vs + C::VX_STAGE;
            const float* vzs = vys + C::VY_STAGE;
            const long long ibase = i * PL;

            for (int e = tid; e < C::VY_STAGE; e += C::NT) {
                const int r = e / C::TK, c = e % C::TK;
                const int jf = j0 - 2 + r, k = k0 + c;
                float v = 0.0f;
                if (jf >= 0 && jf <= ny - 2 && k < nz) {
                    const float* pcol = pst + (c + 4);
                    const float pm = pcol[r * C::PC], p0 = pcol[(r + 1) * C::PC];
                    const float p1 = pcol[(r + 2) * C::PC], p2 = pcol[(r + 3) * C::PC];
                    const float grad = (jf > 0 && jf < ny - 2)
                        ? fadd(fmul(cf.c1, fsub(p1, p0)), fmul(cf.c2, fsub(p2, pm)))
                        : fsub(p1, p0);
                    const float azk = az_s[c + 4];
                    const float aL = fmaxf(fmaxf(axi, ay_s[r]), azk);
                    const float aR = fmaxf(fmaxf(axi, ay_s[r + 1]), azk);
                    v = fmul(fsub(vys[e], fmul(cf.vc, grad)), face_damp(aL, aR, cf.dt));
                    if (r >= 2 && r < C::TJ + 2) vyo[ibase + (long long)jf * sz + k] = v;
                }
                vyn[e] = v;
            }
            for (int e = tid; e < C::TJ * (C::TK + 3); e += C::NT) {
                const int jl = e / (C::TK + 3), c = 2 + e % (C::TK + 3);
                const int j = j0 + jl, kf = k0 - 4 + c;
                float v = 0.0f;
                if (j < ny && kf >= 0 && kf <= nz - 2) {
                    const float* prow = pst + (jl + 3) * C::PC;
                    const float pm = prow[c - 1], p0 = prow[c], p1 = prow[c + 1], p2 = prow[c + 2];
                    const float grad = (kf > 0 && kf < nz - 2)
                        ? fadd(fmul(cf.c1, fsub(p1, p0)), fmul(cf.c2, fsub(p2, pm)))
                        : fsub(p1, p0);
                    const float ay = ay_s[jl + 2];
                    const float aL = fmaxf(fmaxf(axi, ay), az_s[c]);
                    const float aR = fmaxf(fmaxf(axi, ay), az_s[c + 1]);
                    v = fmul(fsub(vzs[jl * C::VZC + c], fmul(cf.vc, grad)), face_damp(aL, aR, cf.dt));
                    if (c >= 4 && c < C::TK + 4) vzo[ibase + (long long)j * sz + kf] = v;
                }
                vzn[jl * C::VZC + c] = v;
            }
            __syncthreads();

            const float pxi = __ldg(a.tb.px + i);
            const float* prow = pst + (w + 3) * C::PC + 4;
#pragma unroll
            for (int c = 0; c < C::CPT; ++c) {
                const int kl = lane + 32 * c, k = k0 + kl;
                if (jr < ny && k < nz) {
                    const float yp = vyn[(w + 2) * C::TK + kl], ym = vyn[(w + 1) * C::TK + kl];
                    const float ypp = vyn[(w + 3) * C::TK + kl], ymm = vyn[w * C::TK + kl];
                    const float* zr = vzn + w * C::VZC + kl;
                    const float zp = zr[4], zm = zr[3], zpp = zr[5], zmm = zr[2];
                    const float d1 = fadd(fadd(fsub(qx[c][2], qx[c][1]), fsub(yp, ym)), fsub(zp, zm));
                    const float d2 = fadd(fadd(fsub(qx[c][3], qx[c][0]), fsub(ypp, ymm)), fsub(zpp, zmm));
                    const float dv = fadd(fmul(cf.c1, d1), fmul(cf.c2, d2));
                    const float pd = fminf(pxi, mpz[c]);
                    pn[ibase + (long long)jr * sz + k] = fmul(fsub(prow[kl], fmul(cf.bulk, dv)), pd);
                }
            }
        }
        // stages u-4 (P) and u-1 (V) were last read before this iteration's barrier
        if (u + C::D <= u1) issue(u + C::D);
        else cp_async_commit();
    }
    cp_async_wait<0>();
}

using FusedCfg = Cfg<8, 64, 2>;

constexpr int kMaxDevices = 64;
int g_slots_per_sm[kMaxDevices];
int g_sms[kMaxDevices];
bool g_configured[kMaxDevices];

}  // namespace

bool fused_supported(const Grid& g)
{
    return g.nx >= 1 && g.ny >= 1 && g.nz >= 1 && (g.sz % 4) == 0;
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
