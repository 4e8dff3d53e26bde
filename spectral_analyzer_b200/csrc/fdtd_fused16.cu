/*
 * fdtd_fused16.cu — single-pass step of the storage-precision study for the
 * 16-bit storage modes: BF16, FP16 (scaled), and their compensated forms
 * (value + 16-bit residual).
 *
 * The march is the FP32 step kernel's (fdtd_fused.cu): a CTA owns an 8 x 128
 * (j, k) tile, marches along i over a segment of planes, and one thread issues
 * the TMA boxes of each plane (P with a 3-row / 8-column halo, Vx, Vy with its
 * halo rows, Vz with its halo columns) into a shared-memory ring D planes
 * ahead, completed by mbarriers with bounded waits.  The boxes carry the
 * stored 16-bit values (two boxes per field when compensated); threads decode
 * them to float where they use them, compute in float, and encode once per
 * store.  The boxes start in k at k0-8 or k0: multiples of 8 two-byte
 * elements, 16 bytes.
 *
 * Exactness: the two-pass kernels of fdtd_precision.cu decode every stored
 * value they read and encode every value they write; the pressure pass reads
 * the velocities as stored.  This kernel does the same: each new velocity is
 * encoded, and the pressure update (and a neighbouring tile's recomputation of
 * a halo face) uses its decoded value, so both schedules produce the same
 * stored bits.  The source deposit is applied to the CTAs' shared-memory copies
 * of the source cell (decode, add, encode), the value the two-pass step
 * deposits into P^n before its velocity pass.  The receivers of the previous
 * step are recorded from this step's input P (8 taps, summed in double).
 *
 * Arithmetic: the reference's velocity and pressure updates
 * (csrc/kernels/acoustic_fdtd.cpp:1099-1148, :1176-1234), every operation
 * separately rounded, as in the two-pass kernels.
 */
#include "acoustic_fdtd_b200.h"
#include "fdtd_internal.h"
#include "fdtd_prec_internal.h"
#include "fdtd_tma.h"

#include <mutex>
#include <type_traits>
#include <vector>

namespace fdtd {
namespace prec {

namespace {

template <int M, int D_>
struct H16 {
    static constexpr bool COMP = Traits<M>::comp;
    static constexpr int NB = COMP ? 2 : 1;     // stored arrays per field
    static constexpr int TJ = 8, TK = 128, NT = 256, D = D_;   // one warp per row, 4 k per lane
    static constexpr int PR = TJ + 6;           // P rows j0-3 .. j0+TJ+2
    static constexpr int PC = TK + 16;          // P / Vz cols k0-8 .. k0+TK+7 (elements)
    static constexpr int VYR = TJ + 3;          // Vy rows j0-2 .. j0+TJ
    static constexpr int ZC = TK + 8;           // float rows of the Vz exchange: k0-4 .. k0+TK+3
    static constexpr int RING = D + 4, VSTAGES = D + 1;
    static constexpr int r128(int b) { return (b + 127) / 128 * 128; }
    // one box of one array, bytes
    static constexpr int P_B = 2 * PR * PC, VX_B = 2 * TJ * TK, VY_B = 2 * VYR * TK, VZ_B = 2 * TJ * PC;
    // stage layouts, byte offsets; the residual box of a field follows its value box
    static constexpr int P_LO = r128(P_B);
    static constexpr int P_STAGE = NB * r128(P_B);
    static constexpr int VX_OFF = 0, VX_LO = r128(VX_B);
    static constexpr int VY_OFF = NB * r128(VX_B), VY_LO = r128(VY_B);
    static constexpr int VZ_OFF = VY_OFF + NB * r128(VY_B), VZ_LO = r128(VZ_B);
    static constexpr int V_STAGE = VZ_OFF + NB * r128(VZ_B);
    // shared-memory map, bytes from a 128-byte aligned base
    static constexpr int RING0 = 0;
    static constexpr int VST0 = RING0 + RING * P_STAGE;
    static constexpr int VYN0 = VST0 + VSTAGES * V_STAGE;          // float [VYR][TK]
    static constexpr int VZN0 = VYN0 + r128(4 * VYR * TK);          // float [TJ][ZC]
    static constexpr int AY0 = VZN0 + r128(4 * TJ * ZC);            // float [TJ+4]
    static constexpr int AZ0 = AY0 + r128(4 * (TJ + 4));            // float [ZC]
    static constexpr int BAR0 = AZ0 + r128(4 * ZC);
    static constexpr size_t SMEM_BYTES = BAR0 + 8 * (RING + VSTAGES) + 128;
    static constexpr unsigned P_BYTES = NB * P_B, VX_BYTES = NB * VX_B, VYZ_BYTES = NB * (VY_B + VZ_B);
    static_assert((PC * 2) % 16 == 0 && (TK * 2) % 16 == 0, "TMA box rows are 16-byte multiples");
    static_assert(PC <= 256 && PR <= 256, "TMA box extent");
};

// Prefetch distance (planes): 3 for the plain 16-bit forms (same box:
// BF16 146.2 -> 146.8, FP16 136.6 -> 138.5 Gcell/s against 2); 2 for the
// compensated forms, whose boxes at 3 leave one CTA per SM (half the rate).
template <int M>
__host__ __device__ constexpr int depth16() { return Traits<M>::comp ? 2 : 3; }

// Exact decode / encode of the stored forms (as ld4 / st4 of the two-pass
// kernels); the residual arguments are ignored by the plain 16-bit forms.
template <int M>
struct Code {
    using S = typename Traits<M>::S;
    static constexpr bool C = Traits<M>::comp;
    // the BF16 forms are stored unscaled (scale and residual scale 1), and a
    // product with 1.0f is the operand itself, so those multiplies are left out
    static constexpr bool U = (M == kBF16 || M == kBF16C);
    union U4 { uint2 u; S s[4]; };

    __device__ static float dec(S h, S l, const Sc& c)
    {
        float x = tofl(h);
        if constexpr (C) x = __fadd_rn(x, U ? tofl(l) : __fmul_rn(tofl(l), c.ils));
        return U ? x : __fmul_rn(x, c.is);
    }
    // four values at element e of a box whose residual box is lo_off bytes on
    __device__ static float4 ld4(const unsigned char* box, int e, int lo_off, const Sc& c)
    {
        U4 h, l;
        h.u = *reinterpret_cast<const uint2*>(box + 2 * e);
        if constexpr (C) l.u = *reinterpret_cast<const uint2*>(box + lo_off + 2 * e);
        else l.u = h.u;
        return make_float4(dec(h.s[0], l.s[0], c), dec(h.s[1], l.s[1], c), dec(h.s[2], l.s[2], c),
                           dec(h.s[3], l.s[3], c));
    }
    __device__ static float ld1(const unsigned char* box, int e, int lo_off, const Sc& c)
    {
        const S h = *reinterpret_cast<const S*>(box + 2 * e);
        if constexpr (C) return dec(h, *reinterpret_cast<const S*>(box + lo_off + 2 * e), c);
        else return dec(h, h, c);
    }
    __device__ static void enc(float v, const Sc& c, S& h, S& l)
    {
        const float xs = U ? v : __fmul_rn(v, c.s);
        h = fromfl<S>(xs);
        if constexpr (C) {
            const float r = __fsub_rn(xs, tofl(h));
            l = fromfl<S>(U ? r : __fmul_rn(r, c.ls));
        } else {
            l = h;
        }
    }
    // encode four values, store them at padded index i (when st), return them decoded
    __device__ static float4 st4(float4 v, const Sc& c, void* hi, void* lo, long long i, bool st)
    {
        U4 h, l;
        float* pv = reinterpret_cast<float*>(&v);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            enc(pv[q], c, h.s[q], l.s[q]);
            pv[q] = dec(h.s[q], l.s[q], c);
        }
        if (st) {
            *reinterpret_cast<uint2*>(static_cast<S*>(hi) + i) = h.u;
            if constexpr (C) *reinterpret_cast<uint2*>(static_cast<S*>(lo) + i) = l.u;
        }
        return v;
    }
    __device__ static float round_trip(float v, const Sc& c)
    {
        S h, l;
        enc(v, c, h, l);
        return dec(h, l, c);
    }
    // the value at padded index i of a stored field in global memory
    __device__ static float ldg(const void* hi, const void* lo, long long i, const Sc& c)
    {
        const S h = static_cast<const S*>(hi)[i];
        if constexpr (C) return dec(h, static_cast<const S*>(lo)[i], c);
        else return dec(h, h, c);
    }
    // the source deposit on a shared-memory copy: x <- x + amp, re-encoded
    __device__ static void add1(unsigned char* box, int e, int lo_off, float amp, const Sc& c)
    {
        S* h = reinterpret_cast<S*>(box + 2 * e);
        const float x = __fadd_rn(ld1(box, e, lo_off, c), amp);
        S hh, ll;
        enc(x, c, hh, ll);
        *h = hh;
        if constexpr (C) *reinterpret_cast<S*>(box + lo_off + 2 * e) = ll;
    }
};

__device__ __forceinline__ float& at4(float4& v, int q) { return reinterpret_cast<float*>(&v)[q]; }

__device__ __forceinline__ float grad(const PCoef<float>& cf, float pm, float p0, float p1, float p2, bool fourth)
{
    return fourth ? __fadd_rn(__fmul_rn(cf.c1, __fsub_rn(p1, p0)), __fmul_rn(cf.c2, __fsub_rn(p2, pm)))
                  : __fsub_rn(p1, p0);
}

__device__ __forceinline__ float vup(const PCoef<float>& cf, float vo, float gr, float dmp)
{
    return __fmul_rn(__fsub_rn(vo, __fmul_rn(cf.vc, gr)), dmp);
}

__device__ __forceinline__ float damp(float aL, float aR, float dt)
{
    return __fsub_rn(1.0f, __fmul_rn(__fmul_rn(0.5f, __fadd_rn(aL, aR)), dt));
}

// four faces; bit q of m4: 4th-order gradient, bit q of ok: the face exists
__device__ __forceinline__ float4 vel4m(const PCoef<float>& cf, float4 pm, float4 p0, float4 p1, float4 p2,
                                        float4 vo, float4 dmp, int m4, int ok)
{
    float4 r;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float gr = grad(cf, at4(pm, q), at4(p0, q), at4(p1, q), at4(p2, q), (m4 >> q) & 1);
        at4(r, q) = ((ok >> q) & 1) ? vup(cf, at4(vo, q), gr, at4(dmp, q)) : 0.0f;
    }
    return r;
}

__device__ __forceinline__ float pup(const PCoef<float>& cf, float p, float xp, float xm, float xpp, float xmm,
                                     float yp, float ym, float ypp, float ymm, float zp, float zm, float zpp,
                                     float zmm, float pd)
{
    const float d1 = __fadd_rn(__fadd_rn(__fsub_rn(xp, xm), __fsub_rn(yp, ym)), __fsub_rn(zp, zm));
    const float d2 = __fadd_rn(__fadd_rn(__fsub_rn(xpp, xmm), __fsub_rn(ypp, ymm)), __fsub_rn(zpp, zmm));
    const float dv = __fadd_rn(__fmul_rn(cf.c1, d1), __fmul_rn(cf.c2, d2));
    return __fmul_rn(__fsub_rn(p, __fmul_rn(cf.bulk, dv)), pd);
}

struct Maps16 {
    CUtensorMap m[8];   // P, Vx, Vy, Vz: value map, then residual map
};

template <int M>
__global__ void __launch_bounds__(256) k_fused16(F16Args a, const __grid_constant__ Maps16 mp, int seg_len,
                                                  int tiles_k)
{
    using C = H16<M, depth16<M>()>;
    using K = Code<M>;
    const Grid g = a.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, sz = g.sz;
    const long long PL = g.plane;
    const PCoef<float> cf = a.cf;
    const int tid = threadIdx.x;

    if (a.rec_out) {   // the previous step's receivers, from this step's input P
        const int nblk = gridDim.x * gridDim.y, b = blockIdx.x + gridDim.x * blockIdx.y;
        for (int r = b + nblk * tid; r < a.n_rec; r += nblk * C::NT) {
            double s = 0.0;
            for (int t = 0; t < 8; ++t)
                s = __dadd_rn(s, __dmul_rn(a.rec_w[8 * r + t],
                                           (double)K::ldg(a.p_hi, a.p_lo, a.rec_idx[8 * r + t], a.sp)));
            a.rec_out[r] = s;
        }
    }
    const int i_beg = blockIdx.y * seg_len;
    if (i_beg >= nx) return;
    const int i_end = min(i_beg + seg_len, nx);

    extern __shared__ unsigned char smem_raw16[];
    unsigned char* const sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw16) + 127) & ~uintptr_t(127));
    const unsigned sbase = smem_u32(sm);
    const unsigned bar0 = sbase + C::BAR0;
    float* const vyn = reinterpret_cast<float*>(sm + C::VYN0);
    float* const vzn = reinterpret_cast<float*>(sm + C::VZN0);
    float* const ay_s = reinterpret_cast<float*>(sm + C::AY0);
    float* const az_s = reinterpret_cast<float*>(sm + C::AZ0);

    const int lane = tid % 32, w = tid / 32;
    const int tile = blockIdx.x, tk = tile % tiles_k, tj = tile / tiles_k;
    const int j0 = tj * C::TJ, k0 = tk * C::TK;

    if (tid == 0) {
        for (int q = 0; q < C::RING + C::VSTAGES; ++q) mbar_init(bar0 + 8u * q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    for (int e = tid; e < C::TJ + 4; e += C::NT) {
        const int j = j0 - 2 + e;
        ay_s[e] = (j >= 0 && j < ny) ? __ldg(cf.ay + j) : 0.0f;
    }
    for (int e = tid; e < C::ZC; e += C::NT) {
        const int k = k0 - 4 + e;
        az_s[e] = (k >= 0 && k < nz) ? __ldg(cf.az + k) : 0.0f;
    }
    __syncthreads();

    int pslot[C::RING], vslot[C::VSTAGES];
#pragma unroll
    for (int q = 0; q < C::RING; ++q) pslot[q] = q;
#pragma unroll
    for (int q = 0; q < C::VSTAGES; ++q) vslot[q] = q;
    unsigned pph = 0, vph = 0;

    // loads feeding iteration u: P plane u, Vx face u-2, Vy / Vz of plane u-3
    auto issue = [&](int u, int ps, int vsg) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        const unsigned pb = bar0 + 8u * ps;
        mbar_expect_tx(pb, C::P_BYTES);
        const unsigned pdst = sbase + C::RING0 + ps * C::P_STAGE;
        tma_load3(pdst, &mp.m[0], k0 - 8, j0 - 3, u, pb);
        if constexpr (C::COMP) tma_load3(pdst + C::P_LO, &mp.m[1], k0 - 8, j0 - 3, u, pb);
        const int f = u - 2, io = u - 3;
        const bool vx = (u >= i_beg && f >= 0 && f <= nx - 2);
        const bool vyz = (io >= i_beg && io < i_end);
        const unsigned vb = bar0 + 8u * (C::RING + vsg);
        const unsigned vdst = sbase + C::VST0 + vsg * C::V_STAGE;
        mbar_expect_tx(vb, (vx ? C::VX_BYTES : 0u) + (vyz ? C::VYZ_BYTES : 0u));
        if (vx) {
            tma_load3(vdst + C::VX_OFF, &mp.m[2], k0, j0, f, vb);
            if constexpr (C::COMP) tma_load3(vdst + C::VX_OFF + C::VX_LO, &mp.m[3], k0, j0, f, vb);
        }
        if (vyz) {
            tma_load3(vdst + C::VY_OFF, &mp.m[4], k0, j0 - 2, io, vb);
            tma_load3(vdst + C::VZ_OFF, &mp.m[6], k0 - 8, j0, io, vb);
            if constexpr (C::COMP) {
                tma_load3(vdst + C::VY_OFF + C::VY_LO, &mp.m[5], k0, j0 - 2, io, vb);
                tma_load3(vdst + C::VZ_OFF + C::VZ_LO, &mp.m[7], k0 - 8, j0, io, vb);
            }
        }
    };

    const int u0 = i_beg - 3, u1 = i_end + 2;
    if (tid == 0)
        for (int q = 0; q < C::D; ++q) issue(u0 + q, pslot[3 + q], vslot[q]);

    // per-thread constants of the own row and columns
    const int jr = j0 + w;
    const int kb = k0 + 4 * lane;
    const bool row_ok = jr < ny;
    const bool kfull = k0 + C::TK <= nz;
    const bool st_ok = row_ok && kb < sz;
    const long long own = row_ok ? (long long)jr * sz + kb : 0;
    const int cP = (w + 3) * C::PC + 4 * lane + 8;    // own cells in a P box (elements)
    int zm4 = 0, zok = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int kf = kb + q;
        zm4 |= (kf > 0 && kf < nz - 2) ? (1 << q) : 0;
        zok |= (kf <= nz - 2) ? (1 << q) : 0;
    }
    int okk = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) okk |= (kb + q < nz) ? (1 << q) : 0;
    float4 myz, mpz, dxi, dzi;
    {
        const float pyj = row_ok ? __ldg(cf.py + jr) : 1.0f;
        const float ayj = ay_s[w + 2];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = kb + q;
            const float azk = az_s[4 * lane + 4 + q];
            at4(myz, q) = fmaxf(ayj, azk);
            at4(mpz, q) = fminf(pyj, k < nz ? __ldg(cf.pz + k) : 1.0f);
            at4(dxi, q) = damp(at4(myz, q), at4(myz, q), cf.dt);
            at4(dzi, q) = damp(fmaxf(ayj, azk), fmaxf(ayj, az_s[4 * lane + 5 + q]), cf.dt);
        }
    }
    float4 dyi[2];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int r = m == 0 ? w : C::TJ + w;
        dyi[m] = make_float4(1.f, 1.f, 1.f, 1.f);
        if (r < C::VYR) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float azk = az_s[4 * lane + 4 + q];
                at4(dyi[m], q) = damp(fmaxf(ay_s[r], azk), fmaxf(ay_s[r + 1], azk), cf.dt);
            }
        }
    }
    // own-column P of planes u-3 .. u (decoded) and new Vx of faces u-5 .. u-2
    float4 pq0 = make_float4(0.f, 0.f, 0.f, 0.f), pq1 = pq0, pq2 = pq0, pq3 = pq0;
    float4 qx0 = pq0, qx1 = pq0, qx2 = pq0, qx3 = pq0;
    auto ax_at = [&](int q) { return (q >= 0 && q < nx) ? __ldg(cf.ax + q) : 0.0f; };
    auto px_at = [&](int q) { return (q >= 0 && q < nx) ? __ldg(cf.px + q) : 1.0f; };
    float axw3 = ax_at(u0 - 3), axw2 = ax_at(u0 - 2), axw1 = ax_at(u0 - 1), axw0 = ax_at(u0);
    float pxw = px_at(u0 - 3);
    int u_fail = u1 + 1;

    // The x-interior iterations of a tile whose columns are all cells run a
    // separately compiled body without the general path: iteration u is
    // interior when plane u-3 and faces u-2 .. u-1 have alpha_x = 0 (px = 1),
    // face u-2 has the 4th-order gradient and plane u-3 is an own plane.  Both
    // bodies evaluate the same expressions there.
    int fast_lo = u1 + 1, fast_hi = u1 + 1;
    if (kfull && a.xi_hi > a.xi_lo) {
        fast_lo = max(max(a.xi_lo + 3, 3), i_beg + 3);
        fast_hi = min(min(a.xi_hi + 1, nx), u1 + 1);
        if (fast_lo >= fast_hi) fast_lo = fast_hi = u1 + 1;
    }

    auto iteration = [&](const int u, auto fast_tag) -> bool {
        constexpr bool FAST = decltype(fast_tag)::value;
        const int ps = pslot[3], vsg = vslot[0];
        const bool ok = mbar_wait(bar0 + 8u * ps, (pph >> ps) & 1u, a.wait_us) &&
                        mbar_wait(bar0 + 8u * (C::RING + vsg), (vph >> vsg) & 1u, a.wait_us);
        unsigned char* const pbox = sm + C::RING0 + ps * C::P_STAGE;
        if (a.dep_amp != 0.0f && u == a.dep_i && tid == 0 && ok) {
            const int dj = a.dep_j - (j0 - 3), dk = a.dep_k - (k0 - 8);
            if (dj >= 0 && dj < C::PR && dk >= 0 && dk < C::PC)
                K::add1(pbox, dj * C::PC + dk, C::P_LO, a.dep_amp, a.sp);
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicMin(a.status + kStatusTimeout, blockIdx.x + gridDim.x * blockIdx.y);
            u_fail = u;
            return false;
        }
        pph ^= 1u << ps;
        vph ^= 1u << vsg;
        if (tid == 0 && u + C::D <= u1) issue(u + C::D, pslot[C::RING - 1], vslot[C::VSTAGES - 1]);
        float ax_next = 0.0f, px_next = 1.0f;
        if constexpr (!FAST) {
            ax_next = ax_at(u + 1);
            px_next = px_at(u - 2);
        }
        const unsigned char* const vs = sm + C::VST0 + vsg * C::V_STAGE;

        pq0 = pq1; pq1 = pq2; pq2 = pq3;
        pq3 = K::ld4(pbox, cP, C::P_LO, a.sp);

        // ---- new Vx on face f = u-2 (planes u-3 .. u) ----
        if (FAST || u >= i_beg) {
            const int f = u - 2;
            float4 vnew = make_float4(0.f, 0.f, 0.f, 0.f);
            if (FAST ? row_ok : (f >= 0 && f <= nx - 2 && row_ok)) {
                const float4 vo = K::ld4(vs + C::VX_OFF, w * C::TK + 4 * lane, C::VX_LO, a.sv);
                float4 v;
                if constexpr (FAST) {
                    v = vel4m(cf, pq0, pq1, pq2, pq3, vo, dxi, 15, 15);
                } else {
                    const bool fourth = (f > 0 && f < nx - 2);
                    const float axf = axw2, axf1 = axw1;
                    if (fourth && axf == 0.0f && axf1 == 0.0f && kfull) {
                        v = vel4m(cf, pq0, pq1, pq2, pq3, vo, dxi, 15, 15);
                    } else {
                        float4 dm;
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            at4(dm, q) = damp(fmaxf(axf, at4(myz, q)), fmaxf(axf1, at4(myz, q)), cf.dt);
                        v = vel4m(cf, pq0, pq1, pq2, pq3, vo, dm, fourth ? 15 : 0, okk);
                    }
                }
                vnew = K::st4(v, a.sv, a.vout_hi[0], a.vout_lo[0], f * PL + own,
                              f >= i_beg && f < i_end && st_ok);
            }
            qx0 = qx1; qx1 = qx2; qx2 = qx3; qx3 = vnew;
        }

        // ---- plane i = u-3: new Vy / Vz (with halos), then P^{n+1} ----
        const int i = u - 3;
        if (FAST || i >= i_beg) {
            const float axi = FAST ? 0.0f : axw3;
            const bool xint = FAST || (axi == 0.0f);
            const unsigned char* const pst = sm + C::RING0 + pslot[0] * C::P_STAGE;
            const unsigned char* const vys = vs + C::VY_OFF;
            const unsigned char* const vzs = vs + C::VZ_OFF;
            const long long ib = (long long)i * PL;
            const float4 pown = pq0;   // own row of plane i

#pragma unroll
            for (int m = 0; m < 2; ++m) {
                const int r = m == 0 ? w : C::TJ + w;
                if (r < C::VYR) {
                    const int jf = j0 - 2 + r;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (jf >= 0 && jf <= ny - 2) {
                        const int c = 4 * lane + 8;
                        const float4 pm = K::ld4(pst, r * C::PC + c, C::P_LO, a.sp);
                        const float4 p0 = K::ld4(pst, (r + 1) * C::PC + c, C::P_LO, a.sp);
                        const float4 p1 = K::ld4(pst, (r + 2) * C::PC + c, C::P_LO, a.sp);
                        // row r+3 of the box is the own row for the first item
                        const float4 p2 = m == 0 ? pown : K::ld4(pst, (r + 3) * C::PC + c, C::P_LO, a.sp);
                        const float4 vo = K::ld4(vys, r * C::TK + 4 * lane, C::VY_LO, a.sv);
                        const bool fourth = (jf > 0 && jf < ny - 2);
                        float4 vv;
                        if constexpr (FAST) {
                            // the row's gradient order is uniform over its threads
                            vv = vel4m(cf, pm, p0, p1, p2, vo, dyi[m], fourth ? 15 : 0, 15);
                        } else if (fourth && xint && kfull) {
                            vv = vel4m(cf, pm, p0, p1, p2, vo, dyi[m], 15, 15);
                        } else {
                            float4 dm;
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float azk = az_s[4 * lane + 4 + q];
                                at4(dm, q) = damp(fmaxf(fmaxf(axi, ay_s[r]), azk), fmaxf(fmaxf(axi, ay_s[r + 1]), azk),
                                                  cf.dt);
                            }
                            vv = vel4m(cf, pm, p0, p1, p2, vo, dm, fourth ? 15 : 0, okk);
                        }
                        v = K::st4(vv, a.sv, a.vout_hi[1], a.vout_lo[1], ib + (long long)jf * sz + kb,
                                   r >= 2 && r < C::TJ + 2 && kb < sz);
                    }
                    *reinterpret_cast<float4*>(vyn + r * C::TK + 4 * lane) = v;
                }
            }

            // Vz: own faces kb .. kb+3 of row jr
            {
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (row_ok) {
                    const int c = (w + 3) * C::PC + 4 * lane + 8;
                    const float4 pb4 = K::ld4(pst, c + 4, C::P_LO, a.sp);
                    const float pl = K::ld1(pst, c - 1, C::P_LO, a.sp);
                    const float4 vo = K::ld4(vzs, w * C::PC + 4 * lane + 8, C::VZ_LO, a.sv);
                    const float4 pm = make_float4(pl, pown.x, pown.y, pown.z);
                    const float4 p1 = make_float4(pown.y, pown.z, pown.w, pb4.x);
                    const float4 p2 = make_float4(pown.z, pown.w, pb4.x, pb4.y);
                    float4 vv;
                    if (xint) {
                        vv = vel4m(cf, pm, pown, p1, p2, vo, dzi, zm4, zok);
                    } else {
                        const float ay = ay_s[w + 2];
                        float4 dm;
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            at4(dm, q) = damp(fmaxf(fmaxf(axi, ay), az_s[4 * lane + 4 + q]),
                                              fmaxf(fmaxf(axi, ay), az_s[4 * lane + 5 + q]), cf.dt);
                        vv = vel4m(cf, pm, pown, p1, p2, vo, dm, zm4, zok);
                    }
                    v = K::st4(vv, a.sv, a.vout_hi[2], a.vout_lo[2], ib + own, st_ok);
                }
                *reinterpret_cast<float4*>(vzn + w * C::ZC + 4 * lane + 4) = v;
            }
            // halo Vz faces k0-2, k0-1, k0+TK of every row (the last warp)
            const int hl = tid - (C::NT - 32);
            if (hl >= 0 && hl < 3 * C::TJ) {
                const int jl = hl / 3, which = hl - 3 * jl;
                const int ch = which < 2 ? 2 + which : C::TK + 4;    // float col: k = k0-4+ch
                const int ce = ch + 4;                               // element col: k = k0-8+ce
                const int kf = k0 - 4 + ch;
                float vh = 0.0f;
                if (j0 + jl < ny && kf >= 0 && kf <= nz - 2) {
                    const bool fourth = (kf > 0 && kf < nz - 2);
                    const float ay = ay_s[jl + 2];
                    const int rb = (jl + 3) * C::PC;
                    const float gr = grad(cf, K::ld1(pst, rb + ce - 1, C::P_LO, a.sp), K::ld1(pst, rb + ce, C::P_LO, a.sp),
                                          K::ld1(pst, rb + ce + 1, C::P_LO, a.sp),
                                          K::ld1(pst, rb + ce + 2, C::P_LO, a.sp), fourth);
                    const float dmp = damp(fmaxf(fmaxf(axi, ay), az_s[ch]), fmaxf(fmaxf(axi, ay), az_s[ch + 1]), cf.dt);
                    vh = K::round_trip(vup(cf, K::ld1(vzs, jl * C::PC + ce, C::VZ_LO, a.sv), gr, dmp), a.sv);
                }
                vzn[jl * C::ZC + ch] = vh;
            }
            __syncthreads();

            // P^{n+1} of the own cells
            if (row_ok) {
                const float* yr = vyn + 4 * lane;
                const float4 ymm = *reinterpret_cast<const float4*>(yr + w * C::TK);
                const float4 ym = *reinterpret_cast<const float4*>(yr + (w + 1) * C::TK);
                const float4 yp = *reinterpret_cast<const float4*>(yr + (w + 2) * C::TK);
                const float4 ypp = *reinterpret_cast<const float4*>(yr + (w + 3) * C::TK);
                const float* zr = vzn + w * C::ZC + 4 * lane;
                const float2 za = *reinterpret_cast<const float2*>(zr + 2);
                const float4 zb = *reinterpret_cast<const float4*>(zr + 4);
                const float zc = zr[8];
                // px[i] = 1 on x-interior planes, so min(px[i], min(py, pz)) = mpz there
                float4 pd = mpz;
                if constexpr (!FAST) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) at4(pd, q) = fminf(pxw, at4(mpz, q));
                }
                float4 out;
                out.x = pup(cf, pown.x, qx2.x, qx1.x, qx3.x, qx0.x, yp.x, ym.x, ypp.x, ymm.x, zb.x, za.y, zb.y, za.x, pd.x);
                out.y = pup(cf, pown.y, qx2.y, qx1.y, qx3.y, qx0.y, yp.y, ym.y, ypp.y, ymm.y, zb.y, zb.x, zb.z, za.y, pd.y);
                out.z = pup(cf, pown.z, qx2.z, qx1.z, qx3.z, qx0.z, yp.z, ym.z, ypp.z, ymm.z, zb.z, zb.y, zb.w, zb.x, pd.z);
                out.w = pup(cf, pown.w, qx2.w, qx1.w, qx3.w, qx0.w, yp.w, ym.w, ypp.w, ymm.w, zb.w, zb.z, zc, zb.y, pd.w);
                if (!FAST && !kfull) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (kb + q >= nz) at4(out, q) = 0.0f;
                }
                K::st4(out, a.sp, a.pn_hi, a.pn_lo, ib + own, kb < sz);
            }
        }

        if constexpr (!FAST) {
            axw3 = axw2; axw2 = axw1; axw1 = axw0; axw0 = ax_next;
            pxw = px_next;
        }
        {
            const int pfree = pslot[0];
#pragma unroll
            for (int q = 0; q + 1 < C::RING; ++q) pslot[q] = pslot[q + 1];
            pslot[C::RING - 1] = pfree;
            const int vfree = vslot[0];
#pragma unroll
            for (int q = 0; q + 1 < C::VSTAGES; ++q) vslot[q] = vslot[q + 1];
            vslot[C::VSTAGES - 1] = vfree;
        }
        return true;
    };

    for (int u = u0; u <= u1;) {
        if (u == fast_lo) {
            bool ran = true;
            for (; u < fast_hi; ++u)
                if (!iteration(u, std::true_type{})) { ran = false; break; }
            if (!ran) break;
            // the alpha_x / px window of the general iterations that follow
            axw3 = ax_at(u - 3); axw2 = ax_at(u - 2); axw1 = ax_at(u - 1); axw0 = ax_at(u);
            pxw = px_at(u - 3);
            continue;
        }
        if (!iteration(u, std::false_type{})) break;
        ++u;
    }

    // after a timed-out wait, the copies of iterations u_fail .. u_fail+D-1 may
    // still be landing: wait for them (bounded) before shared memory is released
    if (u_fail <= u1) {
        if (tid == 0) {
            for (int q = 0; q < C::D && u_fail + q <= u1; ++q) {
                const int ps = pslot[3 + q], vsg = vslot[q];
                mbar_wait(bar0 + 8u * ps, (pph >> ps) & 1u, a.wait_us);
                mbar_wait(bar0 + 8u * (C::RING + vsg), (vph >> vsg) & 1u, a.wait_us);
            }
        }
        __syncthreads();
    }
}

constexpr int kMaxDev16 = 64;
int g_slots16[6][kMaxDev16];
int g_sms16[kMaxDev16];
std::mutex g_cfg16_mu;

template <int M>
cudaError_t launch_of(const F16Args& a, F16Cache* cache, const void* const bases[8], cudaStream_t s)
{
    using C = H16<M, depth16<M>()>;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev16) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lk(g_cfg16_mu);
        if (!g_slots16[M][dev]) {
            e = cudaFuncSetAttribute(k_fused16<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM_BYTES);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&g_sms16[dev], cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            int slots = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&slots, k_fused16<M>, C::NT, C::SMEM_BYTES);
            if (e != cudaSuccess) return e;
            g_slots16[M][dev] = slots > 0 ? slots : 1;
        }
    }
    Maps16 mp;
    const int bx[4] = {C::PC, C::TK, C::TK, C::PC};
    const int by[4] = {C::PR, C::TJ, C::VYR, C::TJ};
    for (int q = 0; q < 8; ++q) {
        if (!bases[q]) { mp.m[q] = mp.m[q & ~1]; continue; }   // no residual array: unused
        e = f16_map(cache, bases[q], a.g, bx[q / 2], by[q / 2], &mp.m[q]);
        if (e != cudaSuccess) return e;
    }
    const Grid& g = a.g;
    const int tiles_j = (g.ny + C::TJ - 1) / C::TJ;
    const int tiles_k = (g.nz + C::TK - 1) / C::TK;
    const long long tiles = (long long)tiles_j * tiles_k;
    const long long slots = (long long)g_slots16[M][dev] * g_sms16[dev];
    long long segs = slots / tiles;
    if (segs < 1) segs = 1;
    if (segs > g.nx) segs = g.nx;
    const int seg_len = (int)((g.nx + segs - 1) / segs);
    segs = (g.nx + seg_len - 1) / seg_len;
    if (tiles > 0x7fffffffLL) return cudaErrorInvalidValue;
    dim3 grid((unsigned)tiles, (unsigned)segs, 1);
    k_fused16<M><<<grid, C::NT, C::SMEM_BYTES, s>>>(a, mp, seg_len, tiles_k);
    return cudaGetLastError();
}

}  // namespace

struct F16Cache {
    struct Entry {
        const void* base;
        int bx, by;
        CUtensorMap map;
    };
    std::vector<Entry> entries;
};

F16Cache* f16_cache_create() { return new F16Cache(); }
void f16_cache_destroy(F16Cache* c) { delete c; }

cudaError_t f16_map(F16Cache* c, const void* base, const Grid& g, int bx, int by, CUtensorMap* out)
{
    for (const auto& e : c->entries)
        if (e.base == base && e.bx == bx && e.by == by) { *out = e.map; return cudaSuccess; }
    F16Cache::Entry e;
    e.base = base;
    e.bx = bx;
    e.by = by;
    cudaError_t err = encode_field_map(&e.map, base, 2, g, bx, by);
    if (err != cudaSuccess) return err;
    c->entries.push_back(e);
    *out = e.map;
    return cudaSuccess;
}

bool f16_supported(int mode, const Grid& g)
{
    return (mode == kBF16 || mode == kFP16 || mode == kBF16C || mode == kFP16C) && g.nx >= 1 && g.ny >= 1 &&
           g.nz >= 1 && g.sz % 8 == 0;
}

size_t f16_smem_bytes(int mode)
{
    switch (mode) {
        case kBF16: return H16<kBF16, depth16<kBF16>()>::SMEM_BYTES;
        case kFP16: return H16<kFP16, depth16<kFP16>()>::SMEM_BYTES;
        case kBF16C: return H16<kBF16C, depth16<kBF16C>()>::SMEM_BYTES;
        case kFP16C: return H16<kFP16C, depth16<kFP16C>()>::SMEM_BYTES;
        default: return 0;
    }
}

cudaError_t launch_fused16(int mode, const F16Args& a, F16Cache* cache, const void* const bases[8], cudaStream_t s)
{
    switch (mode) {
        case kBF16: return launch_of<kBF16>(a, cache, bases, s);
        case kFP16: return launch_of<kFP16>(a, cache, bases, s);
        case kBF16C: return launch_of<kBF16C>(a, cache, bases, s);
        case kFP16C: return launch_of<kFP16C>(a, cache, bases, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace prec
}  // namespace fdtd
