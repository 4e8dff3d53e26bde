/*
 * fdtd_fused.cu — single-pass velocity+pressure step for open rooms (and, with
 * the walled rules of the two-pass kernels, for large walled scenes).
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
 *     Vz of faces k0-2 .. k0+128: faces outside the tile are recomputed here
 *     from V^{n-1/2}, never read back from a neighbour, so the step writes the
 *     other velocity set;
 *   - finishes P^{n+1} of plane i from the 4th-order divergence.
 *
 * Loads: one thread per CTA issues four TMA boxes per plane (P with a 3-cell
 * halo in j and a 4-cell halo in k, Vx, Vy with its halo rows, Vz with its halo
 * columns) into a ring of shared-memory stages D planes ahead of use, each
 * stage completed by an mbarrier; boxes that reach outside the grid are
 * zero-filled by the TMA unit.  The box origin in k is k0-4 or k0, a multiple
 * of 4 floats (16 bytes).  Every mbarrier wait is bounded: a wait that runs
 * out sets a status word, the CTA drains its copies in flight (again bounded)
 * and returns.  Halo rows and columns are shared with neighbouring CTAs that
 * march at the same pace, so they are served mostly from L2.
 *
 * Absorption: on x-interior planes (alpha_x = 0, all but the 2*n_pml PML
 * planes) a face's damping depends on (j, k) only and is a per-thread constant
 * computed once; PML planes take a general path that computes it per face.
 * Both evaluate the same expression, so results do not depend on the path.
 *
 * Arithmetic is the reference's (csrc/kernels/acoustic_fdtd.cpp:1099-1148 for
 * the velocity, :894-952 and :1176-1234 for the pressure) with every operation
 * separately rounded (fadd/fsub/fmul): bit-identical to the two-pass kernels
 * and to the reference.
 */
#include "fdtd_internal.h"
#include "fdtd_tma.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>
#include <type_traits>
#include <vector>

namespace fdtd {

namespace {

// TJ rows x TK = 4*LW columns per CTA; LW threads per row (float4 each), so a
// warp covers 32/LW rows.
template <int TJ_, int D_, int LW_ = 32>
struct Cfg {
    static constexpr int TJ = TJ_;              // rows per CTA
    static constexpr int LW = LW_;              // threads per row
    static constexpr int RW = 32 / LW;          // rows per warp
    static constexpr int TK = 4 * LW;           // columns per CTA
    static constexpr int D = D_;                // prefetch distance (iterations)
    static constexpr int NT = 32 * (TJ / RW);
    static constexpr int HW = (3 * TJ + 31) / 32;   // warps computing the halo Vz faces
    static constexpr int PR = TJ + 6;           // P box rows j0-3 .. j0+TJ+2
    static constexpr int PC = TK + 8;           // P box cols k0-4 .. k0+TK+3
    static constexpr int RING = D + 4;          // planes u-3 .. u in use + D in flight
    static constexpr int VYR = TJ + 3;          // Vy rows j0-2 .. j0+TJ
    // box sizes in floats, and stage strides rounded to 128 bytes
    static constexpr int P_BOX = PR * PC;
    static constexpr int VX_BOX = TJ * TK;
    static constexpr int VY_BOX = VYR * TK;
    static constexpr int VZ_BOX = TJ * PC;      // Vz cols k0-4 .. k0+TK+3
    static constexpr int r32(int n) { return (n + 31) / 32 * 32; }
    static constexpr int P_STAGE = r32(P_BOX);
    static constexpr int VX_OFF = 0;
    static constexpr int VY_OFF = r32(VX_BOX);
    static constexpr int VZ_OFF = VY_OFF + r32(VY_BOX);
    static constexpr int V_STAGE = VZ_OFF + r32(VZ_BOX);
    static constexpr int VSTAGES = D + 1;
    static constexpr int AY_N = TJ + 4;         // alpha_y rows j0-2 .. j0+TJ+1
    // shared-memory map (floats from a 128-byte aligned base)
    static constexpr int RING0 = 0;
    static constexpr int VST0 = RING0 + RING * P_STAGE;
    static constexpr int VYN0 = VST0 + VSTAGES * V_STAGE;
    static constexpr int VZN0 = VYN0 + r32(VY_BOX);
    static constexpr int AY0 = VZN0 + r32(VZ_BOX);
    static constexpr int AZ0 = AY0 + r32(AY_N);
    static constexpr int BAR0 = AZ0 + r32(PC);  // RING + VSTAGES mbarriers (8 B each)
    static constexpr int SMEM_FLOATS = BAR0 + 2 * (RING + VSTAGES);
    static constexpr size_t SMEM_BYTES = sizeof(float) * SMEM_FLOATS + 128;   // + base alignment
    static constexpr unsigned P_BYTES = 4u * P_BOX;
    static constexpr unsigned VX_BYTES = 4u * VX_BOX;
    static constexpr unsigned VYZ_BYTES = 4u * (VY_BOX + VZ_BOX);
    static_assert((PC * 4) % 16 == 0 && (TK * 4) % 16 == 0, "TMA box rows are 16-byte multiples");
    static_assert(PC <= 256 && PR <= 256 && VYR <= 256, "TMA box extent");
    static_assert(VYR <= 2 * TJ, "at most two Vy rows per warp");
    static_assert(LW == 32 || LW == 16, "a row is one warp or half a warp");
    static_assert(TJ % RW == 0 && HW * 32 <= NT, "whole warps of rows; halo warps exist");
};

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void sts4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ void stg4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float& at(float4& v, int q) { return reinterpret_cast<float*>(&v)[q]; }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
// a face whose open fraction is 0 is closed
__device__ __forceinline__ float4 close4(float4 v, const float4& fr)
{
    if (fr.x == 0.0f) v.x = 0.0f;
    if (fr.y == 0.0f) v.y = 0.0f;
    if (fr.z == 0.0f) v.z = 0.0f;
    if (fr.w == 0.0f) v.w = 0.0f;
    return v;
}
__device__ __forceinline__ float4 mul4(const float4& v, const float4& fr)
{
    return make_float4(fmul(v.x, fr.x), fmul(v.y, fr.y), fmul(v.z, fr.z), fmul(v.w, fr.w));
}

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

// four faces, 4th-order gradient, given damping (the x-interior fast path)
__device__ __forceinline__ float4 vel4(const Coef& cf, const float4& pm, const float4& p0,
                                      const float4& p1, const float4& p2, const float4& vo,
                                      const float4& dmp)
{
    float4 r;
    r.x = vupd(cf, vo.x, grad4(cf, pm.x, p0.x, p1.x, p2.x, true), dmp.x);
    r.y = vupd(cf, vo.y, grad4(cf, pm.y, p0.y, p1.y, p2.y, true), dmp.y);
    r.z = vupd(cf, vo.z, grad4(cf, pm.z, p0.z, p1.z, p2.z, true), dmp.z);
    r.w = vupd(cf, vo.w, grad4(cf, pm.w, p0.w, p1.w, p2.w, true), dmp.w);
    return r;
}

// four faces, 2nd-order gradient, given damping (the faces next to a j end)
__device__ __forceinline__ float4 vel4_2nd(const Coef& cf, const float4& p0, const float4& p1,
                                          const float4& vo, const float4& dmp)
{
    float4 r;
    r.x = vupd(cf, vo.x, fsub(p1.x, p0.x), dmp.x);
    r.y = vupd(cf, vo.y, fsub(p1.y, p0.y), dmp.y);
    r.z = vupd(cf, vo.z, fsub(p1.z, p0.z), dmp.z);
    r.w = vupd(cf, vo.w, fsub(p1.w, p0.w), dmp.w);
    return r;
}

// as vel4, with a per-face gradient order (bit q of m4) and existence (bit q of ok)
__device__ __forceinline__ float4 vel4_masked(const Coef& cf, float4 pm, float4 p0, float4 p1,
                                             float4 p2, float4 vo, float4 dmp, int m4, int ok)
{
    float4 r;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float gr = grad4(cf, at(pm, q), at(p0, q), at(p1, q), at(p2, q), (m4 >> q) & 1);
        at(r, q) = ((ok >> q) & 1) ? vupd(cf, at(vo, q), gr, at(dmp, q)) : 0.0f;
    }
    return r;
}

// General-path velocity of four faces: damping from the alphas (PML planes
// and ragged tiles).  Inlined: an out-of-line call here cost the fast path
// about 9 % more instructions through the call's register traffic.
__device__ __forceinline__ float4 vel4_general(Coef cf, float4 pm, float4 p0, float4 p1, float4 p2,
                                            float4 vo, float4 aL, float4 aR, int m4, int ok)
{
    float4 dmp;
#pragma unroll
    for (int q = 0; q < 4; ++q) at(dmp, q) = face_damp(at(aL, q), at(aR, q), cf.dt);
    return vel4_masked(cf, pm, p0, p1, p2, vo, dmp, m4, ok);
}

// P^{n+1} = (P^n - bulk*div) * pd, div = c1*(dx+dy+dz) + c2*(dxx+dyy+dzz)
__device__ __forceinline__ float pupd(const Coef& cf, float p, float xp, float xm, float xpp,
                                      float xmm, float yp, float ym, float ypp, float ymm, float zp,
                                      float zm, float zpp, float zmm, float pd)
{
    const float d1 = fadd(fadd(fsub(xp, xm), fsub(yp, ym)), fsub(zp, zm));
    const float d2 = fadd(fadd(fsub(xpp, xmm), fsub(ypp, ymm)), fsub(zpp, zmm));
    const float dv = fadd(fmul(cf.c1, d1), fmul(cf.c2, d2));
    return fmul(fsub(p, fmul(cf.bulk, dv)), pd);
}

// Load-pipeline state carried by a CTA from one tile to the next: rotating slot
// ids and the mbarrier parity to wait for next, per slot.  Between tiles every
// issued load has been consumed, so pslot[3 .. 3+D] and vslot[0 .. D] are free.
template <class C>
struct Pipe {
    int pslot[C::RING];
    int vslot[C::VSTAGES];
    unsigned pph, vph;
    __device__ void init()
    {
#pragma unroll
        for (int q = 0; q < C::RING; ++q) pslot[q] = q;
#pragma unroll
        for (int q = 0; q < C::VSTAGES; ++q) vslot[q] = q;
        pph = vph = 0;
    }
};

template <class C>
__device__ __forceinline__ unsigned smem_base_u32(float** smem_out)
{
    extern __shared__ float smem_raw[];
    float* const smem = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    *smem_out = smem;
    return smem_u32(smem);
}

template <class C>
__device__ __forceinline__ void init_barriers(unsigned bar0)
{
    if (threadIdx.x == 0) {
        for (int q = 0; q < C::RING + C::VSTAGES; ++q) mbar_init(bar0 + 8u * q, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
}

// One tile (TJ x TK columns, planes [seg*seg_len, ...)) of the fused step.
// Returns false when a load wait ran out (the CTA must stop; status is set).
// PEER = false compiles out the neighbour ghost-plane stores (single rooms and
// batches), which the slab step of a split room needs.  WALLS = true adds the
// walled-scene rules of the two-pass kernels to the general body: a face whose
// open fraction is 0 is closed (its new velocity is 0), the divergence sees
// each face's velocity times its fraction (when fractions were set), and
// solid cells keep P = 0, in both the interior and the general body.
template <class C, bool PEER = true, bool WALLS = false>
__device__ __forceinline__ bool fused_tile(const FusedArgs& a, const CUtensorMap* tmP,
                                           const CUtensorMap* tmX, const CUtensorMap* tmY,
                                           const CUtensorMap* tmZ, int tile, int seg, int seg_len,
                                           int tiles_k, float* smem, unsigned sbase, unsigned bar0,
                                           Pipe<C>& pp, bool acquire_maps = false)
{
    float* const vyn = smem + C::VYN0;
    float* const vzn = smem + C::VZN0;
    float* const ay_s = smem + C::AY0;
    float* const az_s = smem + C::AZ0;
    int* const pslot = pp.pslot;
    int* const vslot = pp.vslot;
    unsigned& pph = pp.pph;
    unsigned& vph = pp.vph;

    const Grid g = a.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, sz = g.sz;
    const long long PL = g.plane;
    // lane = this thread's float4 column in its row, w = its row in the tile
    // (with 32 threads per row: the hardware lane and warp)
    const int tid = threadIdx.x, lane = tid % C::LW, w = tid / C::LW;
    const int tk = tile % tiles_k, tj = tile / tiles_k;
    const int j0 = tj * C::TJ, k0 = tk * C::TK;
    // own planes and the global frame (a slab of a split room, or the whole room)
    const bool slab = a.xs.nxg > 0;
    const int nxg = slab ? a.xs.nxg : nx, xg0 = slab ? a.xs.xg0 : 0;
    const int own_lo = slab ? a.xs.i_lo : 0, own_hi = slab ? a.xs.i_lo + a.xs.n_own : nx;
    const int i_beg = own_lo + seg * seg_len;
    if (i_beg >= own_hi) return true;
    const int i_end = min(i_beg + seg_len, own_hi);
    const Coef cf = a.cf;

    __syncthreads();   // the previous tile's readers of the tables are done
    for (int e = tid; e < C::AY_N; e += C::NT) {
        const int j = j0 - 2 + e;
        ay_s[e] = (j >= 0 && j < ny) ? __ldg(a.tb.ay + j) : 0.0f;
    }
    for (int e = tid; e < C::PC; e += C::NT) {
        const int k = k0 - 4 + e;
        az_s[e] = (k >= 0 && k < nz) ? __ldg(a.tb.az + k) : 0.0f;
    }
    __syncthreads();

    // Loads feeding iteration u (issued by thread 0): P plane u, Vx face u-2,
    // Vy/Vz of plane u-3.  An iteration without V loads still completes its V
    // stage's phase (expect_tx of 0 bytes is a plain arrive).
    auto issue = [&](int u, int ps, int vsg) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        const unsigned pb = bar0 + 8u * ps;
        mbar_expect_tx(pb, C::P_BYTES);
        if (u != a.hold_plane)
            tma_load3(sbase + 4u * (C::RING0 + ps * C::P_STAGE), tmP, k0 - 4, j0 - 3, u, pb);
        const int f = u - 2, io = u - 3, fg = f + xg0;
        const bool vx = (u >= i_beg && fg >= 0 && fg <= nxg - 2);
        const bool vyz = (io >= i_beg && io < i_end);
        const unsigned vb = bar0 + 8u * (C::RING + vsg);
        const unsigned vdst = sbase + 4u * (C::VST0 + vsg * C::V_STAGE);
        mbar_expect_tx(vb, (vx ? C::VX_BYTES : 0u) + (vyz ? C::VYZ_BYTES : 0u));
        if (vx) tma_load3(vdst + 4u * C::VX_OFF, tmX, k0, j0, f, vb);
        if (vyz) {
            tma_load3(vdst + 4u * C::VY_OFF, tmY, k0, j0 - 2, io, vb);
            tma_load3(vdst + 4u * C::VZ_OFF, tmZ, k0 - 4, j0, io, vb);
        }
    };

    if (acquire_maps && tid == 0) {
        acquire_tensormap(tmP);
        acquire_tensormap(tmX);
        acquire_tensormap(tmY);
        acquire_tensormap(tmZ);
    }
    const int u0 = i_beg - 3, u1 = i_end + 2;
    // Slot ids, rotated each iteration.  At iteration u: pslot[0..3] hold planes
    // u-3 .. u, pslot[4 .. 3+D-1] planes u+1 .. u+D-1 in flight, pslot[3+D] is
    // free; vslot[0] holds iteration u's V data, vslot[1 .. D-1] the next
    // iterations' in flight, vslot[D] is free.  pph/vph: parity to wait for, per slot.
    // The first D iterations' loads go into the free slots left by the previous tile.
    if (tid == 0)
        for (int q = 0; q < C::D; ++q) issue(u0 + q, pslot[3 + q], vslot[q]);

    // ---- per-thread constants of the own row and columns
    const int jr = j0 + w;
    const int kb = k0 + 4 * lane;                 // first own k
    const bool row_ok = jr < ny;
    const bool kfull = k0 + C::TK <= nz;          // every own k of the CTA is a cell
    const bool st_ok = row_ok && kb < sz;         // the float4 store stays inside the row
    const int own = row_ok ? jr * sz + kb : 0;    // in-plane offset of the own float4
    const int cP = (w + 3) * C::PC + 4 * lane + 4;    // own cells in a P stage
    int zm4 = 0, zok = 0;                         // own Vz faces: 4th order / existing
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int kf = kb + q;
        zm4 |= (kf > 0 && kf < nz - 2) ? (1 << q) : 0;
        zok |= (kf <= nz - 2) ? (1 << q) : 0;
    }
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
    // Vy items of this thread: row w (all warps) and row TJ+w (the first VYR-TJ warps)
    constexpr int NY_IT = 2;
    float4 dyi[NY_IT];
#pragma unroll
    for (int m = 0; m < NY_IT; ++m) {
        const int r = m == 0 ? w : C::TJ + w;
        dyi[m] = make_float4(1.f, 1.f, 1.f, 1.f);
        if (r < C::VYR) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float azk = az_s[4 * lane + 4 + q];
                at(dyi[m], q) = face_damp(fmaxf(ay_s[r], azk), fmaxf(ay_s[r + 1], azk), cf.dt);
            }
        }
    }
    float4 qx0 = make_float4(0.f, 0.f, 0.f, 0.f), qx1 = qx0, qx2 = qx0, qx3 = qx0;
    int u_fail = u1 + 1;   // iteration whose wait ran out (none)
    // alpha_x / px window: at iteration u, axw{3,2,1,0} = alpha_x[u-3 .. u] and
    // pxw = px[u-3]; the next iteration's values are prefetched one iteration ahead
    auto ax_at = [&](int q) { return (q >= 0 && q < nx) ? __ldg(a.tb.ax + q) : 0.0f; };
    auto px_at = [&](int q) { return (q >= 0 && q < nx) ? __ldg(a.tb.px + q) : 1.0f; };
    float axw3 = ax_at(u0 - 3), axw2 = ax_at(u0 - 2), axw1 = ax_at(u0 - 1), axw0 = ax_at(u0);
    float pxw = px_at(u0 - 3);

    // The interior iterations of a tile whose columns are all cells take a
    // separately compiled body without the general path (the general path
    // present in the loop costs the interior about 12 % although it never runs
    // there).  Iteration u is interior when plane u-3 and faces u-2 .. u-1 have
    // no x absorption, face u-2 has the 4th-order gradient and the planes u-3,
    // u-2 are own ones.  Rows beyond the room and Vy faces at the j ends are
    // warp-uniform cases the interior body handles itself.  Both bodies
    // evaluate the same expressions (alpha_x = 0, px = 1 there), so the results
    // do not depend on the choice.  The step runs in one wave, so a CTA left on
    // the general body for its whole march would set the kernel's time.
    const bool clean = kfull;
    int fast_lo = u1 + 1, fast_hi = u1 + 1;
    if (clean && a.tb.xi_hi > a.tb.xi_lo) {
        fast_lo = max(max(a.tb.xi_lo + 3, 3 - xg0), i_beg + 3);
        fast_hi = min(min(a.tb.xi_hi + 1, nxg - xg0), u1 + 1);
        if (fast_lo >= fast_hi) fast_lo = fast_hi = u1 + 1;
    }

    // One iteration of the march; FAST = the interior body.  False when a load
    // wait ran out (u_fail is then set).
    auto iteration = [&](const int u, auto fast_tag) -> bool {
        constexpr bool FAST = decltype(fast_tag)::value;
        // wait for plane u (P) and iteration u's V data; the decision to stop on a
        // timeout is made by the whole CTA (the barrier below is also the one that
        // separates the previous iteration's reads from this iteration's writes)
        const int ps = pslot[3], vsg = vslot[0];
        // WALLS: this iteration's face fractions and solid flags, loaded before
        // the wait so that their latency overlaps it (they do not depend on it)
        float4 pf_x = make_float4(1.f, 1.f, 1.f, 1.f), pf_y0 = pf_x, pf_y1 = pf_x, pf_z = pf_x;
        float pf_h = 1.0f;
        unsigned pf_s = 0u;
        if constexpr (WALLS) {
            const int f = u - 2, i = u - 3;
            if (a.fr[0] && st_ok && u >= i_beg && f >= 0 && f <= nx - 2) pf_x = ldg4(a.fr[0] + f * PL + own);
            if (i >= i_beg) {
                const long long ib = (long long)i * PL;
                if (a.fr[1] && kb < sz) {
                    const int jf0 = j0 - 2 + w, jf1 = j0 - 2 + C::TJ + w;
                    if (jf0 >= 0 && jf0 <= ny - 2) pf_y0 = ldg4(a.fr[1] + ib + (long long)jf0 * sz + kb);
                    if (C::TJ + w < C::VYR && jf1 >= 0 && jf1 <= ny - 2)
                        pf_y1 = ldg4(a.fr[1] + ib + (long long)jf1 * sz + kb);
                }
                if (a.fr[2] && st_ok) pf_z = ldg4(a.fr[2] + ib + own);
                const int hl = tid - (C::NT - 32 * C::HW);
                if (a.fr[2] && hl >= 0 && hl < 3 * C::TJ) {
                    const int jl = hl / 3, which = hl - 3 * jl;
                    const int kf = k0 - 4 + (which < 2 ? 2 + which : C::TK + 4);
                    if (j0 + jl < ny && kf >= 0 && kf <= nz - 2)
                        pf_h = __ldg(a.fr[2] + ib + (long long)(j0 + jl) * sz + kf);
                }
                if (a.solid && row_ok && kb < sz)
                    pf_s = __ldg(reinterpret_cast<const unsigned*>(a.solid + ib + own));
            }
        }
        const bool ok = mbar_wait(bar0 + 8u * ps, (pph >> ps) & 1u, a.wait_us) &&
                        mbar_wait(bar0 + 8u * (C::RING + vsg), (vph >> vsg) & 1u, a.wait_us);
        // the source deposit, on the arriving plane's shared copy before anyone reads it
        if (a.dep_sig && u == a.dep_i && tid == 0 && ok) {
            const int dj = a.dep_j - (j0 - 3), dk = a.dep_k - (k0 - 4);
            const float amp = a.dep_sig[a.dep_step];
            if (dj >= 0 && dj < C::PR && dk >= 0 && dk < C::PC && amp != 0.0f) {
                float* c = smem + C::RING0 + ps * C::P_STAGE + dj * C::PC + dk;
                *c = fadd(*c, amp);
            }
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicMin(a.status + kStatusTimeout, blockIdx.x + gridDim.x * blockIdx.y);
            u_fail = u;
            return false;
        }
        pph ^= 1u << ps;
        vph ^= 1u << vsg;
        // iteration u+D's loads go into the slots iteration u-1 freed (their last
        // reads came before the barrier above), so thread 0 issues them before
        // its own work of this iteration rather than after it
        if (tid == 0 && u + C::D <= u1) issue(u + C::D, pslot[C::RING - 1], vslot[C::VSTAGES - 1]);
        float ax_next = 0.0f, px_next = 1.0f;
        if constexpr (!FAST) {
            ax_next = ax_at(u + 1);
            px_next = px_at(u - 2);
        }
        const float* vs = smem + C::VST0 + vsg * C::V_STAGE;

        // ---- new Vx on face f = u-2 of the own columns (planes f-1 .. f+2) ----
        if (FAST || u >= i_beg) {
            const int f = u - 2, fg = f + xg0;
            float4 vnew = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 vdiv = vnew;   // WALLS: the value the divergence sees
            if (FAST ? row_ok : (fg >= 0 && fg <= nxg - 2 && row_ok)) {
                const float4 pm = lds4(smem + C::RING0 + pslot[0] * C::P_STAGE + cP);
                const float4 p0 = lds4(smem + C::RING0 + pslot[1] * C::P_STAGE + cP);
                const float4 p1 = lds4(smem + C::RING0 + pslot[2] * C::P_STAGE + cP);
                const float4 p2 = lds4(smem + C::RING0 + pslot[3] * C::P_STAGE + cP);
                const float4 vo = lds4(vs + C::VX_OFF + 4 * tid);
                if constexpr (FAST) {
                    vnew = vel4(cf, pm, p0, p1, p2, vo, dxi);
                } else {
                    const bool fourth = (fg > 0 && fg < nxg - 2);
                    const float axf = axw2, axf1 = axw1;     // alpha_x[f], alpha_x[f+1]
                    if (fourth && axf == 0.0f && axf1 == 0.0f && kfull) {
                        vnew = vel4(cf, pm, p0, p1, p2, vo, dxi);
                    } else {
                        float4 aL, aR;
                        int okx = 0;
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            at(aL, q) = fmaxf(axf, at(myz, q));
                            at(aR, q) = fmaxf(axf1, at(myz, q));
                            okx |= (kb + q < nz) ? (1 << q) : 0;
                        }
                        vnew = vel4_general(cf, pm, p0, p1, p2, vo, aL, aR, fourth ? 15 : 0, okx);
                    }
                }
                if constexpr (WALLS) {
                    vdiv = vnew;
                    if (a.fr[0] && st_ok) {
                        const float4 fr = pf_x;
                        vnew = close4(vnew, fr);
                        vdiv = a.frac_div ? mul4(vnew, fr) : vnew;
                    }
                }
                if (f >= i_beg && f < i_end && st_ok) {
                    stg4(a.vout[0] + f * PL + own, vnew);
#pragma unroll
                    for (int sd = 0; sd < 2; ++sd)   // the neighbours' ghost faces
                        if (PEER && a.pr.vx[sd] && f >= a.pr.v_lo[sd] && f < a.pr.v_hi[sd])
                            stg4(a.pr.vx[sd] + (f + a.pr.dl[sd]) * PL + own, vnew);
                }
            }
            qx0 = qx1; qx1 = qx2; qx2 = qx3; qx3 = WALLS ? vdiv : vnew;
        }

        // ---- plane i = u-3: new Vy / Vz (with halos), then P^{n+1} ----
        {
            const int i = u - 3;
            if (FAST || i >= i_beg) {
                const float axi = FAST ? 0.0f : axw3;    // alpha_x[i]
                const bool xint = FAST || (axi == 0.0f);
                const float* pst = smem + C::RING0 + pslot[0] * C::P_STAGE;
                const float* vys = vs + C::VY_OFF;
                const float* vzs = vs + C::VZ_OFF;
                const long long ib = i * PL;

                // Vy rows: row w, and row TJ+w for the first VYR-TJ warps
#pragma unroll
                for (int m = 0; m < NY_IT; ++m) {
                    const int r = m == 0 ? w : C::TJ + w;
                    if (r < C::VYR) {
                        const int jf = j0 - 2 + r;
                        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (jf >= 0 && jf <= ny - 2) {
                            const float* pc = pst + 4 * lane + 4;
                            const float4 pm = lds4(pc + r * C::PC), p0 = lds4(pc + (r + 1) * C::PC);
                            const float4 p1 = lds4(pc + (r + 2) * C::PC), p2 = lds4(pc + (r + 3) * C::PC);
                            const float4 vo = lds4(vys + r * C::TK + 4 * lane);
                            if constexpr (FAST) {
                                // the row's gradient order is uniform over its threads
                                if (jf > 0 && jf < ny - 2) v = vel4(cf, pm, p0, p1, p2, vo, dyi[m]);
                                else v = vel4_2nd(cf, p0, p1, vo, dyi[m]);
                            } else {
                                const bool fourth = (jf > 0 && jf < ny - 2);
                                if (fourth && xint && kfull) {
                                    v = vel4(cf, pm, p0, p1, p2, vo, dyi[m]);
                                } else {
                                    float4 aL, aR;
                                    int oky = 0;
#pragma unroll
                                    for (int q = 0; q < 4; ++q) {
                                        const float azk = az_s[4 * lane + 4 + q];
                                        at(aL, q) = fmaxf(fmaxf(axi, ay_s[r]), azk);
                                        at(aR, q) = fmaxf(fmaxf(axi, ay_s[r + 1]), azk);
                                        oky |= (kb + q < nz) ? (1 << q) : 0;
                                    }
                                    v = vel4_general(cf, pm, p0, p1, p2, vo, aL, aR, fourth ? 15 : 0, oky);
                                }
                            }
                            float4 fry = make_float4(1.f, 1.f, 1.f, 1.f);
                            if constexpr (WALLS) {
                                if (a.fr[1] && kb < sz) {
                                    fry = m == 0 ? pf_y0 : pf_y1;
                                    v = close4(v, fry);
                                }
                            }
                            if (r >= 2 && r < C::TJ + 2 && kb < sz)
                                stg4(a.vout[1] + ib + (long long)jf * sz + kb, v);
                            if constexpr (WALLS) {
                                if (a.fr[1] && a.frac_div && kb < sz) v = mul4(v, fry);
                            }
                        }
                        sts4(vyn + r * C::TK + 4 * lane, v);
                    }
                }

                // Vz: own faces kb .. kb+3 of row jr
                float4 pown = make_float4(0.f, 0.f, 0.f, 0.f);
                {
                    const float* prow = pst + (w + 3) * C::PC;
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (row_ok) {
                        const int c = 4 * lane + 4;            // col of kb
                        pown = lds4(prow + c);
                        const float4 pb4 = lds4(prow + c + 4);
                        const float pl = prow[c - 1];
                        const float4 vo = lds4(vzs + w * C::PC + c);
                        // faces kb+q use P[kb+q-1 .. kb+q+2]
                        const float4 pm = make_float4(pl, pown.x, pown.y, pown.z);
                        const float4 p1 = make_float4(pown.y, pown.z, pown.w, pb4.x);
                        const float4 p2 = make_float4(pown.z, pown.w, pb4.x, pb4.y);
                        if (xint) {
                            v = vel4_masked(cf, pm, pown, p1, p2, vo, dzi, zm4, zok);
                        } else {
                            const float ay = ay_s[w + 2];
                            float4 aL, aR;
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                at(aL, q) = fmaxf(fmaxf(axi, ay), az_s[c + q]);
                                at(aR, q) = fmaxf(fmaxf(axi, ay), az_s[c + q + 1]);
                            }
                            v = vel4_general(cf, pm, pown, p1, p2, vo, aL, aR, zm4, zok);
                        }
                        float4 frz = make_float4(1.f, 1.f, 1.f, 1.f);
                        if constexpr (WALLS) {
                            if (a.fr[2] && st_ok) {
                                frz = pf_z;
                                v = close4(v, frz);
                            }
                        }
                        if (st_ok) stg4(a.vout[2] + ib + own, v);
                        if constexpr (WALLS) {
                            if (a.fr[2] && a.frac_div && st_ok) v = mul4(v, frz);
                        }
                    }
                    sts4(vzn + w * C::PC + 4 * lane + 4, v);
                }
                // halo Vz faces k0-2, k0-1, k0+TK of every row: 3*TJ faces, one per
                // thread of the last HW warps
                const int hl = tid - (C::NT - 32 * C::HW);
                if (hl >= 0 && hl < 3 * C::TJ) {
                    const int jl = hl / 3, which = hl - 3 * jl;
                    const int ch = which < 2 ? 2 + which : C::TK + 4;
                    const int kf = k0 - 4 + ch;
                    const float* prow = pst + (jl + 3) * C::PC;
                    float vh = 0.0f;
                    if (j0 + jl < ny && kf >= 0 && kf <= nz - 2) {
                        const bool fourth = (kf > 0 && kf < nz - 2);
                        const float ay = ay_s[jl + 2];
                        const float gr = grad4(cf, prow[ch - 1], prow[ch], prow[ch + 1], prow[ch + 2], fourth);
                        const float dmp = face_damp(fmaxf(fmaxf(axi, ay), az_s[ch]),
                                                    fmaxf(fmaxf(axi, ay), az_s[ch + 1]), cf.dt);
                        vh = vupd(cf, vzs[jl * C::PC + ch], gr, dmp);
                        if constexpr (WALLS) {
                            if (a.fr[2]) {
                                const float fz = pf_h;
                                if (fz == 0.0f) vh = 0.0f;
                                if (a.frac_div) vh = fmul(vh, fz);
                            }
                        }
                    }
                    vzn[jl * C::PC + ch] = vh;
                }
                __syncthreads();

                // P^{n+1} of the own cells
                if (row_ok) {
                    const float* yr = vyn + 4 * lane;
                    const float4 ymm = lds4(yr + w * C::TK), ym = lds4(yr + (w + 1) * C::TK);
                    const float4 yp = lds4(yr + (w + 2) * C::TK), ypp = lds4(yr + (w + 3) * C::TK);
                    const float* zr = vzn + w * C::PC + 4 * lane;
                    const float2 za = *reinterpret_cast<const float2*>(zr + 2);   // faces kb-2, kb-1
                    const float4 zb = lds4(zr + 4);                                // faces kb .. kb+3
                    const float zc = zr[8];                                        // face kb+4
                    // px[i] = 1 on x-interior planes, so min(px[i], min(py, pz)) = mpz there
                    float4 pd = mpz;
                    if constexpr (!FAST) {
                        const float pxi = pxw;
#pragma unroll
                        for (int q = 0; q < 4; ++q) at(pd, q) = fminf(pxi, at(mpz, q));
                    }
                    float4 out;
                    out.x = pupd(cf, pown.x, qx2.x, qx1.x, qx3.x, qx0.x, yp.x, ym.x, ypp.x, ymm.x, zb.x, za.y, zb.y, za.x, pd.x);
                    out.y = pupd(cf, pown.y, qx2.y, qx1.y, qx3.y, qx0.y, yp.y, ym.y, ypp.y, ymm.y, zb.y, zb.x, zb.z, za.y, pd.y);
                    out.z = pupd(cf, pown.z, qx2.z, qx1.z, qx3.z, qx0.z, yp.z, ym.z, ypp.z, ymm.z, zb.z, zb.y, zb.w, zb.x, pd.z);
                    out.w = pupd(cf, pown.w, qx2.w, qx1.w, qx3.w, qx0.w, yp.w, ym.w, ypp.w, ymm.w, zb.w, zb.z, zc, zb.y, pd.w);
                    if (!FAST && !kfull) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            if (kb + q >= nz) at(out, q) = 0.0f;
                    }
                    if constexpr (WALLS) {
                        if (a.solid && kb < sz) {   // solid cells keep P = 0
                            const unsigned sol = pf_s;
#pragma unroll
                            for (int q = 0; q < 4; ++q)
                                if ((sol >> (8 * q)) & 0xFFu) at(out, q) = 0.0f;
                        }
                    }
                    if (kb < sz) {
                        stg4(a.pn + ib + own, out);
#pragma unroll
                        for (int sd = 0; sd < 2; ++sd)   // the neighbours' ghost planes
                            if (PEER && a.pr.pn[sd] && i >= a.pr.p_lo[sd] && i < a.pr.p_hi[sd])
                                stg4(a.pr.pn[sd] + (i + a.pr.dl[sd]) * PL + own, out);
                    }
                }
            }
        }

        if constexpr (!FAST) {
            axw3 = axw2; axw2 = axw1; axw1 = axw0; axw0 = ax_next;
            pxw = px_next;
        }
        // rotate: after it pslot[q] holds plane u+1-3+q and vslot[q] iteration u+1+q.
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
            // the window of the general iterations that follow
            axw3 = ax_at(u - 3); axw2 = ax_at(u - 2); axw1 = ax_at(u - 1); axw0 = ax_at(u);
            pxw = px_at(u - 3);
            continue;
        }
        if (!iteration(u, std::false_type{})) break;
        ++u;
    }

    // A normal march waits for every load it issued, so none is in flight here.
    // After a timed-out wait at iteration u_fail, the copies issued for
    // iterations u_fail .. u_fail+D-1 may still be landing: wait for them
    // (bounded) before the CTA's shared memory is released.
    if (u_fail <= u1) {
        if (tid == 0) {
            for (int q = 0; q < C::D && u_fail + q <= u1; ++q) {
                const int ps = pslot[3 + q], vsg = vslot[q];
                mbar_wait(bar0 + 8u * ps, (pph >> ps) & 1u, a.wait_us);
                mbar_wait(bar0 + 8u * (C::RING + vsg), (vph >> vsg) & 1u, a.wait_us);
            }
        }
        __syncthreads();
        return false;
    }
    return true;
}

// Single-room step: one CTA per (tile, segment).
template <class C, bool PEER, bool WALLS = false>
__global__ void __launch_bounds__(C::NT) k_fused_step(FusedArgs a,
                                                      const __grid_constant__ CUtensorMap tmP,
                                                      const __grid_constant__ CUtensorMap tmX,
                                                      const __grid_constant__ CUtensorMap tmY,
                                                      const __grid_constant__ CUtensorMap tmZ,
                                                      int seg_len, int tiles_k)
{
    if (a.n_rec > 0) {   // the previous step's receivers, from this step's input P
        const int nblk = gridDim.x * gridDim.y, b = blockIdx.x + gridDim.x * blockIdx.y;
        for (int r = b + nblk * (int)threadIdx.x; r < a.n_rec; r += nblk * C::NT)
            a.rec_out[r] = sample8(a.p, a.rec_idx + 8 * r, a.rec_w + 8 * r);
    }
    if ((int)blockIdx.y * seg_len >= (a.xs.nxg > 0 ? a.xs.n_own : a.g.nx)) return;
    float* smem;
    const unsigned sbase = smem_base_u32<C>(&smem);
    const unsigned bar0 = sbase + 4u * C::BAR0;
    init_barriers<C>(bar0);
    Pipe<C> pp;
    pp.init();
    fused_tile<C, PEER, WALLS>(a, &tmP, &tmX, &tmY, &tmZ, blockIdx.x, blockIdx.y, seg_len, tiles_k, smem,
                               sbase, bar0, pp);
}


// Batched step: a persistent kernel whose CTAs pull (member, tile, segment)
// work items from a device counter until the list is exhausted; members at
// their step limit are skipped.  Uneven members balance across the SMs.  The
// members' tensor maps live in global memory and are rewritten when the set
// changes, so each work item acquires them before its first TMA load.
template <class C>
__global__ void __launch_bounds__(C::NT, 2) k_fused_batch(BatchMember* __restrict__ mem,
                                                          BatchHeader* __restrict__ hdr,
                                                          const int* __restrict__ item_member,
                                                          unsigned* __restrict__ status)
{
    __shared__ int s_item;
    const int total_items = hdr->total_items;
    int* const counter = &hdr->counter;
    float* smem;
    const unsigned sbase = smem_base_u32<C>(&smem);
    const unsigned bar0 = sbase + 4u * C::BAR0;
    init_barriers<C>(bar0);
    Pipe<C> pp;
    pp.init();
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total_items) break;
        const BatchMember* m = mem + item_member[item];
        const int step = m->step;
        if (step >= m->limit || m->unstable != 0xFFFFFFFFu) continue;   // done, or stopped unstable
        const int par = (step - m->step0) & 1;
        FusedArgs a;
        a.g = m->g;
        a.cf = m->cf;
        a.tb = m->tb;
        a.p = m->p[par];
        a.pn = m->p[par ^ 1];
        for (int c = 0; c < 3; ++c) {
            a.vin[c] = m->v[par][c];
            a.vout[c] = m->v[par ^ 1][c];
        }
        a.status = status;
        a.xs = XSpan{0, 0, 0, 0};
        a.pr = XPeers{};
        const int local = item - m->items_begin;
        if (!fused_tile<C, false>(a, &m->maps[par][0], &m->maps[par][1], &m->maps[par][2], &m->maps[par][3],
                           local % m->tiles, local / m->tiles, m->seg_len, m->tiles_k, smem, sbase,
                           bar0, pp, true))
            break;
    }
}

// After a batched step, per member below its limit: record the receivers from
// the new pressure, advance the step counter, run the 256-step check, then
// deposit the next step's source sample (the order of the single-room path:
// record after step n, deposit before step n+1).  One block per member.  A
// member whose check fails stops at that step without the next deposit, the
// state a single room is left in when its step returns UNSTABLE; the batch
// steps it no further until its set is rebuilt.
__global__ void k_batch_epilogue(BatchMember* __restrict__ mem, const BatchHeader* __restrict__ hdr)
{
    const int r = blockIdx.x;
    if (r >= hdr->n_members) return;
    BatchMember* m = mem + r;
    const int s = m->step;
    if (s >= m->limit || m->unstable != 0xFFFFFFFFu) return;
    const int s1 = s + 1;
    float* P = m->p[(s1 - m->step0) & 1];
    const int slot = m->trace0 + (s - m->step0);
    if (slot < m->trace_cap)
        for (int q = threadIdx.x; q < m->n_rec; q += blockDim.x)
            m->trace[(size_t)slot * m->n_rec + q] = sample8(P, m->rec_idx + 8 * q, m->rec_w + 8 * q);
    if ((s1 & (kCheckPeriod - 1)) == 0) {
        const int n_chk = s1 / kCheckPeriod - m->step0 / kCheckPeriod;
        const long long phase = (m->phase0 + n_chk - 1) % kCheckStride;
        const Grid g = m->g;
        for (long long q = phase + (long long)kCheckStride * threadIdx.x; q < m->n_cells;
             q += (long long)kCheckStride * blockDim.x) {
            const int k = (int)(q % g.nz);
            const long long ij = q / g.nz;
            const float v = P[((ij / g.ny) * g.ny + ij % g.ny) * g.sz + k];
            if (!isfinite(v) || v > 2e3f || v < -2e3f) atomicCAS(&m->unstable, 0xFFFFFFFFu, (unsigned)s1);
        }
    }
    __syncthreads();   // receivers have read P and the check's flags are set
    if (threadIdx.x == 0) {
        const bool stopped = *(volatile unsigned*)&m->unstable != 0xFFFFFFFFu;
        if (!stopped && s1 < m->limit && s1 < m->ps_n) deposit_apply(m->ps, m->ps_sig[s1], P);
        m->step = s1;
    }
}

using FusedCfg = Cfg<8, 2>;          // 8 x 128 tiles: single rooms, and batches by default
using NarrowCfg = Cfg<16, 2, 16>;    // 16 x 64 tiles: batches of rooms with small Nz

constexpr int kMaxDevices = 64;
int g_slots_per_sm[2][kMaxDevices];   // per tile shape and device
int g_sms[2][kMaxDevices];
bool g_configured[2][kMaxDevices];

}  // namespace

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

cudaError_t get_encoder()
{
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return g_encode ? cudaSuccess : cudaErrorNotSupported;
}
}  // namespace

cudaError_t encode_field_map(CUtensorMap* m, const void* base, int elem_bytes, const Grid& g, int bx, int by)
{
    cudaError_t e = get_encoder();
    if (e != cudaSuccess) return e;
    if (elem_bytes != 4 && elem_bytes != 2) return cudaErrorInvalidValue;
    const cuuint64_t eb = (cuuint64_t)elem_bytes;
    cuuint64_t dims[3] = {(cuuint64_t)g.sz, (cuuint64_t)g.ny, (cuuint64_t)g.nx};
    cuuint64_t strides[2] = {(cuuint64_t)g.sz * eb, (cuuint64_t)g.plane * eb};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = g_encode(m, elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 3,
                          const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

struct FusedCache {
    struct Entry {
        const float* base;
        int kind, shape;
        CUtensorMap map;
    };
    std::vector<Entry> entries;
};

FusedCache* fused_cache_create() { return new FusedCache(); }
void fused_cache_destroy(FusedCache* c) { delete c; }

template <class C>
void box_of(int kind, int* bx, int* by)
{
    const int x[4] = {C::PC, C::TK, C::TK, C::PC};
    const int y[4] = {C::PR, C::TJ, C::VYR, C::TJ};
    *bx = x[kind];
    *by = y[kind];
}

static cudaError_t cached_map(FusedCache* c, const float* base, int kind, const Grid& g, CUtensorMap* out,
                              int shape = 0)
{
    for (const auto& e : c->entries)
        if (e.base == base && e.kind == kind && e.shape == shape) { *out = e.map; return cudaSuccess; }
    int bx, by;
    if (shape == 1) box_of<NarrowCfg>(kind, &bx, &by);
    else box_of<FusedCfg>(kind, &bx, &by);
    FusedCache::Entry e;
    e.base = base;
    e.kind = kind;
    e.shape = shape;
    cudaError_t err = encode_field_map(&e.map, base, 4, g, bx, by);
    if (err != cudaSuccess) return err;
    c->entries.push_back(e);
    *out = e.map;
    return cudaSuccess;
}

bool fused_supported(const Grid& g)
{
    return g.nx >= 1 && g.ny >= 1 && g.nz >= 1 && (g.sz % 8) == 0;
}

int fused_kernel_launches_per_step() { return 1; }

template <class C>
static cudaError_t launch_step_of(const FusedArgs& a, FusedCache* cache, cudaStream_t s, int shape)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_configured[shape][dev]) {
        e = cudaFuncSetAttribute(k_fused_step<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_fused_step<C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k_fused_step<C, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&g_sms[shape][dev], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        int slots = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&slots, k_fused_step<C, true>, C::NT, C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        int slots_w = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&slots_w, k_fused_step<C, false, true>, C::NT,
                                                          C::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        slots = slots < slots_w ? slots : slots_w;
        g_slots_per_sm[shape][dev] = slots > 0 ? slots : 1;
        g_configured[shape][dev] = true;
    }
    const Grid& g = a.g;
    CUtensorMap maps[4];
    const float* bases[4] = {a.p, a.vin[0], a.vin[1], a.vin[2]};
    for (int q = 0; q < 4; ++q) {
        e = cached_map(cache, bases[q], q, g, &maps[q], shape);
        if (e != cudaSuccess) return e;
    }
    const int tiles_j = (g.ny + C::TJ - 1) / C::TJ;
    const int tiles_k = (g.nz + C::TK - 1) / C::TK;
    const long long tiles = (long long)tiles_j * tiles_k;
    // segments along i: as many as one wave of resident CTAs holds (every CTA
    // marches the same number of planes, so a single full wave has no tail)
    const long long slots = (long long)g_slots_per_sm[shape][dev] * g_sms[shape][dev];
    const int n_own = a.xs.nxg > 0 ? a.xs.n_own : g.nx;
    long long segs = slots / tiles;
    if (segs < 1) segs = 1;
    if (segs > n_own) segs = n_own;
    const int seg_len = (int)((n_own + segs - 1) / segs);
    segs = (n_own + seg_len - 1) / seg_len;
    dim3 grid((unsigned)tiles, (unsigned)segs, 1);
    const bool peer = a.pr.pn[0] || a.pr.pn[1] || a.pr.vx[0] || a.pr.vx[1];
    const bool walls = a.fr[0] || a.fr[1] || a.fr[2] || a.solid;
    if (walls && (peer || a.xs.nxg > 0)) return cudaErrorInvalidValue;   // walled scenes are whole rooms
    if (walls)
        k_fused_step<C, false, true><<<grid, C::NT, C::SMEM_BYTES, s>>>(a, maps[0], maps[1], maps[2], maps[3],
                                                                        seg_len, tiles_k);
    else if (peer)
        k_fused_step<C, true><<<grid, C::NT, C::SMEM_BYTES, s>>>(a, maps[0], maps[1], maps[2], maps[3], seg_len,
                                                                 tiles_k);
    else
        k_fused_step<C, false><<<grid, C::NT, C::SMEM_BYTES, s>>>(a, maps[0], maps[1], maps[2], maps[3], seg_len,
                                                                  tiles_k);
    return cudaGetLastError();
}

// The tile shape a room's step uses: 16 x 64 tiles when they leave less of the
// last k tile idle than 8 x 128 tiles (e.g. Nz = 32, 48, 144, 160), else 8 x 128.
int fused_step_shape(const Grid& g)
{
    const int w128 = (g.nz + 127) / 128 * 128 - g.nz, w64 = (g.nz + 63) / 64 * 64 - g.nz;
    return w64 < w128 ? 1 : 0;
}

cudaError_t launch_fused_step(const FusedArgs& a, FusedCache* cache, cudaStream_t s)
{
    return fused_step_shape(a.g) == 1 ? launch_step_of<NarrowCfg>(a, cache, s, 1)
                                      : launch_step_of<FusedCfg>(a, cache, s, 0);
}

cudaError_t fused_maps(FusedCache* c, const Grid& g, const float* p, const float* const* v,
                       CUtensorMap out[4], int shape)
{
    const float* bases[4] = {p, v[0], v[1], v[2]};
    for (int q = 0; q < 4; ++q) {
        cudaError_t e = cached_map(c, bases[q], q, g, &out[q], shape);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void fused_tile_shape(int shape, int* tj, int* tk)
{
    *tj = shape == 1 ? NarrowCfg::TJ : FusedCfg::TJ;
    *tk = shape == 1 ? NarrowCfg::TK : FusedCfg::TK;
}

template <class C>
static cudaError_t batch_slots_of(int* slots)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_fused_batch<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)C::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    int sms = 0, per = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fused_batch<C>, C::NT, C::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    *slots = (per > 0 ? per : 1) * sms;
    return cudaSuccess;
}

cudaError_t fused_batch_slots(int shape, int* slots)
{
    return shape == 1 ? batch_slots_of<NarrowCfg>(slots) : batch_slots_of<FusedCfg>(slots);
}

cudaError_t launch_fused_batch_step(BatchMember* members, BatchHeader* hdr, const int* item_member,
                                    unsigned* status, int grid_ctas, int epi_blocks, cudaStream_t s,
                                    int shape)
{
    cudaError_t e = cudaMemsetAsync(&hdr->counter, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    if (shape == 1)
        k_fused_batch<NarrowCfg><<<grid_ctas, NarrowCfg::NT, NarrowCfg::SMEM_BYTES, s>>>(members, hdr, item_member,
                                                                                       status);
    else
        k_fused_batch<FusedCfg><<<grid_ctas, FusedCfg::NT, FusedCfg::SMEM_BYTES, s>>>(members, hdr, item_member,
                                                                                     status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_batch_epilogue<<<epi_blocks, 128, 0, s>>>(members, hdr);
    return cudaGetLastError();
}

}  // namespace fdtd
