/*
 * fdtd_internal.h — device-side types and kernel launchers of the engine.
 *
 * Device layout (HBM): every field (P current, P next, Vx, Vy, Vz, and the
 * optional face fractions and solid mask) is an [Nx][Ny][Sz] array, Sz = Nz
 * rounded up to 8 floats, so each (i, j) row starts on a 32-byte sector and
 * all four fields share one index id = (i*Ny + j)*Sz + k.  Staggered faces
 * that do not exist (Vx plane Nx-1, Vy row Ny-1, Vz element Nz-1) and the row
 * padding hold zero and are never written.  Absorption is stored as three 1-D
 * per-axis tables (alpha and the pressure damping 1/(1+alpha*dt)); a cell's
 * alpha is the max over its three axes, so no per-cell coefficient array is
 * read by the step.
 *
 * All stencil arithmetic goes through fadd/fsub/fmul (round-to-nearest
 * intrinsics), which keeps every operation separately rounded in the
 * reference's order (csrc/kernels/acoustic_fdtd.cpp:1099-1234): the float32
 * results are bit-identical to the reference built without FMA contraction.
 */
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fdtd {

constexpr int kRowAlign = 8;           // floats per row-padding unit (32 B)
constexpr int kCheckStride = 1013;     // stability sample stride (acoustic_fdtd.cpp:1250)
constexpr int kCheckPeriod = 256;      // steps between checks (acoustic_fdtd.cpp:1284)

// Records a CUDA error for fdtd_b200_last_error (defined in fdtd_capi.cu).
void record_cuda_error(cudaError_t e, const char* what);

struct Grid {
    int nx, ny, nz, sz;
    long long plane;   // ny * sz
    long long cells;   // nx * plane (padded)
};

struct Coef {
    float vc;      // dt / (rho*dx)              (acoustic_fdtd.cpp:1091)
    float bulk;    // rho*c*c*dt*(1/dx)          (acoustic_fdtd.cpp:1173)
    float dt;
    float c1;      // 9/8                        (acoustic_fdtd.cpp:889)
    float c2;      // -1/24                      (acoustic_fdtd.cpp:890)
    float inv_dt;  // 1/dt, plate face velocity  (acoustic_fdtd.cpp:1160)
};

struct Tables {        // per-axis absorption tables, lengths nx, ny, nz
    const float* ax;
    const float* ay;
    const float* az;
    const float* px;   // 1/(1 + ax*dt)
    const float* py;
    const float* pz;
    int xi_lo, xi_hi;  // planes [xi_lo, xi_hi) have ax == 0 (x-interior); empty: none
};

// The longest run [lo, hi) of planes with alpha_x == 0 (the interior between
// the x absorbing layers, extended through a layer whose absorption is 0;
// a slab's ghost planes outside the room also have alpha_x == 0, so the
// longest run is taken); empty when there is none.
inline void x_interior_run(const float* ax, int n, int* lo, int* hi)
{
    int best_lo = 0, best_hi = 0;
    for (int a = 0; a < n;) {
        if (ax[a] != 0.0f) { ++a; continue; }
        int b = a;
        while (b < n && ax[b] == 0.0f) ++b;
        if (b - a > best_hi - best_lo) { best_lo = a; best_hi = b; }
        a = b;
    }
    *lo = best_lo;
    *hi = best_hi;
}

struct PlateCoef {
    float a;    // dt^2 / (rho_s h)
    float bh;   // D dt^2 / (rho_s h dx^4)
    float vd;   // 1 - alpha_M dt
    float bk;   // beta_K / dt * bh
};

// Extra jobs of the two-pass velocity pass for a plate scene (code null: none):
// the plate's face velocities (w - w_prev)/dt on the Vz faces below (code bit 0)
// and above (bit 1) each active node, which overwrite the updated faces as
// k_plate_inject does; and, by the first block, the entries of the consumed
// plate forces back to zero (pack/m, m = 0: none).  Both are skipped when the
// gate reports a failed plate update.
struct PlateFaces {
    const uint8_t* code = nullptr;   // [Nx * Ny], node j + Ny * i
    const float* w = nullptr;
    const float* wp = nullptr;
    float inv_dt = 0.0f;
    int iz = -1;
    float* ext = nullptr;
    const int2* pack = nullptr;
    int m = 0;
};

// Targets of one pressure deposit (deposit_pressure_open, acoustic_fdtd.cpp:840-872):
// divisor 0 = add the amplitude to idx[0]; divisor m > 0 = add amp/m to idx[0..n).
struct Deposit {
    int n;
    int divisor;
    long long idx[6];
};

// Status words (unsigned, 0xFFFFFFFF = none), reset with a 0xFF memset:
// first unstable cell of a check, first unstable plate node, first failing
// step latched by async stepping, and a fused-step CTA whose load wait ran out.
enum StatusSlot { kStatusCell = 0, kStatusPlate = 1, kStatusLatch = 2, kStatusTimeout = 3, kStatusWords = 4 };

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Face damping 1 - 0.5*(aL + aR)*dt (acoustic_fdtd.cpp:536-561).
__device__ __forceinline__ float face_damp(float aL, float aR, float dt)
{
    return fsub(1.0f, fmul(fmul(0.5f, fadd(aL, aR)), dt));
}

// One deposit of the open-cell rule (acoustic_fdtd.cpp:840-872); zero amplitude
// is a no-op, a solid cell splits amp/m over its m open face neighbours.
__device__ __forceinline__ void deposit_apply(const Deposit& d, float amp, float* p)
{
    if (amp == 0.0f || d.n == 0) return;
    if (d.divisor == 0) {
        p[d.idx[0]] = fadd(p[d.idx[0]], amp);
        return;
    }
    const float share = __fdiv_rn(amp, (float)d.divisor);
    for (int q = 0; q < d.n; ++q) p[d.idx[q]] = fadd(p[d.idx[q]], share);
}

// 8-tap precomputed sample (acoustic_fdtd.cpp:1673-1674): products in tap
// order, the first one starting the running sum.
__device__ __forceinline__ float sample8(const float* f, const long long* idx, const float* w)
{
    float s = fmul(w[0], f[idx[0]]);
    for (int t = 1; t < 8; ++t) s = fadd(s, fmul(w[t], f[idx[t]]));
    return s;
}

// ---- launchers (fdtd_general.cu) ----
cudaError_t launch_velocity_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* vx, float* vy, float* vz,
                                    const float* fx, const float* fy, const float* fz,
                                    cudaStream_t s, const unsigned* gate = nullptr,
                                    const PlateFaces* pf = nullptr);
// pressure update of listed four-cell groups (plate-face neighbours after a walled single-pass step)
cudaError_t launch_pressure_groups(const Grid& g, const Coef& cf, const Tables& tb, const float* p, float* pn,
                                   const float* vx, const float* vy, const float* vz, const float* fx,
                                   const float* fy, const float* fz, const uint8_t* solid,
                                   const long long* groups, int n_groups, cudaStream_t s);
cudaError_t launch_pressure_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* pn, const float* vx, const float* vy,
                                    const float* vz, const float* fx, const float* fy,
                                    const float* fz, const uint8_t* solid, cudaStream_t s,
                                    const unsigned* gate = nullptr);
cudaError_t launch_plate_step(int n_act, const int* act, const int* nb13, const long long* above,
                              const long long* below, const float* w, const float* wp, float* wt,
                              const float* ext, const float* p, const PlateCoef& pc,
                              unsigned* status, cudaStream_t s);
// plate forces as (node, value) pairs scattered into the zeroed device buffer
// (the velocity pass returns them to zero: PlateFaces)
cudaError_t launch_ext_scatter(float* ext, const int2* pack, int m, cudaStream_t s);
cudaError_t launch_plate_inject(int n_act, const int* act, const long long* vzb,
                                const long long* vza, const float* w, const float* wp,
                                float inv_dt, float* vz, cudaStream_t s,
                                const unsigned* gate = nullptr);
cudaError_t launch_deposit(const Deposit& d, const float* signal, int step, float amp, float* p,
                           cudaStream_t s);
cudaError_t launch_wsum(const float* f, const long long* idx, const float* w, int n_out, int taps,
                        int from_zero, float* out, cudaStream_t s);
cudaError_t launch_check(const Grid& g, const float* p, long long n_cells, int phase,
                         unsigned* status, int step, cudaStream_t s, const unsigned* gate = nullptr);
// Kernels given a gate (the handle's status words) do nothing once this step's
// plate update has recorded a failure in gate[kStatusPlate].
cudaError_t launch_zero_gated(float* x, int n, const unsigned* gate, cudaStream_t s);
cudaError_t launch_slice(const float* f, const Grid& g, int axis, int idx, float* out, int na, int nb,
                         cudaStream_t s);

// ---- fused single-pass step (fdtd_fused.cu) ----
// A slab of a room split along i: the local grid holds planes of the global
// room from xg0 on and the step computes the local planes [i_lo, i_lo+n_own);
// face existence and gradient order follow the global index.  nxg = 0 means
// the local grid is the whole room (all planes own).
struct XSpan {
    int xg0;     // global index of local plane 0
    int nxg;     // global Nx, or 0
    int i_lo;    // first own local plane
    int n_own;   // own planes
};

// Peer slabs' ghost planes written by the step itself (a slab of a split
// room): side 0 = the left neighbour, 1 = the right one.  pn/vx are the
// neighbour's next P buffer and next Vx set (null: no neighbour or no peer
// stores); local plane l of this slab is plane l + dl of the neighbour;
// planes [p_lo, p_hi) of the new P and faces [v_lo, v_hi) of the new Vx go
// there.  Memory may be another GPU's (peer access or IPC mapping).
struct XPeers {
    float* pn[2];
    float* vx[2];
    int dl[2];
    int p_lo[2], p_hi[2], v_lo[2], v_hi[2];
};

// Bounds of every mbarrier wait in the fused kernels: wall time (the
// %globaltimer clock) and, as a backstop, a poll count.
constexpr unsigned kWaitUs = 2000000u;   // 2 s; a load lands in microseconds
constexpr int kWaitPolls = 1 << 26;
// "no plane": plane indices of a march start at -3 (halo planes below i = 0)
constexpr int kNoPlane = -(1 << 30);

struct FusedArgs {
    Grid g;
    Coef cf;
    Tables tb;             // tb.ax / tb.px per local plane
    const float* p;        // P^n
    float* pn;             // P^{n+1}
    const float* vin[3];   // V^{n-1/2}: Vx, Vy, Vz
    float* vout[3];        // V^{n+1/2}
    unsigned* status;      // kStatusTimeout is set if a load wait runs out
    XSpan xs;              // zero: whole room
    XPeers pr;             // zero: no peer stores
    // Failure-path hook (fdtd_b200_debug_hold_load): the P load of this plane is
    // armed on its mbarrier but never issued, so its wait runs out after
    // wait_us microseconds and the kernel takes its timeout exit.
    int hold_plane = kNoPlane;
    unsigned wait_us = kWaitUs;
    // Fused point-source deposit (an open source cell): every CTA that loads
    // cell (dep_i, dep_j, dep_k) adds dep_sig[dep_step] to its shared-memory
    // copy of it when the plane arrives, so the step sees P^n plus the deposit
    // while P^n in HBM is left as it was.  dep_sig null: none.
    const float* dep_sig = nullptr;
    int dep_step = 0, dep_i = kNoPlane, dep_j = 0, dep_k = 0;
    // Fused receiver record of the input pressure (the previous step's
    // result): rec_out[r] = 8-tap sample of receiver r, spread over the CTAs.
    const long long* rec_idx = nullptr;
    const float* rec_w = nullptr;
    float* rec_out = nullptr;
    int n_rec = 0;
    // Walled scenes (whole rooms only): open fractions of the Vx, Vy, Vz faces
    // (null: none; a face with fraction 0 is closed), whether the divergence
    // scales each face by its fraction, and the solid-cell mask (null: none).
    const float* fr[3] = {nullptr, nullptr, nullptr};
    bool frac_div = false;
    const uint8_t* solid = nullptr;
};
struct FusedCache;         // host-side TMA descriptors of a handle's fields
FusedCache* fused_cache_create();
void fused_cache_destroy(FusedCache* c);
bool fused_supported(const Grid& g);
cudaError_t launch_fused_step(const FusedArgs& a, FusedCache* cache, cudaStream_t s);
int fused_kernel_launches_per_step();
// TMA descriptors of the four fields a fused step reads (P, Vx, Vy, Vz).
cudaError_t fused_maps(FusedCache* c, const Grid& g, const float* p, const float* const* v,
                       CUtensorMap out[4], int shape = 0);

// ---- batched step (continuous batching of independent rooms) ----
// Device-resident descriptor of one batch member.  Parity 0 is the member's
// state when it joined the batch; a step taken at parity q reads p[q], v[q]
// and writes p[q^1], v[q^1].
struct alignas(64) BatchMember {
    CUtensorMap maps[2][4];      // per parity: P, Vx, Vy, Vz read by the step
    Grid g;
    Coef cf;
    Tables tb;
    float* p[2];
    float* v[2][3];
    int step;                    // device step counter (advanced by the epilogue)
    int step0, limit;            // step count on joining; stop at this step count
    int items_begin, tiles, tiles_k, seg_len;
    // point source
    Deposit ps;
    const float* ps_sig;
    int ps_n;
    // receivers
    int n_rec, trace0, trace_cap;
    const long long* rec_idx;
    const float* rec_w;
    float* trace;
    // stability check
    int n_cells, phase0;
    unsigned unstable;           // first step whose check failed (0xFFFFFFFF = none)
};
// Tile geometry of the fused step: rows x columns of a tile.
void fused_tile_shape(int shape, int* tj, int* tk);   // shape 0: 8 x 128 tiles, 1: 16 x 64
// Resident CTAs of the batched kernel on the current device (all SMs).
cudaError_t fused_batch_slots(int shape, int* slots);
// Sizes of the current member set, read by the kernels from device memory so
// that a captured graph stays valid when the set changes.
struct BatchHeader {
    int n_members;
    int total_items;
    int counter;                 // work-item counter, reset before each step
};
// One batched step: every member below its limit advances one step (fused
// velocity+pressure over item_member's work items, then the epilogue:
// receivers, step counter, 256-step check, next source sample).  epi_blocks
// is the member capacity (blocks beyond n_members exit at once).
cudaError_t launch_fused_batch_step(BatchMember* members, BatchHeader* hdr, const int* item_member,
                                    unsigned* status, int grid_ctas, int epi_blocks, cudaStream_t s, int shape = 0);

}  // namespace fdtd
