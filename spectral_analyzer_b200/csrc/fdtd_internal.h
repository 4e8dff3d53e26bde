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
#include <cuda_runtime.h>
#include <stdint.h>

namespace fdtd {

constexpr int kRowAlign = 8;           // floats per row-padding unit (32 B)
constexpr int kCheckStride = 1013;     // stability sample stride (acoustic_fdtd.cpp:1250)
constexpr int kCheckPeriod = 256;      // steps between checks (acoustic_fdtd.cpp:1284)

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
};

struct PlateCoef {
    float a;    // dt^2 / (rho_s h)
    float bh;   // D dt^2 / (rho_s h dx^4)
    float vd;   // 1 - alpha_M dt
    float bk;   // beta_K / dt * bh
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

// ---- launchers (fdtd_general.cu) ----
cudaError_t launch_velocity_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* vx, float* vy, float* vz,
                                    const float* fx, const float* fy, const float* fz,
                                    cudaStream_t s);
cudaError_t launch_pressure_general(const Grid& g, const Coef& cf, const Tables& tb,
                                    const float* p, float* pn, const float* vx, const float* vy,
                                    const float* vz, const float* fx, const float* fy,
                                    const float* fz, const uint8_t* solid, cudaStream_t s);
cudaError_t launch_plate_step(int n_act, const int* act, const int* nb13, const long long* above,
                              const long long* below, const float* w, const float* wp, float* wt,
                              const float* ext, const float* p, const PlateCoef& pc,
                              unsigned* status, cudaStream_t s);
cudaError_t launch_plate_inject(int n_act, const int* act, const long long* vzb,
                                const long long* vza, const float* w, const float* wp,
                                float inv_dt, float* vz, cudaStream_t s);
cudaError_t launch_deposit(const Deposit& d, const float* signal, int step, float amp, float* p,
                           cudaStream_t s);
cudaError_t launch_wsum(const float* f, const long long* idx, const float* w, int n_out, int taps,
                        int from_zero, float* out, cudaStream_t s);
cudaError_t launch_check(const Grid& g, const float* p, long long n_cells, int phase,
                         unsigned* status, int step, cudaStream_t s);

// ---- fused single-pass step (fdtd_fused.cu) ----
struct FusedArgs {
    Grid g;
    Coef cf;
    Tables tb;
    const float* p;        // P^n
    float* pn;             // P^{n+1}
    const float* vin[3];   // V^{n-1/2}: Vx, Vy, Vz
    float* vout[3];        // V^{n+1/2}
    unsigned* status;      // kStatusTimeout is set if a load wait runs out
};
struct FusedCache;         // host-side TMA descriptors of a handle's fields
FusedCache* fused_cache_create();
void fused_cache_destroy(FusedCache* c);
bool fused_supported(const Grid& g);
cudaError_t launch_fused_step(const FusedArgs& a, FusedCache* cache, cudaStream_t s);
int fused_kernel_launches_per_step();

}  // namespace fdtd
