// fdtd_prec_internal.h — storage modes of the precision study: the stored
// types, their exact encode/decode and the coefficient block, shared by the
// two-pass kernels (fdtd_precision.cu) and the single-pass 16-bit step
// (fdtd_fused16.cu).
#pragma once

#include "fdtd_internal.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace fdtd {
namespace prec {

enum Mode { kFP32 = 0, kFP64 = 1, kBF16 = 2, kFP16 = 3, kBF16C = 4, kFP16C = 5 };

// exactly rounded ops in both arithmetic types
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }

template <int M> struct Traits;
template <> struct Traits<kFP32> { using A = float; using S = float; static constexpr bool comp = false; };
template <> struct Traits<kFP64> { using A = double; using S = double; static constexpr bool comp = false; };
template <> struct Traits<kBF16> { using A = float; using S = __nv_bfloat16; static constexpr bool comp = false; };
template <> struct Traits<kFP16> { using A = float; using S = __half; static constexpr bool comp = false; };
template <> struct Traits<kBF16C> { using A = float; using S = __nv_bfloat16; static constexpr bool comp = true; };
template <> struct Traits<kFP16C> { using A = float; using S = __half; static constexpr bool comp = true; };

__device__ __forceinline__ float tofl(float v) { return v; }
__device__ __forceinline__ double tofl(double v) { return v; }
__device__ __forceinline__ float tofl(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float tofl(__half v) { return __half2float(v); }
template <class S> __device__ __forceinline__ S fromfl(float v);
template <> __device__ __forceinline__ float fromfl<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 fromfl<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half fromfl<__half>(float v) { return __float2half_rn(v); }

// One stored field: value array, optional residual array, power-of-two scale.
struct Field {
    void* hi;
    void* lo;
    float scale, inv_scale;        // stored value = x * scale
    float lo_scale, inv_lo_scale;  // stored residual = (x*scale - hi) * lo_scale
};

template <int M>
__device__ __forceinline__ typename Traits<M>::A ld(const Field& f, long long i)
{
    using T = Traits<M>;
    using S = typename T::S;
    if constexpr (M == kFP32 || M == kFP64) {
        return static_cast<const S*>(f.hi)[i];
    } else {
        float v = tofl(static_cast<const S*>(f.hi)[i]);
        if constexpr (T::comp)
            v = __fadd_rn(v, __fmul_rn(tofl(static_cast<const S*>(f.lo)[i]), f.inv_lo_scale));
        return __fmul_rn(v, f.inv_scale);
    }
}

template <int M>
__device__ __forceinline__ void st(const Field& f, long long i, typename Traits<M>::A x)
{
    using T = Traits<M>;
    using S = typename T::S;
    if constexpr (M == kFP32 || M == kFP64) {
        static_cast<S*>(f.hi)[i] = x;
    } else {
        const float xs = __fmul_rn(x, f.scale);
        const S h = fromfl<S>(xs);
        static_cast<S*>(f.hi)[i] = h;
        if constexpr (T::comp)
            static_cast<S*>(f.lo)[i] = fromfl<S>(__fmul_rn(__fsub_rn(xs, tofl(h)), f.lo_scale));
    }
}

template <class A>
struct PCoef {
    A vc, bulk, dt, c1, c2;
    const A *ax, *ay, *az, *px, *py, *pz;
};

template <class A>
__device__ __forceinline__ A fdamp(A aL, A aR, A dt)
{
    return rsub(A(1), rmul(rmul(A(0.5), radd(aL, aR)), dt));
}

template <class A>
__device__ __forceinline__ A amax(A a, A b) { return a > b ? a : b; }
template <class A>
__device__ __forceinline__ A amin(A a, A b) { return a < b ? a : b; }

// Four consecutive values (index i a multiple of 4, so the access is aligned:
// rows start on 8-element boundaries).  Each value is decoded exactly as ld().
template <int M>
__device__ __forceinline__ void ld4(const Field& f, long long i, typename Traits<M>::A (&v)[4])
{
    using T = Traits<M>;
    using S = typename T::S;
    if constexpr (M == kFP32) {
        const float4 x = *reinterpret_cast<const float4*>(static_cast<const float*>(f.hi) + i);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else if constexpr (M == kFP64) {
        const double2 x = *reinterpret_cast<const double2*>(static_cast<const double*>(f.hi) + i);
        const double2 y = *reinterpret_cast<const double2*>(static_cast<const double*>(f.hi) + i + 2);
        v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
    } else {
        union { uint2 u; S s[4]; } h, l;
        h.u = *reinterpret_cast<const uint2*>(static_cast<const S*>(f.hi) + i);
        if constexpr (T::comp) l.u = *reinterpret_cast<const uint2*>(static_cast<const S*>(f.lo) + i);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float x = tofl(h.s[q]);
            if constexpr (T::comp) x = __fadd_rn(x, __fmul_rn(tofl(l.s[q]), f.inv_lo_scale));
            v[q] = __fmul_rn(x, f.inv_scale);
        }
    }
}

// Four consecutive values, each encoded exactly as st().
template <int M>
__device__ __forceinline__ void st4(const Field& f, long long i, const typename Traits<M>::A (&v)[4])
{
    using T = Traits<M>;
    using S = typename T::S;
    if constexpr (M == kFP32) {
        *reinterpret_cast<float4*>(static_cast<float*>(f.hi) + i) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (M == kFP64) {
        *reinterpret_cast<double2*>(static_cast<double*>(f.hi) + i) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(static_cast<double*>(f.hi) + i + 2) = make_double2(v[2], v[3]);
    } else {
        union { uint2 u; S s[4]; } h, l;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float xs = __fmul_rn(v[q], f.scale);
            h.s[q] = fromfl<S>(xs);
            if constexpr (T::comp) l.s[q] = fromfl<S>(__fmul_rn(__fsub_rn(xs, tofl(h.s[q])), f.lo_scale));
        }
        *reinterpret_cast<uint2*>(static_cast<S*>(f.hi) + i) = h.u;
        if constexpr (T::comp) *reinterpret_cast<uint2*>(static_cast<S*>(f.lo) + i) = l.u;
    }
}

// ---- single-pass step of the 16-bit storage modes (fdtd_fused16.cu) ----
struct Sc {
    float s, is;       // stored value = x * s;  x = stored * is
    float ls, ils;     // residual scale and its inverse (compensated forms)
};

struct F16Args {
    Grid g;
    PCoef<float> cf;               // coefficients and device axis tables
    const void* p_hi;              // P^n (value, residual)
    const void* p_lo;
    void* pn_hi;                   // P^{n+1}
    void* pn_lo;
    void* vout_hi[3];              // V^{n+1/2}: Vx, Vy, Vz
    void* vout_lo[3];
    Sc sp, sv;                     // pressure and velocity scales
    float dep_amp;                 // this step's source sample (0: none) at (dep_i, dep_j, dep_k)
    int dep_i, dep_j, dep_k;
    int n_rec;                     // receivers of the input P (the previous step's), rec_out null: none
    const long long* rec_idx;
    const double* rec_w;
    double* rec_out;
    unsigned* status;              // kStatusTimeout is set when a load wait runs out
    unsigned wait_us;
    int xi_lo, xi_hi;              // planes [xi_lo, xi_hi) have alpha_x = 0 (empty: none)
};

struct F16Cache;                   // host-side tensor maps of a handle's 16-bit fields
F16Cache* f16_cache_create();
void f16_cache_destroy(F16Cache* c);
cudaError_t f16_map(F16Cache* c, const void* base, const Grid& g, int bx, int by, CUtensorMap* out);
bool f16_supported(int mode, const Grid& g);
size_t f16_smem_bytes(int mode);
// bases: P^n value, P^n residual, then V^{n-1/2} value / residual of Vx, Vy, Vz
// (residuals null for the plain 16-bit modes)
cudaError_t launch_fused16(int mode, const F16Args& a, F16Cache* cache, const void* const bases[8],
                           cudaStream_t s);

}  // namespace prec
}  // namespace fdtd
