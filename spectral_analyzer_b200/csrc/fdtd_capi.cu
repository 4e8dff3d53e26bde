/*
 * fdtd_capi.cu — the C ABI (include/acoustic_fdtd_b200.h) over the CUDA kernels.
 *
 * Host-side work mirrors the reference's fdtd_* functions
 * (csrc/kernels/acoustic_fdtd.cpp, cited per function): create-time setup,
 * sampler index arithmetic and force accumulation are done on the host in
 * float with the reference's operation order; the per-step work runs on the
 * device.  The device layout is described in fdtd_internal.h.
 */
#include "acoustic_fdtd_b200.h"
#include "fdtd_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

using namespace fdtd;

namespace {

std::mutex g_err_mu;
char g_err[512] = "";

void set_err(cudaError_t e, const char* what)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    snprintf(g_err, sizeof(g_err), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
}

}  // namespace

void fdtd::record_cuda_error(cudaError_t e, const char* what) { set_err(e, what); }

namespace {

#define CK(expr)                                   \
    do {                                           \
        cudaError_t e_ = (expr);                   \
        if (e_ != cudaSuccess) {                   \
            set_err(e_, #expr);                    \
            return FDTD_ERR_CUDA;                  \
        }                                          \
    } while (0)

inline bool is_solid(uint8_t c) { return c == FDTD_WALL || c == FDTD_PLATE; }

// pml_sigma with sigma_max scaled per face (acoustic_fdtd.cpp:216-222).
float scaled_sigma(int d, int n_pml, float dt, float scale)
{
    if (n_pml <= 0 || d <= 0) return 0.0f;
    float frac = (float)d / (float)n_pml;
    float sigma_max = scale * (3.45f / (dt * (float)n_pml));
    return sigma_max * frac * frac * frac;
}

// alpha along one axis: low face first, as acoustic_fdtd.cpp:381-383 selects depth.
float axis_alpha(int i, int n, int n_pml, float dt, float a_lo, float a_hi)
{
    if (i < n_pml) return scaled_sigma(n_pml - i, n_pml, dt, a_lo);
    if (i >= n - n_pml) return scaled_sigma(i - (n - n_pml) + 1, n_pml, dt, a_hi);
    return 0.0f;
}

struct ProfEvents {
    std::vector<cudaEvent_t> ev;   // pairs
    int used = 0;
};

}  // namespace

// Everything a co-evolver substep's device work depends on besides memory
// contents: buffer pointers, coefficients, flags.  A substep whose key equals a
// cached one replays that graph (compared byte for byte; zero-filled first).
struct SubstepKey {
    cudaStream_t stream;
    const float *p, *pn, *v0, *v1, *v2, *w_cur, *w_prev, *w_tmp, *frac[3], *ext, *h_ext;
    const int2 *pack, *h_pack;
    const uint8_t* solid;
    const long long *sidx;
    const float *sw;
    float *sout, *h_sout;
    unsigned *status, *h_status;
    Grid g;
    Coef cf;
    Tables tb;
    PlateCoef pc;
    int n_act, n_plate, n_saddle, ext_copy, ext_zero, has_frac, n_pack;
};

struct SubstepGraph {
    SubstepKey key;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
};

struct AcousticFDTDState {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;

    Grid g{};
    int Nx = 0, Ny = 0, Nz = 0, N = 0, N_plate = 0, plate_iz = 0, n_pml = 0;
    float dx = 0, c = 0, rho = 0, dt = 0;
    Coef cf{};
    PlateCoef pc{};
    std::vector<SubstepGraph> sgraphs;   // cached substep graphs (at most kSubstepGraphs)
    float a6[6] = {1, 1, 1, 1, 1, 1};

    float* p[2] = {nullptr, nullptr};
    int cur = 0;
    float* v[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int cv = 0;                      // current velocity set; the fused step writes the other
    bool own_fields = true;
    size_t field_bytes = 0;

    float* d_tab = nullptr;   // ax | ay | az | px | py | pz
    Tables tb{};

    std::vector<uint8_t> cell_type;      // after PML marking and plate enforcement
    std::vector<uint8_t> plate_active;
    bool any_solid = false;
    uint8_t* d_solid = nullptr;
    std::vector<float> frac[3];          // reference layouts, built on first need
    float* d_frac[3] = {nullptr, nullptr, nullptr};
    bool has_frac = false;

    // plate
    int n_act = 0;
    int* d_act = nullptr;
    int* d_nb13 = nullptr;
    long long* d_above = nullptr;
    long long* d_below = nullptr;
    long long* d_vzb = nullptr;
    long long* d_vza = nullptr;
    uint8_t* d_plate_code = nullptr;   // per plate node: bit 0 Vz face below, bit 1 above (PlateFaces)
    // four-cell groups whose divergence reads a plate face (padded index of the
    // group's first cell): recomputed after a walled single-pass step
    long long* d_pfix = nullptr;
    int n_pfix = 0;
    std::vector<int> h_act;
    float* d_w[3] = {nullptr, nullptr, nullptr};
    int wi_cur = 0, wi_prev = 1, wi_tmp = 2;
    float* d_ext = nullptr;
    float* d_slice = nullptr;        // fdtd_b200_get_volume_slice staging, largest plane
    float* h_ext = nullptr;          // pinned, N_plate: forces pending for the next step
    bool ext_pending = false;
    bool dev_ext_nonzero = false;
    // plate nodes holding a pending force, each once, and their (node, value)
    // pairs as the substep sends them (pinned) and as the device receives them
    std::vector<int> ext_nodes;
    std::vector<uint8_t> ext_mark;
    int2* h_ext_pack = nullptr;
    int2* d_ext_pack = nullptr;

    std::vector<int> src_idx;
    std::vector<float> src_wgt;

    // point source
    Deposit ps{};
    float* d_ps_sig = nullptr;
    int ps_n = 0;
    int ps_cell = -1;
    int ps_done_step = -1;           // step whose source sample is already in P
    int rec_pending = -1;            // trace slot the next fused step (or flush_record) records

    // receivers
    int n_rec = 0;
    long long* d_rec_idx = nullptr;
    float* d_rec_w = nullptr;
    float* d_trace = nullptr;
    int trace_cap = 0;
    int trace_len = 0;

    unsigned* d_status = nullptr;
    unsigned* h_status = nullptr;    // pinned
    int step_count = 0;
    int stab_phase = 0;

    int kernel_mode = 0;
    int hold_plane = kNoPlane;       // fdtd_b200_debug_hold_load
    unsigned wait_us = kWaitUs;
    FusedCache* fcache = nullptr;    // TMA descriptors of the fields (fused step)

    long long launches = 0;          // kernels launched by this handle

    bool prof_on = false;
    ProfEvents prof;
    long long prof_launches = 0;     // main-kernel launch groups timed
    long long prof_kernels = 0;      // individual kernel launches in those groups

    // sampling scratch
    size_t s_cap = 0;
    long long* d_sidx = nullptr;
    float* d_sw = nullptr;
    float* d_sout = nullptr;
    long long* h_sidx = nullptr;
    float* h_sw = nullptr;
    float* h_sout = nullptr;
    // sampler results written by the kernel straight into pinned host memory
    // (mapped into the device's address space): no device-to-host copy per call
    float* h_sout_map = nullptr;
    float* d_sout_map = nullptr;
    // what d_sidx / d_sw hold (upload_taps skips a copy of the same taps)
    std::vector<long long> up_idx;
    std::vector<float> up_w;

    long long pad(int i, int j, int k) const { return ((long long)i * Ny + j) * g.sz + k; }
    float* P() const { return p[cur]; }
    float* Pn() const { return p[cur ^ 1]; }
    float* V(int c) const { return v[cv][c]; }
};

namespace {

int dev_guard(const AcousticFDTDState* st)
{
    int d = -1;
    cudaGetDevice(&d);
    if (d != st->device) CK(cudaSetDevice(st->device));
    return FDTD_OK;
}

int build_tables(AcousticFDTDState* st)
{
    const int nx = st->Nx, ny = st->Ny, nz = st->Nz;
    std::vector<float> h((size_t)2 * (nx + ny + nz));
    float* ax = h.data();
    float* ay = ax + nx;
    float* az = ay + ny;
    float* px = az + nz;   // px | py | pz follow the alphas in the same order
    const float dt = st->dt;
    for (int i = 0; i < nx; ++i) ax[i] = axis_alpha(i, nx, st->n_pml, dt, st->a6[0], st->a6[1]);
    for (int j = 0; j < ny; ++j) ay[j] = axis_alpha(j, ny, st->n_pml, dt, st->a6[2], st->a6[3]);
    for (int k = 0; k < nz; ++k) az[k] = axis_alpha(k, nz, st->n_pml, dt, st->a6[4], st->a6[5]);
    // P damping 1/(1 + alpha*dt) (acoustic_fdtd.cpp:469-476) per axis; a cell's is the
    // minimum over its axes because the map alpha -> damping is monotone.
    for (int q = 0; q < nx + ny + nz; ++q) {
        float denom = 1.0f + ax[q] * dt;
        px[q] = 1.0f / denom;
    }
    x_interior_run(ax, nx, &st->tb.xi_lo, &st->tb.xi_hi);
    CK(cudaMemcpyAsync(st->d_tab, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice,
                       st->stream));
    CK(cudaStreamSynchronize(st->stream));
    return FDTD_OK;
}

// Default face fractions (acoustic_fdtd.cpp:492-534): 0 beside a solid cell,
// else 1; the Vz faces on either side of the plate layer stay 1.
void default_fracs(AcousticFDTDState* st)
{
    const int nx = st->Nx, ny = st->Ny, nz = st->Nz, piz = st->plate_iz;
    const uint8_t* ct = st->cell_type.data();
    auto sol = [&](int i, int j, int k) { return is_solid(ct[k + nz * (j + ny * i)]); };
    st->frac[0].assign((size_t)(nx - 1) * ny * nz, 1.0f);
    st->frac[1].assign((size_t)nx * (ny - 1) * nz, 1.0f);
    st->frac[2].assign((size_t)nx * ny * (nz - 1), 1.0f);
    for (int i = 0; i < nx - 1; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                st->frac[0][k + nz * (j + ny * i)] = (sol(i, j, k) || sol(i + 1, j, k)) ? 0.0f : 1.0f;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
                st->frac[1][k + nz * (j + (ny - 1) * i)] =
                    (sol(i, j, k) || sol(i, j + 1, k)) ? 0.0f : 1.0f;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz - 1; ++k) {
                float f;
                if (k == piz - 1 || k == piz) f = 1.0f;
                else f = (sol(i, j, k) || sol(i, j, k + 1)) ? 0.0f : 1.0f;
                st->frac[2][k + (nz - 1) * (j + ny * i)] = f;
            }
}

// Copies a compact [nxa][nya][nza] host block into a padded device field (or back).
int copy_block(AcousticFDTDState* st, float* dfield, float* host, int nxa, int nya, int nza,
               bool to_device)
{
    if (nxa <= 0 || nya <= 0 || nza <= 0) return FDTD_OK;
    cudaMemcpy3DParms prm = {};
    cudaPitchedPtr dev = make_cudaPitchedPtr(dfield, (size_t)st->g.sz * sizeof(float), st->g.sz, st->Ny);
    cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)nza * sizeof(float), nza, nya);
    prm.extent = make_cudaExtent((size_t)nza * sizeof(float), nya, nxa);
    if (to_device) {
        prm.srcPtr = hp;
        prm.dstPtr = dev;
        prm.kind = cudaMemcpyHostToDevice;
    } else {
        prm.srcPtr = dev;
        prm.dstPtr = hp;
        prm.kind = cudaMemcpyDeviceToHost;
    }
    CK(cudaMemcpy3DAsync(&prm, st->stream));
    CK(cudaStreamSynchronize(st->stream));
    return FDTD_OK;
}

int upload_fracs(AcousticFDTDState* st)
{
    for (int c = 0; c < 3; ++c)
        if (!st->d_frac[c]) {
            CK(cudaMalloc(&st->d_frac[c], st->field_bytes));
            CK(cudaMemsetAsync(st->d_frac[c], 0, st->field_bytes, st->stream));
        }
    int rc;
    if ((rc = copy_block(st, st->d_frac[0], st->frac[0].data(), st->Nx - 1, st->Ny, st->Nz, true))) return rc;
    if ((rc = copy_block(st, st->d_frac[1], st->frac[1].data(), st->Nx, st->Ny - 1, st->Nz, true))) return rc;
    if ((rc = copy_block(st, st->d_frac[2], st->frac[2].data(), st->Nx, st->Ny, st->Nz - 1, true))) return rc;
    return FDTD_OK;
}

// Open-cell deposit targets of flat cell `idx` (acoustic_fdtd.cpp:840-872).
Deposit make_deposit(const AcousticFDTDState* st, int idx)
{
    Deposit d{};
    if (idx < 0 || idx >= st->N) return d;
    const int nz = st->Nz, ny = st->Ny, nx = st->Nx;
    const uint8_t* ct = st->cell_type.data();
    int k = idx % nz, t = idx / nz, j = t % ny, i = t / ny;
    if (!is_solid(ct[idx])) {
        d.n = 1;
        d.divisor = 0;
        d.idx[0] = st->pad(i, j, k);
        return d;
    }
    int nb[6][3];
    int m = 0;
    if (i + 1 < nx) { nb[m][0] = i + 1; nb[m][1] = j; nb[m][2] = k; ++m; }
    if (i - 1 >= 0) { nb[m][0] = i - 1; nb[m][1] = j; nb[m][2] = k; ++m; }
    if (j + 1 < ny) { nb[m][0] = i; nb[m][1] = j + 1; nb[m][2] = k; ++m; }
    if (j - 1 >= 0) { nb[m][0] = i; nb[m][1] = j - 1; nb[m][2] = k; ++m; }
    if (k + 1 < nz) { nb[m][0] = i; nb[m][1] = j; nb[m][2] = k + 1; ++m; }
    if (k - 1 >= 0) { nb[m][0] = i; nb[m][1] = j; nb[m][2] = k - 1; ++m; }
    for (int q = 0; q < m; ++q)
        if (!is_solid(ct[nb[q][2] + nz * (nb[q][1] + ny * nb[q][0])]))
            d.idx[d.n++] = st->pad(nb[q][0], nb[q][1], nb[q][2]);
    d.divisor = d.n;   // share = amp / open_count
    return d;
}

int ensure_scratch(AcousticFDTDState* st, size_t n)
{
    if (n <= st->s_cap) return FDTD_OK;
    size_t cap = std::max<size_t>(n, 1024);
    cudaFree(st->d_sidx); cudaFree(st->d_sw); cudaFree(st->d_sout);
    cudaFreeHost(st->h_sidx); cudaFreeHost(st->h_sw); cudaFreeHost(st->h_sout); cudaFreeHost(st->h_sout_map);
    st->d_sidx = nullptr; st->d_sw = st->d_sout = nullptr;
    st->h_sidx = nullptr; st->h_sw = st->h_sout = nullptr;
    st->h_sout_map = st->d_sout_map = nullptr;
    st->s_cap = 0;
    st->up_idx.clear();
    st->up_w.clear();
    CK(cudaMalloc(&st->d_sidx, cap * sizeof(long long)));
    CK(cudaMalloc(&st->d_sw, cap * sizeof(float)));
    CK(cudaMalloc(&st->d_sout, cap * sizeof(float)));
    CK(cudaMallocHost(&st->h_sidx, cap * sizeof(long long)));
    CK(cudaMallocHost(&st->h_sw, cap * sizeof(float)));
    CK(cudaMallocHost(&st->h_sout, cap * sizeof(float)));
    CK(cudaHostAlloc(&st->h_sout_map, cap * sizeof(float), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void**)&st->d_sout_map, st->h_sout_map, 0));
    st->s_cap = cap;
    return FDTD_OK;
}

// Copies the n taps staged in h_sidx / h_sw to the device unless it already
// holds exactly these (a caller sampling the same receivers every step).
int upload_taps(AcousticFDTDState* st, size_t n, cudaStream_t s)
{
    if (n == 0) return FDTD_OK;
    if (st->up_idx.size() == n && memcmp(st->up_idx.data(), st->h_sidx, n * sizeof(long long)) == 0 &&
        memcmp(st->up_w.data(), st->h_sw, n * sizeof(float)) == 0)
        return FDTD_OK;
    st->up_idx.clear();
    st->up_w.clear();
    CK(cudaMemcpyAsync(st->d_sidx, st->h_sidx, n * sizeof(long long), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st->d_sw, st->h_sw, n * sizeof(float), cudaMemcpyHostToDevice, s));
    st->up_idx.assign(st->h_sidx, st->h_sidx + n);
    st->up_w.assign(st->h_sw, st->h_sw + n);
    return FDTD_OK;
}

// Weighted gathers already staged in h_sidx / h_sw (n_out * taps entries):
// runs k_wsum on `field` and copies n_out results to `out`.
int run_wsum(AcousticFDTDState* st, const float* field, int n_out, int taps, int from_zero,
             float* out)
{
    if (n_out <= 0) return FDTD_OK;
    const size_t n = (size_t)n_out * taps;
    if (int rc = upload_taps(st, n, st->stream)) return rc;
    CK(launch_wsum(field, st->d_sidx, st->d_sw, n_out, taps, from_zero, st->d_sout_map, st->stream));
    ++st->launches;
    CK(cudaStreamSynchronize(st->stream));
    memcpy(out, st->h_sout_map, (size_t)n_out * sizeof(float));
    return FDTD_OK;
}

// Field selector for index conversion: 0 P, 1 Vx, 2 Vy, 3 Vz.
struct FieldShape { int nxa, nya, nza; };

FieldShape field_shape(const AcousticFDTDState* st, int f)
{
    return {st->Nx - (f == 1), st->Ny - (f == 2), st->Nz - (f == 3)};
}

// Reference flat index of field f -> padded device index; -1 when out of range.
long long ref_to_pad(const AcousticFDTDState* st, int f, long long flat)
{
    FieldShape s = field_shape(st, f);
    long long len = (long long)s.nxa * s.nya * s.nza;
    if (flat < 0 || flat >= len) return -1;
    int k = (int)(flat % s.nza);
    long long t = flat / s.nza;
    int j = (int)(t % s.nya);
    int i = (int)(t / s.nya);
    return st->pad(i, j, k);
}

const float* field_ptr(const AcousticFDTDState* st, int f)
{
    return f == 0 ? st->P() : st->V(f - 1);
}

// Trilinear taps of the reference samplers (acoustic_fdtd.cpp:1355-1395,
// :1404-1538, :1567-1661).  f = 0 pressure, 1..3 = Vx, Vy, Vz with the
// half-cell shift on their own axis.  Indices are the field's reference flat
// indices; a NaN coordinate is mapped to 0 (the reference would read out of range).
void sampler_taps(const AcousticFDTDState* st, int f, const float* xyz, int* id8, float* w8)
{
    FieldShape s = field_shape(st, f);
    float gx = xyz[0] - (f == 1 ? 0.5f : 0.0f);
    float gy = xyz[1] - (f == 2 ? 0.5f : 0.0f);
    float gz = xyz[2] - (f == 3 ? 0.5f : 0.0f);
    if (gx < 0.0f) gx = 0.0f;
    if (gx > (float)(s.nxa - 1)) gx = (float)(s.nxa - 1);
    if (gy < 0.0f) gy = 0.0f;
    if (gy > (float)(s.nya - 1)) gy = (float)(s.nya - 1);
    if (gz < 0.0f) gz = 0.0f;
    if (gz > (float)(s.nza - 1)) gz = (float)(s.nza - 1);
    if (gx != gx) gx = 0.0f;
    if (gy != gy) gy = 0.0f;
    if (gz != gz) gz = 0.0f;
    int i0 = (int)gx, i1 = (i0 < s.nxa - 1) ? i0 + 1 : i0;
    int j0 = (int)gy, j1 = (j0 < s.nya - 1) ? j0 + 1 : j0;
    int k0 = (int)gz, k1 = (k0 < s.nza - 1) ? k0 + 1 : k0;
    float fx = gx - (float)i0, fy = gy - (float)j0, fz = gz - (float)k0;
    auto FI = [&](int a, int b, int c) { return c + s.nza * (b + s.nya * a); };
    id8[0] = FI(i0, j0, k0); w8[0] = (1 - fx) * (1 - fy) * (1 - fz);
    id8[1] = FI(i1, j0, k0); w8[1] = (fx) * (1 - fy) * (1 - fz);
    id8[2] = FI(i0, j1, k0); w8[2] = (1 - fx) * (fy) * (1 - fz);
    id8[3] = FI(i1, j1, k0); w8[3] = (fx) * (fy) * (1 - fz);
    id8[4] = FI(i0, j0, k1); w8[4] = (1 - fx) * (1 - fy) * (fz);
    id8[5] = FI(i1, j0, k1); w8[5] = (fx) * (1 - fy) * (fz);
    id8[6] = FI(i0, j1, k1); w8[6] = (1 - fx) * (fy) * (fz);
    id8[7] = FI(i1, j1, k1); w8[7] = (fx) * (fy) * (fz);
}

// Stages n samplers of field f (8 taps each, reference indices) into h_sidx/h_sw.
int stage_taps(AcousticFDTDState* st, int f, int n, const int* idx8, const float* wgt8)
{
    int rc = ensure_scratch(st, (size_t)n * 8);
    if (rc) return rc;
    for (long long q = 0; q < (long long)n * 8; ++q) {
        long long pi = ref_to_pad(st, f, idx8[q]);
        if (pi < 0) return FDTD_ERR_ARG;
        st->h_sidx[q] = pi;
        st->h_sw[q] = wgt8[q];
    }
    return FDTD_OK;
}

int direct_samples(AcousticFDTDState* st, int f, int n, const float* xyz, float* out)
{
    int rc = ensure_scratch(st, (size_t)n * 8);
    if (rc) return rc;
    for (int r = 0; r < n; ++r) {
        int id8[8];
        float w8[8];
        sampler_taps(st, f, xyz + 3 * r, id8, w8);
        for (int t = 0; t < 8; ++t) {
            st->h_sidx[8 * r + t] = ref_to_pad(st, f, id8[t]);
            st->h_sw[8 * r + t] = w8[t];
        }
    }
    return run_wsum(st, field_ptr(st, f), n, 8, 1, out);
}

bool fused_eligible(const AcousticFDTDState* st)
{
    return !st->any_solid && !st->has_frac && !st->d_frac[0] && st->n_act == 0 &&
           fused_supported(st->g);
}

// A walled scene (solid cells, face fractions or an active plate) that the
// single-pass step can take: whole room, row padding as the TMA maps need.
bool fused_walled_ok(const AcousticFDTDState* st)
{
    return (st->any_solid || st->d_frac[0] || st->n_act > 0) && fused_supported(st->g);
}

// Walled scenes take the single pass automatically from this many cells on:
// below it the fields stay in L2 and the two-pass kernels are faster (step
// kernels per step, two-pass / single pass: 170x140x74 40 / 67 us,
// 160x128x128 50 / 60; above it 256x200x128 120 / 106, 400x300x256 511 / 430,
// 512x384x256 827 / 558).
constexpr long long kWalledFusedCells = 1LL << 22;

bool use_fused(const AcousticFDTDState* st)
{
    if (st->kernel_mode == 1) return false;
    if (fused_eligible(st)) return true;
    if (!fused_walled_ok(st)) return false;
    return st->kernel_mode == 2 || (long long)st->N >= kWalledFusedCells;
}

int prof_begin(AcousticFDTDState* st, cudaEvent_t* e1)
{
    *e1 = nullptr;
    if (!st->prof_on) return FDTD_OK;
    if (st->prof.used + 2 > (int)st->prof.ev.size()) return FDTD_OK;
    *e1 = st->prof.ev[st->prof.used];
    CK(cudaEventRecord(*e1, st->stream));
    return FDTD_OK;
}

int prof_end(AcousticFDTDState* st, cudaEvent_t e1, int kernels)
{
    if (!st->prof_on || !e1) return FDTD_OK;
    CK(cudaEventRecord(st->prof.ev[st->prof.used + 1], st->stream));
    st->prof.used += 2;
    st->prof_launches += 1;
    st->prof_kernels += kernels;
    return FDTD_OK;
}

// A fused-step CTA whose bounded load wait ran out leaves its blocks' results
// incomplete: reported as a CUDA-level failure (status read from h_status).
int check_timeout(AcousticFDTDState* st)
{
    if (st->h_status[kStatusTimeout] == 0xFFFFFFFFu) return FDTD_OK;
    std::lock_guard<std::mutex> lk(g_err_mu);
    snprintf(g_err, sizeof(g_err), "fused step: a tile's load wait timed out (block %u)",
             st->h_status[kStatusTimeout]);
    return FDTD_ERR_CUDA;
}

void report_unstable_cell(AcousticFDTDState* st, unsigned q)
{
    const int ny = st->Ny, nz = st->Nz;
    int ci = (int)(q / (unsigned)(ny * nz)), cj = (int)((q / (unsigned)nz) % (unsigned)ny),
        ck = (int)(q % (unsigned)nz);
    float v = NAN;
    cudaMemcpy(&v, st->P() + st->pad(ci, cj, ck), sizeof(float), cudaMemcpyDeviceToHost);
    fprintf(stderr, "[fdtd_pressure] UNSTABLE step=%d cell=%u (%d,%d,%d) p=%.3g Pa\n",
            st->step_count, q, ci, cj, ck, (double)v);
    fflush(stderr);
}

// The fused step reads one velocity set and writes the other (neighbouring
// tiles recompute halo faces from the old values, so updates cannot be in
// place).  Engine-owned fields get the second set on first use.
int alloc_second_velocity_set(AcousticFDTDState* st)
{
    const int b = st->cv ^ 1;
    for (int c2 = 0; c2 < 3; ++c2) {
        if (st->v[b][c2]) continue;
        CK(cudaMalloc(&st->v[b][c2], st->field_bytes));
        CK(cudaMemsetAsync(st->v[b][c2], 0, st->field_bytes, st->stream));
    }
    return FDTD_OK;
}

// Records the receivers of the current pressure into the pending trace slot
// (a record a fused step left for the next one to take).
int flush_record(AcousticFDTDState* st)
{
    if (st->rec_pending < 0) return FDTD_OK;
    const int slot = st->rec_pending;
    st->rec_pending = -1;
    CK(launch_wsum(st->P(), st->d_rec_idx, st->d_rec_w, st->n_rec, 8, 0,
                   st->d_trace + (size_t)slot * st->n_rec, st->stream));
    ++st->launches;
    return FDTD_OK;
}

// One time step (acoustic_fdtd.cpp:1272-1290 loop body) plus the engine's
// point-source deposit before it and receiver record after it.
// sync_check: stop and return FDTD_ERR_UNSTABLE at a failed check (fdtd_step);
// otherwise failures are latched on the device (fdtd_b200_step_async).
// defer_record: a fused step leaves its receiver record pending, to be taken
// by the next fused step's kernel from its input pressure; the caller ends
// its run of steps with flush_record.  On the fused path the point-source
// deposit of an open source cell is applied inside the step kernel too.
// A plate node that receives a pending force (recorded once).
inline void note_ext(AcousticFDTDState* st, int pidx)
{
    if (!st->ext_mark[pidx]) {
        st->ext_mark[pidx] = 1;
        st->ext_nodes.push_back(pidx);
    }
}

// The pending forces consumed: their host entries (the only nonzero ones) back to zero.
void clear_ext_host(AcousticFDTDState* st)
{
    for (int pidx : st->ext_nodes) {
        st->h_ext[pidx] = 0.0f;
        st->ext_mark[pidx] = 0;
    }
    st->ext_nodes.clear();
    st->ext_pending = false;
}

int substep_plate(AcousticFDTDState* st, int n_saddle, float* out);

int one_step(AcousticFDTDState* st, bool sync_check, bool defer_record = false)
{
    cudaStream_t s = st->stream;
    const bool fused = use_fused(st);
    if (!fused) {
        if (int rc0 = flush_record(st)) return rc0;
        // A plate scene on the two-pass kernels waits for its plate guard every
        // step anyway: take the substep's schedule (all of the step issued, the
        // guard read with the status words at its end, graph replay where it
        // applies), which leaves the same state and return codes.
        if (st->n_act > 0 && sync_check && !st->prof_on) return substep_plate(st, 0, nullptr);
    }
    // point source: deposit s[n] before step n (applies before the plate reads P)
    bool fuse_deposit = false;
    if (st->ps_n > 0 && st->step_count < st->ps_n && st->ps.n > 0 && st->ps_done_step != st->step_count) {
        fuse_deposit = fused && st->ps.n == 1 && st->ps.divisor == 0;
        if (!fuse_deposit) {
            CK(launch_deposit(st->ps, st->d_ps_sig, st->step_count, 0.0f, st->P(), s));
            ++st->launches;
        }
        st->ps_done_step = st->step_count;
    }

    // plate step (acoustic_fdtd.cpp:984-1053)
    if (st->n_act > 0) {
        if (st->ext_pending) {
            CK(cudaMemcpyAsync(st->d_ext, st->h_ext, (size_t)st->N_plate * sizeof(float),
                               cudaMemcpyHostToDevice, s));
            st->dev_ext_nonzero = true;
        }
        CK(cudaMemsetAsync(st->d_status + kStatusPlate, 0xFF, sizeof(unsigned), s));
        CK(launch_plate_step(st->n_act, st->d_act, st->d_nb13, st->d_above, st->d_below,
                             st->d_w[st->wi_cur], st->d_w[st->wi_prev], st->d_w[st->wi_tmp],
                             st->d_ext, st->P(), st->pc, st->d_status, s));
        ++st->launches;
        CK(cudaMemcpyAsync(st->h_status + kStatusPlate, st->d_status + kStatusPlate,
                           sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        unsigned bad = st->h_status[kStatusPlate];
        if (bad != 0xFFFFFFFFu) {
            int pidx = st->h_act[bad];
            float wn = NAN;
            cudaMemcpy(&wn, st->d_w[st->wi_tmp] + pidx, sizeof(float), cudaMemcpyDeviceToHost);
            fprintf(stderr,
                    "[fdtd_plate] UNSTABLE step=%d plate_node=%d (%d,%d) w_new=%.3g m (limit 0.02 m)\n",
                    st->step_count, pidx, pidx / st->Ny, pidx % st->Ny, (double)wn);
            fflush(stderr);
            return FDTD_ERR_UNSTABLE;   // no rotation; pending forces stay (as the reference)
        }
        // consume the forces (acoustic_fdtd.cpp:1045-1046) and rotate w
        if (st->dev_ext_nonzero) {
            CK(cudaMemsetAsync(st->d_ext, 0, (size_t)st->N_plate * sizeof(float), s));
            st->dev_ext_nonzero = false;
        }
        if (st->ext_pending) clear_ext_host(st);
        int t = st->wi_prev;
        st->wi_prev = st->wi_cur;
        st->wi_cur = st->wi_tmp;
        st->wi_tmp = t;
    } else if (st->ext_pending) {
        clear_ext_host(st);   // consumed with no plate
    }

    // velocity + pressure
    cudaEvent_t e1;
    int rc = prof_begin(st, &e1);
    if (rc) return rc;
    if (fused) {
        if (!st->v[st->cv ^ 1][0]) {
            int rc2 = alloc_second_velocity_set(st);
            if (rc2) return rc2;
        }
        if (!st->fcache) st->fcache = fused_cache_create();
        FusedArgs a{st->g, st->cf, st->tb, st->P(), st->Pn(),
                    {st->V(0), st->V(1), st->V(2)},
                    {st->v[st->cv ^ 1][0], st->v[st->cv ^ 1][1], st->v[st->cv ^ 1][2]},
                    st->d_status};
        a.hold_plane = st->hold_plane;
        a.wait_us = st->wait_us;
        const bool walled = !fused_eligible(st);
        if (walled) {
            for (int c2 = 0; c2 < 3; ++c2) a.fr[c2] = st->d_frac[c2];
            a.frac_div = st->has_frac;
            a.solid = st->d_solid;
        }
        if (fuse_deposit) {
            const long long c = st->ps.idx[0], t = c / st->g.sz;
            a.dep_sig = st->d_ps_sig;
            a.dep_step = st->step_count;
            a.dep_i = (int)(t / st->Ny);
            a.dep_j = (int)(t % st->Ny);
            a.dep_k = (int)(c % st->g.sz);
        }
        if (st->rec_pending >= 0) {
            a.rec_idx = st->d_rec_idx;
            a.rec_w = st->d_rec_w;
            a.rec_out = st->d_trace + (size_t)st->rec_pending * st->n_rec;
            a.n_rec = st->n_rec;
            st->rec_pending = -1;
        }
        CK(launch_fused_step(a, st->fcache, s));
        ++st->launches;
        st->cv ^= 1;
        if (walled && st->n_act > 0) {
            // the plate sets its faces' velocity after the update (as on the
            // two-pass path); the cells whose divergence reads those faces are
            // then updated again from P^n and the new velocities
            CK(launch_plate_inject(st->n_act, st->d_act, st->d_vzb, st->d_vza, st->d_w[st->wi_cur],
                                   st->d_w[st->wi_prev], st->cf.inv_dt, st->V(2), s));
            const bool hf = st->has_frac;
            CK(launch_pressure_groups(st->g, st->cf, st->tb, st->P(), st->Pn(), st->V(0), st->V(1), st->V(2),
                                      hf ? st->d_frac[0] : nullptr, hf ? st->d_frac[1] : nullptr,
                                      hf ? st->d_frac[2] : nullptr, st->d_solid, st->d_pfix, st->n_pfix, s));
            st->launches += 2;
        }
        if ((rc = prof_end(st, e1, fused_kernel_launches_per_step()))) return rc;
    } else {
        PlateFaces pf;   // the plate's face velocities, set inside the velocity pass
        if (st->n_act > 0) {
            pf.code = st->d_plate_code;
            pf.w = st->d_w[st->wi_cur];
            pf.wp = st->d_w[st->wi_prev];
            pf.inv_dt = st->cf.inv_dt;
            pf.iz = st->plate_iz;
        }
        CK(launch_velocity_general(st->g, st->cf, st->tb, st->P(), st->V(0), st->V(1), st->V(2),
                                   st->d_frac[0], st->d_frac[1], st->d_frac[2], s, nullptr, &pf));
        st->launches += 2;
        const bool hf = st->has_frac;
        CK(launch_pressure_general(st->g, st->cf, st->tb, st->P(), st->Pn(), st->V(0), st->V(1),
                                   st->V(2), hf ? st->d_frac[0] : nullptr,
                                   hf ? st->d_frac[1] : nullptr, hf ? st->d_frac[2] : nullptr,
                                   st->d_solid, s));
        if ((rc = prof_end(st, e1, 2))) return rc;
    }
    st->cur ^= 1;
    ++st->step_count;

    // receivers
    if (st->n_rec > 0 && st->trace_len < st->trace_cap) {
        if (fused && defer_record) {
            st->rec_pending = st->trace_len;
        } else {
            CK(launch_wsum(st->P(), st->d_rec_idx, st->d_rec_w, st->n_rec, 8, 0,
                           st->d_trace + (size_t)st->trace_len * st->n_rec, s));
            ++st->launches;
        }
        ++st->trace_len;
    }

    // stability check every 256 steps (acoustic_fdtd.cpp:1284-1287)
    if ((st->step_count & (kCheckPeriod - 1)) == 0) {
        int phase = st->stab_phase;
        st->stab_phase = (phase + 1) % kCheckStride;
        if (sync_check) CK(cudaMemsetAsync(st->d_status + kStatusCell, 0xFF, sizeof(unsigned), s));
        CK(launch_check(st->g, st->P(), st->N, phase, st->d_status, st->step_count, s));
        ++st->launches;
        if (sync_check) {
            CK(cudaMemcpyAsync(st->h_status, st->d_status, kStatusWords * sizeof(unsigned),
                               cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (int rc2 = check_timeout(st)) return rc2;
            unsigned bad = st->h_status[kStatusCell];
            if (bad != 0xFFFFFFFFu) {
                report_unstable_cell(st, bad);
                CK(cudaMemsetAsync(st->d_status + kStatusLatch, 0xFF, sizeof(unsigned), s));
                return FDTD_ERR_UNSTABLE;
            }
        }
    }
    return FDTD_OK;
}

void free_state(AcousticFDTDState* st)
{
    if (!st) return;
    int d = -1;
    cudaGetDevice(&d);
    if (d != st->device) cudaSetDevice(st->device);
    if (st->stream) cudaStreamSynchronize(st->stream);
    for (auto& sg : st->sgraphs)
        if (sg.exec) cudaGraphExecDestroy(sg.exec);
    st->sgraphs.clear();
    if (st->own_fields) {
        cudaFree(st->p[0]); cudaFree(st->p[1]);
        for (int b = 0; b < 2; ++b)
            for (int c2 = 0; c2 < 3; ++c2) cudaFree(st->v[b][c2]);
    }
    cudaFree(st->d_tab);
    cudaFree(st->d_solid);
    for (int c = 0; c < 3; ++c) { cudaFree(st->d_frac[c]); cudaFree(st->d_w[c]); }
    cudaFree(st->d_act); cudaFree(st->d_nb13); cudaFree(st->d_above); cudaFree(st->d_below);
    cudaFree(st->d_vzb); cudaFree(st->d_vza); cudaFree(st->d_pfix); cudaFree(st->d_plate_code); cudaFree(st->d_ext); cudaFree(st->d_slice);
    cudaFreeHost(st->h_ext);
    cudaFreeHost(st->h_ext_pack);
    cudaFree(st->d_ext_pack);
    cudaFree(st->d_ps_sig);
    cudaFree(st->d_rec_idx); cudaFree(st->d_rec_w); cudaFree(st->d_trace);
    cudaFree(st->d_status); cudaFreeHost(st->h_status);
    cudaFree(st->d_sidx); cudaFree(st->d_sw); cudaFree(st->d_sout);
    cudaFreeHost(st->h_sidx); cudaFreeHost(st->h_sw); cudaFreeHost(st->h_sout); cudaFreeHost(st->h_sout_map);
    for (cudaEvent_t e : st->prof.ev) cudaEventDestroy(e);
    fused_cache_destroy(st->fcache);
    if (st->own_stream) cudaStreamDestroy(st->own_stream);
    if (d >= 0 && d != st->device) cudaSetDevice(d);
    delete st;
}

#define CKN(expr)                     \
    do {                              \
        cudaError_t e_ = (expr);      \
        if (e_ != cudaSuccess) {      \
            set_err(e_, #expr);       \
            free_state(st);           \
            return nullptr;           \
        }                             \
    } while (0)

AcousticFDTDState* create_impl(int Nx, int Ny, int Nz, float dx, float c, float rho_air,
                               const uint8_t* cell_type, int plate_iz,
                               const uint8_t* plate_active, float plate_mass_density,
                               float plate_stiffness_D, float plate_alpha_M, float plate_beta_K,
                               int n_pml, int device, float* const* fields)
{
    // argument checks of acoustic_fdtd.cpp:342-344, plus the int index range of the ABI
    if (Nx <= 0 || Ny <= 0 || Nz <= 0 || dx <= 0.0f || c <= 0.0f || cell_type == NULL ||
        plate_active == NULL)
        return nullptr;
    if ((long long)Nx * Ny * Nz > INT_MAX) return nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        set_err(cudaErrorNoDevice, "fdtd_create: no CUDA device");
        cudaGetLastError();
        return nullptr;
    }
    AcousticFDTDState* st = new AcousticFDTDState();
    if (device < 0) CKN(cudaGetDevice(&device));
    st->device = device;
    CKN(cudaSetDevice(device));
    CKN(cudaStreamCreateWithFlags(&st->own_stream, cudaStreamNonBlocking));
    st->stream = st->own_stream;

    // time step and coefficients (acoustic_fdtd.cpp:345-349, :1091, :1171-1173)
    const float dt = 0.77f * dx / (c * 1.732050808f);
    st->Nx = Nx; st->Ny = Ny; st->Nz = Nz;
    st->N = Nx * Ny * Nz;
    st->N_plate = Nx * Ny;
    st->plate_iz = (plate_iz >= 0 && plate_iz < Nz) ? plate_iz : Nz / 2;
    st->n_pml = n_pml;
    st->dx = dx; st->c = c; st->rho = rho_air; st->dt = dt;
    st->cf.vc = dt / (rho_air * dx);
    const float inv_dx = 1.0f / dx;
    st->cf.bulk = rho_air * c * c * dt * inv_dx;
    st->cf.dt = dt;
    st->cf.c1 = 9.0f / 8.0f;
    st->cf.c2 = -1.0f / 24.0f;
    st->cf.inv_dt = 1.0f / dt;
    // plate constants (acoustic_fdtd.cpp:435-449)
    st->pc.a = (dt * dt) / plate_mass_density;
    {
        float dx4 = dx * dx * dx * dx;
        st->pc.bh = plate_stiffness_D * (dt * dt) / (plate_mass_density * dx4);
    }
    st->pc.vd = 1.0f - plate_alpha_M * dt;
    st->pc.bk = (dt > 0.0f) ? (plate_beta_K / dt * st->pc.bh) : 0.0f;

    st->g.nx = Nx; st->g.ny = Ny; st->g.nz = Nz;
    st->g.sz = (Nz + kRowAlign - 1) / kRowAlign * kRowAlign;
    st->g.plane = (long long)Ny * st->g.sz;
    st->g.cells = (long long)Nx * st->g.plane;
    st->field_bytes = (size_t)st->g.cells * sizeof(float);

    // geometry on the host: PML marking (:386-395) and plate mask (:413-425)
    st->cell_type.assign(cell_type, cell_type + st->N);
    st->plate_active.assign(plate_active, plate_active + st->N_plate);
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j) {
            int g = st->plate_iz + Nz * (j + Ny * i);
            if (st->plate_active[j + Ny * i]) {
                if (st->cell_type[g] == FDTD_AIR || st->cell_type[g] == FDTD_PML)
                    st->cell_type[g] = FDTD_PLATE;
            } else if (st->cell_type[g] == FDTD_PLATE) {
                st->cell_type[g] = FDTD_AIR;
            }
        }
    for (int q = 0; q < st->N; ++q)
        if (is_solid(st->cell_type[q])) { st->any_solid = true; break; }

    // fields
    if (fields) {
        for (int q = 0; q < 8; ++q)
            if (!fields[q] || ((uintptr_t)fields[q] & 15u)) {
                free_state(st);
                return nullptr;
            }
        st->own_fields = false;
        st->p[0] = fields[0]; st->p[1] = fields[1];
        for (int c2 = 0; c2 < 3; ++c2) {
            st->v[0][c2] = fields[2 + c2];
            st->v[1][c2] = fields[5 + c2];
        }
    } else {
        st->own_fields = true;
        CKN(cudaMalloc(&st->p[0], st->field_bytes));
        CKN(cudaMalloc(&st->p[1], st->field_bytes));
        for (int c2 = 0; c2 < 3; ++c2) CKN(cudaMalloc(&st->v[0][c2], st->field_bytes));
    }
    for (float* f : {st->p[0], st->p[1], st->v[0][0], st->v[0][1], st->v[0][2], st->v[1][0],
                     st->v[1][1], st->v[1][2]})
        if (f) CKN(cudaMemsetAsync(f, 0, st->field_bytes, st->stream));

    CKN(cudaMalloc(&st->d_tab, sizeof(float) * 2 * (Nx + Ny + Nz)));
    st->tb.ax = st->d_tab;
    st->tb.ay = st->tb.ax + Nx;
    st->tb.az = st->tb.ay + Ny;
    st->tb.px = st->tb.az + Nz;
    st->tb.py = st->tb.px + Nx;
    st->tb.pz = st->tb.py + Ny;
    if (build_tables(st)) { free_state(st); return nullptr; }

    if (st->any_solid) {
        std::vector<uint8_t> m((size_t)st->g.cells, 0);
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < Nz; ++k)
                    m[st->pad(i, j, k)] = is_solid(st->cell_type[k + Nz * (j + Ny * i)]) ? 1 : 0;
        CKN(cudaMalloc(&st->d_solid, m.size()));
        CKN(cudaMemcpy(st->d_solid, m.data(), m.size(), cudaMemcpyHostToDevice));
        default_fracs(st);
        if (upload_fracs(st)) { free_state(st); return nullptr; }
    }

    // plate tables (acoustic_fdtd.cpp:670-752)
    for (int c2 = 0; c2 < 3; ++c2) {
        CKN(cudaMalloc(&st->d_w[c2], sizeof(float) * st->N_plate));
        CKN(cudaMemsetAsync(st->d_w[c2], 0, sizeof(float) * st->N_plate, st->stream));
    }
    CKN(cudaMalloc(&st->d_ext, sizeof(float) * st->N_plate));
    CKN(cudaMemsetAsync(st->d_ext, 0, sizeof(float) * st->N_plate, st->stream));
    CKN(cudaMallocHost(&st->h_ext, sizeof(float) * st->N_plate));
    memset(st->h_ext, 0, sizeof(float) * st->N_plate);
    st->ext_mark.assign((size_t)st->N_plate, 0);
    CKN(cudaMallocHost(&st->h_ext_pack, sizeof(int2) * std::max(st->N_plate, 1)));
    CKN(cudaMalloc(&st->d_ext_pack, sizeof(int2) * std::max(st->N_plate, 1)));
    {
        static const int DI[13] = {0, 1, -1, 0, 0, 1, 1, -1, -1, 2, -2, 0, 0};
        static const int DJ[13] = {0, 0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 2, -2};
        std::vector<int> nb13;
        std::vector<long long> above, below, vzb, vza;
        const int piz = st->plate_iz;
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) {
                int pidx = j + Ny * i;
                if (!st->plate_active[pidx]) continue;
                st->h_act.push_back(pidx);
                above.push_back(piz + 1 < Nz ? st->pad(i, j, piz + 1) : -1);
                below.push_back(piz - 1 >= 0 ? st->pad(i, j, piz - 1) : -1);
                for (int t = 0; t < 13; ++t) {
                    int ii = i + DI[t], jj = j + DJ[t];
                    if (ii < 0 || ii >= Nx || jj < 0 || jj >= Ny || !st->plate_active[jj + Ny * ii]) {
                        ii = i;
                        jj = j;
                    }
                    nb13.push_back(jj + Ny * ii);
                }
                const uint8_t* ct = st->cell_type.data();
                vzb.push_back(piz > 0 && !is_solid(ct[(piz - 1) + Nz * (j + Ny * i)]) ? st->pad(i, j, piz - 1) : -1);
                vza.push_back(piz < Nz - 1 && !is_solid(ct[(piz + 1) + Nz * (j + Ny * i)]) ? st->pad(i, j, piz) : -1);
            }
        st->n_act = (int)st->h_act.size();
        if (st->n_act > 0) {
            const size_t na = st->n_act;
            CKN(cudaMalloc(&st->d_act, na * sizeof(int)));
            CKN(cudaMalloc(&st->d_nb13, na * 13 * sizeof(int)));
            CKN(cudaMalloc(&st->d_above, na * sizeof(long long)));
            CKN(cudaMalloc(&st->d_below, na * sizeof(long long)));
            CKN(cudaMalloc(&st->d_vzb, na * sizeof(long long)));
            CKN(cudaMalloc(&st->d_vza, na * sizeof(long long)));
            CKN(cudaMemcpy(st->d_act, st->h_act.data(), na * sizeof(int), cudaMemcpyHostToDevice));
            CKN(cudaMemcpy(st->d_nb13, nb13.data(), na * 13 * sizeof(int), cudaMemcpyHostToDevice));
            CKN(cudaMemcpy(st->d_above, above.data(), na * sizeof(long long), cudaMemcpyHostToDevice));
            CKN(cudaMemcpy(st->d_below, below.data(), na * sizeof(long long), cudaMemcpyHostToDevice));
            CKN(cudaMemcpy(st->d_vzb, vzb.data(), na * sizeof(long long), cudaMemcpyHostToDevice));
            CKN(cudaMemcpy(st->d_vza, vza.data(), na * sizeof(long long), cudaMemcpyHostToDevice));
            std::vector<uint8_t> code((size_t)st->N_plate, 0);
            for (size_t q = 0; q < na; ++q)
                code[st->h_act[q]] = (uint8_t)((vzb[q] >= 0 ? 1 : 0) | (vza[q] >= 0 ? 2 : 0));
            CKN(cudaMalloc(&st->d_plate_code, code.size()));
            CKN(cudaMemcpy(st->d_plate_code, code.data(), code.size(), cudaMemcpyHostToDevice));
            // cells whose pressure update reads plate face kf: k = kf-1 .. kf+2
            std::vector<long long> fix;
            for (const auto* lst : {&vzb, &vza})
                for (long long q : *lst) {
                    if (q < 0) continue;
                    const int kf = (int)(q % st->g.sz);
                    const long long row = q - kf;
                    for (int k = kf - 1; k <= kf + 2; ++k)
                        if (k >= 0 && k < Nz) fix.push_back(row + (k & ~3));
                }
            std::sort(fix.begin(), fix.end());
            fix.erase(std::unique(fix.begin(), fix.end()), fix.end());
            st->n_pfix = (int)fix.size();
            if (st->n_pfix > 0) {
                CKN(cudaMalloc(&st->d_pfix, fix.size() * sizeof(long long)));
                CKN(cudaMemcpy(st->d_pfix, fix.data(), fix.size() * sizeof(long long), cudaMemcpyHostToDevice));
            }
        }
    }

    CKN(cudaMalloc(&st->d_status, kStatusWords * sizeof(unsigned)));
    CKN(cudaMemsetAsync(st->d_status, 0xFF, kStatusWords * sizeof(unsigned), st->stream));
    CKN(cudaMallocHost(&st->h_status, kStatusWords * sizeof(unsigned)));
    CKN(cudaStreamSynchronize(st->stream));
    return st;
}

}  // namespace

/* ============================== reference entry points ============================== */

extern "C" {

AcousticFDTDState* fdtd_create(int Nx, int Ny, int Nz, float dx, float c, float rho_air,
                               const uint8_t* cell_type, int plate_iz, const uint8_t* plate_active,
                               float plate_mass_density, float plate_stiffness_D,
                               float plate_alpha_M, float plate_beta_K, int n_pml)
{
    return create_impl(Nx, Ny, Nz, dx, c, rho_air, cell_type, plate_iz, plate_active,
                       plate_mass_density, plate_stiffness_D, plate_alpha_M, plate_beta_K, n_pml,
                       -1, nullptr);
}

AcousticFDTDState* fdtd_b200_create_ex(int Nx, int Ny, int Nz, float dx, float c, float rho_air,
                                       const uint8_t* cell_type, int plate_iz,
                                       const uint8_t* plate_active, float plate_mass_density,
                                       float plate_stiffness_D, float plate_alpha_M,
                                       float plate_beta_K, int n_pml, int device,
                                       float* const* fields)
{
    return create_impl(Nx, Ny, Nz, dx, c, rho_air, cell_type, plate_iz, plate_active,
                       plate_mass_density, plate_stiffness_D, plate_alpha_M, plate_beta_K, n_pml,
                       device, fields);
}

void fdtd_destroy(AcousticFDTDState* st) { free_state(st); }

int fdtd_set_bridge_sources(AcousticFDTDState* st, int n_cells, const int* cell_indices,
                            const float* weights)
{   // acoustic_fdtd.cpp:798-830
    if (!st || n_cells <= 0 || !cell_indices || !weights) return FDTD_ERR_NULL;
    float wsum = 0.0f;
    for (int i = 0; i < n_cells; ++i) wsum += fabsf(weights[i]);
    float wscale = (wsum > 1e-12f) ? 1.0f / wsum : 1.0f;
    st->src_idx.assign(cell_indices, cell_indices + n_cells);
    st->src_wgt.resize(n_cells);
    for (int i = 0; i < n_cells; ++i) st->src_wgt[i] = weights[i] * wscale;
    return FDTD_OK;
}

int fdtd_inject_bridge(AcousticFDTDState* st, float signal_val, float signal_ddt, float force_scale)
{   // acoustic_fdtd.cpp:874-885: disabled
    (void)st; (void)signal_val; (void)signal_ddt; (void)force_scale;
    return FDTD_ERR_UNSTABLE;
}

int fdtd_inject_bridge_drive(AcousticFDTDState* st, const float* cell_drives, float force_scale)
{   // acoustic_fdtd.cpp:1699-1721
    if (!st) return FDTD_ERR_NULL;
    if (st->src_idx.empty()) return FDTD_OK;
    if (!cell_drives) return FDTD_ERR_NULL;
    float inv_dx2 = 1.0f / (st->dx * st->dx);
    for (size_t i = 0; i < st->src_idx.size(); ++i) {
        int pidx = st->src_idx[i] / st->Nz;
        if (pidx < 0 || pidx >= st->N_plate) return FDTD_ERR_ARG;
        note_ext(st, pidx);
        st->h_ext[pidx] += force_scale * cell_drives[i] * inv_dx2;
    }
    st->ext_pending = true;
    return FDTD_OK;
}

int fdtd_inject_plate_force(AcousticFDTDState* st, int n_plate, const int* plate_indices,
                            const float* weights, float total_force_N)
{   // acoustic_fdtd.cpp:1723-1742
    if (!st || !plate_indices || !weights) return FDTD_ERR_NULL;
    if (n_plate <= 0 || total_force_N == 0.0f) return FDTD_OK;
    float inv_dx2 = 1.0f / (st->dx * st->dx);
    for (int i = 0; i < n_plate; ++i) {
        int pidx = plate_indices[i];
        if (pidx < 0 || pidx >= st->N_plate) continue;
        if (!st->plate_active[pidx]) continue;
        note_ext(st, pidx);
        st->h_ext[pidx] += total_force_N * weights[i] * inv_dx2;
        st->ext_pending = true;
    }
    return FDTD_OK;
}

int fdtd_set_face_fractions(AcousticFDTDState* st, const float* vx_frac, const float* vy_frac,
                            const float* vz_frac)
{   // acoustic_fdtd.cpp:1064-1077
    if (!st) return FDTD_ERR_NULL;
    if (!vx_frac && !vy_frac && !vz_frac) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    if (st->frac[0].empty()) default_fracs(st);
    if (vx_frac) memcpy(st->frac[0].data(), vx_frac, st->frac[0].size() * sizeof(float));
    if (vy_frac) memcpy(st->frac[1].data(), vy_frac, st->frac[1].size() * sizeof(float));
    if (vz_frac) memcpy(st->frac[2].data(), vz_frac, st->frac[2].size() * sizeof(float));
    st->has_frac = true;
    return upload_fracs(st);
}

int fdtd_sample_plate_weighted(const AcousticFDTDState* cst, int n_plate, const int* plate_indices,
                               const float* weights, float* out_w)
{   // acoustic_fdtd.cpp:1744-1760
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !plate_indices || !weights || !out_w) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc = ensure_scratch(st, n_plate > 0 ? (size_t)n_plate : 1);
    if (rc) return rc;
    int m = 0;
    for (int i = 0; i < n_plate; ++i) {
        int pidx = plate_indices[i];
        if (pidx < 0 || pidx >= st->N_plate) continue;
        st->h_sidx[m] = pidx;
        st->h_sw[m] = weights[i];
        ++m;
    }
    if (m == 0) { *out_w = 0.0f; return FDTD_OK; }
    return run_wsum(st, st->d_w[st->wi_cur], 1, m, 1, out_w);
}

int fdtd_precompute_pressure_samplers(const AcousticFDTDState* st, int n_rec, const float* rec_xyz,
                                      int* out_idx8, float* out_wgt8)
{   // acoustic_fdtd.cpp:1567-1596
    if (!st || !rec_xyz || !out_idx8 || !out_wgt8) return FDTD_ERR_NULL;
    for (int r = 0; r < n_rec; ++r) sampler_taps(st, 0, rec_xyz + 3 * r, out_idx8 + 8 * r, out_wgt8 + 8 * r);
    return FDTD_OK;
}

int fdtd_precompute_velocity_samplers(const AcousticFDTDState* st, int n_rec, const float* rec_xyz,
                                      int* out_vx_idx8, float* out_vx_wgt8, int* out_vy_idx8,
                                      float* out_vy_wgt8, int* out_vz_idx8, float* out_vz_wgt8)
{   // acoustic_fdtd.cpp:1598-1661
    if (!st || !rec_xyz) return FDTD_ERR_NULL;
    if (!out_vx_idx8 || !out_vx_wgt8 || !out_vy_idx8 || !out_vy_wgt8 || !out_vz_idx8 || !out_vz_wgt8)
        return FDTD_ERR_NULL;
    for (int r = 0; r < n_rec; ++r) {
        sampler_taps(st, 1, rec_xyz + 3 * r, out_vx_idx8 + 8 * r, out_vx_wgt8 + 8 * r);
        sampler_taps(st, 2, rec_xyz + 3 * r, out_vy_idx8 + 8 * r, out_vy_wgt8 + 8 * r);
        sampler_taps(st, 3, rec_xyz + 3 * r, out_vz_idx8 + 8 * r, out_vz_wgt8 + 8 * r);
    }
    return FDTD_OK;
}

int fdtd_sample_pressure_precomputed(const AcousticFDTDState* cst, int n_rec, const int* idx8,
                                     const float* wgt8, float* out_p)
{   // acoustic_fdtd.cpp:1663-1676
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !idx8 || !wgt8 || !out_p) return FDTD_ERR_NULL;
    if (n_rec <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc = stage_taps(st, 0, n_rec, idx8, wgt8);
    if (rc) return rc;
    return run_wsum(st, st->P(), n_rec, 8, 0, out_p);
}

int fdtd_sample_velocity_precomputed(const AcousticFDTDState* cst, int n_rec, const int* vx_idx8,
                                     const float* vx_wgt8, const int* vy_idx8,
                                     const float* vy_wgt8, const int* vz_idx8,
                                     const float* vz_wgt8, float* out_vx, float* out_vy,
                                     float* out_vz)
{   // acoustic_fdtd.cpp:1678-1697
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !vx_idx8 || !vx_wgt8 || !vy_idx8 || !vy_wgt8 || !vz_idx8 || !vz_wgt8) return FDTD_ERR_NULL;
    if (!out_vx || !out_vy || !out_vz) return FDTD_ERR_NULL;
    if (n_rec <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    const int* ids[3] = {vx_idx8, vy_idx8, vz_idx8};
    const float* ws[3] = {vx_wgt8, vy_wgt8, vz_wgt8};
    float* outs[3] = {out_vx, out_vy, out_vz};
    for (int c = 0; c < 3; ++c) {
        int rc = stage_taps(st, c + 1, n_rec, ids[c], ws[c]);
        if (rc) return rc;
        if ((rc = run_wsum(st, field_ptr(st, c + 1), n_rec, 8, 1, outs[c]))) return rc;
    }
    return FDTD_OK;
}

int fdtd_step(AcousticFDTDState* st, int n_steps)
{   // acoustic_fdtd.cpp:1272-1290
    if (!st) return FDTD_ERR_NULL;
    if (n_steps <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc = FDTD_OK;
    for (int s = 0; s < n_steps && rc == FDTD_OK; ++s) rc = one_step(st, true, true);
    const int rc_rec = flush_record(st);
    return rc != FDTD_OK ? rc : rc_rec;
}

int fdtd_get_step_count(const AcousticFDTDState* st) { return st ? st->step_count : 0; }
float fdtd_get_dt(const AcousticFDTDState* st) { return st ? st->dt : 0.0f; }

int fdtd_reset(AcousticFDTDState* st)
{   // acoustic_fdtd.cpp:1297-1310; also clears recorded receiver traces
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    for (float* f : {st->p[0], st->p[1], st->v[0][0], st->v[0][1], st->v[0][2], st->v[1][0],
                     st->v[1][1], st->v[1][2]})
        if (f) CK(cudaMemsetAsync(f, 0, st->field_bytes, st->stream));
    for (int c = 0; c < 3; ++c) CK(cudaMemsetAsync(st->d_w[c], 0, sizeof(float) * st->N_plate, st->stream));
    CK(cudaMemsetAsync(st->d_ext, 0, sizeof(float) * st->N_plate, st->stream));
    // a latched fused-step timeout or instability ends with the state it spoiled
    CK(cudaMemsetAsync(st->d_status, 0xFF, kStatusWords * sizeof(unsigned), st->stream));
    CK(cudaStreamSynchronize(st->stream));
    for (int w = 0; w < kStatusWords; ++w) st->h_status[w] = 0xFFFFFFFFu;
    clear_ext_host(st);
    st->dev_ext_nonzero = false;
    st->step_count = 0;
    st->trace_len = 0;
    st->ps_done_step = -1;
    return FDTD_OK;
}

int fdtd_b200_get_volume_slice(const AcousticFDTDState* cst, int axis, int idx, float* out, int out_len)
{   // acoustic_fdtd_bridge.py:737-757 without the full-field copy
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !out) return FDTD_ERR_NULL;
    if (axis < 0 || axis > 2) return FDTD_ERR_ARG;
    const int dims[3] = {st->Nx, st->Ny, st->Nz};
    const int na = axis == 0 ? st->Ny : st->Nx, nb = axis == 2 ? st->Ny : st->Nz;
    if ((long long)out_len != (long long)na * nb) return FDTD_ERR_DIM;
    if (idx < 0) idx = dims[axis] / 2;
    idx = std::min(idx, dims[axis] - 1);
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    if (!st->d_slice) {
        const size_t most = (size_t)std::max({(long long)st->Ny * st->Nz, (long long)st->Nx * st->Nz,
                                              (long long)st->Nx * st->Ny});
        CK(cudaMalloc(&st->d_slice, most * sizeof(float)));
    }
    CK(launch_slice(st->P(), st->g, axis, idx, st->d_slice, na, nb, st->stream));
    CK(cudaMemcpyAsync(out, st->d_slice, sizeof(float) * (size_t)out_len, cudaMemcpyDeviceToHost, st->stream));
    CK(cudaStreamSynchronize(st->stream));
    return FDTD_OK;
}

int fdtd_get_pressure_field(const AcousticFDTDState* cst, float* out, int out_len)
{   // acoustic_fdtd.cpp:1314-1321
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !out) return FDTD_ERR_NULL;
    if (out_len != st->N) return FDTD_ERR_DIM;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    return copy_block(st, st->P(), out, st->Nx, st->Ny, st->Nz, false);
}

int fdtd_get_plate_displacement(const AcousticFDTDState* cst, float* out, int out_len)
{   // acoustic_fdtd.cpp:1323-1330
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !out) return FDTD_ERR_NULL;
    if (out_len != st->N_plate) return FDTD_ERR_DIM;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaMemcpyAsync(out, st->d_w[st->wi_cur], sizeof(float) * st->N_plate, cudaMemcpyDeviceToHost,
                       st->stream));
    CK(cudaStreamSynchronize(st->stream));
    return FDTD_OK;
}

int fdtd_sample_plate_displacement_batch(const AcousticFDTDState* cst, int n_points,
                                         const int* saddle_idx4, const float* saddle_wgt4,
                                         float* out_w)
{   // acoustic_fdtd.cpp:1332-1353
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !saddle_idx4 || !saddle_wgt4 || !out_w) return FDTD_ERR_NULL;
    if (n_points <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc = ensure_scratch(st, (size_t)n_points * 4);
    if (rc) return rc;
    for (long long q = 0; q < (long long)n_points * 4; ++q) {
        if (saddle_idx4[q] < 0 || saddle_idx4[q] >= st->N_plate) return FDTD_ERR_ARG;
        st->h_sidx[q] = saddle_idx4[q];
        st->h_sw[q] = saddle_wgt4[q];
    }
    return run_wsum(st, st->d_w[st->wi_cur], n_points, 4, 0, out_w);
}

int fdtd_sample_pressure(const AcousticFDTDState* cst, int n_rec, const float* rec_xyz, float* out_p)
{   // acoustic_fdtd.cpp:1355-1395
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !rec_xyz || !out_p) return FDTD_ERR_NULL;
    if (n_rec <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    return direct_samples(st, 0, n_rec, rec_xyz, out_p);
}

void fdtd_get_velocity_dims(const AcousticFDTDState* st, int* Nvx, int* Nvy, int* Nvz)
{   // acoustic_fdtd.cpp:1399-1407
    if (!Nvx || !Nvy || !Nvz) return;
    if (!st) { *Nvx = *Nvy = *Nvz = 0; return; }
    *Nvx = (st->Nx - 1) * st->Ny * st->Nz;
    *Nvy = st->Nx * (st->Ny - 1) * st->Nz;
    *Nvz = st->Nx * st->Ny * (st->Nz - 1);
}

static int get_velocity(AcousticFDTDState* st, int f, float* out, int out_len)
{
    if (!st || !out) return FDTD_ERR_NULL;
    FieldShape s = field_shape(st, f);
    if (out_len != s.nxa * s.nya * s.nza) return FDTD_ERR_DIM;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    return copy_block(st, const_cast<float*>(field_ptr(st, f)), out, s.nxa, s.nya, s.nza, false);
}

int fdtd_get_velocity_x(const AcousticFDTDState* st, float* out, int out_len)
{   // acoustic_fdtd.cpp:1409-1415
    return get_velocity(const_cast<AcousticFDTDState*>(st), 1, out, out_len);
}
int fdtd_get_velocity_y(const AcousticFDTDState* st, float* out, int out_len)
{   // acoustic_fdtd.cpp:1417-1423
    return get_velocity(const_cast<AcousticFDTDState*>(st), 2, out, out_len);
}
int fdtd_get_velocity_z(const AcousticFDTDState* st, float* out, int out_len)
{   // acoustic_fdtd.cpp:1425-1431
    return get_velocity(const_cast<AcousticFDTDState*>(st), 3, out, out_len);
}

int fdtd_sample_velocity(const AcousticFDTDState* cst, int n_rec, const float* rec_xyz, float* out_vx,
                         float* out_vy, float* out_vz)
{   // acoustic_fdtd.cpp:1522-1538
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !rec_xyz || !out_vx || !out_vy || !out_vz) return FDTD_ERR_NULL;
    if (n_rec <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc;
    if ((rc = direct_samples(st, 1, n_rec, rec_xyz, out_vx))) return rc;
    if ((rc = direct_samples(st, 2, n_rec, rec_xyz, out_vy))) return rc;
    return direct_samples(st, 3, n_rec, rec_xyz, out_vz);
}

int fdtd_get_surface_emission(const AcousticFDTDState* cst, int n_surf, const float* surf_xyz,
                              const float* surf_normals, float* out_P, float* out_vn)
{   // acoustic_fdtd.cpp:1540-1563
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !surf_xyz || !surf_normals || !out_P || !out_vn) return FDTD_ERR_NULL;
    if (n_surf <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    std::vector<float> vx(n_surf), vy(n_surf), vz(n_surf);
    int rc;
    if ((rc = direct_samples(st, 0, n_surf, surf_xyz, out_P))) return rc;
    if ((rc = direct_samples(st, 1, n_surf, surf_xyz, vx.data()))) return rc;
    if ((rc = direct_samples(st, 2, n_surf, surf_xyz, vy.data()))) return rc;
    if ((rc = direct_samples(st, 3, n_surf, surf_xyz, vz.data()))) return rc;
    for (int s = 0; s < n_surf; ++s)
        out_vn[s] = vx[s] * surf_normals[3 * s] + vy[s] * surf_normals[3 * s + 1] +
                    vz[s] * surf_normals[3 * s + 2];
    return FDTD_OK;
}

/* ================================ extensions ================================ */

int fdtd_b200_field_layout(int Nx, int Ny, int Nz, int* row_stride, size_t* field_bytes)
{
    if (Nx <= 0 || Ny <= 0 || Nz <= 0) return FDTD_ERR_ARG;
    int sz = (Nz + kRowAlign - 1) / kRowAlign * kRowAlign;
    if (row_stride) *row_stride = sz;
    if (field_bytes) *field_bytes = (size_t)Nx * Ny * sz * sizeof(float);
    return FDTD_OK;
}

int fdtd_b200_set_face_absorption(AcousticFDTDState* st, const float* a6)
{
    if (!st || !a6) return FDTD_ERR_NULL;
    for (int q = 0; q < 6; ++q)
        if (!(a6[q] > 0.0f) || !std::isfinite(a6[q])) return FDTD_ERR_ARG;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    memcpy(st->a6, a6, sizeof(st->a6));
    return build_tables(st);
}

int fdtd_b200_add_pressure(AcousticFDTDState* st, int cell_index, float amp)
{
    if (!st) return FDTD_ERR_NULL;
    if (cell_index < 0 || cell_index >= st->N || amp == 0.0f) return 0;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    Deposit d = make_deposit(st, cell_index);
    if (d.n == 0) return 0;
    CK(launch_deposit(d, nullptr, 0, amp, st->P(), st->stream));
    ++st->launches;
    return d.n;
}

int fdtd_b200_set_point_source(AcousticFDTDState* st, int cell_index, const float* signal,
                               int n_signal)
{
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaStreamSynchronize(st->stream));
    cudaFree(st->d_ps_sig);
    st->d_ps_sig = nullptr;
    st->ps_n = 0;
    st->ps = Deposit{};
    st->ps_cell = -1;
    st->ps_done_step = -1;
    if (n_signal <= 0 || !signal) return FDTD_OK;
    if (cell_index < 0 || cell_index >= st->N) return FDTD_ERR_ARG;
    CK(cudaMalloc(&st->d_ps_sig, sizeof(float) * n_signal));
    CK(cudaMemcpy(st->d_ps_sig, signal, sizeof(float) * n_signal, cudaMemcpyHostToDevice));
    st->ps_n = n_signal;
    st->ps_cell = cell_index;
    st->ps = make_deposit(st, cell_index);
    return FDTD_OK;
}

int fdtd_b200_set_receivers(AcousticFDTDState* st, int n_rec, const int* idx8, const float* wgt8,
                            int capacity)
{
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaStreamSynchronize(st->stream));
    cudaFree(st->d_rec_idx); cudaFree(st->d_rec_w); cudaFree(st->d_trace);
    st->d_rec_idx = nullptr; st->d_rec_w = nullptr; st->d_trace = nullptr;
    st->n_rec = 0; st->trace_cap = 0; st->trace_len = 0;
    if (n_rec <= 0) return FDTD_OK;
    if (!idx8 || !wgt8 || capacity <= 0) return FDTD_ERR_ARG;
    std::vector<long long> pidx((size_t)n_rec * 8);
    for (size_t q = 0; q < pidx.size(); ++q) {
        pidx[q] = ref_to_pad(st, 0, idx8[q]);
        if (pidx[q] < 0) return FDTD_ERR_ARG;
    }
    CK(cudaMalloc(&st->d_rec_idx, pidx.size() * sizeof(long long)));
    CK(cudaMalloc(&st->d_rec_w, pidx.size() * sizeof(float)));
    CK(cudaMalloc(&st->d_trace, (size_t)n_rec * capacity * sizeof(float)));
    CK(cudaMemcpy(st->d_rec_idx, pidx.data(), pidx.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(st->d_rec_w, wgt8, pidx.size() * sizeof(float), cudaMemcpyHostToDevice));
    st->n_rec = n_rec;
    st->trace_cap = capacity;
    return FDTD_OK;
}

int fdtd_b200_get_traces(AcousticFDTDState* st, float* out, int out_len, int* n_recorded)
{
    if (!st || !out) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    const long long need = (long long)st->trace_len * st->n_rec;
    if (out_len < need) return FDTD_ERR_DIM;
    if (need > 0)
        CK(cudaMemcpyAsync(out, st->d_trace, (size_t)need * sizeof(float), cudaMemcpyDeviceToHost,
                           st->stream));
    CK(cudaStreamSynchronize(st->stream));
    if (n_recorded) *n_recorded = st->trace_len;
    st->trace_len = 0;
    return FDTD_OK;
}

int fdtd_b200_set_stream(AcousticFDTDState* st, void* stream)
{
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaStreamSynchronize(st->stream));
    st->stream = stream ? (cudaStream_t)stream : st->own_stream;
    return FDTD_OK;
}

void* fdtd_b200_get_stream(const AcousticFDTDState* st) { return st ? (void*)st->stream : nullptr; }

int fdtd_b200_step_async(AcousticFDTDState* st, int n_steps)
{
    if (!st) return FDTD_ERR_NULL;
    if (n_steps <= 0) return FDTD_OK;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc = FDTD_OK;
    for (int s = 0; s < n_steps && rc == FDTD_OK; ++s) rc = one_step(st, false, true);
    const int rc_rec = flush_record(st);
    return rc != FDTD_OK ? rc : rc_rec;
}

int fdtd_b200_synchronize(AcousticFDTDState* st)
{
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaMemcpyAsync(st->h_status, st->d_status, kStatusWords * sizeof(unsigned),
                       cudaMemcpyDeviceToHost, st->stream));
    CK(cudaStreamSynchronize(st->stream));
    if (int rc = check_timeout(st)) return rc;
    if (st->h_status[kStatusLatch] != 0xFFFFFFFFu) {
        fprintf(stderr, "[fdtd_pressure] UNSTABLE at step=%u (async)\n", st->h_status[kStatusLatch]);
        CK(cudaMemsetAsync(st->d_status, 0xFF, kStatusWords * sizeof(unsigned), st->stream));
        CK(cudaStreamSynchronize(st->stream));
        return FDTD_ERR_UNSTABLE;
    }
    return FDTD_OK;
}

int fdtd_b200_debug_hold_load(AcousticFDTDState* st, int plane, int wait_us)
{
    if (!st) return FDTD_ERR_NULL;
    if (plane < -1 || plane >= st->Nx || wait_us < 0 || (unsigned)wait_us > kWaitUs) return FDTD_ERR_ARG;
    st->hold_plane = plane < 0 ? kNoPlane : plane;
    st->wait_us = wait_us > 0 ? (unsigned)wait_us : kWaitUs;
    return FDTD_OK;
}

int fdtd_b200_set_kernel(AcousticFDTDState* st, int mode)
{
    if (!st) return FDTD_ERR_NULL;
    if (mode < 0 || mode > 2) return FDTD_ERR_ARG;
    if (mode == 2 && !fused_eligible(st) && !fused_walled_ok(st)) return FDTD_ERR_ARG;
    st->kernel_mode = mode;
    return FDTD_OK;
}

int fdtd_b200_get_kernel(const AcousticFDTDState* st)
{
    if (!st) return FDTD_ERR_NULL;
    return use_fused(st) ? 2 : 1;
}

int fdtd_b200_device_fields(const AcousticFDTDState* st, void** out5)
{
    if (!st || !out5) return FDTD_ERR_NULL;
    out5[0] = st->P(); out5[1] = st->Pn();
    out5[2] = st->V(0); out5[3] = st->V(1); out5[4] = st->V(2);
    return FDTD_OK;
}

// The step counter, the stability check's rotating phase and the step whose
// source sample is already in P (a batch deposits the next step's sample
// ahead): with the current P and V fields they are the whole state a later
// step depends on (the source schedule and receivers are configuration), so
// a snapshot of the fields plus these three resumes a room exactly.
int fdtd_b200_get_progress(const AcousticFDTDState* st, int* step_count, int* check_phase, int* deposited_step)
{
    if (!st || !step_count || !check_phase || !deposited_step) return FDTD_ERR_NULL;
    *step_count = st->step_count;
    *check_phase = st->stab_phase;
    *deposited_step = st->ps_done_step;
    return FDTD_OK;
}

int fdtd_b200_set_progress(AcousticFDTDState* st, int step_count, int check_phase, int deposited_step)
{
    if (!st) return FDTD_ERR_NULL;
    if (step_count < 0 || check_phase < 0 || check_phase >= kCheckStride || deposited_step < -1)
        return FDTD_ERR_ARG;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaStreamSynchronize(st->stream));
    st->step_count = step_count;
    st->stab_phase = check_phase;
    st->ps_done_step = deposited_step;
    return FDTD_OK;
}

int fdtd_b200_profile(AcousticFDTDState* st, int enable)
{
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaStreamSynchronize(st->stream));
    if (enable && st->prof.ev.empty()) {
        st->prof.ev.resize(2 * 8192);
        for (auto& e : st->prof.ev) CK(cudaEventCreate(&e));
    }
    st->prof.used = 0;
    st->prof_launches = 0;
    st->prof_kernels = 0;
    st->prof_on = enable != 0;
    return FDTD_OK;
}

int fdtd_b200_profile_read(AcousticFDTDState* st, double* total_ms, long long* launches,
                           long long* kernel_launches)
{
    if (!st) return FDTD_ERR_NULL;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    CK(cudaStreamSynchronize(st->stream));
    double tot = 0.0;
    for (int q = 0; q + 1 < st->prof.used; q += 2) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, st->prof.ev[q], st->prof.ev[q + 1]));
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = st->prof_launches;
    if (kernel_launches) *kernel_launches = st->prof_kernels;
    return FDTD_OK;
}

long long fdtd_b200_launch_count(const AcousticFDTDState* st) { return st ? st->launches : 0; }

const char* fdtd_b200_last_error(void) { return g_err; }

}  // extern "C"

/* ================= allocation-free pressure sampler ================= */
/*
 * Some callers cannot allocate: the instrument co-evolver samples its
 * microphones once per audio sample from a real-time audio callback, where a
 * cudaMalloc/cudaMallocHost may block on driver locks for an unbounded time.
 * fdtd_sample_pressure_precomputed grows per-handle scratch on demand; this
 * variant stages its inputs and result in one fixed device array instead.
 * It ends with a synchronisation of the handle's stream (so it also waits for
 * steps queued there, and cannot be called while that stream is captured).
 * The array's device address is looked up on the first call on a device and
 * kept; a cudaDeviceReset of that device makes the kept address stale.
 */
namespace {

constexpr int kNoAllocMaxReceivers = 4096;   // receivers per call (8 taps each)

struct NoAllocScratch {
    int idx[kNoAllocMaxReceivers * 8];
    float wgt[kNoAllocMaxReceivers * 8];
    float out[kNoAllocMaxReceivers];
};

// 272 KB on every device that loads this library, held until the process exits.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Same sum as k_wsum for the precomputed sampler (products in tap order, the
// first one starting the running sum), with the reference's flat indices
// turned into device offsets here rather than on the host.
__global__ void k_sample_noalloc(NoAllocScratch* s, const float* __restrict__ p, Grid g, int n_rec)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rec) return;
    float acc = 0.0f;
    for (int t = 0; t < 8; ++t) {
        const int flat = s->idx[8 * r + t];   // validated in [0, N) on the host
        const int k = flat % g.nz;
        const int ij = flat / g.nz;
        const long long off = ((long long)(ij / g.ny) * g.ny + ij % g.ny) * g.sz + k;
        const float v = fmul(s->wgt[8 * r + t], p[off]);
        acc = t == 0 ? v : fadd(acc, v);
    }
    s->out[r] = acc;
}

std::mutex g_noalloc_mu;
NoAllocScratch* g_noalloc_addr[64];   // device address of the array, per device

}  // namespace

extern "C" int fdtd_b200_sample_pressure_noalloc(const AcousticFDTDState* cst, int n_rec,
                                                 const int* idx8, const float* wgt8, float* out_p)
{
    AcousticFDTDState* st = const_cast<AcousticFDTDState*>(cst);
    if (!st || !idx8 || !wgt8 || !out_p) return FDTD_ERR_NULL;
    if (n_rec <= 0) return FDTD_OK;
    if (n_rec > kNoAllocMaxReceivers) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        snprintf(g_err, sizeof(g_err),
                 "fdtd_b200_sample_pressure_noalloc: %d receivers exceed the maximum of %d per call",
                 n_rec, kNoAllocMaxReceivers);
        return FDTD_ERR_ARG;
    }
    for (long long q = 0; q < (long long)n_rec * 8; ++q)
        if (idx8[q] < 0 || idx8[q] >= st->N) {
            std::lock_guard<std::mutex> lk(g_err_mu);
            snprintf(g_err, sizeof(g_err),
                     "fdtd_b200_sample_pressure_noalloc: tap %lld (receiver %lld) has index %d outside [0, %lld)",
                     q, q / 8, idx8[q], (long long)st->N);
            return FDTD_ERR_ARG;
        }
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    if (st->device < 0 || st->device >= 64) return FDTD_ERR_ARG;
    NoAllocScratch* s;
    {
        // first call on this device (its device current): look up the array's address
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[st->device]) {
            void* addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess) {
                set_err(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
                return FDTD_ERR_CUDA;
            }
            g_noalloc_addr[st->device] = static_cast<NoAllocScratch*>(addr);
        }
        s = g_noalloc_addr[st->device];
    }
    const size_t taps = (size_t)n_rec * 8;
    CK(cudaMemcpyAsync(s->idx, idx8, taps * sizeof(int), cudaMemcpyHostToDevice, st->stream));
    CK(cudaMemcpyAsync(s->wgt, wgt8, taps * sizeof(float), cudaMemcpyHostToDevice, st->stream));
    k_sample_noalloc<<<(n_rec + 127) / 128, 128, 0, st->stream>>>(s, st->P(), st->g, n_rec);
    CK(cudaGetLastError());
    ++st->launches;
    CK(cudaMemcpyAsync(out_p, s->out, (size_t)n_rec * sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    CK(cudaStreamSynchronize(st->stream));
    return FDTD_OK;
}

/* ====================== batched stepping (continuous batching) ====================== */

struct FdtdB200Batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<AcousticFDTDState*> members;
    std::vector<BatchMember> h;          // host copy of the device descriptors
    std::vector<int> cur0, cv0;          // member buffer parities when the batch was set
    BatchMember* d_members = nullptr;
    int cap_members = 0;
    int* d_item_member = nullptr;
    int cap_items = 0;
    int total_items = 0;
    BatchHeader* d_hdr = nullptr;
    unsigned* d_status = nullptr;
    unsigned h_status[kStatusWords];
    int grid_ctas = 0;                   // persistent CTAs of the current tile shape
    int grid_ctas_shape[2] = {0, 0};
    int shape = 0;                       // 0: 8 x 128 tiles, 1: 16 x 64 (fdtd_b200_batch_set_tile)
    int set_shape = 0;                   // the shape the current member set was built with
    int seg_planes = 0;                  // planes per work item, 0 = automatic
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    long long launches = 0;
};

namespace {

void batch_drop_graph(FdtdB200Batch* b)
{
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = 0;
}

// Pull the device step counters back into the member handles.
int batch_pull(FdtdB200Batch* b, int* steps_out, int* status_out)
{
    const int n = (int)b->members.size();
    if (n > 0)
        CK(cudaMemcpyAsync(b->h.data(), b->d_members, sizeof(BatchMember) * n, cudaMemcpyDeviceToHost,
                           b->stream));
    CK(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(b->h_status), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    for (int q = 0; q < n; ++q) {
        AcousticFDTDState* st = b->members[q];
        const BatchMember& m = b->h[q];
        const int done = m.step - m.step0;
        st->step_count = m.step;
        st->cur = b->cur0[q] ^ (done & 1);
        st->cv = b->cv0[q] ^ (done & 1);
        st->trace_len = std::min(m.trace0 + done, m.trace_cap);
        const int n_chk = m.step / kCheckPeriod - m.step0 / kCheckPeriod;
        st->stab_phase = (m.phase0 + n_chk) % kCheckStride;
        // the epilogue deposited step m.step's sample unless the member stopped unstable
        if (m.step < m.limit && m.step < m.ps_n && m.unstable == 0xFFFFFFFFu) st->ps_done_step = m.step;
        if (steps_out) steps_out[q] = m.step;
        if (status_out) status_out[q] = (m.unstable != 0xFFFFFFFFu) ? FDTD_ERR_UNSTABLE : FDTD_OK;
    }
    if (b->h_status[kStatusTimeout] != 0xFFFFFFFFu) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        snprintf(g_err, sizeof(g_err), "batched step: a tile's load wait timed out (block %u)",
                 b->h_status[kStatusTimeout]);
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

}  // namespace

extern "C" {

FdtdB200Batch* fdtd_b200_batch_create(int device)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return nullptr;
    }
    FdtdB200Batch* b = new FdtdB200Batch();
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) { delete b; return nullptr; }
    b->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&b->d_hdr, sizeof(BatchHeader)) != cudaSuccess ||
        cudaMemset(b->d_hdr, 0, sizeof(BatchHeader)) != cudaSuccess ||
        cudaMalloc(&b->d_status, sizeof(unsigned) * kStatusWords) != cudaSuccess ||
        cudaMemset(b->d_status, 0xFF, sizeof(unsigned) * kStatusWords) != cudaSuccess ||
        fused_batch_slots(0, &b->grid_ctas_shape[0]) != cudaSuccess ||
        fused_batch_slots(1, &b->grid_ctas_shape[1]) != cudaSuccess) {
        set_err(cudaGetLastError(), "fdtd_b200_batch_create");
        fdtd_b200_batch_destroy(b);
        return nullptr;
    }
    return b;
}

void fdtd_b200_batch_destroy(FdtdB200Batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    cudaFree(b->d_members);
    cudaFree(b->d_item_member);
    cudaFree(b->d_hdr);
    cudaFree(b->d_status);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int fdtd_b200_batch_set_tile(FdtdB200Batch* b, int tile_k)
{
    if (!b) return FDTD_ERR_NULL;
    if (tile_k != 128 && tile_k != 64) return FDTD_ERR_ARG;
    b->shape = tile_k == 64 ? 1 : 0;
    batch_drop_graph(b);
    return FDTD_OK;
}

int fdtd_b200_batch_set_segment(FdtdB200Batch* b, int planes)
{
    if (!b) return FDTD_ERR_NULL;
    if (planes < 0) return FDTD_ERR_ARG;
    b->seg_planes = planes;
    batch_drop_graph(b);
    return FDTD_OK;
}

int fdtd_b200_batch_set(FdtdB200Batch* b, AcousticFDTDState* const* members, const int* limits, int n)
{
    if (!b || (n > 0 && (!members || !limits))) return FDTD_ERR_NULL;
    if (n < 0) return FDTD_ERR_ARG;
    CK(cudaSetDevice(b->device));
    // the previous members' progress goes back to their handles first
    if (!b->members.empty()) {
        int rc = batch_pull(b, nullptr, nullptr);
        if (rc) return rc;
    }
    b->members.clear();
    b->h.clear();
    b->cur0.clear();
    b->cv0.clear();
    b->total_items = 0;
    if (n == 0) {
        BatchHeader hz{0, 0, 0};
        CK(cudaMemcpyAsync(b->d_hdr, &hz, sizeof(hz), cudaMemcpyHostToDevice, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        return FDTD_OK;
    }
    for (int q = 0; q < n; ++q) {
        AcousticFDTDState* st = members[q];
        if (!st) return FDTD_ERR_NULL;
        if (st->device != b->device || !fused_eligible(st) || limits[q] < st->step_count) return FDTD_ERR_ARG;
    }
    int tj, tk;
    b->set_shape = b->shape;
    b->grid_ctas = b->grid_ctas_shape[b->set_shape];
    fused_tile_shape(b->set_shape, &tj, &tk);
    std::vector<int> item_member;
    for (int q = 0; q < n; ++q) {
        AcousticFDTDState* st = members[q];
        CK(cudaStreamSynchronize(st->stream));
        if (!st->v[st->cv ^ 1][0]) {
            int rc = alloc_second_velocity_set(st);
            if (rc) return rc;
            CK(cudaStreamSynchronize(st->stream));
        }
        if (!st->fcache) st->fcache = fused_cache_create();
        // the member's next source sample goes in before its first batched step
        if (st->ps_n > 0 && st->step_count < st->ps_n && st->ps.n > 0 && st->ps_done_step != st->step_count &&
            st->step_count < limits[q]) {
            CK(launch_deposit(st->ps, st->d_ps_sig, st->step_count, 0.0f, st->P(), b->stream));
            ++b->launches;
            st->ps_done_step = st->step_count;
        }
        BatchMember m;
        memset(&m, 0, sizeof(m));
        const float* v0[3] = {st->V(0), st->V(1), st->V(2)};
        const float* v1[3] = {st->v[st->cv ^ 1][0], st->v[st->cv ^ 1][1], st->v[st->cv ^ 1][2]};
        CK(fused_maps(st->fcache, st->g, st->P(), v0, m.maps[0], b->set_shape));
        CK(fused_maps(st->fcache, st->g, st->Pn(), v1, m.maps[1], b->set_shape));
        m.g = st->g;
        m.cf = st->cf;
        m.tb = st->tb;
        m.p[0] = st->P();
        m.p[1] = st->Pn();
        for (int c = 0; c < 3; ++c) {
            m.v[0][c] = st->V(c);
            m.v[1][c] = st->v[st->cv ^ 1][c];
        }
        m.step = m.step0 = st->step_count;
        m.limit = limits[q];
        const int tiles_j = (st->Ny + tj - 1) / tj, tiles_k = (st->Nz + tk - 1) / tk;
        m.tiles_k = tiles_k;
        m.tiles = tiles_j * tiles_k;
        int segs;
        if (b->seg_planes > 0) {
            segs = (st->Nx + b->seg_planes - 1) / b->seg_planes;
        } else {
            // automatic: about one wave of work items for this member alone
            segs = std::max(1, b->grid_ctas / m.tiles);
        }
        segs = std::min(segs, st->Nx);
        m.seg_len = (st->Nx + segs - 1) / segs;
        segs = (st->Nx + m.seg_len - 1) / m.seg_len;
        m.items_begin = (int)item_member.size();
        for (int t = 0; t < m.tiles * segs; ++t) item_member.push_back(q);
        m.ps = st->ps;
        m.ps_sig = st->d_ps_sig;
        m.ps_n = (st->ps.n > 0 && st->d_ps_sig) ? st->ps_n : 0;
        m.n_rec = st->n_rec;
        m.trace0 = st->trace_len;
        m.trace_cap = st->trace_cap;
        m.rec_idx = st->d_rec_idx;
        m.rec_w = st->d_rec_w;
        m.trace = st->d_trace;
        m.n_cells = st->N;
        m.phase0 = st->stab_phase;
        m.unstable = 0xFFFFFFFFu;
        b->members.push_back(st);
        b->h.push_back(m);
        b->cur0.push_back(st->cur);
        b->cv0.push_back(st->cv);
    }
    // descriptor arrays keep their addresses (and a captured graph stays valid)
    // until a set outgrows them
    if (n > b->cap_members) {
        batch_drop_graph(b);
        cudaFree(b->d_members);
        b->d_members = nullptr;
        b->cap_members = 0;
        const int cap = std::max(n, std::max(64, 2 * b->cap_members));
        CK(cudaMalloc(&b->d_members, sizeof(BatchMember) * cap));
        b->cap_members = cap;
    }
    if ((int)item_member.size() > b->cap_items) {
        batch_drop_graph(b);
        cudaFree(b->d_item_member);
        b->d_item_member = nullptr;
        b->cap_items = 0;
        const int cap = std::max((int)item_member.size(), 1 << 15);
        CK(cudaMalloc(&b->d_item_member, sizeof(int) * cap));
        b->cap_items = cap;
    }
    b->total_items = (int)item_member.size();
    BatchHeader hh{n, b->total_items, 0};
    CK(cudaMemcpyAsync(b->d_members, b->h.data(), sizeof(BatchMember) * n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->d_item_member, item_member.data(), sizeof(int) * item_member.size(),
                       cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->d_hdr, &hh, sizeof(hh), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return FDTD_OK;
}

int fdtd_b200_batch_step(FdtdB200Batch* b, int n_steps, int use_graph)
{
    if (!b) return FDTD_ERR_NULL;
    if (n_steps <= 0 || b->members.empty()) return FDTD_OK;
    CK(cudaSetDevice(b->device));
    if (!use_graph) {
        for (int s = 0; s < n_steps; ++s) {
            CK(launch_fused_batch_step(b->d_members, b->d_hdr, b->d_item_member, b->d_status,
                                       b->grid_ctas, b->cap_members, b->stream, b->set_shape));
            b->launches += 2;
        }
        return FDTD_OK;
    }
    if (!b->graph || b->graph_steps != n_steps) {
        batch_drop_graph(b);
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int s = 0; s < n_steps && e == cudaSuccess; ++s)
            e = launch_fused_batch_step(b->d_members, b->d_hdr, b->d_item_member, b->d_status,
                                        b->grid_ctas, b->cap_members, b->stream, b->set_shape);
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            set_err(e != cudaSuccess ? e : e2, "batch graph capture");
            return FDTD_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->graph = nullptr;
            set_err(e, "cudaGraphInstantiate");
            return FDTD_ERR_CUDA;
        }
        b->graph_steps = n_steps;
    }
    CK(cudaGraphLaunch(b->graph, b->stream));
    b->launches += 2LL * n_steps;
    return FDTD_OK;
}

int fdtd_b200_batch_sync(FdtdB200Batch* b, int* steps_out, int* status_out)
{
    if (!b) return FDTD_ERR_NULL;
    CK(cudaSetDevice(b->device));
    return batch_pull(b, steps_out, status_out);
}

long long fdtd_b200_batch_launch_count(const FdtdB200Batch* b) { return b ? b->launches : 0; }

}  // extern "C"

// ---------------------------------------------------------------- co-evolver substep
// The uniform co-evolver's per-substep calls (acoustic_coevolver.cpp:2072-2121:
// fdtd_inject_bridge_drive, fdtd_inject_plate_force, fdtd_step(st, 1),
// fdtd_sample_plate_displacement_batch) as one call with one stream
// synchronisation.  With an active plate, fdtd_step must wait for the plate
// guard before the velocity and pressure updates; here those kernels (and the
// consumption of the plate forces and the 256-step check) are gated on the
// device by the plate status word instead, the saddle samples are taken from
// the new displacement, and the host reads status and samples together.  If
// the plate update failed, the host undoes its own bookkeeping of the step
// (buffer rotation, step count, trace row, check phase), which leaves the
// handle exactly as fdtd_step leaves it on that failure.
namespace {

constexpr size_t kSubstepGraphs = 12;   // 2 pressure parities x 3 plate rotations, with / without forces

int substep_plate(AcousticFDTDState* st, int n_saddle, float* out)
{
    cudaStream_t s = st->stream;
    if (st->ps_n > 0 && st->step_count < st->ps_n && st->ps.n > 0 && st->ps_done_step != st->step_count) {
        CK(launch_deposit(st->ps, st->d_ps_sig, st->step_count, 0.0f, st->P(), s));
        ++st->launches;
        st->ps_done_step = st->step_count;
    }
    const bool ext_was_pending = st->ext_pending;
    const bool ext_left = st->dev_ext_nonzero && !ext_was_pending;   // not expected; zeroed in full then
    if (st->ext_pending) st->dev_ext_nonzero = true;
    const bool ext_zero = st->dev_ext_nonzero;
    // the pending forces as (node, value) pairs: only their nodes are nonzero on
    // the host, and only they are written to (and later cleared on) the device
    const int n_pack = ext_was_pending ? (int)st->ext_nodes.size() : 0;
    for (int q = 0; q < n_pack; ++q) {
        const int pidx = st->ext_nodes[q];
        int bits;
        memcpy(&bits, &st->h_ext[pidx], 4);
        st->h_ext_pack[q] = make_int2(pidx, bits);
    }
    if (n_saddle > 0)   // the saddle taps (staged by the caller) go up before the step's work
        if (int rc2 = upload_taps(st, (size_t)n_saddle * 4, s)) return rc2;
    const int wp0 = st->wi_prev, wc0 = st->wi_cur, wt0 = st->wi_tmp;
    const bool record = st->n_rec > 0 && st->trace_len < st->trace_cap;
    const int step1 = st->step_count + 1;
    const bool checked = (step1 & (kCheckPeriod - 1)) == 0;
    const int phase0 = st->stab_phase;
    const int trace0 = st->trace_len;
    const unsigned* gate = st->d_status;
    float* const P = st->P();
    float* const Pn = st->Pn();
    const bool hf = st->has_frac;
    // The substep's device work in stream order: the plate update (its guard
    // gates everything after it), the step as if the plate succeeded (the
    // plate's new displacement is d_w[wt0], the previous one d_w[wc0]), then
    // the saddle samples and the status words to the host.
    auto issue = [&]() -> int {
        if (n_pack > 0) {
            CK(cudaMemcpyAsync(st->d_ext_pack, st->h_ext_pack, (size_t)n_pack * sizeof(int2), cudaMemcpyHostToDevice, s));
            CK(launch_ext_scatter(st->d_ext, st->d_ext_pack, n_pack, s));
        }
        CK(cudaMemsetAsync(st->d_status + kStatusPlate, 0xFF, sizeof(unsigned), s));
        CK(launch_plate_step(st->n_act, st->d_act, st->d_nb13, st->d_above, st->d_below, st->d_w[wc0], st->d_w[wp0],
                             st->d_w[wt0], st->d_ext, P, st->pc, st->d_status, s));
        if (ext_left) CK(launch_zero_gated(st->d_ext, st->N_plate, gate, s));
        PlateFaces pf;   // plate face velocities and the consumed forces' zeroing, in the velocity pass
        pf.code = st->d_plate_code;
        pf.w = st->d_w[wt0];
        pf.wp = st->d_w[wc0];
        pf.inv_dt = st->cf.inv_dt;
        pf.iz = st->plate_iz;
        if (!ext_left && ext_zero) {
            pf.ext = st->d_ext;
            pf.pack = st->d_ext_pack;
            pf.m = n_pack;
        }
        CK(launch_velocity_general(st->g, st->cf, st->tb, P, st->V(0), st->V(1), st->V(2), st->d_frac[0],
                                   st->d_frac[1], st->d_frac[2], s, gate, &pf));
        CK(launch_pressure_general(st->g, st->cf, st->tb, P, Pn, st->V(0), st->V(1), st->V(2),
                                   hf ? st->d_frac[0] : nullptr, hf ? st->d_frac[1] : nullptr,
                                   hf ? st->d_frac[2] : nullptr, st->d_solid, s, gate));
        if (record)
            CK(launch_wsum(Pn, st->d_rec_idx, st->d_rec_w, st->n_rec, 8, 0,
                           st->d_trace + (size_t)trace0 * st->n_rec, s));
        if (checked) {
            CK(cudaMemsetAsync(st->d_status + kStatusCell, 0xFF, sizeof(unsigned), s));
            CK(launch_check(st->g, Pn, st->N, phase0, st->d_status, step1, s, gate));
        }
        if (n_saddle > 0) {
            CK(launch_wsum(st->d_w[wt0], st->d_sidx, st->d_sw, n_saddle, 4, 0, st->d_sout, s));
            CK(cudaMemcpyAsync(st->h_sout, st->d_sout, (size_t)n_saddle * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        CK(cudaMemcpyAsync(st->h_status, st->d_status, kStatusWords * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        return FDTD_OK;
    };
    const long long n_launch = 3 + (n_pack > 0 ? 1 : 0) + (ext_left ? 1 : 0) + (record ? 1 : 0) + (checked ? 1 : 0) +
                               (n_saddle > 0 ? 1 : 0);
    bool issued = false;
    if (!record && !checked) {
        // The same work recurs every substep with one of a few pointer sets:
        // replay it as a cached CUDA graph (one launch instead of about ten).
        SubstepKey k;
        memset(&k, 0, sizeof k);
        k.stream = s;
        k.p = P; k.pn = Pn; k.v0 = st->V(0); k.v1 = st->V(1); k.v2 = st->V(2);
        k.w_cur = st->d_w[wc0]; k.w_prev = st->d_w[wp0]; k.w_tmp = st->d_w[wt0];
        for (int c2 = 0; c2 < 3; ++c2) k.frac[c2] = st->d_frac[c2];
        k.ext = st->d_ext; k.h_ext = st->h_ext; k.solid = st->d_solid;
        k.pack = st->d_ext_pack; k.h_pack = st->h_ext_pack; k.n_pack = n_pack;
        k.sidx = st->d_sidx; k.sw = st->d_sw; k.sout = st->d_sout; k.h_sout = st->h_sout;
        k.status = st->d_status; k.h_status = st->h_status;
        k.g = st->g; k.cf = st->cf; k.tb = st->tb; k.pc = st->pc;
        k.n_act = st->n_act; k.n_plate = st->N_plate; k.n_saddle = n_saddle;
        k.ext_copy = ext_was_pending; k.ext_zero = ext_zero; k.has_frac = hf;
        SubstepGraph* hit = nullptr;
        for (auto& sg : st->sgraphs)
            if (memcmp(&sg.key, &k, sizeof k) == 0) hit = &sg;
        const cudaError_t e_begin = hit ? cudaSuccess : cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e_begin != cudaSuccess) cudaGetLastError();   // e.g. the legacy default stream: no capture
        if (!hit && e_begin == cudaSuccess) {
            const int rc_issue = issue();
            cudaGraph_t graph = nullptr;
            const cudaError_t e_end = cudaStreamEndCapture(s, &graph);
            cudaGraphExec_t exec = nullptr;
            const cudaError_t e_inst = (rc_issue == FDTD_OK && e_end == cudaSuccess)
                                           ? cudaGraphInstantiate(&exec, graph, 0) : cudaErrorUnknown;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();   // a capture that failed leaves its error behind; the direct path follows
            if (e_inst == cudaSuccess) {
                if (st->sgraphs.size() >= kSubstepGraphs) {
                    cudaGraphExecDestroy(st->sgraphs.front().exec);
                    st->sgraphs.erase(st->sgraphs.begin());
                }
                SubstepGraph sg;
                sg.key = k;
                sg.exec = exec;
                sg.launches = n_launch;
                st->sgraphs.push_back(sg);
                hit = &st->sgraphs.back();
            }
        }
        if (hit) {
            CK(cudaGraphLaunch(hit->exec, s));
            issued = true;
        }
    }
    if (!issued)
        if (int rc_issue = issue()) return rc_issue;
    st->launches += n_launch;
    // the bookkeeping of a step whose plate update succeeded (undone below if not)
    st->wi_prev = wc0;
    st->wi_cur = wt0;
    st->wi_tmp = wp0;
    st->cur ^= 1;
    st->step_count = step1;
    if (record) ++st->trace_len;
    if (checked) st->stab_phase = (phase0 + 1) % kCheckStride;
    CK(cudaStreamSynchronize(s));

    const unsigned bad = st->h_status[kStatusPlate];
    if (bad != 0xFFFFFFFFu) {   // the plate guard fired: undo the bookkeeping of the gated step
        st->cur ^= 1;
        --st->step_count;
        st->wi_prev = wp0;
        st->wi_cur = wc0;
        st->wi_tmp = wt0;
        st->trace_len = trace0;
        if (checked) st->stab_phase = phase0;
        const int pidx = st->h_act[bad];
        float wn = NAN;
        cudaMemcpy(&wn, st->d_w[st->wi_tmp] + pidx, sizeof(float), cudaMemcpyDeviceToHost);
        fprintf(stderr, "[fdtd_plate] UNSTABLE step=%d plate_node=%d (%d,%d) w_new=%.3g m (limit 0.02 m)\n",
                st->step_count, pidx, pidx / st->Ny, pidx % st->Ny, (double)wn);
        fflush(stderr);
        return FDTD_ERR_UNSTABLE;   // pending forces stay, as after fdtd_step
    }
    st->dev_ext_nonzero = false;    // consumed by the gated zeroing
    if (ext_was_pending) clear_ext_host(st);
    if (checked) {
        if (int rc2 = check_timeout(st)) return rc2;
        const unsigned cell = st->h_status[kStatusCell];
        if (cell != 0xFFFFFFFFu) {
            report_unstable_cell(st, cell);
            CK(cudaMemsetAsync(st->d_status + kStatusLatch, 0xFF, sizeof(unsigned), s));
            return FDTD_ERR_UNSTABLE;
        }
    }
    if (n_saddle > 0) memcpy(out, st->h_sout, (size_t)n_saddle * sizeof(float));
    return FDTD_OK;
}

}  // namespace

extern "C" int fdtd_b200_substep(AcousticFDTDState* st, const float* cell_drives, float drive_scale,
                                 int n_force, const int* force_idx, const float* force_wgt,
                                 float force_total_N, int n_saddle, const int* saddle_idx4,
                                 const float* saddle_wgt4, float* out_saddle_w)
{
    if (!st) return FDTD_ERR_NULL;
    if (n_saddle < 0) return FDTD_ERR_ARG;
    if (n_saddle > 0 && (!saddle_idx4 || !saddle_wgt4 || !out_saddle_w)) return FDTD_ERR_NULL;
    for (long long q = 0; q < (long long)n_saddle * 4; ++q)
        if (saddle_idx4[q] < 0 || saddle_idx4[q] >= st->N_plate) return FDTD_ERR_ARG;
    if (dev_guard(st)) return FDTD_ERR_CUDA;
    int rc;
    if (cell_drives && (rc = fdtd_inject_bridge_drive(st, cell_drives, drive_scale))) return rc;
    if (n_force > 0 && (rc = fdtd_inject_plate_force(st, n_force, force_idx, force_wgt, force_total_N)))
        return rc;
    if (st->n_act == 0) {   // no plate guard: fdtd_step(st, 1) does not wait here
        if ((rc = one_step(st, true))) return rc;
        return n_saddle > 0 ? fdtd_sample_plate_displacement_batch(st, n_saddle, saddle_idx4, saddle_wgt4,
                                                                    out_saddle_w)
                            : FDTD_OK;
    }
    if (n_saddle > 0) {
        if ((rc = ensure_scratch(st, (size_t)n_saddle * 4))) return rc;
        for (long long q = 0; q < (long long)n_saddle * 4; ++q) {
            st->h_sidx[q] = saddle_idx4[q];
            st->h_sw[q] = saddle_wgt4[q];
        }
    }
    return substep_plate(st, n_saddle, out_saddle_w);
}
