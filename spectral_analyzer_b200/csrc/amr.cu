/*
 * amr.cu — the AMR pressure backend on the GPU (include/acoustic_amr_b200.h).
 *
 * Drop-in for the reference's topology-driven AMR stepper
 * (csrc/kernels/acoustic_amr.cpp behind csrc/include/acoustic_amr.h): explicit
 * pressure cells joined by velocity faces, each face with an area, open
 * fraction and centre distance; a Kirchhoff plate coupled through ragged
 * face lists; graded absorbing borders; inverse-distance microphones.
 *
 * Device layout (HBM, structure of arrays, float32/int32):
 *   cells  p, P_damp, P_src_coeff, cell_inv_denom, zero flag (wall/plate),
 *          CSR of incident faces (starts, face index, signed flux weight);
 *   faces  v, V_damp, 1/distance, neg/pos cell, plate boundary code, and for
 *          gradient order 8 the 8-slot Fornberg stencil (cell, coefficient);
 *   plate  three displacement buffers rotated per step, external force,
 *          per-node CSR of the cells above and below.
 * One step = three kernels: k_amr_velocity (face gather; the plate's face
 * velocities are written in the same pass), k_amr_pressure (CSR divergence
 * and pressure update, wall/plate cells zeroed, divergence check fused),
 * k_amr_plate (Kirchhoff plate, force buffer cleared).  A diverged step
 * latches its index in a status word; the later kernels of the window skip.
 *
 * Arithmetic is the reference's, operation for operation, with separately
 * rounded float operations (__fadd_rn/__fmul_rn/__fdiv_rn on the device,
 * -ffp-contract=off on the host): velocity (acoustic_amr.cpp:1129-1151),
 * plate face velocity (:1050-1072), divergence and pressure (:1157-1169),
 * wall cells (:1172-1173), plate (:939-1048), checks (:1182-1192).
 * Create-time coefficients are computed on the host exactly as amr_create,
 * amr_set_border_condition, amr_setup_plate and amr_setup_mic_samplers do
 * (:680-895, :1318-1410, :1412-1532, :1647-1760), then uploaded once.
 */
#include "acoustic_amr_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace {

constexpr int kSW = 4;            // stencil half-width (cells each side) of gradient order 8
constexpr int kSW2 = 2 * kSW;
constexpr unsigned kNone = 0xFFFFFFFFu;

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

// ---------------------------------------------------------------- errors
std::mutex g_err_mu;
char g_err[512] = "";
thread_local std::string g_stage = "ok";
thread_local std::string g_msg;
std::atomic<int> g_prog_active{0}, g_prog_done{0}, g_prog_total{0};

void set_err(const char* what, cudaError_t e)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    snprintf(g_err, sizeof(g_err), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
}

#define AK(expr)                                   \
    do {                                           \
        cudaError_t e_ = (expr);                   \
        if (e_ != cudaSuccess) {                   \
            set_err(#expr, e_);                    \
            return AMR_B200_ERR_CUDA;              \
        }                                          \
    } while (0)

template <class T>
cudaError_t upload(T** d, const std::vector<T>& h)
{
    if (*d) cudaFree(*d);
    *d = nullptr;
    if (h.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(d, h.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// ---------------------------------------------------------------- kernels
struct PlateDev {
    const float* w;      // current displacement
    const float* wp;     // previous
    float* wn;           // next (written by the plate step)
    float* ext;          // external force, cleared by the plate step
    float dt;
};

// Velocity of every face; plate faces take the plate velocity instead
// (the reference overwrites them after the update, acoustic_amr.cpp:1050-1072).
template <int ORDER>
__global__ void k_amr_velocity(int n_faces, const float* __restrict__ p, float* __restrict__ v,
                               const float* __restrict__ vdamp, const float* __restrict__ inv_d,
                               const int* __restrict__ fneg, const int* __restrict__ fpos,
                               const int* __restrict__ s_cells, const float* __restrict__ s_coeff,
                               const int* __restrict__ bc, const int* __restrict__ bc_flat, PlateDev pl,
                               float dt_over_rho, const unsigned* __restrict__ status, unsigned step)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces || *status < step) return;
    const int code = bc ? bc[f] : -1;
    if (code >= 0) {   // plate face: +v_plate above, -v_plate below
        const int flat = bc_flat[code >> 1];
        const float vp = fd(fs(pl.w[flat], pl.wp[flat]), pl.dt);
        v[f] = (code & 1) ? -vp : vp;
        return;
    }
    float grad;
    if (ORDER == 8) {
        grad = 0.0f;
        const int* sc = s_cells + (size_t)f * kSW2;
        const float* sw = s_coeff + (size_t)f * kSW2;
#pragma unroll
        for (int k = 0; k < kSW2; ++k) grad = fa(grad, fm(sw[k], p[sc[k]]));
    } else {
        grad = fm(fs(p[fpos[f]], p[fneg[f]]), inv_d[f]);
    }
    v[f] = fm(fs(v[f], fm(dt_over_rho, grad)), vdamp[f]);
}

// Divergence and pressure of every cell, wall/plate cells zeroed, and the
// divergence check of this step (non-finite anywhere; |p| > 2e3 on steps
// whose count is a multiple of 256).
__global__ void k_amr_pressure(int n_cells, float* __restrict__ p, const float* __restrict__ v,
                               const float* __restrict__ pdamp, const float* __restrict__ psrc,
                               const float* __restrict__ inv_den, const int* __restrict__ cstart,
                               const int* __restrict__ cface, const float* __restrict__ cw,
                               const unsigned char* __restrict__ zero, float bulk,
                               unsigned* __restrict__ status, unsigned step, int check_max)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells || *status < step) return;
    float out = 0.0f;
    if (!zero[c]) {
        float d = 0.0f;
        const int k1 = cstart[c + 1];
        for (int k = cstart[c]; k < k1; ++k) d = fa(d, fm(cw[k], v[cface[k]]));
        out = fs(fm(p[c], pdamp[c]), fm(fm(fm(bulk, d), inv_den[c]), psrc[c]));
    }
    p[c] = out;
    if (!isfinite(out) || (check_max && fabsf(out) > 2e3f)) atomicMin(status, step);
}

// 13-point biharmonic of a plate buffer at (i, j), zero outside the plate.
__device__ __forceinline__ float biharmonic(const float* w, int i, int j, int nx, int ny, float idx4)
{
    auto W = [&](int a, int b) -> float { return (a < 0 || a >= nx || b < 0 || b >= ny) ? 0.0f : w[a * ny + b]; };
    float s = fa(fa(fa(W(i - 2, j), W(i + 2, j)), W(i, j - 2)), W(i, j + 2));
    s = fa(s, fm(2.0f, fa(fa(fa(W(i - 1, j - 1), W(i - 1, j + 1)), W(i + 1, j - 1)), W(i + 1, j + 1))));
    s = fs(s, fm(8.0f, fa(fa(fa(W(i - 1, j), W(i + 1, j)), W(i, j - 1)), W(i, j + 1))));
    s = fa(s, fm(20.0f, W(i, j)));
    return fm(s, idx4);
}

struct PlateCoefs {
    int nx, ny;
    float dx, idx4, dt2, inv_rh, damp_fwd, damp_bwd, cD0, cDp;
};

// One plate step: thread per plate node; active nodes (their last entry in
// the caller's list) integrate, every node's force is cleared.
__global__ void k_amr_plate(int n_nodes, const int* __restrict__ node_entry, const int* __restrict__ a_start,
                            const float* __restrict__ a_wgt, const int* __restrict__ a_cell,
                            const int* __restrict__ b_start, const float* __restrict__ b_wgt,
                            const int* __restrict__ b_cell, const int* __restrict__ cell_above,
                            const int* __restrict__ cell_below, const float* __restrict__ p, PlateDev pl,
                            PlateCoefs k, const unsigned* __restrict__ status, unsigned step)
{
    const int flat = blockIdx.x * blockDim.x + threadIdx.x;
    if (flat >= n_nodes || *status < step) return;
    const int n = node_entry[flat];
    if (n >= 0) {
        float pa = 0.0f, pb = 0.0f;
        if (a_start[n + 1] > a_start[n]) {
            for (int q = a_start[n]; q < a_start[n + 1]; ++q) pa = fa(pa, fm(a_wgt[q], p[a_cell[q]]));
        } else if (cell_above[n] >= 0) {
            pa = p[cell_above[n]];
        }
        if (b_start[n + 1] > b_start[n]) {
            for (int q = b_start[n]; q < b_start[n + 1]; ++q) pb = fa(pb, fm(b_wgt[q], p[b_cell[q]]));
        } else if (cell_below[n] >= 0) {
            pb = p[cell_below[n]];
        }
        const float f_acou = fm(fm(fs(pb, pa), k.dx), k.dx);
        const int i = flat / k.ny, j = flat % k.ny;
        const float l4w = biharmonic(pl.w, i, j, k.nx, k.ny, k.idx4);
        const float l4wp = biharmonic(pl.wp, i, j, k.nx, k.ny, k.idx4);
        const float rhs = fa(fs(fa(f_acou, pl.ext[flat]), fm(k.cD0, l4w)), fm(k.cDp, l4wp));
        pl.wn[flat] = fd(fa(fm(k.damp_bwd, fs(fm(2.0f, pl.w[flat]), pl.wp[flat])), fm(fm(k.dt2, k.inv_rh), rhs)),
                         k.damp_fwd);
    }
    pl.ext[flat] = 0.0f;
}

__global__ void k_amr_add(float* p, int idx, float value) { p[idx] = fa(p[idx], value); }

// Samples of the plate (4-tap batch, or one weighted sum), in tap order.
__global__ void k_amr_plate_taps(const float* __restrict__ w, int n_out, int taps, const int* __restrict__ idx,
                                 const float* __restrict__ wgt, float* __restrict__ out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_out) return;
    float s = 0.0f;
    for (int t = 0; t < taps; ++t) s = fa(s, fm(wgt[q * taps + t], w[idx[q * taps + t]]));
    out[q] = s;
}

// Microphones: pressure from the cell stencil, velocity from the face stencil.
__global__ void k_amr_mics(int n_mics, const float* __restrict__ p, const float* __restrict__ v,
                           const int* __restrict__ ps, const int* __restrict__ pc, const float* __restrict__ pw,
                           const int* __restrict__ vs, const int* __restrict__ vf, const float* __restrict__ wx,
                           const float* __restrict__ wy, const float* __restrict__ wz, float* __restrict__ out)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_mics) return;
    float sp = 0.0f;
    for (int k = ps[m]; k < ps[m + 1]; ++k) sp = fa(sp, fm(pw[k], p[pc[k]]));
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int k = vs[m]; k < vs[m + 1]; ++k) {
        const float vv = v[vf[k]];
        sx = fa(sx, fm(wx[k], vv));
        sy = fa(sy, fm(wy[k], vv));
        sz = fa(sz, fm(wz[k], vv));
    }
    out[m] = sp;
    out[n_mics + m] = sx;
    out[2 * n_mics + m] = sy;
    out[3 * n_mics + m] = sz;
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ================================================================ state
struct AcousticAMRState {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_cells = 0, n_faces = 0, order = 2;
    double c = 343.0, rho = 1.21, dt = 0.0;
    int step_count = 0;               // steps launched (a pending window may still be rolled back)
    int pend0 = 0, pend_n = 0;        // steps queued since the last wait: [pend0, pend0 + pend_n)
    long long launches = 0;

    // host copies used by set-up functions (double inputs, as the reference keeps them)
    std::vector<double> centers, volumes, open_vol, face_area, face_open, face_dist;
    std::vector<int> cell_type, face_neg, face_pos, acoustic;
    std::vector<int> csr_start, csr_face;
    std::vector<float> csr_w;

    // device
    float *d_p = nullptr, *d_v = nullptr, *d_vdamp = nullptr, *d_inv_d = nullptr;
    float *d_pdamp = nullptr, *d_psrc = nullptr, *d_inv_den = nullptr, *d_cw = nullptr, *d_scoef = nullptr;
    int *d_neg = nullptr, *d_pos = nullptr, *d_cstart = nullptr, *d_cface = nullptr, *d_scell = nullptr;
    unsigned char* d_zero = nullptr;
    unsigned* d_status = nullptr;
    float* d_scratch = nullptr;       // staging of sampler weights and results (2 x scratch_n)
    int* d_iscratch = nullptr;        // staging of sampler indices (scratch_n)
    size_t scratch_n = 0;

    // plate
    bool plate = false;
    int pnx = 0, pny = 0, p_nodes = 0, n_act = 0;
    PlateCoefs pk{};
    std::vector<int> act_flat;
    float* d_w[3] = {nullptr, nullptr, nullptr};
    int wi = 0;                       // d_w[wi] current, d_w[(wi+2)%3] previous, d_w[(wi+1)%3] next
    float* d_ext = nullptr;
    int *d_node_entry = nullptr, *d_astart = nullptr, *d_acell = nullptr, *d_bstart = nullptr, *d_bcell = nullptr;
    int *d_cabove = nullptr, *d_cbelow = nullptr, *d_bc = nullptr, *d_bc_flat = nullptr;
    float *d_awgt = nullptr, *d_bwgt = nullptr;
    float* h_ext = nullptr;           // pinned: forces injected since the last step, in call order
    bool ext_pending = false;
    std::vector<int> bridge_idx, neck_idx;
    std::vector<float> bridge_wgt, neck_wgt;

    // microphones
    int n_mics = 0;
    int *d_mps = nullptr, *d_mpc = nullptr, *d_mvs = nullptr, *d_mvf = nullptr;
    float *d_mpw = nullptr, *d_mwx = nullptr, *d_mwy = nullptr, *d_mwz = nullptr;

    // profiling
    bool prof = false;
    std::vector<cudaEvent_t> ev;
    size_t ev_used = 0;
    double prof_ms = 0;
    long long prof_steps = 0;

    float* cur_w() const { return d_w[wi]; }
    float* prev_w() const { return d_w[(wi + 2) % 3]; }
    float* next_w() const { return d_w[(wi + 1) % 3]; }
};

namespace {

void free_all(AcousticAMRState* st)
{
    void* ptrs[] = {st->d_p, st->d_v, st->d_vdamp, st->d_inv_d, st->d_pdamp, st->d_psrc, st->d_inv_den,
                    st->d_cw, st->d_scoef, st->d_neg, st->d_pos, st->d_cstart, st->d_cface, st->d_scell,
                    st->d_zero, st->d_status, st->d_scratch, st->d_iscratch, st->d_w[0], st->d_w[1],
                    st->d_w[2], st->d_ext, st->d_node_entry, st->d_astart, st->d_acell, st->d_bstart,
                    st->d_bcell, st->d_cabove, st->d_cbelow, st->d_bc, st->d_bc_flat, st->d_awgt,
                    st->d_bwgt, st->d_mps, st->d_mpc, st->d_mvs, st->d_mvf, st->d_mpw, st->d_mwx,
                    st->d_mwy, st->d_mwz};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (st->h_ext) cudaFreeHost(st->h_ext);
    for (cudaEvent_t e : st->ev) cudaEventDestroy(e);
    if (st->stream) cudaStreamDestroy(st->stream);
}

int guard(const AcousticAMRState* st)
{
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return -1;
    if (cur != st->device && cudaSetDevice(st->device) != cudaSuccess) return -1;
    return 0;
}

int ensure_scratch(AcousticAMRState* st, size_t n)
{
    if (n <= st->scratch_n) return 0;
    if (st->d_scratch) cudaFree(st->d_scratch);
    if (st->d_iscratch) cudaFree(st->d_iscratch);
    st->d_scratch = nullptr;
    st->d_iscratch = nullptr;
    st->scratch_n = 0;
    AK(cudaMalloc(&st->d_scratch, 2 * n * sizeof(float)));
    AK(cudaMalloc(&st->d_iscratch, n * sizeof(int)));
    st->scratch_n = n;
    return 0;
}

// amr_create's input checks (acoustic_amr.cpp:275-325).
int validate(int n_cells, const double* cc, const double* cv, const double* ov, const uint8_t* ct, int n_faces,
             const int32_t* fn, const int32_t* fp, const double* fa_, const double* fo, const double* fdist,
             double c, double rho, double min_dx)
{
    if (n_cells <= 0 || n_faces <= 0) return SK_ERR_DIM_MISMATCH;
    if (!cc || !cv || !ov || !ct || !fn || !fp || !fa_ || !fo || !fdist) return SK_ERR_NULL_STATE;
    if (c <= 0.0 || rho <= 0.0 || min_dx <= 0.0) return SK_ERR_DIM_MISMATCH;
    for (int i = 0; i < n_cells; ++i)
        if (!(cv[i] > 0.0) || ov[i] < 0.0 || ov[i] > 1.0 || ct[i] > 3) return SK_ERR_DIM_MISMATCH;
    for (int f = 0; f < n_faces; ++f) {
        if (fn[f] < 0 || fn[f] >= n_cells || fp[f] < 0 || fp[f] >= n_cells || fn[f] == fp[f])
            return SK_ERR_DIM_MISMATCH;
        if (!(fa_[f] > 0.0) || fo[f] < 0.0 || fo[f] > 1.0 || !(fdist[f] > 0.0)) return SK_ERR_DIM_MISMATCH;
    }
    return SK_OK;
}

// ------------------------------------------------ gradient order 8 stencil
// Fornberg (1988, SIAM Review 30:4) weights of the first derivative at xi for
// nodes x[0..n), in single precision with the recurrence's operation order
// (as the reference's fornberg_d1, acoustic_amr.cpp:398-428).
void fornberg_first(const float* x, int n, float xi, float* w)
{
    float c0[kSW2] = {}, c1[kSW2] = {};   // weights of derivative order 0 and 1 per node
    float prod_prev = 1.0f;
    c0[0] = 1.0f;
    for (int a = 1; a < n; ++a) {
        float prod = 1.0f;
        const float xa = x[a] - xi;
        for (int b = 0; b < a; ++b) {
            const float diff = x[a] - x[b];
            prod *= diff;
            if (b == a - 1) {
                const float r = prod_prev / prod;
                c1[a] = r * (1.0f * c0[a - 1] - xa * c1[a - 1]);
                c0[a] = r * (-xa) * c0[a - 1];
            }
            c1[b] = (xa * c1[b] - 1.0f * c0[b]) / diff;
            c0[b] = xa * c0[b] / diff;
        }
        prod_prev = prod;
    }
    for (int k = 0; k < n; ++k) w[k] = c1[k];
}

struct Topo {
    const AcousticAMRState* st;
    std::vector<int> nb_pos[3], nb_neg[3];
};

float proj(const AcousticAMRState* st, int ci, const float d[3])
{
    return (float)(st->centers[3 * ci] * d[0] + st->centers[3 * ci + 1] * d[1] + st->centers[3 * ci + 2] * d[2]);
}

// Axis neighbour tables: a face whose centre-to-centre direction is within
// acos(0.9) of an axis links its cells along that axis; a second, different
// link on the same side marks the side ambiguous (acoustic_amr.cpp:329-384).
void build_axis_neighbours(Topo& t)
{
    const AcousticAMRState* st = t.st;
    const int nc = st->n_cells;
    std::vector<unsigned char> sp[3], sn[3];
    for (int a = 0; a < 3; ++a) {
        t.nb_pos[a].assign(nc, -1);
        t.nb_neg[a].assign(nc, -1);
        sp[a].assign(nc, 0);
        sn[a].assign(nc, 0);
    }
    auto link = [](int& nb, unsigned char& s, int other) {
        if (s == 0) {
            nb = other;
            s = 1;
        } else if (s == 1 && nb != other) {
            nb = -1;
            s = 2;
        }
    };
    for (int f = 0; f < st->n_faces; ++f) {
        const int cn = st->face_neg[f], cp = st->face_pos[f];
        const float dx = (float)(st->centers[3 * cp] - st->centers[3 * cn]);
        const float dy = (float)(st->centers[3 * cp + 1] - st->centers[3 * cn + 1]);
        const float dz = (float)(st->centers[3 * cp + 2] - st->centers[3 * cn + 2]);
        const float len = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (len < 1e-15f) continue;
        const float ax = std::abs(dx / len), ay = std::abs(dy / len), az = std::abs(dz / len);
        if (std::max({ax, ay, az}) <= 0.9f) continue;
        const int a = (ax >= ay && ax >= az) ? 0 : (ay >= ax && ay >= az) ? 1 : 2;
        const float sd = a == 0 ? dx : a == 1 ? dy : dz;
        if (sd > 0.0f) {
            link(t.nb_pos[a][cn], sp[a][cn], cp);
            link(t.nb_neg[a][cp], sn[a][cp], cn);
        } else {
            link(t.nb_neg[a][cn], sn[a][cn], cp);
            link(t.nb_pos[a][cp], sp[a][cp], cn);
        }
    }
}

// Cells met walking from `seed` along `walk` (table lookups for axis-aligned
// walks, else the incident face best aligned with `walk`, > 0.5), stopping at
// walls, the plate, the domain edge or `depth` cells; positions are projected
// on `coord` relative to `face_proj` (acoustic_amr.cpp:444-547).
int walk_cells(const Topo& t, int seed, float face_proj, const float coord[3], const float walk[3], int depth,
               int* cells, float* xs)
{
    const AcousticAMRState* st = t.st;
    cells[0] = seed;
    xs[0] = proj(st, seed, coord) - face_proj;
    int found = 1, cur = seed;
    const float ax = std::abs(walk[0]), ay = std::abs(walk[1]), az = std::abs(walk[2]);
    int axis = -1;
    bool up = false;
    if (std::max({ax, ay, az}) > 0.9f) {
        if (ax >= ay && ax >= az) {
            axis = 0;
            up = walk[0] > 0.f;
        } else if (ay >= ax && ay >= az) {
            axis = 1;
            up = walk[1] > 0.f;
        } else {
            axis = 2;
            up = walk[2] > 0.f;
        }
    }
    auto solid = [&](int c) { return st->cell_type[c] == 1 || st->cell_type[c] == 2; };
    if (axis >= 0) {
        const std::vector<int>& tab = up ? t.nb_pos[axis] : t.nb_neg[axis];
        while (found < depth) {
            const int nb = tab[cur];
            if (nb < 0 || nb >= st->n_cells || solid(nb)) break;
            cells[found] = nb;
            xs[found] = proj(st, nb, coord) - face_proj;
            ++found;
            cur = nb;
        }
        return found;
    }
    while (found < depth) {
        int best = -1;
        float best_dot = 0.5f;
        for (int k = st->csr_start[cur]; k < st->csr_start[cur + 1]; ++k) {
            const int fk = st->csr_face[k];
            const float sg = (st->csr_w[k] > 0.f) ? +1.f : -1.f;
            const int a = st->face_neg[fk], b = st->face_pos[fk];
            const float dx = (float)(st->centers[3 * b] - st->centers[3 * a]);
            const float dy = (float)(st->centers[3 * b + 1] - st->centers[3 * a + 1]);
            const float dz = (float)(st->centers[3 * b + 2] - st->centers[3 * a + 2]);
            const float len = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (len < 1e-15f) continue;
            const float dot = sg * (dx * walk[0] + dy * walk[1] + dz * walk[2]) / len;
            if (dot > best_dot) {
                const int nb = (sg > 0.f) ? b : a;
                if (nb >= 0 && nb < st->n_cells && !solid(nb)) {
                    best_dot = dot;
                    best = nb;
                }
            }
        }
        if (best < 0) break;
        cells[found] = best;
        xs[found] = proj(st, best, coord) - face_proj;
        ++found;
        cur = best;
    }
    return found;
}

// Per face: with four cells on each side, Fornberg weights over all eight;
// otherwise the two-cell difference (acoustic_amr.cpp:549-629).  Unused slots
// keep cell 0 and weight 0.
void build_stencil(AcousticAMRState* st, std::vector<int>& sc, std::vector<float>& sw)
{
    Topo t;
    t.st = st;
    build_axis_neighbours(t);
    const int nf = st->n_faces;
    sc.assign((size_t)nf * kSW2, 0);
    sw.assign((size_t)nf * kSW2, 0.0f);
    g_prog_total.store(nf);
    g_prog_done.store(0);
    g_prog_active.store(1);
    for (int f = 0; f < nf; ++f) {
        const int cn = st->face_neg[f], cp = st->face_pos[f];
        const float dxf = (float)(st->centers[3 * cp] - st->centers[3 * cn]);
        const float dyf = (float)(st->centers[3 * cp + 1] - st->centers[3 * cn + 1]);
        const float dzf = (float)(st->centers[3 * cp + 2] - st->centers[3 * cn + 2]);
        const float len = std::sqrt(dxf * dxf + dyf * dyf + dzf * dzf);
        if (len >= 1e-15f) {
            const float dir[3] = {dxf / len, dyf / len, dzf / len};
            const float back[3] = {-dir[0], -dir[1], -dir[2]};
            const float fp = 0.5f * (proj(st, cn, dir) + proj(st, cp, dir));
            int nc_[kSW], pc_[kSW];
            float nx_[kSW], px_[kSW];
            const int nn = walk_cells(t, cn, fp, dir, back, kSW, nc_, nx_);
            const int np = walk_cells(t, cp, fp, dir, dir, kSW, pc_, px_);
            if (nn == kSW && np == kSW) {
                float xs[kSW2], w[kSW2];
                for (int k = 0; k < kSW; ++k) {
                    xs[k] = nx_[kSW - 1 - k];
                    xs[kSW + k] = px_[k];
                }
                fornberg_first(xs, kSW2, 0.0f, w);
                for (int k = 0; k < kSW; ++k) {
                    sc[(size_t)f * kSW2 + k] = nc_[k];          // walk order from the face outward
                    sw[(size_t)f * kSW2 + k] = w[kSW - 1 - k];
                    sc[(size_t)f * kSW2 + kSW + k] = pc_[k];
                    sw[(size_t)f * kSW2 + kSW + k] = w[kSW + k];
                }
            } else if (nn + np >= 2) {
                const float inv = st->face_dist[f] > 0.0 ? 1.0f / (float)st->face_dist[f] : 0.0f;
                sc[(size_t)f * kSW2] = cn;
                sw[(size_t)f * kSW2] = -inv;
                sc[(size_t)f * kSW2 + kSW] = cp;
                sw[(size_t)f * kSW2 + kSW] = inv;
            }
        }
        g_prog_done.store(f + 1);
    }
    g_prog_active.store(0);
}

void prof_mark(AcousticAMRState* st)
{
    if (!st->prof) return;
    if (st->ev_used >= st->ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        st->ev.push_back(e);
    }
    cudaEventRecord(st->ev[st->ev_used++], st->stream);
}

void prof_collect(AcousticAMRState* st)
{
    for (size_t q = 0; q + 1 < st->ev_used; q += 2) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, st->ev[q], st->ev[q + 1]) == cudaSuccess) {
            st->prof_ms += ms;
            ++st->prof_steps;
        }
    }
    st->ev_used = 0;
}

int launch_steps(AcousticAMRState* st, int n_steps)
{
    if (st->pend_n == 0) st->pend0 = st->step_count;
    if (st->ext_pending) {
        AK(cudaMemcpyAsync(st->d_ext, st->h_ext, st->p_nodes * sizeof(float), cudaMemcpyHostToDevice,
                           st->stream));
        AK(cudaStreamSynchronize(st->stream));   // the pinned buffer is reused by the next injection
        std::fill(st->h_ext, st->h_ext + st->p_nodes, 0.0f);
        st->ext_pending = false;
    }
    const float dt = (float)st->dt;
    const float dt_over_rho = dt / (float)st->rho;
    const float bulk = (float)(st->rho * st->c * st->c * st->dt);
    for (int s = 0; s < n_steps; ++s) {
        const unsigned step = (unsigned)(st->step_count + s);
        PlateDev pl{};
        if (st->plate) pl = PlateDev{st->cur_w(), st->prev_w(), st->next_w(), st->d_ext, dt};
        prof_mark(st);
        if (st->order == 8)
            k_amr_velocity<8><<<blocks(st->n_faces, 256), 256, 0, st->stream>>>(
                st->n_faces, st->d_p, st->d_v, st->d_vdamp, st->d_inv_d, st->d_neg, st->d_pos, st->d_scell,
                st->d_scoef, st->plate ? st->d_bc : nullptr, st->d_bc_flat, pl, dt_over_rho, st->d_status, step);
        else
            k_amr_velocity<2><<<blocks(st->n_faces, 256), 256, 0, st->stream>>>(
                st->n_faces, st->d_p, st->d_v, st->d_vdamp, st->d_inv_d, st->d_neg, st->d_pos, nullptr, nullptr,
                st->plate ? st->d_bc : nullptr, st->d_bc_flat, pl, dt_over_rho, st->d_status, step);
        AK(cudaGetLastError());
        k_amr_pressure<<<blocks(st->n_cells, 256), 256, 0, st->stream>>>(
            st->n_cells, st->d_p, st->d_v, st->d_pdamp, st->d_psrc, st->d_inv_den, st->d_cstart, st->d_cface,
            st->d_cw, st->d_zero, bulk, st->d_status, step, (step & 0xFFu) == 0 ? 1 : 0);
        AK(cudaGetLastError());
        st->launches += 2;
        if (st->plate) {
            k_amr_plate<<<blocks(st->p_nodes, 128), 128, 0, st->stream>>>(
                st->p_nodes, st->d_node_entry, st->d_astart, st->d_awgt, st->d_acell, st->d_bstart, st->d_bwgt,
                st->d_bcell, st->d_cabove, st->d_cbelow, st->d_p, pl, st->pk, st->d_status, step);
            AK(cudaGetLastError());
            ++st->launches;
            st->wi = (st->wi + 1) % 3;
        }
        prof_mark(st);
    }
    st->step_count += n_steps;
    st->pend_n += n_steps;
    return SK_OK;
}

// Wait for the queued steps; on a diverged step, roll the step count and the
// plate buffer rotation back to what the reference leaves (the failing step's
// plate update ran; its count was not advanced; later steps did not run).
int finish_steps(AcousticAMRState* st)
{
    AK(cudaStreamSynchronize(st->stream));
    if (st->prof) prof_collect(st);
    const int n = st->pend_n;
    st->pend_n = 0;
    unsigned status = kNone;
    AK(cudaMemcpy(&status, st->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (status == kNone) return SK_OK;
    const int ran = (int)status - st->pend0 + 1;   // plate updates executed in the window
    if (st->plate) st->wi = ((st->wi - n + ran) % 3 + 3) % 3;
    st->step_count = (int)status;
    AK(cudaMemset(st->d_status, 0xFF, sizeof(unsigned)));
    fprintf(stderr, "[amr_step] UNSTABLE step=%d (non-finite or |p| > 2e3 Pa)\n", st->step_count);
    return SK_ERR_DIVERGED;
}

int plate_taps(AcousticAMRState* st, int n_out, int taps, const int* idx, const float* wgt, float* out)
{
    if (n_out <= 0) return SK_OK;
    for (long long q = 0; q < (long long)n_out * taps; ++q)
        if (idx[q] < 0 || idx[q] >= st->p_nodes) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    const size_t m = (size_t)n_out * taps;
    if (ensure_scratch(st, std::max(m, (size_t)n_out))) return AMR_B200_ERR_CUDA;
    float* d_wgt = st->d_scratch;
    float* d_out = st->d_scratch + st->scratch_n;
    AK(cudaMemcpyAsync(st->d_iscratch, idx, m * sizeof(int), cudaMemcpyHostToDevice, st->stream));
    AK(cudaMemcpyAsync(d_wgt, wgt, m * sizeof(float), cudaMemcpyHostToDevice, st->stream));
    k_amr_plate_taps<<<blocks(n_out, 128), 128, 0, st->stream>>>(st->cur_w(), n_out, taps, st->d_iscratch, d_wgt,
                                                                 d_out);
    AK(cudaGetLastError());
    ++st->launches;
    AK(cudaMemcpyAsync(out, d_out, n_out * sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    AK(cudaStreamSynchronize(st->stream));
    return SK_OK;
}

}  // namespace

// ================================================================ C ABI
extern "C" {

AcousticAMRState* amr_create(int n_cells, const double* cc, const double* cv, const double* ov, const uint8_t* ct,
                             int n_faces, const int32_t* fn, const int32_t* fp, const double* fa_,
                             const double* fo, const double* fdist, double c, double rho, double min_dx,
                             int gradient_order)
{
    g_stage = "validate_inputs";
    g_msg.clear();
    if (validate(n_cells, cc, cv, ov, ct, n_faces, fn, fp, fa_, fo, fdist, c, rho, min_dx) != SK_OK) {
        g_msg = "input validation failed";
        return nullptr;
    }
    if (gradient_order != 2 && gradient_order != 8) {
        g_msg = "gradient_order must be 2 or 8";
        return nullptr;
    }
    g_stage = "state.init";
    auto* st = new (std::nothrow) AcousticAMRState();
    if (!st) {
        g_msg = "AcousticAMRState allocation failed";
        return nullptr;
    }
    try {
        cudaGetDevice(&st->device);
        st->n_cells = n_cells;
        st->n_faces = n_faces;
        st->c = c;
        st->rho = rho;
        st->order = gradient_order;
        st->dt = (gradient_order == 8 ? 0.10 : 0.77) * min_dx / (c * std::sqrt(3.0));
        st->centers.assign(cc, cc + 3 * (size_t)n_cells);
        st->volumes.assign(cv, cv + n_cells);
        st->open_vol.assign(ov, ov + n_cells);
        st->cell_type.assign(ct, ct + n_cells);
        st->face_neg.assign(fn, fn + n_faces);
        st->face_pos.assign(fp, fp + n_faces);
        st->face_area.assign(fa_, fa_ + n_faces);
        st->face_open.assign(fo, fo + n_faces);
        st->face_dist.assign(fdist, fdist + n_faces);
        for (int i = 0; i < n_cells; ++i)
            if ((ct[i] == 0 || ct[i] == 3) && ov[i] > 0.0) st->acoustic.push_back(i);
        if (st->acoustic.empty()) {
            g_stage = "acoustic_cells";
            g_msg = "no active acoustic cells after filtering";
            delete st;
            return nullptr;
        }
        g_stage = "coefficients";
        std::vector<float> inv_d(n_faces), flux(n_faces), inv_den(n_cells, 0.0f);
        for (int f = 0; f < n_faces; ++f) {
            inv_d[f] = 1.0f / (float)fdist[f];
            flux[f] = (float)(fa_[f] * fo[f]);
        }
        for (int i : st->acoustic) inv_den[i] = (float)(1.0 / (cv[i] * std::max(ov[i], 1e-12)));
        std::vector<unsigned char> zero(n_cells);
        for (int i = 0; i < n_cells; ++i) zero[i] = (ct[i] == 1 || ct[i] == 2) ? 1 : 0;
        // incident faces of each cell, in face order: +flux on the face's negative side, -flux on its positive side
        st->csr_start.assign(n_cells + 1, 0);
        for (int f = 0; f < n_faces; ++f) {
            st->csr_start[fn[f] + 1]++;
            st->csr_start[fp[f] + 1]++;
        }
        for (int i = 1; i <= n_cells; ++i) st->csr_start[i] += st->csr_start[i - 1];
        st->csr_face.resize(st->csr_start[n_cells]);
        st->csr_w.resize(st->csr_start[n_cells]);
        {
            std::vector<int> fill(n_cells, 0);
            for (int f = 0; f < n_faces; ++f) {
                const int ka = st->csr_start[fn[f]] + fill[fn[f]]++;
                st->csr_face[ka] = f;
                st->csr_w[ka] = +flux[f];
                const int kb = st->csr_start[fp[f]] + fill[fp[f]]++;
                st->csr_face[kb] = f;
                st->csr_w[kb] = -flux[f];
            }
        }
        std::vector<int> scell;
        std::vector<float> scoef;
        if (gradient_order == 8) {
            g_stage = "stencil.build";
            build_stencil(st, scell, scoef);
        }
        g_stage = "device";
        cudaError_t e = cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking);
        std::vector<float> ones_f(n_faces, 1.0f), ones_c(n_cells, 1.0f), zc(n_cells, 0.0f), zf(n_faces, 0.0f);
        if (e == cudaSuccess) e = upload(&st->d_p, zc);
        if (e == cudaSuccess) e = upload(&st->d_v, zf);
        if (e == cudaSuccess) e = upload(&st->d_vdamp, ones_f);
        if (e == cudaSuccess) e = upload(&st->d_inv_d, inv_d);
        if (e == cudaSuccess) e = upload(&st->d_pdamp, ones_c);
        if (e == cudaSuccess) e = upload(&st->d_psrc, ones_c);
        if (e == cudaSuccess) e = upload(&st->d_inv_den, inv_den);
        if (e == cudaSuccess) e = upload(&st->d_neg, st->face_neg);
        if (e == cudaSuccess) e = upload(&st->d_pos, st->face_pos);
        if (e == cudaSuccess) e = upload(&st->d_cstart, st->csr_start);
        if (e == cudaSuccess) e = upload(&st->d_cface, st->csr_face);
        if (e == cudaSuccess) e = upload(&st->d_cw, st->csr_w);
        if (e == cudaSuccess) e = upload(&st->d_zero, zero);
        if (e == cudaSuccess && gradient_order == 8) e = upload(&st->d_scell, scell);
        if (e == cudaSuccess && gradient_order == 8) e = upload(&st->d_scoef, scoef);
        if (e == cudaSuccess) e = cudaMalloc(&st->d_status, sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemset(st->d_status, 0xFF, sizeof(unsigned));
        if (e != cudaSuccess) {
            g_msg = std::string("CUDA: ") + cudaGetErrorString(e);
            set_err("amr_create", e);
            free_all(st);
            delete st;
            return nullptr;
        }
    } catch (const std::bad_alloc&) {
        g_msg = "std::bad_alloc at stage: " + g_stage;
        free_all(st);
        delete st;
        return nullptr;
    }
    g_stage = "ok";
    g_msg.clear();
    return st;
}

const char* amr_get_last_create_error_stage(void) { return g_stage.c_str(); }
const char* amr_get_last_create_error_message(void) { return g_msg.c_str(); }
int amr_get_create_progress_active(void) { return g_prog_active.load(); }
int amr_get_create_progress_done_faces(void) { return g_prog_done.load(); }
int amr_get_create_progress_total_faces(void) { return g_prog_total.load(); }

void amr_destroy(AcousticAMRState* st)
{
    if (!st) return;
    if (guard(st) == 0) {
        cudaStreamSynchronize(st->stream);
        free_all(st);
    }
    delete st;
}

int amr_step(AcousticAMRState* st, int n_steps)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (n_steps < 0) return SK_ERR_DIM_MISMATCH;
    if (n_steps == 0) return SK_OK;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    int rc = launch_steps(st, n_steps);
    if (rc != SK_OK) return rc;
    return finish_steps(st);
}

int amr_b200_step_async(AcousticAMRState* st, int n_steps)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (n_steps < 0) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    return launch_steps(st, n_steps);
}

int amr_b200_synchronize(AcousticAMRState* st)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    return finish_steps(st);
}

int amr_reset(AcousticAMRState* st)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaStreamSynchronize(st->stream));
    AK(cudaMemset(st->d_p, 0, st->n_cells * sizeof(float)));
    AK(cudaMemset(st->d_v, 0, st->n_faces * sizeof(float)));
    if (st->plate) {
        for (int q = 0; q < 3; ++q) AK(cudaMemset(st->d_w[q], 0, st->p_nodes * sizeof(float)));
        AK(cudaMemset(st->d_ext, 0, st->p_nodes * sizeof(float)));
        std::fill(st->h_ext, st->h_ext + st->p_nodes, 0.0f);
        st->ext_pending = false;
    }
    AK(cudaMemset(st->d_status, 0xFF, sizeof(unsigned)));
    st->step_count = 0;
    st->pend_n = 0;
    return SK_OK;
}

int amr_inject_pressure_nearest(AcousticAMRState* st, const double* xyz, float value)
{
    if (!st || !xyz) return SK_ERR_NULL_STATE;
    if (!std::isfinite(value)) return SK_ERR_DIVERGED;
    double best = 1e300;
    int bi = -1;
    for (int i : st->acoustic) {
        const double dx = st->centers[3 * i] - xyz[0], dy = st->centers[3 * i + 1] - xyz[1],
                     dz = st->centers[3 * i + 2] - xyz[2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < best) {
            best = d2;
            bi = i;
        }
    }
    if (bi < 0) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    k_amr_add<<<1, 1, 0, st->stream>>>(st->d_p, bi, value);
    AK(cudaGetLastError());
    ++st->launches;
    AK(cudaStreamSynchronize(st->stream));
    return SK_OK;
}

int amr_get_pressure(const AcousticAMRState* st, float* out, int n)
{
    if (!st || !out) return SK_ERR_NULL_STATE;
    if (n != st->n_cells) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaMemcpyAsync(out, st->d_p, n * sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    AK(cudaStreamSynchronize(st->stream));
    return SK_OK;
}

int amr_get_cell_centers(const AcousticAMRState* st, float* out, int n3)
{
    if (!st || !out) return SK_ERR_NULL_STATE;
    if (n3 < st->n_cells * 3) return SK_ERR_DIM_MISMATCH;
    for (int i = 0; i < 3 * st->n_cells; ++i) out[i] = (float)st->centers[i];
    return SK_OK;
}

int amr_get_velocity(const AcousticAMRState* st, float* out, int n)
{
    if (!st || !out) return SK_ERR_NULL_STATE;
    if (n != st->n_faces) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaMemcpyAsync(out, st->d_v, n * sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    AK(cudaStreamSynchronize(st->stream));
    return SK_OK;
}

double amr_get_dt(const AcousticAMRState* st) { return st ? st->dt : 0.0; }
int amr_get_step_count(const AcousticAMRState* st) { return st ? st->step_count : 0; }

// Nearest voxel per cell, last cell wins (acoustic_amr.cpp:1266-1294); the
// field is read back and scattered on the host (a display helper, not the step).
int amr_scatter_pressure_uniform(const AcousticAMRState* st, int Nx, int Ny, int Nz, const double bmin[3],
                                 const double bmax[3], float* out)
{
    if (!st || !out || !bmin || !bmax) return SK_ERR_NULL_STATE;
    if (Nx <= 0 || Ny <= 0 || Nz <= 0) return SK_ERR_DIM_MISMATCH;
    std::vector<float> p(st->n_cells);
    int rc = amr_get_pressure(st, p.data(), st->n_cells);
    if (rc != SK_OK) return rc;
    std::fill(out, out + (size_t)Nx * Ny * Nz, 0.0f);
    const double rx = Nx > 1 ? (Nx - 1) / (bmax[0] - bmin[0]) : 0.0;
    const double ry = Ny > 1 ? (Ny - 1) / (bmax[1] - bmin[1]) : 0.0;
    const double rz = Nz > 1 ? (Nz - 1) / (bmax[2] - bmin[2]) : 0.0;
    for (int i = 0; i < st->n_cells; ++i) {
        const int ix = (int)std::lround((st->centers[3 * i] - bmin[0]) * rx);
        const int iy = (int)std::lround((st->centers[3 * i + 1] - bmin[1]) * ry);
        const int iz = (int)std::lround((st->centers[3 * i + 2] - bmin[2]) * rz);
        if (ix < 0 || ix >= Nx || iy < 0 || iy >= Ny || iz < 0 || iz >= Nz) continue;
        out[(size_t)ix * (Ny * Nz) + (size_t)iy * Nz + iz] = p[i];
    }
    return SK_OK;
}

// Graded absorption of the PML-type cells and the damping it implies
// (acoustic_amr.cpp:1318-1410): cell alpha = sigma_max * norm^order with norm
// the depth into the layer; P_damp = exp(-s), the integrating factor
// (1 - exp(-s))/s of the source term, faces exp(-s_face dt) with the
// open-volume-weighted harmonic mean of their cells' alpha.
int amr_set_border_condition(AcousticAMRState* st, int mode, float sigma_order, float R, float Z, int n_pml,
                             const double* bmin, const double* bmax)
{
    (void)Z;
    if (!st || !bmin || !bmax) return SK_ERR_NULL_STATE;
    if (n_pml <= 0) return SK_OK;
    const float order = sigma_order > 0.0f ? sigma_order : 3.0f;
    const float dt_f = (float)st->dt;
    const int nc = st->n_cells, nf = st->n_faces;
    float sigma_max = 3.45f / (dt_f * (float)n_pml);
    if (mode == AMR_BORDER_ROOM_PANEL) {
        const float r = std::max(0.0f, std::min(1.0f, R));
        sigma_max *= (1.0f - r);
    }
    const double min_dx = st->dt * st->c * std::sqrt(3.0) / 0.77;
    const double depth = (double)n_pml * min_dx;
    std::vector<float> alpha(nc, 0.0f);
    for (int i = 0; i < nc; ++i) {
        if (st->cell_type[i] != 3) continue;
        const double x = st->centers[3 * i], y = st->centers[3 * i + 1], z = st->centers[3 * i + 2];
        double d = std::min({x - bmin[0], bmax[0] - x, y - bmin[1], bmax[1] - y, z - bmin[2], bmax[2] - z});
        d = std::max(d, 0.0);
        const float norm = (float)std::max(0.0, std::min(1.0, 1.0 - d / depth));
        alpha[i] = sigma_max * std::pow(norm, order);
    }
    std::vector<float> pdamp(nc), psrc(nc), vdamp(nf);
    for (int i = 0; i < nc; ++i) {
        const float s = alpha[i] * dt_f;
        pdamp[i] = std::exp(-s);
        psrc[i] = (s < 1e-6f) ? 1.0f - 0.5f * s : (1.0f - std::exp(-s)) / s;
    }
    for (int f = 0; f < nf; ++f) {
        const int a = st->face_neg[f], b = st->face_pos[f];
        const float vn = (float)st->open_vol[a], vp = (float)st->open_vol[b];
        const float den = vn + vp;
        const float sf = den > 0.f ? 2.0f * (vp * alpha[a] + vn * alpha[b]) / den : 0.5f * (alpha[a] + alpha[b]);
        vdamp[f] = std::exp(-sf * dt_f);
    }
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaStreamSynchronize(st->stream));
    AK(cudaMemcpy(st->d_pdamp, pdamp.data(), nc * sizeof(float), cudaMemcpyHostToDevice));
    AK(cudaMemcpy(st->d_psrc, psrc.data(), nc * sizeof(float), cudaMemcpyHostToDevice));
    AK(cudaMemcpy(st->d_vdamp, vdamp.data(), nf * sizeof(float), cudaMemcpyHostToDevice));
    return SK_OK;
}

int amr_setup_plate(AcousticAMRState* st, int pnx, int pny, float pdx, const float origin[3],
                    const uint8_t* active, float rho_h, float D, float aM, float bK, int n_act,
                    const int32_t* act_idx, const int32_t* a_start, const int32_t* a_idx, const float* a_wgt,
                    const int32_t* b_start, const int32_t* b_idx, const float* b_wgt, const int32_t* cell_above,
                    const int32_t* cell_below)
{
    (void)origin;
    if (!st) return SK_ERR_NULL_STATE;
    if (!active || !act_idx || !a_start || !b_start || !cell_above || !cell_below) return SK_ERR_NULL_STATE;
    if (pnx <= 0 || pny <= 0 || pdx <= 0.0f || rho_h <= 0.0f || D <= 0.0f || n_act < 0) return SK_ERR_DIM_MISMATCH;
    const int nodes = pnx * pny;
    int count = 0;
    for (int k = 0; k < nodes; ++k) count += active[k] ? 1 : 0;
    if (count != n_act) return SK_ERR_DIM_MISMATCH;
    for (int k = 0; k < a_start[n_act]; ++k)
        if (a_idx[k] < 0 || a_idx[k] >= st->n_faces) return SK_ERR_DIM_MISMATCH;
    for (int k = 0; k < b_start[n_act]; ++k)
        if (b_idx[k] < 0 || b_idx[k] >= st->n_faces) return SK_ERR_DIM_MISMATCH;
    for (int n = 0; n < n_act; ++n) {
        if (cell_above[n] != -1 && (cell_above[n] < 0 || cell_above[n] >= st->n_cells)) return SK_ERR_DIM_MISMATCH;
        if (cell_below[n] != -1 && (cell_below[n] < 0 || cell_below[n] >= st->n_cells)) return SK_ERR_DIM_MISMATCH;
        if (a_start[n + 1] == a_start[n] && cell_above[n] < 0) return SK_ERR_DIM_MISMATCH;
        if (b_start[n + 1] == b_start[n] && cell_below[n] < 0) return SK_ERR_DIM_MISMATCH;
        if (act_idx[n] < 0 || act_idx[n] >= nodes) return SK_ERR_DIM_MISMATCH;
    }
    // the cell on the air side of each coupling face: above faces have the
    // plate on their negative side, below faces on their positive side
    std::vector<int> acell(a_start[n_act]), bcell(b_start[n_act]);
    for (int k = 0; k < a_start[n_act]; ++k) acell[k] = st->face_pos[a_idx[k]];
    for (int k = 0; k < b_start[n_act]; ++k) bcell[k] = st->face_neg[b_idx[k]];
    // per plate node, its last entry in the list (a later entry overwrites an earlier one)
    std::vector<int> node_entry(nodes, -1);
    for (int n = 0; n < n_act; ++n) node_entry[act_idx[n]] = n;
    // plate boundary faces: entry*2 (+v above) or entry*2+1 (-v below); the last assignment wins
    std::vector<int> bc(st->n_faces, -1);
    for (int n = 0; n < n_act; ++n) {
        for (int k = a_start[n]; k < a_start[n + 1]; ++k) bc[a_idx[k]] = 2 * n;
        for (int k = b_start[n]; k < b_start[n + 1]; ++k) bc[b_idx[k]] = 2 * n + 1;
    }
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaStreamSynchronize(st->stream));
    st->pnx = pnx;
    st->pny = pny;
    st->p_nodes = nodes;
    st->n_act = n_act;
    st->act_flat.assign(act_idx, act_idx + n_act);
    const float dt = (float)st->dt;
    PlateCoefs& k = st->pk;
    k.nx = pnx;
    k.ny = pny;
    k.dx = pdx;
    k.idx4 = 1.0f / (pdx * pdx * pdx * pdx);
    k.dt2 = dt * dt;
    k.inv_rh = 1.0f / rho_h;
    k.damp_fwd = 1.0f + 0.5f * aM * dt;
    k.damp_bwd = 1.0f - 0.5f * aM * dt;
    k.cD0 = D * (1.0f + bK / dt);
    k.cDp = D * (bK / dt);
    std::vector<float> z(nodes, 0.0f);
    for (int q = 0; q < 3; ++q) AK(upload(&st->d_w[q], z));
    AK(upload(&st->d_ext, z));
    AK(upload(&st->d_node_entry, node_entry));
    AK(upload(&st->d_astart, std::vector<int>(a_start, a_start + n_act + 1)));
    AK(upload(&st->d_bstart, std::vector<int>(b_start, b_start + n_act + 1)));
    AK(upload(&st->d_awgt, std::vector<float>(a_wgt, a_wgt + a_start[n_act])));
    AK(upload(&st->d_bwgt, std::vector<float>(b_wgt, b_wgt + b_start[n_act])));
    AK(upload(&st->d_acell, acell));
    AK(upload(&st->d_bcell, bcell));
    AK(upload(&st->d_cabove, std::vector<int>(cell_above, cell_above + n_act)));
    AK(upload(&st->d_cbelow, std::vector<int>(cell_below, cell_below + n_act)));
    AK(upload(&st->d_bc, bc));
    AK(upload(&st->d_bc_flat, st->act_flat));
    if (st->h_ext) cudaFreeHost(st->h_ext);
    st->h_ext = nullptr;
    AK(cudaMallocHost(&st->h_ext, std::max(nodes, 1) * sizeof(float)));
    std::fill(st->h_ext, st->h_ext + nodes, 0.0f);
    st->ext_pending = false;
    st->wi = 0;
    st->plate = true;
    return SK_OK;
}

int amr_set_bridge_plate_sources(AcousticAMRState* st, int n, const int32_t* idx, const float* wgt)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (!st->plate || n <= 0 || !idx || !wgt) return SK_ERR_DIM_MISMATCH;
    for (int i = 0; i < n; ++i)
        if (idx[i] < 0 || idx[i] >= st->p_nodes) return SK_ERR_DIM_MISMATCH;
    st->bridge_idx.assign(idx, idx + n);
    st->bridge_wgt.assign(wgt, wgt + n);
    return SK_OK;
}

int amr_set_neck_plate_sources(AcousticAMRState* st, int n, const int32_t* idx, const float* wgt)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (n == 0) {
        st->neck_idx.clear();
        st->neck_wgt.clear();
        return SK_OK;
    }
    if (!st->plate || !idx || !wgt) return SK_ERR_DIM_MISMATCH;
    for (int i = 0; i < n; ++i)
        if (idx[i] < 0 || idx[i] >= st->p_nodes) return SK_ERR_DIM_MISMATCH;
    st->neck_idx.assign(idx, idx + n);
    st->neck_wgt.assign(wgt, wgt + n);
    return SK_OK;
}

// Forces accumulate on the host, in call order, into the buffer the next step
// uploads (the device buffer is zero between steps), as the reference
// accumulates into its force array (acoustic_amr.cpp:1567-1598).
int amr_inject_bridge_drive(AcousticAMRState* st, const float* drives, int n, float scale)
{
    if (!st || !drives) return SK_ERR_NULL_STATE;
    if (!st->plate || n != (int)st->bridge_idx.size()) return SK_ERR_DIM_MISMATCH;
    for (int i = 0; i < n; ++i) st->h_ext[st->bridge_idx[i]] += drives[i] * st->bridge_wgt[i] * scale;
    st->ext_pending = true;
    return SK_OK;
}

int amr_inject_plate_force(AcousticAMRState* st, int n, const int32_t* idx, const float* wgt, float total)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (!st->plate || n <= 0 || !idx || !wgt) return SK_ERR_DIM_MISMATCH;
    for (int i = 0; i < n; ++i) {
        if (idx[i] < 0 || idx[i] >= st->p_nodes) return SK_ERR_DIM_MISMATCH;
        st->h_ext[idx[i]] += wgt[i] * total;
        st->ext_pending = true;
    }
    return SK_OK;
}

int amr_sample_plate_displacement_batch(const AcousticAMRState* st, int n, const int* idx4, const float* wgt4,
                                        float* out)
{
    if (!st || !idx4 || !wgt4 || !out) return SK_ERR_NULL_STATE;
    if (!st->plate) return SK_ERR_DIM_MISMATCH;
    return plate_taps(const_cast<AcousticAMRState*>(st), n, 4, idx4, wgt4, out);
}

int amr_sample_plate_weighted(const AcousticAMRState* st, int n, const int* idx, const float* wgt, float* out)
{
    if (!st || !idx || !wgt || !out) return SK_ERR_NULL_STATE;
    if (!st->plate) return SK_ERR_DIM_MISMATCH;
    if (n <= 0) {
        *out = 0.0f;
        return SK_OK;
    }
    return plate_taps(const_cast<AcousticAMRState*>(st), 1, n, idx, wgt, out);
}

int amr_get_plate_displacement(const AcousticAMRState* st, float* out, int n)
{
    if (!st || !out) return SK_ERR_NULL_STATE;
    if (!st->plate || n != st->p_nodes) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaMemcpyAsync(out, st->cur_w(), n * sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    AK(cudaStreamSynchronize(st->stream));
    return SK_OK;
}

// Inverse-distance pressure stencils over the acoustic cells within twice the
// mean cell size, and area-weighted face-normal velocity stencils, per mic
// (acoustic_amr.cpp:1647-1760); mics outside the acoustic cells' box are
// clamped onto it.
int amr_setup_mic_samplers(AcousticAMRState* st, int n_mics, const float* pos, const float* axis, int need_v)
{
    if (!st || !pos || !axis) return SK_ERR_NULL_STATE;
    if (n_mics <= 0) return SK_ERR_DIM_MISMATCH;
    double mean_vol = 0.0;
    float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
                   std::numeric_limits<float>::max()};
    float hi[3] = {std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
                   std::numeric_limits<float>::lowest()};
    for (int i : st->acoustic) {
        mean_vol += st->volumes[i];
        for (int d = 0; d < 3; ++d) {
            const float c = (float)st->centers[3 * i + d];
            if (c < lo[d]) lo[d] = c;
            if (c > hi[d]) hi[d] = c;
        }
    }
    mean_vol /= (double)st->acoustic.size();
    const float search_r = 2.0f * (float)std::cbrt(mean_vol);
    std::vector<int> ps{0}, pc, vs{0}, vf;
    std::vector<float> pw, wx, wy, wz;
    for (int m = 0; m < n_mics; ++m) {
        float mx = pos[3 * m], my = pos[3 * m + 1], mz = pos[3 * m + 2];
        const float cx = std::max(lo[0], std::min(hi[0], mx)), cy = std::max(lo[1], std::min(hi[1], my)),
                    cz = std::max(lo[2], std::min(hi[2], mz));
        if (cx != mx || cy != my || cz != mz) {
            fprintf(stderr, "[amr_mic] mic %d at (%.4f, %.4f, %.4f) is outside the acoustic cells; clamped to "
                            "(%.4f, %.4f, %.4f)\n", m, mx, my, mz, cx, cy, cz);
            mx = cx;
            my = cy;
            mz = cz;
        }
        const size_t p0 = pc.size();
        float wsum = 0.0f;
        for (int i : st->acoustic) {
            const float dx = mx - (float)st->centers[3 * i], dy = my - (float)st->centers[3 * i + 1],
                        dz = mz - (float)st->centers[3 * i + 2];
            const float r = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (r < search_r) {
                const float w = (r < 1e-9f) ? 1e9f : 1.0f / r;
                pc.push_back(i);
                pw.push_back(w);
                wsum += w;
            }
        }
        if (pc.size() == p0) return SK_ERR_DIM_MISMATCH;
        const float inv = 1.0f / wsum;
        for (size_t q = p0; q < pw.size(); ++q) pw[q] *= inv;
        ps.push_back((int)pc.size());
        if (need_v) {
            const size_t v0 = vf.size();
            float total = 0.0f;
            for (int f = 0; f < st->n_faces; ++f) {
                const int a = st->face_neg[f], b = st->face_pos[f];
                const float fx = 0.5f * (float)(st->centers[3 * a] + st->centers[3 * b]);
                const float fy = 0.5f * (float)(st->centers[3 * a + 1] + st->centers[3 * b + 1]);
                const float fz = 0.5f * (float)(st->centers[3 * a + 2] + st->centers[3 * b + 2]);
                const float dx = fx - mx, dy = fy - my, dz = fz - mz;
                const float r = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (r >= search_r || st->face_open[f] < 0.5) continue;
                float nx = (float)(st->centers[3 * b] - st->centers[3 * a]);
                float ny = (float)(st->centers[3 * b + 1] - st->centers[3 * a + 1]);
                float nz = (float)(st->centers[3 * b + 2] - st->centers[3 * a + 2]);
                const float nl = std::sqrt(nx * nx + ny * ny + nz * nz);
                if (nl < 1e-12f) continue;
                nx /= nl;
                ny /= nl;
                nz /= nl;
                const float aw = (float)(st->face_area[f] * st->face_open[f]);
                vf.push_back(f);
                wx.push_back(nx * aw);
                wy.push_back(ny * aw);
                wz.push_back(nz * aw);
                total += aw;
            }
            if (total > 1e-20f) {
                const float inv_a = 1.0f / total;
                for (size_t q = v0; q < vf.size(); ++q) {
                    wx[q] *= inv_a;
                    wy[q] *= inv_a;
                    wz[q] *= inv_a;
                }
            }
        }
        vs.push_back((int)vf.size());
    }
    if (guard(st)) return AMR_B200_ERR_CUDA;
    AK(cudaStreamSynchronize(st->stream));
    if (vf.empty()) {   // keep the device arrays non-null; the ranges are empty, nothing is read
        vf.push_back(0);
        wx.push_back(0.f);
        wy.push_back(0.f);
        wz.push_back(0.f);
    }
    AK(upload(&st->d_mps, ps));
    AK(upload(&st->d_mpc, pc));
    AK(upload(&st->d_mpw, pw));
    AK(upload(&st->d_mvs, vs));
    AK(upload(&st->d_mvf, vf));
    AK(upload(&st->d_mwx, wx));
    AK(upload(&st->d_mwy, wy));
    AK(upload(&st->d_mwz, wz));
    st->n_mics = n_mics;
    return ensure_scratch(st, 4 * (size_t)n_mics) ? AMR_B200_ERR_CUDA : SK_OK;
}

int amr_sample_mics(const AcousticAMRState* cst, int n_mics, float* out_p, float* out_vx, float* out_vy,
                    float* out_vz)
{
    AcousticAMRState* st = const_cast<AcousticAMRState*>(cst);
    if (!st || !out_p) return SK_ERR_NULL_STATE;
    if (n_mics != st->n_mics) return SK_ERR_DIM_MISMATCH;
    if (guard(st)) return AMR_B200_ERR_CUDA;
    k_amr_mics<<<blocks(n_mics, 64), 64, 0, st->stream>>>(n_mics, st->d_p, st->d_v, st->d_mps, st->d_mpc,
                                                          st->d_mpw, st->d_mvs, st->d_mvf, st->d_mwx, st->d_mwy,
                                                          st->d_mwz, st->d_scratch);
    AK(cudaGetLastError());
    ++st->launches;
    std::vector<float> h(4 * (size_t)n_mics);
    AK(cudaMemcpyAsync(h.data(), st->d_scratch, h.size() * sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    AK(cudaStreamSynchronize(st->stream));
    std::copy(h.begin(), h.begin() + n_mics, out_p);
    if (out_vx && out_vy && out_vz) {
        std::copy(h.begin() + n_mics, h.begin() + 2 * n_mics, out_vx);
        std::copy(h.begin() + 2 * n_mics, h.begin() + 3 * n_mics, out_vy);
        std::copy(h.begin() + 3 * n_mics, h.begin() + 4 * n_mics, out_vz);
    }
    return SK_OK;
}

const char* amr_b200_last_error(void) { return g_err; }
long long amr_b200_launch_count(const AcousticAMRState* st) { return st ? st->launches : 0; }

int amr_b200_profile(AcousticAMRState* st, int enable)
{
    if (!st) return SK_ERR_NULL_STATE;
    st->prof = enable != 0;
    st->prof_ms = 0;
    st->prof_steps = 0;
    st->ev_used = 0;
    return SK_OK;
}

int amr_b200_profile_read(AcousticAMRState* st, double* total_ms, long long* steps)
{
    if (!st) return SK_ERR_NULL_STATE;
    if (total_ms) *total_ms = st->prof_ms;
    if (steps) *steps = st->prof_steps;
    return SK_OK;
}

}  // extern "C"
