/*
 * fdtd_slab.cu — one slab of a room split along i across GPUs.
 *
 * A rank owns the planes [i0, i1) of an open room (no walls, fractions or
 * plate) and stores them with three ghost planes on each side: local plane l
 * is global plane x0 + l, x0 = i0 - 3, L = i1 - i0 + 6 planes of the usual
 * [plane][Ny][Sz] layout.  Every boundary decision is taken on the global
 * index, so a slab computes exactly what the whole-room kernels compute for
 * its planes, provided its ghosts hold the neighbours' values.  Two steps:
 *   fused (fdtd_b200_slab_step): the single-pass TMA kernel of
 *     fdtd_fused.cu on the own planes; it recomputes the new Vx of the two
 *     faces left and one face right of the slab from ghost P (local planes
 *     0 .. own+5) and ghost old Vx (local faces 1 .. own+3), so one exchange
 *     per step suffices: 3 planes of the new P and 2 of the new Vx per
 *     neighbour after the step;
 *   two-pass (fdtd_b200_slab_velocity, then _pressure): velocity of the own
 *     faces needs P on local planes 2 .. own+4, pressure of the own cells
 *     needs Vx on local planes 1 .. own+3; Vx is exchanged between the passes
 *     and P after them.
 * (acoustic_fdtd.cpp:1108-1109 and :935-938 are the stencils that need the
 * ghosts.)  A source in a ghost plane is deposited into the ghost copy as
 * well, so the copies stay identical without another exchange.
 *
 * Kernels run on the stream set with fdtd_b200_slab_set_stream (the caller's
 * communication stream order, e.g. torch's current stream).
 */
#include "acoustic_fdtd_b200.h"
#include "fdtd_internal.h"

#include <climits>
#include <vector>

namespace fdtd {
namespace {

struct Slab {
    Grid g;        // local grid: nx = L planes
    int x0;        // global index of local plane 0
    int nxg;       // global Nx
    int own_lo;    // first own local plane (3)
};

__device__ __forceinline__ float slab_alpha(const Tables& tb, int l, float ay, float az)
{
    return fmaxf(fmaxf(__ldg(tb.ax + l), ay), az);
}

// Velocity of the own faces (acoustic_fdtd.cpp:1099-1148), global boundary logic.
__global__ void __launch_bounds__(256) k_slab_vel(Slab s, Coef cf, Tables tb, const float* __restrict__ p,
                                                  float* __restrict__ vx, float* __restrict__ vy,
                                                  float* __restrict__ vz)
{
    const Grid& g = s.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = s.own_lo + blockIdx.z;
    if (k >= g.nz || j >= g.ny) return;
    const int ig = s.x0 + l;
    const long long id = ((long long)l * g.ny + j) * g.sz + k;
    const float ay = __ldg(tb.ay + j), az = __ldg(tb.az + k);
    const float ac = slab_alpha(tb, l, ay, az);
    const float pc = p[id];
    if (ig < s.nxg - 1) {
        const float pr = p[id + g.plane];
        float grad;
        if (ig > 0 && ig < s.nxg - 2)
            grad = fadd(fmul(cf.c1, fsub(pr, pc)), fmul(cf.c2, fsub(p[id + 2 * g.plane], p[id - g.plane])));
        else
            grad = fsub(pr, pc);
        vx[id] = fmul(fsub(vx[id], fmul(cf.vc, grad)), face_damp(ac, slab_alpha(tb, l + 1, ay, az), cf.dt));
    }
    if (j < g.ny - 1) {
        const float pr = p[id + g.sz];
        float grad;
        if (j > 0 && j < g.ny - 2)
            grad = fadd(fmul(cf.c1, fsub(pr, pc)), fmul(cf.c2, fsub(p[id + 2 * g.sz], p[id - g.sz])));
        else
            grad = fsub(pr, pc);
        vy[id] = fmul(fsub(vy[id], fmul(cf.vc, grad)),
                      face_damp(ac, slab_alpha(tb, l, __ldg(tb.ay + j + 1), az), cf.dt));
    }
    if (k < g.nz - 1) {
        const float pr = p[id + 1];
        float grad;
        if (k > 0 && k < g.nz - 2)
            grad = fadd(fmul(cf.c1, fsub(pr, pc)), fmul(cf.c2, fsub(p[id + 2], p[id - 1])));
        else
            grad = fsub(pr, pc);
        vz[id] = fmul(fsub(vz[id], fmul(cf.vc, grad)),
                      face_damp(ac, slab_alpha(tb, l, ay, __ldg(tb.az + k + 1)), cf.dt));
    }
}

// Pressure of the own cells (acoustic_fdtd.cpp:894-952, :1176-1234).
__global__ void __launch_bounds__(256) k_slab_pres(Slab s, Coef cf, Tables tb, const float* __restrict__ p,
                                                   float* __restrict__ pn, const float* __restrict__ vx,
                                                   const float* __restrict__ vy, const float* __restrict__ vz)
{
    const Grid& g = s.g;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = s.own_lo + blockIdx.z;
    if (k >= g.nz || j >= g.ny) return;
    const int ig = s.x0 + l;
    const long long id = ((long long)l * g.ny + j) * g.sz + k;
    const long long P = g.plane, S = g.sz;
    const float xp = (ig < s.nxg - 1) ? vx[id] : 0.0f;
    const float xm = (ig > 0) ? vx[id - P] : 0.0f;
    const float xpp = (ig < s.nxg - 2) ? vx[id + P] : 0.0f;
    const float xmm = (ig > 1) ? vx[id - 2 * P] : 0.0f;
    const float yp = (j < g.ny - 1) ? vy[id] : 0.0f;
    const float ym = (j > 0) ? vy[id - S] : 0.0f;
    const float ypp = (j < g.ny - 2) ? vy[id + S] : 0.0f;
    const float ymm = (j > 1) ? vy[id - 2 * S] : 0.0f;
    const float zp = (k < g.nz - 1) ? vz[id] : 0.0f;
    const float zm = (k > 0) ? vz[id - 1] : 0.0f;
    const float zpp = (k < g.nz - 2) ? vz[id + 1] : 0.0f;
    const float zmm = (k > 1) ? vz[id - 2] : 0.0f;
    const float d1 = fadd(fadd(fsub(xp, xm), fsub(yp, ym)), fsub(zp, zm));
    const float d2 = fadd(fadd(fsub(xpp, xmm), fsub(ypp, ymm)), fsub(zpp, zmm));
    const float dv = fadd(fmul(cf.c1, d1), fmul(cf.c2, d2));
    const float pd = fminf(fminf(__ldg(tb.px + l), __ldg(tb.py + j)), __ldg(tb.pz + k));
    pn[id] = fmul(fsub(p[id], fmul(cf.bulk, dv)), pd);
}

// Open-cell deposit (acoustic_fdtd.cpp:840-872) into the local copy of the source.
__global__ void k_slab_deposit(float* p, long long src, const float* __restrict__ sig, int n)
{
    const float s = sig[n];
    if (s != 0.0f) p[src] = fadd(p[src], s);
}

// The same deposit with the amplitude passed by the host.
__global__ void k_slab_add(float* p, long long src, float amp)
{
    if (amp != 0.0f) p[src] = fadd(p[src], amp);
}

// Stability sample (acoustic_fdtd.cpp:1245-1268) over the own cells: global
// flat indices phase + 1013 t inside [q_lo, q_hi); records the smallest bad one.
__global__ void k_slab_check(Slab s, const float* __restrict__ p, long long q_first, long long q_hi,
                             unsigned long long* __restrict__ bad)
{
    const Grid& g = s.g;
    const long long q = q_first + ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kCheckStride;
    if (q >= q_hi) return;
    const int k = (int)(q % g.nz);
    const long long ij = q / g.nz;
    const int j = (int)(ij % g.ny);
    const int l = (int)(ij / g.ny) - s.x0;
    const float v = p[((long long)l * g.ny + j) * g.sz + k];
    if (!isfinite(v) || v > 2e3f || v < -2e3f) atomicMin(bad, (unsigned long long)q);
}

float scaled_sigma(int d, int n_pml, float dt, float scale)
{   // pml_sigma with a per-face scale on sigma_max (acoustic_fdtd.cpp:216-222)
    if (n_pml <= 0 || d <= 0) return 0.0f;
    float frac = (float)d / (float)n_pml;
    float sigma_max = scale * (3.45f / (dt * (float)n_pml));
    return sigma_max * frac * frac * frac;
}

float axis_alpha(int i, int n, int n_pml, float dt, float a_lo, float a_hi)
{   // low face first, as acoustic_fdtd.cpp:381-383 picks the depth
    if (i < n_pml) return scaled_sigma(n_pml - i, n_pml, dt, a_lo);
    if (i >= n - n_pml) return scaled_sigma(i - (n - n_pml) + 1, n_pml, dt, a_hi);
    return 0.0f;
}

}  // namespace
}  // namespace fdtd

using namespace fdtd;

struct FdtdB200Slab {
    int device = 0;
    cudaStream_t stream = nullptr;
    Slab s{};
    int i0 = 0, i1 = 0, ny = 0, nz = 0;
    Coef cf{};
    Tables tb{};
    float* d_tab = nullptr;
    float* P[2] = {};
    float* V[2][3] = {};
    int cur = 0, cv = 0;
    FusedCache* fcache = nullptr;
    long long src = -1;
    float* d_sig = nullptr;
    int n_sig = 0;
    int n_rec = 0;
    long long* d_ridx = nullptr;
    float* d_rw = nullptr;
    float* d_trace = nullptr;
    int cap = 0, rows = 0;
    unsigned long long* d_bad = nullptr;
    unsigned* d_status = nullptr;   // timeout word of the fused step
    // neighbours whose ghost planes the fused step writes directly (side 0 left, 1 right)
    float* peer_p[2][2] = {};       // [side][buffer]
    float* peer_vx[2][2] = {};      // [side][velocity set]
    int peer_dl[2] = {0, 0};
    long long launches = 0;
};

namespace {

#define SCK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { record_cuda_error(e_, #x); return FDTD_ERR_CUDA; } } while (0)

// global flat (reference order) -> local padded index, -1 when outside the local planes
long long slab_index(const FdtdB200Slab* h, long long flat)
{
    const Grid& g = h->s.g;
    const long long k = flat % h->nz, ij = flat / h->nz, j = ij % h->ny, ig = ij / h->ny;
    const long long l = ig - h->s.x0;
    if (l < 0 || l >= g.nx || ig >= h->s.nxg) return -1;
    return (l * g.ny + j) * g.sz + k;
}

dim3 own_grid(const FdtdB200Slab* h)
{
    return dim3((h->nz + 31) / 32, (h->ny + 7) / 8, h->i1 - h->i0);
}

}  // namespace

extern "C" {

int fdtd_b200_slab_layout(int Nx, int Ny, int Nz, int i0, int i1, int* local_planes, int* sz)
{
    if (Nx < 1 || Ny < 1 || Nz < 1 || i0 < 0 || i1 > Nx || i1 - i0 < 3) return FDTD_ERR_DIM;
    if (local_planes) *local_planes = i1 - i0 + 6;
    if (sz) *sz = (Nz + kRowAlign - 1) / kRowAlign * kRowAlign;
    return FDTD_OK;
}

FdtdB200Slab* fdtd_b200_slab_create(int Nx, int Ny, int Nz, int i0, int i1, float dx, float c,
                                    float rho_air, int n_pml, const float* a6,
                                    float* const* fields, int device)
{
    int L = 0, sz = 0;
    if (fdtd_b200_slab_layout(Nx, Ny, Nz, i0, i1, &L, &sz) != FDTD_OK || !fields || dx <= 0 || c <= 0)
        return nullptr;
    if ((long long)Nx * Ny * Nz > INT_MAX) return nullptr;
    for (int q = 0; q < 8; ++q)
        if (!fields[q]) return nullptr;
    FdtdB200Slab* h = new FdtdB200Slab();
    if (device < 0) cudaGetDevice(&device);
    h->device = device;
    h->i0 = i0; h->i1 = i1; h->ny = Ny; h->nz = Nz;
    Grid& g = h->s.g;
    g.nx = L; g.ny = Ny; g.nz = Nz; g.sz = sz;
    g.plane = (long long)Ny * sz;
    g.cells = (long long)L * g.plane;
    h->s.x0 = i0 - 3;
    h->s.nxg = Nx;
    h->s.own_lo = 3;
    h->P[0] = fields[0]; h->P[1] = fields[1];
    for (int c = 0; c < 3; ++c) {
        h->V[0][c] = fields[2 + c];
        h->V[1][c] = fields[5 + c];
    }
    // coefficients exactly as fdtd_create computes them (acoustic_fdtd.cpp:345-349, :1091, :1173)
    const float dt = 0.77f * dx / (c * 1.732050808f);
    h->cf.vc = dt / (rho_air * dx);
    const float inv_dx = 1.0f / dx;
    h->cf.bulk = rho_air * c * c * dt * inv_dx;
    h->cf.dt = dt;
    h->cf.c1 = 9.0f / 8.0f;
    h->cf.c2 = -1.0f / 24.0f;
    h->cf.inv_dt = 1.0f / dt;
    const float ones[6] = {1, 1, 1, 1, 1, 1};
    if (!a6) a6 = ones;
    std::vector<float> t((size_t)2 * (L + Ny + Nz), 0.0f);
    float* ax = t.data();
    float* ay = ax + L;
    float* az = ay + Ny;
    float* px = az + Nz;
    for (int l = 0; l < L; ++l) {
        const int ig = i0 - 3 + l;
        ax[l] = (ig >= 0 && ig < Nx) ? axis_alpha(ig, Nx, n_pml, dt, a6[0], a6[1]) : 0.0f;
    }
    for (int j = 0; j < Ny; ++j) ay[j] = axis_alpha(j, Ny, n_pml, dt, a6[2], a6[3]);
    for (int k = 0; k < Nz; ++k) az[k] = axis_alpha(k, Nz, n_pml, dt, a6[4], a6[5]);
    for (int q = 0; q < L + Ny + Nz; ++q) {   // P damping 1/(1 + alpha dt) (acoustic_fdtd.cpp:469-476)
        float denom = 1.0f + ax[q] * dt;
        px[q] = 1.0f / denom;
    }
    bool ok = cudaSetDevice(device) == cudaSuccess &&
              cudaMalloc(&h->d_tab, t.size() * sizeof(float)) == cudaSuccess &&
              cudaMemcpy(h->d_tab, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMalloc(&h->d_bad, sizeof(unsigned long long)) == cudaSuccess;
    if (!ok) {
        fdtd_b200_slab_destroy(h);
        return nullptr;
    }
    h->tb.ax = h->d_tab;
    h->tb.ay = h->d_tab + L;
    h->tb.az = h->d_tab + L + Ny;
    h->tb.px = h->d_tab + L + Ny + Nz;
    h->tb.py = h->tb.px + L;
    h->tb.pz = h->tb.py + Ny;
    x_interior_run(ax, L, &h->tb.xi_lo, &h->tb.xi_hi);
    return h;
}

void fdtd_b200_slab_destroy(FdtdB200Slab* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    if (h->fcache) fused_cache_destroy(h->fcache);
    cudaFree(h->d_tab);
    cudaFree(h->d_bad);
    cudaFree(h->d_status);
    cudaFree(h->d_sig);
    cudaFree(h->d_ridx);
    cudaFree(h->d_rw);
    cudaFree(h->d_trace);
    delete h;
}

int fdtd_b200_slab_set_stream(FdtdB200Slab* h, void* stream)
{
    if (!h) return FDTD_ERR_NULL;
    h->stream = (cudaStream_t)stream;
    return FDTD_OK;
}

float fdtd_b200_slab_dt(const FdtdB200Slab* h) { return h ? h->cf.dt : 0.0f; }

int fdtd_b200_slab_current(const FdtdB200Slab* h) { return h ? h->cur : -1; }

int fdtd_b200_slab_vset(const FdtdB200Slab* h) { return h ? h->cv : -1; }

long long fdtd_b200_slab_launch_count(const FdtdB200Slab* h) { return h ? h->launches : 0; }

int fdtd_b200_slab_set_source(FdtdB200Slab* h, int cell, const float* signal, int n)
{
    if (!h) return FDTD_ERR_NULL;
    if (n < 0 || (n > 0 && !signal)) return FDTD_ERR_ARG;
    SCK(cudaSetDevice(h->device));
    cudaFree(h->d_sig);
    h->d_sig = nullptr;
    h->n_sig = 0;
    h->src = (cell >= 0) ? slab_index(h, cell) : -1;
    if (h->src >= 0 && n > 0) {
        SCK(cudaMalloc(&h->d_sig, sizeof(float) * n));
        SCK(cudaMemcpy(h->d_sig, signal, sizeof(float) * n, cudaMemcpyHostToDevice));
        h->n_sig = n;
    }
    return FDTD_OK;
}

int fdtd_b200_slab_set_receivers(FdtdB200Slab* h, int n_rec, const int* idx8, const float* wgt8, int capacity)
{
    if (!h || (n_rec > 0 && (!idx8 || !wgt8))) return FDTD_ERR_NULL;
    if (n_rec < 0 || capacity < 0) return FDTD_ERR_ARG;
    std::vector<long long> li((size_t)n_rec * 8);
    for (size_t q = 0; q < li.size(); ++q) {
        li[q] = slab_index(h, idx8[q]);
        if (li[q] < 0) return FDTD_ERR_ARG;   // a tap outside this slab and its ghosts
    }
    SCK(cudaSetDevice(h->device));
    cudaFree(h->d_ridx); cudaFree(h->d_rw); cudaFree(h->d_trace);
    h->d_ridx = nullptr; h->d_rw = nullptr; h->d_trace = nullptr;
    h->n_rec = n_rec;
    h->cap = capacity;
    h->rows = 0;
    if (n_rec > 0) {
        SCK(cudaMalloc(&h->d_ridx, sizeof(long long) * li.size()));
        SCK(cudaMalloc(&h->d_rw, sizeof(float) * li.size()));
        SCK(cudaMalloc(&h->d_trace, sizeof(float) * (size_t)n_rec * (capacity > 0 ? capacity : 1)));
        SCK(cudaMemcpy(h->d_ridx, li.data(), sizeof(long long) * li.size(), cudaMemcpyHostToDevice));
        SCK(cudaMemcpy(h->d_rw, wgt8, sizeof(float) * li.size(), cudaMemcpyHostToDevice));
    }
    return FDTD_OK;
}

int fdtd_b200_slab_deposit(FdtdB200Slab* h, int n)
{
    if (!h) return FDTD_ERR_NULL;
    if (h->src < 0 || n < 0 || n >= h->n_sig) return FDTD_OK;
    k_slab_deposit<<<1, 1, 0, h->stream>>>(h->P[h->cur], h->src, h->d_sig, n);
    ++h->launches;
    SCK(cudaGetLastError());
    return FDTD_OK;
}

// Deposit amp into the local copy of a cell (global flat index; an own or a
// ghost copy; a no-op when the slab holds no copy of it).
int fdtd_b200_slab_add_pressure(FdtdB200Slab* h, int cell, float amp)
{
    if (!h) return FDTD_ERR_NULL;
    const long long li = slab_index(h, cell);
    if (li < 0) return FDTD_OK;
    k_slab_add<<<1, 1, 0, h->stream>>>(h->P[h->cur], li, amp);
    ++h->launches;
    SCK(cudaGetLastError());
    return FDTD_OK;
}

// The receiver samples of the last recorded step into out[0 .. n_rec), once
// the slab's stream has reached them.
int fdtd_b200_slab_read_last(FdtdB200Slab* h, float* out, int n)
{
    if (!h || (!out && n > 0)) return FDTD_ERR_NULL;
    if (n != h->n_rec) return FDTD_ERR_DIM;
    if (h->n_rec <= 0 || h->rows == 0) return FDTD_OK;
    SCK(cudaMemcpyAsync(out, h->d_trace + (size_t)(h->rows - 1) * h->n_rec, sizeof(float) * h->n_rec,
                        cudaMemcpyDeviceToHost, h->stream));
    SCK(cudaStreamSynchronize(h->stream));
    return FDTD_OK;
}

int fdtd_b200_slab_velocity(FdtdB200Slab* h)
{
    if (!h) return FDTD_ERR_NULL;
    float* const* v = h->V[h->cv];
    k_slab_vel<<<own_grid(h), dim3(32, 8, 1), 0, h->stream>>>(h->s, h->cf, h->tb, h->P[h->cur], v[0], v[1],
                                                             v[2]);
    ++h->launches;
    SCK(cudaGetLastError());
    return FDTD_OK;
}

int fdtd_b200_slab_pressure(FdtdB200Slab* h)
{
    if (!h) return FDTD_ERR_NULL;
    float* const* v = h->V[h->cv];
    k_slab_pres<<<own_grid(h), dim3(32, 8, 1), 0, h->stream>>>(h->s, h->cf, h->tb, h->P[h->cur],
                                                              h->P[h->cur ^ 1], v[0], v[1], v[2]);
    ++h->launches;
    SCK(cudaGetLastError());
    h->cur ^= 1;
    return FDTD_OK;
}

// Neighbour fields for the fused step's direct ghost stores.  fields: the
// neighbour's eight fields {P0, P1, Vx0, Vy0, Vz0, Vx1, Vy1, Vz1} as pointers
// this process can write (the same device, peer access, or an IPC mapping);
// NULL clears the side.  The neighbour must step in lockstep (same buffer
// parities) and own the planes [peer_i0, peer_i1) next to this slab.
int fdtd_b200_slab_set_peer(FdtdB200Slab* h, int side, float* const* fields, int peer_i0, int peer_i1)
{
    if (!h) return FDTD_ERR_NULL;
    if (side != 0 && side != 1) return FDTD_ERR_ARG;
    if (!fields) {
        h->peer_p[side][0] = h->peer_p[side][1] = nullptr;
        h->peer_vx[side][0] = h->peer_vx[side][1] = nullptr;
        return FDTD_OK;
    }
    if (peer_i1 - peer_i0 < 3 || (side == 0 && peer_i1 != h->i0) || (side == 1 && peer_i0 != h->i1))
        return FDTD_ERR_ARG;
    for (int q = 0; q < 8; ++q)
        if (!fields[q]) return FDTD_ERR_NULL;
    h->peer_p[side][0] = fields[0];
    h->peer_p[side][1] = fields[1];
    h->peer_vx[side][0] = fields[2];
    h->peer_vx[side][1] = fields[5];
    h->peer_dl[side] = h->i0 - peer_i0;   // local plane l here is plane l + dl there
    return FDTD_OK;
}

// One fused step of the own planes: P[cur] -> P[cur^1], V set cv -> cv^1.
int fdtd_b200_slab_step(FdtdB200Slab* h)
{
    if (!h) return FDTD_ERR_NULL;
    if (!fused_supported(h->s.g)) return FDTD_ERR_DIM;
    if (!h->fcache) h->fcache = fused_cache_create();
    if (!h->fcache) return FDTD_ERR_CUDA;
    if (!h->d_status) {
        SCK(cudaMalloc(&h->d_status, kStatusWords * sizeof(unsigned)));
        SCK(cudaMemsetAsync(h->d_status, 0xFF, kStatusWords * sizeof(unsigned), h->stream));
    }
    float* const* vi = h->V[h->cv];
    float* const* vo = h->V[h->cv ^ 1];
    FusedArgs a{h->s.g, h->cf, h->tb, h->P[h->cur], h->P[h->cur ^ 1], {vi[0], vi[1], vi[2]},
                {vo[0], vo[1], vo[2]}, h->d_status,
                XSpan{h->s.x0, h->s.nxg, h->s.own_lo, h->i1 - h->i0}};
    const int own = h->i1 - h->i0;
    for (int sd = 0; sd < 2; ++sd) {
        if (!h->peer_p[sd][0]) continue;
        // left neighbour: its ghosts own_L+3 .. own_L+5 (P) and own_L+3, own_L+4 (Vx) are
        // this slab's planes 3 .. 5 and faces 3, 4; right neighbour: its ghosts 0 .. 2 (P)
        // and 1, 2 (Vx) are this slab's planes own .. own+2 and faces own+1, own+2
        a.pr.pn[sd] = h->peer_p[sd][h->cur ^ 1];
        a.pr.vx[sd] = h->peer_vx[sd][h->cv ^ 1];
        a.pr.dl[sd] = h->peer_dl[sd];
        a.pr.p_lo[sd] = sd == 0 ? 3 : own;
        a.pr.p_hi[sd] = sd == 0 ? 6 : own + 3;
        a.pr.v_lo[sd] = sd == 0 ? 3 : own + 1;
        a.pr.v_hi[sd] = sd == 0 ? 5 : own + 3;
    }
    SCK(launch_fused_step(a, h->fcache, h->stream));
    ++h->launches;
    h->cur ^= 1;
    h->cv ^= 1;
    return FDTD_OK;
}

// own planes at each end of a slab that a neighbour keeps as ghosts
constexpr int GHOST_PLANES = 3;

// The fused step in two launches, so that the ghost exchange can overlap the
// interior: part 1 computes the own planes a neighbour keeps as ghosts (the
// first and the last three; the whole slab when it has six planes or fewer),
// part 2 the planes between them and then flips the buffers.  Both parts
// read only the old fields and write only their own planes of the new ones,
// so together they equal fdtd_b200_slab_step bit for bit; part 2 may run on
// another stream than part 1 (fdtd_b200_slab_set_stream before each call).
int fdtd_b200_slab_step_part(FdtdB200Slab* h, int part)
{
    if (!h) return FDTD_ERR_NULL;
    if (part != 1 && part != 2) return FDTD_ERR_ARG;
    if (!fused_supported(h->s.g)) return FDTD_ERR_DIM;
    if (!h->fcache) h->fcache = fused_cache_create();
    if (!h->fcache) return FDTD_ERR_CUDA;
    if (!h->d_status) {
        SCK(cudaMalloc(&h->d_status, kStatusWords * sizeof(unsigned)));
        SCK(cudaMemsetAsync(h->d_status, 0xFF, kStatusWords * sizeof(unsigned), h->stream));
    }
    float* const* vi = h->V[h->cv];
    float* const* vo = h->V[h->cv ^ 1];
    FusedArgs a{h->s.g, h->cf, h->tb, h->P[h->cur], h->P[h->cur ^ 1], {vi[0], vi[1], vi[2]},
                {vo[0], vo[1], vo[2]}, h->d_status, XSpan{h->s.x0, h->s.nxg, h->s.own_lo, 0}};
    const int own = h->i1 - h->i0, lo = h->s.own_lo;
    auto run = [&](int from, int n) -> cudaError_t {
        if (n <= 0) return cudaSuccess;
        a.xs.i_lo = from;
        a.xs.n_own = n;
        ++h->launches;
        return launch_fused_step(a, h->fcache, h->stream);
    };
    if (part == 1) {
        if (own <= 2 * GHOST_PLANES) {
            SCK(run(lo, own));
        } else {
            SCK(run(lo, GHOST_PLANES));
            SCK(run(lo + own - GHOST_PLANES, GHOST_PLANES));
        }
        return FDTD_OK;
    }
    if (own > 2 * GHOST_PLANES) SCK(run(lo + GHOST_PLANES, own - 2 * GHOST_PLANES));
    h->cur ^= 1;
    h->cv ^= 1;
    return FDTD_OK;
}

int fdtd_b200_slab_record(FdtdB200Slab* h)
{
    if (!h) return FDTD_ERR_NULL;
    if (h->n_rec <= 0 || h->rows >= h->cap) return FDTD_OK;
    SCK(launch_wsum(h->P[h->cur], h->d_ridx, h->d_rw, h->n_rec, 8, 0,
                    h->d_trace + (size_t)h->rows * h->n_rec, h->stream));
    ++h->launches;
    ++h->rows;
    return FDTD_OK;
}

// Samples the own cells at global flat indices phase + 1013 t; *bad = the
// smallest failing index or -1.  Waits for the stream; also reports a fused
// step whose load wait ran out (FDTD_ERR_CUDA).
int fdtd_b200_slab_check(FdtdB200Slab* h, int phase, long long* bad)
{
    if (!h || !bad) return FDTD_ERR_NULL;
    const long long per = (long long)h->ny * h->nz;
    const long long q_lo = (long long)h->i0 * per, q_hi = (long long)h->i1 * per;
    long long q_first = phase;
    if (q_first < q_lo) q_first += ((q_lo - q_first + kCheckStride - 1) / kCheckStride) * kCheckStride;
    SCK(cudaMemsetAsync(h->d_bad, 0xFF, sizeof(unsigned long long), h->stream));
    if (q_first < q_hi) {
        const long long n = (q_hi - q_first + kCheckStride - 1) / kCheckStride;
        k_slab_check<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->s, h->P[h->cur], q_first, q_hi, h->d_bad);
        ++h->launches;
        SCK(cudaGetLastError());
    }
    unsigned long long v = 0;
    unsigned tmo = 0xFFFFFFFFu;
    SCK(cudaMemcpyAsync(&v, h->d_bad, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    if (h->d_status)
        SCK(cudaMemcpyAsync(&tmo, h->d_status + kStatusTimeout, sizeof(tmo), cudaMemcpyDeviceToHost, h->stream));
    SCK(cudaStreamSynchronize(h->stream));
    if (tmo != 0xFFFFFFFFu) {
        record_cuda_error(cudaErrorTimeout, "fused slab step: a tile's load wait timed out");
        return FDTD_ERR_CUDA;
    }
    *bad = (v == ~0ULL) ? -1 : (long long)v;
    return FDTD_OK;
}

int fdtd_b200_slab_get_traces(FdtdB200Slab* h, float* out, int out_len, int* n_rows)
{
    if (!h || !out) return FDTD_ERR_NULL;
    const long long need = (long long)h->rows * h->n_rec;
    if (out_len < need) return FDTD_ERR_DIM;
    SCK(cudaStreamSynchronize(h->stream));
    if (need > 0) SCK(cudaMemcpy(out, h->d_trace, sizeof(float) * need, cudaMemcpyDeviceToHost));
    if (n_rows) *n_rows = h->rows;
    return FDTD_OK;
}

}  // extern "C"
