/* ref_shim.cpp — TEST INFRASTRUCTURE ONLY (part of the oracle, never shipped).
 *
 * Compiles the reference's dense acoustic FDTD translation unit
 * (csrc/kernels/acoustic_fdtd.cpp) UNCHANGED, by including it, and adds three
 * hooks the reference has no public entry point for.  oracle/Makefile builds
 * this into oracle/_ref/libfdtd_ref*.so; tests and bench.py's reference arm
 * load it through ctypes.
 *
 *   fdtd_ref_add_pressure        — point-source deposit.  Wraps the
 *                                  reference's own deposit_pressure_open
 *                                  (acoustic_fdtd.cpp:840-872), which the
 *                                  reference defines but never calls.
 *   fdtd_ref_set_face_absorption — per-face scale a_f on the PML's sigma_max.
 *                                  Recomputes pml_alpha / P_damp / V*_damp with
 *                                  the reference's own formulas
 *                                  (acoustic_fdtd.cpp:216-222, :377-396,
 *                                  :469-476, :536-561); at a_f = 1 for all six
 *                                  faces the result is bit-identical to what
 *                                  fdtd_create computed.
 *   fdtd_ref_get_p_damp          — read-back of the per-cell pressure damping,
 *                                  for checking the restated coefficients.
 *
 * REF_FDTD_SOURCE is the path of acoustic_fdtd.cpp, passed by the Makefile.
 */
#include REF_FDTD_SOURCE

#define REF_SHIM_API extern "C" __attribute__((visibility("default")))

REF_SHIM_API int fdtd_ref_add_pressure(AcousticFDTDState* st, int idx, float amp)
{
    return deposit_pressure_open(st, idx, amp);
}

/* sigma(d) with sigma_max scaled by `scale`; the unscaled form is pml_sigma
 * (acoustic_fdtd.cpp:216-222).  scale * x == x exactly at scale == 1. */
static float shim_scaled_sigma(int d, int n_pml, float dt, float scale)
{
    if (n_pml <= 0 || d <= 0) return 0.0f;
    float frac = (float)d / (float)n_pml;
    float sigma_max = scale * (3.45f / (dt * (float)n_pml));
    return sigma_max * frac * frac * frac;
}

/* Depth into the PML along one axis, with the low face taking precedence,
 * exactly as acoustic_fdtd.cpp:381-383 selects it; *face is 0 (low) / 1 (high). */
static int shim_axis_depth(int i, int n, int n_pml, int* face)
{
    if (i < n_pml) { *face = 0; return n_pml - i; }
    if (i >= n - n_pml) { *face = 1; return i - (n - n_pml) + 1; }
    *face = 0;
    return 0;
}

/* a6 = {x_lo, x_hi, y_lo, y_hi, z_lo, z_hi}.  alpha_cell = max over the three
 * axes of a_face * sigma(depth).  With all a = 1 this equals
 * sigma(max depth) because sigma is monotone in d. */
REF_SHIM_API int fdtd_ref_set_face_absorption(AcousticFDTDState* st, int n_pml, const float* a6)
{
    if (!st || !a6) return FDTD_ERR_NULL;
    const int Nx = st->Nx, Ny = st->Ny, Nz = st->Nz;
    const float dt = st->dt;
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                int fx, fy, fz;
                int dxd = shim_axis_depth(i, Nx, n_pml, &fx);
                int dyd = shim_axis_depth(j, Ny, n_pml, &fy);
                int dzd = shim_axis_depth(k, Nz, n_pml, &fz);
                float ax = shim_scaled_sigma(dxd, n_pml, dt, a6[0 + fx]);
                float ay = shim_scaled_sigma(dyd, n_pml, dt, a6[2 + fy]);
                float az = shim_scaled_sigma(dzd, n_pml, dt, a6[4 + fz]);
                float a = ax;
                if (ay > a) a = ay;
                if (az > a) a = az;
                int idx = IDX3(Ny, Nz, i, j, k);
                st->pml_alpha[idx] = a;
                float denom = 1.0f + a * dt;
                st->P_damp[idx] = 1.0f / denom;
            }
    for (int i = 0; i < Nx - 1; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                int vidx = k + Nz * (j + Ny * i);
                int L = IDX3(Ny, Nz, i, j, k), R = IDX3(Ny, Nz, i + 1, j, k);
                st->Vx_damp[vidx] = 1.0f - 0.5f * (st->pml_alpha[L] + st->pml_alpha[R]) * dt;
            }
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny - 1; ++j)
            for (int k = 0; k < Nz; ++k) {
                int vidx = k + Nz * (j + (Ny - 1) * i);
                int L = IDX3(Ny, Nz, i, j, k), R = IDX3(Ny, Nz, i, j + 1, k);
                st->Vy_damp[vidx] = 1.0f - 0.5f * (st->pml_alpha[L] + st->pml_alpha[R]) * dt;
            }
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz - 1; ++k) {
                int vidx = k + (Nz - 1) * (j + Ny * i);
                int L = IDX3(Ny, Nz, i, j, k), R = IDX3(Ny, Nz, i, j, k + 1);
                st->Vz_damp[vidx] = 1.0f - 0.5f * (st->pml_alpha[L] + st->pml_alpha[R]) * dt;
            }
    return FDTD_OK;
}

REF_SHIM_API int fdtd_ref_get_p_damp(const AcousticFDTDState* st, float* out, int out_len)
{
    if (!st || !out) return FDTD_ERR_NULL;
    if (out_len != st->N) return FDTD_ERR_DIM;
    memcpy(out, st->P_damp, (size_t)st->N * sizeof(float));
    return FDTD_OK;
}

/* Number of worker threads the reference's FDTDPool uses (acoustic_fdtd.cpp:758-761). */
REF_SHIM_API int fdtd_ref_pool_threads(void)
{
    int nw = (int)std::thread::hardware_concurrency();
    return nw > 1 ? nw : 1;
}
