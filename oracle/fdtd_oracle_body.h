/* fdtd_oracle_body.h — TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * Plain-C restatement of the reference's dense acoustic FDTD
 * (csrc/kernels/acoustic_fdtd.cpp of sangderenard/spectral-analyzer), written
 * for checking the CUDA engine, never for shipping or timing it.
 *
 * This body is included twice by fdtd_oracle.c: once with R = float (prefix
 * orc_, bit-exact with the reference compiled without FMA contraction) and
 * once with R = double (prefix orc64_, the FP64 oracle for the precision
 * study).  Every arithmetic expression keeps the reference's operand order so
 * that the float build rounds identically; each function cites the reference
 * lines it restates.
 *
 * Layouts are the reference's (acoustic_fdtd.h:67-71, :430-437):
 *   P  [Nx][Ny][Nz]      idx k + Nz*(j + Ny*i)
 *   Vx [Nx-1][Ny][Nz]    idx k + Nz*(j + Ny*i)
 *   Vy [Nx][Ny-1][Nz]    idx k + Nz*(j + (Ny-1)*i)
 *   Vz [Nx][Ny][Nz-1]    idx k + (Nz-1)*(j + Ny*i)
 *
 * Requires before inclusion: R (float|double), L(x) (literal suffix), P_(x)
 * (symbol prefixer), S_ (state struct name).
 */

typedef struct S_ {
    int nx, ny, nz, n, n_plate, plate_iz, n_pml;
    R dx, dt, c, rho;
    R vel_coeff, bulk_coeff;
    uint8_t *cell_type;        /* after PML marking and plate-mask enforcement */
    uint8_t *plate_active;
    R *p, *p_next;             /* P^n and the write target of the next step */
    R *vx, *vy, *vz;
    R *alpha, *pdamp;          /* per cell */
    R *vxd, *vyd, *vzd;        /* per-face damping multipliers */
    R *vxf, *vyf, *vzf;        /* per-face open fractions */
    int has_frac;
    /* Kirchhoff plate */
    R *w, *w_prev, *w_tmp, *ext_force;
    int n_act;
    int *act, *nb13, *above, *below, *vz_below, *vz_above;
    R pl_a, pl_bh, pl_vd, pl_bk;
    /* bridge sources */
    int n_src;
    int *src_idx;
    R *src_wgt;
    int step_count, stab_phase;
    /* config-5 form: a_c = alpha_c * dt given per cell (NULL = PML profile) */
    R *cell_a;
} S_;

static int P_(is_solid)(uint8_t c) { return c == 1 || c == 2; }  /* acoustic_fdtd.cpp:37-40 */

static int P_(idx3)(const S_* s, int i, int j, int k) { return k + s->nz * (j + s->ny * i); }

/* pml_sigma with an optional scale on sigma_max (acoustic_fdtd.cpp:216-222). */
static R P_(sigma)(int d, int n_pml, R dt, R scale)
{
    if (n_pml <= 0 || d <= 0) return L(0.0);
    R frac = (R)d / (R)n_pml;
    R sigma_max = scale * (L(3.45) / (dt * (R)n_pml));
    return sigma_max * frac * frac * frac;
}

static int P_(axis_depth)(int i, int n, int n_pml, int* face)
{   /* depth selection of acoustic_fdtd.cpp:381-383 (low face first) */
    if (i < n_pml) { *face = 0; return n_pml - i; }
    if (i >= n - n_pml) { *face = 1; return i - (n - n_pml) + 1; }
    *face = 0;
    return 0;
}

/* Recompute alpha, P damping and face damping (acoustic_fdtd.cpp:377-396,
 * :469-476, :536-561) with per-face scales a6 = {xlo,xhi,ylo,yhi,zlo,zhi}. */
static void P_(build_damping)(S_* s, const R* a6)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz, np = s->n_pml;
    const R dt = s->dt;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int idx = P_(idx3)(s, i, j, k);
                R a, den;
                if (s->cell_a) {
                    /* per-cell form: alpha*dt = a_c directly */
                    a = s->cell_a[idx];
                    s->alpha[idx] = a;
                    den = L(1.0) + a;
                } else {
                    int fx, fy, fz;
                    int di = P_(axis_depth)(i, nx, np, &fx);
                    int dj = P_(axis_depth)(j, ny, np, &fy);
                    int dk = P_(axis_depth)(k, nz, np, &fz);
                    R ax = P_(sigma)(di, np, dt, a6[0 + fx]);
                    R ay = P_(sigma)(dj, np, dt, a6[2 + fy]);
                    R az = P_(sigma)(dk, np, dt, a6[4 + fz]);
                    a = ax;
                    if (ay > a) a = ay;
                    if (az > a) a = az;
                    s->alpha[idx] = a;
                    den = L(1.0) + a * dt;
                }
                s->pdamp[idx] = L(1.0) / den;
            }
#define FACE_DAMP(L_, R_) (s->cell_a \
        ? (L(1.0) - L(0.5) * (s->alpha[L_] + s->alpha[R_])) \
        : (L(1.0) - L(0.5) * (s->alpha[L_] + s->alpha[R_]) * dt))
    for (int i = 0; i < nx - 1; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                s->vxd[k + nz * (j + ny * i)] =
                    FACE_DAMP(P_(idx3)(s, i, j, k), P_(idx3)(s, i + 1, j, k));
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
                s->vyd[k + nz * (j + (ny - 1) * i)] =
                    FACE_DAMP(P_(idx3)(s, i, j, k), P_(idx3)(s, i, j + 1, k));
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz - 1; ++k)
                s->vzd[k + (nz - 1) * (j + ny * i)] =
                    FACE_DAMP(P_(idx3)(s, i, j, k), P_(idx3)(s, i, j, k + 1));
#undef FACE_DAMP
}

EXPORT void P_(destroy)(S_* s)
{
    if (!s) return;
    free(s->cell_type); free(s->plate_active);
    free(s->p); free(s->p_next); free(s->vx); free(s->vy); free(s->vz);
    free(s->alpha); free(s->pdamp); free(s->vxd); free(s->vyd); free(s->vzd);
    free(s->vxf); free(s->vyf); free(s->vzf);
    free(s->w); free(s->w_prev); free(s->w_tmp); free(s->ext_force);
    free(s->act); free(s->nb13); free(s->above); free(s->below);
    free(s->vz_below); free(s->vz_above);
    free(s->src_idx); free(s->src_wgt); free(s->cell_a);
    free(s);
}

/* fdtd_create (acoustic_fdtd.cpp:327-768): time step, PML, plate-mask
 * enforcement, default face fractions, plate stencil tables. */
EXPORT S_* P_(create)(int nx, int ny, int nz, R dx, R c, R rho,
                      const uint8_t* cell_type, int plate_iz, const uint8_t* plate_active,
                      R plate_mass, R plate_D, R plate_aM, R plate_bK, int n_pml)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || dx <= L(0.0) || c <= L(0.0)
            || !cell_type || !plate_active)
        return NULL;
    S_* s = (S_*)calloc(1, sizeof(S_));
    if (!s) return NULL;
    const int n = nx * ny * nz, npl = nx * ny;
    s->nx = nx; s->ny = ny; s->nz = nz; s->n = n; s->n_plate = npl; s->n_pml = n_pml;
    s->plate_iz = (plate_iz >= 0 && plate_iz < nz) ? plate_iz : nz / 2;   /* :359 */
    s->dx = dx; s->c = c; s->rho = rho;
    s->dt = L(0.77) * dx / (c * L(1.732050808));                          /* :348 */
    s->vel_coeff = s->dt / (rho * dx);                                     /* :1091 */
    s->bulk_coeff = rho * c * c * s->dt * (L(1.0) / dx);                    /* :1173 */

    s->cell_type = (uint8_t*)malloc((size_t)n);
    s->plate_active = (uint8_t*)malloc((size_t)npl);
    s->p = (R*)calloc((size_t)n, sizeof(R));
    s->p_next = (R*)calloc((size_t)n, sizeof(R));
    s->alpha = (R*)calloc((size_t)n, sizeof(R));
    s->pdamp = (R*)calloc((size_t)n, sizeof(R));
    const int nvx = (nx - 1) * ny * nz, nvy = nx * (ny - 1) * nz, nvz = nx * ny * (nz - 1);
    s->vx = (R*)calloc((size_t)(nvx > 0 ? nvx : 1), sizeof(R));
    s->vy = (R*)calloc((size_t)(nvy > 0 ? nvy : 1), sizeof(R));
    s->vz = (R*)calloc((size_t)(nvz > 0 ? nvz : 1), sizeof(R));
    s->vxd = (R*)calloc((size_t)(nvx > 0 ? nvx : 1), sizeof(R));
    s->vyd = (R*)calloc((size_t)(nvy > 0 ? nvy : 1), sizeof(R));
    s->vzd = (R*)calloc((size_t)(nvz > 0 ? nvz : 1), sizeof(R));
    s->vxf = (R*)calloc((size_t)(nvx > 0 ? nvx : 1), sizeof(R));
    s->vyf = (R*)calloc((size_t)(nvy > 0 ? nvy : 1), sizeof(R));
    s->vzf = (R*)calloc((size_t)(nvz > 0 ? nvz : 1), sizeof(R));
    s->w = (R*)calloc((size_t)npl, sizeof(R));
    s->w_prev = (R*)calloc((size_t)npl, sizeof(R));
    s->w_tmp = (R*)calloc((size_t)npl, sizeof(R));
    s->ext_force = (R*)calloc((size_t)npl, sizeof(R));
    if (!s->cell_type || !s->plate_active || !s->p || !s->p_next || !s->alpha || !s->pdamp
            || !s->vx || !s->vy || !s->vz || !s->vxd || !s->vyd || !s->vzd
            || !s->vxf || !s->vyf || !s->vzf || !s->w || !s->w_prev || !s->w_tmp
            || !s->ext_force) {
        P_(destroy)(s);
        return NULL;
    }
    memcpy(s->cell_type, cell_type, (size_t)n);
    memcpy(s->plate_active, plate_active, (size_t)npl);

    /* PML marking of air cells (:377-396); arithmetic uses alpha only. */
    {
        R ones[6] = {L(1.0), L(1.0), L(1.0), L(1.0), L(1.0), L(1.0)};
        P_(build_damping)(s, ones);
        for (int idx = 0; idx < n; ++idx)
            if (s->cell_type[idx] == 0 && s->alpha[idx] > L(0.0)) s->cell_type[idx] = 3;
    }
    /* Plate mask on the pressure grid (:413-425). */
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            int g = P_(idx3)(s, i, j, s->plate_iz);
            if (s->plate_active[j + ny * i]) {
                if (s->cell_type[g] == 0 || s->cell_type[g] == 3) s->cell_type[g] = 2;
            } else if (s->cell_type[g] == 2) {
                s->cell_type[g] = 0;
            }
        }

    /* Plate constants (:435-449). */
    s->pl_a = (s->dt * s->dt) / plate_mass;
    {
        R dx4 = dx * dx * dx * dx;
        s->pl_bh = plate_D * (s->dt * s->dt) / (plate_mass * dx4);
    }
    s->pl_vd = L(1.0) - plate_aM * s->dt;
    s->pl_bk = (s->dt > L(0.0)) ? (plate_bK / s->dt * s->pl_bh) : L(0.0);

    /* Default fractions: 0 next to a solid cell, else 1; plate-layer Vz faces 1 (:492-534). */
    for (int i = 0; i < nx - 1; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                s->vxf[k + nz * (j + ny * i)] =
                    (P_(is_solid)(s->cell_type[P_(idx3)(s, i, j, k)]) ||
                     P_(is_solid)(s->cell_type[P_(idx3)(s, i + 1, j, k)])) ? L(0.0) : L(1.0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k)
                s->vyf[k + nz * (j + (ny - 1) * i)] =
                    (P_(is_solid)(s->cell_type[P_(idx3)(s, i, j, k)]) ||
                     P_(is_solid)(s->cell_type[P_(idx3)(s, i, j + 1, k)])) ? L(0.0) : L(1.0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz - 1; ++k) {
                R f;
                if (k == s->plate_iz - 1 || k == s->plate_iz) f = L(1.0);
                else f = (P_(is_solid)(s->cell_type[P_(idx3)(s, i, j, k)]) ||
                          P_(is_solid)(s->cell_type[P_(idx3)(s, i, j, k + 1)])) ? L(0.0) : L(1.0);
                s->vzf[k + (nz - 1) * (j + ny * i)] = f;
            }

    /* Plate stencil tables (:670-733) and Vz injection faces (:737-752). */
    {
        static const int DI[13] = {0, 1, -1, 0, 0, 1, 1, -1, -1, 2, -2, 0, 0};
        static const int DJ[13] = {0, 0, 0, 1, -1, 1, -1, 1, -1, 0, 0, 2, -2};
        int na = 0;
        for (int q = 0; q < npl; ++q) if (plate_active[q]) ++na;
        s->n_act = na;
        int m = na > 0 ? na : 1;
        s->act = (int*)malloc((size_t)m * sizeof(int));
        s->above = (int*)malloc((size_t)m * sizeof(int));
        s->below = (int*)malloc((size_t)m * sizeof(int));
        s->nb13 = (int*)malloc((size_t)m * 13 * sizeof(int));
        s->vz_below = (int*)malloc((size_t)m * sizeof(int));
        s->vz_above = (int*)malloc((size_t)m * sizeof(int));
        if (!s->act || !s->above || !s->below || !s->nb13 || !s->vz_below || !s->vz_above) {
            P_(destroy)(s);
            return NULL;
        }
        const int piz = s->plate_iz;
        int q = 0;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                int pidx = j + ny * i;
                if (!plate_active[pidx]) continue;
                s->act[q] = pidx;
                s->above[q] = (piz + 1 < nz) ? P_(idx3)(s, i, j, piz + 1) : -1;
                s->below[q] = (piz - 1 >= 0) ? P_(idx3)(s, i, j, piz - 1) : -1;
                for (int t = 0; t < 13; ++t) {
                    int ii = i + DI[t], jj = j + DJ[t];
                    if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || !plate_active[jj + ny * ii]) {
                        ii = i; jj = j;
                    }
                    s->nb13[q * 13 + t] = jj + ny * ii;
                }
                if (piz > 0)
                    s->vz_below[q] = P_(is_solid)(s->cell_type[P_(idx3)(s, i, j, piz - 1)])
                                     ? -1 : (piz - 1) + (nz - 1) * (j + ny * i);
                else
                    s->vz_below[q] = -1;
                if (piz < nz - 1)
                    s->vz_above[q] = P_(is_solid)(s->cell_type[P_(idx3)(s, i, j, piz + 1)])
                                     ? -1 : piz + (nz - 1) * (j + ny * i);
                else
                    s->vz_above[q] = -1;
                ++q;
            }
    }
    /* Solid cells hold zero pressure (:427-433); calloc already did that. */
    return s;
}

/* Per-face absorption scale on sigma_max (the engine's documented extension). */
EXPORT int P_(set_face_absorption)(S_* s, const R* a6)
{
    if (!s || !a6) return -1;
    free(s->cell_a); s->cell_a = NULL;
    P_(build_damping)(s, a6);
    return 0;
}

/* Per-cell absorption a_c = alpha_c*dt in place of the PML profile. */
EXPORT int P_(set_cell_absorption)(S_* s, const R* a_cell)
{
    if (!s || !a_cell) return -1;
    if (!s->cell_a) s->cell_a = (R*)malloc((size_t)s->n * sizeof(R));
    if (!s->cell_a) return -1;
    memcpy(s->cell_a, a_cell, (size_t)s->n * sizeof(R));
    R ones[6] = {L(1.0), L(1.0), L(1.0), L(1.0), L(1.0), L(1.0)};
    P_(build_damping)(s, ones);
    return 0;
}

/* fdtd_set_face_fractions (acoustic_fdtd.cpp:1064-1077). */
EXPORT int P_(set_face_fractions)(S_* s, const R* fx, const R* fy, const R* fz)
{
    if (!s) return -1;
    if (fx) memcpy(s->vxf, fx, (size_t)(s->nx - 1) * s->ny * s->nz * sizeof(R));
    if (fy) memcpy(s->vyf, fy, (size_t)s->nx * (s->ny - 1) * s->nz * sizeof(R));
    if (fz) memcpy(s->vzf, fz, (size_t)s->nx * s->ny * (s->nz - 1) * sizeof(R));
    if (fx || fy || fz) s->has_frac = 1;
    return 0;
}

/* fdtd_set_bridge_sources (acoustic_fdtd.cpp:798-830). */
EXPORT int P_(set_bridge_sources)(S_* s, int n, const int* idx, const R* wgt)
{
    if (!s || n <= 0 || !idx || !wgt) return -1;
    int* ni = (int*)malloc((size_t)n * sizeof(int));
    R* nw = (R*)malloc((size_t)n * sizeof(R));
    if (!ni || !nw) { free(ni); free(nw); return -1; }
    R sum = L(0.0);
    for (int q = 0; q < n; ++q) sum += (wgt[q] < L(0.0) ? -wgt[q] : wgt[q]);
    R scale = (sum > L(1e-12)) ? L(1.0) / sum : L(1.0);
    for (int q = 0; q < n; ++q) { ni[q] = idx[q]; nw[q] = wgt[q] * scale; }
    free(s->src_idx); free(s->src_wgt);
    s->src_idx = ni; s->src_wgt = nw; s->n_src = n;
    return 0;
}

/* fdtd_inject_bridge_drive (acoustic_fdtd.cpp:1699-1721). */
EXPORT int P_(inject_bridge_drive)(S_* s, const R* drives, R force_scale)
{
    if (!s) return -1;
    if (!s->src_idx || s->n_src == 0) return 0;
    if (!drives) return -1;
    R inv_dx2 = L(1.0) / (s->dx * s->dx);
    for (int q = 0; q < s->n_src; ++q) {
        int pidx = s->src_idx[q] / s->nz;
        s->ext_force[pidx] += force_scale * drives[q] * inv_dx2;
    }
    return 0;
}

/* fdtd_inject_plate_force (acoustic_fdtd.cpp:1723-1742). */
EXPORT int P_(inject_plate_force)(S_* s, int n, const int* pidx, const R* wgt, R total)
{
    if (!s || !pidx || !wgt) return -1;
    if (n <= 0 || total == L(0.0)) return 0;
    R inv_dx2 = L(1.0) / (s->dx * s->dx);
    for (int q = 0; q < n; ++q) {
        int p = pidx[q];
        if (p < 0 || p >= s->n_plate) continue;
        if (!s->plate_active[p]) continue;
        s->ext_force[p] += total * wgt[q] * inv_dx2;
    }
    return 0;
}

/* deposit_pressure_open (acoustic_fdtd.cpp:840-872): add into an open cell, or
 * split equally among its open face neighbours when the cell is solid. */
EXPORT int P_(add_pressure)(S_* s, int idx, R amp)
{
    if (!s || idx < 0 || idx >= s->n || amp == L(0.0)) return 0;
    if (!P_(is_solid)(s->cell_type[idx])) { s->p[idx] += amp; return 1; }
    int k = idx % s->nz, t = idx / s->nz, j = t % s->ny, i = t / s->ny;
    int nb[6], m = 0;
    if (i + 1 < s->nx) nb[m++] = P_(idx3)(s, i + 1, j, k);
    if (i - 1 >= 0)    nb[m++] = P_(idx3)(s, i - 1, j, k);
    if (j + 1 < s->ny) nb[m++] = P_(idx3)(s, i, j + 1, k);
    if (j - 1 >= 0)    nb[m++] = P_(idx3)(s, i, j - 1, k);
    if (k + 1 < s->nz) nb[m++] = P_(idx3)(s, i, j, k + 1);
    if (k - 1 >= 0)    nb[m++] = P_(idx3)(s, i, j, k - 1);
    int open = 0;
    for (int q = 0; q < m; ++q) if (!P_(is_solid)(s->cell_type[nb[q]])) ++open;
    if (open <= 0) return 0;
    R share = amp / (R)open;
    for (int q = 0; q < m; ++q)
        if (!P_(is_solid)(s->cell_type[nb[q]])) s->p[nb[q]] += share;
    return open;
}

/* plate_step (acoustic_fdtd.cpp:984-1053). Returns 0 or -3. */
static int P_(plate_step)(S_* s)
{
    static const R W13[13] = {20, -8, -8, -8, -8, 2, 2, 2, 2, 1, 1, 1, 1};
    for (int q = 0; q < s->n_act; ++q) {
        int pidx = s->act[q];
        const int* nb = s->nb13 + q * 13;
        R bh = L(0.0), bhp = L(0.0);
        for (int t = 0; t < 13; ++t) bh += W13[t] * s->w[nb[t]];
        R pa = (s->above[q] >= 0) ? s->p[s->above[q]] : L(0.0);
        R pb = (s->below[q] >= 0) ? s->p[s->below[q]] : L(0.0);
        R fb = s->ext_force[pidx];
        for (int t = 0; t < 13; ++t) bhp += W13[t] * s->w_prev[nb[t]];
        R vel = s->w[pidx] - s->w_prev[pidx];
        R wn = s->w[pidx] + s->pl_vd * vel
             + s->pl_a * ((pb - pa) + fb)
             - s->pl_bh * bh
             - s->pl_bk * (bh - bhp);
        if (!isfinite((double)wn) || (wn < L(0.0) ? -wn : wn) > L(0.02)) {
            fprintf(stderr, "[oracle plate] UNSTABLE step=%d plate_node=%d w_new=%.3g m\n",
                    s->step_count, pidx, (double)wn);
            return -3;
        }
        s->w_tmp[pidx] = wn;
    }
    memset(s->ext_force, 0, (size_t)s->n_plate * sizeof(R));
    R* t = s->w_prev; s->w_prev = s->w; s->w = s->w_tmp; s->w_tmp = t;
    return 0;
}

/* Staggered 4th-order divergence (acoustic_fdtd.cpp:889-952); faces outside
 * the grid read as zero, fractions multiply each face when has_frac. */
static R P_(div_v)(const S_* s, int i, int j, int k)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const R* vx = s->vx; const R* vy = s->vy; const R* vz = s->vz;
#define GX(ii) (s->has_frac ? vx[k + nz * (j + ny * (ii))] * s->vxf[k + nz * (j + ny * (ii))] \
                            : vx[k + nz * (j + ny * (ii))])
#define GY(jj) (s->has_frac ? vy[k + nz * ((jj) + (ny - 1) * i)] * s->vyf[k + nz * ((jj) + (ny - 1) * i)] \
                            : vy[k + nz * ((jj) + (ny - 1) * i)])
#define GZ(kk) (s->has_frac ? vz[(kk) + (nz - 1) * (j + ny * i)] * s->vzf[(kk) + (nz - 1) * (j + ny * i)] \
                            : vz[(kk) + (nz - 1) * (j + ny * i)])
    R xp = (i < nx - 1) ? GX(i) : L(0.0);
    R xm = (i > 0) ? GX(i - 1) : L(0.0);
    R xpp = (i < nx - 2) ? GX(i + 1) : L(0.0);
    R xmm = (i > 1) ? GX(i - 2) : L(0.0);
    R yp = (j < ny - 1) ? GY(j) : L(0.0);
    R ym = (j > 0) ? GY(j - 1) : L(0.0);
    R ypp = (j < ny - 2) ? GY(j + 1) : L(0.0);
    R ymm = (j > 1) ? GY(j - 2) : L(0.0);
    R zp = (k < nz - 1) ? GZ(k) : L(0.0);
    R zm = (k > 0) ? GZ(k - 1) : L(0.0);
    R zpp = (k < nz - 2) ? GZ(k + 1) : L(0.0);
    R zmm = (k > 1) ? GZ(k - 2) : L(0.0);
#undef GX
#undef GY
#undef GZ
    const R C1 = (R)9 / (R)8, C2 = (R)(-1) / (R)24;
    return C1 * ((xp - xm) + (yp - ym) + (zp - zm))
         + C2 * ((xpp - xmm) + (ypp - ymm) + (zpp - zmm));
}

/* pressure_step (acoustic_fdtd.cpp:1081-1241): velocity, face BCs, plate
 * Vz injection, pressure, buffer rotation. */
static void P_(pressure_step)(S_* s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const R* p = s->p;
    const R vc = s->vel_coeff;
    const R C1 = (R)9 / (R)8, C2 = (R)(-1) / (R)24;
    /* velocity (:1099-1148) */
    for (int i = 0; i < nx - 1; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int v = k + nz * (j + ny * i);
                int Lc = P_(idx3)(s, i, j, k), Rc = P_(idx3)(s, i + 1, j, k);
                R g = (i > 0 && i < nx - 2)
                    ? C1 * (p[Rc] - p[Lc]) + C2 * (p[P_(idx3)(s, i + 2, j, k)] - p[P_(idx3)(s, i - 1, j, k)])
                    : p[Rc] - p[Lc];
                s->vx[v] = (s->vx[v] - vc * g) * s->vxd[v];
            }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny - 1; ++j)
            for (int k = 0; k < nz; ++k) {
                int v = k + nz * (j + (ny - 1) * i);
                int Lc = P_(idx3)(s, i, j, k), Rc = P_(idx3)(s, i, j + 1, k);
                R g = (j > 0 && j < ny - 2)
                    ? C1 * (p[Rc] - p[Lc]) + C2 * (p[P_(idx3)(s, i, j + 2, k)] - p[P_(idx3)(s, i, j - 1, k)])
                    : p[Rc] - p[Lc];
                s->vy[v] = (s->vy[v] - vc * g) * s->vyd[v];
            }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz - 1; ++k) {
                int v = k + (nz - 1) * (j + ny * i);
                int Lc = P_(idx3)(s, i, j, k), Rc = P_(idx3)(s, i, j, k + 1);
                R g = (k > 0 && k < nz - 2)
                    ? C1 * (p[Rc] - p[Lc]) + C2 * (p[P_(idx3)(s, i, j, k + 2)] - p[P_(idx3)(s, i, j, k - 1)])
                    : p[Rc] - p[Lc];
                s->vz[v] = (s->vz[v] - vc * g) * s->vzd[v];
            }
    /* closed faces (frac == 0) are zeroed (:1152-1154, list built at :297-323) */
    const int nvx = (nx - 1) * ny * nz, nvy = nx * (ny - 1) * nz, nvz = nx * ny * (nz - 1);
    for (int q = 0; q < nvx; ++q) if (s->vxf[q] == L(0.0)) s->vx[q] = L(0.0);
    for (int q = 0; q < nvy; ++q) if (s->vyf[q] == L(0.0)) s->vy[q] = L(0.0);
    for (int q = 0; q < nvz; ++q) if (s->vzf[q] == L(0.0)) s->vz[q] = L(0.0);
    /* plate velocity on the faces beside the plate (:1158-1163) */
    for (int q = 0; q < s->n_act; ++q) {
        int pidx = s->act[q];
        R vpl = (s->w[pidx] - s->w_prev[pidx]) * (L(1.0) / s->dt);
        if (s->vz_below[q] >= 0) s->vz[s->vz_below[q]] = vpl;
        if (s->vz_above[q] >= 0) s->vz[s->vz_above[q]] = vpl;
    }
    /* pressure on every non-solid cell (:1176-1234) */
    const R bulk = s->bulk_coeff;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int idx = P_(idx3)(s, i, j, k);
                if (P_(is_solid)(s->cell_type[idx])) continue;
                R dv = P_(div_v)(s, i, j, k);
                s->p_next[idx] = (p[idx] - bulk * dv) * s->pdamp[idx];
            }
    R* t = s->p; s->p = s->p_next; s->p_next = t;
}

/* check_stable (acoustic_fdtd.cpp:1245-1268). */
static int P_(check_stable)(S_* s)
{
    int start = s->stab_phase;
    s->stab_phase = (start + 1) % 1013;
    for (int q = start; q < s->n; q += 1013) {
        R v = s->p[q];
        if (!isfinite((double)v) || v > L(2e3) || v < L(-2e3)) {
            fprintf(stderr, "[oracle pressure] UNSTABLE step=%d cell=%d p=%.3g Pa\n",
                    s->step_count, q, (double)v);
            return -3;
        }
    }
    return 0;
}

/* fdtd_step (acoustic_fdtd.cpp:1272-1290). */
EXPORT int P_(step)(S_* s, int n_steps)
{
    if (!s) return -1;
    for (int q = 0; q < n_steps; ++q) {
        int rc = P_(plate_step)(s);
        if (rc) return rc;
        P_(pressure_step)(s);
        ++s->step_count;
        if ((s->step_count & 0xFF) == 0 && P_(check_stable)(s)) return -3;
    }
    return 0;
}

/* fdtd_sample_pressure_precomputed (acoustic_fdtd.cpp:1663-1676). */
EXPORT int P_(sample_pressure_precomputed)(const S_* s, int n_rec, const int* id8, const R* w8, R* out)
{
    if (!s || !id8 || !w8 || !out) return -1;
    const R* P = s->p;
    for (int r = 0; r < n_rec; ++r) {
        const int* id = id8 + r * 8;
        const R* w = w8 + r * 8;
        out[r] = w[0] * P[id[0]] + w[1] * P[id[1]] + w[2] * P[id[2]] + w[3] * P[id[3]]
               + w[4] * P[id[4]] + w[5] * P[id[5]] + w[6] * P[id[6]] + w[7] * P[id[7]];
    }
    return 0;
}

/* Room run: before step n add signal[n] at src_idx with the deposit rule, step,
 * then record every receiver with its precomputed 8-tap sampler. */
EXPORT int P_(run)(S_* s, int n_steps, int src_idx, const R* signal, int n_sig,
                   int n_rec, const int* id8, const R* w8, R* trace)
{
    if (!s) return -1;
    for (int q = 0; q < n_steps; ++q) {
        if (signal && src_idx >= 0 && s->step_count < n_sig)
            P_(add_pressure)(s, src_idx, signal[s->step_count]);
        int rc = P_(step)(s, 1);
        if (rc) return rc;
        if (n_rec > 0 && trace) P_(sample_pressure_precomputed)(s, n_rec, id8, w8, trace + (size_t)q * n_rec);
    }
    return 0;
}

EXPORT int P_(get_step_count)(const S_* s) { return s ? s->step_count : 0; }
EXPORT R P_(get_dt)(const S_* s) { return s ? s->dt : L(0.0); }

/* fdtd_reset (acoustic_fdtd.cpp:1297-1310): P, plate and V are zeroed. */
EXPORT int P_(reset)(S_* s)
{
    if (!s) return -1;
    memset(s->p, 0, (size_t)s->n * sizeof(R));
    memset(s->w, 0, (size_t)s->n_plate * sizeof(R));
    memset(s->w_prev, 0, (size_t)s->n_plate * sizeof(R));
    memset(s->ext_force, 0, (size_t)s->n_plate * sizeof(R));
    memset(s->vx, 0, (size_t)(s->nx - 1) * s->ny * s->nz * sizeof(R));
    memset(s->vy, 0, (size_t)s->nx * (s->ny - 1) * s->nz * sizeof(R));
    memset(s->vz, 0, (size_t)s->nx * s->ny * (s->nz - 1) * sizeof(R));
    s->step_count = 0;
    return 0;
}

/* Field copies with the exact-length check (acoustic_fdtd.cpp:1314-1330, :1399-1430). */
EXPORT int P_(get_pressure_field)(const S_* s, R* out, int len)
{
    if (!s || !out) return -1;
    if (len != s->n) return -2;
    memcpy(out, s->p, (size_t)s->n * sizeof(R));
    return 0;
}
EXPORT int P_(get_velocity_x)(const S_* s, R* out, int len)
{
    if (!s || !out) return -1;
    if (len != (s->nx - 1) * s->ny * s->nz) return -2;
    memcpy(out, s->vx, (size_t)len * sizeof(R));
    return 0;
}
EXPORT int P_(get_velocity_y)(const S_* s, R* out, int len)
{
    if (!s || !out) return -1;
    if (len != s->nx * (s->ny - 1) * s->nz) return -2;
    memcpy(out, s->vy, (size_t)len * sizeof(R));
    return 0;
}
EXPORT int P_(get_velocity_z)(const S_* s, R* out, int len)
{
    if (!s || !out) return -1;
    if (len != s->nx * s->ny * (s->nz - 1)) return -2;
    memcpy(out, s->vz, (size_t)len * sizeof(R));
    return 0;
}
EXPORT int P_(get_plate_displacement)(const S_* s, R* out, int len)
{
    if (!s || !out) return -1;
    if (len != s->n_plate) return -2;
    memcpy(out, s->w, (size_t)len * sizeof(R));
    return 0;
}
EXPORT int P_(get_p_damp)(const S_* s, R* out, int len)
{
    if (!s || !out) return -1;
    if (len != s->n) return -2;
    memcpy(out, s->pdamp, (size_t)len * sizeof(R));
    return 0;
}

/* Trilinear weights and taps shared by the samplers (acoustic_fdtd.cpp:1355-1395,
 * :1567-1596): clamp to [0, n-1], truncate, 8 corners in a fixed order. */
static void P_(taps)(int nxa, int nya, int nza, R gx, R gy, R gz,
                     int* i0, int* i1, int* j0, int* j1, int* k0, int* k1, R* w8)
{
    if (gx < L(0.0)) gx = L(0.0);
    if (gx > (R)(nxa - 1)) gx = (R)(nxa - 1);
    if (gy < L(0.0)) gy = L(0.0);
    if (gy > (R)(nya - 1)) gy = (R)(nya - 1);
    if (gz < L(0.0)) gz = L(0.0);
    if (gz > (R)(nza - 1)) gz = (R)(nza - 1);
    /* a NaN coordinate would make the reference read out of bounds; it is
     * mapped to 0 here (documented divergence on invalid input) */
    if (gx != gx) gx = L(0.0);
    if (gy != gy) gy = L(0.0);
    if (gz != gz) gz = L(0.0);
    *i0 = (int)gx; *i1 = (*i0 < nxa - 1) ? *i0 + 1 : *i0;
    *j0 = (int)gy; *j1 = (*j0 < nya - 1) ? *j0 + 1 : *j0;
    *k0 = (int)gz; *k1 = (*k0 < nza - 1) ? *k0 + 1 : *k0;
    R fx = gx - (R)*i0, fy = gy - (R)*j0, fz = gz - (R)*k0;
    w8[0] = (1 - fx) * (1 - fy) * (1 - fz);
    w8[1] = (fx) * (1 - fy) * (1 - fz);
    w8[2] = (1 - fx) * (fy) * (1 - fz);
    w8[3] = (fx) * (fy) * (1 - fz);
    w8[4] = (1 - fx) * (1 - fy) * (fz);
    w8[5] = (fx) * (1 - fy) * (fz);
    w8[6] = (1 - fx) * (fy) * (fz);
    w8[7] = (fx) * (fy) * (fz);
}

/* axis: -1 pressure, 0/1/2 = Vx/Vy/Vz with their half-cell shift and sizes. */
static void P_(sampler)(const S_* s, int axis, const R* xyz, int* id8, R* w8)
{
    int nxa = s->nx - (axis == 0), nya = s->ny - (axis == 1), nza = s->nz - (axis == 2);
    R gx = xyz[0] - (axis == 0 ? L(0.5) : L(0.0));
    R gy = xyz[1] - (axis == 1 ? L(0.5) : L(0.0));
    R gz = xyz[2] - (axis == 2 ? L(0.5) : L(0.0));
    int i0, i1, j0, j1, k0, k1;
    P_(taps)(nxa, nya, nza, gx, gy, gz, &i0, &i1, &j0, &j1, &k0, &k1, w8);
    /* every field's flat index is k + nza*(j + nya*i) in its own shape */
#define FI(a, b, c) ((c) + nza * ((b) + nya * (a)))
    id8[0] = FI(i0, j0, k0); id8[1] = FI(i1, j0, k0); id8[2] = FI(i0, j1, k0); id8[3] = FI(i1, j1, k0);
    id8[4] = FI(i0, j0, k1); id8[5] = FI(i1, j0, k1); id8[6] = FI(i0, j1, k1); id8[7] = FI(i1, j1, k1);
#undef FI
}

EXPORT int P_(precompute_pressure_samplers)(const S_* s, int n, const R* xyz, int* id8, R* w8)
{
    if (!s || !xyz || !id8 || !w8) return -1;
    for (int r = 0; r < n; ++r) P_(sampler)(s, -1, xyz + 3 * r, id8 + 8 * r, w8 + 8 * r);
    return 0;
}

EXPORT int P_(precompute_velocity_samplers)(const S_* s, int n, const R* xyz,
                                            int* xi, R* xw, int* yi, R* yw, int* zi, R* zw)
{
    if (!s || !xyz || !xi || !xw || !yi || !yw || !zi || !zw) return -1;
    for (int r = 0; r < n; ++r) {
        P_(sampler)(s, 0, xyz + 3 * r, xi + 8 * r, xw + 8 * r);
        P_(sampler)(s, 1, xyz + 3 * r, yi + 8 * r, yw + 8 * r);
        P_(sampler)(s, 2, xyz + 3 * r, zi + 8 * r, zw + 8 * r);
    }
    return 0;
}

/* Direct (not precomputed) trilinear sample: accumulates from 0 in tap order
 * (acoustic_fdtd.cpp:1381-1389, :1456-1464). */
static R P_(sample_one)(const S_* s, int axis, const R* xyz)
{
    int id8[8]; R w8[8];
    P_(sampler)(s, axis, xyz, id8, w8);
    const R* f = axis < 0 ? s->p : axis == 0 ? s->vx : axis == 1 ? s->vy : s->vz;
    R v = L(0.0);
    for (int t = 0; t < 8; ++t) v += w8[t] * f[id8[t]];
    return v;
}

EXPORT int P_(sample_pressure)(const S_* s, int n, const R* xyz, R* out)
{
    if (!s || !xyz || !out) return -1;
    for (int r = 0; r < n; ++r) out[r] = P_(sample_one)(s, -1, xyz + 3 * r);
    return 0;
}

EXPORT int P_(sample_velocity)(const S_* s, int n, const R* xyz, R* ox, R* oy, R* oz)
{
    if (!s || !xyz || !ox || !oy || !oz) return -1;
    for (int r = 0; r < n; ++r) {
        ox[r] = P_(sample_one)(s, 0, xyz + 3 * r);
        oy[r] = P_(sample_one)(s, 1, xyz + 3 * r);
        oz[r] = P_(sample_one)(s, 2, xyz + 3 * r);
    }
    return 0;
}

/* fdtd_sample_velocity_precomputed (acoustic_fdtd.cpp:1678-1697): one running
 * sum per component from 0. */
EXPORT int P_(sample_velocity_precomputed)(const S_* s, int n, const int* xi, const R* xw,
                                           const int* yi, const R* yw, const int* zi, const R* zw,
                                           R* ox, R* oy, R* oz)
{
    if (!s || !xi || !xw || !yi || !yw || !zi || !zw || !ox || !oy || !oz) return -1;
    for (int r = 0; r < n; ++r) {
        R a = L(0.0), b = L(0.0), c = L(0.0);
        for (int t = 0; t < 8; ++t) {
            a += xw[8 * r + t] * s->vx[xi[8 * r + t]];
            b += yw[8 * r + t] * s->vy[yi[8 * r + t]];
            c += zw[8 * r + t] * s->vz[zi[8 * r + t]];
        }
        ox[r] = a; oy[r] = b; oz[r] = c;
    }
    return 0;
}

/* fdtd_get_surface_emission (acoustic_fdtd.cpp:1540-1563). */
EXPORT int P_(get_surface_emission)(const S_* s, int n, const R* xyz, const R* nrm, R* op, R* ovn)
{
    if (!s || !xyz || !nrm || !op || !ovn) return -1;
    for (int q = 0; q < n; ++q) {
        op[q] = P_(sample_one)(s, -1, xyz + 3 * q);
        R a = P_(sample_one)(s, 0, xyz + 3 * q);
        R b = P_(sample_one)(s, 1, xyz + 3 * q);
        R c = P_(sample_one)(s, 2, xyz + 3 * q);
        ovn[q] = a * nrm[3 * q] + b * nrm[3 * q + 1] + c * nrm[3 * q + 2];
    }
    return 0;
}

/* Plate samplers (acoustic_fdtd.cpp:1332-1353, :1744-1760). */
EXPORT int P_(sample_plate_displacement_batch)(const S_* s, int n, const int* i4, const R* w4, R* out)
{
    if (!s || !i4 || !w4 || !out) return -1;
    for (int q = 0; q < n; ++q)
        out[q] = w4[4 * q] * s->w[i4[4 * q]] + w4[4 * q + 1] * s->w[i4[4 * q + 1]]
               + w4[4 * q + 2] * s->w[i4[4 * q + 2]] + w4[4 * q + 3] * s->w[i4[4 * q + 3]];
    return 0;
}

EXPORT int P_(sample_plate_weighted)(const S_* s, int n, const int* pidx, const R* wgt, R* out)
{
    if (!s || !pidx || !wgt || !out) return -1;
    R acc = L(0.0);
    for (int q = 0; q < n; ++q) {
        int p = pidx[q];
        if (p < 0 || p >= s->n_plate) continue;
        acc += s->w[p] * wgt[q];
    }
    *out = acc;
    return 0;
}

EXPORT void P_(set_pressure_field)(S_* s, const R* in) { memcpy(s->p, in, (size_t)s->n * sizeof(R)); }
