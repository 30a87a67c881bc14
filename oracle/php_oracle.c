/*
 * php_oracle.c -- TEST INFRASTRUCTURE: the parity checker and the timed CPU
 * baseline of the B200 FDTD path.  Nothing in the product links it.
 *
 * A CPU restatement of PhP_FDTD's time-step loop (fdtd.c:3116-3884) on one
 * domain, in the reference's own layout (double [nx][ny][nz + 2 halo], z
 * fastest, fdtd.c:261-284) and with its per-cell arithmetic as written:
 * CPML b/c recomputed with exp() in every PML cell and step, rotation
 * cos/sin evaluated per cell, the ADE and ion updates in source order.  The
 * coefficients are derived here independently of libphpfdtd.
 *
 * One deliberate difference: in the tensor ADE update (fdtd.c:3465-3475)
 * the reference forms P^{n+1}[id] from tempvec[0..2] while tempvec[id+1..2]
 * are still unassigned, and overwrites P_ADEo[id] before later components
 * read it.  Both only matter when the ADE matrices have non-zero
 * off-diagonal entries (otherwise those products are exact zeros); there the
 * reference reads uninitialised memory.  This restatement (and the device
 * path) evaluates the tensor update as written in fdtd.c's comments: all
 * of tempvec from P^n and P^{n-1}, then P^{n+1} = gdt2p1_inv . tempvec.
 *
 * Built with -O2 -ffp-contract=off (oracle/Makefile): IEEE double in source
 * order, like the reference binary compiled the same way.
 */
#include "php_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define EPS_INF 20.0 /* fdtd.c:202 */

static char g_err[512];

typedef struct {
    double eps[9], epsi[9], eps_inv[9];
    double sigma, anglez, anglex;
    int use_ade, natom;
    double gdt2p1_inv[9], gdt2m1[9], wp2[9];
    const double *qezv, *qezm, *dmm;
} omat;

struct oracle_ctx {
    php_desc d;
    int nx, ny, nz, L, nzh;
    double *Ex, *Ey, *Ez, *Dx, *Dy, *Dz, *Hx, *Hy, *Hz;
    double *PSI_Dxy, *PSI_Dxz, *PSI_Dyx, *PSI_Dyz, *PSI_Hxy, *PSI_Hxz, *PSI_Hyx, *PSI_Hyz;
    double *PSI_Dzx, *PSI_Dzy, *PSI_Hzx, *PSI_Hzy;
    double *pml_sigma[3], *pml_kappa[3], *pml_alpha[3];
    int* medium; /* [nx][ny][nz] */
    omat* mats;
    int nmat, n3max;
    double *r, *v;    /* [cell][n3max] */
    double *P, *Po;   /* [cell][3] */
    double* owned;    /* ion coefficient copies */
    int t;
};

const char* oracle_last_error(void) { return g_err; }

void oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* field index with the halo of fdtd.c:274: k = -1 .. nz */
#define FI(o, i, j, k) ((((size_t)(i) * (o)->ny + (j)) * (o)->nzh) + (size_t)((k) + 1))
#define CI(o, i, j, k) ((((size_t)(i) * (o)->ny + (j)) * (o)->nz) + (size_t)(k))

/* inverse_dielectric_tensor real part, fdtd.c:555-625 */
static int eps_inverse(const double* e, const double* ei, double* inv)
{
    double det_real = e[0] * (e[4] * e[8] - e[5] * e[7]) - e[1] * (e[3] * e[8] - e[5] * e[6]) + e[2] * (e[3] * e[7] - e[4] * e[6]);
    double det_imag = ei[0] * (ei[4] * ei[8] - ei[5] * ei[7]) - ei[1] * (ei[3] * ei[8] - ei[5] * ei[6]) +
                      ei[2] * (ei[3] * ei[7] - ei[4] * ei[6]);
    double det_magnitude = sqrt(det_real * det_real + det_imag * det_imag);
    if (fabs(det_magnitude) < 1e-12) return -1;
    double a = det_real / (det_real * det_real + det_imag * det_imag);
    double b = -det_imag / (det_real * det_real + det_imag * det_imag);
    inv[0] = a * (e[4] * e[8] - e[5] * e[7]) - b * (ei[4] * ei[8] - ei[5] * ei[7]);
    inv[1] = a * (e[2] * e[7] - e[1] * e[8]) - b * (ei[2] * ei[7] - ei[1] * ei[8]);
    inv[2] = a * (e[1] * e[5] - e[2] * e[4]) - b * (ei[1] * ei[5] - ei[2] * ei[4]);
    inv[3] = a * (e[5] * e[6] - e[3] * e[8]) - b * (ei[5] * ei[6] - ei[3] * ei[8]);
    inv[4] = a * (e[0] * e[8] - e[2] * e[6]) - b * (ei[0] * ei[8] - ei[2] * ei[6]);
    inv[5] = a * (e[2] * e[3] - e[0] * e[5]) - b * (ei[2] * ei[3] - ei[0] * ei[5]);
    inv[6] = a * (e[3] * e[7] - e[4] * e[6]) - b * (ei[3] * ei[7] - ei[4] * ei[6]);
    inv[7] = a * (e[1] * e[6] - e[0] * e[7]) - b * (ei[1] * ei[6] - ei[0] * ei[7]);
    inv[8] = a * (e[0] * e[4] - e[1] * e[3]) - b * (ei[0] * ei[4] - ei[1] * ei[3]);
    return 0;
}

/* determinant / adjoint / inverse, fdtd.c:205-258 */
static int inv3(double m[3][3], double inv[3][3])
{
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    if (fabs(det) < 1e-12) return -1;
    double adj[3][3];
    adj[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    adj[0][1] = -(m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    adj[0][2] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    adj[1][0] = -(m[0][1] * m[2][2] - m[0][2] * m[2][1]);
    adj[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]);
    adj[1][2] = -(m[0][0] * m[2][1] - m[0][1] * m[2][0]);
    adj[2][0] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]);
    adj[2][1] = -(m[0][0] * m[1][2] - m[0][2] * m[1][0]);
    adj[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) inv[i][j] = adj[j][i] / det;
    return 0;
}

/* ADE coefficients, fdtd.c:2478-2528 */
static int ade_coefficients(omat* m, double f, double dt)
{
    double epsr1[3][3], epsr1_inv[3][3], gama[3][3], gp[3][3], gm[3][3], gpi[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) epsr1[a][b] = m->eps[a * 3 + b] - (a == b ? EPS_INF : 0.0);
    if (epsr1[0][0] >= 0 || epsr1[1][1] >= 0 || epsr1[2][2] >= 0) return -1;
    if (inv3(epsr1, epsr1_inv)) return -1;
    const double* ei = m->epsi;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            gama[a][b] = -(ei[a * 3 + 0] * epsr1_inv[0][b] + ei[a * 3 + 1] * epsr1_inv[1][b] + ei[a * 3 + 2] * epsr1_inv[2][b]) * f * 2.0 * M_PI;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            m->wp2[a * 3 + b] = -f * f * 4.0 * M_PI * M_PI * epsr1[a][b] +
                                f * 2.0 * M_PI * (gama[a][0] * ei[0 * 3 + b] + gama[a][1] * ei[1 * 3 + b] + gama[a][2] * ei[2 * 3 + b]);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            gp[a][b] = +gama[a][b] * dt / 2.0;
            gm[a][b] = -gama[a][b] * dt / 2.0;
            if (a == b) { gp[a][b] += 1.0; gm[a][b] += 1.0; }
        }
    if (inv3(gp, gpi)) return -1;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            m->gdt2p1_inv[a * 3 + b] = gpi[a][b];
            m->gdt2m1[a * 3 + b] = gm[a][b];
        }
    return 0;
}

/* init_pml, fdtd.c:962-989 */
static void init_pml(int size, double delta, const php_desc* d, double** s, double** k, double** a)
{
    *s = (double*)calloc(size > 0 ? size : 1, sizeof(double));
    *k = (double*)calloc(size > 0 ? size : 1, sizeof(double));
    *a = (double*)calloc(size > 0 ? size : 1, sizeof(double));
    if (size <= 0) return;
    double m = 3.0, kappa_max = 7.0, alpha_max = 0.05;
    double eta0 = sqrt(d->mu0 / d->epsilon0);
    double sigma_max = -(m + 1) * log(d->pml_reflection) / (2.0 * eta0 * delta * size);
    for (int i = 0; i < size; i++) {
        double r = (double)(size - i) / size;
        (*s)[i] = sigma_max * pow(r, m);
        (*k)[i] = 1.0 + (kappa_max - 1.0) * pow(r, m);
        (*a)[i] = alpha_max * (1.0 - r);
    }
}

/* calculate_source_value, fdtd.c:1923-1947 */
static double source_value(const php_source_desc* s, double time)
{
    if (time < s->start_time || time > s->end_time) return 0.0;
    switch (s->type) {
    case 0: return s->amplitude * exp(-pow((time - s->t0) / s->tau, 2));
    case 1: return s->amplitude * sin(2 * M_PI * s->frequency * time);
    case 2: {
        double t_shift = time - s->t0;
        double arg = M_PI * M_PI * s->frequency * s->frequency * t_shift * t_shift;
        return s->amplitude * (1.0 - 2.0 * arg) * exp(-arg);
    }
    case 3: return s->amplitude * sin(2 * M_PI * s->frequency * time) * exp(-pow((time - s->t0) / s->tau, 2));
    default: return 0.0;
    }
}

void oracle_destroy(oracle_ctx* o)
{
    if (!o) return;
    double* arrs[] = {o->Ex, o->Ey, o->Ez, o->Dx, o->Dy, o->Dz, o->Hx, o->Hy, o->Hz, o->PSI_Dxy, o->PSI_Dxz,
                      o->PSI_Dyx, o->PSI_Dyz, o->PSI_Hxy, o->PSI_Hxz, o->PSI_Hyx, o->PSI_Hyz, o->PSI_Dzx,
                      o->PSI_Dzy, o->PSI_Hzx, o->PSI_Hzy, o->r, o->v, o->P, o->Po, o->owned};
    for (size_t q = 0; q < sizeof(arrs) / sizeof(arrs[0]); q++) free(arrs[q]);
    for (int a = 0; a < 3; a++) { free(o->pml_sigma[a]); free(o->pml_kappa[a]); free(o->pml_alpha[a]); }
    free(o->medium);
    free(o->mats);
    free(o);
}

int oracle_create(const php_desc* d, oracle_ctx** out)
{
    *out = NULL;
    if (!d || d->nx < 2 || d->ny < 2 || d->nz < 1 || d->num_materials < 1) {
        snprintf(g_err, sizeof(g_err), "bad description");
        return PHP_ERR_INPUT;
    }
    oracle_ctx* o = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
    o->d = *d;
    o->nx = d->nx; o->ny = d->ny; o->nz = d->nz; o->L = d->pml_thickness; o->nzh = d->nz + 2;
    const size_t nf = (size_t)o->nx * o->ny * o->nzh, nc = (size_t)o->nx * o->ny * o->nz;
    double** fields[9] = {&o->Ex, &o->Ey, &o->Ez, &o->Dx, &o->Dy, &o->Dz, &o->Hx, &o->Hy, &o->Hz};
    for (int q = 0; q < 9; q++) *fields[q] = (double*)calloc(nf, sizeof(double));
    const int L = o->L;
    const size_t xs = (size_t)2 * L * o->ny * o->nz, ys = (size_t)o->nx * 2 * L * o->nz;
    o->PSI_Dxy = calloc(xs + 1, 8); o->PSI_Dxz = calloc(xs + 1, 8); o->PSI_Hxy = calloc(xs + 1, 8); o->PSI_Hxz = calloc(xs + 1, 8);
    o->PSI_Dyx = calloc(ys + 1, 8); o->PSI_Dyz = calloc(ys + 1, 8); o->PSI_Hyx = calloc(ys + 1, 8); o->PSI_Hyz = calloc(ys + 1, 8);
    /* z-psi over the whole domain, as the reference allocates it on ranks
     * that touch the z-PML (fdtd.c:3040-3049) */
    o->PSI_Dzx = calloc(nc, 8); o->PSI_Dzy = calloc(nc, 8); o->PSI_Hzx = calloc(nc, 8); o->PSI_Hzy = calloc(nc, 8);
    init_pml(L, d->dx, d, &o->pml_sigma[0], &o->pml_kappa[0], &o->pml_alpha[0]);
    init_pml(L, d->dy, d, &o->pml_sigma[1], &o->pml_kappa[1], &o->pml_alpha[1]);
    init_pml(L, d->dz, d, &o->pml_sigma[2], &o->pml_kappa[2], &o->pml_alpha[2]);

    o->nmat = d->num_materials;
    o->mats = (omat*)calloc(o->nmat, sizeof(omat));
    size_t ion_total = 0;
    for (int m = 0; m < o->nmat; m++) ion_total += (size_t)18 * d->materials[m].natom + (size_t)9 * d->materials[m].natom * d->materials[m].natom;
    o->owned = (double*)calloc(ion_total + 1, sizeof(double));
    size_t ion_used = 0;
    for (int m = 0; m < o->nmat; m++) {
        const php_material_desc* s = &d->materials[m];
        omat* t = &o->mats[m];
        memcpy(t->eps, s->eps_re, sizeof(t->eps));
        memcpy(t->epsi, s->eps_im, sizeof(t->epsi));
        t->sigma = s->sigma; t->anglez = s->anglez; t->anglex = s->anglex;
        t->use_ade = s->use_ade; t->natom = s->natom;
        if (eps_inverse(t->eps, t->epsi, t->eps_inv)) {
            snprintf(g_err, sizeof(g_err), "Error: Singular dielectric tensor! (material %d)", m);
            oracle_destroy(o);
            return PHP_ERR_INPUT;
        }
        if (t->use_ade == 1 && ade_coefficients(t, d->source_frequency, d->dt)) {
            snprintf(g_err, sizeof(g_err), "ADE coefficients of material %d invalid", m);
            oracle_destroy(o);
            return PHP_ERR_INPUT;
        }
        if (t->natom > 0) {
            const int N = t->natom;
            double* q = o->owned + ion_used;
            memcpy(q, s->qezv, sizeof(double) * 9 * N);
            memcpy(q + 9 * N, s->qezm, sizeof(double) * 9 * N);
            memcpy(q + 18 * N, s->dmm, sizeof(double) * 9 * N * N);
            t->qezv = q; t->qezm = q + 9 * N; t->dmm = q + 18 * N;
            ion_used += (size_t)18 * N + (size_t)9 * N * N;
            if (3 * N > o->n3max) o->n3max = 3 * N;
        }
    }
    o->medium = (int*)malloc(nc * sizeof(int));
    int any_ade = 0;
    for (size_t c = 0; c < nc; c++) {
        int id = d->medium[c];
        if (id < 0 || id >= o->nmat) {
            snprintf(g_err, sizeof(g_err), "medium id %d outside the material table", id);
            oracle_destroy(o);
            return PHP_ERR_INPUT;
        }
        o->medium[c] = id;
        any_ade |= o->mats[id].use_ade == 1;
    }
    if (o->n3max) {
        o->r = (double*)calloc(nc * o->n3max, sizeof(double));
        o->v = (double*)calloc(nc * o->n3max, sizeof(double));
    }
    if (any_ade) {
        o->P = (double*)calloc(nc * 3, sizeof(double));
        o->Po = (double*)calloc(nc * 3, sizeof(double));
    }
    *out = o;
    return PHP_OK;
}

int oracle_get_step(const oracle_ctx* o) { return o->t; }

/* per-cell CPML b and c exactly as fdtd.c:3146-3151 */
static inline void cpml_bc(const oracle_ctx* o, int axis, int idx, double* kappa, double* b, double* c)
{
    double s = o->pml_sigma[axis][idx];
    *kappa = o->pml_kappa[axis][idx];
    double a = o->pml_alpha[axis][idx];
    double aw = s / (*kappa * o->d.epsilon0) + a / o->d.epsilon0;
    *b = exp(-aw * o->d.dt);
    *c = (aw > 1e-30) ? s / (*kappa * *kappa * o->d.epsilon0) * (*b - 1.0) / aw : 0.0;
}

/* H sweep, fdtd.c:3123-3231 */
static void sweep_h(oracle_ctx* o)
{
    const int nx = o->nx, ny = o->ny, nz = o->nz, L = o->L;
    const double dt = o->d.dt, mu0 = o->d.mu0, dxs = o->d.dx, dys = o->d.dy, dzs = o->d.dz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx - 1; i++) {
        for (int j = 0; j < ny - 1; j++) {
            for (int k = 0; k < nz; k++) {
                double PSI_Hxy_val = 0.0, PSI_Hxz_val = 0.0, PSI_Hyx_val = 0.0, PSI_Hyz_val = 0.0, PSI_Hzx_val = 0.0, PSI_Hzy_val = 0.0;
                double bh_x = 1.0, ch_x = dt, bh_y = 1.0, ch_y = dt, bh_z = 1.0, ch_z = dt;
                double kappa_x = 1.0, kappa_y = 1.0, kappa_z = 1.0;
                const size_t c = FI(o, i, j, k);
                double dEy_dz = (o->Ey[FI(o, i, j, k + 1)] - o->Ey[c]) / dzs;
                double dEz_dy = (o->Ez[FI(o, i, j + 1, k)] - o->Ez[c]) / dys;
                double dEz_dx = (o->Ez[FI(o, i + 1, j, k)] - o->Ez[c]) / dxs;
                double dEx_dz = (o->Ex[FI(o, i, j, k + 1)] - o->Ex[c]) / dzs;
                double dEx_dy = (o->Ex[FI(o, i, j + 1, k)] - o->Ex[c]) / dys;
                double dEy_dx = (o->Ey[FI(o, i + 1, j, k)] - o->Ey[c]) / dxs;
                int gk = k;
                if (L > 0 && i < L) {
                    cpml_bc(o, 0, i, &kappa_x, &bh_x, &ch_x);
                    size_t q = ((size_t)i * ny + j) * nz + k;
                    PSI_Hxy_val = o->PSI_Hxy[q];
                    PSI_Hxz_val = o->PSI_Hxz[q];
                    o->PSI_Hxy[q] = bh_x * PSI_Hxy_val + ch_x * (dEz_dx / mu0);
                    o->PSI_Hxz[q] = bh_x * PSI_Hxz_val + ch_x * (-dEy_dx / mu0);
                } else if (L > 0 && i >= nx - L) {
                    int idx = nx - 1 - i;
                    cpml_bc(o, 0, idx, &kappa_x, &bh_x, &ch_x);
                    size_t q = ((size_t)(L + idx) * ny + j) * nz + k;
                    PSI_Hxy_val = o->PSI_Hxy[q];
                    PSI_Hxz_val = o->PSI_Hxz[q];
                    o->PSI_Hxy[q] = bh_x * PSI_Hxy_val + ch_x * (dEz_dx / mu0);
                    o->PSI_Hxz[q] = bh_x * PSI_Hxz_val + ch_x * (-dEy_dx / mu0);
                }
                if (L > 0 && j < L) {
                    cpml_bc(o, 1, j, &kappa_y, &bh_y, &ch_y);
                    size_t q = ((size_t)i * 2 * L + j) * nz + k;
                    PSI_Hyx_val = o->PSI_Hyx[q];
                    PSI_Hyz_val = o->PSI_Hyz[q];
                    o->PSI_Hyx[q] = bh_y * PSI_Hyx_val + ch_y * (-dEz_dy / mu0);
                    o->PSI_Hyz[q] = bh_y * PSI_Hyz_val + ch_y * (dEx_dy / mu0);
                } else if (j >= ny - L) {
                    int idx = ny - 1 - j;
                    cpml_bc(o, 1, idx, &kappa_y, &bh_y, &ch_y);
                    size_t q = ((size_t)i * 2 * L + (L + idx)) * nz + k;
                    PSI_Hyx_val = o->PSI_Hyx[q];
                    PSI_Hyz_val = o->PSI_Hyz[q];
                    o->PSI_Hyx[q] = bh_y * PSI_Hyx_val + ch_y * (-dEz_dy / mu0);
                    o->PSI_Hyz[q] = bh_y * PSI_Hyz_val + ch_y * (dEx_dy / mu0);
                }
                const int zp = (gk < L || gk >= nz - L);
                const size_t qc = CI(o, i, j, k);
                if (zp) {
                    int idx = (gk < L) ? gk : nz - 1 - gk;
                    cpml_bc(o, 2, idx, &kappa_z, &bh_z, &ch_z);
                    PSI_Hzx_val = o->PSI_Hzx[qc];
                    PSI_Hzy_val = o->PSI_Hzy[qc];
                }
                o->Hx[c] += dt * ((-dEz_dy / mu0) / kappa_y + PSI_Hyx_val + (dEy_dz / mu0) / kappa_z + PSI_Hzx_val);
                o->Hy[c] += dt * ((dEz_dx / mu0) / kappa_x + PSI_Hxy_val + (-dEx_dz / mu0) / kappa_z + PSI_Hzy_val);
                o->Hz[c] += dt * ((-dEy_dx / mu0) / kappa_x + PSI_Hxz_val + (dEx_dy / mu0) / kappa_y + PSI_Hyz_val);
                if (zp) {
                    o->PSI_Hzx[qc] = bh_z * PSI_Hzx_val + ch_z * (dEy_dz / mu0);
                    o->PSI_Hzy[qc] = bh_z * PSI_Hzy_val + ch_z * (-dEx_dz / mu0);
                }
            }
        }
    }
}

/* D sweep with the eps'' term, fdtd.c:3238-3356 */
static void sweep_d(oracle_ctx* o)
{
    const int nx = o->nx, ny = o->ny, nz = o->nz, L = o->L;
    const double dt = o->d.dt, dxs = o->d.dx, dys = o->d.dy, dzs = o->d.dz;
    const double f = o->d.source_frequency, eps0 = o->d.epsilon0;
#pragma omp parallel for schedule(static)
    for (int i = 1; i < nx - 1; i++) {
        for (int j = 1; j < ny - 1; j++) {
            for (int k = 0; k < nz; k++) {
                double PSI_Dxy_val = 0.0, PSI_Dxz_val = 0.0, PSI_Dyx_val = 0.0, PSI_Dyz_val = 0.0, PSI_Dzx_val = 0.0, PSI_Dzy_val = 0.0;
                double b_x = 1.0, c_x = dt, b_y = 1.0, c_y = dt, b_z = 1.0, c_z = dt;
                double kappa_x = 1.0, kappa_y = 1.0, kappa_z = 1.0;
                const size_t c = FI(o, i, j, k);
                double dHz_dy = (o->Hz[c] - o->Hz[FI(o, i, j - 1, k)]) / dys;
                double dHy_dz = (o->Hy[c] - o->Hy[FI(o, i, j, k - 1)]) / dzs;
                double dHx_dz = (o->Hx[c] - o->Hx[FI(o, i, j, k - 1)]) / dzs;
                double dHz_dx = (o->Hz[c] - o->Hz[FI(o, i - 1, j, k)]) / dxs;
                double dHy_dx = (o->Hy[c] - o->Hy[FI(o, i - 1, j, k)]) / dxs;
                double dHx_dy = (o->Hx[c] - o->Hx[FI(o, i, j - 1, k)]) / dys;
                int gk = k;
                if (L > 0 && i < L) {
                    cpml_bc(o, 0, i, &kappa_x, &b_x, &c_x);
                    size_t q = ((size_t)i * ny + j) * nz + k;
                    PSI_Dxy_val = o->PSI_Dxy[q];
                    PSI_Dxz_val = o->PSI_Dxz[q];
                    o->PSI_Dxy[q] = b_x * PSI_Dxy_val + c_x * (-dHz_dx);
                    o->PSI_Dxz[q] = b_x * PSI_Dxz_val + c_x * (dHy_dx);
                } else if (L > 0 && i >= nx - L) {
                    int idx = nx - 1 - i;
                    cpml_bc(o, 0, idx, &kappa_x, &b_x, &c_x);
                    size_t q = ((size_t)(L + idx) * ny + j) * nz + k;
                    PSI_Dxy_val = o->PSI_Dxy[q];
                    PSI_Dxz_val = o->PSI_Dxz[q];
                    o->PSI_Dxy[q] = b_x * PSI_Dxy_val + c_x * (-dHz_dx);
                    o->PSI_Dxz[q] = b_x * PSI_Dxz_val + c_x * (dHy_dx);
                }
                if (L > 0 && j < L) {
                    cpml_bc(o, 1, j, &kappa_y, &b_y, &c_y);
                    size_t q = ((size_t)i * 2 * L + j) * nz + k;
                    PSI_Dyx_val = o->PSI_Dyx[q];
                    PSI_Dyz_val = o->PSI_Dyz[q];
                    o->PSI_Dyx[q] = b_y * PSI_Dyx_val + c_y * (dHz_dy);
                    o->PSI_Dyz[q] = b_y * PSI_Dyz_val + c_y * (-dHx_dy);
                } else if (j >= ny - L) {
                    int idx = ny - 1 - j;
                    cpml_bc(o, 1, idx, &kappa_y, &b_y, &c_y);
                    size_t q = ((size_t)i * 2 * L + (L + idx)) * nz + k;
                    PSI_Dyx_val = o->PSI_Dyx[q];
                    PSI_Dyz_val = o->PSI_Dyz[q];
                    o->PSI_Dyx[q] = b_y * PSI_Dyx_val + c_y * (dHz_dy);
                    o->PSI_Dyz[q] = b_y * PSI_Dyz_val + c_y * (-dHx_dy);
                }
                const int zp = (gk < L || gk >= nz - L);
                const size_t qc = CI(o, i, j, k);
                if (zp) {
                    int idx = (gk < L) ? gk : nz - 1 - gk;
                    cpml_bc(o, 2, idx, &kappa_z, &b_z, &c_z);
                    PSI_Dzx_val = o->PSI_Dzx[qc];
                    PSI_Dzy_val = o->PSI_Dzy[qc];
                }
                o->Dx[c] += dt * ((dHz_dy) / kappa_y + PSI_Dyx_val + (-dHy_dz) / kappa_z + PSI_Dzx_val);
                o->Dy[c] += dt * ((-dHz_dx) / kappa_x + PSI_Dxy_val + (dHx_dz) / kappa_z + PSI_Dzy_val);
                o->Dz[c] += dt * ((dHy_dx) / kappa_x + PSI_Dxz_val + (-dHx_dy) / kappa_y + PSI_Dyz_val);
                if (zp) {
                    o->PSI_Dzx[qc] = b_z * PSI_Dzx_val + c_z * (-dHy_dz);
                    o->PSI_Dzy[qc] = b_z * PSI_Dzy_val + c_z * (dHx_dz);
                }
                const omat* m = &o->mats[o->medium[qc]];
                if (m->use_ade == 0) {
                    const double* e = m->epsi;
                    o->Dx[c] -= dt * f * 2.0 * 3.14159265 * (e[0] * o->Ex[c] + e[1] * o->Ey[c] + e[2] * o->Ez[c]) * eps0;
                    o->Dy[c] -= dt * f * 2.0 * 3.14159265 * (e[3] * o->Ex[c] + e[4] * o->Ey[c] + e[5] * o->Ez[c]) * eps0;
                    o->Dz[c] -= dt * f * 2.0 * 3.14159265 * (e[6] * o->Ex[c] + e[7] * o->Ey[c] + e[8] * o->Ez[c]) * eps0;
                }
            }
        }
    }
}

/* sources, fdtd.c:3363-3396 */
static void add_sources(oracle_ctx* o, double current_time)
{
    for (int s = 0; s < o->d.num_sources; s++) {
        const php_source_desc* src = &o->d.sources[s];
        double value = source_value(src, current_time);
        int i = src->x, j = src->y, k = src->z;
        if (i < 0 || i >= o->nx || j < 0 || j >= o->ny || k < 0 || k >= o->nz) continue;
        size_t c = FI(o, i, j, k);
        switch (src->component) {
        case 'x': o->Dx[c] += value * o->d.dt; break;
        case 'y': o->Dy[c] += value * o->d.dt; break;
        case 'z': o->Dz[c] += value * o->d.dt; break;
        }
    }
}

/* D -> E, ADE and ions, fdtd.c:3404-3528 */
static void sweep_e(oracle_ctx* o)
{
    const int nx = o->nx, ny = o->ny, nz = o->nz, n3max = o->n3max;
    const double dt = o->d.dt, eps0 = o->d.epsilon0;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; i++) {
        double a[192];
        for (int j = 0; j < ny; j++) {
            for (int k = 0; k < nz; k++) {
                const size_t c = FI(o, i, j, k), qc = CI(o, i, j, k);
                const omat* m = &o->mats[o->medium[qc]];
                const double* inv = m->eps_inv;
                const int natom = m->natom;
                double loss_factor = 1.0 / (1.0 + m->sigma * dt / (2 * eps0));
                double loss_term = (m->sigma * dt / (2 * eps0)) * loss_factor;
                double* r = o->r ? o->r + qc * n3max : NULL;
                double* v = o->v ? o->v + qc * n3max : NULL;
                double Pr[3];
                for (int iE = 0; iE < 3; iE++) {
                    Pr[iE] = 0.0;
                    for (int ia = 0; ia < natom; ia++)
                        for (int id = 0; id < 3; id++) Pr[iE] += m->qezv[ia * 9 + iE * 3 + id] * r[ia * 3 + id];
                }
                double Ea, Eb, Ec, Da, Db, Dc;
                const double Exv = o->Ex[c], Eyv = o->Ey[c], Ezv = o->Ez[c], Dxv = o->Dx[c], Dyv = o->Dy[c], Dzv = o->Dz[c];
                if (fabs(m->anglez) > 1e-10) {
                    Ea = Exv * cos(m->anglez) - Eyv * sin(m->anglez);
                    Eb = Exv * sin(m->anglez) + Eyv * cos(m->anglez);
                    Ec = Ezv;
                    Da = Dxv * cos(m->anglez) - Dyv * sin(m->anglez);
                    Db = Dxv * sin(m->anglez) + Dyv * cos(m->anglez);
                    Dc = Dzv;
                } else if (fabs(m->anglex) > 1e-10) {
                    Ea = Exv;
                    Eb = Eyv * cos(-m->anglex) - Ezv * sin(-m->anglex);
                    Ec = Eyv * sin(-m->anglex) + Ezv * cos(-m->anglex);
                    Da = Dxv;
                    Db = Dyv * cos(-m->anglex) - Dzv * sin(-m->anglex);
                    Dc = Dyv * sin(-m->anglex) + Dzv * cos(-m->anglex);
                } else {
                    Ea = Exv; Eb = Eyv; Ec = Ezv;
                    Da = Dxv; Db = Dyv; Dc = Dzv;
                }
                double Da_val = Da - Pr[0], Db_val = Db - Pr[1], Dc_val = Dc - Pr[2];
                double Ea_new, Eb_new, Ec_new;
                if (m->use_ade == 0) {
                    Ea_new = loss_factor * (inv[0] * Da_val + inv[1] * Db_val + inv[2] * Dc_val) / eps0;
                    Eb_new = loss_factor * (inv[3] * Da_val + inv[4] * Db_val + inv[5] * Dc_val) / eps0;
                    Ec_new = loss_factor * (inv[6] * Da_val + inv[7] * Db_val + inv[8] * Dc_val) / eps0;
                } else {
                    double* P = o->P + qc * 3;
                    double* Po = o->Po + qc * 3;
                    double tempvec[3], Pn[3];
                    for (int id = 0; id < 3; id++) {
                        tempvec[id] = 2.0 * P[id];
                        tempvec[id] += -m->gdt2m1[id * 3 + 0] * Po[0] - m->gdt2m1[id * 3 + 1] * Po[1] - m->gdt2m1[id * 3 + 2] * Po[2] +
                                       eps0 * dt * dt * (m->wp2[id * 3 + 0] * Ea + m->wp2[id * 3 + 1] * Eb + m->wp2[id * 3 + 2] * Ec);
                    }
                    for (int id = 0; id < 3; id++) {
                        Pn[id] = 0.0;
                        for (int kk = 0; kk < 3; kk++) Pn[id] += m->gdt2p1_inv[id * 3 + kk] * tempvec[kk];
                    }
                    for (int id = 0; id < 3; id++) { Po[id] = P[id]; P[id] = Pn[id]; }
                    Ea_new = (Da_val - P[0]) / eps0 / EPS_INF;
                    Eb_new = (Db_val - P[1]) / eps0 / EPS_INF;
                    Ec_new = (Dc_val - P[2]) / eps0 / EPS_INF;
                }
                Ea = Ea_new - loss_term * Ea_new;
                Eb = Eb_new - loss_term * Eb_new;
                Ec = Ec_new - loss_term * Ec_new;
                if (fabs(m->anglez) > 1e-10) {
                    o->Ex[c] = Ea * cos(m->anglez) + Eb * sin(m->anglez);
                    o->Ey[c] = -Ea * sin(m->anglez) + Eb * cos(m->anglez);
                    o->Ez[c] = Ec;
                } else if (fabs(m->anglex) > 1e-10) {
                    o->Ex[c] = Ea;
                    o->Ey[c] = Eb * cos(-m->anglex) + Ec * sin(-m->anglex);
                    o->Ez[c] = -Eb * sin(-m->anglex) + Ec * cos(-m->anglex);
                } else {
                    o->Ex[c] = Ea; o->Ey[c] = Eb; o->Ez[c] = Ec;
                }
                for (int ia = 0; ia < natom; ia++)
                    for (int id = 0; id < 3; id++) {
                        double acc = m->qezm[ia * 9 + 0 * 3 + id] * Ea + m->qezm[ia * 9 + 1 * 3 + id] * Eb + m->qezm[ia * 9 + 2 * 3 + id] * Ec;
                        for (int ja = 0; ja < natom; ja++)
                            for (int jd = 0; jd < 3; jd++)
                                acc -= m->dmm[ia * 3 * natom * 3 + id * natom * 3 + ja * 3 + jd] * r[ja * 3 + jd];
                        a[ia * 3 + id] = acc;
                    }
                for (int ia = 0; ia < natom; ia++)
                    for (int id = 0; id < 3; id++) {
                        int q = ia * 3 + id;
                        r[q] += v[q] * dt + 0.5 * a[q] * dt * dt;
                        v[q] += a[q] * dt;
                    }
            }
        }
    }
}

int oracle_step(oracle_ctx* o, int n)
{
    if (o->n3max > 192) {
        snprintf(g_err, sizeof(g_err), "natom above 64");
        return PHP_ERR_UNSUPPORTED;
    }
    for (int s = 0; s < n; s++) {
        double current_time = o->t * o->d.dt; /* fdtd.c:3117 */
        sweep_h(o);
        sweep_d(o);
        add_sources(o, current_time);
        sweep_e(o);
        o->t++;
    }
    return PHP_OK;
}

static double* comp_ptr(oracle_ctx* o, int comp)
{
    double* p[9] = {o->Ex, o->Ey, o->Ez, o->Dx, o->Dy, o->Dz, o->Hx, o->Hy, o->Hz};
    return (comp >= 0 && comp < 9) ? p[comp] : NULL;
}

int oracle_read_volume(oracle_ctx* o, int comp, double* out)
{
    double* f = comp_ptr(o, comp);
    if (!f) return PHP_ERR_INPUT;
    for (int i = 0; i < o->nx; i++)
        for (int j = 0; j < o->ny; j++)
            for (int k = 0; k < o->nz; k++) out[CI(o, i, j, k)] = f[FI(o, i, j, k)];
    return PHP_OK;
}

static double cell_value(oracle_ctx* o, int comp, size_t c)
{
    if (comp == PHP_EMAG) return sqrt(o->Ex[c] * o->Ex[c] + o->Ey[c] * o->Ey[c] + o->Ez[c] * o->Ez[c]);
    return comp_ptr(o, comp)[c];
}

/* save_field_slice_parallel on one rank, fdtd.c:999-1400 */
int oracle_read_slice_f64(oracle_ctx* o, int comp, char axis, int pos, double* out)
{
    if (comp < 0 || comp > 9) return PHP_ERR_INPUT;
    if (axis == 'z') {
        if (pos < 0 || pos >= o->nz) return PHP_ERR_INPUT;
        int local_z = pos + 1; /* fdtd.c:1029 on pointers already offset by the halo */
        for (int i = 0; i < o->nx; i++)
            for (int j = 0; j < o->ny; j++) out[(size_t)i * o->ny + j] = cell_value(o, comp, FI(o, i, j, local_z));
    } else if (axis == 'x') {
        if (pos < 0 || pos >= o->nx) return PHP_ERR_INPUT;
        for (int j = 0; j < o->ny; j++)
            for (int k = 0; k < o->nz; k++) out[(size_t)j * o->nz + k] = cell_value(o, comp, FI(o, pos, j, k));
    } else if (axis == 'y') {
        if (pos < 0 || pos >= o->ny) return PHP_ERR_INPUT;
        for (int i = 0; i < o->nx; i++)
            for (int k = 0; k < o->nz; k++) out[(size_t)i * o->nz + k] = cell_value(o, comp, FI(o, i, pos, k));
    } else {
        return PHP_ERR_INPUT;
    }
    return PHP_OK;
}

int oracle_read_point(oracle_ctx* o, int i, int j, int k, double* out9)
{
    if (i < 0 || i >= o->nx || j < 0 || j >= o->ny || k < -1 || k > o->nz) return PHP_ERR_INPUT;
    for (int q = 0; q < 9; q++) out9[q] = comp_ptr(o, q)[FI(o, i, j, k)];
    return PHP_OK;
}

int oracle_read_cell_state(oracle_ctx* o, int i, int j, int k, int* natom, double* r, double* v, double* p, double* po)
{
    if (i < 0 || i >= o->nx || j < 0 || j >= o->ny || k < 0 || k >= o->nz) return PHP_ERR_INPUT;
    size_t qc = CI(o, i, j, k);
    const omat* m = &o->mats[o->medium[qc]];
    if (natom) *natom = m->natom;
    for (int q = 0; q < 3 * m->natom; q++) {
        if (r) r[q] = o->r[qc * o->n3max + q];
        if (v) v[q] = o->v[qc * o->n3max + q];
    }
    for (int q = 0; q < 3; q++) {
        if (p) p[q] = m->use_ade == 1 ? o->P[qc * 3 + q] : 0.0;
        if (po) po[q] = m->use_ade == 1 ? o->Po[qc * 3 + q] : 0.0;
    }
    return PHP_OK;
}

/* fdtd.c:3537-3597 */
int oracle_diagnostics(oracle_ctx* o, php_diag* out)
{
    double local_max_E = 0.0, local_max_Ex = 0.0, local_max_r = 0.0;
    int max_i = -1, max_j = -1, max_k = -1, max_atom = -1, max_dir = -1;
    for (int i = 0; i < o->nx; i++)
        for (int j = 0; j < o->ny; j++)
            for (int k = 0; k < o->nz; k++) {
                size_t c = FI(o, i, j, k);
                double E_mag = sqrt(o->Ex[c] * o->Ex[c] + o->Ey[c] * o->Ey[c] + o->Ez[c] * o->Ez[c]);
                double Ex_mag = fabs(o->Ex[c]);
                if (E_mag > local_max_E) local_max_E = E_mag;
                if (Ex_mag > local_max_Ex) local_max_Ex = Ex_mag;
            }
    for (int i = 0; i < o->nx; i++)
        for (int j = 0; j < o->ny; j++)
            for (int k = 0; k < o->nz; k++) {
                size_t qc = CI(o, i, j, k);
                int natom = o->mats[o->medium[qc]].natom;
                for (int a = 0; a < natom; a++)
                    for (int d = 0; d < 3; d++) {
                        double r_val = fabs(o->r[qc * o->n3max + a * 3 + d]);
                        if (r_val > local_max_r) {
                            local_max_r = r_val;
                            max_i = i; max_j = j; max_k = k; max_atom = a; max_dir = d;
                        }
                    }
            }
    out->max_e = local_max_E;
    out->max_ex = local_max_Ex;
    out->max_r = local_max_r;
    out->argmax_r[0] = max_i; out->argmax_r[1] = max_j; out->argmax_r[2] = max_k;
    out->argmax_r[3] = max_atom; out->argmax_r[4] = max_dir;
    return PHP_OK;
}
