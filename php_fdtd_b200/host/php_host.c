/*
 * php_host.c -- configuration, material data, medium map and output files
 * for the B200 drop-in of PhP_FDTD's solver.
 *
 * Written against the behaviour of the reference's fdtd.c set-up code (cited
 * per function).  Parsing goes through the same C library scanners
 * (sscanf/strtok/atoi/atof/strtod) so that every accepted spelling, default
 * and quirk of a .cfg file means the same thing here.  Arithmetic that feeds
 * the time loop (the SiO2 built-in, the CFL time step) keeps the reference's
 * expression order; this file is compiled with FP contraction off.
 */
#define _GNU_SOURCE
#include "php_host.h"
#include "php_serve.h"

#include <ctype.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static void set_err(char* err, size_t n, const char* fmt, ...)
{
    if (!err || !n) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, n, fmt, ap);
    va_end(ap);
}

static void add_warning(php_cfg* c, const char* fmt, ...)
{
    size_t used = strlen(c->warnings);
    if (used + 2 >= sizeof(c->warnings)) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->warnings + used, sizeof(c->warnings) - used, fmt, ap);
    va_end(ap);
}

/* trim(), fdtd.c:182-199: strip leading and trailing white space in place. */
static void trim(char* s)
{
    int i = 0, j = 0;
    while (isspace((unsigned char)s[i])) i++;
    while (s[i] != '\0') s[j++] = s[i++];
    s[j] = '\0';
    j = (int)strlen(s) - 1;
    while (j >= 0 && isspace((unsigned char)s[j])) s[j--] = '\0';
}

/* ---------------------------------------------------------------- materials */

static void material_vacuum(php_host_material* m, const char* name)
{
    memset(m, 0, sizeof(*m));
    snprintf(m->name, sizeof(m->name), "%s", name);
    m->eps_re[0] = m->eps_re[4] = m->eps_re[8] = 1.0;
}

/* create_material_library, fdtd.c:628-715: ids 0..3 (vacuum, SiO2 at the
 * source wavenumber, a biaxial crystal, a lossy medium). */
static void material_library(php_cfg* c, double frequency)
{
    c->num_materials = 4;
    c->materials = (php_host_material*)calloc(4, sizeof(php_host_material));
    double omega = frequency / 0.03e12;

    material_vacuum(&c->materials[0], "Vacuum");

    php_host_material* m = &c->materials[1];
    material_vacuum(m, "SiO2");
    double e0 = 1.5, s1 = 231, g1 = 69, w1 = 806, s2 = 866, g2 = 75, w2 = 1063;
    double temp1 = w1 * w1 - omega * omega, temp2 = w2 * w2 - omega * omega;
    double epsr = e0 + s1 * s1 * temp1 / (temp1 * temp1 + omega * omega * g1 * g1)
                + s2 * s2 * temp2 / (temp2 * temp2 + omega * omega * g2 * g2);
    double epsi = s1 * s1 * omega * g1 / (temp1 * temp1 + omega * omega * g1 * g1)
                + s2 * s2 * omega * g2 / (temp2 * temp2 + omega * omega * g2 * g2);
    m->eps_re[0] = m->eps_re[4] = m->eps_re[8] = epsr;
    m->eps_im[0] = m->eps_im[4] = m->eps_im[8] = epsi;
    if (epsr <= 0) m->use_ade = 1;

    m = &c->materials[2];
    material_vacuum(m, "Uniaxial Crystal");
    m->eps_re[0] = 8.0; m->eps_re[4] = 7.0; m->eps_re[8] = 5.0;

    m = &c->materials[3];
    material_vacuum(m, "Lossy Medium");
    m->eps_re[0] = m->eps_re[4] = m->eps_re[8] = 9.0;
    m->sigma = 0.1;
}

/* ------------------------------------------------------------------ sources */

/* parse_source, fdtd.c:1403-1510.  Defaults are evaluated with the values
 * the config holds at that moment: the first pass runs before any key is
 * read, so nx/ny/nz/tsteps are the defaults and dt is -1. */
static int parse_source(php_cfg* c, char* line, char* err, size_t errlen)
{
    php_source_desc* tmp = (php_source_desc*)realloc(c->sources, (size_t)(c->num_sources + 1) * sizeof(*tmp));
    if (!tmp) { set_err(err, errlen, "Memory allocation failed"); return PHP_ERR_OOM; }
    c->sources = tmp;
    php_source_desc* s = &c->sources[c->num_sources];
    memset(s, 0, sizeof(*s));
    s->type = 0;
    s->x = c->nx / 2;
    s->y = c->ny / 2;
    s->z = c->nz / 3;
    s->amplitude = 1.0;
    s->frequency = 1e9;
    s->t0 = 40 * c->dt;
    s->tau = 15 * c->dt;
    s->component = 'z';
    s->start_time = 0.0;
    s->end_time = c->tsteps * c->dt;

    int has_frequency = 0, has_wavenumber = 0;
    double wavenumber = 0.0;
    char *saveptr = NULL;
    char* token = strtok_r(line, ",", &saveptr);
    while (token) {
        char key[32], value[1024];
        if (sscanf(token, " %31[^=] = %1023s", key, value) == 2) {
            trim(key);
            trim(value);
            if (!strcmp(key, "type")) {
                if (!strcmp(value, "gaussian")) s->type = 0;
                else if (!strcmp(value, "sinusoidal")) s->type = 1;
                else if (!strcmp(value, "ricker")) s->type = 2;
                else if (!strcmp(value, "dipole")) s->type = 3;
            } else if (!strcmp(key, "x")) s->x = atoi(value);
            else if (!strcmp(key, "y")) s->y = atoi(value);
            else if (!strcmp(key, "z")) s->z = atoi(value);
            else if (!strcmp(key, "amplitude")) s->amplitude = strtod(value, NULL);
            else if (!strcmp(key, "frequency")) { s->frequency = strtod(value, NULL); has_frequency = 1; }
            else if (!strcmp(key, "wavenumber")) { wavenumber = strtod(value, NULL); has_wavenumber = 1; }
            else if (!strcmp(key, "t0")) s->t0 = strtod(value, NULL);
            else if (!strcmp(key, "tau")) s->tau = strtod(value, NULL);
            else if (!strcmp(key, "component")) s->component = (unsigned char)value[0];
            else if (!strcmp(key, "start_time")) s->start_time = strtod(value, NULL);
            else if (!strcmp(key, "end_time")) s->end_time = strtod(value, NULL);
        }
        token = strtok_r(NULL, ",", &saveptr);
    }
    if (s->type == 3) {
        if (has_frequency && has_wavenumber) {
            set_err(err, errlen, "Error: Cannot specify both frequency and wavenumber for dipole source");
            return PHP_ERR_INPUT;
        }
        if (!has_frequency && !has_wavenumber) {
            set_err(err, errlen, "Error: Must specify either frequency or wavenumber for dipole source");
            return PHP_ERR_INPUT;
        }
        if (has_wavenumber) s->frequency = wavenumber * 0.03e12;
    }
    c->num_sources++;
    return PHP_OK;
}

/* parse_material, fdtd.c:1512-1727. */
static int parse_material(php_cfg* c, char* line)
{
    int mat_id = -1;
    char line_copy[4096];
    strncpy(line_copy, line, sizeof(line_copy));
    line_copy[sizeof(line_copy) - 1] = '\0';
    char *saveptr = NULL;
    char* token = strtok_r(line_copy, ",", &saveptr);
    while (token) {
        char key[32], value[1024];
        if (sscanf(token, " %31[^=] = %1023s", key, value) == 2) {
            trim(key);
            trim(value);
            if (!strcmp(key, "id")) { mat_id = atoi(value); break; }
        }
        token = strtok_r(NULL, ",", &saveptr);
    }
    if (mat_id < 0) {
        add_warning(c, "Error: Material must have a valid ID\n");
        return PHP_OK;
    }
    if (mat_id >= c->num_materials) {
        php_host_material* tmp = (php_host_material*)realloc(c->materials, (size_t)(mat_id + 1) * sizeof(*tmp));
        if (!tmp) return PHP_ERR_OOM;
        c->materials = tmp;
        for (int i = c->num_materials; i <= mat_id; i++) material_vacuum(&c->materials[i], "Vacuum");
        c->num_materials = mat_id + 1;
    }
    php_host_material* m = &c->materials[mat_id];
    static const char* eps_keys[9] = {"eps_xx", "eps_xy", "eps_xz", "eps_yx", "eps_yy",
                                      "eps_yz", "eps_zx", "eps_zy", "eps_zz"};
    static const char* epsi_keys[9] = {"eps_xxi", "eps_xyi", "eps_xzi", "eps_yxi", "eps_yyi",
                                       "eps_yzi", "eps_zxi", "eps_zyi", "eps_zzi"};
    saveptr = NULL;
    token = strtok_r(line, ",", &saveptr);
    while (token) {
        char key[32], value[1024];
        if (sscanf(token, " %31[^=] = %1023s", key, value) == 2) {
            trim(key);
            trim(value);
            int matched = 0;
            for (int q = 0; q < 9 && !matched; q++) {
                if (!strcmp(key, eps_keys[q])) { m->eps_re[q] = atof(value); matched = 1; }
                else if (!strcmp(key, epsi_keys[q])) { m->eps_im[q] = atof(value); matched = 1; }
            }
            if (matched) { /* done */ }
            else if (!strcmp(key, "name")) snprintf(m->name, sizeof(m->name), "%s", value);
            else if (!strcmp(key, "sigma")) m->sigma = atof(value);
            else if (!strcmp(key, "sigma_m")) m->sigma_m = atof(value);
            else if (!strcmp(key, "dielectric")) {
                snprintf(m->dielectric_file, sizeof(m->dielectric_file), "%s", value);
                m->use_dielectric_file = 1;
            } else if (!strcmp(key, "switchxz")) m->switchxz = atoi(value);
            else if (!strcmp(key, "natom")) m->natom = atoi(value);
            else if (!strcmp(key, "QeZV")) { snprintf(m->qezv_file, sizeof(m->qezv_file), "%s", value); m->qezv_set = 1; }
            else if (!strcmp(key, "QeZM")) { snprintf(m->qezm_file, sizeof(m->qezm_file), "%s", value); m->qezm_set = 1; }
            else if (!strcmp(key, "DMM")) { snprintf(m->dmm_file, sizeof(m->dmm_file), "%s", value); m->dmm_set = 1; }
            else if (!strcmp(key, "use_ADE")) {
                m->use_ade = atoi(value);
                if (m->use_ade != 0 && m->use_ade != 1) {
                    /* fdtd.c:1656-1659 reports and abandons the rest of the line */
                    add_warning(c, "Error: use_ADE must be 0 or 1\n");
                    return PHP_OK;
                }
            } else if (!strcmp(key, "anglez")) m->anglez = atof(value);
            else if (!strcmp(key, "anglex")) m->anglex = atof(value);
            else if (!strcmp(key, "born")) {
                if (!strchr(value, '[') && !strchr(value, ']')) {
                    snprintf(m->born_file, sizeof(m->born_file), "%s", value);
                    m->use_born_file_for_eps = 1;
                } else {
                    /* the inline array form cannot survive the comma
                     * tokenizer (fdtd.c:1671-1719); the reference reports it
                     * and abandons the rest of the line */
                    add_warning(c, "Error: born array must be enclosed in square brackets\n");
                    return PHP_OK;
                }
            }
        }
        token = strtok_r(NULL, ",", &saveptr);
    }
    return PHP_OK;
}

/* ------------------------------------------------------------- data files */

/* read_data, fdtd.c:403-420: n whitespace-separated doubles. */
static int read_numbers(const char* path, double* out, int n, char* err, size_t errlen)
{
    FILE* f = fopen(path, "r");
    if (!f) { set_err(err, errlen, "cannot open %s", path); return PHP_ERR_INPUT; }
    for (int i = 0; i < n; i++) {
        if (fscanf(f, "%lf", &out[i]) != 1) {
            fclose(f);
            set_err(err, errlen, "read failure or too few numbers in %s (%d of %d)", path, i, n);
            return PHP_ERR_INPUT;
        }
    }
    fclose(f);
    return PHP_OK;
}

/* read_born_from_file, fdtd.c:423-552: VASP OUTCAR fragment.  Values of the
 * dielectric block and the Born block are appended in file order. */
static int read_born(const char* path, double* born, int natom, double* eps9, int use_eps,
                     char* err, size_t errlen)
{
    FILE* f = fopen(path, "r");
    if (!f) { set_err(err, errlen, "Error opening Born file: %s", path); return PHP_ERR_INPUT; }
    char line[512];
    int nvals = 0, cap = 1000;
    double values[1000];
    int total_required = (use_eps ? 9 : 0) + 9 * natom;
    int in_dielectric = 0, in_born = 0, current_ion = -1, direction = 0, diel_read = 0;
    while (fgets(line, sizeof(line), f)) {
        line[strcspn(line, "\n")] = 0;
        if (strlen(line) == 0) continue;
        if (strstr(line, "MACROSCOPIC STATIC DIELECTRIC TENSOR")) { in_dielectric = 1; diel_read = 0; continue; }
        if (strstr(line, "BORN EFFECTIVE CHARGES")) { in_born = 1; continue; }
        if ((in_dielectric || in_born) && strstr(line, "---")) {
            if (in_born) current_ion = -1;
            continue;
        }
        if (in_dielectric && diel_read < 9) {
            double a, b, cc;
            if (sscanf(line, "%*s %lf %lf %lf", &a, &b, &cc) == 3 || sscanf(line, "%lf %lf %lf", &a, &b, &cc) == 3) {
                if (nvals + 3 <= cap) { values[nvals++] = a; values[nvals++] = b; values[nvals++] = cc; }
                diel_read += 3;
            }
            continue;
        }
        if (in_born) {
            char* ion = strstr(line, "ion");
            if (ion) {
                ion += 3;
                while (*ion && isspace((unsigned char)*ion)) ion++;
                current_ion = atoi(ion);
                direction = 0;
                continue;
            }
            int idx;
            double a, b, cc;
            if (sscanf(line, "%d %lf %lf %lf", &idx, &a, &b, &cc) == 4) {
                if (current_ion >= 1 && current_ion <= natom && direction < 3) {
                    if (nvals + 3 <= cap) { values[nvals++] = a; values[nvals++] = b; values[nvals++] = cc; }
                    direction++;
                }
            }
            continue;
        }
    }
    fclose(f);
    if (nvals < total_required) {
        set_err(err, errlen, "Error: Only %d values read (expected %d) from %s", nvals, total_required, path);
        return PHP_ERR_INPUT;
    }
    int start = 0;
    if (use_eps) {
        for (int q = 0; q < 9; q++) eps9[q] = values[q];
        start = 9;
    }
    for (int q = 0; q < 9 * natom; q++) born[q] = values[start + q];
    return PHP_OK;
}

/* read_dielectric_from_file, fdtd.c:346-401: the 15-column table row whose
 * frequency is closest to the source frequency, filled symmetrically. */
static int read_dielectric(php_cfg* c, const char* path, double frequency, double* re9, double* im9,
                           char* err, size_t errlen)
{
    FILE* f = fopen(path, "r");
    if (!f) { set_err(err, errlen, "Error opening dielectric file: %s", path); return PHP_ERR_INPUT; }
    double best = DBL_MAX;
    double br[9] = {0}, bi[9] = {0};
    int found = 0;
    char line[256];
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        double v[15];
        if (sscanf(line, "%lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf",
                   &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9],
                   &v[10], &v[11], &v[12], &v[13], &v[14]) == 15) {
            double d = fabs(v[0] - frequency);
            if (d < best) {
                best = d;
                /* columns: xx xy xz yy yz zz, then the imaginary parts */
                br[0] = v[3]; br[1] = v[4]; br[2] = v[5];
                br[3] = v[4]; br[4] = v[6]; br[5] = v[7];
                br[6] = v[5]; br[7] = v[7]; br[8] = v[8];
                bi[0] = v[9]; bi[1] = v[10]; bi[2] = v[11];
                bi[3] = v[10]; bi[4] = v[12]; bi[5] = v[13];
                bi[6] = v[11]; bi[7] = v[13]; bi[8] = v[14];
                found = 1;
            }
        }
    }
    fclose(f);
    if (!found) { set_err(err, errlen, "Error: No valid data found in dielectric file: %s", path); return PHP_ERR_INPUT; }
    if (best > 0.1 * frequency)
        add_warning(c, "Warning: No exact frequency match in %s. Using closest frequency (diff: %.2e Hz)\n", path, best);
    memcpy(re9, br, sizeof(br));
    memcpy(im9, bi, sizeof(bi));
    return PHP_OK;
}

/* switchxz: exchange the x and z axes of a 3x3 block, i.e. (a,b) -> (2-a,2-b)
 * (fdtd.c:2270-2316, 2333-2423, 2442-2467). */
static void swap_xz_3x3(double* m, int row_stride)
{
#define SW(a, b) do { double t_ = m[a]; m[a] = m[b]; m[b] = t_; } while (0)
    int r0 = 0, r1 = row_stride, r2 = 2 * row_stride;
    SW(r0 + 0, r2 + 2);
    SW(r0 + 1, r2 + 1);
    SW(r0 + 2, r2 + 0);
    SW(r1 + 0, r1 + 2);
#undef SW
}

/* ---------------------------------------------------------------- read_config */

static int load_materials(php_cfg* c, char* err, size_t errlen)
{
    /* Born / QeZV / QeZM / DMM, fdtd.c:2249-2431 */
    for (int i = 0; i < c->num_materials; i++) {
        php_host_material* m = &c->materials[i];
        int natom = m->natom;
        if (natom > 0 && m->born_file[0] != '\0') {
            free(m->born);
            m->born = (double*)calloc((size_t)9 * natom, sizeof(double));
            double eps9[9];
            int rc = read_born(m->born_file, m->born, natom, eps9, m->use_born_file_for_eps, err, errlen);
            if (rc) return rc;
            if (m->switchxz == 1)
                for (int a = 0; a < natom; a++) swap_xz_3x3(m->born + 9 * a, 3);
            if (m->use_born_file_for_eps) {
                memcpy(m->eps_re, eps9, sizeof(eps9));
                memset(m->eps_im, 0, sizeof(m->eps_im));
                if (m->switchxz == 1) { swap_xz_3x3(m->eps_re, 3); swap_xz_3x3(m->eps_im, 3); }
            }
        }
        if (natom > 0) {
            if (!m->qezv_set) { set_err(err, errlen, "Error: QeZV is not set!"); return PHP_ERR_INPUT; }
            m->qezv = (double*)calloc((size_t)9 * natom, sizeof(double));
            int rc = read_numbers(m->qezv_file, m->qezv, 9 * natom, err, errlen);
            if (rc) return rc;
            if (m->switchxz == 1)
                for (int a = 0; a < natom; a++) swap_xz_3x3(m->qezv + 9 * a, 3);

            if (!m->qezm_set) { set_err(err, errlen, "Error: QeZM is not set!"); return PHP_ERR_INPUT; }
            m->qezm = (double*)calloc((size_t)9 * natom, sizeof(double));
            rc = read_numbers(m->qezm_file, m->qezm, 9 * natom, err, errlen);
            if (rc) return rc;
            if (m->switchxz == 1)
                for (int a = 0; a < natom; a++) swap_xz_3x3(m->qezm + 9 * a, 3);

            if (!m->dmm_set) { set_err(err, errlen, "Error: DMM is not set!"); return PHP_ERR_INPUT; }
            m->dmm = (double*)calloc((size_t)9 * natom * natom, sizeof(double));
            rc = read_numbers(m->dmm_file, m->dmm, 9 * natom * natom, err, errlen);
            if (rc) return rc;
            if (m->switchxz == 1)
                for (int a = 0; a < natom; a++)
                    for (int b = 0; b < natom; b++)
                        swap_xz_3x3(m->dmm + (size_t)a * 9 * natom + (size_t)b * 3, 3 * natom);
        }
    }
    /* dielectric tables, fdtd.c:2434-2477 */
    for (int i = 0; i < c->num_materials; i++) {
        php_host_material* m = &c->materials[i];
        if (!m->use_dielectric_file) continue;
        int rc = read_dielectric(c, m->dielectric_file, c->unique_source_frequency, m->eps_re, m->eps_im, err, errlen);
        if (rc) {
            char inner[512];
            snprintf(inner, sizeof(inner), "%s", err ? err : "");
            set_err(err, errlen, "Failed to read dielectric function from %s for material %d (%s)",
                    m->dielectric_file, i, inner);
            return rc;
        }
        if (m->switchxz == 1) { swap_xz_3x3(m->eps_re, 3); swap_xz_3x3(m->eps_im, 3); }
    }
    /* material rules checked while printing the library, fdtd.c:2863-2872 */
    for (int i = 0; i < c->num_materials; i++) {
        php_host_material* m = &c->materials[i];
        if (m->natom == 0 && m->use_dielectric_file == 0 && m->switchxz != 0) {
            set_err(err, errlen, "Error: Please switch X and Z by hand for this simple material (material %d)", i);
            return PHP_ERR_INPUT;
        }
        if (fabs(m->anglex) > 1e-10 && fabs(m->anglez) > 1e-10) {
            set_err(err, errlen, "Error: Can not rotate along X and Z axis at the same time (material %d)", i);
            return PHP_ERR_INPUT;
        }
    }
    return PHP_OK;
}

int php_cfg_load(const char* path, php_cfg** out, char* err, size_t errlen)
{
    if (!path || !out) { set_err(err, errlen, "null argument"); return PHP_ERR_INPUT; }
    *out = NULL;
    FILE* f = fopen(path, "r");
    if (!f) { set_err(err, errlen, "Error opening config file: %s", path); return PHP_ERR_INPUT; }
    php_cfg* c = (php_cfg*)calloc(1, sizeof(php_cfg));
    if (!c) { fclose(f); return PHP_ERR_OOM; }

    /* defaults, fdtd.c:1739-1762 */
    c->nx = 50; c->ny = 50; c->nz = 50;
    c->tsteps = 500;
    c->delta_x = 0.01; c->delta_y = 0.01; c->delta_z = 0.01;
    c->pml_thickness = 10;
    c->pml_reflection = 0.001;
    c->output_interval = 20;
    strcpy(c->medium_file, "medium_map.bin");
    c->c = 3e8;
    c->epsilon0 = 8.854e-12;
    c->mu0 = M_PI * 4e-7;
    c->dt = -1.0;
    strcpy(c->output_component, "Ex");
    c->output_slice_axis = 'z';
    c->output_slice_position = c->nz / 2;
    c->full_monitor_enabled = 0;
    strcpy(c->full_monitor_output_file, "full_monitor.dat");
    c->unique_source_frequency = -1.0;

    int rc = PHP_OK;
    char line[4096];
    /* pass 1: sources only (fdtd.c:1765-1777) */
    while (fgets(line, sizeof(line), f)) {
        line[strcspn(line, "\n")] = 0;
        if (line[0] == '#' || line[0] == '\n') continue;
        if (strstr(line, "source") == line) {
            rc = parse_source(c, line + 6, err, errlen);
            if (rc) { fclose(f); php_cfg_free(c); return rc; }
            c->unique_source_frequency = c->sources[0].frequency;
        }
    }
    material_library(c, c->unique_source_frequency);

    /* pass 2: materials and key = value lines (fdtd.c:1789-1901) */
    rewind(f);
    while (fgets(line, sizeof(line), f)) {
        line[strcspn(line, "\n")] = 0;
        if (line[0] == '#' || line[0] == '\n') continue;
        if (strstr(line, "material") == line) {
            rc = parse_material(c, line + 8);
            if (rc) { fclose(f); php_cfg_free(c); return rc; }
            continue;
        }
        char key[64], value[1024];
        if (sscanf(line, "%63[^=]=%1023[^\n]", key, value) != 2) continue;
        trim(key);
        trim(value);
        if (!strcmp(key, "nx")) c->nx = atoi(value);
        else if (!strcmp(key, "ny")) c->ny = atoi(value);
        else if (!strcmp(key, "nz")) c->nz = atoi(value);
        else if (!strcmp(key, "tsteps")) c->tsteps = atoi(value);
        else if (!strcmp(key, "delta_x")) c->delta_x = atof(value);
        else if (!strcmp(key, "delta_y")) c->delta_y = atof(value);
        else if (!strcmp(key, "delta_z")) c->delta_z = atof(value);
        else if (!strcmp(key, "pml_thickness")) c->pml_thickness = atoi(value);
        else if (!strcmp(key, "pml_reflection")) c->pml_reflection = atof(value);
        else if (!strcmp(key, "output_interval")) c->output_interval = atoi(value);
        else if (!strcmp(key, "medium_file")) {
            strncpy(c->medium_file, value, sizeof(c->medium_file) - 1);
            c->medium_file[sizeof(c->medium_file) - 1] = '\0';
        }
        else if (!strcmp(key, "dt")) c->dt = atof(value);
        else if (!strcmp(key, "output_component")) {
            strncpy(c->output_component, value, sizeof(c->output_component));
            c->output_component[sizeof(c->output_component) - 1] = '\0';
            const char* ok[] = {"Ex", "Ey", "Ez", "E", "Dx", "Dy", "Dz"};
            int good = 0;
            for (int q = 0; q < 7; q++) good |= !strcmp(c->output_component, ok[q]);
            if (!good) {
                add_warning(c, "output_component must be one of Ex, Ey, Ez, Dx, Dy, Dz, E; using 'Ex'\n");
                strcpy(c->output_component, "Ex");
            }
        } else if (!strcmp(key, "output_slice_axis")) {
            if (strlen(value) > 0) {
                c->output_slice_axis = value[0];
                if (c->output_slice_axis != 'x' && c->output_slice_axis != 'y' && c->output_slice_axis != 'z') {
                    add_warning(c, "output_slice_axis must be 'x', 'y' or 'z'; using 'z'\n");
                    c->output_slice_axis = 'z';
                }
            }
        } else if (!strcmp(key, "output_slice_position")) c->output_slice_position = atoi(value);
        else if (!strcmp(key, "monitor_point")) {
            c->monitor_enabled = 1;
            char copy[1024];
            strncpy(copy, value, sizeof(copy) - 1);
            copy[sizeof(copy) - 1] = '\0';
            char* sp = NULL;
            char* tok = strtok_r(copy, ",", &sp);
            while (tok) {
                char sk[32], sv[1024];
                if (sscanf(tok, "%31[^=]=%1023s", sk, sv) == 2) {
                    trim(sk);
                    trim(sv);
                    if (!strcmp(sk, "x")) c->monitor_x = atoi(sv);
                    else if (!strcmp(sk, "y")) c->monitor_y = atoi(sv);
                    else if (!strcmp(sk, "z")) c->monitor_z = atoi(sv);
                    else if (!strcmp(sk, "atom")) c->monitor_atom = atoi(sv);
                    else if (!strcmp(sk, "dir")) {
                        if (!strcmp(sv, "x")) c->monitor_dir = 0;
                        else if (!strcmp(sv, "y")) c->monitor_dir = 1;
                        else if (!strcmp(sv, "z")) c->monitor_dir = 2;
                        else {
                            add_warning(c, "Warning: Invalid direction '%s' for monitor_point. Using 'x'.\n", sv);
                            c->monitor_dir = 0;
                        }
                    }
                }
                tok = strtok_r(NULL, ",", &sp);
            }
        } else if (!strcmp(key, "monitor_output_file")) {
            strncpy(c->monitor_output_file, value, sizeof(c->monitor_output_file) - 1);
            c->monitor_output_file[sizeof(c->monitor_output_file) - 1] = '\0';
        } else if (!strcmp(key, "full_monitor")) c->full_monitor_enabled = atoi(value);
        else if (!strcmp(key, "full_monitor_output_file")) {
            strncpy(c->full_monitor_output_file, value, sizeof(c->full_monitor_output_file) - 1);
            c->full_monitor_output_file[sizeof(c->full_monitor_output_file) - 1] = '\0';
        }
    }
    fclose(f);

    /* CFL time step, fdtd.c:1906-1910 */
    double min_delta = c->delta_x;
    if (c->delta_y < min_delta) min_delta = c->delta_y;
    if (c->delta_z < min_delta) min_delta = c->delta_z;
    double temp = min_delta / (c->c * sqrt(3.0)) * 0.99;
    if (c->dt < 0 || c->dt > temp) c->dt = temp;
    /* source end time default, fdtd.c:1913-1917 */
    for (int i = 0; i < c->num_sources; i++)
        if (c->sources[i].end_time <= 0) c->sources[i].end_time = c->tsteps * c->dt;

    rc = load_materials(c, err, errlen);
    if (rc) { php_cfg_free(c); return rc; }
    if (c->nx < 1 || c->ny < 1 || c->nz < 1 || c->tsteps < 0 || c->output_interval < 1) {
        set_err(err, errlen, "invalid grid or interval (nx=%d ny=%d nz=%d tsteps=%d output_interval=%d)",
                c->nx, c->ny, c->nz, c->tsteps, c->output_interval);
        php_cfg_free(c);
        return PHP_ERR_INPUT;
    }
    *out = c;
    return PHP_OK;
}

void php_cfg_free(php_cfg* c)
{
    if (!c) return;
    for (int i = 0; i < c->num_materials; i++) {
        free(c->materials[i].born);
        free(c->materials[i].qezv);
        free(c->materials[i].qezm);
        free(c->materials[i].dmm);
    }
    free(c->materials);
    free(c->desc_materials);
    free(c->sources);
    free(c);
}

int php_cfg_to_desc(const php_cfg* cc, const int32_t* medium, int32_t precision, php_desc* d)
{
    if (!cc || !d) return PHP_ERR_INPUT;
    php_cfg* c = (php_cfg*)cc;
    free(c->desc_materials);
    c->desc_materials = (php_material_desc*)calloc((size_t)(c->num_materials ? c->num_materials : 1),
                                                   sizeof(php_material_desc));
    if (!c->desc_materials) return PHP_ERR_OOM;
    for (int i = 0; i < c->num_materials; i++) {
        const php_host_material* m = &c->materials[i];
        php_material_desc* o = &c->desc_materials[i];
        memcpy(o->eps_re, m->eps_re, sizeof(o->eps_re));
        memcpy(o->eps_im, m->eps_im, sizeof(o->eps_im));
        o->sigma = m->sigma;
        o->anglez = m->anglez;
        o->anglex = m->anglex;
        o->use_ade = m->use_ade;
        o->natom = m->natom;
        o->qezv = m->qezv;
        o->qezm = m->qezm;
        o->dmm = m->dmm;
    }
    memset(d, 0, sizeof(*d));
    d->abi_version = PHP_ABI_VERSION;
    d->nx = c->nx; d->ny = c->ny; d->nz = c->nz;
    d->dx = c->delta_x; d->dy = c->delta_y; d->dz = c->delta_z;
    d->dt = c->dt;
    d->epsilon0 = c->epsilon0;
    d->mu0 = c->mu0;
    d->pml_thickness = c->pml_thickness;
    d->pml_reflection = c->pml_reflection;
    d->precision = precision;
    d->source_frequency = c->unique_source_frequency;
    d->num_materials = c->num_materials;
    d->materials = c->desc_materials;
    d->medium = medium;
    d->num_sources = c->num_sources;
    d->sources = c->sources;
    return PHP_OK;
}

/* read_medium_map_parallel, fdtd.c:718-959, single domain. */
int php_medium_load(const char* path, int32_t nx, int32_t ny, int32_t nz, int32_t** out,
                    char* err, size_t errlen)
{
    *out = NULL;
    FILE* f = fopen(path, "rb");
    if (!f) { set_err(err, errlen, "Error opening medium file: %s", path); return PHP_ERR_INPUT; }
    int32_t h[3];
    if (fread(h, sizeof(int32_t), 3, f) != 3) {
        fclose(f);
        set_err(err, errlen, "Error reading medium file header: %s", path);
        return PHP_ERR_INPUT;
    }
    if (h[0] != nx || h[1] != ny || h[2] != nz) {
        fclose(f);
        set_err(err, errlen, "Medium file dimensions (%d,%d,%d) do not match simulation (%d,%d,%d)",
                h[0], h[1], h[2], nx, ny, nz);
        return PHP_ERR_INPUT;
    }
    size_t n = (size_t)nx * ny * nz;
    int32_t* m = (int32_t*)malloc(n * sizeof(int32_t));
    if (!m) { fclose(f); return PHP_ERR_OOM; }
    if (fread(m, sizeof(int32_t), n, f) != n) {
        fclose(f);
        free(m);
        set_err(err, errlen, "Error reading medium data: %s", path);
        return PHP_ERR_INPUT;
    }
    fclose(f);
    *out = m;
    return PHP_OK;
}

/* calculate_source_value, fdtd.c:1923-1947 */
double php_source_value(const php_source_desc* src, double time)
{
    if (time < src->start_time || time > src->end_time) return 0.0;
    switch (src->type) {
    case 0:
        return src->amplitude * exp(-pow((time - src->t0) / src->tau, 2));
    case 1:
        return src->amplitude * sin(2 * M_PI * src->frequency * time);
    case 2: {
        double t_shift = time - src->t0;
        double arg = M_PI * M_PI * src->frequency * src->frequency * t_shift * t_shift;
        return src->amplitude * (1.0 - 2.0 * arg) * exp(-arg);
    }
    case 3:
        return src->amplitude * sin(2 * M_PI * src->frequency * time) * exp(-pow((time - src->t0) / src->tau, 2));
    default:
        return 0.0;
    }
}

/* ------------------------------------------------------------------ writers */

void php_slice_filename(char* buf, size_t n, char axis, int32_t position, int32_t step)
{
    snprintf(buf, n, "field_slice_%c%d_%08d.bin", axis, position, step);
}

int php_write_slice_file(const char* name, char axis, int32_t nx, int32_t ny, int32_t nz, const float* data)
{
    int32_t a, b;
    if (axis == 'z') { a = nx; b = ny; }
    else if (axis == 'x') { a = ny; b = nz; }
    else if (axis == 'y') { a = nx; b = nz; }
    else return PHP_ERR_INPUT;
    FILE* f = fopen(name, "wb");
    if (!f) return PHP_ERR_INPUT;
    fwrite(&a, sizeof(int32_t), 1, f);
    fwrite(&b, sizeof(int32_t), 1, f);
    fwrite(data, sizeof(float), (size_t)a * b, f);
    fclose(f);
    return PHP_OK;
}

int32_t php_component_from_name(const char* s)
{
    if (!strcmp(s, "Ex")) return PHP_EX;
    if (!strcmp(s, "Ey")) return PHP_EY;
    if (!strcmp(s, "Ez")) return PHP_EZ;
    if (!strcmp(s, "E")) return PHP_EMAG;
    if (!strcmp(s, "Dx")) return PHP_DX;
    if (!strcmp(s, "Dy")) return PHP_DY;
    if (!strcmp(s, "Dz")) return PHP_DZ;
    return PHP_EX;
}

void php_monitor_header(FILE* f, int32_t with_rv)
{
    if (with_rv) fprintf(f, "# Time(s)\tEx\tEy\tEz\tDx\tDy\tDz\tHx\tHy\tHz\tR\tV\n");
    else fprintf(f, "# Time(s)\tEx\tEy\tEz\tDx\tDy\tDz\tHx\tHy\tHz\n");
}

void php_monitor_row(FILE* f, double time, const double* q, int32_t with_rv, double r, double v)
{
    fprintf(f, "%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e", time, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8]);
    if (with_rv) fprintf(f, "\t%e\t%e", r, v);
    fprintf(f, "\n");
}

void php_full_monitor_header(FILE* f, int32_t natom)
{
    fprintf(f, "# Time(s)\tEx\tEy\tEz\tDx\tDy\tDz\tHx\tHy\tHz");
    for (int a = 0; a < natom; a++) fprintf(f, "\tr%d_x\tr%d_y\tr%d_z\tv%d_x\tv%d_y\tv%d_z", a, a, a, a, a, a);
    fprintf(f, "\n");
}

void php_full_monitor_row(FILE* f, double time, const double* q, int32_t natom, const double* r, const double* v)
{
    fprintf(f, "%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e", time, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8]);
    for (int a = 0; a < natom; a++) {
        for (int d = 0; d < 3; d++) fprintf(f, "\t%e", r[a * 3 + d]);
        for (int d = 0; d < 3; d++) fprintf(f, "\t%e", v[a * 3 + d]);
    }
    fprintf(f, "\n");
}

int php_write_frequency_slice(const char* name, double freq_hz, int32_t freq_index, double source_frequency,
                              double fs, int32_t nsamples, int32_t nx, int32_t ny, const double* re,
                              const double* im)
{
    FILE* f = fopen(name, "w");
    if (!f) return PHP_ERR_INPUT;
    fprintf(f, "# Frequency slice at %.3e Hz (index: %d)\n", freq_hz, freq_index);
    fprintf(f, "# Source frequency: %.3e Hz\n", source_frequency);
    fprintf(f, "# Difference: %.3e Hz\n", fabs(freq_hz - source_frequency));
    fprintf(f, "# FFT parameters:\n");
    fprintf(f, "#   Time points: %d\n", nsamples);
    fprintf(f, "#   Sampling frequency: %.3e Hz\n", fs);
    fprintf(f, "#   Frequency resolution: %.3e Hz\n", fs / nsamples);
    fprintf(f, "# Slice dimensions: %d x %d\n", nx, ny);
    fprintf(f, "# Format: x_index y_index real_part imag_part magnitude phase(rad) phase(deg)\n");
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            size_t idx = (size_t)i * ny + j;
            if (i > nx * 0.25 && i < nx * 0.75 && j > ny * 0.25 && j < ny * 0.75) {
                double mag = sqrt(re[idx] * re[idx] + im[idx] * im[idx]);
                double ph = atan2(im[idx], re[idx]);
                fprintf(f, "%d %d %.6e %.6e %.6e %.6e %.6e\n", i, j, re[idx], im[idx], mag, ph, ph * 180.0 / M_PI);
            }
        }
    fclose(f);
    return PHP_OK;
}

int php_spectra_config(const char* cfg_path, double* freq_hz, double* dt)
{
    if (!cfg_path || !freq_hz || !dt) return PHP_ERR_INPUT;
    FILE* f = fopen(cfg_path, "r");
    if (!f) return PHP_ERR_INPUT;
    char line[256];
    double found = 0.0;
    *dt = -1.0;
    while (fgets(line, sizeof(line), f)) {
        line[strcspn(line, "\n")] = 0;
        if (line[0] == '#') continue;
        if (strstr(line, "dt") == line) {
            const char* eq = strchr(line, '=');
            if (eq) *dt = atof(eq + 1);
            continue;
        }
        if (strstr(line, "source") != line) continue;
        double fr = 0.0, wn = 0.0;
        int has_f = 0, has_w = 0;
        char* save = NULL;
        for (char* tok = strtok_r(line, ",", &save); tok; tok = strtok_r(NULL, ",", &save)) {
            char* eq = strchr(tok, '=');
            if (!eq) continue;
            if (strstr(tok, "frequency")) {
                fr = atof(eq + 1);
                has_f = 1;
            } else if (strstr(tok, "wavenumber")) {
                wn = atof(eq + 1);
                has_w = 1;
            }
        }
        if (has_f && has_w) {
            fclose(f);
            return PHP_ERR_INPUT;
        }
        if (has_w) fr = wn * 0.03e12, has_f = 1;
        if (has_f) found = fr;
    }
    fclose(f);
    if (!(found > 0.0)) return PHP_ERR_INPUT;
    *freq_hz = found;
    return PHP_OK;
}

int32_t php_spectra_bins(int32_t n, int32_t interval, double dt, double source_frequency, int32_t* index9,
                         double* freq9, double* fs_out)
{
    if (n < 2 || interval < 1 || !index9 || !freq9) return 0;
    /* sample times as the analysis reads them from the slice file names */
    const double t_first = 0.0 * dt, t_last = (double)((int64_t)(n - 1) * interval) * dt;
    const double T = t_last - t_first;
    const double fs = 1.0 / (T / (n - 1));
    int target = -1;
    double best = 1e100;
    for (int i = 0; i < n / 2; i++) {
        const double d = fabs(i * fs / n - source_frequency);
        if (d < best) {
            best = d;
            target = i;
        }
    }
    int32_t count = 0;
    for (int off = -4; off <= 4 && count < 9; off++) {
        const int idx = target + off;
        if (idx >= 0 && idx < n / 2) {
            index9[count] = idx;
            freq9[count] = idx * fs / n;
            count++;
        }
    }
    if (fs_out) *fs_out = fs;
    return count;
}

uint64_t php_host_sizeof(const char* n)
{
    if (!n) return 0;
    if (!strcmp(n, "php_desc")) return sizeof(php_desc);
    if (!strcmp(n, "php_material_desc")) return sizeof(php_material_desc);
    if (!strcmp(n, "php_source_desc")) return sizeof(php_source_desc);
    if (!strcmp(n, "php_diag")) return sizeof(php_diag);
    if (!strcmp(n, "php_cfg")) return sizeof(php_cfg);
    if (!strcmp(n, "php_host_material")) return sizeof(php_host_material);
    if (!strcmp(n, "php_server_desc")) return sizeof(php_server_desc);
    if (!strcmp(n, "php_dft_request")) return sizeof(php_dft_request);
    if (!strcmp(n, "php_job_info")) return sizeof(php_job_info);
    if (!strcmp(n, "php_server_stats")) return sizeof(php_server_stats);
    if (!strcmp(n, "php_frame_req")) return sizeof(php_frame_req);
    if (!strcmp(n, "php_frame")) return sizeof(php_frame);
    return 0;
}
