/*
 * fdtd_b200 -- drop-in replacement for PhP_FDTD's solver executable
 * (fdtd.x, fdtd.c:2075-4083) on one B200.
 *
 *   fdtd_b200 <config.cfg> [fp64|fp64-strict|fp32] [--spectra] [--sync-output]
 *
 * Reads the same .cfg, medium_map.bin and material files, prints the same
 * progress lines and writes the same output files as a single-rank run of
 * the reference:
 *   field_slice_<axis><pos>_<step:08d>.bin   every output_interval steps
 *   monitor_point.dat (monitor_output_file)  every step
 *   full_monitor.dat                         every output_interval steps
 *   source.txt                               every output_interval steps
 * and with --spectra, at the end, the frequency_slice_*.txt files that the
 * reference's post-processor (frequency_analysis.c) derives from the z slices:
 * the same bins, normalisation, columns and central crop, accumulated on the
 * device at the output steps from the float32 slice values instead of an FFT
 * over the slice files.
 * The time loop (fdtd.c:3116-3884) runs on the GPU through libphpfdtd; this
 * file is the host loop around it, with the reference's output cadence and
 * index conventions (monitor and z-slice fields read at k+1, atoms at k,
 * fdtd.c:1029, 3752-3753, 3814-3815).
 *
 * Exit codes: 0 done, 1 usage / divergence abort (as MPI_Abort(1) at
 * fdtd.c:3667), 2 bad input, 3 device failure.
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "php_fdtd.h"
#include "php_host.h"

static double wall(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int device_fail(php_ctx* ctx, const char* what, int rc)
{
    fprintf(stderr, "%s failed (%d): %s\n", what, rc, php_last_error(ctx));
    return rc == PHP_ERR_INPUT ? 2 : 3;
}

static void print_config(const php_cfg* c)
{
    printf("==========================Simulation Configuration===========================\n");
    printf("  Grid size: %d x %d x %d\n", c->nx, c->ny, c->nz);
    printf("  Spatial steps: dx=%.4e m, dy=%.4e m, dz=%.4e m\n", c->delta_x, c->delta_y, c->delta_z);
    printf("  Time steps: %d, dt=%.4e s\n", c->tsteps, c->dt);
    printf("  PML thickness: %d cells\n", c->pml_thickness);
    printf("  PML reflection: %.4g\n", c->pml_reflection);
    printf("  Medium file: %s\n", c->medium_file);
    printf("  Sources: %d\n", c->num_sources);
    for (int i = 0; i < c->num_sources; i++) {
        const php_source_desc* s = &c->sources[i];
        const char* ts = s->type == 1 ? "sinusoidal" : s->type == 2 ? "ricker" : s->type == 3 ? "dipole" : "gaussian";
        printf("    Source %d: type=%s, position=(%d,%d,%d), amplitude=%.2f\n", i + 1, ts, s->x, s->y, s->z, s->amplitude);
        printf("               component=%c, frequency=%.2e Hz, T=%.2e s, t0=%.2e s, tau=%.2e s\n", (char)s->component,
               s->frequency, 1 / s->frequency, s->t0, s->tau);
    }
    printf("Output %.2s at time interval: %.2e s\n", c->output_component, c->output_interval * c->dt);
    printf("Output slice: axis=%c, position=%d\n", c->output_slice_axis, c->output_slice_position);
    printf("\nMaterial library details:\n");
    for (int i = 0; i < c->num_materials; i++) {
        const php_host_material* m = &c->materials[i];
        printf("  Material %d: %s\n", i, m->name);
        printf("    Dielectric tensor (real):\n");
        for (int r = 0; r < 3; r++) printf("      [%.4f, %.4f, %.4f]\n", m->eps_re[3 * r], m->eps_re[3 * r + 1], m->eps_re[3 * r + 2]);
        printf("    Dielectric tensor (imag) should be >= 0:\n");
        for (int r = 0; r < 3; r++) printf("      [%.4f, %.4f, %.4f]\n", m->eps_im[3 * r], m->eps_im[3 * r + 1], m->eps_im[3 * r + 2]);
        printf("    use_ADE: %d\n    Number of atoms: %d\n", m->use_ade, m->natom);
    }
}

static void write_monitor_row(const php_cfg* cfg, FILE** f, int with_rv, int natom, int step, const double* row)
{
    if (step == 0) {
        *f = fopen(cfg->monitor_output_file, "w");
        if (*f) php_monitor_header(*f, with_rv);
    }
    if (!*f) return;
    const int idx = cfg->monitor_atom * 3 + cfg->monitor_dir;
    const double r = with_rv ? row[9 + idx] : 0.0, v = with_rv ? row[9 + 3 * natom + idx] : 0.0;
    php_monitor_row(*f, step * cfg->dt, row, with_rv, r, v);
}

/* ------------------------------------------------------------ the writer
 *
 * The stepping thread enqueues a chunk of steps and its output frame
 * (php_frame_begin) and goes on with the next chunk; the writer takes the
 * frames in order, waits for each, writes what the reference writes at
 * those steps (fdtd.c:3535-3883) and releases it.  The device is never idle
 * for the writer's file output.  With --sync-output the stepping thread
 * writes each frame itself before the next chunk. */

typedef struct {
    int t, next, n;  /* steps t .. next (n of them); t < 0 ends the writer */
    int32_t ticket;
} Item;

#define WRITER_QUEUE (PHP_FRAME_SLOTS + 2)

typedef struct {
    const php_cfg* cfg;
    php_ctx* ctx;
    int nx, ny, nz;
    int monitor_ok, monitor_rv, monitor_natom, full_ok, full_natom;
    FILE *source_file, *monitor_file, *full_file;
    double start;
    atomic_int stop; /* divergence abort or failure: no further chunks */
    int exit_code;
    int dead;        /* after a stop: frames are waited for and released, nothing is written */
    pthread_mutex_t mu;
    pthread_cond_t cv;
    Item q[WRITER_QUEUE];
    int head, count;
} Writer;

static void writer_push(Writer* W, Item it)
{
    pthread_mutex_lock(&W->mu);
    while (W->count == WRITER_QUEUE) pthread_cond_wait(&W->cv, &W->mu);
    W->q[(W->head + W->count) % WRITER_QUEUE] = it;
    W->count++;
    pthread_cond_broadcast(&W->cv);
    pthread_mutex_unlock(&W->mu);
}

static Item writer_pop(Writer* W)
{
    pthread_mutex_lock(&W->mu);
    while (W->count == 0) pthread_cond_wait(&W->cv, &W->mu);
    Item it = W->q[W->head];
    W->head = (W->head + 1) % WRITER_QUEUE;
    W->count--;
    pthread_cond_broadcast(&W->cv);
    pthread_mutex_unlock(&W->mu);
    return it;
}

/* The divergence report of fdtd.c:3626-3668 from the frame's copy of the
 * cell of max |r|. */
static void report_divergence(Writer* W, const php_frame* fr, int last)
{
    const php_cfg* cfg = W->cfg;
    const php_diag* dg = &fr->diag;
    const int* am = dg->argmax_r;
    printf("ERROR: r field too large at step %d\n", last);
    printf("Max r value: %e\n", dg->max_r);
    printf("Location: i=%d, j=%d, k=%d (global k=%d)\n", am[0], am[1], am[2], am[2]);
    printf("Atom: %d, Direction: %d\n", am[3], am[4]);
    const int idx = am[3] * 3 + am[4];
    printf("v value: %e\n", fr->diag_v[idx]);
    /* acceleration recomputed from the lab-frame E, as fdtd.c:3642-3663 */
    const php_host_material* m = NULL;
    int32_t* med = NULL;
    char err[1024];
    if (!php_medium_load(cfg->medium_file, W->nx, W->ny, W->nz, &med, err, sizeof(err))) {
        m = &cfg->materials[med[((size_t)am[0] * W->ny + am[1]) * W->nz + am[2]]];
        free(med);
    }
    if (m && m->qezm && m->dmm) {
        double a_val = 0.0;
        for (int iE = 0; iE < 3; iE++) a_val += m->qezm[am[3] * 9 + iE * 3 + am[4]] * fr->diag_point[iE];
        for (int q = 0; q < 3 * m->natom; q++) a_val -= m->dmm[(size_t)idx * 3 * m->natom + q] * fr->diag_r[q];
        printf("a value: %e\n", a_val);
    }
    fflush(stdout);
}

static void writer_item(Writer* W, const Item* it)
{
    const php_cfg* cfg = W->cfg;
    php_frame fr;
    int rc = php_frame_wait(W->ctx, it->ticket, &fr);
    if (rc || W->dead) {
        if (rc && !W->dead) {
            W->exit_code = device_fail(W->ctx, "php_frame_wait", rc);
            W->dead = 1;
            atomic_store(&W->stop, 1);
        }
        php_frame_release(W->ctx, it->ticket);
        return;
    }
    const int t = it->t, next = it->next, n = it->n;
    /* source.txt rows of the output steps in this chunk (fdtd.c:3359-3400) */
    for (int s = t; s <= next; s++) {
        if (s % cfg->output_interval == 0 && W->source_file) {
            double ct = s * cfg->dt;
            fprintf(W->source_file, "%.4e  ", ct);
            for (int q = 0; q < cfg->num_sources; q++) fprintf(W->source_file, "%.4e  ", php_source_value(&cfg->sources[q], ct));
            fprintf(W->source_file, "\n");
            fflush(W->source_file);
        }
    }
    /* monitor rows (every step, fdtd.c:3806-3883): the row of an output step
     * follows that step's diagnostics, so a divergence abort there drops it,
     * as in the reference */
    const int nrows = fr.nrows, row_len = fr.row_len;
    if (W->monitor_ok)
        for (int q = 0; q < nrows && t + q < next; q++)
            write_monitor_row(cfg, &W->monitor_file, W->monitor_rv, W->monitor_natom, t + q, fr.rows + (size_t)q * row_len);
    const int last = next;
    if (last % cfg->output_interval == 0) {
        const php_diag* dg = &fr.diag;
        double current_time = last * cfg->dt;
        printf("it %d/%d (%.1f%%), t = %.5e s,|E|_max = %.2e V/m,", last, cfg->tsteps, 100.0 * last / cfg->tsteps, current_time,
               dg->max_e);
        printf("r_max = %.2e A,", dg->max_r / 1e-10);
        if (last > 0) {
            double el = wall() - W->start;
            double eta = el / last * (cfg->tsteps - last);
            int eh = (int)(el / 3600), em = (int)((el - eh * 3600) / 60), es = (int)(el - eh * 3600 - em * 60);
            int rh = (int)(eta / 3600), rm = (int)((eta - rh * 3600) / 60), rs = (int)(eta - rh * 3600 - rm * 60);
            printf(" elapsed: %03d:%02d:%02d, ETA: %03d:%02d:%02d", eh, em, es, rh, rm, rs);
        }
        printf("\n");
        fflush(stdout);
        if (dg->max_r > 1e-10) { /* fdtd.c:3626-3668 */
            report_divergence(W, &fr, last);
            W->exit_code = 1;
            W->dead = 1;
            atomic_store(&W->stop, 1);
            php_frame_release(W->ctx, it->ticket);
            return;
        }
        if (fr.slice) {
            char name[256];
            php_slice_filename(name, sizeof(name), (char)cfg->output_slice_axis, cfg->output_slice_position, last);
            php_write_slice_file(name, (char)cfg->output_slice_axis, W->nx, W->ny, W->nz, fr.slice);
        }
        if (W->full_ok) {
            if (last == 0) {
                W->full_file = fopen(cfg->full_monitor_output_file, "w");
                if (W->full_file) php_full_monitor_header(W->full_file, W->full_natom);
            }
            if (W->full_file) php_full_monitor_row(W->full_file, current_time, fr.point, W->full_natom, fr.cell_r, fr.cell_v);
        }
    }
    if (W->monitor_ok && nrows == n)
        write_monitor_row(cfg, &W->monitor_file, W->monitor_rv, W->monitor_natom, next, fr.rows + (size_t)(n - 1) * row_len);
    php_frame_release(W->ctx, it->ticket);
}

static void* writer_main(void* arg)
{
    Writer* W = (Writer*)arg;
    for (;;) {
        Item it = writer_pop(W);
        if (it.t < 0) break;
        writer_item(W, &it);
    }
    return NULL;
}

int main(int argc, char** argv)
{
    printf("FDTD (B200) running on 1 GPU\n");
    if (argc < 2) {
        printf("Usage: %s <config_file.cfg> [fp64|fp64-strict|fp32] [--spectra] [--sync-output]\n", argv[0]);
        return 1;
    }
    int precision = PHP_PREC_FP64;
    int spectra = 0, sync_output = 0;
    const char* pa = getenv("PHP_PRECISION");
    for (int a = 2; a < argc; a++) {
        if (!strcmp(argv[a], "--spectra")) spectra = 1;
        else if (!strcmp(argv[a], "--sync-output")) sync_output = 1;
        else pa = argv[a];
    }
    if (pa) {
        if (!strcmp(pa, "fp64-strict")) precision = PHP_PREC_FP64_STRICT;
        else if (!strcmp(pa, "fp32")) precision = PHP_PREC_FP32;
        else if (!strcmp(pa, "fp64")) precision = PHP_PREC_FP64;
        else {
            fprintf(stderr, "unknown precision '%s'\n", pa);
            return 1;
        }
    }
    char err[1024] = "";
    php_cfg* cfg = NULL;
    if (php_cfg_load(argv[1], &cfg, err, sizeof(err))) {
        fprintf(stderr, "%s\n", err);
        return 2;
    }
    if (cfg->warnings[0]) fprintf(stderr, "%s", cfg->warnings);
    print_config(cfg);
    printf("Using medium file: %s\n", cfg->medium_file);
    int32_t* medium = NULL;
    if (php_medium_load(cfg->medium_file, cfg->nx, cfg->ny, cfg->nz, &medium, err, sizeof(err))) {
        fprintf(stderr, "%s\n", err);
        php_cfg_free(cfg);
        return 2;
    }
    printf("Successfully loaded medium map from %s\n", cfg->medium_file);

    php_desc desc;
    php_cfg_to_desc(cfg, medium, precision, &desc);
    php_ctx* ctx = NULL;
    int rc = php_create(&desc, &ctx);
    if (rc) {
        int code = device_fail(NULL, "php_create", rc);
        free(medium);
        php_cfg_free(cfg);
        return code;
    }

    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    /* monitor point: fields at z+1, atoms at z (fdtd.c:3806-3883) */
    int monitor_ok = 0, monitor_rv = 0, monitor_natom = 0;
    if (cfg->monitor_enabled && cfg->monitor_z >= 0 && cfg->monitor_z < nz && cfg->monitor_x >= 0 && cfg->monitor_x < nx &&
        cfg->monitor_y >= 0 && cfg->monitor_y < ny) {
        monitor_ok = 1;
        int id = medium[((size_t)cfg->monitor_x * ny + cfg->monitor_y) * nz + cfg->monitor_z];
        monitor_natom = cfg->materials[id].natom;
        monitor_rv = cfg->monitor_atom < monitor_natom;
        /* fdtd.c:2932-2951: atoms at the monitor point switch the full monitor on */
        if (!cfg->full_monitor_enabled && monitor_natom > 0) cfg->full_monitor_enabled = 1;
        if ((rc = php_probe_set(ctx, cfg->monitor_x, cfg->monitor_y, cfg->monitor_z + 1, cfg->monitor_z)))
            return device_fail(ctx, "php_probe_set", rc);
    }
    int full_ok = 0, full_natom = 0;
    if (cfg->full_monitor_enabled && cfg->monitor_z >= 0 && cfg->monitor_z < nz && cfg->monitor_x >= 0 && cfg->monitor_x < nx &&
        cfg->monitor_y >= 0 && cfg->monitor_y < ny) {
        full_ok = 1;
        full_natom = cfg->materials[medium[((size_t)cfg->monitor_x * ny + cfg->monitor_y) * nz + cfg->monitor_z]].natom;
    }
    free(medium);
    medium = NULL;

    /* running DFT of the output slice at the post-processor's bins
     * (frequency_analysis.c:363-421): samples at t % output_interval == 0,
     * float32 like the slice files, z slices of a field component */
    int spectra_id = -1, spectra_n = 0, spectra_count = 0;
    int32_t spectra_index[9];
    double spectra_freq[9], spectra_fs = 0.0, spectra_src = 0.0, spectra_dt = -1.0;
    const int spectra_comp = php_component_from_name(cfg->output_component);
    if (spectra) {
        spectra_n = (cfg->tsteps - 1) / cfg->output_interval + 1;
        if (cfg->output_slice_axis != 'z' || spectra_comp < 0 || spectra_comp > PHP_HZ)
            fprintf(stderr, "--spectra: needs a z slice of a field component; skipped\n");
        else if (php_spectra_config(argv[1], &spectra_src, &spectra_dt))
            fprintf(stderr, "--spectra: no source frequency in %s; skipped\n", argv[1]);
        else {
            /* bins and their labels as the post-processor computes them from
             * the .cfg's dt line (the solver's dt when there is none) ... */
            const double label_dt = spectra_dt > 0 ? spectra_dt : cfg->dt;
            spectra_count = php_spectra_bins(spectra_n, cfg->output_interval, label_dt, spectra_src, spectra_index,
                                             spectra_freq, &spectra_fs);
            /* ... and sampled on the solver's own time base, so that bin k
             * is exactly exp(-2 pi i k n / N) over the N output steps */
            double fs_solver = 0.0, f_solver[9];
            int32_t idx_solver[9];
            php_spectra_bins(spectra_n, cfg->output_interval, cfg->dt, spectra_src, idx_solver, f_solver, &fs_solver);
            for (int f = 0; f < spectra_count; f++) f_solver[f] = spectra_index[f] * fs_solver / spectra_n;
            if (spectra_count > 0 &&
                (rc = php_dft_add(ctx, spectra_comp, cfg->output_slice_position + 1, 0, cfg->output_interval,
                                  spectra_count, f_solver, 1, &spectra_id)))
                return device_fail(ctx, "php_dft_add", rc);
        }
    }

    Writer W;
    memset(&W, 0, sizeof(W));
    W.cfg = cfg;
    W.ctx = ctx;
    W.nx = nx;
    W.ny = ny;
    W.nz = nz;
    W.monitor_ok = monitor_ok;
    W.monitor_rv = monitor_rv;
    W.monitor_natom = monitor_natom;
    W.full_ok = full_ok;
    W.full_natom = full_natom;
    W.source_file = fopen("source.txt", "w");
    if (!W.source_file) fprintf(stderr, "Error opening source.txt for writing\n");
    pthread_mutex_init(&W.mu, NULL);
    pthread_cond_init(&W.cv, NULL);

    W.start = wall();
    printf("Entering iteration:\n");
    fflush(stdout);
    pthread_t writer;
    const int threaded = !sync_output && pthread_create(&writer, NULL, writer_main, &W) == 0;
    int t = 0;
    int exit_code = 0;
    while (t < cfg->tsteps && !atomic_load(&W.stop)) {
        /* run to the next output step (t % output_interval == 0) inclusive */
        int next = (t % cfg->output_interval == 0) ? t : (t / cfg->output_interval + 1) * cfg->output_interval;
        if (next > cfg->tsteps - 1) next = cfg->tsteps - 1;
        const int n = next - t + 1;
        if ((rc = php_step(ctx, n))) { exit_code = device_fail(ctx, "php_step", rc); break; }
        /* the frame of this chunk: probe rows of every step, and at an output
         * step the diagnostics, the slice and the full-monitor cell */
        const int out = next % cfg->output_interval == 0;
        php_frame_req q;
        memset(&q, 0, sizeof(q));
        q.diag = out;
        q.slice_comp = out ? php_component_from_name(cfg->output_component) : -1;
        q.slice_axis = cfg->output_slice_axis;
        q.slice_pos = cfg->output_slice_position;
        q.probe = monitor_ok;
        q.point[0] = q.cell[0] = -1;
        if (out && full_ok) {
            q.point[0] = q.cell[0] = cfg->monitor_x;
            q.point[1] = q.cell[1] = cfg->monitor_y;
            q.point[2] = cfg->monitor_z + 1;
            q.cell[2] = cfg->monitor_z;
        }
        Item it = {t, next, n, -1};
        if ((rc = php_frame_begin(ctx, &q, &it.ticket))) {
            if (q.slice_comp >= 0 && rc == PHP_ERR_INPUT) {
                /* a slice the reference refuses (message, no file): the rest of the frame */
                fprintf(stderr, "%s\n", php_last_error(ctx));
                q.slice_comp = -1;
                rc = php_frame_begin(ctx, &q, &it.ticket);
            }
            if (rc) { exit_code = device_fail(ctx, "php_frame_begin", rc); break; }
        }
        if (threaded) writer_push(&W, it);
        else writer_item(&W, &it);
        t = next + 1;
    }
    if (threaded) {
        Item end = {-1, -1, 0, -1};
        writer_push(&W, end);
        pthread_join(writer, NULL);
    }
    if (W.exit_code && !exit_code) exit_code = W.exit_code;
    FILE* source_file = W.source_file;
    FILE* monitor_file = W.monitor_file;
    FILE* full_file = W.full_file;
    const double start = W.start;
    php_sync(ctx);
    if (spectra_id >= 0 && exit_code == 0) {
        double* acc = (double*)malloc(sizeof(double) * 2 * (size_t)spectra_count * nx * ny);
        double* re = (double*)malloc(sizeof(double) * (size_t)nx * ny);
        double* im = (double*)malloc(sizeof(double) * (size_t)nx * ny);
        int32_t ns = 0;
        if (acc && re && im && php_dft_read(ctx, spectra_id, acc, &ns) == PHP_OK) {
            for (int f = 0; f < spectra_count; f++) {
                for (size_t q = 0; q < (size_t)nx * ny; q++) {
                    re[q] = acc[2 * ((size_t)f * nx * ny + q)] / ns;
                    im[q] = acc[2 * ((size_t)f * nx * ny + q) + 1] / ns;
                }
                char name[256];
                snprintf(name, sizeof(name), "frequency_slice_%d_%.3eHz_%.3ecm-1.txt", spectra_index[f], spectra_freq[f],
                         spectra_freq[f] / 0.03e12);
                php_write_frequency_slice(name, spectra_freq[f], spectra_index[f], spectra_src, spectra_fs, ns, nx, ny, re,
                                          im);
                printf("  Results saved to %s\n", name);
            }
        }
        free(acc);
        free(re);
        free(im);
    }
    if (source_file) fclose(source_file);
    if (monitor_file) {
        fclose(monitor_file);
        printf("Monitor data saved to %s\n", cfg->monitor_output_file);
    }
    if (full_file) {
        fclose(full_file);
        printf("Full monitor data saved to %s\n", cfg->full_monitor_output_file);
    }
    if (exit_code == 0) printf("\nSimulation completed in %.2f seconds\n", wall() - start);
    pthread_mutex_destroy(&W.mu);
    pthread_cond_destroy(&W.cv);
    php_destroy(ctx);
    php_cfg_free(cfg);
    return exit_code;
}
