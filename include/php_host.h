/*
 * php_host.h -- host side of the drop-in: configuration, material data,
 * medium map and output files, in C, with the semantics of PhP_FDTD's
 * fdtd.c set-up code and writers.  It produces the php_desc that
 * libphpfdtd (php_fdtd.h) consumes and writes the same files the reference
 * writes.  No CUDA dependency: libphphost.so loads on machines without a
 * GPU.
 */
#ifndef PHP_HOST_H
#define PHP_HOST_H

#include <stdio.h>
#include "php_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One material as the reference holds it (Material, fdtd.c:82-113). */
typedef struct php_host_material {
    char name[64];
    double eps_re[9];
    double eps_im[9];
    double sigma, sigma_m;
    double anglez, anglex;
    int32_t use_ade;
    int32_t natom;
    int32_t switchxz;
    int32_t use_born_file_for_eps;
    int32_t use_dielectric_file;
    int32_t qezv_set, qezm_set, dmm_set;
    char born_file[1024];
    char qezv_file[1024];
    char qezm_file[1024];
    char dmm_file[1024];
    char dielectric_file[1024];
    double* born; /* 9*natom (read but not used by the time loop) */
    double* qezv; /* 9*natom */
    double* qezm; /* 9*natom */
    double* dmm;  /* 9*natom*natom */
} php_host_material;

/* Configuration (Config, fdtd.c:136-169). */
typedef struct php_cfg {
    int32_t nx, ny, nz, tsteps;
    double delta_x, delta_y, delta_z, dt, c, epsilon0, mu0;
    int32_t pml_thickness;
    double pml_reflection;
    int32_t output_interval;
    char medium_file[1024];
    char output_component[10];
    char output_slice_axis;
    int32_t output_slice_position;
    int32_t monitor_enabled, monitor_x, monitor_y, monitor_z, monitor_atom, monitor_dir;
    char monitor_output_file[1024];
    int32_t full_monitor_enabled;
    char full_monitor_output_file[1024];
    double unique_source_frequency;
    int32_t num_sources;
    php_source_desc* sources;
    int32_t num_materials;
    php_host_material* materials;
    /* desc view of materials, filled by php_cfg_to_desc */
    php_material_desc* desc_materials;
    /* non-fatal messages the reference prints while parsing */
    char warnings[2048];
} php_cfg;

/* Parses the .cfg (read_config, fdtd.c:1730-1920, with parse_source
 * fdtd.c:1403-1510 and parse_material fdtd.c:1512-1727), builds the built-in
 * material library (fdtd.c:628-715), then reads every Born / QeZV / QeZM /
 * DMM / dielectric file with the switchxz permutations (fdtd.c:2249-2477)
 * and checks the material rules of fdtd.c:2863-2872.  On failure returns
 * PHP_ERR_INPUT with a message in err (where the reference would exit). */
int php_cfg_load(const char* path, php_cfg** out, char* err, size_t errlen);
void php_cfg_free(php_cfg* cfg);

/* Fills desc from cfg and a medium array (file order).  Pointers in desc
 * point into cfg and medium, which must outlive desc. */
int php_cfg_to_desc(const php_cfg* cfg, const int32_t* medium, int32_t precision, php_desc* desc);

/* Reads medium_map.bin (fdtd.c:718-959): header nx ny nz must match.
 * Returns a malloc'd [nx][ny][nz] int32 array in *out. */
int php_medium_load(const char* path, int32_t nx, int32_t ny, int32_t nz, int32_t** out,
                    char* err, size_t errlen);

/* Source waveform at time t (calculate_source_value, fdtd.c:1923-1947). */
double php_source_value(const php_source_desc* src, double time);

/* Output files with the reference's formats. */
/* field_slice_<axis><pos>_<step:08d>.bin name (fdtd.c:3712) */
void php_slice_filename(char* buf, size_t n, char axis, int32_t position, int32_t step);
/* 2 int32 dims + float32 data (fdtd.c:1080-1093, 1225-1262, 1370-1384) */
int php_write_slice_file(const char* name, char axis, int32_t nx, int32_t ny, int32_t nz,
                         const float* data);
/* component name -> php_component, "E" -> PHP_EMAG; unknown -> PHP_EX */
int32_t php_component_from_name(const char* name);

/* Monitor-point file (fdtd.c:3828-3878): header at t == 0, one row per
 * step.  with_rv selects the 12-column form. */
void php_monitor_header(FILE* f, int32_t with_rv);
void php_monitor_row(FILE* f, double time, const double* fields9, int32_t with_rv, double r, double v);
/* Full-monitor file (fdtd.c:3739-3775). */
void php_full_monitor_header(FILE* f, int32_t natom);
void php_full_monitor_row(FILE* f, double time, const double* fields9, int32_t natom,
                          const double* r, const double* v);

/* sizeof of a public struct by name ("php_desc", "php_material_desc",
 * "php_source_desc", "php_diag", "php_cfg", "php_host_material"), 0 if
 * unknown; lets foreign-function bindings check their layouts. */
uint64_t php_host_sizeof(const char* type_name);

/* DFT output file (save_frequency_result of frequency_analysis.c:275-314):
 * data [i][j] of re/im; writes the central 25-75 % only. */
int php_write_frequency_slice(const char* name, double freq_hz, int32_t freq_index,
                              double source_frequency, double fs, int32_t nsamples,
                              int32_t nx, int32_t ny, const double* re, const double* im);

/* What frequency_analysis.c takes from a .cfg (frequency_analysis.c:56-148):
 * the frequency= (or wavenumber= x 0.03e12) of the last `source` line that
 * has one, and the explicit `dt` line (*dt = -1 when there is none; the
 * solver itself may have lowered dt to the Courant limit, fdtd.c:1910).
 * Returns PHP_ERR_INPUT when the file cannot be read or no source line has
 * a frequency. */
int php_spectra_config(const char* cfg_path, double* freq_hz, double* dt);

/* The DFT bins frequency_analysis.c writes (frequency_analysis.c:363-421)
 * for n_samples slices taken every `interval` steps of dt: the bin nearest
 * source_frequency and up to four on each side below n_samples / 2.  Fills
 * up to 9 indices and their frequencies k fs / N; returns the count (0 if
 * n_samples < 2) and the sampling frequency fs. */
int32_t php_spectra_bins(int32_t n_samples, int32_t interval, double dt, double source_frequency,
                         int32_t* index9, double* freq9, double* fs);

#ifdef __cplusplus
}
#endif

#endif /* PHP_HOST_H */
