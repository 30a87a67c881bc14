/*
 * php_oracle.h -- TEST INFRASTRUCTURE.  CPU restatement of the PhP_FDTD
 * time-step loop (fdtd.c:3116-3884) used as the parity checker of the CUDA
 * path and as the timed CPU baseline.  Never linked into the product.
 *
 * Consumes the same php_desc as libphpfdtd and exposes read-outs with the
 * same meaning, so a test can run both on identical inputs.
 */
#ifndef PHP_ORACLE_H
#define PHP_ORACLE_H

#include "php_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

int oracle_create(const php_desc* d, oracle_ctx** out);
void oracle_destroy(oracle_ctx* o);
const char* oracle_last_error(void);
/* OpenMP threads for the sweeps (results do not depend on it). */
void oracle_set_threads(int n);
int oracle_step(oracle_ctx* o, int n);
int oracle_get_step(const oracle_ctx* o);
int oracle_read_volume(oracle_ctx* o, int comp, double* out);
int oracle_read_slice_f64(oracle_ctx* o, int comp, char axis, int pos, double* out);
int oracle_read_point(oracle_ctx* o, int i, int j, int k, double* out9);
int oracle_read_cell_state(oracle_ctx* o, int i, int j, int k, int* natom, double* r, double* v, double* p,
                           double* po);
int oracle_diagnostics(oracle_ctx* o, php_diag* out);

#ifdef __cplusplus
}
#endif

#endif
