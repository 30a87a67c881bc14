/*
 * Test infrastructure: a stand-in for the few FFTW3 calls of the reference's
 * post-processor (frequency_analysis.c of PhP_FDTD: fftw_malloc/fftw_free
 * :494-495, fftw_plan_dft_1d :496, fftw_execute :557, fftw_destroy_plan :592,
 * fftw_cleanup :615), so that program compiles unmodified on a machine
 * without FFTW.  FFTW is not vendored in the reference; its published
 * definition of the forward transform (FFTW 3 manual, "What FFTW Really
 * Computes") is Y_k = sum_{j=0}^{n-1} X_j exp(-2 pi i j k / n), unnormalised;
 * this header evaluates that sum directly in double precision, O(n^2) per
 * execution, with the twiddle of each product j*k taken from a table indexed
 * by (j*k) mod n.  Only the plan kind frequency_analysis.c makes (complex,
 * 1-D, FFTW_FORWARD or FFTW_BACKWARD) exists.
 *
 * With PHP_WIDE_OUTPUT the post-processor reads float64 slices and prints
 * %.17e (wide_output.h), the counterpart of the widened solver outputs.
 */
#ifndef PHP_ORACLE_FFTW_STUB_H
#define PHP_ORACLE_FFTW_STUB_H

#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef double fftw_complex[2];

typedef struct php_fftw_plan_s {
    int n, sign;
    fftw_complex *in, *out;
    double *cos_t, *sin_t;   /* cos, sign * sin of 2 pi m / n, m < n */
    double *acc;             /* 2n scratch, so in == out works */
} * fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

static inline void* fftw_malloc(size_t n) { return malloc(n ? n : 1); }
static inline void fftw_free(void* p) { free(p); }
static inline void fftw_cleanup(void) {}

static inline fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags)
{
    (void)flags;
    if (n < 1) return NULL;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->n = n;
    p->sign = sign;
    p->in = in;
    p->out = out;
    p->cos_t = (double*)malloc(sizeof(double) * (size_t)n);
    p->sin_t = (double*)malloc(sizeof(double) * (size_t)n);
    p->acc = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    if (!p->cos_t || !p->sin_t || !p->acc) {
        free(p->cos_t); free(p->sin_t); free(p->acc); free(p);
        return NULL;
    }
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < n; m++) {
        const double a = two_pi * (double)m / (double)n;
        p->cos_t[m] = cos(a);
        p->sin_t[m] = (double)sign * sin(a);
    }
    return p;
}

static inline void fftw_execute(const fftw_plan p)
{
    const int n = p->n;
    const double* x = (const double*)p->in;
    for (int k = 0; k < n; k++) {
        double re = 0.0, im = 0.0;
        for (int j = 0; j < n; j++) {
            const int m = (int)(((int64_t)j * k) % n);
            const double c = p->cos_t[m], s = p->sin_t[m];
            const double xr = x[2 * j], xi = x[2 * j + 1];
            re += xr * c - xi * s;
            im += xr * s + xi * c;
        }
        p->acc[2 * k] = re;
        p->acc[2 * k + 1] = im;
    }
    double* y = (double*)p->out;
    for (int k = 0; k < 2 * n; k++) y[k] = p->acc[k];
}

static inline void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    free(p->cos_t);
    free(p->sin_t);
    free(p->acc);
    free(p);
}

#ifdef PHP_WIDE_OUTPUT
#include "../wide_output.h"
#endif

#endif
