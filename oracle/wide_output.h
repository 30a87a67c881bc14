/*
 * Test infrastructure: widens the OUTPUTS of the reference solver (fdtd.c of
 * PhP_FDTD) without touching its arithmetic, so that its results can be
 * compared at 1e-10 and below.  Included last by both MPI stand-ins
 * (mpi_stub/mpi.h, mpi_shm/mpi.h) when PHP_WIDE_OUTPUT is defined:
 *   - `float` becomes `double` for the code after the stand-in, which only
 *     affects the field-slice buffers (fdtd.c:1050-1092, 1115-1261,
 *     1308-1383): slices are written as float64 instead of float32 (the
 *     stand-ins give MPI_FLOAT an 8-byte size under PHP_WIDE_OUTPUT, so the
 *     slice gathers of fdtd.c:1076-1098, 1191-1267, 1357-1390 move the wide
 *     buffers whole);
 *   - every `%e`/`%.Ne` conversion of fprintf becomes `%.17e`, which widens
 *     monitor_point.dat, full_monitor.dat (fdtd.c:3754, 3839, 3865) and
 *     source.txt (fdtd.c:3360, 3367) to round-trip precision.
 */
#ifndef PHP_ORACLE_WIDE_OUTPUT_H
#define PHP_ORACLE_WIDE_OUTPUT_H

#include <stdarg.h>
#include <stdio.h>
#include <string.h>

/* Rewrites every %e conversion (any flags/width/precision) to %.17e. */
static inline int php_wide_fprintf(FILE* f, const char* fmt, ...)
{
    char wide[1024];
    size_t o = 0;
    for (const char* p = fmt; *p && o + 8 < sizeof(wide); ) {
        if (*p != '%') { wide[o++] = *p++; continue; }
        const char* q = p + 1;
        if (*q == '%') { wide[o++] = '%'; wide[o++] = '%'; p = q + 1; continue; }
        while (*q && strchr("-+ #0123456789.", *q)) q++;
        if (*q == 'e') {
            memcpy(wide + o, "%.17e", 5); o += 5; p = q + 1;
        } else {
            while (p <= q && *p && o + 1 < sizeof(wide)) wide[o++] = *p++;
        }
    }
    wide[o] = '\0';
    va_list ap;
    va_start(ap, fmt);
    int n = vfprintf(f, wide, ap);
    va_end(ap);
    return n;
}
#define fprintf php_wide_fprintf
#define float double

#endif
