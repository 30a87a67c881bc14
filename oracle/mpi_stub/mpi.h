/*
 * Single-rank MPI stand-in used ONLY to compile the reference solver
 * (fdtd.c of PhP_FDTD) unmodified on a machine without an MPI
 * installation.  This is test infrastructure: the compiled reference is the
 * parity checker and the CPU baseline, never part of the product path.
 *
 * With one rank every collective fdtd.c issues is a local copy or a no-op:
 *   MPI_Bcast      fdtd.c:2162, 2204, 2214, 2223, 2230, 2242, 2566-2702, 3720
 *   MPI_Allreduce  fdtd.c:1040, 2949, 3559, 3560, 3596, 3630
 *   MPI_Reduce     fdtd.c:62, 3894, 3905
 *   MPI_Scatterv   fdtd.c:853 (rank 0 receives displs[0]..+counts[0])
 * Point-to-point calls (MPI_Send/Recv/Sendrecv, fdtd.c:904-945, 2021, 2044,
 * 1076, 1098, 1191, 1267, 1357, 1390) are only reached when size > 1; here
 * they abort loudly.
 *
 * PHP_WIDE_OUTPUT (compile-time) widens the reference's OUTPUTS without
 * touching its arithmetic (float64 slices, %.17e monitors): wide_output.h.
 */
#ifndef PHP_ORACLE_MPI_STUB_H
#define PHP_ORACLE_MPI_STUB_H

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0

/* datatype handles encode their byte size */
#define MPI_CHAR 1
#define MPI_BYTE 1001
#define MPI_INT 4
#ifdef PHP_WIDE_OUTPUT
#define MPI_FLOAT 2008 /* the slice buffers are double under PHP_WIDE_OUTPUT */
#else
#define MPI_FLOAT 1004
#endif
#define MPI_DOUBLE 8
#define MPI_UNSIGNED_LONG_LONG 1008

#define MPI_MAX 1
#define MPI_SUM 2

static inline size_t php_stub_type_size(MPI_Datatype t) { return (size_t)(t % 1000); }

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; fflush(stdout); exit(code ? code : 1); }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void)op; (void)c; memmove(r, s, (size_t)n * php_stub_type_size(t)); return 0; }
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void)op; (void)root; (void)c; memmove(r, s, (size_t)n * php_stub_type_size(t)); return 0; }
static inline int MPI_Scatterv(const void* s, const int* counts, const int* displs, MPI_Datatype st,
                               void* r, int rc, MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rc; (void)rt; (void)root; (void)c;
    if (s) memmove(r, (const char*)s + (size_t)displs[0] * php_stub_type_size(st),
                   (size_t)counts[0] * php_stub_type_size(st));
    return 0;
}
static inline int php_stub_p2p(void)
{
    fprintf(stderr, "mpi stub: point-to-point call reached with one rank\n");
    exit(70);
}
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return php_stub_p2p(); }
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return php_stub_p2p(); }
static inline int MPI_Sendrecv(const void* sb, int sn, MPI_Datatype st, int d, int stag,
                               void* rb, int rn, MPI_Datatype rt, int s, int rtag, MPI_Comm c, MPI_Status* status)
{
    (void)sb; (void)sn; (void)st; (void)d; (void)stag; (void)rb; (void)rn; (void)rt;
    (void)s; (void)rtag; (void)c; (void)status;
    return php_stub_p2p();
}
static inline double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#ifdef PHP_WIDE_OUTPUT
#include "../wide_output.h"
#endif

#endif
