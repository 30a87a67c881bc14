/*
 * Multi-process MPI stand-in over shared memory, used ONLY to compile the
 * reference solver (fdtd.c of PhP_FDTD) unmodified into a CPU baseline that
 * uses all of a host's cores when no MPI installation exists.  Test and
 * benchmark infrastructure: the timed reference arm, never the product.
 *
 * MPI_Init forks PHP_MPI_NP - 1 children (default 1 rank) after mapping one
 * shared anonymous region; every rank then runs the rest of main().  What
 * fdtd.c uses is implemented:
 *   - MPI_Barrier: sense-reversing barrier on shared counters;
 *   - MPI_Bcast, MPI_Scatterv: through a shared staging area, in chunks;
 *   - MPI_Allreduce, MPI_Reduce (MAX, SUM of int, double, unsigned long long);
 *   - MPI_Send, MPI_Recv, MPI_Sendrecv: one FIFO channel per ordered rank
 *     pair that fdtd.c uses (neighbours in z, and every rank to rank 0),
 *     messages copied through the channel in chunks; MPI_Sendrecv advances
 *     both directions together, so two ranks exchanging large messages do
 *     not wait on each other.  Tags are not matched: fdtd.c sends the
 *     messages of each pair in the order they are received.
 * A rank that calls MPI_Abort marks the region; spinning ranks then exit.
 * Children die with rank 0 (PR_SET_PDEATHSIG); MPI_Finalize on rank 0
 * waits for them.  PHP_WIDE_OUTPUT widens the outputs as in the one-rank
 * stub (wide_output.h).
 */
#ifndef PHP_ORACLE_MPI_SHM_H
#define PHP_ORACLE_MPI_SHM_H

#include <sched.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
/* handles encode the byte size (value % 1000) and the kind */
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

#define PHP_SHM_MAXRANK 512
#define PHP_SHM_CHAN_BYTES ((size_t)32 << 20)
#define PHP_SHM_COLL_BYTES ((size_t)256 << 20)

typedef struct {
    volatile uint64_t posted, taken; /* chunks written / read */
    volatile uint64_t bytes;         /* size of the chunk in the buffer */
    char pad[40];
} php_shm_chan;

typedef struct {
    volatile int count, sense, aborted, np;
    volatile int64_t coll_total;                      /* Scatterv: elements on the root */
    int displs[PHP_SHM_MAXRANK], counts[PHP_SHM_MAXRANK];
} php_shm_hdr;

static php_shm_hdr* php_shm_h;
static php_shm_chan* php_shm_ch;
static char* php_shm_chdata;
static char* php_shm_coll;
static int php_shm_rank, php_shm_np = 1, php_shm_local_sense;
static pid_t php_shm_kids[PHP_SHM_MAXRANK];

static inline size_t php_shm_tsize(MPI_Datatype t) { return (size_t)(t % 1000); }

/* channel of src -> dst: 0..np-2 down (r -> r-1), np-1..2np-3 up (r -> r+1),
 * 2np-2.. to rank 0 from ranks >= 2 */
static inline int php_shm_chan_index(int src, int dst)
{
    const int np = php_shm_np;
    if (dst == src - 1) return src - 1;
    if (dst == src + 1) return (np - 1) + src;
    if (dst == 0 && src >= 2) return 2 * (np - 1) + (src - 2);
    fprintf(stderr, "mpi shm: no channel %d -> %d\n", src, dst);
    exit(71);
}

static inline void php_shm_relax(void)
{
    if (php_shm_h->aborted) _exit(1);
    sched_yield();
}

static inline int MPI_Barrier(MPI_Comm c)
{
    (void)c;
    if (php_shm_np == 1) return 0;
    php_shm_local_sense = !php_shm_local_sense;
    if (__atomic_add_fetch(&php_shm_h->count, 1, __ATOMIC_ACQ_REL) == php_shm_np) {
        __atomic_store_n(&php_shm_h->count, 0, __ATOMIC_RELAXED);
        __atomic_store_n(&php_shm_h->sense, php_shm_local_sense, __ATOMIC_RELEASE);
    } else {
        while (__atomic_load_n(&php_shm_h->sense, __ATOMIC_ACQUIRE) != php_shm_local_sense) php_shm_relax();
    }
    return 0;
}

static inline int MPI_Init(int* argc, char*** argv)
{
    (void)argc; (void)argv;
    const char* e = getenv("PHP_MPI_NP");
    int np = e ? atoi(e) : 1;
    if (np < 1) np = 1;
    if (np > PHP_SHM_MAXRANK) np = PHP_SHM_MAXRANK;
    const size_t nchan = (size_t)3 * np;
    const size_t hdr = (sizeof(php_shm_hdr) + 4095) / 4096 * 4096;
    const size_t chs = (nchan * sizeof(php_shm_chan) + 4095) / 4096 * 4096;
    const size_t total = hdr + chs + nchan * PHP_SHM_CHAN_BYTES + PHP_SHM_COLL_BYTES;
    char* base = (char*)mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (base == MAP_FAILED) {
        perror("mpi shm: mmap");
        exit(72);
    }
    php_shm_h = (php_shm_hdr*)base;
    php_shm_ch = (php_shm_chan*)(base + hdr);
    php_shm_chdata = base + hdr + chs;
    php_shm_coll = php_shm_chdata + nchan * PHP_SHM_CHAN_BYTES;
    php_shm_h->np = np;
    php_shm_np = np;
    fflush(stdout);
    fflush(stderr);
    for (int r = 1; r < np; r++) {
        pid_t p = fork();
        if (p < 0) {
            perror("mpi shm: fork");
            exit(73);
        }
        if (p == 0) {
            prctl(PR_SET_PDEATHSIG, SIGKILL);
            php_shm_rank = r;
            return 0;
        }
        php_shm_kids[r] = p;
    }
    php_shm_rank = 0;
    return 0;
}

static inline int MPI_Finalize(void)
{
    MPI_Barrier(0);
    if (php_shm_rank == 0)
        for (int r = 1; r < php_shm_np; r++) waitpid(php_shm_kids[r], NULL, 0);
    return 0;
}

static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = php_shm_rank; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = php_shm_np; return 0; }

static inline int MPI_Abort(MPI_Comm c, int code)
{
    (void)c;
    if (php_shm_h) php_shm_h->aborted = 1;
    fflush(stdout);
    exit(code ? code : 1);
}

static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)c;
    if (php_shm_np == 1) return 0;
    const size_t bytes = (size_t)n * php_shm_tsize(t);
    for (size_t off = 0; off < bytes; off += PHP_SHM_COLL_BYTES) {
        const size_t len = bytes - off < PHP_SHM_COLL_BYTES ? bytes - off : PHP_SHM_COLL_BYTES;
        if (php_shm_rank == root) memcpy(php_shm_coll, (char*)b + off, len);
        MPI_Barrier(0);
        if (php_shm_rank != root) memcpy((char*)b + off, php_shm_coll, len);
        MPI_Barrier(0);
    }
    return 0;
}

static inline void php_shm_reduce_into(void* r, int n, MPI_Datatype t, MPI_Op op)
{
    const size_t sz = php_shm_tsize(t), bytes = (size_t)n * sz;
    memcpy(r, php_shm_coll, bytes);
    for (int k = 1; k < php_shm_np; k++) {
        const char* x = php_shm_coll + (size_t)k * bytes;
        for (int i = 0; i < n; i++) {
            if (t == MPI_DOUBLE) {
                double* d = (double*)r + i;
                const double v = ((const double*)x)[i];
                *d = op == MPI_MAX ? (v > *d ? v : *d) : *d + v;
            } else if (t == MPI_INT) {
                int* d = (int*)r + i;
                const int v = ((const int*)x)[i];
                *d = op == MPI_MAX ? (v > *d ? v : *d) : *d + v;
            } else if (t == MPI_UNSIGNED_LONG_LONG) {
                unsigned long long* d = (unsigned long long*)r + i;
                const unsigned long long v = ((const unsigned long long*)x)[i];
                *d = op == MPI_MAX ? (v > *d ? v : *d) : *d + v;
            } else if (t == MPI_FLOAT && sz == sizeof(double)) {
                double* d = (double*)r + i;
                const double v = ((const double*)x)[i];
                *d = op == MPI_MAX ? (v > *d ? v : *d) : *d + v;
            } else if (t == MPI_FLOAT) {
                float* d = (float*)r + i;
                const float v = ((const float*)x)[i];
                *d = op == MPI_MAX ? (v > *d ? v : *d) : *d + v;
            } else {
                fprintf(stderr, "mpi shm: reduction of datatype %d\n", t);
                exit(74);
            }
        }
    }
}

static inline int php_shm_reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, int root)
{
    const size_t bytes = (size_t)n * php_shm_tsize(t);
    if (php_shm_np == 1) {
        memmove(r, s, bytes);
        return 0;
    }
    if (bytes * (size_t)php_shm_np > PHP_SHM_COLL_BYTES) {
        fprintf(stderr, "mpi shm: reduction of %zu bytes too large\n", bytes);
        exit(75);
    }
    memcpy(php_shm_coll + (size_t)php_shm_rank * bytes, s, bytes);
    MPI_Barrier(0);
    if (root < 0 || php_shm_rank == root) php_shm_reduce_into(r, n, t, op);
    MPI_Barrier(0);
    return 0;
}

static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)c;
    return php_shm_reduce(s, r, n, t, op, -1);
}

static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)c;
    return php_shm_reduce(s, r, n, t, op, root);
}

static inline int MPI_Scatterv(const void* s, const int* counts, const int* displs, MPI_Datatype st, void* r, int rc,
                               MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rt; (void)c;
    const size_t sz = php_shm_tsize(st);
    if (php_shm_np == 1) {
        if (s) memmove(r, (const char*)s + (size_t)displs[0] * sz, (size_t)counts[0] * sz);
        return 0;
    }
    if (php_shm_rank == root) {
        int64_t total = 0;
        for (int k = 0; k < php_shm_np; k++) {
            php_shm_h->displs[k] = displs[k];
            php_shm_h->counts[k] = counts[k];
            if ((int64_t)displs[k] + counts[k] > total) total = (int64_t)displs[k] + counts[k];
        }
        php_shm_h->coll_total = total;
    }
    MPI_Barrier(0);
    const int64_t total = php_shm_h->coll_total;
    const int64_t my0 = php_shm_h->displs[php_shm_rank], my1 = my0 + rc;
    const int64_t chunk = (int64_t)(PHP_SHM_COLL_BYTES / sz);
    for (int64_t c0 = 0; c0 < total; c0 += chunk) {
        const int64_t c1 = c0 + chunk < total ? c0 + chunk : total;
        if (php_shm_rank == root) memcpy(php_shm_coll, (const char*)s + (size_t)c0 * sz, (size_t)(c1 - c0) * sz);
        MPI_Barrier(0);
        const int64_t a0 = my0 > c0 ? my0 : c0, a1 = my1 < c1 ? my1 : c1;
        if (a1 > a0) memcpy((char*)r + (size_t)(a0 - my0) * sz, php_shm_coll + (size_t)(a0 - c0) * sz, (size_t)(a1 - a0) * sz);
        MPI_Barrier(0);
    }
    return 0;
}

/* non-blocking halves of a channel transfer: one chunk if possible */
static inline int php_shm_try_put(int ch, const char* b, size_t bytes, size_t* done)
{
    php_shm_chan* q = &php_shm_ch[ch];
    if (__atomic_load_n(&q->taken, __ATOMIC_ACQUIRE) != q->posted) return 0;
    const size_t len = bytes - *done < PHP_SHM_CHAN_BYTES ? bytes - *done : PHP_SHM_CHAN_BYTES;
    memcpy(php_shm_chdata + (size_t)ch * PHP_SHM_CHAN_BYTES, b + *done, len);
    q->bytes = len;
    __atomic_store_n(&q->posted, q->posted + 1, __ATOMIC_RELEASE);
    *done += len;
    return 1;
}

static inline int php_shm_try_get(int ch, char* b, size_t bytes, size_t* done)
{
    php_shm_chan* q = &php_shm_ch[ch];
    if (__atomic_load_n(&q->posted, __ATOMIC_ACQUIRE) == q->taken) return 0;
    size_t len = q->bytes;
    if (len > bytes - *done) len = bytes - *done;
    memcpy(b + *done, php_shm_chdata + (size_t)ch * PHP_SHM_CHAN_BYTES, len);
    __atomic_store_n(&q->taken, q->taken + 1, __ATOMIC_RELEASE);
    *done += len;
    return 1;
}

static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{
    (void)tag; (void)c;
    const size_t bytes = (size_t)n * php_shm_tsize(t);
    const int ch = php_shm_chan_index(php_shm_rank, d);
    size_t done = 0;
    do {
        while (!php_shm_try_put(ch, (const char*)b, bytes, &done)) php_shm_relax();
    } while (done < bytes);
    return 0;
}

static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st)
{
    (void)c;
    const size_t bytes = (size_t)n * php_shm_tsize(t);
    const int ch = php_shm_chan_index(s, php_shm_rank);
    size_t done = 0;
    do {
        while (!php_shm_try_get(ch, (char*)b, bytes, &done)) php_shm_relax();
    } while (done < bytes);
    if (st) { st->MPI_SOURCE = s; st->MPI_TAG = tag; st->MPI_ERROR = 0; }
    return 0;
}

static inline int MPI_Sendrecv(const void* sb, int sn, MPI_Datatype stype, int d, int stag, void* rb, int rn,
                               MPI_Datatype rtype, int s, int rtag, MPI_Comm c, MPI_Status* status)
{
    (void)stag; (void)c;
    const size_t sbytes = (size_t)sn * php_shm_tsize(stype), rbytes = (size_t)rn * php_shm_tsize(rtype);
    const int cs = php_shm_chan_index(php_shm_rank, d), cr = php_shm_chan_index(s, php_shm_rank);
    /* every message is at least one chunk (an empty one for zero bytes), as
     * in MPI_Send / MPI_Recv */
    size_t sdone = 0, rdone = 0;
    int sent = 0, got = 0;
    while (!sent || !got) {
        int moved = 0;
        if (!sent && php_shm_try_put(cs, (const char*)sb, sbytes, &sdone)) {
            moved = 1;
            sent = sdone >= sbytes;
        }
        if (!got && php_shm_try_get(cr, (char*)rb, rbytes, &rdone)) {
            moved = 1;
            got = rdone >= rbytes;
        }
        if (!moved) php_shm_relax();
    }
    if (status) { status->MPI_SOURCE = s; status->MPI_TAG = rtag; status->MPI_ERROR = 0; }
    return 0;
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
