/*
 * php_serve.h -- serving loop of libphpfdtd: a stream of independent
 * simulations advanced together on one GPU (continuous batching).
 *
 * The reference runs one simulation per mpirun invocation and has no
 * counterpart; a sweep over wavenumbers or tip heights is a shell loop of
 * separate runs.  Here a server (one per GPU) has admission threads that
 *  - admit submitted simulations in arrival order while the sum of their
 *    device footprints (php_estimate_bytes + DFT planes) stays within the
 *    memory budget and the number of running simulations within max_active,
 *    and build their contexts in parallel;
 * and a stepping thread that
 *  - keeps every admitted simulation's fields on the device and keeps up to
 *    two chunks of its time steps (CUDA graphs, php_step) queued on its own
 *    stream, so that the kernels of all running simulations overlap on the
 *    device;
 *  - when a simulation has run its steps, reads its running-DFT plane back,
 *    frees its memory (stream ordered: the others keep running) and admits
 *    the next ones.
 * Each simulation's arithmetic is exactly that of a php_ctx stepped alone,
 * so its result does not depend on what else runs beside it.
 *
 * Threading: every call may come from any host thread; the server
 * serialises them internally.  Times are seconds on the server's monotonic
 * clock (php_server_clock).
 */
#ifndef PHP_SERVE_H
#define PHP_SERVE_H

#include "php_fdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct php_server php_server;

typedef struct {
    int32_t abi_version;       /* PHP_ABI_VERSION */
    int32_t device;
    uint64_t memory_budget;    /* bytes of device memory the running simulations may hold */
    int32_t max_active;        /* running simulations at most; 0 = memory bound only */
    int32_t chunk_steps;       /* time steps per queued chunk; 0 = 256 */
} php_server_desc;

/* The running DFT a job accumulates (php_dft_add arguments). */
typedef struct {
    int32_t component;         /* PHP_EX .. PHP_HZ */
    int32_t z_plane;           /* field plane index, -1..nz */
    int32_t first_step;
    int32_t interval;
    int32_t nfreq;
    int32_t cast_f32;
    const double* freq_hz;     /* nfreq frequencies */
} php_dft_request;

typedef struct {
    int64_t job;               /* id returned by php_batch_submit */
    uint64_t tag;              /* caller's tag */
    int32_t status;            /* PHP_OK or the PHP_ERR_* code of the failing call */
    int32_t steps;             /* time steps run */
    double t_submit, t_admit, t_done;
    double t_start;            /* context built, first chunk about to be queued */
    uint64_t device_bytes;     /* footprint charged against the budget */
    int32_t nx, ny, nfreq;     /* shape of the DFT result */
    int32_t dft_samples;
    char error[256];           /* php_last_error text when status != PHP_OK */
} php_job_info;

typedef struct {
    int32_t queued, running, finished_unpolled;
    int32_t peak_running;
    uint64_t bytes_in_use, peak_bytes;
    int64_t submitted, completed;
} php_server_stats;

int php_server_create(const php_server_desc* desc, php_server** out);
/* Waits for the queued and running jobs to finish, then frees the server
 * and every result not yet fetched. */
int php_server_destroy(php_server* s);
const char* php_server_last_error(const php_server* s);
int php_server_clock(const php_server* s, double* seconds);
int php_server_stats_read(php_server* s, php_server_stats* out);

/* Queues one simulation of `nsteps` time steps.  The description and the
 * arrays it points to are copied before the call returns.  dft may be NULL
 * (then the job returns no plane). */
int php_batch_submit(php_server* s, const php_desc* desc, int32_t nsteps, const php_dft_request* dft, uint64_t tag,
                     int64_t* job);
/* Moves up to `max` finished jobs into `out` (oldest first), waiting up to
 * timeout_ms for the first one (0: do not wait, <0: wait without limit).
 * *n receives the count. */
int php_batch_poll(php_server* s, php_job_info* out, int32_t max, int32_t timeout_ms, int32_t* n);
/* Copies a polled job's DFT plane, [nfreq][nx][ny][re, im] doubles, and
 * releases the job's result. */
int php_batch_fetch_dft(php_server* s, int64_t job, double* out);
/* Releases a polled job's result without reading it. */
int php_batch_release(php_server* s, int64_t job);

#ifdef __cplusplus
}
#endif

#endif /* PHP_SERVE_H */
