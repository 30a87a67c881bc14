/*
 * php_fdtd.h -- C ABI of libphpfdtd, the B200 implementation of the
 * PhP_FDTD time-step loop.
 *
 * The reference (PhP_FDTD, fdtd.c) has no library interface: its time loop
 * is written inline in main() (fdtd.c:3116-3884) between the host set-up
 * (fdtd.c:2075-3107) and the writers.  This header is the boundary that
 * replaces that inline loop: the host keeps parsing the .cfg, reading the
 * medium map and the Born/QeZV/QeZM/DMM files and writing the output files,
 * and calls these entry points for everything the loop computes.
 *
 * Conventions
 *  - Every call returns PHP_OK (0) or a negative PHP_ERR_* code; the text of
 *    the last error is returned by php_last_error().  Nothing here calls
 *    exit(): where the reference aborts (MPI_Abort/exit) this returns
 *    PHP_ERR_INPUT and the caller decides.
 *  - php_create copies every input to the device; the caller keeps
 *    ownership of all its buffers, and owns every output buffer.
 *  - One host thread per context.  All device work of a context runs on
 *    its own CUDA stream; php_step is asynchronous, the read calls
 *    synchronise.
 *  - Index conventions are the reference's: i along x (0..nx-1), j along y,
 *    k along z; host arrays in "file order" are [nx][ny][nz], z fastest,
 *    exactly as medium_map.bin (fdtd.c:808-817) and the field arrays
 *    (fdtd.c:261-284).
 */
#ifndef PHP_FDTD_H
#define PHP_FDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHP_ABI_VERSION 1

/* status codes */
#define PHP_OK 0
#define PHP_ERR_INPUT (-1)       /* invalid description / argument (reference: MPI_Abort, exit) */
#define PHP_ERR_OOM (-2)         /* device or host allocation failed */
#define PHP_ERR_CUDA (-3)        /* a CUDA call failed; see php_last_error */
#define PHP_ERR_DIVERGED (-4)    /* |r| above the reference's 1e-10 m guard (fdtd.c:3626) */
#define PHP_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define PHP_ERR_STATE (-6)       /* call not valid in the context's current state */
#define PHP_ERR_UNSUPPORTED (-7) /* feature not available in this build / precision */
#define PHP_ERR_NODEVICE (-8)    /* no CUDA device visible */

/* arithmetic of the device path */
typedef enum {
    /* FP64, every operation in the reference's order and rounding (IEEE
     * division, no fused multiply-add): reproduces fdtd.c bit for bit. */
    PHP_PREC_FP64_STRICT = 0,
    /* FP64 with host-folded coefficients (reciprocals, scaled CPML psi)
     * and FMA: the fast plain path, within 1e-10 relative L2 of the
     * reference. */
    PHP_PREC_FP64 = 1,
    /* FP32 fields, psi, ADE currents and ion r/v; coefficients folded on the
     * host in FP64; DFT accumulators stay FP64. */
    PHP_PREC_FP32 = 2
} php_precision;

/* field components (reference names, fdtd.c:3671-3707) */
typedef enum {
    PHP_EX = 0, PHP_EY = 1, PHP_EZ = 2,
    PHP_DX = 3, PHP_DY = 4, PHP_DZ = 5,
    PHP_HX = 6, PHP_HY = 7, PHP_HZ = 8,
    PHP_EMAG = 9 /* sqrt(Ex^2+Ey^2+Ez^2), output_component "E" (fdtd.c:3681-3694) */
} php_component;

/* One material of the material table (Material, fdtd.c:82-113), after every
 * host-side override (born= static tensor, dielectric= table row, switchxz
 * permutations; fdtd.c:2249-2477).  The library derives eps_inv
 * (fdtd.c:555-625), the loss factors (fdtd.c:3414-3415), the rotation
 * (fdtd.c:3429-3452) and the ADE matrices (fdtd.c:2478-2528) itself. */
typedef struct php_material_desc {
    double eps_re[9];   /* eps.xx, xy, xz, yx, yy, yz, zx, zy, zz */
    double eps_im[9];   /* eps.xxi ... zzi (imaginary part, >= 0 convention) */
    double sigma;       /* S/m */
    double anglez;      /* radians, rotation about z (fdtd.c:3429) */
    double anglex;      /* radians, rotation about x, used when anglez == 0 (fdtd.c:3437) */
    int32_t use_ade;    /* 0 or 1 (fdtd.c:107) */
    int32_t natom;      /* atoms per cell, 0 = no lattice dynamics */
    const double* qezv; /* 9*natom, [iatom][iE][idir] (fdtd.c:3424) */
    const double* qezm; /* 9*natom, [iatom][iE][idir] (fdtd.c:3510) */
    const double* dmm;  /* 9*natom*natom, [iatom][idir][jatom][jdir] (fdtd.c:3515) */
} php_material_desc;

/* One excitation source (Source, fdtd.c:123-133) after parsing defaults and
 * the wavenumber conversion (fdtd.c:1403-1510, 1913-1917). */
typedef struct php_source_desc {
    int32_t type;       /* 0 gaussian, 1 sinusoidal, 2 ricker, 3 dipole */
    int32_t x, y, z;    /* cell */
    int32_t component;  /* 'x', 'y' or 'z' */
    int32_t pad_;
    double amplitude;
    double frequency;   /* Hz */
    double t0, tau;     /* s */
    double start_time, end_time; /* s */
} php_source_desc;

/* Everything the time loop needs (Config, fdtd.c:136-169, reduced to what
 * the loop reads). */
typedef struct php_desc {
    int32_t abi_version;     /* PHP_ABI_VERSION */
    int32_t nx, ny, nz;
    double dx, dy, dz, dt;   /* m, m, m, s */
    double epsilon0, mu0;
    int32_t pml_thickness;   /* cells; CPML profile of init_pml (fdtd.c:962-989) */
    int32_t precision;       /* php_precision */
    double pml_reflection;
    double source_frequency; /* unique_source_frequency = first source's frequency (fdtd.c:1774) */
    int32_t num_materials;
    int32_t num_sources;
    const php_material_desc* materials;
    const int32_t* medium;   /* nx*ny*nz material ids in file order (z fastest) */
    const php_source_desc* sources;
    int32_t z_chunk;         /* tuning: planes per thread block along z; 0 = default */
    int32_t device;          /* CUDA device ordinal */
} php_desc;

typedef struct php_ctx php_ctx;

/* Diagnostics of the output interval (fdtd.c:3537-3597). */
typedef struct php_diag {
    double max_e;        /* max over cells of sqrt(Ex^2+Ey^2+Ez^2) */
    double max_ex;       /* max |Ex| */
    double max_r;        /* max |r| over all atom coordinates */
    int32_t argmax_r[5]; /* i, j, k, atom, dir of the first maximum in the
                            reference's loop order; all -1 if max_r == 0 */
    int32_t pad_;
} php_diag;

/* --- lifetime ------------------------------------------------------------ */

/* Validates desc, derives every coefficient, allocates the device state
 * (fields, CPML psi slabs, ADE and ion pools) and uploads the medium.
 * Replaces fdtd.c:2478-2528 (ADE coefficients), 2884-3100 (allocation and
 * zeroing) and 2954-2956 (CPML profiles). */
int php_create(const php_desc* desc, php_ctx** out);
int php_destroy(php_ctx* ctx);

/* Message of the last failed call on ctx (or of the last failed
 * php_create when ctx is NULL). */
const char* php_last_error(const php_ctx* ctx);

/* --- time stepping -------------------------------------------------------- */

/* Advances nsteps time steps from the current step t (t = 0 after create):
 * per step the H sweep (fdtd.c:3123-3231), the D sweep with the lossy
 * eps'' term (fdtd.c:3238-3356), the sources (fdtd.c:3363-3400) and the
 * D->E / ADE / ion sweep (fdtd.c:3404-3528), plus every registered probe
 * and DFT sample of those steps.  Asynchronous: the work is enqueued on the
 * context's stream (as one CUDA graph per distinct nsteps). */
int php_step(php_ctx* ctx, int32_t nsteps);
/* Waits for the context's work.  PHP_ERR_TIMEOUT if a sweep block gave up a
 * bounded wait for its plane loads (it left after its own loads landed; the
 * fields of that step are not valid, the context still answers).  With the
 * environment variable PHP_TEST_STALL_WAIT=1 at php_create, the first block
 * of every H sweep gives up such a wait on purpose (failure-path tests). */
int php_sync(php_ctx* ctx);
int php_get_step(const php_ctx* ctx, int32_t* t);
/* Records (without running) the CUDA graphs that php_step(ctx, nsteps) will
 * launch, so that the first such call does not pay for their capture.
 * Registering a probe or a DFT plane afterwards drops them again. */
int php_prepare(php_ctx* ctx, int32_t nsteps);

/* --- z slabs (several GPUs) ------------------------------------------------ */

/* A context for the planes z0 .. z0+nz_local-1 of the domain `desc`
 * describes (desc->medium and the sources in global coordinates).  This is
 * the reference's z decomposition (fdtd.c:2761-2771) with one slab per GPU:
 * the CPML z profile is the global one, sources outside the slab are
 * skipped, and every index of the read-out calls is local.  The halo planes
 * -1 and nz_local hold the neighbours' planes once the caller has copied
 * them in (see php_halo_planes); at the domain's ends they stay zero. */
int php_create_slab(const php_desc* desc, int32_t z0, int32_t nz_local, php_ctx** out);
/* Device addresses of the x, y, z component planes exchanged between
 * neighbouring slabs (fdtd.c:3120, 3235):
 *   0  E, plane 0          (sent to the slab below, before the H sweep)
 *   1  E, halo plane nz    (received from the slab above)
 *   2  H, plane nz-1       (sent to the slab above, before the E sweep)
 *   3  H, halo plane -1    (received from the slab below)
 * Each plane is plane_bytes long (nx padded, times ny, elements). */
int php_halo_planes(php_ctx* ctx, int32_t which, void** ptrs3, uint64_t* plane_bytes);
/* Half of one time step, enqueued on the context's stream without a graph:
 * half 0 = the H sweep; half 1 = the D/E sweep, ion pass, probe and DFT
 * sample, after which the step counter advances.  A slab's step is
 * [E halo exchange] half 0 [H halo exchange] half 1. */
int php_step_half(php_ctx* ctx, int32_t half);
/* One fifth of a time step, so that a slab can hide its halo exchanges
 * behind the planes that do not need them (the reference exchanges, then
 * sweeps, fdtd.c:3120-3235).  Parts, enqueued on `stream` (a cudaStream_t;
 * NULL = the context's stream):
 *   0  H sweep of the top z chunk (reads the E halo above)
 *   1  H sweep of the other chunks (no halo)
 *   2  fused E sweep of the bottom chunk (reads the H halo below)
 *   3  fused E sweep of the other chunks (no halo)
 *   4  the rest of the step: ion pass, probe, DFT; the step counter advances
 * The first of parts 0 and 1 called in a step also stages the step's source
 * values and DFT phasors on its stream.
 * The caller orders them on the device: 0 and 1 before 2 and 3 (an E chunk
 * reads H of its own plane and the plane below); 2 and 3 before 4
 * and before the next step's 0 and 1; 4 before the next step's 2 and 3.
 * Parts 0 and 1 may run concurrently, and so may 2 and 3.  With one z chunk
 * parts 1 and 3 launch nothing.  A step must not mix parts with
 * php_step_half or php_step. */
int php_step_part(php_ctx* ctx, int32_t part, void* stream);

/* --- outputs -------------------------------------------------------------- */

/* One output slice exactly as save_field_slice_parallel writes its data
 * block (fdtd.c:999-1400) in a single-rank run: axis 'z' gives [i][j]
 * (the reference reads plane position+1 there, fdtd.c:1029 with the halo
 * offset of fdtd.c:274 already in the pointers; position nz-1 reads the
 * zero halo), axis 'x' gives [j][k] at i = position, axis 'y' gives
 * [i][k] at j = position.  `out` holds nx*ny, ny*nz or nx*nz values.
 * Returns PHP_ERR_INPUT where the reference prints an error and writes no
 * file. */
int php_read_slice(php_ctx* ctx, int32_t comp, char axis, int32_t position, float* out);
int php_read_slice_f64(php_ctx* ctx, int32_t comp, char axis, int32_t position, double* out);

/* Whole component in file order [nx][ny][nz]. */
int php_read_volume(php_ctx* ctx, int32_t comp, double* out);

/* Field values at one cell (no index quirk): out[9] = Ex Ey Ez Dx Dy Dz Hx
 * Hy Hz.  k may be -1 or nz (the zero halo planes). */
int php_read_point(php_ctx* ctx, int32_t i, int32_t j, int32_t k, double* out9);

/* Lattice state of one cell: r and v (3*natom each, [iatom][dir]) and, for
 * ADE cells, P and P_old (3 each).  Buffers may be NULL.  *natom receives
 * the cell's atom count. */
int php_read_cell_state(php_ctx* ctx, int32_t i, int32_t j, int32_t k, int32_t* natom,
                        double* r, double* v, double* p_ade, double* p_ade_old);

/* Global maxima of fdtd.c:3537-3597 for the current state. */
int php_diagnostics(php_ctx* ctx, php_diag* out);

/* --- asynchronous output frames (fdtd.c:3535-3883 off the device's path) --- */

/* An output frame holds what the writer of one output step reads: the
 * diagnostics (with the fields and lattice state of the cell of max |r|,
 * which the divergence report prints, fdtd.c:3626-3663), one slice, the
 * probe rows recorded since the last frame, and the fields and lattice
 * state of the full-monitor cell.  php_frame_begin enqueues the gathers and
 * their copies into page-locked host memory on the context's stream, behind
 * the steps enqueued so far, and returns at once: the device goes on with
 * the next php_step while another host thread waits for the frame
 * (php_frame_wait), writes the files and releases it.  Frames are taken and
 * released in ticket order; the library holds PHP_FRAME_SLOTS of them, and
 * php_frame_begin waits (at most 60 s, then PHP_ERR_TIMEOUT) for the oldest
 * to be released when all are taken.  php_frame_wait and php_frame_release
 * may run on another thread than the one that steps the context. */
#define PHP_FRAME_SLOTS 3
#define PHP_FRAME_MAX_N3 192

typedef struct php_frame_req {
    int32_t diag;        /* 1: php_diagnostics, and the max |r| cell's state */
    int32_t slice_comp;  /* php_read_slice component; -1: no slice */
    int32_t slice_axis;  /* 'x', 'y' or 'z' */
    int32_t slice_pos;
    int32_t probe;       /* 1: the probe rows recorded since the last read */
    int32_t point[3];    /* php_read_point (i, j, k); point[0] < 0: none */
    int32_t cell[3];     /* php_read_cell_state r, v of (i, j, k); cell[0] < 0: none */
} php_frame_req;

typedef struct php_frame {
    int32_t step;                       /* steps done when the frame was taken */
    int32_t nrows, row_len;             /* probe rows */
    int32_t diag_natom, cell_natom;
    int32_t pad_;
    php_diag diag;
    double diag_point[9];               /* php_read_point at argmax_r[0..2] */
    double diag_r[PHP_FRAME_MAX_N3], diag_v[PHP_FRAME_MAX_N3];
    double point[9];
    double cell_r[PHP_FRAME_MAX_N3], cell_v[PHP_FRAME_MAX_N3];
    const float* slice;                 /* slice_len values; valid until release */
    int64_t slice_len;
    const double* rows;                 /* nrows x row_len; valid until release */
} php_frame;

int php_frame_begin(php_ctx* ctx, const php_frame_req* req, int32_t* ticket);
int php_frame_wait(php_ctx* ctx, int32_t ticket, php_frame* out);
int php_frame_release(php_ctx* ctx, int32_t ticket);

/* --- per-step probe (monitor_point, fdtd.c:3806-3883) ---------------------- */

/* Records, at the end of every subsequent step, the 9 field values at
 * (i, j, k_field) followed by r and v (3*natom each) of cell (i, j,
 * k_atom).  The reference's monitor reads fields at k+1 and atoms at k
 * (fdtd.c:3814-3815 with fdtd.c:274); the caller passes both indices.  One
 * probe per context; rows accumulate on the device until read. */
int php_probe_set(php_ctx* ctx, int32_t i, int32_t j, int32_t k_field, int32_t k_atom);
/* Copies the rows recorded since the last call (oldest first) into rows,
 * each row_len = 9 + 6*natom doubles; *nrows receives the count.  Fails with
 * PHP_ERR_STATE if more than max_rows rows are pending. */
int php_probe_read(php_ctx* ctx, double* rows, int32_t max_rows, int32_t* nrows, int32_t* row_len);

/* --- running DFT on a plane (the math of frequency_analysis.c:548-570) ---- */

/* Adds a running DFT of component comp on the z plane z_plane.  From step
 * first_step on, every sample_interval steps (at the end of the step t), each
 * pixel accumulates F_f += x(t) * exp(-2*pi*i*f*t*dt) in FP64 for each of the
 * nfreq frequencies (Hz).  If cast_f32 is non-zero x is rounded to float32
 * first, as the slice files hold it.  Returns the plane id in *id. */
int php_dft_add(php_ctx* ctx, int32_t comp, int32_t z_plane, int32_t first_step,
                int32_t sample_interval, int32_t nfreq, const double* freq_hz,
                int32_t cast_f32, int32_t* id);
/* Accumulators of plane id: out[f][i][j][2] (re, im), nfreq*nx*ny*2
 * doubles; *nsamples receives the number of samples taken. */
int php_dft_read(php_ctx* ctx, int32_t id, double* out, int32_t* nsamples);

/* --- information ----------------------------------------------------------- */

/* Device bytes held by the context. */
int php_memory_bytes(const php_ctx* ctx, uint64_t* bytes);
/* Device bytes php_create would allocate for this description (before any
 * php_dft_add / php_probe_set); needs no device.  Used for admission
 * against a memory budget. */
int php_estimate_bytes(const php_desc* desc, uint64_t* bytes);
/* Number of kernel launches enqueued by the last php_step call. */
int php_last_launch_count(const php_ctx* ctx, int32_t* launches);
/* How the sweep kernels split the domain's blocks (a 32 x 8 tile of one z
 * chunk) among their code paths, fixed at php_create: counts[0] fused
 * D/E sweep blocks of one plain isotropic material on the stencil-only path,
 * [1] such blocks with CPML or domain-edge cells, [2] blocks of the one
 * lossy or anisotropic material whose record rides in the kernel
 * parameters, [3] blocks of the few-atom lattice whose ions the fused sweep
 * updates, [4] all other fused-sweep blocks (the general per-cell path),
 * [5] H sweep blocks on the stencil-only path, [6] other H sweep blocks,
 * [7] the total number of blocks of one sweep.  The strict mode runs every
 * block on the general path.  No counterpart in the reference, which has
 * one loop for every cell. */
#define PHP_CENSUS_LEN 8
int php_block_census(const php_ctx* ctx, int64_t* counts);
/* Stream the context enqueues on (a cudaStream_t), for event timing. */
int php_stream(const php_ctx* ctx, void** stream);

/* Per-kernel timing.  While enabled, the recorded step graphs carry CUDA
 * events around every sweep kernel and php_step accumulates their device
 * time: ms[0] H sweep, ms[1] fused D/E sweep, ms[2] probe, ms[3] DFT,
 * ms[4] ion pass of many-atom cells, ms[5] the one-launch step (H, D and E
 * in one sweep, which replaces [0] and [1] where it runs), with the number
 * of launches of each in launches[] (both arrays hold PHP_PROFILE_KINDS
 * entries).  Enabling or disabling resets the sums. */
#define PHP_PROFILE_KINDS 6
int php_profile_enable(php_ctx* ctx, int32_t enable);
int php_profile_read(php_ctx* ctx, double* ms, int64_t* launches);

/* --- allocation-free field maxima ------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory at the moment they need the field maxima: a divergence check on a
 * device whose memory is full (resident domains take most of the HBM, and a
 * failing cudaMalloc would hide the real state), a host whose own allocator
 * owns all device memory, or a latency-critical loop where cudaMalloc /
 * cudaFree would synchronise the device.
 *
 * Computes, from three device arrays of n contiguous doubles, out2[0] =
 * max sqrt(Ex^2+Ey^2+Ez^2) and out2[1] = max |Ex| (the values php_diagnostics
 * reports as max_e and max_ex, fdtd.c:3537-3554) into out2, a device array
 * of 2 doubles, asynchronously on `stream` (a cudaStream_t, NULL = legacy
 * default stream).  It allocates nothing: its scratch is a fixed 256 KB
 * array inside the library, which every GPU that loads the library holds
 * until the process exits.  n above PHP_NOALLOC_MAX_CELLS is rejected with
 * PHP_ERR_INPUT; a larger domain is reduced in pieces of at most that many
 * cells, one call per piece.  The first call on each device looks up the
 * scratch address on that device, and so does the first call after the
 * device's context was destroyed and made anew (cudaDeviceReset); make
 * those calls before any stream capture.  Calls that overlap on the GPU
 * share the scratch and race, so serialise them. */
#define PHP_NOALLOC_MAX_CELLS 67108864 /* 2^26 cells, e.g. 512 x 512 x 256 */
int php_field_maxima_noalloc(const double* ex, const double* ey, const double* ez, int64_t n,
                             double* out2, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PHP_FDTD_H */
