/*
 * php_fdtd.cu -- libphpfdtd: the C ABI of include/php_fdtd.h on one B200.
 *
 * Host side of the device path: derives every per-material and per-axis
 * coefficient once (where the reference recomputes them per cell and step),
 * lays the domain out in HBM (see php_kernels.cuh), records one CUDA graph
 * per distinct step count and replays it, and serves the read-outs.
 *
 * Coefficients used by the strict mode are computed with the reference's
 * expressions and evaluation order (this file is compiled with host FP
 * contraction off), so the device sees the same doubles fdtd.c computes.
 */
#include "php_fdtd.h"
#include "php_kernels.cuh"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace phpdev;

namespace {

constexpr int kMaxChunk = 256;      /* steps per recorded graph */
constexpr int kProfKinds = PHP_PROFILE_KINDS; /* H sweep, E sweep, probe, DFT, ion pass, one-launch step */
constexpr int kProbeCap = 8192;     /* probe rows held on the device */
constexpr double kEpsInf = 20.0;    /* EPS_INF, fdtd.c:202 */
/* The FP32 path keeps the lattice state as 2^48 r and 2^48 v: early in a
 * pulse the reference's displacements are 1e-42 m and below, under FP32's
 * normal range (1.2e-38), where subnormals keep only a few bits; scaled,
 * every displacement from 1e-52 m to the 1e-10 m divergence guard is a
 * normal number.  The factor is folded into QeZM (times 2^48) and QeZV
 * (times 2^-48), so a = QeZM E - DMM r and P_ion = QeZV r need no extra
 * operation, and a power of two changes no rounding.  Read-outs multiply
 * by rv_unit = 2^-48. */
constexpr double kIonScale32 = 281474976710656.0; /* 2^48 */

thread_local std::string g_create_error; /* errors of php_create, per calling thread */

struct DftPlane {
    int comp, z, first, interval, nfreq, cast_f32;
    std::vector<double> freq;
    double* acc = nullptr; /* [nfreq][ny][nx][2], x fastest (php_dft_read reorders) */
    int nsamples = 0;
    int in_off = 0;        /* offset of this plane's flag in a step-input row */
};

} // namespace

struct php_ctx {
    php_desc d{};
    int prec = 0;
    int nx = 0, ny = 0, nz = 0, nxp = 0, L = 0;
    int64_t plane = 0, ncell_dev = 0;
    int zchunk = 1;
    int n3max = 0, namax_tpl = 0;
    int64_t nslot = 0;           /* pool slots, padded to a multiple of 32 */
    int z_off = 0, nz_glob = 0;  /* z slab: global index of local plane 0, global nz */
    int step_part = 7;           /* launches of a step: 1 H sweep, 2 fused E sweep, 4 the rest (ions, probe, DFT) */
    int zc_first = 0, zc_count = -1; /* z chunks the sweeps launch over (-1: all) */
    bool part_staged = false;    /* php_step_part: this step's inputs are on the device */
    int num_sms = 148;
    double rv_unit = 1.0;        /* physical r, v per stored unit (FP32: 2^-48, kIonScale32) */
    /* failure-path test (PHP_TEST_STALL_WAIT=1 at php_create): the first
     * block of every H sweep gives up a bounded wait on a barrier nothing
     * arrives on, so the error flag and PHP_ERR_TIMEOUT can be checked
     * without a fault */
    int32_t stall_test = 0;
    bool any_ade = false, any_atoms = false;
    cudaStream_t stream = nullptr;
    /* php_create's own work (allocation, zeroing, uploads) runs on a stream
     * of the highest priority, so that a context built while others keep the
     * device busy does not queue behind their sweeps; `stream` (default
     * priority) takes over at the end of php_create */
    cudaStream_t setup = nullptr;
    /* page-locked staging of host -> device uploads (upload()) */
    void* up_buf[2] = {};
    cudaEvent_t up_ev[2] = {};
    bool up_used[2] = {};
    int up_next = 0;
    /* last error text: a fixed buffer, so that php_last_error's pointer stays
     * valid while another thread (php_frame_wait) records an error */
    char err[1024] = "";
    std::mutex err_mu;
    uint64_t bytes = 0;
    std::vector<void*> allocs;

    /* device state */
    void* f[9] = {};            /* field bases (plane 0) */
    void* psi[12] = {};
    /* one-launch step (he_sweep_tma): the second buffers of E, H (fo[0..2],
     * fo[6..8]; fo[3..5] = f[3..5]) and of the H CPML state, which the
     * launch writes the new level to; swap_levels exchanges them with f and
     * psi after it.  level: how many swaps since php_create, mod 2 */
    bool fused = false;
    void* fo[9] = {};
    void* psio[6] = {};
    int level = 0;
    uint8_t* plain_hf = nullptr;  /* StepArgs::plain_hf */
    uint8_t* mat = nullptr;
    uint8_t* plain_blk = nullptr; /* plain blocks of the fused sweep (StepArgs::plain_blk) */
    double kdp[3] = {};
    uint8_t* plain_h = nullptr;   /* plain blocks of the H sweep (StepArgs::plain_h) */
    double khp[3] = {};
    int32_t* slot = nullptr;
    int64_t* slot_cell = nullptr;
    uint8_t* slot_mat = nullptr;
    int32_t* slot_n3 = nullptr;
    void *P = nullptr, *Po = nullptr, *r = nullptr, *v = nullptr;
    void* mc = nullptr;          /* MatCoef<R>[nmat] */
    void* ion_coef = nullptr;
    void* axis_tab[3][7] = {};   /* kappa b c kh kd ch cd per axis */
    int32_t* axis_slot[3] = {};
    /* per-step inputs (source values, DFT flags and phasors), double
     * buffered so that the host fills one while the GPU runs the other */
    double* step_in = nullptr;   /* buffer the graph being recorded reads */
    double* step_in_dev[2] = {};  /* [kMaxChunk][row] each */
    double* step_in_host[2] = {}; /* pinned */
    cudaEvent_t staged[2] = {};   /* copy out of step_in_host[b] finished */
    int chunk_no = 0;
    int step_row = 0;
    void* scratch = nullptr;     /* plane gathers, diagnostics */
    size_t scratch_bytes = 0;
    void* host_stage = nullptr;  /* pinned */
    size_t host_stage_bytes = 0;

    /* host copies kept for reads */
    std::vector<int> mat_natom, mat_ade, mat_flags;
    std::vector<double> mat_cs, mat_sn;
    std::vector<int32_t> slot_host_dummy;

    /* sources */
    std::vector<php_source_desc> src;
    int64_t src_cell[kMaxSources] = {};
    int32_t src_comp[kMaxSources] = {};
    int nsrc_active = 0;
    std::vector<int> src_active_index;

    /* stepping */
    int32_t t = 0;
    std::map<int, cudaGraphExec_t> graphs; /* key: 4 * steps + 2 * level + input buffer */
    int last_launches = 0;

    /* probe */
    bool probe = false;
    int64_t probe_cf = 0, probe_slot = -1;
    int probe_ka = 0;            /* plane of the atom cell */
    int probe_n3 = 0;
    double* probe_rows = nullptr;
    int32_t* probe_count = nullptr;

    std::vector<DftPlane> dft;
    /* the E sweep samples E and D planes itself (dft_folded); PHP_DFT_FOLD=0
     * at create keeps a dft_sample launch per plane; likewise it records the
     * monitor row (probe_folded; PHP_PROBE_FOLD=0) */
    bool dft_fold = true, probe_fold = true;

    /* TMA maps of the sweep kernels; maps_o those of the second buffers */
    TmaMaps maps, maps_o;
    int64_t census[PHP_CENSUS_LEN] = {}; /* php_block_census */
    int32_t* err_flag = nullptr;

    /* per-kernel timing (php_profile_enable) */
    bool profile = false;
    std::vector<cudaEvent_t> prof_ev;   /* [kMaxChunk][kProfKinds][begin, end] */
    double prof_ms[kProfKinds] = {};
    int64_t prof_n[kProfKinds] = {};

    /* many-atom cells: ion pass apart from the E sweep (php_ions.cuh) */
    bool ion_split = false, ion_tc = false;
    int ion_np = 0;              /* 3N padded to 16 */
    void* Pr = nullptr;          /* [3][nslot] */
    void* ion_dmm = nullptr;     /* CUDA-core kernel: [np][np] R */
    void* ion_dfrag = nullptr;   /* FP64 ring: m8n8k4 B fragments */
    void* ion_bsplit = nullptr;  /* tensor kernel: DMM hi, lo bf16 images */
    bool ion_pipe = false;       /* TMA-fed pass (ion_pipe) */
    IonMaps ion_maps;
    int n3_ion = 0;
    int ion_off_ref = 0;
    /* the few-atom material (N <= 4) with the most cells: its coefficients
     * ride in the sweep's kernel parameters (StepArgs::ion_k) */
    int ion_k_off = -1;
    std::vector<double> ion_k;
    std::vector<double> iso_scale;   /* StepArgs::iso, per material */
    /* per material: eps_inv, eps_im, cs, sn of the packed record; the
     * chosen one rides in StepArgs::tns_* */
    std::vector<std::array<double, 20>> mat_tns;
    int tns_id = -1;
    /* the few-atom material of ion_k and its packed record (MatCoef<R>
     * bytes), for StepArgs::amc; atom_blocks: kPlainAtoms blocks exist */
    int atom_id = -1;
    std::vector<unsigned char> atom_mc;
    bool atom_blocks = false;

    /* output frames (php_frame_begin): page-locked slots taken in ticket
     * order; state 0 free, 1 taken (begun and not released) */
    struct FrameSlot {
        std::atomic<int> state{0};
        int32_t ticket = -1, step = 0;
        php_frame_req req{};
        int64_t rows_copied = 0, slice_len = 0;
        int32_t row_len = 0;
        cudaEvent_t done = nullptr;
        FrameHead* head = nullptr;   /* pinned */
        float* slice = nullptr;      /* pinned */
        double* rows = nullptr;      /* pinned */
        size_t rows_bytes = 0;
    };
    FrameSlot frames[PHP_FRAME_SLOTS];
    int32_t frame_next = 0;
    FrameHead* frame_head_dev = nullptr;
    int32_t probe_t0 = 0;        /* step of the last probe read (rows pending = t - probe_t0) */
};

/* ------------------------------------------------------------------ utils */

static int fail(php_ctx* c, int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) {
        std::lock_guard<std::mutex> g(c->err_mu);
        memcpy(c->err, buf, sizeof(buf));
    } else {
        g_create_error = buf;
    }
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(ctx, PHP_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                       \
    } while (0)

/* Device buffers come from the device's stream-ordered pool, allocated and
 * freed on the context's stream: destroying one context never waits for the
 * work of the others (cudaFree would synchronise the whole device), which
 * the serving loop relies on. */
static int dalloc(php_ctx* ctx, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(ctx, PHP_ERR_OOM, "cudaMallocAsync(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    ctx->allocs.push_back(*p);
    ctx->bytes += bytes;
    e = cudaMemsetAsync(*p, 0, bytes, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, PHP_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
    return PHP_OK;
}

static int upload(php_ctx* ctx, void* dst, const void* src, size_t bytes);

static size_t rsize(int prec) { return prec == PHP_PREC_FP32 ? sizeof(float) : sizeof(double); }

/* --------------------------------------------------- coefficient derivation */

/* Real part of inverse_dielectric_tensor (fdtd.c:555-625). */
static int complex_inverse_re(const double* e, const double* ei, double* out)
{
    const double xx = e[0], xy = e[1], xz = e[2], yx = e[3], yy = e[4], yz = e[5], zx = e[6], zy = e[7], zz = e[8];
    const double xxi = ei[0], xyi = ei[1], xzi = ei[2], yxi = ei[3], yyi = ei[4], yzi = ei[5], zxi = ei[6],
                 zyi = ei[7], zzi = ei[8];
    double det_real = xx * (yy * zz - yz * zy) - xy * (yx * zz - yz * zx) + xz * (yx * zy - yy * zx);
    double det_imag = xxi * (yyi * zzi - yzi * zyi) - xyi * (yxi * zzi - yzi * zxi) + xzi * (yxi * zyi - yyi * zxi);
    double det_magnitude = sqrt(det_real * det_real + det_imag * det_imag);
    if (fabs(det_magnitude) < 1e-12) return -1;
    double idr = det_real / (det_real * det_real + det_imag * det_imag);
    double idi = -det_imag / (det_real * det_real + det_imag * det_imag);
    out[0] = idr * (yy * zz - yz * zy) - idi * (yyi * zzi - yzi * zyi);
    out[1] = idr * (xz * zy - xy * zz) - idi * (xzi * zyi - xyi * zzi);
    out[2] = idr * (xy * yz - xz * yy) - idi * (xyi * yzi - xzi * yyi);
    out[3] = idr * (yz * zx - yx * zz) - idi * (yzi * zxi - yxi * zzi);
    out[4] = idr * (xx * zz - xz * zx) - idi * (xxi * zzi - xzi * zxi);
    out[5] = idr * (xz * yx - xx * yz) - idi * (xzi * yxi - xxi * yzi);
    out[6] = idr * (yx * zy - yy * zx) - idi * (yxi * zyi - yyi * zxi);
    out[7] = idr * (xy * zx - xx * zy) - idi * (xyi * zxi - xxi * zyi);
    out[8] = idr * (xx * yy - xy * yx) - idi * (xxi * yyi - xyi * yxi);
    return 0;
}

/* 3x3 inverse by the adjugate (fdtd.c:205-258); -1 when |det| < 1e-12. */
static int inverse3(const double m[3][3], double inv[3][3])
{
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    if (fabs(det) < 1e-12) return -1;
    double adj[3][3];
    adj[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    adj[0][1] = -(m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    adj[0][2] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    adj[1][0] = -(m[0][1] * m[2][2] - m[0][2] * m[2][1]);
    adj[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]);
    adj[1][2] = -(m[0][0] * m[2][1] - m[0][1] * m[2][0]);
    adj[2][0] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]);
    adj[2][1] = -(m[0][0] * m[1][2] - m[0][2] * m[1][0]);
    adj[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) inv[i][j] = adj[j][i] / det;
    return 0;
}

/* Double-precision per-material coefficients in the reference's order. */
struct MatD {
    int flags = 0, natom = 0;
    double eps_inv[9] = {}, eps_im[9] = {};
    double lf = 1.0, lt = 0.0, cs = 1.0, sn = 0.0;
    double gp_inv[9] = {}, gm[9] = {}, wp2[9] = {};
};

static int derive_material(php_ctx* ctx, int id, const php_material_desc& m, MatD& o)
{
    const php_desc& d = ctx->d;
    if (complex_inverse_re(m.eps_re, m.eps_im, o.eps_inv))
        return fail(ctx, PHP_ERR_INPUT, "Error: Singular dielectric tensor! (material %d)", id);
    memcpy(o.eps_im, m.eps_im, sizeof(o.eps_im));
    /* fdtd.c:3414-3415 */
    o.lf = 1.0 / (1.0 + m.sigma * d.dt / (2 * d.epsilon0));
    o.lt = (m.sigma * d.dt / (2 * d.epsilon0)) * o.lf;
    if (fabs(m.anglez) > 1e-10) {
        o.flags |= kRotZ;
        o.cs = cos(m.anglez);
        o.sn = sin(m.anglez);
    } else if (fabs(m.anglex) > 1e-10) {
        o.flags |= kRotX;
        o.cs = cos(-m.anglex);
        o.sn = sin(-m.anglex);
    }
    if (m.use_ade != 0 && m.use_ade != 1) return fail(ctx, PHP_ERR_INPUT, "Error: use_ADE must be 0 or 1 (material %d)", id);
    if (m.use_ade == 1) {
        o.flags |= kAde;
        const double f = d.source_frequency;
        double epsr1[3][3], epsr1_inv[3][3], gama[3][3], gdt2p1[3][3], gdt2m1[3][3], gp_inv[3][3];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) epsr1[a][b] = m.eps_re[a * 3 + b];
        epsr1[0][0] = m.eps_re[0] - kEpsInf;
        epsr1[1][1] = m.eps_re[4] - kEpsInf;
        epsr1[2][2] = m.eps_re[8] - kEpsInf;
        if (epsr1[0][0] >= 0 || epsr1[1][1] >= 0 || epsr1[2][2] >= 0)
            return fail(ctx, PHP_ERR_INPUT, "Error: EPS_INF is too small for material %d", id);
        if (inverse3(epsr1, epsr1_inv)) return fail(ctx, PHP_ERR_INPUT, "Error: epsr1 can not be inversed (material %d)", id);
        const double* ei = m.eps_im;
        /* fdtd.c:2490-2498 */
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                gama[a][b] = -(ei[a * 3 + 0] * epsr1_inv[0][b] + ei[a * 3 + 1] * epsr1_inv[1][b] + ei[a * 3 + 2] * epsr1_inv[2][b]) *
                             f * 2.0 * M_PI;
        /* fdtd.c:2499-2507 */
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                o.wp2[a * 3 + b] = -f * f * 4.0 * M_PI * M_PI * epsr1[a][b] +
                                   f * 2.0 * M_PI * (gama[a][0] * ei[0 * 3 + b] + gama[a][1] * ei[1 * 3 + b] + gama[a][2] * ei[2 * 3 + b]);
        /* fdtd.c:2508-2517 */
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                gdt2p1[a][b] = +gama[a][b] * d.dt / 2.0;
                gdt2m1[a][b] = -gama[a][b] * d.dt / 2.0;
                if (a == b) {
                    gdt2p1[a][b] += 1.0;
                    gdt2m1[a][b] += 1.0;
                }
            }
        if (inverse3(gdt2p1, gp_inv)) return fail(ctx, PHP_ERR_INPUT, "Error: gdt2p1 can not be inversed (material %d)", id);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                o.gp_inv[a * 3 + b] = gp_inv[a][b];
                o.gm[a * 3 + b] = gdt2m1[a][b];
            }
    } else {
        bool lossy = false;
        for (int q = 0; q < 9; q++) lossy |= (m.eps_im[q] != 0.0);
        if (lossy) o.flags |= kLossy;
    }
    if (m.natom < 0) return fail(ctx, PHP_ERR_INPUT, "negative natom (material %d)", id);
    if (m.natom > 0) {
        if (!m.qezv || !m.qezm || !m.dmm) return fail(ctx, PHP_ERR_INPUT, "material %d: natom > 0 needs QeZV, QeZM and DMM", id);
        o.flags |= kAtoms;
        o.natom = m.natom;
    }
    return PHP_OK;
}

template <typename R>
static MatCoef<R> pack_material(const php_ctx* ctx, const MatD& s, int ion_off)
{
    MatCoef<R> o;
    memset(&o, 0, sizeof(o));
    o.flags = s.flags;
    o.natom = s.natom;
    o.ion_off = ion_off;
    const php_desc& d = ctx->d;
    const bool strict = ctx->prec == PHP_PREC_FP64_STRICT;
    const double c1 = d.dt * d.source_frequency * 2.0 * 3.14159265;
    const double e0dt2 = d.epsilon0 * d.dt * d.dt;
    for (int q = 0; q < 9; q++) {
        if (strict) {
            o.eps_inv[q] = (R)s.eps_inv[q];
            o.eps_im[q] = (R)s.eps_im[q];
            o.wp2[q] = (R)s.wp2[q];
        } else {
            o.eps_inv[q] = (R)(s.eps_inv[q] * (s.lf * (1.0 - s.lt) / d.epsilon0));
            o.eps_im[q] = (R)(s.eps_im[q] * c1 * d.epsilon0);
            o.wp2[q] = (R)(s.wp2[q] * e0dt2);
        }
        o.gp_inv[q] = (R)s.gp_inv[q];
        o.gm[q] = (R)s.gm[q];
    }
    if (ctx->prec == PHP_PREC_FP32 && (s.flags & kAde)) {
        /* increment form of the ADE recurrence (see e_update):
         * A = (I + G)^-1 2G with G = I - gm, B = (I + G)^-1 eps0 dt^2 wp2,
         * formed in double before rounding */
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
                double av = 0.0, bv = 0.0;
                for (int t = 0; t < 3; t++) {
                    const double g2 = 2.0 * ((t == q ? 1.0 : 0.0) - s.gm[t * 3 + q]); /* 2G[t][q] */
                    av += s.gp_inv[r * 3 + t] * g2;
                    bv += s.gp_inv[r * 3 + t] * s.wp2[t * 3 + q] * e0dt2;
                }
                o.gm[r * 3 + q] = (R)av;
                o.wp2[r * 3 + q] = (R)bv;
            }
    }
    o.lf = (R)s.lf;
    o.lt = (R)s.lt;
    o.cs = (R)s.cs;
    o.sn = (R)s.sn;
    o.ade_scale = (R)((1.0 - s.lt) / (d.epsilon0 * kEpsInf));
    if (!strict && !(s.flags & (kLossy | kAde | kRotZ | kRotX | kAtoms))) {
        const double* e = s.eps_inv;
        if (e[1] == 0.0 && e[2] == 0.0 && e[3] == 0.0 && e[5] == 0.0 && e[6] == 0.0 && e[7] == 0.0 && e[0] == e[4] &&
            e[0] == e[8])
            o.flags |= kIso;
    }
    return o;
}

/* init_pml (fdtd.c:962-989) and the per-cell b, c of fdtd.c:3146-3151. */
struct AxisD {
    std::vector<int32_t> slot;
    std::vector<double> kappa, b, c, kh, kd, ch, cd;
};

static void derive_axis(const php_desc& d, int n, double delta, bool is_z, AxisD& ax)
{
    const int L = d.pml_thickness;
    ax.slot.assign(n, -1);
    ax.kappa.assign(n, 1.0);
    ax.b.assign(n, 1.0);
    ax.c.assign(n, 0.0);
    ax.kh.assign(n, 0.0);
    ax.kd.assign(n, 0.0);
    ax.ch.assign(n, 0.0);
    ax.cd.assign(n, 0.0);
    std::vector<double> sigma(L > 0 ? L : 0), kappa(L > 0 ? L : 0), alpha(L > 0 ? L : 0);
    if (L > 0) {
        double m = 3.0, kappa_max = 7.0, alpha_max = 0.05;
        double eta0 = sqrt(d.mu0 / d.epsilon0);
        double sigma_max = -(m + 1) * log(d.pml_reflection) / (2.0 * eta0 * delta * L);
        for (int i = 0; i < L; i++) {
            double r = (double)(L - i) / L;
            sigma[i] = sigma_max * pow(r, m);
            kappa[i] = 1.0 + (kappa_max - 1.0) * pow(r, m);
            alpha[i] = alpha_max * (1.0 - r);
        }
    }
    for (int i = 0; i < n; i++) {
        int idx = -1, s = -1;
        if (is_z) {
            if (i < L || i >= n - L) {
                idx = (i < L) ? i : n - 1 - i;
                s = (i < L) ? i : L + idx;
            }
        } else if (L > 0 && i < L) {
            idx = i;
            s = i;
        } else if (L > 0 && i >= n - L) {
            idx = n - 1 - i;
            s = L + idx;
        }
        double kap = 1.0, bb = 1.0, cc = 0.0;
        if (idx >= 0) {
            double sx = sigma[idx];
            kap = kappa[idx];
            double ax_ = alpha[idx];
            double aw = sx / (kap * d.epsilon0) + ax_ / d.epsilon0;
            bb = exp(-aw * d.dt);
            cc = (aw > 1e-30) ? sx / (kap * kap * d.epsilon0) * (bb - 1.0) / aw : 0.0;
        }
        ax.slot[i] = s;
        ax.kappa[i] = kap;
        ax.b[i] = bb;
        ax.c[i] = cc;
        ax.kh[i] = d.dt / (d.mu0 * delta * kap);
        ax.kd[i] = d.dt / (delta * kap);
        ax.ch[i] = d.dt * cc / (d.mu0 * delta);
        ax.cd[i] = d.dt * cc / delta;
    }
}

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* calculate_source_value, fdtd.c:1923-1947 */
static double source_value(const php_source_desc* s, double time)
{
    if (time < s->start_time || time > s->end_time) return 0.0;
    switch (s->type) {
    case 0: return s->amplitude * exp(-pow((time - s->t0) / s->tau, 2));
    case 1: return s->amplitude * sin(2 * M_PI * s->frequency * time);
    case 2: {
        double t_shift = time - s->t0;
        double arg = M_PI * M_PI * s->frequency * s->frequency * t_shift * t_shift;
        return s->amplitude * (1.0 - 2.0 * arg) * exp(-arg);
    }
    case 3: return s->amplitude * sin(2 * M_PI * s->frequency * time) * exp(-pow((time - s->t0) / s->tau, 2));
    default: return 0.0;
    }
}

/* ------------------------------------------------------------ kernel args */

/* Whether the E sweep samples DFT plane q itself (StepArgs::dft_*): the first
 * kDftFold planes of E or D components; H planes and the rest take a
 * dft_sample launch after the step. */
static bool dft_folded(const php_ctx* ctx, size_t q)
{
    if (!ctx->dft_fold || ctx->dft[q].comp > PHP_DZ) return false;
    int before = 0;
    for (size_t r = 0; r < q; r++) before += ctx->dft[r].comp <= PHP_DZ;
    return before < kDftFold;
}

/* Whether the E sweep records the monitor row itself (StepArgs::probe_*):
 * the field cell is a plane of the grid (not a halo plane) in the z chunk
 * of the atom cell, whose r and v that sweep updates (no ion pass apart). */
static bool probe_folded(const php_ctx* ctx)
{
    if (!ctx->probe || !ctx->probe_fold || ctx->ion_split) return false;
    const int kf = (int)(ctx->probe_cf / ctx->plane);
    if (ctx->probe_cf < 0 || kf >= ctx->nz) return false;
    return ctx->probe_n3 == 0 || kf / ctx->zchunk == ctx->probe_ka / ctx->zchunk;
}

/* dft_sample launches per step */
static int dft_launched(const php_ctx* ctx)
{
    int n = 0;
    for (size_t q = 0; q < ctx->dft.size(); q++) n += !dft_folded(ctx, q);
    return n;
}

template <typename R>
static StepArgs<R> make_args(php_ctx* ctx, int s_local)
{
    StepArgs<R> a;
    memset(&a, 0, sizeof(a));
    R* const* fp = reinterpret_cast<R* const*>(ctx->f);
    a.f = Fields<R>{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], fp[8]};
    R* const* pp = reinterpret_cast<R* const*>(ctx->psi);
    a.psi = Psi<R>{pp[0], pp[1], pp[2], pp[3], pp[4], pp[5], pp[6], pp[7], pp[8], pp[9], pp[10], pp[11]};
    AxisTab<R>* tabs[3] = {&a.tx, &a.ty, &a.tz};
    for (int ax = 0; ax < 3; ax++) {
        AxisTab<R>& t = *tabs[ax];
        t.slot = ctx->axis_slot[ax];
        t.kappa = (const R*)ctx->axis_tab[ax][0];
        t.b = (const R*)ctx->axis_tab[ax][1];
        t.c = (const R*)ctx->axis_tab[ax][2];
        t.kh = (const R*)ctx->axis_tab[ax][3];
        t.kd = (const R*)ctx->axis_tab[ax][4];
        t.ch = (const R*)ctx->axis_tab[ax][5];
        t.cd = (const R*)ctx->axis_tab[ax][6];
    }
    a.mat = ctx->mat;
    a.slot = ctx->slot;
    a.mc = (const MatCoef<R>*)ctx->mc;
    a.ion_coef = (const R*)ctx->ion_coef;
    a.P = (R*)ctx->P;
    a.Po = (R*)ctx->Po;
    a.r = (R*)ctx->r;
    a.v = (R*)ctx->v;
    a.pr = ctx->ion_split ? (const R*)ctx->Pr : nullptr;
    a.ion_k_off = ctx->ion_k_off;
    for (size_t q = 0; q < ctx->ion_k.size() && q < (size_t)kIonK; q++) a.ion_k[q] = (R)ctx->ion_k[q];
    for (size_t q = 0; q < ctx->iso_scale.size() && q < (size_t)kIsoMats; q++) a.iso[q] = (R)ctx->iso_scale[q];
    a.plain_blk = ctx->plain_blk;
    for (int q = 0; q < 3; q++) a.kdp[q] = (R)ctx->kdp[q];
    a.plain_h = ctx->plain_h;
    for (int q = 0; q < 3; q++) a.khp[q] = (R)ctx->khp[q];
    a.tns_flags = 0;
    a.tns_cs = a.tns_sn = R(0);
    for (int q = 0; q < 9; q++) a.tns_inv[q] = a.tns_im[q] = R(0);
    if (ctx->tns_id >= 0) {
        const std::array<double, 20>& t = ctx->mat_tns[ctx->tns_id];
        a.tns_flags = ctx->mat_flags[ctx->tns_id];
        for (int q = 0; q < 9; q++) {
            a.tns_inv[q] = (R)t[q];
            a.tns_im[q] = (R)t[9 + q];
        }
        a.tns_cs = (R)t[18];
        a.tns_sn = (R)t[19];
    }
    memset(&a.amc, 0, sizeof(a.amc));
    if (ctx->atom_blocks && ctx->atom_mc.size() == sizeof(MatCoef<R>)) memcpy(&a.amc, ctx->atom_mc.data(), sizeof(MatCoef<R>));
    a.nslot = ctx->nslot;
#ifndef PHP_SMEM_MATS
#define PHP_SMEM_MATS 0
#endif
    a.nmat = PHP_SMEM_MATS ? std::min(ctx->d.num_materials, kSmemMats) : 0;
    a.nx = ctx->nx;
    a.ny = ctx->ny;
    a.nz = ctx->nz;
    a.nxp = ctx->nxp;
    a.L = ctx->L;
    a.zchunk = ctx->zchunk;
    a.plane = ctx->plane;
    const php_desc& d = ctx->d;
    a.dt = d.dt;
    a.dxs = d.dx;
    a.dys = d.dy;
    a.dzs = d.dz;
    a.mu0 = d.mu0;
    a.eps0 = d.epsilon0;
    a.c1 = d.dt * d.source_frequency * 2.0 * 3.14159265;
    a.e0dt2 = d.epsilon0 * d.dt * d.dt;
    a.nsrc = ctx->nsrc_active;
    for (int s = 0; s < ctx->nsrc_active; s++) {
        a.src_cell[s] = ctx->src_cell[s];
        a.src_comp[s] = ctx->src_comp[s];
    }
    a.src_val = ctx->step_in + (size_t)s_local * ctx->step_row;
    a.err = ctx->err_flag;
    a.stall_test = ctx->stall_test;
    a.ndft = 0;
    for (size_t q = 0; q < ctx->dft.size(); q++) {
        if (!dft_folded(ctx, q)) continue;
        const DftPlane& p = ctx->dft[q];
        a.dft_z[a.ndft] = p.z;
        a.dft_comp[a.ndft] = p.comp;
        a.dft_nfreq[a.ndft] = p.nfreq;
        a.dft_cast[a.ndft] = p.cast_f32;
        a.dft_off[a.ndft] = p.in_off;
        a.dft_acc[a.ndft] = p.acc;
        a.ndft++;
    }
    a.probe_rows = nullptr;
    if (probe_folded(ctx)) {
        const int64_t cf = ctx->probe_cf;
        a.probe_rows = ctx->probe_rows;
        a.probe_count = ctx->probe_count;
        a.probe_kf = (int32_t)(cf / ctx->plane);
        a.probe_j = (int32_t)((cf % ctx->plane) / ctx->nxp);
        a.probe_i = (int32_t)(cf % ctx->nxp);
        a.probe_n3 = ctx->probe_n3;
        a.probe_slot = ctx->probe_slot;
        a.probe_cap = kProbeCap;
    }
    a.rv_unit = ctx->rv_unit;
    if (ctx->fused) {
        for (int q = 0; q < 3; q++) {
            a.enew[q] = (R*)ctx->fo[PHP_EX + q];
            a.hnew[q] = (R*)ctx->fo[PHP_HX + q];
        }
        for (int q = 0; q < 6; q++) a.psin_h[q] = (R*)ctx->psio[q];
        a.plain_hf = ctx->plain_hf;
    }
    return a;
}

/* After a one-launch step: the buffers it wrote hold the current E, H and H
 * CPML state (on the host side, for every later launch and read). */
static void swap_levels(php_ctx* ctx)
{
    for (int q = 0; q < 3; q++) {
        std::swap(ctx->f[PHP_EX + q], ctx->fo[PHP_EX + q]);
        std::swap(ctx->f[PHP_HX + q], ctx->fo[PHP_HX + q]);
    }
    for (int q = 0; q < 6; q++) std::swap(ctx->psi[q], ctx->psio[q]);
    std::swap(ctx->maps, ctx->maps_o);
    ctx->level ^= 1;
}

static inline void prof_mark(php_ctx* ctx, int s_local, int kind, int end)
{
    if (ctx->profile)
        cudaEventRecordWithFlags(ctx->prof_ev[((size_t)s_local * kProfKinds + kind) * 2 + end], ctx->stream,
                                 cudaEventRecordExternal);
}

template <typename R>
static void launch_ions(php_ctx* ctx)
{
    IonArgs<R> a;
    memset(&a, 0, sizeof(a));
    R* const* fp = reinterpret_cast<R* const*>(ctx->f);
    a.ex = fp[0];
    a.ey = fp[1];
    a.ez = fp[2];
    a.r = (R*)ctx->r;
    a.v = (R*)ctx->v;
    a.pr = (R*)ctx->Pr;
    a.slot_cell = ctx->slot_cell;
    a.slot_n3 = ctx->slot_n3;
    a.slot_mat = ctx->slot_mat;
    a.ion_off_ref = ctx->ion_off_ref;
    a.mat = ctx->mat;
    a.mc = (const MatCoef<R>*)ctx->mc;
    a.ion_coef = (const R*)ctx->ion_coef;
    a.dmm = (const R*)ctx->ion_dmm;
    a.dfrag = (const double*)ctx->ion_dfrag;
    a.bsplit = (const uint32_t*)ctx->ion_bsplit;
    a.nslot = ctx->nslot;
    a.ntiles = (int32_t)((ctx->nslot + kIonTile - 1) / kIonTile);
    a.dt = ctx->d.dt;
    a.err = ctx->err_flag;
    cudaStream_t st = ctx->stream;
    if (ctx->ion_pipe) {
        /* one persistent CTA per SM */
        const int grid = (int)std::min<int64_t>(a.ntiles, ctx->num_sms);
        const int n3 = ctx->n3_ion;
#define PHP_ION_PIPE(NP, S) \
    ion_pipe<R, NP, S><<<grid, IonPipe<R, NP, S>::THREADS, IonPipe<R, NP, S>::SMEM, st>>>(a, ctx->ion_maps, n3)
        if constexpr (sizeof(R) == 4) {
            switch (ctx->ion_np) {
            case 16: PHP_ION_PIPE(16, 3); break;
            case 32: PHP_ION_PIPE(32, 3); break;
            case 48: PHP_ION_PIPE(48, 3); break;
            default: PHP_ION_PIPE(64, 2); break;
            }
        } else {
            switch (ctx->ion_np) {
            case 16: PHP_ION_PIPE(16, 2); break;
            case 32: PHP_ION_PIPE(32, 2); break;
            default: PHP_ION_PIPE(48, 2); break;
            }
        }
#undef PHP_ION_PIPE
        return;
    }
    const int grid = (int)std::min<int64_t>(a.ntiles, 148 * 4);
    ion_update_cc<R, 64><<<grid, kIonTile, 0, st>>>(a);
}

template <typename R, bool STRICT, int NA>
static void launch_step_t(php_ctx* ctx, int s_local, int& launches)
{
    StepArgs<R> a = make_args<R>(ctx, s_local);
    dim3 block(kBlockX, kBlockY, 1);
    const int nchunk = (ctx->nz + ctx->zchunk - 1) / ctx->zchunk;
    a.zc0 = ctx->zc_count < 0 ? 0 : ctx->zc_first;
    dim3 grid((ctx->nx + kBlockX - 1) / kBlockX, (ctx->ny + kBlockY - 1) / kBlockY,
              ctx->zc_count < 0 ? nchunk : ctx->zc_count);
    bool do_h = ctx->step_part & 1, do_e = ctx->step_part & 2;
    const bool do_rest = ctx->step_part & 4;
    if constexpr (!STRICT) {
        if (ctx->fused && do_h && do_e && grid.z > 0) {
            /* the one-launch step: reads this level, writes the other */
            prof_mark(ctx, s_local, 5, 0);
            he_sweep_tma<R, NA><<<grid, block, FusedGeom<R>::SMEM, ctx->stream>>>(a, ctx->maps);
            prof_mark(ctx, s_local, 5, 1);
            launches++;
            swap_levels(ctx);
            do_h = do_e = false;
        }
    }
    if (grid.z == 0) { /* an empty part: no sweep blocks */
    } else if (do_h) {
        prof_mark(ctx, s_local, 0, 0);
        h_sweep_tma<R, STRICT><<<grid, block, TmaGeom<R>::H_SMEM, ctx->stream>>>(a, ctx->maps);
        prof_mark(ctx, s_local, 0, 1);
        launches++;
    }
    if (do_e && grid.z > 0) {
        prof_mark(ctx, s_local, 1, 0);
        e_sweep_tma<R, STRICT, NA><<<grid, block, TmaGeom<R>::E_SMEM + a.nmat * sizeof(MatCoef<R>), ctx->stream>>>(a, ctx->maps);
        prof_mark(ctx, s_local, 1, 1);
        launches++;
    }
    if (!do_rest) return;
    if constexpr (!STRICT && NA == 0) {
        if (ctx->ion_split) {
            prof_mark(ctx, s_local, 4, 0);
            launch_ions<R>(ctx);
            prof_mark(ctx, s_local, 4, 1);
            launches++;
        }
    }
    if (ctx->probe && !probe_folded(ctx)) {
        prof_mark(ctx, s_local, 2, 0);
        R* const* fp = reinterpret_cast<R* const*>(ctx->f);
        Fields<R> f{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], fp[8]};
        const int threads = (9 + 2 * ctx->probe_n3 + 31) / 32 * 32;
        probe_record_counted<R><<<1, threads, 0, ctx->stream>>>(
            f, ctx->probe_cf, (const R*)ctx->r, (const R*)ctx->v, ctx->rv_unit, ctx->nslot, ctx->probe_slot,
            ctx->probe_n3, ctx->probe_rows, ctx->probe_count, kProbeCap, 9 + 2 * ctx->probe_n3);
        prof_mark(ctx, s_local, 2, 1);
        launches++;
    }
    const bool dft_kernels = dft_launched(ctx) > 0;
    if (dft_kernels) prof_mark(ctx, s_local, 3, 0);
    for (size_t q = 0; q < ctx->dft.size(); q++) {
        if (dft_folded(ctx, q)) continue; /* sampled by the E sweep */
        const DftPlane& p = ctx->dft[q];
        R* const* fp = reinterpret_cast<R* const*>(ctx->f);
        const int64_t n = (int64_t)ctx->nx * ctx->ny;
        int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
        dft_sample<R><<<blocks, 256, 0, ctx->stream>>>(fp[p.comp], (int64_t)p.z * ctx->plane, ctx->nx, ctx->ny, ctx->nxp,
                                                       p.nfreq, p.cast_f32, ctx->step_in + (size_t)s_local * ctx->step_row,
                                                       p.in_off, p.in_off + 1, p.acc);
        launches++;
    }
    if (dft_kernels) prof_mark(ctx, s_local, 3, 1);
}

typedef void (*step_fn)(php_ctx*, int, int&);
typedef int (*prep_fn)(php_ctx*);

/* the TMA sweeps need more than the default 48 KB of dynamic shared memory */
template <typename R, bool STRICT, int NA>
static int prepare_t(php_ctx* ctx)
{
    cudaError_t e = cudaFuncSetAttribute(h_sweep_tma<R, STRICT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TmaGeom<R>::H_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(e_sweep_tma<R, STRICT, NA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(TmaGeom<R>::E_SMEM + kSmemMats * sizeof(MatCoef<R>)));
    if constexpr (!STRICT)
        if (e == cudaSuccess && ctx->fused)
            e = cudaFuncSetAttribute(he_sweep_tma<R, NA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)FusedGeom<R>::SMEM);
    if (e != cudaSuccess) return fail(ctx, PHP_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    return PHP_OK;
}

struct StepKernels {
    step_fn launch;
    prep_fn prepare;
};

template <typename R, bool STRICT>
static StepKernels pick_na(int namax)
{
    switch (namax) {
    case 0: return {launch_step_t<R, STRICT, 0>, prepare_t<R, STRICT, 0>};
    case 2: return {launch_step_t<R, STRICT, 2>, prepare_t<R, STRICT, 2>};
    case 4: return {launch_step_t<R, STRICT, 4>, prepare_t<R, STRICT, 4>};
    case 8: return {launch_step_t<R, STRICT, 8>, prepare_t<R, STRICT, 8>};
    case 16: return {launch_step_t<R, STRICT, 16>, prepare_t<R, STRICT, 16>};
    default: return {launch_step_t<R, STRICT, 64>, prepare_t<R, STRICT, 64>};
    }
}

static StepKernels pick_step(const php_ctx* ctx)
{
    /* with the ion pass apart, the E sweep carries no per-atom state */
    const int na = ctx->ion_split ? 0 : ctx->namax_tpl;
    if (ctx->prec == PHP_PREC_FP64_STRICT) return pick_na<double, true>(ctx->namax_tpl);
    if (ctx->prec == PHP_PREC_FP64) return pick_na<double, false>(na);
    return pick_na<float, false>(na);
}

/* ------------------------------------------------------------ tensor maps */

static int encode_map(php_ctx* ctx, CUtensorMap* m, void* base, CUtensorMapDataType dt, size_t esize, uint64_t d0,
                      uint64_t d1, uint64_t d2, uint32_t b0, uint32_t b1)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
            q != cudaDriverEntryPointSuccess)
            return fail(ctx, PHP_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {d0 * esize, d0 * d1 * esize};
    const cuuint32_t box[3] = {b0, b1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ctx, PHP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PHP_OK;
}

/* Maps of the field arrays (planes -1..nz) and the material ids (planes
 * 0..nz-1) with the boxes of php_sweeps_tma.cuh. */
template <typename R>
static int make_maps(php_ctx* ctx)
{
    using G = TmaGeom<R>;
    const CUtensorMapDataType dt = sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const uint64_t nxp = ctx->nxp, ny = ctx->ny, nzh = ctx->nz + 2;
    int rc = PHP_OK;
    using F = FusedGeom<R>;
    /* maps of the current buffers, then (one-launch step) of the second ones */
    for (int set = 0; set < (ctx->fused ? 2 : 1) && !rc; ++set) {
        TmaMaps& m = set ? ctx->maps_o : ctx->maps;
        void* const* fb = set ? ctx->fo : ctx->f;
        auto base = [&](int q) { return (void*)((char*)fb[q] - (size_t)ctx->plane * sizeof(R)); };
        for (int q = 0; q < 3 && !rc; ++q) {
            rc = encode_map(ctx, &m.e_halo[q], base(PHP_EX + q), dt, sizeof(R), nxp, ny, nzh, G::BX, G::BY);
            if (!rc) rc = encode_map(ctx, &m.h_own[q], base(PHP_HX + q), dt, sizeof(R), nxp, ny, nzh, G::TX, G::TY);
            if (!rc) rc = encode_map(ctx, &m.h_halo[q], base(PHP_HX + q), dt, sizeof(R), nxp, ny, nzh, G::BX, G::BY);
            if (!rc) rc = encode_map(ctx, &m.d_own[q], base(PHP_DX + q), dt, sizeof(R), nxp, ny, nzh, G::TX, G::TY);
            if (!rc) rc = encode_map(ctx, &m.e_wide[q], base(PHP_EX + q), dt, sizeof(R), nxp, ny, nzh, F::EX, F::EY);
        }
        if (!rc) rc = encode_map(ctx, &m.mat, ctx->mat, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, nxp, ny, ctx->nz, G::TX, G::TY);
    }
    return rc;
}

/* --------------------------------------------------------------- creation */

template <typename R>
static int upload_tables(php_ctx* ctx, const std::vector<MatD>& mats, const std::vector<int>& ion_off,
                         const std::vector<double>& ion_coef, const AxisD* axes)
{
    std::vector<MatCoef<R>> mc(mats.size());
    ctx->iso_scale.assign(mats.size(), 0.0);
    ctx->mat_tns.assign(mats.size(), {});
    for (size_t i = 0; i < mats.size(); i++) {
        mc[i] = pack_material<R>(ctx, mats[i], ion_off[i]);
        if (mc[i].flags & kIso) ctx->iso_scale[i] = (double)mc[i].eps_inv[0];
        for (int q = 0; q < 9; q++) {
            ctx->mat_tns[i][q] = (double)mc[i].eps_inv[q];
            ctx->mat_tns[i][9 + q] = (double)mc[i].eps_im[q];
        }
        ctx->mat_tns[i][18] = (double)mc[i].cs;
        ctx->mat_tns[i][19] = (double)mc[i].sn;
        if ((int)i == ctx->atom_id) {
            const unsigned char* p = reinterpret_cast<const unsigned char*>(&mc[i]);
            ctx->atom_mc.assign(p, p + sizeof(MatCoef<R>));
        }
    }
    int rc = dalloc(ctx, &ctx->mc, mc.size() * sizeof(MatCoef<R>));
    if (rc) return rc;
    if ((rc = upload(ctx, ctx->mc, mc.data(), mc.size() * sizeof(MatCoef<R>)))) return rc;
    std::vector<R> ic(ion_coef.size() ? ion_coef.size() : 1);
    for (size_t i = 0; i < ion_coef.size(); i++) ic[i] = (R)ion_coef[i];
    rc = dalloc(ctx, &ctx->ion_coef, ic.size() * sizeof(R));
    if (rc) return rc;
    if ((rc = upload(ctx, ctx->ion_coef, ic.data(), ic.size() * sizeof(R)))) return rc;
    for (int ax = 0; ax < 3; ax++) {
        const AxisD& A = axes[ax];
        const std::vector<double>* cols[7] = {&A.kappa, &A.b, &A.c, &A.kh, &A.kd, &A.ch, &A.cd};
        for (int q = 0; q < 7; q++) {
            std::vector<R> h(cols[q]->size());
            for (size_t i = 0; i < h.size(); i++) h[i] = (R)(*cols[q])[i];
            rc = dalloc(ctx, &ctx->axis_tab[ax][q], h.size() * sizeof(R));
            if (rc) return rc;
            if ((rc = upload(ctx, ctx->axis_tab[ax][q], h.data(), h.size() * sizeof(R)))) return rc;
        }
        rc = dalloc(ctx, (void**)&ctx->axis_slot[ax], A.slot.size() * sizeof(int32_t));
        if (rc) return rc;
        if ((rc = upload(ctx, ctx->axis_slot[ax], A.slot.data(), A.slot.size() * sizeof(int32_t)))) return rc;
    }
    /* host tables must stay alive until the copies finish */
    CK(cudaStreamSynchronize(ctx->stream));
    return PHP_OK;
}

/* Page-locked host buffers, kept for reuse by later contexts: freeing one
 * (cudaFreeHost) can wait for the whole device, which would stall the other
 * contexts a serving loop runs beside it. */
static std::mutex g_pinned_mu;
static std::multimap<size_t, void*> g_pinned_free;
static std::map<void*, size_t> g_pinned_size;

static void* pinned_get(size_t bytes)
{
    {
        std::lock_guard<std::mutex> g(g_pinned_mu);
        auto it = g_pinned_free.lower_bound(bytes);
        if (it != g_pinned_free.end() && it->first <= 2 * bytes) {
            void* p = it->second;
            g_pinned_free.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> g(g_pinned_mu);
    g_pinned_size[p] = bytes;
    return p;
}

static void pinned_put(void* p)
{
    if (!p) return;
    std::lock_guard<std::mutex> g(g_pinned_mu);
    g_pinned_free.emplace(g_pinned_size[p], p);
}

/* Host -> device copy through page-locked staging.  A copy from pageable
 * memory is staged by the driver in small synchronous pieces; while other
 * contexts kept the device busy that took up to seconds per context.  Here
 * chunks of up to kUploadChunk go through two pooled page-locked buffers,
 * one copy in flight while the other buffer fills.  The source may be freed
 * on return. */
constexpr size_t kUploadChunk = (size_t)4 << 20;
static int upload(php_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (bytes == 0) return PHP_OK;
    for (int b = 0; b < 2; ++b) {
        if (!ctx->up_buf[b]) {
            ctx->up_buf[b] = pinned_get(kUploadChunk);
            if (!ctx->up_buf[b]) return fail(ctx, PHP_ERR_OOM, "page-locked host allocation failed");
            ctx->up_used[b] = false;
        }
        if (!ctx->up_ev[b]) CK(cudaEventCreateWithFlags(&ctx->up_ev[b], cudaEventDisableTiming));
    }
    for (size_t off = 0; off < bytes;) {
        const int b = ctx->up_next & 1;
        const size_t n = std::min(kUploadChunk, bytes - off);
        if (ctx->up_used[b]) CK(cudaEventSynchronize(ctx->up_ev[b])); /* its last copy has left */
        memcpy(ctx->up_buf[b], (const char*)src + off, n);
        CK(cudaMemcpyAsync((char*)dst + off, ctx->up_buf[b], n, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaEventRecord(ctx->up_ev[b], ctx->stream));
        ctx->up_used[b] = true;
        ctx->up_next++;
        off += n;
    }
    return PHP_OK;
}

/* returns the staging buffers to the pool once their copies are done */
static void upload_release(php_ctx* ctx)
{
    for (int b = 0; b < 2; ++b) {
        if (ctx->up_used[b]) cudaEventSynchronize(ctx->up_ev[b]);
        pinned_put(ctx->up_buf[b]);
        ctx->up_buf[b] = nullptr;
        ctx->up_used[b] = false;
    }
}

static void ctx_free(php_ctx* ctx)
{
    if (!ctx) return;
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
    for (void* p : ctx->allocs) cudaFreeAsync(p, ctx->stream);
    ctx->allocs.clear();
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (cudaEvent_t e : ctx->prof_ev) cudaEventDestroy(e);
    ctx->prof_ev.clear();
    pinned_put(ctx->host_stage);
    for (int b = 0; b < 2; ++b) {
        pinned_put(ctx->step_in_host[b]);
        if (ctx->staged[b]) cudaEventDestroy(ctx->staged[b]);
    }
    upload_release(ctx);
    for (int b = 0; b < 2; ++b)
        if (ctx->up_ev[b]) cudaEventDestroy(ctx->up_ev[b]);
    for (auto& f : ctx->frames) {
        if (f.done) cudaEventDestroy(f.done);
        pinned_put(f.head);
        pinned_put(f.slice);
        pinned_put(f.rows);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->setup && ctx->setup != ctx->stream) {
        cudaStreamSynchronize(ctx->setup);
        cudaStreamDestroy(ctx->setup);
    }
    delete ctx;
}

/* (Re)allocates both per-step input buffers for rows of `row` doubles; the
 * stream must be idle.  Replaced device buffers stay allocated until
 * destroy. */
static int alloc_step_inputs(php_ctx* ctx, int row)
{
    ctx->step_row = row;
    for (int b = 0; b < 2; ++b) {
        int rc = dalloc(ctx, (void**)&ctx->step_in_dev[b], (size_t)kMaxChunk * row * sizeof(double));
        if (rc) return rc;
        pinned_put(ctx->step_in_host[b]);
        ctx->step_in_host[b] = (double*)pinned_get((size_t)kMaxChunk * row * sizeof(double));
        if (!ctx->step_in_host[b]) return fail(ctx, PHP_ERR_OOM, "page-locked host allocation failed");
        if (!ctx->staged[b]) CK(cudaEventCreateWithFlags(&ctx->staged[b], cudaEventDisableTiming));
    }
    ctx->step_in = ctx->step_in_dev[0];
    return PHP_OK;
}

template <typename R, int NP, int S>
static cudaError_t ion_pipe_attr()
{
    return cudaFuncSetAttribute(ion_pipe<R, NP, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)IonPipe<R, NP, S>::SMEM);
}

/* bf16 bits of x, rounded to nearest even (finite inputs) */
static uint16_t bf16_bits(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

static double bf16_value(uint16_t b)
{
    const uint32_t u = (uint32_t)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

/* Many-atom cells (3N >= 24, one DMM shared by every atom material) get the
 * ion pass of php_ions.cuh in the fast FP64 and FP32 paths; PHP_IONS=fused
 * keeps the update inside the E sweep and PHP_IONS=pass moves few-atom cells
 * to the pass too (both for A/B timing). */
static int setup_ion_pass(php_ctx* ctx, const std::vector<MatD>& mats, const std::vector<int>& ion_off, const php_desc& d)
{
    const char* iv = getenv("PHP_IONS");
    const bool force = iv && !strcmp(iv, "pass");
    if ((iv && !strcmp(iv, "fused")) || ctx->prec == PHP_PREC_FP64_STRICT || (ctx->n3max < 24 && !force) ||
        ctx->n3max == 0 || ctx->n3max > 64)
        return PHP_OK;
    int ref = -1;
    for (int i = 0; i < d.num_materials; i++) {
        if (mats[i].natom == 0) continue;
        if (ref < 0) {
            ref = i;
            continue;
        }
        const int N = mats[i].natom;
        if (N != mats[ref].natom || memcmp(d.materials[i].dmm, d.materials[ref].dmm, sizeof(double) * 9 * N * N))
            return PHP_OK; /* several lattices: keep the fused update */
    }
    if (ref < 0) return PHP_OK;
    const int n3 = 3 * mats[ref].natom, np = (n3 + 15) / 16 * 16;
    const double* D = d.materials[ref].dmm;
    const size_t rs = rsize(ctx->prec);
    int rc = dalloc(ctx, &ctx->Pr, 3 * (size_t)ctx->nslot * rs);
    if (rc) return rc;
    if (ctx->prec == PHP_PREC_FP32) {
        /* B operand of D = r DMM^T: row n = output coordinate q, k = p */
        std::vector<uint16_t> img(2 * (size_t)np * np, 0);
        for (int q = 0; q < n3; q++)
            for (int p = 0; p < n3; p++) {
                const double x = D[(size_t)q * n3 + p];
                const uint16_t hi = bf16_bits((float)x);
                const uint16_t lo = bf16_bits((float)(x - bf16_value(hi)));
                const size_t off = umma_kmajor_off(q, p, np) / 2;
                img[off] = hi;
                img[(size_t)np * np + off] = lo;
            }
        if ((rc = dalloc(ctx, &ctx->ion_bsplit, img.size() * 2))) return rc;
        if ((rc = upload(ctx, ctx->ion_bsplit, img.data(), img.size() * 2))) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->ion_tc = true;
    } else {
        std::vector<double> pad((size_t)np * np, 0.0);
        for (int q = 0; q < n3; q++)
            for (int p = 0; p < n3; p++) pad[(size_t)q * np + p] = D[(size_t)q * n3 + p];
        if ((rc = dalloc(ctx, &ctx->ion_dmm, pad.size() * sizeof(double)))) return rc;
        if ((rc = upload(ctx, ctx->ion_dmm, pad.data(), pad.size() * sizeof(double)))) return rc;
        /* the same matrix as B fragments of the m8n8k4 FP64 MMA (B[k][n] =
         * DMM[n][k]): lane l of fragment (ks, nt) holds B[4 ks + l % 4][8 nt + l / 4];
         * then the E step, B[t][q] = -QeZM(q, t) (t < 3), and P_ion's B[p][c] =
         * QeZV(c, p) (c < 3), both of the lattice (fdtd.c:3418-3427, 3507-3528) */
        const double* zv = d.materials[ref].qezv;
        const double* zm = d.materials[ref].qezm;
        std::vector<double> frag((size_t)np * np + (size_t)(np / 8) * 32 + (size_t)(np / 4) * 32, 0.0);
        for (int ks = 0; ks < np / 4; ks++)
            for (int nt = 0; nt < np / 8; nt++)
                for (int l = 0; l < 32; l++) {
                    const int q = nt * 8 + l / 4, p = ks * 4 + l % 4;
                    frag[((size_t)ks * (np / 8) + nt) * 32 + l] = (q < n3 && p < n3) ? D[(size_t)q * n3 + p] : 0.0;
                }
        const size_t fe = (size_t)np * np, fp = fe + (size_t)(np / 8) * 32;
        for (int nt = 0; nt < np / 8; nt++)
            for (int l = 0; l < 32; l++) {
                const int t = l % 4, q = nt * 8 + l / 4;
                frag[fe + (size_t)nt * 32 + l] = (t < 3 && q < n3) ? -zm[(q / 3) * 9 + t * 3 + q % 3] : 0.0;
            }
        for (int ks = 0; ks < np / 4; ks++)
            for (int l = 0; l < 32; l++) {
                const int p = ks * 4 + l % 4, c = l / 4;
                frag[fp + (size_t)ks * 32 + l] = (c < 3 && p < n3) ? zv[(p / 3) * 9 + c * 3 + p % 3] : 0.0;
            }
        if ((rc = dalloc(ctx, &ctx->ion_dfrag, frag.size() * sizeof(double)))) return rc;
        if ((rc = upload(ctx, ctx->ion_dfrag, frag.data(), frag.size() * sizeof(double)))) return rc;
        CK(cudaStreamSynchronize(ctx->stream));
    }
    ctx->ion_np = np;
    ctx->ion_split = true;
    ctx->n3_ion = n3;
    ctx->ion_off_ref = ion_off[ref];
    ctx->ion_pipe = ctx->prec == PHP_PREC_FP32 ? np <= 64 : np <= 48;
    if (ctx->ion_pipe) {
        const CUtensorMapDataType dt = ctx->prec == PHP_PREC_FP32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        rc = encode_map(ctx, &ctx->ion_maps.r, ctx->r, dt, rs, (uint64_t)ctx->nslot, (uint64_t)n3, 1, kIonTile, (uint32_t)n3);
        if (!rc) rc = encode_map(ctx, &ctx->ion_maps.v, ctx->v, dt, rs, (uint64_t)ctx->nslot, (uint64_t)n3, 1, kIonTile, (uint32_t)n3);
        if (rc) return rc;
        cudaError_t e;
        if (ctx->prec == PHP_PREC_FP32)
            e = np == 16 ? ion_pipe_attr<float, 16, 3>() : np == 32 ? ion_pipe_attr<float, 32, 3>()
              : np == 48 ? ion_pipe_attr<float, 48, 3>() : ion_pipe_attr<float, 64, 2>();
        else
            e = np == 16 ? ion_pipe_attr<double, 16, 2>() : np == 32 ? ion_pipe_attr<double, 32, 2>()
                         : ion_pipe_attr<double, 48, 2>();
        if (e != cudaSuccess) return fail(ctx, PHP_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    }
    return PHP_OK;
}

static int create_impl(const php_desc* desc, php_ctx* ctx)
{
    const php_desc& d = *desc;
    if (d.abi_version != PHP_ABI_VERSION) return fail(ctx, PHP_ERR_INPUT, "abi_version %d, library %d", d.abi_version, PHP_ABI_VERSION);
    if (d.nx < 2 || d.ny < 2 || d.nz < 1) return fail(ctx, PHP_ERR_INPUT, "grid %dx%dx%d too small", d.nx, d.ny, d.nz);
    if (!(d.dt > 0) || !(d.dx > 0) || !(d.dy > 0) || !(d.dz > 0))
        return fail(ctx, PHP_ERR_INPUT, "dt and cell sizes must be positive");
    if (d.precision < 0 || d.precision > 2) return fail(ctx, PHP_ERR_INPUT, "unknown precision %d", d.precision);
    if (d.pml_thickness < 0) return fail(ctx, PHP_ERR_INPUT, "negative pml_thickness");
    if (d.num_materials < 1 || d.num_materials > 256 || !d.materials)
        return fail(ctx, PHP_ERR_INPUT, "num_materials must be 1..256 (got %d)", d.num_materials);
    if (!d.medium) return fail(ctx, PHP_ERR_INPUT, "medium is NULL");
    if (d.num_sources < 0 || (d.num_sources > 0 && !d.sources)) return fail(ctx, PHP_ERR_INPUT, "bad sources");
    ctx->d = d;
    if (ctx->nz_glob == 0) ctx->nz_glob = d.nz;
    ctx->prec = d.precision;
    ctx->nx = d.nx;
    ctx->ny = d.ny;
    ctx->nz = d.nz;
    ctx->nxp = (d.nx + 31) / 32 * 32;
    ctx->L = d.pml_thickness;
    ctx->plane = (int64_t)ctx->nxp * d.ny;
    ctx->ncell_dev = ctx->plane * d.nz;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ctx, PHP_ERR_NODEVICE, "no CUDA device visible");
    if (d.device < 0 || d.device >= ndev) return fail(ctx, PHP_ERR_INPUT, "device %d not present", d.device);
    CK(cudaSetDevice(d.device));
    CK(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, d.device));
    {
        int least = 0, greatest = 0;
        CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CK(cudaStreamCreateWithPriority(&ctx->setup, cudaStreamNonBlocking, greatest));
        ctx->stream = ctx->setup;
    }

    /* materials */
    std::vector<MatD> mats(d.num_materials);
    std::vector<int> ion_off(d.num_materials, 0);
    std::vector<double> ion_coef;
    const double ion_scale = ctx->prec == PHP_PREC_FP32 ? kIonScale32 : 1.0;
    ctx->rv_unit = 1.0 / ion_scale;
    for (int i = 0; i < d.num_materials; i++) {
        int rc = derive_material(ctx, i, d.materials[i], mats[i]);
        if (rc) return rc;
        if (mats[i].natom > 0) {
            const int N = mats[i].natom;
            ion_off[i] = (int)ion_coef.size();
            for (int q = 0; q < 9 * N; q++) ion_coef.push_back(d.materials[i].qezv[q] / ion_scale);
            for (int q = 0; q < 9 * N; q++) ion_coef.push_back(d.materials[i].qezm[q] * ion_scale);
            ion_coef.insert(ion_coef.end(), d.materials[i].dmm, d.materials[i].dmm + 9 * N * N);
        }
        ctx->mat_natom.push_back(mats[i].natom);
        ctx->mat_ade.push_back(mats[i].flags & kAde ? 1 : 0);
        ctx->mat_flags.push_back(mats[i].flags);
        ctx->mat_cs.push_back(mats[i].cs);
        ctx->mat_sn.push_back(mats[i].sn);
    }

    /* medium census, slots, device material map */
    const int nx = d.nx, ny = d.ny, nz = d.nz, nxp = ctx->nxp;
    std::vector<uint8_t> mat_dev((size_t)ctx->ncell_dev, 0);
    std::vector<int32_t> slot_dev;
    std::vector<int64_t> slot_cell;
    std::vector<int32_t> slot_n3;
    int n3max = 0;
    std::vector<int64_t> mat_cells(d.num_materials, 0);
    {
        /* the medium from file order (z fastest) into the device layout (x
         * fastest), with the pool slots of ADE and atom cells in device cell
         * order: z-plane ranges on host threads (a 1024 x 1024 x 512 medium
         * is 537 M strided reads), joined in plane order */
        struct Part {
            std::vector<int64_t> cell;
            std::vector<int32_t> n3;
            std::vector<int64_t> count;
            int n3max = 0;
            bool ade = false, atoms = false;
            int bad = 0, bad_id = 0, bi = 0, bj = 0, bk = 0;
        };
        const int nt = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)std::thread::hardware_concurrency(), 32,
                                                                    (int64_t)nz, (int64_t)nx * ny * nz / (1 << 20) + 1}));
        std::vector<Part> parts(nt);
        auto work = [&](int t) {
            Part& P = parts[t];
            P.count.assign(d.num_materials, 0);
            const int k0 = (int)((int64_t)nz * t / nt), k1 = (int)((int64_t)nz * (t + 1) / nt);
            for (int k = k0; k < k1; k++)
                for (int j = 0; j < ny; j++)
                    for (int i = 0; i < nx; i++) {
                        const int32_t id = d.medium[((size_t)i * ny + j) * nz + k];
                        if (id < 0 || id >= d.num_materials) {
                            P.bad = 1;
                            P.bad_id = id;
                            P.bi = i, P.bj = j, P.bk = k;
                            return;
                        }
                        const int64_t c = ((int64_t)k * ny + j) * nxp + i;
                        mat_dev[c] = (uint8_t)id;
                        P.count[id]++;
                        if (mats[id].flags & (kAde | kAtoms)) {
                            P.cell.push_back(c);
                            P.n3.push_back(3 * mats[id].natom);
                            P.n3max = std::max(P.n3max, 3 * mats[id].natom);
                            if (mats[id].flags & kAde) P.ade = true;
                            if (mats[id].flags & kAtoms) P.atoms = true;
                        }
                    }
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nt; t++) th.emplace_back(work, t);
        work(0);
        for (auto& x : th) x.join();
        for (const Part& P : parts) /* the first bad id in the reference's plane order */
            if (P.bad)
                return fail(ctx, PHP_ERR_INPUT, "medium id %d at (%d,%d,%d) outside the material table (0..%d)", P.bad_id,
                            P.bi, P.bj, P.bk, d.num_materials - 1);
        size_t total = 0;
        for (const Part& P : parts) total += P.cell.size();
        slot_cell.reserve(total);
        slot_n3.reserve(total);
        for (const Part& P : parts) {
            slot_cell.insert(slot_cell.end(), P.cell.begin(), P.cell.end());
            slot_n3.insert(slot_n3.end(), P.n3.begin(), P.n3.end());
            for (int m = 0; m < d.num_materials; m++) mat_cells[m] += P.count[m];
            n3max = std::max(n3max, P.n3max);
            ctx->any_ade = ctx->any_ade || P.ade;
            ctx->any_atoms = ctx->any_atoms || P.atoms;
        }
    }
    /* pad the pool to a multiple of 32 slots (16-byte rows for the tensor
     * maps of the ion pass); padding slots have no atoms */
    const int64_t nreal = (int64_t)slot_cell.size();
    while (nreal > 0 && slot_cell.size() % 32) {
        slot_cell.push_back(slot_cell.back());
        slot_n3.push_back(0);
    }
    ctx->nslot = (int64_t)slot_cell.size();
    ctx->n3max = n3max;
    {
        int best = -1;
        for (int i = 0; i < d.num_materials; i++)
            if ((mats[i].flags & kAtoms) && mats[i].natom <= 4 && mat_cells[i] > 0 && (best < 0 || mat_cells[i] > mat_cells[best]))
                best = i;
        if (best >= 0) {
            const int N = mats[best].natom, n3 = 3 * N;
            const php_material_desc& M = d.materials[best];
            ctx->ion_k.assign(kIonK, 0.0);
            for (int q = 0; q < 9 * N; q++) {
                ctx->ion_k[q] = M.qezv[q] / ion_scale;
                ctx->ion_k[kIonKM + q] = M.qezm[q] * ion_scale;
            }
            for (int q = 0; q < n3; q++)
                for (int p = 0; p < n3; p++) ctx->ion_k[kIonKD + q * kIonKQ + p] = M.dmm[(size_t)q * n3 + p];
            ctx->ion_k_off = ion_off[best];
            ctx->atom_id = best;
        }
    }
    const int namax = n3max / 3;
    ctx->namax_tpl = namax == 0 ? 0 : namax <= 2 ? 2 : namax <= 4 ? 4 : namax <= 8 ? 8 : namax <= 16 ? 16 : 64;
    if (namax > 64) return fail(ctx, PHP_ERR_UNSUPPORTED, "natom %d above the supported 64", namax);
    /* the two-atom update holds r, v in registers and indexes its pools with
     * 32-bit offsets (both precisions) */
    if (ctx->namax_tpl == 2 && (uint64_t)ctx->nslot * 6u >= ((uint64_t)1 << 32))
        return fail(ctx, PHP_ERR_UNSUPPORTED, "%lld atom / ADE cells exceed the 2^32-element pools of the two-atom update",
                    (long long)ctx->nslot);

    /* sources */
    if (d.num_sources > kMaxSources) return fail(ctx, PHP_ERR_UNSUPPORTED, "at most %d sources", kMaxSources);
    ctx->src.assign(d.sources, d.sources + d.num_sources);
    for (int s = 0; s < d.num_sources; s++) {
        const php_source_desc& S = d.sources[s];
        /* fdtd.c:3375-3393: sources outside the grid or with an unknown
         * component are skipped (their value still goes to source.txt) */
        if (S.x < 0 || S.x >= nx || S.y < 0 || S.y >= ny || S.z < 0 || S.z >= nz) continue;
        int comp = S.component == 'x' ? 0 : S.component == 'y' ? 1 : S.component == 'z' ? 2 : -1;
        if (comp < 0) continue;
        ctx->src_cell[ctx->nsrc_active] = ((int64_t)S.z * ny + S.y) * nxp + S.x;
        ctx->src_comp[ctx->nsrc_active] = comp;
        ctx->src_active_index.push_back(s);
        ctx->nsrc_active++;
    }

    /* z chunking: short marches while keeping at least ~4 waves of blocks on
     * 148 SMs.  Measured on 256^3 (the tip workload): FP64 fastest with 4
     * planes per block (E sweep 0.331 ms, H 0.210 ms; 8 planes 0.339 and
     * 0.214; 16 planes 0.364 and 0.225), FP32 with 8 (E 0.204 ms; 4 planes
     * 0.210, 16 planes 0.219) */
    {
        const int tiles = ((nx + kBlockX - 1) / kBlockX) * ((ny + kBlockY - 1) / kBlockY);
        int zc = std::min(ctx->prec == PHP_PREC_FP32 ? 8 : 4, nz);
        while (zc > 1 && (int64_t)tiles * ((nz + zc - 1) / zc) < 148 * 4 * 4) zc /= 2;
        ctx->zchunk = d.z_chunk > 0 ? d.z_chunk : zc;
    }
    /* 32-bit cell offsets inside the sweeps */
    if ((int64_t)ctx->plane * (nz + 2) >= ((int64_t)1 << 31))
        return fail(ctx, PHP_ERR_UNSUPPORTED, "grid of %lld padded cells exceeds the 2^31 cell limit of one domain",
                    (long long)ctx->plane * (nz + 2));

    /* allocations */
    const size_t rs = rsize(ctx->prec);
    const size_t field_bytes = (size_t)ctx->plane * (nz + 2) * rs;
    for (int q = 0; q < 9; q++) {
        void* p;
        int rc = dalloc(ctx, &p, field_bytes);
        if (rc) return rc;
        ctx->f[q] = (char*)p + (size_t)ctx->plane * rs; /* plane 0; plane -1 is the low halo */
    }
    const int L = ctx->L;
    const size_t xs = (size_t)nz * ny * 2 * L, ys = (size_t)nz * 2 * L * nxp, zs = (size_t)2 * L * ny * nxp;
    const size_t psz[12] = {xs, xs, ys, ys, zs, zs, xs, xs, ys, ys, zs, zs};
    for (int q = 0; q < 12; q++) {
        int rc = dalloc(ctx, &ctx->psi[q], psz[q] * rs);
        if (rc) return rc;
    }
    /* the one-launch step (he_sweep_tma) on a whole domain in the fast
     * modes, with PHP_FUSED=1 at create: it moves 12 % fewer bytes per step
     * than the two sweeps but measured slower on B200 (occupancy: E and H
     * with their halos in the stage ring, 80-125 registers), so the two
     * sweeps are the default */
    {
        const char* fv = getenv("PHP_FUSED");
        ctx->fused = ctx->prec != PHP_PREC_FP64_STRICT && ctx->z_off == 0 && ctx->nz_glob == nz && fv && !strcmp(fv, "1");
    }
    if (ctx->fused) {
        for (int q = 0; q < 9; q++) {
            if (q >= PHP_DX && q < PHP_DX + 3) {
                ctx->fo[q] = ctx->f[q];
                continue;
            }
            void* p;
            int rc = dalloc(ctx, &p, field_bytes);
            if (rc) return rc;
            ctx->fo[q] = (char*)p + (size_t)ctx->plane * rs;
        }
        for (int q = 0; q < 6; q++) {
            int rc = dalloc(ctx, &ctx->psio[q], psz[q] * rs);
            if (rc) return rc;
        }
    }
    int rc = dalloc(ctx, (void**)&ctx->mat, mat_dev.size());
    if (rc) return rc;
    if ((rc = upload(ctx, ctx->mat, mat_dev.data(), mat_dev.size()))) return rc;
    if (ctx->nslot > 0) {
        slot_dev.assign((size_t)ctx->ncell_dev, -1);
        for (int64_t s = 0; s < nreal; s++) slot_dev[slot_cell[s]] = (int32_t)s;
        rc = dalloc(ctx, (void**)&ctx->slot, slot_dev.size() * sizeof(int32_t));
        if (rc) return rc;
        if ((rc = upload(ctx, ctx->slot, slot_dev.data(), slot_dev.size() * sizeof(int32_t)))) return rc;
        rc = dalloc(ctx, (void**)&ctx->slot_cell, slot_cell.size() * sizeof(int64_t));
        if (rc) return rc;
        if ((rc = upload(ctx, ctx->slot_cell, slot_cell.data(), slot_cell.size() * sizeof(int64_t)))) return rc;
        rc = dalloc(ctx, (void**)&ctx->slot_n3, slot_n3.size() * sizeof(int32_t));
        if (rc) return rc;
        if ((rc = upload(ctx, ctx->slot_n3, slot_n3.data(), slot_n3.size() * sizeof(int32_t)))) return rc;
        std::vector<uint8_t> slot_mat(slot_cell.size(), 0);
        for (int64_t s = 0; s < nreal; s++) slot_mat[s] = mat_dev[slot_cell[s]];
        rc = dalloc(ctx, (void**)&ctx->slot_mat, slot_mat.size());
        if (rc) return rc;
        if ((rc = upload(ctx, ctx->slot_mat, slot_mat.data(), slot_mat.size()))) return rc;
        CK(cudaStreamSynchronize(ctx->stream)); /* the host vectors go out of scope */
    }
    if (ctx->any_ade) {
        if ((rc = dalloc(ctx, &ctx->P, 3 * (size_t)ctx->nslot * rs))) return rc;
        if ((rc = dalloc(ctx, &ctx->Po, 3 * (size_t)ctx->nslot * rs))) return rc;
    }
    if (ctx->any_atoms) {
        if ((rc = dalloc(ctx, &ctx->r, (size_t)n3max * ctx->nslot * rs))) return rc;
        if ((rc = dalloc(ctx, &ctx->v, (size_t)n3max * ctx->nslot * rs))) return rc;
    }
    if ((rc = setup_ion_pass(ctx, mats, ion_off, d))) return rc;

    AxisD axes[3];
    derive_axis(d, nx, d.dx, false, axes[0]);
    derive_axis(d, ny, d.dy, false, axes[1]);
    derive_axis(d, ctx->nz_glob, d.dz, true, axes[2]);
    if (ctx->nz_glob != nz) { /* a z slab: its planes of the global profile */
        AxisD& z = axes[2];
        auto cut = [&](auto& v) { v = std::vector<typename std::decay_t<decltype(v)>::value_type>(
                                      v.begin() + ctx->z_off, v.begin() + ctx->z_off + nz); };
        cut(z.slot); cut(z.kappa); cut(z.b); cut(z.c); cut(z.kh); cut(z.kd); cut(z.ch); cut(z.cd);
    }
    if (ctx->prec == PHP_PREC_FP32) rc = upload_tables<float>(ctx, mats, ion_off, ion_coef, axes);
    else rc = upload_tables<double>(ctx, mats, ion_off, ion_coef, axes);
    if (rc) return rc;

    /* plain blocks of the fused sweep: a 32 x 8 tile and z chunk of cells of
     * one plain isotropic material (id < kIsoMats), none in the CPML, none
     * on the domain's x/y edge, no source.  The sweep updates them without
     * the per-cell material, CPML and source handling; PHP_PLAIN=0 turns it
     * off (A/B timing and tests).  Blocks without a source of the one lossy
     * or anisotropic material (no ADE, no ions) that fills the most blocks
     * take its coefficients from the kernel parameters (kPlainTensor;
     * PHP_PLAIN_TENSOR=0 turns that class off), and so do blocks of the
     * few-atom material whose ions the sweep updates (kPlainAtoms;
     * PHP_PLAIN_ATOMS=0). */
    {
        const char* pv = getenv("PHP_PLAIN");
        const int gx = (nx + kBlockX - 1) / kBlockX, gy = (ny + kBlockY - 1) / kBlockY;
        const int gz = (nz + ctx->zchunk - 1) / ctx->zchunk;
        std::vector<uint8_t> pm((size_t)gx * gy * gz, 255), ph(pm.size(), 0), phf(pm.size(), 0);
        std::vector<char> src_tile(pm.size(), 0);
        for (int s = 0; s < ctx->nsrc_active; s++) {
            const int64_t sc = ctx->src_cell[s];
            const int sk = (int)(sc / ctx->plane), sj = (int)((sc % ctx->plane) / nxp), si = (int)(sc % nxp);
            src_tile[((size_t)(sk / ctx->zchunk) * gy + sj / kBlockY) * gx + si / kBlockX] = 1;
        }
        size_t nplain = 0, nplain_h = 0, nplain_hf = 0;
        const char* tv = getenv("PHP_PLAIN_TENSOR");
        const bool tns_off = tv && !strcmp(tv, "0");
        /* blocks of the few-atom material when the fused sweep updates its
         * ions (two or four atoms, no ion pass apart) */
        const char* av = getenv("PHP_PLAIN_ATOMS");
        const bool atoms_on = !(av && !strcmp(av, "0")) && ctx->atom_id >= 0 && !ctx->ion_split &&
                              (ctx->namax_tpl == 2 || ctx->namax_tpl == 4) &&
                              !(ctx->mat_flags[ctx->atom_id] & kAde) && ctx->atom_mc.size() > 0;
        std::vector<int16_t> uni(pm.size(), -1);
        std::vector<size_t> tns_count(ctx->mat_flags.size(), 0);
        for (int bz = 0; bz < gz && !(pv && !strcmp(pv, "0")) && ctx->prec != PHP_PREC_FP64_STRICT; bz++)
            for (int by = 0; by < gy; by++)
                for (int bx = 0; bx < gx; bx++) {
                    const int i0 = bx * kBlockX, j0 = by * kBlockY, k0 = bz * ctx->zchunk;
                    const int k1 = std::min(k0 + ctx->zchunk, nz);
                    const size_t b = ((size_t)bz * gy + by) * gx + bx;
                    const int i1 = std::min(i0 + kBlockX, nx), j1 = std::min(j0 + kBlockY, ny);
                    bool pml_free = true;
                    for (int i = i0; i < i1 && pml_free; i++) pml_free = axes[0].slot[i] < 0;
                    for (int j = j0; j < j1 && pml_free; j++) pml_free = axes[1].slot[j] < 0;
                    for (int k = k0; k < k1 && pml_free; k++) pml_free = axes[2].slot[k] < 0;
                    const bool full = i0 + kBlockX <= nx - 1 && j0 + kBlockY <= ny - 1; /* every cell has i < nx-1, j < ny-1 */
                    if (full && pml_free) { /* the H sweep needs no more */
                        ph[b] = 1;
                        nplain_h++;
                    }
                    /* the one-launch step computes H one cell further down in
                     * x, y and z: those cells must be outside the CPML too */
                    bool ring_free = pml_free;
                    if (ring_free && i0 >= 1) ring_free = axes[0].slot[i0 - 1] < 0;
                    if (ring_free && j0 >= 1) ring_free = axes[1].slot[j0 - 1] < 0;
                    if (ring_free && k0 >= 1) ring_free = axes[2].slot[k0 - 1] < 0;
                    if (full && ring_free) {
                        phf[b] = 1;
                        nplain_hf++;
                    }
                    if (src_tile[b]) continue;
                    const int id = mat_dev[((size_t)k0 * ny + j0) * nxp + i0];
                    bool ok = id < (int)ctx->mat_flags.size() && id < (int)ctx->iso_scale.size();
                    for (int k = k0; k < k1 && ok; k++)
                        for (int j = j0; j < j1 && ok; j++) {
                            const uint8_t* row = &mat_dev[((size_t)k * ny + j) * nxp];
                            for (int i = i0; i < i1 && ok; i++) ok = row[i] == id;
                        }
                    if (!ok) continue;
                    if (id < kIsoMats && ctx->iso_scale[id] != 0.0) {
                        /* one plain material: the stencil-only path, or with CPML or
                         * domain-edge cells the path that adds their CPML terms */
                        pm[b] = (uint8_t)((full && i0 >= 1 && j0 >= 1 && pml_free) ? id : kPlainCpml + id);
                        nplain++;
                    } else if (atoms_on && id == ctx->atom_id) {
                        pm[b] = (uint8_t)kPlainAtoms;
                        nplain++;
                        ctx->atom_blocks = true;
                    } else if (!(ctx->mat_flags[id] & (kAde | kAtoms)) && ctx->iso_scale[id] == 0.0 && !tns_off) {
                        uni[b] = (int16_t)id; /* a tensor block if id is the material chosen below */
                        tns_count[id]++;
                    }
                }
        /* the lossy or anisotropic material filling the most blocks */
        for (size_t id = 0; id < tns_count.size(); id++)
            if (tns_count[id] && (ctx->tns_id < 0 || tns_count[id] > tns_count[ctx->tns_id])) ctx->tns_id = (int)id;
        if (ctx->tns_id >= 0)
            for (size_t b = 0; b < pm.size(); b++)
                if (uni[b] == ctx->tns_id) {
                    pm[b] = (uint8_t)kPlainTensor;
                    nplain++;
                }
        for (size_t b = 0; b < pm.size(); b++) {
            const int c = pm[b] == 255 ? 4 : pm[b] == kPlainAtoms ? 3 : pm[b] == kPlainTensor ? 2
                        : pm[b] >= kPlainCpml ? 1 : 0;
            ctx->census[c]++;
            ctx->census[ph[b] ? 5 : 6]++;
        }
        ctx->census[7] = (int64_t)pm.size();
        if (nplain) {
            if ((rc = dalloc(ctx, (void**)&ctx->plain_blk, pm.size()))) return rc;
            if ((rc = upload(ctx, ctx->plain_blk, pm.data(), pm.size()))) return rc;
        }
        if (nplain_h) {
            if ((rc = dalloc(ctx, (void**)&ctx->plain_h, ph.size()))) return rc;
            if ((rc = upload(ctx, ctx->plain_h, ph.data(), ph.size()))) return rc;
        }
        if (nplain_hf && ctx->fused) {
            if ((rc = dalloc(ctx, (void**)&ctx->plain_hf, phf.size()))) return rc;
            if ((rc = upload(ctx, ctx->plain_hf, phf.data(), phf.size()))) return rc;
        }
        ctx->khp[0] = d.dt / (d.mu0 * d.dx * 1.0);
        ctx->khp[1] = d.dt / (d.mu0 * d.dy * 1.0);
        ctx->khp[2] = d.dt / (d.mu0 * d.dz * 1.0);
        ctx->kdp[0] = d.dt / (d.dx * 1.0);
        ctx->kdp[1] = d.dt / (d.dy * 1.0);
        ctx->kdp[2] = d.dt / (d.dz * 1.0);
    }

    if (const char* st = getenv("PHP_TEST_STALL_WAIT")) ctx->stall_test = !strcmp(st, "1");
    if (const char* dv = getenv("PHP_DFT_FOLD")) ctx->dft_fold = strcmp(dv, "0") != 0;
    if (const char* pv = getenv("PHP_PROBE_FOLD")) ctx->probe_fold = strcmp(pv, "0") != 0;
    /* sweep kernels: the TMA plane pipeline */
    if ((rc = dalloc(ctx, (void**)&ctx->err_flag, sizeof(int32_t)))) return rc;
    rc = ctx->prec == PHP_PREC_FP32 ? make_maps<float>(ctx) : make_maps<double>(ctx);
    if (!rc) rc = pick_step(ctx).prepare(ctx);
    if (rc) return rc;

    /* per-step inputs, scratch, staging */
    if ((rc = alloc_step_inputs(ctx, std::max(1, ctx->nsrc_active)))) return rc;
    const size_t maxplane = std::max({(size_t)nx * ny, (size_t)ny * nz, (size_t)nx * nz});
    ctx->scratch_bytes = std::max(maxplane * sizeof(double), (size_t)4096 * sizeof(DiagPartial));
    if ((rc = dalloc(ctx, &ctx->scratch, ctx->scratch_bytes))) return rc;
    ctx->host_stage_bytes = ctx->scratch_bytes;
    ctx->host_stage = pinned_get(ctx->host_stage_bytes);
    if (!ctx->host_stage) return fail(ctx, PHP_ERR_OOM, "page-locked host allocation failed");
    CK(cudaStreamSynchronize(ctx->stream));
    upload_release(ctx);
    /* hand over to the context's stream (everything above is complete) */
    cudaStream_t work = nullptr;
    CK(cudaStreamCreateWithFlags(&work, cudaStreamNonBlocking));
    ctx->stream = work;
    cudaStreamDestroy(ctx->setup);
    ctx->setup = nullptr;
    return PHP_OK;
}

/* Device bytes php_create will allocate for a description (the buffers of
 * create_impl, without DFT planes or the probe ring); no device needed. */
static int estimate_bytes(const php_desc& d, uint64_t* out)
{
    if (d.nx < 2 || d.ny < 2 || d.nz < 1 || d.num_materials < 1 || !d.materials || !d.medium || d.pml_thickness < 0 ||
        d.precision < 0 || d.precision > 2)
        return PHP_ERR_INPUT;
    const uint64_t rs = d.precision == PHP_PREC_FP32 ? 4 : 8;
    const uint64_t nxp = (uint64_t)(d.nx + 31) / 32 * 32, plane = nxp * d.ny, ncell = plane * d.nz;
    std::vector<int> n3(d.num_materials, 0);
    std::vector<char> slotted(d.num_materials, 0);
    bool any_ade = false, any_atoms = false;
    for (int m = 0; m < d.num_materials; m++) {
        n3[m] = 3 * std::max(0, (int)d.materials[m].natom);
        slotted[m] = d.materials[m].use_ade == 1 || d.materials[m].natom > 0;
    }
    uint64_t nslot = 0;
    int n3max = 0;
    const size_t V = (size_t)d.nx * d.ny * d.nz;
    for (size_t c = 0; c < V; c++) {
        const int id = d.medium[c];
        if (id < 0 || id >= d.num_materials) return PHP_ERR_INPUT;
        if (slotted[id]) {
            nslot++;
            n3max = std::max(n3max, n3[id]);
            if (d.materials[id].use_ade == 1) any_ade = true;
            if (d.materials[id].natom > 0) any_atoms = true;
        }
    }
    const uint64_t L = d.pml_thickness;
    uint64_t b = 9 * plane * (d.nz + 2) * rs;
    b += 4 * ((uint64_t)d.nz * d.ny * 2 * L + (uint64_t)d.nz * 2 * L * nxp + 2 * L * d.ny * nxp) * rs;
    const char* fv = getenv("PHP_FUSED");
    if (d.precision != PHP_PREC_FP64_STRICT && fv && !strcmp(fv, "1")) { /* second E, H and H CPML buffers */
        b += 6 * plane * (d.nz + 2) * rs;
        b += 2 * ((uint64_t)d.nz * d.ny * 2 * L + (uint64_t)d.nz * 2 * L * nxp + 2 * L * d.ny * nxp) * rs;
    }
    b += ncell; /* material ids */
    if (nslot) b += ncell * 4 + nslot * 12;
    if (any_ade) b += 6 * nslot * rs;
    if (any_atoms) b += 2 * (uint64_t)n3max * nslot * rs;
    if (n3max >= 24 && d.precision != PHP_PREC_FP64_STRICT) b += 3 * nslot * rs + 64 * 64 * 8; /* ion pass */
    b += 7 * (uint64_t)(d.nx + d.ny + d.nz) * (rs + 4);
    b += 2 * (uint64_t)kMaxChunk * (std::max(1, (int)d.num_sources) + 8) * 8;
    b += std::max((uint64_t)std::max({(uint64_t)d.nx * d.ny, (uint64_t)d.ny * d.nz, (uint64_t)d.nx * d.nz}) * 8,
                  (uint64_t)4096 * sizeof(DiagPartial));
    b += (uint64_t)d.num_materials * 512 + (1u << 20); /* tables, pool granularity */
    *out = b;
    return PHP_OK;
}

/* ---------------------------------------------------------------- stepping */

static int record_graph(php_ctx* ctx, int n, int b, cudaGraphExec_t* out);

/* graph of n steps reading per-step input buffer b; a new chunk length
 * records the graphs of both buffers at once, so that a repeated step
 * pattern instantiates nothing after its first pass */
static int graph_key(const php_ctx* ctx, int n, int b) { return 4 * n + 2 * ctx->level + b; }

static int ensure_graph(php_ctx* ctx, int n, int b, cudaGraphExec_t* out)
{
    auto it = ctx->graphs.find(graph_key(ctx, n, b));
    if (it != ctx->graphs.end()) {
        *out = it->second;
        return PHP_OK;
    }
    cudaGraphExec_t other;
    int rc = record_graph(ctx, n, b ^ 1, &other);
    if (rc) return rc;
    return record_graph(ctx, n, b, out);
}

/* The graph of n steps from the current level; each one-launch step of the
 * recording swaps the levels on the host as the step will on the device, so
 * the recording ends by restoring the level it started from. */
static int record_graph(php_ctx* ctx, int n, int b, cudaGraphExec_t* out)
{
    const int key = graph_key(ctx, n, b);
    const int level = ctx->level;
    ctx->step_in = ctx->step_in_dev[b];
    step_fn fn = pick_step(ctx).launch;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    for (int s = 0; s < n; s++) fn(ctx, s, launches);
    if (ctx->level != level) swap_levels(ctx);
    cudaError_t le = cudaGetLastError();
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
    if (le != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(ctx, PHP_ERR_CUDA, "kernel launch during capture failed: %s", cudaGetErrorString(le));
    }
    if (ce != cudaSuccess) return fail(ctx, PHP_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    cudaGraphExec_t ge = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return fail(ctx, PHP_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
    ctx->graphs[key] = ge;
    *out = ge;
    return PHP_OK;
}

static void drop_graphs(php_ctx* ctx)
{
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
}

static int relayout_step_inputs(php_ctx* ctx)
{
    int row = std::max(1, ctx->nsrc_active);
    for (auto& p : ctx->dft) {
        p.in_off = row;
        row += 1 + 2 * p.nfreq;
    }
    if (row == ctx->step_row) return PHP_OK;
    drop_graphs(ctx);
    return alloc_step_inputs(ctx, row);
}

template <typename R>
static void launch_gather_plane(php_ctx* ctx, int comp, int axis, int pos, bool f32)
{
    R* const* fp = reinterpret_cast<R* const*>(ctx->f);
    Fields<R> f{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], fp[8]};
    if (f32) gather_plane<R, float><<<296, 256, 0, ctx->stream>>>(f, comp, axis, pos, ctx->nx, ctx->ny, ctx->nz, ctx->nxp, (float*)ctx->scratch);
    else gather_plane<R, double><<<296, 256, 0, ctx->stream>>>(f, comp, axis, pos, ctx->nx, ctx->ny, ctx->nz, ctx->nxp, (double*)ctx->scratch);
}

/* Fills pinned buffer b with the per-step inputs (source values, DFT
 * sample flags and phasors) of steps t .. t+n-1 and copies it to device
 * buffer b on the stream. */
static int stage_step_inputs(php_ctx* ctx, int n, int b)
{
    const double dt = ctx->d.dt;
    /* the copy out of this pinned buffer two chunks ago must be done; the
     * chunk in between keeps the GPU busy meanwhile */
    CK(cudaEventSynchronize(ctx->staged[b]));
    double* h = ctx->step_in_host[b];
    for (int s = 0; s < n; s++) {
        const int t = ctx->t + s;
        double* row = h + (size_t)s * ctx->step_row;
        const double current_time = t * dt; /* fdtd.c:3117 */
        for (int q = 0; q < ctx->nsrc_active; q++)
            row[q] = source_value(&ctx->src[ctx->src_active_index[q]], current_time);
        for (auto& p : ctx->dft) {
            const bool take = t >= p.first && ((t - p.first) % p.interval) == 0;
            row[p.in_off] = take ? 1.0 : 0.0;
            for (int f = 0; f < p.nfreq; f++) {
                const double ph = -2.0 * M_PI * p.freq[f] * (t * dt);
                row[p.in_off + 1 + 2 * f] = take ? cos(ph) : 0.0;
                row[p.in_off + 2 + 2 * f] = take ? sin(ph) : 0.0;
            }
            if (take) p.nsamples++;
        }
    }
    /* the device buffer b was last read by the work of two chunks back,
     * which precedes this copy on the stream */
    CK(cudaMemcpyAsync(ctx->step_in_dev[b], h, (size_t)n * ctx->step_row * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaEventRecord(ctx->staged[b], ctx->stream));
    return PHP_OK;
}

/* ------------------------------------------------------------- public API */

/* frame gathers (php_frame_begin) */

static int64_t point_index(const php_ctx* ctx, const int32_t* p)
{
    return ((int64_t)p[2] * ctx->ny + p[1]) * ctx->nxp + p[0];
}

template <typename R>
static void launch_frame_gather(php_ctx* ctx, const DiagPartial* fin, int has_point, int64_t pc, int64_t cc)
{
    R* const* fp = reinterpret_cast<R* const*>(ctx->f);
    Fields<R> f{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], fp[8]};
    frame_gather<R><<<1, 256, 0, ctx->stream>>>(f, ctx->mat, ctx->slot, (const MatCoef<R>*)ctx->mc, (const R*)ctx->r,
                                                 (const R*)ctx->v, ctx->rv_unit, ctx->nslot, ctx->nx, ctx->ny, ctx->nz, ctx->nxp,
                                                 ctx->n3max, fin, has_point, pc, cc,
                                                 ctx->probe ? ctx->probe_count : nullptr, ctx->err_flag,
                                                 ctx->frame_head_dev);
}

extern "C" {

int php_create(const php_desc* desc, php_ctx** out)
{
    if (!desc || !out) return fail(nullptr, PHP_ERR_INPUT, "null argument");
    *out = nullptr;
    php_ctx* ctx = new (std::nothrow) php_ctx();
    if (!ctx) return fail(nullptr, PHP_ERR_OOM, "host allocation failed");
    int rc = create_impl(desc, ctx);
    if (rc) {
        g_create_error = ctx->err;
        ctx_free(ctx);
        return rc;
    }
    *out = ctx;
    return PHP_OK;
}

int php_create_slab(const php_desc* desc, int32_t z0, int32_t nz_local, php_ctx** out)
{
    if (!desc || !out) return fail(nullptr, PHP_ERR_INPUT, "null argument");
    *out = nullptr;
    if (!desc->medium || desc->nz < 1 || z0 < 0 || nz_local < 1 || z0 + nz_local > desc->nz)
        return fail(nullptr, PHP_ERR_INPUT, "slab [%d, %d) outside the grid of %d planes", z0, z0 + nz_local, desc->nz);
    if (desc->num_sources < 0 || (desc->num_sources > 0 && !desc->sources))
        return fail(nullptr, PHP_ERR_INPUT, "bad sources");
    /* the slab's medium and sources in local z */
    const size_t nx = desc->nx, ny = desc->ny, nzg = desc->nz;
    std::vector<int32_t> med(nx * ny * (size_t)nz_local);
    for (size_t i = 0; i < nx; i++)
        for (size_t j = 0; j < ny; j++)
            memcpy(&med[(i * ny + j) * nz_local], desc->medium + (i * ny + j) * nzg + z0, sizeof(int32_t) * nz_local);
    std::vector<php_source_desc> src(desc->sources, desc->sources + std::max(0, desc->num_sources));
    for (auto& x : src) x.z -= z0; /* sources outside the slab are skipped like those outside the grid */
    php_desc d = *desc;
    d.nz = nz_local;
    d.medium = med.data();
    d.sources = src.empty() ? nullptr : src.data();
    php_ctx* ctx = new (std::nothrow) php_ctx();
    if (!ctx) return fail(nullptr, PHP_ERR_OOM, "host allocation failed");
    ctx->z_off = z0;
    ctx->nz_glob = desc->nz;
    int rc = create_impl(&d, ctx);
    if (rc) {
        g_create_error = ctx->err;
        ctx_free(ctx);
        return rc;
    }
    ctx->d.medium = nullptr; /* the local copies go out of scope */
    ctx->d.sources = nullptr;
    *out = ctx;
    return PHP_OK;
}

int php_halo_planes(php_ctx* ctx, int32_t which, void** ptrs, uint64_t* plane_bytes)
{
    if (!ctx || !ptrs || which < 0 || which > 3) return PHP_ERR_INPUT;
    /* E plane 0 | E halo above | H top plane | H halo below */
    const int64_t plane_idx[4] = {0, ctx->nz, ctx->nz - 1, -1};
    const int first[4] = {PHP_EX, PHP_EX, PHP_HX, PHP_HX};
    const size_t rs = rsize(ctx->prec);
    for (int q = 0; q < 3; q++)
        ptrs[q] = (char*)ctx->f[first[which] + q] + plane_idx[which] * ctx->plane * (int64_t)rs;
    if (plane_bytes) *plane_bytes = (uint64_t)ctx->plane * rs;
    return PHP_OK;
}

int php_step_half(php_ctx* ctx, int32_t half)
{
    if (!ctx || (half != 0 && half != 1)) return PHP_ERR_INPUT;
    ctx->last_launches = 0;
    int launches = 0;
    const int b = ctx->chunk_no & 1;
    if (half == 1) {
        int rc = stage_step_inputs(ctx, 1, b);
        if (rc) return rc;
    }
    ctx->step_in = ctx->step_in_dev[b];
    ctx->step_part = half == 0 ? 1 : 6;
    pick_step(ctx).launch(ctx, 0, launches);
    ctx->step_part = 7;
    CK(cudaGetLastError());
    if (half == 1) {
        ctx->chunk_no++;
        ctx->t++;
    }
    ctx->last_launches = launches;
    return PHP_OK;
}

int php_step_part(php_ctx* ctx, int32_t part, void* stream)
{
    if (!ctx || part < 0 || part > 4) return PHP_ERR_INPUT;
    ctx->last_launches = 0;
    int launches = 0;
    const int b = ctx->chunk_no & 1;
    const int nchunk = (ctx->nz + ctx->zchunk - 1) / ctx->zchunk;
    cudaStream_t own = ctx->stream;
    if (stream) ctx->stream = static_cast<cudaStream_t>(stream);
    int rc = PHP_OK;
    if (part <= 1 && !ctx->part_staged) { /* the first H part stages the step's source values and DFT phasors */
        rc = stage_step_inputs(ctx, 1, b);
        ctx->part_staged = rc == PHP_OK;
    }
    if (rc == PHP_OK && part != 0 && !ctx->part_staged)
        rc = fail(ctx, PHP_ERR_STATE, "php_step_part %d before an H part (0 or 1) of the step", part);
    if (rc == PHP_OK) {
        ctx->step_in = ctx->step_in_dev[b];
        /* H: part 0 the top chunk, part 1 the others; E: part 2 the bottom
         * chunk, part 3 the others; part 4 the rest of the step */
        static const int kPartBits[5] = {1, 1, 2, 2, 4};
        ctx->step_part = kPartBits[part];
        ctx->zc_first = part == 0 ? nchunk - 1 : part == 3 ? 1 : 0;
        ctx->zc_count = part == 0 || part == 2 ? 1 : part == 4 ? 0 : nchunk - 1;
        pick_step(ctx).launch(ctx, 0, launches);
        ctx->step_part = 7;
        ctx->zc_first = 0;
        ctx->zc_count = -1;
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(ctx, PHP_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
    ctx->stream = own;
    if (rc == PHP_OK && part == 4) {
        ctx->part_staged = false;
        ctx->chunk_no++;
        ctx->t++;
    }
    ctx->last_launches = launches;
    return rc;
}

int php_destroy(php_ctx* ctx)
{
    ctx_free(ctx);
    return PHP_OK;
}

const char* php_last_error(const php_ctx* ctx)
{
    if (!ctx) return g_create_error.c_str();
    return ctx->err;
}

int php_step(php_ctx* ctx, int32_t nsteps)
{
    if (!ctx) return PHP_ERR_INPUT;
    if (nsteps < 0) return fail(ctx, PHP_ERR_INPUT, "negative step count");
    ctx->last_launches = 0;
    while (nsteps > 0) {
        const int n = std::min(nsteps, kMaxChunk);
        const int b = ctx->chunk_no & 1;
        /* the copy out of this pinned buffer two chunks ago must be done;
         * the chunk in between keeps the GPU busy meanwhile */
        int rc = stage_step_inputs(ctx, n, b);
        if (rc) return rc;
        cudaGraphExec_t g;
        rc = ensure_graph(ctx, n, b, &g);
        if (rc) return rc;
        CK(cudaGraphLaunch(g, ctx->stream));
        if (ctx->fused && (n & 1)) swap_levels(ctx); /* the level the graph leaves current */
        ctx->chunk_no++;
        if (ctx->profile) {
            CK(cudaStreamSynchronize(ctx->stream));
            for (int s = 0; s < n; s++)
                for (int kind = 0; kind < kProfKinds; kind++) {
                    if ((kind == 2 && (!ctx->probe || probe_folded(ctx))) || (kind == 3 && dft_launched(ctx) == 0) ||
                        (kind == 4 && !ctx->ion_split) ||
                        (kind <= 1 && ctx->fused) || (kind == 5 && !ctx->fused))
                        continue;
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, ctx->prof_ev[((size_t)s * kProfKinds + kind) * 2],
                                            ctx->prof_ev[((size_t)s * kProfKinds + kind) * 2 + 1]));
                    ctx->prof_ms[kind] += ms;
                    ctx->prof_n[kind] += kind == 3 ? (int64_t)dft_launched(ctx) : 1;
                }
        }
        ctx->last_launches += n * ((ctx->fused ? 1 : 2) + (ctx->ion_split ? 1 : 0) + (ctx->probe && !probe_folded(ctx) ? 1 : 0) +
                                   dft_launched(ctx));
        ctx->t += n;
        nsteps -= n;
    }
    return PHP_OK;
}

int php_prepare(php_ctx* ctx, int32_t nsteps)
{
    if (!ctx) return PHP_ERR_INPUT;
    if (nsteps < 0) return fail(ctx, PHP_ERR_INPUT, "negative step count");
    cudaGraphExec_t g;
    /* with the one-launch step, a chunk of odd length leaves the other level
     * current: the graphs of both levels */
    int rc = PHP_OK;
    for (int lv = 0; lv < (ctx->fused ? 2 : 1) && rc == PHP_OK; lv++) {
        if (lv) swap_levels(ctx);
        if (nsteps >= kMaxChunk) rc = ensure_graph(ctx, kMaxChunk, 0, &g);
        if (rc == PHP_OK && nsteps % kMaxChunk) rc = ensure_graph(ctx, nsteps % kMaxChunk, 0, &g);
        if (lv) swap_levels(ctx);
    }
    return rc;
}

int php_sync(php_ctx* ctx)
{
    if (!ctx) return PHP_ERR_INPUT;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    int32_t flag = 0;
    CK(cudaMemcpy(&flag, ctx->err_flag, sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag) return fail(ctx, PHP_ERR_TIMEOUT, "a sweep kernel gave up waiting for its plane loads");
    return PHP_OK;
}

int php_get_step(const php_ctx* ctx, int32_t* t)
{
    if (!ctx || !t) return PHP_ERR_INPUT;
    *t = ctx->t;
    return PHP_OK;
}

/* Gather geometry of a slice, with the reference's messages for bad ones. */
static int slice_geom(php_ctx* ctx, int32_t comp, char axis, int32_t position, int& ax, int& pos, size_t& n)
{
    if (comp < 0 || comp > 9) return fail(ctx, PHP_ERR_INPUT, "bad component %d", comp);
    if (axis == 'z') {
        if (position < 0 || position >= ctx->nz) return fail(ctx, PHP_ERR_INPUT, "Error: No process contains slice z=%d", position);
        ax = 0;
        pos = position + 1; /* fdtd.c:1029 with the halo already in the pointers (fdtd.c:274) */
        n = (size_t)ctx->nx * ctx->ny;
    } else if (axis == 'x') {
        if (position < 0 || position >= ctx->nx)
            return fail(ctx, PHP_ERR_INPUT, "Error: Invalid x slice position %d (range: 0-%d)", position, ctx->nx - 1);
        ax = 1;
        pos = position;
        n = (size_t)ctx->ny * ctx->nz;
    } else if (axis == 'y') {
        if (position < 0 || position >= ctx->ny)
            return fail(ctx, PHP_ERR_INPUT, "Error: Invalid y slice position %d (range: 0-%d)", position, ctx->ny - 1);
        ax = 2;
        pos = position;
        n = (size_t)ctx->nx * ctx->nz;
    } else {
        return fail(ctx, PHP_ERR_INPUT, "Error: Invalid slice axis '%c'. Must be 'x', 'y', or 'z'.", axis);
    }
    return PHP_OK;
}

static int read_slice_impl(php_ctx* ctx, int32_t comp, char axis, int32_t position, void* out, bool f32)
{
    if (!ctx || !out) return PHP_ERR_INPUT;
    int ax, pos;
    size_t n;
    int rc = slice_geom(ctx, comp, axis, position, ax, pos, n);
    if (rc) return rc;
    if (ctx->prec == PHP_PREC_FP32) launch_gather_plane<float>(ctx, comp, ax, pos, f32);
    else launch_gather_plane<double>(ctx, comp, ax, pos, f32);
    CK(cudaGetLastError());
    const size_t bytes = n * (f32 ? sizeof(float) : sizeof(double));
    CK(cudaMemcpyAsync(ctx->host_stage, ctx->scratch, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    memcpy(out, ctx->host_stage, bytes);
    return PHP_OK;
}

int php_read_slice(php_ctx* ctx, int32_t comp, char axis, int32_t position, float* out)
{
    return read_slice_impl(ctx, comp, axis, position, out, true);
}

int php_read_slice_f64(php_ctx* ctx, int32_t comp, char axis, int32_t position, double* out)
{
    return read_slice_impl(ctx, comp, axis, position, out, false);
}

int php_read_volume(php_ctx* ctx, int32_t comp, double* out)
{
    if (!ctx || !out) return PHP_ERR_INPUT;
    if (comp < 0 || comp > 8) return fail(ctx, PHP_ERR_INPUT, "bad component %d", comp);
    const size_t n = (size_t)ctx->nx * ctx->ny * ctx->nz;
    void* dbuf = nullptr;
    CK(cudaMallocAsync(&dbuf, n * sizeof(double), ctx->stream));
    if (ctx->prec == PHP_PREC_FP32)
        gather_volume<float><<<592, 256, 0, ctx->stream>>>((const float*)ctx->f[comp], ctx->nx, ctx->ny, ctx->nz, ctx->nxp, (double*)dbuf);
    else
        gather_volume<double><<<592, 256, 0, ctx->stream>>>((const double*)ctx->f[comp], ctx->nx, ctx->ny, ctx->nz, ctx->nxp, (double*)dbuf);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dbuf, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaFreeAsync(dbuf, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return PHP_OK;
}

int php_read_point(php_ctx* ctx, int32_t i, int32_t j, int32_t k, double* out9)
{
    if (!ctx || !out9) return PHP_ERR_INPUT;
    if (i < 0 || i >= ctx->nx || j < 0 || j >= ctx->ny || k < -1 || k > ctx->nz)
        return fail(ctx, PHP_ERR_INPUT, "point (%d,%d,%d) outside the grid", i, j, k);
    const int64_t c = ((int64_t)k * ctx->ny + j) * ctx->nxp + i;
    const size_t rs = rsize(ctx->prec);
    char* stage = (char*)ctx->host_stage;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < 9; q++)
        CK(cudaMemcpyAsync(stage + q * rs, (const char*)ctx->f[q] + c * (int64_t)rs, rs, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < 9; q++) out9[q] = rs == 4 ? (double)((float*)stage)[q] : ((double*)stage)[q];
    return PHP_OK;
}

int php_read_cell_state(php_ctx* ctx, int32_t i, int32_t j, int32_t k, int32_t* natom, double* r, double* v,
                        double* p_ade, double* p_ade_old)
{
    if (!ctx) return PHP_ERR_INPUT;
    if (i < 0 || i >= ctx->nx || j < 0 || j >= ctx->ny || k < 0 || k >= ctx->nz)
        return fail(ctx, PHP_ERR_INPUT, "cell (%d,%d,%d) outside the grid", i, j, k);
    const int64_t c = ((int64_t)k * ctx->ny + j) * ctx->nxp + i;
    CK(cudaStreamSynchronize(ctx->stream));
    uint8_t mid = 0;
    CK(cudaMemcpy(&mid, ctx->mat + c, 1, cudaMemcpyDeviceToHost));
    const int na = ctx->mat_natom[mid];
    if (natom) *natom = na;
    int32_t s = -1;
    if (ctx->slot) CK(cudaMemcpy(&s, ctx->slot + c, sizeof(int32_t), cudaMemcpyDeviceToHost));
    const size_t rs = rsize(ctx->prec);
    auto fetch = [&](void* base, int q, double* dst) -> int {
        char tmp[8];
        cudaError_t e = cudaMemcpy(tmp, (const char*)base + ((int64_t)q * ctx->nslot + s) * (int64_t)rs, rs, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail(ctx, PHP_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e));
        *dst = rs == 4 ? (double)*(float*)tmp : *(double*)tmp;
        return PHP_OK;
    };
    for (int q = 0; q < 3 * na; q++) {
        if (r) { int rc = fetch(ctx->r, q, &r[q]); if (rc) return rc; r[q] *= ctx->rv_unit; }
        if (v) { int rc = fetch(ctx->v, q, &v[q]); if (rc) return rc; v[q] *= ctx->rv_unit; }
    }
    if (ctx->mat_ade[mid] && s >= 0) {
        double pq[3], poq[3];
        for (int q = 0; q < 3; q++) {
            double p = 0.0, po = 0.0;
            int rc = fetch(ctx->P, q, &p);
            if (!rc) rc = fetch(ctx->Po, q, &po);
            if (rc) return rc;
            pq[q] = p;
            poq[q] = po;
        }
        if (ctx->prec == PHP_PREC_FP32) {
            /* FP32 keeps Q = D - P (lab frame) in the P pool and
             * J = P - P_old (crystal frame) in the P_old pool */
            double dl[3];
            for (int q = 0; q < 3; q++) {
                float dv = 0.f;
                CK(cudaMemcpy(&dv, (const float*)ctx->f[3 + q] + c, sizeof(float), cudaMemcpyDeviceToHost));
                dl[q] = (double)dv - pq[q];
            }
            const int fl = ctx->mat_flags[mid];
            const double cs = ctx->mat_cs[mid], sn = ctx->mat_sn[mid];
            if (fl & kRotZ) {
                const double u = dl[0] * cs - dl[1] * sn, w = dl[0] * sn + dl[1] * cs;
                dl[0] = u; dl[1] = w;
            } else if (fl & kRotX) {
                const double u = dl[1] * cs - dl[2] * sn, w = dl[1] * sn + dl[2] * cs;
                dl[1] = u; dl[2] = w;
            }
            for (int q = 0; q < 3; q++) {
                poq[q] = dl[q] - poq[q];
                pq[q] = dl[q];
            }
        }
        for (int q = 0; q < 3; q++) {
            if (p_ade) p_ade[q] = pq[q];
            if (p_ade_old) p_ade_old[q] = poq[q];
        }
    } else {
        for (int q = 0; q < 3; q++) {
            if (p_ade) p_ade[q] = 0.0;
            if (p_ade_old) p_ade_old[q] = 0.0;
        }
    }
    return PHP_OK;
}

/* Enqueues the two diagnostics passes; the result lands in *fin (scratch). */
static int enqueue_diag(php_ctx* ctx, DiagPartial** fin_out)
{
    const int blocks = 148 * 4;
    DiagPartial* part = (DiagPartial*)ctx->scratch;
    DiagPartial* fin = part + blocks;
    *fin_out = fin;
    if (ctx->prec == PHP_PREC_FP32) {
        float* const* fp = reinterpret_cast<float* const*>(ctx->f);
        Fields<float> f{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], fp[8]};
        diag_pass1<float><<<blocks, 256, 0, ctx->stream>>>(f, ctx->nx, ctx->ny, ctx->nz, ctx->nxp, (const float*)ctx->r,
                                                           ctx->rv_unit, ctx->any_atoms ? ctx->nslot : 0, ctx->slot_cell, ctx->slot_n3,
                                                           std::max(ctx->n3max, 1), part);
    } else {
        double* const* fp = reinterpret_cast<double* const*>(ctx->f);
        Fields<double> f{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], fp[8]};
        diag_pass1<double><<<blocks, 256, 0, ctx->stream>>>(f, ctx->nx, ctx->ny, ctx->nz, ctx->nxp, (const double*)ctx->r,
                                                            ctx->rv_unit, ctx->any_atoms ? ctx->nslot : 0, ctx->slot_cell, ctx->slot_n3,
                                                            std::max(ctx->n3max, 1), part);
    }
    diag_pass2<<<1, 256, 0, ctx->stream>>>(part, blocks, fin);
    CK(cudaGetLastError());
    return PHP_OK;
}

/* php_diag from the reduced partial (argmax in the reference's loop order) */
static void decode_diag(const php_ctx* ctx, const DiagPartial& h, php_diag* out)
{
    out->max_e = h.max_e;
    out->max_ex = h.max_ex;
    out->max_r = h.max_r;
    if (h.max_r > 0.0 && h.key_r != INT64_MAX) {
        const int64_t n3 = std::max(ctx->n3max, 1);
        int64_t cell = h.key_r / n3;
        const int q = (int)(h.key_r % n3);
        out->argmax_r[2] = (int)(cell % ctx->nz);
        cell /= ctx->nz;
        out->argmax_r[1] = (int)(cell % ctx->ny);
        out->argmax_r[0] = (int)(cell / ctx->ny);
        out->argmax_r[3] = q / 3;
        out->argmax_r[4] = q % 3;
    } else {
        for (int q = 0; q < 5; q++) out->argmax_r[q] = -1;
    }
}

int php_diagnostics(php_ctx* ctx, php_diag* out)
{
    if (!ctx || !out) return PHP_ERR_INPUT;
    DiagPartial* fin = nullptr;
    int rc = enqueue_diag(ctx, &fin);
    if (rc) return rc;
    DiagPartial h;
    CK(cudaMemcpyAsync(ctx->host_stage, fin, sizeof(DiagPartial), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    memcpy(&h, ctx->host_stage, sizeof(h));
    decode_diag(ctx, h, out);
    return PHP_OK;
}

int php_probe_set(php_ctx* ctx, int32_t i, int32_t j, int32_t k_field, int32_t k_atom)
{
    if (!ctx) return PHP_ERR_INPUT;
    if (i < 0 || i >= ctx->nx || j < 0 || j >= ctx->ny || k_field < -1 || k_field > ctx->nz || k_atom < 0 || k_atom >= ctx->nz)
        return fail(ctx, PHP_ERR_INPUT, "probe (%d,%d,%d/%d) outside the grid", i, j, k_field, k_atom);
    drop_graphs(ctx);
    ctx->probe_cf = ((int64_t)k_field * ctx->ny + j) * ctx->nxp + i;
    const int64_t ca = ((int64_t)k_atom * ctx->ny + j) * ctx->nxp + i;
    ctx->probe_ka = k_atom;
    uint8_t mid = 0;
    CK(cudaMemcpy(&mid, ctx->mat + ca, 1, cudaMemcpyDeviceToHost));
    ctx->probe_n3 = 3 * ctx->mat_natom[mid];
    int32_t s = -1;
    if (ctx->slot) CK(cudaMemcpy(&s, ctx->slot + ca, sizeof(int32_t), cudaMemcpyDeviceToHost));
    ctx->probe_slot = s;
    if (ctx->probe_n3 == 0) ctx->probe_slot = 0;
    if (!ctx->probe_rows) {
        int rc = dalloc(ctx, (void**)&ctx->probe_rows, (size_t)kProbeCap * (9 + 2 * std::max(ctx->n3max, 1)) * sizeof(double));
        if (rc) return rc;
        rc = dalloc(ctx, (void**)&ctx->probe_count, 2 * sizeof(int32_t));
        if (rc) return rc;
    }
    CK(cudaMemsetAsync(ctx->probe_count, 0, 2 * sizeof(int32_t), ctx->stream));
    ctx->probe = true;
    ctx->probe_t0 = ctx->t;
    return PHP_OK;
}

int php_probe_read(php_ctx* ctx, double* rows, int32_t max_rows, int32_t* nrows, int32_t* row_len)
{
    if (!ctx || !nrows) return PHP_ERR_INPUT;
    if (!ctx->probe) return fail(ctx, PHP_ERR_STATE, "no probe set");
    int32_t cnt[2];
    CK(cudaMemcpyAsync(cnt, ctx->probe_count, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const int rl = 9 + 2 * ctx->probe_n3;
    if (row_len) *row_len = rl;
    if (cnt[1]) return fail(ctx, PHP_ERR_STATE, "probe buffer overflowed (more than %d rows between reads)", kProbeCap);
    if (cnt[0] > max_rows) return fail(ctx, PHP_ERR_STATE, "%d probe rows pending, buffer holds %d", cnt[0], max_rows);
    if (cnt[0] > 0 && rows)
        CK(cudaMemcpyAsync(rows, ctx->probe_rows, (size_t)cnt[0] * rl * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->probe_count, 0, 2 * sizeof(int32_t), ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *nrows = cnt[0];
    ctx->probe_t0 = ctx->t;
    return PHP_OK;
}

/* ------------------------------------------------------------ output frames */

int php_frame_begin(php_ctx* ctx, const php_frame_req* req, int32_t* ticket)
{
    if (!ctx || !req || !ticket) return PHP_ERR_INPUT;
    int ax = 0, pos = 0;
    size_t slice_n = 0;
    if (req->slice_comp >= 0) {
        int rc = slice_geom(ctx, req->slice_comp, (char)req->slice_axis, req->slice_pos, ax, pos, slice_n);
        if (rc) return rc;
    }
    const bool has_point = req->point[0] >= 0;
    if (has_point && (req->point[0] >= ctx->nx || req->point[1] < 0 || req->point[1] >= ctx->ny || req->point[2] < -1 ||
                      req->point[2] > ctx->nz))
        return fail(ctx, PHP_ERR_INPUT, "point (%d,%d,%d) outside the grid", req->point[0], req->point[1], req->point[2]);
    const bool has_cell = req->cell[0] >= 0;
    if (has_cell && (req->cell[0] >= ctx->nx || req->cell[1] < 0 || req->cell[1] >= ctx->ny || req->cell[2] < 0 ||
                     req->cell[2] >= ctx->nz))
        return fail(ctx, PHP_ERR_INPUT, "cell (%d,%d,%d) outside the grid", req->cell[0], req->cell[1], req->cell[2]);
    if (req->probe && !ctx->probe) return fail(ctx, PHP_ERR_STATE, "no probe set");
    if (!ctx->frame_head_dev) {
        int rc = dalloc(ctx, (void**)&ctx->frame_head_dev, sizeof(FrameHead));
        if (rc) return rc;
    }
    const int32_t tk = ctx->frame_next;
    php_ctx::FrameSlot& F = ctx->frames[tk % PHP_FRAME_SLOTS];
    /* the oldest frame must have been released (bounded wait) */
    const auto t0 = std::chrono::steady_clock::now();
    while (F.state.load(std::memory_order_acquire) != 0) {
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(60))
            return fail(ctx, PHP_ERR_TIMEOUT, "frame %d was not released within 60 s", F.ticket);
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    if (!F.done) CK(cudaEventCreateWithFlags(&F.done, cudaEventDisableTiming));
    if (!F.head) F.head = (FrameHead*)pinned_get(sizeof(FrameHead));
    const size_t slice_cap = std::max({(size_t)ctx->nx * ctx->ny, (size_t)ctx->ny * ctx->nz, (size_t)ctx->nx * ctx->nz});
    if (!F.slice) F.slice = (float*)pinned_get(slice_cap * sizeof(float));
    const int32_t row_len = 9 + 2 * ctx->probe_n3;
    int64_t rows = 0;
    if (req->probe) {
        rows = std::min<int64_t>((int64_t)ctx->t - ctx->probe_t0, kProbeCap);
        const size_t need = (size_t)std::max<int64_t>(rows, 1) * row_len * sizeof(double);
        if (F.rows_bytes < need) {
            pinned_put(F.rows);
            F.rows = (double*)pinned_get(need);
            F.rows_bytes = F.rows ? need : 0;
        }
        if (!F.rows) return fail(ctx, PHP_ERR_OOM, "page-locked host allocation failed");
    }
    if (!F.head || !F.slice) return fail(ctx, PHP_ERR_OOM, "page-locked host allocation failed");

    DiagPartial* fin = nullptr;
    if (req->diag) {
        int rc = enqueue_diag(ctx, &fin);
        if (rc) return rc;
    }
    const int64_t pc = has_point ? point_index(ctx, req->point) : 0;
    const int64_t cc = has_cell ? point_index(ctx, req->cell) : -1;
    if (ctx->prec == PHP_PREC_FP32) launch_frame_gather<float>(ctx, fin, has_point, pc, cc);
    else launch_frame_gather<double>(ctx, fin, has_point, pc, cc);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(F.head, ctx->frame_head_dev, sizeof(FrameHead), cudaMemcpyDeviceToHost, ctx->stream));
    if (req->slice_comp >= 0) {
        if (ctx->prec == PHP_PREC_FP32) launch_gather_plane<float>(ctx, req->slice_comp, ax, pos, true);
        else launch_gather_plane<double>(ctx, req->slice_comp, ax, pos, true);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(F.slice, ctx->scratch, slice_n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (req->probe) {
        if (rows > 0)
            CK(cudaMemcpyAsync(F.rows, ctx->probe_rows, (size_t)rows * row_len * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
        CK(cudaMemsetAsync(ctx->probe_count, 0, 2 * sizeof(int32_t), ctx->stream));
        ctx->probe_t0 = ctx->t;
    }
    CK(cudaEventRecord(F.done, ctx->stream));
    F.ticket = tk;
    F.step = ctx->t;
    F.req = *req;
    F.rows_copied = rows;
    F.row_len = row_len;
    F.slice_len = req->slice_comp >= 0 ? (int64_t)slice_n : 0;
    F.state.store(1, std::memory_order_release);
    ctx->frame_next++;
    *ticket = tk;
    return PHP_OK;
}

int php_frame_wait(php_ctx* ctx, int32_t ticket, php_frame* out)
{
    if (!ctx || !out || ticket < 0) return PHP_ERR_INPUT;
    php_ctx::FrameSlot& F = ctx->frames[ticket % PHP_FRAME_SLOTS];
    if (F.state.load(std::memory_order_acquire) != 1 || F.ticket != ticket)
        return fail(ctx, PHP_ERR_STATE, "frame %d is not taken", ticket);
    CK(cudaEventSynchronize(F.done));
    const FrameHead& h = *F.head;
    if (h.err) return fail(ctx, PHP_ERR_TIMEOUT, "a sweep kernel gave up waiting for its plane loads");
    memset(out, 0, sizeof(*out));
    out->step = F.step;
    if (F.req.diag) {
        decode_diag(ctx, h.diag, &out->diag);
        out->diag_natom = h.diag_natom;
        memcpy(out->diag_point, h.diag_point, sizeof(out->diag_point));
        memcpy(out->diag_r, h.diag_r, sizeof(out->diag_r));
        memcpy(out->diag_v, h.diag_v, sizeof(out->diag_v));
    }
    if (F.req.point[0] >= 0) memcpy(out->point, h.point, sizeof(out->point));
    if (F.req.cell[0] >= 0) {
        out->cell_natom = h.cell_natom;
        memcpy(out->cell_r, h.cell_r, sizeof(out->cell_r));
        memcpy(out->cell_v, h.cell_v, sizeof(out->cell_v));
    }
    out->slice = F.slice_len ? F.slice : nullptr;
    out->slice_len = F.slice_len;
    out->row_len = F.row_len;
    if (F.req.probe) {
        if (h.probe_count[1])
            return fail(ctx, PHP_ERR_STATE, "probe buffer overflowed (more than %d rows between reads)", kProbeCap);
        out->nrows = (int32_t)std::min<int64_t>(h.probe_count[0], F.rows_copied);
        out->rows = F.rows;
    }
    return PHP_OK;
}

int php_frame_release(php_ctx* ctx, int32_t ticket)
{
    if (!ctx || ticket < 0) return PHP_ERR_INPUT;
    php_ctx::FrameSlot& F = ctx->frames[ticket % PHP_FRAME_SLOTS];
    if (F.ticket != ticket) return fail(ctx, PHP_ERR_STATE, "frame %d is not taken", ticket);
    F.state.store(0, std::memory_order_release);
    return PHP_OK;
}

int php_dft_add(php_ctx* ctx, int32_t comp, int32_t z_plane, int32_t first_step, int32_t sample_interval, int32_t nfreq,
                const double* freq_hz, int32_t cast_f32, int32_t* id)
{
    if (!ctx || !freq_hz || !id) return PHP_ERR_INPUT;
    if (comp < 0 || comp > 8) return fail(ctx, PHP_ERR_INPUT, "DFT component must be 0..8");
    if (z_plane < -1 || z_plane > ctx->nz) return fail(ctx, PHP_ERR_INPUT, "DFT plane %d outside -1..nz", z_plane);
    if (sample_interval < 1 || nfreq < 1 || nfreq > 64 || first_step < 0) return fail(ctx, PHP_ERR_INPUT, "bad DFT arguments");
    DftPlane p;
    p.comp = comp;
    p.z = z_plane;
    p.first = first_step;
    p.interval = sample_interval;
    p.nfreq = nfreq;
    p.cast_f32 = cast_f32 ? 1 : 0;
    p.freq.assign(freq_hz, freq_hz + nfreq);
    int rc = dalloc(ctx, (void**)&p.acc, (size_t)nfreq * ctx->nx * ctx->ny * 2 * sizeof(double));
    if (rc) return rc;
    ctx->dft.push_back(p);
    rc = relayout_step_inputs(ctx);
    if (rc) return rc;
    drop_graphs(ctx);
    *id = (int32_t)ctx->dft.size() - 1;
    return PHP_OK;
}

int php_dft_read(php_ctx* ctx, int32_t id, double* out, int32_t* nsamples)
{
    if (!ctx || !out) return PHP_ERR_INPUT;
    if (id < 0 || id >= (int)ctx->dft.size()) return fail(ctx, PHP_ERR_INPUT, "no DFT plane %d", id);
    const DftPlane& p = ctx->dft[id];
    /* the device keeps [nfreq][ny][nx][2] (x fastest for the samplers);
     * the caller gets [nfreq][nx][ny][2] */
    const size_t nx = ctx->nx, ny = ctx->ny;
    std::vector<double> dev((size_t)p.nfreq * nx * ny * 2);
    CK(cudaMemcpyAsync(dev.data(), p.acc, dev.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t f = 0; f < (size_t)p.nfreq; f++)
        for (size_t j = 0; j < ny; j++)
            for (size_t i = 0; i < nx; i++) {
                const double* src = &dev[((f * ny + j) * nx + i) * 2];
                double* dst = out + ((f * nx + i) * ny + j) * 2;
                dst[0] = src[0];
                dst[1] = src[1];
            }
    if (nsamples) *nsamples = p.nsamples;
    return PHP_OK;
}

int php_memory_bytes(const php_ctx* ctx, uint64_t* bytes)
{
    if (!ctx || !bytes) return PHP_ERR_INPUT;
    *bytes = ctx->bytes;
    return PHP_OK;
}

int php_estimate_bytes(const php_desc* desc, uint64_t* bytes)
{
    if (!desc || !bytes) return PHP_ERR_INPUT;
    return estimate_bytes(*desc, bytes);
}

int php_last_launch_count(const php_ctx* ctx, int32_t* launches)
{
    if (!ctx || !launches) return PHP_ERR_INPUT;
    *launches = ctx->last_launches;
    return PHP_OK;
}

int php_block_census(const php_ctx* ctx, int64_t* counts)
{
    if (!ctx || !counts) return PHP_ERR_INPUT;
    for (int q = 0; q < PHP_CENSUS_LEN; q++) counts[q] = ctx->census[q];
    return PHP_OK;
}

int php_stream(const php_ctx* ctx, void** stream)
{
    if (!ctx || !stream) return PHP_ERR_INPUT;
    *stream = (void*)ctx->stream;
    return PHP_OK;
}

int php_profile_enable(php_ctx* ctx, int32_t enable)
{
    if (!ctx) return PHP_ERR_INPUT;
    drop_graphs(ctx);
    if (enable && ctx->prof_ev.empty()) {
        ctx->prof_ev.resize((size_t)kMaxChunk * kProfKinds * 2);
        for (auto& e : ctx->prof_ev) CK(cudaEventCreate(&e));
    }
    ctx->profile = enable != 0;
    for (int q = 0; q < kProfKinds; q++) {
        ctx->prof_ms[q] = 0.0;
        ctx->prof_n[q] = 0;
    }
    return PHP_OK;
}

int php_profile_read(php_ctx* ctx, double* ms, int64_t* launches)
{
    if (!ctx) return PHP_ERR_INPUT;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < kProfKinds; q++) {
        if (ms) ms[q] = ctx->prof_ms[q];
        if (launches) launches[q] = ctx->prof_n[q];
    }
    return PHP_OK;
}

} // extern "C"
