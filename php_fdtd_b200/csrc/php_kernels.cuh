/*
 * php_kernels.cuh -- device types and the small kernels of the PhP_FDTD
 * time step on sm_100a (the sweeps are in php_sweeps*.cuh and
 * php_sweep_fused.cuh, the ion pass in php_ions.cuh).
 *
 * Device layout (one domain per GPU):
 *   field arrays  R[(nz + 2) planes][ny][nxp]   x fastest, nxp = nx rounded up
 *                 to 32 elements; plane -1 and plane nz are zero halos that
 *                 are never written, so the z stencils need no branch
 *                 (the reference's k = -1 / k = local_nz halo, fdtd.c:2006-2056,
 *                 holds zeros on a single rank).
 *   mat           uint8 [nz][ny][nxp] material id
 *   slot          int32 [nz][ny][nxp] index into the ADE / ion pools, -1 else
 *   psi x-slab    [nz][ny][2L]   (low side s = i, high side s = L + nx-1-i)
 *   psi y-slab    [nz][2L][nxp]
 *   psi z-slab    [2L][ny][nxp]
 *   pools         SoA: P[3][nslot], Po[3][nslot], r[3*natom_max][nslot], v[...]
 *
 * Arithmetic modes:
 *   Strict (double): every operation of the reference in its order, with
 *     IEEE division and no contraction (__dadd_rn & co. are never fused),
 *     on coefficient tables derived on the host exactly as fdtd.c derives
 *     them per cell.  Reproduces the reference bit for bit.
 *   Fast (double or float): the same update with host-folded coefficients
 *     (reciprocal spacings, psi stored pre-multiplied by dt, eps^-1 folded
 *     with the loss factors) and FMA.
 */
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace phpdev {

constexpr int kMaxSources = 16;
constexpr int kBlockX = 32;
constexpr int kBlockY = 8;

/* ----------------------------------------------------------------- tables */

/* Per material coefficients.  Strict and fast variants share the layout;
 * fields not used by a mode are zero. */
template <typename R>
struct MatCoef {
    int32_t flags;     /* kLossy | kAde | kRotZ | kRotX | kAtoms */
    int32_t natom;
    int32_t ion_off;   /* offset of QeZV (9N), QeZM (9N), DMM (9N^2) in ion_coef */
    int32_t pad;
    R eps_inv[9];      /* strict: Re eps^-1; fast: (1-lt)*lf/eps0 * Re eps^-1 */
    R eps_im[9];       /* strict: eps''; fast: c1*eps0*eps'' */
    R lf, lt;          /* loss factor and loss term (strict) */
    R cs, sn;          /* rotation cosine / sine */
    R gp_inv[9];       /* ADE (I + gamma dt/2)^-1 */
    R gm[9];           /* ADE (I - gamma dt/2) */
    R wp2[9];          /* strict: wp2; fast: eps0 dt^2 wp2 */
    R ade_scale;       /* fast: (1-lt)/(eps0*EPS_INF) */
    R pad2;
};

/* kIso (fast modes only): no rotation, loss, ADE or atoms and eps^-1 a
 * multiple of the identity, so E = eps_inv[0] * D. */
enum : int32_t { kLossy = 1, kAde = 2, kRotZ = 4, kRotX = 8, kAtoms = 16, kIso = 32 };

/* materials the fused sweep keeps in shared memory (ids above read global) */
constexpr int kSmemMats = 16;

/* Per-axis CPML tables, indexed by the cell index along the axis.  slot < 0
 * outside the PML.  Strict uses kappa, b, c (fdtd.c:3146-3151 evaluated on
 * the host); fast uses kh = dt/(mu0 d kappa), kd = dt/(d kappa),
 * ch = dt c/(mu0 d), cd = dt c/d. */
template <typename R>
struct AxisTab {
    const int32_t* slot;
    const R* kappa;
    const R* b;
    const R* c;
    const R* kh;
    const R* kd;
    const R* ch;
    const R* cd;
};

template <typename R>
struct Fields {
    R *ex, *ey, *ez, *dx, *dy, *dz, *hx, *hy, *hz;
};

template <typename R>
struct Psi {
    R *hxy, *hxz, *hyx, *hyz, *hzx, *hzy;
    R *dxy, *dxz, *dyx, *dyz, *dzx, *dzy;
};

/* The fused sweep's copy of one few-atom material's ion coefficients in the
 * kernel parameters (constant bank): QeZV [9 N], QeZM [9 N] and DMM with row
 * stride kIonKQ, for N <= 4 */
constexpr int kIonKQ = 12;
constexpr int kIonKM = 36;
constexpr int kIonKD = 72;
constexpr int kIonK = kIonKD + kIonKQ * kIonKQ;
constexpr int kIsoMats = 32;
/* running DFT planes the E sweep can sample itself (StepArgs::dft_*) */
constexpr int kDftFold = 4;
/* plain-block codes of the fused sweep: id, or kPlainCpml + id for blocks of
 * one plain material with CPML or domain-edge cells, kPlainTensor for blocks
 * of the tensor material in StepArgs::tns_*, kPlainAtoms for blocks of the
 * few-atom material in StepArgs::amc; 255 = general path */
constexpr int kPlainCpml = 64;
constexpr int kPlainTensor = 128;
constexpr int kPlainAtoms = 129;

template <typename R>
struct StepArgs {
    Fields<R> f;
    Psi<R> psi;
    AxisTab<R> tx, ty, tz;
    const uint8_t* mat;
    const int32_t* slot;
    const MatCoef<R>* mc;
    const R* ion_coef;
    R *P, *Po, *r, *v;         /* pools */
    const R* pr;               /* QeZV . r [3][nslot] when the ion pass runs apart (php_ions.cuh), else null */
    int32_t ion_k_off;         /* ion_coef offset of the material copied in ion_k, -1 for none */
    R ion_k[kIonK];
    /* E = iso[id] * D for the plain isotropic materials (kIso) among the
     * first kIsoMats ids, 0 for the others: the fused sweep's common case
     * without a load of the material record */
    R iso[kIsoMats];
    /* per block of the fused sweep: the material id of a plain block (one
     * plain isotropic material, no CPML or domain-edge cell, no source), 255
     * for the others; nullptr = no plain blocks.  kdp: dt / d of the axes
     * outside the CPML (kappa = 1) */
    const uint8_t* plain_blk;
    R kdp[3];
    /* per block of the H sweep: 1 for a tile and z chunk with no CPML cell
     * and every cell updated (i < nx-1, j < ny-1); kh of kappa = 1 */
    const uint8_t* plain_h;
    R khp[3];
    /* the material record of one lossy or anisotropic material without ADE
     * or ions (the one filling most blocks): blocks of that material alone
     * (kPlainTensor) read it as constant-bank operands */
    R tns_inv[9], tns_im[9], tns_cs, tns_sn;
    int32_t tns_flags;
    /* the material record of the few-atom material whose ion coefficients
     * are in ion_k, for blocks of that material alone (kPlainAtoms) */
    MatCoef<R> amc;
    int64_t nslot;
    int32_t nmat;
    int32_t nx, ny, nz, nxp, L, zchunk;
    int32_t zc0;                /* first z chunk of the launch (blockIdx.z + zc0 is the chunk) */
    int64_t plane;             /* nxp * ny */
    /* strict scalars */
    double dt, dxs, dys, dzs, mu0, eps0, c1, e0dt2;
    /* sources of this step */
    int32_t nsrc;
    int64_t src_cell[kMaxSources];
    int32_t src_comp[kMaxSources];
    const double* src_val;     /* nsrc values of this step */
    int32_t* err;              /* set to 1 by a block whose bounded wait gave up */
    int32_t stall_test;        /* failure-path test: the first H sweep block's wait gives up */
    /* the one-launch step (he_sweep_tma): f's E and H and psi's H arrays hold
     * the old time level, read only during the launch; the new E, H and H
     * CPML state go to these buffers (D, the D CPML state and the pools are
     * updated in place) */
    R *enew[3], *hnew[3];
    R* psin_h[6];              /* hxy hxz hyx hyz hzx hzy */
    /* per block of he_sweep_tma: 1 when the H part needs no CPML term and
     * updates every cell, over the tile, the cells one below it in x and y
     * and the plane below the z chunk */
    const uint8_t* plain_hf;
    /* running DFT planes of E or D components that the E sweep samples
     * after its z march (dft_fold), instead of a dft_sample launch: plane,
     * component (0-5), frequencies, the float32 cast flag, the offset of the
     * plane's flag and phasors in the step's input row (src_val), and the
     * accumulators [nfreq][ny][nx][2] */
    int32_t ndft;
    int32_t dft_z[kDftFold], dft_comp[kDftFold], dft_nfreq[kDftFold], dft_cast[kDftFold], dft_off[kDftFold];
    double* dft_acc[kDftFold];
    /* the monitor row the E sweep records after its z march (probe_fold),
     * instead of a probe_record_counted launch, when the field cell (i, j,
     * kf) and the atom cell of slot (its r and v updated by the sweep) lie in
     * one z chunk; probe_rows null: no such row */
    double* probe_rows;
    int32_t* probe_count;      /* [rows written, overflow flag] */
    int32_t probe_i, probe_j, probe_kf, probe_n3, probe_cap;
    int64_t probe_slot;
    double rv_unit;            /* physical r, v per stored unit */
};

/* ------------------------------------------------------------ arithmetic */

struct SOp {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

/* Read-only loads the compiler may not hoist out of the z loop: PML and
 * material coefficients are only needed inside rare branches, and keeping
 * them live across the loop would cost the registers that hold the next
 * plane in flight. */
__device__ __forceinline__ double ldg_nh(const double* p)
{
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ldg_nh(const float* p)
{
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int32_t ldg_nh(const int32_t* p)
{
    int32_t v;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

/* ========================================================== small kernels */

/* Gathers one plane of a component into out (float or double).
 * axis 0: z plane kk -> [i][j]; axis 1: x plane -> [j][k]; axis 2: y plane
 * -> [i][k].  comp 9 is |E|. */
template <typename R, typename O>
__global__ void gather_plane(const Fields<R> f, int comp, int axis, int pos, int nx, int ny, int nz,
                             int nxp, O* out)
{
    int A, B;
    if (axis == 0) { A = nx; B = ny; }
    else if (axis == 1) { A = ny; B = nz; }
    else { A = nx; B = nz; }
    const int64_t n = (int64_t)A * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int u = (int)(t / B), w = (int)(t % B);
        int i, j, k;
        if (axis == 0) { i = u; j = w; k = pos; }
        else if (axis == 1) { i = pos; j = u; k = w; }
        else { i = u; j = pos; k = w; }
        const int64_t c = ((int64_t)k * ny + j) * nxp + i;
        double val;
        switch (comp) {
        case 0: val = (double)f.ex[c]; break;
        case 1: val = (double)f.ey[c]; break;
        case 2: val = (double)f.ez[c]; break;
        case 3: val = (double)f.dx[c]; break;
        case 4: val = (double)f.dy[c]; break;
        case 5: val = (double)f.dz[c]; break;
        case 6: val = (double)f.hx[c]; break;
        case 7: val = (double)f.hy[c]; break;
        case 8: val = (double)f.hz[c]; break;
        default: {
            const double x = (double)f.ex[c], y = (double)f.ey[c], z = (double)f.ez[c];
            val = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
        }
        }
        out[t] = (O)val;
    }
}

/* Whole component to file order [i][j][k]. */
template <typename R>
__global__ void gather_volume(const R* src, int nx, int ny, int nz, int nxp, double* out)
{
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % nz);
        const int64_t ij = t / nz;
        const int j = (int)(ij % ny), i = (int)(ij / ny);
        out[t] = (double)src[((int64_t)k * ny + j) * nxp + i];
    }
}

/* Probe row appended at count[0]: 9 fields at cf, then r and v of pool slot
 * (3*natom each, times rv_unit: the stored state is scaled in FP32).
 * count[1] is raised instead of writing past cap. */
template <typename R>
__global__ void probe_record_counted(const Fields<R> f, int64_t cf, const R* r, const R* v, double rv_unit,
                                     int64_t nslot, int64_t slot, int n3, double* rows, int32_t* count, int cap,
                                     int row_len)
{
    __shared__ int row;
    if (threadIdx.x == 0) row = count[0];
    __syncthreads();
    if (row >= cap) {
        if (threadIdx.x == 0) count[1] = 1;
        return;
    }
    double* out = rows + (int64_t)row * row_len;
    const int t = threadIdx.x;
    if (t < 9) {
        const R* p[9] = {f.ex, f.ey, f.ez, f.dx, f.dy, f.dz, f.hx, f.hy, f.hz};
        out[t] = (double)p[t][cf];
    } else if (t < 9 + 2 * n3) {
        const int q = t - 9;
        out[t] = rv_unit * ((q < n3) ? (double)r[(int64_t)q * nslot + slot] : (double)v[(int64_t)(q - n3) * nslot + slot]);
    }
    __syncthreads();
    if (threadIdx.x == 0) count[0] = row + 1;
}

/* One cell's running-DFT samples: acc[f][t] += x * (cos, sin) for the
 * phasors of this step (ph[2f], ph[2f+1]), t = j * nx + i of n = nx * ny
 * (x fastest, so that a warp's cells along x update adjacent accumulators;
 * php_dft_read hands them out in [f][i][j] order). */
__device__ __forceinline__ void dft_accumulate(double x, const double* ph, int nfreq, double* acc, int64_t n, int64_t t)
{
    for (int f = 0; f < nfreq; ++f) {
        double* a = acc + ((int64_t)f * n + t) * 2;
        a[0] += x * ph[2 * f];
        a[1] += x * ph[2 * f + 1];
    }
}

/* Running DFT sample of one plane; skipped when flag == 0. */
template <typename R>
__global__ void dft_sample(const R* src, int64_t plane_off, int nx, int ny, int nxp, int nfreq,
                           int cast_f32, const double* step_in, int flag_off, int phasor_off,
                           double* acc)
{
    if (step_in[flag_off] == 0.0) return;
    const int64_t n = (int64_t)nx * ny;
    const double* ph = step_in + phasor_off;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / nx), i = (int)(t % nx);
        double x = (double)src[plane_off + (int64_t)j * nxp + i];
        if (cast_f32) x = (double)(float)x;
        dft_accumulate(x, ph, nfreq, acc, n, t);
    }
}

/* The same samples taken by the E sweep (StepArgs::dft_*): after a block's z
 * march over planes k0 .. k1-1, each of its threads reads back the E or D
 * values it stored at cell (i, j) of every registered plane in that range
 * that this step samples (e3: the E arrays the sweep wrote).  A cell's
 * accumulators belong to the one thread that updates the cell; no register
 * is held for this inside the march. */
template <typename R>
__device__ __forceinline__ void dft_fold(const StepArgs<R>& a, R* const* e3, int i, int j, int k0, int k1)
{
    if (i >= a.nx || j >= a.ny) return;
    for (int q = 0; q < a.ndft; ++q) {
        const int k = a.dft_z[q];
        if (k < k0 || k >= k1 || a.src_val[a.dft_off[q]] == 0.0) continue;
        const int cp = a.dft_comp[q];
        const R* src = cp == 0 ? e3[0] : cp == 1 ? e3[1] : cp == 2 ? e3[2] : cp == 3 ? a.f.dx : cp == 4 ? a.f.dy : a.f.dz;
        double x = (double)src[(k * a.ny + j) * a.nxp + i];
        if (a.dft_cast[q]) x = (double)(float)x;
        dft_accumulate(x, a.src_val + a.dft_off[q] + 1, a.dft_nfreq[q], a.dft_acc[q], (int64_t)a.nx * a.ny,
                       (int64_t)j * a.nx + i);
    }
}

/* The monitor row of probe_record_counted taken by the E sweep
 * (StepArgs::probe_*): the thread of column (i, j), after its z march over
 * planes k0 .. k1-1 that hold the field cell, reads back the E and D it
 * stored there, H (e3, h3: the arrays the step's sweeps wrote), and the r
 * and v it stored for the atom cell of the same column and chunk.  It is the
 * one thread of the launch that touches the row counter. */
template <typename R>
__device__ __forceinline__ void probe_fold(const StepArgs<R>& a, R* const* e3, R* const* h3, int i, int j, int k0, int k1)
{
    if (!a.probe_rows || i != a.probe_i || j != a.probe_j || a.probe_kf < k0 || a.probe_kf >= k1) return;
    const int row = a.probe_count[0];
    if (row >= a.probe_cap) {
        a.probe_count[1] = 1;
        return;
    }
    const int64_t c = ((int64_t)a.probe_kf * a.ny + j) * a.nxp + i;
    double* out = a.probe_rows + (int64_t)row * (9 + 2 * a.probe_n3);
    out[0] = (double)e3[0][c];
    out[1] = (double)e3[1][c];
    out[2] = (double)e3[2][c];
    out[3] = (double)a.f.dx[c];
    out[4] = (double)a.f.dy[c];
    out[5] = (double)a.f.dz[c];
    out[6] = (double)h3[0][c];
    out[7] = (double)h3[1][c];
    out[8] = (double)h3[2][c];
    for (int q = 0; q < a.probe_n3; ++q) {
        out[9 + q] = a.rv_unit * (double)a.r[(int64_t)q * a.nslot + a.probe_slot];
        out[9 + a.probe_n3 + q] = a.rv_unit * (double)a.v[(int64_t)q * a.nslot + a.probe_slot];
    }
    a.probe_count[0] = row + 1;
}

/* ------------------------------------------------------------ diagnostics */

struct DiagPartial {
    double max_e, max_ex, max_r;
    int64_t key_r; /* reference loop-order key of the first max_r */
};

/* The reference keeps the first strictly larger |r| starting from 0
 * (fdtd.c:3567-3586): ties go to the smaller loop-order key and zeros never
 * set an argmax. */
__device__ __forceinline__ void diag_merge(DiagPartial& a, const DiagPartial& b)
{
    a.max_e = fmax(a.max_e, b.max_e);
    a.max_ex = fmax(a.max_ex, b.max_ex);
    if (b.max_r > a.max_r || (b.max_r == a.max_r && b.max_r > 0.0 && b.key_r < a.key_r)) {
        a.max_r = b.max_r;
        a.key_r = b.key_r;
    }
}

/* Pass 1 over cells (|E|, |Ex|) and pool slots (|r|, times rv_unit); one
 * partial per block into scratch.  slot_cell maps a pool slot to its device
 * cell index. */
template <typename R>
__global__ void __launch_bounds__(256) diag_pass1(const Fields<R> f, int nx, int ny, int nz, int nxp,
                                                  const R* r, double rv_unit, int64_t nslot, const int64_t* slot_cell,
                                                  const int32_t* slot_n3, int n3max, DiagPartial* scratch)
{
    DiagPartial acc{0.0, 0.0, 0.0, INT64_MAX};
    const int64_t ncell = (int64_t)nx * ny * nz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ncell; t += stride) {
        const int i = (int)(t % nx);
        const int64_t jk = t / nx;
        const int64_t c = jk * nxp + i;
        const double x = (double)f.ex[c], y = (double)f.ey[c], z = (double)f.ez[c];
        const double e = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
        acc.max_e = fmax(acc.max_e, e);
        acc.max_ex = fmax(acc.max_ex, fabs(x));
    }
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nslot; s += stride) {
        const int n3 = slot_n3[s];
        if (!n3) continue;
        const int64_t c = slot_cell[s];
        const int i = (int)(c % nxp);
        const int64_t jk = c / nxp;
        const int j = (int)(jk % ny), k = (int)(jk / ny);
        const int64_t base = (((int64_t)i * ny + j) * nz + k) * (int64_t)n3max;
        for (int q = 0; q < n3; ++q) {
            const double rv = rv_unit * fabs((double)r[(int64_t)q * nslot + s]);
            if (rv > acc.max_r || (rv == acc.max_r && rv > 0.0 && base + q < acc.key_r)) {
                acc.max_r = rv;
                acc.key_r = base + q;
            }
        }
    }
    __shared__ DiagPartial sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) diag_merge(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) scratch[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(256) diag_pass2(const DiagPartial* scratch, int n, DiagPartial* out)
{
    DiagPartial acc{0.0, 0.0, 0.0, INT64_MAX};
    for (int t = threadIdx.x; t < n; t += blockDim.x) diag_merge(acc, scratch[t]);
    __shared__ DiagPartial sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) diag_merge(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

/* ---------------------------------------------------------- output frames */

constexpr int kFrameMaxN3 = 192; /* 3 N for N <= 64 atoms */

/* The small part of an output frame (php_frame_begin), gathered on the
 * device and copied to page-locked host memory in one piece. */
struct FrameHead {
    DiagPartial diag;                                       /* diag_pass2 result */
    double diag_point[9];                                   /* fields at the max |r| cell */
    double diag_r[kFrameMaxN3], diag_v[kFrameMaxN3];        /* r, v there */
    double point[9];                                        /* fields at the requested point */
    double cell_r[kFrameMaxN3], cell_v[kFrameMaxN3];        /* r, v of the requested cell */
    int32_t diag_natom, cell_natom;
    int32_t probe_count[2];                                 /* rows recorded, overflow flag */
    int32_t err;                                            /* a sweep's bounded wait gave up */
    int32_t pad_;
};

/* Field values (Ex Ey Ez Dx Dy Dz Hx Hy Hz) at device cell c, and r, v of the
 * atom cell c (none when its material has no atoms). */
template <typename R>
__device__ __forceinline__ void frame_cell(const Fields<R>& f, const uint8_t* mat, const int32_t* slot,
                                           const MatCoef<R>* mc, const R* r, const R* v, double rv_unit,
                                           int64_t nslot, int64_t cf, int64_t ca, double* point9, double* rr,
                                           double* vv, int32_t* natom)
{
    const int t = threadIdx.x;
    if (point9 && t < 9) {
        const R* p[9] = {f.ex, f.ey, f.ez, f.dx, f.dy, f.dz, f.hx, f.hy, f.hz};
        point9[t] = (double)p[t][cf];
    }
    if (ca < 0) return;
    const int na = mc[mat[ca]].natom;
    const int64_t s = (na > 0 && slot) ? slot[ca] : -1;
    if (t == 0) *natom = s >= 0 ? na : 0;
    if (s < 0) return;
    for (int q = t; q < 3 * na && q < kFrameMaxN3; q += blockDim.x) {
        rr[q] = rv_unit * (double)r[(int64_t)q * nslot + s];
        vv[q] = rv_unit * (double)v[(int64_t)q * nslot + s];
    }
}

/* One block.  fin: the diagnostics of this frame (nullptr: none); the
 * point's device index (k may be -1 or nz, the halo planes; has_point 0:
 * none) and the cell's (-1: none); probe_count: the probe row counter
 * (nullptr: no probe).  Thread 0 writes every natom field. */
template <typename R>
__global__ void frame_gather(const Fields<R> f, const uint8_t* mat, const int32_t* slot, const MatCoef<R>* mc,
                             const R* r, const R* v, double rv_unit, int64_t nslot, int nx, int ny, int nz, int nxp,
                             int n3max,
                             const DiagPartial* fin, int has_point, int64_t point_c, int64_t cell_c,
                             const int32_t* probe_count,
                             const int32_t* err, FrameHead* head)
{
    const int t = threadIdx.x;
    if (fin) {
        const DiagPartial d = *fin;
        if (t == 0) {
            head->diag = d;
            head->diag_natom = 0;
        }
        if (d.max_r > 0.0 && d.key_r != INT64_MAX) {
            /* reference loop order (i, j, k, coordinate), as php_diagnostics decodes it */
            const int64_t n3 = n3max > 1 ? n3max : 1;
            int64_t cell = d.key_r / n3;
            const int k = (int)(cell % nz);
            cell /= nz;
            const int j = (int)(cell % ny);
            const int i = (int)(cell / ny);
            const int64_t c = ((int64_t)k * ny + j) * nxp + i;
            frame_cell(f, mat, slot, mc, r, v, rv_unit, nslot, c, c, head->diag_point, head->diag_r, head->diag_v,
                       &head->diag_natom);
        }
    }
    if (has_point)
        frame_cell<R>(f, mat, slot, mc, r, v, rv_unit, nslot, point_c, -1, head->point, nullptr, nullptr, nullptr);
    if (cell_c >= 0) {
        if (t == 0) head->cell_natom = 0;
        frame_cell<R>(f, mat, slot, mc, r, v, rv_unit, nslot, cell_c, cell_c, nullptr, head->cell_r, head->cell_v,
                      &head->cell_natom);
    }
    if (t == 0) {
        head->probe_count[0] = probe_count ? probe_count[0] : 0;
        head->probe_count[1] = probe_count ? probe_count[1] : 0;
        head->err = *err;
    }
}

} // namespace phpdev

#include "php_sweeps.cuh"
#include "php_sweeps_tma.cuh"
#include "php_sweep_fused.cuh"
#include "php_ions.cuh"
