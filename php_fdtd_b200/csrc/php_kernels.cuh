/*
 * php_kernels.cuh -- sm_100a kernels of the PhP_FDTD time step.
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
 * Two kernels per step:
 *   h_sweep   H += dt (curl E / kappa + psi_H)          fdtd.c:3123-3231
 *   e_sweep   D += dt (curl H / kappa + psi_D) - eps''  fdtd.c:3238-3356
 *             + sources                                 fdtd.c:3363-3400
 *             D -> E (rotation, eps^-1 or ADE, loss)    fdtd.c:3404-3503
 *             ion equations of motion                   fdtd.c:3505-3528
 * Each thread owns one (i, j) column of a z chunk and marches up in k,
 * carrying the k+1 (H sweep) or k-1 (E sweep) plane in registers; in-plane
 * neighbours come through L1.
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

enum : int32_t { kLossy = 1, kAde = 2, kRotZ = 4, kRotX = 8, kAtoms = 16 };

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
    int64_t nslot;
    int32_t nx, ny, nz, nxp, L, zchunk;
    int64_t plane;             /* nxp * ny */
    /* strict scalars */
    double dt, dxs, dys, dzs, mu0, eps0, c1, e0dt2;
    /* sources of this step */
    int32_t nsrc;
    int64_t src_cell[kMaxSources];
    int32_t src_comp[kMaxSources];
    const double* src_val;     /* nsrc values of this step */
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

/* ================================================================ H sweep */

/* fdtd.c:3123-3231.  Cells i < nx-1, j < ny-1, all k. */
template <typename R, bool STRICT>
__global__ void __launch_bounds__(256) h_sweep(const StepArgs<R> a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= a.nx - 1 || j >= a.ny - 1) return;
    const int k0 = blockIdx.z * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return;

    const int L = a.L;
    const int sx = ldg(a.tx.slot + i);
    const int sy = ldg(a.ty.slot + j);
    const int64_t P = a.plane;
    int64_t c = ((int64_t)k0 * a.ny + j) * a.nxp + i;

    const R* __restrict__ ex = a.f.ex;
    const R* __restrict__ ey = a.f.ey;
    const R* __restrict__ ez = a.f.ez;
    R ex0 = ldg(ex + c), ey0 = ldg(ey + c);

    if constexpr (STRICT) {
        const double kx = ldg(a.tx.kappa + i), bx = ldg(a.tx.b + i), cx = ldg(a.tx.c + i);
        const double ky = ldg(a.ty.kappa + j), by = ldg(a.ty.b + j), cy = ldg(a.ty.c + j);
        const double dt = a.dt, mu0 = a.mu0;
        for (int k = k0; k < k1; ++k, c += P) {
            const double ex1 = ldg(ex + c + P), ey1 = ldg(ey + c + P);
            const double ez0 = ldg(ez + c);
            const double ezi = ldg(ez + c + 1), eyi = ldg(ey + c + 1);
            const double ezj = ldg(ez + c + a.nxp), exj = ldg(ex + c + a.nxp);
            /* fdtd.c:3132-3137 */
            const double dEy_dz = SOp::div(SOp::sub(ey1, ey0), a.dzs);
            const double dEz_dy = SOp::div(SOp::sub(ezj, ez0), a.dys);
            const double dEz_dx = SOp::div(SOp::sub(ezi, ez0), a.dxs);
            const double dEx_dz = SOp::div(SOp::sub(ex1, ex0), a.dzs);
            const double dEx_dy = SOp::div(SOp::sub(exj, ex0), a.dys);
            const double dEy_dx = SOp::div(SOp::sub(eyi, ey0), a.dxs);
            double pxy = 0.0, pxz = 0.0, pyx = 0.0, pyz = 0.0, pzx = 0.0, pzy = 0.0;
            double kappa_x = 1.0, kappa_y = 1.0, kappa_z = 1.0;
            if (sx >= 0) { /* fdtd.c:3143-3170 */
                kappa_x = kx;
                const int64_t q = ((int64_t)k * a.ny + j) * (2 * L) + sx;
                pxy = a.psi.hxy[q];
                pxz = a.psi.hxz[q];
                a.psi.hxy[q] = SOp::add(SOp::mul(bx, pxy), SOp::mul(cx, SOp::div(dEz_dx, mu0)));
                a.psi.hxz[q] = SOp::add(SOp::mul(bx, pxz), SOp::mul(cx, SOp::div(-dEy_dx, mu0)));
            }
            if (sy >= 0) { /* fdtd.c:3173-3200 */
                kappa_y = ky;
                const int64_t q = ((int64_t)k * (2 * L) + sy) * a.nxp + i;
                pyx = a.psi.hyx[q];
                pyz = a.psi.hyz[q];
                a.psi.hyx[q] = SOp::add(SOp::mul(by, pyx), SOp::mul(cy, SOp::div(-dEz_dy, mu0)));
                a.psi.hyz[q] = SOp::add(SOp::mul(by, pyz), SOp::mul(cy, SOp::div(dEx_dy, mu0)));
            }
            const int sz = ldg(a.tz.slot + k);
            double bz = 1.0, cz = 0.0;
            int64_t qz = 0;
            if (sz >= 0) { /* fdtd.c:3203-3219 */
                kappa_z = ldg(a.tz.kappa + k);
                bz = ldg(a.tz.b + k);
                cz = ldg(a.tz.c + k);
                qz = ((int64_t)sz * a.ny + j) * a.nxp + i;
                pzx = a.psi.hzx[qz];
                pzy = a.psi.hzy[qz];
            }
            /* fdtd.c:3222-3224 */
            double sx_ = SOp::add(SOp::add(SOp::add(SOp::div(SOp::div(-dEz_dy, mu0), kappa_y), pyx),
                                           SOp::div(SOp::div(dEy_dz, mu0), kappa_z)), pzx);
            double sy_ = SOp::add(SOp::add(SOp::add(SOp::div(SOp::div(dEz_dx, mu0), kappa_x), pxy),
                                           SOp::div(SOp::div(-dEx_dz, mu0), kappa_z)), pzy);
            double sz_ = SOp::add(SOp::add(SOp::add(SOp::div(SOp::div(-dEy_dx, mu0), kappa_x), pxz),
                                           SOp::div(SOp::div(dEx_dy, mu0), kappa_y)), pyz);
            a.f.hx[c] = SOp::add(a.f.hx[c], SOp::mul(dt, sx_));
            a.f.hy[c] = SOp::add(a.f.hy[c], SOp::mul(dt, sy_));
            a.f.hz[c] = SOp::add(a.f.hz[c], SOp::mul(dt, sz_));
            if (sz >= 0) { /* fdtd.c:3225-3228 */
                a.psi.hzx[qz] = SOp::add(SOp::mul(bz, pzx), SOp::mul(cz, SOp::div(dEy_dz, mu0)));
                a.psi.hzy[qz] = SOp::add(SOp::mul(bz, pzy), SOp::mul(cz, SOp::div(-dEx_dz, mu0)));
            }
            ex0 = ex1;
            ey0 = ey1;
        }
    } else {
        const R khx = ldg(a.tx.kh + i), khy = ldg(a.ty.kh + j);
        const R bx = ldg(a.tx.b + i), chx = ldg(a.tx.ch + i);
        const R by = ldg(a.ty.b + j), chy = ldg(a.ty.ch + j);
        for (int k = k0; k < k1; ++k, c += P) {
            const R ex1 = ldg(ex + c + P), ey1 = ldg(ey + c + P);
            const R ez0 = ldg(ez + c);
            const R ezi = ldg(ez + c + 1), eyi = ldg(ey + c + 1);
            const R ezj = ldg(ez + c + a.nxp), exj = ldg(ex + c + a.nxp);
            const R dEyz = ey1 - ey0, dEzy = ezj - ez0, dEzx = ezi - ez0;
            const R dExz = ex1 - ex0, dExy = exj - ex0, dEyx = eyi - ey0;
            const R khz = ldg(a.tz.kh + k);
            R ux = -khy * dEzy + khz * dEyz;
            R uy = khx * dEzx - khz * dExz;
            R uz = -khx * dEyx + khy * dExy;
            if (sx >= 0) {
                const int64_t q = ((int64_t)k * a.ny + j) * (2 * L) + sx;
                const R pxy = a.psi.hxy[q], pxz = a.psi.hxz[q];
                uy += pxy;
                uz += pxz;
                a.psi.hxy[q] = bx * pxy + chx * dEzx;
                a.psi.hxz[q] = bx * pxz - chx * dEyx;
            }
            if (sy >= 0) {
                const int64_t q = ((int64_t)k * (2 * L) + sy) * a.nxp + i;
                const R pyx = a.psi.hyx[q], pyz = a.psi.hyz[q];
                ux += pyx;
                uz += pyz;
                a.psi.hyx[q] = by * pyx - chy * dEzy;
                a.psi.hyz[q] = by * pyz + chy * dExy;
            }
            const int sz = ldg(a.tz.slot + k);
            if (sz >= 0) {
                const R bz = ldg(a.tz.b + k), chz = ldg(a.tz.ch + k);
                const int64_t q = ((int64_t)sz * a.ny + j) * a.nxp + i;
                const R pzx = a.psi.hzx[q], pzy = a.psi.hzy[q];
                ux += pzx;
                uy += pzy;
                a.psi.hzx[q] = bz * pzx + chz * dEyz;
                a.psi.hzy[q] = bz * pzy - chz * dExz;
            }
            a.f.hx[c] += ux;
            a.f.hy[c] += uy;
            a.f.hz[c] += uz;
            ex0 = ex1;
            ey0 = ey1;
        }
    }
}

/* ================================================================ E sweep */

/* Rotation to the crystal frame and back (fdtd.c:3429-3452, 3489-3503):
 * about z it acts on (x, y), about x on (y, z); cs, sn are cos/sin of anglez,
 * or of -anglex. */
template <bool STRICT, typename R>
__device__ __forceinline__ void rot_fwd(int flags, R cs, R sn, R& u0, R& u1, R& u2)
{
    if (flags & kRotZ) {
        R a, b;
        if constexpr (STRICT) {
            a = SOp::sub(SOp::mul(u0, cs), SOp::mul(u1, sn));
            b = SOp::add(SOp::mul(u0, sn), SOp::mul(u1, cs));
        } else {
            a = u0 * cs - u1 * sn;
            b = u0 * sn + u1 * cs;
        }
        u0 = a; u1 = b;
    } else if (flags & kRotX) {
        R a, b;
        if constexpr (STRICT) {
            a = SOp::sub(SOp::mul(u1, cs), SOp::mul(u2, sn));
            b = SOp::add(SOp::mul(u1, sn), SOp::mul(u2, cs));
        } else {
            a = u1 * cs - u2 * sn;
            b = u1 * sn + u2 * cs;
        }
        u1 = a; u2 = b;
    }
}

template <bool STRICT, typename R>
__device__ __forceinline__ void rot_back(int flags, R cs, R sn, R& u0, R& u1, R& u2)
{
    if (flags & kRotZ) {
        R x, y;
        if constexpr (STRICT) {
            x = SOp::add(SOp::mul(u0, cs), SOp::mul(u1, sn));
            y = SOp::add(SOp::mul(-u0, sn), SOp::mul(u1, cs));
        } else {
            x = u0 * cs + u1 * sn;
            y = -u0 * sn + u1 * cs;
        }
        u0 = x; u1 = y;
    } else if (flags & kRotX) {
        R y, z;
        if constexpr (STRICT) {
            y = SOp::add(SOp::mul(u1, cs), SOp::mul(u2, sn));
            z = SOp::add(SOp::mul(-u1, sn), SOp::mul(u2, cs));
        } else {
            y = u1 * cs + u2 * sn;
            z = -u1 * sn + u2 * cs;
        }
        u1 = y; u2 = z;
    }
}

/* D sweep (fdtd.c:3238-3343) for one interior cell; returns the updated D. */
template <typename R, bool STRICT>
__device__ __forceinline__ void d_update(const StepArgs<R>& a, int i, int j, int k, int64_t c,
                                         int sx, int sy, R hx0, R hy0, R hz0, R hxk, R hyk,
                                         R& dx, R& dy, R& dz)
{
    const R hz_jm = ldg(a.f.hz + c - a.nxp), hx_jm = ldg(a.f.hx + c - a.nxp);
    const R hz_im = ldg(a.f.hz + c - 1), hy_im = ldg(a.f.hy + c - 1);
    const int L = a.L;
    if constexpr (STRICT) {
        const double dHz_dy = SOp::div(SOp::sub(hz0, hz_jm), a.dys);
        const double dHy_dz = SOp::div(SOp::sub(hy0, hyk), a.dzs);
        const double dHx_dz = SOp::div(SOp::sub(hx0, hxk), a.dzs);
        const double dHz_dx = SOp::div(SOp::sub(hz0, hz_im), a.dxs);
        const double dHy_dx = SOp::div(SOp::sub(hy0, hy_im), a.dxs);
        const double dHx_dy = SOp::div(SOp::sub(hx0, hx_jm), a.dys);
        double pxy = 0.0, pxz = 0.0, pyx = 0.0, pyz = 0.0, pzx = 0.0, pzy = 0.0;
        double kappa_x = 1.0, kappa_y = 1.0, kappa_z = 1.0;
        if (sx >= 0) { /* fdtd.c:3258-3285 */
            kappa_x = ldg(a.tx.kappa + i);
            const double b = ldg(a.tx.b + i), cc = ldg(a.tx.c + i);
            const int64_t q = ((int64_t)k * a.ny + j) * (2 * L) + sx;
            pxy = a.psi.dxy[q];
            pxz = a.psi.dxz[q];
            a.psi.dxy[q] = SOp::add(SOp::mul(b, pxy), SOp::mul(cc, -dHz_dx));
            a.psi.dxz[q] = SOp::add(SOp::mul(b, pxz), SOp::mul(cc, dHy_dx));
        }
        if (sy >= 0) { /* fdtd.c:3288-3315 */
            kappa_y = ldg(a.ty.kappa + j);
            const double b = ldg(a.ty.b + j), cc = ldg(a.ty.c + j);
            const int64_t q = ((int64_t)k * (2 * L) + sy) * a.nxp + i;
            pyx = a.psi.dyx[q];
            pyz = a.psi.dyz[q];
            a.psi.dyx[q] = SOp::add(SOp::mul(b, pyx), SOp::mul(cc, dHz_dy));
            a.psi.dyz[q] = SOp::add(SOp::mul(b, pyz), SOp::mul(cc, -dHx_dy));
        }
        const int sz = ldg(a.tz.slot + k);
        double bz = 1.0, cz = 0.0;
        int64_t qz = 0;
        if (sz >= 0) { /* fdtd.c:3318-3334 */
            kappa_z = ldg(a.tz.kappa + k);
            bz = ldg(a.tz.b + k);
            cz = ldg(a.tz.c + k);
            qz = ((int64_t)sz * a.ny + j) * a.nxp + i;
            pzx = a.psi.dzx[qz];
            pzy = a.psi.dzy[qz];
        }
        /* fdtd.c:3337-3339 */
        const double ux = SOp::add(SOp::add(SOp::add(SOp::div(dHz_dy, kappa_y), pyx), SOp::div(-dHy_dz, kappa_z)), pzx);
        const double uy = SOp::add(SOp::add(SOp::add(SOp::div(-dHz_dx, kappa_x), pxy), SOp::div(dHx_dz, kappa_z)), pzy);
        const double uz = SOp::add(SOp::add(SOp::add(SOp::div(dHy_dx, kappa_x), pxz), SOp::div(-dHx_dy, kappa_y)), pyz);
        dx = SOp::add(dx, SOp::mul(a.dt, ux));
        dy = SOp::add(dy, SOp::mul(a.dt, uy));
        dz = SOp::add(dz, SOp::mul(a.dt, uz));
        if (sz >= 0) { /* fdtd.c:3340-3343 */
            a.psi.dzx[qz] = SOp::add(SOp::mul(bz, pzx), SOp::mul(cz, -dHy_dz));
            a.psi.dzy[qz] = SOp::add(SOp::mul(bz, pzy), SOp::mul(cz, dHx_dz));
        }
    } else {
        const R dHzy = hz0 - hz_jm, dHyz = hy0 - hyk, dHxz = hx0 - hxk;
        const R dHzx = hz0 - hz_im, dHyx = hy0 - hy_im, dHxy = hx0 - hx_jm;
        const R kdx = ldg(a.tx.kd + i), kdy = ldg(a.ty.kd + j), kdz = ldg(a.tz.kd + k);
        R ux = kdy * dHzy - kdz * dHyz;
        R uy = -kdx * dHzx + kdz * dHxz;
        R uz = kdx * dHyx - kdy * dHxy;
        if (sx >= 0) {
            const R b = ldg(a.tx.b + i), cd = ldg(a.tx.cd + i);
            const int64_t q = ((int64_t)k * a.ny + j) * (2 * L) + sx;
            const R pxy = a.psi.dxy[q], pxz = a.psi.dxz[q];
            uy += pxy;
            uz += pxz;
            a.psi.dxy[q] = b * pxy - cd * dHzx;
            a.psi.dxz[q] = b * pxz + cd * dHyx;
        }
        if (sy >= 0) {
            const R b = ldg(a.ty.b + j), cd = ldg(a.ty.cd + j);
            const int64_t q = ((int64_t)k * (2 * L) + sy) * a.nxp + i;
            const R pyx = a.psi.dyx[q], pyz = a.psi.dyz[q];
            ux += pyx;
            uz += pyz;
            a.psi.dyx[q] = b * pyx + cd * dHzy;
            a.psi.dyz[q] = b * pyz - cd * dHxy;
        }
        const int sz = ldg(a.tz.slot + k);
        if (sz >= 0) {
            const R b = ldg(a.tz.b + k), cd = ldg(a.tz.cd + k);
            const int64_t q = ((int64_t)sz * a.ny + j) * a.nxp + i;
            const R pzx = a.psi.dzx[q], pzy = a.psi.dzy[q];
            ux += pzx;
            uy += pzy;
            a.psi.dzx[q] = b * pzx - cd * dHyz;
            a.psi.dzy[q] = b * pzy + cd * dHxz;
        }
        dx += ux;
        dy += uy;
        dz += uz;
    }
}

/* D -> E, ADE and ions for one cell (fdtd.c:3404-3528).  ex..ez hold E^n on
 * entry (lab frame) and E^{n+1} on return; dx..dz are D^{n+1}. */
template <typename R, bool STRICT, int NAMAX>
__device__ __forceinline__ void e_update(const StepArgs<R>& a, const MatCoef<R>& m, int64_t c,
                                         R dx, R dy, R dz, R& ex, R& ey, R& ez)
{
    const int flags = m.flags;
    int64_t slot = -1;
    if (flags & (kAde | kAtoms)) slot = a.slot[c];
    const int64_t ns = a.nslot;

    /* P_ion = QeZV . r^n in the crystal frame (fdtd.c:3418-3427) */
    R pr0 = R(0), pr1 = R(0), pr2 = R(0);
    R rold[NAMAX > 0 ? 3 * NAMAX : 1];
    const int n3 = (NAMAX > 0 && (flags & kAtoms)) ? 3 * m.natom : 0;
    if constexpr (NAMAX > 0) {
        if (n3) {
            const R* qv = a.ion_coef + m.ion_off;
#pragma unroll 4
            for (int q = 0; q < n3; ++q) {
                const R rq = a.r[(int64_t)q * ns + slot];
                rold[q] = rq;
                const int at = q / 3, d = q - 3 * (q / 3);
                const R q0 = ldg(qv + at * 9 + 0 * 3 + d);
                const R q1 = ldg(qv + at * 9 + 1 * 3 + d);
                const R q2 = ldg(qv + at * 9 + 2 * 3 + d);
                if constexpr (STRICT) {
                    pr0 = SOp::add(pr0, SOp::mul(q0, rq));
                    pr1 = SOp::add(pr1, SOp::mul(q1, rq));
                    pr2 = SOp::add(pr2, SOp::mul(q2, rq));
                } else {
                    pr0 += q0 * rq;
                    pr1 += q1 * rq;
                    pr2 += q2 * rq;
                }
            }
        }
    }

    R ea = ex, eb = ey, ec = ez; /* E^n, crystal frame after rotation */
    R da = dx, db = dy, dc = dz;
    rot_fwd<STRICT>(flags, m.cs, m.sn, ea, eb, ec);
    rot_fwd<STRICT>(flags, m.cs, m.sn, da, db, dc);
    R dav, dbv, dcv;
    if constexpr (STRICT) {
        dav = SOp::sub(da, pr0); dbv = SOp::sub(db, pr1); dcv = SOp::sub(dc, pr2);
    } else {
        dav = da - pr0; dbv = db - pr1; dcv = dc - pr2;
    }

    R na, nb, nc; /* E^{n+1} in the crystal frame */
    if (!(flags & kAde)) {
        const R* E = m.eps_inv;
        if constexpr (STRICT) { /* fdtd.c:3459-3461 then 3486-3488 */
            na = SOp::div(SOp::mul(m.lf, SOp::add(SOp::add(SOp::mul(E[0], dav), SOp::mul(E[1], dbv)), SOp::mul(E[2], dcv))), a.eps0);
            nb = SOp::div(SOp::mul(m.lf, SOp::add(SOp::add(SOp::mul(E[3], dav), SOp::mul(E[4], dbv)), SOp::mul(E[5], dcv))), a.eps0);
            nc = SOp::div(SOp::mul(m.lf, SOp::add(SOp::add(SOp::mul(E[6], dav), SOp::mul(E[7], dbv)), SOp::mul(E[8], dcv))), a.eps0);
            na = SOp::sub(na, SOp::mul(m.lt, na));
            nb = SOp::sub(nb, SOp::mul(m.lt, nb));
            nc = SOp::sub(nc, SOp::mul(m.lt, nc));
        } else { /* eps_inv already carries lf (1 - lt) / eps0 */
            na = E[0] * dav + E[1] * dbv + E[2] * dcv;
            nb = E[3] * dav + E[4] * dbv + E[5] * dcv;
            nc = E[6] * dav + E[7] * dbv + E[8] * dcv;
        }
    } else {
        /* tensor ADE, fdtd.c:3463-3479: (I + g dt/2) P^{n+1} =
         * 2 P^n - (I - g dt/2) P^{n-1} + eps0 dt^2 wp2 E^n */
        R p0 = a.P[slot], p1 = a.P[ns + slot], p2 = a.P[2 * ns + slot];
        const R o0 = a.Po[slot], o1 = a.Po[ns + slot], o2 = a.Po[2 * ns + slot];
        const R* g = m.gm;
        const R* w = m.wp2;
        const R* gi = m.gp_inv;
        R t0, t1, t2;
        if constexpr (STRICT) {
#define PHP_ADE_TV(id, p)                                                                              \
    SOp::add(SOp::mul(2.0, p),                                                                         \
             SOp::add(SOp::sub(SOp::sub(SOp::mul(-g[id * 3 + 0], o0), SOp::mul(g[id * 3 + 1], o1)),   \
                               SOp::mul(g[id * 3 + 2], o2)),                                           \
                      SOp::mul(a.e0dt2, SOp::add(SOp::add(SOp::mul(w[id * 3 + 0], ea),                 \
                                                          SOp::mul(w[id * 3 + 1], eb)),                \
                                                 SOp::mul(w[id * 3 + 2], ec)))))
            t0 = PHP_ADE_TV(0, p0);
            t1 = PHP_ADE_TV(1, p1);
            t2 = PHP_ADE_TV(2, p2);
#undef PHP_ADE_TV
            const R n0 = SOp::add(SOp::add(SOp::add(0.0, SOp::mul(gi[0], t0)), SOp::mul(gi[1], t1)), SOp::mul(gi[2], t2));
            const R n1 = SOp::add(SOp::add(SOp::add(0.0, SOp::mul(gi[3], t0)), SOp::mul(gi[4], t1)), SOp::mul(gi[5], t2));
            const R n2 = SOp::add(SOp::add(SOp::add(0.0, SOp::mul(gi[6], t0)), SOp::mul(gi[7], t1)), SOp::mul(gi[8], t2));
            a.Po[slot] = p0; a.Po[ns + slot] = p1; a.Po[2 * ns + slot] = p2;
            a.P[slot] = n0; a.P[ns + slot] = n1; a.P[2 * ns + slot] = n2;
            na = SOp::div(SOp::div(SOp::sub(dav, n0), a.eps0), 20.0);
            nb = SOp::div(SOp::div(SOp::sub(dbv, n1), a.eps0), 20.0);
            nc = SOp::div(SOp::div(SOp::sub(dcv, n2), a.eps0), 20.0);
            na = SOp::sub(na, SOp::mul(m.lt, na));
            nb = SOp::sub(nb, SOp::mul(m.lt, nb));
            nc = SOp::sub(nc, SOp::mul(m.lt, nc));
        } else {
            t0 = R(2) * p0 - (g[0] * o0 + g[1] * o1 + g[2] * o2) + (w[0] * ea + w[1] * eb + w[2] * ec);
            t1 = R(2) * p1 - (g[3] * o0 + g[4] * o1 + g[5] * o2) + (w[3] * ea + w[4] * eb + w[5] * ec);
            t2 = R(2) * p2 - (g[6] * o0 + g[7] * o1 + g[8] * o2) + (w[6] * ea + w[7] * eb + w[8] * ec);
            const R n0 = gi[0] * t0 + gi[1] * t1 + gi[2] * t2;
            const R n1 = gi[3] * t0 + gi[4] * t1 + gi[5] * t2;
            const R n2 = gi[6] * t0 + gi[7] * t1 + gi[8] * t2;
            a.Po[slot] = p0; a.Po[ns + slot] = p1; a.Po[2 * ns + slot] = p2;
            a.P[slot] = n0; a.P[ns + slot] = n1; a.P[2 * ns + slot] = n2;
            na = (dav - n0) * m.ade_scale;
            nb = (dbv - n1) * m.ade_scale;
            nc = (dcv - n2) * m.ade_scale;
        }
    }

    /* ions: a = QeZM . E^{n+1} - DMM . r^n; r += v dt + a dt^2/2; v += a dt
     * (fdtd.c:3507-3528), all in the crystal frame */
    if constexpr (NAMAX > 0) {
        if (n3) {
            const R* qm = a.ion_coef + m.ion_off + 3 * n3;
            const R* dmm = qm + 3 * n3;
            const R dt = R(a.dt);
            for (int q = 0; q < n3; ++q) {
                const int at = q / 3, d = q - 3 * (q / 3);
                const R m0 = ldg(qm + at * 9 + 0 * 3 + d);
                const R m1 = ldg(qm + at * 9 + 1 * 3 + d);
                const R m2 = ldg(qm + at * 9 + 2 * 3 + d);
                const R* row = dmm + (int64_t)q * n3;
                R acc;
                if constexpr (STRICT) {
                    acc = SOp::add(SOp::add(SOp::mul(m0, na), SOp::mul(m1, nb)), SOp::mul(m2, nc));
                    for (int p = 0; p < n3; ++p) acc = SOp::sub(acc, SOp::mul(ldg(row + p), rold[p]));
                } else {
                    acc = m0 * na + m1 * nb + m2 * nc;
#pragma unroll 8
                    for (int p = 0; p < n3; ++p) acc -= ldg(row + p) * rold[p];
                }
                const int64_t o = (int64_t)q * ns + slot;
                const R vq = a.v[o];
                if constexpr (STRICT) {
                    a.r[o] = SOp::add(rold[q], SOp::add(SOp::mul(vq, a.dt), SOp::mul(SOp::mul(SOp::mul(0.5, acc), a.dt), a.dt)));
                    a.v[o] = SOp::add(vq, SOp::mul(acc, a.dt));
                } else {
                    a.r[o] = rold[q] + (vq * dt + R(0.5) * acc * dt * dt);
                    a.v[o] = vq + acc * dt;
                }
            }
        }
    }

    rot_back<STRICT>(flags, m.cs, m.sn, na, nb, nc);
    ex = na;
    ey = nb;
    ez = nc;
}

/* fdtd.c:3238-3528 fused: D sweep on the interior (i in [1,nx-1), j in
 * [1,ny-1)), sources, then D -> E / ADE / ions on every cell. */
template <typename R, bool STRICT, int NAMAX>
__global__ void __launch_bounds__(256) e_sweep(const StepArgs<R> a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= a.nx || j >= a.ny) return;
    const int k0 = blockIdx.z * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return;
    const bool interior = (i >= 1 && i < a.nx - 1 && j >= 1 && j < a.ny - 1);
    const int sx = ldg(a.tx.slot + i);
    const int sy = ldg(a.ty.slot + j);
    const int64_t P = a.plane;
    int64_t c = ((int64_t)k0 * a.ny + j) * a.nxp + i;
    R hxk = ldg(a.f.hx + c - P), hyk = ldg(a.f.hy + c - P); /* plane k-1 */

    for (int k = k0; k < k1; ++k, c += P) {
        const R hx0 = ldg(a.f.hx + c), hy0 = ldg(a.f.hy + c), hz0 = ldg(a.f.hz + c);
        const uint8_t mid = a.mat[c];
        const MatCoef<R>& m = a.mc[mid];
        const int flags = m.flags;
        R dx = a.f.dx[c], dy = a.f.dy[c], dz = a.f.dz[c];
        R ex = R(0), ey = R(0), ez = R(0);
        if (flags & (kLossy | kAde)) { ex = a.f.ex[c]; ey = a.f.ey[c]; ez = a.f.ez[c]; }
        if (interior) {
            d_update<R, STRICT>(a, i, j, k, c, sx, sy, hx0, hy0, hz0, hxk, hyk, dx, dy, dz);
            if (flags & kLossy) { /* fdtd.c:3349-3353 */
                const R* q = m.eps_im;
                if constexpr (STRICT) {
                    dx = SOp::sub(dx, SOp::mul(SOp::mul(a.c1, SOp::add(SOp::add(SOp::mul(q[0], ex), SOp::mul(q[1], ey)), SOp::mul(q[2], ez))), a.eps0));
                    dy = SOp::sub(dy, SOp::mul(SOp::mul(a.c1, SOp::add(SOp::add(SOp::mul(q[3], ex), SOp::mul(q[4], ey)), SOp::mul(q[5], ez))), a.eps0));
                    dz = SOp::sub(dz, SOp::mul(SOp::mul(a.c1, SOp::add(SOp::add(SOp::mul(q[6], ex), SOp::mul(q[7], ey)), SOp::mul(q[8], ez))), a.eps0));
                } else {
                    dx -= q[0] * ex + q[1] * ey + q[2] * ez;
                    dy -= q[3] * ex + q[4] * ey + q[5] * ez;
                    dz -= q[6] * ex + q[7] * ey + q[8] * ez;
                }
            }
        }
        /* sources, in source order (fdtd.c:3363-3396) */
        for (int s = 0; s < a.nsrc; ++s) {
            if (a.src_cell[s] == c) {
                const double v = a.src_val[s];
                if constexpr (STRICT) {
                    const double add = SOp::mul(v, a.dt);
                    if (a.src_comp[s] == 0) dx = SOp::add(dx, add);
                    else if (a.src_comp[s] == 1) dy = SOp::add(dy, add);
                    else if (a.src_comp[s] == 2) dz = SOp::add(dz, add);
                } else {
                    const R add = R(v * a.dt);
                    if (a.src_comp[s] == 0) dx += add;
                    else if (a.src_comp[s] == 1) dy += add;
                    else if (a.src_comp[s] == 2) dz += add;
                }
            }
        }
        a.f.dx[c] = dx;
        a.f.dy[c] = dy;
        a.f.dz[c] = dz;
        e_update<R, STRICT, NAMAX>(a, m, c, dx, dy, dz, ex, ey, ez);
        a.f.ex[c] = ex;
        a.f.ey[c] = ey;
        a.f.ez[c] = ez;
        hxk = hx0;
        hyk = hy0;
    }
}

/* ========================================================== small kernels */

/* Gathers one plane of a component into out (float or double).
 * axis 0: z plane kk -> [i][j]; axis 1: x plane -> [j][k]; axis 2: y plane
 * -> [i][k].  comp 9 is |E|. */
template <typename R, typename O>
__global__ void gather_plane(const Fields<R> f, int comp, int axis, int pos, int nx, int ny, int nz,
                             int nxp, O* out)
{
    const int64_t plane = (int64_t)nxp * ny;
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
        (void)plane;
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
 * (3*natom each).  count[1] is raised instead of writing past cap. */
template <typename R>
__global__ void probe_record_counted(const Fields<R> f, int64_t cf, const R* r, const R* v, int64_t nslot,
                                     int64_t slot, int n3, double* rows, int32_t* count, int cap, int row_len)
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
        out[t] = (q < n3) ? (double)r[(int64_t)q * nslot + slot] : (double)v[(int64_t)(q - n3) * nslot + slot];
    }
    __syncthreads();
    if (threadIdx.x == 0) count[0] = row + 1;
}

/* Running DFT sample: acc[f][i][j] += x * (cos, sin) for the phasors of this
 * step (phasor[2*f], phasor[2*f+1]); skipped when flag == 0. */
template <typename R>
__global__ void dft_sample(const R* src, int64_t plane_off, int nx, int ny, int nxp, int nfreq,
                           int cast_f32, const double* step_in, int flag_off, int phasor_off,
                           double* acc)
{
    if (step_in[flag_off] == 0.0) return;
    const int64_t n = (int64_t)nx * ny;
    const double* ph = step_in + phasor_off;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / ny), j = (int)(t % ny);
        double x = (double)src[plane_off + (int64_t)j * nxp + i];
        if (cast_f32) x = (double)(float)x;
        for (int f = 0; f < nfreq; ++f) {
            double* a = acc + ((int64_t)f * n + t) * 2;
            a[0] += x * ph[2 * f];
            a[1] += x * ph[2 * f + 1];
        }
    }
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

/* Pass 1 over cells (|E|, |Ex|) and pool slots (|r|); one partial per block
 * into scratch.  slot_cell maps a pool slot to its device cell index. */
template <typename R>
__global__ void __launch_bounds__(256) diag_pass1(const Fields<R> f, int nx, int ny, int nz, int nxp,
                                                  const R* r, int64_t nslot, const int64_t* slot_cell,
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
            const double rv = fabs((double)r[(int64_t)q * nslot + s]);
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

} // namespace phpdev
