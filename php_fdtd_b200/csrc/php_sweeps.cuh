/*
 * php_sweeps.cuh -- the per-cell physics of one PhP_FDTD time step, shared by
 * the TMA plane-ring sweeps of php_sweeps_tma.cuh and the one-launch step of
 * php_sweep_fused.cuh:
 *
 *   d_update        D += dt (curl H / kappa + psi_D) - eps''  fdtd.c:3238-3356
 *   e_cell_values   D -> E (rotation, eps^-1 or ADE, loss)    fdtd.c:3404-3503
 *   e_update        tensor ADE and the ion equations of motion fdtd.c:3463-3528
 *
 * CPML and material coefficients are loaded only inside the branches that
 * need them, so they never occupy registers across the sweeps' loops.
 */
#pragma once

namespace phpdev {

/* ================================================================ E sweep */

/* Rotation to the crystal frame and back (fdtd.c:3429-3452, 3489-3503):
 * about z it acts on (x, y), about x on (y, z); cs, sn are cos/sin of anglez,
 * or of -anglex. */
template <bool STRICT, typename R>
__device__ __forceinline__ void rot_fwd(int flags, R cs, R sn, R& u0, R& u1, R& u2)
{
    if (flags & kRotZ) {
        R p, q;
        if constexpr (STRICT) {
            p = SOp::sub(SOp::mul(u0, cs), SOp::mul(u1, sn));
            q = SOp::add(SOp::mul(u0, sn), SOp::mul(u1, cs));
        } else {
            p = u0 * cs - u1 * sn;
            q = u0 * sn + u1 * cs;
        }
        u0 = p; u1 = q;
    } else if (flags & kRotX) {
        R p, q;
        if constexpr (STRICT) {
            p = SOp::sub(SOp::mul(u1, cs), SOp::mul(u2, sn));
            q = SOp::add(SOp::mul(u1, sn), SOp::mul(u2, cs));
        } else {
            p = u1 * cs - u2 * sn;
            q = u1 * sn + u2 * cs;
        }
        u1 = p; u2 = q;
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

/* CPML state of one cell read before its update: the z slot of the plane
 * and the old psi values of every PML axis the cell lies in (zero
 * elsewhere).  Loading them apart from the update lets a kernel issue these
 * loads early, before it waits for the plane's other inputs. */
template <typename R>
struct CellPsi {
    int sz;
    R xy, xz, yx, yz, zx, zy;
    R kdz;                     /* dt / (dz kappa_z), FP32/FP64 fast paths */
};

/* psi_D of fdtd.c:3258-3334 (the reads) */
template <typename R>
__device__ __forceinline__ void load_psi_d(const StepArgs<R>& a, int i, int j, int k, int sx, int sy, CellPsi<R>& ps)
{
    const int L2 = 2 * a.L;
    ps.sz = ldg_nh(a.tz.slot + k);
    /* FP64: the z profile with the other early loads (measured faster);
     * FP32 reads it in d_update (measured faster there) */
    ps.kdz = sizeof(R) == 8 ? ldg_nh(a.tz.kd + k) : R(0);
    ps.xy = ps.xz = ps.yx = ps.yz = ps.zx = ps.zy = R(0);
    if (sx >= 0) {
        const int q = (k * a.ny + j) * L2 + sx;
        ps.xy = a.psi.dxy[q];
        ps.xz = a.psi.dxz[q];
    }
    if (sy >= 0) {
        const int q = (k * L2 + sy) * a.nxp + i;
        ps.yx = a.psi.dyx[q];
        ps.yz = a.psi.dyz[q];
    }
    if (ps.sz >= 0) {
        const int q = (ps.sz * a.ny + j) * a.nxp + i;
        ps.zx = a.psi.dzx[q];
        ps.zy = a.psi.dzy[q];
    }
}

/* the lines load_psi_d reads at plane k, requested into L1 a plane ahead */
template <typename R>
__device__ __forceinline__ void prefetch_psi_d(const StepArgs<R>& a, int i, int j, int k, int sx, int sy)
{
    const int L2 = 2 * a.L;
    if (sx >= 0) {
        const int q = (k * a.ny + j) * L2 + sx;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.dxy + q));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.dxz + q));
    }
    if (sy >= 0) {
        const int q = (k * L2 + sy) * a.nxp + i;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.dyx + q));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.dyz + q));
    }
    const int sz = ldg_nh(a.tz.slot + k);
    if (sz >= 0) {
        const int q = (sz * a.ny + j) * a.nxp + i;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.dzx + q));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.dzy + q));
    }
}

/* D sweep (fdtd.c:3238-3343) for one interior cell; hx0..hz0 are H at the
 * cell, hxk/hyk at k-1, hz_jm/hx_jm at j-1, hz_im/hy_im at i-1; ps holds the
 * old psi values (load_psi_d). */
template <typename R, bool STRICT>
__device__ __forceinline__ void d_update(const StepArgs<R>& a, int i, int j, int k, int sx, int sy, R hx0, R hy0,
                                         R hz0, R hxk, R hyk, R hz_jm, R hx_jm, R hz_im, R hy_im,
                                         const CellPsi<R>& ps, R& dx, R& dy, R& dz)
{
    const int L2 = 2 * a.L;
    const int sz = ps.sz;
    if constexpr (STRICT) {
        const double dHz_dy = SOp::div(SOp::sub(hz0, hz_jm), a.dys);
        const double dHy_dz = SOp::div(SOp::sub(hy0, hyk), a.dzs);
        const double dHx_dz = SOp::div(SOp::sub(hx0, hxk), a.dzs);
        const double dHz_dx = SOp::div(SOp::sub(hz0, hz_im), a.dxs);
        const double dHy_dx = SOp::div(SOp::sub(hy0, hy_im), a.dxs);
        const double dHx_dy = SOp::div(SOp::sub(hx0, hx_jm), a.dys);
        double kappa_x = 1.0, kappa_y = 1.0, kappa_z = 1.0;
        if (sx >= 0) { /* fdtd.c:3258-3285 */
            kappa_x = ldg_nh(a.tx.kappa + i);
            const double b = ldg_nh(a.tx.b + i), cc = ldg_nh(a.tx.c + i);
            const int q = (k * a.ny + j) * L2 + sx;
            a.psi.dxy[q] = SOp::add(SOp::mul(b, ps.xy), SOp::mul(cc, -dHz_dx));
            a.psi.dxz[q] = SOp::add(SOp::mul(b, ps.xz), SOp::mul(cc, dHy_dx));
        }
        if (sy >= 0) { /* fdtd.c:3288-3315 */
            kappa_y = ldg_nh(a.ty.kappa + j);
            const double b = ldg_nh(a.ty.b + j), cc = ldg_nh(a.ty.c + j);
            const int q = (k * L2 + sy) * a.nxp + i;
            a.psi.dyx[q] = SOp::add(SOp::mul(b, ps.yx), SOp::mul(cc, dHz_dy));
            a.psi.dyz[q] = SOp::add(SOp::mul(b, ps.yz), SOp::mul(cc, -dHx_dy));
        }
        if (sz >= 0) kappa_z = ldg_nh(a.tz.kappa + k); /* fdtd.c:3318-3334 */
        /* fdtd.c:3337-3339 */
        const double ux = SOp::add(SOp::add(SOp::add(SOp::div(dHz_dy, kappa_y), ps.yx), SOp::div(-dHy_dz, kappa_z)), ps.zx);
        const double uy = SOp::add(SOp::add(SOp::add(SOp::div(-dHz_dx, kappa_x), ps.xy), SOp::div(dHx_dz, kappa_z)), ps.zy);
        const double uz = SOp::add(SOp::add(SOp::add(SOp::div(dHy_dx, kappa_x), ps.xz), SOp::div(-dHx_dy, kappa_y)), ps.yz);
        dx = SOp::add(dx, SOp::mul(a.dt, ux));
        dy = SOp::add(dy, SOp::mul(a.dt, uy));
        dz = SOp::add(dz, SOp::mul(a.dt, uz));
        if (sz >= 0) { /* fdtd.c:3340-3343 */
            const double b = ldg_nh(a.tz.b + k), cc = ldg_nh(a.tz.c + k);
            const int qz = (sz * a.ny + j) * a.nxp + i;
            a.psi.dzx[qz] = SOp::add(SOp::mul(b, ps.zx), SOp::mul(cc, -dHy_dz));
            a.psi.dzy[qz] = SOp::add(SOp::mul(b, ps.zy), SOp::mul(cc, dHx_dz));
        }
    } else {
        const R dHzy = hz0 - hz_jm, dHyz = hy0 - hyk, dHxz = hx0 - hxk;
        const R dHzx = hz0 - hz_im, dHyx = hy0 - hy_im, dHxy = hx0 - hx_jm;
        const R kdx = ldg(a.tx.kd + i), kdy = ldg(a.ty.kd + j);
        const R kdz = sizeof(R) == 8 ? ps.kdz : ldg_nh(a.tz.kd + k);
        /* psi terms enter as zeros outside the PML */
        R ux = kdy * dHzy - kdz * dHyz + ps.yx + ps.zx;
        R uy = -kdx * dHzx + kdz * dHxz + ps.xy + ps.zy;
        R uz = kdx * dHyx - kdy * dHxy + ps.xz + ps.yz;
        if (sx >= 0) {
            const R b = ldg_nh(a.tx.b + i), cd = ldg_nh(a.tx.cd + i);
            const int q = (k * a.ny + j) * L2 + sx;
            a.psi.dxy[q] = b * ps.xy - cd * dHzx;
            a.psi.dxz[q] = b * ps.xz + cd * dHyx;
        }
        if (sy >= 0) {
            const R b = ldg_nh(a.ty.b + j), cd = ldg_nh(a.ty.cd + j);
            const int q = (k * L2 + sy) * a.nxp + i;
            a.psi.dyx[q] = b * ps.yx + cd * dHzy;
            a.psi.dyz[q] = b * ps.yz - cd * dHxy;
        }
        if (sz >= 0) {
            const R b = ldg_nh(a.tz.b + k), cd = ldg_nh(a.tz.cd + k);
            const int q = (sz * a.ny + j) * a.nxp + i;
            a.psi.dzx[q] = b * ps.zx - cd * dHyz;
            a.psi.dzy[q] = b * ps.zy + cd * dHxz;
        }
        dx += ux;
        dy += uy;
        dz += uz;
    }
}

/* FP32: E = iso * D from the kernel parameters for plain isotropic cells
 * (measured 2 % faster on the 256^3 tip workload; FP64 measured slower) */
#ifndef PHP_ISO_PARAM
#define PHP_ISO_PARAM 1
#endif

/* bytes of r (and again of v) per cell up to which the fused sweep holds a
 * cell's ion state in registers: 6 FP32 coordinates (two atoms) fit the
 * 64-register budget of the FP32 sweep without spills, FP64 ones do not */
constexpr int kIonRegBytes = 24;
/* FP64: the same for two atoms (48 bytes), with the fused sweeps that hold
 * them compiled for three resident blocks of 80 registers instead of four of
 * 64 (measured E sweep 1.510 -> 1.464 ms on the 512 x 512 x 256 two-atom
 * slab, 0.0495 -> 0.0435 ms on the 96^3 one; the 64-register budget would
 * spill them) */
#ifndef PHP_ION_REG64
#define PHP_ION_REG64 48
#endif
#ifndef PHP_E_MINBLOCKS64_ATOMS
#define PHP_E_MINBLOCKS64_ATOMS 3
#endif
/* FP32 keeps four blocks of 64 registers for them (three of 80 measured
 * 0.158 -> 0.171 ms on the 192^3 two-atom grid) */
#ifndef PHP_E_MINBLOCKS32_ATOMS
#define PHP_E_MINBLOCKS32_ATOMS 4
#endif
template <typename R>
constexpr int kIonRegBytesR = sizeof(R) == 8 ? PHP_ION_REG64 : kIonRegBytes;
/* whether the fused update of NAMAX atoms holds a cell's r and v in registers */
template <typename R, int NAMAX>
constexpr bool kIonVReg = NAMAX > 0 && 3 * NAMAX * (int)sizeof(R) <= kIonRegBytesR<R>;

/* f(q) for q = 0 .. n3-1 in order; with UNR fully unrolled over the bound
 * QN (predicated), so that arrays indexed by q stay in registers */
template <int QN, bool UNR, typename F>
__device__ __forceinline__ void for_atoms(int n3, F&& f)
{
    if constexpr (UNR) {
#pragma unroll
        for (int q = 0; q < QN; ++q)
            if (q < n3) f(q);
    } else {
#pragma unroll 6
        for (int q = 0; q < n3; ++q) f(q);
    }
}

/* Coefficient sources of the fused ion update: the material's arrays in
 * global memory, or the copy in the kernel parameters, which the unrolled
 * few-atom loops read as constant-bank operands instead of loads. */
template <typename R>
struct IonCoefGlobal {
    const R* qv;
    int n3;
    __device__ __forceinline__ R zv(int i) const { return ldg(qv + i); }
    __device__ __forceinline__ R zm(int i) const { return ldg(qv + 3 * n3 + i); }
    __device__ __forceinline__ R dmm(int q, int p) const { return ldg(qv + 6 * n3 + q * n3 + p); }
};
template <typename R>
struct IonCoefParam {
    const StepArgs<R>& a;
    __device__ __forceinline__ R zv(int i) const { return a.ion_k[i]; }
    __device__ __forceinline__ R zm(int i) const { return a.ion_k[kIonKM + i]; }
    __device__ __forceinline__ R dmm(int q, int p) const { return a.ion_k[kIonKD + q * kIonKQ + p]; }
};

/* A cell's pool slot, read ahead of the stage wait by a caller that knows
 * the cell's material. */
struct IonPre {
    int64_t slot;
};

/* D -> E, ADE and ions for one cell (fdtd.c:3404-3528).  ex..ez hold E^n on
 * entry (lab frame) and E^{n+1} on return; dx..dz are D^{n+1}; ix..iz are
 * D^{n+1} - D^n as summed before rounding into D (FP32 only).  pre: the
 * slot already read, or null. */
template <typename R, bool STRICT, int NAMAX>
__device__ __forceinline__ void e_update(const StepArgs<R>& a, const MatCoef<R>& m, int c,
                                         R dx, R dy, R dz, R ix, R iy, R iz, R& ex, R& ey, R& ez,
                                         const IonPre* pre = nullptr)
{
    const int flags = m.flags;
    if constexpr (!STRICT) {
        if (flags & kIso) { /* vacuum and isotropic lossless dielectrics */
            const R s = m.eps_inv[0];
            ex = s * dx;
            ey = s * dy;
            ez = s * dz;
            return;
        }
    }
    int64_t slot = -1;
    if (pre) slot = pre->slot;
    else if (flags & (kAde | kAtoms)) slot = a.slot[c];
    const int64_t ns = a.nslot;

    /* P_ion = QeZV . r^n in the crystal frame (fdtd.c:3418-3427).  With
     * few atoms (VREG) r and v of the cell sit in registers and all 2 x 3N
     * loads are issued together here. */
    constexpr int QN = NAMAX > 0 ? 3 * NAMAX : 1;
    constexpr bool VREG = NAMAX > 0 && QN * (int)sizeof(R) <= kIonRegBytesR<R>;
    R pr0 = R(0), pr1 = R(0), pr2 = R(0);
    R rold[QN];
    R vold[VREG ? QN : 1];
    const int n3 = (NAMAX > 0 && (flags & kAtoms)) ? 3 * m.natom : 0;
    /* few-atom cells of the material held in the parameters */
    const bool kpar = VREG && NAMAX <= 4 && m.ion_off == a.ion_k_off;
    if constexpr (NAMAX > 0) {
        if (n3) {
            if constexpr (VREG) {
#pragma unroll
                for (int q = 0; q < QN; ++q) {
                    /* 32-bit element offsets: the host keeps few-atom pools
                     * below 2^32 elements */
                    const uint32_t o = (uint32_t)q * (uint32_t)ns + (uint32_t)slot;
                    rold[q] = q < n3 ? a.r[o] : R(0);
                    vold[q] = q < n3 ? a.v[o] : R(0);
                }
            }
            auto ion_pr = [&](const auto& C) {
                for_atoms<QN, VREG>(n3, [&](int q) {
                    R rq;
                    if constexpr (VREG) {
                        rq = rold[q];
                    } else {
                        rq = a.r[(int64_t)q * ns + slot];
                        rold[q] = rq;
                        /* v is read after E^{n+1}: bring it into L1 now */
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.v + (int64_t)q * ns + slot));
                    }
                    const int at = q / 3, d = q - 3 * at;
                    const R q0 = C.zv(at * 9 + 0 * 3 + d);
                    const R q1 = C.zv(at * 9 + 1 * 3 + d);
                    const R q2 = C.zv(at * 9 + 2 * 3 + d);
                    if constexpr (STRICT) {
                        pr0 = SOp::add(pr0, SOp::mul(q0, rq));
                        pr1 = SOp::add(pr1, SOp::mul(q1, rq));
                        pr2 = SOp::add(pr2, SOp::mul(q2, rq));
                    } else {
                        pr0 += q0 * rq;
                        pr1 += q1 * rq;
                        pr2 += q2 * rq;
                    }
                });
            };
            if (kpar) ion_pr(IonCoefParam<R>{a});
            else ion_pr(IonCoefGlobal<R>{a.ion_coef + m.ion_off, n3});
        }
    }

    if constexpr (!STRICT && NAMAX == 0) {
        /* many-atom cells: P_ion = QeZV . r^n left by the ion pass */
        if ((flags & kAtoms) && a.pr) {
            pr0 = a.pr[slot];
            pr1 = a.pr[ns + slot];
            pr2 = a.pr[2 * ns + slot];
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
        const R p0 = a.P[slot], p1 = a.P[ns + slot], p2 = a.P[2 * ns + slot];
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
        } else if constexpr (sizeof(R) == 8) {
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
        } else {
            /* FP32: the same recurrence, rewritten so that no step cancels
             * digits.  With J^n = P^n - P^{n-1},
             *   J^{n+1} = J^n - A J^n + B E^n,  A = 2 (I + g dt/2)^-1 g dt/2,
             *                                   B = (I + g dt/2)^-1 eps0 dt^2 wp2
             * (A in gm, B in wp2), and E^{n+1} is taken from
             * Q = D - P (lab frame), Q^{n+1} = Q^n + (D^{n+1} - D^n) - J^{n+1}
             * in the crystal frame.  The pools hold Q (P pool) and J (P_old
             * pool).  In a metal D and P agree to a few parts in 1e3, and
             * 2 P^n - P^{n-1} to a few parts in 1e3 of P: both differences
             * lose most single-precision digits and drift by percents over
             * thousands of steps. */
            (void)gi;
            const R j0 = o0 - (g[0] * o0 + g[1] * o1 + g[2] * o2) + (w[0] * ea + w[1] * eb + w[2] * ec);
            const R j1 = o1 - (g[3] * o0 + g[4] * o1 + g[5] * o2) + (w[3] * ea + w[4] * eb + w[5] * ec);
            const R j2 = o2 - (g[6] * o0 + g[7] * o1 + g[8] * o2) + (w[6] * ea + w[7] * eb + w[8] * ec);
            R qa = p0 + ix, qb = p1 + iy, qc = p2 + iz;
            rot_fwd<STRICT>(flags, m.cs, m.sn, qa, qb, qc);
            qa -= j0;
            qb -= j1;
            qc -= j2;
            na = (qa - pr0) * m.ade_scale;
            nb = (qb - pr1) * m.ade_scale;
            nc = (qc - pr2) * m.ade_scale;
            rot_back<STRICT>(flags, m.cs, m.sn, qa, qb, qc);
            a.Po[slot] = j0; a.Po[ns + slot] = j1; a.Po[2 * ns + slot] = j2;
            a.P[slot] = qa; a.P[ns + slot] = qb; a.P[2 * ns + slot] = qc;
        }
    }

    /* ions: a = QeZM . E^{n+1} - DMM . r^n; r += v dt + a dt^2/2; v += a dt
     * (fdtd.c:3507-3528), all in the crystal frame */
    if constexpr (NAMAX > 0) {
        const R dt = R(a.dt);
        auto ion_eom = [&](const auto& C) {
            for_atoms<QN, VREG>(n3, [&](int q) {
                const int at = q / 3, d = q - 3 * at;
                const R m0 = C.zm(at * 9 + 0 * 3 + d);
                const R m1 = C.zm(at * 9 + 1 * 3 + d);
                const R m2 = C.zm(at * 9 + 2 * 3 + d);
                R acc;
                if constexpr (STRICT) {
                    acc = SOp::add(SOp::add(SOp::mul(m0, na), SOp::mul(m1, nb)), SOp::mul(m2, nc));
                    for_atoms<QN, VREG>(n3, [&](int p) { acc = SOp::sub(acc, SOp::mul(C.dmm(q, p), rold[p])); });
                } else {
                    acc = m0 * na + m1 * nb + m2 * nc;
                    for_atoms<QN, VREG>(n3, [&](int p) { acc -= C.dmm(q, p) * rold[p]; });
                }
                const int64_t o = VREG ? (int64_t)((uint32_t)q * (uint32_t)ns + (uint32_t)slot) : (int64_t)q * ns + slot;
                R vq;
                if constexpr (VREG) vq = vold[q];
                else vq = a.v[o];
                if constexpr (STRICT) {
                    a.r[o] = SOp::add(rold[q], SOp::add(SOp::mul(vq, a.dt), SOp::mul(SOp::mul(SOp::mul(0.5, acc), a.dt), a.dt)));
                    a.v[o] = SOp::add(vq, SOp::mul(acc, a.dt));
                } else {
                    a.r[o] = rold[q] + (vq * dt + R(0.5) * acc * dt * dt);
                    a.v[o] = vq + acc * dt;
                }
            });
        };
        if (n3) {
            if (kpar) ion_eom(IonCoefParam<R>{a});
            else ion_eom(IonCoefGlobal<R>{a.ion_coef + m.ion_off, n3});
        }
    }

    rot_back<STRICT>(flags, m.cs, m.sn, na, nb, nc);
    ex = na;
    ey = nb;
    ez = nc;
}

/* One cell of the fused sweep once its H values are known: D update on
 * the interior with the lossy eps'' term (fdtd.c:3238-3356), the sources of
 * this step (fdtd.c:3363-3396), D -> E / ADE / ions (fdtd.c:3404-3528).  The
 * new D and E come back in dx..dz and ex_out..ez_out; the caller stores
 * them (e_cell below in place, he_sweep_tma E into the new level). */
template <typename R, bool STRICT, int NAMAX>
__device__ __forceinline__ void e_cell_values(const StepArgs<R>& a, int i, int j, int k, int c, bool interior, int sx,
                                              int sy, R hx0, R hy0, R hz0, R hxk, R hyk, R hz_jm, R hx_jm, R hz_im,
                                              R hy_im, R& dx, R& dy, R& dz, int mid, const MatCoef<R>* mcs,
                                              const CellPsi<R>* pre, R& ex_out, R& ey_out, R& ez_out,
                                              const IonPre* ipre = nullptr)
{
    const R* __restrict__ exp_ = a.f.ex;
    const R* __restrict__ eyp = a.f.ey;
    const R* __restrict__ ezp = a.f.ez;
    /* plain isotropic cells take E = iso * D without the material record */
    const R iso = (!STRICT && PHP_ISO_PARAM && sizeof(R) == 4 && mid < kIsoMats) ? a.iso[mid] : R(0);
    /* mcs: the block's shared-memory copy of the first kSmemMats records */
    const MatCoef<R>* mp = iso != R(0) ? nullptr : ((mcs && mid < a.nmat) ? &mcs[mid] : &a.mc[mid]);
    const int flags = mp ? mp->flags : kIso;
    R ex = R(0), ey = R(0), ez = R(0);
    if (flags & (kLossy | kAde)) { ex = exp_[c]; ey = eyp[c]; ez = ezp[c]; }
    /* FP32 sums this step's D increment on its own before adding it to D:
     * the ADE update needs the increment without D's rounding */
    constexpr bool kInc = !STRICT && sizeof(R) == 4;
    R ix = R(0), iy = R(0), iz = R(0);
    R& ux = kInc ? ix : dx;
    R& uy = kInc ? iy : dy;
    R& uz = kInc ? iz : dz;
    if (interior) {
        CellPsi<R> ps;
        if (pre) ps = *pre;
        else load_psi_d(a, i, j, k, sx, sy, ps);
        d_update<R, STRICT>(a, i, j, k, sx, sy, hx0, hy0, hz0, hxk, hyk, hz_jm, hx_jm, hz_im, hy_im, ps, ux, uy, uz);
        if (flags & kLossy) { /* fdtd.c:3349-3353 */
            const R* q = mp->eps_im;
            if constexpr (STRICT) {
                dx = SOp::sub(dx, SOp::mul(SOp::mul(a.c1, SOp::add(SOp::add(SOp::mul(q[0], ex), SOp::mul(q[1], ey)), SOp::mul(q[2], ez))), a.eps0));
                dy = SOp::sub(dy, SOp::mul(SOp::mul(a.c1, SOp::add(SOp::add(SOp::mul(q[3], ex), SOp::mul(q[4], ey)), SOp::mul(q[5], ez))), a.eps0));
                dz = SOp::sub(dz, SOp::mul(SOp::mul(a.c1, SOp::add(SOp::add(SOp::mul(q[6], ex), SOp::mul(q[7], ey)), SOp::mul(q[8], ez))), a.eps0));
            } else {
                ux -= q[0] * ex + q[1] * ey + q[2] * ez;
                uy -= q[3] * ex + q[4] * ey + q[5] * ez;
                uz -= q[6] * ex + q[7] * ey + q[8] * ez;
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
                if (a.src_comp[s] == 0) ux += add;
                else if (a.src_comp[s] == 1) uy += add;
                else if (a.src_comp[s] == 2) uz += add;
            }
        }
    }
    if constexpr (kInc) {
        dx += ix;
        dy += iy;
        dz += iz;
    }
    if (!mp) {
        ex = iso * dx;
        ey = iso * dy;
        ez = iso * dz;
    } else {
        e_update<R, STRICT, NAMAX>(a, *mp, c, dx, dy, dz, ix, iy, iz, ex, ey, ez, ipre);
    }
    ex_out = ex;
    ey_out = ey;
    ez_out = ez;
}

/* e_cell_values with D and E stored to global memory */
template <typename R, bool STRICT, int NAMAX>
__device__ __forceinline__ void e_cell(const StepArgs<R>& a, int i, int j, int k, int c, bool interior, int sx, int sy,
                                       R hx0, R hy0, R hz0, R hxk, R hyk, R hz_jm, R hx_jm, R hz_im, R hy_im, R dx, R dy,
                                       R dz, int mid, const MatCoef<R>* mcs, const CellPsi<R>* pre,
                                       const IonPre* ipre = nullptr)
{
    R ex, ey, ez;
    e_cell_values<R, STRICT, NAMAX>(a, i, j, k, c, interior, sx, sy, hx0, hy0, hz0, hxk, hyk, hz_jm, hx_jm, hz_im, hy_im,
                                    dx, dy, dz, mid, mcs, pre, ex, ey, ez, ipre);
    a.f.dx[c] = dx;
    a.f.dy[c] = dy;
    a.f.dz[c] = dz;
    a.f.ex[c] = ex;
    a.f.ey[c] = ey;
    a.f.ez[c] = ez;
}

} // namespace phpdev
