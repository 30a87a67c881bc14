/*
 * php_sweep_fused.cuh -- the time step of fdtd.c:3116-3528 in one launch
 * (sm_100a): the H sweep and the fused D / source / E / ADE / ion sweep of
 * php_sweeps_tma.cuh in a single z march per block.
 *
 * The two sweeps move E and H (H sweep), then H again with D and the
 * material ids (E sweep): every step reads H twice.  Here the block of a
 * 32 x 8 tile and z chunk computes, plane by plane, the new H of its tile and
 * of the 41 cells one below it in x and y (its D update needs their H; they
 * belong to the neighbouring tiles and are computed twice), keeps it in
 * shared memory and registers, and updates D and E from it.  H crosses HBM
 * once per step in each direction, and one launch replaces two.
 *
 * Per plane the stage ring holds, loaded by TMA (tile mode, no multicast,
 * this GPU's own memory only): E^n on the tile widened by one cell on every
 * side (x widened to 16 bytes), H^{n-1/2} on the tile and the cells below
 * it, D^n and the material ids of the tile.  The march starts one plane
 * below the chunk (the D update of plane k0 needs the new H of plane k0 - 1,
 * computed again here) and reads E one plane above it.
 *
 * The cells below the tile are updated by their own blocks during the same
 * launch, so their old E, H and H CPML state must stay readable: those are
 * double buffered (the launch reads StepArgs::f and psi, and writes the new
 * level to enew, hnew and psin_h; the host swaps the buffers after the
 * launch).  D, the D CPML state and the ADE and lattice pools belong to one
 * cell each and are updated in place.  The arithmetic per cell is that of
 * the two sweeps, operation for operation, so both paths give the same
 * fields.
 *
 * Waits are bounded as in the two sweeps (kWaitLimit polls, error flag,
 * drain of the loads in flight).
 */
#pragma once

namespace phpdev {

/* ring depth and resident blocks per SM the kernel is compiled for, FP64 and
 * FP32 (measured on the 256^3 tip workload: FP64 0.612 ms per step with 3
 * stages and 3 blocks of 80 registers, 0.684 ms with 4 stages and 2 blocks of
 * 125; FP32 0.359 ms with 3 stages and 4 blocks, 0.404 ms with 4 and 3) */
#ifndef PHP_FUSED_S64
#define PHP_FUSED_S64 3
#endif
#ifndef PHP_FUSED_S32
#define PHP_FUSED_S32 3
#endif
#ifndef PHP_FUSED_MINB64
#define PHP_FUSED_MINB64 3
#endif
#ifndef PHP_FUSED_MINB32
#define PHP_FUSED_MINB32 4
#endif
/* 1: each thread reads D and the material id of its cell from global memory
 * at the start of the pass, before the stage wait (they are used after the
 * H part), instead of having them staged by TMA: the stages hold E and H
 * only, a third less shared memory per stage, which lets three FP64 blocks
 * share an SM; FP64 and FP32 (FP32 measured 0.375 ms with it, 0.359 ms
 * without) */
#ifndef PHP_FUSED_DREG64
#define PHP_FUSED_DREG64 1
#endif
#ifndef PHP_FUSED_DREG32
#define PHP_FUSED_DREG32 0
#endif

__host__ __device__ constexpr uint32_t align128u(uint32_t b) { return (b + 127u) / 128u * 128u; }

template <typename R>
struct FusedGeom {
    static constexpr int TX = kBlockX, TY = kBlockY;
    static constexpr int HALO = 16 / (int)sizeof(R);
    static constexpr int EX = TX + 2 * HALO, EY = TY + 2; /* E box: x from i0 - HALO, y from j0 - 1 */
    static constexpr int HX = TX + HALO, HY = TY + 1;     /* H box: x from i0 - HALO, y from j0 - 1 */
    static constexpr int QX = TX + 1, QY = TY + 1;        /* new-H tile: x from i0 - 1, y from j0 - 1 */
    static constexpr int TILE = QX * QY;                  /* cells of one component of the tile */
    static constexpr int NHALO = TILE - TX * TY;          /* the 41 cells below the block's own */
    static constexpr uint32_t E_BYTES = EX * EY * sizeof(R), H_BYTES = HX * HY * sizeof(R);
    static constexpr uint32_t D_BYTES = TX * TY * sizeof(R), M_BYTES = TX * TY;
    static constexpr uint32_t EB = align128u(E_BYTES), HB = align128u(H_BYTES), DB = align128u(D_BYTES);
    static constexpr bool DREG = (sizeof(R) == 8 ? PHP_FUSED_DREG64 : PHP_FUSED_DREG32) != 0;
    static constexpr uint32_t STAGE = 3 * EB + 3 * HB + (DREG ? 0u : 3 * DB + align128u(M_BYTES));
    static constexpr int S = sizeof(R) == 8 ? PHP_FUSED_S64 : PHP_FUSED_S32;
    /* plane p's H needs planes p and p + 1 staged, and plane p - 1 + S is
     * issued only after the barrier of plane p: fewer than 3 stages would
     * wait for a plane that is never issued */
    static_assert(S >= 3, "he_sweep_tma needs at least 3 stages");
    /* alignment slack, the stages, two planes of the new-H tile, the stage
     * barriers and the failure-path test's barrier */
    static constexpr uint32_t SMEM = 128 + S * STAGE + 2 * 3 * TILE * sizeof(R) + (S + 1) * 8;
};

/* Loads a block has issued when it stops at plane p: planes k0-1 .. k1, the
 * first S at once, then plane q - 1 + S after the barrier of plane q >= k0. */
__device__ __forceinline__ uint32_t fused_loads_issued(int p, int k0, int k1, int S)
{
    return (uint32_t)(min(k1, max(p, k0) + S - 2) - k0 + 2);
}

/* the six E differences of the curl in the H update (fdtd.c:3132-3137),
 * from E boxes of planes p (b0) and p + 1 (b1) with row length EX */
template <typename R, int EX>
struct HCurl {
    R dEyz, dEzy, dEzx, dExz, dExy, dEyx;
    __device__ __forceinline__ HCurl(const R* Ex0, const R* Ey0, const R* Ez0, const R* Ex1, const R* Ey1, int e)
    {
        const R ex0 = Ex0[e], ey0 = Ey0[e], ez0 = Ez0[e];
        dEyz = Ey1[e] - ey0;
        dEzy = Ez0[e + EX] - ez0;
        dEzx = Ez0[e + 1] - ez0;
        dExz = Ex1[e] - ex0;
        dExy = Ex0[e + EX] - ex0;
        dEyx = Ey0[e + 1] - ey0;
    }
};

/* H of one cell with its CPML terms (the general path of h_sweep_tma):
 * psi holds the old pxy pxz pyx pyz pzx pzy (zero outside the PML); with
 * `store` the new ones go to StepArgs::psin_h (the block's own cells; the
 * cells below the tile are only read) */
template <typename R, int EX>
__device__ __forceinline__ void h_cpml(const StepArgs<R>& a, const HCurl<R, EX>& d, R khx, R khy, R khz, const R* psi,
                                       int sx, int sy, int sz, int i, int j, int k, R& hx, R& hy, R& hz, bool store)
{
    const int L2 = 2 * a.L;
    /* psi terms enter as zeros outside the PML */
    hx = hx + (-khy * d.dEzy + khz * d.dEyz + psi[2] + psi[4]);
    hy = hy + (khx * d.dEzx - khz * d.dExz + psi[0] + psi[5]);
    hz = hz + (-khx * d.dEyx + khy * d.dExy + psi[1] + psi[3]);
    if (!store) return;
    if (sx >= 0) {
        const R bb = ldg_nh(a.tx.b + i), ch = ldg_nh(a.tx.ch + i);
        const int q = (k * a.ny + j) * L2 + sx;
        a.psin_h[0][q] = bb * psi[0] + ch * d.dEzx;
        a.psin_h[1][q] = bb * psi[1] - ch * d.dEyx;
    }
    if (sy >= 0) {
        const R bb = ldg_nh(a.ty.b + j), ch = ldg_nh(a.ty.ch + j);
        const int q = (k * L2 + sy) * a.nxp + i;
        a.psin_h[2][q] = bb * psi[2] - ch * d.dEzy;
        a.psin_h[3][q] = bb * psi[3] + ch * d.dExy;
    }
    if (sz >= 0) {
        const R bb = ldg_nh(a.tz.b + k), ch = ldg_nh(a.tz.ch + k);
        const int q = (sz * a.ny + j) * a.nxp + i;
        a.psin_h[4][q] = bb * psi[4] + ch * d.dEyz;
        a.psin_h[5][q] = bb * psi[5] - ch * d.dExz;
    }
}

/* the old H CPML state of cell (i, j) of plane k into psi[6] */
template <typename R>
__device__ __forceinline__ void h_psi_load(const StepArgs<R>& a, int sx, int sy, int sz, int i, int j, int k, R* psi)
{
    const int L2 = 2 * a.L;
    if (sx >= 0) {
        const int q = (k * a.ny + j) * L2 + sx;
        psi[0] = a.psi.hxy[q];
        psi[1] = a.psi.hxz[q];
    }
    if (sy >= 0) {
        const int q = (k * L2 + sy) * a.nxp + i;
        psi[2] = a.psi.hyx[q];
        psi[3] = a.psi.hyz[q];
    }
    if (sz >= 0) {
        const int q = (sz * a.ny + j) * a.nxp + i;
        psi[4] = a.psi.hzx[q];
        psi[5] = a.psi.hzy[q];
    }
}

template <typename R, int NAMAX>
__global__ void __launch_bounds__(kBlockX * kBlockY, (NAMAX > 4 ? 1 : sizeof(R) == 8 ? PHP_FUSED_MINB64 : PHP_FUSED_MINB32))
    he_sweep_tma(const __grid_constant__ StepArgs<R> a, const __grid_constant__ TmaMaps tm)
{
    using G = FusedGeom<R>;
    constexpr int S = G::S;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* smem = ring_base(dyn_smem);
    R* tile = reinterpret_cast<R*>(smem + S * G::STAGE); /* [plane & 1][x, y, z][TILE] */
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * G::STAGE + 2 * 3 * G::TILE * sizeof(R));

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * G::TX + tx;
    const int i0 = blockIdx.x * G::TX, j0 = blockIdx.y * G::TY;
    const int i = i0 + tx, j = j0 + ty;
    const int bz = blockIdx.z + a.zc0;
    const int k0 = bz * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return; /* uniform over the block */
    const size_t blk = ((size_t)bz * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;

    /* plane p = k0-1 .. k1 into stage (p - k0 + 1) % S: E of planes >= 0, H of
     * planes 0 .. k1-1, D and ids of the chunk's planes; plane -1 (k0 = 0)
     * loads nothing and completes its barrier at once */
    auto stage = [&](int p) -> unsigned char* { return smem + (uint32_t)((p - k0 + 1) % S) * G::STAGE; };
    auto issue = [&](int p) {
        const int g = p - k0 + 1;
        uint64_t* bar = &full[g % S];
        unsigned char* b = smem + (uint32_t)(g % S) * G::STAGE;
        const bool e_box = p >= 0, h_box = p >= 0 && p < k1, own = !G::DREG && p >= k0 && p < k1;
        mbar_arrive_expect_tx(bar, (e_box ? 3 * G::E_BYTES : 0u) + (h_box ? 3 * G::H_BYTES : 0u) +
                                       (own ? 3 * G::D_BYTES + G::M_BYTES : 0u));
        if (e_box)
            for (int q = 0; q < 3; ++q) tma_load_3d(b + q * G::EB, &tm.e_wide[q], bar, i0 - G::HALO, j0 - 1, p + 1);
        if (h_box)
            for (int q = 0; q < 3; ++q)
                tma_load_3d(b + 3 * G::EB + q * G::HB, &tm.h_halo[q], bar, i0 - G::HALO, j0 - 1, p + 1);
        if (own) {
            for (int q = 0; q < 3; ++q)
                tma_load_3d(b + 3 * G::EB + 3 * G::HB + q * G::DB, &tm.d_own[q], bar, i0, j0, p + 1);
            tma_load_3d(b + 3 * G::EB + 3 * G::HB + 3 * G::DB, &tm.mat, bar, i0, j0, p);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < S + 1; ++s) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int p = k0 - 1; p <= min(k1, k0 - 1 + S - 1); ++p) issue(p);
    if (a.stall_test && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
        /* failure-path test (StepArgs::stall_test), as in h_sweep_tma */
        const bool ok = mbar_wait_n(&full[S], 0, kStallPolls);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                ring_drain(full, S, fused_loads_issued(k0 - 1, k0, k1, S));
            }
            return;
        }
    }

    /* block classes: the H part (plain or with CPML terms) and the E part
     * (the plain-block codes of StepArgs::plain_blk) */
    const bool hplain = a.plain_hf && a.plain_hf[blk];
    const int pm = a.plain_blk ? a.plain_blk[blk] : 255;

    const bool e_active = (i < a.nx) && (j < a.ny);
    const bool interior = (i >= 1 && i < a.nx - 1 && j >= 1 && j < a.ny - 1);
    const bool h_active = (i < a.nx - 1) && (j < a.ny - 1);
    const int slot_i = e_active ? ldg(a.tx.slot + i) : -1;
    const int slot_j = e_active ? ldg(a.ty.slot + j) : -1;
    const int sxh = h_active ? slot_i : -1, syh = h_active ? slot_j : -1;
    R khx = R(0), khy = R(0);
    if (!hplain && h_active) {
        khx = ldg(a.tx.kh + i);
        khy = ldg(a.ty.kh + j);
    }
    /* the cell below the tile this thread computes H of as well (tid < 41):
     * the row j0 - 1 from i0 - 1, then the column i0 - 1 */
    const int ci = tid < G::QX ? i0 - 1 + tid : i0 - 1;
    const int cj = tid < G::QX ? j0 - 1 : j0 + tid - G::QX;
    const bool halo = tid < G::NHALO && ci >= 0 && cj >= 0 && ci < a.nx && cj < a.ny;
    const bool halo_upd = halo && ci < a.nx - 1 && cj < a.ny - 1;

    /* offsets of the own cell in the boxes and the tile, of the halo cell */
    const int eo = (ty + 1) * G::EX + tx + G::HALO;
    const int ho = (ty + 1) * G::HX + tx + G::HALO;
    const int oo = ty * G::TX + tx;
    const int to = (ty + 1) * G::QX + tx + 1;
    const int ce = (cj - j0 + 1) * G::EX + (ci - i0 + G::HALO);
    const int ch = (cj - j0 + 1) * G::HX + (ci - i0 + G::HALO);
    const int ct = (cj - j0 + 1) * G::QX + (ci - i0 + 1);

    constexpr uint32_t HBW = G::HB / sizeof(R), DBW = G::DB / sizeof(R);
    constexpr bool kInc = sizeof(R) == 4;
    /* pool slot of the cell one plane ahead in the general path (FP32, as
     * e_sweep_tma) */
    const bool slots = PHP_SLOT_AHEAD && sizeof(R) == 4 && pm == 255 && a.slot != nullptr && e_active;
    int slot_next = slots ? ldg(a.slot + (k0 * a.ny + j) * a.nxp + i) : -1;

    R hxk = R(0), hyk = R(0); /* new H of the own cell at plane p - 1 */
    for (int p = k0 - 1; p < k1; ++p) {
        const bool eph = p >= k0; /* D and E of plane p this pass */
        const int c = (p * a.ny + j) * a.nxp + i;
        /* state that does not depend on the stages, read before the wait:
         * the own cell's H CPML state (old level) and D CPML state */
        R psi[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
        int szh = -1;
        if (!hplain && p >= 0) {
            szh = ldg_nh(a.tz.slot + p);
            if (h_active) h_psi_load(a, sxh, syh, szh, i, j, p, psi);
        }
        CellPsi<R> ps;
        ps.sz = -1;
        if (eph && pm >= kPlainCpml && interior) load_psi_d(a, i, j, p, slot_i, slot_j, ps);
        R d0 = R(0), d1 = R(0), d2 = R(0);
        int mid = 0;
        if (G::DREG && eph && e_active) {
            d0 = a.f.dx[c];
            d1 = a.f.dy[c];
            d2 = a.f.dz[c];
            if (pm == 255) mid = a.mat[c];
        }
        IonPre ip;
        ip.slot = -1;
        if (eph && slots) {
            ip.slot = slot_next;
            if (p + 1 < k1) slot_next = ldg(a.slot + ((p + 1) * a.ny + j) * a.nxp + i);
            if (ip.slot >= 0) {
                const int64_t ns = a.nslot;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    if (a.P) {
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.P + q * ns + ip.slot));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.Po + q * ns + ip.slot));
                    }
                    if (NAMAX == 0 && a.pr) asm volatile("prefetch.global.L1 [%0];" ::"l"(a.pr + q * ns + ip.slot));
                }
            }
        }
        if constexpr (NAMAX > 0 && NAMAX <= 4) {
            if (eph && pm == kPlainAtoms && e_active) {
                /* the few-atom cell's slot, and its r and v into L1 */
                constexpr int QN = 3 * NAMAX;
                constexpr bool VREG = QN * (int)sizeof(R) <= kIonRegBytesR<R>;
                const int n3 = 3 * a.amc.natom;
                ip.slot = a.slot[c];
#pragma unroll
                for (int q = 0; q < QN; ++q) {
                    const int64_t o = VREG ? (int64_t)((uint32_t)q * (uint32_t)a.nslot + (uint32_t)ip.slot)
                                           : (int64_t)q * a.nslot + ip.slot;
                    if (q < n3) {
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.r + o));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.v + o));
                    }
                }
            }
        }

        bool ok = true;
        if (p == k0 - 1) ok = mbar_wait(&full[0], 0);
        {
            const int g = p - k0 + 2;
            ok = ok && mbar_wait(&full[g % S], (g / S) & 1);
        }

        /* ---- H of plane p: the own cell, and the cell below the tile */
        R hx = R(0), hy = R(0), hz = R(0); /* plane -1: the zero halo plane */
        R* tb = tile + (p & 1) * 3 * G::TILE;
        if (ok && p >= 0) {
            const unsigned char* b0 = stage(p);
            const unsigned char* b1 = stage(p + 1);
            const R* Ex0 = reinterpret_cast<const R*>(b0);
            const R* Ey0 = reinterpret_cast<const R*>(b0 + G::EB);
            const R* Ez0 = reinterpret_cast<const R*>(b0 + 2 * G::EB);
            const R* Ex1 = reinterpret_cast<const R*>(b1);
            const R* Ey1 = reinterpret_cast<const R*>(b1 + G::EB);
            const R* Hb = reinterpret_cast<const R*>(b0 + 3 * G::EB);
            hx = Hb[ho];
            hy = Hb[HBW + ho];
            hz = Hb[2 * HBW + ho];
            if (hplain) {
                const R kx = a.khp[0], ky = a.khp[1], kz = a.khp[2];
                const HCurl<R, G::EX> d(Ex0, Ey0, Ez0, Ex1, Ey1, eo);
                hx = hx + (-ky * d.dEzy + kz * d.dEyz);
                hy = hy + (kx * d.dEzx - kz * d.dExz);
                hz = hz + (-kx * d.dEyx + ky * d.dExy);
            } else if (h_active) {
                const HCurl<R, G::EX> d(Ex0, Ey0, Ez0, Ex1, Ey1, eo);
                h_cpml(a, d, khx, khy, ldg_nh(a.tz.kh + p), psi, sxh, syh, szh, i, j, p, hx, hy, hz, eph);
            }
            if (eph) {
                if (e_active) {
                    a.hnew[0][c] = hx;
                    a.hnew[1][c] = hy;
                    a.hnew[2][c] = hz;
                }
                tb[to] = hx;
                tb[G::TILE + to] = hy;
                tb[2 * G::TILE + to] = hz;
                if (halo) {
                    R qx = Hb[ch], qy = Hb[HBW + ch], qz = Hb[2 * HBW + ch];
                    if (hplain) {
                        const R kx = a.khp[0], ky = a.khp[1], kz = a.khp[2];
                        const HCurl<R, G::EX> d(Ex0, Ey0, Ez0, Ex1, Ey1, ce);
                        qx = qx + (-ky * d.dEzy + kz * d.dEyz);
                        qy = qy + (kx * d.dEzx - kz * d.dExz);
                        qz = qz + (-kx * d.dEyx + ky * d.dExy);
                    } else if (halo_upd) {
                        const int hsx = ldg(a.tx.slot + ci), hsy = ldg(a.ty.slot + cj);
                        R hpsi[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
                        h_psi_load(a, hsx, hsy, szh, ci, cj, p, hpsi);
                        const HCurl<R, G::EX> d(Ex0, Ey0, Ez0, Ex1, Ey1, ce);
                        h_cpml(a, d, ldg(a.tx.kh + ci), ldg(a.ty.kh + cj), ldg_nh(a.tz.kh + p), hpsi, hsx, hsy, szh,
                               ci, cj, p, qx, qy, qz, false);
                    }
                    tb[ct] = qx;
                    tb[G::TILE + ct] = qy;
                    tb[2 * G::TILE + ct] = qz;
                }
            }
        }
        /* every thread is done with plane p - 1 and has written the tile of
         * plane p: plane p - 1's stage takes plane p - 1 + S */
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                ring_drain(full, S, fused_loads_issued(p, k0, k1, S));
            }
            break;
        }
        if (tid == 0 && eph && p - 1 + S <= k1) {
            fence_proxy_async_smem();
            issue(p - 1 + S);
        }

        /* ---- D and E of plane p */
        if (eph && e_active) {
            const unsigned char* bc = stage(p);
            const R* Eo = reinterpret_cast<const R*>(bc);
            const R hz_jm = tb[2 * G::TILE + to - G::QX], hx_jm = tb[to - G::QX];
            const R hz_im = tb[2 * G::TILE + to - 1], hy_im = tb[G::TILE + to - 1];
            if constexpr (!G::DREG) {
                const R* Ds = reinterpret_cast<const R*>(bc + 3 * G::EB + 3 * G::HB);
                d0 = Ds[oo];
                d1 = Ds[DBW + oo];
                d2 = Ds[2 * DBW + oo];
                mid = reinterpret_cast<const uint8_t*>(bc + 3 * G::EB + 3 * G::HB + 3 * G::DB)[oo];
            }
            R dx = d0, dy = d1, dz = d2;
            R ex, ey, ez;
            if (pm == 255) {
                e_cell_values<R, false, NAMAX>(a, i, j, p, c, interior, slot_i, slot_j, hx, hy, hz, hxk, hyk, hz_jm,
                                               hx_jm, hz_im, hy_im, dx, dy, dz, mid, nullptr, &ps, ex, ey, ez,
                                               slots ? &ip : nullptr);
            } else if (pm < kPlainCpml) {
                /* one plain material, no CPML, edge or source cell */
                const R iso = a.iso[pm];
                const R kdx = a.kdp[0], kdy = a.kdp[1], kdz = a.kdp[2];
                const R dHzy = hz - hz_jm, dHyz = hy - hyk, dHxz = hx - hxk;
                const R dHzx = hz - hz_im, dHyx = hy - hy_im, dHxy = hx - hx_jm;
                const R ux = kdy * dHzy - kdz * dHyz;
                const R uy = -kdx * dHzx + kdz * dHxz;
                const R uz = kdx * dHyx - kdy * dHxy;
                dx = dx + ux;
                dy = dy + uy;
                dz = dz + uz;
                ex = iso * dx;
                ey = iso * dy;
                ez = iso * dz;
            } else {
                R ix = R(0), iy = R(0), iz = R(0);
                R& ux = kInc ? ix : dx;
                R& uy = kInc ? iy : dy;
                R& uz = kInc ? iz : dz;
                if (pm < kPlainTensor) {
                    /* one plain material with CPML or domain-edge cells */
                    if (interior)
                        d_update<R, false>(a, i, j, p, slot_i, slot_j, hx, hy, hz, hxk, hyk, hz_jm, hx_jm, hz_im, hy_im,
                                           ps, ux, uy, uz);
                    if constexpr (kInc) {
                        dx += ix;
                        dy += iy;
                        dz += iz;
                    }
                    const R iso = a.iso[pm - kPlainCpml];
                    ex = iso * dx;
                    ey = iso * dy;
                    ez = iso * dz;
                } else if (pm == kPlainTensor) {
                    /* the one lossy or anisotropic material of StepArgs::tns_* */
                    const int fl = a.tns_flags;
                    R e0 = R(0), e1 = R(0), e2 = R(0);
                    if (interior && (fl & kLossy)) {
                        e0 = Eo[eo];
                        e1 = Eo[G::EB / sizeof(R) + eo];
                        e2 = Eo[2 * (G::EB / sizeof(R)) + eo];
                    }
                    if (interior) {
                        d_update<R, false>(a, i, j, p, slot_i, slot_j, hx, hy, hz, hxk, hyk, hz_jm, hx_jm, hz_im, hy_im,
                                           ps, ux, uy, uz);
                        if (fl & kLossy) { /* fdtd.c:3349-3353 */
                            const R* q = a.tns_im;
                            ux -= q[0] * e0 + q[1] * e1 + q[2] * e2;
                            uy -= q[3] * e0 + q[4] * e1 + q[5] * e2;
                            uz -= q[6] * e0 + q[7] * e1 + q[8] * e2;
                        }
                    }
                    if constexpr (kInc) {
                        dx += ix;
                        dy += iy;
                        dz += iz;
                    }
                    /* fdtd.c:3429-3461, 3486-3503 */
                    R da = dx, db = dy, dc = dz;
                    rot_fwd<false>(fl, a.tns_cs, a.tns_sn, da, db, dc);
                    const R* E = a.tns_inv;
                    ex = E[0] * da + E[1] * db + E[2] * dc;
                    ey = E[3] * da + E[4] * db + E[5] * dc;
                    ez = E[6] * da + E[7] * db + E[8] * dc;
                    rot_back<false>(fl, a.tns_cs, a.tns_sn, ex, ey, ez);
                } else {
                    /* the few-atom material of StepArgs::amc (kPlainAtoms) */
                    if constexpr (NAMAX > 0 && NAMAX <= 4) {
                        const MatCoef<R>& m = a.amc;
                        const bool lossy = (m.flags & kLossy) != 0;
                        ex = ey = ez = R(0);
                        if (interior && lossy) {
                            ex = Eo[eo];
                            ey = Eo[G::EB / sizeof(R) + eo];
                            ez = Eo[2 * (G::EB / sizeof(R)) + eo];
                        }
                        if (interior) {
                            d_update<R, false>(a, i, j, p, slot_i, slot_j, hx, hy, hz, hxk, hyk, hz_jm, hx_jm, hz_im,
                                               hy_im, ps, ux, uy, uz);
                            if (lossy) { /* fdtd.c:3349-3353 */
                                const R* q = m.eps_im;
                                ux -= q[0] * ex + q[1] * ey + q[2] * ez;
                                uy -= q[3] * ex + q[4] * ey + q[5] * ez;
                                uz -= q[6] * ex + q[7] * ey + q[8] * ez;
                            }
                        }
                        if constexpr (kInc) {
                            dx += ix;
                            dy += iy;
                            dz += iz;
                        }
                        e_update<R, false, NAMAX>(a, m, c, dx, dy, dz, ix, iy, iz, ex, ey, ez, &ip);
                    } else {
                        ex = ey = ez = R(0); /* no such blocks without the fused ion update */
                    }
                }
            }
            a.f.dx[c] = dx;
            a.f.dy[c] = dy;
            a.f.dz[c] = dz;
            a.enew[0][c] = ex;
            a.enew[1][c] = ey;
            a.enew[2][c] = ez;
        }
        hxk = hx;
        hyk = hy;
    }
    if (a.ndft) dft_fold(a, a.enew, i, j, k0, k1); /* the new E */
    if (a.probe_rows) probe_fold(a, a.enew, a.hnew, i, j, k0, k1);
}

} // namespace phpdev
