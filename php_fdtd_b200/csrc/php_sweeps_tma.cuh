/*
 * php_sweeps_tma.cuh -- the two sweeps with a TMA plane pipeline (sm_100a).
 *
 * A block owns a 32 x 8 (x, y) tile of a z chunk.  One thread streams whole
 * planes of the tile into a ring of kTmaStages shared-memory stages with
 * cp.async.bulk.tensor (tile mode, no multicast: every byte comes from this
 * GPU's own memory), each stage completed on its own mbarrier; all 256
 * threads compute from shared memory.  The bytes in flight are set by the
 * ring depth instead of by registers, which is what a streaming stencil on
 * HBM needs.
 *
 *   h_sweep_tma: per plane, Ex/Ey/Ez with a +1 halo in x and y (the box is
 *     widened to 16 bytes in x) and Hx/Hy/Hz of the tile; the update at k
 *     reads E planes k and k+1.
 *   e_sweep_tma: per plane, Hx/Hy/Hz with a -1 halo in x and y (the box starts
 *     16 bytes left of the tile so that its x offset stays 16-byte aligned),
 *     Dx/Dy/Dz and the material ids of the tile; the update at k reads H planes
 *     k and k-1.
 * Out-of-range parts of a box read the tensor map's zero fill; those values
 * are only used by cells the reference never updates there (i = nx-1 or
 * j = ny-1 for H, the x/y border for D).
 *
 * Waits on the mbarriers are bounded: after kWaitLimit polls the block sets
 * a device error flag and leaves the loop (the decision is made uniform
 * across the block with __syncthreads_or), and the host reports
 * PHP_ERR_TIMEOUT.
 */
#pragma once

#include <cuda.h>

namespace phpdev {

constexpr int kTmaStages = 4;
constexpr uint32_t kWaitLimit = 1u << 24;

/* tuning: ring depth of the FP64 fused sweep, and whether the CPML state is
 * read before the stage wait (1) or after it (0), per sweep and precision */
#ifndef PHP_TMA_ES64
#define PHP_TMA_ES64 3
#endif
#ifndef PHP_TMA_ES32
#define PHP_TMA_ES32 4
#endif
#ifndef PHP_TMA_HS
#define PHP_TMA_HS 4
#endif
#ifndef PHP_PSI_EARLY_H64
#define PHP_PSI_EARLY_H64 1
#endif
/* FP32 H sweep: early since its CPML coefficients are loaded once per column
 * (256^3 tip workload H 0.1223 -> 0.1191 ms, 192^3 two-atom 0.0684 -> 0.0661
 * ms; before that, late measured faster) */
#ifndef PHP_PSI_EARLY_H32
#define PHP_PSI_EARLY_H32 1
#endif
/* resident blocks the fused sweep is compiled for (register budget), FP64
 * and FP32 */
#ifndef PHP_E_MINBLOCKS
#define PHP_E_MINBLOCKS 4
#endif
#ifndef PHP_E_MINBLOCKS32
#define PHP_E_MINBLOCKS32 4
#endif
#ifndef PHP_PSI_EARLY_E
#define PHP_PSI_EARLY_E 1
#endif
/* the CPML loops request the psi lines of the next plane into L1: both H
 * sweeps and the FP64 fused sweep (the FP32 fused sweep measured slower) */
#ifndef PHP_PSI_AHEAD
#define PHP_PSI_AHEAD 1
#endif
#ifndef PHP_PSI_AHEAD_E32
#define PHP_PSI_AHEAD_E32 0
#endif
#ifndef PHP_PSI_AHEAD_H32
#define PHP_PSI_AHEAD_H32 1
#endif
/* the tensor and few-atom blocks of the fused sweep request the next plane's
 * old E lines into L1 (256^3 tip workload: FP64 E 0.3386 -> 0.3335 ms, FP32
 * 0.2055 -> 0.2039 ms) */
#ifndef PHP_EOLD_AHEAD
#define PHP_EOLD_AHEAD 1
#endif
/* the general path (FP32, where pool slots are read a plane ahead) requests
 * the old E lines of its pooled cells before the stage wait (256^3 tip
 * workload: FP32 E 0.2041 -> 0.2019 ms) */
#ifndef PHP_EOLD_AHEAD_GEN
#define PHP_EOLD_AHEAD_GEN 1
#endif
/* the general path of the FP32 fused sweep reads pool slots one plane ahead
 * (in FP64 the extra live values spill) */
#ifndef PHP_SLOT_AHEAD
#define PHP_SLOT_AHEAD 1
#endif

template <typename R>
constexpr bool kPsiAheadE = PHP_PSI_AHEAD && (sizeof(R) == 8 || PHP_PSI_AHEAD_E32);

/* Tensor maps of the device arrays (3-D: x, y, plane; planes count from the
 * low halo plane of the field arrays). */
struct TmaMaps {
    CUtensorMap e_halo[3]; /* Ex, Ey, Ez: box (32 + 16/s) x 9 at (i0, j0) */
    CUtensorMap h_own[3];  /* Hx, Hy, Hz: box 32 x 8 */
    CUtensorMap h_halo[3]; /* Hx, Hy, Hz: box (32 + 16/s) x 9 at (i0 - 16/s, j0 - 1) */
    CUtensorMap d_own[3];  /* Dx, Dy, Dz: box 32 x 8 */
    CUtensorMap mat;       /* uint8 ids (no halo planes): box 32 x 8 */
    CUtensorMap e_wide[3]; /* Ex, Ey, Ez: box (32 + 32/s) x 10 at (i0 - 16/s, j0 - 1), he_sweep_tma */
};

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n"
        "  .reg .pred p;\n"
        "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "  selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

/* bounded wait: false after `limit` polls (kWaitLimit by default) */
__device__ __forceinline__ bool mbar_wait_n(uint64_t* bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t n = 0; n < limit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    return mbar_wait_n(bar, parity, kWaitLimit);
}

/* After a bounded wait gave up: waits (bounded again) for the block's plane
 * loads that may still be in flight -- at most the last S of the `issued`
 * loads, load g in stage g % S with phase parity (g / S) & 1, since a load
 * is only issued into a stage whose previous load every thread has
 * consumed -- so that none lands in shared memory after the block left. */
__device__ __forceinline__ void ring_drain(uint64_t* full, int S, uint32_t issued)
{
    const uint32_t first = issued > (uint32_t)S ? issued - (uint32_t)S : 0u;
    for (uint32_t g = first; g < issued; ++g) mbar_wait(&full[g % S], (g / S) & 1u);
}

/* Loads a block has issued when it stops after plane k: the H sweep loads
 * planes k0..k1 (the first S at once, then plane j + S after plane j), the
 * fused sweep planes k0-1..k1-1 (then plane j - 1 + S after plane j). */
__device__ __forceinline__ uint32_t h_loads_issued(int k, int k0, int k1, int S)
{
    return (uint32_t)(min(k1, k + S - 1) - k0 + 1);
}
__device__ __forceinline__ uint32_t e_loads_issued(int k, int k0, int k1, int S)
{
    return (uint32_t)(min(k1 - 1, k + S - 2) - k0 + 2);
}

/* polls of the failure-path test's wait on a barrier nothing arrives on */
constexpr uint32_t kStallPolls = 1u << 12;

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

/* orders this thread's generic-proxy accesses to shared memory before the
 * async-proxy (TMA) writes it issues next */
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

template <typename R>
struct TmaGeom {
    static constexpr int TX = kBlockX, TY = kBlockY;
    static constexpr int HALO = 16 / (int)sizeof(R);      /* x halo widened to 16 bytes */
    static constexpr int BX = TX + HALO, BY = TY + 1;      /* halo box */
    static constexpr int HALO_ELEMS = BX * BY, OWN_ELEMS = TX * TY;
    static constexpr uint32_t HALO_BYTES = HALO_ELEMS * sizeof(R), OWN_BYTES = OWN_ELEMS * sizeof(R);
    static constexpr uint32_t MAT_BYTES = OWN_ELEMS;
    __host__ __device__ static constexpr uint32_t align128(uint32_t b) { return (b + 127u) / 128u * 128u; }
    /* H sweep stage: 3 halo E boxes + 3 own H boxes */
    static constexpr uint32_t H_STAGE = align128(3 * align128(HALO_BYTES) + 3 * align128(OWN_BYTES));
    /* E sweep stage: 3 halo H boxes + 3 own D boxes + material ids */
    static constexpr uint32_t E_STAGE = align128(3 * align128(HALO_BYTES) + 3 * align128(OWN_BYTES) + align128(MAT_BYTES));
    /* ring depths: 4 planes, 3 for the FP64 fused sweep so that four
     * blocks (with their material records) fit in one SM's shared memory */
    static constexpr int HS = PHP_TMA_HS;
    static constexpr int ES = sizeof(R) == 8 ? PHP_TMA_ES64 : PHP_TMA_ES32;
    /* dynamic shared memory: 128 bytes of alignment slack, the stages, then
     * the stage barriers */
    static constexpr uint32_t H_SMEM = 128 + HS * H_STAGE + (HS + 1) * 8; /* + the failure-path test's barrier */
    /* the fused sweep adds its material records after 128 bytes of barriers:
     * E_SMEM + nmat * sizeof(MatCoef<R>) */
    static constexpr uint32_t E_SMEM = 128 + ES * E_STAGE + 128;
};

/* 128-byte aligned start of the stage ring inside dynamic shared memory */
__device__ __forceinline__ unsigned char* ring_base(unsigned char* dyn)
{
    const uint32_t a = smem_addr(dyn);
    return dyn + ((128u - (a & 127u)) & 127u);
}

/* ================================================================ H sweep */

/* fdtd.c:3123-3231: cells i < nx-1, j < ny-1, all k.  Compiled for the
 * resident blocks per SM that shared memory allows: six in FP32, four in
 * FP64. */
#ifndef PHP_H_MINBLOCKS32
#define PHP_H_MINBLOCKS32 6
#endif
template <typename R, bool STRICT>
__global__ void __launch_bounds__(kBlockX * kBlockY, sizeof(R) == 4 ? PHP_H_MINBLOCKS32 : 4) h_sweep_tma(const __grid_constant__ StepArgs<R> a,
                                                                 const __grid_constant__ TmaMaps tm)
{
    using G = TmaGeom<R>;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* smem = ring_base(dyn_smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::HS * G::H_STAGE);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * G::TX + tx;
    const int i0 = blockIdx.x * G::TX, j0 = blockIdx.y * G::TY;
    const int i = i0 + tx, j = j0 + ty;
    const int bz = blockIdx.z + a.zc0;
    const int k0 = bz * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return; /* uniform over the block */

    constexpr uint32_t EB = G::align128(G::HALO_BYTES), HB = G::align128(G::OWN_BYTES);
    auto stage = [&](int p) -> unsigned char* { return smem + (uint32_t)((p - k0) % G::HS) * G::H_STAGE; };
    /* plane p = k0..k1: E (halo boxes) of every plane, H of planes < k1 */
    auto issue = [&](int p) {
        uint64_t* bar = &full[(p - k0) % G::HS];
        unsigned char* b = stage(p);
        const bool with_h = p < k1;
        mbar_arrive_expect_tx(bar, 3 * G::HALO_BYTES + (with_h ? 3 * G::OWN_BYTES : 0u));
        for (int q = 0; q < 3; ++q) tma_load_3d(b + q * EB, &tm.e_halo[q], bar, i0, j0, p + 1);
        if (with_h)
            for (int q = 0; q < 3; ++q) tma_load_3d(b + 3 * EB + q * HB, &tm.h_own[q], bar, i0, j0, p + 1);
    };

    if (tid == 0) {
        for (int s = 0; s < G::HS + 1; ++s) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int p = k0; p <= min(k1, k0 + G::HS - 1); ++p) issue(p);
    if (a.stall_test && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
        /* failure-path test (StepArgs::stall_test): a bounded wait on the
         * barrier after the ring's, on which nothing ever arrives, gives up
         * like a wait for a plane that never lands */
        const bool ok = mbar_wait_n(&full[G::HS], 0, kStallPolls);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                ring_drain(full, G::HS, h_loads_issued(k0, k0, k1, G::HS));
            }
            return;
        }
    }

    const int eo = ty * G::BX + tx; /* own cell in a halo box */
    const int ho = ty * G::TX + tx; /* own cell in an own box */

    /* a plain block (no CPML cell, every cell updated; marked on the host):
     * the stencil with the kappa = 1 factors only, the same arithmetic as the
     * general path below takes for such cells */
    if (!STRICT && a.plain_h && a.plain_h[((size_t)bz * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x]) {
        const R khx = a.khp[0], khy = a.khp[1], khz = a.khp[2];
        for (int k = k0; k < k1; ++k) {
            bool ok = true;
            if (k == k0) ok = mbar_wait(&full[0], 0);
            ok = ok && mbar_wait(&full[(k + 1 - k0) % G::HS], ((k + 1 - k0) / G::HS) & 1);
            if (ok) {
                const unsigned char* b0 = stage(k);
                const unsigned char* b1 = stage(k + 1);
                const R* Ex0 = reinterpret_cast<const R*>(b0);
                const R* Ey0 = reinterpret_cast<const R*>(b0 + EB);
                const R* Ez0 = reinterpret_cast<const R*>(b0 + 2 * EB);
                const R* Ex1 = reinterpret_cast<const R*>(b1);
                const R* Ey1 = reinterpret_cast<const R*>(b1 + EB);
                const R* Hs = reinterpret_cast<const R*>(b0 + 3 * EB);
                const R ex0 = Ex0[eo], ey0 = Ey0[eo], ez0 = Ez0[eo];
                const R dEyz = Ey1[eo] - ey0, dEzy = Ez0[eo + G::BX] - ez0, dEzx = Ez0[eo + 1] - ez0;
                const R dExz = Ex1[eo] - ex0, dExy = Ex0[eo + G::BX] - ex0, dEyx = Ey0[eo + 1] - ey0;
                const int c = (k * a.ny + j) * a.nxp + i;
                a.f.hx[c] = Hs[ho] + (-khy * dEzy + khz * dEyz);
                a.f.hy[c] = Hs[HB / sizeof(R) + ho] + (khx * dEzx - khz * dExz);
                a.f.hz[c] = Hs[2 * (HB / sizeof(R)) + ho] + (-khx * dEyx + khy * dExy);
            }
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(a.err, 1);
                    ring_drain(full, G::HS, h_loads_issued(k, k0, k1, G::HS));
                }
                break;
            }
            if (tid == 0 && k + G::HS <= k1) {
                fence_proxy_async_smem();
                issue(k + G::HS);
            }
        }
        return;
    }

    const bool active = (i < a.nx - 1) && (j < a.ny - 1);
    const int L2 = 2 * a.L;
    const int nxp = a.nxp, ny = a.ny;
    const int sx = active ? ldg(a.tx.slot + i) : -1;
    const int sy = active ? ldg(a.ty.slot + j) : -1;
    R khx = R(0), khy = R(0);
    /* the column's CPML coefficients (fast form), loaded once: FP32 H 0.1233
     * -> 0.1223 ms on the 256^3 tip workload, FP64 unchanged */
    R bx = R(0), chx = R(0), by = R(0), chy = R(0);
    if constexpr (!STRICT) {
        if (active) {
            khx = ldg(a.tx.kh + i);
            khy = ldg(a.ty.kh + j);
        }
        if (sx >= 0) {
            bx = ldg(a.tx.b + i);
            chx = ldg(a.tx.ch + i);
        }
        if (sy >= 0) {
            by = ldg(a.ty.b + j);
            chy = ldg(a.ty.ch + j);
        }
    }
    R* __restrict__ hxg = a.f.hx;
    R* __restrict__ hyg = a.f.hy;
    R* __restrict__ hzg = a.f.hz;

    for (int k = k0; k < k1; ++k) {
        /* CPML state and per-plane values do not depend on the staged planes:
         * issue their loads first so their latency overlaps the wait */
        constexpr bool early = sizeof(R) == 8 ? PHP_PSI_EARLY_H64 : PHP_PSI_EARLY_H32;
        const int sz = ldg_nh(a.tz.slot + k);
        R pxy = R(0), pxz = R(0), pyx = R(0), pyz = R(0), pzx = R(0), pzy = R(0);
        const int qx = (k * ny + j) * L2 + sx, qy = (k * L2 + sy) * nxp + i, qz = (sz * ny + j) * nxp + i;
        auto load_psi = [&]() {
            if (active) {
                if (sx >= 0) { pxy = a.psi.hxy[qx]; pxz = a.psi.hxz[qx]; }
                if (sy >= 0) { pyx = a.psi.hyx[qy]; pyz = a.psi.hyz[qy]; }
                if (sz >= 0) { pzx = a.psi.hzx[qz]; pzy = a.psi.hzy[qz]; }
            }
        };
        if constexpr (early) load_psi();
        if (PHP_PSI_AHEAD && (sizeof(R) == 8 || PHP_PSI_AHEAD_H32) && !STRICT && active && k + 1 < k1) {
            /* the lines of plane k + 1 requested into L1 a plane ahead */
            const int sz1 = ldg_nh(a.tz.slot + k + 1);
            if (sx >= 0) {
                const int q = ((k + 1) * ny + j) * L2 + sx;
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.hxy + q));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.hxz + q));
            }
            if (sy >= 0) {
                const int q = ((k + 1) * L2 + sy) * nxp + i;
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.hyx + q));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.hyz + q));
            }
            if (sz1 >= 0) {
                const int q = (sz1 * ny + j) * nxp + i;
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.hzx + q));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.psi.hzy + q));
            }
        }
        R khz = R(0), bz = R(0), chz = R(0); /* the plane's, before the wait */
        if constexpr (!STRICT) {
            khz = ldg_nh(a.tz.kh + k);
            if (sz >= 0) {
                bz = ldg_nh(a.tz.b + k);
                chz = ldg_nh(a.tz.ch + k);
            }
        }

        bool ok = true;
        if (k == k0) ok = mbar_wait(&full[0], 0);
        ok = ok && mbar_wait(&full[(k + 1 - k0) % G::HS], ((k + 1 - k0) / G::HS) & 1);
        if constexpr (!early) load_psi();
        if (ok && active) {
            const unsigned char* b0 = stage(k);
            const unsigned char* b1 = stage(k + 1);
            const R* Ex0 = reinterpret_cast<const R*>(b0);
            const R* Ey0 = reinterpret_cast<const R*>(b0 + EB);
            const R* Ez0 = reinterpret_cast<const R*>(b0 + 2 * EB);
            const R* Ex1 = reinterpret_cast<const R*>(b1);
            const R* Ey1 = reinterpret_cast<const R*>(b1 + EB);
            const R* Hx0 = reinterpret_cast<const R*>(b0 + 3 * EB);
            const R* Hy0 = reinterpret_cast<const R*>(b0 + 3 * EB + HB);
            const R* Hz0 = reinterpret_cast<const R*>(b0 + 3 * EB + 2 * HB);
            const R ex0 = Ex0[eo], ey0 = Ey0[eo], ez0 = Ez0[eo];
            const R ex1 = Ex1[eo], ey1 = Ey1[eo];
            const R ezi = Ez0[eo + 1], eyi = Ey0[eo + 1];
            const R ezj = Ez0[eo + G::BX], exj = Ex0[eo + G::BX];
            const R hx0 = Hx0[ho], hy0 = Hy0[ho], hz0 = Hz0[ho];
            const int c = (k * ny + j) * nxp + i;
            if constexpr (STRICT) {
                const double mu0 = a.mu0;
                /* fdtd.c:3132-3137 */
                const double dEy_dz = SOp::div(SOp::sub(ey1, ey0), a.dzs);
                const double dEz_dy = SOp::div(SOp::sub(ezj, ez0), a.dys);
                const double dEz_dx = SOp::div(SOp::sub(ezi, ez0), a.dxs);
                const double dEx_dz = SOp::div(SOp::sub(ex1, ex0), a.dzs);
                const double dEx_dy = SOp::div(SOp::sub(exj, ex0), a.dys);
                const double dEy_dx = SOp::div(SOp::sub(eyi, ey0), a.dxs);
                double kappa_x = 1.0, kappa_y = 1.0, kappa_z = 1.0;
                if (sx >= 0) { /* fdtd.c:3143-3170 */
                    kappa_x = ldg_nh(a.tx.kappa + i);
                    const double bb = ldg_nh(a.tx.b + i), cc = ldg_nh(a.tx.c + i);
                    a.psi.hxy[qx] = SOp::add(SOp::mul(bb, pxy), SOp::mul(cc, SOp::div(dEz_dx, mu0)));
                    a.psi.hxz[qx] = SOp::add(SOp::mul(bb, pxz), SOp::mul(cc, SOp::div(-dEy_dx, mu0)));
                }
                if (sy >= 0) { /* fdtd.c:3173-3200 */
                    kappa_y = ldg_nh(a.ty.kappa + j);
                    const double bb = ldg_nh(a.ty.b + j), cc = ldg_nh(a.ty.c + j);
                    a.psi.hyx[qy] = SOp::add(SOp::mul(bb, pyx), SOp::mul(cc, SOp::div(-dEz_dy, mu0)));
                    a.psi.hyz[qy] = SOp::add(SOp::mul(bb, pyz), SOp::mul(cc, SOp::div(dEx_dy, mu0)));
                }
                if (sz >= 0) kappa_z = ldg_nh(a.tz.kappa + k); /* fdtd.c:3203-3219 */
                /* fdtd.c:3222-3224 */
                const double ux = SOp::add(SOp::add(SOp::add(SOp::div(SOp::div(-dEz_dy, mu0), kappa_y), pyx),
                                                    SOp::div(SOp::div(dEy_dz, mu0), kappa_z)), pzx);
                const double uy = SOp::add(SOp::add(SOp::add(SOp::div(SOp::div(dEz_dx, mu0), kappa_x), pxy),
                                                    SOp::div(SOp::div(-dEx_dz, mu0), kappa_z)), pzy);
                const double uz = SOp::add(SOp::add(SOp::add(SOp::div(SOp::div(-dEy_dx, mu0), kappa_x), pxz),
                                                    SOp::div(SOp::div(dEx_dy, mu0), kappa_y)), pyz);
                hxg[c] = SOp::add(hx0, SOp::mul(a.dt, ux));
                hyg[c] = SOp::add(hy0, SOp::mul(a.dt, uy));
                hzg[c] = SOp::add(hz0, SOp::mul(a.dt, uz));
                if (sz >= 0) { /* fdtd.c:3225-3228 */
                    const double bb = ldg_nh(a.tz.b + k), cc = ldg_nh(a.tz.c + k);
                    a.psi.hzx[qz] = SOp::add(SOp::mul(bb, pzx), SOp::mul(cc, SOp::div(dEy_dz, mu0)));
                    a.psi.hzy[qz] = SOp::add(SOp::mul(bb, pzy), SOp::mul(cc, SOp::div(-dEx_dz, mu0)));
                }
            } else {
                const R dEyz = ey1 - ey0, dEzy = ezj - ez0, dEzx = ezi - ez0;
                const R dExz = ex1 - ex0, dExy = exj - ex0, dEyx = eyi - ey0;
                /* psi terms enter as zeros outside the PML */
                hxg[c] = hx0 + (-khy * dEzy + khz * dEyz + pyx + pzx);
                hyg[c] = hy0 + (khx * dEzx - khz * dExz + pxy + pzy);
                hzg[c] = hz0 + (-khx * dEyx + khy * dExy + pxz + pyz);
                if (sx >= 0) {
                    a.psi.hxy[qx] = bx * pxy + chx * dEzx;
                    a.psi.hxz[qx] = bx * pxz - chx * dEyx;
                }
                if (sy >= 0) {
                    a.psi.hyx[qy] = by * pyx - chy * dEzy;
                    a.psi.hyz[qy] = by * pyz + chy * dExy;
                }
                if (sz >= 0) {
                    a.psi.hzx[qz] = bz * pzx + chz * dEyz;
                    a.psi.hzy[qz] = bz * pzy - chz * dExz;
                }
            }
        }
        /* every thread is done with plane k: its stage takes plane k + stages */
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                ring_drain(full, G::HS, h_loads_issued(k, k0, k1, G::HS));
            }
            break;
        }
        if (tid == 0 && k + G::HS <= k1) {
            fence_proxy_async_smem();
            issue(k + G::HS);
        }
    }
}

/* ================================================================ E sweep */

/* fdtd.c:3238-3528 fused, as e_sweep, with H, D and the material ids
 * streamed through the stage ring. */
template <typename R, bool STRICT, int NAMAX>
__global__ void __launch_bounds__(kBlockX * kBlockY,
                                  (NAMAX > 4 ? 1
                                   : sizeof(R) == 4 ? (kIonVReg<R, NAMAX> ? PHP_E_MINBLOCKS32_ATOMS : PHP_E_MINBLOCKS32)
                                   : kIonVReg<R, NAMAX> ? PHP_E_MINBLOCKS64_ATOMS : PHP_E_MINBLOCKS))
    e_sweep_tma(const __grid_constant__ StepArgs<R> a, const __grid_constant__ TmaMaps tm)
{
    using G = TmaGeom<R>;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* smem = ring_base(dyn_smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::ES * G::E_STAGE);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * G::TX + tx;
    const int i0 = blockIdx.x * G::TX, j0 = blockIdx.y * G::TY;
    const int i = i0 + tx, j = j0 + ty;
    const int bz = blockIdx.z + a.zc0;
    const int k0 = bz * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return; /* uniform over the block */

    constexpr uint32_t HB = G::align128(G::HALO_BYTES), OB = G::align128(G::OWN_BYTES);
    /* plane p = k0-1 .. k1-1 into stage (p - k0 + 1) % stages */
    auto stage = [&](int p) -> unsigned char* { return smem + (uint32_t)((p - k0 + 1) % G::ES) * G::E_STAGE; };
    auto issue = [&](int p) {
        uint64_t* bar = &full[(p - k0 + 1) % G::ES];
        unsigned char* b = stage(p);
        const bool own = p >= k0;
        mbar_arrive_expect_tx(bar, 3 * G::HALO_BYTES + (own ? 3 * G::OWN_BYTES + G::MAT_BYTES : 0u));
        for (int q = 0; q < 3; ++q) tma_load_3d(b + q * HB, &tm.h_halo[q], bar, i0 - G::HALO, j0 - 1, p + 1);
        if (own) {
            for (int q = 0; q < 3; ++q) tma_load_3d(b + 3 * HB + q * OB, &tm.d_own[q], bar, i0, j0, p + 1);
            tma_load_3d(b + 3 * HB + 3 * OB, &tm.mat, bar, i0, j0, p);
        }
    };

    /* material records of ids < a.nmat, copied after the barriers */
    MatCoef<R>* mcs = reinterpret_cast<MatCoef<R>*>(smem + G::ES * G::E_STAGE + 128);
    if (tid == 0) {
        for (int s = 0; s < G::ES; ++s) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.mc);
        uint32_t* dst = reinterpret_cast<uint32_t*>(mcs);
        const int words = a.nmat * (int)(sizeof(MatCoef<R>) / 4);
        for (int t = tid; t < words; t += G::TX * G::TY) dst[t] = ldg(src + t);
    }
    __syncthreads();
    if (tid == 0)
        for (int p = k0 - 1; p <= min(k1 - 1, k0 - 1 + G::ES - 1); ++p) issue(p);

    const int ho = (ty + 1) * G::BX + tx + G::HALO; /* own cell in a halo box */
    const int oo = ty * G::TX + tx;                 /* own cell in an own box */
    /* after the march: the running DFT samples and the monitor row of this
     * chunk's planes */
    auto fold_dft = [&]() {
        R* const e3[3] = {a.f.ex, a.f.ey, a.f.ez};
        if (a.ndft) dft_fold(a, e3, i, j, k0, k1);
        if (a.probe_rows) {
            R* const h3[3] = {a.f.hx, a.f.hy, a.f.hz};
            probe_fold(a, e3, h3, i, j, k0, k1);
        }
    };

    /* a plain block (one plain isotropic material, no CPML, edge or source
     * cell; marked on the host): D += curl H with the kappa = 1 factors and
     * E = iso D, nothing per cell beyond the stencil (the same arithmetic as
     * the general path below takes for such cells) */
    const int pm = (!STRICT && a.plain_blk) ? a.plain_blk[((size_t)bz * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x]
                                            : 255;
    if constexpr (NAMAX > 0 && NAMAX <= 4) {
        if (pm == kPlainAtoms) {
            /* the few-atom material alone (no ADE, no source): the general
             * path's D update and D -> E with the fused ion update, its
             * material record and ion coefficients from the kernel
             * parameters, the cell's slot (and, held in registers, its r
             * and v) read before the stage wait */
            const MatCoef<R>& m = a.amc;
            constexpr int QN = 3 * NAMAX;
            constexpr bool VREG = QN * (int)sizeof(R) <= kIonRegBytesR<R>;
            const int n3 = 3 * m.natom;
            const bool active = (i < a.nx) && (j < a.ny);
            const bool interior = (i >= 1 && i < a.nx - 1 && j >= 1 && j < a.ny - 1);
            const int sx = active ? ldg(a.tx.slot + i) : -1;
            const int sy = active ? ldg(a.ty.slot + j) : -1;
            const bool lossy = (m.flags & kLossy) != 0;
            constexpr bool kInc = sizeof(R) == 4;
            for (int k = k0; k < k1; ++k) {
                CellPsi<R> ps;
                ps.sz = -1;
                if (active && interior) load_psi_d(a, i, j, k, sx, sy, ps);
                if (kPsiAheadE<R> && active && interior && k + 1 < k1) prefetch_psi_d(a, i, j, k + 1, sx, sy);
                const int c = (k * a.ny + j) * a.nxp + i;
                R ex = R(0), ey = R(0), ez = R(0);
                if (active && interior && lossy) {
                    ex = a.f.ex[c];
                    ey = a.f.ey[c];
                    ez = a.f.ez[c];
                    if (PHP_EOLD_AHEAD && k + 1 < k1) { /* the next plane's lines into L1 */
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ex + c + a.plane));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ey + c + a.plane));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ez + c + a.plane));
                    }
                }
                IonPre ip;
                ip.slot = -1;
                if (active) {
                    ip.slot = a.slot[c];
                    /* r and v into L1 ahead of their reads in e_update */
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
                bool ok = true;
                if (k == k0) ok = mbar_wait(&full[0], 0);
                ok = ok && mbar_wait(&full[(k - k0 + 1) % G::ES], ((k - k0 + 1) / G::ES) & 1);
                if (ok && active) {
                    const unsigned char* bp = stage(k - 1);
                    const unsigned char* bc = stage(k);
                    const R* Hxp = reinterpret_cast<const R*>(bp);
                    const R* Hyp = reinterpret_cast<const R*>(bp + HB);
                    const R* Hx = reinterpret_cast<const R*>(bc);
                    const R* Hy = reinterpret_cast<const R*>(bc + HB);
                    const R* Hz = reinterpret_cast<const R*>(bc + 2 * HB);
                    const R* Ds = reinterpret_cast<const R*>(bc + 3 * HB);
                    R dx = Ds[oo], dy = Ds[OB / sizeof(R) + oo], dz = Ds[2 * (OB / sizeof(R)) + oo];
                    R ix = R(0), iy = R(0), iz = R(0);
                    R& ux = kInc ? ix : dx;
                    R& uy = kInc ? iy : dy;
                    R& uz = kInc ? iz : dz;
                    if (interior) {
                        d_update<R, false>(a, i, j, k, sx, sy, Hx[ho], Hy[ho], Hz[ho], Hxp[ho], Hyp[ho], Hz[ho - G::BX],
                                           Hx[ho - G::BX], Hz[ho - 1], Hy[ho - 1], ps, ux, uy, uz);
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
                    a.f.dx[c] = dx;
                    a.f.dy[c] = dy;
                    a.f.dz[c] = dz;
                    a.f.ex[c] = ex;
                    a.f.ey[c] = ey;
                    a.f.ez[c] = ez;
                }
                if (__syncthreads_or(!ok)) {
                    if (tid == 0) {
                        atomicExch(a.err, 1);
                        ring_drain(full, G::ES, e_loads_issued(k, k0, k1, G::ES));
                    }
                    break;
                }
                if (tid == 0 && k - 1 + G::ES <= k1 - 1) {
                    fence_proxy_async_smem();
                    issue(k - 1 + G::ES);
                }
            }
            fold_dft();
            return;
        }
    }
    if (pm == kPlainTensor) {
        /* one lossy or anisotropic material (no ADE, ions or source): the
         * general path's D update with the eps'' term and E = eps^-1 D in
         * the crystal frame, its coefficients from the kernel parameters and
         * the old E read before the stage wait (it does not depend on the
         * stages) */
        const bool active = (i < a.nx) && (j < a.ny);
        const bool interior = (i >= 1 && i < a.nx - 1 && j >= 1 && j < a.ny - 1);
        const int sx = active ? ldg(a.tx.slot + i) : -1;
        const int sy = active ? ldg(a.ty.slot + j) : -1;
        const int fl = a.tns_flags;
        const bool lossy = (fl & kLossy) != 0;
        constexpr bool kInc = sizeof(R) == 4;
        for (int k = k0; k < k1; ++k) {
            CellPsi<R> ps;
            ps.sz = -1;
            if (active && interior) load_psi_d(a, i, j, k, sx, sy, ps);
            if (kPsiAheadE<R> && active && interior && k + 1 < k1) prefetch_psi_d(a, i, j, k + 1, sx, sy);
            const int c = (k * a.ny + j) * a.nxp + i;
            R ex = R(0), ey = R(0), ez = R(0);
            if (active && interior && lossy) {
                ex = a.f.ex[c];
                ey = a.f.ey[c];
                ez = a.f.ez[c];
                if (PHP_EOLD_AHEAD && k + 1 < k1) { /* the next plane's lines into L1 */
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ex + c + a.plane));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ey + c + a.plane));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ez + c + a.plane));
                }
            }
            bool ok = true;
            if (k == k0) ok = mbar_wait(&full[0], 0);
            ok = ok && mbar_wait(&full[(k - k0 + 1) % G::ES], ((k - k0 + 1) / G::ES) & 1);
            if (ok && active) {
                const unsigned char* bp = stage(k - 1);
                const unsigned char* bc = stage(k);
                const R* Hxp = reinterpret_cast<const R*>(bp);
                const R* Hyp = reinterpret_cast<const R*>(bp + HB);
                const R* Hx = reinterpret_cast<const R*>(bc);
                const R* Hy = reinterpret_cast<const R*>(bc + HB);
                const R* Hz = reinterpret_cast<const R*>(bc + 2 * HB);
                const R* Ds = reinterpret_cast<const R*>(bc + 3 * HB);
                R dx = Ds[oo], dy = Ds[OB / sizeof(R) + oo], dz = Ds[2 * (OB / sizeof(R)) + oo];
                R ix = R(0), iy = R(0), iz = R(0);
                R& ux = kInc ? ix : dx;
                R& uy = kInc ? iy : dy;
                R& uz = kInc ? iz : dz;
                if (interior) {
                    d_update<R, false>(a, i, j, k, sx, sy, Hx[ho], Hy[ho], Hz[ho], Hxp[ho], Hyp[ho], Hz[ho - G::BX],
                                       Hx[ho - G::BX], Hz[ho - 1], Hy[ho - 1], ps, ux, uy, uz);
                    if (lossy) { /* fdtd.c:3349-3353 */
                        const R* q = a.tns_im;
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
                /* fdtd.c:3429-3461, 3486-3503 */
                R da = dx, db = dy, dc = dz;
                rot_fwd<false>(fl, a.tns_cs, a.tns_sn, da, db, dc);
                const R* E = a.tns_inv;
                R na = E[0] * da + E[1] * db + E[2] * dc;
                R nb = E[3] * da + E[4] * db + E[5] * dc;
                R nc = E[6] * da + E[7] * db + E[8] * dc;
                rot_back<false>(fl, a.tns_cs, a.tns_sn, na, nb, nc);
                a.f.dx[c] = dx;
                a.f.dy[c] = dy;
                a.f.dz[c] = dz;
                a.f.ex[c] = na;
                a.f.ey[c] = nb;
                a.f.ez[c] = nc;
            }
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(a.err, 1);
                    ring_drain(full, G::ES, e_loads_issued(k, k0, k1, G::ES));
                }
                break;
            }
            if (tid == 0 && k - 1 + G::ES <= k1 - 1) {
                fence_proxy_async_smem();
                issue(k - 1 + G::ES);
            }
        }
        fold_dft();
        return;
    }
    if (pm != 255 && pm >= kPlainCpml) {
        /* one plain material with CPML or domain-edge cells: the general
         * path's D update (CPML terms included) and E = iso D, without the
         * per-cell material and source handling */
        const R iso = a.iso[pm - kPlainCpml];
        const bool active = (i < a.nx) && (j < a.ny);
        const bool interior = (i >= 1 && i < a.nx - 1 && j >= 1 && j < a.ny - 1);
        const int sx = active ? ldg(a.tx.slot + i) : -1;
        const int sy = active ? ldg(a.ty.slot + j) : -1;
        constexpr bool kInc = sizeof(R) == 4;
        for (int k = k0; k < k1; ++k) {
            CellPsi<R> ps;
            ps.sz = -1;
            if (active && interior) load_psi_d(a, i, j, k, sx, sy, ps);
            if (kPsiAheadE<R> && active && interior && k + 1 < k1) prefetch_psi_d(a, i, j, k + 1, sx, sy);
            bool ok = true;
            if (k == k0) ok = mbar_wait(&full[0], 0);
            ok = ok && mbar_wait(&full[(k - k0 + 1) % G::ES], ((k - k0 + 1) / G::ES) & 1);
            if (ok && active) {
                const unsigned char* bp = stage(k - 1);
                const unsigned char* bc = stage(k);
                const R* Hxp = reinterpret_cast<const R*>(bp);
                const R* Hyp = reinterpret_cast<const R*>(bp + HB);
                const R* Hx = reinterpret_cast<const R*>(bc);
                const R* Hy = reinterpret_cast<const R*>(bc + HB);
                const R* Hz = reinterpret_cast<const R*>(bc + 2 * HB);
                const R* Ds = reinterpret_cast<const R*>(bc + 3 * HB);
                R dx = Ds[oo], dy = Ds[OB / sizeof(R) + oo], dz = Ds[2 * (OB / sizeof(R)) + oo];
                R ix = R(0), iy = R(0), iz = R(0);
                R& ux = kInc ? ix : dx;
                R& uy = kInc ? iy : dy;
                R& uz = kInc ? iz : dz;
                if (interior)
                    d_update<R, false>(a, i, j, k, sx, sy, Hx[ho], Hy[ho], Hz[ho], Hxp[ho], Hyp[ho], Hz[ho - G::BX],
                                       Hx[ho - G::BX], Hz[ho - 1], Hy[ho - 1], ps, ux, uy, uz);
                if constexpr (kInc) {
                    dx += ix;
                    dy += iy;
                    dz += iz;
                }
                const int c = (k * a.ny + j) * a.nxp + i;
                a.f.dx[c] = dx;
                a.f.dy[c] = dy;
                a.f.dz[c] = dz;
                a.f.ex[c] = iso * dx;
                a.f.ey[c] = iso * dy;
                a.f.ez[c] = iso * dz;
            }
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(a.err, 1);
                    ring_drain(full, G::ES, e_loads_issued(k, k0, k1, G::ES));
                }
                break;
            }
            if (tid == 0 && k - 1 + G::ES <= k1 - 1) {
                fence_proxy_async_smem();
                issue(k - 1 + G::ES);
            }
        }
        fold_dft();
        return;
    }
    if (pm != 255) {
        const R iso = a.iso[pm];
        const R kdx = a.kdp[0], kdy = a.kdp[1], kdz = a.kdp[2];
        for (int k = k0; k < k1; ++k) {
            bool ok = true;
            if (k == k0) ok = mbar_wait(&full[0], 0);
            ok = ok && mbar_wait(&full[(k - k0 + 1) % G::ES], ((k - k0 + 1) / G::ES) & 1);
            if (ok) {
                const unsigned char* bp = stage(k - 1);
                const unsigned char* bc = stage(k);
                const R* Hxp = reinterpret_cast<const R*>(bp);
                const R* Hyp = reinterpret_cast<const R*>(bp + HB);
                const R* Hx = reinterpret_cast<const R*>(bc);
                const R* Hy = reinterpret_cast<const R*>(bc + HB);
                const R* Hz = reinterpret_cast<const R*>(bc + 2 * HB);
                const R* Ds = reinterpret_cast<const R*>(bc + 3 * HB);
                const R hx0 = Hx[ho], hy0 = Hy[ho], hz0 = Hz[ho];
                const R dHzy = hz0 - Hz[ho - G::BX], dHyz = hy0 - Hyp[ho], dHxz = hx0 - Hxp[ho];
                const R dHzx = hz0 - Hz[ho - 1], dHyx = hy0 - Hy[ho - 1], dHxy = hx0 - Hx[ho - G::BX];
                const R ux = kdy * dHzy - kdz * dHyz;
                const R uy = -kdx * dHzx + kdz * dHxz;
                const R uz = kdx * dHyx - kdy * dHxy;
                const R dx = Ds[oo] + ux, dy = Ds[OB / sizeof(R) + oo] + uy, dz = Ds[2 * (OB / sizeof(R)) + oo] + uz;
                const int c = (k * a.ny + j) * a.nxp + i;
                a.f.dx[c] = dx;
                a.f.dy[c] = dy;
                a.f.dz[c] = dz;
                a.f.ex[c] = iso * dx;
                a.f.ey[c] = iso * dy;
                a.f.ez[c] = iso * dz;
            }
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(a.err, 1);
                    ring_drain(full, G::ES, e_loads_issued(k, k0, k1, G::ES));
                }
                break;
            }
            if (tid == 0 && k - 1 + G::ES <= k1 - 1) {
                fence_proxy_async_smem();
                issue(k - 1 + G::ES);
            }
        }
        fold_dft();
        return;
    }

    const bool active = (i < a.nx) && (j < a.ny);
    const bool interior = (i >= 1 && i < a.nx - 1 && j >= 1 && j < a.ny - 1);
    const int sx = active ? ldg(a.tx.slot + i) : -1;
    const int sy = active ? ldg(a.ty.slot + j) : -1;
    /* pool slot of the cell one plane ahead (ADE and atom cells, -1 for the
     * others): the lines of P, P_old and P_ion of this plane's cell are
     * requested before the stage wait instead of after the material lookup */
    const bool slots = PHP_SLOT_AHEAD && sizeof(R) == 4 && a.slot != nullptr && active;
    int slot_next = slots ? ldg(a.slot + (k0 * a.ny + j) * a.nxp + i) : -1;

    for (int k = k0; k < k1; ++k) {
        /* CPML state read before the wait (it does not depend on the stages) */
        CellPsi<R> ps;
        ps.sz = -1;
        if (PHP_PSI_EARLY_E && active && interior) load_psi_d(a, i, j, k, sx, sy, ps);
        if (kPsiAheadE<R> && !STRICT && active && interior && k + 1 < k1) prefetch_psi_d(a, i, j, k + 1, sx, sy);
        IonPre ip;
        ip.slot = slot_next;
        if (slots && k + 1 < k1) slot_next = ldg(a.slot + ((k + 1) * a.ny + j) * a.nxp + i);
        if (ip.slot >= 0) {
            const int64_t ns = a.nslot;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (a.P) {
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.P + q * ns + ip.slot));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(a.Po + q * ns + ip.slot));
                }
                if (!STRICT && NAMAX == 0 && a.pr) asm volatile("prefetch.global.L1 [%0];" ::"l"(a.pr + q * ns + ip.slot));
            }
            if (PHP_EOLD_AHEAD_GEN) { /* the old E the ADE update reads, before the wait */
                const int c = (k * a.ny + j) * a.nxp + i;
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ex + c));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ey + c));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.f.ez + c));
            }
        }
        bool ok = true;
        if (k == k0) ok = mbar_wait(&full[0], 0);
        ok = ok && mbar_wait(&full[(k - k0 + 1) % G::ES], ((k - k0 + 1) / G::ES) & 1);
        if (!PHP_PSI_EARLY_E && active && interior) load_psi_d(a, i, j, k, sx, sy, ps);
        if (ok && active) {
            const unsigned char* bp = stage(k - 1);
            const unsigned char* bc = stage(k);
            const R* Hxp = reinterpret_cast<const R*>(bp);
            const R* Hyp = reinterpret_cast<const R*>(bp + HB);
            const R* Hx = reinterpret_cast<const R*>(bc);
            const R* Hy = reinterpret_cast<const R*>(bc + HB);
            const R* Hz = reinterpret_cast<const R*>(bc + 2 * HB);
            const R* Dx = reinterpret_cast<const R*>(bc + 3 * HB);
            const R* Dy = reinterpret_cast<const R*>(bc + 3 * HB + OB);
            const R* Dz = reinterpret_cast<const R*>(bc + 3 * HB + 2 * OB);
            const uint8_t* M = reinterpret_cast<const uint8_t*>(bc + 3 * HB + 3 * OB);
            const int c = (k * a.ny + j) * a.nxp + i;
            e_cell<R, STRICT, NAMAX>(a, i, j, k, c, interior, sx, sy, Hx[ho], Hy[ho], Hz[ho], Hxp[ho], Hyp[ho],
                                     Hz[ho - G::BX], Hx[ho - G::BX], Hz[ho - 1], Hy[ho - 1], Dx[oo], Dy[oo], Dz[oo], M[oo],
                                     mcs, &ps, slots ? &ip : nullptr);
        }
        /* every thread is done with plane k-1: its stage takes plane k-1 + stages */
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                ring_drain(full, G::ES, e_loads_issued(k, k0, k1, G::ES));
            }
            break;
        }
        if (tid == 0 && k - 1 + G::ES <= k1 - 1) {
            fence_proxy_async_smem();
            issue(k - 1 + G::ES);
        }
    }
    fold_dft();
}

} // namespace phpdev
