/*
 * php_ions.cuh -- the ionic equations of motion of many-atom cells as their
 * own pass over the compact atom pool (fdtd.c:3418-3427, 3507-3528).
 *
 * For cells with few atoms the ion update stays inside the fused E sweep.
 * For many atoms (3N >= 24) the per-cell work is a (cells x 3N) . (3N x 3N)
 * contraction, DMM . r, and 12 N words of r and v per cell; inside the
 * stencil sweep it costs registers the plane pipeline needs.  Here it runs
 * after the E sweep, on the pool in slot order (cells in k, j, i order):
 *
 *   a   = QeZM . E^{n+1} - DMM . r^n        (crystal frame)
 *   r  += v dt + a dt^2 / 2,   v += a dt
 *   Pr  = QeZV . r^{n+1}                    (stored for the next E sweep)
 *
 * The E sweep of the next step reads Pr (3 words) instead of recomputing
 * QeZV . r from the 3N-word pool, so the pool is read and written once per
 * step.  The arithmetic is the reference's; only its rounding order differs
 * from the fused form (FP64: within 1e-10 of the reference).
 *
 *  ion_pipe       the pass proper: a TMA-fed ring of pool tiles, two
 *                 consumer warpgroups.  FP32 (mixed path) on the 5th-generation
 *                 tensor cores: per 128-cell tile, r is split into bf16 hi + lo,
 *                 DMM likewise (host), and D = r_hi DMM_hi^T + r_hi DMM_lo^T +
 *                 r_lo DMM_hi^T accumulates in FP32 in tensor memory
 *                 (tcgen05.mma kind::f16, M = 128, N = K = 3N padded to 16);
 *                 the epilogue reads D with tcgen05.ld and does the update.
 *                 The dropped r_lo DMM_lo term and the bf16 representation
 *                 leave about 2^-17 relative error in DMM . r.  FP64 (fast
 *                 plain path): FMA chains against DMM in shared memory.
 *  ion_update_cc  plain loads, FP64, one cell per thread: used where the
 *                 FP64 ring does not fit in shared memory (3N > 48).
 */
#pragma once

#include <cuda_bf16.h>

namespace phpdev {

template <typename R>
struct IonArgs {
    const R *ex, *ey, *ez;       /* E^{n+1}, plane 0 of the field arrays */
    R *r, *v, *pr;               /* pools [3N][nslot], Pr [3][nslot] */
    const int64_t* slot_cell;
    const int32_t* slot_n3;
    const uint8_t* slot_mat;     /* material id per slot */
    const uint8_t* mat;
    const MatCoef<R>* mc;
    const R* ion_coef;
    const R* dmm;                /* [NP][NP], zero padded (CUDA-core kernel) */
    const double* dfrag;         /* FP64 ring: DMM as m8n8k4 B fragments [NP/4][NP/8][32 lanes] */
    const uint32_t* bsplit;      /* DMM hi, lo as bf16 in the UMMA K-major layout (tensor kernel) */
    int64_t nslot;
    int32_t ntiles;
    int32_t ion_off_ref;         /* the lattice's QeZV/QeZM block, staged in shared memory */
    double dt;
    int32_t* err;
};

constexpr int kIonTile = 128;

/* crystal-frame E at a pool cell, and the cell's material record */
template <typename R>
__device__ __forceinline__ const MatCoef<R>& ion_cell_e(const IonArgs<R>& a, int64_t s, R& e0, R& e1, R& e2)
{
    const int64_t c = a.slot_cell[s];
    const MatCoef<R>& m = a.mc[a.mat[c]];
    e0 = a.ex[c];
    e1 = a.ey[c];
    e2 = a.ez[c];
    rot_fwd<false>(m.flags, m.cs, m.sn, e0, e1, e2);
    return m;
}

/* ---------------------------------------------------------- CUDA cores */

template <typename R, int NP>
__global__ void __launch_bounds__(kIonTile) ion_update_cc(const IonArgs<R> a)
{
    __shared__ R D[NP * NP];
    for (int t = threadIdx.x; t < NP * NP; t += kIonTile) D[t] = a.dmm[t];
    __syncthreads();
    const R dt = R(a.dt);
    const int64_t ns = a.nslot;
    for (int64_t s = (int64_t)blockIdx.x * kIonTile + threadIdx.x; s < ns; s += (int64_t)gridDim.x * kIonTile) {
        const int n3 = a.slot_n3[s];
        if (n3 == 0) continue;
        R rold[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) rold[q] = q < n3 ? a.r[(int64_t)q * ns + s] : R(0);
        R e0, e1, e2;
        const MatCoef<R>& m = ion_cell_e(a, s, e0, e1, e2);
        const R* qv = a.ion_coef + m.ion_off;
        const R* qm = qv + 3 * n3;
        R p0 = R(0), p1 = R(0), p2 = R(0);
        /* QG coordinates at a time: QG independent accumulation chains, and
         * their v loads in flight together */
        constexpr int QG = 4;
#pragma unroll 1
        for (int q0 = 0; q0 < n3; q0 += QG) {
            R acc[QG], vq[QG];
#pragma unroll
            for (int u = 0; u < QG; ++u) {
                const int q = q0 + u;
                vq[u] = q < n3 ? a.v[(int64_t)q * ns + s] : R(0);
                const int at = q / 3, d = q - 3 * at;
                acc[u] = q < n3 ? ldg(qm + at * 9 + d) * e0 + ldg(qm + at * 9 + 3 + d) * e1 +
                                      ldg(qm + at * 9 + 6 + d) * e2
                                : R(0);
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) {
#pragma unroll
                for (int u = 0; u < QG; ++u) acc[u] -= D[(q0 + u) * NP + p] * rold[p];
            }
#pragma unroll
            for (int u = 0; u < QG; ++u) {
                const int q = q0 + u;
                if (q < n3) {
                    const int at = q / 3, d = q - 3 * at;
                    const int64_t o = (int64_t)q * ns + s;
                    const R rn = a.r[o] + (vq[u] * dt + R(0.5) * acc[u] * dt * dt); /* r^n again, from L1 */
                    a.r[o] = rn;
                    a.v[o] = vq[u] + acc[u] * dt;
                    p0 += ldg(qv + at * 9 + d) * rn;
                    p1 += ldg(qv + at * 9 + 3 + d) * rn;
                    p2 += ldg(qv + at * 9 + 6 + d) * rn;
                }
            }
        }
        a.pr[s] = p0;
        a.pr[ns + s] = p1;
        a.pr[2 * ns + s] = p2;
    }
}

/* ---------------------------------------------------------- tensor cores */

/* byte offset of element (row, k) of a bf16 operand in the no-swizzle
 * K-major layout: 8 x 16-byte core matrices, row groups 128 B apart, K
 * chunks of 8 elements `rows * 16` bytes apart */
__host__ __device__ constexpr uint32_t umma_kmajor_off(int row, int k, int rows)
{
    return (uint32_t)((k >> 3) * rows * 16 + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46; /* descriptor version of sm_100 */
    /* base offset 0, legacy LBO mode, layout type 0 = no swizzle */
    return d;
}

/* kind::f16 instruction descriptor: bf16 A and B (K-major), f32 D */
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat16 lo_half, __nv_bfloat16 hi_half)
{
    return (uint32_t)__bfloat16_as_ushort(lo_half) | ((uint32_t)__bfloat16_as_ushort(hi_half) << 16);
}

/* ------------------------------------------------- pipelined ion pass
 *
 * One CTA per SM, persistent over 128-cell tiles.  Warp 8 streams the r
 * and v tiles of the pool (box 128 cells x 3N, cp.async.bulk.tensor, no
 * multicast) and the tiles' slot indices (cp.async.bulk) into a ring of S
 * stages; two consumer warpgroups take alternate tiles, so that one group's
 * tensor-core round trip or E gather overlaps the other's epilogue.  The
 * updated r, v go back from the stage with a tensor store.  FP32: DMM . r as
 * BF16 x 3 on tcgen05 (each group its own A buffers and TMEM columns); FP64:
 * CUDA-core FMA chains against DMM in shared memory.
 */
struct IonMaps {
    CUtensorMap r, v; /* pool [3N][ns] as (x = slot, y = coordinate), box 128 x 3N */
};

template <int NP>
__host__ __device__ constexpr int ion_cols() { return NP <= 32 ? 32 : 64; }

template <typename R, int NP, int S>
struct IonPipe {
    static constexpr bool TC = sizeof(R) == 4;
    /* consumer groups: FP32 two groups of 128 threads take alternate tiles
     * (one accumulator row per thread); FP64 one group of 256 threads takes
     * each tile, so that with two stages one tile loads while one computes */
    static constexpr int CONSUMERS = 2 * kIonTile, THREADS = CONSUMERS + 32;
    static constexpr int GT = TC ? kIonTile : 2 * kIonTile, GROUPS = CONSUMERS / GT;
    static constexpr int CELLS_PER_WARP = kIonTile / (GT / 32);  /* FP64: 16 */
    static_assert(CONSUMERS % GT == 0 && GT % kIonTile == 0 && CELLS_PER_WARP % 16 == 0, "consumer layout");
    static constexpr uint32_t BOX = kIonTile * NP * sizeof(R);      /* one array's tile, NP rows */
    /* per stage: r, v, then the slots' cell offsets (int64, 1024 B), atom
     * coordinate counts (int32, 512 B) and material ids (uint8, 128 B) */
    static constexpr uint32_t IDX = 2048;
    /* then the crystal-frame inputs: Ex, Ey, Ez of the tile's cells, gathered
     * by the producer warp with cp.async */
    static constexpr uint32_t E_OFF = 2 * BOX + IDX;
    static constexpr uint32_t EB = 3 * kIonTile * sizeof(R);
    static constexpr uint32_t STAGE = 2 * BOX + IDX + EB;
    static constexpr uint32_t A_BYTES = kIonTile * NP * 2;           /* bf16 rows of one group */
    static constexpr uint32_t B_BYTES = NP * NP * 2;
    /* FP64: DMM, -QeZM (the E step) and QeZV^T (P_ion) as m8n8k4 B fragments */
    static constexpr uint32_t FRAG_E = NP * NP, FRAG_P = FRAG_E + (NP / 8) * 32, FRAG_N = FRAG_P + (NP / 4) * 32;
    static constexpr uint32_t OPS = TC ? GROUPS * 2 * A_BYTES + 2 * B_BYTES : FRAG_N * 8;
    /* FP32: the lattice's QeZV, QeZM (9N each, 9N <= 3 NP) */
    static constexpr uint32_t COEF = TC ? 2 * 3 * NP * sizeof(R) : 0;
    static constexpr uint32_t SMEM = 1024 + S * STAGE + OPS + COEF + 256;
};

__device__ __forceinline__ void named_sync(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

/* barrier `id` over n threads that also ORs a predicate across them */
__device__ __forceinline__ bool named_sync_or(int id, int n, bool v)
{
    uint32_t r;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(r)
                 : "r"((uint32_t)v), "r"(id), "r"(n)
                 : "memory");
    return r != 0;
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
                 ::"l"(map), "r"(smem_addr(src)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

/* untiled bulk copy global -> shared, completing on an mbarrier (both
 * addresses 16-byte aligned, size a multiple of 16) */
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

/* D += A B for one 8 x 8 x 4 FP64 tile (the FP64 tensor path): per lane
 * g = lane / 4, t = lane % 4, a = A[g][t], b = B[t][g], and c0, c1 =
 * C[g][2t], C[g][2t + 1] */
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

/* B-byte asynchronous copy global -> shared (B = 4, 8 or 16) */
template <int B>
__device__ __forceinline__ void cp_async_ca(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"(B) : "memory");
}

/* an arrival on bar once this thread's earlier cp.async copies have landed
 * (counted in the barrier's expected arrivals) */
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

template <typename R, int NP, int S>
__global__ void __launch_bounds__(IonPipe<R, NP, S>::THREADS, 1)
    ion_pipe(const __grid_constant__ IonArgs<R> a, const __grid_constant__ IonMaps maps, int32_t n3)
{
    using P = IonPipe<R, NP, S>;
    static_assert(NP % 16 == 0 && NP >= 16 && NP <= 64, "3N padded to 16..64");
    static_assert(P::SMEM <= 227u * 1024u, "shared memory of one CTA");
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* base = dyn_smem + ((1024u - (smem_addr(dyn_smem) & 1023u)) & 1023u);
    unsigned char* stages = base;
    unsigned char* ops = base + S * P::STAGE;
    R* coef = reinterpret_cast<R*>(ops + P::OPS);
    uint64_t* full = reinterpret_cast<uint64_t*>(ops + P::OPS + P::COEF);
    uint64_t* empty = full + S;
    uint64_t* mma_bar = empty + S;                                 /* one per group */
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + P::GROUPS);
    volatile int32_t* consumed = reinterpret_cast<volatile int32_t*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    const int mine = a.ntiles > (int)blockIdx.x ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    /* DMM (bf16 images for the tensor cores, or the padded FP64 matrix) and
     * the lattice's QeZV, QeZM (cells of other materials read global) */
    {
        const uint4* src = P::TC ? reinterpret_cast<const uint4*>(a.bsplit) : reinterpret_cast<const uint4*>(a.dfrag);
        unsigned char* dst0 = P::TC ? ops + P::GROUPS * 2 * P::A_BYTES : ops;
        const int n16 = (int)((P::TC ? 2 * P::B_BYTES : P::OPS) / 16);
        uint4* dst = reinterpret_cast<uint4*>(dst0);
        for (int t = tid; t < n16; t += P::THREADS) dst[t] = src[t];
        if constexpr (P::TC)
            for (int t = tid; t < 6 * n3; t += P::THREADS) coef[t] = a.ion_coef[a.ion_off_ref + t];
    }
    if constexpr (P::TC) {
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                         "r"(P::GROUPS * ion_cols<NP>()));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
    }
    if (tid == 0) {
        for (int q = 0; q < S; ++q) {
            /* the producer's expect_tx arrival and one cp.async arrival per producer lane */
            mbar_init(&full[q], 1 + 32);
            mbar_init(&empty[q], 1);
        }
        for (int g = 0; g < P::GROUPS; ++g) mbar_init(&mma_bar[g], 1);
        *consumed = 0;
        fence_barrier_init();
    }
    fence_proxy_async_smem();
    if constexpr (P::TC) asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if constexpr (P::TC) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem0 = P::TC ? *tmem_slot : 0u;
    const uint32_t tx_bytes = 2u * kIonTile * (uint32_t)n3 * (uint32_t)sizeof(R);
    bool failed = false;

    if (warp == P::CONSUMERS / 32) {
        /* ------------------------------------------------------ producer */
        const int lane = tid & 31;
        int issued = 0;
        /* lane 0: once the consumers are done with tile kk, its stage goes back
         * with one tensor store per array (the consumers never wait for it) */
        auto store_tile = [&](int kk) -> bool {
            if (!mbar_wait(&empty[kk % S], (kk / S) & 1)) return false;
            const int x = ((int)blockIdx.x + kk * (int)gridDim.x) * kIonTile;
            unsigned char* b = stages + (kk % S) * P::STAGE;
            tma_store_3d(&maps.r, b, x, 0, 0);
            tma_store_3d(&maps.v, b + P::BOX, x, 0, 0);
            bulk_commit();
            return true;
        };
        /* cell offsets of this lane's slots of tile kk (-1 past the pool) */
        int64_t cells[kIonTile / 32];
        auto fetch_cells = [&](int kk) {
            const int64_t xk = (int64_t)((int)blockIdx.x + kk * (int)gridDim.x) * kIonTile;
#pragma unroll
            for (int u = 0; u < kIonTile / 32; ++u) {
                const int64_t sl = xk + lane + 32 * u;
                cells[u] = sl < a.nslot ? a.slot_cell[sl] : -1;
            }
        };
        if (mine > 0) fetch_cells(0);
        for (int k = 0; k < mine; ++k) {
            const int st = k % S;
            bool ok = true;
            if (k >= S && lane == 0) {
                ok = store_tile(k - S);
                if (ok) bulk_wait_read0(); /* the stage is free once the store has read it */
            }
            if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) {
                failed = true;
                break;
            }
            const int x = ((int)blockIdx.x + k * (int)gridDim.x) * kIonTile;
            unsigned char* b = stages + st * P::STAGE;
            if (lane == 0) {
                /* slots left in this tile: a multiple of 32 (the pool is padded) */
                const uint32_t nrem = (uint32_t)min((int64_t)kIonTile, a.nslot - x);
                mbar_arrive_expect_tx(&full[st], tx_bytes + nrem * 13u);
                tma_load_3d(b, &maps.r, &full[st], x, 0, 0);
                tma_load_3d(b + P::BOX, &maps.v, &full[st], x, 0, 0);
                bulk_load(b + 2 * P::BOX, a.slot_cell + x, nrem * 8u, &full[st]);
                bulk_load(b + 2 * P::BOX + 1024, a.slot_n3 + x, nrem * 4u, &full[st]);
                bulk_load(b + 2 * P::BOX + 1536, a.slot_mat + x, nrem, &full[st]);
            }
            /* E^{n+1} of the tile's cells, gathered ahead like the rest of the
             * stage (padding slots repeat the last cell; slots past the pool
             * are not read); their cell offsets were read one tile ahead */
            R* es = reinterpret_cast<R*>(b + P::E_OFF);
#pragma unroll
            for (int u = 0; u < kIonTile / 32; ++u) {
                const int t = lane + 32 * u;
                const int64_t c = cells[u];
                if (c >= 0) {
                    cp_async_ca<sizeof(R)>(es + t, a.ex + c);
                    cp_async_ca<sizeof(R)>(es + kIonTile + t, a.ey + c);
                    cp_async_ca<sizeof(R)>(es + 2 * kIonTile + t, a.ez + c);
                }
            }
            cp_async_arrive_noinc(&full[st]);
            issued = k + 1;
            if (k + 1 < mine) fetch_cells(k + 1);
        }
        if (lane == 0 && !failed)
            for (int kk = max(0, mine - S); kk < mine && !failed; ++kk) failed = !store_tile(kk);
        if (failed && lane == 0) {
            atomicExch(a.err, 1);
            /* loads issued and not consumed land before the CTA leaves */
            for (int k = *consumed; k < issued; ++k) mbar_wait(&full[k % S], (k / S) & 1);
        }
        if (lane == 0) bulk_wait0(); /* stores complete before the CTA leaves */
    } else {
        /* ------------------------------------------------------ consumers */
        const int g = tid / P::GT, gi = tid % P::GT, gt = gi & (kIonTile - 1), bar_id = 1 + g;
        /* FP64: threads gi >= 128 take part in the contraction only */
        const bool cell_thread = gi < kIonTile;
        const int64_t ns = a.nslot;
        const R dt = R(a.dt);
        unsigned char* Ahi = ops + g * 2 * P::A_BYTES;
        unsigned char* Alo = Ahi + P::A_BYTES;
        const unsigned char* Bhi = ops + P::GROUPS * 2 * P::A_BYTES;
        const unsigned char* Blo = Bhi + P::B_BYTES;
        const double* Bfrag = reinterpret_cast<const double*>(ops);
        const uint32_t tmem = tmem0 + (uint32_t)(g * ion_cols<NP>());
        uint32_t mphase = 0;
        for (int k = g; k < mine; k += P::GROUPS) {
            const int st = k % S;
            const int64_t s = (int64_t)((int)blockIdx.x + k * (int)gridDim.x) * kIonTile + gt;
            const bool got = mbar_wait(&full[st], (k / S) & 1);
            if (named_sync_or(bar_id, P::GT, !got)) {
                failed = true;
                break;
            }
            unsigned char* sb = stages + st * P::STAGE;
            R* rs = reinterpret_cast<R*>(sb);
            R* vs = reinterpret_cast<R*>(sb + P::BOX);
            const int n3c = (cell_thread && s < ns) ? reinterpret_cast<const int32_t*>(sb + 2 * P::BOX + 1024)[gt] : 0;
            R e0 = R(0), e1 = R(0), e2 = R(0);
            const MatCoef<R>* mp = nullptr;
            if (n3c) {
                const R* es = reinterpret_cast<const R*>(sb + P::E_OFF);
                mp = &a.mc[(sb + 2 * P::BOX + 1536)[gt]];
                e0 = es[gt];
                e1 = es[kIonTile + gt];
                e2 = es[2 * kIonTile + gt];
                rot_fwd<false>(mp->flags, mp->cs, mp->sn, e0, e1, e2);
            }
            R p0 = R(0), p1 = R(0), p2 = R(0);
            const R* qv = n3c ? (mp->ion_off == a.ion_off_ref ? coef : a.ion_coef + mp->ion_off) : nullptr;
            const R* qm = n3c ? qv + 3 * n3c : nullptr;
            if constexpr (P::TC) {
                /* A rows (this cell) as bf16 hi + lo */
#pragma unroll
                for (int kc = 0; kc < NP / 8; ++kc) {
                    uint32_t h[4], l[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int q = kc * 8 + 2 * u;
                        const float x0 = q < n3 ? (float)rs[q * kIonTile + gt] : 0.f;
                        const float x1 = q + 1 < n3 ? (float)rs[(q + 1) * kIonTile + gt] : 0.f;
                        const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
                        const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
                        const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
                        h[u] = bf16x2_bits(h0, h1);
                        l[u] = bf16x2_bits(l0, l1);
                    }
                    const uint32_t off = umma_kmajor_off(gt, kc * 8, kIonTile);
                    *reinterpret_cast<uint4*>(Ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<uint4*>(Alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
                }
                fence_proxy_async_smem();
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                named_sync(bar_id, P::GT);
                if (gt == 0) {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t idesc = umma_idesc_bf16(kIonTile, NP);
                    const uint32_t sa_hi = smem_addr(Ahi), sa_lo = smem_addr(Alo);
                    const uint32_t sb_hi = smem_addr(Bhi), sb_lo = smem_addr(Blo);
#pragma unroll
                    for (int ks = 0; ks < NP / 16; ++ks) {
                        const uint32_t ao = umma_kmajor_off(0, ks * 16, kIonTile), bo = umma_kmajor_off(0, ks * 16, NP);
                        const uint64_t dah = umma_smem_desc(sa_hi + ao, kIonTile * 16, 128);
                        const uint64_t dal = umma_smem_desc(sa_lo + ao, kIonTile * 16, 128);
                        const uint64_t dbh = umma_smem_desc(sb_hi + bo, NP * 16, 128);
                        const uint64_t dbl = umma_smem_desc(sb_lo + bo, NP * 16, 128);
                        const uint32_t acc0 = ks > 0 ? 1u : 0u;
                        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                     " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                                     ::"r"(tmem), "l"(dah), "l"(dbh), "r"(idesc), "r"(acc0));
                        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                     " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                                     ::"r"(tmem), "l"(dah), "l"(dbl), "r"(idesc), "r"(1u));
                        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                     " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                                     ::"r"(tmem), "l"(dal), "l"(dbh), "r"(idesc), "r"(1u));
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_addr(&mma_bar[g]))
                                 : "memory");
                }
                const bool done = mbar_wait(&mma_bar[g], mphase);
                mphase ^= 1u;
                if (named_sync_or(bar_id, P::GT, !done)) {
                    failed = true;
                    if (gt == 0) mbar_wait(&mma_bar[g], mphase ^ 1u); /* the MMAs in flight finish first */
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                /* epilogue with the coefficients from shared memory when every
                 * cell of the warp has the lattice's, else through qv, qm (the
                 * choice is warp-uniform: tcgen05.ld is warp-collective) */
                auto epilogue = [&](const R* zv, const R* zm) {
#pragma unroll
                for (int cb = 0; cb < NP; cb += 16) {
                    uint32_t d[16];
                    const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)cb;
                    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                                 : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                                   "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
                                   "=r"(d[14]), "=r"(d[15])
                                 : "r"(taddr));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int q = cb + u;
                        if (q < n3c) {
                            const int at = q / 3, dd = q - 3 * at;
                            const R acc = zm[at * 9 + dd] * e0 + zm[at * 9 + 3 + dd] * e1 + zm[at * 9 + 6 + dd] * e2 -
                                          __uint_as_float(d[u]);
                            const int o = q * kIonTile + gt;
                            const R vq = vs[o];
                            const R rn = rs[o] + (vq * dt + R(0.5) * acc * dt * dt);
                            rs[o] = rn;
                            vs[o] = vq + acc * dt;
                            p0 += zv[at * 9 + dd] * rn;
                            p1 += zv[at * 9 + 3 + dd] * rn;
                            p2 += zv[at * 9 + 6 + dd] * rn;
                        }
                    }
                }
                };
                const bool lattice = !n3c || mp->ion_off == a.ion_off_ref;
                if (__all_sync(0xffffffffu, lattice)) epilogue(coef, coef + 3 * n3c);
                else epilogue(qv, qm);
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            } else {
                /* FP64: DMM . r on the FP64 tensor path (mma.sync m8n8k4).
                 * Each thread leaves its cell's crystal-frame E and the
                 * offset of its QeZV, QeZM in the stage; then each warp
                 * takes its 32 cells, 16 at a time: the accumulators hold
                 * (DMM . r)[cell][q] for two 8-cell rows and all NP columns,
                 * and the lanes that hold a (cell, q) pair update that
                 * coordinate's r and v in the stage. */
                R* es = reinterpret_cast<R*>(sb + P::E_OFF);
                int64_t* qoff = reinterpret_cast<int64_t*>(sb + 2 * P::BOX); /* slot cells, no longer read */
                const int32_t* n3s = reinterpret_cast<const int32_t*>(sb + 2 * P::BOX + 1024);
                if (cell_thread) {
                    es[gt] = e0;
                    es[kIonTile + gt] = e1;
                    es[2 * kIonTile + gt] = e2;
                    qoff[gt] = n3c ? (mp->ion_off == a.ion_off_ref ? -1 : (int64_t)mp->ion_off) : 0;
                }
                named_sync(bar_id, P::GT);
                const int lane = tid & 31, grp = lane >> 2, tig = lane & 3;
                const int64_t x0 = (int64_t)((int)blockIdx.x + k * (int)gridDim.x) * kIonTile;
#pragma unroll 1
                for (int pass = 0; pass < P::CELLS_PER_WARP / 16; ++pass) {
                    const int cb = (gi >> 5) * P::CELLS_PER_WARP + pass * 16;
                    int n3l[2];
                    bool lat = true;
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        const int cl = cb + 8 * mt + grp;
                        n3l[mt] = x0 + cl < ns ? n3s[cl] : 0;
                        lat = lat && (n3l[mt] == 0 || qoff[cl] < 0);
                    }
                    /* every cell of the 16 has the lattice's coefficients: QeZM . E
                     * joins the contraction as one more k step and P_ion = QeZV . r
                     * is a second contraction (warp-uniform choice) */
                    const bool fold = __all_sync(0xffffffffu, lat);
                    double acc[2][NP / 8][2];
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                        for (int nt = 0; nt < NP / 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
#pragma unroll 4
                    for (int ks = 0; ks < NP / 4; ++ks) {
                        const int kk = ks * 4 + tig;
                        /* rows past 3N hold no data: A is zero there */
                        const double a0 = kk < n3 ? (double)rs[kk * kIonTile + cb + grp] : 0.0;
                        const double a1 = kk < n3 ? (double)rs[kk * kIonTile + cb + 8 + grp] : 0.0;
#pragma unroll
                        for (int nt = 0; nt < NP / 8; ++nt) {
                            const double b = Bfrag[(ks * (NP / 8) + nt) * 32 + lane];
                            dmma_8x8x4(acc[0][nt][0], acc[0][nt][1], a0, b);
                            dmma_8x8x4(acc[1][nt][0], acc[1][nt][1], a1, b);
                        }
                    }
                    if (fold) {
                        const double a0 = tig < 3 ? (double)es[tig * kIonTile + cb + grp] : 0.0;
                        const double a1 = tig < 3 ? (double)es[tig * kIonTile + cb + 8 + grp] : 0.0;
#pragma unroll
                        for (int nt = 0; nt < NP / 8; ++nt) {
                            const double b = Bfrag[P::FRAG_E + nt * 32 + lane];
                            dmma_8x8x4(acc[0][nt][0], acc[0][nt][1], a0, b);
                            dmma_8x8x4(acc[1][nt][0], acc[1][nt][1], a1, b);
                        }
                        /* acc = DMM . r - QeZM . E = -a.  The update goes cell-major:
                         * lane l takes cell cb + l % 16 and, per step, the coordinate
                         * q of columns 2t + j with t = t2 + 2 (l / 16), shuffled in
                         * from the lane that holds it, so that each shared-memory
                         * access covers 16 consecutive cells of two rows (no bank
                         * conflicts; the accumulator layout would give four rows) */
                        const int me = lane & 15, half = lane >> 4;
                        const int cme = cb + me;
                        const bool live_me = x0 + cme < ns && n3s[cme] != 0;
#pragma unroll
                        for (int nt = 0; nt < NP / 8; ++nt)
#pragma unroll
                            for (int j = 0; j < 2; ++j)
#pragma unroll
                                for (int t2 = 0; t2 < 2; ++t2) {
                                    const int t = t2 + 2 * half;
                                    const int src = (me & 7) * 4 + t;
                                    const double v0 = __shfl_sync(0xffffffffu, acc[0][nt][j], src);
                                    const double v1 = __shfl_sync(0xffffffffu, acc[1][nt][j], src);
                                    const int q = nt * 8 + 2 * t + j;
                                    if (live_me && q < n3) {
                                        const R acc_q = -(R)(me < 8 ? v0 : v1);
                                        const int o = q * kIonTile + cme;
                                        const R vq = vs[o];
                                        rs[o] = rs[o] + (vq * dt + R(0.5) * acc_q * dt * dt);
                                        vs[o] = vq + acc_q * dt;
                                    }
                                }
                        __syncwarp();
                        /* P_ion = QeZV . r^{n+1}: lanes t = 0, 1 of each cell hold
                         * components 2t, 2t + 1 */
                        double pa[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 4
                        for (int ks = 0; ks < NP / 4; ++ks) {
                            const int kk = ks * 4 + tig;
                            const double a0 = kk < n3 ? (double)rs[kk * kIonTile + cb + grp] : 0.0;
                            const double a1 = kk < n3 ? (double)rs[kk * kIonTile + cb + 8 + grp] : 0.0;
                            const double b = Bfrag[P::FRAG_P + ks * 32 + lane];
                            dmma_8x8x4(pa[0][0], pa[0][1], a0, b);
                            dmma_8x8x4(pa[1][0], pa[1][1], a1, b);
                        }
#pragma unroll
                        for (int mt = 0; mt < 2; ++mt) {
                            const int64_t sl = x0 + cb + 8 * mt + grp;
                            if (n3l[mt] && tig == 0) {
                                a.pr[sl] = (R)pa[mt][0];
                                a.pr[ns + sl] = (R)pa[mt][1];
                            }
                            if (n3l[mt] && tig == 1) a.pr[2 * ns + sl] = (R)pa[mt][0];
                        }
                        continue;
                    }
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        const int cl = cb + 8 * mt + grp;
                        R q0 = R(0), q1 = R(0), q2 = R(0);
                        /* cells of several materials: QeZM . E and QeZV . r from
                         * each cell's coefficients in global memory */
                        if (n3l[mt]) {
                            const int64_t qo = qoff[cl];
                            const R* zv = a.ion_coef + (qo < 0 ? (int64_t)a.ion_off_ref : qo);
                            const R* zm = zv + 3 * n3l[mt];
                            const R ex0 = es[cl], ex1 = es[kIonTile + cl], ex2 = es[2 * kIonTile + cl];
#pragma unroll
                            for (int nt = 0; nt < NP / 8; ++nt)
#pragma unroll
                                for (int j = 0; j < 2; ++j) {
                                    const int q = nt * 8 + 2 * tig + j;
                                    if (q < n3l[mt]) {
                                        const int at = q / 3, dd = q - 3 * at;
                                        const R acc_q = zm[at * 9 + dd] * ex0 + zm[at * 9 + 3 + dd] * ex1 +
                                                        zm[at * 9 + 6 + dd] * ex2 - (R)acc[mt][nt][j];
                                        const int o = q * kIonTile + cl;
                                        const R vq = vs[o];
                                        const R rn = rs[o] + (vq * dt + R(0.5) * acc_q * dt * dt);
                                        rs[o] = rn;
                                        vs[o] = vq + acc_q * dt;
                                        q0 += zv[at * 9 + dd] * rn;
                                        q1 += zv[at * 9 + 3 + dd] * rn;
                                        q2 += zv[at * 9 + 6 + dd] * rn;
                                    }
                                }
                        }
                        /* P_ion of the cell: the sum over its four lanes */
#pragma unroll
                        for (int m = 1; m < 4; m <<= 1) {
                            q0 += __shfl_xor_sync(0xffffffffu, q0, m);
                            q1 += __shfl_xor_sync(0xffffffffu, q1, m);
                            q2 += __shfl_xor_sync(0xffffffffu, q2, m);
                        }
                        if (n3l[mt] && tig == 0) {
                            const int64_t sl = x0 + cl;
                            a.pr[sl] = q0;
                            a.pr[ns + sl] = q1;
                            a.pr[2 * ns + sl] = q2;
                        }
                    }
                }
            }
            if (P::TC && n3c) {
                a.pr[s] = p0;
                a.pr[ns + s] = p1;
                a.pr[2 * ns + s] = p2;
            }
            /* the updated tile is complete in the stage: the producer stores it
             * (the writes are ordered before the tensor store's reads by the
             * proxy fence, the barrier and the arrival) */
            fence_proxy_async_smem();
            named_sync(bar_id, P::GT);
            if (gi == 0) {
                atomicMax((int32_t*)consumed, k + 1);
                mbar_arrive(&empty[st]);
            }
        }
        if (failed && gi == 0) atomicExch(a.err, 1);
    }
    if constexpr (P::TC) asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if constexpr (P::TC) {
        if (warp == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem0),
                         "r"(P::GROUPS * ion_cols<NP>()));
        }
    }
}

} // namespace phpdev
