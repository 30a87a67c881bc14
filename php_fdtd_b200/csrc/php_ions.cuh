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
 *  ion_update_cc  CUDA cores, FP64 (the fast plain path): DMM in shared
 *                 memory, one cell per thread.
 *  ion_update_tc  FP32 mixed path on the 5th-generation tensor cores: per
 *                 128-cell tile, r is split into bf16 hi + lo, DMM likewise
 *                 (host), and D = r_hi DMM_hi^T + r_hi DMM_lo^T + r_lo DMM_hi^T
 *                 accumulates in FP32 in tensor memory (tcgen05.mma
 *                 kind::f16, M = 128, N = K = 3N padded to 16); the
 *                 epilogue reads D with tcgen05.ld and does the update.  The
 *                 dropped r_lo DMM_lo term and the bf16 representation leave
 *                 about 2^-17 relative error in DMM . r.
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
    const uint8_t* mat;
    const MatCoef<R>* mc;
    const R* ion_coef;
    const R* dmm;                /* [NP][NP], zero padded (CUDA-core kernel) */
    const uint32_t* bsplit;      /* DMM hi, lo as bf16 in the UMMA K-major layout (tensor kernel) */
    int64_t nslot;
    int32_t ntiles;
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

template <int NP>
struct IonTc {
    static constexpr int COLS = NP <= 32 ? 32 : NP <= 64 ? 64 : 128;   /* TMEM columns */
    static constexpr uint32_t A_BYTES = kIonTile * NP * 2;
    static constexpr uint32_t B_BYTES = NP * NP * 2;
    /* A_hi, A_lo, B_hi, B_lo, then the barrier and the TMEM address */
    static constexpr uint32_t SMEM = 1024 + 2 * A_BYTES + 2 * B_BYTES + 64;
};

template <int NP>
__global__ void __launch_bounds__(kIonTile, 4) ion_update_tc(const IonArgs<float> a)
{
    using T = IonTc<NP>;
    static_assert(NP % 16 == 0 && NP >= 16 && NP <= 64, "3N padded to 16..64");
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* base = dyn_smem + ((1024u - (smem_addr(dyn_smem) & 1023u)) & 1023u);
    unsigned char* Ahi = base;
    unsigned char* Alo = base + T::A_BYTES;
    unsigned char* Bhi = base + 2 * T::A_BYTES;
    unsigned char* Blo = Bhi + T::B_BYTES;
    uint64_t* bar = reinterpret_cast<uint64_t*>(Blo + T::B_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    /* B operands: host-prepared bf16 images, copied once */
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.bsplit);
        uint4* dst = reinterpret_cast<uint4*>(Bhi);
        for (int t = tid; t < (int)(2 * T::B_BYTES / 16); t += kIonTile) dst[t] = src[t];
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(T::COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    fence_proxy_async_smem(); /* B images written with generic stores */
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc_bf16(kIonTile, NP);
    const uint32_t sa_hi = smem_addr(Ahi), sa_lo = smem_addr(Alo), sb_hi = smem_addr(Bhi), sb_lo = smem_addr(Blo);
    const float dt = (float)a.dt;
    const int64_t ns = a.nslot;
    bool ok = true;
    uint32_t phase = 0;

    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int64_t s = (int64_t)tile * kIonTile + tid;
        const bool valid = s < ns;
        const int n3 = valid ? a.slot_n3[s] : 0;
        /* the dependent gather slot -> cell -> material -> E goes first */
        float e0 = 0.f, e1 = 0.f, e2 = 0.f;
        const MatCoef<float>* mp = nullptr;
        if (n3) mp = &ion_cell_e(a, s, e0, e1, e2);
        /* r of this cell: registers (FP32) and bf16 hi/lo rows of A */
        float rold[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) rold[q] = q < n3 ? a.r[(int64_t)q * ns + s] : 0.f;
#pragma unroll
        for (int kc = 0; kc < NP / 8; ++kc) {
            uint32_t h[4], l[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float x0 = rold[kc * 8 + 2 * u], x1 = rold[kc * 8 + 2 * u + 1];
                const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
                const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
                const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
                h[u] = bf16x2_bits(h0, h1);
                l[u] = bf16x2_bits(l0, l1);
            }
            const uint32_t off = umma_kmajor_off(tid, kc * 8, kIonTile);
            *reinterpret_cast<uint4*>(Ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4*>(Alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
        }
        fence_proxy_async_smem();
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
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
                             smem_addr(bar))
                         : "memory");
        }
        const bool got = mbar_wait(bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!got)) {
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

        /* epilogue: this thread's row of D, 16 columns at a time */
        float p0 = 0.f, p1 = 0.f, p2 = 0.f;
        const float* qv = n3 ? a.ion_coef + mp->ion_off : nullptr;
        const float* qm = n3 ? qv + 3 * n3 : nullptr;
#pragma unroll
        for (int cb = 0; cb < NP; cb += 16) {
            uint32_t d[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                           "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
                           "=r"(d[14]), "=r"(d[15])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int q = cb + u;
                if (q < n3) {
                    const int at = q / 3, dd = q - 3 * at;
                    const float acc = ldg(qm + at * 9 + dd) * e0 + ldg(qm + at * 9 + 3 + dd) * e1 +
                                      ldg(qm + at * 9 + 6 + dd) * e2 - __uint_as_float(d[u]);
                    const int64_t o = (int64_t)q * ns + s;
                    const float vq = a.v[o];
                    const float rn = rold[q] + (vq * dt + 0.5f * acc * dt * dt);
                    a.r[o] = rn;
                    a.v[o] = vq + acc * dt;
                    p0 += ldg(qv + at * 9 + dd) * rn;
                    p1 += ldg(qv + at * 9 + 3 + dd) * rn;
                    p2 += ldg(qv + at * 9 + 6 + dd) * rn;
                }
            }
        }
        if (n3) {
            a.pr[s] = p0;
            a.pr[ns + s] = p1;
            a.pr[2 * ns + s] = p2;
        }
        /* D has been read and A may be rewritten */
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok) {
        if (tid == 0) atomicExch(a.err, 1);
        /* the MMAs of the abandoned tile may still run: wait for them (again
         * bounded) before the tensor memory is given back */
        mbar_wait(bar, phase ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::COLS));
    }
}

} // namespace phpdev
