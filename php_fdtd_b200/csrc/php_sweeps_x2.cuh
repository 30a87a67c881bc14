/*
 * php_sweeps_x2.cuh -- the FP32 sweeps with two cells per thread along x.
 *
 * In FP32 a cell moves half the bytes of FP64 for the same instructions, and
 * the one-cell TMA sweeps become issue-bound (about 70 % issue-active on the
 * H sweep).  Here a block of 32 x 8 threads owns a 64 x 8 tile: each thread
 * updates cells i and i+1, reads its shared-memory planes as float2 pairs,
 * stores its results as float2 pairs, and pays the per-plane overhead
 * (barrier waits, CPML slot tests, index arithmetic) once for two cells.
 * Pipeline, boxes and bounded waits are those of php_sweeps_tma.cuh with the
 * wider tile; the per-cell arithmetic is the FP32 fast path of
 * php_sweeps.cuh (d_update / e_cell_values).
 */
#pragma once

namespace phpdev {

__host__ __device__ constexpr uint32_t x2_align128(uint32_t b) { return (b + 127u) / 128u * 128u; }

struct TmaGeomX2 {
    static constexpr int TX = 2 * kBlockX, TY = kBlockY;
    static constexpr int HALO = 4;                      /* 16 bytes of float */
    static constexpr int BX = TX + HALO, BY = TY + 1;
    static constexpr uint32_t HALO_BYTES = BX * BY * 4, OWN_BYTES = TX * TY * 4, MAT_BYTES = TX * TY;
    __host__ __device__ static constexpr uint32_t align128(uint32_t b) { return x2_align128(b); }
    static constexpr uint32_t H_STAGE = x2_align128(3 * x2_align128(HALO_BYTES) + 3 * x2_align128(OWN_BYTES));
    static constexpr uint32_t E_STAGE =
        x2_align128(3 * x2_align128(HALO_BYTES) + 3 * x2_align128(OWN_BYTES) + x2_align128(MAT_BYTES));
    static constexpr int HS = 4, ES = 3;
    static constexpr uint32_t H_SMEM = 128 + HS * H_STAGE + HS * 8;
    static constexpr uint32_t E_SMEM = 128 + ES * E_STAGE + 128;
};

__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float x, float y) { *reinterpret_cast<float2*>(p) = make_float2(x, y); }

/* ================================================================ H sweep */

__global__ void __launch_bounds__(kBlockX * kBlockY) h_sweep_x2(const __grid_constant__ StepArgs<float> a,
                                                                const __grid_constant__ TmaMaps tm)
{
    using G = TmaGeomX2;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* smem = ring_base(dyn_smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::HS * G::H_STAGE);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kBlockX + tx;
    const int i0 = blockIdx.x * G::TX, j0 = blockIdx.y * G::TY;
    const int i = i0 + 2 * tx, j = j0 + ty;
    const int k0 = blockIdx.z * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return;

    constexpr uint32_t EB = G::align128(G::HALO_BYTES), HB = G::align128(G::OWN_BYTES);
    auto stage = [&](int p) -> unsigned char* { return smem + (uint32_t)((p - k0) % G::HS) * G::H_STAGE; };
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
        for (int s = 0; s < G::HS; ++s) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int p = k0; p <= min(k1, k0 + G::HS - 1); ++p) issue(p);

    const bool jok = j < a.ny - 1;
    const bool act0 = jok && i < a.nx - 1, act1 = jok && i + 1 < a.nx - 1;
    const int L2 = 2 * a.L;
    const int nxp = a.nxp, ny = a.ny;
    const int sx0 = act0 ? ldg(a.tx.slot + i) : -1, sx1 = act1 ? ldg(a.tx.slot + i + 1) : -1;
    const int sy = act0 ? ldg(a.ty.slot + j) : -1;
    const float khx0 = act0 ? ldg(a.tx.kh + i) : 0.f, khx1 = act1 ? ldg(a.tx.kh + i + 1) : 0.f;
    const float khy = act0 ? ldg(a.ty.kh + j) : 0.f;
    float* __restrict__ hxg = a.f.hx;
    float* __restrict__ hyg = a.f.hy;
    float* __restrict__ hzg = a.f.hz;
    const int eo = ty * G::BX + 2 * tx;
    const int ho = ty * G::TX + 2 * tx;

    for (int k = k0; k < k1; ++k) {
        const int sz = ldg_nh(a.tz.slot + k);
        const float khz = ldg_nh(a.tz.kh + k);
        bool ok = true;
        if (k == k0) ok = mbar_wait(&full[0], 0);
        ok = ok && mbar_wait(&full[(k + 1 - k0) % G::HS], ((k + 1 - k0) / G::HS) & 1);
        if (ok && act0) {
            const unsigned char* b0 = stage(k);
            const unsigned char* b1 = stage(k + 1);
            const float* Ex0 = reinterpret_cast<const float*>(b0);
            const float* Ey0 = reinterpret_cast<const float*>(b0 + EB);
            const float* Ez0 = reinterpret_cast<const float*>(b0 + 2 * EB);
            const float* Ex1 = reinterpret_cast<const float*>(b1);
            const float* Ey1 = reinterpret_cast<const float*>(b1 + EB);
            const float2 ex0 = ld2(Ex0 + eo), ey0 = ld2(Ey0 + eo), ez0 = ld2(Ez0 + eo);
            const float2 ex1 = ld2(Ex1 + eo), ey1 = ld2(Ey1 + eo);
            const float2 ezr = ld2(Ez0 + eo + 2), eyr = ld2(Ey0 + eo + 2); /* cells i+2, i+3 */
            const float2 ezj = ld2(Ez0 + eo + G::BX), exj = ld2(Ex0 + eo + G::BX);
            const float2 hx = ld2(reinterpret_cast<const float*>(b0 + 3 * EB) + ho);
            const float2 hy = ld2(reinterpret_cast<const float*>(b0 + 3 * EB + HB) + ho);
            const float2 hz = ld2(reinterpret_cast<const float*>(b0 + 3 * EB + 2 * HB) + ho);
            /* differences of both cells: .x cell i, .y cell i+1 */
            const float dEyz0 = ey1.x - ey0.x, dEyz1 = ey1.y - ey0.y;
            const float dExz0 = ex1.x - ex0.x, dExz1 = ex1.y - ex0.y;
            const float dEzy0 = ezj.x - ez0.x, dEzy1 = ezj.y - ez0.y;
            const float dExy0 = exj.x - ex0.x, dExy1 = exj.y - ex0.y;
            const float dEzx0 = ez0.y - ez0.x, dEzx1 = ezr.x - ez0.y;
            const float dEyx0 = ey0.y - ey0.x, dEyx1 = eyr.x - ey0.y;
            float ux0 = -khy * dEzy0 + khz * dEyz0, ux1 = -khy * dEzy1 + khz * dEyz1;
            float uy0 = khx0 * dEzx0 - khz * dExz0, uy1 = khx1 * dEzx1 - khz * dExz1;
            float uz0 = -khx0 * dEyx0 + khy * dExy0, uz1 = -khx1 * dEyx1 + khy * dExy1;
            const int c = (k * ny + j) * nxp + i;
            /* CPML psi (fdtd.c:3143-3228), folded as in h_sweep_tma */
            if (sx0 >= 0) {
                const int q = (k * ny + j) * L2 + sx0;
                const float bb = ldg_nh(a.tx.b + i), ch = ldg_nh(a.tx.ch + i);
                const float pxy = a.psi.hxy[q], pxz = a.psi.hxz[q];
                uy0 += pxy;
                uz0 += pxz;
                a.psi.hxy[q] = bb * pxy + ch * dEzx0;
                a.psi.hxz[q] = bb * pxz - ch * dEyx0;
            }
            if (sx1 >= 0) {
                const int q = (k * ny + j) * L2 + sx1;
                const float bb = ldg_nh(a.tx.b + i + 1), ch = ldg_nh(a.tx.ch + i + 1);
                const float pxy = a.psi.hxy[q], pxz = a.psi.hxz[q];
                uy1 += pxy;
                uz1 += pxz;
                a.psi.hxy[q] = bb * pxy + ch * dEzx1;
                a.psi.hxz[q] = bb * pxz - ch * dEyx1;
            }
            if (sy >= 0) {
                const int q = (k * L2 + sy) * nxp + i;
                const float bb = ldg_nh(a.ty.b + j), ch = ldg_nh(a.ty.ch + j);
                const float2 pyx = ld2(a.psi.hyx + q), pyz = ld2(a.psi.hyz + q);
                ux0 += pyx.x;
                ux1 += pyx.y;
                uz0 += pyz.x;
                uz1 += pyz.y;
                if (act1) {
                    st2(a.psi.hyx + q, bb * pyx.x - ch * dEzy0, bb * pyx.y - ch * dEzy1);
                    st2(a.psi.hyz + q, bb * pyz.x + ch * dExy0, bb * pyz.y + ch * dExy1);
                } else {
                    a.psi.hyx[q] = bb * pyx.x - ch * dEzy0;
                    a.psi.hyz[q] = bb * pyz.x + ch * dExy0;
                }
            }
            if (sz >= 0) {
                const int q = (sz * ny + j) * nxp + i;
                const float bb = ldg_nh(a.tz.b + k), ch = ldg_nh(a.tz.ch + k);
                const float2 pzx = ld2(a.psi.hzx + q), pzy = ld2(a.psi.hzy + q);
                ux0 += pzx.x;
                ux1 += pzx.y;
                uy0 += pzy.x;
                uy1 += pzy.y;
                if (act1) {
                    st2(a.psi.hzx + q, bb * pzx.x + ch * dEyz0, bb * pzx.y + ch * dEyz1);
                    st2(a.psi.hzy + q, bb * pzy.x - ch * dExz0, bb * pzy.y - ch * dExz1);
                } else {
                    a.psi.hzx[q] = bb * pzx.x + ch * dEyz0;
                    a.psi.hzy[q] = bb * pzy.x - ch * dExz0;
                }
            }
            if (act1) {
                st2(hxg + c, hx.x + ux0, hx.y + ux1);
                st2(hyg + c, hy.x + uy0, hy.y + uy1);
                st2(hzg + c, hz.x + uz0, hz.y + uz1);
            } else {
                hxg[c] = hx.x + ux0;
                hyg[c] = hy.x + uy0;
                hzg[c] = hz.x + uz0;
            }
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(a.err, 1);
            break;
        }
        if (tid == 0 && k + G::HS <= k1) {
            fence_proxy_async_smem();
            issue(k + G::HS);
        }
    }
}

/* ================================================================ E sweep */

template <int NAMAX>
__global__ void __launch_bounds__(kBlockX * kBlockY, 3) e_sweep_x2(const __grid_constant__ StepArgs<float> a,
                                                                   const __grid_constant__ TmaMaps tm)
{
    using G = TmaGeomX2;
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* smem = ring_base(dyn_smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::ES * G::E_STAGE);

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kBlockX + tx;
    const int i0 = blockIdx.x * G::TX, j0 = blockIdx.y * G::TY;
    const int i = i0 + 2 * tx, j = j0 + ty;
    const int k0 = blockIdx.z * a.zchunk;
    const int k1 = min(k0 + a.zchunk, a.nz);
    if (k0 >= k1) return;

    constexpr uint32_t HB = G::align128(G::HALO_BYTES), OB = G::align128(G::OWN_BYTES);
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
    if (tid == 0) {
        for (int s = 0; s < G::ES; ++s) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int p = k0 - 1; p <= min(k1 - 1, k0 - 1 + G::ES - 1); ++p) issue(p);

    const bool jok = j < a.ny;
    const bool act0 = jok && i < a.nx, act1 = jok && i + 1 < a.nx;
    const bool jin = j >= 1 && j < a.ny - 1;
    const bool int0 = jin && i >= 1 && i < a.nx - 1, int1 = jin && i + 1 < a.nx - 1;
    const int sx0 = act0 ? ldg(a.tx.slot + i) : -1, sx1 = act1 ? ldg(a.tx.slot + i + 1) : -1;
    const int sy = act0 ? ldg(a.ty.slot + j) : -1;
    const int ho = (ty + 1) * G::BX + 2 * tx + G::HALO; /* cell i in a halo box */
    const int oo = ty * G::TX + 2 * tx;                 /* cell i in an own box */

    for (int k = k0; k < k1; ++k) {
        CellPsi<float> ps0, ps1;
        ps0.sz = ps1.sz = -1;
        if (int0) load_psi_d(a, i, j, k, sx0, sy, ps0);
        if (int1) load_psi_d(a, i + 1, j, k, sx1, sy, ps1);
        bool ok = true;
        if (k == k0) ok = mbar_wait(&full[0], 0);
        ok = ok && mbar_wait(&full[(k - k0 + 1) % G::ES], ((k - k0 + 1) / G::ES) & 1);
        if (ok && act0) {
            const unsigned char* bp = stage(k - 1);
            const unsigned char* bc = stage(k);
            const float* Hxp = reinterpret_cast<const float*>(bp);
            const float* Hyp = reinterpret_cast<const float*>(bp + HB);
            const float* Hx = reinterpret_cast<const float*>(bc);
            const float* Hy = reinterpret_cast<const float*>(bc + HB);
            const float* Hz = reinterpret_cast<const float*>(bc + 2 * HB);
            const float* Dx = reinterpret_cast<const float*>(bc + 3 * HB);
            const float* Dy = reinterpret_cast<const float*>(bc + 3 * HB + OB);
            const float* Dz = reinterpret_cast<const float*>(bc + 3 * HB + 2 * OB);
            const uint8_t* M = reinterpret_cast<const uint8_t*>(bc + 3 * HB + 3 * OB);
            const float2 hx = ld2(Hx + ho), hy = ld2(Hy + ho), hz = ld2(Hz + ho);
            const float2 hxk = ld2(Hxp + ho), hyk = ld2(Hyp + ho);
            const float2 hzj = ld2(Hz + ho - G::BX), hxj = ld2(Hx + ho - G::BX);
            const float2 hzl = ld2(Hz + ho - 2), hyl = ld2(Hy + ho - 2); /* .y: cell i-1 */
            float2 d0 = ld2(Dx + oo), d1 = ld2(Dy + oo), d2 = ld2(Dz + oo);
            const int mid0 = M[oo], mid1 = M[oo + 1];
            const int c = (k * a.ny + j) * a.nxp + i;
            float ex0, ey0, ez0;
            e_cell_values<float, false, NAMAX>(a, i, j, k, c, int0, sx0, sy, hx.x, hy.x, hz.x, hxk.x, hyk.x, hzj.x,
                                               hxj.x, hzl.y, hyl.y, d0.x, d1.x, d2.x, mid0, nullptr, &ps0, ex0, ey0,
                                               ez0);
            if (act1) {
                float ex1, ey1, ez1;
                e_cell_values<float, false, NAMAX>(a, i + 1, j, k, c + 1, int1, sx1, sy, hx.y, hy.y, hz.y, hxk.y,
                                                   hyk.y, hzj.y, hxj.y, hz.x, hy.x, d0.y, d1.y, d2.y, mid1, nullptr,
                                                   &ps1, ex1, ey1, ez1);
                st2(a.f.dx + c, d0.x, d0.y);
                st2(a.f.dy + c, d1.x, d1.y);
                st2(a.f.dz + c, d2.x, d2.y);
                st2(a.f.ex + c, ex0, ex1);
                st2(a.f.ey + c, ey0, ey1);
                st2(a.f.ez + c, ez0, ez1);
            } else {
                a.f.dx[c] = d0.x;
                a.f.dy[c] = d1.x;
                a.f.dz[c] = d2.x;
                a.f.ex[c] = ex0;
                a.f.ey[c] = ey0;
                a.f.ez[c] = ez0;
            }
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(a.err, 1);
            break;
        }
        if (tid == 0 && k - 1 + G::ES <= k1 - 1) {
            fence_proxy_async_smem();
            issue(k - 1 + G::ES);
        }
    }
}

} // namespace phpdev
