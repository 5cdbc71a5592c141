// sm_100a kernels of the D3Q19 acoustic step (family-B semantics of
// 06_transient_localization_dx1.cpp).  Storage is FP32 or FP16 deviations from
// rest equilibrium (see device.hpp for the HBM layout); arithmetic is FP32,
// with FP64 for the source-weight reduction and the probe accumulators.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "device.hpp"
#include "lattice.cuh"

namespace lbm {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// Scalar access.  ld: read-only path (arrays the kernel does not write);
// ldw: coherent load for arrays the same kernel also writes.
template <typename S>
struct Io;

template <>
struct Io<float>
{
    static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
    static __device__ __forceinline__ float ldw(const float* p) { return *p; }
    static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
    static __device__ __forceinline__ float rnd(float v) { return v; }   // value as stored
};

template <>
struct Io<__half>
{
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float ldw(const __half* p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
    static __device__ __forceinline__ float rnd(float v) { return __half2float(__float2half_rn(v)); }
};

// Row part of the pull offset of direction q: src = dst - ex(q) - row_off(q).
__device__ __forceinline__ long long row_off(int q, const Layout& L)
{
    return (long long)ey(q) * L.pitch + (long long)ez(q) * L.plane;
}

__device__ __forceinline__ void moments(const float (&G)[Q], float& rho, float& jx, float& jy, float& jz)
{
    rho = 0.f;
    jx = jy = jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        rho += G[q];
        if (ex(q) > 0) jx += G[q];
        if (ex(q) < 0) jx -= G[q];
        if (ey(q) > 0) jy += G[q];
        if (ey(q) < 0) jy -= G[q];
        if (ez(q) > 0) jz += G[q];
        if (ez(q) < 0) jz -= G[q];
    }
}

__device__ __forceinline__ float dot_c(int q, float x, float y, float z)
{
    float r = 0.f;
    if (ex(q) > 0) r += x;
    if (ex(q) < 0) r -= x;
    if (ey(q) > 0) r += y;
    if (ey(q) < 0) r -= y;
    if (ez(q) > 0) r += z;
    if (ez(q) < 0) r -= z;
    return r;
}

// BGK + sponge in deviation form, in place (06:940-967).  With stored
// G = scale * (f - w):
//   rho' = sum G, J = sum c G, r = 1 + rho'/scale (guard r <= 0 -> 1e-12, 06:948)
//   Geq_q = w_q (rho' + 3 c.J + (4.5 (c.J)^2 - 1.5 J^2) / (scale r))
//   G'    = (1 - sigma) (G - omega (G - Geq))      [sponge blend toward w_q, 06:955-965]
__device__ __forceinline__ void collide(float (&G)[Q], float inv_scale, float omega, float sigma)
{
    float rho, jx, jy, jz;
    moments(G, rho, jx, jy, jz);
    float r = fmaf(rho, inv_scale, 1.0f);
    if (r <= 0.f) r = 1e-12f;
    const float irs = inv_scale / r;
    const float base = rho - 1.5f * irs * (jx * jx + jy * jy + jz * jz);
    const float k45 = 4.5f * irs;
    const float keep = 1.0f - sigma;
    const float cA = keep * (1.0f - omega);
    const float cB = keep * omega;
    G[0] = fmaf(cA, G[0], cB * wf(0) * base);
#pragma unroll
    for (int p = 0; p < 9; ++p)
    {
        const int q = pair_head(p);
        const int qb = inv(q);
        const float cj = dot_c(q, jx, jy, jz);
        const float e = cB * wf(q) * fmaf(k45, cj * cj, base);
        const float o = cB * (3.0f * wf(q)) * cj;
        G[q] = fmaf(cA, G[q], e + o);
        G[qb] = fmaf(cA, G[qb], e - o);
    }
}

__device__ __forceinline__ uint32_t near_word(const StepArgs& a, const Layout& L, int col, int j, int k)
{
    return a.near[((long long)k * (L.ny + 2) + j) * L.words_per_row + (col >> 5)];
}

// Pulled populations of one cell (halo-inclusive coordinates i, j, k),
// halfway bounce-back included (06:918-931); x-halo sources read the x-face
// ghosts.  Used by the probe and field kernels.
template <typename S>
__device__ __forceinline__ void pull_cell(const S* __restrict__ f, const Layout& L, const StepArgs& sa, int i, int j,
                                          int k, float (&G)[Q], bool& solid)
{
    const long long cell = (long long)k * L.plane + (long long)j * L.pitch + (i - 1);
    const uint32_t lk = sa.links[cell];
    solid = (lk & kSolidSelfBit) != 0u;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int si = i - ex(q);
        if ((lk >> q) & 1u) G[q] = Io<S>::ld(f + (long long)inv(q) * L.pop_stride + cell);
        else if (si == 0) G[q] = sa.xf.xgh[sa.xf.gh_index(0, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else if (si == L.nx + 1) G[q] = sa.xf.xgh[sa.xf.gh_index(1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else G[q] = Io<S>::ld(f + (long long)q * L.pop_stride + cell - ex(q) - row_off(q, L));
    }
}

// ---------------------------------------------------------------- step
// Packed FP32x2 arithmetic (sm_100): both cells of a thread's pair in one
// instruction.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }

// Pair version of collide(): the same BGK + sponge update of two cells, in
// lockstep.  A SOLID cell gets cA = 1, cB = 0, so its pulled values pass
// through unchanged (06:933-938).
__device__ __forceinline__ void collide2(float2 (&G)[Q], float inv_scale, float omega, float2 sigma, bool solid0,
                                         bool solid1)
{
    // rho' and J in the family-B order (06:21-23)
    const float2 rho = add2(add2(add2(add2(G[0], G[1]), add2(G[2], G[3])), add2(add2(G[4], G[5]), add2(G[6], G[7]))),
                            add2(add2(add2(G[8], G[9]), add2(G[10], G[11])),
                                 add2(add2(add2(G[12], G[13]), add2(G[14], G[15])), add2(add2(G[16], G[17]), G[18]))));
    const float2 jx = sub2(add2(add2(add2(G[1], G[7]), add2(G[8], G[11])), G[12]),
                           add2(add2(add2(G[2], G[9]), add2(G[10], G[13])), G[14]));
    const float2 jy = sub2(add2(add2(add2(G[3], G[7]), add2(G[9], G[15])), G[16]),
                           add2(add2(add2(G[4], G[8]), add2(G[10], G[17])), G[18]));
    const float2 jz = sub2(add2(add2(add2(G[5], G[11]), add2(G[13], G[15])), G[17]),
                           add2(add2(add2(G[6], G[12]), add2(G[14], G[16])), G[18]));
    float2 r = fma2(rho, f2(inv_scale), f2(1.0f));
    if (r.x <= 0.f) r.x = 1e-12f;   // 06:948
    if (r.y <= 0.f) r.y = 1e-12f;
    const float2 irs = make_float2(__fdividef(inv_scale, r.x), __fdividef(inv_scale, r.y));
    const float2 j2 = fma2(jz, jz, fma2(jy, jy, mul2(jx, jx)));
    const float2 base = fma2(mul2(irs, j2), f2(-1.5f), rho);
    const float2 k45 = mul2(irs, f2(4.5f));
    const float2 keep = sub2(f2(1.0f), sigma);
    float2 cA = mul2(keep, f2(1.0f - omega));
    float2 cB = mul2(keep, f2(omega));
    if (solid0) cA.x = 1.0f, cB.x = 0.0f;
    if (solid1) cA.y = 1.0f, cB.y = 0.0f;
    const float2 cBw1 = mul2(cB, f2(wf(1))), cBw2 = mul2(cB, f2(wf(7)));
    const float2 cBt1 = mul2(cB, f2(3.0f * wf(1))), cBt2 = mul2(cB, f2(3.0f * wf(7)));
    G[0] = fma2(cA, G[0], mul2(mul2(cB, f2(wf(0))), base));
#pragma unroll
    for (int p = 0; p < 9; ++p)
    {
        const int q = pair_head(p);
        const int qb = inv(q);
        float2 cj;
        if (p == 0) cj = jx;                  // q = 1  ( 1, 0, 0)
        else if (p == 1) cj = jy;             // q = 3  ( 0, 1, 0)
        else if (p == 2) cj = jz;             // q = 5  ( 0, 0, 1)
        else if (p == 3) cj = add2(jx, jy);   // q = 7  ( 1, 1, 0)
        else if (p == 4) cj = sub2(jx, jy);   // q = 8  ( 1,-1, 0)
        else if (p == 5) cj = add2(jx, jz);   // q = 11 ( 1, 0, 1)
        else if (p == 6) cj = sub2(jx, jz);   // q = 12 ( 1, 0,-1)
        else if (p == 7) cj = add2(jy, jz);   // q = 15 ( 0, 1, 1)
        else cj = sub2(jy, jz);               // q = 16 ( 0, 1,-1)
        const float2 cBw = q < 7 ? cBw1 : cBw2;
        const float2 cBt = q < 7 ? cBt1 : cBt2;
        const float2 e = mul2(cBw, fma2(k45, mul2(cj, cj), base));
        const float2 o = mul2(cBt, cj);
        G[q] = fma2(cA, G[q], add2(e, o));
        G[qb] = fma2(cA, G[qb], sub2(e, o));
    }
}

template <typename S>
struct PairIo;

template <>
struct PairIo<float>
{
    using V = float2;
    static __device__ __forceinline__ V ld(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
    static __device__ __forceinline__ void st(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
    static __device__ __forceinline__ float2 cvt(V v) { return v; }
    static __device__ __forceinline__ V up(V v) { return make_float2(v.x, __shfl_up_sync(kFull, v.y, 1)); }
    static __device__ __forceinline__ V down(V v) { return make_float2(__shfl_down_sync(kFull, v.x, 1), v.y); }
    static __device__ __forceinline__ float2 left(V prev, V cur) { return make_float2(prev.y, cur.x); }
    static __device__ __forceinline__ float2 right(V cur, V next) { return make_float2(cur.y, next.x); }
    static __device__ __forceinline__ float rnd(float v) { return v; }
};

template <>
struct PairIo<__half>
{
    using V = unsigned;
    static __device__ __forceinline__ V ld(const __half* p) { return __ldg(reinterpret_cast<const unsigned*>(p)); }
    static __device__ __forceinline__ void st(__half* p, float2 v)
    {
        *reinterpret_cast<__half2*>(p) = __float22half2_rn(v);
    }
    static __device__ __forceinline__ float2 cvt(V u)
    {
        __half2 h;
        *reinterpret_cast<unsigned*>(&h) = u;
        return __half22float2(h);
    }
    static __device__ __forceinline__ V up(V v) { return __shfl_up_sync(kFull, v, 1); }
    static __device__ __forceinline__ V down(V v) { return __shfl_down_sync(kFull, v, 1); }
    static __device__ __forceinline__ float2 left(V prev, V cur) { return cvt(__byte_perm(prev, cur, 0x5432)); }
    static __device__ __forceinline__ float2 right(V cur, V next) { return cvt(__byte_perm(cur, next, 0x5432)); }
    static __device__ __forceinline__ float rnd(float v) { return __half2float(__float2half_rn(v)); }
};

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// One thread of the block asks L2 for the 19 source row segments the same
// block position needs `prefetch_rows` rows later, so that by the time that
// block runs its loads hit L2 instead of HBM.  Segments are widened to
// 16-byte boundaries (the bulk-prefetch alignment rule).
template <typename S>
__device__ __forceinline__ void prefetch_ahead(const S* fin, const Layout& L, const StepArgs& a, int j, int k,
                                               int col0, int ncols)
{
    const long long r = (long long)(k - 1) * L.ny + (j - 1) + a.prefetch_rows;
    if (r >= (long long)L.ny * L.nz) return;
    const int jj = 1 + (int)(r % L.ny), kk = 1 + (int)(r / L.ny);
    constexpr int PADE = 16 / (int)sizeof(S);
    const long long cell0 = (long long)kk * L.plane + (long long)jj * L.pitch + col0;
    const uint32_t bytes = (uint32_t)((ncols + 2 * PADE) * (int)sizeof(S) + 15) & ~15u;
#pragma unroll
    for (int q = 0; q < Q; ++q) prefetch_l2(fin + cell0 + a.pull_off[q] - PADE, bytes);
}

// Fused pull-stream + halfway bounce-back + BGK + sponge (06:906-972), two
// x-adjacent cells per thread.  Each direction is read as one aligned vector
// per thread; the +-1 x shift of directions with ex != 0 takes the missing
// neighbour element from the adjacent lane (warp shuffle) and, at the warp
// edge, from one extra aligned load.  The collision runs on the pair with
// packed FP32x2 instructions.  Cells next to the x faces take their x-halo
// sources from the x-face ghosts and export their results for the next ghost
// fill.
template <typename S, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_step(const S* __restrict__ fin, S* __restrict__ fout, Layout L,
                                                      StepArgs a, float inv_scale)
{
    using P = PairIo<S>;
    const int lane = threadIdx.x & 31;
    const int c0r = 2 * (blockIdx.x * blockDim.x + threadIdx.x);   // first column of the pair
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~1);              // inactive lanes shadow a valid pair
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    const long long cell = (long long)k * L.plane + (long long)j * L.pitch + c0;
    const S* tin = fin + cell;
    if (a.prefetch_rows > 0 && threadIdx.x == 0)
    {
        const int col0 = 2 * blockIdx.x * BLOCK;
        prefetch_ahead<S>(fin, L, a, j, k, col0, min(2 * BLOCK, L.nx - col0));
    }

    uint32_t lk0 = 0, lk1 = 0;
    if (active)
    {
        const uint32_t nw = near_word(a, L, c0, j, k);
        const uint32_t b = (nw >> (c0 & 31)) & 3u;
        if (b & 1u) lk0 = a.links[cell];
        if (b & 2u) lk1 = a.links[cell + 1];
    }
    const bool any_link = __any_sync(kFull, (lk0 | lk1) != 0u);

    float2 G[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const S* src = tin + a.pull_off[q];
        const typename P::V cur = P::ld(src);
        if (ex(q) == 0)
        {
            G[q] = P::cvt(cur);
        }
        else if (ex(q) > 0)
        {
            typename P::V prev = P::up(cur);
            if (lane == 0) prev = P::ld(src - 2);
            G[q] = P::left(prev, cur);
        }
        else
        {
            typename P::V next = P::down(cur);
            if (lane == 31) next = P::ld(src + 2);
            G[q] = P::right(cur, next);
        }
    }
    if (any_link)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (((lk0 | lk1) >> q) & 1u)
            {
                const float2 own = P::cvt(P::ld(tin + a.pop_off[inv(q)]));
                if ((lk0 >> q) & 1u) G[q].x = own.x;
                if ((lk1 >> q) & 1u) G[q].y = own.y;
            }
        }
    }
    // x faces: sources in the x halo come from the x-face ghosts.
    const bool xlo = active && c0 == 0;
    const bool xhi0 = active && c0 == L.nx - 1;       // nx odd: first cell of the pair is the last
    const bool xhi1 = active && c0 + 1 == L.nx - 1;   // nx even: second cell is the last
    if (xlo | xhi0 | xhi1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (ex(q) == 0) continue;
            const float g = a.xf.xgh[a.xf.gh_index(ex(q) > 0 ? 0 : 1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
            if (ex(q) > 0 && xlo && !((lk0 >> q) & 1u)) G[q].x = g;
            if (ex(q) < 0 && xhi0 && !((lk0 >> q) & 1u)) G[q].x = g;
            if (ex(q) < 0 && xhi1 && !((lk1 >> q) & 1u)) G[q].y = g;
        }
    }
    if (!active) return;

    const float syz = fmaxf(a.sig_y[j - 1], a.sig_z[k - 1]);
    const float2 sg = make_float2(fmaxf(a.sig_x[c0], syz), fmaxf(c0 + 1 < L.nx ? a.sig_x[c0 + 1] : 0.f, syz));
    collide2(G, inv_scale, a.omega, sg, (lk0 & kSolidSelfBit) != 0u, (lk1 & kSolidSelfBit) != 0u);

    S* tout = fout + cell;
#pragma unroll
    for (int q = 0; q < Q; ++q) P::st(tout + a.pop_off[q], G[q]);

    if (xlo | xhi0 | xhi1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (xlo) a.xf.xexp[a.xf.exp_index(0, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
            if (xhi0) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
            if (xhi1) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].y);
        }
    }
}

// Pair kernel with 32-bit per-thread element offsets: every address is a
// warp-uniform per-direction base pointer (fin + q * pop_stride, from kernel
// parameters) plus a 32-bit cell offset, so per-thread address arithmetic
// stays 32-bit.  The host guarantees pop_stride < 2^31.
template <typename S, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_step32(const S* __restrict__ fin, S* __restrict__ fout, Layout L,
                                                        StepArgs a, float inv_scale)
{
    using P = PairIo<S>;
    const int lane = threadIdx.x & 31;
    const int c0r = 2 * (blockIdx.x * BLOCK + threadIdx.x);
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~1);
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    const uint32_t pitch = (uint32_t)L.pitch, plane = (uint32_t)L.plane;
    const uint32_t cell = (uint32_t)k * plane + (uint32_t)j * pitch + (uint32_t)c0;
    const size_t ps = (size_t)L.pop_stride;
    if (a.prefetch_rows > 0 && threadIdx.x == 0)
    {
        const int col0 = 2 * blockIdx.x * BLOCK;
        prefetch_ahead<S>(fin, L, a, j, k, col0, min(2 * BLOCK, L.nx - col0));
    }
    uint32_t lk0 = 0, lk1 = 0;
    if (active)
    {
        const uint32_t b = (near_word(a, L, c0, j, k) >> (c0 & 31)) & 3u;
        if (b & 1u) lk0 = a.links[cell];
        if (b & 2u) lk1 = a.links[cell + 1];
    }
    const bool any_link = __any_sync(kFull, (lk0 | lk1) != 0u);

    float2 G[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const S* __restrict__ Pq = fin + q * ps;
        const uint32_t src = cell - (uint32_t)(ey(q) * (int)pitch + ez(q) * (int)plane);
        const typename P::V cur = P::ld(Pq + src);
        if (ex(q) == 0)
        {
            G[q] = P::cvt(cur);
        }
        else if (ex(q) > 0)
        {
            typename P::V prev = P::up(cur);
            if (lane == 0) prev = P::ld(Pq + (src - 2u));
            G[q] = P::left(prev, cur);
        }
        else
        {
            typename P::V next = P::down(cur);
            if (lane == 31) next = P::ld(Pq + (src + 2u));
            G[q] = P::right(cur, next);
        }
    }
    if (any_link)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (((lk0 | lk1) >> q) & 1u)
            {
                const float2 own = P::cvt(P::ld(fin + inv(q) * ps + cell));
                if ((lk0 >> q) & 1u) G[q].x = own.x;
                if ((lk1 >> q) & 1u) G[q].y = own.y;
            }
        }
    }
    const bool xlo = active && c0 == 0;
    const bool xhi0 = active && c0 == L.nx - 1;
    const bool xhi1 = active && c0 + 1 == L.nx - 1;
    if (xlo | xhi0 | xhi1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (ex(q) == 0) continue;
            const float g = a.xf.xgh[a.xf.gh_index(ex(q) > 0 ? 0 : 1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
            if (ex(q) > 0 && xlo && !((lk0 >> q) & 1u)) G[q].x = g;
            if (ex(q) < 0 && xhi0 && !((lk0 >> q) & 1u)) G[q].x = g;
            if (ex(q) < 0 && xhi1 && !((lk1 >> q) & 1u)) G[q].y = g;
        }
    }
    if (!active) return;

    const float syz = fmaxf(a.sig_y[j - 1], a.sig_z[k - 1]);
    const float2 sg = make_float2(fmaxf(a.sig_x[c0], syz), fmaxf(c0 + 1 < L.nx ? a.sig_x[c0 + 1] : 0.f, syz));
    collide2(G, inv_scale, a.omega, sg, (lk0 & kSolidSelfBit) != 0u, (lk1 & kSolidSelfBit) != 0u);
#pragma unroll
    for (int q = 0; q < Q; ++q) P::st(fout + q * ps + cell, G[q]);
    if (xlo | xhi0 | xhi1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (xlo) a.xf.xexp[a.xf.exp_index(0, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
            if (xhi0) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
            if (xhi1) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].y);
        }
    }
}

// Four x-adjacent cells per thread, FP16 storage: every direction is one
// aligned 8-byte vector (two half2 words) per thread, so each thread keeps
// twice the bytes in flight of the pair kernel for about the same register
// budget.  The two pairs are collided one after the other (packed FP32x2).
__device__ __forceinline__ uint2 ld_quad(const __half* p) { return __ldg(reinterpret_cast<const uint2*>(p)); }

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_step_quad(const __half* __restrict__ fin, __half* __restrict__ fout,
                                                           Layout L, StepArgs a, float inv_scale)
{
    using P = PairIo<__half>;
    const int lane = threadIdx.x & 31;
    const int c0r = 4 * (blockIdx.x * BLOCK + threadIdx.x);
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~3);
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    const long long cell = (long long)k * L.plane + (long long)j * L.pitch + c0;
    const __half* tin = fin + cell;
    if (a.prefetch_rows > 0 && threadIdx.x == 0)
    {
        const int col0 = 4 * blockIdx.x * BLOCK;
        prefetch_ahead<__half>(fin, L, a, j, k, col0, min(4 * BLOCK, L.nx - col0));
    }
    uint32_t lk[4] = {0, 0, 0, 0};
    if (active)
    {
        const uint32_t b = (near_word(a, L, c0, j, k) >> (c0 & 31)) & 15u;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if ((b >> c) & 1u) lk[c] = a.links[cell + c];
    }
    const bool any_link = __any_sync(kFull, (lk[0] | lk[1] | lk[2] | lk[3]) != 0u);

    // words: w[q].x = cells (c0, c0+1), w[q].y = cells (c0+2, c0+3), shifted per direction
    uint2 w[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const __half* src = tin + a.pull_off[q];
        const uint2 cur = ld_quad(src);
        if (ex(q) == 0)
        {
            w[q] = cur;
        }
        else if (ex(q) > 0)
        {
            unsigned prev = __shfl_up_sync(kFull, cur.y, 1);   // cells (c0-2, c0-1)
            if (lane == 0) prev = ld_quad(src - 4).y;
            w[q] = make_uint2(__byte_perm(prev, cur.x, 0x5432), __byte_perm(cur.x, cur.y, 0x5432));
        }
        else
        {
            unsigned next = __shfl_down_sync(kFull, cur.x, 1);   // cells (c0+4, c0+5)
            if (lane == 31) next = ld_quad(src + 4).x;
            w[q] = make_uint2(__byte_perm(cur.x, cur.y, 0x5432), __byte_perm(cur.y, next, 0x5432));
        }
    }
    if (any_link)
    {
        const uint32_t la = lk[0] | lk[1] | lk[2] | lk[3];
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if ((la >> q) & 1u)
            {
                const uint2 own = ld_quad(tin + a.pop_off[inv(q)]);
                // halfword select: cell c takes `own` when its link bit q is set
                const unsigned m0 = (((lk[0] >> q) & 1u) ? 0x0000ffffu : 0u) | (((lk[1] >> q) & 1u) ? 0xffff0000u : 0u);
                const unsigned m1 = (((lk[2] >> q) & 1u) ? 0x0000ffffu : 0u) | (((lk[3] >> q) & 1u) ? 0xffff0000u : 0u);
                w[q].x = (w[q].x & ~m0) | (own.x & m0);
                w[q].y = (w[q].y & ~m1) | (own.y & m1);
            }
        }
    }
    // x faces (ghost values are float; patched after conversion below)
    const int last = L.nx - 1 - c0;   // position of cell nx-1 in this quad when 0..3
    const bool xlo = active && c0 == 0;
    const bool xhi = active && last >= 0 && last < 4;
    if (!active) return;

    const float syz = fmaxf(a.sig_y[j - 1], a.sig_z[k - 1]);
    __half* tout = fout + cell;
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        float2 G[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) G[q] = P::cvt(h == 0 ? w[q].x : w[q].y);
        const int ca = c0 + 2 * h;
        if (xlo | xhi)
        {
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (ex(q) == 0) continue;
                const float g = a.xf.xgh[a.xf.gh_index(ex(q) > 0 ? 0 : 1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
                if (ex(q) > 0 && xlo && h == 0 && !((lk[0] >> q) & 1u)) G[q].x = g;
                if (ex(q) < 0 && xhi && last == 2 * h && !((lk[2 * h] >> q) & 1u)) G[q].x = g;
                if (ex(q) < 0 && xhi && last == 2 * h + 1 && !((lk[2 * h + 1] >> q) & 1u)) G[q].y = g;
            }
        }
        const float2 sg = make_float2(fmaxf(ca < L.nx ? a.sig_x[ca] : 0.f, syz),
                                      fmaxf(ca + 1 < L.nx ? a.sig_x[ca + 1] : 0.f, syz));
        collide2(G, inv_scale, a.omega, sg, (lk[2 * h] & kSolidSelfBit) != 0u, (lk[2 * h + 1] & kSolidSelfBit) != 0u);
#pragma unroll
        for (int q = 0; q < Q; ++q) P::st(tout + a.pop_off[q] + 2 * h, G[q]);
        if (xlo | xhi)
        {
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (xlo && h == 0) a.xf.xexp[a.xf.exp_index(0, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
                if (xhi && last == 2 * h) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
                if (xhi && last == 2 * h + 1) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].y);
            }
        }
    }
}

// ---------------------------------------------------------------- staged step
// Bulk asynchronous copies (cp.async.bulk, completion counted on an mbarrier)
// stage, for every direction q, the source row segment of a tile in shared
// memory; a persistent CTA keeps NS tiles in flight while it collides the
// oldest one.  Memory-level parallelism no longer depends on registers.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Waits for phase `parity` of the barrier, giving up after `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit)
{
    for (int n = 0; n < limit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbarrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Reads of a staged row (p points at the element of the pair's first cell).
template <typename S>
struct Staged;

template <>
struct Staged<float>
{
    static __device__ __forceinline__ float2 pair(const float* p) { return *reinterpret_cast<const float2*>(p); }
    static __device__ __forceinline__ float2 left(const float* p) { return make_float2(p[-1], p[0]); }
    static __device__ __forceinline__ float2 right(const float* p) { return make_float2(p[1], p[2]); }
};

template <>
struct Staged<__half>
{
    static __device__ __forceinline__ unsigned word(const __half* p) { return *reinterpret_cast<const unsigned*>(p); }
    static __device__ __forceinline__ float2 pair(const __half* p) { return PairIo<__half>::cvt(word(p)); }
    static __device__ __forceinline__ float2 left(const __half* p)
    {
        return PairIo<__half>::cvt(__byte_perm(word(p - 2), word(p), 0x5432));
    }
    static __device__ __forceinline__ float2 right(const __half* p)
    {
        return PairIo<__half>::cvt(__byte_perm(word(p), word(p + 2), 0x5432));
    }
};

constexpr int kStageWaitLimit = 1 << 22;   // mbarrier polls before a stage wait gives up

template <typename S, int TW, int NS>
__global__ void __launch_bounds__(TW / 2) k_step_staged(const S* __restrict__ fin, S* __restrict__ fout, Layout L,
                                                       StepArgs a, float inv_scale, int tiles_per_row,
                                                       long long ntiles)
{
    using P = PairIo<S>;
    using T = Staged<S>;
    constexpr int PADE = 16 / (int)sizeof(S);   // 16-byte alignment margin on both sides of a row
    constexpr int ROW = TW + 2 * PADE;          // staged elements per direction
    constexpr uint32_t ROW_BYTES = ROW * sizeof(S);
    constexpr uint32_t STAGE_BYTES = Q * ROW_BYTES;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    S* const stages = reinterpret_cast<S*>(smem_raw);
    __shared__ __align__(8) uint64_t full[NS];

    const int tid = threadIdx.x;
    if (tid == 0)
    {
        for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
        fence_mbarrier_init();
    }
    __syncthreads();

    // One elected thread stages all 19 source rows of a tile.
    auto issue = [&](int s, long long tile) {
        const long long r = tile / tiles_per_row;
        const int seg = (int)(tile - r * tiles_per_row);
        const int j = 1 + (int)(r % L.ny), k = 1 + (int)(r / L.ny);
        const long long cell0 = (long long)k * L.plane + (long long)j * L.pitch + (long long)seg * TW;
        S* dst = stages + (size_t)s * Q * ROW;
        mbar_expect_tx(&full[s], STAGE_BYTES);
#pragma unroll
        for (int q = 0; q < Q; ++q) bulk_copy_g2s(dst + q * ROW, fin + cell0 + a.pull_off[q] - PADE, ROW_BYTES, &full[s]);
    };
    if (tid == 0)
        for (int s = 0; s < NS; ++s)
        {
            const long long t = blockIdx.x + (long long)s * gridDim.x;
            if (t < ntiles) issue(s, t);
        }

    int it = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it)
    {
        const int s = it % NS;
        const uint32_t parity = (uint32_t)(it / NS) & 1u;
        const bool ok = mbar_wait_bounded(&full[s], parity, kStageWaitLimit);

        const long long r = tile / tiles_per_row;
        const int seg = (int)(tile - r * tiles_per_row);
        const int j = 1 + (int)(r % L.ny), k = 1 + (int)(r / L.ny);
        const int c0 = seg * TW + 2 * tid;
        const bool active = ok && c0 < L.nx;
        if (active)
        {
            const long long cell = (long long)k * L.plane + (long long)j * L.pitch + c0;
            uint32_t lk0 = 0, lk1 = 0;
            const uint32_t b = (near_word(a, L, c0, j, k) >> (c0 & 31)) & 3u;
            if (b & 1u) lk0 = a.links[cell];
            if (b & 2u) lk1 = a.links[cell + 1];
            const S* sp = stages + (size_t)s * Q * ROW + PADE + 2 * tid;
            float2 G[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (ex(q) == 0) G[q] = T::pair(sp + q * ROW);
                else if (ex(q) > 0) G[q] = T::left(sp + q * ROW);
                else G[q] = T::right(sp + q * ROW);
            }
            const S* tin = fin + cell;
            if (lk0 | lk1)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q)
                {
                    if (((lk0 | lk1) >> q) & 1u)
                    {
                        const float2 own = P::cvt(P::ld(tin + a.pop_off[inv(q)]));
                        if ((lk0 >> q) & 1u) G[q].x = own.x;
                        if ((lk1 >> q) & 1u) G[q].y = own.y;
                    }
                }
            }
            const bool xlo = c0 == 0;
            const bool xhi0 = c0 == L.nx - 1;
            const bool xhi1 = c0 + 1 == L.nx - 1;
            if (xlo | xhi0 | xhi1)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q)
                {
                    if (ex(q) == 0) continue;
                    const float g = a.xf.xgh[a.xf.gh_index(ex(q) > 0 ? 0 : 1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
                    if (ex(q) > 0 && xlo && !((lk0 >> q) & 1u)) G[q].x = g;
                    if (ex(q) < 0 && xhi0 && !((lk0 >> q) & 1u)) G[q].x = g;
                    if (ex(q) < 0 && xhi1 && !((lk1 >> q) & 1u)) G[q].y = g;
                }
            }
            const float syz = fmaxf(a.sig_y[j - 1], a.sig_z[k - 1]);
            const float2 sg =
                make_float2(fmaxf(a.sig_x[c0], syz), fmaxf(c0 + 1 < L.nx ? a.sig_x[c0 + 1] : 0.f, syz));
            collide2(G, inv_scale, a.omega, sg, (lk0 & kSolidSelfBit) != 0u, (lk1 & kSolidSelfBit) != 0u);
            S* tout = fout + cell;
#pragma unroll
            for (int q = 0; q < Q; ++q) P::st(tout + a.pop_off[q], G[q]);
            if (xlo | xhi0 | xhi1)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q)
                {
                    if (xlo) a.xf.xexp[a.xf.exp_index(0, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
                    if (xhi0) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].x);
                    if (xhi1) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = P::rnd(G[q].y);
                }
            }
        }
        // every thread is done with stage s (and agrees on whether the wait failed)
        const int failed = __syncthreads_or(!ok);
        if (failed)
        {
            if (tid == 0)
            {
                atomicExch(a.error, kErrStageTimeout);
                // let the copies already in flight land before the CTA exits
                for (int d = 0; d < NS; ++d)
                {
                    const long long t = tile + (long long)d * gridDim.x;
                    if (t < ntiles) mbar_wait_bounded(&full[(it + d) % NS], (uint32_t)((it + d) / NS) & 1u, kStageWaitLimit);
                }
            }
            return;
        }
        if (tid == 0)
        {
            const long long next = tile + (long long)NS * gridDim.x;
            if (next < ntiles)
            {
                fence_proxy_async_smem();   // generic-proxy reads of stage s before the async-proxy refill
                issue(s, next);
            }
        }
    }
}

// ---------------------------------------------------------------- links
// Per interior cell: bit q set when the pull source cell - e_q is SOLID,
// bit 19 when the cell itself is SOLID (mask semantics 06:923, 06:933).
// The near-solid bitmap gets one bit per cell (a warp ballot), so the step
// kernel reads the links word only in warps that touch a solid.
__global__ void __launch_bounds__(128) k_build_links(const uint8_t* __restrict__ m, uint32_t* __restrict__ links,
                                                     uint32_t* __restrict__ near, Layout L)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    const bool active = i0 < L.nx;
    const long long nxt = L.nx + 2, nyt = L.ny + 2;
    uint32_t lk = 0;
    if (active)
    {
        const int i = i0 + 1;
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const long long src = (long long)(i - ex(q)) + (long long)(j - ey(q)) * nxt + (long long)(k - ez(q)) * nxt * nyt;
            if (m[src]) lk |= 1u << q;
        }
        if (m[(long long)i + (long long)j * nxt + (long long)k * nxt * nyt]) lk |= kSolidSelfBit;
        links[(long long)k * L.plane + (long long)j * L.pitch + i0] = lk;
    }
    const uint32_t ball = __ballot_sync(kFull, active && lk != 0u);
    if ((threadIdx.x & 31) == 0 && i0 < L.pitch)
        near[((long long)k * (L.ny + 2) + j) * L.words_per_row + (i0 >> 5)] = ball;
}

// ---------------------------------------------------------------- source
__device__ double block_sum(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) t += red[w];
    return t;
}

// Source injection (LBMSolver::apply_source 06:576-667): weights of the
// (2R+1)^3 Gaussian stencil (or the 8 trilinear weights) are normalised over
// the FLUID cells of the grid, A = mass / sum_w, and every FLUID cell gains
// w_q * A * w_cell in each direction.  One block; sources run in order.
// Cells next to the x faces also update their x-face export.
template <typename S>
__global__ void __launch_bounds__(512) k_source(S* __restrict__ f, Layout L, StepArgs sa, SourceArgs a)
{
    __shared__ double red[32];
    const int tid = threadIdx.x;
    for (int s = 0; s < a.nsrc; ++s)
    {
        SourceEntry e;
        if (a.ctl)
        {
            const long long row = a.ctl->step - a.ctl->table_base;
            e = a.table[row * a.nsrc + s];
        }
        else
        {
            e = a.direct[s];
        }
        if (e.mass == 0.0) continue;
        const SourceStatic st = a.st[s];
        int gi = 0, gj = 0, gk = 0;
        bool in = false;
        double ww = 0.0;
        if (st.injection == 1)
        {
            const double fx = (e.cx - a.x_min) / a.dx - 0.5;
            const double fy = (e.cy - a.y_min) / a.dx - 0.5;
            const double fz = (e.cz - a.z_min) / a.dx - 0.5;
            const int i0 = (int)floor(fx), j0 = (int)floor(fy), k0 = (int)floor(fz);
            const double tx = fx - i0, ty = fy - j0, tz = fz - k0;
            if (tid < 8)
            {
                gi = i0 + (tid & 1);
                gj = j0 + ((tid >> 1) & 1);
                gk = k0 + (tid >> 2);
                ww = ((tid & 1) ? tx : 1.0 - tx) * (((tid >> 1) & 1) ? ty : 1.0 - ty) * ((tid >> 2) ? tz : 1.0 - tz);
                in = true;
            }
        }
        else
        {
            const int R = st.radius, n = 2 * R + 1;
            const int ic = (int)floor((e.cx - a.x_min) / a.dx);
            const int jc = (int)floor((e.cy - a.y_min) / a.dx);
            const int kc = (int)floor((e.cz - a.z_min) / a.dx);
            if (ic < -R || ic >= L.nx + R || jc < -R || jc >= L.ny + R || kc < -R || kc >= L.nz + R) continue;
            if (tid < n * n * n)
            {
                gi = ic + tid % n - R;
                gj = jc + (tid / n) % n - R;
                gk = kc + tid / (n * n) - R;
                const double x = a.x_min + (gi + 0.5) * a.dx;
                const double y = a.y_min + (gj + 0.5) * a.dx;
                const double z = a.z_min + (gk + 0.5) * a.dx;
                const double ddx = x - e.cx, ddy = y - e.cy, ddz = z - e.cz;
                const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                ww = exp(-0.5 * r2 / st.sigma2);
                in = true;
            }
        }
        long long cell = 0;
        bool fluid = false;
        if (in && gi >= 0 && gi < L.nx && gj >= 0 && gj < L.ny && gk >= 0 && gk < L.nz)
        {
            cell = (long long)(gk + 1) * L.plane + (long long)(gj + 1) * L.pitch + gi;
            fluid = (sa.links[cell] & kSolidSelfBit) == 0u;
        }
        const double sum = block_sum(fluid ? ww : 0.0, red);
        if (sum < 1e-30) continue;
        const double A = e.mass / sum;
        if (fluid)
        {
            const double add = A * ww * (double)a.scale;
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                S* p = f + (long long)q * L.pop_stride + cell;
                Io<S>::st(p, Io<S>::ldw(p) + (float)(wd(q) * add));
                if (gi == 0 || gi == L.nx - 1)
                {
                    const float gs = Io<S>::ldw(p);   // the stored value, as the step would export it
                    if (gi == 0) sa.xf.xexp[sa.xf.exp_index(0, q, gj + 1, gk + 1, L.ny, L.nz)] = gs;
                    if (gi == L.nx - 1) sa.xf.xexp[sa.xf.exp_index(1, q, gj + 1, gk + 1, L.ny, L.nz)] = gs;
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- ghosts
// Characteristic open boundary (exchange_halos 06:684-835, MPI size 1): the
// ghost cell next to interior cell I gets
//   f_B = feq(rho_B, u_B) + (f_I - feq(rho_I, u_I)),
// where u_B keeps the tangential velocity of I, and the normal velocity and
// pressure carry only the outgoing invariant (incoming invariant zero).  In
// stored deviation units (Gs = scale * g):
//   geq(rho', r, u) = w (rho' + r (3 c.u + (4.5 (c.u)^2 - 1.5 u^2) / scale)).
__device__ __forceinline__ float geq_dev(int q, float rho, float r, float ux, float uy, float uz, float inv_scale)
{
    const float cu = dot_c(q, ux, uy, uz);
    const float u2 = ux * ux + uy * uy + uz * uz;
    return wf(q) * fmaf(r, fmaf(inv_scale, 4.5f * cu * cu - 1.5f * u2, 3.0f * cu), rho);
}

__device__ __forceinline__ void nscbc(float (&G)[Q], int axis, int side, float inv_scale)
{
    float rho, jx, jy, jz;
    moments(G, rho, jx, jy, jz);
    float rI = fmaf(rho, inv_scale, 1.0f);
    float ux, uy, uz;
    if (rI > 1e-30f)
    {
        ux = jx / rI;
        uy = jy / rI;
        uz = jz / rI;
    }
    else
    {
        rI = 1.0f;
        rho = 0.0f;
        ux = uy = uz = 0.0f;
    }
    const float cs = (float)kCs, cs2 = (float)kCs2;
    const float pI = cs2 * rho;
    const float un = axis == 0 ? ux : (axis == 1 ? uy : uz);
    float unB, pB;
    if (side == 0)
    {
        const float Wm = un - pI / cs;   // Wp = 0 (06:694-698)
        unB = 0.5f * Wm;
        pB = -0.5f * cs * Wm;
    }
    else
    {
        const float Wp = un + pI / cs;   // Wm = 0 (06:721-725)
        unB = 0.5f * Wp;
        pB = 0.5f * cs * Wp;
    }
    const float rhoB = pB / cs2;
    const float rB = fmaf(rhoB, inv_scale, 1.0f);
    const float bx = axis == 0 ? unB : ux, by = axis == 1 ? unB : uy, bz = axis == 2 ? unB : uz;
#pragma unroll
    for (int q = 0; q < Q; ++q)
        G[q] += geq_dev(q, rhoB, rB, bx, by, bz, inv_scale) - geq_dev(q, rho, rI, ux, uy, uz, inv_scale);
}

template <typename S>
__global__ void __launch_bounds__(128) k_ghost(S* __restrict__ f, Layout L, GhostArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.total) return;
    int fi = 0;
    while (fi + 1 < a.nfaces && t >= a.face[fi + 1].first) ++fi;
    const GhostFace F = a.face[fi];
    const long long lt = t - F.first;
    const int u = (int)(lt % F.nu), v = (int)(lt / F.nu);
    const float inv_scale = 1.0f / a.scale;
    float G[Q];
    if (F.axis == 0)
    {
        // x faces: compact export -> compact ghost, both coalesced along j
        const int j = 1 + u, k = 1 + v;
#pragma unroll
        for (int q = 0; q < Q; ++q) G[q] = a.xf.xexp[a.xf.exp_index(F.side, q, j, k, L.ny, L.nz)];
        nscbc(G, 0, F.side, inv_scale);
#pragma unroll
        for (int q = 0; q < Q; ++q) a.xf.xgh[a.xf.gh_index(F.side, q, j, k, L.ny, L.nz)] = G[q];
        return;
    }
    int ci, cj, ck, gj, gk;
    if (F.axis == 1)
    {
        ci = 1 + u;
        ck = gk = 1 + v;
        cj = F.side ? L.ny : 1;
        gj = F.side ? L.ny + 1 : 0;
    }
    else
    {
        ci = 1 + u;
        cj = gj = 1 + v;
        ck = F.side ? L.nz : 1;
        gk = F.side ? L.nz + 1 : 0;
    }
    const long long cI = (long long)ck * L.plane + (long long)cj * L.pitch + (ci - 1);
    const long long cB = (long long)gk * L.plane + (long long)gj * L.pitch + (ci - 1);
#pragma unroll
    for (int q = 0; q < Q; ++q) G[q] = Io<S>::ld(f + (long long)q * L.pop_stride + cI);
    nscbc(G, F.axis, F.side, inv_scale);
#pragma unroll
    for (int q = 0; q < Q; ++q) Io<S>::st(f + (long long)q * L.pop_stride + cB, G[q]);
}

// ---------------------------------------------------------------- probes
// rho - 1 at each probe cell for the step whose pre-step buffer is `f`
// (the value LBMSolver::run records, 06:1085-1092; SOLID cells read 0).
template <typename S>
__global__ void __launch_bounds__(256) k_probe(const S* __restrict__ f, Layout L, StepArgs sa, ProbeArgs a)
{
    const long long row = a.ctl ? a.ctl->step - a.ctl->probe_base : a.direct_row;
    const float inv_scale = 1.0f / a.scale;
    for (int p = threadIdx.x; p < a.n; p += blockDim.x)
    {
        const long long c = a.cell[p];
        double val;
        if (c < 0)
        {
            val = __longlong_as_double(0x7ff8000000000000LL);
        }
        else
        {
            const int k = (int)(c / L.plane);
            const long long rem = c - (long long)k * L.plane;
            const int j = (int)(rem / L.pitch);
            const int i = (int)(rem - (long long)j * L.pitch) + 1;
            bool solid;
            float G[Q];
            pull_cell<S>(f, L, sa, i, j, k, G, solid);
            float rho = 0.f;
#pragma unroll
            for (int q = 0; q < Q; ++q) rho += G[q];
            const float rp = rho * inv_scale;
            if (solid) val = 0.0;
            else if (1.0f + rp <= 0.f) val = 1e-12 - 1.0;
            else val = (double)rp;
            a.energy[p] += val * val;
        }
        a.out[row * a.n + p] = val;
    }
    __syncthreads();
    if (threadIdx.x == 0 && a.ctl) a.ctl->step += 1;
}

template <typename S>
__global__ void __launch_bounds__(128) k_field_rho(const S* __restrict__ f, float* __restrict__ out, Layout L,
                                                   StepArgs sa, float inv_scale)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 >= L.nx) return;
    const int j = blockIdx.y + 1, k = blockIdx.z + 1;
    bool solid;
    float G[Q];
    pull_cell<S>(f, L, sa, i0 + 1, j, k, G, solid);
    float rho = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) rho += G[q];
    out[((long long)(k - 1) * L.ny + (j - 1)) * L.nx + i0] = solid ? 0.f : rho * inv_scale;
}

// ---------------------------------------------------------------- import/export
// Conversions between the device state and FP64 f in the reference's AoS
// halo-inclusive layout; the x-halo columns map to the x-face ghosts and the
// cells next to the x faces are mirrored into the x-face exports.
template <typename S>
__global__ void k_export_f(const S* __restrict__ f, double* __restrict__ out, Layout L, XFace xf, float inv_scale)
{
    const long long nxt = L.nx + 2, nyt = L.ny + 2, n = nxt * nyt * (L.nz + 2);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(idx % nxt);
        const int j = (int)((idx / nxt) % nyt);
        const int k = (int)(idx / (nxt * nyt));
        const long long c = (long long)k * L.plane + (long long)j * L.pitch + (i - 1);
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            float g;
            if (i == 0) g = xf.xgh[xf.gh_index(0, q, j, k, L.ny, L.nz)];
            else if (i == L.nx + 1) g = xf.xgh[xf.gh_index(1, q, j, k, L.ny, L.nz)];
            else g = Io<S>::ld(f + (long long)q * L.pop_stride + c);
            out[idx * Q + q] = wd(q) + (double)g * (double)inv_scale;
        }
    }
}

template <typename S>
__global__ void k_import_f(S* __restrict__ f, const double* __restrict__ in, Layout L, XFace xf, float scale)
{
    const long long nxt = L.nx + 2, nyt = L.ny + 2, n = nxt * nyt * (L.nz + 2);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x)
    {
        const int i = (int)(idx % nxt);
        const int j = (int)((idx / nxt) % nyt);
        const int k = (int)(idx / (nxt * nyt));
        const long long c = (long long)k * L.plane + (long long)j * L.pitch + (i - 1);
        const bool inner = j >= 1 && j <= L.ny && k >= 1 && k <= L.nz;
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const float g = (float)((in[idx * Q + q] - wd(q)) * (double)scale);
            if (i == 0)
            {
                xf.xgh[xf.gh_index(0, q, j, k, L.ny, L.nz)] = g;
                continue;
            }
            if (i == L.nx + 1)
            {
                xf.xgh[xf.gh_index(1, q, j, k, L.ny, L.nz)] = g;
                continue;
            }
            S* p = f + (long long)q * L.pop_stride + c;
            Io<S>::st(p, g);
            const float gs = Io<S>::ldw(p);   // the stored (rounded) value
            if (inner && i == 1) xf.xexp[xf.exp_index(0, q, j, k, L.ny, L.nz)] = gs;
            if (inner && i == L.nx) xf.xexp[xf.exp_index(1, q, j, k, L.ny, L.nz)] = gs;
        }
    }
}

dim3 row_grid(const Layout& L) { return dim3((unsigned)((L.nx + 127) / 128), (unsigned)L.ny, (unsigned)L.nz); }
dim3 pair_grid(const Layout& L, int block)
{
    return dim3((unsigned)(((L.nx + 1) / 2 + block - 1) / block), (unsigned)L.ny, (unsigned)L.nz);
}

template <typename S, int TW, int NS>
constexpr size_t staged_smem()
{
    return (size_t)NS * Q * (TW + 2 * (16 / sizeof(S))) * sizeof(S);
}

template <typename S, int TW, int NS>
cudaError_t launch_staged(const S* fin, S* fout, const Layout& L, const StepArgs& a, float inv_scale, int grid,
                          cudaStream_t stream)
{
    const int tpr = (L.nx + TW - 1) / TW;
    const long long ntiles = (long long)tpr * L.ny * L.nz;
    const int g = (int)std::min<long long>(grid, ntiles);
    k_step_staged<S, TW, NS><<<g, TW / 2, staged_smem<S, TW, NS>(), stream>>>(fin, fout, L, a, inv_scale, tpr, ntiles);
    return cudaGetLastError();
}

template <typename S, int TW, int NS>
cudaError_t prepare_staged(int device, int* grid)
{
    const size_t smem = staged_smem<S, TW, NS>();
    cudaError_t e = cudaFuncSetAttribute(k_step_staged<S, TW, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_staged<S, TW, NS>, TW / 2, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    *grid = std::max(1, per_sm) * sms;
    return cudaSuccess;
}

template <typename S>
cudaError_t launch_step_t(const S* fin, S* fout, const Layout& L, const StepArgs& a, float inv_scale, int variant,
                          int grid, cudaStream_t stream)
{
    switch (variant)
    {
    case 4: return launch_staged<S, 256, 3>(fin, fout, L, a, inv_scale, grid, stream);
    case 5: return launch_staged<S, 256, 2>(fin, fout, L, a, inv_scale, grid, stream);
    case 6: return launch_staged<S, 128, 4>(fin, fout, L, a, inv_scale, grid, stream);
    case 7: return launch_staged<S, 512, 2>(fin, fout, L, a, inv_scale, grid, stream);
    case 8:
        if constexpr (std::is_same<S, __half>::value)
        {
            const dim3 g((unsigned)(((L.nx + 3) / 4 + 127) / 128), (unsigned)L.ny, (unsigned)L.nz);
            k_step_quad<128, 0><<<g, 128, 0, stream>>>(fin, fout, L, a, inv_scale);
            return cudaGetLastError();
        }
        variant = 3;
        break;
    case 10: k_step32<S, 128, 0><<<pair_grid(L, 128), 128, 0, stream>>>(fin, fout, L, a, inv_scale); return cudaGetLastError();
    case 11: k_step32<S, 128, 8><<<pair_grid(L, 128), 128, 0, stream>>>(fin, fout, L, a, inv_scale); return cudaGetLastError();
    case 12: k_step32<S, 64, 0><<<pair_grid(L, 64), 64, 0, stream>>>(fin, fout, L, a, inv_scale); return cudaGetLastError();
    case 9:
        if constexpr (std::is_same<S, __half>::value)
        {
            const dim3 g((unsigned)(((L.nx + 3) / 4 + 127) / 128), (unsigned)L.ny, (unsigned)L.nz);
            k_step_quad<128, 6><<<g, 128, 0, stream>>>(fin, fout, L, a, inv_scale);
            return cudaGetLastError();
        }
        variant = 3;
        break;
    default: break;
    }
    switch (variant)
    {
    case 1: k_step<S, 128, 8><<<pair_grid(L, 128), 128, 0, stream>>>(fin, fout, L, a, inv_scale); break;
    case 2: k_step<S, 256, 4><<<pair_grid(L, 256), 256, 0, stream>>>(fin, fout, L, a, inv_scale); break;
    case 3: k_step<S, 64, 0><<<pair_grid(L, 64), 64, 0, stream>>>(fin, fout, L, a, inv_scale); break;
    default: k_step<S, 128, 0><<<pair_grid(L, 128), 128, 0, stream>>>(fin, fout, L, a, inv_scale); break;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_build_links(const uint8_t* mask_ref, uint32_t* links, uint32_t* near, const Layout& L,
                               cudaStream_t stream)
{
    k_build_links<<<row_grid(L), 128, 0, stream>>>(mask_ref, links, near, L);
    return cudaGetLastError();
}

cudaError_t launch_step(int storage, const void* fin, void* fout, const Layout& L, const StepArgs& a,
                        float scale, int variant, int grid, cudaStream_t stream)
{
    if (storage == 0)
        return launch_step_t<float>((const float*)fin, (float*)fout, L, a, 1.0f, variant, grid, stream);
    return launch_step_t<__half>((const __half*)fin, (__half*)fout, L, a, 1.0f / scale, variant, grid, stream);
}

cudaError_t prepare_step(int storage, int variant, int device, int* grid)
{
    *grid = 0;
    const bool h = storage != 0;
    switch (variant)
    {
    case 4: return h ? prepare_staged<__half, 256, 3>(device, grid) : prepare_staged<float, 256, 3>(device, grid);
    case 5: return h ? prepare_staged<__half, 256, 2>(device, grid) : prepare_staged<float, 256, 2>(device, grid);
    case 6: return h ? prepare_staged<__half, 128, 4>(device, grid) : prepare_staged<float, 128, 4>(device, grid);
    case 7: return h ? prepare_staged<__half, 512, 2>(device, grid) : prepare_staged<float, 512, 2>(device, grid);
    default: return cudaSuccess;
    }
}

cudaError_t launch_source(int storage, void* f, const Layout& L, const StepArgs& sa, const SourceArgs& a,
                          cudaStream_t stream)
{
    if (storage == 0) k_source<float><<<1, 512, 0, stream>>>((float*)f, L, sa, a);
    else k_source<__half><<<1, 512, 0, stream>>>((__half*)f, L, sa, a);
    return cudaGetLastError();
}

cudaError_t launch_ghost(int storage, void* f, const Layout& L, const GhostArgs& a, cudaStream_t stream)
{
    if (a.total <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((a.total + 127) / 128);
    if (storage == 0) k_ghost<float><<<blocks, 128, 0, stream>>>((float*)f, L, a);
    else k_ghost<__half><<<blocks, 128, 0, stream>>>((__half*)f, L, a);
    return cudaGetLastError();
}

cudaError_t launch_probe(int storage, const void* f, const Layout& L, const StepArgs& sa, const ProbeArgs& a,
                         cudaStream_t stream)
{
    if (storage == 0) k_probe<float><<<1, 256, 0, stream>>>((const float*)f, L, sa, a);
    else k_probe<__half><<<1, 256, 0, stream>>>((const __half*)f, L, sa, a);
    return cudaGetLastError();
}

cudaError_t launch_field_rho(int storage, const void* f, float* out, const Layout& L, const StepArgs& sa,
                             float scale, cudaStream_t stream)
{
    if (storage == 0) k_field_rho<float><<<row_grid(L), 128, 0, stream>>>((const float*)f, out, L, sa, 1.0f / scale);
    else k_field_rho<__half><<<row_grid(L), 128, 0, stream>>>((const __half*)f, out, L, sa, 1.0f / scale);
    return cudaGetLastError();
}

cudaError_t launch_export_f(int storage, const void* f, double* out, const Layout& L, const XFace& xf, float scale,
                            cudaStream_t stream)
{
    if (storage == 0) k_export_f<float><<<1184, 256, 0, stream>>>((const float*)f, out, L, xf, 1.0f / scale);
    else k_export_f<__half><<<1184, 256, 0, stream>>>((const __half*)f, out, L, xf, 1.0f / scale);
    return cudaGetLastError();
}

cudaError_t launch_import_f(int storage, void* f, const double* in, const Layout& L, const XFace& xf, float scale,
                            cudaStream_t stream)
{
    if (storage == 0) k_import_f<float><<<1184, 256, 0, stream>>>((float*)f, in, L, xf, scale);
    else k_import_f<__half><<<1184, 256, 0, stream>>>((__half*)f, in, L, xf, scale);
    return cudaGetLastError();
}

}  // namespace lbm
