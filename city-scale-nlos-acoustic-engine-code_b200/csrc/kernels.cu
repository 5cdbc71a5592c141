// sm_100a kernels of the D3Q19 acoustic step (family-B semantics of
// 06_transient_localization_dx1.cpp).  Storage is FP32 or FP16 deviations from
// rest equilibrium in the block-interleaved layout of device.hpp; arithmetic
// is FP32 (packed FP32x2 where two cells go together), with FP64 for the
// source-weight reduction and the probe accumulators.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "check.cuh"
#include "device.hpp"
#include "lattice.cuh"

namespace lbm {
namespace {

constexpr unsigned kFull = 0xffffffffu;

#ifdef LBM_CHECK
// Extents of the side arrays (elements), for the bounds-checked build.
__device__ __forceinline__ long long links_extent(const Layout& L) { return L.plane * (L.nz + 2); }
__device__ __forceinline__ long long near_extent(const Layout& L)
{
    return (long long)L.words_per_row * (L.ny + 2) * (L.nz + 2);
}
__device__ __forceinline__ long long xgh_extent(const Layout& L) { return 2LL * 19 * (L.nz + 2) * (L.ny + 2); }
__device__ __forceinline__ long long xexp_extent(const Layout& L) { return 2LL * 19 * L.nz * L.ny; }
#endif

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
};

template <>
struct Io<__half>
{
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float ldw(const __half* p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
};

// Two x-adjacent cells as one aligned vector: float2 (8 B) or half2 (4 B).
// `V` is the raw register form that is shuffled between lanes.
template <typename S>
struct PairIo;

template <>
struct PairIo<float>
{
    using V = float2;
    static __device__ __forceinline__ V ld(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
    static __device__ __forceinline__ void st(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
    static __device__ __forceinline__ float2 cvt(V v) { return v; }
    static __device__ __forceinline__ float hi_of(V v) { return v.y; }
    static __device__ __forceinline__ float lo_of(V v) { return v.x; }
    // cells (c-1, c) from the previous pair's high element and cur = (c, c+1)
    static __device__ __forceinline__ float2 left(float prev_hi, V cur) { return make_float2(prev_hi, cur.x); }
    // cells (c+1, c+2) from cur = (c, c+1) and the next pair's low element
    static __device__ __forceinline__ float2 right(V cur, float next_lo) { return make_float2(cur.y, next_lo); }
    static __device__ __forceinline__ float rnd(float v) { return v; }   // value as stored
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
    // the whole 32-bit word is shuffled; the byte permute picks the half
    static __device__ __forceinline__ unsigned hi_of(V v) { return v; }
    static __device__ __forceinline__ unsigned lo_of(V v) { return v; }
    static __device__ __forceinline__ float2 left(unsigned prev, V cur) { return cvt(__byte_perm(prev, cur, 0x5432)); }
    static __device__ __forceinline__ float2 right(V cur, unsigned next) { return cvt(__byte_perm(cur, next, 0x5432)); }
    static __device__ __forceinline__ float rnd(float v) { return __half2float(__float2half_rn(v)); }
};

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

__device__ __forceinline__ uint32_t near_bits(const StepArgs& a, const Layout& L, int col, int j, int k)
{
    return a.near[((long long)k * (L.ny + 2) + j) * L.words_per_row + (col >> 5)] >> (col & 31);
}

// Pulled populations of one cell (halo-inclusive coordinates i, j, k),
// halfway bounce-back included (06:918-931); x-halo sources read the x-face
// ghosts.  Used by the probe and field kernels.
template <typename S>
__device__ __forceinline__ void pull_cell(const S* __restrict__ f, const Layout& L, const StepArgs& sa, int i, int j,
                                          int k, float (&G)[Q], bool& solid)
{
    const uint32_t lk = sa.links[L.cell(i, j, k)];
    solid = (lk & kSolidSelfBit) != 0u;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int si = i - ex(q);
        long long e = -1;
        G[q] = 0.f;
        if ((lk >> q) & 1u) e = L.elem(inv(q), i, j, k);
        else if (si == 0) G[q] = sa.xf.xgh[sa.xf.gh_index(0, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else if (si == L.nx + 1) G[q] = sa.xf.xgh[sa.xf.gh_index(1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else e = L.elem(q, si, j - ey(q), k - ez(q));
        if (e >= 0 && LBM_IN(kChkProbe, e, L.total)) G[q] = Io<S>::ld(f + e);
    }
}

// y and z components of the velocities, for per-lane index arithmetic
__constant__ signed char c_ey[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
__constant__ signed char c_ez[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};

// ---------------------------------------------------------------- step
// Packed FP32x2 arithmetic (sm_100): both cells of a thread's pair in one
// instruction.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }

// BGK + sponge of two cells in lockstep, in place, deviation form (06:940-967).
// With stored G = scale * (f - w):
//   rho' = sum G, J = sum c G, r = 1 + rho'/scale (guard r <= 0 -> 1e-12, 06:948)
//   Geq_q = w_q (rho' + 3 c.J + (4.5 (c.J)^2 - 1.5 J^2) / (scale r))
//   G'    = (1 - sigma) (G - omega (G - Geq))      [sponge blend toward w_q, 06:955-965]
// A SOLID cell gets cA = 1, cB = 0, so its pulled values pass through
// unchanged (06:933-938).  on_moments(rho', jx, jy, jz) receives the moments
// of the pulled populations as soon as they are summed (the adjoint's forward
// data), so nothing beyond the collision's own values stays live for them.
template <typename OnMoments>
__device__ __forceinline__ void collide2(float2 (&G)[Q], float inv_scale, float omega, float2 sigma, bool solid0,
                                         bool solid1, OnMoments&& on_moments)
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
    on_moments(rho, jx, jy, jz);
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

// Fused pull-stream + halfway bounce-back + BGK + sponge (06:906-972), two
// x-adjacent cells per thread.  Direction q of the pair comes from the row
// (j - ey, k - ez) of the block-interleaved layout as one aligned vector at
// a compile-time offset from that row's base; the +-1 x shift of directions
// with ex != 0 takes the missing neighbour element from the adjacent lane
// (warp shuffle) and, at the warp edge, from one extra aligned load.  Cells
// next to the x faces take their x-halo sources from the x-face ghosts and
// export their results for the next ghost fill.
// MOM: also write the moments (rho', J) of every cell's pulled populations to
// `mom` (PairMoments: 12-bit floats, one record per x pair), the forward data
// the adjoint's BGK Jacobian needs.
// FP16 bits of x rounded to nearest-even at their 4 lowest mantissa bits:
// sign at bit 11, exponent at bits 6-10, 6 mantissa bits (finite values only).
__device__ __forceinline__ unsigned to_f12(float x)
{
    const unsigned h = (unsigned)__half_as_ushort(__float2half_rn(x));
    const unsigned mag = h & 0x7fffu;
    const unsigned r = min((mag + 7u + ((mag >> 4) & 1u)) >> 4, 0x7bfu);
    return ((h >> 15) << 11) | r;
}
__device__ __forceinline__ PairMoments pack_moments(float4 m0, float4 m1)
{
    const unsigned v0 = to_f12(m0.x), v1 = to_f12(m0.y), v2 = to_f12(m0.z), v3 = to_f12(m0.w);
    const unsigned v4 = to_f12(m1.x), v5 = to_f12(m1.y), v6 = to_f12(m1.z), v7 = to_f12(m1.w);
    return PairMoments{{v0 | (v1 << 12) | (v2 << 24), (v2 >> 8) | (v3 << 4) | (v4 << 16) | (v5 << 28),
                        (v5 >> 4) | (v6 << 8) | (v7 << 20)}};
}

template <typename S, int BLOCK, int MINB, bool MOM = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_step(const S* __restrict__ fin, S* __restrict__ fout, Layout L,
                                                      StepArgs a, float inv_scale,
                                                      PairMoments* __restrict__ mom = nullptr)
{
    using P = PairIo<S>;
    constexpr int BC = block_cells(sizeof(S));   // cells per interleaved block
    constexpr int BE = 19 * BC;                   // elements per block
    const int lane = threadIdx.x & 31;
    const int c0r = 2 * (blockIdx.x * BLOCK + threadIdx.x);   // first column (0-based) of the pair
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~1);         // inactive lanes shadow a valid pair
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    const long long e0 = L.elem(0, c0 + 1, j, k);
    const S* own = fin + e0;
    const long long rs = L.row_stride, ps = L.plane_stride;

    // pair load (the bounds-checked build tests the index first)
    const auto ldp = [&](const S* p) -> typename P::V {
        if (LBM_IN(kChkStepLoad, p - fin, L.total - 1)) return P::ld(p);
        return typename P::V{};
    };

    uint32_t lk0 = 0, lk1 = 0;
    if (active)
    {
        const uint32_t b = near_bits(a, L, c0, j, k) & 3u;
        const long long cl = L.cell(c0 + 1, j, k);
        if (b & 1u) lk0 = a.links[cl];
        if (b & 2u) lk1 = a.links[cl + 1];
    }
    const bool any_link = __any_sync(kFull, (lk0 | lk1) != 0u);

    float2 G[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const S* row = own - (ey(q) * rs + ez(q) * ps);
        const typename P::V cur = ldp(row + q * BC);
        if (ex(q) == 0)
        {
            G[q] = P::cvt(cur);
        }
        else if (ex(q) > 0)
        {
            // lane 0 sits at the start of a block: its left neighbour pair is
            // the last pair of the previous block
            auto prev = __shfl_up_sync(kFull, P::hi_of(cur), 1);
            if (lane == 0) prev = P::hi_of(ldp(row + q * BC - BE + (BC - 2)));
            G[q] = P::left(prev, cur);
        }
        else
        {
            // lane 31 sits at the last pair of a block: its right neighbour
            // pair is the first pair of the next block
            auto next = __shfl_down_sync(kFull, P::lo_of(cur), 1);
            if (lane == 31) next = P::lo_of(ldp(row + q * BC + BE - (BC - 2)));
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
                const float2 o = P::cvt(ldp(own + inv(q) * BC));
                if ((lk0 >> q) & 1u) G[q].x = o.x;
                if ((lk1 >> q) & 1u) G[q].y = o.y;
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
    collide2(G, inv_scale, a.omega, sg, (lk0 & kSolidSelfBit) != 0u, (lk1 & kSolidSelfBit) != 0u,
             [&](float2 rho, float2 jx, float2 jy, float2 jz) {
                 if constexpr (MOM)
                 {
                     const long long pi = ((long long)(k - 1) * L.ny + (j - 1)) * ((L.nx + 1) >> 1) + (c0 >> 1);
                     mom[pi] = pack_moments(make_float4(rho.x, jx.x, jy.x, jz.x),
                                            c0 + 1 < L.nx ? make_float4(rho.y, jx.y, jy.y, jz.y)
                                                          : make_float4(0.f, 0.f, 0.f, 0.f));
                 }
             });

    S* out = fout + e0;
#pragma unroll
    for (int q = 0; q < Q; ++q)
        if (LBM_IN(kChkStepStore, e0 + q * BC, L.total - 1)) P::st(out + q * BC, G[q]);

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

// ---------------------------------------------------------------- FP16 step
// FP16 storage keeps the 19 directions of a cell pair packed as half2 words
// through the whole update: the moment pass and the update pass each convert
// a word to float2 right before use, so no 19 x float2 array is ever live and
// the kernel needs far fewer registers (more warps, more loads in flight).
__device__ __forceinline__ float2 h2f(unsigned u) { return PairIo<__half>::cvt(u); }
__device__ __forceinline__ unsigned f2h(float2 v)
{
    const __half2 h = __float22half2_rn(v);
    return *reinterpret_cast<const unsigned*>(&h);
}
__device__ __forceinline__ unsigned set_lo(unsigned w, float v)
{
    return (w & 0xffff0000u) | (unsigned)__half_as_ushort(__float2half_rn(v));
}
__device__ __forceinline__ unsigned set_hi(unsigned w, float v)
{
    return (w & 0x0000ffffu) | ((unsigned)__half_as_ushort(__float2half_rn(v)) << 16);
}

// collide2() on packed FP16 words: each word is converted to FP32 once; the moments share partial sums
// (rho = g0 + rest + S(x+) + S(x-), jx = S(x+) - S(x-)); each direction of a
// pair (q, inv q) is two FMAs from the pair's equilibrium term
//   e = (cB w k45) (c.J)^2 + cB w base,   G'_q = cA G_q + e +- 3 cB w (c.J).
// Same formulas as collide2(); the rounding order differs.
__device__ __forceinline__ void collide2_grouped(unsigned (&w)[Q], float inv_scale, float omega, float2 sigma,
                                                 bool solid0, bool solid1)
{
    float2 g[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) g[q] = h2f(w[q]);
    const float2 sxp = add2(add2(add2(g[1], g[7]), add2(g[8], g[11])), g[12]);
    const float2 sxn = add2(add2(add2(g[2], g[9]), add2(g[10], g[13])), g[14]);
    const float2 rest = add2(add2(add2(g[3], g[4]), add2(g[5], g[6])), add2(add2(g[15], g[16]), add2(g[17], g[18])));
    const float2 rho = add2(add2(g[0], rest), add2(sxp, sxn));
    const float2 jx = sub2(sxp, sxn);
    const float2 jy = sub2(add2(add2(add2(g[3], g[7]), add2(g[9], g[15])), g[16]),
                           add2(add2(add2(g[4], g[8]), add2(g[10], g[17])), g[18]));
    const float2 jz = sub2(add2(add2(add2(g[5], g[11]), add2(g[13], g[15])), g[17]),
                           add2(add2(add2(g[6], g[12]), add2(g[14], g[16])), g[18]));
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
    const float2 K1 = mul2(cBw1, k45), K2 = mul2(cBw2, k45);
    const float2 B1 = mul2(cBw1, base), B2 = mul2(cBw2, base);
    const float2 T1 = mul2(cB, f2(3.0f * wf(1))), T2 = mul2(cB, f2(3.0f * wf(7)));
    const float2 N1 = mul2(cB, f2(-3.0f * wf(1))), N2 = mul2(cB, f2(-3.0f * wf(7)));
    w[0] = f2h(fma2(cA, g[0], mul2(mul2(cB, f2(wf(0))), base)));
#pragma unroll
    for (int p = 0; p < 9; ++p)
    {
        const int q = pair_head(p);
        const int qb = inv(q);
        float2 cj;
        if (p == 0) cj = jx;
        else if (p == 1) cj = jy;
        else if (p == 2) cj = jz;
        else if (p == 3) cj = add2(jx, jy);
        else if (p == 4) cj = sub2(jx, jy);
        else if (p == 5) cj = add2(jx, jz);
        else if (p == 6) cj = sub2(jx, jz);
        else if (p == 7) cj = add2(jy, jz);
        else cj = sub2(jy, jz);
        const float2 e = fma2(q < 7 ? K1 : K2, mul2(cj, cj), q < 7 ? B1 : B2);
        w[q] = f2h(fma2(q < 7 ? T1 : T2, cj, fma2(cA, g[q], e)));
        w[qb] = f2h(fma2(q < 7 ? N1 : N2, cj, fma2(cA, g[qb], e)));
    }
}

// ---------------------------------------------------------------- FP16 step, warp pipelines
// Each warp walks whole rows one interleaved block (64 cells, two per lane)
// at a time and keeps the source lines of its next P blocks in flight as
// cp.async copies into its own ring of shared-memory slots: the bytes in
// flight no longer depend on registers or on resident warps, and no barrier
// couples the warps of a CTA.  A block's 19 source lines (direction q from
// row (j - ey, k - ez)) are 152 16-byte pieces, five copy instructions per
// lane.  The x neighbour of the block's first / last cell is the last /
// first element of the previous / next block of the same row, which the ring
// still / already holds (at the row ends the x-face ghosts replace it).  The
// near-solid words of a block are loaded one block ahead of its copies and
// its links words travel with the copies when any bit is set.
namespace wp {
constexpr int kPopBytes = 19 * 128;           // one block's 19 source lines
constexpr int kLinkOff = kPopBytes;           // 64 links words
constexpr int kNearOff = kPopBytes + 256;     // the block's 2 near-solid words
constexpr int kGhostOff = kNearOff + 16;      // x-face ghosts of a row-end block: 5 per side
constexpr int kSlotBytes = kGhostOff + 48;
// Directions with ex > 0 (ghosts of the low x face) and ex < 0 (high face).
__device__ __forceinline__ int ghost_dir(int i) { return i < 5 ? (i < 1 ? 1 : i < 3 ? i + 6 : i + 8) : (i < 6 ? 2 : i < 8 ? i + 3 : i + 5); }
}  // namespace wp

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Position of direction q (ex != 0) in a slot's x-face ghosts (inverse of wp::ghost_dir).
__host__ __device__ constexpr int ghost_slot(int q)
{
    constexpr int t[Q] = {-1, 0, 5, -1, -1, -1, -1, 1, 2, 6, 7, 3, 4, 8, 9, -1, -1, -1, -1};
    return t[q];
}

template <int P, int WARPS, int MINB>
__global__ void __launch_bounds__(32 * WARPS, MINB) k_step_hw(const __half* __restrict__ fin,
                                                               __half* __restrict__ fout, Layout L, StepArgs a,
                                                               float inv_scale)
{
    constexpr int S = P + 2;   // ring slots: blocks t - 1 .. t + P
    constexpr uint32_t kDirBits = (1u << Q) - 1u;
    extern __shared__ __align__(128) unsigned char wp_smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned char* ring = wp_smem + warp * (S * wp::kSlotBytes);
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring);
    const int nrows = L.ny * L.nz;
    const int all_warps = gridDim.x * WARPS;
    const int r0 = blockIdx.x * WARPS + warp;   // rows r0, r0 + all_warps, ...; r = (k-1) ny + (j-1)
    if (r0 >= nrows) return;

    // element offsets of this lane's five 16-byte pieces from the destination block
    int poff[5];
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        const int p = i * 32 + lane;
        const int q = min(p >> 3, 18);
        poff[i] = -(c_ey[q] * (int)L.row_stride + c_ez[q] * (int)L.plane_stride) + q * 64 + (p & 7) * 8;
    }

    // lanes 0-4 copy the low-face ghosts of a row-start block, lanes 5-9 the
    // high-face ghosts of a row-end block: ghost of direction q for row
    // (j, k) is xgh[gh_index(side, q, j - ey, k - ez)] = row (k (ny+2) + j) + goff
    const int gq = wp::ghost_dir(lane < 10 ? lane : 0);
    const int goff = (lane < 5 ? 0 : 19) * (L.nz + 2) * (L.ny + 2) + gq * (L.nz + 2) * (L.ny + 2) -
                     c_ez[gq] * (L.ny + 2) - c_ey[gq];

    // ---- copy cursor: the next block whose lines are copied
    int ci_r = r0, ci_b = 0;
    const __half* ci_src = nullptr;     // the block's own position (lines are offset by poff)
    const uint32_t* ci_near = nullptr;  // the block's two near-solid words
    const uint32_t* ci_link = nullptr;  // links words of this lane's two cells
    const float* ci_gh = nullptr;       // this lane's x-face ghost of the row
    const auto ci_row = [&]() {
        const int k = 1 + ci_r / L.ny, j = 1 + ci_r - (k - 1) * L.ny;
        ci_src = fin + L.elem(0, 1, j, k);
        ci_near = a.near + ((long long)k * (L.ny + 2) + j) * L.words_per_row;
        ci_link = a.links + L.cell(1, j, k) + 2 * lane;
        ci_gh = a.xf.xgh + ((long long)k * (L.ny + 2) + j) + goff;
    };
    const auto ci_next = [&]() {
        ci_src += 19 * 64;
        ci_near += 2;
        ci_link += 64;
        if (++ci_b == L.nb)
        {
            ci_b = 0;
            ci_r += all_warps;
            if (ci_r < nrows) ci_row();
        }
    };
    uint32_t n0 = 0u, n1 = 0u;   // near words of the copy cursor's block, loaded one block ahead
    const auto load_near = [&]() {
        n0 = LBM_IN(kChkHwNear, ci_near - a.near, near_extent(L)) ? __ldg(ci_near) : 0u;
        n1 = ci_b * 64 + 32 < L.nx && LBM_IN(kChkHwNear, ci_near + 1 - a.near, near_extent(L)) ? __ldg(ci_near + 1)
                                                                                                   : 0u;
    };
    const auto issue = [&](int slot) {
        const uint32_t dst = ring_s + slot * wp::kSlotBytes;
#pragma unroll
        for (int i = 0; i < 5; ++i)
            if ((i < 4 || lane < 24) && LBM_IN(kChkHwLine, (ci_src - fin) + poff[i], L.total - 7))
                cp_async16(dst + (i * 32 + lane) * 16, ci_src + poff[i]);
        if (lane < 2) reinterpret_cast<uint32_t*>(ring + slot * wp::kSlotBytes + wp::kNearOff)[lane] = lane ? n1 : n0;
        if ((n0 | n1) != 0u && ci_b * 64 + 2 * lane < L.nx &&
            LBM_IN(kChkHwLinks, ci_link - a.links, links_extent(L) - 1))
            cp_async8(dst + wp::kLinkOff + lane * 8, ci_link);
        if (((ci_b == 0 && lane < 5) || (ci_b == L.nb - 1 && lane >= 5 && lane < 10)) &&
            LBM_IN(kChkHwGhost, ci_gh - a.xf.xgh, xgh_extent(L)))
            cp_async4(dst + wp::kGhostOff + lane * 4, ci_gh);
    };

    // ---- update cursor: the block being updated
    int cc_r = r0, cc_b = 0, cc_j = 0, cc_k = 0, c0 = 0;
    const unsigned* own = nullptr;   // this lane's word of line 0 of the block (line q: own[32 q])
    unsigned* outp = nullptr;
    float syz = 0.f;
    const auto cc_row = [&]() {
        cc_k = 1 + cc_r / L.ny;
        cc_j = 1 + cc_r - (cc_k - 1) * L.ny;
        const long long e = L.elem(0, 1, cc_j, cc_k);
        own = reinterpret_cast<const unsigned*>(fin + e) + lane;
        outp = reinterpret_cast<unsigned*>(fout + e) + lane;
        c0 = 2 * lane;
        syz = fmaxf(__ldg(a.sig_y + cc_j - 1), __ldg(a.sig_z + cc_k - 1));
    };
    const auto cc_next = [&]() {
        own += 19 * 32;
        outp += 19 * 32;
        c0 += 64;
        if (++cc_b == L.nb)
        {
            cc_b = 0;
            cc_r += all_warps;
            if (cc_r < nrows) cc_row();
        }
    };

    ci_row();
    cc_row();
#pragma unroll 1
    for (int p = 0; p < P; ++p)
    {
        if (ci_r < nrows)
        {
            load_near();
            issue(p);
            ci_next();
        }
        cp_async_commit();
    }
    if (ci_r < nrows) load_near();

    int st = 0;   // slot of block t
#pragma unroll 1
    while (cc_r < nrows)
    {
        const int sp = st == 0 ? S - 1 : st - 1;
        const int sn = st == S - 1 ? 0 : st + 1;
        int si = st + P;
        if (si >= S) si -= S;
        if (ci_r < nrows)
        {
            issue(si);
            ci_next();
            if (ci_r < nrows) load_near();
        }
        cp_async_commit();
        cp_async_wait<P - 1>();   // blocks up to t + 1 have landed
        __syncwarp();

        const int j = cc_j, k = cc_k;
        const bool active = c0 < L.nx;
        const int last = L.nx - 1 - c0;
        const bool xlo = c0 == 0;
        const bool xhi = last >= 0 && last < 2;
        const bool edge = cc_b == 0 || cc_b == L.nb - 1;
        const unsigned char* slot = ring + st * wp::kSlotBytes;

        // links words of block t (they came with its lines, when a near-solid bit is set)
        // sponge strengths of the two cells, first so that the loads are in flight early
        const float sx0 = active ? __ldg(a.sig_x + c0) : 0.f;
        const float sx1 = c0 + 1 < L.nx ? __ldg(a.sig_x + c0 + 1) : 0.f;
        const uint2 nw = *reinterpret_cast<const uint2*>(slot + wp::kNearOff);
        uint32_t lk0 = 0u, lk1 = 0u;
        bool any_link = false;
        if ((nw.x | nw.y) != 0u)
        {
            const uint32_t bits = active ? ((lane < 16 ? nw.x : nw.y) >> ((2 * lane) & 31)) & 3u : 0u;
            const uint32_t* lw = reinterpret_cast<const uint32_t*>(slot + wp::kLinkOff) + 2 * lane;
            lk0 = (bits & 1u) ? lw[0] : 0u;
            lk1 = (bits & 2u) ? lw[1] : 0u;
            any_link = __any_sync(kFull, ((lk0 | lk1) & kDirBits) != 0u);
        }
        const uint32_t lka = (lk0 | lk1) & kDirBits;

        // pulled words: line q of the slot, shifted by ex(q) across lanes / blocks
        const unsigned* cur = reinterpret_cast<const unsigned*>(slot) + lane;   // line q: cur[32 q]
        const unsigned* prv = lane > 0 ? cur - 1
                                       : (cc_b > 0 ? reinterpret_cast<const unsigned*>(ring + sp * wp::kSlotBytes) + 31
                                                   : cur);
        const unsigned* nxt =
            lane < 31 ? cur + 1
                      : (cc_b + 1 < L.nb ? reinterpret_cast<const unsigned*>(ring + sn * wp::kSlotBytes) : cur);
        unsigned w[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const unsigned v = cur[32 * q];
            if (ex(q) == 0) w[q] = v;
            else if (ex(q) > 0) w[q] = __byte_perm(prv[32 * q], v, 0x5432);
            else w[q] = __byte_perm(v, nxt[32 * q], 0x5432);
        }
        if (any_link)
        {
            // halfway bounce-back: the own cell's word of the opposite direction
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                const unsigned o =
                    ((lka >> q) & 1u) &&
                            LBM_IN(kChkHwBounce, 2 * (own - reinterpret_cast<const unsigned*>(fin)) + inv(q) * 64,
                                   L.total - 1)
                        ? __ldg(own + inv(q) * 32)
                        : 0u;
                const unsigned m = ((0u - ((lk0 >> q) & 1u)) & 0x0000ffffu) | ((0u - ((lk1 >> q) & 1u)) & 0xffff0000u);
                w[q] = (w[q] & ~m) | (o & m);
            }
        }
        if (edge)
        {
            // x-face ghosts of the row ends (they came with the block's lines)
            const float* gs = reinterpret_cast<const float*>(slot + wp::kGhostOff);
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (ex(q) == 0) continue;
                const float g = gs[ghost_slot(q)];
                if (ex(q) > 0 && xlo && !((lk0 >> q) & 1u)) w[q] = set_lo(w[q], g);
                if (ex(q) < 0 && xhi && last == 0 && !((lk0 >> q) & 1u)) w[q] = set_lo(w[q], g);
                if (ex(q) < 0 && xhi && last == 1 && !((lk1 >> q) & 1u)) w[q] = set_hi(w[q], g);
            }
        }
        if (active)
        {
            const float2 sg = make_float2(fmaxf(sx0, syz), fmaxf(sx1, syz));
            collide2_grouped(w, inv_scale, a.omega, sg, (lk0 & kSolidSelfBit) != 0u, (lk1 & kSolidSelfBit) != 0u);
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (LBM_IN(kChkHwStore, 2 * (outp - reinterpret_cast<unsigned*>(fout)) + 64 * q, L.total - 1))
                    outp[32 * q] = w[q];
            if (edge && (xlo | xhi))
            {
#pragma unroll
                for (int q = 0; q < Q; ++q)
                {
                    if (!LBM_IN(kChkHwExport, a.xf.exp_index(xlo ? 0 : 1, q, j, k, L.ny, L.nz), xexp_extent(L)))
                        continue;
                    if (xlo) a.xf.xexp[a.xf.exp_index(0, q, j, k, L.ny, L.nz)] = h2f(w[q]).x;
                    if (xhi && last == 0) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = h2f(w[q]).x;
                    if (xhi && last == 1) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = h2f(w[q]).y;
                }
            }
        }
        __syncwarp();   // every lane is done with slot t - 1 before the next copy lands there
        cc_next();
        st = sn;
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------- z-slab messages
// The populations that cross a z cut: the 5 directions with ez = +1 leave a
// slab's top plane for the upper neighbour's halo plane 0, the 5 with ez = -1
// its bottom plane for the lower neighbour's halo plane nz + 1.  A message holds
// those directions of every row of the plane (y-halo rows included) as whole
// 128-byte lines, [5][ny + 2][nb], then the two x-face ghost rows of the plane
// that the receiving plane's row-end cells pull (the two of the five with
// ex != 0), [2][ny + 2] floats.  The same kernel packs (plane -> message) and
// unpacks (message -> plane); it moves bytes, whatever the storage type.
__host__ __device__ constexpr int cross_dir(int up, int d)
{
    constexpr int u[5] = {5, 11, 13, 15, 17};   // ez = +1
    constexpr int w[5] = {6, 12, 14, 16, 18};   // ez = -1
    return up ? u[d] : w[d];
}
// the x-face ghost directions among them: side 0 (low face, ex > 0), side 1 (high face, ex < 0)
__host__ __device__ constexpr int cross_ghost_dir(int up, int side) { return up ? (side ? 13 : 11) : (side ? 14 : 12); }

template <bool PACK>
__global__ void __launch_bounds__(256) k_slab_msg(unsigned char* __restrict__ f, float* __restrict__ xgh,
                                                  unsigned char* __restrict__ msg, Layout L, int k, int up, int esz)
{
    const long long nl = 5LL * (L.ny + 2) * L.nb * 8;   // 16-byte pieces of the lines
    const long long ng = 2LL * (L.ny + 2);
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nl + ng;
         u += (long long)gridDim.x * blockDim.x)
    {
        if (u < nl)
        {
            const int piece = (int)(u & 7);
            long long line = u >> 3;
            const int b = (int)(line % L.nb);
            line /= L.nb;
            const int j = (int)(line % (L.ny + 2));
            const int d = (int)(line / (L.ny + 2));
            const long long e = kFrontElems + ((long long)k * (L.ny + 2) + j) * L.row_stride + (long long)b * 19 * L.bc +
                                (long long)cross_dir(up, d) * L.bc;
            uint4* fp = reinterpret_cast<uint4*>(f + e * esz) + piece;
            uint4* mp = reinterpret_cast<uint4*>(msg) + u;
            if (PACK) *mp = *fp;
            else *fp = *mp;
        }
        else
        {
            const long long g = u - nl;
            const int side = (int)(g / (L.ny + 2)), j = (int)(g % (L.ny + 2));
            const long long gi = ((long long)(side * 19 + cross_ghost_dir(up, side)) * (L.nz + 2) + k) * (L.ny + 2) + j;
            float* mp = reinterpret_cast<float*>(msg + nl * 16) + g;
            if (PACK) *mp = xgh[gi];
            else xgh[gi] = *mp;
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
        links[L.cell(i, j, k)] = lk;
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
            if (ic < -R || ic >= L.nx + R || jc < -R || jc >= L.ny + R || kc - a.k_off < -R ||
                kc - a.k_off >= L.nz + R)
                continue;
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
        // weights in the coordinates of the whole grid; a z-slab holds layers k_off..
        gk -= a.k_off;
        bool fluid = false;
        if (in && gi >= 0 && gi < L.nx && gj >= 0 && gj < L.ny && gk >= 0 && gk < L.nz)
            fluid = (sa.links[L.cell(gi + 1, gj + 1, gk + 1)] & kSolidSelfBit) == 0u;
        const double bsum = block_sum(fluid ? ww : 0.0, red);
        const double sum = e.wsum > 0.0 ? e.wsum : bsum;   // a stencil across a z-slab cut
        if (sum < 1e-30) continue;
        const double A = e.mass / sum;
        // (the bounds-checked build skips a cell whose 19 directions leave the buffer; no
        // thread leaves the loop early, every thread reaches the barrier below)
        if (fluid && LBM_IN(kChkSource, L.elem(18, gi + 1, gj + 1, gk + 1), L.total))
        {
            const double add = A * ww * (double)a.scale;
            // the 19 directions of one cell are 19 distinct elements: every load
            // first (one round trip), then the stores
            S* p = f + L.elem(0, gi + 1, gj + 1, gk + 1);   // direction q at p + q * bc
            float v[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) v[q] = Io<S>::ldw(p + q * L.bc);
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                Io<S>::st(p + q * L.bc, v[q] + (float)(wd(q) * add));
                if (gi == 0 || gi == L.nx - 1)
                {
                    const float gs = Io<S>::ldw(p + q * L.bc);   // the stored value, as the step would export it
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

//
// Only the 5 directions that point from the ghost into the interior (e_axis =
// +1 on the low side, -1 on the high side) are ever pulled from a ghost cell
// (by the step, the probes, the field output, the slab messages and the
// adjoint); the fill computes and stores those and leaves the other 14 of the
// ghost cell as they are.
template <int AXIS, int SIDE>
__host__ __device__ constexpr bool inward(int q)
{
    return (AXIS == 0 ? ex(q) : AXIS == 1 ? ey(q) : ez(q)) == (SIDE ? -1 : 1);
}

template <int AXIS, int SIDE>
__device__ __forceinline__ void nscbc(float (&G)[Q], float inv_scale)
{
    constexpr int axis = AXIS, side = SIDE;
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
    // geq(B) - geq(I) = w_q (d0 + c.v + c^T M c), a quadratic form in
    // c_q whose ten coefficients are taken once per cell
    const float k45 = 4.5f * inv_scale;
    const float d0 = (rhoB - rho) - 1.5f * inv_scale * (rB * (bx * bx + by * by + bz * bz) - rI * (ux * ux + uy * uy + uz * uz));
    const float vx = 3.0f * (rB * bx - rI * ux), vy = 3.0f * (rB * by - rI * uy), vz = 3.0f * (rB * bz - rI * uz);
    const float mxx = k45 * (rB * bx * bx - rI * ux * ux), myy = k45 * (rB * by * by - rI * uy * uy),
                mzz = k45 * (rB * bz * bz - rI * uz * uz);
    const float mxy = 2.0f * k45 * (rB * bx * by - rI * ux * uy), mxz = 2.0f * k45 * (rB * bx * bz - rI * ux * uz),
                myz = 2.0f * k45 * (rB * by * bz - rI * uy * uz);
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        if (!inward<AXIS, SIDE>(q)) continue;
        float e = d0;
        if (ex(q)) e += mxx;
        if (ey(q)) e += myy;
        if (ez(q)) e += mzz;
        if (ex(q) * ey(q)) e += ex(q) * ey(q) * mxy;
        if (ex(q) * ez(q)) e += ex(q) * ez(q) * mxz;
        if (ey(q) * ez(q)) e += ey(q) * ez(q) * myz;
        if (ex(q)) e += ex(q) * vx;
        if (ey(q)) e += ey(q) * vy;
        if (ez(q)) e += ez(q) * vz;
        G[q] = fmaf(wf(q), e, G[q]);
    }
}

__device__ __forceinline__ void store_moments(const float (&G)[Q], float4* out)
{
    float rho, jx, jy, jz;
    moments(G, rho, jx, jy, jz);
    *out = make_float4(rho, jx, jy, jz);
}

// One face cell (two x-adjacent ones in FP16 y and z faces) of face (AXIS, SIDE).
template <typename S, int AXIS, int SIDE>
__device__ __forceinline__ void ghost_cell(S* __restrict__ f, const Layout& L, const GhostArgs& a, const GhostFace& F,
                                           long long t, int lt)
{
    const int v = lt / F.nu, u = lt - v * F.nu;
    const float inv_scale = 1.0f / a.scale;
    float G[Q];
    if constexpr (AXIS == 0)
    {
        // x faces: compact export -> compact ghost, both coalesced along j
        const int j = 1 + u, k = 1 + v;
        if (!LBM_IN(kChkGhost, a.xf.exp_index(SIDE, 18, j, k, L.ny, L.nz), xexp_extent(L)) ||
            !LBM_IN(kChkGhost, a.xf.gh_index(SIDE, 18, j, k, L.ny, L.nz), xgh_extent(L)))
            return;
#pragma unroll
        for (int q = 0; q < Q; ++q) G[q] = a.xf.xexp[a.xf.exp_index(SIDE, q, j, k, L.ny, L.nz)];
        if (a.face_mom) store_moments(G, a.face_mom + t);
        nscbc<AXIS, SIDE>(G, inv_scale);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (inward<AXIS, SIDE>(q)) a.xf.xgh[a.xf.gh_index(SIDE, q, j, k, L.ny, L.nz)] = G[q];
        return;
    }
    else if constexpr (std::is_same<S, __half>::value)
    {
        // y and z faces in FP16: the first half of the face's threads take two
        // x-adjacent cells each, one half2 per direction (a 64-cell block
        // holds both cells of an even-aligned pair); same values as one cell
        // per thread, half as many 2-byte accesses
        const int npair = (F.nu + 1) >> 1;
        if (lt >= npair * F.nv) return;
        const int vp = lt / npair, up = 2 * (lt - vp * npair);
        const bool two = up + 1 < F.nu;
        const int pi = 1 + up;
        const int pj = AXIS == 1 ? (SIDE ? L.ny : 1) : 1 + vp, pk = AXIS == 1 ? 1 + vp : (SIDE ? L.nz : 1);
        const int qj = AXIS == 1 ? (SIDE ? L.ny + 1 : 0) : pj, qk = AXIS == 1 ? pk : (SIDE ? L.nz + 1 : 0);
        constexpr int BCH = block_cells(sizeof(S));
        if (!LBM_IN(kChkGhost, L.elem(18, pi + (two ? 1 : 0), pj, pk), L.total) ||
            !LBM_IN(kChkGhost, L.elem(18, pi + (two ? 1 : 0), qj, qk), L.total))
            return;
        const __half* I = f + L.elem(0, pi, pj, pk);
        __half* B = f + L.elem(0, pi, qj, qk);
        float G1[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (two)
            {
                const float2 v2 = __half22float2(__ldg(reinterpret_cast<const __half2*>(I + q * BCH)));
                G[q] = v2.x;
                G1[q] = v2.y;
            }
            else
            {
                G[q] = Io<S>::ld(I + q * BCH);
                G1[q] = 0.f;
            }
        }
        const long long cell = F.first + (long long)vp * F.nu + up;   // the face enumeration of one cell a thread
        if (a.face_mom) store_moments(G, a.face_mom + cell);
        nscbc<AXIS, SIDE>(G, inv_scale);
        if (two)
        {
            if (a.face_mom) store_moments(G1, a.face_mom + cell + 1);
            nscbc<AXIS, SIDE>(G1, inv_scale);
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (inward<AXIS, SIDE>(q)) *reinterpret_cast<__half2*>(B + q * BCH) = __floats2half2_rn(G[q], G1[q]);
        }
        else
        {
#pragma unroll
            for (int q = 0; q < Q; ++q)
                if (inward<AXIS, SIDE>(q)) Io<S>::st(B + q * BCH, G[q]);
        }
    }
    else
    {
        const int ci = 1 + u;
        const int cj = AXIS == 1 ? (SIDE ? L.ny : 1) : 1 + v, gj = AXIS == 1 ? (SIDE ? L.ny + 1 : 0) : cj;
        const int ck = AXIS == 1 ? 1 + v : (SIDE ? L.nz : 1), gk = AXIS == 1 ? ck : (SIDE ? L.nz + 1 : 0);
        constexpr int BC = block_cells(sizeof(S));
        if (!LBM_IN(kChkGhost, L.elem(18, ci, cj, ck), L.total) ||
            !LBM_IN(kChkGhost, L.elem(18, ci, gj, gk), L.total) || !LBM_IN(kChkGhost, L.elem(0, ci, gj, gk), L.total))
            return;
        const S* I = f + L.elem(0, ci, cj, ck);
        S* B = f + L.elem(0, ci, gj, gk);
#pragma unroll
        for (int q = 0; q < Q; ++q) G[q] = Io<S>::ld(I + q * BC);
        if (a.face_mom) store_moments(G, a.face_mom + t);
        nscbc<AXIS, SIDE>(G, inv_scale);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (inward<AXIS, SIDE>(q)) Io<S>::st(B + q * BC, G[q]);
    }
}

template <typename S>
__global__ void __launch_bounds__(128) k_ghost(S* __restrict__ f, Layout L, GhostArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.total) return;
    int fi = 0;
    while (fi + 1 < a.nfaces && t >= a.face[fi + 1].first) ++fi;
    const GhostFace F = a.face[fi];
    const int lt = (int)(t - F.first);   // a face has fewer than 2^31 cells (nu, nv are ints of one grid)
    switch (F.axis * 2 + F.side)
    {
    case 0: ghost_cell<S, 0, 0>(f, L, a, F, t, lt); break;
    case 1: ghost_cell<S, 0, 1>(f, L, a, F, t, lt); break;
    case 2: ghost_cell<S, 1, 0>(f, L, a, F, t, lt); break;
    case 3: ghost_cell<S, 1, 1>(f, L, a, F, t, lt); break;
    case 4: ghost_cell<S, 2, 0>(f, L, a, F, t, lt); break;
    default: ghost_cell<S, 2, 1>(f, L, a, F, t, lt); break;
    }
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
        const int i = a.ijk[3 * p], j = a.ijk[3 * p + 1], k = a.ijk[3 * p + 2];
        double val;
        if (i < 0)
        {
            val = __longlong_as_double(0x7ff8000000000000LL);
        }
        else
        {
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
            if (!isfinite(val)) *a.nonfinite = 1;
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
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            float g;
            if (i == 0) g = xf.xgh[xf.gh_index(0, q, j, k, L.ny, L.nz)];
            else if (i == L.nx + 1) g = xf.xgh[xf.gh_index(1, q, j, k, L.ny, L.nz)];
            else g = Io<S>::ld(f + L.elem(q, i, j, k));
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
            S* p = f + L.elem(q, i, j, k);
            Io<S>::st(p, g);
            const float gs = Io<S>::ldw(p);   // the stored (rounded) value
            if (inner && i == 1) xf.xexp[xf.exp_index(0, q, j, k, L.ny, L.nz)] = gs;
            if (inner && i == L.nx) xf.xexp[xf.exp_index(1, q, j, k, L.ny, L.nz)] = gs;
        }
    }
}

// Self-test of the bounds-checked build: lane 5 tests an index one past its
// extent (nothing is accessed), which must be recorded as site kChkSelfTest.
__global__ void k_check_selftest()
{
    const int lane = threadIdx.x & 31;
    if (lane == 5 && !LBM_IN(kChkSelfTest, 32 + lane, 37)) return;
}

// Statically reserved device array for lbm_get_rho_noalloc: the field of
// (rho - 1) passes through it instead of a temporary cudaMalloc buffer.  It
// exists on every GPU that loads this library, for the life of the process.
static __device__ __align__(256) float g_field_scratch[kNoAllocFieldCells];
static_assert(sizeof(g_field_scratch) == sizeof(float) * LBM_NOALLOC_MAX_CELLS,
              "the static field array must hold the grid size lbm_get_rho_noalloc accepts");

dim3 row_grid(const Layout& L) { return dim3((unsigned)((L.nx + 127) / 128), (unsigned)L.ny, (unsigned)L.nz); }
dim3 pair_grid(const Layout& L, int block)
{
    return dim3((unsigned)(((L.nx + 1) / 2 + block - 1) / block), (unsigned)L.ny, (unsigned)L.nz);
}

// Warp-pipelined FP16 step: dynamic shared memory (one ring per warp) and a
// grid of as many CTAs as the GPU holds at once (every warp then walks rows
// all_warps apart).  The attribute and the occupancy are set up once per device.
template <int P, int WARPS, int MINB>
cudaError_t hw_ctas(int* out)
{
    constexpr int smem = WARPS * (P + 2) * wp::kSlotBytes;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    static std::mutex mu;
    static int ctas[kMaxDevices] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (!ctas[dev])
    {
        e = cudaFuncSetAttribute(k_step_hw<P, WARPS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int per_sm = 0, sms = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_hw<P, WARPS, MINB>, 32 * WARPS, smem);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        ctas[dev] = per_sm * sms;
    }
    *out = ctas[dev];
    return cudaSuccess;
}

template <int P, int WARPS, int MINB>
cudaError_t launch_hw(const __half* fin, __half* fout, const Layout& L, const StepArgs& a, float inv_scale,
                      cudaStream_t stream)
{
    // the per-lane source offsets are 32-bit
    if (L.plane_stride + L.row_stride + 19 * 64 > 0x7fffffffLL) return cudaErrorInvalidValue;
    int ctas = 0;
    const cudaError_t e = hw_ctas<P, WARPS, MINB>(&ctas);
    if (e != cudaSuccess) return e;
    const long long need = ((long long)L.ny * L.nz + WARPS - 1) / WARPS;
    const int grid = (int)(need < ctas ? need : ctas);
    k_step_hw<P, WARPS, MINB><<<grid, 32 * WARPS, WARPS * (P + 2) * wp::kSlotBytes, stream>>>(fin, fout, L, a, inv_scale);
    return cudaGetLastError();
}

template <typename S>
cudaError_t launch_step_t(const S* fin, S* fout, const Layout& L, const StepArgs& a, float inv_scale,
                          cudaStream_t stream)
{
    if constexpr (std::is_same<S, __half>::value)
        return launch_hw<2, 4, 5>(fin, fout, L, a, inv_scale, stream);
    k_step<S, 128, 0><<<pair_grid(L, 128), 128, 0, stream>>>(fin, fout, L, a, inv_scale);
    return cudaGetLastError();
}

}  // namespace

cudaError_t field_scratch_address(int device, float** ptr)
{
    // Host code cannot use the array's name as a device address; the address
    // is looked up once per device, with that device current (the caller
    // sets it), and cached.
    static std::mutex mu;
    static float* cached[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!cached[device])
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_field_scratch);
        if (e != cudaSuccess) return e;
        cached[device] = static_cast<float*>(p);
    }
    *ptr = cached[device];
    return cudaSuccess;
}

long long slab_message_bytes(const Layout& L) { return 5LL * (L.ny + 2) * L.nb * 128 + 8LL * (L.ny + 2); }

cudaError_t launch_slab_msg(bool pack, void* f, float* xgh, void* msg, const Layout& L, int k, int up, int esz,
                            cudaStream_t stream)
{
    const long long n = 5LL * (L.ny + 2) * L.nb * 8 + 2LL * (L.ny + 2);
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    if (pack)
        k_slab_msg<true><<<blocks, 256, 0, stream>>>((unsigned char*)f, xgh, (unsigned char*)msg, L, k, up, esz);
    else
        k_slab_msg<false><<<blocks, 256, 0, stream>>>((unsigned char*)f, xgh, (unsigned char*)msg, L, k, up, esz);
    return cudaGetLastError();
}

cudaError_t check_read_kernels(check::Status* out) { return check::read_and_clear(out); }

cudaError_t launch_check_selftest(cudaStream_t stream)
{
    k_check_selftest<<<1, 32, 0, stream>>>();
    return cudaGetLastError();
}

cudaError_t launch_build_links(const uint8_t* mask_ref, uint32_t* links, uint32_t* near, const Layout& L,
                               cudaStream_t stream)
{
    k_build_links<<<row_grid(L), 128, 0, stream>>>(mask_ref, links, near, L);
    return cudaGetLastError();
}

cudaError_t prepare_step(int storage)
{
    if (storage == 0) return cudaSuccess;
    int ctas = 0;
    return hw_ctas<2, 4, 5>(&ctas);
}

cudaError_t launch_step(int storage, const void* fin, void* fout, const Layout& L, const StepArgs& a,
                        float scale, cudaStream_t stream)
{
    if (storage == 0) return launch_step_t<float>((const float*)fin, (float*)fout, L, a, 1.0f, stream);
    return launch_step_t<__half>((const __half*)fin, (__half*)fout, L, a, 1.0f / scale, stream);
}

cudaError_t launch_step_moments(const float* fin, float* fout, const Layout& L, const StepArgs& a,
                                PairMoments* mom, cudaStream_t stream)
{
    k_step<float, 128, 0, true><<<pair_grid(L, 128), 128, 0, stream>>>(fin, fout, L, a, 1.0f, mom);
    return cudaGetLastError();
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
