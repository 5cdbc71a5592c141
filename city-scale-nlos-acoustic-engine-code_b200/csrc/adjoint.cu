// Reverse-time adjoint kernels of the fused D3Q19 step (FP32 storage, scale 1).
// See adjoint.hpp for the recursion.  Every kernel is a gather: the transposed
// pull-stream reads the adjoint populations of the neighbours that pulled
// from a cell, mirroring the forward pull.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "adjoint.hpp"
#include "check.cuh"
#include "lattice.cuh"

namespace lbm {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool interior(const Layout& L, int i, int j, int k)
{
    return i >= 1 && i <= L.nx && j >= 1 && j <= L.ny && k >= 1 && k <= L.nz;
}

// Index of an interior cell within the ghost-adjoint buffer of a face of
// axis `axis` (the same (u, v) enumeration as the forward ghost kernel).
__device__ __forceinline__ long long face_cell(const Layout& L, int axis, int i, int j, int k)
{
    if (axis == 0) return (long long)(j - 1) + (long long)(k - 1) * L.ny;
    if (axis == 1) return (long long)(i - 1) + (long long)(k - 1) * L.nx;
    return (long long)(i - 1) + (long long)(j - 1) * L.nx;
}
__device__ __forceinline__ long long face_cells(const Layout& L, int axis)
{
    if (axis == 0) return (long long)L.ny * L.nz;
    if (axis == 1) return (long long)L.nx * L.nz;
    return (long long)L.nx * L.ny;
}

// lamH^s at interior cell (i, j, k): transposed pull of lamF^s with the
// bounce-back links, plus the ghost-adjoint contributions of every open face
// the cell borders.
__device__ __forceinline__ void gather_lam(const Layout& L, const uint32_t* __restrict__ links,
                                           const float* __restrict__ lam, const float* __restrict__ gadj,
                                           const long long (&gadj_off)[6], int i, int j, int k, float (&lg)[Q])
{
    const uint32_t lk = links[L.cell(i, j, k)];
    const bool fluid = (lk & kSolidSelfBit) == 0u;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        float v = 0.f;
        const int di = i + ex(q), dj = j + ey(q), dk = k + ez(q);
        if (fluid && interior(L, di, dj, dk)) v = lam[L.elem(q, di, dj, dk)];
        if ((lk >> inv(q)) & 1u) v += lam[L.elem(inv(q), i, j, k)];
        lg[q] = v;
    }
    const int at[6] = {i == 1, i == L.nx, j == 1, j == L.ny, k == 1, k == L.nz};
#pragma unroll
    for (int f = 0; f < 6; ++f)
    {
        if (!at[f] || gadj_off[f] < 0) continue;
        const int axis = f / 2;
        const long long n = face_cells(L, axis), c = face_cell(L, axis, i, j, k);
#pragma unroll
        for (int q = 0; q < Q; ++q) lg[q] += gadj[gadj_off[f] + (long long)q * n + c];
    }
}

// ---- dual numbers over the four moments (rho', jx, jy, jz) ----------------
struct D4
{
    float v, d[4];
};
__device__ __forceinline__ D4 dc(float v)
{
    return D4{v, {0.f, 0.f, 0.f, 0.f}};
}
__device__ __forceinline__ D4 operator+(D4 a, D4 b)
{
    return D4{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2], a.d[3] + b.d[3]}};
}
__device__ __forceinline__ D4 operator-(D4 a, D4 b)
{
    return D4{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2], a.d[3] - b.d[3]}};
}
__device__ __forceinline__ D4 operator*(D4 a, D4 b)
{
    return D4{a.v * b.v,
              {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2],
               a.d[3] * b.v + a.v * b.d[3]}};
}
__device__ __forceinline__ D4 operator*(float s, D4 a)
{
    return D4{s * a.v, {s * a.d[0], s * a.d[1], s * a.d[2], s * a.d[3]}};
}
__device__ __forceinline__ D4 operator/(D4 a, D4 b)
{
    const float iv = 1.0f / b.v, iv2 = iv * iv;
    return D4{a.v * iv,
              {(a.d[0] * b.v - a.v * b.d[0]) * iv2, (a.d[1] * b.v - a.v * b.d[1]) * iv2,
               (a.d[2] * b.v - a.v * b.d[2]) * iv2, (a.d[3] * b.v - a.v * b.d[3]) * iv2}};
}

// Ghost delta D_q(m) = geq(rho_B, u_B) - geq(rho_I, u_I) of the open boundary
// (06:684-835) as a function of the interior moments m = (rho', J), with
// geq(q; rho', r, u) = w_q (rho' + r (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)) in
// deviation units with scale 1.  The adjoint needs only sum_q lam_q D_q(m)
// and its gradient in m, which go through the weighted moments of lam:
//   A0 = sum w lam, A1 = sum w lam c, A2 = sum w lam c c^T (xx yy zz xy xz yz),
//   A0 rho' + r (3 A1.u + 4.5 u^T A2 u - 1.5 u^2 A0).
struct LamMoments
{
    float a0, a1[3], a2[6];
};
__device__ __forceinline__ D4 lam_geq4(const LamMoments& A, D4 rho, D4 r, D4 ux, D4 uy, D4 uz)
{
    const D4 cu = A.a1[0] * ux + A.a1[1] * uy + A.a1[2] * uz;
    const D4 xx = ux * ux, yy = uy * uy, zz = uz * uz;
    const D4 quad = A.a2[0] * xx + A.a2[1] * yy + A.a2[2] * zz +
                    2.0f * (A.a2[3] * (ux * uy) + A.a2[4] * (ux * uz) + A.a2[5] * (uy * uz));
    return A.a0 * rho + r * (3.0f * cu + 4.5f * quad - 1.5f * (A.a0 * (xx + yy + zz)));
}

// sum_q lam_q D_q(m), one scalar whose four derivatives are J_ghost^T lam.
__device__ __forceinline__ D4 nscbc_lam4(const LamMoments& A, D4 rho, D4 jx, D4 jy, D4 jz, int axis, int side)
{
    const D4 rI = dc(1.0f) + rho;
    const D4 ux = jx / rI, uy = jy / rI, uz = jz / rI;
    const float cs = (float)kCs, cs2 = (float)kCs2;
    const D4 pI = cs2 * rho;
    const D4 un = axis == 0 ? ux : (axis == 1 ? uy : uz);
    D4 unB, pB;
    if (side == 0)
    {
        const D4 Wm = un - (1.0f / cs) * pI;
        unB = 0.5f * Wm;
        pB = (-0.5f * cs) * Wm;
    }
    else
    {
        const D4 Wp = un + (1.0f / cs) * pI;
        unB = 0.5f * Wp;
        pB = (0.5f * cs) * Wp;
    }
    const D4 rhoB = (1.0f / cs2) * pB;
    const D4 rB = dc(1.0f) + rhoB;
    const D4 bx = axis == 0 ? unB : ux, by = axis == 1 ? unB : uy, bz = axis == 2 ? unB : uz;
    return lam_geq4(A, rhoB, rB, bx, by, bz) - lam_geq4(A, rho, rI, ux, uy, uz);
}

// ---------------------------------------------------------------- kernels

// J_ghost^T of every open-face ghost cell: lamHt at the ghost (what the
// interior cells pulled from it) mapped onto the interior cell it was built
// from.  One thread per face cell, the face (AXIS, SIDE) a template argument:
// only the 5 directions pointing into the interior carry adjoint values.
template <int AXIS, int SIDE>
__host__ __device__ constexpr bool inward(int q)
{
    return (AXIS == 0 ? ex(q) : AXIS == 1 ? ey(q) : ez(q)) == (SIDE ? -1 : 1);
}

template <int AXIS, int SIDE>
__device__ __forceinline__ void adj_ghost_cell(const AdjGhostArgs& a, const GhostFace& F, long long t, int lt)
{
    const int v = lt / F.nu, u = lt - v * F.nu;
    const Layout& L = a.L;
    // ghost cell g (the forward ghost kernel's enumeration of the face)
    int gi, gj, gk;
    if (AXIS == 0)
    {
        gi = SIDE ? L.nx + 1 : 0;
        gj = 1 + u;
        gk = 1 + v;
    }
    else if (AXIS == 1)
    {
        gi = 1 + u;
        gj = SIDE ? L.ny + 1 : 0;
        gk = 1 + v;
    }
    else
    {
        gi = 1 + u;
        gj = 1 + v;
        gk = SIDE ? L.nz + 1 : 0;
    }
    // lamHt at the ghost: what the interior cells y = g + e_q pulled from it,
    // nothing when the ghost cell is SOLID (they bounced back instead).  Bit q
    // of y's links word is that solidity for every such y, so one word is
    // read: that of the interior neighbour along the inward normal.
    const int qn = 1 + 2 * AXIS + SIDE;
    const int ni = AXIS == 0 ? 1 - 2 * SIDE : 0, nj = AXIS == 1 ? 1 - 2 * SIDE : 0,
              nk = AXIS == 2 ? 1 - 2 * SIDE : 0;
    // (loaded beside the adjoint values, not before them: one memory round trip)
    const uint32_t lkn = __ldg(a.links + L.cell(gi + ni, gj + nj, gk + nk));
    float lh[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int di = gi + ex(q), dj = gj + ey(q), dk = gk + ez(q);
        // only the directions pointing into the interior reach an interior cell
        lh[q] = inward<AXIS, SIDE>(q) && interior(L, di, dj, dk) ? __ldg(a.lam_in + L.elem(q, di, dj, dk)) : 0.f;
    }
    if ((lkn >> qn) & 1u)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (inward<AXIS, SIDE>(q)) lh[q] = 0.f;
    }
    // moments of the interior cell the ghost was built from
    const float4 m = __ldg(a.face_mom + t);
    // J_ghost^T lam = grad_m sum_q lam_q D_q(m), through lam's weighted moments
    LamMoments A{};
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        if (!inward<AXIS, SIDE>(q)) continue;   // lh[q] = 0
        const float wl = wf(q) * lh[q];
        A.a0 += wl;
        if (ex(q)) A.a1[0] += ex(q) * wl;
        if (ey(q)) A.a1[1] += ey(q) * wl;
        if (ez(q)) A.a1[2] += ez(q) * wl;
        if (ex(q)) A.a2[0] += wl;
        if (ey(q)) A.a2[1] += wl;
        if (ez(q)) A.a2[2] += wl;
        if (ex(q) * ey(q)) A.a2[3] += ex(q) * ey(q) * wl;
        if (ex(q) * ez(q)) A.a2[4] += ex(q) * ez(q) * wl;
        if (ey(q) * ez(q)) A.a2[5] += ey(q) * ez(q) * wl;
    }
    const D4 S = nscbc_lam4(A, D4{m.x, {1.f, 0.f, 0.f, 0.f}}, D4{m.y, {0.f, 1.f, 0.f, 0.f}},
                            D4{m.z, {0.f, 0.f, 1.f, 0.f}}, D4{m.w, {0.f, 0.f, 0.f, 1.f}}, AXIS, SIDE);
    const float vk[4] = {S.d[0], S.d[1], S.d[2], S.d[3]};
    const long long n = (long long)F.nu * F.nv, off = a.gadj_off[AXIS * 2 + SIDE];
#pragma unroll
    for (int p = 0; p < Q; ++p)
        a.gadj[off + (long long)p * n + lt] = lh[p] + vk[0] + ex(p) * vk[1] + ey(p) * vk[2] + ez(p) * vk[3];
}

__global__ void __launch_bounds__(128) k_adj_ghost(AdjGhostArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ga.total) return;
    int fi = 0;
    while (fi + 1 < a.ga.nfaces && t >= a.ga.face[fi + 1].first) ++fi;
    const GhostFace F = a.ga.face[fi];
    const int lt = (int)(t - F.first);
    switch (F.axis * 2 + F.side)
    {
    case 0: adj_ghost_cell<0, 0>(a, F, t, lt); break;
    case 1: adj_ghost_cell<0, 1>(a, F, t, lt); break;
    case 2: adj_ghost_cell<1, 0>(a, F, t, lt); break;
    case 3: adj_ghost_cell<1, 1>(a, F, t, lt); break;
    case 4: adj_ghost_cell<2, 0>(a, F, t, lt); break;
    default: adj_ghost_cell<2, 1>(a, F, t, lt); break;
    }
}

__device__ __forceinline__ uint32_t near_bits(const StepArgs& a, const Layout& L, int col, int j, int k)
{
    return a.near[((long long)k * (L.ny + 2) + j) * L.words_per_row + (col >> 5)] >> (col & 31);
}

__device__ __forceinline__ float2 ldg2(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }

// 12-bit float (PairMoments) -> float: it is FP16 with the 4 lowest mantissa bits zero
__device__ __forceinline__ float from_f12(unsigned t)
{
    return __half2float(__ushort_as_half((unsigned short)((((t >> 11) & 1u) << 15) | ((t & 0x7ffu) << 4))));
}

// (rho', jx, jy, jz) of the two cells of a PairMoments record
__device__ __forceinline__ void unpack_moments(const PairMoments& p, float4& m0, float4& m1)
{
    const unsigned w0 = p.w[0], w1 = p.w[1], w2 = p.w[2];
    m0 = make_float4(from_f12(w0 & 0xfffu), from_f12((w0 >> 12) & 0xfffu), from_f12((w0 >> 24) | ((w1 & 0xfu) << 8)),
                     from_f12((w1 >> 4) & 0xfffu));
    m1 = make_float4(from_f12((w1 >> 16) & 0xfffu), from_f12((w1 >> 28) | ((w2 & 0xffu) << 4)),
                     from_f12((w2 >> 8) & 0xfffu), from_f12(w2 >> 20));
}

// packed FP32x2 arithmetic (sm_100): both cells of a pair in one instruction
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }
// c_q . (x, y, z) for a pair head q (components 0 or +-1)
__device__ __forceinline__ float2 cdot(int q, float2 x, float2 y, float2 z)
{
    float2 r = f2(0.f);
    bool any = false;
    if (ex(q)) r = ex(q) > 0 ? x : mul2(x, f2(-1.f)), any = true;
    if (ey(q)) r = any ? (ey(q) > 0 ? add2(r, y) : sub2(r, y)) : (ey(q) > 0 ? y : mul2(y, f2(-1.f))), any = true;
    if (ez(q)) r = any ? (ez(q) > 0 ? add2(r, z) : sub2(r, z)) : (ez(q) > 0 ? z : mul2(z, f2(-1.f)));
    return r;
}

// Pair (c0 + d, c0 + 1 + d), d = -1, 0, +1, of the row whose element of
// column c0 is at `row` (block-interleaved layout, 32-cell blocks): one
// aligned float2 per lane; the +-1 shift takes the neighbour element from the
// adjacent lane and, at the warp edge, from the adjacent block (the same
// scheme as the forward step).  Every lane of the warp must call it.
// pair load of buffer `base` (total elements); the bounds-checked build tests the index first
__device__ __forceinline__ float2 ldg2c(const float* p, const float* base, long long total)
{
    return LBM_IN(kChkAdjLoad, p - base, total - 1) ? ldg2(p) : make_float2(0.f, 0.f);
}

template <int D>
__device__ __forceinline__ float2 shifted_pair(const float* row, int lane, const float* base, long long total)
{
    constexpr int BC = 32, BE = 19 * BC;
    const float2 cur = ldg2c(row, base, total);
    if (D == 0) return cur;
    if (D < 0)
    {
        float prev = __shfl_up_sync(kFull, cur.y, 1);
        if (lane == 0) prev = ldg2c(row - BE + (BC - 2), base, total).y;
        return make_float2(prev, cur.x);
    }
    float next = __shfl_down_sync(kFull, cur.x, 1);
    if (lane == 31) next = ldg2c(row + BE - (BC - 2), base, total).x;
    return make_float2(cur.y, next);
}

// lamF^{s-1} = J_C(F^{s-1})^T lamH^s for two x-adjacent cells per thread.
// With F the pulled populations (only their stored moments are read),
// rho' = sum F, J = sum c F, r = 1 + rho':
//   (J_C^T l)_p = a l_p + b (A + c_p . B)
//   A = sum_q l_q w_q (1 - (4.5 (c_q.J)^2 - 1.5 J^2) / r^2)
//   B = sum_q l_q w_q (3 c_q + (9 (c_q.J) c_q - 3 J) / r)
// a = (1 - sigma)(1 - omega), b = (1 - sigma) omega; SOLID cells copy.
// lamH (gather of lamF^s with the bounce-back terms and, at the open faces,
// the ghost-adjoint terms) stays in registers for the output.
// L2 prefetch, one CTA's share, as two bulk prefetches issued by its first
// thread: the columns of this CTA in the storage row first read `dist` rows
// from now (a row of the adjoint layout is contiguous: its blocks' 19 lines
// back to back; rows are first read by the target row one plane and one row
// before them), and the moment records of the target row `dist` rows ahead.
template <int CELLS>
__device__ __forceinline__ void adj_prefetch_rows(const AdjStepArgs& a, int j, int k, int col0)
{
    if (threadIdx.x != 0) return;
    const Layout& L = a.L;
    const long long rows_total = (long long)(L.nz + 2) * (L.ny + 2);
    const long long R = (long long)k * (L.ny + 2) + j + (L.ny + 2) + 1 + a.prefetch_rows;
    if (R < rows_total)
    {
        constexpr int kBlocks = (CELLS + 31) / 32;
        const int b0 = col0 >> 5, nbk = min(kBlocks, L.nb - b0);
        const float* p = a.lam_in + kFrontElems + R * L.row_stride + (long long)b0 * (19 * 32);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(nbk * 19 * 128) : "memory");
    }
    const long long r = (long long)(k - 1) * L.ny + (j - 1) + a.prefetch_rows;
    if (r < (long long)L.ny * L.nz)
    {
        const long long npr = (L.nx + 1) >> 1;
        const long long first = r * npr + (col0 >> 1), last = min(first + CELLS / 2, (r + 1) * npr);
        const long long total = npr * L.ny * L.nz * (long long)sizeof(PairMoments);
        const long long lo = first * (long long)sizeof(PairMoments) & ~15LL;
        const long long hi = min((last * (long long)sizeof(PairMoments) + 15) & ~15LL, total & ~15LL);
        if (hi > lo)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<const char*>(a.mom_prev) + lo),
                         "r"((unsigned)(hi - lo)) : "memory");
    }
}

template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_adj_step(AdjStepArgs a)
{
    constexpr int BC = 32;
    const Layout& L = a.L;
    const int lane = threadIdx.x & 31;
    const int c0r = 2 * (blockIdx.x * BLOCK + threadIdx.x);
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~1);   // inactive lanes shadow a valid pair
    const int j = blockIdx.y + 1, k = blockIdx.z + 1;
    const long long e0 = L.elem(0, c0 + 1, j, k);
    const long long rs = L.row_stride, ps = L.plane_stride;
    if (a.prefetch_rows > 0) adj_prefetch_rows<2 * BLOCK>(a, j, k, 2 * BLOCK * blockIdx.x);

    uint32_t lk0 = 0, lk1 = 0;
    if (active)
    {
        const uint32_t b = near_bits(a.sa, L, c0, j, k) & 3u;
        const long long cl = L.cell(c0 + 1, j, k);
        if (b & 1u) lk0 = a.sa.links[cl];
        if (b & 2u) lk1 = a.sa.links[cl + 1];
    }
    const bool any_link = __any_sync(kFull, (lk0 | lk1) != 0u);
    const bool xlo = c0 == 0;                 // first cell at i = 1
    const bool xhi0 = c0 == L.nx - 1;         // first cell at i = nx (nx odd)
    const bool xhi1 = c0 + 1 == L.nx - 1;     // second cell at i = nx
    const bool has1 = c0 + 1 < L.nx;

    // ---- moments of F^{s-1}, stored by the forward recomputation
    float2 rho, jx, jy, jz;
    {
        const long long pi = ((long long)(k - 1) * L.ny + (j - 1)) * ((L.nx + 1) >> 1) + (c0 >> 1);
        [[maybe_unused]] const long long npair = (long long)((L.nx + 1) >> 1) * L.ny * L.nz;
        PairMoments pm{{0u, 0u, 0u}};
        if (LBM_IN(kChkAdjLoad, pi, npair)) pm = a.mom_prev[pi];
        float4 m0, m1;
        unpack_moments(pm, m0, m1);
        if (!has1) m1 = m0;
        rho = make_float2(m0.x, m1.x);
        jx = make_float2(m0.y, m1.y);
        jy = make_float2(m0.z, m1.z);
        jz = make_float2(m0.w, m1.w);
    }

    // ---- lamH^s of the pair: transposed pull of lamF^s.  Cell y + e_q pulled
    // direction q from y; rows outside the interior pulled nothing, and there
    // the adjoint buffers hold 0 (their halo rows are never written), so the
    // loads need no row test.
    const bool solid0 = (lk0 & kSolidSelfBit) != 0u, solid1 = (lk1 & kSolidSelfBit) != 0u;
    float2 lg[Q];
    {
        const float* own = a.lam_in + e0;
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const float* row = own + (ey(q) * rs + ez(q) * ps) + q * BC;
            if (ex(q) == 0) lg[q] = shifted_pair<0>(row, lane, a.lam_in, L.total);
            else if (ex(q) > 0) lg[q] = shifted_pair<1>(row, lane, a.lam_in, L.total);
            else lg[q] = shifted_pair<-1>(row, lane, a.lam_in, L.total);
        }
        // columns outside the interior pulled nothing (and the neighbour block
        // read there may belong to another row)
        if (xlo | xhi0 | xhi1)
        {
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (ex(q) < 0 && xlo) lg[q].x = 0.f;
                if (ex(q) > 0 && xhi0) lg[q].x = 0.f;
                if (ex(q) > 0 && xhi1) lg[q].y = 0.f;
            }
        }
        if (any_link)
        {
            // a SOLID cell is pulled from by nobody (its neighbours bounce back) ...
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (solid0) lg[q].x = 0.f;
                if (solid1) lg[q].y = 0.f;
            }
            // ... and y pulled direction inv(q) from itself when y + e_q is SOLID
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (((lk0 | lk1) >> inv(q)) & 1u)
                {
                    const float2 o = ldg2c(own + inv(q) * BC, a.lam_in, L.total);
                    if ((lk0 >> inv(q)) & 1u) lg[q].x += o.x;
                    if ((lk1 >> inv(q)) & 1u) lg[q].y += o.y;
                }
            }
        }
    }
    if (!active) return;

    // ---- ghost-adjoint terms of the open faces the pair borders: lamH of a
    // face cell also holds what the ghost fill took from it (k_adj_ghost),
    // and J_C^T is applied to the sum.  y and z faces are whole rows (the
    // branch is uniform across the CTA); the x faces touch the row ends.
    {
        const bool yz = (j == 1 && a.gadj_off[2] >= 0) || (j == L.ny && a.gadj_off[3] >= 0) ||
                        (k == 1 && a.gadj_off[4] >= 0) || (k == L.nz && a.gadj_off[5] >= 0);
        if (yz)
        {
#pragma unroll
            for (int f = 2; f < 6; ++f)
            {
                const bool on = f == 2 ? j == 1 : f == 3 ? j == L.ny : f == 4 ? k == 1 : k == L.nz;
                if (!on || a.gadj_off[f] < 0) continue;
                const int axis = f / 2;
                const long long n = face_cells(L, axis);
                const float* g = a.gadj + a.gadj_off[f] + face_cell(L, axis, c0 + 1, j, k);
#pragma unroll
                for (int q = 0; q < Q; ++q)
                {
                    lg[q].x += __ldg(g + q * n);
                    if (has1) lg[q].y += __ldg(g + q * n + 1);
                }
            }
        }
        if (xlo | xhi0 | xhi1)
        {
            const long long n = face_cells(L, 0), c = face_cell(L, 0, 1, j, k);
#pragma unroll
            for (int f = 0; f < 2; ++f)
            {
                if (a.gadj_off[f] < 0) continue;
                const bool to0 = f == 0 ? xlo : xhi0, to1 = f == 1 && xhi1;
                if (!(to0 | to1)) continue;
                const float* g = a.gadj + a.gadj_off[f] + c;
#pragma unroll
                for (int q = 0; q < Q; ++q)
                {
                    const float v = __ldg(g + q * n);
                    if (to0) lg[q].x += v;
                    if (to1) lg[q].y += v;
                }
            }
        }
    }

    // ---- J_C^T, packed FP32x2 over the pair, directions taken with their
    // opposites (c_qb = -c_q, so both share c.J)
    const float syz = fmaxf(a.sa.sig_y[j - 1], a.sa.sig_z[k - 1]);
    const float sg0 = fmaxf(a.sa.sig_x[c0], syz), sg1 = fmaxf(has1 ? a.sa.sig_x[c0 + 1] : 0.f, syz);
    float2 ca = make_float2((1.0f - sg0) * (1.0f - a.sa.omega), (1.0f - sg1) * (1.0f - a.sa.omega));
    float2 cb = make_float2((1.0f - sg0) * a.sa.omega, (1.0f - sg1) * a.sa.omega);
    if (solid0) ca.x = 1.0f, cb.x = 0.0f;
    if (solid1) ca.y = 1.0f, cb.y = 0.0f;
    if (!has1) ca.y = 0.0f, cb.y = 0.0f;   // no second cell: keep the padding column at 0
    float2 r = add2(rho, f2(1.0f));
    if (r.x <= 0.f) r.x = 1e-12f;
    if (r.y <= 0.f) r.y = 1e-12f;
    const float2 ir = make_float2(1.0f / r.x, 1.0f / r.y);
    const float2 ir2 = mul2(ir, ir);
    const float2 j2 = fma2(jz, jz, fma2(jy, jy, mul2(jx, jx)));
    // s0 = sum w l, s1 = sum w l (c.J)^2, v = sum w l c, u = sum w l (c.J) c
    float2 s0 = mul2(f2(wf(0)), lg[0]), s1 = f2(0.f);
    float2 vx = f2(0.f), vy = vx, vz = vx, ux = vx, uy = vx, uz = vx;
#pragma unroll
    for (int p = 0; p < 9; ++p)
    {
        const int q = pair_head(p), qb = inv(q);
        const float2 cj = cdot(q, jx, jy, jz);
        const float2 sp = mul2(f2(wf(q)), add2(lg[q], lg[qb]));
        const float2 dm = mul2(f2(wf(q)), sub2(lg[q], lg[qb]));
        const float2 t = mul2(sp, cj);
        s0 = add2(s0, sp);
        s1 = fma2(t, cj, s1);
        if (ex(q)) vx = ex(q) > 0 ? add2(vx, dm) : sub2(vx, dm), ux = ex(q) > 0 ? add2(ux, t) : sub2(ux, t);
        if (ey(q)) vy = ey(q) > 0 ? add2(vy, dm) : sub2(vy, dm), uy = ey(q) > 0 ? add2(uy, t) : sub2(uy, t);
        if (ez(q)) vz = ez(q) > 0 ? add2(vz, dm) : sub2(vz, dm), uz = ez(q) > 0 ? add2(uz, t) : sub2(uz, t);
    }
    // A = s0 (1 + 1.5 J^2 / r^2) - 4.5 s1 / r^2;  B = 3 v + (9 u - 3 J s0) / r
    const float2 A = sub2(mul2(s0, fma2(mul2(j2, ir2), f2(1.5f), f2(1.0f))), mul2(mul2(s1, ir2), f2(4.5f)));
    const float2 Bx = fma2(vx, f2(3.0f), mul2(sub2(mul2(ux, f2(9.0f)), mul2(mul2(jx, s0), f2(3.0f))), ir));
    const float2 By = fma2(vy, f2(3.0f), mul2(sub2(mul2(uy, f2(9.0f)), mul2(mul2(jy, s0), f2(3.0f))), ir));
    const float2 Bz = fma2(vz, f2(3.0f), mul2(sub2(mul2(uz, f2(9.0f)), mul2(mul2(jz, s0), f2(3.0f))), ir));
    float* out = a.lam_out + e0;
    if (!LBM_IN(kChkAdjStore, e0 + 18 * BC + 1, L.total)) return;
    const float2 cbA = mul2(cb, A);
    *reinterpret_cast<float2*>(out) = fma2(ca, lg[0], cbA);
#pragma unroll
    for (int p = 0; p < 9; ++p)
    {
        const int q = pair_head(p), qb = inv(q);
        const float2 cB = mul2(cb, cdot(q, Bx, By, Bz));
        *reinterpret_cast<float2*>(out + q * BC) = fma2(ca, lg[q], add2(cbA, cB));
        *reinterpret_cast<float2*>(out + qb * BC) = fma2(ca, lg[qb], sub2(cbA, cB));
    }
}

// Residual of each probe enters the adjoint of every population it summed.
__global__ void k_adj_probe(float* __restrict__ lam, AdjProbeArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int i = a.ijk[3 * p], j = a.ijk[3 * p + 1], k = a.ijk[3 * p + 2];
    const float r = (float)a.resid[p];
    if (i < 0 || r == 0.f) return;
#pragma unroll
    for (int q = 0; q < Q; ++q) atomicAdd(&lam[a.L.elem(q, i, j, k)], r);
}

// Source gradient of one step: Lam_c = sum_q w_q lamH^s[q](c) over the
// injection cells; out = (sum_c w_hat_c Lam_c, sum_c dw_hat_c/dpos Lam_c),
// reduced in FP64.
__global__ void __launch_bounds__(128) k_adj_source(AdjSourceArgs a)
{
    __shared__ double red[4][4];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const AdjSourceCell* cells = a.cells + (long long)a.step * a.ncell;
    for (int c = threadIdx.x; c < a.ncell; c += blockDim.x)
    {
        const AdjSourceCell e = cells[c];
        if (e.i < 0) continue;
        float lg[Q];
        gather_lam(a.L, a.links, a.lam_in, a.gadj, a.gadj_off, e.i, e.j, e.k, lg);
        double lam = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) lam += wd(q) * (double)lg[q];
        acc[0] += e.what * lam;
        acc[1] += e.dwhat[0] * lam;
        acc[2] += e.dwhat[1] * lam;
        acc[3] += e.dwhat[2] * lam;
    }
#pragma unroll
    for (int m = 0; m < 4; ++m)
        for (int o = 16; o > 0; o >>= 1) acc[m] += __shfl_xor_sync(kFull, acc[m], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int m = 0; m < 4; ++m) red[warp][m] = acc[m];
    __syncthreads();
    if (threadIdx.x < 4)
    {
        double t = 0.0;
        for (int w = 0; w < 4; ++w) t += red[w][threadIdx.x];
        a.out[4LL * a.step + threadIdx.x] = t;
    }
}

}  // namespace

cudaError_t launch_adj_ghost(const AdjGhostArgs& a, cudaStream_t stream)
{
    if (a.ga.total <= 0) return cudaSuccess;
    k_adj_ghost<<<(unsigned)((a.ga.total + 127) / 128), 128, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_step(const AdjStepArgs& a, cudaStream_t stream)
{
    // 80 registers, no spills, 24 warps per SM (a 3000-step gradient on the
    // 256x256x128 patch: 1578 ms against 1587 ms at 96 registers); rows of up
    // to 128 columns take 64-thread blocks, so no warp idles
    const int block = a.L.nx <= 128 ? 64 : 128;
    const dim3 g((unsigned)((a.L.nx + 2 * block - 1) / (2 * block)), (unsigned)a.L.ny, (unsigned)a.L.nz);
    if (block == 64) k_adj_step<64, 10><<<g, 64, 0, stream>>>(a);
    else k_adj_step<128, 6><<<g, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_source(const AdjSourceArgs& a, cudaStream_t stream)
{
    k_adj_source<<<1, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_probe(float* lam, const AdjProbeArgs& a, cudaStream_t stream)
{
    if (a.n <= 0) return cudaSuccess;
    k_adj_probe<<<(a.n + 127) / 128, 128, 0, stream>>>(lam, a);
    return cudaGetLastError();
}

cudaError_t check_read_adjoint(check::Status* out) { return check::read_and_clear(out); }

}  // namespace lbm
