// sm_100a kernels of the D3Q19 acoustic step (family-B semantics of
// 06_transient_localization_dx1.cpp).  Storage is FP32 or FP16 deviations from
// rest equilibrium (see device.hpp for the HBM layout); arithmetic is FP32,
// with FP64 for the source-weight reduction and the probe accumulators.
#include <cuda_fp16.h>

#include <cmath>
#include <cstdint>

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

// Two x-adjacent cells as one aligned vector: float2 (8 B) or half2 (4 B).
// `V` is the raw register form that is shuffled between lanes.
template <typename S>
struct Pair;

template <>
struct Pair<float>
{
    using V = float2;
    static __device__ __forceinline__ V ld(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
    static __device__ __forceinline__ void st(float* p, float a, float b)
    {
        *reinterpret_cast<float2*>(p) = make_float2(a, b);
    }
    static __device__ __forceinline__ float lo(V v) { return v.x; }
    static __device__ __forceinline__ float hi(V v) { return v.y; }
    static __device__ __forceinline__ V up(V v)   // element 1 of lane - 1 (element 0 unused)
    {
        return make_float2(v.x, __shfl_up_sync(kFull, v.y, 1));
    }
    static __device__ __forceinline__ V down(V v)   // element 0 of lane + 1 (element 1 unused)
    {
        return make_float2(__shfl_down_sync(kFull, v.x, 1), v.y);
    }
    // cells (c-1, c) from prev = (c-2, c-1) and cur = (c, c+1)
    static __device__ __forceinline__ void left(V prev, V cur, float& a, float& b)
    {
        a = prev.y;
        b = cur.x;
    }
    // cells (c+1, c+2) from cur = (c, c+1) and next = (c+2, c+3)
    static __device__ __forceinline__ void right(V cur, V next, float& a, float& b)
    {
        a = cur.y;
        b = next.x;
    }
};

template <>
struct Pair<__half>
{
    using V = unsigned;
    static __device__ __forceinline__ V ld(const __half* p) { return __ldg(reinterpret_cast<const unsigned*>(p)); }
    static __device__ __forceinline__ void st(__half* p, float a, float b)
    {
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
    }
    static __device__ __forceinline__ float2 f2(unsigned u)
    {
        __half2 h;
        *reinterpret_cast<unsigned*>(&h) = u;
        return __half22float2(h);
    }
    static __device__ __forceinline__ float lo(V v) { return f2(v).x; }
    static __device__ __forceinline__ float hi(V v) { return f2(v).y; }
    static __device__ __forceinline__ V up(V v) { return __shfl_up_sync(kFull, v, 1); }
    static __device__ __forceinline__ V down(V v) { return __shfl_down_sync(kFull, v, 1); }
    static __device__ __forceinline__ void left(V prev, V cur, float& a, float& b)
    {
        const float2 r = f2(__byte_perm(prev, cur, 0x5432));
        a = r.x;
        b = r.y;
    }
    static __device__ __forceinline__ void right(V cur, V next, float& a, float& b)
    {
        const float2 r = f2(__byte_perm(cur, next, 0x5432));
        a = r.x;
        b = r.y;
    }
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
// Fused pull-stream + halfway bounce-back + BGK + sponge (06:906-972), two
// x-adjacent cells per thread.  Each direction is read as one aligned vector
// per thread; the +-1 x shift of directions with ex != 0 takes the missing
// neighbour element from the adjacent lane (warp shuffle) and, at the warp
// edge, from one extra aligned load.  SOLID cells copy the pulled values
// (06:933-938).  Cells next to the x faces take their x-halo sources from
// the x-face ghosts and export their results for the next ghost fill.
template <typename S>
__global__ void __launch_bounds__(128) k_step(const S* __restrict__ fin, S* __restrict__ fout, Layout L,
                                              StepArgs a, float inv_scale)
{
    using P = Pair<S>;
    const int lane = threadIdx.x & 31;
    const int c0r = 2 * (blockIdx.x * blockDim.x + threadIdx.x);   // first column of the pair
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~1);              // inactive lanes shadow a valid pair
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    const long long cell = (long long)k * L.plane + (long long)j * L.pitch + c0;

    uint32_t lk0 = 0, lk1 = 0;
    if (active)
    {
        const uint32_t nw = near_word(a, L, c0, j, k);
        const uint32_t b = (nw >> (c0 & 31)) & 3u;
        if (b & 1u) lk0 = a.links[cell];
        if (b & 2u) lk1 = a.links[cell + 1];
    }
    const bool any_link = __any_sync(kFull, (lk0 | lk1) != 0u);

    float G0[Q], G1[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const S* src = fin + (long long)q * L.pop_stride + cell - row_off(q, L);
        const typename P::V cur = P::ld(src);
        if (ex(q) == 0)
        {
            G0[q] = P::lo(cur);
            G1[q] = P::hi(cur);
        }
        else if (ex(q) > 0)
        {
            typename P::V prev = P::up(cur);
            if (lane == 0) prev = P::ld(src - 2);
            P::left(prev, cur, G0[q], G1[q]);
        }
        else
        {
            typename P::V next = P::down(cur);
            if (lane == 31) next = P::ld(src + 2);
            P::right(cur, next, G0[q], G1[q]);
        }
    }
    if (any_link)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (((lk0 | lk1) >> q) & 1u)
            {
                const typename P::V own = P::ld(fin + (long long)inv(q) * L.pop_stride + cell);
                if ((lk0 >> q) & 1u) G0[q] = P::lo(own);
                if ((lk1 >> q) & 1u) G1[q] = P::hi(own);
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
            if (ex(q) > 0 && xlo && !((lk0 >> q) & 1u)) G0[q] = g;
            if (ex(q) < 0 && xhi0 && !((lk0 >> q) & 1u)) G0[q] = g;
            if (ex(q) < 0 && xhi1 && !((lk1 >> q) & 1u)) G1[q] = g;
        }
    }
    if (!active) return;

    const float syz = fmaxf(a.sig_y[j - 1], a.sig_z[k - 1]);
    const float s0 = fmaxf(a.sig_x[c0], syz);
    const float s1 = fmaxf(c0 + 1 < L.nx ? a.sig_x[c0 + 1] : 0.f, syz);
    if (!(lk0 & kSolidSelfBit)) collide(G0, inv_scale, a.omega, s0);
    if (!(lk1 & kSolidSelfBit)) collide(G1, inv_scale, a.omega, s1);

#pragma unroll
    for (int q = 0; q < Q; ++q) P::st(fout + (long long)q * L.pop_stride + cell, G0[q], G1[q]);

    if (xlo | xhi0 | xhi1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (xlo) a.xf.xexp[a.xf.exp_index(0, q, j, k, L.ny, L.nz)] = Io<S>::rnd(G0[q]);
            if (xhi0) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = Io<S>::rnd(G0[q]);
            if (xhi1) a.xf.xexp[a.xf.exp_index(1, q, j, k, L.ny, L.nz)] = Io<S>::rnd(G1[q]);
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
dim3 pair_grid(const Layout& L)
{
    return dim3((unsigned)(((L.nx + 1) / 2 + 127) / 128), (unsigned)L.ny, (unsigned)L.nz);
}

}  // namespace

cudaError_t launch_build_links(const uint8_t* mask_ref, uint32_t* links, uint32_t* near, const Layout& L,
                               cudaStream_t stream)
{
    k_build_links<<<row_grid(L), 128, 0, stream>>>(mask_ref, links, near, L);
    return cudaGetLastError();
}

cudaError_t launch_step(int storage, const void* fin, void* fout, const Layout& L, const StepArgs& a,
                        float scale, cudaStream_t stream)
{
    if (storage == 0)
        k_step<float><<<pair_grid(L), 128, 0, stream>>>((const float*)fin, (float*)fout, L, a, 1.0f);
    else
        k_step<__half><<<pair_grid(L), 128, 0, stream>>>((const __half*)fin, (__half*)fout, L, a, 1.0f / scale);
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
