// Reverse-time adjoint kernels of the fused D3Q19 step (FP32 storage, scale 1).
// See adjoint.hpp for the recursion.  Every kernel is a gather: the transposed
// pull-stream reads the adjoint populations of the neighbours that pulled
// from a cell, mirroring the forward pull.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "adjoint.hpp"
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

__device__ __forceinline__ D4 dot_c4(int q, D4 x, D4 y, D4 z)
{
    D4 r = dc(0.f);
    if (ex(q) > 0) r = r + x;
    if (ex(q) < 0) r = r - x;
    if (ey(q) > 0) r = r + y;
    if (ey(q) < 0) r = r - y;
    if (ez(q) > 0) r = r + z;
    if (ez(q) < 0) r = r - z;
    return r;
}

// geq(rho', r, u) - w_q rho-free part, in deviation units with scale 1:
//   w_q (rho' + r (3 c.u + 4.5 (c.u)^2 - 1.5 u^2))
__device__ __forceinline__ D4 geq4(int q, D4 rho, D4 r, D4 ux, D4 uy, D4 uz)
{
    const D4 cu = dot_c4(q, ux, uy, uz);
    const D4 u2 = ux * ux + uy * uy + uz * uz;
    return wf(q) * (rho + r * (3.0f * cu + 4.5f * (cu * cu) - 1.5f * u2));
}

// Ghost delta D_q(m) = geq(rho_B, u_B) - geq(rho_I, u_I) of the open boundary
// (06:684-835), as a function of the interior moments m = (rho', J).
__device__ __forceinline__ void nscbc_delta4(D4 rho, D4 jx, D4 jy, D4 jz, int axis, int side, D4 (&D)[Q])
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
#pragma unroll
    for (int q = 0; q < Q; ++q) D[q] = geq4(q, rhoB, rB, bx, by, bz) - geq4(q, rho, rI, ux, uy, uz);
}

// ---------------------------------------------------------------- kernels

// J_ghost^T of every open-face ghost cell: lamHt at the ghost (what the
// interior cells pulled from it) mapped onto the interior cell it was built
// from.  One thread per face cell.
__global__ void __launch_bounds__(128) k_adj_ghost(AdjGhostArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ga.total) return;
    int fi = 0;
    while (fi + 1 < a.ga.nfaces && t >= a.ga.face[fi + 1].first) ++fi;
    const GhostFace F = a.ga.face[fi];
    const long long lt = t - F.first;
    const int u = (int)(lt % F.nu), v = (int)(lt / F.nu);
    const Layout& L = a.L;
    int ci, cj, ck, gi, gj, gk;
    if (F.axis == 0)
    {
        cj = gj = 1 + u;
        ck = gk = 1 + v;
        ci = F.side ? L.nx : 1;
        gi = F.side ? L.nx + 1 : 0;
    }
    else if (F.axis == 1)
    {
        ci = gi = 1 + u;
        ck = gk = 1 + v;
        cj = F.side ? L.ny : 1;
        gj = F.side ? L.ny + 1 : 0;
    }
    else
    {
        ci = gi = 1 + u;
        cj = gj = 1 + v;
        ck = F.side ? L.nz : 1;
        gk = F.side ? L.nz + 1 : 0;
    }
    // lamHt at the ghost: what the interior cells y = g + e_q pulled from it
    // (none when y bounced back, i.e. when the ghost cell is SOLID)
    float lh[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int di = gi + ex(q), dj = gj + ey(q), dk = gk + ez(q);
        float v = 0.f;
        if (interior(L, di, dj, dk) && !((a.links[L.cell(di, dj, dk)] >> q) & 1u))
            v = a.lam_in[L.elem(q, di, dj, dk)];
        lh[q] = v;
    }
    // moments of the interior cell the ghost was built from
    float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const float g = a.fwd[L.elem(q, ci, cj, ck)];
        rho += g;
        if (ex(q) > 0) jx += g;
        if (ex(q) < 0) jx -= g;
        if (ey(q) > 0) jy += g;
        if (ey(q) < 0) jy -= g;
        if (ez(q) > 0) jz += g;
        if (ez(q) < 0) jz -= g;
    }
    D4 D[Q];
    nscbc_delta4(D4{rho, {1.f, 0.f, 0.f, 0.f}}, D4{jx, {0.f, 1.f, 0.f, 0.f}}, D4{jy, {0.f, 0.f, 1.f, 0.f}},
                 D4{jz, {0.f, 0.f, 0.f, 1.f}}, F.axis, F.side, D);
    float vk[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int m = 0; m < 4; ++m) vk[m] += lh[q] * D[q].d[m];
    const long long n = (long long)F.nu * F.nv, off = a.gadj_off[F.axis * 2 + F.side];
#pragma unroll
    for (int p = 0; p < Q; ++p)
        a.gadj[off + (long long)p * n + lt] = lh[p] + vk[0] + ex(p) * vk[1] + ey(p) * vk[2] + ez(p) * vk[3];
}

// lamF^{s-1} = J_C(F^{s-1})^T lamH^s.  With F the pulled populations,
// rho' = sum F, J = sum c F, r = 1 + rho':
//   (J_C^T l)_p = a l_p + b (A + c_p . B)
//   A = sum_q l_q w_q (1 - (4.5 (c_q.J)^2 - 1.5 J^2) / r^2)
//   B = sum_q l_q w_q (3 c_q + (9 (c_q.J) c_q - 3 J) / r)
// with a = (1 - sigma)(1 - omega), b = (1 - sigma) omega; SOLID cells copy.
__global__ void __launch_bounds__(128) k_adj_step(AdjStepArgs a)
{
    const Layout& L = a.L;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > L.nx) return;
    const int j = blockIdx.y + 1, k = blockIdx.z + 1;
    float lg[Q];
    gather_lam(L, a.sa.links, a.lam_in, a.gadj, a.gadj_off, i, j, k, lg);
    const uint32_t lk = a.sa.links[L.cell(i, j, k)];
    const long long e0 = L.elem(0, i, j, k);
    if (lk & kSolidSelfBit)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q) a.lam_out[e0 + q * L.bc] = lg[q];
        return;
    }
    // F^{s-1}: pull from Ht^{s-1} with bounce-back and x-face ghosts
    float F[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int si = i - ex(q);
        if ((lk >> q) & 1u) F[q] = a.fwd_prev[L.elem(inv(q), i, j, k)];
        else if (si == 0) F[q] = a.xgh_prev[a.sa.xf.gh_index(0, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else if (si == L.nx + 1) F[q] = a.xgh_prev[a.sa.xf.gh_index(1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else F[q] = a.fwd_prev[L.elem(q, si, j - ey(q), k - ez(q))];
    }
    float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        rho += F[q];
        if (ex(q) > 0) jx += F[q];
        if (ex(q) < 0) jx -= F[q];
        if (ey(q) > 0) jy += F[q];
        if (ey(q) < 0) jy -= F[q];
        if (ez(q) > 0) jz += F[q];
        if (ez(q) < 0) jz -= F[q];
    }
    float r = 1.0f + rho;
    if (r <= 0.f) r = 1e-12f;
    const float ir = 1.0f / r;
    const float j2 = jx * jx + jy * jy + jz * jz;
    float A = 0.f, Bx = 0.f, By = 0.f, Bz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const float cj = (float)ex(q) * jx + (float)ey(q) * jy + (float)ez(q) * jz;
        const float wl = wf(q) * lg[q];
        A += wl * (1.0f - (4.5f * cj * cj - 1.5f * j2) * ir * ir);
        const float t = 3.0f + 9.0f * cj * ir;
        Bx += wl * ((float)ex(q) * t - 3.0f * jx * ir);
        By += wl * ((float)ey(q) * t - 3.0f * jy * ir);
        Bz += wl * ((float)ez(q) * t - 3.0f * jz * ir);
    }
    const float sg = fmaxf(a.sa.sig_x[i - 1], fmaxf(a.sa.sig_y[j - 1], a.sa.sig_z[k - 1]));
    const float keep = 1.0f - sg;
    const float ca = keep * (1.0f - a.sa.omega), cb = keep * a.sa.omega;
#pragma unroll
    for (int p = 0; p < Q; ++p)
        a.lam_out[e0 + p * L.bc] =
            ca * lg[p] + cb * (A + (float)ex(p) * Bx + (float)ey(p) * By + (float)ez(p) * Bz);
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
    const dim3 g((unsigned)((a.L.nx + 127) / 128), (unsigned)a.L.ny, (unsigned)a.L.nz);
    k_adj_step<<<g, 128, 0, stream>>>(a);
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

}  // namespace lbm
