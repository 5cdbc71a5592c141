// Scheme A of the D3Q19 acoustic step: the update of the reference's family-A
// programs (01-04), FP32 deviation storage.  See SchemeAArgs (device.hpp) for
// the state and the SOLID-neighbour slots; the per-step formulas follow
// 02:363-420 (destination source, SOLID cells skipped) and 03:402-441
// (forcing at the collided cell, zero-gradient halos).
#include <cuda_runtime.h>

#include <cstdint>

#include "check.cuh"
#include "device.hpp"
#include "lattice.cuh"

namespace lbm {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int BC = 32;        // FP32 cells per interleaved block
constexpr int BE = 19 * BC;   // elements per block

__device__ __forceinline__ float2 ldg2(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }

__device__ __forceinline__ uint32_t near_bits(const StepArgs& a, const Layout& L, int col, int j, int k)
{
    return a.near[((long long)k * (L.ny + 2) + j) * L.words_per_row + (col >> 5)] >> (col & 31);
}

// mass (val(t) dt gain) of step s + ahead of the field source
__device__ __forceinline__ float field_mass(const SchemeAArgs& b, int ahead)
{
    if (!b.ctl) return b.mass_direct[ahead];
    const long long row = b.ctl->step - b.ctl->table_base + ahead;
    return (float)b.table[row * b.nsrc + b.src_index].mass;
}

__device__ __forceinline__ float cell_omega(const SchemeAArgs& b, int i, int j, int k)
{
    return fminf(b.om_x[i - 1], fminf(b.om_y[j - 1], b.om_z[k - 1]));
}

// source weight of cell (i, j, k), halo-inclusive (a halo cell takes its
// nearest column's per-column weight); COLS = false: per-axis factors only
template <bool COLS = true>
__device__ __forceinline__ float field_weight(const SchemeAArgs& b, int i, int j, int k)
{
    if (COLS && b.fld_xy)
    {
        const int ci = min(max(i, 1), b.nx_col) - 1, cj = min(max(j, 1), b.ny_col) - 1;
        return b.fld_xy[cj * b.nx_col + ci];
    }
    return b.fld_x[i] * b.fld_y[j] * b.fld_z[k];
}

// strength of the destination blend at interior cell (i, j, k) (01:207-225,
// 04:177-209)
template <bool COLS = true>
__device__ __forceinline__ float cell_blend(const SchemeAArgs& b, int i, int j, int k)
{
    const float s = fmaxf(b.sg_x[i - 1], fmaxf(b.sg_y[j - 1], b.sg_z[k - 1]));
    return COLS && b.sg_xy ? fmaxf(s, b.sg_xy[(j - 1) * b.nx_col + (i - 1)]) : s;
}

// BGK of one cell on deviations d = f - feq(1, u0): with rho' = sum d,
// J' = sum c d (so rho = 1 + rho', J = u0 + J'), the equilibrium deviation is
//   w_q (rho' + 3 c.J' + (4.5 E_q - 1.5 E) / rho),
//   E_q = (c.J)^2 - rho (c.u0)^2 = 2 (c.u0)(c.J') + (c.J')^2 - rho' (c.u0)^2,
//   E   = J^2 - rho u0^2       = 2 u0.J' + J'^2 - rho' u0^2,
// written without the cancellation of feq(rho, u) - feq(1, u0); d' = d - om (d - geq).
__device__ __forceinline__ void moments1(const float (&G)[Q], float& rho, float& jx, float& jy, float& jz)
{
    rho = jx = jy = jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        rho += G[q];
        jx += ex(q) * G[q];
        jy += ey(q) * G[q];
        jz += ez(q) * G[q];
    }
}

__device__ __forceinline__ void collide1(float (&G)[Q], float om, const SchemeAArgs& b)
{
    float rho, jx, jy, jz;
    moments1(G, rho, jx, jy, jz);
    float r = 1.0f + rho;
    if (r <= 0.f) r = 1e-12f;
    const float ir = 1.0f / r;
    const float uj = b.flow[0] * jx + b.flow[1] * jy + b.flow[2] * jz;
    const float E = 2.0f * uj + jx * jx + jy * jy + jz * jz - rho * b.u0sq;
    const float base = rho - 1.5f * E * ir;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const float cj = ex(q) * jx + ey(q) * jy + ez(q) * jz;
        const float Eq = (2.0f * b.cu0[q] + cj) * cj - rho * b.cu0[q] * b.cu0[q];
        const float geq = wf(q) * (base + 3.0f * cj + 4.5f * Eq * ir);
        G[q] = G[q] - om * (G[q] - geq);
    }
}

// forcing term of the collided cell (03:74-78, 03:422-435)
__device__ __forceinline__ float force_term(const SchemeAArgs& b, int q, float s_amp, float om)
{
    return b.fq[q] * (s_amp * (1.0f - 0.5f * om));
}

// Populations arriving at interior cell (i, j, k) in the step that reads f:
// the stored values of the source cells (x-halo sources from the x-face
// array), plus the destination source for those that left a fluid cell.
__device__ __forceinline__ void pull_a(const float* __restrict__ f, const Layout& L, const StepArgs& sa,
                                       const SchemeAArgs& b, int i, int j, int k, float (&G)[Q], uint32_t& lk)
{
    lk = sa.links[L.cell(i, j, k)];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int si = i - ex(q);
        if (si == 0) G[q] = sa.xf.xgh[sa.xf.gh_index(0, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else if (si == L.nx + 1) G[q] = sa.xf.xgh[sa.xf.gh_index(1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
        else G[q] = __ldg(f + L.elem(q, si, j - ey(q), k - ez(q)));
    }
    if (b.field_mode == 0)
    {
        const float S = field_mass(b, 0) * field_weight(b, i, j, k);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (!((lk >> q) & 1u)) G[q] += wf(q) * S;
    }
    // (1 - s) f + s w_q on deviations from feq(1, u0): (1 - s) d - s base_q (01:343-347)
    if (b.blend)
    {
        const float sg = cell_blend(b, i, j, k), keep = 1.0f - sg;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (!((lk >> q) & 1u)) G[q] = fmaf(keep, G[q], -sg * b.base[q]);
    }
}

// ---------------------------------------------------------------- step
// Two x-adjacent cells per thread, aligned float2 loads with warp shuffles
// for the +-1 x shift (the same access scheme as the scheme-B step).  04's
// instance looks up what does not depend on z (the omega and blend profiles
// of the column, its source weights, the step's source masses) once per
// thread, for KZ consecutive planes (the launcher uses one: more planes per
// thread cost registers, and occupancy set this kernel's time).  FEAT: 0 = the
// update of 02 and 03; 1 = with 01's destination blend and periodic z; 2 =
// also with per-column fields and the pre-step source (04).  Each is its own
// instance, so the simpler programs keep the leaner kernel.
struct ColumnValues
{
    float2 om;      // min(om_x, om_y) of the two cells
    float2 blend;   // max(sg_x, sg_y[, sg_xy]) of the two cells
    float2 fw;      // source weight per column (fld_xy), else fld_x fld_y
    float mass0, mass1;   // source mass of this step and of the next
};

template <int FEAT>
__device__ __forceinline__ void step_a_pair(const float* __restrict__ fin, float* __restrict__ fout, const Layout& L,
                                            const StepArgs& a, const SchemeAArgs& b, const ColumnValues& z,
                                            int lane, bool active, bool has1, int c0, int j, int k)
{
    const long long e0 = L.elem(0, c0 + 1, j, k);
    const float* own = fin + e0;
    const long long rs = L.row_stride, ps = L.plane_stride;

    uint32_t lk0 = 0, lk1 = 0;
    if (active)
    {
        const uint32_t nb = near_bits(a, L, c0, j, k) & 3u;
        const long long cl = L.cell(c0 + 1, j, k);
        if (nb & 1u) lk0 = a.links[cl];
        if (nb & 2u) lk1 = a.links[cl + 1];
    }
    const bool any_link = __any_sync(kFull, (lk0 | lk1) != 0u);
    // the pair's source weights: per column (04), or the product of the
    // per-axis factors with this plane's z factor
    const auto pair_weight = [&](float m) -> float2 {
        if constexpr (FEAT == 2)
        {
            if (b.fld_xy) return mul2(f2(m), z.fw);
            const float fz = b.fld_z[k];
            return make_float2(m * (z.fw.x * fz), c0 + 1 < L.nx ? m * (z.fw.y * fz) : 0.f);
        }
        return make_float2(m * field_weight<false>(b, c0 + 1, j, k),
                           c0 + 1 < L.nx ? m * field_weight<false>(b, c0 + 2, j, k) : 0.f);
    };
    const auto mass = [&](int ahead) -> float {
        if constexpr (FEAT == 2) return ahead ? z.mass1 : z.mass0;
        return field_mass(b, ahead);
    };
    // pair load (the bounds-checked build tests the index first)
    const auto ldc = [&](const float* p) {
        return LBM_IN(kChkALoad, p - fin, L.total - 1) ? ldg2(p) : make_float2(0.f, 0.f);
    };
    float2 G[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const float* row = own - (ey(q) * rs + ez(q) * ps) + q * BC;
        const float2 cur = ldc(row);
        if (ex(q) == 0)
        {
            G[q] = cur;
        }
        else if (ex(q) > 0)
        {
            float prev = __shfl_up_sync(kFull, cur.y, 1);
            if (lane == 0) prev = ldc(row - BE + (BC - 2)).y;
            G[q] = make_float2(prev, cur.x);
        }
        else
        {
            float next = __shfl_down_sync(kFull, cur.x, 1);
            if (lane == 31) next = ldc(row + BE - (BC - 2)).x;
            G[q] = make_float2(cur.y, next);
        }
    }
    const bool xlo = active && c0 == 0, xhi0 = active && c0 == L.nx - 1, xhi1 = active && c0 + 1 == L.nx - 1;
    if (xlo | xhi0 | xhi1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if (ex(q) == 0) continue;
            const float g = a.xf.xgh[a.xf.gh_index(ex(q) > 0 ? 0 : 1, q, j - ey(q), k - ez(q), L.ny, L.nz)];
            if (ex(q) > 0 && xlo) G[q].x = g;
            if (ex(q) < 0 && xhi0) G[q].x = g;
            if (ex(q) < 0 && xhi1) G[q].y = g;
        }
    }
    if (!active) return;
    const bool solid0 = (lk0 & kSolidSelfBit) != 0u;
    const bool solid1 = !has1 || (lk1 & kSolidSelfBit) != 0u;
    if (solid0 && solid1) return;   // SOLID cells are not updated (02:371)

    // destination source, for populations that left a fluid cell (02:373, 02:405)
    if (b.field_mode == 0)
    {
        const float2 S = pair_weight(mass(0));
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const float2 add = mul2(f2(wf(q)), S);
            if (!((lk0 >> q) & 1u)) G[q].x += add.x;
            if (!((lk1 >> q) & 1u)) G[q].y += add.y;
        }
    }
    // destination blend toward rest, same populations (01:343-347)
    if (FEAT >= 1 && b.blend)
    {
        float2 sg;
        if constexpr (FEAT == 2)
        {
            const float szk = b.sg_z[k - 1];
            sg = make_float2(fmaxf(z.blend.x, szk), has1 ? fmaxf(z.blend.y, szk) : 0.f);
        }
        else
        {
            sg = make_float2(cell_blend<false>(b, c0 + 1, j, k), has1 ? cell_blend<false>(b, c0 + 2, j, k) : 0.f);
        }
        const float2 keep = sub2(f2(1.0f), sg);
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const float2 v = fma2(keep, G[q], mul2(sg, f2(-b.base[q])));
            if (!((lk0 >> q) & 1u)) G[q].x = v.x;
            if (!((lk1 >> q) & 1u)) G[q].y = v.y;
        }
    }
    // pre-step source of the next step (04:212-235): every population of the
    // cell, before it is bounced back or collided next step
    if (FEAT == 2 && b.field_mode == 2)
    {
        const float2 S = pair_weight(mass(1));
#pragma unroll
        for (int q = 0; q < Q; ++q) G[q] = fma2(f2(wf(q)), S, G[q]);
    }
    // pre-collision values for the SOLID neighbours' slots: the next step
    // pulls direction q from the SOLID cell dst - e_q and must read this
    // cell's own value of direction inv(q) (02:391-394)
    if (any_link)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
#pragma unroll
            for (int c = 0; c < 2; ++c)
            {
                const uint32_t lkc = c ? lk1 : lk0;
                const bool sol = c ? solid1 : solid0;
                if (sol || !((lkc >> q) & 1u)) continue;
                const int si = c0 + 1 + c - ex(q), sj = j - ey(q), sk = k - ez(q);
                const float v = c ? G[inv(q)].y : G[inv(q)].x;
                if (si == 0 || si == L.nx + 1) b.xgh_out[a.xf.gh_index(si == 0 ? 0 : 1, q, sj, sk, L.ny, L.nz)] = v;
                else if (LBM_IN(kChkAStore, L.elem(q, si, sj, sk), L.total)) fout[L.elem(q, si, sj, sk)] = v;
            }
        }
    }

    // BGK with each cell's own omega, FP32x2
    float2 om;
    if constexpr (FEAT == 2)
    {
        const float ozk = b.om_z[k - 1];
        om = make_float2(fminf(z.om.x, ozk), has1 ? fminf(z.om.y, ozk) : 1.0f);
    }
    else
    {
        om = make_float2(cell_omega(b, c0 + 1, j, k), has1 ? cell_omega(b, c0 + 2, j, k) : 1.0f);
    }
    {
        // moments; the 01 instance sums them one direction after another (with the
        // shared partial sums below it spills at its register cap)
        float2 rho, jx, jy, jz;
        if constexpr (FEAT == 1)
        {
            rho = jx = jy = jz = f2(0.f);
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                rho = add2(rho, G[q]);
                if (ex(q) > 0) jx = add2(jx, G[q]);
                if (ex(q) < 0) jx = sub2(jx, G[q]);
                if (ey(q) > 0) jy = add2(jy, G[q]);
                if (ey(q) < 0) jy = sub2(jy, G[q]);
                if (ez(q) > 0) jz = add2(jz, G[q]);
                if (ez(q) < 0) jz = sub2(jz, G[q]);
            }
        }
        else
        {
            // rho' = g0 + rest + S(x+) + S(x-), jx = S(x+) - S(x-)
            const float2 sxp = add2(add2(add2(G[1], G[7]), add2(G[8], G[11])), G[12]);
            const float2 sxn = add2(add2(add2(G[2], G[9]), add2(G[10], G[13])), G[14]);
            const float2 rest =
                add2(add2(add2(G[3], G[4]), add2(G[5], G[6])), add2(add2(G[15], G[16]), add2(G[17], G[18])));
            rho = add2(add2(G[0], rest), add2(sxp, sxn));
            jx = sub2(sxp, sxn);
            jy = sub2(add2(add2(add2(G[3], G[7]), add2(G[9], G[15])), G[16]),
                      add2(add2(add2(G[4], G[8]), add2(G[10], G[17])), G[18]));
            jz = sub2(add2(add2(add2(G[5], G[11]), add2(G[13], G[15])), G[17]),
                      add2(add2(add2(G[6], G[12]), add2(G[14], G[16])), G[18]));
        }
        float2 r = add2(rho, f2(1.0f));
        if (r.x <= 0.f) r.x = 1e-12f;
        if (r.y <= 0.f) r.y = 1e-12f;
        const float2 ir = make_float2(1.0f / r.x, 1.0f / r.y);
        // E = 2 u0.J' + J'^2 - rho' u0^2 (see collide1)
        const float2 uj = fma2(f2(b.flow[2]), jz, fma2(f2(b.flow[1]), jy, mul2(f2(b.flow[0]), jx)));
        const float2 E = fma2(rho, f2(-b.u0sq), fma2(uj, f2(2.0f), fma2(jz, jz, fma2(jy, jy, mul2(jx, jx)))));
        const float2 base = fma2(mul2(ir, E), f2(-1.5f), rho);
        const float2 k45 = mul2(ir, f2(4.5f));
        const float2 keep = sub2(f2(1.0f), om);
        if constexpr (FEAT == 1)
        {
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                float2 cj = f2(0.f);
                if (ex(q) > 0) cj = add2(cj, jx);
                if (ex(q) < 0) cj = sub2(cj, jx);
                if (ey(q) > 0) cj = add2(cj, jy);
                if (ey(q) < 0) cj = sub2(cj, jy);
                if (ez(q) > 0) cj = add2(cj, jz);
                if (ez(q) < 0) cj = sub2(cj, jz);
                const float c0 = b.cu0[q];
                // E_q = (2 c.u0 + c.J') c.J' - rho' (c.u0)^2
                const float2 Eq = fma2(rho, f2(-c0 * c0), mul2(add2(f2(2.0f * c0), cj), cj));
                const float2 geq = mul2(f2(wf(q)), fma2(cj, f2(3.0f), fma2(k45, Eq, base)));
                G[q] = fma2(keep, G[q], mul2(om, geq));
            }
        }
        else
        {
            // rest direction: c = 0, so E_0 = -rho' (c.u0)^2 with c.u0 = 0
            {
                const float c0 = b.cu0[0];
                const float2 Eq = fma2(rho, f2(-c0 * c0), mul2(f2(2.0f * c0), f2(0.f)));
                G[0] = fma2(keep, G[0], mul2(om, mul2(f2(wf(0)), fma2(k45, Eq, base))));
            }
            // a direction q and its opposite share c.J' up to sign and, since
            // c_{inv q}.u0 = -c_q.u0, the same E_q = (2 c.u0 + c.J') c.J' - rho' (c.u0)^2:
            // om geq = om w (base + k45 E_q) +- 3 om w c.J'
            const float2 omw1 = mul2(om, f2(wf(1))), omw2 = mul2(om, f2(wf(7)));
#pragma unroll
            for (int p = 0; p < 9; ++p)
            {
                const int q = pair_head(p), qb = inv(q);
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
                const float c0 = b.cu0[q];
                const float2 Eq = fma2(rho, f2(-c0 * c0), mul2(add2(f2(2.0f * c0), cj), cj));
                const float2 omw = q < 7 ? omw1 : omw2;
                const float2 e = mul2(omw, fma2(k45, Eq, base));
                const float2 t = mul2(omw, mul2(cj, f2(3.0f)));
                G[q] = fma2(keep, G[q], add2(e, t));
                G[qb] = fma2(keep, G[qb], sub2(e, t));
            }
        }
    }
    // forcing of this cell for the populations it sends next (03:424-435)
    if (b.field_mode == 1)
    {
        // force_term() of both cells: w_q (1 + 3 c_q.u0) s (1 - om / 2)
        const float2 sw = mul2(pair_weight(mass(1)), fma2(om, f2(-0.5f), f2(1.0f)));
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            if constexpr (FEAT == 2)
            {
                // 04's instance forms the weight in place: reading fq from the
                // parameter space costs it 36 more bytes of spills at its cap
                const float w = wf(q) * (1.0f + 3.0f * b.cu0[q]);
                G[q].x = fmaf(w, sw.x, G[q].x);
                G[q].y = fmaf(w, sw.y, G[q].y);
            }
            else
            {
                G[q].x = fmaf(b.fq[q], sw.x, G[q].x);
                G[q].y = fmaf(b.fq[q], sw.y, G[q].y);
            }
        }
    }

    const auto store = [&](long long ep) {
        float* out = fout + ep;
        if (!LBM_IN(kChkAStore, ep + 18 * BC + 1, L.total)) return;
        if (!(solid0 | solid1))
        {
#pragma unroll
            for (int q = 0; q < Q; ++q) *reinterpret_cast<float2*>(out + q * BC) = G[q];
        }
        else
        {
            // a SOLID cell's slots hold what its neighbours wrote for the next step
#pragma unroll
            for (int q = 0; q < Q; ++q)
            {
                if (!solid0) out[q * BC] = G[q].x;
                if (!solid1) out[q * BC + 1] = G[q].y;
            }
        }
    };
    store(e0);
    // periodic z (01:286-299): planes nz and 1 are also the next step's halo
    // planes 0 and nz + 1, stored twice here instead of copied afterwards
    if (FEAT >= 1 && b.zper)
    {
        if (k == L.nz) store(e0 - (long long)L.nz * ps);
        if (k == 1) store(e0 + (long long)L.nz * ps);
    }
}

template <int BLOCK, int MINB, int FEAT, int KZ>
__global__ void __launch_bounds__(BLOCK, MINB) k_step_a(const float* __restrict__ fin, float* __restrict__ fout,
                                                        Layout L, StepArgs a, SchemeAArgs b)
{
    const int lane = threadIdx.x & 31;
    const int c0r = 2 * (blockIdx.x * BLOCK + threadIdx.x);
    const bool active = c0r < L.nx;
    const int c0 = active ? c0r : ((L.nx - 1) & ~1);   // inactive lanes shadow a valid pair
    const bool has1 = c0 + 1 < L.nx;
    const int j = blockIdx.y + 1;
    if constexpr (FEAT < 2)
    {
        step_a_pair<FEAT>(fin, fout, L, a, b, ColumnValues{}, lane, active, has1, c0, j, blockIdx.z + 1);
    }
    else
    {
        const int i0 = c0 + 1, i1 = has1 ? c0 + 2 : c0 + 1;
        ColumnValues z{};
        z.om = make_float2(fminf(b.om_x[i0 - 1], b.om_y[j - 1]), fminf(b.om_x[i1 - 1], b.om_y[j - 1]));
        if (b.blend)
        {
            z.blend = make_float2(fmaxf(b.sg_x[i0 - 1], b.sg_y[j - 1]), fmaxf(b.sg_x[i1 - 1], b.sg_y[j - 1]));
            if (b.sg_xy)
                z.blend = make_float2(fmaxf(z.blend.x, b.sg_xy[(j - 1) * b.nx_col + (i0 - 1)]),
                                      fmaxf(z.blend.y, b.sg_xy[(j - 1) * b.nx_col + (i1 - 1)]));
        }
        if (b.field_mode >= 0)
        {
            if (b.fld_xy)
                z.fw = make_float2(field_weight(b, i0, j, 1), has1 ? field_weight(b, i1, j, 1) : 0.f);
            else
                z.fw = make_float2(b.fld_x[i0] * b.fld_y[j], b.fld_x[i1] * b.fld_y[j]);
        }
        z.mass0 = b.field_mode == 0 ? field_mass(b, 0) : 0.f;
        z.mass1 = b.field_mode >= 1 ? field_mass(b, 1) : 0.f;
        const int k0 = blockIdx.z * KZ + 1;
        if (b.prefetch_rows > 0 && threadIdx.x == 0)
        {
            // this CTA's columns of the storage row first read prefetch_rows rows
            // from now, one bulk prefetch into L2 (a row of the layout is contiguous)
            const long long R = (long long)k0 * (L.ny + 2) + j + (L.ny + 2) + 1 + b.prefetch_rows;
            if (R < (long long)(L.nz + 2) * (L.ny + 2))
            {
                constexpr int kBlocks = 2 * BLOCK / BC;
                const int b0 = 2 * BLOCK * (int)blockIdx.x / BC, nbk = min(kBlocks, L.nb - b0);
                const float* p = fin + kFrontElems + R * L.row_stride + (long long)b0 * BE;
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(nbk * BE * 4) : "memory");
            }
        }
#pragma unroll 1
        for (int kk = 0; kk < KZ; ++kk)
        {
            const int k = k0 + kk;
            if (k > L.nz) break;
            step_a_pair<FEAT>(fin, fout, L, a, b, z, lane, active, has1, c0, j, k);
        }
    }
}

// ---------------------------------------------------------------- halo copies
// Zero-gradient halos (03:175-237): every halo cell is a copy of the nearest
// interior cell I taken before the step and then collided like any cell,
// with the halo's own tau (outside every ramp) and source weight.  For the
// step after this one, the halo's post-collision values are
// C_bulk(f(I)) + force(halo), with f(I) the populations arriving at I in this
// step.  One thread per halo cell: x-halo planes (edges and corners
// included), then the y-halo rows, then the z-halo rows.
__global__ void __launch_bounds__(128) k_copy_a(const float* __restrict__ fin, float* __restrict__ fout, Layout L,
                                                 StepArgs a, SchemeAArgs b)
{
    // 32-bit index arithmetic: launch_copy_a rejects grids with 2^31 halo cells or more
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nyt = L.ny + 2, nzt = L.nz + 2;
    const int pX = nyt * nzt, pY = L.nx * nzt, pZ = L.nx * L.ny;   // cells of one face
    int ih, jh, kh;
    if (t < 2 * pX)
    {
        const int r = t < pX ? t : t - pX;
        ih = t < pX ? 0 : L.nx + 1;
        kh = r / nyt;
        jh = r - kh * nyt;
    }
    else if (t < 2 * pX + 2 * pY)
    {
        const int u = t - 2 * pX, r = u < pY ? u : u - pY;
        jh = u < pY ? 0 : L.ny + 1;
        kh = r / L.nx;
        ih = 1 + r - kh * L.nx;
    }
    else if (t < 2 * pX + 2 * pY + 2 * pZ)
    {
        const int u = t - 2 * pX - 2 * pY, r = u < pZ ? u : u - pZ;
        kh = u < pZ ? 0 : L.nz + 1;
        const int jr = r / L.nx;
        ih = 1 + r - jr * L.nx;
        jh = 1 + jr;
    }
    else
    {
        return;
    }
    const int i = min(max(ih, 1), L.nx), j = min(max(jh, 1), L.ny), k = min(max(kh, 1), L.nz);
    float G[Q];
    uint32_t lk;
    pull_a(fin, L, a, b, i, j, k, G, lk);
    collide1(G, b.om_bulk, b);
    if (b.field_mode == 1)
    {
        const float s = field_mass(b, 1) * field_weight(b, ih, jh, kh);
#pragma unroll
        for (int q = 0; q < Q; ++q) G[q] += force_term(b, q, s, b.om_bulk);
    }
    if (ih == 0 || ih == L.nx + 1)
    {
#pragma unroll
        for (int q = 0; q < Q; ++q) b.xgh_out[a.xf.gh_index(ih == 0 ? 0 : 1, q, jh, kh, L.ny, L.nz)] = G[q];
    }
    else
    {
        float* out = fout + L.elem(0, ih, jh, kh);
#pragma unroll
        for (int q = 0; q < Q; ++q) out[q * BC] = G[q];
    }
}

// ---------------------------------------------------------------- set-up
// Initial state of both population buffers and both x-face arrays, as
// deviations from feq(1, u0): fluid cells 0; fluid halo cells 0 with
// zero-gradient halos and rest w_q (-base) otherwise; a SOLID cell's slot q
// holds the value its neighbour cell + e_q would put there, feq(1, u0) of
// direction inv(q).
// mask_ref: the reference's halo-inclusive mask, i fastest.
__global__ void __launch_bounds__(128) k_init_a(float* __restrict__ f0, float* __restrict__ f1,
                                                float* __restrict__ xgh0, float* __restrict__ xgh1,
                                                const uint8_t* __restrict__ m, Layout L, SchemeAArgs b)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;   // 0..nx+1
    const int j = blockIdx.y, k = blockIdx.z;               // halo-inclusive
    if (i0 > L.nx + 1) return;
    const long long nxt = L.nx + 2, nyt = L.ny + 2;
    const bool solid = m[(long long)i0 + j * nxt + k * nxt * nyt] != 0;
    const bool halo = i0 == 0 || i0 == L.nx + 1 || j == 0 || j == L.ny + 1 || k == 0 || k == L.nz + 1;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        float v = 0.f;
        if (solid) v = b.base[inv(q)] - b.base[q];
        else if (halo && !b.copy) v = -b.base[q];
        if (i0 == 0 || i0 == L.nx + 1)
        {
            const long long g = XFace{nullptr, nullptr}.gh_index(i0 == 0 ? 0 : 1, q, j, k, L.ny, L.nz);
            xgh0[g] = v;
            xgh1[g] = v;
        }
        else
        {
            const long long e = L.elem(q, i0, j, k);
            f0[e] = v;
            f1[e] = v;
        }
    }
}

// ---------------------------------------------------------------- periodic z
// 01 exchanges whole z planes with itself at one rank (01:286-299) after the
// x and y halos are set, so halo plane 0 holds plane nz and halo plane nz + 1
// plane 1, at every (i, j).  The stored values are post-collision and a
// halo cell collides like the cell it repeats, so copying the stored values
// of the FLUID interior columns is the exchange; the x- and y-halo cells of
// those planes are rest (REST or WALL faces) and stay as lbm_init left them.
// SOLID cells are not copied: their slots are the mailboxes that the
// interior cells next to them write.  One thread per column and side.
__global__ void __launch_bounds__(128) k_zper_a(float* __restrict__ f, Layout L, StepArgs sa)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ncol = (long long)L.nx * L.ny;
    if (t >= 2 * ncol) return;
    const int side = t >= ncol;
    const long long r = side ? t - ncol : t;
    const int i = 1 + (int)(r % L.nx), j = 1 + (int)(r / L.nx);
    const int ks = side ? 1 : L.nz, kd = side ? L.nz + 1 : 0;
    if (sa.links[L.cell(i, j, ks)] & kSolidSelfBit) return;   // the halo cell is SOLID too
    const long long es = L.elem(0, i, j, ks), ed = L.elem(0, i, j, kd);
    if (!LBM_IN(kChkAStore, ed + 18 * BC, L.total) || !LBM_IN(kChkALoad, es + 18 * BC, L.total)) return;
#pragma unroll
    for (int q = 0; q < Q; ++q) f[ed + q * BC] = f[es + q * BC];
}

// ---------------------------------------------------------------- initial density
// 01's pulse (01:187-205): every FLUID cell starts at f = feq(1 + rho', u0)
// = (1 + rho') (w_q + base_q), an equilibrium, which the collision keeps, so
// the stored post-collision deviation is rho' (w_q + base_q); zero-gradient
// halo cells take the value of their nearest interior cell.  A SOLID
// cell's slot q holds the value its neighbour D = cell + e_q bounces back in
// the first step, f(D) of direction inv(q): base_inv(q) - base_q +
// rho'(D) (w_q + base_inv(q)) for FLUID interior D (w_inv(q) = w_q).  Other
// cells keep the state lbm_init wrote.  One thread per halo-inclusive cell.
__global__ void __launch_bounds__(128) k_set_density_a(float* __restrict__ f, float* __restrict__ xgh,
                                                       const float* __restrict__ rp, const uint8_t* __restrict__ m,
                                                       Layout L, SchemeAArgs b)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;   // 0..nx+1
    const int j = blockIdx.y, k = blockIdx.z;               // halo-inclusive
    if (i0 > L.nx + 1) return;
    const long long nxt = L.nx + 2, nyt = L.ny + 2;
    const auto mref = [&](int ii, int jj, int kk) { return m[(long long)ii + jj * nxt + kk * nxt * nyt]; };
    const auto rho_at = [&](int ii, int jj, int kk) {
        return rp[((long long)(kk - 1) * L.ny + (jj - 1)) * L.nx + (ii - 1)];
    };
    const auto interior = [&](int ii, int jj, int kk) {
        return ii >= 1 && ii <= L.nx && jj >= 1 && jj <= L.ny && kk >= 1 && kk <= L.nz;
    };
    const bool solid = mref(i0, j, k) != 0;
    if (!solid)
    {
        // a zero-gradient halo cell repeats its nearest interior cell I, and
        // collides what I holds (03:175-237): the same equilibrium, I's rho'
        const bool in = interior(i0, j, k);
        if (!in && !b.copy) return;
        const int ii = min(max(i0, 1), L.nx), jj = min(max(j, 1), L.ny), kk = min(max(k, 1), L.nz);
        if (!in && mref(ii, jj, kk) != 0) return;   // a SOLID I holds no density of its own
        const float r = rho_at(ii, jj, kk);
#pragma unroll
        for (int q = 0; q < Q; ++q)
        {
            const float v = r * (wf(q) + b.base[q]);
            if (i0 == 0 || i0 == L.nx + 1)
                xgh[XFace{nullptr, nullptr}.gh_index(i0 == 0 ? 0 : 1, q, j, k, L.ny, L.nz)] = v;
            else if (LBM_IN(kChkAStore, L.elem(q, i0, j, k), L.total))
                f[L.elem(q, i0, j, k)] = v;
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        const int di = i0 + ex(q), dj = j + ey(q), dk = k + ez(q);
        if (!interior(di, dj, dk) || mref(di, dj, dk) != 0) continue;
        const float v = b.base[inv(q)] - b.base[q] + rho_at(di, dj, dk) * (wf(q) + b.base[inv(q)]);
        if (i0 == 0 || i0 == L.nx + 1) xgh[XFace{nullptr, nullptr}.gh_index(i0 == 0 ? 0 : 1, q, j, k, L.ny, L.nz)] = v;
        else if (LBM_IN(kChkAStore, L.elem(q, i0, j, k), L.total)) f[L.elem(q, i0, j, k)] = v;
    }
}

// ---------------------------------------------------------------- probes, field
// rho - 1 after the step that reads f (the reference records rho of the
// arriving populations, 02:411, 03:438); SOLID cells read 0.
__global__ void __launch_bounds__(256) k_probe_a(const float* __restrict__ f, Layout L, StepArgs sa, SchemeAArgs b,
                                                 ProbeArgs a)
{
    const long long row = a.ctl ? a.ctl->step - a.ctl->probe_base : a.direct_row;
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
            float G[Q];
            uint32_t lk;
            pull_a(f, L, sa, b, i, j, k, G, lk);
            float rho = 0.f;
#pragma unroll
            for (int q = 0; q < Q; ++q) rho += G[q];
            val = (lk & kSolidSelfBit) ? 0.0 : (double)rho;
            a.energy[p] += val * val;
            if (!isfinite(val)) *a.nonfinite = 1;
        }
        a.out[row * a.n + p] = val;
    }
    __syncthreads();
    if (threadIdx.x == 0 && a.ctl) a.ctl->step += 1;
}

__global__ void __launch_bounds__(128) k_field_rho_a(const float* __restrict__ f, float* __restrict__ out, Layout L,
                                                     StepArgs sa, SchemeAArgs b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > L.nx) return;
    const int j = blockIdx.y + 1, k = blockIdx.z + 1;
    float G[Q];
    uint32_t lk;
    pull_a(f, L, sa, b, i, j, k, G, lk);
    float rho = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) rho += G[q];
    out[((long long)(k - 1) * L.ny + (j - 1)) * L.nx + (i - 1)] = (lk & kSolidSelfBit) ? 0.f : rho;
}

}  // namespace

cudaError_t launch_step_a(const float* fin, float* fout, const Layout& L, const StepArgs& a, const SchemeAArgs& b,
                          cudaStream_t stream)
{
    if (L.bc != BC) return cudaErrorInvalidValue;
    // every instance takes one plane per thread; 04's, with its column values
    // hoisted, at the lean instances' 72 registers (28 warps per SM): on 04's
    // 208^3 grid 0.309 ms (0.293 ms with the paired collision) against 0.326 ms
    // at 96 registers with four planes per thread, 0.320 ms at 80 registers with
    // two, 0.349-0.367 ms otherwise
    constexpr int kBlock = 128;
    const unsigned gx = (unsigned)((L.nx + 2 * kBlock - 1) / (2 * kBlock));
    if (b.field_mode == 2 || b.sg_xy || b.fld_xy)
        k_step_a<kBlock, 7, 2, 1><<<dim3(gx, L.ny, L.nz), kBlock, 0, stream>>>(fin, fout, L, a, b);
    else if (b.blend || b.zper)
        k_step_a<kBlock, 7, 1, 1><<<dim3(gx, L.ny, L.nz), kBlock, 0, stream>>>(fin, fout, L, a, b);
    else
        k_step_a<kBlock, 7, 0, 1><<<dim3(gx, L.ny, L.nz), kBlock, 0, stream>>>(fin, fout, L, a, b);
    return cudaGetLastError();
}

cudaError_t launch_copy_a(const float* fin, float* fout, const Layout& L, const StepArgs& a, const SchemeAArgs& b,
                          cudaStream_t stream)
{
    const long long n = 2LL * (L.ny + 2) * (L.nz + 2) + 2LL * L.nx * (L.nz + 2) + 2LL * L.nx * L.ny;
    if (n + 127 > 0x7fffffffLL) return cudaErrorInvalidValue;   // the kernel indexes in 32 bits
    k_copy_a<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(fin, fout, L, a, b);
    return cudaGetLastError();
}

cudaError_t launch_init_a(float* f0, float* f1, float* xgh0, float* xgh1, const uint8_t* mask_ref, const Layout& L,
                          const SchemeAArgs& b, cudaStream_t stream)
{
    const dim3 g((unsigned)((L.nx + 2 + 127) / 128), (unsigned)(L.ny + 2), (unsigned)(L.nz + 2));
    k_init_a<<<g, 128, 0, stream>>>(f0, f1, xgh0, xgh1, mask_ref, L, b);
    return cudaGetLastError();
}

cudaError_t launch_probe_a(const float* f, const Layout& L, const StepArgs& sa, const SchemeAArgs& b,
                           const ProbeArgs& a, cudaStream_t stream)
{
    k_probe_a<<<1, 256, 0, stream>>>(f, L, sa, b, a);
    return cudaGetLastError();
}

cudaError_t launch_field_rho_a(const float* f, float* out, const Layout& L, const StepArgs& sa, const SchemeAArgs& b,
                               cudaStream_t stream)
{
    const dim3 g((unsigned)((L.nx + 127) / 128), (unsigned)L.ny, (unsigned)L.nz);
    k_field_rho_a<<<g, 128, 0, stream>>>(f, out, L, sa, b);
    return cudaGetLastError();
}

cudaError_t launch_zper_a(float* f, const Layout& L, const StepArgs& sa, cudaStream_t stream)
{
    const long long n = 2LL * L.nx * L.ny;
    k_zper_a<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(f, L, sa);
    return cudaGetLastError();
}

cudaError_t launch_set_density_a(float* f, float* xgh, const float* rho_prime, const uint8_t* mask_ref,
                                 const Layout& L, const SchemeAArgs& b, cudaStream_t stream)
{
    const dim3 g((unsigned)((L.nx + 2 + 127) / 128), (unsigned)(L.ny + 2), (unsigned)(L.nz + 2));
    k_set_density_a<<<g, 128, 0, stream>>>(f, xgh, rho_prime, mask_ref, L, b);
    return cudaGetLastError();
}

cudaError_t check_read_scheme_a(check::Status* out) { return check::read_and_clear(out); }

}  // namespace lbm
