// Reverse-time adjoint of the fused D3Q19 step (FP32 storage), for the
// gradient of a receiver misfit with respect to the source position and the
// per-step source signal.  Included by api.cpp (g++) and adjoint.cu.
//
// Forward step s (kernels.cu):  G^s -source-> H^s -ghosts-> Ht^s -pull-> F^s
// -BGK/sponge-> G^{s+1};  probe p_s = sum_q F^s_q at each probe cell;
// loss L = 1/2 sum_s sum_p (p_s - d_s)^2.
// Adjoint step s, given lamF^s = dL/dF^s:
//   lamHt^s[q](y) = [y not SOLID] lamF^s[q](y + e_q) + [y + e_q SOLID] lamF^s[inv q](y)   (pull transposed)
//   lamH^s        = lamHt^s on interior cells + J_ghost^T lamHt^s(halo)                   (ghost fill)
//   dL/dm_s       = sum_cells w_hat_c sum_q w_q lamH^s[q](c)                              (source, additive)
//   lamF^{s-1}    = J_C(F^{s-1})^T lamH^s + probe residuals of step s-1
// The pull transposed is a gather: cell y collects what the cells y + e_q
// pulled from it, so no atomics are needed.  J_C(F) depends on F only through
// its moments (rho', J), and the ghost Jacobian on the moments of the interior
// face cell, so the forward recomputation stores those moments per step
// (16 bytes per cell) instead of the populations (76 bytes per cell).
#pragma once

#include <cstdint>

#include "device.hpp"

namespace lbm {

struct AdjStepArgs
{
    Layout L;
    StepArgs sa;            // links, sponge, omega of the forward step
    const float* lam_in;    // lamF^s, population layout
    float* lam_out;         // lamF^{s-1}
    const PairMoments* mom_prev;     // moments (rho', J) of F^{s-1}, dense pair order (launch_step_moments)
    const float* gadj;      // ghost-adjoint contributions of step s, per open face
    long long gadj_off[6];  // offset of face f in gadj, -1 = face not open
    int prefetch_rows;      // > 0: each block prefetches into L2 the storage row first read this many rows ahead
};

struct AdjGhostArgs
{
    Layout L;
    GhostArgs ga;           // open faces (same enumeration as the forward ghost kernel)
    const uint32_t* links;
    const float* lam_in;    // lamF^s
    const float4* face_mom; // moments of H^s at each ghost's interior cell (GhostArgs::face_mom of step s)
    float* gadj;            // out: per open face [Q][nu * nv]
    long long gadj_off[6];
};

// One injection cell of the source at one step.
struct AdjSourceCell
{
    int i, j, k;            // halo-inclusive interior coordinates; i = -1: unused slot
    int pad;
    double what;            // normalised weight w_hat_c (FLUID cells only)
    double dwhat[3];        // d w_hat_c / d (cx, cy, cz), per metre
};

struct AdjSourceArgs
{
    Layout L;
    const uint32_t* links;
    const float* lam_in;    // lamF^s
    const float* gadj;
    long long gadj_off[6];
    const AdjSourceCell* cells;   // [step][ncell]
    int ncell;
    int step;
    double* out;            // [step][4]: sum_c w_hat_c Lam_c, sum_c dw_hat_c Lam_c (3)
};

struct AdjProbeArgs
{
    int n;
    const int* ijk;         // [n][3], i = -1: not owned
    const double* resid;    // [n] residuals of this step (0 for SOLID or unowned probes)
    Layout L;
};

cudaError_t launch_adj_ghost(const AdjGhostArgs& a, cudaStream_t stream);
// J_C^T of the gathered lamF^s (plus, at the open faces, the ghost-adjoint
// terms written by launch_adj_ghost for the same step) over every interior
// cell.
cudaError_t launch_adj_step(const AdjStepArgs& a, cudaStream_t stream);
cudaError_t launch_adj_source(const AdjSourceArgs& a, cudaStream_t stream);
cudaError_t launch_adj_probe(float* lam, const AdjProbeArgs& a, cudaStream_t stream);

}  // namespace lbm
