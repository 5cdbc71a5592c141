// Bounds-checked builds (-DLBM_CHECK, liblbm_b200_check.so).  Each device
// access that could leave its array is tested first with LBM_IN(site, index,
// extent); a failing test records the site and the index in this translation
// unit's flag and the access is skipped, so the kernel runs to its end and the
// host reports the failure (lbm_check_status) instead of the GPU faulting.
// In the product build LBM_IN is the constant true and compiles away.
#pragma once

#include <cuda_runtime.h>

namespace lbm {

// Check sites (the value lbm_check_status reports).
enum CheckSite : int
{
    kChkNone = 0,
    kChkHwLine = 1,      // k_step_hw: source line copy
    kChkHwLinks = 2,     // k_step_hw: links words copy
    kChkHwGhost = 3,     // k_step_hw: x-face ghost copy
    kChkHwNear = 4,      // k_step_hw: near-solid words
    kChkHwBounce = 5,    // k_step_hw: bounce-back word
    kChkHwStore = 6,     // k_step_hw: result store
    kChkHwExport = 7,    // k_step_hw: x-face export
    kChkStepLoad = 8,    // k_step: pulled or bounce-back load
    kChkStepStore = 9,   // k_step: result store
    kChkSource = 10,     // k_source: injected cell
    kChkGhost = 11,      // k_ghost: interior or ghost cell
    kChkProbe = 12,      // k_probe / k_field_rho: pulled value
    kChkAdjLoad = 20,    // k_adj_step: gathered adjoint or moments load
    kChkAdjStore = 21,   // k_adj_step: result store
    kChkALoad = 30,      // k_step_a: pulled load
    kChkAStore = 31,     // k_step_a: result or mailbox store
    kChkSelfTest = 99,   // lbm_check_selftest: an index past its extent on purpose
};

namespace check {

// The first failed check of one kernel file: {site, index} (site 0: none).
struct Status
{
    long long site, index;
};

}  // namespace check
}  // namespace lbm

#if defined(__CUDACC__)
namespace lbm {
namespace check {
#ifdef LBM_CHECK
static __device__ unsigned long long g_flag[2];

__device__ __forceinline__ bool in_range(int site, long long i, long long n)
{
    if (i >= 0 && i < n) return true;
    if (atomicCAS(&g_flag[0], 0ull, (unsigned long long)site) == 0ull) g_flag[1] = (unsigned long long)i;
    return false;
}

// Read and clear this translation unit's flag (current device, synchronous).
static inline cudaError_t read_and_clear(Status* out)
{
    unsigned long long f[2] = {0ull, 0ull};
    cudaError_t e = cudaMemcpyFromSymbol(f, g_flag, sizeof(f));
    if (e != cudaSuccess) return e;
    out->site = (long long)f[0];
    out->index = (long long)f[1];
    if (f[0] == 0ull) return cudaSuccess;
    const unsigned long long z[2] = {0ull, 0ull};
    return cudaMemcpyToSymbol(g_flag, z, sizeof(z));
}
#define LBM_IN(site, i, n) ::lbm::check::in_range((site), (long long)(i), (long long)(n))
#else
static inline cudaError_t read_and_clear(Status* out)
{
    out->site = 0;
    out->index = 0;
    return cudaSuccess;
}
#define LBM_IN(site, i, n) true
#endif
}  // namespace check
}  // namespace lbm
#endif
