// D3Q19 lattice in the reference's family-B velocity order
// (06_transient_localization_dx1.cpp:21-31).  Every accessor is constexpr so
// that fully unrolled loops over q fold to immediate operands on the device.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define LBM_HD __host__ __device__ __forceinline__
#else
#define LBM_HD inline
#endif

namespace lbm {

constexpr int Q = 19;
constexpr uint32_t kSolidSelfBit = 1u << 19;   // links word: bit q = src of q is SOLID, bit 19 = cell SOLID

constexpr double kCs2 = 1.0 / 3.0;                 // 06:17
constexpr double kCs = 0.57735026918962576451;     // 06:18
constexpr double kPi = 3.14159265358979323846;     // 06:19

LBM_HD constexpr int ex(int q)
{
    constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 0, 0, 0, 0};
    return t[q];
}
LBM_HD constexpr int ey(int q)
{
    constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
    return t[q];
}
LBM_HD constexpr int ez(int q)
{
    constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
    return t[q];
}
// Opposite direction: e_{inv(q)} = -e_q (the table 06:301-312 computes at run time).
LBM_HD constexpr int inv(int q)
{
    constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    return t[q];
}
LBM_HD constexpr double wd(int q) { return q == 0 ? 1.0 / 3.0 : (q < 7 ? 1.0 / 18.0 : 1.0 / 36.0); }
LBM_HD constexpr float wf(int q) { return q == 0 ? 1.0f / 3.0f : (q < 7 ? 1.0f / 18.0f : 1.0f / 36.0f); }

// Directions with a positive "first non-zero component"; each forms a pair
// (q, inv(q)) for the symmetric evaluation of the equilibrium.
LBM_HD constexpr int pair_head(int p)
{
    constexpr int t[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
    return t[p];
}

}  // namespace lbm
