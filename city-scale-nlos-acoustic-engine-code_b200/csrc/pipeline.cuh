// Shared-memory pipelines of bulk copies (sm_90+ cp.async.bulk with mbarrier
// completion), used by the FP16 forward step and the adjoint step: a warp
// starts 16-byte-aligned global -> shared copies whose completion is counted
// in bytes on a per-slot mbarrier, and waits for a slot's phase with an
// iteration limit, so a copy that never lands ends in an error flag instead
// of a hang.  No cluster multicast: every copy reads this GPU's own memory
// into the issuing CTA's shared memory.
#pragma once

#include <cstdint>

namespace lbm {
namespace pipe {
constexpr int kSpinLimit = 1 << 22;   // try_wait rounds before a slot wait gives up (seconds)
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Bounded wait for the phase of parity `parity`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < pipe::kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// One bulk copy global -> this CTA's shared memory, completed on `bar`
// (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

}  // namespace lbm
