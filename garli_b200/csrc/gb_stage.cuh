// gb_stage.cuh -- asynchronous copies into shared memory and the bounded
// mbarrier wait: per-lane cp.async prefetch of the precision form's CLA and
// coefficient inputs, and the wait of the tensor-core kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long stage_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// bounded wait for the phase with the given parity (at most 2^24 polls or
// about two seconds); false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    unsigned long long t0 = 0;
    for (long long it = 0; it < (1LL << 24); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 1023) == 0) {
            const unsigned long long t = stage_ns();
            if (it == 0) t0 = t;
            else if (t - t0 > 2000000000ULL) return false;
        }
    }
    return false;
}

// 16-byte asynchronous copy global -> shared through L2 (both addresses
// 16-byte aligned); completion per commit group of the issuing thread
__device__ __forceinline__ void cp16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// 8-byte asynchronous copy global -> shared (both addresses 8-byte aligned)
__device__ __forceinline__ void cp8(uint32_t dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
// 4-byte asynchronous copy global -> shared (both addresses 4-byte aligned)
__device__ __forceinline__ void cp4(uint32_t dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's commit groups are pending
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> shared of this CTA, completion counted on mbar
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(mbar)
        : "memory");
}

}  // namespace gb
