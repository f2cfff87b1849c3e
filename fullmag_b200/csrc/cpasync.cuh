// cpasync.cuh — per-thread asynchronous global -> shared copies (cp.async).
#pragma once

namespace fm {

// 16-byte copy through L2 only (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// copy of one 4-, 8- or 16-byte element to a shared address (16: L2 only)
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(unsigned smem, const void *gmem) {
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem), "l"(gmem), "n"(BYTES) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// wait until at most N of this thread's committed groups are still pending
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all_but_one() { cp_async_wait<1>(); }
__device__ __forceinline__ void cp_async_wait_all() { cp_async_wait<0>(); }

}  // namespace fm
