// Asynchronous global -> shared copies of single complex elements
// (cp.async, sm_80 and later): the copy lands in shared memory without a
// register round trip, so a thread issues all of its tile's loads back to
// back and waits once (async_wait_all) before the barrier that publishes
// the tile.  complex128 elements go through L2 only (.cg, 16 B); complex64
// elements are 8 B, which only the .ca form takes.
#pragma once
#include <cuda_runtime.h>

namespace gm {

__device__ __forceinline__ void cp_async_elem(double2 *dst, const double2 *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_elem(float2 *dst, const float2 *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

// every cp.async this thread issued has landed
__device__ __forceinline__ void async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// the staged tile is complete and visible to the whole CTA
__device__ __forceinline__ void staged_sync() {
    async_wait_all();
    __syncthreads();
}

}  // namespace gm
