// tmem.cuh -- tensor memory (TMEM) as per-lane storage: allocation, and
// 32-bit loads and stores of P consecutive columns of a thread's own lane
// (shape 32x32b: a warp reaches the 32 lanes of its quadrant, warp w of a
// block lanes 32 (w % 4) .. +31).  The register adjoint keeps its tape
// here.  Stores are asynchronous (tm_wait_st before a load reads them);
// tm_ld waits for its own load, and the wait names the loaded registers so
// that no use of them is scheduled before it.  A block allocates with
// tm_alloc (one warp, which also gives up the right to allocate again),
// fences around the barrier that publishes the address, and frees with
// tm_dealloc before it exits.
#pragma once
#include <stdint.h>

#include "vm_ops.cuh"

namespace rsr {

__device__ __forceinline__ void tm_alloc(uint32_t *dst_smem, uint32_t ncols) {
    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tm_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tm_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

template <int P>
__device__ __forceinline__ void tm_st(uint32_t addr, const Vf<P> &v) {
    if constexpr (P == 2) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(addr), "r"(__float_as_uint(v.v[0])),
                     "r"(__float_as_uint(v.v[1])) : "memory");
    } else if constexpr (P == 4) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr),
                     "r"(__float_as_uint(v.v[0])), "r"(__float_as_uint(v.v[1])), "r"(__float_as_uint(v.v[2])),
                     "r"(__float_as_uint(v.v[3])) : "memory");
    } else {
        static_assert(P == 8, "tape slots of 2, 4 or 8 columns");
        asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(addr),
                     "r"(__float_as_uint(v.v[0])), "r"(__float_as_uint(v.v[1])), "r"(__float_as_uint(v.v[2])),
                     "r"(__float_as_uint(v.v[3])), "r"(__float_as_uint(v.v[4])), "r"(__float_as_uint(v.v[5])),
                     "r"(__float_as_uint(v.v[6])), "r"(__float_as_uint(v.v[7])) : "memory");
    }
}

// The wait names the loaded registers, so no use of them is scheduled
// before it.
template <int P>
__device__ __forceinline__ Vf<P> tm_ld(uint32_t addr) {
    uint32_t r[P];
    if constexpr (P == 2) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(addr) : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1])::"memory");
    } else if constexpr (P == 4) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr) : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])::"memory");
    } else {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(addr) : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])::"memory");
    }
    Vf<P> v;
#pragma unroll
    for (int j = 0; j < P; ++j) v.v[j] = __uint_as_float(r[j]);
    return v;
}

}  // namespace rsr
