// Tensor-memory-accelerator (TMA) plumbing for sm_100a kernels: tiled tensor
// maps (built on the host through the driver's cuTensorMapEncodeTiled, looked
// up once at run time so the library does not link libcuda), mbarrier
// arrive/wait with an iteration bound, and the cp.async.bulk.tensor loads and
// stores.  All copies are between this GPU's global memory and the issuing
// CTA's shared memory (no cluster multicast).
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "common.cuh"

namespace aprb {

// A 3-D tiled tensor map over 4-byte elements: dims d[0..2] (d[0] contiguous),
// byte strides s1, s2 of dims 1 and 2, box b[0..2].  Returns false when the
// driver rejects the layout (alignment, stride or box limits); the caller then
// takes a path without TMA.
bool make_tensor_map_3d_f32(CUtensorMap *map, const void *base, const uint64_t d[3], uint64_t s1, uint64_t s2,
                            const uint32_t b[3]);
// A 2-D tiled tensor map (d[0] contiguous, row stride s1 bytes) over uint16 or
// float elements with 128-byte swizzling: the box's rows (128 bytes each) land
// in shared memory with their 16-byte chunks permuted, chunk j of row r at
// position j ^ (r % 8) (the destination must be 1024-byte aligned).
bool make_tensor_map_2d_sw128(CUtensorMap *map, const void *base, bool f32, const uint64_t d[2], uint64_t s1,
                              const uint32_t b[2]);

// cudaFuncSetAttribute(KERN, MaxDynamicSharedMemorySize, bytes) once per
// device for each kernel KERN (a launch needs it once per device)
template <auto KERN>
void set_smem_once(int bytes) {
    static uint64_t done = 0;  // bit d: set on device d
    int dev = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = dev < 64 ? (uint64_t(1) << dev) : 0;
    if (bit && (__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit)) return;
    APRB_CUDA(cudaFuncSetAttribute(KERN, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (bit) __atomic_fetch_or(&done, bit, __ATOMIC_RELEASE);
}

// Iterations of a bounded mbarrier wait (each try_wait may suspend the thread
// for a short, hardware-defined time); a wait that runs out reports failure.
constexpr uint32_t kMbarWaitLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// true once the phase with this parity has completed; false after
// kMbarWaitLimit attempts
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (uint32_t it = 0; it < kMbarWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, const void *src, int c0, int c1) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_addr(src)), "r"(c0), "r"(c1)
                 : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_addr(src)), "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// wait until every committed bulk store has finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// wait until every committed bulk store has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// generic-proxy shared-memory writes become visible to the async proxy (TMA)
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace aprb
