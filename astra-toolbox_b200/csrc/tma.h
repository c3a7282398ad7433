// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a kernels, plus
// the host-side tensor-map encoder (cuTensorMapEncodeTiled, fetched from the
// driver at run time so the library does not link libcuda directly).
//
// Only plain TMA tile loads and tile reduce-adds are used, none of them
// multicast across a cluster.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "b2tomo.h"

namespace b2t {

// Host: encode a tiled tensor map.  rank <= 5; dims/strides/box in elements /
// bytes as cuTensorMapEncodeTiled expects (strides of dims 1..rank-1).  Out of
// range elements read as zero.
b2t_status encode_tensor_map(CUtensorMap *map, CUtensorMapDataType dtype, uint32_t rank, const void *base,
                             const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
                             CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE);

// Device-side error bits: kernels OR them into their translation unit's
// error word instead of trapping; b2t_device_errors() reads and clears them.
enum { B2T_DEVERR_WAIT_TIMEOUT = 1u };

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Add `bytes` to the barrier's expected transaction count without arriving.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// try_wait with a suspend-time hint: the thread may sleep (without issuing)
// for up to `ns` nanoseconds while the phase is incomplete; it resumes as soon
// as the phase completes.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity, uint32_t ns)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return done != 0;
}

// Wait for phase `parity` of a barrier, giving up after ~max_cycles clock
// cycles.  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long max_cycles)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > max_cycles) return false;
    }
    return true;
}

// The same, sleeping between polls instead of spinning, for waits whose
// end matters more than their latency (a producer waiting for room): the
// warp leaves its issue slots to the others.
__device__ __forceinline__ bool mbar_wait_bounded_sleep(uint64_t *bar, uint32_t parity, long long max_cycles)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait_sleep(bar, parity, 20000u)) {
        if (clock64() - t0 > max_cycles) return false;
    }
    return true;
}

// Order this thread's prior generic-proxy shared-memory accesses before
// subsequent async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// Element-wise add of a shared-memory box into the tensor at (c0, c1, c2)
// (cp.reduce.async.bulk.tensor, .add, FP32 in the tensor map), tracked by
// the issuing thread's bulk groups.  The box must lie inside the tensor and
// c0 x the element size be a multiple of 16 bytes.
__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap *map, const void *src, int c0, int c1, int c2)
{
    asm volatile(
        "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void bulk_commit_group() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Wait until at most N of this thread's bulk groups still read their
// shared-memory source (the source may then be overwritten).
template <int N> __device__ __forceinline__ void bulk_wait_group_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Wait until every bulk group of this thread has completed (writes included).
__device__ __forceinline__ void bulk_wait_group_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

#endif  // __CUDACC__

}  // namespace b2t
