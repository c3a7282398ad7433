// Internal helpers shared by the libb2tomo translation units (host side).
#pragma once

#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "b2tomo.h"

namespace b2t {

// Record a failure message for b2t_last_error() on this thread and return st.
b2t_status fail(b2t_status st, const char *fmt, ...);
void clear_error();

// Count kernels launched by the library (reported by b2t_kernel_launches).
void count_launches(int n);

// Map a CUDA error to B2T_ERR_CUDA (or B2T_ERR_NO_MEMORY) with context.
b2t_status cuda_fail(cudaError_t e, const char *where);

// Measured on-chip load bandwidth (onchip_peak.cu).
b2t_status onchip_peak_impl(int32_t which, double *gbs);

#define B2T_CUDA_TRY(expr, where)                                  \
    do {                                                           \
        cudaError_t _e = (expr);                                   \
        if (_e != cudaSuccess) return ::b2t::cuda_fail(_e, where); \
    } while (0)

#define B2T_TRY(expr)                    \
    do {                                 \
        b2t_status _s = (expr);          \
        if (_s != B2T_OK) return _s;     \
    } while (0)

inline size_t dtype_size(int32_t dtype)
{
    return dtype == B2T_F32 ? 4 : 2;
}
inline bool dtype_valid(int32_t dtype)
{
    return dtype == B2T_F32 || dtype == B2T_F16 || dtype == B2T_BF16;
}

// The library's stream-ordered memory pool of the current device (created on
// first use).  Freed scratch stays cached in it between calls, so repeated
// calls do not map and unmap device memory; b2t_release_cached_memory trims it.
cudaMemPool_t scratch_pool(cudaError_t &err);
void trim_scratch_pools();

// Device-allocation bookkeeping of the library (every allocation site calls
// these): alloc_injected_failure() is true for the allocation that
// b2t_debug_fail_alloc armed (its caller then fails with B2T_ERR_NO_MEMORY
// without allocating); alloc_live() tracks the allocations the library holds,
// read by b2t_debug_live_allocations.
bool alloc_injected_failure();
void alloc_live(long long delta);

// Stream-ordered scratch allocation that is freed (stream-ordered) when the
// object goes out of scope.
class Scratch {
public:
    Scratch() = default;
    Scratch(const Scratch &) = delete;
    Scratch &operator=(const Scratch &) = delete;
    ~Scratch() { release(); }
    b2t_status alloc(size_t bytes, cudaStream_t s, const char *what)
    {
        release();
        stream_ = s;
        if (bytes == 0) bytes = 16;
        if (alloc_injected_failure()) return fail(B2T_ERR_NO_MEMORY, "%s: injected allocation failure", what);
        cudaError_t e = cudaSuccess;
        cudaMemPool_t pool = scratch_pool(e);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&ptr_, bytes, pool, s);
        if (e != cudaSuccess) {
            ptr_ = nullptr;
            (void)cudaGetLastError();  // allocation failures are not sticky: clear them
            return cuda_fail(e, what);
        }
        alloc_live(1);
        bytes_ = bytes;
        return B2T_OK;
    }
    void release()
    {
        if (ptr_) {
            cudaFreeAsync(ptr_, stream_);
            alloc_live(-1);
        }
        ptr_ = nullptr;
        bytes_ = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(ptr_); }
    size_t bytes() const { return bytes_; }

private:
    void *ptr_ = nullptr;
    size_t bytes_ = 0;
    cudaStream_t stream_ = nullptr;
};

}  // namespace b2t
