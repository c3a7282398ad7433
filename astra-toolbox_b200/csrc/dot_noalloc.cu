// b2t_dot_f64_noalloc: the FP64 inner product of b2t_dot_f64 without any
// device allocation.
//
// b2t_dot_f64 takes its per-block partial sums from a stream-ordered
// allocation.  Some callers cannot allocate at the point of the call: a
// real-time acquisition loop that must not wait on the allocator, a host
// application that hands all device memory out of its own fixed pool, a
// reconstruction service whose memory budget is already committed.  This
// entry point keeps the partial sums in a fixed array compiled into the
// library instead.  The caller still provides the inputs and the result.
//
// The array (NOALLOC_PARTS doubles, 32 KB) exists on every GPU that loads the
// library and stays there until the process exits.  The reduction runs with
// the launch shape of b2t_dot_f64 (dot_num_blocks(n) blocks), so for every n
// up to DOT_MAX_BLOCKS * NOALLOC_CHUNK elements both entry points sum in the
// same order and return the same bits; above that, blocks of at most
// NOALLOC_CHUNK elements, so n is limited to NOALLOC_PARTS * NOALLOC_CHUNK
// elements and larger n is rejected before any device work.  Every call
// writes the partial sums it reads (nothing is carried over from an earlier
// call), and all calls on one device share the array: calls that overlap on
// the GPU race and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>

#include "arith.h"
#include "b2t_internal.h"

namespace b2t {

namespace {

constexpr size_t NOALLOC_PARTS = 4096;
constexpr size_t NOALLOC_CHUNK = size_t(1) << 20;
static_assert(DOT_MAX_BLOCKS <= (int)NOALLOC_PARTS, "the fixed array must hold b2t_dot_f64's largest launch");

static __device__ __align__(256) double g_noalloc_partials[NOALLOC_PARTS];

// Device address of the array on the current device.  In host code the
// symbol is only a host-side stand-in, so the address is looked up with the
// device current, on every call: a cached address would not survive a
// cudaDeviceReset or a new context on that device.
b2t_status noalloc_partials(double **out)
{
    void *p = nullptr;
    B2T_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_partials), "b2t_dot_f64_noalloc: scratch address");
    *out = static_cast<double *>(p);
    return B2T_OK;
}

}  // namespace

b2t_status dot_noalloc_impl(const void *a, const void *b, size_t n, int32_t dtype, double *result, cudaStream_t s)
{
    if (!a || !b || !result) return fail(B2T_ERR_INVALID_ARG, "b2t_dot_f64_noalloc: null pointer");
    if (!dtype_valid(dtype)) return fail(B2T_ERR_INVALID_ARG, "b2t_dot_f64_noalloc: bad dtype %d", dtype);
    if (n > NOALLOC_PARTS * NOALLOC_CHUNK)
        return fail(B2T_ERR_INVALID_ARG,
                    "b2t_dot_f64_noalloc: %zu elements exceed the maximum of %zu (%zu blocks of %zu) "
                    "that its fixed scratch array holds; use b2t_dot_f64",
                    n, NOALLOC_PARTS * NOALLOC_CHUNK, NOALLOC_PARTS, NOALLOC_CHUNK);
    double *partials = nullptr;
    B2T_TRY(noalloc_partials(&partials));
    const size_t nblocks = std::max((size_t)dot_num_blocks(n), (n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
    return dot_launch(a, b, n, dtype, partials, (int)nblocks, result, s);
}

}  // namespace b2t
