// Element-wise update operations and FP64 inner products for the SIRT/CGLS
// steps.
//
// Reference: processVol3D<op> / processData<op> (cuda/3d/arith3d.cu:44-111,
// 227-451; cuda/2d/arith.cu) launch one kernel per z-slice on a stream they
// create and synchronise per call; dotProduct2D (cuda/2d/util.cu:231-357)
// reduces in float32 with a cudaMalloc/cudaFree and a synchronise per call.
// Here each operation is one grid-stride launch over the whole buffer on the
// caller's stream, and inner products accumulate in FP64 with a fixed-shape,
// deterministic two-pass tree (warp shuffles, then one block over the
// per-block partials).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "arith.h"
#include "b2t_internal.h"

namespace b2t {

namespace {

__device__ __forceinline__ float apply_op(int op, float o, float a, float b, float s)
{
    switch (op) {
    case B2T_OP_SET: return s;
    case B2T_OP_MUL_SCALAR: return o * s;
    case B2T_OP_MUL: return o * a;
    case B2T_OP_ADD_MUL: return fmaf(a, b, o);
    case B2T_OP_ADD_SCALED: return fmaf(a, s, o);
    case B2T_OP_SCALE_AND_ADD: return fmaf(o, s, a);
    case B2T_OP_INVERT: return (o > 0.000001f) ? 1.0f / o : 0.0f;
    case B2T_OP_CLAMP_MIN: return (o < s) ? s : o;
    case B2T_OP_CLAMP_MAX: return (o > s) ? s : o;
    case B2T_OP_ADD: return o + a;
    default: return o;
    }
}

__global__ void vec_op_kernel(int op, float *__restrict__ out, const float *__restrict__ a,
                              const float *__restrict__ b, float s, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float o = (op == B2T_OP_SET) ? 0.0f : out[i];
        const float av = a ? a[i] : 0.0f;
        const float bv = b ? b[i] : 0.0f;
        out[i] = apply_op(op, o, av, bv, s);
    }
}

__global__ void vec_op_kernel4(int op, float4 *__restrict__ out, const float4 *__restrict__ a,
                               const float4 *__restrict__ b, float s, size_t n4)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 o = (op == B2T_OP_SET) ? make_float4(0, 0, 0, 0) : out[i];
        const float4 av = a ? a[i] : make_float4(0, 0, 0, 0);
        const float4 bv = b ? b[i] : make_float4(0, 0, 0, 0);
        o.x = apply_op(op, o.x, av.x, bv.x, s);
        o.y = apply_op(op, o.y, av.y, bv.y, s);
        o.z = apply_op(op, o.z, av.z, bv.z, s);
        o.w = apply_op(op, o.w, av.w, bv.w, s);
        out[i] = o;
    }
}

template <typename T> __device__ __forceinline__ double ldd(const T *p, size_t i);
template <> __device__ __forceinline__ double ldd<float>(const float *p, size_t i) { return (double)__ldg(p + i); }
template <> __device__ __forceinline__ double ldd<__half>(const __half *p, size_t i)
{
    return (double)__half2float(__ldg(p + i));
}
template <> __device__ __forceinline__ double ldd<__nv_bfloat16>(const __nv_bfloat16 *p, size_t i)
{
    return (double)__bfloat162float(__ldg(p + i));
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Pass 1: each block reduces a contiguous chunk into partial[blockIdx.x].
template <typename T>
__global__ void __launch_bounds__(DOT_THREADS) dot_partial_kernel(const T *__restrict__ a, const T *__restrict__ b,
                                                                  size_t n, double *__restrict__ partial)
{
    __shared__ double warp_part[DOT_THREADS / 32];
    const size_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const size_t begin = (size_t)blockIdx.x * chunk;
    const size_t end = min(n, begin + chunk);
    double acc = 0.0;
    for (size_t i = begin + threadIdx.x; i < end; i += DOT_THREADS) {
        const double x = ldd(a, i);
        const double y = (b == a) ? x : ldd(b, i);
        acc = fma(x, y, acc);
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < DOT_THREADS / 32) ? warp_part[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

}  // namespace

// Pass 2: one block sums nparts partials in a fixed order.
__global__ void __launch_bounds__(DOT_THREADS) dot_final_kernel(const double *__restrict__ partial, int nparts,
                                                                double *__restrict__ result)
{
    __shared__ double warp_part[DOT_THREADS / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += DOT_THREADS) acc += partial[i];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < DOT_THREADS / 32) ? warp_part[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) *result = v;
    }
}

int dot_num_blocks(size_t n)
{
    // fixed shape for a given n: deterministic summation order
    size_t blocks = (n + 8 * DOT_THREADS - 1) / (8 * DOT_THREADS);
    if (blocks < 1) blocks = 1;
    if (blocks > DOT_MAX_BLOCKS) blocks = DOT_MAX_BLOCKS;
    return (int)blocks;
}

b2t_status dot_launch(const void *a, const void *b, size_t n, int32_t dtype, double *partial, int nblocks,
                      double *result, cudaStream_t s)
{
    if (dtype == B2T_F32)
        dot_partial_kernel<float><<<nblocks, DOT_THREADS, 0, s>>>(static_cast<const float *>(a),
                                                                  static_cast<const float *>(b), n, partial);
    else if (dtype == B2T_F16)
        dot_partial_kernel<__half><<<nblocks, DOT_THREADS, 0, s>>>(static_cast<const __half *>(a),
                                                                   static_cast<const __half *>(b), n, partial);
    else
        dot_partial_kernel<__nv_bfloat16><<<nblocks, DOT_THREADS, 0, s>>>(
            static_cast<const __nv_bfloat16 *>(a), static_cast<const __nv_bfloat16 *>(b), n, partial);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "dot partial launch");
    dot_final_kernel<<<1, DOT_THREADS, 0, s>>>(partial, nblocks, result);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "dot final launch");
    return B2T_OK;
}

b2t_status vec_op_impl(int32_t op, float *out, const float *a, const float *b, float sc, size_t n,
                       cudaStream_t s)
{
    if (op < B2T_OP_SET || op > B2T_OP_ADD) return fail(B2T_ERR_INVALID_ARG, "b2t_vec_op: bad op %d", op);
    if (n == 0) return B2T_OK;
    if (!out) return fail(B2T_ERR_INVALID_ARG, "b2t_vec_op: null output");
    const bool need_a = (op == B2T_OP_MUL || op == B2T_OP_ADD_MUL || op == B2T_OP_ADD_SCALED ||
                         op == B2T_OP_SCALE_AND_ADD || op == B2T_OP_ADD);
    const bool need_b = (op == B2T_OP_ADD_MUL);
    if ((need_a && !a) || (need_b && !b)) return fail(B2T_ERR_INVALID_ARG, "b2t_vec_op: missing operand");
    if (!need_a) a = nullptr;
    if (!need_b) b = nullptr;
    const bool aligned = ((uintptr_t)out % 16 == 0) && (!a || (uintptr_t)a % 16 == 0) &&
                         (!b || (uintptr_t)b % 16 == 0) && (n % 4 == 0);
    const int threads = 256;
    if (aligned) {
        const size_t n4 = n / 4;
        size_t blocks = (n4 + threads - 1) / threads;
        if (blocks > 148 * 16) blocks = 148 * 16;
        vec_op_kernel4<<<(unsigned)blocks, threads, 0, s>>>(op, reinterpret_cast<float4 *>(out),
                                                             reinterpret_cast<const float4 *>(a),
                                                             reinterpret_cast<const float4 *>(b), sc, n4);
    } else {
        size_t blocks = (n + threads - 1) / threads;
        if (blocks > 148 * 16) blocks = 148 * 16;
        vec_op_kernel<<<(unsigned)blocks, threads, 0, s>>>(op, out, a, b, sc, n);
    }
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "b2t_vec_op launch");
    return B2T_OK;
}

b2t_status dot_impl(const void *a, const void *b, size_t n, int32_t dtype, double *result, cudaStream_t s)
{
    if (!a || !b || !result) return fail(B2T_ERR_INVALID_ARG, "b2t_dot_f64: null pointer");
    if (!dtype_valid(dtype)) return fail(B2T_ERR_INVALID_ARG, "b2t_dot_f64: bad dtype %d", dtype);
    const int nb = dot_num_blocks(n);
    Scratch part;
    B2T_TRY(part.alloc(sizeof(double) * nb, s, "b2t_dot_f64 partials"));
    return dot_launch(a, b, n, dtype, part.as<double>(), nb, result, s);
}

}  // namespace b2t
