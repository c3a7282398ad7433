// Kernels of SART_CUDA (2D): one view per step.
//
// Reference: CCudaSartAlgorithm::run (src/CudaSartAlgorithm.cpp:233-318) with
// FP_SART / BP_SART (cuda/2d/mem2d.cu:332-410), mul_SART (cuda/2d/sart.cu),
// devBP_SART (cuda/2d/par_bp.cu:139-159, host :261-299) and devFanBP_SART
// (cuda/2d/fan_bp.cu:164-201, host :339-376).  A step with view a is
//   r = (b_a - FP_a(x)) * W_line[a]
//   x = clamp(x + lambda * out_scale * BP_SART_a(r))
// where BP_SART samples r with clamp-to-edge addressing and without the
// adjoint's per-view weight (the SART line weights take its place).
//
// Differences by design: the reference issues a device-to-device copy, an FP
// with its own stream and texture, a multiply and a BP with another texture
// per step, each synchronised.  Here a step is two kernels: the residual
// kernel (eight lanes per detector ray, reduced with warp shuffles) and the
// update kernel (one thread per pixel, with the clamps fused), plus a
// one-thread kernel that advances the step counter.  The view comes from a
// device-side step counter and projection order, so one step can be captured
// as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include "b2t_internal.h"
#include "proj2d_dev.cuh"
#include "sart.h"

namespace b2t {

namespace {

constexpr int SART_LANES = 8;  // lanes per detector ray in the residual kernel

__device__ __forceinline__ int sart_view(const int *order, int norder, const long long *step)
{
    return order[(int)(*step % (long long)norder)];
}

// linear interpolation of a row at index q, clamped to the edge texels
__device__ __forceinline__ float lerp_clamp(const float *__restrict__ row, int n, float q)
{
    const float fl = floorf(q);
    const int k = (int)fl;
    const float f = q - fl;
    const float a = __ldg(row + min(max(k, 0), n - 1));
    const float b = __ldg(row + min(max(k + 1, 0), n - 1));
    return fmaf(f, b - a, a);
}

__global__ void __launch_bounds__(128) sart_residual_kernel(const SartResidualLaunch L)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int det = t / SART_LANES, lane = t % SART_LANES;
    const int a = sart_view(L.order, L.norder, L.step);
    float v = 0.0f;
    if (det < L.ndet) {
        if (L.kind == B2T_GEOM_PAR2D)
            v = fp2d_par_ray(L.vol, L.vol_pitch, L.W, L.H, L.par[a], det, L.rays, lane, SART_LANES);
        else
            v = fp2d_fan_ray(L.vol, L.vol_pitch, L.W, L.H, L.fan[a], det, L.rays, L.out_scale, lane, SART_LANES);
    }
    // every lane of the warp takes part (no early return above)
#pragma unroll
    for (int o = SART_LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (det < L.ndet && lane == 0) {
        const size_t i = (size_t)a * L.ndet + det;
        L.r[det] = (L.sino[i] - v) * L.line_weight[i];
    }
}

__global__ void __launch_bounds__(256) sart_update_kernel(const SartUpdateLaunch L)
{
    const int X = blockIdx.x * 32 + threadIdx.x;
    const int Y = blockIdx.y * 8 + threadIdx.y;
    if (X >= L.W || Y >= L.H) return;
    const BPView2D &C = L.views[sart_view(L.order, L.norder, L.step)];
    const float x = (float)X - 0.5f * (float)L.W + 0.5f;
    const float y = (float)Y - 0.5f * (float)L.H + 0.5f;
    float T;
    if (L.kind == B2T_GEOM_PAR2D) {
        T = fmaf(x, C.c[0], fmaf(-y, C.c[1], C.c[2]));
    } else {
        const float yw = -y;  // world y is flipped (fan_bp.cu:184)
        const float num = fmaf(x, C.c[1], fmaf(yw, C.c[2], C.c[0]));
        const float den = fmaf(x, C.c[4], fmaf(yw, C.c[5], C.c[3]));
        T = num * (1.0f / den);
    }
    float u = lerp_clamp(L.r, L.ndet, T - 0.5f) * L.scale;
    const size_t i = (size_t)Y * L.vol_pitch + X;
    if (L.mask) u *= L.mask[(size_t)Y * L.W + X];
    float nx = L.vol[i] + u;
    if (L.use_min) nx = fmaxf(nx, L.min_value);
    if (L.use_max) nx = fminf(nx, L.max_value);
    L.vol[i] = nx;
}

__global__ void sart_advance_kernel(long long *step) { *step += 1; }

}  // namespace

b2t_status sart_residual_launch(const SartResidualLaunch &L, cudaStream_t s)
{
    const int threads = L.ndet * SART_LANES;
    sart_residual_kernel<<<(threads + 127) / 128, 128, 0, s>>>(L);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "sart residual launch");
    return B2T_OK;
}

b2t_status sart_update_launch(const SartUpdateLaunch &L, cudaStream_t s)
{
    sart_update_kernel<<<dim3((L.W + 31) / 32, (L.H + 7) / 8), dim3(32, 8), 0, s>>>(L);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "sart update launch");
    return B2T_OK;
}

b2t_status sart_advance_launch(long long *step, cudaStream_t s)
{
    sart_advance_kernel<<<1, 1, 0, s>>>(step);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "sart advance launch");
    return B2T_OK;
}

}  // namespace b2t
