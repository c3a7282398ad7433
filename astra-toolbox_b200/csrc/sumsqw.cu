// "sum_square_weights" forward projection of parallel-beam geometries.
//
// The reference's ker3d_sum_square_weights (par3D_FP_SumSqW_t and its host
// Par3DFP_SumSqW, cuda/3d/par3d_fp.cu:329-415,607-703): per ray, the sum over
// the slices of the dominant axis of the product of the two plane axes'
// squared linear-interpolation weights, scaled by the squared ray-length
// factor (always the non-cube form, with the reference's Y-direction
// fScale2 = (fY/fY)^2).  The volume is not read.  The result accumulates into
// the projections (or replaces them in B2T_MODE_SET).
//
// One thread per detector pixel and view.  Instead of stepping a position
// along all slices, each slice's texture coordinate is A s + B (one FMA, no
// drift) and the loop covers only the slices where both weights can be
// non-zero.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "b2t_internal.h"
#include "proj3d.h"

namespace b2t {

namespace {

template <typename T> __device__ __forceinline__ float ld_out(const T *p);
template <> __device__ __forceinline__ float ld_out<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float ld_out<__half>(const __half *p) { return __half2float(*p); }
template <> __device__ __forceinline__ float ld_out<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(*p);
}
template <typename T> __device__ __forceinline__ T st_out(float v);
template <> __device__ __forceinline__ float st_out<float>(float v) { return v; }
template <> __device__ __forceinline__ __half st_out<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 st_out<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Squared interpolation weights of one axis at texture coordinate x (texel
// centres at i + 0.5, zero outside 0..n-1): both neighbours inside, one of
// them outside, or none.
__device__ __forceinline__ float dir_sqw(float x, float n)
{
    if (x <= -0.5f) return 0.0f;
    if (x <= 0.5f) return (x + 0.5f) * (x + 0.5f);
    if (x <= n - 0.5f) {
        const float t = x + 0.5f - floorf(x + 0.5f);
        return fmaf(t, t, (1.0f - t) * (1.0f - t));
    }
    if (x <= n + 0.5f) return (n + 0.5f - x) * (n + 0.5f - x);
    return 0.0f;
}

// Narrow [smin, smax] to the slices s with lo <= A s + B <= hi.
__device__ __forceinline__ void clip_range(float A, float B, float lo, float hi, float &smin, float &smax)
{
    if (fabsf(A) < 1e-12f) {
        if (!(B >= lo && B <= hi)) {
            smin = 1.0f;
            smax = 0.0f;
        }
        return;
    }
    const float s1 = (lo - B) / A, s2 = (hi - B) / A;
    smin = fmaxf(smin, fminf(s1, s2));
    smax = fminf(smax, fmaxf(s1, s2));
}

template <typename T>
__global__ void __launch_bounds__(256) fp3d_sumsqw_kernel(const __grid_constant__ FPLaunch L)
{
    const FPView &V = L.views[blockIdx.x];
    const int u = blockIdx.y * 32 + threadIdx.x;
    const int v = blockIdx.z * 8 + threadIdx.y;
    if (u >= L.nu || v >= L.nv) return;
    const float uu = (float)u + 0.5f - 0.5f * (float)L.nu;
    const float vv = (float)v + 0.5f - 0.5f * (float)L.nv;
    // parallel beams: unit denominator, slopes constant over the view; the
    // coefficients give A s + B = texture coordinate - 1
    const float A1 = V.m1[0], A2 = V.m2[0];
    const float B1 = fmaf(vv, V.n1[2], fmaf(uu, V.n1[1], V.n1[0])) + 1.0f;
    const float B2 = fmaf(vv, V.n2[2], fmaf(uu, V.n2[1], V.n2[0])) + 1.0f;
    const float n1 = (float)L.n1, n2 = (float)L.n2;
    // slices where both weights can be non-zero, widened by one slice on
    // each side against rounding (the weights are zero outside anyway)
    float smin = 0.0f, smax = (float)(L.n0 - 1);
    clip_range(A1, B1, -0.5f, n1 + 0.5f, smin, smax);
    clip_range(A2, B2, -0.5f, n2 + 0.5f, smin, smax);
    const int s_lo = (int)fmaxf(0.0f, fminf(floorf(smin) - 1.0f, (float)L.n0));
    const int s_hi = (int)fminf((float)(L.n0 - 1), fmaxf(ceilf(smax) + 1.0f, -1.0f));
    float sum0 = 0.0f, sum1 = 0.0f;
    int s = s_lo;
    for (; s + 1 <= s_hi; s += 2) {
        sum0 = fmaf(dir_sqw(fmaf(A1, (float)s, B1), n1), dir_sqw(fmaf(A2, (float)s, B2), n2), sum0);
        sum1 = fmaf(dir_sqw(fmaf(A1, (float)(s + 1), B1), n1), dir_sqw(fmaf(A2, (float)(s + 1), B2), n2), sum1);
    }
    if (s <= s_hi) sum0 = fmaf(dir_sqw(fmaf(A1, (float)s, B1), n1), dir_sqw(fmaf(A2, (float)s, B2), n2), sum0);
    const float sc2 = fmaf(A1 * A1, L.f1, fmaf(A2 * A2, L.f2, 1.0f)) * (L.mul * L.mul);
    T *out = static_cast<T *>(L.proj) + ((size_t)v * L.na + V.a) * L.proj_pitch + u;
    float r = (sum0 + sum1) * sc2;
    if (L.accumulate) r += ld_out(out);
    *out = st_out<T>(r);
}

}  // namespace

b2t_status fp3d_sumsqw_impl(const b2t_geom3d *g, const b2t_params3d *p, void *proj, size_t proj_pitch,
                            int32_t dtype, int32_t mode, cudaStream_t s)
{
    if (g->kind != B2T_GEOM_PAR3D)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_fp3d: sum_square_weights needs a parallel-beam geometry");
    if (p->det_supersample != 1)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_fp3d: sum_square_weights has no detector supersampling");
    const b2t_dims3d &d = g->dims;
    std::vector<int> dirs(d.angles);
    for (uint32_t a = 0; a < d.angles; ++a) dirs[a] = dominant_axis(g->kind, g->views[a], d);
    FPLaunch *Lp = new FPLaunch;  // large parameter block; filled per launch below
    FPLaunch &P = *Lp;
    b2t_status st = B2T_OK;
    for (int dir = 0; dir < 3 && st == B2T_OK; ++dir) {
        std::vector<int> views;
        for (uint32_t a = 0; a < d.angles; ++a)
            if (dirs[a] == dir) views.push_back((int)a);
        if (views.empty()) continue;
        P.vol = nullptr;
        P.proj = proj;
        P.proj_pitch = (long long)proj_pitch;
        P.nu = d.det_u;
        P.nv = d.det_v;
        P.na = d.angles;
        P.rays = 1;
        P.accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
        fp_scale(g->kind, dir, g->vol_scale, /*force_noncube=*/true, p->output_scale, P.f1, P.f2, P.mul);
        if (dir == 0) { P.n0 = d.vol_x; P.n1 = d.vol_y; P.n2 = d.vol_z; }
        else if (dir == 1) { P.n0 = d.vol_y; P.n1 = d.vol_x; P.n2 = d.vol_z; }
        else { P.n0 = d.vol_z; P.n1 = d.vol_x; P.n2 = d.vol_y; }
        P.st0 = P.st2 = 0;
        for (size_t c0 = 0; c0 < views.size() && st == B2T_OK; c0 += FP_MAX_VIEWS) {
            const size_t cn = std::min(views.size() - c0, (size_t)FP_MAX_VIEWS);
            P.nviews = (int)cn;
            for (size_t i = 0; i < cn; ++i) {
                fp_view_coeffs(g->kind, g->views[views[c0 + i]], d, dir, P.views[i]);
                P.views[i].a = views[c0 + i];
            }
            const dim3 grid((unsigned)cn, (d.det_u + 31) / 32, (d.det_v + 7) / 8);
            if (dtype == B2T_F32) fp3d_sumsqw_kernel<float><<<grid, dim3(32, 8), 0, s>>>(P);
            else if (dtype == B2T_F16) fp3d_sumsqw_kernel<__half><<<grid, dim3(32, 8), 0, s>>>(P);
            else fp3d_sumsqw_kernel<__nv_bfloat16><<<grid, dim3(32, 8), 0, s>>>(P);
            count_launches(1);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) st = fail(B2T_ERR_CUDA, "fp3d_sumsqw_kernel launch: %s", cudaGetErrorString(e));
        }
    }
    delete Lp;
    return st;
}

}  // namespace b2t
