// Device-side bodies of the 2D projectors, shared by the single-problem
// kernels (proj2d.cu) and the batched persistent kernels (batch2d.cu): one
// ray of a forward projection, one pixel of a backprojection.
//
// Model: cuda/2d/par_fp.cu (FPhorizontal_simple / FPvertical_simple, 53-200),
// cuda/2d/fan_fp.cu (FanFPhorizontal / FanFPvertical, 55-193),
// cuda/2d/par_bp.cu (devBP / devBP_SS, 52-137) and cuda/2d/fan_bp.cu
// (devFanBP / devFanBP_SS, 57-161), with explicit FP32 linear interpolation
// and a zero border in place of texture fetches.
#pragma once

#include <cuda_runtime.h>

#include "proj2d.h"

namespace b2t {

// linear interpolation of a 1D line at continuous index q (texel i at q = i),
// zero outside [0, n)
__device__ __forceinline__ float lerp_line(const float *__restrict__ p, long long stride, int n, float q)
{
    const float fl = floorf(q);
    const int k = (int)fl;
    const float f = q - fl;
    const float a = (k >= 0 && k < n) ? __ldg(p + (long long)k * stride) : 0.0f;
    const float b = (k + 1 >= 0 && k + 1 < n) ? __ldg(p + (long long)(k + 1) * stride) : 0.0f;
    return fmaf(f, b - a, a);
}

// Parallel-beam line integral of detector `det` (R sub-rays), scaled; over
// slices s0, s0 + ds, ... (all slices by default; a partial sum otherwise).
__device__ __forceinline__ float fp2d_par_ray(const float *vol, long long pitch, int W, int H, const ParFPView &V,
                                              int det, int R, int s0 = 0, int ds = 1)
{
    float acc = 0.0f;
    for (int r = 0; r < R; ++r) {
        const float p0 = fmaf((float)det + (0.5f + (float)r) / (float)R - 0.5f, V.detstep, V.p0);
        if (!V.vertical) {
            // slices are columns; the sample moves along the rows
            for (int sl = s0; sl < W; sl += ds)
                acc += lerp_line(vol + sl, pitch, H, fmaf((float)sl, V.slicestep, p0) - 0.5f);
        } else {
            for (int sl = s0; sl < H; sl += ds)
                acc += lerp_line(vol + (long long)sl * pitch, 1, W, fmaf((float)sl, V.slicestep, p0) - 0.5f);
        }
    }
    return acc * (V.corr / (float)R);
}

// Fan-beam line integral of detector `det` (R sub-rays), scaled; over slices
// s0, s0 + ds, ... as fp2d_par_ray.
__device__ __forceinline__ float fp2d_fan_ray(const float *vol, long long pitch, int W, int H, const b2t_view2d &V,
                                              int det, int R, float out_scale, int s0 = 0, int ds = 1)
{
    // per-ray orientation choice, in float as the reference evaluates it
    const float fdx = fabsf(fmaf((float)det, V.det_u[0], V.det_s[0]) + 0.5f - V.src[0]);
    const float fdy = fabsf(fmaf((float)det, V.det_u[1], V.det_s[1]) + 0.5f - V.src[1]);
    const bool horizontal = !(fdy > fdx);
    float acc = 0.0f;
    for (int r = 0; r < R; ++r) {
        // ray set-up in FP64: the source sits far from the origin
        const double fdet = det + (0.5 + r) / (double)R;
        const double DX = V.det_s[0] + fdet * V.det_u[0];
        const double DY = V.det_s[1] + fdet * V.det_u[1];
        float sum = 0.0f, corr;
        if (horizontal) {
            const double alpha = (V.src[1] - DY) / (V.src[0] - DX);
            const double beta = V.src[1] - alpha * V.src[0];
            corr = (float)(sqrt(alpha * alpha + 1.0) * out_scale / R);
            const float y0 = (float)(-alpha * (0.5 - 0.5 * W) - beta + 0.5 * H - 0.5);
            const float dy = (float)-alpha;
            for (int sl = s0; sl < W; sl += ds) sum += lerp_line(vol + sl, pitch, H, fmaf((float)sl, dy, y0));
        } else {
            const double alpha = (V.src[0] - DX) / (V.src[1] - DY);
            const double beta = V.src[0] - alpha * V.src[1];
            corr = (float)(sqrt(alpha * alpha + 1.0) * out_scale / R);
            const float x0 = (float)(-alpha * (0.5 - 0.5 * H) + beta + 0.5 * W - 0.5);
            const float dx = (float)-alpha;
            for (int sl = s0; sl < H; sl += ds)
                sum += lerp_line(vol + (long long)sl * pitch, 1, W, fmaf((float)sl, dx, x0));
        }
        acc = fmaf(sum, corr, acc);
    }
    return acc;
}

// Backprojection sum of pixel (X, Y) over views [0, nviews) of `views`
// (sinogram rows row0 .. row0 + nviews - 1), R x R sub-pixels, unscaled.
__device__ __forceinline__ float bp2d_pixel(const float *sino, long long sino_pitch, int row0, int nviews,
                                            const BPView2D *views, int W, int H, int ndet, int R, int kind, int fbp,
                                            int X, int Y)
{
    const float sub = 1.0f / (float)R;
    float acc = 0.0f;
    for (int i = 0; i < nviews; ++i) {
        const BPView2D &C = views[i];
        const float *row = sino + (long long)(row0 + i) * sino_pitch;
        for (int ix = 0; ix < R; ++ix) {
            for (int iy = 0; iy < R; ++iy) {
                float x = (float)X - 0.5f * (float)W + 0.5f;
                float y = (float)Y - 0.5f * (float)H + 0.5f;
                if (R > 1) {
                    x += -0.5f + 0.5f * sub + (float)ix * sub;
                    y += -0.5f + 0.5f * sub + (float)iy * sub;
                }
                if (kind == B2T_GEOM_PAR2D) {
                    // T = x c - y s + offset (par_bp.cu:78-81)
                    const float T = fmaf(x, C.c[0], fmaf(-y, C.c[1], C.c[2]));
                    acc = fmaf(lerp_line(row, 1, ndet, T - 0.5f), C.c[3], acc);
                } else {
                    // world y is flipped (fan_bp.cu:73)
                    const float yw = -y;
                    const float num = fmaf(x, C.c[1], fmaf(yw, C.c[2], C.c[0]));
                    const float den = fmaf(x, C.c[4], fmaf(yw, C.c[5], C.c[3]));
                    const float fr = 1.0f / den;
                    const float w = fbp ? fr * fr : fr;
                    acc = fmaf(lerp_line(row, 1, ndet, num * fr - 0.5f), w, acc);
                }
            }
        }
    }
    return acc;
}

}  // namespace b2t
