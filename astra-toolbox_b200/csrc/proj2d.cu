// 2D forward and back projectors for parallel (parallel / parallel_vec) and
// fan (fanflat / fanflat_vec) geometries.
//
// Model: cuda/2d/par_fp.cu (FPhorizontal_simple / FPvertical_simple, 53-200),
// cuda/2d/fan_fp.cu (FanFPhorizontal / FanFPvertical, 55-193),
// cuda/2d/par_bp.cu (devBP / devBP_SS, 52-137) and cuda/2d/fan_bp.cu
// (devFanBP / devFanBP_SS, 57-161), evaluated with explicit FP32 linear
// interpolation and a zero border instead of texture fetches.  Per-view
// constants are computed on the host in FP64 (the reference evaluates
// __cosf/__sinf on the device) and passed as kernel parameters.
//
// One launch covers every view of a chunk: FP threads own one ray (all
// slices accumulated in registers), BP threads own one pixel (all views of
// the chunk accumulated in registers).  The per-ray and per-pixel bodies live
// in proj2d_dev.cuh, shared with the batched kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "b2t_internal.h"
#include "proj2d.h"
#include "proj2d_dev.cuh"

namespace b2t {

namespace {

__global__ void __launch_bounds__(256) fp2d_par_kernel(const __grid_constant__ FP2DParLaunch L)
{
    const int det = blockIdx.x * blockDim.x + threadIdx.x;
    const int vi = blockIdx.y;
    if (det >= L.ndet) return;
    const ParFPView &V = L.views[vi];
    const float acc = fp2d_par_ray(L.vol, L.vol_pitch, L.W, L.H, V, det, L.rays);
    float *out = L.sino + (long long)V.a * L.sino_pitch + det;
    *out = L.accumulate ? *out + acc : acc;
}

__global__ void __launch_bounds__(256) fp2d_fan_kernel(const __grid_constant__ FP2DFanLaunch L)
{
    const int det = blockIdx.x * blockDim.x + threadIdx.x;
    const int vi = blockIdx.y;
    if (det >= L.ndet) return;
    const float acc = fp2d_fan_ray(L.vol, L.vol_pitch, L.W, L.H, L.views[vi], det, L.rays, L.out_scale);
    float *out = L.sino + (long long)(L.a0 + vi) * L.sino_pitch + det;
    *out = L.accumulate ? *out + acc : acc;
}

__global__ void __launch_bounds__(256) bp2d_kernel(const __grid_constant__ BP2DLaunch L)
{
    const int X = blockIdx.x * 32 + threadIdx.x;
    const int Y = blockIdx.y * 8 + threadIdx.y;
    if (X >= L.W || Y >= L.H) return;
    const float acc = bp2d_pixel(L.sino, L.sino_pitch, L.a0, L.nviews, L.views, L.W, L.H, L.ndet, L.rays, L.kind,
                                 L.fbp, X, Y);
    float *o = L.vol + (long long)Y * L.vol_pitch + X;
    const float r = acc * L.out_scale;
    *o = L.accumulate ? *o + r : r;
}

}  // namespace

b2t_status validate2d(const b2t_geom2d *g, const char *who)
{
    if (!g || !g->views) return fail(B2T_ERR_INVALID_ARG, "%s: null geometry", who);
    if (g->kind != B2T_GEOM_PAR2D && g->kind != B2T_GEOM_FAN2D)
        return fail(B2T_ERR_INVALID_ARG, "%s: geometry kind must be PAR2D or FAN2D", who);
    const b2t_dims2d &d = g->dims;
    if (d.vol_width == 0 || d.vol_height == 0 || d.angles == 0 || d.dets == 0)
        return fail(B2T_ERR_INVALID_ARG, "%s: empty dimension", who);
    if (d.vol_width > 65536 || d.vol_height > 65536 || d.dets > (1u << 20))
        return fail(B2T_ERR_INVALID_ARG, "%s: dimension too large", who);
    return B2T_OK;
}

// getParParameters (src/GeometryUtil2D.cpp:107-131) and the derived FP ray
// constants of FPhorizontal_simple / FPvertical_simple.
void par_fp_view(const b2t_view2d &p, const b2t_dims2d &d, float out_scale, ParFPView &o)
{
    double ux = p.det_u[0], uy = p.det_u[1];
    const double rx = p.src[0], ry = p.src[1];
    double t = (ux * rx + uy * ry) / (rx * rx + ry * ry);
    ux -= t * rx;
    uy -= t * ry;
    const float fAngle = (float)atan2(uy, ux);
    const double norm2 = uy * uy + ux * ux;
    const float fDetSize = (float)sqrt(norm2);
    const float fOffset = (float)(-0.5 * d.dets - (p.det_s[1] * uy + p.det_s[0] * ux) / norm2);
    const double c = cos((double)fAngle), s = sin((double)fAngle);
    const bool vertical = fabsf(p.src[0]) <= fabsf(p.src[1]);
    o.vertical = vertical ? 1 : 0;
    double detstep, slicestep, corr, p0;
    if (!vertical) {
        detstep = -fDetSize / s;
        slicestep = c / s;
        corr = out_scale / std::fabs(s);
        p0 = (0.5 - 0.5 * d.dets - fOffset) * detstep + (0.5 - 0.5 * d.vol_width) * slicestep + 0.5 * d.vol_height;
    } else {
        detstep = fDetSize / c;
        slicestep = s / c;
        corr = out_scale / std::fabs(c);
        p0 = (0.5 - 0.5 * d.dets - fOffset) * detstep + (0.5 - 0.5 * d.vol_height) * slicestep + 0.5 * d.vol_width;
    }
    o.detstep = (float)detstep;
    o.slicestep = (float)slicestep;
    o.corr = (float)corr;
    o.p0 = (float)p0;
}

// BP per-view constants: par_bp.cu:163-191, fan_bp.cu:225-279.
void bp2d_view(int kind, int fbp, const b2t_view2d &p, BPView2D &o)
{
    if (kind == B2T_GEOM_PAR2D) {
        const double d = (double)p.det_u[0] * p.src[1] - (double)p.det_u[1] * p.src[0];
        o.c[0] = (float)(p.src[1] / d);
        o.c[1] = (float)(-p.src[0] / d);
        o.c[2] = (float)(((double)p.det_s[1] * p.src[0] - (double)p.det_s[0] * p.src[1]) / d);
        o.c[3] = (float)(std::sqrt((double)p.src[0] * p.src[0] + (double)p.src[1] * p.src[1]) / std::fabs(d));
        o.c[4] = o.c[5] = 0.0f;
    } else {
        const double ux = p.det_u[0], uy = p.det_u[1], sx = p.src[0], sy = p.src[1];
        const double dx = p.det_s[0], dy = p.det_s[1];
        const double smdx = sx - dx, smdy = sy - dy;
        double scale;
        if (!fbp) scale = std::sqrt(ux * ux + uy * uy) / (ux * smdy - uy * smdx);
        else scale = 1.0 / (ux * sy - uy * sx);
        o.c[0] = (float)(scale * (sx * dy - sy * dx));
        o.c[1] = (float)(scale * smdy);
        o.c[2] = (float)(-scale * smdx);
        o.c[3] = fbp ? 1.0f : (float)(scale * (ux * sy - uy * sx));
        o.c[4] = (float)(scale * uy);
        o.c[5] = (float)(-scale * ux);
    }
}

b2t_status fp2d_impl(const b2t_geom2d *g, uint32_t det_supersample, const float *vol, size_t vol_pitch, float *sino,
                     size_t sino_pitch, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate2d(g, "b2t_fp2d"));
    if (!vol || !sino) return fail(B2T_ERR_INVALID_ARG, "b2t_fp2d: null data pointer");
    if (det_supersample == 0 || det_supersample > 64)
        return fail(B2T_ERR_INVALID_ARG, "b2t_fp2d: detector supersampling must be 1..64");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_fp2d: bad mode");
    const b2t_dims2d &d = g->dims;
    if (vol_pitch == 0) vol_pitch = d.vol_width;
    if (sino_pitch == 0) sino_pitch = d.dets;
    if (vol_pitch < d.vol_width || sino_pitch < d.dets) return fail(B2T_ERR_INVALID_ARG, "b2t_fp2d: pitch below row length");
    const int acc = (mode == B2T_MODE_ADD) ? 1 : 0;
    if (g->kind == B2T_GEOM_PAR2D) {
        FP2DParLaunch *L = new FP2DParLaunch;
        L->vol = vol; L->vol_pitch = (long long)vol_pitch; L->sino = sino; L->sino_pitch = (long long)sino_pitch;
        L->W = d.vol_width; L->H = d.vol_height; L->ndet = d.dets; L->rays = det_supersample; L->accumulate = acc;
        for (uint32_t c0 = 0; c0 < d.angles; c0 += FP2D_MAX_VIEWS) {
            const uint32_t cn = std::min(d.angles - c0, (uint32_t)FP2D_MAX_VIEWS);
            for (uint32_t i = 0; i < cn; ++i) {
                par_fp_view(g->views[c0 + i], d, g->output_scale, L->views[i]);
                L->views[i].a = (int)(c0 + i);
            }
            fp2d_par_kernel<<<dim3((d.dets + 255) / 256, cn), 256, 0, s>>>(*L);
            count_launches(1);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                delete L;
                return cuda_fail(e, "fp2d par launch");
            }
        }
        delete L;
    } else {
        FP2DFanLaunch *L = new FP2DFanLaunch;
        L->vol = vol; L->vol_pitch = (long long)vol_pitch; L->sino = sino; L->sino_pitch = (long long)sino_pitch;
        L->W = d.vol_width; L->H = d.vol_height; L->ndet = d.dets; L->rays = det_supersample; L->accumulate = acc;
        L->out_scale = g->output_scale;
        for (uint32_t c0 = 0; c0 < d.angles; c0 += FP2D_MAX_VIEWS) {
            const uint32_t cn = std::min(d.angles - c0, (uint32_t)FP2D_MAX_VIEWS);
            L->a0 = (int)c0;
            for (uint32_t i = 0; i < cn; ++i) L->views[i] = g->views[c0 + i];
            fp2d_fan_kernel<<<dim3((d.dets + 255) / 256, cn), 256, 0, s>>>(*L);
            count_launches(1);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                delete L;
                return cuda_fail(e, "fp2d fan launch");
            }
        }
        delete L;
    }
    return B2T_OK;
}

b2t_status bp2d_impl(const b2t_geom2d *g, uint32_t pixel_supersample, int32_t fbp_weight, const float *sino,
                     size_t sino_pitch, float *vol, size_t vol_pitch, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate2d(g, "b2t_bp2d"));
    if (!vol || !sino) return fail(B2T_ERR_INVALID_ARG, "b2t_bp2d: null data pointer");
    if (pixel_supersample == 0 || pixel_supersample > 64)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp2d: pixel supersampling must be 1..64");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_bp2d: bad mode");
    if (fbp_weight && g->kind != B2T_GEOM_FAN2D)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_bp2d: FBP weighting applies to fan geometries");
    if (fbp_weight && pixel_supersample > 1)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_bp2d: FBP weighting without supersampling only");
    const b2t_dims2d &d = g->dims;
    if (vol_pitch == 0) vol_pitch = d.vol_width;
    if (sino_pitch == 0) sino_pitch = d.dets;
    if (vol_pitch < d.vol_width || sino_pitch < d.dets) return fail(B2T_ERR_INVALID_ARG, "b2t_bp2d: pitch below row length");
    BP2DLaunch *L = new BP2DLaunch;
    L->sino = sino; L->sino_pitch = (long long)sino_pitch; L->vol = vol; L->vol_pitch = (long long)vol_pitch;
    L->W = d.vol_width; L->H = d.vol_height; L->ndet = d.dets; L->rays = pixel_supersample;
    L->kind = g->kind; L->fbp = fbp_weight ? 1 : 0;
    L->out_scale = g->output_scale / (float)(pixel_supersample * pixel_supersample);
    for (uint32_t c0 = 0; c0 < d.angles; c0 += BP2D_MAX_VIEWS) {
        const uint32_t cn = std::min(d.angles - c0, (uint32_t)BP2D_MAX_VIEWS);
        L->a0 = (int)c0;
        L->nviews = (int)cn;
        L->accumulate = (c0 > 0 || mode == B2T_MODE_ADD) ? 1 : 0;
        for (uint32_t i = 0; i < cn; ++i) bp2d_view(g->kind, L->fbp, g->views[c0 + i], L->views[i]);
        bp2d_kernel<<<dim3((d.vol_width + 31) / 32, (d.vol_height + 7) / 8), dim3(32, 8), 0, s>>>(*L);
        count_launches(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            delete L;
            return cuda_fail(e, "bp2d launch");
        }
    }
    delete L;
    return B2T_OK;
}

}  // namespace b2t
