// Internal declarations of the 2D projector module.
#pragma once

#include <cuda_runtime.h>

#include "b2tomo.h"

namespace b2t {

constexpr int FP2D_MAX_VIEWS = 1024;
constexpr int BP2D_MAX_VIEWS = 1024;

// Parallel FP ray constants of one view: sample coordinate along the
// non-marching axis p(det, slice) = p0 + det * detstep + slice * slicestep.
struct ParFPView {
    float detstep, slicestep, corr, p0;
    int vertical;  // 1: march over rows (|ray x| <= |ray y|)
    int a;         // view index
};

struct FP2DParLaunch {
    const float *vol;
    long long vol_pitch;
    float *sino;
    long long sino_pitch;
    int W, H, ndet, rays, accumulate;
    ParFPView views[FP2D_MAX_VIEWS];
};

struct FP2DFanLaunch {
    const float *vol;
    long long vol_pitch;
    float *sino;
    long long sino_pitch;
    int W, H, ndet, rays, accumulate, a0;
    float out_scale;
    b2t_view2d views[FP2D_MAX_VIEWS];
};

// BP per-view constants: parallel (scaled cos, scaled sin, offset, weight),
// fan (NumC, NumX, NumY, DenC, DenX, DenY).
struct BPView2D {
    float c[6];
};

struct BP2DLaunch {
    const float *sino;
    long long sino_pitch;
    float *vol;
    long long vol_pitch;
    int W, H, ndet, rays, kind, fbp, a0, nviews, accumulate;
    float out_scale;
    BPView2D views[BP2D_MAX_VIEWS];
};

b2t_status validate2d(const b2t_geom2d *g, const char *who);
void par_fp_view(const b2t_view2d &p, const b2t_dims2d &d, float out_scale, ParFPView &o);
void bp2d_view(int kind, int fbp, const b2t_view2d &p, BPView2D &o);
b2t_status fp2d_impl(const b2t_geom2d *g, uint32_t det_supersample, const float *vol, size_t vol_pitch, float *sino,
                     size_t sino_pitch, int32_t mode, cudaStream_t s);
b2t_status bp2d_impl(const b2t_geom2d *g, uint32_t pixel_supersample, int32_t fbp_weight, const float *sino,
                     size_t sino_pitch, float *vol, size_t vol_pitch, int32_t mode, cudaStream_t s);

}  // namespace b2t
