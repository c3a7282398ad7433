// SART_CUDA step kernels (sart.cu).
#pragma once

#include <cuda_runtime.h>

#include "b2tomo.h"
#include "proj2d.h"

namespace b2t {

// r = (b_a - FP_a(vol)) * W_line[a] for the step's view a = order[step % norder].
struct SartResidualLaunch {
    const float *vol;          // volume to project (x, or x * mask)
    long long vol_pitch;
    const float *sino;         // b, [angle][det]
    const float *line_weight;  // W_line, [angle][det]
    float *r;                  // one detector row
    int W, H, ndet, rays, kind;
    float out_scale;           // fan: ray-sum scale (parallel views carry theirs)
    const ParFPView *par;      // device, per view (parallel)
    const b2t_view2d *fan;     // device, per view (fan)
    const int *order;          // device projection order
    int norder;
    const long long *step;     // device step counter
};

// vol = clamp(vol + scale * mask * BP_SART_a(r)).
struct SartUpdateLaunch {
    float *vol;
    long long vol_pitch;
    const float *r;
    const float *mask;         // reconstruction mask, or null
    int W, H, ndet, kind;
    float scale;               // lambda * output scale
    int use_min, use_max;
    float min_value, max_value;
    const BPView2D *views;     // device, per view (non-FBP constants)
    const int *order;
    int norder;
    const long long *step;
};

b2t_status sart_residual_launch(const SartResidualLaunch &L, cudaStream_t s);
b2t_status sart_update_launch(const SartUpdateLaunch &L, cudaStream_t s);
b2t_status sart_advance_launch(long long *step, cudaStream_t s);

}  // namespace b2t
