// Internal declarations of the FDK module.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "b2tomo.h"

namespace b2t {

// Per-call FDK weighting parameters (circular orbit recovered from view 0).
struct FDKWeights {
    int apply;           // 0: filter only (no pre-weighting)
    float central_ray;   // source-origin + origin-detector distance
    float det_usize, det_vsize, zshift;
    float W;             // (D^2 / (du * Rs)) * (pi / 2) / n_angles
    int short_scan;
    float parker_scale;  // scanned range / pi
    float central_fan;   // half fan angle of the central row
};

void fdk_weights(float fSrcOrigin, float fDetOrigin, float fZShift, float fDetUSize, float fDetVSize,
                 uint32_t n_angles, uint32_t det_u, const float *angles, int short_scan, FDKWeights &P,
                 std::vector<float> &rel);
b2t_status fdk_setup(const b2t_geom3d *g, int short_scan, FDKWeights &P, std::vector<float> &rel);
b2t_status filter_rows_impl(float *data, size_t nrows, uint32_t n, size_t pitch, const b2t_filter_config *filter,
                            cudaStream_t s);
b2t_status fbp2d_impl(const b2t_geom2d *g, const b2t_filter_config *filter, int32_t short_scan, const float *sino, size_t sino_pitch,
                      float *vol, size_t vol_pitch, int32_t mode, cudaStream_t s);
b2t_status fdk_weight_filter_impl(const b2t_geom3d *g, const b2t_filter_config *filter, int32_t short_scan, void *proj,
                                  size_t proj_pitch, int32_t dtype, cudaStream_t s);
// FDK pre-weighting and filtering of views [a0, a0 + n) of the scan g, with
// the weights of the whole scan (its angle count and Parker range): src is
// the block's projections [v][n][u] (row pitch src_pitch), dst as for the
// padded BP input (element strides dst_row between views, dst_v between rows).
b2t_status fdk_weight_filter_views(const b2t_geom3d *g, uint32_t a0, uint32_t n, const b2t_filter_config *filter,
                                   int32_t short_scan, const float *src, size_t src_pitch, float *dst,
                                   long long dst_row, long long dst_v, cudaStream_t s);
b2t_status fdk_impl(const b2t_geom3d *g, const b2t_filter_config *filter, int32_t short_scan, float output_scale, const void *proj,
                    size_t proj_pitch, void *vol, size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s);

}  // namespace b2t
