// Internal declarations of the SIRT / CGLS / SART drivers.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "b2tomo.h"

namespace b2t {

b2t_status algo_create3d_impl(int32_t type, const b2t_geom3d *geom, const b2t_params3d *params,
                              const b2t_algo_options *opt, b2t_algo **out);
b2t_status algo_create3d_cyl_impl(int32_t type, const b2t_geom3d_cyl *geom, const b2t_params3d *params,
                                  const b2t_algo_options *opt, b2t_algo **out);
b2t_status algo_create2d_impl(int32_t type, const b2t_geom2d *geom, uint32_t det_ss, uint32_t pix_ss,
                              const b2t_algo_options *opt, b2t_algo **out);
struct Batch2D;
b2t_status algo_create_batch2d_impl(int32_t type, Batch2D *batch, const b2t_algo_options *opt, b2t_algo **out);
b2t_status algo_run_impl(b2t_algo *a, const float *sino, float *vol, int32_t iters, int32_t use_graph, cudaStream_t s);
b2t_status algo_residual_impl(b2t_algo *a, const float *sino, const float *vol, double *norm, cudaStream_t s);
b2t_status algo_set_order_impl(b2t_algo *a, const int32_t *order, uint32_t n);
void algo_abort_impl(b2t_algo *a);
void algo_destroy_impl(b2t_algo *a);

}  // namespace b2t
