// Internal declarations of the element-wise / reduction module.
#pragma once

#include <cuda_runtime.h>

#include "b2tomo.h"

namespace b2t {

constexpr int DOT_THREADS = 512;
constexpr int DOT_MAX_BLOCKS = 1184;  // 8 x 148 SMs

int dot_num_blocks(size_t n);
b2t_status dot_launch(const void *a, const void *b, size_t n, int32_t dtype, double *partial, int nblocks,
                      double *result, cudaStream_t s);
b2t_status vec_op_impl(int32_t op, float *out, const float *a, const float *b, float sc, size_t n,
                       cudaStream_t s);
b2t_status dot_impl(const void *a, const void *b, size_t n, int32_t dtype, double *result, cudaStream_t s);
b2t_status dot_noalloc_impl(const void *a, const void *b, size_t n, int32_t dtype, double *result, cudaStream_t s);

}  // namespace b2t
