// Tensor-core Ram-Lak row filter (ramp_tc.cu): layout of the split operands
// and the host entry point.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "b2tomo.h"

namespace b2t {

// Offsets |d| <= RAMP_TC_BAND of the filter (and the centre tap) are summed
// exactly in FP32 by the split kernel, which writes that near part to the
// output; the tensor cores add the remaining far taps.  The far taps carry
// only ~0.3 % of the filter's weight, so the rounding of the tensor cores'
// FP32 accumulation (toward zero, relative to the running sum) no longer
// meets the filter's strong cancellation.
constexpr int RAMP_TC_BAND = 63;

// Shape of one filter call: M rows of nu detector values.  Inputs and taps are
// deinterleaved by parity (even / odd detector columns) and split into three
// BF16 terms:
//   a: [parity 2][term 3][M][khp]    a[q][l][m][j] = term l of x[m][2j + q]
//   b: [parity 2][term 3][nhp][khp]  b[p][l][i][j] = term l of c(2i + p - (2j + 1 - p)),
//                                     zero inside the near band
struct RampTCPlan {
    int nu;
    long long M;
    int kh;       // ceil(nu / 2): columns of one parity
    int khp;      // row pitch of a and b (elements, multiple of 16)
    int bn;       // output columns (per parity) of one tile, multiple of 16, <= 128
    int ntn;      // tiles along the output columns
    int nhp;      // rows of b per parity (ntn * bn)
    int nkb;      // 64-wide K blocks per parity
    size_t a_elems, b_elems;
};

// Plan a call; false if the shape is outside the tensor-core path (fewer than
// 128 rows or fewer than 127 detector columns), where the SIMT filter runs.
bool ramp_tc_plan(uint32_t nu, long long M, RampTCPlan &plan);

// Add the far taps of the split rows `a` (laid out as above) to dst, which
// already holds the near part: row m = v * na + ang is at dst + v * dst_v +
// ang * dst_row (elements of the storage type), columns 0 .. nu-1.  `taps` is
// scratch of plan.b_elems BF16 values.
b2t_status ramp_tc_filter(const RampTCPlan &plan, const __nv_bfloat16 *a, __nv_bfloat16 *taps, void *dst,
                          long long dst_row, long long dst_v, int na, int32_t dtype, cudaStream_t s);

// Read and clear the device error word of the tensor-core filter.
b2t_status ramp_tc_errors(uint32_t *flags);

// True unless B2T_SIMT_FILTER=1 asks for the SIMT filter everywhere.
bool ramp_tc_enabled();

}  // namespace b2t
