// FDK reconstruction: pre-weighting, Parker short-scan weighting, Ram-Lak
// row filter and the FDK-weighted cone backprojection.
//
// Reference: FDK (cuda/3d/fdk.cu:415-478) runs devFDK_preweight
// (fdk.cu:70-113), optionally devFDK_ParkerWeight (fdk.cu:115-163), then
// FDK_Filter (fdk.cu:266-412: per detector row, memset + pitched copy + cuFFT
// R2C + spectrum multiply + C2R + rescale + copy back), then ConeBP with
// ker3d_fdk_weighting.
//
// Here the weights and the filter are one pass: each CTA loads a few
// projection rows into shared memory with the weights applied, evaluates the
// Ram-Lak filter as the Toeplitz product it equals (y_i = sum_j 2 h(|i-j|) x_j
// with h(0) = 1/4, h(odd k) = -1/(pi k)^2, h(even k != 0) = 0; the reference's
// zero padding to nextpow2(2 nU) makes its FFT convolution identical to this),
// and writes the result straight into the zero-padded buffer the
// backprojector reads, so the filtered projections never make an extra HBM
// round trip.  The filter uses only the odd taps and a sliding register window
// of 8 outputs per thread.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "b2t_internal.h"
#include "fdk.h"
#include "proj2d.h"
#include "proj3d.h"
#include "filters.h"
#include "ramp_tc.h"

namespace b2t {

namespace {

template <typename T> __device__ __forceinline__ float ldf(const T *p);
template <> __device__ __forceinline__ float ldf<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ldf<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(__ldg(p));
}
template <typename T> __device__ __forceinline__ T stf(float v);
template <> __device__ __forceinline__ float stf<float>(float v) { return v; }
template <> __device__ __forceinline__ __half stf<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 stf<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

constexpr int FILT_THREADS = 256;
constexpr int FILT_OUT = 8;  // consecutive outputs per thread

// Parker weight of view a at detector column offset fU (devFDK_ParkerWeight).
__device__ __forceinline__ float parker_weight(float beta, float fU, const FDKWeights &P)
{
    const float gamma = atanf(fU / P.central_ray);
    const float cfa = P.central_fan;
    float w;
    if (beta <= 0.0f) {
        w = 0.0f;
    } else if (beta <= 2.0f * (cfa + gamma)) {
        w = sinf((float)(M_PI / 4.0) * beta / (cfa + gamma));
        w *= w;
    } else if (beta <= (float)M_PI + 2.0f * gamma) {
        w = 1.0f;
    } else if (beta <= (float)M_PI + 2.0f * cfa) {
        w = sinf((float)(M_PI / 4.0) * ((float)M_PI + 2.0f * cfa - beta) / (cfa - gamma));
        w *= w;
    } else {
        w = 0.0f;
    }
    return w * P.parker_scale;
}

// FDK weight of detector column u in a row with vertical offset fV (view at
// relative angle beta): devFDK_preweight times, for short scans, the Parker
// weight.  1 when the weights are off (plain filtering).
__device__ __forceinline__ float fdk_weight(const FDKWeights &P, int u, int nu, float fV, float beta)
{
    if (!P.apply) return 1.0f;
    const float fU = ((float)u - 0.5f * (float)nu + 0.5f) * P.det_usize;
    const float rl = sqrtf(P.central_ray * P.central_ray + fU * fU + fV * fV);
    float w = P.W / rl;
    if (P.short_scan) w *= parker_weight(beta, fU, P);
    return w;
}

__device__ __forceinline__ void split3(float x, __nv_bfloat16 &t0, __nv_bfloat16 &t1, __nv_bfloat16 &t2)
{
    t0 = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(t0);
    t1 = __float2bfloat16_rn(r1);
    t2 = __float2bfloat16_rn(r1 - __bfloat162float(t1));
}

// Weighted rows for the tensor-core filter (ramp_tc.h).  One CTA stages
// SPLIT_ROWS rows in shared memory (FDK weights applied, zero beyond the row)
// and then
//   - writes the exact near part of the filter to dst:
//       near_n = x_n / 2 + sum_{odd d <= RAMP_TC_BAND} c(d) (x_{n-d} + x_{n+d})
//     in FP32 (round to nearest); the tensor cores later add the far taps;
//   - writes the three BF16 terms of x[m][2j] and x[m][2j+1] into the even and
//     odd planes of the split operand (zero past the row and in the pitch).
// Every row is read completely before any of it is written, so src may equal
// dst (in-place filtering).
constexpr int SPLIT_ROWS = 4;
constexpr int SPLIT_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(SPLIT_THREADS) fdk_split_kernel(
    const T *src, long long src_pitch, int nu, int na, int nv, FDKWeights P, const float *__restrict__ rel_angles,
    __nv_bfloat16 *out, int khp, long long M, T *dst, long long dst_row, long long dst_v)
{
    extern __shared__ float xs[];  // SPLIT_ROWS rows of skewed(PADL + nu + PADR) floats
    __shared__ float taps[(RAMP_TC_BAND + 1) / 2];
    // the sliding window below reads x[n0 - BAND - 2 .. n0 + BAND + 9] for
    // output groups n0 <= nu - 1 (its last shift fetches one tap ahead)
    const int PADL = RAMP_TC_BAND + 3, PADR = RAMP_TC_BAND + 9;
    const int W = PADL + nu + PADR;
    // Skewed row layout: logical column i sits at k + k / 8 with k = i + PADL,
    // so lanes whose windows start 8 columns apart hit banks 9 apart
    // (conflict-free) instead of 8 apart (4 banks, 8-way conflicts).
    const int WS = W + W / 8 + 1;
    auto at = [PADL](const float *row, int i) -> float {
        const int k = i + PADL;
        return row[k + (k >> 3)];
    };
    const long long m0 = (long long)blockIdx.x * SPLIT_ROWS;
    const int nr = (int)min((long long)SPLIT_ROWS, M - m0);
    for (int t = threadIdx.x; t < (RAMP_TC_BAND + 1) / 2; t += SPLIT_THREADS) {
        const double d = 2.0 * t + 1.0;
        taps[t] = (float)(-2.0 / (M_PI * M_PI * d * d));
    }
    for (int r = 0; r < nr; ++r) {
        const long long m = m0 + r;
        const int v = (int)(m / na);
        const int a = (int)(m - (long long)v * na);
        const float fV = ((float)v - 0.5f * (float)nv + 0.5f) * P.det_vsize + P.zshift;
        const float beta = P.short_scan ? rel_angles[a] : 0.0f;
        const T *row = src + m * src_pitch;
        float *x = xs + r * WS;
        for (int j = threadIdx.x; j < W; j += SPLIT_THREADS) {
            const int u = j - PADL;
            x[j + (j >> 3)] = (u >= 0 && u < nu) ? ldf(row + u) * fdk_weight(P, u, nu, fV, beta) : 0.0f;
        }
    }
    __syncthreads();
    const long long term = M * khp;
    for (int r = 0; r < nr; ++r) {
        const long long m = m0 + r;
        const float *x = xs + r * WS;  // logical columns -PADL .. nu + PADR - 1 through at()
        const int v = (int)(m / na);
        T *orow = dst + (long long)v * dst_v + (m - (long long)v * na) * dst_row;
        // 8 consecutive outputs per thread; L[j] = x[n0 + j - d], R[j] = x[n0 + j + d],
        // slid by two columns per odd tap d
        for (int g = threadIdx.x; g < (nu + 7) / 8; g += SPLIT_THREADS) {
            const int n0 = 8 * g;
            // column n0 + c of the skewed row is xb[sk(c)]: n0 is a multiple
            // of 8, so with the taps fully unrolled every load is the base
            // plus a compile-time offset
            const float *xb = x + 9 * g;
            auto sk = [PADL](int c) { return (PADL + c) + ((PADL + c) >> 3); };
            float acc[8], Lw[8], Rw[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                acc[j] = 0.5f * xb[sk(j)];
                Lw[j] = xb[sk(j - 1)];
                Rw[j] = xb[sk(j + 1)];
            }
#pragma unroll
            for (int t = 0; t < (RAMP_TC_BAND + 1) / 2; ++t) {
                const float c = taps[t];
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[j] = fmaf(c, Lw[j] + Rw[j], acc[j]);
                const int d = 2 * t + 1;
#pragma unroll
                for (int j = 7; j >= 2; --j) Lw[j] = Lw[j - 2];
                Lw[0] = xb[sk(-d - 2)];
                Lw[1] = xb[sk(-d - 1)];
#pragma unroll
                for (int j = 0; j < 6; ++j) Rw[j] = Rw[j + 2];
                Rw[6] = xb[sk(d + 8)];
                Rw[7] = xb[sk(d + 9)];
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (n0 + j < nu) orow[n0 + j] = stf<T>(acc[j]);
        }
        __nv_bfloat16 *e = out + m * khp;
        for (int j = threadIdx.x; j < khp; j += SPLIT_THREADS) {
            const int u0 = 2 * j, u1 = 2 * j + 1;
            const float x0 = (u0 < nu) ? at(x, u0) : 0.0f;
            const float x1 = (u1 < nu) ? at(x, u1) : 0.0f;
            __nv_bfloat16 t0, t1, t2;
            split3(x0, t0, t1, t2);
            e[j] = t0;
            e[j + term] = t1;
            e[j + 2 * term] = t2;
            split3(x1, t0, t1, t2);
            e[j + 3 * term] = t0;
            e[j + 4 * term] = t1;
            e[j + 5 * term] = t2;
        }
    }
}

// One CTA filters `rows` consecutive rows m = v * na + a of proj (pitch in
// elements).  Shared memory: rows x (3 nu + 32) floats (each row zero-padded
// by nu + 16 on both sides, which covers every window read, including the
// look-ahead loads of the last tap) followed by the odd taps.
template <typename T>
__global__ void __launch_bounds__(FILT_THREADS) fdk_weight_filter_kernel(
    const T *src, long long src_pitch, int nu, int na, int nv, int rows, FDKWeights P,
    const float *__restrict__ rel_angles, int do_filter, T *dst, long long dst_row_stride,
    long long dst_v_stride)
{
    extern __shared__ float sm[];
    const int PADW = nu + 16;
    const int W3 = nu + 2 * PADW;
    float *taps = sm + (size_t)rows * W3;
    const int nodd = (nu + 1) / 2;
    const long long m0 = (long long)blockIdx.x * rows;
    const long long mtot = (long long)na * nv;
    int nr = (int)min((long long)rows, mtot - m0);
    if (nr <= 0) return;

    for (int j = threadIdx.x; j < nodd; j += FILT_THREADS) {
        const double k = 2.0 * j + 1.0;
        taps[j] = (float)(-2.0 / (M_PI * M_PI * k * k));
    }
    // load rows with weights applied, zero padding on both sides
    for (int r = 0; r < nr; ++r) {
        const long long m = m0 + r;
        const int v = (int)(m / na);
        const int a = (int)(m - (long long)v * na);
        const float fV = ((float)v - 0.5f * (float)nv + 0.5f) * P.det_vsize + P.zshift;
        const float beta = P.short_scan ? rel_angles[a] : 0.0f;
        const T *row = src + m * src_pitch;
        float *xs = sm + (size_t)r * W3;
        for (int j = threadIdx.x; j < W3; j += FILT_THREADS) {
            const int u = j - PADW;
            float val = 0.0f;
            if (u >= 0 && u < nu) {
                val = ldf(row + u) * fdk_weight(P, u, nu, fV, beta);
            }
            xs[j] = val;
        }
    }
    __syncthreads();

    const int groups = (nu + FILT_OUT - 1) / FILT_OUT;
    for (int item = threadIdx.x; item < nr * groups; item += FILT_THREADS) {
        const int r = item / groups;
        const int i0 = (item - r * groups) * FILT_OUT;
        const float *xs = sm + (size_t)r * W3 + PADW;  // xs[i] = x_i, i in [-nu-16, 2nu+16)
        float acc[FILT_OUT];
        if (do_filter) {
            float Lw[FILT_OUT + 1], Rw[FILT_OUT + 1];
            // window for k = 1: L[t] = x[i0 + t - 1], R[t] = x[i0 + t + 1]
#pragma unroll
            for (int t = 0; t < FILT_OUT; ++t) {
                acc[t] = 0.5f * xs[i0 + t];
                Lw[t] = xs[i0 + t - 1];
                Rw[t] = xs[i0 + t + 1];
            }
            for (int j = 0; j < nodd; ++j) {
                const float c = taps[j];
#pragma unroll
                for (int t = 0; t < FILT_OUT; ++t) acc[t] = fmaf(c, Lw[t] + Rw[t], acc[t]);
                // advance k by 2: L shifts right by 2 (new x[i0-k-2], x[i0-k-1]),
                // R shifts left by 2 (new x[i0+8+k], x[i0+9+k])
                const int k = 2 * j + 1;
#pragma unroll
                for (int t = FILT_OUT - 1; t >= 2; --t) Lw[t] = Lw[t - 2];
                Lw[1] = xs[i0 - k - 1];
                Lw[0] = xs[i0 - k - 2];
#pragma unroll
                for (int t = 0; t < FILT_OUT - 2; ++t) Rw[t] = Rw[t + 2];
                Rw[FILT_OUT - 2] = xs[i0 + FILT_OUT + k];
                Rw[FILT_OUT - 1] = xs[i0 + FILT_OUT + k + 1];
            }
        } else {
#pragma unroll
            for (int t = 0; t < FILT_OUT; ++t) acc[t] = xs[i0 + t];
        }
        const long long m = m0 + r;
        const int v = (int)(m / na);
        const int a = (int)(m - (long long)v * na);
        T *out = dst + (long long)v * dst_v_stride + (long long)a * dst_row_stride;
#pragma unroll
        for (int t = 0; t < FILT_OUT; ++t)
            if (i0 + t < nu) out[i0 + t] = stf<T>(acc[t]);
    }
}

// Weighted rows filtered with arbitrary taps (any b2t_filter_config other
// than the plain Ram-Lak): y[i] = sum_{d=-(nu-1)}^{nu-1} g[d] x[i - d], taps
// of view a at taps + (per_view ? a : 0) * (2 nu - 1).  Rows staged in
// shared memory as in fdk_weight_filter_kernel (zero-padded by nu + 16 on both
// sides); each thread keeps 8 consecutive outputs and a sliding window of 8
// inputs that moves one column per offset d.
template <typename T>
__global__ void __launch_bounds__(FILT_THREADS) fdk_weight_toeplitz_kernel(
    const T *src, long long src_pitch, int nu, int na, int nv, int rows, FDKWeights P,
    const float *__restrict__ rel_angles, const float *__restrict__ taps, int per_view, T *dst,
    long long dst_row_stride, long long dst_v_stride)
{
    extern __shared__ float sm[];
    const int PADW = nu + 16;
    const int W3 = nu + 2 * PADW;
    const long long m0 = (long long)blockIdx.x * rows;
    const long long mtot = (long long)na * nv;
    const int nr = (int)min((long long)rows, mtot - m0);
    if (nr <= 0) return;
    for (int r = 0; r < nr; ++r) {
        const long long m = m0 + r;
        const int v = (int)(m / na);
        const int a = (int)(m - (long long)v * na);
        const float fV = ((float)v - 0.5f * (float)nv + 0.5f) * P.det_vsize + P.zshift;
        const float beta = P.short_scan ? rel_angles[a] : 0.0f;
        const T *row = src + m * src_pitch;
        float *xs = sm + (size_t)r * W3;
        for (int j = threadIdx.x; j < W3; j += FILT_THREADS) {
            const int u = j - PADW;
            xs[j] = (u >= 0 && u < nu) ? ldf(row + u) * fdk_weight(P, u, nu, fV, beta) : 0.0f;
        }
    }
    __syncthreads();
    const int groups = (nu + FILT_OUT - 1) / FILT_OUT;
    const int ntap = 2 * nu - 1;
    for (int item = threadIdx.x; item < nr * groups; item += FILT_THREADS) {
        const int r = item / groups;
        const int i0 = (item - r * groups) * FILT_OUT;
        const long long m = m0 + r;
        const int v = (int)(m / na);
        const int a = (int)(m - (long long)v * na);
        const float *xs = sm + (size_t)r * W3 + PADW;  // xs[i] = x_i, i in [-nu-16, 2nu+16)
        const float *g = taps + (per_view ? (long long)a * ntap : 0) + (nu - 1);  // g[d], |d| < nu
        float acc[FILT_OUT], w[FILT_OUT];
        // offsets from d = nu - 1 down to -(nu - 1): w[t] = x[i0 + t - d]
#pragma unroll
        for (int t = 0; t < FILT_OUT; ++t) {
            acc[t] = 0.0f;
            w[t] = xs[i0 + t - (nu - 1)];
        }
        for (int d = nu - 1; d >= -(nu - 1); --d) {
            const float c = __ldg(g + d);
#pragma unroll
            for (int t = 0; t < FILT_OUT; ++t) acc[t] = fmaf(c, w[t], acc[t]);
#pragma unroll
            for (int t = 0; t < FILT_OUT - 1; ++t) w[t] = w[t + 1];
            w[FILT_OUT - 1] = xs[i0 + FILT_OUT - d];
        }
        T *out = dst + (long long)v * dst_v_stride + (long long)a * dst_row_stride;
#pragma unroll
        for (int t = 0; t < FILT_OUT; ++t)
            if (i0 + t < nu) out[i0 + t] = stf<T>(acc[t]);
    }
}

}  // namespace

// Weights of FDK_PreWeight (fdk.cu:168-264) for a circular orbit given by its
// source-origin and origin-detector distances, detector pixel sizes, z shift
// and per-view angles; Parker set-up as there (relative angles, scanned range,
// central fan angle), with the reference's float / double mix.
void fdk_weights(float fSrcOrigin, float fDetOrigin, float fZShift, float fDetUSize, float fDetVSize,
                 uint32_t n_angles, uint32_t det_u, const float *angles, int short_scan, FDKWeights &P,
                 std::vector<float> &rel)
{
    P.apply = 1;
    P.central_ray = fSrcOrigin + fDetOrigin;
    P.det_usize = fDetUSize;
    P.det_vsize = fDetVSize;
    P.zshift = fZShift;
    const float fW2 = P.central_ray / (fDetUSize * fSrcOrigin);
    P.W = (float)(P.central_ray * fW2 * (M_PI / 2.0f) / (float)n_angles);
    P.short_scan = 0;
    P.parker_scale = 1.0f;
    P.central_fan = 0.0f;
    rel.clear();
    if (short_scan && n_angles > 1) {
        float fdA = angles[1] - angles[0];
        while (fdA < -M_PI) fdA += 2 * M_PI;
        while (fdA >= M_PI) fdA -= 2 * M_PI;
        float base = (fdA >= 0.0f) ? angles[0] : angles[n_angles - 1];
        rel.resize(n_angles);
        for (uint32_t i = 0; i < n_angles; ++i) {
            float f = angles[i] - base;
            while (f >= 2 * M_PI) f -= 2 * M_PI;
            while (f < 0) f += 2 * M_PI;
            rel[i] = f;
        }
        float range = std::fabs(rel[n_angles - 1] - rel[0]);
        range /= (float)(n_angles - 1);
        range *= (float)n_angles;
        P.parker_scale = (float)(range / M_PI);
        P.central_fan = std::fabs(std::atan(fDetUSize * (det_u * 0.5f) / (fSrcOrigin + fDetOrigin)));
        P.short_scan = 1;
    }
}

// Circular-orbit parameters from view 0 and the per-view angles, exactly as
// FDK() derives them (fdk.cu:425-445).
b2t_status fdk_setup(const b2t_geom3d *g, int short_scan, FDKWeights &P, std::vector<float> &rel)
{
    const b2t_dims3d &d = g->dims;
    const b2t_view3d &p0 = g->views[0];
    float fDetCX = (float)(p0.det_s[0] + 0.5 * d.det_u * p0.det_u[0]);
    float fDetCY = (float)(p0.det_s[1] + 0.5 * d.det_u * p0.det_u[1]);
    float fDetCZ = (float)(p0.det_s[2] + 0.5 * d.det_v * p0.det_v[2]);
    float fSrcOrigin = (float)std::sqrt(p0.src[0] * p0.src[0] + p0.src[1] * p0.src[1]);
    float fDetOrigin = std::sqrt(fDetCX * fDetCX + fDetCY * fDetCY);
    float fDetUSize = (float)std::sqrt(p0.det_u[0] * p0.det_u[0] + p0.det_u[1] * p0.det_u[1]);
    float fDetVSize = (float)std::abs(p0.det_v[2]);
    float fZShift = (float)(fDetCZ - p0.src[2]);
    std::vector<float> angles(d.angles);
    for (uint32_t i = 0; i < d.angles; ++i)
        angles[i] = (float)(-std::atan2(g->views[i].src[0], g->views[i].src[1]) + M_PI);
    fdk_weights(fSrcOrigin, fDetOrigin, fZShift, fDetUSize, fDetVSize, d.angles, d.det_u, angles.data(), short_scan,
                P, rel);
    return B2T_OK;
}

template <typename T>
static b2t_status launch_filter(const void *src, size_t src_pitch, const b2t_dims3d &d, const FDKWeights &P,
                                const float *rel_dev, int do_filter, void *dst, long long dst_row,
                                long long dst_v, cudaStream_t s)
{
    const int nu = d.det_u;
    const size_t row_bytes = sizeof(float) * (3 * (size_t)nu + 32);
    const size_t tap_bytes = sizeof(float) * ((nu + 1) / 2 + 1);
    const size_t budget = 200 * 1024;
    if (row_bytes + tap_bytes > budget)
        return fail(B2T_ERR_UNSUPPORTED, "FDK filter: detector rows of %d pixels exceed shared memory", nu);
    int rows = (int)((budget - tap_bytes) / row_bytes);
    if (rows > 8) rows = 8;
    const size_t smem = rows * row_bytes + tap_bytes;
    auto kern = fdk_weight_filter_kernel<T>;
    B2T_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "FDK filter smem attribute");
    const long long mtot = (long long)d.angles * d.det_v;
    const long long blocks = (mtot + rows - 1) / rows;
    if (blocks > 0x7fffffffLL) return fail(B2T_ERR_UNSUPPORTED, "FDK filter: too many rows");
    kern<<<(unsigned)blocks, FILT_THREADS, smem, s>>>(static_cast<const T *>(src), (long long)src_pitch, nu,
                                                      d.angles, d.det_v, rows, P, rel_dev, do_filter,
                                                      static_cast<T *>(dst), dst_row, dst_v);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "FDK weight/filter launch");
    return B2T_OK;
}

static b2t_status validate_filter(const b2t_filter_config *filter, const char *who)
{
    if (filter && (filter->type < B2T_FILTER_NONE || filter->type > B2T_FILTER_RSINOGRAM))
        return fail(B2T_ERR_INVALID_ARG, "%s: unknown filter type %d", who, filter->type);
    return B2T_OK;
}

template <typename T>
static b2t_status launch_toeplitz(const void *src, size_t src_pitch, const b2t_dims3d &d, const FDKWeights &P,
                                  const float *rel_dev, const float *taps, int per_view, void *dst, long long dst_row,
                                  long long dst_v, cudaStream_t s)
{
    const int nu = d.det_u;
    const size_t row_bytes = sizeof(float) * (3 * (size_t)nu + 32);
    const size_t budget = 200 * 1024;
    if (row_bytes > budget)
        return fail(B2T_ERR_UNSUPPORTED, "filter: detector rows of %d pixels exceed shared memory", nu);
    int rows = (int)(budget / row_bytes);
    if (rows > 8) rows = 8;
    const size_t smem = rows * row_bytes;
    auto kern = fdk_weight_toeplitz_kernel<T>;
    B2T_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "filter smem attribute");
    const long long mtot = (long long)d.angles * d.det_v;
    const long long blocks = (mtot + rows - 1) / rows;
    if (blocks > 0x7fffffffLL) return fail(B2T_ERR_UNSUPPORTED, "filter: too many rows");
    kern<<<(unsigned)blocks, FILT_THREADS, smem, s>>>(static_cast<const T *>(src), (long long)src_pitch, nu,
                                                      d.angles, d.det_v, rows, P, rel_dev, taps, per_view,
                                                      static_cast<T *>(dst), dst_row, dst_v);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "filter launch");
    return B2T_OK;
}

template <typename T>
static b2t_status launch_split(const void *src, size_t src_pitch, const b2t_dims3d &d, const FDKWeights &P,
                               const float *rel_dev, __nv_bfloat16 *a, int khp, long long M, void *dst,
                               long long dst_row, long long dst_v, int blocks, size_t smem, cudaStream_t s)
{
    auto kern = fdk_split_kernel<T>;
    B2T_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "ramp filter split smem attribute");
    kern<<<blocks, SPLIT_THREADS, smem, s>>>(static_cast<const T *>(src), (long long)src_pitch, (int)d.det_u,
                                             (int)d.angles, (int)d.det_v, P, rel_dev, a, khp, M,
                                             static_cast<T *>(dst), dst_row, dst_v);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "ramp filter split launch");
    return B2T_OK;
}

static b2t_status run_filter(const b2t_dims3d &d, const FDKWeights &P, const std::vector<float> &rel,
                             const b2t_filter_config *filter,
                             const void *src, size_t src_pitch, void *dst, long long dst_row, long long dst_v,
                             int32_t dtype, cudaStream_t s)
{
    Scratch rs;
    const float *rel_dev = nullptr;
    if (!rel.empty()) {
        B2T_TRY(rs.alloc(sizeof(float) * rel.size(), s, "Parker angles"));
        B2T_CUDA_TRY(cudaMemcpyAsync(rs.as<void>(), rel.data(), sizeof(float) * rel.size(), cudaMemcpyHostToDevice, s),
                     "Parker angles upload");
        rel_dev = rs.as<float>();
    }
    const int ftype = filter ? filter->type : B2T_FILTER_RAMLAK;
    if (ftype != B2T_FILTER_NONE && !filter_is_plain_ramlak(filter)) {
        // any other filter: its exact spatial taps (filters.cpp), SIMT Toeplitz
        FilterTaps ft;
        B2T_TRY(filter_taps(filter, d.det_u, d.angles, ft));
        Scratch ts;
        B2T_TRY(ts.alloc(sizeof(float) * ft.g.size(), s, "filter taps"));
        B2T_CUDA_TRY(cudaMemcpyAsync(ts.as<void>(), ft.g.data(), sizeof(float) * ft.g.size(), cudaMemcpyHostToDevice,
                                     s),
                     "filter taps upload");
        const int per_view = ft.nsets > 1 ? 1 : 0;
        if (dtype == B2T_F32)
            return launch_toeplitz<float>(src, src_pitch, d, P, rel_dev, ts.as<float>(), per_view, dst, dst_row, dst_v, s);
        if (dtype == B2T_F16)
            return launch_toeplitz<__half>(src, src_pitch, d, P, rel_dev, ts.as<float>(), per_view, dst, dst_row, dst_v,
                                           s);
        return launch_toeplitz<__nv_bfloat16>(src, src_pitch, d, P, rel_dev, ts.as<float>(), per_view, dst, dst_row,
                                              dst_v, s);
    }
    const int do_filter = (ftype == B2T_FILTER_RAMLAK) ? 1 : 0;
    // Ram-Lak on the tensor cores (ramp_tc.cu) when the shape allows it and
    // its scratch fits; otherwise the SIMT Toeplitz kernel below
    RampTCPlan plan;
    const long long M = (long long)d.angles * d.det_v;
    if (do_filter && ramp_tc_enabled() && ramp_tc_plan(d.det_u, M, plan)) {
        Scratch sa, sb;
        b2t_status st = sa.alloc(plan.a_elems * sizeof(__nv_bfloat16), s, "ramp filter split rows");
        if (st == B2T_OK) st = sb.alloc(plan.b_elems * sizeof(__nv_bfloat16), s, "ramp filter taps");
        if (st == B2T_OK) {
            __nv_bfloat16 *a = sa.as<__nv_bfloat16>();
            const long long blocks = (M + SPLIT_ROWS - 1) / SPLIT_ROWS;
            const size_t wrow = (size_t)d.det_u + 2 * RAMP_TC_BAND + 12;  // PADL + nu + PADR
            const size_t smem = sizeof(float) * SPLIT_ROWS * (wrow + wrow / 8 + 1);
            if (blocks > 0x7fffffffLL || smem > 200 * 1024)
                return fail(B2T_ERR_UNSUPPORTED, "ramp filter: %lld rows of %u columns are too many", M, d.det_u);
            if (dtype == B2T_F32)
                st = launch_split<float>(src, src_pitch, d, P, rel_dev, a, plan.khp, M, dst, dst_row, dst_v,
                                         (int)blocks, smem, s);
            else if (dtype == B2T_F16)
                st = launch_split<__half>(src, src_pitch, d, P, rel_dev, a, plan.khp, M, dst, dst_row, dst_v,
                                          (int)blocks, smem, s);
            else
                st = launch_split<__nv_bfloat16>(src, src_pitch, d, P, rel_dev, a, plan.khp, M, dst, dst_row,
                                                 dst_v, (int)blocks, smem, s);
            if (st != B2T_OK) return st;
            return ramp_tc_filter(plan, a, sb.as<__nv_bfloat16>(), dst, dst_row, dst_v, (int)d.angles, dtype, s);
        }
        if (st != B2T_ERR_NO_MEMORY) return st;
        clear_error();  // not enough memory for the split operands: SIMT filter
    }
    if (dtype == B2T_F32) return launch_filter<float>(src, src_pitch, d, P, rel_dev, do_filter, dst, dst_row, dst_v, s);
    if (dtype == B2T_F16) return launch_filter<__half>(src, src_pitch, d, P, rel_dev, do_filter, dst, dst_row, dst_v, s);
    return launch_filter<__nv_bfloat16>(src, src_pitch, d, P, rel_dev, do_filter, dst, dst_row, dst_v, s);
}

b2t_status filter_rows_impl(float *data, size_t nrows, uint32_t n, size_t pitch, const b2t_filter_config *filter,
                            cudaStream_t s)
{
    if (!data) return fail(B2T_ERR_INVALID_ARG, "b2t_filter_rows: null data");
    B2T_TRY(validate_filter(filter, "b2t_filter_rows"));
    if (n == 0 || nrows == 0) return B2T_OK;
    if (nrows > 0xffffffffu) return fail(B2T_ERR_INVALID_ARG, "b2t_filter_rows: too many rows");
    if (pitch == 0) pitch = n;
    if (pitch < n) return fail(B2T_ERR_INVALID_ARG, "b2t_filter_rows: pitch below row length");
    b2t_dims3d d{};
    d.det_u = n;
    d.angles = (uint32_t)nrows;
    d.det_v = 1;
    FDKWeights P{};
    P.apply = 0;
    std::vector<float> rel;
    return run_filter(d, P, rel, filter, data, pitch, data, (long long)pitch, (long long)pitch * nrows, B2T_F32, s);
}

// getFanParameters (src/GeometryUtil2D.cpp:134-178): circular fan parameters
// of one view; false if the view is not a circular fan.
static bool fan_parameters(const b2t_view2d &p, uint32_t ndet, float &angle, float &src_origin, float &origin_det,
                           float &det_size)
{
    double dp = p.src[0] * p.det_u[0] + p.src[1] * p.det_u[1];
    double rel = std::sqrt(((double)p.src[0] * p.src[0] + (double)p.src[1] * p.src[1]) *
                           ((double)p.det_u[0] * p.det_u[0] + (double)p.det_u[1] * p.det_u[1]));
    if (std::abs(dp) > rel * 0.0001) return false;
    src_origin = (float)std::sqrt((double)p.src[0] * p.src[0] + (double)p.src[1] * p.src[1]);
    det_size = (float)std::sqrt((double)p.det_u[0] * p.det_u[0] + (double)p.det_u[1] * p.det_u[1]);
    double t = (-(double)p.det_s[0]) * p.det_u[0] + (-(double)p.det_s[1]) * p.det_u[1];
    t /= ((double)p.det_u[0] * p.det_u[0] + (double)p.det_u[1] * p.det_u[1]);
    origin_det = (float)std::sqrt((p.det_s[0] + t * p.det_u[0]) * (p.det_s[0] + t * p.det_u[0]) +
                                  (p.det_s[1] + t * p.det_u[1]) * (p.det_s[1] + t * p.det_u[1]));
    angle = (float)std::atan2((double)p.det_u[1], (double)p.det_u[0]);
    (void)ndet;
    return true;
}

// FBP_CUDA (cuda/2d/fbp.cu:77-190): parallel = Ram-Lak filter + BP scaled by
// (pi/2)/n_angles; fan = FDK pre-weighting of a one-row cone (+ Parker) +
// filter + fan BP with the FBP weighting.  sino is not modified.
b2t_status fbp2d_impl(const b2t_geom2d *g, const b2t_filter_config *filter, int32_t short_scan, const float *sino,
                      size_t sino_pitch,
                      float *vol, size_t vol_pitch, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate2d(g, "b2t_fbp2d"));
    if (!sino || !vol) return fail(B2T_ERR_INVALID_ARG, "b2t_fbp2d: null data pointer");
    B2T_TRY(validate_filter(filter, "b2t_fbp2d"));
    const b2t_dims2d &dm = g->dims;
    if (sino_pitch == 0) sino_pitch = dm.dets;
    if (sino_pitch < dm.dets) return fail(B2T_ERR_INVALID_ARG, "b2t_fbp2d: pitch below row length");
    b2t_dims3d d{};
    d.det_u = dm.dets;
    d.angles = dm.angles;
    d.det_v = 1;
    FDKWeights P{};
    P.apply = 0;
    std::vector<float> rel;
    b2t_geom2d q = *g;
    if (g->kind == B2T_GEOM_FAN2D) {
        std::vector<float> angles(dm.angles);
        float fs = 0, fd = 0, du = 0;
        for (uint32_t i = 0; i < dm.angles; ++i)
            if (!fan_parameters(g->views[i], dm.dets, angles[i], fs, fd, du))
                return fail(B2T_ERR_UNSUPPORTED, "b2t_fbp2d: view %u is not a circular fan beam", i);
        fdk_weights(fs, fd, 0.0f, du, 1.0f, dm.angles, dm.dets, angles.data(), short_scan, P, rel);
    } else {
        q.output_scale = (float)(q.output_scale * ((M_PI / 2.0f) / (float)dm.angles));
    }
    Scratch tmp;
    B2T_TRY(tmp.alloc(sizeof(float) * (size_t)dm.angles * dm.dets, s, "b2t_fbp2d scratch"));
    B2T_TRY(run_filter(d, P, rel, filter, sino, sino_pitch, tmp.as<void>(), (long long)dm.dets,
                       (long long)dm.dets * dm.angles, B2T_F32, s));
    return bp2d_impl(&q, 1, g->kind == B2T_GEOM_FAN2D ? 1 : 0, tmp.as<float>(), dm.dets, vol, vol_pitch, mode, s);
}

static b2t_status run_weight_filter(const b2t_geom3d *g, const b2t_filter_config *filter, int short_scan, const void *src,
                                    size_t src_pitch, void *dst, long long dst_row, long long dst_v, int32_t dtype,
                                    cudaStream_t s)
{
    FDKWeights P;
    std::vector<float> rel;
    B2T_TRY(fdk_setup(g, short_scan, P, rel));
    return run_filter(g->dims, P, rel, filter, src, src_pitch, dst, dst_row, dst_v, dtype, s);
}

static b2t_status validate_fdk(const b2t_geom3d *g, const b2t_filter_config *filter, int32_t dtype, const char *who)
{
    B2T_TRY(validate3d(g, who));
    if (g->kind != B2T_GEOM_CONE) return fail(B2T_ERR_UNSUPPORTED, "%s: FDK needs a cone geometry", who);
    B2T_TRY(validate_filter(filter, who));
    if (!dtype_valid(dtype)) return fail(B2T_ERR_INVALID_ARG, "%s: bad dtype %d", who, dtype);
    return B2T_OK;
}

b2t_status fdk_weight_filter_views(const b2t_geom3d *g, uint32_t a0, uint32_t n, const b2t_filter_config *filter,
                                   int32_t short_scan, const float *src, size_t src_pitch, float *dst,
                                   long long dst_row, long long dst_v, cudaStream_t s)
{
    B2T_TRY(validate_fdk(g, filter, B2T_F32, "FDK views"));
    if (a0 + n > g->dims.angles || n == 0) return fail(B2T_ERR_INVALID_ARG, "FDK views: range outside the scan");
    const int ftype = filter ? filter->type : B2T_FILTER_RAMLAK;
    if ((ftype == B2T_FILTER_SINOGRAM || ftype == B2T_FILTER_RSINOGRAM) && n != g->dims.angles)
        return fail(B2T_ERR_UNSUPPORTED, "FDK views: per-view custom filters need all views at once");
    FDKWeights P;
    std::vector<float> rel;
    B2T_TRY(fdk_setup(g, short_scan, P, rel));
    std::vector<float> sub;
    if (!rel.empty()) sub.assign(rel.begin() + a0, rel.begin() + a0 + n);
    b2t_dims3d d = g->dims;
    d.angles = n;
    return run_filter(d, P, sub, filter, src, src_pitch, dst, dst_row, dst_v, B2T_F32, s);
}

b2t_status fdk_weight_filter_impl(const b2t_geom3d *g, const b2t_filter_config *filter, int32_t short_scan, void *proj,
                                  size_t proj_pitch, int32_t dtype, cudaStream_t s)
{
    B2T_TRY(validate_fdk(g, filter, dtype, "b2t_fdk_weight_filter"));
    if (!proj) return fail(B2T_ERR_INVALID_ARG, "b2t_fdk_weight_filter: null projections");
    const b2t_dims3d &d = g->dims;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (proj_pitch < d.det_u) return fail(B2T_ERR_INVALID_ARG, "b2t_fdk_weight_filter: pitch below row length");
    // rows are loaded into shared memory before any is written: in place is safe
    return run_weight_filter(g, filter, short_scan, proj, proj_pitch, proj, (long long)proj_pitch,
                             (long long)proj_pitch * d.angles, dtype, s);
}

b2t_status fdk_impl(const b2t_geom3d *g, const b2t_filter_config *filter, int32_t short_scan, float output_scale,
                    const void *proj,
                    size_t proj_pitch, void *vol, size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate_fdk(g, filter, dtype, "b2t_fdk"));
    if (!proj || !vol) return fail(B2T_ERR_INVALID_ARG, "b2t_fdk: null data pointer");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_fdk: bad mode");
    const b2t_dims3d &d = g->dims;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    if (proj_pitch < d.det_u || vol_pitch < d.vol_x) return fail(B2T_ERR_INVALID_ARG, "b2t_fdk: pitch below row length");
    b2t_params3d p;
    p.det_supersample = 1;
    p.voxel_supersample = 1;
    p.output_scale = output_scale;
    p.kernel = B2T_KER_FDK_WEIGHTING;
    const bool pairs = bp_pairs(dtype, &p);
    Scratch sp;
    const size_t bytes = padded_proj_bytes(d, dtype, pairs);
    B2T_TRY(sp.alloc(bytes, s, "b2t_fdk scratch (filtered projections)"));
    if (pairs) {
        // 16-bit pair layout (each element holds a texel and the one below
        // it): filtered rows into a texel buffer, then paired
        Scratch st;
        B2T_TRY(st.alloc((size_t)d.det_u * d.angles * d.det_v * dtype_size(dtype), s,
                         "b2t_fdk scratch (filtered rows)"));
        B2T_TRY(run_weight_filter(g, filter, short_scan, proj, proj_pitch, st.as<void>(), (long long)d.det_u,
                                  (long long)d.det_u * d.angles, dtype, s));
        B2T_TRY(pad_projections_impl(st.as<void>(), d.det_u, d, sp.as<void>(), dtype, true, s));
    } else {
        // filtered projections straight into the zero-padded BP input
        B2T_CUDA_TRY(cudaMemsetAsync(sp.as<void>(), 0, bytes, s), "b2t_fdk memset");
        const long long pu = (long long)padded_pu(d.det_u), pv = pu * d.angles;
        char *interior = sp.as<char>() + (2 * pv + 2) * (long long)dtype_size(dtype);
        B2T_TRY(run_weight_filter(g, filter, short_scan, proj, proj_pitch, interior, pu, pv, dtype, s));
    }
    return bp3d_from_padded(g, &p, sp.as<void>(), vol, vol_pitch, dtype, mode, s);
}

}  // namespace b2t
