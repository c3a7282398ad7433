// Exact adjoint of the forward projector (projection kernel "matched_bp").
//
// The reference has a matched backprojector only for cyl_cone_vec
// (cuda/3d/cone_cyl.cu:309-470, dispatched in cuda/3d/mem3d.cu:463-479): each
// ray scatters its value back along the samples its forward projector read,
// with atomic adds.  This module provides the same construction for the
// flat-panel cone and parallel geometries: the transpose of fp3d_kernel,
// sample for sample, so <A x, y> = <x, A^T y> holds to rounding.
//
// Layout: each marching direction scatters into a zero-padded FP32
// accumulation volume with the same layout its forward pass reads (xyz copy
// for y/z-major views, zxy copy for x-major views); a final pass drops the
// padding, folds the two accumulators and applies SET/ADD.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <vector>

#include "b2t_internal.h"
#include "proj3d.h"

namespace b2t {

namespace {

template <typename T> __device__ __forceinline__ float ldm(const T *p);
template <> __device__ __forceinline__ float ldm<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ldm<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ldm<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(__ldg(p));
}
template <typename T> __device__ __forceinline__ float ldm_plain(const T *p);
template <> __device__ __forceinline__ float ldm_plain<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float ldm_plain<__half>(const __half *p) { return __half2float(*p); }
template <> __device__ __forceinline__ float ldm_plain<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(*p);
}
template <typename T> __device__ __forceinline__ T tom(float v);
template <> __device__ __forceinline__ float tom<float>(float v) { return v; }
template <> __device__ __forceinline__ __half tom<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 tom<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ void clip_slices_m(float A, float B, float lo, float hi, float &smin, float &smax)
{
    if (fabsf(A) < 1e-12f) {
        if (!(B >= lo && B <= hi)) {
            smin = 1.0f;
            smax = 0.0f;
        }
        return;
    }
    float s1 = (lo - B) / A, s2 = (hi - B) / A;
    smin = fmaxf(smin, fminf(s1, s2));
    smax = fminf(smax, fmaxf(s1, s2));
}

// The forward projectors' split (fp3d_col_kernel, fp3d_cell_kernel, fp3d_kernel): sample
// position plus one half qh = A s + (B + 1/2); texel floor(qh) by rounding
// down, weight qh - floor(qh).  Identical arithmetic keeps the transpose exact.
constexpr float SPLIT_M = 12582912.0f;  // 1.5 * 2^23
__device__ __forceinline__ void split_floor_m(float qh, int &k, float &f)
{
    const float t = __fadd_rd(qh, SPLIT_M);
    k = __float_as_int(t) - 0x4B400000;
    f = qh - (t - SPLIT_M);
}

__device__ __forceinline__ bool texel_ok_m(float A, float Bh, int s, int n)
{
    int k;
    float f;
    split_floor_m(fmaf(A, (float)s, Bh), k, f);
    return k >= -2 && k <= n;
}

// Transpose of fp3d_kernel: L.vol is the FP32 padded accumulator (written),
// L.proj the input projections.  Same ray set-up, same slice range, same
// weights; the four bilinear taps are scattered with atomic adds.
template <typename T>
__global__ void __launch_bounds__(256) fp3d_transpose_kernel(const __grid_constant__ FPLaunch L)
{
    const FPView &V = L.views[blockIdx.x];
    const int u = blockIdx.y * 32 + threadIdx.x;
    const int v = blockIdx.z * 8 + threadIdx.y;
    if (u >= L.nu || v >= L.nv) return;
    float *acc = const_cast<float *>(static_cast<const float *>(L.vol));
    const T *pin = static_cast<const T *>(L.proj) + ((size_t)v * L.na + V.a) * L.proj_pitch + u;
    float val = ldm(pin);
    if (val == 0.0f) return;
    const int R = L.rays;
    if (R > 1) val /= (float)(R * R);
    const long long st0 = L.st0, st2 = L.st2;
    const float n0 = (float)L.n0;
    for (int iu = 0; iu < R; ++iu) {
        for (int iv = 0; iv < R; ++iv) {
            float uu = (float)u + 0.5f - 0.5f * (float)L.nu;
            float vv = (float)v + 0.5f - 0.5f * (float)L.nv;
            if (R > 1) {
                uu += -0.5f + (0.5f + (float)iu) / (float)R;
                vv += -0.5f + (0.5f + (float)iv) / (float)R;
            }
            const float den = fmaf(vv, V.e[2], fmaf(uu, V.e[1], V.e[0]));
            const float inv = 1.0f / den;
            const float A1 = fmaf(vv, V.m1[2], fmaf(uu, V.m1[1], V.m1[0])) * inv;
            const float A2 = fmaf(vv, V.m2[2], fmaf(uu, V.m2[1], V.m2[0])) * inv;
            const float B1 = fmaf(vv, V.n1[2], fmaf(uu, V.n1[1], V.n1[0])) * inv;
            const float B2 = fmaf(vv, V.n2[2], fmaf(uu, V.n2[1], V.n2[0])) * inv;
            float smin = 0.0f, smax = n0 - 1.0f;
            clip_slices_m(A1, B1, -1.6f, (float)L.n1 - 0.4f, smin, smax);
            clip_slices_m(A2, B2, -1.6f, (float)L.n2 - 0.4f, smin, smax);
            int s_lo = max(0, (int)ceilf(fmaxf(smin, -1.0f)));
            int s_hi = min(L.n0 - 1, (int)floorf(fminf(smax, n0)));
            const float B1h = B1 + 0.5f, B2h = B2 + 0.5f;
            for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
                if (texel_ok_m(A1, B1h, s_lo, L.n1) && texel_ok_m(A2, B2h, s_lo, L.n2)) break;
                ++s_lo;
            }
            for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
                if (texel_ok_m(A1, B1h, s_hi, L.n1) && texel_ok_m(A2, B2h, s_hi, L.n2)) break;
                --s_hi;
            }
            if (!(texel_ok_m(A1, B1h, s_lo, L.n1) && texel_ok_m(A2, B2h, s_lo, L.n2) &&
                  texel_ok_m(A1, B1h, s_hi, L.n1) && texel_ok_m(A2, B2h, s_hi, L.n2)))
                s_hi = s_lo - 1;
            const float sc = sqrtf(fmaf(A1 * A1, L.f1, fmaf(A2 * A2, L.f2, 1.0f))) * L.mul;
            const float w = val * sc;
            for (int s = s_lo; s <= s_hi; ++s) {
                int k1, k2;
                float f1, f2;
                split_floor_m(fmaf(A1, (float)s, B1h), k1, f1);
                split_floor_m(fmaf(A2, (float)s, B2h), k2, f2);
                float *p = acc + (long long)s * st0 + (long long)k2 * st2 + k1;
                const float g1 = 1.0f - f1, g2 = 1.0f - f2;
                atomicAdd(p, g1 * g2 * w);
                atomicAdd(p + 1, f1 * g2 * w);
                atomicAdd(p + st2, g1 * f2 * w);
                atomicAdd(p + st2 + 1, f1 * f2 * w);
            }
        }
    }
}

__device__ __forceinline__ void red_add_v4(float4 *p, float a, float b, float c, float d)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

// Transpose of the forward projector for x- and y-major views, in the cell
// space of its columns layout: a sample with base texel (k1, k2) at slice s
// adds its four bilinear taps (weights of corners (k1, k2), (k1 + 1, k2),
// (k1, k2 + 1), (k1 + 1, k2 + 1)) to the 16-byte accumulator of cell
// (k1, s, k2), one vector reduction per sample instead of four scalar
// atomics; fold_cells then gathers each voxel's taps from the four cells
// around it.  A warp takes 32 rows of one detector column, so its
// reductions fall on a few contiguous lines.  L.vol is the accumulator's
// first cell (j1 = j2 = 0), index (j1 n0 + s) (n2 + 4) + j2, j = k + 2.
template <typename T, bool AGG>
__global__ void __launch_bounds__(256) fp3d_transpose_cols_kernel(const __grid_constant__ FPLaunch L)
{
    const FPView &V = L.views[blockIdx.x];
    const int v = blockIdx.z * 32 + threadIdx.x;
    const int u = blockIdx.y * 8 + threadIdx.y;
    const int lane = threadIdx.x;
    const bool inside = u < L.nu && v < L.nv;
    if (!AGG && !inside) return;
    float4 *cacc = static_cast<float4 *>(const_cast<void *>(L.vol));
    float val = 0.0f;
    if (inside) val = ldm(static_cast<const T *>(L.proj) + ((size_t)v * L.na + V.a) * L.proj_pitch + u);
    if (!AGG && val == 0.0f) return;
    const bool live = inside && val != 0.0f;
    const int R = L.rays;
    if (R > 1) val /= (float)(R * R);
    const float n0 = (float)L.n0;
    const long long m2 = L.n2 + 4;
    for (int iu = 0; iu < R; ++iu) {
        for (int iv = 0; iv < R; ++iv) {
            float uu = (float)u + 0.5f - 0.5f * (float)L.nu;
            float vv = (float)v + 0.5f - 0.5f * (float)L.nv;
            if (R > 1) {
                uu += -0.5f + (0.5f + (float)iu) / (float)R;
                vv += -0.5f + (0.5f + (float)iv) / (float)R;
            }
            const float den = fmaf(vv, V.e[2], fmaf(uu, V.e[1], V.e[0]));
            const float inv = 1.0f / den;
            const float A1 = fmaf(vv, V.m1[2], fmaf(uu, V.m1[1], V.m1[0])) * inv;
            const float A2 = fmaf(vv, V.m2[2], fmaf(uu, V.m2[1], V.m2[0])) * inv;
            const float B1 = fmaf(vv, V.n1[2], fmaf(uu, V.n1[1], V.n1[0])) * inv;
            const float B2 = fmaf(vv, V.n2[2], fmaf(uu, V.n2[1], V.n2[0])) * inv;
            float smin = 0.0f, smax = n0 - 1.0f;
            clip_slices_m(A1, B1, -1.6f, (float)L.n1 - 0.4f, smin, smax);
            clip_slices_m(A2, B2, -1.6f, (float)L.n2 - 0.4f, smin, smax);
            int s_lo = max(0, (int)ceilf(fmaxf(smin, -1.0f)));
            int s_hi = min(L.n0 - 1, (int)floorf(fminf(smax, n0)));
            const float B1h = B1 + 0.5f, B2h = B2 + 0.5f;
            for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
                if (texel_ok_m(A1, B1h, s_lo, L.n1) && texel_ok_m(A2, B2h, s_lo, L.n2)) break;
                ++s_lo;
            }
            for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
                if (texel_ok_m(A1, B1h, s_hi, L.n1) && texel_ok_m(A2, B2h, s_hi, L.n2)) break;
                --s_hi;
            }
            if (!(texel_ok_m(A1, B1h, s_lo, L.n1) && texel_ok_m(A2, B2h, s_lo, L.n2) &&
                  texel_ok_m(A1, B1h, s_hi, L.n1) && texel_ok_m(A2, B2h, s_hi, L.n2)))
                s_hi = s_lo - 1;
            const float sc = sqrtf(fmaf(A1 * A1, L.f1, fmaf(A2 * A2, L.f2, 1.0f))) * L.mul;
            const float w = val * sc;
            if constexpr (!AGG) {
                for (int s = s_lo; s <= s_hi; ++s) {
                    int k1, k2;
                    float f1, f2;
                    split_floor_m(fmaf(A1, (float)s, B1h), k1, f1);
                    split_floor_m(fmaf(A2, (float)s, B2h), k2, f2);
                    const float g1 = 1.0f - f1, g2 = 1.0f - f2;
                    red_add_v4(cacc + ((long long)(k1 + 2) * L.n0 + s) * m2 + (k2 + 2), g1 * g2 * w,
                               f1 * g2 * w, g1 * f2 * w, f1 * f2 * w);
                }
            } else {
                // The warp's rays (consecutive rows of one column) walk one
                // common slice range; at each slice, neighbouring lanes whose
                // samples share a cell (about 1.5 rays per cell) merge: the
                // head of a run of equal cells adds the taps of the lane after
                // it, which then skips its reduction; later lanes of longer
                // runs reduce on their own.  Lanes without a sample carry
                // distinct keys that match nothing.
                if (!live) {
                    s_lo = 1;
                    s_hi = 0;
                }
                const int S0 = __reduce_min_sync(0xffffffffu, s_lo <= s_hi ? s_lo : 0x7fffffff);
                const int S1 = __reduce_max_sync(0xffffffffu, s_lo <= s_hi ? s_hi : -1);
                for (int s = S0; s <= S1; ++s) {
                    const bool in = s >= s_lo && s <= s_hi;
                    uint32_t key = 0xffffffffu - (uint32_t)lane;
                    float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f, t3 = 0.0f;
                    if (in) {
                        int k1, k2;
                        float f1, f2;
                        split_floor_m(fmaf(A1, (float)s, B1h), k1, f1);
                        split_floor_m(fmaf(A2, (float)s, B2h), k2, f2);
                        const float g1 = 1.0f - f1, g2 = 1.0f - f2;
                        key = ((uint32_t)(k1 + 2) * (uint32_t)L.n0 + (uint32_t)s) * (uint32_t)m2 + (uint32_t)(k2 + 2);
                        t0 = g1 * g2 * w;
                        t1 = f1 * g2 * w;
                        t2 = g1 * f2 * w;
                        t3 = f1 * f2 * w;
                    }
                    const uint32_t kp = __shfl_up_sync(0xffffffffu, key, 1);
                    const uint32_t kp2 = __shfl_up_sync(0xffffffffu, key, 2);
                    const uint32_t kn = __shfl_down_sync(0xffffffffu, key, 1);
                    const float n0v = __shfl_down_sync(0xffffffffu, t0, 1);
                    const float n1v = __shfl_down_sync(0xffffffffu, t1, 1);
                    const float n2v = __shfl_down_sync(0xffffffffu, t2, 1);
                    const float n3v = __shfl_down_sync(0xffffffffu, t3, 1);
                    const bool head = lane == 0 || kp != key;
                    const bool second = !head && (lane == 1 || kp2 != key);
                    if (in && !second) {
                        if (head && lane < 31 && kn == key) {
                            t0 += n0v;
                            t1 += n1v;
                            t2 += n2v;
                            t3 += n3v;
                        }
                        red_add_v4(cacc + key, t0, t1, t2, t3);
                    }
                }
            }
        }
    }
}

// out[z][y][x] (=|+=) the x-major cell taps C0 (k1 = y, s = x, k2 = z), the
// y-major cell taps C1 (k1 = x, s = y, k2 = z) and the z-major padded
// accumulator accA[z+2][y+2][x+2]; a voxel's taps are .x of its own cell,
// .y of the cell before it along k1, .z before it along k2, .w before both.
// Threads run along z, the cells' contiguous axis.
// Views of the slab transpose (fp3d_slab.cu) come as plain FP32 sums per
// voxel in its accumulators m0 (x-major: cell (x, y, z) at (x ay0 + y + 2)
// az + z + 2) and m1 (y-major: (y ay1 + x + 2) az + z + 2).
template <typename T>
__global__ void fold_cells(const float4 *__restrict__ c0, const float4 *__restrict__ c1,
                           const float *__restrict__ accA, const float *__restrict__ m0,
                           const float *__restrict__ m1, long long ay0, long long ay1, long long az, int nx, int ny,
                           int nz, T *__restrict__ out, size_t pitch, int accumulate)
{
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    const int y = blockIdx.z;
    if (z >= nz) return;
    const long long m2 = nz + 4;
    float r = 0.0f;
    auto taps = [&](const float4 *c, long long j1, long long n0, long long sl) {
        const float4 *p = c + (j1 * n0 + sl) * m2 + (z + 2);  // cell (k1, s, k2 = z)
        const float4 *q = p - n0 * m2;                        // k1 - 1
        r += p->x + q->y + (p - 1)->z + (q - 1)->w;
    };
    if (c0) taps(c0, y + 2, nx, x);
    if (c1) taps(c1, x + 2, ny, y);
    if (accA) r += accA[((size_t)(z + 2) * (ny + 4) + (y + 2)) * (nx + 4) + (x + 2)];
    if (m0) r += m0[((long long)x * ay0 + y + 2) * az + z + 2];
    if (m1) r += m1[((long long)y * ay1 + x + 2) * az + z + 2];
    T *o = out + ((size_t)z * ny + y) * pitch + x;
    if (accumulate) r += ldm_plain(o);
    *o = tom<T>(r);
}

// out[z][y][x] (=|+=) accA[z+2][y+2][x+2] + accB[z+2][x+2][y+2]
template <typename T>
__global__ void fold_accumulators(const float *__restrict__ accA, const float *__restrict__ accB, int nx,
                                  int ny, int nz, T *__restrict__ out, size_t pitch, int accumulate)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= nx) return;
    const size_t px = nx + 4, py = ny + 4;
    float r = 0.0f;
    if (accA) r += accA[((size_t)(z + 2) * py + (y + 2)) * px + (x + 2)];
    if (accB) r += accB[((size_t)(z + 2) * px + (x + 2)) * py + (y + 2)];
    T *o = out + ((size_t)z * ny + y) * pitch + x;
    if (accumulate) r += ldm_plain(o);
    *o = tom<T>(r);
}

// B2T_MATCHED_PLAIN=1 selects the per-lane reductions of
// fp3d_transpose_cols_kernel (the path of arrays of 2^32 cells or more)
// instead of the merged ones (same sums, another order; tests compare them).
std::atomic<unsigned long long> g_scatter_launches{0};

bool matched_force_plain()
{
    const char *e = getenv("B2T_MATCHED_PLAIN");
    return e && e[0] == '1';
}

template <typename T> b2t_status launch_T(const FPLaunch &L, dim3 grid, cudaStream_t s)
{
    fp3d_transpose_kernel<T><<<grid, dim3(32, 8), 0, s>>>(L);
    count_launches(1);
    g_scatter_launches.fetch_add(1);
    B2T_CUDA_TRY(cudaGetLastError(), "matched bp kernel launch");
    return B2T_OK;
}

template <typename T>
b2t_status launch_fold(const float *a, const float *b, const b2t_dims3d &d, void *vol, size_t pitch,
                       int accumulate, cudaStream_t s)
{
    dim3 grid((d.vol_x + 127) / 128, d.vol_y, d.vol_z);
    fold_accumulators<T><<<grid, 128, 0, s>>>(a, b, d.vol_x, d.vol_y, d.vol_z, static_cast<T *>(vol), pitch,
                                               accumulate);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "matched bp fold launch");
    return B2T_OK;
}

}  // namespace

unsigned long long matched_scatter_launches_take() { return g_scatter_launches.exchange(0); }

b2t_status matched_bp3d_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *proj,
                             size_t proj_pitch, void *vol, size_t vol_pitch, int32_t dtype,
                             int32_t mode, cudaStream_t s)
{
    const b2t_dims3d &d = g->dims;
    if (p->det_supersample == 0 || p->det_supersample > 16)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d(matched): detector supersampling must be 1..16");
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (vol_pitch < d.vol_x || proj_pitch < d.det_u)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d(matched): pitch below row length");
    std::vector<int> dirs(d.angles);
    bool need[3] = {false, false, false};
    for (uint32_t a = 0; a < d.angles; ++a) {
        dirs[a] = dominant_axis(g->kind, g->views[a], d);
        need[dirs[a]] = true;
    }
    const size_t px = d.vol_x + 4, py = d.vol_y + 4, pz = d.vol_z + 4;
    const size_t padded = px * py * pz;
    {
        // cell-space accumulators for x- and y-major views (one vector
        // reduction per sample); the scalar path below when they do not fit
        Scratch cacc[2], sz, macc[2];
        bool ok = true;
        // the slab transpose for the directions whose views it takes (its
        // accumulators hold single floats), else cell accumulators
        bool slab[2] = {false, false};
        for (int dir = 0; dir < 2; ++dir) {
            if (!need[dir] || !matched_slab_eligible(g, p, dir, dirs)) continue;
            const size_t bytes = matched_slab_acc_bytes(d, dir);
            const b2t_status st = macc[dir].alloc(bytes, s, "matched bp slab accumulator");
            if (st == B2T_ERR_NO_MEMORY) {
                clear_error();
                continue;
            }
            B2T_TRY(st);
            B2T_CUDA_TRY(cudaMemsetAsync(macc[dir].as<void>(), 0, bytes, s), "matched bp memset");
            slab[dir] = true;
        }
        for (int dir = 0; dir < 2 && ok; ++dir) {
            if (!need[dir] || slab[dir]) continue;
            const size_t count = (dir == 0 ? py : px) * (size_t)(dir == 0 ? d.vol_x : d.vol_y) * pz;
            const b2t_status st = cacc[dir].alloc(count * sizeof(float4), s, "matched bp cell accumulator");
            if (st == B2T_ERR_NO_MEMORY) {
                clear_error();
                ok = false;
                break;
            }
            B2T_TRY(st);
            B2T_CUDA_TRY(cudaMemsetAsync(cacc[dir].as<void>(), 0, count * sizeof(float4), s), "matched bp memset");
        }
        if (ok && need[2]) {
            const b2t_status st = sz.alloc(padded * sizeof(float), s, "matched bp accumulator (xyz)");
            if (st == B2T_ERR_NO_MEMORY) {
                clear_error();
                ok = false;
            } else {
                B2T_TRY(st);
                B2T_CUDA_TRY(cudaMemsetAsync(sz.as<void>(), 0, padded * sizeof(float), s), "matched bp memset");
            }
        }
        if (ok) {
            FPLaunch *Lp = new FPLaunch;
            FPLaunch &P = *Lp;
            const bool force_noncube = p->det_supersample > 1;
            b2t_status st = B2T_OK;
            for (int dir = 0; dir < 3 && st == B2T_OK; ++dir) {
                if (!need[dir]) continue;
                if (dir < 2 && slab[dir]) {
                    st = matched_slab_scatter(g, p, proj, proj_pitch, dtype, dir, dirs, macc[dir].as<float>(), s);
                    continue;
                }
                P.proj = const_cast<void *>(proj);
                P.proj_pitch = (long long)proj_pitch;
                P.nu = d.det_u;
                P.nv = d.det_v;
                P.na = d.angles;
                P.rays = p->det_supersample;
                P.accumulate = 0;
                fp_scale(g->kind, dir, g->vol_scale, force_noncube, p->output_scale, P.f1, P.f2, P.mul);
                if (dir == 0) { P.n0 = d.vol_x; P.n1 = d.vol_y; P.n2 = d.vol_z; }
                else if (dir == 1) { P.n0 = d.vol_y; P.n1 = d.vol_x; P.n2 = d.vol_z; }
                else {
                    P.n0 = d.vol_z; P.n1 = d.vol_x; P.n2 = d.vol_y;
                    P.st0 = (long long)(px * py);
                    P.st2 = (long long)px;
                }
                P.vol = (dir == 2) ? static_cast<void *>(sz.as<float>() + 2 * P.st0 + 2 * P.st2 + 2)
                                   : cacc[dir].as<void>();
                std::vector<int> views;
                for (uint32_t a = 0; a < d.angles; ++a)
                    if (dirs[a] == dir) views.push_back((int)a);
                for (size_t c0 = 0; c0 < views.size() && st == B2T_OK; c0 += FP_MAX_VIEWS) {
                    const size_t cn = std::min(views.size() - c0, (size_t)FP_MAX_VIEWS);
                    P.nviews = (int)cn;
                    for (size_t i = 0; i < cn; ++i) {
                        const int a = views[c0 + i];
                        fp_view_coeffs(g->kind, g->views[a], d, dir, P.views[i]);
                        P.views[i].a = a;
                    }
                    if (dir == 2) {
                        dim3 grid((unsigned)cn, (d.det_u + 31) / 32, (d.det_v + 7) / 8);
                        if (dtype == B2T_F32) st = launch_T<float>(P, grid, s);
                        else if (dtype == B2T_F16) st = launch_T<__half>(P, grid, s);
                        else st = launch_T<__nv_bfloat16>(P, grid, s);
                    } else {
                        dim3 grid((unsigned)cn, (d.det_u + 7) / 8, (d.det_v + 31) / 32);
                        // merged reductions key cells by 32-bit index (with
                        // the lanes' sentinels above the cell count)
                        const unsigned long long cells =
                            (unsigned long long)(P.n1 + 4) * P.n0 * (unsigned long long)(P.n2 + 4);
                        const bool agg = cells < (1ull << 32) - 64 && !matched_force_plain();
                        if (dtype == B2T_F32) {
                            if (agg) fp3d_transpose_cols_kernel<float, true><<<grid, dim3(32, 8), 0, s>>>(P);
                            else fp3d_transpose_cols_kernel<float, false><<<grid, dim3(32, 8), 0, s>>>(P);
                        } else if (dtype == B2T_F16) {
                            if (agg) fp3d_transpose_cols_kernel<__half, true><<<grid, dim3(32, 8), 0, s>>>(P);
                            else fp3d_transpose_cols_kernel<__half, false><<<grid, dim3(32, 8), 0, s>>>(P);
                        } else {
                            if (agg) fp3d_transpose_cols_kernel<__nv_bfloat16, true><<<grid, dim3(32, 8), 0, s>>>(P);
                            else fp3d_transpose_cols_kernel<__nv_bfloat16, false><<<grid, dim3(32, 8), 0, s>>>(P);
                        }
                        count_launches(1);
                        g_scatter_launches.fetch_add(1);
                        if (cudaGetLastError() != cudaSuccess) st = fail(B2T_ERR_CUDA, "matched bp (cells) launch");
                    }
                }
            }
            delete Lp;
            B2T_TRY(st);
            const int accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
            dim3 grid((d.vol_z + 127) / 128, d.vol_x, d.vol_y);
            const float4 *c0 = need[0] && !slab[0] ? cacc[0].as<float4>() : nullptr;
            const float4 *c1 = need[1] && !slab[1] ? cacc[1].as<float4>() : nullptr;
            const float *az = need[2] ? sz.as<float>() : nullptr;
            const float *m0 = slab[0] ? macc[0].as<float>() : nullptr;
            const float *m1 = slab[1] ? macc[1].as<float>() : nullptr;
            long long ay0 = 0, ay1 = 0, mz = 0;
            matched_slab_dims(d, 0, ay0, mz);
            matched_slab_dims(d, 1, ay1, mz);
            if (dtype == B2T_F32)
                fold_cells<float><<<grid, 128, 0, s>>>(c0, c1, az, m0, m1, ay0, ay1, mz, d.vol_x, d.vol_y, d.vol_z,
                                                       static_cast<float *>(vol), vol_pitch, accumulate);
            else if (dtype == B2T_F16)
                fold_cells<__half><<<grid, 128, 0, s>>>(c0, c1, az, m0, m1, ay0, ay1, mz, d.vol_x, d.vol_y,
                                                        d.vol_z, static_cast<__half *>(vol), vol_pitch, accumulate);
            else
                fold_cells<__nv_bfloat16><<<grid, 128, 0, s>>>(c0, c1, az, m0, m1, ay0, ay1, mz, d.vol_x, d.vol_y,
                                                               d.vol_z, static_cast<__nv_bfloat16 *>(vol),
                                                               vol_pitch, accumulate);
            count_launches(1);
            B2T_CUDA_TRY(cudaGetLastError(), "matched bp fold launch");
            return B2T_OK;
        }
    }
    Scratch sa, sb;
    if (need[1] || need[2]) {
        B2T_TRY(sa.alloc(padded * sizeof(float), s, "matched bp accumulator (xyz)"));
        B2T_CUDA_TRY(cudaMemsetAsync(sa.as<void>(), 0, padded * sizeof(float), s), "matched bp memset");
    }
    if (need[0]) {
        B2T_TRY(sb.alloc(padded * sizeof(float), s, "matched bp accumulator (zxy)"));
        B2T_CUDA_TRY(cudaMemsetAsync(sb.as<void>(), 0, padded * sizeof(float), s), "matched bp memset");
    }
    FPLaunch *Lp = new FPLaunch;
    FPLaunch &P = *Lp;
    const bool force_noncube = p->det_supersample > 1;
    for (int dir = 0; dir < 3; ++dir) {
        if (!need[dir]) continue;
        P.proj = const_cast<void *>(proj);
        P.proj_pitch = (long long)proj_pitch;
        P.nu = d.det_u;
        P.nv = d.det_v;
        P.na = d.angles;
        P.rays = p->det_supersample;
        P.accumulate = 0;
        fp_scale(g->kind, dir, g->vol_scale, force_noncube, p->output_scale, P.f1, P.f2, P.mul);
        float *base;
        if (dir == 0) {
            base = sb.as<float>();
            P.n0 = d.vol_x; P.n1 = d.vol_y; P.n2 = d.vol_z;
            P.st0 = (long long)py;
            P.st2 = (long long)(px * py);
            base += 2 * P.st2 + 2 * P.st0 + 2;
        } else if (dir == 1) {
            base = sa.as<float>();
            P.n0 = d.vol_y; P.n1 = d.vol_x; P.n2 = d.vol_z;
            P.st0 = (long long)px;
            P.st2 = (long long)(px * py);
            base += 2 * P.st2 + 2 * P.st0 + 2;
        } else {
            base = sa.as<float>();
            P.n0 = d.vol_z; P.n1 = d.vol_x; P.n2 = d.vol_y;
            P.st0 = (long long)(px * py);
            P.st2 = (long long)px;
            base += 2 * P.st0 + 2 * P.st2 + 2;
        }
        P.vol = base;
        std::vector<int> views;
        for (uint32_t a = 0; a < d.angles; ++a)
            if (dirs[a] == dir) views.push_back((int)a);
        for (size_t c0 = 0; c0 < views.size(); c0 += FP_MAX_VIEWS) {
            const size_t cn = std::min(views.size() - c0, (size_t)FP_MAX_VIEWS);
            P.nviews = (int)cn;
            for (size_t i = 0; i < cn; ++i) {
                const int a = views[c0 + i];
                fp_view_coeffs(g->kind, g->views[a], d, dir, P.views[i]);
                P.views[i].a = a;
            }
            dim3 grid((unsigned)cn, (d.det_u + 31) / 32, (d.det_v + 7) / 8);
            b2t_status st;
            if (dtype == B2T_F32) st = launch_T<float>(P, grid, s);
            else if (dtype == B2T_F16) st = launch_T<__half>(P, grid, s);
            else st = launch_T<__nv_bfloat16>(P, grid, s);
            if (st != B2T_OK) {
                delete Lp;
                return st;
            }
        }
    }
    delete Lp;
    const float *a = (need[1] || need[2]) ? sa.as<float>() : nullptr;
    const float *b = need[0] ? sb.as<float>() : nullptr;
    const int accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
    if (dtype == B2T_F32) return launch_fold<float>(a, b, d, vol, vol_pitch, accumulate, s);
    if (dtype == B2T_F16) return launch_fold<__half>(a, b, d, vol, vol_pitch, accumulate, s);
    return launch_fold<__nv_bfloat16>(a, b, d, vol, vol_pitch, accumulate, s);
}

}  // namespace b2t
