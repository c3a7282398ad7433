// 3D forward and back projectors for parallel (par3d / parallel3d_vec) and
// cone (cone / cone_vec) geometries on sm_100a.
//
// Model: the reference's texture-sampled projectors (cuda/3d/cone_fp.cu,
// cuda/3d/par3d_fp.cu, cuda/3d/cone_bp.cu, cuda/3d/par3d_bp.cu) evaluated with
// explicit FP32 interpolation instead of 8-bit texture weights:
//   FP: ray-driven; each ray marches the view's dominant axis at unit steps
//       through voxel centres and sums bilinear samples of the slice plane;
//       the sum is scaled by sqrt(1 + a1^2 + a2^2) * voxel size.
//   BP: voxel-driven; each voxel centre is projected onto every view's
//       detector, the projection is sampled bilinearly and weighted by the
//       ray-density factor 1/Den^2 (or 1/Den for 2d_weighting, FDK weights).
//
// B200 design:
//   - per-view geometry is precomputed on the host in FP64 and passed in a
//     __grid_constant__ kernel parameter block (no module-global __constant__
//     state, so concurrent calls on different streams are safe);
//   - FP: one thread owns one ray and accumulates the whole ray in registers
//     (the reference writes back to HBM every 4 slices); blockIdx.x walks
//     views fastest so the CTAs resident at one time read the same thin slab
//     of the volume and the slab stays in the 126 MB L2;
//   - the volume is read from a zero-padded copy whose contiguous axis is a
//     non-marching axis for every view (a y-fastest copy for x-major views),
//     so a warp of u-adjacent rays issues coalesced loads;
//   - the zero border replaces the texture unit's border mode; per-ray slice
//     ranges are clipped so every access is inside the padded copy;
//   - BP: one thread owns a column of ZB voxels accumulated in registers over
//     all views of a launch; reads come from a zero-padded projection copy.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "b2t_internal.h"
#include "proj3d.h"
#include "proj3d_dev.cuh"

namespace b2t {

// ---------------------------------------------------------------------------
// padded copies
// ---------------------------------------------------------------------------

// dst[z+2][y+2][x+2] = src[z][y][x], zero border of width 2.
template <typename T>
__global__ void pad_volume_xyz(const T *__restrict__ src, size_t src_pitch, int nx, int ny, int nz,
                               T *__restrict__ dst)
{
    const int px = nx + 4, py = ny + 4;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= px) return;
    const int sx = x - 2, sy = y - 2, sz = z - 2;
    T v = from_float<T>(0.0f);
    if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz)
        v = src[((size_t)sz * ny + sy) * src_pitch + sx];
    dst[((size_t)z * py + y) * px + x] = v;
}

// dst[z+2][x+2][y+2] = src[z][y][x] (y fastest), zero border of width 2;
// 32x32 tiles transposed through shared memory.
template <typename T>
__global__ void pad_volume_zxy(const T *__restrict__ src, size_t src_pitch, int nx, int ny, int nz,
                               T *__restrict__ dst)
{
    __shared__ T tile[32][33];
    const int px = nx + 4, py = ny + 4;
    const int z = blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const int sz = z - 2;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int y = y0 + j, x = x0 + threadIdx.x;
        int sx = x - 2, sy = y - 2;
        T v = from_float<T>(0.0f);
        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz)
            v = src[((size_t)sz * ny + sy) * src_pitch + sx];
        tile[j][threadIdx.x] = v;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int x = x0 + j, y = y0 + threadIdx.x;
        if (x < px && y < py) dst[((size_t)z * px + x) * py + y] = tile[threadIdx.x][j];
    }
}

// dst[v+2][a][u+2] = src[v][a][u], zero border of width 2 in u and v (and
// zero columns up to the row pitch pu).
template <typename T>
__global__ void pad_proj(const T *__restrict__ src, size_t src_pitch, int nu, int na, int nv, int pu,
                         T *__restrict__ dst)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    const int v = blockIdx.z;
    if (u >= pu) return;
    const int su = u - 2, sv = v - 2;
    T val = from_float<T>(0.0f);
    if (su >= 0 && su < nu && sv >= 0 && sv < nv) val = src[((size_t)sv * na + a) * src_pitch + su];
    dst[((size_t)v * na + a) * pu + u] = val;
}

// The same in the pair layout of 16-bit texels: dst[v][a][u] is the word
// (x[v][a][u], x[v+1][a][u]) of the padded texels x (the texel and the one
// below it; x past the last row zero).
template <typename T, typename T2>
__global__ void pad_proj_pairs(const T *__restrict__ src, size_t src_pitch, int nu, int na, int nv, int pu,
                               T2 *__restrict__ dst)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int a = blockIdx.y;
    const int v = blockIdx.z;
    if (u >= pu) return;
    const int su = u - 2, sv = v - 2;
    T x0 = from_float<T>(0.0f), x1 = from_float<T>(0.0f);
    if (su >= 0 && su < nu) {
        if (sv >= 0 && sv < nv) x0 = src[((size_t)sv * na + a) * src_pitch + su];
        if (sv + 1 >= 0 && sv + 1 < nv) x1 = src[((size_t)(sv + 1) * na + a) * src_pitch + su];
    }
    T2 w;
    w.x = x0;
    w.y = x1;
    dst[((size_t)v * na + a) * pu + u] = w;
}

// ---------------------------------------------------------------------------
// forward projection
// ---------------------------------------------------------------------------

template <typename T>
__global__ void __launch_bounds__(256) fp3d_kernel(const __grid_constant__ FPLaunch L)
{
    const FPView &V = L.views[blockIdx.x];
    const int u = blockIdx.y * 32 + threadIdx.x;
    const int v = blockIdx.z * 8 + threadIdx.y;
    if (u >= L.nu || v >= L.nv) return;
    const FPPadded<T> Ld{static_cast<const T *>(L.vol), L.st0, L.st2};
    float acc = fp3d_ray(Ld, V, u, v, L.n0, L.n1, L.n2, L.nu, L.nv, L.rays, L.f1, L.f2, L.mul);
    T *out = static_cast<T *>(L.proj) + ((size_t)v * L.na + V.a) * L.proj_pitch + u;
    if (L.accumulate) acc += ldplain(out);
    *out = from_float<T>(acc);
}

// ---------------------------------------------------------------------------
// backprojection
// ---------------------------------------------------------------------------

template <typename T, int KIND, int KER, int ZB>
__global__ void __launch_bounds__(256) bp3d_kernel(const __grid_constant__ BPLaunch L)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * ZB;
    if (x >= L.nx || y >= L.ny) return;
    const float fx = (float)x - 0.5f * (float)L.nx + 0.5f;
    const float fy = (float)y - 0.5f * (float)L.ny + 0.5f;
    const float fz = (float)z0 - 0.5f * (float)L.nz + 0.5f;
    const BPPadded<T> Ld{static_cast<const T *>(L.proj), L.pv, L.pu};
    float acc[ZB];
    bp3d_column<KIND, KER, ZB>(Ld, L.views, L.nviews, L.a0, L.nu, L.nv, fx, fy, fz, acc);
    T *out = static_cast<T *>(L.vol);
#pragma unroll
    for (int j = 0; j < ZB; ++j) {
        const int z = z0 + j;
        if (z < L.nz) {
            T *o = out + ((size_t)z * L.ny + y) * L.vol_pitch + x;
            float r = acc[j] * L.out_scale;
            if (L.accumulate) r += ldplain(o);
            *o = from_float<T>(r);
        }
    }
}

// Voxel-supersampled BP (dev_cone_BP_SS / dev_par3D_BP_SS): R^3 sub-voxels.
template <typename T, int KIND>
__global__ void __launch_bounds__(256) bp3d_ss_kernel(const __grid_constant__ BPLaunch L)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= L.nx || y >= L.ny || z >= L.nz) return;
    const T *__restrict__ proj = static_cast<const T *>(L.proj);
    const int R = L.rays;
    const float sub = 1.0f / (float)R;
    const float bx = (float)x - 0.5f * (float)L.nx + 0.5f - 0.5f + 0.5f * sub;
    const float by = (float)y - 0.5f * (float)L.ny + 0.5f - 0.5f + 0.5f * sub;
    const float bz = (float)z - 0.5f * (float)L.nz + 0.5f - 0.5f + 0.5f * sub;
    float acc = 0.0f;
    for (int i = 0; i < L.nviews; ++i) {
        const BPView &W = L.views[i];
        const T *P = proj + (long long)(L.a0 + i) * L.pu;
        for (int ix = 0; ix < R; ++ix)
            for (int iy = 0; iy < R; ++iy)
                for (int iz = 0; iz < R; ++iz) {
                    const float fx = bx + ix * sub, fy = by + iy * sub, fz = bz + iz * sub;
                    float U = fmaf(fz, W.nu.z, fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)));
                    float Vc = fmaf(fz, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
                    float w;
                    if (KIND == B2T_GEOM_CONE) {
                        const float dn = fmaf(fz, W.den.z, fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w)));
                        const float fr = __frcp_rn(dn);
                        U *= fr;
                        Vc *= fr;
                        w = fr * fr;
                    } else {
                        w = W.den.w;
                    }
                    int ku, kv;
                    float fu, fv;
                    split_texel(U - 1.0f, ku, fu);
                    split_texel(Vc - 1.0f, kv, fv);
                    ku = min(max(ku, -2), L.nu);
                    kv = min(max(kv, -2), L.nv);
                    const T *p = P + (long long)kv * L.pv + ku;
                    const float v00 = ld(p), v10 = ld(p + 1);
                    const float v01 = ld(p + L.pv), v11 = ld(p + L.pv + 1);
                    const float a = fmaf(fu, v10 - v00, v00);
                    const float b = fmaf(fu, v11 - v01, v01);
                    acc = fmaf(fmaf(fv, b - a, a), w, acc);
                }
    }
    T *o = static_cast<T *>(L.vol) + ((size_t)z * L.ny + y) * L.vol_pitch + x;
    float r = acc * L.out_scale;
    if (L.accumulate) r += ldplain(o);
    *o = from_float<T>(r);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

namespace {

struct D3 {
    double v[3];
};

inline double det3x(const double *b, const double *c) { return b[1] * c[2] - b[2] * c[1]; }
inline double det3y(const double *b, const double *c) { return -(b[0] * c[2] - b[2] * c[0]); }
inline double det3z(const double *b, const double *c) { return b[0] * c[1] - b[1] * c[0]; }
inline double det3(const double *a, const double *b, const double *c)
{
    return a[0] * det3x(b, c) + a[1] * det3y(b, c) + a[2] * det3z(b, c);
}
inline double scaled_cross_norm(const double *a, const double *b, const float *sc)
{
    double x = det3x(a, b) * sc[1] * sc[2];
    double y = det3y(a, b) * sc[0] * sc[2];
    double z = det3z(a, b) * sc[0] * sc[1];
    return std::sqrt(x * x + y * y + z * z);
}

const int kPerm[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};

template <typename T> b2t_status launch_fp_typed(const FPLaunch &L, dim3 grid, cudaStream_t s)
{
    fp3d_kernel<T><<<grid, dim3(32, 8), 0, s>>>(L);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "fp3d kernel launch");
    return B2T_OK;
}

template <typename T>
b2t_status pad_volumes(const void *vol, size_t pitch, const b2t_dims3d &d, void *pa, void *pb,
                       cudaStream_t s)
{
    const int nx = d.vol_x, ny = d.vol_y, nz = d.vol_z;
    if (pa) {
        dim3 grid((nx + 4 + 127) / 128, ny + 4, nz + 4);
        pad_volume_xyz<T><<<grid, 128, 0, s>>>(static_cast<const T *>(vol), pitch, nx, ny, nz,
                                               static_cast<T *>(pa));
        count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "pad_volume_xyz launch");
    }
    if (pb) {
        dim3 grid((nx + 4 + 31) / 32, (ny + 4 + 31) / 32, nz + 4);
        pad_volume_zxy<T><<<grid, dim3(32, 8), 0, s>>>(static_cast<const T *>(vol), pitch, nx, ny, nz,
                                                       static_cast<T *>(pb));
        count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "pad_volume_zxy launch");
    }
    return B2T_OK;
}

}  // namespace

b2t_status pad_volumes_f32(const float *vol, size_t pitch, const b2t_dims3d &d, float *xyz, float *zxy,
                           cudaStream_t s)
{
    return pad_volumes<float>(vol, pitch, d, xyz, zxy, s);
}

namespace {

template <typename T>
b2t_status pad_projections(const void *proj, size_t pitch, const b2t_dims3d &d, void *pp, bool pairs,
                           cudaStream_t s)
{
    const int pu = (int)padded_pu(d.det_u);
    dim3 grid((pu + 127) / 128, d.angles, d.det_v + 4);
    if constexpr (sizeof(T) == 2) {
        if (pairs) {
            using T2 = typename std::conditional<std::is_same<T, __half>::value, __half2, __nv_bfloat162>::type;
            pad_proj_pairs<T, T2><<<grid, 128, 0, s>>>(static_cast<const T *>(proj), pitch, d.det_u, d.angles,
                                                       d.det_v, pu, static_cast<T2 *>(pp));
            count_launches(1);
            B2T_CUDA_TRY(cudaGetLastError(), "pad_proj_pairs launch");
            return B2T_OK;
        }
    }
    pad_proj<T><<<grid, 128, 0, s>>>(static_cast<const T *>(proj), pitch, d.det_u, d.angles, d.det_v, pu,
                                     static_cast<T *>(pp));
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "pad_proj launch");
    return B2T_OK;
}

}  // namespace

// Per-view ray coefficients in the dominant frame, FP64 on the host.  Ray
// through detector offset (u', v') from the detector centre (pixels):
//   a_k  = (m_k . [1,u',v']) / (e . [1,u',v'])      (slope along axis k)
//   b'_k = (n_k . [1,u',v']) / (e . [1,u',v'])      (q - 0.5 at slice 0)
// cone (cone_fp.cu:188-204): e = S0 - D0, m_k = S_k - D_k, b_k = S_k - a_k S0;
// par3d (par3d_fp.cu:157-200): e = 1, m_k = R_k/R0, b_k = D_k - a_k D0.
void fp_view_coeffs(int kind, const b2t_view3d &w, const b2t_dims3d &d, int dir, FPView &o)
{
    const int *P = kPerm[dir];
    const double nx[3] = {(double)d.vol_x, (double)d.vol_y, (double)d.vol_z};
    const double N0 = nx[P[0]], N1 = nx[P[1]], N2 = nx[P[2]];
    // detector centre and steps
    double Dc[3], U[3], Vv[3];
    for (int k = 0; k < 3; ++k) {
        Dc[k] = w.det_s[k] + 0.5 * d.det_u * w.det_u[k] + 0.5 * d.det_v * w.det_v[k];
        U[k] = w.det_u[k];
        Vv[k] = w.det_v[k];
    }
    double e[3], m[2][3], n[2][3];
    if (kind == B2T_GEOM_CONE) {
        const double *S = w.src;
        const double s0 = S[P[0]];
        e[0] = s0 - Dc[P[0]];
        e[1] = -U[P[0]];
        e[2] = -Vv[P[0]];
        for (int j = 0; j < 2; ++j) {
            const int c = P[1 + j];
            const double sc = S[c];
            m[j][0] = sc - Dc[c];
            m[j][1] = -U[c];
            m[j][2] = -Vv[c];
            // b = S_c - a S0 = (S0 D_c - S_c D0) / (S0 - D0)
            n[j][0] = s0 * Dc[c] - sc * Dc[P[0]];
            n[j][1] = s0 * U[c] - sc * U[P[0]];
            n[j][2] = s0 * Vv[c] - sc * Vv[P[0]];
        }
    } else {
        const double *R = w.src;
        const double r0 = R[P[0]];
        e[0] = 1.0;
        e[1] = 0.0;
        e[2] = 0.0;
        for (int j = 0; j < 2; ++j) {
            const int c = P[1 + j];
            const double a = R[c] / r0;
            m[j][0] = a;
            m[j][1] = 0.0;
            m[j][2] = 0.0;
            n[j][0] = Dc[c] - a * Dc[P[0]];
            n[j][1] = U[c] - a * U[P[0]];
            n[j][2] = Vv[c] - a * Vv[P[0]];
        }
    }
    // q(s) - 0.5 = a*(s - N0/2 + 0.5) + b + N_k/2 - 1
    const double Nk[2] = {N1, N2};
    for (int j = 0; j < 2; ++j)
        for (int t = 0; t < 3; ++t)
            n[j][t] = n[j][t] + (0.5 * Nk[j] - 1.0) * e[t] + (0.5 - 0.5 * N0) * m[j][t];
    for (int t = 0; t < 3; ++t) {
        o.e[t] = (float)e[t];
        o.m1[t] = (float)m[0][t];
        o.m2[t] = (float)m[1][t];
        o.n1[t] = (float)n[0][t];
        o.n2[t] = (float)n[1][t];
    }
}

// Dominant axis, with the reference's float comparison (cone_fp.cu:375-388,
// par3d_fp.cu:474-487).
int dominant_axis(int kind, const b2t_view3d &w, const b2t_dims3d &d)
{
    float dX, dY, dZ;
    if (kind == B2T_GEOM_CONE) {
        dX = fabsf((float)(w.src[0] - (w.det_s[0] + d.det_u * w.det_u[0] * 0.5f + d.det_v * w.det_v[0] * 0.5f)));
        dY = fabsf((float)(w.src[1] - (w.det_s[1] + d.det_u * w.det_u[1] * 0.5f + d.det_v * w.det_v[1] * 0.5f)));
        dZ = fabsf((float)(w.src[2] - (w.det_s[2] + d.det_u * w.det_u[2] * 0.5f + d.det_v * w.det_v[2] * 0.5f)));
    } else {
        dX = fabsf((float)w.src[0]);
        dY = fabsf((float)w.src[1]);
        dZ = fabsf((float)w.src[2]);
    }
    if (dX >= dY && dX >= dZ) return 0;
    if (dY >= dX && dY >= dZ) return 1;
    return 2;
}

// Ray-sum scale factors (SCALE_CUBE / SCALE_NONCUBE selection,
// cone_fp.cu:335-370, par3d_fp.cu:436-469).
void fp_scale(int kind, int dir, const float *vs, bool force_noncube, float out_scale, float &f1,
              float &f2, float &mul)
{
    bool cube = true;
    if (std::abs(vs[0] / vs[1] - 1.0) > 0.00001) cube = false;
    if (std::abs(vs[0] / vs[2] - 1.0) > 0.00001) cube = false;
    if (cube && !force_noncube) {
        f1 = f2 = 1.0f;
        mul = out_scale * vs[0];
        return;
    }
    float s1, s2;
    if (dir == 0) {
        s1 = vs[1] / vs[0];
        s2 = vs[2] / vs[0];
        mul = out_scale * vs[0];
    } else if (dir == 1) {
        s1 = vs[0] / vs[1];
        s2 = (kind == B2T_GEOM_PAR3D) ? vs[1] / vs[1] : vs[2] / vs[1];
        mul = out_scale * vs[1];
    } else {
        s1 = vs[0] / vs[2];
        s2 = vs[1] / vs[2];
        mul = out_scale * vs[2];
    }
    f1 = s1 * s1;
    f2 = s2 * s2;
}

// BP per-view coefficients (cone: transferConstants, cone_bp.cu:221-302;
// par3d: transferConstants, par3d_bp.cu:202-244), FP64 then rounded.
void bp_view_coeffs(int kind, int kernel, const b2t_view3d &w, const float *vs, BPView &o)
{
    const double *u = w.det_u, *v = w.det_v, *d = w.det_s;
    if (kind == B2T_GEOM_CONE) {
        const double *s = w.src;
        const double smd[3] = {s[0] - d[0], s[1] - d[1], s[2] - d[2]};
        double scale;
        if (kernel == B2T_KER_FDK_WEIGHTING) {
            scale = 1.0 / det3(u, v, s);
        } else if (kernel == B2T_KER_2D_WEIGHTING) {
            const double ez[3] = {0, 0, 1};
            scale = scaled_cross_norm(u, ez, vs) / det3(u, v, smd);
        } else {
            scale = std::sqrt(scaled_cross_norm(u, v, vs)) / det3(u, v, smd);
        }
        o.nu = make_float4((float)(scale * det3x(v, smd)), (float)(scale * det3y(v, smd)),
                           (float)(scale * det3z(v, smd)), (float)(scale * det3(s, v, d)));
        o.nv = make_float4((float)(-scale * det3x(u, smd)), (float)(-scale * det3y(u, smd)),
                           (float)(-scale * det3z(u, smd)), (float)(-scale * det3(s, u, d)));
        o.den = make_float4((float)(-scale * det3x(u, v)), (float)(-scale * det3y(u, v)),
                            (float)(-scale * det3z(u, v)),
                            kernel == B2T_KER_FDK_WEIGHTING ? 1.0f : (float)(scale * det3(u, v, s)));
    } else {
        const double *r = w.src;
        const double den = det3(r, u, v);
        o.nu = make_float4((float)(-det3x(r, v) / den), (float)(-det3y(r, v) / den),
                           (float)(-det3z(r, v) / den), (float)(-det3(r, d, v) / den));
        o.nv = make_float4((float)(det3x(r, u) / den), (float)(det3y(r, u) / den),
                           (float)(det3z(r, u) / den), (float)(det3(r, d, u) / den));
        double sc;
        if (kernel == B2T_KER_2D_WEIGHTING) {
            const double ez[3] = {0, 0, 1};
            sc = 1.0 / scaled_cross_norm(u, ez, vs);
        } else {
            sc = 1.0 / scaled_cross_norm(u, v, vs);
        }
        o.den = make_float4(0.0f, 0.0f, 0.0f, (float)sc);
    }
}

// B2T_SIMPLE_BP=1 selects the direct-load backprojector instead of the
// TMA-staged one (both implement the same model; tests compare them).
bool force_simple_bp()
{
    const char *e = getenv("B2T_SIMPLE_BP");
    return e && e[0] == '1';
}

// B2T_SIMPLE_FP=1 selects the padded-copy forward projector instead of the
// cell one (same model; tests compare them).
bool force_simple_fp()
{
    const char *e = getenv("B2T_SIMPLE_FP");
    return e && e[0] == '1';
}

b2t_status validate3d(const b2t_geom3d *g, const char *who)
{
    if (!g || !g->views) return fail(B2T_ERR_INVALID_ARG, "%s: null geometry", who);
    if (g->kind != B2T_GEOM_CONE && g->kind != B2T_GEOM_PAR3D)
        return fail(B2T_ERR_INVALID_ARG, "%s: geometry kind must be PAR3D or CONE", who);
    const b2t_dims3d &d = g->dims;
    if (d.vol_x == 0 || d.vol_y == 0 || d.vol_z == 0 || d.angles == 0 || d.det_u == 0 || d.det_v == 0)
        return fail(B2T_ERR_INVALID_ARG, "%s: empty dimension", who);
    if (d.vol_x > (1u << 20) || d.vol_y > (1u << 20) || d.vol_z > (1u << 20) || d.det_u > (1u << 20) ||
        d.det_v > (1u << 20))
        return fail(B2T_ERR_INVALID_ARG, "%s: dimension above 2^20", who);
    for (int k = 0; k < 3; ++k)
        if (!(g->vol_scale[k] > 0.0f)) return fail(B2T_ERR_INVALID_ARG, "%s: voxel size must be > 0", who);
    return B2T_OK;
}

b2t_status fp3d_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *vol, size_t vol_pitch,
                     void *proj, size_t proj_pitch, int32_t dtype, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate3d(g, "b2t_fp3d"));
    if (!p) return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: null params");
    if (!proj) return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: null data pointer");
    if (!dtype_valid(dtype)) return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: bad dtype %d", dtype);
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET)
        return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: bad mode %d", mode);
    if (p->kernel < 0 || p->kernel > B2T_KER_MATCHED_BP)
        return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: bad kernel %d", p->kernel);
    if (p->det_supersample == 0 || p->det_supersample > 16)
        return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: detector supersampling must be 1..16");
    const b2t_dims3d &d = g->dims;
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (vol_pitch < d.vol_x || proj_pitch < d.det_u)
        return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: pitch below row length");
    // sum_square_weights reads no volume (vol may be null)
    if (p->kernel == B2T_KER_SUM_SQUARE_WEIGHTS) return fp3d_sumsqw_impl(g, p, proj, proj_pitch, dtype, mode, s);
    if (!vol) return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d: null data pointer");

    std::vector<int> dirs(d.angles);
    bool need[3] = {false, false, false};
    for (uint32_t a = 0; a < d.angles; ++a) {
        dirs[a] = dominant_axis(g->kind, g->views[a], d);
        need[dirs[a]] = true;
    }
    if (!force_simple_fp()) {
        // cell path (fp3d_cells.cu); if its scratch does not fit, use the
        // padded-copy path below, which needs a quarter of the memory
        const b2t_status st = fp3d_cells(g, p, vol, vol_pitch, proj, proj_pitch, dtype, mode, dirs, s);
        if (st != B2T_ERR_NO_MEMORY) return st;
        clear_error();
    }
    const size_t esz = dtype_size(dtype);
    const size_t px = d.vol_x + 4, py = d.vol_y + 4, pz = d.vol_z + 4;
    const size_t padded = px * py * pz;
    Scratch sa, sb;
    if (need[1] || need[2]) B2T_TRY(sa.alloc(padded * esz, s, "b2t_fp3d scratch (xyz copy)"));
    if (need[0]) B2T_TRY(sb.alloc(padded * esz, s, "b2t_fp3d scratch (zxy copy)"));
    void *pa = (need[1] || need[2]) ? sa.as<void>() : nullptr;
    void *pb = need[0] ? sb.as<void>() : nullptr;
    if (dtype == B2T_F32) B2T_TRY(pad_volumes<float>(vol, vol_pitch, d, pa, pb, s));
    else if (dtype == B2T_F16) B2T_TRY(pad_volumes<__half>(vol, vol_pitch, d, pa, pb, s));
    else B2T_TRY(pad_volumes<__nv_bfloat16>(vol, vol_pitch, d, pa, pb, s));

    FPLaunch *Lp = new FPLaunch;  // large parameter block; filled per launch below
    const bool force_noncube = p->det_supersample > 1;
    for (int dir = 0; dir < 3; ++dir) {
        if (!need[dir]) continue;
        FPLaunch &P = *Lp;
        P.proj = proj;
        P.proj_pitch = (long long)proj_pitch;
        P.nu = d.det_u;
        P.nv = d.det_v;
        P.na = d.angles;
        P.rays = p->det_supersample;
        P.accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
        fp_scale(g->kind, dir, g->vol_scale, force_noncube, p->output_scale, P.f1, P.f2, P.mul);
        const char *base;
        if (dir == 0) {
            base = sb.as<char>();
            P.n0 = d.vol_x; P.n1 = d.vol_y; P.n2 = d.vol_z;
            P.st0 = (long long)py;            // x stride in [z][x][y]
            P.st2 = (long long)(px * py);     // z stride
            base += (2 * P.st2 + 2 * P.st0 + 2) * esz;
        } else if (dir == 1) {
            base = sa.as<char>();
            P.n0 = d.vol_y; P.n1 = d.vol_x; P.n2 = d.vol_z;
            P.st0 = (long long)px;            // y stride in [z][y][x]
            P.st2 = (long long)(px * py);     // z stride
            base += (2 * P.st2 + 2 * P.st0 + 2) * esz;
        } else {
            base = sa.as<char>();
            P.n0 = d.vol_z; P.n1 = d.vol_x; P.n2 = d.vol_y;
            P.st0 = (long long)(px * py);     // z stride
            P.st2 = (long long)px;            // y stride
            base += (2 * P.st0 + 2 * P.st2 + 2) * esz;
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
            if (dtype == B2T_F32) st = launch_fp_typed<float>(P, grid, s);
            else if (dtype == B2T_F16) st = launch_fp_typed<__half>(P, grid, s);
            else st = launch_fp_typed<__nv_bfloat16>(P, grid, s);
            if (st != B2T_OK) {
                delete Lp;
                return st;
            }
        }
    }
    delete Lp;
    return B2T_OK;
}

namespace {
template <typename T, int KIND, int KER>
b2t_status launch_bp(const BPLaunch &L, const b2t_dims3d &d, cudaStream_t s)
{
    constexpr int ZB = 8;
    if (L.rays > 1) {
        dim3 grid((d.vol_x + 31) / 32, (d.vol_y + 7) / 8, d.vol_z);
        bp3d_ss_kernel<T, KIND><<<grid, dim3(32, 8), 0, s>>>(L);
    } else {
        dim3 grid((d.vol_x + 31) / 32, (d.vol_y + 7) / 8, (d.vol_z + ZB - 1) / ZB);
        bp3d_kernel<T, KIND, KER, ZB><<<grid, dim3(32, 8), 0, s>>>(L);
    }
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "bp3d kernel launch");
    return B2T_OK;
}

template <typename T>
b2t_status launch_bp_kind(const BPLaunch &L, int kind, int ker, const b2t_dims3d &d, cudaStream_t s)
{
    if (kind == B2T_GEOM_PAR3D) return launch_bp<T, B2T_GEOM_PAR3D, B2T_KER_DEFAULT>(L, d, s);
    if (ker == B2T_KER_2D_WEIGHTING) return launch_bp<T, B2T_GEOM_CONE, B2T_KER_2D_WEIGHTING>(L, d, s);
    return launch_bp<T, B2T_GEOM_CONE, B2T_KER_DEFAULT>(L, d, s);
}
}  // namespace

b2t_status bp3d_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *proj, size_t proj_pitch,
                     void *vol, size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate3d(g, "b2t_bp3d"));
    if (!p) return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d: null params");
    if (!vol || !proj) return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d: null data pointer");
    if (!dtype_valid(dtype)) return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d: bad dtype %d", dtype);
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d: bad mode %d", mode);
    if (p->voxel_supersample == 0 || p->voxel_supersample > 16)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d: voxel supersampling must be 1..16");
    const int ker = p->kernel;
    if (ker == B2T_KER_MATCHED_BP) return matched_bp3d_impl(g, p, proj, proj_pitch, vol, vol_pitch, dtype, mode, s);
    if (ker != B2T_KER_DEFAULT && ker != B2T_KER_FDK_WEIGHTING && ker != B2T_KER_2D_WEIGHTING)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_bp3d: kernel %d has no backprojector", ker);
    if (g->kind == B2T_GEOM_PAR3D && ker == B2T_KER_FDK_WEIGHTING)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_bp3d: fdk_weighting needs a cone geometry");
    if (p->voxel_supersample > 1 && ker != B2T_KER_DEFAULT)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_bp3d: supersampling only with the default kernel");
    const b2t_dims3d &d = g->dims;
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (vol_pitch < d.vol_x || proj_pitch < d.det_u)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d: pitch below row length");

    const bool pairs = bp_pairs(dtype, p);
    Scratch sp;
    B2T_TRY(sp.alloc(padded_proj_bytes(d, dtype, pairs), s, "b2t_bp3d scratch (padded projections)"));
    if (dtype == B2T_F32) B2T_TRY(pad_projections<float>(proj, proj_pitch, d, sp.as<void>(), false, s));
    else if (dtype == B2T_F16) B2T_TRY(pad_projections<__half>(proj, proj_pitch, d, sp.as<void>(), pairs, s));
    else B2T_TRY(pad_projections<__nv_bfloat16>(proj, proj_pitch, d, sp.as<void>(), pairs, s));
    return bp3d_from_padded(g, p, sp.as<void>(), vol, vol_pitch, dtype, mode, s);
}

b2t_status pad_projections_impl(const void *proj, size_t pitch, const b2t_dims3d &d, void *padded, int32_t dtype,
                                bool pairs, cudaStream_t s)
{
    if (dtype == B2T_F32) return pad_projections<float>(proj, pitch, d, padded, false, s);
    if (dtype == B2T_F16) return pad_projections<__half>(proj, pitch, d, padded, pairs, s);
    return pad_projections<__nv_bfloat16>(proj, pitch, d, padded, pairs, s);
}

bool bp_pairs(int32_t dtype, const b2t_params3d *p)
{
    return dtype != B2T_F32 && p->voxel_supersample == 1 && !force_simple_bp();
}

size_t padded_proj_bytes(const b2t_dims3d &d, int32_t dtype, bool pairs)
{
    return padded_pu(d.det_u) * d.angles * (size_t)(d.det_v + 4) * padded_elem_size(dtype, pairs);
}

// BP from a zero-padded projection buffer [v+2][angle][u+2] (pitch
// padded_pu(det_u), border of 2 texels in u and v; pairs of texels when
// bp_pairs(dtype, p)), already validated by the caller.  The direct-load
// kernels below read the texel layout, which bp_pairs selects for them.
b2t_status bp3d_from_padded(const b2t_geom3d *g, const b2t_params3d *p, const void *padded, void *vol,
                            size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s)
{
    const b2t_dims3d &d = g->dims;
    const int ker = p->kernel;
    const size_t esz = dtype_size(dtype);
    const size_t pu = padded_pu(d.det_u);
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    const float *vs0 = g->vol_scale;
    if (p->voxel_supersample == 1 && !force_simple_bp()) {
        const float outs = (g->kind == B2T_GEOM_CONE && ker == B2T_KER_FDK_WEIGHTING)
                               ? p->output_scale / vs0[0]
                               : p->output_scale * (vs0[0] * vs0[1] * vs0[2]);
        return bp3d_tma(g, ker, outs, padded, bp_pairs(dtype, p), vol, vol_pitch, dtype, mode, s);
    }
    BPLaunch *Lp = new BPLaunch;
    BPLaunch &L = *Lp;
    L.pu = (int)pu;
    L.pv = (long long)pu * d.angles;
    L.proj = static_cast<const char *>(padded) + (2 * L.pv + 2) * esz;
    L.vol = vol;
    L.vol_pitch = (long long)vol_pitch;
    L.nx = d.vol_x; L.ny = d.vol_y; L.nz = d.vol_z;
    L.nu = d.det_u; L.nv = d.det_v;
    L.rays = p->voxel_supersample;
    const float *vs = g->vol_scale;
    float outs;
    if (g->kind == B2T_GEOM_CONE && ker == B2T_KER_FDK_WEIGHTING) outs = p->output_scale / vs[0];
    else outs = p->output_scale * (vs[0] * vs[1] * vs[2]);
    if (L.rays > 1) outs /= (float)(L.rays * L.rays * L.rays);
    L.out_scale = outs;
    const int kker = (ker == B2T_KER_FDK_WEIGHTING) ? B2T_KER_DEFAULT : ker;  // fdk: weights in coeffs
    for (uint32_t c0 = 0; c0 < d.angles; c0 += BP_MAX_VIEWS) {
        const uint32_t cn = std::min(d.angles - c0, (uint32_t)BP_MAX_VIEWS);
        L.a0 = (int)c0;
        L.nviews = (int)cn;
        L.accumulate = (c0 > 0 || mode == B2T_MODE_ADD) ? 1 : 0;
        for (uint32_t i = 0; i < cn; ++i) bp_view_coeffs(g->kind, ker, g->views[c0 + i], vs, L.views[i]);
        b2t_status st;
        if (dtype == B2T_F32) st = launch_bp_kind<float>(L, g->kind, kker, d, s);
        else if (dtype == B2T_F16) st = launch_bp_kind<__half>(L, g->kind, kker, d, s);
        else st = launch_bp_kind<__nv_bfloat16>(L, g->kind, kker, d, s);
        if (st != B2T_OK) {
            delete Lp;
            return st;
        }
    }
    delete Lp;
    return B2T_OK;
}

}  // namespace b2t
