// Cone beam on a cylindrical detector (cyl_cone_vec): FP, voxel-driven BP and
// the FP's exact transpose, FP32 data.
//
// Reference: cuda/3d/cone_cyl.cu (transferConstants :80-130, cylcone_FP_t
// :197-306, cylcone_BP_t :308-475, host :477-749) and cuda/3d/cone_cyl_bp.cu
// (dev_cylcone_BP :61-160, transferConstants_conecylbp :162-233, host
// :235-320); cylinder axes getCylConeAxes (src/GeometryUtil3D.cpp:542-561).
//
// The views are not scaled to unit voxels (convertAstraGeometry_unscaled):
// positions are in world units and the kernels divide by the voxel size.
//   FP: pixel (u, v) sits at c + a cos(th) + b sin(th) + v_axis (v - nv/2 + 1/2)
//       with th = (u - nu/2 + 1/2) * |u| / R; the ray from the source to it
//       is sampled bilinearly at every slice of the view's dominant axis
//       (of source - detector centre), times sqrt(1 + a1^2 + a2^2) * voxel
//       size along that axis.  Samples come from the zero-padded copies the
//       flat-panel FP uses, over the clipped slice range.
//   BP: for each voxel centre x and view, the ray source -> x meets the
//       cylinder at s + t (x - s) (larger root); the detector is sampled
//       bilinearly (zero border) at the angular and axial coordinates of that
//       point, weight t^2; times the voxel volume.
//   matched BP: the FP's samples scattered back (atomics), the FP's exact
//       transpose: ray set-up and texel split are one shared function.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "b2t_internal.h"
#include "proj3d.h"

namespace b2t {

namespace {

constexpr int CYL_MAX_VIEWS = 384;

// per view, float (rounded from the FP64 host set-up as the reference does)
struct CylFPView {
    float src[3], c[3], a[3], b[3], v[3];
    float ut;  // angular pitch |u| / R
    int a_idx; // global view index
};

struct CylFPLaunch {
    const float *vol;       // FP: padded copy at texel (0, 0, 0) of the marching frame
    float *vout;            // matched BP: the volume (unpadded), [z][y][x]
    long long vol_pitch;    // matched BP: elements per volume row
    long long st0, st2;     // FP: strides of the marching axis and plane axis 2
    float *proj;            // FP output / matched BP input, [v][angle][u]
    const float *proj_in;
    long long proj_pitch;
    int nx, ny, nz, nu, nv, na;
    int n0, n1, n2;         // extents along the marching axis and the plane axes
    int p0, p1, p2;         // world axis of each (0 x, 1 y, 2 z)
    float vs0, vs1, vs2;    // voxel size along each
    float out_scale;
    int accumulate;
    int nviews;
    CylFPView views[CYL_MAX_VIEWS];
};

struct CylBPView {
    float4 ca, cb, cc;  // cylinder axes (radial, tangential, axial) * sqrt|u x v|, w = -src . axis * same
    float sa, sb, sc;   // (src - cylinder centre) . unit axes
    float ut, inv_norm_v, r;
};

struct CylBPLaunch {
    const float *proj;
    long long proj_pitch;
    float *vol;
    long long vol_pitch;
    int nx, ny, nz, nu, nv, na;
    int a0, nviews, accumulate;
    float vsx, vsy, vsz;
    float out_scale;
    CylBPView views[CYL_MAX_VIEWS];
};

// kernel parameter blocks stay under the 32764-byte limit
static_assert(sizeof(CylFPLaunch) <= 32764, "CylFPLaunch too large");
static_assert(sizeof(CylBPLaunch) <= 32764, "CylBPLaunch too large");

// split of qm = (sample index) - 0.5: k = round(qm), f = qm - k + 0.5, sample
// index k + f (the same round-to-nearest split the flat-panel FP uses)
__device__ __forceinline__ void split_cyl(float qm, int &k, float &f)
{
    const float M = 12582912.0f;
    const float t = __fadd_rn(qm, M);
    const float r = __fadd_rn(t, -M);
    k = __float_as_int(t) - 0x4B400000;
    f = __fadd_rn(__fadd_rn(qm, -r), 0.5f);
}

__device__ __forceinline__ void clip_cyl(float A, float B, float lo, float hi, float &smin, float &smax)
{
    if (fabsf(A) < 1e-12f) {
        if (!(B >= lo && B <= hi)) {
            smin = 1.0f;
            smax = 0.0f;
        }
        return;
    }
    const float s1 = __fdiv_rn(lo - B, A), s2 = __fdiv_rn(hi - B, A);
    smin = fmaxf(smin, fminf(s1, s2));
    smax = fminf(smax, fmaxf(s1, s2));
}

__device__ __forceinline__ bool texel_ok_cyl(float A, float B, int s, int n)
{
    int k;
    float f;
    split_cyl(fmaf(A, (float)s, B), k, f);
    return k >= -2 && k <= n;
}

// Ray of pixel (u, v): qm_j(s) = A_j s + B_j for the two plane axes, the
// ray-length factor per slice, and the clipped slice range whose samples can
// touch the volume.  Every product is an explicit fmaf or rounded multiply,
// so the FP and its transpose compute bit-identical samples.
__device__ __forceinline__ void cyl_ray(const CylFPLaunch &L, const CylFPView &V, int u, int v, float &A1,
                                        float &B1, float &A2, float &B2, float &corr, int &s_lo, int &s_hi)
{
    const float th = __fmul_rn(__fmul_rn((float)(2 * u - L.nu + 1), 0.5f), V.ut);
    float sn, cs;
    sincosf(th, &sn, &cs);
    const float dv = (float)v - 0.5f * (float)L.nv + 0.5f;
    const float Dx = fmaf(V.v[0], dv, fmaf(V.b[0], sn, fmaf(V.a[0], cs, V.c[0])));
    const float Dy = fmaf(V.v[1], dv, fmaf(V.b[1], sn, fmaf(V.a[1], cs, V.c[1])));
    const float Dz = fmaf(V.v[2], dv, fmaf(V.b[2], sn, fmaf(V.a[2], cs, V.c[2])));
    auto pick = [](int p, float x, float y, float z) { return p == 0 ? x : (p == 1 ? y : z); };
    const float S0 = V.src[L.p0], S1 = V.src[L.p1], S2 = V.src[L.p2];
    const float den = __fadd_rn(S0, -pick(L.p0, Dx, Dy, Dz));
    float a1 = __fdiv_rn(__fadd_rn(S1, -pick(L.p1, Dx, Dy, Dz)), den);
    float a2 = __fdiv_rn(__fadd_rn(S2, -pick(L.p2, Dx, Dy, Dz)), den);
    corr = __fmul_rn(__fsqrt_rn(fmaf(a1, a1, fmaf(a2, a2, 1.0f))), L.vs0);
    // world slopes -> texel steps; offsets at the world origin of the marching axis
    a1 = __fdiv_rn(a1, L.vs1);
    a2 = __fdiv_rn(a2, L.vs2);
    const float b1 = fmaf(-a1, S0, __fdiv_rn(S1, L.vs1));
    const float b2 = fmaf(-a2, S0, __fdiv_rn(S2, L.vs2));
    a1 = __fmul_rn(a1, L.vs0);
    a2 = __fmul_rn(a2, L.vs0);
    // texture coordinate at slice s: a (s + 1/2 - n0/2) + b + n/2; qm = that - 1
    const float s_off = 0.5f - 0.5f * (float)L.n0;
    A1 = a1;
    A2 = a2;
    B1 = fmaf(a1, s_off, b1) + (0.5f * (float)L.n1 - 1.0f);
    B2 = fmaf(a2, s_off, b2) + (0.5f * (float)L.n2 - 1.0f);
    float smin = 0.0f, smax = (float)(L.n0 - 1);
    clip_cyl(A1, B1, -1.6f, (float)L.n1 - 0.4f, smin, smax);
    clip_cyl(A2, B2, -1.6f, (float)L.n2 - 0.4f, smin, smax);
    s_lo = max(0, (int)ceilf(fmaxf(smin, -1.0f)));
    s_hi = min(L.n0 - 1, (int)floorf(fminf(smax, (float)L.n0)));
    // every access inside the padded copy: the base texel is monotone in s
    for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
        if (texel_ok_cyl(A1, B1, s_lo, L.n1) && texel_ok_cyl(A2, B2, s_lo, L.n2)) break;
        ++s_lo;
    }
    for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
        if (texel_ok_cyl(A1, B1, s_hi, L.n1) && texel_ok_cyl(A2, B2, s_hi, L.n2)) break;
        --s_hi;
    }
    if (!(texel_ok_cyl(A1, B1, s_lo, L.n1) && texel_ok_cyl(A2, B2, s_lo, L.n2) &&
          texel_ok_cyl(A1, B1, s_hi, L.n1) && texel_ok_cyl(A2, B2, s_hi, L.n2)))
        s_hi = s_lo - 1;
}

__global__ void __launch_bounds__(256) fp3d_cyl_kernel(const __grid_constant__ CylFPLaunch L)
{
    const CylFPView &V = L.views[blockIdx.x];
    const int u = blockIdx.y * 32 + threadIdx.x;
    const int v = blockIdx.z * 8 + threadIdx.y;
    if (u >= L.nu || v >= L.nv) return;
    float A1, B1, A2, B2, corr;
    int s_lo, s_hi;
    cyl_ray(L, V, u, v, A1, B1, A2, B2, corr, s_lo, s_hi);
    float sum = 0.0f;
    for (int s = s_lo; s <= s_hi; ++s) {
        int k1, k2;
        float f1, f2;
        split_cyl(fmaf(A1, (float)s, B1), k1, f1);
        split_cyl(fmaf(A2, (float)s, B2), k2, f2);
        const float *p = L.vol + (long long)s * L.st0 + (long long)k2 * L.st2 + k1;
        const float v00 = __ldg(p), v10 = __ldg(p + 1);
        const float v01 = __ldg(p + L.st2), v11 = __ldg(p + L.st2 + 1);
        const float a = fmaf(f1, v10 - v00, v00);
        const float b = fmaf(f1, v11 - v01, v01);
        sum += fmaf(f2, b - a, a);
    }
    float r = sum * corr * L.out_scale;
    float *out = L.proj + ((size_t)v * L.na + V.a_idx) * L.proj_pitch + u;
    if (L.accumulate) r += *out;
    *out = r;
}

// volume element of marching-frame texel (s, k1, k2), or null outside
__device__ __forceinline__ float *cyl_voxel(const CylFPLaunch &L, int s, int k1, int k2)
{
    if (k1 < 0 || k1 >= L.n1 || k2 < 0 || k2 >= L.n2) return nullptr;
    int x, y, z;
    if (L.p0 == 0) { x = s; y = k1; z = k2; }
    else if (L.p0 == 1) { y = s; x = k1; z = k2; }
    else { z = s; x = k1; y = k2; }
    return L.vout + ((size_t)z * L.ny + y) * L.vol_pitch + x;
}

__global__ void __launch_bounds__(256) bp3d_cyl_matched_kernel(const __grid_constant__ CylFPLaunch L)
{
    const CylFPView &V = L.views[blockIdx.x];
    const int u = blockIdx.y * 32 + threadIdx.x;
    const int v = blockIdx.z * 8 + threadIdx.y;
    if (u >= L.nu || v >= L.nv) return;
    float A1, B1, A2, B2, corr;
    int s_lo, s_hi;
    cyl_ray(L, V, u, v, A1, B1, A2, B2, corr, s_lo, s_hi);
    const float w = L.proj_in[((size_t)v * L.na + V.a_idx) * L.proj_pitch + u] * corr * L.out_scale;
    if (w == 0.0f) return;
    for (int s = s_lo; s <= s_hi; ++s) {
        int k1, k2;
        float f1, f2;
        split_cyl(fmaf(A1, (float)s, B1), k1, f1);
        split_cyl(fmaf(A2, (float)s, B2), k2, f2);
        // the FP's sample: (1-f2)((1-f1) v00 + f1 v10) + f2((1-f1) v01 + f1 v11)
        const float w0 = w * (1.0f - f2), w1 = w * f2;
        if (float *p = cyl_voxel(L, s, k1, k2)) atomicAdd(p, w0 * (1.0f - f1));
        if (float *p = cyl_voxel(L, s, k1 + 1, k2)) atomicAdd(p, w0 * f1);
        if (float *p = cyl_voxel(L, s, k1, k2 + 1)) atomicAdd(p, w1 * (1.0f - f1));
        if (float *p = cyl_voxel(L, s, k1 + 1, k2 + 1)) atomicAdd(p, w1 * f1);
    }
}

// bilinear sample of detector row-major plane (view a) at index (qu, qv), zero outside
__device__ __forceinline__ float sample_det(const CylBPLaunch &L, int a, float qu, float qv)
{
    if (!(fabsf(qu) < 1.0e7f && fabsf(qv) < 1.0e7f)) return 0.0f;  // also NaN
    const float fu = floorf(qu), fv = floorf(qv);
    const int ku = (int)fu, kv = (int)fv;
    const float tu = qu - fu, tv = qv - fv;
    if (ku < -1 || ku >= L.nu || kv < -1 || kv >= L.nv) return 0.0f;
    const float *row = L.proj + (size_t)a * L.proj_pitch;
    const long long pv = (long long)L.na * L.proj_pitch;
    auto at = [&](int iu, int iv) -> float {
        return (iu >= 0 && iu < L.nu && iv >= 0 && iv < L.nv) ? __ldg(row + iv * pv + iu) : 0.0f;
    };
    const float a0 = fmaf(tu, at(ku + 1, kv) - at(ku, kv), at(ku, kv));
    const float a1 = fmaf(tu, at(ku + 1, kv + 1) - at(ku, kv + 1), at(ku, kv + 1));
    return fmaf(tv, a1 - a0, a0);
}

// sample_det with the u split done once for a column of voxels: ku, tu and
// the validity of columns ku, ku + 1 (cu0, cu1) from sample_det's rules
__device__ __forceinline__ float sample_det_col(const CylBPLaunch &L, const float *row, int ku, float tu, bool cu0,
                                                bool cu1, float qv)
{
    if (!(fabsf(qv) < 1.0e7f)) return 0.0f;  // also NaN
    const float fv = floorf(qv);
    const int kv = (int)fv;
    const float tv = qv - fv;
    if (kv < -1 || kv >= L.nv) return 0.0f;
    const long long pv = (long long)L.na * L.proj_pitch;
    const bool r0 = kv >= 0, r1 = kv + 1 < L.nv;
    const float *p0 = row + (long long)kv * pv + ku;
    const float v00 = (cu0 && r0) ? __ldg(p0) : 0.0f, v10 = (cu1 && r0) ? __ldg(p0 + 1) : 0.0f;
    const float v01 = (cu0 && r1) ? __ldg(p0 + pv) : 0.0f, v11 = (cu1 && r1) ? __ldg(p0 + pv + 1) : 0.0f;
    const float a0 = fmaf(tu, v10 - v00, v00);
    const float a1 = fmaf(tu, v11 - v01, v01);
    return fmaf(tv, a1 - a0, a0);
}

constexpr int CYL_BP_Z = 16;

__global__ void __launch_bounds__(256) bp3d_cyl_kernel(const __grid_constant__ CylBPLaunch L)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * CYL_BP_Z;
    if (x >= L.nx || y >= L.ny) return;
    const float fx = L.vsx * ((float)x - 0.5f * (float)L.nx + 0.5f);
    const float fy = L.vsy * ((float)y - 0.5f * (float)L.ny + 0.5f);
    const float fz0 = L.vsz * ((float)z0 - 0.5f * (float)L.nz + 0.5f);
    float acc[CYL_BP_Z];
#pragma unroll
    for (int j = 0; j < CYL_BP_Z; ++j) acc[j] = 0.0f;
    for (int i = 0; i < L.nviews; ++i) {
        const CylBPView &C = L.views[i];
        float ra = fmaf(fz0, C.ca.z, fmaf(fy, C.ca.y, fmaf(fx, C.ca.x, C.ca.w)));
        float rb = fmaf(fz0, C.cb.z, fmaf(fy, C.cb.y, fmaf(fx, C.cb.x, C.cb.w)));
        float rc = fmaf(fz0, C.cc.z, fmaf(fy, C.cc.y, fmaf(fx, C.cc.x, C.cc.w)));
        const float cq = fmaf(C.sa, C.sa, fmaf(C.sb, C.sb, -C.r * C.r));
        if (C.ca.z == 0.0f && C.cb.z == 0.0f) {
            // cylinder axis along z: the ray's in-plane part does not change
            // along the voxel column, so t and the hit angle are the
            // column's (the same values the general loop computes per voxel)
            const float qa = fmaf(ra, ra, rb * rb);
            const float qb = fmaf(ra, C.sa, rb * C.sb);
            const float disc = fmaf(qb, qb, -qa * cq);
            if (!(disc >= 0.0f && qa > 0.0f)) continue;
            const float t = (sqrtf(disc) - qb) / qa;
            const float th = asinf(fmaf(t, rb, C.sb) / C.r) / C.ut;
            const float qu = th + 0.5f * (float)L.nu - 0.5f;
            if (!(fabsf(qu) < 1.0e7f)) continue;
            const float fu = floorf(qu);
            const int ku = (int)fu;
            const float tu = qu - fu;
            if (ku < -1 || ku >= L.nu) continue;
            const bool cu0 = ku >= 0, cu1 = ku + 1 < L.nu;
            const float *row = L.proj + (size_t)(L.a0 + i) * L.proj_pitch;
            const float w = t * t;
#pragma unroll
            for (int j = 0; j < CYL_BP_Z; ++j) {
                const float vv = fmaf(t, rc, C.sc) * C.inv_norm_v;
                acc[j] = fmaf(sample_det_col(L, row, ku, tu, cu0, cu1, vv + 0.5f * (float)L.nv - 0.5f), w, acc[j]);
                rc = fmaf(L.vsz, C.cc.z, rc);
            }
            continue;
        }
#pragma unroll
        for (int j = 0; j < CYL_BP_Z; ++j) {
            // |smc_ab + t r_ab| = R, larger root
            const float qa = fmaf(ra, ra, rb * rb);
            const float qb = fmaf(ra, C.sa, rb * C.sb);
            const float disc = fmaf(qb, qb, -qa * cq);
            if (disc >= 0.0f && qa > 0.0f) {
                const float t = (sqrtf(disc) - qb) / qa;
                const float th = asinf(fmaf(t, rb, C.sb) / C.r) / C.ut;
                const float vv = fmaf(t, rc, C.sc) * C.inv_norm_v;
                // texture coordinates th + nu/2, vv + nv/2; sample index = that - 1/2
                const float val = sample_det(L, L.a0 + i, th + 0.5f * (float)L.nu - 0.5f,
                                             vv + 0.5f * (float)L.nv - 0.5f);
                acc[j] = fmaf(val, t * t, acc[j]);
            }
            ra = fmaf(L.vsz, C.ca.z, ra);
            rb = fmaf(L.vsz, C.cb.z, rb);
            rc = fmaf(L.vsz, C.cc.z, rc);
        }
    }
#pragma unroll
    for (int j = 0; j < CYL_BP_Z; ++j) {
        const int z = z0 + j;
        if (z < L.nz) {
            float *o = L.vol + ((size_t)z * L.ny + y) * L.vol_pitch + x;
            const float r = acc[j] * L.out_scale;
            *o = L.accumulate ? *o + r : r;
        }
    }
}

// ---------------------------------------------------------------------------
// host set-up
// ---------------------------------------------------------------------------

struct V3 {
    double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 vec(const double *p) { return {p[0], p[1], p[2]}; }

// getCylConeAxes (src/GeometryUtil3D.cpp:542-561): radial a (towards the
// detector from the cylinder centre), cylinder centre c, tangential b
struct CylAxes {
    V3 a, b, c;
};
CylAxes cyl_axes(const b2t_view3d_cyl &w)
{
    const V3 u = vec(w.det_u), v = vec(w.det_v), s = vec(w.src), d = vec(w.det_c);
    const double R = w.radius;
    V3 a = cross(u, v) * (-R / (norm(u) * norm(v)));
    if (norm(d - a - s) > norm(d + a - s)) a = a * -1.0;
    return {a, u * (R / norm(u)), d - a};
}

// dominant axis of source - detector centre, compared in float as
// ConeCylFP_Array_internal does (cone_cyl.cu:491-503)
int cyl_dir(const b2t_view3d_cyl &w)
{
    const float dX = fabsf((float)(w.src[0] - w.det_c[0]));
    const float dY = fabsf((float)(w.src[1] - w.det_c[1]));
    const float dZ = fabsf((float)(w.src[2] - w.det_c[2]));
    if (dX >= dY && dX >= dZ) return 0;
    if (dY >= dX && dY >= dZ) return 1;
    return 2;
}

void cyl_fp_view(const b2t_view3d_cyl &w, int a, CylFPView &o)
{
    const CylAxes ax = cyl_axes(w);
    const double ca[3] = {ax.a.x, ax.a.y, ax.a.z}, cb[3] = {ax.b.x, ax.b.y, ax.b.z}, cc[3] = {ax.c.x, ax.c.y, ax.c.z};
    for (int k = 0; k < 3; ++k) {
        o.src[k] = (float)w.src[k];
        o.c[k] = (float)cc[k];
        o.a[k] = (float)ca[k];
        o.b[k] = (float)cb[k];
        o.v[k] = (float)w.det_v[k];
    }
    o.ut = (float)(norm(vec(w.det_u)) / w.radius);
    o.a_idx = a;
}

// transferConstants_conecylbp (cone_cyl_bp.cu:162-233)
void cyl_bp_view(const b2t_view3d_cyl &w, CylBPView &o)
{
    const CylAxes ax = cyl_axes(w);
    const V3 u = vec(w.det_u), v = vec(w.det_v), s = vec(w.src);
    const V3 an = ax.a * (1.0 / norm(ax.a)), bn = ax.b * (1.0 / norm(ax.b)), vn = v * (1.0 / norm(v));
    const double sc = std::sqrt(norm(cross(u, v)));
    o.ca = make_float4((float)(an.x * sc), (float)(an.y * sc), (float)(an.z * sc), (float)(-dot(s, an) * sc));
    o.cb = make_float4((float)(bn.x * sc), (float)(bn.y * sc), (float)(bn.z * sc), (float)(-dot(s, bn) * sc));
    o.cc = make_float4((float)(vn.x * sc), (float)(vn.y * sc), (float)(vn.z * sc), (float)(-dot(s, vn) * sc));
    const V3 smc = s - ax.c;
    o.sa = (float)dot(smc, an);
    o.sb = (float)dot(smc, bn);
    o.sc = (float)dot(smc, vn);
    o.ut = (float)(norm(u) / w.radius);
    o.inv_norm_v = (float)(1.0 / norm(v));
    o.r = (float)w.radius;
}

b2t_status validate_cyl(const b2t_geom3d_cyl *g, const b2t_params3d *p, const char *who)
{
    if (!g || !g->views || !p) return fail(B2T_ERR_INVALID_ARG, "%s: null geometry or params", who);
    const b2t_dims3d &d = g->dims;
    if (d.vol_x == 0 || d.vol_y == 0 || d.vol_z == 0 || d.angles == 0 || d.det_u == 0 || d.det_v == 0)
        return fail(B2T_ERR_INVALID_ARG, "%s: empty dimension", who);
    if (d.vol_x > (1u << 20) || d.vol_y > (1u << 20) || d.vol_z > (1u << 20) || d.det_u > (1u << 20) ||
        d.det_v > (1u << 20))
        return fail(B2T_ERR_INVALID_ARG, "%s: dimension above 2^20", who);
    for (int k = 0; k < 3; ++k)
        if (!(g->vol_scale[k] > 0.0f)) return fail(B2T_ERR_INVALID_ARG, "%s: voxel size must be > 0", who);
    for (uint32_t i = 0; i < d.angles; ++i)
        if (!(g->views[i].radius > 0.0)) return fail(B2T_ERR_INVALID_ARG, "%s: radius must be > 0", who);
    if (p->det_supersample > 1 || p->voxel_supersample > 1)
        return fail(B2T_ERR_UNSUPPORTED, "%s: no supersampling for cyl_cone_vec, as the reference", who);
    return B2T_OK;
}

// the marching frame of direction dir: permutation, extents, voxel sizes
void cyl_frame(int dir, const b2t_geom3d_cyl *g, CylFPLaunch &P)
{
    static const int perm[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
    const uint32_t n[3] = {g->dims.vol_x, g->dims.vol_y, g->dims.vol_z};
    P.p0 = perm[dir][0];
    P.p1 = perm[dir][1];
    P.p2 = perm[dir][2];
    P.n0 = (int)n[P.p0];
    P.n1 = (int)n[P.p1];
    P.n2 = (int)n[P.p2];
    P.vs0 = g->vol_scale[P.p0];
    P.vs1 = g->vol_scale[P.p1];
    P.vs2 = g->vol_scale[P.p2];
}

// Group the views by direction and launch `kern` per group and chunk.
template <typename Launch>
b2t_status cyl_fp_like(const b2t_geom3d_cyl *g, CylFPLaunch &P, Launch launch)
{
    std::vector<int> dirs(g->dims.angles);
    for (uint32_t a = 0; a < g->dims.angles; ++a) dirs[a] = cyl_dir(g->views[a]);
    for (int dir = 0; dir < 3; ++dir) {
        std::vector<int> views;
        for (uint32_t a = 0; a < g->dims.angles; ++a)
            if (dirs[a] == dir) views.push_back((int)a);
        if (views.empty()) continue;
        cyl_frame(dir, g, P);
        for (size_t c0 = 0; c0 < views.size(); c0 += CYL_MAX_VIEWS) {
            const size_t cn = std::min(views.size() - c0, (size_t)CYL_MAX_VIEWS);
            P.nviews = (int)cn;
            for (size_t i = 0; i < cn; ++i) cyl_fp_view(g->views[views[c0 + i]], views[c0 + i], P.views[i]);
            const dim3 grid((unsigned)cn, (g->dims.det_u + 31) / 32, (g->dims.det_v + 7) / 8);
            B2T_TRY(launch(dir, grid));
        }
    }
    return B2T_OK;
}

}  // namespace

b2t_status fp3d_cyl_impl(const b2t_geom3d_cyl *g, const b2t_params3d *p, const float *vol, size_t vol_pitch,
                         float *proj, size_t proj_pitch, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate_cyl(g, p, "b2t_fp3d_cyl"));
    if (!vol || !proj) return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d_cyl: null data pointer");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d_cyl: bad mode");
    if (p->kernel == B2T_KER_SUM_SQUARE_WEIGHTS)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_fp3d_cyl: sum_square_weights needs a parallel-beam geometry");
    const b2t_dims3d &d = g->dims;
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (vol_pitch < d.vol_x || proj_pitch < d.det_u)
        return fail(B2T_ERR_INVALID_ARG, "b2t_fp3d_cyl: pitch below row length");
    bool need[3] = {false, false, false};
    for (uint32_t a = 0; a < d.angles; ++a) need[cyl_dir(g->views[a])] = true;
    const size_t px = d.vol_x + 4, py = d.vol_y + 4, pz = d.vol_z + 4, padded = px * py * pz;
    Scratch sa, sb;
    if (need[1] || need[2]) B2T_TRY(sa.alloc(padded * sizeof(float), s, "b2t_fp3d_cyl scratch (xyz copy)"));
    if (need[0]) B2T_TRY(sb.alloc(padded * sizeof(float), s, "b2t_fp3d_cyl scratch (zxy copy)"));
    B2T_TRY(pad_volumes_f32(vol, vol_pitch, d, (need[1] || need[2]) ? sa.as<float>() : nullptr,
                            need[0] ? sb.as<float>() : nullptr, s));
    std::unique_ptr<CylFPLaunch> P(new CylFPLaunch());
    P->proj = proj;
    P->proj_pitch = (long long)proj_pitch;
    P->nx = d.vol_x; P->ny = d.vol_y; P->nz = d.vol_z;
    P->nu = d.det_u; P->nv = d.det_v; P->na = d.angles;
    P->out_scale = p->output_scale;
    P->accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
    return cyl_fp_like(g, *P, [&](int dir, dim3 grid) -> b2t_status {
        // padded copy of this direction, at texel (0, 0, 0) of the marching frame
        const float *base;
        if (dir == 0) {
            base = sb.as<float>();
            P->st0 = (long long)py;
            P->st2 = (long long)(px * py);
            base += 2 * P->st2 + 2 * P->st0 + 2;
        } else if (dir == 1) {
            base = sa.as<float>();
            P->st0 = (long long)px;
            P->st2 = (long long)(px * py);
            base += 2 * P->st2 + 2 * P->st0 + 2;
        } else {
            base = sa.as<float>();
            P->st0 = (long long)(px * py);
            P->st2 = (long long)px;
            base += 2 * P->st0 + 2 * P->st2 + 2;
        }
        P->vol = base;
        fp3d_cyl_kernel<<<grid, dim3(32, 8), 0, s>>>(*P);
        count_launches(1);
        B2T_CUDA_TRY(cudaGetLastError(), "fp3d_cyl_kernel launch");
        return B2T_OK;
    });
}

b2t_status bp3d_cyl_impl(const b2t_geom3d_cyl *g, const b2t_params3d *p, const float *proj, size_t proj_pitch,
                         float *vol, size_t vol_pitch, int32_t mode, cudaStream_t s)
{
    B2T_TRY(validate_cyl(g, p, "b2t_bp3d_cyl"));
    if (!vol || !proj) return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d_cyl: null data pointer");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d_cyl: bad mode");
    if (p->kernel != B2T_KER_DEFAULT && p->kernel != B2T_KER_MATCHED_BP)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_bp3d_cyl: kernel %d (DEFAULT or MATCHED_BP only)", p->kernel);
    const b2t_dims3d &d = g->dims;
    if (vol_pitch == 0) vol_pitch = d.vol_x;
    if (proj_pitch == 0) proj_pitch = d.det_u;
    if (vol_pitch < d.vol_x || proj_pitch < d.det_u)
        return fail(B2T_ERR_INVALID_ARG, "b2t_bp3d_cyl: pitch below row length");
    if (p->kernel == B2T_KER_MATCHED_BP) {
        if (mode == B2T_MODE_SET) {
            B2T_CUDA_TRY(cudaMemset2DAsync(vol, vol_pitch * sizeof(float), 0, d.vol_x * sizeof(float),
                                           (size_t)d.vol_y * d.vol_z, s),
                         "b2t_bp3d_cyl clear");
        }
        std::unique_ptr<CylFPLaunch> P(new CylFPLaunch());
        P->vout = vol;
        P->vol_pitch = (long long)vol_pitch;
        P->proj_in = proj;
        P->proj_pitch = (long long)proj_pitch;
        P->nx = d.vol_x; P->ny = d.vol_y; P->nz = d.vol_z;
        P->nu = d.det_u; P->nv = d.det_v; P->na = d.angles;
        P->out_scale = p->output_scale;
        return cyl_fp_like(g, *P, [&](int, dim3 grid) -> b2t_status {
            bp3d_cyl_matched_kernel<<<grid, dim3(32, 8), 0, s>>>(*P);
            count_launches(1);
            B2T_CUDA_TRY(cudaGetLastError(), "bp3d_cyl_matched_kernel launch");
            return B2T_OK;
        });
    }
    std::unique_ptr<CylBPLaunch> L(new CylBPLaunch());
    L->proj = proj;
    L->proj_pitch = (long long)proj_pitch;
    L->vol = vol;
    L->vol_pitch = (long long)vol_pitch;
    L->nx = d.vol_x; L->ny = d.vol_y; L->nz = d.vol_z;
    L->nu = d.det_u; L->nv = d.det_v; L->na = d.angles;
    L->vsx = g->vol_scale[0]; L->vsy = g->vol_scale[1]; L->vsz = g->vol_scale[2];
    // ConeCylBP_Array (cone_cyl_bp.cu:248): output scale times the voxel volume
    L->out_scale = p->output_scale * (g->vol_scale[0] * g->vol_scale[1] * g->vol_scale[2]);
    const dim3 grid((d.vol_x + 31) / 32, (d.vol_y + 7) / 8, (d.vol_z + CYL_BP_Z - 1) / CYL_BP_Z);
    for (uint32_t c0 = 0; c0 < d.angles; c0 += CYL_MAX_VIEWS) {
        const uint32_t cn = std::min(d.angles - c0, (uint32_t)CYL_MAX_VIEWS);
        L->a0 = (int)c0;
        L->nviews = (int)cn;
        L->accumulate = (c0 > 0 || mode == B2T_MODE_ADD) ? 1 : 0;
        for (uint32_t i = 0; i < cn; ++i) cyl_bp_view(g->views[c0 + i], L->views[i]);
        bp3d_cyl_kernel<<<grid, dim3(32, 8), 0, s>>>(*L);
        count_launches(1);
        B2T_CUDA_TRY(cudaGetLastError(), "bp3d_cyl_kernel launch");
    }
    return B2T_OK;
}

}  // namespace b2t
