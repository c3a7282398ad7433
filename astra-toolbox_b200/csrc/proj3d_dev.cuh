// Device-side bodies of the direct-load 3D projectors, shared by the
// single-problem kernels (proj3d.cu) and the batched persistent kernels
// (batch3d.cu): one detector ray of a forward projection, one column of
// voxels of a backprojection.
//
// Model: the reference's cone_FP / par3D_FP ray marching (cuda/3d/
// cone_fp.cu:154-231, cuda/3d/par3d_fp.cu:146-220) and dev_cone_BP /
// dev_par3D_BP (cuda/3d/cone_bp.cu:55-133, cuda/3d/par3d_bp.cu:55-120), with
// explicit FP32 interpolation in place of texture fetches.  The texel reads
// go through a loader: a zero-padded copy read without checks (the
// single-problem kernels), or the caller's own array read with bounds checks
// (zero outside, the batched kernels); both give the same values, so the
// arithmetic and the results are the same.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "proj3d.h"

namespace b2t {

template <typename T> __device__ __forceinline__ float ld(const T *p);
template <> __device__ __forceinline__ float ld<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(__ldg(p));
}

template <typename T> __device__ __forceinline__ float ldplain(const T *p);
template <> __device__ __forceinline__ float ldplain<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float ldplain<__half>(const __half *p) { return __half2float(*p); }
template <> __device__ __forceinline__ float ldplain<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(*p);
}

template <typename T> __device__ __forceinline__ T from_float(float v);
template <> __device__ __forceinline__ float from_float<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_float<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_float<__nv_bfloat16>(float v)
{
    return __float2bfloat16_rn(v);
}

// Split a continuous texel index q (texel i at q = i) into the base texel
// k = floor(q) and the weight f = q - k, using the round-to-nearest of the
// FP32 adder (q - 0.5 + 1.5*2^23 holds rint(q - 0.5) in its mantissa) rather
// than the conversion pipe.  qm = q - 0.5 is passed in; valid for |q| < 2^22.
// At exact ties either neighbour is chosen and f is 0 or 1, which selects the
// same texel value.
__device__ __forceinline__ void split_texel(float qm, int &k, float &f)
{
    const float M = 12582912.0f;  // 1.5 * 2^23
    float t = __fadd_rn(qm, M);
    float r = __fadd_rn(t, -M);
    k = __float_as_int(t) - 0x4B400000;
    f = __fadd_rn(__fadd_rn(qm, -r), 0.5f);
}

// Clip the slice range [smin, smax] to where lo <= A*s + B <= hi.
__device__ __forceinline__ void clip_slices(float A, float B, float lo, float hi, float &smin, float &smax)
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

// The FP's split (shared with the cell kernels and the matched BP): sample
// position plus one half qh = A s + (B + 1/2); texel floor(qh) by rounding
// down, weight qh - floor(qh).
constexpr float SPLIT_M = 12582912.0f;  // 1.5 * 2^23
__device__ __forceinline__ void split_floor(float qh, int &k, float &f)
{
    const float t = __fadd_rd(qh, SPLIT_M);
    k = __float_as_int(t) - 0x4B400000;
    f = qh - (t - SPLIT_M);
}

__device__ __forceinline__ bool fp_texel_ok(float A, float Bh, int s, int n)
{
    int k;
    float f;
    split_floor(fmaf(A, (float)s, Bh), k, f);
    return k >= -2 && k <= n;
}

// FP texels (s, k1, k2) of the view's frame (s along the marching axis) from
// a zero-padded copy whose k1 axis is contiguous: every index the ray
// reaches lies inside the copy's 2-texel border.
template <typename T> struct FPPadded {
    const T *base;  // texel (0, 0, 0)
    long long st0, st2;
    __device__ __forceinline__ void quad(int s, int k1, int k2, float &v00, float &v10, float &v01,
                                         float &v11) const
    {
        const T *p = base + (long long)s * st0 + (long long)k2 * st2 + k1;
        v00 = ld(p);
        v10 = ld(p + 1);
        v01 = ld(p + st2);
        v11 = ld(p + st2 + 1);
    }
};

// The same from an unpadded FP32 volume with any strides, zero outside
// [0, n1) x [0, n2) (s is always inside).
struct FPChecked {
    const float *base;
    long long st0, st1, st2;
    int n1, n2;
    __device__ __forceinline__ float at(int s, int k1, int k2) const
    {
        return (k1 >= 0 && k1 < n1 && k2 >= 0 && k2 < n2)
                   ? __ldg(base + (long long)s * st0 + (long long)k1 * st1 + (long long)k2 * st2)
                   : 0.0f;
    }
    __device__ __forceinline__ void quad(int s, int k1, int k2, float &v00, float &v10, float &v01,
                                         float &v11) const
    {
        v00 = at(s, k1, k2);
        v10 = at(s, k1 + 1, k2);
        v01 = at(s, k1, k2 + 1);
        v11 = at(s, k1 + 1, k2 + 1);
    }
};

// The samples of detector pixel (u, v) of view V (R x R sub-rays): the
// marching axis has n0 slices, the in-plane axes n1 and n2 texels.  For each
// sub-ray, visit.begin(sc) with the sub-ray's scale, visit.sample(s, k1, fa,
// k2, fb) for each slice s it crosses (bilinear base texel (k1, k2) and
// weights (fa, fb) of slice s), then visit.end(sc).
template <typename Visit>
__device__ __forceinline__ void fp3d_ray_walk(const FPView &V, int u, int v, int n0, int n1, int n2, int nu, int nv,
                                              int R, float f1, float f2, float mul, Visit &visit)
{
    const float fn0 = (float)n0;
    for (int iu = 0; iu < R; ++iu) {
        for (int iv = 0; iv < R; ++iv) {
            // detector position relative to the detector centre, in pixels
            float uu = (float)u + 0.5f - 0.5f * (float)nu;
            float vv = (float)v + 0.5f - 0.5f * (float)nv;
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
            // slices whose sample can touch the volume: q - 0.5 in [-1.5, n - 0.5)
            float smin = 0.0f, smax = fn0 - 1.0f;
            clip_slices(A1, B1, -1.6f, (float)n1 - 0.4f, smin, smax);
            clip_slices(A2, B2, -1.6f, (float)n2 - 0.4f, smin, smax);
            int s_lo = max(0, (int)ceilf(fmaxf(smin, -1.0f)));
            int s_hi = min(n0 - 1, (int)floorf(fminf(smax, fn0)));
            const float B1h = B1 + 0.5f, B2h = B2 + 0.5f;
            // keep every access within the 2-texel border: the base texel
            // is monotone in s, so checking the end points suffices
            for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
                if (fp_texel_ok(A1, B1h, s_lo, n1) && fp_texel_ok(A2, B2h, s_lo, n2)) break;
                ++s_lo;
            }
            for (int it = 0; it < 3 && s_lo <= s_hi; ++it) {
                if (fp_texel_ok(A1, B1h, s_hi, n1) && fp_texel_ok(A2, B2h, s_hi, n2)) break;
                --s_hi;
            }
            if (!(fp_texel_ok(A1, B1h, s_lo, n1) && fp_texel_ok(A2, B2h, s_lo, n2) &&
                  fp_texel_ok(A1, B1h, s_hi, n1) && fp_texel_ok(A2, B2h, s_hi, n2)))
                s_hi = s_lo - 1;
            const float sc = sqrtf(fmaf(A1 * A1, f1, fmaf(A2 * A2, f2, 1.0f))) * mul;
            visit.begin(sc);
            for (int s = s_lo; s <= s_hi; ++s) {
                int k1, k2;
                float fa, fb;
                split_floor(fmaf(A1, (float)s, B1h), k1, fa);
                split_floor(fmaf(A2, (float)s, B2h), k2, fb);
                visit.sample(s, k1, fa, k2, fb);
            }
            visit.end(sc);
        }
    }
}

// Line integral of detector pixel (u, v) of view V, scaled (the R x R
// sub-rays averaged), reading the texels through loader Ld.
template <typename Loader> struct FPSum {
    const Loader &Ld;
    float acc, sum;
    __device__ __forceinline__ void begin(float) { sum = 0.0f; }
    __device__ __forceinline__ void sample(int s, int k1, float fa, int k2, float fb)
    {
        float v00, v10, v01, v11;
        Ld.quad(s, k1, k2, v00, v10, v01, v11);
        const float a = fmaf(fa, v10 - v00, v00);
        const float b = fmaf(fa, v11 - v01, v01);
        sum += fmaf(fb, b - a, a);
    }
    __device__ __forceinline__ void end(float sc) { acc = fmaf(sum, sc, acc); }
};

template <typename Loader>
__device__ __forceinline__ float fp3d_ray(const Loader &Ld, const FPView &V, int u, int v, int n0, int n1, int n2,
                                          int nu, int nv, int R, float f1, float f2, float mul)
{
    FPSum<Loader> S{Ld, 0.0f, 0.0f};
    fp3d_ray_walk(V, u, v, n0, n1, n2, nu, nv, R, f1, f2, mul, S);
    float acc = S.acc;
    if (R > 1) acc /= (float)(R * R);
    return acc;
}

// BP texels (view a, row kv, column ku) from the zero-padded projections
// [v][angle][u] (rows pv elements apart, views pu): ku, kv within the
// 2-texel border.
template <typename T> struct BPPadded {
    const T *base;  // texel (u 0, angle 0, v 0)
    long long pv;
    int pu;
    __device__ __forceinline__ void quad(int a, int kv, int ku, float &v00, float &v10, float &v01,
                                         float &v11) const
    {
        const T *p = base + (long long)a * pu + (long long)kv * pv + ku;
        v00 = ld(p);
        v10 = ld(p + 1);
        v01 = ld(p + pv);
        v11 = ld(p + pv + 1);
    }
};

// The same from the caller's FP32 projections [v][angle][u] (rows of nu
// texels), zero outside the detector.
struct BPChecked {
    const float *base;
    int nu, nv, na;
    __device__ __forceinline__ float at(int a, int kv, int ku) const
    {
        return (ku >= 0 && ku < nu && kv >= 0 && kv < nv) ? __ldg(base + ((long long)kv * na + a) * nu + ku) : 0.0f;
    }
    __device__ __forceinline__ void quad(int a, int kv, int ku, float &v00, float &v10, float &v01,
                                         float &v11) const
    {
        v00 = at(a, kv, ku);
        v10 = at(a, kv, ku + 1);
        v01 = at(a, kv + 1, ku);
        v11 = at(a, kv + 1, ku + 1);
    }
};

// Unscaled sums of ZB voxels (fx, fy, fz + j), j < ZB, over views [0, nviews)
// of `views` (texels of view i are view a0 + i of the loader's data).
template <int KIND, int KER, int ZB, typename Loader>
__device__ __forceinline__ void bp3d_column(const Loader &Ld, const BPView *views, int nviews, int a0, int nu,
                                            int nv, float fx, float fy, float fz, float *acc)
{
#pragma unroll
    for (int j = 0; j < ZB; ++j) acc[j] = 0.0f;
    for (int i = 0; i < nviews; ++i) {
        const BPView &W = views[i];
        float snu = fmaf(fz, W.nu.z, fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)));
        float snv = fmaf(fz, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
        float dn = fmaf(fz, W.den.z, fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w)));
#pragma unroll
        for (int j = 0; j < ZB; ++j) {
            float U, Vc, w;
            if (KIND == B2T_GEOM_CONE) {
                const float fr = __frcp_rn(dn);
                U = snu * fr;
                Vc = snv * fr;
                w = (KER == B2T_KER_2D_WEIGHTING) ? fr : fr * fr;
            } else {
                U = snu;
                Vc = snv;
                w = W.den.w;
            }
            // texture coordinates (U, V): texel i at i + 0.5 -> q - 0.5 = U - 1
            int ku, kv;
            float fu, fv;
            split_texel(U - 1.0f, ku, fu);
            split_texel(Vc - 1.0f, kv, fv);
            ku = min(max(ku, -2), nu);
            kv = min(max(kv, -2), nv);
            float v00, v10, v01, v11;
            Ld.quad(a0 + i, kv, ku, v00, v10, v01, v11);
            const float a = fmaf(fu, v10 - v00, v00);
            const float b = fmaf(fu, v11 - v01, v01);
            acc[j] = fmaf(fmaf(fv, b - a, a), w, acc[j]);
            snu += W.nu.z;
            snv += W.nv.z;
            dn += W.den.z;
        }
    }
}

}  // namespace b2t
