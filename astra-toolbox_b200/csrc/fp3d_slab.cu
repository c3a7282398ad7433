// Ray-driven 3D forward projection from TMA-staged volume slabs.
//
// Same model as fp3d_kernel / the cell kernels (the reference's cone_FP_t /
// par3D_FP_t, cuda/3d/cone_fp.cu:154-231, cuda/3d/par3d_fp.cu:152-230): per
// ray, the slices of the view's dominant axis are sampled bilinearly at unit
// steps and the sum is scaled by the ray length factor.
//
// For views that march along x or y and whose detector v axis has no
// component along the marching axis or the in-plane axis (every circular
// orbit, parallel or cone), all rays of one detector column lie in a plane
// that contains the z direction: at every slice they share the in-plane
// texel and its weight, and only their z position differs.  The kernel is
// built on that:
//
//   - the volume is copied once per call and marching axis into a slab copy
//     of z-pairs [slice][in-plane texel + 2][z texel + 2] holding
//     (v[z], v[z + 1] - v[z]) (z contiguous, a zero border of two texels), so
//     a bilinear sample is two 8-byte loads and two FMAs along z;
//   - a CTA traces SLAB_W consecutive views x SLAB_U consecutive detector
//     columns x SLAB_ROWS detector rows; a compute warp owns one column, each
//     lane SLAB_R rows of it (v, v + 32, ...) in both views, so the in-plane
//     position, texel split and buffer row of a slice are computed once per
//     view for SLAB_R rays and the slice's wait and release once for all
//     SLAB_W x SLAB_R of them;
//   - a producer warp works out the buffer box of 32 slices at a time (one
//     slice per lane) from the tile's corner rays (the rays of a detector
//     rectangle cross a slice in the convex hull of its corners' crossings),
//     clamped to the zero border, and loads each slice's box with 4-row
//     cp.async.bulk.tensor boxes of one of two widths (96 or 160 texels;
//     plain tile loads, no multicast) into one of SLAB_STAGES slice buffers;
//     a box lands densely, so its width is the buffer's row pitch;
//   - compute warps interpolate from shared memory in FP32.  Samples outside
//     the volume read the zero border (positions clamped to it on the slices
//     where some ray of the warp leaves the volume);
//   - a slice whose box does not fit a buffer (extreme magnification) is read
//     from the slab copy in global memory instead.
//
// Every mbarrier wait is bounded (about a second); on a timeout the kernel
// sets B2T_DEVERR_WAIT_TIMEOUT in its error word, lets its own copies land
// and returns.  The reference has no such kernel; its FP samples a 3D
// texture per slice (cone_fp.cu:154-231).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <string>
#include <vector>

#include "b2t_internal.h"
#include "f32x2.cuh"
#include "proj3d.h"
#include "tma.h"

namespace b2t {

// error word of this translation unit (read by b2t_device_errors)
static __device__ unsigned int g_fp_slab_errors = 0;
// slices staged in shared memory / read from global memory, summed over CTAs
// (read and cleared by b2t_fp_path_stats)
static __device__ unsigned long long g_fp_slab_slices[2] = {0, 0};
// the same for the transpose (slices whose box went through shared memory /
// scattered straight into the accumulator; read by b2t_matched_path_stats)
static __device__ unsigned long long g_mt_slab_slices[2] = {0, 0};

namespace {

constexpr int SLAB_W = 2;                   // views per CTA (every warp traces both)
constexpr int SLAB_U = 11;                  // detector columns per CTA, one compute warp each
constexpr int SLAB_R = 5;                   // rows per lane and view: v, v + 32, ... (384 threads:
                                            // 80 registers at two CTAs per SM, no spills)
constexpr int SLAB_ROWS = 32 * SLAB_R;      // detector rows per CTA
constexpr int SLAB_WARPS = SLAB_U;          // compute warps; one more produces
constexpr int SLAB_THREADS = 32 * (SLAB_WARPS + 1);
constexpr int SLAB_BY = 24;                 // buffer rows (in-plane texels) per slice
constexpr int SLAB_WA = 96, SLAB_WB = 160;  // box widths (z-pairs): the buffer row pitch of a slice
constexpr int SLAB_BOX_Y = 4;               // rows per TMA box
constexpr int SLAB_STAGES = 3;              // slices in flight
constexpr int SLAB_SLOT = SLAB_BY * SLAB_WB;  // z-pairs per slice buffer
constexpr int SLAB_MAX_VIEWS = 448;
constexpr long long SLAB_WAIT = 2000000000LL;  // cycles (about a second)
constexpr float SPLIT_M = 12582912.0f;      // 1.5 * 2^23
constexpr int SPLIT_BITS = 0x4B400000;      // bits of SPLIT_M

static_assert(SLAB_BY % SLAB_BOX_Y == 0, "buffer made of whole boxes");
static_assert(4 * SLAB_W <= 32, "the producer projects the corner rays one per lane");

// The launch record of the FP and of its transpose (bp3d_slab_matched_kernel,
// which reads the projections and writes the accumulator through tmap / acc).
struct alignas(64) SlabLaunch {
    CUtensorMap tmap[2];   // FP: slab copy as 8-byte z-pairs, dims (n2 + 4, n1 + 4, n0); box widths WA, WB
                           // transpose: FP32 accumulator, dims (az, ay, n0); box widths MT_WA, MT_WB
    const float2 *copy;    // z-pair (s, k1, k2) at (s * py + k1 + 2) * pz + k2 + 2
    long long py, pz;
    float *acc;            // transpose: cell (s, k1, k2) at (s * ay + k1 + 2) * az + k2 + 2
    long long ay, az;
    void *proj;            // FP: output projections [v][angle][u]; transpose: its input
    long long proj_pitch;
    int n0, n1, n2, nu, nv, na;
    int accumulate;
    float f1, f2, mul;     // ray length factors and output scale
    int nviews;
    FPView views[SLAB_MAX_VIEWS];
};

// A slice's buffer: sel 0 / 1 the box width WA / WB, -1 read global memory;
// rbase folds the box origin and the texel split's offset into the byte
// address: texel (k1, k2) at slot + rbase + bits1 * 8 pitch + bits2 * 8
struct SlabInfo {
    int sel, rbase, pad0, pad1;
};

__device__ __forceinline__ float ray_setup(const FPView &V, float uu, float vv, float &A1, float &B1h, float &A2,
                                           float &B2h)
{
    const float den = fmaf(vv, V.e[2], fmaf(uu, V.e[1], V.e[0]));
    const float inv = 1.0f / den;
    A1 = fmaf(vv, V.m1[2], fmaf(uu, V.m1[1], V.m1[0])) * inv;
    A2 = fmaf(vv, V.m2[2], fmaf(uu, V.m2[1], V.m2[0])) * inv;
    B1h = fmaf(vv, V.n1[2], fmaf(uu, V.n1[1], V.n1[0])) * inv + 0.5f;
    B2h = fmaf(vv, V.n2[2], fmaf(uu, V.n2[1], V.n2[0])) * inv + 0.5f;
    return den;
}

// Base texel of position qh (floor), by rounding down qh + 1.5 * 2^23.
__device__ __forceinline__ int floor_texel(float qh) { return __float_as_int(__fadd_rd(qh, SPLIT_M)) - SPLIT_BITS; }

// Slices s of [0, n0) at which a ray's base texel along one axis stays in
// [-2, n] (the copy's zero border), intersected into [lo, hi].
__device__ __forceinline__ void clip_axis(float A, float Bh, int n, int n0, int &lo, int &hi)
{
    // qh = A s + Bh in [-2, n + 1) up to rounding (a nearly constant qh: the
    // whole range); then step inwards until the texel of the end slices is
    // inside.  fmaf(A, s, Bh) is monotone in s, so texels inside at both end
    // slices are inside at every slice between them; ends that stay outside
    // leave the range empty.
    float a = -1.0f, b = (float)n0;
    if (fabsf(A) >= 1e-12f) {
        const float s1 = (-2.0f - Bh) / A, s2 = ((float)n + 1.0f - Bh) / A;
        a = fminf(s1, s2);
        b = fmaxf(s1, s2);
    }
    int l = max(lo, (int)ceilf(fmaxf(a, -1.0f)));
    int h = min(hi, (int)floorf(fminf(b, (float)n0)));
    for (int it = 0; it < 4 && l <= h; ++it) {
        const int k = floor_texel(fmaf(A, (float)l, Bh));
        if (k >= -2 && k <= n) break;
        ++l;
    }
    for (int it = 0; it < 4 && l <= h; ++it) {
        const int k = floor_texel(fmaf(A, (float)h, Bh));
        if (k >= -2 && k <= n) break;
        --h;
    }
    if (l <= h) {
        const int kl = floor_texel(fmaf(A, (float)l, Bh)), kh = floor_texel(fmaf(A, (float)h, Bh));
        if (kl < -2 || kl > n || kh < -2 || kh > n) h = l - 1;
    }
    lo = l;
    hi = h;
}

// z-pair at a shared-memory byte address (plus an immediate offset)
template <int OFF> __device__ __forceinline__ float2 lds_pair(uint32_t a)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2+%3];" : "=f"(v.x), "=f"(v.y) : "r"(a), "n"(OFF));
    return v;
}

__device__ __forceinline__ int warp_min(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The detector ray (column u, row v) of a tile, clamped into the detector:
// lanes and corners outside the detector trace a copy of a real ray and
// store nothing.
__device__ __forceinline__ float det_uu(const SlabLaunch &L, int u) { return (float)min(u, L.nu - 1) + 0.5f - 0.5f * (float)L.nu; }
__device__ __forceinline__ float det_vv(const SlabLaunch &L, int v) { return (float)min(v, L.nv - 1) + 0.5f - 0.5f * (float)L.nv; }

// The tile's corner rays (view, column end, row end), set up once: lane
// c < 4 SLAB_W computes corner c, then every lane holds all of them.  The
// rays of a detector rectangle cross a slice inside the convex hull of the
// corners' crossings when their denominators share one sign (hull).
constexpr int SLAB_NC = 4 * SLAB_W;
struct Corners {
    float A1[SLAB_NC], B1[SLAB_NC], A2[SLAB_NC], B2[SLAB_NC];
    bool hull;
};

__device__ __forceinline__ void slab_corners(const SlabLaunch &L, int lane, Corners &C)
{
    const int c = lane % SLAB_NC;
    const int w = c >> 2, uc = c & 1, vc = (c >> 1) & 1;
    const int vi = min((int)blockIdx.x * SLAB_W + w, L.nviews - 1);
    const int u = (int)blockIdx.y * SLAB_U + (uc ? SLAB_U - 1 : 0);
    const int v = (int)blockIdx.z * SLAB_ROWS + (vc ? SLAB_ROWS - 1 : 0);
    float A1, B1h, A2, B2h;
    const float den = ray_setup(L.views[vi], det_uu(L, u), det_vv(L, v), A1, B1h, A2, B2h);
    C.hull = __all_sync(0xffffffffu, den > 1e-6f) || __all_sync(0xffffffffu, den < -1e-6f);
#pragma unroll
    for (int k = 0; k < SLAB_NC; ++k) {
        C.A1[k] = __shfl_sync(0xffffffffu, A1, k);
        C.B1[k] = __shfl_sync(0xffffffffu, B1h, k);
        C.A2[k] = __shfl_sync(0xffffffffu, A2, k);
        C.B2[k] = __shfl_sync(0xffffffffu, B2h, k);
    }
}

// The box of slice sf from the corners' texels, clamped to the zero border,
// one texel of margin for rounding: in-plane texels [y0, y1], z texels
// [zlo, z1].  sane: no corner position so large that its texel saturates.
__device__ __forceinline__ bool slab_box(const SlabLaunch &L, const Corners &C, float sf, int &y0, int &y1,
                                         int &zlo, int &z1)
{
    int k1lo = 0x7fffffff, k1hi = -0x7fffffff, k2lo = 0x7fffffff, k2hi = -0x7fffffff;
    bool sane = true;
#pragma unroll
    for (int k = 0; k < SLAB_NC; ++k) {
        const float q1 = fmaf(C.A1[k], sf, C.B1[k]), q2 = fmaf(C.A2[k], sf, C.B2[k]);
        sane = sane && fabsf(q1) < 1.0e7f && fabsf(q2) < 1.0e7f;
        const int k1 = min(max(floor_texel(q1), -2), L.n1), k2 = min(max(floor_texel(q2), -2), L.n2);
        k1lo = min(k1lo, k1);
        k1hi = max(k1hi, k1);
        k2lo = min(k2lo, k2);
        k2hi = max(k2hi, k2);
    }
    y0 = max(k1lo - 1, -2);
    y1 = min(k1hi + 2, L.n1 + 1);
    zlo = max(k2lo - 1, -2);
    z1 = min(k2hi + 2, L.n2 + 1);
    return sane;
}

// Producer warp: the buffer box of every slice of the CTA's range and its loads.
__device__ __noinline__ void slab_produce(const SlabLaunch &L, float2 *buf, uint64_t *full, uint64_t *empty,
                                          SlabInfo *info, int lane, int s_lo, int s_hi)
{
    Corners C;
    slab_corners(L, lane, C);
    const uint32_t sbuf = smem_u32(buf);
    const int nst = s_hi - s_lo + 1;
    unsigned long long n_staged = 0, n_global = 0;
    for (int b0 = 0; b0 < nst; b0 += 32) {
        // lane k: the buffer box of slice s_lo + b0 + k
        int y0, y1, zlo, z1;
        const bool sane = slab_box(L, C, (float)(s_lo + b0 + lane), y0, y1, zlo, z1);
        const int z0 = ((zlo + 2) & ~1) - 2;  // TMA: (z0 + 2) * 8 bytes on a 16-byte boundary
        const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
        const int sel = (!C.hull || !sane || ny > SLAB_BY || nz > SLAB_WB) ? -1 : (nz <= SLAB_WA ? 0 : 1);
        const int pitch = sel == 0 ? SLAB_WA : SLAB_WB;
        const int nby = (ny + SLAB_BOX_Y - 1) / SLAB_BOX_Y;
        const int cnt = min(32, nst - b0);
        if (lane < cnt) {
            if (sel >= 0) ++n_staged;
            else ++n_global;
        }
        // the slices in order: each waits for its buffer, then its own lane
        // writes the record and issues the loads
        for (int k = 0; k < cnt; ++k) {
            const int st = b0 + k;
            const int slot = st % SLAB_STAGES;
            if (st >= SLAB_STAGES) {
                const uint32_t par = (uint32_t)(((st / SLAB_STAGES) - 1) & 1);
                if (!__all_sync(0xffffffffu, mbar_wait_bounded_sleep(&empty[slot], par, SLAB_WAIT))) {
                    if (lane == 0) atomicOr(&g_fp_slab_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
                    // the loads of the slices still in the buffers land first
                    for (int q = max(0, st - SLAB_STAGES); q < st; ++q)
                        (void)mbar_wait_bounded_sleep(&full[q % SLAB_STAGES], (uint32_t)((q / SLAB_STAGES) & 1),
                                                      SLAB_WAIT);
                    return;
                }
            }
            if (lane == k) {
                SlabInfo r;
                r.sel = sel;
                r.rbase = (int)(0u - (uint32_t)(SPLIT_BITS + y0) * (uint32_t)(8 * pitch) -
                                (uint32_t)(SPLIT_BITS + z0) * 8u);
                r.pad0 = r.pad1 = 0;
                info[slot] = r;
                if (sel >= 0) {
                    // the loads go out after the arrival, whose transaction
                    // count keeps the phase open until they land
                    mbar_arrive_expect_tx(&full[slot], (uint32_t)(nby * SLAB_BOX_Y * pitch * sizeof(float2)));
                    float2 *dst = buf + (size_t)slot * SLAB_SLOT;
                    for (int by = 0; by < nby; ++by)
                        tma_load_3d(dst + (size_t)(by * SLAB_BOX_Y) * pitch, &L.tmap[sel], z0 + 2,
                                    y0 + 2 + by * SLAB_BOX_Y, s_lo + st, &full[slot]);
                } else {
                    mbar_arrive(&full[slot]);
                }
            }
            __syncwarp();
        }
    }
    (void)sbuf;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_staged += __shfl_xor_sync(0xffffffffu, n_staged, o);
        n_global += __shfl_xor_sync(0xffffffffu, n_global, o);
    }
    if (lane == 0) {
        atomicAdd(&g_fp_slab_slices[0], n_staged);
        atomicAdd(&g_fp_slab_slices[1], n_global);
    }
    // the last slices' loads land before the warp leaves
    for (int st = max(0, nst - SLAB_STAGES); st < nst; ++st)
        (void)mbar_wait_bounded_sleep(&full[st % SLAB_STAGES], (uint32_t)((st / SLAB_STAGES) & 1), SLAB_WAIT);
}

// The lane's rays: both views, SLAB_R rows each.
struct Rays {
    float A1[SLAB_W], B1h[SLAB_W];
    float A2[SLAB_W][SLAB_R], B2h[SLAB_W][SLAB_R];
    float acc[SLAB_W][SLAB_R];
};

// One slice of the lane's rays (rows r < RE of each view) from a
// shared-memory buffer of row pitch P (z-pairs).  CLAMP: texels clamped to
// the zero border (slices where a ray of the warp is outside the volume).
// rb = the slot's byte address + rbase.
template <int P, bool CLAMP, int RE>
__device__ __forceinline__ void sample_smem(const SlabLaunch &L, uint32_t rb, float sf, Rays &R)
{
    constexpr uint32_t ROWB = 8u * P;
    static_assert(SLAB_W == 2, "the two views' in-plane splits share packed instructions");
    const uint64_t sf2 = pk2(sf, sf), M2 = pk2(SPLIT_M, SPLIT_M), nM2 = pk2(-SPLIT_M, -SPLIT_M);
    // both views' in-plane position, split and weights in packed f32x2
    // (130.8 against 133.1 ms one view at a time at 512^3 x 720, same bits)
    const uint64_t q1p = fma2(pk2(R.A1[0], R.A1[1]), sf2, pk2(R.B1h[0], R.B1h[1]));
    const uint64_t t1p = add2_rd(q1p, M2);
    const uint64_t f1p = sub2(q1p, add2(t1p, nM2));
    const float2 t1u = upk2(t1p), f1u = upk2(f1p), g1u = upk2(sub2(pk2(1.0f, 1.0f), f1p));
#pragma unroll
    for (int w = 0; w < SLAB_W; ++w) {
        const float f1 = w == 0 ? f1u.x : f1u.y, g1 = w == 0 ? g1u.x : g1u.y;
        int b1 = __float_as_int(w == 0 ? t1u.x : t1u.y);
        if (CLAMP) b1 = min(max(b1, SPLIT_BITS - 2), SPLIT_BITS + L.n1);
        const uint32_t row = (uint32_t)b1 * ROWB + rb;
        // rows r, r + 1 in the two halves of packed f32x2 operations (each
        // half rounds as the scalar form of the odd row below)
        const uint64_t f12 = pk2(f1, f1), g12 = pk2(g1, g1);
#pragma unroll
        for (int r = 0; r + 1 < RE; r += 2) {
            const uint64_t q2 = fma2(pk2(R.A2[w][r], R.A2[w][r + 1]), sf2, pk2(R.B2h[w][r], R.B2h[w][r + 1]));
            const uint64_t t2 = add2_rd(q2, M2);
            const float2 f2 = upk2(sub2(q2, add2(t2, nM2)));
            const float2 tb = upk2(t2);
            int b2a = __float_as_int(tb.x), b2b = __float_as_int(tb.y);
            if (CLAMP) {
                b2a = min(max(b2a, SPLIT_BITS - 2), SPLIT_BITS + L.n2);
                b2b = min(max(b2b, SPLIT_BITS - 2), SPLIT_BITS + L.n2);
            }
            const uint32_t a0 = (uint32_t)b2a * 8u + row, a1 = (uint32_t)b2b * 8u + row;
            const float2 p0a = lds_pair<0>(a0), p1a = lds_pair<(int)ROWB>(a0);
            const float2 p0b = lds_pair<0>(a1), p1b = lds_pair<(int)ROWB>(a1);
            // rows k1 and k1 + 1 interpolated along z, then blended by the
            // shared in-plane weights straight into the sum
            const uint64_t lo = pk2(fmaf(f2.x, p0a.y, p0a.x), fmaf(f2.y, p0b.y, p0b.x));
            const uint64_t hi = pk2(fmaf(f2.x, p1a.y, p1a.x), fmaf(f2.y, p1b.y, p1b.x));
            const float2 acc = upk2(fma2(f12, hi, fma2(g12, lo, pk2(R.acc[w][r], R.acc[w][r + 1]))));
            R.acc[w][r] = acc.x;
            R.acc[w][r + 1] = acc.y;
        }
        if constexpr (RE % 2 == 1) {
            constexpr int r = RE - 1;
            const float q2 = fmaf(R.A2[w][r], sf, R.B2h[w][r]);
            const float t2 = __fadd_rd(q2, SPLIT_M);
            const float f2 = q2 - (t2 - SPLIT_M);
            int b2 = __float_as_int(t2);
            if (CLAMP) b2 = min(max(b2, SPLIT_BITS - 2), SPLIT_BITS + L.n2);
            const uint32_t a = (uint32_t)b2 * 8u + row;
            const float2 p0 = lds_pair<0>(a), p1 = lds_pair<(int)ROWB>(a);
            const float lo = fmaf(f2, p0.y, p0.x), hi = fmaf(f2, p1.y, p1.x);
            R.acc[w][r] = fmaf(f1, hi, fmaf(g1, lo, R.acc[w][r]));
        }
    }
}

// The same from the slab copy in global memory (a slice whose box did not fit).
template <int RE>
__device__ __forceinline__ void sample_global(const SlabLaunch &L, int s, float sf, Rays &R)
{
#pragma unroll
    for (int w = 0; w < SLAB_W; ++w) {
        const float q1 = fmaf(R.A1[w], sf, R.B1h[w]);
        const float t1 = __fadd_rd(q1, SPLIT_M);
        const float f1 = q1 - (t1 - SPLIT_M);
        const float g1 = 1.0f - f1;
        const int k1 = min(max(__float_as_int(t1) - SPLIT_BITS, -2), L.n1);
        const float2 *row = L.copy + ((long long)s * L.py + k1 + 2) * L.pz + 2;
#pragma unroll
        for (int r = 0; r < RE; ++r) {
            const float q2 = fmaf(R.A2[w][r], sf, R.B2h[w][r]);
            const float t2 = __fadd_rd(q2, SPLIT_M);
            const float f2 = q2 - (t2 - SPLIT_M);
            const int k2 = min(max(__float_as_int(t2) - SPLIT_BITS, -2), L.n2);
            const float2 p0 = __ldg(row + k2), p1 = __ldg(row + L.pz + k2);
            // the arithmetic of sample_smem, so that a ray's sum does not
            // depend on where its slices were read from
            const float lo = fmaf(f2, p0.y, p0.x), hi = fmaf(f2, p1.y, p1.x);
            R.acc[w][r] = fmaf(f1, hi, fmaf(g1, lo, R.acc[w][r]));
        }
    }
}

// The CTA's slice range [s_lo, s_hi] and the warp's union [wlo, whi] and
// intersection [ilo, ihi] of its rays' ranges.
struct Range {
    int s_lo, s_hi, wlo, whi, ilo, ihi;
};

// Slices [s0, s1] of a compute warp's pass (rows r < RE of each view): wait
// for each slice's buffer, sample it (KIND 0: no ray of the warp samples
// these slices, 1: some ray leaves the volume, texels clamped, 2: fast),
// release it.  False when a wait gave up.
template <int RE, int KIND>
__device__ __forceinline__ bool slab_slices(const SlabLaunch &L, uint32_t sbase, uint64_t *full, uint64_t *empty,
                                            const SlabInfo *info, int lane, int s0, int s1, int &slot,
                                            uint32_t &par, Rays &R)
{
    float sf = (float)s0;
    for (int s = s0; s <= s1; ++s, sf += 1.0f) {
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[slot], par, SLAB_WAIT))) {
            if (lane == 0) atomicOr(&g_fp_slab_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
            return false;
        }
        if constexpr (KIND > 0) {
            const SlabInfo I = info[slot];
            const uint32_t rb = sbase + (uint32_t)slot * (SLAB_SLOT * 8u) + (uint32_t)I.rbase;
            if (I.sel == 0) sample_smem<SLAB_WA, KIND == 1, RE>(L, rb, sf, R);
            else if (I.sel == 1) sample_smem<SLAB_WB, KIND == 1, RE>(L, rb, sf, R);
            else sample_global<RE>(L, s, sf, R);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
        if (++slot == SLAB_STAGES) {
            slot = 0;
            par ^= 1u;
        }
    }
    return true;
}

// A compute warp's pass over the CTA's slices, split into the segments
// where its sampling is the same for every slice (no per-slice range tests;
// 137.0 -> 133.4 ms at 512^3 x 720, bit-identical).
template <int RE>
__device__ __forceinline__ bool slab_consume(const SlabLaunch &L, const float2 *buf, uint64_t *full, uint64_t *empty,
                                             const SlabInfo *info, int lane, const Range &rg, Rays &R)
{
    const uint32_t sbase = smem_u32(buf);
    int slot = 0;
    uint32_t par = 0;
    // the warp's slices in segments: none of its rays, clamped, fast, clamped, none
    const bool any = rg.wlo <= rg.whi;
    const int w0 = any ? rg.wlo : rg.s_hi + 1, w1 = any ? rg.whi : rg.s_hi;
    const bool hasf = any && rg.ilo <= rg.ihi;
    const int f0 = hasf ? max(rg.ilo, w0) : w1 + 1, f1 = hasf ? min(rg.ihi, w1) : w1;
    if (!slab_slices<RE, 0>(L, sbase, full, empty, info, lane, rg.s_lo, w0 - 1, slot, par, R)) return false;
    if (!slab_slices<RE, 1>(L, sbase, full, empty, info, lane, w0, f0 - 1, slot, par, R)) return false;
    if (!slab_slices<RE, 2>(L, sbase, full, empty, info, lane, f0, f1, slot, par, R)) return false;
    if (!slab_slices<RE, 1>(L, sbase, full, empty, info, lane, f1 + 1, w1, slot, par, R)) return false;
    return slab_slices<RE, 0>(L, sbase, full, empty, info, lane, w1 + 1, rg.s_hi, slot, par, R);
}

// slab_consume for the rows in use, re in [1, RE]
template <int RE>
__device__ __forceinline__ bool slab_consume_rows(int re, const SlabLaunch &L, const float2 *buf, uint64_t *full,
                                                  uint64_t *empty, const SlabInfo *info, int lane, const Range &rg,
                                                  Rays &R)
{
    if constexpr (RE == 1) {
        return slab_consume<1>(L, buf, full, empty, info, lane, rg, R);
    } else {
        if (re >= RE) return slab_consume<RE>(L, buf, full, empty, info, lane, rg, R);
        return slab_consume_rows<RE - 1>(re, L, buf, full, empty, info, lane, rg, R);
    }
}

__global__ void __launch_bounds__(SLAB_THREADS, 2) fp3d_slab_kernel(const __grid_constant__ SlabLaunch L)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    float2 *buf = reinterpret_cast<float2 *>(smraw);
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw + (size_t)SLAB_STAGES * SLAB_SLOT * sizeof(float2));
    uint64_t *empty = full + SLAB_STAGES;
    SlabInfo *info = reinterpret_cast<SlabInfo *>(empty + SLAB_STAGES);
    int *range = reinterpret_cast<int *>(info + SLAB_STAGES);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int k = 0; k < SLAB_STAGES; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], SLAB_WARPS);
        }
        range[0] = 0x7fffffff;
        range[1] = -0x7fffffff;
        mbar_fence_init();
        tma_prefetch_map(&L.tmap[0]);
        tma_prefetch_map(&L.tmap[1]);
    }
    __syncthreads();

    // ---- ray set-up (compute warps): column `warp`, both views, SLAB_R rows per lane
    const int u_raw = (int)blockIdx.y * SLAB_U + warp;
    Rays R;
    int wlo = 1, whi = 0, ilo = 1, ihi = 0;  // union and intersection of the warp's ray ranges
    if (warp < SLAB_WARPS) {
        const float uu = det_uu(L, u_raw);
        int lo_u = 0x7fffffff, hi_u = -0x7fffffff, lo_i = -0x7fffffff, hi_i = 0x7fffffff;
#pragma unroll
        for (int w = 0; w < SLAB_W; ++w) {
            const FPView &V = L.views[min((int)blockIdx.x * SLAB_W + w, L.nviews - 1)];
#pragma unroll
            for (int r = 0; r < SLAB_R; ++r) {
                const int v = (int)blockIdx.z * SLAB_ROWS + lane + 32 * r;
                float a1, b1;
                ray_setup(V, uu, det_vv(L, v), a1, b1, R.A2[w][r], R.B2h[w][r]);
                // the same for every row: a column's rays share the in-plane position
                R.A1[w] = a1;
                R.B1h[w] = b1;
                R.acc[w][r] = 0.0f;
                int lo = 0, hi = L.n0 - 1;
                clip_axis(a1, b1, L.n1, L.n0, lo, hi);
                clip_axis(R.A2[w][r], R.B2h[w][r], L.n2, L.n0, lo, hi);
                if (lo <= hi) {
                    lo_u = min(lo_u, lo);
                    hi_u = max(hi_u, hi);
                }
                lo_i = max(lo_i, lo);
                hi_i = min(hi_i, hi);
            }
        }
        wlo = warp_min(lo_u);
        whi = warp_max(hi_u);
        ilo = warp_max(lo_i);
        ihi = warp_min(hi_i);
        if (lane == 0 && wlo <= whi) {
            atomicMin(&range[0], wlo);
            atomicMax(&range[1], whi);
        }
    }
    __syncthreads();
    const int s_lo = range[0], s_hi = range[1];

    if (warp == SLAB_WARPS) {
        if (s_lo <= s_hi) slab_produce(L, buf, full, empty, info, lane, s_lo, s_hi);
        return;
    }

    // ---- compute warps: the rows in use (the last row block of the
    // detector may hold fewer than SLAB_ROWS)
    const int re = min(SLAB_R, (L.nv - (int)blockIdx.z * SLAB_ROWS + 31) >> 5);
    const Range rg{s_lo, s_hi, wlo, whi, ilo, ihi};
    bool ok;
    ok = slab_consume_rows<SLAB_R>(re, L, buf, full, empty, info, lane, rg, R);
    if (!ok || u_raw >= L.nu) return;
    // ---- results
#pragma unroll
    for (int w = 0; w < SLAB_W; ++w) {
        const int vi = (int)blockIdx.x * SLAB_W + w;
        if (vi >= L.nviews) break;
        const int a = L.views[vi].a;
#pragma unroll
        for (int r = 0; r < SLAB_R; ++r) {
            const int v = (int)blockIdx.z * SLAB_ROWS + lane + 32 * r;
            if (v >= L.nv) continue;
            const float sc =
                sqrtf(fmaf(R.A1[w] * R.A1[w], L.f1, fmaf(R.A2[w][r] * R.A2[w][r], L.f2, 1.0f))) * L.mul;
            float *out = static_cast<float *>(L.proj) + ((size_t)v * L.na + a) * L.proj_pitch + u_raw;
            float val = fmaf(R.acc[w][r], sc, 0.0f);
            if (L.accumulate) val += *out;
            *out = val;
        }
    }
}

// ---------------------------------------------------------------------------
// The FP's transpose on the same tiles (projection kernel "matched_bp" for
// the views the slab FP takes).  A CTA takes the rays of one FP tile
// (SLAB_W views x SLAB_U columns x SLAB_ROWS rows) and walks the same slices:
// each sample's four bilinear taps, weighted as the FP weighs the texels it
// reads at that sample, are added with shared-memory reductions into an
// FP32 box of the slice (the FP's buffer box, as single floats); the
// producer warp zeroes each box before its slice and, MT_LAG slices after
// the compute warps have finished it, adds the box into an FP32
// accumulator in global memory with TMA reduce-adds (cp.reduce.async.bulk
// .tensor .add, one per SLAB_BOX_Y rows).  The accumulator has the slab
// copy's layout (slice, in-plane texel + 2, z texel + 2) with room past the
// far borders, so that no box leaves it; fold_cells (matched.cu) adds its
// interior into the volume.  Global memory sees one reduction per box cell
// instead of one per tap.
//
// Measured on B200 (512^3 x 720 views, 832^2 detector) this is 4.1x slower
// than the per-sample global reductions of matched.cu (1538 against 372 ms;
// 98.5 against 23.3 ms at 256^3 x 360, 416^2): FP32 reductions into shared
// memory are not a native operation there (ncu counts 13.5 shared-memory
// atomic instructions and 88 instructions per warp-sample where the kernel
// issues 4 reductions), while the same kernel with 32-bit integer reductions
// at the same addresses takes 29.9 ms and with plain stores 16.8 ms, which
// bounds any shared-memory accumulation of this tiling at 0.72x of the
// scatter.  So the scatter kernels stay the default and this kernel runs
// only when B2T_MATCHED_PATH=slab selects it.
//
// A tap lands inside its box for the reason an FP sample reads inside it:
// at a slice, the rays of a detector rectangle whose denominators share a
// sign cross it inside the hull of the corner rays' crossings, and the box
// is that hull's texel range with a texel of margin; samples outside the
// volume are clamped to the zero border exactly as the FP clamps them (their
// taps land on border cells, which the fold drops).
constexpr int MT_STAGES = 4;              // slice boxes in flight
constexpr int MT_LAG = 2;                 // slices between a box's last scatter and its flush
constexpr int MT_WA = 96, MT_WB = 160;    // box widths (floats): a box's row pitch
constexpr int MT_SLOT = SLAB_BY * MT_WB;  // floats per box
static_assert(MT_LAG >= 1 && MT_LAG < MT_STAGES, "a box is flushed before its slot comes round again");
static_assert((MT_WA * 4 * SLAB_BOX_Y) % 128 == 0 && (MT_WB * 4 * SLAB_BOX_Y) % 128 == 0,
              "TMA boxes start on 128-byte boundaries of a slot");

// A slice's box: sel 0 / 1 the width MT_WA / MT_WB, -1 scattered straight
// into the accumulator; rbase as in SlabInfo (4-byte cells); (zc, yc) the
// box origin in accumulator coordinates, nby its TMA boxes, s the slice
struct MTInfo {
    int sel, rbase, zc, yc, nby, s, pad0, pad1;
};

// The lane's rays: both views, SLAB_R rows each, with the value each
// carries back (projection value x the FP's output scale of the ray)
struct TRays {
    float A1[SLAB_W], B1h[SLAB_W];
    float A2[SLAB_W][SLAB_R], B2h[SLAB_W][SLAB_R];
    float wv[SLAB_W][SLAB_R];
};

template <typename T> __device__ __forceinline__ float ld_proj(const T *p);
template <> __device__ __forceinline__ float ld_proj<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_proj<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ld_proj<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(__ldg(p));
}

template <int OFF> __device__ __forceinline__ void red_smem(uint32_t a, float v)
{
    asm volatile("red.shared.add.f32 [%0+%1], %2;" ::"r"(a), "n"(OFF), "f"(v) : "memory");
}

// One slice of the lane's rays into a box of row pitch P (floats); CLAMP as
// in sample_smem.  The taps of a sample at base texel (k1, k2) with weights
// f1 (in-plane) and f2 (z): (1 - f1) (1 - f2), (1 - f1) f2, f1 (1 - f2),
// f1 f2 at (k1, k2), (k1, k2 + 1), (k1 + 1, k2), (k1 + 1, k2 + 1).
template <int P, bool CLAMP, int RE>
__device__ __forceinline__ void scatter_smem(const SlabLaunch &L, uint32_t rb, float sf, const TRays &R)
{
    constexpr uint32_t ROWB = 4u * P;
#pragma unroll
    for (int w = 0; w < SLAB_W; ++w) {
        const float q1 = fmaf(R.A1[w], sf, R.B1h[w]);
        const float t1 = __fadd_rd(q1, SPLIT_M);
        const float f1 = q1 - (t1 - SPLIT_M);
        const float g1 = 1.0f - f1;
        int b1 = __float_as_int(t1);
        if (CLAMP) b1 = min(max(b1, SPLIT_BITS - 2), SPLIT_BITS + L.n1);
        const uint32_t row = (uint32_t)b1 * ROWB + rb;
        const uint64_t sf2 = pk2(sf, sf), M2 = pk2(SPLIT_M, SPLIT_M), nM2 = pk2(-SPLIT_M, -SPLIT_M);
        const uint64_t f12 = pk2(f1, f1), g12 = pk2(g1, g1);
#pragma unroll
        for (int r = 0; r + 1 < RE; r += 2) {
            const uint64_t q2 = fma2(pk2(R.A2[w][r], R.A2[w][r + 1]), sf2, pk2(R.B2h[w][r], R.B2h[w][r + 1]));
            const uint64_t t2 = add2_rd(q2, M2);
            const uint64_t f2 = sub2(q2, add2(t2, nM2));
            const float2 tb = upk2(t2);
            int b2a = __float_as_int(tb.x), b2b = __float_as_int(tb.y);
            if (CLAMP) {
                b2a = min(max(b2a, SPLIT_BITS - 2), SPLIT_BITS + L.n2);
                b2b = min(max(b2b, SPLIT_BITS - 2), SPLIT_BITS + L.n2);
            }
            const uint32_t a0 = (uint32_t)b2a * 4u + row, a1 = (uint32_t)b2b * 4u + row;
            const uint64_t c = pk2(R.wv[w][r], R.wv[w][r + 1]);
            const uint64_t cb = mul2(c, f2), ca = sub2(c, cb);
            const float2 la = upk2(mul2(g12, ca)), lb = upk2(mul2(g12, cb));
            const float2 ha = upk2(mul2(f12, ca)), hb = upk2(mul2(f12, cb));
            red_smem<0>(a0, la.x);
            red_smem<4>(a0, lb.x);
            red_smem<(int)ROWB>(a0, ha.x);
            red_smem<(int)ROWB + 4>(a0, hb.x);
            red_smem<0>(a1, la.y);
            red_smem<4>(a1, lb.y);
            red_smem<(int)ROWB>(a1, ha.y);
            red_smem<(int)ROWB + 4>(a1, hb.y);
        }
        if constexpr (RE % 2 == 1) {
            constexpr int r = RE - 1;
            const float q2 = fmaf(R.A2[w][r], sf, R.B2h[w][r]);
            const float t2 = __fadd_rd(q2, SPLIT_M);
            const float f2 = q2 - (t2 - SPLIT_M);
            int b2 = __float_as_int(t2);
            if (CLAMP) b2 = min(max(b2, SPLIT_BITS - 2), SPLIT_BITS + L.n2);
            const uint32_t a = (uint32_t)b2 * 4u + row;
            const float cb = R.wv[w][r] * f2, ca = R.wv[w][r] - cb;
            red_smem<0>(a, g1 * ca);
            red_smem<4>(a, g1 * cb);
            red_smem<(int)ROWB>(a, f1 * ca);
            red_smem<(int)ROWB + 4>(a, f1 * cb);
        }
    }
}

// The same straight into the accumulator (a slice whose box did not fit).
template <int RE>
__device__ __forceinline__ void scatter_global(const SlabLaunch &L, int s, float sf, const TRays &R)
{
#pragma unroll
    for (int w = 0; w < SLAB_W; ++w) {
        const float q1 = fmaf(R.A1[w], sf, R.B1h[w]);
        const float t1 = __fadd_rd(q1, SPLIT_M);
        const float f1 = q1 - (t1 - SPLIT_M);
        const float g1 = 1.0f - f1;
        const int k1 = min(max(__float_as_int(t1) - SPLIT_BITS, -2), L.n1);
        float *row = L.acc + ((long long)s * L.ay + k1 + 2) * L.az + 2;
#pragma unroll
        for (int r = 0; r < RE; ++r) {
            const float q2 = fmaf(R.A2[w][r], sf, R.B2h[w][r]);
            const float t2 = __fadd_rd(q2, SPLIT_M);
            const float f2 = q2 - (t2 - SPLIT_M);
            const int k2 = min(max(__float_as_int(t2) - SPLIT_BITS, -2), L.n2);
            const float cb = R.wv[w][r] * f2, ca = R.wv[w][r] - cb;
            atomicAdd(row + k2, g1 * ca);
            atomicAdd(row + k2 + 1, g1 * cb);
            atomicAdd(row + L.az + k2, f1 * ca);
            atomicAdd(row + L.az + k2 + 1, f1 * cb);
        }
    }
}

// Producer warp of the transpose: for every slice of the CTA's range, in
// order, flush the box finished MT_LAG slices earlier, then zero the slot
// of this slice's box and hand it to the compute warps.
__device__ __noinline__ void mt_produce(const SlabLaunch &L, float *buf, uint64_t *ready, uint64_t *done,
                                        MTInfo *info, int lane, int s_lo, int s_hi)
{
    Corners C;
    slab_corners(L, lane, C);
    const int nst = s_hi - s_lo + 1;
    unsigned long long n_staged = 0, n_global = 0;
    bool ok = true;
    // wait for the compute warps to finish slice st, then (lane 0) reduce its
    // box into the accumulator; every slice commits one bulk group
    auto flush = [&](int st) -> bool {
        const int slot = st % MT_STAGES;
        if (!__all_sync(0xffffffffu,
                        mbar_wait_bounded_sleep(&done[slot], (uint32_t)((st / MT_STAGES) & 1), SLAB_WAIT))) {
            if (lane == 0) atomicOr(&g_fp_slab_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
            return false;
        }
        if (lane == 0) {
            const MTInfo I = info[slot];
            if (I.sel >= 0) {
                const int pitch = I.sel == 0 ? MT_WA : MT_WB;
                const float *src = buf + (size_t)slot * MT_SLOT;
                for (int by = 0; by < I.nby; ++by)
                    tma_reduce_add_3d(&L.tmap[I.sel], src + (size_t)(by * SLAB_BOX_Y) * pitch, I.zc,
                                      I.yc + by * SLAB_BOX_Y, I.s);
            }
            bulk_commit_group();
        }
        __syncwarp();
        return true;
    };
    for (int b0 = 0; b0 < nst && ok; b0 += 32) {
        // lane k: the box of slice s_lo + b0 + k
        int y0, y1, zlo, z1;
        const bool sane = slab_box(L, C, (float)(s_lo + b0 + lane), y0, y1, zlo, z1);
        const int z0 = ((zlo + 2) & ~3) - 2;  // TMA: (z0 + 2) * 4 bytes on a 16-byte boundary
        const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
        const int sel_l = (!C.hull || !sane || ny > SLAB_BY || nz > MT_WB) ? -1 : (nz <= MT_WA ? 0 : 1);
        const int nby_l = (ny + SLAB_BOX_Y - 1) / SLAB_BOX_Y;
        const int cnt = min(32, nst - b0);
        if (lane < cnt) {
            if (sel_l >= 0) ++n_staged;
            else ++n_global;
        }
        for (int k = 0; k < cnt; ++k) {
            const int st = b0 + k;
            const int slot = st % MT_STAGES;
            if (st >= MT_LAG && !flush(st - MT_LAG)) {
                ok = false;
                break;
            }
            // the slot's previous box (slice st - MT_STAGES) has been read by
            // its reduce: it was committed MT_STAGES - MT_LAG groups ago
            if (st >= MT_STAGES && lane == 0) bulk_wait_group_read<MT_STAGES - MT_LAG>();
            __syncwarp();
            const int sel = __shfl_sync(0xffffffffu, sel_l, k);
            const int y0k = __shfl_sync(0xffffffffu, y0, k);
            const int z0k = __shfl_sync(0xffffffffu, z0, k);
            const int nby = __shfl_sync(0xffffffffu, nby_l, k);
            float *slotp = buf + (size_t)slot * MT_SLOT;
            if (sel >= 0) {
                const int n4 = nby * SLAB_BOX_Y * (sel == 0 ? MT_WA : MT_WB) / 4;
                float4 *z4 = reinterpret_cast<float4 *>(slotp);
                for (int i = lane; i < n4; i += 32) z4[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            if (lane == 0) {
                const int pitch = sel == 0 ? MT_WA : MT_WB;
                MTInfo r;
                r.sel = sel;
                r.rbase = (int)(0u - (uint32_t)(SPLIT_BITS + y0k) * (uint32_t)(4 * pitch) -
                                (uint32_t)(SPLIT_BITS + z0k) * 4u);
                r.zc = z0k + 2;
                r.yc = y0k + 2;
                r.nby = nby;
                r.s = s_lo + st;
                r.pad0 = r.pad1 = 0;
                info[slot] = r;
            }
            // every lane releases its own zero stores
            mbar_arrive(&ready[slot]);
        }
    }
    if (ok) {
        for (int st = max(0, nst - MT_LAG); st < nst; ++st) {
            if (!flush(st)) {
                ok = false;
                break;
            }
        }
    }
    // the reduces complete before the CTA leaves (on a timeout too)
    if (lane == 0) bulk_wait_group_all();
    __syncwarp();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_staged += __shfl_xor_sync(0xffffffffu, n_staged, o);
        n_global += __shfl_xor_sync(0xffffffffu, n_global, o);
    }
    if (lane == 0) {
        atomicAdd(&g_mt_slab_slices[0], n_staged);
        atomicAdd(&g_mt_slab_slices[1], n_global);
    }
}

// A compute warp's pass over the CTA's slices (rows r < RE): wait for the
// slice's zeroed box, scatter, hand it back.  False when a wait gave up.
template <int RE>
__device__ __forceinline__ bool mt_consume(const SlabLaunch &L, const float *buf, uint64_t *ready, uint64_t *done,
                                           const MTInfo *info, int lane, const Range &rg, const TRays &R)
{
    const uint32_t sbase = smem_u32(buf);
    int slot = 0;
    uint32_t par = 0;
    float sf = (float)rg.s_lo;
    for (int s = rg.s_lo; s <= rg.s_hi; ++s, sf += 1.0f) {
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&ready[slot], par, SLAB_WAIT))) {
            if (lane == 0) atomicOr(&g_fp_slab_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
            return false;
        }
        if (s >= rg.wlo && s <= rg.whi) {
            const MTInfo &I = info[slot];
            const int sel = I.sel;
            const uint32_t rb = sbase + (uint32_t)slot * (MT_SLOT * 4u) + (uint32_t)I.rbase;
            const bool fast = s >= rg.ilo && s <= rg.ihi;
            if (sel == 0) {
                if (fast) scatter_smem<MT_WA, false, RE>(L, rb, sf, R);
                else scatter_smem<MT_WA, true, RE>(L, rb, sf, R);
            } else if (sel == 1) {
                if (fast) scatter_smem<MT_WB, false, RE>(L, rb, sf, R);
                else scatter_smem<MT_WB, true, RE>(L, rb, sf, R);
            } else {
                scatter_global<RE>(L, s, sf, R);
            }
            // the reductions are visible to the TMA reduce that reads the box
            if (sel >= 0) fence_proxy_async_smem();
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&done[slot]);
        if (++slot == MT_STAGES) {
            slot = 0;
            par ^= 1u;
        }
    }
    return true;
}

// mt_consume for the rows in use, re in [1, RE]
template <int RE>
__device__ __forceinline__ bool mt_consume_rows(int re, const SlabLaunch &L, const float *buf, uint64_t *ready,
                                                uint64_t *done, const MTInfo *info, int lane, const Range &rg,
                                                const TRays &R)
{
    if constexpr (RE == 1) {
        return mt_consume<1>(L, buf, ready, done, info, lane, rg, R);
    } else {
        if (re >= RE) return mt_consume<RE>(L, buf, ready, done, info, lane, rg, R);
        return mt_consume_rows<RE - 1>(re, L, buf, ready, done, info, lane, rg, R);
    }
}

template <typename T>
__global__ void __launch_bounds__(SLAB_THREADS, 2) bp3d_slab_matched_kernel(const __grid_constant__ SlabLaunch L)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    float *buf = reinterpret_cast<float *>(smraw);
    uint64_t *ready = reinterpret_cast<uint64_t *>(smraw + (size_t)MT_STAGES * MT_SLOT * sizeof(float));
    uint64_t *done = ready + MT_STAGES;
    MTInfo *info = reinterpret_cast<MTInfo *>(done + MT_STAGES);
    int *range = reinterpret_cast<int *>(info + MT_STAGES);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int k = 0; k < MT_STAGES; ++k) {
            mbar_init(&ready[k], 32);
            mbar_init(&done[k], SLAB_WARPS);
        }
        range[0] = 0x7fffffff;
        range[1] = -0x7fffffff;
        mbar_fence_init();
        tma_prefetch_map(&L.tmap[0]);
        tma_prefetch_map(&L.tmap[1]);
    }
    __syncthreads();

    // ---- ray set-up (compute warps), as in fp3d_slab_kernel, plus the
    // value each ray carries back: rays off the detector carry zero
    const int u_raw = (int)blockIdx.y * SLAB_U + warp;
    TRays R;
    int wlo = 1, whi = 0, ilo = 1, ihi = 0;
    if (warp < SLAB_WARPS) {
        const float uu = det_uu(L, u_raw);
        int lo_u = 0x7fffffff, hi_u = -0x7fffffff, lo_i = -0x7fffffff, hi_i = 0x7fffffff;
#pragma unroll
        for (int w = 0; w < SLAB_W; ++w) {
            const int vi = (int)blockIdx.x * SLAB_W + w;
            const FPView &V = L.views[min(vi, L.nviews - 1)];
#pragma unroll
            for (int r = 0; r < SLAB_R; ++r) {
                const int v = (int)blockIdx.z * SLAB_ROWS + lane + 32 * r;
                float a1, b1;
                ray_setup(V, uu, det_vv(L, v), a1, b1, R.A2[w][r], R.B2h[w][r]);
                R.A1[w] = a1;
                R.B1h[w] = b1;
                float val = 0.0f;
                if (vi < L.nviews && u_raw < L.nu && v < L.nv)
                    val = ld_proj(static_cast<const T *>(L.proj) + ((size_t)v * L.na + V.a) * L.proj_pitch + u_raw);
                const float sc =
                    sqrtf(fmaf(a1 * a1, L.f1, fmaf(R.A2[w][r] * R.A2[w][r], L.f2, 1.0f))) * L.mul;
                R.wv[w][r] = val * sc;
                int lo = 0, hi = L.n0 - 1;
                clip_axis(a1, b1, L.n1, L.n0, lo, hi);
                clip_axis(R.A2[w][r], R.B2h[w][r], L.n2, L.n0, lo, hi);
                if (lo <= hi) {
                    lo_u = min(lo_u, lo);
                    hi_u = max(hi_u, hi);
                }
                lo_i = max(lo_i, lo);
                hi_i = min(hi_i, hi);
            }
        }
        wlo = warp_min(lo_u);
        whi = warp_max(hi_u);
        ilo = warp_max(lo_i);
        ihi = warp_min(hi_i);
        if (lane == 0 && wlo <= whi) {
            atomicMin(&range[0], wlo);
            atomicMax(&range[1], whi);
        }
    }
    __syncthreads();
    const int s_lo = range[0], s_hi = range[1];

    if (warp == SLAB_WARPS) {
        if (s_lo <= s_hi) mt_produce(L, buf, ready, done, info, lane, s_lo, s_hi);
        return;
    }
    const int re = min(SLAB_R, (L.nv - (int)blockIdx.z * SLAB_ROWS + 31) >> 5);
    const Range rg{s_lo, s_hi, wlo, whi, ilo, ihi};
    (void)mt_consume_rows<SLAB_R>(re, L, buf, ready, done, info, lane, rg, R);
}

// Slab copy of marching axis dir (0: slices along x, in-plane axis y; 1:
// slices along y, in-plane axis x) as z-pairs: texel (s, k1, k2) holds
// (v[k2], v[k2 + 1] - v[k2]) at (s * py + k1 + 2) * pz + k2 + 2, written for
// k1 in [0, n1) and k2 in [-1, n2 - 1] (the pair below the volume carries
// v[0] as its difference); everything else stays zero from a memset.  A CTA
// transposes a (z, x) tile of one y plane through shared memory.
__global__ void __launch_bounds__(256) build_slab_copy(const float *__restrict__ vol, size_t pitch, int nx, int ny,
                                                       int nz, int dir, long long py, long long pz,
                                                       float2 *__restrict__ out)
{
    __shared__ float t[34][33];  // t[i][xi] = v(z0 - 1 + i, y, x0 + xi), zero outside the volume
    const int z0 = blockIdx.x * 32, x0 = blockIdx.y * 32, y = blockIdx.z;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int i = ty; i < 34; i += 8) {
        const int z = z0 - 1 + i, x = x0 + tx;
        t[i][tx] = (z >= 0 && z < nz && x < nx) ? __ldg(vol + ((size_t)z * ny + y) * pitch + x) : 0.0f;
    }
    __syncthreads();
    for (int xi = ty; xi < 32; xi += 8) {
        const int x = x0 + xi;
        if (x >= nx) continue;
        const long long s = (dir == 0) ? x : y, k1 = (dir == 0) ? y : x;
        float2 *row = out + (s * py + k1 + 2) * pz + 2;
        const int z = z0 + tx;
        if (z < nz) row[z] = make_float2(t[tx + 1][xi], t[tx + 2][xi] - t[tx + 1][xi]);
        if (z0 == 0 && tx == 0) row[-1] = make_float2(0.0f, t[1][xi]);
    }
}

bool slab_enabled()
{
    const char *e = std::getenv("B2T_FP_PATH");
    return !(e && e[0] == 'c');  // B2T_FP_PATH=cells keeps the cell kernels for every view
}

long long slab_pz(const b2t_dims3d &d) { return ((long long)d.vol_z + 4 + 1) & ~1ll; }

}  // namespace

static std::atomic<unsigned long long> g_slab_launches{0};

b2t_status fp_path_stats_impl(uint64_t *stats)
{
    unsigned long long v[2] = {0, 0};
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(v, g_fp_slab_slices, sizeof(v)), "read FP path statistics");
    const unsigned long long zero[2] = {0, 0};
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_fp_slab_slices, zero, sizeof(zero)), "clear FP path statistics");
    stats[0] = v[0];
    stats[1] = v[1];
    stats[2] = g_slab_launches.exchange(0);
    stats[3] = fp_cell_launches_take();
    return B2T_OK;
}

b2t_status fp_slab_errors(uint32_t *flags)
{
    unsigned int v = 0;
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_fp_slab_errors, sizeof(v)), "read FP error word");
    const unsigned int zero = 0;
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_fp_slab_errors, &zero, sizeof(zero)), "clear FP error word");
    *flags = v;
    return B2T_OK;
}

bool fp_slab_eligible(const b2t_geom3d *g, const b2t_params3d *p, int32_t dtype, int dir, const std::vector<int> &dirs)
{
    if (!slab_enabled() || dtype != B2T_F32 || dir > 1 || p->det_supersample != 1) return false;
    const b2t_dims3d &d = g->dims;
    for (uint32_t a = 0; a < d.angles; ++a) {
        if (dirs[a] != dir) continue;
        FPView w;
        fp_view_coeffs(g->kind, g->views[a], d, dir, w);
        if (w.e[2] != 0.0f || w.m1[2] != 0.0f || w.n1[2] != 0.0f) return false;
    }
    return true;
}

size_t fp_slab_copy_bytes(const b2t_dims3d &d, int dir)
{
    const size_t n0 = dir == 0 ? d.vol_x : d.vol_y, n1 = dir == 0 ? d.vol_y : d.vol_x;
    return n0 * (n1 + 4) * (size_t)slab_pz(d) * sizeof(float2);
}

b2t_status fp_slab_build(const b2t_dims3d &d, const float *vol, size_t vol_pitch, int dir, void *copy,
                         cudaStream_t s)
{
    const long long n1 = dir == 0 ? d.vol_y : d.vol_x;
    B2T_CUDA_TRY(cudaMemsetAsync(copy, 0, fp_slab_copy_bytes(d, dir), s), "slab copy clear");
    dim3 grid((d.vol_z + 31) / 32, (d.vol_x + 31) / 32, d.vol_y);
    build_slab_copy<<<grid, 256, 0, s>>>(vol, vol_pitch, d.vol_x, d.vol_y, d.vol_z, dir, n1 + 4, slab_pz(d),
                                         static_cast<float2 *>(copy));
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "slab copy launch");
    return B2T_OK;
}

b2t_status fp_slab_project(const b2t_geom3d *g, const b2t_params3d *p, const void *copy, int dir, void *proj,
                           size_t proj_pitch, int32_t mode, const std::vector<int> &dirs, cudaStream_t s)
{
    const b2t_dims3d &d = g->dims;
    SlabLaunch *Lp = new SlabLaunch;
    SlabLaunch &L = *Lp;
    L.n0 = dir == 0 ? d.vol_x : d.vol_y;
    L.n1 = dir == 0 ? d.vol_y : d.vol_x;
    L.n2 = d.vol_z;
    L.py = L.n1 + 4;
    L.pz = slab_pz(d);
    L.copy = static_cast<const float2 *>(copy);
    // 8-byte elements (the z-pairs, copied bit for bit); zero fill outside
    const uint64_t dims[3] = {(uint64_t)L.n2 + 4, (uint64_t)L.py, (uint64_t)L.n0};
    const uint64_t strides[2] = {(uint64_t)L.pz * sizeof(float2), (uint64_t)(L.pz * L.py) * sizeof(float2)};
    b2t_status st = B2T_OK;
    for (int k = 0; k < 2 && st == B2T_OK; ++k) {
        const uint32_t box[3] = {(uint32_t)(k == 0 ? SLAB_WA : SLAB_WB), SLAB_BOX_Y, 1};
        st = encode_tensor_map(&L.tmap[k], CU_TENSOR_MAP_DATA_TYPE_INT64, 3, copy, dims, strides, box);
    }
    if (st != B2T_OK) {
        delete Lp;
        return st;
    }
    L.proj = proj;
    L.proj_pitch = (long long)proj_pitch;
    L.nu = d.det_u;
    L.nv = d.det_v;
    L.na = d.angles;
    L.accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
    fp_scale(g->kind, dir, g->vol_scale, false, p->output_scale, L.f1, L.f2, L.mul);
    std::vector<int> views;
    for (uint32_t a = 0; a < d.angles; ++a)
        if (dirs[a] == dir) views.push_back((int)a);
    const size_t smem = (size_t)SLAB_STAGES * SLAB_SLOT * sizeof(float2) +
                        SLAB_STAGES * (2 * sizeof(uint64_t) + sizeof(SlabInfo)) + 2 * sizeof(int);
    static bool attr_set = false;
    if (!attr_set) {
        B2T_CUDA_TRY(cudaFuncSetAttribute(fp3d_slab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     "slab FP shared memory attribute");
        attr_set = true;
    }
    for (size_t c0 = 0; c0 < views.size() && st == B2T_OK; c0 += SLAB_MAX_VIEWS) {
        const size_t cn = std::min(views.size() - c0, (size_t)SLAB_MAX_VIEWS);
        L.nviews = (int)cn;
        for (size_t i = 0; i < cn; ++i) {
            fp_view_coeffs(g->kind, g->views[views[c0 + i]], d, dir, L.views[i]);
            L.views[i].a = views[c0 + i];
        }
        dim3 grid((unsigned)((cn + SLAB_W - 1) / SLAB_W), (d.det_u + SLAB_U - 1) / SLAB_U,
                  (d.det_v + SLAB_ROWS - 1) / SLAB_ROWS);
        fp3d_slab_kernel<<<grid, SLAB_THREADS, smem, s>>>(L);
        count_launches(1);
        g_slab_launches.fetch_add(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "fp3d_slab_kernel launch");
    }
    delete Lp;
    return st;
}

// ---- the FP's transpose (matched BP) for the views the slab FP takes

static std::atomic<unsigned long long> g_mt_launches{0};

bool matched_slab_eligible(const b2t_geom3d *g, const b2t_params3d *p, int dir, const std::vector<int> &dirs)
{
    // opt-in (B2T_MATCHED_PATH=slab): the per-sample global reductions of
    // matched.cu are faster on this hardware, see the kernel's comment
    const char *e = std::getenv("B2T_MATCHED_PATH");
    if (!(e && std::string(e) == "slab") || dir > 1 || p->det_supersample != 1) return false;
    const b2t_dims3d &d = g->dims;
    for (uint32_t a = 0; a < d.angles; ++a) {
        if (dirs[a] != dir) continue;
        FPView w;
        fp_view_coeffs(g->kind, g->views[a], d, dir, w);
        if (w.e[2] != 0.0f || w.m1[2] != 0.0f || w.n1[2] != 0.0f) return false;
    }
    return true;
}

void matched_slab_dims(const b2t_dims3d &d, int dir, long long &ay, long long &az)
{
    // room for a whole box past the far border: no TMA reduce leaves the array
    ay = (long long)(dir == 0 ? d.vol_y : d.vol_x) + 4 + SLAB_BY;
    az = ((long long)d.vol_z + 4 + MT_WB + 3) & ~3ll;
}

size_t matched_slab_acc_bytes(const b2t_dims3d &d, int dir)
{
    long long ay, az;
    matched_slab_dims(d, dir, ay, az);
    return (size_t)(dir == 0 ? d.vol_x : d.vol_y) * (size_t)ay * (size_t)az * sizeof(float);
}

template <typename T> static b2t_status launch_mt(const SlabLaunch &L, dim3 grid, size_t smem, cudaStream_t s)
{
    static bool attr_set = false;
    if (!attr_set) {
        B2T_CUDA_TRY(cudaFuncSetAttribute(bp3d_slab_matched_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem),
                     "slab matched BP shared memory attribute");
        attr_set = true;
    }
    bp3d_slab_matched_kernel<T><<<grid, SLAB_THREADS, smem, s>>>(L);
    count_launches(1);
    g_mt_launches.fetch_add(1);
    B2T_CUDA_TRY(cudaGetLastError(), "bp3d_slab_matched_kernel launch");
    return B2T_OK;
}

b2t_status matched_slab_scatter(const b2t_geom3d *g, const b2t_params3d *p, const void *proj, size_t proj_pitch,
                                int32_t dtype, int dir, const std::vector<int> &dirs, float *acc, cudaStream_t s)
{
    const b2t_dims3d &d = g->dims;
    SlabLaunch *Lp = new SlabLaunch;
    SlabLaunch &L = *Lp;
    L.n0 = dir == 0 ? d.vol_x : d.vol_y;
    L.n1 = dir == 0 ? d.vol_y : d.vol_x;
    L.n2 = d.vol_z;
    L.copy = nullptr;
    L.py = L.pz = 0;
    L.acc = acc;
    matched_slab_dims(d, dir, L.ay, L.az);
    const uint64_t dims[3] = {(uint64_t)L.az, (uint64_t)L.ay, (uint64_t)L.n0};
    const uint64_t strides[2] = {(uint64_t)L.az * sizeof(float), (uint64_t)(L.az * L.ay) * sizeof(float)};
    b2t_status st = B2T_OK;
    for (int k = 0; k < 2 && st == B2T_OK; ++k) {
        const uint32_t box[3] = {(uint32_t)(k == 0 ? MT_WA : MT_WB), SLAB_BOX_Y, 1};
        st = encode_tensor_map(&L.tmap[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, acc, dims, strides, box);
    }
    if (st != B2T_OK) {
        delete Lp;
        return st;
    }
    L.proj = const_cast<void *>(proj);
    L.proj_pitch = (long long)proj_pitch;
    L.nu = d.det_u;
    L.nv = d.det_v;
    L.na = d.angles;
    L.accumulate = 0;
    fp_scale(g->kind, dir, g->vol_scale, false, p->output_scale, L.f1, L.f2, L.mul);
    std::vector<int> views;
    for (uint32_t a = 0; a < d.angles; ++a)
        if (dirs[a] == dir) views.push_back((int)a);
    const size_t smem = (size_t)MT_STAGES * MT_SLOT * sizeof(float) +
                        MT_STAGES * (2 * sizeof(uint64_t) + sizeof(MTInfo)) + 2 * sizeof(int);
    for (size_t c0 = 0; c0 < views.size() && st == B2T_OK; c0 += SLAB_MAX_VIEWS) {
        const size_t cn = std::min(views.size() - c0, (size_t)SLAB_MAX_VIEWS);
        L.nviews = (int)cn;
        for (size_t i = 0; i < cn; ++i) {
            fp_view_coeffs(g->kind, g->views[views[c0 + i]], d, dir, L.views[i]);
            L.views[i].a = views[c0 + i];
        }
        dim3 grid((unsigned)((cn + SLAB_W - 1) / SLAB_W), (d.det_u + SLAB_U - 1) / SLAB_U,
                  (d.det_v + SLAB_ROWS - 1) / SLAB_ROWS);
        if (dtype == B2T_F32) st = launch_mt<float>(L, grid, smem, s);
        else if (dtype == B2T_F16) st = launch_mt<__half>(L, grid, smem, s);
        else st = launch_mt<__nv_bfloat16>(L, grid, smem, s);
    }
    delete Lp;
    return st;
}

b2t_status matched_path_stats_impl(uint64_t *stats)
{
    unsigned long long v[2] = {0, 0};
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(v, g_mt_slab_slices, sizeof(v)), "read matched BP path statistics");
    const unsigned long long zero[2] = {0, 0};
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_mt_slab_slices, zero, sizeof(zero)), "clear matched BP path statistics");
    stats[0] = v[0];
    stats[1] = v[1];
    stats[2] = g_mt_launches.exchange(0);
    stats[3] = matched_scatter_launches_take();
    return B2T_OK;
}

}  // namespace b2t
