// Voxel-driven 3D backprojection with TMA-staged projection tiles.
//
// Same model as bp3d_kernel (the reference's dev_cone_BP / dev_par3D_BP,
// cuda/3d/cone_bp.cu:55-133, cuda/3d/par3d_bp.cu:55-120): every voxel centre
// is projected onto each view, the projection is sampled bilinearly and
// weighted.  The difference is where the samples come from:
//
//   - a CTA owns a 32 x 8 x 32 voxel block and walks all views of the launch
//     with eight compute warps and one producer warp;
//   - for each view the producer projects the block's eight corner voxels,
//     takes the bounding box of their detector coordinates (plus one texel of
//     margin), reserves the rows of that box in a ring of shared memory and
//     loads them from the zero-padded projections with 8-row
//     cp.async.bulk.tensor boxes, signalling the view's mbarrier.  Tiles take
//     only the rows their footprint needs, so the ring holds several views
//     (up to eight) ahead of the compute warps;
//   - the compute warps interpolate from shared memory.  For circular
//     geometries (detector v axis along z) the detector u coordinate and the
//     ray-density weight do not depend on z, so each thread computes them once
//     per view (from affine forms the producer folds per block) and only v
//     changes along its 32-voxel column; voxels j and j + 1 of the column
//     share packed f32x2 instructions (sm_100a), and 16-bit projections are
//     staged as pairs of vertically adjacent texels, so that a sample takes
//     two 32-bit shared loads and one packed 16-bit interpolation along u;
//   - a tile that does not fit (extreme magnification) is read from the padded
//     projections in global memory instead.
//
// Every mbarrier wait is bounded (about a second); on timeout the kernel sets
// B2T_DEVERR_WAIT_TIMEOUT in g_b2t_device_errors and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "b2t_internal.h"
#include "f32x2.cuh"
#include "proj3d.h"
#include "ramp_tc.h"
#include "tma.h"

namespace b2t {

// error word of this translation unit (see b2t_device_errors)
static __device__ unsigned int g_b2t_device_errors = 0;

// Path statistics of the TMA backprojection, read and cleared by
// b2t_bp_path_stats.  In voxel-column views (one thread's column of 16 or 32
// voxels for one view): [0] the circular fast path (all samples from the
// shared-memory tile), [1] the general path (other orbits, columns whose
// rows leave the tile, views read from global memory), [2] lanes idle
// because their column lies outside the volume; [3] SM cycles the compute
// warps spent in their view loops, summed over warps.
static __device__ unsigned long long g_bp_path_stats[4] = {0, 0, 0, 0};

namespace {

template <typename T> __device__ __forceinline__ float lds(const T *p);
template <> __device__ __forceinline__ float lds<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float lds<__half>(const __half *p) { return __half2float(*p); }
template <> __device__ __forceinline__ float lds<__nv_bfloat16>(const __nv_bfloat16 *p) { return __bfloat162float(*p); }

template <typename T> __device__ __forceinline__ float ldgt(const T *p);
template <> __device__ __forceinline__ float ldgt<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ldgt<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float ldgt<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(__ldg(p));
}
template <typename T> __device__ __forceinline__ T tot(float v);
template <> __device__ __forceinline__ float tot<float>(float v) { return v; }
template <> __device__ __forceinline__ __half tot<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 tot<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ void split_texel_t(float qm, int &k, float &f)
{
    const float M = 12582912.0f;
    float t = __fadd_rn(qm, M);
    float r = __fadd_rn(t, -M);
    k = __float_as_int(t) - 0x4B400000;
    f = __fadd_rn(__fadd_rn(qm, -r), 0.5f);
}

// FP32 texel at 32-bit shared address a + OFF (OFF an immediate of the
// instruction, so the texels of a sample share one address register).
template <typename T, int OFF> __device__ __forceinline__ float lds_sh(uint32_t a)
{
    static_assert(sizeof(T) == 4, "16-bit texels are read as pairs");
    float v;
    asm volatile("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(a), "n"(OFF));
    return v;
}

// A pair of 16-bit texels in one 32-bit word, as two floats.
template <typename T, typename E> __device__ __forceinline__ float2 pair_f2(E v)
{
    if constexpr (std::is_same<T, __half>::value) return __half22float2(v);
    else return __bfloat1622float2(v);
}
// The 32-bit word at shared address a + OFF.
template <int OFF> __device__ __forceinline__ uint32_t lds_b32(uint32_t a)
{
    uint32_t v;
    asm volatile("ld.shared.b32 %0, [%1+%2];" : "=r"(v) : "r"(a), "n"(OFF));
    return v;
}

// Storage of the padded projections the kernel reads: FP32 texels, or for
// the 16-bit types the pair layout (padded_elem_size), whose element (v, u)
// is the 32-bit word (x[v][u], x[v+1][u]), a texel and the one below it.  A
// bilinear sample then takes two 32-bit loads from one row of pairs (columns
// u and u + 1) instead of four 16-bit loads, half the shared-memory
// wavefronts, and the interpolation along u of both rows is one packed
// 16-bit fused multiply-add.
template <typename T, bool PAIR> struct Elem {
    using type = T;
};
template <> struct Elem<__half, true> {
    using type = __half2;
};
template <> struct Elem<__nv_bfloat16, true> {
    using type = __nv_bfloat162;
};
template <typename T, bool PAIR> using elem_t = typename Elem<T, PAIR>::type;

// x in both halves of a 16-bit pair (x itself for FP32).
template <typename T> __device__ __forceinline__ elem_t<T, true> splat2(float x)
{
    if constexpr (std::is_same<T, __half>::value) return __float2half2_rn(x);
    else if constexpr (std::is_same<T, __nv_bfloat16>::value) return __float2bfloat162_rn(x);
    else return x;
}

// Bilinear sample with weights fu (along u) and fv (along v) from element p
// of shared memory (GLOBAL false) or of the padded projections in global
// memory, rows rs elements apart.
template <typename T, bool PAIR, bool GLOBAL>
__device__ __forceinline__ float bilerp(const elem_t<T, PAIR> *p, long long rs, float fu, float fv)
{
    float v00, v10, v01, v11;
    if constexpr (PAIR) {
        // columns u and u + 1 of the pair row (rs unused)
        const float2 c0 = pair_f2<T>(GLOBAL ? __ldg(p) : p[0]), c1 = pair_f2<T>(GLOBAL ? __ldg(p + 1) : p[1]);
        v00 = c0.x;
        v01 = c0.y;
        v10 = c1.x;
        v11 = c1.y;
    } else {
        v00 = GLOBAL ? ldgt(p) : lds(p);
        v10 = GLOBAL ? ldgt(p + 1) : lds(p + 1);
        v01 = GLOBAL ? ldgt(p + rs) : lds(p + rs);
        v11 = GLOBAL ? ldgt(p + rs + 1) : lds(p + rs + 1);
    }
    const float a = fmaf(fu, v10 - v00, v00);
    const float b = fmaf(fu, v11 - v01, v01);
    return fmaf(fv, b - a, a);
}

// Tile width and ring row pitch in 4-byte elements: a TMA box row must be a
// multiple of 16 bytes, and rows that share shared-memory banks should be far
// apart (84 x 4 B: 8 rows).
template <typename E> __host__ __device__ constexpr int tile_bu()
{
    static_assert(sizeof(E) == 4, "tile elements are FP32 texels or 16-bit pairs");
    return 84;
}
// Ring rows (multiple of BPT_CHUNK) in the BPT_RING_BYTES of shared memory.
// An 8-row chunk is a multiple of 128 bytes, so every chunk destination (ring
// rows are allocated in whole chunks) is 128-byte aligned.
template <typename E> __host__ __device__ constexpr int ring_rows()
{
    return (BPT_RING_BYTES / (tile_bu<E>() * (int)sizeof(E))) & ~(BPT_CHUNK - 1);
}
static_assert(BPT_CHUNK * 84 * 4 % 128 == 0, "chunk alignment");
static_assert((84 * 4) % 16 == 0, "TMA box row bytes");
static_assert(ring_rows<float>() >= BPT_BV, "the ring holds the largest view");

// View i's coefficients from the launch record: 10 floats a view in circular
// launches (nu.z and den.z are zero there), 12 otherwise.
template <bool CIRC> __device__ __forceinline__ BPView view_rec(const BPTmaLaunch &L, int i)
{
    BPView W;
    if constexpr (CIRC) {
        const float *f = L.vrec + 10 * i;
        W.nu = make_float4(f[0], f[1], 0.0f, f[2]);
        W.nv = make_float4(f[3], f[4], f[5], f[6]);
        W.den = make_float4(f[7], f[8], 0.0f, f[9]);
    } else {
        const float *f = L.vrec + 12 * i;
        W.nu = make_float4(f[0], f[1], f[2], f[3]);
        W.nv = make_float4(f[4], f[5], f[6], f[7]);
        W.den = make_float4(f[8], f[9], f[10], f[11]);
    }
    return W;
}

// Per-view record written by the producer warp: the tile's origin in padded
// texels (u0, v0), its first ring row and its row count (0: the footprint does
// not fit a tile, read global memory), and for circular geometries the
// view's coefficients folded into affine forms of the thread's offset
// (lx, ly) inside the CTA's block at the block's first z slice, with the
// tile origin absorbed:
//   cone:     U = (cu.w + cu.x lx + cu.y ly) / D,  V_j = (cv.w + cv.x lx + cv.y ly + j cv.z) / D,
//             D = cd.w + cd.x lx + cd.y ly
//   parallel: the same without the division; cd.w is the ray weight
// U and V are tile-relative sample positions (texel k = floor, weight frac on
// k + 1).
struct StageInfo {
    int u0, v0, row0, nrows;
    float4 cu, cv, cd;
};

// Projected detector coordinates (texture units) of voxel centre (fx, fy, fz).
// D is the cone denominator (1 for parallel beams).
template <int KIND>
__device__ __forceinline__ void project(const BPView &W, float fx, float fy, float fz, float &U, float &V, float &D)
{
    float nu = fmaf(fz, W.nu.z, fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)));
    float nv = fmaf(fz, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
    if (KIND == B2T_GEOM_CONE) {
        const float dn = fmaf(fz, W.den.z, fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w)));
        const float fr = __frcp_rn(dn);
        U = nu * fr;
        V = nv * fr;
        D = dn;
    } else {
        U = nu;
        V = nv;
        D = 1.0f;
    }
}

// c.w + c.x ox + c.y oy + c.z oz + k (d.w + d.x ox + d.y oy + d.z oz), in FP64
__device__ __forceinline__ float4 fold_form(float4 c, float4 d, double k, double ox, double oy, double oz, bool keep_z)
{
    const double cx = (double)c.x + k * d.x, cy = (double)c.y + k * d.y, cz = (double)c.z + k * d.z;
    const double cw = (double)c.w + k * d.w;
    const double w0 = cw + cx * ox + cy * oy + cz * oz;
    return make_float4((float)cx, (float)cy, keep_z ? (float)cz : 0.0f, (float)w0);
}

// Producer warp of bp3d_tma_kernel (a separate function so that its
// registers are allocated apart from the compute warps' accumulators).
// Lane l works out view vb + l of each batch of 32: its footprint, tile
// origin, row count and folded record, all independent of where the tile
// lands in the ring.  The views then go through the ring one at a time: the
// warp finds room together (waiting for the oldest views to be released) and
// the view's own lane issues the loads and writes the record.
template <typename E, int KIND, bool CIRC, int ZB>
__device__ __noinline__ void bp_produce(const BPTmaLaunch &L, E *ring, uint64_t *full, uint64_t *empty,
                                        StageInfo *info, int lane, float cx,
                                        float cy, float fz0)
{
    constexpr int R = ring_rows<E>();
    constexpr int BU = tile_bu<E>();
    // voxel-centre extent of the block; along z the block's full ZB
    // slices, so that the voxels computed past the volume's last slice
    // (and discarded) also project inside the tile
    const float bx0 = (float)(blockIdx.x * 32) + cx, bx1 = (float)(min(L.nx, (int)blockIdx.x * 32 + 32) - 1) + cx;
    const float by0 = (float)(blockIdx.y * 8) + cy, by1 = (float)(min(L.ny, (int)blockIdx.y * 8 + 8) - 1) + cy;
    const float bz0 = fz0, bz1 = fz0 + (float)(ZB - 1);
    int j0 = 0;         // oldest view still held by the compute warps
    int head = 0;       // next free ring row
    int slot_row0 = 0;  // lane s < BPT_SLOTS: first ring row of the view in slot s
    int slot_rows = 0;  // lane s < BPT_SLOTS: its row count (0: it reads global memory)
    for (int vb = 0; vb < L.nviews; vb += 32) {
        const int v = vb + lane;
        StageInfo r;
        r.u0 = r.v0 = r.row0 = r.nrows = 0;
        r.cu = r.cv = r.cd = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (v < L.nviews) {
            const BPView W = view_rec<CIRC>(L, v);
            float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f, dmin = 3.0e38f;
#pragma unroll 1
            for (int c = 0; c < 8; ++c) {
                float U, V, D;
                project<KIND>(W, (c & 1) ? bx1 : bx0, (c & 2) ? by1 : by0, (c & 4) ? bz1 : bz0, U, V, D);
                umin = fminf(umin, U);
                umax = fmaxf(umax, U);
                vmin = fminf(vmin, V);
                vmax = fmaxf(vmax, V);
                dmin = fminf(dmin, D);
            }
            // padded texel index of continuous coordinate c is floor(c - 0.5) + 2;
            // one texel of margin on each side for rounding in the consumers.
            // A cone denominator positive at all eight corners is positive on
            // the whole block, which then projects inside the corners' box.
            const float lim = 1.0e7f;
            if (dmin > 0.0f && umin > -lim && umax < lim && vmin > -lim && vmax < lim) {
                const int ua = (int)floorf(umin - 0.5f) + 2 - 1;
                const int ub = (int)floorf(umax - 0.5f) + 2 + 2;
                const int va = (int)floorf(vmin - 0.5f) + 2 - 1;
                const int vb2 = (int)floorf(vmax - 0.5f) + 2 + 2;
                const int u0 = ua & ~7;  // TMA: x * element size must be 16-byte aligned
                const int rows = (vb2 - va + BPT_CHUNK) & ~(BPT_CHUNK - 1);  // rows va..vb2, whole chunks
                if (ub - u0 < BU && rows <= BPT_BV) {
                    r.u0 = u0;
                    r.v0 = va;
                    r.nrows = rows;
                }
            }
            if (CIRC && r.nrows > 0) {
                // sample position in tile texels: c + 1.5 - origin (c the
                // continuous detector coordinate, origin the padded index)
                const double ox = bx0, oy = by0, oz = bz0;
                if (KIND == B2T_GEOM_CONE) {
                    r.cu = fold_form(W.nu, W.den, 1.5 - r.u0, ox, oy, oz, false);
                    r.cv = fold_form(W.nv, W.den, 1.5 - r.v0, ox, oy, oz, true);
                    r.cd = fold_form(W.den, W.den, 0.0, ox, oy, oz, false);
                } else {
                    const float4 one = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
                    r.cu = fold_form(W.nu, one, 1.5 - r.u0, ox, oy, oz, false);
                    r.cv = fold_form(W.nv, one, 1.5 - r.v0, ox, oy, oz, true);
                    r.cd = make_float4(0.0f, 0.0f, 0.0f, W.den.w);
                }
            }
        }
        const int cnt = min(32, L.nviews - vb);
        for (int k = 0; k < cnt; ++k) {
            // warp-uniform from here on: every lane follows the same room
            // search, so each lane also acquires the released views itself
            const int nrows = __shfl_sync(0xffffffffu, r.nrows, k);
            const int vk = vb + k;
            const int slot = vk % BPT_SLOTS;
            int at = 0;
            // room: a free slot and nrows contiguous ring rows; views leave
            // the ring in order, so wait for the oldest
            for (;;) {
                const int live = vk - j0;
                if (live < BPT_SLOTS) {
                    if (nrows == 0) {
                        at = head;
                        break;
                    }
                    // the occupied rows start at the oldest live view that
                    // holds rows; with none the ring is empty
                    int tail = -1;
                    for (int q = j0; q < vk && tail < 0; ++q) {
                        const int r0 = __shfl_sync(0xffffffffu, slot_row0, q % BPT_SLOTS);
                        if (__shfl_sync(0xffffffffu, slot_rows, q % BPT_SLOTS) > 0) tail = r0;
                    }
                    if (tail < 0) {
                        head = 0;
                        at = 0;
                        break;
                    }
                    if (head > tail) {
                        if (R - head >= nrows) {
                            at = head;
                            break;
                        }
                        if (tail >= nrows) {
                            at = 0;
                            break;
                        }
                    } else if (head < tail && tail - head >= nrows) {
                        at = head;
                        break;
                    }
                }
                if (!__all_sync(0xffffffffu, mbar_wait_bounded_sleep(&empty[j0 % BPT_SLOTS],
                                                               (uint32_t)((j0 / BPT_SLOTS) & 1), 2000000000LL))) {
                    if (lane == 0) atomicOr(&g_b2t_device_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
                    // the copies already issued (views j0 .. vk - 1, one per
                    // slot) land before the warp leaves
                    for (int q = j0; q < vk; ++q)
                        (void)mbar_wait_bounded_sleep(&full[q % BPT_SLOTS], (uint32_t)((q / BPT_SLOTS) & 1),
                                                      2000000000LL);
                    return;
                }
                ++j0;
            }
            if (lane == slot) {
                slot_row0 = at;
                slot_rows = nrows;
            }
            if (nrows > 0) head = at + nrows;
            if (lane == k) {
                // the loads go out before the record is written: the view's
                // phase cannot complete before the arrival, which releases
                // the record
                if (nrows > 0) {
                    mbar_expect_tx(&full[slot], (uint32_t)(nrows * BU * sizeof(E)));
                    for (int c = 0; c < nrows; c += BPT_CHUNK)
                        tma_load_3d(ring + (size_t)(at + c) * BU, &L.tmap, r.u0, L.a0 + vk, r.v0 + c, &full[slot]);
                }
                r.row0 = at;
                info[slot] = r;
                mbar_arrive(&full[slot]);
            }
        }
    }
    // the last views' copies land before the warp leaves: the CTA cannot end
    // with bulk copies in flight, even when the compute warps give up on a
    // wait (views j0 .. nviews - 1 hold one slot each)
    for (int q = j0; q < L.nviews; ++q)
        (void)mbar_wait_bounded_sleep(&full[q % BPT_SLOTS], (uint32_t)((q / BPT_SLOTS) & 1), 2000000000LL);
}

// 288 threads: warps 0-7 backproject a 32 x 8 x ZB voxel block, warp 8
// streams the views' tiles into the ring ahead of them.
template <typename T, int KIND, int KER, bool CIRC, int ZB>
__global__ void __launch_bounds__(288, BPT_CTAS_PER_SM) bp3d_tma_kernel(const __grid_constant__ BPTmaLaunch L)
{
    constexpr bool PAIR = sizeof(T) == 2;  // 16-bit texels are stored as pairs
    using E = elem_t<T, PAIR>;
    constexpr int R = ring_rows<E>();
    constexpr int BU = tile_bu<E>();
    extern __shared__ __align__(128) unsigned char smraw[];
    E *ring = reinterpret_cast<E *>(smraw);
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw + (size_t)R * BU * sizeof(E));
    uint64_t *empty = full + BPT_SLOTS;
    StageInfo *info = reinterpret_cast<StageInfo *>(empty + BPT_SLOTS);

    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int z0 = blockIdx.z * ZB;

    if (tid == 0) {
        for (int s = 0; s < BPT_SLOTS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);  // one arrival per compute warp when it is done with the view
        }
        mbar_fence_init();
        tma_prefetch_map(&L.tmap);
    }
    __syncthreads();

    if (warp == 8) {
        const float cx = 0.5f - 0.5f * (float)L.nx, cy = 0.5f - 0.5f * (float)L.ny;
        const float fz0 = (float)z0 + 0.5f - 0.5f * (float)L.nz;
        bp_produce<E, KIND, CIRC, ZB>(L, ring, full, empty, info, lane, cx, cy, fz0);
        return;
    }

    // ---- compute warps
    // a warp covers 8 x 4 voxels, so its detector footprint in a tile row
    // stays under 32 texels; the 8 warps tile the 32 x 8 block
    const int x = blockIdx.x * 32 + (warp & 3) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 2) * 4 + (lane >> 3);
    const bool active = (x < L.nx) && (y < L.ny);
    // this thread's offset inside the block
    const float lx = (float)(x - (int)blockIdx.x * 32), ly = (float)(y - (int)blockIdx.y * 8);

    float acc[ZB];
#pragma unroll
    for (int j = 0; j < ZB; ++j) acc[j] = 0.0f;

    unsigned long long n_fast = 0, n_general = 0, n_idle = 0;  // this thread's column-views by path
    const long long t_loop = clock64();
    int slot = 0;
    uint32_t parity = 0;
    for (int i = 0; i < L.nviews; ++i) {
        // every wait is bounded: a warp that gives up records the error and
        // leaves; the producer then gives up on the release it no longer
        // gets, so the kernel always ends
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[slot], parity, 2000000000LL))) {
            if (lane == 0) atomicOr(&g_b2t_device_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
            return;
        }
        const int4 hd = *reinterpret_cast<const int4 *>(&info[slot]);  // u0, v0, row0, nrows
        const E *tile = ring + (size_t)hd.z * BU;
        bool done = false;
        if (CIRC && active && hd.w > 0) {
            // u and the weight are independent of z, v is linear in z
            const float4 cu = info[slot].cu, cv = info[slot].cv, cd = info[slot].cd;
            float Uq = fmaf(ly, cu.y, fmaf(lx, cu.x, cu.w));
            float Vq = fmaf(ly, cv.y, fmaf(lx, cv.x, cv.w));
            float dV = cv.z, w;
            if (KIND == B2T_GEOM_CONE) {
                const float fr = __frcp_rn(fmaf(ly, cd.y, fmaf(lx, cd.x, cd.w)));
                Uq *= fr;
                Vq *= fr;
                dV *= fr;
                w = (KER == B2T_KER_2D_WEIGHTING) ? fr : fr * fr;
            } else {
                w = cd.w;
            }
            const float M = 12582912.0f;  // 1.5 * 2^23: q + M rounded down holds floor(q) in its mantissa
            // q_j = Vq + j dV is monotone in j (fmaf and rounding down are
            // monotone), so the rows of all ZB voxels are inside the tile
            // when the first and the last are
            const int ka = __float_as_int(__fadd_rd(Vq, M)) - 0x4B400000;
            const int kb = __float_as_int(__fadd_rd(fmaf((float)(ZB - 1), dV, Vq), M)) - 0x4B400000;
            if (min(ka, kb) >= 0 && max(ka, kb) <= hd.w - 2) {
                const float tU = __fadd_rd(Uq, M);
                const float fu = Uq - (tU - M);
                const int ku = min(max(__float_as_int(tU) - 0x4B400000, 0), BU - 2);
                // shared address of row floor(q_j), column ku, is
                // bits(q_j + M) * row bytes + abase (32-bit wrap-around)
                constexpr uint32_t ROWB = BU * sizeof(E);
                // the row bytes come from the launch record: with the literal
                // constant the compiled loop issued about three ALU-pipe
                // instructions per address below instead of one multiply-add
                // (measured: 4.6 against 1.8 ALU instructions per warp-sample)
                const uint32_t rowb = L.tile_row_bytes;
                const uint32_t abase = smem_u32(tile) + (uint32_t)ku * (uint32_t)sizeof(E) - 0x4B400000u * rowb;
                // voxels j, j + 1 in the two halves of packed f32x2
                // operations; each half rounds as the scalar texel form
                // fmaf(fv, b - a, a), a = fmaf(fu, v10 - v00, v00), ...
                const uint64_t dV2 = pk2(dV, dV), Vq2 = pk2(Vq, Vq), w2 = pk2(w, w), fu2 = pk2(fu, fu);
                const uint64_t M2 = pk2(M, M), nM2 = pk2(-M, -M), two2 = pk2(2.0f, 2.0f);
                // (j, j + 1), stepped by exact additions (the literal pairs
                // would take two register moves each)
                uint64_t j2 = pk2(0.0f, 1.0f);
                using H2 = elem_t<T, true>;
                const H2 fuh = splat2<T>(fu);  // 16-bit pairs: fu for the packed interpolation along u
#pragma unroll
                for (int j = 0; j < ZB; j += 2, j2 = add2(j2, two2)) {
                    const uint64_t q2 = fma2(j2, dV2, Vq2);
                    const uint64_t t2 = add2_rd(q2, M2);
                    const uint64_t fv2 = sub2(q2, add2(t2, nM2));
                    const float2 t = upk2(t2);
                    const uint32_t a0 = (uint32_t)__float_as_int(t.x) * rowb + abase;
                    const uint32_t a1 = (uint32_t)__float_as_int(t.y) * rowb + abase;
                    uint64_t av, bv;
                    if constexpr (PAIR) {
                        // (a, b) = (v00, v01) + fu ((v10, v11) - (v00, v01))
                        // in 16-bit arithmetic, then the blend along v in FP32
                        float2 ab[2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const uint32_t c0 = lds_b32<0>(h ? a1 : a0), c1 = lds_b32<4>(h ? a1 : a0);
                            const H2 x0 = *reinterpret_cast<const H2 *>(&c0), x1 = *reinterpret_cast<const H2 *>(&c1);
                            ab[h] = pair_f2<T>(__hfma2(fuh, __hsub2(x1, x0), x0));
                        }
                        av = pk2(ab[0].x, ab[1].x);
                        bv = pk2(ab[0].y, ab[1].y);
                    } else {
                        const uint64_t v00 = pk2(lds_sh<T, 0>(a0), lds_sh<T, 0>(a1));
                        const uint64_t v10 = pk2(lds_sh<T, 4>(a0), lds_sh<T, 4>(a1));
                        const uint64_t v01 = pk2(lds_sh<T, (int)ROWB>(a0), lds_sh<T, (int)ROWB>(a1));
                        const uint64_t v11 = pk2(lds_sh<T, (int)ROWB + 4>(a0), lds_sh<T, (int)ROWB + 4>(a1));
                        av = fma2(fu2, sub2(v10, v00), v00);
                        bv = fma2(fu2, sub2(v11, v01), v01);
                    }
                    const float2 r = upk2(fma2(fma2(fv2, sub2(bv, av), av), w2, pk2(acc[j], acc[j + 1])));
                    acc[j] = r.x;
                    acc[j + 1] = r.y;
                }
                done = true;
            }
        }
        if (done) ++n_fast;
        else if (active) ++n_general;
        else ++n_idle;
        if (active && !done) {
            // the general paths recompute the voxel centre here rather than
            // keeping it live across the hot loop above
            const E *gproj = static_cast<const E *>(L.proj);
            const float fx = (float)(blockIdx.x * 32 + (warp & 3) * 8 + (lane & 7)) + 0.5f - 0.5f * (float)L.nx;
            const float fy = (float)(blockIdx.y * 8 + (warp >> 2) * 4 + (lane >> 3)) + 0.5f - 0.5f * (float)L.ny;
            const float fz0 = (float)(blockIdx.z * ZB) + 0.5f - 0.5f * (float)L.nz;
            const BPView W = view_rec<CIRC>(L, i);
            const int u0 = hd.x, v0 = hd.y, nrows = hd.w;
            if (CIRC) {
                // u, weight independent of z; v linear in z
                float U, w, Vb, dV;
                if (KIND == B2T_GEOM_CONE) {
                    const float dn = fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w));
                    const float fr = __frcp_rn(dn);
                    U = fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)) * fr;
                    Vb = fmaf(fz0, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w))) * fr;
                    dV = W.nv.z * fr;
                    w = (KER == B2T_KER_2D_WEIGHTING) ? fr : fr * fr;
                } else {
                    U = fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w));
                    Vb = fmaf(fz0, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
                    dV = W.nv.z;
                    w = W.den.w;
                }
                if (nrows > 0) {
                    int ku;
                    float fu;
                    split_texel_t(U + 1.0f - (float)u0, ku, fu);
                    ku = min(max(ku, 0), BU - 2);
                    const float vofs = 1.0f - (float)v0;
#pragma unroll
                    for (int j = 0; j < ZB; ++j) {
                        int kv;
                        float fv;
                        split_texel_t(fmaf((float)j, dV, Vb) + vofs, kv, fv);
                        kv = min(max(kv, 0), nrows - 2);
                        acc[j] = fmaf(bilerp<T, PAIR, false>(tile + kv * BU + ku, BU, fu, fv), w, acc[j]);
                    }
                } else {
                    const E *P = gproj + (long long)(L.a0 + i) * L.pu;
                    int ku;
                    float fu;
                    split_texel_t(U - 1.0f, ku, fu);
                    ku = min(max(ku, -2), L.nu);
#pragma unroll
                    for (int j = 0; j < ZB; ++j) {
                        int kv;
                        float fv;
                        split_texel_t(fmaf((float)j, dV, Vb) - 1.0f, kv, fv);
                        kv = min(max(kv, -2), L.nv);
                        acc[j] = fmaf(bilerp<T, PAIR, true>(P + (long long)kv * L.pv + ku, L.pv, fu, fv), w, acc[j]);
                    }
                }
            } else {
                // general orientation: everything varies along z
                float nu = fmaf(fz0, W.nu.z, fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)));
                float nv = fmaf(fz0, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
                float dn = fmaf(fz0, W.den.z, fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w)));
#pragma unroll
                for (int j = 0; j < ZB; ++j) {
                    float U, Vc, w;
                    if (KIND == B2T_GEOM_CONE) {
                        const float fr = __frcp_rn(dn);
                        U = nu * fr;
                        Vc = nv * fr;
                        w = (KER == B2T_KER_2D_WEIGHTING) ? fr : fr * fr;
                    } else {
                        U = nu;
                        Vc = nv;
                        w = W.den.w;
                    }
                    int ku, kv;
                    float fu, fv, r;
                    if (nrows > 0) {
                        split_texel_t(U + 1.0f - (float)u0, ku, fu);
                        split_texel_t(Vc + 1.0f - (float)v0, kv, fv);
                        ku = min(max(ku, 0), BU - 2);
                        kv = min(max(kv, 0), nrows - 2);
                        r = bilerp<T, PAIR, false>(tile + kv * BU + ku, BU, fu, fv);
                    } else {
                        split_texel_t(U - 1.0f, ku, fu);
                        split_texel_t(Vc - 1.0f, kv, fv);
                        ku = min(max(ku, -2), L.nu);
                        kv = min(max(kv, -2), L.nv);
                        r = bilerp<T, PAIR, true>(gproj + (long long)(L.a0 + i) * L.pu + (long long)kv * L.pv + ku,
                                                  L.pv, fu, fv);
                    }
                    acc[j] = fmaf(r, w, acc[j]);
                    nu += W.nu.z;
                    nv += W.nv.z;
                    dn += W.den.z;
                }
            }
        }
        // release the view: one arrival per warp once all its lanes are done
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
        if (++slot == BPT_SLOTS) {
            slot = 0;
            parity ^= 1u;
        }
    }

    // per-thread counts are at most the launch's views, so 32-bit sums hold
    const unsigned w_fast = __reduce_add_sync(0xffffffffu, (unsigned)n_fast);
    const unsigned w_general = __reduce_add_sync(0xffffffffu, (unsigned)n_general);
    const unsigned w_idle = __reduce_add_sync(0xffffffffu, (unsigned)n_idle);
    if (lane == 0) {
        atomicAdd(&g_bp_path_stats[0], (unsigned long long)w_fast);
        atomicAdd(&g_bp_path_stats[1], (unsigned long long)w_general);
        atomicAdd(&g_bp_path_stats[2], (unsigned long long)w_idle);
        atomicAdd(&g_bp_path_stats[3], (unsigned long long)(clock64() - t_loop));
    }
    // the voxel indices are recomputed here rather than kept live across
    // the view loop (register pressure: 32 accumulators at 96 registers)
    const int xo = blockIdx.x * 32 + (threadIdx.y & 3) * 8 + (threadIdx.x & 7);
    const int yo = blockIdx.y * 8 + (threadIdx.y >> 2) * 4 + (threadIdx.x >> 3);
    if (xo < L.nx && yo < L.ny) {
        T *out = static_cast<T *>(L.vol);
#pragma unroll
        for (int j = 0; j < ZB; ++j) {
            const int z = (int)blockIdx.z * ZB + j;
            if (z < L.nz) {
                T *o = out + ((size_t)z * L.ny + yo) * L.vol_pitch + xo;
                float r = acc[j] * L.out_scale;
                if (L.accumulate) r += lds(o);
                *o = tot<T>(r);
            }
        }
    }
}

template <typename T, int KIND, int KER, bool CIRC, int ZB>
b2t_status launch_one(const BPTmaLaunch &L, const b2t_dims3d &d, cudaStream_t s)
{
    using E = elem_t<T, sizeof(T) == 2>;
    const size_t smem = (size_t)ring_rows<E>() * tile_bu<E>() * sizeof(E) +
                        BPT_SLOTS * (2 * sizeof(uint64_t) + sizeof(StageInfo));
    auto kern = bp3d_tma_kernel<T, KIND, KER, CIRC, ZB>;
    B2T_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "bp3d_tma smem attribute");
    dim3 grid((d.vol_x + 31) / 32, (d.vol_y + 7) / 8, (d.vol_z + ZB - 1) / ZB);
    kern<<<grid, dim3(32, 9), smem, s>>>(L);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "bp3d_tma launch");
    return B2T_OK;
}

template <typename T, int ZB>
b2t_status launch_kind(const BPTmaLaunch &L, int kind, int ker, bool circ, const b2t_dims3d &d, cudaStream_t s)
{
    if (kind == B2T_GEOM_PAR3D)
        return circ ? launch_one<T, B2T_GEOM_PAR3D, B2T_KER_DEFAULT, true, ZB>(L, d, s)
                    : launch_one<T, B2T_GEOM_PAR3D, B2T_KER_DEFAULT, false, ZB>(L, d, s);
    if (ker == B2T_KER_2D_WEIGHTING)
        return circ ? launch_one<T, B2T_GEOM_CONE, B2T_KER_2D_WEIGHTING, true, ZB>(L, d, s)
                    : launch_one<T, B2T_GEOM_CONE, B2T_KER_2D_WEIGHTING, false, ZB>(L, d, s);
    return circ ? launch_one<T, B2T_GEOM_CONE, B2T_KER_DEFAULT, true, ZB>(L, d, s)
                : launch_one<T, B2T_GEOM_CONE, B2T_KER_DEFAULT, false, ZB>(L, d, s);
}

template <typename T>
b2t_status launch_shape(const BPTmaLaunch &L, int kind, int ker, bool circ, int vpt, const b2t_dims3d &d,
                        cudaStream_t s)
{
    return vpt == 16 ? launch_kind<T, 16>(L, kind, ker, circ, d, s) : launch_kind<T, 32>(L, kind, ker, circ, d, s);
}

// Voxels per thread chosen by b2t_autotune_bp3d, per problem class, for this
// process; the autotuner's candidate while it times one on this thread.
std::mutex g_vpt_mutex;
std::map<std::string, int> g_vpt;
thread_local int t_vpt_override = 0;

std::string vpt_key(const b2t_geom3d *g, int32_t dtype)
{
    const b2t_dims3d &d = g->dims;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "%d/%d/%u/%u/%u/%u/%u/%u", g->kind, dtype, d.vol_x, d.vol_y, d.vol_z, d.angles,
                  d.det_u, d.det_v);
    return buf;
}

// The autotuner's candidate; else B2T_BP_VPT (16 or 32) from the
// environment; else the tuned shape of this problem class; else 32, unless
// the volume's depth leaves 32-voxel columns mostly past its last slice: a
// 16-voxel column costs about 1.1 times a 32-voxel one per slice (measured
// on B200 at 128^3 to 512^3), so 16 when 1.1 x the slices it computes is
// fewer than the 32-voxel shape computes.
int choose_vpt(const b2t_geom3d *g, int32_t dtype)
{
    if (t_vpt_override) return t_vpt_override;
    if (const char *e = std::getenv("B2T_BP_VPT")) return std::atoi(e) == 16 ? 16 : 32;
    {
        std::lock_guard<std::mutex> lock(g_vpt_mutex);
        auto it = g_vpt.find(vpt_key(g, dtype));
        if (it != g_vpt.end()) return it->second;
    }
    const double nz = g->dims.vol_z;
    const double z16 = 16.0 * std::ceil(nz / 16.0), z32 = 32.0 * std::ceil(nz / 32.0);
    return 1.1 * z16 < z32 ? 16 : 32;
}

}  // namespace

b2t_status bp3d_tma(const b2t_geom3d *g, int ker, float out_scale, const void *padded, bool pairs, void *vol,
                    size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s)
{
    const b2t_dims3d &d = g->dims;
    if (pairs != (dtype != B2T_F32))
        return fail(B2T_ERR_INVALID_ARG, "bp3d_tma: 16-bit projections in the pair layout, FP32 as texels");
    const size_t esz = padded_elem_size(dtype, pairs);  // 4 bytes: FP32 texels or 16-bit pairs
    const size_t pu = padded_pu(d.det_u);
    BPTmaLaunch *Lp = new BPTmaLaunch;
    BPTmaLaunch &L = *Lp;
    const uint64_t dims[3] = {pu, d.angles, (uint64_t)d.det_v + 4};
    const uint64_t strides[2] = {pu * esz, pu * esz * d.angles};
    const uint32_t box[3] = {(uint32_t)tile_bu<float>(), 1u, (uint32_t)BPT_CHUNK};
    // a pair is moved as one 32-bit element (a TMA copy does no arithmetic)
    const CUtensorMapDataType tdt = pairs ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    b2t_status st = encode_tensor_map(&L.tmap, tdt, 3, padded, dims, strides, box);
    if (st != B2T_OK) {
        delete Lp;
        return st;
    }
    L.pu = (int)pu;
    L.pv = (long long)pu * d.angles;
    L.proj = static_cast<const char *>(padded) + (2 * L.pv + 2) * esz;
    L.vol = vol;
    L.vol_pitch = (long long)vol_pitch;
    L.nx = d.vol_x; L.ny = d.vol_y; L.nz = d.vol_z;
    L.nu = d.det_u; L.nv = d.det_v; L.na = d.angles;
    L.out_scale = out_scale;
    L.tile_row_bytes = (uint32_t)(tile_bu<float>() * esz);
    const int vpt = choose_vpt(g, dtype);
    const int kker = (ker == B2T_KER_FDK_WEIGHTING) ? B2T_KER_DEFAULT : ker;
    std::vector<BPView> W(d.angles);
    for (uint32_t a = 0; a < d.angles; ++a) bp_view_coeffs(g->kind, ker, g->views[a], g->vol_scale, W[a]);
    auto circular = [&](const BPView &w) { return w.nu.z == 0.0f && (g->kind != B2T_GEOM_CONE || w.den.z == 0.0f); };
    for (uint32_t c0 = 0, cn = 0; c0 < d.angles && st == B2T_OK; c0 += cn) {
        // a launch of circular views holds more of them
        cn = std::min(d.angles - c0, (uint32_t)BPT_MAX_VIEWS_CIRC);
        bool circ = true;
        for (uint32_t i = 0; i < cn && circ; ++i) circ = circular(W[c0 + i]);
        if (!circ) {
            cn = std::min(cn, (uint32_t)BPT_MAX_VIEWS);
            circ = true;
            for (uint32_t i = 0; i < cn && circ; ++i) circ = circular(W[c0 + i]);
        }
        L.a0 = (int)c0;
        L.nviews = (int)cn;
        L.accumulate = (c0 > 0 || mode == B2T_MODE_ADD) ? 1 : 0;
        for (uint32_t i = 0; i < cn; ++i) {
            const BPView &w = W[c0 + i];
            float *f = L.vrec + (circ ? 10 : 12) * i;
            if (circ) {
                const float r[10] = {w.nu.x, w.nu.y, w.nu.w, w.nv.x, w.nv.y, w.nv.z, w.nv.w, w.den.x, w.den.y, w.den.w};
                std::copy(r, r + 10, f);
            } else {
                const float r[12] = {w.nu.x, w.nu.y, w.nu.z, w.nu.w, w.nv.x, w.nv.y,
                                     w.nv.z, w.nv.w, w.den.x, w.den.y, w.den.z, w.den.w};
                std::copy(r, r + 12, f);
            }
        }
        if (dtype == B2T_F32) st = launch_shape<float>(L, g->kind, kker, circ, vpt, d, s);
        else if (dtype == B2T_F16) st = launch_shape<__half>(L, g->kind, kker, circ, vpt, d, s);
        else st = launch_shape<__nv_bfloat16>(L, g->kind, kker, circ, vpt, d, s);
    }
    delete Lp;
    return st;
}

b2t_status bp3d_autotune_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *proj, size_t proj_pitch,
                              void *vol, size_t vol_pitch, int32_t dtype, cudaStream_t s, int32_t *vpt_out)
{
    B2T_TRY(validate3d(g, "b2t_autotune_bp3d"));
    if (!p || !vol || !proj) return fail(B2T_ERR_INVALID_ARG, "b2t_autotune_bp3d: null argument");
    if (!dtype_valid(dtype)) return fail(B2T_ERR_INVALID_ARG, "b2t_autotune_bp3d: bad dtype %d", dtype);
    if (p->voxel_supersample != 1 || p->kernel == B2T_KER_MATCHED_BP || force_simple_bp())
        return fail(B2T_ERR_UNSUPPORTED, "b2t_autotune_bp3d: only the TMA backprojector has launch shapes to choose");
    static const int cands[] = {32, 16};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    B2T_CUDA_TRY(cudaEventCreate(&e0), "autotune event");
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(ce, "autotune event");
    }
    int best = 32;
    float best_ms = 1e30f;
    b2t_status st = B2T_OK;
    for (const int c : cands) {
        t_vpt_override = c;
        // one untimed run, then the best of two timed runs of the whole call
        st = bp3d_impl(g, p, proj, proj_pitch, vol, vol_pitch, dtype, B2T_MODE_SET, s);
        float ms = 1e30f;
        for (int rep = 0; rep < 2 && st == B2T_OK; ++rep) {
            cudaEventRecord(e0, s);
            st = bp3d_impl(g, p, proj, proj_pitch, vol, vol_pitch, dtype, B2T_MODE_SET, s);
            cudaEventRecord(e1, s);
            ce = cudaEventSynchronize(e1);
            if (ce != cudaSuccess) {
                st = cuda_fail(ce, "autotune timing");
                break;
            }
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        t_vpt_override = 0;
        if (st != B2T_OK) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != B2T_OK) return st;
    {
        std::lock_guard<std::mutex> lock(g_vpt_mutex);
        g_vpt[vpt_key(g, dtype)] = best;
    }
    if (vpt_out) *vpt_out = best;
    return B2T_OK;
}

b2t_status encode_tensor_map(CUtensorMap *map, CUtensorMapDataType dtype, uint32_t rank, const void *base,
                             const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
                             CUtensorMapSwizzle swizzle)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return fail(B2T_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t gdim[5];
    cuuint64_t gstr[4];
    cuuint32_t bdim[5], estr[5];
    for (uint32_t k = 0; k < rank; ++k) {
        gdim[k] = dims[k];
        bdim[k] = box[k];
        estr[k] = 1;
        if (k + 1 < rank) gstr[k] = strides_bytes[k];
    }
    CUresult r = encode(map, dtype, rank, const_cast<void *>(base), gdim, gstr, bdim, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(B2T_ERR_CUDA, "cuTensorMapEncodeTiled failed (CUresult %d)", (int)r);
    return B2T_OK;
}

b2t_status bp_path_stats_impl(uint64_t *stats)
{
    unsigned long long v[4] = {0, 0, 0, 0};
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(v, g_bp_path_stats, sizeof(v)), "read BP path statistics");
    const unsigned long long zero[4] = {0, 0, 0, 0};
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_bp_path_stats, zero, sizeof(zero)), "clear BP path statistics");
    for (int k = 0; k < 4; ++k) stats[k] = v[k];
    return B2T_OK;
}

namespace {

// Set by nothing: the flag the self-test waits for.
static __device__ unsigned int g_selftest_flag = 0;

// The bounded waits of the pipelined kernels, run where nothing can end them:
// one warp waits for phase 0 of an mbarrier that expects one arrival and
// never gets it (which 0), or polls a device flag that nothing sets
// (which 1).  Either wait gives up after `limit` cycles, records
// B2T_DEVERR_WAIT_TIMEOUT in the error word and returns, as bp3d_tma_kernel
// and ramp_tc_kernel do on a timeout.  No copy is in flight.
__global__ void __launch_bounds__(32) wait_selftest_kernel(int which, long long limit)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    bool ok;
    if (which == 0) {
        ok = mbar_wait_bounded(&bar, 0u, limit);
    } else {
        const long long t0 = clock64();
        ok = true;
        while (*reinterpret_cast<volatile unsigned int *>(&g_selftest_flag) == 0u) {
            if (clock64() - t0 > limit) {
                ok = false;
                break;
            }
            __nanosleep(1000);
        }
    }
    if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicOr(&g_b2t_device_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
}

}  // namespace

b2t_status selftest_wait_impl(int which, long long limit, cudaStream_t s)
{
    wait_selftest_kernel<<<1, 32, 0, s>>>(which, limit);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "wait self-test launch");
    B2T_CUDA_TRY(cudaStreamSynchronize(s), "wait self-test synchronize");
    uint32_t flags = 0;
    B2T_TRY(device_errors_impl(&flags));
    if (flags & B2T_DEVERR_WAIT_TIMEOUT)
        return fail(B2T_ERR_TIMEOUT, "b2t_selftest_bounded_wait: the wait gave up after %lld cycles", limit);
    return B2T_OK;
}

b2t_status device_errors_impl(uint32_t *flags)
{
    unsigned int v = 0;
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_b2t_device_errors, sizeof(v)), "read device error word");
    const unsigned int zero = 0;
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_b2t_device_errors, &zero, sizeof(zero)), "clear device error word");
    uint32_t w = 0, f = 0;
    B2T_TRY(ramp_tc_errors(&w));
    B2T_TRY(fp_slab_errors(&f));
    *flags = v | w | f;
    return B2T_OK;
}

}  // namespace b2t
