// Voxel-driven 3D backprojection with TMA-staged projection tiles.
//
// Same model as bp3d_kernel (the reference's dev_cone_BP / dev_par3D_BP,
// cuda/3d/cone_bp.cu:55-133, cuda/3d/par3d_bp.cu:55-120): every voxel centre
// is projected onto each view, the projection is sampled bilinearly and
// weighted.  The difference is where the samples come from:
//
//   - a CTA owns a 32 x 8 x 16 voxel block and walks all views of the launch;
//   - for each view, warp 0 projects the block's eight corner voxels, takes
//     the bounding box of their detector coordinates (plus one texel of
//     margin) and issues one cp.async.bulk.tensor load of that tile of the
//     zero-padded projections into a ring of shared-memory stages, signalling
//     an mbarrier; loads run STAGES-1 views ahead of the compute;
//   - all 256 threads then interpolate from shared memory.  For circular
//     geometries (detector v axis along z) the detector u coordinate and the
//     ray-density weight do not depend on z, so each thread computes them once
//     per view and only v changes along its 16-voxel column;
//   - a tile that does not fit the stage (extreme magnification) is read from
//     the padded projections in global memory instead.
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

#include "b2t_internal.h"
#include "proj3d.h"
#include "ramp_tc.h"
#include "tma.h"

namespace b2t {

// error word of this translation unit (see b2t_device_errors)
static __device__ unsigned int g_b2t_device_errors = 0;

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

struct StageInfo {
    int u0, v0, fits, pad;
};

// Projected detector coordinates (texture units) of voxel centre (fx, fy, fz).
template <int KIND>
__device__ __forceinline__ void project(const BPView &W, float fx, float fy, float fz, float &U, float &V)
{
    float nu = fmaf(fz, W.nu.z, fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)));
    float nv = fmaf(fz, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
    if (KIND == B2T_GEOM_CONE) {
        const float dn = fmaf(fz, W.den.z, fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w)));
        const float fr = __frcp_rn(dn);
        U = nu * fr;
        V = nv * fr;
    } else {
        U = nu;
        V = nv;
    }
}

template <typename T, int KIND, int KER, bool CIRC>
__global__ void __launch_bounds__(256, 3) bp3d_tma_kernel(const __grid_constant__ BPTmaLaunch L)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    T *tiles = reinterpret_cast<T *>(smraw);
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw + (size_t)BPT_STAGES * BPT_BV * BPT_BU * sizeof(T));
    uint64_t *empty = full + BPT_STAGES;
    StageInfo *info = reinterpret_cast<StageInfo *>(empty + BPT_STAGES);

    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    // a warp covers 8 x 4 voxels, so its detector footprint in a tile row
    // stays under 32 texels (no shared-memory bank conflicts between lanes
    // of one row); the 8 warps tile the 32 x 8 block
    const int x = blockIdx.x * 32 + (warp & 3) * 8 + (lane & 7);
    const int y = blockIdx.y * 8 + (warp >> 2) * 4 + (lane >> 3);
    const int z0 = blockIdx.z * BPT_Z;
    const bool active = (x < L.nx) && (y < L.ny);
    const float cx = 0.5f - 0.5f * (float)L.nx, cy = 0.5f - 0.5f * (float)L.ny, cz = 0.5f - 0.5f * (float)L.nz;
    const float fx = (float)x + cx, fy = (float)y + cy, fz0 = (float)z0 + cz;
    // voxel-centre extent of this block (for the footprint)
    const float bx0 = (float)(blockIdx.x * 32) + cx, bx1 = (float)(min(L.nx, (int)blockIdx.x * 32 + 32) - 1) + cx;
    const float by0 = (float)(blockIdx.y * 8) + cy, by1 = (float)(min(L.ny, (int)blockIdx.y * 8 + 8) - 1) + cy;
    const float bz0 = fz0, bz1 = (float)(min(L.nz, z0 + BPT_Z) - 1) + cz;

    if (tid == 0) {
        for (int s = 0; s < BPT_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 8);  // one arrival per warp when it is done with the stage
        }
        mbar_fence_init();
        tma_prefetch_map(&L.tmap);
    }
    __syncthreads();

    // warp 0: footprint of view i and its tile load
    auto produce = [&](int i) {
        const int stage = i % BPT_STAGES;
        const BPView &W = L.views[i];
        float U = 0.0f, V = 0.0f;
        if (lane < 8) {
            project<KIND>(W, (lane & 1) ? bx1 : bx0, (lane & 2) ? by1 : by0, (lane & 4) ? bz1 : bz0, U, V);
        }
        float umin = (lane < 8) ? U : 3.0e38f, umax = (lane < 8) ? U : -3.0e38f;
        float vmin = (lane < 8) ? V : 3.0e38f, vmax = (lane < 8) ? V : -3.0e38f;
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, o));
            umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, o));
            vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
            vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        }
        if (lane == 0) {
            // padded texel index of continuous coordinate c is floor(c - 0.5) + 2;
            // one texel of margin on each side for rounding in the consumers
            int fits = 0, u0 = 0, v0 = 0;
            const float lim = 1.0e7f;
            if (umin > -lim && umax < lim && vmin > -lim && vmax < lim) {
                const int ua = (int)floorf(umin - 0.5f) + 2 - 1;
                const int ub = (int)floorf(umax - 0.5f) + 2 + 2;
                const int va = (int)floorf(vmin - 0.5f) + 2 - 1;
                const int vb = (int)floorf(vmax - 0.5f) + 2 + 2;
                u0 = ua & ~7;  // TMA: x * element size must be 16-byte aligned
                v0 = va;
                fits = (ub - u0 < BPT_BU) && (vb - v0 < BPT_BV);
            }
            info[stage] = StageInfo{u0, v0, fits, 0};
            if (fits) {
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(&full[stage], (uint32_t)(BPT_BU * BPT_BV * sizeof(T)));
                tma_load_3d(tiles + (size_t)stage * BPT_BV * BPT_BU, &L.tmap, u0, L.a0 + i, v0, &full[stage]);
            } else {
                mbar_arrive(&full[stage]);
            }
        }
    };

    if (warp == 0) {
        const int n0 = min(BPT_STAGES, L.nviews);
        for (int i = 0; i < n0; ++i) produce(i);
    }

    float acc[BPT_Z];
#pragma unroll
    for (int j = 0; j < BPT_Z; ++j) acc[j] = 0.0f;

    const T *gproj = static_cast<const T *>(L.proj);
    for (int i = 0; i < L.nviews; ++i) {
        const int stage = i % BPT_STAGES;
        const uint32_t parity = (uint32_t)((i / BPT_STAGES) & 1);
        // every wait is bounded: a thread that gives up records the error
        // and leaves; the others then give up on the barriers it no longer
        // arrives on, so the kernel always ends
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[stage], parity, 2000000000LL))) {
            if (lane == 0) atomicOr(&g_b2t_device_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
            return;
        }
        const StageInfo si = info[stage];
        const BPView &W = L.views[i];
        if (active) {
            const T *tile = tiles + (size_t)stage * BPT_BV * BPT_BU;
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
                if (si.fits) {
                    int ku;
                    float fu;
                    split_texel_t(U + 1.0f - (float)si.u0, ku, fu);
                    ku = min(max(ku, 0), BPT_BU - 2);
                    const float vofs = 1.0f - (float)si.v0;
#pragma unroll
                    for (int j = 0; j < BPT_Z; ++j) {
                        int kv;
                        float fv;
                        split_texel_t(fmaf((float)j, dV, Vb) + vofs, kv, fv);
                        kv = min(max(kv, 0), BPT_BV - 2);
                        const T *p = tile + kv * BPT_BU + ku;
                        const float v00 = lds(p), v10 = lds(p + 1);
                        const float v01 = lds(p + BPT_BU), v11 = lds(p + BPT_BU + 1);
                        const float a = fmaf(fu, v10 - v00, v00);
                        const float b = fmaf(fu, v11 - v01, v01);
                        acc[j] = fmaf(fmaf(fv, b - a, a), w, acc[j]);
                    }
                } else {
                    const T *P = gproj + (long long)(L.a0 + i) * L.pu;
                    int ku;
                    float fu;
                    split_texel_t(U - 1.0f, ku, fu);
                    ku = min(max(ku, -2), L.nu);
#pragma unroll
                    for (int j = 0; j < BPT_Z; ++j) {
                        int kv;
                        float fv;
                        split_texel_t(fmaf((float)j, dV, Vb) - 1.0f, kv, fv);
                        kv = min(max(kv, -2), L.nv);
                        const T *p = P + (long long)kv * L.pv + ku;
                        const float v00 = ldgt(p), v10 = ldgt(p + 1);
                        const float v01 = ldgt(p + L.pv), v11 = ldgt(p + L.pv + 1);
                        const float a = fmaf(fu, v10 - v00, v00);
                        const float b = fmaf(fu, v11 - v01, v01);
                        acc[j] = fmaf(fmaf(fv, b - a, a), w, acc[j]);
                    }
                }
            } else {
                // general orientation: everything varies along z
                float nu = fmaf(fz0, W.nu.z, fmaf(fy, W.nu.y, fmaf(fx, W.nu.x, W.nu.w)));
                float nv = fmaf(fz0, W.nv.z, fmaf(fy, W.nv.y, fmaf(fx, W.nv.x, W.nv.w)));
                float dn = fmaf(fz0, W.den.z, fmaf(fy, W.den.y, fmaf(fx, W.den.x, W.den.w)));
#pragma unroll
                for (int j = 0; j < BPT_Z; ++j) {
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
                    float fu, fv;
                    float v00, v10, v01, v11;
                    if (si.fits) {
                        split_texel_t(U + 1.0f - (float)si.u0, ku, fu);
                        split_texel_t(Vc + 1.0f - (float)si.v0, kv, fv);
                        ku = min(max(ku, 0), BPT_BU - 2);
                        kv = min(max(kv, 0), BPT_BV - 2);
                        const T *p = tile + kv * BPT_BU + ku;
                        v00 = lds(p);
                        v10 = lds(p + 1);
                        v01 = lds(p + BPT_BU);
                        v11 = lds(p + BPT_BU + 1);
                    } else {
                        split_texel_t(U - 1.0f, ku, fu);
                        split_texel_t(Vc - 1.0f, kv, fv);
                        ku = min(max(ku, -2), L.nu);
                        kv = min(max(kv, -2), L.nv);
                        const T *p = gproj + (long long)(L.a0 + i) * L.pu + (long long)kv * L.pv + ku;
                        v00 = ldgt(p);
                        v10 = ldgt(p + 1);
                        v01 = ldgt(p + L.pv);
                        v11 = ldgt(p + L.pv + 1);
                    }
                    const float a = fmaf(fu, v10 - v00, v00);
                    const float b = fmaf(fu, v11 - v01, v01);
                    acc[j] = fmaf(fmaf(fv, b - a, a), w, acc[j]);
                    nu += W.nu.z;
                    nv += W.nv.z;
                    dn += W.den.z;
                }
            }
        }
        // release the stage: one arrival per warp once all its lanes are done
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
        // warp 0 refills it for view i + STAGES once every warp has released
        // it; the other warps run ahead on the stages already loaded
        if (warp == 0 && i + BPT_STAGES < L.nviews) {
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(&empty[stage], parity, 2000000000LL))) {
                if (lane == 0) atomicOr(&g_b2t_device_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
                return;
            }
            produce(i + BPT_STAGES);
        }
    }

    if (active) {
        T *out = static_cast<T *>(L.vol);
#pragma unroll
        for (int j = 0; j < BPT_Z; ++j) {
            const int z = z0 + j;
            if (z < L.nz) {
                T *o = out + ((size_t)z * L.ny + y) * L.vol_pitch + x;
                float r = acc[j] * L.out_scale;
                if (L.accumulate) r += lds(o);
                *o = tot<T>(r);
            }
        }
    }
}

template <typename T, int KIND, int KER, bool CIRC>
b2t_status launch_one(const BPTmaLaunch &L, const b2t_dims3d &d, cudaStream_t s)
{
    const size_t smem = (size_t)BPT_STAGES * BPT_BV * BPT_BU * sizeof(T) + BPT_STAGES * (2 * sizeof(uint64_t) + 16) + 64;
    auto kern = bp3d_tma_kernel<T, KIND, KER, CIRC>;
    B2T_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "bp3d_tma smem attribute");
    dim3 grid((d.vol_x + 31) / 32, (d.vol_y + 7) / 8, (d.vol_z + BPT_Z - 1) / BPT_Z);
    kern<<<grid, dim3(32, 8), smem, s>>>(L);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "bp3d_tma launch");
    return B2T_OK;
}

template <typename T>
b2t_status launch_kind(const BPTmaLaunch &L, int kind, int ker, bool circ, const b2t_dims3d &d, cudaStream_t s)
{
    if (kind == B2T_GEOM_PAR3D)
        return circ ? launch_one<T, B2T_GEOM_PAR3D, B2T_KER_DEFAULT, true>(L, d, s)
                    : launch_one<T, B2T_GEOM_PAR3D, B2T_KER_DEFAULT, false>(L, d, s);
    if (ker == B2T_KER_2D_WEIGHTING)
        return circ ? launch_one<T, B2T_GEOM_CONE, B2T_KER_2D_WEIGHTING, true>(L, d, s)
                    : launch_one<T, B2T_GEOM_CONE, B2T_KER_2D_WEIGHTING, false>(L, d, s);
    return circ ? launch_one<T, B2T_GEOM_CONE, B2T_KER_DEFAULT, true>(L, d, s)
                : launch_one<T, B2T_GEOM_CONE, B2T_KER_DEFAULT, false>(L, d, s);
}

}  // namespace

b2t_status bp3d_tma(const b2t_geom3d *g, int ker, float out_scale, const void *padded, void *vol, size_t vol_pitch,
                    int32_t dtype, int32_t mode, cudaStream_t s)
{
    const b2t_dims3d &d = g->dims;
    const size_t esz = dtype_size(dtype);
    const size_t pu = padded_pu(d.det_u);
    BPTmaLaunch *Lp = new BPTmaLaunch;
    BPTmaLaunch &L = *Lp;
    const uint64_t dims[3] = {pu, d.angles, (uint64_t)d.det_v + 4};
    const uint64_t strides[2] = {pu * esz, pu * esz * d.angles};
    const uint32_t box[3] = {(uint32_t)BPT_BU, 1u, (uint32_t)BPT_BV};
    const CUtensorMapDataType tdt = (dtype == B2T_F32) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                    : (dtype == B2T_F16) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                         : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
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
    const int kker = (ker == B2T_KER_FDK_WEIGHTING) ? B2T_KER_DEFAULT : ker;
    for (uint32_t c0 = 0; c0 < d.angles && st == B2T_OK; c0 += BPT_MAX_VIEWS) {
        const uint32_t cn = std::min(d.angles - c0, (uint32_t)BPT_MAX_VIEWS);
        L.a0 = (int)c0;
        L.nviews = (int)cn;
        L.accumulate = (c0 > 0 || mode == B2T_MODE_ADD) ? 1 : 0;
        bool circ = true;
        for (uint32_t i = 0; i < cn; ++i) {
            bp_view_coeffs(g->kind, ker, g->views[c0 + i], g->vol_scale, L.views[i]);
            const BPView &w = L.views[i];
            if (w.nu.z != 0.0f || (g->kind == B2T_GEOM_CONE && w.den.z != 0.0f)) circ = false;
        }
        if (dtype == B2T_F32) st = launch_kind<float>(L, g->kind, kker, circ, d, s);
        else if (dtype == B2T_F16) st = launch_kind<__half>(L, g->kind, kker, circ, d, s);
        else st = launch_kind<__nv_bfloat16>(L, g->kind, kker, circ, d, s);
    }
    delete Lp;
    return st;
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

b2t_status device_errors_impl(uint32_t *flags)
{
    unsigned int v = 0;
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_b2t_device_errors, sizeof(v)), "read device error word");
    const unsigned int zero = 0;
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_b2t_device_errors, &zero, sizeof(zero)), "clear device error word");
    uint32_t w = 0;
    B2T_TRY(ramp_tc_errors(&w));
    *flags = v | w;
    return B2T_OK;
}

}  // namespace b2t
