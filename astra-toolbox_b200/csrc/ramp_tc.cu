// Ram-Lak row filter on the 5th-generation tensor cores (tcgen05).
//
// The filter is a Toeplitz product along every detector row:
//     y_n = sum_k c(n - k) x_k,  c(0) = 1/2, c(odd d) = -2 / (pi d)^2, c(even d != 0) = 0,
// which is what the reference's zero-padded FFT convolution computes
// (cuda/3d/fdk.cu FDK_Filter with the Ram-Lak filter of cuda/2d/fft.cu
// genFilter).  Because c vanishes at even offsets, even outputs only see odd
// inputs and odd outputs only even inputs:
//     y_even = x_even / 2 + E x_odd,   E[i][j] = c(2(i - j) - 1)
//     y_odd  = x_odd  / 2 + O x_even,  O[i][j] = c(2(i - j) + 1)
// Both E and O are dense.  Stacking all detector rows of all views as the M
// dimension (M = det_v * angles) turns each parity into one GEMM of
// M x ceil(nu/2) x ceil(nu/2): half the multiply-adds of the dense nu x nu
// Toeplitz matrix, with no zero taps.
//
// Precision.  The ramp filter cancels strongly on projection data (outputs
// about 100x smaller than inputs), so the work is split in two:
//   - the centre tap and the near taps |d| <= RAMP_TC_BAND carry ~99.7 % of
//     the filter's weight; the split kernel (fdk.cu) sums them exactly in
//     FP32 and writes them to the output;
//   - the far taps run on the tensor cores.  BF16 operands are split in three
//     terms (x = x0 + x1 + x2 with x0 = bf16(x), x1 = bf16(x - x0),
//     x2 = bf16(x - x0 - x1); the taps likewise, from FP64) and the six
//     products at or above 2^-24 relative are accumulated in FP32 in tensor
//     memory: x2 c0 + x1 c1 + x0 c2 + x1 c0 + x0 c1 + x0 c0.
// The tensor cores' FP32 accumulation truncates each step relative to the
// running sum; on the full filter that costs ~1e-5 (127 columns) to ~6e-4
// (1500 columns) relative error, on the far taps alone ~1e-6 to ~3e-6.  The
// epilogue adds the far part to the near part in FP32.
//
// Kernel.  Persistent, one CTA per SM, 6 warps; a tile is 128 rows x bn
// output columns of BOTH parities:
//   warp 0     TMA producer: per 64-wide K block, 3 A tiles (128 x 64) and 3 B
//              tiles (bn x 64), 128-byte swizzled, into a 2-stage ring;
//   warp 1     owns the tensor memory and issues 24 tcgen05.mma per K block
//              into the tile's two FP32 accumulators (one per parity), double
//              buffered across tiles (4 x 128 of the 512 columns);
//   warps 2-5  epilogue: tcgen05.ld of both accumulators, interleave
//              even/odd, transpose through shared memory, add to the near
//              part in full 128-byte row segments.
// Every mbarrier wait is bounded; on a timeout the kernel sets
// B2T_DEVERR_WAIT_TIMEOUT, waits (bounded) for its own loads and MMAs in
// flight, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "b2t_internal.h"
#include "ramp_tc.h"
#include "tc.h"
#include "tma.h"

namespace b2t {

// error word of this translation unit (see b2t_device_errors)
static __device__ unsigned int g_ramp_tc_errors = 0;

namespace {

constexpr int RT_BM = 128;            // rows per tile (TMEM lanes)
constexpr int RT_BK = 64;             // K per stage: one 128-byte swizzle row of BF16
constexpr int RT_STAGES = 2;
constexpr int RT_THREADS = 192;
constexpr uint32_t RT_TMEM_COLS = 512;
constexpr int RT_A_TILE = RT_BM * RT_BK * 2;         // bytes of one A term tile
constexpr int RT_EPI_STRIDE = 33;                    // floats per staged row (conflict-free)
constexpr int RT_EPI_BYTES = 4 * 32 * RT_EPI_STRIDE * 4;
constexpr long long RT_WAIT = 2000000000LL;          // clock cycles, about a second

struct RampTCLaunch {
    CUtensorMap amap;     // split inputs, dims (kh, M, 3, 2)
    CUtensorMap bmap;     // split taps,   dims (kh, nhp, 3, 2)
    void *dst;
    long long dst_row, dst_v;
    long long M;
    long long ntiles;
    int khp, kh, nu, na, nkb, bn, ntn;
    int stage_bytes;
    uint32_t idesc;
};

template <typename T> __device__ __forceinline__ T to_out(float v);
template <> __device__ __forceinline__ float to_out<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_out<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_out<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ float from_out(float v) { return v; }
__device__ __forceinline__ float from_out(__half v) { return __half2float(v); }
__device__ __forceinline__ float from_out(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T>
__global__ void __launch_bounds__(RT_THREADS, 1) ramp_tc_kernel(const __grid_constant__ RampTCLaunch L)
{
    extern __shared__ unsigned char rt_raw[];
    const uint32_t raw = smem_u32(rt_raw);
    unsigned char *sm = rt_raw + (((raw + 1023u) & ~1023u) - raw);
    float *epi = reinterpret_cast<float *>(sm + RT_STAGES * L.stage_bytes);
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + RT_STAGES * L.stage_bytes + RT_EPI_BYTES);
    uint64_t *empty = full + RT_STAGES;
    uint64_t *tfull = empty + RT_STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *drain = tempty + 2;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < RT_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        mbar_fence_init();
        tma_prefetch_map(&L.amap);
        tma_prefetch_map(&L.bmap);
    }
    if (warp == 1) tmem_alloc(tslot, RT_TMEM_COLS);
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = *tslot;
    const int b_bytes = L.bn * RT_BK * 2;
    const int nblk = 2 * L.nkb;  // K blocks of both parities

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t ph = 0;
            long long issued = 0;
            bool ok = true;
            for (long long t = blockIdx.x; ok && t < L.ntiles; t += gridDim.x) {
                if (*abort_flag) break;
                const int nt = (int)(t % L.ntn);
                const int mt = (int)(t / L.ntn);
                for (int blk = 0; blk < nblk; ++blk) {
                    const int p = blk >= L.nkb ? 1 : 0;  // output parity
                    const int kb = blk - p * L.nkb;
                    if (!mbar_wait_bounded(&empty[stage], ph ^ 1u, RT_WAIT)) {
                        ok = false;
                        break;
                    }
                    unsigned char *st = sm + stage * L.stage_bytes;
                    mbar_arrive_expect_tx(&full[stage], (uint32_t)L.stage_bytes);
#pragma unroll
                    for (int l = 0; l < 3; ++l)
                        tma_load_4d(st + l * RT_A_TILE, &L.amap, kb * RT_BK, mt * RT_BM, l, 1 - p, &full[stage]);
#pragma unroll
                    for (int l = 0; l < 3; ++l)
                        tma_load_4d(st + 3 * RT_A_TILE + l * b_bytes, &L.bmap, kb * RT_BK, nt * L.bn, l, p,
                                    &full[stage]);
                    ++issued;
                    if (++stage == RT_STAGES) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok) {
                atomicOr(&g_ramp_tc_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
                *abort_flag = 1;
            }
            // every load issued lands before the CTA may exit
            for (int k = 0; k < RT_STAGES && k < issued; ++k) {
                if (--stage < 0) {
                    stage = RT_STAGES - 1;
                    ph ^= 1u;
                }
                (void)mbar_wait_bounded(&full[stage], ph, RT_WAIT);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0;
            uint32_t ph = 0;
            int buf = 0;
            uint32_t bph = 0;
            bool ok = true;
            const uint32_t sbase = smem_u32(sm);
            for (long long t = blockIdx.x; ok && t < L.ntiles; t += gridDim.x) {
                if (*abort_flag) break;
                if (!mbar_wait_bounded(&tempty[buf], bph ^ 1u, RT_WAIT)) {
                    ok = false;
                    break;
                }
                tc_fence_after_sync();
                for (int blk = 0; blk < nblk; ++blk) {
                    const int p = blk >= L.nkb ? 1 : 0;
                    const int kb = blk - p * L.nkb;
                    const uint32_t d = tmem + (uint32_t)buf * 256u + (uint32_t)p * 128u;
                    if (!mbar_wait_bounded(&full[stage], ph, RT_WAIT)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after_sync();
                    const uint32_t sa = sbase + (uint32_t)(stage * L.stage_bytes);
                    const uint32_t sb = sa + 3u * RT_A_TILE;
#pragma unroll
                    for (int kk = 0; kk < RT_BK / 16; ++kk) {
                        const uint32_t o = (uint32_t)kk * 32u;
                        const uint64_t a0 = umma_desc_sw128(sa + o);
                        const uint64_t a1 = umma_desc_sw128(sa + RT_A_TILE + o);
                        const uint64_t a2 = umma_desc_sw128(sa + 2 * RT_A_TILE + o);
                        const uint64_t b0 = umma_desc_sw128(sb + o);
                        const uint64_t b1 = umma_desc_sw128(sb + b_bytes + o);
                        const uint64_t b2 = umma_desc_sw128(sb + 2 * b_bytes + o);
                        const uint32_t acc = (kb == 0 && kk == 0) ? 0u : 1u;
                        umma_bf16(d, a2, b0, L.idesc, acc);
                        umma_bf16(d, a1, b1, L.idesc, 1u);
                        umma_bf16(d, a0, b2, L.idesc, 1u);
                        umma_bf16(d, a1, b0, L.idesc, 1u);
                        umma_bf16(d, a0, b1, L.idesc, 1u);
                        umma_bf16(d, a0, b0, L.idesc, 1u);
                    }
                    umma_commit(&empty[stage]);  // frees the stage once these MMAs have read it
                    if (++stage == RT_STAGES) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(&tfull[buf]);
                if (++buf == 2) {
                    buf = 0;
                    bph ^= 1u;
                }
            }
            if (!ok) {
                atomicOr(&g_ramp_tc_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
                *abort_flag = 1;
            }
            // every MMA issued completes before tensor memory is freed
            umma_commit(drain);
            (void)mbar_wait_bounded(drain, 0, RT_WAIT);
        }
    } else {
        // epilogue: warp w may read TMEM lanes 32 (w % 4) .. +31
        const int q = warp & 3;
        float *stg = epi + (warp - 2) * 32 * RT_EPI_STRIDE;
        T *dst = static_cast<T *>(L.dst);
        int buf = 0;
        uint32_t bph = 0;
        bool ok = true;
        for (long long t = blockIdx.x; t < L.ntiles; t += gridDim.x) {
            if (*abort_flag) break;
            const int nt = (int)(t % L.ntn);
            const int mt = (int)(t / L.ntn);
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(&tfull[buf], bph, RT_WAIT))) {
                ok = false;
                break;
            }
            tc_fence_after_sync();
            // this lane's row and its output base
            const long long m = (long long)mt * RT_BM + q * 32 + lane;
            const bool row_ok = m < L.M;
            T *orow = dst;
            if (row_ok) {
                const long long v = m / L.na;
                orow = dst + v * L.dst_v + (m - v * L.na) * L.dst_row;
            }
            const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)buf * 256u;
            for (int c = 0; c < L.bn; c += 16) {
                uint32_t re[16], ro[16];
                tmem_ld16(tb + (uint32_t)c, re);
                tmem_ld16(tb + 128u + (uint32_t)c, ro);
                tmem_ld_wait();
                const int i0 = nt * L.bn + c;  // first column of this chunk (per parity)
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    stg[lane * RT_EPI_STRIDE + 2 * j] = __uint_as_float(re[j]);
                    stg[lane * RT_EPI_STRIDE + 2 * j + 1] = __uint_as_float(ro[j]);
                }
                __syncwarp();
                // row r of this warp's 32 rows: 32 consecutive outputs, one per
                // lane.  All 32 near-part loads are issued before any store, so
                // they are in flight together.
                const int n = 2 * i0 + lane;
                const bool col_ok = n < L.nu;
                float near[32];
#pragma unroll
                for (int r = 0; r < 32; ++r) {
                    T *rp = reinterpret_cast<T *>(
                        __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(orow), r));
                    const bool ok = col_ok && (long long)mt * RT_BM + q * 32 + r < L.M;
                    near[r] = ok ? from_out(rp[n]) : 0.0f;
                }
#pragma unroll
                for (int r = 0; r < 32; ++r) {
                    T *rp = reinterpret_cast<T *>(
                        __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(orow), r));
                    const bool ok = col_ok && (long long)mt * RT_BM + q * 32 + r < L.M;
                    if (ok) rp[n] = to_out<T>(near[r] + stg[r * RT_EPI_STRIDE + lane]);
                }
                __syncwarp();
            }
            tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
            if (++buf == 2) {
                buf = 0;
                bph ^= 1u;
            }
        }
        if (!ok && lane == 0) {
            atomicOr(&g_ramp_tc_errors, (unsigned)B2T_DEVERR_WAIT_TIMEOUT);
            *abort_flag = 1;
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after_sync();
        tmem_free(tmem, RT_TMEM_COLS);
    }
}

// Split far taps: b[p][l][i][j] = term l of c(2i + p - (2j + 1 - p)) when both
// the output column 2i + p and the input column 2j + 1 - p lie in [0, nu) and
// they are more than RAMP_TC_BAND apart, else 0.
__global__ void ramp_taps_kernel(__nv_bfloat16 *b, int nu, int nhp, int khp)
{
    const long long per = (long long)nhp * khp;
    const long long total = 2 * per;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(idx / per);
        const long long r = idx - p * per;
        const int i = (int)(r / khp);
        const int j = (int)(r - (long long)i * khp);
        const int n = 2 * i + p, k = 2 * j + 1 - p;
        double c = 0.0;
        if (n < nu && k < nu && abs(n - k) > RAMP_TC_BAND) {
            const double dd = (double)(n - k);  // always odd
            c = -2.0 / (M_PI * M_PI * dd * dd);
        }
        const __nv_bfloat16 t0 = __double2bfloat16(c);
        const double r1 = c - (double)__bfloat162float(t0);
        const __nv_bfloat16 t1 = __double2bfloat16(r1);
        const double r2 = r1 - (double)__bfloat162float(t1);
        const __nv_bfloat16 t2 = __double2bfloat16(r2);
        __nv_bfloat16 *base = b + ((long long)p * 3) * per + r;
        base[0] = t0;
        base[per] = t1;
        base[2 * per] = t2;
    }
}

}  // namespace

bool ramp_tc_enabled()
{
    const char *e = std::getenv("B2T_SIMT_FILTER");
    return !(e && e[0] == '1');
}

bool ramp_tc_plan(uint32_t nu, long long M, RampTCPlan &plan)
{
    if (nu < 127 || M < RT_BM) return false;
    plan.nu = (int)nu;
    plan.M = M;
    plan.kh = (int)((nu + 1) / 2);
    plan.khp = (plan.kh + 15) & ~15;
    const int t = (plan.kh + 127) / 128;
    plan.bn = (((plan.kh + t - 1) / t) + 15) & ~15;
    plan.ntn = (plan.kh + plan.bn - 1) / plan.bn;
    plan.nhp = plan.ntn * plan.bn;
    plan.nkb = (plan.kh + RT_BK - 1) / RT_BK;
    plan.a_elems = (size_t)6 * (size_t)M * plan.khp;
    plan.b_elems = (size_t)6 * (size_t)plan.nhp * plan.khp;
    return true;
}

template <typename T>
static b2t_status launch_ramp(const RampTCLaunch &L, int grid, size_t smem, cudaStream_t s)
{
    auto kern = ramp_tc_kernel<T>;
    B2T_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "ramp filter smem attribute");
    kern<<<grid, RT_THREADS, smem, s>>>(L);
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "ramp filter launch");
    return B2T_OK;
}

b2t_status ramp_tc_filter(const RampTCPlan &P, const __nv_bfloat16 *a, __nv_bfloat16 *taps, void *dst,
                          long long dst_row, long long dst_v, int na, int32_t dtype, cudaStream_t s)
{
    if (!a || !taps || !dst || na <= 0) return fail(B2T_ERR_INVALID_ARG, "ramp filter: bad arguments");
    {
        const long long total = 2LL * P.nhp * P.khp;
        const int blocks = (int)std::min<long long>((total + 255) / 256, 4096);
        ramp_taps_kernel<<<blocks, 256, 0, s>>>(taps, P.nu, P.nhp, P.khp);
        count_launches(1);
        B2T_CUDA_TRY(cudaGetLastError(), "ramp taps launch");
    }
    auto *Lp = new RampTCLaunch();
    RampTCLaunch &L = *Lp;
    const uint64_t pitch = (uint64_t)P.khp * 2;
    {
        const uint64_t dims[4] = {(uint64_t)P.kh, (uint64_t)P.M, 3, 2};
        const uint64_t strides[3] = {pitch, pitch * (uint64_t)P.M, pitch * (uint64_t)P.M * 3};
        const uint32_t box[4] = {(uint32_t)RT_BK, (uint32_t)RT_BM, 1, 1};
        b2t_status st = encode_tensor_map(&L.amap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, a, dims, strides, box,
                                          CU_TENSOR_MAP_SWIZZLE_128B);
        if (st != B2T_OK) {
            delete Lp;
            return st;
        }
    }
    {
        const uint64_t dims[4] = {(uint64_t)P.kh, (uint64_t)P.nhp, 3, 2};
        const uint64_t strides[3] = {pitch, pitch * (uint64_t)P.nhp, pitch * (uint64_t)P.nhp * 3};
        const uint32_t box[4] = {(uint32_t)RT_BK, (uint32_t)P.bn, 1, 1};
        b2t_status st = encode_tensor_map(&L.bmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, taps, dims, strides, box,
                                          CU_TENSOR_MAP_SWIZZLE_128B);
        if (st != B2T_OK) {
            delete Lp;
            return st;
        }
    }
    L.dst = dst;
    L.dst_row = dst_row;
    L.dst_v = dst_v;
    L.M = P.M;
    L.khp = P.khp;
    L.kh = P.kh;
    L.nu = P.nu;
    L.na = na;
    L.nkb = P.nkb;
    L.bn = P.bn;
    L.ntn = P.ntn;
    const long long mtiles = (P.M + RT_BM - 1) / RT_BM;
    L.ntiles = mtiles * P.ntn;
    L.stage_bytes = 3 * RT_A_TILE + 3 * P.bn * RT_BK * 2;
    L.idesc = umma_idesc_bf16_f32(RT_BM, (uint32_t)P.bn);
    const size_t smem = 1024 + (size_t)RT_STAGES * L.stage_bytes + RT_EPI_BYTES + 8 * (2 * RT_STAGES + 5) + 16;
    int dev = 0, sms = 0;
    b2t_status st = B2T_OK;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) st = cuda_fail(e, "ramp filter device query");
    if (st == B2T_OK) {
        const int grid = (int)std::min<long long>(L.ntiles, (long long)sms);
        if (dtype == B2T_F32) st = launch_ramp<float>(L, grid, smem, s);
        else if (dtype == B2T_F16) st = launch_ramp<__half>(L, grid, smem, s);
        else st = launch_ramp<__nv_bfloat16>(L, grid, smem, s);
    }
    delete Lp;
    return st;
}

b2t_status ramp_tc_errors(uint32_t *flags)
{
    unsigned int v = 0;
    B2T_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_ramp_tc_errors, sizeof(v)), "read filter error word");
    const unsigned int zero = 0;
    B2T_CUDA_TRY(cudaMemcpyToSymbol(g_ramp_tc_errors, &zero, sizeof(zero)), "clear filter error word");
    *flags = v;
    return B2T_OK;
}

}  // namespace b2t
