// extern "C" entry points of libb2tomo and the per-thread error state.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "algorithms.h"
#include "arith.h"
#include "batch2d.h"
#include "batch3d.h"
#include "b2t_internal.h"
#include "fdk.h"
#include "filters.h"
#include "proj2d.h"
#include "proj3d.h"

namespace b2t {

static thread_local std::string g_last_error;

constexpr int MAX_POOL_DEVICES = 64;
static std::mutex g_pool_mutex;
static cudaMemPool_t g_pools[MAX_POOL_DEVICES] = {};

cudaMemPool_t scratch_pool(cudaError_t &err)
{
    int dev = 0;
    err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= MAX_POOL_DEVICES) {
        err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        err = cudaMemPoolCreate(&pool, &props);
        if (err != cudaSuccess) return nullptr;
        uint64_t keep = UINT64_MAX;  // never hand freed blocks back on synchronisation
        err = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (err != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return nullptr;
        }
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

void trim_scratch_pools()
{
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    for (int d = 0; d < MAX_POOL_DEVICES; ++d)
        if (g_pools[d]) cudaMemPoolTrimTo(g_pools[d], 0);
}
static std::atomic<unsigned long long> g_launches{0};

void count_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

// Allocations still to go before the armed one fails (0: none armed), and the
// number of device allocations the library holds.
static std::atomic<long long> g_alloc_countdown{0};
static std::atomic<long long> g_live_allocs{0};

bool alloc_injected_failure()
{
    long long c = g_alloc_countdown.load();
    while (c > 0) {
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    }
    return false;
}

void alloc_live(long long delta) { g_live_allocs.fetch_add(delta); }

b2t_status fail(b2t_status st, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

void clear_error() { g_last_error.clear(); }

b2t_status cuda_fail(cudaError_t e, const char *where)
{
    const b2t_status st = (e == cudaErrorMemoryAllocation) ? B2T_ERR_NO_MEMORY : B2T_ERR_CUDA;
    return fail(st, "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
}

}  // namespace b2t

using namespace b2t;

extern "C" {

const char *b2t_last_error(void) { return g_last_error.c_str(); }

int32_t b2t_version(void) { return 100; }

uint64_t b2t_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

b2t_status b2t_set_device(int32_t device)
{
    clear_error();
    B2T_CUDA_TRY(cudaSetDevice(device), "b2t_set_device");
    return B2T_OK;
}

b2t_status b2t_device_errors(uint32_t *flags)
{
    clear_error();
    if (!flags) return fail(B2T_ERR_INVALID_ARG, "b2t_device_errors: null pointer");
    B2T_CUDA_TRY(cudaDeviceSynchronize(), "b2t_device_errors synchronize");
    return device_errors_impl(flags);
}

b2t_status b2t_debug_fail_alloc(int64_t nth, int64_t *pending)
{
    clear_error();
    if (nth < 0) return fail(B2T_ERR_INVALID_ARG, "b2t_debug_fail_alloc: negative count %lld", (long long)nth);
    const long long before = g_alloc_countdown.exchange(nth);
    if (pending) *pending = before;
    return B2T_OK;
}

int64_t b2t_debug_live_allocations(void) { return g_live_allocs.load(); }

b2t_status b2t_selftest_bounded_wait(int32_t which, uint64_t limit_cycles, void *stream)
{
    clear_error();
    if (which != 0 && which != 1) return fail(B2T_ERR_INVALID_ARG, "b2t_selftest_bounded_wait: which must be 0 or 1");
    if (limit_cycles == 0 || limit_cycles > 4000000000ull)
        return fail(B2T_ERR_INVALID_ARG, "b2t_selftest_bounded_wait: limit must be 1..4e9 cycles");
    return selftest_wait_impl(which, (long long)limit_cycles, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_fp_path_stats(uint64_t *stats)
{
    clear_error();
    if (!stats) return fail(B2T_ERR_INVALID_ARG, "b2t_fp_path_stats: null pointer");
    B2T_CUDA_TRY(cudaDeviceSynchronize(), "b2t_fp_path_stats synchronize");
    return fp_path_stats_impl(stats);
}

b2t_status b2t_matched_path_stats(uint64_t *stats)
{
    clear_error();
    if (!stats) return fail(B2T_ERR_INVALID_ARG, "b2t_matched_path_stats: null pointer");
    B2T_CUDA_TRY(cudaDeviceSynchronize(), "b2t_matched_path_stats synchronize");
    return matched_path_stats_impl(stats);
}

b2t_status b2t_bp_path_stats(uint64_t *stats)
{
    clear_error();
    if (!stats) return fail(B2T_ERR_INVALID_ARG, "b2t_bp_path_stats: null pointer");
    B2T_CUDA_TRY(cudaDeviceSynchronize(), "b2t_bp_path_stats synchronize");
    return bp_path_stats_impl(stats);
}

b2t_status b2t_fp3d(const b2t_geom3d *geom, const b2t_params3d *params, const void *vol, size_t vol_pitch,
                    void *proj, size_t proj_pitch, int32_t dtype, int32_t mode, void *stream)
{
    clear_error();
    return fp3d_impl(geom, params, vol, vol_pitch, proj, proj_pitch, dtype, mode,
                     static_cast<cudaStream_t>(stream));
}

b2t_status b2t_bp3d(const b2t_geom3d *geom, const b2t_params3d *params, const void *proj, size_t proj_pitch,
                    void *vol, size_t vol_pitch, int32_t dtype, int32_t mode, void *stream)
{
    clear_error();
    return bp3d_impl(geom, params, proj, proj_pitch, vol, vol_pitch, dtype, mode,
                     static_cast<cudaStream_t>(stream));
}

b2t_status b2t_fp3d_host(const b2t_geom3d *geom, const b2t_params3d *params, const float *vol, float *proj,
                         int32_t mode, const b2t_stream_config *cfg)
{
    clear_error();
    return stream3d_run(0, geom, params, nullptr, 0, 1.0f, vol, proj, mode, cfg);
}

b2t_status b2t_bp3d_host(const b2t_geom3d *geom, const b2t_params3d *params, const float *proj, float *vol,
                         int32_t mode, const b2t_stream_config *cfg)
{
    clear_error();
    return stream3d_run(1, geom, params, nullptr, 0, 1.0f, proj, vol, mode, cfg);
}

b2t_status b2t_fdk_host(const b2t_geom3d *geom, const b2t_filter_config *filter, int32_t short_scan,
                        float output_scale, const float *proj, float *vol, int32_t mode,
                        const b2t_stream_config *cfg)
{
    clear_error();
    return stream3d_run(2, geom, nullptr, filter, short_scan, output_scale, proj, vol, mode, cfg);
}

b2t_status b2t_stream_plan(int32_t op, const b2t_geom3d *geom, const b2t_stream_config *cfg, uint32_t *slab,
                           uint32_t *block)
{
    clear_error();
    return stream3d_plan(op, geom, cfg, slab, block);
}

b2t_status b2t_fp3d_cyl(const b2t_geom3d_cyl *geom, const b2t_params3d *params, const float *vol,
                        size_t vol_pitch, float *proj, size_t proj_pitch, int32_t mode, void *stream)
{
    clear_error();
    return fp3d_cyl_impl(geom, params, vol, vol_pitch, proj, proj_pitch, mode, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_bp3d_cyl(const b2t_geom3d_cyl *geom, const b2t_params3d *params, const float *proj,
                        size_t proj_pitch, float *vol, size_t vol_pitch, int32_t mode, void *stream)
{
    clear_error();
    return bp3d_cyl_impl(geom, params, proj, proj_pitch, vol, vol_pitch, mode, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_fp2d(const b2t_geom2d *geom, uint32_t det_supersample, const float *vol, size_t vol_pitch, float *sino,
                    size_t sino_pitch, int32_t mode, void *stream)
{
    clear_error();
    return fp2d_impl(geom, det_supersample, vol, vol_pitch, sino, sino_pitch, mode, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_bp2d(const b2t_geom2d *geom, uint32_t pixel_supersample, int32_t fbp_weight, const float *sino,
                    size_t sino_pitch, float *vol, size_t vol_pitch, int32_t mode, void *stream)
{
    clear_error();
    return bp2d_impl(geom, pixel_supersample, fbp_weight, sino, sino_pitch, vol, vol_pitch, mode,
                     static_cast<cudaStream_t>(stream));
}

b2t_status b2t_fdk(const b2t_geom3d *geom, const b2t_filter_config *filter, int32_t short_scan, float output_scale, const void *proj,
                   size_t proj_pitch, void *vol, size_t vol_pitch, int32_t dtype, int32_t mode, void *stream)
{
    clear_error();
    return fdk_impl(geom, filter, short_scan, output_scale, proj, proj_pitch, vol, vol_pitch, dtype, mode,
                    static_cast<cudaStream_t>(stream));
}

b2t_status b2t_fdk_weight_filter(const b2t_geom3d *geom, const b2t_filter_config *filter, int32_t short_scan, void *proj,
                                 size_t proj_pitch, int32_t dtype, void *stream)
{
    clear_error();
    return fdk_weight_filter_impl(geom, filter, short_scan, proj, proj_pitch, dtype, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_filter_rows(float *data, size_t nrows, uint32_t n, size_t pitch, const b2t_filter_config *filter,
                           void *stream)
{
    clear_error();
    return filter_rows_impl(data, nrows, n, pitch, filter, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_fbp2d(const b2t_geom2d *geom, const b2t_filter_config *filter, int32_t short_scan, const float *sino,
                     size_t sino_pitch, float *vol, size_t vol_pitch, int32_t mode, void *stream)
{
    clear_error();
    return fbp2d_impl(geom, filter, short_scan, sino, sino_pitch, vol, vol_pitch, mode,
                      static_cast<cudaStream_t>(stream));
}

b2t_status b2t_algo_create3d(int32_t type, const b2t_geom3d *geom, const b2t_params3d *params,
                             const b2t_algo_options *options, b2t_algo **out)
{
    clear_error();
    return algo_create3d_impl(type, geom, params, options, out);
}

b2t_status b2t_algo_create3d_cyl(int32_t type, const b2t_geom3d_cyl *geom, const b2t_params3d *params,
                                 const b2t_algo_options *options, b2t_algo **out)
{
    clear_error();
    return algo_create3d_cyl_impl(type, geom, params, options, out);
}

b2t_status b2t_algo_create2d(int32_t type, const b2t_geom2d *geom, uint32_t det_supersample,
                             uint32_t pixel_supersample, const b2t_algo_options *options, b2t_algo **out)
{
    clear_error();
    return algo_create2d_impl(type, geom, det_supersample, pixel_supersample, options, out);
}

b2t_status b2t_algo_run(b2t_algo *algo, const float *sino, float *vol, int32_t iterations, int32_t use_graph,
                        void *stream)
{
    clear_error();
    return algo_run_impl(algo, sino, vol, iterations, use_graph, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_algo_residual_norm(b2t_algo *algo, const float *sino, const float *vol, double *norm, void *stream)
{
    clear_error();
    return algo_residual_impl(algo, sino, vol, norm, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_algo_set_projection_order(b2t_algo *algo, const int32_t *order, uint32_t n)
{
    clear_error();
    return algo_set_order_impl(algo, order, n);
}

void b2t_algo_abort(b2t_algo *algo) { algo_abort_impl(algo); }

void b2t_algo_destroy(b2t_algo *algo) { algo_destroy_impl(algo); }

b2t_status b2t_vec_op(int32_t op, float *out, const float *a, const float *b, float s, size_t n, void *stream)
{
    clear_error();
    return vec_op_impl(op, out, a, b, s, n, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_dot_f64(const void *a, const void *b, size_t n, int32_t dtype, double *result, void *stream)
{
    clear_error();
    return dot_impl(a, b, n, dtype, result, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_dot_f64_noalloc(const void *a, const void *b, size_t n, int32_t dtype, double *result, void *stream)
{
    clear_error();
    return dot_noalloc_impl(a, b, n, dtype, result, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_batch2d_create(const b2t_problem2d *problems, int32_t n, b2t_batch2d **out)
{
    clear_error();
    return batch2d_create_impl(problems, n, reinterpret_cast<Batch2D **>(out));
}

b2t_status b2t_batch2d_layout(const b2t_batch2d *batch, uint64_t *vol_offsets, uint64_t *sino_offsets,
                              uint64_t *vol_total, uint64_t *sino_total)
{
    clear_error();
    const Batch2D *b = reinterpret_cast<const Batch2D *>(batch);
    if (!b) return fail(B2T_ERR_INVALID_ARG, "b2t_batch2d_layout: null batch");
    for (size_t i = 0; i < b->probs.size(); ++i) {
        if (vol_offsets) vol_offsets[i] = (uint64_t)b->probs[i].vol_off;
        if (sino_offsets) sino_offsets[i] = (uint64_t)b->probs[i].sino_off;
    }
    if (vol_total) *vol_total = b->vol_total;
    if (sino_total) *sino_total = b->sino_total;
    return B2T_OK;
}

b2t_status b2t_batch2d_fp(b2t_batch2d *batch, const float *vols, float *sinos, int32_t mode, void *stream)
{
    clear_error();
    return batch2d_fp_impl(reinterpret_cast<Batch2D *>(batch), vols, sinos, 1.0f, mode,
                           static_cast<cudaStream_t>(stream));
}

b2t_status b2t_batch2d_bp(b2t_batch2d *batch, const float *sinos, float *vols, int32_t mode, void *stream)
{
    clear_error();
    return batch2d_bp_impl(reinterpret_cast<Batch2D *>(batch), sinos, vols, 1.0f, mode,
                           static_cast<cudaStream_t>(stream));
}

b2t_status b2t_algo_create_batch2d(int32_t type, b2t_batch2d *batch, const b2t_algo_options *options,
                                   b2t_algo **out)
{
    clear_error();
    return algo_create_batch2d_impl(type, reinterpret_cast<Batch2D *>(batch), options, out);
}

void b2t_batch2d_destroy(b2t_batch2d *batch)
{
    delete reinterpret_cast<Batch2D *>(batch);
}

b2t_status b2t_batch3d_create(const b2t_problem3d *problems, int32_t n, b2t_batch3d **out)
{
    clear_error();
    return batch3d_create_impl(problems, n, reinterpret_cast<Batch3D **>(out));
}

b2t_status b2t_batch3d_layout(const b2t_batch3d *batch, uint64_t *vol_offsets, uint64_t *proj_offsets,
                              uint64_t *vol_total, uint64_t *proj_total)
{
    clear_error();
    const Batch3D *b = reinterpret_cast<const Batch3D *>(batch);
    if (!b) return fail(B2T_ERR_INVALID_ARG, "b2t_batch3d_layout: null batch");
    for (size_t i = 0; i < b->probs.size(); ++i) {
        if (vol_offsets) vol_offsets[i] = (uint64_t)b->probs[i].vol_off;
        if (proj_offsets) proj_offsets[i] = (uint64_t)b->probs[i].proj_off;
    }
    if (vol_total) *vol_total = b->vol_total;
    if (proj_total) *proj_total = b->proj_total;
    return B2T_OK;
}

b2t_status b2t_batch3d_fp(b2t_batch3d *batch, const float *vols, float *projs, int32_t mode, void *stream)
{
    clear_error();
    return batch3d_fp_impl(reinterpret_cast<Batch3D *>(batch), vols, projs, mode, static_cast<cudaStream_t>(stream));
}

b2t_status b2t_batch3d_bp(b2t_batch3d *batch, const float *projs, float *vols, int32_t mode, void *stream)
{
    clear_error();
    return batch3d_bp_impl(reinterpret_cast<Batch3D *>(batch), projs, vols, mode, false,
                           static_cast<cudaStream_t>(stream));
}

b2t_status b2t_batch3d_matched_bp(b2t_batch3d *batch, const float *projs, float *vols, int32_t mode, void *stream)
{
    clear_error();
    return batch3d_bp_impl(reinterpret_cast<Batch3D *>(batch), projs, vols, mode, true,
                           static_cast<cudaStream_t>(stream));
}

void b2t_batch3d_destroy(b2t_batch3d *batch)
{
    delete reinterpret_cast<Batch3D *>(batch);
}

b2t_status b2t_filter_taps(const b2t_filter_config *filter, uint32_t n, uint32_t n_views, float *out, size_t *count)
{
    clear_error();
    if (!count) return fail(B2T_ERR_INVALID_ARG, "b2t_filter_taps: null count");
    if (!filter || filter->type == B2T_FILTER_NONE)
        return fail(B2T_ERR_INVALID_ARG, "b2t_filter_taps: a filter type with taps is needed");
    FilterTaps ft;
    B2T_TRY(filter_taps(filter, n, n_views, ft));
    const size_t need = ft.g.size();
    if (out) {
        if (*count < need) return fail(B2T_ERR_INVALID_ARG, "b2t_filter_taps: output holds %zu of %zu taps", *count, need);
        std::copy(ft.g.begin(), ft.g.end(), out);
    }
    *count = need;
    return B2T_OK;
}

b2t_status b2t_autotune_fp3d(const b2t_geom3d *geom, const b2t_params3d *params, const void *vol, size_t vol_pitch,
                             void *proj, size_t proj_pitch, int32_t dtype, void *stream, int32_t *vpc)
{
    clear_error();
    return fp3d_autotune_impl(geom, params, vol, vol_pitch, proj, proj_pitch, dtype, static_cast<cudaStream_t>(stream),
                              vpc);
}

b2t_status b2t_autotune_bp3d(const b2t_geom3d *geom, const b2t_params3d *params, const void *proj, size_t proj_pitch,
                             void *vol, size_t vol_pitch, int32_t dtype, void *stream, int32_t *vpt)
{
    clear_error();
    return bp3d_autotune_impl(geom, params, proj, proj_pitch, vol, vol_pitch, dtype, static_cast<cudaStream_t>(stream),
                              vpt);
}

b2t_status b2t_release_cached_memory(void)
{
    clear_error();
    B2T_CUDA_TRY(cudaDeviceSynchronize(), "b2t_release_cached_memory synchronize");
    trim_scratch_pools();
    return B2T_OK;
}

b2t_status b2t_onchip_peak(int32_t which, double *gbs)
{
    clear_error();
    return onchip_peak_impl(which, gbs);
}

}  // extern "C"
