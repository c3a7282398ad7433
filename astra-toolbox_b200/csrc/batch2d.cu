// Batched 2D projection: many parallel / fan problems of different sizes,
// angle counts and geometries, forward- or back-projected in ONE persistent
// launch per operation.
//
// The reference projects a set of problems one call at a time (cuda/2d
// FP / FanFP / BP / FanBP, include/astra/cuda/2d/par_fp.h:33, fan_fp.h,
// par_bp.h, fan_bp.h:33-44), one or more launches each, so small problems
// leave most of the GPU idle and every call pays its launch and set-up cost.
// Here:
//   - a batch is planned once (b2t_batch2d_create): per-view constants of all
//     problems go to the device, volumes and sinograms live packed in two
//     flat buffers, and the work is cut into items ordered by decreasing cost;
//   - an FP item is one view x 128 detectors of one problem (one ray per
//     thread); a BP item is one 32 x 8 pixel tile of one problem, summed over
//     all of that problem's views (one pixel per thread);
//   - the kernels are persistent: every CTA takes the next item from an
//     atomic counter until the list is exhausted, so long and short items
//     balance across the SMs without a launch per problem.
// The arithmetic per ray and per pixel is the single-problem kernels' own
// (proj2d_dev.cuh): batched forward projections equal per-problem ones bit
// for bit, and so do backprojections of up to 1024 views (the single-problem
// path sums longer scans in chunks of 1024 views, a different rounding).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "b2t_internal.h"
#include "batch2d.h"
#include "proj2d.h"
#include "proj2d_dev.cuh"

namespace b2t {

namespace {

constexpr int BFP_THREADS = 128;  // detectors per FP item
constexpr int BBP_TX = 32, BBP_TY = 8;

struct BatchLaunch {
    const BatchProb *probs;
    const ParFPView *par;
    const b2t_view2d *fan;
    const BPView2D *bp;
    const int4 *items;
    int *counter;
    int nitems;
    int accumulate;
    float scale;
    const float *src;  // FP: packed volumes;   BP: packed sinograms
    float *dst;        // FP: packed sinograms; BP: packed volumes
};

// Next item for this CTA (thread 0 draws it, everyone reads it).
__device__ __forceinline__ int next_item(int *counter)
{
    __shared__ int s_item;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    return s_item;
}

__global__ void __launch_bounds__(BFP_THREADS) batch2d_fp_kernel(const __grid_constant__ BatchLaunch L)
{
    for (;;) {
        const int it = next_item(L.counter);
        if (it >= L.nitems) return;
        const int4 item = L.items[it];
        const BatchProb &P = L.probs[item.x];
        const int a = item.y;
        const int det = item.z + threadIdx.x;
        if (det < P.ndet) {
            const float *vol = L.src + P.vol_off;
            float acc;
            if (P.kind == B2T_GEOM_PAR2D)
                acc = fp2d_par_ray(vol, P.W, P.W, P.H, L.par[P.view_off + a], det, P.det_ss);
            else
                acc = fp2d_fan_ray(vol, P.W, P.W, P.H, L.fan[P.view_off + a], det, P.det_ss, P.out_scale);
            acc *= L.scale;
            float *out = L.dst + P.sino_off + (long long)a * P.ndet + det;
            *out = L.accumulate ? *out + acc : acc;
        }
    }
}

__global__ void __launch_bounds__(BBP_TX * BBP_TY) batch2d_bp_kernel(const __grid_constant__ BatchLaunch L)
{
    for (;;) {
        const int it = next_item(L.counter);
        if (it >= L.nitems) return;
        const int4 item = L.items[it];
        const BatchProb &P = L.probs[item.x];
        const int X = item.y * BBP_TX + threadIdx.x;
        const int Y = item.z * BBP_TY + threadIdx.y;
        if (X < P.W && Y < P.H) {
            const float acc = bp2d_pixel(L.src + P.sino_off, P.ndet, 0, P.nang, L.bp + P.view_off, P.W, P.H, P.ndet,
                                         P.pix_ss, P.kind, 0, X, Y);
            const float r = acc * (P.out_scale / (float)(P.pix_ss * P.pix_ss)) * L.scale;
            float *o = L.dst + P.vol_off + (long long)Y * P.W + X;
            *o = L.accumulate ? *o + r : r;
        }
    }
}

// Persistent grid: as many CTAs as fit on the GPU at once.
template <typename K>
static b2t_status persistent_grid(K kern, int threads, int nitems, int &grid)
{
    int dev = 0, sms = 0, per_sm = 0;
    B2T_CUDA_TRY(cudaGetDevice(&dev), "batch2d device");
    B2T_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "batch2d SM count");
    B2T_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0), "batch2d occupancy");
    grid = std::max(1, std::min(nitems, sms * std::max(1, per_sm)));
    return B2T_OK;
}

}  // namespace

Batch2D::~Batch2D()
{
    if (mem) {
        cudaFree(mem);
        alloc_live(-1);
    }
}

b2t_status batch2d_create_impl(const b2t_problem2d *problems, int32_t n, Batch2D **out)
{
    if (!out) return fail(B2T_ERR_INVALID_ARG, "b2t_batch2d_create: null output");
    *out = nullptr;
    if (!problems || n <= 0) return fail(B2T_ERR_INVALID_ARG, "b2t_batch2d_create: no problems");
    Batch2D *b = new Batch2D();
    cudaGetDevice(&b->device);
    b->probs.resize(n);
    b->views.resize(n);
    long long vo = 0, so = 0;
    int view_off = 0;
    for (int i = 0; i < n; ++i) {
        const b2t_problem2d &q = problems[i];
        b2t_status st = validate2d(&q.geom, "b2t_batch2d_create");
        if (st == B2T_OK && (q.det_supersample == 0 || q.det_supersample > 64 || q.pixel_supersample == 0 ||
                             q.pixel_supersample > 64))
            st = fail(B2T_ERR_INVALID_ARG, "b2t_batch2d_create: problem %d: supersampling must be 1..64", i);
        if (st != B2T_OK) {
            delete b;
            return st;
        }
        const b2t_dims2d &d = q.geom.dims;
        BatchProb &P = b->probs[i];
        P.kind = q.geom.kind;
        P.W = (int)d.vol_width;
        P.H = (int)d.vol_height;
        P.ndet = (int)d.dets;
        P.nang = (int)d.angles;
        P.det_ss = (int)q.det_supersample;
        P.pix_ss = (int)q.pixel_supersample;
        P.pad = 0;
        P.out_scale = q.geom.output_scale;
        P.view_off = view_off;
        P.vol_off = vo;
        P.sino_off = so;
        b->views[i].assign(q.geom.views, q.geom.views + d.angles);
        view_off += (int)d.angles;
        // every problem starts on a 128-byte boundary of the packed buffers
        vo += ((long long)d.vol_width * d.vol_height + 31) & ~31LL;
        so += ((long long)d.angles * d.dets + 31) & ~31LL;
    }
    b->vol_total = (size_t)vo;
    b->sino_total = (size_t)so;

    // per-view constants
    std::vector<ParFPView> par(view_off);
    std::vector<b2t_view2d> fan(view_off);
    std::vector<BPView2D> bp(view_off);
    for (int i = 0; i < n; ++i) {
        const BatchProb &P = b->probs[i];
        b2t_dims2d d{(uint32_t)P.W, (uint32_t)P.H, (uint32_t)P.nang, (uint32_t)P.ndet};
        for (int a = 0; a < P.nang; ++a) {
            const b2t_view2d &w = b->views[i][a];
            fan[P.view_off + a] = w;
            if (P.kind == B2T_GEOM_PAR2D) {
                par_fp_view(w, d, P.out_scale, par[P.view_off + a]);
                par[P.view_off + a].a = a;
            } else {
                par[P.view_off + a] = ParFPView{};
            }
            bp2d_view(P.kind, 0, w, bp[P.view_off + a]);
        }
    }
    // work items, most expensive first: an FP ray costs W (or H) samples per
    // sub-ray, a BP pixel costs one sample per view and sub-pixel
    struct Keyed {
        double cost;
        int4 item;
    };
    std::vector<Keyed> fpi, bpi;
    for (int i = 0; i < n; ++i) {
        const BatchProb &P = b->probs[i];
        const double cf = (double)std::max(P.W, P.H) * P.det_ss;
        for (int a = 0; a < P.nang; ++a)
            for (int d0 = 0; d0 < P.ndet; d0 += BFP_THREADS) fpi.push_back({cf, make_int4(i, a, d0, 0)});
        const double cb = (double)P.nang * P.pix_ss * P.pix_ss;
        for (int ty = 0; ty < (P.H + BBP_TY - 1) / BBP_TY; ++ty)
            for (int tx = 0; tx < (P.W + BBP_TX - 1) / BBP_TX; ++tx) bpi.push_back({cb, make_int4(i, tx, ty, 0)});
    }
    auto by_cost = [](const Keyed &x, const Keyed &y) { return x.cost > y.cost; };
    std::stable_sort(fpi.begin(), fpi.end(), by_cost);
    std::stable_sort(bpi.begin(), bpi.end(), by_cost);
    if (fpi.size() > 0x7fffffff || bpi.size() > 0x7fffffff) {
        delete b;
        return fail(B2T_ERR_UNSUPPORTED, "b2t_batch2d_create: too many work items");
    }
    b->n_fp_items = (int)fpi.size();
    b->n_bp_items = (int)bpi.size();

    // chunk tables of the packed buffers (per-problem reductions)
    std::vector<SegChunk> vch, sch;
    std::vector<int> vfirst(n + 1), sfirst(n + 1);
    for (int i = 0; i < n; ++i) {
        const BatchProb &P = b->probs[i];
        const long long nvol = (long long)P.W * P.H, nsino = (long long)P.nang * P.ndet;
        vfirst[i] = (int)vch.size();
        for (long long o = 0; o < nvol; o += SEG_CHUNK)
            vch.push_back({P.vol_off + o, (int)std::min<long long>(SEG_CHUNK, nvol - o), i});
        sfirst[i] = (int)sch.size();
        for (long long o = 0; o < nsino; o += SEG_CHUNK)
            sch.push_back({P.sino_off + o, (int)std::min<long long>(SEG_CHUNK, nsino - o), i});
    }
    vfirst[n] = (int)vch.size();
    sfirst[n] = (int)sch.size();

    // one device allocation for every table
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_probs = 0;
    const size_t o_par = align(o_probs + sizeof(BatchProb) * n);
    const size_t o_fan = align(o_par + sizeof(ParFPView) * view_off);
    const size_t o_bp = align(o_fan + sizeof(b2t_view2d) * view_off);
    const size_t o_fpi = align(o_bp + sizeof(BPView2D) * view_off);
    const size_t o_bpi = align(o_fpi + sizeof(int4) * fpi.size());
    const size_t o_cnt = align(o_bpi + sizeof(int4) * bpi.size());
    const size_t o_vch = align(o_cnt + 256);
    const size_t o_sch = align(o_vch + sizeof(SegChunk) * vch.size());
    const size_t o_vfi = align(o_sch + sizeof(SegChunk) * sch.size());
    const size_t o_sfi = align(o_vfi + sizeof(int) * (n + 1));
    const size_t total = o_sfi + sizeof(int) * (n + 1);
    if (alloc_injected_failure()) {
        delete b;
        return fail(B2T_ERR_NO_MEMORY, "b2t_batch2d_create: device tables: injected allocation failure");
    }
    cudaError_t e = cudaMalloc(&b->mem, total);
    if (e != cudaSuccess) {
        b->mem = nullptr;
        delete b;
        return cuda_fail(e, "b2t_batch2d_create: device tables");
    }
    alloc_live(1);
    char *base = static_cast<char *>(b->mem);
    b->d_probs = reinterpret_cast<BatchProb *>(base + o_probs);
    b->d_par = reinterpret_cast<ParFPView *>(base + o_par);
    b->d_fan = reinterpret_cast<b2t_view2d *>(base + o_fan);
    b->d_bp = reinterpret_cast<BPView2D *>(base + o_bp);
    b->d_fp_items = reinterpret_cast<int4 *>(base + o_fpi);
    b->d_bp_items = reinterpret_cast<int4 *>(base + o_bpi);
    b->d_counters = reinterpret_cast<int *>(base + o_cnt);
    b->vol_segs = SegTable{reinterpret_cast<SegChunk *>(base + o_vch), reinterpret_cast<int *>(base + o_vfi),
                           (int)vch.size(), n};
    b->sino_segs = SegTable{reinterpret_cast<SegChunk *>(base + o_sch), reinterpret_cast<int *>(base + o_sfi),
                            (int)sch.size(), n};
    std::vector<int4> fp_items(fpi.size()), bp_items(bpi.size());
    for (size_t k = 0; k < fpi.size(); ++k) fp_items[k] = fpi[k].item;
    for (size_t k = 0; k < bpi.size(); ++k) bp_items[k] = bpi[k].item;
    struct Up {
        void *dst;
        const void *src;
        size_t bytes;
    } ups[] = {{b->d_probs, b->probs.data(), sizeof(BatchProb) * n},
               {b->d_par, par.data(), sizeof(ParFPView) * view_off},
               {b->d_fan, fan.data(), sizeof(b2t_view2d) * view_off},
               {b->d_bp, bp.data(), sizeof(BPView2D) * view_off},
               {b->d_fp_items, fp_items.data(), sizeof(int4) * fp_items.size()},
               {b->d_bp_items, bp_items.data(), sizeof(int4) * bp_items.size()},
               {base + o_vch, vch.data(), sizeof(SegChunk) * vch.size()},
               {base + o_sch, sch.data(), sizeof(SegChunk) * sch.size()},
               {base + o_vfi, vfirst.data(), sizeof(int) * (n + 1)},
               {base + o_sfi, sfirst.data(), sizeof(int) * (n + 1)}};
    for (const Up &u : ups) {
        if (u.bytes == 0) continue;
        e = cudaMemcpy(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            delete b;
            return cuda_fail(e, "b2t_batch2d_create: table upload");
        }
    }
    *out = b;
    return B2T_OK;
}

static b2t_status batch2d_run(Batch2D *b, bool is_fp, const float *src, float *dst, float scale, int32_t mode,
                              cudaStream_t s)
{
    if (!b) return fail(B2T_ERR_INVALID_ARG, "b2t_batch2d: null batch");
    if (!src || !dst) return fail(B2T_ERR_INVALID_ARG, "b2t_batch2d: null data pointer");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_batch2d: bad mode");
    BatchLaunch L;
    L.probs = b->d_probs;
    L.par = b->d_par;
    L.fan = b->d_fan;
    L.bp = b->d_bp;
    L.items = is_fp ? b->d_fp_items : b->d_bp_items;
    L.counter = b->d_counters + (is_fp ? 0 : 1);
    L.nitems = is_fp ? b->n_fp_items : b->n_bp_items;
    L.accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
    L.scale = scale;
    L.src = src;
    L.dst = dst;
    if (L.nitems == 0) return B2T_OK;
    // the counter restarts at zero for every launch (stream-ordered, so a
    // captured CUDA graph replays it too)
    B2T_CUDA_TRY(cudaMemsetAsync(L.counter, 0, sizeof(int), s), "b2t_batch2d counter reset");
    int grid = 1;
    if (is_fp) {
        B2T_TRY(persistent_grid(batch2d_fp_kernel, BFP_THREADS, L.nitems, grid));
        batch2d_fp_kernel<<<grid, BFP_THREADS, 0, s>>>(L);
    } else {
        B2T_TRY(persistent_grid(batch2d_bp_kernel, BBP_TX * BBP_TY, L.nitems, grid));
        batch2d_bp_kernel<<<grid, dim3(BBP_TX, BBP_TY), 0, s>>>(L);
    }
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), is_fp ? "batch2d FP launch" : "batch2d BP launch");
    return B2T_OK;
}

b2t_status batch2d_fp_impl(Batch2D *b, const float *vols, float *sinos, float scale, int32_t mode, cudaStream_t s)
{
    return batch2d_run(b, true, vols, sinos, scale, mode, s);
}

b2t_status batch2d_bp_impl(Batch2D *b, const float *sinos, float *vols, float scale, int32_t mode, cudaStream_t s)
{
    return batch2d_run(b, false, sinos, vols, scale, mode, s);
}

}  // namespace b2t
