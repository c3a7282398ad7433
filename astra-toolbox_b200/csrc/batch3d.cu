// Batched 3D projection: many parallel-beam and cone-beam problems of
// different sizes, view counts and geometries (parallel3d, parallel3d_vec,
// cone, cone_vec), forward- or back-projected in ONE persistent launch per
// operation.
//
// The reference projects such a set one call at a time (astraCUDA3d::FP / BP,
// include/astra/cuda/3d/mem3d.h:107-113, reaching ConeFP / Par3DFP /
// ConeBP / Par3DBP), each with its own texture set-up and launches, so a set
// of small problems leaves most of the GPU idle.  Here:
//   - a batch is planned once (b2t_batch3d_create): per-view constants of all
//     problems go to the device, volumes and projections live packed in two
//     flat FP32 buffers, and the work is cut into items ordered by
//     decreasing cost;
//   - an FP item is 32 x 8 detector pixels of one view of one problem (one
//     ray per thread); a BP item is a 32 x 8 x 8 voxel block of one problem,
//     summed over all of that problem's views;
//   - the kernels are persistent: every CTA takes the next item from an
//     atomic counter until the list is exhausted;
//   - the texels come straight from the packed buffers, bounds-checked (zero
//     outside), so no padded copies are made;
//   - the exact adjoint of the batched FP (for gradients) walks the same rays
//     and scatters each detector value over the texels its samples read.
// The per-ray and per-voxel arithmetic is the direct-load projectors' own
// (proj3d_dev.cuh): batched results equal b2t_fp3d / b2t_bp3d on the
// direct-load path (B2T_SIMPLE_FP / B2T_SIMPLE_BP) bit for bit, for
// backprojections of up to BP_MAX_VIEWS views (longer scans are summed there
// in chunks, a different rounding).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "b2t_internal.h"
#include "batch3d.h"
#include "proj3d.h"
#include "proj3d_dev.cuh"

namespace b2t {

namespace {

constexpr int B3_TX = 32, B3_TY = 8;  // FP: detector pixels; BP: voxels in x, y
constexpr int B3_ZB = 8;              // BP voxels per thread along z (the direct BP's)

struct Batch3DLaunch {
    const Batch3DProb *probs;
    const FPView *fpv;
    const BPView *bpv;
    const int4 *items;
    int *counter;
    int nitems;
    int accumulate;
    const float *src;  // FP: packed volumes;     BP: packed projections
    float *dst;        // FP: packed projections; BP: packed volumes
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

__global__ void __launch_bounds__(B3_TX *B3_TY) batch3d_fp_kernel(const __grid_constant__ Batch3DLaunch L)
{
    for (;;) {
        const int it = next_item(L.counter);
        if (it >= L.nitems) return;
        const int4 item = L.items[it];  // (problem, view of the problem, tile, marching axis)
        const Batch3DProb &P = L.probs[item.x];
        const FPView &V = L.fpv[P.fpview_off + item.y];
        const int ntu = (P.nu + B3_TX - 1) / B3_TX;
        const int u = (item.z % ntu) * B3_TX + threadIdx.x;
        const int v = (item.z / ntu) * B3_TY + threadIdx.y;
        if (u >= P.nu || v >= P.nv) continue;
        // the view's frame over the volume [z][y][x]: marching axis s,
        // in-plane axes k1 and k2 (the direct FP's frames)
        const long long sx = 1, sy = P.nx, sz = (long long)P.nx * P.ny;
        const int dir = item.w;
        FPChecked Ld;
        Ld.base = L.src + P.vol_off;
        int n0, n1, n2;
        if (dir == 0) {
            Ld.st0 = sx, Ld.st1 = sy, Ld.st2 = sz;
            n0 = P.nx, n1 = P.ny, n2 = P.nz;
        } else if (dir == 1) {
            Ld.st0 = sy, Ld.st1 = sx, Ld.st2 = sz;
            n0 = P.ny, n1 = P.nx, n2 = P.nz;
        } else {
            Ld.st0 = sz, Ld.st1 = sx, Ld.st2 = sy;
            n0 = P.nz, n1 = P.nx, n2 = P.ny;
        }
        Ld.n1 = n1;
        Ld.n2 = n2;
        const float acc = fp3d_ray(Ld, V, u, v, n0, n1, n2, P.nu, P.nv, P.rays, P.fsc[dir][0], P.fsc[dir][1],
                                   P.fsc[dir][2]);
        float *out = L.dst + P.proj_off + ((long long)v * P.na + V.a) * P.nu + u;
        *out = L.accumulate ? *out + acc : acc;
    }
}

// The transpose of one FP ray: its detector value g spread over the texels
// its samples read, with the FP's bilinear weights and scale (atomics: the
// rays of a view overlap).
struct FPScatter {
    float *base;
    long long st0, st1, st2;
    int n1, n2;
    float g, rr, gw;  // detector value, 1 / R^2, scaled value of the sub-ray
    __device__ __forceinline__ void add(int s, int k1, int k2, float w) const
    {
        if (k1 >= 0 && k1 < n1 && k2 >= 0 && k2 < n2)
            atomicAdd(base + (long long)s * st0 + (long long)k1 * st1 + (long long)k2 * st2, w);
    }
    __device__ __forceinline__ void begin(float sc) { gw = g * sc * rr; }
    __device__ __forceinline__ void sample(int s, int k1, float fa, int k2, float fb)
    {
        const float ga = 1.0f - fa, gb = 1.0f - fb;
        add(s, k1, k2, gw * (ga * gb));
        add(s, k1 + 1, k2, gw * (fa * gb));
        add(s, k1, k2 + 1, gw * (ga * fb));
        add(s, k1 + 1, k2 + 1, gw * (fa * fb));
    }
    __device__ __forceinline__ void end(float) {}
};

// vols += A^T projs: the exact adjoint of batch3d_fp_kernel, item for item.
__global__ void __launch_bounds__(B3_TX *B3_TY) batch3d_fpt_kernel(const __grid_constant__ Batch3DLaunch L)
{
    for (;;) {
        const int it = next_item(L.counter);
        if (it >= L.nitems) return;
        const int4 item = L.items[it];  // (problem, view of the problem, tile, marching axis)
        const Batch3DProb &P = L.probs[item.x];
        const FPView &V = L.fpv[P.fpview_off + item.y];
        const int ntu = (P.nu + B3_TX - 1) / B3_TX;
        const int u = (item.z % ntu) * B3_TX + threadIdx.x;
        const int v = (item.z / ntu) * B3_TY + threadIdx.y;
        if (u >= P.nu || v >= P.nv) continue;
        const float g = __ldg(L.src + P.proj_off + ((long long)v * P.na + V.a) * P.nu + u);
        if (g == 0.0f) continue;
        const long long sx = 1, sy = P.nx, sz = (long long)P.nx * P.ny;
        const int dir = item.w;
        FPScatter S;
        S.base = L.dst + P.vol_off;
        int n0;
        if (dir == 0) {
            S.st0 = sx, S.st1 = sy, S.st2 = sz;
            n0 = P.nx, S.n1 = P.ny, S.n2 = P.nz;
        } else if (dir == 1) {
            S.st0 = sy, S.st1 = sx, S.st2 = sz;
            n0 = P.ny, S.n1 = P.nx, S.n2 = P.nz;
        } else {
            S.st0 = sz, S.st1 = sx, S.st2 = sy;
            n0 = P.nz, S.n1 = P.nx, S.n2 = P.ny;
        }
        S.g = g;
        S.rr = 1.0f / (float)(P.rays * P.rays);
        S.gw = 0.0f;
        fp3d_ray_walk(V, u, v, n0, S.n1, S.n2, P.nu, P.nv, P.rays, P.fsc[dir][0], P.fsc[dir][1], P.fsc[dir][2], S);
    }
}

__global__ void __launch_bounds__(B3_TX *B3_TY) batch3d_bp_kernel(const __grid_constant__ Batch3DLaunch L)
{
    for (;;) {
        const int it = next_item(L.counter);
        if (it >= L.nitems) return;
        const int4 item = L.items[it];  // (problem, block x, block y, block z)
        const Batch3DProb &P = L.probs[item.x];
        const int x = item.y * B3_TX + threadIdx.x;
        const int y = item.z * B3_TY + threadIdx.y;
        const int z0 = item.w * B3_ZB;
        if (x >= P.nx || y >= P.ny) continue;
        const float fx = (float)x - 0.5f * (float)P.nx + 0.5f;
        const float fy = (float)y - 0.5f * (float)P.ny + 0.5f;
        const float fz = (float)z0 - 0.5f * (float)P.nz + 0.5f;
        const BPChecked Ld{L.src + P.proj_off, P.nu, P.nv, P.na};
        float acc[B3_ZB];
        if (P.kind == B2T_GEOM_CONE)
            bp3d_column<B2T_GEOM_CONE, B2T_KER_DEFAULT, B3_ZB>(Ld, L.bpv + P.bpview_off, P.na, 0, P.nu, P.nv, fx,
                                                               fy, fz, acc);
        else
            bp3d_column<B2T_GEOM_PAR3D, B2T_KER_DEFAULT, B3_ZB>(Ld, L.bpv + P.bpview_off, P.na, 0, P.nu, P.nv, fx,
                                                                fy, fz, acc);
#pragma unroll
        for (int j = 0; j < B3_ZB; ++j) {
            const int z = z0 + j;
            if (z < P.nz) {
                float *o = L.dst + P.vol_off + ((long long)z * P.ny + y) * P.nx + x;
                const float r = acc[j] * P.bp_scale;
                *o = L.accumulate ? *o + r : r;
            }
        }
    }
}

// Persistent grid: as many CTAs as fit on the GPU at once.
template <typename K> b2t_status persistent_grid(K kern, int threads, int nitems, int &grid)
{
    int dev = 0, sms = 0, per_sm = 0;
    B2T_CUDA_TRY(cudaGetDevice(&dev), "batch3d device");
    B2T_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "batch3d SM count");
    B2T_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0), "batch3d occupancy");
    grid = std::max(1, std::min(nitems, sms * std::max(1, per_sm)));
    return B2T_OK;
}

}  // namespace

Batch3D::~Batch3D()
{
    if (mem) {
        cudaFree(mem);
        alloc_live(-1);
    }
}

b2t_status batch3d_create_impl(const b2t_problem3d *problems, int32_t n, Batch3D **out)
{
    if (!out) return fail(B2T_ERR_INVALID_ARG, "b2t_batch3d_create: null output");
    *out = nullptr;
    if (!problems || n <= 0) return fail(B2T_ERR_INVALID_ARG, "b2t_batch3d_create: no problems");
    Batch3D *b = new Batch3D();
    cudaGetDevice(&b->device);
    b->probs.resize(n);
    long long vo = 0, po = 0;
    int fpv = 0;
    std::vector<FPView> fpviews;
    std::vector<BPView> bpviews;
    struct Keyed {
        double cost;
        int4 item;
    };
    std::vector<Keyed> fpi, bpi;
    for (int i = 0; i < n; ++i) {
        const b2t_problem3d &q = problems[i];
        b2t_status st = validate3d(&q.geom, "b2t_batch3d_create");
        if (st == B2T_OK && (q.det_supersample == 0 || q.det_supersample > 16))
            st = fail(B2T_ERR_INVALID_ARG, "b2t_batch3d_create: problem %d: detector supersampling must be 1..16", i);
        if (st == B2T_OK && q.geom.dims.angles > (1u << 24))
            st = fail(B2T_ERR_INVALID_ARG, "b2t_batch3d_create: problem %d: too many views", i);
        if (st != B2T_OK) {
            delete b;
            return st;
        }
        const b2t_geom3d &g = q.geom;
        const b2t_dims3d &d = g.dims;
        Batch3DProb &P = b->probs[i];
        P.kind = g.kind;
        P.nx = (int)d.vol_x;
        P.ny = (int)d.vol_y;
        P.nz = (int)d.vol_z;
        P.na = (int)d.angles;
        P.nu = (int)d.det_u;
        P.nv = (int)d.det_v;
        P.rays = (int)q.det_supersample;
        const float *vs = g.vol_scale;
        for (int dir = 0; dir < 3; ++dir)
            fp_scale(g.kind, dir, vs, q.det_supersample > 1, q.output_scale, P.fsc[dir][0], P.fsc[dir][1],
                     P.fsc[dir][2]);
        P.bp_scale = q.output_scale * (vs[0] * vs[1] * vs[2]);
        P.fpview_off = fpv;
        P.bpview_off = fpv;
        P.vol_off = vo;
        P.proj_off = po;
        // every problem starts on a 128-byte boundary of the packed buffers
        vo += ((long long)d.vol_x * d.vol_y * d.vol_z + 31) & ~31LL;
        po += ((long long)d.angles * d.det_u * d.det_v + 31) & ~31LL;
        const int ntiles = (P.nu + B3_TX - 1) / B3_TX * ((P.nv + B3_TY - 1) / B3_TY);
        for (int a = 0; a < P.na; ++a) {
            const int dir = dominant_axis(g.kind, g.views[a], d);
            FPView fv;
            fp_view_coeffs(g.kind, g.views[a], d, dir, fv);
            fv.a = a;
            fpviews.push_back(fv);
            BPView bv;
            bp_view_coeffs(g.kind, B2T_KER_DEFAULT, g.views[a], vs, bv);
            bpviews.push_back(bv);
            // an FP ray costs about one sample per slice of its marching axis
            const double cf = (double)(dir == 0 ? P.nx : dir == 1 ? P.ny : P.nz) * P.rays * P.rays;
            for (int t = 0; t < ntiles; ++t) fpi.push_back({cf, make_int4(i, a, t, dir)});
        }
        fpv += P.na;
        // a BP block costs one sample per voxel and view
        const double cb = (double)P.na;
        for (int bz = 0; bz < (P.nz + B3_ZB - 1) / B3_ZB; ++bz)
            for (int by = 0; by < (P.ny + B3_TY - 1) / B3_TY; ++by)
                for (int bx = 0; bx < (P.nx + B3_TX - 1) / B3_TX; ++bx) bpi.push_back({cb, make_int4(i, bx, by, bz)});
    }
    b->vol_total = (size_t)vo;
    b->proj_total = (size_t)po;
    auto by_cost = [](const Keyed &x, const Keyed &y) { return x.cost > y.cost; };
    std::stable_sort(fpi.begin(), fpi.end(), by_cost);
    std::stable_sort(bpi.begin(), bpi.end(), by_cost);
    if (fpi.size() > 0x7fffffff || bpi.size() > 0x7fffffff) {
        delete b;
        return fail(B2T_ERR_UNSUPPORTED, "b2t_batch3d_create: too many work items");
    }
    b->n_fp_items = (int)fpi.size();
    b->n_bp_items = (int)bpi.size();

    // one device allocation for every table
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_probs = 0;
    const size_t o_fpv = align(o_probs + sizeof(Batch3DProb) * n);
    const size_t o_bpv = align(o_fpv + sizeof(FPView) * fpviews.size());
    const size_t o_fpi = align(o_bpv + sizeof(BPView) * bpviews.size());
    const size_t o_bpi = align(o_fpi + sizeof(int4) * fpi.size());
    const size_t o_cnt = align(o_bpi + sizeof(int4) * bpi.size());
    const size_t total = o_cnt + 256;
    if (alloc_injected_failure()) {
        delete b;
        return fail(B2T_ERR_NO_MEMORY, "b2t_batch3d_create: device tables: injected allocation failure");
    }
    cudaError_t e = cudaMalloc(&b->mem, total);
    if (e != cudaSuccess) {
        b->mem = nullptr;
        delete b;
        return cuda_fail(e, "b2t_batch3d_create: device tables");
    }
    alloc_live(1);
    char *base = static_cast<char *>(b->mem);
    b->d_probs = reinterpret_cast<Batch3DProb *>(base + o_probs);
    b->d_fpv = reinterpret_cast<FPView *>(base + o_fpv);
    b->d_bpv = reinterpret_cast<BPView *>(base + o_bpv);
    b->d_fp_items = reinterpret_cast<int4 *>(base + o_fpi);
    b->d_bp_items = reinterpret_cast<int4 *>(base + o_bpi);
    b->d_counters = reinterpret_cast<int *>(base + o_cnt);
    std::vector<int4> fp_items(fpi.size()), bp_items(bpi.size());
    for (size_t k = 0; k < fpi.size(); ++k) fp_items[k] = fpi[k].item;
    for (size_t k = 0; k < bpi.size(); ++k) bp_items[k] = bpi[k].item;
    struct Up {
        void *dst;
        const void *src;
        size_t bytes;
    } ups[] = {{b->d_probs, b->probs.data(), sizeof(Batch3DProb) * n},
               {b->d_fpv, fpviews.data(), sizeof(FPView) * fpviews.size()},
               {b->d_bpv, bpviews.data(), sizeof(BPView) * bpviews.size()},
               {b->d_fp_items, fp_items.data(), sizeof(int4) * fp_items.size()},
               {b->d_bp_items, bp_items.data(), sizeof(int4) * bp_items.size()}};
    for (const Up &u : ups) {
        if (u.bytes == 0) continue;
        e = cudaMemcpy(u.dst, u.src, u.bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            delete b;
            return cuda_fail(e, "b2t_batch3d_create: table upload");
        }
    }
    *out = b;
    return B2T_OK;
}

enum class B3Op { fp, bp, fpt };

static b2t_status batch3d_run(Batch3D *b, B3Op op, const float *src, float *dst, int32_t mode, cudaStream_t s)
{
    const bool is_fp = op == B3Op::fp, rays = op != B3Op::bp;
    if (!b) return fail(B2T_ERR_INVALID_ARG, "b2t_batch3d: null batch");
    if (!src || !dst) return fail(B2T_ERR_INVALID_ARG, "b2t_batch3d: null data pointer");
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "b2t_batch3d: bad mode");
    Batch3DLaunch L;
    L.probs = b->d_probs;
    L.fpv = b->d_fpv;
    L.bpv = b->d_bpv;
    L.items = rays ? b->d_fp_items : b->d_bp_items;
    L.counter = b->d_counters + (rays ? 0 : 1);
    L.nitems = rays ? b->n_fp_items : b->n_bp_items;
    L.accumulate = (mode == B2T_MODE_ADD) ? 1 : 0;
    L.src = src;
    L.dst = dst;
    if (L.nitems == 0) return B2T_OK;
    // the counter restarts at zero for every launch (stream-ordered)
    B2T_CUDA_TRY(cudaMemsetAsync(L.counter, 0, sizeof(int), s), "b2t_batch3d counter reset");
    int grid = 1;
    if (op == B3Op::fpt) {
        // the scatter accumulates: SET starts from zero
        if (mode == B2T_MODE_SET)
            B2T_CUDA_TRY(cudaMemsetAsync(dst, 0, b->vol_total * sizeof(float), s), "b2t_batch3d volume clear");
        B2T_TRY(persistent_grid(batch3d_fpt_kernel, B3_TX * B3_TY, L.nitems, grid));
        batch3d_fpt_kernel<<<grid, dim3(B3_TX, B3_TY), 0, s>>>(L);
    } else if (is_fp) {
        B2T_TRY(persistent_grid(batch3d_fp_kernel, B3_TX * B3_TY, L.nitems, grid));
        batch3d_fp_kernel<<<grid, dim3(B3_TX, B3_TY), 0, s>>>(L);
    } else {
        B2T_TRY(persistent_grid(batch3d_bp_kernel, B3_TX * B3_TY, L.nitems, grid));
        batch3d_bp_kernel<<<grid, dim3(B3_TX, B3_TY), 0, s>>>(L);
    }
    count_launches(1);
    B2T_CUDA_TRY(cudaGetLastError(), "batch3d launch");
    return B2T_OK;
}

b2t_status batch3d_fp_impl(Batch3D *b, const float *vols, float *projs, int32_t mode, cudaStream_t s)
{
    return batch3d_run(b, B3Op::fp, vols, projs, mode, s);
}

b2t_status batch3d_bp_impl(Batch3D *b, const float *projs, float *vols, int32_t mode, bool matched, cudaStream_t s)
{
    return batch3d_run(b, matched ? B3Op::fpt : B3Op::bp, projs, vols, mode, s);
}

}  // namespace b2t
