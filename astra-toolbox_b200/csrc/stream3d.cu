// Streamed 3D projection of host-resident data: volumes and projections
// larger than the device memory budget.
//
// The reference's CompositeGeometryManager (src/CompositeGeometryManager.cpp:
// job splitting :218-379, execution :1115-1280, 1409-1477) splits volume and
// projections into blocks that fit the GPU and copies each block to the
// device per job.  Here:
//   - the volume is cut into z-slabs and the projections into angle blocks;
//     a slab's geometry is the full geometry with the views shifted along z
//     (views are volume-centred, in voxel units), an angle block's is the
//     subset of views; FP and BP are linear, so the FP of the whole volume is
//     the sum of the slabs' FPs (ADD mode), and a slab's BP is the full BP
//     restricted to its voxels (the sum over angle blocks);
//   - FP jobs are angle blocks (each accumulates over the slabs), BP and FDK
//     jobs are slabs (each accumulates over the angle blocks); a job's inputs
//     stream through two device buffers on a copy stream while the compute
//     stream works on the other, and its output is copied back on a third
//     stream while the next job computes; an input that fits whole is copied
//     once per device and kept;
//   - FDK weights and filters each angle block with the weights of the whole
//     scan (its angle count and Parker range);
//   - jobs are spread over the listed GPUs, one host thread each, writing
//     disjoint parts of the output (no exchange between GPUs).
// Host buffers may be pageable; pinned host memory lets the copies overlap
// the compute.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "b2t_internal.h"
#include "fdk.h"
#include "proj3d.h"

namespace b2t {

namespace {

enum class Op { fp, bp, fdk };

struct Req {
    Op op;
    const b2t_geom3d *g;
    b2t_params3d params;
    const b2t_filter_config *filter;
    int32_t short_scan;
    float fdk_scale;
    const float *in;   // host input: volume (FP) or projections (BP, FDK)
    float *out;        // host output
    int32_t mode;
    uint32_t slab, block;  // z-slab thickness and angle block size
};

// A device buffer of a streamed call, from the library's stream-ordered
// memory pool (cached between calls, so repeated calls map no memory),
// allocated and released on the worker's compute stream.
struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf()
    {
        if (p) {
            cudaFreeAsync(p, s);
            alloc_live(-1);
        }
    }
    b2t_status alloc(size_t bytes, cudaStream_t st, const char *what)
    {
        if (alloc_injected_failure()) return fail(B2T_ERR_NO_MEMORY, "%s: injected allocation failure", what);
        cudaError_t e = cudaSuccess;
        cudaMemPool_t pool = scratch_pool(e);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, st);
        if (e != cudaSuccess) {
            p = nullptr;
            (void)cudaGetLastError();
            return cuda_fail(e, what);
        }
        alloc_live(1);
        s = st;
        return B2T_OK;
    }
    float *f() const { return static_cast<float *>(p); }
};

struct Stream {
    cudaStream_t s = nullptr;
    ~Stream()
    {
        if (s) cudaStreamDestroy(s);
    }
};
struct Event {
    cudaEvent_t e = nullptr;
    ~Event()
    {
        if (e) cudaEventDestroy(e);
    }
};
// Drains a worker's three streams when it leaves, on every path, before its
// buffers go back to the pool (declared after the buffers, so destroyed first).
struct Drain {
    Stream *st[3];
    ~Drain()
    {
        for (Stream *x : st)
            if (x->s) cudaStreamSynchronize(x->s);
    }
};

// The geometry of views [a0, a0 + n) and z-slab [z0, z0 + nz) of g.
struct SubGeom {
    b2t_geom3d g;
    std::vector<b2t_view3d> views;
    void set(const b2t_geom3d &full, uint32_t a0, uint32_t n, uint32_t z0, uint32_t nz)
    {
        g = full;
        views.assign(full.views + a0, full.views + a0 + n);
        // slab centre relative to the volume centre, in voxels
        const double dz = (double)z0 + 0.5 * nz - 0.5 * full.dims.vol_z;
        for (b2t_view3d &v : views) {
            if (full.kind == B2T_GEOM_CONE) v.src[2] -= dz;  // parallel: src is the ray direction
            v.det_s[2] -= dz;
        }
        g.views = views.data();
        g.dims.angles = n;
        g.dims.vol_z = nz;
    }
};

// host <-> device copies of an angle block [a0, a0 + n) of the projections
// [v][angle][u] (rows of n * nu floats, pitch na * nu) and of a slab
b2t_status copy_block(float *dst, const float *src, const b2t_dims3d &d, uint32_t a0, uint32_t n, bool to_device,
                      cudaStream_t s)
{
    const size_t row = (size_t)n * d.det_u * sizeof(float), full = (size_t)d.angles * d.det_u * sizeof(float);
    const size_t off = (size_t)a0 * d.det_u;
    if (to_device)
        B2T_CUDA_TRY(cudaMemcpy2DAsync(dst, row, src + off, full, row, d.det_v, cudaMemcpyHostToDevice, s),
                     "projection block upload");
    else
        B2T_CUDA_TRY(cudaMemcpy2DAsync(dst + off, full, src, row, row, d.det_v, cudaMemcpyDeviceToHost, s),
                     "projection block download");
    return B2T_OK;
}

b2t_status copy_slab(float *dst, const float *src, const b2t_dims3d &d, uint32_t z0, uint32_t nz, bool to_device,
                     cudaStream_t s)
{
    const size_t plane = (size_t)d.vol_x * d.vol_y;
    if (to_device)
        B2T_CUDA_TRY(cudaMemcpyAsync(dst, src + z0 * plane, plane * nz * sizeof(float), cudaMemcpyHostToDevice, s),
                     "volume slab upload");
    else
        B2T_CUDA_TRY(cudaMemcpyAsync(dst + z0 * plane, src, plane * nz * sizeof(float), cudaMemcpyDeviceToHost, s),
                     "volume slab download");
    return B2T_OK;
}

// One GPU's share of the jobs (job j = angle block j for FP, slab j for
// BP / FDK).
// The angle blocks of a streamed call, (first view, count): blocks of at
// most `step` views, balanced, and, when the views are split at all, one
// block of at most 16 views at the end of the pipeline whose transfer no
// compute hides: last for the FP (its final download), first for the BP and
// FDK (their first upload).
std::vector<std::pair<uint32_t, uint32_t>> angle_blocks(uint32_t n, uint32_t step, bool small_last)
{
    std::vector<std::pair<uint32_t, uint32_t>> r;
    const uint32_t edge = n > step ? std::min<uint32_t>(16, step) : 0;
    const uint32_t rest = n - edge;
    const uint32_t nb = (rest + step - 1) / step;
    uint32_t a = 0;
    if (!small_last && edge) {
        r.push_back({0, edge});
        a = edge;
    }
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t len = rest / nb + (b < rest % nb ? 1u : 0u);
        r.push_back({a, len});
        a += len;
    }
    if (small_last && edge) r.push_back({a, edge});
    return r;
}

b2t_status run_worker(const Req &R, int device, const std::vector<uint32_t> &jobs)
{
    B2T_CUDA_TRY(cudaSetDevice(device), "stream worker device");
    const b2t_geom3d &G = *R.g;
    const b2t_dims3d &d = G.dims;
    const bool fp = R.op == Op::fp;
    // inner chunks (the streamed input) and outer jobs (the accumulated output)
    const uint32_t in_n = fp ? d.vol_z : d.angles, in_step = fp ? R.slab : R.block;
    const uint32_t out_step = fp ? R.block : R.slab;
    const uint32_t out_n = fp ? d.angles : d.vol_z;
    const std::vector<std::pair<uint32_t, uint32_t>> ablocks = angle_blocks(d.angles, R.block, fp);
    const uint32_t nin = fp ? (in_n + in_step - 1) / in_step : (uint32_t)ablocks.size();
    const size_t in_elems = fp ? (size_t)d.vol_x * d.vol_y * in_step : (size_t)d.det_u * d.det_v * in_step;
    const size_t out_elems = fp ? (size_t)d.det_u * d.det_v * out_step : (size_t)d.vol_x * d.vol_y * out_step;
    const bool resident = nin == 1;  // the whole input fits: copy it once

    Stream cs, hs, os;
    for (Stream *st : {&cs, &hs, &os})
        B2T_CUDA_TRY(cudaStreamCreateWithFlags(&st->s, cudaStreamNonBlocking), "stream create");
    DevBuf inb[2], outb[2], padded;
    Drain drain{{&cs, &hs, &os}};
    Event in_ready[2], in_free[2], out_done[2], out_copied[2], allocated;
    for (int k = 0; k < 2; ++k) {
        if (k == 0 || !resident) B2T_TRY(inb[k].alloc(in_elems * sizeof(float), cs.s, "streamed input buffer"));
        B2T_TRY(outb[k].alloc(out_elems * sizeof(float), cs.s, "streamed output buffer"));
    }
    if (R.op == Op::fdk) {
        b2t_dims3d db = d;
        db.angles = R.block;
        B2T_TRY(padded.alloc(padded_proj_bytes(db, B2T_F32, false), cs.s, "streamed FDK filtered block"));
    }
    // the copy streams touch the buffers only after their allocation
    B2T_CUDA_TRY(cudaEventCreateWithFlags(&allocated.e, cudaEventDisableTiming), "event create");
    B2T_CUDA_TRY(cudaEventRecord(allocated.e, cs.s), "event record");
    B2T_CUDA_TRY(cudaStreamWaitEvent(hs.s, allocated.e, 0), "wait");
    B2T_CUDA_TRY(cudaStreamWaitEvent(os.s, allocated.e, 0), "wait");
    for (int k = 0; k < 2; ++k) {
        for (Event *e : {&in_ready[k], &in_free[k], &out_done[k], &out_copied[k]})
            B2T_CUDA_TRY(cudaEventCreateWithFlags(&e->e, cudaEventDisableTiming), "event create");
        B2T_CUDA_TRY(cudaEventRecord(in_free[k].e, cs.s), "event record");
        B2T_CUDA_TRY(cudaEventRecord(out_copied[k].e, os.s), "event record");
    }
    // input chunk c: a z-slab of the FP, an angle block of the BP / FDK
    auto in_chunk = [&](uint32_t c, uint32_t &c0, uint32_t &cn) {
        if (fp) {
            c0 = c * in_step;
            cn = std::min(in_step, in_n - c0);
        } else {
            c0 = ablocks[c].first;
            cn = ablocks[c].second;
        }
    };
    auto upload = [&](uint32_t c, int buf) -> b2t_status {
        uint32_t c0, cn;
        in_chunk(c, c0, cn);
        B2T_CUDA_TRY(cudaStreamWaitEvent(hs.s, in_free[buf].e, 0), "wait");
        if (fp) B2T_TRY(copy_slab(inb[buf].f(), R.in, d, c0, cn, true, hs.s));
        else B2T_TRY(copy_block(inb[buf].f(), R.in, d, c0, cn, true, hs.s));
        B2T_CUDA_TRY(cudaEventRecord(in_ready[buf].e, hs.s), "event record");
        return B2T_OK;
    };
    if (resident) B2T_TRY(upload(0, 0));
    // a resident FP input (the whole volume in one slab) is laid out in
    // cells once; every angle block projects from them
    FPCells cells;
    bool have_cells = false;
    if (fp && resident && R.params.kernel == B2T_KER_DEFAULT && !force_simple_fp()) {
        bool need[3] = {false, false, false};
        for (uint32_t a = 0; a < d.angles; ++a) need[dominant_axis(G.kind, G.views[a], d)] = true;
        B2T_CUDA_TRY(cudaStreamWaitEvent(cs.s, in_ready[0].e, 0), "wait");
        const b2t_status bs = fp3d_cells_build(&G, &R.params, inb[0].f(), 0, B2T_F32, need, cs.s, cells);
        if (bs == B2T_OK) have_cells = true;
        else if (bs == B2T_ERR_NO_MEMORY) clear_error();  // project block by block instead
        else return bs;
    }

    // The BP's and FDK's last angle block of a job runs in z-chunks, each
    // downloaded as soon as it is final, so that the volume's download
    // overlaps the last block's compute instead of following it (projections
    // padded, or weighted and filtered, once).
    const bool split_tail = (R.op == Op::bp && R.params.kernel == B2T_KER_DEFAULT &&
                             R.params.voxel_supersample >= 1 && R.params.voxel_supersample <= 16) ||
                            (R.op == Op::fdk && R.params.voxel_supersample >= 1 &&
                             R.params.voxel_supersample <= 16);
    DevBuf tailpad;
    if (split_tail && R.op == Op::bp) {
        b2t_dims3d db = d;
        db.angles = R.block;
        B2T_TRY(tailpad.alloc(padded_proj_bytes(db, B2T_F32, false), cs.s, "streamed BP padded block"));
    }
    std::vector<Event> tail_ev(8);
    for (Event &e : tail_ev) B2T_CUDA_TRY(cudaEventCreateWithFlags(&e.e, cudaEventDisableTiming), "event create");
    const size_t plane = (size_t)d.vol_x * d.vol_y;
    SubGeom sub;
    // BP of views [c0, c0 + cn) from a padded block into slab [o0, o0 + on)
    // of obuf in z-chunks, each downloaded once computed
    auto bp_tail = [&](const void *pad, const b2t_params3d &p, uint32_t c0, uint32_t cn, uint32_t o0, uint32_t on,
                       float *obuf, int32_t mode) -> b2t_status {
        const uint32_t nch = std::min<uint32_t>((uint32_t)tail_ev.size(), std::max<uint32_t>(1, on / 16));
        const uint32_t zc = (on + nch - 1) / nch;
        for (uint32_t k = 0; k * zc < on; ++k) {
            const uint32_t z0 = o0 + k * zc, nz = std::min(zc, o0 + on - z0);
            sub.set(G, c0, cn, z0, nz);
            float *part = obuf + (size_t)(z0 - o0) * plane;
            B2T_TRY(bp3d_from_padded(&sub.g, &p, pad, part, 0, B2T_F32, mode, cs.s));
            B2T_CUDA_TRY(cudaEventRecord(tail_ev[k].e, cs.s), "event record");
            B2T_CUDA_TRY(cudaStreamWaitEvent(os.s, tail_ev[k].e, 0), "wait");
            B2T_TRY(copy_slab(R.out, part, d, z0, nz, false, os.s));
        }
        return B2T_OK;
    };

    for (size_t jn = 0; jn < jobs.size(); ++jn) {
        const uint32_t j = jobs[jn];
        uint32_t o0 = j * out_step, on = std::min(out_step, out_n - std::min(o0, out_n));
        if (fp) {
            o0 = ablocks[j].first;
            on = ablocks[j].second;
        }
        const int ob = (int)(jn & 1);
        float *obuf = outb[ob].f();
        // the output buffer's previous download must be complete
        B2T_CUDA_TRY(cudaStreamWaitEvent(cs.s, out_copied[ob].e, 0), "wait");
        bool first = R.mode == B2T_MODE_SET;
        if (!first) {  // ADD: start from the host's current values
            B2T_CUDA_TRY(cudaStreamWaitEvent(hs.s, out_copied[ob].e, 0), "wait");
            if (fp) B2T_TRY(copy_block(obuf, R.out, d, o0, on, true, hs.s));
            else B2T_TRY(copy_slab(obuf, R.out, d, o0, on, true, hs.s));
            Event got;
            B2T_CUDA_TRY(cudaEventCreateWithFlags(&got.e, cudaEventDisableTiming), "event create");
            B2T_CUDA_TRY(cudaEventRecord(got.e, hs.s), "event record");
            B2T_CUDA_TRY(cudaStreamWaitEvent(cs.s, got.e, 0), "wait");
        }
        if (!resident) B2T_TRY(upload(0, 0));
        bool downloaded = false;
        for (uint32_t c = 0; c < nin; ++c) {
            const int ib = resident ? 0 : (int)(c & 1);
            if (!resident && c + 1 < nin) B2T_TRY(upload(c + 1, (int)((c + 1) & 1)));
            B2T_CUDA_TRY(cudaStreamWaitEvent(cs.s, in_ready[ib].e, 0), "wait");
            uint32_t c0, cn;
            in_chunk(c, c0, cn);
            const int32_t mode = first ? B2T_MODE_SET : B2T_MODE_ADD;
            first = false;
            if (fp) {
                sub.set(G, o0, on, c0, cn);
                if (have_cells) B2T_TRY(fp3d_cells_project(&sub.g, &R.params, cells, obuf, 0, mode, cs.s));
                else B2T_TRY(fp3d_impl(&sub.g, &R.params, inb[ib].f(), 0, obuf, 0, B2T_F32, mode, cs.s));
            } else if (R.op == Op::bp && split_tail && c + 1 == nin) {
                sub.set(G, c0, cn, o0, on);
                B2T_TRY(pad_projections_impl(inb[ib].f(), d.det_u, sub.g.dims, tailpad.p, B2T_F32, false, cs.s));
                B2T_TRY(bp_tail(tailpad.p, R.params, c0, cn, o0, on, obuf, mode));
                downloaded = true;
            } else if (R.op == Op::bp) {
                sub.set(G, c0, cn, o0, on);
                B2T_TRY(bp3d_impl(&sub.g, &R.params, inb[ib].f(), 0, obuf, 0, B2T_F32, mode, cs.s));
            } else {
                sub.set(G, c0, cn, o0, on);
                const size_t pbytes = padded_proj_bytes(sub.g.dims, B2T_F32, false);
                B2T_CUDA_TRY(cudaMemsetAsync(padded.p, 0, pbytes, cs.s), "FDK block clear");
                const long long pu = (long long)padded_pu(d.det_u), pv = pu * cn;
                float *interior = padded.f() + 2 * pv + 2;
                B2T_TRY(fdk_weight_filter_views(&G, c0, cn, R.filter, R.short_scan, inb[ib].f(), d.det_u, interior,
                                                pu, pv, cs.s));
                b2t_params3d p = R.params;
                p.kernel = B2T_KER_FDK_WEIGHTING;
                p.output_scale = R.fdk_scale;
                if (split_tail && c + 1 == nin) {
                    B2T_TRY(bp_tail(padded.p, p, c0, cn, o0, on, obuf, mode));
                    downloaded = true;
                } else {
                    B2T_TRY(bp3d_from_padded(&sub.g, &p, padded.p, obuf, 0, B2T_F32, mode, cs.s));
                }
            }
            if (!resident) B2T_CUDA_TRY(cudaEventRecord(in_free[ib].e, cs.s), "event record");
        }
        // download this job's output while the next job computes
        B2T_CUDA_TRY(cudaEventRecord(out_done[ob].e, cs.s), "event record");
        B2T_CUDA_TRY(cudaStreamWaitEvent(os.s, out_done[ob].e, 0), "wait");
        if (fp) B2T_TRY(copy_block(R.out, obuf, d, o0, on, false, os.s));
        else if (!downloaded) B2T_TRY(copy_slab(R.out, obuf, d, o0, on, false, os.s));
        B2T_CUDA_TRY(cudaEventRecord(out_copied[ob].e, os.s), "event record");
    }
    for (Stream *st : {&cs, &hs, &os}) B2T_CUDA_TRY(cudaStreamSynchronize(st->s), "stream worker synchronize");
    return B2T_OK;
}

// Devices and chunk sizes of a streamed call: the budget per device is the
// configured bytes, else the free memory of the first device less 2 GiB.
// Bytes per streamed element: FP, the slab double-buffered plus the FP's cell
// scratch (two marching directions, 16 B each) and the output block
// double-buffered; BP, the block double-buffered plus its padded copy, FDK
// adding the filter's operand scratch (6 x 2 B per value) and the filtered
// block, and the slab double-buffered.  The streamed input takes at most half
// the budget, the accumulated output the rest.
b2t_status stream3d_plan_impl(int32_t op, const b2t_geom3d *g, const b2t_stream_config *cfg, const char *who,
                              std::vector<int> &devs, uint32_t &slab, uint32_t &block)
{
    devs.clear();
    if (cfg && cfg->n_devices > 0) {
        if (!cfg->devices) return fail(B2T_ERR_INVALID_ARG, "%s: null device list", who);
        devs.assign(cfg->devices, cfg->devices + cfg->n_devices);
    } else {
        int cur = 0;
        B2T_CUDA_TRY(cudaGetDevice(&cur), "current device");
        devs.push_back(cur);
    }
    size_t budget = cfg ? cfg->device_bytes : 0;
    if (budget == 0) {
        int cur = 0;
        B2T_CUDA_TRY(cudaGetDevice(&cur), "current device");
        B2T_CUDA_TRY(cudaSetDevice(devs[0]), "budget device");
        size_t fr = 0, tot = 0;
        const cudaError_t e = cudaMemGetInfo(&fr, &tot);
        cudaSetDevice(cur);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
        budget = fr > ((size_t)2 << 30) ? fr - ((size_t)2 << 30) : fr / 2;
    }
    const b2t_dims3d &d = g->dims;
    const double plane = (double)d.vol_x * d.vol_y, view = (double)d.det_u * d.det_v;
    const double vox_in = 8.0 + 32.0, pix_out = 8.0;                                   // FP
    const double pix_in = op == 2 ? 8.0 + 4.2 + 12.0 + 4.2 : 8.0 + 4.2, vox_out = 8.0;  // BP / FDK
    const double B = (double)budget;
    double z, a;
    if (op == 0) {
        z = std::min((double)d.vol_z, std::floor(0.5 * B / (plane * vox_in)));
        if (z < 1) return fail(B2T_ERR_NO_MEMORY, "%s: one volume slice does not fit %zu bytes", who, budget);
        a = std::min((double)d.angles, std::floor((B - z * plane * vox_in) / (view * pix_out)));
        if (a < 1) return fail(B2T_ERR_NO_MEMORY, "%s: one projection does not fit %zu bytes", who, budget);
    } else {
        a = std::min((double)d.angles, std::floor(0.5 * B / (view * pix_in)));
        if (a < 1) return fail(B2T_ERR_NO_MEMORY, "%s: one projection does not fit %zu bytes", who, budget);
        z = std::min((double)d.vol_z, std::floor((B - a * view * pix_in) / (plane * vox_out)));
        if (z < 1) return fail(B2T_ERR_NO_MEMORY, "%s: one volume slice does not fit %zu bytes", who, budget);
    }
    // angle blocks of at most an eighth of the views (and at least 16 views):
    // the FP downloads one block while it computes the next, the BP and FDK
    // upload the next block while they compute one, so transfers overlap
    // compute even when everything would fit at once
    const double overlap_block = std::max(16.0, std::ceil(d.angles / 8.0));
    a = std::min(a, overlap_block);
    slab = (uint32_t)z;
    block = (uint32_t)a;
    return B2T_OK;
}

}  // namespace

b2t_status stream3d_run(int32_t op, const b2t_geom3d *g, const b2t_params3d *params,
                        const b2t_filter_config *filter, int32_t short_scan, float fdk_scale, const float *in,
                        float *out, int32_t mode, const b2t_stream_config *cfg)
{
    const char *who = op == 0 ? "b2t_fp3d_host" : (op == 1 ? "b2t_bp3d_host" : "b2t_fdk_host");
    B2T_TRY(validate3d(g, who));
    if (!in || !out) return fail(B2T_ERR_INVALID_ARG, "%s: null data pointer", who);
    if (mode != B2T_MODE_ADD && mode != B2T_MODE_SET) return fail(B2T_ERR_INVALID_ARG, "%s: bad mode", who);
    if (op == 2 && g->kind != B2T_GEOM_CONE) return fail(B2T_ERR_UNSUPPORTED, "%s: FDK needs a cone geometry", who);
    Req R;
    R.op = op == 0 ? Op::fp : (op == 1 ? Op::bp : Op::fdk);
    R.g = g;
    if (params) {
        R.params = *params;
    } else {
        R.params = b2t_params3d{1, 1, 1.0f, B2T_KER_DEFAULT};
    }
    R.filter = filter;
    R.short_scan = short_scan;
    R.fdk_scale = fdk_scale;
    R.in = in;
    R.out = out;
    R.mode = mode;
    std::vector<int> devs;
    B2T_TRY(stream3d_plan_impl(op, g, cfg, who, devs, R.slab, R.block));
    const b2t_dims3d &d = g->dims;
    const uint32_t njobs = op == 0 ? (uint32_t)angle_blocks(d.angles, R.block, true).size()
                                   : (d.vol_z + R.slab - 1) / R.slab;
    const size_t nw = std::min<size_t>(devs.size(), njobs);
    std::vector<std::vector<uint32_t>> share(nw);
    for (uint32_t j = 0; j < njobs; ++j) share[j % nw].push_back(j);
    std::vector<b2t_status> st(nw, B2T_OK);
    std::vector<std::string> msg(nw);
    auto work = [&](size_t w) {
        st[w] = run_worker(R, devs[w], share[w]);
        if (st[w] != B2T_OK) {
            const char *m = b2t_last_error();
            msg[w] = m ? m : "";
        }
    };
    int cur = 0;
    B2T_CUDA_TRY(cudaGetDevice(&cur), "current device");
    if (nw == 1) {
        work(0);
    } else {
        std::vector<std::thread> threads;
        for (size_t w = 0; w < nw; ++w) threads.emplace_back(work, w);
        for (std::thread &t : threads) t.join();
    }
    cudaSetDevice(cur);
    for (size_t w = 0; w < nw; ++w)
        if (st[w] != B2T_OK) return fail(st[w], "%s (device %d): %s", who, devs[w], msg[w].c_str());
    return B2T_OK;
}


b2t_status stream3d_plan(int32_t op, const b2t_geom3d *g, const b2t_stream_config *cfg, uint32_t *slab,
                         uint32_t *block)
{
    B2T_TRY(validate3d(g, "b2t_stream_plan"));
    if (op < 0 || op > 2 || !slab || !block) return fail(B2T_ERR_INVALID_ARG, "b2t_stream_plan: bad argument");
    std::vector<int> devs;
    return stream3d_plan_impl(op, g, cfg, "b2t_stream_plan", devs, *slab, *block);
}

}  // namespace b2t
