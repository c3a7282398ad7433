// Internal declarations of the batched 2D projector (batch2d.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "b2tomo.h"
#include "proj2d.h"

namespace b2t {

// Device table entry of one problem of a batch.
struct BatchProb {
    int kind, W, H, ndet, nang, det_ss, pix_ss, pad;
    float out_scale;
    int view_off;              // first view of this problem in the view tables
    long long vol_off, sino_off;  // element offsets in the packed buffers
};

// Chunks of the packed buffers, each inside one problem's segment, for the
// per-problem reductions and updates of CGLS on a batch: chunk c covers
// elements [begin, begin + len) of segment (problem) seg; the chunks of
// segment p are first[p] .. first[p + 1] - 1, in order.
struct SegChunk {
    long long begin;
    int len;
    int seg;
};
struct SegTable {
    const SegChunk *chunks = nullptr;  // device
    const int *first = nullptr;        // device, nseg + 1 entries
    int nchunks = 0;
    int nseg = 0;
};
constexpr int SEG_CHUNK = 32768;

// A batch: problems, their packed layout, per-view constants on the device
// and the work items of the persistent kernels, ordered by decreasing cost.
struct Batch2D {
    std::vector<BatchProb> probs;
    std::vector<std::vector<b2t_view2d>> views;  // host copies of each problem's views
    size_t vol_total = 0, sino_total = 0;
    int n_fp_items = 0, n_bp_items = 0;
    int device = 0;
    // device memory (one allocation, carved up)
    void *mem = nullptr;
    BatchProb *d_probs = nullptr;
    ParFPView *d_par = nullptr;    // FP constants of parallel views
    b2t_view2d *d_fan = nullptr;   // raw fan views
    BPView2D *d_bp = nullptr;      // BP constants of every view
    int4 *d_fp_items = nullptr;    // (problem, view, first detector, 0)
    int4 *d_bp_items = nullptr;    // (problem, tile x, tile y, 0)
    int *d_counters = nullptr;     // work counters of the FP and BP launches
    SegTable vol_segs, sino_segs;  // chunk tables of the packed buffers
    ~Batch2D();
};

b2t_status batch2d_create_impl(const b2t_problem2d *problems, int32_t n, Batch2D **out);
b2t_status batch2d_fp_impl(Batch2D *b, const float *vols, float *sinos, float scale, int32_t mode, cudaStream_t s);
b2t_status batch2d_bp_impl(Batch2D *b, const float *sinos, float *vols, float scale, int32_t mode, cudaStream_t s);

}  // namespace b2t
