// Internal declarations of the batched 3D projector (batch3d.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "b2tomo.h"
#include "proj3d.h"

namespace b2t {

// Device table entry of one problem of a 3D batch.
struct Batch3DProb {
    int kind, nx, ny, nz, na, nu, nv, rays;
    float fsc[3][3];           // FP ray scale (f1, f2, mul) per marching axis
    float bp_scale;            // BP output scale
    int fpview_off, bpview_off;   // first view of this problem in the view tables
    long long vol_off, proj_off;  // element offsets in the packed buffers
};

// A batch: problems, their packed layout, per-view constants on the device
// and the work items of the persistent kernels, ordered by decreasing cost.
struct Batch3D {
    std::vector<Batch3DProb> probs;
    size_t vol_total = 0, proj_total = 0;
    int n_fp_items = 0, n_bp_items = 0;
    int device = 0;
    // device memory (one allocation, carved up)
    void *mem = nullptr;
    Batch3DProb *d_probs = nullptr;
    FPView *d_fpv = nullptr;     // FP constants of every view (in its marching frame)
    BPView *d_bpv = nullptr;     // BP constants of every view
    int4 *d_fp_items = nullptr;  // (problem, view, detector tile, marching axis)
    int4 *d_bp_items = nullptr;  // (problem, block x, block y, block z)
    int *d_counters = nullptr;   // work counters of the FP and BP launches
    ~Batch3D();
};

b2t_status batch3d_create_impl(const b2t_problem3d *problems, int32_t n, Batch3D **out);
b2t_status batch3d_fp_impl(Batch3D *b, const float *vols, float *projs, int32_t mode, cudaStream_t s);
b2t_status batch3d_bp_impl(Batch3D *b, const float *projs, float *vols, int32_t mode, bool matched, cudaStream_t s);

}  // namespace b2t
