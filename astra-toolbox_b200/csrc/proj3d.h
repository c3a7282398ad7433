// Internal declarations of the 3D projector module (launch parameter blocks
// and host entry points behind b2t_fp3d / b2t_bp3d).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "b2tomo.h"

namespace b2t {

// Per-view forward-projection coefficients in the view's dominant frame
// (see fp_view_coeffs): den, slopes a1/a2 and offsets b1/b2 are affine in the
// detector offset (u', v') and share the denominator.  64 bytes.
struct FPView {
    float e[3];
    float m1[3], m2[3];
    float n1[3], n2[3];
    int a;  // global view index
};

// Views per forward-projection launch: the parameter block stays under the
// 32764-byte kernel parameter limit.
constexpr int FP_MAX_VIEWS = 448;

struct FPLaunch {
    const void *vol;        // padded volume, pointing at texel (s=0, k1=0, k2=0)
    void *proj;             // output projections [v][angle][u]
    long long proj_pitch;   // elements
    long long st0, st1, st2; // element strides of the marching axis, axis 1 and axis 2 (the direct
                             // kernel's padded volume has st1 = 1)
    int n0, n1, n2;         // extents along marching axis, axis 1, axis 2
    int nu, nv, na;
    int rays;               // detector supersampling per dimension
    int accumulate;         // 1: proj += result, 0: proj = result
    float f1, f2, mul;      // ray length factors and output scale
    int nviews;
    FPView views[FP_MAX_VIEWS];
};

// Per-view backprojection coefficients: texture u = nu.(x,y,z,1) / den.(x,y,z,1)
// (cone) or nu.(x,y,z,1) (parallel, den.w = per-view weight).  48 bytes.
struct BPView {
    float4 nu, nv, den;
};

constexpr int BP_MAX_VIEWS = 640;

struct BPLaunch {
    const void *proj;       // padded projections, pointing at texel (u=0, angle 0, v=0)
    long long pv;           // element stride between detector rows
    int pu;                 // element stride between views
    void *vol;
    long long vol_pitch;
    int nx, ny, nz, nu, nv;
    int a0, nviews;         // first view of this launch and count
    int rays;               // voxel supersampling per dimension
    int accumulate;
    float out_scale;
    BPView views[BP_MAX_VIEWS];
};

// TMA-staged backprojection (bp3d_tma.cu): voxel block, tile geometry and
// the shared-memory ring the tiles stream through.
// voxels per thread along z: 32 unless b2t_autotune_bp3d (or the volume's
// depth) chose 16 for the problem class
constexpr int BPT_CHUNK = 8;          // tile rows per TMA box; a view loads the chunks its footprint needs
constexpr int BPT_BV = 96;            // most rows one view's tile may take
constexpr int BPT_RING_BYTES = 75264; // ring of tile rows (224 rows of 84 4-byte elements: FP32 texels or
                                      // 16-bit pairs); three CTAs of ring + records (and the 1 KB each
                                      // reserves) fit an SM's 228 KB
constexpr int BPT_CTAS_PER_SM = 3;    // resident CTAs (72 registers a thread with 32 accumulators)
constexpr int BPT_SLOTS = 8;          // views in flight at most (barrier pairs and stage records)
// Views per launch: their coefficients travel in the launch record, 12
// floats a view, 10 when every view is circular (nu.z = den.z = 0).
constexpr int BPT_VIEW_FLOATS = 7680;
constexpr int BPT_MAX_VIEWS = BPT_VIEW_FLOATS / 12;
constexpr int BPT_MAX_VIEWS_CIRC = BPT_VIEW_FLOATS / 10;

struct alignas(64) BPTmaLaunch {
    CUtensorMap tmap;       // padded projections: dims (pu, angles, det_v + 4)
    const void *proj;       // padded projections at texel (u=0, angle 0, v=0)
    long long pv;
    int pu;
    void *vol;
    long long vol_pitch;
    int nx, ny, nz, nu, nv, na;
    int a0, nviews, accumulate;
    float out_scale;
    uint32_t tile_row_bytes;  // bytes per ring row (a launch value: see the kernel's addressing)
    float vrec[BPT_VIEW_FLOATS];  // the views' BPView coefficients, packed (see BPT_MAX_VIEWS)
};

// Row pitch (elements) of the zero-padded projection buffer: det_u plus a
// 2-texel border on each side, rounded up to 8 so rows are 16-byte aligned
// for TMA in every storage type.
inline size_t padded_pu(uint32_t det_u) { return ((size_t)det_u + 4 + 7) & ~(size_t)7; }

// Bytes per element of the padded projection buffer.  16-bit projections
// bound for the TMA backprojector use the pair layout: element (v, a, u) is
// the 32-bit word (x[v][a][u], x[v+1][a][u]), the texel and the one below it
// (x past the last row zero); every other case stores the texels themselves.
inline size_t padded_elem_size(int32_t dtype, bool pairs) { return (pairs || dtype == B2T_F32) ? 4 : 2; }

b2t_status bp3d_tma(const b2t_geom3d *g, int ker, float out_scale, const void *padded, bool pairs, void *vol,
                    size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s);
b2t_status device_errors_impl(uint32_t *flags);
b2t_status bp_path_stats_impl(uint64_t *stats);
b2t_status bp3d_autotune_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *proj, size_t proj_pitch,
                              void *vol, size_t vol_pitch, int32_t dtype, cudaStream_t s, int32_t *vpt_out);
// One warp waits, bounded by limit cycles, for an mbarrier phase (which 0) or
// a device flag (which 1) that nothing completes; B2T_ERR_TIMEOUT when the
// wait gave up and set the device error word.
b2t_status selftest_wait_impl(int which, long long limit, cudaStream_t s);

int dominant_axis(int kind, const b2t_view3d &w, const b2t_dims3d &d);
void fp_view_coeffs(int kind, const b2t_view3d &w, const b2t_dims3d &d, int dir, FPView &o);
void fp_scale(int kind, int dir, const float *vs, bool force_noncube, float out_scale, float &f1,
              float &f2, float &mul);
void bp_view_coeffs(int kind, int kernel, const b2t_view3d &w, const float *vs, BPView &o);
b2t_status validate3d(const b2t_geom3d *g, const char *who);
bool force_simple_bp();
bool force_simple_fp();
b2t_status fp3d_cells(const b2t_geom3d *g, const b2t_params3d *p, const void *vol, size_t vol_pitch, void *proj,
                      size_t proj_pitch, int32_t dtype, int32_t mode, const std::vector<int> &dirs, cudaStream_t s);

// The cell copies of one volume for the cell forward projector
// (fp3d_cells.cu), built once and projected by any number of calls over
// subsets of the views (the streamed executor's angle blocks).
class Scratch;
struct FPCells {
    FPCells();
    ~FPCells();
    FPCells(const FPCells &) = delete;
    FPCells &operator=(const FPCells &) = delete;
    std::unique_ptr<Scratch> mem[3];
    const void *base[3] = {nullptr, nullptr, nullptr};  // cell of texels (0, 0), slice 0, per marching axis
    long long st0[3] = {0, 0, 0}, st1[3] = {0, 0, 0}, st2[3] = {0, 0, 0};
    // marching axes held as a slab copy for the TMA-staged kernel
    // (fp3d_slab.cu) instead of cells; base[] then points at the copy
    bool slab[3] = {false, false, false};
    int32_t dtype = B2T_F32;
    uint32_t vol_x = 0, vol_y = 0, vol_z = 0;
};
// Builds the cells (or slab copies) of the marching axes marked in need[]
// (x, y, z) for the views of g projected with parameters p.
b2t_status fp3d_cells_build(const b2t_geom3d *g, const b2t_params3d *p, const void *vol, size_t vol_pitch,
                            int32_t dtype, const bool need[3], cudaStream_t s, FPCells &c);

// TMA-staged slab forward projector (fp3d_slab.cu) for x- and y-major views
// whose rays share the in-plane position along a detector column: FP32,
// no detector supersampling.
bool fp_slab_eligible(const b2t_geom3d *g, const b2t_params3d *p, int32_t dtype, int dir, const std::vector<int> &dirs);
size_t fp_slab_copy_bytes(const b2t_dims3d &d, int dir);
b2t_status fp_slab_build(const b2t_dims3d &d, const float *vol, size_t vol_pitch, int dir, void *copy,
                         cudaStream_t s);
b2t_status fp_slab_project(const b2t_geom3d *g, const b2t_params3d *p, const void *copy, int dir, void *proj,
                           size_t proj_pitch, int32_t mode, const std::vector<int> &dirs, cudaStream_t s);
b2t_status fp_slab_errors(uint32_t *flags);
b2t_status fp_path_stats_impl(uint64_t *stats);
unsigned long long fp_cell_launches_take();

// The slab FP's transpose (fp3d_slab.cu), the matched BP of the views the
// slab FP takes (any projection storage type): scatters into an FP32
// accumulator of matched_slab_acc_bytes (zeroed by the caller), cell (s, k1,
// k2) at (s * ay + k1 + 2) * az + k2 + 2 with (ay, az) from matched_slab_dims.
bool matched_slab_eligible(const b2t_geom3d *g, const b2t_params3d *p, int dir, const std::vector<int> &dirs);
void matched_slab_dims(const b2t_dims3d &d, int dir, long long &ay, long long &az);
size_t matched_slab_acc_bytes(const b2t_dims3d &d, int dir);
b2t_status matched_slab_scatter(const b2t_geom3d *g, const b2t_params3d *p, const void *proj, size_t proj_pitch,
                                int32_t dtype, int dir, const std::vector<int> &dirs, float *acc, cudaStream_t s);
b2t_status matched_path_stats_impl(uint64_t *stats);
// launches of matched.cu's scatter kernels since the last call
unsigned long long matched_scatter_launches_take();
// proj (=|+=) FP of the volume the cells hold, for the views of g (same
// volume dimensions as at build time; every view's marching axis built).
b2t_status fp3d_cells_project(const b2t_geom3d *g, const b2t_params3d *p, const FPCells &c, void *proj,
                              size_t proj_pitch, int32_t mode, cudaStream_t s);

// Zero-padded FP32 volume copies (2-voxel border): xyz = [z+2][y+2][x+2],
// zxy = [z+2][x+2][y+2] (either may be null).
b2t_status pad_volumes_f32(const float *vol, size_t pitch, const b2t_dims3d &d, float *xyz, float *zxy,
                           cudaStream_t s);
b2t_status fp3d_cyl_impl(const b2t_geom3d_cyl *g, const b2t_params3d *p, const float *vol, size_t vol_pitch,
                         float *proj, size_t proj_pitch, int32_t mode, cudaStream_t s);
b2t_status bp3d_cyl_impl(const b2t_geom3d_cyl *g, const b2t_params3d *p, const float *proj, size_t proj_pitch,
                         float *vol, size_t vol_pitch, int32_t mode, cudaStream_t s);
b2t_status stream3d_run(int32_t op, const b2t_geom3d *g, const b2t_params3d *params,
                        const b2t_filter_config *filter, int32_t short_scan, float fdk_scale, const float *in,
                        float *out, int32_t mode, const b2t_stream_config *cfg);
b2t_status stream3d_plan(int32_t op, const b2t_geom3d *g, const b2t_stream_config *cfg, uint32_t *slab,
                         uint32_t *block);
b2t_status fp3d_sumsqw_impl(const b2t_geom3d *g, const b2t_params3d *p, void *proj, size_t proj_pitch,
                            int32_t dtype, int32_t mode, cudaStream_t s);
b2t_status fp3d_autotune_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *vol, size_t vol_pitch,
                              void *proj, size_t proj_pitch, int32_t dtype, cudaStream_t s, int32_t *vpc_out);
b2t_status fp3d_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *vol, size_t vol_pitch,
                     void *proj, size_t proj_pitch, int32_t dtype, int32_t mode, cudaStream_t s);
b2t_status bp3d_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *proj, size_t proj_pitch,
                     void *vol, size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s);
// Whether the padded projections of a backprojection with these parameters
// use the pair layout (padded_elem_size).
bool bp_pairs(int32_t dtype, const b2t_params3d *p);
size_t padded_proj_bytes(const b2t_dims3d &d, int32_t dtype, bool pairs);
// The zero-padded projection buffer of projections proj (row pitch in
// texels) in the layout bp_pairs selects.
b2t_status pad_projections_impl(const void *proj, size_t pitch, const b2t_dims3d &d, void *padded, int32_t dtype,
                                bool pairs, cudaStream_t s);
// BP from a zero-padded projection buffer in the layout bp_pairs(dtype, p)
// names.
b2t_status bp3d_from_padded(const b2t_geom3d *g, const b2t_params3d *p, const void *padded, void *vol,
                            size_t vol_pitch, int32_t dtype, int32_t mode, cudaStream_t s);
b2t_status matched_bp3d_impl(const b2t_geom3d *g, const b2t_params3d *p, const void *proj,
                             size_t proj_pitch, void *vol, size_t vol_pitch, int32_t dtype,
                             int32_t mode, cudaStream_t s);

}  // namespace b2t
