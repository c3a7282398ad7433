/*
 * b2tomo.h -- C ABI of libb2tomo, a B200-native (sm_100a) implementation of
 * the ASTRA Toolbox CUDA projection core.
 *
 * Conventions (the reference's own, kept so the library drops in for
 * cuda/2d and cuda/3d):
 *   - volume [z][y][x] (x fastest), projections [v][angle][u] (u fastest);
 *     2D volume [row][col], sinogram [angle][det]
 *     (python/astra/src/dlpack.cpp:145-147, cuda/3d/mem3d.cu:348-353).
 *   - Row pitches are in ELEMENTS (>= the row length); pitch 0 means
 *     "contiguous".  All data pointers are device pointers unless a function
 *     says otherwise; all of them are caller-owned.
 *   - mode B2T_MODE_ADD accumulates (+=) into the output, B2T_MODE_SET
 *     overwrites it (CompositeGeometryManager.h:127-129 MODE_ADD / MODE_SET).
 *   - Every call is stream-ordered on the given cudaStream_t (passed as
 *     void*, NULL = the legacy default stream) and returns without a device
 *     synchronisation unless it says it returns a host value.  Per-view
 *     geometry travels in kernel parameters, so concurrent calls on different
 *     streams do not share state (the reference's module-global __constant__
 *     arrays, cuda/3d/cone_fp.cu:46-57, are gone).
 *   - Every function returns a b2t_status and never aborts or traps;
 *     b2t_last_error() gives the message of the last failure on the calling
 *     thread (the reference returns bool and logs through ASTRA_ERROR,
 *     cuda/2d/util.cu:359-375).
 */
#ifndef B2TOMO_H
#define B2TOMO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* status, errors, version                                                 */
/* ---------------------------------------------------------------------- */

typedef int32_t b2t_status;
enum {
    B2T_OK = 0,
    B2T_ERR_INVALID_ARG = 1,   /* bad geometry, sizes, pointers or options   */
    B2T_ERR_UNSUPPORTED = 2,   /* combination the reference also refuses     */
    B2T_ERR_CUDA = 3,          /* a CUDA runtime error                        */
    B2T_ERR_NO_MEMORY = 4,     /* device allocation failed                    */
    B2T_ERR_ABORTED = 5,       /* iteration stopped by b2t_request_abort      */
    B2T_ERR_TIMEOUT = 6        /* a bounded device-side wait gave up          */
};

/* Message of the last failing call on this thread ("" if none). */
const char *b2t_last_error(void);
/* Library version, e.g. 100 for 1.0.0. */
int32_t b2t_version(void);
/* Number of CUDA kernels this library has launched since it was loaded
 * (all threads); lets callers verify which work ran on the device. */
uint64_t b2t_kernel_launches(void);
/* Select the CUDA device for this host thread (astraCUDA::setGPUIndex,
 * cuda/2d/astra.cu:60-75). */
b2t_status b2t_set_device(int32_t device);
/* Read and clear the device-side error bits of the current device (bit 0:
 * a bounded wait inside a kernel gave up; the kernel returned early and its
 * output is incomplete).  Synchronises the device.  The reference has no
 * device-side waits and no counterpart. */
b2t_status b2t_device_errors(uint32_t *flags);
/* Read and clear, for the current device, the path statistics of the
 * TMA-staged cone/parallel backprojection since the last call.  Counts are in
 * voxel-column views (one thread's column of 32 voxels for one view):
 * stats[0] took the circular-orbit fast path (detector u fixed along the
 * column, every sample from the shared-memory tile of the view's footprint);
 * stats[1] took the general path (non-circular orbits, columns whose rows
 * leave the tile, views whose footprint does not fit a tile and read global
 * memory); stats[2] were idle lanes (columns outside the volume).  stats[3]
 * is the SM cycles the compute warps spent in their view loops, summed over
 * warps.  Synchronises the device.  A performance diagnostic; the reference
 * has no counterpart. */
b2t_status b2t_bp_path_stats(uint64_t stats[4]);
/* Read and clear the path statistics of the cone/parallel forward projection
 * since the last call: stats[0] slices that CTAs of the TMA-staged slab
 * kernel read from shared memory, stats[1] slices they read from the slab
 * copy in global memory (a box too large for a slice buffer), stats[2] slab
 * kernel launches, stats[3] cell kernel launches (views the slab kernel does
 * not take).  Synchronises the device.  A performance diagnostic; the
 * reference has no counterpart. */
b2t_status b2t_fp_path_stats(uint64_t stats[4]);
/* Read and clear the path statistics of the matched (exact-transpose)
 * backprojection since the last call: stats[0] slices whose accumulation box
 * CTAs of the slab transpose kept in shared memory, stats[1] slices they
 * scattered straight into global memory (a box too large for a slice
 * buffer), stats[2] slab transpose launches, stats[3] launches of the
 * per-sample scatter kernels (views the slab transpose does not take).
 * Synchronises the device.  A performance diagnostic; the reference has no
 * counterpart. */
b2t_status b2t_matched_path_stats(uint64_t stats[4]);

/* Failure-handling test hooks; the reference has no counterpart.
 * b2t_debug_fail_alloc(n), n >= 1: the n-th device allocation the library
 * makes from now on (any thread) fails with B2T_ERR_NO_MEMORY without
 * allocating, as a real out-of-memory would; n = 0 disarms it.  *pending (if
 * not null) receives the allocations that were still to go before the
 * previously armed failure (0: it fired, or none was armed).
 * b2t_debug_live_allocations: the device allocations the library holds now
 * (scratch, algorithm buffers, batch tables), to check that a failed call
 * released what it had taken.
 * b2t_selftest_bounded_wait: one warp waits for something nothing completes,
 * an mbarrier phase (which = 0) or a device flag (which = 1), with the
 * bounded wait the pipelined kernels use, limited to limit_cycles (at most
 * 4e9, about two seconds); the wait gives up, records bit 0 of the device
 * error word and returns.  Synchronises the stream, reads and clears the
 * error word and returns B2T_ERR_TIMEOUT when the bit was set. */
b2t_status b2t_debug_fail_alloc(int64_t nth, int64_t *pending);
int64_t b2t_debug_live_allocations(void);
b2t_status b2t_selftest_bounded_wait(int32_t which, uint64_t limit_cycles, void *stream);

/* Scratch buffers (padded copies, cell copies, filter operands) come from a
 * stream-ordered memory pool of the library, one per device, that keeps freed
 * blocks cached so repeated calls do not map device memory again.  This
 * synchronises the current device and returns the cached blocks of every
 * device to the driver.  The reference allocates and frees per call with
 * cudaMalloc / cudaFree (cuda/3d/mem3d.cu:82-166, cuda/3d/fdk.cu:341). */
b2t_status b2t_release_cached_memory(void);

/* ---------------------------------------------------------------------- */
/* enumerations                                                            */
/* ---------------------------------------------------------------------- */

enum { B2T_MODE_ADD = 0, B2T_MODE_SET = 1 };

/* storage types of volume / projection data; all arithmetic is FP32 */
enum { B2T_F32 = 0, B2T_F16 = 1, B2T_BF16 = 2 };

/* geometry kinds */
enum {
    B2T_GEOM_PAR3D = 1,   /* parallel3d, parallel3d_vec -> SPar3DProjection  */
    B2T_GEOM_CONE = 2,    /* cone, cone_vec            -> SConeProjection   */
    B2T_GEOM_PAR2D = 3,   /* parallel, parallel_vec    -> SParProjection    */
    B2T_GEOM_FAN2D = 4,   /* fanflat, fanflat_vec      -> SFanProjection    */
    B2T_GEOM_CYLCONE = 5  /* cyl_cone_vec -> SCylConeProjection (b2t_geom3d_cyl) */
};

/* projection kernels: Cuda3DProjectionKernel (cuda/3d/dims3d.h:45-51) */
enum {
    B2T_KER_DEFAULT = 0,
    B2T_KER_SUM_SQUARE_WEIGHTS = 1,
    B2T_KER_FDK_WEIGHTING = 2,
    B2T_KER_2D_WEIGHTING = 3,
    B2T_KER_MATCHED_BP = 4     /* exact transpose of the forward projector   */
};

/* filter types: E_FBPFILTER (include/astra/Filters.h:43-66) in the same order
 * without its leading FILTER_ERROR, i.e. B2T value = E_FBPFILTER value - 1 */
enum {
    B2T_FILTER_NONE = 0,
    B2T_FILTER_RAMLAK = 1,
    B2T_FILTER_SHEPPLOGAN = 2,
    B2T_FILTER_COSINE = 3,
    B2T_FILTER_HAMMING = 4,
    B2T_FILTER_HANN = 5,
    B2T_FILTER_TUKEY = 6,          /* parameter: alpha (default 0.5)           */
    B2T_FILTER_LANCZOS = 7,
    B2T_FILTER_TRIANGULAR = 8,
    B2T_FILTER_GAUSSIAN = 9,       /* parameter: sigma (default 0.4)           */
    B2T_FILTER_BARTLETTHANN = 10,
    B2T_FILTER_BLACKMAN = 11,      /* parameter: alpha (default 0.16)          */
    B2T_FILTER_NUTTALL = 12,
    B2T_FILTER_BLACKMANHARRIS = 13,
    B2T_FILTER_BLACKMANNUTTALL = 14,
    B2T_FILTER_FLATTOP = 15,
    B2T_FILTER_KAISER = 16,        /* parameter: alpha (default 3)             */
    B2T_FILTER_PARZEN = 17,
    B2T_FILTER_PROJECTION = 18,    /* custom spectrum, shared by all views     */
    B2T_FILTER_SINOGRAM = 19,      /* custom spectrum per view                 */
    B2T_FILTER_RPROJECTION = 20,   /* custom spatial filter, shared            */
    B2T_FILTER_RSINOGRAM = 21      /* custom spatial filter per view           */
};

/* SFilterConfig (include/astra/Filters.h:70-82).  d: frequency cut-off
 * scale (FilterD, spectrum zero beyond w = pi d); parameter: FilterParameter
 * (< 0 = the type's default).  custom: host array, custom_height rows of
 * custom_width values: for PROJECTION / SINOGRAM the real spectrum on
 * nextpow2(2 det) / 2 + 1 bins, for RPROJECTION / RSINOGRAM a spatial filter
 * of any width centred on its element width / 2; one row, or one per view
 * for the SINOGRAM types.  A NULL config means Ram-Lak with d = 1. */
typedef struct b2t_filter_config {
    int32_t type;
    float d;
    float parameter;
    const float *custom;
    uint32_t custom_width;
    uint32_t custom_height;
} b2t_filter_config;

/* element-wise operations: processVol3D<op> (cuda/3d/arith3d.cu:44-111) */
enum {
    B2T_OP_SET = 0,          /* out = s                                     */
    B2T_OP_MUL_SCALAR = 1,   /* out *= s                                    */
    B2T_OP_MUL = 2,          /* out *= a                                    */
    B2T_OP_ADD_MUL = 3,      /* out += a * b           (opAddMul)           */
    B2T_OP_ADD_SCALED = 4,   /* out += a * s           (opAddScaled)        */
    B2T_OP_SCALE_AND_ADD = 5,/* out = a + out * s      (opScaleAndAdd)      */
    B2T_OP_INVERT = 6,       /* out = out > 1e-6 ? 1/out : 0 (opInvert)     */
    B2T_OP_CLAMP_MIN = 7,    /* out = max(out, s)                           */
    B2T_OP_CLAMP_MAX = 8,    /* out = min(out, s)                           */
    B2T_OP_ADD = 9           /* out += a                                    */
};

/* ---------------------------------------------------------------------- */
/* geometry                                                                */
/* ---------------------------------------------------------------------- */

/* One 3D view.  Same layout and meaning as SConeProjection / SPar3DProjection
 * (include/astra/GeometryUtil3D.h:47-115): src = source position (cone) or
 * ray direction (parallel); det_s = detector corner ("bottom left" of pixel
 * (0,0)); det_u / det_v = one pixel step along u / v. */
typedef struct b2t_view3d {
    double src[3];
    double det_s[3];
    double det_u[3];
    double det_v[3];
} b2t_view3d;

/* SDimensions3D (include/astra/GeometryUtil3D.h:150-157) */
typedef struct b2t_dims3d {
    uint32_t vol_x, vol_y, vol_z;
    uint32_t angles, det_u, det_v;
} b2t_dims3d;

/* Normalised 3D geometry: views already translated/scaled to unit voxels
 * centred on the origin.  Geometry3DParameters (GeometryUtil3D.h:172-227). */
typedef struct b2t_geom3d {
    int32_t kind;              /* B2T_GEOM_PAR3D or B2T_GEOM_CONE            */
    b2t_dims3d dims;
    float vol_scale[3];        /* SVolScale3D: voxel size x, y, z            */
    const b2t_view3d *views;   /* host array of dims.angles views            */
} b2t_geom3d;

/* SProjectorParams3D (cuda/3d/dims3d.h:53-66) minus volScale */
typedef struct b2t_params3d {
    uint32_t det_supersample;    /* iRaysPerDetDim   (DetectorSuperSampling) */
    uint32_t voxel_supersample;  /* iRaysPerVoxelDim (VoxelSuperSampling)    */
    float output_scale;          /* fOutputScale                             */
    int32_t kernel;              /* B2T_KER_*                                */
} b2t_params3d;

/* CVolumeGeometry3D window (src/VolumeGeometry3D.cpp:140-180): grid counts
 * and window extents, float32 as the reference stores them. */
typedef struct b2t_volgeom3d {
    uint32_t cols, rows, slices;  /* x, y, z */
    float min_x, max_x, min_y, max_y, min_z, max_z;
} b2t_volgeom3d;

/* genConeProjections (src/GeometryUtil3D.cpp:42-83). */
b2t_status b2t_cone_views(uint32_t n_angles, uint32_t det_cols, uint32_t det_rows,
                          float src_origin, float origin_det, float det_spacing_x,
                          float det_spacing_y, const float *angles, b2t_view3d *out);
/* genPar3DProjections (src/GeometryUtil3D.cpp:133-172). */
b2t_status b2t_par3d_views(uint32_t n_angles, uint32_t det_cols, uint32_t det_rows,
                           float det_spacing_x, float det_spacing_y, const float *angles,
                           b2t_view3d *out);
/* cone_vec / parallel3d_vec rows (12 doubles: src-or-ray, detector CENTRE, u,
 * v) to corner-based views: CConeVecProjectionGeometry3D /
 * CParallelVecProjectionGeometry3D initialisation
 * (src/ConeVecProjectionGeometry3D.cpp:96-110). */
b2t_status b2t_vec_views3d(uint32_t n_angles, uint32_t det_cols, uint32_t det_rows,
                           const double *vectors, b2t_view3d *out);
/* convertAstraGeometry_internal (src/GeometryUtil3D.cpp:569-593): translate by
 * the float window centre, scale by the float inverse voxel size, in place.
 * Writes the voxel size to vol_scale_out[3]. */
b2t_status b2t_normalize_views3d(const b2t_volgeom3d *vol, int32_t kind, uint32_t n,
                                 b2t_view3d *views, float *vol_scale_out);

/* cyl_cone_vec: one view of a cone beam on a detector curved around an axis,
 * layout-identical to SCylConeProjection (include/astra/GeometryUtil3D.h:125-150).
 * det_c = centre of the detector (on the cylinder); det_u = tangent from pixel
 * (0,0) to (0,1), its length the pixel's arc length; det_v = pixel (0,0) to
 * (1,0) along the cylinder axis; radius = cylinder radius. */
typedef struct b2t_view3d_cyl {
    double src[3];
    double det_c[3];
    double det_u[3];
    double det_v[3];
    double radius;
} b2t_view3d_cyl;

typedef struct b2t_geom3d_cyl {
    b2t_dims3d dims;
    float vol_scale[3];            /* voxel size x, y, z (world units)           */
    const b2t_view3d_cyl *views;   /* host array of dims.angles views            */
} b2t_geom3d_cyl;

/* convertAstraGeometry for cyl_cone_vec (src/GeometryUtil3D.cpp:733-752 with
 * convertAstraGeometry_unscaled_internal :597-617): translate source and
 * detector centre so the volume is centred; no scaling (the kernels take the
 * voxel size).  Writes the voxel size. */
b2t_status b2t_normalize_views3d_cyl(const b2t_volgeom3d *vol, uint32_t n, b2t_view3d_cyl *views,
                                     float *vol_scale_out);

/* One 2D view: SFanProjection / SParProjection (GeometryUtil2D.h:53-105),
 * float fields.  src = source (fan) or ray direction (parallel); det_s =
 * detector start (pixel 0 corner); det_u = one detector pixel step. */
typedef struct b2t_view2d {
    float src[2];
    float det_s[2];
    float det_u[2];
} b2t_view2d;

/* SDimensions (include/astra/GeometryUtil2D.h:41-51) */
typedef struct b2t_dims2d {
    uint32_t vol_width, vol_height;
    uint32_t angles, dets;
} b2t_dims2d;

/* Normalised 2D geometry: Geometry2DParameters (GeometryUtil2D.h:107-150). */
typedef struct b2t_geom2d {
    int32_t kind;              /* B2T_GEOM_PAR2D or B2T_GEOM_FAN2D            */
    b2t_dims2d dims;
    float output_scale;        /* pixel size (convertAstraGeometry, 2D)       */
    const b2t_view2d *views;   /* host array of dims.angles views             */
} b2t_geom2d;

/* CVolumeGeometry2D window (src/VolumeGeometry2D.cpp:190-205). */
typedef struct b2t_volgeom2d {
    uint32_t cols, rows;
    float min_x, max_x, min_y, max_y;
} b2t_volgeom2d;

/* genParProjections (src/GeometryUtil2D.cpp:40-78), no extra offsets. */
b2t_status b2t_par_views(uint32_t n_angles, uint32_t n_dets, float det_width,
                         const float *angles, b2t_view2d *out);
/* genFanProjections (src/GeometryUtil2D.cpp:81-104). */
b2t_status b2t_fan_views(uint32_t n_angles, uint32_t n_dets, float src_origin, float origin_det,
                         float det_width, const float *angles, b2t_view2d *out);
/* parallel_vec / fanflat_vec rows (6 doubles: src-or-ray, detector CENTRE,
 * u) to corner-based views (src/FanFlatVecProjectionGeometry2D.cpp:108-124). */
b2t_status b2t_vec_views2d(uint32_t n_angles, uint32_t n_dets, const double *vectors,
                           b2t_view2d *out);
/* convertAstraGeometry_internal, 2D (src/GeometryUtil2D.cpp:182-209); refuses
 * non-square pixels as the reference does.  Writes the output scale. */
b2t_status b2t_normalize_views2d(const b2t_volgeom2d *vol, int32_t kind, uint32_t n,
                                 b2t_view2d *views, float *output_scale);

/* ---------------------------------------------------------------------- */
/* 3D projectors                                                           */
/* ---------------------------------------------------------------------- */

/* Forward projection proj (+)= A vol.  Replaces astraCUDA3d::FP
 * (include/astra/cuda/3d/mem3d.h:107), ConeFP (cone_fp.h:33-36) and Par3DFP
 * (par3d_fp.h:33-36).  Kernels: DEFAULT, 2D_WEIGHTING, FDK_WEIGHTING and
 * MATCHED_BP project identically (cuda/3d/mem3d.cu:355-386).
 * SUM_SQUARE_WEIGHTS (parallel-beam geometries, no detector supersampling)
 * writes each ray's sum of squared interpolation weights times the squared
 * ray-length factor instead, as Par3DFP_SumSqW (par3d_fp.h:43, par3d_fp.cu:607);
 * it reads no volume and vol may be NULL.  vol and proj have storage type
 * dtype (B2T_F32/F16/BF16). */
b2t_status b2t_fp3d(const b2t_geom3d *geom, const b2t_params3d *params,
                    const void *vol, size_t vol_pitch, void *proj, size_t proj_pitch,
                    int32_t dtype, int32_t mode, void *stream);

/* Backprojection vol (+)= B proj.  Replaces astraCUDA3d::BP (mem3d.h:109),
 * ConeBP (cone_bp.h:33-36) and Par3DBP (par3d_bp.h:33-36).  kernel DEFAULT is
 * ASTRA's voxel-driven BP (not the exact adjoint), FDK_WEIGHTING and
 * 2D_WEIGHTING its weight variants (cone_bp.cu:99-123, 226-269), MATCHED_BP
 * the exact transpose of b2t_fp3d (ker3d_matched_bp, mem3d.cu:463-479, which
 * the reference implements only for cyl_cone_vec). */
b2t_status b2t_bp3d(const b2t_geom3d *geom, const b2t_params3d *params,
                    const void *proj, size_t proj_pitch, void *vol, size_t vol_pitch,
                    int32_t dtype, int32_t mode, void *stream);

/* Streamed projection of host-resident FP32 data larger than the device
 * memory (the reference's CompositeGeometryManager,
 * src/CompositeGeometryManager.cpp:218-379, 1115-1280, 1409-1477, behind
 * astraCUDA3d::FP/BP/FDK and astra.set_gpu_index(..., memory=...)).  The
 * volume is cut into z-slabs, the projections into angle blocks; blocks
 * stream through double-buffered device memory with the copies overlapping
 * the compute (pinned host memory), jobs spread over the listed GPUs.
 * Host arrays are tightly packed ([z][y][x], [v][angle][u]).  Calls block
 * until the output is in host memory. */
typedef struct b2t_stream_config {
    size_t device_bytes;       /* device memory per GPU (0: free memory less 2 GiB) */
    uint32_t n_devices;        /* GPUs to spread jobs over (0: the current device) */
    const int32_t *devices;    /* their ordinals                                  */
} b2t_stream_config;
b2t_status b2t_fp3d_host(const b2t_geom3d *geom, const b2t_params3d *params, const float *vol, float *proj,
                         int32_t mode, const b2t_stream_config *cfg);
b2t_status b2t_bp3d_host(const b2t_geom3d *geom, const b2t_params3d *params, const float *proj, float *vol,
                         int32_t mode, const b2t_stream_config *cfg);
b2t_status b2t_fdk_host(const b2t_geom3d *geom, const b2t_filter_config *filter, int32_t short_scan,
                        float output_scale, const float *proj, float *vol, int32_t mode,
                        const b2t_stream_config *cfg);
/* The split a streamed call would use: op 0 FP, 1 BP, 2 FDK; z-slab
 * thickness and angle block size. */
b2t_status b2t_stream_plan(int32_t op, const b2t_geom3d *geom, const b2t_stream_config *cfg, uint32_t *slab,
                           uint32_t *block);

/* Cone beam on a cylindrical detector (cyl_cone_vec), FP32 data.
 * b2t_fp3d_cyl replaces astraCUDA3d::ConeCylFP (cuda/3d/cone_cyl.cu:197-306,
 * 477-546, 622-682):
 * per ray from the source to the pixel centre on the cylinder, unit steps
 * along the dominant axis of (source - detector centre), bilinear samples,
 * times the ray length per step.  b2t_bp3d_cyl: kernel DEFAULT replaces
 * ConeCylBP (voxel-driven: the ray through
 * the voxel centre meets the cylinder, weight t^2, times the voxel volume;
 * cone_cyl_bp.cu:61-160, 235-320); MATCHED_BP is the exact transpose of
 * b2t_fp3d_cyl (the reference's ConeCylBP_matched, cone_cyl.cu:308-475,
 * 684-749, scatters the same model, without the output scale).
 * No supersampling, as the reference. */
b2t_status b2t_fp3d_cyl(const b2t_geom3d_cyl *geom, const b2t_params3d *params, const float *vol,
                        size_t vol_pitch, float *proj, size_t proj_pitch, int32_t mode, void *stream);
b2t_status b2t_bp3d_cyl(const b2t_geom3d_cyl *geom, const b2t_params3d *params, const float *proj,
                        size_t proj_pitch, float *vol, size_t vol_pitch, int32_t mode, void *stream);

/* ---------------------------------------------------------------------- */
/* 2D projectors (f32 data)                                                */
/* ---------------------------------------------------------------------- */

/* sino (+)= A vol.  Replaces astraCUDA::FP (include/astra/cuda/2d/par_fp.h:33,
 * cuda/2d/par_fp.cu:340) and astraCUDA::FanFP (fan_fp.h:33, fan_fp.cu:260);
 * det_supersample = iRaysPerDet (DetectorSuperSampling). */
b2t_status b2t_fp2d(const b2t_geom2d *geom, uint32_t det_supersample, const float *vol, size_t vol_pitch,
                    float *sino, size_t sino_pitch, int32_t mode, void *stream);

/* vol (+)= B sino.  Replaces astraCUDA::BP (par_bp.h:35, par_bp.cu:224),
 * FanBP and FanBP_FBPWeighted (fan_bp.h:33-48, fan_bp.cu:380-448);
 * fbp_weight != 0 selects the fan FBP weight 1/Den^2. */
b2t_status b2t_bp2d(const b2t_geom2d *geom, uint32_t pixel_supersample, int32_t fbp_weight, const float *sino,
                    size_t sino_pitch, float *vol, size_t vol_pitch, int32_t mode, void *stream);

/* ---------------------------------------------------------------------- */
/* FDK                                                                     */
/* ---------------------------------------------------------------------- */

/* FDK reconstruction of a cone geometry with a circular orbit: cosine /
 * magnification pre-weight, Parker weight if short_scan, Ram-Lak (or no)
 * filter along u (any b2t_filter_config), then the FDK-weighted cone BP;
 * vol (+)= result * scale.
 * Replaces astraCUDA3d::FDK (include/astra/cuda/3d/mem3d.h:113,
 * cuda/3d/fdk.cu:415-478).  Unlike the reference, proj is left unmodified:
 * the filtered projections go to a stream-ordered scratch buffer. */
b2t_status b2t_fdk(const b2t_geom3d *geom, const b2t_filter_config *filter, int32_t short_scan, float output_scale,
                   const void *proj, size_t proj_pitch, void *vol, size_t vol_pitch, int32_t dtype,
                   int32_t mode, void *stream);

/* Pre-weighting (+ Parker) and filtering of proj in place: FDK_PreWeight +
 * FDK_Filter (cuda/3d/fdk.cu:168-412). */
b2t_status b2t_fdk_weight_filter(const b2t_geom3d *geom, const b2t_filter_config *filter, int32_t short_scan, void *proj,
                                 size_t proj_pitch, int32_t dtype, void *stream);

/* Filtering of nrows rows of n f32 samples in place (row pitch in
 * elements): the zero-padded FFT convolution of runCudaFFT / applyFilter /
 * runCudaIFFT (cuda/2d/fft.cu:52-336) evaluated as its exact Toeplitz form.
 * For the per-view filter types row r uses the filter of view r. */
b2t_status b2t_filter_rows(float *data, size_t nrows, uint32_t n, size_t pitch, const b2t_filter_config *filter,
                           void *stream);

/* Host only: the spatial taps of a filter for rows of n samples, the exact
 * Toeplitz form of the reference's filtering (genFilter, src/Filters.cpp:
 * 131-488, and the custom types of cuda/2d/fft.cu:447-595).  out receives
 * n_sets x (2n - 1) floats, tap of offset d (y[i] = sum_k g[i - k] x[k]) at
 * d + n - 1; n_sets = n_views for the SINOGRAM types, else 1 (n_views is
 * then ignored).  *count (in: capacity of out in floats, out: needed) may be
 * queried with out = NULL. */
b2t_status b2t_filter_taps(const b2t_filter_config *filter, uint32_t n, uint32_t n_views, float *out,
                           size_t *count);

/* 2D filtered backprojection, vol (+)= FBP(sino); sino is not modified.
 * Replaces astraCUDA::FBP (cuda/2d/fbp.cu:77-190): parallel = filter + BP
 * scaled by (pi/2)/n_angles; fan = FDK pre-weighting of a one-row cone (+
 * Parker if short_scan) + filter + FBP-weighted fan BP. */
b2t_status b2t_fbp2d(const b2t_geom2d *geom, const b2t_filter_config *filter, int32_t short_scan, const float *sino,
                     size_t sino_pitch, float *vol, size_t vol_pitch, int32_t mode, void *stream);

/* ---------------------------------------------------------------------- */
/* element-wise operations and reductions                                  */
/* ---------------------------------------------------------------------- */

/* out = op(out, a, b, s) over n contiguous f32 elements (processVol3D<op>,
 * include/astra/cuda/3d/arith3d.h; processData<op>, cuda/2d/arith.cu). */
b2t_status b2t_vec_op(int32_t op, float *out, const float *a, const float *b, float s, size_t n,
                      void *stream);

/* sum(a[i] * b[i]) over n elements accumulated in FP64, written to the DEVICE
 * double *result.  b may equal a (squared norm).  Replaces dotProduct2D /
 * dotProduct3D (cuda/2d/util.cu:304-357, cuda/3d/mem3d.cu:581-590), which
 * accumulate in float32.  Uses a device scratch buffer that the call
 * allocates and frees in stream order. */
b2t_status b2t_dot_f64(const void *a, const void *b, size_t n, int32_t dtype, double *result,
                       void *stream);

/* The same FP64 inner product, allocating nothing.  No counterpart in the
 * reference.  For callers that cannot allocate device memory when they call
 * it (a real-time loop that must not wait on the allocator, a host that
 * hands out all device memory from its own fixed pool): the partial sums live
 * in a fixed 32 KB array built into the library, present on every GPU that
 * loads it until the process exits.  Limit: n <= 4096 * 2^20 elements; larger
 * n returns B2T_ERR_INVALID_ARG before any device work.  Up to 1184 * 2^20
 * elements it launches exactly as b2t_dot_f64 does and returns the same
 * bits.  All calls on one device share the array, so calls that overlap on
 * the GPU race: serialise them.  Every call looks up the array's device
 * address on the current device (a cheap host lookup that stays valid after
 * a cudaDeviceReset). */
b2t_status b2t_dot_f64_noalloc(const void *a, const void *b, size_t n, int32_t dtype, double *result,
                               void *stream);

/* ---------------------------------------------------------------------- */
/* SIRT / CGLS / SART reconstruction                                       */
/* ---------------------------------------------------------------------- */

enum { B2T_ALGO_SIRT = 1, B2T_ALGO_CGLS = 2, B2T_ALGO_SART = 3 /* 2D only */ };

/* Options of SIRT3D_CUDA / CGLS3D_CUDA / SIRT_CUDA / CGLS_CUDA
 * (src/ReconstructionAlgorithm3D.cpp:95-120, CudaSirtAlgorithm3D.cpp:141).
 * Mask and bound arrays are device pointers (NULL = unused) that must stay
 * valid while the algorithm is used. */
typedef struct b2t_algo_options {
    float relaxation;          /* SIRT "Relaxation" (default 1)                 */
    int32_t use_min;           /* MinConstraint                                 */
    float min_value;
    int32_t use_max;           /* MaxConstraint                                 */
    float max_value;
    const float *vol_mask;     /* ReconstructionMaskId                          */
    const float *sino_mask;    /* SinogramMaskId (SIRT)                         */
    const float *min_mask;     /* per-pixel lower bound (2D SIRT MinMaskId)     */
    const float *max_mask;     /* per-pixel upper bound (2D SIRT MaxMaskId)     */
} b2t_algo_options;

typedef struct b2t_algo b2t_algo;  /* opaque: operator, weights, work buffers */

/* SIRT3D_CUDA / CGLS3D_CUDA (src/CudaSirtAlgorithm3D.cpp,
 * src/CudaCglsAlgorithm3D.cpp).  Allocates the work buffers (cudaMalloc). */
b2t_status b2t_algo_create3d(int32_t type, const b2t_geom3d *geom, const b2t_params3d *params,
                             const b2t_algo_options *options, b2t_algo **out);
/* SIRT3D_CUDA / CGLS3D_CUDA on a cyl_cone_vec geometry (no supersampling:
 * CudaSirtAlgorithm3D.cpp:155-158, CudaCglsAlgorithm3D.cpp:156-159). */
b2t_status b2t_algo_create3d_cyl(int32_t type, const b2t_geom3d_cyl *geom, const b2t_params3d *params,
                                 const b2t_algo_options *options, b2t_algo **out);
/* SIRT_CUDA / CGLS_CUDA / SART_CUDA (src/CudaSirtAlgorithm.cpp,
 * src/CudaCglsAlgorithm.cpp, src/CudaSartAlgorithm.cpp).  SART: one iteration
 * is one view (in the order of b2t_algo_set_projection_order, sequential by
 * default); "relaxation" is its lambda; no sinogram mask, no per-pixel bounds
 * and no pixel supersampling, as the reference. */
b2t_status b2t_algo_create2d(int32_t type, const b2t_geom2d *geom, uint32_t det_supersample,
                             uint32_t pixel_supersample, const b2t_algo_options *options, b2t_algo **out);
/* run(iterations) (CudaSirtAlgorithm3D.cpp:301-381, CudaCglsAlgorithm3D.cpp:264-355):
 * iterates on device f32 data; vol is updated in place, sino is read.  CGLS
 * restarts at every call, as the reference does.  use_graph != 0 replays a
 * CUDA graph of the iteration (captured on first use). */
b2t_status b2t_algo_run(b2t_algo *algo, const float *sino, float *vol, int32_t iterations, int32_t use_graph,
                        void *stream);
/* getResidualNorm (CudaSirtAlgorithm3D.cpp:383-418): ||sino - A vol||_2,
 * accumulated in FP64; synchronises the stream. */
b2t_status b2t_algo_residual_norm(b2t_algo *algo, const float *sino, const float *vol, double *norm,
                                  void *stream);
/* SART's projection order (CudaSartAlgorithm.cpp:76-109, "ProjectionOrder" /
 * "ProjectionOrderList"): n view indices, used cyclically from the
 * algorithm's running step count.  B2T_ERR_INVALID_ARG for other algorithms
 * or out-of-range views. */
b2t_status b2t_algo_set_projection_order(b2t_algo *algo, const int32_t *order, uint32_t n);
/* Ask a running b2t_algo_run (on another thread) to stop between iterations
 * (astra::shouldAbort, src/Globals.cpp:49-58). */
void b2t_algo_abort(b2t_algo *algo);
void b2t_algo_destroy(b2t_algo *algo);

/* ---------------------------------------------------------------------- */
/* batched 2D problems                                                     */
/* ---------------------------------------------------------------------- */

/* One problem of a batch: its normalised geometry and supersampling. */
typedef struct b2t_problem2d {
    b2t_geom2d geom;              /* kind, dims, output scale, host views        */
    uint32_t det_supersample;     /* FP rays per detector (DetectorSuperSampling) */
    uint32_t pixel_supersample;   /* BP sub-pixels per axis (PixelSuperSampling)  */
} b2t_problem2d;

typedef struct b2t_batch2d b2t_batch2d;  /* opaque: device tables + work list */

/* Plan a batch of n independent 2D problems (parallel and fan mixed, any
 * sizes).  No counterpart in the reference, which projects such a set one
 * problem at a time through FP / FanFP / BP / FanBP
 * (include/astra/cuda/2d/par_fp.h:33, fan_fp.h, par_bp.h, fan_bp.h:33-44), at
 * least one launch each.  Copies the geometry to the device (synchronous,
 * allocates with cudaMalloc).  Problem i's volume (H x W, row-major) and
 * sinogram (angles x dets) live in two packed buffers at the element offsets
 * b2t_batch2d_layout reports. */
b2t_status b2t_batch2d_create(const b2t_problem2d *problems, int32_t n, b2t_batch2d **out);
/* Offsets (elements) of every problem in the packed buffers, and the buffer
 * lengths.  vol_offsets / sino_offsets hold n entries each (may be NULL). */
b2t_status b2t_batch2d_layout(const b2t_batch2d *batch, uint64_t *vol_offsets, uint64_t *sino_offsets,
                              uint64_t *vol_total, uint64_t *sino_total);
/* sinos (=|+=) A vols for every problem, in one persistent launch. */
b2t_status b2t_batch2d_fp(b2t_batch2d *batch, const float *vols, float *sinos, int32_t mode, void *stream);
/* vols (=|+=) A^T-style backprojection of sinos for every problem (the
 * reference's unmatched BP), in one persistent launch. */
b2t_status b2t_batch2d_bp(b2t_batch2d *batch, const float *sinos, float *vols, int32_t mode, void *stream);
/* SIRT_CUDA or CGLS_CUDA on every problem of the batch at once
 * (src/CudaSirtAlgorithm.cpp, src/CudaCglsAlgorithm.cpp): run with
 * b2t_algo_run / b2t_algo_residual_norm on the packed buffers.  Each problem
 * keeps its own CGLS step sizes (per-problem FP64 inner products), so the
 * iterates equal per-problem runs; the residual norm is over the whole batch.
 * Options as for b2t_algo_create2d, without masks.  The batch must outlive
 * the algorithm. */
b2t_status b2t_algo_create_batch2d(int32_t type, b2t_batch2d *batch, const b2t_algo_options *options,
                                   b2t_algo **out);
void b2t_batch2d_destroy(b2t_batch2d *batch);

/* ---------------------------------------------------------------------- */
/* batched 3D problems                                                     */
/* ---------------------------------------------------------------------- */

/* One problem of a 3D batch: a parallel3d / parallel3d_vec or cone / cone_vec
 * geometry (views as for b2t_fp3d), FP32 storage, the default kernel. */
typedef struct b2t_problem3d {
    b2t_geom3d geom;              /* kind, dims, voxel size, host views           */
    uint32_t det_supersample;     /* FP rays per detector pixel side (1..16)       */
    float output_scale;           /* as b2t_params3d.output_scale                  */
} b2t_problem3d;

typedef struct b2t_batch3d b2t_batch3d;  /* opaque: device tables + work list */

/* Plan a batch of n independent 3D problems (parallel and cone mixed, any
 * sizes and view counts).  No counterpart in the reference, which projects
 * such a set one problem at a time through astraCUDA3d::FP / BP
 * (include/astra/cuda/3d/mem3d.h:107-113), at least one launch each.
 * Copies the geometry to the device (synchronous, allocates with
 * cudaMalloc).  Problem i's volume (z, y, x) and projections (v, angle, u)
 * live in two packed buffers at the element offsets b2t_batch3d_layout
 * reports. */
b2t_status b2t_batch3d_create(const b2t_problem3d *problems, int32_t n, b2t_batch3d **out);
/* Offsets (elements) of every problem in the packed buffers, and the buffer
 * lengths.  vol_offsets / proj_offsets hold n entries each (may be NULL). */
b2t_status b2t_batch3d_layout(const b2t_batch3d *batch, uint64_t *vol_offsets, uint64_t *proj_offsets,
                              uint64_t *vol_total, uint64_t *proj_total);
/* projs (=|+=) FP of vols for every problem, in one persistent launch:
 * b2t_fp3d's direct-load ray model (cuda/3d/cone_fp.cu:154-231,
 * par3d_fp.cu:146-220). */
b2t_status b2t_batch3d_fp(b2t_batch3d *batch, const float *vols, float *projs, int32_t mode, void *stream);
/* vols (=|+=) BP of projs for every problem (the reference's BP, default
 * weighting: cuda/3d/cone_bp.cu:55-133, par3d_bp.cu:55-120), in one
 * persistent launch. */
b2t_status b2t_batch3d_bp(b2t_batch3d *batch, const float *projs, float *vols, int32_t mode, void *stream);
/* vols (=|+=) A^T projs for every problem: the exact adjoint of
 * b2t_batch3d_fp (its rays walked again, each detector value scattered over
 * the texels its samples read with the same weights), for gradients; the
 * scatter's atomic sums make the last bits depend on timing.  No counterpart
 * in the reference, whose only matched backprojector is the cylindrical
 * one (cuda/3d/cone_cyl.cu:309-470).  One persistent launch (plus a clear
 * for B2T_MODE_SET). */
b2t_status b2t_batch3d_matched_bp(b2t_batch3d *batch, const float *projs, float *vols, int32_t mode, void *stream);
void b2t_batch3d_destroy(b2t_batch3d *batch);

/* ---------------------------------------------------------------------- */
/* measurement and tuning                                                  */
/* ---------------------------------------------------------------------- */

/* Choose the launch shape of the 3D forward projector for this problem class
 * (geometry kind, storage type, volume and detector sizes, view count,
 * supersampling) by timing every candidate on the caller's buffers: 1, 2, 4
 * or 8 consecutive views per CTA.  The choice is kept for the process and
 * used by every later b2t_fp3d of the same class (B2T_FP_VPC in the
 * environment still overrides it).  Overwrites proj with A vol; synchronises
 * the stream.  No counterpart in the reference, whose launch shapes are
 * compile-time constants (cuda/3d/cone_fp.cu:47-53).  vpc may be NULL. */
b2t_status b2t_autotune_fp3d(const b2t_geom3d *geom, const b2t_params3d *params, const void *vol, size_t vol_pitch,
                             void *proj, size_t proj_pitch, int32_t dtype, void *stream, int32_t *vpc);

/* Choose the launch shape of the TMA 3D backprojector for this problem class
 * (geometry kind, storage type, volume and detector sizes, view count) by
 * timing both on the caller's buffers: 32 or 16 voxels per thread along z
 * (the per-view set-up amortised over more voxels, or fewer slices computed
 * past the volume's depth).
 * The choice is kept for the process and used by every later b2t_bp3d (and
 * the BP of b2t_fdk) of the same class; B2T_BP_VPT in the environment still
 * overrides it.  Overwrites vol with B proj; synchronises the stream.
 * B2T_ERR_UNSUPPORTED for voxel supersampling or the matched BP, which have
 * one shape.  No counterpart in the reference, whose launch shapes are
 * compile-time constants (cuda/3d/cone_bp.cu:38-42).  vpt may be NULL. */
b2t_status b2t_autotune_bp3d(const b2t_geom3d *geom, const b2t_params3d *params, const void *proj, size_t proj_pitch,
                             void *vol, size_t vol_pitch, int32_t dtype, void *stream, int32_t *vpt);

/* On-chip load bandwidth of the current GPU in GB/s (no counterpart in the
 * reference): which = 0 streams 16-byte shared-memory loads, which = 1
 * streams 16-byte global loads that hit L1.  The projectors' interpolation
 * reads are bound by this roof rather than by HBM.  Synchronous; allocates
 * nothing. */
b2t_status b2t_onchip_peak(int32_t which, double *gbs);

#ifdef __cplusplus
}
#endif

#endif /* B2TOMO_H */
