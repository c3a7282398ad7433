// ref_shim.cu -- the reference's cuda/3d projector entry points implemented on
// libb2tomo: the integration a maintainer makes when dropping
// cuda/3d/{cone,par3d}_{fp,bp}.cu from the reference's build.  Compiled
// against the reference's own headers and linked with its unchanged host
// sources and remaining CUDA files by oracle/ref_shim.mk into
// oracle/_ref/libastra_ref_shim.so, so that the tests run the reference's
// CompositeGeometryManager (astraCUDA3d::FP / BP dispatch, cuda/3d/mem3d.cu:
// 338-484), its FDK (cuda/3d/fdk.cu, whose BP lands here) and its algorithm
// objects on top of the library.
//
// TEST INFRASTRUCTURE ONLY: nothing in astra-toolbox_b200 links this.
//
// Replaced (declarations in include/astra/cuda/3d/):
//   ConeFP, ConeFP_Array                cone_fp.h:33-41
//   ConeBP, ConeBP_Array                cone_bp.h:33-41
//   Par3DFP, Par3DFP_Array, Par3DFP_SumSqW  par3d_fp.h:33-46
//   Par3DBP, Par3DBP_Array              par3d_bp.h:33-41
#include <cstddef>

#include "astra/cuda/gpu_runtime_wrapper.h"
#include "astra/GeometryUtil3D.h"
#include "astra/Logging.h"
// dims3d.h first: the projector headers use its names
#include "astra/cuda/3d/dims3d.h"
#include "astra/cuda/3d/cone_bp.h"
#include "astra/cuda/3d/cone_fp.h"
#include "astra/cuda/3d/par3d_bp.h"
#include "astra/cuda/3d/par3d_fp.h"
#include "b2tomo.h"

// The geometry structs cross the boundary by pointer: the layouts must be
// the same.
static_assert(sizeof(astra::SConeProjection) == sizeof(b2t_view3d), "SConeProjection size");
static_assert(offsetof(astra::SConeProjection, fSrcX) == offsetof(b2t_view3d, src), "SConeProjection src");
static_assert(offsetof(astra::SConeProjection, fDetSX) == offsetof(b2t_view3d, det_s), "SConeProjection det_s");
static_assert(offsetof(astra::SConeProjection, fDetUX) == offsetof(b2t_view3d, det_u), "SConeProjection det_u");
static_assert(offsetof(astra::SConeProjection, fDetVX) == offsetof(b2t_view3d, det_v), "SConeProjection det_v");
static_assert(sizeof(astra::SPar3DProjection) == sizeof(b2t_view3d), "SPar3DProjection size");
static_assert(offsetof(astra::SPar3DProjection, fRayX) == offsetof(b2t_view3d, src), "SPar3DProjection ray");
static_assert(offsetof(astra::SPar3DProjection, fDetSX) == offsetof(b2t_view3d, det_s), "SPar3DProjection det_s");
static_assert(offsetof(astra::SPar3DProjection, fDetUX) == offsetof(b2t_view3d, det_u), "SPar3DProjection det_u");
static_assert(offsetof(astra::SPar3DProjection, fDetVX) == offsetof(b2t_view3d, det_v), "SPar3DProjection det_v");
static_assert(sizeof(astra::SDimensions3D) == sizeof(b2t_dims3d), "SDimensions3D size");
static_assert(offsetof(astra::SDimensions3D, iVolX) == offsetof(b2t_dims3d, vol_x), "iVolX");
static_assert(offsetof(astra::SDimensions3D, iVolY) == offsetof(b2t_dims3d, vol_y), "iVolY");
static_assert(offsetof(astra::SDimensions3D, iVolZ) == offsetof(b2t_dims3d, vol_z), "iVolZ");
static_assert(offsetof(astra::SDimensions3D, iProjAngles) == offsetof(b2t_dims3d, angles), "iProjAngles");
static_assert(offsetof(astra::SDimensions3D, iProjU) == offsetof(b2t_dims3d, det_u), "iProjU");
static_assert(offsetof(astra::SDimensions3D, iProjV) == offsetof(b2t_dims3d, det_v), "iProjV");
static_assert((int)astraCUDA3d::ker3d_default == B2T_KER_DEFAULT, "ker3d_default");
static_assert((int)astraCUDA3d::ker3d_sum_square_weights == B2T_KER_SUM_SQUARE_WEIGHTS, "sum_square_weights");
static_assert((int)astraCUDA3d::ker3d_fdk_weighting == B2T_KER_FDK_WEIGHTING, "fdk_weighting");
static_assert((int)astraCUDA3d::ker3d_2d_weighting == B2T_KER_2D_WEIGHTING, "2d_weighting");
static_assert((int)astraCUDA3d::ker3d_matched_bp == B2T_KER_MATCHED_BP, "matched_bp");

namespace astraCUDA3d {

namespace {

// A pitched pointer as the library's (pointer, row pitch in elements); the
// library's slices follow each other at row pitch x rows, so the pointer's
// ysize must be the row count.
bool pitched(const cudaPitchedPtr &p, unsigned rows, size_t &pitch_elems)
{
    if (p.pitch % sizeof(float) != 0 || (p.ysize != 0 && p.ysize != rows)) {
        ASTRA_ERROR("libb2tomo shim: unsupported pitched layout (pitch %zu, ysize %zu)", p.pitch, p.ysize);
        return false;
    }
    pitch_elems = p.pitch / sizeof(float);
    return true;
}

b2t_geom3d geom(int32_t kind, const SDimensions3D &dims, const void *views, const SProjectorParams3D &params)
{
    b2t_geom3d g;
    g.kind = kind;
    g.dims = {dims.iVolX, dims.iVolY, dims.iVolZ, dims.iProjAngles, dims.iProjU, dims.iProjV};
    g.vol_scale[0] = params.volScale.fX;
    g.vol_scale[1] = params.volScale.fY;
    g.vol_scale[2] = params.volScale.fZ;
    g.views = static_cast<const b2t_view3d *>(views);
    return g;
}

b2t_params3d prm(const SProjectorParams3D &params, int32_t kernel)
{
    return b2t_params3d{params.iRaysPerDetDim, params.iRaysPerVoxelDim, params.fOutputScale, kernel};
}

// The reference's projectors accumulate and return after their work is
// done; the library is stream-ordered, so synchronise the default stream.
bool finish(b2t_status st, const char *who)
{
    if (st != B2T_OK) {
        ASTRA_ERROR("%s: %s", who, b2t_last_error());
        return false;
    }
    return cudaStreamSynchronize(0) == cudaSuccess;
}

bool fp(int32_t kind, cudaPitchedPtr vol, cudaPitchedPtr proj, const SDimensions3D &dims, const void *views,
        const SProjectorParams3D &params, int32_t kernel, const char *who)
{
    size_t vp, pp;
    if (!pitched(vol, dims.iVolY, vp) || !pitched(proj, dims.iProjAngles, pp)) return false;
    const b2t_geom3d g = geom(kind, dims, views, params);
    const b2t_params3d p = prm(params, kernel);
    return finish(b2t_fp3d(&g, &p, vol.ptr, vp, proj.ptr, pp, B2T_F32, B2T_MODE_ADD, nullptr), who);
}

bool bp(int32_t kind, cudaPitchedPtr vol, cudaPitchedPtr proj, const SDimensions3D &dims, const void *views,
        const SProjectorParams3D &params, const char *who)
{
    size_t vp, pp;
    if (!pitched(vol, dims.iVolY, vp) || !pitched(proj, dims.iProjAngles, pp)) return false;
    const b2t_geom3d g = geom(kind, dims, views, params);
    const b2t_params3d p = prm(params, (int32_t)params.projKernel);
    return finish(b2t_bp3d(&g, &p, proj.ptr, pp, vol.ptr, vp, B2T_F32, B2T_MODE_ADD, nullptr), who);
}

// A cudaArray (the reference's texture-backed storage) copied into linear
// memory of width x rows x depth floats.
struct Linear {
    cudaPitchedPtr p{};
    bool from(cudaArray *a, unsigned width, unsigned rows, unsigned depth)
    {
        if (cudaMalloc3D(&p, make_cudaExtent(sizeof(float) * width, rows, depth)) != cudaSuccess) return false;
        cudaMemcpy3DParms c = {};
        c.srcArray = a;
        c.dstPtr = p;
        c.extent = make_cudaExtent(width, rows, depth);
        c.kind = cudaMemcpyDeviceToDevice;
        return cudaMemcpy3D(&c) == cudaSuccess;
    }
    ~Linear()
    {
        if (p.ptr) cudaFree(p.ptr);
    }
};

}  // namespace

bool ConeFP(cudaPitchedPtr D_volumeData, cudaPitchedPtr D_projData, const SDimensions3D &dims,
            const SConeProjection *angles, const SProjectorParams3D &params)
{
    return fp(B2T_GEOM_CONE, D_volumeData, D_projData, dims, angles, params, B2T_KER_DEFAULT, "ConeFP");
}

bool ConeFP_Array(cudaArray *D_volArray, cudaPitchedPtr D_projData, const SDimensions3D &dims,
                  const SConeProjection *angles, const SProjectorParams3D &params)
{
    Linear v;
    if (!v.from(D_volArray, dims.iVolX, dims.iVolY, dims.iVolZ)) return false;
    return ConeFP(v.p, D_projData, dims, angles, params);
}

bool Par3DFP(cudaPitchedPtr D_volumeData, cudaPitchedPtr D_projData, const SDimensions3D &dims,
             const SPar3DProjection *angles, const SProjectorParams3D &params)
{
    return fp(B2T_GEOM_PAR3D, D_volumeData, D_projData, dims, angles, params, B2T_KER_DEFAULT, "Par3DFP");
}

bool Par3DFP_Array(cudaArray *D_volArray, cudaPitchedPtr D_projData, const SDimensions3D &dims,
                   const SPar3DProjection *angles, const SProjectorParams3D &params)
{
    Linear v;
    if (!v.from(D_volArray, dims.iVolX, dims.iVolY, dims.iVolZ)) return false;
    return Par3DFP(v.p, D_projData, dims, angles, params);
}

bool Par3DFP_SumSqW(cudaPitchedPtr D_volumeData, cudaPitchedPtr D_projData, const SDimensions3D &dims,
                    const SPar3DProjection *angles, const SProjectorParams3D &params)
{
    return fp(B2T_GEOM_PAR3D, D_volumeData, D_projData, dims, angles, params, B2T_KER_SUM_SQUARE_WEIGHTS,
              "Par3DFP_SumSqW");
}

bool ConeBP(cudaPitchedPtr D_volumeData, cudaPitchedPtr D_projData, const SDimensions3D &dims,
            const SConeProjection *angles, const SProjectorParams3D &params)
{
    return bp(B2T_GEOM_CONE, D_volumeData, D_projData, dims, angles, params, "ConeBP");
}

bool ConeBP_Array(cudaPitchedPtr D_volumeData, cudaArray *D_projArray, const SDimensions3D &dims,
                  const SConeProjection *angles, const SProjectorParams3D &params)
{
    Linear p;
    if (!p.from(D_projArray, dims.iProjU, dims.iProjAngles, dims.iProjV)) return false;
    return ConeBP(D_volumeData, p.p, dims, angles, params);
}

bool Par3DBP(cudaPitchedPtr D_volumeData, cudaPitchedPtr D_projData, const SDimensions3D &dims,
             const SPar3DProjection *angles, const SProjectorParams3D &params)
{
    return bp(B2T_GEOM_PAR3D, D_volumeData, D_projData, dims, angles, params, "Par3DBP");
}

bool Par3DBP_Array(cudaPitchedPtr D_volumeData, cudaArray *D_projArray, const SDimensions3D &dims,
                   const SPar3DProjection *angles, const SProjectorParams3D &params)
{
    Linear p;
    if (!p.from(D_projArray, dims.iProjU, dims.iProjAngles, dims.iProjV)) return false;
    return Par3DBP(D_volumeData, p.p, dims, angles, params);
}

}  // namespace astraCUDA3d
