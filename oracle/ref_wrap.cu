// ref_wrap.cu -- extern "C" entry points into the reference ASTRA Toolbox,
// built from its own sources by oracle/ref.mk into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY.  These wrappers let the tests (and the reference
// leg of bench.py) call the reference's geometry conversion, its CUDA
// projectors and its FDK on the same inputs as libb2tomo.  Nothing in
// astra-toolbox_b200 links or calls this.
//
// Called reference functions:
//   astra::convertAstraGeometry      src/GeometryUtil3D.cpp:754, GeometryUtil2D.cpp:357
//   astraCUDA3d::ConeFP / Par3DFP    cuda/3d/cone_fp.cu:444, par3d_fp.cu:564
//   astraCUDA3d::Par3DFP_SumSqW      cuda/3d/par3d_fp.cu:607
//   astraCUDA3d::ConeCylFP / ConeCylBP / ConeCylBP_matched
//                                    cuda/3d/cone_cyl.cu:622,724, cone_cyl_bp.cu:300
//   astraCUDA3d::ConeBP / Par3DBP    cuda/3d/cone_bp.cu:380, par3d_bp.cu:318
//   astraCUDA3d::FDK                 cuda/3d/fdk.cu:415
//   astraCUDA::FP / FanFP            cuda/2d/par_fp.cu:340, fan_fp.cu:260
//   astraCUDA::BP / FanBP            cuda/2d/par_bp.cu:224, fan_bp.cu:380
//   astra::CCudaSartAlgorithm        src/CudaSartAlgorithm.cpp (C++ initialize: sequential
//                                    projection order, relaxation 1)
#include <cstring>
#include <memory>
#include <vector>

#include "astra/cuda/gpu_runtime_wrapper.h"
#include "astra/cuda/2d/util.h"
#include "astra/cuda/3d/util3d.h"
#include "astra/cuda/3d/dims3d.h"
#include "astra/ConeProjectionGeometry3D.h"
#include "astra/CudaSartAlgorithm.h"
#include "astra/Data2D.h"
#include "astra/ConeVecProjectionGeometry3D.h"
#include "astra/CylConeVecProjectionGeometry3D.h"
#include "astra/FanFlatProjectionGeometry2D.h"
#include "astra/FanFlatVecProjectionGeometry2D.h"
#include "astra/Filters.h"
#include "astra/GeometryUtil2D.h"
#include "astra/GeometryUtil3D.h"
#include "astra/ParallelProjectionGeometry2D.h"
#include "astra/ParallelProjectionGeometry3D.h"
#include "astra/ParallelVecProjectionGeometry2D.h"
#include "astra/ParallelVecProjectionGeometry3D.h"
#include "astra/VolumeGeometry2D.h"
#include "astra/VolumeGeometry3D.h"
#include "astra/cuda/2d/fan_bp.h"
#include "astra/cuda/2d/fan_fp.h"
#include "astra/cuda/2d/par_bp.h"
#include "astra/cuda/2d/par_fp.h"
#include "astra/cuda/3d/cone_bp.h"
#include "astra/cuda/3d/cone_cyl.h"
#include "astra/cuda/3d/cone_fp.h"
#include "astra/cuda/3d/dims3d.h"
#include "astra/cuda/3d/fdk.h"
#include "astra/cuda/3d/par3d_bp.h"
#include "astra/cuda/3d/par3d_fp.h"
#include "astra/cuda/3d/mem3d.h"
#include "astra/CompositeGeometryManager.h"
#include "astra/CudaCglsAlgorithm3D.h"
#include "astra/CudaFDKAlgorithm3D.h"
#include "astra/CudaProjector3D.h"
#include "astra/CudaSirtAlgorithm3D.h"
#include "astra/Data3D.h"

using namespace astra;

namespace {

void copy_cone(const SConeProjection &p, double *o)
{
    const double v[12] = {p.fSrcX, p.fSrcY, p.fSrcZ, p.fDetSX, p.fDetSY, p.fDetSZ,
                          p.fDetUX, p.fDetUY, p.fDetUZ, p.fDetVX, p.fDetVY, p.fDetVZ};
    memcpy(o, v, sizeof(v));
}
void copy_cyl(const SCylConeProjection &p, double *o)
{
    const double v[13] = {p.fSrcX, p.fSrcY, p.fSrcZ, p.fDetCX, p.fDetCY, p.fDetCZ, p.fDetUX, p.fDetUY,
                          p.fDetUZ, p.fDetVX, p.fDetVY, p.fDetVZ, p.fDetR};
    std::memcpy(o, v, sizeof(v));
}

SCylConeProjection to_cyl(const double *d)
{
    SCylConeProjection p;
    p.fSrcX = d[0]; p.fSrcY = d[1]; p.fSrcZ = d[2];
    p.fDetCX = d[3]; p.fDetCY = d[4]; p.fDetCZ = d[5];
    p.fDetUX = d[6]; p.fDetUY = d[7]; p.fDetUZ = d[8];
    p.fDetVX = d[9]; p.fDetVY = d[10]; p.fDetVZ = d[11];
    p.fDetR = d[12];
    return p;
}

void copy_par(const SPar3DProjection &p, double *o)
{
    const double v[12] = {p.fRayX, p.fRayY, p.fRayZ, p.fDetSX, p.fDetSY, p.fDetSZ,
                          p.fDetUX, p.fDetUY, p.fDetUZ, p.fDetVX, p.fDetVY, p.fDetVZ};
    memcpy(o, v, sizeof(v));
}
SConeProjection to_cone(const double *o)
{
    SConeProjection p;
    p.fSrcX = o[0]; p.fSrcY = o[1]; p.fSrcZ = o[2];
    p.fDetSX = o[3]; p.fDetSY = o[4]; p.fDetSZ = o[5];
    p.fDetUX = o[6]; p.fDetUY = o[7]; p.fDetUZ = o[8];
    p.fDetVX = o[9]; p.fDetVY = o[10]; p.fDetVZ = o[11];
    return p;
}
SPar3DProjection to_par(const double *o)
{
    SPar3DProjection p;
    p.fRayX = o[0]; p.fRayY = o[1]; p.fRayZ = o[2];
    p.fDetSX = o[3]; p.fDetSY = o[4]; p.fDetSZ = o[5];
    p.fDetUX = o[6]; p.fDetUY = o[7]; p.fDetUZ = o[8];
    p.fDetVX = o[9]; p.fDetVY = o[10]; p.fDetVZ = o[11];
    return p;
}
SDimensions3D dims3(int nx, int ny, int nz, int na, int nu, int nv)
{
    SDimensions3D d;
    d.iVolX = nx; d.iVolY = ny; d.iVolZ = nz;
    d.iProjAngles = na; d.iProjU = nu; d.iProjV = nv;
    return d;
}
cudaPitchedPtr pitched(const float *p, int x, int y)
{
    return make_cudaPitchedPtr((void *)p, sizeof(float) * x, x, y);
}

// The reference binds 2D data as pitched textures, which need the pitch
// alignment cudaMallocPitch provides; stage tightly packed buffers through one.
struct Pitched2D {
    float *ptr = nullptr;
    size_t pitch = 0;  // bytes
    int w = 0, h = 0;
    bool alloc(int width, int height)
    {
        w = width;
        h = height;
        return cudaMallocPitch((void **)&ptr, &pitch, sizeof(float) * width, height) == cudaSuccess;
    }
    void upload(const float *src) { cudaMemcpy2D(ptr, pitch, src, sizeof(float) * w, sizeof(float) * w, h, cudaMemcpyDeviceToDevice); }
    void download(float *dst) { cudaMemcpy2D(dst, sizeof(float) * w, ptr, pitch, sizeof(float) * w, h, cudaMemcpyDeviceToDevice); }
    unsigned elems() const { return (unsigned)(pitch / sizeof(float)); }
    ~Pitched2D() { if (ptr) cudaFree(ptr); }
};

}  // namespace

extern "C" {

// type: 0 parallel3d, 1 cone, 2 parallel3d_vec, 3 cone_vec.
// window: min_x, max_x, min_y, max_y, min_z, max_z.  vecs: (na, 12) centre-based rows.
int ref_geom3d(int type, int cols, int rows, int slices, const float *window, int na, int det_rows,
               int det_cols, float sx, float sy, const float *angles, float sod, float odd,
               const double *vecs, double *out_views, float *out_volscale)
{
    CVolumeGeometry3D vg(cols, rows, slices, window[0], window[2], window[4], window[1], window[3], window[5]);
    std::unique_ptr<CProjectionGeometry3D> pg;
    if (type == 0 || type == 1) {
        std::vector<float32> a(angles, angles + na);
        if (type == 0)
            pg.reset(new CParallelProjectionGeometry3D(na, det_rows, det_cols, sx, sy, std::move(a)));
        else
            pg.reset(new CConeProjectionGeometry3D(na, det_rows, det_cols, sx, sy, std::move(a), sod, odd));
    } else if (type == 2) {
        std::vector<SPar3DProjection> v(na);
        for (int i = 0; i < na; ++i) {
            const double *d = vecs + 12 * i;
            SPar3DProjection &p = v[i];
            p.fRayX = d[0]; p.fRayY = d[1]; p.fRayZ = d[2];
            p.fDetUX = d[6]; p.fDetUY = d[7]; p.fDetUZ = d[8];
            p.fDetVX = d[9]; p.fDetVY = d[10]; p.fDetVZ = d[11];
            p.fDetSX = d[3] - 0.5 * det_rows * p.fDetVX - 0.5 * det_cols * p.fDetUX;
            p.fDetSY = d[4] - 0.5 * det_rows * p.fDetVY - 0.5 * det_cols * p.fDetUY;
            p.fDetSZ = d[5] - 0.5 * det_rows * p.fDetVZ - 0.5 * det_cols * p.fDetUZ;
        }
        pg.reset(new CParallelVecProjectionGeometry3D(na, det_rows, det_cols, std::move(v)));
    } else if (type == 4) {
        std::vector<SCylConeProjection> v(na);
        for (int i = 0; i < na; ++i) v[i] = to_cyl(vecs + 13 * i);
        pg.reset(new CCylConeVecProjectionGeometry3D(na, det_rows, det_cols, std::move(v)));
    } else {
        std::vector<SConeProjection> v(na);
        for (int i = 0; i < na; ++i) {
            const double *d = vecs + 12 * i;
            SConeProjection &p = v[i];
            p.fSrcX = d[0]; p.fSrcY = d[1]; p.fSrcZ = d[2];
            p.fDetUX = d[6]; p.fDetUY = d[7]; p.fDetUZ = d[8];
            p.fDetVX = d[9]; p.fDetVY = d[10]; p.fDetVZ = d[11];
            p.fDetSX = d[3] - 0.5 * det_rows * p.fDetVX - 0.5 * det_cols * p.fDetUX;
            p.fDetSY = d[4] - 0.5 * det_rows * p.fDetVY - 0.5 * det_cols * p.fDetUY;
            p.fDetSZ = d[5] - 0.5 * det_rows * p.fDetVZ - 0.5 * det_cols * p.fDetUZ;
        }
        pg.reset(new CConeVecProjectionGeometry3D(na, det_rows, det_cols, std::move(v)));
    }
    Geometry3DParameters g = convertAstraGeometry(&vg, pg.get());
    if (!g.isValid()) return 1;
    for (int i = 0; i < na; ++i) {
        if (g.isCylCone()) copy_cyl(g.getCylCone()[i], out_views + 13 * i);
        else if (g.isCone()) copy_cone(g.getCone()[i], out_views + 12 * i);
        else copy_par(g.getParallel()[i], out_views + 12 * i);
    }
    out_volscale[0] = g.getVolScale().fX;
    out_volscale[1] = g.getVolScale().fY;
    out_volscale[2] = g.getVolScale().fZ;
    return 0;
}

// type: 0 parallel, 1 fanflat, 2 parallel_vec, 3 fanflat_vec.  window: min_x, max_x, min_y, max_y.
static std::unique_ptr<CProjectionGeometry2D> make_proj_geom2d(int type, int na, int ndet, float width,
                                                               const float *angles, float sod, float odd,
                                                               const double *vecs)
{
    std::unique_ptr<CProjectionGeometry2D> pg;
    if (type == 0 || type == 1) {
        std::vector<float32> a(angles, angles + na);
        if (type == 0) pg.reset(new CParallelProjectionGeometry2D(na, ndet, width, std::move(a)));
        else pg.reset(new CFanFlatProjectionGeometry2D(na, ndet, width, std::move(a), sod, odd));
    } else if (type == 2) {
        std::vector<SParProjection> v(na);
        for (int i = 0; i < na; ++i) {
            const double *d = vecs + 6 * i;
            SParProjection &p = v[i];
            p.fRayX = d[0]; p.fRayY = d[1]; p.fDetUX = d[4]; p.fDetUY = d[5];
            p.fDetSX = d[2] - 0.5 * ndet * p.fDetUX;
            p.fDetSY = d[3] - 0.5 * ndet * p.fDetUY;
        }
        pg.reset(new CParallelVecProjectionGeometry2D(na, ndet, std::move(v)));
    } else {
        std::vector<SFanProjection> v(na);
        for (int i = 0; i < na; ++i) {
            const double *d = vecs + 6 * i;
            SFanProjection &p = v[i];
            p.fSrcX = d[0]; p.fSrcY = d[1]; p.fDetUX = d[4]; p.fDetUY = d[5];
            p.fDetSX = d[2] - 0.5 * ndet * p.fDetUX;
            p.fDetSY = d[3] - 0.5 * ndet * p.fDetUY;
        }
        pg.reset(new CFanFlatVecProjectionGeometry2D(na, ndet, std::move(v)));
    }
    return pg;
}

int ref_geom2d(int type, int cols, int rows, const float *window, int na, int ndet, float width,
               const float *angles, float sod, float odd, const double *vecs, float *out_views,
               float *out_scale)
{
    CVolumeGeometry2D vg(cols, rows, window[0], window[2], window[1], window[3]);
    std::unique_ptr<CProjectionGeometry2D> pg = make_proj_geom2d(type, na, ndet, width, angles, sod, odd, vecs);
    Geometry2DParameters g = convertAstraGeometry(&vg, pg.get());
    if (!g.isValid()) return 1;
    for (int i = 0; i < na; ++i) {
        float *o = out_views + 6 * i;
        if (g.isParallel()) {
            const SParProjection &p = g.getParallel()[i];
            o[0] = p.fRayX; o[1] = p.fRayY; o[2] = p.fDetSX; o[3] = p.fDetSY; o[4] = p.fDetUX; o[5] = p.fDetUY;
        } else {
            const SFanProjection &p = g.getFan()[i];
            o[0] = p.fSrcX; o[1] = p.fSrcY; o[2] = p.fDetSX; o[3] = p.fDetSY; o[4] = p.fDetUX; o[5] = p.fDetUY;
        }
    }
    *out_scale = g.getOutputScale();
    return 0;
}

// SART_CUDA on host buffers: sino (na, ndet), vol (rows, cols) updated in
// place by `iterations` single-angle steps in sequential order.
int ref_sart2d(int type, int cols, int rows, const float *window, int na, int ndet, float width,
               const float *angles, float sod, float odd, const double *vecs, const float *sino, float *vol,
               int iterations, int use_min, float min_value, int use_max, float max_value)
{
    CVolumeGeometry2D vg(cols, rows, window[0], window[2], window[1], window[3]);
    std::unique_ptr<CProjectionGeometry2D> pg = make_proj_geom2d(type, na, ndet, width, angles, sod, odd, vecs);
    std::unique_ptr<CFloat32ProjectionData2D> S(createCFloat32ProjectionData2DMemory(*pg));
    std::unique_ptr<CFloat32VolumeData2D> V(createCFloat32VolumeData2DMemory(vg));
    std::memcpy(S->getFloat32Memory(), sino, sizeof(float) * (size_t)na * ndet);
    std::memcpy(V->getFloat32Memory(), vol, sizeof(float) * (size_t)rows * cols);
    CCudaSartAlgorithm alg;
    if (!alg.initialize(nullptr, S.get(), V.get())) return 1;
    alg.setConstraints(use_min != 0, min_value, use_max != 0, max_value);
    if (!alg.run(iterations)) return 2;
    std::memcpy(vol, V->getFloat32Memory(), sizeof(float) * (size_t)rows * cols);
    return 0;
}

// kind: 1 par3d, 2 cone (same codes as libb2tomo).  Device pointers; the
// reference accumulates into d_proj (callers zero it for SET semantics).
int ref_cuda_fp3d(int kind, const double *views, int nx, int ny, int nz, int na, int nu, int nv,
                  const float *vs, float out_scale, int rays, const float *d_vol, float *d_proj)
{
    astraCUDA3d::SProjectorParams3D params;
    params.volScale.fX = vs[0];
    params.volScale.fY = vs[1];
    params.volScale.fZ = vs[2];
    params.iRaysPerDetDim = rays;
    params.fOutputScale = out_scale;
    SDimensions3D d = dims3(nx, ny, nz, na, nu, nv);
    bool ok;
    if (kind == 2) {
        std::vector<SConeProjection> p(na);
        for (int i = 0; i < na; ++i) p[i] = to_cone(views + 12 * i);
        ok = astraCUDA3d::ConeFP(pitched(d_vol, nx, ny), pitched(d_proj, nu, na), d, &p[0], params);
    } else {
        std::vector<SPar3DProjection> p(na);
        for (int i = 0; i < na; ++i) p[i] = to_par(views + 12 * i);
        ok = astraCUDA3d::Par3DFP(pitched(d_vol, nx, ny), pitched(d_proj, nu, na), d, &p[0], params);
    }
    return ok ? 0 : 1;
}

// cyl_cone_vec projectors: op 0 ConeCylFP (d_in volume, d_out projections),
// 1 ConeCylBP, 2 ConeCylBP_matched (d_in projections, d_out volume).  views
// (na, 13) as normalised by ref_geom3d.  Accumulates into d_out.
int ref_cuda_cyl(int op, const double *views, int nx, int ny, int nz, int na, int nu, int nv, const float *vs,
                 float out_scale, const float *d_in, float *d_out)
{
    astraCUDA3d::SProjectorParams3D params;
    params.volScale.fX = vs[0];
    params.volScale.fY = vs[1];
    params.volScale.fZ = vs[2];
    params.fOutputScale = out_scale;
    SDimensions3D d = dims3(nx, ny, nz, na, nu, nv);
    std::vector<SCylConeProjection> p(na);
    for (int i = 0; i < na; ++i) p[i] = to_cyl(views + 13 * i);
    bool ok;
    if (op == 0)
        ok = astraCUDA3d::ConeCylFP(pitched(d_in, nx, ny), pitched(d_out, nu, na), d, &p[0], params);
    else if (op == 1)
        ok = astraCUDA3d::ConeCylBP(pitched(d_out, nx, ny), pitched(d_in, nu, na), d, &p[0], params);
    else
        ok = astraCUDA3d::ConeCylBP_matched(pitched(d_out, nx, ny), pitched(d_in, nu, na), d, &p[0], params);
    return ok ? 0 : 1;
}

// Par3DFP_SumSqW (cuda/3d/par3d_fp.cu:607): accumulates into d_proj; the
// volume is not read.
int ref_cuda_sumsqw(const double *views, int nx, int ny, int nz, int na, int nu, int nv, const float *vs,
                    float out_scale, float *d_proj)
{
    astraCUDA3d::SProjectorParams3D params;
    params.volScale.fX = vs[0];
    params.volScale.fY = vs[1];
    params.volScale.fZ = vs[2];
    params.iRaysPerDetDim = 1;
    params.fOutputScale = out_scale;
    params.projKernel = astraCUDA3d::ker3d_sum_square_weights;
    SDimensions3D d = dims3(nx, ny, nz, na, nu, nv);
    std::vector<SPar3DProjection> p(na);
    for (int i = 0; i < na; ++i) p[i] = to_par(views + 12 * i);
    cudaPitchedPtr none = pitched(nullptr, nx, ny);
    return astraCUDA3d::Par3DFP_SumSqW(none, pitched(d_proj, nu, na), d, &p[0], params) ? 0 : 1;
}

// kernel: 0 default, 2 fdk_weighting, 3 2d_weighting.  Accumulates into d_vol.
int ref_cuda_bp3d(int kind, int kernel, const double *views, int nx, int ny, int nz, int na, int nu, int nv,
                  const float *vs, float out_scale, int rays, const float *d_proj, float *d_vol)
{
    astraCUDA3d::SProjectorParams3D params;
    params.volScale.fX = vs[0];
    params.volScale.fY = vs[1];
    params.volScale.fZ = vs[2];
    params.iRaysPerVoxelDim = rays;
    params.fOutputScale = out_scale;
    params.projKernel = (astraCUDA3d::Cuda3DProjectionKernel)kernel;
    SDimensions3D d = dims3(nx, ny, nz, na, nu, nv);
    bool ok;
    if (kind == 2) {
        std::vector<SConeProjection> p(na);
        for (int i = 0; i < na; ++i) p[i] = to_cone(views + 12 * i);
        ok = astraCUDA3d::ConeBP(pitched(d_vol, nx, ny), pitched(d_proj, nu, na), d, &p[0], params);
    } else {
        std::vector<SPar3DProjection> p(na);
        for (int i = 0; i < na; ++i) p[i] = to_par(views + 12 * i);
        ok = astraCUDA3d::Par3DBP(pitched(d_vol, nx, ny), pitched(d_proj, nu, na), d, &p[0], params);
    }
    return ok ? 0 : 1;
}

// FDK with the Ram-Lak filter; d_proj is weighted and filtered in place and
// the result accumulated into d_vol.
int ref_cuda_fdk(const double *views, int nx, int ny, int nz, int na, int nu, int nv, const float *vs,
                 int short_scan, float out_scale, float *d_proj, float *d_vol)
{
    astraCUDA3d::SProjectorParams3D params;
    params.volScale.fX = vs[0];
    params.volScale.fY = vs[1];
    params.volScale.fZ = vs[2];
    params.fOutputScale = out_scale;
    params.projKernel = astraCUDA3d::ker3d_fdk_weighting;
    SDimensions3D d = dims3(nx, ny, nz, na, nu, nv);
    std::vector<SConeProjection> p(na);
    for (int i = 0; i < na; ++i) p[i] = to_cone(views + 12 * i);
    SFilterConfig cfg;
    cfg.m_eType = FILTER_RAMLAK;
    // The weighting kernels (devFDK_preweight, devFDK_ParkerWeight) do not
    // bound-check u and rely on the row padding of pitched allocations, so
    // the projections are staged through a cudaMallocPitch buffer as in ASTRA.
    Pitched2D P;
    if (!P.alloc(nu, na * nv)) return 2;
    P.upload(d_proj);
    cudaPitchedPtr pp = make_cudaPitchedPtr(P.ptr, P.pitch, nu, na);
    bool ok = astraCUDA3d::FDK(pitched(d_vol, nx, ny), pp, &p[0], d, params, short_scan != 0, cfg);
    P.download(d_proj);
    return ok ? 0 : 1;
}

// 2D: kind 3 parallel, 4 fan.  views: (na, 6) floats.  Accumulates.
int ref_cuda_fp2d(int kind, const float *views, int W, int H, int na, int ndet, float out_scale, int rays,
                  float *d_vol, float *d_sino)
{
    SDimensions d;
    d.iVolWidth = W; d.iVolHeight = H; d.iProjAngles = na; d.iProjDets = ndet;
    astraCUDA::SProjectorParams2D params;
    params.iRaysPerDet = rays;
    params.fOutputScale = out_scale;
    bool ok;
    if (kind == 3) {
        std::vector<SParProjection> p(na);
        for (int i = 0; i < na; ++i) {
            const float *o = views + 6 * i;
            p[i].fRayX = o[0]; p[i].fRayY = o[1]; p[i].fDetSX = o[2]; p[i].fDetSY = o[3];
            p[i].fDetUX = o[4]; p[i].fDetUY = o[5];
        }
        Pitched2D V, S;
        if (!V.alloc(W, H) || !S.alloc(ndet, na)) return 2;
        V.upload(d_vol);
        S.upload(d_sino);
        ok = astraCUDA::FP(V.ptr, V.elems(), S.ptr, S.elems(), d, params, &p[0]);
        S.download(d_sino);
    } else {
        std::vector<SFanProjection> p(na);
        for (int i = 0; i < na; ++i) {
            const float *o = views + 6 * i;
            p[i].fSrcX = o[0]; p[i].fSrcY = o[1]; p[i].fDetSX = o[2]; p[i].fDetSY = o[3];
            p[i].fDetUX = o[4]; p[i].fDetUY = o[5];
        }
        Pitched2D V, S;
        if (!V.alloc(W, H) || !S.alloc(ndet, na)) return 2;
        V.upload(d_vol);
        S.upload(d_sino);
        ok = astraCUDA::FanFP(V.ptr, V.elems(), S.ptr, S.elems(), d, params, &p[0]);
        S.download(d_sino);
    }
    return ok ? 0 : 1;
}

int ref_cuda_bp2d(int kind, const float *views, int W, int H, int na, int ndet, float out_scale, int rays,
                  int fbp, float *d_sino, float *d_vol)
{
    SDimensions d;
    d.iVolWidth = W; d.iVolHeight = H; d.iProjAngles = na; d.iProjDets = ndet;
    astraCUDA::SProjectorParams2D params;
    params.iRaysPerPixelDim = rays;
    params.fOutputScale = out_scale;
    bool ok;
    if (kind == 3) {
        std::vector<SParProjection> p(na);
        for (int i = 0; i < na; ++i) {
            const float *o = views + 6 * i;
            p[i].fRayX = o[0]; p[i].fRayY = o[1]; p[i].fDetSX = o[2]; p[i].fDetSY = o[3];
            p[i].fDetUX = o[4]; p[i].fDetUY = o[5];
        }
        Pitched2D V, S;
        if (!V.alloc(W, H) || !S.alloc(ndet, na)) return 2;
        V.upload(d_vol);
        S.upload(d_sino);
        ok = astraCUDA::BP(V.ptr, V.elems(), S.ptr, S.elems(), d, params, &p[0]);
        V.download(d_vol);
    } else {
        std::vector<SFanProjection> p(na);
        for (int i = 0; i < na; ++i) {
            const float *o = views + 6 * i;
            p[i].fSrcX = o[0]; p[i].fSrcY = o[1]; p[i].fDetSX = o[2]; p[i].fDetSY = o[3];
            p[i].fDetUX = o[4]; p[i].fDetUY = o[5];
        }
        Pitched2D V, S;
        if (!V.alloc(W, H) || !S.alloc(ndet, na)) return 2;
        V.upload(d_vol);
        S.upload(d_sino);
        if (fbp) ok = astraCUDA::FanBP_FBPWeighted(V.ptr, V.elems(), S.ptr, S.elems(), d, params, &p[0]);
        else ok = astraCUDA::FanBP(V.ptr, V.elems(), S.ptr, S.elems(), d, params, &p[0]);
        V.download(d_vol);
    }
    return ok ? 0 : 1;
}

// The reference's filter spectrum (astra::genFilter, src/Filters.cpp:131-488)
// for an FFT of N samples: writes N / 2 + 1 floats.  type = E_FBPFILTER value.
// Host code only (no GPU needed).
int ref_gen_filter(int type, float d, float parameter, int N, float *out)
{
    astra::SFilterConfig cfg;
    cfg.m_eType = (astra::E_FBPFILTER)type;
    cfg.m_fD = d;
    cfg.m_fParameter = parameter;
    const int F = astra::calcFFTFourierSize(N);
    float *f = astra::genFilter(cfg, N, F);
    if (!f) return 1;
    std::memcpy(out, f, sizeof(float) * F);
    delete[] f;
    return 0;
}

// A reference 3D algorithm object (type 0: SIRT3D_CUDA, 1: CGLS3D_CUDA,
// 2: FDK_CUDA with the Ram-Lak filter; src/CudaSirtAlgorithm3D.cpp,
// CudaCglsAlgorithm3D.cpp, CudaFDKAlgorithm3D.cpp, unchanged) for a circular
// cone geometry over caller device buffers: projections [v][angle][u],
// volume [z][y][x].  FDK takes them linked as the reference's GPU data
// (astraCUDA3d::wrapHandle, cuda/3d/mem3d.cu:521, the path its DLPack
// interface takes); SIRT3D and CGLS3D accept host-memory data only
// (CudaSirtAlgorithm3D.cpp, CudaCglsAlgorithm3D.cpp initialisation checks),
// so their projections are copied to host memory at creation and every run
// copies its result back into the device volume.
struct RefAlgo3D {
    std::unique_ptr<CConeProjectionGeometry3D> pg;
    std::unique_ptr<CVolumeGeometry3D> vg;
    std::unique_ptr<CCudaProjector3D> proj;
    std::unique_ptr<CFloat32ProjectionData3D> sino;
    std::unique_ptr<CFloat32VolumeData3D> vol;
    std::unique_ptr<CReconstructionAlgorithm3D> alg;
    float *d_vol = nullptr;  // host-memory volume: copied here after each run
    size_t vol_bytes = 0;
};

void *ref_algo3d_create(int type, int nx, int ny, int nz, int na, int nu, int nv, float du, float dv,
                        const float *angles, float sod, float odd, float *d_proj, float *d_vol)
{
    auto *h = new RefAlgo3D;
    h->pg.reset(new CConeProjectionGeometry3D(na, nv, nu, du, dv, std::vector<float32>(angles, angles + na), sod,
                                              odd));
    h->vg.reset(new CVolumeGeometry3D(nx, ny, nz));
    h->proj.reset(new CCudaProjector3D(*h->pg, *h->vg));
    if (type == 2) {
        h->sino.reset(new CFloat32ProjectionData3D(*h->pg, astraCUDA3d::wrapHandle(d_proj, nu, na, nv, nu)));
        h->vol.reset(new CFloat32VolumeData3D(*h->vg, astraCUDA3d::wrapHandle(d_vol, nx, ny, nz, nx)));
    } else {
        h->sino.reset(createCFloat32ProjectionData3DMemory(*h->pg));
        h->vol.reset(createCFloat32VolumeData3DMemory(*h->vg));
        h->vol_bytes = sizeof(float) * (size_t)nx * ny * nz;
        h->d_vol = d_vol;
        if (cudaMemcpy(h->sino->getFloat32Memory(), d_proj, sizeof(float) * (size_t)nu * na * nv,
                       cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(h->vol->getFloat32Memory(), d_vol, h->vol_bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
            delete h;
            return nullptr;
        }
    }
    if (type == 0) {
        h->alg.reset(new CCudaSirtAlgorithm3D(h->proj.get(), h->sino.get(), h->vol.get()));
    } else if (type == 1) {
        h->alg.reset(new CCudaCglsAlgorithm3D(h->proj.get(), h->sino.get(), h->vol.get()));
    } else if (type == 2) {
        SFilterConfig f;
        f.m_eType = FILTER_RAMLAK;
        h->alg.reset(new CCudaFDKAlgorithm3D(h->proj.get(), h->sino.get(), h->vol.get(), f, false));
    }
    if (!h->alg || !h->alg->isInitialized()) {
        delete h;
        return nullptr;
    }
    return h;
}

// iterations (ignored by FDK); synchronises the device
int ref_algo3d_run(void *p, int iterations)
{
    auto *h = static_cast<RefAlgo3D *>(p);
    const bool ok = h->alg->run(iterations);
    cudaDeviceSynchronize();
    if (ok && h->d_vol &&
        cudaMemcpy(h->d_vol, h->vol->getFloat32Memory(), h->vol_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return 2;
    return ok ? 0 : 1;
}

int ref_algo3d_residual(void *p, float *norm)
{
    auto *h = static_cast<RefAlgo3D *>(p);
    float32 v = 0.0f;
    if (!h->alg->getResidualNorm(v)) return 1;
    *norm = v;
    return 0;
}

void ref_algo3d_destroy(void *p) { delete static_cast<RefAlgo3D *>(p); }

// The reference's CompositeGeometryManager doFP (op 0) / doBP (op 1) in
// MODE_SET on a circular cone geometry: the path under
// astra.experimental.direct_FP3D / direct_BP3D (linked device data, gpu_data
// = 1; python/astra/experimental.pyx:172-227) and create_sino3d_gpu /
// create_backprojection3d_gpu (host data, gpu_data = 0), with the GPU memory
// limit of astra.set_gpu_index(0, memory) (0: none), under which the manager
// splits the job (src/CompositeGeometryManager.cpp:218-379).
int ref_cgm_cone(int op, int gpu_data, size_t memory, int nx, int ny, int nz, int na, int nu, int nv, float du,
                 float dv, const float *angles, float sod, float odd, float *proj, float *vol)
{
    CConeProjectionGeometry3D pg(na, nv, nu, du, dv, std::vector<float32>(angles, angles + na), sod, odd);
    CVolumeGeometry3D vg(nx, ny, nz);
    CCudaProjector3D projector(pg, vg);
    std::unique_ptr<CFloat32ProjectionData3D> P;
    std::unique_ptr<CFloat32VolumeData3D> V;
    if (gpu_data) {
        P.reset(new CFloat32ProjectionData3D(pg, astraCUDA3d::wrapHandle(proj, nu, na, nv, nu)));
        V.reset(new CFloat32VolumeData3D(vg, astraCUDA3d::wrapHandle(vol, nx, ny, nz, nx)));
    } else {
        P.reset(createCFloat32ProjectionData3DMemory(pg));
        V.reset(createCFloat32VolumeData3DMemory(vg));
        std::memcpy(op == 0 ? (void *)V->getFloat32Memory() : (void *)P->getFloat32Memory(), op == 0 ? vol : proj,
                    sizeof(float) * (op == 0 ? (size_t)nx * ny * nz : (size_t)nu * na * nv));
    }
    SGPUParams gp;
    gp.GPUIndices.push_back(0);
    gp.memory = memory;
    CCompositeGeometryManager::setGlobalGPUParams(gp);
    CCompositeGeometryManager m;
    std::vector<CFloat32VolumeData3D *> vv{V.get()};
    std::vector<CFloat32ProjectionData3D *> pv{P.get()};
    const bool ok = op == 0 ? m.doFP(&projector, vv, pv, CCompositeGeometryManager::MODE_SET)
                            : m.doBP(&projector, vv, pv, CCompositeGeometryManager::MODE_SET);
    SGPUParams none;
    none.GPUIndices.push_back(0);
    none.memory = 0;
    CCompositeGeometryManager::setGlobalGPUParams(none);
    if (!ok) return 1;
    if (!gpu_data)
        std::memcpy(op == 0 ? proj : vol, op == 0 ? (void *)P->getFloat32Memory() : (void *)V->getFloat32Memory(),
                    sizeof(float) * (op == 0 ? (size_t)nu * na * nv : (size_t)nx * ny * nz));
    cudaDeviceSynchronize();
    return 0;
}

}  // extern "C"
