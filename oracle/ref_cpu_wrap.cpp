// ref_cpu_wrap.cpp -- extern "C" entry points into the reference ASTRA
// Toolbox's CPU 2D path, built from its own sources without CUDA by
// oracle/ref_cpu.mk into oracle/_ref/libastra_ref_cpu.so.
//
// TEST INFRASTRUCTURE ONLY: the tests compare the library's 2D CUDA
// projectors with the reference's CPU projectors, and bench.py times the
// reference's CPU path on the host cores.  Nothing in astra-toolbox_b200
// links or calls this.
//
// Called reference classes (all single-threaded CPU code):
//   CParallelBeamLineKernelProjector2D     src/ParallelBeamLineKernelProjector2D.cpp
//   CParallelBeamLinearKernelProjector2D   src/ParallelBeamLinearKernelProjector2D.cpp
//   CParallelBeamStripKernelProjector2D    src/ParallelBeamStripKernelProjector2D.cpp
//   CFanFlatBeamLineKernelProjector2D      src/FanFlatBeamLineKernelProjector2D.cpp
//   CFanFlatBeamStripKernelProjector2D     src/FanFlatBeamStripKernelProjector2D.cpp
//   CForwardProjectionAlgorithm / CBackProjectionAlgorithm / CSirtAlgorithm
//                                          src/ForwardProjectionAlgorithm.cpp,
//                                          BackProjectionAlgorithm.cpp, SirtAlgorithm.cpp
#include <cstring>
#include <memory>
#include <vector>

#include "astra/BackProjectionAlgorithm.h"
#include "astra/Data2D.h"
#include "astra/FanFlatBeamLineKernelProjector2D.h"
#include "astra/FanFlatBeamStripKernelProjector2D.h"
#include "astra/FanFlatProjectionGeometry2D.h"
#include "astra/ForwardProjectionAlgorithm.h"
#include "astra/ParallelBeamLineKernelProjector2D.h"
#include "astra/ParallelBeamLinearKernelProjector2D.h"
#include "astra/ParallelBeamStripKernelProjector2D.h"
#include "astra/ParallelProjectionGeometry2D.h"
#include "astra/SirtAlgorithm.h"
#include "astra/VolumeGeometry2D.h"

using namespace astra;

namespace {

// geom 0: parallel, 1: fanflat; kernel 0: line, 1: linear (parallel only), 2: strip
struct Problem {
    std::unique_ptr<CVolumeGeometry2D> vg;
    std::unique_ptr<CProjectionGeometry2D> pg;
    std::unique_ptr<CProjector2D> proj;
    std::unique_ptr<CFloat32VolumeData2D> vol;
    std::unique_ptr<CFloat32ProjectionData2D> sino;

    bool make(int geom, int kernel, int cols, int rows, int na, int ndet, float det_width, const float *angles,
              float sod, float odd)
    {
        vg.reset(new CVolumeGeometry2D(cols, rows));
        std::vector<float32> ang(angles, angles + na);
        if (geom == 0) {
            auto *p = new CParallelProjectionGeometry2D(na, ndet, det_width, std::move(ang));
            pg.reset(p);
            if (kernel == 0) proj.reset(new CParallelBeamLineKernelProjector2D(*p, *vg));
            else if (kernel == 1) proj.reset(new CParallelBeamLinearKernelProjector2D(*p, *vg));
            else if (kernel == 2) proj.reset(new CParallelBeamStripKernelProjector2D(*p, *vg));
            else return false;
        } else if (geom == 1) {
            auto *p = new CFanFlatProjectionGeometry2D(na, ndet, det_width, std::move(ang), sod, odd);
            pg.reset(p);
            if (kernel == 0) proj.reset(new CFanFlatBeamLineKernelProjector2D(*p, *vg));
            else if (kernel == 2) proj.reset(new CFanFlatBeamStripKernelProjector2D(*p, *vg));
            else return false;
        } else {
            return false;
        }
        vol.reset(createCFloat32VolumeData2DMemory(*vg));
        sino.reset(createCFloat32ProjectionData2DMemory(*pg));
        return vol && sino && proj->isInitialized();
    }
    size_t nvol() const { return (size_t)vg->getGridTotCount(); }
    size_t nsino() const { return (size_t)pg->getProjectionAngleCount() * pg->getDetectorCount(); }
};

}  // namespace

extern "C" {

// sino [na][ndet] = FP of vol [rows][cols]
int refcpu_fp2d(int geom, int kernel, int cols, int rows, int na, int ndet, float det_width, const float *angles,
                float sod, float odd, const float *vol, float *sino)
{
    Problem P;
    if (!P.make(geom, kernel, cols, rows, na, ndet, det_width, angles, sod, odd)) return 1;
    std::memcpy(P.vol->getFloat32Memory(), vol, sizeof(float) * P.nvol());
    CForwardProjectionAlgorithm alg(P.proj.get(), P.vol.get(), P.sino.get());
    if (!alg.isInitialized() || !alg.run()) return 2;
    std::memcpy(sino, P.sino->getFloat32Memory(), sizeof(float) * P.nsino());
    return 0;
}

// vol [rows][cols] = BP of sino [na][ndet]
int refcpu_bp2d(int geom, int kernel, int cols, int rows, int na, int ndet, float det_width, const float *angles,
                float sod, float odd, const float *sino, float *vol)
{
    Problem P;
    if (!P.make(geom, kernel, cols, rows, na, ndet, det_width, angles, sod, odd)) return 1;
    std::memcpy(P.sino->getFloat32Memory(), sino, sizeof(float) * P.nsino());
    CBackProjectionAlgorithm alg;
    if (!alg.initialize(P.proj.get(), P.sino.get(), P.vol.get()) || !alg.run()) return 2;
    std::memcpy(vol, P.vol->getFloat32Memory(), sizeof(float) * P.nvol());
    return 0;
}

// vol [rows][cols]: SIRT iterations on sino, starting from vol's content
int refcpu_sirt2d(int geom, int kernel, int cols, int rows, int na, int ndet, float det_width, const float *angles,
                  float sod, float odd, const float *sino, float *vol, int iterations)
{
    Problem P;
    if (!P.make(geom, kernel, cols, rows, na, ndet, det_width, angles, sod, odd)) return 1;
    std::memcpy(P.sino->getFloat32Memory(), sino, sizeof(float) * P.nsino());
    std::memcpy(P.vol->getFloat32Memory(), vol, sizeof(float) * P.nvol());
    CSirtAlgorithm alg;
    if (!alg.initialize(P.proj.get(), P.sino.get(), P.vol.get()) || !alg.run(iterations)) return 2;
    std::memcpy(vol, P.vol->getFloat32Memory(), sizeof(float) * P.nvol());
    return 0;
}

}  // extern "C"
