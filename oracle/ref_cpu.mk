# Builds the reference ASTRA Toolbox's CPU-only configuration (its host
# sources without ASTRA_CUDA, the object list of its own build's BASE_OBJECTS,
# build/linux/Makefile.in) plus ref_cpu_wrap.cpp into
# _ref/libastra_ref_cpu.so.  Test infrastructure only: the product never links
# it.  Outputs go to _ref/ (git-ignored).
#   make -f ref_cpu.mk REF=/path/to/astra-toolbox -j8
ifeq ($(REF),)
$(error REF=<reference source tree> is required)
endif
OUT = _ref
BASE = Algorithm ReconstructionAlgorithm2D ReconstructionAlgorithm3D ArtAlgorithm AstraObjectFactory \
  AstraObjectManager BackProjectionAlgorithm CglsAlgorithm CompositeGeometryManager ConeProjectionGeometry3D \
  ConeVecProjectionGeometry3D CylConeVecProjectionGeometry3D Config Data2D Data3D DataProjector \
  DataProjectorPolicies FanFlatBeamLineKernelProjector2D FanFlatBeamStripKernelProjector2D \
  FanFlatProjectionGeometry2D FanFlatVecProjectionGeometry2D Features FilteredBackProjectionAlgorithm Filters \
  ForwardProjectionAlgorithm Fourier GeometryUtil2D GeometryUtil3D Globals Logging \
  ParallelBeamBlobKernelProjector2D ParallelBeamDistanceDrivenProjector2D ParallelBeamLinearKernelProjector2D \
  ParallelBeamLineKernelProjector2D ParallelBeamStripKernelProjector2D ParallelProjectionGeometry2D \
  ParallelVecProjectionGeometry2D ParallelProjectionGeometry3D ParallelVecProjectionGeometry3D \
  PluginAlgorithmFactory ProjectionGeometry2D ProjectionGeometry2DFactory ProjectionGeometry3D \
  ProjectionGeometry3DFactory Projector2D Projector3D SartAlgorithm SheppLogan SirtAlgorithm \
  SparseMatrixProjectionGeometry2D SparseMatrixProjector2D SparseMatrix Utilities VolumeGeometry2D \
  VolumeGeometry3D XMLConfig XMLDocument XMLNode
OBJS = $(patsubst %,$(OUT)/objcpu/%.o,$(BASE)) $(OUT)/objcpu/ref_cpu_wrap.o
CXXFLAGS = -O2 -fPIC -std=c++17 -w -I$(REF)/include -I$(REF)/lib/include

all: $(OUT)/libastra_ref_cpu.so

$(OUT)/objcpu/%.o: $(REF)/src/%.cpp
	@mkdir -p $(dir $@)
	g++ $(CXXFLAGS) -c $< -o $@

$(OUT)/objcpu/ref_cpu_wrap.o: ref_cpu_wrap.cpp
	@mkdir -p $(dir $@)
	g++ $(CXXFLAGS) -c $< -o $@

$(OUT)/libastra_ref_cpu.so: $(OBJS)
	g++ -shared -o $@ $(OBJS) -lpthread

clean:
	rm -rf $(OUT)/objcpu $(OUT)/libastra_ref_cpu.so

.PHONY: all clean
