# Builds the reference ASTRA Toolbox with its cuda/3d projectors replaced by
# libb2tomo: every host source and CUDA file of ref.mk except
# cuda/3d/{cone,par3d}_{fp,bp}.cu, plus ref_shim.cu (those entry points on the
# C ABI) and ref_wrap.cu, linked with astra-toolbox_b200/libb2tomo.so into
# _ref/libastra_ref_shim.so.  The integration a maintainer makes, compiled
# against the reference's own headers.  Test infrastructure only.  Objects are
# shared with ref.mk (same flags).  Run after libb2tomo.so is built.
#   make -f ref_shim.mk REF=/path/to/astra-toolbox -j8
ifeq ($(REF),)
$(error REF=<reference source tree> is required)
endif
OUT = _ref
DROP = $(REF)/cuda/3d/cone_fp.cu $(REF)/cuda/3d/cone_bp.cu $(REF)/cuda/3d/par3d_fp.cu $(REF)/cuda/3d/par3d_bp.cu
SRCS = $(wildcard $(REF)/src/*.cpp)
CUS = $(filter-out $(DROP),$(wildcard $(REF)/cuda/*.cu) $(wildcard $(REF)/cuda/2d/*.cu) $(wildcard $(REF)/cuda/3d/*.cu))
OBJS = $(patsubst $(REF)/%.cpp,$(OUT)/obj/%.o,$(SRCS)) $(patsubst $(REF)/%.cu,$(OUT)/obj/%.cu.o,$(CUS)) \
       $(OUT)/obj/ref_wrap.cu.o $(OUT)/obj/ref_shim.cu.o
DEFS = -DASTRA_CUDA -DASTRA_BUILDING_CUDA
INC = -I$(REF)/include -I$(REF)/lib/include
CXXFLAGS = -O2 -fPIC -std=c++17 -w $(DEFS) $(INC) -I/usr/local/cuda/include
NVFLAGS = -O2 -std=c++17 -w -Xcompiler -fPIC $(DEFS) $(INC) -gencode arch=compute_100a,code=sm_100a
B2T = ../astra-toolbox_b200

all: $(OUT)/libastra_ref_shim.so

$(OUT)/obj/%.o: $(REF)/%.cpp
	@mkdir -p $(dir $@)
	g++ $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/%.cu.o: $(REF)/%.cu
	@mkdir -p $(dir $@)
	nvcc $(NVFLAGS) -c $< -o $@

$(OUT)/obj/ref_wrap.cu.o: ref_wrap.cu
	@mkdir -p $(dir $@)
	nvcc $(NVFLAGS) -c $< -o $@

$(OUT)/obj/ref_shim.cu.o: ref_shim.cu ../include/b2tomo.h
	@mkdir -p $(dir $@)
	nvcc $(NVFLAGS) -I../include -c $< -o $@

$(OUT)/libastra_ref_shim.so: $(OBJS) $(B2T)/libb2tomo.so
	nvcc -shared -gencode arch=compute_100a,code=sm_100a -o $@ $(OBJS) -L$(B2T) -lb2tomo \
	    -Xlinker -rpath,'$$ORIGIN/../../astra-toolbox_b200' -lcufft -lcudart_static -lrt -lpthread -ldl

clean:
	rm -f $(OUT)/libastra_ref_shim.so $(OUT)/obj/ref_shim.cu.o

.PHONY: all clean
