# Builds the reference ASTRA Toolbox (host sources + CUDA kernels, sm_100a)
# from the read-only source tree REF, plus ref_wrap.cu, into _ref/libastra_ref.so.
# Test infrastructure only: the product never links it.  Outputs go to _ref/
# (git-ignored; the built .so travels with the repository snapshot).
#   make -f ref.mk REF=/path/to/astra-toolbox -j8
ifeq ($(REF),)
$(error REF=<reference source tree> is required)
endif
OUT = _ref
SRCS = $(wildcard $(REF)/src/*.cpp)
CUS = $(wildcard $(REF)/cuda/*.cu) $(wildcard $(REF)/cuda/2d/*.cu) $(wildcard $(REF)/cuda/3d/*.cu)
OBJS = $(patsubst $(REF)/%.cpp,$(OUT)/obj/%.o,$(SRCS)) $(patsubst $(REF)/%.cu,$(OUT)/obj/%.cu.o,$(CUS)) $(OUT)/obj/ref_wrap.cu.o
DEFS = -DASTRA_CUDA -DASTRA_BUILDING_CUDA
INC = -I$(REF)/include -I$(REF)/lib/include
CXXFLAGS = -O2 -fPIC -std=c++17 -w $(DEFS) $(INC) -I/usr/local/cuda/include
NVFLAGS = -O2 -std=c++17 -w -Xcompiler -fPIC $(DEFS) $(INC) -gencode arch=compute_100a,code=sm_100a

all: $(OUT)/libastra_ref.so

$(OUT)/obj/%.o: $(REF)/%.cpp
	@mkdir -p $(dir $@)
	g++ $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/%.cu.o: $(REF)/%.cu
	@mkdir -p $(dir $@)
	nvcc $(NVFLAGS) -c $< -o $@

$(OUT)/obj/ref_wrap.cu.o: ref_wrap.cu
	@mkdir -p $(dir $@)
	nvcc $(NVFLAGS) -c $< -o $@

$(OUT)/libastra_ref.so: $(OBJS)
	nvcc -shared -gencode arch=compute_100a,code=sm_100a -o $@ $(OBJS) -lcufft -lcudart_static -lrt -lpthread -ldl

clean:
	rm -rf $(OUT)

.PHONY: all clean
