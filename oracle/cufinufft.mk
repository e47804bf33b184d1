# Builds the reference's own cuFINUFFT (vendored in thatstar/sqcalc under
# external/finufft) for sm_100a, straight from its sources, into
# oracle/_ref/libcufinufft.so.  TEST AND BASELINE INFRASTRUCTURE ONLY: the
# benchmark's reference-bar leg times it next to this library's type-1 entry
# points; the product never links or calls it.
#
#   make -C oracle -f cufinufft.mk REF=<path of the sqcalc checkout> [-j8]
#
# Sources: the cuFINUFFT list of external/finufft/src/cuda/CMakeLists.txt
# (precision-independent + 1d/2d/3d wrappers + plan/memtransfer/deconvolve/
# common) and the CPU kernel-parameter helpers it calls (external/finufft/src/
# common/{kernel,utils,pswf}.cpp).  Flags as that CMakeLists sets them
# (C++17, --extended-lambda, --extra-device-vectorization), default symbol
# visibility so the C entry points of include/cufinufft.h are exported.
ifndef REF
$(error REF=<path of the sqcalc checkout> is required)
endif
FI := $(REF)/external/finufft
OUT := _ref
OBJ := $(OUT)/cufinufft_obj
NVCC ?= $(firstword $(wildcard /usr/local/cuda/bin/nvcc) nvcc)
CXX := $(firstword $(wildcard /usr/bin/g++) g++)
ARCH := -gencode arch=compute_100a,code=sm_100a
NVFLAGS := -O3 -std=c++17 $(ARCH) --extended-lambda --extra-device-vectorization \
           -Xcompiler -fPIC -ccbin $(CXX) -I$(FI)/include -w
CXXFLAGS := -O3 -std=c++17 -fPIC -I$(FI)/include -I/usr/local/cuda/include -w

# 1d/spread1d_wrapper.cu crashes the CUDA 12.9 device front end for sm_100a
# (cicc segmentation fault); cufinufft_no1d.cu stands in for its entry points.
CU := precision_independent.cu 1d/cufinufft1d.cu 1d/interp1d_wrapper.cu \
      2d/cufinufft2d.cu 2d/spread2d_wrapper.cu 2d/interp2d_wrapper.cu \
      3d/spread3d_wrapper.cu 3d/interp3d_wrapper.cu 3d/cufinufft3d.cu \
      memtransfer_wrapper.cu deconvolve_wrapper.cu cufinufft.cu common.cu
CUOBJ := $(addprefix $(OBJ)/,$(subst /,_,$(CU:.cu=.o)))
CPPOBJ := $(OBJ)/spreadinterp_cpp.o $(OBJ)/common_kernel.o $(OBJ)/common_utils.o \
          $(OBJ)/common_pswf.o $(OBJ)/no1d.o

all: $(OUT)/libcufinufft.so

$(OBJ):
	mkdir -p $(OBJ)

$(OBJ)/1d_%.o: $(FI)/src/cuda/1d/%.cu | $(OBJ)
	$(NVCC) $(NVFLAGS) -dc -o $@ $<
$(OBJ)/2d_%.o: $(FI)/src/cuda/2d/%.cu | $(OBJ)
	$(NVCC) $(NVFLAGS) -dc -o $@ $<
$(OBJ)/3d_%.o: $(FI)/src/cuda/3d/%.cu | $(OBJ)
	$(NVCC) $(NVFLAGS) -dc -o $@ $<
$(OBJ)/%.o: $(FI)/src/cuda/%.cu | $(OBJ)
	$(NVCC) $(NVFLAGS) -dc -o $@ $<

$(OBJ)/no1d.o: cufinufft_no1d.cu | $(OBJ)
	$(NVCC) $(NVFLAGS) -dc -o $@ $<
$(OBJ)/spreadinterp_cpp.o: | $(OBJ)
	$(CXX) $(CXXFLAGS) -c -o $@ $(FI)/src/cuda/spreadinterp.cpp
$(OBJ)/common_%.o: | $(OBJ)
	$(CXX) $(CXXFLAGS) -c -o $@ $(FI)/src/common/$*.cpp

$(OUT)/libcufinufft.so: $(CUOBJ) $(CPPOBJ)
	$(NVCC) $(ARCH) -rdc=true -shared -Xcompiler -fPIC -ccbin $(CXX) -o $@ $^ -L/usr/local/cuda/lib64 \
	    -lcufft -lcudart -Xlinker -rpath=/usr/local/cuda/lib64

clean:
	rm -rf $(OBJ) $(OUT)/libcufinufft.so

.PHONY: all clean
