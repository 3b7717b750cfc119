# Host (CPU) build of the reference's legacy Baseline search body,
# plugins/GPUWorkerBaseline.cu lines 21-206 (binarySearchGeq, reduceEarlyIdx,
# TMotifMatching_NextMatch, MotifMatching_dispatch), compiled where it lies in
# the reference tree through a macro shim (ref_shim.h): __device__/__global__
# become host functions, a loop over root ids replaces the CUDA grid, and
# atomicAdd becomes a relaxed atomic add.  Nothing is copied into the
# repository: the extracted lines go to $(OUT) (git-ignored) only.
REF ?= $(EVX_REFERENCE_ROOT)
ifeq ($(strip $(REF)),)
$(error set EVX_REFERENCE_ROOT (or REF=) to the reference checkout)
endif
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
OUT ?= $(HERE)_ref
SRC := $(REF)/plugins/GPUWorkerBaseline.cu

$(OUT)/libref_baseline.so: $(SRC) $(HERE)ref_shim.h $(HERE)ref_driver.cc
	mkdir -p $(OUT)
	sed -n '21,206p' $(SRC) > $(OUT)/baseline_body.inc
	head -1 $(OUT)/baseline_body.inc | grep -q 'binarySearchGeq'
	grep -q 'EXITKERNEL:' $(OUT)/baseline_body.inc
	tail -1 $(OUT)/baseline_body.inc | grep -q '^}'
	g++ -O3 -march=x86-64-v2 -fopenmp -fPIC -shared -std=c++17 -I$(OUT) -I$(HERE) \
	    -o $@ $(HERE)ref_driver.cc

# Device build of the same kernel body for sm_100a (a parity and speed
# comparator for the GPU tests; never linked by the product).
$(OUT)/libref_baseline_gpu.so: $(OUT)/libref_baseline.so $(HERE)ref_gpu_driver.cu
	nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Xcompiler -fPIC -shared \
	    -I$(OUT) -o $@ $(HERE)ref_gpu_driver.cu
