# Builds the reference's own programs from their sources where they lie, into
# oracle/_ref/ (git-ignored; travels with the tree to the GPU host).
#
#   make -f oracle/ref.mk REF=<reference checkout>
#
# hot-path binaries (the reference's dump/timing driver, cuda_native_impl/benchmark.cu):
#   ref_h64  cuda_native_impl/{benchmark.cu,hydro-cal-src}                  variant H, fp64
#   ref_f64  cuda_native_impl/baselines/native_cuda_v0/fp64/...             variant F, fp64
#   ref_h32  cuda_native_impl/fp32_src/...                                  variant H, fp32
#   ref_f32  cuda_native_impl/baselines/native_cuda_v0/fp32/...             variant F, fp32
# with the flags of each tree's build.sh (-O3 -rdc=true, default fmad; only
# fp32_src/build.sh adds --fmad=false) and -arch=sm_100a in place of sm_80.
#
# CPU solver: hydro-cal-fortan/calculate.cpp, g++ -O3.
#   calculate       no source change; reads ./origin/changjiangkou/ relative
#                   to its working directory.
#   calculate_open  the same source with the documented minimal patch applied
#                   by oracle/calc_patch.sed to a copy under oracle/_ref/ (the
#                   reference tree is never written): the discharge series
#                   buffers are sized before they are filled and the day-table
#                   indices are put in [cell][day] order with the last day
#                   clamped, so decks with open boundaries (NQ, NZ > 0) run
#                   without undefined behaviour.
ifndef REF
$(error REF is not set: make -f oracle/ref.mk REF=<reference checkout>)
endif
OUT := $(dir $(lastword $(MAKEFILE_LIST)))_ref
HERE := $(dir $(lastword $(MAKEFILE_LIST)))
NVCC ?= nvcc
ARCH ?= sm_100a
CNI := $(REF)/cuda_native_impl

define ref_bin
$(OUT)/$(1): $$(wildcard $(2)/benchmark.cu $(2)/hydro-cal-src/src/* $(2)/hydro-cal-src/include/*.hpp $(2)/hydro-cal-src/include/*/*.hpp)
	@mkdir -p $(OUT)
	$(NVCC) -O3 -arch=$(ARCH) -rdc=true --std=c++17 $(3) -I$(2)/hydro-cal-src/include \
	    $(2)/benchmark.cu $(2)/hydro-cal-src/src/functors.cu $(2)/hydro-cal-src/src/mesh.cpp \
	    $(2)/hydro-cal-src/src/cell.cpp $(2)/hydro-cal-src/src/side.cpp -o $$@ -lcudadevrt
endef

all: $(OUT)/ref_h64 $(OUT)/ref_f64 $(OUT)/ref_h32 $(OUT)/ref_f32 $(OUT)/ref_dropin $(OUT)/calculate $(OUT)/calculate_open

$(eval $(call ref_bin,ref_h64,$(CNI),))
$(eval $(call ref_bin,ref_f64,$(CNI)/baselines/native_cuda_v0/fp64,))
$(eval $(call ref_bin,ref_h32,$(CNI)/fp32_src,--fmad=false))
$(eval $(call ref_bin,ref_f32,$(CNI)/baselines/native_cuda_v0/fp32,))

# The link-level drop-in: the reference's own driver and host code
# (benchmark.cu, mesh.cpp, cell.cpp, side.cpp) built exactly as build.sh builds
# them but with functors.cu left out, linked against libhydrob200.so, which
# exports CalculateFlux / UpdateCell with the reference's mangled names
# (functors.cuh:59-65).  The library is found next to the tree at run time.
LIBDIR := $(abspath $(HERE)../hydro-bench_b200/hydrob200)
$(OUT)/ref_dropin: $(CNI)/benchmark.cu $(LIBDIR)/libhydrob200.so
	@mkdir -p $(OUT)
	$(NVCC) -O3 -arch=$(ARCH) -rdc=true --std=c++17 -I$(CNI)/hydro-cal-src/include \
	    $(CNI)/benchmark.cu $(CNI)/hydro-cal-src/src/mesh.cpp $(CNI)/hydro-cal-src/src/cell.cpp \
	    $(CNI)/hydro-cal-src/src/side.cpp -L$(LIBDIR) -lhydrob200 \
	    -Xlinker -rpath='$$ORIGIN/../../hydro-bench_b200/hydrob200' -o $@ -lcudadevrt

$(OUT)/calculate: $(REF)/hydro-cal-fortan/calculate.cpp
	@mkdir -p $(OUT)
	g++ -O3 -std=c++17 -w -I$(REF)/hydro-cal-fortan $< -o $@

$(OUT)/calculate_open: $(REF)/hydro-cal-fortan/calculate.cpp $(HERE)calc_patch.sed
	@mkdir -p $(OUT)
	sed -f $(HERE)calc_patch.sed $< | g++ -O3 -std=c++17 -w -I$(REF)/hydro-cal-fortan -x c++ - -o $@

.PHONY: all
