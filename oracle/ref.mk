# TEST INFRASTRUCTURE: the reference's own solver, compiled from its sources for sm_100a so that
# it runs on the B200 beside this build (GPU parity of its operators, its step time). Outputs go
# only to oracle/_ref/ (not committed). The flags are those the reference's Makefile uses
# (-O3 -use_fast_math -lineinfo --extended-lambda, libcufft), with HDF5 off (libhdf5 is not in
# this image):
#   _ref/nse2d_ref           the solver (src/*.cu, -DNO_HDF5)
#   _ref/nse2d_ref_freeslip  the same with -DFREE_SLIP_WALLS (its WALLS=freeslip build)
#   _ref/libnse2d_ref.so     the operators and the C-linkage test API (-DEXPORT_TEST_API
#                            -DNSE2D_BUILD_AS_LIB, src/test_api.cu)
#   _ref/libnse2d_refloop.so the reference's time loop driven through its own launchers
#                            (ref_loop.cu, this directory), for field parity on seeded inputs
# make -f ref.mk REF=/path/to/reference; without REF: $(NSE2D_REFERENCE_DIR), else the directory
# "reference" beside this repository
REF   ?= $(if $(NSE2D_REFERENCE_DIR),$(NSE2D_REFERENCE_DIR),$(abspath $(CURDIR)/../../reference))
NVCC  ?= /usr/local/cuda/bin/nvcc
OUT   := _ref
SRCS  := $(addprefix $(REF)/src/,io.cu grid.cu ops.cu diag.cu poisson.cu init.cu main.cu)
FLAGS := --extended-lambda -O3 -use_fast_math -lineinfo -std=c++17 -gencode arch=compute_100a,code=sm_100a -DNO_HDF5
LIBS  := -lcufft

all: $(OUT)/nse2d_ref $(OUT)/nse2d_ref_freeslip $(OUT)/libnse2d_ref.so $(OUT)/libnse2d_refloop.so

$(OUT):
	mkdir -p $(OUT)

$(OUT)/nse2d_ref: $(SRCS) | $(OUT)
	$(NVCC) $(FLAGS) $(SRCS) $(LIBS) -o $@

$(OUT)/nse2d_ref_freeslip: $(SRCS) | $(OUT)
	$(NVCC) $(FLAGS) -DFREE_SLIP_WALLS $(SRCS) $(LIBS) -o $@

$(OUT)/libnse2d_ref.so: $(SRCS) $(REF)/src/test_api.cu | $(OUT)
	$(NVCC) $(FLAGS) -DEXPORT_TEST_API -DNSE2D_BUILD_AS_LIB -Xcompiler -fPIC -shared $(SRCS) $(REF)/src/test_api.cu $(LIBS) -o $@

$(OUT)/libnse2d_refloop.so: ref_loop.cu $(SRCS) | $(OUT)
	$(NVCC) $(FLAGS) -DNSE2D_BUILD_AS_LIB -I$(REF)/src -Xcompiler -fPIC -shared ref_loop.cu $(SRCS) $(LIBS) -o $@

.PHONY: all
