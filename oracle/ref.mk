# Builds 3DI's own hot-path CUDA sources, unmodified, into oracle/_ref/ for pinning the oracle
# (test infrastructure only; nothing in the product links these libraries).
#
#   make -f ref.mk            (from oracle/; needs the reference checkout at $(REF))
#
# Sources compiled as they lie: src/lib/funcs.cu, newfuncs.cu, rotation_header.cu. Their
# OpenCV includes resolve to the stand-in headers of refstub/ (OpenCV is used there only in
# host display helpers that are never called). Flags: the definitions of the reference's
# src/CMakeLists.txt:1; nvcc's defaults otherwise (the reference's CMake build passes no
# maths flags to its CUDA targets), once as is (libtdi_ref.so) and once without FMA
# contraction (libtdi_ref_nofma.so), the arithmetic contract of the oracle. CUDA 12's thrust
# no longer includes <thrust/extrema.h> from the headers funcs.h names, so it is included on
# the command line.
REF ?= /root/reference/src/lib
NVCC ?= /usr/local/cuda/bin/nvcc
OUT := _ref
SRCS := $(REF)/funcs.cu $(REF)/newfuncs.cu $(REF)/rotation_header.cu ref_harness.cu
FLAGS := -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
	-DKERNEL_RADIUS=7 -DWRITE_OBJ_FILE=0 -D_IGNORE_BOUNDS=0 \
	-include thrust/extrema.h -Irefstub -I$(REF) -Xcompiler -fPIC -shared -w -lcublas
STUBS := $(wildcard refstub/opencv2/*.hpp)

all: $(OUT)/libtdi_ref.so $(OUT)/libtdi_ref_nofma.so

$(OUT)/libtdi_ref.so: $(SRCS) $(STUBS)
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -o $@ $(SRCS)

$(OUT)/libtdi_ref_nofma.so: $(SRCS) $(STUBS)
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -fmad=false -o $@ $(SRCS)

clean:
	rm -f $(OUT)/libtdi_ref.so $(OUT)/libtdi_ref_nofma.so

.PHONY: all clean
