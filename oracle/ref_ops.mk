# Builds the reference's own CUDA operators (fft, beamform, equalize) from
# the reference tree, in place, with the C shim ref_shim.cu, into
# _ref/libref_ops.so.  Test infrastructure only; nothing is copied from the
# reference tree.  Usage: make -f ref_ops.mk REF=<reference tree>
ifeq ($(REF),)
$(error REF=<MegaStation tree> is required)
endif
OPS := $(REF)/src/operators
NVCC ?= nvcc
SITE := $(shell python -c "import site; print(site.getsitepackages()[0])" 2>/dev/null)
CUTLASS ?= $(SITE)/flashinfer/data/cutlass/include
SRCS := $(OPS)/fft/fft_op.cu $(OPS)/beamform/beamform.cu $(OPS)/sgemv/equalize.cu ref_shim.cu
OUT := _ref/libref_ops.so

all: $(OUT)

$(OUT): $(SRCS)
	mkdir -p _ref
	$(NVCC) -std=c++20 -O3 -gencode arch=compute_100a,code=sm_100a --expt-relaxed-constexpr \
	  -Xcompiler -fPIC -shared -I$(OPS) -I$(REF)/src -I$(CUTLASS) \
	  $(SRCS) -o $@ -lcufft -lcublas -lcusolver

.PHONY: all
