# Builds the reference's MATLAB-generated data generator (its NR LDPC encoder
# among it) from the reference tree, in place, into _ref/libref_ldpc.so.
# Test infrastructure only: tests/golden/make_ldpc_golden.py calls its
# encoder to make the LDPC fixtures; nothing is copied from the reference
# tree.  Usage: make -f ref_ldpc.mk REF=<reference tree>
ifeq ($(REF),)
$(error REF=<MegaStation tree> is required)
endif
DG := $(REF)/matlab/codegen/lib/data_generator
SRCS := $(wildcard $(DG)/*.c)
OUT := _ref/libref_ldpc.so

all: $(OUT)

$(OUT): $(SRCS)
	mkdir -p _ref
	gcc -O2 -fPIC -shared -fopenmp -I$(DG) $(SRCS) -o $@ -lm

.PHONY: all
