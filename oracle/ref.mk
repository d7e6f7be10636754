# Builds pieces of the reference itself from its own sources, where they lie
# under the read-only reference tree, into oracle/_ref/ (git-ignored; the
# built files travel to the GPU box with the working tree).  Used only to pin
# the oracle and as the GPU parity reference of the tests.  Never copies
# reference sources into this repository.
#
#   make -f oracle/ref.mk REF=/path/to/reference
REF     ?= /root/reference
OUT     := oracle/_ref
CXX     := g++
NVCC    ?= nvcc
# the reference's own device flags (src/make/main.mk:18-26), for sm_100a
REF_NVCC := -gencode arch=compute_100a,code=sm_100a -std=c++11 -O3 -g -use_fast_math -restrict -DNDEBUG

all: $(OUT)/gen_random $(OUT)/librefkern.so

# the reference's fixture generator (pre/units/gen_random.cpp, plain C++)
$(OUT)/gen_random: $(REF)/pre/units/gen_random.cpp $(REF)/pre/units/common/dump.cpp
	mkdir -p $(OUT)
	$(CXX) -O2 -I$(REF)/pre/units -o $@ $^

# reference device code (src/math/rnd/dev.h, src/pair/dev.h, ...) behind a C
# shim; oracle/refkern/conf.h stands in for the generated build configuration
$(OUT)/librefkern.so: oracle/refkern/refkern.cu oracle/refkern/conf.h
	mkdir -p $(OUT)
	$(NVCC) $(REF_NVCC) -Ioracle/refkern -I$(REF)/src -Xcompiler -fPIC -shared -o $@ oracle/refkern/refkern.cu

.PHONY: all
