# Builds pieces of the reference itself from its own sources, where they lie
# under the read-only reference tree, into oracle/_ref/ (git-ignored; the
# built files travel to the GPU box with the working tree).  Used only to pin
# the oracle and as the GPU parity reference of the tests.  Never copies
# reference sources into this repository.
#
#   make -f oracle/ref.mk REF=/path/to/reference
# the reference tree: $(CTC_REFERENCE) when set, else its usual place in the
# build container
CTC_REFERENCE ?= /root/reference
REF     ?= $(CTC_REFERENCE)
OUT     := oracle/_ref
CXX     := g++
NVCC    ?= nvcc
# the reference's own device flags (src/make/main.mk:18-26), for sm_100a
REF_NVCC := -gencode arch=compute_100a,code=sm_100a -std=c++11 -O3 -g -use_fast_math -restrict -DNDEBUG

all: $(OUT)/gen_random $(OUT)/librefkern.so $(OUT)/librefsdf.so $(OUT)/librefhost.so

# the reference's fixture generator (pre/units/gen_random.cpp, plain C++)
$(OUT)/gen_random: $(REF)/pre/units/gen_random.cpp $(REF)/pre/units/common/dump.cpp
	mkdir -p $(OUT)
	$(CXX) -O2 -I$(REF)/pre/units -o $@ $^

# reference device code (src/math/rnd/dev.h, src/pair/dev.h, ...) behind a C
# shim; oracle/refkern/conf.h stands in for the generated build configuration
$(OUT)/librefkern.so: oracle/refkern/refkern.cu oracle/refkern/refwall.cu oracle/refkern/refobj.cu oracle/refkern/conf.h
	mkdir -p $(OUT)
	$(NVCC) $(REF_NVCC) -Ioracle/refkern -Ictc_b200/compat/check -I$(REF)/src -Xcompiler -fPIC -shared -o $@ \
	    oracle/refkern/refkern.cu \
	    oracle/refkern/refwall.cu \
	    oracle/refkern/refobj.cu

# the reference's host-side SDF pipeline (field reading, scaling, B-spline
# resampling, grid transforms) from its sources, with the reference's host
# flags (src/make/main.mk: -std=c++11 -O3); oracle/refkern/refsdf.cpp holds
# the one-rank coordinate accessors and stubs for the log and the HDF5 writer;
# <stdio.h> comes first as the real <mpi.h> brings it
REF_SDF_SRC := $(REF)/src/utils/error.cpp $(REF)/src/utils/imp.cpp $(REF)/src/utils/os.cpp \
	$(REF)/src/math/tform/imp.cpp $(REF)/src/wall/sdf/field/imp.cpp $(REF)/src/wall/sdf/tform/imp.cpp
$(OUT)/librefsdf.so: oracle/refkern/refsdf.cpp oracle/refkern/conf.h $(REF_SDF_SRC)
	mkdir -p $(OUT)
	$(CXX) -std=c++11 -O3 -fPIC -shared -include stdio.h -Ioracle/refkern -Ictc_b200/compat/check -I$(REF)/src \
	    -I/usr/local/cuda/include -o $@ oracle/refkern/refsdf.cpp $(REF_SDF_SRC)

.PHONY: all

# the reference's host-side membrane pieces from its sources: the ring
# adjacency (src/rbc/adj, src/algo/edg) and the host build of the Kantor
# dihedral forces (src/mesh/force/kantor0/imp.cpp); oracle/refkern/refhost.cpp
# holds the entry points and stubs for the device calls it never makes
REF_HOST_SRC := $(REF)/src/rbc/adj/imp.cpp $(REF)/src/algo/edg/imp.cpp $(REF)/src/mesh/force/kantor0/imp.cpp \
	$(REF)/src/utils/error.cpp $(REF)/src/utils/imp.cpp $(REF)/src/utils/os.cpp
$(OUT)/librefhost.so: oracle/refkern/refhost.cpp oracle/refkern/conf.h $(REF_HOST_SRC)
	mkdir -p $(OUT)
	$(CXX) -std=c++11 -O3 -fPIC -shared -include stdio.h -Ioracle/refkern -Ictc_b200/compat/check -I$(REF)/src \
	    -I$(REF)/src/algo/edg -I/usr/local/cuda/include -o $@ oracle/refkern/refhost.cpp $(REF_HOST_SRC)
