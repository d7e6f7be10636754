# Builds pieces of the reference itself from its own sources, where they lie
# under the read-only reference tree, into oracle/_ref/ (git-ignored; the
# built files travel to the GPU box with the working tree).  Used only to pin
# the oracle.  Never copies reference sources into this repository.
#
#   make -f oracle/ref.mk REF=/path/to/reference
REF     ?= /root/reference
OUT     := oracle/_ref
CXX     := g++

all: $(OUT)/gen_random

# the reference's fixture generator (pre/units/gen_random.cpp, plain C++)
$(OUT)/gen_random: $(REF)/pre/units/gen_random.cpp $(REF)/pre/units/common/dump.cpp
	mkdir -p $(OUT)
	$(CXX) -O2 -I$(REF)/pre/units -o $@ $^

.PHONY: all
