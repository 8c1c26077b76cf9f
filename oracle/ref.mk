# Build hotspin's own CUDA kernel library (libhotspin.so) from the reference sources, for
# sm_100a, into oracle/_ref/.  TEST INFRASTRUCTURE: the reference kernels are the parity and
# timing baseline of the replayed reference path; nothing in the product links them.
#
#   make -f oracle/ref.mk            (needs the reference checkout: $HOTSPIN_REF, default
#                                     /root/reference, or REF=<its src/libhotspin>)
#
# The flags are those of src/Make.inc with the gencode list replaced by sm_100a.
HOTSPIN_REF ?= /root/reference
REF  ?= $(HOTSPIN_REF)/src/libhotspin
OUT  ?= $(dir $(abspath $(lastword $(MAKEFILE_LIST))))_ref
NVCC ?= nvcc
ARCH  = -gencode arch=compute_100a,code=sm_100a
FLAGS = -std=c++14 --compiler-options -fPIC --fmad=true $(ARCH) -O3 -I$(REF)

CU  := $(wildcard $(REF)/*.cu)
CPP := $(wildcard $(REF)/*.cpp)
OBJ := $(patsubst $(REF)/%.cu,$(OUT)/obj/%.o,$(CU)) $(patsubst $(REF)/%.cpp,$(OUT)/obj/%.o,$(CPP))

all: $(OUT)/libhotspin.so

$(OUT)/obj/%.o: $(REF)/%.cu
	@mkdir -p $(dir $@)
	$(NVCC) $(FLAGS) -dc $< -o $@

$(OUT)/obj/%.o: $(REF)/%.cpp
	@mkdir -p $(dir $@)
	g++ -fPIC -O2 -I/usr/local/cuda/include -I$(REF) -c $< -o $@

$(OUT)/libhotspin.so: $(OBJ)
	$(NVCC) $(ARCH) -shared $(OBJ) -o $@ -lcufft -lcudart

clean:
	rm -rf $(OUT)/obj $(OUT)/libhotspin.so

.PHONY: all clean
