# Build recipe for libghb (the sm_100a kernels behind the C ABI in include/ghb.h)
# and for the CPU checkers under oracle/.
#   make            -> graphhet_b200/libghb.so, oracle/liboracle.so, oracle/_ref/* (when the
#                      reference tree is present)
NVCC      ?= nvcc
CXX       := g++
CC        := gcc
ARCH      := -gencode arch=compute_100a,code=sm_100a
NVFLAGS   := $(ARCH) -O3 -lineinfo -std=c++17 -Xcompiler -fPIC -Iinclude --expt-relaxed-constexpr
REF_ROOT  ?= /root/reference
BUILD     := build/obj

CU_SRC    := $(wildcard graphhet_b200/csrc/*.cu)
CU_OBJ    := $(patsubst graphhet_b200/csrc/%.cu,$(BUILD)/%.o,$(CU_SRC))
CU_HDR    := $(wildcard graphhet_b200/csrc/*.cuh) include/ghb.h include/ghb_gen.h

all: graphhet_b200/libghb.so oracle

graphhet_b200/libghb.so: $(CU_OBJ)
	$(NVCC) $(ARCH) -shared -cudart static -o $@ $^ -lrt -ldl -lpthread

$(BUILD)/%.o: graphhet_b200/csrc/%.cu $(CU_HDR)
	@mkdir -p $(BUILD)
	$(NVCC) $(NVFLAGS) -c $< -o $@

oracle:
	$(MAKE) -C oracle REF_ROOT=$(REF_ROOT)

clean:
	rm -rf build graphhet_b200/libghb.so
	$(MAKE) -C oracle clean

.PHONY: all oracle clean
