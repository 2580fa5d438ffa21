# Build recipe for libghb (the sm_100a kernels behind the C ABI in include/ghb.h)
# and for the CPU checkers under oracle/.
#   make            -> graphhet_b200/libghb.so, oracle/liboracle.so, oracle/_ref/* (when the
#                      reference tree is present)
NVCC      ?= nvcc
CXX       := g++
CC        := gcc
ARCH      := -gencode arch=compute_100a,code=sm_100a
NVFLAGS   := $(ARCH) -O3 -lineinfo -std=c++17 -Xcompiler -fPIC -Iinclude --expt-relaxed-constexpr
# REF_ROOT: path to the GraphHET source tree (MDNDDD/GraphHET).  Required for
# oracle/_ref and the drop-in build; both are skipped when it is not given.
REF_ROOT  ?=
BUILD     := build/obj

CU_SRC    := $(wildcard graphhet_b200/csrc/*.cu)
CU_OBJ    := $(patsubst graphhet_b200/csrc/%.cu,$(BUILD)/%.o,$(CU_SRC))
CU_HDR    := $(wildcard graphhet_b200/csrc/*.cuh) include/ghb.h include/ghb_gen.h

all: graphhet_b200/libghb.so oracle dropin

graphhet_b200/libghb.so: $(CU_OBJ)
	$(NVCC) $(ARCH) -shared -cudart static -o $@ $^ -lrt -ldl -lpthread

$(BUILD)/%.o: graphhet_b200/csrc/%.cu $(CU_HDR)
	@mkdir -p $(BUILD)
	$(NVCC) $(NVFLAGS) -c $< -o $@

oracle:
	$(MAKE) -C oracle REF_ROOT=$(REF_ROOT)

# The reference's own GPU drivers (GPU_csr_example.cu, LDBC_GPU_csr.cu,
# GPU_gpma_example.cu, LDBC_GPU_gpma.cu), compiled unchanged from where they
# lie against this repository's include/GPU_csr and include/GPU_gpma headers
# and linked to libghb.so: the drop-in check.
DROPIN    := build/dropin
dropin: graphhet_b200/libghb.so
	@if [ -n "$(REF_ROOT)" ] && [ -f "$(REF_ROOT)/src/LDBC/LDBC_GPU_csr.cu" ]; then \
	  mkdir -p $(DROPIN) && \
	  $(NVCC) $(ARCH) -O2 -std=c++17 -Iinclude -I$(REF_ROOT)/include $(REF_ROOT)/src/GPU_csr/GPU_csr_example.cu \
	    -o $(DROPIN)/GPU_csr_example -Lgraphhet_b200 -lghb -Xlinker -rpath -Xlinker '$$ORIGIN/../../graphhet_b200' && \
	  $(NVCC) $(ARCH) -O2 -std=c++17 -Iinclude -I$(REF_ROOT)/include $(REF_ROOT)/src/LDBC/LDBC_GPU_csr.cu \
	    -o $(DROPIN)/LDBC_GPU_csr -Lgraphhet_b200 -lghb -Xlinker -rpath -Xlinker '$$ORIGIN/../../graphhet_b200' && \
	  $(NVCC) $(ARCH) -O2 -std=c++17 -Iinclude -I$(REF_ROOT)/include $(REF_ROOT)/src/GPU_gpma/GPU_gpma_example.cu \
	    -o $(DROPIN)/GPU_gpma_example -Lgraphhet_b200 -lghb -Xlinker -rpath -Xlinker '$$ORIGIN/../../graphhet_b200' && \
	  $(NVCC) $(ARCH) -O2 -std=c++17 -Iinclude -I$(REF_ROOT)/include $(REF_ROOT)/src/LDBC/LDBC_GPU_gpma.cu \
	    -o $(DROPIN)/LDBC_GPU_gpma -Lgraphhet_b200 -lghb -Xlinker -rpath -Xlinker '$$ORIGIN/../../graphhet_b200' && \
	  $(NVCC) $(ARCH) -O3 -std=c++17 -Iinclude -I$(REF_ROOT)/include graphhet_b200/dropin_bfs_bench.cu \
	    -o $(DROPIN)/dropin_bfs_bench -Lgraphhet_b200 -lghb -Xlinker -rpath -Xlinker '$$ORIGIN/../../graphhet_b200' ; \
	else echo "REF_ROOT (the GraphHET source tree) not given or without src/: skipping the drop-in build"; fi

clean:
	rm -rf build graphhet_b200/libghb.so
	$(MAKE) -C oracle clean

.PHONY: all oracle dropin clean
