# Builds the reference router's own code, from its sources where they lie,
# into oracle/_ref/ (git-ignored; travels to the GPU box with the snapshot):
#   ref_harness  -- oracle/ref_harness.cu compiled against the reference headers
#   ref_harness_ggr -- the same with GROTOR_GGR_ROUTING (integer wire costs and
#                   the Z-shape pipeline of the reference's grotor_ggr build)
#   grotor       -- the reference router itself (its src/main.cu, CPU-batching
#                   build), the stock program a drop-in is compared with
#   grotor_ggr   -- the same program with GROTOR_GGR_ROUTING (its grotor_ggr
#                   build: the Z-shape pipeline)
#   grotor_cugr2 -- the same program with GROTOR_CUGR2_ROUTING (its
#                   grotor_cugr2 build: L-shape, FLT and maze stages)
#   evaluator    -- the reference's scoring program (resources/evaluator.cpp)
#   POWV9.dat, POST9.dat -- FLUTE lookup tables the reference reads at run time
# Usage: make -C oracle -f ref.mk REF=/path/to/GRotor
# (REF has no default: the caller names the reference checkout.)
ifeq ($(REF),)
$(error REF=<path to the GRotor sources> is required)
endif
NVCC ?= nvcc
HOSTCXX ?= /usr/bin/g++
OUT := _ref

all: $(OUT)/ref_harness $(OUT)/ref_harness_ggr $(OUT)/grotor $(OUT)/grotor_ggr $(OUT)/grotor_cugr2 $(OUT)/evaluator \
     $(OUT)/POWV9.dat \
     $(OUT)/POST9.dat

$(OUT):
	mkdir -p $(OUT)

$(OUT)/ref_harness: ref_harness.cu | $(OUT)
	$(NVCC) -ccbin $(HOSTCXX) -std=c++17 -O3 -UNDEBUG -gencode arch=compute_100a,code=sm_100a \
	  -Xcompiler -fopenmp -I$(REF)/include -I$(REF)/src -I$(REF)/third_party \
	  -DG_ROTOR_RESOURCE_DIR=\"$(OUT)\" -x cu ref_harness.cu -o $@

$(OUT)/ref_harness_ggr: ref_harness.cu | $(OUT)
	$(NVCC) -ccbin $(HOSTCXX) -std=c++17 -O3 -UNDEBUG -gencode arch=compute_100a,code=sm_100a \
	  -Xcompiler -fopenmp -I$(REF)/include -I$(REF)/src -I$(REF)/third_party -DGROTOR_GGR_ROUTING=1 \
	  -DG_ROTOR_RESOURCE_DIR=\"$(OUT)\" -x cu ref_harness.cu -o $@

$(OUT)/grotor: $(REF)/src/main.cu | $(OUT)
	$(NVCC) -ccbin $(HOSTCXX) -std=c++17 -O3 -UNDEBUG -gencode arch=compute_100a,code=sm_100a \
	  -Xcompiler -fopenmp -I$(REF)/include -I$(REF)/src -I$(REF)/third_party \
	  -DG_ROTOR_RESOURCE_DIR=\"$(OUT)\" -x cu $< -o $@

$(OUT)/grotor_ggr: $(REF)/src/main.cu | $(OUT)
	$(NVCC) -ccbin $(HOSTCXX) -std=c++17 -O3 -UNDEBUG -gencode arch=compute_100a,code=sm_100a \
	  -Xcompiler -fopenmp -I$(REF)/include -I$(REF)/src -I$(REF)/third_party -DGROTOR_GGR_ROUTING=1 \
	  -DG_ROTOR_RESOURCE_DIR=\"$(OUT)\" -x cu $< -o $@

$(OUT)/grotor_cugr2: $(REF)/src/main.cu | $(OUT)
	$(NVCC) -ccbin $(HOSTCXX) -std=c++17 -O3 -UNDEBUG -gencode arch=compute_100a,code=sm_100a \
	  -Xcompiler -fopenmp -I$(REF)/include -I$(REF)/src -I$(REF)/third_party -DGROTOR_CUGR2_ROUTING=1 \
	  -DG_ROTOR_RESOURCE_DIR=\"$(OUT)\" -x cu $< -o $@

$(OUT)/evaluator: $(REF)/resources/evaluator.cpp | $(OUT)
	$(HOSTCXX) -O3 -UNDEBUG -std=c++17 $< -o $@

$(OUT)/%.dat: $(REF)/resources/flute/%.dat | $(OUT)
	cp $< $@

.PHONY: all
