# Compiles the unmodified reference sources (read in place) for sm_100a into _ref/:
#   _ref/gpu-tild      the reference program (drop-in comparison on the same GPU)
#   _ref/ref_harness   reference objects minus main.o + ref_harness_main.cu: runs
#                      initialize(); forces(); and dumps forces, densities and stencils
# Nothing here is product code.  Usage: make -f ref.mk REF=<path to the gpu-tild sources>
ifeq ($(REF),)
$(error REF=<path to the gpu-tild sources> is required)
endif
NVCC     ?= nvcc
OUT      := _ref
FLAGS    := -std=c++14 -rdc=true -gencode arch=compute_100a,code=sm_100a -O3 -w
SRCS     := $(filter-out $(REF)/main.cu,$(wildcard $(REF)/*.cu))
OBJS     := $(patsubst $(REF)/%.cu,$(OUT)/obj/%.o,$(SRCS))

all: $(OUT)/gpu-tild $(OUT)/ref_harness

$(OUT)/obj/%.o: $(REF)/%.cu
	@mkdir -p $(OUT)/obj
	$(NVCC) $(FLAGS) -I$(REF) -c $< -o $@

$(OUT)/obj/main.o: $(REF)/main.cu
	@mkdir -p $(OUT)/obj
	$(NVCC) $(FLAGS) -I$(REF) -c $< -o $@

$(OUT)/obj/ref_harness_main.o: ref_harness_main.cu
	@mkdir -p $(OUT)/obj
	$(NVCC) $(FLAGS) -I$(REF) -c $< -o $@

$(OUT)/gpu-tild: $(OBJS) $(OUT)/obj/main.o
	$(NVCC) $(FLAGS) -o $@ $^ -lcufft -lm

$(OUT)/ref_harness: $(OBJS) $(OUT)/obj/ref_harness_main.o
	$(NVCC) $(FLAGS) -o $@ $^ -lcufft -lm

.PHONY: all
