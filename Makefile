# B200 ACO-for-CVRP build (sm_100a only).
#
#   make            -> vehicleroutingproblem_b200/libaco_b200.so + aco_vrp_cuda.out
#   make cuda       -> aco_vrp_cuda.out (drop-in for the reference's `make cuda`)
#   make lib        -> the shared library behind the C ABI (include/aco_b200.h)
#   make oracle     -> oracle/liboracle.so (test infrastructure)
#   make ref        -> oracle/_ref/ (the reference built from its sources)

NVCC ?= nvcc
CC := gcc
CUDA_ARCH ?= -gencode arch=compute_100a,code=sm_100a
NVCC_FLAGS = -O3 -std=c++17 $(CUDA_ARCH) -lineinfo -Iinclude -Xcompiler -fPIC \
             -Xcompiler -fvisibility=hidden
C_FLAGS = -O2 -std=c11 -Wall -Iinclude -fPIC -fvisibility=hidden

PKG := vehicleroutingproblem_b200
CSRC := $(PKG)/csrc
BUILD := $(PKG)/_build
LIB := $(PKG)/libaco_b200.so
CLI := aco_vrp_cuda.out

CU_SRCS := $(CSRC)/cuda/aco_kernels.cu $(CSRC)/cuda/aco_solver.cu $(CSRC)/cuda/aco_compat.cu $(CSRC)/cuda/aco_prior.cu \
           $(CSRC)/cuda/aco_noalloc.cu $(CSRC)/cuda/aco_batch.cu $(CSRC)/cuda/aco_seq_update.cu
C_SRCS := $(CSRC)/common/solution.c $(CSRC)/common/instance_parser.c \
          $(CSRC)/common/aco_config.c $(CSRC)/common/cli_common.c
CU_OBJS := $(patsubst $(CSRC)/cuda/%.cu,$(BUILD)/%.o,$(CU_SRCS))
C_OBJS := $(patsubst $(CSRC)/common/%.c,$(BUILD)/%.o,$(C_SRCS))
HDRS := $(wildcard include/*.h) $(wildcard $(CSRC)/cuda/*.cuh) $(wildcard $(CSRC)/cuda/*.h)

all: lib cuda

lib: $(LIB)
cuda: $(CLI)

$(BUILD):
	mkdir -p $(BUILD)

$(BUILD)/%.o: $(CSRC)/cuda/%.cu $(HDRS) | $(BUILD)
	$(NVCC) $(NVCC_FLAGS) -c $< -o $@

$(BUILD)/%.o: $(CSRC)/common/%.c $(HDRS) | $(BUILD)
	$(CC) $(C_FLAGS) -c $< -o $@

$(LIB): $(CU_OBJS) $(C_OBJS)
	$(NVCC) $(CUDA_ARCH) -shared -Xcompiler -fvisibility=hidden $^ -o $@

$(CLI): $(CSRC)/main_vrp.c $(LIB)
	$(CC) -O2 -std=c11 -Wall -Iinclude $< -L$(PKG) -laco_b200 -Wl,-rpath,'$$ORIGIN/$(PKG)' -o $@

oracle:
	$(MAKE) -C oracle all

ref:
	$(MAKE) -C oracle ref

ptxas:
	$(NVCC) $(NVCC_FLAGS) -Xptxas -v -c $(CSRC)/cuda/aco_kernels.cu -o /dev/null

clean:
	rm -rf $(BUILD) $(LIB) $(CLI)

.PHONY: all lib cuda oracle ref ptxas clean
