# Build recipe for oracle/_ref/libpdhcg_ref.so: the reference solver compiled
# from its own sources, where they lie under REF (read-only), with outputs
# only under oracle/_ref/.  Test infrastructure: it is the reference run as a
# checker (host-side functions are called on the CPU by the tests; the GPU
# solve is run beside ours on a GPU host).  It is never linked into the
# product.
#
#   make -f oracle/ref.mk REF=<reference source tree> -j8
#
# REF defaults to $(PDHCG_REFERENCE_SRC), else a "reference" directory
# beside the repository.
#
# The reference's own CMake build is not used.  The source list mirrors
# what that build puts in its core library for a single-GPU build: every
# src/*.c except the CLI, every src/*.cu and src/kernels/*.cu, plus the two
# distributed stubs.  It links the CUDA toolkit's cuSPARSE, cuBLAS and
# cuSOLVER and zlib, all present in the image.

REF ?= $(if $(PDHCG_REFERENCE_SRC),$(PDHCG_REFERENCE_SRC),$(abspath ../reference))
OUT := oracle/_ref
NVCC ?= nvcc
CC ?= gcc
ARCH := -gencode arch=compute_100a,code=sm_100a
DEFS := -DPDHCG_VERSION=\"0.3.0\" -DCUSPARSE_ENABLE_EXPERIMENTAL_API
INCS := -I$(REF)/include -I$(REF)/internal -I$(REF)/distributed

C_SRCS := $(filter-out $(REF)/src/cli.c,$(wildcard $(REF)/src/*.c)) \
          $(REF)/distributed/distributed_ops_stub.c \
          $(REF)/distributed/distributed_conic_stub.c
CU_SRCS := $(wildcard $(REF)/src/*.cu) $(wildcard $(REF)/src/kernels/*.cu)

C_OBJS := $(patsubst $(REF)/%.c,$(OUT)/obj/%.o,$(C_SRCS))
CU_OBJS := $(patsubst $(REF)/%.cu,$(OUT)/obj/%.o,$(CU_SRCS))

all: $(OUT)/libpdhcg_ref.so

$(OUT)/obj/%.o: $(REF)/%.c
	@mkdir -p $(dir $@)
	$(CC) -std=gnu99 -O3 -fPIC $(DEFS) $(INCS) -I/usr/local/cuda/include -c $< -o $@

$(OUT)/obj/%.o: $(REF)/%.cu
	@mkdir -p $(dir $@)
	$(NVCC) -std=c++17 -O3 -rdc=true -Xcompiler -fPIC $(ARCH) $(DEFS) $(INCS) -c $< -o $@

$(OUT)/libpdhcg_ref.so: $(C_OBJS) $(CU_OBJS)
	$(NVCC) -shared -rdc=true $(ARCH) -Xlinker -Bsymbolic $^ -o $@ -lcusparse -lcublas -lcusolver -lz

clean:
	rm -rf $(OUT)

.PHONY: all clean
