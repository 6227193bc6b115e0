# Builds the reference's eight CLI binaries from its own sources, in place under
# REF (read-only; required: make -f oracle/ref.mk REF=<reference checkout>),
# into oracle/_ref/.  Flags follow the reference Makefile
# (Makefile:1-4 there) with the device architecture fixed to sm_100a and a
# portable host -march (the GPU box CPU may differ from the build host).  The binaries are
# test infrastructure: they produce golden streams on a GPU box and are never
# linked into or called by the product library.
ifndef REF
$(error REF=<path of the reference checkout> is required)
endif
OUT ?= $(dir $(lastword $(MAKEFILE_LIST)))_ref
NVCC ?= nvcc
FLAGS = -arch=sm_100a -O3 -DUSE_GPU -DNDEBUG -fmad=false \
        -Xcompiler "-O3 -march=x86-64-v2 -mno-fma -ffp-contract=off" -std=c++17 -I$(REF)

BINS = store init_send init_recv resi_send resi_recv store_bench init_bench resi_bench
all: $(addprefix $(OUT)/,$(BINS))

$(OUT)/store: $(REF)/src/cortado_store.cu ; mkdir -p $(OUT) && $(NVCC) $(FLAGS) -o $@ $<
$(OUT)/store_bench: $(REF)/src/cortado_store.cu ; mkdir -p $(OUT) && $(NVCC) -DBENCHMARK $(FLAGS) -o $@ $<
$(OUT)/init_send: $(REF)/src/cortado_init.cu ; mkdir -p $(OUT) && $(NVCC) -DSEND $(FLAGS) -o $@ $<
$(OUT)/init_recv: $(REF)/src/cortado_init.cu ; mkdir -p $(OUT) && $(NVCC) -DRECV $(FLAGS) -o $@ $<
$(OUT)/init_bench: $(REF)/src/cortado_init.cu ; mkdir -p $(OUT) && $(NVCC) -DBENCHMARK $(FLAGS) -o $@ $<
$(OUT)/resi_send: $(REF)/src/cortado_resi.cu ; mkdir -p $(OUT) && $(NVCC) -DSEND $(FLAGS) -o $@ $<
$(OUT)/resi_recv: $(REF)/src/cortado_resi.cu ; mkdir -p $(OUT) && $(NVCC) -DRECV $(FLAGS) -o $@ $<
$(OUT)/resi_bench: $(REF)/src/cortado_resi.cu ; mkdir -p $(OUT) && $(NVCC) -DBENCHMARK $(FLAGS) -o $@ $<
