# Compiles the reference's own host sources for decycle and the BFS matching
# order (cpuGraph.cpp, decycle.cpp, order.cpp), where they lie in the
# reference checkout, together with ref_harness.cpp into oracle/_ref/libref.so
# (test infrastructure; outputs only under oracle/_ref/).  The sources include
# CUDA headers, so nvcc compiles them (host code only is used).
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
REF ?= /root/reference
OUT := $(HERE)_ref
NVCC ?= /usr/local/cuda/bin/nvcc
FLAGS := -x cu -std=c++17 -O1 -DNDEBUG -w -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a \
         -Wno-deprecated-gpu-targets -I$(REF)

OBJS := $(OUT)/cpuGraph.o $(OUT)/decycle.o $(OUT)/order.o $(OUT)/ref_harness.o

all: $(OUT)/libref.so

$(OUT)/%.o: $(REF)/%.cpp
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/ref_harness.o: $(HERE)ref_harness.cpp
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/libref.so: $(OBJS)
	$(NVCC) -shared -gencode arch=compute_100a,code=sm_100a -o $@ $(OBJS) -lcudart

.PHONY: all
