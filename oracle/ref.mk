# Builds the reference 3D-RISM-CUDA executable from its own sources, in place
# where they lie, for sm_100a.  Objects and the binary go to oracle/_ref/
# (git-ignored; it travels to the GPU box beside the other built files).
# The reference is used only as a checker and as the timed reference arm.
#
#   make -f oracle/ref.mk REFERENCE=<reference checkout> -j8
#
# REFERENCE (or the environment variable of that name) is the checkout of the
# reference project; the default is where the build container mounts it.
REFERENCE ?= /root/reference
REF     ?= $(REFERENCE)/src-cuda
OUT     ?= $(dir $(lastword $(MAKEFILE_LIST)))_ref
CUDA    ?= /usr/local/cuda
NVCC    ?= $(CUDA)/bin/nvcc
# The image exports CXX as a wrapper without OpenMP support; use the system g++.
CXX     := $(shell test -x /usr/bin/g++ && echo /usr/bin/g++ || echo g++)
NVFLAGS  = -O3 -m64 -gencode arch=compute_100a,code=sm_100a -I$(CUDA)/include
CXXFLAGS = -O3 -fomit-frame-pointer -fopenmp -std=c++14

CU_SRCS := $(wildcard $(REF)/*.cu)
CC_SRCS := $(filter-out $(REF)/index.cc,$(wildcard $(REF)/*.cc))
OBJS    := $(patsubst $(REF)/%.cu,$(OUT)/obj/%.o,$(CU_SRCS)) \
           $(patsubst $(REF)/%.cc,$(OUT)/obj/%.o,$(CC_SRCS))

all: $(OUT)/3drism-cuda

$(OUT)/3drism-cuda: $(OBJS)
	$(CXX) $(CXXFLAGS) $(OBJS) -L$(CUDA)/lib64 -lcufft -lcuda -lcudart -o $@

$(OUT)/obj/%.o: $(REF)/%.cu | $(OUT)/obj
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OUT)/obj/%.o: $(REF)/%.cc | $(OUT)/obj
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/obj:
	mkdir -p $@

.PHONY: all
