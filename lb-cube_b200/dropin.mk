# Builds LB-Cube's own drivers (src/main.cpp -> lbm_sim, src/simulate_reaction.cpp
# -> lbm_reaction_sim), unmodified, against this engine: include/lattice_cuda.cuh
# shadows the reference's header and liblbcube_b200.so replaces the lbm::cuda
# library. Eigen and <mdspan> come from the oracle's stand-ins because neither
# is installed here; a user with real Eigen drops SHIM.
#
#   make -f lb-cube_b200/dropin.mk REF=/path/to/LB-Cube
# (default: a checkout named reference next to this repository)
HERE    := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
REF     ?= $(abspath $(HERE)../../reference)
CUDA    ?= /usr/local/cuda
OUT     := $(HERE)_build/dropin
SHIM    := -I$(HERE)../oracle/shim
CXXFLAGS := -std=c++23 -O2 -ffp-contract=off -w -DLB_CUBE_ENABLE_CUDA=1 \
            -I$(HERE)../include $(SHIM) -I$(REF)/include -I$(CUDA)/targets/x86_64-linux/include
LDFLAGS := -L$(HERE) -llbcube_b200 -Wl,-rpath,$(HERE) -L$(CUDA)/lib64 -lcudart -Wl,-rpath,$(CUDA)/lib64

.PHONY: all
all: $(OUT)/lbm_sim $(OUT)/lbm_reaction_sim

$(OUT)/lbm_sim: $(REF)/src/main.cpp $(HERE)../include/lattice_cuda.cuh $(HERE)liblbcube_b200.so
	mkdir -p $(OUT) && g++ $(CXXFLAGS) $< -o $@ $(LDFLAGS)

$(OUT)/lbm_reaction_sim: $(REF)/src/simulate_reaction.cpp $(HERE)../include/lattice_cuda.cuh $(HERE)liblbcube_b200.so
	mkdir -p $(OUT) && g++ $(CXXFLAGS) $< -o $@ $(LDFLAGS)
