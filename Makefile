# B200 PageRank engine: native build.
#
#   make            libgapbs_graph.so (host builder), libgapbs_pr.so (CUDA
#                   engine, sm_100a), pr_gpu (the pr_spmv-compatible CLI),
#                   cc_gpu and bfs_gpu (the cc- and bfs-compatible CLIs)
#   make oracle     oracle/liboracle.so and, where the reference tree exists,
#                   oracle/_ref/ (test infrastructure only)
#
# Everything is built in-tree under gapbs_b200/lib and gapbs_b200/bin.

CXX   := /usr/bin/g++
NVCC  ?= /usr/local/cuda/bin/nvcc
CUDA  ?= /usr/local/cuda
ARCH  := -gencode arch=compute_100a,code=sm_100a

PKG   := gapbs_b200
SRC   := $(PKG)/csrc
LIB   := $(PKG)/lib
BIN   := $(PKG)/bin

HOST_CXXFLAGS := -std=c++17 -O3 -Wall -fopenmp -fPIC -Iinclude -I$(SRC)/host
NVCC_FLAGS    := $(ARCH) -lineinfo -O3 -std=c++17 -Xcompiler -fPIC,-Wall \
                 -Iinclude -I$(SRC) --expt-relaxed-constexpr

HOST_SRCS := $(SRC)/host/builder.cc $(SRC)/host/graph_capi.cc
HOST_HDRS := $(wildcard $(SRC)/host/*.h) include/gapbs_graph.h
CU_SRCS   := $(wildcard $(SRC)/engine/*.cu)
CU_HDRS   := $(wildcard $(SRC)/engine/*.cuh) $(wildcard $(SRC)/engine/*.h) include/pr_gpu.h
CU_OBJS   := $(patsubst $(SRC)/engine/%.cu,$(LIB)/obj/%.o,$(CU_SRCS))

.PHONY: all graph engine cli oracle clean
all: graph engine cli

graph: $(LIB)/libgapbs_graph.so
engine: $(LIB)/libgapbs_pr.so
cli: $(BIN)/pr_gpu $(BIN)/cc_gpu $(BIN)/bfs_gpu

$(LIB)/libgapbs_graph.so: $(HOST_SRCS) $(HOST_HDRS)
	mkdir -p $(LIB)
	$(CXX) $(HOST_CXXFLAGS) -shared $(HOST_SRCS) -o $@

$(LIB)/obj/%.o: $(SRC)/engine/%.cu $(CU_HDRS)
	mkdir -p $(LIB)/obj
	$(NVCC) $(NVCC_FLAGS) -c $< -o $@

$(LIB)/libgapbs_pr.so: $(CU_OBJS)
	mkdir -p $(LIB)
	$(NVCC) $(ARCH) -shared $(CU_OBJS) -o $@ -lcudart

$(BIN)/pr_gpu: $(SRC)/host/pr_main.cc $(HOST_SRCS) $(HOST_HDRS) $(LIB)/libgapbs_pr.so include/pr_gpu.h
	mkdir -p $(BIN)
	$(CXX) $(HOST_CXXFLAGS) $(SRC)/host/pr_main.cc $(HOST_SRCS) -o $@ \
	    -L$(LIB) -lgapbs_pr -Wl,-rpath,'$$ORIGIN/../lib'

$(BIN)/cc_gpu: $(SRC)/host/cc_main.cc $(HOST_SRCS) $(HOST_HDRS) $(LIB)/libgapbs_pr.so include/pr_gpu.h
	mkdir -p $(BIN)
	$(CXX) $(HOST_CXXFLAGS) $(SRC)/host/cc_main.cc $(HOST_SRCS) -o $@ \
	    -L$(LIB) -lgapbs_pr -Wl,-rpath,'$$ORIGIN/../lib'

$(BIN)/bfs_gpu: $(SRC)/host/bfs_main.cc $(HOST_SRCS) $(HOST_HDRS) $(LIB)/libgapbs_pr.so include/pr_gpu.h
	mkdir -p $(BIN)
	$(CXX) $(HOST_CXXFLAGS) $(SRC)/host/bfs_main.cc $(HOST_SRCS) -o $@ \
	    -L$(LIB) -lgapbs_pr -Wl,-rpath,'$$ORIGIN/../lib'

oracle:
	$(MAKE) -C oracle

clean:
	rm -rf $(LIB) $(BIN)
