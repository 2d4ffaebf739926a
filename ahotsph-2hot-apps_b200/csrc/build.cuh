// build.cuh -- the GPU tree builder's interface inside libgravcuda (build.cu
// builds; batch.cu turns the result into a plan).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "nlnhost.h"
#include "nlnlists.h"

// A tree built on the device: every table and list in device memory
// (cudaMalloc'd; ownership passes to whoever takes them), plus host copies
// of the small arrays a plan's work queue is built from.
struct DevTree {
    int64_t n = 0, ncells = 0, ngroups = 0;
    double box = 0.0;
    float4 *points = nullptr;       // n + ncells: bodies in tree order, then cell monopoles
    nln_qcell *qcells = nullptr;    // ncells
    nln_hcell *hcells = nullptr;    // ncells
    nln_group *groups = nullptr;    // ngroups
    uint32_t *list[4] = {nullptr, nullptr, nullptr, nullptr};  // P, Q, H, correction
    int64_t len[4] = {0, 0, 0, 0};
    int64_t *order = nullptr;       // n: tree position -> input index
    int64_t *cell_first = nullptr;  // ncells
    int32_t *cell_count = nullptr, *cell_child = nullptr, *cell_nchild = nullptr,
            *cell_level = nullptr;
    int64_t counts[4] = {0, 0, 0, 0};  // interactions: body, monopole cell, quadrupole, order 4
    std::vector<nln_group> groups_h;
    std::vector<int64_t> ptr_h[4];  // ngroups + 1 list offsets per kind
    double seconds[6] = {0, 0, 0, 0, 0, 0};  // sort, cells, moments, groups, walk passes, lists
    cudaMemPool_t pool = nullptr;   // the pool the buffers came from (cudaFreeAsync them)
};

// Build the tree, moments, critical radii, sink groups and interaction
// lists of n bodies (device float4 x, y, z, m, any order) with the
// semantics and arithmetic of nlnhost.h's nln_tree_build + nln_tree_walk
// (bit-identical results); enqueued on st and synchronised.  Returns 0, -1
// for bad arguments or positions (message recorded), or a CUDA status.
// pool: when set, every device buffer comes from it (stream-ordered on st)
// and is returned to it; the tree's buffers must then be freed with
// cudaFreeAsync.
int gpu_tree_build(const nln_params &p, const float4 *bodies, int64_t n, cudaStream_t st,
                   DevTree &out, cudaMemPool_t pool = nullptr);
void dev_tree_free(DevTree &t, cudaMemPool_t pool = nullptr);
