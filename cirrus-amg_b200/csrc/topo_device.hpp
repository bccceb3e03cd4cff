// Octree refinement, ghost spawning and the canonical tables built on the device
// (topo_device.cu) for the built-in refinement targets.
#pragma once
#include <cuda_runtime.h>

#include "topology.hpp"

namespace cmg {

constexpr int kDevTopoMaxParams = 64;

// Device memory from the per-device stream-ordered pool that also holds the grids' channel
// planes and tables; freed memory stays in the pool for the next octree (cmg_impl.cu).
cudaError_t pool_malloc(void** p, size_t bytes, int dev, cudaStream_t st);
void pool_release(void* p, cudaStream_t st);

// Device work space of the builder: tile pool, hash table, sort buffers (grow-only).
struct DeviceTopoBuilder {
    int cap = 0;         // tile records
    unsigned hcap = 0;   // hash slots (power of two, at least twice cap)
    unsigned long long *hk = nullptr, *keys = nullptr, *keys2 = nullptr;
    int *hv = nullptr, *type0 = nullptr, *flag = nullptr, *idx = nullptr, *idx2 = nullptr, *nb = nullptr, *child = nullptr;
    int* scal = nullptr;
    int4 *rec = nullptr, *rec2 = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    cudaStream_t st = nullptr;  // the stream the builder's work and its allocations run on
    int dev = 0;                // the device of the grid that owns the builder
    cudaError_t reserve(int tiles);
    void release();
    ~DeviceTopoBuilder();
};

// Cases the device builder computes exactly as the host (case_target): 0-3, 6, 7.
bool device_case_supported(int case_id);
// Topology::iterative_refine with case_target, then the ghost layer and the canonical
// order and tables, on the device; the result is adopted by `topo`.  0 on success, 1 for
// an unsupported case or bad parameters, 2 for a CUDA error.
int device_refine_case(DeviceTopoBuilder& B, Topology& topo, int case_id, const double* params, int nparams, cudaStream_t st,
                       int* steps);

// CreateTestGrid's LEAF cell types of the built-in cases on the device (all but the star
// case 5, whose corner test uses transcendental functions): the same values as the host's
// case_cell_type, written into the cell-type plane of the given LEAF tiles
bool device_cell_types_supported(int case_id);
cudaError_t device_leaf_cell_types(const int4* meta, uint8_t* ctype, const int* leaf, int nleaf, int case_id, float h0, cudaStream_t st);

}  // namespace cmg
