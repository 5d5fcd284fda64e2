// pfs_staged.cuh — the staged shape of the FP32 neighbour passes
// (pfs_staged.cu): sizes shared with the host code and the launchers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"

namespace pfs {

struct StepBuffers;

// Threads of a staged pass's thread block (one particle each).
constexpr int ST_THREADS_HOST = 128;
// Candidates one block stages in shared memory (its union: the block's cells
// and one layer around them); blocks with more are walked from global memory.
constexpr int ST_CAP = 1024;
// Union cells a block shape may have.
constexpr int ST_UMAX = 512;
// Device counters of the staged density pass (StepBuffers::st_counters):
// non-empty blocks listed this substep, and the pass's work counter.
enum { ST_CTR_BLOCKS = 0, ST_CTR_DENSITY = 1, ST_CTR_WORDS = 4 };

// Block shape of the staged passes for a world of n particles with about
// `per_cell` particles per occupied cell and a table of `slots` slots:
// extents 2^sbx x 2^sby x 2^sbz cells.  Fills the staged fields of P (nsx.. from the grid); returns false
// when the grid is too large for fine buckets (more than `bucket_cap`).
bool configure_staged(DevParams* P, double per_cell, double slots, uint64_t bucket_cap);
// Fine buckets (cells, padded to whole blocks) of a staged configuration.
uint64_t staged_buckets(const DevParams& P);
// Particles per occupied cell of an initial state (host positions).
double occupied_cell_density(const float* pos4, uint32_t n, const float box_min[3],
                             const float box_max[3], float h);

cudaError_t launch_bucket_alloc_staged(const DevParams& P, const StepBuffers& b, cudaStream_t s);
cudaError_t launch_density_staged(const DevParams& P, const StepBuffers& b, bool fast, cudaStream_t s);

}  // namespace pfs
