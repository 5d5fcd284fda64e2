// pfs_world_impl.cuh — host-side pieces shared by the world and the batch.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pfs.h"

namespace pfs {

// Internal flag: ids buffers carved (PFS_FLAG_IDS requested).
constexpr int PFS_FLAG_IDS_INTERNAL = 1 << 16;

int status_from_cuda(cudaError_t e);

// One cudaMalloc carved into 256-byte aligned pieces.
struct Arena {
    void* base = nullptr;
    size_t bytes = 0;
    size_t used = 0;
    ~Arena();
    cudaError_t reserve(size_t total);
    void* take(size_t n);
    void release();
};

// Device bytes one world of n particles holds (blocks: spatial-order
// buckets; staged_blocks: blocks of the staged shape, 0 without it).
size_t world_arena_bytes(uint32_t n, int flags, int precision, uint32_t blocks, uint32_t list_cap,
                         uint32_t staged_blocks);

}  // namespace pfs
