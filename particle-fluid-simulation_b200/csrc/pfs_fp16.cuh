// pfs_fp16.cuh — the bandwidth (FP16-cell) form of the neighbour passes.
//
// Sorted positions and velocities are stored for the neighbour loops as one
// 16-byte record per particle: the integer cell of x* (three 10-bit fields,
// biased by one) plus FP16 offsets of x* from that cell's origin in units of
// h, and the velocity in FP16 in units of h/dt.  A force candidate then costs
// 16 + 8 bytes instead of 16 + 16 + 8.  All accumulation stays FP32 (the
// density sum compensated), and the integrator, cell keys and table are the
// FP32 form's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_step.cuh"
#include "pfs_world_impl.cuh"

namespace pfs {

struct Fp16Buffers {
    uint4* rec;  // n records: cell, half2(ox, oy), half2(oz, vx), half2(vy, vz)
};

// Cells per axis the 10-bit fields can hold (bias -1 .. 1022).
constexpr int FP16_MAX_CELLS = 1020;

size_t fp16_arena_bytes(uint32_t n);
bool fp16_carve(Arena& a, uint32_t n, Fp16Buffers* out);
// PFS_EINVAL when the box spans more than FP16_MAX_CELLS cells on an axis or
// dt <= 0 (the velocity unit is h/dt).
int fp16_check_box(const pfs_params& p);

cudaError_t launch_reorder_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                                cudaStream_t s);
cudaError_t launch_density_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                                cudaStream_t s);
cudaError_t launch_force_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                              cudaStream_t s);

}  // namespace pfs
