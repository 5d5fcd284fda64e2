// pfs_record.cuh — the 16-byte neighbour record of the FP16-cell form.
//
//   x: cell of x* — three 10-bit fields, each biased by one (-1 .. 1022)
//   y: half2 (ox, oy)   offsets of x* from the cell origin, units of h
//   z: half2 (oz, vx)   vx, vy, vz: velocity, units of h / dt
//   w: half2 (vy, vz)
// Offsets are in [0, 1); velocities saturate at the FP16 range.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "pfs_common.cuh"

namespace pfs {

__device__ __forceinline__ uint32_t rec_pack_cell(int32_t cx, int32_t cy, int32_t cz) {
    return ((uint32_t)(cx + 1) & 1023u) | (((uint32_t)(cy + 1) & 1023u) << 10) |
           (((uint32_t)(cz + 1) & 1023u) << 20);
}

__device__ __forceinline__ float rec_sat(float x) { return fminf(fmaxf(x, -65504.0f), 65504.0f); }

__device__ __forceinline__ uint32_t rec_h2u(float a, float b) {
    const __half2 v = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float2 rec_u2f(uint32_t u) {
    __half2 v;
    *reinterpret_cast<uint32_t*>(&v) = u;
    return __half22float2(v);
}

struct Unpacked {
    float px, py, pz;  // position in units of h: cell + offset
    float vx, vy, vz;  // velocity in units of h/dt
};

// A biased 10-bit cell field as the float (field - 1): the bits 0x4B000000
// are the float 2^23, whose mantissa step is 1, so with the field in the low
// mantissa bits the float is exactly 2^23 + field, and subtracting 2^23 + 1
// is exact.  Same value as an integer-to-float conversion, in two
// instructions.
__device__ __forceinline__ float rec_cell_f(uint32_t field10) {
    return __int_as_float(0x4B000000u | field10) - 8388609.0f;
}

__device__ __forceinline__ Unpacked rec_unpack(const uint4 r) {
    Unpacked u;
    const float2 a = rec_u2f(r.y), b = rec_u2f(r.z), c = rec_u2f(r.w);
    u.px = rec_cell_f(r.x & 1023u) + a.x;
    u.py = rec_cell_f((r.x >> 10) & 1023u) + a.y;
    u.pz = rec_cell_f((r.x >> 20) & 1023u) + b.x;
    u.vx = b.y;
    u.vy = c.x;
    u.vz = c.y;
    return u;
}

// Record of a predicted position and a (pre-force) velocity.
__device__ __forceinline__ uint4 make_record(const DevParams& P, float3 pos, float4 vel) {
    const float tx = (pos.x - P.minx) / P.h, ty = (pos.y - P.miny) / P.h, tz = (pos.z - P.minz) / P.h;
    const float fx = floorf(tx), fy = floorf(ty), fz = floorf(tz);
    const float vscale = P.dt / P.h;
    uint4 r;
    r.x = rec_pack_cell((int32_t)fx, (int32_t)fy, (int32_t)fz);
    r.y = rec_h2u(tx - fx, ty - fy);
    r.z = rec_h2u(tz - fz, rec_sat(vel.x * vscale));
    r.w = rec_h2u(rec_sat(vel.y * vscale), rec_sat(vel.z * vscale));
    return r;
}

}  // namespace pfs
