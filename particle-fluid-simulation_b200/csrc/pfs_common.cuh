// pfs_common.cuh — device-side parameter block and the arithmetic shared by
// every step kernel.
//
// All float arithmetic on the parity path goes through the *_rn intrinsics
// below: one IEEE round-to-nearest operation each, never fused into an FMA, in
// the order the reference shaders write the expression.  Together with the
// host-derived constants (same code as the oracle) this makes the FP32 step
// bit-identical to the CPU restatement of the shaders.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pfs.h"

namespace pfs {

// Device error word bits (atomicOr'd by kernels whose own bounds checks trip).
enum : uint32_t {
    ERR_TABLE_RANGE = 1u << 0,   // a cell table range outside [0, n]
    ERR_PERM_RANGE  = 1u << 1,   // a sort permutation entry >= n
    ERR_KEY_RANGE   = 1u << 2,   // a sorted key > mask
    ERR_SORT_COUNT  = 1u << 3,   // radix pass placed an element out of range
    ERR_SCENE_RANGE = 1u << 4,   // batched: scene id / segment out of range
    ERR_SORT_WAIT   = 1u << 5,   // a sort tile gave up waiting on an earlier tile
};

// Parameters as the kernels see them: the public pfs_params plus the
// constants derived on the host (pfs_derive, identical to the oracle's).
struct DevParams {
    float h, rho0, k, kn, visc, m;
    float gx, gy, gz, dt;
    float minx, miny, minz, maxx, maxy, maxz;
    float margin_p, margin_i;
    float rest[6];
    float volume, near_inv, slope_scale, near_slope_scale, r2, skip_d2;
    uint32_t mask;
    uint32_t n;
    int32_t flags;
    // spatial processing order of the neighbour passes: x* cells clamped to
    // [0, ng?-1] are grouped into blocks of 2^bshift cells per axis, nb? blocks
    // per axis (row-major block id)
    uint32_t ngx, ngy, ngz;
    uint32_t nbx, nby, nbz;
    int32_t bshift;
    // batched scenes: the scene's slice of the shared key space (table slots
    // key_base .. key_base + mask) and of the spatial-order blocks; 0 for a
    // world.  n is the particle count of the whole table either way.
    uint32_t key_base;
    uint32_t block_base;
    // neighbour search: 0 scans the table ranges, 1 finds the in-range
    // candidates through the spatial grid (same results, pfs_geo.cuh)
    uint32_t geo;
    // rows of the neighbour-list buffer: particles with more in-range
    // neighbours than this are scanned by the force pass instead
    uint32_t list_cap;
    // staged shape (pfs_staged.cu): blocks of 2^sbx x 2^sby x 2^sbz cells,
    // nsx x nsy x nsz of them; when `staged` is set the spatial order
    // buckets particles by (block, cell in block), so each block's
    // particles are contiguous and in cell order
    uint32_t staged;
    int32_t sbx, sby, sbz;
    uint32_t nsx, nsy, nsz;
    // the least float whose square root is at least 1e-7 (the force pass's
    // coincident-particle cut, applyPressureAndViscosityForce.comp:150)
    float min_d2;
};

// Per-slot scene parameters of a batch (null scenes: one world, the kernel's
// own DevParams apply to every slot).
struct SceneRef {
    const DevParams* __restrict__ scenes;
    const uint32_t* __restrict__ sid;
};

// Parameters that apply to slot s: kernels take a copy, so only the fields
// they use are loaded.
template <bool BATCH>
__device__ __forceinline__ DevParams params_of(const DevParams& P0, const SceneRef& sr, uint32_t s) {
    if constexpr (BATCH) {
        return sr.scenes[sr.sid[s]];
    } else {
        return P0;
    }
}

// Block (bucket) of a predicted position for the spatial processing order.
__device__ __forceinline__ uint32_t spatial_block(const DevParams& P, float x, float y, float z) {
    int32_t cx = __float2int_rz(floorf(__fdiv_rn(__fsub_rn(x, P.minx), P.h)));
    int32_t cy = __float2int_rz(floorf(__fdiv_rn(__fsub_rn(y, P.miny), P.h)));
    int32_t cz = __float2int_rz(floorf(__fdiv_rn(__fsub_rn(z, P.minz), P.h)));
    cx = min(max(cx, 0), (int32_t)P.ngx - 1);
    cy = min(max(cy, 0), (int32_t)P.ngy - 1);
    cz = min(max(cz, 0), (int32_t)P.ngz - 1);
    const uint32_t bx = (uint32_t)cx >> P.bshift, by = (uint32_t)cy >> P.bshift,
                   bz = (uint32_t)cz >> P.bshift;
    return P.block_base + bx + P.nbx * (by + P.nby * bz);
}

// Bucket of the spatial processing order: the block of x* (spatial_block),
// or with the staged shape the (block, cell in block) fine bucket, numbered
// so that each block's cells are consecutive.
__device__ __forceinline__ uint32_t spatial_bucket(const DevParams& P, float x, float y, float z) {
    if (!P.staged) return spatial_block(P, x, y, z);
    int32_t cx = __float2int_rz(floorf(__fdiv_rn(__fsub_rn(x, P.minx), P.h)));
    int32_t cy = __float2int_rz(floorf(__fdiv_rn(__fsub_rn(y, P.miny), P.h)));
    int32_t cz = __float2int_rz(floorf(__fdiv_rn(__fsub_rn(z, P.minz), P.h)));
    cx = min(max(cx, 0), (int32_t)P.ngx - 1);
    cy = min(max(cy, 0), (int32_t)P.ngy - 1);
    cz = min(max(cz, 0), (int32_t)P.ngz - 1);
    const uint32_t bx = (uint32_t)cx >> P.sbx, by = (uint32_t)cy >> P.sby, bz = (uint32_t)cz >> P.sbz;
    const uint32_t lx = (uint32_t)cx & ((1u << P.sbx) - 1u), ly = (uint32_t)cy & ((1u << P.sby) - 1u),
                   lz = (uint32_t)cz & ((1u << P.sbz) - 1u);
    const uint32_t blk = bx + P.nsx * (by + P.nsy * bz);
    return (blk << (P.sbx + P.sby + P.sbz)) | lx | (ly << P.sbx) | (lz << (P.sbx + P.sby));
}

#define PFS_ADD(a, b) __fadd_rn((a), (b))
#define PFS_SUB(a, b) __fsub_rn((a), (b))
#define PFS_MUL(a, b) __fmul_rn((a), (b))
#define PFS_DIV(a, b) __fdiv_rn((a), (b))
#define PFS_SQRT(a)   __fsqrt_rn((a))

// cellCoordToHash (updateCellEntries.comp:36-52): the xor of the three
// products is split so callers can precompute per-axis products.
__device__ __forceinline__ uint32_t hash_finalize(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}
__device__ __forceinline__ uint32_t cell_hash(uint32_t cx, uint32_t cy, uint32_t cz) {
    return hash_finalize((cx * 73856093u) ^ (cy * 19349663u) ^ (cz * 83492791u));
}

// ivec3(floor((p - minXYZ) / smoothingRadius)), one axis.  cvt.rzi.s32.f32
// saturates out-of-range values and maps NaN to 0.
__device__ __forceinline__ int32_t cell_coord(float v, float lo, float h) {
    return __float2int_rz(floorf(PFS_DIV(PFS_SUB(v, lo), h)));
}

// Key of a position (updateCellEntries.comp:72-79), as a slot of the shared
// table (key_base is 0 for a world).
__device__ __forceinline__ uint32_t point_key(const DevParams& P, float x, float y, float z) {
    uint32_t cx = (uint32_t)cell_coord(x, P.minx, P.h);
    uint32_t cy = (uint32_t)cell_coord(y, P.miny, P.h);
    uint32_t cz = (uint32_t)cell_coord(z, P.minz, P.h);
    return P.key_base + (cell_hash(cx, cy, cz) & P.mask);
}

// Table slot of a hash: the scene's slice of the shared table.
__device__ __forceinline__ uint32_t slot_of(const DevParams& P, uint32_t hash) {
    return P.key_base + (hash & P.mask);
}

// Wall clamp + reflect for one axis (predictPositions.comp:80-113,
// updateVelocities.comp:83-115): negate the hit component, then scale it by
// that wall's restitution (reference: 1.0 everywhere except z-min 0.95).
__device__ __forceinline__ void wall_axis(float lo0, float hi0, float margin, float r_lo,
                                          float r_hi, float& x, float& v) {
    const float lo = PFS_ADD(lo0, margin);
    const float hi = PFS_SUB(hi0, margin);
    if (x < lo) {
        x = lo;
        v = PFS_MUL(PFS_MUL(v, -1.0f), r_lo);
    } else if (x > hi) {
        x = hi;
        v = PFS_MUL(PFS_MUL(v, -1.0f), r_hi);
    }
}

__device__ __forceinline__ void walls(const DevParams& P, float margin, float3& pos, float3& vel) {
    wall_axis(P.minx, P.maxx, margin, P.rest[0], P.rest[1], pos.x, vel.x);
    wall_axis(P.miny, P.maxy, margin, P.rest[2], P.rest[3], pos.y, vel.y);
    wall_axis(P.minz, P.maxz, margin, P.rest[4], P.rest[5], pos.z, vel.z);
}

// v += g dt; x += v dt; walls.  Shared by predict (margin particleRadius,
// predictPositions.comp:74-113) and integrate (margin particleRadius + 0.5,
// updateVelocities.comp:75-115; its extra "* dt_scale" with dt_scale = 1.0
// is an exact identity).
__device__ __forceinline__ void euler_walls(const DevParams& P, float margin, float3& pos,
                                            float3& vel) {
    vel.x = PFS_ADD(vel.x, PFS_MUL(P.gx, P.dt));
    vel.y = PFS_ADD(vel.y, PFS_MUL(P.gy, P.dt));
    vel.z = PFS_ADD(vel.z, PFS_MUL(P.gz, P.dt));
    pos.x = PFS_ADD(pos.x, PFS_MUL(vel.x, P.dt));
    pos.y = PFS_ADD(pos.y, PFS_MUL(vel.y, P.dt));
    pos.z = PFS_ADD(pos.z, PFS_MUL(vel.z, P.dt));
    walls(P, margin, pos, vel);
}

// Speed colour ramp (updateVelocities.comp:120-141).
__device__ __forceinline__ float4 speed_color(float3 v) {
    const float speed =
        PFS_SQRT(PFS_ADD(PFS_ADD(PFS_MUL(v.x, v.x), PFS_MUL(v.y, v.y)), PFS_MUL(v.z, v.z)));
    float t = PFS_DIV(speed, 60.0f);
    t = t < 0.0f ? 0.0f : t;
    t = t > 1.0f ? 1.0f : t;
    float3 a, b;
    float u;
    if (t < 0.33f) {
        a = make_float3(0.3f, 0.3f, 1.0f); b = make_float3(0.0f, 1.0f, 1.0f);
        u = PFS_DIV(t, 0.33f);
    } else if (t < 0.66f) {
        a = make_float3(0.0f, 1.0f, 1.0f); b = make_float3(1.0f, 1.0f, 0.0f);
        u = PFS_DIV(PFS_SUB(t, 0.33f), 0.33f);
    } else {
        a = make_float3(1.0f, 1.0f, 0.0f); b = make_float3(1.0f, 0.3f, 0.3f);
        u = PFS_DIV(PFS_SUB(t, 0.66f), 0.34f);
    }
    const float w = PFS_SUB(1.0f, u);
    return make_float4(PFS_ADD(PFS_MUL(a.x, w), PFS_MUL(b.x, u)),
                       PFS_ADD(PFS_MUL(a.y, w), PFS_MUL(b.y, u)),
                       PFS_ADD(PFS_MUL(a.z, w), PFS_MUL(b.z, u)), 1.0f);
}

// Host: derive DevParams from pfs_params (same arithmetic as the oracle's
// pfso_derive, which the GPU parity tests rely on).
// search: -1 automatic (or PFS_NEIGHBOR_SEARCH), 0 table scan, 1 grid search
// (where the grid bound allows it).
void derive_params(const pfs_params& p, uint32_t n, DevParams* out, int search = -1);
// The grid search is possible for this table and box.
bool grid_search_allowed(const pfs_params& p, uint32_t n);
// Buckets of the spatial processing order.
uint32_t spatial_blocks(const DevParams& P);
// Coarsen the spatial-order blocks until at most `cap` remain.
void fit_spatial_blocks(DevParams* P, uint32_t cap);

}  // namespace pfs
