// pfs_geo.cuh — grid search of the neighbour passes (one warp per particle).
//
// The cell table is keyed by hash & (n - 1), so when n - 1 has few set bits
// the table has far fewer slots than particles (n = 300000 leaves 4096) and
// every slot range holds particles of many distant cells.  Scanning those
// ranges is what the shaders do (calculateDensities.comp:114-131,
// applyPressureAndViscosityForce.comp:134-171), but almost every candidate
// fails the distance test.
//
// The grid search finds the same in-range candidates through the spatial
// grid of x* the reorder already builds (order / bcount / boffset: slots
// bucketed by block of 2^bshift cells of x*), sorts them by slot, and then
// walks the 27 table ranges exactly as the scan does, taking from each range
// [start, end) only its in-range members, in slot order.  The lanes of a warp
// gather, sort and evaluate the terms in parallel; the per-particle sums are
// then accumulated in that order by one lane per sum, so they see the same
// terms in the same order as the table scan and the results are
// bit-identical.  Only candidates that cannot contribute are never loaded.
//
// Completeness: a candidate passes the distance test only if it lies within
// h (1 + 2^-20) of x* on every axis.  The grid coordinate u = (x - min) / h
// is computed with two rounded operations, so on a grid of at most
// GEO_MAX_CELLS cells per axis two such points differ in u by less than
// 1 + 2^-10, and the cells floor(u - GEO_REACH) .. floor(u + GEO_REACH)
// (GEO_REACH = 1 + 2^-6) hold every one of them.  Clamping to the grid is
// monotone, so points outside the box land in the edge cells on both sides
// of the comparison.  NaN coordinates give cell 0 and never pass a distance
// test.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"

namespace pfs {

constexpr float GEO_REACH = 1.0f + 1.0f / 64.0f;
// Largest grid (cells per axis) the rounding bound above covers.
constexpr uint32_t GEO_MAX_CELLS = 1024;
// Warps per thread block of the grid-search kernels.
constexpr int GEO_WARPS = 4;

__device__ __forceinline__ void geo_axis(float x, float mn, float h, uint32_t ng, uint32_t shift,
                                         uint32_t& lo, uint32_t& hi) {
    const float u = __fdiv_rn(__fsub_rn(x, mn), h);
    const int32_t top = (int32_t)ng - 1;
    const int32_t a = min(max(__float2int_rz(floorf(__fsub_rn(u, GEO_REACH))), 0), top);
    const int32_t b = min(max(__float2int_rz(floorf(__fadd_rn(u, GEO_REACH))), 0), top);
    lo = (uint32_t)a >> shift;
    hi = (uint32_t)b >> shift;
}

// Called by all 32 lanes: collect the slots j of the spatial-grid blocks
// around (x, y, z) for which test(j) holds into s_j[0, cap).  Returns how many
// passed (entries beyond cap are counted but not stored).  The blocks (at
// most 4 per axis) are flattened into one candidate sequence that the lanes
// walk 32 at a time.
template <class Test>
__device__ __forceinline__ int warp_gather(const DevParams& P, float x, float y, float z,
                                           const uint32_t* __restrict__ bcount,
                                           const uint32_t* __restrict__ boffset,
                                           const uint32_t* __restrict__ order, int32_t* s_j,
                                           int cap, uint32_t* __restrict__ err, Test&& test) {
    const int lane = threadIdx.x & 31;
    const uint32_t n = P.n;
    const uint32_t sh = (uint32_t)P.bshift;
    uint32_t x0, x1, y0, y1, z0, z1;
    geo_axis(x, P.minx, P.h, P.ngx, sh, x0, x1);
    geo_axis(y, P.miny, P.h, P.ngy, sh, y0, y1);
    geo_axis(z, P.minz, P.h, P.ngz, sh, z0, z1);
    const uint32_t wx = x1 - x0 + 1, wy = y1 - y0 + 1;
    const uint32_t nb = wx * wy * (z1 - z0 + 1);  // <= 64
    int m = 0;
    for (uint32_t round = 0; round < nb; round += 32) {
        // lane b holds block round + b: its candidate count and first entry
        const uint32_t b = round + (uint32_t)lane;
        uint32_t c = 0, o = 0;
        if (b < nb) {
            const uint32_t bx = x0 + b % wx, by = y0 + (b / wx) % wy, bz = z0 + b / (wx * wy);
            const uint32_t blk = P.block_base + bx + P.nbx * (by + P.nby * bz);
            c = __ldg(bcount + blk);
            if (c) {
                o = __ldg(boffset + blk);
                if (o > n || c > n - o) {
                    atomicOr(err, ERR_SORT_COUNT);
                    c = 0;
                }
            }
        }
        uint32_t incl = c;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, s);
            if (lane >= s) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t base = 0; base < total; base += 32) {
            const uint32_t t = base + (uint32_t)lane;
            // block of candidate t: the first lane whose inclusive count exceeds t
            int lo = 0, hi = 31;
#pragma unroll
            for (int s = 0; s < 5; s++) {
                const int mid = (lo + hi) >> 1;
                const uint32_t v = __shfl_sync(0xffffffffu, incl, mid);
                if (v <= t)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            const uint32_t bincl = __shfl_sync(0xffffffffu, incl, lo);
            const uint32_t bc = __shfl_sync(0xffffffffu, c, lo);
            const uint32_t bo = __shfl_sync(0xffffffffu, o, lo);
            bool in = false;
            int32_t j = 0;
            if (t < total) {
                j = (int32_t)__ldg(order + bo + (t - (bincl - bc)));
                if ((uint32_t)j >= n)
                    atomicOr(err, ERR_PERM_RANGE);
                else
                    in = test(j);
            }
            const uint32_t mask = __ballot_sync(0xffffffffu, in);
            const int pos = m + __popc(mask & ((1u << lane) - 1u));
            if (in && pos < cap) s_j[pos] = j;
            m += __popc(mask);
        }
    }
    __syncwarp();
    return m;
}

// Called by all 32 lanes: sort s_j[0, m) ascending (bitonic over the next
// power of two, padded with INT32_MAX; that size must not exceed cap).
__device__ __forceinline__ void warp_sort(int32_t* s_j, int m) {
    const int lane = threadIdx.x & 31;
    int p = 2;
    while (p < m) p <<= 1;
    for (int k = m + lane; k < p; k += 32) s_j[k] = 0x7fffffff;
    __syncwarp();
    for (int k = 2; k <= p; k <<= 1) {
        for (int s = k >> 1; s > 0; s >>= 1) {
            for (int q = lane; q < (p >> 1); q += 32) {
                const int a = ((q & ~(s - 1)) << 1) | (q & (s - 1));
                const int b = a + s;
                const int32_t va = s_j[a], vb = s_j[b];
                const bool up = (a & k) == 0;
                if ((va > vb) == up) {
                    s_j[a] = vb;
                    s_j[b] = va;
                }
            }
            __syncwarp();
        }
    }
}

// Work stealing of the persistent grid-search kernels: a warp takes the next
// GEO_CHUNK items from a counter the reorder zeroes each substep (lane 0
// adds, the warp shares the result).  Particles of dense scenes cost many
// times those of sparse ones, so the warps of a batch take work as they free
// up instead of a fixed stride of it.  Called by all 32 lanes.
constexpr uint32_t GEO_CHUNK = 4;
__device__ __forceinline__ uint32_t warp_take(uint32_t* ctr) {
    uint32_t base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(ctr, GEO_CHUNK);
    return __shfl_sync(0xffffffffu, base, 0);
}

// First position k in a[0, m) with a[k] >= key.
__device__ __forceinline__ int geo_lower(const int32_t* a, int m, int32_t key) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Position of slot i in the processing order (n when its block is invalid).
__device__ __forceinline__ uint32_t order_position(uint32_t i, uint32_t n, uint32_t nblocks,
                                                   const uint32_t* __restrict__ bucket,
                                                   const uint32_t* __restrict__ brank,
                                                   const uint32_t* __restrict__ boffset) {
    const uint32_t blk = __ldg(bucket + i);
    if (blk >= nblocks) return n;
    const uint32_t t = __ldg(boffset + blk) + __ldg(brank + i);
    return t < n ? t : n;
}

// Queue of grid-search particles whose force pass must evaluate in full: it
// shares the scan queue's array, filled from the top (entries n-1, n-2, ...)
// and counted in scanq_n[1].
__device__ __forceinline__ uint32_t* geo_queue_entry(uint32_t* scanq, uint32_t n, uint32_t k) {
    return scanq + (n - 1u - k);
}

}  // namespace pfs
