// pfs_flat.cuh — the flat walk over a particle's 27 table ranges, shared by
// the FP32 density pass (k_density_flat, pfs_neighbors.cu) and the FP16-cell
// density pass (k_density16_flat, pfs_fp16.cu).  The candidates and their
// order are calculateDensities.comp:114-131's (27 sample cells in order, each
// slot's run in table order); only the layout of the work on the warp is
// this file's:
//   1. each thread looks up its own particle's 27 table ranges (a row's nine
//      entries loaded together) and keeps the non-empty ones, in walk order,
//      as packed words in shared memory (start | length << 24 | sample-point
//      flag << 31; a range longer than FLAT_LEN_MAX takes several words);
//   2. the block sorts its particles by candidate total (bitonic: in-warp
//      stages by shuffle, cross-warp stages through shared memory), so the
//      lanes of a warp walk totals of similar length; the particles of one
//      cell have equal totals and stay next to each other, so their
//      candidate loads still coincide; each thread then moves the words of
//      the particle it walks into its own column;
//   3. one loop of warp-uniform, even trip count (the largest total of the
//      warp's particles) runs over the concatenated ranges, two candidates
//      per iteration: each step tests the lane's current candidate (lanes
//      past their total test their own slot and discard it) and moves a
//      branch-free cursor to the next one, whose data is loaded one step
//      ahead; warps whose ranges all have in-box sample points run a copy of
//      the loop that keeps no flag.
// A particle whose ranges need more than FLAT_RCAP words walks the table
// from global memory instead (the caller's fallback) and goes to the force
// pass's scan queue.  Indices fit the packed start: n <= 2^24.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "pfs_common.cuh"

namespace pfs {
namespace {

constexpr int FLAT_THREADS = 128;       // threads per block (column in 7 bits)
constexpr int FLAT_RCAP = 28;           // range words per particle (a multiple of 4)
constexpr uint32_t FLAT_LEN_MAX = 127;  // candidates per range word
static_assert(PFS_MAX_PARTICLES <= (1u << 24), "packed range start");
static_assert(FLAT_RCAP % 4 == 0, "moved in four parts");

// Per-column flags of phase 1.
enum : uint32_t { FLAT_LIVE = 1u, FLAT_LIST_OK = 4u, FLAT_OVER = 8u, FLAT_ALLF = 16u };

struct FlatShared {
    uint32_t rng[FLAT_RCAP][FLAT_THREADS];  // per column: packed ranges
    uint32_t key[FLAT_THREADS];             // sort exchange buffer
    uint8_t meta[FLAT_THREADS];             // per column: FLAT_* flags
};

// Phase 1: the ranges of this thread's own particle (column threadIdx.x).
// Returns its sort key, candidate total << 7 | column (total 0 for a
// particle that walks nothing here).
template <bool BATCH>
__device__ __forceinline__ uint32_t flat_ranges(const DevParams& P0, const SceneRef& sr,
                                                const float4* __restrict__ xp,
                                                const int2* __restrict__ table,
                                                const uint32_t* __restrict__ order,
                                                uint32_t* __restrict__ err, FlatShared& S) {
    const int tid = threadIdx.x;
    const uint32_t n = P0.n;
    const uint32_t t = blockIdx.x * FLAT_THREADS + tid;
    uint32_t i = 0;
    bool live = t < n;
    if (live) {
        i = order[t];
        if (i >= n) {
            atomicOr(err, ERR_PERM_RANGE);
            live = false;
        }
    }
    const DevParams P = params_of<BATCH>(P0, sr, live ? i : 0u);
    if (P.geo) live = false;  // the grid-search pass takes it
    const float4 sp = live ? xp[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float h = P.h;
    const float off[3] = {PFS_MUL(h, -1.0f), PFS_MUL(h, 0.0f), h};
    uint32_t hx[3], hy[3], hz[3];
    bool vx[3], vy[3], vz[3];
    int32_t cx[3], cy[3], cz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float sx = PFS_ADD(sp.x, off[a]), sy = PFS_ADD(sp.y, off[a]), sz = PFS_ADD(sp.z, off[a]);
        vx[a] = live && !(sx < P.minx) && !(sx > P.maxx);
        vy[a] = !(sy < P.miny) && !(sy > P.maxy);
        vz[a] = !(sz < P.minz) && !(sz > P.maxz);
        cx[a] = cell_coord(sx, P.minx, h);
        cy[a] = cell_coord(sy, P.miny, h);
        cz[a] = cell_coord(sz, P.minz, h);
    }
    // the sample-point cells are the force pass's 27 cell offsets: the
    // particle's in-range candidates are its force-pass list
    const bool listing = vx[1] && vy[1] && vz[1] && (!vx[0] || cx[0] == cx[1] - 1) &&
                         (!vx[2] || cx[2] == cx[1] + 1) && (!vy[0] || cy[0] == cy[1] - 1) &&
                         (!vy[2] || cy[2] == cy[1] + 1) && (!vz[0] || cz[0] == cz[1] - 1) &&
                         (!vz[2] || cz[2] == cz[1] + 1);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        hx[a] = (uint32_t)(listing ? cx[1] + a - 1 : cx[a]) * 73856093u;
        hy[a] = (uint32_t)(listing ? cy[1] + a - 1 : cy[a]) * 19349663u;
        hz[a] = (uint32_t)(listing ? cz[1] + a - 1 : cz[a]) * 83492791u;
    }
    bool list_ok = listing;
    int nr = 0;
    uint32_t tot = 0;
    bool allf = true;  // every stored range has its sample point in the box
#pragma unroll 1
    for (int dz = 0; dz < 3; dz++) {
        const bool vzz = dz == 0 ? vz[0] : (dz == 1 ? vz[1] : vz[2]);
        const uint32_t hzz = dz == 0 ? hz[0] : (dz == 1 ? hz[1] : hz[2]);
        // the row's nine table entries are loaded together (a slot is always
        // inside the table), then taken in walk order
        int2 row[9];
#pragma unroll
        for (int q = 0; q < 9; q++)
            row[q] = __ldg(table + slot_of(P, hash_finalize(hx[q % 3] ^ hy[q / 3] ^ hzz)));
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int dy = q / 3, dx = q % 3;
            const bool dens = vx[dx] && vy[dy] && vzz;
            if (!(dens || listing)) continue;
            const int2 se = row[q];
            if (se.x == -1) continue;
            if (se.x < 0 || se.y > (int32_t)n || se.x > se.y) {
                atomicOr(err, ERR_TABLE_RANGE);
                list_ok = false;
                continue;
            }
            uint32_t s0 = (uint32_t)se.x, len = (uint32_t)(se.y - se.x);
            tot += len;
            allf = allf && (dens || len == 0);
            const uint32_t flag = dens ? 0x80000000u : 0u;
            if (len - 1u < FLAT_LEN_MAX) {  // one word (empty ranges take none)
                if (nr < FLAT_RCAP) S.rng[nr][tid] = s0 | (len << 24) | flag;
                nr++;
            } else {
                while (len > 0) {
                    const uint32_t l = min(len, FLAT_LEN_MAX);
                    if (nr < FLAT_RCAP) S.rng[nr][tid] = s0 | (l << 24) | flag;
                    nr++;
                    s0 += l;
                    len -= l;
                }
            }
        }
    }
    const bool over = nr > FLAT_RCAP;
    if (nr == 0 || over) S.rng[0][tid] = 0u;  // an empty walk
    S.meta[tid] = (uint8_t)((live ? FLAT_LIVE : 0u) | (list_ok ? FLAT_LIST_OK : 0u) | (over ? FLAT_OVER : 0u) |
                            (allf ? FLAT_ALLF : 0u));
    return ((over ? 0u : tot) << 7) | (uint32_t)tid;
}

// Phase 2: the block's keys in ascending order, thread k holding the k-th.
// In-warp partners by shuffle; cross-warp partners through S.key and buf1
// taken in turn (one barrier per such stage; the first also publishes phase
// 1's words and flags).  buf1 holds FLAT_THREADS words the caller does not
// use until the walk.
__device__ __forceinline__ uint32_t flat_sort(uint32_t key, uint32_t* buf1, FlatShared& S) {
    const int tid = threadIdx.x;
    uint32_t* buf[2] = {S.key, buf1};
    int nb = 0;
#pragma unroll
    for (int k = 2; k <= FLAT_THREADS; k <<= 1) {
#pragma unroll
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            uint32_t pk;
            if (jj < 32) {
                pk = __shfl_xor_sync(0xffffffffu, key, jj);
            } else {
                buf[nb][tid] = key;
                __syncthreads();
                pk = buf[nb][tid ^ jj];
                nb ^= 1;
            }
            const bool keep_min = ((tid & jj) == 0) == ((tid & k) == 0);
            key = keep_min ? min(key, pk) : max(key, pk);
        }
    }
    return key;
}

// The words of column src into this thread's own column: the columns a warp
// walks are scattered over the block, so reading them in place would collide
// in the shared-memory banks on every step of the walk.
__device__ __forceinline__ void flat_move(int src, FlatShared& S) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int c0 = 0; c0 < FLAT_RCAP; c0 += FLAT_RCAP / 4) {
        uint32_t wv[FLAT_RCAP / 4];
#pragma unroll
        for (int k = 0; k < FLAT_RCAP / 4; k++) wv[k] = S.rng[c0 + k][src];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < FLAT_RCAP / 4; k++) S.rng[c0 + k][tid] = wv[k];
        __syncthreads();
    }
}

// Phase 3: the walk of this thread's column, tot candidates; load(j) loads
// candidate j's data, test(q, j, flagged, valid) takes it, pair() runs after
// every second step (the caller's buffer drain).  Lanes past their total
// load their own slot self and test it as invalid.
template <class Load, class Test, class Pair>
__device__ __forceinline__ void flat_walk(const FlatShared& S, int32_t tot, int32_t self, bool all_flagged,
                                          Load&& load, Test&& test, Pair&& pair) {
    const int tid = threadIdx.x;
    // an even trip count, so the loop body takes two candidates without a
    // mid-body exit
    const int32_t trips = (__reduce_max_sync(0xffffffffu, tot) + 1) & ~1;
    auto walk = [&](auto allf_tag) {
        constexpr bool ALLF = decltype(allf_tag)::value;
        // cursor: candidate j of range word r (end jend, sample-point flag
        // f); it steps to the next word only while the lane has candidates
        // left, so it never passes the column's last word
        int r = 0;
        int32_t j, jend;
        bool f;
        {
            const uint32_t w = S.rng[0][tid];
            j = (int32_t)(w & 0xffffffu);
            jend = j + (int32_t)((w >> 24) & 127u);
            f = (int32_t)w < 0;
        }
        auto step = [&](bool more) {
            j++;
            const bool adv = more && j == jend;
            r += adv ? 1 : 0;
            const uint32_t w = S.rng[r][tid];
            const int32_t js = (int32_t)(w & 0xffffffu);
            j = adv ? js : j;
            jend = adv ? js + (int32_t)((w >> 24) & 127u) : jend;
            if constexpr (!ALLF) f = adv ? (int32_t)w < 0 : f;
        };
        int32_t ja = j;
        bool fa = ALLF || f;
        auto qa = load(0 < tot ? j : self);
        step(0 < tot);
        for (int32_t k = 0; k < trips; k += 2) {
            const int32_t jb = j;
            const bool fb = ALLF || f;
            const auto qb = load(k + 1 < tot ? j : self);
            step(k + 1 < tot);
            test(qa, ja, fa, k < tot);
            ja = j;
            fa = ALLF || f;
            qa = load(k + 2 < tot ? j : self);
            step(k + 2 < tot);
            test(qb, jb, fb, k + 1 < tot);
            pair();
        }
    };
    if (__all_sync(0xffffffffu, all_flagged))
        walk(std::true_type{});
    else
        walk(std::false_type{});
}

// The scan queue: positions whose density pass wrote no usable list.
__device__ __forceinline__ void flat_enqueue(bool scan, uint32_t t, uint32_t* __restrict__ scanq,
                                             uint32_t* __restrict__ scanq_n) {
    const int lane = threadIdx.x & 31;
    const uint32_t want = __ballot_sync(0xffffffffu, scan);
    if (want) {
        const int leader = __ffs(want) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(scanq_n, (uint32_t)__popc(want));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (scan) scanq[base + __popc(want & ((1u << lane) - 1u))] = t;
    }
}

}  // namespace
}  // namespace pfs
