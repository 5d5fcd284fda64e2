// pfs_sort.cu — stable LSD radix sort of (cell key, slot) pairs.
//
// Order contract: the permutation of the reference's VkRadixSort passes
// (src/shaders/multiRadixSortHistograms.comp:39-59,
//  src/shaders/multiRadixSort.comp:54-139, driven by commands.c:106-161):
// sorted by key, ties in ascending slot index.  The reference always runs
// four 8-bit passes; keys here are < n <= 2^24, so only the ceil(log2 n / 8)
// passes that can see a non-zero digit run — a pass over an all-zero digit is
// a stable identity, so the permutation is the same.
//
// One sweep per pass (decoupled look-back), so a sort of P passes is one
// memset and P + 1 kernels instead of the reference's 2 dispatches per pass
// plus barriers:
//   k_sort_upsweep   one read of the keys: the 256-bin histogram of every
//                    pass's digit at once, summed into ghist[P][256]
//   k_sort_onesweep  per pass, tiles of SORT_TILE keys taken in launch order
//                    (a tile counter): stable in-tile rank (warp match +
//                    per-warp counters in the tile's key order), then each
//                    digit's count is published in the tile's look-back word
//                    and the counts of all earlier tiles are summed by
//                    walking back until a tile that already published its
//                    inclusive prefix; the tile then reorders locally in
//                    shared memory and scatters coalesced runs to
//                    base(d) + earlier tiles' count(d) + local rank.
// A look-back word is flag << 30 | count (flag 1: this tile's count, 2: the
// inclusive prefix through this tile).  A tile waits only on tiles that took
// their ids before it, which are resident and publish their count before
// waiting on anything, so every wait ends; the waits are still bounded and
// set ERR_SORT_WAIT if a bound is ever reached.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_sort.cuh"

namespace pfs {

namespace {

constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_IPT = 16;
constexpr int SORT_TILE = SORT_THREADS * SORT_IPT;
constexpr int RADIX = 256;
constexpr int MAX_PASSES = 4;
constexpr uint32_t LB_AGG = 1u << 30;
constexpr uint32_t LB_PREFIX = 2u << 30;
constexpr uint32_t LB_COUNT = (1u << 30) - 1u;
constexpr uint32_t LB_SPIN_LIMIT = 1u << 22;
constexpr int LB_BATCH = 16;  // look-back words loaded at once
// scratch header: ghist (MAX_PASSES * RADIX words), then the tile counters
constexpr size_t HEADER_WORDS = (size_t)MAX_PASSES * RADIX + 64;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Exclusive scan of two sums at once (low and high 32 bits of v, neither
// overflowing) across a 256-thread block.
__device__ __forceinline__ uint64_t block_exclusive_scan2(uint64_t v, uint64_t* s_warp_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp_tot[warp] = incl;
    __syncthreads();
    uint64_t before = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) before += w < warp ? s_warp_tot[w] : 0ull;
    __syncthreads();
    return before + incl - v;
}

// Histograms of all passes' digits in one read of the keys; also clears the
// look-back words the onesweep passes will use (look_words of them).
__global__ void __launch_bounds__(SORT_THREADS)
k_sort_upsweep(const uint32_t* __restrict__ keys, uint32_t n, int passes,
               uint32_t* __restrict__ ghist, uint32_t* __restrict__ look, size_t look_words) {
    __shared__ uint32_t s_h[MAX_PASSES][RADIX];
    for (int i = threadIdx.x; i < MAX_PASSES * RADIX; i += SORT_THREADS) (&s_h[0][0])[i] = 0u;
    __syncthreads();
    const size_t stride = (size_t)gridDim.x * SORT_THREADS;
    for (size_t i = (size_t)blockIdx.x * SORT_THREADS + threadIdx.x; i < look_words; i += stride)
        look[i] = 0u;
    // eight keys in flight per thread before their histogram updates
    constexpr int UP = 8;
    for (size_t i0 = (size_t)blockIdx.x * SORT_THREADS + threadIdx.x; i0 < n; i0 += UP * stride) {
        uint32_t k[UP];
#pragma unroll
        for (int u = 0; u < UP; u++) {
            const size_t i = i0 + (size_t)u * stride;
            k[u] = i < n ? __ldg(keys + i) : 0u;
        }
#pragma unroll
        for (int u = 0; u < UP; u++) {
            if (i0 + (size_t)u * stride >= n) break;
            for (int p = 0; p < passes; p++) atomicAdd(&s_h[p][(k[u] >> (8 * p)) & (RADIX - 1)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RADIX; i += SORT_THREADS) {
        const uint32_t c = (&s_h[0][0])[i];
        if (c) atomicAdd(ghist + i, c);
    }
}

template <bool FIRST>
__global__ void __launch_bounds__(SORT_THREADS, 2)
k_sort_onesweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                int shift, const uint32_t* __restrict__ ghist, uint32_t* __restrict__ tile_ctr,
                uint32_t* __restrict__ look, uint32_t* __restrict__ err) {
    __shared__ uint32_t s_keys[SORT_TILE];
    __shared__ uint32_t s_vals[SORT_TILE];
    __shared__ uint32_t s_warp[SORT_WARPS][RADIX];
    __shared__ uint32_t s_local[RADIX];
    __shared__ uint32_t s_base[RADIX];
    __shared__ uint32_t s_tile;

    __shared__ uint64_t s_tot2[SORT_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    const uint32_t gh = ghist[threadIdx.x];  // this thread's digit total, loaded early
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&s_warp[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t tile = s_tile;

    const uint64_t tile_base = (uint64_t)tile * SORT_TILE;
    const uint64_t base = tile_base + (uint64_t)warp * (32 * SORT_IPT);
    const uint32_t lt = lanemask_lt();
    uint32_t k[SORT_IPT], v[SORT_IPT], r[SORT_IPT];
#pragma unroll
    // every key and value of the thread is loaded before the first match:
    // the ranks are serial (one match per key), the loads need not be
    for (int it = 0; it < SORT_IPT; it++) {
        const uint64_t idx = base + (uint64_t)it * 32 + lane;
        const bool valid = idx < n;
        k[it] = valid ? __ldg(keys_in + idx) : 0xffffffffu;
        v[it] = valid ? (FIRST ? (uint32_t)idx : __ldg(vals_in + idx)) : 0u;
    }
#pragma unroll
    for (int it = 0; it < SORT_IPT; it++) {
        const uint64_t idx = base + (uint64_t)it * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((k[it] >> shift) & (RADIX - 1)) : RADIX;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (valid && lane == leader) {
            before = s_warp[warp][d];
            s_warp[warp][d] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        r[it] = before + __popc(peers & lt);
    }
    __syncthreads();
    // per digit: exclusive offsets across warps (tile key order is warp-major)
    const int d = threadIdx.x;  // SORT_THREADS == RADIX
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) {
        const uint32_t c = s_warp[w][d];
        s_warp[w][d] = cnt;
        cnt += c;
    }
    // publish this tile's count, then sum the earlier tiles' counts
    uint32_t* mine = look + (size_t)tile * RADIX + d;
    uint32_t excl = 0;
    if (tile == 0) {
        st_relaxed(mine, LB_PREFIX | cnt);
    } else {
        st_relaxed(mine, LB_AGG | cnt);
        // LB_BATCH earlier tiles' words are loaded at once, then summed in
        // order (nearest first) up to the first inclusive prefix; a word not
        // yet published is waited for, with a bound
        bool done = false;
        for (int32_t t = (int32_t)tile - 1; t >= 0 && !done; t -= LB_BATCH) {
            uint32_t word[LB_BATCH];
#pragma unroll
            for (int q = 0; q < LB_BATCH; q++)
                word[q] = t - q >= 0 ? ld_relaxed(look + (size_t)(t - q) * RADIX + d) : LB_PREFIX;
#pragma unroll
            for (int q = 0; q < LB_BATCH; q++) {
                if (done) break;
                uint32_t wq = word[q];
                if ((wq & ~LB_COUNT) == 0u) {
                    const uint32_t* wp = look + (size_t)(t - q) * RADIX + d;
                    uint32_t spins = 0;
                    while ((wq & ~LB_COUNT) == 0u && ++spins < LB_SPIN_LIMIT) {
                        __nanosleep(20);
                        wq = ld_relaxed(wp);
                    }
                    if ((wq & ~LB_COUNT) == 0u) {
                        atomicOr(err, ERR_SORT_WAIT);
                        done = true;
                        break;
                    }
                }
                excl += wq & LB_COUNT;
                if ((wq & ~LB_COUNT) == LB_PREFIX) done = true;
            }
        }
        st_relaxed(mine, LB_PREFIX | ((excl + cnt) & LB_COUNT));
    }
    // the tile's digit offsets and the digits' global bases in one scan
    const uint64_t both = block_exclusive_scan2(((uint64_t)gh << 32) | cnt, s_tot2);
    s_local[d] = (uint32_t)both;
    s_base[d] = (uint32_t)(both >> 32) + excl;
    __syncthreads();
#pragma unroll
    for (int it = 0; it < SORT_IPT; it++) {
        const uint64_t idx = base + (uint64_t)it * 32 + lane;
        if (idx < n) {
            const uint32_t dd = (k[it] >> shift) & (RADIX - 1);
            const uint32_t pos = s_local[dd] + s_warp[warp][dd] + r[it];
            if (pos < SORT_TILE) {
                s_keys[pos] = k[it];
                s_vals[pos] = v[it];
            } else {
                atomicOr(err, ERR_SORT_COUNT);
            }
        }
    }
    __syncthreads();
    const uint32_t count = tile_base < n ? (uint32_t)min((uint64_t)SORT_TILE, (uint64_t)n - tile_base) : 0u;
    for (uint32_t i = threadIdx.x; i < count; i += SORT_THREADS) {
        const uint32_t key = s_keys[i];
        const uint32_t dd = (key >> shift) & (RADIX - 1);
        const uint32_t dst = s_base[dd] + (i - s_local[dd]);
        if (dst < n) {
            keys_out[dst] = key;
            vals_out[dst] = s_vals[i];
        } else {
            atomicOr(err, ERR_SORT_COUNT);
        }
    }
}

__global__ void k_identity(const uint32_t* __restrict__ keys_in, uint32_t n,
                           uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        keys_out[i] = keys_in[i];
        vals_out[i] = i;
    }
}

// Upsweep grid: a few blocks per SM, striding over the keys (measured: one
// block per SM leaves the pass latency-bound, 21 us against 14 us at 1M).
unsigned upsweep_blocks(uint32_t n) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const unsigned want = (n + SORT_TILE - 1) / SORT_TILE;
    return std::max(1u, std::min(want, (unsigned)(4 * sms)));
}

}  // namespace

int sort_key_bits(uint32_t n) { return n <= 1 ? 0 : 32 - __builtin_clz(n - 1u); }

int sort_passes(uint32_t n) { return (sort_key_bits(n) + 7) / 8; }

uint32_t sort_tiles(uint32_t n) { return (n + SORT_TILE - 1) / SORT_TILE; }

size_t sort_scratch_words(uint32_t n, int key_bits) {
    const int passes = (key_bits + 7) / 8;
    const size_t tiles = sort_tiles(n) > 0 ? sort_tiles(n) : 1;
    return HEADER_WORDS + (size_t)(passes > 0 ? passes : 1) * tiles * RADIX;
}

int sort_launches(uint32_t n) {
    const int p = sort_passes(n);
    return p == 0 ? 1 : 1 + p;
}

cudaError_t sort_pairs(const uint32_t* keys_in, uint32_t n, int key_bits, uint32_t* keys_out,
                       uint32_t* vals_out, uint32_t* keys_tmp, uint32_t* vals_tmp,
                       uint32_t* scratch, uint32_t* err, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const int passes = (key_bits + 7) / 8;
    if (passes == 0) {
        k_identity<<<(n + 255) / 256, 256, 0, stream>>>(keys_in, n, keys_out, vals_out);
        return cudaGetLastError();
    }
    if (passes > MAX_PASSES) return cudaErrorInvalidValue;
    const uint32_t tiles = sort_tiles(n);
    uint32_t* ghist = scratch;
    uint32_t* tile_ctr = scratch + (size_t)MAX_PASSES * RADIX;
    uint32_t* look = scratch + HEADER_WORDS;
    const size_t look_words = (size_t)passes * tiles * RADIX;
    cudaError_t e = cudaMemsetAsync(scratch, 0, HEADER_WORDS * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    k_sort_upsweep<<<upsweep_blocks(n), SORT_THREADS, 0, stream>>>(keys_in, n, passes, ghist, look,
                                                                    look_words);
    const uint32_t* kin = keys_in;
    const uint32_t* vin = nullptr;
    for (int p = 0; p < passes; p++) {
        // the last pass lands in keys_out/vals_out
        const bool to_final = ((passes - 1 - p) % 2) == 0;
        uint32_t* kout = to_final ? keys_out : keys_tmp;
        uint32_t* vout = to_final ? vals_out : vals_tmp;
        const int shift = 8 * p;
        uint32_t* lp = look + (size_t)p * tiles * RADIX;
        if (p == 0)
            k_sort_onesweep<true><<<tiles, SORT_THREADS, 0, stream>>>(
                kin, vin, kout, vout, n, shift, ghist + p * RADIX, tile_ctr + p, lp, err);
        else
            k_sort_onesweep<false><<<tiles, SORT_THREADS, 0, stream>>>(
                kin, vin, kout, vout, n, shift, ghist + p * RADIX, tile_ctr + p, lp, err);
        kin = kout;
        vin = vout;
    }
    return cudaGetLastError();
}

}  // namespace pfs
