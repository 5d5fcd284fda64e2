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
// Each pass is reduce-then-scan over tiles of SORT_TILE keys:
//   k_radix_hist     per-tile digit histogram, bin-major  hist[d * T + t]
//   k_radix_scan     per-digit exclusive scan over tiles + digit totals
//   k_radix_scatter  stable in-tile rank (warp match + per-warp counters in
//                    the tile's key order), local reorder in shared memory,
//                    coalesced scatter to  base(d) + hist[d][t] + local rank.
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

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread across a 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp_tot,
                                                         uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < SORT_WARPS ? s_warp_tot[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < SORT_WARPS) s_warp_tot[lane] = wi - w;
        if (lane == SORT_WARPS - 1 && total) *total = wi;
    }
    __syncthreads();
    const uint32_t r = s_warp_tot[warp] + incl - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SORT_THREADS)
k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, int shift, uint32_t tiles,
             uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_h[SORT_WARPS][RADIX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&s_h[0][0])[i] = 0u;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * SORT_TILE + (uint64_t)warp * (32 * SORT_IPT);
#pragma unroll 4
    for (int it = 0; it < SORT_IPT; it++) {
        const uint64_t idx = base + (uint64_t)it * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((__ldg(keys + idx) >> shift) & (RADIX - 1)) : RADIX;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (valid && lane == __ffs(peers) - 1) s_h[warp][d] += __popc(peers);
    }
    __syncthreads();
    const int d = threadIdx.x;  // SORT_THREADS == RADIX
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) c += s_h[w][d];
    hist[(size_t)d * tiles + blockIdx.x] = c;
}

// One block per digit: exclusive scan of hist[d][0..tiles) in place.
__global__ void __launch_bounds__(SORT_THREADS)
k_radix_scan(uint32_t* __restrict__ hist, uint32_t tiles, uint32_t* __restrict__ digit_total) {
    __shared__ uint32_t s_tot[SORT_WARPS];
    __shared__ uint32_t s_total;
    uint32_t* row = hist + (size_t)blockIdx.x * tiles;
    const uint32_t per = (tiles + SORT_THREADS - 1) / SORT_THREADS;
    const uint32_t b = threadIdx.x * per;
    const uint32_t e = min(b + per, tiles);
    uint32_t sum = 0;
    for (uint32_t t = b; t < e; t++) sum += row[t];
    uint32_t run = block_exclusive_scan(sum, s_tot, &s_total);
    for (uint32_t t = b; t < e; t++) {
        const uint32_t c = row[t];
        row[t] = run;
        run += c;
    }
    if (threadIdx.x == 0) digit_total[blockIdx.x] = s_total;
}

template <bool FIRST>
__global__ void __launch_bounds__(SORT_THREADS)
k_radix_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
                int shift, uint32_t tiles, const uint32_t* __restrict__ hist,
                const uint32_t* __restrict__ digit_total, uint32_t* __restrict__ err) {
    __shared__ uint32_t s_keys[SORT_TILE];
    __shared__ uint32_t s_vals[SORT_TILE];
    __shared__ uint32_t s_warp[SORT_WARPS][RADIX];
    __shared__ uint32_t s_local[RADIX];
    __shared__ uint32_t s_base[RADIX];
    __shared__ uint32_t s_tot[SORT_WARPS];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&s_warp[0][0])[i] = 0u;
    __syncthreads();

    const uint64_t tile_base = (uint64_t)blockIdx.x * SORT_TILE;
    const uint64_t base = tile_base + (uint64_t)warp * (32 * SORT_IPT);
    const uint32_t lt = lanemask_lt();
    uint32_t k[SORT_IPT], v[SORT_IPT], r[SORT_IPT];
#pragma unroll
    for (int it = 0; it < SORT_IPT; it++) {
        const uint64_t idx = base + (uint64_t)it * 32 + lane;
        const bool valid = idx < n;
        k[it] = valid ? __ldg(keys_in + idx) : 0xffffffffu;
        v[it] = valid ? (FIRST ? (uint32_t)idx : __ldg(vals_in + idx)) : 0u;
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
    const int d = threadIdx.x;
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) {
        const uint32_t c = s_warp[w][d];
        s_warp[w][d] = cnt;
        cnt += c;
    }
    const uint32_t local = block_exclusive_scan(cnt, s_tot, nullptr);
    const uint32_t dtot = digit_total[d];
    const uint32_t dbase = block_exclusive_scan(dtot, s_tot, nullptr);
    s_local[d] = local;
    s_base[d] = dbase + hist[(size_t)d * tiles + blockIdx.x];
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
    const uint32_t count = (uint32_t)min((uint64_t)SORT_TILE, (uint64_t)n - tile_base);
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

}  // namespace

int sort_key_bits(uint32_t n) { return n <= 1 ? 0 : 32 - __builtin_clz(n - 1u); }

int sort_passes(uint32_t n) { return (sort_key_bits(n) + 7) / 8; }

uint32_t sort_tiles(uint32_t n) { return (n + SORT_TILE - 1) / SORT_TILE; }

size_t sort_hist_words(uint32_t n) { return (size_t)RADIX * (sort_tiles(n) > 0 ? sort_tiles(n) : 1); }

int sort_launches(uint32_t n) {
    const int p = sort_passes(n);
    return p == 0 ? 1 : 3 * p;
}

cudaError_t sort_pairs(const uint32_t* keys_in, uint32_t n, int key_bits, uint32_t* keys_out,
                       uint32_t* vals_out, uint32_t* keys_tmp, uint32_t* vals_tmp,
                       uint32_t* hist, uint32_t* digit_total, uint32_t* err,
                       cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const int passes = (key_bits + 7) / 8;
    if (passes == 0) {
        k_identity<<<(n + 255) / 256, 256, 0, stream>>>(keys_in, n, keys_out, vals_out);
        return cudaGetLastError();
    }
    const uint32_t tiles = sort_tiles(n);
    const uint32_t* kin = keys_in;
    const uint32_t* vin = nullptr;
    for (int p = 0; p < passes; p++) {
        // the last pass lands in keys_out/vals_out
        const bool to_final = ((passes - 1 - p) % 2) == 0;
        uint32_t* kout = to_final ? keys_out : keys_tmp;
        uint32_t* vout = to_final ? vals_out : vals_tmp;
        const int shift = 8 * p;
        k_radix_hist<<<tiles, SORT_THREADS, 0, stream>>>(kin, n, shift, tiles, hist);
        k_radix_scan<<<RADIX, SORT_THREADS, 0, stream>>>(hist, tiles, digit_total);
        if (p == 0)
            k_radix_scatter<true><<<tiles, SORT_THREADS, 0, stream>>>(
                kin, vin, kout, vout, n, shift, tiles, hist, digit_total, err);
        else
            k_radix_scatter<false><<<tiles, SORT_THREADS, 0, stream>>>(
                kin, vin, kout, vout, n, shift, tiles, hist, digit_total, err);
        kin = kout;
        vin = vout;
    }
    return cudaGetLastError();
}

}  // namespace pfs
