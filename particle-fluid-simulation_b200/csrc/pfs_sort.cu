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
// Tiles of SORT_TILE keys; per pass a digit's output range for tile t starts
// at (keys of smaller digits) + (keys of this digit in tiles before t).  The
// per-tile digit counts come for free: the first pass's from one histogram
// kernel, every later pass's from the scatter before it, which knows where
// each key lands (its destination tile) and adds one to that tile's count of
// the key's next digit.  So a sort of P passes is 1 + 2P launches:
//   k_sort_count0    per tile, the 256-bin histogram of digit 0 (and the
//                    later passes' count rows cleared)
//   k_sort_scan      per digit (one thread block each), the exclusive scan
//                    of its count over the tiles, in place, and its total
//   k_sort_scatter   per tile: stable in-tile rank (warp match + per-warp
//                    counters in the tile's key order), local reorder in
//                    shared memory, coalesced scatter to
//                    base(d) + earlier tiles' count(d) + local rank, and the
//                    next pass's per-tile counts (global atomics on counts)
// Every step is a plain data-parallel kernel: no tile waits on another.  (A
// single sweep per pass with decoupled look-back was measured first: with
// all 256 tiles of a 1M-key pass resident at once, each tile's walk back over
// the earlier tiles' counts was a chain of dependent global reads, 22-24 us
// per pass.)
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
constexpr int SCAN_THREADS = 1024;

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

// Per tile: the histogram of digit 0 into cnt[0][tile][*]; the count rows of
// the later passes (cnt[1..passes-1][tile][*]) are cleared for the scatters'
// atomics.
__global__ void __launch_bounds__(SORT_THREADS)
k_sort_count0(const uint32_t* __restrict__ keys, uint32_t n, int passes, uint32_t tiles,
              uint32_t* __restrict__ cnt) {
    __shared__ uint32_t s_h[SORT_WARPS][RADIX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&s_h[0][0])[i] = 0u;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * SORT_TILE + (uint64_t)warp * (32 * SORT_IPT);
#pragma unroll 4
    for (int it = 0; it < SORT_IPT; it++) {
        const uint64_t idx = base + (uint64_t)it * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? (__ldg(keys + idx) & (RADIX - 1)) : RADIX;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (valid && lane == __ffs(peers) - 1) s_h[warp][d] += __popc(peers);
    }
    __syncthreads();
    const int d = threadIdx.x;  // SORT_THREADS == RADIX
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) c += s_h[w][d];
    cnt[(size_t)blockIdx.x * RADIX + d] = c;
    for (int p = 1; p < passes; p++) cnt[((size_t)p * tiles + blockIdx.x) * RADIX + d] = 0u;
}

// One thread block per digit: cnt[tile][d] over the tiles becomes its
// exclusive prefix (in place), tot[d] the digit's total.  Each thread takes
// a run of consecutive tiles.
__global__ void __launch_bounds__(SCAN_THREADS)
k_sort_scan(uint32_t* __restrict__ cnt, uint32_t tiles, uint32_t* __restrict__ tot) {
    __shared__ uint32_t s_w[SCAN_THREADS / 32];
    const int d = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t per = (tiles + SCAN_THREADS - 1) / SCAN_THREADS;
    const uint32_t t0 = min(threadIdx.x * per, tiles), t1 = min(t0 + per, tiles);
    uint32_t sum = 0;
    for (uint32_t t = t0; t < t1; t++) sum += cnt[(size_t)t * RADIX + d];
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < SCAN_THREADS / 32 ? s_w[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += v;
        }
        if (lane < SCAN_THREADS / 32) s_w[lane] = wi - w;
        if (lane == SCAN_THREADS / 32 - 1) tot[d] = wi;
    }
    __syncthreads();
    uint32_t run = s_w[warp] + incl - sum;
    for (uint32_t t = t0; t < t1; t++) {
        uint32_t* c = cnt + (size_t)t * RADIX + d;
        const uint32_t v = *c;
        *c = run;
        run += v;
    }
}

// One tile of one pass.  pre: the scanned counts of this pass (earlier
// tiles' keys per digit), tot: the digit totals; next: the next pass's count
// rows (null on the last pass), next_shift its digit.
template <bool FIRST>
__global__ void __launch_bounds__(SORT_THREADS, 2)
k_sort_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
               uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t n,
               int shift, const uint32_t* __restrict__ pre, const uint32_t* __restrict__ tot,
               uint32_t* __restrict__ next, int next_shift, uint32_t* __restrict__ err) {
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
    const int d = threadIdx.x;  // SORT_THREADS == RADIX
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; w++) {
        const uint32_t c = s_warp[w][d];
        s_warp[w][d] = cnt;
        cnt += c;
    }
    const uint32_t local = block_exclusive_scan(cnt, s_tot, nullptr);
    const uint32_t dbase = block_exclusive_scan(tot[d], s_tot, nullptr);
    s_local[d] = local;
    s_base[d] = dbase + pre[(size_t)blockIdx.x * RADIX + d];
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
            // the next pass's tile dst / SORT_TILE holds this key
            if (next) atomicAdd(next + (size_t)(dst / SORT_TILE) * RADIX + ((key >> next_shift) & (RADIX - 1)), 1u);
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

// Per pass: the tiles' digit counts (scanned in place) and the digit totals.
size_t sort_scratch_words(uint32_t n, int key_bits) {
    const int passes = (key_bits + 7) / 8;
    const size_t tiles = sort_tiles(n) > 0 ? sort_tiles(n) : 1;
    return (size_t)(passes > 0 ? passes : 1) * (tiles + 1) * RADIX;
}

int sort_launches(uint32_t n) {
    const int p = sort_passes(n);
    return p == 0 ? 1 : 1 + 2 * p;
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
    uint32_t* cnt = scratch;                                  // passes x tiles x RADIX
    uint32_t* tot = scratch + (size_t)passes * tiles * RADIX;  // passes x RADIX
    k_sort_count0<<<tiles, SORT_THREADS, 0, stream>>>(keys_in, n, passes, tiles, cnt);
    const uint32_t* kin = keys_in;
    const uint32_t* vin = nullptr;
    for (int p = 0; p < passes; p++) {
        // the last pass lands in keys_out/vals_out
        const bool to_final = ((passes - 1 - p) % 2) == 0;
        uint32_t* kout = to_final ? keys_out : keys_tmp;
        uint32_t* vout = to_final ? vals_out : vals_tmp;
        uint32_t* cp = cnt + (size_t)p * tiles * RADIX;
        uint32_t* tp = tot + (size_t)p * RADIX;
        uint32_t* next = p + 1 < passes ? cnt + (size_t)(p + 1) * tiles * RADIX : nullptr;
        k_sort_scan<<<RADIX, SCAN_THREADS, 0, stream>>>(cp, tiles, tp);
        if (p == 0)
            k_sort_scatter<true><<<tiles, SORT_THREADS, 0, stream>>>(
                kin, vin, kout, vout, n, 8 * p, cp, tp, next, 8 * (p + 1), err);
        else
            k_sort_scatter<false><<<tiles, SORT_THREADS, 0, stream>>>(
                kin, vin, kout, vout, n, 8 * p, cp, tp, next, 8 * (p + 1), err);
        kin = kout;
        vin = vout;
    }
    return cudaGetLastError();
}

}  // namespace pfs
