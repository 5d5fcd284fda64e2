// pfs_staged.cu — the staged shape of the FP32 density pass.
//
// Same sums as every other shape (calculateDensities.comp:96-153): the 27
// sample-point cells of x* (z outer, x inner, out-of-box sample points
// skipped, duplicate slots walked twice, self included), each cell's table
// range in slot order; and the same neighbour lists for the force pass
// (applyPressureAndViscosityForce.comp:121-183: the 27 cells around the cell
// of x*, self and d < 1e-7 left out), which the list shape's force pass
// evaluates (pfs_neighbors.cu).
//
// Work is organised by spatial block instead of by particle:
//   - the spatial order buckets particles by (block of 2^sbx x 2^sby x 2^sbz
//     cells of x*, cell in the block), so a block's particles are one
//     contiguous, cell-ordered segment of `order`; k_bucket_alloc_staged
//     places the segments and lists the non-empty blocks;
//   - one thread block takes one spatial block at a time from that list (a
//     persistent grid and a work counter), looks up the table ranges of the
//     block's cells and the layer of cells around them (the "union": every
//     cell any of its particles visits), and copies those ranges'
//     candidates (x* and slot) into shared memory with coalesced loads, cell
//     by cell in union order;
//   - each thread then walks its particle's 27 cells as nine rows of three
//     cells, which are consecutive in the staged array, in one loop whose
//     trip count is the warp's longest walk, so the warp stays converged.
//     Lanes hold particles in cell order, so a warp's lanes mostly share
//     cells, walk lengths and (broadcast) shared-memory addresses.
//
// Exactness: the walk visits each particle's candidates in the reference's
// order, so with FAST = false every term and sum is the reference's IEEE
// operation sequence and the results equal the oracle bit for bit.  With
// FAST = true (the PFS_FP32_FAST form) the same candidates are summed with
// fused multiply-adds and hardware reciprocal square roots; keys, sort,
// table, predict, force and integrate stay exact.
//
// Fallbacks, with the same results: a particle whose sample-point cells are
// not its cell's neighbours (cell-boundary rounding, x* outside the box), or
// whose cell lies outside its bucket's block, or a block whose union holds
// more than ST_CAP candidates, is walked from global memory by its own
// thread (exact arithmetic, either form) and goes to the force pass's scan
// queue, as does a particle with more neighbours than a list holds.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_nbr.cuh"
#include "pfs_staged.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int ST_THREADS = ST_THREADS_HOST;
constexpr int ST_WARPS = ST_THREADS / 32;
constexpr int ST_DCAP = 16;  // deferred density terms per lane

// ---- spatial order: place each block's cells contiguously -----------------

// One warp per staged block: the block's fine-bucket counts (one per cell,
// V = 2^(sbx+sby+sbz) of them) are summed, the block reserves one segment of
// `order`, its cells get consecutive offsets inside it (cell order), and a
// non-empty block is appended to the work list.
__global__ void __launch_bounds__(256)
k_bucket_alloc_staged(uint32_t nblocks, uint32_t cells_per_block, const uint32_t* __restrict__ fcount,
                      uint32_t* __restrict__ foffset, uint32_t* __restrict__ bseg,
                      uint32_t* __restrict__ btot, uint32_t* __restrict__ blist,
                      uint32_t* __restrict__ counters, uint32_t* __restrict__ bcounter) {
    const uint32_t blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (blk >= nblocks) return;
    const uint32_t V = cells_per_block;
    const uint32_t* fc = fcount + (size_t)blk * V;
    uint32_t sum = 0;
    for (uint32_t c = lane; c < V; c += 32) sum += fc[c];
    sum = __reduce_add_sync(0xffffffffu, sum);
    if (sum == 0) return;
    uint32_t seg = 0;
    if (lane == 0) {
        seg = atomicAdd(bcounter, sum);
        const uint32_t k = atomicAdd(counters + ST_CTR_BLOCKS, 1u);
        blist[k] = blk;
        bseg[blk] = seg;
        btot[blk] = sum;
    }
    uint32_t run = __shfl_sync(0xffffffffu, seg, 0);
    for (uint32_t base = 0; base < V; base += 32) {
        const uint32_t c = base + lane;
        const uint32_t v = c < V ? fc[c] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (c < V) foffset[(size_t)blk * V + c] = run + incl - v;
        run += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// ---- shared pieces of both passes ------------------------------------------

struct Union {
    int ox, oy, oz;  // first cell of the block
    int ux, uy, uz;  // union extents (block + one cell on each side)
    int U;           // union cells
};

__device__ __forceinline__ Union block_union(const DevParams& P, uint32_t blk) {
    Union u;
    const uint32_t bx = blk % P.nsx, r = blk / P.nsx, by = r % P.nsy, bz = r / P.nsy;
    u.ox = (int)(bx << P.sbx);
    u.oy = (int)(by << P.sby);
    u.oz = (int)(bz << P.sbz);
    u.ux = (1 << P.sbx) + 2;
    u.uy = (1 << P.sby) + 2;
    u.uz = (1 << P.sbz) + 2;
    u.U = u.ux * u.uy * u.uz;
    return u;
}

// Exclusive scan over the thread block (ST_THREADS threads).
__device__ __forceinline__ uint32_t st_exclusive_scan(uint32_t v, uint32_t* s_tmp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_tmp[warp] = incl;
    __syncthreads();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < ST_WARPS; w++) {
        const uint32_t x = s_tmp[w];
        before += w < warp ? x : 0u;
        all += x;
    }
    __syncthreads();
    *total = all;
    return before + incl - v;
}

// Table ranges of the union cells: s_start[u] and the prefix offsets
// s_off[0..U] of their lengths in union order (x fastest).  Returns the
// number of candidates; called by every thread of the block.
__device__ __forceinline__ uint32_t stage_ranges(const DevParams& P, const Union& un,
                                                 const int2* __restrict__ table, int32_t* s_off,
                                                 int32_t* s_start, uint32_t* s_tmp,
                                                 uint32_t* __restrict__ err) {
    constexpr int PER = ST_UMAX / ST_THREADS;
    const int u0 = threadIdx.x * PER;
    int32_t len[PER];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const int u = u0 + k;
        len[k] = 0;
        if (u < un.U) {
            const int lx = u % un.ux, ly = (u / un.ux) % un.uy, lz = u / (un.ux * un.uy);
            // cell coordinates as the force pass forms them: one below the
            // grid wraps to 2^32 - 1 (applyPressureAndViscosityForce.comp:136-137)
            const uint32_t cx = (uint32_t)(un.ox - 1 + lx), cy = (uint32_t)(un.oy - 1 + ly),
                           cz = (uint32_t)(un.oz - 1 + lz);
            const int2 se = __ldg(table + slot_of(P, cell_hash(cx, cy, cz)));
            int32_t st = 0;
            if (se.x != -1) {
                if (table_range_ok(se, P.n)) {
                    len[k] = se.y - se.x;
                    st = se.x;
                } else {
                    atomicOr(err, ERR_TABLE_RANGE);
                }
            }
            s_start[u] = st;
            sum += (uint32_t)len[k];
        }
    }
    uint32_t total;
    uint32_t run = st_exclusive_scan(sum, s_tmp, &total);
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const int u = u0 + k;
        if (u < un.U) {
            s_off[u] = (int32_t)run;
            run += (uint32_t)len[k];
        }
    }
    if (threadIdx.x == 0) s_off[un.U] = (int32_t)total;
    __syncthreads();
    return total;
}

// Union cell of staged candidate c: the last u with s_off[u] <= c.
__device__ __forceinline__ int union_cell_of(const int32_t* s_off, int U, int32_t c) {
    int lo = 0, hi = U;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_off[mid] <= c) lo = mid; else hi = mid;
    }
    return lo;
}

// Per-particle set-up shared by both passes: the sample points' validity and
// cells (calculateDensities.comp:117-118, samplePointToKey), whether they are
// exactly the 27 cells around the cell of x* (then the force pass visits the
// same cells), and the particle's cell inside the block.
struct Walker {
    bool vx[3], vy[3], vz[3];
    int32_t cx[3], cy[3], cz[3];
    bool listing;
    int lx, ly, lz;  // cell of x* relative to the block's first cell
    bool inside;     // that cell lies in the block
};

__device__ __forceinline__ void walker_setup(const DevParams& P, const float4 sp, const Union& un,
                                             bool live, Walker& w) {
    const float h = P.h;
    const float off[3] = {PFS_MUL(h, -1.0f), PFS_MUL(h, 0.0f), h};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float sx = PFS_ADD(sp.x, off[a]), sy = PFS_ADD(sp.y, off[a]), sz = PFS_ADD(sp.z, off[a]);
        w.vx[a] = !(sx < P.minx) && !(sx > P.maxx);
        w.vy[a] = !(sy < P.miny) && !(sy > P.maxy);
        w.vz[a] = !(sz < P.minz) && !(sz > P.maxz);
        w.cx[a] = cell_coord(sx, P.minx, h);
        w.cy[a] = cell_coord(sy, P.miny, h);
        w.cz[a] = cell_coord(sz, P.minz, h);
    }
    w.listing = live && w.vx[1] && w.vy[1] && w.vz[1] && (!w.vx[0] || w.cx[0] == w.cx[1] - 1) &&
                (!w.vx[2] || w.cx[2] == w.cx[1] + 1) && (!w.vy[0] || w.cy[0] == w.cy[1] - 1) &&
                (!w.vy[2] || w.cy[2] == w.cy[1] + 1) && (!w.vz[0] || w.cz[0] == w.cz[1] - 1) &&
                (!w.vz[2] || w.cz[2] == w.cz[1] + 1);
    w.lx = w.cx[1] - un.ox;
    w.ly = w.cy[1] - un.oy;
    w.lz = w.cz[1] - un.oz;
    w.inside = w.lx >= 0 && w.ly >= 0 && w.lz >= 0 && w.lx < un.ux - 2 && w.ly < un.uy - 2 &&
               w.lz < un.uz - 2;
}

// First union cell of row (dy, dz) of the particle's 27 cells: the cell
// (lx - 1, ly + dy - 1, lz + dz - 1) of the block sits at union index
// lx + ux * ((ly + dy) + uy * (lz + dz)).
__device__ __forceinline__ int row_cell(const Union& un, const Walker& w, int dy, int dz) {
    return w.lx + un.ux * ((w.ly + dy) + un.uy * (w.lz + dz));
}

// Distance squared, as the reference's distance() / dot(d, d) forms it
// (exact), or with fused multiply-adds (fast).
template <bool FAST>
__device__ __forceinline__ float st_dist2(const float4 q, const float4 sp) {
    if constexpr (FAST) {
        const float d0 = __fsub_rn(q.x, sp.x), d1 = __fsub_rn(q.y, sp.y), d2 = __fsub_rn(q.z, sp.z);
        return __fmaf_rn(d0, d0, __fmaf_rn(d1, d1, __fmul_rn(d2, d2)));
    } else {
        float d0, d1, d2;
        return dist2(q, sp, d0, d1, d2);
    }
}

template <bool FAST>
__device__ __forceinline__ void st_density_term(float dd, float h, float m, float& total, float& total_near) {
    if constexpr (FAST) {
        const float d = dd > 0.0f ? __fmul_rn(dd, rsqrtf(dd)) : 0.0f;
        const float a = __fsub_rn(h, d);
        const float a2 = __fmul_rn(a, a);
        total = __fadd_rn(total, a2);
        total_near = __fmaf_rn(a2, a, total_near);
    } else {
        density_term(dd, h, m, total, total_near);
    }
}

template <bool FAST>
__device__ __forceinline__ float2 st_density_finish(const DevParams& P, float total, float total_near) {
    if constexpr (FAST) {
        // the fast sums leave out the particle mass: scale once here
        return density_finish(P, __fmul_rn(total, P.m), __fmul_rn(total_near, P.m));
    } else {
        return density_finish(P, total, total_near);
    }
}

// ---- density pass -----------------------------------------------------------

struct DensSmem {
    float4 x[ST_CAP];    // staged x*
    int32_t j[ST_CAP];   // its slot (the force pass's list entry)
    int32_t off[ST_UMAX + 1];
    int32_t start[ST_UMAX];
    float dd[ST_DCAP][ST_THREADS];
    uint32_t tmp[ST_WARPS];
    uint32_t item;
};

// One particle's walk over its nine rows in the staged array: the row, the
// candidate position, the row's end and its density window [ds, de) (the
// cells whose sample point is in the box).
struct Cursor {
    int row;
    int32_t c, end, ds, de;
};

__device__ __forceinline__ void cursor_row(const Union& un, const Walker& w, const int32_t* s_off,
                                           int row, Cursor& k) {
    const int dy = row % 3, dz = row / 3;
    const int u = row_cell(un, w, dy, dz);
    const int32_t c0 = s_off[u], c1 = s_off[u + 1], c2 = s_off[u + 2], c3 = s_off[u + 3];
    const bool rowv = pickb(dy, w.vy[0], w.vy[1], w.vy[2]) && pickb(dz, w.vz[0], w.vz[1], w.vz[2]);
    k.row = row;
    k.c = c0;
    k.end = c3;
    k.ds = rowv ? (w.vx[0] ? c0 : c1) : c3;
    k.de = rowv ? (w.vx[2] ? c3 : c2) : c3;
}

// Candidates of all nine rows of a particle.
__device__ __forceinline__ int32_t walk_length(const Union& un, const Walker& w, const int32_t* s_off) {
    int32_t t = 0;
#pragma unroll
    for (int row = 0; row < 9; row++) {
        const int u = row_cell(un, w, row % 3, row / 3);
        t += s_off[u + 3] - s_off[u];
    }
    return t;
}

// Density pass of the staged shape.  Per thread block and spatial block:
// stage the union's x* (and slots) in shared memory; then the block's
// particles, 128 at a time in cell order, walk their nine rows in one loop
// whose trip count is the warp's longest walk (lanes with shorter walks idle
// through the tail), so the warp stays converged.  In-range terms of cells
// with an in-box sample point are deferred in order and evaluated in order;
// the force pass's neighbours (all 27 cells, not itself, d >= 1e-7, in walk
// order, i.e. the force pass's own order) go to the neighbour list as
// slots.  Particles that cannot
// walk the stage (see the file comment) take the global 27-cell walk and
// the force pass's scan queue, as in the list shape.
template <bool FAST>
__global__ void __launch_bounds__(ST_THREADS)
k_density_staged(DevParams P, const float4* __restrict__ xp,
                 const int2* __restrict__ table, const uint32_t* __restrict__ order,
                 const uint32_t* __restrict__ bseg, const uint32_t* __restrict__ btot,
                 const uint32_t* __restrict__ blist, uint32_t* __restrict__ counters,
                 float2* __restrict__ rr, int32_t* __restrict__ nlist,
                 int32_t* __restrict__ ncount, uint32_t* __restrict__ scanq,
                 uint32_t* __restrict__ scanq_n, uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char st_smem[];
    DensSmem& S = *reinterpret_cast<DensSmem*>(st_smem);
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t full = 0xffffffffu;
    const uint32_t n = P.n;
    const uint32_t items = counters[ST_CTR_BLOCKS];
    const float h = P.h, m = P.m, skip = P.skip_d2, min_d2 = P.min_d2;
    const int32_t cap = (int32_t)P.list_cap;
    for (;;) {
        if (tid == 0) S.item = atomicAdd(counters + ST_CTR_DENSITY, 1u);
        __syncthreads();
        const uint32_t item = S.item;
        if (item >= items) break;
        const uint32_t blk = blist[item];
        const uint32_t seg = bseg[blk], cnt = btot[blk];
        const Union un = block_union(P, blk);
        const uint32_t total = stage_ranges(P, un, table, S.off, S.start, S.tmp, err);
        const bool staged = total <= (uint32_t)ST_CAP;
        if (staged) {
            for (int32_t c = tid; c < (int32_t)total; c += ST_THREADS) {
                const int u = union_cell_of(S.off, un.U, c);
                const int32_t j = S.start[u] + (c - S.off[u]);
                S.x[c] = __ldg(xp + j);
                S.j[c] = j;
            }
        }
        __syncthreads();
        for (uint32_t pb = 0; pb < cnt; pb += ST_THREADS) {
            const uint32_t r = pb + tid;
            bool live = r < cnt;
            const uint32_t t = seg + r;
            uint32_t i = 0;
            if (live) {
                i = order[t];
                if (i >= n || t >= n) {
                    atomicOr(err, ERR_PERM_RANGE);
                    live = false;
                }
            }
            const float4 sp = live ? xp[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            Walker w;
            walker_setup(P, sp, un, live, w);
            const bool walk = live && staged && w.listing && w.inside;
            // the warp's loop: every lane takes part, lanes without a staged
            // walk with length 0
            const int32_t len = walk ? walk_length(un, w, S.off) : 0;
            const int32_t trips = __reduce_max_sync(full, len);
            float tot = 0.0f, tot_n = 0.0f;
            int cd = 0;
            int32_t nl = 0;
            if (trips > 0) {
                Cursor k{0, 0, 0, 0, 0};
                if (walk) {
                    cursor_row(un, w, S.off, 0, k);
                    while (k.c == k.end && k.row < 8) cursor_row(un, w, S.off, k.row + 1, k);
                }
                for (int32_t q = 0; q < trips; q++) {
                    const bool valid = q < len;
                    const int32_t c = valid ? k.c : 0;
                    const float dd = st_dist2<FAST>(S.x[c], sp);
                    const bool in = valid && in_reach(dd, skip);
                    const bool dens = in && c >= k.ds && c < k.de;
                    const bool lst = in && !(dd < min_d2);
                    S.dd[cd][tid] = dd;
                    cd += dens ? 1 : 0;
                    if (lst && nl < cap) __stcs(nlist + (size_t)nl * n + t, S.j[c]);
                    nl += lst ? 1 : 0;
                    if (valid) {
                        k.c++;
                        while (k.c == k.end && k.row < 8) cursor_row(un, w, S.off, k.row + 1, k);
                    }
                    // all lanes evaluate their deferred terms once one buffer is full
                    if (__any_sync(full, cd == ST_DCAP)) {
                        for (int e = 0; e < ST_DCAP; e++)
                            if (e < cd) st_density_term<FAST>(S.dd[e][tid], h, m, tot, tot_n);
                        cd = 0;
                    }
                }
            }
            if (walk) {
                for (int e = 0; e < cd; e++) st_density_term<FAST>(S.dd[e][tid], h, m, tot, tot_n);
                rr[i] = st_density_finish<FAST>(P, tot, tot_n);
            } else if (live) {
                rr[i] = density_scan_one(P, sp, xp, table, err);
            }
            // the force pass: a list, or its scan queue
            const bool scan = live && !(walk && nl <= cap);
            if (live) ncount[t] = scan ? -1 : nl;
            const uint32_t want = __ballot_sync(full, scan);
            if (want) {
                const int leader = __ffs(want) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(scanq_n, (uint32_t)__popc(want));
                base = __shfl_sync(full, base, leader);
                if (scan) scanq[base + __popc(want & ((1u << lane) - 1u))] = t;
            }
        }
        __syncthreads();  // the next block restages
    }
}

// Resident thread blocks of a staged kernel on the current device (the grid
// of the persistent loop).
template <class K>
unsigned staged_grid(K kernel, size_t smem) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, ST_THREADS, smem);
    return (unsigned)std::max(1, per_sm) * (unsigned)sms;
}

template <class K>
cudaError_t allow_smem(K kernel, size_t smem) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace

cudaError_t launch_bucket_alloc_staged(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    const uint32_t nblocks = P.nsx * P.nsy * P.nsz;
    const uint32_t V = 1u << (P.sbx + P.sby + P.sbz);
    const unsigned grid = (unsigned)(((size_t)nblocks * 32 + 255) / 256);
    k_bucket_alloc_staged<<<grid, 256, 0, s>>>(nblocks, V, b.bcount, b.boffset, b.bseg, b.btot, b.blist,
                                               b.st_counters, b.bcounter);
    return cudaGetLastError();
}

cudaError_t launch_density_staged(const DevParams& P, const StepBuffers& b, bool fast, cudaStream_t s) {
    const size_t smem = sizeof(DensSmem);
    cudaError_t e;
    if (fast) {
        auto k = k_density_staged<true>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<staged_grid(k, smem), ST_THREADS, smem, s>>>(P, b.xp, b.table, b.order, b.bseg, b.btot,
                                                         b.blist, b.st_counters, b.rr, b.nlist,
                                                         b.ncount, b.scanq, b.scanq_n, b.err);
    } else {
        auto k = k_density_staged<false>;
        if ((e = allow_smem(k, smem)) != cudaSuccess) return e;
        k<<<staged_grid(k, smem), ST_THREADS, smem, s>>>(P, b.xp, b.table, b.order, b.bseg, b.btot,
                                                         b.blist, b.st_counters, b.rr, b.nlist,
                                                         b.ncount, b.scanq, b.scanq_n, b.err);
    }
    return cudaGetLastError();
}

}  // namespace pfs

namespace pfs {

uint64_t staged_buckets(const DevParams& P) {
    return (uint64_t)P.nsx * P.nsy * P.nsz << (P.sbx + P.sby + P.sbz);
}

// Among block shapes whose union fits ST_UMAX cells, pick the one that fills
// the thread block's lanes best at this density (expected particles per
// block against the lanes its chunks of ST_THREADS take), with room for the
// expected union (its cells' table ranges, hash collisions included) in
// ST_CAP with a quarter to spare; ties go to the shape that stages the
// fewest union cells per block cell.
bool configure_staged(DevParams* P, double per_cell, double slots, uint64_t bucket_cap) {
    if (!(per_cell > 0.0)) per_cell = 2.0;
    // a union cell's table range also holds the particles of other cells
    // hashed to the same slot: about n / per_cell occupied cells share the
    // slots
    const double per_range = per_cell * (1.0 + (double)P->n / (per_cell * std::max(slots, 1.0)));
    double best = -1.0, best_ratio = 0.0;
    int bx = 1, by = 1, bz = 1;
    for (int sx = 0; sx <= 3; sx++)
        for (int sy = 0; sy <= 3; sy++)
            for (int sz = 0; sz <= 3; sz++) {
                const int ex = 1 << sx, ey = 1 << sy, ez = 1 << sz;
                const int U = (ex + 2) * (ey + 2) * (ez + 2);
                if (U > ST_UMAX) continue;
                if ((double)U * per_range * 1.25 > (double)ST_CAP) continue;
                const double parts = (double)(ex * ey * ez) * per_cell;
                const double lanes = ST_THREADS_HOST * std::ceil(std::max(parts, 1.0) / ST_THREADS_HOST);
                const double fill = parts / lanes;
                const double ratio = (double)U / (double)(ex * ey * ez);
                if (fill > best + 1e-9 || (fill > best - 1e-9 && ratio < best_ratio)) {
                    best = fill;
                    best_ratio = ratio;
                    bx = sx;
                    by = sy;
                    bz = sz;
                }
            }
    if (best < 0.0) return false;  // even single cells overflow the stage
    P->sbx = bx;
    P->sby = by;
    P->sbz = bz;
    P->nsx = ((P->ngx - 1) >> bx) + 1;
    P->nsy = ((P->ngy - 1) >> by) + 1;
    P->nsz = ((P->ngz - 1) >> bz) + 1;
    if (staged_buckets(*P) > bucket_cap) return false;
    return true;
}

// n over the cells of the initial state's bounding box (inside the world
// box): particles per cell where the particles are.
double occupied_cell_density(const float* pos4, uint32_t n, const float box_min[3],
                             const float box_max[3], float h) {
    if (!pos4 || n == 0) return 0.0;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            const double v = pos4[4 * (size_t)i + a];
            if (v >= box_min[a] && v <= box_max[a]) {
                lo[a] = std::min(lo[a], v);
                hi[a] = std::max(hi[a], v);
            }
        }
    double cells = 1.0;
    for (int a = 0; a < 3; a++) {
        if (!(hi[a] >= lo[a])) return 0.0;
        cells *= std::max(1.0, std::ceil((hi[a] - lo[a]) / (double)h));
    }
    return (double)n / cells;
}

}  // namespace pfs
