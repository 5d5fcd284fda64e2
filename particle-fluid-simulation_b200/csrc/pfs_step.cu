// pfs_step.cu — FP32 SPH substep kernels (plain form).
//
// Data flow of one substep (reference dispatch order commands.c:193-402):
//   keys (from the integrate of the previous substep, or k_keys)
//   -> radix sort -> (skeys, perm)
//   -> k_reorder:   xs, vs = gather(x, v, perm); xp, vp = predict(xs, vs);
//                   table[skey] = (run start, run end)
//   -> density:     rr = (density, near density) from xp and the table
//   -> force:       v  = vs + F / density * dt        (Jacobi: reads vs)
//                   (both neighbour passes live in pfs_neighbors.cu)
//   -> k_integrate: x, v = integrate(xs, v); keys = key(x); clear the table
//                   slots this substep set
// Predict is per particle, so running it on the gathered state equals the
// reference's predict-then-scatter (predictPositions.comp, scatterPass.comp).
// The state stays in sort order between substeps, as the reference's
// ping-pong buffers do.
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_record.cuh"
#include "pfs_sort.cuh"
#include "pfs_staged.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int ELEM_THREADS = 256;

template <bool BATCH>
__global__ void __launch_bounds__(ELEM_THREADS)
k_keys(DevParams P0, SceneRef sr, const float4* __restrict__ x, uint32_t* __restrict__ keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P0.n) return;
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 p = x[i];
    keys[i] = point_key(P, p.x, p.y, p.z);
}

__global__ void __launch_bounds__(ELEM_THREADS)
k_table_clear(uint32_t n, int2* __restrict__ table) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) table[i] = make_int2(-1, -1);
}

// scatterPass.comp:50-65 (gather by permutation) + predictPositions.comp:69-117
// + updateStartIndices.comp:40-64 (run heads set start, run tails set end).
template <bool BATCH>
__global__ void __launch_bounds__(ELEM_THREADS)
k_reorder(DevParams P0, SceneRef sr, const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ perm,
          const float4* __restrict__ x, const float4* __restrict__ v,
          const uint32_t* __restrict__ ids, float4* __restrict__ xs, float4* __restrict__ vs,
          float4* __restrict__ xp, float4* __restrict__ vp, uint32_t* __restrict__ ids_s,
          int2* __restrict__ table, uint32_t* __restrict__ bucket, uint32_t* __restrict__ brank,
          uint32_t* __restrict__ bcount, uint32_t* __restrict__ bcounter,
          uint32_t* __restrict__ scanq_n, uint4* __restrict__ rec, uint32_t* __restrict__ st_counters,
          uint32_t* __restrict__ err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = P0.n;
    if (s == 0) {
        *bcounter = 0u;
        scanq_n[0] = 0u;  // scan queue
        scanq_n[1] = 0u;  // grid-search queue
        scanq_n[2] = 0u;  // grid-search density pass: work counter
        scanq_n[3] = 0u;  // grid-search force pass: work counter
        if (st_counters) {  // staged passes: block list and work counters
            st_counters[ST_CTR_BLOCKS] = 0u;
            st_counters[ST_CTR_DENSITY] = 0u;
        }
    }
    if (s >= n) return;
    const DevParams P = params_of<BATCH>(P0, sr, s);
    const uint32_t p = perm[s];
    const uint32_t k = skeys[s];
    if (p >= n || k >= n) {
        atomicOr(err, p >= n ? ERR_PERM_RANGE : ERR_KEY_RANGE);
        bucket[s] = 0xffffffffu;
        return;
    }
    const float4 xo = x[p];
    const float4 vo = v[p];
    xs[s] = xo;
    vs[s] = vo;
    float3 pos = make_float3(xo.x, xo.y, xo.z);
    float3 vel = make_float3(vo.x, vo.y, vo.z);
    euler_walls(P, P.margin_p, pos, vel);
    xp[s] = make_float4(pos.x, pos.y, pos.z, 1.0f);
    vp[s] = make_float4(vel.x, vel.y, vel.z, 1.0f);
    if (rec) rec[s] = make_record(P, pos, vo);  // FP16-cell form
    // block of x* for the neighbour passes' processing order (any order gives
    // the same results; this one keeps a warp's neighbours in cache)
    const uint32_t blk = spatial_bucket(P, pos.x, pos.y, pos.z);
    bucket[s] = blk;
    brank[s] = atomicAdd(bcount + blk, 1u);
    if (ids) ids_s[s] = ids[p];
    const bool head = (s == 0) || (skeys[s - 1] != k);
    const bool tail = (s == n - 1) || (skeys[s + 1] != k);
    if (head) table[k].x = (int32_t)s;
    if (tail) table[k].y = (int32_t)(s + 1);
}

// Spatial processing order, step 2: each block reserves its segment of
// `order`.  One thread per block id: a thread block scans the counts of 256
// consecutive block ids and reserves one contiguous range for them, so
// segments land in about block-id order (row-major in space) and the
// neighbour passes, which take positions in order, sweep space coherently:
// a neighbourhood's data is reused from L2 while it is hot.
__global__ void __launch_bounds__(ELEM_THREADS)
k_bucket_alloc(uint32_t nblocks, const uint32_t* __restrict__ bcount, uint32_t* __restrict__ boffset,
               uint32_t* __restrict__ bcounter) {
    __shared__ uint32_t s_warp[ELEM_THREADS / 32];
    __shared__ uint32_t s_base;
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t c = b < nblocks ? bcount[b] : 0u;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < ELEM_THREADS / 32; w++) {
            const uint32_t t = s_warp[w];
            s_warp[w] = run;
            run += t;
        }
        s_base = run ? atomicAdd(bcounter, run) : 0u;
    }
    __syncthreads();
    if (c) boffset[b] = s_base + s_warp[warp] + incl - c;
}

// Step 3: place each slot in its block's segment.  The block counters are
// zeroed here for the next substep, or, when the grid search reads them
// during the neighbour passes (keep), by k_integrate.
__global__ void __launch_bounds__(ELEM_THREADS)
k_bucket_scatter(uint32_t n, uint32_t nblocks, const uint32_t* __restrict__ bucket,
                 const uint32_t* __restrict__ brank, const uint32_t* __restrict__ boffset,
                 uint32_t* __restrict__ bcount, uint32_t keep, uint32_t* __restrict__ order,
                 uint32_t* __restrict__ err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t blk = bucket[s];
    if (blk >= nblocks) {
        atomicOr(err, ERR_SORT_COUNT);
        return;
    }
    const uint32_t r = brank[s];
    const uint32_t dst = boffset[blk] + r;
    if (dst < n)
        order[dst] = s;
    else
        atomicOr(err, ERR_SORT_COUNT);
    if (r == 0u && !keep) bcount[blk] = 0u;
}

// updateVelocities.comp:71-141 + the next substep's updateCellEntries
// (keys of the integrated positions) + reset of the table slots this
// substep's run heads set, so the next table starts empty without a full
// clear.  Slot s is read only by itself here, so x/v update in place.
template <bool BATCH>
__global__ void __launch_bounds__(ELEM_THREADS)
k_integrate(DevParams P0, SceneRef sr, const float4* __restrict__ xs, float4* __restrict__ x,
            float4* __restrict__ v, uint32_t* __restrict__ keys,
            const uint32_t* __restrict__ skeys, int2* __restrict__ table,
            const uint32_t* __restrict__ ids_s, uint32_t* __restrict__ ids,
            float4* __restrict__ color, const uint32_t* __restrict__ bucket,
            const uint32_t* __restrict__ brank, uint32_t* __restrict__ bcount, uint32_t nblocks) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P0.n) return;
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 xo = xs[i];
    const float4 vo = v[i];
    float3 pos = make_float3(xo.x, xo.y, xo.z);
    float3 vel = make_float3(vo.x, vo.y, vo.z);
    euler_walls(P, P.margin_i, pos, vel);
    x[i] = make_float4(pos.x, pos.y, pos.z, 1.0f);
    v[i] = make_float4(vel.x, vel.y, vel.z, 1.0f);
    keys[i] = point_key(P, pos.x, pos.y, pos.z);
    if (color) color[i] = speed_color(vel);
    if (ids) ids[i] = ids_s[i];
    const uint32_t k = skeys[i];
    if (k < P0.n && (i == 0 || skeys[i - 1] != k)) table[k] = make_int2(-1, -1);
    // block counters kept for the grid search start the next substep at zero
    if (bcount) {
        const uint32_t blk = bucket[i];
        if (blk < nblocks && brank[i] == 0u) bcount[blk] = 0u;
    }
}

inline unsigned grid_for(uint32_t n, int threads) { return (n + threads - 1) / threads; }

}  // namespace

cudaError_t launch_keys(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, ELEM_THREADS);
    if (b.sr.scenes)
        k_keys<true><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.x, b.keys);
    else
        k_keys<false><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.x, b.keys);
    return cudaGetLastError();
}

cudaError_t launch_table_clear(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_table_clear<<<grid_for(P.n, ELEM_THREADS), ELEM_THREADS, 0, s>>>(P.n, b.table);
    return cudaGetLastError();
}

cudaError_t launch_sort(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    return sort_pairs(b.keys, P.n, sort_key_bits(P.n), b.skeys, b.perm, b.keys_tmp, b.vals_tmp,
                      b.sort_scratch, b.err, s);
}

cudaError_t launch_reorder(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, ELEM_THREADS);
    if (b.sr.scenes)
        k_reorder<true><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.skeys, b.perm, b.x, b.v, b.ids, b.xs,
                                                   b.vs, b.xp, b.vp, b.ids_s, b.table, b.bucket,
                                                   b.brank, b.bcount, b.bcounter, b.scanq_n, b.rec,
                                                   b.st_counters, b.err);
    else
        k_reorder<false><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.skeys, b.perm, b.x, b.v, b.ids, b.xs,
                                                    b.vs, b.xp, b.vp, b.ids_s, b.table, b.bucket,
                                                    b.brank, b.bcount, b.bcounter, b.scanq_n, b.rec,
                                                    b.st_counters, b.err);
    const uint32_t nb = b.nblocks;
    if (P.staged) {
        // fine buckets: each staged block's cells get one contiguous segment
        const cudaError_t e = launch_bucket_alloc_staged(P, b, s);
        if (e != cudaSuccess) return e;
    } else if (nb > 0) {
        k_bucket_alloc<<<grid_for(nb, ELEM_THREADS), ELEM_THREADS, 0, s>>>(nb, b.bcount, b.boffset,
                                                                            b.bcounter);
    }
    k_bucket_scatter<<<g, ELEM_THREADS, 0, s>>>(P.n, nb, b.bucket, b.brank, b.boffset, b.bcount,
                                                b.geo_any, b.order, b.err);
    return cudaGetLastError();
}

cudaError_t launch_integrate(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, ELEM_THREADS);
    if (b.sr.scenes)
        k_integrate<true><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.xs, b.x, b.v, b.keys, b.skeys,
                                                     b.table, b.ids_s, b.ids, b.color, b.bucket,
                                                     b.brank, b.geo_any ? b.bcount : nullptr,
                                                     b.nblocks);
    else
        k_integrate<false><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.xs, b.x, b.v, b.keys, b.skeys,
                                                      b.table, b.ids_s, b.ids, b.color, b.bucket,
                                                      b.brank, b.geo_any ? b.bcount : nullptr,
                                                      b.nblocks);
    return cudaGetLastError();
}

// sort + reorder/bucket (3) + density + force + integrate (+ the two
// grid-search passes)
int substep_launches(uint32_t n, bool geo) {
    return n == 0 ? 0 : sort_launches(n) + 6 + (geo ? 2 : 0);
}

}  // namespace pfs
