// pfs_step.cuh — launchers of the SPH substep kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"

namespace pfs {

// Device buffers of one table (one world, or one batch of scenes).
// Particle arrays are n float4 (xyz + w); the cell table is n int2
// (start, end) with start = -1 for an empty slot.
struct StepBuffers {
    float4* x;          // state positions (order of the previous sort)
    float4* v;          // state velocities; also the force pass output
    float4* xs;         // positions gathered into the current sort order
    float4* vs;         // velocities gathered into the current sort order
    float4* xp;         // predicted positions x*
    float4* vp;         // predicted velocities v*
    float2* rr;         // (density, near density)
    uint32_t* keys;     // keys of the state positions (next sort's input)
    uint32_t* skeys;    // sorted keys
    uint32_t* perm;     // sort permutation
    uint32_t* keys_tmp; // sort scratch
    uint32_t* vals_tmp;
    uint32_t* sort_scratch;  // sort_scratch_words(n, sort_key_bits(n))
    int2* table;        // (start, end) per key slot
    uint32_t* ids;      // optional creation index per slot
    uint32_t* ids_s;    // optional, gathered ids
    float4* color;      // optional speed colours
    uint32_t* err;      // device error word
    // spatial processing order of the neighbour passes (a permutation of the
    // sorted slots grouping particles by block of x*; any order gives the
    // same results, this one gives cache reuse)
    uint32_t* order;    // n
    uint32_t* bucket;   // n: block of each slot
    uint32_t* brank;    // n: rank of the slot inside its block
    uint32_t* bcount;   // blocks: particles per block (zero between substeps)
    uint32_t* boffset;  // blocks: start of each block's segment of order
    uint32_t* bcounter; // 1: segment allocator
    // neighbour lists the density pass leaves for the force pass, indexed by
    // position in `order`: nlist[k * n + t] is the k-th in-range neighbour
    // (force enumeration order, self excluded) of particle order[t];
    // ncount[t] < 0 means the force pass must scan for itself
    int32_t* nlist;     // list_cap * n (DevParams::list_cap)
    int32_t* ncount;    // n
    uint32_t* scanq;    // n: positions t whose force pass must scan
    uint32_t* scanq_n;  // 1: entries in scanq
    // batch of scenes: per-slot scene parameters (null for one world) and
    // the spatial-order blocks of all scenes together
    SceneRef sr;
    uint32_t nblocks;
    // FP16-cell form: 16-byte neighbour records the reorder writes (null for
    // the FP32 form)
    uint4* rec;
    // some particle uses the grid search (pfs_geo.cuh): the block counters
    // then stay set through the neighbour passes and the grid-search kernels
    // run after the per-thread ones
    uint32_t geo_any;
    // kernel shape of the FP32 neighbour passes (NBR_*; all give the same bits)
    int32_t variant;
    // staged shape (pfs_staged.cu): per block of the staged order its
    // segment of `order` and particle count, the non-empty blocks of this
    // substep, and the density pass's counters (ST_CTR_*)
    uint32_t* bseg;
    uint32_t* btot;
    uint32_t* blist;
    uint32_t* st_counters;
    // arithmetic of the staged passes: 0 the reference's IEEE sequence
    // (bit-exact), 1 fused multiply-adds and hardware reciprocals
    // (PFS_FP32_FAST)
    int32_t fast;
};

// Neighbours a list holds per particle.
// Neighbour-list rows per particle: worlds size them from the density of
// their initial state (at least NLIST_CAP, rounded up to 16), batches use
// NLIST_CAP_MAX so scenes of any density added later keep their lists.
constexpr int NLIST_CAP = 48;
constexpr int NLIST_CAP_MAX = 512;
// Length bins of the force pass's per-block ordering (longer lists share the
// last bin; the order only balances the warps' work).
constexpr int LEN_BINS = 64;

#ifdef __CUDACC__
// Position this thread evaluates in a force-pass block that starts at tb:
// the block's positions in ascending list length (a counting sort over
// ncount in shared memory; queued and past-the-end positions first), so the
// lanes of a warp walk lists of similar length while the block keeps its
// spatial neighbourhood.  Called by every thread of a block of at most 256
// threads.
__device__ __forceinline__ uint32_t list_length_order(uint32_t tb, uint32_t n, const int32_t* __restrict__ ncount) {
    __shared__ uint32_t s_cnt[LEN_BINS], s_pos[LEN_BINS];
    __shared__ uint8_t s_tid[256];
    const uint32_t t_own = tb + threadIdx.x;
    const int32_t c_own = t_own < n ? ncount[t_own] : -1;
    const int bin = c_own < 0 ? 0 : min(c_own, LEN_BINS - 2) + 1;
    for (int k = threadIdx.x; k < LEN_BINS; k += blockDim.x) s_cnt[k] = 0u;
    __syncthreads();
    atomicAdd(&s_cnt[bin], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int k = 0; k < LEN_BINS; k++) {
            s_pos[k] = run;
            run += s_cnt[k];
        }
    }
    __syncthreads();
    s_tid[atomicAdd(&s_pos[bin], 1u)] = (uint8_t)threadIdx.x;
    __syncthreads();
    return tb + s_tid[threadIdx.x];
}
#endif

// Keys of the state positions (updateCellEntries.comp:69-80).
cudaError_t launch_keys(const DevParams& P, const StepBuffers& b, cudaStream_t s);
// Table slots all empty.
cudaError_t launch_table_clear(const DevParams& P, const StepBuffers& b, cudaStream_t s);
// Sort keys -> (skeys, perm).
cudaError_t launch_sort(const DevParams& P, const StepBuffers& b, cudaStream_t s);
// Gather by perm + predict + table set.
cudaError_t launch_reorder(const DevParams& P, const StepBuffers& b, cudaStream_t s);
cudaError_t launch_density(const DevParams& P, const StepBuffers& b, cudaStream_t s);
cudaError_t launch_force(const DevParams& P, const StepBuffers& b, cudaStream_t s);
// Integrate + next keys + table slot reset (+ colours, ids).
cudaError_t launch_integrate(const DevParams& P, const StepBuffers& b, cudaStream_t s);

// Density map of the state x (in the order of the last sort, skeys) over an
// image of image[] voxels of cell_size, with the shader's bounds rule at
// bound[], into out on the device (the reference's updateDensityMap.comp).
cudaError_t launch_density_map(const DevParams& P, const StepBuffers& b, float cell_size,
                               const int32_t image[3], const int32_t bound[3], float* out,
                               cudaStream_t s);

// Volumetric rendering (pfs_render.cu): light volume of ldims voxels of
// light_step marched toward sun over the density map dmap (ddims), and the
// view-ray march of a width x height RGBA image (cam = position, forward,
// right, up; half_h = tan(FOV / 2), half_w = half_h * width / height; ext =
// normalised extinction coefficients).
cudaError_t launch_light_volume(const DevParams& P, const float* dmap, const int32_t ddims[3],
                                float light_step, const float sun[3], const int32_t ldims[3],
                                float* out, cudaStream_t s);
cudaError_t launch_volumetric(const DevParams& P, const float* dmap, const int32_t ddims[3],
                              const float* lvol, const int32_t ldims[3], const float cam[12],
                              float half_h, float half_w, float step, const float ext[3],
                              uint32_t width, uint32_t height, float* rgba, cudaStream_t s);
cudaError_t launch_splats(uint32_t n, const float4* x, const float4* color, const float mvp[16],
                          const float right[3], const float up[3], float radius, uint32_t width,
                          uint32_t height, unsigned long long* keys, float* rgba, float* depth,
                          uint32_t* err, cudaStream_t s);
cudaError_t launch_fxaa(const float* in, uint32_t width, uint32_t height, float* out, cudaStream_t s);
cudaError_t launch_refractive(const DevParams& P, const float* dmap, const int32_t ddims[3], const float cam[12],
                              float half_h, float half_w, float step, float light_step, const float ext[3],
                              int32_t num_refractions, float threshold, float ior, uint32_t width,
                              uint32_t height, float* rgba, cudaStream_t s);

// Neighbour-pass kernel variants (the values of PFS_SHAPE_* in pfs.h).
enum { NBR_SIMPLE = 0, NBR_COMPACT = 1, NBR_LIST = 2, NBR_FLAT = 3, NBR_STAGED = 4 };
// Default shape of new worlds and batches (PFS_NBR_VARIANT=simple|slab|list|flat).
int nbr_variant();

// Launches one substep issues (sort included; geo: grid search in use).
int substep_launches(uint32_t n, bool geo);

}  // namespace pfs
