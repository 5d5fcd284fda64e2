// pfs_batch.cu — many independent scenes stepped by one set of launches.
//
// Layout: resident scenes are packed back to back; scene s owns particle
// slots and table slots [off_s, off_s + n_s).  Its keys are
// off_s + (hash & (n_s - 1)) (DevParams::key_base / mask), so one stable sort
// of all keys leaves every scene in its own slots, in exactly the order its
// own world's sort gives, and every per-particle kernel reads the scene's
// parameters through the per-slot scene id.  Results per scene are therefore
// bit-identical to a world holding that scene alone; the batch only shares
// the launches (one sort, one launch per stage, one CUDA graph per step).
//
// Scenes are added at the end and removed by moving the later scenes down
// (device copies on the batch's stream), between steps, when the table is
// empty (each substep's integrate clears the slots it set).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pfs.h"
#include "pfs_common.cuh"
#include "pfs_fp16.cuh"
#include "pfs_sort.cuh"
#include "pfs_step.cuh"
#include "pfs_world_impl.cuh"

using namespace pfs;

namespace {

struct Scene {
    int32_t id;
    uint32_t off, n;
    pfs_params params;
    DevParams dp;
};

// Spatial-order buckets a batch reserves per particle and per scene: the
// cap a world uses (derive_params: max(4 n, 4096) blocks), so a scene's
// grid search reads the same blocks (single cells where they fit) as the
// scene's own world.  Coarser blocks made the gather test up to several
// times as many candidates.
constexpr uint32_t kBlocksPerParticle = 4;
constexpr uint32_t kBlocksPerScene = 4096;

__global__ void k_fill_sid(uint32_t n, const uint32_t* __restrict__ offs, uint32_t scenes,
                           uint32_t* __restrict__ sid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // last scene whose offset <= i
    uint32_t lo = 0, hi = scenes;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (offs[mid] <= i) lo = mid; else hi = mid;
    }
    sid[i] = lo;
}

__global__ void k_density_out(uint32_t n, const float2* __restrict__ rr, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = rr[i].x;
}

unsigned grid256(uint32_t n) { return (n + 255) / 256; }

}  // namespace

struct pfs_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t cap_n = 0, cap_s = 0, blocks_cap = 0;
    int32_t precision = PFS_FP32, substeps = 1;
    Arena arena;
    StepBuffers b{};
    Fp16Buffers h16{};
    DevParams* d_scenes = nullptr;
    uint32_t* d_sid = nullptr;
    uint32_t* d_offs = nullptr;
    std::vector<Scene> scenes;
    int32_t next_id = 0;
    uint32_t n_total = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;
    bool layout_dirty = false;  // scenes added/removed since the last repack_tables
    bool stepped = false;
    // input states of the resident scenes (packed like x, v); in feed mode
    // every step starts from them
    float4* x0 = nullptr;
    float4* v0 = nullptr;
    bool feed = false;
};

namespace {

void drop_graph(pfs_batch* B) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
}

size_t batch_arena_bytes(uint32_t cap_n, uint32_t cap_s, int precision, uint32_t blocks_cap) {
    size_t b = world_arena_bytes(cap_n, 0, precision, blocks_cap, NLIST_CAP_MAX, 0);
    b += (size_t)cap_s * sizeof(DevParams) + (size_t)cap_n * 4 /*sid*/ + ((size_t)cap_s + 1) * 4;
    b += 2 * (size_t)cap_n * 16; /* x0 v0 */
    return b + 8 * 256;
}

DevParams global_params(uint32_t n, uint32_t blocks) {
    DevParams P{};
    P.n = n;
    P.mask = n ? n - 1 : 0;
    P.nbx = blocks;
    P.nby = P.nbz = 1;
    P.list_cap = NLIST_CAP_MAX;
    return P;
}

// Re-derive every scene's device parameters for the current packing, upload
// them, refill the per-slot scene ids and recompute all keys.
int repack_tables(pfs_batch* B) {
    uint32_t block_base = 0;
    uint32_t geo_any = 0;
    std::vector<DevParams> dps(B->scenes.size());
    std::vector<uint32_t> offs(B->scenes.size() + 1);
    for (size_t k = 0; k < B->scenes.size(); k++) {
        Scene& s = B->scenes[k];
        DevParams d = s.dp;
        d.n = B->n_total;
        d.key_base = s.off;
        d.block_base = block_base;
        d.list_cap = NLIST_CAP_MAX;
        block_base += spatial_blocks(d);
        geo_any |= d.geo;
        dps[k] = d;
        offs[k] = s.off;
    }
    offs[B->scenes.size()] = B->n_total;
    if (block_base > B->blocks_cap) return PFS_ERANGE;  // cannot happen: blocks are capped per scene
    B->b.nblocks = block_base;
    B->b.geo_any = geo_any;
    cudaError_t e = cudaSuccess;
    if (!dps.empty())
        e = cudaMemcpyAsync(B->d_scenes, dps.data(), dps.size() * sizeof(DevParams),
                            cudaMemcpyHostToDevice, B->stream);
    if (e == cudaSuccess && B->n_total) {
        e = cudaMemcpyAsync(B->d_offs, offs.data(), offs.size() * 4, cudaMemcpyHostToDevice,
                            B->stream);
        if (e == cudaSuccess) {
            k_fill_sid<<<grid256(B->n_total), 256, 0, B->stream>>>(
                B->n_total, B->d_offs, (uint32_t)B->scenes.size(), B->d_sid);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = launch_keys(global_params(B->n_total, block_base), B->b, B->stream);
    }
    // the host vectors must outlive the async copies
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    B->dirty = true;
    B->layout_dirty = false;
    return status_from_cuda(e);
}

// Scenes added or removed since the last repack: repack once, before the
// next use of the packed layout (so admitting many scenes costs one repack).
int ensure_layout(pfs_batch* B) {
    return B->layout_dirty ? repack_tables(B) : PFS_OK;
}

// Feed mode: restore the input states and their keys.
cudaError_t run_batch_feed(pfs_batch* B) {
    const size_t f4 = (size_t)B->n_total * 16;
    cudaError_t e = cudaMemcpyAsync(B->b.x, B->x0, f4, cudaMemcpyDeviceToDevice, B->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B->b.v, B->v0, f4, cudaMemcpyDeviceToDevice, B->stream);
    if (e == cudaSuccess) e = launch_keys(global_params(B->n_total, B->b.nblocks), B->b, B->stream);
    return e;
}

cudaError_t run_batch_substep(pfs_batch* B) {
    const DevParams P = global_params(B->n_total, B->b.nblocks);
    cudaError_t e;
    if ((e = launch_sort(P, B->b, B->stream)) != cudaSuccess) return e;
    if (B->precision == PFS_FP16_CELL) {
        if ((e = launch_reorder_fp16(P, B->b, B->h16, B->stream)) != cudaSuccess) return e;
        if ((e = launch_density_fp16(P, B->b, B->h16, B->stream)) != cudaSuccess) return e;
        if ((e = launch_force_fp16(P, B->b, B->h16, B->stream)) != cudaSuccess) return e;
    } else {
        if ((e = launch_reorder(P, B->b, B->stream)) != cudaSuccess) return e;
        if ((e = launch_density(P, B->b, B->stream)) != cudaSuccess) return e;
        if ((e = launch_force(P, B->b, B->stream)) != cudaSuccess) return e;
    }
    return launch_integrate(P, B->b, B->stream);
}

Scene* find_scene(pfs_batch* B, int32_t id, size_t* index = nullptr) {
    for (size_t k = 0; k < B->scenes.size(); k++)
        if (B->scenes[k].id == id) {
            if (index) *index = k;
            return &B->scenes[k];
        }
    return nullptr;
}

}  // namespace

extern "C" {

uint64_t pfs_batch_bytes(uint32_t max_particles, uint32_t max_scenes, int32_t precision) {
    const uint32_t blocks = kBlocksPerParticle * max_particles + kBlocksPerScene * max_scenes;
    return batch_arena_bytes(max_particles, max_scenes, precision, blocks);
}

int pfs_batch_create(uint32_t max_particles, uint32_t max_scenes, int32_t precision,
                     int32_t substeps, pfs_batch** out) {
    if (!out) return PFS_EINVAL;
    *out = nullptr;
    if (max_particles == 0 || max_scenes == 0) return PFS_EINVAL;
    if (max_particles > PFS_MAX_PARTICLES || max_scenes > (1u << 16)) return PFS_ERANGE;
    if (precision != PFS_FP32 && precision != PFS_FP16_CELL) return PFS_EINVAL;
    if (substeps < 1 || substeps > 1000000) return PFS_EINVAL;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return PFS_ENODEV;
    pfs_batch* B = new (std::nothrow) pfs_batch();
    if (!B) return PFS_ENOMEM;
    cudaGetDevice(&B->device);
    B->cap_n = max_particles;
    B->cap_s = max_scenes;
    B->precision = precision;
    B->substeps = substeps;
    B->blocks_cap = kBlocksPerParticle * max_particles + kBlocksPerScene * max_scenes;
    cudaError_t e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = B->arena.reserve(batch_arena_bytes(max_particles, max_scenes, precision, B->blocks_cap));
    if (e != cudaSuccess) {
        pfs_batch_destroy(B);
        return status_from_cuda(e);
    }
    Arena& a = B->arena;
    const size_t f4 = (size_t)max_particles * 16, u = (size_t)max_particles * 4;
    StepBuffers& b = B->b;
    b.x = (float4*)a.take(f4);
    b.v = (float4*)a.take(f4);
    b.xs = (float4*)a.take(f4);
    b.vs = (float4*)a.take(f4);
    b.xp = (float4*)a.take(f4);
    b.vp = (float4*)a.take(f4);
    b.rr = (float2*)a.take((size_t)max_particles * 8);
    b.keys = (uint32_t*)a.take(u);
    b.skeys = (uint32_t*)a.take(u);
    b.perm = (uint32_t*)a.take(u);
    b.keys_tmp = (uint32_t*)a.take(u);
    b.vals_tmp = (uint32_t*)a.take(u);
    b.sort_scratch = (uint32_t*)a.take(sort_scratch_words(max_particles, sort_key_bits(max_particles)) * 4);
    b.table = (int2*)a.take((size_t)max_particles * 8);
    b.err = (uint32_t*)a.take(256);
    b.order = (uint32_t*)a.take(u);
    b.bucket = (uint32_t*)a.take(u);
    b.brank = (uint32_t*)a.take(u);
    b.bcount = (uint32_t*)a.take((size_t)B->blocks_cap * 4);
    b.boffset = (uint32_t*)a.take((size_t)B->blocks_cap * 4);
    b.bcounter = (uint32_t*)a.take(256);
    b.nlist = (int32_t*)a.take((size_t)NLIST_CAP_MAX * u);
    b.ncount = (int32_t*)a.take(u);
    b.scanq = (uint32_t*)a.take(u);
    b.scanq_n = (uint32_t*)a.take(256);
    B->d_scenes = (DevParams*)a.take((size_t)max_scenes * sizeof(DevParams));
    B->d_sid = (uint32_t*)a.take(u);
    B->d_offs = (uint32_t*)a.take(((size_t)max_scenes + 1) * 4);
    B->x0 = (float4*)a.take(f4);
    B->v0 = (float4*)a.take(f4);
    b.sr = SceneRef{B->d_scenes, B->d_sid};
    b.nblocks = 0;
    b.variant = B->precision == PFS_FP16_CELL ? (int)NBR_LIST : nbr_variant();
    bool ok = b.x && b.v && b.xs && b.vs && b.xp && b.vp && b.rr && b.keys && b.skeys && b.perm &&
              b.keys_tmp && b.vals_tmp && b.sort_scratch && b.table && b.err && b.order &&
              b.bucket && b.brank && b.bcount && b.boffset && b.bcounter && b.nlist && b.ncount &&
              b.scanq && b.scanq_n && B->d_scenes && B->d_sid && B->d_offs && B->x0 && B->v0;
    if (ok && precision == PFS_FP16_CELL) ok = fp16_carve(a, max_particles, &B->h16);
    if (!ok) {
        pfs_batch_destroy(B);
        return PFS_ENOMEM;
    }
    e = cudaMemsetAsync(b.err, 0, 4, B->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.bcount, 0, (size_t)B->blocks_cap * 4, B->stream);
    if (e == cudaSuccess) e = launch_table_clear(global_params(max_particles, 0), b, B->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    if (e != cudaSuccess) {
        pfs_batch_destroy(B);
        return status_from_cuda(e);
    }
    *out = B;
    return PFS_OK;
}

int pfs_batch_add_scene(pfs_batch* B, const pfs_params* p, uint32_t n, const float* pos4,
                        const float* vel4, int32_t* scene_id) {
    if (!B || !pos4 || n == 0) return PFS_EINVAL;
    int rc = pfs_params_validate(p);
    if (rc) return rc;
    if (p->precision != B->precision || p->substeps != B->substeps) return PFS_EINVAL;
    if ((uint64_t)B->n_total + n > B->cap_n || B->scenes.size() >= B->cap_s) return PFS_EBUDGET;
    if ((rc = status_from_cuda(cudaSetDevice(B->device)))) return rc;
    Scene s{};
    s.id = B->next_id++;
    s.off = B->n_total;
    s.n = n;
    s.params = *p;
    derive_params(*p, n, &s.dp);
    fit_spatial_blocks(&s.dp, std::max(kBlocksPerParticle * n, kBlocksPerScene));
    const size_t f4 = (size_t)n * 16;
    cudaError_t e = cudaMemcpyAsync(B->b.x + s.off, pos4, f4, cudaMemcpyDefault, B->stream);
    if (e == cudaSuccess) {
        if (vel4)
            e = cudaMemcpyAsync(B->b.v + s.off, vel4, f4, cudaMemcpyDefault, B->stream);
        else
            e = cudaMemsetAsync(B->b.v + s.off, 0, f4, B->stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->x0 + s.off, B->b.x + s.off, f4, cudaMemcpyDeviceToDevice, B->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->v0 + s.off, B->b.v + s.off, f4, cudaMemcpyDeviceToDevice, B->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    B->scenes.push_back(s);
    B->n_total += n;
    B->layout_dirty = true;
    B->dirty = true;
    if (scene_id) *scene_id = s.id;
    return PFS_OK;
}

int pfs_batch_remove_scene(pfs_batch* B, int32_t id) {
    if (!B) return PFS_EINVAL;
    size_t k = 0;
    Scene* s = find_scene(B, id, &k);
    if (!s) return PFS_ENOTFOUND;
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    const uint32_t off = s->off, n = s->n;
    const uint32_t tail = B->n_total - (off + n);
    cudaError_t e = cudaSuccess;
    if (tail) {
        // move the later scenes down through the gather buffers (regions overlap)
        const size_t f4 = (size_t)tail * 16;
        e = cudaMemcpyAsync(B->b.xs, B->b.x + off + n, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.vs, B->b.v + off + n, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.x + off, B->b.xs, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.v + off, B->b.vs, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.xs, B->x0 + off + n, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.vs, B->v0 + off + n, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->x0 + off, B->b.xs, f4, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->v0 + off, B->b.vs, f4, cudaMemcpyDeviceToDevice, B->stream);
        // densities of the moved scenes stay readable (read_scene reports them)
        const size_t f2 = (size_t)tail * 8;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.xp, B->b.rr + off + n, f2, cudaMemcpyDeviceToDevice, B->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(B->b.rr + off, B->b.xp, f2, cudaMemcpyDeviceToDevice, B->stream);
    }
    if (e != cudaSuccess) return status_from_cuda(e);
    B->scenes.erase(B->scenes.begin() + (long)k);
    for (size_t q = k; q < B->scenes.size(); q++) B->scenes[q].off -= n;
    B->n_total -= n;
    B->layout_dirty = true;
    B->dirty = true;
    return PFS_OK;
}

int pfs_batch_step(pfs_batch* B, uint32_t nsteps) {
    if (!B) return PFS_EINVAL;
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    if (nsteps == 0 || B->n_total == 0) return PFS_OK;
    if ((rc = ensure_layout(B))) return rc;
    if (B->dirty || !B->exec) {
        drop_graph(B);
        cudaError_t e = cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return status_from_cuda(e);
        cudaError_t le = B->feed ? run_batch_feed(B) : cudaSuccess;
        for (int k = 0; k < B->substeps && le == cudaSuccess; k++) le = run_batch_substep(B);
        e = cudaStreamEndCapture(B->stream, &B->graph);
        if (le != cudaSuccess || e != cudaSuccess) {
            drop_graph(B);
            return status_from_cuda(le != cudaSuccess ? le : e);
        }
        e = cudaGraphInstantiate(&B->exec, B->graph, 0);
        if (e != cudaSuccess) {
            drop_graph(B);
            return status_from_cuda(e);
        }
        B->dirty = false;
    }
    for (uint32_t s = 0; s < nsteps; s++) {
        cudaError_t e = cudaGraphLaunch(B->exec, B->stream);
        if (e != cudaSuccess) return status_from_cuda(e);
    }
    B->stepped = true;
    return PFS_OK;
}

int pfs_batch_sync(pfs_batch* B, uint64_t timeout_ns) {
    if (!B) return PFS_EINVAL;
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    if (timeout_ns == 0) {
        rc = status_from_cuda(cudaStreamSynchronize(B->stream));
    } else {
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            cudaError_t e = cudaStreamQuery(B->stream);
            if (e == cudaSuccess) break;
            if (e != cudaErrorNotReady) return status_from_cuda(e);
            const auto dt = std::chrono::steady_clock::now() - t0;
            if ((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(dt).count() >= timeout_ns)
                return PFS_ETIMEDOUT;
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
    if (rc) return rc;
    uint32_t word = 0;
    cudaError_t e = cudaMemcpy(&word, B->b.err, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return status_from_cuda(e);
    return word ? PFS_EDEVICE : PFS_OK;
}

int pfs_batch_read_scene(pfs_batch* B, int32_t id, float* pos4, float* vel4, float* density) {
    if (!B) return PFS_EINVAL;
    Scene* s = find_scene(B, id);
    if (!s) return PFS_ENOTFOUND;
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    const size_t f4 = (size_t)s->n * 16;
    cudaError_t e = cudaSuccess;
    if (pos4) e = cudaMemcpyAsync(pos4, B->b.x + s->off, f4, cudaMemcpyDefault, B->stream);
    if (vel4 && e == cudaSuccess)
        e = cudaMemcpyAsync(vel4, B->b.v + s->off, f4, cudaMemcpyDefault, B->stream);
    if (density && e == cudaSuccess) {
        if (!B->stepped) return PFS_EINVAL;
        float* tmp = reinterpret_cast<float*>(B->b.keys_tmp);
        k_density_out<<<grid256(s->n), 256, 0, B->stream>>>(s->n, B->b.rr + s->off, tmp);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(density, tmp, (size_t)s->n * 4, cudaMemcpyDefault, B->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    return status_from_cuda(e);
}

int pfs_batch_write_scene(pfs_batch* B, int32_t id, const float* pos4, const float* vel4) {
    if (!B || !pos4) return PFS_EINVAL;
    Scene* s = find_scene(B, id);
    if (!s) return PFS_ENOTFOUND;
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    const size_t f4 = (size_t)s->n * 16;
    cudaError_t e = cudaMemcpyAsync(B->b.x + s->off, pos4, f4, cudaMemcpyDefault, B->stream);
    if (e == cudaSuccess) {
        if (vel4)
            e = cudaMemcpyAsync(B->b.v + s->off, vel4, f4, cudaMemcpyDefault, B->stream);
        else
            e = cudaMemsetAsync(B->b.v + s->off, 0, f4, B->stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->x0 + s->off, B->b.x + s->off, f4, cudaMemcpyDeviceToDevice, B->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(B->v0 + s->off, B->b.v + s->off, f4, cudaMemcpyDeviceToDevice, B->stream);
    // keys of the new state (a pending repack recomputes all keys anyway)
    if (e == cudaSuccess && !B->layout_dirty)
        e = launch_keys(global_params(B->n_total, B->b.nblocks), B->b, B->stream);
    return status_from_cuda(e);
}

// Kernel shape of the batch and neighbour search of every scene (search -1:
// each scene's automatic choice); takes effect at the next step.
static int batch_apply_shape(pfs_batch* B, int32_t shape, int32_t search) {
    if (shape < NBR_SIMPLE || shape > NBR_FLAT || search < -1 || search > 1) return PFS_EINVAL;
    B->b.variant = shape;
    for (Scene& s : B->scenes) {
        derive_params(s.params, s.n, &s.dp, search);
        fit_spatial_blocks(&s.dp, std::max(kBlocksPerParticle * s.n, kBlocksPerScene));
    }
    B->layout_dirty = true;
    B->dirty = true;
    return PFS_OK;
}

int pfs_batch_set_shape(pfs_batch* B, int32_t shape, int32_t search) {
    if (!B) return PFS_EINVAL;
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    rc = status_from_cuda(cudaStreamSynchronize(B->stream));
    return rc ? rc : batch_apply_shape(B, shape, search);
}

int pfs_batch_autotune(pfs_batch* B, uint32_t trial_steps, pfs_tune_result* out) {
    if (!B || !out) return PFS_EINVAL;
    std::memset(out, 0, sizeof(*out));
    int rc = status_from_cuda(cudaSetDevice(B->device));
    if (rc) return rc;
    if (B->n_total == 0) return PFS_OK;
    if ((rc = status_from_cuda(cudaStreamSynchronize(B->stream)))) return rc;
    if (trial_steps == 0) trial_steps = 2;
    const int32_t keep_shape = B->b.variant;
    std::vector<std::pair<int32_t, int32_t>> cand;
    const bool fp16 = B->precision == PFS_FP16_CELL;
    for (int32_t shape : {NBR_LIST, NBR_FLAT, NBR_COMPACT, NBR_SIMPLE}) {
        if (fp16 && shape != NBR_LIST) continue;
        cand.push_back({shape, -1});
        cand.push_back({shape, 0});
    }
    const size_t f4 = (size_t)B->n_total * 16, f2 = (size_t)B->n_total * 8;
    char* snap = nullptr;
    cudaError_t e = cudaMalloc(&snap, 2 * f4 + f2);
    if (e != cudaSuccess) return status_from_cuda(e);
    auto copy_state = [&](bool save) -> cudaError_t {
        char* q = snap;
        auto one = [&](void* dev, size_t bytes) -> cudaError_t {
            cudaError_t r = save ? cudaMemcpyAsync(q, dev, bytes, cudaMemcpyDeviceToDevice, B->stream)
                                 : cudaMemcpyAsync(dev, q, bytes, cudaMemcpyDeviceToDevice, B->stream);
            q += bytes;
            return r;
        };
        cudaError_t r = one(B->b.x, f4);
        if (r == cudaSuccess) r = one(B->b.v, f4);
        if (r == cudaSuccess) r = one(B->b.rr, f2);
        return r;
    };
    if ((rc = ensure_layout(B))) {
        cudaFree(snap);
        return rc;
    }
    e = copy_state(true);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best = INFINITY;
    int32_t chosen = -1;
    auto restore = [&]() -> int {
        cudaError_t r = copy_state(false);
        if (r == cudaSuccess)
            r = launch_keys(global_params(B->n_total, B->b.nblocks), B->b, B->stream);
        return status_from_cuda(r);
    };
    for (size_t k = 0; k < cand.size() && k < PFS_TUNE_MAX && e == cudaSuccess; k++) {
        if ((rc = batch_apply_shape(B, cand[k].first, cand[k].second))) break;
        if ((rc = ensure_layout(B))) break;
        if ((rc = restore())) break;
        if ((rc = pfs_batch_step(B, 1))) break;
        if ((rc = restore())) break;
        if ((e = cudaEventRecord(e0, B->stream)) != cudaSuccess) break;
        if ((rc = pfs_batch_step(B, trial_steps))) break;
        if ((e = cudaEventRecord(e1, B->stream)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        out->shape[out->candidates] = cand[k].first;
        out->search[out->candidates] = cand[k].second;
        out->ms_per_step[out->candidates] = ms / (float)trial_steps;
        if (ms < best) {
            best = ms;
            chosen = out->candidates;
        }
        out->candidates++;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    const bool ok = rc == PFS_OK && e == cudaSuccess && chosen >= 0;
    int rc2 = ok ? batch_apply_shape(B, out->shape[chosen], out->search[chosen])
                 : batch_apply_shape(B, keep_shape, -1);
    out->chosen = ok ? chosen : -1;
    if (!rc2) rc2 = ensure_layout(B);
    if (!rc2) rc2 = restore();
    if (!rc2) rc2 = status_from_cuda(cudaStreamSynchronize(B->stream));
    cudaFree(snap);
    if (rc) return rc;
    if (e != cudaSuccess) return status_from_cuda(e);
    return rc2;
}

int pfs_batch_set_feed(pfs_batch* B, int enable) {
    if (!B) return PFS_EINVAL;
    if ((enable != 0) != B->feed) B->dirty = true;
    B->feed = enable != 0;
    return PFS_OK;
}

int pfs_batch_info_get(pfs_batch* B, pfs_batch_info* out) {
    if (!B || !out) return PFS_EINVAL;
    std::memset(out, 0, sizeof(*out));
    out->particles = B->n_total;
    out->scenes = (uint32_t)B->scenes.size();
    out->max_particles = B->cap_n;
    out->max_scenes = B->cap_s;
    out->device_bytes = B->arena.bytes;
    bool geo = false;
    for (const Scene& s : B->scenes) geo = geo || s.dp.geo != 0;
    out->launches_per_substep = substep_launches(B->n_total ? B->n_total : 1, geo);
    return PFS_OK;
}

void* pfs_batch_stream(pfs_batch* B) { return B ? (void*)B->stream : nullptr; }

int pfs_batch_destroy(pfs_batch* B) {
    if (!B) return PFS_EINVAL;
    cudaSetDevice(B->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    drop_graph(B);
    B->arena.release();
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
    return PFS_OK;
}

}  // extern "C"
