// pfs_world.cu — the C ABI of one SPH world (include/pfs.h).
//
// Replaces the reference's substep block (src/renderer/commands.c:193-402)
// and its buffer setup (src/renderer/renderer.c:510-754).  The host side owns
// one CUDA stream per world, one device arena holding every particle array,
// and a CUDA graph of one step (params.substeps substeps) captured on first
// use, so a step costs one graph launch instead of ~13 kernel launches per
// substep re-recorded every frame (renderer.c:404).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <new>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pfs.h"
#include "pfs_common.cuh"
#include "pfs_fp16.cuh"
#include "pfs_geo.cuh"
#include "pfs_sort.cuh"
#include "pfs_staged.cuh"
#include "pfs_step.cuh"
#include "pfs_world_impl.cuh"

namespace pfs {

// Neighbour search of a table of n particles over a grid of g cells per
// axis.  The table has 2^popcount(n - 1) slots; when that is a quarter of n
// or less, slot ranges mix many distant cells and the grid search
// (pfs_geo.cuh) reads far fewer candidates.  PFS_NEIGHBOR_SEARCH=table|grid
// forces one (grid only where the grid bound allows it).
static bool choose_grid_search(uint32_t n, const uint32_t g[3], int search) {
    for (int a = 0; a < 3; a++)
        if (g[a] > GEO_MAX_CELLS) return false;
    if (search == 0) return false;
    if (search == 1) return n > 0;
    const char* e = getenv("PFS_NEIGHBOR_SEARCH");
    if (e && strcmp(e, "table") == 0) return false;
    if (e && strcmp(e, "grid") == 0) return n > 0;
    if (n < 2) return false;
    const uint64_t slots = 1ull << __builtin_popcount(n - 1u);
    return slots * 4 <= (uint64_t)n;
}

// Same arithmetic as the oracle's pfso_derive: volume per main.c:349 in
// double, kernel scales per calculateDensities.comp:110 and
// applyPressureAndViscosityForce.comp:89,104 in float, PI = 3.14159265359f.
void derive_params(const pfs_params& p, uint32_t n, DevParams* o, int search) {
    const float PI = 3.14159265359f;
    const float h = p.h;
    o->h = h;
    o->rho0 = p.target_density;
    o->k = p.pressure_multiplier;
    o->kn = p.near_pressure_multiplier;
    o->visc = p.viscosity;
    o->m = p.particle_mass;
    o->gx = p.gravity[0]; o->gy = p.gravity[1]; o->gz = p.gravity[2];
    o->dt = p.dt;
    o->minx = p.box_min[0]; o->miny = p.box_min[1]; o->minz = p.box_min[2];
    o->maxx = p.box_max[0]; o->maxy = p.box_max[1]; o->maxz = p.box_max[2];
    o->margin_p = p.margin_predict;
    o->margin_i = p.margin_integrate;
    for (int i = 0; i < 6; i++) o->rest[i] = p.restitution[i];
    if (p.volume > 0.0f)
        o->volume = p.volume;
    else
        o->volume = (float)(2.0f * M_PI * pow((double)h, 5) / 15.0f);
    o->near_inv = 15.0f / (PI * powf(h, 6.0f));
    o->slope_scale = 15.0f / (PI * powf(h, 5.0f));
    o->near_slope_scale = -45.0f / (PI * powf(h, 6.0f));
    o->r2 = h * h;
    float t = h * h;
    while (t > 0.0f && sqrtf(nextafterf(t, 0.0f)) >= h) t = nextafterf(t, 0.0f);
    while (sqrtf(t) < h) t = nextafterf(t, INFINITY);
    o->skip_d2 = t;
    o->mask = n > 0 ? n - 1u : 0u;
    o->n = n;
    o->flags = p.flags;
    // grid of cells over the box and the blocks the spatial order groups them
    // into: 2x2x2 cells, coarser when the box is large against n
    uint32_t g[3];
    for (int a = 0; a < 3; a++) {
        double cells = std::floor(((double)p.box_max[a] - (double)p.box_min[a]) / (double)h) + 1.0;
        g[a] = (uint32_t)std::min(std::max(cells, 1.0), (double)(1u << 20));
    }
    o->ngx = g[0]; o->ngy = g[1]; o->ngz = g[2];
    o->geo = choose_grid_search(n, g, search) ? 1u : 0u;
    const double cap = std::max(4.0 * (double)n, 4096.0);
    // the grid search reads single cells when the buffers allow it
    int s = o->geo ? 0 : 1;
    for (;; s++) {
        const double nb = (double)((g[0] - 1) >> s) + 1.0;
        const double blocks = nb * ((double)((g[1] - 1) >> s) + 1.0) * ((double)((g[2] - 1) >> s) + 1.0);
        if (blocks <= cap || s >= 20) break;
    }
    o->bshift = s;
    o->nbx = ((g[0] - 1) >> s) + 1;
    o->nby = ((g[1] - 1) >> s) + 1;
    o->nbz = ((g[2] - 1) >> s) + 1;
    o->key_base = 0;
    o->block_base = 0;
    o->list_cap = NLIST_CAP;
    o->staged = 0;
    o->sbx = o->sby = o->sbz = 0;
    o->nsx = o->nsy = o->nsz = 1;
    {
        const float c = 1e-7f;
        float m = c * c;
        while (m > 0.0f && sqrtf(nextafterf(m, 0.0f)) >= c) m = nextafterf(m, 0.0f);
        while (sqrtf(m) < c) m = nextafterf(m, INFINITY);
        o->min_d2 = m;
    }
}

uint32_t spatial_blocks(const DevParams& P) { return P.nbx * P.nby * P.nbz; }

bool grid_search_allowed(const pfs_params& p, uint32_t n) {
    DevParams d{};
    derive_params(p, n, &d, 1);
    return d.geo != 0;
}

// Coarsen the spatial-order blocks until they fit buffers sized for `cap`.
void fit_spatial_blocks(DevParams* o, uint32_t cap) {
    while (spatial_blocks(*o) > cap && o->bshift < 20) {
        o->bshift++;
        o->nbx = ((o->ngx - 1) >> o->bshift) + 1;
        o->nby = ((o->ngy - 1) >> o->bshift) + 1;
        o->nbz = ((o->ngz - 1) >> o->bshift) + 1;
    }
}

int status_from_cuda(cudaError_t e) {
    if (e == cudaSuccess) return PFS_OK;
    if (e == cudaErrorMemoryAllocation) return PFS_ENOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return PFS_ENODEV;
    return PFS_ECUDA;
}

Arena::~Arena() { release(); }

void Arena::release() {
    if (base) cudaFree(base);
    base = nullptr;
    bytes = used = 0;
}

cudaError_t Arena::reserve(size_t total) {
    release();
    if (total == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&base, total);
    if (e != cudaSuccess) {
        base = nullptr;
        return e;
    }
    bytes = total;
    used = 0;
    return cudaSuccess;
}

void* Arena::take(size_t n) {
    const size_t off = (used + 255) & ~size_t(255);
    if (off + n > bytes) return nullptr;
    used = off + n;
    return static_cast<char*>(base) + off;
}

size_t world_arena_bytes(uint32_t n, int flags, int precision, uint32_t blocks, uint32_t list_cap,
                         uint32_t staged_blocks) {
    const size_t f4 = (size_t)n * 16, u = (size_t)n * 4;
    size_t b = 6 * f4 /*x v xs vs xp vp*/ + (size_t)n * 8 /*rr*/ + 5 * u /*keys skeys perm tmp x2*/ +
               sort_scratch_words(n, sort_key_bits(n)) * 4 + (size_t)n * 8 /*table*/ + 256 /*err*/ +
               3 * u /*order bucket brank*/ + 2 * (size_t)blocks * 4 /*bcount boffset*/ + 256 +
               (size_t)(list_cap + 2) * u /*nlist ncount scanq*/ + 256;
    b += 3 * ((size_t)staged_blocks + 1) * 4 + 256;  // bseg btot blist, staged counters
    if (flags & PFS_FLAG_IDS_INTERNAL) b += 2 * u;
    if (flags & PFS_FLAG_COLORS) b += f4;
    if (precision == PFS_FP16_CELL) b += fp16_arena_bytes(n);
    return b + 32 * 256;  // alignment slack
}

}  // namespace pfs

using namespace pfs;

struct pfs_world {
    int device = 0;
    cudaStream_t stream = nullptr;
    pfs_params params{};
    DevParams dp{};
    uint32_t n = 0;
    int flags = 0;
    Arena arena;
    StepBuffers b{};
    Fp16Buffers h16{};
    uint32_t* err = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool profiling = false;
    std::vector<cudaEvent_t> pending;  // profiling events, 6 per substep
    pfs_stage_times times{};
    bool sorted_valid = false;  // skeys/perm hold a sort result
    uint32_t blocks_cap = 0;    // spatial-order buckets the arena holds
    int search = -1;            // neighbour search: -1 automatic, 0 table, 1 grid
    // staged shape (pfs_staged.cu): block shape picked from the initial
    // state's density, or unavailable (grid too large for fine buckets)
    bool staged_ok = false;
    DevParams staged_cfg{};
    uint32_t staged_blocks = 0;  // nsx * nsy * nsz
    uint32_t list_cap = NLIST_CAP;  // neighbour-list rows (list_rows_for)
    float* map_buf = nullptr;   // device grid of pfs_world_density_map (grown on demand)
    size_t map_cap = 0;         // floats it holds
    float* lv_buf = nullptr;    // light volume and image of pfs_world_render_volumetric
    size_t lv_cap = 0;
    // pfs_world_run_pipelined: copy streams, double-buffered staging
    // (input pos, vel and output pos, vel per slot) and their events
    cudaStream_t h2d = nullptr, d2h = nullptr;
    float* pipe_buf = nullptr;
    size_t pipe_cap = 0;
    cudaEvent_t pipe_ev[9] = {};  // in_ready[2], in_free[2], out_ready[2], out_free[2], start
};

namespace {

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

void drop_graph(pfs_world* w) {
    if (w->exec) cudaGraphExecDestroy(w->exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    w->exec = nullptr;
    w->graph = nullptr;
}

unsigned grid256(uint32_t n) { return (n + 255) / 256; }

__global__ void k_iota(uint32_t n, uint32_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

__global__ void k_fill_w(uint32_t n, float4* v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void k_split2(uint32_t n, const float2* in, float* a, float* b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float2 v = in[i];
        if (a) a[i] = v.x;
        if (b) b[i] = v.y;
    }
}

// One substep on the world's stream.  With profiling on, events bracket the
// five stages.
cudaError_t run_substep(pfs_world* w) {
    const DevParams& P = w->dp;
    cudaEvent_t ev[PFS_STAGE_COUNT + 1] = {};
    if (w->profiling) {
        for (auto& e : ev) {
            cudaError_t ce = cudaEventCreate(&e);
            if (ce != cudaSuccess) return ce;
        }
        cudaEventRecord(ev[0], w->stream);
    }
    cudaError_t e;
    if ((e = launch_sort(P, w->b, w->stream)) != cudaSuccess) return e;
    if (w->profiling) cudaEventRecord(ev[1], w->stream);
    if (w->params.precision == PFS_FP16_CELL) {
        if ((e = launch_reorder_fp16(P, w->b, w->h16, w->stream)) != cudaSuccess) return e;
        if (w->profiling) cudaEventRecord(ev[2], w->stream);
        if ((e = launch_density_fp16(P, w->b, w->h16, w->stream)) != cudaSuccess) return e;
        if (w->profiling) cudaEventRecord(ev[3], w->stream);
        if ((e = launch_force_fp16(P, w->b, w->h16, w->stream)) != cudaSuccess) return e;
    } else {
        if ((e = launch_reorder(P, w->b, w->stream)) != cudaSuccess) return e;
        if (w->profiling) cudaEventRecord(ev[2], w->stream);
        if ((e = launch_density(P, w->b, w->stream)) != cudaSuccess) return e;
        if (w->profiling) cudaEventRecord(ev[3], w->stream);
        if ((e = launch_force(P, w->b, w->stream)) != cudaSuccess) return e;
    }
    if (w->profiling) cudaEventRecord(ev[4], w->stream);
    if ((e = launch_integrate(P, w->b, w->stream)) != cudaSuccess) return e;
    if (w->profiling) {
        cudaEventRecord(ev[5], w->stream);
        for (auto& x : ev) w->pending.push_back(x);
    }
    w->sorted_valid = true;
    return cudaSuccess;
}

int capture_graph(pfs_world* w) {
    drop_graph(w);
    cudaError_t e = cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return status_from_cuda(e);
    const int subs = w->params.substeps;
    cudaError_t le = cudaSuccess;
    for (int s = 0; s < subs && le == cudaSuccess; s++) le = run_substep(w);
    e = cudaStreamEndCapture(w->stream, &w->graph);
    if (le != cudaSuccess) {
        drop_graph(w);
        return status_from_cuda(le);
    }
    if (e != cudaSuccess) {
        drop_graph(w);
        return status_from_cuda(e);
    }
    e = cudaGraphInstantiate(&w->exec, w->graph, 0);
    if (e != cudaSuccess) {
        drop_graph(w);
        return status_from_cuda(e);
    }
    return PFS_OK;
}

int set_device(pfs_world* w) { return status_from_cuda(cudaSetDevice(w->device)); }

int carve(pfs_world* w) {
    const uint32_t n = w->n;
    Arena& a = w->arena;
    // bucket counters hold the spatial blocks, or the staged shape's fine
    // buckets (cells padded to whole blocks) where that is more
    uint32_t blocks = spatial_blocks(w->dp);
    if (w->staged_ok) blocks = std::max<uint32_t>(blocks, (uint32_t)staged_buckets(w->staged_cfg));
    w->blocks_cap = blocks;
    cudaError_t e = a.reserve(world_arena_bytes(n, w->flags, w->params.precision, blocks, w->list_cap,
                                                w->staged_blocks));
    if (e != cudaSuccess) return status_from_cuda(e);
    const size_t f4 = (size_t)n * 16, u = (size_t)n * 4;
    StepBuffers& b = w->b;
    b.x = (float4*)a.take(f4);
    b.v = (float4*)a.take(f4);
    b.xs = (float4*)a.take(f4);
    b.vs = (float4*)a.take(f4);
    b.xp = (float4*)a.take(f4);
    b.vp = (float4*)a.take(f4);
    b.rr = (float2*)a.take((size_t)n * 8);
    b.keys = (uint32_t*)a.take(u);
    b.skeys = (uint32_t*)a.take(u);
    b.perm = (uint32_t*)a.take(u);
    b.keys_tmp = (uint32_t*)a.take(u);
    b.vals_tmp = (uint32_t*)a.take(u);
    b.sort_scratch = (uint32_t*)a.take(sort_scratch_words(n, sort_key_bits(n)) * 4);
    b.table = (int2*)a.take((size_t)n * 8);
    b.err = (uint32_t*)a.take(256);
    b.order = (uint32_t*)a.take(u);
    b.bucket = (uint32_t*)a.take(u);
    b.brank = (uint32_t*)a.take(u);
    b.bcount = (uint32_t*)a.take((size_t)blocks * 4);
    b.boffset = (uint32_t*)a.take((size_t)blocks * 4);
    b.bcounter = (uint32_t*)a.take(256);
    b.nlist = (int32_t*)a.take((size_t)w->list_cap * u);
    b.ncount = (int32_t*)a.take(u);
    b.scanq = (uint32_t*)a.take(u);
    b.scanq_n = (uint32_t*)a.take(256);
    b.bseg = (uint32_t*)a.take(((size_t)w->staged_blocks + 1) * 4);
    b.btot = (uint32_t*)a.take(((size_t)w->staged_blocks + 1) * 4);
    b.blist = (uint32_t*)a.take(((size_t)w->staged_blocks + 1) * 4);
    b.st_counters = (uint32_t*)a.take(256);
    b.fast = w->params.precision == PFS_FP32_FAST ? 1 : 0;
    b.sr = SceneRef{nullptr, nullptr};
    b.nblocks = spatial_blocks(w->dp);
    b.geo_any = w->dp.geo;
    // the FP16-cell form has one shape, the list shape's
    b.variant = w->params.precision == PFS_FP16_CELL ? (int)NBR_LIST : nbr_variant();
    if (!b.order || !b.bucket || !b.brank || !b.bcount || !b.boffset || !b.bcounter ||
        !b.nlist || !b.ncount || !b.scanq || !b.scanq_n || !b.bseg || !b.btot || !b.blist ||
        !b.st_counters)
        return PFS_ENOMEM;
    b.ids = b.ids_s = nullptr;
    b.color = nullptr;
    if (w->flags & PFS_FLAG_IDS_INTERNAL) {
        b.ids = (uint32_t*)a.take(u);
        b.ids_s = (uint32_t*)a.take(u);
    }
    if (w->flags & PFS_FLAG_COLORS) b.color = (float4*)a.take(f4);
    if (w->params.precision == PFS_FP16_CELL) {
        if (!fp16_carve(a, n, &w->h16)) return PFS_ENOMEM;
    }
    if (!b.x || !b.v || !b.xs || !b.vs || !b.xp || !b.vp || !b.rr || !b.keys || !b.skeys ||
        !b.perm || !b.keys_tmp || !b.vals_tmp || !b.sort_scratch || !b.table || !b.err)
        return PFS_ENOMEM;
    w->err = b.err;
    return PFS_OK;
}

int upload_state(pfs_world* w, const float* pos4, const float* vel4) {
    const size_t f4 = (size_t)w->n * 16;
    cudaError_t e = cudaMemcpyAsync(w->b.x, pos4, f4, cudaMemcpyDefault, w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    if (vel4) {
        e = cudaMemcpyAsync(w->b.v, vel4, f4, cudaMemcpyDefault, w->stream);
    } else {
        k_fill_w<<<grid256(w->n), 256, 0, w->stream>>>(w->n, w->b.v);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return status_from_cuda(e);
    if ((e = launch_keys(w->dp, w->b, w->stream)) != cudaSuccess) return status_from_cuda(e);
    if (w->b.ids) {
        k_iota<<<grid256(w->n), 256, 0, w->stream>>>(w->n, w->b.ids);
        if ((e = cudaGetLastError()) != cudaSuccess) return status_from_cuda(e);
    }
    w->sorted_valid = false;
    return PFS_OK;
}

int wait_stream(pfs_world* w, uint64_t timeout_ns) {
    if (timeout_ns == 0) return status_from_cuda(cudaStreamSynchronize(w->stream));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(w->stream);
        if (e == cudaSuccess) return PFS_OK;
        if (e != cudaErrorNotReady) return status_from_cuda(e);
        const auto dt = std::chrono::steady_clock::now() - t0;
        if ((uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(dt).count() >= timeout_ns)
            return PFS_ETIMEDOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

int check_err_word(pfs_world* w) {
    uint32_t word = 0;
    cudaError_t e = cudaMemcpy(&word, w->err, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return status_from_cuda(e);
    return word ? PFS_EDEVICE : PFS_OK;
}

}  // namespace

extern "C" {

void pfs_params_reference_default(pfs_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // src/main.c:11-22, 53-63, 356-358
    p->h = 2.5f;
    p->target_density = 1.0f;
    p->pressure_multiplier = 15000.0f;
    p->near_pressure_multiplier = 0.0f;
    p->viscosity = 1.0f;
    p->particle_mass = 1.0f;
    p->gravity[0] = 0.0f;
    p->gravity[1] = 0.0f;
    p->gravity[2] = -100.0f;
    p->dt = (float)(0.01 / (float)1);
    const float s = 40.0f;
    p->box_min[0] = (float)(-3.5 * s); p->box_min[1] = (float)(-1.00 * s); p->box_min[2] = (float)(-1.00 * s);
    p->box_max[0] = (float)(3.5 * s);  p->box_max[1] = (float)(1.00 * s);  p->box_max[2] = (float)(1.00 * s);
    const float radius = (float)0.3;
    p->margin_predict = radius;
    p->margin_integrate = radius + 0.5f;
    for (int i = 0; i < 6; i++) p->restitution[i] = 1.0f;
    p->restitution[4] = 0.95f;
    p->volume = 0.0f;
    p->substeps = 1;
    p->precision = PFS_FP32;
    p->flags = 0;
}

int pfs_params_validate(const pfs_params* p) {
    if (!p) return PFS_EINVAL;
    if (!(std::isfinite(p->h) && p->h > 0.0f)) return PFS_EINVAL;
    if (!(std::isfinite(p->dt) && p->dt >= 0.0f)) return PFS_EINVAL;
    if (!std::isfinite(p->target_density) || !std::isfinite(p->pressure_multiplier) ||
        !std::isfinite(p->near_pressure_multiplier) || !std::isfinite(p->viscosity) ||
        !std::isfinite(p->particle_mass) || !std::isfinite(p->volume))
        return PFS_EINVAL;
    if (!finite3(p->gravity) || !finite3(p->box_min) || !finite3(p->box_max)) return PFS_EINVAL;
    for (int a = 0; a < 3; a++)
        if (!(p->box_min[a] < p->box_max[a])) return PFS_EINVAL;
    if (!std::isfinite(p->margin_predict) || !std::isfinite(p->margin_integrate)) return PFS_EINVAL;
    for (int i = 0; i < 6; i++)
        if (!std::isfinite(p->restitution[i])) return PFS_EINVAL;
    if (p->substeps < 1 || p->substeps > 1000000) return PFS_EINVAL;
    if (p->precision != PFS_FP32 && p->precision != PFS_FP16_CELL && p->precision != PFS_FP32_FAST)
        return PFS_EINVAL;
    if (p->flags & ~(PFS_FLAG_COLORS | PFS_FLAG_IDS)) return PFS_EINVAL;
    if (p->precision == PFS_FP16_CELL) {
        const int rc = fp16_check_box(*p);
        if (rc) return rc;
    }
    return PFS_OK;
}

const char* pfs_strerror(int s) {
    switch (s) {
        case PFS_OK: return "ok";
        case PFS_EINVAL: return "invalid argument or parameter set";
        case PFS_ENOMEM: return "out of memory";
        case PFS_ECUDA: return "CUDA runtime error";
        case PFS_ETIMEDOUT: return "timed out";
        case PFS_ENODEV: return "no usable CUDA device";
        case PFS_EDEVICE: return "device-side bounds check tripped";
        case PFS_ERANGE: return "size out of range";
        case PFS_EBUDGET: return "refused by the HBM budget";
        case PFS_ENOTFOUND: return "unknown handle";
        default: return "unknown status";
    }
}

int pfs_version(void) { return 10000; }

// Neighbour-list rows of a new world: twice the mean neighbour count of its
// initial state (particles in their bounding box, clipped to the world box,
// times the volume of a sphere of radius h), rounded up to 16 and kept within
// [NLIST_CAP, NLIST_CAP_MAX].  Particles of denser regions than that fall back
// to the force pass's scan, with the same results.
static bool is_device_ptr(const void* p);
static int apply_shape(pfs_world* w, int32_t shape, int32_t search);

static uint32_t list_rows_for(const pfs_params& p, uint32_t n, const float* pos4) {
    if (n == 0 || !pos4) return NLIST_CAP;
    double lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = INFINITY;
        hi[a] = -INFINITY;
    }
    const bool dev = [&] {
        cudaPointerAttributes attr{};
        if (cudaPointerGetAttributes(&attr, pos4) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return attr.type == cudaMemoryTypeDevice;
    }();
    if (dev) return NLIST_CAP_MAX;  // device input: no host pass over it
    for (uint32_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            const double v = pos4[4 * (size_t)i + a];
            if (v >= p.box_min[a] && v <= p.box_max[a]) {
                lo[a] = std::min(lo[a], v);
                hi[a] = std::max(hi[a], v);
            }
        }
    double vol = 1.0;
    for (int a = 0; a < 3; a++) vol *= std::max(hi[a] - lo[a], (double)p.h);
    const double h = p.h;
    const double nb = 2.0 * (double)n / vol * (4.0 / 3.0) * 3.14159265358979 * h * h * h;
    if (!(nb > NLIST_CAP)) return NLIST_CAP;
    if (nb >= NLIST_CAP_MAX) return NLIST_CAP_MAX;
    return std::min<uint32_t>(((uint32_t)nb + 15u) & ~15u, NLIST_CAP_MAX);
}

int pfs_world_create(const pfs_params* p, uint32_t n, const float* pos4, const float* vel4,
                     pfs_world** out) {
    if (!out) return PFS_EINVAL;
    *out = nullptr;
    int rc = pfs_params_validate(p);
    if (rc) return rc;
    if (n == 0 || !pos4) return PFS_EINVAL;
    if (n > PFS_MAX_PARTICLES) return PFS_ERANGE;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return PFS_ENODEV;
    pfs_world* w = new (std::nothrow) pfs_world();
    if (!w) return PFS_ENOMEM;
    cudaGetDevice(&w->device);
    w->params = *p;
    w->n = n;
    w->flags = p->flags;
    if (w->flags & PFS_FLAG_IDS) w->flags |= PFS_FLAG_IDS_INTERNAL;
    derive_params(*p, n, &w->dp);
    w->list_cap = list_rows_for(*p, n, pos4);
    w->dp.list_cap = w->list_cap;
    {
        // staged block shape from the initial state's particles per cell
        // (device input: an assumed 2); FP32 forms only
        const double per_cell = is_device_ptr(pos4)
                                    ? 2.0
                                    : occupied_cell_density(pos4, n, p->box_min, p->box_max, p->h);
        w->staged_cfg = w->dp;
        w->staged_ok = p->precision != PFS_FP16_CELL &&
                       configure_staged(&w->staged_cfg, per_cell,
                                        (double)(1ull << __builtin_popcount(n - 1u)),
                                        8ull * n + 65536ull);
        w->staged_cfg.staged = w->staged_ok ? 1u : 0u;
        w->staged_blocks = w->staged_ok ? w->staged_cfg.nsx * w->staged_cfg.nsy * w->staged_cfg.nsz : 0u;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete w;
        return status_from_cuda(e);
    }
    rc = carve(w);
    if (rc == PFS_OK) {
        e = cudaMemsetAsync(w->err, 0, 4, w->stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(w->b.bcount, 0, (size_t)w->blocks_cap * 4, w->stream);
        if (e == cudaSuccess) e = launch_table_clear(w->dp, w->b, w->stream);
        rc = status_from_cuda(e);
    }
    // the staged shape (PFS_NBR_VARIANT=staged) needs its block
    // configuration applied; without one the flat shape runs
    if (rc == PFS_OK) {
        const bool want_staged = w->b.variant == NBR_STAGED;
        if (want_staged && w->staged_ok)
            rc = apply_shape(w, NBR_STAGED, 0);
        else if (w->b.variant == NBR_STAGED)
            w->b.variant = NBR_FLAT;
    }
    if (rc == PFS_OK) rc = upload_state(w, pos4, vel4);
    if (rc == PFS_OK) rc = status_from_cuda(cudaStreamSynchronize(w->stream));
    if (rc != PFS_OK) {
        pfs_world_destroy(w);
        return rc;
    }
    *out = w;
    return PFS_OK;
}

int pfs_world_set_params(pfs_world* w, const pfs_params* p) {
    if (!w) return PFS_EINVAL;
    int rc = pfs_params_validate(p);
    if (rc) return rc;
    if (p->precision != w->params.precision || (p->flags & ~w->params.flags)) return PFS_EINVAL;
    if ((rc = set_device(w))) return rc;
    if ((rc = wait_stream(w, 0))) return rc;
    const bool rekey = p->h != w->params.h || std::memcmp(p->box_min, w->params.box_min, 12) != 0;
    w->params = *p;
    derive_params(*p, w->n, &w->dp, w->search);
    w->dp.list_cap = w->list_cap;
    fit_spatial_blocks(&w->dp, w->blocks_cap);
    w->b.nblocks = spatial_blocks(w->dp);
    w->b.geo_any = w->dp.geo;
    drop_graph(w);
    if (rekey) {
        cudaError_t e = launch_keys(w->dp, w->b, w->stream);
        if (e != cudaSuccess) return status_from_cuda(e);
    }
    return PFS_OK;
}

int pfs_world_step(pfs_world* w, uint32_t nsteps) {
    if (!w) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    if (nsteps == 0) return PFS_OK;
    if (w->profiling) {
        for (uint32_t s = 0; s < nsteps; s++)
            for (int k = 0; k < w->params.substeps; k++) {
                cudaError_t e = run_substep(w);
                if (e != cudaSuccess) return status_from_cuda(e);
            }
        return PFS_OK;
    }
    if (!w->exec && (rc = capture_graph(w))) return rc;
    for (uint32_t s = 0; s < nsteps; s++) {
        cudaError_t e = cudaGraphLaunch(w->exec, w->stream);
        if (e != cudaSuccess) return status_from_cuda(e);
    }
    w->sorted_valid = true;
    return PFS_OK;
}

int pfs_world_run_pipelined(pfs_world* w, uint32_t count, const float* const* pos_in,
                            const float* const* vel_in, float* const* pos_out, float* const* vel_out,
                            uint32_t steps_each) {
    if (!w || !pos_in || !pos_out || steps_each == 0) return PFS_EINVAL;
    if (count == 0) return PFS_OK;
    for (uint32_t k = 0; k < count; k++)
        if (!pos_in[k] || !pos_out[k]) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    if (w->profiling) {  // stage timing has no pipelined form: run the plain sequence
        for (uint32_t k = 0; k < count; k++) {
            if ((rc = pfs_world_write(w, pos_in[k], vel_in ? vel_in[k] : nullptr))) return rc;
            if ((rc = pfs_world_step(w, steps_each))) return rc;
            if ((rc = pfs_world_read(w, pos_out[k], vel_out ? vel_out[k] : nullptr, nullptr, nullptr, nullptr)))
                return rc;
        }
        return PFS_OK;
    }
    cudaError_t e = cudaSuccess;
    if (!w->h2d) e = cudaStreamCreateWithFlags(&w->h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess && !w->d2h) e = cudaStreamCreateWithFlags(&w->d2h, cudaStreamNonBlocking);
    for (auto& ev : w->pipe_ev)
        if (e == cudaSuccess && !ev) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return status_from_cuda(e);
    const size_t f4 = (size_t)w->n * 16, fl = (size_t)w->n * 4;  // bytes, floats of one float4 array
    if (w->pipe_cap < 8 * fl) {
        if ((rc = wait_stream(w, 0))) return rc;
        if (w->pipe_buf) cudaFree(w->pipe_buf);
        w->pipe_buf = nullptr;
        w->pipe_cap = 0;
        if ((e = cudaMalloc(&w->pipe_buf, 8 * fl * sizeof(float))) != cudaSuccess) return status_from_cuda(e);
        w->pipe_cap = 8 * fl;
    }
    if (!w->exec && (rc = capture_graph(w))) return rc;
    cudaEvent_t* in_ready = w->pipe_ev;
    cudaEvent_t* in_free = w->pipe_ev + 2;
    cudaEvent_t* out_ready = w->pipe_ev + 4;
    cudaEvent_t* out_free = w->pipe_ev + 6;
    cudaEvent_t start = w->pipe_ev[8];
    auto in_pos = [&](uint32_t s) { return w->pipe_buf + (size_t)s * 2 * fl; };
    auto in_vel = [&](uint32_t s) { return w->pipe_buf + (size_t)s * 2 * fl + fl; };
    auto out_pos = [&](uint32_t s) { return w->pipe_buf + 4 * fl + (size_t)s * 2 * fl; };
    auto out_vel = [&](uint32_t s) { return w->pipe_buf + 4 * fl + (size_t)s * 2 * fl + fl; };
    // everything already queued on the world's stream comes first; the slot
    // events start out recorded so the first waits on them are satisfied
    e = cudaEventRecord(start, w->stream);
    for (int k = 0; k < 8 && e == cudaSuccess; k++) e = cudaEventRecord(w->pipe_ev[k], w->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w->h2d, start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w->d2h, start, 0);
    auto upload = [&](uint32_t k) -> cudaError_t {
        const uint32_t s = k & 1u;
        cudaError_t r = cudaStreamWaitEvent(w->h2d, in_free[s], 0);
        if (r == cudaSuccess) r = cudaMemcpyAsync(in_pos(s), pos_in[k], f4, cudaMemcpyDefault, w->h2d);
        if (r == cudaSuccess && vel_in && vel_in[k])
            r = cudaMemcpyAsync(in_vel(s), vel_in[k], f4, cudaMemcpyDefault, w->h2d);
        if (r == cudaSuccess) r = cudaEventRecord(in_ready[s], w->h2d);
        return r;
    };
    if (e == cudaSuccess) e = upload(0);
    for (uint32_t k = 0; k < count && e == cudaSuccess; k++) {
        const uint32_t s = k & 1u;
        // input k + 1 crosses the bus while input k steps
        if (k + 1 < count && (e = upload(k + 1)) != cudaSuccess) break;
        if ((e = cudaStreamWaitEvent(w->stream, in_ready[s], 0)) != cudaSuccess) break;
        if ((rc = upload_state(w, in_pos(s), vel_in && vel_in[k] ? in_vel(s) : nullptr))) {
            // no copy may still touch the caller's buffers when the call returns
            cudaStreamSynchronize(w->h2d);
            cudaStreamSynchronize(w->d2h);
            return rc;
        }
        if ((e = cudaEventRecord(in_free[s], w->stream)) != cudaSuccess) break;
        for (uint32_t t = 0; t < steps_each && e == cudaSuccess; t++) e = cudaGraphLaunch(w->exec, w->stream);
        if (e != cudaSuccess) break;
        w->sorted_valid = true;
        // the result leaves through a staging slot, so the next input can
        // overwrite the state while it is read back
        if ((e = cudaStreamWaitEvent(w->stream, out_free[s], 0)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(out_pos(s), w->b.x, f4, cudaMemcpyDeviceToDevice, w->stream)) != cudaSuccess) break;
        if (vel_out && vel_out[k] &&
            (e = cudaMemcpyAsync(out_vel(s), w->b.v, f4, cudaMemcpyDeviceToDevice, w->stream)) != cudaSuccess)
            break;
        if ((e = cudaEventRecord(out_ready[s], w->stream)) != cudaSuccess) break;
        if ((e = cudaStreamWaitEvent(w->d2h, out_ready[s], 0)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(pos_out[k], out_pos(s), f4, cudaMemcpyDefault, w->d2h)) != cudaSuccess) break;
        if (vel_out && vel_out[k] &&
            (e = cudaMemcpyAsync(vel_out[k], out_vel(s), f4, cudaMemcpyDefault, w->d2h)) != cudaSuccess)
            break;
        if ((e = cudaEventRecord(out_free[s], w->d2h)) != cudaSuccess) break;
    }
    // the world's stream ends after the last read-back
    if (e == cudaSuccess) e = cudaEventRecord(start, w->d2h);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w->stream, start, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->h2d);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) {
        // no copy may still touch the caller's buffers when the call returns
        cudaStreamSynchronize(w->h2d);
        cudaStreamSynchronize(w->d2h);
        return status_from_cuda(e);
    }
    return check_err_word(w);
}

int pfs_world_sync(pfs_world* w, uint64_t timeout_ns) {
    if (!w) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    if ((rc = wait_stream(w, timeout_ns))) return rc;
    return check_err_word(w);
}

int pfs_world_read(pfs_world* w, float* pos4, float* vel4, float* density, uint32_t* keys,
                   uint32_t* perm) {
    if (!w) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    // keys, perm and density exist only once a substep ran; refuse before
    // any copy is queued into the caller's buffers
    if ((keys || perm || density) && !w->sorted_valid) return PFS_EINVAL;
    const uint32_t n = w->n;
    const size_t f4 = (size_t)n * 16, u = (size_t)n * 4;
    cudaError_t e = cudaSuccess;
    if (pos4 && e == cudaSuccess) e = cudaMemcpyAsync(pos4, w->b.x, f4, cudaMemcpyDefault, w->stream);
    if (vel4 && e == cudaSuccess) e = cudaMemcpyAsync(vel4, w->b.v, f4, cudaMemcpyDefault, w->stream);
    if (density && e == cudaSuccess) {
        float* tmp = reinterpret_cast<float*>(w->b.keys_tmp);
        k_split2<<<grid256(n), 256, 0, w->stream>>>(n, w->b.rr, tmp, nullptr);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(density, tmp, u, cudaMemcpyDefault, w->stream);
    }
    if (keys && e == cudaSuccess) e = cudaMemcpyAsync(keys, w->b.skeys, u, cudaMemcpyDefault, w->stream);
    if (perm && e == cudaSuccess) e = cudaMemcpyAsync(perm, w->b.perm, u, cudaMemcpyDefault, w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    if ((rc = wait_stream(w, 0))) return rc;
    return check_err_word(w);
}

int pfs_world_read_colors(pfs_world* w, float* rgba4) {
    if (!w || !rgba4 || !w->b.color) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(rgba4, w->b.color, (size_t)w->n * 16, cudaMemcpyDeviceToHost, w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    return wait_stream(w, 0);
}

int pfs_world_read_ids(pfs_world* w, uint32_t* ids) {
    if (!w || !ids || !w->b.ids) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(ids, w->b.ids, (size_t)w->n * 4, cudaMemcpyDeviceToHost, w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    return wait_stream(w, 0);
}

int pfs_world_write(pfs_world* w, const float* pos4, const float* vel4) {
    if (!w || !pos4) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    return upload_state(w, pos4, vel4);
}

int pfs_world_destroy(pfs_world* w) {
    if (!w) return PFS_EINVAL;
    cudaSetDevice(w->device);
    if (w->stream) cudaStreamSynchronize(w->stream);
    for (auto e : w->pending) cudaEventDestroy(e);
    drop_graph(w);
    w->arena.release();
    if (w->map_buf) cudaFree(w->map_buf);
    if (w->lv_buf) cudaFree(w->lv_buf);
    if (w->h2d) cudaStreamSynchronize(w->h2d);
    if (w->d2h) cudaStreamSynchronize(w->d2h);
    if (w->pipe_buf) cudaFree(w->pipe_buf);
    for (auto& e : w->pipe_ev)
        if (e) cudaEventDestroy(e);
    if (w->h2d) cudaStreamDestroy(w->h2d);
    if (w->d2h) cudaStreamDestroy(w->d2h);
    if (w->stream) cudaStreamDestroy(w->stream);
    delete w;
    return PFS_OK;
}

// Density map extents: the image the reference allocates,
// (int)ceil((maxXYZ - minXYZ) * (1 / densityCellSize)) in float
// (renderer.c:774-781), and the shader's own bound
// ivec3(ceil((maxXYZ - minXYZ) / densityCellSize)) (updateDensityMap.comp:94).
static int density_map_extent(const pfs_params& p, float cell_size, int32_t image[3],
                              int32_t bound[3]) {
    if (!(cell_size > 0.0f) || !std::isfinite(cell_size)) return PFS_EINVAL;
    const float inv = 1.0f / cell_size;
    uint64_t voxels = 1;
    for (int a = 0; a < 3; a++) {
        const float ext = p.box_max[a] - p.box_min[a];
        const double img = std::ceil((double)(ext * inv));
        const float bnd = ceilf(ext / cell_size);
        if (!(img >= 0.0) || img > 65536.0 || !(bnd >= 0.0f) || bnd > 65536.0f) return PFS_ERANGE;
        image[a] = (int32_t)img;
        bound[a] = (int32_t)bnd;
        voxels *= (uint64_t)image[a];
    }
    return voxels > (1ull << 31) ? PFS_ERANGE : PFS_OK;
}

int pfs_world_density_map_dims(const pfs_world* w, float cell_size, uint32_t dims[3]) {
    if (!w || !dims) return PFS_EINVAL;
    int32_t img[3], bnd[3];
    const int rc = density_map_extent(w->params, cell_size, img, bnd);
    if (rc) return rc;
    for (int a = 0; a < 3; a++) dims[a] = (uint32_t)img[a];
    return PFS_OK;
}

// Light volume extent: (int)ceil((maxXYZ - minXYZ) * (1 / lightMarchStepSize))
// in float (renderer.c:812-819).
static int light_volume_extent(const pfs_params& p, float step, int32_t dims[3]) {
    if (!(step > 0.0f) || !std::isfinite(step)) return PFS_EINVAL;
    const float inv = 1.0f / step;
    uint64_t voxels = 1;
    for (int a = 0; a < 3; a++) {
        const double d = std::ceil((double)((p.box_max[a] - p.box_min[a]) * inv));
        if (!(d >= 0.0) || d > 65536.0) return PFS_ERANGE;
        dims[a] = (int32_t)d;
        voxels *= (uint64_t)dims[a];
    }
    return voxels > (1ull << 31) ? PFS_ERANGE : PFS_OK;
}

int pfs_world_light_volume_dims(const pfs_world* w, float light_step_size, uint32_t dims[3]) {
    if (!w || !dims) return PFS_EINVAL;
    int32_t d[3];
    const int rc = light_volume_extent(w->params, light_step_size, d);
    if (rc) return rc;
    for (int a = 0; a < 3; a++) dims[a] = (uint32_t)d[a];
    return PFS_OK;
}

static bool is_device_ptr(const void* p) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Grow a world-owned device buffer to hold `floats` (waits for the stream).
static int grow(pfs_world* w, float** buf, size_t* cap, size_t floats) {
    if (*cap >= floats) return PFS_OK;
    int rc = wait_stream(w, 0);
    if (rc) return rc;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(buf, floats * sizeof(float));
    if (e != cudaSuccess) return status_from_cuda(e);
    *cap = floats;
    return PFS_OK;
}

int pfs_world_render_volumetric(pfs_world* w, const pfs_volume_view* v, uint32_t width,
                                uint32_t height, float* rgba, float* light_volume) {
    if (!w || !v || !rgba || width == 0 || height == 0) return PFS_EINVAL;
    if ((uint64_t)width * height > (1ull << 28)) return PFS_ERANGE;
    for (int a = 0; a < 3; a++)
        if (!std::isfinite(v->position[a]) || !std::isfinite(v->forward[a]) ||
            !std::isfinite(v->right[a]) || !std::isfinite(v->up[a]) || !std::isfinite(v->extinction[a]) ||
            !std::isfinite(v->dir_to_sun[a]))
            return PFS_EINVAL;
    if (!(v->step_size > 0.0f) || !std::isfinite(v->fov)) return PFS_EINVAL;
    const float el = sqrtf(v->extinction[0] * v->extinction[0] + v->extinction[1] * v->extinction[1] +
                           v->extinction[2] * v->extinction[2]);
    if (!(el > 0.0f)) return PFS_EINVAL;
    int32_t img[3], bnd[3], ld[3];
    int rc = density_map_extent(w->params, v->density_cell_size, img, bnd);
    if (rc) return rc;
    if ((rc = light_volume_extent(w->params, v->light_step_size, ld))) return rc;
    if (!w->sorted_valid) return PFS_EINVAL;  // the map needs the table of a step's sort
    if ((rc = set_device(w))) return rc;
    const size_t nd = (size_t)img[0] * img[1] * img[2], nl = (size_t)ld[0] * ld[1] * ld[2];
    if (nd == 0 || nl == 0) return PFS_EINVAL;  // the samplers need a non-empty grid
    const size_t npx = (size_t)width * height * 4;
    const bool dev_out = is_device_ptr(rgba);
    if ((rc = grow(w, &w->map_buf, &w->map_cap, std::max<size_t>(nd, 1)))) return rc;
    if ((rc = grow(w, &w->lv_buf, &w->lv_cap, std::max<size_t>(nl, 1) + (dev_out ? 0 : npx)))) return rc;
    float* lvol = w->lv_buf;
    float* img_dev = dev_out ? rgba : w->lv_buf + std::max<size_t>(nl, 1);
    // the camera constants the shader computes per pixel from uniforms
    const float half_h = tanf(0.5f * v->fov);
    const float half_w = half_h * (float)width / (float)height;
    float ext[3];
    for (int a = 0; a < 3; a++) ext[a] = 1.0f * (v->extinction[a] / el);
    float cam[12];
    for (int a = 0; a < 3; a++) {
        cam[a] = v->position[a];
        cam[3 + a] = v->forward[a];
        cam[6 + a] = v->right[a];
        cam[9 + a] = v->up[a];
    }
    cudaError_t e = nd ? launch_density_map(w->dp, w->b, v->density_cell_size, img, bnd, w->map_buf, w->stream)
                       : cudaSuccess;
    if (e == cudaSuccess && nl)
        e = launch_light_volume(w->dp, w->map_buf, img, v->light_step_size, v->dir_to_sun, ld, lvol,
                                w->stream);
    if (e == cudaSuccess)
        e = launch_volumetric(w->dp, w->map_buf, img, lvol, ld, cam, half_h, half_w, v->step_size, ext,
                              width, height, img_dev, w->stream);
    if (e == cudaSuccess && !dev_out)
        e = cudaMemcpyAsync(rgba, img_dev, npx * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess && light_volume && nl)
        e = cudaMemcpyAsync(light_volume, lvol, nl * sizeof(float), cudaMemcpyDefault, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    return check_err_word(w);
}

int pfs_world_render_refractive(pfs_world* w, const pfs_volume_view* v, const pfs_refraction* r,
                                uint32_t width, uint32_t height, float* rgba) {
    if (!w || !v || !r || !rgba || width == 0 || height == 0) return PFS_EINVAL;
    if ((uint64_t)width * height > (1ull << 28)) return PFS_ERANGE;
    for (int a = 0; a < 3; a++)
        if (!std::isfinite(v->position[a]) || !std::isfinite(v->forward[a]) ||
            !std::isfinite(v->right[a]) || !std::isfinite(v->up[a]) || !std::isfinite(v->extinction[a]))
            return PFS_EINVAL;
    if (!(v->step_size > 0.0f) || !(v->light_step_size > 0.0f) || !std::isfinite(v->fov)) return PFS_EINVAL;
    if (r->num_refractions < 0 || r->num_refractions > 64 || !std::isfinite(r->surface_density_threshold) ||
        !(r->index_of_refraction > 0.0f) || !std::isfinite(r->index_of_refraction))
        return PFS_EINVAL;
    int32_t img[3], bnd[3];
    int rc = density_map_extent(w->params, v->density_cell_size, img, bnd);
    if (rc) return rc;
    if (!w->sorted_valid) return PFS_EINVAL;  // the map needs the table of a step's sort
    if ((rc = set_device(w))) return rc;
    const size_t nd = (size_t)img[0] * img[1] * img[2];
    if (nd == 0) return PFS_EINVAL;  // the sampler needs a non-empty grid
    const size_t npx = (size_t)width * height * 4;
    const bool dev_out = is_device_ptr(rgba);
    if ((rc = grow(w, &w->map_buf, &w->map_cap, nd))) return rc;
    if (!dev_out && (rc = grow(w, &w->lv_buf, &w->lv_cap, npx))) return rc;
    float* img_dev = dev_out ? rgba : w->lv_buf;
    // the camera constants the shader computes per pixel from uniforms
    const float half_h = tanf(0.5f * v->fov);
    const float half_w = half_h * (float)width / (float)height;
    float cam[12];
    for (int a = 0; a < 3; a++) {
        cam[a] = v->position[a];
        cam[3 + a] = v->forward[a];
        cam[6 + a] = v->right[a];
        cam[9 + a] = v->up[a];
    }
    cudaError_t e = launch_density_map(w->dp, w->b, v->density_cell_size, img, bnd, w->map_buf, w->stream);
    if (e == cudaSuccess)
        e = launch_refractive(w->dp, w->map_buf, img, cam, half_h, half_w, v->step_size, v->light_step_size,
                              v->extinction, r->num_refractions, r->surface_density_threshold,
                              r->index_of_refraction, width, height, img_dev, w->stream);
    if (e == cudaSuccess && !dev_out)
        e = cudaMemcpyAsync(rgba, img_dev, npx * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    return check_err_word(w);
}

// mvp = (proj * view) * model and the camera's right / up (the first two
// rows of view's rotation), as the oracle's pfso_splat_camera computes them.
static void splat_camera(const pfs_splat_view* v, float mvp[16], float right[3], float up[3]) {
    float pv[16];
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++)
            pv[c * 4 + r] = v->proj[0 * 4 + r] * v->view[c * 4 + 0] + v->proj[1 * 4 + r] * v->view[c * 4 + 1] +
                            v->proj[2 * 4 + r] * v->view[c * 4 + 2] + v->proj[3 * 4 + r] * v->view[c * 4 + 3];
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++)
            mvp[c * 4 + r] = pv[0 * 4 + r] * v->model[c * 4 + 0] + pv[1 * 4 + r] * v->model[c * 4 + 1] +
                             pv[2 * 4 + r] * v->model[c * 4 + 2] + pv[3 * 4 + r] * v->model[c * 4 + 3];
    for (int a = 0; a < 3; a++) {
        right[a] = v->view[a * 4 + 0];
        up[a] = v->view[a * 4 + 1];
    }
}

int pfs_world_render_splats(pfs_world* w, const pfs_splat_view* v, uint32_t width, uint32_t height,
                            float* rgba, float* depth) {
    if (!w || !v || !rgba || width == 0 || height == 0) return PFS_EINVAL;
    if ((uint64_t)width * height > (1ull << 28)) return PFS_ERANGE;
    if (!w->b.color) return PFS_EINVAL;  // the splats take the speed colour ramp
    for (int k = 0; k < 16; k++)
        if (!std::isfinite(v->model[k]) || !std::isfinite(v->view[k]) || !std::isfinite(v->proj[k]))
            return PFS_EINVAL;
    if (!(v->particle_radius >= 0.0f) || !std::isfinite(v->particle_radius)) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    const size_t npx = (size_t)width * height;
    const bool dev_rgba = is_device_ptr(rgba), dev_depth = depth && is_device_ptr(depth);
    const size_t need = 2 * npx + (dev_rgba ? 0 : 4 * npx) + (depth && !dev_depth ? npx : 0);
    if ((rc = grow(w, &w->lv_buf, &w->lv_cap, need))) return rc;
    auto* keys = reinterpret_cast<unsigned long long*>(w->lv_buf);
    float* img = dev_rgba ? rgba : w->lv_buf + 2 * npx;
    float* dep = depth ? (dev_depth ? depth : w->lv_buf + 2 * npx + (dev_rgba ? 0 : 4 * npx)) : nullptr;
    float mvp[16], right[3], up[3];
    splat_camera(v, mvp, right, up);
    cudaError_t e = launch_splats(w->n, w->b.x, w->b.color, mvp, right, up, v->particle_radius, width, height,
                                  keys, img, dep, w->b.err, w->stream);
    if (e == cudaSuccess && !dev_rgba)
        e = cudaMemcpyAsync(rgba, img, 4 * npx * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess && depth && !dev_depth)
        e = cudaMemcpyAsync(depth, dep, npx * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    return check_err_word(w);
}

int pfs_world_fxaa(pfs_world* w, const float* rgba_in, uint32_t width, uint32_t height, float* rgba_out) {
    if (!w || !rgba_in || !rgba_out || width == 0 || height == 0 || rgba_in == rgba_out) return PFS_EINVAL;
    if ((uint64_t)width * height > (1ull << 28)) return PFS_ERANGE;
    int rc = set_device(w);
    if (rc) return rc;
    const size_t n4 = (size_t)width * height * 4;
    const bool dev_in = is_device_ptr(rgba_in), dev_out = is_device_ptr(rgba_out);
    const size_t need = (dev_in ? 0 : n4) + (dev_out ? 0 : n4);
    if (need && (rc = grow(w, &w->lv_buf, &w->lv_cap, need))) return rc;
    const float* src = rgba_in;
    float* dst = dev_out ? rgba_out : w->lv_buf + (dev_in ? 0 : n4);
    cudaError_t e = cudaSuccess;
    if (!dev_in) {
        e = cudaMemcpyAsync(w->lv_buf, rgba_in, n4 * sizeof(float), cudaMemcpyHostToDevice, w->stream);
        src = w->lv_buf;
    }
    if (e == cudaSuccess) e = launch_fxaa(src, width, height, dst, w->stream);
    if (e == cudaSuccess && !dev_out)
        e = cudaMemcpyAsync(rgba_out, dst, n4 * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    return e == cudaSuccess ? PFS_OK : status_from_cuda(e);
}

int pfs_world_density_map(pfs_world* w, float cell_size, float* out) {
    if (!w || !out) return PFS_EINVAL;
    int32_t img[3], bnd[3];
    int rc = density_map_extent(w->params, cell_size, img, bnd);
    if (rc) return rc;
    if (!w->sorted_valid) return PFS_EINVAL;  // the map needs the table of a step's sort
    if ((rc = set_device(w))) return rc;
    const size_t voxels = (size_t)img[0] * (size_t)img[1] * (size_t)img[2];
    if (voxels == 0) return PFS_OK;
    cudaPointerAttributes attr{};
    bool on_device = false;
    if (cudaPointerGetAttributes(&attr, out) == cudaSuccess)
        on_device = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
    else
        cudaGetLastError();
    float* dst = out;
    if (!on_device) {
        if (w->map_cap < voxels) {
            if ((rc = wait_stream(w, 0))) return rc;
            if (w->map_buf) cudaFree(w->map_buf);
            w->map_buf = nullptr;
            w->map_cap = 0;
            cudaError_t e = cudaMalloc(&w->map_buf, voxels * sizeof(float));
            if (e != cudaSuccess) return status_from_cuda(e);
            w->map_cap = voxels;
        }
        dst = w->map_buf;
    }
    cudaError_t e = launch_density_map(w->dp, w->b, cell_size, img, bnd, dst, w->stream);
    if (e == cudaSuccess && !on_device)
        e = cudaMemcpyAsync(out, dst, voxels * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    if (e != cudaSuccess) return status_from_cuda(e);
    return check_err_word(w);
}

uint32_t pfs_world_size(const pfs_world* w) { return w ? w->n : 0u; }

void* pfs_world_stream(pfs_world* w) { return w ? (void*)w->stream : nullptr; }

int pfs_world_device_state(pfs_world* w, void** pos4_dev, void** vel4_dev) {
    if (!w) return PFS_EINVAL;
    if (pos4_dev) *pos4_dev = w->b.x;
    if (vel4_dev) *vel4_dev = w->b.v;
    return PFS_OK;
}

int pfs_world_profile(pfs_world* w, int enable) {
    if (!w) return PFS_EINVAL;
    w->profiling = enable != 0;
    return PFS_OK;
}

int pfs_world_stage_times(pfs_world* w, pfs_stage_times* out) {
    if (!w || !out) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    if ((rc = wait_stream(w, 0))) return rc;
    const size_t per = PFS_STAGE_COUNT + 1;
    for (size_t s = 0; s + per <= w->pending.size(); s += per) {
        for (int k = 0; k < PFS_STAGE_COUNT; k++) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, w->pending[s + k], w->pending[s + k + 1]);
            w->times.ms_total[k] += ms;
        }
        const int sort_l = sort_launches(w->n);
        w->times.launches[PFS_STAGE_SORT] += sort_l;
        for (int k = 1; k < PFS_STAGE_COUNT; k++) w->times.launches[k] += 1;
        w->times.substeps += 1;
    }
    for (auto e : w->pending) cudaEventDestroy(e);
    w->pending.clear();
    *out = w->times;
    std::memset(&w->times, 0, sizeof(w->times));
    return PFS_OK;
}

int pfs_world_launches_per_substep(const pfs_world* w) {
    return w ? substep_launches(w->n, w->dp.geo != 0) : 0;
}

int pfs_world_debug_substep(pfs_world* w, pfs_debug_substep* o) {
    if (!w || !o) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    const uint32_t n = w->n;
    const size_t f4 = (size_t)n * 16, u = (size_t)n * 4;
    const DevParams& P = w->dp;
    cudaStream_t s = w->stream;
    auto d2h = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
        if (!dst) return cudaSuccess;
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    };
    cudaError_t e = d2h(o->keys_in, w->b.keys, u);
    if (e == cudaSuccess) e = launch_sort(P, w->b, s);
    if (e == cudaSuccess) e = d2h(o->keys, w->b.skeys, u);
    if (e == cudaSuccess) e = d2h(o->perm, w->b.perm, u);
    const bool fp16 = w->params.precision == PFS_FP16_CELL;
    if (e == cudaSuccess) e = fp16 ? launch_reorder_fp16(P, w->b, w->h16, s) : launch_reorder(P, w->b, s);
    if (e == cudaSuccess && (o->start || o->end)) {
        std::vector<int32_t> t((size_t)n * 2);
        e = d2h(t.data(), w->b.table, (size_t)n * 8);
        for (uint32_t k = 0; k < n && e == cudaSuccess; k++) {
            if (o->start) o->start[k] = t[2 * (size_t)k];
            if (o->end) o->end[k] = t[2 * (size_t)k + 1];
        }
    }
    if (e == cudaSuccess) e = d2h(o->xp, w->b.xp, f4);
    if (e == cudaSuccess) e = d2h(o->vp, w->b.vp, f4);
    if (e == cudaSuccess) e = fp16 ? launch_density_fp16(P, w->b, w->h16, s) : launch_density(P, w->b, s);
    if (e == cudaSuccess && (o->density || o->near_density)) {
        std::vector<float> t((size_t)n * 2);
        e = d2h(t.data(), w->b.rr, (size_t)n * 8);
        for (uint32_t k = 0; k < n && e == cudaSuccess; k++) {
            if (o->density) o->density[k] = t[2 * (size_t)k];
            if (o->near_density) o->near_density[k] = t[2 * (size_t)k + 1];
        }
    }
    if (e == cudaSuccess) e = fp16 ? launch_force_fp16(P, w->b, w->h16, s) : launch_force(P, w->b, s);
    if (e == cudaSuccess) e = d2h(o->vel_force, w->b.v, f4);
    if (e == cudaSuccess) e = launch_integrate(P, w->b, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return status_from_cuda(e);
    w->sorted_valid = true;
    return check_err_word(w);
}

// Kernel shape and neighbour search of a world: re-derive the parameters
// with the search, refit the spatial blocks to the arena, drop the graph.
static int apply_shape(pfs_world* w, int32_t shape, int32_t search) {
    if (shape < NBR_SIMPLE || shape > NBR_STAGED || search < -1 || search > 1) return PFS_EINVAL;
    if (search == 1 && !grid_search_allowed(w->params, w->n)) return PFS_EINVAL;
    if (shape == NBR_STAGED) {
        // the staged passes scan table ranges (no grid search); they need a
        // block shape whose fine buckets fit the world's counters
        if (!w->staged_ok || search == 1) return PFS_EINVAL;
        search = 0;
    }
    w->b.variant = shape;
    w->search = search;
    derive_params(w->params, w->n, &w->dp, search);
    w->dp.list_cap = w->list_cap;
    if (shape == NBR_STAGED) {
        const DevParams& c = w->staged_cfg;
        w->dp.staged = 1;
        w->dp.sbx = c.sbx;
        w->dp.sby = c.sby;
        w->dp.sbz = c.sbz;
        w->dp.nsx = c.nsx;
        w->dp.nsy = c.nsy;
        w->dp.nsz = c.nsz;
        w->b.nblocks = (uint32_t)staged_buckets(w->dp);
    } else {
        fit_spatial_blocks(&w->dp, w->blocks_cap);
        w->b.nblocks = spatial_blocks(w->dp);
    }
    w->b.geo_any = w->dp.geo;
    drop_graph(w);
    return PFS_OK;
}

int pfs_world_shape_available(const pfs_world* w, int32_t shape) {
    if (!w || shape < NBR_SIMPLE || shape > NBR_STAGED) return 0;
    return shape == NBR_STAGED ? (w->staged_ok ? 1 : 0) : 1;
}

int pfs_world_set_shape(pfs_world* w, int32_t shape, int32_t search) {
    if (!w) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    if ((rc = wait_stream(w, 0))) return rc;
    return apply_shape(w, shape, search);
}

int pfs_world_autotune(pfs_world* w, uint32_t trial_steps, pfs_tune_result* out) {
    if (!w || !out) return PFS_EINVAL;
    std::memset(out, 0, sizeof(*out));
    int rc = set_device(w);
    if (rc) return rc;
    if ((rc = wait_stream(w, 0))) return rc;
    if (trial_steps == 0) trial_steps = 2;
    const int32_t keep_shape = w->b.variant, keep_search = w->search;
    // candidates: every shape the form has, with each search it allows
    std::vector<std::pair<int32_t, int32_t>> cand;
    const bool fp16 = w->params.precision == PFS_FP16_CELL;
    const bool grid = grid_search_allowed(w->params, w->n);
    for (int32_t shape : {NBR_STAGED, NBR_LIST, NBR_FLAT, NBR_COMPACT, NBR_SIMPLE}) {
        if (fp16 && shape != NBR_LIST) continue;  // one shape in the FP16-cell form
        if (shape == NBR_STAGED) {
            if (w->staged_ok) cand.push_back({shape, 0});  // table scan only
            continue;
        }
        cand.push_back({shape, 0});
        if (grid) cand.push_back({shape, 1});
    }
    // the state every trial starts from, restored at the end
    const size_t f4 = (size_t)w->n * 16, u = (size_t)w->n * 4;
    char* snap = nullptr;
    const size_t snap_bytes = 2 * f4 + 2 * u + (w->b.ids ? u : 0);
    cudaError_t e = cudaMalloc(&snap, snap_bytes);
    if (e != cudaSuccess) return status_from_cuda(e);
    auto copy_state = [&](bool save) -> cudaError_t {
        char* q = snap;
        auto one = [&](void* dev, size_t bytes) -> cudaError_t {
            cudaError_t r = save ? cudaMemcpyAsync(q, dev, bytes, cudaMemcpyDeviceToDevice, w->stream)
                                 : cudaMemcpyAsync(dev, q, bytes, cudaMemcpyDeviceToDevice, w->stream);
            q += bytes;
            return r;
        };
        cudaError_t r = one(w->b.x, f4);
        if (r == cudaSuccess) r = one(w->b.v, f4);
        if (r == cudaSuccess) r = one(w->b.skeys, u);
        if (r == cudaSuccess) r = one(w->b.perm, u);
        if (r == cudaSuccess && w->b.ids) r = one(w->b.ids, u);
        if (r == cudaSuccess && !save) r = launch_keys(w->dp, w->b, w->stream);
        return r;
    };
    const bool keep_sorted = w->sorted_valid;
    e = copy_state(true);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best = INFINITY;
    int32_t chosen = -1;
    for (size_t k = 0; k < cand.size() && k < PFS_TUNE_MAX && e == cudaSuccess; k++) {
        if ((rc = apply_shape(w, cand[k].first, cand[k].second))) break;
        if ((e = copy_state(false)) != cudaSuccess) break;
        if ((rc = pfs_world_step(w, 1))) break;  // captures the graph, warms caches
        // trial_steps single steps, each from the saved state; the fastest
        // counts (steps differ by a few percent between shapes, about the
        // noise of one timing)
        float ms = INFINITY;
        for (uint32_t r = 0; r < trial_steps; r++) {
            if ((e = copy_state(false)) != cudaSuccess) break;
            if ((e = cudaEventRecord(e0, w->stream)) != cudaSuccess) break;
            if ((rc = pfs_world_step(w, 1))) break;
            if ((e = cudaEventRecord(e1, w->stream)) != cudaSuccess) break;
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
            float one = 0.0f;
            cudaEventElapsedTime(&one, e0, e1);
            ms = std::min(ms, one);
        }
        if (rc || e != cudaSuccess) break;
        out->shape[out->candidates] = cand[k].first;
        out->search[out->candidates] = cand[k].second;
        out->ms_per_step[out->candidates] = ms;
        if (ms < best) {
            best = ms;
            chosen = out->candidates;
        }
        out->candidates++;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    // keep the fastest (or the previous choice if a trial failed), restore the state
    const int rc2 = chosen >= 0 && rc == PFS_OK && e == cudaSuccess
                        ? apply_shape(w, out->shape[chosen], out->search[chosen])
                        : apply_shape(w, keep_shape, keep_search);
    out->chosen = (rc == PFS_OK && e == cudaSuccess) ? chosen : -1;
    cudaError_t e2 = copy_state(false);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(w->stream);
    cudaFree(snap);
    w->sorted_valid = keep_sorted;
    if (rc) return rc;
    if (e != cudaSuccess) return status_from_cuda(e);
    if (rc2) return rc2;
    if (e2 != cudaSuccess) return status_from_cuda(e2);
    return check_err_word(w);
}

int pfs_world_device_error(pfs_world* w, uint32_t* word) {
    if (!w || !word) return PFS_EINVAL;
    int rc = set_device(w);
    if (rc) return rc;
    if ((rc = wait_stream(w, 0))) return rc;
    cudaError_t e = cudaMemcpy(word, w->err, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(w->err, 0, 4);
    return status_from_cuda(e);
}

}  // extern "C"
