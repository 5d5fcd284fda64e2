// pfs_fp16.cu — FP16-cell neighbour passes (bandwidth form).
//
// Same neighbour enumeration as the FP32 form (calculateDensities.comp:114-131,
// applyPressureAndViscosityForce.comp:134-171): the 27 cell keys are taken
// from the FP32 x* exactly as the reference takes them, only the candidate
// data is compressed.  Arithmetic here may use FMA (explicit fmaf).
#include <cmath>
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_fp16.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int ELEM_THREADS = 256;
constexpr int NBR_THREADS = 128;

__device__ __forceinline__ uint32_t pack_cell(int32_t cx, int32_t cy, int32_t cz) {
    return ((uint32_t)(cx + 1) & 1023u) | (((uint32_t)(cy + 1) & 1023u) << 10) |
           (((uint32_t)(cz + 1) & 1023u) << 20);
}

__device__ __forceinline__ float sat_half_range(float x) {
    return fminf(fmaxf(x, -65504.0f), 65504.0f);
}

__device__ __forceinline__ uint32_t h2u(float a, float b) {
    const __half2 v = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float2 u2f(uint32_t u) {
    __half2 v;
    *reinterpret_cast<uint32_t*>(&v) = u;
    return __half22float2(v);
}

struct Unpacked {
    float px, py, pz;  // position in units of h, cell + offset
    float vx, vy, vz;  // velocity in units of h/dt
};

__device__ __forceinline__ Unpacked unpack(const uint4 r) {
    Unpacked u;
    const float2 a = u2f(r.y), b = u2f(r.z), c = u2f(r.w);
    u.px = (float)((int32_t)(r.x & 1023u) - 1) + a.x;
    u.py = (float)((int32_t)((r.x >> 10) & 1023u) - 1) + a.y;
    u.pz = (float)((int32_t)((r.x >> 20) & 1023u) - 1) + b.x;
    u.vx = b.y;
    u.vy = c.x;
    u.vz = c.y;
    return u;
}

__device__ __forceinline__ uint4 make_record(const DevParams& P, float3 pos, float4 vel) {
    const float tx = (pos.x - P.minx) / P.h, ty = (pos.y - P.miny) / P.h, tz = (pos.z - P.minz) / P.h;
    const float fx = floorf(tx), fy = floorf(ty), fz = floorf(tz);
    const float vscale = P.dt / P.h;
    uint4 r;
    r.x = pack_cell((int32_t)fx, (int32_t)fy, (int32_t)fz);
    r.y = h2u(tx - fx, ty - fy);
    r.z = h2u(tz - fz, sat_half_range(vel.x * vscale));
    r.w = h2u(sat_half_range(vel.y * vscale), sat_half_range(vel.z * vscale));
    return r;
}

// k_reorder of the FP32 form plus the 16-byte neighbour record of x* and v.
template <bool BATCH>
__global__ void __launch_bounds__(ELEM_THREADS)
k_reorder_fp16(DevParams P0, SceneRef sr, const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ perm,
               const float4* __restrict__ x, const float4* __restrict__ v,
               const uint32_t* __restrict__ ids, float4* __restrict__ xs, float4* __restrict__ vs,
               float4* __restrict__ xp, float4* __restrict__ vp, uint32_t* __restrict__ ids_s,
               int2* __restrict__ table, uint4* __restrict__ rec, uint32_t* __restrict__ err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = P0.n;
    if (s >= n) return;
    const DevParams P = params_of<BATCH>(P0, sr, s);
    const uint32_t p = perm[s];
    const uint32_t k = skeys[s];
    if (p >= n || k >= n) {
        atomicOr(err, p >= n ? ERR_PERM_RANGE : ERR_KEY_RANGE);
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
    rec[s] = make_record(P, pos, vo);
    if (ids) ids_s[s] = ids[p];
    const bool head = (s == 0) || (skeys[s - 1] != k);
    const bool tail = (s == n - 1) || (skeys[s + 1] != k);
    if (head) table[k].x = (int32_t)s;
    if (tail) table[k].y = (int32_t)(s + 1);
}

__device__ __forceinline__ uint32_t pick3(int i, uint32_t a, uint32_t b, uint32_t c) {
    return i == 0 ? a : (i == 1 ? b : c);
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS)
k_density_fp16(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const uint4* __restrict__ rec,
               const int2* __restrict__ table, float2* __restrict__ rr,
               uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P0.n) return;
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 sp = xp[i];
    const Unpacked me = unpack(rec[i]);
    const float h = P.h, m = P.m;
    const float off0 = PFS_MUL(h, -1.0f), off1 = PFS_MUL(h, 0.0f), off2 = h;
    uint32_t hx[3], hy[3], hz[3];
    bool vx[3], vy[3], vz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float o = a == 0 ? off0 : (a == 1 ? off1 : off2);
        const float sx = PFS_ADD(sp.x, o), sy = PFS_ADD(sp.y, o), sz = PFS_ADD(sp.z, o);
        vx[a] = !(sx < P.minx) && !(sx > P.maxx);
        vy[a] = !(sy < P.miny) && !(sy > P.maxy);
        vz[a] = !(sz < P.minz) && !(sz > P.maxz);
        hx[a] = (uint32_t)cell_coord(sx, P.minx, h) * 73856093u;
        hy[a] = (uint32_t)cell_coord(sy, P.miny, h) * 19349663u;
        hz[a] = (uint32_t)cell_coord(sz, P.minz, h) * 83492791u;
    }
    // compensated (Kahan) sums in units of h: sum (1 - d/h)^2 and ^3
    float s2 = 0.0f, c2 = 0.0f, s3 = 0.0f, c3 = 0.0f;
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const bool ok = (dx == 0 ? vx[0] : dx == 1 ? vx[1] : vx[2]) &&
                        (dy == 0 ? vy[0] : dy == 1 ? vy[1] : vy[2]) &&
                        (dz == 0 ? vz[0] : dz == 1 ? vz[1] : vz[2]);
        if (!ok) continue;
        const uint32_t key = slot_of(P, hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                                      pick3(dy, hy[0], hy[1], hy[2]) ^
                                                      pick3(dz, hz[0], hz[1], hz[2])));
        const int2 se = __ldg(table + key);
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)P.n || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            const Unpacked o = unpack(__ldg(rec + j));
            const float ex = o.px - me.px, ey = o.py - me.py, ez = o.pz - me.pz;
            const float q2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            if (q2 >= 1.0f) continue;
            const float a = 1.0f - sqrtf(q2);
            const float a2 = a * a;
            float y = a2 - c2;
            float t = s2 + y;
            c2 = (t - s2) - y;
            s2 = t;
            y = a2 * a - c3;
            t = s3 + y;
            c3 = (t - s3) - y;
            s3 = t;
        }
    }
    const float h2 = h * h;
    const float d = (m * (s2 * h2)) / P.volume;
    const float nd = (m * (s3 * h2 * h)) * P.near_inv;
    rr[i] = make_float2((0.01f < d) ? d : 0.01f, (0.01f < nd) ? nd : 0.01f);
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS)
k_force_fp16(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
             const float4* __restrict__ vs, const uint4* __restrict__ rec,
             const float2* __restrict__ rr, const int2* __restrict__ table,
             float4* __restrict__ vout, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P0.n) return;
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 sp = xp[i];
    const float4 pv = vp[i];
    const float2 rri = rr[i];
    const Unpacked me = unpack(rec[i]);
    const float h = P.h, m = P.m, rho0 = P.rho0, k = P.k, kn = P.kn;
    const float vunit = P.h / P.dt;
    const bool inside = !(sp.x < P.minx) && !(sp.y < P.miny) && !(sp.z < P.minz) &&
                        !(sp.x > P.maxx) && !(sp.y > P.maxy) && !(sp.z > P.maxz);
    const int32_t cx = inside ? cell_coord(sp.x, P.minx, h) : -1;
    const int32_t cy = inside ? cell_coord(sp.y, P.miny, h) : -1;
    const int32_t cz = inside ? cell_coord(sp.z, P.minz, h) : -1;
    uint32_t hx[3], hy[3], hz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        hx[a] = ((uint32_t)cx + (uint32_t)(a - 1)) * 73856093u;
        hy[a] = ((uint32_t)cy + (uint32_t)(a - 1)) * 19349663u;
        hz[a] = ((uint32_t)cz + (uint32_t)(a - 1)) * 83492791u;
    }
    const float my_density = rri.x;
    const float my_p = (my_density - rho0) * k;
    const float near_p = rri.y * kn;
    // pressure kernel derivative (d - h) * slope_scale written in units of h
    const float slope_h = h * P.slope_scale;
    const float nslope_h2 = h * h * P.near_slope_scale;
    const float h2m = h * h * m;
    const float pvx = pv.x / vunit, pvy = pv.y / vunit, pvz = pv.z / vunit;
    float fpx = 0.0f, fpy = 0.0f, fpz = 0.0f, fvx = 0.0f, fvy = 0.0f, fvz = 0.0f;
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const uint32_t key = slot_of(P, hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                                      pick3(dy, hy[0], hy[1], hy[2]) ^
                                                      pick3(dz, hz[0], hz[1], hz[2])));
        const int2 se = __ldg(table + key);
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)P.n || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            if (j == (int32_t)i) continue;
            const Unpacked o = unpack(__ldg(rec + j));
            const float ex = o.px - me.px, ey = o.py - me.py, ez = o.pz - me.pz;
            const float q2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
            if (q2 >= 1.0f) continue;
            const float q = sqrtf(q2);
            if (q * h < 1e-7f) continue;
            const float inv_q = 1.0f / q;
            const float2 rrj = __ldg(rr + j);
            const float dj = rrj.x, nnd = rrj.y;
            const float a = 1.0f - q;
            const float shared = 0.5f * ((dj - rho0) * k + my_p);
            const float coef = shared * (-a * slope_h) * m / dj;
            const float shared_near = 0.5f * (near_p + nnd * kn);
            const float ncoef = shared_near * (a * a * nslope_h2) * m / nnd;
            const float pc = (coef + ncoef) * inv_q;
            fpx = fmaf(pc, ex, fpx);
            fpy = fmaf(pc, ey, fpy);
            fpz = fmaf(pc, ez, fpz);
            const float vcoef = h2m * a * a / dj;
            fvx = fmaf(vcoef, o.vx - pvx, fvx);
            fvy = fmaf(vcoef, o.vy - pvy, fvy);
            fvz = fmaf(vcoef, o.vz - pvz, fvz);
        }
    }
    const float4 vi = vs[i];
    const float sv = P.visc * vunit;
    const float tx = fpx + sv * fvx, ty = fpy + sv * fvy, tz = fpz + sv * fvz;
    const float g = P.dt / my_density;
    vout[i] = make_float4(vi.x + tx * g, vi.y + ty * g, vi.z + tz * g, vi.w + 1.0f);
}

inline unsigned grid_for(uint32_t n, int threads) { return (n + threads - 1) / threads; }

}  // namespace

size_t fp16_arena_bytes(uint32_t n) { return (size_t)n * 16 + 256; }

bool fp16_carve(Arena& a, uint32_t n, Fp16Buffers* out) {
    out->rec = (uint4*)a.take((size_t)n * 16);
    return out->rec != nullptr;
}

int fp16_check_box(const pfs_params& p) {
    if (!(p.dt > 0.0f)) return PFS_EINVAL;
    for (int a = 0; a < 3; a++) {
        const double cells = ((double)p.box_max[a] - (double)p.box_min[a]) / (double)p.h;
        if (!(cells < (double)FP16_MAX_CELLS)) return PFS_EINVAL;
    }
    return PFS_OK;
}

cudaError_t launch_reorder_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                                cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, ELEM_THREADS);
    if (b.sr.scenes)
        k_reorder_fp16<true><<<g, ELEM_THREADS, 0, s>>>(P, b.sr, b.skeys, b.perm, b.x, b.v, b.ids,
                                                        b.xs, b.vs, b.xp, b.vp, b.ids_s, b.table,
                                                        f.rec, b.err);
    else
        k_reorder_fp16<false><<<g, ELEM_THREADS, 0, s>>>(
        P, b.sr, b.skeys, b.perm, b.x, b.v, b.ids, b.xs, b.vs, b.xp, b.vp, b.ids_s, b.table, f.rec, b.err);
    return cudaGetLastError();
}

cudaError_t launch_density_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                                cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, NBR_THREADS);
    if (b.sr.scenes)
        k_density_fp16<true><<<g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, f.rec, b.table, b.rr, b.err);
    else
        k_density_fp16<false><<<g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, f.rec, b.table, b.rr, b.err);
    return cudaGetLastError();
}

cudaError_t launch_force_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                              cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, NBR_THREADS);
    if (b.sr.scenes)
        k_force_fp16<true><<<g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, f.rec, b.rr, b.table,
                                                     b.v, b.err);
    else
        k_force_fp16<false><<<g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, f.rec, b.rr,
                                                      b.table, b.v, b.err);
    return cudaGetLastError();
}

}  // namespace pfs
