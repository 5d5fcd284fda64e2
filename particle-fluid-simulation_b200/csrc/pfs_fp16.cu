// pfs_fp16.cu — FP16-cell neighbour passes (bandwidth form).
//
// Same neighbour enumeration as the FP32 form (calculateDensities.comp:114-131,
// applyPressureAndViscosityForce.comp:134-171): the 27 cell keys come from
// the FP32 x* exactly as the reference takes them; only the candidate data
// is the 16-byte record (pfs_record.cuh) the reorder writes, so a density
// candidate costs 16 bytes and a force neighbour 16 + 8 instead of 16 + 16 + 8.
// Distances are taken in units of h from the records (cell difference plus
// FP16 offsets), accumulation is FP32 (the density sums compensated), and
// the processing order, density-built neighbour lists, full-scan queue and
// grid search are the FP32 form's (pfs_neighbors.cu, pfs_geo.cuh).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_flat.cuh"
#include "pfs_fp16.cuh"
#include "pfs_geo.cuh"
#include "pfs_record.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int NBR_THREADS = 128;

__device__ __forceinline__ uint32_t pick3(int i, uint32_t a, uint32_t b, uint32_t c) {
    return i == 0 ? a : (i == 1 ? b : c);
}
__device__ __forceinline__ bool pickb(int i, bool a, bool b, bool c) {
    return i == 0 ? a : (i == 1 ? b : c);
}

__device__ __forceinline__ float rec_q2(const Unpacked& o, const Unpacked& me, float& ex, float& ey,
                                        float& ez) {
    ex = o.px - me.px;
    ey = o.py - me.py;
    ez = o.pz - me.pz;
    return fmaf(ex, ex, fmaf(ey, ey, ez * ez));
}

// Kahan-compensated add.
__device__ __forceinline__ void kahan(float& s, float& c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// This form is held to a tolerance against FP64, not to the reference's
// bits, so its square roots and reciprocals use the hardware approximations
// (a few ulp) instead of the IEEE-exact sequences.
//
// Density and near-density terms (1 - q)^2 and (1 - q)^3 of a candidate at
// q2 = (r / h)^2 < 1 (q2 = 0 gives q = 0).  Every density pass of the form
// uses this, so the table scan and the grid search give the same bits.
__device__ __forceinline__ void dens16_terms(float q2, float& a2, float& a3) {
    const float q = q2 > 0.0f ? q2 * rsqrtf(q2) : 0.0f;
    const float a = 1.0f - q;
    a2 = a * a;
    a3 = a2 * a;
}

// ---- flat shape of the FP16-cell density pass -------------------------------
// The flat walk of pfs_flat.cuh over the 16-byte records: each thread packs
// its particle's 27 table ranges into shared memory, the block sorts its
// particles by candidate total, and each warp walks all 27 ranges in one
// loop of uniform trip count.  The candidates and
// their order are those of the 27-cell table walk (density16_scan_one), so
// the compensated sums, in that order, and the list and queue decisions are
// the same bits as a particle's own walk.
constexpr int D16_CAP = 12;  // deferred q2 per lane

// Density sums of one particle by its own 27-cell walk from global memory
// in the reference's order: the fallback of the flat shape.
__device__ __forceinline__ void density16_scan_one(const DevParams& P, const float4 sp, const Unpacked& me,
                                                   const uint4* __restrict__ rec,
                                                   const int2* __restrict__ table, uint32_t n_all,
                                                   uint32_t* __restrict__ err, float& s2, float& c2, float& s3,
                                                   float& c3) {
    const float h = P.h;
    const float off[3] = {PFS_MUL(h, -1.0f), PFS_MUL(h, 0.0f), h};
    uint32_t hx[3], hy[3], hz[3];
    bool vx[3], vy[3], vz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float sx = PFS_ADD(sp.x, off[a]), sy = PFS_ADD(sp.y, off[a]), sz = PFS_ADD(sp.z, off[a]);
        vx[a] = !(sx < P.minx) && !(sx > P.maxx);
        vy[a] = !(sy < P.miny) && !(sy > P.maxy);
        vz[a] = !(sz < P.minz) && !(sz > P.maxz);
        hx[a] = (uint32_t)cell_coord(sx, P.minx, h) * 73856093u;
        hy[a] = (uint32_t)cell_coord(sy, P.miny, h) * 19349663u;
        hz[a] = (uint32_t)cell_coord(sz, P.minz, h) * 83492791u;
    }
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        if (!(pickb(dx, vx[0], vx[1], vx[2]) && pickb(dy, vy[0], vy[1], vy[2]) &&
              pickb(dz, vz[0], vz[1], vz[2])))
            continue;
        const int2 se = __ldg(table + slot_of(P, hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                                               pick3(dy, hy[0], hy[1], hy[2]) ^
                                                               pick3(dz, hz[0], hz[1], hz[2]))));
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)n_all || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            float ex, ey, ez;
            const float q2 = rec_q2(rec_unpack(__ldg(rec + j)), me, ex, ey, ez);
            if (q2 < 1.0f) {
                float a2, a3;
                dens16_terms(q2, a2, a3);
                kahan(s2, c2, a2);
                kahan(s3, c3, a3);
            }
        }
    }
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS, BATCH ? 8 : 9)
k_density16_flat(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const uint4* __restrict__ rec,
                 const int2* __restrict__ table, const uint32_t* __restrict__ order,
                 float2* __restrict__ rr, int32_t* __restrict__ nlist, int32_t* __restrict__ ncount,
                 uint32_t* __restrict__ scanq, uint32_t* __restrict__ scanq_n,
                 uint32_t* __restrict__ err) {
    static_assert(NBR_THREADS == FLAT_THREADS, "the flat walk's block");
    __shared__ FlatShared S;
    __shared__ float s_q2[D16_CAP][NBR_THREADS];  // per thread: deferred q2
    const int tid = threadIdx.x;
    const uint32_t n = P0.n;
    uint32_t key = flat_ranges<BATCH>(P0, sr, xp, table, order, err, S);
    key = flat_sort(key, reinterpret_cast<uint32_t*>(&s_q2[0][0]), S);
    const int src = (int)(key & 127u);
    const int32_t tot = (int32_t)(key >> 7);
    const uint32_t meta = S.meta[src];
    flat_move(src, S);
    const bool live = (meta & FLAT_LIVE) != 0, over = (meta & FLAT_OVER) != 0;
    const uint32_t t = blockIdx.x * NBR_THREADS + (uint32_t)src;
    const uint32_t i = live ? order[t] : 0u;
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const Unpacked me = rec_unpack(live ? rec[i] : make_uint4(0u, 0u, 0u, 0u));
    const int32_t self = (int32_t)i;
    float s2 = 0.0f, c2 = 0.0f, s3 = 0.0f, c3 = 0.0f;
    float* dp = &s_q2[0][tid];
    float* const dfull = &s_q2[D16_CAP - 1][tid];
    int32_t cnt = 0;
    const int32_t lcap1 = (int32_t)P.list_cap - 1;
    auto test = [&](const uint4 q, int32_t jq, bool fq, bool valid) {
        float ex, ey, ez;
        const float q2 = rec_q2(rec_unpack(q), me, ex, ey, ez);
        const bool in = valid && q2 < 1.0f;
        *dp = q2;
        dp += (in && fq) ? NBR_THREADS : 0;
        // a list past its capacity keeps overwriting its last row (its count
        // sends the particle to the scan queue)
        const bool le = in && jq != self;
        if (le) __stcs(nlist + (size_t)min(cnt, lcap1) * n + t, jq);
        cnt += le ? 1 : 0;
    };
    auto term = [&](float q2) {
        float a2, a3;
        dens16_terms(q2, a2, a3);
        kahan(s2, c2, a2);
        kahan(s3, c3, a3);
    };
    // all lanes drain together once one of them has no room for a pair
    auto drain_if_full = [&]() {
        if (__any_sync(0xffffffffu, dp >= dfull)) {
            for (int c = 0; c < D16_CAP; c++)
                if (&s_q2[c][tid] < dp) term(s_q2[c][tid]);
            dp = &s_q2[0][tid];
        }
    };
    flat_walk(S, tot, self, (meta & FLAT_ALLF) != 0, [&](int32_t j) { return __ldg(rec + j); }, test,
              drain_if_full);
    for (const float* e = &s_q2[0][tid]; e < dp; e += NBR_THREADS) term(*e);
    const bool scan = live && (over || !((meta & FLAT_LIST_OK) != 0 && cnt <= (int32_t)P.list_cap));
    if (live) {
        if (over) density16_scan_one(P, xp[i], me, rec, table, n, err, s2, c2, s3, c3);
        const float h = P.h, h2 = h * h;
        const float d = (P.m * (s2 * h2)) / P.volume;
        const float nd = (P.m * (s3 * h2 * h)) * P.near_inv;
        rr[i] = make_float2((0.01f < d) ? d : 0.01f, (0.01f < nd) ? nd : 0.01f);
        ncount[t] = scan ? -1 : cnt;
    }
    flat_enqueue(scan, t, scanq, scanq_n);
}

// Particle-side constants of the force terms in the units of the records.
struct Self16 {
    Unpacked me;
    float pvx, pvy, pvz;     // v*_i in units of h/dt
    float my_p, near_p;      // (rho_i - rho0) k, rho_near_i kn
};

struct Acc16 {
    float fpx, fpy, fpz, fvx, fvy, fvz;
};

// One neighbour's force increments in record units: inc[0..2] pressure
// (pressure and near pressure combined), inc[3..5] viscosity.  Zero for
// candidates out of range or closer than 1e-7 (r^2 < 1e-14; adding +0
// leaves a sum that started at +0 unchanged).  Densities are at least 0.01
// (the density pass clamps them), so the approximate reciprocals are safe.
__device__ __forceinline__ void force16_incr(const DevParams& P, const Self16& s, const Unpacked& o,
                                             const float2 rrj, float inc[6]) {
    float ex, ey, ez;
    const float q2 = rec_q2(o, s.me, ex, ey, ez);
    if (q2 >= 1.0f || q2 * (P.h * P.h) < 1e-14f) {
#pragma unroll
        for (int c = 0; c < 6; c++) inc[c] = 0.0f;
        return;
    }
    const float inv_q = rsqrtf(q2);
    const float q = q2 * inv_q;
    const float dj = rrj.x, nnd = rrj.y;
    const float inv_dj = __fdividef(1.0f, dj), inv_nnd = __fdividef(1.0f, nnd);
    const float a = 1.0f - q;
    const float shared = 0.5f * ((dj - P.rho0) * P.k + s.my_p);
    const float coef = shared * (-a * (P.h * P.slope_scale)) * P.m * inv_dj;
    const float shared_near = 0.5f * (s.near_p + nnd * P.kn);
    const float ncoef = shared_near * (a * a * (P.h * P.h * P.near_slope_scale)) * P.m * inv_nnd;
    const float pc = (coef + ncoef) * inv_q;
    inc[0] = pc * ex;
    inc[1] = pc * ey;
    inc[2] = pc * ez;
    const float vcoef = P.h * P.h * P.m * a * a * inv_dj;
    inc[3] = vcoef * (o.vx - s.pvx);
    inc[4] = vcoef * (o.vy - s.pvy);
    inc[5] = vcoef * (o.vz - s.pvz);
}

__device__ __forceinline__ void force16_term(const DevParams& P, const Self16& s, const Unpacked& o,
                                             const float2 rrj, Acc16& f) {
    float v[6];
    force16_incr(P, s, o, rrj, v);
    f.fpx += v[0];
    f.fpy += v[1];
    f.fpz += v[2];
    f.fvx += v[3];
    f.fvy += v[4];
    f.fvz += v[5];
}

__device__ __forceinline__ Self16 self16(const DevParams& P, const uint4 ri, const float4 pv,
                                         const float2 rri) {
    Self16 s;
    s.me = rec_unpack(ri);
    const float vunit = P.h / P.dt;
    s.pvx = pv.x / vunit;
    s.pvy = pv.y / vunit;
    s.pvz = pv.z / vunit;
    s.my_p = (rri.x - P.rho0) * P.k;
    s.near_p = rri.y * P.kn;
    return s;
}

__device__ __forceinline__ float4 force16_finish(const DevParams& P, const Acc16& f, float4 vi,
                                                 float my_density) {
    const float sv = P.visc * (P.h / P.dt);
    const float tx = f.fpx + sv * f.fvx, ty = f.fpy + sv * f.fvy, tz = f.fpz + sv * f.fvz;
    const float g = P.dt / my_density;
    return make_float4(vi.x + tx * g, vi.y + ty * g, vi.z + tz * g, vi.w + 1.0f);
}

// Full 27-cell scan for one particle (queued: no list).
__device__ __forceinline__ float4 force16_scan_one(const DevParams& P, uint32_t i,
                                                   const float4* __restrict__ xp,
                                                   const float4* __restrict__ vp,
                                                   const float4* __restrict__ vs,
                                                   const uint4* __restrict__ rec,
                                                   const float2* __restrict__ rr,
                                                   const int2* __restrict__ table,
                                                   uint32_t* __restrict__ err) {
    const uint32_t n = P.n;
    const float4 sp = xp[i];
    const float2 rri = rr[i];
    const Self16 s = self16(P, rec[i], vp[i], rri);
    const bool inside = !(sp.x < P.minx) && !(sp.y < P.miny) && !(sp.z < P.minz) &&
                        !(sp.x > P.maxx) && !(sp.y > P.maxy) && !(sp.z > P.maxz);
    const int32_t cx = inside ? cell_coord(sp.x, P.minx, P.h) : -1;
    const int32_t cy = inside ? cell_coord(sp.y, P.miny, P.h) : -1;
    const int32_t cz = inside ? cell_coord(sp.z, P.minz, P.h) : -1;
    uint32_t hx[3], hy[3], hz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        hx[a] = ((uint32_t)cx + (uint32_t)(a - 1)) * 73856093u;
        hy[a] = ((uint32_t)cy + (uint32_t)(a - 1)) * 19349663u;
        hz[a] = ((uint32_t)cz + (uint32_t)(a - 1)) * 83492791u;
    }
    Acc16 f = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const int2 se = __ldg(table + slot_of(P, hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                                               pick3(dy, hy[0], hy[1], hy[2]) ^
                                                               pick3(dz, hz[0], hz[1], hz[2]))));
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)n || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            if (j == (int32_t)i) continue;
            force16_term(P, s, rec_unpack(__ldg(rec + j)), __ldg(rr + j), f);
        }
    }
    return force16_finish(P, f, vs[i], rri.x);
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS)
k_force16(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
          const float4* __restrict__ vs, const uint4* __restrict__ rec,
          const float2* __restrict__ rr, const int2* __restrict__ table,
          const uint32_t* __restrict__ order, const int32_t* __restrict__ nlist,
          const int32_t* __restrict__ ncount, const uint32_t* __restrict__ scanq,
          const uint32_t* __restrict__ scanq_n, uint32_t qblocks, float4* __restrict__ vout,
          uint32_t* __restrict__ err) {
    const uint32_t n = P0.n;
    if (blockIdx.x < qblocks) {
        const uint32_t total = min(*scanq_n, n);
        for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += qblocks * blockDim.x) {
            const uint32_t t = scanq[q];
            const uint32_t i = t < n ? order[t] : n;
            if (i >= n) {
                atomicOr(err, ERR_PERM_RANGE);
                continue;
            }
            vout[i] = force16_scan_one(params_of<BATCH>(P0, sr, i), i, xp, vp, vs, rec, rr, table, err);
        }
        return;
    }
    const uint32_t t = list_length_order((blockIdx.x - qblocks) * blockDim.x, n, ncount);
    if (t >= n) return;
    const int32_t cnt = ncount[t];
    if (cnt < 0) return;
    const uint32_t i = order[t];
    if (i >= n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float2 rri = rr[i];
    const Self16 s = self16(P, rec[i], vp[i], rri);
    Acc16 f = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    auto index = [&](int32_t k) -> int32_t {
        const int32_t j = k < cnt ? __ldg(nlist + (size_t)k * n + t) : (int32_t)i;
        if ((uint32_t)j >= n) {
            atomicOr(err, ERR_TABLE_RANGE);
            return (int32_t)i;  // self: distance 0, skipped
        }
        return j;
    };
    int32_t jn = index(1);
    int32_t j = index(0);
    uint4 r = __ldg(rec + j);
    float2 rj = __ldg(rr + j);
    for (int32_t k = 0; k < cnt; k++) {
        const int32_t jnn = index(k + 2);
        const uint4 rn = __ldg(rec + jn);
        const float2 rjn = __ldg(rr + jn);
        force16_term(P, s, rec_unpack(r), rj, f);
        r = rn;
        rj = rjn;
        jn = jnn;
    }
    vout[i] = force16_finish(P, f, vs[i], rri.x);
}

// ---- grid search (pfs_geo.cuh): one warp per particle ------------------------

constexpr int GEO16_DCAP = 512;
constexpr int GEO16_FCAP = 256;

__device__ __forceinline__ bool geo16_skip(const DevParams& P0, SceneRef sr, uint32_t i, bool batch) {
    return batch ? !__ldg(&sr.scenes[__ldg(sr.sid + i)].geo) : !P0.geo;
}

// Density pass of the grid-search particles, as k_density16_flat (same sums in
// the same order, same list and queue decisions).  Nine blocks per SM, as
// k_density_geo.
template <bool BATCH>
__global__ void __launch_bounds__(GEO_WARPS * 32, 9)
k_density16_geo(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const uint4* __restrict__ rec,
                const int2* __restrict__ table, const uint32_t* __restrict__ order,
                const uint32_t* __restrict__ bucket, const uint32_t* __restrict__ brank,
                const uint32_t* __restrict__ bcount, const uint32_t* __restrict__ boffset,
                uint32_t nblocks, float2* __restrict__ rr, int32_t* __restrict__ nlist,
                int32_t* __restrict__ ncount, uint32_t* __restrict__ scanq,
                uint32_t* __restrict__ scanq_n, uint32_t* __restrict__ err) {
    __shared__ int32_t s_j[GEO_WARPS][GEO16_DCAP];
    __shared__ float s_a[GEO_WARPS][GEO16_DCAP];
    __shared__ float s_b[GEO_WARPS][GEO16_DCAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full = 0xffffffffu, lt = (1u << lane) - 1u;
    int32_t* sj = s_j[w];
    float* sa = s_a[w];
    float* sb = s_b[w];
    const uint32_t n = P0.n;
    for (uint32_t i = blockIdx.x * GEO_WARPS + w; i < n; i += gridDim.x * GEO_WARPS) {
        if (geo16_skip(P0, sr, i, BATCH)) continue;
        const DevParams P = params_of<BATCH>(P0, sr, i);
        const float4 sp = xp[i];
        const Unpacked me = rec_unpack(rec[i]);
        const float h = P.h;
        const float off[3] = {PFS_MUL(h, -1.0f), PFS_MUL(h, 0.0f), h};
        bool vx[3], vy[3], vz[3];
        int32_t cx[3], cy[3], cz[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float sx = PFS_ADD(sp.x, off[a]), sy = PFS_ADD(sp.y, off[a]), sz = PFS_ADD(sp.z, off[a]);
            vx[a] = !(sx < P.minx) && !(sx > P.maxx);
            vy[a] = !(sy < P.miny) && !(sy > P.maxy);
            vz[a] = !(sz < P.minz) && !(sz > P.maxz);
            cx[a] = cell_coord(sx, P.minx, h);
            cy[a] = cell_coord(sy, P.miny, h);
            cz[a] = cell_coord(sz, P.minz, h);
        }
        const bool listing = vx[1] && vy[1] && vz[1] && (!vx[0] || cx[0] == cx[1] - 1) &&
                             (!vx[2] || cx[2] == cx[1] + 1) && (!vy[0] || cy[0] == cy[1] - 1) &&
                             (!vy[2] || cy[2] == cy[1] + 1) && (!vz[0] || cz[0] == cz[1] - 1) &&
                             (!vz[2] || cz[2] == cz[1] + 1);
        bool dens = false, bad = false;
        int2 se = make_int2(-1, -1);
        if (lane < 27) {
            const int dz = lane / 9, dy = (lane / 3) % 3, dx = lane % 3;
            dens = pickb(dx, vx[0], vx[1], vx[2]) && pickb(dy, vy[0], vy[1], vy[2]) &&
                   pickb(dz, vz[0], vz[1], vz[2]);
            if (dens || listing) {
                const int32_t kx = listing ? cx[1] + dx - 1 : (dx == 0 ? cx[0] : (dx == 1 ? cx[1] : cx[2]));
                const int32_t ky = listing ? cy[1] + dy - 1 : (dy == 0 ? cy[0] : (dy == 1 ? cy[1] : cy[2]));
                const int32_t kz = listing ? cz[1] + dz - 1 : (dz == 0 ? cz[0] : (dz == 1 ? cz[1] : cz[2]));
                se = __ldg(table + slot_of(P, hash_finalize(((uint32_t)kx * 73856093u) ^
                                                            ((uint32_t)ky * 19349663u) ^
                                                            ((uint32_t)kz * 83492791u))));
                if (se.x != -1 && (se.x < 0 || se.y > (int32_t)n || se.x > se.y)) {
                    atomicOr(err, ERR_TABLE_RANGE);
                    bad = true;
                    se = make_int2(-1, -1);
                }
            }
        }
        bool list_ok = listing && !__any_sync(full, bad);
        const int m = warp_gather(P, sp.x, sp.y, sp.z, bcount, boffset, order, sj, GEO16_DCAP, err,
                                  [&](int32_t j) {
                                      float ex, ey, ez;
                                      return rec_q2(rec_unpack(__ldg(rec + j)), me, ex, ey, ez) < 1.0f;
                                  });
        float s2 = 0.0f, c2 = 0.0f, s3 = 0.0f, c3 = 0.0f;  // lane 0: s2 c2, lane 1: s3 c3
        int32_t cnt = 0;
        const uint32_t t = order_position(i, n, nblocks, bucket, brank, boffset);
        if (m <= GEO16_DCAP) {
            warp_sort(sj, m);
            for (int k = lane; k < m; k += 32) {
                float ex, ey, ez;
                const float q2 = rec_q2(rec_unpack(__ldg(rec + sj[k])), me, ex, ey, ez);
                dens16_terms(q2, sa[k], sb[k]);
            }
            int lo = 0, hi = 0;
            if (se.x != -1) {
                lo = geo_lower(sj, m, se.x);
                hi = geo_lower(sj, m, se.y);
            }
            __syncwarp();
            // list length first (self excluded); an overflowing list is not written
            bool write_list = false;
            if (listing) {
                const int mine = hi - lo - ((se.x != -1 && se.x <= (int32_t)i && (int32_t)i < se.y) ? 1 : 0);
                int len = lane < 27 ? mine : 0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) len += __shfl_xor_sync(full, len, o);
                write_list = len <= (int)P.list_cap;
                if (!write_list) {
                    list_ok = false;
                    cnt = len;
                }
            }
            for (int d = 0; d < 27; d++) {
                const bool dd_ = __shfl_sync(full, dens, d);
                const int l = __shfl_sync(full, lo, d), u = __shfl_sync(full, hi, d);
                if (dd_) {
                    // lanes 0 and 1 run the two sums side by side in one loop
                    if (lane < 2) {
                        const float* src = lane == 0 ? sa : sb;
                        float s = lane == 0 ? s2 : s3, c = lane == 0 ? c2 : c3;
                        for (int k = l; k < u; k++) kahan(s, c, src[k]);
                        if (lane == 0) {
                            s2 = s;
                            c2 = c;
                        } else {
                            s3 = s;
                            c3 = c;
                        }
                    }
                }
                if (write_list) {
                    for (int base = l; base < u; base += 32) {
                        const int k = base + lane;
                        const int32_t j = k < u ? sj[k] : (int32_t)i;
                        const bool e = j != (int32_t)i;
                        const uint32_t mk = __ballot_sync(full, e);
                        const int32_t pos = cnt + __popc(mk & lt);
                        if (e && pos < (int32_t)P.list_cap && t < n) nlist[(size_t)pos * n + t] = j;
                        cnt += __popc(mk);
                    }
                }
            }
        } else {
            list_ok = false;
            for (int d = 0; d < 27; d++) {
                const bool dd_ = __shfl_sync(full, dens, d);
                const int32_t r0 = __shfl_sync(full, se.x, d), r1 = __shfl_sync(full, se.y, d);
                if (!dd_ || r0 == -1) continue;
                for (int32_t base = r0; base < r1; base += 32) {
                    const int32_t j = base + lane;
                    bool in = false;
                    if (j < r1) {
                        float ex, ey, ez;
                        const float q2 = rec_q2(rec_unpack(__ldg(rec + j)), me, ex, ey, ez);
                        in = q2 < 1.0f;
                        if (in) dens16_terms(q2, sa[lane], sb[lane]);
                    }
                    uint32_t mk = __ballot_sync(full, in);
                    __syncwarp();
                    if (lane < 2) {
                        const float* src = lane == 0 ? sa : sb;
                        float acc = lane == 0 ? s2 : s3, comp = lane == 0 ? c2 : c3;
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1u;
                            kahan(acc, comp, src[k]);
                        }
                        if (lane == 0) {
                            s2 = acc;
                            c2 = comp;
                        } else {
                            s3 = acc;
                            c3 = comp;
                        }
                    }
                    __syncwarp();
                }
            }
        }
        s2 = __shfl_sync(full, s2, 0);
        s3 = __shfl_sync(full, s3, 1);
        if (lane == 0) {
            const float h2 = h * h;
            const float dn = (P.m * (s2 * h2)) / P.volume;
            const float nd = (P.m * (s3 * h2 * h)) * P.near_inv;
            rr[i] = make_float2((0.01f < dn) ? dn : 0.01f, (0.01f < nd) ? nd : 0.01f);
            if (t < n) {
                const bool scan = !(list_ok && cnt <= (int32_t)P.list_cap);
                ncount[t] = scan ? -1 : cnt;
                if (scan) {
                    const uint32_t q = atomicAdd(scanq_n + 1, 1u);
                    if (q < n) *geo_queue_entry(scanq, n, q) = i;
                }
            } else {
                atomicOr(err, ERR_PERM_RANGE);
            }
        }
        __syncwarp();
    }
}

// Force pass of the grid-search queue, as force16_scan_one.
template <bool BATCH>
__global__ void __launch_bounds__(GEO_WARPS * 32)
k_force16_geo(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
              const float4* __restrict__ vs, const uint4* __restrict__ rec,
              const float2* __restrict__ rr, const int2* __restrict__ table,
              const uint32_t* __restrict__ order, const uint32_t* __restrict__ bcount,
              const uint32_t* __restrict__ boffset, const uint32_t* __restrict__ scanq,
              const uint32_t* __restrict__ scanq_n, float4* __restrict__ vout,
              uint32_t* __restrict__ err) {
    __shared__ int32_t s_j[GEO_WARPS][GEO16_FCAP];
    __shared__ float s_inc[GEO_WARPS][6][GEO16_FCAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full = 0xffffffffu;
    int32_t* sj = s_j[w];
    float(*inc)[GEO16_FCAP] = s_inc[w];
    const uint32_t n = P0.n;
    const uint32_t total_q = min(scanq_n[1], n);
    for (uint32_t q = blockIdx.x * GEO_WARPS + w; q < total_q; q += gridDim.x * GEO_WARPS) {
        const uint32_t i = scanq[n - 1u - q];
        if (i >= n) {
            if (lane == 0) atomicOr(err, ERR_PERM_RANGE);
            continue;
        }
        const DevParams P = params_of<BATCH>(P0, sr, i);
        const float4 sp = xp[i];
        const float2 rri = rr[i];
        const Self16 s = self16(P, rec[i], vp[i], rri);
        const bool inside = !(sp.x < P.minx) && !(sp.y < P.miny) && !(sp.z < P.minz) &&
                            !(sp.x > P.maxx) && !(sp.y > P.maxy) && !(sp.z > P.maxz);
        const int32_t cx = inside ? cell_coord(sp.x, P.minx, P.h) : -1;
        const int32_t cy = inside ? cell_coord(sp.y, P.miny, P.h) : -1;
        const int32_t cz = inside ? cell_coord(sp.z, P.minz, P.h) : -1;
        int2 se = make_int2(-1, -1);
        if (lane < 27) {
            const int dz = lane / 9, dy = (lane / 3) % 3, dx = lane % 3;
            se = __ldg(table + slot_of(P, hash_finalize(
                                              (((uint32_t)cx + (uint32_t)(dx - 1)) * 73856093u) ^
                                              (((uint32_t)cy + (uint32_t)(dy - 1)) * 19349663u) ^
                                              (((uint32_t)cz + (uint32_t)(dz - 1)) * 83492791u))));
            if (se.x != -1 && (se.x < 0 || se.y > (int32_t)n || se.x > se.y)) {
                atomicOr(err, ERR_TABLE_RANGE);
                se = make_int2(-1, -1);
            }
        }
        const int m = warp_gather(P, sp.x, sp.y, sp.z, bcount, boffset, order, sj, GEO16_FCAP, err,
                                  [&](int32_t j) {
                                      if (j == (int32_t)i) return false;
                                      float ex, ey, ez;
                                      return rec_q2(rec_unpack(__ldg(rec + j)), s.me, ex, ey, ez) < 1.0f;
                                  });
        float acc = 0.0f;  // lanes 0..5: fpx fpy fpz fvx fvy fvz
        if (m <= GEO16_FCAP) {
            warp_sort(sj, m);
            for (int k = lane; k < m; k += 32) {
                const int32_t j = sj[k];
                float v[6];
                force16_incr(P, s, rec_unpack(__ldg(rec + j)), __ldg(rr + j), v);
#pragma unroll
                for (int c = 0; c < 6; c++) inc[c][k] = v[c];
            }
            int lo = 0, hi = 0;
            if (se.x != -1) {
                lo = geo_lower(sj, m, se.x);
                hi = geo_lower(sj, m, se.y);
            }
            __syncwarp();
            for (int d = 0; d < 27; d++) {
                const int l = __shfl_sync(full, lo, d), u = __shfl_sync(full, hi, d);
                if (lane < 6)
                    for (int k = l; k < u; k++) acc += inc[lane][k];
            }
        } else {
            for (int d = 0; d < 27; d++) {
                const int32_t r0 = __shfl_sync(full, se.x, d), r1 = __shfl_sync(full, se.y, d);
                if (r0 == -1) continue;
                for (int32_t base = r0; base < r1; base += 32) {
                    const int32_t j = base + lane;
                    const bool in = j < r1 && j != (int32_t)i;
                    if (in) {
                        float v[6];
                        force16_incr(P, s, rec_unpack(__ldg(rec + j)), __ldg(rr + j), v);
#pragma unroll
                        for (int c = 0; c < 6; c++) inc[c][lane] = v[c];
                    }
                    uint32_t mk = __ballot_sync(full, in);
                    __syncwarp();
                    if (lane < 6) {
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1u;
                            acc += inc[lane][k];
                        }
                    }
                    __syncwarp();
                }
            }
        }
        Acc16 f;
        f.fpx = __shfl_sync(full, acc, 0);
        f.fpy = __shfl_sync(full, acc, 1);
        f.fpz = __shfl_sync(full, acc, 2);
        f.fvx = __shfl_sync(full, acc, 3);
        f.fvy = __shfl_sync(full, acc, 4);
        f.fvz = __shfl_sync(full, acc, 5);
        if (lane == 0) vout[i] = force16_finish(P, f, vs[i], rri.x);
        __syncwarp();
    }
}

// Thread blocks of kernel k (GEO_WARPS warps each) that are resident at once
// on the current device, at most one warp per item: the grid-search kernels
// stride over their items, so a grid beyond one resident wave would leave a
// second wave of whole strides behind the first.
template <class K>
unsigned geo16_grid(K kernel, uint32_t items) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, GEO_WARPS * 32, 0);
    const unsigned resident = (unsigned)std::max(1, per_sm) * (unsigned)std::max(1, sms);
    return std::max(1u, std::min(resident, (items + GEO_WARPS - 1) / GEO_WARPS));
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
    StepBuffers bb = b;
    bb.rec = f.rec;  // the shared reorder writes the records
    return launch_reorder(P, bb, s);
}

cudaError_t launch_density_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                                cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, NBR_THREADS);
    if (b.sr.scenes)
        k_density16_flat<true><<<g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, f.rec, b.table, b.order, b.rr,
                                                          b.nlist, b.ncount, b.scanq, b.scanq_n, b.err);
    else
        k_density16_flat<false><<<g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, f.rec, b.table, b.order, b.rr,
                                                           b.nlist, b.ncount, b.scanq, b.scanq_n, b.err);
    if (b.geo_any) {
                if (b.sr.scenes)
            k_density16_geo<true><<<geo16_grid(k_density16_geo<true>, P.n), GEO_WARPS * 32, 0, s>>>(
                P, b.sr, b.xp, f.rec, b.table, b.order, b.bucket, b.brank, b.bcount, b.boffset,
                b.nblocks, b.rr, b.nlist, b.ncount, b.scanq, b.scanq_n, b.err);
        else
            k_density16_geo<false><<<geo16_grid(k_density16_geo<false>, P.n), GEO_WARPS * 32, 0, s>>>(
                P, b.sr, b.xp, f.rec, b.table, b.order, b.bucket, b.brank, b.bcount, b.boffset,
                b.nblocks, b.rr, b.nlist, b.ncount, b.scanq, b.scanq_n, b.err);
    }
    return cudaGetLastError();
}

cudaError_t launch_force_fp16(const DevParams& P, const StepBuffers& b, const Fp16Buffers& f,
                              cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, NBR_THREADS);
    // one queue thread per possible entry: dense scenes can send most
    // particles to the queue (lists overflow); surplus queue blocks exit at once
    const unsigned qb = g;
    if (b.sr.scenes)
        k_force16<true><<<qb + g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, f.rec, b.rr, b.table,
                                                       b.order, b.nlist, b.ncount, b.scanq,
                                                       b.scanq_n, qb, b.v, b.err);
    else
        k_force16<false><<<qb + g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, f.rec, b.rr,
                                                        b.table, b.order, b.nlist, b.ncount,
                                                        b.scanq, b.scanq_n, qb, b.v, b.err);
    if (b.geo_any) {
                if (b.sr.scenes)
            k_force16_geo<true><<<geo16_grid(k_force16_geo<true>, P.n), GEO_WARPS * 32, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, f.rec, b.rr,
                                                              b.table, b.order, b.bcount, b.boffset,
                                                              b.scanq, b.scanq_n, b.v, b.err);
        else
            k_force16_geo<false><<<geo16_grid(k_force16_geo<false>, P.n), GEO_WARPS * 32, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, f.rec, b.rr,
                                                               b.table, b.order, b.bcount, b.boffset,
                                                               b.scanq, b.scanq_n, b.v, b.err);
    }
    return cudaGetLastError();
}

}  // namespace pfs
