// pfs_nbr.cuh — device helpers shared by the FP32 neighbour-pass kernels
// (pfs_neighbors.cu, pfs_staged.cu): table ranges, sample-point and cell
// offsets, the distance, and the density and force terms in the reference
// shaders' operation order (calculateDensities.comp:96-131,
// applyPressureAndViscosityForce.comp:121-182), one IEEE round-to-nearest
// operation each.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"

namespace pfs {
namespace {

__device__ __forceinline__ uint32_t pick3(int i, uint32_t a, uint32_t b, uint32_t c) {
    return i == 0 ? a : (i == 1 ? b : c);
}
__device__ __forceinline__ bool pickb(int i, bool a, bool b, bool c) {
    return i == 0 ? a : (i == 1 ? b : c);
}

__device__ __forceinline__ bool table_range_ok(const int2 se, uint32_t n) {
    return se.x >= 0 && se.y <= (int32_t)n && se.x <= se.y;
}

// Per-particle neighbourhood set-up shared by both shapes of the density pass:
// sample-point validity and hash partial products per axis.
struct DensityCells {
    uint32_t hx[3], hy[3], hz[3];
    bool vx[3], vy[3], vz[3];
};

__device__ __forceinline__ void density_cells(const DevParams& P, const float4 sp, DensityCells& c) {
    const float h = P.h;
    const float off[3] = {PFS_MUL(h, -1.0f), PFS_MUL(h, 0.0f), h};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float sx = PFS_ADD(sp.x, off[a]), sy = PFS_ADD(sp.y, off[a]), sz = PFS_ADD(sp.z, off[a]);
        c.vx[a] = !(sx < P.minx) && !(sx > P.maxx);
        c.vy[a] = !(sy < P.miny) && !(sy > P.maxy);
        c.vz[a] = !(sz < P.minz) && !(sz > P.maxz);
        c.hx[a] = (uint32_t)cell_coord(sx, P.minx, h) * 73856093u;
        c.hy[a] = (uint32_t)cell_coord(sy, P.miny, h) * 19349663u;
        c.hz[a] = (uint32_t)cell_coord(sz, P.minz, h) * 83492791u;
    }
}

// Hash partial products of the 27 cell offsets around the cell of x*
// (samplePointToCellCoord returns (-1,-1,-1) outside the box).
struct ForceCells {
    uint32_t hx[3], hy[3], hz[3];
};

__device__ __forceinline__ void force_cells(const DevParams& P, const float4 sp, ForceCells& c) {
    const bool inside = !(sp.x < P.minx) && !(sp.y < P.miny) && !(sp.z < P.minz) &&
                        !(sp.x > P.maxx) && !(sp.y > P.maxy) && !(sp.z > P.maxz);
    const int32_t cx = inside ? cell_coord(sp.x, P.minx, P.h) : -1;
    const int32_t cy = inside ? cell_coord(sp.y, P.miny, P.h) : -1;
    const int32_t cz = inside ? cell_coord(sp.z, P.minz, P.h) : -1;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        c.hx[a] = ((uint32_t)cx + (uint32_t)(a - 1)) * 73856093u;
        c.hy[a] = ((uint32_t)cy + (uint32_t)(a - 1)) * 19349663u;
        c.hz[a] = ((uint32_t)cz + (uint32_t)(a - 1)) * 83492791u;
    }
}

__device__ __forceinline__ float dist2(const float4 q, const float4 sp, float& d0, float& d1, float& d2) {
    d0 = PFS_SUB(q.x, sp.x);
    d1 = PFS_SUB(q.y, sp.y);
    d2 = PFS_SUB(q.z, sp.z);
    return PFS_ADD(PFS_ADD(PFS_MUL(d0, d0), PFS_MUL(d1, d1)), PFS_MUL(d2, d2));
}

// Whether a candidate at squared distance dd takes part in a neighbour sum:
// every dd below skip_d2 (distance below h), and a NaN distance, which the
// shaders' own tests (dist >= h, dist2 > h^2) do not skip either, so its NaN
// terms reach the sums as they do in the reference.
__device__ __forceinline__ bool in_reach(float dd, float skip) { return !(dd >= skip); }

// Scan candidates [j0, j1) in table order and hand each in-range one
// (d2 < skip, slot != self) to emit(j, d2) in order.
template <class Emit>
__device__ __forceinline__ void scan_range(const float4* __restrict__ xp, int32_t j0, int32_t j1,
                                           const float4 sp, float skip, int32_t self, Emit&& emit) {
    for (int32_t j = j0; j < j1; j++) {
        float d0, d1, d2;
        const float dd = dist2(__ldg(xp + j), sp, d0, d1, d2);
        if (j != self && in_reach(dd, skip)) emit(j, dd);
    }
}

// ---- density ---------------------------------------------------------------

__device__ __forceinline__ void density_term(float dd, float h, float m, float& total,
                                             float& total_near) {
    const float a = PFS_SUB(h, PFS_SQRT(dd));
    const float a2 = PFS_MUL(a, a);
    total = PFS_ADD(total, PFS_MUL(m, a2));
    total_near = PFS_ADD(total_near, PFS_MUL(m, PFS_MUL(a2, a)));
}

__device__ __forceinline__ float2 density_finish(const DevParams& P, float total, float total_near) {
    const float d = PFS_DIV(total, P.volume);
    const float nd = PFS_MUL(total_near, P.near_inv);
    return make_float2((0.01f < d) ? d : 0.01f, (0.01f < nd) ? nd : 0.01f);
}

// Density of one particle by its own 27-cell walk from global memory (the
// fallback; exact arithmetic).
__device__ __forceinline__ float2 density_scan_one(const DevParams& P, const float4 sp,
                                                   const float4* __restrict__ xp,
                                                   const int2* __restrict__ table,
                                                   uint32_t* __restrict__ err) {
    DensityCells cl;
    density_cells(P, sp, cl);
    float total = 0.0f, total_near = 0.0f;
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        if (!(pickb(dx, cl.vx[0], cl.vx[1], cl.vx[2]) && pickb(dy, cl.vy[0], cl.vy[1], cl.vy[2]) &&
              pickb(dz, cl.vz[0], cl.vz[1], cl.vz[2])))
            continue;
        const uint32_t key = slot_of(P, hash_finalize(pick3(dx, cl.hx[0], cl.hx[1], cl.hx[2]) ^
                                                      pick3(dy, cl.hy[0], cl.hy[1], cl.hy[2]) ^
                                                      pick3(dz, cl.hz[0], cl.hz[1], cl.hz[2])));
        const int2 se = __ldg(table + key);
        if (se.x == -1) continue;
        if (!table_range_ok(se, P.n)) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            float d0, d1, d2;
            const float dd = dist2(__ldg(xp + j), sp, d0, d1, d2);
            if (in_reach(dd, P.skip_d2)) density_term(dd, P.h, P.m, total, total_near);
        }
    }
    return density_finish(P, total, total_near);
}

// ---- force -----------------------------------------------------------------

struct ForceAcc {
    float fpx, fpy, fpz, fvx, fvy, fvz;
};

struct ForceSelf {
    float4 sp, pv;
    float my_pressure_term, near_pressure;
};

// One neighbour's pressure, viscosity and near-pressure terms from its
// already loaded x*_j, (rho_j, rho_near_j) and v_j.
__device__ __forceinline__ void force_term_pre(const DevParams& P, const ForceSelf& me,
                                               const float4 q, const float2 rrj, const float4 vj,
                                               ForceAcc& f);

__device__ __forceinline__ void force_term(const DevParams& P, const ForceSelf& me, int32_t j,
                                           const float4* __restrict__ xp,
                                           const float4* __restrict__ vs,
                                           const float2* __restrict__ rr, ForceAcc& f) {
    force_term_pre(P, me, __ldg(xp + j), __ldg(rr + j), __ldg(vs + j), f);
}

__device__ __forceinline__ void force_term_pre(const DevParams& P, const ForceSelf& me,
                                               const float4 q, const float2 rrj, const float4 vj,
                                               ForceAcc& f) {
    const float h = P.h, m = P.m;
    float d0, d1, d2;
    const float dd = dist2(q, me.sp, d0, d1, d2);
    const float dist = PFS_SQRT(dd);
    if (fabsf(dist) < 1e-7f) return;
    const float dirx = PFS_DIV(d0, dist), diry = PFS_DIV(d1, dist), dirz = PFS_DIV(d2, dist);
    const float slope = PFS_MUL(PFS_SUB(dist, h), P.slope_scale);
    const float dj = rrj.x;
    // (a + b) / 2 and (a + b) * 0.5 are the same correctly rounded value
    const float shared = PFS_MUL(PFS_ADD(PFS_MUL(PFS_SUB(dj, P.rho0), P.k), me.my_pressure_term), 0.5f);
    const float coef = PFS_DIV(PFS_MUL(PFS_MUL(shared, slope), m), dj);
    f.fpx = PFS_ADD(f.fpx, PFS_MUL(coef, dirx));
    f.fpy = PFS_ADD(f.fpy, PFS_MUL(coef, diry));
    f.fpz = PFS_ADD(f.fpz, PFS_MUL(coef, dirz));
    const float a = PFS_SUB(h, dist);
    const float a2 = PFS_MUL(a, a);
    const float vcoef = PFS_DIV(PFS_MUL(m, a2), dj);
    f.fvx = PFS_ADD(f.fvx, PFS_MUL(vcoef, PFS_SUB(vj.x, me.pv.x)));
    f.fvy = PFS_ADD(f.fvy, PFS_MUL(vcoef, PFS_SUB(vj.y, me.pv.y)));
    f.fvz = PFS_ADD(f.fvz, PFS_MUL(vcoef, PFS_SUB(vj.z, me.pv.z)));
    const float nnd = rrj.y;
    const float shared_near = PFS_MUL(PFS_ADD(me.near_pressure, PFS_MUL(nnd, P.kn)), 0.5f);
    const float nslope = PFS_MUL(a2, P.near_slope_scale);
    const float ncoef = PFS_DIV(PFS_MUL(PFS_MUL(shared_near, nslope), m), nnd);
    f.fpx = PFS_ADD(f.fpx, PFS_MUL(ncoef, dirx));
    f.fpy = PFS_ADD(f.fpy, PFS_MUL(ncoef, diry));
    f.fpz = PFS_ADD(f.fpz, PFS_MUL(ncoef, dirz));
}

__device__ __forceinline__ float4 force_finish(const DevParams& P, const ForceAcc& f, float4 vi,
                                               float my_density) {
    const float tx = PFS_ADD(PFS_ADD(f.fpx, PFS_MUL(P.visc, f.fvx)), 0.0f);
    const float ty = PFS_ADD(PFS_ADD(f.fpy, PFS_MUL(P.visc, f.fvy)), 0.0f);
    const float tz = PFS_ADD(PFS_ADD(f.fpz, PFS_MUL(P.visc, f.fvz)), 0.0f);
    return make_float4(PFS_ADD(vi.x, PFS_MUL(PFS_DIV(tx, my_density), P.dt)),
                       PFS_ADD(vi.y, PFS_MUL(PFS_DIV(ty, my_density), P.dt)),
                       PFS_ADD(vi.z, PFS_MUL(PFS_DIV(tz, my_density), P.dt)), PFS_ADD(vi.w, 1.0f));
}

__device__ __forceinline__ ForceSelf force_self(const DevParams& P, float4 sp, float4 pv, float2 rri) {
    ForceSelf me;
    me.sp = sp;
    me.pv = pv;
    me.my_pressure_term = PFS_MUL(PFS_SUB(rri.x, P.rho0), P.k);
    me.near_pressure = PFS_MUL(rri.y, P.kn);
    return me;
}

// Full 27-cell force evaluation of one particle (the *_simple walk).
__device__ __forceinline__ float4 force_scan_one(const DevParams& P, uint32_t i,
                                                 const float4* __restrict__ xp,
                                                 const float4* __restrict__ vp,
                                                 const float4* __restrict__ vs,
                                                 const float2* __restrict__ rr,
                                                 const int2* __restrict__ table,
                                                 uint32_t* __restrict__ err) {
    const uint32_t n = P.n;
    const float2 rri = rr[i];
    const ForceSelf me = force_self(P, xp[i], vp[i], rri);
    ForceAcc f = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    ForceCells cl;
    force_cells(P, me.sp, cl);
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const uint32_t key = slot_of(P, hash_finalize(pick3(dx, cl.hx[0], cl.hx[1], cl.hx[2]) ^
                                                      pick3(dy, cl.hy[0], cl.hy[1], cl.hy[2]) ^
                                                      pick3(dz, cl.hz[0], cl.hz[1], cl.hz[2])));
        const int2 se = __ldg(table + key);
        if (se.x == -1) continue;
        if (!table_range_ok(se, n)) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            if (j == (int32_t)i) continue;
            float d0, d1, d2;
            if (in_reach(dist2(__ldg(xp + j), me.sp, d0, d1, d2), P.skip_d2)) force_term(P, me, j, xp, vs, rr, f);
        }
    }
    return force_finish(P, f, vs[i], rri.x);
}

// One neighbour's pressure, viscosity and near-pressure terms in the
// PFS_FP32_FAST form: the same terms as force_term_pre, from the neighbour's
// record a = (x*, density), b = (v, near density), with fused multiply-adds,
// a hardware reciprocal square root for the distance and direction, and
// hardware reciprocals of the densities.
__device__ __forceinline__ void force_term_fast(const DevParams& P, const ForceSelf& me,
                                                const float4 a, const float4 b, ForceAcc& f) {
    const float d0 = __fsub_rn(a.x, me.sp.x), d1 = __fsub_rn(a.y, me.sp.y), d2 = __fsub_rn(a.z, me.sp.z);
    const float dd = __fmaf_rn(d0, d0, __fmaf_rn(d1, d1, __fmul_rn(d2, d2)));
    if (dd < P.min_d2) return;  // d < 1e-7: skipped, as the shader skips it
    const float inv = rsqrtf(dd);
    const float dist = __fmul_rn(dd, inv);
    const float mrj = __fmul_rn(P.m, __fdividef(1.0f, a.w));
    const float mrnj = __fmul_rn(P.m, __fdividef(1.0f, b.w));
    const float slope = __fmul_rn(__fsub_rn(dist, P.h), P.slope_scale);
    const float shared = __fmul_rn(__fmaf_rn(__fsub_rn(a.w, P.rho0), P.k, me.my_pressure_term), 0.5f);
    const float aa = __fsub_rn(P.h, dist);
    const float a2 = __fmul_rn(aa, aa);
    const float shared_near = __fmul_rn(__fmaf_rn(b.w, P.kn, me.near_pressure), 0.5f);
    const float ncoef = __fmul_rn(__fmul_rn(shared_near, __fmul_rn(a2, P.near_slope_scale)), mrnj);
    const float pc = __fmul_rn(__fmaf_rn(__fmul_rn(shared, slope), mrj, ncoef), inv);
    f.fpx = __fmaf_rn(pc, d0, f.fpx);
    f.fpy = __fmaf_rn(pc, d1, f.fpy);
    f.fpz = __fmaf_rn(pc, d2, f.fpz);
    const float vcoef = __fmul_rn(a2, mrj);
    f.fvx = __fmaf_rn(vcoef, __fsub_rn(b.x, me.pv.x), f.fvx);
    f.fvy = __fmaf_rn(vcoef, __fsub_rn(b.y, me.pv.y), f.fvy);
    f.fvz = __fmaf_rn(vcoef, __fsub_rn(b.z, me.pv.z), f.fvz);
}

}  // namespace
}  // namespace pfs
