// pfs_neighbors.cu — the two FP32 neighbour passes of the substep.
//
//   density: calculateDensities.comp:96-153 — 27 sample points x* + h*(dx,dy,dz)
//            (z outer, x inner), out-of-box sample points skipped, duplicate
//            keys not de-duplicated, self included, clamp at 0.01.
//   force:   applyPressureAndViscosityForce.comp:121-183 — 27 cell offsets
//            around the cell of x*, self / d2 > h^2 / dist < 1e-7 skipped,
//            shared pressure with the spiky derivative, viscosity on
//            (v_j - v*_i) with pre-update v_j (Jacobi), near pressure,
//            v_i += (F_p + F_v + 0) / rho_i * dt.
//
// Exactness: every float operation is one IEEE round-to-nearest operation in
// the shaders' order (PFS_* macros), and each particle's sums run over its
// candidates in table order, so results equal the oracle bit for bit.
// Candidates with d2 >= skip_d2 have distance >= h, where every kernel is
// zero: their exact +-0 terms cannot change a sum that starts at +0 (it never
// becomes -0), so they are skipped.  That test also covers the force pass's
// d2 > h^2 cut because skip_d2 <= h*h.  A NaN distance is not skipped
// (in_reach), as the shaders' tests do not skip it; so a state holding NaN
// gives the reference's NaN sums in the table-scan shapes.  The grid search
// finds candidates by the cell of x*, which a NaN x* does not have, so it
// leaves NaN candidates out: the two searches agree on finite states.  A
// candidate with d2 in [skip_d2, h*h] and a non-finite velocity difference
// would add 0 * Inf = NaN to the reference's viscosity sum, and nothing here.
//
// Kernel shapes per pass (all bit-identical; see also the list shape below):
//   *_simple  one thread per sorted particle walking its 27 cells; the heavy
//             in-range body runs whenever any lane of the warp has an in-range
//             candidate (~15% lane utilisation on dense scenes).
//   *_slab    the 27 cells in three z-slabs of nine: a slab's nine
//             table entries are fetched together, each lane scans its
//             candidates and appends the in-range ones to a per-lane list in
//             shared memory, and the list is processed densely (flushed early
//             only when it fills).  Same order, so same bits.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <type_traits>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_flat.cuh"
#include "pfs_geo.cuh"
#include "pfs_nbr.cuh"
#include "pfs_staged.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int NBR_THREADS = 128;
constexpr int NBR_CAP = 32;

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS)
k_density_simple(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const int2* __restrict__ table,
                 const uint32_t* __restrict__ order, float2* __restrict__ rr, uint32_t* __restrict__ err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P0.n) return;
    const uint32_t i = order[t];
    if (i >= P0.n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 sp = xp[i];
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
    rr[i] = density_finish(P, total, total_near);
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS, 6)
k_density_slab(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const int2* __restrict__ table,
               const uint32_t* __restrict__ order, float2* __restrict__ rr, uint32_t* __restrict__ err) {
    __shared__ float s_dd[NBR_CAP][NBR_THREADS];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P0.n) return;
    const uint32_t i = order[t];
    if (i >= P0.n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 sp = xp[i];
    DensityCells cl;
    density_cells(P, sp, cl);
    const float h = P.h, m = P.m, skip = P.skip_d2;
    float total = 0.0f, total_near = 0.0f;
    int cnt = 0;
    for (int dz = 0; dz < 3; dz++) {
        const uint32_t hz = pick3(dz, cl.hz[0], cl.hz[1], cl.hz[2]);
        const bool vz = pickb(dz, cl.vz[0], cl.vz[1], cl.vz[2]);
        int2 se[9];
#pragma unroll
        for (int q = 0; q < 9; q++) {
            const int dy = q / 3, dx = q % 3;
            if (vz && cl.vy[dy] && cl.vx[dx])
                se[q] = __ldg(table + slot_of(P, hash_finalize(cl.hx[dx] ^ cl.hy[dy] ^ hz)));
            else
                se[q] = make_int2(-1, -1);
        }
#pragma unroll
        for (int q = 0; q < 9; q++) {
            if (se[q].x == -1) continue;
            if (!table_range_ok(se[q], P.n)) {
                atomicOr(err, ERR_TABLE_RANGE);
                continue;
            }
            scan_range(xp, se[q].x, se[q].y, sp, skip, -1, [&](int32_t, float dd) {
                if (cnt == NBR_CAP) {
                    for (int t = 0; t < NBR_CAP; t++)
                        density_term(s_dd[t][threadIdx.x], h, m, total, total_near);
                    cnt = 0;
                }
                s_dd[cnt++][threadIdx.x] = dd;
            });
        }
    }
    for (int t = 0; t < cnt; t++) density_term(s_dd[t][threadIdx.x], h, m, total, total_near);
    rr[i] = density_finish(P, total, total_near);
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS)
k_force_simple(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
               const float4* __restrict__ vs, const float2* __restrict__ rr,
               const int2* __restrict__ table, const uint32_t* __restrict__ order, float4* __restrict__ vout,
               uint32_t* __restrict__ err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P0.n) return;
    const uint32_t i = order[t];
    if (i >= P0.n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float2 rri = rr[i];
    const ForceSelf me = force_self(P, xp[i], vp[i], rri);
    ForceCells cl;
    force_cells(P, me.sp, cl);
    ForceAcc f = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
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
            if (j == (int32_t)i) continue;
            float d0, d1, d2;
            if (in_reach(dist2(__ldg(xp + j), me.sp, d0, d1, d2), P.skip_d2)) force_term(P, me, j, xp, vs, rr, f);
        }
    }
    vout[i] = force_finish(P, f, vs[i], rri.x);
}

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS, 5)
k_force_slab(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
             const float4* __restrict__ vs, const float2* __restrict__ rr,
             const int2* __restrict__ table, const uint32_t* __restrict__ order, float4* __restrict__ vout,
             uint32_t* __restrict__ err) {
    __shared__ int32_t s_j[NBR_CAP][NBR_THREADS];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P0.n) return;
    const uint32_t i = order[t];
    if (i >= P0.n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float2 rri = rr[i];
    const ForceSelf me = force_self(P, xp[i], vp[i], rri);
    ForceCells cl;
    force_cells(P, me.sp, cl);
    const float skip = P.skip_d2;
    ForceAcc f = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    int cnt = 0;
    for (int dz = 0; dz < 3; dz++) {
        const uint32_t hz = pick3(dz, cl.hz[0], cl.hz[1], cl.hz[2]);
        int2 se[9];
#pragma unroll
        for (int q = 0; q < 9; q++)
            se[q] = __ldg(table + slot_of(P, hash_finalize(cl.hx[q % 3] ^ cl.hy[q / 3] ^ hz)));
#pragma unroll
        for (int q = 0; q < 9; q++) {
            if (se[q].x == -1) continue;
            if (!table_range_ok(se[q], P.n)) {
                atomicOr(err, ERR_TABLE_RANGE);
                continue;
            }
            scan_range(xp, se[q].x, se[q].y, me.sp, skip, (int32_t)i, [&](int32_t j, float) {
                if (cnt == NBR_CAP) {
                    for (int t = 0; t < NBR_CAP; t++) force_term(P, me, s_j[t][threadIdx.x], xp, vs, rr, f);
                    cnt = 0;
                }
                s_j[cnt++][threadIdx.x] = j;
            });
        }
    }
    for (int t = 0; t < cnt; t++) force_term(P, me, s_j[t][threadIdx.x], xp, vs, rr, f);
    vout[i] = force_finish(P, f, vs[i], rri.x);
}

// ---- list shape (default) ----------------------------------------------------
// The density pass walks its 27 sample-point cells exactly as *_simple does
// and, for each particle whose sample-point cells are exactly the force
// pass's 27 cell offsets (all sample points in the box and
// cell(x* + h*d) = cell(x*) + d on every axis — true away from walls and
// cell-boundary rounding), it also records its in-range candidates except
// itself: that is precisely the force pass's list of contributing
// neighbours, in the force pass's order.  The force pass then evaluates the
// list instead of rescanning ~100 candidates; particles without a list
// (ncount < 0: cells differ, or more than list_cap neighbours) are scanned
// as in *_simple.

// Force pass of the list shape.  The first qblocks thread blocks work
// through the queue of positions without a list (full scans, long latency
// chains, issued first so they overlap the list work); the others evaluate
// one listed particle per thread, a block's 128 positions in ascending list
// length.
template <bool BATCH, bool FAST>
__global__ void __launch_bounds__(NBR_THREADS)
k_force_list(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
             const float4* __restrict__ vs, const float2* __restrict__ rr,
             const int2* __restrict__ table, const uint32_t* __restrict__ order,
             const int32_t* __restrict__ nlist, const int32_t* __restrict__ ncount,
             const uint32_t* __restrict__ scanq, const uint32_t* __restrict__ scanq_n,
             uint32_t qblocks, float4* __restrict__ vout,
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
            vout[i] = force_scan_one(params_of<BATCH>(P0, sr, i), i, xp, vp, vs, rr, table, err);
        }
        return;
    }
    const uint32_t t = list_length_order((blockIdx.x - qblocks) * blockDim.x, n, ncount);
    if (t >= n) return;
    const int32_t cnt = ncount[t];
    if (cnt < 0) return;  // in the queue
    const uint32_t i = order[t];
    if (i >= n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    // the particle's own data and result are touched once: streaming loads
    // and stores, so the neighbours' data stay in L2
    const float2 rri = __ldcs(rr + i);
    const ForceSelf me = force_self(P, __ldcs(xp + i), __ldcs(vp + i), rri);
    ForceAcc f = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    // software pipeline: the index of neighbour k+2 and the data of k+1 are
    // in flight while neighbour k is evaluated
    auto index = [&](int32_t k) -> int32_t {
        const int32_t j = k < cnt ? __ldcs(nlist + (size_t)k * n + t) : (int32_t)i;
        if ((uint32_t)j >= n) {
            atomicOr(err, ERR_TABLE_RANGE);
            return (int32_t)i;  // evaluated as self: d = 0, skipped
        }
        return j;
    };
    int32_t jn = index(1);
    int32_t j = index(0);
    float4 q = __ldg(xp + j), vj = __ldg(vs + j);
    float2 rj = __ldg(rr + j);
    for (int32_t k = 0; k < cnt; k++) {
        const int32_t jnn = index(k + 2);
        const float4 qn = __ldg(xp + jn), vn = __ldg(vs + jn);
        const float2 rn = __ldg(rr + jn);
        if constexpr (FAST)
            force_term_fast(P, me, make_float4(q.x, q.y, q.z, rj.x), make_float4(vj.x, vj.y, vj.z, rj.y), f);
        else
            force_term_pre(P, me, q, rj, vj, f);
        q = qn;
        vj = vn;
        rj = rn;
        jn = jnn;
    }
    __stcs(vout + i, force_finish(P, f, __ldcs(vs + i), rri.x));
}

// Density pass of the list shape: the walk of *_simple, plus the list, with
// in-range distances deferred: they go to a
// per-lane list in shared memory and their kernel terms are evaluated
// densely afterwards (in the same order), so the scan loop carries only the
// load, the distance and an append.  (Unrolling the 27-cell walk overflows
// the instruction cache; the walk stays a loop.)
constexpr int DENS_CAP = 32;

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS, 8)
k_density_list(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const int2* __restrict__ table,
                const uint32_t* __restrict__ order, float2* __restrict__ rr,
                int32_t* __restrict__ nlist, int32_t* __restrict__ ncount,
                uint32_t* __restrict__ scanq, uint32_t* __restrict__ scanq_n,
                uint32_t* __restrict__ err) {
    __shared__ float s_dd[DENS_CAP][NBR_THREADS];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = P0.n;
    if (t >= n) return;
    const uint32_t i = order[t];
    if (i >= n) {
        atomicOr(err, ERR_PERM_RANGE);
        return;
    }
    const DevParams P = params_of<BATCH>(P0, sr, i);
    if (P.geo) return;  // k_density_geo
    const float4 sp = xp[i];
    const float h = P.h, m = P.m, skip = P.skip_d2;
    const float off[3] = {PFS_MUL(h, -1.0f), PFS_MUL(h, 0.0f), h};
    uint32_t hx[3], hy[3], hz[3];
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
#pragma unroll
    for (int a = 0; a < 3; a++) {
        hx[a] = (uint32_t)(listing ? cx[1] + a - 1 : cx[a]) * 73856093u;
        hy[a] = (uint32_t)(listing ? cy[1] + a - 1 : cy[a]) * 19349663u;
        hz[a] = (uint32_t)(listing ? cz[1] + a - 1 : cz[a]) * 83492791u;
    }
    float total = 0.0f, total_near = 0.0f;
    int cd = 0;        // deferred density terms in s_dd
    int32_t cnt = 0;   // list entries
    bool list_ok = listing;
#pragma unroll 1
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const bool dens = pickb(dx, vx[0], vx[1], vx[2]) && pickb(dy, vy[0], vy[1], vy[2]) &&
                          pickb(dz, vz[0], vz[1], vz[2]);
        if (dens || listing) {
            const int2 se = __ldg(table + slot_of(P, hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                                                   pick3(dy, hy[0], hy[1], hy[2]) ^
                                                                   pick3(dz, hz[0], hz[1], hz[2]))));
            if (se.x != -1) {
                if (!table_range_ok(se, n)) {
                    atomicOr(err, ERR_TABLE_RANGE);
                    list_ok = false;
                } else {
                    for (int32_t j = se.x; j < se.y; j++) {
                        float d0, d1, d2;
                        const float dd = dist2(__ldg(xp + j), sp, d0, d1, d2);
                        if (in_reach(dd, skip)) {
                            if (dens) {
                                if (cd == DENS_CAP) {
                                    for (int k = 0; k < DENS_CAP; k++)
                                        density_term(s_dd[k][threadIdx.x], h, m, total, total_near);
                                    cd = 0;
                                }
                                s_dd[cd++][threadIdx.x] = dd;
                            }
                            if (listing && j != (int32_t)i) {
                                if (cnt < (int32_t)P.list_cap) __stcs(nlist + (size_t)cnt * n + t, j);
                                cnt++;
                            }
                        }
                    }
                }
            }
        }
    }
    for (int k = 0; k < cd; k++) density_term(s_dd[k][threadIdx.x], h, m, total, total_near);
    const bool scan = !(list_ok && cnt <= (int32_t)P.list_cap);
    ncount[t] = scan ? -1 : cnt;
    rr[i] = density_finish(P, total, total_near);
    const uint32_t active = __activemask();
    const uint32_t want = __ballot_sync(active, scan);
    if (want) {
        const int leader = __ffs(want) - 1;
        const int lane = threadIdx.x & 31;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(scanq_n, (uint32_t)__popc(want));
        base = __shfl_sync(active, base, leader);
        if (scan) scanq[base + __popc(want & ((1u << lane) - 1u))] = t;
    }
}

// ---- flat shape ----------------------------------------------------------------
// Same sums, list and queue as k_density_list, on the flat walk of
// pfs_flat.cuh (warp-uniform control flow; in the list shape branches and
// reconvergence outnumber the arithmetic several times over).  In-range
// distances of cells with an in-box sample point are appended to a per-lane
// buffer whose terms are evaluated in order (all lanes together, once one
// buffer has no room for the next pair, and at the end); list entries are
// written as they are found.  Appends store unconditionally and advance the
// count by the predicate.  A particle whose ranges do not fit the walk's
// stage walks the table from global memory (density_scan_one).
constexpr int FLAT_CAP = 14;  // buffered density terms per lane

template <bool BATCH>
__global__ void __launch_bounds__(NBR_THREADS, BATCH ? 8 : 10)
k_density_flat(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const int2* __restrict__ table,
               const uint32_t* __restrict__ order, float2* __restrict__ rr,
               int32_t* __restrict__ nlist, int32_t* __restrict__ ncount,
               uint32_t* __restrict__ scanq, uint32_t* __restrict__ scanq_n,
               uint32_t* __restrict__ err) {
    static_assert(NBR_THREADS == FLAT_THREADS, "the flat walk's block");
    __shared__ FlatShared S;
    __shared__ float s_dd[FLAT_CAP][NBR_THREADS];  // per thread: deferred terms
    const int tid = threadIdx.x;
    const uint32_t n = P0.n;
    uint32_t key = flat_ranges<BATCH>(P0, sr, xp, table, order, err, S);
    key = flat_sort(key, reinterpret_cast<uint32_t*>(&s_dd[0][0]), S);
    const int src = (int)(key & 127u);
    const int32_t tot = (int32_t)(key >> 7);
    const uint32_t meta = S.meta[src];
    flat_move(src, S);
    const bool live = (meta & FLAT_LIVE) != 0, over = (meta & FLAT_OVER) != 0;
    const uint32_t t = blockIdx.x * NBR_THREADS + (uint32_t)src;
    const uint32_t i = live ? order[t] : 0u;
    const DevParams P = params_of<BATCH>(P0, sr, i);
    const float4 sp = live ? xp[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float h = P.h, m = P.m, skip = P.skip_d2;
    const int32_t self = (int32_t)i;
    float total = 0.0f, total_near = 0.0f;
    // next free slot of this thread's deferred terms (column tid of s_dd)
    float* dp = &s_dd[0][tid];
    float* const dfull = &s_dd[FLAT_CAP - 1][tid];
    int32_t cnt = 0;  // list entries
    const int32_t lcap1 = (int32_t)P.list_cap - 1;
    auto test = [&](const float4 q, int32_t jq, bool fq, bool valid) {
        float d0, d1, d2;
        const float dd = dist2(q, sp, d0, d1, d2);
        const bool in = valid && in_reach(dd, skip);
        *dp = dd;
        dp += (in && fq) ? NBR_THREADS : 0;
        // a list past its capacity keeps overwriting its last row: its count
        // sends the particle to the scan queue, which ignores the list (so do
        // lists of particles that are not listing)
        const bool le = in && jq != self;
        if (le) __stcs(nlist + (size_t)min(cnt, lcap1) * n + t, jq);
        cnt += le ? 1 : 0;
    };
    // all lanes drain their buffers together once one of them has no room
    // for the next pair of candidates
    auto drain_if_full = [&]() {
        if (__any_sync(0xffffffffu, dp >= dfull)) {
            for (int c = 0; c < FLAT_CAP; c++)
                if (&s_dd[c][tid] < dp) density_term(s_dd[c][tid], h, m, total, total_near);
            dp = &s_dd[0][tid];
        }
    };
    flat_walk(S, tot, self, (meta & FLAT_ALLF) != 0, [&](int32_t j) { return __ldg(xp + j); }, test,
              drain_if_full);
    for (const float* e = &s_dd[0][tid]; e < dp; e += NBR_THREADS) density_term(*e, h, m, total, total_near);
    const bool scan = live && (over || !((meta & FLAT_LIST_OK) != 0 && cnt <= (int32_t)P.list_cap));
    if (live) {
        ncount[t] = scan ? -1 : cnt;
        rr[i] = over ? density_scan_one(P, sp, xp, table, err) : density_finish(P, total, total_near);
    }
    flat_enqueue(scan, t, scanq, scanq_n);
}

// ---- grid search (pfs_geo.cuh): one warp per particle ------------------------

// In-range candidates a warp holds per particle (beyond them it walks the
// table ranges instead; same results).
constexpr int GEO_DCAP = 512;
constexpr int GEO_FCAP = 256;
constexpr int FORCE_INCS = 9;

// force_term_pre's per-neighbour increments, in its operation order:
// inc[0..2] pressure, inc[3..5] viscosity, inc[6..8] near pressure; each
// accumulator takes fp += inc[a] then fp += inc[6 + a], fv += inc[3 + a].
// Candidates closer than 1e-7 contribute nothing (all increments +0, which
// leaves a sum that started at +0 unchanged).
__device__ __forceinline__ void force_incr(const DevParams& P, const ForceSelf& me, const float4 q,
                                           const float2 rrj, const float4 vj, float inc[FORCE_INCS]) {
    const float h = P.h, m = P.m;
    float d0, d1, d2;
    const float dd = dist2(q, me.sp, d0, d1, d2);
    const float dist = PFS_SQRT(dd);
    if (fabsf(dist) < 1e-7f) {
#pragma unroll
        for (int c = 0; c < FORCE_INCS; c++) inc[c] = 0.0f;
        return;
    }
    const float dirx = PFS_DIV(d0, dist), diry = PFS_DIV(d1, dist), dirz = PFS_DIV(d2, dist);
    const float slope = PFS_MUL(PFS_SUB(dist, h), P.slope_scale);
    const float dj = rrj.x;
    const float shared = PFS_MUL(PFS_ADD(PFS_MUL(PFS_SUB(dj, P.rho0), P.k), me.my_pressure_term), 0.5f);
    const float coef = PFS_DIV(PFS_MUL(PFS_MUL(shared, slope), m), dj);
    inc[0] = PFS_MUL(coef, dirx);
    inc[1] = PFS_MUL(coef, diry);
    inc[2] = PFS_MUL(coef, dirz);
    const float a = PFS_SUB(h, dist);
    const float a2 = PFS_MUL(a, a);
    const float vcoef = PFS_DIV(PFS_MUL(m, a2), dj);
    inc[3] = PFS_MUL(vcoef, PFS_SUB(vj.x, me.pv.x));
    inc[4] = PFS_MUL(vcoef, PFS_SUB(vj.y, me.pv.y));
    inc[5] = PFS_MUL(vcoef, PFS_SUB(vj.z, me.pv.z));
    const float nnd = rrj.y;
    const float shared_near = PFS_MUL(PFS_ADD(me.near_pressure, PFS_MUL(nnd, P.kn)), 0.5f);
    const float nslope = PFS_MUL(a2, P.near_slope_scale);
    const float ncoef = PFS_DIV(PFS_MUL(PFS_MUL(shared_near, nslope), m), nnd);
    inc[6] = PFS_MUL(ncoef, dirx);
    inc[7] = PFS_MUL(ncoef, diry);
    inc[8] = PFS_MUL(ncoef, dirz);
}

// Accumulator `lane` (0..5: fpx fpy fpz fvx fvy fvz) takes one candidate's
// increments from column k of inc.
__device__ __forceinline__ float force_chain_add(float acc, int lane, const float (*inc)[GEO_FCAP],
                                                 int k) {
    if (lane < 3) return PFS_ADD(PFS_ADD(acc, inc[lane][k]), inc[6 + lane][k]);
    return PFS_ADD(acc, inc[lane][k]);
}

__device__ __forceinline__ bool geo_skip(const DevParams& P0, SceneRef sr, uint32_t i, bool batch) {
    return batch ? !__ldg(&sr.scenes[__ldg(sr.sid + i)].geo) : !P0.geo;
}

// Density pass of the grid-search particles: warp w walks slots w, w + W, ...
// and handles those whose scene uses the grid search.  Same sums, list and
// queue decisions as k_density_list; particles it cannot list go to the
// grid-search queue.  Nine blocks of 24 KB fill an SM's shared memory; the
// register cap of 56 per thread lets the batch form (per-scene parameters)
// keep all nine resident as well.
template <bool BATCH>
__global__ void __launch_bounds__(GEO_WARPS * 32, 9)
k_density_geo(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const int2* __restrict__ table,
              const uint32_t* __restrict__ order, const uint32_t* __restrict__ bucket,
              const uint32_t* __restrict__ brank, const uint32_t* __restrict__ bcount,
              const uint32_t* __restrict__ boffset, uint32_t nblocks, float2* __restrict__ rr,
              int32_t* __restrict__ nlist, int32_t* __restrict__ ncount, uint32_t* __restrict__ scanq,
              uint32_t* __restrict__ scanq_n, uint32_t* __restrict__ err) {
    __shared__ int32_t s_j[GEO_WARPS][GEO_DCAP];
    __shared__ float s_a[GEO_WARPS][GEO_DCAP];
    __shared__ float s_b[GEO_WARPS][GEO_DCAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full = 0xffffffffu, lt = (1u << lane) - 1u;
    int32_t* sj = s_j[w];
    float* sa = s_a[w];
    float* sb = s_b[w];
    const uint32_t n = P0.n;
    for (uint32_t base = warp_take(scanq_n + 2); base < n; base = warp_take(scanq_n + 2))
    for (uint32_t i = base; i < min(base + GEO_CHUNK, n); i++) {
        if (geo_skip(P0, sr, i, BATCH)) continue;
        const DevParams P = params_of<BATCH>(P0, sr, i);
        const float4 sp = xp[i];
        const float h = P.h, skip = P.skip_d2;
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
        // lane d < 27: sample d (z outer, x inner) and its table range
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
                if (se.x != -1 && !table_range_ok(se, n)) {
                    atomicOr(err, ERR_TABLE_RANGE);
                    bad = true;
                    se = make_int2(-1, -1);
                }
            }
        }
        bool list_ok = listing && !__any_sync(full, bad);
        const int m = warp_gather(P, sp.x, sp.y, sp.z, bcount, boffset, order, sj, GEO_DCAP, err,
                                  [&](int32_t j) {
                                      float d0, d1, d2;
                                      return dist2(__ldg(xp + j), sp, d0, d1, d2) < skip;
                                  });
        float total = 0.0f, total_near = 0.0f;
        int32_t cnt = 0;
        const uint32_t t = order_position(i, n, nblocks, bucket, brank, boffset);
        if (m <= GEO_DCAP) {
            warp_sort(sj, m);
            for (int k = lane; k < m; k += 32) {
                float d0, d1, d2;
                const float dd = dist2(__ldg(xp + sj[k]), sp, d0, d1, d2);
                const float a = PFS_SUB(h, PFS_SQRT(dd));
                const float a2 = PFS_MUL(a, a);
                sa[k] = PFS_MUL(P.m, a2);
                sb[k] = PFS_MUL(P.m, PFS_MUL(a2, a));
            }
            int lo = 0, hi = 0;  // this lane's range, as positions in sj
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
                        float acc = lane == 0 ? total : total_near;
                        for (int k = l; k < u; k++) acc = PFS_ADD(acc, src[k]);
                        if (lane == 0)
                            total = acc;
                        else
                            total_near = acc;
                    }
                }
                if (write_list) {
                    for (int base = l; base < u; base += 32) {
                        const int k = base + lane;
                        const int32_t j = k < u ? sj[k] : (int32_t)i;
                        const bool e = j != (int32_t)i;
                        const uint32_t mk = __ballot_sync(full, e);
                        const int32_t pos = cnt + __popc(mk & lt);
                        if (e && pos < (int32_t)P.list_cap && t < n) __stcs(nlist + (size_t)pos * n + t, j);
                        cnt += __popc(mk);
                    }
                }
            }
        } else {
            // too many for the warp's buffer: walk the table ranges in table order
            list_ok = false;
            for (int d = 0; d < 27; d++) {
                const bool dd_ = __shfl_sync(full, dens, d);
                const int32_t r0 = __shfl_sync(full, se.x, d), r1 = __shfl_sync(full, se.y, d);
                if (!dd_ || r0 == -1) continue;
                for (int32_t base = r0; base < r1; base += 32) {
                    const int32_t j = base + lane;
                    bool in = false;
                    if (j < r1) {
                        float d0, d1, d2;
                        const float dd = dist2(__ldg(xp + j), sp, d0, d1, d2);
                        in = dd < skip;
                        if (in) {
                            const float a = PFS_SUB(h, PFS_SQRT(dd));
                            const float a2 = PFS_MUL(a, a);
                            sa[lane] = PFS_MUL(P.m, a2);
                            sb[lane] = PFS_MUL(P.m, PFS_MUL(a2, a));
                        }
                    }
                    uint32_t mk = __ballot_sync(full, in);
                    __syncwarp();
                    if (lane < 2) {
                        const float* src = lane == 0 ? sa : sb;
                        float acc = lane == 0 ? total : total_near;
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1u;
                            acc = PFS_ADD(acc, src[k]);
                        }
                        if (lane == 0)
                            total = acc;
                        else
                            total_near = acc;
                    }
                    __syncwarp();
                }
            }
        }
        total = __shfl_sync(full, total, 0);
        total_near = __shfl_sync(full, total_near, 1);
        if (lane == 0) {
            rr[i] = density_finish(P, total, total_near);
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

// Force pass of the grid-search queue (one warp per queued particle): the 27
// cells around the cell of x*, in-range candidates self excluded, as in
// force_scan_one.
template <bool BATCH>
__global__ void __launch_bounds__(GEO_WARPS * 32)
k_force_geo(DevParams P0, SceneRef sr, const float4* __restrict__ xp, const float4* __restrict__ vp,
            const float4* __restrict__ vs, const float2* __restrict__ rr,
            const int2* __restrict__ table, const uint32_t* __restrict__ order,
            const uint32_t* __restrict__ bcount, const uint32_t* __restrict__ boffset,
            const uint32_t* __restrict__ scanq, uint32_t* __restrict__ scanq_n,
            float4* __restrict__ vout, uint32_t* __restrict__ err) {
    __shared__ int32_t s_j[GEO_WARPS][GEO_FCAP];
    __shared__ float s_inc[GEO_WARPS][FORCE_INCS][GEO_FCAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full = 0xffffffffu;
    int32_t* sj = s_j[w];
    float(*inc)[GEO_FCAP] = s_inc[w];
    const uint32_t n = P0.n;
    const uint32_t total_q = min(scanq_n[1], n);
    for (uint32_t base = warp_take(scanq_n + 3); base < total_q; base = warp_take(scanq_n + 3))
    for (uint32_t q = base; q < min(base + GEO_CHUNK, total_q); q++) {
        const uint32_t i = scanq[n - 1u - q];
        if (i >= n) {
            if (lane == 0) atomicOr(err, ERR_PERM_RANGE);
            continue;
        }
        const DevParams P = params_of<BATCH>(P0, sr, i);
        const float2 rri = rr[i];
        const ForceSelf me = force_self(P, xp[i], vp[i], rri);
        ForceCells cl;
        force_cells(P, me.sp, cl);
        int2 se = make_int2(-1, -1);
        if (lane < 27) {
            const int dz = lane / 9, dy = (lane / 3) % 3, dx = lane % 3;
            se = __ldg(table + slot_of(P, hash_finalize(pick3(dx, cl.hx[0], cl.hx[1], cl.hx[2]) ^
                                                        pick3(dy, cl.hy[0], cl.hy[1], cl.hy[2]) ^
                                                        pick3(dz, cl.hz[0], cl.hz[1], cl.hz[2]))));
            if (se.x != -1 && !table_range_ok(se, n)) {
                atomicOr(err, ERR_TABLE_RANGE);
                se = make_int2(-1, -1);
            }
        }
        const int m = warp_gather(P, me.sp.x, me.sp.y, me.sp.z, bcount, boffset, order, sj, GEO_FCAP,
                                  err, [&](int32_t j) {
                                      if (j == (int32_t)i) return false;
                                      float d0, d1, d2;
                                      return dist2(__ldg(xp + j), me.sp, d0, d1, d2) < P.skip_d2;
                                  });
        float acc = 0.0f;  // lanes 0..5: fpx fpy fpz fvx fvy fvz
        if (m <= GEO_FCAP) {
            warp_sort(sj, m);
            for (int k = lane; k < m; k += 32) {
                const int32_t j = sj[k];
                float v[FORCE_INCS];
                force_incr(P, me, __ldg(xp + j), __ldg(rr + j), __ldg(vs + j), v);
#pragma unroll
                for (int c = 0; c < FORCE_INCS; c++) inc[c][k] = v[c];
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
                    for (int k = l; k < u; k++) acc = force_chain_add(acc, lane, inc, k);
            }
        } else {
            for (int d = 0; d < 27; d++) {
                const int32_t r0 = __shfl_sync(full, se.x, d), r1 = __shfl_sync(full, se.y, d);
                if (r0 == -1) continue;
                for (int32_t base = r0; base < r1; base += 32) {
                    const int32_t j = base + lane;
                    bool in = false;
                    if (j < r1 && j != (int32_t)i) {
                        float d0, d1, d2;
                        in = dist2(__ldg(xp + j), me.sp, d0, d1, d2) < P.skip_d2;
                        if (in) {
                            float v[FORCE_INCS];
                            force_incr(P, me, __ldg(xp + j), __ldg(rr + j), __ldg(vs + j), v);
#pragma unroll
                            for (int c = 0; c < FORCE_INCS; c++) inc[c][lane] = v[c];
                        }
                    }
                    uint32_t mk = __ballot_sync(full, in);
                    __syncwarp();
                    if (lane < 6) {
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1u;
                            acc = force_chain_add(acc, lane, inc, k);
                        }
                    }
                    __syncwarp();
                }
            }
        }
        ForceAcc f;
        f.fpx = __shfl_sync(full, acc, 0);
        f.fpy = __shfl_sync(full, acc, 1);
        f.fpz = __shfl_sync(full, acc, 2);
        f.fvx = __shfl_sync(full, acc, 3);
        f.fvy = __shfl_sync(full, acc, 4);
        f.fvz = __shfl_sync(full, acc, 5);
        if (lane == 0) vout[i] = force_finish(P, f, vs[i], rri.x);
        __syncwarp();
    }
}

// Thread blocks of kernel k (GEO_WARPS warps each) that are resident at once
// on the current device, at most one warp per item: the grid-search kernels
// stride over their items, so a grid beyond one resident wave would leave a
// second wave of whole strides behind the first.
template <class K>
unsigned geo_grid(K kernel, uint32_t items) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, GEO_WARPS * 32, 0);
    const unsigned resident = (unsigned)std::max(1, per_sm) * (unsigned)std::max(1, sms);
    return std::max(1u, std::min(resident, (items + GEO_WARPS - 1) / GEO_WARPS));
}

inline unsigned grid_for(uint32_t n, int threads) { return (n + threads - 1) / threads; }

}  // namespace

// PFS_NBR_VARIANT=simple|slab|list|flat|staged picks the default kernel shape
// of new worlds and batches (all give the same bits); flat when unset.
int nbr_variant() {
    static const int v = [] {
        const char* e = getenv("PFS_NBR_VARIANT");
        if (e && strcmp(e, "simple") == 0) return (int)NBR_SIMPLE;
        if (e && strcmp(e, "slab") == 0) return (int)NBR_COMPACT;
        if (e && strcmp(e, "list") == 0) return (int)NBR_LIST;
        if (e && strcmp(e, "staged") == 0) return (int)NBR_STAGED;
        return (int)NBR_FLAT;
    }();
    return v;
}

// Launch kernel K in its one-world or batch form.
#define PFS_LAUNCH(K, grid, ...)                                          \
    do {                                                                  \
        if (b.sr.scenes)                                                  \
            K<true><<<(grid), NBR_THREADS, 0, s>>>(P, b.sr, __VA_ARGS__);  \
        else                                                              \
            K<false><<<(grid), NBR_THREADS, 0, s>>>(P, b.sr, __VA_ARGS__); \
    } while (0)

cudaError_t launch_density(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, NBR_THREADS);
    if (b.variant == NBR_STAGED && P.staged && !b.sr.scenes) return launch_density_staged(P, b, b.fast != 0, s);
    switch (b.variant) {
        case NBR_SIMPLE:
            PFS_LAUNCH(k_density_simple, g, b.xp, b.table, b.order, b.rr, b.err);
            break;
        case NBR_COMPACT:
            PFS_LAUNCH(k_density_slab, g, b.xp, b.table, b.order, b.rr, b.err);
            break;
        default:
            if (b.variant == NBR_FLAT)
                PFS_LAUNCH(k_density_flat, g, b.xp, b.table, b.order, b.rr, b.nlist, b.ncount, b.scanq,
                           b.scanq_n, b.err);
            else
                PFS_LAUNCH(k_density_list, g, b.xp, b.table, b.order, b.rr, b.nlist, b.ncount, b.scanq,
                           b.scanq_n, b.err);
            if (b.geo_any) {
                if (b.sr.scenes)
                    k_density_geo<true><<<geo_grid(k_density_geo<true>, P.n), GEO_WARPS * 32, 0, s>>>(
                        P, b.sr, b.xp, b.table, b.order, b.bucket, b.brank, b.bcount, b.boffset,
                        b.nblocks, b.rr, b.nlist, b.ncount, b.scanq, b.scanq_n, b.err);
                else
                    k_density_geo<false><<<geo_grid(k_density_geo<false>, P.n), GEO_WARPS * 32, 0, s>>>(
                        P, b.sr, b.xp, b.table, b.order, b.bucket, b.brank, b.bcount, b.boffset,
                        b.nblocks, b.rr, b.nlist, b.ncount, b.scanq, b.scanq_n, b.err);
            }
    }
    return cudaGetLastError();
}

cudaError_t launch_force(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    const unsigned g = grid_for(P.n, NBR_THREADS);
    switch (b.variant) {
        case NBR_SIMPLE:
            PFS_LAUNCH(k_force_simple, g, b.xp, b.vp, b.vs, b.rr, b.table, b.order, b.v, b.err);
            break;
        case NBR_COMPACT:
            PFS_LAUNCH(k_force_slab, g, b.xp, b.vp, b.vs, b.rr, b.table, b.order, b.v, b.err);
            break;
        default: {
            // one queue thread per possible entry: dense scenes can send most
            // particles to the queue (lists overflow), sparse ones very few;
            // surplus queue blocks exit at once
            const unsigned qb = g;
            // the fast form sums the listed terms with fused arithmetic
            auto kf = b.sr.scenes ? (b.fast ? k_force_list<true, true> : k_force_list<true, false>)
                                  : (b.fast ? k_force_list<false, true> : k_force_list<false, false>);
            kf<<<qb + g, NBR_THREADS, 0, s>>>(P, b.sr, b.xp, b.vp, b.vs, b.rr, b.table, b.order, b.nlist,
                                              b.ncount, b.scanq, b.scanq_n, qb, b.v, b.err);
            if (b.geo_any) {
                if (b.sr.scenes)
                    k_force_geo<true><<<geo_grid(k_force_geo<true>, P.n), GEO_WARPS * 32, 0, s>>>(
                        P, b.sr, b.xp, b.vp, b.vs, b.rr, b.table, b.order, b.bcount, b.boffset,
                        b.scanq, b.scanq_n, b.v, b.err);
                else
                    k_force_geo<false><<<geo_grid(k_force_geo<false>, P.n), GEO_WARPS * 32, 0, s>>>(
                        P, b.sr, b.xp, b.vp, b.vs, b.rr, b.table, b.order, b.bcount, b.boffset,
                        b.scanq, b.scanq_n, b.v, b.err);
            }
        }
    }
    return cudaGetLastError();
}

#undef PFS_LAUNCH

}  // namespace pfs
