// pfs_step.cu — FP32 SPH substep kernels (plain form).
//
// Data flow of one substep (reference dispatch order commands.c:193-402):
//   keys (from the integrate of the previous substep, or k_keys)
//   -> radix sort -> (skeys, perm)
//   -> k_reorder:   xs, vs = gather(x, v, perm); xp, vp = predict(xs, vs);
//                   table[skey] = (run start, run end)
//   -> k_density:   rr = (density, near density) from xp and the table
//   -> k_force:     v  = vs + F / density * dt        (Jacobi: reads vs)
//   -> k_integrate: x, v = integrate(xs, v); keys = key(x); clear the table
//                   slots this substep set
// Predict is per particle, so running it on the gathered state equals the
// reference's predict-then-scatter (predictPositions.comp, scatterPass.comp).
// The state stays in sort order between substeps, as the reference's
// ping-pong buffers do.
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_sort.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int ELEM_THREADS = 256;
constexpr int NBR_THREADS = 128;

__global__ void __launch_bounds__(ELEM_THREADS)
k_keys(DevParams P, const float4* __restrict__ x, uint32_t* __restrict__ keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
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
__global__ void __launch_bounds__(ELEM_THREADS)
k_reorder(DevParams P, const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ perm,
          const float4* __restrict__ x, const float4* __restrict__ v,
          const uint32_t* __restrict__ ids, float4* __restrict__ xs, float4* __restrict__ vs,
          float4* __restrict__ xp, float4* __restrict__ vp, uint32_t* __restrict__ ids_s,
          int2* __restrict__ table, uint32_t* __restrict__ err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = P.n;
    if (s >= n) return;
    const uint32_t p = perm[s];
    const uint32_t k = skeys[s];
    if (p >= n || k > P.mask) {
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
    if (ids) ids_s[s] = ids[p];
    const bool head = (s == 0) || (skeys[s - 1] != k);
    const bool tail = (s == n - 1) || (skeys[s + 1] != k);
    if (head) table[k].x = (int32_t)s;
    if (tail) table[k].y = (int32_t)(s + 1);
}

__device__ __forceinline__ uint32_t pick3(int i, uint32_t a, uint32_t b, uint32_t c) {
    return i == 0 ? a : (i == 1 ? b : c);
}

// calculateDensities.comp:96-153.  One thread per sorted particle, the 27
// sample-point cells in the reference's z-outer / x-inner order, candidates
// in table order: the float sums are taken in exactly the reference's order.
// Candidates with d2 >= skip_d2 (distance >= h) add an exact +0 in the
// reference and are skipped here.
__global__ void __launch_bounds__(NBR_THREADS)
k_density(DevParams P, const float4* __restrict__ xp, const int2* __restrict__ table,
          float2* __restrict__ rr, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const float4 sp = xp[i];
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
    float total = 0.0f, total_near = 0.0f;
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const bool ok = (dx == 0 ? vx[0] : dx == 1 ? vx[1] : vx[2]) &&
                        (dy == 0 ? vy[0] : dy == 1 ? vy[1] : vy[2]) &&
                        (dz == 0 ? vz[0] : dz == 1 ? vz[1] : vz[2]);
        if (!ok) continue;
        const uint32_t key = hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                           pick3(dy, hy[0], hy[1], hy[2]) ^
                                           pick3(dz, hz[0], hz[1], hz[2])) & P.mask;
        const int2 se = __ldg(table + key);
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)P.n || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            const float4 q = __ldg(xp + j);
            const float d0 = PFS_SUB(q.x, sp.x), d1 = PFS_SUB(q.y, sp.y), d2 = PFS_SUB(q.z, sp.z);
            const float dd = PFS_ADD(PFS_ADD(PFS_MUL(d0, d0), PFS_MUL(d1, d1)), PFS_MUL(d2, d2));
            if (dd >= P.skip_d2) continue;
            const float a = PFS_SUB(h, PFS_SQRT(dd));
            const float a2 = PFS_MUL(a, a);
            total = PFS_ADD(total, PFS_MUL(m, a2));
            total_near = PFS_ADD(total_near, PFS_MUL(m, PFS_MUL(a2, a)));
        }
    }
    const float d = PFS_DIV(total, P.volume);
    const float nd = PFS_MUL(total_near, P.near_inv);
    rr[i] = make_float2((0.01f < d) ? d : 0.01f, (0.01f < nd) ? nd : 0.01f);
}

// applyPressureAndViscosityForce.comp:121-183.  27 cell offsets around the
// cell of x*, candidates in table order, reference expression order.
// Neighbour velocities come from vs (pre-update, Jacobi), the result goes to
// v.  Candidates with d2 >= skip_d2 have distance >= h, where slope,
// viscosity and near-pressure kernels are all zero; their exact +-0
// contributions leave the (never negative-zero) sums unchanged and are
// skipped.  That test also covers the reference's d2 > h^2 cut, since
// skip_d2 <= h*h.
__global__ void __launch_bounds__(NBR_THREADS)
k_force(DevParams P, const float4* __restrict__ xp, const float4* __restrict__ vp,
        const float4* __restrict__ vs, const float2* __restrict__ rr,
        const int2* __restrict__ table, float4* __restrict__ vout, uint32_t* __restrict__ err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const float4 sp = xp[i];
    const float4 pv = vp[i];
    const float2 rri = rr[i];
    const float h = P.h, m = P.m, rho0 = P.rho0, k = P.k, kn = P.kn;
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
    const float my_pressure_term = PFS_MUL(PFS_SUB(my_density, rho0), k);
    const float near_pressure = PFS_MUL(rri.y, kn);
    float fpx = 0.0f, fpy = 0.0f, fpz = 0.0f, fvx = 0.0f, fvy = 0.0f, fvz = 0.0f;
    for (int c = 0; c < 27; c++) {
        const int dz = c / 9, dy = (c / 3) % 3, dx = c % 3;
        const uint32_t key = hash_finalize(pick3(dx, hx[0], hx[1], hx[2]) ^
                                           pick3(dy, hy[0], hy[1], hy[2]) ^
                                           pick3(dz, hz[0], hz[1], hz[2])) & P.mask;
        const int2 se = __ldg(table + key);
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)P.n || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t j = se.x; j < se.y; j++) {
            if (j == (int32_t)i) continue;
            const float4 q = __ldg(xp + j);
            const float d0 = PFS_SUB(q.x, sp.x), d1 = PFS_SUB(q.y, sp.y), d2 = PFS_SUB(q.z, sp.z);
            const float dd = PFS_ADD(PFS_ADD(PFS_MUL(d0, d0), PFS_MUL(d1, d1)), PFS_MUL(d2, d2));
            if (dd >= P.skip_d2) continue;
            const float dist = PFS_SQRT(dd);
            if (fabsf(dist) < 1e-7f) continue;
            const float dirx = PFS_DIV(d0, dist), diry = PFS_DIV(d1, dist), dirz = PFS_DIV(d2, dist);
            const float slope = PFS_MUL(PFS_SUB(dist, h), P.slope_scale);
            const float2 rrj = __ldg(rr + j);
            const float dj = rrj.x;
            const float shared = PFS_DIV(PFS_ADD(PFS_MUL(PFS_SUB(dj, rho0), k), my_pressure_term), 2.0f);
            const float coef = PFS_DIV(PFS_MUL(PFS_MUL(shared, slope), m), dj);
            fpx = PFS_ADD(fpx, PFS_MUL(coef, dirx));
            fpy = PFS_ADD(fpy, PFS_MUL(coef, diry));
            fpz = PFS_ADD(fpz, PFS_MUL(coef, dirz));
            const float a = PFS_SUB(h, dist);
            const float a2 = PFS_MUL(a, a);
            const float vcoef = PFS_DIV(PFS_MUL(m, a2), dj);
            const float4 vj = __ldg(vs + j);
            fvx = PFS_ADD(fvx, PFS_MUL(vcoef, PFS_SUB(vj.x, pv.x)));
            fvy = PFS_ADD(fvy, PFS_MUL(vcoef, PFS_SUB(vj.y, pv.y)));
            fvz = PFS_ADD(fvz, PFS_MUL(vcoef, PFS_SUB(vj.z, pv.z)));
            const float nnd = rrj.y;
            const float shared_near = PFS_DIV(PFS_ADD(near_pressure, PFS_MUL(nnd, kn)), 2.0f);
            const float nslope = PFS_MUL(a2, P.near_slope_scale);
            const float ncoef = PFS_DIV(PFS_MUL(PFS_MUL(shared_near, nslope), m), nnd);
            fpx = PFS_ADD(fpx, PFS_MUL(ncoef, dirx));
            fpy = PFS_ADD(fpy, PFS_MUL(ncoef, diry));
            fpz = PFS_ADD(fpz, PFS_MUL(ncoef, dirz));
        }
    }
    const float4 vi = vs[i];
    const float tx = PFS_ADD(PFS_ADD(fpx, PFS_MUL(P.visc, fvx)), 0.0f);
    const float ty = PFS_ADD(PFS_ADD(fpy, PFS_MUL(P.visc, fvy)), 0.0f);
    const float tz = PFS_ADD(PFS_ADD(fpz, PFS_MUL(P.visc, fvz)), 0.0f);
    vout[i] = make_float4(PFS_ADD(vi.x, PFS_MUL(PFS_DIV(tx, my_density), P.dt)),
                          PFS_ADD(vi.y, PFS_MUL(PFS_DIV(ty, my_density), P.dt)),
                          PFS_ADD(vi.z, PFS_MUL(PFS_DIV(tz, my_density), P.dt)),
                          PFS_ADD(vi.w, 1.0f));
}

// updateVelocities.comp:71-141 + the next substep's updateCellEntries
// (keys of the integrated positions) + reset of the table slots this
// substep's run heads set, so the next table starts empty without a full
// clear.  Slot s is read only by itself here, so x/v update in place.
__global__ void __launch_bounds__(ELEM_THREADS)
k_integrate(DevParams P, const float4* __restrict__ xs, float4* __restrict__ x,
            float4* __restrict__ v, uint32_t* __restrict__ keys,
            const uint32_t* __restrict__ skeys, int2* __restrict__ table,
            const uint32_t* __restrict__ ids_s, uint32_t* __restrict__ ids,
            float4* __restrict__ color) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
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
    if (k <= P.mask && (i == 0 || skeys[i - 1] != k)) table[k] = make_int2(-1, -1);
}

inline unsigned grid_for(uint32_t n, int threads) { return (n + threads - 1) / threads; }

}  // namespace

cudaError_t launch_keys(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_keys<<<grid_for(P.n, ELEM_THREADS), ELEM_THREADS, 0, s>>>(P, b.x, b.keys);
    return cudaGetLastError();
}

cudaError_t launch_table_clear(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_table_clear<<<grid_for(P.n, ELEM_THREADS), ELEM_THREADS, 0, s>>>(P.n, b.table);
    return cudaGetLastError();
}

cudaError_t launch_sort(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    return sort_pairs(b.keys, P.n, sort_key_bits(P.n), b.skeys, b.perm, b.keys_tmp, b.vals_tmp,
                      b.hist, b.digit_total, b.err, s);
}

cudaError_t launch_reorder(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_reorder<<<grid_for(P.n, ELEM_THREADS), ELEM_THREADS, 0, s>>>(
        P, b.skeys, b.perm, b.x, b.v, b.ids, b.xs, b.vs, b.xp, b.vp, b.ids_s, b.table, b.err);
    return cudaGetLastError();
}

cudaError_t launch_density(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_density<<<grid_for(P.n, NBR_THREADS), NBR_THREADS, 0, s>>>(P, b.xp, b.table, b.rr, b.err);
    return cudaGetLastError();
}

cudaError_t launch_force(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_force<<<grid_for(P.n, NBR_THREADS), NBR_THREADS, 0, s>>>(P, b.xp, b.vp, b.vs, b.rr, b.table,
                                                                b.v, b.err);
    return cudaGetLastError();
}

cudaError_t launch_integrate(const DevParams& P, const StepBuffers& b, cudaStream_t s) {
    if (P.n == 0) return cudaSuccess;
    k_integrate<<<grid_for(P.n, ELEM_THREADS), ELEM_THREADS, 0, s>>>(
        P, b.xs, b.x, b.v, b.keys, b.skeys, b.table, b.ids_s, b.ids, b.color);
    return cudaGetLastError();
}

int substep_launches(uint32_t n) { return n == 0 ? 0 : sort_launches(n) + 4; }

}  // namespace pfs
