// pfs_density_map.cu — density map of a world's state into a headless float
// grid: the reference's updateDensityMap.comp (:93-147), which fills the 3-D
// image its ray-marching renderers sample.
//
// One thread per voxel of the image the reference allocates
// (renderer.c:774-781): the cell of the voxel centre ((-1,-1,-1) outside the
// box), the 27 cells around it in the shader's order (z outer, x inner), each
// skipped when out of bounds by the shader's voxel rule, and over the table
// range of each cell's key the smoothing kernel m (h - d)^2 of every position
// with d^2 < h^2, divided by the volume.  Every float operation is one IEEE
// round-to-nearest operation in the shader's order, so the map equals the
// oracle's bit for bit.  The table of the last sort is rebuilt from its
// sorted keys for the call (the step's integrate clears it) and cleared again.
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int MAP_THREADS = 256;

// outOfBounds (updateDensityMap.comp:93-96): negative, beyond the extent, or
// the far corner itself.
__device__ __forceinline__ bool map_out(int32_t x, int32_t y, int32_t z, int3 m) {
    if (x < 0 || y < 0 || z < 0) return true;
    if (x > m.x || y > m.y || z > m.z) return true;
    return x == m.x && y == m.y && z == m.z;
}

__global__ void __launch_bounds__(MAP_THREADS)
k_table_runs(uint32_t n, const uint32_t* __restrict__ skeys, int2* __restrict__ table, int set) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t k = skeys[s];
    if (k >= n) return;
    const bool head = (s == 0) || (skeys[s - 1] != k);
    const bool tail = (s == n - 1) || (skeys[s + 1] != k);
    if (!set) {
        if (head) table[k] = make_int2(-1, -1);
        return;
    }
    if (head) table[k].x = (int32_t)s;
    if (tail) table[k].y = (int32_t)(s + 1);
}

__global__ void __launch_bounds__(MAP_THREADS)
k_density_map(DevParams P, float cs, int3 img, int3 m, const float4* __restrict__ x,
              const int2* __restrict__ table, float* __restrict__ out, uint32_t* __restrict__ err) {
    const uint64_t nx = (uint64_t)img.x, ny = (uint64_t)img.y, nz = (uint64_t)img.z;
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nx * ny * nz) return;
    const int32_t vx = (int32_t)(idx % nx), vy = (int32_t)((idx / nx) % ny), vz = (int32_t)(idx / (nx * ny));
    if (map_out(vx, vy, vz, m)) {
        out[idx] = 0.0f;  // skipped by the shader
        return;
    }
    const float h = P.h;
    const float cxp = PFS_ADD(P.minx, PFS_MUL(PFS_ADD((float)vx, 0.5f), cs));
    const float cyp = PFS_ADD(P.miny, PFS_MUL(PFS_ADD((float)vy, 0.5f), cs));
    const float czp = PFS_ADD(P.minz, PFS_MUL(PFS_ADD((float)vz, 0.5f), cs));
    int32_t c0 = -1, c1 = -1, c2 = -1;
    if (!(cxp < P.minx || cyp < P.miny || czp < P.minz || cxp > P.maxx || cyp > P.maxy || czp > P.maxz)) {
        c0 = cell_coord(cxp, P.minx, h);
        c1 = cell_coord(cyp, P.miny, h);
        c2 = cell_coord(czp, P.minz, h);
    }
    const uint32_t n = P.n;
    float density = 0.0f;
#pragma unroll 1
    for (int q = 0; q < 27; q++) {
        const int32_t kx = c0 + q % 3 - 1, ky = c1 + (q / 3) % 3 - 1, kz = c2 + q / 9 - 1;
        if (map_out(kx, ky, kz, m)) continue;
        const int2 se = __ldg(table + slot_of(P, cell_hash((uint32_t)kx, (uint32_t)ky, (uint32_t)kz)));
        if (se.x == -1) continue;
        if (se.x < 0 || se.y > (int32_t)n || se.x > se.y) {
            atomicOr(err, ERR_TABLE_RANGE);
            continue;
        }
        for (int32_t i = se.x; i < se.y; i++) {
            const float4 p = __ldg(x + i);
            const float d0 = PFS_SUB(cxp, p.x), d1 = PFS_SUB(cyp, p.y), d2 = PFS_SUB(czp, p.z);
            const float dist2 = PFS_ADD(PFS_ADD(PFS_MUL(d0, d0), PFS_MUL(d1, d1)), PFS_MUL(d2, d2));
            if (dist2 < P.r2) {
                const float dist = PFS_SQRT(dist2);
                const float k = dist >= h ? 0.0f : PFS_MUL(PFS_SUB(h, dist), PFS_SUB(h, dist));
                density = PFS_ADD(density, PFS_MUL(P.m, k));
            }
        }
    }
    density = PFS_MUL(density, 1.0f);
    out[idx] = PFS_DIV(density, P.volume);
}

}  // namespace

cudaError_t launch_density_map(const DevParams& P, const StepBuffers& b, float cell_size,
                               const int32_t image[3], const int32_t bound[3], float* out,
                               cudaStream_t s) {
    const uint32_t n = P.n;
    if (n == 0) return cudaSuccess;
    const unsigned g = (n + MAP_THREADS - 1) / MAP_THREADS;
    k_table_runs<<<g, MAP_THREADS, 0, s>>>(n, b.skeys, b.table, 1);
    const int3 img = make_int3(image[0], image[1], image[2]);
    const int3 m = make_int3(bound[0], bound[1], bound[2]);
    const uint64_t voxels = (uint64_t)img.x * (uint64_t)img.y * (uint64_t)img.z;
    if (voxels)
        k_density_map<<<(unsigned)((voxels + MAP_THREADS - 1) / MAP_THREADS), MAP_THREADS, 0, s>>>(
            P, cell_size, img, m, b.x, b.table, out, b.err);
    k_table_runs<<<g, MAP_THREADS, 0, s>>>(n, b.skeys, b.table, 0);
    return cudaGetLastError();
}

}  // namespace pfs
