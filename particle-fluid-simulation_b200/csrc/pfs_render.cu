// pfs_render.cu — volumetric rendering of a world's state into a headless
// RGBA buffer: the reference's calculateLightVolume.comp (:193-219) and
// volumetricFluid.comp (:196-263), which it runs as compute shaders over the
// density map (pfs_density_map.cu).
//
// texture() of the reference's sampler (linear, clamp to edge, normalised
// coordinates; image.c:134-164) is restated as float trilinear interpolation
// in a fixed term order (tex3d), and every other float operation is one IEEE
// round-to-nearest operation in the shaders' order, so results equal the
// oracle's up to expf, whose device and host versions may differ in the last
// bits.
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int RENDER_THREADS = 256;

// Trilinear sample of an x-fastest float image of dims (W, H, D) at
// normalised uvw, with the oracle's term order (pfso_texture3d).
__device__ __forceinline__ float tex3d(const float* __restrict__ img, int3 d, float u0, float u1,
                                       float u2) {
    const float uu[3] = {u0, u1, u2};
    const int32_t dd[3] = {d.x, d.y, d.z};
    int32_t i0[3], i1[3];
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float u = PFS_SUB(PFS_MUL(uu[a], (float)dd[a]), 0.5f);
        const float fl = floorf(u);
        f[a] = PFS_SUB(u, fl);
        const int32_t k = __float2int_rz(fl);  // NaN -> 0, out of range saturates
        const int32_t top = dd[a] - 1;
        i0[a] = min(max(k, 0), top);
        const int32_t k1 = k == INT32_MAX ? k : k + 1;
        i1[a] = min(max(k1, 0), top);
    }
    const int64_t W = d.x, H = d.y;
    auto T = [&](int32_t x, int32_t y, int32_t z) { return __ldg(img + ((int64_t)z * H + y) * W + x); };
    const float a0 = PFS_SUB(1.0f, f[0]), a1 = f[0], b0 = PFS_SUB(1.0f, f[1]), b1 = f[1],
                c0 = PFS_SUB(1.0f, f[2]), c1 = f[2];
    float r = 0.0f;
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a0, b0), c0), T(i0[0], i0[1], i0[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a1, b0), c0), T(i1[0], i0[1], i0[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a0, b1), c0), T(i0[0], i1[1], i0[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a1, b1), c0), T(i1[0], i1[1], i0[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a0, b0), c1), T(i0[0], i0[1], i1[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a1, b0), c1), T(i1[0], i0[1], i1[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a0, b1), c1), T(i0[0], i1[1], i1[2])));
    r = PFS_ADD(r, PFS_MUL(PFS_MUL(PFS_MUL(a1, b1), c1), T(i1[0], i1[1], i1[2])));
    return r;
}

// intersectVolume: slab test, march interval [max(tNear + pad_near, 0), tFar + pad_far].
__device__ __forceinline__ bool ray_box(const DevParams& P, float3 o, float3 d, float pad_near,
                                        float pad_far, float* t0, float* t1) {
    const float mn[3] = {P.minx, P.miny, P.minz}, mx[3] = {P.maxx, P.maxy, P.maxz};
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    float tn[3], tf[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float inv = PFS_DIV(1.0f, dd[a]);
        const float ta = PFS_MUL(PFS_SUB(mn[a], oo[a]), inv), tb = PFS_MUL(PFS_SUB(mx[a], oo[a]), inv);
        tn[a] = (tb < ta) ? tb : ta;
        tf[a] = (ta < tb) ? tb : ta;
    }
    const float m = (tn[0] < tn[1]) ? tn[1] : tn[0];
    const float t_near = (m < tn[2]) ? tn[2] : m;
    const float q = (tf[1] < tf[0]) ? tf[1] : tf[0];
    const float t_far = (tf[2] < q) ? tf[2] : q;
    if (!(t_near <= t_far && t_far >= 0.0f)) return false;
    const float a = PFS_ADD(t_near, pad_near);
    *t0 = (a < 0.0f) ? 0.0f : a;
    *t1 = PFS_ADD(t_far, pad_far);
    return true;
}

__global__ void __launch_bounds__(RENDER_THREADS)
k_light_volume(DevParams P, const float* __restrict__ dmap, int3 dd, float ls, float3 sun, int3 ld,
               float* __restrict__ out) {
    const uint64_t nx = (uint64_t)ld.x, ny = (uint64_t)ld.y, nz = (uint64_t)ld.z;
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nx * ny * nz) return;
    const int32_t vx = (int32_t)(idx % nx), vy = (int32_t)((idx / nx) % ny), vz = (int32_t)(idx / (nx * ny));
    out[idx] = 0.0f;
    const float sx = PFS_SUB(P.maxx, P.minx), sy = PFS_SUB(P.maxy, P.miny), sz = PFS_SUB(P.maxz, P.minz);
    if ((float)vx > sx || (float)vy > sy || (float)vz > sz) return;
    const float3 c = make_float3(PFS_ADD(P.minx, PFS_MUL(PFS_ADD((float)vx, 0.5f), ls)),
                                 PFS_ADD(P.miny, PFS_MUL(PFS_ADD((float)vy, 0.5f), ls)),
                                 PFS_ADD(P.minz, PFS_MUL(PFS_ADD((float)vz, 0.5f), ls)));
    float t0, t1;
    if (!ray_box(P, c, sun, -1.0f, 1.0f, &t0, &t1)) return;
    float acc = 0.0f;
    for (float t = (t0 < 0.0f) ? 0.0f : t0; t < t1; t = PFS_ADD(t, ls)) {
        const float u0 = PFS_DIV(PFS_SUB(PFS_ADD(c.x, PFS_MUL(t, sun.x)), P.minx), sx);
        const float u1 = PFS_DIV(PFS_SUB(PFS_ADD(c.y, PFS_MUL(t, sun.y)), P.miny), sy);
        const float u2 = PFS_DIV(PFS_SUB(PFS_ADD(c.z, PFS_MUL(t, sun.z)), P.minz), sz);
        acc = PFS_ADD(acc, PFS_MUL(tex3d(dmap, dd, u0, u1, u2), ls));
    }
    out[idx] = acc;
}

struct ViewArgs {
    float3 pos, fwd, right, up;
    float half_h, half_w, step;
    float3 ext;  // normalize(extinctionCoefficients)
};

__device__ __forceinline__ float clamp01(float w) {
    const float m = (w < 0.0f) ? 0.0f : w;
    return (1.0f < m) ? 1.0f : m;
}

__global__ void __launch_bounds__(RENDER_THREADS)
k_volumetric(DevParams P, const float* __restrict__ dmap, int3 dd, const float* __restrict__ lvol,
             int3 ld, ViewArgs V, uint32_t width, uint32_t height, float4* __restrict__ rgba) {
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (uint64_t)width * height) return;
    const int32_t x = (int32_t)(idx % width), y = (int32_t)(idx / width);
    const float px = PFS_ADD((float)x, 0.5f), py = PFS_ADD((float)y, 0.5f);
    const float u = PFS_SUB(PFS_MUL(PFS_DIV(px, (float)width), 2.0f), 1.0f);
    const float v = PFS_SUB(PFS_MUL(PFS_DIV(py, (float)height), 2.0f), 1.0f);
    const float uw = PFS_MUL(u, V.half_w), vh = PFS_MUL(v, V.half_h);
    float3 d;
    d.x = PFS_SUB(PFS_SUB(PFS_ADD(PFS_ADD(V.pos.x, V.fwd.x), PFS_MUL(uw, V.right.x)), PFS_MUL(vh, V.up.x)), V.pos.x);
    d.y = PFS_SUB(PFS_SUB(PFS_ADD(PFS_ADD(V.pos.y, V.fwd.y), PFS_MUL(uw, V.right.y)), PFS_MUL(vh, V.up.y)), V.pos.y);
    d.z = PFS_SUB(PFS_SUB(PFS_ADD(PFS_ADD(V.pos.z, V.fwd.z), PFS_MUL(uw, V.right.z)), PFS_MUL(vh, V.up.z)), V.pos.z);
    const float dl = PFS_SQRT(PFS_ADD(PFS_ADD(PFS_MUL(d.x, d.x), PFS_MUL(d.y, d.y)), PFS_MUL(d.z, d.z)));
    d.x = PFS_DIV(d.x, dl);
    d.y = PFS_DIV(d.y, dl);
    d.z = PFS_DIV(d.z, dl);
    const float sx = PFS_SUB(P.maxx, P.minx), sy = PFS_SUB(P.maxy, P.miny), sz = PFS_SUB(P.maxz, P.minz);
    const float amb[3] = {0.529f, 0.808f, 0.922f};
    const float ext[3] = {V.ext.x, V.ext.y, V.ext.z};
    float light[3] = {0.0f, 0.0f, 0.0f};
    float t0, t1;
    if (ray_box(P, V.pos, d, 1.0f, -1.0f, &t0, &t1)) {
        float view = 0.0f;
        for (float t = PFS_ADD((t0 < 0.0f) ? 0.0f : t0, V.step); t < PFS_SUB(t1, V.step); t = PFS_ADD(t, V.step)) {
            const float w0 = clamp01(PFS_DIV(PFS_SUB(PFS_ADD(V.pos.x, PFS_MUL(t, d.x)), P.minx), sx));
            const float w1 = clamp01(PFS_DIV(PFS_SUB(PFS_ADD(V.pos.y, PFS_MUL(t, d.y)), P.miny), sy));
            const float w2 = clamp01(PFS_DIV(PFS_SUB(PFS_ADD(V.pos.z, PFS_MUL(t, d.z)), P.minz), sz));
            const float dens = PFS_MUL(tex3d(dmap, dd, w0, w1, w2), 0.05f);
            view = PFS_ADD(view, PFS_MUL(dens, V.step));
            const float sun = tex3d(lvol, ld, w0, w1, w2);
            float in[3], vt[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const float tr = PFS_MUL(expf(PFS_MUL(-sun, ext[a])), amb[a]);
                in[a] = PFS_MUL(PFS_MUL(tr, dens), ext[a]);
                vt[a] = expf(PFS_MUL(-view, ext[a]));
            }
            const float mx = (vt[1] < vt[2]) ? vt[2] : vt[1];
            const float mm = (vt[0] < mx) ? mx : vt[0];
            if (mm < 0.01f) break;
#pragma unroll
            for (int a = 0; a < 3; a++) light[a] = PFS_ADD(light[a], PFS_MUL(in[a], vt[a]));
        }
        if (light[0] > 0.00001f && light[1] > 0.00001f && light[2] > 0.00001f)
#pragma unroll
            for (int a = 0; a < 3; a++) light[a] = PFS_ADD(light[a], 0.05f);
    }
    rgba[idx] = make_float4(light[0], light[1], light[2], 1.0f);
}

}  // namespace

cudaError_t launch_light_volume(const DevParams& P, const float* dmap, const int32_t ddims[3],
                                float light_step, const float sun[3], const int32_t ldims[3],
                                float* out, cudaStream_t s) {
    const uint64_t n = (uint64_t)ldims[0] * ldims[1] * ldims[2];
    if (n == 0) return cudaSuccess;
    k_light_volume<<<(unsigned)((n + RENDER_THREADS - 1) / RENDER_THREADS), RENDER_THREADS, 0, s>>>(
        P, dmap, make_int3(ddims[0], ddims[1], ddims[2]), light_step, make_float3(sun[0], sun[1], sun[2]),
        make_int3(ldims[0], ldims[1], ldims[2]), out);
    return cudaGetLastError();
}

cudaError_t launch_volumetric(const DevParams& P, const float* dmap, const int32_t ddims[3],
                              const float* lvol, const int32_t ldims[3], const float cam[12],
                              float half_h, float half_w, float step, const float ext[3],
                              uint32_t width, uint32_t height, float* rgba, cudaStream_t s) {
    const uint64_t n = (uint64_t)width * height;
    if (n == 0) return cudaSuccess;
    ViewArgs V;
    V.pos = make_float3(cam[0], cam[1], cam[2]);
    V.fwd = make_float3(cam[3], cam[4], cam[5]);
    V.right = make_float3(cam[6], cam[7], cam[8]);
    V.up = make_float3(cam[9], cam[10], cam[11]);
    V.half_h = half_h;
    V.half_w = half_w;
    V.step = step;
    V.ext = make_float3(ext[0], ext[1], ext[2]);
    k_volumetric<<<(unsigned)((n + RENDER_THREADS - 1) / RENDER_THREADS), RENDER_THREADS, 0, s>>>(
        P, dmap, make_int3(ddims[0], ddims[1], ddims[2]), lvol, make_int3(ldims[0], ldims[1], ldims[2]),
        V, width, height, reinterpret_cast<float4*>(rgba));
    return cudaGetLastError();
}

}  // namespace pfs
