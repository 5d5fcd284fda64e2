// pfs_render.cu — ray-marched rendering of a world's state into a headless
// RGBA buffer: the reference's volumetric mode, calculateLightVolume.comp
// (:193-219) and volumetricFluid.comp (:196-263), and its refractive mode,
// properFluid.comp (:151-614), which it runs as compute shaders over the
// density map (pfs_density_map.cu).
//
// texture() of the reference's sampler (linear, clamp to edge, normalised
// coordinates; image.c:134-164) is restated as float trilinear interpolation
// in a fixed term order (tex3d), and every other float operation is one IEEE
// round-to-nearest operation in the shaders' order, so results equal the
// oracle's up to expf and powf, whose device and host versions may differ in
// the last bits.
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

// ---- refractive mode (properFluid.comp) --------------------------------------
// GLSL built-ins by their specification formulas, left to right (the oracle's
// definitions): dot, normalize = v / sqrt(dot(v, v)), smoothstep, reflect,
// refract; the environment is white (environmentLight returns vec3(1) before
// its floor and sky code).

__device__ __forceinline__ float dot3(float3 a, float3 b) {
    return PFS_ADD(PFS_ADD(PFS_MUL(a.x, b.x), PFS_MUL(a.y, b.y)), PFS_MUL(a.z, b.z));
}
__device__ __forceinline__ float3 normalize3(float3 v) {
    const float l = PFS_SQRT(dot3(v, v));
    return make_float3(PFS_DIV(v.x, l), PFS_DIV(v.y, l), PFS_DIV(v.z, l));
}
__device__ __forceinline__ float gmin(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return (x < y) ? y : x; }
__device__ __forceinline__ float gclamp(float x, float a, float b) { return gmin(gmax(x, a), b); }
__device__ __forceinline__ float gsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ float smoothstep(float e0, float e1, float x) {
    const float t = gclamp(PFS_DIV(PFS_SUB(x, e0), PFS_SUB(e1, e0)), 0.0f, 1.0f);
    return PFS_MUL(PFS_MUL(t, t), PFS_SUB(3.0f, PFS_MUL(2.0f, t)));
}

struct RefrArgs {
    float3 pos, fwd, right, up;
    float half_h, half_w, step, light_step, threshold, ior;
    float3 ext;  // extinctionCoefficients as given
    int32_t num_refr;
};

struct RefrMap {
    const float* __restrict__ img;
    int3 d;
    float3 size;
};

__device__ __forceinline__ float map_at(const DevParams& P, const RefrMap& M, float3 q) {
    return tex3d(M.img, M.d, PFS_DIV(PFS_SUB(q.x, P.minx), M.size.x), PFS_DIV(PFS_SUB(q.y, P.miny), M.size.y),
                 PFS_DIV(PFS_SUB(q.z, P.minz), M.size.z));
}

__device__ __forceinline__ float3 along(float3 o, float t, float3 d) {
    return make_float3(PFS_ADD(o.x, PFS_MUL(t, d.x)), PFS_ADD(o.y, PFS_MUL(t, d.y)), PFS_ADD(o.z, PFS_MUL(t, d.z)));
}

// calculateDensityAlongRay (:205-218), intersectVolume padded by +-1e-4.
__device__ float refr_density_along(const DevParams& P, const RefrMap& M, float3 o, float3 d, float sstep) {
    float t0, t1;
    if (!ray_box(P, o, d, 1e-4f, -1e-4f, &t0, &t1)) return 0.0f;
    float acc = 0.0f;
    for (float t = PFS_ADD(gmax(t0, 0.0f), sstep); t < PFS_SUB(t1, sstep); t = PFS_ADD(t, sstep))
        acc = PFS_ADD(acc, PFS_MUL(map_at(P, M, along(o, t, d)), sstep));
    return acc;
}

// getSurfaceNormal (:230-260) with calculateClosestFaceNormal (:193-203).
__device__ float3 refr_normal(const DevParams& P, const RefrMap& M, float3 pos) {
    const float mn[3] = {P.minx, P.miny, P.minz}, mx[3] = {P.maxx, P.maxy, P.maxz};
    const float pp[3] = {pos.x, pos.y, pos.z}, sz[3] = {M.size.x, M.size.y, M.size.z};
    const int32_t dd[3] = {M.d.x, M.d.y, M.d.z};
    float uvw[3], texel[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        uvw[a] = gclamp(PFS_DIV(PFS_SUB(pp[a], mn[a]), sz[a]), 0.0f, 1.0f);
        texel[a] = PFS_DIV(1.0f, (float)dd[a]);
    }
    float g[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float up[3], dn[3];
#pragma unroll
        for (int b = 0; b < 3; b++) {
            up[b] = PFS_ADD(uvw[b], a == b ? texel[a] : 0.0f);
            dn[b] = PFS_SUB(uvw[b], a == b ? texel[a] : 0.0f);
        }
        g[a] = PFS_SUB(tex3d(M.img, M.d, up[0], up[1], up[2]), tex3d(M.img, M.d, dn[0], dn[1], dn[2]));
    }
    const float3 vn = normalize3(make_float3(g[0], g[1], g[2]));
    float o[3], local[3], dl[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        o[a] = PFS_SUB(PFS_DIV(sz[a], 2.0f), fabsf(pp[a]));
        local[a] = PFS_SUB(pp[a], PFS_MUL(0.5f, PFS_ADD(mn[a], mx[a])));
        dl[a] = PFS_SUB(PFS_MUL(0.5f, sz[a]), fabsf(local[a]));
    }
    float fw = gmin(o[0], gmin(o[1], o[2]));
    float3 fn = make_float3(0.0f, 0.0f, 0.0f);
    if (dl[0] < dl[1] && dl[0] < dl[2]) fn.x = gsign(local[0]);
    else if (dl[1] < dl[2]) fn.y = gsign(local[1]);
    else fn.z = gsign(local[2]);
    fw = PFS_MUL(PFS_SUB(1.0f, smoothstep(0.0f, 0.3f, fw)), PFS_SUB(1.0f, powf(gclamp(vn.z, 0.0f, 1.0f), 5.0f)));
    const float keep = PFS_SUB(1.0f, fw);
    return normalize3(make_float3(PFS_ADD(PFS_MUL(vn.x, keep), PFS_MUL(fn.x, fw)),
                                  PFS_ADD(PFS_MUL(vn.y, keep), PFS_MUL(fn.y, fw)),
                                  PFS_ADD(PFS_MUL(vn.z, keep), PFS_MUL(fn.z, fw))));
}

struct RefrSurface {
    float3 pos, normal;
    float dens;
    bool found, entering;
};

// findNextSurface (:277-325).
__device__ RefrSurface refr_next_surface(const DevParams& P, const RefrMap& M, const RefrArgs& A, float3 o,
                                         float3 d, bool inside) {
    RefrSurface s;
    s.pos = make_float3(0.0f, 0.0f, 0.0f);
    s.normal = s.pos;
    s.dens = 0.0f;
    s.found = s.entering = false;
    float t0, t1;
    if (!ray_box(P, o, d, 1e-4f, -1e-4f, &t0, &t1)) return s;
    const bool out_of_fluid = !(o.x >= P.minx && o.y >= P.miny && o.z >= P.minz && o.x <= P.maxx &&
                                o.y <= P.maxy && o.z <= P.maxz);
    const float t = inside ? 0.0f : gmax(t0, 0.0f);
    o = along(o, PFS_ADD(t, A.step), d);
    float prev = out_of_fluid ? 0.0f : map_at(P, M, o);
    float dens = 0.0f;
    for (float tt = t; tt < t1; tt = PFS_ADD(tt, A.step)) {
        o = along(o, A.step, d);
        const float density = map_at(P, M, o);
        dens = PFS_ADD(dens, PFS_MUL(density, A.step));
        const bool entering = prev < A.threshold && density >= A.threshold;
        const bool exiting = prev >= A.threshold && density < A.threshold;
        if (inside ? exiting : entering) {
            float3 n = refr_normal(P, M, o);
            if (dot3(n, d) > 0.0f) n = make_float3(-n.x, -n.y, -n.z);
            s.pos = o;
            s.normal = n;
            s.dens = dens;
            s.found = true;
            s.entering = entering;
            return s;
        }
        prev = density;
    }
    s.pos = o;
    s.dens = dens;
    return s;
}

// calculateReflectance (:329-345).
__device__ __forceinline__ float refr_reflectance(float3 in, float3 n, float ia, float ib) {
    const float ratio = PFS_DIV(ia, ib);
    const float cos_in = -dot3(in, n);
    const float sin2 = PFS_MUL(PFS_MUL(ratio, ratio), PFS_SUB(1.0f, PFS_MUL(cos_in, cos_in)));
    if (sin2 >= 1.0f) return 1.0f;
    const float cos_r = PFS_SQRT(PFS_SUB(1.0f, sin2));
    float rs = PFS_DIV(PFS_SUB(PFS_MUL(ia, cos_in), PFS_MUL(ib, cos_r)), PFS_ADD(PFS_MUL(ia, cos_in), PFS_MUL(ib, cos_r)));
    rs = PFS_MUL(rs, rs);
    float rp = PFS_DIV(PFS_SUB(PFS_MUL(ib, cos_in), PFS_MUL(ia, cos_r)), PFS_ADD(PFS_MUL(ib, cos_in), PFS_MUL(ia, cos_r)));
    rp = PFS_MUL(rp, rp);
    return PFS_DIV(PFS_ADD(rs, rp), 2.0f);
}

__device__ __forceinline__ float3 offset(float3 p, float3 n, float s) {
    return make_float3(PFS_ADD(p.x, PFS_MUL(n.x, s)), PFS_ADD(p.y, PFS_MUL(n.y, s)), PFS_ADD(p.z, PFS_MUL(n.z, s)));
}

// marchRayExpensive (:498-573) for one camera ray.
__device__ float3 refr_march(const DevParams& P, const RefrMap& M, const RefrArgs& A, float3 o, float3 d) {
    float tr[3] = {1.0f, 1.0f, 1.0f};
    float light[3] = {0.0f, 0.0f, 0.0f};
    const float ext[3] = {A.ext.x, A.ext.y, A.ext.z};
    bool in_fluid = false;
    for (int i = 0; i < A.num_refr; i++) {
        if (isnan(d.x) || isnan(d.y) || isnan(d.z)) return make_float3(1.0f, 0.0f, 1.0f);
        if (PFS_SQRT(dot3(d, d)) < 1e-6f) return make_float3(1.0f, 1.0f, 0.0f);
        const RefrSurface s = refr_next_surface(P, M, A, o, d, in_fluid);
#pragma unroll
        for (int a = 0; a < 3; a++) tr[a] = PFS_MUL(tr[a], expf(PFS_MUL(-s.dens, ext[a])));
        if (!s.found) break;
        const float ia = s.entering ? 1.0f : A.ior, ib = s.entering ? A.ior : 1.0f;
        // calculateReflectionAndRefraction (:354-372)
        const float3 in = normalize3(d), n = normalize3(s.normal);
        const float rw = refr_reflectance(in, n, ia, ib);
        const float fw = PFS_SUB(1.0f, rw);
        const float dni = dot3(n, in);
        const float two_d = PFS_MUL(2.0f, dni);
        const float3 rdir = normalize3(make_float3(PFS_SUB(in.x, PFS_MUL(two_d, n.x)), PFS_SUB(in.y, PFS_MUL(two_d, n.y)),
                                                   PFS_SUB(in.z, PFS_MUL(two_d, n.z))));
        const float eta = PFS_DIV(ia, ib);
        const float k = PFS_SUB(1.0f, PFS_MUL(PFS_MUL(eta, eta), PFS_SUB(1.0f, PFS_MUL(dni, dni))));
        float3 refr = make_float3(0.0f, 0.0f, 0.0f);
        if (!(k < 0.0f)) {
            const float c = PFS_ADD(PFS_MUL(eta, dni), PFS_SQRT(k));
            refr = make_float3(PFS_SUB(PFS_MUL(eta, in.x), PFS_MUL(c, n.x)), PFS_SUB(PFS_MUL(eta, in.y), PFS_MUL(c, n.y)),
                               PFS_SUB(PFS_MUL(eta, in.z), PFS_MUL(c, n.z)));
        }
        const float3 fdir = dot3(refr, refr) > 1e-12f ? normalize3(refr) : make_float3(0.0f, 0.0f, 0.0f);
        const float3 fo = offset(s.pos, s.normal, -1e-3f), ro = offset(s.pos, s.normal, 1e-3f);
        const bool follow = fw > rw && PFS_SQRT(dot3(fdir, fdir)) > 1e-6f;
        if (follow) in_fluid = !in_fluid;
        if (!follow) {
            if (fw > 0.0f) {
                const float dr = refr_density_along(P, M, fo, fdir, A.light_step);
#pragma unroll
                for (int a = 0; a < 3; a++)
                    light[a] = PFS_ADD(light[a], PFS_MUL(PFS_MUL(PFS_MUL(1.0f, tr[a]), expf(PFS_MUL(-dr, ext[a]))), fw));
            }
        } else {
            const float dr = refr_density_along(P, M, ro, rdir, A.light_step);
#pragma unroll
            for (int a = 0; a < 3; a++)
                light[a] = PFS_ADD(light[a], PFS_MUL(PFS_MUL(PFS_MUL(1.0f, tr[a]), expf(PFS_MUL(-dr, ext[a]))), rw));
        }
        o = follow ? fo : ro;
        d = follow ? fdir : rdir;
        const float wsel = follow ? fw : rw;
#pragma unroll
        for (int a = 0; a < 3; a++) tr[a] = PFS_MUL(tr[a], wsel);
        if (gmax(tr[0], gmax(tr[1], tr[2])) < 0.02f) break;
    }
    const float dr = refr_density_along(P, M, o, d, A.light_step);
#pragma unroll
    for (int a = 0; a < 3; a++)
        light[a] = PFS_ADD(light[a], PFS_MUL(PFS_MUL(1.0f, tr[a]), expf(PFS_MUL(-dr, ext[a]))));
    return make_float3(light[0], light[1], light[2]);
}

// properFluid main (:600-614): one thread per pixel, 16 x 16 pixel tiles as
// the reference's workgroups, so neighbouring rays march together.
__global__ void __launch_bounds__(256)
k_refractive(DevParams P, RefrMap M, RefrArgs A, uint32_t width, uint32_t height, float4* __restrict__ rgba) {
    const uint32_t x = blockIdx.x * 16 + threadIdx.x % 16, y = blockIdx.y * 16 + threadIdx.x / 16;
    if (x >= width || y >= height) return;
    const float u = PFS_SUB(PFS_MUL(PFS_DIV(PFS_ADD((float)x, 0.5f), (float)width), 2.0f), 1.0f);
    const float v = PFS_SUB(PFS_MUL(PFS_DIV(PFS_ADD((float)y, 0.5f), (float)height), 2.0f), 1.0f);
    const float uw = PFS_MUL(u, A.half_w), vh = PFS_MUL(v, A.half_h);
    float3 d;
    d.x = PFS_SUB(PFS_SUB(PFS_ADD(PFS_ADD(A.pos.x, A.fwd.x), PFS_MUL(uw, A.right.x)), PFS_MUL(vh, A.up.x)), A.pos.x);
    d.y = PFS_SUB(PFS_SUB(PFS_ADD(PFS_ADD(A.pos.y, A.fwd.y), PFS_MUL(uw, A.right.y)), PFS_MUL(vh, A.up.y)), A.pos.y);
    d.z = PFS_SUB(PFS_SUB(PFS_ADD(PFS_ADD(A.pos.z, A.fwd.z), PFS_MUL(uw, A.right.z)), PFS_MUL(vh, A.up.z)), A.pos.z);
    const float3 c = refr_march(P, M, A, A.pos, normalize3(d));
    rgba[(size_t)y * width + x] = make_float4(c.x, c.y, c.z, 1.0f);
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

cudaError_t launch_refractive(const DevParams& P, const float* dmap, const int32_t ddims[3], const float cam[12],
                              float half_h, float half_w, float step, float light_step, const float ext[3],
                              int32_t num_refractions, float threshold, float ior, uint32_t width,
                              uint32_t height, float* rgba, cudaStream_t s) {
    if ((uint64_t)width * height == 0) return cudaSuccess;
    RefrMap M;
    M.img = dmap;
    M.d = make_int3(ddims[0], ddims[1], ddims[2]);
    M.size = make_float3(P.maxx - P.minx, P.maxy - P.miny, P.maxz - P.minz);
    RefrArgs A;
    A.pos = make_float3(cam[0], cam[1], cam[2]);
    A.fwd = make_float3(cam[3], cam[4], cam[5]);
    A.right = make_float3(cam[6], cam[7], cam[8]);
    A.up = make_float3(cam[9], cam[10], cam[11]);
    A.half_h = half_h;
    A.half_w = half_w;
    A.step = step;
    A.light_step = light_step;
    A.threshold = threshold;
    A.ior = ior;
    A.ext = make_float3(ext[0], ext[1], ext[2]);
    A.num_refr = num_refractions;
    const dim3 grid((width + 15) / 16, (height + 15) / 16);
    k_refractive<<<grid, 256, 0, s>>>(P, M, A, width, height, reinterpret_cast<float4*>(rgba));
    return cudaGetLastError();
}

}  // namespace pfs
