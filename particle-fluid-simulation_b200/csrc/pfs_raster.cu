// pfs_raster.cu — the reference's default render (RENDER_TYPE RASTERIZATION):
// camera-facing point splats of shader.vert:27-57 / shader.frag:56-87 with
// depth test LESS and no blending, and the FXAA pass of
// raymarchShader.frag:15-73 that presents the ray-marched modes, as CUDA
// kernels writing headless float4 buffers.
//
// Splats (the oracle's restatement, pfso_splats): each quad projects to a
// screen-aligned square between its corners (-1,-1) and (1,1); pixel centres
// in [min, max) on both axes are fragments, fragQuadPos is linear across the
// square, the depth is the projected z / w of the particle centre and
// fragments with |fragQuadPos|^2 > 1 are discarded.  Sequential drawing in
// slot order with LESS keeps, per pixel, the first particle of the smallest
// depth, i.e. the minimum of (depth bits << 32 | slot) over the fragments
// (depths lie in [0, 1), where float bits order like the floats): pass 1
// takes that minimum with 64-bit atomicMin, pass 2 shades each pixel from its
// winner.  Every float operation is one IEEE round-to-nearest operation in
// the oracle's order, so images equal the oracle's bit for bit.
#include <cstdint>
#include <cuda_runtime.h>

#include "pfs_common.cuh"
#include "pfs_step.cuh"

namespace pfs {

namespace {

constexpr int RASTER_THREADS = 256;
constexpr unsigned long long EMPTY = ~0ull;

__device__ __forceinline__ float fmin_g(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float fmax_g(float x, float y) { return (x < y) ? y : x; }

struct SplatCam {
    float mvp[16];
    float right[3], up[3];
    float radius;
};

__device__ __forceinline__ void splat_clip(const SplatCam& C, float4 p, float qx, float qy, float clip[4]) {
    const float pp[3] = {p.x, p.y, p.z};
    float wp[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
        wp[a] = PFS_ADD(pp[a], PFS_MUL(C.radius, PFS_ADD(PFS_MUL(qx, C.right[a]), PFS_MUL(qy, C.up[a]))));
#pragma unroll
    for (int k = 0; k < 4; k++)
        clip[k] = PFS_ADD(PFS_ADD(PFS_ADD(PFS_MUL(C.mvp[k], wp[0]), PFS_MUL(C.mvp[4 + k], wp[1])),
                                  PFS_MUL(C.mvp[8 + k], wp[2])),
                          PFS_MUL(C.mvp[12 + k], 1.0f));
}

// pfso_splat_geometry: screen square (corner (-1,-1) x, y, corner (1,1) x, y)
// and depth; false when clipped.
__device__ __forceinline__ bool splat_geometry(const SplatCam& C, float4 p, uint32_t width, uint32_t height,
                                               float sq[4], float* depth) {
    float c0[4], ca[4], cb[4];
    splat_clip(C, p, 0.0f, 0.0f, c0);
    splat_clip(C, p, -1.0f, -1.0f, ca);
    splat_clip(C, p, 1.0f, 1.0f, cb);
    if (!(c0[3] > 0.0f && ca[3] > 0.0f && cb[3] > 0.0f)) return false;
    const float z = PFS_DIV(c0[2], c0[3]);
    if (!(z >= 0.0f && z <= 1.0f)) return false;
    const float hw = PFS_MUL((float)width, 0.5f), hh = PFS_MUL((float)height, 0.5f);
    sq[0] = PFS_ADD(PFS_MUL(PFS_DIV(ca[0], ca[3]), hw), hw);
    sq[1] = PFS_ADD(PFS_MUL(PFS_DIV(ca[1], ca[3]), hh), hh);
    sq[2] = PFS_ADD(PFS_MUL(PFS_DIV(cb[0], cb[3]), hw), hw);
    sq[3] = PFS_ADD(PFS_MUL(PFS_DIV(cb[1], cb[3]), hh), hh);
    *depth = z;
    return true;
}

__device__ __forceinline__ bool splat_quadpos(const float sq[4], int32_t x, int32_t y, float* qx, float* qy) {
    const float px = PFS_ADD((float)x, 0.5f), py = PFS_ADD((float)y, 0.5f);
    const float x0 = fmin_g(sq[0], sq[2]), x1 = fmax_g(sq[0], sq[2]);
    const float y0 = fmin_g(sq[1], sq[3]), y1 = fmax_g(sq[1], sq[3]);
    if (!(px >= x0 && px < x1 && py >= y0 && py < y1)) return false;
    *qx = PFS_ADD(-1.0f, PFS_MUL(2.0f, PFS_DIV(PFS_SUB(px, sq[0]), PFS_SUB(sq[2], sq[0]))));
    *qy = PFS_ADD(-1.0f, PFS_MUL(2.0f, PFS_DIV(PFS_SUB(py, sq[1]), PFS_SUB(sq[3], sq[1]))));
    return true;
}

__global__ void __launch_bounds__(RASTER_THREADS)
k_splat_raster(uint32_t n, const float4* __restrict__ x, SplatCam C, uint32_t width, uint32_t height,
               unsigned long long* __restrict__ keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float sq[4], z;
    if (!splat_geometry(C, x[i], width, height, sq, &z)) return;
    if (!(z < 1.0f)) return;  // LESS against the cleared depth 1
    const float x0 = fmin_g(sq[0], sq[2]), x1 = fmax_g(sq[0], sq[2]);
    const float y0 = fmin_g(sq[1], sq[3]), y1 = fmax_g(sq[1], sq[3]);
    if (!(x1 >= 0.0f && y1 >= 0.0f && x0 <= (float)width && y0 <= (float)height)) return;
    const int32_t xa = x0 < 1.0f ? 0 : (int32_t)x0 - 1, ya = y0 < 1.0f ? 0 : (int32_t)y0 - 1;
    const int32_t xb = x1 >= (float)width ? (int32_t)width - 1 : (int32_t)x1 + 1;
    const int32_t yb = y1 >= (float)height ? (int32_t)height - 1 : (int32_t)y1 + 1;
    const unsigned long long key = ((unsigned long long)__float_as_uint(z) << 32) | i;
    for (int32_t py = ya; py <= yb; py++)
        for (int32_t px = xa; px <= xb; px++) {
            float qx, qy;
            if (!splat_quadpos(sq, px, py, &qx, &qy)) continue;
            if (PFS_ADD(PFS_MUL(qx, qx), PFS_MUL(qy, qy)) > 1.0f) continue;  // discard
            atomicMin(keys + (size_t)py * width + px, key);
        }
}

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) {
    return PFS_ADD(PFS_ADD(PFS_MUL(a[0], b[0]), PFS_MUL(a[1], b[1])), PFS_MUL(a[2], b[2]));
}

__global__ void __launch_bounds__(RASTER_THREADS)
k_splat_shade(uint32_t n, const float4* __restrict__ x, const float4* __restrict__ color, SplatCam C,
              uint32_t width, uint32_t height, const unsigned long long* __restrict__ keys,
              float4* __restrict__ rgba, float* __restrict__ depth, uint32_t* __restrict__ err) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (uint64_t)width * height) return;
    const unsigned long long key = keys[k];
    float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float z = 1.0f;
    if (key != EMPTY) {
        const uint32_t i = (uint32_t)(key & 0xffffffffu);
        float sq[4], zi, qx, qy;
        if (i >= n || !splat_geometry(C, x[i], width, height, sq, &zi) ||
            !splat_quadpos(sq, (int32_t)(k % width), (int32_t)(k / width), &qx, &qy)) {
            atomicOr(err, ERR_PERM_RANGE);
        } else {
            z = zi;
            // pfso_splat_shade (shader.frag:63-85)
            const float r2 = PFS_ADD(PFS_MUL(qx, qx), PFS_MUL(qy, qy));
            float nrm[3] = {-qx, -qy, PFS_SQRT(PFS_SUB(1.0f, r2))};
            const float nl = PFS_SQRT(dot3(nrm, nrm));
#pragma unroll
            for (int a = 0; a < 3; a++) nrm[a] = PFS_DIV(nrm[a], nl);
            float ld[3] = {-0.5f, -0.5f, 1.0f};
            const float ll = PFS_SQRT(dot3(ld, ld));
#pragma unroll
            for (int a = 0; a < 3; a++) ld[a] = PFS_DIV(ld[a], ll);
            const float lighting = fmax_g(dot3(nrm, ld), 0.0f);
            const float t = fmin_g(fmax_g(PFS_DIV(PFS_SUB(PFS_SQRT(r2), 0.8f), PFS_SUB(1.0f, 0.8f)), 0.0f), 1.0f);
            const float alpha = PFS_SUB(1.0f, PFS_MUL(PFS_MUL(t, t), PFS_SUB(3.0f, PFS_MUL(2.0f, t))));
            const float s = PFS_ADD(PFS_SUB(1.0f, 0.3f), PFS_MUL(0.3f, lighting));
            const float4 c = color[i];
            out = make_float4(PFS_MUL(c.x, s), PFS_MUL(c.y, s), PFS_MUL(c.z, s), alpha);
        }
    }
    rgba[k] = out;
    if (depth) depth[k] = z;
}

// ---- FXAA (raymarchShader.frag:15-73, the oracle's pfso_fxaa) ---------------

__device__ __forceinline__ float3 tex2d_rgb(const float4* __restrict__ img, int32_t w, int32_t h, float u,
                                            float v) {
    const float uu[2] = {u, v};
    const int32_t dd[2] = {w, h};
    int32_t i0[2], i1[2];
    float f[2];
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const float t = PFS_SUB(PFS_MUL(uu[a], (float)dd[a]), 0.5f);
        const float fl = floorf(t);
        f[a] = PFS_SUB(t, fl);
        const int32_t kk = __float2int_rz(fl);  // NaN -> 0, out of range saturates
        const int32_t top = dd[a] - 1;
        i0[a] = min(max(kk, 0), top);
        const int32_t k1 = kk == INT32_MAX ? kk : kk + 1;
        i1[a] = min(max(k1, 0), top);
    }
    const float a0 = PFS_SUB(1.0f, f[0]), a1 = f[0], b0 = PFS_SUB(1.0f, f[1]), b1 = f[1];
    const float w00 = PFS_MUL(a0, b0), w10 = PFS_MUL(a1, b0), w01 = PFS_MUL(a0, b1), w11 = PFS_MUL(a1, b1);
    const float4 t00 = __ldg(img + (size_t)i0[1] * w + i0[0]), t10 = __ldg(img + (size_t)i0[1] * w + i1[0]);
    const float4 t01 = __ldg(img + (size_t)i1[1] * w + i0[0]), t11 = __ldg(img + (size_t)i1[1] * w + i1[0]);
    float3 r;
    r.x = PFS_ADD(PFS_ADD(PFS_ADD(PFS_ADD(0.0f, PFS_MUL(w00, t00.x)), PFS_MUL(w10, t10.x)), PFS_MUL(w01, t01.x)),
                  PFS_MUL(w11, t11.x));
    r.y = PFS_ADD(PFS_ADD(PFS_ADD(PFS_ADD(0.0f, PFS_MUL(w00, t00.y)), PFS_MUL(w10, t10.y)), PFS_MUL(w01, t01.y)),
                  PFS_MUL(w11, t11.y));
    r.z = PFS_ADD(PFS_ADD(PFS_ADD(PFS_ADD(0.0f, PFS_MUL(w00, t00.z)), PFS_MUL(w10, t10.z)), PFS_MUL(w01, t01.z)),
                  PFS_MUL(w11, t11.z));
    return r;
}

__device__ __forceinline__ float luma(float3 c) {
    return PFS_ADD(PFS_ADD(PFS_MUL(c.x, 0.299f), PFS_MUL(c.y, 0.587f)), PFS_MUL(c.z, 0.114f));
}

__global__ void __launch_bounds__(RASTER_THREADS)
k_fxaa(const float4* __restrict__ in, uint32_t width, uint32_t height, float tx, float ty, float4* __restrict__ out) {
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (uint64_t)width * height) return;
    const int32_t W = (int32_t)width, H = (int32_t)height;
    const int32_t x = (int32_t)(idx % width), y = (int32_t)(idx / width);
    const float nx = PFS_SUB(PFS_MUL(PFS_DIV(PFS_ADD((float)x, 0.5f), (float)width), 2.0f), 1.0f);
    const float ny = PFS_SUB(PFS_MUL(PFS_DIV(PFS_ADD((float)y, 0.5f), (float)height), 2.0f), 1.0f);
    const float u = PFS_ADD(PFS_MUL(nx, 0.5f), 0.5f), v = PFS_ADD(PFS_MUL(ny, 0.5f), 0.5f);
    const float mtx = PFS_MUL(-1.0f, tx), mty = PFS_MUL(-1.0f, ty), ptx = PFS_MUL(1.0f, tx), pty = PFS_MUL(1.0f, ty);
    const float lnw = luma(tex2d_rgb(in, W, H, PFS_ADD(u, mtx), PFS_ADD(v, mty)));
    const float lne = luma(tex2d_rgb(in, W, H, PFS_ADD(u, ptx), PFS_ADD(v, mty)));
    const float lsw = luma(tex2d_rgb(in, W, H, PFS_ADD(u, mtx), PFS_ADD(v, pty)));
    const float lse = luma(tex2d_rgb(in, W, H, PFS_ADD(u, ptx), PFS_ADD(v, pty)));
    const float lm = luma(tex2d_rgb(in, W, H, u, v));
    const float lmin = fmin_g(lm, fmin_g(fmin_g(lnw, lne), fmin_g(lsw, lse)));
    const float lmax = fmax_g(lm, fmax_g(fmax_g(lnw, lne), fmax_g(lsw, lse)));
    float dx = -PFS_SUB(PFS_ADD(lnw, lne), PFS_ADD(lsw, lse));
    float dy = PFS_SUB(PFS_ADD(lnw, lsw), PFS_ADD(lne, lse));
    const float reduce = fmax_g(PFS_MUL(PFS_ADD(PFS_ADD(PFS_ADD(lnw, lne), lsw), lse), 0.03125f), 0.0078125f);
    const float rcp = PFS_DIV(1.0f, PFS_ADD(fmin_g(fabsf(dx), fabsf(dy)), reduce));
    dx = PFS_MUL(fmin_g(fmax_g(PFS_MUL(dx, rcp), -8.0f), 8.0f), tx);
    dy = PFS_MUL(fmin_g(fmax_g(PFS_MUL(dy, rcp), -8.0f), 8.0f), ty);
    const float k1 = PFS_SUB(PFS_DIV(1.0f, 3.0f), 0.5f), k2 = PFS_SUB(PFS_DIV(2.0f, 3.0f), 0.5f);
    const float3 a1 = tex2d_rgb(in, W, H, PFS_ADD(u, PFS_MUL(dx, k1)), PFS_ADD(v, PFS_MUL(dy, k1)));
    const float3 a2 = tex2d_rgb(in, W, H, PFS_ADD(u, PFS_MUL(dx, k2)), PFS_ADD(v, PFS_MUL(dy, k2)));
    const float3 b1 = tex2d_rgb(in, W, H, PFS_ADD(u, PFS_MUL(dx, -0.5f)), PFS_ADD(v, PFS_MUL(dy, -0.5f)));
    const float3 b2 = tex2d_rgb(in, W, H, PFS_ADD(u, PFS_MUL(dx, 0.5f)), PFS_ADD(v, PFS_MUL(dy, 0.5f)));
    const float3 ra = make_float3(PFS_MUL(0.5f, PFS_ADD(a1.x, a2.x)), PFS_MUL(0.5f, PFS_ADD(a1.y, a2.y)),
                                  PFS_MUL(0.5f, PFS_ADD(a1.z, a2.z)));
    const float3 rb = make_float3(PFS_ADD(PFS_MUL(ra.x, 0.5f), PFS_MUL(0.25f, PFS_ADD(b1.x, b2.x))),
                                  PFS_ADD(PFS_MUL(ra.y, 0.5f), PFS_MUL(0.25f, PFS_ADD(b1.y, b2.y))),
                                  PFS_ADD(PFS_MUL(ra.z, 0.5f), PFS_MUL(0.25f, PFS_ADD(b1.z, b2.z))));
    const float lb = luma(rb);
    const float3 c = (lb < lmin || lb > lmax) ? ra : rb;
    out[idx] = make_float4(c.x, c.y, c.z, 1.0f);
}

}  // namespace

cudaError_t launch_splats(uint32_t n, const float4* x, const float4* color, const float mvp[16],
                          const float right[3], const float up[3], float radius, uint32_t width,
                          uint32_t height, unsigned long long* keys, float* rgba, float* depth,
                          uint32_t* err, cudaStream_t s) {
    const uint64_t npx = (uint64_t)width * height;
    if (npx == 0) return cudaSuccess;
    SplatCam C;
    for (int k = 0; k < 16; k++) C.mvp[k] = mvp[k];
    for (int a = 0; a < 3; a++) {
        C.right[a] = right[a];
        C.up[a] = up[a];
    }
    C.radius = radius;
    cudaError_t e = cudaMemsetAsync(keys, 0xff, npx * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (n) k_splat_raster<<<(n + RASTER_THREADS - 1) / RASTER_THREADS, RASTER_THREADS, 0, s>>>(n, x, C, width,
                                                                                               height, keys);
    k_splat_shade<<<(unsigned)((npx + RASTER_THREADS - 1) / RASTER_THREADS), RASTER_THREADS, 0, s>>>(
        n, x, color, C, width, height, keys, reinterpret_cast<float4*>(rgba), depth, err);
    return cudaGetLastError();
}

cudaError_t launch_fxaa(const float* in, uint32_t width, uint32_t height, float* out, cudaStream_t s) {
    const uint64_t npx = (uint64_t)width * height;
    if (npx == 0) return cudaSuccess;
    const float tx = 1.0f / (float)width, ty = 1.0f / (float)height;
    k_fxaa<<<(unsigned)((npx + RASTER_THREADS - 1) / RASTER_THREADS), RASTER_THREADS, 0, s>>>(
        reinterpret_cast<const float4*>(in), width, height, tx, ty, reinterpret_cast<float4*>(out));
    return cudaGetLastError();
}

}  // namespace pfs
