// glsl_emu.hpp — just enough of GLSL 4.50 compute to execute the reference's
// step shaders on the CPU (TEST INFRASTRUCTURE: used only by the harness that
// pins the oracle; see glsl_ref.py).
//
// Semantics follow the GLSL 4.50 specification with IEEE float32 arithmetic
// (the harness is compiled with -ffp-contract=off): vector operators are
// component-wise, dot/length/distance sum x, y, z left to right, max(x, y) is
// (x < y) ? y : x, min(x, y) is (y < x) ? y : x, clamp = min(max(x, lo), hi),
// mix(x, y, a) = x * (1 - a) + y * a.  Workgroups with barrier() run one
// std::thread per invocation; subgroup operations of uniform control flow are
// emulated through workgroup shared exchange slots (subgroup size 32).
#pragma once
#include <climits>

#include <atomic>
#include <barrier>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace glsl {

typedef unsigned int uint;

struct bvec3 {
    bool x, y, z;
};

struct vec3;
struct ivec3;
struct uvec3;

struct vec3 {
    float x, y, z;
    vec3() = default;
    vec3(float s) : x(s), y(s), z(s) {}
    explicit vec3(const ivec3& v);
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    vec3(int a, int b, int c) : x((float)a), y((float)b), z((float)c) {}
    vec3(float a, float b, int c) : x(a), y(b), z((float)c) {}
    vec3(int a, int b, float c) : x((float)a), y((float)b), z(c) {}
    vec3(float a, int b, int c) : x(a), y((float)b), z((float)c) {}
    vec3(int a, float b, int c) : x((float)a), y(b), z((float)c) {}
    vec3(float a, int b, float c) : x(a), y((float)b), z(c) {}
    vec3(int a, float b, float c) : x((float)a), y(b), z(c) {}
    vec3(double a, double b, double c) : x((float)a), y((float)b), z((float)c) {}
    vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
    vec3& operator*=(float s) { x = x * s; y = y * s; z = z * s; return *this; }
    vec3& operator*=(const vec3& o) { x = x * o.x; y = y * o.y; z = z * o.z; return *this; }
};

struct vec4 {
    float x, y, z, w;
    vec4() = default;
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    vec4(const vec3& v, int d) : x(v.x), y(v.y), z(v.z), w((float)d) {}
    vec4(const vec3& v, double d) : x(v.x), y(v.y), z(v.z), w((float)d) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    // the shaders only read .xyz; the generator rewrites it to .xyz()
    vec3 xyz() const { return vec3(x, y, z); }
    vec4& operator+=(const vec4& o) { x = x + o.x; y = y + o.y; z = z + o.z; w = w + o.w; return *this; }
};

struct ivec3 {
    int x, y, z;
    ivec3() = default;
    explicit ivec3(int s) : x(s), y(s), z(s) {}
    ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit ivec3(const vec3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
    explicit ivec3(const uvec3& v);
};

struct uvec2 {
    uint x, y;
};

struct ivec2 {
    int x, y;
    ivec2() = default;
    ivec2(int a, int b) : x(a), y(b) {}
    explicit ivec2(const uvec2& v) : x((int)v.x), y((int)v.y) {}
};

struct vec2 {
    float x, y;
    vec2() = default;
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
    vec2(int a, int b) : x((float)a), y((float)b) {}
    explicit vec2(const ivec2& v) : x((float)v.x), y((float)v.y) {}
};
inline vec2 operator+(const vec2& a, const vec2& b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator*(const vec2& a, const vec2& b) { return vec2(a.x * b.x, a.y * b.y); }
inline vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }
inline vec2 operator*(float s, const vec2& a) { return vec2(s * a.x, s * a.y); }
inline vec2 operator+(const vec2& a, float s) { return vec2(a.x + s, a.y + s); }
inline vec2 operator/(float s, const vec2& a) { return vec2(s / a.x, s / a.y); }

struct uvec3 {
    uint x, y, z;
    uvec3() = default;
    uvec3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
    // GLSL 4.00+: int -> uint conversions are implicit and keep the bits
    uvec3(const ivec3& v) : x((uint)v.x), y((uint)v.y), z((uint)v.z) {}
    // float -> uint of non-negative in-range values (the shaders only convert
    // in-box coordinates); negative values go through int so bits wrap
    explicit uvec3(const vec3& v)
        : x((uint)(int)v.x), y((uint)(int)v.y), z((uint)(int)v.z) {}
    uvec3 xyz() const { return *this; }
    uvec2 xy() const { return {x, y}; }
};

inline vec3::vec3(const ivec3& v) : x((float)v.x), y((float)v.y), z((float)v.z) {}
inline ivec3::ivec3(const uvec3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}

inline ivec3 operator+(const ivec3& a, const ivec3& b) {
    return ivec3((int)((uint)a.x + (uint)b.x), (int)((uint)a.y + (uint)b.y), (int)((uint)a.z + (uint)b.z));
}

inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline vec3 operator/(float s, const vec3& a) { return vec3(s / a.x, s / a.y, s / a.z); }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }

inline float floor(float v) { return ::floorf(v); }
inline vec3 floor(const vec3& v) { return vec3(::floorf(v.x), ::floorf(v.y), ::floorf(v.z)); }
inline vec3 ceil(const vec3& v) { return vec3(::ceilf(v.x), ::ceilf(v.y), ::ceilf(v.z)); }
inline float sqrt(float v) { return ::sqrtf(v); }
inline float tan(float v) { return ::tanf(v); }
inline float exp(float v) { return ::expf(v); }
inline vec3 exp(const vec3& v) { return vec3(::expf(v.x), ::expf(v.y), ::expf(v.z)); }
inline float abs(float v) { return ::fabsf(v); }
inline float pow(float a, float b) { return ::powf(a, b); }
inline vec3 abs(const vec3& v) { return vec3(::fabsf(v.x), ::fabsf(v.y), ::fabsf(v.z)); }
inline float sign(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(const vec3& a) { return ::sqrtf(dot(a, a)); }
// normalize(v) = v / length(v) (the restatement's definition; GLSL leaves it open)
inline vec3 normalize(const vec3& a) { return a / length(a); }
inline float distance(const vec3& a, const vec3& b) { return length(a - b); }
inline float max(float a, float b) { return (a < b) ? b : a; }
inline float min(float a, float b) { return (b < a) ? b : a; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline vec3 clamp(const vec3& x, float lo, float hi) {
    return vec3(clamp(x.x, lo, hi), clamp(x.y, lo, hi), clamp(x.z, lo, hi));
}
inline vec3 mix(const vec3& x, const vec3& y, float a) { return x * (1.0f - a) + y * a; }
// smoothstep, reflect and refract by the formulas of the GLSL specification,
// evaluated left to right
inline float smoothstep(float e0, float e1, float x) {
    const float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline vec3 reflect(const vec3& i, const vec3& n) { return i - 2.0f * dot(n, i) * n; }
inline vec3 refract(const vec3& i, const vec3& n, float eta) {
    const float k = 1.0f - eta * eta * (1.0f - dot(n, i) * dot(n, i));
    if (k < 0.0f) return vec3(0.0f);
    return eta * i - (eta * dot(n, i) + ::sqrtf(k)) * n;
}
inline bvec3 isnan(const vec3& v) { return {v.x != v.x, v.y != v.y, v.z != v.z}; }
inline bvec3 greaterThanEqual(const vec3& a, const vec3& b) { return {a.x >= b.x, a.y >= b.y, a.z >= b.z}; }
inline bvec3 lessThanEqual(const vec3& a, const vec3& b) { return {a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline bvec3 lessThan(const vec3& a, const vec3& b) { return {a.x < b.x, a.y < b.y, a.z < b.z}; }
inline bvec3 greaterThan(const vec3& a, const vec3& b) { return {a.x > b.x, a.y > b.y, a.z > b.z}; }
inline bool any(const bvec3& b) { return b.x || b.y || b.z; }
inline bool all(const bvec3& b) { return b.x && b.y && b.z; }
inline bvec3 lessThan(const ivec3& a, const ivec3& b) { return {a.x < b.x, a.y < b.y, a.z < b.z}; }
inline bvec3 greaterThan(const ivec3& a, const ivec3& b) { return {a.x > b.x, a.y > b.y, a.z > b.z}; }
inline bvec3 equal(const ivec3& a, const ivec3& b) { return {a.x == b.x, a.y == b.y, a.z == b.z}; }
inline bvec3 greaterThan(const ivec3& a, const vec3& b) {
    return {(float)a.x > b.x, (float)a.y > b.y, (float)a.z > b.z};
}

// A sampler3D of the reference's sampler (linear, clamp to edge, normalised
// coordinates, one level), as float trilinear interpolation in the term order
// of the oracle's pfso_texture3d.
struct Sampler3D {
    const float* data = nullptr;
    int nx = 0, ny = 0, nz = 0;
};
inline vec4 texture(const Sampler3D& t, const vec3& uvw) {
    const float uu[3] = {uvw.x, uvw.y, uvw.z};
    const int dd[3] = {t.nx, t.ny, t.nz};
    int i0[3], i1[3];
    float f[3];
    for (int a = 0; a < 3; a++) {
        const float u = uu[a] * (float)dd[a] - 0.5f;
        const float fl = ::floorf(u);
        f[a] = u - fl;
        const int k = fl != fl ? 0 : (fl < -2147483648.0f ? INT_MIN : (fl >= 2147483647.0f ? INT_MAX : (int)fl));
        const int top = dd[a] - 1;
        i0[a] = k < 0 ? 0 : (k > top ? top : k);
        const int k1 = k == INT_MAX ? k : k + 1;
        i1[a] = k1 < 0 ? 0 : (k1 > top ? top : k1);
    }
    auto T = [&](int x, int y, int z) { return t.data[((size_t)z * t.ny + y) * t.nx + x]; };
    const float a0 = 1.0f - f[0], a1 = f[0], b0 = 1.0f - f[1], b1 = f[1], c0 = 1.0f - f[2], c1 = f[2];
    float r = 0.0f;
    r = r + (a0 * b0) * c0 * T(i0[0], i0[1], i0[2]);
    r = r + (a1 * b0) * c0 * T(i1[0], i0[1], i0[2]);
    r = r + (a0 * b1) * c0 * T(i0[0], i1[1], i0[2]);
    r = r + (a1 * b1) * c0 * T(i1[0], i1[1], i0[2]);
    r = r + (a0 * b0) * c1 * T(i0[0], i0[1], i1[2]);
    r = r + (a1 * b0) * c1 * T(i1[0], i0[1], i1[2]);
    r = r + (a0 * b1) * c1 * T(i0[0], i1[1], i1[2]);
    r = r + (a1 * b1) * c1 * T(i1[0], i1[1], i1[2]);
    return vec4(r, r, r, r);
}

inline vec2 clamp(const vec2& x, const vec2& lo, const vec2& hi) {
    return vec2(clamp(x.x, lo.x, hi.x), clamp(x.y, lo.y, hi.y));
}

// A sampler2D of the reference's sampler (linear, clamp to edge, normalised
// coordinates) over an rgba32f image, as float bilinear interpolation in the
// term order of the oracle's tex2d_rgb.
struct Sampler2D {
    const float* data = nullptr;  // x-fastest float4 texels
    int nx = 0, ny = 0;
};
inline ivec2 textureSize(const Sampler2D& t, int) { return ivec2(t.nx, t.ny); }
inline vec4 texture(const Sampler2D& t, const vec2& uv) {
    const float uu[2] = {uv.x, uv.y};
    const int dd[2] = {t.nx, t.ny};
    int i0[2], i1[2];
    float f[2];
    for (int a = 0; a < 2; a++) {
        const float u = uu[a] * (float)dd[a] - 0.5f;
        const float fl = ::floorf(u);
        f[a] = u - fl;
        const int k = fl != fl ? 0 : (fl < -2147483648.0f ? INT_MIN : (fl >= 2147483647.0f ? INT_MAX : (int)fl));
        const int top = dd[a] - 1;
        i0[a] = k < 0 ? 0 : (k > top ? top : k);
        const int k1 = k == INT_MAX ? k : k + 1;
        i1[a] = k1 < 0 ? 0 : (k1 > top ? top : k1);
    }
    const float a0 = 1.0f - f[0], a1 = f[0], b0 = 1.0f - f[1], b1 = f[1];
    float r[4];
    for (int c = 0; c < 4; c++) {
        auto T = [&](int x, int y) { return t.data[4 * ((size_t)y * t.nx + x) + c]; };
        float v = 0.0f;
        v = v + (a0 * b0) * T(i0[0], i0[1]);
        v = v + (a1 * b0) * T(i1[0], i0[1]);
        v = v + (a0 * b1) * T(i0[0], i1[1]);
        v = v + (a1 * b1) * T(i1[0], i1[1]);
        r[c] = v;
    }
    return vec4(r[0], r[1], r[2], r[3]);
}

// A writeonly rgba32f image2D.
struct Image2D {
    float* data = nullptr;
    int nx = 0, ny = 0;
};
inline void imageStore(Image2D& im, const ivec2& c, const vec4& v) {
    if (c.x < 0 || c.y < 0 || c.x >= im.nx || c.y >= im.ny) return;
    float* q = im.data + 4 * ((size_t)c.y * im.nx + c.x);
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
}

// A writeonly r32f image3D: imageStore keeps .x; stores outside the image
// are dropped (the reference's image is smaller than the shader's bound).
struct Image3D {
    float* data = nullptr;
    int nx = 0, ny = 0, nz = 0;
};
inline ivec3 imageSize(const Image3D& im) { return ivec3(im.nx, im.ny, im.nz); }
inline void imageStore(Image3D& im, const ivec3& c, const vec4& v) {
    if (c.x < 0 || c.y < 0 || c.z < 0 || c.x >= im.nx || c.y >= im.ny || c.z >= im.nz) return;
    im.data[((size_t)c.z * im.ny + c.y) * im.nx + c.x] = v.x;
}
inline uint bitCount(uint v) { return (uint)__builtin_popcount(v); }
inline uint atomicAdd(uint& mem, uint v) { return std::atomic_ref<uint>(mem).fetch_add(v); }

// Column-major matrices (m[column * 4 + row]); products sum over k left to
// right, the order the oracle's pfso_splat_camera uses.
struct mat4 {
    float m[16];
};
struct mat3 {
    vec3 c[3];
    mat3() = default;
    explicit mat3(const mat4& a) {
        for (int k = 0; k < 3; k++) c[k] = vec3(a.m[k * 4 + 0], a.m[k * 4 + 1], a.m[k * 4 + 2]);
    }
    vec3 operator[](int k) const { return c[k]; }
};
inline mat3 transpose(const mat3& a) {
    mat3 t;
    t.c[0] = vec3(a.c[0].x, a.c[1].x, a.c[2].x);
    t.c[1] = vec3(a.c[0].y, a.c[1].y, a.c[2].y);
    t.c[2] = vec3(a.c[0].z, a.c[1].z, a.c[2].z);
    return t;
}
inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r;
    for (int c = 0; c < 4; c++)
        for (int w = 0; w < 4; w++)
            r.m[c * 4 + w] = a.m[0 * 4 + w] * b.m[c * 4 + 0] + a.m[1 * 4 + w] * b.m[c * 4 + 1] +
                             a.m[2 * 4 + w] * b.m[c * 4 + 2] + a.m[3 * 4 + w] * b.m[c * 4 + 3];
    return r;
}
inline vec4 operator*(const mat4& a, const vec4& v) {
    float r[4];
    for (int w = 0; w < 4; w++)
        r[w] = a.m[0 * 4 + w] * v.x + a.m[1 * 4 + w] * v.y + a.m[2 * 4 + w] * v.z + a.m[3 * 4 + w] * v.w;
    return vec4(r[0], r[1], r[2], r[3]);
}
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }

// Per-workgroup context shared by its invocations.
struct Workgroup {
    std::barrier<>* bar = nullptr;
    uint exchange[1024];
    alignas(16) char smem[65536];
};

// Built-ins and workgroup operations of one invocation.
struct Invocation {
    // graphics-stage built-ins (vertex and fragment shaders)
    vec4 gl_Position{0.0f, 0.0f, 0.0f, 0.0f};
    int gl_InstanceIndex = 0;
    bool discarded = false;
    uvec3 gl_GlobalInvocationID{0, 0, 0};
    uvec3 gl_LocalInvocationID{0, 0, 0};
    uvec3 gl_WorkGroupID{0, 0, 0};
    uint gl_SubgroupID = 0;
    uint gl_SubgroupInvocationID = 0;
    Workgroup* wg = nullptr;

    void barrier() {
        if (wg && wg->bar) wg->bar->arrive_and_wait();
    }
    uint subgroupAdd(uint v) {
        const uint lid = gl_LocalInvocationID.x;
        wg->exchange[lid] = v;
        barrier();
        uint s = 0;
        for (uint k = gl_SubgroupID * 32; k < gl_SubgroupID * 32 + 32; k++) s += wg->exchange[k];
        barrier();
        return s;
    }
    uint subgroupExclusiveAdd(uint v) {
        const uint lid = gl_LocalInvocationID.x;
        wg->exchange[lid] = v;
        barrier();
        uint s = 0;
        for (uint k = gl_SubgroupID * 32; k < lid; k++) s += wg->exchange[k];
        barrier();
        return s;
    }
    bool subgroupElect() { return gl_SubgroupInvocationID == 0; }
};

}  // namespace glsl
