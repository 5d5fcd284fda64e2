// glsl_driver.cpp — replays the reference's substep (src/renderer/commands.c
// :193-402) on the CPU over the reference's own shader sources, which
// glsl_ref.py turns into C++ structs (TEST INFRASTRUCTURE: pins the oracle).
//
// Buffers and descriptor sets follow renderer.c:510-754 and
// descriptors.c:144-289: everything but startIndices, endIndices and
// histograms exists twice; descriptor set p binds the [p] buffers at bindings
// 2-9 and 19, and the [1-p] buffers at the output bindings 10-16 and 20.
// multiRadixSort() is commands.c:106-161 (4 passes, ping toggled per pass).
//
// One deliberate difference, switchable: with jacobi = 1 the force pass reads
// every neighbour's velocity from before the pass (the reference's shader
// reads velocities[j] from the buffer it is updating, a data race on the GPU;
// run serially it would be Gauss-Seidel in slot order).
#include <cstdint>
#include <cstring>
#include <vector>

#include "glsl_dispatch.hpp"

using glsl::RefUbo;
using glsl::uint;

#define DECLARE(name)                                                                     \
    extern "C" void ref_dispatch_##name(const RefUbo* u, void* const* bindings, uint groups, \
                                        glsl::InvocationHook hook, void* ctx)
DECLARE(predictPositions);
DECLARE(updateCellEntries);
DECLARE(multiRadixSortHistograms);
DECLARE(multiRadixSort);
DECLARE(scatterPass);
DECLARE(clearStartIndices);
DECLARE(updateStartIndices);
DECLARE(calculateDensities);
DECLARE(applyPressureAndViscosityForce);
DECLARE(updateVelocities);
extern "C" void ref_dispatch3_updateDensityMap(const RefUbo* u, void* const* bindings, uint nx,
                                               uint ny, uint nz, float* img, int ix, int iy, int iz);
extern "C" void ref_dispatch_rt_calculateLightVolume(const RefUbo* u, void* const* bindings, uint nx,
                                                     uint ny, uint nz, const glsl::RtBind* rb);
extern "C" void ref_dispatch_rt_volumetricFluid(const RefUbo* u, void* const* bindings, uint nx,
                                                uint ny, uint nz, const glsl::RtBind* rb);
extern "C" void ref_vertex_shader_vert(const RefUbo* u, float qx, float qy, const float pos[3], int instance,
                                       float clip[4]);
extern "C" int ref_fragment_shader_frag(const RefUbo* u, void* const* bindings, int index, float qx, float qy,
                                        float out[4]);
extern "C" void ref_dispatch_rt_properFluid(const RefUbo* u, void* const* bindings, uint nx, uint ny,
                                            uint nz, const glsl::RtBind* rb);

extern "C" {

typedef struct ref_params {
    float particleRadius, smoothingRadius, g;
    float minXYZ[3];
    float dt;
    float maxXYZ[3];
    float particleMass, pressureMultiplier, targetDensity, viscosityStrength, volume,
        nearPressureMultiplier;
    uint32_t numBlocksPerWorkGroup;
} ref_params;

typedef struct ref_trace {
    uint32_t* keys_in;
    uint32_t* keys;
    uint32_t* perm;
    int32_t* start;
    int32_t* end;
    float* xp;
    float* vp;
    float* density;
    float* near_density;
    float* vel_force;
    float* colors;
} ref_trace;

}  // extern "C"

namespace {

struct Entry {
    uint32_t key, particleIndex;
};

struct Jacobi {
    uint32_t n;
    float* live;        // velocities buffer the shader updates in place
    const float* orig;  // velocities before the pass
    float* out;         // collected results
};

void jacobi_hook(void* ctx, uint gid) {
    Jacobi* j = static_cast<Jacobi*>(ctx);
    if (gid >= j->n) return;  // guarded invocations of the last workgroup
    // slot gid is the only element invocation gid writes
    std::memcpy(j->out + 4 * (size_t)gid, j->live + 4 * (size_t)gid, 16);
    std::memcpy(j->live + 4 * (size_t)gid, j->orig + 4 * (size_t)gid, 16);
}

}  // namespace

extern "C" int ref_substep(const ref_params* p, uint32_t n, float* pos4, float* vel4,
                           ref_trace* tr, int jacobi) {
    if (n == 0) return 0;
    const size_t n4 = (size_t)n * 4;
    const uint32_t WG = 128;  // WORKGROUP_SIZE_X (commands.h:4)
    std::vector<float> pos[2], vel[2], ppos[2], pvel[2], dens[2], col[2], near[2];
    std::vector<Entry> cells[2];
    for (int k = 0; k < 2; k++) {
        pos[k].assign(pos4, pos4 + n4);                     // renderer.c:595-605
        vel[k].assign(vel4, vel4 + n4);                     // renderer.c:646-656
        ppos[k].assign(n4, 0.0f);
        pvel[k].assign(n4, 0.0f);
        dens[k].assign(n, 0.0f);
        near[k].assign(n, 0.0f);
        col[k].assign(n4, 1.0f);
        cells[k].resize(n);
        for (uint32_t i = 0; i < n; i++) cells[k][i] = {0u, i};  // renderer.c:684
    }
    std::vector<int32_t> start(n, 0), end(n, 0);
    const uint32_t blocks = p->numBlocksPerWorkGroup;
    const uint32_t per_group_host = WG * blocks;  // commands.c:112
    const uint32_t sort_groups = (n + per_group_host - 1) / per_group_host;
    // the histogram buffer holds n words (renderer.c:536); the shaders index
    // 256 per workgroup, so small n needs the larger of the two
    std::vector<uint32_t> hist(std::max<size_t>(n, 256 * (size_t)sort_groups), 0u);

    RefUbo u{};
    u.numParticles = (int)n;
    u.particleRadius = p->particleRadius;
    u.smoothingRadius = p->smoothingRadius;
    u.g = p->g;
    for (int a = 0; a < 3; a++) { u.minXYZ[a] = p->minXYZ[a]; u.maxXYZ[a] = p->maxXYZ[a]; }
    u.dt = p->dt;
    u.particleMass = p->particleMass;
    u.pressureMultiplier = p->pressureMultiplier;
    u.targetDensity = p->targetDensity;
    u.viscosityStrength = p->viscosityStrength;
    u.volume = p->volume;
    u.nearPressureMultiplier = p->nearPressureMultiplier;

    int ping = 0;  // main.c:384
    auto set = [&](int q, void** b) {
        for (int i = 0; i < 32; i++) b[i] = nullptr;
        const int o = 1 - q;
        b[2] = pos[q].data(); b[3] = vel[q].data(); b[4] = ppos[q].data(); b[5] = pvel[q].data();
        b[6] = cells[q].data(); b[7] = dens[q].data(); b[8] = start.data(); b[9] = col[q].data();
        b[10] = pos[o].data(); b[11] = vel[o].data(); b[12] = ppos[o].data(); b[13] = pvel[o].data();
        b[14] = dens[o].data(); b[15] = col[o].data(); b[16] = cells[o].data();
        b[17] = hist.data(); b[18] = end.data(); b[19] = near[q].data(); b[20] = near[o].data();
    };
    void* b[32];
    const uint32_t g64 = (n + 63) / 64, g128 = (n + WG - 1) / WG;

    set(ping, b);  // commands.c:196-200
    ref_dispatch_predictPositions(&u, b, g64, nullptr, nullptr);
    ref_dispatch_updateCellEntries(&u, b, g64, nullptr, nullptr);  // :222-226
    if (tr && tr->keys_in)
        for (uint32_t i = 0; i < n; i++) tr->keys_in[i] = cells[ping][i].key;
    for (int pass = 0; pass < 4; pass++) {  // multiRadixSort, commands.c:106-161
        u.g_num_elements = n;
        u.g_shift = 8u * pass;
        u.g_num_workgroups = sort_groups;
        u.g_num_blocks_per_workgroup = blocks;
        set(ping, b);
        ref_dispatch_multiRadixSortHistograms(&u, b, sort_groups, nullptr, nullptr);
        ref_dispatch_multiRadixSort(&u, b, sort_groups, nullptr, nullptr);
        ping = 1 - ping;
    }
    if (tr) {
        for (uint32_t i = 0; i < n; i++) {
            if (tr->keys) tr->keys[i] = cells[ping][i].key;
            if (tr->perm) tr->perm[i] = cells[ping][i].particleIndex;
        }
    }
    set(ping, b);
    ref_dispatch_scatterPass(&u, b, g128, nullptr, nullptr);  // :249-253
    ping = 1 - ping;                                          // :255
    set(ping, b);
    ref_dispatch_clearStartIndices(&u, b, g128, nullptr, nullptr);   // :268-272
    ref_dispatch_updateStartIndices(&u, b, g128, nullptr, nullptr);  // :295-299
    if (tr) {
        if (tr->start) std::memcpy(tr->start, start.data(), n * 4);
        if (tr->end) std::memcpy(tr->end, end.data(), n * 4);
        if (tr->xp) std::memcpy(tr->xp, ppos[ping].data(), n4 * 4);
        if (tr->vp) std::memcpy(tr->vp, pvel[ping].data(), n4 * 4);
    }
    ref_dispatch_calculateDensities(&u, b, g128, nullptr, nullptr);  // :322-326
    if (tr) {
        if (tr->density) std::memcpy(tr->density, dens[ping].data(), n * 4);
        if (tr->near_density) std::memcpy(tr->near_density, near[ping].data(), n * 4);
    }
    if (jacobi) {  // :339-343 with pre-pass neighbour velocities
        std::vector<float> orig = vel[ping], out(n4);
        Jacobi j{n, vel[ping].data(), orig.data(), out.data()};
        ref_dispatch_applyPressureAndViscosityForce(&u, b, g128, jacobi_hook, &j);
        vel[ping] = out;
    } else {
        ref_dispatch_applyPressureAndViscosityForce(&u, b, g128, nullptr, nullptr);
    }
    if (tr && tr->vel_force) std::memcpy(tr->vel_force, vel[ping].data(), n4 * 4);
    ref_dispatch_updateVelocities(&u, b, g128, nullptr, nullptr);  // :367-371
    if (tr && tr->colors) std::memcpy(tr->colors, col[ping].data(), n4 * 4);
    std::memcpy(pos4, pos[ping].data(), n4 * 4);
    std::memcpy(vel4, vel[ping].data(), n4 * 4);
    return 0;
}

// The four radix passes alone (commands.c:106-161) over caller keys with
// particleIndex = slot, as testSort() drives them (main.c:274-338).
extern "C" int ref_sort(uint32_t n, const uint32_t* keys, uint32_t blocks, uint32_t* out_keys,
                        uint32_t* out_vals) {
    if (n == 0) return 0;
    std::vector<Entry> cells[2];
    for (int k = 0; k < 2; k++) cells[k].resize(n);
    for (uint32_t i = 0; i < n; i++) cells[0][i] = {keys[i], i};
    const uint32_t per_group_host = 128u * blocks;
    const uint32_t groups = (n + per_group_host - 1) / per_group_host;
    std::vector<uint32_t> hist(std::max<size_t>(n, 256 * (size_t)groups), 0u);
    RefUbo u{};
    u.numParticles = (int)n;
    int ping = 0;
    void* b[32];
    for (int pass = 0; pass < 4; pass++) {
        for (int i = 0; i < 32; i++) b[i] = nullptr;
        b[6] = cells[ping].data();
        b[16] = cells[1 - ping].data();
        b[17] = hist.data();
        u.g_num_elements = n;
        u.g_shift = 8u * pass;
        u.g_num_workgroups = groups;
        u.g_num_blocks_per_workgroup = blocks;
        ref_dispatch_multiRadixSortHistograms(&u, b, groups, nullptr, nullptr);
        ref_dispatch_multiRadixSort(&u, b, groups, nullptr, nullptr);
        ping = 1 - ping;
    }
    for (uint32_t i = 0; i < n; i++) {
        out_keys[i] = cells[ping][i].key;
        out_vals[i] = cells[ping][i].particleIndex;
    }
    return 0;
}

// updateDensityMap as commands.c:416-424 dispatches it: ceil(image / 8)
// workgroups of 8^3 per axis over the image renderer.c:774-781 allocates
// (ix x iy x iz voxels, x fastest), reading the positions and the cell table
// of the last sort through descriptor set ping (bindings 2, 8 and 18).
// Voxels the shader skips keep the 0 written here first.
extern "C" int ref_density_map(const ref_params* p, uint32_t n, const float* pos4,
                               const int32_t* start, const int32_t* end, float cell_size, int ix,
                               int iy, int iz, float* out) {
    if (ix <= 0 || iy <= 0 || iz <= 0) return 0;
    RefUbo u{};
    u.numParticles = (int)n;
    u.particleRadius = p->particleRadius;
    u.smoothingRadius = p->smoothingRadius;
    u.g = p->g;
    for (int a = 0; a < 3; a++) { u.minXYZ[a] = p->minXYZ[a]; u.maxXYZ[a] = p->maxXYZ[a]; }
    u.dt = p->dt;
    u.particleMass = p->particleMass;
    u.pressureMultiplier = p->pressureMultiplier;
    u.targetDensity = p->targetDensity;
    u.viscosityStrength = p->viscosityStrength;
    u.volume = p->volume;
    u.nearPressureMultiplier = p->nearPressureMultiplier;
    u.densityCellSize = cell_size;
    void* b[32] = {};
    b[2] = const_cast<float*>(pos4);
    b[8] = const_cast<int32_t*>(start);
    b[18] = const_cast<int32_t*>(end);
    for (size_t k = 0; k < (size_t)ix * iy * iz; k++) out[k] = 0.0f;
    ref_dispatch3_updateDensityMap(&u, b, (uint)((ix + 7) / 8 * 8), (uint)((iy + 7) / 8 * 8),
                                   (uint)((iz + 7) / 8 * 8), out, ix, iy, iz);
    return 0;
}

static RefUbo render_ubo(const ref_params* p) {
    RefUbo u{};
    u.numParticles = 1;
    u.particleRadius = p->particleRadius;
    u.smoothingRadius = p->smoothingRadius;
    u.g = p->g;
    for (int a = 0; a < 3; a++) { u.minXYZ[a] = p->minXYZ[a]; u.maxXYZ[a] = p->maxXYZ[a]; }
    u.dt = p->dt;
    u.particleMass = p->particleMass;
    u.volume = p->volume;
    return u;
}

// calculateLightVolume as commands.c:437-445 dispatches it over the light
// volume (ceil(dims / 8) workgroups of 8^3), sampling the density map dmap
// (ddims, x fastest) through binding 22.
extern "C" int ref_light_volume(const ref_params* p, const float* dmap, const int32_t ddims[3],
                                float light_step, const float sun[3], const int32_t ldims[3],
                                float* out) {
    RefUbo u = render_ubo(p);
    u.lightMarchStepSize = light_step;
    for (int a = 0; a < 3; a++) u.dirToSun[a] = sun[a];
    void* b[32] = {};
    glsl::RtBind rb{};
    rb.img3.data = out;
    rb.img3.nx = ldims[0]; rb.img3.ny = ldims[1]; rb.img3.nz = ldims[2];
    rb.tex[22].data = dmap;
    rb.tex[22].nx = ddims[0]; rb.tex[22].ny = ddims[1]; rb.tex[22].nz = ddims[2];
    for (size_t k = 0; k < (size_t)ldims[0] * ldims[1] * ldims[2]; k++) out[k] = 0.0f;
    ref_dispatch_rt_calculateLightVolume(&u, b, (uint)((ldims[0] + 7) / 8 * 8), (uint)((ldims[1] + 7) / 8 * 8),
                                         (uint)((ldims[2] + 7) / 8 * 8), &rb);
    return 0;
}

// volumetricFluid as commands.c:447-453 dispatches it (16 x 16 workgroups
// over width x height), with the density map at binding 22 and the light
// volume at binding 24; rgba is x-fastest float4.
extern "C" int ref_volumetric(const ref_params* p, const float* dmap, const int32_t ddims[3],
                              const float* lvol, const int32_t ldims[3], const float cam[12],
                              float fov, float step, const float ext[3], int width, int height,
                              float* rgba) {
    RefUbo u = render_ubo(p);
    u.width = width;
    u.height = height;
    u.stepSize = step;
    u.FOV = fov;
    for (int a = 0; a < 3; a++) {
        u.extinctionCoefficients[a] = ext[a];
        u.camPosition[a] = cam[a];
        u.camForward[a] = cam[3 + a];
        u.camRight[a] = cam[6 + a];
        u.camUp[a] = cam[9 + a];
    }
    void* b[32] = {};
    glsl::RtBind rb{};
    rb.img2.data = rgba;
    rb.img2.nx = width; rb.img2.ny = height;
    rb.tex[22].data = dmap;
    rb.tex[22].nx = ddims[0]; rb.tex[22].ny = ddims[1]; rb.tex[22].nz = ddims[2];
    rb.tex[24].data = lvol;
    rb.tex[24].nx = ldims[0]; rb.tex[24].ny = ldims[1]; rb.tex[24].nz = ldims[2];
    for (size_t k = 0; k < (size_t)width * height * 4; k++) rgba[k] = 0.0f;
    ref_dispatch_rt_volumetricFluid(&u, b, (uint)((width + 15) / 16 * 16), (uint)((height + 15) / 16 * 16),
                                    1u, &rb);
    return 0;
}

// properFluid as commands.c:461-467 dispatches it (16 x 16 workgroups over
// width x height), with the density map as sampler (binding 22) and as the
// image whose size the normal's finite differences use (binding 21).
extern "C" int ref_refractive(const ref_params* p, const float* dmap, const int32_t ddims[3],
                              const float cam[12], float fov, float step, float light_step,
                              const float ext[3], int num_refractions, float threshold, float ior,
                              int width, int height, float* rgba) {
    RefUbo u = render_ubo(p);
    u.width = width;
    u.height = height;
    u.stepSize = step;
    u.lightMarchStepSize = light_step;
    u.FOV = fov;
    u.numRefractions = num_refractions;
    u.surfaceDensityThreshold = threshold;
    u.indexOfRefraction = ior;
    for (int a = 0; a < 3; a++) {
        u.extinctionCoefficients[a] = ext[a];
        u.camPosition[a] = cam[a];
        u.camForward[a] = cam[3 + a];
        u.camRight[a] = cam[6 + a];
        u.camUp[a] = cam[9 + a];
    }
    void* b[32] = {};
    glsl::RtBind rb{};
    rb.img2.data = rgba;
    rb.img2.nx = width; rb.img2.ny = height;
    rb.img3.data = const_cast<float*>(dmap);
    rb.img3.nx = ddims[0]; rb.img3.ny = ddims[1]; rb.img3.nz = ddims[2];
    rb.tex[22].data = dmap;
    rb.tex[22].nx = ddims[0]; rb.tex[22].ny = ddims[1]; rb.tex[22].nz = ddims[2];
    for (size_t k = 0; k < (size_t)width * height * 4; k++) rgba[k] = 0.0f;
    ref_dispatch_rt_properFluid(&u, b, (uint)((width + 15) / 16 * 16), (uint)((height + 15) / 16 * 16),
                                1u, &rb);
    return 0;
}

// The rasterisation pipeline's vertex stage (shader.vert) for one quad corner
// of instance `instance`, with the UBO's matrices and particleRadius.
extern "C" void ref_splat_vertex(const float model[16], const float view[16], const float proj[16], float radius,
                                 float qx, float qy, const float pos[3], int instance, float clip[4]) {
    RefUbo u{};
    u.particleRadius = radius;
    for (int k = 0; k < 16; k++) {
        u.model[k] = model[k];
        u.view[k] = view[k];
        u.proj[k] = proj[k];
    }
    ref_vertex_shader_vert(&u, qx, qy, pos, instance, clip);
}

// Its fragment stage (shader.frag) for particle `index` (colors: float4 per
// particle, binding 9) at fragQuadPos; returns 1 if the fragment is discarded.
extern "C" int ref_splat_fragment(const float* colors, int index, float qx, float qy, float out[4]) {
    RefUbo u{};
    void* b[32] = {};
    b[9] = const_cast<float*>(colors);
    return ref_fragment_shader_frag(&u, b, index, qx, qy, out);
}
