// glsl_dispatch.hpp — vkCmdDispatch emulation for the shader structs the
// harness generator writes (TEST INFRASTRUCTURE, see glsl_ref.py).
#pragma once

#include <cstdint>
#include <memory>
#include <thread>
#include <vector>

#include "glsl_emu.hpp"

namespace glsl {

// Uniform block + push constants as the reference's host fills them
// (src/main.c:53-63, src/renderer/commands.c:118-143).
struct RefUbo {
    int numParticles;
    float particleRadius, smoothingRadius, g;
    float minXYZ[3];
    float dt;
    float maxXYZ[3];
    float particleMass, pressureMultiplier, targetDensity, viscosityStrength, volume,
        nearPressureMultiplier;
    uint g_num_elements, g_shift, g_num_workgroups, g_num_blocks_per_workgroup;
    float densityCellSize;
    // render-mode uniforms (volumetricFluid.comp / calculateLightVolume.comp UBO)
    int width, height, frameCount;
    float stepSize, lightMarchStepSize, FOV;
    float extinctionCoefficients[3], dirToSun[3];
    float camPosition[3], camForward[3], camRight[3], camUp[3];
    // UBO matrices (column-major), read by the rasterisation shaders
    float model[16], view[16], proj[16];
    // refractive mode (properFluid.comp UBO)
    int numRefractions;
    float surfaceDensityThreshold, indexOfRefraction;
};

// Images and samplers of a render-mode dispatch: the shader's image3D and
// image2D, and its sampler3D uniforms by binding.
struct RtBind {
    Image3D img3;
    Image2D img2;
    Sampler3D tex[32];
};

template <class S>
void set_uniforms(S& s, const RefUbo& u) {
    if constexpr (requires { s.numParticles; }) s.numParticles = u.numParticles;
    if constexpr (requires { s.particleRadius; }) s.particleRadius = u.particleRadius;
    if constexpr (requires { s.smoothingRadius; }) s.smoothingRadius = u.smoothingRadius;
    if constexpr (requires { s.g; }) s.g = u.g;
    if constexpr (requires { s.minXYZ; }) s.minXYZ = vec3(u.minXYZ[0], u.minXYZ[1], u.minXYZ[2]);
    if constexpr (requires { s.maxXYZ; }) s.maxXYZ = vec3(u.maxXYZ[0], u.maxXYZ[1], u.maxXYZ[2]);
    if constexpr (requires { s.dt; }) s.dt = u.dt;
    if constexpr (requires { s.particleMass; }) s.particleMass = u.particleMass;
    if constexpr (requires { s.pressureMultiplier; }) s.pressureMultiplier = u.pressureMultiplier;
    if constexpr (requires { s.targetDensity; }) s.targetDensity = u.targetDensity;
    // the shaders spell this field three ways; none of them reads it
    if constexpr (requires { s.viscosityStrength; }) s.viscosityStrength = u.viscosityStrength;
    if constexpr (requires { s.visocosityStrength; }) s.visocosityStrength = u.viscosityStrength;
    if constexpr (requires { s.visosityStrength; }) s.visosityStrength = u.viscosityStrength;
    if constexpr (requires { s.volume; }) s.volume = u.volume;
    if constexpr (requires { s.nearPressureMultiplier; }) s.nearPressureMultiplier = u.nearPressureMultiplier;
    if constexpr (requires { s.g_num_elements; }) s.g_num_elements = u.g_num_elements;
    if constexpr (requires { s.g_shift; }) s.g_shift = u.g_shift;
    if constexpr (requires { s.g_num_workgroups; }) s.g_num_workgroups = u.g_num_workgroups;
    if constexpr (requires { s.g_num_blocks_per_workgroup; })
        s.g_num_blocks_per_workgroup = u.g_num_blocks_per_workgroup;
    if constexpr (requires { s.densityCellSize; }) s.densityCellSize = u.densityCellSize;
    if constexpr (requires { s.width; }) s.width = u.width;
    if constexpr (requires { s.height; }) s.height = u.height;
    if constexpr (requires { s.frameCount; }) s.frameCount = u.frameCount;
    if constexpr (requires { s.stepSize; }) s.stepSize = u.stepSize;
    if constexpr (requires { s.lightMarchStepSize; }) s.lightMarchStepSize = u.lightMarchStepSize;
    if constexpr (requires { s.FOV; }) s.FOV = u.FOV;
    if constexpr (requires { s.extinctionCoefficients; })
        s.extinctionCoefficients =
            vec3(u.extinctionCoefficients[0], u.extinctionCoefficients[1], u.extinctionCoefficients[2]);
    if constexpr (requires { s.dirToSun; }) s.dirToSun = vec3(u.dirToSun[0], u.dirToSun[1], u.dirToSun[2]);
    if constexpr (requires { s.model.m; }) {
        for (int k = 0; k < 16; k++) {
            s.model.m[k] = u.model[k];
            s.view.m[k] = u.view[k];
            s.proj.m[k] = u.proj[k];
        }
    }
    if constexpr (requires { s.numRefractions; }) s.numRefractions = u.numRefractions;
    if constexpr (requires { s.surfaceDensityThreshold; }) s.surfaceDensityThreshold = u.surfaceDensityThreshold;
    if constexpr (requires { s.indexOfRefraction; }) s.indexOfRefraction = u.indexOfRefraction;
    if constexpr (requires { s.camera.position; }) {
        s.camera.position = vec3(u.camPosition[0], u.camPosition[1], u.camPosition[2]);
        s.camera.forward = vec3(u.camForward[0], u.camForward[1], u.camForward[2]);
        s.camera.right = vec3(u.camRight[0], u.camRight[1], u.camRight[2]);
        s.camera.up = vec3(u.camUp[0], u.camUp[1], u.camUp[2]);
    }
}

// Barrier-free dispatch of nx x ny x nz invocations with images and samplers.
template <class S>
void dispatch_rt(const RefUbo& u, void* const* bindings, uint nx, uint ny, uint nz, const RtBind& rb) {
    for (uint z = 0; z < nz; z++)
        for (uint y = 0; y < ny; y++)
            for (uint x = 0; x < nx; x++) {
                auto s = std::make_unique<S>();
                s->gl_GlobalInvocationID = uvec3(x, y, z);
                set_uniforms(*s, u);
                for (int b = 0; b < 32; b++)
                    if (bindings[b]) s->bind(b, bindings[b]);
                s->bind_rt(rb);
                s->main();
            }
}

// Barrier-free 3-D dispatch of nx x ny x nz invocations (workgroups of 8^3 in
// the reference; without shared memory the grouping does not matter), with
// the shader's image bound to img.
template <class S>
void dispatch3(const RefUbo& u, void* const* bindings, uint nx, uint ny, uint nz, Image3D img) {
    for (uint z = 0; z < nz; z++)
        for (uint y = 0; y < ny; y++)
            for (uint x = 0; x < nx; x++) {
                auto s = std::make_unique<S>();
                s->gl_GlobalInvocationID = uvec3(x, y, z);
                set_uniforms(*s, u);
                for (int b = 0; b < 32; b++)
                    if (bindings[b]) s->bind(b, bindings[b]);
                s->bind_image(img);
                s->main();
            }
}

// Called after each invocation of a barrier-free dispatch (the harness uses
// it to give the force pass Jacobi semantics).
typedef void (*InvocationHook)(void* ctx, uint global_id);

template <class S>
void dispatch(const RefUbo& u, void* const* bindings, uint groups, uint local, bool workgroup_threads,
              InvocationHook hook, void* ctx) {
    if (!workgroup_threads) {
        for (uint g = 0; g < groups; g++)
            for (uint l = 0; l < local; l++) {
                auto s = std::make_unique<S>();
                s->gl_GlobalInvocationID = uvec3(g * local + l, 0u, 0u);
                s->gl_LocalInvocationID = uvec3(l, 0u, 0u);
                s->gl_WorkGroupID = uvec3(g, 0u, 0u);
                s->gl_SubgroupID = l / 32;
                s->gl_SubgroupInvocationID = l % 32;
                set_uniforms(*s, u);
                for (int b = 0; b < 32; b++)
                    if (bindings[b]) s->bind(b, bindings[b]);
                s->main();
                if (hook) hook(ctx, g * local + l);
            }
        return;
    }
    for (uint g = 0; g < groups; g++) {
        auto wg = std::make_unique<Workgroup>();
        std::barrier<> bar((std::ptrdiff_t)local);
        wg->bar = &bar;
        std::vector<std::thread> threads;
        threads.reserve(local);
        for (uint l = 0; l < local; l++) {
            threads.emplace_back([&, l]() {
                auto s = std::make_unique<S>();
                s->gl_GlobalInvocationID = uvec3(g * local + l, 0u, 0u);
                s->gl_LocalInvocationID = uvec3(l, 0u, 0u);
                s->gl_WorkGroupID = uvec3(g, 0u, 0u);
                s->gl_SubgroupID = l / 32;
                s->gl_SubgroupInvocationID = l % 32;
                s->wg = wg.get();
                set_uniforms(*s, u);
                for (int b = 0; b < 32; b++)
                    if (bindings[b]) s->bind(b, bindings[b]);
                s->bind_shared(wg->smem);
                s->main();
            });
        }
        for (auto& t : threads) t.join();
    }
}

}  // namespace glsl
