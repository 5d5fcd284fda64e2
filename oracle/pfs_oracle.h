/*
 * pfs_oracle.h — CPU restatement of the reference's SPH world step.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA step and
 * the timed CPU baseline of bench.py; only tests/, __graft_entry__.smoke()
 * and bench.py's CPU legs load it.  The product library never links it and has
 * no CPU fallback.
 *
 * Parity pin: the reference publishes no tests or golden vectors.  This
 * restatement is pinned against the reference's own shader sources executed
 * on the CPU (oracle/glsl_ref.py compiles the src/shaders compute shaders as C++ under a
 * GLSL emulation header and replays commands.c:193-402), and against the
 * golden fixtures in tests/golden/ that script produced.
 *
 * Arithmetic contract: IEEE float32, round to nearest, no contraction
 * (built with -O2 -ffp-contract=off, never -ffast-math), expressions evaluated
 * in the shaders' order.  Derived constants are computed once on the host
 * (pfso_derive) and shared with the device.
 *
 * Deliberate differences from the reference, each stated where it applies:
 *   - viscosity reads the neighbours' pre-update velocities (Jacobi); the
 *     reference races on the same buffer (applyPressureAndViscosityForce.comp
 *     :159 reads velocities[j] while :182 writes velocities[i]);
 *   - the cell table is built from the fully sorted order (the reference
 *     reads the pass-2 output, identical whenever keys < 2^24, which
 *     PFS_MAX_PARTICLES guarantees);
 *   - float -> cell coordinate conversion saturates (int range, NaN -> 0)
 *     where GLSL leaves out-of-range conversions undefined.
 */
#ifndef PFS_ORACLE_H
#define PFS_ORACLE_H

#include <stdint.h>
#include "../include/pfs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfso_consts {
    float    volume;            /* 2*pi*h^5/15, double -> float (main.c:349)          */
    float    near_inv;          /* 15/(PI*h^6)  (calculateDensities.comp:110)          */
    float    slope_scale;       /* 15/(PI*h^5)  (applyPressureAndViscosityForce:89)    */
    float    near_slope_scale;  /* -45/(PI*h^6) (applyPressureAndViscosityForce:104)   */
    float    r2;                /* h*h          (applyPressureAndViscosityForce:128)   */
    float    skip_d2;           /* least d2 with sqrtf(d2) >= h: candidates at or above
                                   it contribute exactly zero                           */
    float    margin_i;          /* integrate wall margin                                */
    uint32_t mask;              /* n - 1        (updateCellEntries.comp:54-57)          */
} pfso_consts;

void     pfso_derive(const pfs_params* p, uint32_t n, pfso_consts* c);
uint32_t pfso_cell_hash(uint32_t cx, uint32_t cy, uint32_t cz);
int32_t  pfso_cell_coord(float v, float lo, float h);
uint32_t pfso_point_key(const pfs_params* p, uint32_t mask, const float* xyz);

void pfso_keys(const pfs_params* p, uint32_t n, const float* pos4, uint32_t* keys);
void pfso_sort(uint32_t n, const uint32_t* keys, uint32_t* sorted_keys,
               uint32_t* perm);
void pfso_table(uint32_t n, const uint32_t* sorted_keys, int32_t* start,
                int32_t* end);
void pfso_predict(const pfs_params* p, uint32_t n, const float* pos4,
                  const float* vel4, float* xp4, float* vp4);
void pfso_density(const pfs_params* p, uint32_t n, const float* xp4,
                  const int32_t* start, const int32_t* end, float* density,
                  float* near_density);
void pfso_force(const pfs_params* p, uint32_t n, const float* xp4,
                const float* vp4, const float* vel4, const float* density,
                const float* near_density, const int32_t* start,
                const int32_t* end, float* vel_out4);
void pfso_integrate(const pfs_params* p, uint32_t n, float* pos4, float* vel4,
                    float* rgba4);
void pfso_color(const float* vel4, float* rgba4);

/* One substep in place: pos4/vel4 (n float4) end in sorted order, as the
 * reference's buffers do.  trace (optional) receives every stage output;
 * density/near_density (optional, n) receive the substep's densities;
 * ids (optional, n) is permuted along with the particles. */
int pfso_substep(const pfs_params* p, uint32_t n, float* pos4, float* vel4,
                 pfs_debug_substep* trace, float* density, uint32_t* ids,
                 float* rgba4);
/* nsteps * p->substeps substeps. */
int pfso_step(const pfs_params* p, uint32_t n, float* pos4, float* vel4,
              uint32_t nsteps, float* density, uint32_t* ids);

/* FP64 evaluation of one substep's density and velocity update for a subset
 * of sorted slots, on the same neighbour sets the float path visits (cell
 * keys and table decisions in float as the reference takes them, all
 * accumulation in double).  Inputs are the sorted float state after the
 * reorder stage: xp4, vp4, vel4 (pre-force velocities), start/end.
 * Outputs per subset entry: density, near density, velocity after the force
 * pass (3 doubles). */
void pfso_subset_f64(const pfs_params* p, uint32_t n, const float* xp4,
                     const float* vp4, const float* vel4, const int32_t* start,
                     const int32_t* end, uint32_t m, const uint32_t* subset,
                     double* density, double* near_density, double* vel3);

/* Threads the OpenMP loops use (0 = runtime default). */
/* Density map of the state (updateDensityMap.comp:93-147), see pfs_oracle.c. */
void pfso_density_map_extent(const pfs_params* p, float cell_size, int32_t image[3],
                             int32_t bound[3]);
void pfso_density_map(const pfs_params* p, uint32_t n, const float* pos4, const int32_t* start,
                      const int32_t* end, float cell_size, float* out);

/* Volumetric rendering over the density map (calculateLightVolume.comp,
 * volumetricFluid.comp), see pfs_oracle.c.  cam = position, forward, right,
 * up (3 floats each). */
float pfso_texture3d(const float* img, const int32_t dims[3], const float uvw[3]);
void pfso_light_volume(const pfs_params* p, const float* dmap, const int32_t ddims[3],
                       float light_step, const float sun[3], const int32_t ldims[3], float* out);
void pfso_volumetric(const pfs_params* p, const float* dmap, const int32_t ddims[3],
                     const float* lvol, const int32_t ldims[3], const float cam[12],
                     float half_height, float step, const float extinction[3], uint32_t width,
                     uint32_t height, float* rgba);

/* Refractive render mode (properFluid.comp) over the density map, see
 * pfs_oracle.c. */
void pfso_refractive(const pfs_params* p, const float* dmap, const int32_t ddims[3], const float cam[12],
                     float half_height, float step, float light_step, const float extinction[3],
                     int32_t num_refractions, float threshold, float ior, uint32_t width,
                     uint32_t height, float* rgba);

/* FXAA of a width x height float4 image (raymarchShader.frag) and the
 * point-splat rasteriser (shader.vert / shader.frag), see pfs_oracle.c. */
void pfso_fxaa(const float* in, uint32_t width, uint32_t height, float* out);
void pfso_splat_camera(const float model[16], const float view[16], const float proj[16], float mvp[16],
                       float right[3], float up[3]);
void pfso_splat_clip(const float mvp[16], const float pos[3], const float right[3], const float up[3],
                     float r, float qx, float qy, float clip[4]);
int pfso_splat_geometry(const float mvp[16], const float right[3], const float up[3], float r,
                        const float pos[3], uint32_t width, uint32_t height, float sq[4], float* depth);
int pfso_splat_quadpos(const float sq[4], int32_t x, int32_t y, float* qx, float* qy);
void pfso_splat_shade(const float color[4], float qx, float qy, float out[4]);
void pfso_splats(uint32_t n, const float* pos4, const float* color4, const float mvp[16],
                 const float right[3], const float up[3], float radius, uint32_t width, uint32_t height,
                 float* rgba, float* depth);

void pfso_set_threads(int threads);
int  pfso_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
