/*
 * pfs.h — C ABI of the B200 SPH world step.
 *
 * The reference (mojofill/particle-fluid-simulation) has no library API: its
 * world step is the substep block recorded by recordCommands()
 * (src/renderer/commands.c:193-402), fed by the uniform buffer written in
 * updateUniforms() (src/main.c:37-82) and by the particle buffers created in
 * initialize*Buffer() (src/renderer/renderer.c:510-754).  The entry points
 * below replace that block for a host application: the caller owns host
 * arrays, the world owns device state, every call returns 0 or a negative
 * PFS_E* code and none ever exits the process.
 *
 * Threading: one world must not be used by two host threads at once; distinct
 * worlds may be used concurrently.  All device work of a world runs on the
 * world's own CUDA stream.
 *
 * Layouts: pos4/vel4/rgba4 are arrays of n float4 (x, y, z, w) in std430 vec4
 * order, as the reference's PositionsBuffer/VelocitiesBuffer
 * (src/shaders/predictPositions.comp:27-28).  After a step the particles are
 * stored in the order of the last cell-key sort, exactly as the reference
 * leaves its ping-pong buffers (src/shaders/scatterPass.comp:50-65).
 */
#ifndef PFS_H
#define PFS_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PFS_API __attribute__((visibility("default")))
#else
#define PFS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define PFS_OK          0
#define PFS_EINVAL     (-1)  /* bad argument or parameter set               */
#define PFS_ENOMEM     (-2)  /* device or host allocation failed            */
#define PFS_ECUDA      (-3)  /* a CUDA runtime call failed                   */
#define PFS_ETIMEDOUT  (-4)  /* bounded wait ran out                         */
#define PFS_ENODEV     (-5)  /* no usable CUDA device                        */
#define PFS_EDEVICE    (-6)  /* a kernel's own bounds check tripped          */
#define PFS_ERANGE     (-7)  /* a size beyond a documented limit             */
#define PFS_EBUDGET    (-8)  /* request refused by the HBM budget            */
#define PFS_ENOTFOUND  (-9)  /* unknown scene / request handle               */

/* The cell table has one slot per particle and keys are masked by n-1
 * (src/shaders/updateCellEntries.comp:54-57).  The reference's table read
 * (src/renderer/commands.c:295-299) is only the fully sorted order when all
 * keys fit in 24 bits, so n is limited to 2^24 per table. */
#define PFS_MAX_PARTICLES (1u << 24)

/* ---- precision forms ----------------------------------------------------- */
#define PFS_FP32       0  /* plain form: FP32 throughout, the reference's IEEE
                             operation sequence (bit-exact with the oracle)   */
#define PFS_FP16_CELL  1  /* bandwidth form: FP16 cell-relative neighbor data  */
#define PFS_FP32_FAST  2  /* plain form with fused multiply-adds and hardware
                             reciprocal square roots in the neighbour sums:
                             same candidates, FP32 throughout, held to 1e-5
                             relative density and velocity error per step;
                             keys, sort and table stay bit-exact             */

/* ---- flags --------------------------------------------------------------- */
#define PFS_FLAG_COLORS  1  /* write the speed colour ramp every substep
                               (src/shaders/updateVelocities.comp:120-141)   */
#define PFS_FLAG_IDS     2  /* track each slot's creation index
                               (pfs_world_read_ids)                           */

/*
 * Physics parameters.  Field ↔ reference uniform (src/renderer/vk_types.h:48-65,
 * filled in src/main.c:53-63):
 *   h                         smoothingRadius
 *   target_density            targetDensity
 *   pressure_multiplier       pressureMultiplier
 *   near_pressure_multiplier  nearPressureMultiplier
 *   viscosity                 scale on the viscosity sum; the reference leaves
 *                             the sum unscaled (its visocosityStrength is never
 *                             read), which is viscosity = 1
 *   particle_mass             particleMass
 *   gravity                   the reference hardcodes (0, 0, -g)
 *   dt                        per-substep dt (DELTA_TIME / NUM_SUBSTEPS, main.c:57)
 *   box_min / box_max         minXYZ / maxXYZ
 *   margin_predict            wall margin of the predict pass (particleRadius)
 *   margin_integrate          wall margin of the integrate pass
 *                             (particleRadius + 0.5, updateVelocities.comp:81)
 *   restitution[6]            velocity factor after a wall hit, walls in the
 *                             order -x,+x,-y,+y,-z,+z; reference 1,1,1,1,0.95,1
 *   volume                    density normaliser; <= 0 derives 2*pi*h^5/15 in
 *                             double precision as main.c:349 does
 *   substeps                  substeps per pfs_world_step step (NUM_SUBSTEPS)
 *   precision                 PFS_FP32, PFS_FP32_FAST or PFS_FP16_CELL
 *   flags                     PFS_FLAG_*
 */
typedef struct pfs_params {
    float   h;
    float   target_density;
    float   pressure_multiplier;
    float   near_pressure_multiplier;
    float   viscosity;
    float   particle_mass;
    float   gravity[3];
    float   dt;
    float   box_min[3];
    float   box_max[3];
    float   margin_predict;
    float   margin_integrate;
    float   restitution[6];
    float   volume;
    int32_t substeps;
    int32_t precision;
    int32_t flags;
    int32_t reserved;
} pfs_params;

/* Fill p with the reference's compile-time defaults (src/main.c:11-30,
 * 349-358): h = 2.5, g = 100 along -z, dt = 0.01, one substep, mass 1,
 * pressure multiplier 15000, target density 1, viscosity term unscaled,
 * near-pressure 0, box [-140,140]x[-40,40]x[-40,40], particle radius 0.3. */
PFS_API void pfs_params_reference_default(pfs_params* p);

/* Check a parameter set without touching the GPU.  Returns PFS_OK or
 * PFS_EINVAL. */
PFS_API int pfs_params_validate(const pfs_params* p);

PFS_API const char* pfs_strerror(int status);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
PFS_API int pfs_version(void);

/* ---- world: one scene ------------------------------------------------------
 * pfs_world_create  replaces initRenderer's particle buffer setup
 *                   (renderer.c:510-754) for caller-supplied initial state.
 * pfs_world_step    replaces the substep loop of recordCommands
 *                   (commands.c:193-402) + vkQueueSubmit (renderer.c:419);
 *                   runs nsteps * params.substeps substeps asynchronously.
 * pfs_world_sync    replaces vkQueueWaitIdle (renderer.c:449) with a bounded
 *                   wait (timeout_ns = 0 waits without limit).
 * pfs_world_read    copies state out (any pointer may be NULL):
 *                   pos4/vel4 (n float4), density (n floats, last substep),
 *                   keys (n sorted cell keys of the last sort, the key field of
 *                   cellEntries after multiRadixSort, commands.c:240-243) and
 *                   perm (n indices: sorted slot s came from pre-sort slot
 *                   perm[s], the particleIndex field before scatterPass.comp:64
 *                   resets it).
 * pfs_world_write   replaces the state (the R-key reset path, main.c:85-98).
 */
typedef struct pfs_world pfs_world;

PFS_API int pfs_world_create(const pfs_params* p, uint32_t n, const float* pos4,
                     const float* vel4, pfs_world** out);
PFS_API int pfs_world_set_params(pfs_world* w, const pfs_params* p);
PFS_API int pfs_world_step(pfs_world* w, uint32_t nsteps);
PFS_API int pfs_world_sync(pfs_world* w, uint64_t timeout_ns);

/* Pipelined host-to-host stepping (no reference counterpart): for each k in
 * [0, count), the same as pfs_world_write(pos_in[k], vel_in[k]),
 * pfs_world_step(steps_each), pfs_world_read(pos_out[k], vel_out[k]) in
 * turn, with the same results, but input k + 1 is uploaded and output k - 1
 * read back on the world's own copy streams while input k steps
 * (double-buffered device staging, 128 bytes per particle, kept until
 * destroy).  The host buffers must stay untouched until the call returns;
 * pinned memory lets the copies overlap the steps.  vel_in, vel_out and their
 * entries may be NULL (zero velocities in; velocities not read back).
 * Returns when every output is written. */
PFS_API int pfs_world_run_pipelined(pfs_world* w, uint32_t count, const float* const* pos_in,
                                    const float* const* vel_in, float* const* pos_out,
                                    float* const* vel_out, uint32_t steps_each);
PFS_API int pfs_world_read(pfs_world* w, float* pos4, float* vel4, float* density,
                   uint32_t* keys, uint32_t* perm);
PFS_API int pfs_world_write(pfs_world* w, const float* pos4, const float* vel4);
PFS_API int pfs_world_destroy(pfs_world* w);

/* Extra reads.  colors: n float4 speed ramp of the last substep (needs
 * PFS_FLAG_COLORS).  ids: n creation indices (slot s holds the particle that
 * was created at ids[s]); the reference does not track identity. */
PFS_API int pfs_world_read_colors(pfs_world* w, float* rgba4);
PFS_API int pfs_world_read_ids(pfs_world* w, uint32_t* ids);

/* Number of particles and the world's CUDA stream (cudaStream_t). */
PFS_API uint32_t pfs_world_size(const pfs_world* w);
PFS_API void*    pfs_world_stream(pfs_world* w);

/* Device-resident state: the world's current position/velocity buffers
 * (n float4 each, device pointers).  Valid until the next step. */
PFS_API int pfs_world_device_state(pfs_world* w, void** pos4_dev, void** vel4_dev);

/* ---- per-stage timing (the reference's vkCmdWriteTimestamp pairs,
 * commands.h:12-43, renderer.c:451-503) ---------------------------------- */
enum {
    PFS_STAGE_SORT = 0,      /* QUERY_SORT (+ QUERY_UPDATE_CELL, fused)        */
    PFS_STAGE_REORDER,       /* QUERY_PREDICT + QUERY_SCATTER + table set       */
    PFS_STAGE_DENSITY,       /* QUERY_DENSITY                                   */
    PFS_STAGE_FORCE,         /* QUERY_PRESSURE_AND_VISCOSITY                    */
    PFS_STAGE_INTEGRATE,     /* QUERY_UPDATE_VELOCITY + next keys + table clear */
    PFS_STAGE_COUNT
};
typedef struct pfs_stage_times {
    double   ms_total[PFS_STAGE_COUNT];  /* summed device time per stage        */
    uint64_t launches[PFS_STAGE_COUNT];  /* kernel launches per stage           */
    uint64_t substeps;                   /* substeps timed                      */
} pfs_stage_times;

/* enable != 0: record CUDA events around every stage of every substep
 * (adds per-stage event overhead; for profiling runs only). */
PFS_API int pfs_world_profile(pfs_world* w, int enable);
/* Read and reset the accumulated stage times (synchronises the world). */
PFS_API int pfs_world_stage_times(pfs_world* w, pfs_stage_times* out);
/* Kernel launches one substep issues (for launch accounting). */
PFS_API int pfs_world_launches_per_substep(const pfs_world* w);

/* ---- staged substep for verification ---------------------------------------
 * Runs ONE substep stage by stage and copies each stage's output to the
 * caller's arrays (any may be NULL):
 *   keys_in   n   cell keys of the state before the sort
 *   keys      n   sorted keys;  perm n  sort permutation
 *   start/end n   cell table after it is built (-1 = empty slot)
 *   xp/vp     4n  predicted positions / velocities (sorted order)
 *   density/near_density n
 *   vel_force 4n  velocities after the pressure/viscosity pass
 * After the call the world holds the integrated state, as after one substep.
 */
typedef struct pfs_debug_substep {
    uint32_t* keys_in;
    uint32_t* keys;
    uint32_t* perm;
    int32_t*  start;
    int32_t*  end;
    float*    xp;
    float*    vp;
    float*    density;
    float*    near_density;
    float*    vel_force;
} pfs_debug_substep;
PFS_API int pfs_world_debug_substep(pfs_world* w, pfs_debug_substep* out);

/* ---- batch: many independent scenes stepped together ------------------------
 * No counterpart in the reference (one scene per app).  Scenes share one
 * table, one sort and one launch per stage: scene s owns particle slots
 * [offset_s, offset_s + n_s) and table slots with the same range, so its cell
 * keys are offset_s + (hash & (n_s - 1)) and one stable sort of all keys keeps
 * every scene contiguous and in exactly the order its own world would have.
 * Each scene's results are therefore bit-identical to stepping it alone.
 * Scenes may be added and removed between steps (the batch repacks on its
 * stream); all scenes of a batch share precision and substep count.
 * Capacity is fixed at creation: max_particles in total, max_scenes. */
typedef struct pfs_batch pfs_batch;

typedef struct pfs_batch_info {
    uint32_t particles;       /* particles of all resident scenes              */
    uint32_t scenes;          /* resident scenes                                */
    uint32_t max_particles;
    uint32_t max_scenes;
    uint64_t device_bytes;    /* device memory the batch holds                  */
    int32_t  launches_per_substep;
    int32_t  reserved;
} pfs_batch_info;

PFS_API int pfs_batch_create(uint32_t max_particles, uint32_t max_scenes, int32_t precision,
                             int32_t substeps, pfs_batch** out);
/* Device bytes a batch of this capacity holds (for admission budgets). */
PFS_API uint64_t pfs_batch_bytes(uint32_t max_particles, uint32_t max_scenes, int32_t precision);
PFS_API int pfs_batch_add_scene(pfs_batch* b, const pfs_params* p, uint32_t n, const float* pos4,
                                const float* vel4, int32_t* scene_id);
PFS_API int pfs_batch_remove_scene(pfs_batch* b, int32_t scene_id);
PFS_API int pfs_batch_step(pfs_batch* b, uint32_t nsteps);
PFS_API int pfs_batch_sync(pfs_batch* b, uint64_t timeout_ns);
PFS_API int pfs_batch_read_scene(pfs_batch* b, int32_t scene_id, float* pos4, float* vel4,
                                 float* density);
PFS_API int pfs_batch_write_scene(pfs_batch* b, int32_t scene_id, const float* pos4,
                                  const float* vel4);
PFS_API int pfs_batch_info_get(pfs_batch* b, pfs_batch_info* out);
/* Feed mode (enable != 0): every step starts from the scenes' input states
 * (the state given to add_scene / write_scene, kept resident), so repeated
 * steps re-run the same inputs; off (default): steps continue the rollout. */
PFS_API int pfs_batch_set_feed(pfs_batch* b, int enable);
PFS_API void* pfs_batch_stream(pfs_batch* b);
PFS_API int pfs_batch_destroy(pfs_batch* b);

/* ---- sorting without allocation ---------------------------------------------
 * No counterpart in the reference (its sort always runs inside the frame's
 * command buffer, commands.c:240-243, on buffers the app allocated up front).
 * For hosts that cannot let a library allocate device memory — an engine or
 * renderer that owns the device heap through its own pools, or a frame loop
 * whose memory plan is fixed, where cudaMalloc would fail or stall the device.
 * Sorts n device-resident keys stably (value = slot index) into the caller's
 * sorted_keys_dev / perm_dev, the same order and kernels as the world step's
 * sort, asynchronously on `stream` (a cudaStream_t; NULL = legacy default).
 * key_bits: low key bits to sort, 1..32; 0 = keys are < n (cell keys).
 * keys_dev, sorted_keys_dev and perm_dev must not overlap (PFS_EINVAL).
 * The scratch is a static device array of about 9 MiB in this library,
 * held on every GPU that loads it until exit; n > PFS_STATIC_SORT_MAX_KEYS
 * returns PFS_ERANGE.  All calls share that array: calls that overlap on the
 * GPU race, so serialise them.  The first call on a device (and the first
 * after a device reset) looks up the array's device address; make it before
 * any stream capture begins. */
#define PFS_STATIC_SORT_MAX_KEYS (1u << 20)
PFS_API int pfs_sort_keys_static(const uint32_t* keys_dev, uint32_t n, uint32_t key_bits,
                                 uint32_t* sorted_keys_dev, uint32_t* perm_dev, void* stream);
/* Device-side status of the last pfs_sort_keys_static call on the current
 * device: waits for `stream` (the stream that call used), then returns
 * PFS_EDEVICE if its kernels' own range checks or bounded waits tripped (the
 * result is then not a valid sort), else PFS_OK. */
PFS_API int pfs_sort_static_status(void* stream);

/* Device error word of the world's kernels (0 = clean).  Reading it
 * synchronises the world. */
PFS_API int pfs_world_device_error(pfs_world* w, uint32_t* word);

/* ---- kernel shapes and the autotuner (no reference counterpart) ----------
 * The FP32 neighbour passes come in five shapes and two neighbour searches
 * (table scan, or the grid search where the grid bound allows it); every
 * combination gives the same results bit for bit, only the time differs
 * (in the PFS_FP32_FAST form the staged shape sums with fused arithmetic and
 * the others exactly).  The staged shape stages each spatial block's
 * neighbourhood in shared memory; it scans table ranges only and needs a
 * grid of at most about 8n cells (PFS_EINVAL otherwise).
 * pfs_world_set_shape picks one; pfs_world_autotune times every candidate
 * over trial_steps steps (0: 2), each started from the world's own state,
 * takes the fastest of them, keeps the fastest candidate and restores the
 * state, so tuning changes no result.  It allocates a snapshot of the state
 * for the duration of the call. */
#define PFS_SHAPE_SIMPLE   0
#define PFS_SHAPE_SLAB     1
#define PFS_SHAPE_LIST     2   /* default */
#define PFS_SHAPE_FLAT     3
#define PFS_SHAPE_STAGED   4
#define PFS_SEARCH_AUTO  (-1)  /* grid when the table has <= n/4 slots */
#define PFS_SEARCH_TABLE   0
#define PFS_SEARCH_GRID    1
#define PFS_TUNE_MAX      12

typedef struct pfs_tune_result {
    int32_t candidates;                /* trials run                         */
    int32_t chosen;                    /* index kept (-1: a trial failed)    */
    int32_t shape[PFS_TUNE_MAX];       /* PFS_SHAPE_* of each trial          */
    int32_t search[PFS_TUNE_MAX];      /* PFS_SEARCH_* of each trial         */
    float   ms_per_step[PFS_TUNE_MAX]; /* device time of each trial          */
} pfs_tune_result;

PFS_API int pfs_world_set_shape(pfs_world* w, int32_t shape, int32_t search);
/* 1 when the world can take the shape (the staged shape needs its
 * shared-memory stage to hold a block's neighbourhood: not for tables with
 * few slots or very dense initial states), else 0. */
PFS_API int pfs_world_shape_available(const pfs_world* w, int32_t shape);
PFS_API int pfs_world_autotune(pfs_world* w, uint32_t trial_steps, pfs_tune_result* out);
/* Batch: one shape for all scenes; search -1 lets each scene choose, 0 forces
 * the table scan everywhere (the candidates the batch autotuner tries). */
PFS_API int pfs_batch_set_shape(pfs_batch* b, int32_t shape, int32_t search);
PFS_API int pfs_batch_autotune(pfs_batch* b, uint32_t trial_steps, pfs_tune_result* out);

/* ---- density map (the reference's updateDensityMap.comp:93-147) ----------
 * The per-voxel density the reference's ray-marching renderers sample (a 3-D
 * image there, a plain float grid here).  dims = the image the reference
 * allocates (renderer.c:774-781): (int)ceil((box_max - box_min) *
 * (1 / cell_size)) voxels per axis in float arithmetic, x fastest.  Each
 * voxel gathers the 27 cells around the cell of its centre with the shader's
 * bounds rule and sums m (h - d)^2 / volume over the table ranges of the last
 * sort (bit-exact); voxels the shader's rule skips are 0.  The world must
 * have stepped since its last write (PFS_EINVAL otherwise).  out: host or
 * device memory of dims[0] * dims[1] * dims[2] floats; the call returns when
 * it is written.  PFS_ERANGE when a dimension exceeds 65536 or the grid 2^31
 * voxels. */
PFS_API int pfs_world_density_map_dims(const pfs_world* w, float cell_size, uint32_t dims[3]);
PFS_API int pfs_world_density_map(pfs_world* w, float cell_size, float* out);

/* ---- volumetric rendering (calculateLightVolume.comp:193-219,
 *      volumetricFluid.comp:196-263) ---------------------------------------
 * The reference's volumetric render mode, headless: the density map above at
 * density_cell_size, a light volume of ceil((box_max - box_min) *
 * (1 / light_step_size)) voxels (renderer.c:812-819) marched toward
 * dir_to_sun, then one ray per pixel from the camera (y = 0 at the top)
 * marched through the box with Beer-Lambert transmittance.  texture() is
 * float trilinear interpolation with clamp to edge (the reference's sampler,
 * image.c:134-164).  As in the shader, light voxels whose index exceeds the
 * box size in world units stay 0 (the reference runs with
 * light_step_size = 1).  rgba: width * height float4 (alpha 1), host or
 * device memory; light_volume: NULL or the light volume's floats. */
typedef struct pfs_volume_view {
    float position[3], forward[3], right[3], up[3];  /* camera (vk_types.h Camera) */
    float fov;                  /* radians (FOV, main.c:25)                        */
    float density_cell_size;    /* densityCellSize (main.c:14)                     */
    float step_size;            /* stepSize (main.c:23)                            */
    float light_step_size;      /* lightMarchStepSize (main.c:24)                  */
    float extinction[3];        /* extinctionCoefficients (main.c:389-390)         */
    float dir_to_sun[3];        /* dirToSun, normalised (main.c:393-394)           */
} pfs_volume_view;

PFS_API int pfs_world_light_volume_dims(const pfs_world* w, float light_step_size, uint32_t dims[3]);
PFS_API int pfs_world_render_volumetric(pfs_world* w, const pfs_volume_view* v, uint32_t width,
                                        uint32_t height, float* rgba, float* light_volume);

/* Refractive render mode (RAYMARCH_FLUID): the density map of the last step
 * (v->density_cell_size) marched per pixel for surface crossings of
 * surface_density_threshold, with reflection and refraction at each crossing
 * and Beer-Lambert attenuation by v->extinction (as given, not normalised),
 * under a white environment (properFluid.comp:151-614; replaces the
 * properFluid dispatch of commands.c:461-467).  Uses the camera, fov,
 * step_size and light_step_size of v (dir_to_sun is not read); rgba as in
 * pfs_world_render_volumetric.  Results equal the oracle's up to the last
 * bits of expf / powf. */
typedef struct pfs_refraction {
    int32_t num_refractions;          /* NUM_REFRACTIONS [3] (main.c:27)            */
    float   surface_density_threshold; /* SURFACE_DENSITY_THRESHOLD [0.75] (main.c:28) */
    float   index_of_refraction;      /* INDEX_OF_REFRACTION [1.333] (main.c:29)    */
    float   reserved;                 /* 0                                           */
} pfs_refraction;

PFS_API int pfs_world_render_refractive(pfs_world* w, const pfs_volume_view* v, const pfs_refraction* r,
                                        uint32_t width, uint32_t height, float* rgba);

/* ---- rasterised splats (shader.vert:27-57, shader.frag:56-87) and FXAA
 *      (raymarchShader.frag:15-73) --------------------------------------------
 * The reference's default render (RENDER_TYPE RASTERIZATION, main.c:32),
 * headless: one camera-facing disc of radius particle_radius per particle at
 * the world's positions (slot order, as the reference binds them), shaded
 * from the speed colour ramp (the world needs PFS_FLAG_COLORS) with the
 * fragment shader's Lambert term and edge alpha; depth test LESS with depth
 * writes, no blending, clear colour 0 and depth 1 (commands.c:186-188,
 * graphics_pipeline.c:114-134).  The matrices are the UBO's (column-major
 * mat4; main.c:37-51 fills them with cglm's lookat / perspective and flips
 * proj[1][1]).  Each quad projects to a screen-aligned square: pixel centres
 * in [min, max) of its corners' screen positions are fragments, fragQuadPos
 * is linear across it, the depth is the particle centre's z / w; a pixel
 * keeps the first particle (slot order) of the smallest depth.  rgba:
 * width * height float4; depth: NULL or width * height floats; host or
 * device memory.  Replaces the vkCmdDraw of commands.c:520-526. */
typedef struct pfs_splat_view {
    float model[16], view[16], proj[16];   /* UniformBufferObject mat4s (vk_types.h) */
    float particle_radius;                 /* particleRadius (main.c:11)            */
    float reserved[3];                     /* 0                                     */
} pfs_splat_view;

PFS_API int pfs_world_render_splats(pfs_world* w, const pfs_splat_view* v, uint32_t width, uint32_t height,
                                    float* rgba, float* depth);

/* FXAA of a width x height float4 image as raymarchShader.frag presents the
 * ray-marched modes (full-screen quad, linear clamp-to-edge sampler of
 * image.c:135-161, fragment (x, y) at outNDC = ((x + 0.5) / width * 2 - 1,
 * (y + 0.5) / height * 2 - 1)); alpha 1.  In and out: host or device memory,
 * not the same buffer; runs on the world's stream. */
PFS_API int pfs_world_fxaa(pfs_world* w, const float* rgba_in, uint32_t width, uint32_t height,
                           float* rgba_out);

#ifdef __cplusplus
}
#endif
#endif /* PFS_H */
