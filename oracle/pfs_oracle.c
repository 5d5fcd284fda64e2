/*
 * pfs_oracle.c — CPU restatement of the reference's SPH world step.
 *
 * TEST INFRASTRUCTURE ONLY (see pfs_oracle.h).  Each function cites the
 * shader lines it restates; file paths are relative to the reference project
 * root.  Build: gcc -O2 -ffp-contract=off -fopenmp (oracle/Makefile).
 */
#include "pfs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* const float PI = 3.14159265359f;  (calculateDensities.comp:75) */
#define REF_PI 3.14159265359f

static int g_threads = 0;

void pfso_set_threads(int threads) { g_threads = threads; }

int pfso_max_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

#ifdef _OPENMP
#define PAR_FOR _Pragma("omp parallel for schedule(static) num_threads(pfso_max_threads())")
#define PAR_FOR_DYN _Pragma("omp parallel for schedule(dynamic, 256) num_threads(pfso_max_threads())")
#else
#define PAR_FOR
#define PAR_FOR_DYN
#endif

/* Derived constants, computed once on the host.  volume follows main.c:349
 * (double arithmetic, stored as float); the three kernel scales follow the
 * float expressions of calculateDensities.comp:110 and
 * applyPressureAndViscosityForce.comp:89,104. */
void pfso_derive(const pfs_params* p, uint32_t n, pfso_consts* c) {
    const float h = p->h;
    if (p->volume > 0.0f)
        c->volume = p->volume;
    else
        c->volume = (float)(2.0f * M_PI * pow((double)h, 5) / 15.0f);
    c->near_inv = 15.0f / (REF_PI * powf(h, 6.0f));
    c->slope_scale = 15.0f / (REF_PI * powf(h, 5.0f));
    c->near_slope_scale = -45.0f / (REF_PI * powf(h, 6.0f));
    c->r2 = h * h;
    /* least t with sqrtf(t) >= h; sqrtf is correctly rounded and monotone, so
     * "d2 >= t" is exactly "distance >= h", where every kernel returns 0 */
    float t = h * h;
    while (t > 0.0f && sqrtf(nextafterf(t, 0.0f)) >= h) t = nextafterf(t, 0.0f);
    while (sqrtf(t) < h) t = nextafterf(t, INFINITY);
    c->skip_d2 = t;
    c->margin_i = p->margin_integrate;
    c->mask = n > 0 ? n - 1u : 0u;
}

/* cellCoordToHash: multiply-xor spatial hash + avalanche finaliser
 * (updateCellEntries.comp:36-52). */
uint32_t pfso_cell_hash(uint32_t cx, uint32_t cy, uint32_t cz) {
    uint32_t h = (cx * 73856093u) ^ (cy * 19349663u) ^ (cz * 83492791u);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}

/* ivec3(floor((point - minXYZ) / smoothingRadius)), one axis
 * (updateCellEntries.comp:65).  Out-of-range conversions saturate and NaN
 * maps to 0, as the GPU's float->int conversion does. */
int32_t pfso_cell_coord(float v, float lo, float h) {
    float f = floorf((v - lo) / h);
    if (f != f) return 0;
    if (f >= 2147483648.0f) return INT32_MAX;
    if (f < -2147483648.0f) return INT32_MIN;
    return (int32_t)f;
}

/* cellCoordToKey(uvec3(floor((pos - minXYZ)/smoothingRadius)))
 * (updateCellEntries.comp:72-79, 54-61). */
uint32_t pfso_point_key(const pfs_params* p, uint32_t mask, const float* xyz) {
    uint32_t cx = (uint32_t)pfso_cell_coord(xyz[0], p->box_min[0], p->h);
    uint32_t cy = (uint32_t)pfso_cell_coord(xyz[1], p->box_min[1], p->h);
    uint32_t cz = (uint32_t)pfso_cell_coord(xyz[2], p->box_min[2], p->h);
    return pfso_cell_hash(cx, cy, cz) & mask;
}

/* updateCellEntries main (updateCellEntries.comp:69-80): key from the
 * substep-start position x (not the prediction), value = slot index. */
void pfso_keys(const pfs_params* p, uint32_t n, const float* pos4, uint32_t* keys) {
    const uint32_t mask = n > 0 ? n - 1u : 0u;
    PAR_FOR
    for (int64_t i = 0; i < (int64_t)n; i++) keys[i] = pfso_point_key(p, mask, pos4 + 4 * i);
}

/* Stable sort by key, ties in ascending slot index: the order the 4-pass
 * LSD radix sort of multiRadixSort.comp:54-139 produces (per-workgroup block
 * order + in-block ballot rank).  Keys are < n, so one counting pass over the
 * n-slot key space gives the same permutation. */
void pfso_sort(uint32_t n, const uint32_t* keys, uint32_t* sorted_keys, uint32_t* perm) {
    uint32_t* count = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++) count[keys[i] + 1]++;
    for (uint32_t k = 0; k < n; k++) count[k + 1] += count[k];
    for (uint32_t i = 0; i < n; i++) {
        uint32_t dst = count[keys[i]]++;
        sorted_keys[dst] = keys[i];
        perm[dst] = i;
    }
    free(count);
}

/* clearStartIndices (clearStartIndices.comp:39-45) then updateStartIndices
 * (updateStartIndices.comp:40-64): start at each run head, end exclusive,
 * untouched slots stay -1. */
void pfso_table(uint32_t n, const uint32_t* sk, int32_t* start, int32_t* end) {
    for (uint32_t k = 0; k < n; k++) { start[k] = -1; end[k] = -1; }
    for (uint32_t s = 0; s < n; s++) {
        uint32_t cur = sk[s];
        if (s == 0) {
            start[cur] = 0;
        } else if (cur != sk[s - 1]) {
            start[cur] = (int32_t)s;
            end[sk[s - 1]] = (int32_t)s;
        }
        if (s == n - 1) end[cur] = (int32_t)n;
    }
}

/* Wall clamp + reflect (predictPositions.comp:80-113 with margin
 * particleRadius; updateVelocities.comp:81-115 with particleRadius + 0.5).
 * The reference negates the hit component and then scales either the whole
 * vector by 1.00 or (z-min) that component by 0.95; scaling the component by
 * restitution[wall] reduces to exactly that for the reference values. */
static void walls(const pfs_params* p, float margin, float* pos, float* vel) {
    for (int a = 0; a < 3; a++) {
        float lo = p->box_min[a] + margin;
        float hi = p->box_max[a] - margin;
        if (pos[a] < lo) {
            pos[a] = lo;
            vel[a] = vel[a] * -1.0f;
            vel[a] = vel[a] * p->restitution[2 * a];
        } else if (pos[a] > hi) {
            pos[a] = hi;
            vel[a] = vel[a] * -1.0f;
            vel[a] = vel[a] * p->restitution[2 * a + 1];
        }
    }
}

/* predictPositions main (predictPositions.comp:69-117):
 * v* = v + g dt; x* = x + v* dt; walls with margin particleRadius. */
void pfso_predict(const pfs_params* p, uint32_t n, const float* pos4, const float* vel4,
                  float* xp4, float* vp4) {
    PAR_FOR
    for (int64_t i = 0; i < (int64_t)n; i++) {
        float pos[3], vel[3];
        for (int a = 0; a < 3; a++) {
            vel[a] = vel4[4 * i + a] + p->gravity[a] * p->dt;
            pos[a] = pos4[4 * i + a] + vel[a] * p->dt;
        }
        walls(p, p->margin_predict, pos, vel);
        for (int a = 0; a < 3; a++) { xp4[4 * i + a] = pos[a]; vp4[4 * i + a] = vel[a]; }
        xp4[4 * i + 3] = 1.0f;
        vp4[4 * i + 3] = 1.0f;
    }
}

/* calculateDensities (calculateDensities.comp:96-153): 27 sample points
 * x* + h*(dx,dy,dz), z outer, x inner; out-of-box sample points are skipped
 * (samplePointToKey, :69-73); no de-duplication of colliding keys; self
 * included; clamp at 0.01. */
void pfso_density(const pfs_params* p, uint32_t n, const float* xp4, const int32_t* start,
                  const int32_t* end, float* density, float* near_density) {
    pfso_consts c;
    pfso_derive(p, n, &c);
    const float h = p->h, m = p->particle_mass;
    PAR_FOR_DYN
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const float* sp = xp4 + 4 * i;
        float total = 0.0f, total_near = 0.0f;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    float s[3] = {sp[0] + h * (float)dx, sp[1] + h * (float)dy,
                                  sp[2] + h * (float)dz};
                    if (s[0] < p->box_min[0] || s[1] < p->box_min[1] || s[2] < p->box_min[2] ||
                        s[0] > p->box_max[0] || s[1] > p->box_max[1] || s[2] > p->box_max[2])
                        continue;
                    uint32_t key = pfso_point_key(p, c.mask, s);
                    int32_t st = start[key];
                    if (st == -1) continue;
                    int32_t en = end[key];
                    for (int32_t j = st; j < en; j++) {
                        const float* q = xp4 + 4 * (int64_t)j;
                        float d0 = q[0] - sp[0], d1 = q[1] - sp[1], d2 = q[2] - sp[2];
                        float dist = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
                        float infl = dist >= h ? 0.0f : (h - dist) * (h - dist);
                        total = total + m * infl;
                        float ninfl = dist >= h ? 0.0f : (h - dist) * (h - dist) * (h - dist);
                        total_near = total_near + m * ninfl;
                    }
                }
        float d = total / c.volume;
        float nd = total_near * c.near_inv;
        /* GLSL max(x, y) is (x < y) ? y : x */
        density[i] = (0.01f < d) ? d : 0.01f;
        near_density[i] = (0.01f < nd) ? nd : 0.01f;
    }
}

/* Density map extents.  image: the 3-D image the reference allocates,
 * (int)ceil((maxXYZ - minXYZ) * (1 / densityCellSize)) voxels per axis in
 * float (renderer.c:774-781); the dispatch covers it and stores beyond it are
 * dropped.  bound: the shader's own ivec3(ceil((maxXYZ - minXYZ) /
 * densityCellSize)) (updateDensityMap.comp:94), under which a voxel or cell
 * is out of bounds when a coordinate is negative or above it, or all three
 * equal it. */
void pfso_density_map_extent(const pfs_params* p, float cell_size, int32_t image[3],
                             int32_t bound[3]) {
    const float inv = 1.0f / cell_size;
    for (int a = 0; a < 3; a++) {
        const float ext = p->box_max[a] - p->box_min[a];
        image[a] = (int32_t)ceil((double)(ext * inv));
        bound[a] = (int32_t)ceilf(ext / cell_size);
    }
}

static int map_out_of_bounds(const int32_t v[3], const int32_t m[3]) {
    if (v[0] < 0 || v[1] < 0 || v[2] < 0) return 1;
    if (v[0] > m[0] || v[1] > m[1] || v[2] > m[2]) return 1;
    return v[0] == m[0] && v[1] == m[1] && v[2] == m[2];
}

/* updateDensityMap main (updateDensityMap.comp:109-147): for every voxel of
 * the image, the cell of its centre (samplePointToCellCoord :103-107,
 * (-1,-1,-1) outside the box) and the 27 cells around it (z outer, x inner),
 * each skipped when out of bounds; over the table range of each cell's key,
 * m * (h - d)^2 for d^2 < h^2 (smoothingKernel :98-101); divided by volume.
 * pos4 are the positions in the order of the sort that built start/end.  out
 * is x-fastest over the image; voxels the shader skips are 0. */
void pfso_density_map(const pfs_params* p, uint32_t n, const float* pos4, const int32_t* start,
                      const int32_t* end, float cell_size, float* out) {
    pfso_consts c;
    pfso_derive(p, n, &c);
    int32_t img[3], m[3];
    pfso_density_map_extent(p, cell_size, img, m);
    const int64_t nx = img[0], ny = img[1], nz = img[2];
    const float h = p->h, r2 = h * h, mass = p->particle_mass;
    PAR_FOR_DYN
    for (int64_t idx = 0; idx < nx * ny * nz; idx++) {
        const int32_t v[3] = {(int32_t)(idx % nx), (int32_t)((idx / nx) % ny), (int32_t)(idx / (nx * ny))};
        if (map_out_of_bounds(v, m)) {
            out[idx] = 0.0f;
            continue;
        }
        float ctr[3];
        for (int a = 0; a < 3; a++) ctr[a] = p->box_min[a] + ((float)v[a] + 0.5f) * cell_size;
        int32_t vc[3] = {-1, -1, -1};
        if (!(ctr[0] < p->box_min[0] || ctr[1] < p->box_min[1] || ctr[2] < p->box_min[2] ||
              ctr[0] > p->box_max[0] || ctr[1] > p->box_max[1] || ctr[2] > p->box_max[2]))
            for (int a = 0; a < 3; a++) vc[a] = pfso_cell_coord(ctr[a], p->box_min[a], h);
        float density = 0.0f;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int32_t cell[3] = {vc[0] + dx, vc[1] + dy, vc[2] + dz};
                    if (map_out_of_bounds(cell, m)) continue;
                    const uint32_t key =
                        pfso_cell_hash((uint32_t)cell[0], (uint32_t)cell[1], (uint32_t)cell[2]) & c.mask;
                    const int32_t st = start[key];
                    if (st == -1) continue;
                    const int32_t en = end[key];
                    for (int32_t i = st; i < en; i++) {
                        const float* q = pos4 + 4 * (int64_t)i;
                        const float d0 = ctr[0] - q[0], d1 = ctr[1] - q[1], d2 = ctr[2] - q[2];
                        const float dist2 = d0 * d0 + d1 * d1 + d2 * d2;
                        if (dist2 < r2) {
                            const float dist = sqrtf(dist2);
                            const float k = dist >= h ? 0.0f : (h - dist) * (h - dist);
                            density = density + mass * k;
                        }
                    }
                }
        density = density * 1.0f;
        out[idx] = density / c.volume;
    }
}

/* texture(sampler3D, uvw).r with the reference's sampler (image.c:134-164:
 * linear filter, clamp to edge, normalised coordinates, one level), in the
 * Vulkan specification's form computed in float: u = s * W - 0.5, i0 =
 * floor(u), alpha = u - i0, texels clamped to [0, W - 1], and the eight
 * weighted texels summed in the order (i0,j0,k0), (i1,j0,k0), (i0,j1,k0),
 * (i1,j1,k0), then the same with k1; weights ((1-a or a) * (1-b or b)) *
 * (1-c or c).  img is x-fastest, dims (W, H, D). */
float pfso_texture3d(const float* img, const int32_t dims[3], const float uvw[3]) {
    int32_t i0[3], i1[3];
    float f[3];
    for (int a = 0; a < 3; a++) {
        const float u = uvw[a] * (float)dims[a] - 0.5f;
        const float fl = floorf(u);
        f[a] = u - fl;
        int32_t k = fl != fl ? 0 : (fl < -2147483648.0f ? INT32_MIN : (fl >= 2147483647.0f ? INT32_MAX : (int32_t)fl));
        const int32_t top = dims[a] - 1;
        i0[a] = k < 0 ? 0 : (k > top ? top : k);
        const int32_t k1 = k == INT32_MAX ? k : k + 1;
        i1[a] = k1 < 0 ? 0 : (k1 > top ? top : k1);
    }
    const int64_t W = dims[0], H = dims[1];
#define TX(x, y, z) img[((int64_t)(z) * H + (y)) * W + (x)]
    const float a0 = 1.0f - f[0], a1 = f[0], b0 = 1.0f - f[1], b1 = f[1], c0 = 1.0f - f[2], c1 = f[2];
    float r = 0.0f;
    r = r + (a0 * b0) * c0 * TX(i0[0], i0[1], i0[2]);
    r = r + (a1 * b0) * c0 * TX(i1[0], i0[1], i0[2]);
    r = r + (a0 * b1) * c0 * TX(i0[0], i1[1], i0[2]);
    r = r + (a1 * b1) * c0 * TX(i1[0], i1[1], i0[2]);
    r = r + (a0 * b0) * c1 * TX(i0[0], i0[1], i1[2]);
    r = r + (a1 * b0) * c1 * TX(i1[0], i0[1], i1[2]);
    r = r + (a0 * b1) * c1 * TX(i0[0], i1[1], i1[2]);
    r = r + (a1 * b1) * c1 * TX(i1[0], i1[1], i1[2]);
#undef TX
    return r;
}

/* Ray against the box (intersectVolume, calculateLightVolume.comp:156-178 and
 * volumetricFluid.comp:157-179): slab test with invDir = 1 / dir; on a hit
 * the march interval is [max(tNear + pad_near, 0), tFar + pad_far] (the light
 * volume pads -1 / +1, the view ray +1 / -1).  Returns 0 on a miss. */
static int ray_box(const pfs_params* p, const float o[3], const float d[3], float pad_near,
                   float pad_far, float* t0, float* t1) {
    float tn[3], tf[3];
    for (int a = 0; a < 3; a++) {
        const float inv = 1.0f / d[a];
        const float ta = (p->box_min[a] - o[a]) * inv, tb = (p->box_max[a] - o[a]) * inv;
        /* GLSL min(x, y) = (y < x) ? y : x, max(x, y) = (x < y) ? y : x */
        tn[a] = (tb < ta) ? tb : ta;
        tf[a] = (ta < tb) ? tb : ta;
    }
    float m = (tn[0] < tn[1]) ? tn[1] : tn[0];
    const float t_near = (m < tn[2]) ? tn[2] : m;
    float q = (tf[1] < tf[0]) ? tf[1] : tf[0];
    const float t_far = (tf[2] < q) ? tf[2] : q;
    if (!(t_near <= t_far && t_far >= 0.0f)) return 0;
    const float a = t_near + pad_near;
    *t0 = (a < 0.0f) ? 0.0f : a;
    *t1 = t_far + pad_far;
    return 1;
}

/* calculateLightVolume main (calculateLightVolume.comp:193-219) over the image
 * renderer.c:812-819 allocates, (int)ceil((maxXYZ - minXYZ) * (1 / step)):
 * voxels whose coordinate exceeds the box size in world units are skipped (the
 * shader compares them with maxXYZ - minXYZ) and stay 0; the others march from
 * their centre toward the sun over the density map, summing texture * step
 * (calculateDensityAlongSunRay :180-194). */
void pfso_light_volume(const pfs_params* p, const float* dmap, const int32_t ddims[3],
                       float light_step, const float sun[3], const int32_t ldims[3], float* out) {
    float size[3];
    for (int a = 0; a < 3; a++) size[a] = p->box_max[a] - p->box_min[a];
    const int64_t nx = ldims[0], ny = ldims[1], nz = ldims[2];
    PAR_FOR_DYN
    for (int64_t idx = 0; idx < nx * ny * nz; idx++) {
        const int32_t v[3] = {(int32_t)(idx % nx), (int32_t)((idx / nx) % ny), (int32_t)(idx / (nx * ny))};
        out[idx] = 0.0f;
        if ((float)v[0] > size[0] || (float)v[1] > size[1] || (float)v[2] > size[2]) continue;
        float c[3];
        for (int a = 0; a < 3; a++) c[a] = p->box_min[a] + ((float)v[a] + 0.5f) * light_step;
        float t0, t1;
        if (!ray_box(p, c, sun, -1.0f, 1.0f, &t0, &t1)) continue;
        float acc = 0.0f;
        for (float t = (t0 < 0.0f) ? 0.0f : t0; t < t1; t += light_step) {
            float uvw[3];
            for (int a = 0; a < 3; a++) uvw[a] = ((c[a] + t * sun[a]) - p->box_min[a]) / size[a];
            acc = acc + pfso_texture3d(dmap, ddims, uvw) * light_step;
        }
        out[idx] = acc;
    }
}

/* volumetricFluid main (volumetricFluid.comp:196-263): one ray per pixel from
 * the camera through the pixel centre (makeRayFromCameraThroughPixel
 * :231-252, y = 0 at the top; half_height = tan(0.5 * FOV), computed by the
 * caller once), marched through the box (marchRay :196-229): density map
 * sample * 0.05, light volume sample, Beer-Lambert transmittance with
 * extinction normalize(extinctionCoefficients), early exit when the view
 * transmittance drops below 0.01 on every channel, + 0.05 when every channel
 * of the result exceeds 1e-5; sky colour 0 on a miss.  rgba is x-fastest,
 * alpha 1.  normalize(v) is v / sqrt(dot(v, v)). */
void pfso_volumetric(const pfs_params* p, const float* dmap, const int32_t ddims[3],
                     const float* lvol, const int32_t ldims[3], const float cam[12],
                     float half_height, float step, const float extinction[3], uint32_t width,
                     uint32_t height, float* rgba) {
    const float* pos = cam;
    const float* fwd = cam + 3;
    const float* right = cam + 6;
    const float* up = cam + 9;
    float size[3];
    for (int a = 0; a < 3; a++) size[a] = p->box_max[a] - p->box_min[a];
    const float el = sqrtf(extinction[0] * extinction[0] + extinction[1] * extinction[1] +
                           extinction[2] * extinction[2]);
    float ext[3];
    for (int a = 0; a < 3; a++) ext[a] = 1.0f * (extinction[a] / el);
    const float amb[3] = {0.529f, 0.808f, 0.922f};
    const float half_width = half_height * (float)width / (float)height;
    PAR_FOR_DYN
    for (int64_t idx = 0; idx < (int64_t)width * height; idx++) {
        const int32_t x = (int32_t)(idx % width), y = (int32_t)(idx / width);
        const float px = (float)x + 0.5f, py = (float)y + 0.5f;
        const float u = (px / (float)width) * 2.0f - 1.0f;
        const float v = (py / (float)height) * 2.0f - 1.0f;
        float dir[3];
        for (int a = 0; a < 3; a++) {
            const float center = pos[a] + fwd[a];
            float pp = center + (u * half_width) * right[a];
            pp = pp - (v * half_height) * up[a];
            dir[a] = pp - pos[a];
        }
        const float dl = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
        for (int a = 0; a < 3; a++) dir[a] = dir[a] / dl;
        float light[3] = {0.0f, 0.0f, 0.0f};
        float t0, t1;
        if (ray_box(p, pos, dir, 1.0f, -1.0f, &t0, &t1)) {
            float view = 0.0f;
            for (float t = ((t0 < 0.0f) ? 0.0f : t0) + step; t < t1 - step; t += step) {
                float uvw[3];
                for (int a = 0; a < 3; a++) {
                    float w = ((pos[a] + t * dir[a]) - p->box_min[a]) / size[a];
                    uvw[a] = (w < 0.0f) ? 0.0f : ((1.0f < w) ? 1.0f : w);  /* clamp (min(max)) */
                }
                const float dens = pfso_texture3d(dmap, ddims, uvw) * 0.05f;
                view = view + dens * step;
                const float sun = pfso_texture3d(lvol, ldims, uvw);
                float in[3], vt[3];
                for (int a = 0; a < 3; a++) {
                    const float tr = expf(-sun * ext[a]) * amb[a];
                    in[a] = (tr * dens) * ext[a];
                    vt[a] = expf(-view * ext[a]);
                }
                const float mx = (vt[1] < vt[2]) ? vt[2] : vt[1];
                const float mm = (vt[0] < mx) ? mx : vt[0];
                if (mm < 0.01f) break;
                for (int a = 0; a < 3; a++) light[a] = light[a] + in[a] * vt[a];
            }
            if (light[0] > 0.00001f && light[1] > 0.00001f && light[2] > 0.00001f)
                for (int a = 0; a < 3; a++) light[a] = light[a] + 0.05f;
        }
        for (int a = 0; a < 3; a++) rgba[4 * idx + a] = light[a];
        rgba[4 * idx + 3] = 1.0f;
    }
}

/* ---- refractive render mode (properFluid.comp) --------------------------
 * Restated from properFluid.comp:151-614 with GLSL's built-ins written out by
 * their specification formulas, evaluated left to right in float:
 *   dot(a, b) = a.x*b.x + a.y*b.y + a.z*b.z, length = sqrt(dot(v, v)),
 *   normalize(v) = v / length(v), min(x, y) = (y < x) ? y : x,
 *   max(x, y) = (x < y) ? y : x, clamp(x, a, b) = min(max(x, a), b),
 *   sign(x) = 1 / -1 / 0, smoothstep(e0, e1, x) = t*t*(3 - 2t) with
 *   t = clamp((x - e0) / (e1 - e0), 0, 1), pow = powf, exp = expf,
 *   reflect(I, N) = I - 2*dot(N, I)*N,
 *   refract(I, N, eta) = k < 0 ? 0 : eta*I - (eta*dot(N, I) + sqrt(k))*N,
 *   k = 1 - eta*eta*(1 - dot(N, I)*dot(N, I)). */
static float g_min(float x, float y) { return (y < x) ? y : x; }
static float g_max(float x, float y) { return (x < y) ? y : x; }
static float g_clamp(float x, float a, float b) { return g_min(g_max(x, a), b); }
static float g_dot(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static float g_sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
static void g_normalize(float v[3]) {
    const float l = sqrtf(g_dot(v, v));
    for (int a = 0; a < 3; a++) v[a] = v[a] / l;
}
static float g_smoothstep(float e0, float e1, float x) {
    const float t = g_clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

typedef struct {
    const pfs_params* p;
    const float* dmap;
    const int32_t* ddims;
    float size[3];
    float step, light_step, threshold, ior;
    const float* ext;
} refr_ctx;

/* calculateDensityAlongRay (properFluid.comp:205-218); intersectVolume pads
 * the interval by +1e-4 / -1e-4 (:157-178). */
static float refr_density_along(const refr_ctx* c, const float o[3], const float d[3], float sstep) {
    float t0, t1;
    if (!ray_box(c->p, o, d, 1e-4f, -1e-4f, &t0, &t1)) return 0.0f;
    float acc = 0.0f;
    for (float t = g_max(t0, 0.0f) + sstep; t < t1 - sstep; t += sstep) {
        float uvw[3];
        for (int a = 0; a < 3; a++) uvw[a] = ((o[a] + t * d[a]) - c->p->box_min[a]) / c->size[a];
        acc = acc + pfso_texture3d(c->dmap, c->ddims, uvw) * sstep;
    }
    return acc;
}

/* getSurfaceNormal (:230-260) with calculateClosestFaceNormal (:193-203). */
static void refr_normal(const refr_ctx* c, const float pos[3], float out[3]) {
    const pfs_params* p = c->p;
    float uvw[3], texel[3];
    for (int a = 0; a < 3; a++) {
        uvw[a] = g_clamp((pos[a] - p->box_min[a]) / c->size[a], 0.0f, 1.0f);
        texel[a] = 1.0f / (float)c->ddims[a];
    }
    float g[3];
    for (int a = 0; a < 3; a++) {
        float up[3] = {uvw[0], uvw[1], uvw[2]}, dn[3] = {uvw[0], uvw[1], uvw[2]};
        for (int b = 0; b < 3; b++) {
            up[b] = uvw[b] + (a == b ? texel[a] : 0.0f);
            dn[b] = uvw[b] - (a == b ? texel[a] : 0.0f);
        }
        g[a] = pfso_texture3d(c->dmap, c->ddims, up) - pfso_texture3d(c->dmap, c->ddims, dn);
    }
    g_normalize(g);
    float o[3];
    for (int a = 0; a < 3; a++) o[a] = c->size[a] / 2.0f - fabsf(pos[a]);
    float fw = g_min(o[0], g_min(o[1], o[2]));
    float fn[3] = {0.0f, 0.0f, 0.0f}, local[3], dd[3];
    for (int a = 0; a < 3; a++) {
        const float center = 0.5f * (p->box_min[a] + p->box_max[a]);
        local[a] = pos[a] - center;
        dd[a] = 0.5f * c->size[a] - fabsf(local[a]);
    }
    if (dd[0] < dd[1] && dd[0] < dd[2]) fn[0] = g_sign(local[0]);
    else if (dd[1] < dd[2]) fn[1] = g_sign(local[1]);
    else fn[2] = g_sign(local[2]);
    fw = (1.0f - g_smoothstep(0.0f, 0.3f, fw)) * (1.0f - powf(g_clamp(g[2], 0.0f, 1.0f), 5.0f));
    for (int a = 0; a < 3; a++) out[a] = g[a] * (1.0f - fw) + fn[a] * fw;
    g_normalize(out);
}

typedef struct {
    float pos[3], normal[3], dens;
    int found, entering;
} refr_surface;

/* findNextSurface (:277-325): march the density map from the box entry (or
 * from the origin when inside the fluid) until it crosses the surface
 * threshold upward (outside) or downward (inside). */
static refr_surface refr_next_surface(const refr_ctx* c, const float o_in[3], const float d[3], int inside) {
    refr_surface s;
    memset(&s, 0, sizeof(s));
    const pfs_params* p = c->p;
    float t0, t1;
    if (!ray_box(p, o_in, d, 1e-4f, -1e-4f, &t0, &t1)) return s;
    const int out_of_fluid = !(o_in[0] >= p->box_min[0] && o_in[1] >= p->box_min[1] && o_in[2] >= p->box_min[2] &&
                               o_in[0] <= p->box_max[0] && o_in[1] <= p->box_max[1] && o_in[2] <= p->box_max[2]);
    const float t = inside ? 0.0f : g_max(t0, 0.0f);
    float o[3];
    for (int a = 0; a < 3; a++) o[a] = o_in[a] + (t + c->step) * d[a];
    float uvw[3];
    for (int a = 0; a < 3; a++) uvw[a] = (o[a] - p->box_min[a]) / c->size[a];
    float prev = out_of_fluid ? 0.0f : pfso_texture3d(c->dmap, c->ddims, uvw);
    float dens = 0.0f;
    for (float tt = t; tt < t1; tt += c->step) {
        for (int a = 0; a < 3; a++) o[a] = o[a] + c->step * d[a];
        for (int a = 0; a < 3; a++) uvw[a] = (o[a] - p->box_min[a]) / c->size[a];
        const float density = pfso_texture3d(c->dmap, c->ddims, uvw);
        dens = dens + density * c->step;
        const int entering = prev < c->threshold && density >= c->threshold;
        const int exiting = prev >= c->threshold && density < c->threshold;
        if (inside ? exiting : entering) {
            refr_normal(c, o, s.normal);
            if (g_dot(s.normal, d) > 0.0f)
                for (int a = 0; a < 3; a++) s.normal[a] = -s.normal[a];
            for (int a = 0; a < 3; a++) s.pos[a] = o[a];
            s.dens = dens;
            s.found = 1;
            s.entering = entering;
            return s;
        }
        prev = density;
    }
    for (int a = 0; a < 3; a++) s.pos[a] = o[a];
    s.dens = dens;
    return s;
}

/* calculateReflectance (:329-345). */
static float refr_reflectance(const float in[3], const float n[3], float ia, float ib) {
    const float ratio = ia / ib;
    const float cos_in = -g_dot(in, n);
    const float sin2 = ratio * ratio * (1.0f - cos_in * cos_in);
    if (sin2 >= 1.0f) return 1.0f;
    const float cos_r = sqrtf(1.0f - sin2);
    float rs = (ia * cos_in - ib * cos_r) / (ia * cos_in + ib * cos_r);
    rs = rs * rs;
    float rp = (ib * cos_in - ia * cos_r) / (ib * cos_in + ia * cos_r);
    rp = rp * rp;
    return (rs + rp) / 2.0f;
}

/* marchRayExpensive (:498-573) for one camera ray; environmentLight returns
 * vec3(1) before its floor and sky code (:418), so the environment is white. */
static void refr_march(const refr_ctx* c, float o[3], float d[3], int num_refr, float light[3]) {
    float tr[3] = {1.0f, 1.0f, 1.0f};
    for (int a = 0; a < 3; a++) light[a] = 0.0f;
    int in_fluid = 0;
    for (int i = 0; i < num_refr; i++) {
        if (isnan(d[0]) || isnan(d[1]) || isnan(d[2])) {
            light[0] = 1.0f; light[1] = 0.0f; light[2] = 1.0f;
            return;
        }
        if (sqrtf(g_dot(d, d)) < 1e-6f) {
            light[0] = 1.0f; light[1] = 1.0f; light[2] = 0.0f;
            return;
        }
        const refr_surface s = refr_next_surface(c, o, d, in_fluid);
        for (int a = 0; a < 3; a++) tr[a] = tr[a] * expf(-s.dens * c->ext[a]);
        if (!s.found) break;
        const float ia = s.entering ? 1.0f : c->ior, ib = s.entering ? c->ior : 1.0f;
        /* calculateReflectionAndRefraction (:354-372) */
        float in[3] = {d[0], d[1], d[2]}, n[3] = {s.normal[0], s.normal[1], s.normal[2]};
        g_normalize(in);
        g_normalize(n);
        const float rw = refr_reflectance(in, n, ia, ib);
        const float fw = 1.0f - rw;
        float rdir[3], fdir[3];
        const float dni = g_dot(n, in);
        for (int a = 0; a < 3; a++) rdir[a] = in[a] - 2.0f * dni * n[a];
        g_normalize(rdir);
        const float eta = ia / ib;
        const float k = 1.0f - eta * eta * (1.0f - dni * dni);
        float refr[3];
        if (k < 0.0f) {
            refr[0] = refr[1] = refr[2] = 0.0f;
        } else {
            const float sk = sqrtf(k);
            for (int a = 0; a < 3; a++) refr[a] = eta * in[a] - (eta * dni + sk) * n[a];
        }
        if (g_dot(refr, refr) > 1e-12f) {
            for (int a = 0; a < 3; a++) fdir[a] = refr[a];
            g_normalize(fdir);
        } else {
            fdir[0] = fdir[1] = fdir[2] = 0.0f;
        }
        int follow = fw > rw;
        float fo[3], ro[3];
        for (int a = 0; a < 3; a++) {
            fo[a] = s.pos[a] - s.normal[a] * 1e-3f;
            ro[a] = s.pos[a] + s.normal[a] * 1e-3f;
        }
        const int did = follow && sqrtf(g_dot(fdir, fdir)) > 1e-6f;
        if (did) in_fluid = !in_fluid;
        follow = did;
        if (!follow) {
            if (fw > 0.0f) {
                const float dr = refr_density_along(c, fo, fdir, c->light_step);
                for (int a = 0; a < 3; a++) light[a] = light[a] + 1.0f * tr[a] * expf(-dr * c->ext[a]) * fw;
            }
        } else {
            const float dr = refr_density_along(c, ro, rdir, c->light_step);
            for (int a = 0; a < 3; a++) light[a] = light[a] + 1.0f * tr[a] * expf(-dr * c->ext[a]) * rw;
        }
        for (int a = 0; a < 3; a++) {
            o[a] = follow ? fo[a] : ro[a];
            d[a] = follow ? fdir[a] : rdir[a];
        }
        const float wsel = follow ? fw : rw;
        for (int a = 0; a < 3; a++) tr[a] = tr[a] * wsel;
        if (g_max(tr[0], g_max(tr[1], tr[2])) < 0.02f) break;
    }
    const float dr = refr_density_along(c, o, d, c->light_step);
    for (int a = 0; a < 3; a++) light[a] = light[a] + 1.0f * tr[a] * expf(-dr * c->ext[a]);
}

/* properFluid main (:600-614) with makeRayFromCameraThroughPixel (:575-598,
 * the volumetric mode's camera): rgba x-fastest, alpha 1. */
void pfso_refractive(const pfs_params* p, const float* dmap, const int32_t ddims[3], const float cam[12],
                     float half_height, float step, float light_step, const float extinction[3],
                     int32_t num_refractions, float threshold, float ior, uint32_t width,
                     uint32_t height, float* rgba) {
    refr_ctx c;
    c.p = p;
    c.dmap = dmap;
    c.ddims = ddims;
    for (int a = 0; a < 3; a++) c.size[a] = p->box_max[a] - p->box_min[a];
    c.step = step;
    c.light_step = light_step;
    c.threshold = threshold;
    c.ior = ior;
    c.ext = extinction;
    const float* pos = cam;
    const float* fwd = cam + 3;
    const float* right = cam + 6;
    const float* up = cam + 9;
    const float half_width = half_height * (float)width / (float)height;
    PAR_FOR_DYN
    for (int64_t idx = 0; idx < (int64_t)width * height; idx++) {
        const int32_t x = (int32_t)(idx % width), y = (int32_t)(idx / width);
        const float u = (((float)x + 0.5f) / (float)width) * 2.0f - 1.0f;
        const float v = (((float)y + 0.5f) / (float)height) * 2.0f - 1.0f;
        float o[3], d[3];
        for (int a = 0; a < 3; a++) {
            const float center = pos[a] + fwd[a];
            float pp = center + (u * half_width) * right[a];
            pp = pp - (v * half_height) * up[a];
            d[a] = pp - pos[a];
            o[a] = pos[a];
        }
        g_normalize(d);
        float light[3];
        refr_march(&c, o, d, num_refractions, light);
        for (int a = 0; a < 3; a++) rgba[4 * idx + a] = light[a];
        rgba[4 * idx + 3] = 1.0f;
    }
}

/* ---- FXAA post-process (raymarchShader.frag:15-73) -------------------------
 * The reference draws the compute-rendered image on a full-screen quad
 * through raymarchShader.frag, which samples it with the linear,
 * clamp-to-edge sampler (image.c:135-161) and applies this FXAA variant.
 * Fragment (x, y) of a width x height target gets outNDC = ((x + 0.5) / width
 * * 2 - 1, (y + 0.5) / height * 2 - 1); texture() is float bilinear
 * interpolation in the term order of pfso_texture3d. */
static void tex2d_rgb(const float* img, int32_t w, int32_t h, float u, float v, float out[3]) {
    const float uu[2] = {u, v};
    const int32_t dd[2] = {w, h};
    int32_t i0[2], i1[2];
    float f[2];
    for (int a = 0; a < 2; a++) {
        const float t = uu[a] * (float)dd[a] - 0.5f;
        const float fl = floorf(t);
        f[a] = t - fl;
        int32_t k = fl != fl ? 0 : (fl < -2147483648.0f ? INT32_MIN : (fl >= 2147483647.0f ? INT32_MAX : (int32_t)fl));
        const int32_t top = dd[a] - 1;
        i0[a] = k < 0 ? 0 : (k > top ? top : k);
        const int32_t k1 = k == INT32_MAX ? k : k + 1;
        i1[a] = k1 < 0 ? 0 : (k1 > top ? top : k1);
    }
    const float a0 = 1.0f - f[0], a1 = f[0], b0 = 1.0f - f[1], b1 = f[1];
    for (int c = 0; c < 3; c++) {
#define TX(x, y) img[4 * ((int64_t)(y) * w + (x)) + c]
        float r = 0.0f;
        r = r + (a0 * b0) * TX(i0[0], i0[1]);
        r = r + (a1 * b0) * TX(i1[0], i0[1]);
        r = r + (a0 * b1) * TX(i0[0], i1[1]);
        r = r + (a1 * b1) * TX(i1[0], i1[1]);
#undef TX
        out[c] = r;
    }
}

static float luminance(const float c[3]) { return c[0] * 0.299f + c[1] * 0.587f + c[2] * 0.114f; }

void pfso_fxaa(const float* in, uint32_t width, uint32_t height, float* out) {
    const float tx = 1.0f / (float)width, ty = 1.0f / (float)height;
    PAR_FOR
    for (int64_t idx = 0; idx < (int64_t)width * height; idx++) {
        const int32_t x = (int32_t)(idx % width), y = (int32_t)(idx / width);
        const float nx = ((float)x + 0.5f) / (float)width * 2.0f - 1.0f;
        const float ny = ((float)y + 0.5f) / (float)height * 2.0f - 1.0f;
        const float u = nx * 0.5f + 0.5f, v = ny * 0.5f + 0.5f;
        float nw[3], ne[3], sw[3], se[3], m[3];
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + -1.0f * tx, v + -1.0f * ty, nw);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + 1.0f * tx, v + -1.0f * ty, ne);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + -1.0f * tx, v + 1.0f * ty, sw);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + 1.0f * tx, v + 1.0f * ty, se);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u, v, m);
        const float lnw = luminance(nw), lne = luminance(ne), lsw = luminance(sw), lse = luminance(se),
                    lm = luminance(m);
        const float lmin = g_min(lm, g_min(g_min(lnw, lne), g_min(lsw, lse)));
        const float lmax = g_max(lm, g_max(g_max(lnw, lne), g_max(lsw, lse)));
        float dx = -((lnw + lne) - (lsw + lse));
        float dy = (lnw + lsw) - (lne + lse);
        const float reduce = g_max((lnw + lne + lsw + lse) * (0.25f * (1.0f / 8.0f)), 1.0f / 128.0f);
        const float rcp = 1.0f / (g_min(fabsf(dx), fabsf(dy)) + reduce);
        dx = g_min(g_max(dx * rcp, -8.0f), 8.0f) * tx;
        dy = g_min(g_max(dy * rcp, -8.0f), 8.0f) * ty;
        const float k1 = 1.0f / 3.0f - 0.5f, k2 = 2.0f / 3.0f - 0.5f;
        float a1[3], a2[3], b1[3], b2[3], ra[3], rb[3];
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + dx * k1, v + dy * k1, a1);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + dx * k2, v + dy * k2, a2);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + dx * -0.5f, v + dy * -0.5f, b1);
        tex2d_rgb(in, (int32_t)width, (int32_t)height, u + dx * 0.5f, v + dy * 0.5f, b2);
        for (int c = 0; c < 3; c++) {
            ra[c] = 0.5f * (a1[c] + a2[c]);
            rb[c] = ra[c] * 0.5f + 0.25f * (b1[c] + b2[c]);
        }
        const float lb = luminance(rb);
        const float* pick = (lb < lmin || lb > lmax) ? ra : rb;
        for (int c = 0; c < 3; c++) out[4 * idx + c] = pick[c];
        out[4 * idx + 3] = 1.0f;
    }
}

/* ---- point-splat rasteriser (shader.vert:27-57, shader.frag:56-87) --------
 * The reference's default render (RENDER_TYPE RASTERIZATION, main.c:32):
 * one camera-facing quad of half-size particleRadius per particle,
 * gl_Position = proj * view * model * (pos + r * (qx * right + qy * up), 1)
 * with right / up the first two rows of view's rotation, depth test LESS with
 * depth writes, no blending, clear colour 0 and depth 1 (commands.c:186-188,
 * graphics_pipeline.c:114-134).  Restated headless: the quad is parallel to
 * the image plane, so it projects to a screen-aligned square between its
 * corners (-1,-1) and (1,1); a pixel whose centre lies in [min, max) on both
 * axes is a fragment, fragQuadPos is interpolated linearly across the square,
 * the fragment's depth is the projected z / w of the particle centre, and
 * fragments with |fragQuadPos|^2 > 1 are discarded.  Particles are drawn in
 * slot order (gl_InstanceIndex), so a pixel keeps the first particle of the
 * smallest depth.  The fragment colour is colors[i].xyz scaled by Lambert
 * lighting of the disc normal (0.7 + 0.3 * lighting), alpha
 * 1 - smoothstep(0.8, 1, |fragQuadPos|).  mvp = (proj * view) * model and
 * right / up are computed by the caller (column-major mat4, GLSL order). */
/* mvp = (proj * view) * model (GLSL mat4 products, column-major, sums left
 * to right) and the camera's right / up: transpose(mat3(view)) rows 0 and 1
 * (shader.vert:29-32). */
void pfso_splat_camera(const float model[16], const float view[16], const float proj[16], float mvp[16],
                       float right[3], float up[3]) {
    float pv[16];
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++)
            pv[c * 4 + r] = proj[0 * 4 + r] * view[c * 4 + 0] + proj[1 * 4 + r] * view[c * 4 + 1] +
                            proj[2 * 4 + r] * view[c * 4 + 2] + proj[3 * 4 + r] * view[c * 4 + 3];
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++)
            mvp[c * 4 + r] = pv[0 * 4 + r] * model[c * 4 + 0] + pv[1 * 4 + r] * model[c * 4 + 1] +
                             pv[2 * 4 + r] * model[c * 4 + 2] + pv[3 * 4 + r] * model[c * 4 + 3];
    for (int a = 0; a < 3; a++) {
        right[a] = view[a * 4 + 0];
        up[a] = view[a * 4 + 1];
    }
}

void pfso_splat_clip(const float mvp[16], const float pos[3], const float right[3], const float up[3],
                     float r, float qx, float qy, float clip[4]) {
    float wp[3];
    for (int a = 0; a < 3; a++) wp[a] = pos[a] + r * (qx * right[a] + qy * up[a]);
    for (int k = 0; k < 4; k++)
        clip[k] = mvp[0 * 4 + k] * wp[0] + mvp[1 * 4 + k] * wp[1] + mvp[2 * 4 + k] * wp[2] + mvp[3 * 4 + k] * 1.0f;
}

/* Screen square and depth of particle i; returns 0 when it is clipped. */
int pfso_splat_geometry(const float mvp[16], const float right[3], const float up[3], float r,
                        const float pos[3], uint32_t width, uint32_t height, float sq[4], float* depth) {
    float c0[4], ca[4], cb[4];
    pfso_splat_clip(mvp, pos, right, up, r, 0.0f, 0.0f, c0);
    pfso_splat_clip(mvp, pos, right, up, r, -1.0f, -1.0f, ca);
    pfso_splat_clip(mvp, pos, right, up, r, 1.0f, 1.0f, cb);
    if (!(c0[3] > 0.0f && ca[3] > 0.0f && cb[3] > 0.0f)) return 0;
    const float z = c0[2] / c0[3];
    if (!(z >= 0.0f && z <= 1.0f)) return 0;
    const float hw = (float)width * 0.5f, hh = (float)height * 0.5f;
    sq[0] = (ca[0] / ca[3]) * hw + hw;   /* screen position of corner (-1, -1) */
    sq[1] = (ca[1] / ca[3]) * hh + hh;
    sq[2] = (cb[0] / cb[3]) * hw + hw;   /* and of corner (1, 1) */
    sq[3] = (cb[1] / cb[3]) * hh + hh;
    *depth = z;
    return 1;
}

/* fragQuadPos of pixel (x, y) in the square; returns 0 outside it. */
int pfso_splat_quadpos(const float sq[4], int32_t x, int32_t y, float* qx, float* qy) {
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    const float x0 = g_min(sq[0], sq[2]), x1 = g_max(sq[0], sq[2]);
    const float y0 = g_min(sq[1], sq[3]), y1 = g_max(sq[1], sq[3]);
    if (!(px >= x0 && px < x1 && py >= y0 && py < y1)) return 0;
    *qx = -1.0f + 2.0f * ((px - sq[0]) / (sq[2] - sq[0]));
    *qy = -1.0f + 2.0f * ((py - sq[1]) / (sq[3] - sq[1]));
    return 1;
}

void pfso_splat_shade(const float color[4], float qx, float qy, float out[4]) {
    const float r2 = qx * qx + qy * qy;
    const float z = sqrtf(1.0f - r2);
    float nrm[3] = {-qx, -qy, z};
    g_normalize(nrm);
    float ld[3] = {-0.5f, -0.5f, 1.0f};
    g_normalize(ld);
    const float lighting = g_max(g_dot(nrm, ld), 0.0f);
    const float alpha = 1.0f - g_smoothstep(0.8f, 1.0f, sqrtf(r2));
    const float k = 1.0f - 0.3f + 0.3f * lighting;
    for (int a = 0; a < 3; a++) out[a] = color[a] * k;
    out[3] = alpha;
}

void pfso_splats(uint32_t n, const float* pos4, const float* color4, const float mvp[16],
                 const float right[3], const float up[3], float radius, uint32_t width, uint32_t height,
                 float* rgba, float* depth) {
    const int64_t npx = (int64_t)width * height;
    for (int64_t k = 0; k < npx; k++) {
        depth[k] = 1.0f;
        rgba[4 * k] = rgba[4 * k + 1] = rgba[4 * k + 2] = rgba[4 * k + 3] = 0.0f;
    }
    for (uint32_t i = 0; i < n; i++) {
        float sq[4], z;
        if (!pfso_splat_geometry(mvp, right, up, radius, pos4 + 4 * (size_t)i, width, height, sq, &z)) continue;
        const float x0 = g_min(sq[0], sq[2]), x1 = g_max(sq[0], sq[2]);
        const float y0 = g_min(sq[1], sq[3]), y1 = g_max(sq[1], sq[3]);
        if (!(x1 >= 0.0f && y1 >= 0.0f && x0 <= (float)width && y0 <= (float)height)) continue;
        const int32_t xa = x0 < 1.0f ? 0 : (int32_t)x0 - 1, ya = y0 < 1.0f ? 0 : (int32_t)y0 - 1;
        const int32_t xb = x1 >= (float)width ? (int32_t)width - 1 : (int32_t)x1 + 1;
        const int32_t yb = y1 >= (float)height ? (int32_t)height - 1 : (int32_t)y1 + 1;
        for (int32_t y = ya; y <= yb; y++)
            for (int32_t x = xa; x <= xb; x++) {
                float qx, qy;
                if (!pfso_splat_quadpos(sq, x, y, &qx, &qy)) continue;
                if (qx * qx + qy * qy > 1.0f) continue;   /* discard */
                const int64_t k = (int64_t)y * width + x;
                if (!(z < depth[k])) continue;             /* VK_COMPARE_OP_LESS */
                depth[k] = z;
                pfso_splat_shade(color4 + 4 * (size_t)i, qx, qy, rgba + 4 * k);
            }
    }
}

/* applyPressureAndViscosityForce (applyPressureAndViscosityForce.comp:121-183):
 * 27 cell offsets around the cell of x* ((-1,-1,-1) when x* is outside the
 * box), skip self, d2 > h^2 and dist < 1e-7; symmetric shared pressure with
 * the spiky derivative, viscosity (h-d)^2 on (v_j - v*_i), near pressure;
 * v_i += (F_p + F_v + 0) / rho_i * dt.  v_j are the pre-update velocities. */
void pfso_force(const pfs_params* p, uint32_t n, const float* xp4, const float* vp4,
                const float* vel4, const float* density, const float* near_density,
                const int32_t* start, const int32_t* end, float* vel_out4) {
    pfso_consts c;
    pfso_derive(p, n, &c);
    const float h = p->h, m = p->particle_mass;
    const float rho0 = p->target_density, k = p->pressure_multiplier;
    const float kn = p->near_pressure_multiplier;
    PAR_FOR_DYN
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const float* sp = xp4 + 4 * i;
        const float* pv = vp4 + 4 * i;
        const float my_density = density[i];
        int32_t cell[3];
        if (sp[0] < p->box_min[0] || sp[1] < p->box_min[1] || sp[2] < p->box_min[2] ||
            sp[0] > p->box_max[0] || sp[1] > p->box_max[1] || sp[2] > p->box_max[2]) {
            cell[0] = cell[1] = cell[2] = -1;
        } else {
            for (int a = 0; a < 3; a++) cell[a] = pfso_cell_coord(sp[a], p->box_min[a], h);
        }
        const float near_pressure = near_density[i] * kn;
        float fp[3] = {0.0f, 0.0f, 0.0f}, fv[3] = {0.0f, 0.0f, 0.0f};
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    uint32_t key = pfso_cell_hash((uint32_t)cell[0] + (uint32_t)dx,
                                                  (uint32_t)cell[1] + (uint32_t)dy,
                                                  (uint32_t)cell[2] + (uint32_t)dz) & c.mask;
                    if (key == 0xFFFFFFFFu) continue;
                    int32_t st = start[key];
                    if (st == -1) continue;
                    int32_t en = end[key];
                    for (int32_t j = st; j < en; j++) {
                        if (j == (int32_t)i) continue;
                        const float* q = xp4 + 4 * (int64_t)j;
                        float d[3] = {q[0] - sp[0], q[1] - sp[1], q[2] - sp[2]};
                        float dist2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        if (dist2 > c.r2) continue;
                        float dist = sqrtf(dist2);
                        if (fabsf(dist) < 1e-7f) continue;
                        float dir[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
                        float slope = dist >= h ? 0.0f : (dist - h) * c.slope_scale;
                        float dj = density[j];
                        float shared = ((dj - rho0) * k + (my_density - rho0) * k) / 2.0f;
                        float coef = shared * slope * m / dj;
                        for (int a = 0; a < 3; a++) fp[a] = fp[a] + coef * dir[a];
                        float infl = dist >= h ? 0.0f : (h - dist) * (h - dist);
                        float vcoef = m * infl / dj;
                        const float* vj = vel4 + 4 * (int64_t)j;
                        for (int a = 0; a < 3; a++) fv[a] = fv[a] + vcoef * (vj[a] - pv[a]);
                        float nnd = near_density[j];
                        float shared_near = (near_pressure + nnd * kn) / 2.0f;
                        float x = h - dist;
                        float nslope = dist >= h ? 0.0f : x * x * c.near_slope_scale;
                        float ncoef = shared_near * nslope * m / nnd;
                        for (int a = 0; a < 3; a++) fp[a] = fp[a] + ncoef * dir[a];
                    }
                }
        const float* vi = vel4 + 4 * i;
        for (int a = 0; a < 3; a++) {
            float total = (fp[a] + p->viscosity * fv[a]) + 0.0f;
            vel_out4[4 * i + a] = vi[a] + total / my_density * p->dt;
        }
        vel_out4[4 * i + 3] = vi[3] + 1.0f;
    }
}

/* Speed colour ramp (updateVelocities.comp:120-141). */
void pfso_color(const float* v, float* rgba) {
    static const float c0[3] = {0.3f, 0.3f, 1.0f}, c1[3] = {0.0f, 1.0f, 1.0f},
                       c2[3] = {1.0f, 1.0f, 0.0f}, c3[3] = {1.0f, 0.3f, 0.3f};
    float speed = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    float t = speed / 60.0f;
    t = (t < 0.0f) ? 0.0f : t;  /* clamp = min(max(x, 0), 1) */
    t = (1.0f < t) ? 1.0f : t;
    const float *a, *b;
    float u;
    if (t < 0.33f) { a = c0; b = c1; u = t / 0.33f; }
    else if (t < 0.66f) { a = c1; b = c2; u = (t - 0.33f) / 0.33f; }
    else { a = c2; b = c3; u = (t - 0.66f) / 0.34f; }
    for (int k = 0; k < 3; k++) rgba[k] = a[k] * (1.0f - u) + b[k] * u; /* mix */
    rgba[3] = 1.0f;
}

/* updateVelocities main (updateVelocities.comp:71-118): v += g dt;
 * x += v dt (dt_scale = 1); walls with margin particleRadius + 0.5. */
void pfso_integrate(const pfs_params* p, uint32_t n, float* pos4, float* vel4, float* rgba4) {
    PAR_FOR
    for (int64_t i = 0; i < (int64_t)n; i++) {
        float pos[3], vel[3];
        for (int a = 0; a < 3; a++) {
            vel[a] = vel4[4 * i + a] + p->gravity[a] * p->dt;
            pos[a] = pos4[4 * i + a] + vel[a] * p->dt * 1.0f;
        }
        walls(p, p->margin_integrate, pos, vel);
        for (int a = 0; a < 3; a++) { pos4[4 * i + a] = pos[a]; vel4[4 * i + a] = vel[a]; }
        pos4[4 * i + 3] = 1.0f;
        vel4[4 * i + 3] = 1.0f;
        if (rgba4) pfso_color(vel4 + 4 * i, rgba4 + 4 * i);
    }
}

/* One substep in the dispatch order of commands.c:193-402: keys from x,
 * stable sort, reorder (scatterPass.comp:50-65) with the prediction applied
 * to the reordered state (predict is per particle, so predict-then-gather and
 * gather-then-predict agree), table, density, force, integrate. */
int pfso_substep(const pfs_params* p, uint32_t n, float* pos4, float* vel4,
                 pfs_debug_substep* tr, float* density_out, uint32_t* ids, float* rgba4) {
    if (n == 0) return PFS_OK;
    size_t n4 = (size_t)n * 4;
    uint32_t* keys = malloc(n * sizeof(uint32_t));
    uint32_t* sk = malloc(n * sizeof(uint32_t));
    uint32_t* perm = malloc(n * sizeof(uint32_t));
    int32_t* start = malloc(n * sizeof(int32_t));
    int32_t* end = malloc(n * sizeof(int32_t));
    float* xs = malloc(n4 * sizeof(float));
    float* vs = malloc(n4 * sizeof(float));
    float* xp = malloc(n4 * sizeof(float));
    float* vp = malloc(n4 * sizeof(float));
    float* vf = malloc(n4 * sizeof(float));
    float* rho = malloc(n * sizeof(float));
    float* rhon = malloc(n * sizeof(float));
    if (!keys || !sk || !perm || !start || !end || !xs || !vs || !xp || !vp || !vf || !rho || !rhon) {
        free(keys); free(sk); free(perm); free(start); free(end); free(xs); free(vs);
        free(xp); free(vp); free(vf); free(rho); free(rhon);
        return PFS_ENOMEM;
    }
    pfso_keys(p, n, pos4, keys);
    pfso_sort(n, keys, sk, perm);
    PAR_FOR
    for (int64_t s = 0; s < (int64_t)n; s++) {
        memcpy(xs + 4 * s, pos4 + 4 * (size_t)perm[s], 16);
        memcpy(vs + 4 * s, vel4 + 4 * (size_t)perm[s], 16);
    }
    pfso_predict(p, n, xs, vs, xp, vp);
    pfso_table(n, sk, start, end);
    pfso_density(p, n, xp, start, end, rho, rhon);
    pfso_force(p, n, xp, vp, vs, rho, rhon, start, end, vf);
    if (tr) {
        if (tr->keys_in) memcpy(tr->keys_in, keys, n * sizeof(uint32_t));
        if (tr->keys) memcpy(tr->keys, sk, n * sizeof(uint32_t));
        if (tr->perm) memcpy(tr->perm, perm, n * sizeof(uint32_t));
        if (tr->start) memcpy(tr->start, start, n * sizeof(int32_t));
        if (tr->end) memcpy(tr->end, end, n * sizeof(int32_t));
        if (tr->xp) memcpy(tr->xp, xp, n4 * sizeof(float));
        if (tr->vp) memcpy(tr->vp, vp, n4 * sizeof(float));
        if (tr->density) memcpy(tr->density, rho, n * sizeof(float));
        if (tr->near_density) memcpy(tr->near_density, rhon, n * sizeof(float));
        if (tr->vel_force) memcpy(tr->vel_force, vf, n4 * sizeof(float));
    }
    memcpy(pos4, xs, n4 * sizeof(float));
    memcpy(vel4, vf, n4 * sizeof(float));
    pfso_integrate(p, n, pos4, vel4, rgba4);
    if (density_out) memcpy(density_out, rho, n * sizeof(float));
    if (ids) {
        for (uint32_t s = 0; s < n; s++) keys[s] = ids[perm[s]];
        memcpy(ids, keys, n * sizeof(uint32_t));
    }
    free(keys); free(sk); free(perm); free(start); free(end); free(xs); free(vs);
    free(xp); free(vp); free(vf); free(rho); free(rhon);
    return PFS_OK;
}

int pfso_step(const pfs_params* p, uint32_t n, float* pos4, float* vel4, uint32_t nsteps,
              float* density, uint32_t* ids) {
    int subs = p->substeps > 0 ? p->substeps : 1;
    for (uint32_t s = 0; s < nsteps; s++)
        for (int k = 0; k < subs; k++) {
            int rc = pfso_substep(p, n, pos4, vel4, NULL, density, ids, NULL);
            if (rc) return rc;
        }
    return PFS_OK;
}

/* FP64 reference for a subset of sorted slots: same neighbour enumeration
 * (cell decisions in float, as the reference takes them), double arithmetic
 * for distances, kernels, accumulation and the velocity update. */
void pfso_subset_f64(const pfs_params* p, uint32_t n, const float* xp4, const float* vp4,
                     const float* vel4, const int32_t* start, const int32_t* end, uint32_t m_cnt,
                     const uint32_t* subset, double* dens_out, double* near_out, double* vel3) {
    pfso_consts c;
    pfso_derive(p, n, &c);
    const double h = p->h, m = p->particle_mass, PI = M_PI;
    const double volume = p->volume > 0.0f ? (double)p->volume : 2.0 * PI * pow(h, 5) / 15.0;
    const double near_inv = 15.0 / (PI * pow(h, 6));
    const double slope_scale = 15.0 / (PI * pow(h, 5));
    const double near_slope = -45.0 / (PI * pow(h, 6));
    double* rho = malloc(sizeof(double) * (size_t)n);
    double* rhon = malloc(sizeof(double) * (size_t)n);
    /* densities of every slot are needed for the force terms of the subset;
     * computed in double for all slots */
    PAR_FOR_DYN
    for (int64_t i = 0; i < (int64_t)n; i++) {
        const float* sp = xp4 + 4 * i;
        double t = 0.0, tn = 0.0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    float s[3] = {sp[0] + p->h * (float)dx, sp[1] + p->h * (float)dy,
                                  sp[2] + p->h * (float)dz};
                    if (s[0] < p->box_min[0] || s[1] < p->box_min[1] || s[2] < p->box_min[2] ||
                        s[0] > p->box_max[0] || s[1] > p->box_max[1] || s[2] > p->box_max[2])
                        continue;
                    uint32_t key = pfso_point_key(p, c.mask, s);
                    if (start[key] == -1) continue;
                    for (int32_t j = start[key]; j < end[key]; j++) {
                        const float* q = xp4 + 4 * (int64_t)j;
                        double a = (double)q[0] - sp[0], b = (double)q[1] - sp[1], e = (double)q[2] - sp[2];
                        double dist = sqrt(a * a + b * b + e * e);
                        if (dist >= h) continue;
                        t += m * (h - dist) * (h - dist);
                        tn += m * (h - dist) * (h - dist) * (h - dist);
                    }
                }
        double d = t / volume, nd = tn * near_inv;
        rho[i] = d < 0.01 ? 0.01 : d;
        rhon[i] = nd < 0.01 ? 0.01 : nd;
    }
    PAR_FOR_DYN
    for (int64_t u = 0; u < (int64_t)m_cnt; u++) {
        uint32_t i = subset[u];
        const float* sp = xp4 + 4 * (size_t)i;
        const float* pv = vp4 + 4 * (size_t)i;
        int32_t cell[3];
        if (sp[0] < p->box_min[0] || sp[1] < p->box_min[1] || sp[2] < p->box_min[2] ||
            sp[0] > p->box_max[0] || sp[1] > p->box_max[1] || sp[2] > p->box_max[2]) {
            cell[0] = cell[1] = cell[2] = -1;
        } else {
            for (int a = 0; a < 3; a++) cell[a] = pfso_cell_coord(sp[a], p->box_min[a], p->h);
        }
        double fp[3] = {0, 0, 0}, fv[3] = {0, 0, 0};
        double np_i = rhon[i] * p->near_pressure_multiplier;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    uint32_t key = pfso_cell_hash((uint32_t)cell[0] + (uint32_t)dx,
                                                  (uint32_t)cell[1] + (uint32_t)dy,
                                                  (uint32_t)cell[2] + (uint32_t)dz) & c.mask;
                    if (start[key] == -1) continue;
                    for (int32_t j = start[key]; j < end[key]; j++) {
                        if (j == (int32_t)i) continue;
                        const float* q = xp4 + 4 * (int64_t)j;
                        double d[3] = {(double)q[0] - sp[0], (double)q[1] - sp[1], (double)q[2] - sp[2]};
                        double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                        if (dist >= h || dist < 1e-7) continue;
                        double shared = ((rho[j] - p->target_density) * p->pressure_multiplier +
                                         (rho[i] - p->target_density) * p->pressure_multiplier) / 2.0;
                        double coef = shared * (dist - h) * slope_scale * m / rho[j];
                        double vcoef = m * (h - dist) * (h - dist) / rho[j];
                        double snp = (np_i + rhon[j] * p->near_pressure_multiplier) / 2.0;
                        double ncoef = snp * (h - dist) * (h - dist) * near_slope * m / rhon[j];
                        const float* vj = vel4 + 4 * (int64_t)j;
                        for (int a = 0; a < 3; a++) {
                            fp[a] += (coef + ncoef) * d[a] / dist;
                            fv[a] += vcoef * ((double)vj[a] - pv[a]);
                        }
                    }
                }
        dens_out[u] = rho[i];
        near_out[u] = rhon[i];
        for (int a = 0; a < 3; a++)
            vel3[3 * u + a] = (double)vel4[4 * (size_t)i + a] +
                              (fp[a] + (double)p->viscosity * fv[a]) / rho[i] * (double)p->dt;
    }
    free(rho);
    free(rhon);
}
