/* A C host calling the world step as the reference's C program would, in
 * place of the substep block of recordCommands (src/renderer/commands.c:
 * 193-402): create a world from host particle arrays and parameters, step,
 * read back, render a frame.  Built and run by the CPU tests; without a GPU
 * every device call must fail with a status, never abort.  With a path
 * argument it also writes n, the parameters, the input positions and the
 * stepped positions there (raw, native byte order) so a GPU test can check
 * the step against the oracle. */
#include <stdio.h>
#include <stdlib.h>

#include "pfs.h"

static pfs_world *g_world;
static pfs_params g_params;

static int sph_init(const float *pos4, const float *vel4, uint32_t n) {
    pfs_params p;
    pfs_params_reference_default(&p);
    p.h = 0.035f;
    p.target_density = 1000.0f;
    p.pressure_multiplier = 200.0f;
    p.viscosity = 0.05f;
    p.dt = (1.0f / 120.0f) / 3.0f;
    p.substeps = 3;
    p.flags |= PFS_FLAG_COLORS; /* the splats read the speed colour ramp */
    g_params = p;
    int rc = pfs_params_validate(&p);
    if (rc) return rc;
    return pfs_world_create(&p, n, pos4, vel4, &g_world);
}

static int sph_frame(float *pos4_out, float *rgba_out, uint32_t w, uint32_t h) {
    int rc = pfs_world_step(g_world, 1);
    if (!rc) rc = pfs_world_sync(g_world, 100000000ull);
    if (!rc) rc = pfs_world_read(g_world, pos4_out, NULL, NULL, NULL, NULL);
    if (!rc) {
        pfs_splat_view sv = {0};
        sv.model[0] = sv.model[5] = sv.model[10] = sv.model[15] = 1.0f;
        sv.view[0] = sv.view[5] = sv.view[10] = sv.view[15] = 1.0f;
        sv.proj[0] = sv.proj[5] = sv.proj[10] = sv.proj[15] = 1.0f;
        sv.particle_radius = 0.01f;
        rc = pfs_world_render_splats(g_world, &sv, w, h, rgba_out, NULL);
    }
    return rc;
}

static int dump(const char *path, uint32_t n, const float *pos_in, const float *pos_out) {
    FILE *f = fopen(path, "wb");
    if (!f) return 1;
    int bad = fwrite(&n, sizeof n, 1, f) != 1 || fwrite(&g_params, sizeof g_params, 1, f) != 1 ||
              fwrite(pos_in, 16, n, f) != n || fwrite(pos_out, 16, n, f) != n;
    return fclose(f) != 0 || bad;
}

int main(int argc, char **argv) {
    const uint32_t n = 64;
    float *pos = calloc(4 * n, sizeof(float)), *vel = calloc(4 * n, sizeof(float));
    float *out = calloc(4 * n, sizeof(float)), *rgba = calloc(4 * 16 * 16, sizeof(float));
    if (!pos || !vel || !out || !rgba) return 2;
    for (uint32_t i = 0; i < n; i++) {
        pos[4 * i + 0] = 0.1f + 0.01f * (float)(i % 4);
        pos[4 * i + 1] = 0.1f + 0.01f * (float)((i / 4) % 4);
        pos[4 * i + 2] = 0.1f + 0.01f * (float)(i / 16);
    }
    int rc = sph_init(pos, vel, n);
    if (!rc) rc = sph_frame(out, rgba, 16, 16);
    printf("status %d: %s\n", rc, pfs_strerror(rc));
    if (!rc && argc > 1 && dump(argv[1], n, pos, out)) return 3;
    if (g_world) pfs_world_destroy(g_world);
    free(pos);
    free(vel);
    free(out);
    free(rgba);
    /* a failure is reported as a status, never by exiting from the library */
    return 0;
}
