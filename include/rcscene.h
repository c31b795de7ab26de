/*
 * rcscene.h — seeded synthetic scene renderer for the dense-MVS path.
 *
 * The reference publishes no synthetic MVS scene (its demo scene feeds SfM
 * only, sfm-lite/src/demo.rs:41-116), so this renderer has no reference
 * counterpart.  It ray-casts a room made of rectangles, axis-aligned boxes
 * and spheres, textured with 4-octave value noise plus flat rectangles, and
 * writes grey images with analytic ground-truth depth (z in the camera) and
 * normals.  Cameras are pinhole (k = 0) with the reference's pixel-centre
 * convention (sfm-lite/src/geom.rs:28-42).  The CPU and GPU paths compute
 * the same IEEE operations in the same order and give identical images.
 */
#ifndef RCSCENE_H
#define RCSCENE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define RCSCENE_RECT 0   /* p: origin[3], u[3], v[3] (unit, orthogonal), U, V */
#define RCSCENE_BOX 1    /* p: min[3], max[3] */
#define RCSCENE_SPHERE 2 /* p: centre[3], radius */

typedef struct rcscene_prim {
    int32_t kind;
    int32_t tex_seed;
    float tex_freq;   /* base noise frequency (cycles per unit) */
    float tex_lo;     /* grey at noise 0 */
    float tex_hi;     /* grey at noise 1 */
    float p[11];
} rcscene_prim;

/* Flat-intensity rectangle painted on a RECT primitive, in its (u, v)
 * coordinates. Later rectangles paint over earlier ones. */
typedef struct rcscene_patch {
    int32_t prim;
    float u0, v0, u1, v1;
    float value;
} rcscene_patch;

typedef struct rcscene_cam {
    int32_t w, h;
    double f, cx, cy;
    double R[9];      /* world->camera, row-major */
    double t[3];
} rcscene_cam;

/* Renders n_cams views.  gray_out[i]: w*h u8; depth_out[i]: w*h f32 (0 = no
 * hit); normal_out (nullable) [i]: 3*w*h f32 unit normal in the camera
 * frame.  supersample: s*s sub-rays per pixel for the grey value (depth and
 * normal come from the pixel-centre ray).  device < 0: CPU threads;
 * otherwise the CUDA device index.  Returns 0 on success. */
int rcscene_render(const rcscene_prim* prims, int32_t n_prims, const rcscene_patch* patches,
                   int32_t n_patches, const rcscene_cam* cams, int32_t n_cams, int32_t supersample,
                   int32_t device, uint8_t* const* gray_out, float* const* depth_out,
                   float* const* normal_out);

const char* rcscene_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
