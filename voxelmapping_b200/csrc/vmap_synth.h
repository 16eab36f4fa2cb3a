// Synthetic RGB-D scene generator (input data for tests and benchmarks; the
// reference has no counterpart: its example reads TUM-format datasets).
#ifndef VMAP_SYNTH_H
#define VMAP_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VMAP_SYNTH_MAX_SPHERES 16

enum { VMAP_TRAJ_CIRCLE = 0, VMAP_TRAJ_FIGURE8 = 1 };

typedef struct vmap_scene_desc {
    uint64_t seed;
    double size[3];     /* room extent x, y (centred on 0) and height z (from 0) */
    int n_spheres;      /* radius U(0.1, 0.5) m, scaled down for rooms under 4 m */
    double cam_radius;  /* camera path half-width, kept clear of spheres */
    double cam_height;
} vmap_scene_desc;

typedef struct vmap_scene vmap_scene;

int vmap_synth_scene_create(const vmap_scene_desc* desc, vmap_scene** out);
void vmap_synth_scene_destroy(vmap_scene* s);
/* Writes n_spheres x (cx, cy, cz, r); returns n_spheres. */
int vmap_synth_scene_spheres(const vmap_scene* s, double* out);

/* n camera-to-world poses (row-major 4x4 doubles) on a circle of `radius`
 * looking at the room centre, or on a figure-8. */
int vmap_synth_trajectory(int kind, int n, double radius, double height, double* poses);

/* Render one frame. depth_mm: uint16 millimetres (0 = no measurement); with
 * `noisy`, N(0, 0.0012 + 0.0019 (z - 0.4)^2) m axial noise; `dropout` is the
 * fraction of pixels zeroed. rgb: uint8x3 per pixel; depth_true: exact depth in
 * metres (float). Any output may be NULL. */
int vmap_synth_render(const vmap_scene* s, const double* pose, int w, int h, double fx, double fy, double cx,
                      double cy, uint64_t frame_seed, int noisy, double dropout, uint16_t* depth_mm, uint8_t* rgb,
                      float* depth_true);

#ifdef __cplusplus
}
#endif
#endif
