/*
 * nicp_synth.h -- seeded synthetic depth frames for NICP workloads.
 *
 * Renders uint16 depth images (millimetres) of a procedural room -- an
 * axis-aligned box with random spheres and random axis-aligned boxes inside
 * -- by ray casting through a pinhole camera, then adds depth noise
 * N(0, (sigma_coef * z^2)^2) metres and zeroes a random fraction of pixels.
 * Every pixel draws its noise from a counter-based hash of (noise_seed,
 * pixel), so output is identical for any thread count.
 *
 * This is input generation for tests and benchmarks; it is not part of the
 * registration path.
 */
#ifndef NICP_SYNTH_H
#define NICP_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NICP_SYNTH_MAX_OBJ 16

typedef struct {
  double room_min[3], room_max[3];
  int num_spheres;
  double spheres[NICP_SYNTH_MAX_OBJ][4]; /* cx, cy, cz, r */
  int num_boxes;
  double boxes[NICP_SYNTH_MAX_OBJ][6];   /* min xyz, max xyz */
} nicp_synth_scene;

enum {
  NICP_SYNTH_ROOM = 0,      /* 3 x 3 x 4 m room, 6 spheres r 0.1-0.4, 4 boxes */
  NICP_SYNTH_FAR_ROOM = 1   /* 8 x 4 x 8.5 m hall: depths 0.5 - 8 m        */
};

/* Fills *out with a scene drawn from `seed`.  Returns 0 on success. */
int nicp_synth_scene_make(uint64_t seed, int kind, nicp_synth_scene *out);

/* Renders one frame.  pose16: camera-to-world, row-major 4x4 (camera axes:
 * x right, y down, z forward).  Returns the number of non-zero pixels. */
int nicp_synth_render(const nicp_synth_scene *scene, const double *pose16, float fx, float fy, float cx,
                      float cy, int rows, int cols, uint64_t noise_seed, double sigma_coef,
                      double drop_prob, uint16_t *out);

#ifdef __cplusplus
}
#endif
#endif
