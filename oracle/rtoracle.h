/*
 * Oracle (test infrastructure only): a plain-C, double-precision restatement of
 * the reference CPU renderer's algorithm for the path-tracing hot path. It is the
 * checker the GPU path is compared against, never part of the product.
 *
 * Input is a compiled scene in the reference's own layout (the record formats of
 * rtg_scene_view in include/rtg.h). Pinned against the reference itself (built
 * from its sources by oracle/Makefile into oracle/_ref/) by tests/test_oracle.py.
 */
#ifndef RTORACLE_H
#define RTORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ro_scene {
  uint64_t n_prims, n_planes, n_nodes, n_order, n_lights, n_point_lights, n_materials;
  const double* prims;        /* 24 per primitive */
  const double* planes;       /* 8 per plane */
  const double* nodes;        /* 10 per node */
  const uint32_t* order;      /* Bvh::prim_indices */
  const uint32_t* lights;     /* 2 per light */
  const double* point_lights; /* 6 per point light */
  const double* materials;    /* 16 per material */
  double camera[19];
  double background[8];
  /* light_sampling: 0 off, 1 NEE (the reference), 2 NEE with MIS (the GPU's opt-in extension) */
  int32_t width, height, spp, max_depth, rr_min_depth, integrator, light_sampling, use_bvh;
  uint64_t seed;
} ro_scene;

/* Raw PCG32 stream of Rng::for_sample(seed, pixel, sample). */
void ro_rng(uint64_t seed, uint64_t pixel, uint64_t sample, uint32_t* out, int32_t n);

/* Scene::intersect (brute = 0) or Scene::intersect_brute (brute = 1).
 * rays: n x 8 (o(3), tmin, d(3), tmax). Outputs: t, prim (-1 miss), is_plane,
 * geometric normal facing the ray (3 per ray; may be NULL). */
void ro_closest(const ro_scene* s, const double* rays, int64_t n, int32_t brute, double* t, int32_t* prim,
                int32_t* is_plane, double* gn);

/* Scene::occluded(ray, tmax) with tmin = 1e-6: rays n x 8 (tmax taken from the record). */
void ro_occluded(const ro_scene* s, const double* rays, int64_t n, uint8_t* out);

/* Camera::generate for n (i, j, sx, sy) records (lens draws from the sample's
 * stream when the aperture is open): out n x 6 (origin, direction). */
void ro_camera(const ro_scene* s, const double* pix, int64_t n, uint64_t pixel_for_rng, double* out);

/* Renders rows [y0, y1) with samples [s0, s1) of every pixel, accumulating the
 * per-pixel sum and sum of squares of the sample radiance (3 doubles per pixel,
 * indexed y * width + x over the full image) exactly as Renderer::render_tile
 * does (non-finite or negative samples count as invalid and become black).
 * stats: [rays, shadow_rays, rr_terminated, invalid]. */
void ro_render_rows(const ro_scene* s, int32_t y0, int32_t y1, uint32_t s0, uint32_t s1, double* sum, double* sumsq,
                    uint64_t* stats);

/* Radiance of one explicit primary sample (pixel x, y, sample index). */
void ro_sample(const ro_scene* s, int32_t x, int32_t y, uint32_t sample, double* rgb);

/* tone_map (op 0 clamp, 1 reinhard, 2 aces) then linear_to_srgb8 per channel. */
void ro_tone_map_srgb8(const double* rgb, int64_t n, int32_t op, double exposure, uint8_t* out);

#ifdef __cplusplus
}
#endif

#endif
