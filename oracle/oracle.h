// Test infrastructure only: CPU oracle for the GPU path tracer.
//
// A plain-C restatement of nodebleed's hot path (rend.c), used by tests/ and
// by the CPU-baseline leg of bench.py as the checker.  Never linked into the
// product.  Parity is pinned by comparing this restatement with the reference
// compiled from its own sources (_ref/libnbref.so) on the same rays.

#ifndef NB_ORACLE_H
#define NB_ORACLE_H

#include <stdint.h>
#include "../nodebleed_b200/csrc/host/nb_rdata.h"

#ifdef __cplusplus
extern "C" {
#endif

// A ray: ox oy oz tmax dx dy dz pad (32 bytes).  A hit: t u v id (16 bytes),
// id = tri << 12 | inst (rend.c:24-25), t = FLT_MAX on a miss.
struct orc_hit {
	float    t, u, v;
	uint32_t id;
};

// Visit counts of the reference algorithm: inner-node fetches (256 B
// each), leaf4 fetches (192 B), instance transforms (64 B), rays.
struct orc_counts {
	uint64_t nodes, leaves, insts, rays;
};

// Signatures of rend.c:1976 intersect_tlas and rend.c:2883
// intersect_any_tlas, so the path tracer can run on either the restatement
// below or the compiled reference.
typedef void (*orc_closest_fn)(float *t, float *u, float *v, unsigned int *id,
                               float ox, float oy, float oz,
                               float dx, float dy, float dz,
                               struct nb_bnode8 *nodes, struct nb_rinst *insts,
                               unsigned int tlasofs);
typedef int (*orc_any_fn)(float tfar, float ox, float oy, float oz,
                          float dx, float dy, float dz,
                          struct nb_bnode8 *nodes, struct nb_rinst *insts,
                          unsigned int tlasofs);

// Restatement of intersect_tlas / intersect_any_tlas (1/det by an exact
// division instead of rcpps).  The _cnt variant adds visit counts.
void orc_intersect_tlas(float *t, float *u, float *v, unsigned int *id,
                        float ox, float oy, float oz,
                        float dx, float dy, float dz,
                        struct nb_bnode8 *nodes, struct nb_rinst *insts,
                        unsigned int tlasofs);
int  orc_intersect_any_tlas(float tfar, float ox, float oy, float oz,
                            float dx, float dy, float dz,
                            struct nb_bnode8 *nodes, struct nb_rinst *insts,
                            unsigned int tlasofs);

// Batches over threads.  counts may be NULL.
void orc_trace(const struct nb_rdata *rd, const float *rays, uint32_t n,
               struct orc_hit *hits, struct orc_counts *counts, int nthreads);
void orc_occluded(const struct nb_rdata *rd, const float *rays, uint32_t n,
                  uint8_t *occl, int nthreads);

// Object-space ray of instance `inst` (the fixed FP32 transform both the
// GPU kernel and this oracle use), and the refined hit (t, u, v) of triangle
// `prim` of that instance: t by double-float plane intersection, u/v by
// Moeller-Trumbore with exact division.
void orc_object_ray(const struct nb_rdata *rd, uint32_t inst,
                    const float o[3], const float d[3], float oo[3],
                    float od[3]);
void orc_refine(const struct nb_rdata *rd, const float *rays, uint32_t n,
                struct orc_hit *hits);

// FP64 re-intersection of the hit triangle (id) with the FP32 object-space
// ray: writes t and the barycentrics (b0, b1, b2) per ray; NaN on no id.
void orc_reintersect_f64(const struct nb_rdata *rd, const float *rays,
                         const uint32_t *ids, uint32_t n, double *t64,
                         double *bary64);

// First-order forward error bounds of Moeller-Trumbore evaluated in FP32
// (rend.c:843-926) for triangle `id` of each ray: out[3i..3i+2] = bounds on
// |du|, |dv| and |dt| (8 units of 2^-24 per rounded term, plus the relative
// error of det carried into u, v, t).  Large for grazing rays and for
// triangles small against their distance from the ray origin.
void orc_mt_bounds(const struct nb_rdata *rd, const float *rays,
                   const uint32_t *ids, uint32_t n, double *out);

// Closest hit in FP64 by testing every triangle of every instance whose
// world box the ray enters (ground truth for a handful of rays): id and t per
// ray, t = INFINITY and id = 0 on a miss.
void orc_bruteforce_f64(const struct nb_rdata *rd, const float *rays,
                        uint32_t n, uint32_t *ids, double *t);

// Light table entry: 20 floats = v0[3] e0[3] e1[3] n[3] emit[3] cdf area
// pad[3] (world space; n the emitting side; cdf the running area fraction).
#define ORC_LIGHT_FLOATS 20

enum { ORC_MODE_PATH = 0, ORC_MODE_PRIMARY = 1 };

struct orc_pt_cfg {
	uint64_t       seed;
	uint32_t       depth;      // closest-hit rays per path at most
	uint32_t       mode;       // ORC_MODE_*
	int            nthreads;
	uint32_t       nlights;
	const float    *lights;    // nlights * ORC_LIGHT_FLOATS
	float          light_area; // total emitting area
	uint32_t       x0, y0, x1, y1; // pixel window [x0,x1) x [y0,y1)
	orc_closest_fn closest;    // NULL: the restatement
	orc_any_fn     any;        // NULL: the restatement
	struct orc_counts *counts; // visit counts of closest-hit traversals
	                           // (restatement only); may be NULL
};

// One frame of `rd->spp` samples per pixel for the pixels of the window:
// rad[(y*W + x)*3 + c] = sum over the samples of the path radiance.  Frame key
// is rd->samples (rd is not modified).  Returns the rays traced (closest +
// shadow), counted as rend.c:3154/3264 do.
uint64_t orc_render(const struct nb_rdata *rd, const struct orc_pt_cfg *cfg,
                    float *rad);

// acc += rad over the whole image, then buf = ARGB8 of acc / (samples+spp)
// (rend.c:3565-3580); the caller then bumps rd->samples.
void orc_accumulate(struct nb_rdata *rd, const float *rad);

// Per-path PCG32 and the sampling helpers, exported for unit tests.
uint32_t orc_pcg_first(uint64_t seed, uint32_t frame, uint64_t path,
                       uint32_t count, uint32_t *out);
void     orc_sincos2pi(float u, float *s, float *c);

// GGX conductor of the path tracer, exported for unit tests: for shading
// normal n, outgoing direction wo (both unit, n.wo > 0), roughness alpha
// and uniforms r0, r1, the sampled direction wi and the sample weight
// F G1(wo) G1(wi) (wo.m) / ((n.wo) (n.m)) with F0 = f0 (w[3]); returns 0
// when the sample leaves the hemisphere.  orc_ggx_eval gives f(wo, wi)
// (the BRDF, per channel).
int  orc_ggx_sample(const float n[3], const float wo[3], float alpha,
                    const float f0[3], float r0, float r1, float wi[3],
                    float w[3]);
void orc_ggx_eval(const float n[3], const float wo[3], const float wi[3],
                  float alpha, const float f0[3], float f[3]);

#ifdef __cplusplus
}
#endif

#endif
