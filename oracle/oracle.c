// Test infrastructure only: CPU oracle for the GPU path tracer (see oracle.h).
//
// Contents, each citing the reference code it restates:
//   closest-hit traversal   intersect_tlas rend.c:1976-2155,
//                           intersect_blas rend.c:714-968
//   any-hit traversal       intersect_any_tlas rend.c:2883-2998,
//                           intersect_any_blas rend.c:1797-1973
//   camera rays             make_camray_pckt rend.c:3293-3402 (one ray)
//   primary shading         trace_rays/calc_nrm rend.c:3404-3445, 3109-3116
//   path tracing            trace3 rend.c:3205-3291 (NEE + cosine bounce),
//                           create_onb rend.c:3126, rand_hemicos rend.c:3135
//   accumulation            accum_pckt rend.c:3565-3580
// Deviations, all deliberate and shared with the GPU kernels:
//   * 1/det of Moeller-Trumbore is an exact division (the reference uses
//     rcpps, 12-bit), camera directions are normalised with 1/sqrtf (the
//     reference uses rsqrtps); hit ids then differ only at ties.
//   * after the closest hit is found, t is recomputed by a double-float
//     plane intersection and u/v by Moeller-Trumbore with exact division,
//     so t is good to ~1 ulp of the FP32 inputs.
//   * random numbers are PCG32 per path (the reference: xorshift128+ per
//     block); sin/cos of the sampling angles use the Taylor polynomials below
//     so CPU and GPU produce the same bits.
//   * lights are the emissive triangles of the scene (trace3 hard-codes a
//     quad), shading normals face the incoming ray, mirrors reflect.
// Every float expression is written without contraction (compile with
// -ffp-contract=off); fused operations are explicit fmaf calls.

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define NODE_LEAF  0x80000000u
#define INST_BITS  12
#define INST_MASK  0xfffu
#define EPS2F      1e-3f          // util.h:8
#define INV_PI_F   0.318309886f   // util.h:11, 1/3.14159265

// ------------------------------------------------- SSE-like helpers --------

static inline float mm_max(float a, float b) { return a > b ? a : b; }
static inline float mm_min(float a, float b) { return a < b ? a : b; }
static inline int   le_oq(float a, float b) { return a <= b; }

// ------------------------------------------------- traversal ---------------

// Compact the first `spos` stack entries keeping those with dist <= t, in
// order (rend.c:928-959).
static unsigned int compact(unsigned int *stack, float *dstack,
                            unsigned int spos, float t)
{
	unsigned int k = 0;
	for (unsigned int i = 0; i < spos; i++)
		if (le_oq(dstack[i], t)) {
			stack[k] = stack[i];
			dstack[k] = dstack[i];
			k++;
		}
	return k;
}

struct slab {
	float idx, idy, idz, rx, ry, rz;
	int bdx, bdy, bdz;
	unsigned int shft;
};

static void slab_init(struct slab *s, float ox, float oy, float oz, float dx,
                      float dy, float dz)
{
	s->idx = 1.0f / dx;
	s->idy = 1.0f / dy;
	s->idz = 1.0f / dz;
	s->rx = ox * s->idx;
	s->ry = oy * s->idy;
	s->rz = oz * s->idz;
	s->bdx = dx >= 0.0f;
	s->bdy = dy >= 0.0f;
	s->bdz = dz >= 0.0f;
	s->shft = (unsigned int)((s->bdz << 2) | (s->bdy << 1) | s->bdx) * 3;
}

// 8 slab tests of one node (rend.c:757-787): hit mask and entry distances.
static unsigned int slab8(const struct slab *s, const struct nb_bnode8 *n,
                          float tcur, float tmin[8])
{
	unsigned int mask = 0;
	for (int i = 0; i < 8; i++) {
		float t0x = fmaf(s->bdx ? n->minx8[i] : n->maxx8[i], s->idx, -s->rx);
		float t0y = fmaf(s->bdy ? n->miny8[i] : n->maxy8[i], s->idy, -s->ry);
		float t0z = fmaf(s->bdz ? n->minz8[i] : n->maxz8[i], s->idz, -s->rz);
		float t1x = fmaf(s->bdx ? n->maxx8[i] : n->minx8[i], s->idx, -s->rx);
		float t1y = fmaf(s->bdy ? n->maxy8[i] : n->miny8[i], s->idy, -s->ry);
		float t1z = fmaf(s->bdz ? n->maxz8[i] : n->minz8[i], s->idz, -s->rz);
		float lo = mm_max(mm_max(mm_max(t0x, t0y), t0z), 0.0f);
		float hi = mm_min(mm_min(mm_min(t1x, t1y), t1z), tcur);
		tmin[i] = lo;
		if (le_oq(lo, hi))
			mask |= 1u << i;
	}
	return mask;
}

static inline int highest_bit(unsigned int m)
{
	return 31 - __builtin_clz(m);
}

// Ordered push of the hit children (rend.c:803-838): children sorted by the
// node's octant permutation, hits compressed to the front; the last one is
// taken next.  Returns the node to continue with.
static unsigned int push_ordered(const struct nb_bnode8 *n, unsigned int mask,
                                 const float tmin[8], unsigned int shft,
                                 unsigned int *stack, float *dstack,
                                 unsigned int *spos)
{
	unsigned int k = *spos;
	for (int i = 0; i < 8; i++) {
		unsigned int c = (n->perm8[i] >> shft) & 7u;
		if (mask & (1u << c)) {
			stack[k] = n->children8[c];
			dstack[k] = tmin[c];
			k++;
		}
	}
	*spos = k - 1;
	return stack[k - 1];
}

// Moeller-Trumbore x4 of one leaf4 (rend.c:843-926) with exact 1/det.
static int leaf_hit(const struct nb_leaf4 *l, float ox, float oy, float oz,
                    float dx, float dy, float dz, float tcur, float *t,
                    float *u, float *v, unsigned int *lane)
{
	float tt[4], uu[4], vv[4];
	int mask = 0;
	for (int i = 0; i < 4; i++) {
		float pvx = fmaf(dy, l->e1z4[i], -(dz * l->e1y4[i]));
		float pvy = fmaf(dz, l->e1x4[i], -(dx * l->e1z4[i]));
		float pvz = fmaf(dx, l->e1y4[i], -(dy * l->e1x4[i]));
		float tvx = ox - l->v0x4[i];
		float tvy = oy - l->v0y4[i];
		float tvz = oz - l->v0z4[i];
		float det = fmaf(l->e0x4[i], pvx, fmaf(l->e0y4[i], pvy,
		  l->e0z4[i] * pvz));
		float qvx = fmaf(tvy, l->e0z4[i], -(tvz * l->e0y4[i]));
		float qvy = fmaf(tvz, l->e0x4[i], -(tvx * l->e0z4[i]));
		float qvz = fmaf(tvx, l->e0y4[i], -(tvy * l->e0x4[i]));
		float idet = 1.0f / det;
		uu[i] = idet * fmaf(tvx, pvx, fmaf(tvy, pvy, tvz * pvz));
		vv[i] = idet * fmaf(dx, qvx, fmaf(dy, qvy, dz * qvz));
		tt[i] = idet * fmaf(l->e1x4[i], qvx, fmaf(l->e1y4[i], qvy,
		  l->e1z4[i] * qvz));
		if (uu[i] >= 0.0f && vv[i] >= 0.0f && uu[i] + vv[i] <= 1.0f &&
		  tt[i] > 0.0f && tt[i] < tcur)
			mask |= 1 << i;
	}
	if (!mask)
		return 0;
	// closest; among equal t the highest lane (rend.c:898-905)
	float best = FLT_MAX;
	for (int i = 0; i < 4; i++)
		if ((mask >> i) & 1)
			best = mm_min(tt[i], best);
	int pick = 0;
	for (int i = 0; i < 4; i++)
		if (((mask >> i) & 1 ? tt[i] : FLT_MAX) == best)
			pick = i;
	*t = tt[pick];
	*u = uu[pick];
	*v = vv[pick];
	*lane = (unsigned int)pick;
	return 1;
}

struct tcount { uint64_t nodes, leaves, insts; };

static void blas_closest(float *t, float *u, float *v, unsigned int *id,
                         float ox, float oy, float oz, float dx, float dy,
                         float dz, const struct nb_bnode8 *blas,
                         unsigned int instid, struct tcount *tc)
{
	unsigned int stack[72];
	float dstack[72];
	unsigned int spos = 0, ofs = 0;
	const unsigned char *ptr = (const unsigned char *)blas;
	struct slab s;
	slab_init(&s, ox, oy, oz, dx, dy, dz);
	float tmin[8];
	for (;;) {
		while (!(ofs & NODE_LEAF)) {
			const struct nb_bnode8 *n =
			  (const struct nb_bnode8 *)(ptr + ofs);
			if (tc)
				tc->nodes++;
			unsigned int m = slab8(&s, n, *t, tmin);
			int cnt = __builtin_popcount(m);
			if (cnt == 0) {
				if (!spos)
					return;
				ofs = stack[--spos];
			} else if (cnt == 1) {
				ofs = n->children8[highest_bit(m)];
			} else {
				ofs = push_ordered(n, m, tmin, s.shft, stack,
				  dstack, &spos);
			}
		}
		const struct nb_leaf4 *l =
		  (const struct nb_leaf4 *)(ptr + (ofs & ~NODE_LEAF));
		if (tc)
			tc->leaves++;
		float lt, lu, lv;
		unsigned int lane;
		if (leaf_hit(l, ox, oy, oz, dx, dy, dz, *t, &lt, &lu, &lv,
		  &lane)) {
			*t = lt;
			*u = lu;
			*v = lv;
			*id = (l->id4[lane] << INST_BITS) | instid;
			spos = compact(stack, dstack, spos, *t);
		}
		if (!spos)
			return;
		ofs = stack[--spos];
	}
}

// World -> object with the instance's 3x4 (rend.c:2096-2102), written as a
// fixed sequence of fused operations; the GPU kernel uses the same sequence.
static inline void xform_pos(const float *m, float x, float y, float z,
                             float *o)
{
	o[0] = fmaf(m[0], x, fmaf(m[1], y, fmaf(m[2], z, m[3])));
	o[1] = fmaf(m[4], x, fmaf(m[5], y, fmaf(m[6], z, m[7])));
	o[2] = fmaf(m[8], x, fmaf(m[9], y, fmaf(m[10], z, m[11])));
}

static inline void xform_dir(const float *m, float x, float y, float z,
                             float *o)
{
	o[0] = fmaf(m[0], x, fmaf(m[1], y, m[2] * z));
	o[1] = fmaf(m[4], x, fmaf(m[5], y, m[6] * z));
	o[2] = fmaf(m[8], x, fmaf(m[9], y, m[10] * z));
}

static void tlas_closest(float *t, float *u, float *v, unsigned int *id,
                         float ox, float oy, float oz, float dx, float dy,
                         float dz, const struct nb_bnode8 *nodes,
                         const struct nb_rinst *insts, unsigned int tlasofs,
                         struct tcount *tc)
{
	unsigned int stack[72];
	float dstack[72];
	unsigned int spos = 0, ofs = 0;
	const unsigned char *ptr = (const unsigned char *)&nodes[tlasofs];
	struct slab s;
	slab_init(&s, ox, oy, oz, dx, dy, dz);
	float tmin[8];
	for (;;) {
		while (!(ofs & NODE_LEAF)) {
			const struct nb_bnode8 *n =
			  (const struct nb_bnode8 *)(ptr + ofs);
			if (tc)
				tc->nodes++;
			unsigned int m = slab8(&s, n, *t, tmin);
			int cnt = __builtin_popcount(m);
			if (cnt == 0) {
				if (!spos)
					return;
				ofs = stack[--spos];
			} else if (cnt == 1) {
				ofs = n->children8[highest_bit(m)];
			} else {
				ofs = push_ordered(n, m, tmin, s.shft, stack,
				  dstack, &spos);
			}
		}
		unsigned int inst = ofs & ~NODE_LEAF;
		const struct nb_rinst *ri = &insts[inst];
		if (tc)
			tc->insts++;
		float lo[3], ld[3];
		xform_pos(ri->globinv, ox, oy, oz, lo);
		xform_dir(ri->globinv, dx, dy, dz, ld);
		float tt = *t;
		blas_closest(t, u, v, id, lo[0], lo[1], lo[2], ld[0], ld[1],
		  ld[2], &nodes[(size_t)ri->triofs << 1], inst, tc);
		if (*t < tt)
			spos = compact(stack, dstack, spos, *t);
		if (!spos)
			return;
		ofs = stack[--spos];
	}
}

void orc_intersect_tlas(float *t, float *u, float *v, unsigned int *id,
                        float ox, float oy, float oz,
                        float dx, float dy, float dz,
                        struct nb_bnode8 *nodes, struct nb_rinst *insts,
                        unsigned int tlasofs)
{
	tlas_closest(t, u, v, id, ox, oy, oz, dx, dy, dz, nodes, insts,
	  tlasofs, NULL);
}

static int blas_any(float tfar, float ox, float oy, float oz, float dx,
                    float dy, float dz, const struct nb_bnode8 *blas)
{
	unsigned int stack[72];
	unsigned int spos = 0, ofs = 0;
	const unsigned char *ptr = (const unsigned char *)blas;
	struct slab s;
	slab_init(&s, ox, oy, oz, dx, dy, dz);
	float tmin[8];
	for (;;) {
		while (!(ofs & NODE_LEAF)) {
			const struct nb_bnode8 *n =
			  (const struct nb_bnode8 *)(ptr + ofs);
			unsigned int m = slab8(&s, n, tfar, tmin);
			int cnt = __builtin_popcount(m);
			if (cnt == 0) {
				if (!spos)
					return 0;
				ofs = stack[--spos];
			} else if (cnt == 1) {
				ofs = n->children8[highest_bit(m)];
			} else {
				// unordered, lane order (rend.c:1883-1896)
				for (int i = 0; i < 8; i++)
					if (m & (1u << i))
						stack[spos++] = n->children8[i];
				ofs = stack[--spos];
			}
		}
		const struct nb_leaf4 *l =
		  (const struct nb_leaf4 *)(ptr + (ofs & ~NODE_LEAF));
		float lt, lu, lv;
		unsigned int lane;
		if (leaf_hit(l, ox, oy, oz, dx, dy, dz, tfar, &lt, &lu, &lv,
		  &lane))
			return 1;
		if (!spos)
			return 0;
		ofs = stack[--spos];
	}
}

int orc_intersect_any_tlas(float tfar, float ox, float oy, float oz,
                           float dx, float dy, float dz,
                           struct nb_bnode8 *nodes, struct nb_rinst *insts,
                           unsigned int tlasofs)
{
	unsigned int stack[72];
	unsigned int spos = 0, ofs = 0;
	const unsigned char *ptr = (const unsigned char *)&nodes[tlasofs];
	struct slab s;
	slab_init(&s, ox, oy, oz, dx, dy, dz);
	float tmin[8];
	for (;;) {
		while (!(ofs & NODE_LEAF)) {
			const struct nb_bnode8 *n =
			  (const struct nb_bnode8 *)(ptr + ofs);
			unsigned int m = slab8(&s, n, tfar, tmin);
			int cnt = __builtin_popcount(m);
			if (cnt == 0) {
				if (!spos)
					return 0;
				ofs = stack[--spos];
			} else if (cnt == 1) {
				ofs = n->children8[highest_bit(m)];
			} else {
				for (int i = 0; i < 8; i++)
					if (m & (1u << i))
						stack[spos++] = n->children8[i];
				ofs = stack[--spos];
			}
		}
		const struct nb_rinst *ri = &insts[ofs & ~NODE_LEAF];
		float lo[3], ld[3];
		xform_pos(ri->globinv, ox, oy, oz, lo);
		xform_dir(ri->globinv, dx, dy, dz, ld);
		if (blas_any(tfar, lo[0], lo[1], lo[2], ld[0], ld[1], ld[2],
		  &nodes[(size_t)ri->triofs << 1]))
			return 1;
		if (!spos)
			return 0;
		ofs = stack[--spos];
	}
}

// ------------------------------------------------- refinement --------------

// Double-float helpers (Dekker / Knuth error-free transforms).
struct df { float hi, lo; };

static inline struct df two_sum(float a, float b)
{
	float s = a + b;
	float bb = s - a;
	float e = (a - (s - bb)) + (b - bb);
	return (struct df){s, e};
}

static inline struct df fast_two_sum(float a, float b)
{
	float s = a + b;
	float e = b - (s - a);
	return (struct df){s, e};
}

static inline struct df two_prod(float a, float b)
{
	float p = a * b;
	return (struct df){p, fmaf(a, b, -p)};
}

static inline struct df df_add(struct df x, struct df y)
{
	struct df s = two_sum(x.hi, y.hi);
	float e = s.lo + (x.lo + y.lo);
	return fast_two_sum(s.hi, e);
}

static inline struct df df_neg(struct df x)
{
	return (struct df){-x.hi, -x.lo};
}

static inline struct df df_mul(struct df x, struct df y)
{
	struct df p = two_prod(x.hi, y.hi);
	float e = p.lo + (x.hi * y.lo + x.lo * y.hi);
	return fast_two_sum(p.hi, e);
}

static inline struct df df_div(struct df x, struct df y)
{
	float q1 = x.hi / y.hi;
	struct df r = df_add(x, df_neg(df_mul((struct df){q1, 0.0f}, y)));
	float q2 = r.hi / y.hi;
	return fast_two_sum(q1, q2);
}

// t of the plane through (v0, v1, v2) along o + t d, in double-float.
static float refine_t(const float o[3], const float d[3], const float v0[3],
                      const float v1[3], const float v2[3], float tfallback)
{
	struct df e0[3], e1[3], w[3];
	for (int a = 0; a < 3; a++) {
		e0[a] = two_sum(v1[a], -v0[a]);
		e1[a] = two_sum(v2[a], -v0[a]);
		w[a] = two_sum(v0[a], -o[a]);
	}
	struct df n[3];
	n[0] = df_add(df_mul(e0[1], e1[2]), df_neg(df_mul(e0[2], e1[1])));
	n[1] = df_add(df_mul(e0[2], e1[0]), df_neg(df_mul(e0[0], e1[2])));
	n[2] = df_add(df_mul(e0[0], e1[1]), df_neg(df_mul(e0[1], e1[0])));
	struct df num = df_add(df_add(df_mul(n[0], w[0]), df_mul(n[1], w[1])),
	  df_mul(n[2], w[2]));
	struct df den = df_add(df_add(
	  df_mul(n[0], (struct df){d[0], 0.0f}),
	  df_mul(n[1], (struct df){d[1], 0.0f})),
	  df_mul(n[2], (struct df){d[2], 0.0f}));
	if (den.hi == 0.0f)
		return tfallback;
	return df_div(num, den).hi;
}

// Barycentrics u, v by Moeller-Trumbore with an exact division, no fusion.
static void refine_uv(const float o[3], const float d[3], const float v0[3],
                      const float v1[3], const float v2[3], float *u,
                      float *v)
{
	float e0[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
	float e1[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
	float pv[3] = {d[1] * e1[2] - d[2] * e1[1], d[2] * e1[0] - d[0] * e1[2],
	  d[0] * e1[1] - d[1] * e1[0]};
	float det = e0[0] * pv[0] + e0[1] * pv[1] + e0[2] * pv[2];
	float tv[3] = {o[0] - v0[0], o[1] - v0[1], o[2] - v0[2]};
	float qv[3] = {tv[1] * e0[2] - tv[2] * e0[1],
	  tv[2] * e0[0] - tv[0] * e0[2], tv[0] * e0[1] - tv[1] * e0[0]};
	float uu = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) / det;
	float vv = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) / det;
	*u = uu == uu ? uu : 0.0f;
	*v = vv == vv ? vv : 0.0f;
}

void orc_object_ray(const struct nb_rdata *rd, uint32_t inst,
                    const float o[3], const float d[3], float oo[3],
                    float od[3])
{
	const float *m = rd->insts[inst].globinv;
	xform_pos(m, o[0], o[1], o[2], oo);
	xform_dir(m, d[0], d[1], d[2], od);
}

static void tri_verts(const struct nb_rdata *rd, uint32_t inst, uint32_t prim,
                      float v0[3], float v1[3], float v2[3])
{
	const struct nb_rtri *t = &rd->tris[rd->insts[inst].triofs + prim];
	v0[0] = t->v0.x; v0[1] = t->v0.y; v0[2] = t->v0.z;
	v1[0] = t->v1.x; v1[1] = t->v1.y; v1[2] = t->v1.z;
	v2[0] = t->v2.x; v2[1] = t->v2.y; v2[2] = t->v2.z;
}

static void refine_hit(const struct nb_rdata *rd, const float o[3],
                       const float d[3], struct orc_hit *h)
{
	uint32_t inst = h->id & INST_MASK, prim = h->id >> INST_BITS;
	float oo[3], od[3], v0[3], v1[3], v2[3];
	orc_object_ray(rd, inst, o, d, oo, od);
	tri_verts(rd, inst, prim, v0, v1, v2);
	h->t = refine_t(oo, od, v0, v1, v2, h->t);
	refine_uv(oo, od, v0, v1, v2, &h->u, &h->v);
}

void orc_refine(const struct nb_rdata *rd, const float *rays, uint32_t n,
                struct orc_hit *hits)
{
	for (uint32_t i = 0; i < n; i++) {
		if (hits[i].t == FLT_MAX)
			continue;
		const float *r = rays + 8ull * i;
		float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
		refine_hit(rd, o, d, &hits[i]);
	}
}

void orc_reintersect_f64(const struct nb_rdata *rd, const float *rays,
                         const uint32_t *ids, uint32_t n, double *t64,
                         double *bary64)
{
	for (uint32_t i = 0; i < n; i++) {
		const float *r = rays + 8ull * i;
		uint32_t inst = ids[i] & INST_MASK, prim = ids[i] >> INST_BITS;
		if (inst >= rd->instcnt) {
			t64[i] = NAN;
			bary64[3 * i] = bary64[3 * i + 1] = bary64[3 * i + 2] = NAN;
			continue;
		}
		float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
		float oo[3], od[3], v0[3], v1[3], v2[3];
		orc_object_ray(rd, inst, o, d, oo, od);
		tri_verts(rd, inst, prim, v0, v1, v2);
		double e0[3], e1[3], w[3], n3[3], q[3];
		for (int a = 0; a < 3; a++) {
			e0[a] = (double)v1[a] - v0[a];
			e1[a] = (double)v2[a] - v0[a];
			w[a] = (double)v0[a] - oo[a];
		}
		n3[0] = e0[1] * e1[2] - e0[2] * e1[1];
		n3[1] = e0[2] * e1[0] - e0[0] * e1[2];
		n3[2] = e0[0] * e1[1] - e0[1] * e1[0];
		double num = n3[0] * w[0] + n3[1] * w[1] + n3[2] * w[2];
		double den = n3[0] * od[0] + n3[1] * od[1] + n3[2] * od[2];
		double t = num / den;
		t64[i] = t;
		// barycentrics of the hit point: areas against the normal
		double p[3];
		for (int a = 0; a < 3; a++)
			p[a] = (double)oo[a] + t * od[a] - v0[a];
		double nn = n3[0] * n3[0] + n3[1] * n3[1] + n3[2] * n3[2];
		// b1 = ((p x e1) . n) / nn, b2 = ((e0 x p) . n) / nn
		q[0] = p[1] * e1[2] - p[2] * e1[1];
		q[1] = p[2] * e1[0] - p[0] * e1[2];
		q[2] = p[0] * e1[1] - p[1] * e1[0];
		double b1 = (q[0] * n3[0] + q[1] * n3[1] + q[2] * n3[2]) / nn;
		q[0] = e0[1] * p[2] - e0[2] * p[1];
		q[1] = e0[2] * p[0] - e0[0] * p[2];
		q[2] = e0[0] * p[1] - e0[1] * p[0];
		double b2 = (q[0] * n3[0] + q[1] * n3[1] + q[2] * n3[2]) / nn;
		bary64[3 * i] = 1.0 - b1 - b2;
		bary64[3 * i + 1] = b1;
		bary64[3 * i + 2] = b2;
	}
}

static double vlen3(const double *a)
{
	return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}

static double absdot3(const double *a, const double *b)
{
	return fabs(a[0] * b[0]) + fabs(a[1] * b[1]) + fabs(a[2] * b[2]);
}

void orc_mt_bounds(const struct nb_rdata *rd, const float *rays,
                   const uint32_t *ids, uint32_t n, double *out)
{
	const double eps = 8.0 * ldexp(1.0, -24);
	for (uint32_t i = 0; i < n; i++) {
		const float *r = rays + 8ull * i;
		uint32_t inst = ids[i] & INST_MASK, prim = ids[i] >> INST_BITS;
		if (inst >= rd->instcnt) {
			out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = 0.0;
			continue;
		}
		float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
		float oo[3], od[3], v0[3], v1[3], v2[3];
		orc_object_ray(rd, inst, o, d, oo, od);
		tri_verts(rd, inst, prim, v0, v1, v2);
		double e0[3], e1[3], tv[3], dd[3], pv[3], qv[3];
		for (int a = 0; a < 3; a++) {
			e0[a] = (double)v1[a] - v0[a];
			e1[a] = (double)v2[a] - v0[a];
			tv[a] = (double)oo[a] - v0[a];
			dd[a] = od[a];
		}
		pv[0] = dd[1] * e1[2] - dd[2] * e1[1];
		pv[1] = dd[2] * e1[0] - dd[0] * e1[2];
		pv[2] = dd[0] * e1[1] - dd[1] * e1[0];
		qv[0] = tv[1] * e0[2] - tv[2] * e0[1];
		qv[1] = tv[2] * e0[0] - tv[0] * e0[2];
		qv[2] = tv[0] * e0[1] - tv[1] * e0[0];
		double det = e0[0] * pv[0] + e0[1] * pv[1] + e0[2] * pv[2];
		double adet = fabs(det);
		if (adet == 0.0) {
			out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = INFINITY;
			continue;
		}
		double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) / det;
		double v = (dd[0] * qv[0] + dd[1] * qv[1] + dd[2] * qv[2]) / det;
		double t = (e1[0] * qv[0] + e1[1] * qv[1] + e1[2] * qv[2]) / det;
		double ld = vlen3(dd), l0 = vlen3(e0), l1 = vlen3(e1);
		double lt = vlen3(tv);
		double rdet = eps * (absdot3(e0, pv) + l0 * ld * l1) / adet;
		out[3 * i] = eps * (absdot3(tv, pv) + lt * ld * l1) / adet +
		  fabs(u) * rdet;
		out[3 * i + 1] = eps * (absdot3(dd, qv) + ld * lt * l0) / adet +
		  fabs(v) * rdet;
		out[3 * i + 2] = eps * (absdot3(e1, qv) + l1 * lt * l0) / adet +
		  fabs(t) * rdet;
	}
}

static int slab_f64(const double *o, const double *d, const struct nb_aabb *b,
                    double tbest)
{
	double lo = 0.0, hi = tbest;
	const float mn[3] = {b->min.x, b->min.y, b->min.z};
	const float mx[3] = {b->max.x, b->max.y, b->max.z};
	for (int a = 0; a < 3; a++) {
		if (d[a] == 0.0) {
			if (o[a] < mn[a] || o[a] > mx[a])
				return 0;
			continue;
		}
		double t0 = (mn[a] - o[a]) / d[a], t1 = (mx[a] - o[a]) / d[a];
		if (t0 > t1) {
			double x = t0;
			t0 = t1;
			t1 = x;
		}
		lo = t0 > lo ? t0 : lo;
		hi = t1 < hi ? t1 : hi;
	}
	return lo <= hi * (1.0 + 1e-9);
}

void orc_bruteforce_f64(const struct nb_rdata *rd, const float *rays,
                        uint32_t n, uint32_t *ids, double *tout)
{
	for (uint32_t i = 0; i < n; i++) {
		const float *r = rays + 8ull * i;
		double o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
		double best = r[3] == FLT_MAX ? INFINITY : (double)r[3];
		uint32_t bid = 0;
		for (uint32_t k = 0; k < rd->instcnt; k++) {
			if (!slab_f64(o, d, &rd->aabbs[k], best))
				continue;
			const struct nb_rinst *ri = &rd->insts[k];
			const float *g = ri->globinv;
			double oo[3], od[3];
			for (int a = 0; a < 3; a++) {
				oo[a] = g[4 * a] * o[0] + g[4 * a + 1] * o[1] +
				  g[4 * a + 2] * o[2] + g[4 * a + 3];
				od[a] = g[4 * a] * d[0] + g[4 * a + 1] * d[1] +
				  g[4 * a + 2] * d[2];
			}
			for (uint32_t p = 0; p < ri->tricnt; p++) {
				const struct nb_rtri *t = &rd->tris[ri->triofs + p];
				double v0[3] = {t->v0.x, t->v0.y, t->v0.z};
				double e0[3] = {t->v1.x - v0[0], t->v1.y - v0[1],
				  t->v1.z - v0[2]};
				double e1[3] = {t->v2.x - v0[0], t->v2.y - v0[1],
				  t->v2.z - v0[2]};
				double pv[3] = {od[1] * e1[2] - od[2] * e1[1],
				  od[2] * e1[0] - od[0] * e1[2],
				  od[0] * e1[1] - od[1] * e1[0]};
				double det = e0[0] * pv[0] + e0[1] * pv[1] +
				  e0[2] * pv[2];
				if (det == 0.0)
					continue;
				double tv[3] = {oo[0] - v0[0], oo[1] - v0[1],
				  oo[2] - v0[2]};
				double u = (tv[0] * pv[0] + tv[1] * pv[1] +
				  tv[2] * pv[2]) / det;
				if (u < 0.0 || u > 1.0)
					continue;
				double qv[3] = {tv[1] * e0[2] - tv[2] * e0[1],
				  tv[2] * e0[0] - tv[0] * e0[2],
				  tv[0] * e0[1] - tv[1] * e0[0]};
				double v = (od[0] * qv[0] + od[1] * qv[1] +
				  od[2] * qv[2]) / det;
				if (v < 0.0 || u + v > 1.0)
					continue;
				double tt = (e1[0] * qv[0] + e1[1] * qv[1] +
				  e1[2] * qv[2]) / det;
				if (tt > 0.0 && tt < best) {
					best = tt;
					bid = (p << INST_BITS) | k;
				}
			}
		}
		ids[i] = bid;
		tout[i] = best;
	}
}

// ------------------------------------------------- batches -----------------

struct tbatch {
	const struct nb_rdata *rd;
	const float *rays;
	struct orc_hit *hits;
	uint8_t *occl;
	uint32_t n;
	int next;
	pthread_mutex_t mu;
	struct orc_counts *counts;
};

static void *tbatch_run(void *arg)
{
	struct tbatch *b = arg;
	struct tcount tc = {0, 0, 0};
	uint64_t rays = 0;
	for (;;) {
		int c = __atomic_fetch_add(&b->next, 1, __ATOMIC_SEQ_CST);
		uint32_t s = (uint32_t)c * 256u;
		if (s >= b->n)
			break;
		uint32_t e = s + 256u < b->n ? s + 256u : b->n;
		for (uint32_t i = s; i < e; i++) {
			const float *r = b->rays + 8ull * i;
			if (b->occl) {
				b->occl[i] = (uint8_t)orc_intersect_any_tlas(
				  r[3], r[0], r[1], r[2], r[4], r[5], r[6],
				  b->rd->bnodes, b->rd->insts, b->rd->tlasofs);
				continue;
			}
			struct orc_hit h = {r[3], 0.0f, 0.0f, 0u};
			tlas_closest(&h.t, &h.u, &h.v, &h.id, r[0], r[1], r[2],
			  r[4], r[5], r[6], b->rd->bnodes, b->rd->insts,
			  b->rd->tlasofs, b->counts ? &tc : NULL);
			b->hits[i] = h;
			rays++;
		}
	}
	if (b->counts) {
		pthread_mutex_lock(&b->mu);
		b->counts->nodes += tc.nodes;
		b->counts->leaves += tc.leaves;
		b->counts->insts += tc.insts;
		b->counts->rays += rays;
		pthread_mutex_unlock(&b->mu);
	}
	return NULL;
}

static void run_threads(void *(*fn)(void *), void *arg, int nthreads)
{
	if (nthreads < 1)
		nthreads = 1;
	pthread_t *th = malloc(sizeof(*th) * (size_t)nthreads);
	for (int i = 0; i < nthreads; i++)
		pthread_create(&th[i], NULL, fn, arg);
	for (int i = 0; i < nthreads; i++)
		pthread_join(th[i], NULL);
	free(th);
}

void orc_trace(const struct nb_rdata *rd, const float *rays, uint32_t n,
               struct orc_hit *hits, struct orc_counts *counts, int nthreads)
{
	struct tbatch b = {rd, rays, hits, NULL, n, 0,
	  PTHREAD_MUTEX_INITIALIZER, counts};
	run_threads(tbatch_run, &b, nthreads);
}

void orc_occluded(const struct nb_rdata *rd, const float *rays, uint32_t n,
                  uint8_t *occl, int nthreads)
{
	struct tbatch b = {rd, rays, NULL, occl, n, 0,
	  PTHREAD_MUTEX_INITIALIZER, NULL};
	run_threads(tbatch_run, &b, nthreads);
}

// ------------------------------------------------- sampling ----------------

struct pcg { uint64_t state, inc; };

static inline uint32_t pcg_next(struct pcg *r)
{
	uint64_t old = r->state;
	r->state = old * 6364136223846793005ull + r->inc;
	uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

// Path stream: state from (seed, frame), sequence = path id.
static inline void pcg_path(struct pcg *r, uint64_t seed, uint32_t frame,
                            uint64_t path)
{
	r->state = 0;
	r->inc = (path << 1u) | 1u;
	pcg_next(r);
	r->state += seed + 0x9e3779b97f4a7c15ull * ((uint64_t)frame + 1u);
	pcg_next(r);
}

static inline float rnd01(struct pcg *r)
{
	return (float)(pcg_next(r) >> 8) * 0x1p-24f;
}

uint32_t orc_pcg_first(uint64_t seed, uint32_t frame, uint64_t path,
                       uint32_t count, uint32_t *out)
{
	struct pcg r;
	pcg_path(&r, seed, frame, path);
	for (uint32_t i = 0; i < count; i++)
		out[i] = pcg_next(&r);
	return count;
}

// sin and cos of 2*pi*u for u in [0,1): quadrant by 4u, then Taylor
// polynomials of sin/cos(pi/2 * f) for f in [0,1) (terms to f^11 / f^12).
void orc_sincos2pi(float u, float *s, float *c)
{
	float u4 = u * 4.0f;
	int q = (int)u4;
	float f = u4 - (float)q;
	float f2 = f * f;
	float sp = f * (1.57079633f + f2 * (-0.645964098f + f2 * (0.0796926262f +
	  f2 * (-0.00468175414f + f2 * (0.000160441185f +
	  f2 * -3.59884324e-06f)))));
	float cp = 1.0f + f2 * (-1.23370055f + f2 * (0.253669508f + f2 *
	  (-0.0208634808f + f2 * (0.000919260275f + f2 * (-2.52020424e-05f +
	  f2 * 4.71087478e-07f)))));
	switch (q & 3) {
	case 0: *s = sp; *c = cp; break;
	case 1: *s = cp; *c = -sp; break;
	case 2: *s = -sp; *c = -cp; break;
	default: *s = -cp; *c = sp; break;
	}
}

struct v3 { float x, y, z; };

static inline struct v3 v3(float x, float y, float z)
{
	return (struct v3){x, y, z};
}
static inline struct v3 vadd(struct v3 a, struct v3 b)
{
	return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
static inline struct v3 vsub(struct v3 a, struct v3 b)
{
	return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
static inline struct v3 vmul(struct v3 a, struct v3 b)
{
	return v3(a.x * b.x, a.y * b.y, a.z * b.z);
}
static inline struct v3 vscale(struct v3 a, float s)
{
	return v3(a.x * s, a.y * s, a.z * s);
}
static inline float vdot(struct v3 a, struct v3 b)
{
	return a.x * b.x + a.y * b.y + a.z * b.z;
}
static inline struct v3 vfma(struct v3 a, float s, struct v3 b) // a*s + b
{
	return v3(fmaf(a.x, s, b.x), fmaf(a.y, s, b.y), fmaf(a.z, s, b.z));
}
static inline struct v3 vunit(struct v3 a) // vec3_unit, vec3.c:49
{
	float il = 1.0f / sqrtf(vdot(a, a));
	return vscale(a, il);
}

// Camera ray of pixel (x, y) (rend.c:3293-3402, one lane).
static void camera_ray(const struct nb_rcam *c, uint32_t x, uint32_t y,
                       struct pcg *r, struct v3 *o, struct v3 *d)
{
	float u0 = rnd01(r), u1 = rnd01(r);
	float sx = (float)x + (u0 - 0.5f);
	float sy = (float)y + (u1 - 0.5f);
	sx = fmaf(sx, c->rw8[0], -0.5f);
	sy = fmaf(sy, c->rh8[0], -0.5f);
	sx = sx * c->fovfdist8[0];
	sy = sy * c->fovfdist8[0];
	sx = sx * c->aspect8[0];
	struct v3 eye = v3(c->eye.x, c->eye.y, c->eye.z);
	struct v3 ri = v3(c->ri.x, c->ri.y, c->ri.z);
	struct v3 up = v3(c->up.x, c->up.y, c->up.z);
	struct v3 fw = v3(c->fwd.x, c->fwd.y, c->fwd.z);
	struct v3 ups = vscale(up, sy);
	struct v3 riup = v3(fmaf(ri.x, sx, -ups.x), fmaf(ri.y, sx, -ups.y),
	  fmaf(ri.z, sx, -ups.z));
	struct v3 td;
	if (c->tanfangle > 0.0f) {
		float u2 = rnd01(r), u3 = rnd01(r);
		float rad = sqrtf(u2), sn, cs;
		orc_sincos2pi(u3, &sn, &cs);
		float lx = cs * rad, ly = sn * rad;
		float fr = c->focrad8[0];
		*o = v3(fmaf(fmaf(ri.x, lx, up.x * ly), fr, eye.x),
		  fmaf(fmaf(ri.y, lx, up.y * ly), fr, eye.y),
		  fmaf(fmaf(ri.z, lx, up.z * ly), fr, eye.z));
		struct v3 fe = vfma(fw, c->fdist8[0], eye);
		td = vsub(vadd(fe, riup), *o);
	} else {
		*o = eye;
		td = vfma(fw, c->fdist8[0], riup);
	}
	float l2 = fmaf(td.x, td.x, fmaf(td.y, td.y, td.z * td.z));
	float il = 1.0f / sqrtf(l2);
	*d = vscale(td, il);
}

// Interpolated normal through the inverse transpose (rend.c:3109-3116 with
// the transpose of rend.c:3181-3184).
static struct v3 shading_normal(const struct nb_rnrm *rn, const float *g,
                                float u, float v)
{
	float w = (1.0f - u) - v;
	struct v3 n = vadd(vscale(v3(rn->n1.x, rn->n1.y, rn->n1.z), u),
	  vadd(vscale(v3(rn->n2.x, rn->n2.y, rn->n2.z), v),
	  vscale(v3(rn->n0.x, rn->n0.y, rn->n0.z), w)));
	struct v3 m = v3(g[0] * n.x + g[4] * n.y + g[8] * n.z,
	  g[1] * n.x + g[5] * n.y + g[9] * n.z,
	  g[2] * n.x + g[6] * n.y + g[10] * n.z);
	return vunit(m);
}

// Orthonormal basis around n (rend.c:3126-3133).
static void onb(struct v3 n, struct v3 *b1, struct v3 *b2)
{
	float sgn = copysignf(1.0f, n.z);
	float a = -1.0f / (sgn + n.z);
	float b = n.x * n.y * a;
	*b1 = v3(1.0f + sgn * n.x * n.x * a, sgn * b, -sgn * n.x);
	*b2 = v3(b, sgn + n.y * n.y * a, -n.y);
}

static uint32_t pick_light(const float *lights, uint32_t n, float r)
{
	uint32_t lo = 0, hi = n - 1;
	while (lo < hi) {
		uint32_t mid = (lo + hi) >> 1;
		if (r < lights[ORC_LIGHT_FLOATS * mid + 15])
			hi = mid;
		else
			lo = mid + 1;
	}
	return lo;
}

struct shadow { struct v3 o, d, c; float tfar; int live; };

// GGX (Trowbridge-Reitz) microfacet conductor with alpha = roughness
// (Walter, Marschner, Li, Torrance 2007): Smith's separable masking term
// for GGX, G1(v) = 2 n.v / (n.v + sqrt(a^2 + (1 - a^2) (n.v)^2)), and
// Schlick's Fresnel with F0 = the albedo.  The reference carries metallic
// and roughness in rmtl (rend.h:54-61) but never shades with them.
static float ggx_g1(float a2, float nv)
{
	return (2.0f * nv) / (nv + sqrtf(a2 + (1.0f - a2) * (nv * nv)));
}

static struct v3 schlick(struct v3 f0, float c)
{
	float m = 1.0f - c;
	float m2 = m * m;
	float m5 = (m2 * m2) * m;
	return v3(f0.x + (1.0f - f0.x) * m5, f0.y + (1.0f - f0.y) * m5,
	  f0.z + (1.0f - f0.z) * m5);
}

// Radiance of one path (the GPU wavefront kernels follow the same steps,
// bounce by bounce).
static struct v3 path_radiance(const struct nb_rdata *rd,
                               const struct orc_pt_cfg *cfg, struct pcg *r,
                               uint32_t x, uint32_t y, uint64_t *rays,
                               struct tcount *tc)
{
	orc_closest_fn closest = cfg->closest ? cfg->closest : orc_intersect_tlas;
	orc_any_fn any = cfg->any ? cfg->any : orc_intersect_any_tlas;
	struct v3 o, d, L = v3(0, 0, 0), T = v3(1, 1, 1);
	camera_ray(&rd->cam, x, y, r, &o, &d);
	int spec = 0;
	struct v3 bg = v3(rd->bgcol.x, rd->bgcol.y, rd->bgcol.z);
	for (uint32_t k = 0; k < cfg->depth; k++) {
		struct orc_hit h = {FLT_MAX, 0.0f, 0.0f, 0u};
		if (tc && !cfg->closest)
			tlas_closest(&h.t, &h.u, &h.v, &h.id, o.x, o.y, o.z, d.x,
			  d.y, d.z, rd->bnodes, rd->insts, rd->tlasofs, tc);
		else
			closest(&h.t, &h.u, &h.v, &h.id, o.x, o.y, o.z, d.x,
			  d.y, d.z, rd->bnodes, rd->insts, rd->tlasofs);
		(*rays)++;
		if (h.t == FLT_MAX) {
			L = vadd(L, vmul(T, bg));
			break;
		}
		float of[3] = {o.x, o.y, o.z}, dfv[3] = {d.x, d.y, d.z};
		refine_hit(rd, of, dfv, &h);
		uint32_t inst = h.id & INST_MASK, prim = h.id >> INST_BITS;
		const struct nb_rinst *ri = &rd->insts[inst];
		const struct nb_rnrm *rn = &rd->nrms[ri->triofs + prim];
		const struct nb_rmtl *mt = &rd->mtls[rn->mtlid];
		struct v3 col = v3(mt->col.x, mt->col.y, mt->col.z);
		struct v3 n = shading_normal(rn, ri->globinv, h.u, h.v);
		if (cfg->mode == ORC_MODE_PRIMARY) {
			// rend.c:3435-3441: (n + 1) / 2 * albedo
			struct v3 c = vscale(vadd(n, v3(1, 1, 1)), 0.5f);
			L = vmul(c, col);
			break;
		}
		struct v3 pos = vfma(d, h.t, o);
		int front = vdot(n, d) < 0.0f;
		if (!front)
			n = vscale(n, -1.0f);
		float rl = rnd01(r), ra = rnd01(r), rb = rnd01(r);
		float r0 = rnd01(r), r1 = rnd01(r);
		if (mt->flags & NB_FLAG_EMISSIVE) {
			if ((k == 0 || spec) && front)
				L = vadd(L, vmul(T, col));
			break;
		}
		int glossy = mt->metallic >= 0.5f && mt->roughness > 0.0f;
		if (mt->metallic >= 0.5f && !glossy) { // perfect mirror
			float dn = vdot(d, n);
			d = vsub(d, vscale(n, 2.0f * dn));
			T = vmul(T, col);
			o = vfma(d, EPS2F, pos);
			spec = 1;
			continue;
		}
		spec = 0;
		struct v3 wo = vscale(d, -1.0f);
		float nwo = vdot(n, wo);
		float a2 = mt->roughness * mt->roughness;
		if (glossy && !(nwo > 0.0f))
			break;
		// next-event estimation to one point on the emitters
		// (rend.c:3243-3267)
		if (cfg->nlights) {
			const float *lt = cfg->lights + ORC_LIGHT_FLOATS *
			  pick_light(cfg->lights, cfg->nlights, rl);
			float su = sqrtf(ra);
			float b1 = su * (1.0f - rb), b2 = su * rb;
			struct v3 lp = vadd(vadd(v3(lt[0], lt[1], lt[2]),
			  vscale(v3(lt[3], lt[4], lt[5]), b1)),
			  vscale(v3(lt[6], lt[7], lt[8]), b2));
			struct v3 ld = vsub(lp, pos);
			float l2 = vdot(ld, ld);
			float ldist = sqrtf(l2);
			ld = vscale(ld, 1.0f / ldist);
			float ndotl = vdot(n, ld);
			float cosl = -vdot(v3(lt[9], lt[10], lt[11]), ld);
			float tfar = ldist - 2.0f * EPS2F;
			if (ndotl > 0.0f && cosl > 0.0f && tfar > 0.0f) {
				struct v3 c;
				if (glossy) {
					// f = F D G / (4 n.wo n.l); times n.l cosl
					// area / l^2
					struct v3 h = vunit(vadd(wo, ld));
					float nh = vdot(n, h), lh = vdot(ld, h);
					float dd = (nh * nh) * (a2 - 1.0f) + 1.0f;
					float D = (a2 * INV_PI_F) / (dd * dd);
					float G = ggx_g1(a2, nwo) * ggx_g1(a2, ndotl);
					float wgt = ((D * G) / (4.0f * nwo)) * cosl;
					wgt = wgt * cfg->light_area;
					wgt = wgt / l2;
					c = vscale(vmul(vmul(T, schlick(col, lh)),
					  v3(lt[12], lt[13], lt[14])), wgt);
				} else {
					float wgt = ndotl * cosl;
					wgt = wgt * (INV_PI_F * cfg->light_area);
					wgt = wgt / l2;
					c = vscale(vmul(vmul(T, col),
					  v3(lt[12], lt[13], lt[14])), wgt);
				}
				struct v3 so = vfma(ld, EPS2F, pos);
				(*rays)++;
				if (!any(tfar, so.x, so.y, so.z, ld.x, ld.y,
				  ld.z, rd->bnodes, rd->insts, rd->tlasofs))
					L = vadd(L, c);
			}
		}
		if (k + 1 >= cfg->depth)
			break;
		if (glossy) {
			// microfacet normal from D(m) (m.n): cos^2 = (1 - r1) /
			// (1 + (a^2 - 1) r1); reflect wo; weight F G1(wo) G1(wi)
			// (wo.m) / ((n.wo) (n.m))
			float ct2 = (1.0f - r1) / (1.0f + (a2 - 1.0f) * r1);
			float ct = sqrtf(ct2);
			float s2 = 1.0f - ct2;
			float st = sqrtf(s2 > 0.0f ? s2 : 0.0f);
			float sn, cs;
			orc_sincos2pi(r0, &sn, &cs);
			struct v3 ta, bta;
			onb(n, &ta, &bta);
			struct v3 m = vadd(vadd(vscale(ta, st * cs),
			  vscale(bta, st * sn)), vscale(n, ct));
			float wom = vdot(wo, m);
			struct v3 wi = vsub(vscale(m, 2.0f * wom), wo);
			float nwi = vdot(n, wi);
			if (!(wom > 0.0f) || !(nwi > 0.0f))
				break;
			float w = ((ggx_g1(a2, nwo) * ggx_g1(a2, nwi)) * wom) /
			  (nwo * ct);
			T = vscale(vmul(T, schlick(col, wom)), w);
			d = wi;
			o = vfma(d, EPS2F, pos);
			continue;
		}
		// cosine-weighted bounce (rend.c:3135-3140, 3270-3288)
		float sn, cs;
		orc_sincos2pi(r0, &sn, &cs);
		float s1 = sqrtf(r1);
		struct v3 loc = v3(cs * s1, sn * s1, sqrtf(1.0f - r1));
		struct v3 ta, bta;
		onb(n, &ta, &bta);
		d = vadd(vadd(vscale(ta, loc.x), vscale(bta, loc.y)),
		  vscale(n, loc.z));
		T = vmul(T, col);
		o = vfma(d, EPS2F, pos);
	}
	return L;
}

int orc_ggx_sample(const float nn[3], const float wwo[3], float alpha,
                   const float f0[3], float r0, float r1, float wi[3],
                   float w[3])
{
	struct v3 n = v3(nn[0], nn[1], nn[2]), wo = v3(wwo[0], wwo[1], wwo[2]);
	float a2 = alpha * alpha, nwo = vdot(n, wo);
	float ct2 = (1.0f - r1) / (1.0f + (a2 - 1.0f) * r1);
	float ct = sqrtf(ct2);
	float s2 = 1.0f - ct2;
	float st = sqrtf(s2 > 0.0f ? s2 : 0.0f);
	float sn, cs;
	orc_sincos2pi(r0, &sn, &cs);
	struct v3 ta, bta;
	onb(n, &ta, &bta);
	struct v3 m = vadd(vadd(vscale(ta, st * cs), vscale(bta, st * sn)),
	  vscale(n, ct));
	float wom = vdot(wo, m);
	struct v3 d = vsub(vscale(m, 2.0f * wom), wo);
	float nwi = vdot(n, d);
	wi[0] = d.x;
	wi[1] = d.y;
	wi[2] = d.z;
	if (!(wom > 0.0f) || !(nwi > 0.0f) || !(nwo > 0.0f))
		return 0;
	float g = ((ggx_g1(a2, nwo) * ggx_g1(a2, nwi)) * wom) / (nwo * ct);
	struct v3 F = schlick(v3(f0[0], f0[1], f0[2]), wom);
	w[0] = F.x * g;
	w[1] = F.y * g;
	w[2] = F.z * g;
	return 1;
}

void orc_ggx_eval(const float nn[3], const float wwo[3], const float wwi[3],
                  float alpha, const float f0[3], float f[3])
{
	struct v3 n = v3(nn[0], nn[1], nn[2]), wo = v3(wwo[0], wwo[1], wwo[2]);
	struct v3 ld = v3(wwi[0], wwi[1], wwi[2]);
	float a2 = alpha * alpha, nwo = vdot(n, wo), ndotl = vdot(n, ld);
	struct v3 h = vunit(vadd(wo, ld));
	float nh = vdot(n, h), lh = vdot(ld, h);
	float dd = (nh * nh) * (a2 - 1.0f) + 1.0f;
	float D = (a2 * INV_PI_F) / (dd * dd);
	float G = ggx_g1(a2, nwo) * ggx_g1(a2, ndotl);
	float k = (D * G) / ((4.0f * nwo) * ndotl);
	struct v3 F = schlick(v3(f0[0], f0[1], f0[2]), lh);
	f[0] = F.x * k;
	f[1] = F.y * k;
	f[2] = F.z * k;
}

struct rbatch {
	const struct nb_rdata *rd;
	const struct orc_pt_cfg *cfg;
	float *rad;
	int next;
	uint32_t tw, th, ntiles;
	uint64_t rays;
	pthread_mutex_t mu;
};

#define TILE_W 16
#define TILE_H 8

static void *render_run(void *arg)
{
	struct rbatch *b = arg;
	const struct nb_rdata *rd = b->rd;
	const struct orc_pt_cfg *cfg = b->cfg;
	uint64_t rays = 0;
	struct tcount tc = {0, 0, 0};
	struct tcount *tcp = cfg->counts ? &tc : NULL;
	uint32_t W = rd->width, spp = rd->spp ? rd->spp : 1;
	for (;;) {
		int tix = __atomic_fetch_add(&b->next, 1, __ATOMIC_SEQ_CST);
		if ((uint32_t)tix >= b->ntiles)
			break;
		uint32_t bx = cfg->x0 + ((uint32_t)tix % b->tw) * TILE_W;
		uint32_t by = cfg->y0 + ((uint32_t)tix / b->tw) * TILE_H;
		for (uint32_t y = by; y < by + TILE_H && y < cfg->y1; y++)
			for (uint32_t x = bx; x < bx + TILE_W && x < cfg->x1;
			  x++) {
				struct v3 sum = v3(0, 0, 0);
				for (uint32_t s = 0; s < spp; s++) {
					struct pcg r;
					uint64_t pid = ((uint64_t)y * W + x) *
					  spp + s;
					pcg_path(&r, cfg->seed, rd->samples, pid);
					sum = vadd(sum, path_radiance(rd, cfg,
					  &r, x, y, &rays, tcp));
				}
				float *o = b->rad + 3ull * ((uint64_t)y * W + x);
				o[0] = sum.x;
				o[1] = sum.y;
				o[2] = sum.z;
			}
	}
	__atomic_fetch_add(&b->rays, rays, __ATOMIC_SEQ_CST);
	if (tcp) {
		pthread_mutex_lock(&b->mu);
		cfg->counts->nodes += tc.nodes;
		cfg->counts->leaves += tc.leaves;
		cfg->counts->insts += tc.insts;
		pthread_mutex_unlock(&b->mu);
	}
	return NULL;
}

uint64_t orc_render(const struct nb_rdata *rd, const struct orc_pt_cfg *cfg,
                    float *rad)
{
	struct rbatch b;
	memset(&b, 0, sizeof(b));
	b.rd = rd;
	b.cfg = cfg;
	b.rad = rad;
	pthread_mutex_init(&b.mu, NULL);
	uint32_t w = cfg->x1 > cfg->x0 ? cfg->x1 - cfg->x0 : 0;
	uint32_t h = cfg->y1 > cfg->y0 ? cfg->y1 - cfg->y0 : 0;
	b.tw = (w + TILE_W - 1) / TILE_W;
	b.th = (h + TILE_H - 1) / TILE_H;
	b.ntiles = b.tw * b.th;
	run_threads(render_run, &b, cfg->nthreads);
	return b.rays;
}

void orc_accumulate(struct nb_rdata *rd, const float *rad)
{
	uint32_t n = rd->width * rd->height;
	float inv = 1.0f / (float)(rd->samples + rd->spp);
	for (uint32_t i = 0; i < n; i++) {
		struct nb_vec3 *a = &rd->acc[i];
		a->x = a->x + rad[3 * i];
		a->y = a->y + rad[3 * i + 1];
		a->z = a->z + rad[3 * i + 2];
		if (rd->buf) {
			float cx = a->x * inv, cy = a->y * inv, cz = a->z * inv;
			rd->buf[i] = 0xffu << 24 |
			  ((unsigned int)(255.0f * cx) & 0xffu) << 16 |
			  ((unsigned int)(255.0f * cy) & 0xffu) << 8 |
			  ((unsigned int)(255.0f * cz) & 0xffu);
		}
	}
}
