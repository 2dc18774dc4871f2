// Device side of the two-level BVH traversal (sm_100a).
//
// One ray per thread.  A node visit loads the 80-byte quantised node with
// five 16-byte read-only loads and tests its 8 child boxes; hit inner children
// form a "node group" (first child index, 8-bit hit mask keyed by
// slot ^ octant, inner mask) and hit leaf items a "triangle group" (first item,
// 32-bit mask).  Only node groups with remaining siblings, and at a BLAS
// entry the remaining instance group of the TLAS node, go on the stack, so a
// ray needs at most depth(TLAS) + depth(BLAS) entries; the stack lives in
// shared memory, one column per thread.  Triangles use the watertight test of
// Woop, Benthin and Wald (JCGT 2013) with Kahan's difference of products for
// the edge functions, which gives their exact sign without double precision.
//
// Closest-hit semantics follow intersect_tlas (rend.c:1976): hits with
// 0 < t < tmax, edges inclusive, the ray transformed into object space per
// instance without renormalisation (t stays in world units).

#ifndef NB_TRACE_CUH
#define NB_TRACE_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "gpulayout.h"
#include "host/nb_rdata.h"

namespace nb {

constexpr uint32_t kIGroup = 0x100u;          // stack entry holds instances
constexpr float kWiden = 1.00000095367431640625f; // 1 + 2^-20

struct DScene {
	const nb_qnode *blas;
	const float4   *tris;   // nb_gtri as 3 float4
	const nb_qnode *tlas;
	const uint32_t *irefs;
	const float4   *insts;  // nb_ginst as 4 float4
	const nb_rnrm  *nrms;
	const nb_rmtl  *mtls;
	const float4   *lights; // nb_glight as 5 float4
	uint32_t        nlights;
	float           light_area;
	float           bg[3];
};

// Ray state in the space being traversed.
struct TRay {
	float ox, oy, oz, dx, dy, dz;
	float ix, iy, iz;
	uint32_t oct;
	uint32_t kx, ky, kz;
	float sx, sy, sz;
};

__device__ __forceinline__ float sel3(float x, float y, float z, uint32_t k)
{
	return k == 0 ? x : (k == 1 ? y : z);
}

__device__ __forceinline__ void tray_slab(TRay &r, float ox, float oy,
                                          float oz, float dx, float dy,
                                          float dz)
{
	r.ox = ox;
	r.oy = oy;
	r.oz = oz;
	r.dx = dx;
	r.dy = dy;
	r.dz = dz;
	r.ix = 1.0f / dx;
	r.iy = 1.0f / dy;
	r.iz = 1.0f / dz;
	r.oct = (signbit(r.ix) ? 1u : 0u) | (signbit(r.iy) ? 2u : 0u) |
	  (signbit(r.iz) ? 4u : 0u);
}

__device__ __forceinline__ void tray_watertight(TRay &r)
{
	float ax = fabsf(r.dx), ay = fabsf(r.dy), az = fabsf(r.dz);
	uint32_t kz = ax >= ay ? (ax >= az ? 0u : 2u) : (ay >= az ? 1u : 2u);
	uint32_t kx = kz == 2u ? 0u : kz + 1u;
	uint32_t ky = kx == 2u ? 0u : kx + 1u;
	float dkz = sel3(r.dx, r.dy, r.dz, kz);
	if (dkz < 0.0f) {
		uint32_t t = kx;
		kx = ky;
		ky = t;
	}
	r.kx = kx;
	r.ky = ky;
	r.kz = kz;
	r.sx = sel3(r.dx, r.dy, r.dz, kx) / dkz;
	r.sy = sel3(r.dx, r.dy, r.dz, ky) / dkz;
	r.sz = 1.0f / dkz;
}

__device__ __forceinline__ uint32_t qb(uint32_t w, int k)
{
	return (w >> (8 * k)) & 0xffu;
}

// Test the 8 children of node `ni`; returns the node and triangle groups.
__device__ __forceinline__ void visit(const nb_qnode *__restrict__ nodes,
                                      uint32_t ni, const TRay &r, float tmax,
                                      uint2 &ng, uint2 &tg)
{
	const uint4 *p = reinterpret_cast<const uint4 *>(nodes + ni);
	uint4 w0 = __ldg(p);
	uint4 w1 = __ldg(p + 1);
	uint4 w2 = __ldg(p + 2);
	uint4 w3 = __ldg(p + 3);
	uint4 w4 = __ldg(p + 4);
	uint32_t imask = w0.w >> 24;
	float scx = __uint_as_float((w0.w & 0xffu) << 23) * r.ix;
	float scy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23) * r.iy;
	float scz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23) * r.iz;
	float bx = (__uint_as_float(w0.x) - r.ox) * r.ix;
	float by = (__uint_as_float(w0.y) - r.oy) * r.iy;
	float bz = (__uint_as_float(w0.z) - r.oz) * r.iz;
	bool fx = signbit(r.ix), fy = signbit(r.iy), fz = signbit(r.iz);
	// lo/hi words: x lo = w2.x,w2.y  y lo = w2.z,w2.w  z lo = w3.x,w3.y
	//              x hi = w3.z,w3.w  y hi = w4.x,w4.y  z hi = w4.z,w4.w
	uint32_t nx0 = fx ? w3.z : w2.x, nx1 = fx ? w3.w : w2.y;
	uint32_t fx0 = fx ? w2.x : w3.z, fx1 = fx ? w2.y : w3.w;
	uint32_t ny0 = fy ? w4.x : w2.z, ny1 = fy ? w4.y : w2.w;
	uint32_t fy0 = fy ? w2.z : w4.x, fy1 = fy ? w2.w : w4.y;
	uint32_t nz0 = fz ? w4.z : w3.x, nz1 = fz ? w4.w : w3.y;
	uint32_t fz0 = fz ? w3.x : w4.z, fz1 = fz ? w3.y : w4.w;
	float tcap = tmax * kWiden;
	uint32_t hits = 0, tbits = 0;
#pragma unroll
	for (int s = 0; s < 8; s++) {
		int b = s & 3;
		uint32_t wnx = s < 4 ? nx0 : nx1, wfx = s < 4 ? fx0 : fx1;
		uint32_t wny = s < 4 ? ny0 : ny1, wfy = s < 4 ? fy0 : fy1;
		uint32_t wnz = s < 4 ? nz0 : nz1, wfz = s < 4 ? fz0 : fz1;
		float tnx = __fmaf_rn((float)qb(wnx, b), scx, bx);
		float tny = __fmaf_rn((float)qb(wny, b), scy, by);
		float tnz = __fmaf_rn((float)qb(wnz, b), scz, bz);
		float tfx = __fmaf_rn((float)qb(wfx, b), scx, bx);
		float tfy = __fmaf_rn((float)qb(wfy, b), scy, by);
		float tfz = __fmaf_rn((float)qb(wfz, b), scz, bz);
		float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
		float tf = fminf(fminf(tfx, tfy), tfz) * kWiden;
		if (tn <= fminf(tf, tcap)) {
			if ((imask >> s) & 1u) {
				hits |= 1u << (s ^ r.oct);
			} else {
				uint32_t m = qb(s < 4 ? w1.z : w1.w, b);
				if (m & NB_META_LEAF) {
					uint32_t cnt = ((m >> 5) & 3u) + 1u;
					tbits |= ((1u << cnt) - 1u) << (m & 31u);
				}
			}
		}
	}
	ng = make_uint2(w1.x, (hits << 24) | imask);
	tg = make_uint2(w1.y, tbits);
}

// a*b - c*d with Kahan's error compensation (relative error <= 2 ulp, so
// the sign is exact).
__device__ __forceinline__ float dop(float a, float b, float c, float d)
{
	float cd = c * d;
	float err = __fmaf_rn(-c, d, cd);
	float r = __fmaf_rn(a, b, -cd);
	return r + err;
}

// Watertight ray/triangle test of triangle `idx`; t in (0, tbest).
__device__ __forceinline__ bool tri_hit(const float4 *__restrict__ tris,
                                        uint32_t idx, const TRay &r,
                                        float tbest, float *tout)
{
	float4 a = __ldg(tris + 3u * idx);
	float4 b = __ldg(tris + 3u * idx + 1u);
	float4 c = __ldg(tris + 3u * idx + 2u);
	float ax = a.x - r.ox, ay = a.y - r.oy, az = a.z - r.oz;
	float bx = b.x - r.ox, by = b.y - r.oy, bz = b.z - r.oz;
	float cx = c.x - r.ox, cy = c.y - r.oy, cz = c.z - r.oz;
	float akz = sel3(ax, ay, az, r.kz), bkz = sel3(bx, by, bz, r.kz);
	float ckz = sel3(cx, cy, cz, r.kz);
	float Ax = __fmaf_rn(-r.sx, akz, sel3(ax, ay, az, r.kx));
	float Ay = __fmaf_rn(-r.sy, akz, sel3(ax, ay, az, r.ky));
	float Bx = __fmaf_rn(-r.sx, bkz, sel3(bx, by, bz, r.kx));
	float By = __fmaf_rn(-r.sy, bkz, sel3(bx, by, bz, r.ky));
	float Cx = __fmaf_rn(-r.sx, ckz, sel3(cx, cy, cz, r.kx));
	float Cy = __fmaf_rn(-r.sy, ckz, sel3(cx, cy, cz, r.ky));
	float U = dop(Cx, By, Cy, Bx);
	float V = dop(Ax, Cy, Ay, Cx);
	float W = dop(Bx, Ay, By, Ax);
	if ((U < 0.0f || V < 0.0f || W < 0.0f) &&
	    (U > 0.0f || V > 0.0f || W > 0.0f))
		return false;
	float det = U + V + W;
	if (det == 0.0f)
		return false;
	float T = __fmaf_rn(U, r.sz * akz, __fmaf_rn(V, r.sz * bkz,
	  W * (r.sz * ckz)));
	if (det < 0.0f) {
		T = -T;
		det = -det;
	}
	if (!(T > 0.0f) || T >= tbest * det)
		return false;
	float t = T / det;
	if (!(t < tbest))
		return false;
	*tout = t;
	return true;
}

// World -> object with the instance 3x4; the oracle uses the same sequence.
__device__ __forceinline__ void xform(const float4 &m0, const float4 &m1,
                                      const float4 &m2, float x, float y,
                                      float z, float dx, float dy, float dz,
                                      float *o, float *d)
{
	o[0] = __fmaf_rn(m0.x, x, __fmaf_rn(m0.y, y, __fmaf_rn(m0.z, z, m0.w)));
	o[1] = __fmaf_rn(m1.x, x, __fmaf_rn(m1.y, y, __fmaf_rn(m1.z, z, m1.w)));
	o[2] = __fmaf_rn(m2.x, x, __fmaf_rn(m2.y, y, __fmaf_rn(m2.z, z, m2.w)));
	d[0] = __fmaf_rn(m0.x, dx, __fmaf_rn(m0.y, dy, __fmul_rn(m0.z, dz)));
	d[1] = __fmaf_rn(m1.x, dx, __fmaf_rn(m1.y, dy, __fmul_rn(m1.z, dz)));
	d[2] = __fmaf_rn(m2.x, dx, __fmaf_rn(m2.y, dy, __fmul_rn(m2.z, dz)));
}

struct THit {
	float    t;
	uint32_t tri;  // index into the triangle array
	uint32_t inst;
};

// Traverse the scene.  ANY: stop at the first hit (occlusion).  `stk` is
// this thread's stack column (entry k at stk[k * stride]).  Returns true on
// a hit; sets *err on a stack overflow (the ray is then abandoned).
template <bool ANY, int STACK>
__device__ __forceinline__ bool traverse(const DScene &S, float wox,
                                         float woy, float woz, float wdx,
                                         float wdy, float wdz, float tmax,
                                         uint2 *stk, uint32_t stride,
                                         THit &h, uint32_t &err)
{
	TRay r;
	tray_slab(r, wox, woy, woz, wdx, wdy, wdz);
	uint2 ng, tg;
	visit(S.tlas, 0u, r, tmax, ng, tg);
	int sp = 0, blas_sp = -1;
	uint32_t level = 0, cinst = 0;
	float bt = tmax;
	bool found = false;
	for (;;) {
		while (tg.y) {
			uint32_t i = __ffs(tg.y) - 1;
			tg.y &= tg.y - 1u;
			uint32_t item = tg.x + i;
			if (level == 0u) {
				uint32_t inst = __ldg(S.irefs + item);
				if (ng.y >> 24) {
					if (sp >= STACK) {
						err = 1u;
						return found;
					}
					stk[(uint32_t)sp++ * stride] = ng;
				}
				if (tg.y) {
					if (sp >= STACK) {
						err = 1u;
						return found;
					}
					stk[(uint32_t)sp++ * stride] =
					  make_uint2(tg.x, (tg.y << 24) | kIGroup);
				}
				blas_sp = sp;
				level = 1u;
				cinst = inst;
				const float4 *ip = S.insts + 4u * inst;
				float4 m0 = __ldg(ip), m1 = __ldg(ip + 1);
				float4 m2 = __ldg(ip + 2);
				uint32_t root = __float_as_uint(__ldg(ip + 3).x);
				float o[3], d[3];
				xform(m0, m1, m2, wox, woy, woz, wdx, wdy, wdz, o, d);
				tray_slab(r, o[0], o[1], o[2], d[0], d[1], d[2]);
				tray_watertight(r);
				visit(S.blas, root, r, bt, ng, tg);
				continue;
			}
			float t;
			if (tri_hit(S.tris, item, r, bt, &t)) {
				bt = t;
				h.t = t;
				h.tri = item;
				h.inst = cinst;
				found = true;
				if (ANY)
					return true;
			}
		}
		uint32_t hm = ng.y >> 24;
		if (hm) {
			uint32_t key = __ffs(hm) - 1;
			hm &= hm - 1u;
			uint32_t slot = key ^ r.oct;
			uint32_t child = ng.x + __popc(ng.y & ((1u << slot) - 1u) &
			  0xffu);
			ng.y = (hm << 24) | (ng.y & 0xffu);
			if (hm) {
				if (sp >= STACK) {
					err = 1u;
					return found;
				}
				stk[(uint32_t)sp++ * stride] = ng;
			}
			visit(level ? S.blas : S.tlas, child, r, bt, ng, tg);
			continue;
		}
		if (level == 1u && sp == blas_sp) {
			level = 0u;
			tray_slab(r, wox, woy, woz, wdx, wdy, wdz);
		}
		if (sp == 0)
			return found;
		uint2 e = stk[(uint32_t)(--sp) * stride];
		if (e.y & kIGroup) {
			tg = make_uint2(e.x, e.y >> 24);
			ng = make_uint2(0u, 0u);
		} else {
			ng = e;
			tg.y = 0u;
		}
	}
}

// ---------------------------------------------------------- refinement --

struct df {
	float hi, lo;
};

__device__ __forceinline__ df two_sum(float a, float b)
{
	float s = __fadd_rn(a, b);
	float bb = __fsub_rn(s, a);
	float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
	return {s, e};
}

__device__ __forceinline__ df fast_two_sum(float a, float b)
{
	float s = __fadd_rn(a, b);
	return {s, __fsub_rn(b, __fsub_rn(s, a))};
}

__device__ __forceinline__ df two_prod(float a, float b)
{
	float p = __fmul_rn(a, b);
	return {p, __fmaf_rn(a, b, -p)};
}

__device__ __forceinline__ df df_add(df x, df y)
{
	df s = two_sum(x.hi, y.hi);
	float e = __fadd_rn(s.lo, __fadd_rn(x.lo, y.lo));
	return fast_two_sum(s.hi, e);
}

__device__ __forceinline__ df df_neg(df x)
{
	return {-x.hi, -x.lo};
}

__device__ __forceinline__ df df_mul(df x, df y)
{
	df p = two_prod(x.hi, y.hi);
	float e = __fadd_rn(p.lo, __fadd_rn(__fmul_rn(x.hi, y.lo),
	  __fmul_rn(x.lo, y.hi)));
	return fast_two_sum(p.hi, e);
}

__device__ __forceinline__ df df_div(df x, df y)
{
	float q1 = __fdiv_rn(x.hi, y.hi);
	df r = df_add(x, df_neg(df_mul({q1, 0.0f}, y)));
	float q2 = __fdiv_rn(r.hi, y.hi);
	return fast_two_sum(q1, q2);
}

// t of the plane of (v0, v1, v2) along o + t d in double-float arithmetic;
// u, v by Moeller-Trumbore with an exact division.  Same operation sequence
// as the CPU oracle, so both produce identical bits.
__device__ __forceinline__ void refine(const float *o, const float *d,
                                       const float *v0, const float *v1,
                                       const float *v2, float *t, float *u,
                                       float *v)
{
	df e0[3], e1[3], w[3];
#pragma unroll
	for (int a = 0; a < 3; a++) {
		e0[a] = two_sum(v1[a], -v0[a]);
		e1[a] = two_sum(v2[a], -v0[a]);
		w[a] = two_sum(v0[a], -o[a]);
	}
	df n0 = df_add(df_mul(e0[1], e1[2]), df_neg(df_mul(e0[2], e1[1])));
	df n1 = df_add(df_mul(e0[2], e1[0]), df_neg(df_mul(e0[0], e1[2])));
	df n2 = df_add(df_mul(e0[0], e1[1]), df_neg(df_mul(e0[1], e1[0])));
	df num = df_add(df_add(df_mul(n0, w[0]), df_mul(n1, w[1])),
	  df_mul(n2, w[2]));
	df den = df_add(df_add(df_mul(n0, {d[0], 0.0f}),
	  df_mul(n1, {d[1], 0.0f})), df_mul(n2, {d[2], 0.0f}));
	if (den.hi != 0.0f)
		*t = df_div(num, den).hi;
	float f0[3] = {__fsub_rn(v1[0], v0[0]), __fsub_rn(v1[1], v0[1]),
	  __fsub_rn(v1[2], v0[2])};
	float f1[3] = {__fsub_rn(v2[0], v0[0]), __fsub_rn(v2[1], v0[1]),
	  __fsub_rn(v2[2], v0[2])};
	float pv0 = __fsub_rn(__fmul_rn(d[1], f1[2]), __fmul_rn(d[2], f1[1]));
	float pv1 = __fsub_rn(__fmul_rn(d[2], f1[0]), __fmul_rn(d[0], f1[2]));
	float pv2 = __fsub_rn(__fmul_rn(d[0], f1[1]), __fmul_rn(d[1], f1[0]));
	float det = __fadd_rn(__fadd_rn(__fmul_rn(f0[0], pv0),
	  __fmul_rn(f0[1], pv1)), __fmul_rn(f0[2], pv2));
	float tv0 = __fsub_rn(o[0], v0[0]), tv1 = __fsub_rn(o[1], v0[1]);
	float tv2 = __fsub_rn(o[2], v0[2]);
	float qv0 = __fsub_rn(__fmul_rn(tv1, f0[2]), __fmul_rn(tv2, f0[1]));
	float qv1 = __fsub_rn(__fmul_rn(tv2, f0[0]), __fmul_rn(tv0, f0[2]));
	float qv2 = __fsub_rn(__fmul_rn(tv0, f0[1]), __fmul_rn(tv1, f0[0]));
	float uu = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(tv0, pv0),
	  __fmul_rn(tv1, pv1)), __fmul_rn(tv2, pv2)), det);
	float vv = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(d[0], qv0),
	  __fmul_rn(d[1], qv1)), __fmul_rn(d[2], qv2)), det);
	*u = uu == uu ? uu : 0.0f;
	*v = vv == vv ? vv : 0.0f;
}

// Refined hit record in the reference's form (t, u, v, tri << 12 | inst).
__device__ __forceinline__ float4 finish_hit(const DScene &S, float wox,
                                             float woy, float woz, float wdx,
                                             float wdy, float wdz,
                                             const THit &h)
{
	const float4 *ip = S.insts + 4u * h.inst;
	float o[3], d[3];
	xform(__ldg(ip), __ldg(ip + 1), __ldg(ip + 2), wox, woy, woz, wdx, wdy,
	  wdz, o, d);
	float4 a = __ldg(S.tris + 3u * h.tri);
	float4 b = __ldg(S.tris + 3u * h.tri + 1u);
	float4 c = __ldg(S.tris + 3u * h.tri + 2u);
	float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z};
	float v2[3] = {c.x, c.y, c.z};
	float t = h.t, u, v;
	refine(o, d, v0, v1, v2, &t, &u, &v);
	uint32_t id = (__float_as_uint(a.w) << NB_INST_ID_BITS) | h.inst;
	return make_float4(t, u, v, __uint_as_float(id));
}

} // namespace nb

#endif
