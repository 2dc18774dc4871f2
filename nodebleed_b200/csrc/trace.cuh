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

constexpr float kWiden = 1.00000095367431640625f; // 1 + 2^-20

// Per-scene parameters of a frame (one entry per scene of a batch; a
// single-scene context is a batch of one).  A scene's paths, pixels and
// camera-ray slots are consecutive ranges starting at its bases; its PCG32
// streams and pixel order are those of the scene rendered alone.
struct ScenePar {
	uint32_t tlas_root, light_off, light_cnt, depth;
	uint32_t W, H, spp, frame;             // frame: rd->samples
	uint32_t path_base, pix_base, slot_base, nrc_stride;
	uint32_t nrc_offset, resolve, pad0[2]; // resolve: rendgpu_set_resolve op
	float    light_area, inv, exposure, pad1; // inv: 1 / (samples + spp)
	float    bg[3], tanfangle;
	float    eye[3], rw;
	float    ri[3], rh;
	float    up[3], fovfdist;
	float    fwd[3], aspect;
	float    fdist, focrad, pad2[2];
	uint64_t seed, pad3;
	// radiance cache: position -> [0,1]^3 in this scene's box, plus nrc_off
	// (0 for scene 0, else 2 k: the scene's one-hot feature k, 1..14)
	float    nrc_lo[3], nrc_off;
	float    nrc_inv[3], pad4;
};

struct DScene {
	const nb_qnode *blas;
	const float4   *tris;   // nb_gtri as 3 float4
	const nb_qnode *tlas;
	const uint32_t *irefs;
	const float4   *insts;  // nb_ginst as 4 float4
	const nb_rnrm  *nrms;
	const nb_rmtl  *mtls;
	const float4   *lights; // nb_glight as 5 float4
	const ScenePar *sp;
	uint32_t        nscenes;
};

// Scene owning global index `key` in the range that starts at field
// `base` of each entry: the last scene whose base <= key (bases ascend).
template <class Base>
__device__ __forceinline__ uint32_t scene_search(const DScene &S,
                                                 uint32_t key, Base base)
{
	uint32_t lo = 0, hi = S.nscenes - 1u;
	while (lo < hi) {
		uint32_t mid = (lo + hi + 1u) >> 1;
		if (base(S.sp + mid) <= key)
			lo = mid;
		else
			hi = mid - 1u;
	}
	return lo;
}

__device__ __forceinline__ uint32_t scene_of_path(const DScene &S,
                                                  uint32_t path)
{
	return scene_search(S, path, [](const ScenePar *p) {
		return __ldg(&p->path_base); });
}

// Position of the j-th (from 0) set bit of m (j < popc(m)).
__device__ __forceinline__ uint32_t nth_bit(uint32_t m, uint32_t j)
{
	uint32_t pos = 0, c;
	c = __popc(m & 0xffffu);
	if (j >= c) { j -= c; pos += 16; m >>= 16; }
	c = __popc(m & 0xffu);
	if (j >= c) { j -= c; pos += 8; m >>= 8; }
	c = __popc(m & 0xfu);
	if (j >= c) { j -= c; pos += 4; m >>= 4; }
	c = __popc(m & 0x3u);
	if (j >= c) { j -= c; pos += 2; m >>= 2; }
	c = m & 1u;
	if (j >= c) pos += 1;
	return pos;
}

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

// Hardware reciprocal (relative error below 2^-22; 0 -> inf with the sign
// kept).  Slab distances computed with it carry that relative error on
// every axis alike within 2 ulp, which the far-plane widening 1 + 2^-20
// covers, so no box the ray enters is culled: node pruning only, hits are
// decided by the triangle test.
__device__ __forceinline__ float rcp_approx(float x)
{
	float r;
	asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
	return r;
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
	r.ix = rcp_approx(dx);
	r.iy = rcp_approx(dy);
	r.iz = rcp_approx(dz);
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
	// any per-ray constants keep the test watertight (shared vertices
	// project identically); one rounded reciprocal and two products are
	// cheaper than two divisions
	r.sz = __frcp_rn(dkz);
	r.sx = sel3(r.dx, r.dy, r.dz, kx) * r.sz;
	r.sy = sel3(r.dx, r.dy, r.dz, ky) * r.sz;
}

__device__ __forceinline__ uint32_t qb(uint32_t w, int k)
{
	return (w >> (8 * k)) & 0xffu;
}

// Three-input min / max (sm_100 PTX); a NaN operand is ignored as in fminf.
__device__ __forceinline__ float fmax3(float a, float b, float c)
{
	float r;
	asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
	return r;
}

__device__ __forceinline__ float fmin3(float a, float b, float c)
{
	float r;
	asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
	return r;
}

// Byte k of w as the float 2^23 + 256 * byte (one byte permute: the byte
// goes into bits 8..15 of the mantissa of 2^23).
__device__ __forceinline__ float qbf(uint32_t w, int k)
{
	return __uint_as_float(__byte_perm(w, 0x4b000000u, 0x7404u + 16u * k));
}

// Test the 8 children of node `ni`; returns the node and triangle groups.
// Plane distances are fma(2^23 + 256 q, s, b - 2^23 s) with s = scale / (256
// d) (the stored exponent carries the 1/256) and b = (origin - o) / d.  In
// units of the quantum Q = scale / d the absolute errors are: rounding
// b - 2^23 s (a float near 2^15 Q) at most 2^-9 Q; rounding b, relative
// 2^-23 of |b| <= |t| + 255 Q, at most 2^-14 Q beyond a part relative to t.
// Child planes lie at least 1/32 Q outside the child box (qnode.h), and the
// relative parts (with the reciprocal's) are covered by kWiden.
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
	float bx = __fmaf_rn(-8388608.0f, scx,
	  (__uint_as_float(w0.x) - r.ox) * r.ix);
	float by = __fmaf_rn(-8388608.0f, scy,
	  (__uint_as_float(w0.y) - r.oy) * r.iy);
	float bz = __fmaf_rn(-8388608.0f, scz,
	  (__uint_as_float(w0.z) - r.oz) * r.iz);
	bool fx = signbit(r.ix), fy = signbit(r.iy), fz = signbit(r.iz);
	// lo/hi words: x lo = w2.x,w2.y  y lo = w2.z,w2.w  z lo = w3.x,w3.y
	//              x hi = w3.z,w3.w  y hi = w4.x,w4.y  z hi = w4.z,w4.w
	uint32_t nx0 = fx ? w3.z : w2.x, nx1 = fx ? w3.w : w2.y;
	uint32_t fx0 = fx ? w2.x : w3.z, fx1 = fx ? w2.y : w3.w;
	uint32_t ny0 = fy ? w4.x : w2.z, ny1 = fy ? w4.y : w2.w;
	uint32_t fy0 = fy ? w2.z : w4.x, fy1 = fy ? w2.w : w4.y;
	uint32_t nz0 = fz ? w4.z : w3.x, nz1 = fz ? w4.w : w3.y;
	uint32_t fz0 = fz ? w3.x : w4.z, fz1 = fz ? w3.y : w4.w;
	uint32_t hits = 0, tbits = 0, lhit = 0;
	float gmin = FLT_MAX;
#pragma unroll
	for (int s = 0; s < 8; s++) {
		int b = s & 3;
		uint32_t wnx = s < 4 ? nx0 : nx1, wfx = s < 4 ? fx0 : fx1;
		uint32_t wny = s < 4 ? ny0 : ny1, wfy = s < 4 ? fy0 : fy1;
		uint32_t wnz = s < 4 ? nz0 : nz1, wfz = s < 4 ? fz0 : fz1;
		float tnx = __fmaf_rn(qbf(wnx, b), scx, bx);
		float tny = __fmaf_rn(qbf(wny, b), scy, by);
		float tnz = __fmaf_rn(qbf(wnz, b), scz, bz);
		float tfx = __fmaf_rn(qbf(wfx, b), scx, bx);
		float tfy = __fmaf_rn(qbf(wfy, b), scy, by);
		float tfz = __fmaf_rn(qbf(wfz, b), scz, bz);
		float tn = fmax3(tnx, tny, fmaxf(tnz, 0.0f));
		float tf = fmin3(tfx, tfy, fminf(tfz, tmax));
		if (tn <= tf * kWiden) {
			if ((imask >> s) & 1u) {
				hits |= 1u << s;
				gmin = fminf(gmin, tn);
			} else {
				lhit |= 1u << s;
			}
		}
	}
	// inner hits by slot -> by key (slot ^ octant)
	{
		const uint32_t o = r.oct;
		hits = (o & 1u) ? ((hits & 0x55u) << 1) | ((hits >> 1) & 0x55u) : hits;
		hits = (o & 2u) ? ((hits & 0x33u) << 2) | ((hits >> 2) & 0x33u) : hits;
		hits = (o & 4u) ? ((hits & 0x0fu) << 4) | ((hits >> 4) & 0x0fu) : hits;
	}
	// items of the hit leaf children (typically few)
	while (lhit) {
		uint32_t sl = __ffs(lhit) - 1;
		lhit &= lhit - 1u;
		uint32_t m = ((sl < 4u ? w1.z : w1.w) >> (8u * (sl & 3u))) & 0xffu;
		if (m & NB_META_LEAF) {
			uint32_t cnt = ((m >> 5) & 3u) + 1u;
			tbits |= ((1u << cnt) - 1u) << (m & 31u);
		}
	}
	// node group: first child, hit mask (24..31), entry distance lower
	// bound of the hit children as bf16 truncated towards zero (8..23),
	// inner mask (0..7)
	ng = make_uint2(w1.x, (hits << 24) | ((__float_as_uint(gmin) >> 16) << 8) |
	  imask);
	tg = make_uint2(w1.y, tbits);
}

// Lower bound on the entry distance of a node group's remaining children.
__device__ __forceinline__ float group_tmin(uint32_t y)
{
	return __uint_as_float((y << 8) & 0xffff0000u);
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

constexpr uint32_t kItemGroup = 0x80000000u; // stack entry .x: item group
constexpr uint32_t kFull = 0xffffffffu;

// Per-lane traversal state of the persistent kernels.
struct Trav {
	TRay     r;
	uint2    ng, tg;
	int      sp, blas_sp;
	uint32_t level, cinst;
	float    bt;
	uint32_t btri, binst;
	bool     found;
	uint32_t nvisit, ntest; // counting kernels only
};

constexpr uint32_t kNone = 0xffffffffu;
constexpr int kRefill = 8; // refill a warp once this many lanes idle

// New ray: state reset; the caller visits the TLAS root (node 0).
__device__ __forceinline__ void trav_start(Trav &T, float4 a, float4 b)
{
	tray_slab(T.r, a.x, a.y, a.z, b.x, b.y, b.z);
	T.sp = 0;
	T.blas_sp = -1;
	T.level = 0;
	T.cinst = 0;
	T.bt = a.w;
	T.btri = 0;
	T.binst = 0;
	T.found = false;
	T.ng = make_uint2(0u, 0u);
	T.tg = make_uint2(0u, 0u);
	T.nvisit = 0;
	T.ntest = 0;
}

// Push a stack entry; false (and err set) when the stack is full.
template <int STACK>
__device__ __forceinline__ bool push(Trav &T, uint2 *stk, uint32_t stride,
                                     uint2 e, uint32_t &err)
{
	if (T.sp >= STACK) {
		err = 1u;
		return false;
	}
	stk[(uint32_t)T.sp++ * stride] = e;
	return true;
}

// Take the next child of the node group; false if the group is empty or
// lies entirely beyond the closest hit so far.  Pushes the rest.
template <int STACK>
__device__ __forceinline__ bool next_child(Trav &T, uint2 *stk,
                                           uint32_t stride, uint32_t *vnode,
                                           uint32_t &err)
{
	uint32_t hm = T.ng.y >> 24;
	if (!hm)
		return false;
	if (group_tmin(T.ng.y) > T.bt * kWiden) {
		T.ng.y = 0u;
		return false;
	}
	uint32_t key = __ffs(hm) - 1;
	hm &= hm - 1u;
	uint32_t slot = key ^ T.r.oct;
	*vnode = T.ng.x + __popc(T.ng.y & ((1u << slot) - 1u) & 0xffu);
	T.ng.y = (hm << 24) | (T.ng.y & 0x00ffffffu);
	if (hm && !push<STACK>(T, stk, stride, T.ng, err))
		return false;
	return true;
}

// One node-phase step of a lane that holds no BLAS triangles: enter the
// next instance of a TLAS leaf group (transform, then visit the BLAS
// root), visit the next child of the node group, or pop.  Returns true when
// the ray is finished (or on a stack overflow, with err set).
template <int STACK>
__device__ __forceinline__ bool node_step(Trav &T, const DScene &S,
                                          const float4 *rays, uint32_t ridx,
                                          uint2 *stk, uint32_t stride,
                                          uint32_t &err, uint32_t *vnode)
{
	for (;;) {
		if (T.tg.y) { // level 0: instance references
			uint32_t i = __ffs(T.tg.y) - 1;
			T.tg.y &= T.tg.y - 1u;
			uint32_t inst = __ldg(S.irefs + T.tg.x + i);
			if ((T.ng.y >> 24) && !push<STACK>(T, stk, stride, T.ng, err))
				return true;
			if (T.tg.y && !push<STACK>(T, stk, stride,
			  make_uint2(T.tg.x | kItemGroup, T.tg.y), err))
				return true;
			T.ng.y = 0u;
			T.tg.y = 0u;
			T.blas_sp = T.sp;
			T.level = 1u;
			T.cinst = inst;
			const float4 *ip = S.insts + 4u * inst;
			float4 m0 = __ldg(ip), m1 = __ldg(ip + 1);
			float4 m2 = __ldg(ip + 2);
			*vnode = __float_as_uint(__ldg(ip + 3).x);
			float o[3], d[3];
			xform(m0, m1, m2, T.r.ox, T.r.oy, T.r.oz, T.r.dx, T.r.dy,
			  T.r.dz, o, d);
			tray_slab(T.r, o[0], o[1], o[2], d[0], d[1], d[2]);
			tray_watertight(T.r);
			return false;
		}
		if (next_child<STACK>(T, stk, stride, vnode, err))
			return false;
		if (err)
			return true;
		if (T.level == 1u && T.sp == T.blas_sp) {
			T.level = 0u;
			float4 a = rays[2u * ridx], b = rays[2u * ridx + 1u];
			tray_slab(T.r, a.x, a.y, a.z, b.x, b.y, b.z);
		}
		if (T.sp == 0)
			return true;
		uint2 e = stk[(uint32_t)(--T.sp) * stride];
		if (e.x & kItemGroup) {
			T.tg = make_uint2(e.x & ~kItemGroup, e.y);
			T.ng = make_uint2(0u, 0u);
			if (T.level == 1u)
				return false; // triangles: the triangle phase takes them
		} else {
			T.ng = e;
			T.tg.y = 0u;
		}
	}
}

// Decide this lane's next step: a triangle to test (*titem), a node to
// visit (*vnode: a child, or a BLAS root after entering an instance), or a
// pop.  Stack pushes and the object-space transform happen here; the
// triangle test and the node visit run afterwards in one place for the whole
// warp.  `postpone`: this lane's triangle group goes on the stack so the
// warp keeps visiting nodes together.  Returns true when the ray is done.
template <int STACK>
__device__ __forceinline__ bool trav_decide(Trav &T, const DScene &S,
                                            const float4 *rays, uint32_t ridx,
                                            uint2 *stk, uint32_t stride,
                                            bool postpone, uint32_t &err,
                                            uint32_t *vnode, uint32_t *titem)
{
	bool has_nodes = (T.ng.y >> 24) != 0u;
	if (T.tg.y && has_nodes && postpone) {
		if (T.sp >= STACK) {
			err = 1u;
			return true;
		}
		stk[(uint32_t)T.sp++ * stride] = make_uint2(T.tg.x | kItemGroup,
		  T.tg.y);
		T.tg.y = 0u;
	}
	if (T.tg.y) {
		uint32_t i = __ffs(T.tg.y) - 1;
		T.tg.y &= T.tg.y - 1u;
		uint32_t item = T.tg.x + i;
		if (T.level != 0u) {
			*titem = item;
			return false;
		}
		// enter an instance: keep the TLAS work on the stack
		uint32_t inst = __ldg(S.irefs + item);
		if (has_nodes) {
			if (T.sp >= STACK) {
				err = 1u;
				return true;
			}
			stk[(uint32_t)T.sp++ * stride] = T.ng;
		}
		if (T.tg.y) {
			if (T.sp >= STACK) {
				err = 1u;
				return true;
			}
			stk[(uint32_t)T.sp++ * stride] =
			  make_uint2(T.tg.x | kItemGroup, T.tg.y);
		}
		T.blas_sp = T.sp;
		T.level = 1u;
		T.cinst = inst;
		const float4 *ip = S.insts + 4u * inst;
		float4 m0 = __ldg(ip), m1 = __ldg(ip + 1);
		float4 m2 = __ldg(ip + 2);
		*vnode = __float_as_uint(__ldg(ip + 3).x);
		float o[3], d[3];
		xform(m0, m1, m2, T.r.ox, T.r.oy, T.r.oz, T.r.dx, T.r.dy, T.r.dz,
		  o, d);
		tray_slab(T.r, o[0], o[1], o[2], d[0], d[1], d[2]);
		tray_watertight(T.r);
		return false;
	}
	if (has_nodes) {
		uint32_t hm = T.ng.y >> 24;
		uint32_t key = __ffs(hm) - 1;
		hm &= hm - 1u;
		uint32_t slot = key ^ T.r.oct;
		*vnode = T.ng.x + __popc(T.ng.y & ((1u << slot) - 1u) & 0xffu);
		T.ng.y = (hm << 24) | (T.ng.y & 0xffu);
		if (hm) {
			if (T.sp >= STACK) {
				err = 1u;
				return true;
			}
			stk[(uint32_t)T.sp++ * stride] = T.ng;
		}
		return false;
	}
	if (T.level == 1u && T.sp == T.blas_sp) {
		T.level = 0u;
		float4 a = rays[2u * ridx], b = rays[2u * ridx + 1u];
		tray_slab(T.r, a.x, a.y, a.z, b.x, b.y, b.z);
	}
	if (T.sp == 0)
		return true;
	uint2 e = stk[(uint32_t)(--T.sp) * stride];
	if (e.x & kItemGroup) {
		T.tg = make_uint2(e.x & ~kItemGroup, e.y);
		T.ng = make_uint2(0u, 0u);
	} else {
		T.ng = e;
		T.tg.y = 0u;
	}
	return false;
}

// One triangle test and one node visit per iteration (each from a single
// call site), with Ylitie-style postponing of triangle groups when fewer
// than a fifth of the active lanes want them.
template <bool ANY, int STACK, bool COUNT, class Sink>
__device__ __forceinline__ void trace_step(const DScene &S,
                                                 const float4 *rays,
                                                 uint32_t n, uint32_t *work,
                                                 uint2 *stk, uint32_t stride,
                                                 Sink &sink)
{
	const uint32_t lane = threadIdx.x & 31u;
	bool active = false, exhausted = false;
	uint32_t ridx = 0, err = 0;
	Trav T;
	for (;;) {
		uint32_t vnode = kNone, titem = kNone;
		uint32_t idle = __ballot_sync(kFull, !active);
		if (!exhausted && __popc(idle) >= kRefill) {
			uint32_t cnt = __popc(idle);
			uint32_t leader = __ffs(idle) - 1;
			uint32_t base = 0;
			if (lane == leader)
				base = atomicAdd(work, cnt);
			base = __shfl_sync(kFull, base, leader);
			if (base + cnt >= n)
				exhausted = true;
			if (!active) {
				uint32_t my = base + __popc(idle & ((1u << lane) - 1u));
				if (my < n) {
					ridx = my;
					err = 0;
					float4 rb = rays[2u * my + 1u];
					trav_start(T, rays[2u * my], rb);
					vnode = S.nscenes > 1u ? __ldg(&S.sp[scene_of_path(S,
					  __float_as_uint(rb.w))].tlas_root) : 0u;
					active = true;
				}
			}
		}
		uint32_t act = __ballot_sync(kFull, active);
		if (!act) {
			if (exhausted)
				return;
			continue;
		}
		uint32_t want_tri = __ballot_sync(kFull, active && T.tg.y != 0u);
		bool postpone = __popc(want_tri) * 5u < __popc(act);
		if (active && vnode == kNone) {
			if (trav_decide<STACK>(T, S, rays, ridx, stk, stride, postpone,
			  err, &vnode, &titem)) {
				sink(ridx, T, err);
				active = false;
			}
		}
		if (titem != kNone) {
			float t;
			if (COUNT)
				T.ntest++;
			if (tri_hit(S.tris, titem, T.r, T.bt, &t)) {
				T.bt = t;
				T.btri = titem;
				T.binst = T.cinst;
				T.found = true;
				if (ANY) {
					sink(ridx, T, err);
					active = false;
				}
			}
		}
		if (vnode != kNone) {
			if (COUNT)
				T.nvisit++;
			visit(T.level ? S.blas : S.tlas, vnode, T.r, T.bt, T.ng, T.tg);
		}
	}
}

// Persistent traversal of `n` rays (2 float4 each: (o, tmax),
// (d, payload)) in alternating phases, after Aila and Laine (HPG 2009):
// in the node phase every lane without BLAS triangles visits one node per
// iteration until all lanes hold triangles or are done (lanes that already
// hold triangles keep visiting speculatively and push what they find); in
// the triangle phase all lanes test one triangle per iteration.  Idle lanes
// are refilled from a global work counter once at least kRefill of a warp's
// lanes are idle.  `sink` gets every finished ray: (index, state, error).
template <bool ANY, int STACK, bool COUNT, class Sink>
__device__ __forceinline__ void trace_phase(const DScene &S,
                                                 const float4 *rays,
                                                 uint32_t n, uint32_t *work,
                                                 uint2 *stk, uint32_t stride,
                                                 Sink &sink)
{
	const uint32_t lane = threadIdx.x & 31u;
	bool active = false, exhausted = false;
	uint32_t ridx = 0, err = 0;
	Trav T;
	for (;;) {
		uint32_t vnode = kNone;
		uint32_t idle = __ballot_sync(kFull, !active);
		if (!exhausted && __popc(idle) >= kRefill) {
			uint32_t cnt = __popc(idle);
			uint32_t leader = __ffs(idle) - 1;
			uint32_t base = 0;
			if (lane == leader)
				base = atomicAdd(work, cnt);
			base = __shfl_sync(kFull, base, leader);
			if (base + cnt >= n)
				exhausted = true;
			if (!active) {
				uint32_t my = base + __popc(idle & ((1u << lane) - 1u));
				if (my < n) {
					ridx = my;
					err = 0;
					float4 rb = rays[2u * my + 1u];
					trav_start(T, rays[2u * my], rb);
					vnode = S.nscenes > 1u ? __ldg(&S.sp[scene_of_path(S,
					  __float_as_uint(rb.w))].tlas_root) : 0u;
					active = true;
				}
			}
		}
		if (!__any_sync(kFull, active)) {
			if (exhausted)
				return;
			continue;
		}
		// node phase
		for (;;) {
			bool holding = active && T.level == 1u && T.tg.y != 0u;
			bool searching = active && !holding;
			if (!__any_sync(kFull, searching || vnode != kNone))
				break;
			bool spec = false;
			if (searching && vnode == kNone) {
				if (node_step<STACK>(T, S, rays, ridx, stk, stride, err,
				  &vnode)) {
					sink(ridx, T, err);
					active = false;
				}
			} else if (holding && T.sp + 2 <= STACK) {
				uint32_t e2 = 0;
				spec = next_child<STACK>(T, stk, stride, &vnode, e2);
			}
			if (vnode != kNone) {
				uint2 held = T.tg;
				if (COUNT)
					T.nvisit++;
				visit(T.level ? S.blas : S.tlas, vnode, T.r, T.bt, T.ng,
				  T.tg);
				if (spec) {
					if (T.tg.y)
						stk[(uint32_t)T.sp++ * stride] =
						  make_uint2(T.tg.x | kItemGroup, T.tg.y);
					T.tg = held;
				}
				vnode = kNone;
			}
		}
		// triangle phase
		for (;;) {
			bool want = active && T.level == 1u && T.tg.y != 0u;
			if (!__any_sync(kFull, want))
				break;
			if (want) {
				uint32_t i = __ffs(T.tg.y) - 1;
				T.tg.y &= T.tg.y - 1u;
				float t;
				if (COUNT)
					T.ntest++;
				if (tri_hit(S.tris, T.tg.x + i, T.r, T.bt, &t)) {
					T.bt = t;
					T.btri = T.tg.x + i;
					T.binst = T.cinst;
					T.found = true;
					if (ANY) {
						sink(ridx, T, err);
						active = false;
					}
				}
			}
		}
	}
}

// Node visit, then the triangle group (Ylitie, Karras and Laine, HPG
// 2017): each iteration a lane without BLAS triangles takes one node step
// (instance entry, child visit or pop); then all lanes holding triangles test
// them one per inner iteration, unless fewer than a fifth of the active lanes
// hold any: then those that still have nodes to visit push their triangles
// and the warp goes back to visiting nodes.
template <bool ANY, int STACK, bool COUNT, class Sink, bool TWO = false,
          class Sink2 = Sink>
__device__ __forceinline__ void trace_ylitie(const DScene &S,
                                             const float4 *rays, uint32_t n,
                                             uint32_t *work, uint2 *stk,
                                             uint32_t stride, Sink &sink,
                                             const float4 *rays2 = nullptr,
                                             uint32_t n2 = 0u,
                                             Sink2 *sink2 = nullptr)
{
	// TWO: work items n .. n + n2 - 1 are any-hit rays of a second queue
	// (rays2, reported to sink2), taken once the first queue is drained
	const uint32_t ntot = TWO ? n + n2 : n;
	bool second = false;
	const uint32_t lane = threadIdx.x & 31u;
	bool active = false, exhausted = false;
	uint32_t ridx = 0, err = 0;
	Trav T;
	// a warp keeps at most `share` rays in flight: 32 when the launch has
	// at least 32 rays per resident warp; fewer in small launches, which
	// then spread over every warp instead of filling a few (a warp runs
	// until its slowest ray ends).  Only the launches that can be small
	// (bounces: fused or any-hit) use it; the primary closest-hit launch
	// keeps 32 and its register.
	const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
	const uint32_t share = (TWO || ANY) ?
	  min(32u, max(1u, (ntot + nwarps - 1u) / nwarps)) : 32u;
	const uint32_t need = min((uint32_t)kRefill, share);
	for (;;) {
		uint32_t vnode = kNone;
		uint32_t idle = __ballot_sync(kFull, !active);
		uint32_t nidle = __popc(idle), nact = 32u - nidle;
		uint32_t room = min(nidle, share > nact ? share - nact : 0u);
		if (!exhausted && room >= need) {
			uint32_t cnt = room;
			uint32_t leader = __ffs(idle) - 1;
			uint32_t base = 0;
			if (lane == leader)
				base = atomicAdd(work, cnt);
			base = __shfl_sync(kFull, base, leader);
			if (base + cnt >= ntot)
				exhausted = true;
			if (!active) {
				uint32_t rank = __popc(idle & ((1u << lane) - 1u));
				uint32_t my = base + rank;
				if (rank < cnt && my < ntot) {
					second = TWO && my >= n;
					ridx = second ? my - n : my;
					err = 0;
					const float4 *rq = second ? rays2 : rays;
					float4 rb = rq[2u * ridx + 1u];
					trav_start(T, rq[2u * ridx], rb);
					vnode = S.nscenes > 1u ? __ldg(&S.sp[scene_of_path(S,
					  __float_as_uint(rb.w))].tlas_root) : 0u;
					active = true;
				}
			}
		}
		if (!__any_sync(kFull, active)) {
			if (exhausted)
				return;
			continue;
		}
		bool holding = active && T.level == 1u && T.tg.y != 0u;
		if (active && !holding && vnode == kNone) {
			if (node_step<STACK>(T, S, TWO && second ? rays2 : rays, ridx,
			  stk, stride, err, &vnode)) {
				if (TWO && second)
					(*sink2)(ridx, T, err);
				else
					sink(ridx, T, err);
				active = false;
			}
		}
		if (vnode != kNone) {
			if (COUNT)
				T.nvisit++;
			visit(T.level ? S.blas : S.tlas, vnode, T.r, T.bt, T.ng, T.tg);
		}
		for (;;) {
			bool want = active && T.level == 1u && T.tg.y != 0u;
			uint32_t wm = __ballot_sync(kFull, want);
			if (!wm)
				break;
			if (__popc(wm) * 5u < __popc(__ballot_sync(kFull, active))) {
				if (want && (T.ng.y >> 24) && T.sp < STACK) {
					stk[(uint32_t)T.sp++ * stride] =
					  make_uint2(T.tg.x | kItemGroup, T.tg.y);
					T.tg.y = 0u;
				}
				break;
			}
			// One round of the triangle phase: the first 32 pending
			// triangles of the warp (in lane order) are tested by all 32
			// lanes, each with its owner's ray taken by shuffle; an
			// owner keeps the nearest hit of its testers (lowest item on
			// equal t, as sequential testing would).  Lanes that test
			// their own triangles one by one leave about 3/4 of the warp
			// idle (7.7 active lanes per iteration measured on the
			// 1080p workload).
			uint32_t k = want ? __popc(T.tg.y) : 0u;
			uint32_t incl = k;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				uint32_t x = __shfl_up_sync(kFull, incl, o);
				if (lane >= (uint32_t)o)
					incl += x;
			}
			uint32_t total = __shfl_sync(kFull, incl, 31);
			uint32_t excl = incl - k;
			// owner of work item `lane`: first lane whose prefix exceeds it
			uint32_t owner = 0;
#pragma unroll
			for (int step = 16; step >= 1; step >>= 1) {
				uint32_t v = __shfl_sync(kFull, incl, owner + step - 1);
				if (v <= lane)
					owner += step;
			}
			owner = min(owner, 31u);
			bool has = lane < total;
			uint32_t o_excl = __shfl_sync(kFull, excl, owner);
			uint32_t o_tgy = __shfl_sync(kFull, T.tg.y, owner);
			uint32_t o_tgx = __shfl_sync(kFull, T.tg.x, owner);
			TRay rr;
			rr.ox = __shfl_sync(kFull, T.r.ox, owner);
			rr.oy = __shfl_sync(kFull, T.r.oy, owner);
			rr.oz = __shfl_sync(kFull, T.r.oz, owner);
			rr.sx = __shfl_sync(kFull, T.r.sx, owner);
			rr.sy = __shfl_sync(kFull, T.r.sy, owner);
			rr.sz = __shfl_sync(kFull, T.r.sz, owner);
			uint32_t kk = __shfl_sync(kFull, T.r.kx | (T.r.ky << 2) |
			  (T.r.kz << 4), owner);
			rr.kx = kk & 3u;
			rr.ky = (kk >> 2) & 3u;
			rr.kz = (kk >> 4) & 3u;
			float obt = __shfl_sync(kFull, T.bt, owner);
			uint32_t item = has ? o_tgx + nth_bit(o_tgy, lane - o_excl) : 0u;
			float t = 0.0f;
			bool hit = has && tri_hit(S.tris, item, rr, obt, &t);
			uint32_t grp = __match_any_sync(kFull, has ? owner : 32u);
			uint32_t key = hit ? __float_as_uint(t) : 0x7f800000u;
			uint32_t tmin = __reduce_min_sync(grp, key);
			uint32_t imin = __reduce_min_sync(grp, (hit && key == tmin) ?
			  item : kNone);
			uint32_t src = (want && excl < 32u) ? excl : lane;
			uint32_t got_t = __shfl_sync(kFull, tmin, src);
			uint32_t got_i = __shfl_sync(kFull, imin, src);
			if (want && excl < 32u) {
				uint32_t ntest = min(k, 32u - excl);
				if (COUNT)
					T.ntest += ntest;
				T.tg.y = ntest >= k ? 0u :
				  (T.tg.y & ~((1u << nth_bit(T.tg.y, ntest)) - 1u));
				if (got_i != kNone && __uint_as_float(got_t) < T.bt) {
					T.bt = __uint_as_float(got_t);
					T.btri = got_i;
					T.binst = T.cinst;
					T.found = true;
					if (ANY) {
						sink(ridx, T, err);
						active = false;
						T.tg.y = 0u;
					} else if (TWO && second) {
						(*sink2)(ridx, T, err);
						active = false;
						T.tg.y = 0u;
					}
				}
			}
		}
	}
}

// Traversal schedules (see trace_step, trace_phase, trace_ylitie).
enum { kSchedStep = 0, kSchedPhase = 1, kSchedYlitie = 2 };

template <int SCHED, bool ANY, int STACK, bool COUNT, class Sink>
__device__ __forceinline__ void trace_persistent(const DScene &S,
                                                 const float4 *rays,
                                                 uint32_t n, uint32_t *work,
                                                 uint2 *stk, uint32_t stride,
                                                 Sink &sink)
{
	if (SCHED == kSchedStep)
		trace_step<ANY, STACK, COUNT>(S, rays, n, work, stk, stride, sink);
	else if (SCHED == kSchedPhase)
		trace_phase<ANY, STACK, COUNT>(S, rays, n, work, stk, stride, sink);
	else
		trace_ylitie<ANY, STACK, COUNT>(S, rays, n, work, stk, stride,
		  sink);
}

// Closest hits of one queue, then any hits of a second queue, in one
// persistent loop (Ylitie schedule).
template <int STACK, bool COUNT, class Sink, class Sink2>
__device__ __forceinline__ void trace_two(const DScene &S,
                                          const float4 *rays, uint32_t n,
                                          const float4 *rays2, uint32_t n2,
                                          uint32_t *work, uint2 *stk,
                                          uint32_t stride, Sink &sink,
                                          Sink2 &sink2)
{
	trace_ylitie<false, STACK, COUNT, Sink, true, Sink2>(S, rays, n, work,
	  stk, stride, sink, rays2, n2, &sink2);
}

// --------------------------------------------------------------- sinks --

// Raw closest hit: (t, triangle index, instance, 0); t = FLT_MAX on a miss
// or on a device error (counted in errs).
struct SinkRaw {
	float4   *hits;
	uint32_t *errs;
	unsigned long long *counts; // visits, tests (counting kernels)
	__device__ void operator()(uint32_t i, const Trav &T, uint32_t err)
	{
		if (counts) {
			atomicAdd(&counts[0], (unsigned long long)T.nvisit);
			atomicAdd(&counts[1], (unsigned long long)T.ntest);
		}
		if (err)
			atomicAdd(errs, 1u);
		hits[i] = (T.found && !err) ? make_float4(T.bt,
		  __uint_as_float(T.btri), __uint_as_float(T.binst), 0.0f) :
		  make_float4(FLT_MAX, 0.0f, 0.0f, 0.0f);
	}
};

// Occlusion answer; a ray abandoned by a device error reports occluded, the
// conservative answer (no light leaks through), as SinkShadow adds no light
// for it.
struct SinkOccl {
	uint8_t  *occl;
	uint32_t *errs;
	__device__ void operator()(uint32_t i, const Trav &T, uint32_t err)
	{
		if (err)
			atomicAdd(errs, 1u);
		occl[i] = (T.found || err) ? 1 : 0;
	}
};

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
	if (h.t == FLT_MAX)
		return make_float4(FLT_MAX, 0.0f, 0.0f, 0.0f);
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
