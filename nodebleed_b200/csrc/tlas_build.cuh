// Device-side update of a dynamic scene (sm_100a).
//
// The reference redoes three host steps every frame in which a transform
// changed (main.c:257-264): upd_rinsts (main.c:117-157) inverts each
// instance's object->world matrix (mat4_inv, mat4.c:299) and bounds the
// instance in world space by the 8 transformed corners of its BLAS root box;
// rend_prepdynamic (rend.c:3073-3090) rebuilds the TLAS with build_bvh8
// (rend.c:458-709); the light table follows the instances.  Here all three
// run on the device, fed only by the new matrices:
//
//   k_inst_update   inverse (the FP64 cofactor sequence of the host bridge,
//                   so world->object bits match it) and world box per instance
//   k_tlas_init, k_tlas_level, k_tlas_finish
//                   top-down binned SAH straight into the 8-wide quantised
//                   node layout (gpulayout.h), one launch per tree level,
//                   one warp per open node over all SMs
//   k_tlas_refit    same topology, child boxes recomputed from the instance
//                   ranges the last build recorded, all nodes in parallel
//   k_light_update  world-space emitting triangles and their area CDF (the
//                   host's build_lights sequence)
//
// The build is this library's own algorithm, not the reference's: each node
// is split horizontally (its child of largest surface area is split by a
// 16-bin SAH over centroids on the best of three axes) until it has 8
// children, inner children become the next level's open nodes.  A depth
// limit switches a subtree to count-balanced median splits when SAH splits
// could exceed it, so the traversal stack the host sized still holds.

#ifndef NB_TLAS_BUILD_CUH
#define NB_TLAS_BUILD_CUH

#include "qnode.h"
#include "trace.cuh"

namespace nb {

constexpr uint32_t kTbMaxInst = 4096; // hit ids keep 12 instance bits
constexpr int kTbBins = 16;

// ------------------------------------------------------ instance update --

// Per instance: world->object 3x4 from the inverse of glob (row-major 4x4,
// object->world), written into rows 0-2 of the device instance record;
// world box from the 8 corners of the BLAS root box (rootbox: min, max).
// The inverse follows the host bridge's cofactor expansion over 2x2 minors
// in FP64 operation by operation (no contraction), so the FP32 results are
// bit-identical to it.  A singular matrix zeroes the transform (the
// instance is never hit) and counts into *err.
__global__ void __launch_bounds__(128) k_inst_update(
  const float *__restrict__ glob, uint32_t n,
  const float4 *__restrict__ rootbox, float4 *insts, float4 *wbox,
  uint32_t *err)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const float *g = glob + 16u * i;
	double a[16];
	float gf[16];
	for (int k = 0; k < 16; k++) {
		gf[k] = g[k];
		a[k] = gf[k];
	}
	double s0 = a[0] * a[5] - a[4] * a[1];
	double s1 = a[0] * a[6] - a[4] * a[2];
	double s2 = a[0] * a[7] - a[4] * a[3];
	double s3 = a[1] * a[6] - a[5] * a[2];
	double s4 = a[1] * a[7] - a[5] * a[3];
	double s5 = a[2] * a[7] - a[6] * a[3];
	double c5 = a[10] * a[15] - a[14] * a[11];
	double c4 = a[9] * a[15] - a[13] * a[11];
	double c3 = a[9] * a[14] - a[13] * a[10];
	double c2 = a[8] * a[15] - a[12] * a[11];
	double c1 = a[8] * a[14] - a[12] * a[10];
	double c0 = a[8] * a[13] - a[12] * a[9];
	double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
	float inv[12];
	if (det == 0.0) {
		for (int k = 0; k < 12; k++)
			inv[k] = 0.0f;
		atomicAdd(err, 1u);
	} else {
		double id = 1.0 / det;
		double r[12] = {
		  (a[5] * c5 - a[6] * c4 + a[7] * c3),
		  (-a[1] * c5 + a[2] * c4 - a[3] * c3),
		  (a[13] * s5 - a[14] * s4 + a[15] * s3),
		  (-a[9] * s5 + a[10] * s4 - a[11] * s3),
		  (-a[4] * c5 + a[6] * c2 - a[7] * c1),
		  (a[0] * c5 - a[2] * c2 + a[3] * c1),
		  (-a[12] * s5 + a[14] * s2 - a[15] * s1),
		  (a[8] * s5 - a[10] * s2 + a[11] * s1),
		  (a[4] * c4 - a[5] * c2 + a[7] * c0),
		  (-a[0] * c4 + a[1] * c2 - a[3] * c0),
		  (a[12] * s4 - a[13] * s2 + a[15] * s0),
		  (-a[8] * s4 + a[9] * s2 - a[11] * s0)};
		for (int k = 0; k < 12; k++)
			inv[k] = (float)(r[k] * id);
	}
	float4 *ip = insts + 4u * i;
	ip[0] = make_float4(inv[0], inv[1], inv[2], inv[3]);
	ip[1] = make_float4(inv[4], inv[5], inv[6], inv[7]);
	ip[2] = make_float4(inv[8], inv[9], inv[10], inv[11]);
	float4 bl = rootbox[2u * i], bh = rootbox[2u * i + 1u];
	float mi[3] = {bl.x, bl.y, bl.z}, ma[3] = {bh.x, bh.y, bh.z};
	float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
	float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	for (int c = 0; c < 8; c++) {
		float x = c & 1 ? mi[0] : ma[0];
		float y = c & 2 ? mi[1] : ma[1];
		float z = c & 4 ? mi[2] : ma[2];
		float v[3];
		for (int r = 0; r < 3; r++)
			v[r] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(gf[4 * r], x),
			  __fmul_rn(gf[4 * r + 1], y)), __fmul_rn(gf[4 * r + 2], z)),
			  gf[4 * r + 3]);
		for (int r = 0; r < 3; r++) {
			lo[r] = v[r] < lo[r] ? v[r] : lo[r];
			hi[r] = v[r] > hi[r] ? v[r] : hi[r];
		}
	}
	wbox[2u * i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
	wbox[2u * i + 1u] = make_float4(hi[0], hi[1], hi[2], 0.0f);
}

// Object->world 4x4 (row-major) of each instance from its uploaded
// world->object 3x4, inverted in FP64 (the affine inverse: 3x3 by
// cofactors, translation -A^-1 b).  Feeds k_inst_tight when the TLAS is
// rebuilt at upload time, where only the render data's inverse matrices
// exist; the tight boxes it yields are padded by the TLAS quantisation, so
// the inverse's rounding does not matter.  A singular matrix gives zeros.
__global__ void __launch_bounds__(128) k_inst_glob(const float4 *insts,
                                                   uint32_t n, float *glob)
{
	uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const float4 *ip = insts + 4u * i;
	float4 r0 = ip[0], r1 = ip[1], r2 = ip[2];
	double A[9] = {r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, r2.x, r2.y, r2.z};
	double b[3] = {r0.w, r1.w, r2.w};
	double c0 = A[4] * A[8] - A[5] * A[7], c1 = A[5] * A[6] - A[3] * A[8];
	double c2 = A[3] * A[7] - A[4] * A[6];
	double det = A[0] * c0 + A[1] * c1 + A[2] * c2;
	float *g = glob + 16u * i;
	for (int k = 0; k < 16; k++)
		g[k] = 0.0f;
	if (det == 0.0)
		return;
	double I[9] = {c0 / det, (A[2] * A[7] - A[1] * A[8]) / det,
	  (A[1] * A[5] - A[2] * A[4]) / det, c1 / det,
	  (A[0] * A[8] - A[2] * A[6]) / det, (A[2] * A[3] - A[0] * A[5]) / det,
	  c2 / det, (A[1] * A[6] - A[0] * A[7]) / det,
	  (A[0] * A[4] - A[1] * A[3]) / det};
	for (int r = 0; r < 3; r++) {
		for (int k = 0; k < 3; k++)
			g[4 * r + k] = (float)I[3 * r + k];
		g[4 * r + 3] = (float)-(I[3 * r] * b[0] + I[3 * r + 1] * b[1] +
		  I[3 * r + 2] * b[2]);
	}
	g[15] = 1.0f;
}

// Tight world box of each instance: the bounds of every vertex of its BLAS
// (trange: first triangle and count in the device triangle array) after
// glob, one CTA per instance.  The reference bounds an instance by the 8
// transformed corners of its root box, which a rotation inflates; a TLAS
// over the tight boxes lets fewer rays enter instances they never touch.
// The quantised TLAS boxes are padded by at least one quantum of 2^-22 of
// the coordinates' magnitude, which covers the rounding of the transform.
__device__ __forceinline__ void tb_warp_box(float lo[3], float hi[3]);

__global__ void __launch_bounds__(256) k_inst_tight(
  const float *__restrict__ glob, uint32_t n, const uint2 *__restrict__ trange,
  const float4 *__restrict__ tris, float4 *wbox)
{
	__shared__ float part[8][6];
	uint32_t i = blockIdx.x;
	if (i >= n)
		return;
	const float *g = glob + 16u * i;
	float m[12];
	for (int k = 0; k < 12; k++)
		m[k] = g[k];
	uint2 r = trange[i];
	float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
	float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	for (uint32_t t = r.x + threadIdx.x; t < r.x + r.y; t += blockDim.x)
		for (int v = 0; v < 3; v++) {
			float4 p = __ldg(tris + 3u * t + v);
			for (int a = 0; a < 3; a++) {
				float w = __fadd_rn(__fadd_rn(__fadd_rn(
				  __fmul_rn(m[4 * a], p.x), __fmul_rn(m[4 * a + 1], p.y)),
				  __fmul_rn(m[4 * a + 2], p.z)), m[4 * a + 3]);
				lo[a] = fminf(lo[a], w);
				hi[a] = fmaxf(hi[a], w);
			}
		}
	tb_warp_box(lo, hi);
	uint32_t w = threadIdx.x >> 5;
	if ((threadIdx.x & 31u) == 0)
		for (int a = 0; a < 3; a++) {
			part[w][a] = lo[a];
			part[w][3 + a] = hi[a];
		}
	__syncthreads();
	if (threadIdx.x == 0) {
		for (uint32_t k = 1; k < (blockDim.x >> 5); k++)
			for (int a = 0; a < 3; a++) {
				part[0][a] = fminf(part[0][a], part[k][a]);
				part[0][3 + a] = fmaxf(part[0][3 + a], part[k][3 + a]);
			}
		wbox[2u * i] = make_float4(part[0][0], part[0][1], part[0][2], 0.0f);
		wbox[2u * i + 1u] = make_float4(part[0][3], part[0][4], part[0][5],
		  0.0f);
	}
}

// ----------------------------------------------------------- TLAS build --

struct TbNode { // an open node: its instance range and box
	uint32_t start, cnt, node, depth;
	float    lo[3], hi[3];
};

struct TbArgs {
	const float4 *wbox;     // world boxes (min, max) per instance
	uint32_t      n;        // instances (<= kTbMaxInst)
	uint32_t      inst_base;
	nb_qnode     *nodes;    // capacity node_cap, root at 0
	uint32_t      node_cap;
	uint32_t     *irefs;    // n leaf items
	TbNode       *qa, *qb;  // level queues, n entries each
	uint2        *ranges;   // per node and slot: (start, cnt) for the refit
	uint32_t     *order;    // instance order of the ranges (n)
	uint32_t     *info;     // [0] nodes, [1] depth, [2] overflow
	uint32_t      depth_limit;
	uint16_t     *idx, *tmp; // instance order being partitioned (n each)
	uint32_t     *ctr;       // [0] nodes, [1] items, [2]/[3] queue a/b
};

struct TbBin {
	uint32_t cnt;
	int      lo[3], hi[3]; // float bits in signed-orderable form
};

struct TbChild {
	uint32_t start, cnt;
	float    lo[3], hi[3];
};

// Float <-> int with the same order under signed comparison (for shared
// atomicMin/Max on floats).
__device__ __forceinline__ int tb_ord(float f)
{
	int b = __float_as_int(f);
	return b >= 0 ? b : b ^ 0x7fffffff;
}

__device__ __forceinline__ float tb_unord(int b)
{
	return __int_as_float(b >= 0 ? b : b ^ 0x7fffffff);
}

__device__ __forceinline__ float tb_area(const float lo[3], const float hi[3])
{
	float dx = fmaxf(hi[0] - lo[0], 0.0f), dy = fmaxf(hi[1] - lo[1], 0.0f);
	float dz = fmaxf(hi[2] - lo[2], 0.0f);
	return dx * dy + dy * dz + dz * dx;
}

// Bin of coordinate c along an axis with centroid range [cmn, cmn + ext).
__device__ __forceinline__ int tb_bin(float c, float cmn, float scale)
{
	int b = (int)((c - cmn) * scale);
	return b < 0 ? 0 : (b > kTbBins - 1 ? kTbBins - 1 : b);
}

// Box of instance i (wbox in global or, in the build, shared memory),
// widened per axis by 2^-20 of its coordinates' magnitude: the world boxes
// come from transformed vertices or corners rounded to FP32, and the
// widening covers that rounding whatever the quantisation of the TLAS
// (whose planes only keep 1/32 of a quantum outside a child box, and a
// node of coplanar instances has a tiny quantum along that axis).
__device__ __forceinline__ void tb_load(const float4 *wbox, uint32_t i,
                                        float lo[3], float hi[3])
{
	float4 a = wbox[2u * i], b = wbox[2u * i + 1u];
	lo[0] = a.x; lo[1] = a.y; lo[2] = a.z;
	hi[0] = b.x; hi[1] = b.y; hi[2] = b.z;
	for (int k = 0; k < 3; k++) {
		float pad = __fmul_ru(fmaxf(fabsf(lo[k]), fabsf(hi[k])), 0x1p-20f);
		lo[k] = __fsub_rd(lo[k], pad);
		hi[k] = __fadd_ru(hi[k], pad);
	}
}

// Warp-wide min / max of 3-vectors.
__device__ __forceinline__ void tb_warp_box(float lo[3], float hi[3])
{
	for (int o = 16; o > 0; o >>= 1)
		for (int a = 0; a < 3; a++) {
			lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
			hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
		}
}

// Box of the instances idx[start, start + cnt) (whole warp).
__device__ void tb_range_box(const float4 *wbox, const uint16_t *idx,
                             uint32_t start, uint32_t cnt, float lo[3],
                             float hi[3])
{
	const uint32_t lane = threadIdx.x & 31u;
	for (int a = 0; a < 3; a++) {
		lo[a] = FLT_MAX;
		hi[a] = -FLT_MAX;
	}
	for (uint32_t i = lane; i < cnt; i += 32u) {
		float l[3], h[3];
		tb_load(wbox, idx[start + i], l, h);
		for (int a = 0; a < 3; a++) {
			lo[a] = fminf(lo[a], l[a]);
			hi[a] = fmaxf(hi[a], h[a]);
		}
	}
	tb_warp_box(lo, hi);
}

// Split idx[start, start + cnt) (cnt >= 2) in two, in place (whole warp,
// uniform arguments).  SAH over 16 centroid bins per axis unless `median`
// or no bin boundary separates the centroids; then the first cnt / 2 in
// index order go left.  Returns the left count.
__device__ uint32_t tb_split(const float4 *wbox, uint16_t *idx,
                             uint16_t *tmp, TbBin *bins, uint32_t start,
                             uint32_t cnt, bool median)
{
	const uint32_t lane = threadIdx.x & 31u;
	int axis = -1, kbest = -1;
	float cmn[3], cmx[3], scale[3];
	if (!median) {
		for (int a = 0; a < 3; a++) {
			cmn[a] = FLT_MAX;
			cmx[a] = -FLT_MAX;
		}
		for (uint32_t i = lane; i < cnt; i += 32u) {
			float l[3], h[3];
			tb_load(wbox, idx[start + i], l, h);
			for (int a = 0; a < 3; a++) {
				float c = 0.5f * (l[a] + h[a]);
				cmn[a] = fminf(cmn[a], c);
				cmx[a] = fmaxf(cmx[a], c);
			}
		}
		tb_warp_box(cmn, cmx);
		for (int a = 0; a < 3; a++) {
			float ext = cmx[a] - cmn[a];
			scale[a] = ext > 0.0f ? (float)kTbBins / ext : 0.0f;
		}
		for (int k = (int)lane; k < 3 * kTbBins; k += 32) {
			bins[k].cnt = 0u;
			for (int a = 0; a < 3; a++) {
				bins[k].lo[a] = tb_ord(FLT_MAX);
				bins[k].hi[a] = tb_ord(-FLT_MAX);
			}
		}
		__syncwarp();
		for (uint32_t i = lane; i < cnt; i += 32u) {
			float l[3], h[3];
			tb_load(wbox, idx[start + i], l, h);
			for (int a = 0; a < 3; a++) {
				if (scale[a] == 0.0f)
					continue;
				float c = 0.5f * (l[a] + h[a]);
				TbBin *b = bins + a * kTbBins + tb_bin(c, cmn[a], scale[a]);
				atomicAdd(&b->cnt, 1u);
				for (int d = 0; d < 3; d++) {
					atomicMin(&b->lo[d], tb_ord(l[d]));
					atomicMax(&b->hi[d], tb_ord(h[d]));
				}
			}
		}
		__syncwarp();
		// lane a sweeps axis a: cost of "bins 0..k left" for k in 0..14
		float best = FLT_MAX;
		int bk = -1;
		if (lane < 3u && scale[lane] > 0.0f) {
			const TbBin *B = bins + lane * kTbBins;
			float rarea[kTbBins];
			uint32_t rcnt[kTbBins];
			float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
			float rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
			uint32_t rc = 0;
			for (int k = kTbBins - 1; k >= 1; k--) {
				rc += B[k].cnt;
				for (int d = 0; d < 3; d++) {
					rlo[d] = fminf(rlo[d], tb_unord(B[k].lo[d]));
					rhi[d] = fmaxf(rhi[d], tb_unord(B[k].hi[d]));
				}
				rarea[k] = tb_area(rlo, rhi);
				rcnt[k] = rc;
			}
			float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
			float lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
			uint32_t lc = 0;
			for (int k = 0; k < kTbBins - 1; k++) {
				lc += B[k].cnt;
				for (int d = 0; d < 3; d++) {
					llo[d] = fminf(llo[d], tb_unord(B[k].lo[d]));
					lhi[d] = fmaxf(lhi[d], tb_unord(B[k].hi[d]));
				}
				if (lc == 0u || rcnt[k + 1] == 0u)
					continue;
				float cost = tb_area(llo, lhi) * (float)lc +
				  rarea[k + 1] * (float)rcnt[k + 1];
				if (cost < best) {
					best = cost;
					bk = k;
				}
			}
		}
		// best over the three axes (lowest axis on equal cost)
		float b0 = __shfl_sync(kFull, best, 0);
		float b1 = __shfl_sync(kFull, best, 1);
		float b2 = __shfl_sync(kFull, best, 2);
		int k0 = __shfl_sync(kFull, bk, 0), k1 = __shfl_sync(kFull, bk, 1);
		int k2 = __shfl_sync(kFull, bk, 2);
		if (k0 >= 0) {
			axis = 0;
			kbest = k0;
		}
		if (k1 >= 0 && (axis < 0 || b1 < b0)) {
			axis = 1;
			kbest = k1;
			b0 = b1;
		}
		if (k2 >= 0 && (axis < 0 || b2 < b0)) {
			axis = 2;
			kbest = k2;
		}
	}
	uint32_t lcnt = cnt / 2u;
	if (axis >= 0) {
		// stable partition through tmp: left items first
		uint32_t nl = 0;
		for (uint32_t i0 = 0; i0 < cnt; i0 += 32u) {
			uint32_t i = i0 + lane;
			bool left = false;
			if (i < cnt) {
				float l[3], h[3];
				tb_load(wbox, idx[start + i], l, h);
				float c = 0.5f * (l[axis] + h[axis]);
				left = tb_bin(c, cmn[axis], scale[axis]) <= kbest;
			}
			nl += __popc(__ballot_sync(kFull, left));
		}
		uint32_t pl = 0, pr = nl;
		for (uint32_t i0 = 0; i0 < cnt; i0 += 32u) {
			uint32_t i = i0 + lane;
			bool live = i < cnt, left = false;
			uint16_t v = 0;
			if (live) {
				v = idx[start + i];
				float l[3], h[3];
				tb_load(wbox, v, l, h);
				float c = 0.5f * (l[axis] + h[axis]);
				left = tb_bin(c, cmn[axis], scale[axis]) <= kbest;
			}
			uint32_t ml = __ballot_sync(kFull, live && left);
			uint32_t mr = __ballot_sync(kFull, live && !left);
			uint32_t below = (1u << lane) - 1u;
			if (live)
				tmp[start + (left ? pl + __popc(ml & below) :
				  pr + __popc(mr & below))] = v;
			pl += __popc(ml);
			pr += __popc(mr);
		}
		__syncwarp();
		for (uint32_t i = lane; i < cnt; i += 32u)
			idx[start + i] = tmp[start + i];
		__syncwarp();
		lcnt = nl;
	}
	if (lcnt == 0u || lcnt >= cnt)
		lcnt = cnt / 2u;
	return lcnt;
}

// Levels a balanced 8-wide subtree over cnt items needs (this node
// included).
__device__ __forceinline__ uint32_t tb_levels(uint32_t cnt)
{
	uint32_t l = 1, cap = 8;
	while (cap < cnt) {
		cap *= 8u;
		l++;
	}
	return l;
}

// Build one node from its open range (whole warp): horizontal splits until
// 8 children, then encode, allocate its inner children (contiguous) and
// leaf items (contiguous), and queue the inner children.
__device__ void tb_node(const TbArgs &A, uint16_t *idx, uint16_t *tmp,
                        TbBin *bins, TbChild *ch, const TbNode &nd,
                        TbNode *next, uint32_t *next_cnt,
                        uint32_t *node_ctr, uint32_t *item_ctr)
{
	const uint32_t lane = threadIdx.x & 31u;
	// SAH only while a balanced finish of the subtree still fits the limit
	bool median = nd.depth + tb_levels(nd.cnt) - 1u >= A.depth_limit;
	if (lane == 0) {
		ch[0].start = nd.start;
		ch[0].cnt = nd.cnt;
		for (int a = 0; a < 3; a++) {
			ch[0].lo[a] = nd.lo[a];
			ch[0].hi[a] = nd.hi[a];
		}
	}
	__syncwarp();
	int nch = 1;
	while (nch < 8) {
		int j = -1;
		float best = -1.0f;
		for (int c = 0; c < nch; c++) {
			if (ch[c].cnt < 2u)
				continue;
			float key = median ? (float)ch[c].cnt :
			  tb_area(ch[c].lo, ch[c].hi);
			if (key > best) {
				best = key;
				j = c;
			}
		}
		if (j < 0)
			break;
		uint32_t s = ch[j].start, cnt = ch[j].cnt;
		uint32_t lc = tb_split(A.wbox, idx, tmp, bins, s, cnt, median);
		float llo[3], lhi[3], rlo[3], rhi[3];
		tb_range_box(A.wbox, idx, s, lc, llo, lhi);
		tb_range_box(A.wbox, idx, s + lc, cnt - lc, rlo, rhi);
		__syncwarp();
		if (lane == 0) {
			ch[j].cnt = lc;
			ch[nch].start = s + lc;
			ch[nch].cnt = cnt - lc;
			for (int a = 0; a < 3; a++) {
				ch[j].lo[a] = llo[a];
				ch[j].hi[a] = lhi[a];
				ch[nch].lo[a] = rlo[a];
				ch[nch].hi[a] = rhi[a];
			}
		}
		__syncwarp();
		nch++;
	}
	if (lane != 0)
		return;
	float cen[8][3], ncen[3], cmin[8][3], cmax[8][3];
	for (int c = 0; c < nch; c++)
		for (int a = 0; a < 3; a++)
			cen[c][a] = 0.5f * (ch[c].lo[a] + ch[c].hi[a]);
	for (int a = 0; a < 3; a++)
		ncen[a] = 0.5f * (nd.lo[a] + nd.hi[a]);
	int slot_of[8], child_at[8];
	assign_slots(nch, cen, ncen, slot_of);
	for (int s = 0; s < 8; s++)
		child_at[s] = -1;
	for (int c = 0; c < nch; c++)
		child_at[slot_of[c]] = c;
	uint32_t ninner = 0, nleaf = 0;
	for (int s = 0; s < 8; s++) {
		int c = child_at[s];
		for (int a = 0; a < 3; a++) {
			cmin[s][a] = c < 0 ? 1.0f : ch[c].lo[a];
			cmax[s][a] = c < 0 ? -1.0f : ch[c].hi[a];
		}
		if (c >= 0) {
			if (ch[c].cnt > 1u)
				ninner++;
			else
				nleaf++;
		}
	}
	nb_qnode q;
	memset(&q, 0, sizeof(q));
	quantise_node_hd(cmin, cmax, &q);
	uint32_t cb = ninner ? atomicAdd(node_ctr, ninner) : 0u;
	uint32_t ib = nleaf ? atomicAdd(item_ctr, nleaf) : 0u;
	q.child_base = cb;
	q.item_base = ib;
	uint32_t ji = 0, jl = 0;
	for (int s = 0; s < 8; s++) {
		int c = child_at[s];
		uint2 rg = make_uint2(0u, 0u);
		if (c >= 0) {
			rg = make_uint2(ch[c].start, ch[c].cnt);
			if (ch[c].cnt > 1u) {
				q.imask |= (uint8_t)(1u << s);
				uint32_t k = atomicAdd(next_cnt, 1u);
				TbNode o;
				o.start = ch[c].start;
				o.cnt = ch[c].cnt;
				o.node = cb + ji;
				o.depth = nd.depth + 1u;
				for (int a = 0; a < 3; a++) {
					o.lo[a] = ch[c].lo[a];
					o.hi[a] = ch[c].hi[a];
				}
				if (k < A.n)
					next[k] = o;
				ji++;
			} else {
				q.meta[s] = (uint8_t)(NB_META_LEAF | jl);
				if (ib + jl < A.n)
					A.irefs[ib + jl] = A.inst_base + idx[ch[c].start];
				jl++;
			}
		}
		if (nd.node < A.node_cap)
			A.ranges[8u * nd.node + s] = rg;
	}
	if (nd.node < A.node_cap && cb + ninner <= A.node_cap)
		A.nodes[nd.node] = q;
	else
		atomicExch(&A.info[2], 1u);
	atomicMax(&A.info[1], nd.depth);
}

// The build, level by level: k_tlas_init opens the root, then one
// k_tlas_level launch per tree level builds that level's open nodes, one
// warp per node over all SMs (the nodes of a level are independent), and
// k_tlas_finish records the node count and the instance order.  State
// between launches lives in global memory: the instance order (A.idx,
// A.tmp), the two level queues and the counters A.ctr: [0] nodes, [1] leaf
// items, [2] / [3] entries of queue a / b.

// Root node over all instances (one CTA), counters reset.
__global__ void __launch_bounds__(512) k_tlas_init(TbArgs A)
{
	__shared__ float part[16][6];
	const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
	float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	for (uint32_t i = tid; i < A.n; i += blockDim.x) {
		A.idx[i] = (uint16_t)i;
		float l[3], h[3];
		tb_load(A.wbox, i, l, h);
		for (int a = 0; a < 3; a++) {
			lo[a] = fminf(lo[a], l[a]);
			hi[a] = fmaxf(hi[a], h[a]);
		}
	}
	tb_warp_box(lo, hi);
	if (lane == 0)
		for (int a = 0; a < 3; a++) {
			part[warp][a] = lo[a];
			part[warp][3 + a] = hi[a];
		}
	__syncthreads();
	if (tid != 0)
		return;
	for (uint32_t w = 1; w < (blockDim.x >> 5); w++)
		for (int a = 0; a < 3; a++) {
			part[0][a] = fminf(part[0][a], part[w][a]);
			part[0][3 + a] = fmaxf(part[0][3 + a], part[w][3 + a]);
		}
	TbNode r;
	r.start = 0u;
	r.cnt = A.n;
	r.node = 0u;
	r.depth = 1u;
	for (int a = 0; a < 3; a++) {
		r.lo[a] = part[0][a];
		r.hi[a] = part[0][3 + a];
	}
	A.qa[0] = r;
	A.ctr[0] = 1u;
	A.ctr[1] = 0u;
	A.ctr[2] = A.n ? 1u : 0u;
	A.ctr[3] = 0u;
	A.info[1] = 1u;
	A.info[2] = 0u;
	if (A.n == 0u) {
		// no instances: a root without children
		float cmin[8][3], cmax[8][3];
		for (int s = 0; s < 8; s++)
			for (int a = 0; a < 3; a++) {
				cmin[s][a] = 1.0f;
				cmax[s][a] = -1.0f;
			}
		nb_qnode q;
		memset(&q, 0, sizeof(q));
		quantise_node_hd(cmin, cmax, &q);
		A.nodes[0] = q;
		for (int s = 0; s < 8; s++)
			A.ranges[s] = make_uint2(0u, 0u);
	}
}

constexpr int kTbLevelWarps = 4; // warps (open nodes in flight) per CTA

// The open nodes of one level (queue a for even levels, b for odd ones),
// one warp each; their inner children go to the other queue, whose count
// the host zeroed before the launch.
__global__ void __launch_bounds__(kTbLevelWarps * 32) k_tlas_level(
  TbArgs A, uint32_t level)
{
	__shared__ TbBin bins[kTbLevelWarps][3 * kTbBins];
	__shared__ TbChild chs[kTbLevelWarps][8];
	const uint32_t warp = threadIdx.x >> 5;
	const uint32_t cur = level & 1u;
	const TbNode *q = cur ? A.qb : A.qa;
	TbNode *nq = cur ? A.qa : A.qb;
	const uint32_t cnt = A.ctr[2u + cur];
	const uint32_t nw = gridDim.x * (uint32_t)kTbLevelWarps;
	for (uint32_t k = blockIdx.x * (uint32_t)kTbLevelWarps + warp; k < cnt;
	     k += nw)
		tb_node(A, A.idx, A.tmp, bins[warp], chs[warp], q[k], nq,
		  &A.ctr[2u + (cur ^ 1u)], &A.ctr[0], &A.ctr[1]);
}

// Node count and the instance order of the node ranges (for the refit).
__global__ void k_tlas_finish(TbArgs A)
{
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n;
	     i += gridDim.x * blockDim.x)
		A.order[i] = A.idx[i];
	if (blockIdx.x == 0 && threadIdx.x == 0)
		A.info[0] = A.ctr[0];
}

// Refit: the topology of the last build, child boxes recomputed from the
// instance ranges it recorded (one warp per node; slots, child and item
// bases, masks and leaf items stay).
__global__ void __launch_bounds__(256) k_tlas_refit(const float4 *wbox,
                                                   const uint32_t *order,
                                                   const uint2 *ranges,
                                                   const uint32_t *info,
                                                   nb_qnode *nodes)
{
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t nnodes = info[0];
	for (uint32_t nd = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	     nd < nnodes; nd += (gridDim.x * blockDim.x) >> 5) {
		float cmin[8][3], cmax[8][3];
		for (int s = 0; s < 8; s++) {
			uint2 rg = ranges[8u * nd + s];
			float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
			float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
			for (uint32_t i = lane; i < rg.y; i += 32u) {
				float l[3], h[3];
				tb_load(wbox, order[rg.x + i], l, h);
				for (int a = 0; a < 3; a++) {
					lo[a] = fminf(lo[a], l[a]);
					hi[a] = fmaxf(hi[a], h[a]);
				}
			}
			tb_warp_box(lo, hi);
			for (int a = 0; a < 3; a++) {
				cmin[s][a] = rg.y ? lo[a] : 1.0f;
				cmax[s][a] = rg.y ? hi[a] : -1.0f;
			}
		}
		if (lane == 0) {
			nb_qnode q = nodes[nd];
			quantise_node_hd(cmin, cmax, &q);
			nodes[nd] = q;
		}
	}
}

// ---------------------------------------------------------- light table --

// One emitting triangle of one instance, fixed at upload: instance, the
// object-space vertices, the three vertex normals and the emission.
struct EmitSrc {
	uint32_t inst, pad[3];
	float    v[3][3];
	float    n[3][3];
	float    emit[3];
};

// World-space light table from the device instance records (the host's
// build_lights sequence in FP64: the forward transform from the inverse of
// the world->object 3x4, edges, unit normal towards the emitting side,
// area, running CDF).  One thread: the tables hold a few dozen entries.
// A degenerate entry keeps its place with zero area (never sampled).
// out_area: the total area.
__global__ void k_light_update(const EmitSrc *src, uint32_t n,
                               const float4 *insts, float4 *lights,
                               float *out_area)
{
	if (blockIdx.x != 0 || threadIdx.x != 0)
		return;
	double total = 0.0;
	for (uint32_t i = 0; i < n; i++) {
		const EmitSrc &E = src[i];
		const float4 *ip = insts + 4u * E.inst;
		float4 r0 = ip[0], r1 = ip[1], r2 = ip[2];
		double A[9] = {r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, r2.x, r2.y, r2.z};
		double b[3] = {r0.w, r1.w, r2.w};
		double det = A[0] * (A[4] * A[8] - A[5] * A[7]) -
		  A[1] * (A[3] * A[8] - A[5] * A[6]) +
		  A[2] * (A[3] * A[7] - A[4] * A[6]);
		float L[20];
		for (int k = 0; k < 20; k++)
			L[k] = 0.0f;
		double area = 0.0;
		if (det != 0.0) {
			double I[9] = {
			  (A[4] * A[8] - A[5] * A[7]) / det,
			  (A[2] * A[7] - A[1] * A[8]) / det,
			  (A[1] * A[5] - A[2] * A[4]) / det,
			  (A[5] * A[6] - A[3] * A[8]) / det,
			  (A[0] * A[8] - A[2] * A[6]) / det,
			  (A[2] * A[3] - A[0] * A[5]) / det,
			  (A[3] * A[7] - A[4] * A[6]) / det,
			  (A[1] * A[6] - A[0] * A[7]) / det,
			  (A[0] * A[4] - A[1] * A[3]) / det};
			double w[3][3];
			for (int k = 0; k < 3; k++) {
				double x[3] = {E.v[k][0] - b[0], E.v[k][1] - b[1],
				  E.v[k][2] - b[2]};
				for (int a = 0; a < 3; a++)
					w[k][a] = I[3 * a] * x[0] + I[3 * a + 1] * x[1] +
					  I[3 * a + 2] * x[2];
			}
			double e0[3], e1[3], c[3];
			for (int a = 0; a < 3; a++) {
				e0[a] = w[1][a] - w[0][a];
				e1[a] = w[2][a] - w[0][a];
			}
			c[0] = e0[1] * e1[2] - e0[2] * e1[1];
			c[1] = e0[2] * e1[0] - e0[0] * e1[2];
			c[2] = e0[0] * e1[1] - e0[1] * e1[0];
			double len = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
			if (len != 0.0) {
				double no[3] = {
				  (double)E.n[0][0] + E.n[1][0] + E.n[2][0],
				  (double)E.n[0][1] + E.n[1][1] + E.n[2][1],
				  (double)E.n[0][2] + E.n[1][2] + E.n[2][2]};
				double nw[3] = {A[0] * no[0] + A[3] * no[1] + A[6] * no[2],
				  A[1] * no[0] + A[4] * no[1] + A[7] * no[2],
				  A[2] * no[0] + A[5] * no[1] + A[8] * no[2]};
				double sgn = (c[0] * nw[0] + c[1] * nw[1] + c[2] * nw[2])
				  < 0 ? -1.0 : 1.0;
				for (int a = 0; a < 3; a++) {
					L[a] = (float)w[0][a];
					L[3 + a] = (float)e0[a];
					L[6 + a] = (float)e1[a];
					L[9 + a] = (float)(sgn * c[a] / len);
				}
				area = 0.5 * len;
			}
		}
		for (int a = 0; a < 3; a++)
			L[12 + a] = E.emit[a];
		L[16] = (float)area;
		total += area;
		// the FP64 area rides in the last two pad words until the second
		// pass, which forms the CDF once the total is known
		unsigned long long ab = (unsigned long long)__double_as_longlong(area);
		L[18] = __uint_as_float((uint32_t)ab);
		L[19] = __uint_as_float((uint32_t)(ab >> 32));
		for (int k = 0; k < 5; k++)
			lights[5u * i + k] = make_float4(L[4 * k], L[4 * k + 1],
			  L[4 * k + 2], L[4 * k + 3]);
	}
	double run = 0.0;
	for (uint32_t i = 0; i < n; i++) {
		float4 e = lights[5u * i + 4u]; // (area, pad, area64 lo, hi)
		float4 c = lights[5u * i + 3u]; // (emit xyz, cdf)
		unsigned long long ab = (unsigned long long)__float_as_uint(e.z) |
		  ((unsigned long long)__float_as_uint(e.w) << 32);
		run += __longlong_as_double((long long)ab);
		c.w = i + 1u == n ? 1.0f : (float)(run / total);
		lights[5u * i + 3u] = c;
		lights[5u * i + 4u] = make_float4(e.x, 0.0f, 0.0f, 0.0f);
	}
	*out_area = (float)total;
}

} // namespace nb

#endif
