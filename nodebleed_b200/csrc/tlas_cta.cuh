// TLAS build in one launch of one CTA (sm_100a): a binary SAH tree over the
// instance boxes, collapsed into 8-wide nodes by cost, encoded into the GPU
// node layout (gpulayout.h) with the outputs the refit reads.
//
// The level-by-level build (tlas_build.cuh) splits each open node greedily
// into 8 children, one warp per node, and its top levels keep one warp busy
// for most of the build.  Here 1024 threads share the work:
//   1. binary tree, level by level: nodes of at least kCbBig instances are
//      split by the whole CTA one after another, smaller ones by one warp
//      each; 32 (CTA) or 16 (warp) centroid bins per axis, the children's
//      boxes taken from the bins of the winning split;
//   2. the collapse of Ylitie, Karras and Laine (HPG 2017) bottom-up: per
//      binary node and budget 1..8 the cheapest forest of 8-wide nodes, cost
//      = surface area of each 8-wide node (every leaf holds one instance, so
//      the leaves add the same to every tree and drop out);
//   3. the 8-wide nodes top-down, one warp per node on levels of up to
//      kCbWarpEmitMax nodes (the slot assignment across the warp), one
//      thread per node on wider ones, encoded as the greedy build encodes
//      them (qnode.h), with per-slot instance ranges for the refit.
// Depth: the traversal stack was sized for depth_limit TLAS levels.  SAH
// splits are kept only while a median-split finish of the subtree stays
// within binary depth 3 * depth_limit, and if the collapse by cost comes
// out deeper than the limit the tree is emitted again with the widest
// collapse (4 + 4, 2 + 2, 1 + 1 of the budget), whose node at level l holds
// binary depth 3 (l - 1): depth ceil(binary depth / 3) <= depth_limit.

#ifndef NB_TLAS_CTA_CUH
#define NB_TLAS_CTA_CUH

#include "tlas_build.cuh"

namespace nb {

constexpr int kCbThreads = 1024;
constexpr int kCbWarps = kCbThreads / 32;
constexpr int kCbBins = 32;      // bins per axis of a CTA split
constexpr int kCbWarpBins = 16;  // bins per axis of a warp split
constexpr uint32_t kCbBig = 512; // nodes split by the whole CTA
constexpr int kCbMaxLevels = 160; // binary levels (3 * depth_limit bound)
constexpr uint32_t kCbWarpEmitMax = 128; // levels emitted a warp per node

struct TcNode { // binary node
	float    lo[3], hi[3];
	uint32_t start, cnt;
	uint32_t left;  // first of its two children, or kNone
	uint32_t depth; // binary depth, root 0
};

struct TcArgs {
	TbArgs    A;      // outputs, as the level-by-level build writes them
	TcNode   *bn;     // up to 2n - 1 binary nodes
	float    *cost;   // 8 per binary node: cheapest forest of 1..8 roots
	uint8_t  *kd;     // 8 per binary node: left child's share of budget j
	uint8_t  *prev;   // per binary node, bit j: budget j + 1 no better
	                  // than budget j
	uint32_t *qa, *qb; // emission queues, 3 words per entry
};

struct TcShared {
	TbBin    cbins[3 * kCbBins];                  // CTA split
	TbBin    wbins[kCbWarps][3 * kCbWarpBins];    // warp splits
	uint32_t lv[kCbMaxLevels + 2];                // first node of each level
	uint32_t wsum[kCbWarps];                      // block scan
	float    red[kCbWarps][6];                    // block box reduction
	uint32_t nnodes, nitems, nout, qn, qn2, maxd, over, nlev, stot;
	int      axis, kbest;
	uint32_t lcnt;
	float    lbox[6], rbox[6];
	uint32_t big[8];                              // a level's CTA splits
};

__device__ __forceinline__ uint32_t tc_ceil_log2(uint32_t x)
{
	return x <= 1u ? 0u : 32u - (uint32_t)__clz(x - 1u);
}

__device__ __forceinline__ int tc_bin(float c, float cmn, float scale,
                                      int nb)
{
	int b = (int)((c - cmn) * scale);
	return b < 0 ? 0 : (b > nb - 1 ? nb - 1 : b);
}

__device__ __forceinline__ void tc_bins_clear(TbBin *b, int n, uint32_t t,
                                              uint32_t nt)
{
	for (uint32_t k = t; k < (uint32_t)n; k += nt) {
		b[k].cnt = 0u;
		for (int a = 0; a < 3; a++) {
			b[k].lo[a] = tb_ord(FLT_MAX);
			b[k].hi[a] = tb_ord(-FLT_MAX);
		}
	}
}

// Add this lane's item (box l/h, bin `key` in b, or key < 0: none) to the
// shared bins.  (Combining the lanes of a bin first, by a match and six
// group reductions, measured about 8 times slower than these atomics.)
__device__ __forceinline__ void tc_bin_add(TbBin *b, int key,
                                           const float l[3],
                                           const float h[3])
{
	if (key < 0)
		return;
	TbBin *t = b + key;
	atomicAdd(&t->cnt, 1u);
	for (int d = 0; d < 3; d++) {
		atomicMin(&t->lo[d], tb_ord(l[d]));
		atomicMax(&t->hi[d], tb_ord(h[d]));
	}
}

// SAH sweep of axis a over nb bins: best "bins 0..k left" (cost, k), k = -1
// when no boundary separates items.  One lane.
__device__ __forceinline__ void tc_sweep(const TbBin *B, int nb, float *best,
                                         int *bk)
{
	float rarea[kCbBins];
	uint32_t rcnt[kCbBins];
	float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
	float rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	uint32_t rc = 0;
	for (int k = nb - 1; k >= 1; k--) {
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
	*best = FLT_MAX;
	*bk = -1;
	for (int k = 0; k < nb - 1; k++) {
		lc += B[k].cnt;
		for (int d = 0; d < 3; d++) {
			llo[d] = fminf(llo[d], tb_unord(B[k].lo[d]));
			lhi[d] = fmaxf(lhi[d], tb_unord(B[k].hi[d]));
		}
		if (lc == 0u || rcnt[k + 1] == 0u)
			continue;
		float cost = tb_area(llo, lhi) * (float)lc +
		  rarea[k + 1] * (float)rcnt[k + 1];
		if (cost < *best) {
			*best = cost;
			*bk = k;
		}
	}
}

// Boxes and left count of "bins 0..k left" on one axis.  One lane.
__device__ __forceinline__ void tc_split_boxes(const TbBin *B, int nb, int k,
                                               float lb[6], float rb[6],
                                               uint32_t *lcnt)
{
	for (int d = 0; d < 3; d++) {
		lb[d] = rb[d] = FLT_MAX;
		lb[3 + d] = rb[3 + d] = -FLT_MAX;
	}
	uint32_t lc = 0;
	for (int j = 0; j < nb; j++) {
		float *t = j <= k ? lb : rb;
		if (j <= k)
			lc += B[j].cnt;
		for (int d = 0; d < 3; d++) {
			t[d] = fminf(t[d], tb_unord(B[j].lo[d]));
			t[3 + d] = fmaxf(t[3 + d], tb_unord(B[j].hi[d]));
		}
	}
	*lcnt = lc;
}


// Children c0, c0 + 1 of binary node q over [start, start + lc) and the
// rest, boxes lb / rb (one thread).
__device__ __forceinline__ void tc_make_children(const TcArgs &T,
                                                 uint32_t *nnodes, uint32_t q,
                                                 const TcNode &nd, uint32_t lc,
                                                 const float lb[6],
                                                 const float rb[6])
{
	uint32_t c0 = atomicAdd(nnodes, 2u);
	TcNode l, r;
	for (int d = 0; d < 3; d++) {
		l.lo[d] = lb[d];
		l.hi[d] = lb[3 + d];
		r.lo[d] = rb[d];
		r.hi[d] = rb[3 + d];
	}
	l.start = nd.start;
	l.cnt = lc;
	r.start = nd.start + lc;
	r.cnt = nd.cnt - lc;
	l.left = r.left = kNone;
	l.depth = r.depth = nd.depth + 1u;
	T.bn[c0] = l;
	T.bn[c0 + 1u] = r;
	T.bn[q].left = c0;
}

// SAH over the 16-bin axes of B with the whole warp: in each of two passes
// a half-warp scans one axis's bins (lane & 15 = bin) from both ends, and the
// lane of split "bins 0..k left" prices it; the cheapest split (lowest axis,
// then lowest k, on equal cost) wins.  Returns its axis (-1: none) and, in
// every lane, its bin k, boxes and left count.
__device__ __forceinline__ int tc_sweep_warp(const TbBin *B,
                                             const float scale[3], int *kbest,
                                             float lb[6], float rb[6],
                                             uint32_t *lcnt)
{
	const uint32_t lane = threadIdx.x & 31u, k = lane & 15u;
	int win_axis = -1;
	uint32_t win_bits = 0xffffffffu;
	for (int pass = 0; pass < 2; pass++) {
		int axis = pass == 0 ? (int)(lane >> 4) : 2;
		bool valid = (pass == 0 || lane < 16u) && scale[axis] > 0.0f;
		uint32_t c = 0;
		float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
		float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
		if (valid) {
			const TbBin &b = B[axis * kCbWarpBins + (int)k];
			c = b.cnt;
			for (int d = 0; d < 3; d++) {
				lo[d] = tb_unord(b.lo[d]);
				hi[d] = tb_unord(b.hi[d]);
			}
		}
		// inclusive prefix (left of and at bin k) and suffix (k and right)
		uint32_t lc = c, rc = c;
		float llo[3], lhi[3], rlo[3], rhi[3];
		for (int d = 0; d < 3; d++) {
			llo[d] = rlo[d] = lo[d];
			lhi[d] = rhi[d] = hi[d];
		}
		for (int o = 1; o < 16; o <<= 1) {
			uint32_t xc = __shfl_up_sync(kFull, lc, o, 16);
			uint32_t yc = __shfl_down_sync(kFull, rc, o, 16);
			float xl[3], xh[3], yl[3], yh[3];
			for (int d = 0; d < 3; d++) {
				xl[d] = __shfl_up_sync(kFull, llo[d], o, 16);
				xh[d] = __shfl_up_sync(kFull, lhi[d], o, 16);
				yl[d] = __shfl_down_sync(kFull, rlo[d], o, 16);
				yh[d] = __shfl_down_sync(kFull, rhi[d], o, 16);
			}
			if (k >= (uint32_t)o) {
				lc += xc;
				for (int d = 0; d < 3; d++) {
					llo[d] = fminf(llo[d], xl[d]);
					lhi[d] = fmaxf(lhi[d], xh[d]);
				}
			}
			if (k + (uint32_t)o < 16u) {
				rc += yc;
				for (int d = 0; d < 3; d++) {
					rlo[d] = fminf(rlo[d], yl[d]);
					rhi[d] = fmaxf(rhi[d], yh[d]);
				}
			}
		}
		// the right side of split k starts at bin k + 1
		uint32_t rc1 = __shfl_down_sync(kFull, rc, 1, 16);
		float r1l[3], r1h[3];
		for (int d = 0; d < 3; d++) {
			r1l[d] = __shfl_down_sync(kFull, rlo[d], 1, 16);
			r1h[d] = __shfl_down_sync(kFull, rhi[d], 1, 16);
		}
		bool ok = valid && k < 15u && lc > 0u && rc1 > 0u;
		float cost = ok ? tb_area(llo, lhi) * (float)lc +
		  tb_area(r1l, r1h) * (float)rc1 : FLT_MAX;
		// cost >= 0: its bits order as unsigned integers
		uint32_t bits = ok ? __float_as_uint(cost) : 0xffffffffu;
		uint32_t mb = __reduce_min_sync(kFull, bits);
		uint32_t who = __reduce_min_sync(kFull, ok && bits == mb ?
		  (uint32_t)axis * 16u + k : 0xffffffffu);
		if (who != 0xffffffffu && mb < win_bits) {
			win_bits = mb;
			win_axis = (int)(who >> 4);
			uint32_t src = pass == 0 ? who : (who & 15u);
			*kbest = (int)(who & 15u);
			*lcnt = __shfl_sync(kFull, lc, src);
			for (int d = 0; d < 3; d++) {
				lb[d] = __shfl_sync(kFull, llo[d], src);
				lb[3 + d] = __shfl_sync(kFull, lhi[d], src);
				rb[d] = __shfl_sync(kFull, r1l[d], src);
				rb[3 + d] = __shfl_sync(kFull, r1h[d], src);
			}
		}
	}
	return win_axis;
}

// Split binary node q (2 <= cnt < kCbBig) with one warp: SAH over 16
// centroid bins per axis when `sah`, else (or when no bin boundary
// separates the centroids) the first cnt / 2 in index order go left.
__device__ void tc_warp_split(const TcArgs &T, TcShared &S, uint32_t q,
                              bool sah)
{
	const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
	const float4 *wbox = T.A.wbox;
	uint16_t *idx = T.A.idx, *tmp = T.A.tmp;
	const TcNode nd = T.bn[q];
	const uint32_t s = nd.start, cnt = nd.cnt;
	int axis = -1, kbest = -1;
	float cmn[3], scale[3], lb[6], rb[6];
	uint32_t lc = cnt / 2u;
	if (cnt == 2u) {
		// one instance on each side, whatever the heuristic
		if (lane == 0) {
			float l[3], h[3];
			tb_load(wbox, idx[s], l, h);
			for (int d = 0; d < 3; d++) {
				lb[d] = l[d];
				lb[3 + d] = h[d];
			}
			tb_load(wbox, idx[s + 1u], l, h);
			for (int d = 0; d < 3; d++) {
				rb[d] = l[d];
				rb[3 + d] = h[d];
			}
			tc_make_children(T, &S.nnodes, q, nd, 1u, lb, rb);
		}
		__syncwarp();
		return;
	}
	if (sah) {
		float cmx[3];
		for (int a = 0; a < 3; a++) {
			cmn[a] = FLT_MAX;
			cmx[a] = -FLT_MAX;
		}
		for (uint32_t i = lane; i < cnt; i += 32u) {
			float l[3], h[3];
			tb_load(wbox, idx[s + i], l, h);
			for (int a = 0; a < 3; a++) {
				float c = 0.5f * (l[a] + h[a]);
				cmn[a] = fminf(cmn[a], c);
				cmx[a] = fmaxf(cmx[a], c);
			}
		}
		tb_warp_box(cmn, cmx);
		for (int a = 0; a < 3; a++) {
			float ext = cmx[a] - cmn[a];
			scale[a] = ext > 0.0f ? (float)kCbWarpBins / ext : 0.0f;
		}
		TbBin *B = S.wbins[warp];
		tc_bins_clear(B, 3 * kCbWarpBins, lane, 32u);
		__syncwarp();
		for (uint32_t i0 = 0; i0 < cnt; i0 += 32u) {
			uint32_t i = i0 + lane;
			float l[3] = {0, 0, 0}, h[3] = {0, 0, 0};
			if (i < cnt)
				tb_load(wbox, idx[s + i], l, h);
			for (int a = 0; a < 3; a++) {
				int key = -1;
				if (i < cnt && scale[a] > 0.0f)
					key = a * kCbWarpBins + tc_bin(0.5f * (l[a] + h[a]),
					  cmn[a], scale[a], kCbWarpBins);
				tc_bin_add(B, key, l, h);
			}
		}
		__syncwarp();
		axis = tc_sweep_warp(B, scale, &kbest, lb, rb, &lc);
	}
	if (axis >= 0) {
		// stable partition through tmp: left items first
		uint32_t pl = 0, pr = lc;
		for (uint32_t i0 = 0; i0 < cnt; i0 += 32u) {
			uint32_t i = i0 + lane;
			bool live = i < cnt, left = false;
			uint16_t v = 0;
			if (live) {
				v = idx[s + i];
				float l[3], h[3];
				tb_load(wbox, v, l, h);
				left = tc_bin(0.5f * (l[axis] + h[axis]), cmn[axis],
				  scale[axis], kCbWarpBins) <= kbest;
			}
			uint32_t ml = __ballot_sync(kFull, live && left);
			uint32_t mr = __ballot_sync(kFull, live && !left);
			uint32_t below = (1u << lane) - 1u;
			if (live)
				tmp[s + (left ? pl + __popc(ml & below) :
				  pr + __popc(mr & below))] = v;
			pl += __popc(ml);
			pr += __popc(mr);
		}
		__syncwarp();
		for (uint32_t i = lane; i < cnt; i += 32u)
			idx[s + i] = tmp[s + i];
		__syncwarp();
	} else {
		lc = cnt / 2u;
		float l[3], h[3];
		tb_range_box(wbox, idx, s, lc, l, h);
		for (int d = 0; d < 3; d++) {
			lb[d] = l[d];
			lb[3 + d] = h[d];
		}
		tb_range_box(wbox, idx, s + lc, cnt - lc, l, h);
		for (int d = 0; d < 3; d++) {
			rb[d] = l[d];
			rb[3 + d] = h[d];
		}
	}
	if (lane == 0)
		tc_make_children(T, &S.nnodes, q, nd, lc, lb, rb);
	__syncwarp();
}

// Box of idx[start, start + cnt) reduced over the CTA into S.red[0].
__device__ void tc_cta_range_box(const TcArgs &T, TcShared &S, uint32_t start,
                                 uint32_t cnt, float out[6])
{
	const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
	float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	for (uint32_t i = tid; i < cnt; i += kCbThreads) {
		float l[3], h[3];
		tb_load(T.A.wbox, T.A.idx[start + i], l, h);
		for (int a = 0; a < 3; a++) {
			lo[a] = fminf(lo[a], l[a]);
			hi[a] = fmaxf(hi[a], h[a]);
		}
	}
	tb_warp_box(lo, hi);
	if (lane == 0)
		for (int a = 0; a < 3; a++) {
			S.red[warp][a] = lo[a];
			S.red[warp][3 + a] = hi[a];
		}
	__syncthreads();
	if (warp == 0) {
		for (int a = 0; a < 3; a++) {
			lo[a] = S.red[lane][a];
			hi[a] = S.red[lane][3 + a];
		}
		tb_warp_box(lo, hi);
	}
	__syncthreads();
	if (tid == 0)
		for (int a = 0; a < 3; a++) {
			S.red[0][a] = lo[a];
			S.red[0][3 + a] = hi[a];
		}
	__syncthreads();
	for (int a = 0; a < 6; a++)
		out[a] = S.red[0][a];
	__syncthreads();
}

// Split binary node q (cnt >= kCbBig) with the whole CTA: SAH over 32
// centroid bins per axis when `sah`, else (or when no bin boundary
// separates the centroids) the first cnt / 2 in index order go left.
__device__ void tc_cta_split(const TcArgs &T, TcShared &S, uint32_t q,
                             bool sah)
{
	const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	const float4 *wbox = T.A.wbox;
	uint16_t *idx = T.A.idx, *tmp = T.A.tmp;
	const TcNode nd = T.bn[q];
	const uint32_t s = nd.start, cnt = nd.cnt;
	float cmn[3], cmx[3], scale[3];
	for (int a = 0; a < 3; a++) {
		cmn[a] = FLT_MAX;
		cmx[a] = -FLT_MAX;
	}
	for (uint32_t i = tid; i < cnt; i += kCbThreads) {
		float l[3], h[3];
		tb_load(wbox, idx[s + i], l, h);
		for (int a = 0; a < 3; a++) {
			float c = 0.5f * (l[a] + h[a]);
			cmn[a] = fminf(cmn[a], c);
			cmx[a] = fmaxf(cmx[a], c);
		}
	}
	tb_warp_box(cmn, cmx);
	if (lane == 0)
		for (int a = 0; a < 3; a++) {
			S.red[warp][a] = cmn[a];
			S.red[warp][3 + a] = cmx[a];
		}
	tc_bins_clear(S.cbins, 3 * kCbBins, tid, kCbThreads);
	if (tid == 0)
		S.axis = -1;
	__syncthreads();
	if (warp == 0) {
		for (int a = 0; a < 3; a++) {
			cmn[a] = S.red[lane][a];
			cmx[a] = S.red[lane][3 + a];
		}
		tb_warp_box(cmn, cmx);
	}
	__syncthreads();
	if (tid == 0)
		for (int a = 0; a < 3; a++) {
			S.red[0][a] = cmn[a];
			S.red[0][3 + a] = cmx[a];
		}
	__syncthreads();
	for (int a = 0; a < 3; a++) {
		cmn[a] = S.red[0][a];
		float ext = S.red[0][3 + a] - cmn[a];
		scale[a] = sah && ext > 0.0f ? (float)kCbBins / ext : 0.0f;
	}
	for (uint32_t i0 = 0; i0 < cnt; i0 += kCbThreads) {
		uint32_t i = i0 + tid;
		float l[3] = {0, 0, 0}, h[3] = {0, 0, 0};
		if (i < cnt)
			tb_load(wbox, idx[s + i], l, h);
		for (int a = 0; a < 3; a++) {
			int key = -1;
			if (i < cnt && scale[a] > 0.0f)
				key = a * kCbBins + tc_bin(0.5f * (l[a] + h[a]), cmn[a],
				  scale[a], kCbBins);
			tc_bin_add(S.cbins, key, l, h);
		}
	}
	__syncthreads();
	if (warp == 0) {
		float best = FLT_MAX;
		int bk = -1;
		if (lane < 3u && scale[lane] > 0.0f)
			tc_sweep(S.cbins + lane * kCbBins, kCbBins, &best, &bk);
		float b0 = __shfl_sync(kFull, best, 0);
		float b1 = __shfl_sync(kFull, best, 1);
		float b2 = __shfl_sync(kFull, best, 2);
		int k0 = __shfl_sync(kFull, bk, 0), k1 = __shfl_sync(kFull, bk, 1);
		int k2 = __shfl_sync(kFull, bk, 2);
		int axis = -1, kbest = -1;
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
		if (lane == 0 && axis >= 0) {
			S.axis = axis;
			S.kbest = kbest;
			tc_split_boxes(S.cbins + axis * kCbBins, kCbBins, kbest, S.lbox,
			  S.rbox, &S.lcnt);
		}
	}
	__syncthreads();
	const int axis = S.axis, kbest = S.kbest;
	if (axis >= 0) {
		// stable partition through tmp, rounds of kCbThreads items: each
		// warp's left / right counts packed into one word (<= 32 each) and
		// scanned by warp 0
		uint32_t bl = 0, br = S.lcnt;
		for (uint32_t i0 = 0; i0 < cnt; i0 += kCbThreads) {
			uint32_t i = i0 + tid;
			bool live = i < cnt, left = false;
			uint16_t v = 0;
			if (live) {
				v = idx[s + i];
				float l[3], h[3];
				tb_load(wbox, v, l, h);
				left = tc_bin(0.5f * (l[axis] + h[axis]), cmn[axis],
				  scale[axis], kCbBins) <= kbest;
			}
			uint32_t ml = __ballot_sync(kFull, live && left);
			uint32_t mr = __ballot_sync(kFull, live && !left);
			if (lane == 0)
				S.wsum[warp] = (uint32_t)__popc(ml) |
				  ((uint32_t)__popc(mr) << 16);
			__syncthreads();
			if (warp == 0) {
				uint32_t x = S.wsum[lane], incl = x;
				for (int o = 1; o < 32; o <<= 1) {
					uint32_t y = __shfl_up_sync(kFull, incl, o);
					if (lane >= (uint32_t)o)
						incl += y;
				}
				S.wsum[lane] = incl - x;
				if (lane == 31u)
					S.stot = incl;
			}
			__syncthreads();
			uint32_t pre = S.wsum[warp], below = (1u << lane) - 1u;
			if (live)
				tmp[s + (left ? bl + (pre & 0xffffu) + __popc(ml & below) :
				  br + (pre >> 16) + __popc(mr & below))] = v;
			bl += S.stot & 0xffffu;
			br += S.stot >> 16;
			__syncthreads();
		}
		for (uint32_t i = tid; i < cnt; i += kCbThreads)
			idx[s + i] = tmp[s + i];
		__syncthreads();
		if (tid == 0)
			tc_make_children(T, &S.nnodes, q, nd, S.lcnt, S.lbox, S.rbox);
	} else {
		uint32_t lc = cnt / 2u;
		float lb[6], rb[6];
		tc_cta_range_box(T, S, s, lc, lb);
		tc_cta_range_box(T, S, s + lc, cnt - lc, rb);
		if (tid == 0)
			tc_make_children(T, &S.nnodes, q, nd, lc, lb, rb);
	}
	__syncthreads();
}

// Collapse tables of binary node q from its children's (one thread).
// Leaves cost nothing (each holds one instance, at every budget); an inner
// node as an 8-wide node costs its area plus its best 8-root forest.
__device__ void tc_collapse_node(const TcArgs &T, uint32_t q)
{
	const TcNode b = T.bn[q];
	float *C = T.cost + 8u * q;
	if (b.left == kNone) {
		for (int i = 0; i < 8; i++)
			C[i] = 0.0f;
		T.prev[q] = 0xfe;
		return;
	}
	const float *L = T.cost + 8u * b.left;
	const float *R = T.cost + 8u * (b.left + 1u);
	float dist[9];
	for (int j = 2; j <= 8; j++) {
		float best = FLT_MAX;
		int bk = 1;
		for (int k = 1; k < j; k++) {
			float v = L[k - 1] + R[j - k - 1];
			if (v < best) {
				best = v;
				bk = k;
			}
		}
		dist[j] = best;
		T.kd[8u * q + (uint32_t)(j - 1)] = (uint8_t)bk;
	}
	C[0] = tb_area(b.lo, b.hi) + dist[8];
	uint8_t pv = 0;
	for (int i = 2; i <= 8; i++) {
		if (dist[i] < C[i - 2]) {
			C[i - 1] = dist[i];
		} else {
			C[i - 1] = C[i - 2];
			pv |= (uint8_t)(1u << (i - 1));
		}
	}
	T.prev[q] = pv;
}

// The widest collapse of binary node q: budget j split evenly between the
// children, all of it to the inner one next to a leaf (one thread).
__device__ void tc_widest_node(const TcArgs &T, uint32_t q)
{
	const TcNode b = T.bn[q];
	T.prev[q] = 0;
	if (b.left == kNone)
		return;
	bool ll = T.bn[b.left].left == kNone;
	bool rl = T.bn[b.left + 1u].left == kNone;
	for (uint32_t j = 2; j <= 8; j++)
		T.kd[8u * q + j - 1u] = (uint8_t)(ll ? 1u : (rl ? j - 1u : j / 2u));
}

// assign_slots (qnode.h) with the whole warp: each lane scores two of the
// 64 (child, slot) pairs, and each greedy round takes the best remaining
// pair by a warp argmax (the lowest pair index c * 8 + s on equal scores,
// the order in which the sequential loop keeps the first maximum), so every
// lane gets the sequential assignment.  Scores are clamped to -FLT_MAX
// (NaN included): a total order on which all lanes agree, and the lowest
// free pair when nothing beats -FLT_MAX, as in the sequential loop.
__device__ void tc_assign_slots_warp(int nchild, const float cen[8][3],
                                     const float nc[3], int slot_of[8])
{
	const int lane = (int)(threadIdx.x & 31u);
	float sc[2];
	bool ok[2];
	for (int h = 0; h < 2; h++) {
		int p = lane + 32 * h, c = p >> 3, sl = p & 7;
		ok[h] = c < nchild;
		float v = 0.0f;
		if (ok[h])
			for (int a = 0; a < 3; a++)
				v += (cen[c][a] - nc[a]) * ((sl >> a) & 1 ? 1.0f : -1.0f);
		sc[h] = fmaxf(v, -FLT_MAX);
	}
	for (int i = 0; i < 8; i++)
		slot_of[i] = -1;
	for (int round = 0; round < nchild; round++) {
		float bv = -FLT_MAX;
		int bi = -1;
		for (int h = 0; h < 2; h++)
			if (ok[h] && (bi < 0 || sc[h] > bv)) {
				bv = sc[h];
				bi = lane + 32 * h;
			}
		for (int o = 16; o > 0; o >>= 1) {
			float ov = __shfl_xor_sync(kFull, bv, o);
			int oi = __shfl_xor_sync(kFull, bi, o);
			if (oi >= 0 && (bi < 0 || ov > bv || (ov == bv && oi < bi))) {
				bv = ov;
				bi = oi;
			}
		}
		int bc = bi >> 3, bs = bi & 7;
		slot_of[bc] = bs;
		for (int h = 0; h < 2; h++) {
			int p = lane + 32 * h;
			if ((p >> 3) == bc || (p & 7) == bs)
				ok[h] = false;
		}
	}
}

// Encode the 8-wide node `out` for binary node q at depth `depth`: its
// children from the collapse tables, slots, quantised boxes, leaf items,
// refit ranges; inner children go to the next queue.  One thread, or with
// `warp` the whole warp: every lane finds the children, the warp assigns
// the slots, lane 0 encodes and writes.
__device__ void tc_emit_node(const TcArgs &T, TcShared &S, uint32_t q,
                             uint32_t out, uint32_t depth, uint32_t *nextq,
                             bool warp)
{
	const TbArgs &A = T.A;
	const TcNode nd = T.bn[q];
	uint32_t kids[8];
	int nk = 0;
	if (nd.left == kNone) {
		kids[nk++] = q; // a single instance
	} else {
		uint32_t st[16][2];
		int sp = 0;
		uint32_t k = T.kd[8u * q + 7u];
		st[sp][0] = nd.left + 1u;
		st[sp++][1] = 8u - k;
		st[sp][0] = nd.left;
		st[sp++][1] = k;
		while (sp > 0) {
			sp--;
			uint32_t x = st[sp][0], j = st[sp][1];
			const uint32_t xl = T.bn[x].left;
			if (xl != kNone) {
				uint8_t pv = T.prev[x];
				while (j >= 2u && ((pv >> (j - 1u)) & 1u))
					j--;
			}
			if (xl == kNone || j <= 1u || sp >= 14) {
				if (nk < 8)
					kids[nk++] = x;
				else
					atomicExch(&S.over, 1u);
				continue;
			}
			uint32_t kk = T.kd[8u * x + j - 1u];
			st[sp][0] = xl + 1u;
			st[sp++][1] = j - kk;
			st[sp][0] = xl;
			st[sp++][1] = kk;
		}
	}
	float cen[8][3], ncen[3], cmin[8][3], cmax[8][3];
	for (int c = 0; c < nk; c++)
		for (int a = 0; a < 3; a++) {
			const TcNode &b = T.bn[kids[c]];
			cen[c][a] = 0.5f * (b.lo[a] + b.hi[a]);
		}
	for (int a = 0; a < 3; a++)
		ncen[a] = 0.5f * (nd.lo[a] + nd.hi[a]);
	int slot_of[8], child_at[8];
	if (warp) {
		tc_assign_slots_warp(nk, cen, ncen, slot_of);
		if ((threadIdx.x & 31u) != 0u)
			return;
	} else {
		assign_slots(nk, cen, ncen, slot_of);
	}
	for (int s = 0; s < 8; s++)
		child_at[s] = -1;
	for (int c = 0; c < nk; c++)
		child_at[slot_of[c]] = c;
	uint32_t ninner = 0, nleaf = 0;
	for (int s = 0; s < 8; s++) {
		int c = child_at[s];
		for (int a = 0; a < 3; a++) {
			cmin[s][a] = c < 0 ? 1.0f : T.bn[kids[c]].lo[a];
			cmax[s][a] = c < 0 ? -1.0f : T.bn[kids[c]].hi[a];
		}
		if (c >= 0) {
			if (T.bn[kids[c]].left != kNone)
				ninner++;
			else
				nleaf++;
		}
	}
	nb_qnode qn;
	memset(&qn, 0, sizeof(qn));
	quantise_node_hd(cmin, cmax, &qn);
	uint32_t cb = ninner ? atomicAdd(&S.nout, ninner) : 0u;
	uint32_t ib = nleaf ? atomicAdd(&S.nitems, nleaf) : 0u;
	qn.child_base = cb;
	qn.item_base = ib;
	uint32_t ji = 0, jl = 0;
	for (int s = 0; s < 8; s++) {
		int c = child_at[s];
		uint2 rg = make_uint2(0u, 0u);
		if (c >= 0) {
			const TcNode b = T.bn[kids[c]];
			rg = make_uint2(b.start, b.cnt);
			if (b.left != kNone) {
				qn.imask |= (uint8_t)(1u << s);
				uint32_t e = atomicAdd(&S.qn2, 1u);
				if (e < A.n) {
					nextq[3u * e] = kids[c];
					nextq[3u * e + 1u] = cb + ji;
					nextq[3u * e + 2u] = depth + 1u;
				} else {
					atomicExch(&S.over, 1u);
				}
				ji++;
			} else {
				qn.meta[s] = (uint8_t)(NB_META_LEAF | jl);
				if (ib + jl < A.n)
					A.irefs[ib + jl] = A.inst_base + A.idx[b.start];
				jl++;
			}
		}
		if (out < A.node_cap)
			A.ranges[8u * out + s] = rg;
	}
	if (out < A.node_cap && cb + ninner <= A.node_cap)
		A.nodes[out] = qn;
	else
		atomicExch(&S.over, 1u);
	atomicMax(&S.maxd, depth);
}

// Emit the whole 8-wide tree from the collapse tables (whole CTA).
__device__ void tc_emit(const TcArgs &T, TcShared &S)
{
	const uint32_t tid = threadIdx.x;
	if (tid == 0) {
		S.nout = 1u;
		S.nitems = 0u;
		S.maxd = 1u;
		S.qn = 1u;
		S.qn2 = 0u;
		T.qa[0] = 0u;
		T.qa[1] = 0u;
		T.qa[2] = 1u;
	}
	__syncthreads();
	uint32_t *cur = T.qa, *nxt = T.qb;
	for (;;) {
		uint32_t nq = S.qn;
		if (nq == 0u)
			break;
		// A warp per node while that takes a few rounds of the 32 warps;
		// on wider levels lane 0's serial encoding would queue up, and a
		// thread per node is faster.
		if (nq <= kCbWarpEmitMax) {
			for (uint32_t e = tid >> 5; e < nq; e += (uint32_t)kCbWarps)
				tc_emit_node(T, S, cur[3u * e], cur[3u * e + 1u],
				  cur[3u * e + 2u], nxt, true);
		} else {
			for (uint32_t e = tid; e < nq; e += (uint32_t)kCbThreads)
				tc_emit_node(T, S, cur[3u * e], cur[3u * e + 1u],
				  cur[3u * e + 2u], nxt, false);
		}
		__syncthreads();
		if (tid == 0) {
			S.qn = S.qn2;
			S.qn2 = 0u;
		}
		__syncthreads();
		uint32_t *t = cur;
		cur = nxt;
		nxt = t;
	}
}

// Dynamic shared memory of the build over n instances: their boxes (two
// float4 each, as in wbox) and the two instance orders.
__host__ __device__ inline size_t tc_dyn_smem(uint32_t n)
{
	return (size_t)n * 32u + (((size_t)n * 4u + 15u) & ~(size_t)15u);
}

// The whole build (one CTA of kCbThreads threads).  The instance boxes and
// orders live in shared memory for the build; the world boxes in global
// memory stay as they are for the refit.
__global__ void __launch_bounds__(kCbThreads, 1) k_tlas_cta(TcArgs Tg)
{
	__shared__ TcShared S;
	extern __shared__ float4 tc_dyn[];
	TcArgs T = Tg;
	{
		float4 *sbox = tc_dyn;
		uint16_t *sidx = reinterpret_cast<uint16_t *>(tc_dyn + 2u * Tg.A.n);
		for (uint32_t i = threadIdx.x; i < 2u * Tg.A.n; i += kCbThreads)
			sbox[i] = Tg.A.wbox[i];
		T.A.wbox = sbox;
		T.A.idx = sidx;
		T.A.tmp = sidx + Tg.A.n;
	}
	const TbArgs &A = T.A;
	const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
	const uint32_t n = A.n;
	if (n == 0u) {
		if (tid == 0) {
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
			A.info[0] = 1u;
			A.info[1] = 1u;
			A.info[2] = 0u;
		}
		return;
	}
	const uint32_t cap = 3u * A.depth_limit; // deepest binary leaf allowed
	for (uint32_t i = tid; i < n; i += kCbThreads)
		A.idx[i] = (uint16_t)i;
	__syncthreads(); // the boxes copied above
	if (tid == 0) {
		S.over = 0u;
		S.nnodes = 1u;
		S.lv[0] = 0u;
		S.lv[1] = 1u;
	}
	__syncthreads();
	float rb[6];
	tc_cta_range_box(T, S, 0u, n, rb);
	if (tid == 0) {
		TcNode r;
		for (int a = 0; a < 3; a++) {
			r.lo[a] = rb[a];
			r.hi[a] = rb[3 + a];
		}
		r.start = 0u;
		r.cnt = n;
		r.left = kNone;
		r.depth = 0u;
		T.bn[0] = r;
	}
	__syncthreads();
	// 1. binary tree, level by level
	uint32_t nlev = 0;
	for (uint32_t L = 0; L < (uint32_t)kCbMaxLevels; L++) {
		const uint32_t b = S.lv[L], e = S.lv[L + 1];
		if (b == e)
			break;
		nlev = L + 1u;
		if (tid == 0)
			S.qn = 0u;
		__syncthreads();
		for (uint32_t q = b + tid; q < e; q += kCbThreads)
			if (T.bn[q].cnt >= kCbBig) {
				uint32_t k = atomicAdd(&S.qn, 1u);
				if (k < 8u)
					S.big[k] = q;
			}
		__syncthreads();
		const uint32_t nbig = min(S.qn, 8u);
		for (uint32_t k = 0; k < nbig; k++) {
			const uint32_t q = S.big[k];
			const TcNode nd = T.bn[q];
			tc_cta_split(T, S, q,
			  nd.depth + tc_ceil_log2(nd.cnt) + 1u <= cap);
		}
		for (uint32_t q = b + warp; q < e; q += (uint32_t)kCbWarps) {
			const TcNode nd = T.bn[q];
			if (nd.cnt >= 2u && nd.cnt < kCbBig)
				tc_warp_split(T, S, q,
				  nd.depth + tc_ceil_log2(nd.cnt) + 1u <= cap);
		}
		__syncthreads();
		if (tid == 0)
			S.lv[L + 2] = S.nnodes;
		__syncthreads();
	}
	if (tid == 0 && S.lv[nlev] != S.lv[nlev + 1])
		S.over = 1u; // more levels than kCbMaxLevels (cannot happen)
	// 2. collapse tables, deepest level first
	for (int L = (int)nlev - 1; L >= 0; L--) {
		for (uint32_t q = S.lv[L] + tid; q < S.lv[L + 1]; q += kCbThreads)
			tc_collapse_node(T, q);
		__syncthreads();
	}
	// 3. the 8-wide tree; the widest collapse if the one by cost is too deep
	tc_emit(T, S);
	if (S.maxd > A.depth_limit) {
		for (uint32_t q = tid; q < S.lv[nlev]; q += kCbThreads)
			tc_widest_node(T, q);
		__syncthreads();
		tc_emit(T, S);
	}
	for (uint32_t i = tid; i < n; i += kCbThreads)
		A.order[i] = A.idx[i];
	if (tid == 0) {
		A.info[0] = S.nout;
		A.info[1] = S.maxd;
		A.info[2] = S.over | (S.maxd > A.depth_limit ? 1u : 0u);
	}
	(void)lane;
}

} // namespace nb

#endif
