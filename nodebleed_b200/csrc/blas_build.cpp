// BLAS built for the GPU traversal, as an alternative to converting the
// reference's BVH8 (rend.c:458-709) node for node.
//
// A binary BVH is built top-down with the surface area heuristic down to one
// triangle per leaf: a full sweep over the sorted centroids for ranges of at
// most kSweepMax triangles, kBins bins over the centroid bounds above that.
// It is then collapsed into 8-wide nodes by the dynamic program of Ylitie,
// Karras and Laine (HPG 2017, "Efficient incoherent ray traversal on GPUs
// through compressed wide BVHs"): for every binary node n and every budget
// i = 1..8 it finds the cheapest way to represent n's subtree by at most i
// subtrees, each a leaf of at most 4 triangles (cost c_tri * A * count) or an
// 8-wide node (cost c_node * A plus its own children), A being the box's
// surface area.  The 8-wide nodes are encoded exactly like the converted ones
// (qnode.h: slot order by octant, conservative 8-bit planes), so the device
// traversal reads either tree.
//
// The closest hit of a ray does not depend on the tree: the triangle test is
// the same and boxes only prune.  Among triangles hit at exactly the same t
// the one found first wins, and that can differ from the reference's tree.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

#include "layout.hpp"
#include "qnode.h"

namespace nb {

namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kSweepMax = 128;
constexpr int kBins = 32;
constexpr int kLeafMax = 4; // items per leaf child (2-bit count in meta)

struct Box {
	float lo[3], hi[3];
	void clear()
	{
		for (int a = 0; a < 3; a++) {
			lo[a] = FLT_MAX;
			hi[a] = -FLT_MAX;
		}
	}
	void grow(const Box &b)
	{
		for (int a = 0; a < 3; a++) {
			lo[a] = std::min(lo[a], b.lo[a]);
			hi[a] = std::max(hi[a], b.hi[a]);
		}
	}
	double area() const
	{
		double dx = (double)hi[0] - lo[0], dy = (double)hi[1] - lo[1],
		  dz = (double)hi[2] - lo[2];
		if (!(dx >= 0.0 && dy >= 0.0 && dz >= 0.0))
			return 0.0;
		return dx * dy + dy * dz + dz * dx;
	}
};

struct BNode {
	Box box;
	uint32_t left, right; // kNone for a leaf
	uint32_t start, count;
};

struct Builder {
	std::vector<Box> pbox;
	std::vector<float> cen; // 3 per triangle
	std::vector<uint32_t> idx;
	std::vector<BNode> bn;

	Box range_box(uint32_t s, uint32_t n) const
	{
		Box b;
		b.clear();
		for (uint32_t i = s; i < s + n; i++)
			b.grow(pbox[idx[i]]);
		return b;
	}

	// Best split of [s, s+n) by a sweep over the centroids sorted along
	// each axis; the range is left sorted along the chosen axis and the
	// left side's count is returned (0 if no split beats none).
	uint32_t sweep_split(uint32_t s, uint32_t n, double *best_cost)
	{
		std::vector<uint32_t> tmp(idx.begin() + s, idx.begin() + s + n);
		std::vector<double> rarea(n);
		double best = DBL_MAX;
		int bax = -1;
		uint32_t bpos = 0;
		for (int a = 0; a < 3; a++) {
			std::stable_sort(tmp.begin(), tmp.end(),
			  [&](uint32_t x, uint32_t y) {
				return cen[3 * x + a] < cen[3 * y + a];
			});
			Box b;
			b.clear();
			for (uint32_t i = n - 1; i > 0; i--) {
				b.grow(pbox[tmp[i]]);
				rarea[i] = b.area();
			}
			b.clear();
			for (uint32_t i = 0; i + 1 < n; i++) {
				b.grow(pbox[tmp[i]]);
				double c = b.area() * (i + 1) +
				  rarea[i + 1] * (n - i - 1);
				if (c < best) {
					best = c;
					bax = a;
					bpos = i + 1;
				}
			}
		}
		std::stable_sort(idx.begin() + s, idx.begin() + s + n,
		  [&](uint32_t x, uint32_t y) {
			return cen[3 * x + bax] < cen[3 * y + bax];
		});
		*best_cost = best;
		return bpos;
	}

	// Binned split of [s, s+n) over the centroid bounds; partitions the
	// range and returns the left count (0 when the centroids coincide).
	uint32_t binned_split(uint32_t s, uint32_t n)
	{
		float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
		float chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
		for (uint32_t i = s; i < s + n; i++)
			for (int a = 0; a < 3; a++) {
				float c = cen[3 * idx[i] + a];
				clo[a] = std::min(clo[a], c);
				chi[a] = std::max(chi[a], c);
			}
		double best = DBL_MAX;
		int bax = -1, bbin = 0;
		for (int a = 0; a < 3; a++) {
			double ext = (double)chi[a] - clo[a];
			if (!(ext > 0.0))
				continue;
			Box bb[kBins];
			uint32_t bc[kBins] = {};
			for (int k = 0; k < kBins; k++)
				bb[k].clear();
			double sc = kBins / ext;
			for (uint32_t i = s; i < s + n; i++) {
				uint32_t t = idx[i];
				int k = (int)(((double)cen[3 * t + a] - clo[a]) * sc);
				k = std::min(std::max(k, 0), kBins - 1);
				bb[k].grow(pbox[t]);
				bc[k]++;
			}
			double ra[kBins];
			uint32_t rc[kBins];
			Box b;
			b.clear();
			uint32_t c = 0;
			for (int k = kBins - 1; k > 0; k--) {
				b.grow(bb[k]);
				c += bc[k];
				ra[k] = b.area();
				rc[k] = c;
			}
			b.clear();
			c = 0;
			for (int k = 0; k + 1 < kBins; k++) {
				b.grow(bb[k]);
				c += bc[k];
				if (c == 0 || rc[k + 1] == 0)
					continue;
				double cost = b.area() * c + ra[k + 1] * rc[k + 1];
				if (cost < best) {
					best = cost;
					bax = a;
					bbin = k;
				}
			}
		}
		if (bax < 0)
			return 0;
		double sc = kBins / ((double)chi[bax] - clo[bax]);
		auto mid = std::partition(idx.begin() + s, idx.begin() + s + n,
		  [&](uint32_t t) {
			int k = (int)(((double)cen[3 * t + bax] - clo[bax]) * sc);
			k = std::min(std::max(k, 0), kBins - 1);
			return k <= bbin;
		});
		return (uint32_t)(mid - (idx.begin() + s));
	}

	void build_binary()
	{
		uint32_t n = (uint32_t)idx.size();
		bn.clear();
		bn.reserve(2 * (size_t)n);
		BNode root;
		root.box = range_box(0, n);
		root.left = root.right = kNone;
		root.start = 0;
		root.count = n;
		bn.push_back(root);
		std::vector<uint32_t> todo;
		todo.push_back(0);
		while (!todo.empty()) {
			uint32_t i = todo.back();
			todo.pop_back();
			uint32_t s = bn[i].start, c = bn[i].count;
			if (c <= 1)
				continue;
			uint32_t lc;
			if (c <= kSweepMax) {
				double cost;
				lc = sweep_split(s, c, &cost);
			} else {
				lc = binned_split(s, c);
			}
			if (lc == 0 || lc >= c) {
				// coincident centroids: halve the range
				lc = c / 2;
			}
			BNode l, r;
			l.left = l.right = r.left = r.right = kNone;
			l.start = s;
			l.count = lc;
			r.start = s + lc;
			r.count = c - lc;
			l.box = range_box(l.start, l.count);
			r.box = range_box(r.start, r.count);
			uint32_t li = (uint32_t)bn.size();
			bn.push_back(l);
			bn.push_back(r);
			bn[i].left = li;
			bn[i].right = li + 1;
			todo.push_back(li);
			todo.push_back(li + 1);
		}
	}

	// Collapse tables (Ylitie et al. 2017, section 3.1).
	std::vector<double> cost;    // 8 per binary node: budget 1..8
	std::vector<uint8_t> kd;     // 8 per node: left budget of budget j
	std::vector<uint8_t> prev;   // bit j: cost[j] taken from budget j-1
	std::vector<uint8_t> asleaf; // budget 1 is a leaf

	// In double: surface areas of boxes with coordinates near the float
	// range (1e20 and up) overflow a float, and infinite costs would make a
	// node of more than kLeafMax triangles look no worse as a leaf.
	void collapse_costs(double c_node, double c_tri)
	{
		size_t m = bn.size();
		cost.assign(8 * m, 0.0f);
		kd.assign(8 * m, 0);
		prev.assign(m, 0);
		asleaf.assign(m, 0);
		for (size_t q = m; q-- > 0;) {
			const BNode &b = bn[q];
			double A = b.box.area();
			bool fits = b.count <= (uint32_t)kLeafMax;
			double cl = fits ? A * c_tri * (double)b.count : HUGE_VAL;
			double *C = &cost[8 * q];
			if (b.left == kNone) {
				for (int i = 0; i < 8; i++)
					C[i] = cl;
				asleaf[q] = 1;
				prev[q] = 0xfe;
				continue;
			}
			const double *L = &cost[8 * (size_t)b.left];
			const double *R = &cost[8 * (size_t)b.right];
			double dist[9];
			uint8_t karg[9] = {};
			for (int j = 2; j <= 8; j++) {
				double best = HUGE_VAL;
				int bk = 1;
				for (int k = 1; k < j; k++) {
					double v = L[k - 1] + R[j - k - 1];
					if (v < best) {
						best = v;
						bk = k;
					}
				}
				dist[j] = best;
				karg[j] = (uint8_t)bk;
				kd[8 * q + (j - 1)] = (uint8_t)bk;
			}
			double cn = A * c_node + dist[8];
			if (fits && cl <= cn) {
				C[0] = cl;
				asleaf[q] = 1;
			} else {
				C[0] = cn;
			}
			uint8_t pv = 0;
			for (int i = 2; i <= 8; i++) {
				if (dist[i] < C[i - 2]) {
					C[i - 1] = dist[i];
				} else {
					C[i - 1] = C[i - 2];
					pv |= (uint8_t)(1u << (i - 1));
				}
			}
			prev[q] = pv;
			(void)karg;
		}
	}

	// Subtrees that represent node q with at most j roots.
	void collect(uint32_t q, int j, std::vector<uint32_t> &out) const
	{
		const BNode &b = bn[q];
		if (b.left == kNone) {
			out.push_back(q);
			return;
		}
		while (j >= 2 && (prev[q] >> (j - 1) & 1u))
			j--;
		if (j == 1) {
			out.push_back(q);
			return;
		}
		int k = kd[8 * q + (j - 1)];
		collect(b.left, k, out);
		collect(b.right, j - k, out);
	}
};

} // namespace

bool build_blas(const nb_rdata *rd, uint32_t triofs, uint32_t tricnt,
                const blas_params &prm, blas_out *out, std::string *err)
{
	out->nodes.clear();
	out->tris.clear();
	out->depth = 0;
	if (tricnt == 0) {
		*err = "mesh without triangles";
		return false;
	}
	Builder B;
	B.pbox.resize(tricnt);
	B.cen.resize(3 * (size_t)tricnt);
	B.idx.resize(tricnt);
	for (uint32_t i = 0; i < tricnt; i++) {
		const nb_rtri &t = rd->tris[triofs + i];
		Box b;
		b.lo[0] = std::min(std::min(t.v0.x, t.v1.x), t.v2.x);
		b.lo[1] = std::min(std::min(t.v0.y, t.v1.y), t.v2.y);
		b.lo[2] = std::min(std::min(t.v0.z, t.v1.z), t.v2.z);
		b.hi[0] = std::max(std::max(t.v0.x, t.v1.x), t.v2.x);
		b.hi[1] = std::max(std::max(t.v0.y, t.v1.y), t.v2.y);
		b.hi[2] = std::max(std::max(t.v0.z, t.v1.z), t.v2.z);
		// the vertices themselves: std::min and std::max drop a NaN
		const float vs[9] = {t.v0.x, t.v0.y, t.v0.z, t.v1.x, t.v1.y,
		  t.v1.z, t.v2.x, t.v2.y, t.v2.z};
		for (float v : vs)
			if (!std::isfinite(v)) {
				*err = "non-finite vertex in triangle " +
				  std::to_string(i);
				return false;
			}
		for (int a = 0; a < 3; a++)
			B.cen[3 * (size_t)i + a] = 0.5f * b.lo[a] + 0.5f * b.hi[a];
		B.pbox[i] = b;
		B.idx[i] = i;
	}
	B.build_binary();
	B.collapse_costs(prm.c_node, prm.c_tri);

	struct item {
		uint32_t q;     // binary node represented by the 8-wide node
		uint32_t index; // its output index
		uint32_t depth;
	};
	std::vector<item> fifo;
	fifo.push_back({0u, 0u, 1u});
	out->nodes.emplace_back();
	std::vector<uint32_t> kids;
	for (size_t head = 0; head < fifo.size(); head++) {
		item it = fifo[head];
		out->depth = std::max(out->depth, it.depth);
		const BNode &b = B.bn[it.q];
		kids.clear();
		if (b.left == kNone || B.asleaf[it.q]) {
			kids.push_back(it.q); // a mesh of at most 4 triangles
		} else {
			int k = B.kd[8 * (size_t)it.q + 7];
			B.collect(b.left, k, kids);
			B.collect(b.right, 8 - k, kids);
		}
		int nchild = (int)kids.size();
		if (nchild < 1 || nchild > 8) {
			*err = "collapse produced " + std::to_string(nchild) +
			  " children";
			return false;
		}
		float cen[8][3], nlo[3], nhi[3];
		for (int a = 0; a < 3; a++) {
			nlo[a] = FLT_MAX;
			nhi[a] = -FLT_MAX;
		}
		for (int c = 0; c < nchild; c++) {
			const Box &cb = B.bn[kids[c]].box;
			for (int a = 0; a < 3; a++) {
				cen[c][a] = 0.5f * (cb.lo[a] + cb.hi[a]);
				nlo[a] = std::fmin(nlo[a], cb.lo[a]);
				nhi[a] = std::fmax(nhi[a], cb.hi[a]);
			}
		}
		float nc[3];
		for (int a = 0; a < 3; a++)
			nc[a] = 0.5f * (nlo[a] + nhi[a]);
		int slot_of[8];
		assign_slots(nchild, cen, nc, slot_of);
		int child_at[8];
		for (int s = 0; s < 8; s++)
			child_at[s] = -1;
		for (int c = 0; c < nchild; c++)
			child_at[slot_of[c]] = c;
		float cmin[8][3], cmax[8][3];
		nb_qnode qn;
		std::memset(&qn, 0, sizeof(qn));
		for (int s = 0; s < 8; s++) {
			int c = child_at[s];
			for (int a = 0; a < 3; a++) {
				cmin[s][a] = 1.0f;
				cmax[s][a] = -1.0f;
			}
			if (c < 0)
				continue;
			const Box &cb = B.bn[kids[c]].box;
			for (int a = 0; a < 3; a++) {
				cmin[s][a] = cb.lo[a];
				cmax[s][a] = cb.hi[a];
			}
		}
		quantise_node(cmin, cmax, &qn);
		auto is_leaf = [&](uint32_t q) {
			return B.bn[q].left == kNone || B.asleaf[q] ||
			  q == it.q;
		};
		qn.child_base = (uint32_t)out->nodes.size();
		uint32_t ninner = 0;
		for (int s = 0; s < 8; s++) {
			int c = child_at[s];
			if (c < 0 || is_leaf(kids[c]))
				continue;
			qn.imask |= (uint8_t)(1u << s);
			fifo.push_back({kids[c], qn.child_base + ninner,
			  it.depth + 1});
			ninner++;
		}
		out->nodes.resize(out->nodes.size() + ninner);
		uint32_t off = 0;
		qn.item_base = (uint32_t)out->tris.size();
		for (int s = 0; s < 8; s++) {
			int c = child_at[s];
			if (c < 0 || !is_leaf(kids[c]))
				continue;
			const BNode &lb = B.bn[kids[c]];
			if (lb.count < 1 || lb.count > (uint32_t)kLeafMax ||
			  off + lb.count > 32) {
				*err = "leaf of " + std::to_string(lb.count) +
				  " triangles";
				return false;
			}
			for (uint32_t k = 0; k < lb.count; k++) {
				uint32_t prim = B.idx[lb.start + k];
				const nb_rtri &t = rd->tris[triofs + prim];
				nb_gtri g;
				g.v0[0] = t.v0.x; g.v0[1] = t.v0.y; g.v0[2] = t.v0.z;
				g.v1[0] = t.v1.x; g.v1[1] = t.v1.y; g.v1[2] = t.v1.z;
				g.v2[0] = t.v2.x; g.v2[1] = t.v2.y; g.v2[2] = t.v2.z;
				g.prim = prim;
				g.pad1 = g.pad2 = 0;
				out->tris.push_back(g);
			}
			qn.meta[s] = (uint8_t)(NB_META_LEAF |
			  (lb.count - 1) << 5 | off);
			off += lb.count;
		}
		if (off == 0)
			qn.item_base = 0;
		out->nodes[it.index] = qn;
	}
	return true;
}

void append_blas(const blas_out &b, std::vector<nb_qnode> &nodes,
                 std::vector<nb_gtri> &tris, uint32_t *root)
{
	uint32_t nb = (uint32_t)nodes.size(), tb = (uint32_t)tris.size();
	*root = nb;
	nodes.reserve(nodes.size() + b.nodes.size());
	for (nb_qnode q : b.nodes) {
		q.child_base += nb;
		q.item_base += tb;
		nodes.push_back(q);
	}
	tris.insert(tris.end(), b.tris.begin(), b.tris.end());
}

bool build_blas_many(const nb_rdata *rd, const std::vector<uint32_t> &triofs,
                     const std::vector<uint32_t> &tricnt,
                     const blas_params &prm, std::vector<blas_out> &out,
                     std::string *err)
{
	size_t n = triofs.size();
	out.assign(n, blas_out());
	std::vector<std::string> errs(n);
	std::vector<uint8_t> ok(n, 0);
	unsigned hw = std::thread::hardware_concurrency();
	size_t nt = std::min<size_t>(n, hw ? std::min(hw, 32u) : 4u);
	// largest meshes first, taken from a shared counter
	std::vector<size_t> order(n);
	for (size_t i = 0; i < n; i++)
		order[i] = i;
	std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
		return tricnt[a] > tricnt[b];
	});
	std::atomic<size_t> next(0);
	auto work = [&]() {
		for (;;) {
			size_t k = next.fetch_add(1);
			if (k >= n)
				return;
			size_t i = order[k];
			ok[i] = build_blas(rd, triofs[i], tricnt[i], prm, &out[i],
			  &errs[i]) ? 1 : 0;
		}
	};
	if (nt <= 1) {
		work();
	} else {
		std::vector<std::thread> th;
		for (size_t t = 0; t < nt; t++)
			th.emplace_back(work);
		for (std::thread &t : th)
			t.join();
	}
	for (size_t i = 0; i < n; i++)
		if (!ok[i]) {
			*err = "BLAS of triofs " + std::to_string(triofs[i]) +
			  ": " + errs[i];
			return false;
		}
	return true;
}

} // namespace nb
