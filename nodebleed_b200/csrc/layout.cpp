// Conversion of the reference BVH8 into the GPU node layout (gpulayout.h).
//
// Input is exactly what nodebleed's host code leaves in rd->bnodes after
// rend_prepstatic/rend_prepdynamic (rend.c:458-709): per BLAS a tree of
// 256-byte bnode8 nodes with embedded 192-byte leaf4 records, addressed by
// byte offsets from the BLAS root at node index 2*triofs; the TLAS at node
// index tlasofs with instance ids in its leaves.  The tree shape (which
// children each node has, which triangles each leaf holds) is kept 1:1;
// only the encoding changes.

#include "layout.hpp"
#include "qnode.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>

namespace nb {

namespace {

struct qitem {
	uint32_t ofs;   // byte offset of the bnode8 from the tree base
	uint32_t index; // its node index in the output
	uint32_t depth;
};

bool empty_child(const nb_bnode8 *n, int j)
{
	return !(n->minx8[j] <= n->maxx8[j]) || !(n->miny8[j] <= n->maxy8[j]) ||
	  !(n->minz8[j] <= n->maxz8[j]);
}

} // namespace

void quantise_node(const float cmin[8][3], const float cmax[8][3],
                   nb_qnode *n)
{
	quantise_node_hd(cmin, cmax, n);
}

namespace {

// Shared conversion of one tree.  leaf(ofs, items) appends the leaf's items
// and returns their count (0 = malformed).
// Widen [lo, hi] by 2^-20 of its magnitude, rounded outwards (world boxes
// of a TLAS: they come from transformed corners rounded to FP32, and the
// quantised planes keep only 1/32 of a quantum outside a child box).
void widen_box(float *lo, float *hi)
{
	double m = std::fmax(std::fabs((double)*lo), std::fabs((double)*hi)) *
	  std::ldexp(1.0, -20);
	double l = (double)*lo - m, h = (double)*hi + m;
	float lf = (float)l, hf = (float)h;
	if ((double)lf > l)
		lf = std::nextafter(lf, -FLT_MAX);
	if ((double)hf < h)
		hf = std::nextafter(hf, FLT_MAX);
	*lo = lf;
	*hi = hf;
}

template <class LeafFn>
bool convert_tree(const uint8_t *base, uint64_t limit,
                  std::vector<nb_qnode> &nodes, uint32_t root_index,
                  LeafFn leaf, bvh_stats *st, std::string *err,
                  bool widen = false)
{
	std::deque<qitem> q;
	q.push_back({0u, root_index, 1u});
	uint32_t maxdepth = 0, count = 0;
	while (!q.empty()) {
		qitem it = q.front();
		q.pop_front();
		if (it.ofs % 64 || (uint64_t)it.ofs + sizeof(nb_bnode8) > limit) {
			*err = "node offset out of range";
			return false;
		}
		if (++count > (1u << 28)) {
			*err = "too many nodes";
			return false;
		}
		maxdepth = it.depth > maxdepth ? it.depth : maxdepth;
		const nb_bnode8 *bn = (const nb_bnode8 *)(base + it.ofs);
		int nchild = 0, idx[8];
		float cmin[8][3], cmax[8][3], cen[8][3];
		float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
		float nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
		for (int j = 0; j < 8; j++) {
			if (empty_child(bn, j))
				continue;
			idx[nchild] = j;
			float mi[3] = {bn->minx8[j], bn->miny8[j], bn->minz8[j]};
			float ma[3] = {bn->maxx8[j], bn->maxy8[j], bn->maxz8[j]};
			for (int a = 0; a < 3; a++) {
				cen[nchild][a] = 0.5f * (mi[a] + ma[a]);
				nlo[a] = std::fmin(nlo[a], mi[a]);
				nhi[a] = std::fmax(nhi[a], ma[a]);
			}
			nchild++;
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
			child_at[slot_of[c]] = idx[c];
		nb_qnode qn;
		std::memset(&qn, 0, sizeof(qn));
		for (int s = 0; s < 8; s++) {
			int j = child_at[s];
			for (int a = 0; a < 3; a++) {
				cmin[s][a] = 1.0f;
				cmax[s][a] = -1.0f;
			}
			if (j < 0)
				continue;
			cmin[s][0] = bn->minx8[j];
			cmin[s][1] = bn->miny8[j];
			cmin[s][2] = bn->minz8[j];
			cmax[s][0] = bn->maxx8[j];
			cmax[s][1] = bn->maxy8[j];
			cmax[s][2] = bn->maxz8[j];
			if (widen)
				for (int a = 0; a < 3; a++)
					widen_box(&cmin[s][a], &cmax[s][a]);
		}
		quantise_node(cmin, cmax, &qn);
		// inner children contiguous in slot order
		qn.child_base = (uint32_t)nodes.size();
		uint32_t ninner = 0;
		for (int s = 0; s < 8; s++) {
			int j = child_at[s];
			if (j < 0 || (bn->children8[j] & NB_NODE_LEAF))
				continue;
			qn.imask |= (uint8_t)(1u << s);
			q.push_back({bn->children8[j], qn.child_base + ninner,
			  it.depth + 1});
			ninner++;
		}
		nodes.resize(nodes.size() + ninner);
		// leaf items contiguous in slot order
		uint32_t off = 0;
		qn.item_base = UINT32_MAX;
		for (int s = 0; s < 8; s++) {
			int j = child_at[s];
			if (j < 0 || !(bn->children8[j] & NB_NODE_LEAF))
				continue;
			uint32_t first = 0;
			uint32_t cnt = leaf(bn->children8[j] & ~NB_NODE_LEAF, &first);
			if (cnt == 0 || cnt > 4 || off + cnt > 32) {
				*err = "malformed leaf";
				return false;
			}
			if (qn.item_base == UINT32_MAX)
				qn.item_base = first;
			qn.meta[s] = (uint8_t)(NB_META_LEAF | (cnt - 1) << 5 | off);
			off += cnt;
		}
		if (qn.item_base == UINT32_MAX)
			qn.item_base = 0;
		nodes[it.index] = qn;
	}
	st->depth = maxdepth;
	st->nodes = count;
	return true;
}

} // namespace

bool convert_blas(const nb_rdata *rd, uint32_t triofs,
                  std::vector<nb_qnode> &nodes, std::vector<nb_gtri> &tris,
                  uint32_t *root, bvh_stats *st, std::string *err)
{
	uint32_t tricnt = 0;
	for (uint32_t i = 0; i < rd->instcnt; i++)
		if (rd->insts[i].triofs == triofs)
			tricnt = rd->insts[i].tricnt;
	const uint8_t *base = (const uint8_t *)&rd->bnodes[(size_t)triofs << 1];
	uint64_t limit = (uint64_t)2 * (tricnt ? tricnt : 1) *
	  sizeof(nb_bnode8);
	*root = (uint32_t)nodes.size();
	nodes.emplace_back();
	uint32_t items0 = (uint32_t)tris.size();
	auto leaf = [&](uint32_t ofs, uint32_t *first) -> uint32_t {
		if (ofs % 64 || (uint64_t)ofs + sizeof(nb_leaf4) > limit)
			return 0;
		const nb_leaf4 *l = (const nb_leaf4 *)(base + ofs);
		uint32_t cnt = l->tricnt;
		if (cnt < 1 || cnt > 4)
			return 0;
		*first = (uint32_t)tris.size();
		for (uint32_t k = 0; k < cnt; k++) {
			uint32_t prim = l->id4[k];
			if (prim >= tricnt)
				return 0;
			const nb_rtri *t = &rd->tris[triofs + prim];
			nb_gtri g;
			g.v0[0] = t->v0.x; g.v0[1] = t->v0.y; g.v0[2] = t->v0.z;
			g.v1[0] = t->v1.x; g.v1[1] = t->v1.y; g.v1[2] = t->v1.z;
			g.v2[0] = t->v2.x; g.v2[1] = t->v2.y; g.v2[2] = t->v2.z;
			g.prim = prim;
			g.pad1 = g.pad2 = 0;
			tris.push_back(g);
		}
		return cnt;
	};
	bool ok = convert_tree(base, limit, nodes, *root, leaf, st, err);
	st->items = (uint32_t)tris.size() - items0;
	return ok;
}

bool convert_tlas(const nb_rdata *rd, std::vector<nb_qnode> &nodes,
                  std::vector<uint32_t> &irefs, uint32_t inst_base,
                  uint32_t *root, bvh_stats *st, std::string *err)
{
	const uint8_t *base = (const uint8_t *)&rd->bnodes[rd->tlasofs];
	uint64_t limit = (uint64_t)2 * (rd->instcnt ? rd->instcnt : 1) *
	  sizeof(nb_bnode8);
	*root = (uint32_t)nodes.size();
	nodes.emplace_back();
	uint32_t items0 = (uint32_t)irefs.size();
	auto leaf = [&](uint32_t inst, uint32_t *first) -> uint32_t {
		if (inst >= rd->instcnt)
			return 0;
		*first = (uint32_t)irefs.size();
		irefs.push_back(inst_base + inst);
		return 1;
	};
	bool ok = convert_tree(base, limit, nodes, *root, leaf, st, err, true);
	st->items = (uint32_t)irefs.size() - items0;
	return ok;
}

void find_emitters(const nb_rdata *rd,
                   std::unordered_map<uint32_t, std::vector<uint32_t>> &out)
{
	out.clear();
	for (uint32_t i = 0; i < rd->instcnt; i++) {
		const nb_rinst *ri = &rd->insts[i];
		if (out.count(ri->triofs))
			continue;
		std::vector<uint32_t> &e = out[ri->triofs];
		for (uint32_t t = 0; t < ri->tricnt; t++) {
			const nb_rnrm *rn = &rd->nrms[ri->triofs + t];
			if (rd->mtls[rn->mtlid].flags & NB_FLAG_EMISSIVE)
				e.push_back(t);
		}
	}
}

float build_lights(const nb_rdata *rd, std::vector<nb_glight> &lights,
                   const std::unordered_map<uint32_t,
                   std::vector<uint32_t>> *emitters)
{
	lights.clear();
	double total = 0.0;
	std::vector<double> areas;
	for (uint32_t i = 0; i < rd->instcnt; i++) {
		const nb_rinst *ri = &rd->insts[i];
		const float *g = ri->globinv;
		// forward = inverse of the 3x3 part, translation -A^-1 b
		double A[9] = {g[0], g[1], g[2], g[4], g[5], g[6], g[8], g[9], g[10]};
		double b[3] = {g[3], g[7], g[11]};
		double det = A[0] * (A[4] * A[8] - A[5] * A[7]) -
		  A[1] * (A[3] * A[8] - A[5] * A[6]) +
		  A[2] * (A[3] * A[7] - A[4] * A[6]);
		if (det == 0.0)
			continue;
		double I[9] = {
		  (A[4] * A[8] - A[5] * A[7]) / det, (A[2] * A[7] - A[1] * A[8]) / det,
		  (A[1] * A[5] - A[2] * A[4]) / det, (A[5] * A[6] - A[3] * A[8]) / det,
		  (A[0] * A[8] - A[2] * A[6]) / det, (A[2] * A[3] - A[0] * A[5]) / det,
		  (A[3] * A[7] - A[4] * A[6]) / det, (A[1] * A[6] - A[0] * A[7]) / det,
		  (A[0] * A[4] - A[1] * A[3]) / det};
		const std::vector<uint32_t> *em = nullptr;
		if (emitters) {
			auto it = emitters->find(ri->triofs);
			if (it == emitters->end() || it->second.empty())
				continue;
			em = &it->second;
		}
		uint32_t cnt = em ? (uint32_t)em->size() : ri->tricnt;
		for (uint32_t k = 0; k < cnt; k++) {
			uint32_t t = em ? (*em)[k] : k;
			const nb_rnrm *rn = &rd->nrms[ri->triofs + t];
			const nb_rmtl *m = &rd->mtls[rn->mtlid];
			if (!(m->flags & NB_FLAG_EMISSIVE))
				continue;
			const nb_rtri *tr = &rd->tris[ri->triofs + t];
			const nb_vec3 *vv[3] = {&tr->v0, &tr->v1, &tr->v2};
			double w[3][3];
			for (int k = 0; k < 3; k++) {
				double x[3] = {vv[k]->x - b[0], vv[k]->y - b[1],
				  vv[k]->z - b[2]};
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
			double len = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
			if (len == 0.0)
				continue;
			// emitting side: the world-space interpolated normal at
			// the centroid (normals map by the transpose of A)
			double no[3] = {
			  (double)rn->n0.x + rn->n1.x + rn->n2.x,
			  (double)rn->n0.y + rn->n1.y + rn->n2.y,
			  (double)rn->n0.z + rn->n1.z + rn->n2.z};
			double nw[3] = {A[0] * no[0] + A[3] * no[1] + A[6] * no[2],
			  A[1] * no[0] + A[4] * no[1] + A[7] * no[2],
			  A[2] * no[0] + A[5] * no[1] + A[8] * no[2]};
			double sgn = (c[0] * nw[0] + c[1] * nw[1] + c[2] * nw[2]) < 0
			  ? -1.0 : 1.0;
			nb_glight L;
			std::memset(&L, 0, sizeof(L));
			for (int a = 0; a < 3; a++) {
				L.v0[a] = (float)w[0][a];
				L.e0[a] = (float)e0[a];
				L.e1[a] = (float)e1[a];
				L.n[a] = (float)(sgn * c[a] / len);
			}
			L.emit[0] = m->col.x;
			L.emit[1] = m->col.y;
			L.emit[2] = m->col.z;
			L.area = (float)(0.5 * len);
			lights.push_back(L);
			areas.push_back(0.5 * len);
			total += 0.5 * len;
		}
	}
	double run = 0.0;
	for (size_t i = 0; i < lights.size(); i++) {
		run += areas[i];
		lights[i].cdf = (float)(run / total);
	}
	if (!lights.empty())
		lights.back().cdf = 1.0f;
	return (float)total;
}

} // namespace nb
