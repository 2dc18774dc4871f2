// BVH8 build and render-data allocation, restating nodebleed's host code.
//
// The node bytes this writes are the upload format of the GPU library, so the
// build follows the reference step for step (rend.c:266-709, 3000-3107):
// 16-bin centroid SAH with cost cnt*area/8, an in-place partition, "horizontal"
// splits of the widest-area child until a node has 8 children, then one
// "vertical" split per remaining inner child into a new 2-child node, leaves of
// up to 4 triangles embedded as 192-byte leaf4 records in the node byte space,
// and a per-octant child order (perm8).  tests/test_bvh_build.py checks the
// bytes against the reference build.

#include <float.h>
#include <stdlib.h>
#include <string.h>

#include "nb_host.h"

#define NB_BINS 16 // rend.c:27 INTERVAL_CNT

static inline float fminr(float a, float b) { return a < b ? a : b; }
static inline float fmaxr(float a, float b) { return a > b ? a : b; }

static inline struct nb_vec3 v3min(struct nb_vec3 a, struct nb_vec3 b)
{
	return (struct nb_vec3){fminr(a.x, b.x), fminr(a.y, b.y),
	  fminr(a.z, b.z)};
}

static inline struct nb_vec3 v3max(struct nb_vec3 a, struct nb_vec3 b)
{
	return (struct nb_vec3){fmaxr(a.x, b.x), fmaxr(a.y, b.y),
	  fmaxr(a.z, b.z)};
}

static inline float v3get(struct nb_vec3 v, int a)
{
	return a == 0 ? v.x : (a == 1 ? v.y : v.z);
}

// Half surface area of a box (rend.c:266 calc_area).
static inline float half_area(struct nb_vec3 mi, struct nb_vec3 ma)
{
	float dx = ma.x - mi.x, dy = ma.y - mi.y, dz = ma.z - mi.z;
	return dx * dy + dy * dz + dz * dx;
}

static inline int clampbin(float c)
{
	int b = (int)c;
	b = b > 0 ? b : 0;
	return b < NB_BINS - 1 ? b : NB_BINS - 1;
}

struct split { // rend.c:76-85
	float          cost;
	int            axis;
	unsigned int   pos;
	struct nb_vec3 lmin, lmax, rmin, rmax;
	struct nb_vec3 invd;
};

// Binned SAH split search (rend.c:274-386).
static void best_split(struct split *best, unsigned int start,
                       unsigned int cnt, struct nb_vec3 nmin,
                       struct nb_vec3 nmax, struct nb_vec3 minext,
                       const struct nb_aabb *aabbs, const unsigned int *imap)
{
	struct nb_vec3 bmin[3][NB_BINS], bmax[3][NB_BINS];
	unsigned int bcnt[3][NB_BINS];
	const struct nb_vec3 big = {FLT_MAX, FLT_MAX, FLT_MAX};
	const struct nb_vec3 nbig = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	for (int a = 0; a < 3; a++)
		for (int i = 0; i < NB_BINS; i++) {
			bmin[a][i] = big;
			bmax[a][i] = nbig;
			bcnt[a][i] = 0;
		}

	best->invd = (struct nb_vec3){(float)NB_BINS / (nmax.x - nmin.x),
	  (float)NB_BINS / (nmax.y - nmin.y),
	  (float)NB_BINS / (nmax.z - nmin.z)};

	for (unsigned int i = 0; i < cnt; i++) {
		const struct nb_aabb *b = &aabbs[imap[start + i]];
		float cx = ((b->min.x + b->max.x) * 0.5f - nmin.x) * best->invd.x;
		float cy = ((b->min.y + b->max.y) * 0.5f - nmin.y) * best->invd.y;
		float cz = ((b->min.z + b->max.z) * 0.5f - nmin.z) * best->invd.z;
		int bin[3] = {clampbin(cx), clampbin(cy), clampbin(cz)};
		for (int a = 0; a < 3; a++) {
			bcnt[a][bin[a]]++;
			bmin[a][bin[a]] = v3min(bmin[a][bin[a]], b->min);
			bmax[a][bin[a]] = v3max(bmax[a][bin[a]], b->max);
		}
	}

	best->cost = FLT_MAX;
	// Deviation: the reference leaves the split unset when no plane beats
	// FLT_MAX (all centroids in one bin); here it stays the node box.
	best->axis = 0;
	best->pos = 0;
	best->lmin = best->rmin = nmin;
	best->lmax = best->rmax = nmax;

	for (int a = 0; a < 3; a++) {
		if (v3get(nmax, a) - v3get(nmin, a) < v3get(minext, a))
			continue; // flat axis
		struct nb_vec3 lmin[NB_BINS - 1], lmax[NB_BINS - 1];
		struct nb_vec3 rmin[NB_BINS - 1], rmax[NB_BINS - 1];
		float lcost[NB_BINS - 1], rcost[NB_BINS - 1];
		struct nb_vec3 lmi = big, lma = nbig, rmi = big, rma = nbig;
		unsigned int lc = 0, rc = 0;
		for (int i = 0; i < NB_BINS - 1; i++) {
			lmi = v3min(lmi, bmin[a][i]);
			lma = v3max(lma, bmax[a][i]);
			lmin[i] = lmi;
			lmax[i] = lma;
			lc += bcnt[a][i];
			lcost[i] = lc > 0 ? (float)lc * half_area(lmi, lma) /
			  NB_BRANCH_MAX : FLT_MAX;

			int r = NB_BINS - 1 - i;
			rmi = v3min(rmi, bmin[a][r]);
			rma = v3max(rma, bmax[a][r]);
			rmin[r - 1] = rmi;
			rmax[r - 1] = rma;
			rc += bcnt[a][r];
			rcost[r - 1] = rc > 0 ? (float)rc * half_area(rmi, rma) /
			  NB_BRANCH_MAX : FLT_MAX;
		}
		for (int i = 0; i < NB_BINS - 1; i++) {
			float c = lcost[i] + rcost[i];
			if (c < best->cost) {
				best->cost = c;
				best->axis = a;
				best->pos = (unsigned int)i;
				best->lmin = lmin[i];
				best->lmax = lmax[i];
				best->rmin = rmin[i];
				best->rmax = rmax[i];
			}
		}
	}
}

// In-place partition by split bin (rend.c:389-414); returns the left count.
static unsigned int split_items(unsigned int start, unsigned int cnt,
                                struct nb_vec3 nmin,
                                const struct nb_aabb *aabbs,
                                unsigned int *imap, const struct split *s)
{
	unsigned int l = start, r = start + cnt;
	float invd = v3get(s->invd, s->axis);
	float lo = v3get(nmin, s->axis);
	for (unsigned int i = 0; i < cnt; i++) {
		unsigned int id = imap[l];
		const struct nb_aabb *b = &aabbs[id];
		float c = ((v3get(b->min, s->axis) + v3get(b->max, s->axis)) *
		  0.5f - lo) * invd;
		if ((unsigned int)clampbin(c) <= s->pos) {
			l++;
		} else {
			imap[l] = imap[--r];
			imap[r] = id;
		}
	}
	return l - start;
}

// Write one leaf4 record of up to 4 triangles at byte offset ofs; the last
// triangle is repeated into unused lanes (rend.c:416-456).
static unsigned int write_leaf(unsigned char *base, unsigned int ofs,
                               unsigned int start, unsigned int cnt,
                               const unsigned int *imap,
                               const struct nb_rtri *tris)
{
	struct nb_leaf4 *l = (struct nb_leaf4 *)(base + ofs);
	unsigned int k = start;
	for (int i = 0; i < 4; i++) {
		const struct nb_rtri *t = &tris[imap[k]];
		l->v0x4[i] = t->v0.x;
		l->v0y4[i] = t->v0.y;
		l->v0z4[i] = t->v0.z;
		l->e0x4[i] = t->v1.x - t->v0.x;
		l->e0y4[i] = t->v1.y - t->v0.y;
		l->e0z4[i] = t->v1.z - t->v0.z;
		l->e1x4[i] = t->v2.x - t->v0.x;
		l->e1y4[i] = t->v2.y - t->v0.y;
		l->e1z4[i] = t->v2.z - t->v0.z;
		l->id4[i] = imap[k];
		if ((unsigned int)i + 1 < cnt)
			k++;
	}
	l->tricnt = cnt;
	return (unsigned int)sizeof(*l);
}

struct slotdist { // rend.c:87-90
	float         dist;
	unsigned char id;
};

// Descending by distance, ties unordered: same comparator contract as
// rend.c:92-96 (never returns 0), so qsort permutes identically.
static int slot_cmp(const void *a, const void *b)
{
	return ((const struct slotdist *)a)->dist <
	  ((const struct slotdist *)b)->dist ? 1 : -1;
}

static inline void set_child_box(struct nb_bnode8 *n, int j,
                                 struct nb_vec3 mi, struct nb_vec3 ma)
{
	n->minx8[j] = mi.x;
	n->miny8[j] = mi.y;
	n->minz8[j] = mi.z;
	n->maxx8[j] = ma.x;
	n->maxy8[j] = ma.y;
	n->maxz8[j] = ma.z;
}

// Turn child j (holding `cnt` items from `start`) into a leaf: an embedded
// leaf4 for a BLAS, the instance id for the TLAS.
static void make_leaf(struct nb_bnode8 *n, int j, unsigned char *base,
                      unsigned int *ofs, unsigned int start, unsigned int cnt,
                      const unsigned int *imap, const struct nb_rtri *tris)
{
	if (tris) {
		n->children8[j] = NB_NODE_LEAF | *ofs;
		*ofs += write_leaf(base, *ofs, start, cnt, imap, tris);
	} else {
		n->children8[j] = NB_NODE_LEAF | imap[start];
	}
	n->perm8[j] = 0;
}

// rend.c:458-709.  During the build children8[j] holds the item count and
// perm8[j] the first item index of a not yet split child.
unsigned int nbh_build_bvh8(struct nb_bnode8 *nodes, struct nb_aabb *aabbs,
                            unsigned int *imap, const struct nb_rtri *tris,
                            unsigned int pcnt,
                            struct nb_vec3 rootmin, struct nb_vec3 rootmax)
{
	// Nodes waiting for their horizontal pass, taken last-in first-out as
	// in the reference (whose 64-entry stack is only assert-checked).
	enum { TODO_CAP = 4096 };
	unsigned int todo[TODO_CAP];
	unsigned int ntodo = 0;
	unsigned char *base = (unsigned char *)nodes;
	struct nb_bnode8 *n = nodes;
	unsigned int ofs = sizeof(*n);
	unsigned int childcnt = 1;
	unsigned int ncnt = 1;
	const unsigned int leafmax = tris ? NB_BLAS_LEAF_MAX : NB_TLAS_LEAF_MAX;

	memset(n, 0, sizeof(*n));
	set_child_box(n, 0, rootmin, rootmax);
	n->children8[0] = pcnt;

	struct nb_vec3 minext = {(rootmax.x - rootmin.x) * 0.00000001f,
	  (rootmax.y - rootmin.y) * 0.00000001f,
	  (rootmax.z - rootmin.z) * 0.00000001f};

	for (;;) {
		// Horizontal: split the inner child of largest area until full.
		while (childcnt < NB_BRANCH_MAX) {
			int j = -1;
			float barea = 0.0f;
			struct nb_vec3 bmin = {0, 0, 0}, bmax = {0, 0, 0};
			for (unsigned int i = 0; i < childcnt; i++) {
				if (n->children8[i] & NB_NODE_LEAF)
					continue;
				struct nb_vec3 mi = {n->minx8[i], n->miny8[i],
				  n->minz8[i]};
				struct nb_vec3 ma = {n->maxx8[i], n->maxy8[i],
				  n->maxz8[i]};
				float a = half_area(mi, ma);
				if (a > barea) {
					barea = a;
					j = (int)i;
					bmin = mi;
					bmax = ma;
				}
			}
			if (j < 0)
				break;

			unsigned int cnt = n->children8[j];
			unsigned int start = n->perm8[j];
			if (cnt <= leafmax) {
				make_leaf(n, j, base, &ofs, start, cnt, imap,
				  tris);
				continue;
			}

			struct split s;
			best_split(&s, start, cnt, bmin, bmax, minext, aabbs,
			  imap);
			unsigned int lcnt = split_items(start, cnt, bmin, aabbs,
			  imap, &s);
			if (lcnt == 0)
				lcnt = 1; // rend.c:564 forces a 1-item side
			else if (lcnt == cnt)
				lcnt = cnt - 1;

			n->children8[childcnt] = cnt - lcnt;
			n->perm8[childcnt] = start + lcnt;
			set_child_box(n, (int)childcnt, s.rmin, s.rmax);
			childcnt++;

			n->children8[j] = lcnt;
			set_child_box(n, j, s.lmin, s.lmax);
		}

		// Vertical: each remaining inner child becomes a new 2-child
		// node, queued for its own horizontal pass.
		for (unsigned int j = 0; j < childcnt; j++) {
			unsigned int cnt = n->children8[j];
			if (cnt & NB_NODE_LEAF)
				continue;
			unsigned int start = n->perm8[j];
			if (cnt <= leafmax) {
				make_leaf(n, (int)j, base, &ofs, start, cnt,
				  imap, tris);
				continue;
			}
			struct nb_vec3 mi = {n->minx8[j], n->miny8[j],
			  n->minz8[j]};
			struct nb_vec3 ma = {n->maxx8[j], n->maxy8[j],
			  n->maxz8[j]};
			struct split s;
			best_split(&s, start, cnt, mi, ma, minext, aabbs, imap);
			unsigned int lcnt = split_items(start, cnt, mi, aabbs,
			  imap, &s);
			if (lcnt == 0 || lcnt == cnt)
				continue; // rend.c:614-620

			struct nb_bnode8 *c = (struct nb_bnode8 *)(base + ofs);
			memset(c, 0, sizeof(*c));
			c->children8[0] = lcnt;
			c->perm8[0] = start;
			set_child_box(c, 0, s.lmin, s.lmax);
			c->children8[1] = cnt - lcnt;
			c->perm8[1] = start + lcnt;
			set_child_box(c, 1, s.rmin, s.rmax);

			n->children8[j] = ofs;
			n->perm8[j] = 0;
			if (ntodo >= TODO_CAP)
				return 0; // too deep: report failure
			todo[ntodo++] = ofs;
			ofs += sizeof(*c);
			ncnt++;
		}

		// Child order per ray octant: sort children by the box corner
		// nearest to the octant direction (rend.c:658-687).
		for (unsigned int q = 0; q < NB_BRANCH_MAX; q++) {
			float sx = (q & 1) ? 1.0f : -1.0f;
			float sy = (q & 2) ? 1.0f : -1.0f;
			float sz = (q & 4) ? 1.0f : -1.0f;
			struct slotdist sd[NB_BRANCH_MAX];
			for (unsigned int i = 0; i < NB_BRANCH_MAX; i++) {
				sd[i].id = (unsigned char)i;
				if (i < childcnt) {
					float cx = (q & 1) ? n->minx8[i] : n->maxx8[i];
					float cy = (q & 2) ? n->miny8[i] : n->maxy8[i];
					float cz = (q & 4) ? n->minz8[i] : n->maxz8[i];
					sd[i].dist = sx * cx + sy * cy + sz * cz;
				} else {
					sd[i].dist = FLT_MAX;
				}
			}
			qsort(sd, NB_BRANCH_MAX, sizeof(*sd), slot_cmp);
			for (unsigned int i = 0; i < NB_BRANCH_MAX; i++)
				n->perm8[i] |= (uint32_t)sd[i].id << (q * 3);
		}

		for (; childcnt < NB_BRANCH_MAX; childcnt++) {
			struct nb_vec3 e0 = {FLT_MAX, FLT_MAX, FLT_MAX};
			struct nb_vec3 e1 = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
			set_child_box(n, (int)childcnt, e0, e1);
		}

		if (ntodo == 0)
			break;
		n = (struct nb_bnode8 *)(base + todo[--ntodo]);
		childcnt = 2;
	}
	return ncnt;
}

// One BLAS per distinct mesh (triofs), at node index 2*triofs; a mesh whose
// root already has children is skipped (rend.c:3033-3071).
void nbh_prepstatic(struct nb_rdata *rd)
{
	for (unsigned int j = 0; j < rd->instcnt; j++) {
		const struct nb_rinst *ri = &rd->insts[j];
		struct nb_bnode8 *root = &rd->bnodes[(size_t)ri->triofs << 1];
		if (root->children8[0])
			continue;
		unsigned int tc = ri->tricnt;
		const struct nb_rtri *tp = &rd->tris[ri->triofs];
		unsigned int *imap = malloc(sizeof(*imap) * (tc ? tc : 1));
		struct nb_aabb *bx = malloc(sizeof(*bx) * (tc ? tc : 1));
		struct nb_vec3 rmin = {FLT_MAX, FLT_MAX, FLT_MAX};
		struct nb_vec3 rmax = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
		for (unsigned int i = 0; i < tc; i++) {
			struct nb_vec3 mi = v3min(v3min(tp[i].v0, tp[i].v1),
			  tp[i].v2);
			struct nb_vec3 ma = v3max(v3max(tp[i].v0, tp[i].v1),
			  tp[i].v2);
			bx[i].min = mi;
			bx[i].max = ma;
			bx[i].pad0 = bx[i].pad1 = 0.0f;
			rmin = v3min(rmin, mi);
			rmax = v3max(rmax, ma);
			imap[i] = i;
		}
		nbh_build_bvh8(root, bx, imap, tp, tc, rmin, rmax);
		free(bx);
		free(imap);
	}
}

// TLAS over the world-space instance boxes (rend.c:3073-3090).
void nbh_prepdynamic(struct nb_rdata *rd)
{
	unsigned int n = rd->instcnt;
	unsigned int *imap = malloc(sizeof(*imap) * (n ? n : 1));
	struct nb_vec3 rmin = {FLT_MAX, FLT_MAX, FLT_MAX};
	struct nb_vec3 rmax = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
	for (unsigned int i = 0; i < n; i++) {
		rmin = v3min(rmin, rd->aabbs[i].min);
		rmax = v3max(rmax, rd->aabbs[i].max);
		imap[i] = i;
	}
	nbh_build_bvh8(&rd->bnodes[rd->tlasofs], rd->aabbs, imap, NULL, n,
	  rmin, rmax);
	free(imap);
}

struct nb_rdata *nbh_rdata_new(void)
{
	struct nb_rdata *rd = aligned_alloc(64, (sizeof(*rd) + 63) & ~63ul);
	if (rd)
		memset(rd, 0, sizeof(*rd));
	return rd;
}

void nbh_rdata_delete(struct nb_rdata *rd)
{
	free(rd);
}

static void *zalloc64(size_t bytes)
{
	size_t sz = (bytes + 63) & ~(size_t)63;
	void *p = aligned_alloc(64, sz ? sz : 64);
	if (p)
		memset(p, 0, sz ? sz : 64);
	return p;
}

// rend.c:3000-3023: node space for 2*(tris+insts) nodes, TLAS at 2*maxtris.
int nbh_rend_init(struct nb_rdata *rd, unsigned int maxmtls,
                  unsigned int maxtris, unsigned int maxinsts,
                  unsigned int spp)
{
	rd->mtls = zalloc64((size_t)maxmtls * sizeof(*rd->mtls));
	rd->tris = zalloc64((size_t)maxtris * sizeof(*rd->tris));
	rd->nrms = zalloc64((size_t)maxtris * sizeof(*rd->nrms));
	rd->insts = zalloc64((size_t)maxinsts * sizeof(*rd->insts));
	rd->aabbs = zalloc64((size_t)maxinsts * sizeof(*rd->aabbs));
	rd->bnodes = zalloc64(2 * ((size_t)maxtris + maxinsts) *
	  sizeof(*rd->bnodes));
	rd->tlasofs = 2 * maxtris;
	rd->spp = spp;
	if (!rd->mtls || !rd->tris || !rd->nrms || !rd->insts || !rd->aabbs ||
	  !rd->bnodes)
		return -1;
	return 0;
}

void nbh_rend_release(struct nb_rdata *rd)
{
	free(rd->acc);
	free(rd->bnodes);
	free(rd->aabbs);
	free(rd->insts);
	free(rd->nrms);
	free(rd->tris);
	free(rd->mtls);
	rd->acc = NULL;
	rd->bnodes = NULL;
	rd->aabbs = NULL;
	rd->insts = NULL;
	rd->nrms = NULL;
	rd->tris = NULL;
	rd->mtls = NULL;
}

int nbh_rend_resaccum(struct nb_rdata *rd, unsigned int w, unsigned int h)
{
	free(rd->acc);
	rd->acc = zalloc64((size_t)w * h * sizeof(*rd->acc));
	rd->width = w;
	rd->height = h;
	nbh_rend_clraccum(rd);
	return rd->acc ? 0 : -1;
}

void nbh_rend_clraccum(struct nb_rdata *rd)
{
	if (rd->acc)
		memset(rd->acc, 0, (size_t)rd->width * rd->height *
		  sizeof(*rd->acc));
	rd->samples = 0;
}
