// Test infrastructure only: a headless driver for the reference renderer.
//
// Compiled together with the reference's own rend.c/util.c/... (see Makefile)
// into _ref/libnbref.so.  It replaces the SDL2 frame loop of main.c with
// plain entry points that tests and the CPU baseline call through ctypes:
//
//   refh_layout        sizeof/offsetof of the reference structs (rend.h:17-147)
//   refh_render_frame  N threads on rend_render, as main.c:409-412,424-426
//   refh_trace         intersect_tlas (rend.c:1976) over a ray batch, threaded
//   refh_trace_pckts   intersect_pckts_tlas (rend.c:2472) over 8-ray packets
//   refh_occluded      intersect_any_tlas (rend.c:2883) over a ray batch
//   refh_camrays       make_camray_pckt (rend.c:3293) for one image block
//
// Nothing here changes the reference's arithmetic; it only calls it.

#include <pthread.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <math.h>

#include "rend.h"
#include "util.h"

// Non-static functions of rend.c that rend.h does not declare.
void intersect_tlas(float *t, float *u, float *v, unsigned int *id,
                    float ox, float oy, float oz,
                    float dx, float dy, float dz,
                    struct bnode8 *nodes, struct rinst *insts,
                    unsigned int tlasofs);
void intersect_pckts_tlas(__m256 *t8, __m256 *u8, __m256 *v8, __m256i *id8,
                          __m256 *ox8, __m256 *oy8, __m256 *oz8,
                          __m256 *dx8, __m256 *dy8, __m256 *dz8,
                          unsigned char pcnt,
                          struct bnode8 *nodes, struct rinst *insts,
                          unsigned int tlasofs);
bool intersect_any_tlas(float tfar, float ox, float oy, float oz, float dx,
                        float dy, float dz, struct bnode8 *nodes,
                        struct rinst *insts, unsigned int tlasofs);
void make_camray_pckt(__m256 *ox8, __m256 *oy8, __m256 *oz8,
                      __m256 *dx8, __m256 *dy8, __m256 *dz8,
                      unsigned int x, unsigned int y,
                      __m256 xofs8, __m256 yofs8,
                      struct rcam *c, struct rngstate8 *rngstate);

#define OFS(T, f) ((unsigned long long)offsetof(struct T, f))

// Layout of the reference structs, for the C-ABI mirror check.
int refh_layout(unsigned long long *out, int cap)
{
	unsigned long long v[] = {
	  sizeof(struct rdata), OFS(rdata, mtls), OFS(rdata, tris),
	  OFS(rdata, nrms), OFS(rdata, instcnt), OFS(rdata, insts),
	  OFS(rdata, aabbs), OFS(rdata, bnodes), OFS(rdata, tlasofs),
	  OFS(rdata, cam), OFS(rdata, bgcol), OFS(rdata, width),
	  OFS(rdata, height), OFS(rdata, acc), OFS(rdata, buf),
	  OFS(rdata, blknum), OFS(rdata, rays), OFS(rdata, spp),
	  OFS(rdata, samples),
	  sizeof(struct rcam), OFS(rcam, eyex8), OFS(rcam, focrad8),
	  sizeof(struct bnode8), sizeof(struct leaf4), sizeof(struct rinst),
	  sizeof(struct rtri), sizeof(struct rnrm), sizeof(struct rmtl),
	  sizeof(struct aabb), OFS(leaf4, id4), OFS(leaf4, tricnt),
	  OFS(rinst, flags), OFS(rinst, triofs), OFS(rinst, tricnt)};
	int n = (int)(sizeof(v) / sizeof(*v));
	for (int i = 0; i < n && i < cap; i++)
		out[i] = v[i];
	return n;
}

struct frame_arg {
	struct rdata *rd;
};

static void *render_thread(void *a)
{
	rend_render(((struct frame_arg *)a)->rd);
	return NULL;
}

// One frame of the live renderer on nthreads threads (main.c:409-412), then
// the bookkeeping main.c does after the join (main.c:424-426).  Returns the
// ray count of the frame.
unsigned int refh_render_frame(struct rdata *rd, int nthreads)
{
	if (nthreads < 1)
		nthreads = 1;
	pthread_t *th = malloc(sizeof(*th) * (size_t)nthreads);
	struct frame_arg fa = {rd};
	for (int i = 0; i < nthreads; i++)
		pthread_create(&th[i], NULL, render_thread, &fa);
	for (int i = 0; i < nthreads; i++)
		pthread_join(th[i], NULL);
	free(th);
	unsigned int rays = rd->rays;
	rd->blknum = 0;
	rd->rays = 0;
	rd->samples += rd->spp;
	return rays;
}

// Rays: 8 floats each (ox oy oz tmax dx dy dz pad).  Hits: 4 words each
// (t u v id) with id = tri << 12 | inst as in rend.c:2109/890.
struct batch {
	const float *rays;
	unsigned int *hits; // t,u,v as float bits + id
	unsigned char *occl;
	unsigned int n;
	struct rdata *rd;
	int next; // atomic chunk counter
	int mode; // 0 closest, 1 any, 2 packets
};

#define CHUNK 256

// Direction-sign mask shared by the 8 rays of a packet, or -1 if they
// differ (iscohval3, rend.c:225-247).
static int packet_mask(const float *r)
{
	int m = -1;
	for (int k = 0; k < 8; k++) {
		const float *q = r + 8 * k;
		int mk = (int)signbit(q[4]) | (int)signbit(q[5]) << 1 |
		  (int)signbit(q[6]) << 2;
		if (m >= 0 && mk != m)
			return -1;
		m = mk;
	}
	return m;
}

static void trace_single(struct batch *b, unsigned int s, unsigned int e)
{
	struct rdata *rd = b->rd;
	for (unsigned int i = s; i < e; i++) {
		const float *r = b->rays + 8ull * i;
		float t = r[3], u = 0.0f, v = 0.0f;
		unsigned int id = 0;
		intersect_tlas(&t, &u, &v, &id, r[0], r[1], r[2], r[4], r[5],
		  r[6], rd->bnodes, rd->insts, rd->tlasofs);
		unsigned int *h = b->hits + 4ull * i;
		memcpy(&h[0], &t, 4);
		memcpy(&h[1], &u, 4);
		memcpy(&h[2], &v, 4);
		h[3] = id;
	}
}

static void trace_packets(struct batch *b, unsigned int p, unsigned int pc)
{
	struct rdata *rd = b->rd;
	__m256 ox8[16], oy8[16], oz8[16];
	__m256 dx8[16], dy8[16], dz8[16];
	__m256 t8[16], u8[16], v8[16];
	__m256i id8[16];
	for (unsigned int j = 0; j < pc; j++) {
		for (int k = 0; k < 8; k++) {
			const float *r = b->rays + 8ull * (p + 8 * j + k);
			ox8[j][k] = r[0];
			oy8[j][k] = r[1];
			oz8[j][k] = r[2];
			dx8[j][k] = r[4];
			dy8[j][k] = r[5];
			dz8[j][k] = r[6];
			t8[j][k] = r[3];
			u8[j][k] = 0.0f;
			v8[j][k] = 0.0f;
		}
		id8[j] = _mm256_setzero_si256();
	}
	intersect_pckts_tlas(t8, u8, v8, id8, ox8, oy8, oz8, dx8, dy8, dz8,
	  (unsigned char)pc, rd->bnodes, rd->insts, rd->tlasofs);
	for (unsigned int j = 0; j < pc; j++)
		for (int k = 0; k < 8; k++) {
			unsigned int *h = b->hits + 4ull * (p + 8 * j + k);
			memcpy(&h[0], &t8[j][k], 4);
			memcpy(&h[1], &u8[j][k], 4);
			memcpy(&h[2], &v8[j][k], 4);
			h[3] = ((unsigned int *)&id8[j])[k];
		}
}

static void *trace_thread(void *a)
{
	struct batch *b = a;
	struct rdata *rd = b->rd;
	while (1) {
		int c = __atomic_fetch_add(&b->next, 1, __ATOMIC_SEQ_CST);
		unsigned int s = (unsigned int)c * CHUNK;
		if (s >= b->n)
			break;
		unsigned int e = s + CHUNK < b->n ? s + CHUNK : b->n;
		if (b->mode == 2) {
			// Packets of 8 consecutive rays, traced the way rend_render
			// groups them (rend.c:3636-3700): runs of up to 16 packets
			// whose rays all share one direction-sign mask go to
			// intersect_pckts_tlas, an incoherent packet goes ray by ray
			// to intersect_tlas.  n is a multiple of 8.
			unsigned int p = s;
			while (p < e) {
				unsigned int run = 0;
				int mask0 = -1;
				while (p + 8 * run < e && run < 16) {
					int m = packet_mask(b->rays + 8ull * (p + 8 * run));
					if (m < 0 || (mask0 >= 0 && m != mask0))
						break;
					mask0 = m;
					run++;
				}
				if (run == 0) {
					trace_single(b, p, p + 8);
					p += 8;
					continue;
				}
				trace_packets(b, p, run);
				p += 8 * run;
			}
			continue;
		}
		for (unsigned int i = s; i < e; i++) {
			const float *r = b->rays + 8ull * i;
			if (b->mode == 1) {
				b->occl[i] = intersect_any_tlas(r[3], r[0],
				  r[1], r[2], r[4], r[5], r[6], rd->bnodes,
				  rd->insts, rd->tlasofs);
				continue;
			}
			float t = r[3], u = 0.0f, v = 0.0f;
			unsigned int id = 0;
			intersect_tlas(&t, &u, &v, &id, r[0], r[1], r[2],
			  r[4], r[5], r[6], rd->bnodes, rd->insts,
			  rd->tlasofs);
			unsigned int *h = b->hits + 4ull * i;
			memcpy(&h[0], &t, 4);
			memcpy(&h[1], &u, 4);
			memcpy(&h[2], &v, 4);
			h[3] = id;
		}
	}
	return NULL;
}

static void run_batch(struct batch *b, int nthreads)
{
	if (nthreads < 1)
		nthreads = 1;
	pthread_t *th = malloc(sizeof(*th) * (size_t)nthreads);
	for (int i = 0; i < nthreads; i++)
		pthread_create(&th[i], NULL, trace_thread, b);
	for (int i = 0; i < nthreads; i++)
		pthread_join(th[i], NULL);
	free(th);
}

void refh_trace(struct rdata *rd, const float *rays, unsigned int n,
                unsigned int *hits, int nthreads)
{
	struct batch b = {rays, hits, NULL, n, rd, 0, 0};
	run_batch(&b, nthreads);
}

void refh_trace_pckts(struct rdata *rd, const float *rays, unsigned int n,
                      unsigned int *hits, int nthreads)
{
	struct batch b = {rays, hits, NULL, n, rd, 0, 2};
	run_batch(&b, nthreads);
}

void refh_occluded(struct rdata *rd, const float *rays, unsigned int n,
                   unsigned char *occl, int nthreads)
{
	struct batch b = {rays, NULL, occl, n, rd, 0, 1};
	run_batch(&b, nthreads);
}

// Camera rays of one 4x2 packet at pixel (x, y), drawn the way rend_render
// draws them (rend.c:3627, 3642): the caller passes the reseed values.
// Output: 8 rays of 8 floats (ox oy oz FLT_MAX dx dy dz 0), packet lane order
// pcktxofs8/pcktyofs8 (rend.c:131-132): lanes 0-3 row y, lanes 4-7 row y+1.
void refh_camrays(struct rdata *rd, unsigned int x, unsigned int y,
                  unsigned long long seed0, unsigned long long seed1,
                  unsigned int npckts, const unsigned int *pxy, float *out)
{
	struct rngstate8 rng;
	rand8_init(&rng, seed0, seed1);
	__m256 xo = _mm256_set_ps(3, 2, 1, 0, 3, 2, 1, 0);
	__m256 yo = _mm256_set_ps(1, 1, 1, 1, 0, 0, 0, 0);
	for (unsigned int p = 0; p < npckts; p++) {
		__m256 ox8, oy8, oz8, dx8, dy8, dz8;
		unsigned int px = pxy ? pxy[2 * p] : x;
		unsigned int py = pxy ? pxy[2 * p + 1] : y;
		make_camray_pckt(&ox8, &oy8, &oz8, &dx8, &dy8, &dz8, px, py,
		  xo, yo, &rd->cam, &rng);
		for (int k = 0; k < 8; k++) {
			float *r = out + 64ull * p + 8 * k;
			r[0] = ox8[k];
			r[1] = oy8[k];
			r[2] = oz8[k];
			r[3] = FLT_MAX;
			r[4] = dx8[k];
			r[5] = dy8[k];
			r[6] = dz8[k];
			r[7] = 0.0f;
		}
	}
}

// Import a glTF file with nodebleed's own importer (imp_gltf_f,
// gltfimp.c:415) and report what the render-data bridge would take from it
// (cpy_rdata main.c:53, upd_rinsts main.c:117, the camera of
// scene_updcams scene.c:411).  counts: [0] meshes, [1] vertices, [2]
// indices, [3] materials, [4] mesh nodes.  With non-NULL buffers it also
// copies, mesh after mesh: vertices and normals (3 floats each), indices
// (mesh-local), the material of each triangle; per material col, metallic,
// roughness, ior and the flags as a float's bits (7 floats); per mesh node
// its mesh and its world matrix (16 floats); the camera's eye, fwd, ri, up
// and vfov (13 floats).  Buffers must hold the counts of a first call.
#include "scene.h"
#include "gltfimp.h"
#include "types.h"

int refh_gltf_import(const char *path, unsigned int *counts, float *vrts,
                     float *nrms, unsigned int *inds, unsigned int *trimtl,
                     float *mtls, unsigned int *node_mesh, float *globs,
                     float *cam)
{
	struct scene s;
	memset(&s, 0, sizeof(s));
	char name[4096];
	size_t n = strlen(path);
	if (n >= sizeof(name))
		return -1;
	memcpy(name, path, n + 1);
	imp_gltf_f(&s, name);
	scene_updtransforms(&s);
	scene_updcams(&s);
	unsigned int nv = 0, ni = 0, nn = 0;
	for (unsigned int k = 0; k < s.meshcnt; k++) {
		nv += s.meshes[k].vcnt;
		ni += s.meshes[k].icnt;
	}
	for (unsigned int i = 0; i < s.nodecnt; i++)
		if (s.objs[i].flags & MESH)
			nn++;
	counts[0] = s.meshcnt;
	counts[1] = nv;
	counts[2] = ni;
	counts[3] = s.mtlcnt;
	counts[4] = nn;
	if (vrts) {
		unsigned int v = 0, ix = 0, t = 0;
		for (unsigned int k = 0; k < s.meshcnt; k++) {
			struct mesh *m = &s.meshes[k];
			memcpy(vrts + 3ull * v, m->vrts, 12ull * m->vcnt);
			memcpy(nrms + 3ull * v, m->nrms, 12ull * m->vcnt);
			memcpy(inds + ix, m->inds, 4ull * m->icnt);
			for (unsigned int j = 0; j < m->mcnt; j++)
				for (unsigned int q = 0; q < m->mtls[j].tricnt; q++)
					trimtl[t++] = m->mtls[j].mtlid;
			v += m->vcnt;
			ix += m->icnt;
		}
		for (unsigned int i = 0; i < s.mtlcnt; i++) {
			struct mtl *m = &s.mtls[i];
			float *o = mtls + 7ull * i;
			o[0] = m->col.x;
			o[1] = m->col.y;
			o[2] = m->col.z;
			o[3] = m->metallic;
			o[4] = m->roughness;
			o[5] = m->ior;
			memcpy(&o[6], &m->flags, 4);
		}
		unsigned int q = 0;
		for (unsigned int i = 0; i < s.nodecnt; i++)
			if (s.objs[i].flags & MESH) {
				node_mesh[q] = (unsigned int)s.objs[i].objid;
				memcpy(globs + 16ull * q, s.tfmats[i].glob, 64);
				q++;
			}
		struct cam *c = &s.cams[s.currcam];
		float cv[13] = {c->eye.x, c->eye.y, c->eye.z, c->fwd.x, c->fwd.y,
		  c->fwd.z, c->ri.x, c->ri.y, c->ri.z, c->up.x, c->up.y, c->up.z,
		  c->vfov};
		memcpy(cam, cv, sizeof(cv));
	}
	scene_release(&s);
	return 0;
}

// rend.c:171, declared by main.c:114.
void mulpos(float *ox, float *oy, float *oz, float m[16], float x, float y,
            float z);

// A render data built entirely by nodebleed's own host code from a glTF
// file, in the order its frame loop runs (main.c:226-249, 252-270):
// imp_gltf_f, rend_init, rend_resaccum, the mesh/material/instance copy,
// rend_prepstatic, scene_updtransforms and scene_updcams, the instance
// update, rend_prepdynamic and the camera constants.  The copy (cpy_rdata
// main.c:53-112), the instance update (upd_rinsts main.c:117-157) and the
// camera constants (upd_rcam main.c:159-195) sit in main.c, which needs
// SDL2, so their steps are written out below; they call the reference's own
// mat4_inv, mulpos and bcmin8/bcmax8.  NULL on failure; free with
// refh_rdata_free.  rend_staticinit must have run.
struct rdata *refh_gltf_rdata(const char *path, unsigned int w,
                              unsigned int h, unsigned int spp)
{
	struct scene s;
	memset(&s, 0, sizeof(s));
	char name[4096];
	size_t len = strlen(path);
	if (len >= sizeof(name))
		return NULL;
	memcpy(name, path, len + 1);
	imp_gltf_f(&s, name);
	s.bgcol = (struct vec3){0.4f, 0.4f, 0.4f}; // main.c:230
	unsigned int maxtris = 0, maxinsts = 0;
	for (unsigned int k = 0; k < s.meshcnt; k++)
		maxtris += s.meshes[k].icnt / 3;
	for (unsigned int i = 0; i < s.nodecnt; i++)
		if (s.objs[i].flags & MESH)
			maxinsts++;
	struct rdata *rd = aligned_alloc(64, (sizeof(*rd) + 63) & ~(size_t)63);
	if (!rd) {
		scene_release(&s);
		return NULL;
	}
	memset(rd, 0, sizeof(*rd));
	rend_init(rd, s.mtlmax, maxtris, maxinsts, spp);
	rend_resaccum(rd, w, h);

	// meshes: triangles and per-triangle normals with the material of
	// their run; each mesh's first triangle and count
	unsigned int *triofs = calloc(s.meshcnt ? s.meshcnt : 1, sizeof(int));
	unsigned int *tricnt = calloc(s.meshcnt ? s.meshcnt : 1, sizeof(int));
	unsigned int t = 0;
	for (unsigned int k = 0; k < s.meshcnt; k++) {
		const struct mesh *m = &s.meshes[k];
		const unsigned int *ix = m->inds;
		triofs[k] = t;
		for (unsigned int r = 0; r < m->mcnt; r++)
			for (unsigned int q = 0; q < m->mtls[r].tricnt; q++) {
				rd->tris[t].v0 = m->vrts[ix[0]];
				rd->tris[t].v1 = m->vrts[ix[1]];
				rd->tris[t].v2 = m->vrts[ix[2]];
				rd->nrms[t].n0 = m->nrms[ix[0]];
				rd->nrms[t].n1 = m->nrms[ix[1]];
				rd->nrms[t].n2 = m->nrms[ix[2]];
				rd->nrms[t].mtlid = m->mtls[r].mtlid;
				ix += 3;
				t++;
			}
		tricnt[k] = m->icnt / 3;
	}
	for (unsigned int i = 0; i < s.mtlcnt; i++)
		memcpy(&rd->mtls[i], &s.mtls[i], sizeof(*rd->mtls));
	unsigned int n = 0;
	for (unsigned int i = 0; i < s.nodecnt; i++) {
		struct obj *o = &s.objs[i];
		if (!(o->flags & MESH))
			continue;
		memset(&rd->insts[n], 0, sizeof(rd->insts[n]));
		rd->insts[n].flags = o->flags;
		rd->insts[n].triofs = triofs[o->objid];
		rd->insts[n].tricnt = tricnt[o->objid];
		o->instid = (int)n++;
	}
	rd->instcnt = n;
	rd->bgcol = s.bgcol;
	free(triofs);
	free(tricnt);

	rend_prepstatic(rd);
	scene_updtransforms(&s);
	scene_updcams(&s);

	// instances: world->object 3x4 from the inverse of the node's matrix,
	// world box from the 8 corners of the BLAS root's box after the matrix
	for (unsigned int i = 0; i < s.nodecnt; i++) {
		struct obj *o = &s.objs[i];
		if (!(o->flags & MESH))
			continue;
		struct rinst *ri = &rd->insts[o->instid];
		float *g = s.tfmats[i].glob;
		float inv[16];
		mat4_inv(inv, g);
		memcpy(ri->globinv, inv, sizeof(ri->globinv));
		struct bnode8 *root = &rd->bnodes[ri->triofs << 1];
		float lo[3] = {bcmin8(root->minx8)[0], bcmin8(root->miny8)[0],
		  bcmin8(root->minz8)[0]};
		float hi[3] = {bcmax8(root->maxx8)[0], bcmax8(root->maxy8)[0],
		  bcmax8(root->maxz8)[0]};
		struct vec3 mi = {FLT_MAX, FLT_MAX, FLT_MAX};
		struct vec3 ma = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
		for (int c = 0; c < 8; c++) {
			struct vec3 v;
			mulpos(&v.x, &v.y, &v.z, g, c & 1 ? lo[0] : hi[0],
			  c & 2 ? lo[1] : hi[1], c & 4 ? lo[2] : hi[2]);
			mi = vec3_min(mi, v);
			ma = vec3_max(ma, v);
		}
		rd->aabbs[o->instid] = (struct aabb){.min = mi, .max = ma};
	}
	rend_prepdynamic(rd);

	// camera constants of the current camera
	const struct cam *c = &s.cams[s.currcam];
	float aspect = (float)w / (float)h;
	float tv = tanf(0.5f * c->vfov * PI / 180.0f);
	float tf = tanf(0.5f * c->focangle * PI / 180.0f);
	struct rcam *rc = &rd->cam;
	memset(rc, 0, sizeof(*rc));
	rc->eye = c->eye;
	rc->tanvfov = tv;
	rc->ri = c->ri;
	rc->focdist = c->focdist;
	rc->up = c->up;
	rc->tanfangle = tf;
	rc->fwd = c->fwd;
	rc->aspect = aspect;
	rc->eyex8 = _mm256_set1_ps(c->eye.x);
	rc->eyey8 = _mm256_set1_ps(c->eye.y);
	rc->eyez8 = _mm256_set1_ps(c->eye.z);
	rc->rix8 = _mm256_set1_ps(c->ri.x);
	rc->riy8 = _mm256_set1_ps(c->ri.y);
	rc->riz8 = _mm256_set1_ps(c->ri.z);
	rc->upx8 = _mm256_set1_ps(c->up.x);
	rc->upy8 = _mm256_set1_ps(c->up.y);
	rc->upz8 = _mm256_set1_ps(c->up.z);
	rc->fwdx8 = _mm256_set1_ps(c->fwd.x);
	rc->fwdy8 = _mm256_set1_ps(c->fwd.y);
	rc->fwdz8 = _mm256_set1_ps(c->fwd.z);
	rc->rw8 = _mm256_set1_ps(1.0f / (float)w);
	rc->rh8 = _mm256_set1_ps(1.0f / (float)h);
	rc->aspect8 = _mm256_set1_ps(aspect);
	rc->fdist8 = _mm256_set1_ps(c->focdist);
	rc->fovfdist8 = _mm256_set1_ps(2.0f * tv * c->focdist);
	rc->focangle8 = _mm256_set1_ps(tf);
	rc->focrad8 = _mm256_set1_ps(tf * c->focdist);
	scene_release(&s);
	return rd;
}

void refh_rdata_free(struct rdata *rd)
{
	if (!rd)
		return;
	rend_release(rd);
	free(rd);
}
