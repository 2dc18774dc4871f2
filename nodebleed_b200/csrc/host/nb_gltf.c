// glTF 2.0 scenes for the host library: a loader that turns a .gltf + .bin
// pair straight into the host scene (nbh_scene) the render-data bridge
// flattens, and a writer for the synthetic scenes.
//
// The loader reads the subset nodebleed's own importer reads (gltf.h:4-11,
// gltfimp.c:125-435): one external binary buffer; per mesh primitive a
// float VEC3 POSITION and NORMAL and u8/u16/u32 indices, each primitive a
// run of one material (imp_mesh, gltfimp.c:125-242); materials from
// pbrMetallicRoughness.baseColorFactor/metallicFactor/roughnessFactor,
// emissiveFactor times KHR_materials_emissive_strength (an emissive material
// takes its emission as colour, imp_mtl gltfimp.c:110-123),
// KHR_materials_ior and KHR_materials_transmission (refractive flag); nodes
// with translation / rotation (quaternion xyzw) / scale, composed
// T * R * S under their parent, from the roots of the default scene; the
// first perspective camera (yfov), its node's -Z the view direction.  No
// camera: a proxy camera on the scene root (identity transform) with the
// reference's vfov quirk (gltfimp.c:377-380, radians passed as degrees).
// Animations are not read.
// Beyond the reference's subset it accepts a node "matrix", and the
// exact-transform extras the writer emits ("extras": {"nodebleed":
// {"glob": [16 row-major floats]}} per node, and the camera vectors on the
// camera node), so a written scene loads back bit for bit.
//
// The JSON reader is a small tokenizer of this library: a flat token array
// in document order, each token knowing where its subtree ends.

#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "nb_host.h"

// ----------------------------------------------------------------- JSON --

enum { J_OBJ, J_ARR, J_STR, J_NUM, J_LIT };

struct jtok {
	int type;
	int start, end; // content bytes (strings without quotes)
	int n;          // object: key/value pairs; array: elements
	int next;       // index of the first token after this subtree
};

struct jdoc {
	const char  *s;
	size_t       len;
	struct jtok *t;
	int          nt, cap;
	size_t       pos;
	int          depth;
};

static int j_new(struct jdoc *d, int type, int start)
{
	if (d->nt == d->cap) {
		int cap = d->cap ? 2 * d->cap : 1024;
		struct jtok *p = realloc(d->t, sizeof(*p) * (size_t)cap);
		if (!p)
			return -1;
		d->t = p;
		d->cap = cap;
	}
	struct jtok *k = &d->t[d->nt];
	k->type = type;
	k->start = k->end = start;
	k->n = 0;
	k->next = d->nt + 1;
	return d->nt++;
}

static void j_ws(struct jdoc *d)
{
	while (d->pos < d->len && isspace((unsigned char)d->s[d->pos]))
		d->pos++;
}

static int j_value(struct jdoc *d);

static int j_string(struct jdoc *d)
{
	size_t p = ++d->pos; // after the quote
	while (p < d->len && d->s[p] != '"') {
		if (d->s[p] == '\\')
			p++;
		p++;
	}
	if (p >= d->len)
		return -1;
	int k = j_new(d, J_STR, (int)d->pos);
	if (k < 0)
		return -1;
	d->t[k].end = (int)p;
	d->pos = p + 1;
	return k;
}

static int j_value(struct jdoc *d)
{
	j_ws(d);
	if (d->pos >= d->len || ++d->depth > 64)
		return -1;
	char c = d->s[d->pos];
	int k;
	if (c == '{' || c == '[') {
		int obj = c == '{';
		k = j_new(d, obj ? J_OBJ : J_ARR, (int)d->pos);
		if (k < 0)
			return -1;
		d->pos++;
		j_ws(d);
		if (d->pos < d->len && d->s[d->pos] == (obj ? '}' : ']')) {
			d->pos++;
		} else {
			for (;;) {
				if (obj) {
					j_ws(d);
					if (d->pos >= d->len || d->s[d->pos] != '"' ||
					  j_string(d) < 0)
						return -1;
					j_ws(d);
					if (d->pos >= d->len || d->s[d->pos] != ':')
						return -1;
					d->pos++;
				}
				if (j_value(d) < 0)
					return -1;
				d->t[k].n++;
				j_ws(d);
				if (d->pos >= d->len)
					return -1;
				if (d->s[d->pos] == ',') {
					d->pos++;
					continue;
				}
				if (d->s[d->pos] != (obj ? '}' : ']'))
					return -1;
				d->pos++;
				break;
			}
		}
	} else if (c == '"') {
		k = j_string(d);
		if (k < 0)
			return -1;
	} else {
		size_t p = d->pos;
		while (p < d->len && (isalnum((unsigned char)d->s[p]) ||
		  d->s[p] == '-' || d->s[p] == '+' || d->s[p] == '.'))
			p++;
		if (p == d->pos)
			return -1;
		k = j_new(d, (c == '-' || isdigit((unsigned char)c)) ? J_NUM :
		  J_LIT, (int)d->pos);
		if (k < 0)
			return -1;
		d->t[k].end = (int)p;
		d->pos = p;
	}
	d->t[k].next = d->nt;
	d->depth--;
	return k;
}

static int j_parse(struct jdoc *d, const char *s, size_t len)
{
	memset(d, 0, sizeof(*d));
	d->s = s;
	d->len = len;
	return j_value(d) == 0 ? 0 : -1;
}

static int j_eq(const struct jdoc *d, int k, const char *str)
{
	size_t n = strlen(str);
	return d->t[k].type == J_STR &&
	  (size_t)(d->t[k].end - d->t[k].start) == n &&
	  memcmp(d->s + d->t[k].start, str, n) == 0;
}

// Value of key `key` in object token `obj`, or -1.
static int j_get(const struct jdoc *d, int obj, const char *key)
{
	if (obj < 0 || d->t[obj].type != J_OBJ)
		return -1;
	int k = obj + 1;
	for (int i = 0; i < d->t[obj].n; i++) {
		int v = k + 1;
		if (j_eq(d, k, key))
			return v;
		k = d->t[v].next;
	}
	return -1;
}

// Element i of array token `arr`, or -1.
static int j_at(const struct jdoc *d, int arr, int i)
{
	if (arr < 0 || d->t[arr].type != J_ARR || i < 0 || i >= d->t[arr].n)
		return -1;
	int k = arr + 1;
	while (i--)
		k = d->t[k].next;
	return k;
}

static int j_len(const struct jdoc *d, int arr)
{
	return arr >= 0 && d->t[arr].type == J_ARR ? d->t[arr].n : 0;
}

static double j_num(const struct jdoc *d, int k, double dflt)
{
	if (k < 0 || d->t[k].type != J_NUM)
		return dflt;
	char buf[64];
	int n = d->t[k].end - d->t[k].start;
	if (n <= 0 || n >= (int)sizeof(buf))
		return dflt;
	memcpy(buf, d->s + d->t[k].start, (size_t)n);
	buf[n] = '\0';
	return strtod(buf, NULL);
}

// n numbers of array `arr` into out (as floats); 0 if the array has them.
static int j_floats(const struct jdoc *d, int arr, float *out, int n)
{
	if (j_len(d, arr) < n)
		return -1;
	for (int i = 0; i < n; i++) {
		int k = j_at(d, arr, i);
		if (d->t[k].type != J_NUM)
			return -1;
		out[i] = (float)j_num(d, k, 0.0);
	}
	return 0;
}

// ---------------------------------------------------------------- files --

static char *read_file(const char *path, size_t *len)
{
	FILE *f = fopen(path, "rb");
	if (!f)
		return NULL;
	char *buf = NULL;
	if (fseek(f, 0, SEEK_END) == 0) {
		long n = ftell(f);
		if (n >= 0 && fseek(f, 0, SEEK_SET) == 0) {
			buf = malloc((size_t)n + 1);
			if (buf && fread(buf, 1, (size_t)n, f) != (size_t)n) {
				free(buf);
				buf = NULL;
			} else if (buf) {
				buf[n] = '\0';
				*len = (size_t)n;
			}
		}
	}
	fclose(f);
	return buf;
}

// dir of `path` (with its slash) + name
static char *sibling(const char *path, const char *name, size_t nlen)
{
	const char *sl = strrchr(path, '/');
	size_t dl = sl ? (size_t)(sl - path + 1) : 0;
	char *out = malloc(dl + nlen + 1);
	if (!out)
		return NULL;
	memcpy(out, path, dl);
	memcpy(out + dl, name, nlen);
	out[dl + nlen] = '\0';
	return out;
}

// ------------------------------------------------------------- loading --

struct gl_view {
	uint32_t off, len, stride;
};

struct gl_acc {
	int      view;
	uint32_t off, cnt, comp;
	int      ncomp;
};

struct gl_load {
	struct jdoc      d;
	const uint8_t   *bin;
	size_t           binlen;
	struct gl_view  *views;
	int              nviews;
	struct gl_acc   *accs;
	int              naccs;
	struct nbh_scene *s;
	unsigned int     flags;
	int              cam_done;
	unsigned int     instcap;
	int              err;
	uint8_t         *seen;   // per node: reached from a scene root
};

// Integer fields: the default when absent; a number that is not an integer
// within [lo, hi] sets L->err, which fails the load, and gives the default
// (instead of an out-of-range conversion to int, undefined in C).
static double j_intval(struct gl_load *L, int k, double dflt, double lo,
                       double hi)
{
	double v = j_num(&L->d, k, dflt);
	if (k >= 0 && L->d.t[k].type == J_NUM &&
	  !(v >= lo && v <= hi && v == floor(v))) {
		L->err = 1;
		return dflt;
	}
	return v;
}

static int j_index(struct gl_load *L, int k, int dflt)
{
	return (int)j_intval(L, k, dflt, 0.0, 2147483647.0);
}

static uint32_t j_u32(struct gl_load *L, int k, uint32_t dflt)
{
	return (uint32_t)j_intval(L, k, dflt, 0.0, 4294967295.0);
}

static int comp_size(uint32_t c)
{
	return c == 5121 ? 1 : c == 5123 ? 2 : c == 5125 || c == 5126 ? 4 : 0;
}

// Byte address of element i of accessor a, or NULL out of range.
static const uint8_t *acc_elem(const struct gl_load *L, int a, uint32_t i,
                               int elem_bytes)
{
	if (a < 0 || a >= L->naccs)
		return NULL;
	const struct gl_acc *A = &L->accs[a];
	if (A->view < 0 || A->view >= L->nviews || i >= A->cnt)
		return NULL;
	const struct gl_view *V = &L->views[A->view];
	uint32_t stride = V->stride ? V->stride : (uint32_t)elem_bytes;
	uint64_t at = (uint64_t)V->off + A->off + (uint64_t)i * stride;
	if (at + (uint64_t)elem_bytes > L->binlen ||
	    (uint64_t)A->off + (uint64_t)i * stride + elem_bytes > V->len)
		return NULL;
	return L->bin + at;
}

static int load_materials(struct gl_load *L)
{
	const struct jdoc *d = &L->d;
	int arr = j_get(d, 0, "materials");
	int n = j_len(d, arr);
	struct nbh_scene *s = L->s;
	s->mtlcnt = n > 0 ? (unsigned int)n : 1u;
	s->mtls = calloc(s->mtlcnt, sizeof(*s->mtls));
	if (!s->mtls)
		return -1;
	if (n == 0) {
		// no materials: the reference's default (gltfimp.c:354-357)
		s->mtls[0].col = (struct nb_vec3){0.5f, 0.0f, 0.5f};
		s->mtls[0].roughness = 0.5f;
		s->mtls[0].ior = 1.5f;
		return 0;
	}
	for (int i = 0; i < n; i++) {
		int m = j_at(d, arr, i);
		struct nb_rmtl *o = &s->mtls[i];
		// the reference reader's defaults (read_mtl, gltf.c:176-190):
		// metallic 0, roughness 0.5, ior 1.5, emission factor 1 and
		// strength 0 (no KHR_materials_emissive_strength: not emissive)
		float col[4] = {1.0f, 1.0f, 1.0f, 1.0f}, em[3] = {1, 1, 1};
		o->metallic = 0.0f;
		o->roughness = 0.5f;
		o->ior = 1.5f;
		int pbr = j_get(d, m, "pbrMetallicRoughness");
		if (pbr >= 0) {
			int c = j_get(d, pbr, "baseColorFactor");
			if (c >= 0 && j_floats(d, c, col, 4))
				return -1;
			o->metallic = (float)j_num(d, j_get(d, pbr, "metallicFactor"),
			  0.0);
			o->roughness = (float)j_num(d, j_get(d, pbr,
			  "roughnessFactor"), 0.5);
		}
		int e = j_get(d, m, "emissiveFactor");
		if (e >= 0 && j_floats(d, e, em, 3))
			return -1;
		int ext = j_get(d, m, "extensions");
		float strength = (float)j_num(d, j_get(d, j_get(d, ext,
		  "KHR_materials_emissive_strength"), "emissiveStrength"), 0.0);
		for (int a = 0; a < 3; a++)
			em[a] *= strength;
		o->ior = (float)j_num(d, j_get(d, j_get(d, ext,
		  "KHR_materials_ior"), "ior"), 1.5);
		float tr = (float)j_num(d, j_get(d, j_get(d, ext,
		  "KHR_materials_transmission"), "transmissionFactor"), 0.0);
		o->col = (struct nb_vec3){col[0], col[1], col[2]};
		o->flags = 0;
		if (tr != 0.0f)
			o->flags |= 0x2000u; // REFRACTIVE (types.h)
		if (em[0] + em[1] + em[2] > 0.0f) {
			o->flags |= NB_FLAG_EMISSIVE;
			o->col = (struct nb_vec3){em[0], em[1], em[2]};
		}
	}
	return 0;
}

// One glTF mesh: every primitive's vertices and triangles appended, each
// primitive a run of its material (imp_mesh, gltfimp.c:125-242).
static int load_mesh(struct gl_load *L, int mesh, struct nbh_mesh *o)
{
	const struct jdoc *d = &L->d;
	int prims = j_get(d, mesh, "primitives");
	int np = j_len(d, prims);
	uint64_t vcnt = 0, icnt = 0;
	for (int p = 0; p < np; p++) {
		int pr = j_at(d, prims, p);
		int attr = j_get(d, pr, "attributes");
		int pa = j_index(L, j_get(d, attr, "POSITION"), -1);
		int ia = j_index(L, j_get(d, pr, "indices"), -1);
		if (pa < 0 || pa >= L->naccs || ia < 0 || ia >= L->naccs)
			return -1;
		vcnt += L->accs[pa].cnt;
		icnt += L->accs[ia].cnt;
	}
	if (vcnt == 0 || icnt < 3 || vcnt > 0xffffffffu || icnt > 0xffffffffu)
		return -1;
	memset(o, 0, sizeof(*o));
	o->vrts = malloc(sizeof(float) * 3 * vcnt);
	o->nrms = malloc(sizeof(float) * 3 * vcnt);
	o->inds = malloc(sizeof(unsigned int) * icnt);
	o->tmtl = malloc(sizeof(unsigned int) * (icnt / 3 + 1));
	if (!o->vrts || !o->nrms || !o->inds || !o->tmtl)
		return -1;
	for (int p = 0; p < np; p++) {
		int pr = j_at(d, prims, p);
		int attr = j_get(d, pr, "attributes");
		int pa = j_index(L, j_get(d, attr, "POSITION"), -1);
		int na = j_index(L, j_get(d, attr, "NORMAL"), -1);
		int ia = j_index(L, j_get(d, pr, "indices"), -1);
		int mi = j_index(L, j_get(d, pr, "material"), 0);
		if (mi < 0 || (unsigned int)mi >= L->s->mtlcnt)
			mi = 0;
		// POSITION and NORMAL: float VEC3; indices: u8/u16/u32 SCALAR
		if (na < 0 || na >= L->naccs || L->accs[pa].comp != 5126 ||
		  L->accs[pa].ncomp != 3 || L->accs[na].comp != 5126 ||
		  L->accs[na].ncomp != 3 || L->accs[na].cnt != L->accs[pa].cnt ||
		  L->accs[ia].ncomp != 1 || comp_size(L->accs[ia].comp) == 0 ||
		  L->accs[ia].comp == 5126 || L->accs[ia].cnt % 3)
			return -1;
		uint32_t base = o->vcnt;
		for (uint32_t i = 0; i < L->accs[pa].cnt; i++) {
			const uint8_t *pv = acc_elem(L, pa, i, 12);
			const uint8_t *pn = acc_elem(L, na, i, 12);
			if (!pv || !pn)
				return -1;
			memcpy(&o->vrts[3 * (size_t)(base + i)], pv, 12);
			memcpy(&o->nrms[3 * (size_t)(base + i)], pn, 12);
		}
		int cs = comp_size(L->accs[ia].comp);
		for (uint32_t i = 0; i < L->accs[ia].cnt; i++) {
			const uint8_t *pi = acc_elem(L, ia, i, cs);
			if (!pi)
				return -1;
			uint32_t v = cs == 1 ? pi[0] : cs == 2 ?
			  (uint32_t)(pi[0] | pi[1] << 8) :
			  (uint32_t)pi[0] | (uint32_t)pi[1] << 8 |
			  (uint32_t)pi[2] << 16 | (uint32_t)pi[3] << 24;
			if (v >= L->accs[pa].cnt)
				return -1;
			o->inds[o->icnt + i] = base + v;
		}
		for (uint32_t t = 0; t < L->accs[ia].cnt / 3; t++)
			o->tmtl[o->icnt / 3 + t] = (unsigned int)mi;
		o->icnt += L->accs[ia].cnt;
		o->vcnt += L->accs[pa].cnt;
		if (p == 0)
			o->mtlid = (unsigned int)mi;
	}
	return 0;
}

static void mat4_mul_f(float dst[16], const float a[16], const float b[16])
{
	float r[16];
	for (int i = 0; i < 4; i++)
		for (int j = 0; j < 4; j++)
			r[4 * i + j] = a[4 * i] * b[j] + a[4 * i + 1] * b[4 + j] +
			  a[4 * i + 2] * b[8 + j] + a[4 * i + 3] * b[12 + j];
	memcpy(dst, r, sizeof(r));
}

// Local matrix of a node (row-major): matrix, else T * R * S.
static int node_local(const struct jdoc *d, int node, float m[16])
{
	int mk = j_get(d, node, "matrix");
	if (mk >= 0) {
		float c[16];
		if (j_floats(d, mk, c, 16))
			return -1;
		for (int i = 0; i < 4; i++) // glTF stores columns
			for (int j = 0; j < 4; j++)
				m[4 * i + j] = c[4 * j + i];
		return 0;
	}
	float t[3] = {0, 0, 0}, q[4] = {0, 0, 0, 1}, s[3] = {1, 1, 1};
	int k;
	if ((k = j_get(d, node, "translation")) >= 0 && j_floats(d, k, t, 3))
		return -1;
	if ((k = j_get(d, node, "rotation")) >= 0 && j_floats(d, k, q, 4))
		return -1;
	if ((k = j_get(d, node, "scale")) >= 0 && j_floats(d, k, s, 3))
		return -1;
	float x = q[0], y = q[1], z = q[2], w = q[3];
	float R[9] = {
	  1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
	  2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
	  2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)};
	for (int i = 0; i < 3; i++) {
		for (int j = 0; j < 3; j++)
			m[4 * i + j] = R[3 * i + j] * s[j];
		m[4 * i + 3] = t[i];
	}
	m[12] = m[13] = m[14] = 0.0f;
	m[15] = 1.0f;
	return 0;
}

static void unit3(float v[3])
{
	float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
	if (l > 0.0f)
		for (int a = 0; a < 3; a++)
			v[a] /= l;
}

// Camera from its node's world matrix (calc_cam, scene.c:400-409): eye at
// the translation, fwd = unit(-Z column), ri = unit(fwd x +Y),
// up = unit(ri x fwd).
static void cam_from(struct nbh_cam *c, const float g[16], float vfov)
{
	float f[3] = {-g[2], -g[6], -g[10]};
	unit3(f);
	float ri[3] = {f[1] * 0.0f - f[2] * 1.0f, f[2] * 0.0f - f[0] * 0.0f,
	  f[0] * 1.0f - f[1] * 0.0f};
	unit3(ri);
	float up[3] = {ri[1] * f[2] - ri[2] * f[1], ri[2] * f[0] - ri[0] * f[2],
	  ri[0] * f[1] - ri[1] * f[0]};
	unit3(up);
	c->eye = (struct nb_vec3){g[3], g[7], g[11]};
	c->fwd = (struct nb_vec3){f[0], f[1], f[2]};
	c->ri = (struct nb_vec3){ri[0], ri[1], ri[2]};
	c->up = (struct nb_vec3){up[0], up[1], up[2]};
	c->vfov = vfov;
	c->focdist = 10.0f; // gltfimp.c:107
	c->focangle = 0.0f;
}

static int add_instance(struct gl_load *L, unsigned int mesh,
                        const float g[16])
{
	struct nbh_scene *s = L->s;
	if (s->instcnt == L->instcap) {
		L->instcap = L->instcap * 2 + 16;
		struct nbh_inst *p = realloc(s->insts, sizeof(*p) * L->instcap);
		if (!p)
			return -1;
		s->insts = p;
	}
	struct nbh_inst *o = &s->insts[s->instcnt++];
	o->mesh = mesh;
	// a mesh node carries the flags of its mesh's materials (imp_nodes,
	// gltfimp.c:254-256)
	const struct nbh_mesh *m = &s->meshes[mesh];
	unsigned int f = NB_FLAG_MESH;
	for (unsigned int t = 0; t < m->icnt / 3; t++)
		f |= s->mtls[m->tmtl ? m->tmtl[t] : m->mtlid].flags &
		  NB_FLAG_EMISSIVE;
	o->flags = f;
	memcpy(o->glob, g, sizeof(o->glob));
	return 0;
}

static int load_nodes(struct gl_load *L, int node_id, const float pg[16],
                      int depth)
{
	const struct jdoc *d = &L->d;
	int nodes = j_get(d, 0, "nodes");
	int node = j_at(d, nodes, node_id);
	if (node < 0 || depth > 64)
		return -1;
	// glTF nodes form trees (at most one parent each): a node reached twice
	// is a cycle or a shared child, and shared children repeated on every
	// level would take up to 2^64 visits within the depth bound
	if (L->seen[node_id])
		return -1;
	L->seen[node_id] = 1;
	float loc[16], g[16];
	if (node_local(d, node, loc))
		return -1;
	mat4_mul_f(g, pg, loc);
	int ex = j_get(d, j_get(d, node, "extras"), "nodebleed");
	if (!(L->flags & NBH_GLTF_NO_EXTRAS) && ex >= 0) {
		int gk = j_get(d, ex, "glob");
		if (gk >= 0 && j_floats(d, gk, g, 16))
			return -1;
	}
	int mesh = j_index(L, j_get(d, node, "mesh"), -1);
	int cam = j_index(L, j_get(d, node, "camera"), -1);
	if (cam >= 0) {
		if (L->cam_done)
			goto children; // the first camera node only

		int cams = j_get(d, 0, "cameras");
		int ck = j_at(d, cams, cam);
		float yfov = (float)j_num(d, j_get(d, j_get(d, ck, "perspective"),
		  "yfov"), 1.0);
		cam_from(&L->s->cam, g, yfov * 180.0f / 3.14159265358979f);
		int cv = ex >= 0 && !(L->flags & NBH_GLTF_NO_EXTRAS) ?
		  j_get(d, ex, "camera") : -1;
		if (cv >= 0) {
			float v[14];
			if (j_floats(d, cv, v, 14))
				return -1;
			L->s->cam.eye = (struct nb_vec3){v[0], v[1], v[2]};
			L->s->cam.fwd = (struct nb_vec3){v[3], v[4], v[5]};
			L->s->cam.ri = (struct nb_vec3){v[6], v[7], v[8]};
			L->s->cam.up = (struct nb_vec3){v[9], v[10], v[11]};
			L->s->cam.vfov = v[12];
			L->s->cam.focdist = v[13];
		}
		L->cam_done = 1;
	} else if (mesh >= 0) { // a camera node's mesh is ignored
		if ((unsigned int)mesh >= L->s->meshcnt)
			return -1;
		if (add_instance(L, (unsigned int)mesh, g))
			return -1;
	}
children:;
	int ch = j_get(d, node, "children");
	for (int i = 0; i < j_len(d, ch); i++) {
		int c = j_index(L, j_at(d, ch, i), -1);
		if (c < 0 || load_nodes(L, c, g, depth + 1))
			return -1;
	}
	return 0;
}

int nbh_scene_load_gltf(struct nbh_scene *s, const char *path,
                        unsigned int flags)
{
	memset(s, 0, sizeof(*s));
	struct gl_load L;
	memset(&L, 0, sizeof(L));
	L.s = s;
	L.flags = flags;
	size_t len = 0, binlen = 0;
	char *txt = read_file(path, &len);
	uint8_t *bin = NULL;
	int rc = -1;
	if (!txt || j_parse(&L.d, txt, len))
		goto out;
	const struct jdoc *d = &L.d;
	// the one external buffer (the reference assumes the .gltf's name
	// with .bin, gltfimp.c:420-428; the uri names it here)
	int buf0 = j_at(d, j_get(d, 0, "buffers"), 0);
	int uri = j_get(d, buf0, "uri");
	char *bpath = NULL;
	if (uri >= 0 && d->t[uri].type == J_STR)
		bpath = sibling(path, d->s + d->t[uri].start,
		  (size_t)(d->t[uri].end - d->t[uri].start));
	if (!bpath || !(bin = (uint8_t *)read_file(bpath, &binlen))) {
		free(bpath);
		goto out;
	}
	free(bpath);
	L.bin = bin;
	L.binlen = binlen;
	int va = j_get(d, 0, "bufferViews");
	L.nviews = j_len(d, va);
	L.views = calloc((size_t)L.nviews + 1, sizeof(*L.views));
	for (int i = 0; L.views && i < L.nviews; i++) {
		int v = j_at(d, va, i);
		L.views[i].off = j_u32(&L, j_get(d, v, "byteOffset"), 0);
		L.views[i].len = j_u32(&L, j_get(d, v, "byteLength"), 0);
		L.views[i].stride = j_u32(&L, j_get(d, v, "byteStride"),
		  0);
	}
	int aa = j_get(d, 0, "accessors");
	L.naccs = j_len(d, aa);
	L.accs = calloc((size_t)L.naccs + 1, sizeof(*L.accs));
	if (!L.views || !L.accs)
		goto out;
	for (int i = 0; i < L.naccs; i++) {
		int a = j_at(d, aa, i);
		struct gl_acc *A = &L.accs[i];
		A->view = j_index(&L, j_get(d, a, "bufferView"), -1);
		A->off = j_u32(&L, j_get(d, a, "byteOffset"), 0);
		A->cnt = j_u32(&L, j_get(d, a, "count"), 0);
		A->comp = j_u32(&L, j_get(d, a, "componentType"), 0);
		int ty = j_get(d, a, "type");
		A->ncomp = j_eq(d, ty, "SCALAR") ? 1 : j_eq(d, ty, "VEC2") ? 2 :
		  j_eq(d, ty, "VEC3") ? 3 : j_eq(d, ty, "VEC4") ? 4 : 0;
	}
	if (L.err)
		goto out;
	if (load_materials(&L))
		goto out;
	int ma = j_get(d, 0, "meshes");
	int nm = j_len(d, ma);
	if (nm == 0)
		goto out;
	s->meshes = calloc((size_t)nm, sizeof(*s->meshes));
	if (!s->meshes)
		goto out;
	for (int i = 0; i < nm; i++) {
		s->meshcnt = (unsigned int)i + 1u;
		if (load_mesh(&L, j_at(d, ma, i), &s->meshes[i]))
			goto out;
	}
	// roots of the default scene (scene, else 0)
	int sc = j_at(d, j_get(d, 0, "scenes"),
	  j_index(&L, j_get(d, 0, "scene"), 0));
	int roots = j_get(d, sc, "nodes");
	L.seen = calloc((size_t)j_len(d, j_get(d, 0, "nodes")) + 1, 1);
	if (!L.seen)
		goto out;
	static const float ident[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0,
	  0, 0, 0, 1};
	for (int i = 0; i < j_len(d, roots); i++)
		if (load_nodes(&L, j_index(&L, j_at(d, roots, i), -1), ident,
		  0))
			goto out;
	if (s->instcnt == 0)
		goto out;
	if (!L.cam_done) {
		// proxy camera on the scene's root node, whose transform is the
		// identity (gltfimp.c:377-380; the vfov passes radians as degrees)
		static const float root[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0,
		  0, 0, 0, 1};
		cam_from(&s->cam, root, 60.0f * 180.0f / 3.14159265358979f);
	}
	// glTF has no background: nodebleed's frame loop sets 0.4 grey after
	// the import (main.c:230); the writer keeps the scene's in extras
	s->bgcol = (struct nb_vec3){0.4f, 0.4f, 0.4f};
	int bgk = j_get(d, j_get(d, j_get(d, sc, "extras"), "nodebleed"),
	  "bgcol");
	if (!(flags & NBH_GLTF_NO_EXTRAS) && bgk >= 0) {
		float bg[3];
		if (j_floats(d, bgk, bg, 3))
			goto out;
		s->bgcol = (struct nb_vec3){bg[0], bg[1], bg[2]};
	}
	s->width = 640;
	s->height = 360;
	s->spp = 1;
	s->depth = 5;
	if (L.err)
		goto out;
	rc = 0;
out:
	if (rc)
		nbh_scene_free(s);
	free(L.views);
	free(L.accs);
	free(L.seen);
	free(L.d.t);
	free(txt);
	free(bin);
	return rc;
}

// -------------------------------------------------------------- writing --

static void put_floats(FILE *f, const float *v, int n)
{
	fputc('[', f);
	for (int i = 0; i < n; i++)
		fprintf(f, "%s%.9g", i ? "," : "", (double)v[i]);
	fputc(']', f);
}

// T, R (quaternion xyzw), S of a row-major matrix without shear.
static void decompose(const float g[16], float t[3], float q[4], float s[3])
{
	double c[3][3];
	for (int j = 0; j < 3; j++) {
		double l = sqrt((double)g[j] * g[j] + (double)g[4 + j] * g[4 + j] +
		  (double)g[8 + j] * g[8 + j]);
		s[j] = (float)l;
		for (int i = 0; i < 3; i++)
			c[i][j] = l > 0.0 ? g[4 * i + j] / l : (i == j);
	}
	for (int i = 0; i < 3; i++)
		t[i] = g[4 * i + 3];
	double tr = c[0][0] + c[1][1] + c[2][2], x, y, z, w;
	if (tr > 0.0) {
		double r = sqrt(1.0 + tr) * 2.0;
		w = 0.25 * r;
		x = (c[2][1] - c[1][2]) / r;
		y = (c[0][2] - c[2][0]) / r;
		z = (c[1][0] - c[0][1]) / r;
	} else if (c[0][0] > c[1][1] && c[0][0] > c[2][2]) {
		double r = sqrt(1.0 + c[0][0] - c[1][1] - c[2][2]) * 2.0;
		w = (c[2][1] - c[1][2]) / r;
		x = 0.25 * r;
		y = (c[0][1] + c[1][0]) / r;
		z = (c[0][2] + c[2][0]) / r;
	} else if (c[1][1] > c[2][2]) {
		double r = sqrt(1.0 + c[1][1] - c[0][0] - c[2][2]) * 2.0;
		w = (c[0][2] - c[2][0]) / r;
		x = (c[0][1] + c[1][0]) / r;
		y = 0.25 * r;
		z = (c[1][2] + c[2][1]) / r;
	} else {
		double r = sqrt(1.0 + c[2][2] - c[0][0] - c[1][1]) * 2.0;
		w = (c[1][0] - c[0][1]) / r;
		x = (c[0][2] + c[2][0]) / r;
		y = (c[1][2] + c[2][1]) / r;
		z = 0.25 * r;
	}
	q[0] = (float)x;
	q[1] = (float)y;
	q[2] = (float)z;
	q[3] = (float)w;
}

int nbh_scene_save_gltf(const struct nbh_scene *s, const char *path)
{
	size_t pl = strlen(path);
	if (pl < 6 || strcmp(path + pl - 5, ".gltf") != 0)
		return -1;
	char *bpath = malloc(pl);
	if (!bpath)
		return -1;
	memcpy(bpath, path, pl - 4);
	memcpy(bpath + pl - 4, "bin", 4); // x.gltf -> x.bin
	const char *bname = strrchr(bpath, '/');
	bname = bname ? bname + 1 : bpath;
	FILE *fb = fopen(bpath, "wb");
	FILE *f = fopen(path, "w");
	int rc = -1;
	if (!fb || !f)
		goto out;
	// binary: per mesh positions, normals, u32 indices
	uint64_t off = 0;
	uint64_t *moff = calloc(s->meshcnt + 1, sizeof(*moff));
	if (!moff)
		goto out;
	for (unsigned int k = 0; k < s->meshcnt; k++) {
		const struct nbh_mesh *m = &s->meshes[k];
		moff[k] = off;
		if (fwrite(m->vrts, 12, m->vcnt, fb) != m->vcnt ||
		  fwrite(m->nrms, 12, m->vcnt, fb) != m->vcnt ||
		  fwrite(m->inds, 4, m->icnt, fb) != m->icnt) {
			free(moff);
			goto out;
		}
		off += (uint64_t)m->vcnt * 24 + (uint64_t)m->icnt * 4;
	}
	if (off > 0xffffffffu) {
		free(moff);
		goto out;
	}
	fprintf(f, "{\"asset\":{\"version\":\"2.0\",\"generator\":"
	  "\"nodebleed_b200\"},\"extensionsUsed\":["
	  "\"KHR_materials_emissive_strength\",\"KHR_materials_ior\"],\n");
	fprintf(f, "\"buffers\":[{\"uri\":\"%s\",\"byteLength\":%llu}],\n",
	  bname, (unsigned long long)off);
	fprintf(f, "\"bufferViews\":[");
	for (unsigned int k = 0; k < s->meshcnt; k++) {
		const struct nbh_mesh *m = &s->meshes[k];
		unsigned long long o = moff[k];
		fprintf(f, "%s{\"buffer\":0,\"byteOffset\":%llu,\"byteLength\":%u},"
		  "{\"buffer\":0,\"byteOffset\":%llu,\"byteLength\":%u},"
		  "{\"buffer\":0,\"byteOffset\":%llu,\"byteLength\":%u}",
		  k ? ",\n" : "", o, m->vcnt * 12, o + m->vcnt * 12ull,
		  m->vcnt * 12, o + m->vcnt * 24ull, m->icnt * 4);
	}
	fprintf(f, "],\n\"accessors\":[");
	for (unsigned int k = 0; k < s->meshcnt; k++) {
		const struct nbh_mesh *m = &s->meshes[k];
		float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f};
		float hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
		for (unsigned int i = 0; i < m->vcnt; i++)
			for (int a = 0; a < 3; a++) {
				float v = m->vrts[3 * (size_t)i + a];
				lo[a] = v < lo[a] ? v : lo[a];
				hi[a] = v > hi[a] ? v : hi[a];
			}
		fprintf(f, "%s{\"bufferView\":%u,\"componentType\":5126,\"count\":%u,"
		  "\"type\":\"VEC3\",\"min\":", k ? ",\n" : "", 3 * k, m->vcnt);
		put_floats(f, lo, 3);
		fprintf(f, ",\"max\":");
		put_floats(f, hi, 3);
		fprintf(f, "},{\"bufferView\":%u,\"componentType\":5126,"
		  "\"count\":%u,\"type\":\"VEC3\"},{\"bufferView\":%u,"
		  "\"componentType\":5125,\"count\":%u,\"type\":\"SCALAR\"}",
		  3 * k + 1, m->vcnt, 3 * k + 2, m->icnt);
	}
	free(moff);
	fprintf(f, "],\n\"materials\":[");
	for (unsigned int i = 0; i < s->mtlcnt; i++) {
		const struct nb_rmtl *m = &s->mtls[i];
		float base[4] = {m->col.x, m->col.y, m->col.z, 1.0f};
		fprintf(f, "%s{\"pbrMetallicRoughness\":{\"baseColorFactor\":",
		  i ? ",\n" : "");
		int em = (m->flags & NB_FLAG_EMISSIVE) != 0;
		if (em)
			base[0] = base[1] = base[2] = 1.0f;
		put_floats(f, base, 4);
		fprintf(f, ",\"metallicFactor\":%.9g,\"roughnessFactor\":%.9g}",
		  (double)m->metallic, (double)m->roughness);
		if (em) {
			// emission = factor (in [0, 1]) x strength
			float mx = m->col.x > m->col.y ? m->col.x : m->col.y;
			mx = mx > m->col.z ? mx : m->col.z;
			float fac[3] = {m->col.x / mx, m->col.y / mx, m->col.z / mx};
			fprintf(f, ",\"emissiveFactor\":");
			put_floats(f, fac, 3);
			fprintf(f, ",\"extensions\":{\"KHR_materials_emissive_strength\":"
			  "{\"emissiveStrength\":%.9g},\"KHR_materials_ior\":"
			  "{\"ior\":%.9g}}}", (double)mx, (double)m->ior);
		} else {
			fprintf(f, ",\"extensions\":{\"KHR_materials_ior\":{\"ior\":"
			  "%.9g}}}", (double)m->ior);
		}
	}
	fprintf(f, "],\n\"meshes\":[");
	for (unsigned int k = 0; k < s->meshcnt; k++) {
		const struct nbh_mesh *m = &s->meshes[k];
		fprintf(f, "%s{\"primitives\":[", k ? "," : "");
		// one primitive per run of equal material ids
		unsigned int nt = m->icnt / 3, t0 = 0;
		int first = 1;
		while (t0 < nt) {
			unsigned int mt = m->tmtl ? m->tmtl[t0] : m->mtlid, t1 = t0;
			while (t1 < nt && (m->tmtl ? m->tmtl[t1] : m->mtlid) == mt)
				t1++;
			if (t0 == 0 && t1 == nt) {
				fprintf(f, "{\"attributes\":{\"POSITION\":%u,\"NORMAL\":%u},"
				  "\"indices\":%u,\"material\":%u}", 3 * k, 3 * k + 1,
				  3 * k + 2, mt);
			} else {
				// runs need their own index accessors: not written
				fclose(f);
				f = NULL;
				goto out;
			}
			(void)first;
			first = 0;
			t0 = t1;
		}
		fprintf(f, "]}");
	}
	// nodes: one per instance, then the camera
	fprintf(f, "],\n\"cameras\":[{\"type\":\"perspective\",\"perspective\":"
	  "{\"yfov\":%.9g,\"aspectRatio\":%.9g,\"znear\":0.01}}],\n\"nodes\":[",
	  (double)(s->cam.vfov * 3.14159265358979f / 180.0f),
	  s->height ? (double)s->width / s->height : 1.0);
	for (unsigned int i = 0; i < s->instcnt; i++) {
		const struct nbh_inst *in = &s->insts[i];
		float t[3], q[4], sc[3];
		decompose(in->glob, t, q, sc);
		fprintf(f, "%s{\"mesh\":%u,\"translation\":", i ? ",\n" : "",
		  in->mesh);
		put_floats(f, t, 3);
		fprintf(f, ",\"rotation\":");
		put_floats(f, q, 4);
		fprintf(f, ",\"scale\":");
		put_floats(f, sc, 3);
		fprintf(f, ",\"extras\":{\"nodebleed\":{\"glob\":");
		put_floats(f, in->glob, 16);
		fprintf(f, "}}}");
	}
	{
		// camera node: columns ri, up, -fwd, translation eye
		const struct nbh_cam *c = &s->cam;
		float g[16] = {c->ri.x, c->up.x, -c->fwd.x, c->eye.x,
		  c->ri.y, c->up.y, -c->fwd.y, c->eye.y,
		  c->ri.z, c->up.z, -c->fwd.z, c->eye.z, 0, 0, 0, 1};
		float t[3], q[4], sc[3];
		decompose(g, t, q, sc);
		float v[14] = {c->eye.x, c->eye.y, c->eye.z, c->fwd.x, c->fwd.y,
		  c->fwd.z, c->ri.x, c->ri.y, c->ri.z, c->up.x, c->up.y, c->up.z,
		  c->vfov, c->focdist};
		fprintf(f, "%s{\"camera\":0,\"translation\":",
		  s->instcnt ? ",\n" : "");
		put_floats(f, t, 3);
		fprintf(f, ",\"rotation\":");
		put_floats(f, q, 4);
		fprintf(f, ",\"extras\":{\"nodebleed\":{\"camera\":");
		put_floats(f, v, 14);
		fprintf(f, "}}}");
	}
	fprintf(f, "],\n\"scenes\":[{\"extras\":{\"nodebleed\":{\"bgcol\":");
	float bg[3] = {s->bgcol.x, s->bgcol.y, s->bgcol.z};
	put_floats(f, bg, 3);
	fprintf(f, "}},\"nodes\":[");
	for (unsigned int i = 0; i <= s->instcnt; i++)
		fprintf(f, "%s%u", i ? "," : "", i);
	// a trailing newline: nodebleed's reader calls strlen on the mapped
	// file (gltf.c:1017), so the text must end before the page does
	fprintf(f, "]}],\"scene\":0}\n");
	rc = 0;
out:
	if (f && fclose(f) != 0)
		rc = -1;
	if (fb && fclose(fb) != 0)
		rc = -1;
	free(bpath);
	return rc;
}
