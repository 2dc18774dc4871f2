// Seeded synthetic scenes and the scene -> render-data bridge.
//
// The scenes stand in for glTF files: meshes with per-vertex normals and one
// material each, mesh nodes with object->world transforms, a pinhole camera.
// The bridge restates main.c:53-195 (cpy_rdata, upd_rinsts, upd_rcam) so the
// resulting `struct rdata` is what nodebleed's own frame loop would hand to a
// renderer.  All randomness is PCG32 (O'Neill 2014) from the given seed.

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "nb_host.h"

#define NB_PI 3.14159265 // util.h:9 (a double literal there too)

// ------------------------------------------------------------------ PCG32 --

struct pcg { uint64_t state, inc; };

static uint32_t pcg_next(struct pcg *r)
{
	uint64_t old = r->state;
	r->state = old * 6364136223846793005ull + r->inc;
	uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	uint32_t rot = (uint32_t)(old >> 59u);
	return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

static void pcg_seed(struct pcg *r, uint64_t initstate, uint64_t initseq)
{
	r->state = 0;
	r->inc = (initseq << 1u) | 1u;
	pcg_next(r);
	r->state += initstate;
	pcg_next(r);
}

static double rnd(struct pcg *r) // [0,1) with 32 random bits
{
	return pcg_next(r) * (1.0 / 4294967296.0);
}

static double rnd_range(struct pcg *r, double a, double b)
{
	return a + (b - a) * rnd(r);
}

static double rnd_normal(struct pcg *r) // Box-Muller
{
	double u1 = 1.0 - rnd(r), u2 = rnd(r);
	return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

static double rnd_loguniform(struct pcg *r, double a, double b)
{
	return exp(log(a) + (log(b) - log(a)) * rnd(r));
}

// ------------------------------------------------------------- mesh build --

struct mbuf {
	unsigned int vcnt, vcap, icnt, icap;
	float *v, *n;
	unsigned int *i;
};

static int mb_reserve(struct mbuf *m, unsigned int nv, unsigned int ni)
{
	if (m->vcnt + nv > m->vcap) {
		unsigned int c = (m->vcnt + nv) * 2 + 16;
		float *v = realloc(m->v, sizeof(float) * 3 * c);
		float *n = realloc(m->n, sizeof(float) * 3 * c);
		if (!v || !n)
			return -1;
		m->v = v;
		m->n = n;
		m->vcap = c;
	}
	if (m->icnt + ni > m->icap) {
		unsigned int c = (m->icnt + ni) * 2 + 16;
		unsigned int *i = realloc(m->i, sizeof(unsigned int) * c);
		if (!i)
			return -1;
		m->i = i;
		m->icap = c;
	}
	return 0;
}

static unsigned int mb_vert(struct mbuf *m, const double p[3],
                            const double n[3])
{
	unsigned int k = m->vcnt++;
	for (int a = 0; a < 3; a++) {
		m->v[3 * k + a] = (float)p[a];
		m->n[3 * k + a] = (float)n[a];
	}
	return k;
}

static void mb_tri(struct mbuf *m, unsigned int a, unsigned int b,
                   unsigned int c)
{
	m->i[m->icnt++] = a;
	m->i[m->icnt++] = b;
	m->i[m->icnt++] = c;
}

static void normalize3(double v[3])
{
	double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
	if (l > 0) {
		v[0] /= l;
		v[1] /= l;
		v[2] /= l;
	}
}

static void cross3(double r[3], const double a[3], const double b[3])
{
	r[0] = a[1] * b[2] - a[2] * b[1];
	r[1] = a[2] * b[0] - a[0] * b[2];
	r[2] = a[0] * b[1] - a[1] * b[0];
}

// Icosahedron subdivided at frequency f (20 f^2 triangles, 10 f^2 + 2
// vertices), projected on the unit sphere.  Vertices on icosahedron edges
// are shared between faces (computed once per edge), so the mesh is closed.
// Subdivision level k of the usual icosphere is f = 2^k.
struct sphere_vtx { unsigned int *edge; unsigned int corner[12]; };

static const int ico_face[20][3] = {
  {0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
  {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
  {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
  {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};

static void ico_corner(double p[3], int k)
{
	const double t = (1.0 + sqrt(5.0)) / 2.0;
	const double c[12][3] = {
	  {-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
	  {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
	  {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
	p[0] = c[k][0];
	p[1] = c[k][1];
	p[2] = c[k][2];
	normalize3(p);
}

// Position on the sphere for barycentric grid point (i, j) of a face.
static void face_point(double p[3], const double A[3], const double B[3],
                       const double C[3], int i, int j, int f)
{
	double wa = (double)(f - i - j) / f, wb = (double)i / f,
	  wc = (double)j / f;
	for (int a = 0; a < 3; a++)
		p[a] = A[a] * wa + B[a] * wb + C[a] * wc;
	normalize3(p);
}

static int edge_id(int a, int b, int *ea, int *eb, int *ne)
{
	int lo = a < b ? a : b, hi = a < b ? b : a;
	for (int e = 0; e < *ne; e++)
		if (ea[e] == lo && eb[e] == hi)
			return e;
	ea[*ne] = lo;
	eb[*ne] = hi;
	return (*ne)++;
}

// Vertex index of grid point (i,j) of face fc; creates it on first use.
static unsigned int sphere_index(struct mbuf *m, struct sphere_vtx *sv,
                                 const double P[12][3], int fc, int i, int j,
                                 int f, int *ea, int *eb, int *ne)
{
	const int *F = ico_face[fc];
	int w[3] = {f - i - j, i, j};
	for (int c = 0; c < 3; c++)
		if (w[c] == f)
			return sv->corner[F[c]];
	for (int c = 0; c < 3; c++) {
		if (w[c] != 0)
			continue;
		int a = F[(c + 1) % 3], b = F[(c + 2) % 3];
		int wa = w[(c + 1) % 3]; // weight of corner a
		int e = edge_id(a, b, ea, eb, ne);
		int lo = ea[e];
		// position k along edge from lo to hi (1..f-1)
		int k = (a == lo) ? f - wa : wa;
		unsigned int *slot = &sv->edge[e * (f - 1) + (k - 1)];
		if (*slot == 0xffffffffu) {
			double q[3];
			double t = (double)k / f;
			const double *L = P[lo], *H = P[eb[e]];
			for (int x = 0; x < 3; x++)
				q[x] = L[x] * (1.0 - t) + H[x] * t;
			normalize3(q);
			*slot = mb_vert(m, q, q);
		}
		return *slot;
	}
	// interior: unique to this face
	double q[3];
	face_point(q, P[F[0]], P[F[1]], P[F[2]], i, j, f);
	return mb_vert(m, q, q);
}

static int gen_sphere(struct mbuf *m, int f)
{
	double P[12][3];
	for (int k = 0; k < 12; k++)
		ico_corner(P[k], k);
	unsigned int nv = 10u * f * f + 2, ni = 60u * f * f;
	if (mb_reserve(m, nv, ni))
		return -1;
	struct sphere_vtx sv;
	sv.edge = malloc(sizeof(unsigned int) * 30 * (f > 1 ? f - 1 : 1));
	memset(sv.edge, 0xff, sizeof(unsigned int) * 30 * (f > 1 ? f - 1 : 1));
	for (int k = 0; k < 12; k++)
		sv.corner[k] = mb_vert(m, P[k], P[k]);
	int ea[30], eb[30], ne = 0;
	unsigned int *idx = malloc(sizeof(unsigned int) * (f + 1) * (f + 1));
	for (int fc = 0; fc < 20; fc++) {
		for (int i = 0; i <= f; i++)
			for (int j = 0; i + j <= f; j++)
				idx[i * (f + 1) + j] = sphere_index(m, &sv, P,
				  fc, i, j, f, ea, eb, &ne);
		for (int i = 0; i < f; i++)
			for (int j = 0; i + j < f; j++) {
				unsigned int a = idx[i * (f + 1) + j];
				unsigned int b = idx[(i + 1) * (f + 1) + j];
				unsigned int c = idx[i * (f + 1) + j + 1];
				mb_tri(m, a, b, c);
				if (i + j + 1 < f) {
					unsigned int d =
					  idx[(i + 1) * (f + 1) + j + 1];
					mb_tri(m, b, d, c);
				}
			}
	}
	free(idx);
	free(sv.edge);
	return 0;
}

// Area-weighted vertex normals from the faces.
static void smooth_normals(struct mbuf *m)
{
	double *acc = calloc((size_t)m->vcnt * 3, sizeof(double));
	for (unsigned int t = 0; t < m->icnt; t += 3) {
		unsigned int a = m->i[t], b = m->i[t + 1], c = m->i[t + 2];
		double e0[3], e1[3], n[3];
		for (int x = 0; x < 3; x++) {
			e0[x] = (double)m->v[3 * b + x] - m->v[3 * a + x];
			e1[x] = (double)m->v[3 * c + x] - m->v[3 * a + x];
		}
		cross3(n, e0, e1);
		for (int x = 0; x < 3; x++) {
			acc[3 * a + x] += n[x];
			acc[3 * b + x] += n[x];
			acc[3 * c + x] += n[x];
		}
	}
	for (unsigned int v = 0; v < m->vcnt; v++) {
		normalize3(&acc[3 * v]);
		for (int x = 0; x < 3; x++)
			m->n[3 * v + x] = (float)acc[3 * v + x];
	}
	free(acc);
}

// Icosphere (unit radius) with N(0, sigma) jitter on every coordinate;
// normals stay the unjittered radial directions.
static int gen_jitter_sphere(struct mbuf *m, int f, double sigma,
                             struct pcg *r)
{
	if (gen_sphere(m, f))
		return -1;
	for (unsigned int v = 0; v < m->vcnt; v++)
		for (int x = 0; x < 3; x++)
			m->v[3 * v + x] = (float)(m->v[3 * v + x] +
			  sigma * rnd_normal(r));
	return 0;
}

// Sphere of radius 0.4 centred in the unit box, radially displaced by a sum
// of four random plane waves (amplitude up to 15 %), smooth normals.
static int gen_displaced_sphere(struct mbuf *m, int f, struct pcg *r)
{
	if (gen_sphere(m, f))
		return -1;
	double k[4][3], ph[4], amp[4];
	for (int w = 0; w < 4; w++) {
		double d[3] = {rnd_normal(r), rnd_normal(r), rnd_normal(r)};
		normalize3(d);
		double fr = rnd_range(r, 2.0, 9.0);
		for (int x = 0; x < 3; x++)
			k[w][x] = d[x] * fr;
		ph[w] = rnd_range(r, 0.0, 2.0 * M_PI);
		amp[w] = rnd_range(r, 0.01, 0.0375);
	}
	for (unsigned int v = 0; v < m->vcnt; v++) {
		double p[3] = {m->v[3 * v], m->v[3 * v + 1], m->v[3 * v + 2]};
		double s = 1.0;
		for (int w = 0; w < 4; w++)
			s += amp[w] * sin(k[w][0] * p[0] + k[w][1] * p[1] +
			  k[w][2] * p[2] + ph[w]);
		for (int x = 0; x < 3; x++)
			m->v[3 * v + x] = (float)(0.5 + 0.4 * s * p[x]);
	}
	smooth_normals(m);
	return 0;
}

// `cnt` equilateral triangles with centres uniform in the unit box, random
// orientation and edge length U[emin, emax]; flat normals.
static int gen_soup(struct mbuf *m, unsigned int cnt, double emin, double emax,
                    struct pcg *r)
{
	if (mb_reserve(m, 3 * cnt, 3 * cnt))
		return -1;
	for (unsigned int t = 0; t < cnt; t++) {
		double c[3] = {rnd(r), rnd(r), rnd(r)};
		double n[3] = {rnd_normal(r), rnd_normal(r), rnd_normal(r)};
		normalize3(n);
		double h[3] = {fabs(n[0]) < 0.9 ? 1.0 : 0.0,
		  fabs(n[0]) < 0.9 ? 0.0 : 1.0, 0.0}, u[3], w[3];
		cross3(u, n, h);
		normalize3(u);
		cross3(w, n, u);
		double e = rnd_range(r, emin, emax), rad = e / sqrt(3.0);
		double th = rnd_range(r, 0.0, 2.0 * M_PI);
		unsigned int id[3];
		for (int k = 0; k < 3; k++) {
			double a = th + 2.0 * M_PI * k / 3.0, p[3];
			for (int x = 0; x < 3; x++)
				p[x] = c[x] + rad * (cos(a) * u[x] + sin(a) * w[x]);
			id[k] = mb_vert(m, p, n);
		}
		mb_tri(m, id[0], id[1], id[2]);
	}
	return 0;
}

// Axis-aligned quad in the xz plane at height y, centred at (cx, cz), side
// lengths sx, sz; normal +y (up = 1) or -y (up = 0), wound to match.
static int gen_quad(struct mbuf *m, double cx, double y, double cz, double sx,
                    double sz, int up)
{
	if (mb_reserve(m, 4, 6))
		return -1;
	double n[3] = {0.0, up ? 1.0 : -1.0, 0.0};
	double p[4][3] = {{cx - sx / 2, y, cz - sz / 2},
	  {cx + sx / 2, y, cz - sz / 2}, {cx + sx / 2, y, cz + sz / 2},
	  {cx - sx / 2, y, cz + sz / 2}};
	unsigned int b = m->vcnt;
	for (int k = 0; k < 4; k++)
		mb_vert(m, p[k], n);
	if (up) { // (p3-p0) x (p1-p0) points +y
		mb_tri(m, b, b + 3, b + 2);
		mb_tri(m, b, b + 2, b + 1);
	} else {
		mb_tri(m, b, b + 1, b + 2);
		mb_tri(m, b, b + 2, b + 3);
	}
	return 0;
}

// --------------------------------------------------------------- assembly --

struct sbuild {
	struct nbh_scene *s;
	unsigned int meshcap, mtlcap, instcap;
};

static int add_mesh(struct sbuild *b, struct mbuf *m, unsigned int mtl)
{
	struct nbh_scene *s = b->s;
	if (s->meshcnt == b->meshcap) {
		b->meshcap = b->meshcap * 2 + 8;
		struct nbh_mesh *p = realloc(s->meshes,
		  sizeof(*p) * b->meshcap);
		if (!p)
			return -1;
		s->meshes = p;
	}
	struct nbh_mesh *o = &s->meshes[s->meshcnt];
	o->vcnt = m->vcnt;
	o->vrts = m->v;
	o->nrms = m->n;
	o->icnt = m->icnt;
	o->inds = m->i;
	o->mtlid = mtl;
	o->tmtl = NULL;
	memset(m, 0, sizeof(*m));
	return (int)s->meshcnt++;
}

static int add_mtl(struct sbuild *b, double r, double g, double bl,
                   double metallic, double rough, unsigned int flags)
{
	struct nbh_scene *s = b->s;
	if (s->mtlcnt == b->mtlcap) {
		b->mtlcap = b->mtlcap * 2 + 8;
		struct nb_rmtl *p = realloc(s->mtls, sizeof(*p) * b->mtlcap);
		if (!p)
			return -1;
		s->mtls = p;
	}
	s->mtls[s->mtlcnt] = (struct nb_rmtl){
	  .col = {(float)r, (float)g, (float)bl}, .metallic = (float)metallic,
	  .roughness = (float)rough, .ior = 1.5f, .flags = flags};
	return (int)s->mtlcnt++;
}

// Object->world = T * R * S (scene.c:176-185), R from a unit quaternion.
static void trs(float dst[16], const double t[3], const double q[4],
                const double sc[3])
{
	double x = q[0], y = q[1], z = q[2], w = q[3];
	double R[9] = {
	  1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
	  2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
	  2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)};
	for (int i = 0; i < 3; i++) {
		for (int j = 0; j < 3; j++)
			dst[4 * i + j] = (float)(R[3 * i + j] * sc[j]);
		dst[4 * i + 3] = (float)t[i];
	}
	dst[12] = dst[13] = dst[14] = 0.0f;
	dst[15] = 1.0f;
}

static void rnd_quat(double q[4], struct pcg *r) // Shoemake, uniform
{
	double u1 = rnd(r), u2 = rnd(r), u3 = rnd(r);
	double a = sqrt(1 - u1), b = sqrt(u1);
	q[0] = a * sin(2 * M_PI * u2);
	q[1] = a * cos(2 * M_PI * u2);
	q[2] = b * sin(2 * M_PI * u3);
	q[3] = b * cos(2 * M_PI * u3);
}

static int add_inst(struct sbuild *b, unsigned int mesh, const float glob[16])
{
	struct nbh_scene *s = b->s;
	if (s->instcnt == b->instcap) {
		b->instcap = b->instcap * 2 + 16;
		struct nbh_inst *p = realloc(s->insts, sizeof(*p) * b->instcap);
		if (!p)
			return -1;
		s->insts = p;
	}
	struct nbh_inst *o = &s->insts[s->instcnt];
	o->mesh = mesh;
	o->flags = NB_FLAG_MESH |
	  (s->mtls[s->meshes[mesh].mtlid].flags & NB_FLAG_EMISSIVE);
	memcpy(o->glob, glob, sizeof(o->glob));
	return (int)s->instcnt++;
}

static void place(struct sbuild *b, unsigned int mesh, const double t[3],
                  const double q[4], const double sc[3])
{
	float g[16];
	trs(g, t, q, sc);
	add_inst(b, mesh, g);
}

static void look_at(struct nbh_cam *c, double ex, double ey, double ez,
                    double tx, double ty, double tz, float vfov)
{
	double f[3] = {tx - ex, ty - ey, tz - ez};
	normalize3(f);
	c->eye = (struct nb_vec3){(float)ex, (float)ey, (float)ez};
	c->fwd = (struct nb_vec3){(float)f[0], (float)f[1], (float)f[2]};
	c->vfov = vfov;
	c->focdist = 10.0f; // gltfimp.c:107
	c->focangle = 0.0f;
	// cam_calcbase (main.c:197): ri = unit(fwd x up), up = unit(ri x fwd)
	double upw[3] = {0, 1, 0}, ri[3], up[3];
	cross3(ri, f, upw);
	normalize3(ri);
	cross3(up, ri, f);
	normalize3(up);
	c->ri = (struct nb_vec3){(float)ri[0], (float)ri[1], (float)ri[2]};
	c->up = (struct nb_vec3){(float)up[0], (float)up[1], (float)up[2]};
}

static int sphere_freq_for(double tris)
{
	int f = (int)floor(sqrt(tris / 20.0) + 0.5);
	return f < 1 ? 1 : f;
}

// Small family: icosphere BLAS (f = 2^5 -> 20480 tris) x4 instances, ground
// quad, one quad light of emission 10.
static int scene_small(struct sbuild *b, struct pcg *r, int freq,
                       unsigned int w, unsigned int h, unsigned int spp,
                       unsigned int depth)
{
	struct nbh_scene *s = b->s;
	struct mbuf m = {0};
	int sph_mtl = add_mtl(b, rnd_range(r, 0.2, 0.8), rnd_range(r, 0.2, 0.8),
	  rnd_range(r, 0.2, 0.8), 0.0, 1.0, 0);
	int gnd_mtl = add_mtl(b, rnd_range(r, 0.2, 0.8), rnd_range(r, 0.2, 0.8),
	  rnd_range(r, 0.2, 0.8), 0.0, 1.0, 0);
	int lgt_mtl = add_mtl(b, 10.0, 10.0, 10.0, 0.0, 1.0, NB_FLAG_EMISSIVE);
	if (gen_jitter_sphere(&m, freq, 0.01, r))
		return -1;
	int sph = add_mesh(b, &m, (unsigned int)sph_mtl);
	if (gen_quad(&m, 0.0, -7.5, 0.0, 40.0, 40.0, 1))
		return -1;
	int gnd = add_mesh(b, &m, (unsigned int)gnd_mtl);
	if (gen_quad(&m, 0.0, 10.0, 0.0, 6.0, 6.0, 0))
		return -1;
	int lgt = add_mesh(b, &m, (unsigned int)lgt_mtl);
	for (int i = 0; i < 4; i++) {
		double q[4], t[3], sc;
		rnd_quat(q, r);
		sc = rnd_range(r, 0.5, 2.0);
		for (int a = 0; a < 3; a++)
			t[a] = rnd_range(r, -5.0, 5.0);
		double s3[3] = {sc, sc, sc};
		place(b, (unsigned int)sph, t, q, s3);
	}
	double id[4] = {0, 0, 0, 1}, z[3] = {0, 0, 0}, one[3] = {1, 1, 1};
	place(b, (unsigned int)gnd, z, id, one);
	place(b, (unsigned int)lgt, z, id, one);
	look_at(&s->cam, 0.0, 4.0, 21.0, 0.0, -1.0, 0.0, 50.0f);
	s->bgcol = (struct nb_vec3){0.1f, 0.1f, 0.1f};
	s->width = w;
	s->height = h;
	s->spp = spp;
	s->depth = depth;
	return 0;
}

// Scale/stress family: `nblas` BLAS of log-uniform size (displaced sphere or
// triangle soup in the unit box), `ninst` instances with random rotation,
// per-axis scale U[0.5,2] and position over a 50 x 8 x 50 region, a ground
// quad and `nlights` quad lights.  Material mix per BLAS: mirror fraction
// `pmirror`, GGX fraction `pggx`, rest Lambertian.
static int scene_field(struct sbuild *b, struct pcg *r, unsigned int nblas,
                       double tmin, double tmax, unsigned int ninst,
                       unsigned int nlights, double pmirror, double pggx,
                       unsigned int w, unsigned int h, unsigned int spp,
                       unsigned int depth, double extent)
{
	struct nbh_scene *s = b->s;
	struct mbuf m = {0};
	for (unsigned int k = 0; k < nblas; k++) {
		double n = rnd_loguniform(r, tmin, tmax);
		int soup = rnd(r) < 0.5;
		double u = rnd(r);
		int mtl;
		double c0 = rnd_range(r, 0.2, 0.8), c1 = rnd_range(r, 0.2, 0.8),
		  c2 = rnd_range(r, 0.2, 0.8), rough = rnd_range(r, 0.05, 0.5);
		if (u < pmirror)
			mtl = add_mtl(b, 0.5 + 0.5 * c0, 0.5 + 0.5 * c1,
			  0.5 + 0.5 * c2, 1.0, 0.0, 0);
		else if (u < pmirror + pggx)
			mtl = add_mtl(b, 0.5 + 0.5 * c0, 0.5 + 0.5 * c1,
			  0.5 + 0.5 * c2, 1.0, rough, 0);
		else
			mtl = add_mtl(b, c0, c1, c2, 0.0, 1.0, 0);
		int rc = soup ? gen_soup(&m, (unsigned int)(n + 0.5), 0.005,
		  0.05, r) : gen_displaced_sphere(&m, sphere_freq_for(n), r);
		if (rc)
			return -1;
		add_mesh(b, &m, (unsigned int)mtl);
	}
	int gnd_mtl = add_mtl(b, 0.5, 0.5, 0.5, 0.0, 1.0, 0);
	if (gen_quad(&m, 0.0, -0.5, 0.0, 6 * extent, 6 * extent, 1))
		return -1;
	int gnd = add_mesh(b, &m, (unsigned int)gnd_mtl);
	for (unsigned int i = 0; i < ninst; i++) {
		double q[4], t[3], sc[3];
		unsigned int mesh = (unsigned int)(rnd(r) * nblas);
		rnd_quat(q, r);
		for (int a = 0; a < 3; a++)
			sc[a] = rnd_range(r, 0.5, 2.0);
		t[0] = rnd_range(r, -extent, extent);
		t[1] = rnd_range(r, 0.0, 8.0);
		t[2] = rnd_range(r, -extent, extent);
		place(b, mesh, t, q, sc);
	}
	double id[4] = {0, 0, 0, 1}, z[3] = {0, 0, 0}, one[3] = {1, 1, 1};
	place(b, (unsigned int)gnd, z, id, one);
	for (unsigned int l = 0; l < nlights; l++) {
		double e = nlights == 1 ? 10.0 : rnd_range(r, 6.0, 14.0);
		double cx = nlights == 1 ? 0.0 : rnd_range(r, -extent, extent);
		double cz = nlights == 1 ? 0.0 : rnd_range(r, -extent, extent);
		double sz = nlights == 1 ? 0.4 * extent : rnd_range(r, 3.0, 8.0);
		int lm = add_mtl(b, e, e * 0.95, e * 0.9, 0.0, 1.0,
		  NB_FLAG_EMISSIVE);
		if (gen_quad(&m, cx, 20.0, cz, sz, sz, 0))
			return -1;
		int lg = add_mesh(b, &m, (unsigned int)lm);
		place(b, (unsigned int)lg, z, id, one);
	}
	look_at(&s->cam, 0.0, 0.3 * extent + 4.0, 1.5 * extent,
	  0.0, 2.0, 0.0, 50.0f);
	s->bgcol = (struct nb_vec3){0.25f, 0.3f, 0.35f};
	s->width = w;
	s->height = h;
	s->spp = spp;
	s->depth = depth;
	return 0;
}

int nbh_scene_gen(struct nbh_scene *s, int family, uint64_t seed,
                  unsigned int param)
{
	memset(s, 0, sizeof(*s));
	struct sbuild b = {s, 0, 0, 0};
	struct pcg r;
	pcg_seed(&r, seed, (uint64_t)family * 0x9e3779b97f4a7c15ull + param);
	int rc = -1;
	int field = family == NBH_SCENE_SCALE || family == NBH_SCENE_STRESS ||
	  family == NBH_SCENE_GLOSSY;
	if ((family == NBH_SCENE_SMALL || family == NBH_SCENE_TINY) &&
	  param > NBH_MAX_SPHERE_FREQ)
		return -1;
	if (field && param > NBH_MAX_BLAS)
		return -1;
	switch (family) {
	case NBH_SCENE_SMALL:
		rc = scene_small(&b, &r, param ? (int)param : 32, 640, 360, 1, 5);
		break;
	case NBH_SCENE_TINY:
		rc = scene_small(&b, &r, param ? (int)param : 4, 64, 48, 1, 3);
		break;
	case NBH_SCENE_BATCH: {
		static const unsigned int res[4][2] = {{320, 180}, {640, 360},
		  {1280, 720}, {1920, 1080}};
		static const unsigned int spps[3] = {1, 4, 16};
		static const unsigned int depths[3] = {4, 8, 12};
		double n = rnd_loguniform(&r, 1000.0, 1000000.0);
		unsigned int ri = (unsigned int)(rnd(&r) * 4);
		unsigned int si = (unsigned int)(rnd(&r) * 3);
		unsigned int di = (unsigned int)(rnd(&r) * 3);
		rc = scene_small(&b, &r, sphere_freq_for(n), res[ri][0],
		  res[ri][1], spps[si], depths[di]);
		break;
	}
	case NBH_SCENE_SCALE:
		rc = scene_field(&b, &r, param ? param : 64, 2000.0, 64000.0,
		  1024, 1, 0.2, 0.0, 1920, 1080, 4, 8, 25.0);
		break;
	case NBH_SCENE_STRESS:
		// 4087 random instances + ground + 8 lights = 4096, the
		// reference's instance cap (INST_ID_BITS = 12, rend.c:24)
		rc = scene_field(&b, &r, param ? param : 128, 1000.0, 200000.0,
		  4087, 8, 1.0 / 3.0, 1.0 / 3.0, 3840, 2160, 1, 16, 50.0);
		break;
	case NBH_SCENE_GLOSSY:
		rc = scene_field(&b, &r, param ? param : 6, 200.0, 3000.0, 40, 8,
		  1.0 / 3.0, 1.0 / 3.0, 160, 96, 1, 8, 8.0);
		break;
	default:
		rc = -1;
	}
	if (rc)
		nbh_scene_free(s);
	return rc;
}

void nbh_scene_free(struct nbh_scene *s)
{
	for (unsigned int i = 0; i < s->meshcnt; i++) {
		free(s->meshes[i].vrts);
		free(s->meshes[i].nrms);
		free(s->meshes[i].inds);
		free(s->meshes[i].tmtl);
	}
	free(s->meshes);
	free(s->mtls);
	free(s->insts);
	memset(s, 0, sizeof(*s));
}

unsigned int nbh_scene_tricnt(const struct nbh_scene *s)
{
	unsigned int n = 0;
	for (unsigned int i = 0; i < s->meshcnt; i++)
		n += s->meshes[i].icnt / 3;
	return n;
}

unsigned int nbh_scene_instcnt(const struct nbh_scene *s)
{
	return s->instcnt;
}

double nbh_scene_insttris(const struct nbh_scene *s)
{
	double n = 0;
	for (unsigned int i = 0; i < s->instcnt; i++)
		n += s->meshes[s->insts[i].mesh].icnt / 3;
	return n;
}

// ----------------------------------------------------------------- bridge --

// main.c:53-113: flatten meshes into rtri/rnrm, copy materials, one rinst per
// mesh node.
int nbh_cpy_rdata(struct nb_rdata *rd, const struct nbh_scene *s)
{
	unsigned int *triofs = malloc(sizeof(unsigned int) * (s->meshcnt + 1));
	unsigned int ofs = 0;
	for (unsigned int k = 0; k < s->meshcnt; k++) {
		const struct nbh_mesh *m = &s->meshes[k];
		for (unsigned int t = 0; t < m->icnt / 3; t++) {
			struct nb_rtri *rt = &rd->tris[ofs + t];
			struct nb_rnrm *rn = &rd->nrms[ofs + t];
			const unsigned int *ip = &m->inds[3 * t];
			memset(rt, 0, sizeof(*rt));
			memset(rn, 0, sizeof(*rn));
			memcpy(&rt->v0, &m->vrts[3 * ip[0]], 12);
			memcpy(&rt->v1, &m->vrts[3 * ip[1]], 12);
			memcpy(&rt->v2, &m->vrts[3 * ip[2]], 12);
			memcpy(&rn->n0, &m->nrms[3 * ip[0]], 12);
			memcpy(&rn->n1, &m->nrms[3 * ip[1]], 12);
			memcpy(&rn->n2, &m->nrms[3 * ip[2]], 12);
			rn->mtlid = m->tmtl ? m->tmtl[t] : m->mtlid;
		}
		triofs[k] = ofs;
		ofs += m->icnt / 3;
	}
	memcpy(rd->mtls, s->mtls, sizeof(*rd->mtls) * s->mtlcnt);
	for (unsigned int i = 0; i < s->instcnt; i++) {
		const struct nbh_inst *in = &s->insts[i];
		memset(&rd->insts[i], 0, sizeof(rd->insts[i]));
		rd->insts[i].flags = in->flags;
		rd->insts[i].triofs = triofs[in->mesh];
		rd->insts[i].tricnt = s->meshes[in->mesh].icnt / 3;
	}
	rd->instcnt = s->instcnt;
	rd->bgcol = s->bgcol;
	free(triofs);
	return 0;
}

// Inverse of a row-major 4x4 by cofactors over 2x2 minors; 1 if singular.
int nbh_mat4_inv(float dst[16], const float m[16])
{
	double a[16];
	for (int i = 0; i < 16; i++)
		a[i] = m[i];
	// 2x2 minors of the top two rows (s) and bottom two rows (c)
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
	if (det == 0.0)
		return 1;
	double id = 1.0 / det;
	double r[16] = {
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
	  (-a[8] * s4 + a[9] * s2 - a[11] * s0),
	  (-a[4] * c3 + a[5] * c1 - a[6] * c0),
	  (a[0] * c3 - a[1] * c1 + a[2] * c0),
	  (-a[12] * s3 + a[13] * s1 - a[14] * s0),
	  (a[8] * s3 - a[9] * s1 + a[10] * s0)};
	for (int i = 0; i < 16; i++)
		dst[i] = (float)(r[i] * id);
	return 0;
}

static inline void xf_pos(const float *m, float x, float y, float z,
                          float *o)
{
	o[0] = m[0] * x + m[1] * y + m[2] * z + m[3];
	o[1] = m[4] * x + m[5] * y + m[6] * z + m[7];
	o[2] = m[8] * x + m[9] * y + m[10] * z + m[11];
}

// main.c:117-157: world->object 3x4 from the inverse of the node transform,
// world box from the 8 transformed corners of the BLAS root box.
int nbh_upd_rinsts(struct nb_rdata *rd, const struct nbh_scene *s)
{
	int bad = 0;
	for (unsigned int i = 0; i < s->instcnt; i++) {
		const float *g = s->insts[i].glob;
		struct nb_rinst *ri = &rd->insts[i];
		float inv[16];
		bad |= nbh_mat4_inv(inv, g);
		memcpy(ri->globinv, inv, sizeof(ri->globinv));
		const struct nb_bnode8 *n = &rd->bnodes[(size_t)ri->triofs << 1];
		float mi[3] = {n->minx8[0], n->miny8[0], n->minz8[0]};
		float ma[3] = {n->maxx8[0], n->maxy8[0], n->maxz8[0]};
		for (int k = 1; k < 8; k++) {
			mi[0] = n->minx8[k] < mi[0] ? n->minx8[k] : mi[0];
			mi[1] = n->miny8[k] < mi[1] ? n->miny8[k] : mi[1];
			mi[2] = n->minz8[k] < mi[2] ? n->minz8[k] : mi[2];
			ma[0] = n->maxx8[k] > ma[0] ? n->maxx8[k] : ma[0];
			ma[1] = n->maxy8[k] > ma[1] ? n->maxy8[k] : ma[1];
			ma[2] = n->maxz8[k] > ma[2] ? n->maxz8[k] : ma[2];
		}
		struct nb_aabb bx = {{3.402823466e+38f, 3.402823466e+38f,
		  3.402823466e+38f}, 0.0f, {-3.402823466e+38f,
		  -3.402823466e+38f, -3.402823466e+38f}, 0.0f};
		for (int c = 0; c < 8; c++) {
			float v[3];
			xf_pos(g, c & 1 ? mi[0] : ma[0], c & 2 ? mi[1] : ma[1],
			  c & 4 ? mi[2] : ma[2], v);
			bx.min.x = v[0] < bx.min.x ? v[0] : bx.min.x;
			bx.min.y = v[1] < bx.min.y ? v[1] : bx.min.y;
			bx.min.z = v[2] < bx.min.z ? v[2] : bx.min.z;
			bx.max.x = v[0] > bx.max.x ? v[0] : bx.max.x;
			bx.max.y = v[1] > bx.max.y ? v[1] : bx.max.y;
			bx.max.z = v[2] > bx.max.z ? v[2] : bx.max.z;
		}
		rd->aabbs[i] = bx;
	}
	return bad ? -1 : 0;
}

static void bcast8(float *dst, float v)
{
	for (int i = 0; i < 8; i++)
		dst[i] = v;
}

// main.c:159-195: camera constants for ray generation.
void nbh_upd_rcam(struct nb_rdata *rd, const struct nbh_cam *c, float w,
                  float h)
{
	struct nb_rcam *rc = &rd->cam;
	float aspect = w / h;
	float tanvfov = tanf((float)(0.5f * c->vfov * NB_PI / 180.0f));
	float tanfangle = tanf((float)(0.5f * c->focangle * NB_PI / 180.0f));
	memset(rc, 0, sizeof(*rc));
	rc->eye = c->eye;
	rc->tanvfov = tanvfov;
	rc->ri = c->ri;
	rc->focdist = c->focdist;
	rc->up = c->up;
	rc->tanfangle = tanfangle;
	rc->fwd = c->fwd;
	rc->aspect = aspect;
	bcast8(rc->eyex8, c->eye.x);
	bcast8(rc->eyey8, c->eye.y);
	bcast8(rc->eyez8, c->eye.z);
	bcast8(rc->rix8, c->ri.x);
	bcast8(rc->riy8, c->ri.y);
	bcast8(rc->riz8, c->ri.z);
	bcast8(rc->upx8, c->up.x);
	bcast8(rc->upy8, c->up.y);
	bcast8(rc->upz8, c->up.z);
	bcast8(rc->fwdx8, c->fwd.x);
	bcast8(rc->fwdy8, c->fwd.y);
	bcast8(rc->fwdz8, c->fwd.z);
	bcast8(rc->rw8, 1.0f / w);
	bcast8(rc->rh8, 1.0f / h);
	bcast8(rc->aspect8, aspect);
	bcast8(rc->fdist8, c->focdist);
	bcast8(rc->fovfdist8, 2.0f * tanvfov * c->focdist);
	bcast8(rc->focangle8, tanfangle);
	bcast8(rc->focrad8, tanfangle * c->focdist);
}

int nbh_rdata_from_scene(struct nb_rdata *rd, const struct nbh_scene *s)
{
	unsigned int tris = nbh_scene_tricnt(s);
	if (nbh_rend_init(rd, s->mtlcnt ? s->mtlcnt : 1, tris, s->instcnt,
	  s->spp))
		return -1;
	nbh_cpy_rdata(rd, s);
	nbh_prepstatic(rd);
	if (nbh_upd_rinsts(rd, s))
		return -2;
	nbh_prepdynamic(rd);
	if (nbh_rend_resaccum(rd, s->width, s->height))
		return -1;
	nbh_upd_rcam(rd, &s->cam, (float)s->width, (float)s->height);
	return 0;
}
