// Host side of the GPU path tracer: render-data bridge, BVH8 build and the
// seeded synthetic scenes the benchmarks and tests render.
//
// These are C restatements of the host code nodebleed keeps on the CPU:
//   nbh_rend_init / _release / _resaccum / _clraccum   rend.c:3000-3107
//   nbh_prepstatic / nbh_prepdynamic / nbh_build_bvh8 rend.c:3033/3073/458
//   nbh_cpy_rdata / nbh_upd_rinsts / nbh_upd_rcam      main.c:53/117/159
// and they fill the same `struct rdata` bytes (nb_rdata.h), so an
// application can use either these or its own rend.c before handing the
// render data to the GPU library (rendgpu.h).

#ifndef NB_HOST_H
#define NB_HOST_H

#include <stdint.h>
#include "nb_rdata.h"

#ifdef __cplusplus
extern "C" {
#endif

// ---------------------------------------------------------------- scenes --

// One triangle mesh.  scene.h:34 keeps a list of material runs per mesh;
// here tmtl holds each triangle's material (glTF meshes of several
// primitives), or is NULL and every triangle has mtlid (the synthetic
// scenes).
struct nbh_mesh {
	unsigned int vcnt;
	float        *vrts; // vcnt * 3
	float        *nrms; // vcnt * 3
	unsigned int icnt;
	unsigned int *inds; // icnt, 3 per triangle
	unsigned int mtlid;
	unsigned int *tmtl; // icnt / 3 material ids, or NULL
};

// A mesh node: mesh id + object->world 4x4 row-major (tfmat.glob,
// scene.h:56) + node flags (types.h).
struct nbh_inst {
	unsigned int mesh;
	unsigned int flags;
	float        glob[16];
};

struct nbh_cam { // scene.h:18-27 (vfov and focangle in degrees)
	struct nb_vec3 eye;
	float          vfov;
	struct nb_vec3 fwd;
	float          focdist;
	struct nb_vec3 ri;
	float          focangle;
	struct nb_vec3 up;
	unsigned int   pad;
};

struct nbh_scene {
	unsigned int    meshcnt;
	struct nbh_mesh *meshes;
	unsigned int    mtlcnt;
	struct nb_rmtl  *mtls;
	unsigned int    instcnt;
	struct nbh_inst *insts;
	struct nbh_cam  cam;
	struct nb_vec3  bgcol;
	// Render settings the workload prescribes.
	unsigned int    width, height, spp, depth;
	unsigned int    pad;
};

#define NBH_MAX_SPHERE_FREQ 1024u // 21 M triangles
#define NBH_MAX_BLAS 4096u        // the reference's instance cap

// Workload ids (one per synthetic scene family).
enum {
	NBH_SCENE_SMALL = 1,   // 1 icosphere BLAS x4 + ground + quad light
	NBH_SCENE_SCALE = 2,   // 64 BLAS (displaced spheres / soups), 1024 inst
	NBH_SCENE_BATCH = 3,   // one scene of the 16-scene batch (small family)
	NBH_SCENE_STRESS = 5,  // 128 BLAS, 4096 inst, GGX/mirror, 8 lights
	NBH_SCENE_GLOSSY = 6,  // the stress mix at test size: 6 BLAS, 40 inst
	NBH_SCENE_TINY = 9     // few hundred tris, for fast parity tests
};

// Generate a seeded scene.  `param` tunes the family: for BATCH it is the
// scene index 0..15; for SMALL/TINY it scales the triangle budget (0 =
// default, at most NBH_MAX_SPHERE_FREQ: the sphere's subdivision, 20 f^2
// triangles); for SCALE/STRESS/GLOSSY it is the BLAS count (0 = default, at
// most NBH_MAX_BLAS).  Returns -1 for an unknown family or a param above
// its bound.
int  nbh_scene_gen(struct nbh_scene *s, int family, uint64_t seed,
                   unsigned int param);
void nbh_scene_free(struct nbh_scene *s);

unsigned int nbh_scene_tricnt(const struct nbh_scene *s);   // unique tris
unsigned int nbh_scene_instcnt(const struct nbh_scene *s);  // mesh nodes
double       nbh_scene_insttris(const struct nbh_scene *s); // instanced tris

// glTF 2.0 (nb_gltf.c).  Load the subset nodebleed's importer reads
// (gltf.h:4-11, gltfimp.c): one external .bin buffer, float VEC3 POSITION and
// NORMAL, u8/u16/u32 indices, PBR base colour / metallic / roughness,
// emissive factor x KHR_materials_emissive_strength, node TRS (or matrix)
// hierarchies, the first perspective camera.  The resolution, spp and depth
// fields get 640x360, 1, 5.  NBH_GLTF_NO_EXTRAS ignores the exact
// transforms this library's writer stores in node extras (so the scene is
// read as nodebleed would read it).  Returns 0, or -1 on any error (the
// scene is then empty).  The writer emits one glTF mesh per host mesh, each
// of a single material run, one node per instance (TRS plus the exact matrix in
// extras) and a camera node; the .bin goes beside the .gltf with the same
// basename, as nodebleed's importer expects (gltfimp.c:420-428).
#define NBH_GLTF_NO_EXTRAS 1u
int nbh_scene_load_gltf(struct nbh_scene *s, const char *path,
                        unsigned int flags);
int nbh_scene_save_gltf(const struct nbh_scene *s, const char *path);

// ------------------------------------------------------------ render data --

struct nb_rdata *nbh_rdata_new(void);   // zeroed, 32-byte aligned
void             nbh_rdata_delete(struct nb_rdata *rd);

int  nbh_rend_init(struct nb_rdata *rd, unsigned int maxmtls,
                   unsigned int maxtris, unsigned int maxinsts,
                   unsigned int spp);
void nbh_rend_release(struct nb_rdata *rd);
int  nbh_rend_resaccum(struct nb_rdata *rd, unsigned int w, unsigned int h);
void nbh_rend_clraccum(struct nb_rdata *rd);

// Bridge: scene -> render data.
int  nbh_cpy_rdata(struct nb_rdata *rd, const struct nbh_scene *s);
int  nbh_upd_rinsts(struct nb_rdata *rd, const struct nbh_scene *s);
void nbh_upd_rcam(struct nb_rdata *rd, const struct nbh_cam *c,
                  float w, float h);

// BVH8 build (16-bin SAH, 8-wide, 4 tris / 1 instance per leaf).
void         nbh_prepstatic(struct nb_rdata *rd);
void         nbh_prepdynamic(struct nb_rdata *rd);
unsigned int nbh_build_bvh8(struct nb_bnode8 *nodes, struct nb_aabb *aabbs,
                            unsigned int *imap, const struct nb_rtri *tris,
                            unsigned int pcnt,
                            struct nb_vec3 rootmin, struct nb_vec3 rootmax);

// Convenience: everything from scene to a ready render data in one call
// (rend_init, cpy_rdata, prepstatic, upd_rinsts, prepdynamic, resaccum,
// upd_rcam) with the scene's own resolution and spp.
int nbh_rdata_from_scene(struct nb_rdata *rd, const struct nbh_scene *s);

// 4x4 row-major inverse (mat4.c:299); returns 1 if singular.
int nbh_mat4_inv(float dst[16], const float m[16]);

#ifdef __cplusplus
}
#endif

#endif
