// Byte-compatible mirror of nodebleed's render-data structs (rend.h:15-147).
//
// The GPU library reads the application's `struct rdata` directly, so every
// struct here has the size, field order and offsets of its rend.h namesake.
// The AVX types of rend.h (__m256, __m256i, __m128, __m128i) become plain
// arrays with the same size and alignment, so this header needs no
// <immintrin.h> and compiles under nvcc.  tests/test_layout.py compares every
// size and offset with the compiled reference.

#ifndef NB_RDATA_H
#define NB_RDATA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NB_BRANCH_MAX     8          // rend.h:9
#define NB_BLAS_LEAF_MAX  4          // rend.h:10
#define NB_TLAS_LEAF_MAX  1          // rend.h:11
#define NB_NODE_LEAF      0x80000000u // rend.h:13
#define NB_INST_ID_BITS   12         // rend.c:24
#define NB_INST_ID_MASK   0xfffu     // rend.c:25

// Flags of types.h:4-18 that the renderer reads.
#define NB_FLAG_MESH       0x0001u
#define NB_FLAG_DISABLED   0x0100u
#define NB_FLAG_INVISIBLE  0x0400u
#define NB_FLAG_NOSHADOW   0x0800u
#define NB_FLAG_EMISSIVE   0x1000u

#define NB_A32 __attribute__((aligned(32)))
#define NB_A16 __attribute__((aligned(16)))

struct nb_vec3 { // vec3.h:4
	float x, y, z;
};

struct nb_bnode8 { // rend.h:17-30, 256 bytes
	float    minx8[8] NB_A32;
	float    maxx8[8] NB_A32;
	float    miny8[8] NB_A32;
	float    maxy8[8] NB_A32;
	float    minz8[8] NB_A32;
	float    maxz8[8] NB_A32;
	uint32_t children8[8] NB_A32; // NODE_LEAF | byte ofs, or byte ofs
	uint32_t perm8[8] NB_A32;     // 8 octants x 3 bit child order
} NB_A32;

struct nb_leaf4 { // rend.h:32-45, 192 bytes
	float    v0x4[4] NB_A16;
	float    v0y4[4] NB_A16;
	float    v0z4[4] NB_A16;
	float    e0x4[4] NB_A16;
	float    e0y4[4] NB_A16;
	float    e0z4[4] NB_A16;
	float    e1x4[4] NB_A16;
	float    e1y4[4] NB_A16;
	float    e1z4[4] NB_A16;
	uint32_t id4[4] NB_A16;
	uint32_t tricnt;
	uint32_t pad[7];
} NB_A16;

struct nb_aabb { // rend.h:47-52, 32 bytes
	struct nb_vec3 min;
	float          pad0;
	struct nb_vec3 max;
	float          pad1;
};

struct nb_rmtl { // rend.h:54-61, 32 bytes
	struct nb_vec3 col;
	float          metallic;
	float          roughness;
	float          ior;
	uint32_t       flags;
	uint32_t       pad0;
};

struct nb_rtri { // rend.h:63-70, 48 bytes
	struct nb_vec3 v0;
	float          pad0;
	struct nb_vec3 v1;
	float          pad1;
	struct nb_vec3 v2;
	float          pad2;
};

struct nb_rnrm { // rend.h:72-79, 48 bytes
	struct nb_vec3 n0;
	uint32_t       mtlid;
	struct nb_vec3 n1;
	uint32_t       pad0;
	struct nb_vec3 n2;
	uint32_t       pad1;
};

struct nb_rinst { // rend.h:81-87, 64 bytes
	float    globinv[12]; // world -> object, row-major 3x4
	uint32_t flags;
	uint32_t triofs;
	uint32_t tricnt;
	uint32_t pad0;
};

struct nb_rcam { // rend.h:89-117
	struct nb_vec3 eye;
	float          tanvfov;
	struct nb_vec3 ri;
	float          focdist;
	struct nb_vec3 up;
	float          tanfangle;
	struct nb_vec3 fwd;
	float          aspect;
	float eyex8[8] NB_A32, eyey8[8] NB_A32, eyez8[8] NB_A32;
	float rix8[8] NB_A32, riy8[8] NB_A32, riz8[8] NB_A32;
	float upx8[8] NB_A32, upy8[8] NB_A32, upz8[8] NB_A32;
	float fwdx8[8] NB_A32, fwdy8[8] NB_A32, fwdz8[8] NB_A32;
	float rw8[8] NB_A32;
	float rh8[8] NB_A32;
	float aspect8[8] NB_A32;
	float fdist8[8] NB_A32;
	float fovfdist8[8] NB_A32;
	float focangle8[8] NB_A32;
	float focrad8[8] NB_A32;
} NB_A32;

struct nb_rdata { // rend.h:119-147
	struct nb_rmtl   *mtls;
	struct nb_rtri   *tris;
	struct nb_rnrm   *nrms;
	unsigned int     instcnt;
	struct nb_rinst  *insts;
	struct nb_aabb   *aabbs;
	struct nb_bnode8 *bnodes;
	unsigned int     tlasofs;
	struct nb_rcam   cam;
	struct nb_vec3   bgcol;
	unsigned int     width;
	unsigned int     height;
	struct nb_vec3   *acc;
	unsigned int     *buf;
	int              blknum;
	unsigned int     rays;
	unsigned int     spp;
	unsigned int     samples;
} NB_A32;

#ifdef __cplusplus
}
#endif

#endif
