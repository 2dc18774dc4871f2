// GPU layout of the two-level BVH (host conversion and device traversal).
//
// The reference's 256-byte bnode8 (8 child boxes as FP32 SoA + offsets +
// a per-octant child order) becomes an 80-byte node with the child boxes
// quantised to 8 bits per plane against a per-node origin and power-of-two
// scale (five 16-byte loads per node instead of sixteen).  Inner children of a
// node are stored contiguously in slot order; leaf items (triangles of the
// BLAS, instance references of the TLAS) of a node are stored contiguously.
// Slots are assigned so that visiting them in the order key = slot ^ octant
// approximates near-to-far for a ray of that octant.
//
// Quantised boxes are conservative: every child plane lies at least 1/32 of a
// quantum outside the FP32 child box, which covers the absolute rounding
// error of the device's plane distances, and the device test widens the far
// distance by a relative 2^-20, so no ray that enters an FP32 child box
// misses its quantised box.

#ifndef NB_GPULAYOUT_H
#define NB_GPULAYOUT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// meta byte of a slot: 0 = empty, inner children are in imask,
// leaf = 0x80 | (count - 1) << 5 | offset from the node's item base.
#define NB_META_LEAF 0x80u

struct nb_qnode { // 80 bytes, 16-byte aligned
	float    px, py, pz;     // origin of the quantisation grid
	uint8_t  ex, ey, ez;     // scale = 2^(e - 119) per axis
	uint8_t  imask;          // bit s: slot s is an inner node
	uint32_t child_base;     // node index of the first inner child
	uint32_t item_base;      // index of the first leaf item
	uint8_t  meta[8];
	uint8_t  qlox[8], qloy[8], qloz[8];
	uint8_t  qhix[8], qhiy[8], qhiz[8];
};

// A BLAS triangle as its three original vertices (48 bytes); .w of the first
// holds the mesh-local triangle id (as the reference's leaf4 id4).
struct nb_gtri {
	float v0[3];
	uint32_t prim;
	float v1[3];
	uint32_t pad1;
	float v2[3];
	uint32_t pad2;
};

// An instance: world->object 3x4, BLAS root node, first triangle of its mesh
// in the render data (for rnrm lookups), flags (64 bytes).
struct nb_ginst {
	float    m[12];
	uint32_t root;
	uint32_t triofs;
	uint32_t flags;
	uint32_t pad;
};

// Light table entry (80 bytes): an emitting triangle in world space.
struct nb_glight {
	float v0[3], e0[3], e1[3], n[3], emit[3];
	float cdf, area, pad[3];
};

#define NB_MAX_DEPTH_LIMIT 64

#ifdef __cplusplus
}
#endif

#endif
