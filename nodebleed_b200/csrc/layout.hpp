// Host conversion of the reference BVH8 (bnode8/leaf4 byte trees in
// rd->bnodes) into the GPU layout of gpulayout.h, and the light table.

#ifndef NB_LAYOUT_HPP
#define NB_LAYOUT_HPP

#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "gpulayout.h"
#include "host/nb_rdata.h"

namespace nb {

struct bvh_stats {
	uint32_t depth = 0;  // longest root-to-leaf chain of nodes
	uint32_t nodes = 0;
	uint32_t items = 0;
};

// Append the BLAS rooted at bnodes[2 * triofs] to `nodes`/`tris`; returns
// the root node index.  Triangles come from rd->tris (original vertices).
// Returns false with `err` set on a malformed tree.
bool convert_blas(const nb_rdata *rd, uint32_t triofs,
                  std::vector<nb_qnode> &nodes, std::vector<nb_gtri> &tris,
                  uint32_t *root, bvh_stats *st, std::string *err);

// Append the TLAS rooted at bnodes[tlasofs] to `nodes` (its root index in
// *root) and its instance references, offset by inst_base, to `irefs`.
bool convert_tlas(const nb_rdata *rd, std::vector<nb_qnode> &nodes,
                  std::vector<uint32_t> &irefs, uint32_t inst_base,
                  uint32_t *root, bvh_stats *st, std::string *err);

// Mesh-local ids of the EMISSIVE triangles of every mesh (keyed by its
// triofs) that an instance of rd uses: the per-mesh scan build_lights
// needs, done once per static upload.
void find_emitters(const nb_rdata *rd,
                   std::unordered_map<uint32_t, std::vector<uint32_t>> &out);

// World-space emitting triangles of instances whose material is EMISSIVE,
// with an area CDF; returns the total area.  `emitters` (from
// find_emitters) limits the scan to emissive triangles; null scans every
// triangle of every instance.
float build_lights(const nb_rdata *rd, std::vector<nb_glight> &lights,
                   const std::unordered_map<uint32_t,
                   std::vector<uint32_t>> *emitters = nullptr);

// Settings of the BLAS build (blas_build.cpp): SAH cost of visiting an
// 8-wide node and of testing one triangle, per unit of box area.
struct blas_params {
	float c_node = 1.0f;
	float c_tri = 0.3f;
};

// One BLAS in the GPU layout with node and item indices from 0 (append_blas
// moves them to their place in the shared arrays).
struct blas_out {
	std::vector<nb_qnode> nodes;
	std::vector<nb_gtri> tris;
	uint32_t depth = 0;
};

// SAH binary build + optimal 8-wide collapse of the mesh's triangles
// rd->tris[triofs .. triofs + tricnt).  Returns false with `err` set on a
// mesh it cannot build (no triangles, non-finite vertices).
bool build_blas(const nb_rdata *rd, uint32_t triofs, uint32_t tricnt,
                const blas_params &prm, blas_out *out, std::string *err);

// build_blas of several meshes on the host's cores.
bool build_blas_many(const nb_rdata *rd, const std::vector<uint32_t> &triofs,
                     const std::vector<uint32_t> &tricnt,
                     const blas_params &prm, std::vector<blas_out> &out,
                     std::string *err);

// Append a built BLAS to the shared node and triangle arrays; *root gets
// its root node index.
void append_blas(const blas_out &b, std::vector<nb_qnode> &nodes,
                 std::vector<nb_gtri> &tris, uint32_t *root);

// Quantise one node: child boxes (min/max per slot; empty slots have
// min > max) into n (origin, exponents, qlo/qhi).  Exposed for tests.
void quantise_node(const float cmin[8][3], const float cmax[8][3],
                   nb_qnode *n);

} // namespace nb

#endif
