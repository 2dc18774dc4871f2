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

// Quantise one node: child boxes (min/max per slot; empty slots have
// min > max) into n (origin, exponents, qlo/qhi).  Exposed for tests.
void quantise_node(const float cmin[8][3], const float cmax[8][3],
                   nb_qnode *n);

} // namespace nb

#endif
