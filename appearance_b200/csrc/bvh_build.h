// Host builder of the compressed 8-wide BVH consumed by traverse.cuh.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "scene_layout.h"

namespace ap {

struct BvhStats {
  uint32_t num_nodes = 0;
  uint32_t num_tris = 0;
  uint32_t max_depth = 0;
  uint32_t max_stack = 0;  // worst-case traversal stack entries
  double build_ms = 0.0;
  double sah_cost = 0.0;
};

struct WideBvh {
  std::vector<WideNode> nodes;
  std::vector<TriRec> tris;
  BvhStats stats;
};

// Builds from world-space triangles (9 floats each, global id = index).
// Returns false with `err` set when the tree would exceed `max_stack` entries
// of traversal stack.
bool build_wide_bvh(const float* tri_verts, uint32_t num_tris, uint32_t max_stack, WideBvh* out,
                    std::string* err);

}  // namespace ap
