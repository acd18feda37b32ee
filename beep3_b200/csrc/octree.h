// Flat description of the adaptive octree shared by the near-field builder,
// the FMM schedule and the test exporter.
#pragma once

#include <cstdint>
#include <vector>

namespace bp {

enum : int32_t { TREE_HAS_CHILDREN = 1, TREE_LEAF = 2, TREE_SHADOW = 4 };

struct TreeNode {
  int32_t level;
  uint32_t ix, iy, iz;
  double centre[3];
  double edge;
  int32_t flags;
  int32_t parent;
  int32_t children[8];     // child id c+1 at index c, -1 when absent
  int32_t neighbours[27];  // same-level neighbour nodes, -1 when absent
  int64_t content_start;   // into TreeInfo::contents
  int32_t content_count;
  int32_t mp_idx;          // multipole / plane-wave slot in its level, -1 if empty
  int32_t lc_idx;          // local-expansion slot in its level, -1 if shadow
};

struct TreeInfo {
  int n_levels = 0;
  std::vector<TreeNode> nodes;     // level by level, map order inside a level
  std::vector<int> level_start;    // n_levels + 1
  std::vector<int32_t> contents;   // patch indices, insertion order per node
  std::vector<int> n_mp_per_level, n_lc_per_level;
};

void build_reference_tree(const double* centroids, int n, const double centre[3], double edge, int nbsize,
                          TreeInfo& out);

}  // namespace bp
