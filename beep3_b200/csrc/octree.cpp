// Host-side adaptive octree with the reference libBEEP refinement rules.
//
// The octree decides which patch pairs are integrated explicitly (the 27-box
// neighbourhood of every leaf) and which interact through the FMM, so the
// near field and the FMM of the matvec are only comparable with the
// reference when this tree matches the reference's.  Rules restated from
// src/fmm/octree.h:
//   * non-strict insertion: a childless node splits once it holds more than
//     4*nbsize items (src/fmm/octree.h:1118-1148); children take the parent's
//     items in insertion order (src/fmm/octree.h:120-131);
//   * build_neighbourhoods: every node with children makes its 27 neighbours
//     split too, the new children being "shadow" non-leaves
//     (src/fmm/octree.h:780-806, :1187-1235);
//   * optimize_neighbourhoods: repeatedly split the fattest leaves (by the
//     cached neighbourhood count, which the reference never invalidates)
//     until floor(mean explicit work per item) <= nbsize
//     (src/fmm/octree.h:867-986);
//   * remove_empty_nodes (src/fmm/octree.h:1052-1083);
//   * node order inside a level is the std::map order of OctreeIndexer,
//     i.e. x + y*2^L + z*4^L (src/common/octree_indexer.h:142-185);
//   * neighbour numbering nb = 9*(dz+1) + 3*(dy+1) + (dx+1)
//     (src/common/octree_indexer.h:350-391); child ids 1..8 with
//     x = (id-1)&1, y = ((id-1)>>1)&1, z = (id-1)>>2 (src/fmm/octree.h:84-113).
// FMM bookkeeping (src/fmm/fmm_bem_hybrid.h:644-720): walking levels
// bottom-up in map order, every non-shadow node gets a local-expansion slot
// and every non-empty node a multipole / plane-wave slot.
#include "octree.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <stdexcept>
#include <unordered_map>

namespace bp {

namespace {

constexpr int kMaxDepth = 20;  // OctreeIndexer::MAX_LEVELS for 64-bit longs

struct Node {
  int level;
  uint32_t ix, iy, iz;
  double c[3];
  double edge;
  bool has_children = false, is_leaf = true, is_shadow = false, is_deleted = false, removed = false;
  int parent = -1;
  int children[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
  std::vector<int> contents;
  int cached_nb = -1;
};

inline uint64_t key(uint32_t x, uint32_t y, uint32_t z, int level) {
  uint64_t e = 1ull << level;
  return (uint64_t)x + (uint64_t)y * e + (uint64_t)z * e * e;
}

class RefTree {
 public:
  RefTree(const double* pts, int n, const double centre[3], double edge, int nbsize)
      : pts_(pts), nbsize_(nbsize), edge_(edge) {
    Node root;
    root.level = 0;
    root.ix = root.iy = root.iz = 0;
    for (int k = 0; k < 3; ++k) root.c[k] = centre[k];
    root.edge = edge;
    nodes_.push_back(root);
    levels_.emplace_back();
    levels_[0][0] = 0;
    index_.emplace_back();
    index_[0][0] = 0;
    for (int i = 0; i < n; ++i) add(i);
  }

  void build_neighbourhoods() {
    for (int level = 0; level < (int)levels_.size(); ++level) {
      std::vector<int> with_children;
      for (auto& kv : levels_[level]) {
        const Node& nd = nodes_[kv.second];
        if (nd.has_children && !nd.is_shadow) with_children.push_back(kv.second);
      }
      for (int id : with_children) subdivide_neighbourhood(id);
    }
  }

  void optimize_neighbourhoods() {
    size_t total_items = 0;
    for (auto& lvl : levels_)
      for (auto& kv : lvl) {
        const Node& nd = nodes_[kv.second];
        if (!nd.is_shadow && nd.is_leaf && !nd.is_deleted) total_items += nd.contents.size();
      }
    if (total_items == 0) return;
    double avg = (double)neighbourhood_interacts() / total_items;
    while (std::floor(avg) > nbsize_) {
      std::vector<int> sorted;
      for (auto& lvl : levels_)
        for (auto& kv : lvl) {
          const Node& nd = nodes_[kv.second];
          if (!nd.is_shadow && nd.is_leaf && !nd.contents.empty()) {
            if (cached_nb(kv.second) > (size_t)nbsize_) sorted.push_back(kv.second);
          }
        }
      std::sort(sorted.begin(), sorted.end(),
                [&](int a, int b) { return nodes_[a].cached_nb > nodes_[b].cached_nb; });
      int fatty = 0;
      int estimate = 1 + (int)std::ceil(sorted.size() * (avg - nbsize_) / avg);
      for (int id : sorted) {
        nodes_[id].is_leaf = false;
        if (nodes_[id].has_children) {
          for (int c = 0; c < 8; ++c) {
            int ch = nodes_[id].children[c];
            if (ch < 0) continue;
            nodes_[ch].is_shadow = false;
            nodes_[ch].is_leaf = true;
          }
        } else {
          subdivide(id);
        }
        subdivide_neighbourhood(id);
        if (++fatty >= estimate) break;
      }
      avg = (double)neighbourhood_interacts() / total_items;
    }
  }

  void remove_empty_nodes() {
    for (int level = (int)levels_.size() - 1; level >= 0; --level) {
      std::vector<uint64_t> empties;
      for (auto& kv : levels_[level]) {
        Node& nd = nodes_[kv.second];
        if (nd.contents.empty() && kv.second != 0) {
          empties.push_back(kv.first);
          if (nd.parent >= 0) nodes_[nd.parent].children[child_id(nd) - 1] = -1;
        }
      }
      for (uint64_t k : empties) {
        nodes_[levels_[level][k]].removed = true;
        levels_[level].erase(k);
        index_[level].erase(k);
      }
    }
  }

  void export_to(TreeInfo& out) const {
    out.n_levels = (int)levels_.size();
    out.nodes.clear();
    std::vector<int> remap(nodes_.size(), -1);
    for (int level = 0; level < (int)levels_.size(); ++level)
      for (auto& kv : levels_[level]) {
        remap[kv.second] = (int)out.nodes.size();
        TreeNode tn;
        const Node& nd = nodes_[kv.second];
        tn.level = nd.level;
        tn.ix = nd.ix; tn.iy = nd.iy; tn.iz = nd.iz;
        for (int k = 0; k < 3; ++k) tn.centre[k] = nd.c[k];
        tn.edge = nd.edge;
        tn.flags = (nd.has_children ? TREE_HAS_CHILDREN : 0) | (nd.is_leaf ? TREE_LEAF : 0) |
                   (nd.is_shadow ? TREE_SHADOW : 0);
        out.nodes.push_back(tn);
      }
    out.level_start.assign(out.n_levels + 1, 0);
    for (auto& tn : out.nodes) out.level_start[tn.level + 1]++;
    for (int l = 0; l < out.n_levels; ++l) out.level_start[l + 1] += out.level_start[l];
    out.contents.clear();
    for (size_t i = 0; i < nodes_.size(); ++i) {
      if (remap[i] < 0) continue;
      TreeNode& tn = out.nodes[remap[i]];
      const Node& nd = nodes_[i];
      tn.parent = nd.parent >= 0 ? remap[nd.parent] : -1;
      for (int c = 0; c < 8; ++c) tn.children[c] = nd.children[c] >= 0 ? remap[nd.children[c]] : -1;
    }
    std::vector<int> inv(out.nodes.size(), -1);
    for (size_t i = 0; i < nodes_.size(); ++i)
      if (remap[i] >= 0) inv[remap[i]] = (int)i;
    for (size_t j = 0; j < out.nodes.size(); ++j) {
      const Node& nd = nodes_[inv[j]];
      out.nodes[j].content_start = (int64_t)out.contents.size();
      out.nodes[j].content_count = (int)nd.contents.size();
      out.contents.insert(out.contents.end(), nd.contents.begin(), nd.contents.end());
    }
    // neighbour lookup by (level, ix, iy, iz)
    for (size_t j = 0; j < out.nodes.size(); ++j) {
      TreeNode& tn = out.nodes[j];
      uint32_t E = 1u << tn.level;
      for (int nb = 0; nb < 27; ++nb) {
        int dz = nb / 9 - 1, dy = (nb % 9) / 3 - 1, dx = nb % 3 - 1;
        long x = (long)tn.ix + dx, y = (long)tn.iy + dy, z = (long)tn.iz + dz;
        tn.neighbours[nb] = -1;
        if (x < 0 || y < 0 || z < 0 || x >= (long)E || y >= (long)E || z >= (long)E) continue;
        auto it = index_[tn.level].find(key((uint32_t)x, (uint32_t)y, (uint32_t)z, tn.level));
        if (it != index_[tn.level].end()) tn.neighbours[nb] = remap[it->second];
      }
    }
    // FMM slots (bottom-up, map order)
    std::vector<int> mp(out.n_levels, 0), lc(out.n_levels, 0);
    for (int level = out.n_levels - 1; level >= 0; --level)
      for (int j = out.level_start[level]; j < out.level_start[level + 1]; ++j) {
        TreeNode& tn = out.nodes[j];
        tn.lc_idx = (tn.flags & TREE_SHADOW) ? -1 : lc[level]++;
        tn.mp_idx = tn.content_count > 0 ? mp[level]++ : -1;
      }
    out.n_mp_per_level = mp;
    out.n_lc_per_level = lc;
  }

 private:
  const double* pts_;
  int nbsize_;
  double edge_;
  std::vector<Node> nodes_;
  std::vector<std::map<uint64_t, int>> levels_;  // ordered: the node order of a level
  std::vector<std::unordered_map<uint64_t, int>> index_;  // the same nodes, for lookups
  std::vector<uint8_t> cid_;  // scratch: child of each item of the node being split

  static int child_id(const Node& nd) {
    return 1 + (nd.ix & 1) + 2 * (nd.iy & 1) + 4 * (nd.iz & 1);
  }

  int child_for(const Node& nd, int item) const {
    const double* p = pts_ + 3 * (size_t)item;
    int id = 1;
    if (p[0] > nd.c[0]) id += 1;
    if (p[1] > nd.c[1]) id += 2;
    if (p[2] > nd.c[2]) id += 4;
    return id;
  }

  void add(int item) {
    int id = 0;
    while (true) {
      Node& nd = nodes_[id];
      const double* p = pts_ + 3 * (size_t)item;
      for (int k = 0; k < 3; ++k) {
        double d = std::fabs(2.0 * (p[k] - nd.c[k]) / nd.edge);
        if (d > 1.0 + 1e-9) throw std::invalid_argument("patch centroid outside the bounding cube");
      }
      nd.contents.push_back(item);
      if (!nd.has_children) {
        if (nd.contents.size() > (size_t)nbsize_ * 4 && nd.level < kMaxDepth) {
          subdivide(id);
          nodes_[id].is_leaf = false;
        }
        return;
      }
      id = nd.children[child_for(nd, item) - 1];
    }
  }

  int find(int level, long x, long y, long z) const {
    if (level >= (int)levels_.size()) return -1;
    long E = 1l << level;
    if (x < 0 || y < 0 || z < 0 || x >= E || y >= E || z >= E) return -1;
    auto it = index_[level].find(key((uint32_t)x, (uint32_t)y, (uint32_t)z, level));
    return it == index_[level].end() ? -1 : it->second;
  }

  void subdivide(int id) {
    if (nodes_[id].has_children) return;
    nodes_[id].has_children = true;
    int new_level = nodes_[id].level + 1;
    while ((int)levels_.size() <= new_level) {
      levels_.emplace_back();
      index_.emplace_back();
    }
    const int first = (int)nodes_.size();
    nodes_.resize(first + 8);
    const Node& par = nodes_[id];
    for (int o = 0; o < 8; ++o) {
      Node& ch = nodes_[first + o];
      ch.level = new_level;
      ch.edge = par.edge / 2.0;
      ch.ix = par.ix * 2 + (o & 1);
      ch.iy = par.iy * 2 + ((o >> 1) & 1);
      ch.iz = par.iz * 2 + (o >> 2);
      ch.c[0] = par.c[0] + ((o & 1) ? ch.edge / 2.0 : -ch.edge / 2.0);
      ch.c[1] = par.c[1] + (((o >> 1) & 1) ? ch.edge / 2.0 : -ch.edge / 2.0);
      ch.c[2] = par.c[2] + ((o >> 2) ? ch.edge / 2.0 : -ch.edge / 2.0);
      ch.parent = id;
    }
    // children take the parent's items in its insertion order
    const size_t m = par.contents.size();
    cid_.resize(m);
    size_t count[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t i = 0; i < m; ++i) {
      const double* p = pts_ + 3 * (size_t)par.contents[i];
      const int o = (p[0] > par.c[0]) + 2 * (p[1] > par.c[1]) + 4 * (p[2] > par.c[2]);
      cid_[i] = (uint8_t)o;
      ++count[o];
    }
    int* out[8];
    for (int o = 0; o < 8; ++o) {
      nodes_[first + o].contents.resize(count[o]);
      out[o] = nodes_[first + o].contents.data();
    }
    for (size_t i = 0; i < m; ++i) *out[cid_[i]]++ = par.contents[i];
    for (int o = 0; o < 8; ++o) {
      nodes_[id].children[o] = first + o;
      const Node& ch = nodes_[first + o];
      const uint64_t k = key(ch.ix, ch.iy, ch.iz, new_level);
      levels_[new_level].emplace(k, first + o);
      index_[new_level].emplace(k, first + o);
    }
  }

  void subdivide_neighbourhood(int id) {
    const int level = nodes_[id].level;
    const long bx = nodes_[id].ix, by = nodes_[id].iy, bz = nodes_[id].iz;
    for (int nb = 0; nb < 27; ++nb) {
      int dz = nb / 9 - 1, dy = (nb % 9) / 3 - 1, dx = nb % 3 - 1;
      int nid = find(level, bx + dx, by + dy, bz + dz);
      if (nid < 0) continue;
      if (!nodes_[nid].has_children) {
        subdivide(nid);
        for (int c = 0; c < 8; ++c) {
          Node& ch = nodes_[nodes_[nid].children[c]];
          ch.is_leaf = false;
          ch.is_shadow = true;
        }
      } else {
        for (int c = 0; c < 8; ++c) {
          int ch = nodes_[nid].children[c];
          if (ch < 0) break;
          nodes_[ch].is_deleted = false;
        }
      }
    }
  }

  size_t count_nb(int id) const {
    const Node& nd = nodes_[id];
    size_t r = nd.contents.size();
    for (int nb = 0; nb < 27; ++nb) {
      if (nb == 13) continue;
      int dz = nb / 9 - 1, dy = (nb % 9) / 3 - 1, dx = nb % 3 - 1;
      int nid = find(nd.level, (long)nd.ix + dx, (long)nd.iy + dy, (long)nd.iz + dz);
      if (nid >= 0) r += nodes_[nid].contents.size();
    }
    return r;
  }

  size_t cached_nb(int id) {
    Node& nd = nodes_[id];
    if (nd.cached_nb == -1) nd.cached_nb = (int)count_nb(id);
    return (size_t)nd.cached_nb;
  }

  size_t neighbourhood_interacts() {
    size_t total = 0;
    for (int level = 0; level < (int)levels_.size() && level < kMaxDepth; ++level)
      for (auto& kv : levels_[level]) {
        const Node& nd = nodes_[kv.second];
        if (nd.is_leaf && !nd.is_shadow && !nd.is_deleted) {
          long nbs = (long)cached_nb(kv.second);
          total += nbs * nodes_[kv.second].contents.size();
        }
      }
    return total;
  }
};

}  // namespace

void build_reference_tree(const double* centroids, int n, const double centre[3], double edge, int nbsize,
                          TreeInfo& out) {
  if (nbsize <= 0) throw std::invalid_argument("nbsize must be positive");
  if (!(edge > 0)) throw std::invalid_argument("bounding cube edge must be positive");
  RefTree t(centroids, n, centre, edge, nbsize);
  t.build_neighbourhoods();
  t.optimize_neighbourhoods();
  t.remove_empty_nodes();
  t.export_to(out);
}

}  // namespace bp
