// Leaf-capped octree built on the device from Morton codes: the engine's
// performance tree, beside the reference-rule tree of octree.cpp.
//
// Rules (the reference's adaptive octree, src/fmm/octree.h, with its
// nbsize-driven refinement replaced by a cap on the patches of a leaf):
//   * a node with more than `cap` patches splits (down to level 20, the
//     reference's OctreeIndexer depth); its children are leaves unless they
//     split in turn;
//   * build_neighbourhoods (src/fmm/octree.h:780-806, :1187-1235): level by
//     level, every non-shadow node that split makes each of its existing 26
//     same-level neighbours split too; a neighbour split this way keeps its
//     own flags and its new children are shadows (not leaves, never split by
//     size, split only as neighbours of a split non-shadow node);
//   * empty nodes do not exist (remove_empty_nodes, :1052-1083).
// A patch's cell at the finest level comes from its centroid:
// i = floor((p - (c - e/2)) / e * 2^20), clamped to [0, 2^20); a node of
// level l is the cell prefix i >> (20 - l), child o = x + 2y + 4z of the
// next bits.  Morton codes interleave the cells (x lowest of each triple),
// so after a radix sort by code every node's patches are one contiguous
// range, in code order.
//
// The device does the per-patch work: codes, the sort, and per level the
// segmentation of the still-active patches into nodes (run heads and an
// exclusive scan).  The host decides per node (split by size, split as a
// neighbour, shadow and leaf flags: thousands of nodes, not patches) and
// assembles the same TreeInfo as the reference-rule builder: levels in map
// order (x + y 2^L + z 4^L), contents per node and level, neighbours, FMM
// slots.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace bp {
namespace {

constexpr int kDepth = 20;  // cell bits per axis

__device__ __forceinline__ uint64_t spread3(uint32_t v) {  // bit b of v -> bit 3b
  uint64_t x = v & 0x1FFFFFu;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// cube = {lower corner x y z, centre x y z, edge}; a centroid outside the
// cube (beyond the host tree's 1e-9 relative slack) sets *bad
struct Cube {
  double lo[3], c[3], edge;
};

__global__ void morton_kernel(int n, const double* __restrict__ cen, Cube cube, uint64_t* __restrict__ codes,
                              int32_t* __restrict__ ids, int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c[3];
  for (int k = 0; k < 3; ++k) {
    const double p = cen[3 * (size_t)i + k];
    if (fabs(2.0 * (p - cube.c[k]) / cube.edge) > 1.0 + 1e-9) atomicOr(bad, 1);
    const double t = floor((p - cube.lo[k]) / cube.edge * (double)(1 << kDepth));
    c[k] = (uint32_t)fmin(fmax(t, 0.0), (double)((1 << kDepth) - 1));
  }
  codes[i] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
  ids[i] = i;
}

// heads[i] = 1 where an active patch starts a node of this level (its
// prefix differs from the previous active patch's, or that one is inactive)
__global__ void level_heads_kernel(int n, const uint64_t* __restrict__ codes, const uint8_t* __restrict__ active,
                                   int shift, int32_t* __restrict__ heads) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int h = 0;
  if (active[i]) h = (i == 0 || !active[i - 1] || (codes[i] >> shift) != (codes[i - 1] >> shift)) ? 1 : 0;
  heads[i] = h;
}

// per node k of the level: start, end and code prefix; node_of[i] for every
// active patch; idx = inclusive scan of heads, so a patch's node is idx - 1
__global__ void level_nodes_kernel(int n, const uint64_t* __restrict__ codes, const uint8_t* __restrict__ active,
                                   int shift, const int32_t* __restrict__ heads, const int32_t* __restrict__ idx,
                                   int32_t* __restrict__ start, int32_t* __restrict__ end, uint64_t* __restrict__ key,
                                   int32_t* __restrict__ node_of) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !active[i]) return;
  const int k = idx[i] - 1;
  node_of[i] = k;
  if (heads[i]) {
    start[k] = i;
    key[k] = codes[i] >> shift;
  }
  if (i == n - 1 || !active[i + 1] || heads[i + 1]) end[k] = i + 1;
}

// a patch stays active at the next level when its node splits
__global__ void next_active_kernel(int n, uint8_t* __restrict__ active, const int32_t* __restrict__ node_of,
                                   const uint8_t* __restrict__ split) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !active[i]) return;
  active[i] = split[node_of[i]];
}

uint32_t compact3(uint64_t k, int axis) {  // bits axis, axis+3, ... of k
  uint32_t v = 0;
  for (int b = 0; b < 21; ++b) v |= (uint32_t)((k >> (3 * b + axis)) & 1u) << b;
  return v;
}

struct LevelNode {
  uint64_t key;
  int32_t start, count, parent;  // parent: index in the previous level's list
  bool shadow = false, split_size = false, split_forced = false;
  uint32_t x, y, z;
};

}  // namespace

void build_device_tree(Ctx* c, const double* d_centroids, int n, const double centre[3], double edge, int cap,
                       TreeInfo& out) {
  if (cap <= 0) throw std::invalid_argument("leaf capacity must be positive");
  if (!(edge > 0)) throw std::invalid_argument("bounding cube edge must be positive");
  if (n <= 0) throw std::invalid_argument("no patches");
  cudaStream_t st = c->stream;
  const int threads = 256, blocks = (n + threads - 1) / threads;
  DevBuf codes(c, sizeof(uint64_t) * n), ids(c, sizeof(int32_t) * n), scodes(c, sizeof(uint64_t) * n),
      sids(c, sizeof(int32_t) * n), bad(c, sizeof(int));
  Cube cube;
  for (int k = 0; k < 3; ++k) {
    cube.lo[k] = centre[k] - edge / 2.0;
    cube.c[k] = centre[k];
  }
  cube.edge = edge;
  BP_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), st));
  morton_kernel<<<blocks, threads, 0, st>>>(n, d_centroids, cube, codes.as<uint64_t>(), ids.as<int32_t>(),
                                            bad.as<int>());
  BP_LAUNCH_CHECK();
  int h_bad = 0;
  BP_CUDA(cudaMemcpyAsync(&h_bad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  if (h_bad) throw std::invalid_argument("patch centroid outside the bounding cube");
  size_t tmp_sort = 0, tmp_scan = 0;
  BP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, codes.as<uint64_t>(), scodes.as<uint64_t>(),
                                          ids.as<int32_t>(), sids.as<int32_t>(), n, 0, 3 * kDepth, st));
  BP_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_scan, (int32_t*)nullptr, (int32_t*)nullptr, n, st));
  DevBuf tmp(c, std::max<size_t>(std::max(tmp_sort, tmp_scan), 16));
  BP_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_sort, codes.as<uint64_t>(), scodes.as<uint64_t>(),
                                          ids.as<int32_t>(), sids.as<int32_t>(), n, 0, 3 * kDepth, st));
  DevBuf active(c, n), heads(c, sizeof(int32_t) * n), idx(c, sizeof(int32_t) * n), node_of(c, sizeof(int32_t) * n);
  DevBuf nstart(c, sizeof(int32_t) * n), nend(c, sizeof(int32_t) * n), nkey(c, sizeof(uint64_t) * n),
      nsplit(c, n);
  BP_CUDA(cudaMemsetAsync(active.get(), 1, n, st));
  std::vector<std::vector<LevelNode>> levels;
  std::vector<int32_t> h_start, h_end;
  std::vector<uint64_t> h_key;
  std::vector<int32_t> h_node_of_prev;  // node (previous level) of every patch, at its sorted position
  for (int l = 0; l <= kDepth; ++l) {
    const int shift = 3 * (kDepth - l);
    level_heads_kernel<<<blocks, threads, 0, st>>>(n, scodes.as<uint64_t>(), active.as<uint8_t>(), shift,
                                                   heads.as<int32_t>());
    BP_LAUNCH_CHECK();
    BP_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tmp_scan, heads.as<int32_t>(), idx.as<int32_t>(), n, st));
    int32_t nn = 0;
    BP_CUDA(cudaMemcpyAsync(&nn, idx.as<int32_t>() + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    if (nn == 0) break;
    level_nodes_kernel<<<blocks, threads, 0, st>>>(n, scodes.as<uint64_t>(), active.as<uint8_t>(), shift,
                                                   heads.as<int32_t>(), idx.as<int32_t>(), nstart.as<int32_t>(),
                                                   nend.as<int32_t>(), nkey.as<uint64_t>(), node_of.as<int32_t>());
    BP_LAUNCH_CHECK();
    h_start.resize(nn);
    h_end.resize(nn);
    h_key.resize(nn);
    BP_CUDA(cudaMemcpyAsync(h_start.data(), nstart.get(), sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaMemcpyAsync(h_end.data(), nend.get(), sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaMemcpyAsync(h_key.data(), nkey.get(), sizeof(uint64_t) * nn, cudaMemcpyDeviceToHost, st));
    std::vector<int32_t> h_node_of(n);
    BP_CUDA(cudaMemcpyAsync(h_node_of.data(), node_of.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    std::vector<LevelNode> lv(nn);
    std::unordered_map<uint64_t, int> at;
    at.reserve(2 * (size_t)nn);
    for (int k = 0; k < nn; ++k) {
      LevelNode& nd = lv[k];
      nd.key = h_key[k];
      nd.start = h_start[k];
      nd.count = h_end[k] - h_start[k];
      nd.parent = l == 0 ? -1 : h_node_of_prev[nd.start];
      nd.x = compact3(nd.key, 0);
      nd.y = compact3(nd.key, 1);
      nd.z = compact3(nd.key, 2);
      if (l > 0) nd.shadow = levels[l - 1][nd.parent].split_forced;
      nd.split_size = !nd.shadow && nd.count > cap && l < kDepth;
      at.emplace(nd.key, k);
    }
    // neighbours of split non-shadow nodes split too (shadow children)
    if (l < kDepth) {
      const long E = 1l << l;
      for (int k = 0; k < nn; ++k) {
        if (!lv[k].split_size) continue;
        for (int nb = 0; nb < 27; ++nb) {
          if (nb == 13) continue;
          const long x = (long)lv[k].x + nb % 3 - 1, y = (long)lv[k].y + (nb % 9) / 3 - 1, z = (long)lv[k].z + nb / 9 - 1;
          if (x < 0 || y < 0 || z < 0 || x >= E || y >= E || z >= E) continue;
          uint64_t kk = 0;
          for (int b = 0; b < l; ++b)
            kk |= (((uint64_t)(x >> b) & 1) << (3 * b)) | (((uint64_t)(y >> b) & 1) << (3 * b + 1)) |
                  (((uint64_t)(z >> b) & 1) << (3 * b + 2));
          auto it = at.find(kk);
          if (it == at.end()) continue;
          LevelNode& m = lv[it->second];
          if (!m.split_size) m.split_forced = true;
        }
      }
    }
    std::vector<uint8_t> split(nn);
    bool any = false;
    for (int k = 0; k < nn; ++k) {
      split[k] = (lv[k].split_size || lv[k].split_forced) ? 1 : 0;
      any = any || split[k];
    }
    levels.push_back(std::move(lv));
    h_node_of_prev = std::move(h_node_of);
    if (!any) break;
    BP_CUDA(cudaMemcpyAsync(nsplit.get(), split.data(), nn, cudaMemcpyHostToDevice, st));
    next_active_kernel<<<blocks, threads, 0, st>>>(n, active.as<uint8_t>(), node_of.as<int32_t>(),
                                                   nsplit.as<uint8_t>());
    BP_LAUNCH_CHECK();
    BP_CUDA(cudaStreamSynchronize(st));  // `split` is a host vector
  }
  std::vector<int32_t> order(n);
  BP_CUDA(cudaMemcpyAsync(order.data(), sids.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  BP_CUDA(cudaStreamSynchronize(st));
  // TreeInfo: per level the nodes in map order
  out = TreeInfo();
  out.n_levels = (int)levels.size();
  std::vector<std::vector<int>> pos(levels.size());  // list index -> TreeInfo index
  for (int l = 0; l < out.n_levels; ++l) {
    std::vector<int> perm(levels[l].size());
    for (size_t k = 0; k < perm.size(); ++k) perm[k] = (int)k;
    const uint64_t E = 1ull << l;
    auto map_key = [&](const LevelNode& nd) { return (uint64_t)nd.x + (uint64_t)nd.y * E + (uint64_t)nd.z * E * E; };
    std::sort(perm.begin(), perm.end(),
              [&](int a, int b) { return map_key(levels[l][a]) < map_key(levels[l][b]); });
    pos[l].assign(perm.size(), -1);
    for (int k : perm) {
      pos[l][k] = (int)out.nodes.size();
      const LevelNode& nd = levels[l][k];
      TreeNode tn{};
      tn.level = l;
      tn.ix = nd.x;
      tn.iy = nd.y;
      tn.iz = nd.z;
      tn.edge = edge / (double)(1ull << l);
      tn.centre[0] = centre[0] - edge / 2.0 + (nd.x + 0.5) * tn.edge;
      tn.centre[1] = centre[1] - edge / 2.0 + (nd.y + 0.5) * tn.edge;
      tn.centre[2] = centre[2] - edge / 2.0 + (nd.z + 0.5) * tn.edge;
      const bool has_children = nd.split_size || nd.split_forced;
      const bool leaf = !nd.shadow && !nd.split_size;
      tn.flags = (has_children ? TREE_HAS_CHILDREN : 0) | (leaf ? TREE_LEAF : 0) | (nd.shadow ? TREE_SHADOW : 0);
      tn.parent = -1;
      for (int ch = 0; ch < 8; ++ch) tn.children[ch] = -1;
      tn.content_start = (int64_t)out.contents.size();
      tn.content_count = nd.count;
      out.contents.insert(out.contents.end(), order.begin() + nd.start, order.begin() + nd.start + nd.count);
      out.nodes.push_back(tn);
    }
  }
  out.level_start.assign(out.n_levels + 1, 0);
  for (int l = 0; l < out.n_levels; ++l) out.level_start[l + 1] = out.level_start[l] + (int)levels[l].size();
  for (int l = 1; l < out.n_levels; ++l)
    for (size_t k = 0; k < levels[l].size(); ++k) {
      TreeNode& tn = out.nodes[pos[l][k]];
      const int p = pos[l - 1][levels[l][k].parent];
      tn.parent = p;
      const int o = (int)(tn.ix & 1) + 2 * (int)(tn.iy & 1) + 4 * (int)(tn.iz & 1);
      out.nodes[p].children[o] = pos[l][k];
    }
  // same-level neighbours
  for (int l = 0; l < out.n_levels; ++l) {
    std::unordered_map<uint64_t, int> at;
    const uint64_t E = 1ull << l;
    for (int j = out.level_start[l]; j < out.level_start[l + 1]; ++j) {
      const TreeNode& tn = out.nodes[j];
      at.emplace((uint64_t)tn.ix + (uint64_t)tn.iy * E + (uint64_t)tn.iz * E * E, j);
    }
    for (int j = out.level_start[l]; j < out.level_start[l + 1]; ++j) {
      TreeNode& tn = out.nodes[j];
      for (int nb = 0; nb < 27; ++nb) {
        const long x = (long)tn.ix + nb % 3 - 1, y = (long)tn.iy + (nb % 9) / 3 - 1, z = (long)tn.iz + nb / 9 - 1;
        tn.neighbours[nb] = -1;
        if (x < 0 || y < 0 || z < 0 || x >= (long)E || y >= (long)E || z >= (long)E) continue;
        auto it = at.find((uint64_t)x + (uint64_t)y * E + (uint64_t)z * E * E);
        if (it != at.end()) tn.neighbours[nb] = it->second;
      }
    }
  }
  // FMM slots (bottom-up, map order), as the reference-rule builder
  std::vector<int> mp(out.n_levels, 0), lc(out.n_levels, 0);
  for (int l = out.n_levels - 1; l >= 0; --l)
    for (int j = out.level_start[l]; j < out.level_start[l + 1]; ++j) {
      TreeNode& tn = out.nodes[j];
      tn.lc_idx = (tn.flags & TREE_SHADOW) ? -1 : lc[l]++;
      tn.mp_idx = tn.content_count > 0 ? mp[l]++ : -1;
    }
  out.n_mp_per_level = mp;
  out.n_lc_per_level = lc;
}

}  // namespace bp
