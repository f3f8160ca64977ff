// Host-side cluster tree and close/far lists (one process per GPU; every GPU
// builds its own copy, which is cheaper than broadcasting it).
#pragma once

#include <cstdint>
#include <vector>

namespace hignn {

struct TreeNode {
  int64_t child0, child1, start, end, level;
};

struct ClusterTree {
  std::vector<TreeNode> nodes;   // row layout of src/Build.cpp: [c0, c1, start, end, level]
  std::vector<int64_t> perm;     // tree position -> caller index (reorderedMap)
};

struct BlockLists {
  std::vector<int64_t> closeI, closeJ;  // leaf pairs, reference order
  std::vector<int64_t> farI, farJ;      // node pairs, reference order
  std::vector<int64_t> leaves;          // leaves in BFS order (mLeafNodeList)
  std::vector<float> aux;               // 6 floats per node: xmin,xmax,ymin,ymax,zmin,zmax
};

struct NodeRange {
  int64_t start, end;
};

// The reference treats a split index of 0 as a leaf (src/Build.cpp:71,160). An empty child
// (coincident points) would make it recurse forever; a leaf here.
inline bool split_ok(int64_t d, int64_t first, int64_t last) { return d != 0 && d != first && d != last; }

// Build of src/Build.cpp:17-265 for one rank: the tree rows, with the divisions delegated to
// divide_level(ranges, splits), which divides every range (all larger than `leaf`) -- permuting
// the particle order inside it -- and returns each split position. The host and the device
// builds share this driver and differ only in divide_level.
//   Sequential stage (:38-97): one rank => initial level 0, the root is divided once (rows 1, 2).
//   Parallel stage (:108-180): the local tree restarts from node 0 and divides it again; the
//   nodes of a level are divided together and their children numbered in BFS order.
//   Merge (:199-247): rows 0..2 from the sequential stage, local nodes from row 3 with child ids
//   shifted by +2, the root re-pointed at rows 3, 4 (rows 1, 2 become orphans).
template <class DivideLevel>
std::vector<TreeNode> build_tree_rows(int64_t n, int64_t leaf, DivideLevel&& divide_level) {
  TreeNode init[3] = {{0, 0, 0, n, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};
  std::vector<NodeRange> rg;
  std::vector<int64_t> sp;
  if (n > leaf) {
    rg.assign(1, NodeRange{0, n});
    divide_level(rg, sp);
    const int64_t d = sp[0];
    if (split_ok(d, 0, n)) {
      init[0].child0 = 1;
      init[0].child1 = 2;
      init[1] = {0, 0, 0, d, 1};
      init[2] = {0, 0, d, n, 1};
    }
  }
  std::vector<TreeNode> local;
  local.push_back(init[0]);
  std::vector<int64_t> frontier{0}, next, todo;
  while (!frontier.empty()) {
    rg.clear();
    todo.clear();
    for (int64_t node : frontier) {
      const TreeNode& nd = local[node];
      if (nd.end - nd.start > leaf) {
        rg.push_back(NodeRange{nd.start, nd.end});
        todo.push_back(node);
      } else {
        local[node].child0 = local[node].child1 = 0;
      }
    }
    sp.clear();
    if (!rg.empty()) divide_level(rg, sp);
    next.clear();
    for (size_t q = 0; q < todo.size(); q++) {
      const int64_t node = todo[q];
      const TreeNode nd = local[node];
      if (!split_ok(sp[q], nd.start, nd.end)) {
        local[node].child0 = local[node].child1 = 0;
        continue;
      }
      const int64_t c0 = (int64_t)local.size();
      local.push_back({0, 0, nd.start, sp[q], nd.level + 1});
      local.push_back({0, 0, sp[q], nd.end, nd.level + 1});
      local[node].child0 = c0;
      local[node].child1 = c0 + 1;
      next.push_back(c0);
      next.push_back(c0 + 1);
    }
    frontier.swap(next);
  }
  const int64_t nloc = (int64_t)local.size() - 1;
  std::vector<TreeNode> rows;
  if (nloc == 0) {
    // N <= leaf: the reference points the root at rows 3, 4 of a 3-row tree
    // (src/Build.cpp:239-240); here the root is a single leaf.
    rows.push_back({0, 0, 0, n, 0});
    return rows;
  }
  rows.resize(nloc + 3);
  for (int i = 0; i < 3; i++) rows[i] = init[i];
  for (int64_t i = 0; i < nloc; i++) {
    TreeNode r = local[i + 1];
    if (r.child0 != 0) {
      r.child0 += 2;
      r.child1 += 2;
    }
    rows[3 + i] = r;
  }
  rows[0].child0 = 3;
  rows[0].child1 = 4;
  return rows;
}

// Divide + Build of src/HignnModel.cpp:119-198 and src/Build.cpp:17-265 for one rank, on the host.
ClusterTree build_tree(const float* xyz, int64_t n, int64_t leaf, int num_threads);

// ComputeAux + dual traversal + flattening, src/CloseFarCheck.cpp:11-454.
// num_threads: OpenMP threads of the two parallel loops (the lists do not depend on it).
BlockLists build_lists(const ClusterTree& t, const float* xyz_tree, int64_t max_relative_coord,
                       bool use_symmetry, int num_threads);

// HignnModel::CloseFarCheck(aux, n1, n2), src/HignnModel.cpp:482-518.
bool is_far(const float* a, const float* b);


}  // namespace hignn
