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

// Divide + Build of src/HignnModel.cpp:119-198 and src/Build.cpp:17-265 for one rank.
ClusterTree build_tree(const float* xyz, int64_t n, int64_t leaf, int num_threads);

// ComputeAux + dual traversal + flattening, src/CloseFarCheck.cpp:11-454.
// num_threads: OpenMP threads of the two parallel loops (the lists do not depend on it).
BlockLists build_lists(const ClusterTree& t, const float* xyz_tree, int64_t max_relative_coord,
                       bool use_symmetry, int num_threads);

// HignnModel::CloseFarCheck(aux, n1, n2), src/HignnModel.cpp:482-518.
bool is_far(const float* a, const float* b);

// Dominant eigenvector of a symmetric 3x3 (cyclic Jacobi, FP64).
void jacobi_dominant_axis(const double cov[3][3], double u[3]);

}  // namespace hignn
