// Device build of the cluster tree (tree_dev.cu): the same rows and permutation as build_tree.
#pragma once

#include <cuda_runtime.h>

#include "common.h"
#include "tree.h"

namespace hignn {

// Device buffers of the tree build, kept by the model between builds (grown, never shrunk).
struct TreeDevScratch {
  DevBuf xyz;          // caller-order coordinates (n, 3)
  DevBuf xt, xt2;      // positions in the current particle order (float4), double-buffered
  DevBuf perm, perm2;  // particle order (int32), double-buffered
  DevBuf keys, keys2, vals, vals2, cpos, cub_tmp;
  DevBuf lvl_i32, lvl_f4, lvl_f8;  // per-level node and block tables
  DevBuf node_i32, aux, lst_i32, near_pool, far_pool, flat_i32, outI, outJ, err;  // lists
  void release();
};

// Tree of the n caller-order coordinates at d_xyz (device, (n, 3) float) with leaf size `leaf`.
// On return S.xt holds the positions in tree order (x, y, z, 0) and S.perm the permutation
// (tree position -> caller index); both are also in the returned tree (perm on the host).
ClusterTree build_tree_device(const float* d_xyz, int64_t n, int64_t leaf, TreeDevScratch& S, cudaStream_t st);

// Close and far lists of tree t (ComputeAux + CloseFarCheck, src/CloseFarCheck.cpp:11-465) on the
// device, from the tree-order positions d_xt; the same lists, in the same order, as build_lists.
// Returns false (L untouched) when the tree is too deep for the device traversal's expansion stack;
// the caller then builds the lists on the host.
bool build_lists_device(const ClusterTree& t, const float4* d_xt, int64_t max_relative_coord, bool use_symmetry,
                        TreeDevScratch& S, cudaStream_t st, BlockLists& L);

}  // namespace hignn
