// Device neighbour lists: the two-body and three-body edge lists of the reference's NeighborLists
// class (include/NeighborLists.hpp), built on the GPU from a cell list instead of a kd-tree.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.h"
#include "kernels.h"

namespace hignn {

// Kinds of edge list (the reference's getters, include/NeighborLists.hpp:289-464).
enum EdgeKind : int {
  kEdgesTwoBody = 0,        // (2, E): (i, j), j a neighbour of i at the two-body epsilon
  kEdgesThreeBody = 1,      // (3, E): (i, j, k), j a neighbour of i, k one of j other than i
  kEdgesThreeBodySelf = 2,  // (2, E): (i, j), j a neighbour of i at the three-body epsilon
};

// Neighbours j != i of every particle within one radius, as CSR: nbr[off[i] .. off[i + 1]) in
// ascending order.
struct NeighbourCsr {
  int64_t edges = 0;
  bool host_off_valid = false;
  DevBuf deg, off, nbr;
  std::vector<int64_t> h_off;
};

class NeighbourLists {
 public:
  explicit NeighbourLists(int device);
  ~NeighbourLists();
  NeighbourLists(const NeighbourLists&) = delete;
  NeighbourLists& operator=(const NeighbourLists&) = delete;

  void update_coord(const float* xyz, int64_t n);
  // The same from device positions (float4, w unused); the caller's writes to x4 must be complete.
  void update_coord_device(const float4* x4, int64_t n);
  void set_two_body_epsilon(float e) { eps2_ = e; }
  void set_three_body_epsilon(float e) { eps3_ = e; }
  void build_two_body();
  void build_three_body();
  int64_t size() const { return n_; }

  // Edge count of one list, or (by_index) of its ByIndex variant for the nindex targets.
  int64_t count(int kind, bool by_index, const uint64_t* index, int64_t nindex);
  // Writes that (rows, count) list, row-major, to host memory out.
  void copy_out(int kind, bool by_index, const uint64_t* index, int64_t nindex, uint64_t* out);
  // The whole list on the device, (rows, edges) row-major, owned by this object.
  const uint64_t* device_list(int kind, int64_t* edges) const;
  cudaStream_t stream() const { return stream_; }
  const float4* positions() const { return x4_.as<float4>(); }
  int device() const { return device_; }
  double last_build_ms() const { return build_ms_; }

 private:
  void build_csr(float eps, NeighbourCsr& c);
  void ensure_host_off(NeighbourCsr& c, int64_t n);
  void check_index(const uint64_t* index, int64_t nindex) const;
  int rows(int kind) const { return kind == kEdgesThreeBody ? 3 : 2; }

  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  int64_t n_ = 0;
  float eps2_ = 0.f, eps3_ = 0.f;
  bool built2_ = false, built3_ = false;
  double build_ms_ = 0.0;
  DevBuf x4_, scan_tmp_, index_, loc_off_, out_;
  CellList cells_;
  NeighbourCsr two_, three_;
  DevBuf info2_, self3_, info3_;  // uint64 edge lists, (rows, E) row-major
  NeighbourCsr trip_;             // three-body triplet counts and offsets (nbr unused)
};

}  // namespace hignn
