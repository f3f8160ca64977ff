// Device neighbour lists (the reference's NeighborLists, include/NeighborLists.hpp).
//
// The reference finds, per particle, every source within epsilon with a nanoflann kd-tree radius
// search (include/PointCloudSearch.hpp:274-450; metric sqrt(sum (double)(x_j - x_i)^2) squared,
// strict < epsilon^2 with epsilon squared in float), swaps the particle itself to the front
// (include/NeighborLists.hpp:166-225), and from those lists builds
//   two-body edges   (i, j)     for j in N(i) \ {i}                      (:466-510)
//   three-body edges (i, j, k)  for j in N(i) \ {i}, k in N(j) \ {j, i}  (:512-585)
//   self edges       (i, j)     for j in N(i) \ {i} at the three-body epsilon.
// Here the same neighbour test runs on a uniform cell grid (cells no smaller than epsilon), so the
// sets are identical; each particle's neighbours are kept in ascending order, so the edges come
// out sorted by (i, j, k). The reference's order within a particle is the kd-tree's traversal
// order, which depends on its tree build; callers use the lists as index sets.
//
// Layout in HBM: per radius a CSR (deg / off int64[n + 1], nbr int32[E]); the edge lists as the
// reference returns them, uint64 (rows, E) row-major. The triplets of particle i start at
// trip.off[i] = sum over earlier particles of sum_j (|N(j)| - [i in N(j)]).
#include <cub/device/device_scan.cuh>

#include <chrono>
#include <cmath>
#include <cstring>

#include "neighbors.h"

namespace hignn {

namespace {

inline unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Edge list (i, j) of a CSR: one warp per particle, lanes over its neighbours.
__global__ void k_pairs(const int64_t* __restrict__ off, const int* __restrict__ nbr, int64_t n,
                        uint64_t* __restrict__ out, int64_t e) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  for (int64_t t = off[w] + lane; t < off[w + 1]; t += 32) {
    out[t] = (uint64_t)w;
    out[e + t] = (uint64_t)nbr[t];
  }
}

__device__ __forceinline__ bool sorted_contains(const int* __restrict__ a, int64_t lo, int64_t hi, int v) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int x = a[mid];
    if (x == v) return true;
    if (x < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return false;
}

// Triplets of each particle: sum over j in N(i) of |N(j) \ {i}| (include/NeighborLists.hpp:520-529
// counts |N(j)| - 2 with the self entry included, i.e. assumes i in N(j); here it is checked).
__global__ void k_triplet_count(const int64_t* __restrict__ off, const int* __restrict__ nbr, int64_t n,
                                int64_t* __restrict__ cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  if (i == n) {
    cnt[n] = 0;
    return;
  }
  int64_t c = 0;
  for (int64_t t = off[i]; t < off[i + 1]; t++) {
    const int j = nbr[t];
    const int64_t b = off[j], e = off[j + 1];
    c += (e - b) - (sorted_contains(nbr, b, e, (int)i) ? 1 : 0);
  }
  cnt[i] = c;
}

// Triplets (i, j, k), one warp per particle i: j over N(i) in order, lanes over N(j) \ {i}.
__global__ void k_triplets(const int64_t* __restrict__ off, const int* __restrict__ nbr,
                           const int64_t* __restrict__ off3, int64_t n, uint64_t* __restrict__ out, int64_t e3) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const unsigned below = (1u << lane) - 1u;
  int64_t pos = off3[w];
  for (int64_t t = off[w]; t < off[w + 1]; t++) {
    const int j = nbr[t];
    const int64_t b = off[j], e = off[j + 1];
    for (int64_t q0 = b; q0 < e; q0 += 32) {  // bounds are the same in every lane
      const int64_t q = q0 + lane;
      const int k = q < e ? nbr[q] : -1;
      const bool keep = q < e && k != (int)w;
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int64_t p = pos + __popc(m & below);
        out[p] = (uint64_t)w;
        out[e3 + p] = (uint64_t)j;
        out[2 * e3 + p] = (uint64_t)k;
      }
      pos += __popc(m);
    }
  }
}

// GetTwoBodyEdgeInfoByIndex (include/NeighborLists.hpp:309-340): for every target p, all
// j != p in ascending order, rows (j, p).
__global__ void k_all_others(const uint64_t* __restrict__ idx, int64_t m, int64_t n, uint64_t* __restrict__ out) {
  const int64_t per = n - 1, total = m * per;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = e / per, r = e - t * per;
    const uint64_t p = idx[t];
    out[e] = (uint64_t)r < p ? (uint64_t)r : (uint64_t)r + 1;
    out[total + e] = p;
  }
}

// ByIndex variants of the three-body lists (include/NeighborLists.hpp:362-464): the edges of
// each target in turn, rows reversed ((k, j, i) and (j, i)). One warp per target.
__global__ void k_gather_reversed(const uint64_t* __restrict__ info, int64_t e, int rows,
                                  const int64_t* __restrict__ off, const uint64_t* __restrict__ idx,
                                  const int64_t* __restrict__ loc, int64_t m, uint64_t* __restrict__ out,
                                  int64_t total) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= m) return;
  const uint64_t p = idx[w];
  const int64_t src = off[p], cnt = off[p + 1] - src, dst = loc[w];
  for (int64_t q = lane; q < cnt; q += 32)
    for (int r = 0; r < rows; r++) out[r * total + dst + q] = info[(int64_t)(rows - 1 - r) * e + src + q];
}

void exclusive_scan(DevBuf& tmp, const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
  size_t bytes = 0;
  HIGNN_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
  tmp.ensure(bytes > 0 ? bytes : 1);
  HIGNN_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n, s));
}

int64_t read_last(const DevBuf& off, int64_t n, cudaStream_t s) {
  int64_t v = 0;
  HIGNN_CUDA(cudaMemcpyAsync(&v, off.as<int64_t>() + n, sizeof(v), cudaMemcpyDeviceToHost, s));
  HIGNN_CUDA(cudaStreamSynchronize(s));
  return v;
}

}  // namespace

NeighbourLists::NeighbourLists(int device) : device_(device) {
  HIGNN_CUDA(cudaSetDevice(device_));
  HIGNN_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
}

NeighbourLists::~NeighbourLists() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (DevBuf* b : {&x4_, &scan_tmp_, &index_, &loc_off_, &out_, &info2_, &self3_, &info3_}) b->release();
  cells_.release();
  for (NeighbourCsr* c : {&two_, &three_, &trip_}) {
    c->deg.release();
    c->off.release();
    c->nbr.release();
  }
  if (stream_) cudaStreamDestroy(stream_);
}

// NeighborLists::UpdateCoord (include/NeighborLists.hpp:252-279): copies the coordinates; lists
// built before stay as they are until the next build.
void NeighbourLists::update_coord(const float* xyz, int64_t n) {
  if (n < 0 || (n > 0 && !xyz)) throw Error(-1, "neighbour lists: bad coordinates");
  if (n > (int64_t)INT32_MAX - 1) throw Error(-1, "neighbour lists: more than 2^31 - 2 particles");
  std::vector<float4> h(n);
  for (int64_t i = 0; i < n; i++) {
    const float a = xyz[3 * i], b = xyz[3 * i + 1], c = xyz[3 * i + 2];
    if (!(std::isfinite(a) && std::isfinite(b) && std::isfinite(c)))
      throw Error(-1, "neighbour lists: coordinates must be finite");
    h[i] = make_float4(a, b, c, 0.f);
  }
  HIGNN_CUDA(cudaSetDevice(device_));
  x4_.ensure(sizeof(float4) * (n > 0 ? n : 1));
  if (n > 0) HIGNN_CUDA(cudaMemcpyAsync(x4_.p, h.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, stream_));
  HIGNN_CUDA(cudaStreamSynchronize(stream_));
  n_ = n;
}

void NeighbourLists::update_coord_device(const float4* x4, int64_t n) {
  if (n < 0 || (n > 0 && !x4)) throw Error(-1, "neighbour lists: bad coordinates");
  if (n > (int64_t)INT32_MAX - 1) throw Error(-1, "neighbour lists: more than 2^31 - 2 particles");
  HIGNN_CUDA(cudaSetDevice(device_));
  x4_.ensure(sizeof(float4) * (n > 0 ? n : 1));
  if (n > 0) HIGNN_CUDA(cudaMemcpyAsync(x4_.p, x4, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
  HIGNN_CUDA(cudaStreamSynchronize(stream_));
  n_ = n;
}

void NeighbourLists::build_csr(float eps, NeighbourCsr& c) {
  if (!(eps > 0.f)) throw Error(-1, "neighbour lists: the epsilon must be positive");
  const int64_t n = n_;
  c.deg.ensure(sizeof(int64_t) * (n + 1));
  c.off.ensure(sizeof(int64_t) * (n + 1));
  c.host_off_valid = false;
  HIGNN_CUDA(cudaMemsetAsync(c.deg.p, 0, sizeof(int64_t) * (n + 1), stream_));
  if (n > 0) {
    cells_.build(x4_.as<float4>(), n, eps, stream_);
    launch_neighbours(x4_.as<float4>(), n, cells_, eps, c.deg.as<int64_t>(), nullptr, nullptr, stream_);
  }
  exclusive_scan(scan_tmp_, c.deg.as<int64_t>(), c.off.as<int64_t>(), n + 1, stream_);
  c.edges = read_last(c.off, n, stream_);
  c.nbr.ensure(sizeof(int) * (c.edges > 0 ? c.edges : 1));
  if (c.edges > 0)
    launch_neighbours(x4_.as<float4>(), n, cells_, eps, nullptr, c.off.as<int64_t>(), c.nbr.as<int>(), stream_);
}

// NeighborLists::BuildTwoBodyInfo (include/NeighborLists.hpp:466-510).
void NeighbourLists::build_two_body() {
  HIGNN_CUDA(cudaSetDevice(device_));
  const auto t0 = std::chrono::steady_clock::now();
  build_csr(eps2_, two_);
  info2_.ensure(sizeof(uint64_t) * 2 * (two_.edges > 0 ? two_.edges : 1));
  if (two_.edges > 0) {
    k_pairs<<<nblocks(n_ * 32, 256), 256, 0, stream_>>>(two_.off.as<int64_t>(), two_.nbr.as<int>(), n_,
                                                        info2_.as<uint64_t>(), two_.edges);
    HIGNN_CHECK_LAUNCH();
  }
  HIGNN_CUDA(cudaStreamSynchronize(stream_));
  build_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  built2_ = true;
}

// NeighborLists::BuildThreeBodyInfo (include/NeighborLists.hpp:512-585).
void NeighbourLists::build_three_body() {
  HIGNN_CUDA(cudaSetDevice(device_));
  const auto t0 = std::chrono::steady_clock::now();
  build_csr(eps3_, three_);
  const int64_t n = n_;
  self3_.ensure(sizeof(uint64_t) * 2 * (three_.edges > 0 ? three_.edges : 1));
  if (three_.edges > 0) {
    k_pairs<<<nblocks(n * 32, 256), 256, 0, stream_>>>(three_.off.as<int64_t>(), three_.nbr.as<int>(), n,
                                                       self3_.as<uint64_t>(), three_.edges);
    HIGNN_CHECK_LAUNCH();
  }
  trip_.deg.ensure(sizeof(int64_t) * (n + 1));
  trip_.off.ensure(sizeof(int64_t) * (n + 1));
  trip_.host_off_valid = false;
  k_triplet_count<<<nblocks(n + 1, 256), 256, 0, stream_>>>(three_.off.as<int64_t>(), three_.nbr.as<int>(), n,
                                                            trip_.deg.as<int64_t>());
  HIGNN_CHECK_LAUNCH();
  exclusive_scan(scan_tmp_, trip_.deg.as<int64_t>(), trip_.off.as<int64_t>(), n + 1, stream_);
  trip_.edges = read_last(trip_.off, n, stream_);
  info3_.ensure(sizeof(uint64_t) * 3 * (trip_.edges > 0 ? trip_.edges : 1));
  if (trip_.edges > 0) {
    k_triplets<<<nblocks(n * 32, 256), 256, 0, stream_>>>(three_.off.as<int64_t>(), three_.nbr.as<int>(),
                                                          trip_.off.as<int64_t>(), n, info3_.as<uint64_t>(),
                                                          trip_.edges);
    HIGNN_CHECK_LAUNCH();
  }
  HIGNN_CUDA(cudaStreamSynchronize(stream_));
  build_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  built3_ = true;
}

void NeighbourLists::ensure_host_off(NeighbourCsr& c, int64_t n) {
  if (c.host_off_valid) return;
  c.h_off.resize(n + 1);
  HIGNN_CUDA(cudaMemcpyAsync(c.h_off.data(), c.off.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, stream_));
  HIGNN_CUDA(cudaStreamSynchronize(stream_));
  c.host_off_valid = true;
}

void NeighbourLists::check_index(const uint64_t* index, int64_t nindex) const {
  if (nindex < 0 || (nindex > 0 && !index)) throw Error(-1, "neighbour lists: bad target index array");
  for (int64_t t = 0; t < nindex; t++)
    if (index[t] >= (uint64_t)n_) throw Error(-1, "neighbour lists: target index out of range");
}

const uint64_t* NeighbourLists::device_list(int kind, int64_t* edges) const {
  switch (kind) {
    case kEdgesTwoBody:
      *edges = built2_ ? two_.edges : 0;
      return built2_ ? info2_.as<uint64_t>() : nullptr;
    case kEdgesThreeBody:
      *edges = built3_ ? trip_.edges : 0;
      return built3_ ? info3_.as<uint64_t>() : nullptr;
    case kEdgesThreeBodySelf:
      *edges = built3_ ? three_.edges : 0;
      return built3_ ? self3_.as<uint64_t>() : nullptr;
    default:
      throw Error(-1, "neighbour lists: unknown edge kind");
  }
}

int64_t NeighbourLists::count(int kind, bool by_index, const uint64_t* index, int64_t nindex) {
  int64_t e = 0;
  device_list(kind, &e);  // validates kind
  if (!by_index) return e;
  check_index(index, nindex);
  if (kind == kEdgesTwoBody) return n_ > 0 ? nindex * (n_ - 1) : 0;
  if (!built3_) return 0;
  NeighbourCsr& c = kind == kEdgesThreeBody ? trip_ : three_;
  ensure_host_off(c, n_);
  int64_t total = 0;
  for (int64_t t = 0; t < nindex; t++) total += c.h_off[index[t] + 1] - c.h_off[index[t]];
  return total;
}

void NeighbourLists::copy_out(int kind, bool by_index, const uint64_t* index, int64_t nindex, uint64_t* out) {
  HIGNN_CUDA(cudaSetDevice(device_));
  const int64_t total = count(kind, by_index, index, nindex);
  const int r = rows(kind);
  if (total == 0) return;
  if (!out) throw Error(-1, "neighbour lists: null output");
  if (!by_index) {
    int64_t e = 0;
    const uint64_t* d = device_list(kind, &e);
    HIGNN_CUDA(cudaMemcpyAsync(out, d, sizeof(uint64_t) * r * e, cudaMemcpyDeviceToHost, stream_));
    HIGNN_CUDA(cudaStreamSynchronize(stream_));
    return;
  }
  index_.ensure(sizeof(uint64_t) * nindex);
  HIGNN_CUDA(cudaMemcpyAsync(index_.p, index, sizeof(uint64_t) * nindex, cudaMemcpyHostToDevice, stream_));
  out_.ensure(sizeof(uint64_t) * r * total);
  if (kind == kEdgesTwoBody) {
    k_all_others<<<nblocks(total, 256) < 148 * 64 ? nblocks(total, 256) : 148 * 64, 256, 0, stream_>>>(
        index_.as<uint64_t>(), nindex, n_, out_.as<uint64_t>());
    HIGNN_CHECK_LAUNCH();
  } else {
    NeighbourCsr& c = kind == kEdgesThreeBody ? trip_ : three_;
    std::vector<int64_t> loc(nindex);
    int64_t acc = 0;
    for (int64_t t = 0; t < nindex; t++) {
      loc[t] = acc;
      acc += c.h_off[index[t] + 1] - c.h_off[index[t]];
    }
    loc_off_.ensure(sizeof(int64_t) * nindex);
    HIGNN_CUDA(cudaMemcpyAsync(loc_off_.p, loc.data(), sizeof(int64_t) * nindex, cudaMemcpyHostToDevice, stream_));
    int64_t e = 0;
    const uint64_t* info = device_list(kind, &e);
    k_gather_reversed<<<nblocks(nindex * 32, 256), 256, 0, stream_>>>(info, e, r, c.off.as<int64_t>(),
                                                                      index_.as<uint64_t>(), loc_off_.as<int64_t>(),
                                                                      nindex, out_.as<uint64_t>(), total);
    HIGNN_CHECK_LAUNCH();
    HIGNN_CUDA(cudaStreamSynchronize(stream_));  // loc must outlive the copy above
  }
  HIGNN_CUDA(cudaMemcpyAsync(out, out_.p, sizeof(uint64_t) * r * total, cudaMemcpyDeviceToHost, stream_));
  HIGNN_CUDA(cudaStreamSynchronize(stream_));
}

}  // namespace hignn
