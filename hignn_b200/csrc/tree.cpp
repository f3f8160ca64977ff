// Cluster tree (PCA bisection at the mean) and close/far block lists, host C++.
//
// Restates src/HignnModel.cpp:119-198 (Divide), src/Build.cpp:17-265 (Build for
// one rank), src/CloseFarCheck.cpp:11-454 (bounding boxes, dual traversal,
// list flattening) and src/HignnModel.cpp:482-518 (admissibility). Compiled
// with -ffp-contract=off so that every float/double operation rounds exactly
// as written; the lists are then bit-identical to the oracle's restatement.
//
// Choices where the reference is solver-defined: the principal axis is the
// dominant eigenvector of the FP64 covariance (cyclic Jacobi) rounded to float,
// sign chosen so its largest-magnitude component is positive (the reference
// uses Eigen's JacobiSVD, whose sign is implementation-defined); the sort by
// projection is stable (the reference's std::sort is not).
#include "tree.h"
#include "tree_math.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <utility>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace hignn {

namespace {

// Scratch of one thread's divisions, allocated once per tree build (fresh allocations of the
// top nodes' sizes at every division cost more in first-touch page faults than the work).
struct DivideScratch {
  std::vector<float> vh, tv;
  std::vector<uint32_t> kb, order;
  std::vector<uint64_t> ra, rb;
  std::vector<int64_t> pcopy;
  std::vector<std::pair<float, int64_t>> key;
};

// Stable sort of positions 0..L-1 by kb (ascending), written to s.order: the permutation
// std::stable_sort gives with operator< on the floats behind the keys. LSD radix, 8-bit
// digits, digits on which all keys agree skipped. With `threads` > 1 each pass histograms
// and scatters contiguous chunks per thread; the chunk-major prefix keeps it stable.
void radix_order(DivideScratch& s, int64_t L, int threads) {
  std::vector<uint64_t>& a = s.ra;
  std::vector<uint64_t>& b = s.rb;
  a.resize(L);
  b.resize(L);
  for (int64_t i = 0; i < L; i++) a[i] = ((uint64_t)s.kb[i] << 32) | (uint64_t)i;
  const int T = threads > 1 ? threads : 1;
  std::vector<int64_t> hist((size_t)T * 256);
  for (int shift = 32; shift < 64; shift += 8) {
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T) if (T > 1)
    {
#ifdef _OPENMP
      const int th = T > 1 ? omp_get_thread_num() : 0;
#else
      const int th = 0;
#endif
      const int64_t lo = L * th / T, hi = L * (th + 1) / T;
      int64_t* h = &hist[(size_t)th * 256];
      for (int64_t i = lo; i < hi; i++) h[(a[i] >> shift) & 255]++;
    }
    bool trivial = false;
    for (int d = 0; d < 256 && !trivial; d++) {
      int64_t c = 0;
      for (int th = 0; th < T; th++) c += hist[(size_t)th * 256 + d];
      trivial = (c == L);
    }
    if (trivial) continue;
    int64_t run = 0;  // exclusive prefix over (digit, chunk)
    for (int d = 0; d < 256; d++)
      for (int th = 0; th < T; th++) {
        const int64_t c = hist[(size_t)th * 256 + d];
        hist[(size_t)th * 256 + d] = run;
        run += c;
      }
#pragma omp parallel num_threads(T) if (T > 1)
    {
#ifdef _OPENMP
      const int th = T > 1 ? omp_get_thread_num() : 0;
#else
      const int th = 0;
#endif
      const int64_t lo = L * th / T, hi = L * (th + 1) / T;
      int64_t* h = &hist[(size_t)th * 256];
      for (int64_t i = lo; i < hi; i++) b[h[(a[i] >> shift) & 255]++] = a[i];
    }
    a.swap(b);
  }
  s.order.resize(L);
  for (int64_t i = 0; i < L; i++) s.order[i] = (uint32_t)(a[i] & 0xffffffffu);
}

// Nodes at least this large sort their projections by radix, smaller ones by comparison;
// from kParallelSortMin on (the top divisions) the radix passes use several threads.
constexpr int64_t kRadixMin = 4096;
constexpr int64_t kParallelSortMin = int64_t(1) << 18;

// HignnModel::Divide: returns the split index (first position with t > 0).
int64_t divide(const float* xyz, int64_t* perm, int64_t first, int64_t last, int sort_threads, DivideScratch& s) {
  const int64_t L = last - first;
  // the mean: blocks of kSumBlock consecutive particles summed sequentially, then the block sums
  float mean[3] = {0.f, 0.f, 0.f};
  for (int64_t b0 = first; b0 < last; b0 += kSumBlock) {
    const int64_t b1 = std::min(last, b0 + kSumBlock);
    float bs[3] = {0.f, 0.f, 0.f};
    for (int64_t i = b0; i < b1; i++) {
      const float* p = xyz + 3 * perm[i];
      bs[0] += p[0];
      bs[1] += p[1];
      bs[2] += p[2];
    }
    mean[0] += bs[0];
    mean[1] += bs[1];
    mean[2] += bs[2];
  }
  for (int d = 0; d < 3; d++) mean[d] /= (float)L;
  std::vector<float>& vh = s.vh;
  vh.resize(3 * L);
  double cov[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int64_t i = 0; i < L; i++) {
    const float* p = xyz + 3 * perm[first + i];
    float* q = &vh[3 * i];
    q[0] = p[0] - mean[0];
    q[1] = p[1] - mean[1];
    q[2] = p[2] - mean[2];
  }
  {
    // six sums, blocked as the mean: sequential within each block, then over the block sums
    double s00 = 0.0, s01 = 0.0, s02 = 0.0, s11 = 0.0, s12 = 0.0, s22 = 0.0;
    for (int64_t b0 = 0; b0 < L; b0 += kSumBlock) {
      const int64_t b1 = std::min(L, b0 + kSumBlock);
      double t00 = 0.0, t01 = 0.0, t02 = 0.0, t11 = 0.0, t12 = 0.0, t22 = 0.0;
      for (int64_t i = b0; i < b1; i++) {
        const double x = vh[3 * i], y = vh[3 * i + 1], z = vh[3 * i + 2];
        t00 += x * x;
        t01 += x * y;
        t02 += x * z;
        t11 += y * y;
        t12 += y * z;
        t22 += z * z;
      }
      s00 += t00;
      s01 += t01;
      s02 += t02;
      s11 += t11;
      s12 += t12;
      s22 += t22;
    }
    cov[0][0] = s00;
    cov[0][1] = cov[1][0] = s01;
    cov[0][2] = cov[2][0] = s02;
    cov[1][1] = s11;
    cov[1][2] = cov[2][1] = s12;
    cov[2][2] = s22;
  }
  double ud[3];
  jacobi_dominant_axis(cov, ud);
  const float u0 = (float)ud[0], u1 = (float)ud[1], u2 = (float)ud[2];
  auto project = [&](int64_t i) {
    const float* q = &vh[3 * i];
    return project_axis(u0, u1, u2, q[0], q[1], q[2]);
  };
  // upper_bound(t, 0) over the sorted projections: first position with t strictly above zero
  auto first_positive = [L](auto&& sorted_t) {
    int64_t lo = 0, hi = L;
    while (lo < hi) {
      int64_t mid = (lo + hi) / 2;
      if (0.0f < sorted_t(mid))
        hi = mid;
      else
        lo = mid + 1;
    }
    return lo;
  };
  int64_t split;
  if (L >= kRadixMin) {
    // the permutation a stable comparison sort gives (below), by radix; whole-machine threads
    // for the top divisions, which run outside the per-level parallel loop
    s.tv.resize(L);
    s.kb.resize(L);
    for (int64_t i = 0; i < L; i++) {
      s.tv[i] = project(i);
      s.kb[i] = float_key(s.tv[i]);
    }
#ifdef _OPENMP
    const int threads = (omp_in_parallel() || L < kParallelSortMin) ? 1 : sort_threads;
#else
    const int threads = 1;
#endif
    radix_order(s, L, threads);
    s.pcopy.assign(perm + first, perm + last);
    for (int64_t i = 0; i < L; i++) perm[first + i] = s.pcopy[s.order[i]];
    split = first_positive([&](int64_t k) { return s.tv[s.order[k]]; });
  } else {
    std::vector<std::pair<float, int64_t>>& key = s.key;
    key.resize(L);
    for (int64_t i = 0; i < L; i++) key[i] = {project(i), perm[first + i]};
    std::stable_sort(key.begin(), key.end(),
                     [](const std::pair<float, int64_t>& x, const std::pair<float, int64_t>& y) {
                       return x.first < y.first;
                     });
    for (int64_t i = 0; i < L; i++) perm[first + i] = key[i].second;
    split = first_positive([&](int64_t k) { return key[k].first; });
  }
  return split + first;
}

}  // namespace

ClusterTree build_tree(const float* xyz, int64_t n, int64_t leaf, int num_threads) {
  ClusterTree t;
  t.perm.resize(n);
  std::iota(t.perm.begin(), t.perm.end(), (int64_t)0);
  std::vector<DivideScratch> scratch((size_t)std::max(1, num_threads));
  t.nodes = build_tree_rows(n, leaf, [&](const std::vector<NodeRange>& rg, std::vector<int64_t>& split) {
    const int64_t m = (int64_t)rg.size();
    split.assign(m, 0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads) if (m > 1)
    for (int64_t i = 0; i < m; i++) {
#ifdef _OPENMP
      DivideScratch& sc = scratch[omp_in_parallel() ? omp_get_thread_num() : 0];
#else
      DivideScratch& sc = scratch[0];
#endif
      split[i] = divide(xyz, t.perm.data(), rg[i].start, rg[i].end, num_threads, sc);
    }
  });
  return t;
}

bool is_far(const float* a, const float* b) {
  if (!(a[0] > b[1] || a[1] < b[0] || a[2] > b[3] || a[3] < b[2] || a[4] > b[5] || a[5] < b[4]))
    return false;
  float d0 = 0.f, d1 = 0.f, dist = 0.f, tmp;
  for (int j = 0; j < 3; j++) {
    tmp = a[2 * j] - a[2 * j + 1];
    d0 += tmp * tmp;
    tmp = b[2 * j] - b[2 * j + 1];
    d1 += tmp * tmp;
    tmp = a[2 * j] + a[2 * j + 1] - b[2 * j] - b[2 * j + 1];
    dist += tmp * tmp;
  }
  dist *= 0.25f;
  return (dist > d0) && (dist > d1);
}

BlockLists build_lists(const ClusterTree& t, const float* xt, int64_t max_rel, bool use_symmetry, int num_threads) {
  const int nthr = num_threads > 0 ? num_threads : 1;
  BlockLists L;
  const int64_t nn = (int64_t)t.nodes.size();
  L.aux.assign(6 * nn, 0.f);
  for (int64_t i = 0; i < nn; i++) L.aux[6 * i] = -FLT_MAX;
  // bounding boxes of every node reachable from the root (src/CloseFarCheck.cpp:19-175);
  // an internal node's box is min/max of its children, i.e. of its whole range.
  {
    std::vector<int64_t> st{0};
    std::vector<int64_t> reach;
    while (!st.empty()) {
      int64_t nd = st.back();
      st.pop_back();
      reach.push_back(nd);
      if (t.nodes[nd].child0 != 0) {
        st.push_back(t.nodes[nd].child0);
        st.push_back(t.nodes[nd].child1);
      }
    }
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthr)
    for (int64_t r = 0; r < (int64_t)reach.size(); r++) {
      const int64_t nd = reach[r];
      float bx[6] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
      for (int64_t i = t.nodes[nd].start; i < t.nodes[nd].end; i++)
        for (int d = 0; d < 3; d++) {
          const float v = xt[3 * i + d];
          bx[2 * d] = (bx[2 * d] > v) ? v : bx[2 * d];
          bx[2 * d + 1] = (bx[2 * d + 1] < v) ? v : bx[2 * d + 1];
        }
      for (int k = 0; k < 6; k++) L.aux[6 * nd + k] = bx[k];
    }
  }
  auto size = [&](int64_t nd) { return t.nodes[nd].end - t.nodes[nd].start; };
  auto leafq = [&](int64_t nd) { return t.nodes[nd].child0 == 0; };
  std::vector<std::vector<int64_t>> farM(nn), closeM(nn);
  closeM[0].push_back(0);
  // dual traversal (src/CloseFarCheck.cpp:186-290), breadth first over the row tree. A FIFO
  // queue visits the tree level by level, each level in the order its parents were visited;
  // here the levels are taken one at a time in that order, and the nodes of a level in
  // parallel (a node reads its own close list and writes only its own far list and its
  // children's or its own close list), so every list comes out as the queue would build it.
  auto visit = [&](int64_t i) {
    const float* ai = &L.aux[6 * i];
    if (!leafq(i)) {
      std::vector<int64_t> childClose;
      for (int64_t j : closeM[i]) {
        bool far = is_far(ai, &L.aux[6 * j]) && size(i) < max_rel && size(j) < max_rel;
        if (far) {
          farM[i].push_back(j);
        } else if (!leafq(j)) {
          childClose.push_back(t.nodes[j].child0);
          childClose.push_back(t.nodes[j].child1);
        } else {
          childClose.push_back(j);
        }
      }
      closeM[t.nodes[i].child0] = childClose;
      closeM[t.nodes[i].child1] = std::move(childClose);
    } else {
      std::vector<int64_t> newClose;
      for (int64_t j : closeM[i]) {
        if (is_far(ai, &L.aux[6 * j])) {
          if (size(j) < max_rel) {
            farM[i].push_back(j);
          } else {
            std::vector<int64_t> st{j};
            while (!st.empty()) {
              int64_t c = st.back();
              st.pop_back();
              if (size(c) < max_rel) {
                farM[i].push_back(c);
              } else {
                st.push_back(t.nodes[c].child0);
                st.push_back(t.nodes[c].child1);
              }
            }
          }
        } else if (leafq(j)) {
          newClose.push_back(j);
        } else {
          std::vector<int64_t> st{j};
          while (!st.empty()) {
            int64_t c = st.back();
            st.pop_back();
            if (!leafq(c)) {
              st.push_back(t.nodes[c].child0);
              st.push_back(t.nodes[c].child1);
            } else {
              newClose.push_back(c);
            }
          }
        }
      }
      closeM[i].swap(newClose);
    }
  };
  std::vector<int64_t> level{0}, next;
  while (!level.empty()) {
    const int64_t m = (int64_t)level.size();
#pragma omp parallel for schedule(dynamic, 16) if (m > 64) num_threads(nthr)
    for (int64_t q = 0; q < m; q++) visit(level[q]);
    next.clear();
    for (int64_t i : level) {
      if (leafq(i)) {
        L.leaves.push_back(i);
      } else {
        next.push_back(t.nodes[i].child0);
        next.push_back(t.nodes[i].child1);
      }
    }
    level.swap(next);
  }
  // flattening (src/CloseFarCheck.cpp:298-336, 385-408), one rank
  for (int64_t i : L.leaves)
    for (int64_t j : closeM[i])
      if (!use_symmetry || j >= i) {
        L.closeI.push_back(i);
        L.closeJ.push_back(j);
      }
  for (int64_t i = 0; i < nn; i++)
    for (int64_t j : farM[i])
      if (!use_symmetry || j >= i) {
        L.farI.push_back(i);
        L.farJ.push_back(j);
      }
  return L;
}

}  // namespace hignn
