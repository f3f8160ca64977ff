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

void jacobi_dominant_axis(const double cov[3][3], double u[3]) {
  double a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a[i][j] = cov[i][j];
  static const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-36 * diag || off == 0.0) break;
    for (int r = 0; r < 3; r++) {
      const int p = P[r], q = Q[r];
      double apq = a[p][q];
      if (apq == 0.0) continue;
      double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      double t = 1.0 / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
      if (theta < 0.0) t = -t;
      double c = 1.0 / std::sqrt(t * t + 1.0);
      double s = t * c;
      for (int k = 0; k < 3; k++) {
        double akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - s * akq;
        a[k][q] = s * akp + c * akq;
      }
      for (int k = 0; k < 3; k++) {
        double apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - s * aqk;
        a[q][k] = s * apk + c * aqk;
      }
      for (int k = 0; k < 3; k++) {
        double vkp = v[k][p], vkq = v[k][q];
        v[k][p] = c * vkp - s * vkq;
        v[k][q] = s * vkp + c * vkq;
      }
    }
  }
  int best = 0;
  for (int k = 1; k < 3; k++)
    if (a[k][k] > a[best][best]) best = k;
  for (int k = 0; k < 3; k++) u[k] = v[k][best];
  int big = 0;
  for (int k = 1; k < 3; k++)
    if (std::fabs(u[k]) > std::fabs(u[big])) big = k;
  if (u[big] < 0.0)
    for (int k = 0; k < 3; k++) u[k] = -u[k];
}

namespace {

// Order-preserving unsigned image of a finite float; -0.0 and +0.0 share one image, as they
// compare equal under operator<.
inline uint32_t float_key(float f) {
  uint32_t u;
  if (f == 0.0f) f = 0.0f;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

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
  float mean[3] = {0.f, 0.f, 0.f};
  for (int64_t i = first; i < last; i++) {
    const float* p = xyz + 3 * perm[i];
    mean[0] += p[0];
    mean[1] += p[1];
    mean[2] += p[2];
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
    // six sums in one pass; each is still accumulated in index order
    double s00 = 0.0, s01 = 0.0, s02 = 0.0, s11 = 0.0, s12 = 0.0, s22 = 0.0;
    for (int64_t i = 0; i < L; i++) {
      const double x = vh[3 * i], y = vh[3 * i + 1], z = vh[3 * i + 2];
      s00 += x * x;
      s01 += x * y;
      s02 += x * z;
      s11 += y * y;
      s12 += y * z;
      s22 += z * z;
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
    float t = u0 * q[0];
    t = t + u1 * q[1];
    t = t + u2 * q[2];
    return t;
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

// The reference treats a split index of 0 as a leaf (src/Build.cpp:71,160). An
// empty child (coincident points) would make it recurse forever; a leaf here.
inline bool split_ok(int64_t d, int64_t first, int64_t last) {
  return d != 0 && d != first && d != last;
}

}  // namespace

ClusterTree build_tree(const float* xyz, int64_t n, int64_t leaf, int num_threads) {
  ClusterTree t;
  t.perm.resize(n);
  std::iota(t.perm.begin(), t.perm.end(), (int64_t)0);
  // Sequential stage (src/Build.cpp:38-97): one rank => initialLevel 0, the root is divided once.
  TreeNode init[3] = {{0, 0, 0, n, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};
  std::vector<DivideScratch> scratch((size_t)std::max(1, num_threads));
  if (n > leaf) {
    int64_t d = divide(xyz, t.perm.data(), 0, n, num_threads, scratch[0]);
    if (split_ok(d, 0, n)) {
      init[0].child0 = 1;
      init[0].child1 = 2;
      init[1] = {0, 0, 0, d, 1};
      init[2] = {0, 0, d, n, 1};
    }
  }
  // Parallel stage (src/Build.cpp:108-180): the local tree restarts from node 0 and
  // divides it again; children are numbered in BFS order.
  std::vector<TreeNode> local;
  local.push_back(init[0]);
  std::vector<int64_t> frontier{0};
  while (!frontier.empty()) {
    const int64_t m = (int64_t)frontier.size();
    std::vector<int64_t> split(m, 0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(num_threads) if (m > 1)
    for (int64_t i = 0; i < m; i++) {
      const TreeNode nd = local[frontier[i]];
#ifdef _OPENMP
      DivideScratch& sc = scratch[omp_in_parallel() ? omp_get_thread_num() : 0];
#else
      DivideScratch& sc = scratch[0];
#endif
      split[i] = (nd.end - nd.start > leaf) ? divide(xyz, t.perm.data(), nd.start, nd.end, num_threads, sc) : 0;
    }
    std::vector<int64_t> next;
    for (int64_t i = 0; i < m; i++) {
      const int64_t node = frontier[i];
      TreeNode nd = local[node];
      if (!split_ok(split[i], nd.start, nd.end)) {
        local[node].child0 = local[node].child1 = 0;
        continue;
      }
      const int64_t c0 = (int64_t)local.size();
      local.push_back({0, 0, nd.start, split[i], nd.level + 1});
      local.push_back({0, 0, split[i], nd.end, nd.level + 1});
      local[node].child0 = c0;
      local[node].child1 = c0 + 1;
      next.push_back(c0);
      next.push_back(c0 + 1);
    }
    frontier.swap(next);
  }
  const int64_t nloc = (int64_t)local.size() - 1;
  if (nloc == 0) {
    // N <= leaf: the reference points the root at rows 3, 4 of a 3-row tree
    // (src/Build.cpp:239-240); here the root is a single leaf.
    t.nodes.push_back({0, 0, 0, n, 0});
    return t;
  }
  // Merge (src/Build.cpp:199-247): rows 0..2 from the sequential stage, local nodes from row 3
  // with child ids shifted by +2, root re-pointed at rows 3, 4 (rows 1, 2 become orphans).
  t.nodes.resize(nloc + 3);
  for (int i = 0; i < 3; i++) t.nodes[i] = init[i];
  for (int64_t i = 0; i < nloc; i++) {
    TreeNode r = local[i + 1];
    if (r.child0 != 0) {
      r.child0 += 2;
      r.child1 += 2;
    }
    t.nodes[3 + i] = r;
  }
  t.nodes[0].child0 = 3;
  t.nodes[0].child1 = 4;
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
