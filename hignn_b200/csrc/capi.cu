// C ABI of the native library: the model object and the HignnModel operations.
//
// One model = one device + one stream. The tree and lists are built on the
// host (hignn::build_tree / build_lists); everything the matvec touches lives
// in device memory, laid out in tree order:
//   x4   float4[n]   positions (x, y, z, 0)          -- HignnModel::Reorder(map)
//   perm int32[n]    tree position -> caller index    -- mReorderedMap
//   f4   float4[n]   forces, gathered per dot
//   u    double[3n]  velocity accumulator (FP64, src/HignnModel.cpp:555)
// Near-field work is a list of PairWork (one per close leaf pair) consumed by a
// persistent kernel; the far field is cut into ACA batches whose C/Q pools fit
// HIGNN_P_FAR_POOL_MB (allocated once and reused).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../include/hignn_b200.h"
#include "common.h"
#include "kernels.h"
#include "model_view.h"
#include "neighbors.h"
#include "three_body.h"
#include "tree.h"
#include "tree_dev.h"

using hignn::Error;

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& m) { g_last_error = m; }

template <class F>
int guard(F&& f) {
  try {
    f();
    return HIGNN_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return HIGNN_ERR_ARG;
  } catch (const std::exception& e) {
    set_error(e.what());
    return HIGNN_ERR_ARG;
  }
}

using hignn::DevBuf;

// Threads of the host tree build: the cores this process may run on (OpenMP's count, which
// follows the affinity mask and OMP_NUM_THREADS) shared among the ranks of this node
// (LOCAL_WORLD_SIZE, as torchrun sets it), at most 32; HIGNN_HOST_THREADS overrides. The tree
// and the lists do not depend on the thread count.
int host_threads() {
  if (const char* e = std::getenv("HIGNN_HOST_THREADS")) return std::max(1, std::atoi(e));
#ifdef _OPENMP
  int cores = omp_get_max_threads();
#else
  int cores = (int)std::thread::hardware_concurrency();
#endif
  if (cores <= 0) cores = 8;
  int ranks = 1;
  if (const char* w = std::getenv("LOCAL_WORLD_SIZE")) ranks = std::max(1, std::atoi(w));
  return std::max(1, std::min(32, cores / ranks));
}

}  // namespace

struct hignn_model {
  int device = -1;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int64_t n = 0;
  int block_size = 128;
  // reference parameters (src/HignnModel.cpp:337-379)
  double epsilon = 0.05, eta = 1.0, max_far_field_distance = 1000.0;
  int max_iter = 100, mat_pool_size_factor = 40, max_far_dot_work_node_size = 5000;
  int64_t max_relative_coord = 500000;
  bool post_check = false, use_symmetry = true;
  // this implementation
  int precision = 0;
  int64_t far_batch_rows = int64_t(1) << 26;
  int64_t far_pool_bytes = int64_t(24) << 30;  // C + Q pool memory of one ACA batch
  int rank_hint_offset = 0;                      // added to recorded ranks when planning (tests)
  int max_leaf = 0;                              // largest leaf of the close list
  // shard of the block lists this model computes (hignn_set_shard): close pairs [sh_c0, sh_c1),
  // far pairs [sh_f0, sh_f1) of the lists
  int shard_rank = 0, shard_world = 1;
  int64_t sh_c0 = 0, sh_c1 = 0, sh_f0 = 0, sh_f1 = 0;
  bool shard_ready = false;
  int timing = 0;
  hignn::FarTimer far_timer;
  double student_tol = 1e-3;
  int fields = 3;
  bool record_pivots = false;
  std::vector<int32_t> piv_rank, piv_rows, piv_cols;
  int piv_ld = 0;

  std::vector<float> xyz;  // caller order
  hignn::ClusterTree tree;
  hignn::BlockLists lists;
  std::vector<float> xt;   // tree order
  std::vector<int64_t> inv_perm;
  bool tree_ready = false;
  bool lists_sym = true;
  int64_t lists_max_rel = 500000;

  bool has_weights = false;
  std::vector<float> hw;  // device-layout weights, host copy
  bool has_student = false;
  DevBuf student;         // 2537 FP32 parameters of the far-field student network

  DevBuf x4, perm, slot, f4, u, io_f, io_u, close_work, weights, weights_tc, counter;
  DevBuf far_blocks, far_state, far_rows, far_cols, far_used_row, far_used_col, far_C, far_Q, far_xc, far_act,
      far_preI, far_preJ, far_ctr, far_stats, far_rank, far_retry, far_check;
  DevBuf tmp_work, tmp_x, tmp_u, tmp_pos, dp_k, dp_err, near_prof;
  hignn::CellList cells;  // neighbour search of the pair forces
  // CUDA graph of the rank-planned H-matvec (HIGNN_P_GRAPH): captured once per plan and buffer
  // layout, replayed by every later product on the same tree and settings
  bool use_graph = true;
  bool keep_ranks = true;  // HIGNN_P_KEEP_RANKS: ACA ranks carried across tree rebuilds
  cudaGraphExec_t gexec = nullptr;       // near field (after the force gather)
  cudaGraphExec_t gexec_far = nullptr;   // far field (before the velocity scatter)
  uint64_t graph_sig = 0;
  int64_t graph_kernels = 0;
  int graph_iters = 0;
  DevBuf far_status;  // graph form: status[8], then the lists of blocks to rerun
  bool tree_on_device = true;     // HIGNN_P_TREE_DEVICE
  bool tree_built_on_device = false;
  hignn::TreeDevScratch tree_dev;
  hignn_tb* tb = nullptr;  // three-body near field added to the velocity of the device time loops
  int32_t* host_ctr = nullptr;

  // far-field plan: blocks in batch order; iters > 0 when every block's rank is known
  struct Batch {
    int b0, b1, iters;
  };
  std::vector<hignn::FarBlock> far_plan;
  std::vector<Batch> batches;
  bool plan_ready = false;
  bool plan_hinted = false;
  int plan_max_iter = -1;
  int64_t plan_rows = -1, plan_pool = -1;
  int plan_offset = 0;
  // ACA ranks of the last far field (far-list order), valid for the same tree and settings
  std::vector<int32_t> rank_hint;
  bool hint_valid = false;
  int hint_precision = -1, hint_max_iter = -1;
  double hint_epsilon = -1.0;

  hignn_stats stats{};
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t lev[4] = {nullptr, nullptr, nullptr, nullptr};  // phases of the device time loops
  // phases of the last time loop (hignn_loop_profile): wall, rebuild, forces, matvec, three-body,
  // steps, velocity evaluations, matvecs that ran eagerly (no complete rank plan)
  double loop_prof[8] = {0, 0, 0, 0, 0, 0, 0, 0};

  hignn::MlpF32 wdev() const {
    hignn::MlpF32 w;
    const float* base = weights.as<float>();
    w.w1b1 = reinterpret_cast<const float4*>(base);
    w.w2t = base + 4 * hignn::kH1;
    w.b2 = w.w2t + hignn::kH1 * hignn::kH2;
    w.w3 = w.b2 + hignn::kH2;
    w.b3 = w.w3 + hignn::kOut * hignn::kH2;
    return w;
  }
  hignn::TcWeights wtc() const {
    const hignn::MlpF32 f = wdev();
    hignn::TcWeights w;
    w.w2img = weights_tc.as<uint4>();
    w.w3img = reinterpret_cast<const uint4*>(weights_tc.as<uint8_t>() + hignn::kH2 * hignn::kH1 * 2);
    w.w1b1 = f.w1b1;
    w.b2 = f.b2;
    w.b3 = f.b3;
    return w;
  }
  int* err_flag() const { return counter.as<int>() + 1; }
};

namespace {

void require_device(hignn_model* m) {
  if (m->device < 0) throw Error(HIGNN_ERR_NODEV, "model was created without a CUDA device (host-only)");
  HIGNN_CUDA(cudaSetDevice(m->device));
}

// Builds the tree and lists of m->xyz and, on a device model, uploads the tree-order positions
// and the close work list. Everything is built and checked before the model changes: a tree that
// the device kernels cannot take (a leaf above kMaxLeaf particles, which coincident points can
// give whatever the block size) leaves the model without a tree (tree_ready false), so that no
// later call runs on lists that do not belong to the uploaded positions.
void build_structures(hignn_model* m) {
  const auto t0 = std::chrono::steady_clock::now();
  // ACA ranks of the previous far field, keyed by the two nodes of each block (ids and particle
  // ranges): a block of the new lists that joins the same two nodes starts from that rank
  struct Carried {
    int64_t sI, eI, sJ, eJ;
    int32_t rank;
  };
  std::unordered_map<uint64_t, Carried> carried;
  const bool carry = m->keep_ranks && m->hint_valid && m->rank_hint.size() == m->lists.farI.size() && m->tree_ready;
  if (carry)
    for (size_t q = 0; q < m->lists.farI.size(); q++) {
      const auto& I = m->tree.nodes[m->lists.farI[q]];
      const auto& J = m->tree.nodes[m->lists.farJ[q]];
      carried[((uint64_t)m->lists.farI[q] << 32) | (uint64_t)m->lists.farJ[q]] =
          Carried{I.start, I.end, J.start, J.end, m->rank_hint[q]};
    }
  m->tree_ready = false;
  m->plan_ready = false;
  m->hint_valid = false;
  m->shard_ready = false;
  const bool on_dev = m->device >= 0 && m->tree_on_device;
  hignn::ClusterTree tree;
  if (on_dev) {
    HIGNN_CUDA(cudaSetDevice(m->device));
    m->tree_dev.xyz.ensure(sizeof(float) * 3 * m->n);
    HIGNN_CUDA(cudaMemcpyAsync(m->tree_dev.xyz.p, m->xyz.data(), sizeof(float) * 3 * m->n, cudaMemcpyHostToDevice,
                               m->stream));
    tree = hignn::build_tree_device(m->tree_dev.xyz.as<float>(), m->n, m->block_size, m->tree_dev, m->stream);
  } else {
    tree = hignn::build_tree(m->xyz.data(), m->n, m->block_size, host_threads());
  }
  m->tree_built_on_device = on_dev;
  std::vector<float> xt(3 * m->n);
  std::vector<int64_t> inv_perm(m->n);
  for (int64_t i = 0; i < m->n; i++) {
    const int64_t p = tree.perm[i];
    xt[3 * i] = m->xyz[3 * p];
    xt[3 * i + 1] = m->xyz[3 * p + 1];
    xt[3 * i + 2] = m->xyz[3 * p + 2];
    inv_perm[p] = i;
  }
  hignn::BlockLists lists;
  if (!on_dev || !hignn::build_lists_device(tree, m->tree_dev.xt.as<float4>(), m->max_relative_coord,
                                            m->use_symmetry, m->tree_dev, m->stream, lists))
    lists = hignn::build_lists(tree, xt.data(), m->max_relative_coord, m->use_symmetry, host_threads());
  if (m->device >= 0)
    for (int64_t L : lists.leaves) {
      const int64_t sz = tree.nodes[L].end - tree.nodes[L].start;
      if (sz > hignn::kMaxLeaf)
        throw Error(HIGNN_ERR_ARG, "leaf of " + std::to_string(sz) + " particles (more than " +
                                       std::to_string(hignn::kMaxLeaf) +
                                       "; coincident points or block_size > " + std::to_string(hignn::kMaxLeaf) +
                                       "): the device kernels stage at most " + std::to_string(hignn::kMaxLeaf) +
                                       " particles per leaf");
    }
  m->tree = std::move(tree);
  m->xt = std::move(xt);
  m->inv_perm = std::move(inv_perm);
  m->lists = std::move(lists);
  m->lists_sym = m->use_symmetry;
  m->lists_max_rel = m->max_relative_coord;
  if (carry) {  // hints for the new lists; -1 = not known (planned at full capacity)
    m->rank_hint.assign(m->lists.farI.size(), -1);
    for (size_t q = 0; q < m->lists.farI.size(); q++) {
      const auto it = carried.find(((uint64_t)m->lists.farI[q] << 32) | (uint64_t)m->lists.farJ[q]);
      if (it == carried.end()) continue;
      const auto& I = m->tree.nodes[m->lists.farI[q]];
      const auto& J = m->tree.nodes[m->lists.farJ[q]];
      const Carried& c = it->second;
      if (c.sI == I.start && c.eI == I.end && c.sJ == J.start && c.eJ == J.end) m->rank_hint[q] = c.rank;
    }
    m->hint_valid = true;
  }
  const auto t1 = std::chrono::steady_clock::now();
  m->stats.t_build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  m->stats.n = m->n;
  m->stats.num_nodes = (int64_t)m->tree.nodes.size();
  m->stats.num_leaves = (int64_t)m->lists.leaves.size();
  m->stats.num_close = (int64_t)m->lists.closeI.size();
  m->stats.num_far = (int64_t)m->lists.farI.size();
  if (m->device < 0) {
    m->tree_ready = true;
    return;
  }
  // device copies
  HIGNN_CUDA(cudaSetDevice(m->device));
  const int64_t n = m->n;
  std::vector<float4> x4(n);
  std::vector<int32_t> perm(n), slot(n);
  for (int64_t i = 0; i < n; i++) {
    x4[i] = make_float4(m->xt[3 * i], m->xt[3 * i + 1], m->xt[3 * i + 2], 0.f);
    perm[i] = (int32_t)m->tree.perm[i];
    slot[i] = (int32_t)m->inv_perm[i];
  }
  // close work list (src/CloseFarCheck.cpp:298-336 order)
  std::vector<hignn::PairWork> work(m->lists.closeI.size());
  int64_t evals = 0;
  for (size_t q = 0; q < work.size(); q++) {
    const auto& I = m->tree.nodes[m->lists.closeI[q]];
    const auto& J = m->tree.nodes[m->lists.closeJ[q]];
    hignn::PairWork w{};
    w.sI = (int32_t)I.start;
    w.nI = (int32_t)(I.end - I.start);
    w.sJ = (int32_t)J.start;
    w.nJ = (int32_t)(J.end - J.start);
    w.flags = (m->use_symmetry && m->lists.closeJ[q] > m->lists.closeI[q]) ? hignn::kPairTransposed : 0;
    evals += (int64_t)w.nI * w.nJ;
    work[q] = w;
  }
  m->stats.close_evals = evals;
  m->max_leaf = 0;
  for (const auto& w : work) m->max_leaf = std::max(m->max_leaf, std::max(w.nI, w.nJ));
  m->x4.ensure(sizeof(float4) * n);
  m->perm.ensure(sizeof(int32_t) * n);
  m->slot.ensure(sizeof(int32_t) * n);
  m->f4.ensure(sizeof(float4) * n);
  m->u.ensure(sizeof(double) * 3 * n);
  m->io_f.ensure(sizeof(float) * 3 * n);
  m->io_u.ensure(sizeof(float) * 3 * n);
  m->close_work.ensure(sizeof(hignn::PairWork) * std::max<size_t>(1, work.size()));
  m->counter.ensure(64);
  HIGNN_CUDA(cudaMemcpyAsync(m->slot.p, slot.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, m->stream));
  if (on_dev) {  // tree-order positions and the permutation are already on the device
    HIGNN_CUDA(cudaMemcpyAsync(m->x4.p, m->tree_dev.xt.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, m->stream));
    HIGNN_CUDA(cudaMemcpyAsync(m->perm.p, m->tree_dev.perm.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice,
                               m->stream));
  } else {
    HIGNN_CUDA(cudaMemcpyAsync(m->x4.p, x4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, m->stream));
    HIGNN_CUDA(cudaMemcpyAsync(m->perm.p, perm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, m->stream));
  }
  if (!work.empty())
    HIGNN_CUDA(cudaMemcpyAsync(m->close_work.p, work.data(), sizeof(hignn::PairWork) * work.size(),
                               cudaMemcpyHostToDevice, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  m->tree_ready = true;
}

void ensure_tree(hignn_model* m) {
  if (!m->tree_ready || m->lists_sym != m->use_symmetry || m->lists_max_rel != m->max_relative_coord)
    build_structures(m);
}

// Contiguous range of `cost` owned by `rank` of `world` with about equal cost per rank.
void balanced_range(const std::vector<double>& cost, int rank, int world, int64_t* lo, int64_t* hi) {
  const size_t n = cost.size();
  std::vector<double> pre(n + 1, 0.0);
  for (size_t q = 0; q < n; q++) pre[q + 1] = pre[q] + cost[q];
  auto cut = [&](int r) -> int64_t {
    if (r <= 0) return 0;
    if (r >= world) return (int64_t)n;
    const double target = pre[n] * r / world;
    return (int64_t)(std::lower_bound(pre.begin(), pre.end(), target) - pre.begin());
  };
  *lo = std::min<int64_t>(cut(rank), (int64_t)n);
  *hi = std::max(*lo, std::min<int64_t>(cut(rank + 1), (int64_t)n));
}

// The shard of this model: close pairs balanced by |I||J| evaluations, far pairs by
// (|I| + |J|) min(kmax, 32) (query rows times a typical rank), contiguous in list order as the
// reference's ranks take interleaved shares of the same lists (src/CloseFarCheck.cpp:309,394).
void ensure_shard(hignn_model* m) {
  if (m->shard_ready) return;
  std::vector<double> cc(m->lists.closeI.size()), fc(m->lists.farI.size());
  for (size_t q = 0; q < cc.size(); q++) {
    const auto& I = m->tree.nodes[m->lists.closeI[q]];
    const auto& J = m->tree.nodes[m->lists.closeJ[q]];
    cc[q] = (double)(I.end - I.start) * (double)(J.end - J.start);
  }
  for (size_t q = 0; q < fc.size(); q++) {
    const auto& I = m->tree.nodes[m->lists.farI[q]];
    const auto& J = m->tree.nodes[m->lists.farJ[q]];
    const int64_t nI = I.end - I.start, nJ = J.end - J.start;
    fc[q] = (double)(nI + nJ) * (double)std::min<int64_t>(std::min<int64_t>(m->max_iter, std::min(nI, nJ)), 32);
  }
  balanced_range(cc, m->shard_rank, m->shard_world, &m->sh_c0, &m->sh_c1);
  balanced_range(fc, m->shard_rank, m->shard_world, &m->sh_f0, &m->sh_f1);
  int64_t evals = 0;
  for (int64_t q = m->sh_c0; q < m->sh_c1; q++) evals += (int64_t)cc[q];
  m->stats.close_evals = evals;
  m->shard_ready = true;
}

bool hints_usable(const hignn_model* m) {
  return m->hint_valid && m->hint_precision == m->precision && m->hint_epsilon == m->epsilon &&
         m->hint_max_iter == m->max_iter && m->rank_hint.size() == m->lists.farI.size();
}

// Lays out far blocks `idx` (far-list positions) with pool capacities `kcap` into ACA batches:
// a batch is cut when its C + Q pools (9 doubles per particle and term) would exceed
// far_pool_bytes or its rows (sum of |I| + |J|) far_batch_rows. Grows the device buffers to
// the largest batch. Returns the blocks in batch order.
std::vector<hignn::FarBlock> layout_batches(hignn_model* m, const std::vector<int>& idx, const std::vector<int>& kcap,
                                            bool known, std::vector<hignn_model::Batch>& batches) {
  std::vector<hignn::FarBlock> out(idx.size());
  batches.clear();
  int64_t rows = 0, cE = 0, qE = 0, xE = 0, maxC = 0, maxQ = 0, maxX = 0;
  int32_t rOff = 0, colOff = 0, maxR = 0, maxCol = 0;
  int b0 = 0, maxNb = 0, iters = 0;
  for (size_t p = 0; p < idx.size(); p++) {
    const int q = idx[p];
    const auto& I = m->tree.nodes[m->lists.farI[q]];
    const auto& J = m->tree.nodes[m->lists.farJ[q]];
    const int32_t nI = (int32_t)(I.end - I.start), nJ = (int32_t)(J.end - J.start);
    const int cnt = (int)p - b0;
    const int64_t add = (int64_t)kcap[p] * (nI + nJ) * 9 * (int64_t)sizeof(hignn::pool_t);
    if (cnt > 0 && ((cE + qE) * 9 * (int64_t)sizeof(hignn::pool_t) + add > m->far_pool_bytes ||
                    rows + nI + nJ > m->far_batch_rows)) {
      batches.push_back({b0, (int)p, known ? iters : 0});
      maxNb = std::max(maxNb, cnt);
      b0 = (int)p;
      rows = cE = qE = xE = 0;
      rOff = colOff = 0;
      iters = 0;
    }
    hignn::FarBlock fb{};
    fb.sI = (int32_t)I.start;
    fb.nI = nI;
    fb.sJ = (int32_t)J.start;
    fb.nJ = nJ;
    fb.kcap = kcap[p];
    fb.list_idx = q;
    fb.cOff = cE;
    fb.qOff = qE;
    fb.xOff = xE;
    fb.rOff = rOff;
    fb.colOff = colOff;
    cE += (int64_t)fb.kcap * nI;
    qE += (int64_t)fb.kcap * nJ;
    xE += hignn::kXcHead + 9 * (int64_t)fb.kcap;
    rOff += nI;
    colOff += nJ;
    rows += nI + nJ;
    iters = std::max(iters, fb.kcap);
    maxC = std::max(maxC, cE);
    maxQ = std::max(maxQ, qE);
    maxX = std::max(maxX, xE);
    maxR = std::max(maxR, rOff);
    maxCol = std::max(maxCol, colOff);
    out[p] = fb;
  }
  if (!idx.empty()) {
    batches.push_back({b0, (int)idx.size(), known ? iters : 0});
    maxNb = std::max(maxNb, (int)idx.size() - b0);
  }
  if (m->device >= 0 && !idx.empty()) {
    const int ldr = m->max_iter + 1;
    m->far_state.ensure(sizeof(hignn::FarState) * maxNb);
    m->far_rows.ensure(sizeof(int32_t) * (size_t)maxNb * ldr);
    m->far_cols.ensure(sizeof(int32_t) * (size_t)maxNb * ldr);
    m->far_used_row.ensure((size_t)maxR + 16);
    m->far_used_col.ensure((size_t)maxCol + 16);
    m->far_C.ensure(sizeof(hignn::pool_t) * 9 * (size_t)maxC);
    m->far_Q.ensure(sizeof(hignn::pool_t) * 9 * (size_t)maxQ);
    m->far_xc.ensure(sizeof(float) * (size_t)maxX);
    m->far_act.ensure(sizeof(int32_t) * (maxNb + 1));
    m->far_preI.ensure(sizeof(int32_t) * (maxNb + 1));
    m->far_preJ.ensure(sizeof(int32_t) * (maxNb + 1));
    m->far_ctr.ensure(sizeof(int32_t) * hignn::kCtrCount);
    m->far_stats.ensure(sizeof(unsigned long long) * 4);
    m->far_rank.ensure(sizeof(int32_t) * std::max<size_t>(1, m->lists.farI.size()));
  }
  return out;
}

// ACA plan of the far list. Without rank information every block gets the pool capacity
// min(max_iter, |I|, |J|, kFirstPlanCap) and the batches follow the list order
// (src/FarDot.cpp:191-340 batches the list in order); a block that needs more terms is deferred
// and rerun with min(max_iter, |I|, |J|), so the cap only decides how many blocks share a batch. When the previous far field on the same tree and settings
// recorded every block's rank, each block gets exactly that capacity, the blocks are sorted by
// rank (batches of similar ranks need fewer iterations) and each batch runs its known
// iteration count without reading counters back; a block that would need more terms than
// recorded is deferred and rerun with the full capacity, so the result never depends on the
// hint.
// Pool capacity of a block without a recorded rank: about twice the largest rank of the
// benchmark's far blocks at epsilon 1e-2 (14-18), so that the first far field on a tree packs up to
// three times more blocks per batch than at the full capacity of max_iter = 100 terms.
constexpr int kFirstPlanCap = 32;

void ensure_far_plan(hignn_model* m) {
  ensure_shard(m);
  const bool use_hints = hints_usable(m);
  if (m->plan_ready && m->plan_hinted == use_hints && m->plan_max_iter == m->max_iter &&
      m->plan_rows == m->far_batch_rows && m->plan_pool == m->far_pool_bytes &&
      m->plan_offset == m->rank_hint_offset)
    return;
  const size_t nf = (size_t)(m->sh_f1 - m->sh_f0);
  std::vector<int> idx(nf), kcap(nf);
  std::vector<int> full(m->lists.farI.size());
  for (size_t p = 0; p < nf; p++) {
    const size_t q = (size_t)m->sh_f0 + p;
    const auto& I = m->tree.nodes[m->lists.farI[q]];
    const auto& J = m->tree.nodes[m->lists.farJ[q]];
    const int nI = (int)(I.end - I.start), nJ = (int)(J.end - J.start);
    full[q] = std::max(1, std::min(m->max_iter, std::min(nI, nJ)));
    idx[p] = (int)q;
  }
  if (use_hints) {  // a block whose rank is not known (hint < 0) gets the full capacity
    std::vector<int> kc(m->lists.farI.size());
    for (int q : idx)
      kc[q] = m->rank_hint[q] < 0 ? full[q] : std::max(1, std::min(full[q], m->rank_hint[q] + m->rank_hint_offset));
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return kc[x] > kc[y]; });
    for (size_t p = 0; p < nf; p++) kcap[p] = kc[idx[p]];
  } else {
    for (size_t p = 0; p < nf; p++) kcap[p] = std::min(full[idx[p]], kFirstPlanCap);
  }
  m->far_plan = layout_batches(m, idx, kcap, use_hints, m->batches);
  if (m->device >= 0 && nf > 0) {
    m->far_blocks.ensure(sizeof(hignn::FarBlock) * nf);
    HIGNN_CUDA(cudaMemcpyAsync(m->far_blocks.p, m->far_plan.data(), sizeof(hignn::FarBlock) * nf,
                               cudaMemcpyHostToDevice, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  }
  m->plan_ready = true;
  m->plan_hinted = use_hints;
  m->plan_max_iter = m->max_iter;
  m->plan_rows = m->far_batch_rows;
  m->plan_pool = m->far_pool_bytes;
  m->plan_offset = m->rank_hint_offset;
}

// IEEE binary16, round to nearest even (subnormals kept, overflow to infinity)
uint16_t f16_bits(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
  const uint32_t ax = x & 0x7fffffffu;
  if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u);  // NaN
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds above 65504: infinity
  if (ax < 0x38800000u) {                                     // below 2^-14: subnormal or zero
    if (ax < 0x33000000u) return sign;                        // below half the smallest subnormal
    const uint32_t e = ax >> 23, m = (ax & 0x7fffffu) | 0x800000u;
    const uint32_t shift = 126 - e;                           // 14..24: value = m * 2^(e-150)
    uint32_t q = m >> shift;
    const uint32_t rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
    if (rem > half || (rem == half && (q & 1u))) q++;
    return (uint16_t)(sign | q);
  }
  uint32_t r = ax - 0x38000000u;  // rebias the exponent (127 -> 15)
  const uint32_t rem = r & 0x1fffu;
  r >>= 13;
  if (rem > 0x1000u || (rem == 0x1000u && (r & 1u))) r++;
  return (uint16_t)(sign | r);
}

void check_device_error(hignn_model* m) {
  int e = 0;
  HIGNN_CUDA(cudaMemcpyAsync(&e, m->err_flag(), sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  if (e != 0) {
    HIGNN_CUDA(cudaMemsetAsync(m->err_flag(), 0, sizeof(int), m->stream));
    throw Error(HIGNN_ERR_LIMIT, "tensor-core kernel: a bounded wait timed out (code " + std::to_string(e) + ")");
  }
}

void require_student_if_needed(hignn_model* m) {
  if (m->precision == 2 && !m->has_student)
    throw Error(HIGNN_ERR_STATE, "precision 2 needs a student network (hignn_train_student or hignn_set_student)");
}

void require_weights(hignn_model* m) {
  if (!m->has_weights) throw Error(HIGNN_ERR_STATE, "no two-body model loaded (call load_two_body_model)");
}

void upload_weights(hignn_model* m, const std::vector<std::vector<float>>& W, const std::vector<std::vector<float>>& B,
                    const std::vector<int>& dims) {
  using namespace hignn;
  if (dims.size() != 4 || dims[0] != 3 || dims[1] != kH1 || dims[2] != kH2 || dims[3] != kOut)
    throw Error(HIGNN_ERR_ARG, "two-body network must be 3 -> 128 -> 512 -> 9 (tanh)");
  std::vector<float>& hw = m->hw;
  hw.assign(4 * kH1 + kH1 * kH2 + kH2 + kOut * kH2 + 16, 0.f);
  for (int k = 0; k < kH1; k++) {
    hw[4 * k] = W[0][3 * k];
    hw[4 * k + 1] = W[0][3 * k + 1];
    hw[4 * k + 2] = W[0][3 * k + 2];
    hw[4 * k + 3] = B[0][k];
  }
  float* w2t = hw.data() + 4 * kH1;
  for (int nn = 0; nn < kH2; nn++)
    for (int k = 0; k < kH1; k++) w2t[(size_t)k * kH2 + nn] = W[1][(size_t)nn * kH1 + k];
  float* b2 = w2t + kH1 * kH2;
  for (int nn = 0; nn < kH2; nn++) b2[nn] = B[1][nn];
  float* w3 = b2 + kH2;
  for (int q = 0; q < kOut * kH2; q++) w3[q] = W[2][q];
  float* b3 = w3 + kOut * kH2;
  for (int q = 0; q < kOut; q++) b3[q] = B[2][q];
  // tensor-core images: K-major rows of 64 FP16 (128 B) per 64-wide K slab, 8-row groups of
  // 1024 B, 16-byte chunk c of row r stored at chunk position c ^ (r % 8) (128-byte swizzle)
  auto swz = [](int row, int k, int rows_per_slab) -> size_t {
    const int slab = k >> 6, kc = k & 63;
    return (size_t)slab * rows_per_slab * 128 + (size_t)(row >> 3) * 1024 + (row & 7) * 128 +
           (size_t)(((kc >> 3) ^ (row & 7)) * 16) + (kc & 7) * 2;
  };
  // W2 (512 x 128) and W3 (rows 0-8 of 16 x 512) in FP16; layer 1 stays FP32 (MlpF32::w1b1)
  const size_t w3off = (size_t)kH2 * kH1 * 2;
  std::vector<uint8_t> img(w3off + (size_t)16 * kH2 * 2, 0);
  auto put = [&](size_t off, uint16_t v) { std::memcpy(img.data() + off, &v, 2); };
  for (int nn = 0; nn < kH2; nn++)
    for (int k = 0; k < kH1; k++) put(swz(nn, k, kH2), f16_bits(W[1][(size_t)nn * kH1 + k]));
  for (int o = 0; o < kOut; o++)
    for (int k = 0; k < kH2; k++) put(w3off + swz(o, k, 16), f16_bits(W[2][(size_t)o * kH2 + k]));
  m->has_weights = true;
  m->hint_valid = false;  // ACA ranks depend on the network
  if (m->device < 0) return;
  HIGNN_CUDA(cudaSetDevice(m->device));
  m->weights.ensure(sizeof(float) * hw.size());
  HIGNN_CUDA(cudaMemcpyAsync(m->weights.p, hw.data(), sizeof(float) * hw.size(), cudaMemcpyHostToDevice, m->stream));
  m->weights_tc.ensure(img.size());
  HIGNN_CUDA(cudaMemcpyAsync(m->weights_tc.p, img.data(), img.size(), cudaMemcpyHostToDevice, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
}

struct FarOutcome {
  std::vector<int> deferred;  // far-list positions that outgrew their pool capacity
  std::vector<int> fallback;  // far-list positions the student check sent to the teacher
};

// Runs the ACA batches of `plan` (device copy at d_blocks). student_pass: queries by the
// student network, each converged block applied only after its sampled residual against the
// teacher passed (student_tol); otherwise queries by the teacher (tensor cores from precision 1
// on, FP32 SIMT at precision 0).
// Kernel arguments of ACA batch bt (device block table at d_blocks).
hignn::FarArgs far_args(hignn_model* m, const hignn_model::Batch& bt, const hignn::FarBlock* d_blocks,
                      bool student_pass) {
  hignn::FarArgs a{};
  a.blocks = d_blocks + bt.b0;
  a.nb = bt.b1 - bt.b0;
  a.state = m->far_state.as<hignn::FarState>();
  a.rows = m->far_rows.as<int32_t>();
  a.cols = m->far_cols.as<int32_t>();
  a.ldr = m->max_iter + 1;
  a.usedRow = m->far_used_row.as<uint8_t>();
  a.usedCol = m->far_used_col.as<uint8_t>();
  a.C = m->far_C.as<hignn::pool_t>();
  a.Q = m->far_Q.as<hignn::pool_t>();
  a.xc = m->far_xc.as<float>();
  a.act = m->far_act.as<int32_t>();
  a.preI = m->far_preI.as<int32_t>();
  a.preJ = m->far_preJ.as<int32_t>();
  a.ctr = m->far_ctr.as<int32_t>();
  a.rank_sum = m->far_stats.as<unsigned long long>();
  a.evals = m->far_stats.as<unsigned long long>() + 1;
  a.rank_out = m->far_rank.as<int32_t>();
  a.x = m->x4.as<float4>();
  a.f = m->f4.as<float4>();
  a.u = m->u.as<double>();
  a.max_iter = m->max_iter;
  a.eps2 = m->epsilon * m->epsilon;
  a.use_symmetry = m->use_symmetry ? 1 : 0;
  a.defer_apply = student_pass ? 1 : 0;
  a.fast_pivots = m->precision >= 1 ? 1 : 0;
  return a;
}

FarOutcome run_far_batches(hignn_model* m, const std::vector<hignn::FarBlock>& plan,
                           const std::vector<hignn_model::Batch>& batches, const hignn::FarBlock* d_blocks,
                           bool student_pass, int* iterations) {
  const hignn::MlpF32 w = m->wdev();
  const hignn::TcWeights tcw = m->wtc();
  const float* student = student_pass ? m->student.as<float>() : nullptr;
  FarOutcome out;
  std::vector<int>& deferred = out.deferred;
  for (const auto& bt : batches) {
    const hignn::FarArgs a = far_args(m, bt, d_blocks, student_pass);
    const auto& last = plan[bt.b1 - 1];
    HIGNN_CUDA(cudaMemsetAsync(m->far_used_row.p, 0, (size_t)last.rOff + last.nI, m->stream));
    HIGNN_CUDA(cudaMemsetAsync(m->far_used_col.p, 0, (size_t)last.colOff + last.nJ, m->stream));
    hignn::FarTimer* tm = m->timing >= 2 ? &m->far_timer : nullptr;
    const int nd = hignn::far_batch_plain(a, w, m->precision >= 1 ? &tcw : nullptr, student, m->err_flag(),
                                          m->num_sms, m->host_ctr, m->stream, bt.iters, iterations, tm);
    m->stats.far_rank_max = std::max(m->stats.far_rank_max, m->host_ctr[hignn::kCtrRankMax]);
    m->stats.gpu_launches += 1;
    const int nb = bt.b1 - bt.b0, ld = a.ldr;
    int nfail = 0;
    if (student_pass) {
      const size_t ns = (size_t)nb * hignn::kFarSamples;
      m->far_check.ensure(sizeof(float) * ns * 21 + 64);
      float* feat = m->far_check.as<float>();
      // The student cannot represent the teacher's fine texture (its residual from the RPY tensor has
      // ~3e-3 relative amplitude and a correlation length of 1-2 radii at every distance), so a
      // block is sent back to the teacher when the student's sampled error exceeds the accuracy
      // the ACA block is held to anyway: the larger of student_tol and epsilon.
      const float tol = (float)std::max(m->student_tol, m->epsilon);
      if (tm) HIGNN_CUDA(cudaEventRecord(m->ev[3], m->stream));
      nfail = hignn::far_student_check(a, tcw, student, tol, feat, feat + 3 * ns, feat + 12 * ns,
                                       reinterpret_cast<int*>(feat + 21 * ns), m->err_flag(), m->num_sms, m->stream);
      if (tm) {  // far_student_check synchronised the stream
        HIGNN_CUDA(cudaEventRecord(m->ev[2], m->stream));
        HIGNN_CUDA(cudaEventSynchronize(m->ev[2]));
        float ms = 0;
        HIGNN_CUDA(cudaEventElapsedTime(&ms, m->ev[3], m->ev[2]));
        m->stats.t_far_check_ms += ms;
      }
      m->stats.student_fallback_blocks += nfail;
      m->stats.gpu_launches += 5;
    }
    std::vector<hignn::FarState> st;
    if (nd > 0 || nfail > 0 || m->record_pivots) {
      st.resize(nb);
      HIGNN_CUDA(cudaMemcpyAsync(st.data(), a.state, sizeof(hignn::FarState) * nb, cudaMemcpyDeviceToHost, m->stream));
      HIGNN_CUDA(cudaStreamSynchronize(m->stream));
      for (int q = 0; q < nb; q++) {
        if (st[q].done == 2) deferred.push_back(plan[bt.b0 + q].list_idx);
        if (st[q].done == 3) out.fallback.push_back(plan[bt.b0 + q].list_idx);
      }
    }
    if (m->record_pivots) {
      std::vector<int32_t> rows((size_t)nb * ld), cols((size_t)nb * ld);
      HIGNN_CUDA(cudaMemcpyAsync(rows.data(), a.rows, sizeof(int32_t) * nb * ld, cudaMemcpyDeviceToHost, m->stream));
      HIGNN_CUDA(cudaMemcpyAsync(cols.data(), a.cols, sizeof(int32_t) * nb * ld, cudaMemcpyDeviceToHost, m->stream));
      HIGNN_CUDA(cudaStreamSynchronize(m->stream));
      for (int q = 0; q < nb; q++) {
        if (st[q].done != 1) continue;
        const int li = plan[bt.b0 + q].list_idx;
        m->piv_rank[li] = st[q].k;
        std::copy(rows.begin() + (size_t)q * ld, rows.begin() + (size_t)(q + 1) * ld,
                  m->piv_rows.begin() + (size_t)li * ld);
        std::copy(cols.begin() + (size_t)q * ld, cols.begin() + (size_t)(q + 1) * ld,
                  m->piv_cols.begin() + (size_t)li * ld);
      }
    }
  }
  return out;
}

// Full-capacity plan of the given far-list positions (deferred blocks, student fallbacks).
void run_far_subset(hignn_model* m, const std::vector<int>& subset, bool student_pass, int* iterations,
                    FarOutcome* out) {
  std::vector<int> kcap(subset.size());
  for (size_t p = 0; p < subset.size(); p++) {
    const auto& I = m->tree.nodes[m->lists.farI[subset[p]]];
    const auto& J = m->tree.nodes[m->lists.farJ[subset[p]]];
    kcap[p] = std::max(1, std::min(m->max_iter, (int)std::min(I.end - I.start, J.end - J.start)));
  }
  std::vector<hignn_model::Batch> rb;
  const std::vector<hignn::FarBlock> rplan = layout_batches(m, subset, kcap, false, rb);
  m->far_retry.ensure(sizeof(hignn::FarBlock) * rplan.size());
  HIGNN_CUDA(cudaMemcpyAsync(m->far_retry.p, rplan.data(), sizeof(hignn::FarBlock) * rplan.size(),
                             cudaMemcpyHostToDevice, m->stream));
  *out = run_far_batches(m, rplan, rb, m->far_retry.as<hignn::FarBlock>(), student_pass, iterations);
}

void far_field(hignn_model* m) {
  ensure_far_plan(m);
  m->stats.far_evals = 0;
  m->stats.far_rank_sum = 0;
  m->stats.far_rank_max = 0;
  m->stats.far_iterations = 0;
  if (m->batches.empty()) return;
  const size_t nf = m->lists.farI.size();  // pivots and ranks are kept in far-list order
  if (m->record_pivots) {
    m->piv_ld = m->max_iter + 1;
    m->piv_rank.assign(nf, 0);
    m->piv_rows.assign(nf * (size_t)m->piv_ld, -1);
    m->piv_cols.assign(nf * (size_t)m->piv_ld, -1);
  }
  HIGNN_CUDA(cudaMemsetAsync(m->far_stats.p, 0, sizeof(unsigned long long) * 4, m->stream));
  m->stats.student_fallback_blocks = 0;
  m->stats.t_far_query_ms = m->stats.t_far_pivot_ms = m->stats.t_far_active_ms = m->stats.t_far_check_ms = 0;
  m->far_timer.active_ms = m->far_timer.query_ms = m->far_timer.pivot_ms = 0;
  int iterations = 0;
  const bool student_pass = m->precision == 2 && m->has_student;
  FarOutcome res =
      run_far_batches(m, m->far_plan, m->batches, m->far_blocks.as<hignn::FarBlock>(), student_pass, &iterations);
  const bool had_deferred = !res.deferred.empty();
  std::vector<int> fallback = res.fallback;
  if (had_deferred) {  // blocks that outgrew their recorded rank: rerun with the full capacity
    FarOutcome r2;
    run_far_subset(m, res.deferred, student_pass, &iterations, &r2);
    if (!r2.deferred.empty()) throw Error(HIGNN_ERR_LIMIT, "ACA: a block was deferred at its full capacity");
    fallback.insert(fallback.end(), r2.fallback.begin(), r2.fallback.end());
  }
  if (!fallback.empty()) {  // student residual above tolerance: the teacher network for these blocks
    FarOutcome r3;
    run_far_subset(m, fallback, false, &iterations, &r3);
    if (!r3.deferred.empty()) throw Error(HIGNN_ERR_LIMIT, "ACA: a block was deferred at its full capacity");
  }
  unsigned long long st[2];
  HIGNN_CUDA(cudaMemcpyAsync(st, m->far_stats.p, sizeof(st), cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  m->stats.far_rank_sum = (int64_t)st[0];
  m->stats.far_evals = (int64_t)st[1];
  m->stats.far_iterations = iterations;
  m->stats.t_far_query_ms = m->far_timer.query_ms;
  m->stats.t_far_pivot_ms = m->far_timer.pivot_ms;
  m->stats.t_far_active_ms = m->far_timer.active_ms;
  // per ACA iteration: active list, column eval, column pivot, row eval, row pivot
  m->stats.gpu_launches += 5 * (int64_t)iterations;
  if (!m->plan_hinted || had_deferred) {  // record the ranks for the next far field on this tree
    m->rank_hint.resize(nf);
    HIGNN_CUDA(cudaMemcpyAsync(m->rank_hint.data(), m->far_rank.p, sizeof(int32_t) * nf, cudaMemcpyDeviceToHost,
                               m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    m->hint_valid = true;
    m->hint_precision = m->precision;
    m->hint_epsilon = m->epsilon;
    m->hint_max_iter = m->max_iter;
  }
}

void near_field(hignn_model* m) {
  hignn::NearArgs a{};
  ensure_shard(m);
  a.work = m->close_work.as<hignn::PairWork>() + m->sh_c0;
  a.nwork = (int)(m->sh_c1 - m->sh_c0);
  a.xI = a.xJ = m->x4.as<float4>();
  a.fI = a.fJ = m->f4.as<float4>();
  a.uI = a.uJ = m->u.as<double>();
  if (m->precision >= 1) {
    if (m->max_leaf > hignn::kTcMaxLeaf)
      throw Error(HIGNN_ERR_ARG, "the tensor-core forms (precision 1, 2) need leaves of at most " +
                                     std::to_string(hignn::kTcMaxLeaf) + " particles (block_size <= " +
                                     std::to_string(hignn::kTcMaxLeaf) + ")");
    hignn::TcWeights tw = m->wtc();
    if (m->timing >= 3) {  // wait profile of the engine, accumulated until hignn_near_wait_profile
      if (!m->near_prof.p) {
        m->near_prof.ensure(sizeof(unsigned long long) * 16);
        HIGNN_CUDA(cudaMemsetAsync(m->near_prof.p, 0, sizeof(unsigned long long) * 16, m->stream));
      }
      tw.prof = m->near_prof.as<unsigned long long>();
    }
    hignn::launch_near_tc(a, tw, m->counter.as<int>(), m->err_flag(), m->num_sms, m->stream);
  }
  else
    hignn::launch_near_simt(a, m->wdev(), m->counter.as<int>(), m->num_sms, m->stream);
}

// u (tree order, FP64) = M f for f already gathered into f4.
void matvec_tree_order(hignn_model* m) {
  if (m->timing) HIGNN_CUDA(cudaEventRecord(m->ev[0], m->stream));
  if (m->fields & 1) {
    near_field(m);
    if (!m->lists.closeI.empty()) m->stats.gpu_launches += 1;
  }
  if (m->timing) HIGNN_CUDA(cudaEventRecord(m->ev[1], m->stream));
  if (m->fields & 2) far_field(m);
  if (m->timing) {
    HIGNN_CUDA(cudaEventRecord(m->ev[2], m->stream));
    HIGNN_CUDA(cudaEventSynchronize(m->ev[2]));
    float a = 0, b = 0;
    HIGNN_CUDA(cudaEventElapsedTime(&a, m->ev[0], m->ev[1]));
    HIGNN_CUDA(cudaEventElapsedTime(&b, m->ev[1], m->ev[2]));
    m->stats.t_close_ms = a;
    m->stats.t_far_ms = b;
    m->stats.t_dot_ms = a + b;
  }
}

void post_check(hignn_model* m);

// New positions (m->xyz, caller order) on the existing tree: x4 and the tree-order host copy are
// refreshed, the tree, the lists and the ACA plan are kept.
void refit_positions(hignn_model* m) {
  const int64_t n = m->n;
  std::vector<float4> x4(n);
  for (int64_t i = 0; i < n; i++) {
    const int64_t p = m->tree.perm[i];
    m->xt[3 * i] = m->xyz[3 * p];
    m->xt[3 * i + 1] = m->xyz[3 * p + 1];
    m->xt[3 * i + 2] = m->xyz[3 * p + 2];
    x4[i] = make_float4(m->xt[3 * i], m->xt[3 * i + 1], m->xt[3 * i + 2], 0.f);
  }
  if (m->device < 0) return;
  HIGNN_CUDA(cudaMemcpyAsync(m->x4.p, x4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
}

// Current device positions (tree order) back into m->xyz (caller order) and m->xt.
void download_positions(hignn_model* m) {
  const int64_t n = m->n;
  std::vector<float4> x4(n);
  HIGNN_CUDA(cudaMemcpyAsync(x4.data(), m->x4.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  for (int64_t i = 0; i < n; i++) {
    const int64_t p = m->tree.perm[i];
    m->xyz[3 * p] = m->xt[3 * i] = x4[i].x;
    m->xyz[3 * p + 1] = m->xt[3 * i + 1] = x4[i].y;
    m->xyz[3 * p + 2] = m->xt[3 * i + 2] = x4[i].z;
  }
}

// ---------------------------------------------------------------- graph form of the planned matvec
// The rank-planned H-matvec (every far block's ACA rank recorded by a previous product on the same
// tree and settings) needs no host decision between its launches: each batch runs its known number
// of iterations, and what would need the host -- blocks deferred past their recorded rank, blocks
// the student check sends back to the teacher, error counters -- is collected on the device
// (k_batch_end) and read once after the whole product. The launches from the force gather to the
// velocity scatter are captured into one CUDA graph (caller-order staging io_f -> io_u) and
// replayed; the rare reruns run eagerly afterwards.

bool graph_eligible(hignn_model* m) {
  return m->use_graph && m->device >= 0 && m->timing <= 1 && !m->record_pivots && !m->post_check &&
         m->n > 0 && hints_usable(m);
}

// Pointers and settings baked into the captured launches: a change means a new capture.
uint64_t graph_signature(hignn_model* m) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    h ^= v;
    h *= 1099511628211ull;
  };
  for (const DevBuf* b : {&m->x4, &m->perm, &m->f4, &m->u, &m->io_f, &m->io_u, &m->close_work, &m->weights,
                          &m->weights_tc, &m->counter, &m->student, &m->far_blocks, &m->far_state, &m->far_rows,
                          &m->far_cols, &m->far_used_row, &m->far_used_col, &m->far_C, &m->far_Q, &m->far_xc, &m->far_act,
                          &m->far_preI, &m->far_preJ, &m->far_ctr, &m->far_stats, &m->far_rank, &m->far_check,
                          &m->far_status})
    mix((uint64_t)(uintptr_t)b->p);
  mix((uint64_t)m->precision);
  mix((uint64_t)m->fields);
  mix((uint64_t)m->timing);
  mix((uint64_t)m->max_iter);
  mix((uint64_t)m->use_symmetry);
  mix((uint64_t)m->has_student);
  mix((uint64_t)m->sh_c0);
  mix((uint64_t)m->sh_c1);
  mix((uint64_t)m->batches.size());
  for (const auto& bt : m->batches) mix(((uint64_t)bt.b0 << 40) ^ ((uint64_t)bt.b1 << 16) ^ (uint64_t)bt.iters);
  uint64_t e, t;
  std::memcpy(&e, &m->epsilon, 8);
  const double tol = std::max(m->student_tol, m->epsilon);
  std::memcpy(&t, &tol, 8);
  mix(e);
  mix(t);
  return h;
}

void release_graph(hignn_model* m) {
  if (m->gexec) cudaGraphExecDestroy(m->gexec);
  if (m->gexec_far) cudaGraphExecDestroy(m->gexec_far);
  m->gexec = nullptr;
  m->gexec_far = nullptr;
  m->graph_sig = 0;
}

// The launches of the two graphs (issued on the capturing stream): the force gather (caller-order
// products) and the near field; the far field and the velocity scatter. Two graphs rather than
// one so that the near/far split can be timed with events between the launches.
void graph_near_body(hignn_model* m, bool caller_order) {
  if (caller_order)
    hignn::launch_gather_forces(m->io_f.as<float>(), m->perm.as<int32_t>(), m->f4.as<float4>(), m->u.as<double>(),
                                m->n, m->stream);
  if ((m->fields & 1) && !m->lists.closeI.empty()) near_field(m);
}

void graph_far_body(hignn_model* m, bool caller_order) {
  if ((m->fields & 2) && !m->batches.empty()) {
    const bool student_pass = m->precision == 2 && m->has_student;
    const hignn::MlpF32 w = m->wdev();
    const hignn::TcWeights tcw = m->wtc();
    const float* student = student_pass ? m->student.as<float>() : nullptr;
    int* status = m->far_status.as<int>();
    int32_t* lists = status + 8;
    const int cap = (int)(m->sh_f1 - m->sh_f0);
    HIGNN_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 8, m->stream));
    HIGNN_CUDA(cudaMemsetAsync(m->far_stats.p, 0, sizeof(unsigned long long) * 4, m->stream));
    const hignn::FarBlock* d_blocks = m->far_blocks.as<hignn::FarBlock>();
    for (const auto& bt : m->batches) {
      const hignn::FarArgs a = far_args(m, bt, d_blocks, student_pass);
      const auto& last = m->far_plan[bt.b1 - 1];
      HIGNN_CUDA(cudaMemsetAsync(m->far_used_row.p, 0, (size_t)last.rOff + last.nI, m->stream));
      HIGNN_CUDA(cudaMemsetAsync(m->far_used_col.p, 0, (size_t)last.colOff + last.nJ, m->stream));
      hignn::far_batch_launch(a, w, m->precision >= 1 ? &tcw : nullptr, student, m->err_flag(), m->num_sms,
                              m->stream, bt.iters);
      if (student_pass) {
        const size_t ns = (size_t)a.nb * hignn::kFarSamples;
        float* feat = m->far_check.as<float>();
        const float tol = (float)std::max(m->student_tol, m->epsilon);
        hignn::far_student_check_launch(a, tcw, student, tol, feat, feat + 3 * ns, feat + 12 * ns,
                                        reinterpret_cast<int*>(feat + 21 * ns), m->err_flag(), m->num_sms,
                                        m->stream);
      }
      hignn::far_batch_end(a, status, lists, cap, m->stream);
    }
  }
  if (caller_order)
    hignn::launch_scatter_velocities(m->u.as<double>(), m->perm.as<int32_t>(), m->io_u.as<float>(), m->n,
                                     m->stream);
}

// Captures body(m, caller_order) on the model's stream into an executable graph; returns its
// kernel launches.
template <class Body>
cudaGraphExec_t capture_graph(hignn_model* m, bool caller_order, Body&& body, int64_t* kernels) {
  cudaGraph_t g = nullptr;
  HIGNN_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  try {
    body(m, caller_order);
  } catch (...) {
    cudaStreamEndCapture(m->stream, &g);
    if (g) cudaGraphDestroy(g);
    (void)cudaGetLastError();
    throw;
  }
  HIGNN_CUDA(cudaStreamEndCapture(m->stream, &g));
  size_t nnodes = 0;
  cudaError_t e = cudaGraphGetNodes(g, nullptr, &nnodes);
  std::vector<cudaGraphNode_t> nodes(nnodes);
  if (e == cudaSuccess && nnodes) e = cudaGraphGetNodes(g, nodes.data(), &nnodes);
  int64_t k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType ty;
    if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) k++;
  }
  cudaGraphExec_t x = nullptr;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  HIGNN_CUDA(e);
  *kernels += k;
  return x;
}

// io_f -> io_u through the graph; returns false when the product has no complete rank plan yet
// (the caller runs the eager form, which records the ranks).
bool dot_graph(hignn_model* m, bool caller_order) {
  ensure_far_plan(m);
  if (!m->plan_hinted) return false;
  for (const auto& bt : m->batches)
    if (bt.iters <= 0) return false;
  const size_t nf = (size_t)(m->sh_f1 - m->sh_f0);
  m->far_status.ensure(sizeof(int) * (8 + 2 * std::max<size_t>(nf, 1)));
  if (m->precision == 2 && m->has_student) {
    int maxnb = 1;
    for (const auto& bt : m->batches) maxnb = std::max(maxnb, bt.b1 - bt.b0);
    m->far_check.ensure(sizeof(float) * (size_t)maxnb * hignn::kFarSamples * 21 + 64);
  }
  const uint64_t sig = graph_signature(m) ^ (caller_order ? 0x9e3779b97f4a7c15ull : 0ull);
  if (!m->gexec || !m->gexec_far || sig != m->graph_sig) {
    release_graph(m);
    m->graph_kernels = 0;
    m->gexec = capture_graph(m, caller_order, graph_near_body, &m->graph_kernels);
    m->gexec_far = capture_graph(m, caller_order, graph_far_body, &m->graph_kernels);
    m->graph_sig = sig;
    m->graph_iters = 0;
    for (const auto& bt : m->batches) m->graph_iters += bt.iters;
  }
  if (m->timing) HIGNN_CUDA(cudaEventRecord(m->ev[0], m->stream));
  HIGNN_CUDA(cudaGraphLaunch(m->gexec, m->stream));
  if (m->timing) HIGNN_CUDA(cudaEventRecord(m->ev[1], m->stream));
  HIGNN_CUDA(cudaGraphLaunch(m->gexec_far, m->stream));
  if (m->timing) HIGNN_CUDA(cudaEventRecord(m->ev[2], m->stream));
  // one read-back: the far-field status and statistics and the tensor-core error flag
  int status[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long fst[2] = {0, 0};
  int err = 0;
  const bool far_on = (m->fields & 2) && !m->batches.empty();
  if (far_on) {
    HIGNN_CUDA(cudaMemcpyAsync(status, m->far_status.p, sizeof(status), cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaMemcpyAsync(fst, m->far_stats.p, sizeof(fst), cudaMemcpyDeviceToHost, m->stream));
  }
  HIGNN_CUDA(cudaMemcpyAsync(&err, m->err_flag(), sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  if (err != 0) {
    HIGNN_CUDA(cudaMemsetAsync(m->err_flag(), 0, sizeof(int), m->stream));
    throw Error(HIGNN_ERR_LIMIT, "tensor-core kernel: a bounded wait timed out (code " + std::to_string(err) + ")");
  }
  if (status[2] != 0) throw Error(-5, "ACA: pivot search found no unused row/column (non-finite block entries?)");
  if (status[3] != 0) throw Error(-5, "ACA did not converge within max_iter iterations");
  m->stats.gpu_launches = m->graph_kernels;
  m->stats.far_rank_max = status[4];
  m->stats.student_fallback_blocks = status[1];
  m->stats.far_iterations = m->graph_iters;
  if (m->timing) {
    float a = 0, b = 0;
    HIGNN_CUDA(cudaEventElapsedTime(&a, m->ev[0], m->ev[1]));
    HIGNN_CUDA(cudaEventElapsedTime(&b, m->ev[1], m->ev[2]));
    m->stats.t_close_ms = a;
    m->stats.t_far_ms = b;
    m->stats.t_dot_ms = a + b;
  }
  if (far_on && (status[0] > 0 || status[1] > 0)) {  // reruns, eagerly, then the scatter again
    const int cap = (int)nf;
    std::vector<int32_t> lists(2 * (size_t)cap);
    HIGNN_CUDA(cudaMemcpyAsync(lists.data(), m->far_status.as<int>() + 8, sizeof(int32_t) * 2 * cap,
                               cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    std::vector<int> deferred(lists.begin(), lists.begin() + std::min(status[0], cap));
    std::vector<int> fallback(lists.begin() + cap, lists.begin() + cap + std::min(status[1], cap));
    std::sort(deferred.begin(), deferred.end());
    std::sort(fallback.begin(), fallback.end());
    const bool student_pass = m->precision == 2 && m->has_student;
    int iters = 0;
    if (!deferred.empty()) {
      FarOutcome r2;
      run_far_subset(m, deferred, student_pass, &iters, &r2);
      if (!r2.deferred.empty()) throw Error(HIGNN_ERR_LIMIT, "ACA: a block was deferred at its full capacity");
      fallback.insert(fallback.end(), r2.fallback.begin(), r2.fallback.end());
    }
    if (!fallback.empty()) {
      FarOutcome r3;
      run_far_subset(m, fallback, false, &iters, &r3);
      if (!r3.deferred.empty()) throw Error(HIGNN_ERR_LIMIT, "ACA: a block was deferred at its full capacity");
    }
    m->stats.far_iterations += iters;
    m->stats.gpu_launches += 5 * (int64_t)iters + (caller_order ? 1 : 0);
    if (caller_order)
      hignn::launch_scatter_velocities(m->u.as<double>(), m->perm.as<int32_t>(), m->io_u.as<float>(), m->n,
                                       m->stream);
    HIGNN_CUDA(cudaMemcpyAsync(fst, m->far_stats.p, sizeof(fst), cudaMemcpyDeviceToHost, m->stream));
    if (!deferred.empty()) {  // ranks recorded again for the next plan
      m->rank_hint.resize(m->lists.farI.size());
      HIGNN_CUDA(cudaMemcpyAsync(m->rank_hint.data(), m->far_rank.p, sizeof(int32_t) * m->rank_hint.size(),
                                 cudaMemcpyDeviceToHost, m->stream));
    }
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    if (m->precision >= 1) check_device_error(m);
  }
  m->stats.far_rank_sum = (int64_t)fst[0];
  m->stats.far_evals = (int64_t)fst[1];
  return true;
}

// The matvec of the time loops (forces already in f4, u zeroed, tree order) as a graph: the same
// launches as graph_near_body and graph_far_body without the gather and the scatter. Returns false when it cannot run
// (no complete rank plan yet, or graphs off); the caller then runs the eager form.
bool matvec_graph_tree_order(hignn_model* m) {
  if (!graph_eligible(m)) return false;
  return dot_graph(m, false);
}

void dot_impl(hignn_model* m, float* d_u, const float* d_f) {
  if (graph_eligible(m)) {  // the graph reads io_f and writes io_u
    if (d_f != m->io_f.as<float>())
      HIGNN_CUDA(cudaMemcpyAsync(m->io_f.p, d_f, sizeof(float) * 3 * m->n, cudaMemcpyDeviceToDevice, m->stream));
    if (dot_graph(m, true)) {
      if (d_u != m->io_u.as<float>())
        HIGNN_CUDA(cudaMemcpyAsync(d_u, m->io_u.p, sizeof(float) * 3 * m->n, cudaMemcpyDeviceToDevice, m->stream));
      return;
    }
  }
  m->stats.gpu_launches = 2;  // gather + scatter
  hignn::launch_gather_forces(d_f, m->perm.as<int32_t>(), m->f4.as<float4>(), m->u.as<double>(), m->n, m->stream);
  matvec_tree_order(m);
  if (m->post_check) post_check(m);
  hignn::launch_scatter_velocities(m->u.as<double>(), m->perm.as<int32_t>(), d_u, m->n, m->stream);
  if (m->precision >= 1) check_device_error(m);
}

// Dense product over all leaf pairs into m->u (tree order); f4 already gathered.
void dense_tree_order(hignn_model* m, double* u_out) {
  const auto& lv = m->lists.leaves;
  // one work item per leaf pair, counted in 32 bits on the device
  if ((double)lv.size() * (double)lv.size() > 2147483647.0)
    throw Error(HIGNN_ERR_ARG, "dense product: " + std::to_string(lv.size()) +
                                   " leaves give more leaf pairs than one launch takes; use hignn_dense_rows");
  std::vector<hignn::PairWork> work;
  work.reserve(lv.size() * lv.size());
  for (int64_t I : lv)
    for (int64_t J : lv) {
      const auto& a = m->tree.nodes[I];
      const auto& b = m->tree.nodes[J];
      hignn::PairWork w{};
      w.sI = (int32_t)a.start;
      w.nI = (int32_t)(a.end - a.start);
      w.sJ = (int32_t)b.start;
      w.nJ = (int32_t)(b.end - b.start);
      w.flags = hignn::kPairSymmetrize;
      work.push_back(w);
    }
  m->tmp_work.ensure(sizeof(hignn::PairWork) * std::max<size_t>(1, work.size()));
  HIGNN_CUDA(cudaMemcpyAsync(m->tmp_work.p, work.data(), sizeof(hignn::PairWork) * work.size(),
                             cudaMemcpyHostToDevice, m->stream));
  HIGNN_CUDA(cudaMemsetAsync(u_out, 0, sizeof(double) * 3 * m->n, m->stream));
  hignn::NearArgs a{};
  a.work = m->tmp_work.as<hignn::PairWork>();
  a.nwork = (int)work.size();
  a.xI = a.xJ = m->x4.as<float4>();
  a.fI = a.fJ = m->f4.as<float4>();
  a.uI = a.uJ = u_out;
  hignn::launch_near_simt(a, m->wdev(), m->counter.as<int>(), m->num_sms, m->stream);
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
}

// PostCheckDot (src/PostCheckDot.cpp:351-377): relative L2 of the H-matrix result vs the dense product.
void post_check(hignn_model* m) {
  DevBuf ud;
  ud.ensure(sizeof(double) * 3 * m->n);
  dense_tree_order(m, ud.as<double>());
  std::vector<double> a(3 * m->n), b(3 * m->n);
  HIGNN_CUDA(cudaMemcpyAsync(a.data(), m->u.p, sizeof(double) * 3 * m->n, cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaMemcpyAsync(b.data(), ud.p, sizeof(double) * 3 * m->n, cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); i++) {
    num += (a[i] - b[i]) * (a[i] - b[i]);
    den += b[i] * b[i];
  }
  std::printf("relative error of the H-matrix product vs the dense product: %.6e\n", std::sqrt(num / den));
  std::fflush(stdout);
  ud.release();
}

}  // namespace

namespace hignn {

void model_view(hignn_model* m, ModelView& v) {
  v = ModelView{};
  if (!m) return;
  v.device = m->device;
  v.stream = m->stream;
  v.num_sms = m->num_sms;
  v.n = m->n;
  v.ready = m->device >= 0 && m->has_weights && m->tree_ready && m->x4.p && m->f4.p && m->io_f.p;
  if (!v.ready) return;
  v.x4 = m->x4.as<float4>();
  v.f4 = m->f4.as<float4>();
  v.perm = m->perm.as<int32_t>();
  v.io_f = m->io_f.as<float>();
  v.w = m->wdev();
  v.nodes = &m->tree.nodes;
  v.leaves = &m->lists.leaves;
  v.inv_perm = &m->inv_perm;
}

void set_last_error(const char* msg) { set_error(msg); }

}  // namespace hignn

extern "C" {

int hignn_last_error(char* buf, size_t size) {
  if (!buf || size == 0) return HIGNN_ERR_ARG;
  std::snprintf(buf, size, "%s", g_last_error.c_str());
  return HIGNN_OK;
}

int hignn_version(void) { return 100; }

int hignn_create(const float* xyz, int64_t n, int block_size, int device, hignn_model** out) {
  return guard([&] {
    if (!out) throw Error(HIGNN_ERR_ARG, "out is null");
    *out = nullptr;
    if (!xyz || n <= 0) throw Error(HIGNN_ERR_ARG, "coordinates must be a non-empty (n, 3) array");
    if (n >= (int64_t(1) << 31)) throw Error(HIGNN_ERR_ARG, "n must be below 2^31");
    if (block_size <= 0) throw Error(HIGNN_ERR_ARG, "block_size must be positive");
    if (device >= 0 && block_size > hignn::kMaxLeaf)
      throw Error(HIGNN_ERR_ARG, "block_size must be at most " + std::to_string(hignn::kMaxLeaf) +
                                     " on a device (the near-field kernels stage one leaf in shared memory)");
    auto* m = new hignn_model();
    try {
      m->n = n;
      m->block_size = block_size;
      m->xyz.assign(xyz, xyz + 3 * n);
      for (float v : m->xyz)
        if (!std::isfinite(v)) throw Error(HIGNN_ERR_ARG, "coordinates must be finite");
      m->device = device;
      if (device >= 0) {
        int count = 0;
        HIGNN_CUDA(cudaGetDeviceCount(&count));
        if (device >= count) throw Error(HIGNN_ERR_ARG, "no CUDA device " + std::to_string(device));
        HIGNN_CUDA(cudaSetDevice(device));
        HIGNN_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        HIGNN_CUDA(cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device));
        HIGNN_CUDA(cudaMallocHost((void**)&m->host_ctr, sizeof(int32_t) * hignn::kCtrCount));
        for (auto& e : m->lev)
      if (e) cudaEventDestroy(e);
    for (auto& e : m->ev) HIGNN_CUDA(cudaEventCreate(&e));
        for (auto& e : m->lev) HIGNN_CUDA(cudaEventCreate(&e));
        m->counter.ensure(64);
        HIGNN_CUDA(cudaMemsetAsync(m->counter.p, 0, 64, m->stream));
      }
      m->stats.n = n;
    } catch (...) {
      hignn_destroy(m);
      throw;
    }
    *out = m;
  });
}

int hignn_destroy(hignn_model* m) {
  if (!m) return HIGNN_OK;
  if (m->device >= 0) {
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (DevBuf* b : {&m->x4, &m->perm, &m->slot, &m->f4, &m->u, &m->io_f, &m->io_u, &m->close_work, &m->weights,
                      &m->weights_tc, &m->counter, &m->student,
                      &m->far_blocks, &m->far_state, &m->far_rows, &m->far_cols, &m->far_used_row, &m->far_used_col,
                      &m->far_C, &m->far_Q, &m->far_xc, &m->far_act, &m->far_preI, &m->far_preJ, &m->far_ctr, &m->far_stats,
                      &m->far_rank, &m->far_retry, &m->far_check, &m->tmp_work, &m->tmp_x, &m->tmp_u, &m->tmp_pos,
                      &m->dp_k, &m->dp_err, &m->near_prof, &m->far_status})
      b->release();
    m->cells.release();
    m->tree_dev.release();
    release_graph(m);
    for (auto& e : m->ev)
      if (e) cudaEventDestroy(e);
    if (m->host_ctr) cudaFreeHost(m->host_ctr);
    if (m->stream) cudaStreamDestroy(m->stream);
  }
  delete m;
  return HIGNN_OK;
}

namespace {

// An HGNW weight file (hignn_b200/weights.py): dense layers W (out x in, row-major) and b.
void read_hgnw(const char* path, uint32_t want_wrap, std::vector<std::vector<float>>& W,
               std::vector<std::vector<float>>& B, std::vector<int>& dims) {
  std::ifstream fh(path, std::ios::binary);
  if (!fh) throw Error(HIGNN_ERR_IO, std::string("cannot open weight file ") + path);
  std::vector<char> data((std::istreambuf_iterator<char>(fh)), std::istreambuf_iterator<char>());
  auto rd32 = [&](size_t off) {
    if (off + 4 > data.size()) throw Error(HIGNN_ERR_IO, "truncated weight file");
    uint32_t v;
    std::memcpy(&v, data.data() + off, 4);
    return v;
  };
  if (data.size() < 20 || std::memcmp(data.data(), "HGNW", 4) != 0)
    throw Error(HIGNN_ERR_IO, std::string(path) + " is not an HGNW weight file");
  if (rd32(4) != 1) throw Error(HIGNN_ERR_IO, "unsupported HGNW version");
  const uint32_t L = rd32(8), act = rd32(12), wrap = rd32(16);
  if (act != 1 || wrap != want_wrap) throw Error(HIGNN_ERR_IO, std::string(path) + ": not the expected tanh network");
  if (L < 1 || L > 16) throw Error(HIGNN_ERR_IO, "bad layer count in weight file");
  size_t off = 20;
  std::vector<std::pair<uint32_t, uint32_t>> shp;
  for (uint32_t l = 0; l < L; l++) {
    shp.push_back({rd32(off), rd32(off + 4)});
    off += 8;
  }
  dims.assign(1, (int)shp[0].second);
  for (auto& sh : shp) dims.push_back((int)sh.first);
  W.clear();
  B.clear();
  for (auto& sh : shp) {
    const size_t nw = (size_t)sh.first * sh.second;
    if (off + 4 * (nw + sh.first) > data.size()) throw Error(HIGNN_ERR_IO, "truncated weight file");
    std::vector<float> w(nw), b(sh.first);
    std::memcpy(w.data(), data.data() + off, 4 * nw);
    off += 4 * nw;
    std::memcpy(b.data(), data.data() + off, 4 * sh.first);
    off += 4 * sh.first;
    W.push_back(std::move(w));
    B.push_back(std::move(b));
  }
  if (off != data.size()) throw Error(HIGNN_ERR_IO, "trailing bytes in weight file");
}

}  // namespace

int hignn_load_two_body(hignn_model* m, const char* path) {
  return guard([&] {
    if (!m || !path) throw Error(HIGNN_ERR_ARG, "null argument");
    std::vector<std::vector<float>> W, B;
    std::vector<int> dims;
    read_hgnw(path, 1, W, B, dims);
    if (W.size() != 3) throw Error(HIGNN_ERR_ARG, "two-body network must have 3 dense layers");
    upload_weights(m, W, B, dims);
  });
}

int hignn_load_two_body_mem(hignn_model* m, int num_layers, const int32_t* dims, const float* params,
                            int activation) {
  return guard([&] {
    if (!m || !dims || !params) throw Error(HIGNN_ERR_ARG, "null argument");
    if (activation != 1) throw Error(HIGNN_ERR_ARG, "two-body network activation must be tanh (1)");
    // the shape is checked before any weight is read from `params`
    if (num_layers != 3 || dims[0] != 3 || dims[1] != hignn::kH1 || dims[2] != hignn::kH2 || dims[3] != hignn::kOut)
      throw Error(HIGNN_ERR_ARG, "two-body network must be 3 -> 128 -> 512 -> 9 (tanh)");
    std::vector<int> d(dims, dims + num_layers + 1);
    std::vector<std::vector<float>> W, B;
    const float* p = params;
    for (int l = 0; l < num_layers; l++) {
      const size_t o = d[l + 1], i = d[l];
      W.emplace_back(p, p + o * i);
      p += o * i;
      B.emplace_back(p, p + o);
      p += o;
    }
    upload_weights(m, W, B, d);
  });
}

int hignn_set_param(hignn_model* m, int key, double v) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    switch (key) {
      case HIGNN_P_EPSILON: m->epsilon = v; break;
      case HIGNN_P_ETA: m->eta = v; break;
      case HIGNN_P_MAX_ITER:
        if (v < 1 || v > hignn::kMaxIterCap)
          throw Error(HIGNN_ERR_ARG, "max_iter must be in [1, " + std::to_string(hignn::kMaxIterCap) + "]");
        m->max_iter = (int)v;
        break;
      case HIGNN_P_MAT_POOL_SIZE_FACTOR: m->mat_pool_size_factor = (int)v; break;
      case HIGNN_P_MAX_FAR_DOT_WORK_NODE_SIZE:
        if (v < 1) throw Error(HIGNN_ERR_ARG, "max_far_dot_work_node_size must be >= 1");
        m->max_far_dot_work_node_size = (int)v;
        break;
      case HIGNN_P_MAX_RELATIVE_COORD:
        if (v < 1) throw Error(HIGNN_ERR_ARG, "max_relative_coord must be >= 1");
        m->max_relative_coord = (int64_t)v;
        break;
      case HIGNN_P_POST_CHECK_FLAG: m->post_check = v != 0; break;
      case HIGNN_P_USE_SYMMETRY: m->use_symmetry = v != 0; break;
      case HIGNN_P_MAX_FAR_FIELD_DISTANCE: m->max_far_field_distance = v; break;
      case HIGNN_P_PRECISION:
        if (v != 0 && v != 1 && v != 2) throw Error(HIGNN_ERR_ARG, "precision must be 0, 1 or 2");
        m->precision = (int)v;
        break;
      case HIGNN_P_FAR_BATCH_ROWS:
        // a batch's row offsets and prefix sums are 32-bit on the device
        if (!(v >= 1024 && v <= (double)(int64_t(1) << 30)))
          throw Error(HIGNN_ERR_ARG, "far_batch_rows must be in [1024, 2^30]");
        m->far_batch_rows = (int64_t)v;
        break;
      case HIGNN_P_FAR_POOL_MB:
        if (!(v >= 1 && v <= (double)(int64_t(1) << 24)))
          throw Error(HIGNN_ERR_ARG, "far_pool_mb must be in [1, 2^24]");
        m->far_pool_bytes = (int64_t)(v * 1048576.0);
        break;
      case HIGNN_P_RANK_HINT_OFFSET: m->rank_hint_offset = (int)v; break;
      case HIGNN_P_TIMING: m->timing = (int)v; break;
      case HIGNN_P_STUDENT_TOL: m->student_tol = v; break;
      case HIGNN_P_FIELDS:
        if (v < 0 || v > 3) throw Error(HIGNN_ERR_ARG, "fields must be in [0, 3]");
        m->fields = (int)v;
        break;
      case HIGNN_P_RECORD_PIVOTS: m->record_pivots = v != 0; break;
      case HIGNN_P_TREE_DEVICE:
        if ((v != 0) != m->tree_on_device) m->tree_ready = false;  // rebuilt by the chosen builder
        m->tree_on_device = v != 0;
        break;
      case HIGNN_P_GRAPH:
        m->use_graph = v != 0;
        if (!m->use_graph) release_graph(m);
        break;
      case HIGNN_P_KEEP_RANKS: m->keep_ranks = v != 0; break;
      default: throw Error(HIGNN_ERR_ARG, "unknown parameter key " + std::to_string(key));
    }
  });
}

int hignn_get_param(hignn_model* m, int key, double* v) {
  return guard([&] {
    if (!m || !v) throw Error(HIGNN_ERR_ARG, "null argument");
    switch (key) {
      case HIGNN_P_EPSILON: *v = m->epsilon; break;
      case HIGNN_P_ETA: *v = m->eta; break;
      case HIGNN_P_MAX_ITER: *v = m->max_iter; break;
      case HIGNN_P_MAT_POOL_SIZE_FACTOR: *v = m->mat_pool_size_factor; break;
      case HIGNN_P_MAX_FAR_DOT_WORK_NODE_SIZE: *v = m->max_far_dot_work_node_size; break;
      case HIGNN_P_MAX_RELATIVE_COORD: *v = (double)m->max_relative_coord; break;
      case HIGNN_P_POST_CHECK_FLAG: *v = m->post_check; break;
      case HIGNN_P_USE_SYMMETRY: *v = m->use_symmetry; break;
      case HIGNN_P_MAX_FAR_FIELD_DISTANCE: *v = m->max_far_field_distance; break;
      case HIGNN_P_PRECISION: *v = m->precision; break;
      case HIGNN_P_FAR_BATCH_ROWS: *v = (double)m->far_batch_rows; break;
      case HIGNN_P_FAR_POOL_MB: *v = (double)m->far_pool_bytes / 1048576.0; break;
      case HIGNN_P_RANK_HINT_OFFSET: *v = m->rank_hint_offset; break;
      case HIGNN_P_TIMING: *v = m->timing; break;
      case HIGNN_P_STUDENT_TOL: *v = m->student_tol; break;
      case HIGNN_P_FIELDS: *v = m->fields; break;
      case HIGNN_P_RECORD_PIVOTS: *v = m->record_pivots; break;
      case HIGNN_P_TREE_DEVICE: *v = m->tree_on_device; break;
      case HIGNN_P_GRAPH: *v = m->use_graph; break;
      case HIGNN_P_KEEP_RANKS: *v = m->keep_ranks; break;
      default: throw Error(HIGNN_ERR_ARG, "unknown parameter key " + std::to_string(key));
    }
  });
}

int hignn_update_coord(hignn_model* m, const float* xyz, int64_t n) {
  return guard([&] {
    if (!m || !xyz) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n != m->n)
      throw Error(HIGNN_ERR_ARG, "update_coord: expected " + std::to_string(m->n) + " particles, got " +
                                     std::to_string(n));
    for (int64_t i = 0; i < 3 * n; i++)
      if (!std::isfinite(xyz[i])) throw Error(HIGNN_ERR_ARG, "coordinates must be finite");
    m->xyz.assign(xyz, xyz + 3 * n);
    build_structures(m);
  });
}

int hignn_update_coord_keep_tree(hignn_model* m, const float* xyz, int64_t n) {
  return guard([&] {
    if (!m || !xyz) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n != m->n)
      throw Error(HIGNN_ERR_ARG, "update_coord_keep_tree: expected " + std::to_string(m->n) + " particles, got " +
                                     std::to_string(n));
    for (int64_t i = 0; i < 3 * n; i++)
      if (!std::isfinite(xyz[i])) throw Error(HIGNN_ERR_ARG, "coordinates must be finite");
    ensure_tree(m);
    m->xyz.assign(xyz, xyz + 3 * n);
    refit_positions(m);
  });
}

int hignn_pair_forces(hignn_model* m, const float* xyz, float* f, int64_t n, const float* gravity, double De,
                      double a, double re, double cutoff) {
  return guard([&] {
    if (!m || !xyz || !f) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n <= 0) throw Error(HIGNN_ERR_ARG, "pair_forces: n must be positive");
    if (cutoff < 0) throw Error(HIGNN_ERR_ARG, "pair_forces: cutoff must be >= 0");
    require_device(m);
    m->tmp_x.ensure(sizeof(float4) * n);
    m->io_f.ensure(sizeof(float) * 3 * n);
    m->io_u.ensure(sizeof(float) * 3 * n);
    HIGNN_CUDA(cudaMemcpyAsync(m->io_f.p, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, m->stream));
    hignn::launch_pack_positions(m->io_f.as<float>(), n, m->tmp_x.as<float4>(), m->stream);
    const hignn::MorseParams mp{(float)De, (float)a, (float)re, cutoff};
    if (cutoff > 0) m->cells.build(m->tmp_x.as<float4>(), n, cutoff, m->stream);
    const float3 g = gravity ? make_float3(gravity[0], gravity[1], gravity[2]) : make_float3(0.f, 0.f, 0.f);
    hignn::launch_morse(m->tmp_x.as<float4>(), n, m->cells, mp, g, nullptr, m->io_u.as<float>(), m->stream);
    HIGNN_CUDA(cudaMemcpyAsync(f, m->io_u.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

namespace {

void check_force_model(const hignn_force_model& fm, int64_t n) {
  if (!(fm.morse_cutoff >= 0)) throw Error(HIGNN_ERR_ARG, "forces: the Morse cutoff must be >= 0");
  if (fm.n_filament < 0 || fm.n_chain < 0 || (fm.n_filament > 0 && fm.n_chain < 1))
    throw Error(HIGNN_ERR_ARG, "forces: bad filament counts");
  if (fm.n_filament > 0 && fm.n_filament * (int64_t)fm.n_chain > n)
    throw Error(HIGNN_ERR_ARG, "forces: the filaments hold more rows than there are particles");
}

// Forces of fm at positions x (slot[row] = position of caller row `row` in x, or null: x in
// caller order) into f4 or f3 (same order as x).
void apply_forces(hignn_model* m, const float4* x, int64_t n, const int32_t* slot, const hignn_force_model& fm,
                  float4* f4, float* f3) {
  const hignn::MorseParams mp{(float)fm.morse_De, (float)fm.morse_a, (float)fm.morse_re, fm.morse_cutoff};
  if (fm.morse_cutoff > 0) m->cells.build(x, n, fm.morse_cutoff, m->stream);
  const float3 g = make_float3(fm.gravity[0], fm.gravity[1], fm.gravity[2]);
  hignn::launch_morse(x, n, m->cells, mp, g, f4, f3, m->stream);
  const hignn::FilamentParams fp{fm.n_filament, fm.n_chain, (float)fm.rest_length, (float)fm.k_t, fm.k_b};
  hignn::launch_filaments(x, slot, fp, f4, f3, m->stream);
}

}  // namespace

int hignn_forces(hignn_model* m, const float* xyz, float* f, int64_t n, const hignn_force_model* fm) {
  return guard([&] {
    if (!m || !xyz || !f || !fm) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n <= 0) throw Error(HIGNN_ERR_ARG, "forces: n must be positive");
    check_force_model(*fm, n);
    require_device(m);
    m->tmp_x.ensure(sizeof(float4) * n);
    m->io_f.ensure(sizeof(float) * 3 * n);
    m->io_u.ensure(sizeof(float) * 3 * n);
    HIGNN_CUDA(cudaMemcpyAsync(m->io_f.p, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, m->stream));
    hignn::launch_pack_positions(m->io_f.as<float>(), n, m->tmp_x.as<float4>(), m->stream);
    apply_forces(m, m->tmp_x.as<float4>(), n, nullptr, *fm, nullptr, m->io_u.as<float>());
    HIGNN_CUDA(cudaMemcpyAsync(f, m->io_u.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

namespace {

void tb_add_device(hignn_tb* t, hignn_model* m);

// u (tree order, FP64) = M(x) F(x) at the device positions m->x4, plus the three-body and self
// terms when a three-body object is attached.
void step_velocity(hignn_model* m, const hignn_force_model& fm) {
  const int64_t n = m->n;
  HIGNN_CUDA(cudaEventRecord(m->lev[0], m->stream));
  apply_forces(m, m->x4.as<float4>(), n, m->slot.as<int32_t>(), fm, m->f4.as<float4>(), nullptr);
  HIGNN_CUDA(cudaMemsetAsync(m->u.p, 0, sizeof(double) * 3 * n, m->stream));
  HIGNN_CUDA(cudaEventRecord(m->lev[1], m->stream));
  if (!matvec_graph_tree_order(m)) {
    matvec_tree_order(m);
    m->loop_prof[7] += 1;
  }
  HIGNN_CUDA(cudaEventRecord(m->lev[2], m->stream));
  if (m->tb) tb_add_device(m->tb, m);
  HIGNN_CUDA(cudaEventRecord(m->lev[3], m->stream));
  if (m->precision >= 1) check_device_error(m);
  HIGNN_CUDA(cudaEventSynchronize(m->lev[3]));
  float a = 0, b = 0, c = 0;
  HIGNN_CUDA(cudaEventElapsedTime(&a, m->lev[0], m->lev[1]));
  HIGNN_CUDA(cudaEventElapsedTime(&b, m->lev[1], m->lev[2]));
  HIGNN_CUDA(cudaEventElapsedTime(&c, m->lev[2], m->lev[3]));
  m->loop_prof[2] += a;
  m->loop_prof[3] += b;
  m->loop_prof[4] += c;
  m->loop_prof[6] += 1;
}

// The device time loop: method 0 = explicit Euler, 1 = explicit midpoint (RK2).
void run_steps(hignn_model* m, float* xyz, int64_t n, int steps, double dt, int rebuild_every,
               const hignn_force_model* fm, int method, const char* name) {
  if (!m || !xyz || !fm) throw Error(HIGNN_ERR_ARG, "null argument");
  if (n != m->n) throw Error(HIGNN_ERR_ARG, std::string(name) + ": particle count differs from the model's");
  if (steps < 0 || !(dt > 0) || rebuild_every < 0)
    throw Error(HIGNN_ERR_ARG, std::string(name) + ": need steps >= 0, dt > 0, rebuild_every >= 0");
  check_force_model(*fm, n);
  require_device(m);
  require_weights(m);
  require_student_if_needed(m);
  if (m->shard_world != 1)
    throw Error(HIGNN_ERR_STATE, std::string(name) + " needs the whole product (shard world 1): a sharded step "
                                                     "would need the all-reduce of u between the matvec and the update");
  for (int64_t i = 0; i < 3 * n; i++)
    if (!std::isfinite(xyz[i])) throw Error(HIGNN_ERR_ARG, "coordinates must be finite");
  // start from xyz with a tree built for it
  const auto w0 = std::chrono::steady_clock::now();
  for (double& v : m->loop_prof) v = 0.0;
  m->xyz.assign(xyz, xyz + 3 * n);
  build_structures(m);
  if (method == 1) m->tmp_x.ensure(sizeof(float4) * n);
  for (int s = 0; s < steps; s++) {
    if (s > 0 && rebuild_every > 0 && s % rebuild_every == 0) {
      const auto r0 = std::chrono::steady_clock::now();
      download_positions(m);  // m->xyz <- current positions
      build_structures(m);
      m->loop_prof[1] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r0).count();
    }
    step_velocity(m, *fm);  // forces at the current positions, in tree order, into the matvec
    if (method == 1) {
      // midpoint: x_mid = x + (dt / 2) u(x) on the kept tree, then x += dt u(x_mid)
      HIGNN_CUDA(cudaMemcpyAsync(m->tmp_x.p, m->x4.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, m->stream));
      hignn::launch_advance(m->x4.as<float4>(), m->u.as<double>(), n, (float)(0.5 * dt), m->stream);
      step_velocity(m, *fm);
      HIGNN_CUDA(cudaMemcpyAsync(m->x4.p, m->tmp_x.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, m->stream));
    }
    hignn::launch_advance(m->x4.as<float4>(), m->u.as<double>(), n, (float)dt, m->stream);
  }
  download_positions(m);
  std::copy(m->xyz.begin(), m->xyz.end(), xyz);
  m->loop_prof[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
  m->loop_prof[5] = steps;
}

}  // namespace

int hignn_run_euler(hignn_model* m, float* xyz, int64_t n, int steps, double dt, int rebuild_every,
                    const hignn_force_model* fm) {
  return guard([&] { run_steps(m, xyz, n, steps, dt, rebuild_every, fm, 0, "run_euler"); });
}

int hignn_run_rk2(hignn_model* m, float* xyz, int64_t n, int steps, double dt, int rebuild_every,
                  const hignn_force_model* fm) {
  return guard([&] { run_steps(m, xyz, n, steps, dt, rebuild_every, fm, 1, "run_rk2"); });
}

// ExplicitRk4::Run (include/TimeIntegrator.hpp:602-860) with the velocity on the device: adaptive
// Dormand-Prince 5(4), FSAL, the reference's float stage arithmetic and step control (k1 zero on
// the first step; a grown step size is discarded because the next step starts from
// min(h0, tf - t)). The initial velocity evaluation the reference makes for its output callback
// is skipped (there is no callback).
int hignn_run_dp45(hignn_model* m, float* xyz, int64_t n, double tf, double dt0, double threshold,
                   int rebuild_every, const hignn_force_model* fm, int64_t* steps_taken) {
  return guard([&] {
    if (!m || !xyz || !fm) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n != m->n) throw Error(HIGNN_ERR_ARG, "run_dp45: particle count differs from the model's");
    if (!(tf >= 0) || !(dt0 > 0) || !(threshold > 0) || rebuild_every < 0)
      throw Error(HIGNN_ERR_ARG, "run_dp45: need tf >= 0, dt0 > 0, threshold > 0, rebuild_every >= 0");
    check_force_model(*fm, n);
    require_device(m);
    require_weights(m);
    require_student_if_needed(m);
    if (m->shard_world != 1) throw Error(HIGNN_ERR_STATE, "run_dp45 needs the whole product (shard world 1)");
    for (int64_t i = 0; i < 3 * n; i++)
      if (!std::isfinite(xyz[i])) throw Error(HIGNN_ERR_ARG, "coordinates must be finite");
    // Dormand-Prince tableau (include/TimeIntegrator.hpp:503-549), float constants
    const float A[7][6] = {{0, 0, 0, 0, 0, 0},
                           {1.f / 5.f, 0, 0, 0, 0, 0},
                           {3.f / 40.f, 9.f / 40.f, 0, 0, 0, 0},
                           {44.f / 45.f, -56.f / 15.f, 32.f / 9.f, 0, 0, 0},
                           {19372.f / 6561.f, -25360.f / 2187.f, 64448.f / 6561.f, -212.f / 729.f, 0, 0},
                           {9017.f / 3168.f, -355.f / 33.f, 46732.f / 5247.f, 49.f / 176.f, -5103.f / 18656.f, 0},
                           {35.f / 384.f, 0.f, 500.f / 1113.f, 125.f / 192.f, -2187.f / 6784.f, 11.f / 84.f}};
    const float b1 = 35.f / 384.f, b3 = 500.f / 1113.f, b4 = 125.f / 192.f, b5 = -2187.f / 6784.f, b6 = 11.f / 84.f;
    const float dc[6] = {b1 - 5179.f / 57600.f, b3 - 7571.f / 16695.f, b4 - 393.f / 640.f,
                         b5 - (-92097.f) / 339200.f, b6 - 187.f / 2100.f, -1.f / 40.f};
    m->xyz.assign(xyz, xyz + 3 * n);
    build_structures(m);
    const size_t m3 = 3 * (size_t)n;
    m->dp_k.ensure(sizeof(float) * 7 * m3);
    m->dp_err.ensure(sizeof(double));
    m->tmp_x.ensure(sizeof(float4) * n);
    HIGNN_CUDA(cudaMemsetAsync(m->dp_k.p, 0, sizeof(float) * 7 * m3, m->stream));  // k1 = 0 on the first step
    float* k = m->dp_k.as<float>();
    double t = 0.0;
    int64_t count = 0;
    const double h0 = dt0;
    while (t < tf - 1e-5) {
      double dt = std::min(h0, tf - t);
      if (count > 0 && rebuild_every > 0 && count % rebuild_every == 0) {
        // k1 (the last step's k7) is stored in tree order: carry it over to the new tree's order
        // through the caller's order, as the positions are
        std::vector<float> kt(m3), kc(m3);
        HIGNN_CUDA(cudaMemcpyAsync(kt.data(), k, sizeof(float) * m3, cudaMemcpyDeviceToHost, m->stream));
        download_positions(m);  // synchronises the stream, so kt is complete
        for (int64_t i = 0; i < n; i++) {
          const int64_t p = m->tree.perm[i];
          for (int c = 0; c < 3; c++) kc[3 * p + c] = kt[3 * i + c];
        }
        build_structures(m);
        for (int64_t i = 0; i < n; i++) {
          const int64_t p = m->tree.perm[i];
          for (int c = 0; c < 3; c++) kt[3 * i + c] = kc[3 * p + c];
        }
        HIGNN_CUDA(cudaMemcpyAsync(k, kt.data(), sizeof(float) * m3, cudaMemcpyHostToDevice, m->stream));
        HIGNN_CUDA(cudaStreamSynchronize(m->stream));  // kt is released at the end of this block
      }
      HIGNN_CUDA(cudaMemcpyAsync(m->tmp_x.p, m->x4.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, m->stream));
      double err = 100.0;
      while (err > threshold) {
        for (int i = 1; i < 7; i++) {
          hignn::Dp45Terms tm{};
          for (int jj = 0; jj < 6; jj++) {
            const float coef = A[i][jj];
            if (i < 6 ? jj < i : coef != 0.f) {  // stage i uses k_1 .. k_i; the solution row skips k_2
              tm.j[tm.n] = jj + 1;
              tm.c[tm.n] = (float)(coef * dt);
              tm.n++;
            }
          }
          hignn::launch_dp45_stage(m->tmp_x.as<float4>(), k, n, tm, m->x4.as<float4>(), m->stream);
          step_velocity(m, *fm);
          hignn::launch_velocity_to_float(m->u.as<double>(), (int64_t)m3, k + (size_t)i * m3, m->stream);
        }
        const hignn::Dp45Error de{{dc[0], dc[1], dc[2], dc[3], dc[4], dc[5]}, (float)dt};
        hignn::launch_dp45_error(k, n, de, m->dp_err.as<double>(), m->stream);
        double e2 = 0.0;
        HIGNN_CUDA(cudaMemcpyAsync(&e2, m->dp_err.p, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        HIGNN_CUDA(cudaStreamSynchronize(m->stream));
        err = std::sqrt(e2);
        if (!std::isfinite(err)) throw Error(HIGNN_ERR_LIMIT, "run_dp45: non-finite error estimate");
        if (err > threshold) {
          dt = dt * std::max(0.8 * std::pow(err / threshold, -0.2), 0.1);
          dt = std::max(dt, 1e-6);
        }
      }
      t += dt;
      // first-same-as-last: k1 <- k7
      HIGNN_CUDA(cudaMemcpyAsync(k, k + 6 * m3, sizeof(float) * m3, cudaMemcpyDeviceToDevice, m->stream));
      count++;
    }
    download_positions(m);
    std::copy(m->xyz.begin(), m->xyz.end(), xyz);
    if (steps_taken) *steps_taken = count;
  });
}

int hignn_dot(hignn_model* m, float* u, const float* f, int64_t n) {
  return guard([&] {
    if (!m || !u || !f) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n != m->n) throw Error(HIGNN_ERR_ARG, "dot: size mismatch");
    require_device(m);
    require_weights(m);
    require_student_if_needed(m);
    ensure_tree(m);
    HIGNN_CUDA(cudaMemcpyAsync(m->io_f.p, f, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, m->stream));
    dot_impl(m, m->io_u.as<float>(), m->io_f.as<float>());
    HIGNN_CUDA(cudaMemcpyAsync(u, m->io_u.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_dot_device(hignn_model* m, float* d_u, const float* d_f, int64_t n) {
  return guard([&] {
    if (!m || !d_u || !d_f) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n != m->n) throw Error(HIGNN_ERR_ARG, "dot: size mismatch");
    require_device(m);
    require_weights(m);
    require_student_if_needed(m);
    ensure_tree(m);
    dot_impl(m, d_u, d_f);
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_dense_dot(hignn_model* m, float* u, const float* f, int64_t n) {
  return guard([&] {
    if (!m || !u || !f) throw Error(HIGNN_ERR_ARG, "null argument");
    if (n != m->n) throw Error(HIGNN_ERR_ARG, "dense_dot: size mismatch");
    require_device(m);
    require_weights(m);
    ensure_tree(m);
    HIGNN_CUDA(cudaMemcpyAsync(m->io_f.p, f, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, m->stream));
    hignn::launch_gather_forces(m->io_f.as<float>(), m->perm.as<int32_t>(), m->f4.as<float4>(), m->u.as<double>(),
                                n, m->stream);
    dense_tree_order(m, m->u.as<double>());
    hignn::launch_scatter_velocities(m->u.as<double>(), m->perm.as<int32_t>(), m->io_u.as<float>(), n, m->stream);
    HIGNN_CUDA(cudaMemcpyAsync(u, m->io_u.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_dense_rows(hignn_model* m, double* u_rows, const float* f, const int64_t* rows, int64_t nrows,
                     int precision) {
  return guard([&] {
    if (!m || !u_rows || !f || (!rows && nrows > 0)) throw Error(HIGNN_ERR_ARG, "null argument");
    if (precision != 0 && precision != HIGNN_DENSE_F64)
      throw Error(HIGNN_ERR_ARG, "dense_rows: precision must be 0 (FP32 network) or HIGNN_DENSE_F64 (FP64 network)");
    require_device(m);
    require_weights(m);
    ensure_tree(m);
    if (nrows <= 0) return;
    const auto& lv = m->lists.leaves;
    // one work item per (chunk of 128 rows, leaf), counted and offset in 32 bits on the device
    if (nrows > 2147483647 - 128 || (double)((nrows + 127) / 128) * (double)lv.size() > 2147483647.0)
      throw Error(HIGNN_ERR_ARG, "dense_rows: too many rows for one call; split the rows over several calls");
    std::vector<int32_t> pos(nrows);
    for (int64_t q = 0; q < nrows; q++) {
      if (rows[q] < 0 || rows[q] >= m->n) throw Error(HIGNN_ERR_ARG, "row index out of range");
      pos[q] = (int32_t)m->inv_perm[rows[q]];
    }
    std::vector<hignn::PairWork> work;
    for (int64_t c0 = 0; c0 < nrows; c0 += 128)
      for (int64_t J : lv) {
        const auto& b = m->tree.nodes[J];
        hignn::PairWork w{};
        w.sI = (int32_t)c0;
        w.nI = (int32_t)std::min<int64_t>(128, nrows - c0);
        w.sJ = (int32_t)b.start;
        w.nJ = (int32_t)(b.end - b.start);
        w.flags = hignn::kPairSymmetrize;
        work.push_back(w);
      }
    m->tmp_pos.ensure(sizeof(int32_t) * nrows);
    m->tmp_x.ensure(sizeof(float4) * nrows);
    m->tmp_u.ensure(sizeof(double) * 3 * nrows);
    m->tmp_work.ensure(sizeof(hignn::PairWork) * work.size());
    HIGNN_CUDA(cudaMemcpyAsync(m->tmp_pos.p, pos.data(), sizeof(int32_t) * nrows, cudaMemcpyHostToDevice, m->stream));
    HIGNN_CUDA(cudaMemcpyAsync(m->tmp_work.p, work.data(), sizeof(hignn::PairWork) * work.size(),
                               cudaMemcpyHostToDevice, m->stream));
    HIGNN_CUDA(cudaMemcpyAsync(m->io_f.p, f, sizeof(float) * 3 * m->n, cudaMemcpyHostToDevice, m->stream));
    hignn::launch_gather_forces(m->io_f.as<float>(), m->perm.as<int32_t>(), m->f4.as<float4>(), m->u.as<double>(),
                                m->n, m->stream);
    hignn::launch_gather_positions(m->x4.as<float4>(), m->tmp_pos.as<int32_t>(), m->tmp_x.as<float4>(), nrows,
                                   m->stream);
    HIGNN_CUDA(cudaMemsetAsync(m->tmp_u.p, 0, sizeof(double) * 3 * nrows, m->stream));
    hignn::NearArgs a{};
    a.work = m->tmp_work.as<hignn::PairWork>();
    a.nwork = (int)work.size();
    a.xI = m->tmp_x.as<float4>();
    a.fI = m->tmp_x.as<float4>();  // unused without the transposed update
    a.uI = m->tmp_u.as<double>();
    a.xJ = m->x4.as<float4>();
    a.fJ = m->f4.as<float4>();
    a.uJ = m->u.as<double>();
    if (precision == HIGNN_DENSE_F64)
      hignn::launch_dense_f64(a, m->wdev(), m->counter.as<int>(), m->num_sms, m->stream);
    else
      hignn::launch_near_simt(a, m->wdev(), m->counter.as<int>(), m->num_sms, m->stream);
    HIGNN_CUDA(cudaMemcpyAsync(u_rows, m->tmp_u.p, sizeof(double) * 3 * nrows, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_two_body_eval(hignn_model* m, const float* d_r, float* d_y, int64_t n, int precision) {
  return guard([&] {
    if (!m || (!d_r && n > 0) || (!d_y && n > 0)) throw Error(HIGNN_ERR_ARG, "null argument");
    if (precision != 0 && precision != 1) throw Error(HIGNN_ERR_ARG, "unsupported precision");
    require_device(m);
    require_weights(m);
    if (precision == 1) {
      hignn::launch_eval_tc(d_r, d_y, n, m->wtc(), m->err_flag(), m->num_sms, m->stream);
      check_device_error(m);
    } else {
      hignn::launch_eval_simt(d_r, d_y, n, m->wdev(), m->num_sms, m->stream);
    }
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_get_stats(hignn_model* m, hignn_stats* out) {
  return guard([&] {
    if (!m || !out) throw Error(HIGNN_ERR_ARG, "null argument");
    ensure_tree(m);
    *out = m->stats;
  });
}

int hignn_get_tree(hignn_model* m, int64_t* tree5, int64_t* perm) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    ensure_tree(m);
    if (tree5)
      for (size_t i = 0; i < m->tree.nodes.size(); i++) {
        const auto& t = m->tree.nodes[i];
        tree5[5 * i] = t.child0;
        tree5[5 * i + 1] = t.child1;
        tree5[5 * i + 2] = t.start;
        tree5[5 * i + 3] = t.end;
        tree5[5 * i + 4] = t.level;
      }
    if (perm) std::copy(m->tree.perm.begin(), m->tree.perm.end(), perm);
  });
}

int hignn_get_lists(hignn_model* m, int64_t* ci, int64_t* cj, int64_t* fi, int64_t* fj) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    ensure_tree(m);
    if (ci) std::copy(m->lists.closeI.begin(), m->lists.closeI.end(), ci);
    if (cj) std::copy(m->lists.closeJ.begin(), m->lists.closeJ.end(), cj);
    if (fi) std::copy(m->lists.farI.begin(), m->lists.farI.end(), fi);
    if (fj) std::copy(m->lists.farJ.begin(), m->lists.farJ.end(), fj);
  });
}

int hignn_set_shard(hignn_model* m, int rank, int world) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    if (world < 1 || rank < 0 || rank >= world) throw Error(HIGNN_ERR_ARG, "shard: need 0 <= rank < world");
    m->shard_rank = rank;
    m->shard_world = world;
    m->shard_ready = false;
    m->plan_ready = false;
  });
}

int hignn_get_shard(hignn_model* m, int64_t* ranges) {
  return guard([&] {
    if (!m || !ranges) throw Error(HIGNN_ERR_ARG, "null argument");
    ensure_tree(m);
    ensure_shard(m);
    ranges[0] = m->sh_c0;
    ranges[1] = m->sh_c1;
    ranges[2] = m->sh_f0;
    ranges[3] = m->sh_f1;
  });
}

int hignn_set_student(hignn_model* m, const float* params, int nparams) {
  return guard([&] {
    if (!m || !params) throw Error(HIGNN_ERR_ARG, "null argument");
    if (nparams != hignn::kStudentParams)
      throw Error(HIGNN_ERR_ARG, "student network has " + std::to_string(hignn::kStudentParams) + " parameters");
    require_device(m);
    m->student.ensure(sizeof(float) * hignn::kStudentParams);
    HIGNN_CUDA(cudaMemcpyAsync(m->student.p, params, sizeof(float) * hignn::kStudentParams, cudaMemcpyHostToDevice,
                               m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    m->has_student = true;
    m->hint_valid = false;
  });
}

int hignn_get_student(hignn_model* m, float* params, int nparams) {
  return guard([&] {
    if (!m || !params) throw Error(HIGNN_ERR_ARG, "null argument");
    if (nparams != hignn::kStudentParams)
      throw Error(HIGNN_ERR_ARG, "student network has " + std::to_string(hignn::kStudentParams) + " parameters");
    if (!m->has_student) throw Error(HIGNN_ERR_STATE, "no student network (train or set one first)");
    require_device(m);
    HIGNN_CUDA(cudaMemcpyAsync(params, m->student.p, sizeof(float) * hignn::kStudentParams, cudaMemcpyDeviceToHost,
                               m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_student_eval(hignn_model* m, const float* d_r, float* d_y, int64_t n) {
  return guard([&] {
    if (!m || (n > 0 && (!d_r || !d_y))) throw Error(HIGNN_ERR_ARG, "null argument");
    if (!m->has_student) throw Error(HIGNN_ERR_STATE, "no student network (train or set one first)");
    require_device(m);
    hignn::launch_student_eval(m->student.as<float>(), d_r, d_y, n, m->num_sms, m->stream);
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_student_grad(hignn_model* m, const float* d_r, const float* d_t, int64_t n, float* grad, double* loss) {
  return guard([&] {
    if (!m || !d_r || !d_t || !grad || n <= 0) throw Error(HIGNN_ERR_ARG, "null argument or empty batch");
    if (!m->has_student) throw Error(HIGNN_ERR_STATE, "no student network (train or set one first)");
    require_device(m);
    const int nparts = (int)((n + 127) / 128);
    DevBuf partial, lpart, g, l;
    partial.ensure(sizeof(float) * (size_t)nparts * hignn::kStudentParams);
    lpart.ensure(sizeof(float) * nparts);
    g.ensure(sizeof(float) * hignn::kStudentParams);
    l.ensure(sizeof(float));
    hignn::launch_student_grad(m->student.as<float>(), d_r, d_t, n, n, 0, partial.as<float>(), lpart.as<float>(),
                               g.as<float>(), l.as<float>(), m->stream);
    float lh = 0.f;
    HIGNN_CUDA(cudaMemcpyAsync(grad, g.p, sizeof(float) * hignn::kStudentParams, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaMemcpyAsync(&lh, l.p, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    if (loss) *loss = (double)lh / (9.0 * (double)n);
    for (DevBuf* b : {&partial, &lpart, &g, &l}) b->release();
  });
}

int hignn_train_student(hignn_model* m, int steps, int batch, int64_t nsamples, double lr, uint64_t seed,
                        double* final_loss) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    if (steps < 0 || batch < 128 || nsamples < batch || lr <= 0)
      throw Error(HIGNN_ERR_ARG, "train_student: need steps >= 0, batch >= 128, nsamples >= batch, lr > 0");
    require_device(m);
    require_weights(m);
    using hignn::kStudentParams;
    // initial parameters: uniform Glorot weights from the seed, zero biases, small last layer
    std::vector<float> p(kStudentParams, 0.f);
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto rnd = [&]() {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      return (float)((st >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f;
    };
    const int offs[4] = {0, 128, 1184, 2240}, fin[4] = {3, 32, 32, 32}, fout[4] = {32, 32, 32, 9};
    for (int l = 0; l < 4; l++) {
      const float a = std::sqrt(6.f / (fin[l] + fout[l])) * (l == 3 ? 0.1f : 1.f);
      for (int q = 0; q < fin[l] * fout[l]; q++) p[offs[l] + q] = a * rnd();
    }
    m->student.ensure(sizeof(float) * kStudentParams);
    HIGNN_CUDA(cudaMemcpyAsync(m->student.p, p.data(), sizeof(float) * kStudentParams, cudaMemcpyHostToDevice,
                               m->stream));
    DevBuf r, t, partial, lpart, g, m1, m2, l;
    r.ensure(sizeof(float) * 3 * (size_t)nsamples);
    t.ensure(sizeof(float) * 9 * (size_t)nsamples);
    const int nparts = (batch + 127) / 128;
    partial.ensure(sizeof(float) * (size_t)nparts * kStudentParams);
    lpart.ensure(sizeof(float) * nparts);
    g.ensure(sizeof(float) * kStudentParams);
    m1.ensure(sizeof(float) * kStudentParams);
    m2.ensure(sizeof(float) * kStudentParams);
    l.ensure(sizeof(float));
    HIGNN_CUDA(cudaMemsetAsync(m1.p, 0, sizeof(float) * kStudentParams, m->stream));
    HIGNN_CUDA(cudaMemsetAsync(m2.p, 0, sizeof(float) * kStudentParams, m->stream));
    // teacher evaluations at admissible separations (FP32 network), as residuals of the RPY tensor
    hignn::launch_student_samples(r.as<float>(), nsamples, seed ^ 0x5EEDull, 4.0f, 400.0f, m->stream);
    hignn::launch_eval_simt(r.as<float>(), t.as<float>(), nsamples, m->wdev(), m->num_sms, m->stream);
    hignn::launch_student_targets(r.as<float>(), t.as<float>(), nsamples, m->stream);
    double b1t = 1.0, b2t = 1.0;
    for (int k = 0; k < steps; k++) {
      const double lrk = lr * (0.01 + 0.99 * 0.5 * (1.0 + std::cos(3.14159265358979323846 * k / std::max(1, steps))));
      hignn::launch_student_grad(m->student.as<float>(), r.as<float>(), t.as<float>(), nsamples, batch,
                                 (seed + 1) * 0x9E3779B97F4A7C15ull + (uint64_t)k + 1, partial.as<float>(),
                                 lpart.as<float>(), g.as<float>(), nullptr, m->stream);
      b1t *= 0.9;
      b2t *= 0.999;
      hignn::launch_student_adam(m->student.as<float>(), g.as<float>(), m1.as<float>(), m2.as<float>(), (float)lrk,
                                 (float)b1t, (float)b2t, m->stream);
    }
    // loss on one more random batch
    hignn::launch_student_grad(m->student.as<float>(), r.as<float>(), t.as<float>(), nsamples, batch,
                               seed * 31 + 7, partial.as<float>(), lpart.as<float>(), g.as<float>(), l.as<float>(),
                               m->stream);
    float lh = 0.f;
    HIGNN_CUDA(cudaMemcpyAsync(&lh, l.p, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    if (final_loss) *final_loss = (double)lh / (9.0 * (double)batch);
    for (DevBuf* b : {&r, &t, &partial, &lpart, &g, &m1, &m2, &l}) b->release();
    m->has_student = true;
    m->hint_valid = false;
  });
}

int hignn_get_far_pivots(hignn_model* m, int32_t* ranks, int32_t* rows, int32_t* cols, int ld) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    if (m->piv_rank.size() != m->lists.farI.size() || m->piv_ld == 0)
      throw Error(HIGNN_ERR_STATE, "no pivots recorded (set HIGNN_P_RECORD_PIVOTS and run a dot)");
    if (ld < m->piv_ld) throw Error(HIGNN_ERR_ARG, "ld must be >= max_iter + 1");
    const size_t nf = m->piv_rank.size();
    if (ranks) std::copy(m->piv_rank.begin(), m->piv_rank.end(), ranks);
    for (size_t b = 0; b < nf; b++)
      for (int l = 0; l < m->piv_ld; l++) {
        if (rows) rows[b * ld + l] = m->piv_rows[b * m->piv_ld + l];
        if (cols) cols[b * ld + l] = m->piv_cols[b * m->piv_ld + l];
      }
  });
}

int hignn_near_wait_profile(hignn_model* m, uint64_t* counters) {
  return guard([&] {
    if (!m || !counters) throw Error(HIGNN_ERR_ARG, "null argument");
    std::memset(counters, 0, sizeof(uint64_t) * 16);
    if (!m->near_prof.p) return;
    require_device(m);
    HIGNN_CUDA(cudaMemcpyAsync(counters, m->near_prof.p, sizeof(uint64_t) * 16, cudaMemcpyDeviceToHost, m->stream));
    HIGNN_CUDA(cudaMemsetAsync(m->near_prof.p, 0, sizeof(uint64_t) * 16, m->stream));
    HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int hignn_loop_profile(hignn_model* m, double* ms) {
  return guard([&] {
    if (!m || !ms) throw Error(HIGNN_ERR_ARG, "null argument");
    for (int i = 0; i < 8; i++) ms[i] = m->loop_prof[i];
  });
}

int hignn_synchronize(hignn_model* m) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null model");
    if (m->device >= 0) {
      HIGNN_CUDA(cudaSetDevice(m->device));
      HIGNN_CUDA(cudaStreamSynchronize(m->stream));
    }
  });
}

int hignn_get_stream(hignn_model* m, void** stream) {
  return guard([&] {
    if (!m || !stream) throw Error(HIGNN_ERR_ARG, "null argument");
    *stream = (void*)m->stream;
  });
}

}  // extern "C"

// ---------------------------------------------------------------- neighbour lists

struct hignn_nbl {
  hignn::NeighbourLists lists;
  explicit hignn_nbl(int device) : lists(device) {}
};

int hignn_nbl_create(int device, hignn_nbl** out) {
  return guard([&] {
    if (!out) throw Error(HIGNN_ERR_ARG, "null argument");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Error(HIGNN_ERR_NODEV, "neighbour lists: no CUDA device");
    }
    if (device < 0 || device >= count) throw Error(HIGNN_ERR_ARG, "neighbour lists: bad device");
    *out = new hignn_nbl(device);
  });
}

void hignn_nbl_destroy(hignn_nbl* l) { delete l; }

int hignn_nbl_update_coord(hignn_nbl* l, const float* xyz, int64_t n) {
  return guard([&] {
    if (!l) throw Error(HIGNN_ERR_ARG, "null argument");
    l->lists.update_coord(xyz, n);
  });
}

int hignn_nbl_set_two_body_epsilon(hignn_nbl* l, float eps) {
  return guard([&] {
    if (!l) throw Error(HIGNN_ERR_ARG, "null argument");
    l->lists.set_two_body_epsilon(eps);
  });
}

int hignn_nbl_set_three_body_epsilon(hignn_nbl* l, float eps) {
  return guard([&] {
    if (!l) throw Error(HIGNN_ERR_ARG, "null argument");
    l->lists.set_three_body_epsilon(eps);
  });
}

int hignn_nbl_build_two_body_info(hignn_nbl* l) {
  return guard([&] {
    if (!l) throw Error(HIGNN_ERR_ARG, "null argument");
    l->lists.build_two_body();
  });
}

int hignn_nbl_build_three_body_info(hignn_nbl* l) {
  return guard([&] {
    if (!l) throw Error(HIGNN_ERR_ARG, "null argument");
    l->lists.build_three_body();
  });
}

int hignn_nbl_get_edge_info(hignn_nbl* l, int kind, int by_index, const uint64_t* index, int64_t nindex,
                            uint64_t* out, int64_t cap, int64_t* num_edges) {
  return guard([&] {
    if (!l || !num_edges) throw Error(HIGNN_ERR_ARG, "null argument");
    if (kind < HIGNN_EDGES_TWO_BODY || kind > HIGNN_EDGES_THREE_BODY_SELF)
      throw Error(HIGNN_ERR_ARG, "neighbour lists: unknown edge kind");
    const int64_t e = l->lists.count(kind, by_index != 0, index, nindex);
    *num_edges = e;
    if (!out) return;
    const int rows = kind == HIGNN_EDGES_THREE_BODY ? 3 : 2;
    if (cap < rows * e) throw Error(HIGNN_ERR_ARG, "neighbour lists: output holds fewer than rows * edges entries");
    l->lists.copy_out(kind, by_index != 0, index, nindex, out);
  });
}

int hignn_nbl_edge_info_device(hignn_nbl* l, int kind, const uint64_t** d_info, int64_t* num_edges) {
  return guard([&] {
    if (!l || !d_info || !num_edges) throw Error(HIGNN_ERR_ARG, "null argument");
    *d_info = l->lists.device_list(kind, num_edges);
  });
}

int hignn_nbl_last_build_ms(hignn_nbl* l, double* ms) {
  return guard([&] {
    if (!l || !ms) throw Error(HIGNN_ERR_ARG, "null argument");
    *ms = l->lists.last_build_ms();
  });
}

int hignn_nbl_get_stream(hignn_nbl* l, void** stream) {
  return guard([&] {
    if (!l || !stream) throw Error(HIGNN_ERR_ARG, "null argument");
    *stream = (void*)l->lists.stream();
  });
}

// ---------------------------------------------------------------- three-body near field

struct hignn_tb {
  hignn::NeighbourLists lists;
  hignn::TbNet nets[2];
  int num_sms = 0;
  float eps = 5.0f;
  DevBuf f4, fin, u, err, prof, etri, eself;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  double ms_lists = 0, ms_three = 0, ms_self = 0;
  int64_t triplets = 0, pairs = 0;
  explicit hignn_tb(int device) : lists(device) {
    HIGNN_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    for (auto& e : ev) HIGNN_CUDA(cudaEventCreate(&e));
  }
  ~hignn_tb() {
    cudaSetDevice(lists.device());
    cudaStreamSynchronize(lists.stream());
    for (DevBuf* b : {&f4, &fin, &u, &err, &prof, &etri, &eself}) b->release();
    for (auto& n : nets)
      n.d_img.release();
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

namespace {

void tb_set(hignn_tb* t, int which, const std::vector<std::vector<float>>& W, const std::vector<std::vector<float>>& B,
            const std::vector<int>& dims) {
  if (which != HIGNN_TB_THREE_BODY && which != HIGNN_TB_SELF) throw Error(HIGNN_ERR_ARG, "unknown network kind");
  const int kin = which == HIGNN_TB_THREE_BODY ? 6 : 3;
  if (dims.size() != 5 || dims[0] != kin || dims[1] != hignn::kTbH1 || dims[2] != hignn::kTbH2 ||
      dims[3] != hignn::kTbH3 || dims[4] != 9)
    throw Error(HIGNN_ERR_ARG, which == HIGNN_TB_THREE_BODY ? "three-body network must be 6 -> 256 -> 1024 -> 512 -> 9"
                                                            : "self network must be 3 -> 256 -> 1024 -> 512 -> 9");
  HIGNN_CUDA(cudaSetDevice(t->lists.device()));
  hignn::tb_upload(t->nets[which], kin, W, B, t->lists.stream());
}

}  // namespace

namespace {

// The three-body and self terms at the model's device positions (tree order), added into its
// FP64 velocities: the edge lists are built from a copy of those positions, so their indices are
// tree positions, as are the forces f4 and the velocities u.
void tb_add_device(hignn_tb* t, hignn_model* m) {
  const int64_t n = m->n;
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));  // positions, forces and the matvec are complete
  const auto t0 = std::chrono::steady_clock::now();
  t->lists.update_coord_device(m->x4.as<float4>(), n);
  t->lists.set_three_body_epsilon(t->eps);
  t->lists.build_three_body();
  t->ms_lists = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  int64_t e3 = 0, es = 0;
  const uint64_t* tri = t->lists.device_list(hignn::kEdgesThreeBody, &e3);
  const uint64_t* self = t->lists.device_list(hignn::kEdgesThreeBodySelf, &es);
  t->triplets = e3;
  t->pairs = es;
  t->err.ensure(sizeof(int));
  HIGNN_CUDA(cudaMemsetAsync(t->err.p, 0, sizeof(int), m->stream));
  hignn::launch_three_body(hignn::kTbThreeBody, t->nets[0].dev(), t->nets[0].cst, tri, e3, t->lists.positions(),
                           m->f4.as<float4>(), m->u.as<double>(), t->err.as<int>(), nullptr, t->num_sms, m->stream);
  hignn::launch_three_body(hignn::kTbSelf, t->nets[1].dev(), t->nets[1].cst, self, es, t->lists.positions(),
                           m->f4.as<float4>(), m->u.as<double>(), t->err.as<int>(), nullptr, t->num_sms, m->stream);
  int e = 0;
  HIGNN_CUDA(cudaMemcpyAsync(&e, t->err.p, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  HIGNN_CUDA(cudaStreamSynchronize(m->stream));
  if (e != 0) throw Error(HIGNN_ERR_LIMIT, "three-body kernel: a wait timed out (code " + std::to_string(e) + ")");
}

}  // namespace

int hignn_set_three_body(hignn_model* m, hignn_tb* t) {
  return guard([&] {
    if (!m) throw Error(HIGNN_ERR_ARG, "null argument");
    if (t) {
      require_device(m);
      if (t->lists.device() != m->device) throw Error(HIGNN_ERR_ARG, "three-body object on another device");
      if (!t->nets[0].loaded || !t->nets[1].loaded)
        throw Error(HIGNN_ERR_STATE, "three-body: load both the three-body and the self network");
    }
    m->tb = t;
  });
}

int hignn_tb_create(int device, hignn_tb** out) {
  return guard([&] {
    if (!out) throw Error(HIGNN_ERR_ARG, "null argument");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Error(HIGNN_ERR_NODEV, "three-body: no CUDA device");
    }
    if (device < 0 || device >= count) throw Error(HIGNN_ERR_ARG, "three-body: bad device");
    *out = new hignn_tb(device);
  });
}

void hignn_tb_destroy(hignn_tb* t) { delete t; }

int hignn_tb_load(hignn_tb* t, int which, const char* path) {
  return guard([&] {
    if (!t || !path) throw Error(HIGNN_ERR_ARG, "null argument");
    std::vector<std::vector<float>> W, B;
    std::vector<int> dims;
    read_hgnw(path, which == HIGNN_TB_SELF ? 3u : 2u, W, B, dims);
    tb_set(t, which, W, B, dims);
  });
}

int hignn_tb_load_mem(hignn_tb* t, int which, int num_layers, const int32_t* dims, const float* params) {
  return guard([&] {
    if (!t || !dims || !params) throw Error(HIGNN_ERR_ARG, "null argument");
    if (num_layers != 4) throw Error(HIGNN_ERR_ARG, "three-body networks have 4 dense layers");
    // the shape is checked before any weight is read from `params`
    if (which != HIGNN_TB_THREE_BODY && which != HIGNN_TB_SELF) throw Error(HIGNN_ERR_ARG, "unknown network kind");
    const int kin = which == HIGNN_TB_THREE_BODY ? 6 : 3;
    if (dims[0] != kin || dims[1] != hignn::kTbH1 || dims[2] != hignn::kTbH2 || dims[3] != hignn::kTbH3 || dims[4] != 9)
      throw Error(HIGNN_ERR_ARG, which == HIGNN_TB_THREE_BODY ? "three-body network must be 6 -> 256 -> 1024 -> 512 -> 9"
                                                              : "self network must be 3 -> 256 -> 1024 -> 512 -> 9");
    std::vector<int> d(dims, dims + num_layers + 1);
    std::vector<std::vector<float>> W, B;
    const float* p = params;
    for (int l = 0; l < num_layers; l++) {
      const size_t o = d[l + 1], i = d[l];
      W.emplace_back(p, p + o * i);
      p += o * i;
      B.emplace_back(p, p + o);
      p += o;
    }
    tb_set(t, which, W, B, d);
  });
}

int hignn_tb_set_epsilon(hignn_tb* t, float eps) {
  return guard([&] {
    if (!t) throw Error(HIGNN_ERR_ARG, "null argument");
    if (!(eps > 0.f)) throw Error(HIGNN_ERR_ARG, "three-body: epsilon must be positive");
    t->eps = eps;
  });
}

namespace {

// The two kernels on the device edge lists tri (3, e3) and self (2, es) at the positions already
// in t->lists; f and u are host arrays.
void tb_run(hignn_tb* t, const float* f, float* u, int64_t n, const uint64_t* tri, int64_t e3, const uint64_t* self,
            int64_t es) {
  cudaStream_t s = t->lists.stream();
  t->triplets = e3;
  t->pairs = es;
  t->fin.ensure(sizeof(float) * 3 * n);
  t->f4.ensure(sizeof(float4) * n);
  t->u.ensure(sizeof(float) * 3 * n);
  t->err.ensure(sizeof(int));
  t->prof.ensure(sizeof(unsigned long long) * 12);
  HIGNN_CUDA(cudaMemsetAsync(t->prof.p, 0, sizeof(unsigned long long) * 12, s));
  HIGNN_CUDA(cudaMemcpyAsync(t->fin.p, f, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
  hignn::launch_pack_positions(t->fin.as<float>(), n, t->f4.as<float4>(), s);
  HIGNN_CUDA(cudaMemsetAsync(t->u.p, 0, sizeof(float) * 3 * n, s));
  HIGNN_CUDA(cudaMemsetAsync(t->err.p, 0, sizeof(int), s));
  HIGNN_CUDA(cudaEventRecord(t->ev[0], s));
  hignn::launch_three_body(hignn::kTbThreeBody, t->nets[0].dev(), t->nets[0].cst, tri, e3, t->lists.positions(),
                           t->f4.as<float4>(), t->u.as<float>(), t->err.as<int>(), t->prof.as<unsigned long long>(),
                           t->num_sms, s);
  HIGNN_CUDA(cudaEventRecord(t->ev[1], s));
  hignn::launch_three_body(hignn::kTbSelf, t->nets[1].dev(), t->nets[1].cst, self, es, t->lists.positions(),
                           t->f4.as<float4>(), t->u.as<float>(), t->err.as<int>(),
                           t->prof.as<unsigned long long>() + 6, t->num_sms, s);
  HIGNN_CUDA(cudaEventRecord(t->ev[2], s));
  int e = 0;
  HIGNN_CUDA(cudaMemcpyAsync(u, t->u.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, s));
  HIGNN_CUDA(cudaMemcpyAsync(&e, t->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  HIGNN_CUDA(cudaStreamSynchronize(s));
  float a = 0, b = 0;
  HIGNN_CUDA(cudaEventElapsedTime(&a, t->ev[0], t->ev[1]));
  HIGNN_CUDA(cudaEventElapsedTime(&b, t->ev[1], t->ev[2]));
  t->ms_three = a;
  t->ms_self = b;
  if (e != 0) throw Error(HIGNN_ERR_LIMIT, "three-body kernel: a wait timed out (code " + std::to_string(e) + ")");
}

void tb_check(hignn_tb* t, const float* xyz, const float* f, float* u, int64_t n) {
  if (!t || !xyz || !f || !u) throw Error(HIGNN_ERR_ARG, "null argument");
  if (n <= 0) throw Error(HIGNN_ERR_ARG, "three-body: n must be positive");
  if (!t->nets[0].loaded || !t->nets[1].loaded)
    throw Error(HIGNN_ERR_STATE, "three-body: load both the three-body and the self network");
}

}  // namespace

int hignn_tb_velocity(hignn_tb* t, const float* xyz, const float* f, float* u, int64_t n) {
  return guard([&] {
    tb_check(t, xyz, f, u, n);
    HIGNN_CUDA(cudaSetDevice(t->lists.device()));
    const auto t0 = std::chrono::steady_clock::now();
    t->lists.update_coord(xyz, n);
    t->lists.set_three_body_epsilon(t->eps);
    t->lists.build_three_body();
    t->ms_lists = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    int64_t e3 = 0, es = 0;
    const uint64_t* tri = t->lists.device_list(hignn::kEdgesThreeBody, &e3);
    const uint64_t* self = t->lists.device_list(hignn::kEdgesThreeBodySelf, &es);
    tb_run(t, f, u, n, tri, e3, self, es);
  });
}

int hignn_tb_velocity_edges(hignn_tb* t, const float* xyz, const float* f, float* u, int64_t n, const uint64_t* tri,
                            int64_t e3, const uint64_t* self_edges, int64_t es) {
  return guard([&] {
    tb_check(t, xyz, f, u, n);
    if (e3 < 0 || es < 0 || (e3 > 0 && !tri) || (es > 0 && !self_edges))
      throw Error(HIGNN_ERR_ARG, "three-body: bad edge lists");
    for (int64_t q = 0; q < 3 * e3; q++)
      if (tri[q] >= (uint64_t)n) throw Error(HIGNN_ERR_ARG, "three-body: triplet index out of range");
    for (int64_t q = 0; q < 2 * es; q++)
      if (self_edges[q] >= (uint64_t)n) throw Error(HIGNN_ERR_ARG, "three-body: self-edge index out of range");
    HIGNN_CUDA(cudaSetDevice(t->lists.device()));
    cudaStream_t s = t->lists.stream();
    t->lists.update_coord(xyz, n);
    t->ms_lists = 0.0;
    t->etri.ensure(sizeof(uint64_t) * 3 * (e3 > 0 ? e3 : 1));
    t->eself.ensure(sizeof(uint64_t) * 2 * (es > 0 ? es : 1));
    if (e3 > 0) HIGNN_CUDA(cudaMemcpyAsync(t->etri.p, tri, sizeof(uint64_t) * 3 * e3, cudaMemcpyHostToDevice, s));
    if (es > 0)
      HIGNN_CUDA(cudaMemcpyAsync(t->eself.p, self_edges, sizeof(uint64_t) * 2 * es, cudaMemcpyHostToDevice, s));
    tb_run(t, f, u, n, t->etri.as<uint64_t>(), e3, t->eself.as<uint64_t>(), es);
  });
}

int hignn_tb_wait_profile(hignn_tb* t, uint64_t* counters) {
  return guard([&] {
    if (!t || !counters) throw Error(HIGNN_ERR_ARG, "null argument");
    HIGNN_CUDA(cudaSetDevice(t->lists.device()));
    std::memset(counters, 0, sizeof(uint64_t) * 12);
    if (!t->prof.p) return;
    HIGNN_CUDA(cudaMemcpy(counters, t->prof.p, sizeof(uint64_t) * 12, cudaMemcpyDeviceToHost));
  });
}

int hignn_tb_stats(hignn_tb* t, double* ms_lists, double* ms_three, double* ms_self, int64_t* triplets,
                   int64_t* pairs) {
  return guard([&] {
    if (!t) throw Error(HIGNN_ERR_ARG, "null argument");
    if (ms_lists) *ms_lists = t->ms_lists;
    if (ms_three) *ms_three = t->ms_three;
    if (ms_self) *ms_self = t->ms_self;
    if (triplets) *triplets = t->triplets;
    if (pairs) *pairs = t->pairs;
  });
}
