// Cluster tree on the device: the divisions of HignnModel::Divide (src/HignnModel.cpp:119-198)
// for all nodes of a level at once, driven by the host build's level loop (build_tree_rows,
// src/Build.cpp:17-265), giving the same rows and permutation as the host build bit for bit.
//
// Per level (the nodes to divide, all larger than the leaf size):
//   k_block_mean : one thread per block of kSumBlock consecutive particles of a node: the block's
//                  sequential FP32 coordinate sums;
//   k_node_mean  : one thread per node: sequential sum of its block sums, mean = sum / L;
//   k_block_cov  : one thread per block: centred coordinates (FP32) and the six FP64 products,
//                  summed sequentially;
//   k_node_axis  : one thread per node: sequential sum of the block sums, cyclic Jacobi on the
//                  3x3 covariance, the dominant axis rounded to FP32;
//   k_project    : one thread per particle: projection on the axis, a 64-bit sort key
//                  (node rank, order-preserving image of the projection), the count of
//                  projections <= 0 per node (the split: upper_bound(t, 0));
//   CUB radix sort of the keys (stable: equal projections keep their order, as the host's
//   stable sort does), then k_apply_order permutes the particle order and the positions.
// The positions are kept in the current particle order (x_t[i] = x[perm[i]]) so every pass reads
// contiguous memory. Files compiled with -fmad=false: every FP32/FP64 operation rounds as
// written, exactly as the host build compiled with -ffp-contract=off.
#include <cub/cub.cuh>

#include <cfloat>

#include <vector>

#include "../../include/hignn_b200.h"
#include "common.h"
#include "tree.h"
#include "tree_dev.h"
#include "tree_math.h"

namespace hignn {

namespace {

constexpr int kThreads = 128;

__global__ void k_init_order(const float* __restrict__ xyz, int64_t n, float4* __restrict__ xt,
                             int32_t* __restrict__ perm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xt[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.f);
  perm[i] = (int32_t)i;
}

// Block b covers particles [bstart[b], bstart[b] + blen[b]) of node bnode[b].
struct LevelArgs {
  int nnodes, nblocks;
  const int32_t* nstart;  // [nnodes]
  const int32_t* nlen;
  const int32_t* nblk0;   // first block of each node
  const int32_t* nnblk;   // blocks of each node
  const int32_t* bstart;  // [nblocks]
  const int32_t* blen;
  const int32_t* boff;    // compact offset of the block's first particle among this level's particles
  const int32_t* bnode;
  float4* bsum;           // [nblocks] FP32 coordinate sums
  double* bcov;           // [nblocks][6]
  float4* nmean;          // [nnodes]
  float4* naxis;          // [nnodes]
  int32_t* ncount;        // [nnodes] projections <= 0
};

__global__ void k_block_mean(LevelArgs a, const float4* __restrict__ xt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nblocks) return;
  const int s = a.bstart[b], L = a.blen[b];
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll 8
  for (int i = 0; i < L; i++) {
    const float4 p = xt[s + i];
    sx = sx + p.x;
    sy = sy + p.y;
    sz = sz + p.z;
  }
  a.bsum[b] = make_float4(sx, sy, sz, 0.f);
}

__global__ void k_node_mean(LevelArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.nnodes) return;
  float mx = 0.f, my = 0.f, mz = 0.f;
  const int b0 = a.nblk0[q], nb = a.nnblk[q];
  for (int b = b0; b < b0 + nb; b++) {
    const float4 s = a.bsum[b];
    mx = mx + s.x;
    my = my + s.y;
    mz = mz + s.z;
  }
  const float L = (float)a.nlen[q];
  a.nmean[q] = make_float4(mx / L, my / L, mz / L, 0.f);
  a.ncount[q] = 0;
}

__global__ void k_block_cov(LevelArgs a, const float4* __restrict__ xt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.nblocks) return;
  const int s = a.bstart[b], L = a.blen[b];
  const float4 m = a.nmean[a.bnode[b]];
  double t00 = 0.0, t01 = 0.0, t02 = 0.0, t11 = 0.0, t12 = 0.0, t22 = 0.0;
#pragma unroll 4
  for (int i = 0; i < L; i++) {
    const float4 p = xt[s + i];
    const double x = (double)(p.x - m.x), y = (double)(p.y - m.y), z = (double)(p.z - m.z);
    t00 = t00 + x * x;
    t01 = t01 + x * y;
    t02 = t02 + x * z;
    t11 = t11 + y * y;
    t12 = t12 + y * z;
    t22 = t22 + z * z;
  }
  double* o = a.bcov + 6 * (size_t)b;
  o[0] = t00;
  o[1] = t01;
  o[2] = t02;
  o[3] = t11;
  o[4] = t12;
  o[5] = t22;
}

__global__ void k_node_axis(LevelArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.nnodes) return;
  double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int b0 = a.nblk0[q], nb = a.nnblk[q];
  for (int b = b0; b < b0 + nb; b++)
    for (int k = 0; k < 6; k++) s[k] = s[k] + a.bcov[6 * (size_t)b + k];
  const double cov[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
  double u[3];
  jacobi_dominant_axis(cov, u);
  a.naxis[q] = make_float4((float)u[0], (float)u[1], (float)u[2], 0.f);
}

// One CTA per block (blen <= kSumBlock particles).
__global__ void k_project(LevelArgs a, const float4* __restrict__ xt, uint64_t* __restrict__ keys,
                          int32_t* __restrict__ vals, int32_t* __restrict__ cpos) {
  const int b = blockIdx.x;
  const int i = threadIdx.x;
  if (i >= a.blen[b]) return;
  const int q = a.bnode[b];
  const int p = a.bstart[b] + i;
  const float4 m = a.nmean[q], u = a.naxis[q], x = xt[p];
  const float t = project_axis(u.x, u.y, u.z, x.x - m.x, x.y - m.y, x.z - m.z);
  const int c = a.boff[b] + i;
  keys[c] = ((uint64_t)(uint32_t)q << 32) | (uint64_t)float_key(t);
  vals[c] = p;
  cpos[c] = p;
  if (!(0.0f < t)) atomicAdd(&a.ncount[q], 1);
}

// The sorted c-th particle of the level goes to position cpos[c] (the level's particles in
// position order; each node's sorted run lands in its own range).
__global__ void k_apply_order(int nact, const int32_t* __restrict__ vals_sorted, const int32_t* __restrict__ cpos,
                              const float4* __restrict__ xt, const int32_t* __restrict__ perm,
                              float4* __restrict__ xt2, int32_t* __restrict__ perm2) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nact) return;
  const int src = vals_sorted[c], dst = cpos[c];
  xt2[dst] = xt[src];
  perm2[dst] = perm[src];
}

// ----------------------------------------------------------------------------------------------
// Close / far lists (ComputeAux + CloseFarCheck, src/CloseFarCheck.cpp:11-465) on the device.

struct ListArgs {
  const int32_t* c0;   // node rows: children, range
  const int32_t* c1;
  const int32_t* st;
  const int32_t* en;
  const float* aux;    // [nn][6] bounding boxes (xmin, xmax, ymin, ymax, zmin, zmax)
  int64_t max_rel;
};

// Bounding box of every node over its whole particle range (one CTA per node; min / max are exact
// in any order, so this equals the host's per-node scan).
__global__ void k_node_aux(const int32_t* __restrict__ nodes, int count, const int32_t* __restrict__ st,
                           const int32_t* __restrict__ en, const float4* __restrict__ xt, float* __restrict__ aux) {
  __shared__ float red[6][32];
  const int q = blockIdx.x;
  if (q >= count) return;
  const int nd = nodes[q];
  float b[6] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
  for (int i = st[nd] + threadIdx.x; i < en[nd]; i += blockDim.x) {
    const float4 p = xt[i];
    b[0] = fminf(b[0], p.x);
    b[1] = fmaxf(b[1], p.x);
    b[2] = fminf(b[2], p.y);
    b[3] = fmaxf(b[3], p.y);
    b[4] = fminf(b[4], p.z);
    b[5] = fmaxf(b[5], p.z);
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 6; k++) {
      const float v = __shfl_down_sync(0xffffffffu, b[k], o);
      b[k] = (k & 1) ? fmaxf(b[k], v) : fminf(b[k], v);
    }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 6; k++) red[k][w] = b[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ww++)
      for (int k = 0; k < 6; k++) b[k] = (k & 1) ? fmaxf(b[k], red[k][ww]) : fminf(b[k], red[k][ww]);
    for (int k = 0; k < 6; k++) aux[6 * (size_t)nd + k] = b[k];
  }
}

// HignnModel::CloseFarCheck(aux, n1, n2), src/HignnModel.cpp:482-518 (the host's is_far, the same
// FP32 operations in the same order).
__device__ __forceinline__ bool dev_is_far(const float* a, const float* b) {
  if (!(a[0] > b[1] || a[1] < b[0] || a[2] > b[3] || a[3] < b[2] || a[4] > b[5] || a[5] < b[4])) return false;
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

constexpr int kDfsStack = 64;  // the host uses the device lists only for trees less deep than this

// Visit of the nodes of one level (src/CloseFarCheck.cpp:186-290), one thread per node, in two
// passes: WRITE = false counts the far entries and the near list (the children's shared close list
// of an internal node, the final close list of a leaf); WRITE = true writes them at the offsets the
// host computed. Expansions walk the subtree depth first with the host's stack order (children
// pushed 0 then 1, so child 1 is visited first).
template <bool WRITE>
__global__ void k_visit(ListArgs a, int nl, const int32_t* __restrict__ lvl, const int32_t* __restrict__ cl_off,
                        const int32_t* __restrict__ cl_len, const int32_t* __restrict__ near_in,
                        int32_t* __restrict__ far_cnt, int32_t* __restrict__ near_cnt,
                        const int32_t* __restrict__ far_off, const int32_t* __restrict__ near_off,
                        int32_t* __restrict__ far_pool, int32_t* __restrict__ near_pool, int* err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nl) return;
  const int i = lvl[q];
  const float* ai = a.aux + 6 * (size_t)i;
  const bool leaf_i = a.c0[i] == 0;
  const int64_t size_i = a.en[i] - a.st[i];
  int nf = 0, nn = 0;
  int* fo = WRITE ? far_pool + far_off[q] : nullptr;
  int* no = WRITE ? near_pool + near_off[q] : nullptr;
  auto put_far = [&](int j) {
    if (WRITE) fo[nf] = j;
    nf++;
  };
  auto put_near = [&](int j) {
    if (WRITE) no[nn] = j;
    nn++;
  };
  int stk[kDfsStack];
  const int* cl = near_in + cl_off[q];
  const int ncl = cl_len[q];
  for (int e = 0; e < ncl; e++) {
    const int j = cl[e];
    const int64_t size_j = a.en[j] - a.st[j];
    const bool leaf_j = a.c0[j] == 0;
    const bool adm = dev_is_far(ai, a.aux + 6 * (size_t)j);
    if (!leaf_i) {
      if (adm && size_i < a.max_rel && size_j < a.max_rel) {
        put_far(j);
      } else if (!leaf_j) {
        put_near(a.c0[j]);
        put_near(a.c1[j]);
      } else {
        put_near(j);
      }
    } else if (adm) {
      if (size_j < a.max_rel) {
        put_far(j);
      } else {  // size gate: the subtree's nodes below the gate
        int sp = 0;
        stk[sp++] = j;
        while (sp > 0) {
          const int c = stk[--sp];
          if (a.en[c] - a.st[c] < a.max_rel) {
            put_far(c);
          } else if (sp + 2 <= kDfsStack) {
            stk[sp++] = a.c0[c];
            stk[sp++] = a.c1[c];
          } else {
            atomicExch(err, 1);
            sp = 0;
          }
        }
      }
    } else if (leaf_j) {
      put_near(j);
    } else {  // a non-admissible internal node: all its leaves
      int sp = 0;
      stk[sp++] = j;
      while (sp > 0) {
        const int c = stk[--sp];
        if (a.c0[c] != 0) {
          if (sp + 2 <= kDfsStack) {
            stk[sp++] = a.c0[c];
            stk[sp++] = a.c1[c];
          } else {
            atomicExch(err, 1);
            sp = 0;
          }
        } else {
          put_near(c);
        }
      }
    }
  }
  if (!WRITE) {
    far_cnt[q] = nf;
    near_cnt[q] = nn;
  }
}

// Flattening (src/CloseFarCheck.cpp:298-336, 385-408): for each row node i (in the given order)
// the entries j of its segment, those with j >= i only under symmetry. COUNT = true counts.
template <bool COUNT>
__global__ void k_flatten(int nrows, const int32_t* __restrict__ rows, const int32_t* __restrict__ seg_off,
                          const int32_t* __restrict__ seg_len, const int32_t* __restrict__ pool, int sym,
                          int32_t* __restrict__ cnt, const int32_t* __restrict__ out_off, int32_t* __restrict__ outI,
                          int32_t* __restrict__ outJ) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  const int i = rows[r];
  const int* sg = pool + seg_off[r];
  const int len = seg_len[r];
  int k = 0;
  for (int e = 0; e < len; e++) {
    const int j = sg[e];
    if (sym && j < i) continue;
    if (!COUNT) {
      outI[out_off[r] + k] = i;
      outJ[out_off[r] + k] = j;
    }
    k++;
  }
  if (COUNT) cnt[r] = k;
}

}  // namespace

void TreeDevScratch::release() {
  for (DevBuf* b : {&xyz, &xt, &xt2, &perm, &perm2, &keys, &keys2, &vals, &vals2, &cpos, &cub_tmp, &lvl_i32, &lvl_f4,
                    &lvl_f8, &node_i32, &aux, &lst_i32, &near_pool, &far_pool, &flat_i32, &outI, &outJ, &err})
    b->release();
}

namespace {

// Grows a device buffer to `need` bytes keeping its first `used` bytes.
void grow_keep(DevBuf& b, size_t need, size_t used, cudaStream_t st) {
  if (need <= b.bytes && b.p) return;
  DevBuf nb;
  nb.ensure(std::max(need, 2 * b.bytes));
  if (used) HIGNN_CUDA(cudaMemcpyAsync(nb.p, b.p, used, cudaMemcpyDeviceToDevice, st));
  HIGNN_CUDA(cudaStreamSynchronize(st));
  b.release();
  b = nb;
}

// Counts then writes the flattened pairs (i, j) of the rows' segments; returns them on the host.
void flatten(TreeDevScratch& S, const std::vector<int32_t>& rows, const std::vector<int32_t>& off,
             const std::vector<int32_t>& len, const int32_t* pool, bool sym, std::vector<int64_t>& I,
             std::vector<int64_t>& J, cudaStream_t st) {
  const int nr = (int)rows.size();
  I.clear();
  J.clear();
  if (nr == 0) return;
  S.flat_i32.ensure(sizeof(int32_t) * 5 * (size_t)nr);
  int32_t* d = S.flat_i32.as<int32_t>();
  HIGNN_CUDA(cudaMemcpyAsync(d, rows.data(), sizeof(int32_t) * nr, cudaMemcpyHostToDevice, st));
  HIGNN_CUDA(cudaMemcpyAsync(d + nr, off.data(), sizeof(int32_t) * nr, cudaMemcpyHostToDevice, st));
  HIGNN_CUDA(cudaMemcpyAsync(d + 2 * nr, len.data(), sizeof(int32_t) * nr, cudaMemcpyHostToDevice, st));
  k_flatten<true><<<(nr + 127) / 128, 128, 0, st>>>(nr, d, d + nr, d + 2 * nr, pool, sym ? 1 : 0, d + 3 * nr,
                                                    nullptr, nullptr, nullptr);
  HIGNN_CHECK_LAUNCH();
  std::vector<int32_t> cnt(nr), oo(nr);
  HIGNN_CUDA(cudaMemcpyAsync(cnt.data(), d + 3 * nr, sizeof(int32_t) * nr, cudaMemcpyDeviceToHost, st));
  HIGNN_CUDA(cudaStreamSynchronize(st));
  int64_t tot = 0;
  for (int r = 0; r < nr; r++) {
    oo[r] = (int32_t)tot;
    tot += cnt[r];
  }
  if (tot == 0) return;
  if (tot >= (int64_t(1) << 31)) throw Error(HIGNN_ERR_ARG, "device lists: more than 2^31 pairs");
  HIGNN_CUDA(cudaMemcpyAsync(d + 4 * nr, oo.data(), sizeof(int32_t) * nr, cudaMemcpyHostToDevice, st));
  S.outI.ensure(sizeof(int32_t) * tot);
  S.outJ.ensure(sizeof(int32_t) * tot);
  k_flatten<false><<<(nr + 127) / 128, 128, 0, st>>>(nr, d, d + nr, d + 2 * nr, pool, sym ? 1 : 0, nullptr,
                                                     d + 4 * nr, S.outI.as<int32_t>(), S.outJ.as<int32_t>());
  HIGNN_CHECK_LAUNCH();
  std::vector<int32_t> hi(tot), hj(tot);
  HIGNN_CUDA(cudaMemcpyAsync(hi.data(), S.outI.p, sizeof(int32_t) * tot, cudaMemcpyDeviceToHost, st));
  HIGNN_CUDA(cudaMemcpyAsync(hj.data(), S.outJ.p, sizeof(int32_t) * tot, cudaMemcpyDeviceToHost, st));
  HIGNN_CUDA(cudaStreamSynchronize(st));
  I.assign(hi.begin(), hi.end());
  J.assign(hj.begin(), hj.end());
}

}  // namespace

bool build_lists_device(const ClusterTree& t, const float4* d_xt, int64_t max_rel, bool use_symmetry,
                        TreeDevScratch& S, cudaStream_t st, BlockLists& L) {
  const int nn = (int)t.nodes.size();
  // BFS levels from the root (the order of the host's level-by-level traversal)
  std::vector<std::vector<int32_t>> levels;
  std::vector<int32_t> level{0}, next;
  while (!level.empty()) {
    levels.push_back(level);
    next.clear();
    for (int32_t i : level)
      if (t.nodes[i].child0 != 0) {
        next.push_back((int32_t)t.nodes[i].child0);
        next.push_back((int32_t)t.nodes[i].child1);
      }
    level.swap(next);
  }
  if ((int)levels.size() + 2 >= kDfsStack) return false;  // deeper than the expansion stack: host lists
  std::vector<int32_t> rows(4 * (size_t)nn);
  for (int i = 0; i < nn; i++) {
    rows[i] = (int32_t)t.nodes[i].child0;
    rows[nn + i] = (int32_t)t.nodes[i].child1;
    rows[2 * nn + i] = (int32_t)t.nodes[i].start;
    rows[3 * nn + i] = (int32_t)t.nodes[i].end;
  }
  S.node_i32.ensure(sizeof(int32_t) * 4 * (size_t)nn);
  HIGNN_CUDA(cudaMemcpyAsync(S.node_i32.p, rows.data(), sizeof(int32_t) * rows.size(), cudaMemcpyHostToDevice, st));
  ListArgs a;
  a.c0 = S.node_i32.as<int32_t>();
  a.c1 = a.c0 + nn;
  a.st = a.c0 + 2 * nn;
  a.en = a.c0 + 3 * nn;
  a.max_rel = max_rel;
  // bounding boxes of the reachable nodes
  std::vector<int32_t> reach;
  for (const auto& lv : levels) reach.insert(reach.end(), lv.begin(), lv.end());
  S.aux.ensure(sizeof(float) * 6 * (size_t)nn);
  S.lst_i32.ensure(sizeof(int32_t) * std::max<size_t>(reach.size(), 7 * (size_t)nn));
  HIGNN_CUDA(cudaMemcpyAsync(S.lst_i32.p, reach.data(), sizeof(int32_t) * reach.size(), cudaMemcpyHostToDevice, st));
  k_node_aux<<<(int)reach.size(), 256, 0, st>>>(S.lst_i32.as<int32_t>(), (int)reach.size(), a.st, a.en, d_xt,
                                                S.aux.as<float>());
  HIGNN_CHECK_LAUNCH();
  a.aux = S.aux.as<float>();
  S.err.ensure(sizeof(int));
  HIGNN_CUDA(cudaMemsetAsync(S.err.p, 0, sizeof(int), st));
  // the root's close list is {0}
  size_t near_used = 1, far_used = 0;
  grow_keep(S.near_pool, sizeof(int32_t) * 1024, 0, st);
  grow_keep(S.far_pool, sizeof(int32_t) * 1024, 0, st);
  const int32_t zero = 0;
  HIGNN_CUDA(cudaMemcpyAsync(S.near_pool.p, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  std::vector<int32_t> cl_off{0}, cl_len{1};
  std::vector<int32_t> far_seg_off(nn, 0), far_seg_len(nn, 0);
  std::vector<int32_t> leaf_rows, leaf_off, leaf_len;
  std::vector<int32_t> hbuf;
  for (const auto& lv : levels) {
    const int nl = (int)lv.size();
    hbuf.assign(3 * (size_t)nl, 0);
    std::copy(lv.begin(), lv.end(), hbuf.begin());
    std::copy(cl_off.begin(), cl_off.end(), hbuf.begin() + nl);
    std::copy(cl_len.begin(), cl_len.end(), hbuf.begin() + 2 * nl);
    int32_t* d = S.lst_i32.as<int32_t>();  // lvl, cl_off, cl_len, far_cnt, near_cnt, far_off, near_off
    HIGNN_CUDA(cudaMemcpyAsync(d, hbuf.data(), sizeof(int32_t) * 3 * nl, cudaMemcpyHostToDevice, st));
    const int grid = (nl + 127) / 128;
    k_visit<false><<<grid, 128, 0, st>>>(a, nl, d, d + nl, d + 2 * nl, S.near_pool.as<int32_t>(), d + 3 * nl,
                                          d + 4 * nl, nullptr, nullptr, nullptr, nullptr, S.err.as<int>());
    HIGNN_CHECK_LAUNCH();
    std::vector<int32_t> cnt(2 * (size_t)nl);
    HIGNN_CUDA(cudaMemcpyAsync(cnt.data(), d + 3 * nl, sizeof(int32_t) * 2 * nl, cudaMemcpyDeviceToHost, st));
    HIGNN_CUDA(cudaStreamSynchronize(st));
    std::vector<int32_t> offs(2 * (size_t)nl);
    size_t fu = far_used, nu = near_used;
    for (int q = 0; q < nl; q++) {
      offs[q] = (int32_t)fu;
      fu += cnt[q];
      offs[nl + q] = (int32_t)nu;
      nu += cnt[nl + q];
    }
    if (nu >= (size_t(1) << 31) || fu >= (size_t(1) << 31))
      throw Error(HIGNN_ERR_ARG, "device lists: more than 2^31 list entries");
    grow_keep(S.near_pool, sizeof(int32_t) * nu, sizeof(int32_t) * near_used, st);
    grow_keep(S.far_pool, sizeof(int32_t) * std::max<size_t>(fu, 1), sizeof(int32_t) * far_used, st);
    HIGNN_CUDA(cudaMemcpyAsync(d + 5 * nl, offs.data(), sizeof(int32_t) * 2 * nl, cudaMemcpyHostToDevice, st));
    k_visit<true><<<grid, 128, 0, st>>>(a, nl, d, d + nl, d + 2 * nl, S.near_pool.as<int32_t>(), nullptr, nullptr,
                                         d + 5 * nl, d + 6 * nl, S.far_pool.as<int32_t>(), S.near_pool.as<int32_t>(),
                                         S.err.as<int>());
    HIGNN_CHECK_LAUNCH();
    // the next level's close lists: both children of an internal node share its near list
    cl_off.clear();
    cl_len.clear();
    for (int q = 0; q < nl; q++) {
      const int32_t i = lv[q];
      far_seg_off[i] = offs[q];
      far_seg_len[i] = cnt[q];
      if (t.nodes[i].child0 != 0) {
        for (int c = 0; c < 2; c++) {
          cl_off.push_back(offs[nl + q]);
          cl_len.push_back(cnt[nl + q]);
        }
      } else {
        leaf_rows.push_back(i);
        leaf_off.push_back(offs[nl + q]);
        leaf_len.push_back(cnt[nl + q]);
      }
    }
    far_used = fu;
    near_used = nu;
  }
  int herr = 0;
  HIGNN_CUDA(cudaMemcpyAsync(&herr, S.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  HIGNN_CUDA(cudaStreamSynchronize(st));
  if (herr) return false;  // an expansion outgrew its stack: host lists
  L.leaves.assign(leaf_rows.begin(), leaf_rows.end());
  flatten(S, leaf_rows, leaf_off, leaf_len, S.near_pool.as<int32_t>(), use_symmetry, L.closeI, L.closeJ, st);
  std::vector<int32_t> all(nn);
  for (int i = 0; i < nn; i++) all[i] = i;
  flatten(S, all, far_seg_off, far_seg_len, S.far_pool.as<int32_t>(), use_symmetry, L.farI, L.farJ, st);
  L.aux.assign(6 * (size_t)nn, 0.f);
  HIGNN_CUDA(cudaMemcpyAsync(L.aux.data(), S.aux.p, sizeof(float) * 6 * nn, cudaMemcpyDeviceToHost, st));
  HIGNN_CUDA(cudaStreamSynchronize(st));
  std::vector<char> seen(nn, 0);
  for (int32_t i : reach) seen[i] = 1;
  for (int i = 0; i < nn; i++)
    if (!seen[i]) {
      for (int k = 0; k < 6; k++) L.aux[6 * (size_t)i + k] = 0.f;
      L.aux[6 * (size_t)i] = -FLT_MAX;
    }
  return true;
}

ClusterTree build_tree_device(const float* d_xyz, int64_t n, int64_t leaf, TreeDevScratch& S, cudaStream_t st) {
  if (n >= (int64_t(1) << 31)) throw Error(HIGNN_ERR_ARG, "device tree build: n must be below 2^31");
  ClusterTree t;
  S.xt.ensure(sizeof(float4) * n);
  S.xt2.ensure(sizeof(float4) * n);
  S.perm.ensure(sizeof(int32_t) * n);
  S.perm2.ensure(sizeof(int32_t) * n);
  S.keys.ensure(sizeof(uint64_t) * n);
  S.keys2.ensure(sizeof(uint64_t) * n);
  S.vals.ensure(sizeof(int32_t) * n);
  S.vals2.ensure(sizeof(int32_t) * n);
  S.cpos.ensure(sizeof(int32_t) * n);
  k_init_order<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_xyz, n, S.xt.as<float4>(), S.perm.as<int32_t>());
  HIGNN_CHECK_LAUNCH();
  std::vector<int32_t> h_lvl;
  std::vector<int32_t> h_count;
  t.nodes = build_tree_rows(n, leaf, [&](const std::vector<NodeRange>& rg, std::vector<int64_t>& split) {
    const int m = (int)rg.size();
    // block table: per node (start, len, first block, block count), per block (start, len,
    // compact offset, node)
    int nb = 0;
    for (const NodeRange& r : rg) nb += (int)((r.end - r.start + kSumBlock - 1) / kSumBlock);
    h_lvl.assign((size_t)4 * m + 4 * nb, 0);
    int32_t* ns = h_lvl.data();
    int32_t* nl = ns + m;
    int32_t* n0 = nl + m;
    int32_t* nn = n0 + m;
    int32_t* bs = nn + m;
    int32_t* bl = bs + nb;
    int32_t* bo = bl + nb;
    int32_t* bn = bo + nb;
    int b = 0, off = 0;
    for (int q = 0; q < m; q++) {
      const int64_t s0 = rg[q].start, L = rg[q].end - rg[q].start;
      ns[q] = (int32_t)s0;
      nl[q] = (int32_t)L;
      n0[q] = b;
      nn[q] = (int32_t)((L + kSumBlock - 1) / kSumBlock);
      for (int64_t i = 0; i < L; i += kSumBlock) {
        bs[b] = (int32_t)(s0 + i);
        bl[b] = (int32_t)std::min<int64_t>(kSumBlock, L - i);
        bo[b] = off;
        bn[b] = q;
        off += bl[b];
        b++;
      }
    }
    const int nact = off;
    S.lvl_i32.ensure(sizeof(int32_t) * (h_lvl.size() + m));
    S.lvl_f4.ensure(sizeof(float4) * ((size_t)nb + 2 * (size_t)m));
    S.lvl_f8.ensure(sizeof(double) * 6 * (size_t)nb);
    HIGNN_CUDA(cudaMemcpyAsync(S.lvl_i32.p, h_lvl.data(), sizeof(int32_t) * h_lvl.size(), cudaMemcpyHostToDevice, st));
    LevelArgs a;
    a.nnodes = m;
    a.nblocks = nb;
    const int32_t* d = S.lvl_i32.as<int32_t>();
    a.nstart = d;
    a.nlen = d + m;
    a.nblk0 = d + 2 * m;
    a.nnblk = d + 3 * m;
    a.bstart = d + 4 * m;
    a.blen = a.bstart + nb;
    a.boff = a.blen + nb;
    a.bnode = a.boff + nb;
    a.ncount = S.lvl_i32.as<int32_t>() + h_lvl.size();
    a.bsum = S.lvl_f4.as<float4>();
    a.nmean = a.bsum + nb;
    a.naxis = a.nmean + m;
    a.bcov = S.lvl_f8.as<double>();
    const float4* xt = S.xt.as<float4>();
    k_block_mean<<<(nb + kThreads - 1) / kThreads, kThreads, 0, st>>>(a, xt);
    k_node_mean<<<(m + kThreads - 1) / kThreads, kThreads, 0, st>>>(a);
    k_block_cov<<<(nb + kThreads - 1) / kThreads, kThreads, 0, st>>>(a, xt);
    k_node_axis<<<(m + kThreads - 1) / kThreads, kThreads, 0, st>>>(a);
    k_project<<<nb, (int)kSumBlock, 0, st>>>(a, xt, S.keys.as<uint64_t>(), S.vals.as<int32_t>(),
                                            S.cpos.as<int32_t>());
    HIGNN_CHECK_LAUNCH();
    int end_bit = 32;
    while (end_bit < 64 && (uint64_t)(m - 1) >> (end_bit - 32)) end_bit++;
    size_t tmp = 0;
    HIGNN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, S.keys.as<uint64_t>(), S.keys2.as<uint64_t>(),
                                               S.vals.as<int32_t>(), S.vals2.as<int32_t>(), nact, 0, end_bit, st));
    S.cub_tmp.ensure(std::max<size_t>(tmp, 16));
    HIGNN_CUDA(cub::DeviceRadixSort::SortPairs(S.cub_tmp.p, tmp, S.keys.as<uint64_t>(), S.keys2.as<uint64_t>(),
                                               S.vals.as<int32_t>(), S.vals2.as<int32_t>(), nact, 0, end_bit, st));
    // particles outside this level's nodes keep their place
    HIGNN_CUDA(cudaMemcpyAsync(S.xt2.p, S.xt.p, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st));
    HIGNN_CUDA(cudaMemcpyAsync(S.perm2.p, S.perm.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    k_apply_order<<<(nact + 255) / 256, 256, 0, st>>>(nact, S.vals2.as<int32_t>(), S.cpos.as<int32_t>(),
                                                      S.xt.as<float4>(), S.perm.as<int32_t>(), S.xt2.as<float4>(),
                                                      S.perm2.as<int32_t>());
    HIGNN_CHECK_LAUNCH();
    std::swap(S.xt, S.xt2);
    std::swap(S.perm, S.perm2);
    h_count.resize(m);
    HIGNN_CUDA(cudaMemcpyAsync(h_count.data(), a.ncount, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, st));
    HIGNN_CUDA(cudaStreamSynchronize(st));
    split.resize(m);
    for (int q = 0; q < m; q++) split[q] = rg[q].start + h_count[q];
  });
  std::vector<int32_t> perm(n);
  HIGNN_CUDA(cudaMemcpyAsync(perm.data(), S.perm.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  HIGNN_CUDA(cudaStreamSynchronize(st));
  t.perm.assign(perm.begin(), perm.end());
  return t;
}

}  // namespace hignn
