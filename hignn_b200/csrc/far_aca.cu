// Plain FP32 far field: adaptive cross approximation with FP64 bookkeeping.
//
// Restates HignnModel::FarDot (src/FarDot.cpp:64-1696). Each admissible block
// A(i, j) = 0.5 (M + M^T)(x_j - x_i), i in I, j in J, is approximated by
// sum_l C_l(i) Q_l(j) (3x3 blocks) with the reference's rules:
//   * first column |J|/2 (:257); column query, symmetrised 3x3 (:348-458);
//   * C_k -= sum_{l<k} C_l Q_l(jk) (:474-512); row pivot = max signed det over
//     unused rows (:520-576); C_k <- C_k inv(C_k(ik)) by adjugate (:586-656);
//   * row query (:672-781); Q_k -= sum_{l<k} C_l(ik) Q_l (:797-841); next
//     column = max signed det over columns not yet used, current included (:846-903);
//   * nu2 = ||C_k Q_k||_F^2; mu2 += nu2 + sum_{l<k-1} 2 |C_k^T C_l| |Q_k Q_l^T|
//     (:919-1078); stop when nu2 < mu2 eps^2, k >= maxIter or k >= min(|I|,|J|);
//   * apply u_I += sum_l C_l (Q_l f_J), u_J += sum_l Q_l^T (C_l^T f_I) (:1194-1388).
// The reference compacts converged blocks out of its arrays with O(w^2)
// launches; here every block carries its own iteration counter and an active
// list is rebuilt by one CTA per iteration. This file is compiled with
// -fmad=false so the FP64 determinant, inverse and products round as written.
#include <cfloat>

#include "common.h"
#include "kernels.h"
#include "mlp_simt.cuh"

namespace hignn {

namespace {

// Pivot CTAs work on one block at a time through a chain of dependent phases (orthogonalisation,
// argmax, norms, cross terms), so their rate is set by how many blocks are in flight per SM: the
// pivot kernels run 128-thread CTAs capped at 64 registers per thread, eight per SM (357 ms of
// pivots at N = 1M, against 527 ms for 256-thread CTAs at ~126 registers, two per SM; a cap of
// 40 registers spills too much and is slower).
constexpr int kPivThreads = 128;
// FP32 bookkeeping (the fast forms): 64 registers, no spills; 10 or 12 CTAs per SM spill and ran
// slower at N = 1M (287 ms of pivots at 8, 297 at 10, 315 at 12, 337 for the FP64 form)
constexpr int kPivBlocksF32 = 8;
constexpr int kApplyThreads = 256;  // the deferred apply: few phases, wider CTAs

template <typename T>
__device__ __forceinline__ T det3(const T* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

template <typename T>
__device__ __forceinline__ T lowest();
template <>
__device__ __forceinline__ double lowest<double>() { return -DBL_MAX; }
template <>
__device__ __forceinline__ float lowest<float>() { return -FLT_MAX; }

// argmax with the first index winning ties (Kokkos MaxLoc over a strict '>').
template <typename T>
__device__ __forceinline__ void better(T& v, int& i, T v2, int i2) {
  if (i2 >= 0 && (i < 0 || v2 > v || (v2 == v && i2 < i))) {
    v = v2;
    i = i2;
  }
}

template <typename T>
__device__ void block_argmax(T& v, int& i, T* sv, int* si) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    T v2 = __shfl_down_sync(0xffffffffu, v, o);
    int i2 = __shfl_down_sync(0xffffffffu, i, o);
    better(v, i, v2, i2);
  }
  if (lane == 0) {
    sv[wid] = v;
    si[wid] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T bv = sv[0];
    int bi = si[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) better(bv, bi, sv[w], si[w]);
    sv[0] = bv;
    si[0] = bi;
  }
  __syncthreads();
  v = sv[0];
  i = si[0];
  __syncthreads();
}

template <int N, typename T>
__device__ void block_sum(T (&v)[N], T* scratch /* [32][N] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; q++)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < N; q++) scratch[wid * N + q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int q = 0; q < N; q++) {
      T s = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += scratch[w * N + q];
      scratch[q] = s;
    }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < N; q++) v[q] = scratch[q];
  __syncthreads();
}

// block_argmax and block_sum<12> in one pass: the same per-warp and per-CTA orders, two barriers
// instead of six (sv / si / scratch are not written again before the caller's next barrier).
template <typename T>
__device__ void block_argmax_sum(T& best, int& bi, T (&v)[12], T* sv, int* si, T* scratch /* [32][12] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    T v2 = __shfl_down_sync(0xffffffffu, best, o);
    int i2 = __shfl_down_sync(0xffffffffu, bi, o);
    better(best, bi, v2, i2);
  }
#pragma unroll
  for (int q = 0; q < 12; q++)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  if (lane == 0) {
    sv[wid] = best;
    si[wid] = bi;
#pragma unroll
    for (int q = 0; q < 12; q++) scratch[wid * 12 + q] = v[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T bv = sv[0];
    int bj = si[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) better(bv, bj, sv[w], si[w]);
    sv[0] = bv;
    si[0] = bj;
    for (int q = 0; q < 12; q++) {
      T s = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += scratch[w * 12 + q];
      scratch[q] = s;
    }
  }
  __syncthreads();
  best = sv[0];
  bi = si[0];
#pragma unroll
  for (int q = 0; q < 12; q++) v[q] = scratch[q];
}

__global__ void k_far_init(FarArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0) {
    a.ctr[kCtrRemaining] = a.nb;
    a.ctr[kCtrError] = 0;
    a.ctr[kCtrRankMax] = 0;
    a.ctr[kCtrDeferred] = 0;
  }
  if (b >= a.nb) return;
  a.state[b].k = 0;
  a.state[b].done = 0;
  a.state[b].mu2 = 0.0;
  a.state[b].nu2 = 0.0;
  a.cols[(size_t)b * a.ldr] = a.blocks[b].nJ / 2;
}

// Active list and prefix sums of |I| and |J| over active blocks (one CTA).
__global__ void __launch_bounds__(1024) k_far_active(FarArgs a) {
  __shared__ int sA[32], sI[32], sJ[32];
  __shared__ int baseA, baseI, baseJ;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  if (t == 0) baseA = baseI = baseJ = 0;
  __syncthreads();
  for (int b0 = 0; b0 < a.nb; b0 += 1024) {
    const int b = b0 + t;
    const bool act = b < a.nb && !a.state[b].done;
    int vA = act ? 1 : 0, vI = act ? a.blocks[b].nI : 0, vJ = act ? a.blocks[b].nJ : 0;
    int xA = vA, xI = vI, xJ = vJ;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      int yA = __shfl_up_sync(0xffffffffu, xA, o), yI = __shfl_up_sync(0xffffffffu, xI, o),
          yJ = __shfl_up_sync(0xffffffffu, xJ, o);
      if (lane >= o) {
        xA += yA;
        xI += yI;
        xJ += yJ;
      }
    }
    if (lane == 31) {
      sA[wid] = xA;
      sI[wid] = xI;
      sJ[wid] = xJ;
    }
    __syncthreads();
    if (wid == 0) {
      int zA = sA[lane], zI = sI[lane], zJ = sJ[lane];
      for (int o = 1; o < 32; o <<= 1) {
        int yA = __shfl_up_sync(0xffffffffu, zA, o), yI = __shfl_up_sync(0xffffffffu, zI, o),
            yJ = __shfl_up_sync(0xffffffffu, zJ, o);
        if (lane >= o) {
          zA += yA;
          zI += yI;
          zJ += yJ;
        }
      }
      sA[lane] = zA;
      sI[lane] = zI;
      sJ[lane] = zJ;
    }
    __syncthreads();
    const int offA = baseA + (wid ? sA[wid - 1] : 0) + xA - vA;
    const int offI = baseI + (wid ? sI[wid - 1] : 0) + xI - vI;
    const int offJ = baseJ + (wid ? sJ[wid - 1] : 0) + xJ - vJ;
    if (act) {
      a.act[offA] = b;
      a.preI[offA] = offI;
      a.preJ[offA] = offJ;
    }
    __syncthreads();
    if (t == 0) {
      baseA += sA[31];
      baseI += sI[31];
      baseJ += sJ[31];
    }
    __syncthreads();
  }
  if (t == 0) {
    a.preI[baseA] = baseI;
    a.preJ[baseA] = baseJ;
    a.ctr[kCtrActive] = baseA;
    a.ctr[kCtrTotI] = baseI;
    a.ctr[kCtrTotJ] = baseJ;
  }
}

struct EvalSmem {
  simt::Smem mlp;
  int32_t blk[simt::kTile];
  int32_t loc[simt::kTile];
};

// Column (which = 0) or row (which = 1) queries of every active block, 128 per tile.
__global__ void __launch_bounds__(simt::kThreads, 1) k_far_eval(FarArgs a, MlpF32 w, int which) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EvalSmem& s = *reinterpret_cast<EvalSmem*>(smem_raw);
  const int t = threadIdx.x;
  const int nact = a.ctr[kCtrActive];
  const int tot = which ? a.ctr[kCtrTotJ] : a.ctr[kCtrTotI];
  const int32_t* pre = which ? a.preJ : a.preI;
  if ((int)blockIdx.x * simt::kTile >= tot) return;
  simt::load_weights(s.mlp, w);
  for (int tile = blockIdx.x; tile * simt::kTile < tot; tile += gridDim.x) {
    if (t < simt::kTile) {
      const int e = tile * simt::kTile + t;
      if (e < tot) {
        int lo = 0, hi = nact;  // last active index with pre[idx] <= e
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (pre[mid] <= e)
            lo = mid;
          else
            hi = mid;
        }
        const int b = a.act[lo];
        const int loc = e - pre[lo];
        const FarBlock bk = a.blocks[b];
        const int k = a.state[b].k;
        float4 xi, xj;
        if (which == 0) {
          xj = a.x[bk.sJ + a.cols[(size_t)b * a.ldr + k]];
          xi = a.x[bk.sI + loc];
        } else {
          xj = a.x[bk.sJ + loc];
          xi = a.x[bk.sI + a.rows[(size_t)b * a.ldr + k]];
        }
        s.mlp.r[t] = make_float4(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, 0.f);
        s.blk[t] = b;
        s.loc[t] = loc;
      } else {
        s.mlp.r[t] = make_float4(1.f, 0.f, 0.f, 0.f);
        s.blk[t] = -1;
      }
    }
    __syncthreads();
    simt::mlp_tile(s.mlp, w);
    if (t < simt::kTile && s.blk[t] >= 0) {
      const int b = s.blk[t], loc = s.loc[t];
      const FarBlock bk = a.blocks[b];
      const int k = a.state[b].k;
      pool_t* dst = which == 0 ? a.C + 9 * (bk.cOff + (int64_t)k * bk.nI + loc)
                               : a.Q + 9 * (bk.qOff + (int64_t)k * bk.nJ + loc);
      const float* y = s.mlp.y[t];
      // src/FarDot.cpp:445-456: diagonal copied, off-diagonal 0.5 * (float sum)
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          if (r == c)
            dst[3 * r + c] = (double)y[3 * r + c];
          else
            dst[3 * r + c] = 0.5 * (double)__fadd_rn(y[3 * r + c], y[3 * c + r]);
        }
    }
  }
  if (t == 0 && blockIdx.x == 0) atomicAdd(a.evals, (unsigned long long)tot);
}

// Orthogonalise the new column, pick the pivot row, normalise (one CTA per active block).
template <typename T, int MinBlocks>
__global__ void __launch_bounds__(kPivThreads, MinBlocks) k_far_col_pivot(FarArgs a) {
  extern __shared__ __align__(16) double dsm[];
  T* qj = reinterpret_cast<T*>(dsm);  // [k][9]
  __shared__ T sv[32], inv[9];
  __shared__ int si[32];
  const int nact = a.ctr[kCtrActive];
  for (int ai = blockIdx.x; ai < nact; ai += gridDim.x) {
  const int b = a.act[ai];
  const FarBlock bk = a.blocks[b];
  const int k = a.state[b].k;
  const int jk = a.cols[(size_t)b * a.ldr + k];
  for (int q = threadIdx.x; q < 9 * k; q += blockDim.x) {
    const int l = q / 9, e = q - (q / 9) * 9;
    qj[q] = a.Q[9 * (bk.qOff + (int64_t)l * bk.nJ + jk) + e];
  }
  __syncthreads();
  T best = lowest<T>();
  int bi = -1;
  pool_t* Ck = a.C + 9 * (bk.cOff + (int64_t)k * bk.nI);
  for (int i = threadIdx.x; i < bk.nI; i += blockDim.x) {
    T c[9];
#pragma unroll
    for (int q = 0; q < 9; q++) c[q] = Ck[9 * i + q];
    if (k > 0) {
      T s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int l = 0; l < k; l++) {
        const pool_t* cl = a.C + 9 * (bk.cOff + (int64_t)l * bk.nI + i);
        const T* ql = qj + 9 * l;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int cc = 0; cc < 3; cc++)
#pragma unroll
            for (int m = 0; m < 3; m++) s[3 * r + cc] += cl[3 * r + m] * ql[3 * m + cc];
      }
#pragma unroll
      for (int q = 0; q < 9; q++) {  // stored rounded; the pivot search sees the stored value
        c[q] = (T)(pool_t)(c[q] - s[q]);
        Ck[9 * i + q] = (pool_t)c[q];
      }
    }
    const T d = det3(c);
    if (!a.usedRow[bk.rOff + i] && (bi < 0 || d > best)) {
      best = d;
      bi = i;
    }
  }
  block_argmax(best, bi, sv, si);
  if (bi < 0) {  // CTA-uniform
    if (threadIdx.x == 0) {
      a.ctr[kCtrError] = 1;
      a.rows[(size_t)b * a.ldr + k] = 0;
    }
    __syncthreads();
    continue;
  }
  if (threadIdx.x == 0) {
    a.rows[(size_t)b * a.ldr + k] = bi;
    a.usedRow[bk.rOff + bi] = 1;
    const pool_t* m = Ck + 9 * bi;
    const double A = m[0], B = m[1], C = m[2], D = m[3], E = m[4], F = m[5], G = m[6], H = m[7], I = m[8];
    const double det = A * (E * I - F * H) - B * (D * I - F * G) + C * (D * H - E * G);
    inv[0] = (T)((E * I - F * H) / det);
    inv[1] = (T)(-(B * I - C * H) / det);
    inv[2] = (T)((B * F - C * E) / det);
    inv[3] = (T)(-(D * I - F * G) / det);
    inv[4] = (T)((A * I - C * G) / det);
    inv[5] = (T)(-(A * F - C * D) / det);
    inv[6] = (T)((D * H - E * G) / det);
    inv[7] = (T)(-(A * H - B * G) / det);
    inv[8] = (T)((A * E - B * D) / det);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bk.nI; i += blockDim.x) {
    T c[9], o[9];
#pragma unroll
    for (int q = 0; q < 9; q++) c[q] = Ck[9 * i + q];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int cc = 0; cc < 3; cc++) {
        T acc = c[3 * r] * inv[cc];
        acc = acc + c[3 * r + 1] * inv[3 + cc];
        acc = acc + c[3 * r + 2] * inv[6 + cc];
        o[3 * r + cc] = acc;
      }
#pragma unroll
    for (int q = 0; q < 9; q++) Ck[9 * i + q] = o[q];
  }
  __syncthreads();  // shared state is reused by the next active block
  }
}

// u_I += sum_l C_l (Q_l f_J) and, with symmetry, u_J += sum_l Q_l^T (C_l^T f_I) for one
// converged block (src/FarDot.cpp:1225-1387); all threads of the CTA call it.
__device__ void apply_block(const FarArgs& a, const FarBlock& bk, int rank, double* mid, double* mid2) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int l = wid; l < rank; l += blockDim.x >> 5) {
    const pool_t* Ql = a.Q + 9 * (bk.qOff + (int64_t)l * bk.nJ);
    const pool_t* Cl = a.C + 9 * (bk.cOff + (int64_t)l * bk.nI);
    double m[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
    for (int j = lane; j < bk.nJ; j += 32) {
      const float4 fj = a.f[bk.sJ + j];
      const pool_t* q = Ql + 9 * j;
#pragma unroll
      for (int r = 0; r < 3; r++)
        m[r] += q[3 * r] * (double)fj.x + q[3 * r + 1] * (double)fj.y + q[3 * r + 2] * (double)fj.z;
    }
    if (a.use_symmetry)
      for (int i = lane; i < bk.nI; i += 32) {
        const float4 fi = a.f[bk.sI + i];
        const pool_t* c = Cl + 9 * i;
#pragma unroll
        for (int r = 0; r < 3; r++)
          m2[r] += c[r] * (double)fi.x + c[3 + r] * (double)fi.y + c[6 + r] * (double)fi.z;
      }
#pragma unroll
    for (int r = 0; r < 3; r++)
      for (int o = 16; o > 0; o >>= 1) {
        m[r] += __shfl_down_sync(0xffffffffu, m[r], o);
        m2[r] += __shfl_down_sync(0xffffffffu, m2[r], o);
      }
    if (lane == 0)
#pragma unroll
      for (int r = 0; r < 3; r++) {
        mid[3 * l + r] = m[r];
        mid2[3 * l + r] = m2[r];
      }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bk.nI; i += blockDim.x) {
    double acc[3] = {0, 0, 0};
    for (int l = 0; l < rank; l++) {
      const pool_t* c = a.C + 9 * (bk.cOff + (int64_t)l * bk.nI + i);
#pragma unroll
      for (int r = 0; r < 3; r++)
        acc[r] += c[3 * r] * mid[3 * l] + c[3 * r + 1] * mid[3 * l + 1] + c[3 * r + 2] * mid[3 * l + 2];
    }
#pragma unroll
    for (int r = 0; r < 3; r++) atomicAdd(&a.u[3 * (size_t)(bk.sI + i) + r], acc[r]);
  }
  if (a.use_symmetry)
    for (int j = threadIdx.x; j < bk.nJ; j += blockDim.x) {
      double acc[3] = {0, 0, 0};
      for (int l = 0; l < rank; l++) {
        const pool_t* q = a.Q + 9 * (bk.qOff + (int64_t)l * bk.nJ + j);
#pragma unroll
        for (int r = 0; r < 3; r++)
          acc[r] += q[r] * mid2[3 * l] + q[3 + r] * mid2[3 * l + 1] + q[6 + r] * mid2[3 * l + 2];
      }
#pragma unroll
      for (int r = 0; r < 3; r++) atomicAdd(&a.u[3 * (size_t)(bk.sJ + j) + r], acc[r]);
    }
}

// Stopping rule of iteration k (src/FarDot.cpp:1079-1109) and the block's state update, by one
// thread; done_out: the block converged (apply it), rank_out: its rank.
__device__ void stop_test(const FarArgs& a, int b, const FarBlock& bk, int k, int bj, double nu2, double mu2,
                        int& done_out, int& rank_out) {
  const int k1 = k + 1;
  const int mn = bk.nI < bk.nJ ? bk.nI : bk.nJ;
  int done = (nu2 < mu2 * a.eps2) || k1 >= a.max_iter || k1 >= mn;
  if (!done && bj < 0) {  // no unused column left: cannot continue
    done = 1;
    a.ctr[kCtrError] = 2;
  }
  a.state[b].nu2 = nu2;
  a.state[b].mu2 = mu2;
  a.state[b].k = k1;
  if (k1 < a.ldr) a.cols[(size_t)b * a.ldr + k1] = bj < 0 ? 0 : bj;
  int deferred = 0;
  if (!done && k1 >= bk.kcap) {  // the next term would not fit this block's pool share
    deferred = 1;
    a.state[b].done = 2;
    atomicSub(&a.ctr[kCtrRemaining], 1);
    atomicAdd(&a.ctr[kCtrDeferred], 1);
  }
  if (done) {
    a.state[b].done = 1;
    atomicSub(&a.ctr[kCtrRemaining], 1);
    atomicMax(&a.ctr[kCtrRankMax], k1);
    atomicAdd(a.rank_sum, (unsigned long long)k1);
    if (a.rank_out) a.rank_out[bk.list_idx] = k1;
  }
  done_out = done && !deferred;
  rank_out = k1;
}

// Orthogonalise the new row, pick the next column, stop test, and apply a finished block.
template <typename T, int MinBlocks>
__global__ void __launch_bounds__(kPivThreads, MinBlocks) k_far_row_pivot(FarArgs a) {
  extern __shared__ __align__(16) double dsm[];
  T* ci = reinterpret_cast<T*>(dsm);  // [k][9]
  double* mid = dsm + 9 * a.ldr;      // [rank][3]
  double* mid2 = mid + 3 * a.ldr;     // [rank][3]
  __shared__ T sv[32], cross[8][18], red[32 * 12];
  __shared__ int si[32];
  __shared__ int s_done, s_rank;
  const int nact = a.ctr[kCtrActive];
  for (int ai = blockIdx.x; ai < nact; ai += gridDim.x) {
  const int b = a.act[ai];
  const FarBlock bk = a.blocks[b];
  const int k = a.state[b].k;
  const int ik = a.rows[(size_t)b * a.ldr + k];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = threadIdx.x; q < 9 * k; q += blockDim.x) {
    const int l = q / 9, e = q - (q / 9) * 9;
    ci[q] = a.C[9 * (bk.cOff + (int64_t)l * bk.nI + ik) + e];
  }
  if (threadIdx.x == 0) a.usedCol[bk.colOff + a.cols[(size_t)b * a.ldr + k]] = 1;
  __syncthreads();
  T best = lowest<T>();
  int bj = -1;
  pool_t* Qk = a.Q + 9 * (bk.qOff + (int64_t)k * bk.nJ);
  // nu2 = ||C_k Q_k||_F^2 from column norms/dots of C_k (v[0..5]) and row norms/dots of Q_k
  // (v[6..11], accumulated as each row of Q_k is finished)
  T v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int j = threadIdx.x; j < bk.nJ; j += blockDim.x) {
    T q[9];
#pragma unroll
    for (int e = 0; e < 9; e++) q[e] = Qk[9 * j + e];
    if (k > 0) {
      T s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int l = 0; l < k; l++) {
        const pool_t* ql = a.Q + 9 * (bk.qOff + (int64_t)l * bk.nJ + j);
        const T* cl = ci + 9 * l;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int cc = 0; cc < 3; cc++)
#pragma unroll
            for (int m = 0; m < 3; m++) s[3 * r + cc] += cl[3 * r + m] * ql[3 * m + cc];
      }
#pragma unroll
      for (int e = 0; e < 9; e++) {  // stored rounded; the pivot search sees the stored value
        q[e] = (T)(pool_t)(q[e] - s[e]);
        Qk[9 * j + e] = (pool_t)q[e];
      }
    }
    v[6] += q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    v[7] += q[3] * q[3] + q[4] * q[4] + q[5] * q[5];
    v[8] += q[6] * q[6] + q[7] * q[7] + q[8] * q[8];
    v[9] += q[0] * q[3] + q[1] * q[4] + q[2] * q[5];
    v[10] += q[3] * q[6] + q[4] * q[7] + q[5] * q[8];
    v[11] += q[6] * q[0] + q[7] * q[1] + q[8] * q[2];
    const T d = det3(q);
    if (!a.usedCol[bk.colOff + j] && (bj < 0 || d > best)) {
      best = d;
      bj = j;
    }
  }
  const pool_t* Ck = a.C + 9 * (bk.cOff + (int64_t)k * bk.nI);
  for (int i = threadIdx.x; i < bk.nI; i += blockDim.x) {
    T c[9];
#pragma unroll
    for (int e = 0; e < 9; e++) c[e] = Ck[9 * i + e];
#pragma unroll
    for (int cc = 0; cc < 3; cc++) {
      v[cc] += c[cc] * c[cc] + c[cc + 3] * c[cc + 3] + c[cc + 6] * c[cc + 6];
      const int c1 = (cc + 1) % 3;
      v[3 + cc] += c[cc] * c[c1] + c[cc + 3] * c[c1 + 3] + c[cc + 6] * c[c1 + 6];
    }
  }
  // one reduction for the column pivot and the twelve sums (its barriers also make the Q_k
  // writes visible to the cross terms below)
  block_argmax_sum(best, bj, v, sv, si, red);
  const double nu2 = (T)(v[0] * v[6] + v[1] * v[7] + v[2] * v[8] + T(2) * v[9] * v[3] + T(2) * v[10] * v[4] +
                        T(2) * v[11] * v[5]);
  double mu2 = a.state[b].mu2 + nu2;  // every thread tracks the same value; thread 0 stores it
  // cross terms for l < k - 1 (src/FarDot.cpp:1041-1077), eight l per pass, one warp per l
  const int nw = blockDim.x >> 5;  // at most 8 (cross)
  for (int lb = 0; lb < k - 1; lb += nw) {
    const int l = lb + wid;
    if (l < k - 1) {
      T acc[18];
#pragma unroll
      for (int q = 0; q < 18; q++) acc[q] = 0.0;
      const pool_t* Cl = a.C + 9 * (bk.cOff + (int64_t)l * bk.nI);
      const pool_t* Ql = a.Q + 9 * (bk.qOff + (int64_t)l * bk.nJ);
      for (int i = lane; i < bk.nI; i += 32) {
        T c[9], d[9];
#pragma unroll
        for (int e = 0; e < 9; e++) {
          c[e] = Ck[9 * i + e];
          d[e] = Cl[9 * i + e];
        }
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
          for (int d2 = 0; d2 < 3; d2++)
            acc[3 * d1 + d2] += c[d1] * d[d2] + c[d1 + 3] * d[d2 + 3] + c[d1 + 6] * d[d2 + 6];
      }
      for (int j = lane; j < bk.nJ; j += 32) {
        T q[9], p[9];
#pragma unroll
        for (int e = 0; e < 9; e++) {
          q[e] = Qk[9 * j + e];
          p[e] = Ql[9 * j + e];
        }
#pragma unroll
        for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
          for (int d2 = 0; d2 < 3; d2++)
            acc[9 + 3 * d1 + d2] += q[3 * d1] * p[3 * d2] + q[3 * d1 + 1] * p[3 * d2 + 1] +
                                    q[3 * d1 + 2] * p[3 * d2 + 2];
      }
#pragma unroll
      for (int q = 0; q < 18; q++)
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
      if (lane == 0)
#pragma unroll
        for (int q = 0; q < 18; q++) cross[wid][q] = acc[q];
    }
    __syncthreads();
    for (int ww = 0; ww < nw && lb + ww < k - 1; ww++)
      for (int q = 0; q < 9; q++) mu2 += 2.0 * fabs(cross[ww][q]) * fabs(cross[ww][9 + q]);
    __syncthreads();
  }
  if (threadIdx.x == 0) stop_test(a, b, bk, k, bj, nu2, mu2, s_done, s_rank);
  __syncthreads();
  if (!s_done) continue;  // CTA-uniform; the loop-end barrier protects the shared state
  if (!a.defer_apply) apply_block(a, bk, s_rank, mid, mid2);
  __syncthreads();
  }
}

// ---------------------------------------------------------------- FP32 bookkeeping (fast forms)
// The pivot kernels of the fast forms keep the orthogonalisation, the pivot search and the
// stopping norms in FP32 and read every earlier factor once per iteration. The |.| cross terms of
// the stopping norm (column d1 of C_k . column d2 of C_l and row d1 of Q_k . row d2 of Q_l, for
// l < k - 1; src/FarDot.cpp:1036-1078) are summed chunk by chunk (128 entries) right after the
// orthogonalisation of the same entries: the new entries are staged in shared memory and the
// earlier factors, just read, come from L1 / L2; one warp per l. The C side is summed in the
// column kernel on the orthogonalised column and mapped through the pivot inverse (C_k = c inv,
// so column d1 of C_k is sum_e inv[e][d1] column e of c); it reaches the row kernel of the same
// iteration through the block's scratch at FarBlock::xOff: [0, 6) the column norms and
// adjacent-column dots of C_k, [kXcHead + 9 l, + 9) the cross terms with C_l.

__device__ __forceinline__ void warp_sum9(float (&v)[9]) {
#pragma unroll
  for (int q = 0; q < 9; q++)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
}

size_t col_smem_f32(int ldr) { return sizeof(float) * (18 * (size_t)ldr + 9 * kPivThreads); }
size_t row_smem_f32(int ldr) { return sizeof(double) * 6 * (size_t)ldr + col_smem_f32(ldr); }

__global__ void __launch_bounds__(kPivThreads, kPivBlocksF32) k_far_col_pivot_f32(FarArgs a) {
  extern __shared__ __align__(16) float fsm[];
  float* qj = fsm;             // [k][9]: Q_l[j_k]
  float* xo = qj + 9 * a.ldr;  // [k - 1][9]: cross terms of the orthogonalised column with C_l
  float* cs = xo + 9 * a.ldr;  // [128][9]: the chunk's orthogonalised entries
  __shared__ float sv[32], inv[9], red[32 * 6];
  __shared__ int si[32];
  const int nact = a.ctr[kCtrActive];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int ai = blockIdx.x; ai < nact; ai += gridDim.x) {
    const int b = a.act[ai];
    const FarBlock bk = a.blocks[b];
    const int k = a.state[b].k;
    const int jk = a.cols[(size_t)b * a.ldr + k];
    const int ncross = k > 1 ? k - 1 : 0;
    for (int q = threadIdx.x; q < 9 * k; q += blockDim.x) {
      const int l = q / 9, e = q - (q / 9) * 9;
      qj[q] = a.Q[9 * (bk.qOff + (int64_t)l * bk.nJ + jk) + e];
    }
    for (int q = threadIdx.x; q < 9 * ncross; q += blockDim.x) xo[q] = 0.f;
    __syncthreads();
    float best = -FLT_MAX;
    int bi = -1;
    pool_t* Ck = a.C + 9 * (bk.cOff + (int64_t)k * bk.nI);
    for (int i0 = 0; i0 < bk.nI; i0 += blockDim.x) {
      const int i = i0 + threadIdx.x;
      if (i < bk.nI) {
        float c[9];
#pragma unroll
        for (int q = 0; q < 9; q++) c[q] = Ck[9 * i + q];
        if (k > 0) {
          float s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          for (int l = 0; l < k; l++) {
            const pool_t* cl = a.C + 9 * (bk.cOff + (int64_t)l * bk.nI + i);
            const float* ql = qj + 9 * l;
            float cv[9];
#pragma unroll
            for (int q = 0; q < 9; q++) cv[q] = cl[q];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
              for (int cc = 0; cc < 3; cc++)
#pragma unroll
                for (int m = 0; m < 3; m++) s[3 * r + cc] += cv[3 * r + m] * ql[3 * m + cc];
          }
#pragma unroll
          for (int q = 0; q < 9; q++) {
            c[q] = c[q] - s[q];
            Ck[9 * i + q] = c[q];
          }
        }
        const float d = det3(c);
        if (!a.usedRow[bk.rOff + i] && (bi < 0 || d > best)) {
          best = d;
          bi = i;
        }
        if (ncross > 0)
#pragma unroll
          for (int q = 0; q < 9; q++) cs[9 * threadIdx.x + q] = c[q];
      }
      if (ncross > 0) {  // CTA-uniform
        __syncthreads();
        const int cnt = bk.nI - i0 < (int)blockDim.x ? bk.nI - i0 : (int)blockDim.x;
        for (int l = wid; l < ncross; l += nw) {
          float acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          const pool_t* Cl = a.C + 9 * (bk.cOff + (int64_t)l * bk.nI + i0);
          for (int r = lane; r < cnt; r += 32) {
            const float* c = cs + 9 * r;
            float dv[9];
#pragma unroll
            for (int q = 0; q < 9; q++) dv[q] = Cl[9 * r + q];
#pragma unroll
            for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
              for (int d2 = 0; d2 < 3; d2++)
                acc[3 * d1 + d2] += c[d1] * dv[d2] + c[d1 + 3] * dv[d2 + 3] + c[d1 + 6] * dv[d2 + 6];
          }
          warp_sum9(acc);
          if (lane == 0)
#pragma unroll
            for (int q = 0; q < 9; q++) xo[9 * l + q] += acc[q];
        }
        __syncthreads();
      }
    }
    block_argmax(best, bi, sv, si);
    if (bi < 0) {  // CTA-uniform
      if (threadIdx.x == 0) {
        a.ctr[kCtrError] = 1;
        a.rows[(size_t)b * a.ldr + k] = 0;
      }
      __syncthreads();
      continue;
    }
    if (threadIdx.x == 0) {
      a.rows[(size_t)b * a.ldr + k] = bi;
      a.usedRow[bk.rOff + bi] = 1;
      const pool_t* m = Ck + 9 * bi;
      const double A = m[0], B = m[1], C = m[2], D = m[3], E = m[4], F = m[5], G = m[6], H = m[7], I = m[8];
      const double det = A * (E * I - F * H) - B * (D * I - F * G) + C * (D * H - E * G);
      inv[0] = (float)((E * I - F * H) / det);
      inv[1] = (float)(-(B * I - C * H) / det);
      inv[2] = (float)((B * F - C * E) / det);
      inv[3] = (float)(-(D * I - F * G) / det);
      inv[4] = (float)((A * I - C * G) / det);
      inv[5] = (float)(-(A * F - C * D) / det);
      inv[6] = (float)((D * H - E * G) / det);
      inv[7] = (float)(-(A * H - B * G) / det);
      inv[8] = (float)((A * E - B * D) / det);
    }
    __syncthreads();
    float* xc = a.xc + bk.xOff;
    for (int q = threadIdx.x; q < 9 * ncross; q += blockDim.x) {  // cross terms of the final C_k
      const int l = q / 9, e = q - (q / 9) * 9, d1 = e / 3, d2 = e - (e / 3) * 3;
      const float* x = xo + 9 * l;
      xc[kXcHead + q] = inv[d1] * x[d2] + inv[3 + d1] * x[3 + d2] + inv[6 + d1] * x[6 + d2];
    }
    float v[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < bk.nI; i += blockDim.x) {
      float c[9], o[9];
#pragma unroll
      for (int q = 0; q < 9; q++) c[q] = Ck[9 * i + q];
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
          float acc = c[3 * r] * inv[cc];
          acc = acc + c[3 * r + 1] * inv[3 + cc];
          acc = acc + c[3 * r + 2] * inv[6 + cc];
          o[3 * r + cc] = acc;
        }
#pragma unroll
      for (int q = 0; q < 9; q++) Ck[9 * i + q] = o[q];
#pragma unroll
      for (int cc = 0; cc < 3; cc++) {  // column norms and adjacent-column dots of the final C_k
        const int c1 = (cc + 1) % 3;
        v[cc] += o[cc] * o[cc] + o[cc + 3] * o[cc + 3] + o[cc + 6] * o[cc + 6];
        v[3 + cc] += o[cc] * o[c1] + o[cc + 3] * o[c1 + 3] + o[cc + 6] * o[c1 + 6];
      }
    }
    block_sum<6>(v, red);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < 6; q++) xc[q] = v[q];
    __syncthreads();  // shared state is reused by the next active block
  }
}

__global__ void __launch_bounds__(kPivThreads, kPivBlocksF32) k_far_row_pivot_f32(FarArgs a) {
  extern __shared__ __align__(16) double dsm[];
  double* mid = dsm;                                       // [rank][3] (apply)
  double* mid2 = mid + 3 * a.ldr;                          // [rank][3]
  float* ci = reinterpret_cast<float*>(mid2 + 3 * a.ldr);  // [k][9]: C_l[i_k]
  float* xq = ci + 9 * a.ldr;                              // [k - 1][9]: cross terms of Q_k with Q_l
  float* qs = xq + 9 * a.ldr;                              // [128][9]: the chunk's orthogonalised entries
  __shared__ float sv[32], red[32 * 6];
  __shared__ int si[32];
  __shared__ int s_done, s_rank;
  const int nact = a.ctr[kCtrActive];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int ai = blockIdx.x; ai < nact; ai += gridDim.x) {
    const int b = a.act[ai];
    const FarBlock bk = a.blocks[b];
    const int k = a.state[b].k;
    const int ik = a.rows[(size_t)b * a.ldr + k];
    const int ncross = k > 1 ? k - 1 : 0;
    for (int q = threadIdx.x; q < 9 * k; q += blockDim.x) {
      const int l = q / 9, e = q - (q / 9) * 9;
      ci[q] = a.C[9 * (bk.cOff + (int64_t)l * bk.nI + ik) + e];
    }
    for (int q = threadIdx.x; q < 9 * ncross; q += blockDim.x) xq[q] = 0.f;
    if (threadIdx.x == 0) a.usedCol[bk.colOff + a.cols[(size_t)b * a.ldr + k]] = 1;
    __syncthreads();
    float best = -FLT_MAX;
    int bj = -1;
    float v[6] = {0, 0, 0, 0, 0, 0};  // row norms and adjacent-row dots of Q_k
    pool_t* Qk = a.Q + 9 * (bk.qOff + (int64_t)k * bk.nJ);
    for (int j0 = 0; j0 < bk.nJ; j0 += blockDim.x) {
      const int j = j0 + threadIdx.x;
      if (j < bk.nJ) {
        float q[9];
#pragma unroll
        for (int e = 0; e < 9; e++) q[e] = Qk[9 * j + e];
        if (k > 0) {
          float s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          for (int l = 0; l < k; l++) {
            const pool_t* ql = a.Q + 9 * (bk.qOff + (int64_t)l * bk.nJ + j);
            const float* cl = ci + 9 * l;
            float qv[9];
#pragma unroll
            for (int e = 0; e < 9; e++) qv[e] = ql[e];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
              for (int cc = 0; cc < 3; cc++)
#pragma unroll
                for (int m = 0; m < 3; m++) s[3 * r + cc] += cl[3 * r + m] * qv[3 * m + cc];
          }
#pragma unroll
          for (int e = 0; e < 9; e++) {
            q[e] = q[e] - s[e];
            Qk[9 * j + e] = q[e];
          }
        }
        v[0] += q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        v[1] += q[3] * q[3] + q[4] * q[4] + q[5] * q[5];
        v[2] += q[6] * q[6] + q[7] * q[7] + q[8] * q[8];
        v[3] += q[0] * q[3] + q[1] * q[4] + q[2] * q[5];
        v[4] += q[3] * q[6] + q[4] * q[7] + q[5] * q[8];
        v[5] += q[6] * q[0] + q[7] * q[1] + q[8] * q[2];
        const float d = det3(q);
        if (!a.usedCol[bk.colOff + j] && (bj < 0 || d > best)) {
          best = d;
          bj = j;
        }
        if (ncross > 0)
#pragma unroll
          for (int e = 0; e < 9; e++) qs[9 * threadIdx.x + e] = q[e];
      }
      if (ncross > 0) {  // CTA-uniform
        __syncthreads();
        const int cnt = bk.nJ - j0 < (int)blockDim.x ? bk.nJ - j0 : (int)blockDim.x;
        for (int l = wid; l < ncross; l += nw) {
          float acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
          const pool_t* Ql = a.Q + 9 * (bk.qOff + (int64_t)l * bk.nJ + j0);
          for (int r = lane; r < cnt; r += 32) {
            const float* q = qs + 9 * r;
            float p[9];
#pragma unroll
            for (int e = 0; e < 9; e++) p[e] = Ql[9 * r + e];
#pragma unroll
            for (int d1 = 0; d1 < 3; d1++)
#pragma unroll
              for (int d2 = 0; d2 < 3; d2++)
                acc[3 * d1 + d2] += q[3 * d1] * p[3 * d2] + q[3 * d1 + 1] * p[3 * d2 + 1] + q[3 * d1 + 2] * p[3 * d2 + 2];
          }
          warp_sum9(acc);
          if (lane == 0)
#pragma unroll
            for (int e = 0; e < 9; e++) xq[9 * l + e] += acc[e];
        }
        __syncthreads();
      }
    }
    block_argmax(best, bj, sv, si);
    block_sum<6>(v, red);
    const float* xc = a.xc + bk.xOff;  // written by this iteration's column kernel
    const double nu2 = (float)(xc[0] * v[0] + xc[1] * v[1] + xc[2] * v[2] + 2.f * v[3] * xc[3] + 2.f * v[4] * xc[4] +
                               2.f * v[5] * xc[5]);
    double mu2 = a.state[b].mu2 + nu2;  // every thread tracks the same value; thread 0 stores it
    for (int l = 0; l < ncross; l++)
      for (int e = 0; e < 9; e++) mu2 += 2.0 * fabs((double)xc[kXcHead + 9 * l + e]) * fabs((double)xq[9 * l + e]);
    if (threadIdx.x == 0) stop_test(a, b, bk, k, bj, nu2, mu2, s_done, s_rank);
    __syncthreads();
    if (!s_done) continue;  // CTA-uniform; the loop-end barrier protects the shared state
    if (!a.defer_apply) apply_block(a, bk, s_rank, mid, mid2);
    __syncthreads();
  }
}

// Applies every converged block of the batch (state done == 1): the student path defers the
// apply until the sampled residual check has accepted the block.
__global__ void __launch_bounds__(kApplyThreads) k_far_apply(FarArgs a) {
  extern __shared__ __align__(16) double dsm[];
  double* mid = dsm;
  double* mid2 = dsm + 3 * a.ldr;
  for (int b = blockIdx.x; b < a.nb; b += gridDim.x) {
    if (a.state[b].done != 1) continue;  // CTA-uniform
    const FarBlock bk = a.blocks[b];
    apply_block(a, bk, a.state[b].k, mid, mid2);
    __syncthreads();
  }
}

__device__ __forceinline__ uint64_t mix_hash(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// kFarSamples entries (i, j) per converged block, drawn by a hash of the block's far-list
// position: features x_j - x_i for the teacher / student residual check.
__global__ void k_far_samples(FarArgs a, float* __restrict__ feat) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)a.nb * kFarSamples) return;
  const int b = (int)(g / kFarSamples), q = (int)(g % kFarSamples);
  const FarBlock bk = a.blocks[b];
  const uint64_t h = mix_hash(((uint64_t)bk.list_idx << 8) ^ (uint64_t)q);
  const int i = (int)((h & 0xffffffffull) % (uint64_t)bk.nI), j = (int)((h >> 32) % (uint64_t)bk.nJ);
  const float4 xi = a.x[bk.sI + i], xj = a.x[bk.sJ + j];
  feat[3 * g] = xj.x - xi.x;
  feat[3 * g + 1] = xj.y - xi.y;
  feat[3 * g + 2] = xj.z - xi.z;
}

// One warp per block: relative Frobenius residual of the student against the teacher over the
// block's samples (symmetrised 3x3 blocks, as the far field uses them). A converged block whose
// residual exceeds tol is marked for the teacher (done = 3).
__global__ void k_far_check(FarArgs a, const float* __restrict__ yt, const float* __restrict__ ys, float tol2,
                            int* nfail) {
  const int lane = threadIdx.x & 31;
  const int b = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (b >= a.nb) return;
  if (a.state[b].done != 1) return;  // warp-uniform
  float e2 = 0.f, t2 = 0.f;
  for (int q = lane; q < kFarSamples; q += 32) {
    const float* t = yt + 9 * ((int64_t)b * kFarSamples + q);
    const float* st = ys + 9 * ((int64_t)b * kFarSamples + q);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float tv = 0.5f * (t[3 * r + c] + t[3 * c + r]);
        const float sv = 0.5f * (st[3 * r + c] + st[3 * c + r]);
        e2 += (sv - tv) * (sv - tv);
        t2 += tv * tv;
      }
  }
  for (int o = 16; o > 0; o >>= 1) {
    e2 += __shfl_down_sync(0xffffffffu, e2, o);
    t2 += __shfl_down_sync(0xffffffffu, t2, o);
  }
  if (lane == 0 && !(e2 <= tol2 * t2)) {
    a.state[b].done = 3;
    atomicAdd(nfail, 1);
  }
}

}  // namespace

cudaEvent_t FarTimer::next() {
  if (used == ev.size()) {
    cudaEvent_t e;
    HIGNN_CUDA(cudaEventCreate(&e));
    ev.push_back(e);
  }
  return ev[used++];
}

// events are recorded in groups of six per iteration: before the active list, after it, after
// the column query, after the column pivot, after the row query, after the row pivot
void FarTimer::collect() {
  for (size_t g = 0; g + 6 <= used; g += 6) {
    float t[5];
    for (int q = 0; q < 5; q++) HIGNN_CUDA(cudaEventElapsedTime(&t[q], ev[g + q], ev[g + q + 1]));
    active_ms += t[0];
    query_ms += t[1] + t[3];
    pivot_ms += t[2] + t[4];
  }
  used = 0;
}

FarTimer::~FarTimer() {
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

namespace {

// One ACA iteration of every active block of a batch: active list, column queries, column pivot,
// row queries, row pivot (with the stop test and, unless deferred, the apply).
void far_iteration(const FarArgs& a, const MlpF32& w, const TcWeights* tcw, const float* student, int* err,
                   int num_sms, cudaStream_t s, FarTimer* timer) {
  auto mark = [&]() {
    if (timer) HIGNN_CUDA(cudaEventRecord(timer->next(), s));
  };
  const size_t eval_smem = sizeof(EvalSmem);
  const size_t row_smem = sizeof(double) * (9 + 3 + 3) * a.ldr;
  const size_t col_smem = sizeof(double) * 9 * a.ldr;
  const int piv_grid = a.nb < 16 * num_sms ? a.nb : 16 * num_sms;  // grid-stride over active blocks
  mark();
  k_far_active<<<1, 1024, 0, s>>>(a);
  mark();
  if (student)
    launch_far_student(a, student, 0, err, num_sms, s);
  else if (tcw)
    launch_far_tc(a, *tcw, 0, err, num_sms, s);
  else
    k_far_eval<<<num_sms, simt::kThreads, eval_smem, s>>>(a, w, 0);
  mark();
  if (a.fast_pivots)
    k_far_col_pivot_f32<<<piv_grid, kPivThreads, col_smem_f32(a.ldr), s>>>(a);
  else
    k_far_col_pivot<double, 8><<<piv_grid, kPivThreads, col_smem, s>>>(a);
  mark();
  if (student)
    launch_far_student(a, student, 1, err, num_sms, s);
  else if (tcw)
    launch_far_tc(a, *tcw, 1, err, num_sms, s);
  else
    k_far_eval<<<num_sms, simt::kThreads, eval_smem, s>>>(a, w, 1);
  mark();
  if (a.fast_pivots)
    k_far_row_pivot_f32<<<piv_grid, kPivThreads, row_smem_f32(a.ldr), s>>>(a);
  else
    k_far_row_pivot<double, 8><<<piv_grid, kPivThreads, row_smem, s>>>(a);
  mark();
  HIGNN_CHECK_LAUNCH();
}

// Shared-memory attributes and the state of a batch (first column |J|/2, counters).
void far_batch_start(const FarArgs& a, cudaStream_t s) {
  const size_t eval_smem = sizeof(EvalSmem);
  const size_t row_smem = sizeof(double) * (9 + 3 + 3) * a.ldr;
  const size_t col_smem = sizeof(double) * 9 * a.ldr;
  set_max_dynamic_smem(k_far_eval, eval_smem, s);
  set_max_dynamic_smem(k_far_row_pivot<double, 8>, row_smem, s);
  set_max_dynamic_smem(k_far_col_pivot<double, 8>, col_smem, s);
  set_max_dynamic_smem(k_far_row_pivot_f32, row_smem_f32(a.ldr), s);
  set_max_dynamic_smem(k_far_col_pivot_f32, col_smem_f32(a.ldr), s);
  k_far_init<<<(a.nb + 255) / 256, 256, 0, s>>>(a);
  HIGNN_CHECK_LAUNCH();
}

// End of a batch in the graph form: its counters folded into the matvec's status and the blocks
// to rerun (deferred: done 2; sent back to the teacher: done 3) appended to the status lists.
// status: [0] deferred, [1] fallback, [2] pivot error, [3] blocks left unfinished, [4] largest
// rank; lists: deferred far-list positions at [0, cap), fallback ones at [cap, 2 cap).
__global__ void k_batch_end(FarArgs a, int* __restrict__ status, int32_t* __restrict__ lists, int cap) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0) {
    if (a.ctr[kCtrError]) atomicOr(&status[2], a.ctr[kCtrError]);
    atomicAdd(&status[3], a.ctr[kCtrRemaining]);
    atomicMax(&status[4], a.ctr[kCtrRankMax]);
  }
  if (b >= a.nb) return;
  const int d = a.state[b].done;
  if (d == 2 || d == 3) {
    const int q = atomicAdd(&status[d == 2 ? 0 : 1], 1);
    if (q < cap) lists[(d == 2 ? 0 : cap) + q] = a.blocks[b].list_idx;
  }
}

}  // namespace

void far_batch_launch(const FarArgs& a, const MlpF32& w, const TcWeights* tcw, const float* student, int* err,
                      int num_sms, cudaStream_t s, int iters) {
  if (a.nb <= 0) return;
  far_batch_start(a, s);
  for (int q = 0; q < iters; q++) far_iteration(a, w, tcw, student, err, num_sms, s, nullptr);
}

void far_batch_end(const FarArgs& a, int* status, int32_t* lists, int cap, cudaStream_t s) {
  if (a.nb <= 0) return;
  k_batch_end<<<(a.nb + 255) / 256, 256, 0, s>>>(a, status, lists, cap);
  HIGNN_CHECK_LAUNCH();
}

int far_batch_plain(const FarArgs& a, const MlpF32& w, const TcWeights* tcw, const float* student, int* err,
                    int num_sms, int32_t* host_ctr, cudaStream_t s, int known_iters, int* iterations,
                    FarTimer* timer) {
  if (a.nb <= 0) return 0;
  far_batch_start(a, s);
  // Without a known bound the counters are read back every kCheck iterations; the kernels of
  // an iteration with no active block return at once.
  constexpr int kCheck = 4;
  const int limit = known_iters > 0 ? known_iters : a.max_iter + 1;
  int it = 0;
  bool finished = false;
  while (it < limit && !finished) {
    const int span = known_iters > 0 ? limit : (it + kCheck < limit ? kCheck : limit - it);
    for (int q = 0; q < span; q++, it++) far_iteration(a, w, tcw, student, err, num_sms, s, timer);
    HIGNN_CUDA(cudaMemcpyAsync(host_ctr, a.ctr, sizeof(int32_t) * kCtrCount, cudaMemcpyDeviceToHost, s));
    HIGNN_CUDA(cudaStreamSynchronize(s));
    if (timer) timer->collect();
    if (host_ctr[kCtrError] != 0)
      throw Error(-5, "ACA: pivot search found no unused row/column (non-finite block entries?)");
    finished = host_ctr[kCtrRemaining] == 0;
  }
  if (!finished) throw Error(-5, "ACA did not converge within max_iter iterations");
  if (iterations) *iterations += it;
  return host_ctr[kCtrDeferred];
}

void far_student_check_launch(const FarArgs& a, const TcWeights& tcw, const float* student, float tol, float* feat,
                              float* yt, float* ys, int* nfail_dev, int* err, int num_sms, cudaStream_t s) {
  if (a.nb <= 0) return;
  const int64_t ns = (int64_t)a.nb * kFarSamples;
  HIGNN_CUDA(cudaMemsetAsync(nfail_dev, 0, sizeof(int), s));
  k_far_samples<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(a, feat);
  HIGNN_CHECK_LAUNCH();
  launch_student_eval(student, feat, ys, ns, num_sms, s);
  launch_eval_tc(feat, yt, ns, tcw, err, num_sms, s);
  k_far_check<<<(unsigned)((a.nb * 32 + 255) / 256), 256, 0, s>>>(a, yt, ys, tol * tol, nfail_dev);
  HIGNN_CHECK_LAUNCH();
  const size_t smem = sizeof(double) * 6 * a.ldr;
  const int grid = a.nb < 8 * num_sms ? a.nb : 8 * num_sms;
  k_far_apply<<<grid, kApplyThreads, smem, s>>>(a);
  HIGNN_CHECK_LAUNCH();
}

int far_student_check(const FarArgs& a, const TcWeights& tcw, const float* student, float tol, float* feat, float* yt,
                      float* ys, int* nfail_dev, int* err, int num_sms, cudaStream_t s) {
  if (a.nb <= 0) return 0;
  far_student_check_launch(a, tcw, student, tol, feat, yt, ys, nfail_dev, err, num_sms, s);
  int nfail = 0;
  HIGNN_CUDA(cudaMemcpyAsync(&nfail, nfail_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
  HIGNN_CUDA(cudaStreamSynchronize(s));
  return nfail;
}

}  // namespace hignn
