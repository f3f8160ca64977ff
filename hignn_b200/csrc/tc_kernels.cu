// Tensor-core (tcgen05) forms of the near field, the ACA queries and the stand-alone evaluation.
//
// All three kernels are persistent (one CTA per SM, up to ~227 KB shared
// memory, 512 TMEM columns) and drive the tile engine of tc_mlp.cuh with a
// stream of 128-evaluation tiles; the epilogue threads compute the features of
// the next tile before the engine retires the current one:
//   k_near_tc : close pairs (I, J) fetched from a global counter, staged in
//               shared memory (two buffers: the pair being retired and the next)
//               and flattened into tiles; the contraction u_I += M f_J (and
//               u_J += M f_I for J > I) is reduced per particle in shared memory
//               and flushed with one FP64 atomic per particle and component per
//               pair (src/CloseDot.cpp:245-299).
//   k_far_tc  : column / row queries of all active ACA blocks, symmetrised into
//               the FP64 C / Q pools (src/FarDot.cpp:348-458, 672-781).
//   k_eval_tc : M(r) for an array of features.
#include "common.h"
#include "kernels.h"
#include "tc_mlp.cuh"

namespace hignn {

namespace {

__device__ __forceinline__ uint8_t* align1k(uint8_t* p) {
  const uint32_t a = tc::saddr(p);
  return p + ((1024u - (a & 1023u)) & 1023u);
}

struct NearStage {
  float4 xI[kMaxLeaf], xJ[kMaxLeaf], fI[kMaxLeaf], fJ[kMaxLeaf];
  float uI[kMaxLeaf][3], uJ[kMaxLeaf][3];
};

struct NearTcSmem {
  tc::Smem tcs;
  NearStage st[2];
  int item[2];
};
static_assert(sizeof(NearTcSmem) + 1024 <= 232448, "near-field shared memory exceeds 227 KB per CTA");

// u_I[i] += v for the rows of a warp: rows of a tile share few i (contiguous), so lanes with
// equal i are summed by a segmented shuffle reduction and only segment heads add to shared memory.
__device__ __forceinline__ void add_segmented(float (*uI)[3], int i, float v0, float v1, float v2) {
  const unsigned act = __activemask();
  if (act == 0xffffffffu) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float t0 = __shfl_down_sync(act, v0, o), t1 = __shfl_down_sync(act, v1, o),
                  t2 = __shfl_down_sync(act, v2, o);
      const int ko = __shfl_down_sync(act, i, o);
      if (lane + o < 32 && ko == i) {
        v0 += t0;
        v1 += t1;
        v2 += t2;
      }
    }
    const int kp = __shfl_up_sync(act, i, 1);
    if (lane == 0 || kp != i) {
      atomicAdd(&uI[i][0], v0);
      atomicAdd(&uI[i][1], v1);
      atomicAdd(&uI[i][2], v2);
    }
  } else {
    atomicAdd(&uI[i][0], v0);
    atomicAdd(&uI[i][1], v1);
    atomicAdd(&uI[i][2], v2);
  }
}

// Position of one 128-evaluation tile in the near-field stream.
struct NearCursor {
  int buf, item, t0;
  PairWork pw;
};

// Next close pair from the global counter, staged into buffer b (all epilogue threads).
__device__ __forceinline__ bool near_fetch(NearTcSmem& S, const NearArgs& a, int* counter, int b, NearCursor& c) {
  const int e = threadIdx.x;
  if (e == 0) S.item[b] = atomicAdd(counter, 1);
  tc::epi_bar();  // also: every thread is done with the pair last staged in buffer b
  const int item = S.item[b];
  if (item >= a.nwork) return false;
  const PairWork pw = a.work[item];
  NearStage& G = S.st[b];
  for (int i = e; i < pw.nI; i += tc::kEpiThreads) {
    G.xI[i] = a.xI[pw.sI + i];
    G.fI[i] = a.fI[pw.sI + i];
    G.uI[i][0] = G.uI[i][1] = G.uI[i][2] = 0.f;
  }
  for (int j = e; j < pw.nJ; j += tc::kEpiThreads) {
    G.xJ[j] = a.xJ[pw.sJ + j];
    G.fJ[j] = a.fJ[pw.sJ + j];
    G.uJ[j][0] = G.uJ[j][1] = G.uJ[j][2] = 0.f;
  }
  tc::epi_bar();
  c.buf = b;
  c.item = item;
  c.t0 = 0;
  c.pw = pw;
  return true;
}

// This thread's row of a tile: (i, j) and the feature r = x_j - x_i (a dummy for padding rows).
__device__ __forceinline__ bool near_row(const NearTcSmem& S, const NearCursor& c, int row, int& i, int& j,
                                         float (&r)[3]) {
  const int total = c.pw.nI * c.pw.nJ;
  const int flat = c.t0 + row;
  const bool valid = flat < total;
  i = valid ? flat / c.pw.nJ : 0;
  j = valid ? flat - i * c.pw.nJ : 0;
  r[0] = 1.f;
  r[1] = r[2] = 0.f;
  if (valid) {
    const float4 xi = S.st[c.buf].xI[i], xj = S.st[c.buf].xJ[j];
    r[0] = xj.x - xi.x;
    r[1] = xj.y - xi.y;
    r[2] = xj.z - xi.z;
  }
  return valid;
}

__global__ void __launch_bounds__(tc::kThreads, 1)
    k_near_tc(NearArgs a, TcWeights w, int* work_counter, int* err) {
  extern __shared__ uint8_t smem_raw[];
  NearTcSmem& S = *reinterpret_cast<NearTcSmem*>(align1k(smem_raw));
  tc::cta_setup(S.tcs, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == tc::kMmaWarp) {
    if (lane == 0) tc::mma_loop(S.tcs, err);
    __syncwarp();
  } else {
    const int e = threadIdx.x, row = tc::epi_row(), p = tc::epi_part();
    tc::Epi eng{S.tcs, err, S.tcs.tmem_base + ((uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16), p};
    NearCursor cur;
    bool have = near_fetch(S, a, work_counter, 0, cur);
    int i = 0, j = 0;
    float r[3];
    bool valid = have && near_row(S, cur, row, i, j, r);
    eng.start(have, r[0], r[1], r[2]);
    while (have) {
      // the next tile: the rest of this pair, or the next pair staged into the other buffer
      NearCursor nxt = cur;
      nxt.t0 += tc::kTile;
      const bool last = nxt.t0 >= cur.pw.nI * cur.pw.nJ;
      bool has_next = true;
      if (last) has_next = near_fetch(S, a, work_counter, cur.buf ^ 1, nxt);
      int ni = 0, nj = 0;
      float nr[3] = {1.f, 0.f, 0.f};
      const bool nvalid = has_next && near_row(S, nxt, row, ni, nj, nr);
      float M[9];
      const bool ok = tc::epi_all(eng.step(has_next, nr[0], nr[1], nr[2], r[0], r[1], r[2], M));
      if (!ok) break;
      NearStage& G = S.st[cur.buf];
      const bool trans = (cur.pw.flags & kPairTransposed) != 0;
      if (valid && p < 2) {
        if (cur.pw.flags & kPairSymmetrize) {
#pragma unroll
          for (int q = 0; q < 3; q++)
#pragma unroll
            for (int c = q + 1; c < 3; c++) {
              const float v = 0.5f * (M[3 * q + c] + M[3 * c + q]);
              M[3 * q + c] = v;
              M[3 * c + q] = v;
            }
        }
        if (p == 0) {  // u_I[i] += M f_J[j]
          const float4 fj = G.fJ[j];
          add_segmented(G.uI, i, M[0] * fj.x + M[1] * fj.y + M[2] * fj.z, M[3] * fj.x + M[4] * fj.y + M[5] * fj.z,
                        M[6] * fj.x + M[7] * fj.y + M[8] * fj.z);
        } else if (trans) {  // u_J[j] += M f_I[i] (same M, src/CloseDot.cpp:281-298)
          const float4 fi = G.fI[i];
          atomicAdd(&G.uJ[j][0], M[0] * fi.x + M[1] * fi.y + M[2] * fi.z);
          atomicAdd(&G.uJ[j][1], M[3] * fi.x + M[4] * fi.y + M[5] * fi.z);
          atomicAdd(&G.uJ[j][2], M[6] * fi.x + M[7] * fi.y + M[8] * fi.z);
        }
      }
      if (last) {  // the pair is complete: flush its velocities
        tc::epi_bar();
        for (int q = e; q < 3 * cur.pw.nI; q += tc::kEpiThreads)
          atomicAdd(&a.uI[3 * (size_t)cur.pw.sI + q], (double)(&G.uI[0][0])[q]);
        if (trans)
          for (int q = e; q < 3 * cur.pw.nJ; q += tc::kEpiThreads)
            atomicAdd(&a.uJ[3 * (size_t)cur.pw.sJ + q], (double)(&G.uJ[0][0])[q]);
      }
      if (!has_next) break;
      cur = nxt;
      i = ni;
      j = nj;
      valid = nvalid;
      r[0] = nr[0];
      r[1] = nr[1];
      r[2] = nr[2];
    }
  }
  tc::cta_teardown(S.tcs);
}

struct FarTcSmem {
  tc::Smem tcs;
};

// This thread's row of far tile `tile`: block b, local index loc, term k, feature r.
__device__ __forceinline__ bool far_row(const FarArgs& a, int which, int nact, int tot, int tile, int row, int& b,
                                        int& loc, int& k, float (&r)[3]) {
  const int g = tile * tc::kTile + row;
  r[0] = 1.f;
  r[1] = r[2] = 0.f;
  if (g >= tot) return false;
  const int32_t* pre = which ? a.preJ : a.preI;
  int lo = 0, hi = nact;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  b = a.act[lo];
  loc = g - pre[lo];
  const FarBlock bk = a.blocks[b];
  k = a.state[b].k;
  float4 xi, xj;
  if (which == 0) {
    xj = a.x[bk.sJ + a.cols[(size_t)b * a.ldr + k]];
    xi = a.x[bk.sI + loc];
  } else {
    xj = a.x[bk.sJ + loc];
    xi = a.x[bk.sI + a.rows[(size_t)b * a.ldr + k]];
  }
  r[0] = xj.x - xi.x;
  r[1] = xj.y - xi.y;
  r[2] = xj.z - xi.z;
  return true;
}

__global__ void __launch_bounds__(tc::kThreads, 1) k_far_tc(FarArgs a, TcWeights w, int which, int* err) {
  extern __shared__ uint8_t smem_raw[];
  FarTcSmem& S = *reinterpret_cast<FarTcSmem*>(align1k(smem_raw));
  const int nact = a.ctr[kCtrActive];
  const int tot = which ? a.ctr[kCtrTotJ] : a.ctr[kCtrTotI];
  if ((int)blockIdx.x * tc::kTile >= tot) return;  // uniform: before any setup
  tc::cta_setup(S.tcs, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == tc::kMmaWarp) {
    if (lane == 0) tc::mma_loop(S.tcs, err);
    __syncwarp();
  } else {
    const int row = tc::epi_row(), p = tc::epi_part();
    tc::Epi eng{S.tcs, err, S.tcs.tmem_base + ((uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16), p};
    int tile = blockIdx.x, b = 0, loc = 0, k = 0;
    float r[3];
    bool valid = far_row(a, which, nact, tot, tile, row, b, loc, k, r);
    eng.start(true, r[0], r[1], r[2]);
    for (;;) {
      const int nt = tile + gridDim.x;
      const bool has_next = nt * tc::kTile < tot;
      int nb = 0, nloc = 0, nk = 0;
      float nr[3] = {1.f, 0.f, 0.f};
      const bool nvalid = has_next && far_row(a, which, nact, tot, nt, row, nb, nloc, nk, nr);
      float M[9];
      if (!tc::epi_all(eng.step(has_next, nr[0], nr[1], nr[2], r[0], r[1], r[2], M))) break;
      if (valid && p < 2) {  // the two threads of a row store alternate entries
        const FarBlock bk = a.blocks[b];
        pool_t* dst = which == 0 ? a.C + 9 * (bk.cOff + (int64_t)k * bk.nI + loc)
                                 : a.Q + 9 * (bk.qOff + (int64_t)k * bk.nJ + loc);
#pragma unroll
        for (int q = 0; q < 9; q++) {
          if ((q & 1) != p) continue;
          const int rr = q / 3, c = q % 3;
          dst[q] = (rr == c) ? (double)M[q] : 0.5 * (double)(M[3 * rr + c] + M[3 * c + rr]);
        }
      }
      if (!has_next) break;
      tile = nt;
      b = nb;
      loc = nloc;
      k = nk;
      valid = nvalid;
      r[0] = nr[0];
      r[1] = nr[1];
      r[2] = nr[2];
    }
  }
  tc::cta_teardown(S.tcs);
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(a.evals, (unsigned long long)tot);
}

struct EvalTcSmem {
  tc::Smem tcs;
};

__device__ __forceinline__ bool eval_row(const float* __restrict__ r, int64_t n, int64_t tile, int row,
                                         float (&f)[3]) {
  const int64_t g = tile * tc::kTile + row;
  f[0] = 1.f;
  f[1] = f[2] = 0.f;
  if (g >= n) return false;
  f[0] = r[3 * g];
  f[1] = r[3 * g + 1];
  f[2] = r[3 * g + 2];
  return true;
}

__global__ void __launch_bounds__(tc::kThreads, 1)
    k_eval_tc(const float* __restrict__ r, float* __restrict__ y, int64_t n, TcWeights w, int* err) {
  extern __shared__ uint8_t smem_raw[];
  EvalTcSmem& S = *reinterpret_cast<EvalTcSmem*>(align1k(smem_raw));
  tc::cta_setup(S.tcs, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == tc::kMmaWarp) {
    if (lane == 0) tc::mma_loop(S.tcs, err);
    __syncwarp();
  } else {
    const int row = tc::epi_row(), p = tc::epi_part();
    tc::Epi eng{S.tcs, err, S.tcs.tmem_base + ((uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16), p};
    int64_t tile = blockIdx.x;
    float f[3];
    bool valid = eval_row(r, n, tile, row, f);
    eng.start(true, f[0], f[1], f[2]);
    for (;;) {
      const int64_t nt = tile + gridDim.x;
      const bool has_next = nt * tc::kTile < n;
      float nf[3] = {1.f, 0.f, 0.f};
      const bool nvalid = has_next && eval_row(r, n, nt, row, nf);
      float M[9];
      if (!tc::epi_all(eng.step(has_next, nf[0], nf[1], nf[2], f[0], f[1], f[2], M))) break;
      if (valid && p < 2) {
        const int64_t g = tile * tc::kTile + row;
#pragma unroll
        for (int q = 0; q < 9; q++)
          if ((q & 1) == p) y[9 * g + q] = M[q];
      }
      if (!has_next) break;
      tile = nt;
      valid = nvalid;
      f[0] = nf[0];
      f[1] = nf[1];
      f[2] = nf[2];
    }
  }
  tc::cta_teardown(S.tcs);
}

template <class K>
void set_smem(K kernel, size_t bytes) {
  HIGNN_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

size_t near_tc_smem_bytes() { return sizeof(NearTcSmem) + 1024; }

void launch_near_tc(const NearArgs& a, const TcWeights& w, int* work_counter, int* err, int num_sms,
                    cudaStream_t s) {
  if (a.nwork <= 0) return;
  const size_t smem = sizeof(NearTcSmem) + 1024;
  set_smem(k_near_tc, smem);
  HIGNN_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(int), s));
  const int grid = a.nwork < num_sms ? a.nwork : num_sms;
  k_near_tc<<<grid, tc::kThreads, smem, s>>>(a, w, work_counter, err);
  HIGNN_CHECK_LAUNCH();
}

void launch_far_tc(const FarArgs& a, const TcWeights& w, int which, int* err, int num_sms, cudaStream_t s) {
  const size_t smem = sizeof(FarTcSmem) + 1024;
  set_smem(k_far_tc, smem);
  k_far_tc<<<num_sms, tc::kThreads, smem, s>>>(a, w, which, err);
  HIGNN_CHECK_LAUNCH();
}

void launch_eval_tc(const float* r, float* y, int64_t n, const TcWeights& w, int* err, int num_sms,
                    cudaStream_t s) {
  if (n <= 0) return;
  const size_t smem = sizeof(EvalTcSmem) + 1024;
  set_smem(k_eval_tc, smem);
  const int64_t tiles = (n + tc::kTile - 1) / tc::kTile;
  const int grid = (int)(tiles < num_sms ? tiles : num_sms);
  k_eval_tc<<<grid, tc::kThreads, smem, s>>>(r, y, n, w, err);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
