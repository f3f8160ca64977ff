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

// Leaves up to kTcLeaf particles (the tensor-core forms need block_size <= 128).
constexpr int kTcLeaf = kTcMaxLeaf;

struct NearStage {
  float4 xI[kTcLeaf], xJ[kTcLeaf], fI[kTcLeaf], fJ[kTcLeaf];
  float uI[kTcLeaf][3], uJ[kTcLeaf][3];
};

// Three staging buffers: the pair of the tile being retired, of the tile in flight and of the
// next tile can all differ (pairs of a single tile).
struct NearTcSmem {
  tc::Smem tcs;
  NearStage st[3];
  PairWork pw[3];
  int item[3];
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

// Position of one 128-evaluation tile in the near-field stream and this thread's row of it.
struct NearTile {
  int buf, t0;  // the pair itself is S.pw[buf]
  int i, j;
  bool valid, last;  // last: the final tile of its pair
  float r[3];
};

// Next close pair from the global counter, staged into buffer b (all epilogue threads).
__device__ __forceinline__ bool near_fetch(NearTcSmem& S, const NearArgs& a, int* counter, int b, NearTile& c) {
  const int e = threadIdx.x;
  // after an abort the stream ends here for every thread (the item is broadcast)
  if (e == 0) S.item[b] = *(volatile int*)&S.tcs.abort_flag ? a.nwork : atomicAdd(counter, 1);
  tc::epi_bar();  // also: every thread is done with the pair last staged in buffer b
  const int item = S.item[b];
  if (item >= a.nwork) return false;
  const PairWork pw = a.work[item];
  if (e == 0) S.pw[b] = pw;
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
  c.t0 = 0;
  return true;
}

// This thread's row of a tile: (i, j) and the feature r = x_j - x_i (a dummy for padding rows).
__device__ __forceinline__ void near_row(const NearTcSmem& S, NearTile& c, int row) {
  const int nJ = S.pw[c.buf].nJ, total = S.pw[c.buf].nI * nJ;
  const int flat = c.t0 + row;
  c.valid = flat < total;
  c.last = c.t0 + tc::kTile >= total;
  c.i = c.valid ? flat / nJ : 0;
  c.j = c.valid ? flat - c.i * nJ : 0;
  c.r[0] = 1.f;
  c.r[1] = c.r[2] = 0.f;
  if (c.valid) {
    const float4 xi = S.st[c.buf].xI[c.i], xj = S.st[c.buf].xJ[c.j];
    c.r[0] = xj.x - xi.x;
    c.r[1] = xj.y - xi.y;
    c.r[2] = xj.z - xi.z;
  }
}

// Contraction of one retired tile: u_I += M f_J (part 0), u_J += M f_I for J > I (part 1)
// (src/CloseDot.cpp:245-299), into the pair's shared-memory accumulators.
__device__ __forceinline__ void near_use(NearTcSmem& S, const NearTile& c, int p, float (&M)[9]) {
  if (!c.valid || p >= 2) return;
  NearStage& G = S.st[c.buf];
  const int flags = S.pw[c.buf].flags;
  if (flags & kPairSymmetrize) {
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int k = q + 1; k < 3; k++) {
        const float v = 0.5f * (M[3 * q + k] + M[3 * k + q]);
        M[3 * q + k] = v;
        M[3 * k + q] = v;
      }
  }
  if (p == 0) {
    const float4 fj = G.fJ[c.j];
    add_segmented(G.uI, c.i, M[0] * fj.x + M[1] * fj.y + M[2] * fj.z, M[3] * fj.x + M[4] * fj.y + M[5] * fj.z,
                  M[6] * fj.x + M[7] * fj.y + M[8] * fj.z);
  } else if (flags & kPairTransposed) {  // same M, not transposed (src/CloseDot.cpp:281-298)
    const float4 fi = G.fI[c.i];
    atomicAdd(&G.uJ[c.j][0], M[0] * fi.x + M[1] * fi.y + M[2] * fi.z);
    atomicAdd(&G.uJ[c.j][1], M[3] * fi.x + M[4] * fi.y + M[5] * fi.z);
    atomicAdd(&G.uJ[c.j][2], M[6] * fi.x + M[7] * fi.y + M[8] * fi.z);
  }
}

// The pair of a retired last tile is complete: flush its velocities (all epilogue threads).
__device__ __forceinline__ void near_flush(NearTcSmem& S, const NearArgs& a, const NearTile& c) {
  tc::epi_bar();
  if (*(volatile int*)&S.tcs.abort_flag) return;  // the launch reports an error; nothing is added
  const NearStage& G = S.st[c.buf];
  const PairWork pw = S.pw[c.buf];
  for (int q = threadIdx.x; q < 3 * pw.nI; q += tc::kEpiThreads)
    atomicAdd(&a.uI[3 * (size_t)pw.sI + q], (double)(&G.uI[0][0])[q]);
  if (pw.flags & kPairTransposed)
    for (int q = threadIdx.x; q < 3 * pw.nJ; q += tc::kEpiThreads)
      atomicAdd(&a.uJ[3 * (size_t)pw.sJ + q], (double)(&G.uJ[0][0])[q]);
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
    const long long t_start = clock64();
    const int row = tc::epi_row(), p = tc::epi_part();
    tc::Epi eng{S.tcs, err, S.tcs.tmem_base + ((uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16), p};
    NearTile prev{}, cur{};
    int nbuf = 0;  // staging buffers are used in turn
    const bool have = near_fetch(S, a, work_counter, nbuf, cur);
    nbuf = (nbuf + 1) % 3;
    if (have) near_row(S, cur, row);
    eng.start(have, cur.r[0], cur.r[1], cur.r[2]);
    bool has_prev = false;
    // The control flow is uniform over the epilogue threads (tile positions and work items are
    // shared), so the named barriers of near_fetch / near_flush are always reached by all of them;
    // after an abort the engine calls return at once and near_fetch ends the stream.
    while (have) {
      // the next tile: the rest of this pair, or the next pair staged into the next buffer
      NearTile nxt = cur;
      nxt.t0 += tc::kTile;
      bool has_next = true;
      if (cur.last) {
        has_next = near_fetch(S, a, work_counter, nbuf, nxt);
        nbuf = (nbuf + 1) % 3;
      }
      if (has_next) near_row(S, nxt, row);
      eng.step(has_next, nxt.r[0], nxt.r[1], nxt.r[2], prev.r[0], prev.r[1], prev.r[2],
               [&](float (&M)[9]) { near_use(S, prev, p, M); });
      if (has_prev && prev.last) near_flush(S, a, prev);
      prev = cur;
      has_prev = true;
      if (!has_next) break;
      cur = nxt;
    }
    if (has_prev) {
      eng.finish(prev.r[0], prev.r[1], prev.r[2], [&](float (&M)[9]) { near_use(S, prev, p, M); });
      near_flush(S, a, prev);
    }
    if (S.tcs.prof && threadIdx.x == 0) S.tcs.wprof[12] += (unsigned long long)(clock64() - t_start);
  }
  tc::cta_teardown(S.tcs);
}

struct FarTcSmem {
  tc::Smem tcs;
};

// This thread's row of far tile `tile`: block b, local index loc, term k, feature r.
struct FarRow {
  int b, loc, k;
  bool valid;
  float r[3];
};

__device__ __forceinline__ void far_row(const FarArgs& a, int which, int nact, int tot, int tile, int row, FarRow& f) {
  const int g = tile * tc::kTile + row;
  f.r[0] = 1.f;
  f.r[1] = f.r[2] = 0.f;
  f.valid = g < tot;
  if (!f.valid) return;
  const int32_t* pre = which ? a.preJ : a.preI;
  int lo = 0, hi = nact;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  f.b = a.act[lo];
  f.loc = g - pre[lo];
  const FarBlock bk = a.blocks[f.b];
  f.k = a.state[f.b].k;
  float4 xi, xj;
  if (which == 0) {
    xj = a.x[bk.sJ + a.cols[(size_t)f.b * a.ldr + f.k]];
    xi = a.x[bk.sI + f.loc];
  } else {
    xj = a.x[bk.sJ + f.loc];
    xi = a.x[bk.sI + a.rows[(size_t)f.b * a.ldr + f.k]];
  }
  f.r[0] = xj.x - xi.x;
  f.r[1] = xj.y - xi.y;
  f.r[2] = xj.z - xi.z;
}

// symmetrised 3x3 of a retired far row into the C (which = 0) or Q pool; the two threads of a
// row store alternate entries (src/FarDot.cpp:445-456: diagonal copied, off-diagonal halved sum)
__device__ __forceinline__ void far_use(const FarArgs& a, int which, const FarRow& f, int p, const float (&M)[9]) {
  if (!f.valid || p >= 2) return;
  const FarBlock bk = a.blocks[f.b];
  pool_t* dst = which == 0 ? a.C + 9 * (bk.cOff + (int64_t)f.k * bk.nI + f.loc)
                           : a.Q + 9 * (bk.qOff + (int64_t)f.k * bk.nJ + f.loc);
#pragma unroll
  for (int q = 0; q < 9; q++) {
    if ((q & 1) != p) continue;
    const int rr = q / 3, c = q % 3;
    dst[q] = (rr == c) ? M[q] : 0.5f * (M[3 * rr + c] + M[3 * c + rr]);  // the FP32 half-sum is exact in FP64 too
  }
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
    int tile = blockIdx.x;
    FarRow prev{}, cur{};
    far_row(a, which, nact, tot, tile, row, cur);
    eng.start(true, cur.r[0], cur.r[1], cur.r[2]);
    for (;;) {  // uniform over the epilogue threads; after an abort the engine calls return at once
      const int nt = tile + gridDim.x;
      const bool has_next = nt * tc::kTile < tot;
      FarRow nxt{};
      nxt.r[0] = 1.f;
      if (has_next) far_row(a, which, nact, tot, nt, row, nxt);
      eng.step(has_next, nxt.r[0], nxt.r[1], nxt.r[2], prev.r[0], prev.r[1], prev.r[2],
               [&](float (&M)[9]) { far_use(a, which, prev, p, M); });
      prev = cur;
      if (!has_next) break;
      tile = nt;
      cur = nxt;
    }
    eng.finish(prev.r[0], prev.r[1], prev.r[2], [&](float (&M)[9]) { far_use(a, which, prev, p, M); });
  }
  tc::cta_teardown(S.tcs);
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(a.evals, (unsigned long long)tot);
}

struct EvalTcSmem {
  tc::Smem tcs;
};

struct EvalRow {
  int64_t g;
  bool valid;
  float r[3];
};

__device__ __forceinline__ void eval_row(const float* __restrict__ r, int64_t n, int64_t tile, int row, EvalRow& f) {
  f.g = tile * tc::kTile + row;
  f.valid = f.g < n;
  f.r[0] = 1.f;
  f.r[1] = f.r[2] = 0.f;
  if (!f.valid) return;
  f.r[0] = r[3 * f.g];
  f.r[1] = r[3 * f.g + 1];
  f.r[2] = r[3 * f.g + 2];
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
    auto use = [&](const EvalRow& f, float(&M)[9]) {
      if (f.valid && p < 2)  // the two threads of a row store alternate entries
#pragma unroll
        for (int q = 0; q < 9; q++)
          if ((q & 1) == p) y[9 * f.g + q] = M[q];
    };
    int64_t tile = blockIdx.x;
    EvalRow prev{}, cur{};
    eval_row(r, n, tile, row, cur);
    eng.start(true, cur.r[0], cur.r[1], cur.r[2]);
    for (;;) {  // uniform over the epilogue threads; after an abort the engine calls return at once
      const int64_t nt = tile + gridDim.x;
      const bool has_next = nt * tc::kTile < n;
      EvalRow nxt{};
      nxt.r[0] = 1.f;
      if (has_next) eval_row(r, n, nt, row, nxt);
      eng.step(has_next, nxt.r[0], nxt.r[1], nxt.r[2], prev.r[0], prev.r[1], prev.r[2],
               [&](float (&M)[9]) { use(prev, M); });
      prev = cur;
      if (!has_next) break;
      tile = nt;
      cur = nxt;
    }
    eng.finish(prev.r[0], prev.r[1], prev.r[2], [&](float (&M)[9]) { use(prev, M); });
  }
  tc::cta_teardown(S.tcs);
}

template <class K>
void set_smem(K kernel, size_t bytes, cudaStream_t s) {
  set_max_dynamic_smem(kernel, bytes, s);
}

}  // namespace

size_t near_tc_smem_bytes() { return sizeof(NearTcSmem) + 1024; }

void launch_near_tc(const NearArgs& a, const TcWeights& w, int* work_counter, int* err, int num_sms,
                    cudaStream_t s) {
  if (a.nwork <= 0) return;
  const size_t smem = sizeof(NearTcSmem) + 1024;
  set_smem(k_near_tc, smem, s);
  HIGNN_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(int), s));
  const int grid = a.nwork < num_sms ? a.nwork : num_sms;
  k_near_tc<<<grid, tc::kThreads, smem, s>>>(a, w, work_counter, err);
  HIGNN_CHECK_LAUNCH();
}

void launch_far_tc(const FarArgs& a, const TcWeights& w, int which, int* err, int num_sms, cudaStream_t s) {
  const size_t smem = sizeof(FarTcSmem) + 1024;
  set_smem(k_far_tc, smem, s);
  k_far_tc<<<num_sms, tc::kThreads, smem, s>>>(a, w, which, err);
  HIGNN_CHECK_LAUNCH();
}

void launch_eval_tc(const float* r, float* y, int64_t n, const TcWeights& w, int* err, int num_sms,
                    cudaStream_t s) {
  if (n <= 0) return;
  const size_t smem = sizeof(EvalTcSmem) + 1024;
  set_smem(k_eval_tc, smem, s);
  const int64_t tiles = (n + tc::kTile - 1) / tc::kTile;
  const int grid = (int)(tiles < num_sms ? tiles : num_sms);
  k_eval_tc<<<grid, tc::kThreads, smem, s>>>(r, y, n, w, err);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
