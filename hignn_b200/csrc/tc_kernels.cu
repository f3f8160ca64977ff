// Tensor-core (tcgen05) forms of the near field, the ACA queries and the stand-alone evaluation.
//
// All three kernels are persistent (one CTA per SM, up to ~213 KB shared
// memory, 512 TMEM columns) and share the tile engine of tc_mlp.cuh. Each CTA
// runs two independent epilogue groups (tile contexts); every group walks its
// own share of the work:
//   k_near_tc : close pairs (I, J) fetched from a global counter, flattened into
//               128-evaluation tiles; the contraction u_I += M f_J (and u_J +=
//               M f_I for J > I) is reduced per particle in shared memory and
//               flushed with one FP64 atomic per particle and component per pair
//               (src/CloseDot.cpp:245-299).
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
  int item;
};

struct NearTcSmem {
  tc::Smem tcs;
  NearStage st[2];
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
    NearStage& G = S.st[tc::epi_group()];
    const int e = tc::epi_gthread();  // staging / flush index within the group
    const int row = tc::epi_row(), h = tc::epi_half();
    tc::EpiState st;
    bool ok = true;
    for (;;) {
      if (e == 0) G.item = atomicAdd(work_counter, 1);
      tc::epi_bar();
      const int item = G.item;
      if (item >= a.nwork) break;
      const PairWork pw = a.work[item];
      const bool trans = (pw.flags & kPairTransposed) != 0;
      const bool symm = (pw.flags & kPairSymmetrize) != 0;
      for (int i = e; i < pw.nI; i += tc::kGroupThreads) {
        G.xI[i] = a.xI[pw.sI + i];
        G.fI[i] = a.fI[pw.sI + i];
        G.uI[i][0] = G.uI[i][1] = G.uI[i][2] = 0.f;
      }
      for (int j = e; j < pw.nJ; j += tc::kGroupThreads) {
        G.xJ[j] = a.xJ[pw.sJ + j];
        G.fJ[j] = a.fJ[pw.sJ + j];
        G.uJ[j][0] = G.uJ[j][1] = G.uJ[j][2] = 0.f;
      }
      tc::epi_bar();
      const int total = pw.nI * pw.nJ;
      for (int t0 = 0; t0 < total; t0 += tc::kTile) {
        const int flat = t0 + row;
        const bool valid = flat < total;
        const int i = valid ? flat / pw.nJ : 0;
        const int j = valid ? flat - i * pw.nJ : 0;
        float rx = 1.f, ry = 0.f, rz = 0.f;
        if (valid) {
          const float4 xi = G.xI[i], xj = G.xJ[j];
          rx = xj.x - xi.x;
          ry = xj.y - xi.y;
          rz = xj.z - xi.z;
        }
        float M[9];
        ok = tc::run_tile(S.tcs, st, rx, ry, rz, M, err);
        if (!ok) break;
        if (valid) {
          if (symm) {
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
              for (int c = r + 1; c < 3; c++) {
                const float v = 0.5f * (M[3 * r + c] + M[3 * c + r]);
                M[3 * r + c] = v;
                M[3 * c + r] = v;
              }
          }
          if (h == 0) {  // u_I[i] += M f_J[j]
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
      }
      if (!ok) break;
      tc::epi_bar();
      for (int q = e; q < 3 * pw.nI; q += tc::kGroupThreads)
        atomicAdd(&a.uI[3 * (size_t)pw.sI + q], (double)(&G.uI[0][0])[q]);
      if (trans)
        for (int q = e; q < 3 * pw.nJ; q += tc::kGroupThreads)
          atomicAdd(&a.uJ[3 * (size_t)pw.sJ + q], (double)(&G.uJ[0][0])[q]);
      tc::epi_bar();
    }
    if (ok) tc::epi_finish(S.tcs);
  }
  tc::cta_teardown(S.tcs);
}

struct FarTcSmem {
  tc::Smem tcs;
};

__global__ void __launch_bounds__(tc::kThreads, 1) k_far_tc(FarArgs a, TcWeights w, int which, int* err) {
  extern __shared__ uint8_t smem_raw[];
  FarTcSmem& S = *reinterpret_cast<FarTcSmem*>(align1k(smem_raw));
  const int nact = a.ctr[kCtrActive];
  const int tot = which ? a.ctr[kCtrTotJ] : a.ctr[kCtrTotI];
  if (2 * (int)blockIdx.x * tc::kTile >= tot) return;  // uniform: before any setup
  tc::cta_setup(S.tcs, w);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == tc::kMmaWarp) {
    if (lane == 0) tc::mma_loop(S.tcs, err);
    __syncwarp();
  } else {
    const int row = tc::epi_row(), h = tc::epi_half();
    const int32_t* pre = which ? a.preJ : a.preI;
    tc::EpiState st;
    bool ok = true;
    for (int tile = 2 * blockIdx.x + tc::epi_group(); tile * tc::kTile < tot; tile += 2 * gridDim.x) {
      const int g = tile * tc::kTile + row;
      const bool valid = g < tot;
      float rx = 1.f, ry = 0.f, rz = 0.f;
      int b = 0, loc = 0, k = 0;
      if (valid) {
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
        rx = xj.x - xi.x;
        ry = xj.y - xi.y;
        rz = xj.z - xi.z;
      }
      float M[9];
      ok = tc::run_tile(S.tcs, st, rx, ry, rz, M, err);
      if (!ok) break;
      if (valid) {  // the two threads of a row store alternate entries
        const FarBlock bk = a.blocks[b];
        double* dst = which == 0 ? a.C + 9 * (bk.cOff + (int64_t)k * bk.nI + loc)
                                 : a.Q + 9 * (bk.qOff + (int64_t)k * bk.nJ + loc);
#pragma unroll
        for (int q = 0; q < 9; q++) {
          if ((q & 1) != h) continue;
          const int r = q / 3, c = q % 3;
          dst[q] = (r == c) ? (double)M[q] : 0.5 * (double)(M[3 * r + c] + M[3 * c + r]);
        }
      }
    }
    if (ok) tc::epi_finish(S.tcs);
  }
  tc::cta_teardown(S.tcs);
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(a.evals, (unsigned long long)tot);
}

struct EvalTcSmem {
  tc::Smem tcs;
};

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
    const int row = tc::epi_row(), h = tc::epi_half();
    tc::EpiState st;
    bool ok = true;
    for (int64_t tile = 2 * (int64_t)blockIdx.x + tc::epi_group(); tile * tc::kTile < n;
         tile += 2 * (int64_t)gridDim.x) {
      const int64_t g = tile * tc::kTile + row;
      float rx = 1.f, ry = 0.f, rz = 0.f;
      if (g < n) {
        rx = r[3 * g];
        ry = r[3 * g + 1];
        rz = r[3 * g + 2];
      }
      float M[9];
      ok = tc::run_tile(S.tcs, st, rx, ry, rz, M, err);
      if (!ok) break;
      if (g < n)
#pragma unroll
        for (int q = 0; q < 9; q++)
          if ((q & 1) == h) y[9 * g + q] = M[q];
    }
    if (ok) tc::epi_finish(S.tcs);
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
  const int64_t pairs = (tiles + 1) / 2;
  const int grid = (int)(pairs < num_sms ? pairs : num_sms);
  k_eval_tc<<<grid, tc::kThreads, smem, s>>>(r, y, n, w, err);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
