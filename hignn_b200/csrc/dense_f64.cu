// FP64 dense rows: u_i = sum_j 0.5 (M + M^T)(x_j - x_i) f_j with the two-body network evaluated
// in FP64 (weights promoted from their FP32 values), FP64 sums over all sources.
//
// This is the dense FP64 evaluation the H-matrix product's error is measured against
// (src/PostCheckDot.cpp:351-376 compares against a dense product; here the network itself runs
// in FP64 so that the reference point carries no FP32 network rounding). It takes the same work
// list as the FP32 dense rows (PairWork items flagged kPairSymmetrize: up to 128 gathered target
// rows against one source leaf of up to kMaxLeaf particles).
//
// One persistent CTA per SM, 256 threads, tiles of 128 evaluations:
//   layer 1: h1[k][e] = tanh(W1[k] . r_e + b1[k]) (128 x 128 doubles in shared memory);
//   layer 2: eight chunks of 64 hidden units, each a 128 x 64 x 128 register-tiled DGEMM (8
//            evaluations x 4 units per thread) on one W2^T chunk staged in shared memory as
//            doubles; the chunk buffer then receives tanh(acc + b2) as [unit][evaluation];
//   layer 3: y[e][o] += sum_n h2[n][e] W3[o][n], W3 read through the read-only cache;
//   wrapper: (y + b3 + I) / |r|, identity below |r| = 1e-5 (python/convert.py:11-20).
#include "common.h"
#include "kernels.h"

namespace hignn {

namespace {

constexpr int kF64Threads = 256;
constexpr int kF64Tile = 128;
constexpr int kF64Chunk = 64;
constexpr int kH2Stride = kF64Tile + 2;  // h2 rows padded: the [unit][evaluation] stores spread over the banks

struct F64Smem {
  double h1[kH1][kF64Tile];          // 128 KB
  double buf[kF64Chunk * kH2Stride];  // 65 KB: W2^T chunk [k][n], then h2 [n][e] (row stride kH2Stride)
  double r[kF64Tile][3];
  double y[kF64Tile][kOut];
  double uI[kF64Tile][3];
  float4 xI[kF64Tile];
  float4 xJ[kMaxLeaf], fJ[kMaxLeaf];
  int16_t ei[kF64Tile], ej[kF64Tile];
  int item;
};
static_assert(sizeof(F64Smem) <= 232448, "FP64 dense-rows shared memory exceeds 227 KB per CTA");

__device__ __forceinline__ void f64_tile(F64Smem& s, const MlpF32& w) {
  const int t = threadIdx.x;
  // layer 1
  for (int idx = t; idx < kH1 * kF64Tile; idx += kF64Threads) {
    const int k = idx / kF64Tile, e = idx % kF64Tile;
    const float4 wk = __ldg(&w.w1b1[k]);
    const double z = (double)wk.w + (double)wk.x * s.r[e][0] + (double)wk.y * s.r[e][1] + (double)wk.z * s.r[e][2];
    s.h1[k][e] = tanh(z);
  }
  const int tn = t & 15, te = t >> 4;            // layer-2 micro tile: evals te*8..+8, units tn*4..+4
  const int e3 = t & (kF64Tile - 1), og = t >> 7;  // layer-3 owner: eval e3, outputs og*5..
  const int o0 = og * 5, on = og ? 4 : 5;
  double y3[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int c = 0; c < kH2 / kF64Chunk; c++) {
    __syncthreads();  // layer 1 done / previous chunk's h2 readers done
    for (int idx = t; idx < kH1 * kF64Chunk; idx += kF64Threads) {
      const int k = idx / kF64Chunk, n = idx % kF64Chunk;
      s.buf[idx] = (double)__ldg(&w.w2t[(size_t)k * kH2 + c * kF64Chunk + n]);
    }
    __syncthreads();
    double acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
#pragma unroll 2
    for (int k = 0; k < kH1; k++) {
      const double2* ap = reinterpret_cast<const double2*>(&s.h1[k][te * 8]);
      const double2* bp = reinterpret_cast<const double2*>(&s.buf[k * kF64Chunk + tn * 4]);
      const double2 a0 = ap[0], a1 = ap[1], a2 = ap[2], a3 = ap[3];
      const double2 b0 = bp[0], b1 = bp[1];
      const double av[8] = {a0.x, a0.y, a1.x, a1.y, a2.x, a2.y, a3.x, a3.y};
      const double bv[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    __syncthreads();  // every thread is done with the W2 chunk: the buffer takes h2
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = tn * 4 + j;
      const double bias = (double)__ldg(&w.b2[c * kF64Chunk + n]);
#pragma unroll
      for (int i = 0; i < 8; i++) s.buf[n * kH2Stride + te * 8 + i] = tanh(acc[i][j] + bias);
    }
    __syncthreads();
    for (int n = 0; n < kF64Chunk; n++) {
      const double h = s.buf[n * kH2Stride + e3];
#pragma unroll
      for (int o = 0; o < 5; o++)
        if (o < on) y3[o] = fma(h, (double)__ldg(&w.w3[(o0 + o) * kH2 + c * kF64Chunk + n]), y3[o]);
    }
  }
  const double rx = s.r[e3][0], ry = s.r[e3][1], rz = s.r[e3][2];
  const double nr = sqrt(rx * rx + ry * ry + rz * rz);
  for (int o = 0; o < on; o++) {
    const int oo = o0 + o;
    double v = y3[o] + (double)__ldg(&w.b3[oo]);
    const bool dg = (oo == 0 || oo == 4 || oo == 8);
    if (dg) v += 1.0;
    v = v / nr;
    if (nr < 1e-5) v = dg ? 1.0 : 0.0;
    s.y[e3][oo] = v;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kF64Threads, 1) k_dense_rows_f64(NearArgs a, MlpF32 w, int* counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  F64Smem& s = *reinterpret_cast<F64Smem*>(smem_raw);
  const int t = threadIdx.x;
  for (;;) {
    __syncthreads();
    if (t == 0) s.item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = s.item;
    if (item >= a.nwork) break;
    const PairWork pw = a.work[item];
    for (int i = t; i < pw.nI; i += kF64Threads) {
      s.xI[i] = a.xI[pw.sI + i];
      s.uI[i][0] = s.uI[i][1] = s.uI[i][2] = 0.0;
    }
    for (int j = t; j < pw.nJ; j += kF64Threads) {
      s.xJ[j] = a.xJ[pw.sJ + j];
      s.fJ[j] = a.fJ[pw.sJ + j];
    }
    __syncthreads();
    const int total = pw.nI * pw.nJ;
    for (int t0 = 0; t0 < total; t0 += kF64Tile) {
      if (t < kF64Tile) {
        const int flat = t0 + t;
        if (flat < total) {
          const int i = flat / pw.nJ, j = flat - (flat / pw.nJ) * pw.nJ;
          const float4 xi = s.xI[i], xj = s.xJ[j];
          s.r[t][0] = (double)xj.x - (double)xi.x;
          s.r[t][1] = (double)xj.y - (double)xi.y;
          s.r[t][2] = (double)xj.z - (double)xi.z;
          s.ei[t] = (int16_t)i;
          s.ej[t] = (int16_t)j;
        } else {
          s.r[t][0] = 1.0;
          s.r[t][1] = s.r[t][2] = 0.0;
          s.ei[t] = -1;
        }
      }
      __syncthreads();
      f64_tile(s, w);
      if (t < kF64Tile && s.ei[t] >= 0) {
        const int i = s.ei[t], j = s.ej[t];
        double M[9];
#pragma unroll
        for (int q = 0; q < 9; q++) M[q] = s.y[t][q];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = r + 1; c < 3; c++) {
            const double v = 0.5 * (M[3 * r + c] + M[3 * c + r]);
            M[3 * r + c] = v;
            M[3 * c + r] = v;
          }
        const float4 fj = s.fJ[j];
        const double fx = fj.x, fy = fj.y, fz = fj.z;
        atomicAdd(&s.uI[i][0], M[0] * fx + M[1] * fy + M[2] * fz);
        atomicAdd(&s.uI[i][1], M[3] * fx + M[4] * fy + M[5] * fz);
        atomicAdd(&s.uI[i][2], M[6] * fx + M[7] * fy + M[8] * fz);
      }
    }
    __syncthreads();
    for (int q = t; q < 3 * pw.nI; q += kF64Threads) atomicAdd(&a.uI[3 * (size_t)pw.sI + q], (&s.uI[0][0])[q]);
  }
}

}  // namespace

void launch_dense_f64(const NearArgs& a, const MlpF32& w, int* work_counter, int num_sms, cudaStream_t s) {
  if (a.nwork <= 0) return;
  const size_t smem = sizeof(F64Smem);
  HIGNN_CUDA(cudaFuncSetAttribute(k_dense_rows_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  HIGNN_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(int), s));
  const int grid = a.nwork < num_sms ? a.nwork : num_sms;
  k_dense_rows_f64<<<grid, kF64Threads, smem, s>>>(a, w, work_counter);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
