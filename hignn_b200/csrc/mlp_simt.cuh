// FP32 SIMT evaluation of the two-body network, 128 evaluations per tile.
//
// This is the "plain FP32" form: every layer in FP32 on the CUDA cores, the same
// arithmetic class as the reference's libtorch FP32 forward (src/CloseDot.cpp:233).
// Layer widths 3 -> 128 -> 512 -> 9. Every operation is a single correctly rounded
// FP32 operation in a fixed order (explicit fused multiply-adds, _rn intrinsics,
// the tanh of tanh_f32.cuh), so each output is a function of its feature alone:
//   h1[k] = tanh(fma(W1[k][2], r_z, fma(W1[k][1], r_y, fma(W1[k][0], r_x, b1[k]))))
//   h2[n] = tanh((sum_k fma(h1[k], W2[n][k], .), k ascending from 0) + b2[n])
//   y[o]  = (sum_n fma(h2[n], W3[o][n], .), n ascending from 0) + b3[o] (+ 1 on the
//           diagonal), divided by |r| = sqrt(fma(r_z, r_z, fma(r_y, r_y, r_x r_x))).
//
// Tile schedule (256 threads): layer 1 fills h1[k][e]; layer 2 runs in 8
// chunks of 64 hidden units, each a 128x64x128 register-tiled GEMM (8 evals x
// 4 units per thread) on W2 chunks double-buffered in shared memory with
// cp.async; each chunk is tanh'd into h2[n][e] and immediately folded into
// the 9 layer-3 outputs, so the 512-wide activation never leaves the SM.
#pragma once

#include <cuda_runtime.h>

#include "common.h"
#include "tanh_f32.cuh"

namespace hignn {
namespace simt {

constexpr int kThreads = 256;
constexpr int kTile = 128;
constexpr int kChunk = 64;
constexpr int kNumChunks = kH2 / kChunk;

struct Smem {
  float h1[kH1][kTile];           // 64 KB, [k][e]
  float w2[2][kH1][kChunk];       // 64 KB, W2^T chunks [k][n]
  float h2[kChunk][kTile];        // 32 KB, [n][e]
  float w3[kOut][kH2];            // 18 KB
  float b2[kH2];                  // 2 KB
  float4 w1b1[kH1];               // 2 KB
  float b3[16];
  float4 r[kTile];                // features (x, y, z, unused)
  float y[kTile][kOut + 1];       // network outputs after the wrapper
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Per-CTA weight staging (once per kernel).
__device__ __forceinline__ void load_weights(Smem& s, const MlpF32& w) {
  const int t = threadIdx.x;
  for (int i = t; i < kOut * kH2; i += kThreads) (&s.w3[0][0])[i] = w.w3[i];
  for (int i = t; i < kH2; i += kThreads) s.b2[i] = w.b2[i];
  for (int i = t; i < kH1; i += kThreads) s.w1b1[i] = w.w1b1[i];
  if (t < 16) s.b3[t] = t < kOut ? w.b3[t] : 0.f;
}

__device__ __forceinline__ void load_w2_chunk(Smem& s, const MlpF32& w, int chunk, int buf) {
  // 128 rows x 64 floats = 2048 x 16 B, 8 per thread
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    int idx = t + q * kThreads;  // 0..2047
    int k = idx >> 4, c4 = idx & 15;
    cp_async16(&s.w2[buf][k][c4 * 4], w.w2t + (size_t)k * kH2 + chunk * kChunk + c4 * 4);
  }
  cp_async_commit();
}

// Evaluates M(r) for s.r[0..127] (caller has written them and synchronized).
// On return s.y[e][0..8] holds M row-major and the block is synchronized.
__device__ __forceinline__ void mlp_tile(Smem& s, const MlpF32& w) {
  const int t = threadIdx.x;
  load_w2_chunk(s, w, 0, 0);
  // layer 1: h1[k][e] = tanh(W1[k] . r_e + b1[k])
  for (int idx = t; idx < kH1 * kTile; idx += kThreads) {
    const int k = idx / kTile, e = idx % kTile;
    const float4 wk = s.w1b1[k];
    const float4 r = s.r[e];
    s.h1[k][e] = tanh_f32(__fmaf_rn(wk.z, r.z, __fmaf_rn(wk.y, r.y, __fmaf_rn(wk.x, r.x, wk.w))));
  }
  const int tn = t & 15, te = t >> 4;   // layer-2 micro tile: evals te*8..+8, units tn*4..+4
  const int e3 = t & (kTile - 1), og = t >> 7;  // layer-3 owner: eval e3, outputs og*5..
  const int o0 = og * 5, on = og ? 4 : 5;
  float y3[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int c = 0; c < kNumChunks; c++) {
    const int buf = c & 1;
    cp_async_wait_all();
    __syncthreads();  // chunk c visible; previous chunk's h2 consumers done
    if (c + 1 < kNumChunks) load_w2_chunk(s, w, c + 1, buf ^ 1);
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
#pragma unroll 4
    for (int k = 0; k < kH1; k++) {
      const float4 a0 = *reinterpret_cast<const float4*>(&s.h1[k][te * 8]);
      const float4 a1 = *reinterpret_cast<const float4*>(&s.h1[k][te * 8 + 4]);
      const float4 b = *reinterpret_cast<const float4*>(&s.w2[buf][k][tn * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = __fmaf_rn(av[i], bv[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = tn * 4 + j;
      const float bias = s.b2[c * kChunk + n];
      float4 v0, v1;
      v0.x = tanh_f32(__fadd_rn(acc[0][j], bias));
      v0.y = tanh_f32(__fadd_rn(acc[1][j], bias));
      v0.z = tanh_f32(__fadd_rn(acc[2][j], bias));
      v0.w = tanh_f32(__fadd_rn(acc[3][j], bias));
      v1.x = tanh_f32(__fadd_rn(acc[4][j], bias));
      v1.y = tanh_f32(__fadd_rn(acc[5][j], bias));
      v1.z = tanh_f32(__fadd_rn(acc[6][j], bias));
      v1.w = tanh_f32(__fadd_rn(acc[7][j], bias));
      *reinterpret_cast<float4*>(&s.h2[n][te * 8]) = v0;
      *reinterpret_cast<float4*>(&s.h2[n][te * 8 + 4]) = v1;
    }
    __syncthreads();
    // layer 3 partial: y[e3][o] += sum_n h2[n][e3] * W3[o][c*64 + n]
#pragma unroll 8
    for (int n = 0; n < kChunk; n++) {
      const float h = s.h2[n][e3];
#pragma unroll
      for (int o = 0; o < 5; o++)
        if (o < on) y3[o] = __fmaf_rn(h, s.w3[o0 + o][c * kChunk + n], y3[o]);
    }
  }
  // wrapper of python/convert.py:11-20: (y + b3 + I) / |r|, identity for |r| < 1e-5
  const float4 r = s.r[e3];
  const float nr = __fsqrt_rn(__fmaf_rn(r.z, r.z, __fmaf_rn(r.y, r.y, __fmul_rn(r.x, r.x))));
  for (int o = 0; o < on; o++) {
    const int oo = o0 + o;
    float v = __fadd_rn(y3[o], s.b3[oo]);
    if (oo == 0 || oo == 4 || oo == 8) v = __fadd_rn(v, 1.0f);
    v = __fdiv_rn(v, nr);
    if (nr < 1e-5f) v = (oo == 0 || oo == 4 || oo == 8) ? 1.0f : 0.0f;
    s.y[e3][oo] = v;
  }
  __syncthreads();
}

}  // namespace simt
}  // namespace hignn
