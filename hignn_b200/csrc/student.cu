// Student network for far-field entries: trained on the device, evaluated inside ACA.
//
// The student replaces the two-body teacher network only for admissible
// (far) blocks. Architecture: 3 -> 32 -> 32 -> 32 -> 9 with SiLU, on the input
// encoding x = r_hat * ln(|r| / 2). It predicts the residual of the teacher's
// inner output with respect to the Rotne-Prager-Yamakawa tensor of two unit
// spheres, so that
//     y(r) = rpy(r) + net(x),  M(r) = (y + I) / |r|  (the teacher's wrapper,
//     python/convert.py:11-20), rpy(r) = 0.75 [(1 + 2/(3 r^2)) I + (1 - 2/r^2) r_hat r_hat^T] - I.
// RPY carries the smooth long-range physics; the network learns the part of
// the teacher that is smooth on far-field scales.
//
// Training (all on the device, FP32): teacher evaluations at separations drawn
// log-uniform in [r_min, r_max] with uniform directions (hash-based counter
// RNG), targets = teacher inner output - rpy; loss = mean squared error over
// all outputs of a mini-batch; one kernel computes forward, backward and the
// per-CTA gradient sums of 128 samples, a second sums the CTA partials, a
// third applies Adam with a cosine-decayed learning rate.
#include <cmath>
#include <cstdint>

#include <cuda_fp16.h>

#include "common.h"
#include "kernels.h"
#include "tc_mlp.cuh"

namespace hignn {

namespace {

constexpr int kS = 32;  // hidden width
constexpr int kOffW1 = 0, kOffB1 = 96, kOffW2 = 128, kOffB2 = 1152, kOffW3 = 1184, kOffB3 = 2208, kOffW4 = 2240,
              kOffB4 = 2528;
static_assert(kOffB4 + 9 == kStudentParams, "student layout");

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ float u01(uint64_t h) { return ((h >> 40) + 0.5f) * (1.0f / 16777216.0f); }

__device__ __forceinline__ void rpy_inner(float rx, float ry, float rz, float (&y)[9]) {
  const float d2 = rx * rx + ry * ry + rz * rz;
  const float inv2 = 1.0f / d2;
  const float a = 0.75f * (1.0f + (2.0f / 3.0f) * inv2) - 1.0f;
  const float b = 0.75f * (1.0f - 2.0f * inv2) * inv2;  // multiplies r r^T (r_hat r_hat^T / ... folded)
  const float r[3] = {rx, ry, rz};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) y[3 * i + j] = b * r[i] * r[j] + (i == j ? a : 0.0f);
}

__device__ __forceinline__ float silu_fast(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// Forward of the student on one feature; p points at the 2537 parameters (shared memory).
__device__ __forceinline__ void student_forward(const float* __restrict__ p, float rx, float ry, float rz,
                                                float (&M)[9]) {
  const float nr = sqrtf(rx * rx + ry * ry + rz * rz);
  if (nr < 1e-5f) {
#pragma unroll
    for (int o = 0; o < 9; o++) M[o] = (o == 0 || o == 4 || o == 8) ? 1.0f : 0.0f;
    return;
  }
  const float sc = __logf(nr * 0.5f) / nr;
  const float x0 = rx * sc, x1 = ry * sc, x2 = rz * sc;
  float h1[kS], h2[kS];
#pragma unroll
  for (int k = 0; k < kS; k++) {
    const float z = fmaf(p[kOffW1 + 3 * k + 2], x2, fmaf(p[kOffW1 + 3 * k + 1], x1, fmaf(p[kOffW1 + 3 * k], x0, p[kOffB1 + k])));
    h1[k] = silu_fast(z);
  }
  // rows of W2, W3, W4 start on 16-byte boundaries (offsets 128, 1184, 2240 floats): one
  // 128-bit shared-memory broadcast feeds four FMAs
#pragma unroll
  for (int k = 0; k < kS; k++) {
    float z = p[kOffB2 + k];
    const float4* w = reinterpret_cast<const float4*>(p + kOffW2 + kS * k);
#pragma unroll
    for (int m = 0; m < kS / 4; m++) {
      const float4 wv = w[m];
      z = fmaf(wv.x, h1[4 * m], z);
      z = fmaf(wv.y, h1[4 * m + 1], z);
      z = fmaf(wv.z, h1[4 * m + 2], z);
      z = fmaf(wv.w, h1[4 * m + 3], z);
    }
    h2[k] = silu_fast(z);
  }
#pragma unroll
  for (int k = 0; k < kS; k++) {
    float z = p[kOffB3 + k];
    const float4* w = reinterpret_cast<const float4*>(p + kOffW3 + kS * k);
#pragma unroll
    for (int m = 0; m < kS / 4; m++) {
      const float4 wv = w[m];
      z = fmaf(wv.x, h2[4 * m], z);
      z = fmaf(wv.y, h2[4 * m + 1], z);
      z = fmaf(wv.z, h2[4 * m + 2], z);
      z = fmaf(wv.w, h2[4 * m + 3], z);
    }
    h1[k] = silu_fast(z);  // h3
  }
  float y[9];
  rpy_inner(rx, ry, rz, y);
#pragma unroll
  for (int o = 0; o < 9; o++) {
    float z = p[kOffB4 + o];
    const float4* w = reinterpret_cast<const float4*>(p + kOffW4 + kS * o);
#pragma unroll
    for (int m = 0; m < kS / 4; m++) {
      const float4 wv = w[m];
      z = fmaf(wv.x, h1[4 * m], z);
      z = fmaf(wv.y, h1[4 * m + 1], z);
      z = fmaf(wv.z, h1[4 * m + 2], z);
      z = fmaf(wv.w, h1[4 * m + 3], z);
    }
    y[o] += z;
  }
#pragma unroll
  for (int o = 0; o < 9; o++) {
    float v = y[o];
    if (o == 0 || o == 4 || o == 8) v += 1.0f;
    M[o] = v / nr;
  }
}

__global__ void k_student_samples(float* __restrict__ r, int64_t n, uint64_t seed, float rmin, float rmax) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const uint64_t h0 = mix64(seed ^ (uint64_t)(4 * s)), h1 = mix64(h0 ^ 0x1234567ull), h2 = mix64(h1 ^ 0x89ABCDEFull);
  const float cz = 2.0f * u01(h0) - 1.0f;               // uniform direction
  const float ph = 6.283185307179586f * u01(h1);
  const float sz = sqrtf(fmaxf(0.0f, 1.0f - cz * cz));
  const float lo = logf(rmin), hi = logf(rmax);
  const float d = expf(lo + (hi - lo) * u01(h2));      // log-uniform distance
  r[3 * s] = d * sz * cosf(ph);
  r[3 * s + 1] = d * sz * sinf(ph);
  r[3 * s + 2] = d * cz;
}

// teacher M -> training target: (M |r| - I) - rpy(r)
__global__ void k_student_targets(const float* __restrict__ r, float* __restrict__ t, int64_t n) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float rx = r[3 * s], ry = r[3 * s + 1], rz = r[3 * s + 2];
  const float nr = sqrtf(rx * rx + ry * ry + rz * rz);
  float y[9];
  rpy_inner(rx, ry, rz, y);
#pragma unroll
  for (int o = 0; o < 9; o++) {
    float v = t[9 * s + o] * nr;
    if (o == 0 || o == 4 || o == 8) v -= 1.0f;
    t[9 * s + o] = v - y[o];
  }
}

constexpr int kGradThreads = 128;

struct GradSmem {
  float p[kStudentParams + 7];
  float x[kGradThreads][4];
  float h1[kGradThreads][kS + 1], h2[kGradThreads][kS + 1], h3[kGradThreads][kS + 1];
  float d1[kGradThreads][kS + 1], d2[kGradThreads][kS + 1], d3[kGradThreads][kS + 1];
  float dy[kGradThreads][9];
  float loss[kGradThreads / 32];
};

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

// Forward + backward of 128 samples per CTA; writes the CTA's gradient sum and loss sum.
// idx == nullptr: samples [base, base + 128); else samples idx[...] (a mini-batch).
__global__ void __launch_bounds__(kGradThreads)
    k_student_grad(const float* __restrict__ params, const float* __restrict__ r, const float* __restrict__ t,
                   int64_t nsamples, int64_t batch, uint64_t step_seed, float* __restrict__ partial,
                   float* __restrict__ loss_partial, float scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradSmem& s = *reinterpret_cast<GradSmem*>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < kStudentParams; i += blockDim.x) s.p[i] = params[i];
  __syncthreads();
  const int64_t gi = (int64_t)blockIdx.x * kGradThreads + tid;
  const bool valid = gi < batch;
  int64_t si = gi;
  if (step_seed != 0) si = (int64_t)(mix64(step_seed ^ (uint64_t)gi) % (uint64_t)nsamples);
  float l = 0.0f;
  // forward
  {
    float rx = 0.f, ry = 0.f, rz = 1.f;
    if (valid) {
      rx = r[3 * si];
      ry = r[3 * si + 1];
      rz = r[3 * si + 2];
    }
    const float nr = sqrtf(rx * rx + ry * ry + rz * rz);
    const float sc = logf(nr * 0.5f) / nr;
    const float x[3] = {rx * sc, ry * sc, rz * sc};
    s.x[tid][0] = x[0];
    s.x[tid][1] = x[1];
    s.x[tid][2] = x[2];
    float z1[kS], z2[kS], z3[kS];
    for (int k = 0; k < kS; k++) {
      z1[k] = s.p[kOffB1 + k] + s.p[kOffW1 + 3 * k] * x[0] + s.p[kOffW1 + 3 * k + 1] * x[1] +
              s.p[kOffW1 + 3 * k + 2] * x[2];
      s.h1[tid][k] = z1[k] * sigm(z1[k]);
    }
    for (int k = 0; k < kS; k++) {
      float z = s.p[kOffB2 + k];
      for (int m = 0; m < kS; m++) z += s.p[kOffW2 + kS * k + m] * s.h1[tid][m];
      z2[k] = z;
      s.h2[tid][k] = z * sigm(z);
    }
    for (int k = 0; k < kS; k++) {
      float z = s.p[kOffB3 + k];
      for (int m = 0; m < kS; m++) z += s.p[kOffW3 + kS * k + m] * s.h2[tid][m];
      z3[k] = z;
      s.h3[tid][k] = z * sigm(z);
    }
    float dy[9];
    for (int o = 0; o < 9; o++) {
      float z = s.p[kOffB4 + o];
      for (int m = 0; m < kS; m++) z += s.p[kOffW4 + kS * o + m] * s.h3[tid][m];
      const float e = valid ? z - t[9 * si + o] : 0.0f;
      l += e * e;
      dy[o] = 2.0f * e * scale;
      s.dy[tid][o] = dy[o];
    }
    // backward through the hidden layers (silu'(z) = sg (1 + z (1 - sg)))
    float d3[kS];
    for (int k = 0; k < kS; k++) {
      float g = 0.f;
      for (int o = 0; o < 9; o++) g += s.p[kOffW4 + kS * o + k] * dy[o];
      const float sg = sigm(z3[k]);
      d3[k] = g * sg * (1.0f + z3[k] * (1.0f - sg));
      s.d3[tid][k] = d3[k];
    }
    float d2[kS];
    for (int m = 0; m < kS; m++) {
      float g = 0.f;
      for (int k = 0; k < kS; k++) g += s.p[kOffW3 + kS * k + m] * d3[k];
      const float sg = sigm(z2[m]);
      d2[m] = g * sg * (1.0f + z2[m] * (1.0f - sg));
      s.d2[tid][m] = d2[m];
    }
    for (int m = 0; m < kS; m++) {
      float g = 0.f;
      for (int k = 0; k < kS; k++) g += s.p[kOffW2 + kS * k + m] * d2[k];
      const float sg = sigm(z1[m]);
      s.d1[tid][m] = g * sg * (1.0f + z1[m] * (1.0f - sg));
    }
  }
  // loss
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((tid & 31) == 0) s.loss[tid >> 5] = l;
  __syncthreads();
  // gradient sums over the CTA's samples (parameter entries spread over threads)
  float* out = partial + (size_t)blockIdx.x * kStudentParams;
  for (int q = tid; q < kStudentParams; q += blockDim.x) {
    float g = 0.f;
    if (q < kOffB1) {
      const int k = q / 3, c = q % 3;
      for (int j = 0; j < kGradThreads; j++) g += s.d1[j][k] * s.x[j][c];
    } else if (q < kOffW2) {
      const int k = q - kOffB1;
      for (int j = 0; j < kGradThreads; j++) g += s.d1[j][k];
    } else if (q < kOffB2) {
      const int k = (q - kOffW2) / kS, m = (q - kOffW2) % kS;
      for (int j = 0; j < kGradThreads; j++) g += s.d2[j][k] * s.h1[j][m];
    } else if (q < kOffW3) {
      const int k = q - kOffB2;
      for (int j = 0; j < kGradThreads; j++) g += s.d2[j][k];
    } else if (q < kOffB3) {
      const int k = (q - kOffW3) / kS, m = (q - kOffW3) % kS;
      for (int j = 0; j < kGradThreads; j++) g += s.d3[j][k] * s.h2[j][m];
    } else if (q < kOffW4) {
      const int k = q - kOffB3;
      for (int j = 0; j < kGradThreads; j++) g += s.d3[j][k];
    } else if (q < kOffB4) {
      const int o = (q - kOffW4) / kS, m = (q - kOffW4) % kS;
      for (int j = 0; j < kGradThreads; j++) g += s.dy[j][o] * s.h3[j][m];
    } else {
      const int o = q - kOffB4;
      for (int j = 0; j < kGradThreads; j++) g += s.dy[j][o];
    }
    out[q] = g;
  }
  if (tid == 0) {
    float ls = 0.f;
    for (int w = 0; w < kGradThreads / 32; w++) ls += s.loss[w];
    loss_partial[blockIdx.x] = ls;
  }
}

__global__ void k_student_reduce(const float* __restrict__ partial, int nparts, float* __restrict__ grad,
                                 const float* __restrict__ loss_partial, float* __restrict__ loss_out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < kStudentParams) {
    float g = 0.f;
    for (int c = 0; c < nparts; c++) g += partial[(size_t)c * kStudentParams + q];
    grad[q] = g;
  }
  if (q == 0 && loss_out) {
    float l = 0.f;
    for (int c = 0; c < nparts; c++) l += loss_partial[c];
    *loss_out = l;
  }
}

__global__ void k_student_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                               float* __restrict__ m2, float lr, float b1t, float b2t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kStudentParams) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float gq = g[q];
  const float a = b1 * m1[q] + (1.0f - b1) * gq;
  const float v = b2 * m2[q] + (1.0f - b2) * gq * gq;
  m1[q] = a;
  m2[q] = v;
  const float mh = a / (1.0f - b1t), vh = v / (1.0f - b2t);
  p[q] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_student_eval(const float* __restrict__ params, const float* __restrict__ r, float* __restrict__ y,
                               int64_t n) {
  __shared__ __align__(16) float p[kStudentParams];
  for (int i = threadIdx.x; i < kStudentParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    float M[9];
    student_forward(p, r[3 * s], r[3 * s + 1], r[3 * s + 2], M);
#pragma unroll
    for (int o = 0; o < 9; o++) y[9 * s + o] = M[o];
  }
}

// ---------------------------------------------------------------- student queries on tcgen05
// ACA column (which = 0) / row (which = 1) queries of all active blocks with the student, 128
// entries per tile and one tile at a time per CTA:
// every thread owns one entry (row) and one tensor-memory lane. Layer 1 (3 -> 32) runs in FP32 on
// the CUDA cores; layers 2, 3 (32 -> 32) and 4 (32 -> 9, padded to 16) are tcgen05 MMAs, M = 128,
// with FP16 operands (the A operand in tensor memory, the weights in shared memory as 128-byte
// swizzled K-major tiles padded to K = 64) and FP32 accumulation. SiLU between layers is
// z / 2 (1 + tanh(z / 2)) on FP16 pairs (one tanh.approx.f16x2 per pair), written back as the
// next A operand. A tile's three MMA rounds wait on one another, so several CTAs share an SM
// (64 tensor-memory columns each: A [0, 16), layer 2/3 accumulator [16, 48), layer 4 [48, 64)).
// Waits are bounded; a timeout records an error code and the CTA stops after draining its MMAs.
constexpr int kStcThreads = 128;
constexpr uint32_t kStcA = 0, kStcD = 16, kStcD4 = 48, kStcCols = 64;
constexpr long long kStcWait = 4000000000LL;

struct StcSmem {
  uint8_t w2[32 * 128];  // 32 rows (outputs) x 64 K (32 used), FP16, swizzled
  uint8_t w3[32 * 128];
  uint8_t w4[16 * 128];  // 9 rows used
  float w1b1[32 * 4];    // W1 row k (3), b1[k]
  float b2[32], b3[32], b4[16];
  uint64_t bar;
  uint32_t tmem;
};
// Eight CTAs per SM (8 x 64 tensor-memory columns): 26 KB of shared memory and at most 64
// registers per thread let eight fit.
constexpr size_t kStcSmemBytes = 26 * 1024;
static_assert(sizeof(StcSmem) + 1024 <= kStcSmemBytes, "student tile shared memory");

__device__ __forceinline__ uint32_t stc_swz(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + (((k >> 3) ^ (row & 7)) << 4) + (k & 7) * 2);
}

// SiLU of two FP32 pre-activations as one FP16 pair: (z / 2)(1 + tanh(z / 2))
__device__ __forceinline__ uint32_t silu_f16x2(float z0, float z1) {
  const __half2 hz = __floats2half2_rn(0.5f * z0, 0.5f * z1);
  uint32_t t;
  asm("tanh.approx.f16x2 %0, %1;\n" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t*>(&hz)));
  const __half2 r = __hfma2(hz, *reinterpret_cast<const __half2*>(&t), hz);
  return *reinterpret_cast<const uint32_t*>(&r);
}

__global__ void __launch_bounds__(kStcThreads, 8) k_far_student_tc(FarArgs a, const float* __restrict__ params, int which,
                                                                int* err) {
  extern __shared__ uint8_t raw[];
  const uint32_t rb = tc::saddr(raw);
  StcSmem& S = *reinterpret_cast<StcSmem*>(raw + (((rb + 1023u) & ~1023u) - rb));
  const int tid = threadIdx.x, warp = tid >> 5;
  const int nact = a.ctr[kCtrActive];
  const int tot = which ? a.ctr[kCtrTotJ] : a.ctr[kCtrTotI];
  const int ntiles = (tot + kStcThreads - 1) / kStcThreads;
  if ((int)blockIdx.x >= ntiles) return;
  // weights: FP16 swizzled tiles of W2, W3, W4 (rows = outputs, K = inputs), FP32 W1/b1 and biases
  for (int i = tid; i < 32 * 128 / 4; i += kStcThreads) {
    reinterpret_cast<uint32_t*>(S.w2)[i] = 0u;
    reinterpret_cast<uint32_t*>(S.w3)[i] = 0u;
    if (i < 16 * 128 / 4) reinterpret_cast<uint32_t*>(S.w4)[i] = 0u;
  }
  __syncthreads();
  for (int i = tid; i < 32 * 32; i += kStcThreads) {
    const int n = i >> 5, k = i & 31;
    *reinterpret_cast<__half*>(S.w2 + stc_swz(n, k)) = __float2half_rn(params[kOffW2 + i]);
    *reinterpret_cast<__half*>(S.w3 + stc_swz(n, k)) = __float2half_rn(params[kOffW3 + i]);
    if (n < 9) *reinterpret_cast<__half*>(S.w4 + stc_swz(n, k)) = __float2half_rn(params[kOffW4 + i]);
  }
  if (tid < 32) {
    S.w1b1[4 * tid] = params[kOffW1 + 3 * tid];
    S.w1b1[4 * tid + 1] = params[kOffW1 + 3 * tid + 1];
    S.w1b1[4 * tid + 2] = params[kOffW1 + 3 * tid + 2];
    S.w1b1[4 * tid + 3] = params[kOffB1 + tid];
    S.b2[tid] = params[kOffB2 + tid];
    S.b3[tid] = params[kOffB3 + tid];
    S.b4[tid & 15] = (tid & 15) < 9 ? params[kOffB4 + (tid & 15)] : 0.f;
  }
  if (tid == 0) {
    tc::mbar_init(&S.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (warp == 0) tc::tmem_alloc(&S.tmem, kStcCols);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tb = S.tmem, tl = tb + ((uint32_t)(32 * warp) << 16);
  const uint64_t d2 = tc::sdesc(tc::saddr(S.w2)), d3 = tc::sdesc(tc::saddr(S.w3)), d4 = tc::sdesc(tc::saddr(S.w4));
  const int32_t* pre = which ? a.preJ : a.preI;
  uint32_t phase = 0;
  bool ok = true;
  // one MMA round: everyone's A is in tensor memory; thread 0 issues, all wait for the commit
  // one MMA round: everyone's A is in tensor memory; thread 0 issues (issue), all wait for the
  // commit (await); work that does not touch tensor memory may run in between
  auto issue = [&](uint64_t bdesc, uint32_t d, uint32_t idesc) {
    tc::tmem_wait_st();
    tc::fence_before();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      tc::mma_ts(tb + d, tb + kStcA, bdesc, idesc, 0u);
      tc::mma_ts(tb + d, tb + kStcA + 8, bdesc + 2, idesc, 1u);
      tc::mma_commit(&S.bar);
    }
  };
  auto await = [&]() {
    const long long t0 = clock64();
    while (!tc::mbar_try_sleep(&S.bar, phase & 1, 2000u)) {
      if (clock64() - t0 > kStcWait) {
        atomicCAS(err, 0, 71);
        ok = false;
        break;
      }
    }
    phase++;
    tc::fence_after();
    ok = __syncthreads_and(ok);
  };
  // The entry of this thread in tile t: its block through a 128-way search of the active blocks'
  // row prefix (all threads probe, three rounds for up to 2M blocks), then the positions.
  struct Entry {
    float rx, ry, rz;
    pool_t* dst;
  };
  auto lookup = [&](int t) {
    Entry en{0.f, 0.f, 0.f, nullptr};
    const int g0 = t * kStcThreads, g = g0 + tid;
    int lo = 0, hi = nact;  // pre[lo] <= g0 < pre[hi]
    while (hi - lo > 1) {
      const int step = (hi - lo + kStcThreads - 1) / kStcThreads;
      const int p = lo + tid * step;
      const int cnt = __syncthreads_count(tid > 0 && p < hi && pre[p] <= g0);
      lo += cnt * step;
      hi = min(hi, lo + step);
    }
    if (g < tot) {
      while (pre[lo + 1] <= g) lo++;
      const int b = a.act[lo];
      const int loc = g - pre[lo];
      const FarBlock bk = a.blocks[b];
      const int k = a.state[b].k;
      float4 xi, xj;
      if (which == 0) {
        xj = a.x[bk.sJ + a.cols[(size_t)b * a.ldr + k]];
        xi = a.x[bk.sI + loc];
        en.dst = a.C + 9 * (bk.cOff + (int64_t)k * bk.nI + loc);
      } else {
        xj = a.x[bk.sJ + loc];
        xi = a.x[bk.sI + a.rows[(size_t)b * a.ldr + k]];
        en.dst = a.Q + 9 * (bk.qOff + (int64_t)k * bk.nJ + loc);
      }
      en.rx = xj.x - xi.x, en.ry = xj.y - xi.y, en.rz = xj.z - xi.z;
    }
    return en;
  };
  Entry cur = lookup(blockIdx.x);
  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const float rx = cur.rx, ry = cur.ry, rz = cur.rz;
    const float nr = sqrtf(rx * rx + ry * ry + rz * rz);
    const float sc = nr >= 1e-5f ? __logf(nr * 0.5f) / nr : 0.f;
    const float x0 = rx * sc, x1 = ry * sc, x2 = rz * sc;
    {  // layer 1 -> A
      uint32_t pk[16];
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const float4 w0 = *reinterpret_cast<const float4*>(&S.w1b1[8 * j]);
        const float4 w1 = *reinterpret_cast<const float4*>(&S.w1b1[8 * j + 4]);
        pk[j] = silu_f16x2(fmaf(w0.z, x2, fmaf(w0.y, x1, fmaf(w0.x, x0, w0.w))),
                           fmaf(w1.z, x2, fmaf(w1.y, x1, fmaf(w1.x, x0, w1.w))));
      }
      tc::tmem_st16(tl + kStcA, pk);
    }
    // layers 2 and 3; the next tile's entries are fetched while layer 2 runs
    Entry nxt{0.f, 0.f, 0.f, nullptr};
    for (int l = 0; l < 2; l++) {
      issue(l == 0 ? d2 : d3, kStcD, tc::idesc_f16x(128, 32));
      if (l == 0 && t + (int)gridDim.x < ntiles) nxt = lookup(t + gridDim.x);
      await();
      if (!ok) break;
      uint32_t v[32];
      tc::tmem_ld32(tl + kStcD, v);
      tc::tmem_wait_ld();
      const float* bb = l == 0 ? S.b2 : S.b3;
      uint32_t pk[16];
#pragma unroll
      for (int j = 0; j < 16; j++)
        pk[j] = silu_f16x2(__uint_as_float(v[2 * j]) + bb[2 * j], __uint_as_float(v[2 * j + 1]) + bb[2 * j + 1]);
      tc::tmem_st16(tl + kStcA, pk);
    }
    if (!ok) break;
    issue(d4, kStcD4, tc::idesc_f16x(128, 16));
    await();
    if (!ok) break;
    uint32_t v[16];
    tc::tmem_ld16(tl + kStcD4, v);
    tc::tmem_wait_ld();
    if (cur.dst) {
      float M[9];
      if (nr < 1e-5f) {
#pragma unroll
        for (int o = 0; o < 9; o++) M[o] = (o == 0 || o == 4 || o == 8) ? 1.0f : 0.0f;
      } else {
        float y[9];
        rpy_inner(rx, ry, rz, y);
        const float inv_nr = 1.0f / nr;  // one division, not nine: the MUFU is this kernel's busiest unit
#pragma unroll
        for (int o = 0; o < 9; o++) {
          float z = y[o] + __uint_as_float(v[o]) + S.b4[o];
          if (o == 0 || o == 4 || o == 8) z += 1.0f;
          M[o] = z * inv_nr;
        }
      }
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++)
          cur.dst[3 * r + c] = (r == c) ? M[3 * r + c] : 0.5f * (M[3 * r + c] + M[3 * c + r]);  // as FP64, exact
    }
    cur = nxt;
  }
  // no MMA of this CTA may be in flight when its tensor memory is freed
  if (tid == 0) {
    tc::mma_commit(&S.bar);
    const long long t0 = clock64();
    while (!tc::mbar_try(&S.bar, phase & 1) && clock64() - t0 < kStcWait) {
    }
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0) tc::tmem_dealloc(tb, kStcCols);
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(a.evals, (unsigned long long)tot);
}

}  // namespace

size_t student_grad_smem() { return sizeof(GradSmem); }

void launch_student_samples(float* r, int64_t n, uint64_t seed, float rmin, float rmax, cudaStream_t s) {
  if (n <= 0) return;
  k_student_samples<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(r, n, seed, rmin, rmax);
  HIGNN_CHECK_LAUNCH();
}

void launch_student_targets(const float* r, float* t, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  k_student_targets<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(r, t, n);
  HIGNN_CHECK_LAUNCH();
}

// Gradient of mean((net(x) - t)^2) over a batch: samples [0, batch) of (r, t) when step_seed == 0,
// else batch random draws from nsamples. partial: [ceil(batch/128)][kStudentParams].
void launch_student_grad(const float* params, const float* r, const float* t, int64_t nsamples, int64_t batch,
                         uint64_t step_seed, float* partial, float* loss_partial, float* grad, float* loss,
                         cudaStream_t s) {
  const int nparts = (int)((batch + kGradThreads - 1) / kGradThreads);
  const size_t smem = sizeof(GradSmem);
  HIGNN_CUDA(cudaFuncSetAttribute(k_student_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const float scale = 1.0f / (9.0f * (float)batch);
  k_student_grad<<<nparts, kGradThreads, smem, s>>>(params, r, t, nsamples, batch, step_seed, partial, loss_partial,
                                                    scale);
  HIGNN_CHECK_LAUNCH();
  k_student_reduce<<<(kStudentParams + 255) / 256, 256, 0, s>>>(partial, nparts, grad, loss_partial, loss);
  HIGNN_CHECK_LAUNCH();
}

void launch_student_adam(float* p, const float* g, float* m1, float* m2, float lr, float b1t, float b2t,
                         cudaStream_t s) {
  k_student_adam<<<(kStudentParams + 255) / 256, 256, 0, s>>>(p, g, m1, m2, lr, b1t, b2t);
  HIGNN_CHECK_LAUNCH();
}

void launch_student_eval(const float* params, const float* r, float* y, int64_t n, int num_sms, cudaStream_t s) {
  if (n <= 0) return;
  const int64_t blocks = (n + 255) / 256;
  k_student_eval<<<(unsigned)(blocks < 8 * num_sms ? blocks : 8 * num_sms), 256, 0, s>>>(params, r, y, n);
  HIGNN_CHECK_LAUNCH();
}

void launch_far_student(const FarArgs& a, const float* params, int which, int* err, int num_sms, cudaStream_t s) {
  set_max_dynamic_smem(k_far_student_tc, kStcSmemBytes, s);
  k_far_student_tc<<<8 * num_sms, kStcThreads, kStcSmemBytes, s>>>(a, params, which, err);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
