// Two-body network on the 5th-generation tensor cores (tcgen05, TMEM), 128 evaluations per tile.
//
// All three layers are tcgen05 MMAs with FP32 accumulation in tensor memory:
//   layer 1 (3 -> 128): one K = 16 BF16 MMA on split operands. Each feature r is
//       written as r_hi + r_lo (two BF16 numbers) and each W1 entry as W_hi + W_lo,
//       so the row [r_hi, r_lo, r_hi, 1, 1] against [W_hi, W_hi, W_lo, b1_hi, b1_lo]
//       gives W1 r + b1 to about 2^-16 relative, bias included;
//   layer 2 (128 -> 512): four quarters of N = 128, K = 128 (BF16);
//   layer 3 (512 -> 9): N = 32, K = 512 (BF16), W3 split into a BF16 high part
//       (rows 0-8) and a BF16 residual (rows 16-24): W3 rounding is the dominant
//       systematic error of a plain BF16 layer 3, and the split removes it.
// Between layers the epilogue warps read the accumulator (tcgen05.ld), add the
// FP32 layer-2 bias, round to BF16 pairs and apply tanh.approx.bf16x2 (two per
// MUFU op), and write the pairs back into tensor memory as the next A operand.
//
// Two tile contexts per CTA so that tanh work of one overlaps the MMAs of the
// other. CTA = 17 warps:
//   warps 0-7   epilogue group 0 (context 0), warps 8-15 epilogue group 1;
//               warp w reaches TMEM lanes 32*(w%4)..+31, so the evaluation (row)
//               e = 32*(w%4) + lane of a context is handled by two threads
//               (warps w and w+4 of the group), each owning one half of every
//               row's columns;
//   warp 16     allocates tensor memory; one lane issues every MMA, serving the
//               two contexts as their operands become ready (non-blocking
//               mbarrier tests, so one context never holds up the other).
// Tensor memory (512 columns allocated), per context c at column 256c:
//   [  0, 64)  A1: tanh(layer 1) as packed BF16 pairs (A operand of layer 2)
//   [ 64,192)  slot: FP32 accumulator of layer 1, then of each layer-2 quarter
//              (128 hidden units); after the epilogue reads a quarter, its
//              tanh'd BF16 pairs are written back into slot columns [0,32)
//              (units 0-63, half 0) and [64,96) (units 64-127, half 1) -- each
//              half writes only columns it read itself -- as layer 3's A operand
//   [192,224)  layer-3 accumulator (hi part in columns 0-8, residual in 16-24)
//   [224,232)  A0: the split features (K = 16 BF16) of layer 1
// Shared memory: W2 (512 x 128), W3 (32 x 512) and W1 (128 x 16, in a 64-wide
// slab) as BF16 in the canonical K-major 128-byte-swizzle layout, loaded once
// per CTA; FP32 biases b2, b3; mbarriers.
//
// Per context and tile: features -> A0; MMA L1 -> slot; epilogue tanh -> A1;
// then for each quarter q: MMA L2(q) -> slot, epilogue bias + tanh -> A2(q) in
// the slot, MMA L3(q) -> D3. Every wait is bounded (about two seconds of
// clock): on a timeout the CTA records an error, stops issuing work, drains
// its MMAs and frees its tensor memory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace hignn {
namespace tc {

using hignn::TcWeights;

constexpr int kTile = 128;
constexpr int kGroupThreads = 256;
constexpr int kEpiThreads = 512;
constexpr int kThreads = 544;
constexpr int kMmaWarp = 16;
constexpr uint32_t kCtxCols = 256, kOffA1 = 0, kOffSlot = 64, kOffD3 = 192, kOffA0 = 224;
constexpr int kW2Bytes = kH2 * kH1 * 2;      // 131072
constexpr int kW3Rows = 32;
constexpr int kW3Bytes = kW3Rows * kH2 * 2;  // 32768
constexpr int kW1Bytes = kH1 * 64 * 2;       // 16384: 128 rows x one 64-wide K slab (K 0-15 used)
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

struct CtxBars {
  uint64_t a0_full, d1_full, a1_full, d2_full, a2_full, slot_free, d3_full, d3_free;
  int exit_flag;
  int pad;
};

struct alignas(1024) Smem {
  uint8_t w2[kW2Bytes];
  uint8_t w3[kW3Bytes];
  uint8_t w1[kW1Bytes];
  CtxBars ctx[2];
  uint64_t drain;
  uint32_t tmem_base;
  int abort_flag;
  alignas(16) float b2[kH2];  // FP32 layer-2 bias, added before rounding to BF16
  float b3[16];
};

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(b)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("{\n.reg .b64 st;\nmbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking test of a phase (never suspends the thread): the MMA lane polls two contexts.
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and raises the CTA abort flag) if the phase never completes.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int* abort_flag, int* err, int code) {
  const long long t0 = clock64();
  while (!mbar_try(b, parity)) {
    if (*(volatile int*)abort_flag) return false;
    if (clock64() - t0 > kWaitCycles) {
      atomicExch(abort_flag, 1);
      atomicCAS(err, 0, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(dst)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}

// D[tmem] (+)= A[tmem] * B[smem desc]^T, kind::f16 (BF16 inputs, FP32 accumulate)
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d),
      "r"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(saddr(bar))
               : "memory");
}

// 32 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
      "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]),
      "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]),
      "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}

// 4 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint32_t v0, uint32_t v1, uint32_t v2, uint32_t v3) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};\n" ::"r"(taddr), "r"(v0), "r"(v1), "r"(v2),
               "r"(v3)
               : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ uint32_t add_bf16x2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("add.rn.bf16x2 %0, %1, %2;\n" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t tanh_bf16x2(uint32_t x) {
  uint32_t y;
  asm("tanh.approx.bf16x2 %0, %1;\n" : "=r"(y) : "r"(x));
  return y;
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr_bytes & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;            // leading byte offset (unused by swizzled K-major): 16 B
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset between 8-row groups
  d |= (uint64_t)1 << 46;            // descriptor version of sm_100
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}
// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ------------------------------------------------------------------ per-CTA setup / teardown
__device__ __forceinline__ void cta_setup(Smem& s, const TcWeights& w) {
  const int t = threadIdx.x;
  const uint4* src2 = w.w2img;
  uint4* dst2 = reinterpret_cast<uint4*>(s.w2);
  for (int i = t; i < kW2Bytes / 16; i += blockDim.x) dst2[i] = src2[i];
  const uint4* src3 = w.w3img;
  uint4* dst3 = reinterpret_cast<uint4*>(s.w3);
  for (int i = t; i < kW3Bytes / 16; i += blockDim.x) dst3[i] = src3[i];
  const uint4* src1 = w.w1img;
  uint4* dst1 = reinterpret_cast<uint4*>(s.w1);
  for (int i = t; i < kW1Bytes / 16; i += blockDim.x) dst1[i] = src1[i];
  for (int i = t; i < kH2; i += blockDim.x) s.b2[i] = w.b2[i];
  if (t < 16) s.b3[t] = t < kOut ? w.b3[t] : 0.f;
  if (t == 0) {
    for (int c = 0; c < 2; c++) {
      CtxBars& b = s.ctx[c];
      mbar_init(&b.a0_full, kGroupThreads);
      mbar_init(&b.d1_full, 1);
      mbar_init(&b.a1_full, kGroupThreads);
      mbar_init(&b.d2_full, 1);
      mbar_init(&b.a2_full, kGroupThreads);
      mbar_init(&b.slot_free, 1);
      mbar_init(&b.d3_full, 1);
      mbar_init(&b.d3_free, kGroupThreads);
      b.exit_flag = 0;
    }
    mbar_init(&s.drain, 1);
    s.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // generic-proxy writes of the weight images must be visible to the tensor core (async proxy)
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if ((t >> 5) == kMmaWarp) tmem_alloc(&s.tmem_base, 512);
  fence_before();
  __syncthreads();
  fence_after();
}

__device__ __forceinline__ void cta_teardown(Smem& s) {
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == kMmaWarp) tmem_dealloc(s.tmem_base, 512);
}

// ------------------------------------------------------------------ MMA lane
// Non-blocking state machine per context; mma_loop returns when both epilogue groups
// raised their exit flags (or the CTA aborted / nothing progressed for kWaitCycles).
//   state 0: features of the next tile in A0 (and the slot free) -> layer 1
//   state 1: A1 written -> layer 2 of quarter q
//   state 2: A2(q) written (and, for q = 0, D3 read) -> layer 3 of quarter q
//   state 3: layer 3 of quarter q released the slot -> layer 2 of quarter q + 1
struct MmaCtx {
  uint32_t tile = 0, q = 0, state = 0, l2s = 0, l3s = 0;
  bool done = false;
};

__device__ __forceinline__ void issue_l2(uint32_t base, uint32_t q, uint32_t w2) {
  const uint32_t id_l2 = idesc_bf16(128, 128);
#pragma unroll
  for (uint32_t kk = 0; kk < 8; kk++) {
    const uint32_t bb = w2 + (kk >> 2) * (kH2 * 128) + q * (128 * 128) + (kk & 3) * 32;
    mma_ts(base + kOffSlot, base + kOffA1 + 8 * kk, sdesc(bb), id_l2, kk > 0);
  }
}

__device__ __forceinline__ bool mma_step(Smem& s, MmaCtx& x, uint32_t c, uint32_t tbase, uint32_t w1, uint32_t w2,
                                         uint32_t w3) {
  CtxBars& b = s.ctx[c];
  const uint32_t base = tbase + c * kCtxCols;
  if (x.state == 0) {
    if (!mbar_test(&b.a0_full, x.tile & 1)) return false;
    if (x.l3s > 0 && !mbar_test(&b.slot_free, (x.l3s - 1) & 1)) return false;
    fence_after();
    if (*(volatile int*)&b.exit_flag) {
      x.done = true;
      return true;
    }
    mma_ts(base + kOffSlot, base + kOffA0, sdesc(w1), idesc_bf16(128, 128), 0u);
    mma_commit(&b.d1_full);
    x.q = 0;
    x.state = 1;
    return true;
  }
  if (x.state == 1) {
    if (!mbar_test(&b.a1_full, x.tile & 1)) return false;
    fence_after();
    issue_l2(base, 0, w2);
    mma_commit(&b.d2_full);
    x.l2s++;
    x.state = 2;
    return true;
  }
  if (x.state == 3) {
    if (!mbar_test(&b.slot_free, (x.l3s - 1) & 1)) return false;
    fence_after();
    issue_l2(base, x.q, w2);
    mma_commit(&b.d2_full);
    x.l2s++;
    x.state = 2;
    return true;
  }
  // state 2: layer 3 of quarter q
  if (!mbar_test(&b.a2_full, (x.l2s - 1) & 1)) return false;
  if (x.q == 0 && x.tile > 0 && !mbar_test(&b.d3_free, (x.tile - 1) & 1)) return false;
  fence_after();
  const uint32_t id_l3 = idesc_bf16(128, kW3Rows);
#pragma unroll
  for (uint32_t kk = 0; kk < 8; kk++) {
    const uint32_t kg = x.q * 128 + kk * 16;  // global K of layer 3
    const uint32_t bb = w3 + (kg >> 6) * (kW3Rows * 128) + ((kg & 63) >> 3) * 16;
    const uint32_t a_off = kk < 4 ? 8 * kk : 64 + 8 * (kk - 4);  // A2 halves at slot columns 0 and 64
    mma_ts(base + kOffD3, base + kOffSlot + a_off, sdesc(bb), id_l3, (x.q > 0 || kk > 0) ? 1u : 0u);
  }
  mma_commit(&b.slot_free);
  x.l3s++;
  if (x.q == 3) {
    mma_commit(&b.d3_full);
    x.tile++;
    x.state = 0;
  } else {
    x.q++;
    x.state = 3;
  }
  return true;
}

__device__ __forceinline__ void mma_loop(Smem& s, int* err) {
  const uint32_t tbase = s.tmem_base;
  const uint32_t w1 = saddr(s.w1), w2 = saddr(s.w2), w3 = saddr(s.w3);
  MmaCtx x[2];
  long long last = clock64();
  while (!(x[0].done && x[1].done)) {
    bool prog = false;
    if (!x[0].done) prog |= mma_step(s, x[0], 0, tbase, w1, w2, w3);
    if (!x[1].done) prog |= mma_step(s, x[1], 1, tbase, w1, w2, w3);
    if (prog) {
      last = clock64();
    } else {
      if (*(volatile int*)&s.abort_flag) break;
      if (clock64() - last > kWaitCycles) {
        atomicExch(&s.abort_flag, 1);
        atomicCAS(err, 0, 11);
        break;
      }
    }
  }
  // drain: every MMA issued so far completes before tensor memory is released
  mma_commit(&s.drain);
  const long long t0 = clock64();
  while (!mbar_try(&s.drain, 0) && clock64() - t0 < kWaitCycles) {
  }
}

// ------------------------------------------------------------------ epilogue side
struct EpiState {
  uint32_t tile = 0, quarters = 0;
};

__device__ __forceinline__ int epi_group() { return threadIdx.x >> 8; }                      // context 0 / 1
__device__ __forceinline__ int epi_gthread() { return threadIdx.x & 255; }                   // 0..255 in group
__device__ __forceinline__ int epi_row() { return 32 * ((threadIdx.x >> 5) & 3) + (threadIdx.x & 31); }
__device__ __forceinline__ int epi_half() { return (threadIdx.x >> 7) & 1; }                 // column half
__device__ __forceinline__ void epi_bar() {
  if (epi_group() == 0)
    asm volatile("bar.sync 1, 256;\n" ::: "memory");
  else
    asm volatile("bar.sync 2, 256;\n" ::: "memory");
}

__device__ __forceinline__ float bf16_round(float x) { return __uint_as_float(pack_bf16(x, 0.f) << 16); }

// Layer-1 operand of one row: K = 16 BF16 values [r_hi(3), r_lo(3), r_hi(3), 1, 1, 0 x 5] packed in
// pairs; half 0 writes columns 0-3, half 1 columns 4-7.
__device__ __forceinline__ void write_features(uint32_t ta0, int h, float rx, float ry, float rz) {
  const float hx = bf16_round(rx), hy = bf16_round(ry), hz = bf16_round(rz);
  if (h == 0) {
    const float lx = rx - hx, ly = ry - hy, lz = rz - hz;  // exact in FP32
    tmem_st4(ta0, pack_bf16(hx, hy), pack_bf16(hz, lx), pack_bf16(ly, lz), pack_bf16(hx, hy));
  } else {
    tmem_st4(ta0 + 4, pack_bf16(hz, 1.f), pack_bf16(1.f, 0.f), 0u, 0u);
  }
}

// One tile for this thread's evaluation (row) with features r; writes M (row-major 3x3) into
// both threads of the row. Returns false if the CTA aborted. All 256 threads of the group
// call it together.
__device__ __forceinline__ bool run_tile(Smem& s, EpiState& st, float rx, float ry, float rz, float (&M)[9],
                                         int* err) {
  const int c = epi_group(), h = epi_half();
  CtxBars& b = s.ctx[c];
  const uint32_t tb = s.tmem_base + c * kCtxCols + ((uint32_t)(32 * ((threadIdx.x >> 5) & 3)) << 16);
  write_features(tb + kOffA0, h, rx, ry, rz);
  tmem_wait_st();
  fence_before();
  mbar_arrive(&b.a0_full);
  // layer 1 accumulator (bias included) -> tanh -> A1
  if (!mbar_wait(&b.d1_full, st.tile & 1, &s.abort_flag, err, 21)) return false;
  fence_after();
  {
    uint32_t out[32];
#pragma unroll
    for (int part = 0; part < 2; part++) {
      uint32_t v[32];
      tmem_ld32(tb + kOffSlot + 64 * h + 32 * part, v);
      tmem_wait_ld();
#pragma unroll
      for (int k = 0; k < 16; k++)
        out[16 * part + k] = tanh_bf16x2(pack_bf16(__uint_as_float(v[2 * k]), __uint_as_float(v[2 * k + 1])));
    }
    tmem_st32(tb + kOffA1 + 32 * h, out);
  }
  tmem_wait_st();
  fence_before();
  mbar_arrive(&b.a1_full);
  for (uint32_t q = 0; q < 4; q++) {
    if (!mbar_wait(&b.d2_full, st.quarters & 1, &s.abort_flag, err, 22)) return false;
    fence_after();
    const uint32_t col = tb + kOffSlot + 64 * h;
    uint32_t out[32];
#pragma unroll
    for (int part = 0; part < 2; part++) {
      uint32_t v[32];
      tmem_ld32(col + 32 * part, v);
      tmem_wait_ld();
      const float4* bb = reinterpret_cast<const float4*>(s.b2 + q * 128 + 64 * h + 32 * part);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const float4 bv = bb[k];
        uint32_t* o = out + 16 * part + 2 * k;
        o[0] = tanh_bf16x2(pack_bf16(__uint_as_float(v[4 * k + 0]) + bv.x, __uint_as_float(v[4 * k + 1]) + bv.y));
        o[1] = tanh_bf16x2(pack_bf16(__uint_as_float(v[4 * k + 2]) + bv.z, __uint_as_float(v[4 * k + 3]) + bv.w));
      }
    }
    tmem_st32(col, out);  // inside the columns this thread read itself
    tmem_wait_st();
    fence_before();
    mbar_arrive(&b.a2_full);
    st.quarters++;
  }
  if (!mbar_wait(&b.d3_full, st.tile & 1, &s.abort_flag, err, 23)) return false;
  fence_after();
  {
    uint32_t v[32];
    tmem_ld32(tb + kOffD3, v);
    tmem_wait_ld();
    fence_before();
    mbar_arrive(&b.d3_free);
    const float nr = sqrtf(rx * rx + ry * ry + rz * rz);
    const float inv = __frcp_rn(nr);
#pragma unroll
    for (int o = 0; o < 9; o++) {
      float y = __uint_as_float(v[o]) + __uint_as_float(v[16 + o]) + s.b3[o];
      const bool dg = (o == 0 || o == 4 || o == 8);
      if (dg) y += 1.0f;
      y = y * inv;
      if (nr < 1e-5f) y = dg ? 1.0f : 0.0f;
      M[o] = y;
    }
  }
  st.tile++;
  return true;
}

// Tells the MMA lane that this group has no more tiles (all 256 threads of the group call it).
__device__ __forceinline__ void epi_finish(Smem& s) {
  CtxBars& b = s.ctx[epi_group()];
  if (epi_gthread() == 0) *(volatile int*)&b.exit_flag = 1;
  epi_bar();
  mbar_arrive(&b.a0_full);
}

}  // namespace tc
}  // namespace hignn
