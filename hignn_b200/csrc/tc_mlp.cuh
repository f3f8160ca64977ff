// Two-body network on the 5th-generation tensor cores (tcgen05, TMEM), 128 evaluations per tile.
//
// Layer 1 (3 -> 128) runs on the CUDA cores in FP32 (three FMAs per hidden unit from the
// features in registers); layers 2 and 3 are tcgen05 MMAs with FP32 accumulation in tensor
// memory:
//   layer 2 (128 -> 512): four quarters of N = 128, K = 128, FP16 operands;
//   layer 3 (512 -> 9): N = 16, K = 512, FP16 operands (W3 rows 0-8, rows 9-15 zero).
// FP16 rather than BF16 for layers 2 and 3: their operands are tanh outputs in [-1, 1] and
// weights well inside FP16's range, so the 11-bit significand costs no range and rounds 8x finer.
// The epilogue warps read a layer-2 accumulator (tcgen05.ld), round it to FP16 pairs, add the
// bias as FP16 pairs, apply tanh.approx.f16x2 and write the pairs back into tensor memory as
// layer 3's A operand; layer 1's tanh'd pairs go the same way into layer 2's A operand.
//
// The bound is the MUFU: 640 tanh per evaluation at 16 tanh per clock per SM (tanh.approx.f16x2
// issues at half the rate of tanh.approx.f32, measured on B200: packing saves issue slots, not
// MUFU time), i.e. 40 clocks per evaluation per SM, against ~32 clocks of tensor-pipe occupancy
// (every MMA holds the pipe >= ~64 cycles whatever its N). The schedule keeps the epilogue -- and
// so the MUFU -- from waiting on the tensor core. Per tile t the epilogue handles
//   quarter 0, quarter 1, the retirement of tile t-1, quarter 2, layer 1 of tile t+1, quarter 3
// and the MMA lane issues each layer-2 quarter two epilogue phases before it is read:
//   L2(t,0), L2(t,1) after layer 1 of t and quarter 3 of t-1; L2(t,2) after quarter 0;
//   L2(t,3) after quarter 1; L3(t,q) after quarter q, behind the layer-2 MMA issued with it.
// Layer 1 of tile t+1 is stored into A1 once quarter 3's accumulator is complete (the last MMA
// reading A1), so no layer-2 quarter of t+1 waits for a layer-1 MMA and its epilogue, and the
// first quarter of t+1 is on the tensor cores while quarter 3 of t is in the epilogue. Tile t-1
// is retired from the other of two layer-3 accumulators.
//
// CTA = 17 warps:
//   warps 0-15  epilogue; warp w reaches TMEM lanes 32 (w % 4) .. + 31, so the
//               evaluation (row) e = 32 (w % 4) + lane is handled by four
//               threads (part p = w / 4 owns hidden units 32p .. 32p + 31 of layer 1
//               and columns 32p .. 32p + 31 of every layer-2 quarter);
//   warp 16     allocates tensor memory; one lane issues every MMA.
// Tensor memory (512 columns allocated):
//   [  0, 64)  A1: tanh(layer 1) as packed FP16 pairs (A operand of layer 2)
//   [ 64,192)  slot 0 (quarters 0, 2) and [192,320) slot 1 (quarters 1, 3): FP32 accumulators
//   [320,384)  and [384,448): A2 of even / odd quarters, the tanh'd FP16 pairs of a quarter
//              (A operand of layer 3)
//   [448,464)  and [464,480): layer-3 accumulators of even / odd tiles (M in columns 0-8)
// Shared memory: W2 (512 x 128) and W3 (16 x 512) as FP16, canonical K-major 128-byte-swizzle
// layout, loaded once per CTA; FP32 (W1, b1) per hidden unit, b2 as FP16 pairs, FP32 b3; mbarriers. A
// barrier that completes twice per tile (the per-slot and per-buffer ones) is waited with the
// parity of its position in the tile, and no waiter can fall two phases behind: every phase
// needs the arrival of all epilogue threads or follows one that did. Every wait is bounded
// (about two seconds of clock): on a timeout the CTA records an error, every later wait of the
// CTA returns at once, and the CTA drains its MMAs and frees its tensor memory. The callers keep
// their control flow uniform across the epilogue threads (tile counts and work items are
// broadcast), so no named barrier is left waiting for a thread that gave up.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace hignn {
namespace tc {

using hignn::TcWeights;

constexpr int kTile = 128;
constexpr int kEpiThreads = 512;
constexpr int kThreads = 544;
constexpr int kMmaWarp = 16;
constexpr uint32_t kOffA1 = 0, kOffS0 = 64, kOffS1 = 192, kOffA2a = 320, kOffA2b = 384, kOffD3a = 448,
                   kOffD3b = 464;
constexpr int kW2Bytes = kH2 * kH1 * 2;      // 131072
constexpr int kW3Rows = 16;
constexpr int kW3Bytes = kW3Rows * kH2 * 2;  // 16384
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz
// Wait profile (TcWeights::prof non-null): slot c - 13 sums the cycles that lane 0 of every warp
// spent in bounded waits with code c (13-18 the MMA lane: 13 layer 1 in A1, 14-17 quarters 0-3
// in A2, 18 layer-3 accumulator free; 21-24 the epilogue warps: 21 layer-2 accumulator of
// quarters 0-2, 22 quarter 3's accumulator (A1 free), 23 layer-3 accumulator, 24 A2 buffer
// free); slot 12 the cycles of warp 0's whole epilogue; slot 13 the tiles processed.
constexpr int kProfSlots = 16;

struct alignas(1024) Smem {
  uint8_t w2[kW2Bytes];
  uint8_t w3[kW3Bytes];
  uint64_t a1_full, d2_full[2], a2_full[2], a2_free[2], d3_full[2], d3_free[2], drain;
  uint32_t tmem_base;
  int exit_flag;
  int abort_flag;
  unsigned long long* prof;          // optional wait profile (global, kProfSlots counters) or null
  unsigned long long wprof[16];      // per-CTA wait cycles by barrier code (lane 0 of each warp)
  alignas(16) float4 w1b1[kH1];      // FP32 layer 1: (W1[k][0..2], b1[k]) per hidden unit
  alignas(16) uint32_t b2h[kH2 / 2];  // layer-2 bias as FP16 pairs, added to the rounded accumulator
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
// As mbar_try, but the thread may stay suspended in hardware for up to hint_ns while the phase is
// incomplete (it resumes as soon as the phase completes): waiting warps then issue nothing, and
// in particular do not fill the MIO queue that the MUFU instructions of the working warps share.
__device__ __forceinline__ bool mbar_try_sleep(uint64_t* b, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\nselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and raises the CTA abort flag) if the phase never completes.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int* abort_flag, int* err, int code) {
  const long long t0 = clock64();
  while (!mbar_try_sleep(b, parity, 20000u)) {
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

// 16 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
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
__device__ __forceinline__ uint32_t pack_f16(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.f16x2.f32 %0, %1, %2;\n" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ uint32_t tanh_f16x2(uint32_t x) {
  uint32_t y;
  asm("tanh.approx.f16x2 %0, %1;\n" : "=r"(y) : "r"(x));
  return y;
}
__device__ __forceinline__ uint32_t add_f16x2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("add.rn.f16x2 %0, %1, %2;\n" : "=r"(r) : "r"(a), "r"(b));
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

// Instruction descriptor: FP16 x FP16 -> FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16x(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// 16 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
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
  for (int i = t; i < kH1; i += blockDim.x) s.w1b1[i] = w.w1b1[i];
  for (int i = t; i < kH2 / 2; i += blockDim.x) s.b2h[i] = pack_f16(w.b2[2 * i], w.b2[2 * i + 1]);
  if (t < 16) s.b3[t] = t < kOut ? w.b3[t] : 0.f;
  if (t < 16) s.wprof[t] = 0ull;
  if (t == 0) {
    s.prof = w.prof;
    mbar_init(&s.a1_full, kEpiThreads);
    for (int i = 0; i < 2; i++) {
      mbar_init(&s.d2_full[i], 1);
      mbar_init(&s.a2_full[i], kEpiThreads);
      mbar_init(&s.a2_free[i], 1);
      mbar_init(&s.d3_full[i], 1);
      mbar_init(&s.d3_free[i], kEpiThreads);
    }
    mbar_init(&s.drain, 1);
    s.exit_flag = 0;
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
  if (s.prof && threadIdx.x < kProfSlots) atomicAdd(&s.prof[threadIdx.x], s.wprof[threadIdx.x]);
  if ((threadIdx.x >> 5) == kMmaWarp) tmem_dealloc(s.tmem_base, 512);
}

// ------------------------------------------------------------------ MMA lane
// One thread issues every MMA; quarter q of a tile reads accumulator slot q % 2 and A2 buffer
// q % 2, tile t writes layer-3 accumulator t % 2. Per tile t, in this order:
//   L2(t,2)->slot 0, L3(t,0)<-A2[0]         after a2(q0): slot 0 read, A2[0] written
//   L2(t,3)->slot 1, L3(t,1)<-A2[1]         after a2(q1)
//   L3(t,2)<-A2[0]                          after a2(q2)
//   L2(t+1,0)->slot 0                       after a1_full(t+1): layer 1 of t+1 in A1
//   L2(t+1,1)->slot 1, L3(t,3)<-A2[1], commit d3_full[t % 2]   after a2(q3)
// A layer-2 quarter is queued ahead of the layer-3 MMAs issued with it: the epilogue reads it two
// phases later, while layer 3 is needed only at retirement. An accumulator slot is reused as soon
// as the epilogue has read it (its tanh'd pairs go to a separate A2 buffer), so the lane never
// waits for an MMA of its own: the ~500-cycle latency from an MMA's issue to its commit reaching
// a waiting thread is paid only by threads that have other work queued. L3(t,0) overwrites the
// layer-3 accumulator of tile t - 2, so it also waits until the epilogue has read that (d3_free).
struct MmaLane {
  Smem& s;
  int* err;
  uint32_t tb, w2, w3;
  bool ok = true;

  __device__ __forceinline__ bool wait(uint64_t* b, uint32_t parity, int code) {
    if (!ok) return false;
    const long long t0 = s.prof ? clock64() : 0;
    ok = mbar_wait(b, parity, &s.abort_flag, err, code);
    if (s.prof) atomicAdd(&s.wprof[code - 13], (unsigned long long)(clock64() - t0));
    if (ok) fence_after();
    return ok;
  }
  __device__ __forceinline__ uint32_t slot(uint32_t q) const { return tb + (q & 1 ? kOffS1 : kOffS0); }
  // layer-2 quarter q of the tile whose layer 1 is in A1
  __device__ __forceinline__ void l2(uint32_t q) {
    const uint32_t id = idesc_f16x(128, 128);
#pragma unroll
    for (uint32_t kk = 0; kk < 8; kk++) {
      const uint32_t bb = w2 + (kk >> 2) * (kH2 * 128) + q * (128 * 128) + (kk & 3) * 32;
      mma_ts(slot(q), tb + kOffA1 + 8 * kk, sdesc(bb), id, kk > 0);
    }
    mma_commit(&s.d2_full[q & 1]);
  }
  // layer 3 of quarter q of tile t from its A2 buffer into the tile's layer-3 accumulator
  __device__ __forceinline__ void l3(uint32_t t, uint32_t q) {
    const uint32_t id = idesc_f16x(128, kW3Rows);
    const uint32_t a2 = tb + (q & 1 ? kOffA2b : kOffA2a);
    const uint32_t d3 = tb + (t & 1 ? kOffD3b : kOffD3a);
#pragma unroll
    for (uint32_t kk = 0; kk < 8; kk++) {
      const uint32_t kg = q * 128 + kk * 16;  // global K of layer 3
      const uint32_t bb = w3 + (kg >> 6) * (kW3Rows * 128) + ((kg & 63) >> 3) * 16;
      mma_ts(d3, a2 + 8 * kk, sdesc(bb), id, (q > 0 || kk > 0) ? 1u : 0u);
    }
    mma_commit(&s.a2_free[q & 1]);
  }
  // the epilogue wrote the A2 pairs of quarter q. Each a2_full barrier completes twice per tile
  // (quarters q and q + 2), so the phase parity is q / 2.
  __device__ __forceinline__ bool a2(uint32_t q) { return wait(&s.a2_full[q & 1], q >> 1, 14 + (int)q); }

  __device__ void run() {
    // tile 0: its layer 1 in A1, or the end of an empty stream
    if (!wait(&s.a1_full, 0, 13)) return;
    if (*(volatile int*)&s.exit_flag) return;
    l2(0);
    l2(1);
    for (uint32_t t = 0;; t++) {
      if (!a2(0)) return;
      l2(2);
      if (t >= 2 && !wait(&s.d3_free[t & 1], ((t - 2) >> 1) & 1, 18)) return;
      l3(t, 0);
      if (!a2(1)) return;
      l2(3);
      l3(t, 1);
      if (!a2(2)) return;
      l3(t, 2);
      if (!wait(&s.a1_full, (t + 1) & 1, 13)) return;  // layer 1 of the next tile, or the end
      const bool more = !*(volatile int*)&s.exit_flag;
      if (more) l2(0);
      if (!a2(3)) return;
      if (more) l2(1);
      l3(t, 3);
      mma_commit(&s.d3_full[t & 1]);
      if (!more) return;
    }
  }
};

__device__ __forceinline__ void mma_loop(Smem& s, int* err) {
  MmaLane lane{s, err, s.tmem_base, saddr(s.w2), saddr(s.w3)};
  lane.run();
  // drain: every MMA issued so far completes before tensor memory is released
  mma_commit(&s.drain);
  const long long t0 = clock64();
  while (!mbar_try(&s.drain, 0) && clock64() - t0 < kWaitCycles) {
  }
}

// ------------------------------------------------------------------ epilogue side
// Warp w (0-15) reaches TMEM lanes 32 (w % 4) ..; the evaluation (row) e = 32 (w % 4) + lane is
// handled by four threads (warps w % 4 + 4 p, p = 0..3), thread p owning hidden units
// 32p..32p+31 of layer 1, columns 32p..32p+31 of every layer-2 quarter and packed columns
// 16p..16p+15 of A1 and of the A2 buffers.
__device__ __forceinline__ int epi_row() { return 32 * ((threadIdx.x >> 5) & 3) + (threadIdx.x & 31); }
__device__ __forceinline__ int epi_part() { return (threadIdx.x >> 7) & 3; }
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 512;\n" ::: "memory"); }

// The tile engine seen from the epilogue threads. Tiles are retired one step late: step(t)
// computes the network of tile t up to its layer-3 MMAs, layer 1 of tile t + 1, and hands the
// finished M of tile t - 1 to `use`, called between quarters 1 and 2 of tile t. finish() retires
// the last tile. Every call returns false once the CTA has aborted (and then does nothing).
struct Epi {
  Smem& s;
  int* err;
  uint32_t tl;  // TMEM base with this warp's lane field
  int p;
  uint32_t tile = 0;
  bool ok = true;

  __device__ __forceinline__ bool wait(uint64_t* b, uint32_t parity, int code) {
    if (!ok) return false;
    const bool rec = s.prof && (threadIdx.x & 31) == 0;
    const long long t0 = rec ? clock64() : 0;
    ok = mbar_wait(b, parity, &s.abort_flag, err, code);
    if (rec) atomicAdd(&s.wprof[code - 13], (unsigned long long)(clock64() - t0));
    if (ok) fence_after();
    return ok;
  }
  __device__ __forceinline__ uint32_t slot(uint32_t q) const { return tl + (q & 1 ? kOffS1 : kOffS0); }

  // tanh(W1 r + b1) of this thread's 32 hidden units as FP16 pairs (FP32 FMAs, bias first)
  __device__ __forceinline__ void layer1(float rx, float ry, float rz, uint32_t (&out)[16]) const {
    const float4* w = s.w1b1 + 32 * p;
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const float4 a = w[2 * k], b = w[2 * k + 1];
      const float h0 = fmaf(a.z, rz, fmaf(a.y, ry, fmaf(a.x, rx, a.w)));
      const float h1 = fmaf(b.z, rz, fmaf(b.y, ry, fmaf(b.x, rx, b.w)));
      out[k] = tanh_f16x2(pack_f16(h0, h1));
    }
  }
  // A1 <- out, then the lane may issue the tile's layer-2 quarters (or learns of the end)
  __device__ __forceinline__ void publish_a1(bool has, const uint32_t (&out)[16]) {
    if (has) {
      tmem_st16(tl + kOffA1 + 16 * p, out);
      tmem_wait_st();
    } else if (threadIdx.x == 0) {
      *(volatile int*)&s.exit_flag = 1;  // released by this thread's arrival below
    }
    fence_before();
    mbar_arrive(&s.a1_full);
  }

  // layer 1 of the first tile (has = false: nothing to do at all)
  __device__ __forceinline__ void start(bool has, float rx, float ry, float rz) {
    uint32_t out[16];
    if (has) layer1(rx, ry, rz, out);
    publish_a1(has, out);
  }

  // Quarter q: accumulator slot q % 2 (+ FP32 bias) -> tanh -> A2 buffer q % 2. Quarter 3's
  // accumulator was already waited for (before A1 was rewritten).
  __device__ __forceinline__ bool quarter(uint32_t q) {
    // each d2_full / a2_full barrier completes twice per tile (quarters q and q + 2): parity q / 2
    if (q != 3 && !wait(&s.d2_full[q & 1], q >> 1, 21)) return false;
    uint32_t v[32], out[16];
    tmem_ld32(slot(q) + 32 * p, v);
    tmem_wait_ld();
    // one rounding to FP16 pairs, the FP16 bias added to the pairs (one instruction per pair
    // instead of two FP32 adds)
    const uint4* bb = reinterpret_cast<const uint4*>(s.b2h + (q * 128 + 32 * p) / 2);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint4 bv = bb[k];
      out[4 * k] = tanh_f16x2(add_f16x2(pack_f16(__uint_as_float(v[8 * k]), __uint_as_float(v[8 * k + 1])), bv.x));
      out[4 * k + 1] =
          tanh_f16x2(add_f16x2(pack_f16(__uint_as_float(v[8 * k + 2]), __uint_as_float(v[8 * k + 3])), bv.y));
      out[4 * k + 2] =
          tanh_f16x2(add_f16x2(pack_f16(__uint_as_float(v[8 * k + 4]), __uint_as_float(v[8 * k + 5])), bv.z));
      out[4 * k + 3] =
          tanh_f16x2(add_f16x2(pack_f16(__uint_as_float(v[8 * k + 6]), __uint_as_float(v[8 * k + 7])), bv.w));
    }
    // A2 buffer q % 2 was last read by L3 of quarter q - 2 (this tile, first commit on its
    // barrier: parity 0) or of quarter q + 2 of the previous tile (second commit: parity 1)
    if ((tile > 0 || q >= 2) && !wait(&s.a2_free[q & 1], q >= 2 ? 0u : 1u, 24)) return false;
    tmem_st16(tl + (q & 1 ? kOffA2b : kOffA2a) + 16 * p, out);
    tmem_wait_st();
    fence_before();
    mbar_arrive(&s.a2_full[q & 1]);
    return true;
  }

  // M (row-major 3x3) of tile t, from its layer-3 accumulator (parts 0 and 1 read it; both end
  // up with all nine entries)
  __device__ __forceinline__ bool read_d3(uint32_t t, float rx, float ry, float rz, float (&M)[9]) {
    if (!wait(&s.d3_full[t & 1], (t >> 1) & 1, 23)) return false;
    if (p < 2) {
      uint32_t v[16];
      tmem_ld16(tl + (t & 1 ? kOffD3b : kOffD3a), v);
      tmem_wait_ld();
      const float nr = sqrtf(rx * rx + ry * ry + rz * rz);
      const float inv = __frcp_rn(nr);
#pragma unroll
      for (int o = 0; o < 9; o++) {
        float y = __uint_as_float(v[o]) + s.b3[o];
        const bool dg = (o == 0 || o == 4 || o == 8);
        if (dg) y += 1.0f;
        y = y * inv;
        if (nr < 1e-5f) y = dg ? 1.0f : 0.0f;
        M[o] = y;
      }
    }
    fence_before();
    mbar_arrive(&s.d3_free[t & 1]);
    return true;
  }

  // Tile `tile`: quarters 0 and 1, retirement of the previous tile (use(M) with its features
  // (px, py, pz)), quarter 2, layer 1 of the next tile (features nx, ny, nz; has_next = false:
  // the end of the stream), quarter 3. All 512 epilogue threads call it.
  template <class Use>
  __device__ __forceinline__ bool step(bool has_next, float nx, float ny, float nz, float px, float py, float pz,
                                       Use&& use) {
    if (!quarter(0) || !quarter(1)) return false;
    if (tile > 0) {  // retire the previous tile while L2(tile, 2) and L3(tile, 0) run
      float M[9];
      if (!read_d3(tile - 1, px, py, pz, M)) return false;
      use(M);
    }
    if (!quarter(2)) return false;
    {
      uint32_t out[16];
      if (has_next) layer1(nx, ny, nz, out);
      // quarter 3's accumulator complete: every layer-2 MMA of this tile has read A1
      if (!wait(&s.d2_full[1], 1, 22)) return false;
      publish_a1(has_next, out);
    }
    if (!quarter(3)) return false;
    if (s.prof && threadIdx.x == 0) s.wprof[13]++;
    tile++;
    return true;
  }

  // Retires the last tile (features px, py, pz) after its final step.
  template <class Use>
  __device__ __forceinline__ bool finish(float px, float py, float pz, Use&& use) {
    if (tile == 0) return true;
    float M[9];
    if (!read_d3(tile - 1, px, py, pz, M)) return false;
    use(M);
    return true;
  }
};

}  // namespace tc
}  // namespace hignn
