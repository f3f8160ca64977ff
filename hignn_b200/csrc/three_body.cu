// Three-body and self near field on the tensor cores (python/HIGNN/model_structure.py:41-139).
//
// The reference evaluates, for every triplet (a, b, c) of the three-body edge list
// (include/NeighborLists.hpp:512-585; the model reads its rows as (j, k, i)),
//     M = Three_body_net(x_b - x_a, x_c - x_b) = net(.) / |x_b - x_a| / |x_c - x_b|   (3 x 3)
//     u_c += M f_a                                                              (:94-101)
// and for every self pair (a, b) of the self edge list,
//     M = Two_body_self_net(x_a - x_b) = net(.) / |x_a - x_b| / |x_a - x_b|,   u_b += M f_b
// (:57-67, 120-125), with torch FP32 Linear layers kin -> 256 -> 1024 -> 512 -> 9 and tanh.
//
// Here one persistent kernel per list does gather -> network -> bmm -> scatter for 128 edges per
// tile. Layer 1 (kin <= 6 inputs) runs on the CUDA cores in FP32 and writes tanh'd FP16 pairs
// into tensor memory as the A operand of layer 2. Layers 2, 3 and 4 are tcgen05 MMAs (FP16 in,
// FP32 accumulated in tensor memory); layer 4 (512 -> 9, N = 16) takes each pass's tanh'd layer-3
// values from tensor memory, where they replace the read accumulator. Tensor memory (512
// columns) holds the layer-1 activations (128 columns of FP16
// pairs), one 128-column layer-2 accumulator and a 256-column layer-3 accumulator. The 512
// layer-3 outputs therefore take two passes per tile, each recomputing layer 2 (1.33x the
// network's FLOPs) -- the layer-2 activations of a tile (128 x 1024 FP16 = 256 KB) fit neither
// shared nor tensor memory.
// Layer 2 is cut into sixteen chunks of 128 outputs (eight per pass); the epilogue releases the
// layer-2 accumulator as soon as it has read it, then writes the chunk's tanh'd FP16 values to a
// shared-memory buffer (two, in turn) that is the K-slice of layer 3 (N = 256). The MMA lane
// interleaves the chunks, L2(g + 1) before L3(g), so the tensor pipe has a layer-3 slice to run
// while the epilogue turns an accumulator around.
// The weights (1.6 MB of FP16) stream through a five-deep ring of 32 KB shared-memory stages,
// filled by bulk copies from a host-built image laid out in the order the MMAs consume it.
//
// CTA = 18 warps: 0-15 epilogue (warp w reaches TMEM lanes 32 (w % 4) + 0..31, so row
// e = 32 (w % 4) + lane has four threads, part p = w / 4), 16 MMA lane, 17 producer.
// Every wait is bounded (about two seconds of clock); on a timeout the CTA records an error,
// stops, lets its copies and MMAs drain and frees its tensor memory.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>

#include "three_body.h"
#include "tc_mlp.cuh"

namespace hignn {

namespace {

using tc::fence_after;
using tc::fence_before;
using tc::mbar_arrive;
using tc::mbar_init;
using tc::mbar_try_sleep;
using tc::mma_commit;
using tc::saddr;
using tc::sdesc;
using tc::tmem_ld32;
using tc::tmem_wait_ld;

constexpr int kEpiThreads = 512;
constexpr int kMmaWarp = 16, kProdWarp = 17, kThreads = 576;
constexpr int kRing = 5;
// tensor-memory columns: layer 1 (A of layer 2), layer-2 accumulator, layer-3 accumulator; once
// the layer-3 accumulator of a pass is read, its first 128 columns take that pass's tanh'd
// layer-3 values (A of layer 4) and columns 384-399 the layer-4 accumulator
constexpr uint32_t kOffA1 = 0, kOffD2 = 128, kOffD3 = 256, kOffA3 = 256, kOffD4 = 384;
constexpr long long kWait = 4000000000LL;      // ~2 s at 1.9 GHz

struct TbSmem {
  uint8_t act2[2][2][16384];  // A of layer 3, two buffers of 128 rows x 128 K (FP16)
  uint8_t ring[kRing][kTbStageBytes];
  uint64_t act1_full, d2_full, d2_free, act2_full[2], d3_full, act3_full, d4_full, d3_free, ring_full[kRing],
      ring_empty[kRing], drain;
  uint32_t tmem_base;
  int abort_flag;
};
constexpr size_t kSmemBytes = sizeof(TbSmem) + 1024;  // + alignment slack
static_assert(kSmemBytes <= 232448, "three-body shared memory exceeds the per-CTA limit");
static_assert(sizeof(TbConst) + 128 <= 32764, "three-body kernel parameters exceed the launch limit");

__device__ __forceinline__ bool wait_bar(uint64_t* b, uint32_t parity, int* abort_flag, int* err, int code,
                                         bool honour_abort = true) {
  const long long t0 = clock64();
  while (!mbar_try_sleep(b, parity, 20000u)) {
    if (honour_abort && *(volatile int*)abort_flag) return false;
    if (clock64() - t0 > kWait) {
      atomicExch(abort_flag, 1);
      atomicCAS(err, 0, code);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(saddr(dst)),
      "l"(src), "r"(bytes), "r"(saddr(bar))
      : "memory");
}

// FP16 operands: layer inputs are tanh outputs in [-1, 1] and the weights stay below 1 in
// magnitude, so FP16's 11-bit significand (BF16 has 8) costs no range and cuts the rounding
// error of the tensor-core layers about eightfold at the same MMA rate.
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
// Instruction descriptor: F16 x F16 -> FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, const uint32_t* v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3])
               : "memory");
}

__device__ __forceinline__ bool epi_all(bool ok) {
  uint32_t r;
  asm volatile("{\n.reg .pred p, q;\nsetp.ne.u32 p, %1, 0;\nbar.red.and.pred q, 1, 512, p;\nselp.u32 %0, 1, 0, q;\n}\n"
               : "=r"(r)
               : "r"((uint32_t)ok)
               : "memory");
  return r != 0;
}
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 512;\n" ::: "memory"); }

// Byte offset of (row, k) in a 128-row, 64-wide K block (K-major, 128-byte swizzle) for the
// 16-byte chunk kc8 = k / 8.
__device__ __forceinline__ uint32_t swz_chunk(int row, int kc8) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((kc8 ^ (row & 7)) << 4));
}

// The network input of edge q (6 features; the self net uses the first 3) and its endpoints.
template <int KIND>
__device__ __forceinline__ void edge_input(const uint64_t* __restrict__ edges, int64_t E, int64_t q,
                                           const float4* __restrict__ x, float (&in)[6], int64_t& src, int64_t& dst) {
  if (KIND == kTbThreeBody) {
    const int64_t a = (int64_t)edges[q], b = (int64_t)edges[E + q], c = (int64_t)edges[2 * E + q];
    const float4 xa = x[a], xb = x[b], xc = x[c];
    in[0] = xb.x - xa.x, in[1] = xb.y - xa.y, in[2] = xb.z - xa.z;
    in[3] = xc.x - xb.x, in[4] = xc.y - xb.y, in[5] = xc.z - xb.z;
    src = a, dst = c;
  } else {
    const int64_t a = (int64_t)edges[q], b = (int64_t)edges[E + q];
    const float4 xa = x[a], xb = x[b];
    in[0] = xa.x - xb.x, in[1] = xa.y - xb.y, in[2] = xa.z - xb.z;
    in[3] = in[4] = in[5] = 0.f;
    src = b, dst = b;
  }
}

__device__ __forceinline__ float norm3f(float a, float b, float c) { return sqrtf(a * a + b * b + c * c); }

// ------------------------------------------------------------------ epilogue warps
template <int KIND, typename OUT>
struct Epi {
  TbSmem& s;
  const TbConst& c;
  TbWeightsDev w;
  const uint64_t* edges;
  int64_t E;
  const float4* x;
  const float4* f;
  OUT* u;
  int* err;
  int e, part;     // row of the tile, column part
  uint32_t tlane;  // TMEM address of this warp's lane quarter
  bool ok = true;

  __device__ __forceinline__ bool wait(uint64_t* b, uint32_t parity, int code) {
    if (!ok) return false;
    ok = wait_bar(b, parity, &s.abort_flag, err, code);
    if (ok) fence_after();
    return ok;
  }

  // features and layer 1 of tile t into the tensor-memory A operand of layer 2 (this thread:
  // outputs 64 part .. + 63 of row e, as FP16 pairs in columns 32 part .. + 31). The part is a
  // template argument, so every weight is read at a constant offset of the kernel parameter.
  __device__ void layer1(int64_t t) {
    switch (part) {
      case 0: layer1_part<0>(t); break;
      case 1: layer1_part<1>(t); break;
      case 2: layer1_part<2>(t); break;
      default: layer1_part<3>(t); break;
    }
  }
  template <int PART>
  __device__ void layer1_part(int64_t t) {
    const int64_t q = t * 128 + e;
    float in[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int64_t src, dst;
    if (q < E) edge_input<KIND>(edges, E, q, x, in, src, dst);
#pragma unroll
    for (int half = 0; half < 2; half++) {
      uint32_t pk[16];
#pragma unroll
      for (int pr = 0; pr < 16; pr++) {
        float acc[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int n = 64 * PART + 32 * half + 2 * pr + h;
          const float* wr = c.w1 + 7 * n;
          float a = wr[6];  // b1
#pragma unroll
          for (int k = 0; k < 6; k++) a = fmaf(wr[k], in[k], a);
          acc[h] = a;
        }
        pk[pr] = tanh_f16x2(pack_f16(acc[0], acc[1]));
      }
      tc::tmem_st16(tlane + kOffA1 + 32 * PART + 16 * half, pk);
    }
    tc::tmem_wait_st();
    fence_before();
    mbar_arrive(&s.act1_full);
  }

  // layer-2 chunk g: the accumulator (released once read) -> tanh'd FP16 into act2[g & 1]
  __device__ void layer2(uint32_t g) {
    const uint32_t b = g & 1;
    if (wait(&s.d2_full, g & 1, 41)) {
      uint32_t v[32];
      tmem_ld32(tlane + kOffD2 + 32 * part, v);
      tmem_wait_ld();
      fence_before();
      mbar_arrive(&s.d2_free);
      const float* b2 = c.b2 + (g & 7) * 128 + 32 * part;
      uint32_t pk[16];
#pragma unroll
      for (int j = 0; j < 16; j++)
        pk[j] = tanh_f16x2(pack_f16(__uint_as_float(v[2 * j]) + b2[2 * j], __uint_as_float(v[2 * j + 1]) + b2[2 * j + 1]));
      const uint32_t base = saddr(s.act2[b][part >> 1]);
#pragma unroll
      for (int jj = 0; jj < 4; jj++) st_shared_v4(base + swz_chunk(e, 4 * (part & 1) + jj), pk + 4 * jj);
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    } else {
      mbar_arrive(&s.d2_free);
    }
    mbar_arrive(&s.act2_full[b]);
  }

  // Layer 3 of pass h: read the accumulator (D3 columns 64 part .. + 63), add b3, tanh into FP16
  // pairs, and once every thread has read its columns, write the pairs back as the A operand of
  // layer 4 (columns 256 + 32 part ..). Every epilogue thread runs this (it holds a barrier).
  __device__ void layer3(uint32_t P, int h) {
    uint32_t a3[32];
    const bool got = wait(&s.d3_full, P & 1, 42);
    if (got) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint32_t v[16];
        tc::tmem_ld16(tlane + kOffD3 + 64 * part + 16 * q, v);
        tmem_wait_ld();
        const float* b3 = c.b3 + h * 256 + 64 * part + 16 * q;
#pragma unroll
        for (int j = 0; j < 8; j++)
          a3[8 * q + j] =
              tanh_f16x2(pack_f16(__uint_as_float(v[2 * j]) + b3[2 * j], __uint_as_float(v[2 * j + 1]) + b3[2 * j + 1]));
      }
    }
    fence_before();
    epi_bar();  // every column of D3 has been read before any is overwritten
    fence_after();
    if (got) {
      tc::tmem_st32(tlane + kOffA3 + 32 * part, a3);
      tc::tmem_wait_st();
    }
    fence_before();
    mbar_arrive(&s.act3_full);
  }

  // Layer 4 of pass P (part 0): add the accumulator's nine columns to y and release D3 / D4.
  __device__ void layer4(uint32_t P, float (&y)[9]) {
    if (wait(&s.d4_full, P & 1, 43)) {
      uint32_t v[16];
      tc::tmem_ld16(tlane + kOffD4, v);
      tmem_wait_ld();
#pragma unroll
      for (int o = 0; o < 9; o++) y[o] += __uint_as_float(v[o]);
    }
    fence_before();
    mbar_arrive(&s.d3_free);
  }

  // layer 4's two passes plus b4, the wrapper, 3x3 times the force, scatter (part 0)
  __device__ void output(int64_t t, const float (&y)[9]) {
    const int64_t q = t * 128 + e;
    if (q >= E) return;
    float yy[9];
#pragma unroll
    for (int o = 0; o < 9; o++) yy[o] = y[o] + c.b4[o];
    float in[6];
    int64_t src, dst;
    edge_input<KIND>(edges, E, q, x, in, src, dst);
    if (KIND == kTbThreeBody) {
      const float r1 = norm3f(in[0], in[1], in[2]), r2 = norm3f(in[3], in[4], in[5]);
#pragma unroll
      for (int o = 0; o < 9; o++) yy[o] = yy[o] / r1 / r2;
    } else {
      const float r = norm3f(in[0], in[1], in[2]);
#pragma unroll
      for (int o = 0; o < 9; o++) yy[o] = yy[o] / r / r;
    }
    const float4 fs = f[src];
#pragma unroll
    for (int i = 0; i < 3; i++)
      atomicAdd(&u[3 * dst + i], (OUT)(yy[3 * i] * fs.x + yy[3 * i + 1] * fs.y + yy[3 * i + 2] * fs.z));
  }

  // The epilogue follows the MMA lane's order: per tile E2 of chunks 0..15, layer 3 of pass 0
  // after chunk 8 and its layer 4 (part 0) after chunk 9, the next tile's layer 1 after chunk 15,
  // then layer 3 of pass 1; layer 4 of pass 1 and the output come after the next tile's first
  // chunk (the MMA lane issues that chunk's layer 2 before layer 4 of pass 1).
  __device__ void run(int64_t ntiles) {
    uint32_t g = 0, P = 0;
    float y[9];
#pragma unroll
    for (int o = 0; o < 9; o++) y[o] = 0.f;
    if ((int64_t)blockIdx.x < ntiles) layer1(blockIdx.x);
    bool go = true;
    int64_t prev = -1;
    for (int64_t t = blockIdx.x; t < ntiles && go; t += gridDim.x) {
#pragma unroll 1
      for (int cc = 0; cc < 16; cc++, g++) {
        layer2(g);
        if (cc == 0 && prev >= 0) {  // finish the previous tile
          if (part == 0) {
            layer4(P - 1, y);
            output(prev, y);
          }
          go = epi_all(ok);
          if (!go) break;
#pragma unroll
          for (int o = 0; o < 9; o++) y[o] = 0.f;
        }
        if (cc == 8) layer3(P++, 0);
        if (cc == 9 && part == 0) layer4(P - 1, y);
      }
      if (!go) break;
      if (ok && t + gridDim.x < ntiles) layer1(t + gridDim.x);
      layer3(P++, 1);
      prev = t;
    }
    if (go && prev >= 0) {
      if (part == 0) {
        layer4(P - 1, y);
        output(prev, y);
      }
      epi_all(ok);
    }
  }
};

// ------------------------------------------------------------------ MMA lane
struct MmaLaneTb {
  TbSmem& s;
  int* err;
  uint32_t tb;
  uint32_t S = 0;  // weight stages consumed
  bool ok = true;
  long long waited[4] = {0, 0, 0, 0};  // clocks spent waiting for act1, weight stages, epilogues, D3

  __device__ __forceinline__ bool wait(uint64_t* b, uint32_t parity, int code) {
    if (!ok) return false;
    const long long t0 = clock64();
    ok = wait_bar(b, parity, &s.abort_flag, err, code);
    waited[code == 50 ? 0 : code == 51 ? 1 : code == 54 ? 3 : 2] += clock64() - t0;
    if (ok) fence_after();
    return ok;
  }
  __device__ __forceinline__ bool stage_ready() { return wait(&s.ring_full[S % kRing], (S / kRing) & 1, 51); }
  __device__ __forceinline__ void stage_done() {
    mma_commit(&s.ring_empty[S % kRing]);
    S++;
  }
  // layer-2 chunk g (global chunk index; the accumulator is free once the epilogue has read
  // chunk g - 1): A = layer 1 in tensor memory, two 32 KB stages of W2 (K 0-127, 128-255)
  __device__ bool l2(uint32_t g) {
    if (g > 0 && !wait(&s.d2_free, (g - 1) & 1, 52)) return false;
    const uint32_t id = idesc_f16(128, 128);
    for (uint32_t st = 0; st < 2; st++) {
      if (!stage_ready()) return false;
      const uint64_t b0 = sdesc(saddr(s.ring[S % kRing]));
#pragma unroll
      for (uint32_t i = 0; i < 8; i++) {
        const uint32_t k16 = 8 * st + i;  // K = 16 k16 .. + 15
        const uint64_t bd = b0 + (i >> 2) * (16384 >> 4) + (i & 3) * 2;
        tc::mma_ts(tb + kOffD2, tb + kOffA1 + 8 * k16, bd, id, k16 != 0);
      }
      stage_done();
    }
    mma_commit(&s.d2_full);
    return true;
  }
  // layer-3 K-slice of chunk g (local chunk c, pass P) into D3: N = 256, two 32 KB stages of W3
  // (256 rows x 64 K each)
  __device__ bool l3(uint32_t g, uint32_t c, uint32_t P) {
    if (!wait(&s.act2_full[g & 1], (g >> 1) & 1, 53)) return false;
    if (c == 0 && P > 0 && !wait(&s.d3_free, (P - 1) & 1, 54)) return false;
    const uint32_t id = idesc_f16(128, 256);
    for (uint32_t kb = 0; kb < 2; kb++) {
      if (!stage_ready()) return false;
      const uint64_t a0 = sdesc(saddr(s.act2[g & 1][kb])), b0 = sdesc(saddr(s.ring[S % kRing]));
#pragma unroll
      for (uint32_t kk = 0; kk < 4; kk++) mma_ss(tb + kOffD3, a0 + 2 * kk, b0 + 2 * kk, id, (c | kb | kk) != 0);
      stage_done();
    }
    if (c == 7) mma_commit(&s.d3_full);
    return true;
  }

  // layer 4 of pass P: A = the tanh'd layer 3 in tensor memory, one stage with W4's rows for
  // this pass (16 rows, 9 used, x 256 K, four 2 KB K blocks)
  __device__ bool l4(uint32_t P) {
    if (!wait(&s.act3_full, P & 1, 58)) return false;
    if (!stage_ready()) return false;
    const uint64_t b0 = sdesc(saddr(s.ring[S % kRing]));
    const uint32_t id = idesc_f16(128, 16);
#pragma unroll
    for (uint32_t k16 = 0; k16 < 16; k16++)
      tc::mma_ts(tb + kOffD4, tb + kOffA3 + 8 * k16, b0 + (k16 >> 2) * (2048 >> 4) + (k16 & 3) * 2, id, k16 != 0);
    stage_done();
    mma_commit(&s.d4_full);
    return true;
  }

  __device__ void run(int64_t ntiles, unsigned long long* prof) {
    const long long start = clock64();
    uint32_t g = 0, k = 0;
    // per tile: [L2(0) for the first tile], then L2(c + 1) L3(c) for c = 0..15 (no L2(16)) with
    // L4 of pass 0 before L3(8); then the next tile's L2(0) and L4 of pass 1. Chunks 0-7 are
    // pass 0, 8-15 pass 1.
    if ((int64_t)blockIdx.x < ntiles && wait(&s.act1_full, 0, 50)) l2(0);
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x, k++, g += 16) {
      for (uint32_t c = 0; c < 16 && ok; c++) {
        if (c < 15) l2(g + c + 1);
        if (c == 8 && ok) l4(2 * k);
        if (ok) l3(g + c, c & 7, 2 * k + (c >> 3));
      }
      if (ok && t + gridDim.x < ntiles && wait(&s.act1_full, (k + 1) & 1, 50)) l2(g + 16);
      if (ok) l4(2 * k + 1);
    }
    // let every issued MMA finish before the tensor memory is freed
    mma_commit(&s.drain);
    wait_bar(&s.drain, 0, &s.abort_flag, err, 55, false);
    if (prof) {
      for (int i = 0; i < 4; i++) atomicAdd(&prof[i], (unsigned long long)waited[i]);
      atomicAdd(&prof[4], (unsigned long long)(clock64() - start));
    }
  }
};

// ------------------------------------------------------------------ producer
__device__ void producer(TbSmem& s, const uint8_t* img, int64_t ntiles, int* err, unsigned long long* prof) {
  uint32_t S = 0;
  bool ok = true;
  long long waited = 0;
  // per tile: [segment A for the first tile], segment B, [segment A if a tile follows], W4 of
  // pass 1 -- the MMA lane's order (the image holds A | B | W4 of pass 1)
  for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const bool first = t == (int64_t)blockIdx.x, next = t + gridDim.x < ntiles;
    const int count = (first ? kTbSegA : 0) + kTbSegB + (next ? kTbSegA : 0) + 1;
    for (int i = 0; i < count; i++, S++) {
      int st = i;
      if (!first) st += kTbSegA;                          // skip the leading segment A
      if (st >= kTbSegA + kTbSegB) {                      // past segment B
        const int r = st - kTbSegA - kTbSegB;
        st = (next && r < kTbSegA) ? r : kTbSegA + kTbSegB;  // segment A again, then W4
      }
      const uint32_t slot = S % kRing;
      const long long t0 = clock64();
      const bool got = S < kRing || wait_bar(&s.ring_empty[slot], ((S / kRing) - 1) & 1, &s.abort_flag, err, 56);
      waited += clock64() - t0;
      if (!got) {
        ok = false;
        break;
      }
      bulk_load(s.ring[slot], img + (size_t)st * kTbStageBytes, kTbStageBytes, &s.ring_full[slot]);
    }
  }
  // every issued copy must land before the CTA exits
  const uint32_t first = S > (uint32_t)kRing ? S - kRing : 0;
  for (uint32_t q = first; q < S; q++) wait_bar(&s.ring_full[q % kRing], (q / kRing) & 1, &s.abort_flag, err, 57, false);
  if (prof) atomicAdd(&prof[5], (unsigned long long)waited);
}

template <int KIND, typename OUT>
__global__ void __launch_bounds__(kThreads, 1)
    k_three_body(const __grid_constant__ TbConst cst, TbWeightsDev w, const uint64_t* __restrict__ edges, int64_t E,
                 int64_t ntiles,
                 const float4* __restrict__ x, const float4* __restrict__ f, OUT* __restrict__ u, int* err,
                 unsigned long long* prof) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = saddr(smem_raw);
  TbSmem& s = *reinterpret_cast<TbSmem*>(smem_raw + (((raw + 1023u) & ~1023u) - raw));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&s.act1_full, kEpiThreads);
    mbar_init(&s.d2_full, 1);
    mbar_init(&s.d2_free, kEpiThreads);
    for (int b = 0; b < 2; b++) mbar_init(&s.act2_full[b], kEpiThreads);
    mbar_init(&s.d3_full, 1);
    mbar_init(&s.act3_full, kEpiThreads);
    mbar_init(&s.d4_full, 1);
    mbar_init(&s.d3_free, kEpiThreads / 4);  // part 0 reads layer 4
    for (int r = 0; r < kRing; r++) {
      mbar_init(&s.ring_full[r], 1);
      mbar_init(&s.ring_empty[r], 1);
    }
    mbar_init(&s.drain, 1);
    s.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == kMmaWarp) tc::tmem_alloc(&s.tmem_base, 512);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp < kMmaWarp) {
    Epi<KIND, OUT> ep{s, cst, w, edges, E, x, f, u, err};
    ep.e = 32 * (warp & 3) + lane;
    ep.part = warp >> 2;
    ep.tlane = s.tmem_base + ((uint32_t)(32 * (warp & 3)) << 16);
    ep.run(ntiles);
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      MmaLaneTb ml{s, err, s.tmem_base};
      ml.run(ntiles, prof);
    }
  } else if (warp == kProdWarp && lane == 0) {
    producer(s, w.img, ntiles, err, prof);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == kMmaWarp) {
    __syncwarp();
    tc::tmem_dealloc(s.tmem_base, 512);
  }
}

template <int KIND, typename OUT>
void launch_kind(const TbWeightsDev& w, const TbConst& c, const uint64_t* edges, int64_t E, int64_t ntiles,
                 const float4* x, const float4* f, OUT* u, int* err, unsigned long long* prof, int num_sms,
                 cudaStream_t s) {
  HIGNN_CUDA(
      cudaFuncSetAttribute(k_three_body<KIND, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  const int grid = (int)(ntiles < num_sms ? ntiles : num_sms);
  k_three_body<KIND, OUT><<<grid, kThreads, kSmemBytes, s>>>(c, w, edges, E, ntiles, x, f, u, err, prof);
  HIGNN_CHECK_LAUNCH();
}

uint16_t f16_of(float v) {
  const __half h = __float2half_rn(v);
  uint16_t b;
  std::memcpy(&b, &h, 2);
  return b;
}

template <typename OUT>
int64_t launch_any(int kind, const TbWeightsDev& w, const TbConst& c, const uint64_t* edges, int64_t num_edges,
                   const float4* x, const float4* f, OUT* u, int* err, unsigned long long* prof, int num_sms,
                   cudaStream_t s) {
  const int64_t ntiles = (num_edges + 127) / 128;
  if (ntiles == 0) return 0;
  if (kind == kTbThreeBody)
    launch_kind<kTbThreeBody, OUT>(w, c, edges, num_edges, ntiles, x, f, u, err, prof, num_sms, s);
  else
    launch_kind<kTbSelf, OUT>(w, c, edges, num_edges, ntiles, x, f, u, err, prof, num_sms, s);
  return ntiles;
}

}  // namespace

int64_t launch_three_body(int kind, const TbWeightsDev& w, const TbConst& c, const uint64_t* edges, int64_t num_edges,
                          const float4* x, const float4* f, float* u, int* err, unsigned long long* prof, int num_sms,
                          cudaStream_t s) {
  return launch_any<float>(kind, w, c, edges, num_edges, x, f, u, err, prof, num_sms, s);
}

int64_t launch_three_body(int kind, const TbWeightsDev& w, const TbConst& c, const uint64_t* edges, int64_t num_edges,
                          const float4* x, const float4* f, double* u, int* err, unsigned long long* prof, int num_sms,
                          cudaStream_t s) {
  return launch_any<double>(kind, w, c, edges, num_edges, x, f, u, err, prof, num_sms, s);
}

void tb_upload(TbNet& net, int kin, const std::vector<std::vector<float>>& W, const std::vector<std::vector<float>>& B,
               cudaStream_t s) {
  if (W.size() != 4 || B.size() != 4) throw Error(-1, "three-body network: need 4 dense layers");
  const size_t want[4][2] = {{kTbH1, (size_t)kin}, {kTbH2, kTbH1}, {kTbH3, kTbH2}, {9, kTbH3}};
  for (int l = 0; l < 4; l++)
    if (W[l].size() != want[l][0] * want[l][1] || B[l].size() != want[l][0])
      throw Error(-1, "three-body network: layer sizes must be kin -> 256 -> 1024 -> 512 -> 9");
  net.kin = kin;
  net.cst = TbConst{};
  for (int n = 0; n < kTbH1; n++) {
    for (int k = 0; k < kin; k++) net.cst.w1[n * 7 + k] = W[0][(size_t)n * kin + k];
    net.cst.w1[n * 7 + 6] = B[0][n];
  }
  std::copy(B[1].begin(), B[1].end(), net.cst.b2);
  std::copy(B[2].begin(), B[2].end(), net.cst.b3);
  std::copy(B[3].begin(), B[3].end(), net.cst.b4);
  // layers 2 and 3 as 32 KB FP16 stages (K-major, 128-byte swizzle; a 64-wide K block of R rows
  // is R x 128 B, 8-row groups 1024 B apart) in the MMA lane's order per tile: L2(0), then
  // L2(c + 1) L3(c) for c = 0..15 (no L2(16)). An L2 chunk c (pass c / 8, W2 rows (c % 8) 128 ..)
  // is two stages of two 128-row K blocks (K 0-127, 128-255); an L3 slice c is two stages of one
  // 256-row K block: W3 rows (c / 8) 256 .., columns (c % 8) 128 + 64 kb ...
  std::vector<uint8_t> img(kTbImageBytes, 0);
  auto swz = [](int row, int kc) -> size_t {
    return (size_t)(row >> 3) * 1024 + (row & 7) * 128 + (size_t)(((kc >> 3) ^ (row & 7)) * 16) + (kc & 7) * 2;
  };
  size_t st = 0;
  auto put_block = [&](uint8_t* dst, const std::vector<float>& M, int ld, int rows, int row0, int col0) {
    for (int n = 0; n < rows; n++)
      for (int kc = 0; kc < 64; kc++) {
        const uint16_t v = f16_of(M[(size_t)(row0 + n) * ld + col0 + kc]);
        std::memcpy(dst + swz(n, kc), &v, 2);
      }
  };
  auto put_l2 = [&](int c) {
    for (int half = 0; half < 2; half++, st++)
      for (int i = 0; i < 2; i++)
        put_block(img.data() + st * kTbStageBytes + i * 16384, W[1], kTbH1, 128, (c % 8) * 128, (2 * half + i) * 64);
  };
  auto put_l3 = [&](int c) {
    for (int kb = 0; kb < 2; kb++, st++)
      put_block(img.data() + st * kTbStageBytes, W[2], kTbH2, 256, (c / 8) * 256, (c % 8) * 128 + kb * 64);
  };
  // W4 rows of pass h: 16 rows (outputs, 9 used) x 256 K (layer-3 outputs h 256 ..), four
  // 64-wide K blocks of 2 KB at the start of a stage
  auto put_l4 = [&](int h) {
    uint8_t* dst = img.data() + st * kTbStageBytes;
    for (int kb = 0; kb < 4; kb++)
      for (int o = 0; o < 9; o++)
        for (int kc = 0; kc < 64; kc++) {
          const uint16_t v = f16_of(W[3][(size_t)o * kTbH3 + h * 256 + kb * 64 + kc]);
          std::memcpy(dst + kb * 2048 + swz(o, kc), &v, 2);
        }
    st++;
  };
  put_l2(0);  // segment A
  for (int c = 0; c < 16; c++) {  // segment B
    if (c < 15) put_l2(c + 1);
    if (c == 8) put_l4(0);
    put_l3(c);
  }
  put_l4(1);
  if (st != (size_t)kTbStagesPerTile) throw Error(-1, "three-body image: stage count mismatch");
  net.d_img.ensure(img.size());
  HIGNN_CUDA(cudaMemcpyAsync(net.d_img.p, img.data(), img.size(), cudaMemcpyHostToDevice, s));
  HIGNN_CUDA(cudaStreamSynchronize(s));
  net.loaded = true;
}

}  // namespace hignn
