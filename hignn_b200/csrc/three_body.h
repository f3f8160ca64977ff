// Three-body and self near field (python/HIGNN/model_structure.py:41-139) on the tensor cores.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.h"
#include "neighbors.h"

namespace hignn {

constexpr int kTbH1 = 256, kTbH2 = 1024, kTbH3 = 512;
constexpr int kTbStageBytes = 32768;                // one weight stage: 256 rows x 64 K or 128 x 128 K (FP16)
constexpr int kTbStagesPerTile = 64;                 // 16 layer-2 chunks and 16 layer-3 slices, 2 stages each
constexpr int kTbImageBytes = kTbStagesPerTile * kTbStageBytes;  // 2 MB

// Device weights of one three-body-shaped network (kin -> 256 -> 1024 -> 512 -> 9, tanh).
struct TbWeightsDev {
  const uint8_t* img;  // layers 2 and 3 as FP16 stages in the order the MMA lane consumes them
  const float* w1;     // [256][8]: W1 row (kin entries, zero padded to 6), b1, 0
  const float* b2;     // [1024]
  const float* b3;     // [512]
  const float* w4;     // [512][12]: column n of W4 (9 entries), zero padded
  const float* b4;     // [9]
};

enum TbKind : int { kTbThreeBody = 0, kTbSelf = 1 };

// One network's host copy and device image.
struct TbNet {
  bool loaded = false;
  int kin = 0;
  std::vector<float> w1, b2, b3, w4, b4;
  DevBuf d_img, d_w1, d_b2, d_b3, d_w4, d_b4;
  TbWeightsDev dev() const {
    return {d_img.as<uint8_t>(), d_w1.as<float>(), d_b2.as<float>(), d_b3.as<float>(), d_w4.as<float>(),
            d_b4.as<float>()};
  }
};

// u[c] += ((net(x_b - x_a, x_c - x_b) / |x_b - x_a| / |x_c - x_b|) as 3x3) f[a] for every triplet
// (a, b, c) of the list (rows of the (3, E) uint64 edge list), kind kTbThreeBody; or
// u[b] += ((net(x_a - x_b) / |x_a - x_b|^2) as 3x3) f[b] for every pair (a, b), kind kTbSelf.
// x, f as float4 (w unused), u float (n, 3). prof (optional, 6 counters, summed over CTAs):
// clocks the MMA lane waited for layer-1 operands, weight stages, layer-2 epilogues and the
// layer-3 accumulator, its total clocks, and clocks the producer waited for free ring slots.
// Returns the number of 128-edge tiles launched.
int64_t launch_three_body(int kind, const TbWeightsDev& w, const uint64_t* edges, int64_t num_edges, const float4* x,
                          const float4* f, float* u, int* err, unsigned long long* prof, int num_sms, cudaStream_t s);

// Builds the device image of a network from its dense layers (W row-major out x in, b).
void tb_upload(TbNet& net, int kin, const std::vector<std::vector<float>>& W, const std::vector<std::vector<float>>& B,
               cudaStream_t s);

}  // namespace hignn
