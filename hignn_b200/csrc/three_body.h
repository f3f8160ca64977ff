// Three-body and self near field (python/HIGNN/model_structure.py:41-139) on the tensor cores.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.h"
#include "neighbors.h"

namespace hignn {

constexpr int kTbH1 = 256, kTbH2 = 1024, kTbH3 = 512;
constexpr int kTbStageBytes = 32768;  // one weight stage: 256 rows x 64 K or 128 x 128 K (FP16)
// Image segments in the MMA lane's order: A = layer 2 chunk 0 (2 stages), B = the rest of a tile
// (15 layer-2 chunks and 16 layer-3 slices of 2 stages, layer 4 of pass 0), then layer 4 of pass 1
constexpr int kTbSegA = 2, kTbSegB = 15 * 2 + 16 * 2 + 1;
constexpr int kTbStagesPerTile = kTbSegA + kTbSegB + 1;
constexpr int kTbImageBytes = kTbStagesPerTile * kTbStageBytes;  // 2.06 MB

// Small per-network constants, passed to the kernel as a parameter: the epilogue reads them
// with warp-uniform indices, which the constant bank serves without a memory round trip.
struct TbConst {
  float w1[kTbH1 * 7];  // row n: W1[n][0..kin) zero padded to 6, then b1[n]
  float b2[kTbH2];
  float b3[kTbH3];
  float b4[9];
};

// Device weights of one three-body-shaped network (kin -> 256 -> 1024 -> 512 -> 9, tanh).
struct TbWeightsDev {
  const uint8_t* img;  // layers 2 and 3 as FP16 stages in the order the MMA lane consumes them
};

enum TbKind : int { kTbThreeBody = 0, kTbSelf = 1 };

// One network's host copy and device image.
struct TbNet {
  bool loaded = false;
  int kin = 0;
  TbConst cst{};
  DevBuf d_img;
  TbWeightsDev dev() const { return {d_img.as<uint8_t>()}; }
};

// u[c] += ((net(x_b - x_a, x_c - x_b) / |x_b - x_a| / |x_c - x_b|) as 3x3) f[a] for every triplet
// (a, b, c) of the list (rows of the (3, E) uint64 edge list), kind kTbThreeBody; or
// u[b] += ((net(x_a - x_b) / |x_a - x_b|^2) as 3x3) f[b] for every pair (a, b), kind kTbSelf.
// x, f as float4 (w unused), u float (n, 3). prof (optional, 6 counters, summed over CTAs):
// clocks the MMA lane waited for layer-1 operands, weight stages, layer-2 epilogues and the
// layer-3 accumulator, its total clocks, and clocks the producer waited for free ring slots.
// Returns the number of 128-edge tiles launched.
int64_t launch_three_body(int kind, const TbWeightsDev& w, const TbConst& c, const uint64_t* edges, int64_t num_edges,
                          const float4* x, const float4* f, float* u, int* err, unsigned long long* prof, int num_sms,
                          cudaStream_t s);
// The same, accumulating into FP64 velocities (the H-matvec's accumulator).
int64_t launch_three_body(int kind, const TbWeightsDev& w, const TbConst& c, const uint64_t* edges, int64_t num_edges,
                          const float4* x, const float4* f, double* u, int* err, unsigned long long* prof, int num_sms,
                          cudaStream_t s);

// Builds the device image of a network from its dense layers (W row-major out x in, b).
void tb_upload(TbNet& net, int kin, const std::vector<std::vector<float>>& W, const std::vector<std::vector<float>>& B,
               cudaStream_t s);

}  // namespace hignn
