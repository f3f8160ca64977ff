// Read-only view of a model's device state for entry points implemented outside capi.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.h"
#include "tree.h"

struct hignn_model;

namespace hignn {

struct ModelView {
  bool ready = false;            // device, weights, tree and device buffers all present
  int device = -1;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int64_t n = 0;
  const float4* x4 = nullptr;    // positions, tree order
  float4* f4 = nullptr;          // force buffer, tree order
  const int32_t* perm = nullptr; // tree position -> caller index
  float* io_f = nullptr;         // (n, 3) staging buffer, caller order
  MlpF32 w{};
  const std::vector<TreeNode>* nodes = nullptr;
  const std::vector<int64_t>* leaves = nullptr;
  const std::vector<int64_t>* inv_perm = nullptr;  // caller index -> tree position
};

// Fills v from m without allocating anything (host or device).
void model_view(hignn_model* m, ModelView& v);

// Records an error message for hignn_last_error() of the calling thread.
void set_last_error(const char* msg);

}  // namespace hignn
