// Reorder kernels and the stand-alone two-body evaluation.
//
// HignnModel::Reorder(map, v) / BackwardReorder (src/HignnModel.cpp:252-320)
// gather f into tree order and scatter u back; here the gather also converts
// the caller's (n,3) float32 rows to float4 and zeroes the FP64 accumulator,
// and the scatter converts the accumulator to the caller's float32 rows
// (src/HignnModel.cpp:618-624), so each is one pass over HBM.
#include "common.h"
#include "kernels.h"
#include "mlp_simt.cuh"

namespace hignn {

namespace {

__global__ void k_gather_forces(const float* __restrict__ f, const int32_t* __restrict__ perm,
                                float4* __restrict__ f4, double* __restrict__ u, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = perm[i];
  f4[i] = make_float4(f[3 * p], f[3 * p + 1], f[3 * p + 2], 0.f);
  u[3 * i] = 0.0;
  u[3 * i + 1] = 0.0;
  u[3 * i + 2] = 0.0;
}

__global__ void k_scatter_velocities(const double* __restrict__ u, const int32_t* __restrict__ perm,
                                     float* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = perm[i];
  out[3 * p] = (float)u[3 * i];
  out[3 * p + 1] = (float)u[3 * i + 1];
  out[3 * p + 2] = (float)u[3 * i + 2];
}

__global__ void k_gather_positions(const float4* __restrict__ x4, const int32_t* __restrict__ pos,
                                   float4* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = x4[pos[i]];
}

__global__ void __launch_bounds__(simt::kThreads, 1)
    k_eval_simt(const float* __restrict__ r, float* __restrict__ y, int64_t n, MlpF32 w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  simt::Smem& s = *reinterpret_cast<simt::Smem*>(smem_raw);
  const int t = threadIdx.x;
  simt::load_weights(s, w);
  for (int64_t base = (int64_t)blockIdx.x * simt::kTile; base < n; base += (int64_t)gridDim.x * simt::kTile) {
    if (t < simt::kTile) {
      const int64_t e = base + t;
      s.r[t] = e < n ? make_float4(r[3 * e], r[3 * e + 1], r[3 * e + 2], 0.f) : make_float4(1.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    simt::mlp_tile(s, w);
    if (t < simt::kTile && base + t < n)
#pragma unroll
      for (int q = 0; q < 9; q++) y[9 * (base + t) + q] = s.y[t][q];
  }
}

}  // namespace

void launch_gather_forces(const float* f, const int32_t* perm, float4* f4, double* u, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_forces<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f, perm, f4, u, n);
  HIGNN_CHECK_LAUNCH();
}

void launch_scatter_velocities(const double* u, const int32_t* perm, float* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  k_scatter_velocities<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(u, perm, out, n);
  HIGNN_CHECK_LAUNCH();
}

void launch_gather_positions(const float4* x4, const int32_t* pos, float4* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_positions<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x4, pos, out, n);
  HIGNN_CHECK_LAUNCH();
}

void launch_eval_simt(const float* r, float* y, int64_t n, const MlpF32& w, int num_sms, cudaStream_t s) {
  if (n <= 0) return;
  const size_t smem = sizeof(simt::Smem);
  HIGNN_CUDA(cudaFuncSetAttribute(k_eval_simt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int64_t tiles = (n + simt::kTile - 1) / simt::kTile;
  int grid = (int)(tiles < num_sms ? tiles : num_sms);
  k_eval_simt<<<grid, simt::kThreads, smem, s>>>(r, y, n, w);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
