// Plain FP32 near field: fused pair features -> two-body network -> 3x3 contraction.
//
// Restates HignnModel::CloseDot (src/CloseDot.cpp:177-299): for every close
// leaf pair (I, J), u_I[i] += M(x_J[j] - x_I[i]) f_J[j], and when J > I with
// symmetry on, u_J[j] += (the same M) f_I[i] (not transposed, not
// re-evaluated). The reference writes the features to HBM, runs libtorch and
// scatters with one FP64 atomic per evaluation; here one CTA owns a pair,
// stages both leaves in shared memory, evaluates 128 pairs per tile, reduces
// the contributions per particle in shared memory and issues one FP64 atomic
// per particle and component per pair. With kSymmetrize the 3x3 is replaced by
// 0.5 (M + M^T) and only u_I is updated: DenseDot's contraction
// (src/DenseDot.cpp:227-243).
#include "common.h"
#include "kernels.h"
#include "mlp_simt.cuh"

namespace hignn {

namespace {

struct NearSmem {
  simt::Smem mlp;
  float4 xI[kMaxLeaf], xJ[kMaxLeaf], fI[kMaxLeaf], fJ[kMaxLeaf];
  float uI[kMaxLeaf][3], uJ[kMaxLeaf][3];
  int16_t ei[simt::kTile], ej[simt::kTile];
  int item;
};

__global__ void __launch_bounds__(simt::kThreads, 1)
    k_near_simt(NearArgs a, MlpF32 w, int* work_counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  NearSmem& s = *reinterpret_cast<NearSmem*>(smem_raw);
  const int t = threadIdx.x;
  simt::load_weights(s.mlp, w);
  for (;;) {
    __syncthreads();
    if (t == 0) s.item = atomicAdd(work_counter, 1);
    __syncthreads();
    const int item = s.item;
    if (item >= a.nwork) break;
    const PairWork pw = a.work[item];
    const bool trans = (pw.flags & kPairTransposed) != 0;
    const bool symm = (pw.flags & kPairSymmetrize) != 0;
    for (int i = t; i < pw.nI; i += simt::kThreads) {
      s.xI[i] = a.xI[pw.sI + i];
      s.fI[i] = a.fI[pw.sI + i];
      s.uI[i][0] = s.uI[i][1] = s.uI[i][2] = 0.f;
    }
    for (int j = t; j < pw.nJ; j += simt::kThreads) {
      s.xJ[j] = a.xJ[pw.sJ + j];
      s.fJ[j] = a.fJ[pw.sJ + j];
      s.uJ[j][0] = s.uJ[j][1] = s.uJ[j][2] = 0.f;
    }
    __syncthreads();
    const int total = pw.nI * pw.nJ;
    for (int t0 = 0; t0 < total; t0 += simt::kTile) {
      if (t < simt::kTile) {
        const int flat = t0 + t;
        if (flat < total) {
          const int i = flat / pw.nJ, j = flat - (flat / pw.nJ) * pw.nJ;
          const float4 xi = s.xI[i], xj = s.xJ[j];
          s.mlp.r[t] = make_float4(xj.x - xi.x, xj.y - xi.y, xj.z - xi.z, 0.f);
          s.ei[t] = (int16_t)i;
          s.ej[t] = (int16_t)j;
        } else {
          s.mlp.r[t] = make_float4(1.f, 0.f, 0.f, 0.f);
          s.ei[t] = -1;
        }
      }
      __syncthreads();
      simt::mlp_tile(s.mlp, w);
      if (t < simt::kTile && s.ei[t] >= 0) {
        const int i = s.ei[t], j = s.ej[t];
        float M[9];
#pragma unroll
        for (int q = 0; q < 9; q++) M[q] = s.mlp.y[t][q];
        if (symm) {
#pragma unroll
          for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = r + 1; c < 3; c++) {
              const float v = 0.5f * (M[3 * r + c] + M[3 * c + r]);
              M[3 * r + c] = v;
              M[3 * c + r] = v;
            }
        }
        const float4 fj = s.fJ[j];
        atomicAdd(&s.uI[i][0], M[0] * fj.x + M[1] * fj.y + M[2] * fj.z);
        atomicAdd(&s.uI[i][1], M[3] * fj.x + M[4] * fj.y + M[5] * fj.z);
        atomicAdd(&s.uI[i][2], M[6] * fj.x + M[7] * fj.y + M[8] * fj.z);
        if (trans) {
          const float4 fi = s.fI[i];
          atomicAdd(&s.uJ[j][0], M[0] * fi.x + M[1] * fi.y + M[2] * fi.z);
          atomicAdd(&s.uJ[j][1], M[3] * fi.x + M[4] * fi.y + M[5] * fi.z);
          atomicAdd(&s.uJ[j][2], M[6] * fi.x + M[7] * fi.y + M[8] * fi.z);
        }
      }
    }
    __syncthreads();
    for (int q = t; q < 3 * pw.nI; q += simt::kThreads)
      atomicAdd(&a.uI[3 * (size_t)pw.sI + q], (double)(&s.uI[0][0])[q]);
    if (trans)
      for (int q = t; q < 3 * pw.nJ; q += simt::kThreads)
        atomicAdd(&a.uJ[3 * (size_t)pw.sJ + q], (double)(&s.uJ[0][0])[q]);
  }
}

}  // namespace

size_t near_simt_smem_bytes() { return sizeof(NearSmem); }

void launch_near_simt(const NearArgs& a, const MlpF32& w, int* work_counter, int num_sms,
                      cudaStream_t stream) {
  if (a.nwork <= 0) return;
  const size_t smem = sizeof(NearSmem);
  set_max_dynamic_smem(k_near_simt, smem, stream);
  HIGNN_CUDA(cudaMemsetAsync(work_counter, 0, sizeof(int), stream));
  const int grid = a.nwork < num_sms ? a.nwork : num_sms;
  k_near_simt<<<grid, simt::kThreads, smem, stream>>>(a, w, work_counter);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
