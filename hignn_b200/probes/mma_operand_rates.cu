// Probe of the tensor-pipe rate of tcgen05.mma (M = 128, K = 16, BF16, FP32 accumulate) by
// operand source: A in tensor memory (ts) or in shared memory (ss), B in shared memory, for
// N = 128 and 256. With both operands read from shared memory every MMA costs shared-memory
// bandwidth, so the ss forms show whether those reads, not the tensor pipe, set the rate. One CTA
// per SM on every SM; one thread issues batches of MMAs and waits for each batch (bounded).
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        -o mma_operand_rates hignn_b200/probes/mma_operand_rates.cu && ./mma_operand_rates
#include <cstdint>
#include <cstdio>

#include <cuda_runtime.h>

#include "../csrc/tc_mlp.cuh"
using namespace hignn::tc;

__device__ __forceinline__ void mma_ss_probe(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// SS: 1 = A from shared memory, 0 = A from tensor memory
template <int N, int SS>
__global__ void k(int NI, int R, long long* out) {
  extern __shared__ uint8_t raw[];
  uint8_t* base = raw + ((1024 - (saddr(raw) & 1023)) & 1023);
  uint8_t* a = base;          // 128 rows x 64 K: 16 KB
  uint8_t* b = base + 16384;  // 256 rows x 64 K: 32 KB
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  for (int i = threadIdx.x; i < 49152 / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(base)[i] = 0;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (threadIdx.x < 32) tmem_alloc(&tbase, 512);
  fence_before();
  __syncthreads();
  fence_after();
  if (threadIdx.x == 0) {
    const uint32_t id = idesc_bf16(128, N);
    long long t0 = clock64();
    bool ok = true;
    for (int r = 0; r < R && ok; r++) {
      for (int i = 0; i < NI; i++) {
        const uint64_t bd = sdesc(saddr(b) + 32 * (i & 3));
        if (SS)
          mma_ss_probe(tbase + 256, sdesc(saddr(a) + 32 * (i & 3)), bd, id, i > 0);
        else
          mma_ts(tbase + 256, tbase + 8 * (i & 7), bd, id, i > 0);
      }
      mma_commit(&bar);
      const long long tw = clock64();
      while (!mbar_try(&bar, r & 1))
        if (clock64() - tw > 200000000LL) {
          ok = false;
          break;
        }
    }
    if (blockIdx.x == 0) out[0] = ok ? clock64() - t0 : -1;
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (threadIdx.x < 32) tmem_dealloc(tbase, 512);
}

template <int N, int SS>
void run(int sms, int NI, int R) {
  long long* d;
  cudaMalloc(&d, 16);
  long long h = 0;
  const int smem = 120 * 1024;  // one CTA per SM (49 KB used)
  cudaFuncSetAttribute(k<N, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k<N, SS><<<sms, 128, smem>>>(NI, R, d);
  const cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(&h, d, 8, cudaMemcpyDeviceToHost);
  const double per = (double)h / R / NI;
  printf("%s N=%3d: %.1f cycles per MMA (tensor-pipe rate %.1f), %.0f B/clk of shared-memory operand reads err=%d\n",
         SS ? "ss" : "ts", N, per, 128.0 * N * 16 * 2 / 8192, ((SS ? 4096.0 : 0.0) + N * 32.0) / per, (int)e);
  cudaFree(d);
}

int main() {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  run<128, 0>(sms, 64, 200);
  run<128, 1>(sms, 64, 200);
  run<256, 0>(sms, 64, 200);
  run<256, 1>(sms, 64, 200);
  return 0;
}
