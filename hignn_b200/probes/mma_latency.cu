// Probe of the tensor-pipe cost of tcgen05.mma (M = 128, K = 16, A in tensor memory) against N
// and batch length, of the issue-to-commit latency, and of an mbarrier round trip between two
// warps. One CTA; every wait is bounded. Build and run on a B200:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -I include \
//        -o mma_latency hignn_b200/probes/mma_latency.cu && ./mma_latency

#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "../csrc/tc_mlp.cuh"
using namespace hignn::tc;
// one CTA, 128 threads; thread 0 issues NI MMAs (M=128, N, K=16, A in TMEM, B in smem), commits,
// waits; repeats R times. smem B: 256 rows x 64 K bf16 = 32 KB (zeros).
template <int N>
__global__ void k(int NI, int R, long long* out) {
  __shared__ alignas(1024) uint8_t b[256 * 128];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  for (int i = threadIdx.x; i < 256 * 128 / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(b)[i] = 0;
  if (threadIdx.x == 0) { mbar_init(&bar, 1); asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (threadIdx.x < 32) tmem_alloc(&tbase, 512);
  fence_before(); __syncthreads(); fence_after();
  if (threadIdx.x == 0) {
    const uint32_t id = idesc_bf16(128, N);
    const uint64_t d = sdesc(saddr(b));
    long long t0 = clock64();
    for (int r = 0; r < R; r++) {
      for (int i = 0; i < NI; i++) mma_ts(tbase + 256, tbase + 8 * (i & 7), d, id, i > 0);
      mma_commit(&bar);
      long long tw = clock64();
      while (!mbar_try(&bar, r & 1) && clock64() - tw < 100000000LL) {}
    }
    out[0] = clock64() - t0;
  }
  fence_before(); __syncthreads(); fence_after();
  if (threadIdx.x < 32) tmem_dealloc(tbase, 512);
}
// ping-pong: warp 0 lane 0 arrives on b0, warp 1 lane 0 waits b0 and arrives b1, warp0 waits b1
__global__ void kpp(int R, long long* out) {
  __shared__ uint64_t b0, b1;
  if (threadIdx.x == 0) { mbar_init(&b0, 1); mbar_init(&b1, 1); asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
  __syncthreads();
  long long t0 = clock64();
  if (threadIdx.x == 0) {
    for (int r = 0; r < R; r++) { mbar_arrive(&b0); long long tw=clock64(); while (!mbar_try(&b1, r & 1) && clock64()-tw < 100000000LL) {} }
    out[1] = clock64() - t0;
  } else if (threadIdx.x == 32) {
    for (int r = 0; r < R; r++) { long long tw=clock64(); while (!mbar_try(&b0, r & 1) && clock64()-tw < 100000000LL) {} mbar_arrive(&b1); }
  }
}
template <int N> void run(int NI, int R) {
  long long* d; cudaMalloc(&d, 16); long long h[2];
  k<N><<<1, 128>>>(NI, R, d); cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(h, d, 16, cudaMemcpyDeviceToHost);
  double per = (double)h[0] / R;
  printf("N=%3d NI=%3d: %.0f cycles per batch, %.1f per MMA (ideal compute %.1f) err=%d\n", N, NI, per, per / NI, 128.0 * N * 16 * 2 / 8192, (int)e);
  cudaFree(d);
}
int main() {
  run<32>(1, 200); run<32>(8, 200); run<32>(32, 100);
  run<64>(8, 200); run<64>(32, 100);
  run<128>(1, 200); run<128>(8, 200); run<128>(32, 100); run<128>(64, 50);
  run<256>(8, 200); run<256>(32, 100);
  long long* d; cudaMalloc(&d, 16); long long h[2];
  kpp<<<1, 64>>>(1000, d); cudaError_t e = cudaDeviceSynchronize(); cudaMemcpy(h, d, 16, cudaMemcpyDeviceToHost);
  printf("mbarrier ping-pong: %.0f cycles per round trip err=%d\n", (double)h[1] / 1000, (int)e);
  return 0;
}
