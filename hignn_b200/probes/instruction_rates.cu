// Throughput probe: lane-operations per clock per SM of single instructions (tanh / ex2 in
// f32, f16x2 and bf16x2 forms, conversions, integer and FP adds), eight independent chains per
// thread, 2 CTAs x 1024 threads per SM, clock64 per CTA. Build and run on a B200:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o instruction_rates \
//        hignn_b200/probes/instruction_rates.cu && ./instruction_rates [occupancy]
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#define ITERS 2048
template <int OP>
__global__ void k(uint32_t* out, long long* cyc) {
  uint32_t v[8];
  for (int c = 0; c < 8; c++) v[c] = 0x3f000000u + threadIdx.x * 17 + c * 1234;
  __syncthreads();
  long long t0 = clock64();
  for (int it = 0; it < ITERS; it++) {
#pragma unroll
    for (int c = 0; c < 8; c++) {
      uint32_t x = v[c];
      if (OP == 0) asm volatile("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(x) : "f"(__uint_as_float(x)), "f"(__uint_as_float(x ^ 0x10u)));
      if (OP == 1) asm volatile("tanh.approx.bf16x2 %0, %0;" : "+r"(x));
      if (OP == 2) asm volatile("tanh.approx.f32 %0, %0;" : "+r"(x));
      if (OP == 3) asm volatile("prmt.b32 %0, %0, %0, 0x7632;" : "+r"(x));
      if (OP == 4) asm volatile("add.u32 %0, %0, 0x8000;" : "+r"(x));
      if (OP == 5) asm volatile("add.f32 %0, %0, 0f3F800000;" : "+r"(x));
      if (OP == 6) asm volatile("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(x) : "f"(__uint_as_float(x)), "f"(__uint_as_float(x ^ 0x10u)));
      if (OP == 7) asm volatile("tanh.approx.f16x2 %0, %0;" : "+r"(x));
      if (OP == 8) asm volatile("{.reg .b32 t; cvt.rn.bf16x2.f32 t, %0, %0; tanh.approx.bf16x2 %0, t;}" : "+r"(x));
      if (OP == 9) asm volatile("rcp.approx.ftz.f32 %0, %0;" : "+r"(x));
      if (OP == 10) asm volatile("ex2.approx.ftz.bf16x2 %0, %0;" : "+r"(x));
      if (OP == 11) asm volatile("fma.rn.bf16x2 %0, %0, %0, %0;" : "+r"(x));
      if (OP == 12) asm volatile("{.reg .b32 a, b; add.u32 a, %0, 0x8000; add.u32 b, %0, 0x8010; prmt.b32 %0, a, b, 0x7632;}" : "+r"(x));
      if (OP == 13) asm volatile("{.reg .b32 t; prmt.b32 t, %0, %0, 0x7632; tanh.approx.bf16x2 %0, t;}" : "+r"(x));
      if (OP == 14) asm volatile("cvt.rn.satfinite.bf16x2.f32 %0, %1, %2;" : "=r"(x) : "f"(__uint_as_float(x)), "f"(__uint_as_float(x ^ 0x10u)));
      if (OP == 15) asm volatile("ex2.approx.f16x2 %0, %0;" : "+r"(x));
      v[c] = x;
    }
  }
  long long t1 = clock64();
  uint32_t s = 0;
  for (int c = 0; c < 8; c++) s ^= v[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
  if (threadIdx.x == 0) cyc[blockIdx.x] = t1 - t0;
}
template <int OP>
void run(const char* name, int blocks_per_sm, int threads) {
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  int nb = sms * blocks_per_sm;
  uint32_t* out; long long* cyc;
  cudaMalloc(&out, sizeof(uint32_t) * nb * threads);
  cudaMalloc(&cyc, sizeof(long long) * nb);
  k<OP><<<nb, threads>>>(out, cyc);
  k<OP><<<nb, threads>>>(out, cyc);
  cudaError_t e = cudaDeviceSynchronize();
  long long* h = new long long[nb];
  cudaMemcpy(h, cyc, sizeof(long long) * nb, cudaMemcpyDeviceToHost);
  long long mx = 0; for (int i = 0; i < nb; i++) mx = h[i] > mx ? h[i] : mx;
  double ops_per_sm = (double)blocks_per_sm * threads * 8 * ITERS;
  printf("%-28s err=%d  cycles=%lld  lane-ops/clk/SM=%.2f\n", name, (int)e, mx, ops_per_sm / mx);
  cudaFree(out); cudaFree(cyc); delete[] h;
}
int main(int argc, char** argv) {
  if (argc > 1) {  // occupancy sweep of the packed tanh: lanes/clk/SM with fewer resident warps
    run<1>("tanh.approx.bf16x2 1x128", 1, 128);
    run<1>("tanh.approx.bf16x2 1x256", 1, 256);
    run<1>("tanh.approx.bf16x2 1x512", 1, 512);
    run<1>("tanh.approx.bf16x2 1x1024", 1, 1024);
    run<8>("cvt+tanh 1x512", 1, 512);
    run<2>("tanh.approx.f32 1x512", 1, 512);
    return 0;
  }
  run<5>("fadd.f32", 2, 1024);
  run<0>("cvt.rn.bf16x2.f32", 2, 1024);
  run<14>("cvt.rn.satfinite.bf16x2", 2, 1024);
  run<6>("cvt.rn.f16x2.f32", 2, 1024);
  run<1>("tanh.approx.bf16x2", 2, 1024);
  run<7>("tanh.approx.f16x2", 2, 1024);
  run<2>("tanh.approx.f32", 2, 1024);
  run<10>("ex2.approx.bf16x2", 2, 1024);
  run<15>("ex2.approx.f16x2", 2, 1024);
  run<3>("prmt", 2, 1024);
  run<11>("fma.rn.bf16x2", 2, 1024);
  run<8>("cvt+tanh (2 instr)", 2, 1024);
  run<12>("2 iadd + prmt (3 instr)", 2, 1024);
  run<13>("prmt + tanh (2 instr)", 2, 1024);
  return 0;
}
