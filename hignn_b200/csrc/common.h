// Shared definitions of the native library (host and device).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace hignn {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// A failed call throws; the runtime's record of a non-sticky error is cleared first, so that a
// later, unrelated check (cudaGetLastError after a launch) does not report it again.
#define HIGNN_CUDA(call)                                                                              \
  do {                                                                                                \
    cudaError_t _e = (call);                                                                          \
    if (_e != cudaSuccess) {                                                                          \
      (void)cudaGetLastError();                                                                       \
      throw ::hignn::Error(-2, std::string(#call " failed: ") + cudaGetErrorString(_e) + " at " +   \
                                   __FILE__ + ":" + std::to_string(__LINE__));                      \
    }                                                                                                 \
  } while (0)

#define HIGNN_CHECK_LAUNCH() HIGNN_CUDA(cudaGetLastError())

// Shared-memory size attribute of a kernel, set outside stream capture only: a graph is captured
// after the same launches have run eagerly once, which set the attributes (they persist).
template <class K>
inline void set_max_dynamic_smem(K kernel, size_t bytes, cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  HIGNN_CUDA(cudaStreamIsCapturing(s, &st));
  if (st == cudaStreamCaptureStatusNone)
    HIGNN_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// Device allocation owned by the model (grown on demand, never shrunk; contents not kept).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  // the caller's file and line go into the error of a failed allocation
  void ensure(size_t b, const char* file = __builtin_FILE(), int line = __builtin_LINE()) {
    if (b <= bytes && p) return;
    release();
    if (b == 0) return;
    const cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
      throw Error(-2, std::string("cudaMalloc of ") + std::to_string(b) + " bytes failed: " + cudaGetErrorString(e) +
                          " (buffer grown at " + file + ":" + std::to_string(line) + ")");
    }
    bytes = b;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

constexpr int kMaxLeaf = 256;   // largest leaf the near-field kernels stage in shared memory
constexpr int kTcMaxLeaf = 128; // largest leaf of the tensor-core near field (three staging buffers)
constexpr int kH1 = 128;        // two-body network widths (python/convert.py:6-20 over nn/*.pkl)
constexpr int kH2 = 512;
constexpr int kOut = 9;
constexpr int kStudentParams = 2537;  // 3-32-32-32-9 student network (weights + biases)

// FP32 weights of the two-body network as the SIMT kernels read them.
struct MlpF32 {
  const float4* w1b1;  // [kH1]: (W1[k][0], W1[k][1], W1[k][2], b1[k])
  const float* w2t;    // [kH1][kH2]: w2t[k*kH2 + n] = W2[n][k]
  const float* b2;     // [kH2]
  const float* w3;     // [kOut][kH2]
  const float* b3;     // [kOut]
};

// Tensor-core weights: swizzled FP16 images of W2 and W3 plus FP32 layer 1 (W1, b1) and FP32
// biases of layers 2 and 3.
struct TcWeights {
  const uint4* w2img;   // 512 x 128 FP16, K-major 128-byte swizzle (131072 B)
  const uint4* w3img;   // 16 x 512 FP16 (rows 0-8 W3, rows 9-15 zero) (16384 B)
  const float4* w1b1;   // [128]: (W1[k][0], W1[k][1], W1[k][2], b1[k])
  const float* b2;      // [512]
  const float* b3;      // [9]
  unsigned long long* prof = nullptr;  // optional wait profile of the engine (tc::kProfSlots counters)
};

// One unit of near-field (or dense) work: target range I against source range J.
constexpr int32_t kPairTransposed = 1;  // also u_J += M f_I (symmetric close pair, J > I)
constexpr int32_t kPairSymmetrize = 2;  // use 0.5 (M + M^T) (dense product)
struct PairWork {
  int32_t sI, nI, sJ, nJ, flags, pad0, pad1, pad2;
};

}  // namespace hignn
