// Allocation-free dense rows: hignn_dense_rows_noalloc.
//
// Some callers cannot allocate device memory once they are running: a
// time-stepping code that fixes its device-memory budget at start-up, a host
// framework whose own caching allocator owns the GPU, or a step that must keep
// a constant memory footprint between calls. For them this entry point
// computes the same dense rows as hignn_dense_rows without any cudaMalloc,
// cudaFree or allocating library call: its per-call scratch (target positions,
// leaf table, FP64 accumulators, work counter) lives in one file-scope
// __device__ array of kNaScratchBytes bytes, which every GPU that loads this
// library keeps until the process exits. The model's own buffers, allocated
// when its tree was built, hold the forces.
//
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture. All calls share the array and it keeps the last
// call's contents, so every call clears the accumulators and the counter
// itself. Calls from one process are serialised by a process-wide lock that
// is held until the call's GPU work has finished -- calls on different GPUs
// included, since the host staging arrays are shared too -- so two calls of
// this entry point never overlap on the GPU. What can race is other GPU work
// that the caller issues, on another stream, against the same model's
// buffers while a call runs: the call overwrites the model's force buffers
// (the caller-order staging and the tree-order forces) and reads its
// positions.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/hignn_b200.h"
#include "common.h"
#include "mlp_simt.cuh"
#include "model_view.h"

namespace hignn {

namespace {

constexpr int64_t kNaMaxRows = HIGNN_NOALLOC_MAX_ROWS;
constexpr int64_t kNaMaxLeaves = HIGNN_NOALLOC_MAX_LEAVES;
constexpr size_t kNaOffLeaf = 0;                                              // int2 [kNaMaxLeaves]
constexpr size_t kNaOffPos = kNaOffLeaf + sizeof(int2) * kNaMaxLeaves;        // int32 [kNaMaxRows]
constexpr size_t kNaOffX = kNaOffPos + sizeof(int32_t) * kNaMaxRows;          // float4 [kNaMaxRows]
constexpr size_t kNaOffU = kNaOffX + sizeof(float4) * kNaMaxRows;             // double [3 kNaMaxRows]
constexpr size_t kNaOffCtr = kNaOffU + sizeof(double) * 3 * kNaMaxRows;       // int [64]
constexpr size_t kNaScratchBytes = kNaOffCtr + 256;                           // about 6.3 MB
constexpr int kNaMaxDevices = 64;

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

// Host-side set-up state and staging (static: no heap allocation per call).
std::mutex g_na_mutex;
void* g_na_dev_ptr[kNaMaxDevices] = {};
int32_t g_na_pos[kNaMaxRows];
int2 g_na_leaf[kNaMaxLeaves];

struct NaArgs {
  const int2* leaf;   // (start, count) of each leaf, tree order
  int nleaves;
  const float4* xT;   // target positions
  double* uT;         // target velocities, FP64 (nrows, 3)
  int nrows;
  const float4* x4;   // source positions, tree order
  const float4* f4;   // source forces, tree order
  int* counter;
};

__global__ void k_na_gather_forces(const float* __restrict__ f, const int32_t* __restrict__ perm,
                                   float4* __restrict__ f4, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = perm[i];
  f4[i] = make_float4(f[3 * p], f[3 * p + 1], f[3 * p + 2], 0.f);
}

// Targets gathered, accumulators and the work counter cleared (the array keeps old contents).
__global__ void k_na_prepare(const float4* __restrict__ x4, const int32_t* __restrict__ pos,
                             float4* __restrict__ xT, double* __restrict__ uT, int* __restrict__ counter, int nrows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *counter = 0;
  if (i >= nrows) return;
  xT[i] = x4[pos[i]];
  uT[3 * i] = 0.0;
  uT[3 * i + 1] = 0.0;
  uT[3 * i + 2] = 0.0;
}

struct NaSmem {
  simt::Smem mlp;
  float4 xI[simt::kTile];
  float4 xJ[kMaxLeaf], fJ[kMaxLeaf];
  float uI[simt::kTile][3];
  int16_t ei[simt::kTile], ej[simt::kTile];
  int item;
};

// One work item = 128 target rows against one source leaf; the symmetrised 3x3
// 0.5 (M + M^T) of src/DenseDot.cpp:227-243 contracted with the leaf's forces.
__global__ void __launch_bounds__(simt::kThreads, 1) k_na_dense_rows(NaArgs a, MlpF32 w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  NaSmem& s = *reinterpret_cast<NaSmem*>(smem_raw);
  const int t = threadIdx.x;
  const int nchunks = (a.nrows + simt::kTile - 1) / simt::kTile;
  const int nitems = nchunks * a.nleaves;
  simt::load_weights(s.mlp, w);
  for (;;) {
    __syncthreads();
    if (t == 0) s.item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = s.item;
    if (item >= nitems) break;
    const int chunk = item / a.nleaves, leaf = item - chunk * a.nleaves;
    const int sI = chunk * simt::kTile;
    const int nI = min(simt::kTile, a.nrows - sI);
    const int2 lj = a.leaf[leaf];
    const int sJ = lj.x, nJ = lj.y;
    for (int i = t; i < nI; i += simt::kThreads) {
      s.xI[i] = a.xT[sI + i];
      s.uI[i][0] = s.uI[i][1] = s.uI[i][2] = 0.f;
    }
    for (int j = t; j < nJ; j += simt::kThreads) {
      s.xJ[j] = a.x4[sJ + j];
      s.fJ[j] = a.f4[sJ + j];
    }
    __syncthreads();
    const int total = nI * nJ;
    for (int t0 = 0; t0 < total; t0 += simt::kTile) {
      if (t < simt::kTile) {
        const int flat = t0 + t;
        if (flat < total) {
          const int i = flat / nJ, j = flat - (flat / nJ) * nJ;
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
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = r + 1; c < 3; c++) {
            const float v = 0.5f * (M[3 * r + c] + M[3 * c + r]);
            M[3 * r + c] = v;
            M[3 * c + r] = v;
          }
        const float4 fj = s.fJ[j];
        atomicAdd(&s.uI[i][0], M[0] * fj.x + M[1] * fj.y + M[2] * fj.z);
        atomicAdd(&s.uI[i][1], M[3] * fj.x + M[4] * fj.y + M[5] * fj.z);
        atomicAdd(&s.uI[i][2], M[6] * fj.x + M[7] * fj.y + M[8] * fj.z);
      }
    }
    __syncthreads();
    for (int q = t; q < 3 * nI; q += simt::kThreads) atomicAdd(&a.uT[3 * (size_t)sI + q], (double)(&s.uI[0][0])[q]);
  }
}

// Device address of the scratch array for the current device (looked up once per device).
unsigned char* scratch_for(int device) {
  if (device < 0 || device >= kNaMaxDevices) throw Error(HIGNN_ERR_ARG, "device index out of range");
  if (!g_na_dev_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Error(HIGNN_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                      cudaGetErrorString(e));
    g_na_dev_ptr[device] = p;
  }
  return static_cast<unsigned char*>(g_na_dev_ptr[device]);
}

void dense_rows_noalloc(hignn_model* m, double* u_rows, const float* f, const int64_t* rows, int64_t nrows,
                        int precision) {
  if (!m || !u_rows || !f || (!rows && nrows > 0)) throw Error(HIGNN_ERR_ARG, "null argument");
  if (precision != 0) throw Error(HIGNN_ERR_ARG, "dense_rows_noalloc supports precision 0 (FP32 network)");
  if (nrows < 0 || nrows > kNaMaxRows)
    throw Error(HIGNN_ERR_ARG, "dense_rows_noalloc: nrows must be in [0, " + std::to_string(kNaMaxRows) +
                                   "] (size of the static scratch array)");
  ModelView v;
  model_view(m, v);
  if (!v.ready)
    throw Error(HIGNN_ERR_STATE,
                "dense_rows_noalloc needs a device model with weights and a built tree "
                "(call hignn_update_coord or hignn_dot once first; those may allocate)");
  const int64_t nleaves = (int64_t)v.leaves->size();
  if (nleaves > kNaMaxLeaves)
    throw Error(HIGNN_ERR_ARG, "dense_rows_noalloc: the tree has more than " + std::to_string(kNaMaxLeaves) +
                                   " leaves (size of the static scratch array)");
  if (nrows == 0) return;
  HIGNN_CUDA(cudaSetDevice(v.device));
  std::lock_guard<std::mutex> lock(g_na_mutex);
  unsigned char* base = scratch_for(v.device);
  for (int64_t q = 0; q < nrows; q++) {
    if (rows[q] < 0 || rows[q] >= v.n) throw Error(HIGNN_ERR_ARG, "row index out of range");
    g_na_pos[q] = (int32_t)(*v.inv_perm)[rows[q]];
  }
  for (int64_t l = 0; l < nleaves; l++) {
    const TreeNode& nd = (*v.nodes)[(*v.leaves)[l]];
    if (nd.end - nd.start > kMaxLeaf)  // the kernel stages one source leaf in shared memory
      throw Error(HIGNN_ERR_ARG, "dense_rows_noalloc: a leaf holds more than " + std::to_string(kMaxLeaf) +
                                     " particles");
    g_na_leaf[l] = make_int2((int)nd.start, (int)(nd.end - nd.start));
  }
  int2* d_leaf = reinterpret_cast<int2*>(base + kNaOffLeaf);
  int32_t* d_pos = reinterpret_cast<int32_t*>(base + kNaOffPos);
  float4* d_x = reinterpret_cast<float4*>(base + kNaOffX);
  double* d_u = reinterpret_cast<double*>(base + kNaOffU);
  int* d_ctr = reinterpret_cast<int*>(base + kNaOffCtr);
  cudaStream_t s = v.stream;
  HIGNN_CUDA(cudaMemcpyAsync(d_leaf, g_na_leaf, sizeof(int2) * nleaves, cudaMemcpyHostToDevice, s));
  HIGNN_CUDA(cudaMemcpyAsync(d_pos, g_na_pos, sizeof(int32_t) * nrows, cudaMemcpyHostToDevice, s));
  HIGNN_CUDA(cudaMemcpyAsync(v.io_f, f, sizeof(float) * 3 * v.n, cudaMemcpyHostToDevice, s));
  k_na_gather_forces<<<(unsigned)((v.n + 255) / 256), 256, 0, s>>>(v.io_f, v.perm, v.f4, v.n);
  HIGNN_CHECK_LAUNCH();
  k_na_prepare<<<(unsigned)((nrows + 255) / 256), 256, 0, s>>>(v.x4, d_pos, d_x, d_u, d_ctr, (int)nrows);
  HIGNN_CHECK_LAUNCH();
  NaArgs a;
  a.leaf = d_leaf;
  a.nleaves = (int)nleaves;
  a.xT = d_x;
  a.uT = d_u;
  a.nrows = (int)nrows;
  a.x4 = v.x4;
  a.f4 = v.f4;
  a.counter = d_ctr;
  const size_t smem = sizeof(NaSmem);
  HIGNN_CUDA(cudaFuncSetAttribute(k_na_dense_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t nitems = ((nrows + simt::kTile - 1) / simt::kTile) * nleaves;
  const int grid = (int)(nitems < v.num_sms ? nitems : v.num_sms);
  k_na_dense_rows<<<grid, simt::kThreads, smem, s>>>(a, v.w);
  HIGNN_CHECK_LAUNCH();
  HIGNN_CUDA(cudaMemcpyAsync(u_rows, d_u, sizeof(double) * 3 * nrows, cudaMemcpyDeviceToHost, s));
  HIGNN_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

}  // namespace hignn

extern "C" int hignn_dense_rows_noalloc(hignn_model* m, double* u_rows, const float* f, const int64_t* rows,
                                        int64_t nrows, int precision) {
  try {
    hignn::dense_rows_noalloc(m, u_rows, f, rows, nrows, precision);
    return HIGNN_OK;
  } catch (const hignn::Error& e) {
    hignn::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    hignn::set_last_error(e.what());
    return HIGNN_ERR_ARG;
  }
}
