// Kernel argument blocks and launchers of the native library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.h"

namespace hignn {

constexpr int kMaxIterCap = 512;  // largest ACA iteration cap (set_max_iter) the kernels accept

// Storage type of the ACA factors C_l, Q_l (9 entries per particle and term). The reference keeps
// them in FP64 (src/FarDot.cpp:104-107); here they are stored in FP32 and every operation on them
// (orthogonalisation, pivot determinants and inverses, the stopping norms, the apply) is carried
// out in FP64: the factors are the bulk of the far field's memory traffic, and their FP32 rounding
// (1e-7 relative) is far below the ACA tolerance.
using pool_t = float;

// ---------------------------------------------------------------- near field / dense
struct NearArgs {
  const PairWork* work;
  int nwork;
  const float4* xI;  // target positions (x, y, z, 0)
  const float4* fI;  // target forces
  double* uI;        // target velocities, (n, 3) FP64
  const float4* xJ;  // source positions
  const float4* fJ;
  double* uJ;
};

size_t near_simt_smem_bytes();
void launch_near_simt(const NearArgs& a, const MlpF32& w, int* work_counter, int num_sms, cudaStream_t s);
// Dense rows with the network in FP64 (kPairSymmetrize items, I side only; dense_f64.cu).
void launch_dense_f64(const NearArgs& a, const MlpF32& w, int* work_counter, int num_sms, cudaStream_t s);

// ---------------------------------------------------------------- far field (ACA)
constexpr int kXcHead = 8;  // FP32 pivot scratch of a block: 8 norm terms, then 9 floats per term

struct FarBlock {
  int32_t sI, nI, sJ, nJ;
  int64_t cOff, qOff;      // batch-relative entry offsets into the C / Q pools
  int32_t rOff, colOff;    // batch-relative offsets into the used-row / used-column flags
  int32_t kcap;            // pool capacity in ACA terms, <= min(max_iter, nI, nJ)
  int32_t list_idx;        // position in the far list (ranks are recorded there)
  int64_t xOff;            // batch-relative offset into the FP32 pivot scratch (kXcHead + 9 kcap floats)
};

// done: 0 = iterating, 1 = converged (applied to u), 2 = deferred (reached its pool
// capacity kcap before the stopping rule; not applied, to be rerun with a larger pool)
struct FarState {
  int32_t k, done;
  double mu2, nu2;
};

// Counters kept on the device per batch.
enum FarCtr { kCtrActive = 0, kCtrTotI, kCtrTotJ, kCtrRemaining, kCtrError, kCtrRankMax, kCtrDeferred, kCtrCount = 8 };

struct FarArgs {
  const FarBlock* blocks;
  int nb;
  FarState* state;
  int32_t* rows;      // [nb][ldr]
  int32_t* cols;      // [nb][ldr]
  int ldr;            // max_iter + 1
  uint8_t* usedRow;
  uint8_t* usedCol;
  pool_t* C;          // [entries][9]
  pool_t* Q;
  float* xc;          // per-block scratch of the FP32 pivot kernels (C-side norm terms)
  int32_t* act;       // active block list
  int32_t* preI;      // exclusive prefix of nI over active blocks (nact + 1)
  int32_t* preJ;
  int32_t* ctr;       // FarCtr counters
  unsigned long long* rank_sum;
  unsigned long long* evals;
  int32_t* rank_out;  // [far list size]: ACA rank of each converged block
  const float4* x;
  const float4* f;
  double* u;
  int max_iter;
  double eps2;
  int use_symmetry;
  int defer_apply;  // 1: converged blocks are applied later by far_student_check
  int fast_pivots;  // 1: orthogonalisation, pivot search and stopping norms in FP32 (the fast
                    // forms); 0: in FP64, as the restated reference
};

constexpr int kFarSamples = 64;  // sampled entries per block in the student residual check

// One ACA batch to completion. Queries: student != nullptr -> student network; else
// tcw != nullptr -> teacher on the tensor cores; else teacher FP32 SIMT. known_iters > 0:
// every block stops (converges or is deferred) within that many iterations, so they are
// launched without reading the counters back in between; 0: counters are read every
// few iterations. Returns the number of deferred blocks.
// Optional per-category timing of a batch: CUDA events around every launch, summed after the
// batch (milliseconds added to the four totals).
struct FarTimer {
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  double active_ms = 0, query_ms = 0, pivot_ms = 0;
  cudaEvent_t next();  // records nothing; returns a fresh event from the pool
  void collect();      // sums the recorded batch (after the stream has synchronised)
  ~FarTimer();
};

int far_batch_plain(const FarArgs& a, const MlpF32& w, const TcWeights* tcw, const float* student, int* err,
                    int num_sms, int32_t* host_ctr, cudaStream_t s, int known_iters, int* iterations,
                    FarTimer* timer = nullptr);

// Graph form of a batch (no host read-back): its state and `iters` iterations, every block's rank
// known in advance; far_batch_end folds its counters into `status` and lists the blocks to rerun
// (see k_batch_end in far_aca.cu).
void far_batch_launch(const FarArgs& a, const MlpF32& w, const TcWeights* tcw, const float* student, int* err,
                      int num_sms, cudaStream_t s, int iters);
void far_batch_end(const FarArgs& a, int* status, int32_t* lists, int cap, cudaStream_t s);
// far_student_check without the read-back of the count of blocks sent back to the teacher.
void far_student_check_launch(const FarArgs& a, const TcWeights& tcw, const float* student, float tol, float* feat,
                              float* yt, float* ys, int* nfail_dev, int* err, int num_sms, cudaStream_t s);

// Student residual check of a finished batch run with defer_apply = 1: kFarSamples entries per
// converged block are evaluated by the student and by the teacher (tensor cores); blocks whose
// relative residual exceeds tol are marked done = 3 (to be rerun with the teacher), the others
// are applied to u. feat / yt / ys: device scratch of nb * kFarSamples * (3 / 9 / 9) floats.
// Returns the number of marked blocks.
int far_student_check(const FarArgs& a, const TcWeights& tcw, const float* student, float tol, float* feat, float* yt,
                      float* ys, int* nfail_dev, int* err, int num_sms, cudaStream_t s);

// student network (student.cu)
size_t student_grad_smem();
void launch_student_samples(float* r, int64_t n, uint64_t seed, float rmin, float rmax, cudaStream_t s);
void launch_student_targets(const float* r, float* t, int64_t n, cudaStream_t s);
void launch_student_grad(const float* params, const float* r, const float* t, int64_t nsamples, int64_t batch,
                         uint64_t step_seed, float* partial, float* loss_partial, float* grad, float* loss,
                         cudaStream_t s);
void launch_student_adam(float* p, const float* g, float* m1, float* m2, float lr, float b1t, float b2t,
                         cudaStream_t s);
void launch_student_eval(const float* params, const float* r, float* y, int64_t n, int num_sms, cudaStream_t s);
void launch_far_student(const FarArgs& a, const float* params, int which, int* err, int num_sms, cudaStream_t s);

// tensor-core kernels (tc_kernels.cu); err receives a nonzero code if a bounded wait timed out
void launch_near_tc(const NearArgs& a, const TcWeights& w, int* work_counter, int* err, int num_sms, cudaStream_t s);
void launch_far_tc(const FarArgs& a, const TcWeights& w, int which, int* err, int num_sms, cudaStream_t s);
void launch_eval_tc(const float* r, float* y, int64_t n, const TcWeights& w, int* err, int num_sms, cudaStream_t s);

// ---------------------------------------------------------------- time step (step.cu)
// The reference's squared search radius: epsilon is a float and is squared in float
// (include/PointCloudSearch.hpp:395-397, epsilons(i) * epsilons(i) of a float view), then widened.
__host__ __device__ inline double radius_sq(double eps) {
  const float e = (float)eps;
#ifdef __CUDA_ARCH__
  return (double)__fmul_rn(e, e);
#else
  return (double)(e * e);
#endif
}

struct CellGrid {
  double3 lo;
  double inv;  // 1 / cell size (cell coordinates in double: exact to far below the cell margin)
  int nx, ny, nz, ncell;
};

// Morse pair force parameters (include/PotentialForce.hpp:115-140 hard-codes De = 1, a = 1,
// re = 2.5); cutoff = radius of the neighbour search (0: no pair forces).
struct MorseParams {
  float De, a, re;
  double cutoff;
};

constexpr int kMaxCells = 16 * 1024 * 1024;

// Filament forces of python/simulate.py:14-88. rest_length and k_t meet float32 arrays there and
// act as float32; k_b scales the float64 bending sum.
struct FilamentParams {
  int64_t n_filament;
  int n_chain;
  float rest_length, k_t;
  double k_b;
};

// Uniform grid of cells no smaller than the cutoff over the positions' bounding box; items lists
// the positions cell by cell (start[c] .. start[c + 1]).
struct CellList {
  CellGrid grid{};
  DevBuf box, cell, items, count, start, sums, iota, sorted_cell, sort_tmp;
  void build(const float4* x, int64_t n, double cutoff, cudaStream_t s);
  void release() {
    for (DevBuf* b : {&box, &cell, &items, &count, &start, &sums, &iota, &sorted_cell, &sort_tmp}) b->release();
  }
};

// f = gravity + Morse forces of every position (f4 and / or f3 (n, 3); either may be null).
void launch_morse(const float4* x, int64_t n, const CellList& cl, const MorseParams& mp, float3 grav, float4* f4,
                  float* f3, cudaStream_t s);
// Neighbours j != i within the cutoff (the reference's radius-search test): per-particle counts
// (out null) or the sorted lists at out[off[i] ..].
void launch_neighbours(const float4* x, int64_t n, const CellList& cl, double cutoff, int64_t* count,
                       const int64_t* off, int* out, cudaStream_t s);
void launch_advance(float4* x, const double* u, int64_t n, float dt, cudaStream_t s);

// Dormand-Prince stage positions x = x0 + sum_t k[j_t] c_t (k: 7 stage velocities, float (n, 3)
// each, k_j at offset (j - 1) 3n) and the error estimate (summed into *err, zeroed first).
struct Dp45Terms {
  int n;
  int j[5];
  float c[5];
};
struct Dp45Error {
  float dc[6];  // k1, k3, k4, k5, k6, k7
  float dt;
};
void launch_dp45_stage(const float4* x0, const float* k, int64_t n, const Dp45Terms& tm, float4* x, cudaStream_t s);
void launch_velocity_to_float(const double* u, int64_t m, float* k, cudaStream_t s);
void launch_dp45_error(const float* k, int64_t n, const Dp45Error& de, double* err, cudaStream_t s);
// f += bending, then f += tension, for the filament rows (row -> slot of x and f: slot[row], or
// the row itself when slot is null); f4 or f3 (n, 3) as in launch_morse.
void launch_filaments(const float4* x, const int32_t* slot, const FilamentParams& fp, float4* f4, float* f3,
                      cudaStream_t s);
void launch_pack_positions(const float* xyz, int64_t n, float4* x4, cudaStream_t s);

// ---------------------------------------------------------------- reorder / misc
void launch_gather_forces(const float* f, const int32_t* perm, float4* f4, double* u, int64_t n, cudaStream_t s);
void launch_scatter_velocities(const double* u, const int32_t* perm, float* out, int64_t n, cudaStream_t s);
void launch_eval_simt(const float* r, float* y, int64_t n, const MlpF32& w, int num_sms, cudaStream_t s);
void launch_gather_positions(const float4* x4, const int32_t* pos, float4* out, int64_t n, cudaStream_t s);

}  // namespace hignn
