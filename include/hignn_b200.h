/*
 * hignn_b200 -- C ABI of the B200-native H-HIGNN mobility matvec U = M(x) F.
 *
 * Each entry point replaces a method of the reference's HignnModel, which its
 * pybind11 module `hignn` exposes (interface/HignnInterface.cpp:17-35). Plain
 * pointers and sizes only; every call returns an int status (0 = ok, < 0 =
 * error) and hignn_last_error() gives the message of the calling thread's last
 * failure. A model owns one CUDA stream on its device; calls on one model are
 * not thread-safe, calls on different models are. Host arrays are (n, 3)
 * row-major float32 in the caller's particle order, as the reference's numpy
 * arrays are (src/HignnModel.cpp:569-570).
 */
#ifndef HIGNN_B200_H
#define HIGNN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HIGNN_OK 0
#define HIGNN_ERR_ARG (-1)     /* bad argument: null pointer, size mismatch, bad key   */
#define HIGNN_ERR_CUDA (-2)    /* a CUDA runtime call failed                             */
#define HIGNN_ERR_STATE (-3)   /* call out of order: no weights, no tree, no device    */
#define HIGNN_ERR_IO (-4)      /* weight file missing or malformed                       */
#define HIGNN_ERR_LIMIT (-5)   /* a device loop hit its iteration cap; see message       */
#define HIGNN_ERR_NODEV (-6)   /* model was created without a device (host-only)        */

typedef struct hignn_model hignn_model;

/* Parameter keys for hignn_set_param / hignn_get_param. The first nine are the
 * reference's setters (src/HignnModel.cpp:773-874), defaults from its
 * constructor (src/HignnModel.cpp:337-379). */
enum hignn_param {
  HIGNN_P_EPSILON = 0,                    /* ACA tolerance, default 0.05                 */
  HIGNN_P_ETA = 1,                        /* stored, unused (as in the reference)       */
  HIGNN_P_MAX_ITER = 2,                   /* ACA iteration cap, default 100              */
  HIGNN_P_MAT_POOL_SIZE_FACTOR = 3,       /* stored; pools here are sized per batch     */
  HIGNN_P_MAX_FAR_DOT_WORK_NODE_SIZE = 4, /* stored; batches are sized by pool memory    */
  HIGNN_P_MAX_RELATIVE_COORD = 5,         /* far-size gate of the close/far check, 500000 */
  HIGNN_P_POST_CHECK_FLAG = 6,            /* dense re-check after each dot, default 0   */
  HIGNN_P_USE_SYMMETRY = 7,               /* J >= I lists + transposed update, default 1 */
  HIGNN_P_MAX_FAR_FIELD_DISTANCE = 8,     /* stored, unused (as in the reference)       */
  /* keys of this implementation */
  HIGNN_P_PRECISION = 100,       /* 0 = plain FP32 (default), 1 = BF16 tensor cores, 2 = BF16 + student far field;
                                    1 and 2 need block_size <= 128                               */
  HIGNN_P_FAR_BATCH_ROWS = 101,  /* max rows (sum of |I|+|J|) per ACA batch, default 1<<26, at most 1<<30 */
  HIGNN_P_TIMING = 102,          /* 1 = per-phase CUDA-event times in hignn_stats, 2 = also the
                                    far-field breakdown (events around every far launch)        */
  HIGNN_P_STUDENT_TOL = 103,     /* student fallback: a far block whose 64 sampled entries differ from
                                    the teacher by more than max(this, epsilon) relative (Frobenius)
                                    is recomputed with the teacher; default 1e-3                   */
  HIGNN_P_FIELDS = 104,          /* bit 0 = near field, bit 1 = far field (default 3), for diagnostics */
  HIGNN_P_RECORD_PIVOTS = 105,   /* 1 = keep every far block's ACA rank and pivots (hignn_get_far_pivots) */
  HIGNN_P_FAR_POOL_MB = 106,     /* C + Q pool memory of one ACA batch in MiB, default 24576, at most 1<<24 */
  HIGNN_P_RANK_HINT_OFFSET = 107, /* added to the recorded ACA ranks when planning (default 0; a
                                    negative value exercises the deferral path in tests)        */
  HIGNN_P_TREE_DEVICE = 108,      /* 1 (default on a device model) = build the cluster tree on the
                                     device, 0 = on the host; both give the same tree and lists */
  HIGNN_P_GRAPH = 109,            /* 1 (default) = a rank-planned H-matvec (the ACA ranks of every far
                                     block recorded by a previous product on the same tree and
                                     settings) runs as one captured CUDA graph with a single
                                     read-back; 0 = every launch from the host */
  HIGNN_P_KEEP_RANKS = 110        /* 1 (default) = a tree rebuild keeps the recorded ACA rank of every
                                     far block that joins the same two nodes (ids and particle
                                     ranges) as before, so the next product is planned; 0 = every
                                     rebuild forgets the ranks, and the next product is a first one,
                                     as every product of the reference's time loop. The result does
                                     not depend on it. */
};

typedef struct hignn_stats {
  int64_t n;               /* particles                                          */
  int64_t num_nodes;       /* cluster-tree rows (orphan rows 1, 2 included)      */
  int64_t num_leaves;
  int64_t num_close;       /* close leaf pairs in the list (J >= I with symmetry) */
  int64_t num_far;         /* far node pairs in the list                         */
  int64_t close_evals;     /* two-body evaluations of the last near field       */
  int64_t far_evals;       /* two-body evaluations of the last ACA               */
  int64_t far_rank_sum;    /* sum of ACA ranks of the last far field            */
  int32_t far_rank_max;
  int32_t far_iterations;  /* ACA iterations summed over batches                 */
  int64_t student_fallback_blocks; /* far blocks that fell back to the teacher   */
  double t_build_ms;       /* host tree + lists of the last update_coord        */
  double t_close_ms;       /* device time of the last near field (TIMING = 1)   */
  double t_far_ms;         /* device time of the last far field (TIMING = 1)    */
  double t_dot_ms;         /* device time of the last dot (TIMING = 1)          */
  int64_t gpu_launches;    /* kernels launched by the last dot                    */
  /* far-field breakdown of the last dot (TIMING = 2; CUDA events around each launch) */
  double t_far_query_ms;   /* column / row queries (network evaluations)         */
  double t_far_pivot_ms;   /* orthogonalisation, pivots, stopping norms, apply    */
  double t_far_active_ms;  /* active lists                                       */
  double t_far_check_ms;   /* student residual check and deferred apply          */
} hignn_stats;

/* Message of the calling thread's last error (empty string if none). */
int hignn_last_error(char* buf, size_t size);

/* Library version, e.g. 100 for 0.1.0. */
int hignn_version(void);

/* HignnModel(coord, blockSize) -- src/HignnModel.cpp:335-386, plus the first
 * Update() (src/HignnModel.cpp:457-461) so the model is ready for dot.
 * device >= 0 selects a CUDA device; device = -1 makes a host-only model whose
 * tree and lists can be inspected but whose dot calls fail (no CPU fallback). */
int hignn_create(const float* xyz, int64_t n, int block_size, int device, hignn_model** out);

int hignn_destroy(hignn_model* m);

/* LoadTwoBodyModel -- src/HignnModel.cpp:402-433. `path` names an .hgnw weight
 * blob (see hignn_b200/weights.py) instead of a TorchScript file. */
int hignn_load_two_body(hignn_model* m, const char* path);

/* Weights from memory: dims = {3, h1, ..., 9}, w/b concatenated per layer
 * (row-major out x in, then bias), activation 1 = tanh. */
int hignn_load_two_body_mem(hignn_model* m, int num_layers, const int32_t* dims, const float* params,
                            int activation);

/* Setters of src/HignnModel.cpp:773-874 and this implementation's keys. */
int hignn_set_param(hignn_model* m, int key, double value);
int hignn_get_param(hignn_model* m, int key, double* value);

/* UpdateCoord -- src/HignnModel.cpp:744-762: copy coordinates, rebuild the tree
 * (src/Build.cpp:17-265) and the close/far lists (src/CloseFarCheck.cpp:11-465). */
int hignn_update_coord(hignn_model* m, const float* xyz, int64_t n);

/* New coordinates on the existing tree: the positions are replaced, the cluster tree, the
 * close/far lists and the ACA plan are kept (the reference always rebuilds,
 * src/HignnModel.cpp:744-762; a simulation that rebuilds every k steps moves the particles in
 * between with this call). */
int hignn_update_coord_keep_tree(hignn_model* m, const float* xyz, int64_t n);

/* Pair forces of PotentialForce::GetPotentialForce (include/PotentialForce.hpp:468-593) plus a
 * uniform body force: f_i = gravity + sum over j != i with |x_i - x_j| < cutoff and
 * |r| > 1e-3 of r fMag / |r|, r = x_i - x_j, fMag = -2 a De (exp(-a(|r| - re)) - exp(-2a(|r| - re)))
 * (the reference hard-codes De = 1, a = 1, re = 2.5). Neighbours from a device cell list.
 * Host pointers, (n, 3) float32; gravity may be null; cutoff = 0 gives gravity only. */
int hignn_pair_forces(hignn_model* m, const float* xyz, float* f, int64_t n, const float* gravity, double De,
                      double a, double re, double cutoff);

/* The forces of a step: a body force, Morse pair forces (as hignn_pair_forces; cutoff 0: none)
 * and the filament forces of python/simulate.py:14-88 (chain_bending, then chain_tension, each
 * added to the float32 force as velocity_update does at :130-142). Filament f holds rows
 * f * n_chain .. (f + 1) * n_chain - 1 for f < n_filament; the rest are free particles. The
 * filament arithmetic follows numpy's: float32 arms, norms, crosses and tension, float64 sums. */
typedef struct hignn_force_model {
  float gravity[3];
  double morse_De, morse_a, morse_re, morse_cutoff;
  int64_t n_filament;
  int32_t n_chain;
  double rest_length, k_t, k_b;
} hignn_force_model;

/* f (n, 3) = the forces of fm at positions xyz (n, 3); host pointers. */
int hignn_forces(hignn_model* m, const float* xyz, float* f, int64_t n, const hignn_force_model* fm);

/* ExplicitEuler::Run (include/TimeIntegrator.hpp:431-488) with the velocity callback's work on
 * the device: per step f = the forces of fm (as hignn_forces), u = M(x) f (as hignn_dot,
 * current settings), x += u dt (float). The tree and lists are built for xyz and rebuilt
 * every `rebuild_every` steps (0: never); in between positions move on the kept tree.
 * xyz (n, 3) is read as the start and overwritten with the final positions. */
int hignn_run_euler(hignn_model* m, float* xyz, int64_t n, int steps, double dt, int rebuild_every,
                    const hignn_force_model* fm);

/* As hignn_run_euler with the explicit midpoint rule (second order; an addition -- the reference
 * integrates with Euler or Dormand-Prince): x_mid = x + (dt/2) u(x) on the kept tree, then
 * x += dt u(x_mid), each u = M F with the forces of fm at those positions. */
int hignn_run_rk2(hignn_model* m, float* xyz, int64_t n, int steps, double dt, int rebuild_every,
                  const hignn_force_model* fm);

/* ExplicitRk4::Run (include/TimeIntegrator.hpp:602-860) with the velocity of fm (and of an
 * attached three-body object) on the device: adaptive Dormand-Prince 5(4) from t = 0 to tf with
 * the reference's float stage arithmetic, error norm and step control (initial step dt0, error
 * threshold), tree rebuilt every `rebuild_every` accepted steps (0: never). *steps_taken (may be
 * NULL) receives the number of accepted steps. */
int hignn_run_dp45(hignn_model* m, float* xyz, int64_t n, double tf, double dt0, double threshold,
                   int rebuild_every, const hignn_force_model* fm, int64_t* steps_taken);

/* Dot -- src/HignnModel.cpp:545-634: u = M(x) f through the H-matrix (close
 * field + ACA far field). Host pointers; u is written, its input ignored. */
int hignn_dot(hignn_model* m, float* u, const float* f, int64_t n);

/* Same operation on device pointers (caller's order), stream-ordered on the
 * model's stream; returns when the result is in d_u. */
int hignn_dot_device(hignn_model* m, float* d_u, const float* d_f, int64_t n);

/* DenseDot -- src/HignnModel.cpp:660-728 with src/DenseDot.cpp:22-320:
 * u_i = sum_j 0.5 (M + M^T)(x_j - x_i) f_j over all pairs, FP32 network,
 * FP64 accumulation. Host pointers. */
int hignn_dense_dot(hignn_model* m, float* u, const float* f, int64_t n);

/* Dense rows for accuracy checks (PostCheckDot, src/PostCheckDot.cpp:351-376, on chosen rows):
 * for each listed target row (caller's order) u_row = sum over all j of
 * 0.5 (M + M^T)(x_j - x_row) f_j, accumulated in FP64. precision 0: the FP32 network;
 * HIGNN_DENSE_F64: the network in FP64 (weights promoted from FP32, features x_j - x_row
 * in FP64) -- the FP64 dense evaluation the H-matrix error is stated against. Host
 * pointers; u_rows is (nrows, 3); rows may repeat. */
#define HIGNN_DENSE_F64 64
int hignn_dense_rows(hignn_model* m, double* u_rows, const float* f, const int64_t* rows, int64_t nrows,
                     int precision);

/* Allocation-free variant of hignn_dense_rows (same arguments and results); it has
 * no counterpart in the reference. It serves callers that cannot allocate device
 * memory once they are running -- a time-stepping code whose device-memory budget
 * is fixed at start-up, or a host framework whose own caching allocator owns the
 * GPU: it calls no cudaMalloc, cudaFree or allocating library routine. Its per-call
 * scratch lives in one static device array of about 6.3 MB that every GPU which
 * loads this library holds until the process exits. Limits: nrows <=
 * HIGNN_NOALLOC_MAX_ROWS and a tree of at most HIGNN_NOALLOC_MAX_LEAVES leaves
 * (larger sizes return HIGNN_ERR_ARG); precision 0 only. The model must already
 * hold weights and a built tree (hignn_update_coord or hignn_dot once: those may
 * allocate). The first call on a device looks up the array's address; make it
 * before any stream capture. All calls share the array; a process-wide lock,
 * held until a call's GPU work has finished, serialises the calls (on every GPU),
 * so the race to avoid is with the caller's own GPU work on the same model's force
 * and position buffers, issued on another stream while a call runs. */
#define HIGNN_NOALLOC_MAX_ROWS 131072
#define HIGNN_NOALLOC_MAX_LEAVES 65536
int hignn_dense_rows_noalloc(hignn_model* m, double* u_rows, const float* f, const int64_t* rows, int64_t nrows,
                             int precision);

/* Two-body kernel M(r) on n features (device pointers, r: (n,3), y: (n,9) row-major
 * 3x3): python/convert.py:11-20. precision 0 = FP32 SIMT, 1 = BF16 tensor cores. */
int hignn_two_body_eval(hignn_model* m, const float* d_r, float* d_y, int64_t n, int precision);

/* Far-field student network (no counterpart in the reference; the student is new work).
 * A 3-32-32-32-9 SiLU network on x = r_hat ln(|r|/2) predicting the teacher's inner
 * output minus the Rotne-Prager-Yamakawa tensor; used for the ACA queries of
 * admissible blocks when HIGNN_P_PRECISION = 2. Parameters (2537 floats): W1 (32x3),
 * b1, W2 (32x32), b2, W3 (32x32), b3, W4 (9x32), b4, row-major. */
#define HIGNN_STUDENT_PARAMS 2537

/* Trains the student on the device from teacher evaluations at separations drawn
 * log-uniform in [4, 400] with uniform directions: nsamples teacher samples, Adam
 * (cosine-decayed from lr), mini-batches of `batch`. final_loss: mean squared error
 * of the inner output on one more batch. */
int hignn_train_student(hignn_model* m, int steps, int batch, int64_t nsamples, double lr, uint64_t seed,
                        double* final_loss);
int hignn_set_student(hignn_model* m, const float* params, int nparams);
int hignn_get_student(hignn_model* m, float* params, int nparams);

/* Student M(r) on n features (device pointers, r: (n,3), y: (n,9)). */
int hignn_student_eval(hignn_model* m, const float* d_r, float* d_y, int64_t n);

/* Gradient (host array of HIGNN_STUDENT_PARAMS floats) and loss of mean((net(x(r)) - t)^2)
 * over a batch of features d_r (n,3) and residual targets d_t (n,9), device pointers. */
int hignn_student_grad(hignn_model* m, const float* d_r, const float* d_t, int64_t n, float* grad, double* loss);

/* Sizes of the tree and lists built by the last update. */
int hignn_get_stats(hignn_model* m, hignn_stats* out);

/* Tree rows [child0, child1, start, end, level] (num_nodes x 5) and the
 * permutation (tree position -> caller index), as src/Build.cpp leaves them. */
int hignn_get_tree(hignn_model* m, int64_t* tree5, int64_t* perm);

/* Close leaf pairs and far node pairs in the reference's list order
 * (src/CloseFarCheck.cpp:298-408). Arrays sized from hignn_get_stats. */
int hignn_get_lists(hignn_model* m, int64_t* close_i, int64_t* close_j, int64_t* far_i, int64_t* far_j);

/* Shard of the block lists for one of `world` processes (one GPU each), no counterpart
 * of its own in the reference: there MPI ranks take interleaved shares of the close and far
 * lists (src/CloseFarCheck.cpp:309,323,394,401) and all-reduce u (src/HignnModel.cpp:602).
 * Here each rank takes a contiguous, cost-balanced range of each list; hignn_dot and
 * hignn_dot_device then return this rank's partial velocities, which the caller sums over
 * the ranks (an NCCL all-reduce of the (n, 3) float32 result). rank = 0, world = 1 (the
 * default) is the whole product. */
int hignn_set_shard(hignn_model* m, int rank, int world);

/* The shard's ranges: ranges[4] = {close begin, close end, far begin, far end} in list order. */
int hignn_get_shard(hignn_model* m, int64_t* ranges);

/* ACA ranks and pivot sequences of the last far field (needs HIGNN_P_RECORD_PIVOTS = 1):
 * ranks[num_far]; rows / cols [num_far][ld] with ld >= max_iter + 1, block-local indices
 * (rows[b][l] = pivot row of iteration l, cols[b][l] = its column), in list order. */
int hignn_get_far_pivots(hignn_model* m, int32_t* ranks, int32_t* rows, int32_t* cols, int ld);

/* Synchronize the model's stream. */
int hignn_synchronize(hignn_model* m);

/* The model's CUDA stream (cudaStream_t), for callers that order their own work. */
int hignn_get_stream(hignn_model* m, void** stream);

/* ---------------------------------------------------------------- neighbour lists
 * The reference's NeighborLists class (include/NeighborLists.hpp, bound at
 * interface/HignnInterface.cpp:73-91), built on the device. A neighbour of i is any j with
 * sqrt(sum (double)(x_j - x_i)^2)^2 < (float)eps * (float)eps (the kd-tree radius search of
 * include/PointCloudSearch.hpp:274-450). Each particle's neighbours come out in ascending
 * index order (the reference's follow its kd-tree traversal; the sets are the same). */
typedef struct hignn_nbl hignn_nbl;

#define HIGNN_EDGES_TWO_BODY 0        /* (2, E): (i, j), j in N(i) \ {i} at the two-body eps   */
#define HIGNN_EDGES_THREE_BODY 1      /* (3, E): (i, j, k), j in N(i) \ {i}, k in N(j) \ {j, i} */
#define HIGNN_EDGES_THREE_BODY_SELF 2 /* (2, E): (i, j), j in N(i) \ {i} at the three-body eps */

/* NeighborLists::NeighborLists: an empty set of lists on `device`. */
int hignn_nbl_create(int device, hignn_nbl** out);
void hignn_nbl_destroy(hignn_nbl* l);

/* NeighborLists::UpdateCoord (include/NeighborLists.hpp:252-279): copy n float32 (x, y, z)
 * rows (host). Lists built before stay until the next build. */
int hignn_nbl_update_coord(hignn_nbl* l, const float* xyz, int64_t n);

/* SetTwoBodyEpsilon / SetThreeBodyEpsilon (include/NeighborLists.hpp:281-287). */
int hignn_nbl_set_two_body_epsilon(hignn_nbl* l, float eps);
int hignn_nbl_set_three_body_epsilon(hignn_nbl* l, float eps);

/* BuildTwoBodyInfo (include/NeighborLists.hpp:466-510) and BuildThreeBodyInfo (:512-585; the
 * triplets and the self edges). The epsilon must be positive (the reference's lists underflow
 * at 0). */
int hignn_nbl_build_two_body_info(hignn_nbl* l);
int hignn_nbl_build_three_body_info(hignn_nbl* l);

/* The getters of include/NeighborLists.hpp:289-464, two calls: with out = NULL only
 * *num_edges is set; then out (host, uint64 (rows, *num_edges) row-major, cap entries) is
 * filled. by_index = 0: Get{TwoBody,ThreeBody,ThreeBodySelf}EdgeInfo; by_index = 1: the
 * ByIndex variant for the nindex targets index[] (< n): two-body lists all j != p for each
 * target p, rows (j, p); three-body the target's triplets with rows (k, j, i); self rows
 * (j, i). A list that was never built has 0 edges. */
int hignn_nbl_get_edge_info(hignn_nbl* l, int kind, int by_index, const uint64_t* index, int64_t nindex,
                            uint64_t* out, int64_t cap, int64_t* num_edges);

/* A whole list on the device (uint64 (rows, *num_edges) row-major, owned by l, valid until
 * the next build or hignn_nbl_destroy); NULL when not built. */
int hignn_nbl_edge_info_device(hignn_nbl* l, int kind, const uint64_t** d_info, int64_t* num_edges);

/* Wall time of the last build (ms), and the lists' CUDA stream. */
int hignn_nbl_last_build_ms(hignn_nbl* l, double* ms);
int hignn_nbl_get_stream(hignn_nbl* l, void** stream);

/* ---------------------------------------------------------------- three-body near field
 * The three-body and self terms of HIGNN_model.forward (python/HIGNN/model_structure.py:76-139)
 * with Three_body_net (:41-55) and Two_body_self_net (:58-70): for every triplet (a, b, c) of
 * the three-body edge list at epsilon (NeighborLists::BuildThreeBodyInfo, read as (j, k, i)),
 *     u_c += (net3(x_b - x_a, x_c - x_b) / |x_b - x_a| / |x_c - x_b|) f_a
 * and for every self edge (a, b),  u_b += (net_self(x_a - x_b) / |x_a - x_b|^2) f_b
 * (the two-body term is the H-matrix product, hignn_dot). Networks kin -> 256 -> 1024 -> 512
 * -> 9 with tanh (kin 6 and 3); layer 1 in FP32 on the CUDA cores, layers 2, 3 and 4 on the
 * tensor cores (FP16 operands, FP32 accumulation). */
typedef struct hignn_tb hignn_tb;

#define HIGNN_TB_THREE_BODY 0
#define HIGNN_TB_SELF 1

int hignn_tb_create(int device, hignn_tb** out);
void hignn_tb_destroy(hignn_tb* t);

/* Load the three-body (which = HIGNN_TB_THREE_BODY, HGNW wrapper 2) or self (HIGNN_TB_SELF,
 * wrapper 3) network from an HGNW file, or from memory: dims[num_layers + 1], params = per layer
 * W (out x in, row-major) then b, float32. */
int hignn_tb_load(hignn_tb* t, int which, const char* path);
int hignn_tb_load_mem(hignn_tb* t, int which, int num_layers, const int32_t* dims, const float* params);

/* Three-body cutoff (the NeighborLists three-body epsilon; default 5). */
int hignn_tb_set_epsilon(hignn_tb* t, float eps);

/* u (n, 3) = three-body + self velocities for positions xyz and forces f (host, float32 (n, 3)).
 * Builds the edge lists on the device, then runs both networks. */
int hignn_tb_velocity(hignn_tb* t, const float* xyz, const float* f, float* u, int64_t n);

/* As hignn_tb_velocity, on edge lists the caller gives instead of the internal ones: tri (3, e3)
 * and self_edges (2, es), uint64 row-major host arrays with the rows of the reference's
 * NeighborLists::GetThreeBodyEdgeInfo / GetThreeBodyEdgeSelfInfo (include/NeighborLists.hpp:
 * 342-360, 405-422), in any edge order -- what python/gravity_field.py:31-52 passes to the torch
 * model. Every index must be < n. */
int hignn_tb_velocity_edges(hignn_tb* t, const float* xyz, const float* f, float* u, int64_t n, const uint64_t* tri,
                            int64_t e3, const uint64_t* self_edges, int64_t es);

/* Last call: ms of the list build, the three-body and the self kernels, and the edge counts. */
int hignn_tb_stats(hignn_tb* t, double* ms_lists, double* ms_three, double* ms_self, int64_t* triplets,
                   int64_t* pairs);

/* Attach a three-body object to a model (t = NULL detaches): hignn_run_euler, hignn_run_rk2 and
 * hignn_run_dp45 then add its three-body and self velocities (edge lists rebuilt at every evaluation at t's
 * epsilon, from the current positions) to u = M F -- the whole velocity of the HIGNN model
 * (python/HIGNN/model_structure.py:76-139 with the two-body part from the H-matrix). hignn_dot
 * is unchanged. t must outlive the attachment and live on the model's device. */
int hignn_set_three_body(hignn_model* m, hignn_tb* t);

/* Where the last call's kernels waited, summed over CTAs (12 counters: three-body, then self):
 * clocks the MMA lane waited for layer-1 operands, weight stages, layer-2 epilogues and the
 * layer-3 accumulator; its total clocks; clocks the producer waited for free weight slots. */
int hignn_tb_wait_profile(hignn_tb* t, uint64_t* counters);

/* Wait profile of the tensor-core near field (no counterpart in the reference; a tuning aid),
 * accumulated over the near fields run with HIGNN_P_TIMING >= 3 since the last call, then reset.
 * counters[16]: [c - 13] cycles that lane 0 of every warp spent in bounded waits with code c
 * (13-19 the MMA lane: features, layer-1 epilogue, quarters 0-3 read, layer-3 accumulator free;
 * 21-25 the epilogue: layer-1, layer-2, layer-3 accumulator, A2 buffer free, quarter 3's MMA
 * before the next A1), [13] cycles of one epilogue warp's whole run summed over CTAs, [15] tiles. */
int hignn_near_wait_profile(hignn_model* m, uint64_t* counters);

/* Phases of the last device time loop (hignn_run_euler / hignn_run_rk2; no counterpart in the
 * reference), ms[8]: wall milliseconds of the whole call, tree rebuilds (wall), forces, matvecs,
 * three-body terms (device time), steps, velocity evaluations, evaluations whose matvec ran
 * eagerly (no complete ACA rank plan yet; the others replayed a CUDA graph). */
int hignn_loop_profile(hignn_model* m, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* HIGNN_B200_H */
