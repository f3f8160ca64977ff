// Device time step: pair forces on a cell list, and the explicit Euler update.
//
// The reference assembles the forces in Python every step (python/simulate.py:14-144) -- gravity
// plus, for Morse suspensions, PotentialForce::GetPotentialForce (include/PotentialForce.hpp:
// 468-593): for each particle i, every neighbour j != i with |x_i - x_j| < cutoff (kd-tree radius
// search, metric sqrt(sum (double) d^2) squared against cutoff^2, strict,
// include/PointCloudSearch.hpp:231-240) contributes
//     f_i += r fMag / |r|,  r = x_i - x_j,  fMag = -2 a De (exp(-a (|r| - re)) - exp(-2 a (|r| - re)))
// when |r| > 1e-3 (include/PotentialForce.hpp:115-140; the reference hard-codes De = 1, a = 1,
// re = 2.5, here they are parameters). ExplicitEuler::Run (include/TimeIntegrator.hpp:431-488)
// then moves x += u dt with u the H-matvec of those forces. Here the whole step stays on the
// device: a uniform grid of cells no smaller than the cutoff replaces the kd-tree (the same
// neighbour set: every pair within the cutoff lies in adjacent cells), positions stay in tree
// order, and only the cluster tree is rebuilt on the host, every `rebuild_every` steps.
#include <cub/device/device_radix_sort.cuh>

#include <cfloat>
#include <cmath>
#include <cstring>

#include "common.h"
#include "kernels.h"

namespace hignn {

namespace {

// float <-> order-preserving unsigned int, for atomic min / max of floats
__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_bbox(const float4* __restrict__ x, int64_t n, unsigned* __restrict__ box /* [6] */) {
  unsigned lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float4 p = x[i];
    const unsigned k[3] = {fkey(p.x), fkey(p.y), fkey(p.z)};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo[d] = min(lo[d], k[d]);
      hi[d] = max(hi[d], k[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; d++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_down_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_down_sync(0xffffffffu, hi[d], o));
    }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int d = 0; d < 3; d++) {
      atomicMin(&box[d], lo[d]);
      atomicMax(&box[3 + d], hi[d]);
    }
}

__device__ __forceinline__ int3 cell_of(const float4 p, const CellGrid& g) {
  int cx = (int)floor(((double)p.x - g.lo.x) * g.inv), cy = (int)floor(((double)p.y - g.lo.y) * g.inv),
      cz = (int)floor(((double)p.z - g.lo.z) * g.inv);
  cx = min(max(cx, 0), g.nx - 1);
  cy = min(max(cy, 0), g.ny - 1);
  cz = min(max(cz, 0), g.nz - 1);
  return make_int3(cx, cy, cz);
}

__global__ void k_cell_count(const float4* __restrict__ x, int64_t n, CellGrid g, int* __restrict__ cell,
                             int* __restrict__ count) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int3 c = cell_of(x[i], g);
  const int id = (c.z * g.ny + c.y) * g.nx + c.x;
  cell[i] = id;
  atomicAdd(&count[id], 1);
}

// Exclusive scan of count[0, m) into start[0, m] (start[m] = total), two levels: blocks of 4096
// entries (1024 threads x 4), then one block over the block sums (m <= 4096 * 4096).
constexpr int kScanThreads = 1024, kScanPer = 4, kScanChunk = kScanThreads * kScanPer;

__device__ __forceinline__ int block_excl_scan(int v, int* warp_sums, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int z = warp_sums[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += y;
    }
    warp_sums[lane] = z;
  }
  __syncthreads();
  const int excl = (wid ? warp_sums[wid - 1] : 0) + x - v;
  if (total && threadIdx.x == 0) *total = warp_sums[31];
  __syncthreads();
  return excl;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(const int* __restrict__ count, int m,
                                                              int* __restrict__ start, int* __restrict__ sums) {
  __shared__ int ws[32];
  __shared__ int tot;
  const int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanPer;
  int v[kScanPer], s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer; q++) {
    v[q] = base + q < m ? count[base + q] : 0;
    s += v[q];
  }
  int e = block_excl_scan(s, ws, &tot);
#pragma unroll
  for (int q = 0; q < kScanPer; q++) {
    if (base + q < m) start[base + q] = e;
    e += v[q];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int* __restrict__ sums, int nb, int* __restrict__ total) {
  __shared__ int ws[32];
  __shared__ int tot;
  int v[kScanPer], s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer; q++) {
    const int k = threadIdx.x * kScanPer + q;
    v[q] = k < nb ? sums[k] : 0;
    s += v[q];
  }
  int e = block_excl_scan(s, ws, &tot);
#pragma unroll
  for (int q = 0; q < kScanPer; q++) {
    const int k = threadIdx.x * kScanPer + q;
    if (k < nb) sums[k] = e;
    e += v[q];
  }
  if (threadIdx.x == 0) *total = tot;
}

__global__ void k_scan_add(int* __restrict__ start, int m, const int* __restrict__ sums) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) start[k] += sums[k / kScanChunk];
}

__global__ void k_iota(int* __restrict__ v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int)i;
}

// f_i = g + sum of Morse forces of the neighbours of i within the cutoff (order of the reference's
// float arithmetic kept; the accumulation order follows the cell list).
__global__ void k_morse(const float4* __restrict__ x, int64_t n, CellGrid g, const int* __restrict__ start,
                        const int* __restrict__ items, MorseParams mp, float3 grav, float4* __restrict__ f4,
                        float* __restrict__ f3) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 xi = x[i];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (mp.cutoff > 0.0) {
    const int3 c = cell_of(xi, g);
    const double c2 = radius_sq(mp.cutoff);
    for (int dz = -1; dz <= 1; dz++) {
      const int z = c.z + dz;
      if (z < 0 || z >= g.nz) continue;
      for (int dy = -1; dy <= 1; dy++) {
        const int y = c.y + dy;
        if (y < 0 || y >= g.ny) continue;
        for (int dx = -1; dx <= 1; dx++) {
          const int xx = c.x + dx;
          if (xx < 0 || xx >= g.nx) continue;
          const int id = (z * g.ny + y) * g.nx + xx;
          for (int k = start[id]; k < start[id + 1]; k++) {
            const int j = items[k];
            if (j == (int)i) continue;
            const float4 xj = x[j];
            const double ddx = (double)xj.x - (double)xi.x, ddy = (double)xj.y - (double)xi.y,
                         ddz = (double)xj.z - (double)xi.z;
            const double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            if (!(dist * dist < c2)) continue;
            const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
            const float rn = sqrtf(rx * rx + ry * ry + rz * rz);
            if (!(rn > 1e-3f)) continue;
            const float e1 = expf(-mp.a * (rn - mp.re)), e2 = expf(-2.0f * mp.a * (rn - mp.re));
            const float fmag = (float)(-2.0 * (double)mp.a * (double)mp.De * (double)(e1 - e2));
            const float ratio = fmag / rn;
            fx += rx * ratio;
            fy += ry * ratio;
            fz += rz * ratio;
          }
        }
      }
    }
  }
  fx += grav.x;
  fy += grav.y;
  fz += grav.z;
  if (f4) f4[i] = make_float4(fx, fy, fz, 0.f);
  if (f3) {
    f3[3 * i] = fx;
    f3[3 * i + 1] = fy;
    f3[3 * i + 2] = fz;
  }
}

// The reference's neighbour test (kd-tree radius search): the distance sqrt(sum (double)(x_j -
// x_i)^2), squared, against cutoff^2, strict (include/PointCloudSearch.hpp:231-240, nanoflann
// RadiusResultSet::addPoint).
__device__ __forceinline__ bool is_neighbour(const float4 xi, const float4 xj, double c2) {
  const double dx = (double)xj.x - (double)xi.x, dy = (double)xj.y - (double)xi.y, dz = (double)xj.z - (double)xi.z;
  const double d = sqrt(dx * dx + dy * dy + dz * dz);
  return d * d < c2;
}

// Neighbours j != i of every i within the cutoff: count (out == nullptr) or write them, ascending,
// at out[off[i] ..] (insertion into the sorted run as they are found).
__global__ void k_neighbours(const float4* __restrict__ x, int64_t n, CellGrid g, const int* __restrict__ start,
                             const int* __restrict__ items, double cutoff, int64_t* __restrict__ count,
                             const int64_t* __restrict__ off, int* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 xi = x[i];
  const double c2 = radius_sq(cutoff);
  const int3 c = cell_of(xi, g);
  int cnt = 0;
  int* dst = out ? out + off[i] : nullptr;
  for (int dz = -1; dz <= 1; dz++) {
    const int z = c.z + dz;
    if (z < 0 || z >= g.nz) continue;
    for (int dy = -1; dy <= 1; dy++) {
      const int y = c.y + dy;
      if (y < 0 || y >= g.ny) continue;
      for (int dx = -1; dx <= 1; dx++) {
        const int xx = c.x + dx;
        if (xx < 0 || xx >= g.nx) continue;
        const int id = (z * g.ny + y) * g.nx + xx;
        for (int k = start[id]; k < start[id + 1]; k++) {
          const int j = items[k];
          if (j == (int)i || !is_neighbour(xi, x[j], c2)) continue;
          if (dst) {
            int q = cnt;
            while (q > 0 && dst[q - 1] > j) {
              dst[q] = dst[q - 1];
              q--;
            }
            dst[q] = j;
          }
          cnt++;
        }
      }
    }
  }
  if (count) count[i] = cnt;
}

// ---- filaments (python/simulate.py:14-88), numpy's arithmetic: every float32 operation rounded on
// its own (no contraction), the bending and tension sums in float64.
__device__ __forceinline__ float3 sub3(float3 a, float3 b) {
  return make_float3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
// np.linalg.norm(v, axis=1): sqrt((x^2 + y^2) + z^2) in float32
__device__ __forceinline__ float norm3(float3 a) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z)));
}
__device__ __forceinline__ float3 div3(float3 a, float d) {
  return make_float3(__fdiv_rn(a.x, d), __fdiv_rn(a.y, d), __fdiv_rn(a.z, d));
}
// np.cross: (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0), products rounded before the difference
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
                     __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                     __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// chain_bending's f21 and f23 of the angle at beads (p0, p1, p2) (python/simulate.py:33-50)
__device__ void bend_terms(float3 p0, float3 p1, float3 p2, float3& f21, float3& f23) {
  float3 a1 = sub3(p1, p0), a2 = sub3(p2, p1);
  a1 = div3(a1, norm3(a1));
  a2 = div3(a2, norm3(a2));
  const float c = __fadd_rn(__fadd_rn(__fmul_rn(a1.x, a2.x), __fmul_rn(a1.y, a2.y)), __fmul_rn(a1.z, a2.z));
  float t = __fsub_rn(1.0f, __fmul_rn(c, c));
  if (t < 0.f) t = 0.f;
  const float sn = __fsqrt_rn(t);
  const float3 uv = cross3(a1, a2);
  const float3 tq = make_float3(__fmul_rn(-uv.x, sn), __fmul_rn(-uv.y, sn), __fmul_rn(-uv.z, sn));
  f21 = cross3(tq, a1);
  f23 = cross3(tq, a2);
}

// chain_tension's nodal force of the bond (p0, p1) (python/simulate.py:77-86)
__device__ float3 tension_term(float3 p0, float3 p1, float rest, float kt) {
  const float3 r = sub3(p0, p1);
  const float rn = norm3(r);
  const float fm = __fmul_rn(kt, __fsub_rn(rn, rest));
  const float3 e = div3(r, rn);
  return make_float3(__fmul_rn(e.x, fm), __fmul_rn(e.y, fm), __fmul_rn(e.z, fm));
}

__global__ void k_filaments(const float4* __restrict__ x, const int32_t* __restrict__ slot, FilamentParams fp,
                            float4* __restrict__ f4, float* __restrict__ f3) {
  const int64_t rows = fp.n_filament * fp.n_chain;
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const int N = fp.n_chain;
  const int s = (int)(r % N);
  const int64_t base = r - s;
  auto pos = [&](int q) {
    const int64_t row = base + q;
    const float4 v = x[slot ? slot[row] : row];
    return make_float3(v.x, v.y, v.z);
  };
  // F[0:N-2] += f21; F[1:N-1] -= f21 + f23; F[2:N] += f23; F *= k_b
  double b[3] = {0.0, 0.0, 0.0};
  float3 f21, f23;
  if (s <= N - 3) {
    bend_terms(pos(s), pos(s + 1), pos(s + 2), f21, f23);
    b[0] = __dadd_rn(b[0], (double)f21.x);
    b[1] = __dadd_rn(b[1], (double)f21.y);
    b[2] = __dadd_rn(b[2], (double)f21.z);
  }
  if (s >= 1 && s <= N - 2) {
    bend_terms(pos(s - 1), pos(s), pos(s + 1), f21, f23);
    b[0] = __dsub_rn(b[0], (double)__fadd_rn(f21.x, f23.x));
    b[1] = __dsub_rn(b[1], (double)__fadd_rn(f21.y, f23.y));
    b[2] = __dsub_rn(b[2], (double)__fadd_rn(f21.z, f23.z));
  }
  if (s >= 2) {
    bend_terms(pos(s - 2), pos(s - 1), pos(s), f21, f23);
    b[0] = __dadd_rn(b[0], (double)f23.x);
    b[1] = __dadd_rn(b[1], (double)f23.y);
    b[2] = __dadd_rn(b[2], (double)f23.z);
  }
  // F[0:N-1] -= nodal; F[1:N] += nodal
  double t[3] = {0.0, 0.0, 0.0};
  if (s <= N - 2) {
    const float3 q = tension_term(pos(s), pos(s + 1), fp.rest_length, fp.k_t);
    t[0] = __dsub_rn(t[0], (double)q.x);
    t[1] = __dsub_rn(t[1], (double)q.y);
    t[2] = __dsub_rn(t[2], (double)q.z);
  }
  if (s >= 1) {
    const float3 q = tension_term(pos(s - 1), pos(s), fp.rest_length, fp.k_t);
    t[0] = __dadd_rn(t[0], (double)q.x);
    t[1] = __dadd_rn(t[1], (double)q.y);
    t[2] = __dadd_rn(t[2], (double)q.z);
  }
  const int64_t o = slot ? slot[r] : r;
  float v[3];
  if (f4) {
    const float4 w = f4[o];
    v[0] = w.x, v[1] = w.y, v[2] = w.z;
  } else {
    v[0] = f3[3 * o], v[1] = f3[3 * o + 1], v[2] = f3[3 * o + 2];
  }
#pragma unroll
  for (int d = 0; d < 3; d++) {
    v[d] = __double2float_rn(__dadd_rn((double)v[d], __dmul_rn(fp.k_b, b[d])));
    v[d] = __double2float_rn(__dadd_rn((double)v[d], t[d]));
  }
  if (f4)
    f4[o] = make_float4(v[0], v[1], v[2], 0.f);
  else
    f3[3 * o] = v[0], f3[3 * o + 1] = v[1], f3[3 * o + 2] = v[2];
}

// x += (float) u dt (include/TimeIntegrator.hpp:452: mPosition + mVelocity * dt, float velocity)
__global__ void k_advance(float4* __restrict__ x, const double* __restrict__ u, int64_t n, float dt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = x[i];  // a product and a sum, each rounded (no fused multiply-add), as the reference's host loop
  p.x = __fadd_rn(p.x, __fmul_rn((float)u[3 * i], dt));
  p.y = __fadd_rn(p.y, __fmul_rn((float)u[3 * i + 1], dt));
  p.z = __fadd_rn(p.z, __fmul_rn((float)u[3 * i + 2], dt));
  x[i] = p;
}

// ---- Dormand-Prince stages (ExplicitRk4::Run, include/TimeIntegrator.hpp:602-860): float
// arithmetic in the reference's order, each product and sum rounded on its own.
// x = x0 + k_j1 c_1 + k_j2 c_2 + ... (left to right), k_j the stage velocities (float, (n, 3)).
__global__ void k_dp45_stage(const float4* __restrict__ x0, const float* __restrict__ k, int64_t n, Dp45Terms tm,
                             float4* __restrict__ x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = x0[i];
  for (int t = 0; t < tm.n; t++) {
    const float* kj = k + (size_t)(tm.j[t] - 1) * 3 * n + 3 * i;
    p.x = __fadd_rn(p.x, __fmul_rn(kj[0], tm.c[t]));
    p.y = __fadd_rn(p.y, __fmul_rn(kj[1], tm.c[t]));
    p.z = __fadd_rn(p.z, __fmul_rn(kj[2], tm.c[t]));
  }
  x[i] = p;
}

__global__ void k_velocity_to_float(const double* __restrict__ u, int64_t m, float* __restrict__ k) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < m) k[q] = (float)u[q];
}

// Error estimate: ve = (k1 dc1 + k3 dc3 + k4 dc4 + k5 dc5 + k6 dc6 + k7 dc7) dt in float, |ve|^2 in
// float (Vec3::SquareMag), summed in double.
__global__ void k_dp45_error(const float* __restrict__ k, int64_t n, Dp45Error de, double* __restrict__ err) {
  double acc = 0.0;
  const size_t m = 3 * (size_t)n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float ve[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const size_t q = 3 * i + d;
      float v = __fmul_rn(k[q], de.dc[0]);
      v = __fadd_rn(v, __fmul_rn(k[2 * m + q], de.dc[1]));
      v = __fadd_rn(v, __fmul_rn(k[3 * m + q], de.dc[2]));
      v = __fadd_rn(v, __fmul_rn(k[4 * m + q], de.dc[3]));
      v = __fadd_rn(v, __fmul_rn(k[5 * m + q], de.dc[4]));
      v = __fadd_rn(v, __fmul_rn(k[6 * m + q], de.dc[5]));
      ve[d] = __fmul_rn(v, de.dt);
    }
    acc += (double)__fadd_rn(__fadd_rn(__fmul_rn(ve[0], ve[0]), __fmul_rn(ve[1], ve[1])), __fmul_rn(ve[2], ve[2]));
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(err, acc);
}

__global__ void k_pack_positions(const float* __restrict__ xyz, int64_t n, float4* __restrict__ x4) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x4[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.f);
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void CellList::build(const float4* x, int64_t n, double cutoff, cudaStream_t s) {
  grid = CellGrid{};
  if (n <= 0) return;
  if (!(cutoff > 0.0)) throw Error(-1, "cell list: cutoff must be positive");
  box.ensure(sizeof(unsigned) * 8);
  const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  HIGNN_CUDA(cudaMemcpyAsync(box.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
  k_bbox<<<nblk(n, 256) < 1024 ? nblk(n, 256) : 1024, 256, 0, s>>>(x, n, box.as<unsigned>());
  HIGNN_CHECK_LAUNCH();
  unsigned hb[6];
  HIGNN_CUDA(cudaMemcpyAsync(hb, box.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
  HIGNN_CUDA(cudaStreamSynchronize(s));
  auto unkey = [](unsigned k) {
    const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  };
  float lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = unkey(hb[d]);
    hi[d] = unkey(hb[3 + d]);
    if (!(std::isfinite(lo[d]) && std::isfinite(hi[d]))) throw Error(-1, "cell list: non-finite positions");
  }
  // cells no smaller than the cutoff (a little larger, so rounding never splits a neighbour pair
  // across non-adjacent cells), at most kMaxCells of them
  double size = cutoff * (1.0 + 1e-5);
  // counts in double: a far-flung position must coarsen the grid, not overflow the product
  auto dims = [&](double sz, int* nd) {
    double tot = 1.0;
    for (int d = 0; d < 3; d++) {
      const double c = std::floor((double)(hi[d] - lo[d]) / sz) + 1.0;
      tot *= c;
      nd[d] = (int)std::min(c, (double)kMaxCells);
    }
    return tot;
  };
  int nd[3];
  while (dims(size, nd) > (double)kMaxCells) size *= 1.26;
  grid.lo = make_double3(lo[0], lo[1], lo[2]);
  grid.inv = 1.0 / size;
  grid.nx = nd[0];
  grid.ny = nd[1];
  grid.nz = nd[2];
  grid.ncell = nd[0] * nd[1] * nd[2];
  const int m = grid.ncell;
  const int nb = (m + kScanChunk - 1) / kScanChunk;
  cell.ensure(sizeof(int) * n);
  items.ensure(sizeof(int) * n);
  count.ensure(sizeof(int) * (m + 1));
  start.ensure(sizeof(int) * (m + 1));
  sums.ensure(sizeof(int) * (nb + 1));
  HIGNN_CUDA(cudaMemsetAsync(count.p, 0, sizeof(int) * (m + 1), s));
  k_cell_count<<<nblk(n, 256), 256, 0, s>>>(x, n, grid, cell.as<int>(), count.as<int>());
  k_scan_blocks<<<nb, kScanThreads, 0, s>>>(count.as<int>(), m, start.as<int>(), sums.as<int>());
  k_scan_sums<<<1, kScanThreads, 0, s>>>(sums.as<int>(), nb, start.as<int>() + m);
  k_scan_add<<<nblk(m, 256), 256, 0, s>>>(start.as<int>(), m, sums.as<int>());
  // items: particle indices ordered by (cell, index), by a stable radix sort of the cell ids, so
  // every sum over a cell's items runs in the same order on every build
  iota.ensure(sizeof(int) * n);
  sorted_cell.ensure(sizeof(int) * n);
  k_iota<<<nblk(n, 256), 256, 0, s>>>(iota.as<int>(), n);
  HIGNN_CHECK_LAUNCH();
  int bits = 1;
  while (bits < 31 && (1 << bits) < m) bits++;
  size_t tmp_bytes = 0;
  HIGNN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, cell.as<int>(), sorted_cell.as<int>(),
                                             iota.as<int>(), items.as<int>(), (int)n, 0, bits, s));
  sort_tmp.ensure(tmp_bytes > 0 ? tmp_bytes : 1);
  HIGNN_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp.p, tmp_bytes, cell.as<int>(), sorted_cell.as<int>(),
                                             iota.as<int>(), items.as<int>(), (int)n, 0, bits, s));
}

void launch_morse(const float4* x, int64_t n, const CellList& cl, const MorseParams& mp, float3 grav, float4* f4,
                  float* f3, cudaStream_t s) {
  if (n <= 0) return;
  k_morse<<<nblk(n, 128), 128, 0, s>>>(x, n, cl.grid, cl.start.as<int>(), cl.items.as<int>(), mp, grav, f4, f3);
  HIGNN_CHECK_LAUNCH();
}

void launch_neighbours(const float4* x, int64_t n, const CellList& cl, double cutoff, int64_t* count,
                       const int64_t* off, int* out, cudaStream_t s) {
  if (n <= 0) return;
  k_neighbours<<<nblk(n, 128), 128, 0, s>>>(x, n, cl.grid, cl.start.as<int>(), cl.items.as<int>(), cutoff, count, off,
                                            out);
  HIGNN_CHECK_LAUNCH();
}

void launch_advance(float4* x, const double* u, int64_t n, float dt, cudaStream_t s) {
  if (n <= 0) return;
  k_advance<<<nblk(n, 256), 256, 0, s>>>(x, u, n, dt);
  HIGNN_CHECK_LAUNCH();
}

void launch_filaments(const float4* x, const int32_t* slot, const FilamentParams& fp, float4* f4, float* f3,
                      cudaStream_t s) {
  const int64_t rows = fp.n_filament * (int64_t)fp.n_chain;
  if (rows <= 0) return;
  k_filaments<<<nblk(rows, 128), 128, 0, s>>>(x, slot, fp, f4, f3);
  HIGNN_CHECK_LAUNCH();
}

void launch_dp45_stage(const float4* x0, const float* k, int64_t n, const Dp45Terms& tm, float4* x, cudaStream_t s) {
  if (n <= 0) return;
  k_dp45_stage<<<nblk(n, 256), 256, 0, s>>>(x0, k, n, tm, x);
  HIGNN_CHECK_LAUNCH();
}

void launch_velocity_to_float(const double* u, int64_t m, float* k, cudaStream_t s) {
  if (m <= 0) return;
  k_velocity_to_float<<<nblk(m, 256), 256, 0, s>>>(u, m, k);
  HIGNN_CHECK_LAUNCH();
}

void launch_dp45_error(const float* k, int64_t n, const Dp45Error& de, double* err, cudaStream_t s) {
  HIGNN_CUDA(cudaMemsetAsync(err, 0, sizeof(double), s));
  if (n <= 0) return;
  const unsigned g = nblk(n, 256) < 1184 ? nblk(n, 256) : 1184;
  k_dp45_error<<<g, 256, 0, s>>>(k, n, de, err);
  HIGNN_CHECK_LAUNCH();
}

void launch_pack_positions(const float* xyz, int64_t n, float4* x4, cudaStream_t s) {
  if (n <= 0) return;
  k_pack_positions<<<nblk(n, 256), 256, 0, s>>>(xyz, n, x4);
  HIGNN_CHECK_LAUNCH();
}

}  // namespace hignn
