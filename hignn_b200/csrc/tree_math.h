// Arithmetic of the cluster-tree division shared by the host build (tree.cpp, g++ with
// -ffp-contract=off) and the device build (tree_dev.cu, nvcc with -fmad=false): the same source
// compiled both ways, so that both builds round every operation alike and give the same tree.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define HIGNN_HD __host__ __device__
#else
#define HIGNN_HD
#endif

namespace hignn {

// The mean and covariance sums of a node run in blocks of kSumBlock consecutive particles: each
// block summed sequentially from zero, then the block sums sequentially from zero (the
// reference sums the mean sequentially, src/HignnModel.cpp:130-135; the blocked order lets the
// device form the same values in parallel).
constexpr int64_t kSumBlock = 256;

// Dominant eigenvector of a symmetric 3x3 (cyclic Jacobi, FP64), sign chosen so that its
// largest-magnitude component is positive.
HIGNN_HD inline void jacobi_dominant_axis(const double cov[3][3], double u[3]) {
  double a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a[i][j] = cov[i][j];
  const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-36 * diag || off == 0.0) break;
    for (int r = 0; r < 3; r++) {
      const int p = P[r], q = Q[r];
      double apq = a[p][q];
      if (apq == 0.0) continue;
      double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      double t = 1.0 / (fabs(theta) + sqrt(theta * theta + 1.0));
      if (theta < 0.0) t = -t;
      double c = 1.0 / sqrt(t * t + 1.0);
      double s = t * c;
      for (int k = 0; k < 3; k++) {
        double akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - s * akq;
        a[k][q] = s * akp + c * akq;
      }
      for (int k = 0; k < 3; k++) {
        double apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - s * aqk;
        a[q][k] = s * apk + c * aqk;
      }
      for (int k = 0; k < 3; k++) {
        double vkp = v[k][p], vkq = v[k][q];
        v[k][p] = c * vkp - s * vkq;
        v[k][q] = s * vkp + c * vkq;
      }
    }
  }
  int best = 0;
  for (int k = 1; k < 3; k++)
    if (a[k][k] > a[best][best]) best = k;
  for (int k = 0; k < 3; k++) u[k] = v[k][best];
  int big = 0;
  for (int k = 1; k < 3; k++)
    if (fabs(u[k]) > fabs(u[big])) big = k;
  if (u[big] < 0.0)
    for (int k = 0; k < 3; k++) u[k] = -u[k];
}

// Order-preserving unsigned image of a finite float; -0.0 and +0.0 share one image, as they
// compare equal under operator<.
HIGNN_HD inline uint32_t float_key(float f) {
  uint32_t u;
  if (f == 0.0f) f = 0.0f;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(f);
#else
  std::memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Projection of a centred position on the (float) axis: three roundings, in this order
// (src/HignnModel.cpp:155-160 accumulates temp[i] += U(d, 0) * vertexHat(d, i) from zero).
HIGNN_HD inline float project_axis(float u0, float u1, float u2, float q0, float q1, float q2) {
  float t = u0 * q0;
  t = t + u1 * q1;
  t = t + u2 * q2;
  return t;
}

}  // namespace hignn
