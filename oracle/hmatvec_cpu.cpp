// Oracle (test infrastructure and the CPU baseline; never linked into the library): the
// H-matvec of the reference path restated in C++ with OpenMP over the host cores.
//
// It performs what the numpy restatement (hignn_oracle.py: close_dot, aca_blocks, aca_apply)
// performs, block for block, with the FP32 network of twobody_f32.c (the plain device network's
// operations, bit for bit):
//   CloseDot (src/CloseDot.cpp:177-299): for every close leaf pair (I, J), u_I += M(x_J - x_I) f_J
//     and, for J > I under symmetry, u_J += (the same M) f_I; FP64 accumulation.
//   FarDot (src/FarDot.cpp:191-1388): ACA per admissible block on symmetrised 3x3 queries: first
//     column |J|/2; C_k = A(:, j_k) - sum_l C_l Q_l(j_k); row pivot = first maximal signed
//     determinant over unused rows; C_k <- C_k inv(C_k(i_k)) (adjugate / det); Q_k = A(i_k, :) -
//     sum_l C_l(i_k) Q_l; next column = first maximal signed determinant over unused columns;
//     nu2 = ||C_k Q_k||^2, mu2 += nu2 + sum_{l < k-1} 2 |C_k^T C_l| |Q_k Q_l^T|; stop when
//     nu2 < mu2 eps^2, k >= max_iter or k >= min(|I|, |J|); u_I += sum_l C_l (Q_l f_J), and under
//     symmetry u_J += sum_l Q_l^T (C_l^T f_I). Factors stored rounded to FP32, arithmetic in FP64.
// Blocks run in parallel (dynamic schedule); each block's contribution is accumulated locally and
// added to u under a per-particle atomic.
#include <cmath>
#include <cstdint>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" void oracle_twobody_batch(const float* W1, const float* b1, const float* W2, const float* b2,
                                     const float* W3, const float* b3, const float* r, int nb, float* y);

namespace {

constexpr int kBatch = 16;

struct Net {
  const float *W1, *b1, *W2, *b2, *W3, *b3;
  // y (n, 9) = M(r) for n features
  void eval(const float* r, int64_t n, float* y) const {
    for (int64_t s = 0; s < n; s += kBatch) {
      const int nb = (int)(n - s < kBatch ? n - s : kBatch);
      oracle_twobody_batch(W1, b1, W2, b2, W3, b3, r + 3 * s, nb, y + 9 * s);
    }
  }
};

inline void atomic_add(double* p, double v) {
#pragma omp atomic
  *p += v;
}

inline double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

inline double f32(double v) { return (double)(float)v; }

// symmetrised 3x3 of a network output (src/FarDot.cpp:445-456): diagonal copied, off-diagonal
// 0.5 * (FP32 sum) formed in double
inline void symmetrize(const float* y, double* o) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      o[3 * r + c] = (r == c) ? (double)y[3 * r + c] : 0.5 * (double)(float)(y[3 * r + c] + y[3 * c + r]);
}

struct Block {
  int64_t sI, nI, sJ, nJ;
};

// ACA of one block; C (kmax x nI x 9), Q (kmax x nJ x 9) as FP32 values in doubles. Returns the rank.
int aca_block(const Net& net, const float* xt, const Block& b, double eps2, int max_iter, std::vector<double>& C,
              std::vector<double>& Q) {
  const int64_t nI = b.nI, nJ = b.nJ;
  const int kmax = std::max<int64_t>(1, std::min<int64_t>(max_iter, std::min(nI, nJ)));
  C.assign((size_t)kmax * nI * 9, 0.0);
  Q.assign((size_t)kmax * nJ * 9, 0.0);
  std::vector<char> used_row(nI, 0), used_col(nJ, 0);
  std::vector<float> r(3 * std::max(nI, nJ)), y(9 * std::max(nI, nJ));
  std::vector<double> Ck(9 * nI), Qk(9 * nJ);
  int jk = (int)(nJ / 2);
  double mu2 = 0.0;
  int k = 0;
  for (;;) {
    // column query (src/FarDot.cpp:348-458) and orthogonalisation (:474-512)
    const float* xj = xt + 3 * (b.sJ + jk);
    for (int64_t i = 0; i < nI; i++)
      for (int d = 0; d < 3; d++) r[3 * i + d] = xj[d] - xt[3 * (b.sI + i) + d];
    net.eval(r.data(), nI, y.data());
    used_col[jk] = 1;
    for (int64_t i = 0; i < nI; i++) {
      double c[9];
      symmetrize(&y[9 * i], c);
      if (k > 0) {
        double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int l = 0; l < k; l++) {
          const double* cl = &C[((size_t)l * nI + i) * 9];
          const double* ql = &Q[((size_t)l * nJ + jk) * 9];
          for (int rr = 0; rr < 3; rr++)
            for (int cc = 0; cc < 3; cc++)
              for (int m = 0; m < 3; m++) s[3 * rr + cc] += cl[3 * rr + m] * ql[3 * m + cc];
        }
        for (int q = 0; q < 9; q++) c[q] = f32(c[q] - s[q]);
      }
      for (int q = 0; q < 9; q++) Ck[9 * i + q] = c[q];
    }
    // row pivot: first maximal signed determinant over unused rows (:520-576)
    int ik = -1;
    double best = 0.0;
    for (int64_t i = 0; i < nI; i++) {
      if (used_row[i]) continue;
      const double d = det3(&Ck[9 * i]);
      if (ik < 0 || d > best) {
        best = d;
        ik = (int)i;
      }
    }
    if (ik < 0) return -1;
    used_row[ik] = 1;
    {  // C_k <- C_k inv(C_k(i_k)), adjugate / det (:586-656)
      const double* m = &Ck[9 * ik];
      const double A = m[0], B = m[1], Cc = m[2], D = m[3], E = m[4], F = m[5], G = m[6], H = m[7], I = m[8];
      const double det = A * (E * I - F * H) - B * (D * I - F * G) + Cc * (D * H - E * G);
      const double inv[9] = {(E * I - F * H) / det,  -(B * I - Cc * H) / det, (B * F - Cc * E) / det,
                             -(D * I - F * G) / det, (A * I - Cc * G) / det,  -(A * F - Cc * D) / det,
                             (D * H - E * G) / det,  -(A * H - B * G) / det,  (A * E - B * D) / det};
      for (int64_t i = 0; i < nI; i++) {
        const double* c = &Ck[9 * i];
        double* o = &C[((size_t)k * nI + i) * 9];
        for (int rr = 0; rr < 3; rr++)
          for (int cc = 0; cc < 3; cc++) {
            double acc = c[3 * rr] * inv[cc];
            acc = acc + c[3 * rr + 1] * inv[3 + cc];
            acc = acc + c[3 * rr + 2] * inv[6 + cc];
            o[3 * rr + cc] = f32(acc);
          }
      }
    }
    // row query (:672-781) and orthogonalisation (:797-841)
    const float* xi = xt + 3 * (b.sI + ik);
    for (int64_t j = 0; j < nJ; j++)
      for (int d = 0; d < 3; d++) r[3 * j + d] = xt[3 * (b.sJ + j) + d] - xi[d];
    net.eval(r.data(), nJ, y.data());
    for (int64_t j = 0; j < nJ; j++) {
      double q[9];
      symmetrize(&y[9 * j], q);
      if (k > 0) {
        double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int l = 0; l < k; l++) {
          const double* cl = &C[((size_t)l * nI + ik) * 9];
          const double* ql = &Q[((size_t)l * nJ + j) * 9];
          for (int rr = 0; rr < 3; rr++)
            for (int cc = 0; cc < 3; cc++)
              for (int m = 0; m < 3; m++) s[3 * rr + cc] += cl[3 * rr + m] * ql[3 * m + cc];
        }
        for (int e = 0; e < 9; e++) q[e] = f32(q[e] - s[e]);
      }
      for (int e = 0; e < 9; e++) Q[((size_t)k * nJ + j) * 9 + e] = q[e];
    }
    // next column: first maximal signed determinant over columns not yet used (:846-903)
    int jn = -1;
    best = 0.0;
    for (int64_t j = 0; j < nJ; j++) {
      if (used_col[j]) continue;
      const double d = det3(&Q[((size_t)k * nJ + j) * 9]);
      if (jn < 0 || d > best) {
        best = d;
        jn = (int)j;
      }
    }
    // nu2, mu2 (:919-1078)
    const double* Cn = &C[(size_t)k * nI * 9];
    const double* Qn = &Q[(size_t)k * nJ * 9];
    double cn[3] = {0, 0, 0}, cd[3] = {0, 0, 0}, qn[3] = {0, 0, 0}, qd[3] = {0, 0, 0};
    for (int64_t i = 0; i < nI; i++) {
      const double* c = Cn + 9 * i;
      for (int cc = 0; cc < 3; cc++) {
        const int c1 = (cc + 1) % 3;
        cn[cc] += c[cc] * c[cc] + c[cc + 3] * c[cc + 3] + c[cc + 6] * c[cc + 6];
        cd[cc] += c[cc] * c[c1] + c[cc + 3] * c[c1 + 3] + c[cc + 6] * c[c1 + 6];
      }
    }
    for (int64_t j = 0; j < nJ; j++) {
      const double* q = Qn + 9 * j;
      for (int d = 0; d < 3; d++) qn[d] += q[3 * d] * q[3 * d] + q[3 * d + 1] * q[3 * d + 1] + q[3 * d + 2] * q[3 * d + 2];
      qd[0] += q[0] * q[3] + q[1] * q[4] + q[2] * q[5];
      qd[1] += q[3] * q[6] + q[4] * q[7] + q[5] * q[8];
      qd[2] += q[6] * q[0] + q[7] * q[1] + q[8] * q[2];
    }
    const double nu2 = cn[0] * qn[0] + cn[1] * qn[1] + cn[2] * qn[2] + 2.0 * qd[0] * cd[0] + 2.0 * qd[1] * cd[1] +
                       2.0 * qd[2] * cd[2];
    mu2 += nu2;
    for (int l = 0; l + 1 < k; l++) {  // |.| cross terms, l = k - 1 skipped (:1041)
      double xc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, xq[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const double* Cl = &C[(size_t)l * nI * 9];
      const double* Ql = &Q[(size_t)l * nJ * 9];
      for (int64_t i = 0; i < nI; i++) {
        const double *c = Cn + 9 * i, *d = Cl + 9 * i;
        for (int d1 = 0; d1 < 3; d1++)
          for (int d2 = 0; d2 < 3; d2++) xc[3 * d1 + d2] += c[d1] * d[d2] + c[d1 + 3] * d[d2 + 3] + c[d1 + 6] * d[d2 + 6];
      }
      for (int64_t j = 0; j < nJ; j++) {
        const double *q = Qn + 9 * j, *p = Ql + 9 * j;
        for (int d1 = 0; d1 < 3; d1++)
          for (int d2 = 0; d2 < 3; d2++)
            xq[3 * d1 + d2] += q[3 * d1] * p[3 * d2] + q[3 * d1 + 1] * p[3 * d2 + 1] + q[3 * d1 + 2] * p[3 * d2 + 2];
      }
      for (int e = 0; e < 9; e++) mu2 += 2.0 * std::fabs(xc[e]) * std::fabs(xq[e]);
    }
    k++;
    if (nu2 < mu2 * eps2 || k >= max_iter || k >= std::min(nI, nJ) || jn < 0) return k;
    jk = jn;
  }
}

}  // namespace

extern "C" {

// CloseDot over close pairs [p0, p1) of the lists (tree order); adds into u (n x 3, FP64).
void oracle_close_dot(const float* W1, const float* b1, const float* W2, const float* b2, const float* W3,
                      const float* b3, const float* xt, const float* ft, const int64_t* nstart, const int64_t* nend,
                      const int64_t* closeI, const int64_t* closeJ, int64_t p0, int64_t p1, int use_symmetry,
                      int nthreads, double* u) {
  const Net net{W1, b1, W2, b2, W3, b3};
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    std::vector<float> r, y;
    std::vector<double> uI, uJ;
#pragma omp for schedule(dynamic, 4)
    for (int64_t p = p0; p < p1; p++) {
      const int64_t I = closeI[p], J = closeJ[p];
      const int64_t sI = nstart[I], nI = nend[I] - sI, sJ = nstart[J], nJ = nend[J] - sJ;
      uI.assign(3 * nI, 0.0);
      const bool tr = use_symmetry && J > I;
      uJ.assign(tr ? 3 * nJ : 0, 0.0);
      // in chunks of kChunk evaluations, so that features and outputs stay in the core's cache
      constexpr int64_t kChunk = 256;
      r.resize(3 * kChunk);
      y.resize(9 * kChunk);
      const int64_t total = nI * nJ;
      for (int64_t c0 = 0; c0 < total; c0 += kChunk) {
        const int64_t cn = total - c0 < kChunk ? total - c0 : kChunk;
        for (int64_t e = 0; e < cn; e++) {
          const int64_t i = (c0 + e) / nJ, j = (c0 + e) - i * nJ;
          for (int d = 0; d < 3; d++) r[3 * e + d] = xt[3 * (sJ + j) + d] - xt[3 * (sI + i) + d];
        }
        net.eval(r.data(), cn, y.data());
        for (int64_t e = 0; e < cn; e++) {
          const int64_t i = (c0 + e) / nJ, j = (c0 + e) - i * nJ;
          const float* m = &y[9 * e];
          const double fj[3] = {ft[3 * (sJ + j)], ft[3 * (sJ + j) + 1], ft[3 * (sJ + j) + 2]};
          for (int rr = 0; rr < 3; rr++)
            uI[3 * i + rr] += (double)m[3 * rr] * fj[0] + (double)m[3 * rr + 1] * fj[1] + (double)m[3 * rr + 2] * fj[2];
          if (tr) {
            const double fi[3] = {ft[3 * (sI + i)], ft[3 * (sI + i) + 1], ft[3 * (sI + i) + 2]};
            for (int rr = 0; rr < 3; rr++)
              uJ[3 * j + rr] +=
                  (double)m[3 * rr] * fi[0] + (double)m[3 * rr + 1] * fi[1] + (double)m[3 * rr + 2] * fi[2];
          }
        }
      }
      for (int64_t q = 0; q < 3 * nI; q++) atomic_add(&u[3 * sI + q], uI[q]);
      if (tr)
        for (int64_t q = 0; q < 3 * nJ; q++) atomic_add(&u[3 * sJ + q], uJ[q]);
    }
  }
}

// FarDot over far pairs [p0, p1) of the lists (tree order); adds into u; ranks[p - p0] = ACA rank
// (or -1 when a pivot search found no unused row). Returns the number of ACA evaluations.
int64_t oracle_far_dot(const float* W1, const float* b1, const float* W2, const float* b2, const float* W3,
                       const float* b3, const float* xt, const float* ft, const int64_t* nstart, const int64_t* nend,
                       const int64_t* farI, const int64_t* farJ, int64_t p0, int64_t p1, double epsilon,
                       int max_iter, int use_symmetry, int nthreads, double* u, int32_t* ranks) {
  const Net net{W1, b1, W2, b2, W3, b3};
  const double eps2 = epsilon * epsilon;
  int64_t evals = 0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : evals)
  {
    std::vector<double> C, Q, mid, mid2, uI, uJ;
#pragma omp for schedule(dynamic, 1)
    for (int64_t p = p0; p < p1; p++) {
      const int64_t I = farI[p], J = farJ[p];
      const Block b{nstart[I], nend[I] - nstart[I], nstart[J], nend[J] - nstart[J]};
      const int k = aca_block(net, xt, b, eps2, max_iter, C, Q);
      if (ranks) ranks[p - p0] = k;
      if (k <= 0) continue;
      evals += (int64_t)k * (b.nI + b.nJ);
      // apply (:1194-1388): mid_l = Q_l f_J, u_I = sum_l C_l mid_l; mid2_l = C_l^T f_I, u_J = sum_l Q_l^T mid2_l
      mid.assign(3 * k, 0.0);
      mid2.assign(3 * k, 0.0);
      for (int l = 0; l < k; l++)
        for (int64_t j = 0; j < b.nJ; j++) {
          const double* q = &Q[((size_t)l * b.nJ + j) * 9];
          const float* f = ft + 3 * (b.sJ + j);
          for (int rr = 0; rr < 3; rr++) mid[3 * l + rr] += q[3 * rr] * f[0] + q[3 * rr + 1] * f[1] + q[3 * rr + 2] * f[2];
        }
      uI.assign(3 * b.nI, 0.0);
      for (int64_t i = 0; i < b.nI; i++)
        for (int l = 0; l < k; l++) {
          const double* c = &C[((size_t)l * b.nI + i) * 9];
          for (int rr = 0; rr < 3; rr++)
            uI[3 * i + rr] += c[3 * rr] * mid[3 * l] + c[3 * rr + 1] * mid[3 * l + 1] + c[3 * rr + 2] * mid[3 * l + 2];
        }
      for (int64_t q = 0; q < 3 * b.nI; q++) atomic_add(&u[3 * b.sI + q], uI[q]);
      if (use_symmetry) {
        for (int l = 0; l < k; l++)
          for (int64_t i = 0; i < b.nI; i++) {
            const double* c = &C[((size_t)l * b.nI + i) * 9];
            const float* f = ft + 3 * (b.sI + i);
            for (int rr = 0; rr < 3; rr++) mid2[3 * l + rr] += c[rr] * f[0] + c[3 + rr] * f[1] + c[6 + rr] * f[2];
          }
        uJ.assign(3 * b.nJ, 0.0);
        for (int64_t j = 0; j < b.nJ; j++)
          for (int l = 0; l < k; l++) {
            const double* q = &Q[((size_t)l * b.nJ + j) * 9];
            for (int rr = 0; rr < 3; rr++)
              uJ[3 * j + rr] += q[rr] * mid2[3 * l] + q[3 + rr] * mid2[3 * l + 1] + q[6 + rr] * mid2[3 * l + 2];
          }
        for (int64_t q = 0; q < 3 * b.nJ; q++) atomic_add(&u[3 * b.sJ + q], uJ[q]);
      }
    }
  }
  return evals;
}

}  // extern "C"
