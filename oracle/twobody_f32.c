/* Oracle (test infrastructure, never linked into the library): the FP32 two-body network of
 * the plain form, restated in C so that it reproduces the device's FP32 outputs bit for bit.
 *
 * The reference evaluates the network with libtorch in FP32 (python/convert.py:11-20, called at
 * src/CloseDot.cpp:233 and src/FarDot.cpp:414,739). Any two FP32 evaluations that round in a
 * different order differ in the last bits, and the ACA pivot search takes the maximum of signed
 * 3x3 determinants of network outputs (src/FarDot.cpp:557-573, 883-893), so near-ties then pick
 * other, equally valid pivots. To compare whole H-matrix products free-running, this restatement
 * performs exactly the operations the plain device network performs, one correctly rounded FP32
 * operation at a time and in the same order:
 *   h1[k] = tanh(fma(W1[k][2], r_z, fma(W1[k][1], r_y, fma(W1[k][0], r_x, b1[k]))))
 *   h2[n] = tanh(acc_n + b2[n]),  acc_n = fma(h1[127], W2[n][127], ... fma(h1[0], W2[n][0], 0))
 *   y[o]  = fma(h2[511], W3[o][511], ... fma(h2[0], W3[o][0], 0)) + b3[o] (+ 1 on the diagonal),
 *           divided by |r| = sqrt(fma(r_z, r_z, fma(r_y, r_y, r_x r_x))); identity for |r| < 1e-5
 * with the tanh below. Compiled with -ffp-contract=off: only the fmaf calls fuse.
 *
 * tanh (the same method and FP32 constants as the device's): for a = |x|,
 *   a < 0.8 : a + a s P(s), s = a^2, P the degree-5 fit of (tanh(a)/a - 1)/s on [0, 0.8];
 *   a < 9.5 : 1 - 2 / (exp(2a) + 1), exp(2a) = 2^k exp(r), k = rint(2a / ln 2), r by Cody-Waite
 *             reduction with ln 2 = 0x1.62e4p-1 + 0x1.7f7d1cp-20, exp(r) by Taylor to degree 7;
 *   a >= 9.5: 1.
 * The branches are computed for every lane and selected, so the loops vectorise; the exp
 * branch runs on min(a, 9.5), which is a itself wherever it is selected.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define H1 128
#define H2 512
#define NOUT 9
#define BATCH 16

static inline float scale2(float kf) {
  const uint32_t bits = (uint32_t)((int32_t)kf + 127) << 23;
  float s;
  memcpy(&s, &bits, 4);
  return s;
}

static inline float own_tanh(float x) {
  const float a = fabsf(x);
  const float s = a * a;
  float p = 0x1.a19af4p-10f;
  p = fmaf(p, s, -0x1.e69e6cp-8f);
  p = fmaf(p, s, 0x1.5d356ep-6f);
  p = fmaf(p, s, -0x1.b92feap-5f);
  p = fmaf(p, s, 0x1.110b7ep-3f);
  p = fmaf(p, s, -0x1.55553ep-2f);
  const float tp = fmaf(a, s * p, a);
  const float ac = a < 9.5f ? a : 9.5f;
  const float y = ac + ac;
  const float kf = rintf(y * 0x1.715476p+0f);
  const float r = fmaf(kf, -0x1.7f7d1cp-20f, fmaf(kf, -0x1.62e4p-1f, y));
  float q = 0x1.a01a02p-13f;
  q = fmaf(q, r, 0x1.6c16c2p-10f);
  q = fmaf(q, r, 0x1.111112p-7f);
  q = fmaf(q, r, 0x1.555556p-5f);
  q = fmaf(q, r, 0x1.555556p-3f);
  q = fmaf(q, r, 0.5f);
  q = fmaf(q, r, 1.0f);
  q = fmaf(q, r, 1.0f);
  const float e = q * scale2(kf);
  const float te = 1.0f - 2.0f / (e + 1.0f);
  const float t = a < 0.8f ? tp : (a < 9.5f ? te : (a == a ? 1.0f : a));
  return copysignf(t, x);
}

/* One batch of up to BATCH features. */
__attribute__((target_clones("arch=x86-64-v4", "arch=x86-64-v3", "default")))
static void eval_batch(const float* W1, const float* b1, const float* W2, const float* b2, const float* W3,
                       const float* b3, const float* r, int nb, float* y) {
  float rx[BATCH], ry[BATCH], rz[BATCH];
  float h1[H1][BATCH];
  float y3[NOUT][BATCH];
  for (int e = 0; e < BATCH; e++) {
    const int s = e < nb ? e : 0;
    rx[e] = r[3 * s];
    ry[e] = r[3 * s + 1];
    rz[e] = r[3 * s + 2];
  }
  for (int k = 0; k < H1; k++) {
    const float w0 = W1[3 * k], w1 = W1[3 * k + 1], w2 = W1[3 * k + 2], bk = b1[k];
    for (int e = 0; e < BATCH; e++) h1[k][e] = own_tanh(fmaf(w2, rz[e], fmaf(w1, ry[e], fmaf(w0, rx[e], bk))));
  }
  for (int o = 0; o < NOUT; o++)
    for (int e = 0; e < BATCH; e++) y3[o][e] = 0.0f;
  /* four hidden units at a time (each accumulation still runs over k in order) */
  for (int n0 = 0; n0 < H2; n0 += 4) {
    float acc[4][BATCH];
    for (int j = 0; j < 4; j++)
      for (int e = 0; e < BATCH; e++) acc[j][e] = 0.0f;
    const float* w0 = W2 + (size_t)n0 * H1;
    for (int k = 0; k < H1; k++) {
      const float a0 = w0[k], a1 = w0[H1 + k], a2 = w0[2 * H1 + k], a3 = w0[3 * H1 + k];
      for (int e = 0; e < BATCH; e++) {
        const float h = h1[k][e];
        acc[0][e] = fmaf(h, a0, acc[0][e]);
        acc[1][e] = fmaf(h, a1, acc[1][e]);
        acc[2][e] = fmaf(h, a2, acc[2][e]);
        acc[3][e] = fmaf(h, a3, acc[3][e]);
      }
    }
    for (int j = 0; j < 4; j++) {
      const int n = n0 + j;
      const float bn = b2[n];
      float h2[BATCH];
      for (int e = 0; e < BATCH; e++) h2[e] = own_tanh(acc[j][e] + bn);
      for (int o = 0; o < NOUT; o++) {
        const float w = W3[(size_t)o * H2 + n];
        for (int e = 0; e < BATCH; e++) y3[o][e] = fmaf(h2[e], w, y3[o][e]);
      }
    }
  }
  for (int e = 0; e < nb; e++) {
    const float nr = sqrtf(fmaf(rz[e], rz[e], fmaf(ry[e], ry[e], rx[e] * rx[e])));
    for (int o = 0; o < NOUT; o++) {
      float v = y3[o][e] + b3[o];
      const int dg = (o == 0 || o == 4 || o == 8);
      if (dg) v = v + 1.0f;
      v = v / nr;
      if (nr < 1e-5f) v = dg ? 1.0f : 0.0f;
      y[9 * e + o] = v;
    }
  }
}

/* y (n, 9) = M(r) for features r (n, 3); W1 (128, 3), W2 (512, 128), W3 (9, 512) row-major. */
void oracle_twobody_eval32(const float* W1, const float* b1, const float* W2, const float* b2, const float* W3,
                           const float* b3, const float* r, int64_t n, float* y, int nthreads) {
  const int64_t nbatch = (n + BATCH - 1) / BATCH;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t q = 0; q < nbatch; q++) {
    const int64_t s = q * BATCH;
    const int nb = (int)(n - s < BATCH ? n - s : BATCH);
    eval_batch(W1, b1, W2, b2, W3, b3, r + 3 * s, nb, y + 9 * s);
  }
}

/* tanh of the plain form for an array (tests of the method against a double tanh). */
void oracle_tanh_f32(const float* x, int64_t n, float* t) {
  for (int64_t i = 0; i < n; i++) t[i] = own_tanh(x[i]);
}

/* One batch of nb <= 16 features (the C++ restatement of the H-matvec evaluates through this). */
void oracle_twobody_batch(const float* W1, const float* b1, const float* W2, const float* b2, const float* W3,
                          const float* b3, const float* r, int nb, float* y) {
  eval_batch(W1, b1, W2, b2, W3, b3, r, nb, y);
}
