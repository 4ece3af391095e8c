// host_util.cpp -- the host-side helpers of xgpu.h (xGPU's cpu_util.c and
// omp_xengine.c API): test-input generation, reordering, checking, the DP4A
// input swizzle, Hermitian expansion and a host X-engine.  They work on the
// build's default sizes, like xGPU's, and are never called by the device
// path.  Matrix words are 32-bit; whether they hold floats or ints is the
// build's default output type (int with make DP4A=yes, float otherwise),
// matching the Complex type of callers built the same way.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "internal.h"

namespace {

XGPUInfo defaults() {
  XGPUInfo i;
  xgpuInfo(&i);
  return i;
}

bool int_words() {
  XGPUConfig c;
  xgpuDefaultConfig(&c);
  return c.output_type == XGPU_INT32;
}

inline double word_value(const uint32_t *w, long long idx, bool is_int) {
  if (is_int) return (double)(int32_t)w[idx];
  float f;
  memcpy(&f, &w[idx], 4);
  return (double)f;
}

}  // namespace

extern "C" {

// Box-Muller Gaussian, sigma 2.5, rounded, saturated to [-7, 7] and scaled by
// 16 (cpu_util.c:13-55), drawing two rand() values per complex sample.
void xgpuRandomComplex(ComplexInput *random_num, long long unsigned int length) {
  const double sigma = 2.5;
  for (long long unsigned int q = 0; q < length; q++) {
    double u1 = rand() / (double)RAND_MAX;
    double u2 = rand() / (double)RAND_MAX;
    if (u1 == 0.0) u1 = 0.5 / RAND_MAX;
    if (u2 == 0.0) u2 = 0.5 / RAND_MAX;
    const double r = sigma * sqrt(-2.0 * log(u1));
    const double theta = 2 * M_PI * u2;
    double a = round(r * cos(theta));
    double b = round(r * sin(theta));
    a = a > 7.0 ? 7.0 : (a < -7.0 ? -7.0 : a);
    b = b > 7.0 ? 7.0 : (b < -7.0 ? -7.0 : b);
    random_num[q].real = (ReImInput)(((int)a) * 16);
    random_num[q].imag = (ReImInput)(((int)b) * 16);
  }
}

// Default order -> TRIANGULAR_ORDER, in place (cpu_util.c:57-132).  Register
// tile entries are visited in the reference's loop order, so the one slot per
// diagonal 2x2 tile that holds no baseline is written and then overwritten
// exactly as there.
void xgpuReorderMatrix(Complex *matrix) {
  const XGPUInfo in = defaults();
  if (in.matrix_order == TRIANGULAR_ORDER) return;
  const long long n = in.nstation, nf = in.nfrequency, ml = (long long)in.matLength;
  uint32_t *m = (uint32_t *)matrix;
  std::vector<uint32_t> tmp((size_t)ml * 2, 0u);
  if (in.matrix_order == REGISTER_TILE_TRIANGULAR_ORDER) {
    const long long rtn = (n / 2 + 1) * (n / 4);
    for (long long f = 0; f < nf; f++)
      for (long long I = 0; I < n / 2; I++)
        for (int rx = 0; rx < 2; rx++)
          for (long long J = 0; J <= I; J++)
            for (int ry = 0; ry < 2; ry++) {
              const long long a = 2 * I + rx, b = 2 * J + ry;
              const long long k = f * (n + 1) * (n / 2) + a * (a + 1) / 2 + b;
              const long long l = f * 4 * rtn + (2 * ry + rx) * rtn + I * (I + 1) / 2 + J;
              for (int pp = 0; pp < 4; pp++) {
                tmp[2 * (4 * k + pp)] = m[4 * l + pp];
                tmp[2 * (4 * k + pp) + 1] = m[4 * l + pp + ml];
              }
            }
  } else {
    const long long tl = nf * (n + 1) * (n / 2) * 4;
    for (long long q = 0; q < tl; q++) {
      tmp[2 * q] = m[q];
      tmp[2 * q + 1] = m[q + ml];
    }
  }
  memcpy(m, tmp.data(), (size_t)ml * 2 * sizeof(uint32_t));
}

// Relative complex error check with xGPU's tolerances and report
// (cpu_util.c:134-232): 1e-5 for fixed-point input.  When the output is float
// (xGPU's FIXED_POINT build without DP4A) the GPU matrix is rounded to
// integers in place first, as xGPU does (cpu_util.c:164-167): callers see the
// rounded values afterwards.
void xgpuCheckResult(Complex *gpu, Complex *cpu, int verbose, ComplexInput *array_h) {
  const XGPUInfo in = defaults();
  const bool is_int = int_words();
  const double tol = 1e-5;
  printf("Checking result (tolerance == %g)...\n", tol);
  fflush(stdout);
  uint32_t *g = (uint32_t *)gpu;
  const uint32_t *c = (const uint32_t *)cpu;
  const long long n = in.nstation, nf = in.nfrequency;
  long long errors = 0;
  double max_err = 0.0;
  for (long long i = 0; i < n; i++)
    for (long long j = 0; j <= i; j++)
      for (int p1 = 0; p1 < 2; p1++)
        for (int p2 = 0; p2 < 2; p2++)
          for (long long f = 0; f < nf; f++) {
            const long long k = f * (n + 1) * (n / 2) + i * (i + 1) / 2 + j;
            const long long idx = (k * 2 + p1) * 2 + p2;
            double gr = word_value(g, 2 * idx, is_int), gi = word_value(g, 2 * idx + 1, is_int);
            const double cr = word_value(c, 2 * idx, is_int), ci = word_value(c, 2 * idx + 1, is_int);
            if (!is_int) {
              gr = round(gr);
              gi = round(gi);
              const float fr = (float)gr, fi = (float)gi;
              memcpy(&g[2 * idx], &fr, 4);
              memcpy(&g[2 * idx + 1], &fi, 4);
            }
            const double cabs = sqrt(cr * cr + ci * ci);
            const double dr = cr - gr, di = ci - gi;
            const double err = cabs == 0 ? sqrt(gr * gr + gi * gi) : sqrt(dr * dr + di * di) / cabs;
            if (err > max_err) max_err = err;
            if (err > tol) {
              if (verbose > 0) {
                if (errors == 0)
                  printf("freq  i   j    k px py  linear   cpu.real      gpu.real     cpu.imag      gpu.imag\n");
                printf("%3lld %3lld %3lld %4lld %2d %2d %5lld %12g  %12g  %12g  %12g\n", f, i, j, k, p1,
                       p2, idx, cr, gr, ci, gi);
                if (verbose > 1 && array_h) {
                  long long sr = 0, si = 0;
                  for (long long t = 0; t < (long long)in.ntime; t++) {
                    const ComplexInput a = array_h[((t * nf + f) * n + i) * 2 + p1];
                    const ComplexInput b = array_h[((t * nf + f) * n + j) * 2 + p2];
                    const int pr = a.real * b.real + a.imag * b.imag;
                    const int pi = a.imag * b.real - a.real * b.imag;
                    sr += pr;
                    si += pi;
                    printf(" %4lld (%4d,%4d) (%4d,%4d) -> (%6d, %6d)\n", t, a.real, a.imag, b.real,
                           b.imag, pr, pi);
                  }
                  // the per-sample products' sum, as xGPU prints it
                  printf("                                 (%6lld, %6lld)\n", sr, si);
                }
              }
              errors++;
            }
          }
  if (errors)
    printf("Outer product summation failed with %lld deviations (max error %g)\n\n", errors, max_err);
  else
    printf("Outer product summation successful (max error %g)\n\n", max_err);
}

// [t][f][s][p][c] -> [t/4][f][s][p][c][t%4] (cpu_util.c:235-255).
void xgpuSwizzleInput(ComplexInput *out, const ComplexInput *in_) {
  const XGPUInfo in = defaults();
  const long long nt = in.ntime, nf = in.nfrequency, n = in.nstation;
  int8_t *o = (int8_t *)out;
  const int8_t *x = (const int8_t *)in_;
  for (long long t = 0; t < nt; t++)
    for (long long f = 0; f < nf; f++)
      for (long long s = 0; s < n; s++)
        for (int p = 0; p < 2; p++)
          for (int c = 0; c < 2; c++)
            o[((((t / 4) * nf + f) * n + s) * 2 + p) * 8 + c * 4 + t % 4] =
                x[(((t * nf + f) * n + s) * 2 + p) * 2 + c];
}

// Triangular -> full Hermitian matrix [f][i][j][p1][p2] (cpu_util.c:258-279).
void xgpuExtractMatrix(Complex *matrix, Complex *packed) {
  const XGPUInfo in = defaults();
  const bool is_int = int_words();
  const long long n = in.nstation, nf = in.nfrequency, nb = (long long)in.nbaseline;
  uint32_t *full = (uint32_t *)matrix;
  const uint32_t *pk = (const uint32_t *)packed;
  for (long long f = 0; f < nf; f++)
    for (long long i = 0; i < n; i++)
      for (long long j = 0; j <= i; j++)
        for (int p1 = 0; p1 < 2; p1++)
          for (int p2 = 0; p2 < 2; p2++) {
            const long long ix = ((f * nb + i * (i + 1) / 2 + j) * 2 + p1) * 2 + p2;
            const long long a = (((f * n + i) * n + j) * 2 + p1) * 2 + p2;
            const long long b = (((f * n + j) * n + i) * 2 + p2) * 2 + p1;
            const uint32_t re = pk[2 * ix], im = pk[2 * ix + 1];
            uint32_t neg;
            if (is_int) {
              neg = (uint32_t)(-(int32_t)im);
            } else {
              float v;
              memcpy(&v, &im, 4);
              v = -v;
              memcpy(&neg, &v, 4);
            }
            full[2 * a] = re;
            full[2 * a + 1] = im;
            full[2 * b] = re;
            full[2 * b + 1] = neg;
          }
}

// Host X-engine in triangular order (omp_xengine.c:36-93) with exact int64
// sums, one OpenMP task per (channel, baseline).
void xgpuOmpXengine(Complex *matrix_h, ComplexInput *array_h) {
  const XGPUInfo in = defaults();
  const bool is_int = int_words();
  const long long n = in.nstation, nf = in.nfrequency, nt = in.ntime, nb = (long long)in.nbaseline;
  const int8_t *x = (const int8_t *)array_h;
  uint32_t *out = (uint32_t *)matrix_h;
#pragma omp parallel for schedule(dynamic, 64)
  for (long long idx = 0; idx < nf * nb; idx++) {
    const long long f = idx / nb, k = idx - f * nb;
    long long i = (long long)(-0.5 + sqrt(0.25 + 2.0 * (double)k));
    while (i * (i + 1) / 2 > k) i--;
    while ((i + 1) * (i + 2) / 2 <= k) i++;
    const long long j = k - i * (i + 1) / 2;
    long long acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long long t = 0; t < nt; t++) {
      const int8_t *r = x + ((t * nf + f) * n + i) * 4;
      const int8_t *c = x + ((t * nf + f) * n + j) * 4;
      for (int p1 = 0; p1 < 2; p1++)
        for (int p2 = 0; p2 < 2; p2++) {
          acc[(p1 * 2 + p2) * 2] += r[2 * p1] * c[2 * p2] + r[2 * p1 + 1] * c[2 * p2 + 1];
          acc[(p1 * 2 + p2) * 2 + 1] += r[2 * p1 + 1] * c[2 * p2] - r[2 * p1] * c[2 * p2 + 1];
        }
    }
    for (int q = 0; q < 8; q++) {
      if (is_int) {
        out[idx * 8 + q] = (uint32_t)(int32_t)acc[q];
      } else {
        const float v = (float)acc[q];
        memcpy(&out[idx * 8 + q], &v, 4);
      }
    }
  }
}

}  // extern "C"
