/*
 * xgpu_oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * A plain-C restatement of the reference's CPU path (xGPU src/omp_xengine.c
 * and src/cpu_util.c) with runtime sizes, used only by tests/, the smoke
 * check and bench.py's CPU baseline to check and time the CUDA library.
 * Nothing in libxgpu.so links or calls this file.
 *
 * Differences from the reference, on purpose:
 *  - sizes are arguments instead of compile-time macros;
 *  - oracle_xengine_i64 sums in int64, so it stays exact where the
 *    reference's float sums (omp_xengine.c:24-28) round above 2^24;
 *    oracle_xengine_f32 keeps the reference's float arithmetic, term for
 *    term, for the FP32 comparisons.
 *
 * Layouts (N stations, F channels, T samples, 2 polarisations):
 *   input    [t][f][s][p][c]                 int8, c = re, im
 *   tri      [f][k][p1][p2][c], k = i(i+1)/2 + j, i >= j   (TRIANGULAR_ORDER)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NPOL 2

/* k -> (i, j) with i >= j, the baseline decode of omp_xengine.c:48-49,
 * corrected with integer checks so it stays right for large k. */
static void tri_decode(long k, int *i, int *j) {
  long r = (long)(-0.5 + sqrt(0.25 + 2.0 * (double)k));
  while (r * (r + 1) / 2 > k) r--;
  while ((r + 1) * (r + 2) / 2 <= k) r++;
  *i = (int)r;
  *j = (int)(k - r * (r + 1) / 2);
}

/* Exact X-engine: out[f][k][p1][p2][re,im] += sum_t x_i,p1 * conj(x_j,p2)
 * (omp_xengine.c:41-92 with int64 accumulators).  accumulate=0 overwrites. */
void oracle_xengine_i64(const int8_t *in, int N, int F, int T, int64_t *out, int accumulate) {
  const long NB = (long)N * (N + 1) / 2;
  const long total = (long)F * NB;
#pragma omp parallel for schedule(dynamic, 64)
  for (long idx = 0; idx < total; idx++) {
    int f = (int)(idx / NB);
    long k = idx - (long)f * NB;
    int i, j;
    tri_decode(k, &i, &j);
    int64_t acc[NPOL][NPOL][2];
    memset(acc, 0, sizeof(acc));
    for (int t = 0; t < T; t++) {
      const int8_t *row = in + (((size_t)t * F + f) * N + i) * NPOL * 2;
      const int8_t *col = in + (((size_t)t * F + f) * N + j) * NPOL * 2;
      for (int p1 = 0; p1 < NPOL; p1++) {
        int ar = row[2 * p1], ai = row[2 * p1 + 1];
        for (int p2 = 0; p2 < NPOL; p2++) {
          int br = col[2 * p2], bi = col[2 * p2 + 1];
          acc[p1][p2][0] += (int64_t)(ar * br + ai * bi);
          acc[p1][p2][1] += (int64_t)(ai * br - ar * bi);
        }
      }
    }
    int64_t *o = out + idx * NPOL * NPOL * 2;
    for (int q = 0; q < NPOL * NPOL * 2; q++) {
      int64_t v = ((int64_t *)acc)[q];
      o[q] = accumulate ? o[q] + v : v;
    }
  }
}

/* The reference's float engine, term for term: each product is formed from
 * float-converted samples and added to a float accumulator in time order
 * (omp_xengine.c:24-28, 55-84).  Output is triangular float re/im pairs. */
void oracle_xengine_f32(const int8_t *in, int N, int F, int T, float *out) {
  const long NB = (long)N * (N + 1) / 2;
  const long total = (long)F * NB;
#pragma omp parallel for schedule(dynamic, 64)
  for (long idx = 0; idx < total; idx++) {
    int f = (int)(idx / NB);
    long k = idx - (long)f * NB;
    int i, j;
    tri_decode(k, &i, &j);
    float acc[NPOL][NPOL][2];
    memset(acc, 0, sizeof(acc));
    for (int t = 0; t < T; t++) {
      const int8_t *row = in + (((size_t)t * F + f) * N + i) * NPOL * 2;
      const int8_t *col = in + (((size_t)t * F + f) * N + j) * NPOL * 2;
      for (int p1 = 0; p1 < NPOL; p1++) {
        float ar = row[2 * p1], ai = row[2 * p1 + 1];
        for (int p2 = 0; p2 < NPOL; p2++) {
          float br = col[2 * p2], bi = col[2 * p2 + 1];
          acc[p1][p2][0] += ar * br + ai * bi;
          acc[p1][p2][1] += ai * br - ar * bi;
        }
      }
    }
    memcpy(out + idx * NPOL * NPOL * 2, acc, sizeof(acc));
  }
}

/* Register-tile (REGISTER_TILE_TRIANGULAR_ORDER) word index of the real part
 * of (f, i, j, p1, p2); the imaginary part sits matLength words later.  This
 * is the inverse of the map in cpu_util.c:66-79 (kernel.cuh:49-71). */
static long regtile_word(int N, int f, int i, int j, int p1, int p2) {
  long rtn = (long)(N / 2 + 1) * (N / 4);
  int I = i / 2, J = j / 2, rx = i % 2, ry = j % 2;
  long l = (long)f * 4 * rtn + (long)(2 * ry + rx) * rtn + (long)I * (I + 1) / 2 + J;
  return (l * NPOL + p1) * NPOL + p2;
}

long oracle_mat_length(int N, int F, int order) {
  if (order == 3000) return (long)F * (N / 2 + 1) * (N / 4) * NPOL * NPOL * 4;
  return (long)F * N * (N + 1) / 2 * NPOL * NPOL;
}

/* Triangular re/im 32-bit words -> the given matrix order (words of the same
 * type).  Slots of the register-tile order that hold no baseline (the upper
 * corner of diagonal 2x2 tiles, kernel.cuh:65-71) are left zero. */
void oracle_tri_to_order(const uint32_t *tri, int N, int F, int order, uint32_t *out) {
  const long NB = (long)N * (N + 1) / 2;
  const long ml = oracle_mat_length(N, F, order);
  memset(out, 0, (size_t)ml * 2 * sizeof(uint32_t));
  for (int f = 0; f < F; f++)
    for (int i = 0; i < N; i++)
      for (int j = 0; j <= i; j++)
        for (int p1 = 0; p1 < NPOL; p1++)
          for (int p2 = 0; p2 < NPOL; p2++) {
            long t = (((long)f * NB + (long)i * (i + 1) / 2 + j) * NPOL + p1) * NPOL + p2;
            uint32_t re = tri[2 * t], im = tri[2 * t + 1];
            if (order == 1000) {
              out[2 * t] = re; out[2 * t + 1] = im;
            } else if (order == 2000) {
              out[t] = re; out[t + ml] = im;
            } else {
              long w = regtile_word(N, f, i, j, p1, p2);
              out[w] = re; out[w + ml] = im;
            }
          }
}

/* In-place reorder to triangular order, following cpu_util.c:57-132 loop for
 * loop (including the register-tile diagonal slot that is written first and
 * overwritten later, cpu_util.c:67-93). */
void oracle_reorder_matrix(uint32_t *matrix, int N, int F, int order) {
  if (order == 1000) return;
  const long ml = oracle_mat_length(N, F, order);
  uint32_t *tmp = (uint32_t *)calloc((size_t)ml * 2, sizeof(uint32_t));
  if (order == 3000) {
    long rtn = (long)(N / 2 + 1) * (N / 4);
    for (int f = 0; f < F; f++)
      for (int i = 0; i < N / 2; i++)
        for (int rx = 0; rx < 2; rx++)
          for (int j = 0; j <= i; j++)
            for (int ry = 0; ry < 2; ry++) {
              long k = (long)f * (N + 1) * (N / 2) + (long)(2 * i + rx) * (2 * i + rx + 1) / 2 + 2 * j + ry;
              long l = (long)f * 4 * rtn + (long)(2 * ry + rx) * rtn + (long)i * (i + 1) / 2 + j;
              for (int p1 = 0; p1 < NPOL; p1++)
                for (int p2 = 0; p2 < NPOL; p2++) {
                  long ti = (k * NPOL + p1) * NPOL + p2;
                  long ri = (l * NPOL + p1) * NPOL + p2;
                  tmp[2 * ti] = matrix[ri];
                  tmp[2 * ti + 1] = matrix[ri + ml];
                }
            }
  } else {
    for (int f = 0; f < F; f++)
      for (int i = 0; i < N; i++)
        for (int j = 0; j <= i; j++) {
          long k = (long)f * (N + 1) * (N / 2) + (long)i * (i + 1) / 2 + j;
          for (int p1 = 0; p1 < NPOL; p1++)
            for (int p2 = 0; p2 < NPOL; p2++) {
              long ix = (k * NPOL + p1) * NPOL + p2;
              tmp[2 * ix] = matrix[ix];
              tmp[2 * ix + 1] = matrix[ix + ml];
            }
        }
  }
  memcpy(matrix, tmp, (size_t)ml * 2 * sizeof(uint32_t));
  free(tmp);
}

/* [t][f][s][p][c] -> [t/4][f][s][p][c][t%4] (cpu_util.c:235-255). */
void oracle_swizzle_input(const int8_t *in, int N, int F, int T, int8_t *out) {
  for (int t = 0; t < T; t++)
    for (int f = 0; f < F; f++)
      for (int s = 0; s < N; s++)
        for (int p = 0; p < NPOL; p++)
          for (int c = 0; c < 2; c++)
            out[((((size_t)(t / 4) * F + f) * N + s) * NPOL + p) * 2 * 4 + c * 4 + t % 4] =
                in[((((size_t)t * F + f) * N + s) * NPOL + p) * 2 + c];
}

/* [t][f][s][p]{re,im} -> xGPU's COMPLEX_BLOCK_SIZE=32 layout, the inverse of
 * the reader in omp_xengine.c:61-78.  The flat (t,f,s) station index g falls
 * in 64-byte block g/16 at slot k = g%16: bytes 2k, 2k+1 hold the real parts
 * of polarisations X, Y and bytes 32+2k, 33+2k their imaginary parts.
 * nbytes = 4*T*F*N, a multiple of 64. */
void oracle_block32_input(const int8_t *in, size_t nbytes, int8_t *out) {
  for (size_t g = 0; g < nbytes / 4; g++) {
    int8_t *b = out + 64 * (g / 16) + 2 * (g % 16);
    b[0] = in[4 * g + 0];
    b[1] = in[4 * g + 2];
    b[32] = in[4 * g + 1];
    b[33] = in[4 * g + 3];
  }
}

/* Triangular -> full Hermitian [f][i][j][p1][p2] for float re/im pairs
 * (cpu_util.c:258-279). */
void oracle_extract_matrix_f32(const float *packed, int N, int F, float *full) {
  const long NB = (long)N * (N + 1) / 2;
  for (int f = 0; f < F; f++)
    for (int i = 0; i < N; i++)
      for (int j = 0; j <= i; j++)
        for (int p1 = 0; p1 < NPOL; p1++)
          for (int p2 = 0; p2 < NPOL; p2++) {
            long ix = (((long)f * NB + (long)i * (i + 1) / 2 + j) * NPOL + p1) * NPOL + p2;
            long a = ((((long)f * N + i) * N + j) * NPOL + p1) * NPOL + p2;
            long b = ((((long)f * N + j) * N + i) * NPOL + p2) * NPOL + p1;
            full[2 * a] = packed[2 * ix];
            full[2 * a + 1] = packed[2 * ix + 1];
            full[2 * b] = packed[2 * ix];
            full[2 * b + 1] = -packed[2 * ix + 1];
          }
}

/* ---- seeded synthetic input (not in the reference; its own generator is
 * rand()-based, cpu_util.c:13-55) ------------------------------------------
 * Counter based: byte n of a buffer depends only on (seed, n).  A splitmix64
 * finaliser gives a 32-bit uniform u; a Gaussian byte is the smallest k in
 * [-127,127] with u < thr[k], where thr[k] = floor(2^32 * Phi((k+0.5)/sigma))
 * is the CDF of round(N(0, sigma^2)) clipped to [-127,127]. */
static uint32_t hash32(uint64_t seed, uint64_t n) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ull + n + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (uint32_t)(z >> 32);
}

void oracle_gauss_thresholds(double sigma, uint32_t *thr /* 254 entries */) {
  for (int k = -127; k < 127; k++) {
    double p = 0.5 * erfc(-((k + 0.5) / sigma) / sqrt(2.0));
    double s = floor(p * 4294967296.0);
    if (s > 4294967295.0) s = 4294967295.0;
    if (s < 0) s = 0;
    thr[k + 127] = (uint32_t)s;
  }
}

/* Bytes [offset, offset + nbytes) of the stream (kind, seed, sigma). */
void oracle_generate_range(int8_t *out, size_t nbytes, int kind, uint64_t seed, double sigma,
                           uint64_t offset) {
  uint32_t thr[254];
  if (kind == 0) oracle_gauss_thresholds(sigma, thr);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < (long)nbytes; q++) {
    const uint64_t n = offset + (uint64_t)q;
    int8_t *o = out + q;
    uint32_t u = hash32(seed, n);
    if (kind == 0) {
      int lo = 0, hi = 254; /* first index with u < thr[idx], 254 if none */
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (u < thr[mid]) hi = mid; else lo = mid + 1;
      }
      *o = (int8_t)(lo - 127);
    } else if (kind == 1) {
      uint32_t v = hash32(seed ^ 0x5A5A5A5A5A5A5A5Aull, n);
      int re = (int)(((uint64_t)u * 15u) >> 32) - 7;
      int im = (int)(((uint64_t)v * 15u) >> 32) - 7;
      *o = (int8_t)(((re & 0xF) << 4) | (im & 0xF));
    } else {
      *o = (int8_t)((int)(((uint64_t)u * 15u) >> 32) - 7);
    }
  }
}

void oracle_generate(int8_t *out, size_t nbytes, int kind, uint64_t seed, double sigma) {
  oracle_generate_range(out, nbytes, kind, seed, sigma, 0);
}

/* Packed 4+4-bit -> int8 re/im pairs (re = high nibble, im = low nibble). */
void oracle_unpack4(const uint8_t *in, size_t n, int8_t *out) {
  for (size_t q = 0; q < n; q++) {
    int8_t b = (int8_t)in[q];
    out[2 * q] = (int8_t)(b >> 4);
    out[2 * q + 1] = (int8_t)((int8_t)(in[q] << 4) >> 4);
  }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
