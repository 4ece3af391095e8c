// format.cu -- device-side input conversion, output formatting and synthetic
// input.
//
// Output orders (xgpu.h:45-47) are produced on the device from the triangular
// integration buffer, so a dump copies exactly the requested layout to the
// host.  The index maps follow the reference's writers and reorderers:
//   TRIANGULAR_ORDER            kernel.cuh:96-117, cpu_util.c:161-162
//   REAL_IMAG_TRIANGULAR_ORDER  kernel.cuh:72-95,  cpu_util.c:112-115
//   REGISTER_TILE_...           kernel.cuh:49-71,  cpu_util.c:66-79
#include <math.h>

#include "internal.h"
#include "packed4.cuh"

namespace xgpu {

namespace fmt {

struct Params {
  const void *state;
  int state_is_float;
  int n, f;
  long long nbaseline, mat_length;
  int order, out_type;
  uint32_t *out;  // matLength Complex = 2*matLength 32-bit words
  long long u0, u1;   // the (channel, baseline, product) range formatted
};

__device__ __forceinline__ uint32_t convert(const void *state, int is_float, long long idx,
                                            int out_type) {
  if (is_float) {
    const float v = ((const float *)state)[idx];
    if (out_type == XGPU_INT32) return (uint32_t)__float2int_rn(v);
    return __float_as_uint(v);
  }
  const long long v = ((const long long *)state)[idx];
  if (out_type == XGPU_INT32) return (uint32_t)(unsigned long long)v;  // wraps like int32 sums
  return __float_as_uint(__ll2float_rn(v));
}

// One thread per (channel, baseline, polarisation product).
__global__ void format_kernel(const Params p) {
  for (long long u = p.u0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; u < p.u1;
       u += (long long)gridDim.x * blockDim.x) {
    const int pp = (int)(u & 3);
    const long long fk = u >> 2;
    const int f = (int)(fk / p.nbaseline);
    const long long k = fk - (long long)f * p.nbaseline;
    const uint32_t re = convert(p.state, p.state_is_float, 2 * u, p.out_type);
    const uint32_t im = convert(p.state, p.state_is_float, 2 * u + 1, p.out_type);
    if (p.order == TRIANGULAR_ORDER) {
      *(uint2 *)(p.out + 2 * u) = make_uint2(re, im);
    } else if (p.order == REAL_IMAG_TRIANGULAR_ORDER) {
      p.out[u] = re;
      p.out[u + p.mat_length] = im;
    } else {
      int i = (int)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
      while ((long long)i * (i + 1) / 2 > k) --i;
      while ((long long)(i + 1) * (i + 2) / 2 <= k) ++i;
      const int j = (int)(k - (long long)i * (i + 1) / 2);
      const long long rtn = (long long)(p.n / 2 + 1) * (p.n / 4);
      const int I = i >> 1, J = j >> 1, rx = i & 1, ry = j & 1;
      const long long l =
          (long long)f * 4 * rtn + (long long)(2 * ry + rx) * rtn + (long long)I * (I + 1) / 2 + J;
      const long long w = l * 4 + pp;
      p.out[w] = re;
      p.out[w + p.mat_length] = im;
    }
  }
}

// 16 packed samples per thread: one 16-byte load, two 16-byte stores.
__global__ void unpack4_kernel(const uint4 *in, uint4 *out, long long nquads) {
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nquads;
       u += (long long)gridDim.x * blockDim.x) {
    const uint4 w = in[u];
    const uint2 a = expand_packed4(w.x), b = expand_packed4(w.y), c = expand_packed4(w.z),
                d = expand_packed4(w.w);
    out[2 * u] = make_uint4(a.x, a.y, b.x, b.y);
    out[2 * u + 1] = make_uint4(c.x, c.y, d.x, d.y);
  }
}

// xgpuSwizzleInput's layout (cpu_util.c:235-255) back to [t][f][s][p][c]:
// byte e of row-group tq holds samples 4tq..4tq+3 of input byte e.  One thread
// takes 16 bytes (input bytes 4e4..4e4+3, four samples each), transposes them
// 4x4 with byte permutes, and writes one 4-byte word to each of the four
// sample rows (consecutive threads write consecutive words of a row).
__global__ void unswizzle_kernel(const uint4 *in, uint32_t *out, long long quads,
                                 long long row_words) {
  // quads = (t/4) * row_words; row_words = f*n (4 bytes per station)
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < quads;
       u += (long long)gridDim.x * blockDim.x) {
    const long long tq = u / row_words, e4 = u - tq * row_words;
    const uint4 w = in[u];
    const uint32_t lo01 = __byte_perm(w.x, w.y, 0x5140), hi01 = __byte_perm(w.x, w.y, 0x7362);
    const uint32_t lo23 = __byte_perm(w.z, w.w, 0x5140), hi23 = __byte_perm(w.z, w.w, 0x7362);
    uint32_t *o = out + 4 * tq * row_words + e4;
    o[0] = __byte_perm(lo01, lo23, 0x5410);
    o[row_words] = __byte_perm(lo01, lo23, 0x7632);
    o[2 * row_words] = __byte_perm(hi01, hi23, 0x5410);
    o[3 * row_words] = __byte_perm(hi01, hi23, 0x7632);
  }
}

// xGPU's COMPLEX_BLOCK_SIZE=32 input (read by omp_xengine.c:61-78,
// shared_transfer_4.cuh:69-86) -> [t][f][s][p]{re,im}.  A 64-byte block holds
// 16 consecutive (t,f,s) stations: {X.re,Y.re} pairs in bytes 0-31, {X.im,Y.im}
// pairs in bytes 32-63.  One thread turns 4 stations (8 + 8 bytes) into 16.
__global__ void unblock32_kernel(const uint2 *in, uint4 *out, long long quads) {
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < quads;
       u += (long long)gridDim.x * blockDim.x) {
    const long long blk = u >> 2;
    const int q = (int)(u & 3);
    const uint2 re = in[blk * 8 + q];      // bytes 8q .. 8q+7 of the block
    const uint2 im = in[blk * 8 + 4 + q];  // bytes 32+8q ..
    uint4 o;
    o.x = __byte_perm(re.x, im.x, 0x5140);
    o.y = __byte_perm(re.x, im.x, 0x7362);
    o.z = __byte_perm(re.y, im.y, 0x5140);
    o.w = __byte_perm(re.y, im.y, 0x7362);
    out[u] = o;
  }
}

// Seeded synthetic bytes; the same hash and tables as the host generator.
struct GenParams {
  uint32_t thr[254];
  int kind;
  unsigned long long seed;
};

__device__ __forceinline__ uint32_t hash32(unsigned long long seed, unsigned long long n) {
  unsigned long long z = seed * 0x9E3779B97F4A7C15ull + n + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (uint32_t)(z >> 32);
}

__device__ __forceinline__ int8_t gen_byte(const GenParams &g, const uint32_t *thr,
                                           unsigned long long n) {
  const uint32_t u = hash32(g.seed, n);
  if (g.kind == 0) {
    int lo = 0, hi = 254;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (u < thr[mid]) hi = mid; else lo = mid + 1;
    }
    return (int8_t)(lo - 127);
  } else if (g.kind == 1) {
    const uint32_t v = hash32(g.seed ^ 0x5A5A5A5A5A5A5A5Aull, n);
    const int re = (int)(((unsigned long long)u * 15u) >> 32) - 7;
    const int im = (int)(((unsigned long long)v * 15u) >> 32) - 7;
    return (int8_t)(((re & 0xF) << 4) | (im & 0xF));
  }
  return (int8_t)((int)(((unsigned long long)u * 15u) >> 32) - 7);
}

__global__ void generate_kernel(int8_t *out, unsigned long long nbytes, const GenParams g) {
  __shared__ uint32_t thr[254];
  for (int q = threadIdx.x; q < 254; q += blockDim.x) thr[q] = g.thr[q];
  __syncthreads();
  const unsigned long long nwords = nbytes / 4;
  for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
       w < nwords; w += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t v = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) v |= (uint32_t)(uint8_t)gen_byte(g, thr, 4 * w + b) << (8 * b);
    ((uint32_t *)out)[w] = v;
  }
  if (blockIdx.x == 0)
    for (unsigned long long n = nwords * 4 + threadIdx.x; n < nbytes; n += blockDim.x)
      out[n] = gen_byte(g, thr, n);
}

static unsigned grid_for(long long work, int threads) {
  long long b = (work + threads - 1) / threads;
  if (b > 148LL * 16) b = 148LL * 16;
  if (b < 1) b = 1;
  return (unsigned)b;
}

}  // namespace fmt

cudaError_t launch_format(const void *state, int state_is_float, const Sizes &s, int order,
                          int out_type, void *out, cudaStream_t st, int f0, int fcount) {
  if (fcount < 0) fcount = s.f - f0;
  if (f0 < 0 || fcount < 1 || f0 + fcount > s.f) return cudaErrorInvalidValue;
  if (order == REGISTER_TILE_TRIANGULAR_ORDER) {
    // Slots that hold no baseline (kernel.cuh:65-71) stay zero: clear the
    // channel range's words in both planes.
    const long long per = s.mat_length / s.f;   // 32-bit words per channel and plane
    for (int plane = 0; plane < 2; ++plane) {
      cudaError_t e = cudaMemsetAsync((uint32_t *)out + plane * s.mat_length + f0 * per, 0,
                                      (size_t)(fcount * per) * 4, st);
      if (e != cudaSuccess) return e;
    }
  }
  const long long per_ch = s.nbaseline * 4;
  fmt::Params p{state, state_is_float, s.n, s.f, s.nbaseline, s.mat_length, order, out_type,
                (uint32_t *)out, f0 * per_ch, (f0 + fcount) * per_ch};
  const long long work = fcount * per_ch;
  fmt::format_kernel<<<fmt::grid_for(work, 256), 256, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_unpack4(const uint8_t *in, int8_t *out, long long nsamples, cudaStream_t st) {
  const long long nquads = nsamples / 16;  // nsamples = 2*n*f*t, a multiple of 32 (n % 16 == 0)
  fmt::unpack4_kernel<<<fmt::grid_for(nquads, 256), 256, 0, st>>>((const uint4 *)in,
                                                                  (uint4 *)out, nquads);
  return cudaGetLastError();
}

cudaError_t launch_unswizzle_dp4a(const int8_t *in, int8_t *out, const Sizes &s,
                                  cudaStream_t st) {
  const long long row_words = (long long)s.f * s.n;   // t is a multiple of 4 (ntimepipe % 16 == 0)
  const long long quads = (long long)(s.t / 4) * row_words;
  fmt::unswizzle_kernel<<<fmt::grid_for(quads, 256), 256, 0, st>>>((const uint4 *)in,
                                                                   (uint32_t *)out, quads, row_words);
  return cudaGetLastError();
}

cudaError_t launch_unblock32(const int8_t *in, int8_t *out, long long nbytes, cudaStream_t st) {
  const long long quads = nbytes / 16;
  fmt::unblock32_kernel<<<fmt::grid_for(quads, 256), 256, 0, st>>>((const uint2 *)in,
                                                                   (uint4 *)out, quads);
  return cudaGetLastError();
}

void gauss_thresholds(double sigma, uint32_t thr[254]) {
  for (int k = -127; k < 127; k++) {
    double pr = 0.5 * erfc(-((k + 0.5) / sigma) / sqrt(2.0));
    double sc = floor(pr * 4294967296.0);
    if (sc > 4294967295.0) sc = 4294967295.0;
    if (sc < 0) sc = 0;
    thr[k + 127] = (uint32_t)sc;
  }
}

cudaError_t launch_generate(void *out, size_t nbytes, int kind, unsigned long long seed,
                            double sigma, cudaStream_t st) {
  fmt::GenParams g;
  g.kind = kind;
  g.seed = seed;
  if (kind == 0) gauss_thresholds(sigma, g.thr);
  else for (int q = 0; q < 254; ++q) g.thr[q] = 0;
  fmt::generate_kernel<<<fmt::grid_for((long long)(nbytes / 4) + 1, 256), 256, 0, st>>>(
      (int8_t *)out, (unsigned long long)nbytes, g);
  return cudaGetLastError();
}

}  // namespace xgpu
