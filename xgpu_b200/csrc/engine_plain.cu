// engine_plain.cu -- CUDA-core X-engine: 2x2 register tile, FP32 and dp4a.
//
// The B200 counterpart of xGPU's shared2x2 kernels (kernel.cuh:238-422 FP32,
// kernel.cuh:427-591 dp4a, compute macros shared_transfer_4.cuh:91-156 and
// shared_transfer_4_dp4a.cuh:99-164).  The arithmetic per thread is the same:
// each thread owns a 2x2 block of stations (rows i, i+1 x columns j, j+1) and
// all 4 polarisation products of each, i.e. 16 complex visibilities.
//   FP32: 32 float accumulators, 64 FMAs per sample.
//   dp4a: 48 int32 accumulators (re, im1, im2 as in kernel.cuh:464-479,574),
//         64 dp4a per group of 4 samples.
// What changes is the data path.  xGPU fetches one sample at a time through
// textures and swizzled input; here a CTA of 256 threads covers a 32x32
// station block of one channel, stages 128-byte panels of the natural
// [t][f][s][p][c] input into shared memory with 16-byte cp.async loads
// (double buffered), and converts them in shared memory -- to 4-sample
// words for dp4a (a 4x4 byte transpose with PRMT) or to floats -- in an order
// that makes the 128-bit shared loads of the compute loop conflict-free.
// One launch covers a whole time range (not one NTIME_PIPE chunk), and the
// sums are added to the integration buffer once, at the end.
#include "internal.h"

namespace xgpu {
namespace plain {

constexpr int kBlk = 32;        // stations per block side
constexpr int kThreads = 256;   // 16 x 16 threads, 2x2 stations each
constexpr int kRowBytes = kBlk * 4;   // one sample of one panel: 32 stations x 2 pol x re/im

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void decode_block(int k, int &rb, int &cb) {
  int r = (int)((sqrtf(8.0f * (float)k + 1.0f) - 1.0f) * 0.5f);
  while (r * (r + 1) / 2 > k) --r;
  while ((r + 1) * (r + 2) / 2 <= k) ++r;
  rb = r;
  cb = k - r * (r + 1) / 2;
}

// Slot of station s (0..31) inside a converted panel: thread column tx reads
// stations 2tx and 2tx+1, stored at slots tx and 16+tx so that 16 threads
// read 256 contiguous bytes.
__device__ __forceinline__ int slot_of(int s) { return (s & 1) * 16 + (s >> 1); }

struct Params {
  const int8_t *in;
  int n, f;
  int t0, tcount;
  long long nbaseline;
  void *state;
  int overwrite;
  int per;        // samples per time split (blockIdx.z); == tcount without splits
};

// Issue the cp.async loads of samples [tb, tb+nt) of one panel (32 stations
// from s0) into raw (nt rows of 128 bytes).  Samples past tend and stations
// past n are zero-filled.
template <int NT>
__device__ __forceinline__ void load_panel(uint8_t *raw, const Params &p, int f, int s0, int tb,
                                           int tend) {
  constexpr int kPieces = NT * (kRowBytes / 16);
  for (int q = threadIdx.x; q < kPieces; q += kThreads) {
    const int r = q >> 3, piece = q & 7;
    const int t = tb + r;
    const int s = s0 + piece * 4;   // 16 bytes = 4 stations
    const bool ok = (t < tend) && (s < p.n);
    const int8_t *src =
        ok ? p.in + (((long long)t * p.f + f) * p.n + s) * 4 : p.in;
    cp_async16((uint32_t)__cvta_generic_to_shared(raw + r * kRowBytes + piece * 16), src,
               ok ? 16 : 0);
  }
}

// ---------------------------------------------------------------- dp4a ----
constexpr int kTcD = 64;                        // samples per chunk
constexpr int kGroups = kTcD / 4;               // 4-sample groups per chunk
constexpr int kRawPanel = kTcD * kRowBytes;     // 8 KiB
constexpr int kWordPanel = kGroups * kBlk * 16; // 8 KiB: [group][slot][Xr,Xi,Yr,Yi]

__device__ __forceinline__ int dp4a(int a, int b, int c) {
  int d;
  asm("dp4a.s32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// raw [sample][station][4 bytes] -> words [group][slot][4 words of 4 samples]
__device__ __forceinline__ void to_words(const uint8_t *raw, int4 *words) {
  for (int u = threadIdx.x; u < kGroups * kBlk; u += kThreads) {
    const int g = u / kBlk, s = u % kBlk;
    const uint32_t *r = (const uint32_t *)(raw + (4 * g) * kRowBytes) + s;
    const uint32_t w0 = r[0], w1 = r[kRowBytes / 4], w2 = r[2 * kRowBytes / 4],
                   w3 = r[3 * kRowBytes / 4];
    const uint32_t lo01 = __byte_perm(w0, w1, 0x5140), hi01 = __byte_perm(w0, w1, 0x7362);
    const uint32_t lo23 = __byte_perm(w2, w3, 0x5140), hi23 = __byte_perm(w2, w3, 0x7362);
    int4 o;
    o.x = (int)__byte_perm(lo01, lo23, 0x5410);  // X re, samples 0..3
    o.y = (int)__byte_perm(lo01, lo23, 0x7632);  // X im
    o.z = (int)__byte_perm(hi01, hi23, 0x5410);  // Y re
    o.w = (int)__byte_perm(hi01, hi23, 0x7632);  // Y im
    words[g * kBlk + slot_of(s)] = o;
  }
}

__global__ void __launch_bounds__(kThreads, 2) xengine_dp4a_kernel(const Params p) {
  __shared__ __align__(16) uint8_t raw[2][2][kRawPanel];
  __shared__ __align__(16) int4 words[2][kWordPanel / 16];

  const int f = blockIdx.y;
  int rb, cb;
  decode_block(blockIdx.x, rb, cb);
  const bool diag = (rb == cb);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  // Time split blockIdx.z covers samples [tbeg, tend) of the call's range.
  const int tbeg = p.t0 + (int)blockIdx.z * p.per;
  const int tend = min(p.t0 + p.tcount, tbeg + p.per);
  const int nchunks = (tend - tbeg + kTcD - 1) / kTcD;

  int re[2][2][2][2], i1[2][2][2][2], i2[2][2][2][2];   // [rs][cs][p1][p2]
#pragma unroll
  for (int a = 0; a < 16; ++a) {
    (&re[0][0][0][0])[a] = 0;
    (&i1[0][0][0][0])[a] = 0;
    (&i2[0][0][0][0])[a] = 0;
  }

  load_panel<kTcD>(raw[0][0], p, f, rb * kBlk, tbeg, tend);
  if (!diag) load_panel<kTcD>(raw[0][1], p, f, cb * kBlk, tbeg, tend);
  cp_async_commit();

  for (int ch = 0; ch < nchunks; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nchunks) {
      const int tb = tbeg + (ch + 1) * kTcD;
      load_panel<kTcD>(raw[buf ^ 1][0], p, f, rb * kBlk, tb, tend);
      if (!diag) load_panel<kTcD>(raw[buf ^ 1][1], p, f, cb * kBlk, tb, tend);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    to_words(raw[buf][0], words[0]);
    if (!diag) to_words(raw[buf][1], words[1]);
    __syncthreads();
    const int4 *rw = words[0];
    const int4 *cw = diag ? words[0] : words[1];
#pragma unroll 1
    for (int g = 0; g < kGroups; ++g) {
      int4 r[2], c[2];
      r[0] = rw[g * kBlk + ty];
      r[1] = rw[g * kBlk + 16 + ty];
      c[0] = cw[g * kBlk + tx];
      c[1] = cw[g * kBlk + 16 + tx];
#pragma unroll
      for (int rs = 0; rs < 2; ++rs)
#pragma unroll
        for (int cs = 0; cs < 2; ++cs) {
          const int ar[2] = {r[rs].x, r[rs].z}, ai[2] = {r[rs].y, r[rs].w};
          const int br[2] = {c[cs].x, c[cs].z}, bi[2] = {c[cs].y, c[cs].w};
#pragma unroll
          for (int p1 = 0; p1 < 2; ++p1)
#pragma unroll
            for (int p2 = 0; p2 < 2; ++p2) {
              re[rs][cs][p1][p2] = dp4a(ar[p1], br[p2], re[rs][cs][p1][p2]);
              re[rs][cs][p1][p2] = dp4a(ai[p1], bi[p2], re[rs][cs][p1][p2]);
              i1[rs][cs][p1][p2] = dp4a(ai[p1], br[p2], i1[rs][cs][p1][p2]);
              i2[rs][cs][p1][p2] = dp4a(ar[p1], bi[p2], i2[rs][cs][p1][p2]);
            }
        }
    }
    __syncthreads();
  }

  int64_t *state = (int64_t *)p.state;
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 2; ++cs) {
      const int i = rb * kBlk + 2 * ty + rs, j = cb * kBlk + 2 * tx + cs;
      if (i >= p.n || j > i) continue;
      longlong2 *dst = (longlong2 *)(state + ((long long)f * p.nbaseline +
                                              (long long)i * (i + 1) / 2 + j) * 8);
#pragma unroll
      for (int p1 = 0; p1 < 2; ++p1)
#pragma unroll
        for (int p2 = 0; p2 < 2; ++p2) {
          const long long vr = re[rs][cs][p1][p2];
          const long long vi = (long long)i1[rs][cs][p1][p2] - (long long)i2[rs][cs][p1][p2];
          longlong2 *d = dst + p1 * 2 + p2;
          if (gridDim.z > 1) {
            // Time splits of one block add exactly, in any order.
            atomicAdd((unsigned long long *)&d->x, (unsigned long long)vr);
            atomicAdd((unsigned long long *)&d->y, (unsigned long long)vi);
          } else if (p.overwrite) {
            *d = make_longlong2(vr, vi);
          } else {
            longlong2 o = *d;
            o.x += vr;
            o.y += vi;
            *d = o;
          }
        }
    }
}

// ---------------------------------------------------------------- FP32 ----
constexpr int kTcF = 32;                         // samples per chunk
constexpr int kRawPanelF = kTcF * kRowBytes;     // 4 KiB
constexpr int kFloatPanel = kTcF * kBlk;         // float4 entries: [sample][slot]

__device__ __forceinline__ void to_floats(const uint8_t *raw, float4 *fl) {
  for (int u = threadIdx.x; u < kTcF * kBlk; u += kThreads) {
    const int t = u / kBlk, s = u % kBlk;
    const char4 b = *(const char4 *)(raw + t * kRowBytes + s * 4);
    fl[t * kBlk + slot_of(s)] = make_float4((float)b.x, (float)b.y, (float)b.z, (float)b.w);
  }
}

__global__ void __launch_bounds__(kThreads) xengine_fp32_kernel(const Params p) {
  __shared__ __align__(16) uint8_t raw[2][2][kRawPanelF];
  __shared__ __align__(16) float4 fl[2][kFloatPanel];

  const int f = blockIdx.y;
  int rb, cb;
  decode_block(blockIdx.x, rb, cb);
  const bool diag = (rb == cb);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int tend = p.t0 + p.tcount;
  const int nchunks = (p.tcount + kTcF - 1) / kTcF;

  float sr[2][2][2][2], si[2][2][2][2];
#pragma unroll
  for (int a = 0; a < 16; ++a) {
    (&sr[0][0][0][0])[a] = 0.f;
    (&si[0][0][0][0])[a] = 0.f;
  }

  load_panel<kTcF>(raw[0][0], p, f, rb * kBlk, p.t0, tend);
  if (!diag) load_panel<kTcF>(raw[0][1], p, f, cb * kBlk, p.t0, tend);
  cp_async_commit();

  for (int ch = 0; ch < nchunks; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nchunks) {
      const int tb = p.t0 + (ch + 1) * kTcF;
      load_panel<kTcF>(raw[buf ^ 1][0], p, f, rb * kBlk, tb, tend);
      if (!diag) load_panel<kTcF>(raw[buf ^ 1][1], p, f, cb * kBlk, tb, tend);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    to_floats(raw[buf][0], fl[0]);
    if (!diag) to_floats(raw[buf][1], fl[1]);
    __syncthreads();
    const float4 *rw = fl[0];
    const float4 *cw = diag ? fl[0] : fl[1];
#pragma unroll 4
    for (int t = 0; t < kTcF; ++t) {
      float4 r[2], c[2];
      r[0] = rw[t * kBlk + ty];
      r[1] = rw[t * kBlk + 16 + ty];
      c[0] = cw[t * kBlk + tx];
      c[1] = cw[t * kBlk + 16 + tx];
#pragma unroll
      for (int rs = 0; rs < 2; ++rs)
#pragma unroll
        for (int cs = 0; cs < 2; ++cs) {
          const float ar[2] = {r[rs].x, r[rs].z}, ai[2] = {r[rs].y, r[rs].w};
          const float br[2] = {c[cs].x, c[cs].z}, bi[2] = {c[cs].y, c[cs].w};
#pragma unroll
          for (int p1 = 0; p1 < 2; ++p1)
#pragma unroll
            for (int p2 = 0; p2 < 2; ++p2) {
              float &x = sr[rs][cs][p1][p2];
              float &y = si[rs][cs][p1][p2];
              x = fmaf(ar[p1], br[p2], x);
              x = fmaf(ai[p1], bi[p2], x);
              y = fmaf(ai[p1], br[p2], y);
              y = fmaf(-ar[p1], bi[p2], y);
            }
        }
    }
    __syncthreads();
  }

  float *state = (float *)p.state;
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 2; ++cs) {
      const int i = rb * kBlk + 2 * ty + rs, j = cb * kBlk + 2 * tx + cs;
      if (i >= p.n || j > i) continue;
      float4 *dst = (float4 *)(state + ((long long)f * p.nbaseline +
                                        (long long)i * (i + 1) / 2 + j) * 8);
#pragma unroll
      for (int p1 = 0; p1 < 2; ++p1) {
        float4 v = make_float4(sr[rs][cs][p1][0], si[rs][cs][p1][0], sr[rs][cs][p1][1],
                               si[rs][cs][p1][1]);
        if (!p.overwrite) {
          const float4 o = dst[p1];
          v.x += o.x;
          v.y += o.y;
          v.z += o.z;
          v.w += o.w;
        }
        dst[p1] = v;
      }
    }
}

}  // namespace plain

static dim3 plain_grid(const Sizes &s, int ksplit = 1) {
  const int nb = (s.n + plain::kBlk - 1) / plain::kBlk;
  return dim3((unsigned)(nb * (nb + 1) / 2), (unsigned)s.f, (unsigned)ksplit);
}

// Time splits for the dp4a kernel.  With fewer 32x32-station blocks than two
// waves of resident CTAs (two per SM), SMs idle: at N=256, F=10 the 360 blocks
// leave the second wave mostly empty, and at N=64 the 30 blocks occupy a fifth
// of the GPU.  Split each block's samples until there are about two waves,
// keeping at least 256 samples per split and at most 8 splits (each split adds
// its 8192 sums per block with int64 atomics).  Measured at F=10, T=1024:
// N=256 155 -> 137 us (2 splits), N=64 60 -> 27 us (4 splits).
static int plain_splits(const Sizes &s, int tcount) {
  const int slots = 2 * current_device_sms();
  if (!slots) return 1;
  const dim3 g = plain_grid(s);
  const long long blocks = (long long)g.x * g.y;
  long long k = (2LL * slots + blocks - 1) / blocks;
  if (k > tcount / 256) k = tcount / 256;
  if (k > 8) k = 8;
  return k < 1 ? 1 : (int)k;
}

cudaError_t launch_plain_dp4a(const int8_t *in, const Sizes &s, int t0, int tcount,
                              int64_t *state, int overwrite, cudaStream_t st) {
  const int ks = plain_splits(s, tcount);
  // samples per split: a whole number of 64-sample chunks
  int per = (tcount + ks - 1) / ks;
  per = (per + plain::kTcD - 1) / plain::kTcD * plain::kTcD;
  const int used = (tcount + per - 1) / per;
  if (used > 1 && overwrite) {
    cudaError_t e = cudaMemsetAsync(state, 0, (size_t)s.state_elems * 8, st);
    if (e != cudaSuccess) return e;
  }
  plain::Params p{in, s.n, s.f, t0, tcount, s.nbaseline, state, overwrite, per};
  plain::xengine_dp4a_kernel<<<plain_grid(s, used), plain::kThreads, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_plain_fp32(const int8_t *in, const Sizes &s, int t0, int tcount, float *state,
                              int overwrite, cudaStream_t st) {
  plain::Params p{in, s.n, s.f, t0, tcount, s.nbaseline, state, overwrite, tcount};
  plain::xengine_fp32_kernel<<<plain_grid(s), plain::kThreads, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace xgpu
