// engine_plain.cu -- CUDA-core X-engine: 2x2 register tile, FP32 and dp4a.
//
// The B200 counterpart of xGPU's shared2x2 kernels (kernel.cuh:238-422 FP32,
// kernel.cuh:427-591 dp4a, compute macros shared_transfer_4.cuh:91-156 and
// shared_transfer_4_dp4a.cuh:99-164).  The arithmetic per thread is the same:
// each thread owns a 2x2 block of stations (rows i, i+1 x columns j, j+1) and
// all 4 polarisation products of each, i.e. 16 complex visibilities.
//   FP32: 32 float accumulators; per sample and visibility the two products
//         of the real (and of the imaginary) part are summed exactly and the
//         sum is added with one rounding, as xGPU's float engine does
//         (omp_xengine.c:24-28), so the sums equal its own bit for bit:
//         3 FP32 instructions per component, 96 per sample.
//   dp4a: 48 int32 accumulators (re, im1, im2 as in kernel.cuh:464-479,574),
//         64 dp4a per group of 4 samples.
// What changes is the data path.  xGPU fetches one sample at a time through
// textures and swizzled input; here a CTA of 128 threads covers a block of
// 16 x 32 stations of one channel (small CTAs balance the SMs: the FP32
// engine may not split time), stages 128-byte panels of the natural
// [t][f][s][p][c] input into shared memory with TMA (one thread issues each
// chunk's panels on an mbarrier, double buffered; stations past n and samples
// past the input are zero-filled), and converts them in shared memory -- to 4-sample
// words for dp4a (a 4x4 byte transpose with PRMT) or to floats -- in an order
// that makes the 128-bit shared loads of the compute loop conflict-free.
// One launch covers a whole time range (not one NTIME_PIPE chunk), and the
// sums are added to the integration buffer once, at the end.
#include <atomic>

#include "internal.h"
#include "tc_common.cuh"

namespace xgpu {
namespace plain {

// A CTA covers a block of 16 (rows) x 32 (columns) stations of one channel
// with 128 threads, 8 x 16, each a 2x2 station tile.  Small CTAs balance the
// SMs: at N=256, F=10 there are 720 of them, five resident per SM, all at
// once (32 x 32 blocks of 256 threads gave 360 CTAs, two or three per SM).
constexpr int kBlk = 32;        // stations per column block
constexpr int kRows = 16;       // stations per row block
constexpr int kThreads = (kRows / 2) * (kBlk / 2);   // 128
constexpr int kRowBytes = kBlk * 4;   // one sample of one panel: 32 stations x 2 pol x re/im

// Block k -> (row block r of 16 stations, column block c of 32), 2c <= r:
// row blocks 2m and 2m + 1 both have m + 1 column blocks at or left of the
// diagonal, so blocks m(m+1) .. (m+1)^2 - 1 are row 2m, (m+1)^2 ..
// (m+1)(m+2) - 1 row 2m + 1.
__device__ __forceinline__ void decode_block(int k, int &rb, int &cb) {
  int m = (int)((sqrtf(4.0f * (float)k + 1.0f) - 1.0f) * 0.5f);
  while (m * (m + 1) > k) --m;
  while ((m + 1) * (m + 2) <= k) ++m;
  if (k < (m + 1) * (m + 1)) {
    rb = 2 * m;
    cb = k - m * (m + 1);
  } else {
    rb = 2 * m + 1;
    cb = k - (m + 1) * (m + 1);
  }
}

// Station (0..31) held in slot q of a converted panel: thread column tx reads
// stations 2tx and 2tx+1 from slots tx and 16+tx, so that 16 threads read 256
// contiguous bytes.  The conversions fill slot q from lane q, so a warp's
// stores are 32 consecutive slots (no bank conflicts).
__device__ __forceinline__ int station_of_slot(int q) { return q < 16 ? 2 * q : 2 * (q - 16) + 1; }

// Station (0..15) in slot q of a converted row panel: thread row ty reads
// stations 2ty and 2ty+1 from slots ty and 8+ty.
__device__ __forceinline__ int row_station_of_slot(int q) { return q < 8 ? 2 * q : 2 * (q - 8) + 1; }

struct Params {
  CUtensorMap map;  // the input, boxes of 128 bytes x one chunk of samples
  int n, f;
  int t0, tcount;
  long long nbaseline;
  void *state;
  int overwrite;
  int per;          // samples per time split (blockIdx.z); == tcount without splits
  int *err;         // receives kErrTimeoutPanel (may be null)
  int stall;        // test switch: issue no panel loads (the waits on them expire)
  int f0;           // first channel (blockIdx.y counts from it)
  int overlap;      // dp4a: may run beside the previous (adding) launch of the stream
};

// Queue the TMA loads of samples [tb, tb+NT) of the row panel and the column
// panel into raw[0] / raw[1], completing on bar.  Called by one thread.  The
// row panel is the 32 stations from station 16 rb (its 16 row stations are
// the first half; stations past n are zero-filled), the column panel the
// column block's 32 stations.
template <int NT>
__device__ __forceinline__ void issue_panels(uint8_t (*raw)[NT * kRowBytes], uint32_t bar,
                                             const Params &p, int f, int rb, int cb, int tb) {
  if (p.stall) return;
  tc::mbar_expect_tx(bar, 2 * NT * kRowBytes);
  tc::tma_load_3d(tc::smem_u32(raw[0]), &p.map, bar, rb * kRows * 4, f, tb);
  tc::tma_load_3d(tc::smem_u32(raw[1]), &p.map, bar, cb * kRowBytes, f, tb);
}

// A panel that never arrived (bounded wait expired): record it and leave
// without touching the integration buffer, after the other buffer's load (if
// one is in flight) has landed or its wait has expired too.
__device__ __forceinline__ void panel_timeout(const Params &p, uint32_t other_bar,
                                              uint32_t other_parity, bool other_in_flight) {
  if (threadIdx.x == 0) {
    if (p.err) atomicExch(p.err, kErrTimeoutPanel);
    if (other_in_flight && !p.stall) tc::mbar_wait(other_bar, other_parity, nullptr);
  }
}

// ---------------------------------------------------------------- dp4a ----
constexpr int kTcD = 64;                        // samples per chunk
constexpr int kGroups = kTcD / 4;               // 4-sample groups per chunk
constexpr int kRawPanel = kTcD * kRowBytes;     // 8 KiB
constexpr int kWordPanel = kGroups * kBlk * 16; // 8 KiB: [group][slot][Xr,Xi,Yr,Yi]
constexpr int kWordPanelRows = kGroups * kRows * 16;   // 4 KiB: the row block's 16 stations

__device__ __forceinline__ int dp4a(int a, int b, int c) {
  int d;
  asm("dp4a.s32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// raw [sample][station][4 bytes] -> words [group][slot][4 words of 4 samples]
// for the `slots` stations of a panel (32, or the row panel's first 16).
template <int kSlots>
__device__ __forceinline__ void to_words(const uint8_t *raw, int4 *words) {
  for (int u = threadIdx.x; u < kGroups * kSlots; u += kThreads) {
    const int g = u / kSlots, q = u % kSlots;
    const int s = kSlots == kBlk ? station_of_slot(q) : row_station_of_slot(q);
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
    words[g * kSlots + q] = o;
  }
}

// Epilogue staging (in the panels' memory): 8 block rows of 32 baselines x
// 4 products x {re, im} int64, thread tx's two baselines (128 bytes) at
// tx * kEpiSeg in its row, 16 bytes apart from the next thread's, so that the
// eight lanes of each 16-byte store phase write eight different bank groups.
constexpr int kEpiSeg = 144;
constexpr int kEpiRow = 16 * kEpiSeg;

// Dynamic shared memory of the dp4a kernel: raw panels [2 buffers][row,
// column], the converted row and column words, two mbarriers, and room to
// align the panels to 128 bytes (TMA destinations): 45.2 KB, five CTAs per
// SM (95 registers a thread).
constexpr int kSmemDp4a = 2 * 2 * kRawPanel + kWordPanelRows + kWordPanel + 16 + 128;
static_assert(5 * (kSmemDp4a + 1024) <= 228 * 1024, "five dp4a CTAs per SM");
static_assert((kRows / 2) * kEpiRow <= 2 * 2 * kRawPanel, "epilogue staging fits the panels");

__global__ void __launch_bounds__(kThreads, 5) xengine_dp4a_kernel(const __grid_constant__ Params p) {
  extern __shared__ __align__(128) uint8_t dsm_raw[];
  uint8_t *dsm = (uint8_t *)(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
  auto raw = (uint8_t(*)[2][kRawPanel])dsm;
  int4 *wrow = (int4 *)(dsm + 2 * 2 * kRawPanel);   // row words, 16 slots
  int4 *wcol = wrow + kGroups * kRows;               // column words, 32 slots
  uint64_t *bars = (uint64_t *)(wcol + kGroups * kBlk);

  const int f = p.f0 + (int)blockIdx.y;
  int rb, cb;   // row block of 16 stations, column block of 32
  decode_block(blockIdx.x, rb, cb);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // ty 0..7
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

  // Programmatic launch (as the tensor-core kernels): unless this launch only
  // adds into sums that the previous launch of the stream also only adds
  // into, nothing below reads or writes global memory before that launch has
  // finished; an overlapping launch waits for it at the end instead, so it
  // never completes first.  Either way the next launch may start now.
  if (!p.overlap) tc::pdl_wait();
  tc::pdl_trigger();
  const uint32_t bar0 = tc::smem_u32(&bars[0]);
  if (threadIdx.x == 0) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&p.map) : "memory");
    tc::mbar_init(bar0, 1);
    tc::mbar_init(bar0 + 8, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    issue_panels<kTcD>(raw[0], bar0, p, f, rb, cb, tbeg);
  }
  __syncthreads();

  for (int ch = 0; ch < nchunks; ++ch) {
    const int buf = ch & 1;
    // Chunk ch+1 goes into the other buffer, free since the end of chunk ch-1.
    if (threadIdx.x == 0 && ch + 1 < nchunks)
      issue_panels<kTcD>(raw[buf ^ 1], bar0 + 8 * (buf ^ 1), p, f, rb, cb,
                         tbeg + (ch + 1) * kTcD);
    const bool got = tc::mbar_wait(bar0 + 8 * buf, (ch >> 1) & 1, nullptr);
    if (__syncthreads_or(!got)) {
      panel_timeout(p, bar0 + 8 * (buf ^ 1), ((ch + 1) >> 1) & 1, ch + 1 < nchunks);
      if (p.overlap) tc::pdl_wait();
      return;
    }
    to_words<kRows>(raw[buf][0], wrow);
    to_words<kBlk>(raw[buf][1], wcol);
    __syncthreads();
#pragma unroll 1
    for (int g = 0; g < kGroups; ++g) {
      int4 r[2], c[2];
      r[0] = wrow[g * kRows + ty];
      r[1] = wrow[g * kRows + 8 + ty];
      c[0] = wcol[g * kBlk + tx];
      c[1] = wcol[g * kBlk + 16 + tx];
      // Four sweeps over the 16 visibilities of the 2x2 tile, so that the two
      // dp4a of one real part are 48 instructions apart, not back to back.
#pragma unroll
      for (int sweep = 0; sweep < 4; ++sweep)
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
                if (sweep == 0) re[rs][cs][p1][p2] = dp4a(ar[p1], br[p2], re[rs][cs][p1][p2]);
                if (sweep == 1) i1[rs][cs][p1][p2] = dp4a(ai[p1], br[p2], i1[rs][cs][p1][p2]);
                if (sweep == 2) i2[rs][cs][p1][p2] = dp4a(ar[p1], bi[p2], i2[rs][cs][p1][p2]);
                if (sweep == 3) re[rs][cs][p1][p2] = dp4a(ai[p1], bi[p2], re[rs][cs][p1][p2]);
              }
          }
    }
    __syncthreads();
  }

  // Sums out, half of the block's rows at a time (rs = 0: even rows, 1: odd
  // rows): the threads stage them in shared memory (the panels are free) in
  // the buffer's order, and each of the four warps then adds two of the eight
  // staged rows with 32
  // consecutive words per instruction -- 256 contiguous bytes, where adding
  // straight from the threads' 2x2 tiles scatters every instruction over 32
  // lines (measured: the epilogue took 20 of 135 us at N=256, F=10, T=1024).
  // Time splits of one block add exactly, in any order, as does an adding
  // call; a storing call without splits stores.
  int64_t *state = (int64_t *)p.state;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool store = p.overwrite && gridDim.z == 1;
#pragma unroll
  for (int rs = 0; rs < 2; ++rs) {
    uint8_t *seg = dsm + ty * kEpiRow + tx * kEpiSeg;
#pragma unroll
    for (int cs = 0; cs < 2; ++cs)
#pragma unroll
      for (int p1 = 0; p1 < 2; ++p1)
#pragma unroll
        for (int p2 = 0; p2 < 2; ++p2) {
          const long long vr = re[rs][cs][p1][p2];
          const long long vi = (long long)i1[rs][cs][p1][p2] - (long long)i2[rs][cs][p1][p2];
          *(longlong2 *)(seg + (cs * 4 + p1 * 2 + p2) * 16) = make_longlong2(vr, vi);
        }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = warp + 4 * h;              // staged row: station i of the block
      const int i = rb * kRows + 2 * r + rs;
      if (i < p.n) {
        // the row's baselines (i, cb*32 .. cb*32+31) are 256 consecutive
        // words of the buffer; on the diagonal only columns j <= i count
        int64_t *row = state + ((long long)f * p.nbaseline + (long long)i * (i + 1) / 2 +
                                cb * kBlk) * 8;
        const int jmax = i - cb * kBlk;
#pragma unroll
        for (int it = 0; it < 8; ++it) {
          const int w = it * 32 + lane;         // word w: baseline w / 8 of the row
          if ((w >> 3) <= jmax) {
            const long long v =
                *(const long long *)(dsm + r * kEpiRow + (w >> 4) * kEpiSeg + (w & 15) * 8);
            if (store) row[w] = v;
            else atomicAdd((unsigned long long *)(row + w), (unsigned long long)v);
          }
        }
      }
    }
    __syncthreads();
  }
  if (p.overlap) tc::pdl_wait();
}

// ---------------------------------------------------------------- FP32 ----
// The FP32 engine may not split time (its sums keep xGPU's order); the small
// blocks balance its SMs.
constexpr int kTcF = 32;                         // samples per chunk
constexpr int kRawPanelF = kTcF * kRowBytes;     // 4 KiB
constexpr int kFloatPanel = kTcF * kBlk;         // float4 entries: [sample][slot]
constexpr int kFloatPanelRows = kTcF * kRows;    // the row block's 16 stations

__device__ __forceinline__ void to_floats(const uint8_t *raw, float4 *fl) {
  for (int u = threadIdx.x; u < kTcF * kBlk; u += kThreads) {
    const int t = u / kBlk, q = u % kBlk, s = station_of_slot(q);
    const char4 b = *(const char4 *)(raw + t * kRowBytes + s * 4);
    fl[t * kBlk + q] = make_float4((float)b.x, (float)b.y, (float)b.z, (float)b.w);
  }
}

// The row panel: the first 16 stations of a 32-station panel.
__device__ __forceinline__ void to_floats_rows(const uint8_t *raw, float4 *fl) {
  for (int u = threadIdx.x; u < kTcF * kRows; u += kThreads) {
    const int t = u / kRows, q = u % kRows, s = row_station_of_slot(q);
    const char4 b = *(const char4 *)(raw + t * kRowBytes + s * 4);
    fl[t * kRows + q] = make_float4((float)b.x, (float)b.y, (float)b.z, (float)b.w);
  }
}

// Dynamic shared memory of the FP32 kernel: raw panels [2 buffers][row,
// column], the converted row and column panels, two mbarriers, and room to
// align the panels to 128 bytes.
constexpr int kSmemFp32 =
    2 * 2 * kRawPanelF + (kFloatPanelRows + kFloatPanel) * 16 + 16 + 128;
// five CTAs per SM by shared memory (80 registers a thread would allow six)
static_assert(5 * (kSmemFp32 + 1024) <= 228 * 1024, "five FP32 CTAs per SM");

__global__ void __launch_bounds__(kThreads) xengine_fp32_kernel(const __grid_constant__ Params p) {
  extern __shared__ __align__(128) uint8_t dsm_raw[];
  uint8_t *dsm = (uint8_t *)(((uintptr_t)dsm_raw + 127) & ~(uintptr_t)127);
  auto raw = (uint8_t(*)[2][kRawPanelF])dsm;
  float4 *flr = (float4 *)(dsm + 2 * 2 * kRawPanelF);   // row panel, 16 slots
  float4 *flc = flr + kFloatPanelRows;                   // column panel, 32 slots
  uint64_t *bars = (uint64_t *)(flc + kFloatPanel);

  const int f = p.f0 + (int)blockIdx.y;
  int rb, cb;   // row block of 16 stations, column block of 32
  decode_block(blockIdx.x, rb, cb);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // ty 0..7
  const int nchunks = (p.tcount + kTcF - 1) / kTcF;

  // The accumulators continue the integration buffer's sums (0 after a
  // clear), so an integration over several calls is one sum in time order.
  float sr[2][2][2][2], si[2][2][2][2];
  float *state = (float *)p.state;
#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 2; ++cs) {
      const int i = rb * kRows + 2 * ty + rs, j = cb * kBlk + 2 * tx + cs;
      const bool mine = !p.overwrite && i < p.n && j <= i;
      const float4 *src = (const float4 *)(state + ((long long)f * p.nbaseline +
                                                    (long long)i * (i + 1) / 2 + j) * 8);
#pragma unroll
      for (int p1 = 0; p1 < 2; ++p1) {
        const float4 o = mine ? src[p1] : make_float4(0.f, 0.f, 0.f, 0.f);
        sr[rs][cs][p1][0] = o.x;
        si[rs][cs][p1][0] = o.y;
        sr[rs][cs][p1][1] = o.z;
        si[rs][cs][p1][1] = o.w;
      }
    }

  const uint32_t bar0 = tc::smem_u32(&bars[0]);
  if (threadIdx.x == 0) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&p.map) : "memory");
    tc::mbar_init(bar0, 1);
    tc::mbar_init(bar0 + 8, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    issue_panels<kTcF>(raw[0], bar0, p, f, rb, cb, p.t0);
  }
  __syncthreads();

  for (int ch = 0; ch < nchunks; ++ch) {
    const int buf = ch & 1;
    // Chunk ch+1 goes into the other buffer, free since the end of chunk ch-1.
    if (threadIdx.x == 0 && ch + 1 < nchunks)
      issue_panels<kTcF>(raw[buf ^ 1], bar0 + 8 * (buf ^ 1), p, f, rb, cb, p.t0 + (ch + 1) * kTcF);
    const bool got = tc::mbar_wait(bar0 + 8 * buf, (ch >> 1) & 1, nullptr);
    if (__syncthreads_or(!got)) {
      panel_timeout(p, bar0 + 8 * (buf ^ 1), ((ch + 1) >> 1) & 1, ch + 1 < nchunks);
      return;
    }
    to_floats_rows(raw[buf][0], flr);
    to_floats(raw[buf][1], flc);
    __syncthreads();
#pragma unroll 4
    for (int t = 0; t < kTcF; ++t) {
      float4 r[2], c[2];
      r[0] = flr[t * kRows + ty];
      r[1] = flr[t * kRows + 8 + ty];
      c[0] = flc[t * kBlk + tx];
      c[1] = flc[t * kBlk + 16 + tx];
#pragma unroll
      for (int rs = 0; rs < 2; ++rs)
#pragma unroll
        for (int cs = 0; cs < 2; ++cs) {
          const float ar[2] = {r[rs].x, r[rs].z}, ai[2] = {r[rs].y, r[rs].w};
          const float br[2] = {c[cs].x, c[cs].z}, bi[2] = {c[cs].y, c[cs].w};
          // xGPU's float arithmetic (omp_xengine.c:24-28): a sample's
          // two products are summed first -- exactly: products of int8
          // values and their sums are integers below 2^24 -- and the sum is
          // added to the accumulator with one rounding.
#pragma unroll
          for (int p1 = 0; p1 < 2; ++p1)
#pragma unroll
            for (int p2 = 0; p2 < 2; ++p2) {
              float &x = sr[rs][cs][p1][p2];
              float &y = si[rs][cs][p1][p2];
              x = __fadd_rn(x, __fmaf_rn(ai[p1], bi[p2], __fmul_rn(ar[p1], br[p2])));
              y = __fadd_rn(y, __fmaf_rn(ai[p1], br[p2], -__fmul_rn(ar[p1], bi[p2])));
            }
        }
    }
    __syncthreads();
  }

#pragma unroll
  for (int rs = 0; rs < 2; ++rs)
#pragma unroll
    for (int cs = 0; cs < 2; ++cs) {
      const int i = rb * kRows + 2 * ty + rs, j = cb * kBlk + 2 * tx + cs;
      if (i >= p.n || j > i) continue;
      float4 *dst = (float4 *)(state + ((long long)f * p.nbaseline +
                                        (long long)i * (i + 1) / 2 + j) * 8);
#pragma unroll
      for (int p1 = 0; p1 < 2; ++p1)
        dst[p1] = make_float4(sr[rs][cs][p1][0], si[rs][cs][p1][0], sr[rs][cs][p1][1],
                              si[rs][cs][p1][1]);
    }
}

}  // namespace plain

// Blocks of 16-station rows r and 32-station columns c <= r / 2
// (decode_block), per channel, times the time splits.
static dim3 plain_grid(const Sizes &s, int fcount, int ksplit = 1) {
  const int nr = (s.n + plain::kRows - 1) / plain::kRows;
  const int m = nr / 2;
  const int blocks = nr % 2 == 0 ? m * (m + 1) : (m + 1) * (m + 1);
  return dim3((unsigned)blocks, (unsigned)fcount, (unsigned)ksplit);
}

// Time splits of a dp4a launch: enough CTAs for one wave of resident CTAs
// (five per SM), or for half of one when the launch may overlap the previous
// adding launch (whose last CTAs, and the next launch's, fill the rest; each
// split costs its ramp and its atomics), at least 256 samples per split and
// at most 8 splits.
static int plain_splits(const Sizes &s, int fcount, int tcount, bool overlap) {
  const int slots = 5 * current_device_sms();   // resident dp4a CTAs
  if (!slots) return 1;
  const dim3 g = plain_grid(s, fcount);
  const long long blocks = (long long)g.x * g.y;
  const long long target = overlap ? slots / 2 : slots;
  long long k = (target + blocks - 1) / blocks;
  if (k > tcount / 256) k = tcount / 256;
  if (k > 8) k = 8;
  return k < 1 ? 1 : (int)k;
}

// The kernels' dynamic shared memory (45.2 and 41.1 KB), allowed once per
// device.
static cudaError_t plain_configure_device() {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < kDeviceCache) ? 1ull << dev : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(plain::xengine_dp4a_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           plain::kSmemDp4a);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(plain::xengine_fp32_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, plain::kSmemFp32);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
  return e;
}

static int plain_params(plain::Params *p, const int8_t *in, const Sizes &s, int t0, int tcount,
                        void *state, int overwrite, int per, int rows, int *err, int stall,
                        int f0) {
  if (make_panel_map(&p->map, in, s, rows) != 0) return -1;
  p->n = s.n;
  p->f = s.f;
  p->t0 = t0;
  p->tcount = tcount;
  p->nbaseline = s.nbaseline;
  p->state = state;
  p->overwrite = overwrite;
  p->per = per;
  p->err = err;
  p->stall = stall;
  p->f0 = f0;
  p->overlap = 0;
  return 0;
}

cudaError_t launch_plain_dp4a(const int8_t *in, const Sizes &s, int t0, int tcount,
                              int64_t *state, int overwrite, cudaStream_t st, int *err,
                              int stall, int f0, int fcount, int overlap) {
  if (fcount < 0) fcount = s.f - f0;
  if (f0 < 0 || fcount < 1 || f0 + fcount > s.f) return cudaErrorInvalidValue;
  const int ks = plain_splits(s, fcount, tcount, overlap && !overwrite);
  // samples per split: a whole number of 64-sample chunks
  int per = (tcount + ks - 1) / ks;
  per = (per + plain::kTcD - 1) / plain::kTcD * plain::kTcD;
  const int used = (tcount + per - 1) / per;
  if (used > 1 && overwrite) {   // the splits add: clear the channel range first
    const size_t per_channel = (size_t)s.state_elems / s.f;
    cudaError_t e = cudaMemsetAsync(state + (size_t)f0 * per_channel, 0,
                                    (size_t)fcount * per_channel * 8, st);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = plain_configure_device();
  if (e != cudaSuccess) return e;
  plain::Params p;
  if (plain_params(&p, in, s, t0, tcount, state, overwrite, per, plain::kTcD, err, stall, f0) != 0)
    return cudaErrorInvalidValue;
  p.overlap = (overlap && !overwrite) ? 1 : 0;
  // Programmatic launch: the grid may start beside the previous kernel's last
  // CTAs (the kernel waits for it where it must).
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = plain_grid(s, fcount, used);
  cfg.blockDim = dim3(plain::kThreads);
  cfg.dynamicSmemBytes = plain::kSmemDp4a;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, plain::xengine_dp4a_kernel, p);
}

cudaError_t launch_plain_fp32(const int8_t *in, const Sizes &s, int t0, int tcount, float *state,
                              int overwrite, cudaStream_t st, int *err, int stall, int f0,
                              int fcount) {
  if (fcount < 0) fcount = s.f - f0;
  if (f0 < 0 || fcount < 1 || f0 + fcount > s.f) return cudaErrorInvalidValue;
  cudaError_t e = plain_configure_device();
  if (e != cudaSuccess) return e;
  plain::Params p;
  if (plain_params(&p, in, s, t0, tcount, state, overwrite, tcount, plain::kTcF, err, stall,
                   f0) != 0)
    return cudaErrorInvalidValue;
  plain::xengine_fp32_kernel<<<plain_grid(s, fcount), plain::kThreads, plain::kSmemFp32,
                               st>>>(p);
  return cudaGetLastError();
}

}  // namespace xgpu
