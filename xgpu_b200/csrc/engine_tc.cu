// engine_tc.cu -- tcgen05 int8 tensor-core X-engine (single jobs and batches).
//
// The visibility matrix of one channel is the Hermitian rank-T update
// V = sum_t x(t) x(t)^H over the 2N station-polarisation inputs
// (xGPU kernel.cuh:238-422 computes the same sums with FP32 FMAs, and
// omp_xengine.c:45-89 on the host).  This engine treats the real and imaginary
// parts of every input as separate real rows: with A[m][t] = the int8 byte m
// of sample t in the input layout [t][f][s][p][c] (m = 4s + 2p + c), the real
// Gram matrix G = A A^T holds everything:
//   Re V[(i,p1),(j,p2)] = G[(i,p1,re),(j,p2,re)] + G[(i,p1,im),(j,p2,im)]
//   Im V[(i,p1),(j,p2)] = G[(i,p1,im),(j,p2,re)] - G[(i,p1,re),(j,p2,im)]
// G is a plain int8 x int8 -> int32 GEMM with both operands "MN-major" (the
// 4N input bytes of one sample are contiguous), so the kernel reads the input
// exactly as it lies in HBM: no corner turn, no negation of -128, one
// accumulator.  The two sums of each complex part are formed in int64 when
// the accumulator is drained, so the result is exact.
//
// Work items: (job, channel, time split, 128x128 tile of G on or below the
// diagonal), a tile being 32 stations x 2 pols x re/im on each side.  A
// persistent grid (one CTA per SM) takes items from a static stride or from a
// global atomic work queue (uneven batches); the producer publishes each item
// to the other roles through a small shared-memory ring.  Six warps:
//   warp 0    scheduler + TMA producer: 3-D tiled loads (128 bytes x 128
//             samples, 128-byte swizzle) of row and column panels, 5 stages
//   warp 1    TMEM owner and MMA issuer: tcgen05.mma.cta_group::1.kind::i8,
//             M=N=128, K=32, into one of two TMEM accumulators (2 x 128
//             columns), so a tile's drain overlaps the next tile's MMAs
//   warps 2-5 epilogue: drain TMEM (tcgen05.ld 32x32b), combine the re/im
//             rows of every input with two warp shuffles into int64 (re, im)
//             pairs staged in shared memory (one 2 KB row per station), then
//             32 lanes hand the rows to the bulk-copy engine: a plain bulk
//             store when the item is the only writer of a zero buffer, a bulk
//             reduce-add (cp.reduce.async.bulk .add.u64) otherwise -- the int64
//             accumulation happens in L2 and the old values never travel to
//             the SM, and time splits of one tile add up exactly.
// Every mbarrier wait is bounded; a timeout writes an error code, raises a
// CTA-wide abort flag so the other roles stop waiting, and the kernel still
// waits (bounded) for its own copies and MMAs, frees its TMEM and returns.
// Single-job launches are programmatic (PDL): the prologue overlaps the
// previous kernel of the stream, and a launch that only adds into sums the
// previous launch also only adds into runs beside it (see the kernel body).
#include <cudaTypedefs.h>

#include <atomic>

#include "internal.h"
#include "tc_job.h"
#include "tc_common.cuh"

namespace xgpu {
namespace tc {

constexpr int kTile = 128;                 // G rows (and columns) per tile
constexpr int kStations = kTile / 4;       // 32 stations per tile side
constexpr int kKt = kTcSamplesPerStage;    // samples per pipeline stage
constexpr int kStages = 5;
constexpr int kSched = 4;                  // work-item ring between the roles
constexpr int kBoxBytes = kTile * kKt;     // one operand of one stage: 16 KiB
constexpr int kStageBytes = 2 * kBoxBytes;
// Staging of one 32x32-station block of drained sums (staging_row).
constexpr int kStateBytes = kStagingBytes;
constexpr int kBarrierBytes = 512;    // barriers, work-item ring, TMEM slot
constexpr int kSmemBytes = kStages * kStageBytes + kStateBytes + kBarrierBytes + 1024;
static_assert(kSmemBytes <= 227 * 1024, "dynamic shared memory of one CTA");
constexpr uint32_t kTmemCols = 2 * kTile;  // two accumulators
constexpr int kThreads = 192;

constexpr uint32_t kIdesc = i8_idesc(kTile, kTile);

struct Params {
  Job single;          // the job when jobs == nullptr (its tensor map is a parameter)
  const Job *jobs;     // batched: job table in global memory, ordered by item_begin
  int njobs;
  int total;           // work items over all jobs
  int *queue;          // dynamic work counter (zeroed before launch); nullptr: static stride
  int *err;
  int stall;           // test switch: issue no loads (the waits on them expire)
  int streamk;         // single job: each CTA takes an equal share of all (tile, stage) steps
  int overlap;         // may run alongside the previous (accumulating) launch of the stream
};

// A decoded work item.  The scheduler decodes each item once and publishes it
// in a shared-memory ring; the MMA issuer and the epilogue copy it to
// registers, so neither reads the job table on its critical path.
struct Item {
  int u;               // work item index (>= total: no more work)
  int f, tr, tc;
  int step0, nsteps;   // pipeline stages of this item (its time split)
  int n, store, t0, pad;
  long long nbaseline;
  int64_t *state;
  const CUtensorMap *map;
};

__device__ __forceinline__ Item decode_job(const Job &j, int u) {
  Item it;
  it.u = u;
  const int v = u - j.item_begin;
  const int k = v % j.npairs;          // tile within the channel
  const int rest = v / j.npairs;
  const int split = rest % j.ksplit;
  it.f = j.f0 + rest / j.ksplit;
  int r = (int)((sqrtf(8.0f * (float)k + 1.0f) - 1.0f) * 0.5f);
  while (r * (r + 1) / 2 > k) --r;
  while ((r + 1) * (r + 2) / 2 <= k) ++r;
  it.tr = r;
  it.tc = k - r * (r + 1) / 2;
  it.step0 = split * j.steps_per_split;
  const int ns = j.total_steps - it.step0;
  it.nsteps = ns < j.steps_per_split ? ns : j.steps_per_split;
  it.n = j.n;
  it.store = j.store;
  it.t0 = j.t0;
  it.pad = 0;
  it.nbaseline = j.nbaseline;
  it.state = j.state;
  it.map = &j.map;
  return it;
}

__device__ __forceinline__ Item decode_item(const Params &p, int u) {
  if (p.jobs) {
    int lo = 0, hi = p.njobs - 1;   // last job with item_begin <= u
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (p.jobs[mid].item_begin <= u) lo = mid; else hi = mid - 1;
    }
    return decode_job(p.jobs[lo], u);
  }
  // Named parameter fields: constant-bank reads rather than generic loads
  // through a pointer that may point to either space.
  return decode_job(p.single, u);
}

// Bytes of station row il (0..31) of the item's tile inside the integration
// buffer: baselines (i, j) with j in the tile's column block, j <= i, j < n.
__device__ __forceinline__ int row_bytes(const Item &t, int il) {
  const int i = t.tr * kStations + il;
  if (i >= t.n) return 0;
  int cnt = t.n - t.tc * kStations;
  if (cnt > kStations) cnt = kStations;
  if (t.tr == t.tc && il + 1 < cnt) cnt = il + 1;
  return cnt * 64;
}

__device__ __forceinline__ int64_t *row_ptr(const Item &t, int il) {
  const long long i = (long long)t.tr * kStations + il;
  return t.state + ((long long)t.f * t.nbaseline + i * (i + 1) / 2 + (long long)t.tc * kStations) * 8;
}

__global__ void __launch_bounds__(kThreads, 1) xengine_tc_kernel(const __grid_constant__ Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *sstate = smem + kStages * kStageBytes;
  uint64_t *bars = (uint64_t *)(sstate + kStateBytes);
  // full[kStages] empty[kStages] tfull[2] tempty[2] sfull[kSched] sempty[kSched] mma_done
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages),
                 tfull0 = smem_u32(bars + 2 * kStages), tempty0 = smem_u32(bars + 2 * kStages + 2),
                 sfull0 = smem_u32(bars + 2 * kStages + 4),
                 sempty0 = smem_u32(bars + 2 * kStages + 4 + kSched),
                 mma_done = smem_u32(bars + 2 * kStages + 4 + 2 * kSched);
  Item *ring = (Item *)(bars + 2 * kStages + 6 + 2 * kSched);   // 8-byte aligned
  uint32_t *tmem_slot = (uint32_t *)(ring + kSched);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull0 + 8 * a, 1);
      mbar_init(tempty0 + 8 * a, kEpiThreads / 32);
    }
    for (int q = 0; q < kSched; ++q) {
      mbar_init(sfull0 + 8 * q, 1);
      mbar_init(sempty0 + 8 * q, 2);   // MMA issuer + epilogue
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t stage0 = smem_u32(smem);
  // Prologue done.  Unless this launch only adds into sums that the previous
  // launch of the stream (an engine launch of the same context) also only
  // adds into, nothing below touches global memory before the previous launch
  // has finished; an overlapping launch waits for it at the end instead, so it
  // never completes first.  The next launch may start once this one has
  // waited: a chain of overlapping launches thus only ever runs beside
  // launches that add, never beside a store or anything else queued earlier.
  if (!p.overlap) pdl_wait();
  pdl_trigger();

  auto fail = [&](int code) {
    atomicExch(p.err, code);
    *abort_flag = 1;
  };

  if (warp == 0) {
    // ------------------------------------------------ scheduler + producer --
    if (lane == 0) {
      if (!p.jobs) asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&p.single.map) : "memory");
      uint32_t g = 0, g_loaded = 0;
      bool ok = true;
      // Stream-K: CTA b covers steps [b*W/G, (b+1)*W/G) of the W = items x
      // stages of the job, cutting tiles where the ranges meet; the pieces of
      // a cut tile add up exactly in the integration buffer (reduce-add).
      const long long sk_w = p.streamk ? (long long)p.total * p.single.total_steps : 0;
      long long sk_pos = p.streamk ? sk_w * blockIdx.x / gridDim.x : 0;
      const long long sk_end = p.streamk ? sk_w * (blockIdx.x + 1) / gridDim.x : 0;
      for (int i = 0; ok; ++i) {
        const int slot = i % kSched;
        if (i >= kSched && !mbar_wait(sempty0 + 8 * slot, ((i / kSched) - 1) & 1, abort_flag)) {
          fail(kErrTimeoutProducer);
          break;
        }
        Item t;
        if (p.streamk) {
          if (sk_pos < sk_end) {
            const int ts = p.single.total_steps;
            const int item = (int)(sk_pos / ts);
            const int s0 = (int)(sk_pos % ts);
            const long long left = sk_end - sk_pos;
            const int ns = (int)(ts - s0 < left ? ts - s0 : left);
            t = decode_item(p, item);
            t.step0 = s0;
            t.nsteps = ns;
            t.store = (s0 == 0 && ns == ts) ? t.store : 0;
            sk_pos += ns;
          } else {
            t.u = p.total;
          }
        } else {
          const int u = p.queue ? atomicAdd(p.queue, 1) : (int)blockIdx.x + i * (int)gridDim.x;
          if (u < p.total) {
            t = decode_item(p, u);
          } else {
            t.u = u;
          }
        }
        const int u = t.u;
        ring[slot] = t;
        mbar_arrive(sfull0 + 8 * slot);   // release: the entry is visible to the waiters
        if (u >= p.total) break;
        const bool diag = (t.tr == t.tc);
        const CUtensorMap *map = t.map;
        for (int ks = 0; ks < t.nsteps; ++ks, ++g) {
          const uint32_t s = g % kStages;
          if (g >= (uint32_t)kStages &&
              !mbar_wait(empty0 + 8 * s, ((g / kStages) - 1) & 1, abort_flag)) {
            fail(kErrTimeoutProducer);
            ok = false;
            break;
          }
          if (p.stall) continue;
          const uint32_t dst = stage0 + s * kStageBytes;
          mbar_expect_tx(full0 + 8 * s, diag ? kBoxBytes : 2 * kBoxBytes);
          const int z = t.t0 + (t.step0 + ks) * kKt;
          tma_load_3d(dst, map, full0 + 8 * s, t.tr * kTile, t.f, z);
          if (!diag) tma_load_3d(dst + kBoxBytes, map, full0 + 8 * s, t.tc * kTile, t.f, z);
          g_loaded = g + 1;
        }
      }
      // Loads still in flight land before the CTA leaves (a no-op normally).
      for (uint32_t q = (g_loaded > (uint32_t)kStages ? g_loaded - kStages : 0); q < g_loaded; ++q)
        mbar_wait(full0 + 8 * (q % kStages), (q / kStages) & 1, nullptr);
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA --
    if (lane == 0) {
      uint32_t g = 0;
      bool ok = true;
      for (int i = 0; ok; ++i) {
        const int slot = i % kSched;
        if (!mbar_wait(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag)) {
          fail(kErrTimeoutMma);
          break;
        }
        const Item t = ring[slot];
        mbar_arrive(sempty0 + 8 * slot);
        if (t.u >= p.total) break;
        const bool diag = (t.tr == t.tc);
        const int acc = i & 1;
        if (i >= 2 && !mbar_wait(tempty0 + 8 * acc, ((i >> 1) - 1) & 1, abort_flag)) {
          fail(kErrTimeoutMma);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * kTile);
        for (int ks = 0; ks < t.nsteps; ++ks, ++g) {
          const uint32_t s = g % kStages;
          if (!mbar_wait(full0 + 8 * s, (g / kStages) & 1, abort_flag)) {
            fail(kErrTimeoutMma);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a = stage0 + s * kStageBytes;
          const uint32_t b = diag ? a : a + kBoxBytes;
#pragma unroll
          for (int kk = 0; kk < kKt / 32; ++kk) {
            // 32 samples = 4 swizzle atoms = 4096 bytes per instruction.
            mma_i8(d, mn_sw128_desc(a + kk * 4096, kBoxBytes), mn_sw128_desc(b + kk * 4096, kBoxBytes),
                   kIdesc, (ks | kk) != 0 ? 1u : 0u);
          }
          mma_commit(empty0 + 8 * s);
        }
        if (ok) mma_commit(tfull0 + 8 * acc);
      }
      // Every MMA issued by this CTA has completed once mma_done fires.
      mma_commit(mma_done);
      mbar_wait(mma_done, 0, nullptr);
    }
  } else {
    // ---------------------------------------------------------- epilogue --
    const int ew = warp - 2;                 // 0..3; warp ew == 0 issues the copies
    const int quarter = warp & 3;            // TMEM lanes 32*quarter .. +31
    const int m = quarter * 32 + lane;       // G row of this thread
    const int c = m & 1;                     // 0: real row, 1: imaginary row
    const int p1 = (m >> 1) & 1;
    const int il = m >> 2;                   // station within the row block
    const bool copier = (ew == 0);           // lane r copies staging row r
    for (int i = 0;; ++i) {
      const int slot = i % kSched;
      const bool got = mbar_wait(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag);
      Item t;
      if (got) t = ring[slot];
      if (copier) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // staging free
      if (epi_any(!got)) {
        if (ew == 0 && lane == 0) fail(kErrTimeoutDrain);
        break;
      }
      // every epilogue thread has copied the entry
      if (ew == 0 && lane == 0) mbar_arrive(sempty0 + 8 * slot);
      if (t.u >= p.total) break;
      const int acc = i & 1;
      const bool have = mbar_wait(tfull0 + 8 * acc, (i >> 1) & 1, abort_flag);
      if (epi_any(!have)) {
        if (ew == 0 && lane == 0) fail(kErrTimeoutDrain);
        break;
      }
      __syncwarp();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint8_t *srow = sstate + staging_row(il) + (p1 * 2 + c) * 16;
      int jmax = t.n - t.tc * kStations;
      if (jmax > kStations) jmax = kStations;
      if (t.tr == t.tc && il + 1 < jmax) jmax = il + 1;
      if (t.tr * kStations + il >= t.n) jmax = 0;
      uint32_t v[kTile / 32][32];
      tmem_ld128(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kTile), v);
      // Accumulator fully read: the MMA warp may reuse it.
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty0 + 8 * acc);
#pragma unroll
      for (int q = 0; q < kTile / 32; ++q) {
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          // Columns 4jj..4jj+3: (p2=0 re, p2=0 im, p2=1 re, p2=1 im) of station
          // j.  The real-row lane produces p2 = 0, the imaginary-row lane p2 = 1;
          // each needs two values from its partner lane.
          const int v0 = (int)v[q][4 * jj], v1 = (int)v[q][4 * jj + 1];
          const int v2 = (int)v[q][4 * jj + 2], v3 = (int)v[q][4 * jj + 3];
          const int ra = __shfl_xor_sync(0xffffffffu, c ? v0 : v2, 1);
          const int rb = __shfl_xor_sync(0xffffffffu, c ? v1 : v3, 1);
          const long long re = c ? (long long)ra + v3 : (long long)v0 + rb;
          const long long im = c ? (long long)v2 - rb : (long long)ra - v1;
          const int jl = q * 8 + jj;
          if (jl < jmax) *(longlong2 *)(srow + jl * 64) = make_longlong2(re, im);
        }
      }
      // Staging rows complete: hand them to the bulk-copy engine.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      epi_barrier();
      if (copier) {
        const int nb = row_bytes(t, lane);
        if (nb) {
          const uint32_t src = smem_u32(sstate + staging_row(lane));
          if (t.store) bulk_store(row_ptr(t, lane), src, nb);
          else bulk_reduce_add(row_ptr(t, lane), src, nb);
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      }
    }
    if (copier) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }

  __syncwarp();   // lanes 1-31 of the producer and MMA warps wait for lane 0
  if (p.overlap) pdl_wait();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

}  // namespace tc

// cuTensorMapEncodeTiled, resolved once through the runtime.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return nullptr;
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  return encode;
}

// {x: 4n bytes, y: f, z: t} over [t][f][s][p][c] int8 input with s.fin
// channels per sample (the map covers f of them); boxes of 128 bytes (32
// stations) x `rows` samples.
static int input_map(CUtensorMap *map, const void *dev_in, const Sizes &s, int rows,
                     CUtensorMapSwizzle swizzle) {
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return -1;
  if (((uintptr_t)dev_in & 15) != 0 || s.fin < s.f) return -2;
  cuuint64_t dims[3] = {(cuuint64_t)4 * s.n, (cuuint64_t)s.f, (cuuint64_t)s.t};
  cuuint64_t strides[2] = {(cuuint64_t)4 * s.n, (cuuint64_t)4 * s.n * s.fin};
  cuuint32_t box[3] = {(cuuint32_t)tc::kTile, 1, (cuuint32_t)rows};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(dev_in), dims,
                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -3;
}

int make_tc_tensor_map(CUtensorMap *map, const void *dev_in, const Sizes &s) {
  return input_map(map, dev_in, s, tc::kKt, CU_TENSOR_MAP_SWIZZLE_128B);
}

int make_panel_map(CUtensorMap *map, const void *dev_in, const Sizes &s, int rows) {
  return input_map(map, dev_in, s, rows, CU_TENSOR_MAP_SWIZZLE_NONE);
}

int make_packed_map(CUtensorMap *map, const void *dev_in, const Sizes &s) {
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return -1;
  if (((uintptr_t)dev_in & 15) != 0 || s.n % 8 != 0 || s.fin < s.f) return -2;
  cuuint64_t dims[3] = {(cuuint64_t)2 * s.n, (cuuint64_t)s.f, (cuuint64_t)s.t};
  cuuint64_t strides[2] = {(cuuint64_t)2 * s.n, (cuuint64_t)2 * s.n * s.fin};
  cuuint32_t box[3] = {(cuuint32_t)tc::kTile / 2, 1, (cuuint32_t)tc::kKt};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(dev_in), dims,
                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -3;
}

int current_device_sms() {
  static std::atomic<int> cache[kDeviceCache];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (dev >= 0 && dev < kDeviceCache) {
    const int n = cache[dev].load(std::memory_order_relaxed);
    if (n) return n;
  }
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (dev >= 0 && dev < kDeviceCache) cache[dev].store(n, std::memory_order_relaxed);
  return n;
}

// Both tcgen05 kernels use more than 48 KB of dynamic shared memory, which a
// kernel must be allowed on every device it runs on: set it once per device.
cudaError_t tc_configure_device() {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < kDeviceCache) ? 1ull << dev : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(tc::xengine_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           tc::kSmemBytes);
  if (e == cudaSuccess) e = tc2_set_smem_attribute();
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
  return e;
}

cudaError_t tc_check_device() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, tc::xengine_tc_kernel);
  if (e != cudaSuccess) return e;
  return tc_configure_device();
}

int tc_fill_job(Job *job, const void *dev_in, const Sizes &s, int t0, int tcount, int64_t *state,
                int store, int ksplit, int item_begin, int pair) {
  if (make_tc_tensor_map(&job->map, dev_in, s) != 0) return -1;
  const long long tile = pair ? 2 * tc::kTile : tc::kTile;
  const long long ntl = (4LL * s.n + tile - 1) / tile;
  const long long npairs = ntl * (ntl + 1) / 2;
  const int total_steps = (tcount + tc::kKt - 1) / tc::kKt;
  if (ksplit < 1) ksplit = 1;
  if (ksplit > total_steps) ksplit = total_steps;
  const int per = (total_steps + ksplit - 1) / ksplit;
  ksplit = (total_steps + per - 1) / per;   // every split non-empty
  if ((long long)s.f * npairs * ksplit + item_begin > 0x7fffffffLL) return -2;
  job->state = state;
  job->nbaseline = s.nbaseline;
  job->n = s.n;
  job->f = s.f;
  job->f0 = 0;
  job->t0 = t0;
  job->total_steps = total_steps;
  job->steps_per_split = per;
  job->ksplit = ksplit;
  job->npairs = (int)npairs;
  job->items = (int)(s.f * npairs * ksplit);
  job->item_begin = item_begin;
  job->store = (store && ksplit == 1) ? 1 : 0;
  return 0;
}

cudaError_t launch_tc(const CUtensorMap &map, const Sizes &s, int t0, int tcount, int64_t *state,
                      int overwrite, int *err, cudaStream_t st) {
  TcTuning tune;   // single CTAs, no time split, one CTA per SM
  return launch_tc_tuned(map, s, t0, tcount, state, overwrite, err, st, tune, 0);
}

cudaError_t launch_tc_tuned(const CUtensorMap &map, const Sizes &s, int t0, int tcount,
                            int64_t *state, int overwrite, int *err, cudaStream_t st,
                            const TcTuning &tune, int overlap, int f0, int fcount,
                            const void *packed_in, uint64_t *words, int words_store) {
  if (fcount < 0) fcount = s.f - f0;
  if (f0 < 0 || fcount < 1 || f0 + fcount > s.f) return cudaErrorInvalidValue;
  if (tune.wide)
    return launch_tc2(map, s, t0, tcount, state, overwrite, err, st, tune, overlap, f0, fcount,
                      packed_in, words, words_store);
  if (packed_in) return cudaErrorInvalidValue;   // only the CTA-pair kernel expands packed input
  const int sms = current_device_sms();
  if (!sms) return cudaErrorInvalidDevice;
  {
    const cudaError_t e = tc_configure_device();
    if (e != cudaSuccess) return e;
  }
  tc::Params p;
  p.single.map = map;
  // the map was encoded for `map`'s own buffer; fill the rest of the job
  Job &j = p.single;
  const long long ntl = (4LL * s.n + tc::kTile - 1) / tc::kTile;
  const long long npairs = ntl * (ntl + 1) / 2;
  const int total_steps = (tcount + tc::kKt - 1) / tc::kKt;
  int ksplit = tune.ksplit < 1 ? 1 : (tune.ksplit > total_steps ? total_steps : tune.ksplit);
  const int per = (total_steps + ksplit - 1) / ksplit;
  ksplit = (total_steps + per - 1) / per;
  if ((long long)fcount * npairs * ksplit > 0x7fffffffLL) return cudaErrorInvalidValue;
  // Split items of one tile all add into the buffer: a zero buffer must be
  // cleared first (its channel range) when it would otherwise be stored into.
  if (overwrite && ksplit > 1) {
    const size_t per_channel = (size_t)s.state_elems / s.f;   // int64 words
    cudaError_t e = cudaMemsetAsync(state + (size_t)f0 * per_channel, 0,
                                    (size_t)fcount * per_channel * 8, st);
    if (e != cudaSuccess) return e;
  }
  j.state = state;
  j.nbaseline = s.nbaseline;
  j.n = s.n;
  j.f = fcount;
  j.f0 = f0;
  j.t0 = t0;
  j.total_steps = total_steps;
  j.steps_per_split = per;
  j.ksplit = ksplit;
  j.npairs = (int)npairs;
  j.items = (int)(fcount * npairs * ksplit);
  j.item_begin = 0;
  j.store = (overwrite && ksplit == 1) ? 1 : 0;
  p.jobs = nullptr;
  p.njobs = 1;
  p.total = j.items;
  p.queue = nullptr;
  p.err = err;
  p.stall = tune.stall;
  // Stream-K only when every piece adds into existing sums (no stores).
  p.streamk = (tune.streamk && !j.store && ksplit == 1) ? 1 : 0;
  p.overlap = (overlap && !overwrite) ? 1 : 0;
  int grid = tune.grid > 0 ? tune.grid : sms;
  if (grid > p.total) grid = p.total;
  // Programmatic launch: this grid's prologue overlaps the previous kernel's
  // tail (the kernel waits for it before touching global memory).
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(tc::kThreads);
  cfg.dynamicSmemBytes = tc::kSmemBytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, tc::xengine_tc_kernel, p);
}

cudaError_t launch_tc_batch(const Job *dev_jobs, int njobs, int total_items, int *queue, int *err,
                            int grid, cudaStream_t st) {
  const int sms = current_device_sms();
  if (!sms) return cudaErrorInvalidDevice;
  cudaError_t e = tc_configure_device();
  if (e != cudaSuccess) return e;
  if (queue) {
    e = cudaMemsetAsync(queue, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
  }
  tc::Params p;
  memset(&p.single, 0, sizeof(p.single));
  p.jobs = dev_jobs;
  p.njobs = njobs;
  p.total = total_items;
  p.queue = queue;
  p.err = err;
  p.stall = 0;
  p.streamk = 0;
  p.overlap = 0;
  if (grid <= 0) grid = sms;
  if (grid > total_items) grid = total_items;
  if (grid < 1) return cudaSuccess;
  tc::xengine_tc_kernel<<<grid, tc::kThreads, tc::kSmemBytes, st>>>(p);
  return cudaGetLastError();
}

}  // namespace xgpu
