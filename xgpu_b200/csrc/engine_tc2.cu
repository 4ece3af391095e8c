// engine_tc2.cu -- tcgen05 int8 X-engine on CTA pairs (cta_group::2), 256x256
// tiles of the Gram matrix.
//
// Same arithmetic as engine_tc.cu (G = A A^T over the int8 input bytes of
// each sample, MN-major operands straight from HBM, re/im combined in int64
// when draining), with the tile doubled in both directions and shared by the
// two SMs of a cluster:
//   * the pair computes rows [256R, 256R+256) x columns [256C, 256C+256) of G
//     (64 x 64 stations) for one channel, R >= C;
//   * CTA r loads its own 128 rows of A (32 stations) and half r of the 256
//     columns of B into its shared memory; the leader CTA issues
//     tcgen05.mma.cta_group::2.kind::i8 with M = N = 256, which reads both
//     CTAs' halves, and each CTA's TMEM receives its 128 rows x 256 columns;
//   * per CTA and per 128 samples that is 32 KiB of loads for 128x256 output
//     columns -- half the bytes per MMA operation of the single-CTA kernel, so
//     the load pipeline's latency is covered with the same shared memory.
// Cross-CTA signalling: each CTA's TMA loads fill only its own shared memory
// and complete on the leader's "full" barrier (.cta_group::2 form, the peer's
// copy names the leader's barrier; only the leader registers the expected bytes, so the
// producers issue no cross-CTA fence), the leader's MMA commits once to each CTA's "empty" and
// "accumulator full" barriers, and the peer's epilogue arrives remotely on the
// leader's "accumulator empty" barrier.  Every wait is bounded (as in
// engine_tc.cu); both CTAs meet at a cluster barrier before releasing TMEM.
// Like engine_tc.cu the kernel is launched programmatically (an adding launch
// may run beside the previous one), and its epilogue has two schedules, joint
// and split per warp, chosen by the length of the launch's items.
// A second instantiation (kPacked) reads packed 4+4-bit input: each CTA's
// producer loads its packed boxes with TMA into a ring of packed slots, four
// converter warps expand every stage from there into an operand stage (the
// ring of operand stages is shorter, so that both rings fit), scaled by 16,
// and report it on the leader's "full" barrier; the drain divides the sums
// by 256.
#include <cudaTypedefs.h>
#include <string.h>

#include "internal.h"
#include "tc_common.cuh"
#include "tc_job.h"

namespace xgpu {
namespace tc2 {

using namespace tc;

constexpr int kHalf = 128;                  // G rows per CTA; B columns per CTA
// Items of at most this many pipeline stages use the split epilogue (their
// drains and copies outlast their MMAs); longer ones the joint one, which
// measured 3-10% faster there.
constexpr int kSplitEpilogueSteps = 8;
constexpr int kStations = kHalf / 4;        // 32 stations
constexpr int kKt = kTcSamplesPerStage;     // samples per pipeline stage
constexpr int kStages = 5;
constexpr int kSched = 4;
constexpr int kBoxBytes = kHalf * kKt;      // 16 KiB
constexpr int kStageBytes = 2 * kBoxBytes;  // A rows + B half
// Staging of one 32x32-station block of drained sums (staging_row).
constexpr int kStateBytes = kStagingBytes;
constexpr int kBarrierBytes = 512;    // barriers, work-item ring, TMEM slot
constexpr int kSmemBytes = kStages * kStageBytes + kStateBytes + kBarrierBytes + 1024;
static_assert(kSmemBytes <= 227 * 1024, "dynamic shared memory of one CTA");
constexpr uint32_t kAccCols = 2 * kHalf;    // 256 columns per accumulator
constexpr uint32_t kTmemCols = 2 * kAccCols;
constexpr int kThreads = 192;
constexpr uint32_t kIdesc = i8_idesc(2 * kHalf, 2 * kHalf);
// Word buffer (word mode): per channel, per 32 x 32-station block (rb >= cb,
// index rb(rb+1)/2 + cb) 4096 words, ordered (epilogue warp q: stations 8q ..
// 8q+7) x (baseline jl of the block's 32) x (station 8q + ilq) x (product).
constexpr int kWordsWarpBytes = 8 * kStations * 4 * 8;   // 8 KB
static_assert(4 * kWordsWarpBytes <= kStagingBytes, "word staging fits the staging area");
__host__ __device__ __forceinline__ long long word_offset(int f, long long nblk, int rb, int cb) {
  return ((long long)f * nblk + (long long)rb * (rb + 1) / 2 + cb) * 4096;
}
// Packed 4+4-bit input (one byte per complex sample, 2n bytes per sample):
// the producer loads each CTA's packed boxes (64 bytes per sample row: 32
// stations) with TMA into a ring of kPackedSlots slots of its own, and
// kConvWarps converter warps expand every stage from there into an operand
// ring of kStagesPacked stages -- the two rings take the shared memory of the
// int8 kernel's kStages stages.  Each converter warp owns 32 sample rows of
// both boxes of every stage, so a stage's expansion is spread over four warps
// and the packed loads run up to kPackedSlots stages ahead of it.
constexpr int kPackedRow = kStations * 2;                // 64 packed bytes per sample
constexpr int kPackedBox = kPackedRow * kKt;             // 8 KiB
constexpr int kPackedSlotBytes = 2 * kPackedBox;         // A and B boxes
constexpr int kStagesPacked = 3;
constexpr int kPackedSlots = 4;
static_assert(kStagesPacked * kStageBytes + kPackedSlots * kPackedSlotBytes <= kStages * kStageBytes,
              "the packed rings fit the int8 kernel's stages");
constexpr int kConvWarps = 4;
static_assert(kConvWarps * 32 == kKt, "32 sample rows per converter warp");
constexpr int kThreadsPacked = kThreads + 32 * kConvWarps;
// barriers (full/empty per stage, 2 x 2 accumulator, ring, mma_done, one
// spare), work-item ring, TMEM slot and abort flag; packed input adds its
// slots' loaded/free barriers and contents
static_assert((2 * kStages + 6 + 2 * kSched) * 8 + kSched * 64 + 8 <= kBarrierBytes, "barriers");
static_assert((2 * kStagesPacked + 6 + 2 * kSched) * 8 + kSched * 64 + 8 + kPackedSlots * 17 <=
                  kBarrierBytes,
              "barriers of the packed instantiation");

struct Params {
  Job job;             // the job when jobs == nullptr (npairs counts 256x256 tiles)
  const Job *jobs;     // batched: job table in global memory, ordered by item_begin
  int njobs;
  int total;           // work items over all jobs
  int *queue;          // dynamic work counter (zeroed before launch); nullptr: static stride
  int *err;
  int stall;           // test switch: issue no loads (the waits on them expire)
  int overlap;         // may run alongside the previous (accumulating) launch of the stream
  int split_epi;       // epilogue schedule: 0 joint, 1 split per warp
  // Word mode (single-job launches, split epilogue): the call's sums go to
  // this block-major word buffer instead of the int64 buffer (word_offset);
  // words_nblk = 32-station blocks per channel.  words_store: the launch
  // stores its words (one item per tile: each word has one writer) instead of
  // adding them.
  uint64_t *words;
  long long words_nblk;
  int words_store;
};

// A decoded work item, 64 bytes; the leader's scheduler writes it into both
// CTAs' rings.
struct Item {
  int u;               // >= total: no more work
  int f, R, C;         // channel and 256x256 tile (R >= C)
  int step0, nsteps;
  int n, store, t0, pad;
  long long nbaseline;
  int64_t *state;
  const CUtensorMap *map;
};
static_assert(sizeof(Item) == 64, "ring entries are copied as 8 words");

__device__ __forceinline__ Item decode_job(const Job &j, int u);

__device__ __forceinline__ Item decode(const Params &p, int u) {
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
  return decode_job(p.job, u);
}

__device__ __forceinline__ Item decode_job(const Job &j, int u) {
  Item it;
  it.u = u;
  const int v = u - j.item_begin;
  const int k = v % j.npairs;
  const int rest = v / j.npairs;
  const int split = rest % j.ksplit;
  it.f = j.f0 + rest / j.ksplit;
  int r = (int)((sqrtf(8.0f * (float)k + 1.0f) - 1.0f) * 0.5f);
  while (r * (r + 1) / 2 > k) --r;
  while ((r + 1) * (r + 2) / 2 <= k) ++r;
  it.R = r;
  it.C = k - r * (r + 1) / 2;
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

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(uint32_t local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}

__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

// Arrive on a barrier of either CTA of the pair (default semantics: no
// cluster-scope fence on the arriving thread).
__device__ __forceinline__ void remote_arrive(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}

// Arrive with cluster-scope release: shared-memory stores the thread made in
// the peer CTA before the arrival are visible to the peer's waiters.
__device__ __forceinline__ void remote_arrive_release(uint32_t cluster_bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar)
               : "memory");
}

__device__ __forceinline__ bool try_wait_cluster(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// mbar_wait with cluster-scope acquire, for entries the other CTA wrote.
__device__ __forceinline__ bool mbar_wait_cluster(uint32_t bar, uint32_t parity,
                                                  const volatile int *abort_flag) {
  if (try_wait_cluster(bar, parity)) return true;
  const uint64_t start = globaltimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (try_wait_cluster(bar, parity)) return true;
    if ((it & 63u) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (globaltimer_ns() - start > 2000000000ull) return false;
    }
  }
}

__device__ __forceinline__ void st_cluster_u64(uint32_t cluster_addr, uint64_t v) {
  asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(cluster_addr), "l"(v) : "memory");
}

__device__ __forceinline__ void tma_load_3d_pair(uint32_t dst, const CUtensorMap *map,
                                                 uint32_t cluster_bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(cluster_bar)
      : "memory");
}

__device__ __forceinline__ void mma_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

// Packed input: 4 packed samples (one word, real part in each byte's high
// nibble, imaginary part in its low nibble) -> 8 int8 bytes {re, im, ...},
// each 16 times the 4-bit two's-complement value: a nibble moved to (or left
// in) the high half of its byte is already that multiple, and |16 x 7| = 112
// fits int8.  The Gram sums then come out exactly 256 times too large, and the
// drain divides them back (unscale).
__device__ __forceinline__ uint2 expand_scaled(uint32_t w) {
  const uint32_t re = w & 0xF0F0F0F0u, im = (w << 4) & 0xF0F0F0F0u;
  return make_uint2(__byte_perm(re, im, 0x5140), __byte_perm(re, im, 0x7362));
}

template <bool kPacked>
__device__ __forceinline__ long long unscale(long long v) {
  return kPacked ? v >> 8 : v;   // exact: every packed-input sum is a multiple of 256
}

// A converter warp's share of one packed box in shared memory (64 bytes per
// sample row): rows r0 .. r0 + 31.  Lane l reads 16 bytes -- part m = l % 4 of
// row r0 + 8k + l / 4 -- in each of four loads k (each load reads eight whole
// rows: 512 contiguous bytes, conflict-free).
__device__ __forceinline__ void load_packed_rows(const uint8_t *pbox, int r0, int lane,
                                                 uint4 (&v)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k)
    v[k] = *(const uint4 *)(pbox + (r0 + 8 * k + (lane >> 2)) * kPackedRow + 16 * (lane & 3));
}

// Expands what load_packed_rows read into rows r0 .. r0 + 31 of a 16 KiB
// operand box: 128 int8 bytes per row in the 128-byte swizzled layout
// (16-byte chunk j of row r at r*128 + ((j ^ (r & 7)) << 4)).  Part m of a row
// becomes chunks 2m and 2m + 1.  A quarter-warp's eight lanes hold the four
// parts of two consecutive rows r (even) and r + 1: their even (odd) chunks
// land on complementary halves of the banks, so each store is conflict-free.
__device__ __forceinline__ void store_expanded_rows(uint8_t *box, int r0, int lane,
                                                    const uint4 (&v)[4]) {
  const int m = lane & 3;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = r0 + 8 * k + (lane >> 2);
    const uint2 e0 = expand_scaled(v[k].x), e1 = expand_scaled(v[k].y);
    const uint2 e2 = expand_scaled(v[k].z), e3 = expand_scaled(v[k].w);
    uint8_t *row = box + r * 128;
    *(uint4 *)(row + (((2 * m) ^ (r & 7)) << 4)) = make_uint4(e0.x, e0.y, e1.x, e1.y);
    *(uint4 *)(row + (((2 * m + 1) ^ (r & 7)) << 4)) = make_uint4(e2.x, e2.y, e3.x, e3.y);
  }
}

__device__ __forceinline__ void commit_pair(uint32_t cluster_bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   cluster_bar)
               : "memory");
}

template <bool kPacked>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPacked ? kThreadsPacked : kThreads, 1)
    xengine_tc2_kernel(const __grid_constant__ Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  // operand stages the MMA reads (packed input: the rest of the int8
  // kernel's stage memory holds the packed slots)
  constexpr int S = kPacked ? kStagesPacked : kStages;
  uint8_t *sstate = smem + kStages * kStageBytes;
  uint8_t *packed_slots = smem + S * kStageBytes;   // kPacked only
  uint64_t *bars = (uint64_t *)(sstate + kStateBytes);
  // full[S] empty[S] tfull[2] tempty[2] sfull[kSched] sempty[kSched] mma_done
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + S),
                 tfull0 = smem_u32(bars + 2 * S), tempty0 = smem_u32(bars + 2 * S + 2),
                 sfull0 = smem_u32(bars + 2 * S + 4),
                 sempty0 = smem_u32(bars + 2 * S + 4 + kSched),
                 mma_done = smem_u32(bars + 2 * S + 4 + 2 * kSched);
  Item *ring = (Item *)(bars + 2 * S + 6 + 2 * kSched);
  uint32_t *tmem_slot = (uint32_t *)(ring + kSched);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);
  // packed input: each slot's "loaded" barrier (the producer's TMA bytes) and
  // "free" barrier (every converter warp has read it), and its content
  // (0: A and B boxes, 1: A only (diagonal tile), -1: no more stages)
  const uint32_t praw0 = smem_u32(tmem_slot + 2), pfree0 = praw0 + 8 * kPackedSlots;
  volatile signed char *slot_info = (volatile signed char *)(tmem_slot + 2 + 4 * kPackedSlots);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = (rank == 0);
  const int cid = (int)(blockIdx.x >> 1), ncl = (int)(gridDim.x >> 1);

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      // int8 input: the leader's arrival, and both CTAs' loads complete on it;
      // packed input: every converter warp of both CTAs
      mbar_init(full0 + 8 * s, kPacked ? 2 * kConvWarps : 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    if (kPacked) {
      for (int q = 0; q < kPackedSlots; ++q) {
        mbar_init(praw0 + 8 * q, 1);
        mbar_init(pfree0 + 8 * q, kConvWarps);
      }
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(tfull0 + 8 * a, 1);
      mbar_init(tempty0 + 8 * a, 2 * kEpiThreads / 32);   // epilogue warps of both CTAs
    }
    for (int q = 0; q < kSched; ++q) {
      mbar_init(sfull0 + 8 * q, 1);
      // leader's ring slot is free once the leader's MMA issuer and epilogue
      // (each epilogue warp under the split schedule) and the peer's producer
      // and epilogue have copied the entry
      mbar_init(sempty0 + 8 * q, p.split_epi ? 2 + 2 * kEpiThreads / 32 : 4);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  cluster_sync();
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
    // The leader's lane takes the next item (queue or stride), decodes it once
    // and publishes it to both CTAs' rings; the peer's producer follows its ring.
    if (lane == 0) {
      if (!p.jobs && leader) asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&p.job.map) : "memory");
      uint32_t g = 0;
      bool ok = true;
      for (int i = 0; ok; ++i) {
        const int slot = i % kSched;
        Item t;
        if (leader) {
          if (i >= kSched && !mbar_wait(sempty0 + 8 * slot, ((i / kSched) - 1) & 1, abort_flag)) {
            fail(kErrTimeoutProducer);
            break;
          }
          const int u = p.queue ? atomicAdd(p.queue, 1) : cid + i * ncl;
          if (u < p.total) t = decode(p, u); else t.u = u;
          ring[slot] = t;
          const uint32_t remote = peer_addr(smem_u32(&ring[slot]), 1);
#pragma unroll
          for (int w = 0; w < 8; ++w) st_cluster_u64(remote + 8 * w, ((const uint64_t *)&t)[w]);
          mbar_arrive(sfull0 + 8 * slot);
          remote_arrive_release(peer_addr(sfull0 + 8 * slot, 1));
        } else {
          if (!mbar_wait_cluster(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag)) {
            fail(kErrTimeoutProducer);
            break;
          }
          t = ring[slot];
          remote_arrive(peer_addr(sempty0 + 8 * slot, 0));
        }
        if (t.u >= p.total) break;
        const bool diag = (t.R == t.C);
        const int rb = 2 * t.R + (int)rank, cbb = 2 * t.C + (int)rank;
        if (kPacked) {
          // this CTA's packed boxes into the next packed slot, for the
          // converter warps of this CTA
          for (int ks = 0; ks < t.nsteps; ++ks, ++g) {
            const uint32_t q = g % kPackedSlots;
            if (g >= (uint32_t)kPackedSlots &&
                !mbar_wait(pfree0 + 8 * q, ((g / kPackedSlots) - 1) & 1, abort_flag)) {
              fail(kErrTimeoutProducer);
              ok = false;
              break;
            }
            if (p.stall) continue;
            const uint32_t dst = smem_u32(packed_slots + q * kPackedSlotBytes);
            const int z = t.t0 + (t.step0 + ks) * kKt;
            slot_info[q] = diag ? 1 : 0;
            mbar_expect_tx(praw0 + 8 * q, diag ? kPackedBox : 2 * kPackedBox);
            tma_load_3d(dst, t.map, praw0 + 8 * q, rb * kPackedRow, t.f, z);
            if (!diag)
              tma_load_3d(dst + kPackedBox, t.map, praw0 + 8 * q, cbb * kPackedRow, t.f, z);
          }
        } else {
          for (int ks = 0; ks < t.nsteps; ++ks, ++g) {
            const uint32_t s = g % S;
            if (g >= (uint32_t)S &&
                !mbar_wait(empty0 + 8 * s, ((g / S) - 1) & 1, abort_flag)) {
              fail(kErrTimeoutProducer);
              ok = false;
              break;
            }
            if (p.stall) continue;
            const uint32_t dst = stage0 + s * kStageBytes;
            const int z = t.t0 + (t.step0 + ks) * kKt;
            const uint32_t fbar = peer_addr(full0 + 8 * s, 0);
            // The leader expects the bytes of both CTAs; the peer's loads may land
            // first (the transaction count then dips below zero until it does).
            if (leader) mbar_expect_tx(full0 + 8 * s, diag ? 2 * kBoxBytes : 4 * kBoxBytes);
            tma_load_3d_pair(dst, t.map, fbar, rb * kHalf, t.f, z);
            if (!diag) tma_load_3d_pair(dst + kBoxBytes, t.map, fbar, cbb * kHalf, t.f, z);
          }
        }
      }
      if (kPacked && ok && !p.stall) {
        // No stage follows: one slot says so to every converter warp.
        const uint32_t q = g % kPackedSlots;
        if (g < (uint32_t)kPackedSlots ||
            mbar_wait(pfree0 + 8 * q, ((g / kPackedSlots) - 1) & 1, abort_flag)) {
          slot_info[q] = -1;
          mbar_arrive(praw0 + 8 * q);
        } else {
          fail(kErrTimeoutProducer);
        }
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA --
    if (lane == 0 && leader) {
      uint32_t g = 0;
      bool ok = true;
      bool issued = false;
      for (int i = 0; ok; ++i) {
        const int slot = i % kSched;
        if (!mbar_wait(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag)) {
          fail(kErrTimeoutMma);
          break;
        }
        const Item t = ring[slot];
        mbar_arrive(sempty0 + 8 * slot);
        if (t.u >= p.total) break;
        const bool diag = (t.R == t.C);
        const int acc = i & 1;
        if (i >= 2 && !mbar_wait(tempty0 + 8 * acc, ((i >> 1) - 1) & 1, abort_flag)) {
          fail(kErrTimeoutMma);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(acc * kAccCols);
        for (int ks = 0; ks < t.nsteps; ++ks, ++g) {
          const uint32_t s = g % S;
          // packed input: both CTAs' converters arrived (the peer's from its CTA)
          if (!(kPacked ? mbar_wait_cluster(full0 + 8 * s, (g / S) & 1, abort_flag)
                        : mbar_wait(full0 + 8 * s, (g / S) & 1, abort_flag))) {
            fail(kErrTimeoutMma);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a = stage0 + s * kStageBytes;
          const uint32_t b = diag ? a : a + kBoxBytes;
#pragma unroll
          for (int kk = 0; kk < kKt / 32; ++kk)
            mma_pair(d, mn_sw128_desc(a + kk * 4096, kBoxBytes), mn_sw128_desc(b + kk * 4096, kBoxBytes),
                     (ks | kk) != 0 ? 1u : 0u);
          issued = true;
          commit_pair(peer_addr(empty0 + 8 * s, 0));
          commit_pair(peer_addr(empty0 + 8 * s, 1));
        }
        if (ok) {
          commit_pair(peer_addr(tfull0 + 8 * acc, 0));
          commit_pair(peer_addr(tfull0 + 8 * acc, 1));
        }
      }
      if (issued) {
        // Every MMA of the pair has completed once mma_done fires.
        commit_pair(peer_addr(mma_done, 0));
        mbar_wait(mma_done, 0, nullptr);
      }
    }
  } else if (!kPacked || warp < 6) {
    // ---------------------------------------------------------- epilogue --
    // Two schedules.  Joint: the four warps drain a column block, meet at a
    // barrier, and warp 0 hands all 32 staging rows to the bulk-copy engine.
    // Split (launches whose items are at most 8 pipeline stages, where the
    // drain and copies outlast the MMAs): each warp owns its 8 stations'
    // staging rows and its lanes 0-7 issue their copies, with no barrier
    // between warps, so one warp's copies overlap the others' drains.
    const int ew = warp - 2;
    const int quarter = warp & 3;            // TMEM lanes 32*quarter .. +31
    const int m = quarter * 32 + lane;
    const int c = m & 1;
    const int p1 = (m >> 1) & 1;
    const int il = m >> 2;
    if (!p.split_epi) {
      const bool copier = (ew == 0);
      for (int i = 0;; ++i) {
        const int slot = i % kSched;
        const bool got = leader ? mbar_wait(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag)
                                : mbar_wait_cluster(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag);
        Item t;
        if (got) t = ring[slot];
        if (copier) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        if (epi_any(!got)) {
          if (ew == 0 && lane == 0) fail(kErrTimeoutDrain);
          break;
        }
        if (ew == 0 && lane == 0) {
          if (leader) mbar_arrive(sempty0 + 8 * slot);
          else remote_arrive(peer_addr(sempty0 + 8 * slot, 0));
        }
        if (t.u >= p.total) break;
        const int acc = i & 1;
        const bool have = mbar_wait(tfull0 + 8 * acc, (i >> 1) & 1, abort_flag);
        if (epi_any(!have)) {
          if (ew == 0 && lane == 0) fail(kErrTimeoutDrain);
          break;
        }
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int rb = 2 * t.R + (int)rank;    // this CTA's 32-station row block
        const long long i_glob = (long long)rb * kStations + il;
        for (int h = 0; h < 2; ++h) {
          const int cb = 2 * t.C + h;          // 32-station column block
          if (cb > rb) continue;               // above the diagonal (uniform in the CTA)
          if (h == 1) {
            // the staging rows of column block 2C must have been read
            if (copier) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            epi_barrier();
          }
          uint8_t *srow = sstate + staging_row(il) + (p1 * 2 + c) * 16;
          int jmax = t.n - cb * kStations;
          if (jmax > kStations) jmax = kStations;
          if (cb == rb && il + 1 < jmax) jmax = il + 1;
          if (i_glob >= t.n) jmax = 0;
          uint32_t v[kHalf / 32][32];
          tmem_ld128(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kAccCols + h * kHalf),
                     v);
#pragma unroll
          for (int q = 0; q < kHalf / 32; ++q) {
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const int v0 = (int)v[q][4 * jj], v1 = (int)v[q][4 * jj + 1];
              const int v2 = (int)v[q][4 * jj + 2], v3 = (int)v[q][4 * jj + 3];
              const int ra = __shfl_xor_sync(0xffffffffu, c ? v0 : v2, 1);
              const int rb2 = __shfl_xor_sync(0xffffffffu, c ? v1 : v3, 1);
              const long long re = unscale<kPacked>(c ? (long long)ra + v3 : (long long)v0 + rb2);
              const long long im = unscale<kPacked>(c ? (long long)v2 - rb2 : (long long)ra - v1);
              const int jl = q * 8 + jj;
              if (jl < jmax) *(longlong2 *)(srow + jl * 64) = make_longlong2(re, im);
            }
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          epi_barrier();
          if (copier) {
            // row `lane` of the staging block -> baselines (32 rb + lane, 32 cb .. )
            const long long ig = (long long)rb * kStations + lane;
            int cnt = t.n - cb * kStations;
            if (cnt > kStations) cnt = kStations;
            if (cb == rb && lane + 1 < cnt) cnt = lane + 1;
            if (ig >= t.n) cnt = 0;
            if (cnt > 0) {
              int64_t *dst = t.state + ((long long)t.f * t.nbaseline + ig * (ig + 1) / 2 +
                                        (long long)cb * kStations) * 8;
              const uint32_t src = smem_u32(sstate + staging_row(lane));
              if (t.store) bulk_store(dst, src, cnt * 64);
              else bulk_reduce_add(dst, src, cnt * 64);
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        }
        // The accumulator has been read (or was not needed): release it.
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) remote_arrive(peer_addr(tempty0 + 8 * acc, 0));
      }
      if (copier) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    } else {
      const bool copier = lane < 8;          // copies staging row crow
      const int crow = quarter * 8 + lane;
      for (int i = 0;; ++i) {
        const int slot = i % kSched;
        const bool got = leader ? mbar_wait(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag)
                                : mbar_wait_cluster(sfull0 + 8 * slot, (i / kSched) & 1, abort_flag);
        if (!__all_sync(0xffffffffu, got)) {
          if (lane == 0) fail(kErrTimeoutDrain);
          break;
        }
        const Item t = ring[slot];
        __syncwarp();
        if (lane == 0) {                     // this warp has copied the entry
          if (leader) mbar_arrive(sempty0 + 8 * slot);
          else remote_arrive(peer_addr(sempty0 + 8 * slot, 0));
        }
        if (t.u >= p.total) break;
        const int acc = i & 1;
        if (!__all_sync(0xffffffffu, mbar_wait(tfull0 + 8 * acc, (i >> 1) & 1, abort_flag))) {
          if (lane == 0) fail(kErrTimeoutDrain);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int rb = 2 * t.R + (int)rank;
        const long long i_glob = (long long)rb * kStations + il;
        const int hlast = (2 * t.C + 1 > rb) ? 0 : 1;   // last column block at or below the diagonal
        for (int h = 0; h <= hlast; ++h) {
          const int cb = 2 * t.C + h;
          if (p.words) {
            // Word mode: each visibility's sums of this call as one 64-bit
            // word, im * 2^32 + re, staged as this warp's 8 KB of the block
            // (32 baselines x its 8 stations x 4 products: 32 consecutive
            // words per store) and added with one bulk reduce-add.
            uint32_t v[kHalf / 32][32];
            tmem_ld128(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kAccCols + h * kHalf),
                       v);
            if (h == hlast) {
              asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
              __syncwarp();
              if (lane == 0) remote_arrive(peer_addr(tempty0 + 8 * acc, 0));
            }
            // The second CTA of a pair tile that ends past the last station
            // holds a block with no stations: it has no place in the words
            // (its offset would be another block's).
            if (rb * kStations >= t.n) continue;
            // lane 0 committed this warp's previous copy: its staging is free
            // once that copy has read it
            if (copier) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            __syncwarp();
            uint64_t *wst = (uint64_t *)(sstate + quarter * kWordsWarpBytes);
#pragma unroll
            for (int q = 0; q < kHalf / 32; ++q) {
#pragma unroll
              for (int jj = 0; jj < 8; ++jj) {
                const int v0 = (int)v[q][4 * jj], v1 = (int)v[q][4 * jj + 1];
                const int v2 = (int)v[q][4 * jj + 2], v3 = (int)v[q][4 * jj + 3];
                const int ra = __shfl_xor_sync(0xffffffffu, c ? v0 : v2, 1);
                const int rb2 = __shfl_xor_sync(0xffffffffu, c ? v1 : v3, 1);
                const long long re = unscale<kPacked>(c ? (long long)ra + v3 : (long long)v0 + rb2);
                const long long im = unscale<kPacked>(c ? (long long)v2 - rb2 : (long long)ra - v1);
                wst[(q * 8 + jj) * 32 + lane] =
                    ((unsigned long long)im << 32) + (unsigned long long)re;
              }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
              uint64_t *dst = p.words + word_offset(t.f, p.words_nblk, rb, cb) + quarter * 1024;
              if (p.words_store) bulk_store(dst, smem_u32(wst), kWordsWarpBytes);
              else bulk_reduce_add(dst, smem_u32(wst), kWordsWarpBytes);
              asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            }
            continue;
          }
          uint8_t *srow = sstate + staging_row(il) + (p1 * 2 + c) * 16;
          int jmax = t.n - cb * kStations;
          if (jmax > kStations) jmax = kStations;
          if (cb == rb && il + 1 < jmax) jmax = il + 1;
          if (i_glob >= t.n) jmax = 0;
          uint32_t v[kHalf / 32][32];
          tmem_ld128(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kAccCols + h * kHalf),
                     v);
          if (h == hlast) {
            // The accumulator has been read: release it to the leader's MMA issuer.
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) remote_arrive(peer_addr(tempty0 + 8 * acc, 0));
          }
          // This warp's staging rows are free once its previous copies have read them.
          if (copier) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          __syncwarp();
#pragma unroll
          for (int q = 0; q < kHalf / 32; ++q) {
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const int v0 = (int)v[q][4 * jj], v1 = (int)v[q][4 * jj + 1];
              const int v2 = (int)v[q][4 * jj + 2], v3 = (int)v[q][4 * jj + 3];
              const int ra = __shfl_xor_sync(0xffffffffu, c ? v0 : v2, 1);
              const int rb2 = __shfl_xor_sync(0xffffffffu, c ? v1 : v3, 1);
              const long long re = unscale<kPacked>(c ? (long long)ra + v3 : (long long)v0 + rb2);
              const long long im = unscale<kPacked>(c ? (long long)v2 - rb2 : (long long)ra - v1);
              const int jl = q * 8 + jj;
              if (jl < jmax) *(longlong2 *)(srow + jl * 64) = make_longlong2(re, im);
            }
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (copier) {
            const long long ig = (long long)rb * kStations + crow;
            int cnt = t.n - cb * kStations;
            if (cnt > kStations) cnt = kStations;
            if (cb == rb && crow + 1 < cnt) cnt = crow + 1;
            if (ig >= t.n) cnt = 0;
            if (cnt > 0) {
              int64_t *dst = t.state + ((long long)t.f * t.nbaseline + ig * (ig + 1) / 2 +
                                        (long long)cb * kStations) * 8;
              const uint32_t src = smem_u32(sstate + staging_row(crow));
              if (t.store) bulk_store(dst, src, cnt * 64);
              else bulk_reduce_add(dst, src, cnt * 64);
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        }
      }
      if (copier) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
  } else {
    // -------------------------------------------------------- converters --
    // Packed input only.  Converter warp w expands sample rows 32w .. 32w + 31
    // of both boxes of every stage: it waits for the stage's packed slot and
    // for its operand stage to be free (the MMA has read it), expands its rows
    // into it, makes them visible to the tensor cores, reports on the leader's
    // "full" barrier and frees its share of the packed slot.
    const int r0 = (warp - 6) * 32;
    for (uint32_t g = 0;; ++g) {
      const uint32_t q = g % kPackedSlots;
      if (!__all_sync(0xffffffffu,
                      mbar_wait(praw0 + 8 * q, (g / kPackedSlots) & 1, abort_flag))) {
        if (lane == 0) fail(kErrTimeoutConvert);
        break;
      }
      const int info = slot_info[q];
      if (info < 0) break;
      const uint32_t s = g % S;
      if (g >= (uint32_t)S &&
          !__all_sync(0xffffffffu, mbar_wait(empty0 + 8 * s, ((g / S) - 1) & 1, abort_flag))) {
        if (lane == 0) fail(kErrTimeoutConvert);
        break;
      }
      const uint8_t *pk = packed_slots + q * kPackedSlotBytes;
      uint8_t *box = smem + s * kStageBytes;
      uint4 v[4];
      load_packed_rows(pk, r0, lane, v);
      store_expanded_rows(box, r0, lane, v);
      if (info == 0) {
        load_packed_rows(pk + kPackedBox, r0, lane, v);
        store_expanded_rows(box + kBoxBytes, r0, lane, v);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        if (leader) mbar_arrive(full0 + 8 * s);
        else remote_arrive(peer_addr(full0 + 8 * s, 0));
        mbar_arrive(pfree0 + 8 * q);
      }
    }
  }

  __syncwarp();   // lanes 1-31 of the producer and MMA warps wait for lane 0
  if (p.overlap) pdl_wait();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  cluster_sync();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// The fold: one CTA per quarter of a 32x32-station block of one channel
// (grid x = 4 * block within the channel's triangle of blocks + quarter q,
// y = channel): the quarter's 1024 words, rows 8q..8q+7 of the block, are 8 KB
// contiguous, [column jl][row ilq][product pp].  The CTA reads them with
// contiguous 16-byte loads into shared memory (columns padded to 36 words, so
// that the reads below take the minimum two wavefronts); warp ilq then adds
// its row's words, split into their int32 parts, to the row's 32 int64
// (re, im) pairs of each product -- or stores them there (store_state: the
// int64 buffer holds nothing yet) -- 2 KB contiguous, four 512-byte loads and
// stores per warp, all loads first.  Rows i < n, columns j <= i only (the
// block's other entries hold nothing).  Each int64 value has one writer.  The
// words are left as they are: the next launch that uses them stores its own
// (or they are cleared first).  Launched programmatically behind the engine
// launch that filled the words: it waits for that launch (and so for the
// chain before it) before touching memory, and lets the next launch start its
// prologue at once.
constexpr int kFoldColWords = 36;
__global__ void __launch_bounds__(256) fold_words_kernel(const uint64_t *__restrict__ words,
                                                         int64_t *__restrict__ state, int n,
                                                         long long nbaseline, int nblk,
                                                         int store_state) {
  __shared__ __align__(16) unsigned long long sw[32 * kFoldColWords];
  pdl_wait();
  pdl_trigger();
  const int k = blockIdx.x >> 2, f = blockIdx.y, q = blockIdx.x & 3;
  int rb = (int)((sqrtf(8.0f * (float)k + 1.0f) - 1.0f) * 0.5f);
  while (rb * (rb + 1) / 2 > k) --rb;
  while ((rb + 1) * (rb + 2) / 2 <= k) ++rb;
  const int cb = k - rb * (rb + 1) / 2;
  const ulonglong2 *src =
      reinterpret_cast<const ulonglong2 *>(words + ((long long)f * nblk + k) * 4096 + q * 1024);
  const int t = threadIdx.x;
  const ulonglong2 a0 = src[t], a1 = src[t + 256];   // words 2t, 2t+1 and 512 + 2t, 513 + 2t
  const int ilq = t >> 5, lane = t & 31;
  const long long i = (long long)rb * kStations + q * 8 + ilq;
  const bool row_live = i < n;
  const long long jbase = (long long)cb * kStations;
  longlong2 *d = reinterpret_cast<longlong2 *>(
      state + ((long long)f * nbaseline + (row_live ? i * (i + 1) / 2 : 0) + jbase) * 8);
  // lane's products: column r * 8 + lane / 4, product lane % 4, r = 0..3
  longlong2 acc[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    acc[r] = make_longlong2(0, 0);
    if (!store_state && row_live && jbase + r * 8 + (lane >> 2) <= i) acc[r] = d[r * 32 + lane];
  }
  {
    // word w = jl * 32 + ilq * 4 + pp goes to sw[jl * 36 + ilq * 4 + pp]
    const int w0 = 2 * t, w1 = 512 + 2 * t;
    *reinterpret_cast<ulonglong2 *>(&sw[(w0 >> 5) * kFoldColWords + (w0 & 31)]) = a0;
    *reinterpret_cast<ulonglong2 *>(&sw[(w1 >> 5) * kFoldColWords + (w1 & 31)]) = a1;
  }
  __syncthreads();
  if (!row_live) return;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int jl = r * 8 + (lane >> 2);
    if (jbase + jl > i) continue;
    const unsigned long long v = sw[jl * kFoldColWords + ilq * 4 + (lane & 3)];
    const long long re = (long long)(int)(uint32_t)v;                   // low part, signed
    const long long im = (long long)(v - (unsigned long long)re) >> 32;  // exact: |re| < 2^31
    acc[r].x += re;
    acc[r].y += im;
    d[r * 32 + lane] = acc[r];
  }
}

}  // namespace tc2

// Items of at most kSplitEpilogueSteps stages drain with the split epilogue,
// where the reduce-adds outlast the MMAs: those add words.  Longer items keep
// the joint epilogue and add into the int64 buffer.
bool tc2_uses_words(int tcount, const TcTuning &tune) {
  const int total_steps = (tcount + tc2::kKt - 1) / tc2::kKt;
  int ksplit = tune.ksplit < 1 ? 1 : (tune.ksplit > total_steps ? total_steps : tune.ksplit);
  const int per = (total_steps + ksplit - 1) / ksplit;
  return per <= tc2::kSplitEpilogueSteps;
}

bool tc2_single_item(int tcount, const TcTuning &tune) {
  const int total_steps = (tcount + tc2::kKt - 1) / tc2::kKt;
  int ksplit = tune.ksplit < 1 ? 1 : (tune.ksplit > total_steps ? total_steps : tune.ksplit);
  const int per = (total_steps + ksplit - 1) / ksplit;
  return (total_steps + per - 1) / per == 1;
}

long long words_blocks(const Sizes &s) {
  const long long nb = (s.n + tc2::kStations - 1) / tc2::kStations;
  return nb * (nb + 1) / 2;
}

long long words_elems(const Sizes &s) { return (long long)s.f * words_blocks(s) * 4096; }

cudaError_t launch_fold_words(const uint64_t *words, int64_t *state, const Sizes &s,
                              cudaStream_t st, int overlap, int store_state) {
  if (s.f > 65535) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(4 * words_blocks(s)), (unsigned)s.f);
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = overlap ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, tc2::fold_words_kernel, words, state, s.n, s.nbaseline,
                            (int)words_blocks(s), store_state);
}

cudaError_t tc2_set_smem_attribute() {
  cudaError_t e = cudaFuncSetAttribute(tc2::xengine_tc2_kernel<false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, tc2::kSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(tc2::xengine_tc2_kernel<true>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, tc2::kSmemBytes);
}

cudaError_t launch_tc2(const CUtensorMap &map, const Sizes &s, int t0, int tcount, int64_t *state,
                       int overwrite, int *err, cudaStream_t st, const TcTuning &tune, int overlap,
                       int f0, int fcount, const void *packed_in, uint64_t *words,
                       int words_store) {
  if (fcount < 0) fcount = s.f - f0;
  if (f0 < 0 || fcount < 1 || f0 + fcount > s.f) return cudaErrorInvalidValue;
  const bool packed = packed_in != nullptr;   // `map` describes it (make_packed_map)
  const int num_sms = current_device_sms();
  if (!num_sms) return cudaErrorInvalidDevice;
  {
    const cudaError_t e = tc_configure_device();
    if (e != cudaSuccess) return e;
  }
  tc2::Params p;
  Job &j = p.job;
  j.map = map;
  const long long ntl = (4LL * s.n + 2 * tc2::kHalf - 1) / (2 * tc2::kHalf);
  const long long npairs = ntl * (ntl + 1) / 2;
  const int total_steps = (tcount + tc2::kKt - 1) / tc2::kKt;
  int ksplit = tune.ksplit < 1 ? 1 : (tune.ksplit > total_steps ? total_steps : tune.ksplit);
  const int per = (total_steps + ksplit - 1) / ksplit;
  ksplit = (total_steps + per - 1) / per;
  if ((long long)fcount * npairs * ksplit > 0x7fffffffLL) return cudaErrorInvalidValue;
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
  p.queue = nullptr;
  p.total = j.items;
  p.err = err;
  p.stall = tune.stall;
  // word mode: launches of short items (tc2_uses_words), split epilogue; a
  // launch that stores its words has one item per tile and overlaps nothing
  p.words = (!overwrite && per <= tc2::kSplitEpilogueSteps) ? words : nullptr;
  p.words_nblk = words_blocks(s);
  p.words_store = (p.words && words_store) ? 1 : 0;
  if (p.words_store && ksplit > 1) return cudaErrorInvalidValue;
  p.overlap = (overlap && !overwrite && !p.words_store) ? 1 : 0;
  p.split_epi = (p.words || per <= tc2::kSplitEpilogueSteps) ? 1 : 0;
  int clusters = (tune.grid > 0 ? tune.grid : num_sms) / 2;
  if (clusters > p.total) clusters = p.total;
  if (clusters < 1) clusters = 1;
  // Programmatic launch: this grid's prologue overlaps the previous kernel's
  // tail (the kernel waits for it before touching global memory).
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(2 * clusters));
  cfg.blockDim = dim3(packed ? tc2::kThreadsPacked : tc2::kThreads);
  cfg.dynamicSmemBytes = tc2::kSmemBytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return packed ? cudaLaunchKernelEx(&cfg, tc2::xengine_tc2_kernel<true>, p)
                : cudaLaunchKernelEx(&cfg, tc2::xengine_tc2_kernel<false>, p);
}

cudaError_t launch_tc2_batch(const Job *dev_jobs, int njobs, int total_items, int *queue, int *err,
                             int grid, cudaStream_t st, int max_item_steps) {
  const int sms = current_device_sms();
  if (!sms) return cudaErrorInvalidDevice;
  cudaError_t e = tc_configure_device();
  if (e != cudaSuccess) return e;
  if (queue) {
    e = cudaMemsetAsync(queue, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
  }
  tc2::Params p;
  memset(&p.job, 0, sizeof(p.job));
  p.jobs = dev_jobs;
  p.njobs = njobs;
  p.total = total_items;
  p.queue = queue;
  p.err = err;
  p.stall = 0;
  p.overlap = 0;
  p.words = nullptr;
  p.words_nblk = 0;
  p.words_store = 0;
  p.split_epi = max_item_steps <= tc2::kSplitEpilogueSteps ? 1 : 0;
  int clusters = (grid > 0 ? grid : sms) / 2;
  if (clusters > total_items) clusters = total_items;
  if (clusters < 1) return cudaSuccess;
  tc2::xengine_tc2_kernel<false><<<2 * clusters, tc2::kThreads, tc2::kSmemBytes, st>>>(p);
  return cudaGetLastError();
}

}  // namespace xgpu
