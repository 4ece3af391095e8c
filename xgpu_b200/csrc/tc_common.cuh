// tc_common.cuh -- PTX wrappers shared by the tensor-core kernels: shared
// memory descriptors, mbarriers with bounded waits, TMA and bulk copies,
// tcgen05 MMA / commit / TMEM loads, and the epilogue's named barrier.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace xgpu {
namespace tc {

// Shared-memory matrix descriptor for an MN-major operand with 128-byte
// swizzle: one swizzle atom is 8 samples x 128 bytes (1024 B), atoms follow
// each other along K (the sample axis) every 1024 bytes (stride byte offset).
// lbo is the distance to the next 128-byte block along M/N (unused by a
// 128-wide operand, which has only one).
__device__ __forceinline__ uint64_t mn_sw128_desc(uint32_t saddr, uint32_t lbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for tcgen05
  d |= (uint64_t)2 << 61;   // SWIZZLE_128B
  return d;
}

// Instruction descriptor of tcgen05 .kind::i8: D s32, A and B signed 8-bit,
// both MN-major, N (bits 17-22, >>3), M (bits 24-28, >>4).
constexpr uint32_t i8_idesc(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity to complete.  Gives up (false)
// after ~2 s, or as soon as another role raised the CTA's abort flag when
// abort_flag is given (teardown waits pass nullptr and only time out).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          const volatile int *abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t start = globaltimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (globaltimer_ns() - start > 2000000000ull) return false;
    }
  }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void bulk_store(void *dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_reduce_add(void *dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.u64 [%0], [%1], %2;" ::"l"(
                   dst),
               "r"(src), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

// tcgen05.ld of 32 columns x 32 lanes (one register per column) without the
// wait; tmem_ld_wait below completes it.
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
        "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
        "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// Ties the registers of an earlier tmem_ld32_async to a point after
// tcgen05.wait::ld, so the compiler cannot move their uses above the wait.
__device__ __forceinline__ void tmem_regs_after_wait(uint32_t (&v)[32]) {
  asm volatile(""
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                 "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                 "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]),
                 "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]),
                 "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]),
                 "+r"(v[30]), "+r"(v[31])
               :
               : "memory");
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Four 32-column loads in flight, one wait: 128 columns of this warp's lanes.
__device__ __forceinline__ void tmem_ld128(uint32_t taddr, uint32_t (&v)[4][32]) {
  tmem_ld32_async(taddr, v[0]);
  tmem_ld32_async(taddr + 32, v[1]);
  tmem_ld32_async(taddr + 64, v[2]);
  tmem_ld32_async(taddr + 96, v[3]);
  tmem_ld_wait();
  tmem_regs_after_wait(v[0]);
  tmem_regs_after_wait(v[1]);
  tmem_regs_after_wait(v[2]);
  tmem_regs_after_wait(v[3]);
}

// Programmatic dependent launch.  pdl_trigger lets the next kernel of the
// stream start its prologue now; pdl_wait blocks until the previous kernel of
// the stream (when this one was launched programmatically) has completed and
// its memory is visible.  Both are no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}


constexpr int kEpiThreads = 128;   // four epilogue warps, one per TMEM lane quarter

// Staging of drained sums: one 2 KB row per station of a 32-station block (32
// baselines x 4 polarisation products x int64 (re, im)), handed row by row to
// the bulk-copy engine.  An epilogue warp's 16-byte stores reach two stations'
// rows per quarter-warp (stations 2a and 2a + 1, one baseline, 64 bytes each).
// Rows go in pairs of 4160 bytes, the odd row 2112 bytes after the even one:
// 64 bytes apart in the banks, so the two segments fall on disjoint halves.
__device__ __forceinline__ int staging_row(int il) { return (il >> 1) * 4160 + (il & 1) * 2112; }
constexpr int kStagingBytes = 16 * 4160;

__device__ __forceinline__ void epi_barrier() {
  asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory");
}

// Barrier over the epilogue warps that also returns whether any of their
// threads passed v = true, so they all take the same branch afterwards.
__device__ __forceinline__ bool epi_any(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(kEpiThreads)
      : "memory");
  return r != 0;
}


}  // namespace tc
}  // namespace xgpu
