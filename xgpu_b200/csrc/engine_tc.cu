// engine_tc.cu -- tcgen05 int8 tensor-core X-engine.
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
// One CTA computes one 128x128 tile of G (32 stations x 2 pols x re/im on each
// side) for one channel; only tiles on or below the diagonal are issued.
//   warp 0 lane 0 : TMA producer, 3-D tiled loads with 128-byte swizzle
//   warp 1 lane 0 : MMA issuer, tcgen05.mma.cta_group::1.kind::i8, M=N=128,
//                   K=32 per instruction, accumulator in TMEM (128 columns)
//   all 4 warps   : drain TMEM -> registers (tcgen05.ld 32x32b), combine the
//                   re/im rows of each input with two warp shuffles, and add
//                   into the int64 triangular integration buffer.
// Every wait on an mbarrier is bounded; a timeout writes an error code and the
// kernel still releases its TMEM and returns.
#include <cudaTypedefs.h>

#include "internal.h"

namespace xgpu {
namespace tc {

constexpr int kTile = 128;                 // G rows (and columns) per tile
constexpr int kStations = kTile / 4;       // 32 stations per tile side
constexpr int kKt = 128;                   // samples per pipeline stage
constexpr int kStages = 3;
constexpr int kBoxBytes = kTile * kKt;     // one operand of one stage: 16 KiB
constexpr int kStageBytes = 2 * kBoxBytes;
constexpr int kBarrierBytes = 256;
constexpr int kSmemBytes = kStages * kStageBytes + kBarrierBytes + 1024;  // + alignment slack
constexpr uint32_t kTmemCols = 128;
constexpr int kThreads = 128;

// Instruction descriptor (tcgen05 .kind::i8): D s32, A and B signed 8-bit,
// both MN-major, N = 128 (bits 17-22, >>3), M = 128 (bits 24-28, >>4).
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                            ((uint32_t)(kTile >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);

// Shared-memory matrix descriptor for an MN-major operand with 128-byte
// swizzle: one swizzle atom is 8 samples x 128 bytes (1024 B), atoms follow
// each other along K (the sample axis) every 1024 bytes (stride byte offset).
// The leading byte offset would step to a second 128-byte block along M/N; a
// 128-wide operand has only one, so it is set to the distance it would have.
__device__ __forceinline__ uint64_t mn_sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((kBoxBytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version for tcgen05
  d |= (uint64_t)2 << 61;   // SWIZZLE_128B
  return d;
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

// Wait for the phase with the given parity to complete; false after ~2 s.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t start = globaltimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0 && globaltimer_ns() - start > 2000000000ull) return false;
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

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
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
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct Params {
  int n, f;
  int t0;          // first sample of this launch
  int nsteps;      // pipeline stages of kKt samples
  int ntiles;      // tiles per side = ceil(4n / 128)
  long long nbaseline;
  int64_t *state;
  int overwrite;
  int *err;
};

__global__ void __launch_bounds__(kThreads, 1)
    xengine_tc_kernel(const __grid_constant__ CUtensorMap map, const Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *bars = (uint64_t *)(smem + kStages * kStageBytes);
  uint32_t *tmem_slot = (uint32_t *)(bars + 2 * kStages + 1);
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages),
                 done_bar = smem_u32(bars + 2 * kStages);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // Work item: channel and lower-triangle tile (tr >= tc).
  const int npairs = p.ntiles * (p.ntiles + 1) / 2;
  const int f = blockIdx.x / npairs;
  const int k = blockIdx.x - f * npairs;
  int tr = (int)((sqrtf(8.0f * (float)k + 1.0f) - 1.0f) * 0.5f);
  while (tr * (tr + 1) / 2 > k) --tr;
  while ((tr + 1) * (tr + 2) / 2 <= k) ++tr;
  const int tcol = k - tr * (tr + 1) / 2;
  const bool diag = (tr == tcol);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t stage0 = smem_u32(smem);

  if (warp == 0 && lane == 0) {
    // Producer: stage s holds the row panel at +0 and the column panel at
    // +kBoxBytes (diagonal tiles load one panel and use it for both).
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&map) : "memory");
    for (int ks = 0; ks < p.nsteps; ++ks) {
      const int s = ks % kStages;
      if (ks >= kStages && !mbar_wait(empty0 + 8 * s, ((ks / kStages) - 1) & 1)) {
        atomicExch(p.err, kErrTimeoutProducer);
        break;
      }
      const uint32_t dst = stage0 + s * kStageBytes;
      mbar_expect_tx(full0 + 8 * s, diag ? kBoxBytes : 2 * kBoxBytes);
      const int z = p.t0 + ks * kKt;
      tma_load_3d(dst, &map, full0 + 8 * s, tr * kTile, f, z);
      if (!diag) tma_load_3d(dst + kBoxBytes, &map, full0 + 8 * s, tcol * kTile, f, z);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer.
    bool ok = true;
    for (int ks = 0; ks < p.nsteps; ++ks) {
      const int s = ks % kStages;
      if (!mbar_wait(full0 + 8 * s, (ks / kStages) & 1)) {
        atomicExch(p.err, kErrTimeoutMma);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a = stage0 + s * kStageBytes;
      const uint32_t b = diag ? a : a + kBoxBytes;
#pragma unroll
      for (int kk = 0; kk < kKt / 32; ++kk) {
        // 32 samples = 4 swizzle atoms = 4096 bytes per instruction.
        mma_i8(tmem, mn_sw128_desc(a + kk * 4096), mn_sw128_desc(b + kk * 4096),
               (ks | kk) != 0 ? 1u : 0u);
      }
      mma_commit(empty0 + 8 * s);
    }
    if (ok) mma_commit(done_bar);
  }
  __syncwarp();

  // Epilogue: warp w owns TMEM lanes (= G rows) 32w .. 32w+31.
  const bool have = mbar_wait(done_bar, 0);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!have) {
    if (lane == 0) atomicExch(p.err, kErrTimeoutDrain);
  } else {
    const int m = warp * 32 + lane;
    const int c = m & 1;               // 0: real row, 1: imaginary row
    const int p1 = (m >> 1) & 1;
    const int i = tr * kStations + (m >> 2);
    const long long row_base = (long long)f * p.nbaseline + (long long)i * (i + 1) / 2;
#pragma unroll 1
    for (int q = 0; q < kTile / 32; ++q) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * 32), v);
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        // Columns 4jj..4jj+3 of this chunk: (p2=0 re, p2=0 im, p2=1 re, p2=1 im)
        // of station j.  The real-row lane produces p2 = 0, the imaginary-row
        // lane p2 = 1; each needs two values from its partner lane.
        const int v0 = (int)v[4 * jj], v1 = (int)v[4 * jj + 1];
        const int v2 = (int)v[4 * jj + 2], v3 = (int)v[4 * jj + 3];
        const int ra = __shfl_xor_sync(0xffffffffu, c ? v0 : v2, 1);
        const int rb = __shfl_xor_sync(0xffffffffu, c ? v1 : v3, 1);
        const long long re = c ? (long long)ra + v3 : (long long)v0 + rb;
        const long long im = c ? (long long)v2 - rb : (long long)ra - v1;
        const int j = tcol * kStations + q * 8 + jj;
        if (i < p.n && j < p.n && j <= i) {
          longlong2 *dst = (longlong2 *)(p.state + ((row_base + j) * 4 + p1 * 2 + c) * 2);
          if (p.overwrite) {
            *dst = make_longlong2(re, im);
          } else {
            longlong2 o = *dst;
            o.x += re;
            o.y += im;
            *dst = o;
          }
        }
      }
    }
  }

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

}  // namespace tc

int make_tc_tensor_map(CUtensorMap *map, const void *dev_in, const Sizes &s) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return -1;
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  if (((uintptr_t)dev_in & 15) != 0) return -2;
  cuuint64_t dims[3] = {(cuuint64_t)4 * s.n, (cuuint64_t)s.f, (cuuint64_t)s.t};
  cuuint64_t strides[2] = {(cuuint64_t)4 * s.n, (cuuint64_t)4 * s.n * s.f};
  cuuint32_t box[3] = {(cuuint32_t)tc::kTile, 1, (cuuint32_t)tc::kKt};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(dev_in), dims,
                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -3;
}

cudaError_t tc_check_device() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, tc::xengine_tc_kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(tc::xengine_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              tc::kSmemBytes);
}

cudaError_t launch_tc(const CUtensorMap &map, const Sizes &s, int t0, int tcount, int64_t *state,
                      int overwrite, int *err, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(
        tc::xengine_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  tc::Params p;
  p.n = s.n;
  p.f = s.f;
  p.t0 = t0;
  p.nsteps = (tcount + tc::kKt - 1) / tc::kKt;
  p.ntiles = (4 * s.n + tc::kTile - 1) / tc::kTile;
  p.nbaseline = s.nbaseline;
  p.state = state;
  p.overwrite = overwrite;
  p.err = err;
  const long long grid = (long long)s.f * p.ntiles * (p.ntiles + 1) / 2;
  tc::xengine_tc_kernel<<<(unsigned)grid, tc::kThreads, tc::kSmemBytes, st>>>(map, p);
  return cudaGetLastError();
}

}  // namespace xgpu
