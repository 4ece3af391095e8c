// peak.cu -- CUDA-core throughput of the plain engines' arithmetic, measured
// on the device: the denominators of the dp4a and FP32 engines' rooflines.
//
// Every thread runs 8 independent chains of one instruction (dp4a or FP32
// FMA), each step taking the chain's previous value as a multiplicand, so no
// step can be folded into another and the register-resident loop issues
// nothing but the measured instruction (plus one loop branch per 128).  The
// grid fills every SM to 2048 threads.
#include <cuda_runtime.h>

#include "internal.h"

namespace xgpu {
namespace peak {

constexpr int kThreads = 256;
constexpr int kChains = 8;
constexpr int kUnroll = 16;   // steps per chain per loop iteration

__global__ void __launch_bounds__(kThreads) dp4a_peak_kernel(int iters, int seed, int *sink) {
  int acc[kChains], b[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) {
    acc[k] = seed + (int)threadIdx.x * kChains + k;
    b[k] = (int)(0x01010101u * (unsigned)(k + 1)) ^ (int)blockIdx.x;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int k = 0; k < kChains; ++k) acc[k] = __dp4a(acc[k], b[k], acc[k]);
  }
  int s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s ^= acc[k];
  if (s == 0x7fffffff) sink[0] = s;   // keeps the chains live; practically never taken
}

__global__ void __launch_bounds__(kThreads) fma_peak_kernel(int iters, int seed, int *sink) {
  float acc[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) acc[k] = (float)(seed + (int)threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int k = 0; k < kChains; ++k) acc[k] = fmaf(acc[k], 0.999f, 0.001f);   // tends to 1
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += acc[k];
  if (s == -1.f) sink[0] = 1;   // keeps the chains live; never taken
}

}  // namespace peak
}  // namespace xgpu

using namespace xgpu;

#define PEAK_CHECK(call)                                   \
  do {                                                     \
    if ((call) != cudaSuccess) {                           \
      cudaGetLastError();                                  \
      code = XGPU_CUDA_ERROR;                              \
      goto done;                                           \
    }                                                      \
  } while (0)

extern "C" int xgpuMeasureCorePeak(int device, int kind, double *ops_per_second) {
  if (!ops_per_second || kind < 0 || kind > 1) return XGPU_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return XGPU_CUDA_ERROR;
  }
  int code = XGPU_OK, sms = 0;
  int *sink = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = 0.f;
  int iters = 64;
  PEAK_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  PEAK_CHECK(cudaMalloc(&sink, sizeof(int)));
  PEAK_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  PEAK_CHECK(cudaEventCreate(&e0));
  PEAK_CHECK(cudaEventCreate(&e1));
  {
    const dim3 grid((unsigned)(sms * (2048 / peak::kThreads)));
    // Grow the loop count until one launch runs for at least 20 ms (at most
    // eight launches; each one's duration is bounded by its loop count).
    for (int round = 0; round < 8; ++round) {
      PEAK_CHECK(cudaEventRecord(e0, st));
      if (kind == 0)
        peak::dp4a_peak_kernel<<<grid, peak::kThreads, 0, st>>>(iters, 12345, sink);
      else
        peak::fma_peak_kernel<<<grid, peak::kThreads, 0, st>>>(iters, 12345, sink);
      PEAK_CHECK(cudaGetLastError());
      PEAK_CHECK(cudaEventRecord(e1, st));
      PEAK_CHECK(cudaEventSynchronize(e1));
      PEAK_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      if (ms >= 20.f || iters >= (1 << 24)) break;
      const double want = 25.0 / (ms > 0.01f ? ms : 0.01f) * iters;
      iters = want > (double)(1 << 24) ? (1 << 24) : (int)want;
    }
    const double instr = (double)grid.x * peak::kThreads * peak::kChains * peak::kUnroll * iters;
    // X-engine operations per instruction: a dp4a is four int8 products and
    // their sum (8), an FMA a product and a sum (2).
    *ops_per_second = instr * (kind == 0 ? 8.0 : 2.0) / (ms * 1e-3);
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (sink) cudaFree(sink);
  return code;
}
