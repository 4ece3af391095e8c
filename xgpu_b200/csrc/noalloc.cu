// noalloc.cu -- xgpuCorrelateStatic: one correlation that allocates nothing.
//
// Some callers cannot call cudaMalloc at the point where they correlate: a
// real-time capture thread that must never block (cudaMalloc and cudaFree
// can synchronise the whole device and stall every other stream), or a
// plugin inside a host framework that owns all device memory and forbids
// allocations of its own.  They hand in their input and output buffers; the
// only other memory this path needs -- the int64 integration buffer between
// the tensor-core engine and the output formatting -- lives in the
// file-scope array below.
//
// The array is kNoAllocScratchBytes (32 MiB) of device memory that every GPU
// which loads libxgpu.so holds until the process exits.  Its first 256 bytes
// hold the kernels' error word; the rest holds the integration buffer,
// 64 * F * N(N+1)/2 bytes, which therefore limits F * N(N+1)/2 to
// 524,284 (e.g. N=256 with F <= 15, N=512 with F <= 3).
//
// All calls share the array and it keeps the last call's contents.  The
// engine stores (does not add) every element of the integration buffer that
// the formatting reads, so nothing has to start at zero except the error
// word, which each call clears.  Calls whose work overlaps on the GPU (two
// host threads, or two streams) race on the array and give wrong results:
// serialise them.
//
// In host code `g_noalloc_scratch` is only a host-side stand-in for the
// device array: its device address comes from cudaGetSymbolAddress, taken
// once per device with that device current, on the first call made on that
// device, and kept for the life of the process (a cudaDeviceReset of that
// device invalidates it: make no call on a device after resetting it).
// Because that first call does this set-up, make it before any stream
// capture begins.
//
// Every call waits for its own work (cudaStreamSynchronize) and reads the
// error word back into host memory.  The caller's current device is the same
// after the call as before.
#include <string.h>

#include <mutex>

#include "internal.h"

using namespace xgpu;

namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr size_t kErrBytes = 256;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (current); nullptr on error.
void *scratch_on(int device) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      fprintf(stderr, "xgpuCorrelateStatic: cudaGetSymbolAddress failed: %s\n",
              cudaGetErrorString(e));
      return nullptr;
    }
    g_scratch_addr[device] = p;
  }
  return g_scratch_addr[device];
}

int correlate_static(const void *device_input, void *device_output, const XGPUConfig &c,
                     const Sizes &s, int device, void *stream);

}  // namespace

extern "C" int xgpuCorrelateStatic(const void *device_input, void *device_output,
                                   const XGPUConfig *cfg, int device, void *stream) {
  if (!device_input || !device_output || !cfg) return XGPU_INVALID_ARGUMENT;
  if (((uintptr_t)device_input & 15) != 0 || ((uintptr_t)device_output & 7) != 0)
    return XGPU_INVALID_ARGUMENT;
  if (device < 0 || device >= kMaxDevices) return XGPU_INVALID_ARGUMENT;
  XGPUConfig c = *cfg;
  if (c.engine == XGPU_ENGINE_DEFAULT) c.engine = XGPU_ENGINE_TENSOR;
  // xgpuInitEx's ranges (sample count included), then this path's own limits:
  // the tensor-core engine on int8 input covering the whole buffer
  if (!validate_config(c)) return XGPU_INVALID_ARGUMENT;
  if (c.compute_type != XGPU_INT8 || c.input_format != XGPU_INPUT_INT8 ||
      c.engine != XGPU_ENGINE_TENSOR || c.channel_offset != 0 ||
      (c.input_nfrequency != 0 && c.input_nfrequency != c.nfrequency))
    return XGPU_INVALID_ARGUMENT;

  const Sizes s = make_sizes(c);
  const size_t state_bytes = (size_t)s.state_elems * sizeof(int64_t);
  if (state_bytes > kNoAllocScratchBytes - kErrBytes) {
    fprintf(stderr,
            "xgpuCorrelateStatic: integration buffer of %zu bytes (N=%u, F=%u) exceeds the "
            "static maximum of %zu bytes\n",
            state_bytes, c.nstation, c.nfrequency, kNoAllocScratchBytes - kErrBytes);
    return XGPU_INVALID_ARGUMENT;
  }

  int caller_device = 0;
  if (cudaGetDevice(&caller_device) != cudaSuccess) return XGPU_CUDA_ERROR;
  if (cudaSetDevice(device) != cudaSuccess) return XGPU_CUDA_ERROR;
  const int rc = correlate_static(device_input, device_output, c, s, device, stream);
  cudaSetDevice(caller_device);
  return rc;
}

namespace {

// The body of xgpuCorrelateStatic with `device` current.
int correlate_static(const void *device_input, void *device_output, const XGPUConfig &c,
                     const Sizes &s, int device, void *stream) {
  unsigned char *base = (unsigned char *)scratch_on(device);
  if (!base) return XGPU_CUDA_ERROR;
  int *err = (int *)base;
  int64_t *state = (int64_t *)(base + kErrBytes);
  cudaStream_t st = (cudaStream_t)stream;

  CUtensorMap map;
  if (make_tc_tensor_map(&map, device_input, s) != 0) return XGPU_INVALID_ARGUMENT;
  if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return XGPU_CUDA_ERROR;
  // The kernel a context starts with (it cannot autotune here: that takes
  // scratch buffers): CTA pairs from 384 stations on, single CTAs below, one
  // CTA per SM, no time splits.
  TcTuning tune;
  tune.wide = c.nstation >= 384 ? 1 : 0;
  for (int t0 = 0; t0 < s.t; t0 += kSegment) {
    const int tc = s.t - t0 < kSegment ? s.t - t0 : kSegment;
    if (launch_tc_tuned(map, s, t0, tc, state, t0 == 0 ? 1 : 0, err, st, tune, 0) != cudaSuccess)
      return XGPU_CUDA_ERROR;
  }
  if (launch_format(state, 0, s, (int)c.matrix_order, (int)c.output_type, device_output, st) !=
      cudaSuccess)
    return XGPU_CUDA_ERROR;
  int h_err = 0;
  if (cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return XGPU_CUDA_ERROR;
  if (h_err != 0) {
    fprintf(stderr, "xgpuCorrelateStatic: device wait timed out (code %d)\n", h_err);
    return XGPU_CUDA_ERROR;
  }
  return XGPU_OK;
}

}  // namespace
