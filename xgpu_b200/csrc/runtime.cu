// runtime.cu -- the xgpu.h C ABI: contexts, host buffers, the per-call
// pipeline and dumps.
//
// Counterpart of xGPU's src/cuda_xengine.cu (host side).  Differences by
// design:
//  * sizes are per context (xgpuInitEx) with the build's defaults for
//    xgpuInit; all state lives in the context, so contexts are re-entrant
//    (xGPU keeps textures as file-scope globals, cuda_xengine.cu:73-87);
//  * a call copies its whole input with one host-to-device transfer into one
//    of two device buffers and runs one engine launch over all its samples
//    (xGPU launches once per NTIME_PIPE chunk and re-reads/writes the whole
//    integration buffer each time, cuda_xengine.cu:599-653).  Consecutive
//    calls still overlap: the transfer of call k+1 runs while call k computes;
//  * the integer engines integrate into an int64 buffer, converted to the
//    caller's Complex type and matrix order on the device at dump time;
//  * xgpuClearDeviceIntegrationBuffer is lazy: the next engine launch stores
//    instead of adding, so a cleared buffer is never read.
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <mutex>
#include <new>

#include "internal.h"

#ifndef NSTATION
#define NSTATION 256
#endif
#ifndef NFREQUENCY
#define NFREQUENCY 10
#endif
#ifndef NTIME
#define NTIME 1024
#endif
#ifndef NTIME_PIPE
#define NTIME_PIPE 128
#endif
#if defined MATRIX_ORDER_TRIANGULAR
#define XGPU_DEFAULT_ORDER TRIANGULAR_ORDER
#elif defined MATRIX_ORDER_REAL_IMAG
#define XGPU_DEFAULT_ORDER REAL_IMAG_TRIANGULAR_ORDER
#else
#define XGPU_DEFAULT_ORDER REGISTER_TILE_TRIANGULAR_ORDER
#endif
#ifdef DP4A
#define XGPU_DEFAULT_OUTPUT XGPU_INT32
#else
#define XGPU_DEFAULT_OUTPUT XGPU_FLOAT32
#endif
#ifndef XGPU_VERSION
#define XGPU_VERSION "xgpu-b200-1.0"
#endif

using namespace xgpu;

namespace {

// Channel groups of a dumping call with host buffers (see the note at
// dump_call_grouped): at most this many, each at least kGroupMinBytes of input.
constexpr int kMaxGroups = 8;
constexpr long long kGroupMinBytes = 1 << 20;

struct Internal {
  int device = 0;
  XGPUConfig cfg{};
  Sizes sz{};    // the context's sizes; input geometry of the caller's full-band device input
  Sizes szc{};   // the same for a compact copy of this context's channels (d_in, d_conv)
  bool int_state = true;  // int64 buffer (integer engines) or float (FP32)

  void *d_in[2] = {nullptr, nullptr};  // one call's input, as supplied
  // Packed 4+4-bit (unless the CTA-pair kernel expands it itself:
  // packed_in_kernel), DP4A-swizzled and block-32 input is converted to int8
  // [t][f][s][p][c] on its own stream into one of two buffers, so the
  // conversion of call k+1 is queued without waiting for the engine of call
  // k (measured: the two kernels seldom share the SMs, so a converted call
  // costs its conversion plus its engine launch).
  int8_t *d_conv[2] = {nullptr, nullptr};
  cudaStream_t s_conv = nullptr;
  cudaEvent_t conv_done[2] = {nullptr, nullptr};
  cudaEvent_t conv_free[2] = {nullptr, nullptr};   // engine that read d_conv[k] finished
  bool conv_used[2] = {false, false};
  int conv_cur = 0;
  cudaEvent_t caller_ev = nullptr;                 // orders caller-stream work before a conversion
  // A context of a channel range with a converted format gathers its channels
  // of device-resident input here (on s_conv) before converting them.
  void *d_slice = nullptr;
  void *d_state = nullptr;             // integration buffer
  // Launches of the CTA-pair kernel with short items put their sums into
  // this word buffer (one 64-bit word per visibility, im * 2^32 + re: half
  // the bytes of the int64 buffer's pairs); a fold moves the words into
  // d_state before it is read and before more than kWordsMaxSamples samples
  // have gone in.  nullptr: no word buffer (it could not be allocated, or
  // another engine).
  uint64_t *d_words = nullptr;
  long long words_samples = 0;         // samples in the words since the last fold
  bool words_dirty = false;            // the words hold sums not yet in d_state
  bool words_stale = false;            // the words hold nothing, but are not zero
  void *d_out = nullptr;               // formatted dump
  int *d_err = nullptr;                // device error word
  int *h_err = nullptr;                // pinned copy of it

  cudaStream_t s_copy = nullptr, s_comp = nullptr;
  cudaStream_t s_own = nullptr;  // the context's own compute stream
  // A dumping call over host buffers moves its channels in groups: group k+1
  // goes host-to-device while group k's results go device-to-host on s_dump
  // (the two directions' copy engines run at once).
  cudaStream_t s_dump = nullptr;
  cudaEvent_t group_in[kMaxGroups + 2] = {};    // a group's input is on the device
  cudaEvent_t group_out[kMaxGroups + 2] = {};   // a group's sums (or formatted results) are ready
  cudaEvent_t copy_done[2] = {nullptr, nullptr};
  cudaEvent_t comp_done[2] = {nullptr, nullptr};
  int cur = 0;
  bool state_zero = true;
  TcTuning tune;   // tensor-core kernel, time splits and grid
  // The last operation queued on s_comp is an engine launch that only added
  // into the integration buffer (no store), on the context's own stream: the
  // next accumulating launch over other input may overlap it.
  bool adding_tail = false;

  // tensor maps, cached by device pointer: enough entries for a pipeline
  // that rotates over a ring of input buffers (a miss costs a host-side
  // encode per call); replaced round-robin
  static constexpr int kMaps = 16;
  struct MapEntry {
    const void *ptr;
    bool packed;     // packed 4+4-bit geometry (make_packed_map)
    int fin;         // channels per sample of the buffer
    CUtensorMap map;
  } maps[kMaps];
  int nmaps = 0;
  int next_map = 0;   // the entry a miss replaces once all are in use

  ComplexInput *free_array_h = nullptr, *unregister_array_h = nullptr;
  bool array_h_set = false, register_host_array = true;
  Complex *free_matrix_h = nullptr, *unregister_matrix_h = nullptr;
  bool matrix_h_set = false, register_host_matrix = true;
};

const long kPageSize = sysconf(_SC_PAGE_SIZE);

#define XGPU_CHECK(call)                                                               \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "(CUDA) %s (%s:%d)\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return XGPU_CUDA_ERROR;                                                          \
    }                                                                                  \
  } while (0)

Internal *get(XGPUContext *c) { return c ? (Internal *)c->internal : nullptr; }

XGPUConfig default_config() {
  XGPUConfig c;
  c.nstation = NSTATION;
  c.nfrequency = NFREQUENCY;
  c.ntime = NTIME;
  c.ntimepipe = NTIME_PIPE;
  c.compute_type = XGPU_INT8;
  c.output_type = XGPU_DEFAULT_OUTPUT;
  c.matrix_order = XGPU_DEFAULT_ORDER;
  c.engine = XGPU_ENGINE_TENSOR;
  c.input_format = XGPU_INPUT_INT8;
  c.channel_offset = 0;
  c.input_nfrequency = 0;
  return c;
}

void fill_info(const XGPUConfig &c, const Sizes &s, XGPUInfo *info) {
  info->npol = kNpol;
  info->nstation = c.nstation;
  info->nbaseline = (unsigned)s.nbaseline;
  info->nfrequency = c.nfrequency;
  info->ntime = c.ntime;
  info->ntimepipe = c.ntimepipe;
  info->input_type = XGPU_INT8;
  info->compute_type = c.compute_type;
  // the caller's input holds the whole band (s.fband channels)
  info->vecLength = (unsigned long long)s.t * s.fband * s.n * kNpol;
  info->vecLengthPipe = (unsigned long long)s.fband * c.ntimepipe * c.nstation * kNpol;
  info->matLength = (unsigned long long)s.mat_length;
  info->triLength = (unsigned long long)s.tri_length;
  info->matrix_order = c.matrix_order;
  info->shared_atomic_size = 4;
  info->complex_block_size = c.input_format == XGPU_INPUT_BLOCK32 ? 32 : 1;
}

int free_device(Internal *in) {
  cudaSetDevice(in->device);
  if (in->s_copy) cudaStreamSynchronize(in->s_copy);
  if (in->s_comp) cudaStreamSynchronize(in->s_comp);
  for (int b = 0; b < 2; ++b) {
    if (in->copy_done[b]) cudaEventDestroy(in->copy_done[b]);
    if (in->comp_done[b]) cudaEventDestroy(in->comp_done[b]);
    if (in->d_in[b]) cudaFree(in->d_in[b]);
  }
  if (in->s_copy) cudaStreamDestroy(in->s_copy);
  if (in->s_own) cudaStreamDestroy(in->s_own);
  if (in->s_dump) {
    cudaStreamSynchronize(in->s_dump);
    cudaStreamDestroy(in->s_dump);
  }
  for (int k = 0; k < kMaxGroups + 2; ++k) {
    if (in->group_in[k]) cudaEventDestroy(in->group_in[k]);
    if (in->group_out[k]) cudaEventDestroy(in->group_out[k]);
  }
  for (int k = 0; k < 2; ++k) {
    if (in->d_conv[k]) cudaFree(in->d_conv[k]);
    if (in->conv_done[k]) cudaEventDestroy(in->conv_done[k]);
    if (in->conv_free[k]) cudaEventDestroy(in->conv_free[k]);
  }
  if (in->s_conv) {
    cudaStreamSynchronize(in->s_conv);
    cudaStreamDestroy(in->s_conv);
  }
  if (in->caller_ev) cudaEventDestroy(in->caller_ev);
  if (in->d_slice) cudaFree(in->d_slice);
  if (in->d_state) cudaFree(in->d_state);
  if (in->d_words) cudaFree(in->d_words);
  if (in->d_out) cudaFree(in->d_out);
  if (in->d_err) cudaFree(in->d_err);
  if (in->h_err) cudaFreeHost(in->h_err);
  return XGPU_OK;
}

// Register caller memory page-rounded, as cuda_xengine.cu:386-412 does.
// Memory the caller pinned already (cudaHostAlloc or its own registration) is
// accepted as it is when both ends of the range are pinned; a range that
// shares pages with other registered memory fails, as in xGPU.
cudaError_t register_range(void *p, size_t bytes, void **registered) {
  uintptr_t a = (uintptr_t)p, base = a - (a % kPageSize);
  size_t len = bytes + (a - base);
  len = (len + kPageSize - 1) / kPageSize * kPageSize;
  *registered = nullptr;
  cudaError_t e = cudaHostRegister((void *)base, len, cudaHostRegisterDefault);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {
    cudaGetLastError();
    unsigned int fl;
    if (bytes > 0 && cudaHostGetFlags(&fl, p) == cudaSuccess &&
        cudaHostGetFlags(&fl, (char *)p + bytes - 1) == cudaSuccess)
      return cudaSuccess;
    cudaGetLastError();
    return e;
  }
  if (e == cudaSuccess) *registered = (void *)base;
  return e;
}

// Tensor map over input at ptr with geometry g (g.fin channels per sample).
const CUtensorMap *tensor_map(Internal *in, const void *ptr, const Sizes &g, bool packed = false) {
  for (int q = 0; q < in->nmaps; ++q)
    if (in->maps[q].ptr == ptr && in->maps[q].packed == packed && in->maps[q].fin == g.fin)
      return &in->maps[q].map;
  int slot;
  if (in->nmaps < Internal::kMaps) {
    slot = in->nmaps++;
  } else {
    slot = in->next_map;
    in->next_map = (in->next_map + 1) % Internal::kMaps;
  }
  const int r = packed ? make_packed_map(&in->maps[slot].map, ptr, g)
                       : make_tc_tensor_map(&in->maps[slot].map, ptr, g);
  if (r != 0) {
    in->maps[slot].ptr = nullptr;
    return nullptr;
  }
  in->maps[slot].ptr = ptr;
  in->maps[slot].packed = packed;
  in->maps[slot].fin = g.fin;
  return &in->maps[slot].map;
}

// Packed 4+4-bit input goes straight to the CTA-pair kernel, which expands it
// in shared memory; other kernels (and engines) read it converted to int8 by a
// pre-pass.
bool packed_in_kernel(const Internal *in) {
  return in->cfg.input_format == XGPU_INPUT_PACKED4 && in->int_state &&
         in->cfg.engine == XGPU_ENGINE_TENSOR && in->tune.wide;
}

// Queue the engine over channels [f0, f0 + fcount) of int8 input x (packed
// input when `packed`: packed_in_kernel) on s_comp, in time segments; the
// first segment stores when the buffer is known to be zero.  x has geometry s
// (in->szc for the context's compact buffers, in->sz for a full-band device
// input read in place, x then pointing at the context's first channel).
// Add the words into the int64 buffer (and zero them), on s_comp after
// everything queued there: before the buffer is read, and before the words
// would hold more than kWordsMaxSamples samples.  after_adding: the last
// launch on s_comp is an adding engine launch of this context, which the fold
// may then start beside (it waits for it before touching memory).  The next
// engine launch does not overlap the fold; it only starts its prologue early.
int fold_words(Internal *in, bool after_adding = false) {
  if (!in->words_dirty) return XGPU_OK;
  // an integration held only in the words is stored into d_state
  XGPU_CHECK(launch_fold_words(in->d_words, (int64_t *)in->d_state, in->szc, in->s_comp,
                               after_adding && in->s_comp == in->s_own ? 1 : 0,
                               in->state_zero ? 1 : 0));
  in->state_zero = false;
  in->words_dirty = false;
  in->words_stale = true;
  in->words_samples = 0;
  in->adding_tail = false;
  return XGPU_OK;
}

// *tail: in, the launch may overlap the adding launch before it; out, the
// last launch queued only added.  allow_words: launches of the CTA-pair
// kernel with short items may put their sums into the word buffer.  The first
// launch into the int64 buffer while it holds nothing (state_zero) stores;
// *wrote_state (if given) tells whether any launch went there, after which
// the caller clears state_zero.
int launch_engine(Internal *in, const int8_t *x, const Sizes &s, int f0, int fcount, bool *tail,
                  bool packed = false, bool allow_words = true, bool *wrote_state = nullptr) {
  if (wrote_state) *wrote_state = true;
  const int ow = in->state_zero ? 1 : 0;
  if (!in->int_state) {
    XGPU_CHECK(launch_plain_fp32(x, s, 0, s.t, (float *)in->d_state, ow, in->s_comp, in->d_err,
                                 in->tune.stall, f0, fcount));
  } else if (in->cfg.engine == XGPU_ENGINE_PLAIN) {
    for (int t0 = 0; t0 < s.t; t0 += kSegment) {
      const int tc = s.t - t0 < kSegment ? s.t - t0 : kSegment;
      const int store = ow && t0 == 0;
      XGPU_CHECK(launch_plain_dp4a(x, s, t0, tc, (int64_t *)in->d_state, store, in->s_comp,
                                   in->d_err, in->tune.stall, f0, fcount,
                                   *tail && !store ? 1 : 0));
      *tail = !store;   // the next segment follows an adding launch
    }
  } else {
    const CUtensorMap *map = tensor_map(in, x, s, packed);
    if (!map) {
      fprintf(stderr, "xgpu: cannot describe the input buffer to the tensor memory accelerator\n");
      return XGPU_CUDA_ERROR;
    }
    bool state_written = false;
    for (int t0 = 0; t0 < s.t; t0 += kSegment) {
      const int tc = s.t - t0 < kSegment ? s.t - t0 : kSegment;
      const bool words = allow_words && in->d_words && in->tune.wide && tc2_uses_words(tc, in->tune);
      if (!words) {
        const int store = in->state_zero && !state_written ? 1 : 0;
        XGPU_CHECK(launch_tc_tuned(*map, s, t0, tc, (int64_t *)in->d_state, store, in->d_err,
                                   in->s_comp, in->tune, *tail && !store ? 1 : 0, f0, fcount,
                                   packed ? (const void *)x : nullptr));
        state_written = true;
        *tail = !store;   // the next segment follows an adding launch
        continue;
      }
      if (in->words_samples + tc > kWordsMaxSamples) {
        const int r = fold_words(in, *tail);
        if (r != XGPU_OK) return r;
        *tail = false;
      }
      // Words that hold nothing are overwritten by a launch with one item per
      // tile; a launch with time splits adds, into words cleared first.
      int wstore = 0;
      if (!in->words_dirty) {
        if (tc2_single_item(tc, in->tune)) {
          wstore = 1;
        } else if (in->words_stale) {
          XGPU_CHECK(cudaMemsetAsync(in->d_words, 0, (size_t)words_elems(in->szc) * 8, in->s_comp));
          *tail = false;
        }
      }
      XGPU_CHECK(launch_tc_tuned(*map, s, t0, tc, (int64_t *)in->d_state, 0, in->d_err, in->s_comp,
                                 in->tune, *tail && !wstore ? 1 : 0, f0, fcount,
                                 packed ? (const void *)x : nullptr, in->d_words, wstore));
      in->words_samples += tc;
      in->words_dirty = true;
      in->words_stale = false;
      *tail = !wstore;   // the next segment may overlap only a launch that added
    }
    if (wrote_state) *wrote_state = state_written;
  }
  return XGPU_OK;
}

// Queue the engine over one call's device input (any format) on s_comp.
// input_ready, when given, is the event after which the input is complete
// (the host-to-device copy); converted formats wait for it on s_conv.
// compact: d_input holds only this context's channels (the copy the host path
// makes); otherwise it is the caller's full-band input, read in place (int8,
// or packed input the CTA-pair kernel expands) or gathered into d_slice
// before its conversion (the other formats).
int run_engine(Internal *in, const void *d_input, cudaEvent_t input_ready, bool compact) {
  const Sizes &s = in->sz;
  const bool ranged = !compact && s.fin != s.f;
  const int8_t *x = (const int8_t *)d_input;
  const Sizes *geom = &in->szc;
  int conv = -1;
  // Overlap with the previous launch only when nothing else sits between them
  // on the stream (no conversion, no copy to wait for) and that launch only
  // added into the buffer.
  const bool packed = packed_in_kernel(in);
  bool tail = in->adding_tail && in->s_comp == in->s_own && !input_ready &&
              (in->cfg.input_format == XGPU_INPUT_INT8 || packed);
  in->adding_tail = false;
  if (in->cfg.input_format != XGPU_INPUT_INT8 && !packed) {
    conv = in->conv_cur;
    in->conv_cur ^= 1;
    if (in->conv_used[conv]) XGPU_CHECK(cudaStreamWaitEvent(in->s_conv, in->conv_free[conv], 0));
    if (input_ready) XGPU_CHECK(cudaStreamWaitEvent(in->s_conv, input_ready, 0));
    if (in->s_comp != in->s_own) {
      // The caller's stream may have produced the input: convert after it.
      XGPU_CHECK(cudaEventRecord(in->caller_ev, in->s_comp));
      XGPU_CHECK(cudaStreamWaitEvent(in->s_conv, in->caller_ev, 0));
    }
    const void *src = d_input;
    if (ranged) {
      // this context's channels of every row of the band, gathered in order
      XGPU_CHECK(cudaMemcpy2DAsync(in->d_slice, (size_t)(s.f * s.chan_bytes),
                                   (const char *)d_input + s.fin0 * s.chan_bytes,
                                   (size_t)(s.fband * s.chan_bytes), (size_t)(s.f * s.chan_bytes),
                                   (size_t)s.rows, cudaMemcpyDeviceToDevice, in->s_conv));
      src = in->d_slice;
    }
    if (in->cfg.input_format == XGPU_INPUT_PACKED4)
      XGPU_CHECK(launch_unpack4((const uint8_t *)src, in->d_conv[conv], s.vec_length, in->s_conv));
    else if (in->cfg.input_format == XGPU_INPUT_BLOCK32)
      XGPU_CHECK(launch_unblock32((const int8_t *)src, in->d_conv[conv], 2 * s.vec_length,
                                  in->s_conv));
    else
      XGPU_CHECK(launch_unswizzle_dp4a((const int8_t *)src, in->d_conv[conv], in->szc, in->s_conv));
    XGPU_CHECK(cudaEventRecord(in->conv_done[conv], in->s_conv));
    XGPU_CHECK(cudaStreamWaitEvent(in->s_comp, in->conv_done[conv], 0));
    x = in->d_conv[conv];
  } else {
    if (input_ready) XGPU_CHECK(cudaStreamWaitEvent(in->s_comp, input_ready, 0));
    if (ranged) {
      x += s.fin0 * s.chan_bytes;   // the maps step the band's fin channels per sample
      geom = &in->sz;
    }
  }
  bool wrote_state = true;
  const int r = launch_engine(in, x, *geom, 0, s.f, &tail, packed, true, &wrote_state);
  if (r != XGPU_OK) return r;
  if (in->int_state) in->adding_tail = tail && conv < 0;   // tensor or dp4a engine
  if (wrote_state) in->state_zero = false;   // otherwise the call went to the words
  if (conv >= 0) {
    XGPU_CHECK(cudaEventRecord(in->conv_free[conv], in->s_comp));
    in->conv_used[conv] = true;
  }
  return XGPU_OK;
}

// Read and clear the device error word.
// Queued on `st` (default s_comp), which must be the stream whose completion
// implies every engine launch's: the read and the wait are one round trip.
int check_device_error(Internal *in, cudaStream_t st = nullptr) {
  in->adding_tail = false;
  if (!st) st = in->s_comp;
  XGPU_CHECK(cudaMemcpyAsync(in->h_err, in->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  XGPU_CHECK(cudaStreamSynchronize(st));
  if (*in->h_err != 0) {
    fprintf(stderr, "xgpu: device wait timed out (code %d); results of this integration are invalid\n",
            *in->h_err);
    XGPU_CHECK(cudaMemsetAsync(in->d_err, 0, sizeof(int), in->s_comp));
    XGPU_CHECK(cudaStreamSynchronize(in->s_comp));
    return XGPU_CUDA_ERROR;
  }
  return XGPU_OK;
}

// The device address of the caller's output (the host buffer at
// output_offset) when the formatting kernel can store the dump straight into
// it: triangular and real-imag orders, whose words the kernel writes in runs,
// into page-locked memory the device maps, 8-byte aligned.  Those stores
// cross the host link at the rate of a copy.  Otherwise nullptr: the dump is
// formatted in device memory and copied.
void *direct_output(XGPUContext *ctx, Internal *in) {
  if (in->cfg.matrix_order == REGISTER_TILE_TRIANGULAR_ORDER) return nullptr;
  void *p = nullptr;
  if (cudaHostGetDevicePointer(&p, ctx->matrix_h + ctx->output_offset, 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return ((uintptr_t)p & 7) == 0 ? p : nullptr;
}

int dump(XGPUContext *ctx, Internal *in) {
  const bool after_adding = in->adding_tail;
  in->adding_tail = false;
  if (!in->matrix_h_set || !ctx->matrix_h) return XGPU_HOST_BUFFER_NOT_SET;
  if (ctx->matrix_len && ctx->output_offset + (size_t)in->sz.mat_length > ctx->matrix_len)
    return XGPU_INVALID_ARGUMENT;
  {
    const int r = fold_words(in, after_adding);
    if (r != XGPU_OK) return r;
  }
  if (in->state_zero) {
    XGPU_CHECK(cudaMemsetAsync(in->d_state, 0, (size_t)in->sz.state_elems * (in->int_state ? 8 : 4),
                               in->s_comp));
  }
  void *direct = direct_output(ctx, in);
  XGPU_CHECK(launch_format(in->d_state, in->int_state ? 0 : 1, in->sz, in->cfg.matrix_order,
                           in->cfg.output_type, direct ? direct : in->d_out, in->s_comp));
  if (!direct)
    XGPU_CHECK(cudaMemcpyAsync(ctx->matrix_h + ctx->output_offset, in->d_out,
                               (size_t)in->sz.mat_length * sizeof(Complex),
                               cudaMemcpyDeviceToHost, in->s_comp));
  return check_device_error(in);   // waits for the formatting and the copy too
}

// Channel groups for a dumping call over host buffers, 0 when the call goes
// whole: int8 input, or packed input that the CTA-pair kernel expands (a
// converted format is converted in one pass), at least two groups of
// kGroupMinBytes, an output buffer that takes the dump.
int dump_groups(XGPUContext *ctx, Internal *in) {
  const Sizes &s = in->sz;
  if ((in->cfg.input_format != XGPU_INPUT_INT8 && !packed_in_kernel(in)) || s.f < 2) return 0;
  if (!in->matrix_h_set || !ctx->matrix_h) return 0;
  if (ctx->matrix_len && ctx->output_offset + (size_t)s.mat_length > ctx->matrix_len) return 0;
  long long g = s.input_bytes / kGroupMinBytes;
  if (g > kMaxGroups) g = kMaxGroups;
  if (g > s.f) g = s.f;
  if (g < 2) return 0;
  const int per = (int)((s.f + g - 1) / g);
  return (s.f + per - 1) / per;
}

// xgpuCudaXengine(SYNCOP_DUMP) over host buffers, channel group by channel
// group, on three streams: each group's channels go host-to-device on s_copy
// (one 2-D copy: ntime rows of the group's stations), through the engine on
// s_comp, and through the formatting, which stores either straight into the
// caller's output on s_dump (direct_output; the engine of group k+1 then runs
// beside the formatting of group k, on other channels of the buffer) or into
// device memory on s_comp, copied device-to-host on s_dump.  The input of
// later groups crosses the host link while the results of earlier ones cross
// it the other way.  The input copies are all queued before the first
// device-to-host copy, which may block the host when the output buffer is
// pageable.  Results are the same as the whole call's: each channel's sums
// see the same samples in the same order.
int dump_call_grouped(XGPUContext *ctx, Internal *in, int b, int groups) {
  const Sizes &s = in->sz;
  const int per = (s.f + groups - 1) / groups;
  const bool packed = packed_in_kernel(in);
  // bytes of one channel at one sample: {re, im} bytes, or one packed byte,
  // per station and polarisation; the host rows hold the whole band, the
  // device copy this context's channels
  const size_t row = (size_t)s.chan_bytes;
  const size_t pitch = row * s.f, src_pitch = row * s.fband;
  const char *src = (const char *)(ctx->array_h + ctx->input_offset) + (size_t)s.fin0 * row;
  int8_t *dst = (int8_t *)in->d_in[b];
  in->adding_tail = false;
  // Channel boundaries: the first and last groups hold half as many channels
  // (at least one) as the others, so the first input copy and the last
  // results -- the stretches in which only one direction of the host link
  // is busy -- are short.  At most groups + 2 groups (2 <= 2 * half <= per
  // <= f / 2).
  int bound[kMaxGroups + 4];
  int ng = 0;
  {
    const int half = per > 1 ? per / 2 : 1;
    const int last0 = s.f - half;   // first channel of the last group
    int f = half;
    bound[0] = 0;
    bound[++ng] = f;
    while (f < last0) {
      f = f + per < last0 ? f + per : last0;
      bound[++ng] = f;
    }
    bound[++ng] = s.f;
  }
  // Earlier calls' words go into the int64 buffer first: each group's
  // results are formatted from it right after the group's own launch, which
  // adds there directly.
  {
    const int r = fold_words(in);
    if (r != XGPU_OK) return r;
  }
  // The buffer is free once the engine launch that last read it has finished.
  XGPU_CHECK(cudaStreamWaitEvent(in->s_copy, in->comp_done[b], 0));
  for (int k = 0; k < ng; ++k) {
    const int f0 = bound[k], fc = bound[k + 1] - bound[k];
    XGPU_CHECK(cudaMemcpy2DAsync(dst + f0 * row, pitch, src + f0 * row, src_pitch, fc * row,
                                 (size_t)s.rows, cudaMemcpyHostToDevice, in->s_copy));
    XGPU_CHECK(cudaEventRecord(in->group_in[k], in->s_copy));
  }
  XGPU_CHECK(cudaEventRecord(in->copy_done[b], in->s_copy));
  // Direct stores format on s_dump, beside the next group's engine; results
  // formatted in device memory (register-tile order) format on s_comp and
  // leave s_dump to the copies.
  void *direct = direct_output(ctx, in);
  cudaStream_t s_fmt = direct ? in->s_dump : in->s_comp;
  for (int k = 0; k < ng; ++k) {
    const int f0 = bound[k], fc = bound[k + 1] - bound[k];
    XGPU_CHECK(cudaStreamWaitEvent(in->s_comp, in->group_in[k], 0));
    bool tail = false;
    int r = launch_engine(in, dst, in->szc, f0, fc, &tail, packed, false);
    if (r != XGPU_OK) return r;
    if (direct) {
      XGPU_CHECK(cudaEventRecord(in->group_out[k], in->s_comp));
      XGPU_CHECK(cudaStreamWaitEvent(in->s_dump, in->group_out[k], 0));
    }
    XGPU_CHECK(launch_format(in->d_state, in->int_state ? 0 : 1, s, in->cfg.matrix_order,
                             in->cfg.output_type, direct ? direct : in->d_out, s_fmt, f0, fc));
    if (!direct) XGPU_CHECK(cudaEventRecord(in->group_out[k], in->s_comp));
  }
  in->state_zero = false;
  XGPU_CHECK(cudaEventRecord(in->comp_done[b], in->s_comp));
  if (!direct) {
    // 32-bit words of the output per channel, and the plane stride (the
    // real-imag and register-tile orders keep real and imaginary planes).
    const bool planes = in->cfg.matrix_order != TRIANGULAR_ORDER;
    const size_t words =
        planes ? (size_t)(s.mat_length / s.f) : (size_t)(2 * s.mat_length / s.f);
    char *host = (char *)(ctx->matrix_h + ctx->output_offset);
    const char *dev = (const char *)in->d_out;
    for (int k = 0; k < ng; ++k) {
      const int f0 = bound[k], fc = bound[k + 1] - bound[k];
      XGPU_CHECK(cudaStreamWaitEvent(in->s_dump, in->group_out[k], 0));
      for (int plane = 0; plane < (planes ? 2 : 1); ++plane) {
        const size_t off = ((size_t)plane * s.mat_length + (size_t)f0 * words) * 4;
        XGPU_CHECK(cudaMemcpyAsync(host + off, dev + off, (size_t)fc * words * 4,
                                   cudaMemcpyDeviceToHost, in->s_dump));
      }
    }
  }
  // s_dump's last work follows the last group's engine launch
  return check_device_error(in, in->s_dump);
}

int finish_call(XGPUContext *ctx, Internal *in, int syncOp) {
  switch (syncOp) {
    case SYNCOP_DUMP:
      return dump(ctx, in);
    case SYNCOP_SYNC_TRANSFER:
      XGPU_CHECK(cudaStreamSynchronize(in->s_copy));
      return XGPU_OK;
    case SYNCOP_SYNC_COMPUTE:
      XGPU_CHECK(cudaStreamSynchronize(in->s_comp));
      return check_device_error(in);
    default:
      return XGPU_OK;
  }
}

}  // namespace

namespace xgpu {

int validate_config(const XGPUConfig &c) {
  if (c.nstation < 16 || c.nstation % 16 != 0 || c.nstation > 8192) return 0;
  if (c.nfrequency < 1 || c.nfrequency > 65535) return 0;
  if (c.ntimepipe < 16 || c.ntimepipe % 16 != 0) return 0;
  if (c.ntime < c.ntimepipe || c.ntime % c.ntimepipe != 0) return 0;
  // the engines count samples in int and step through them kSegment at a time
  if (c.ntime > 0x7fffffffu - (unsigned)kSegment) return 0;
  if (c.compute_type != XGPU_INT8 && c.compute_type != XGPU_FLOAT32) return 0;
  if (c.output_type != XGPU_INT32 && c.output_type != XGPU_FLOAT32) return 0;
  if (c.matrix_order != TRIANGULAR_ORDER && c.matrix_order != REAL_IMAG_TRIANGULAR_ORDER &&
      c.matrix_order != REGISTER_TILE_TRIANGULAR_ORDER)
    return 0;
  if (c.engine > XGPU_ENGINE_TENSOR) return 0;
  if (c.engine == XGPU_ENGINE_TENSOR && c.compute_type != XGPU_INT8) return 0;
  if (c.input_format > XGPU_INPUT_BLOCK32) return 0;
  // channel range: [channel_offset, channel_offset + nfrequency) of the band
  const unsigned band = c.input_nfrequency ? c.input_nfrequency : c.nfrequency;
  if (!c.input_nfrequency && c.channel_offset) return 0;
  if (band > 65535 || c.channel_offset > band || band - c.channel_offset < c.nfrequency) return 0;
  // input bytes of one call must fit the 32-bit sample index space of the engines
  const double bytes = 4.0 * c.nstation * band * (double)c.ntime;
  if (bytes > 1.0e12) return 0;
  return 1;
}

Sizes make_sizes(const XGPUConfig &c) {
  Sizes s;
  s.n = (int)c.nstation;
  s.f = (int)c.nfrequency;
  s.t = (int)c.ntime;
  s.tp = (int)c.ntimepipe;
  s.nbaseline = (long long)s.n * (s.n + 1) / 2;
  s.vec_length = (long long)s.t * s.f * s.n * kNpol;
  s.input_bytes = c.input_format == XGPU_INPUT_PACKED4 ? s.vec_length : 2 * s.vec_length;
  s.tri_length = (long long)s.f * s.nbaseline * kNpol * kNpol;
  s.mat_length = c.matrix_order == REGISTER_TILE_TRIANGULAR_ORDER
                     ? (long long)s.f * (s.n / 2 + 1) * (s.n / 4) * kNpol * kNpol * 4
                     : s.tri_length;
  s.state_elems = 2 * s.tri_length;
  s.fband = c.input_nfrequency ? (int)c.input_nfrequency : s.f;
  s.fin = s.fband;
  s.fin0 = (int)c.channel_offset;
  // One row of the input holds every channel of one sample (of four samples
  // in xGPU's DP4A swizzle), each channel's bytes contiguous.
  switch (c.input_format) {
    case XGPU_INPUT_PACKED4:
      s.chan_bytes = (long long)s.n * kNpol;
      s.rows = s.t;
      break;
    case XGPU_INPUT_DP4A_SWIZZLED:
      s.chan_bytes = (long long)s.n * kNpol * 2 * 4;
      s.rows = s.t / 4;
      break;
    default:   // int8 and xGPU's COMPLEX_BLOCK_SIZE=32 (blocks of 16 stations of one channel)
      s.chan_bytes = (long long)s.n * kNpol * 2;
      s.rows = s.t;
      break;
  }
  s.band_bytes = s.rows * s.fband * s.chan_bytes;
  return s;
}

}  // namespace xgpu

extern "C" {

const char *xgpuVersionString() { return XGPU_VERSION " (sm_100a; engines: tcgen05-int8, dp4a, fp32)"; }

void xgpuDefaultConfig(XGPUConfig *cfg) {
  if (cfg) *cfg = default_config();
}

void xgpuInfo(XGPUInfo *pcxs) {
  if (!pcxs) return;
  XGPUConfig c = default_config();
  fill_info(c, make_sizes(c), pcxs);
}

int xgpuContextInfo(XGPUContext *context, XGPUInfo *info) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  if (!info) return XGPU_INVALID_ARGUMENT;
  fill_info(in->cfg, in->sz, info);
  return XGPU_OK;
}

const char *xgpuEngineName(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return "none";
  if (!in->int_state) return "plain-fp32";
  return in->cfg.engine == XGPU_ENGINE_PLAIN ? "plain-dp4a" : "tensor-tcgen05-int8";
}

int xgpuInitEx(XGPUContext *context, int device_flags, const XGPUConfig *cfg_in) {
  if (!context || !cfg_in) return XGPU_INVALID_ARGUMENT;
  XGPUConfig cfg = *cfg_in;
  if (cfg.engine == XGPU_ENGINE_DEFAULT)
    cfg.engine = cfg.compute_type == XGPU_INT8 ? XGPU_ENGINE_TENSOR : XGPU_ENGINE_PLAIN;
  if (!validate_config(cfg)) return XGPU_INVALID_ARGUMENT;

  Internal *in = new (std::nothrow) Internal();
  if (!in) return XGPU_OUT_OF_MEMORY;
  context->internal = in;
  in->device = device_flags & XGPU_DEVICE_MASK;
  in->register_host_array = !(device_flags & XGPU_DONT_REGISTER_ARRAY);
  in->register_host_matrix = !(device_flags & XGPU_DONT_REGISTER_MATRIX);
  in->cfg = cfg;
  in->sz = make_sizes(cfg);
  in->szc = compact_sizes(in->sz);
  in->int_state = cfg.compute_type == XGPU_INT8;
  // CTA-pair 256x256 tiles pay off once a channel has several of them; the
  // autotuner (xgpuTune) revisits the choice per shape.
  in->tune.wide = cfg.nstation >= 384 ? 1 : 0;

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    fprintf(stderr, "xgpu: no CUDA devices found\n");
    delete in;
    context->internal = nullptr;
    return XGPU_CUDA_ERROR;
  }
  if (in->device >= ndev) {
    delete in;
    context->internal = nullptr;
    return XGPU_INVALID_ARGUMENT;
  }
  auto fail = [&](int code) {
    free_device(in);
    delete in;
    context->internal = nullptr;
    return code;
  };
  if (cudaSetDevice(in->device) != cudaSuccess) return fail(XGPU_CUDA_ERROR);
  if (cfg.engine == XGPU_ENGINE_TENSOR && tc_check_device() != cudaSuccess) {
    cudaGetLastError();
    fprintf(stderr, "xgpu: the tensor-core engine needs an sm_100 (B200-class) device\n");
    return fail(XGPU_CUDA_ERROR);
  }

  const Sizes &s = in->sz;
  const size_t in_bytes = (size_t)((s.input_bytes + 255) / 256 * 256);
  const size_t state_bytes = (size_t)s.state_elems * (in->int_state ? 8 : 4);
  if (cudaMalloc(&in->d_in[0], in_bytes) != cudaSuccess ||
      cudaMalloc(&in->d_in[1], in_bytes) != cudaSuccess ||
      cudaMalloc(&in->d_state, state_bytes) != cudaSuccess ||
      cudaMalloc(&in->d_out, (size_t)s.mat_length * sizeof(Complex)) != cudaSuccess ||
      cudaMalloc(&in->d_err, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&in->h_err, sizeof(int)) != cudaSuccess ||
      (cfg.input_format != XGPU_INPUT_INT8 &&
       (cudaMalloc(&in->d_conv[0], (size_t)(2 * s.vec_length + 255) / 256 * 256) != cudaSuccess ||
        cudaMalloc(&in->d_conv[1], (size_t)(2 * s.vec_length + 255) / 256 * 256) != cudaSuccess ||
        (s.fband != s.f && cudaMalloc(&in->d_slice, in_bytes) != cudaSuccess)))) {
    cudaGetLastError();
    return fail(XGPU_OUT_OF_MEMORY);
  }
  if (cudaStreamCreateWithFlags(&in->s_copy, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&in->s_own, cudaStreamNonBlocking) != cudaSuccess)
    return fail(XGPU_CUDA_ERROR);
  in->s_comp = in->s_own;
  for (int b = 0; b < 2; ++b) {
    if (cudaEventCreateWithFlags(&in->copy_done[b], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&in->comp_done[b], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&in->conv_done[b], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&in->conv_free[b], cudaEventDisableTiming) != cudaSuccess)
      return fail(XGPU_CUDA_ERROR);
  }
  if (cudaStreamCreateWithFlags(&in->s_conv, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&in->s_dump, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&in->caller_ev, cudaEventDisableTiming) != cudaSuccess)
    return fail(XGPU_CUDA_ERROR);
  for (int k = 0; k < kMaxGroups + 2; ++k) {
    if (cudaEventCreateWithFlags(&in->group_in[k], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&in->group_out[k], cudaEventDisableTiming) != cudaSuccess)
      return fail(XGPU_CUDA_ERROR);
  }
  if (in->int_state && cfg.engine == XGPU_ENGINE_TENSOR) {
    const size_t wbytes = (size_t)words_elems(in->szc) * 8;
    if (cudaMalloc(&in->d_words, wbytes) != cudaSuccess) {
      cudaGetLastError();   // the engine then adds into the int64 buffer directly
      in->d_words = nullptr;
    } else if (cudaMemsetAsync(in->d_words, 0, wbytes, in->s_comp) != cudaSuccess) {
      return fail(XGPU_CUDA_ERROR);
    }
  }
  if (cudaMemsetAsync(in->d_err, 0, sizeof(int), in->s_comp) != cudaSuccess ||
      cudaMemsetAsync(in->d_state, 0, state_bytes, in->s_comp) != cudaSuccess ||
      cudaStreamSynchronize(in->s_comp) != cudaSuccess)
    return fail(XGPU_CUDA_ERROR);
  in->state_zero = true;

  if (in->register_host_array) {
    int r = xgpuSetHostInputBuffer(context);
    if (r != XGPU_OK) return fail(r);
  }
  if (in->register_host_matrix) {
    int r = xgpuSetHostOutputBuffer(context);
    if (r != XGPU_OK) return fail(r);
  }
  return XGPU_OK;
}

int xgpuInit(XGPUContext *context, int device_flags) {
  XGPUConfig cfg = default_config();
  const char *e = getenv("XGPU_ENGINE");
  if (e && strcmp(e, "plain") == 0) cfg.engine = XGPU_ENGINE_PLAIN;
  if (e && strcmp(e, "fp32") == 0) {
    cfg.engine = XGPU_ENGINE_PLAIN;
    cfg.compute_type = XGPU_FLOAT32;
  }
  return xgpuInitEx(context, device_flags, &cfg);
}

int xgpuClearDeviceIntegrationBuffer(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  XGPU_CHECK(cudaSetDevice(in->device));
  // The next launch into either buffer overwrites it (or clears it first).
  // Words not yet folded belong to the integration being discarded.
  if (in->words_dirty) {
    in->words_dirty = false;
    in->words_stale = true;
    in->words_samples = 0;
  }
  in->adding_tail = false;
  in->state_zero = true;
  return XGPU_OK;
}

int xgpuSetHostInputBuffer(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  XGPU_CHECK(cudaSetDevice(in->device));
  XGPU_CHECK(cudaStreamSynchronize(in->s_copy));
  // Called again with the buffer this library allocated: keep it (freeing it
  // and then registering the freed pointer as a caller's buffer, which is
  // what taking the steps below in order would do, is undefined).
  if (in->free_array_h && context->array_h == in->free_array_h) {
    in->array_h_set = true;
    context->input_offset = 0;
    return XGPU_OK;
  }
  if (in->free_array_h) {
    cudaFreeHost(in->free_array_h);
    in->free_array_h = nullptr;
  }
  if (in->unregister_array_h) {
    cudaHostUnregister(in->unregister_array_h);
    in->unregister_array_h = nullptr;
  }
  in->array_h_set = true;
  if (context->array_h) {
    if (in->register_host_array) {
      void *reg = nullptr;
      XGPU_CHECK(register_range(context->array_h, context->array_len * sizeof(ComplexInput), &reg));
      in->unregister_array_h = (ComplexInput *)reg;
    }
  } else {
    const size_t bytes = (size_t)in->sz.band_bytes;
    // array_len counts ComplexInput elements (2 bytes); packed input needs half.
    context->array_len = (bytes + sizeof(ComplexInput) - 1) / sizeof(ComplexInput);
    XGPU_CHECK(cudaMallocHost((void **)&context->array_h, context->array_len * sizeof(ComplexInput)));
    in->free_array_h = context->array_h;
  }
  context->input_offset = 0;
  return XGPU_OK;
}

int xgpuSetHostOutputBuffer(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  XGPU_CHECK(cudaSetDevice(in->device));
  XGPU_CHECK(cudaStreamSynchronize(in->s_comp));
  // As for the input buffer: the library's own buffer, passed again, stays.
  if (in->free_matrix_h && context->matrix_h == in->free_matrix_h) {
    in->matrix_h_set = true;
    context->output_offset = 0;
    return XGPU_OK;
  }
  if (in->free_matrix_h) {
    cudaFreeHost(in->free_matrix_h);
    in->free_matrix_h = nullptr;
  }
  if (in->unregister_matrix_h) {
    cudaHostUnregister(in->unregister_matrix_h);
    in->unregister_matrix_h = nullptr;
  }
  in->matrix_h_set = true;
  if (context->matrix_h) {
    if (in->register_host_matrix) {
      void *reg = nullptr;
      XGPU_CHECK(register_range(context->matrix_h, context->matrix_len * sizeof(Complex), &reg));
      in->unregister_matrix_h = (Complex *)reg;
    }
  } else {
    context->matrix_len = (size_t)in->sz.mat_length;
    XGPU_CHECK(cudaMallocHost((void **)&context->matrix_h, context->matrix_len * sizeof(Complex)));
    in->free_matrix_h = context->matrix_h;
  }
  context->output_offset = 0;
  return XGPU_OK;
}

void xgpuFree(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return;
  cudaSetDevice(in->device);
  if (in->s_copy) cudaStreamSynchronize(in->s_copy);
  if (in->s_comp) cudaStreamSynchronize(in->s_comp);
  if (in->free_array_h) {
    cudaFreeHost(in->free_array_h);
    context->array_h = nullptr;
  }
  if (in->unregister_array_h) {
    cudaHostUnregister(in->unregister_array_h);
    context->array_h = nullptr;
  }
  if (in->free_matrix_h) {
    cudaFreeHost(in->free_matrix_h);
    context->matrix_h = nullptr;
  }
  if (in->unregister_matrix_h) {
    cudaHostUnregister(in->unregister_matrix_h);
    context->matrix_h = nullptr;
  }
  free_device(in);
  delete in;
  context->internal = nullptr;
}

int xgpuCudaXengine(XGPUContext *context, int syncOp) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  if (!in->array_h_set || !in->matrix_h_set) return XGPU_HOST_BUFFER_NOT_SET;
  if (syncOp < SYNCOP_NONE || syncOp > SYNCOP_SYNC_COMPUTE) return XGPU_INVALID_ARGUMENT;
  if (!context->array_h) return XGPU_HOST_BUFFER_NOT_SET;
  const size_t need = (size_t)((in->sz.band_bytes + 1) / 2);  // in ComplexInput units
  if (context->array_len && context->input_offset + need > context->array_len)
    return XGPU_INVALID_ARGUMENT;
  XGPU_CHECK(cudaSetDevice(in->device));

  const int b = in->cur;
  in->cur ^= 1;
  if (syncOp == SYNCOP_DUMP) {
    const int groups = dump_groups(context, in);
    if (groups > 0) return dump_call_grouped(context, in, b, groups);
  }
  // The buffer is free once the engine launch that last read it has finished.
  XGPU_CHECK(cudaStreamWaitEvent(in->s_copy, in->comp_done[b], 0));
  const Sizes &s = in->sz;
  if (s.fband == s.f) {
    XGPU_CHECK(cudaMemcpyAsync(in->d_in[b], context->array_h + context->input_offset,
                               (size_t)s.input_bytes, cudaMemcpyHostToDevice, in->s_copy));
  } else {
    // this context's channels of every row of the band
    XGPU_CHECK(cudaMemcpy2DAsync(in->d_in[b], (size_t)(s.f * s.chan_bytes),
                                 (const char *)(context->array_h + context->input_offset) +
                                     s.fin0 * s.chan_bytes,
                                 (size_t)(s.fband * s.chan_bytes), (size_t)(s.f * s.chan_bytes),
                                 (size_t)s.rows, cudaMemcpyHostToDevice, in->s_copy));
  }
  XGPU_CHECK(cudaEventRecord(in->copy_done[b], in->s_copy));
  int r = run_engine(in, in->d_in[b], in->copy_done[b], true);
  if (r != XGPU_OK) return r;
  XGPU_CHECK(cudaEventRecord(in->comp_done[b], in->s_comp));
  in->adding_tail = false;
  return finish_call(context, in, syncOp);
}

int xgpuCudaXengineDevice(XGPUContext *context, const void *device_input, int syncOp) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  if (!device_input || ((uintptr_t)device_input & 15) != 0) return XGPU_INVALID_ARGUMENT;
  if (syncOp < SYNCOP_NONE || syncOp > SYNCOP_SYNC_COMPUTE) return XGPU_INVALID_ARGUMENT;
  XGPU_CHECK(cudaSetDevice(in->device));
  int r = run_engine(in, device_input, nullptr, false);
  if (r != XGPU_OK) return r;
  return finish_call(context, in, syncOp);
}

int xgpuDumpDeviceIntegrationBuffer(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  XGPU_CHECK(cudaSetDevice(in->device));
  return dump(context, in);
}

int xgpuDumpDeviceIntegrationBufferInt64(XGPUContext *context, long long *host_out) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  if (!host_out || !in->int_state) return XGPU_INVALID_ARGUMENT;
  XGPU_CHECK(cudaSetDevice(in->device));
  const bool after_adding = in->adding_tail;
  in->adding_tail = false;
  const size_t bytes = (size_t)in->sz.state_elems * 8;
  {
    const int r = fold_words(in, after_adding);
    if (r != XGPU_OK) return r;
  }
  if (in->state_zero) {
    XGPU_CHECK(cudaStreamSynchronize(in->s_comp));
    memset(host_out, 0, bytes);
    return check_device_error(in);
  }
  XGPU_CHECK(cudaMemcpyAsync(host_out, in->d_state, bytes, cudaMemcpyDeviceToHost, in->s_comp));
  XGPU_CHECK(cudaStreamSynchronize(in->s_comp));
  return check_device_error(in);
}

int xgpuFlushIntegrationBuffer(XGPUContext *context) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  XGPU_CHECK(cudaSetDevice(in->device));
  return fold_words(in, in->adding_tail);
}

int xgpuSetComputeStream(XGPUContext *context, void *stream) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  XGPU_CHECK(cudaSetDevice(in->device));
  cudaStream_t next = stream ? (cudaStream_t)stream : in->s_own;
  if (next == in->s_comp) return XGPU_OK;
  in->adding_tail = false;
  // Order the new stream after everything queued on the old one.
  cudaEvent_t ev;
  XGPU_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  XGPU_CHECK(cudaEventRecord(ev, in->s_comp));
  XGPU_CHECK(cudaStreamWaitEvent(next, ev, 0));
  XGPU_CHECK(cudaEventDestroy(ev));
  in->s_comp = next;
  return XGPU_OK;
}

void *xgpuComputeStream(XGPUContext *context) {
  Internal *in = get(context);
  return in ? (void *)in->s_comp : nullptr;
}

int xgpuTune(XGPUContext *context, int ksplit, int grid, int pair) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  if (ksplit < 0 || grid < 0 || pair < 0 || pair > 2) return XGPU_INVALID_ARGUMENT;
  in->adding_tail = false;
  if (ksplit > 0) {
    in->tune.ksplit = ksplit;
    in->tune.grid = grid;
    in->tune.wide = pair == 1 ? 1 : 0;
    in->tune.streamk = pair == 2 ? 1 : 0;
    return XGPU_OK;
  }
  if (!in->int_state || in->cfg.engine != XGPU_ENGINE_TENSOR) return XGPU_OK;  // nothing to tune
  XGPU_CHECK(cudaSetDevice(in->device));
  XGPU_CHECK(cudaStreamSynchronize(in->s_comp));
  const Sizes &s = in->szc;   // the tuning input is a compact buffer
  // Synthetic int8 input where the engine reads it -- the first input buffer
  // of an int8 context (its contents are replaced by the next call anyway),
  // the first conversion buffer of the other formats (the input buffers of a
  // packed context hold only one byte per sample) -- and a scratch
  // integration buffer.
  void *tune_in = in->cfg.input_format == XGPU_INPUT_INT8 ? in->d_in[0] : (void *)in->d_conv[0];
  const size_t call_bytes = (size_t)(2 * s.vec_length);
  // Calls stream their input: each reads it from HBM, not from the 126 MB L2.
  // So the candidates are timed on a rotation of input buffers of together
  // about 256 MB (up to 16 calls' worth; temporary), or on the context's own
  // buffer when one call's input is larger than 128 MB or the rotation cannot
  // be allocated.
  const size_t slot_bytes = (call_bytes + 255) / 256 * 256;
  int nrot = call_bytes > (128u << 20) ? 1 : (int)(((size_t)256 << 20) / slot_bytes);
  nrot = nrot < 1 ? 1 : (nrot > 16 ? 16 : nrot);
  void *rot = nullptr;
  if (nrot > 1 && cudaMalloc(&rot, nrot * slot_bytes) != cudaSuccess) {
    cudaGetLastError();
    rot = nullptr;
    nrot = 1;
  }
  if ((rot ? launch_generate(rot, nrot * slot_bytes, 0, 12345, 16.0, in->s_comp)
           : launch_generate(tune_in, call_bytes, 0, 12345, 16.0, in->s_comp)) != cudaSuccess) {
    if (rot) cudaFree(rot);
    return XGPU_CUDA_ERROR;
  }
  // Scratch integration buffer; CTA-pair candidates add into it as words
  // when the context has a word buffer (as their calls will).
  void *scratch = nullptr;
  size_t scratch_bytes = (size_t)s.state_elems * 8;
  if (in->d_words && (size_t)words_elems(s) * 8 > scratch_bytes)
    scratch_bytes = (size_t)words_elems(s) * 8;
  if (cudaMalloc(&scratch, scratch_bytes) != cudaSuccess) {
    cudaGetLastError();
    if (rot) cudaFree(rot);
    return XGPU_OUT_OF_MEMORY;
  }
  CUtensorMap maps[16];
  for (int q = 0; q < nrot; ++q) {
    const void *buf = rot ? (const void *)((const char *)rot + q * slot_bytes) : tune_in;
    if (make_tc_tensor_map(&maps[q], buf, s) != 0) {
      cudaFree(scratch);
      if (rot) cudaFree(rot);
      return XGPU_CUDA_ERROR;
    }
  }
  int next_map = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  TcTuning best_t = in->tune;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, in->device);
  // Candidates: single CTAs and CTA pairs with 1-8 time splits on every SM,
  // stream-K, and smaller grids, which pay off when consecutive calls overlap
  // (each call then runs on part of the GPU with more tiles per CTA, so the
  // per-CTA prologue and last drain are spread thinner).
  struct Cand {
    int ksplit, grid, wide, streamk;
  };
  Cand cands[32];
  int ncand = 0;
  const int splits[] = {1, 2, 3, 4, 6, 8};
  for (int wide = 0; wide < 2; ++wide)
    for (int q = 0; q < 6; ++q) cands[ncand++] = {splits[q], 0, wide, 0};
  cands[ncand++] = {1, 0, 0, 1};
  if (sms >= 16) {
    for (int d : {2, 4, 6, 8}) cands[ncand++] = {1, sms / d, 0, 0};
    cands[ncand++] = {2, sms / 2, 0, 0};
    cands[ncand++] = {2, sms / 4, 0, 0};
    for (int d : {2, 4, 6, 8}) cands[ncand++] = {1, sms / d, 1, 0};
  }
  int rc = XGPU_OK;
  // Two passes over the candidates, each candidate keeping its faster time:
  // consecutive timings of one candidate differ by several percent, enough
  // to choose a slower setting from one noisy pass.
  float cand_ms[32];
  for (int ci = 0; ci < ncand; ++ci) cand_ms[ci] = 1e30f;
  for (int pass = 0; pass < 2 * ncand && rc == XGPU_OK; ++pass) {
    const int ci = pass % ncand;
    TcTuning t;
    t.ksplit = cands[ci].ksplit;
    t.grid = cands[ci].grid;
    t.wide = cands[ci].wide;
    t.streamk = cands[ci].streamk;
    // Timed as calls run: on the context's own stream an accumulating launch
    // overlaps the previous one (the first launch of a candidate does not).
    const int chain = in->s_comp == in->s_own ? 1 : 0;
    auto run = [&](int overlap) {
      const CUtensorMap &map = maps[next_map];
      next_map = (next_map + 1) % nrot;
      for (int t0 = 0; t0 < s.t; t0 += kSegment) {
        const int tc = s.t - t0 < kSegment ? s.t - t0 : kSegment;
        uint64_t *words =
            (in->d_words && t.wide && tc2_uses_words(tc, t)) ? (uint64_t *)scratch : nullptr;
        if (launch_tc_tuned(map, s, t0, tc, (int64_t *)scratch, 0, in->d_err, in->s_comp, t,
                            overlap, 0, -1, nullptr, words) != cudaSuccess)
          return false;
        overlap = chain;
      }
      return true;
    };
    // One warm run sizes the repetitions: enough for the overlap to settle
    // (up to 16), about 2 ms of work per candidate, at least 3.
    cudaEventRecord(e0, in->s_comp);
    if (!run(0)) { rc = XGPU_CUDA_ERROR; break; }
    cudaEventRecord(e1, in->s_comp);
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = XGPU_CUDA_ERROR; break; }
    float one = 0.f;
    cudaEventElapsedTime(&one, e0, e1);
    int reps = one > 0.f ? (int)(2.0f / one) : 16;
    reps = reps < 3 ? 3 : (reps > 16 ? 16 : reps);
    cudaEventRecord(e0, in->s_comp);
    for (int r = 0; r < reps; ++r) run(chain);
    cudaEventRecord(e1, in->s_comp);
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = XGPU_CUDA_ERROR; break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)reps;
    if (ms < cand_ms[ci]) cand_ms[ci] = ms;
    if (pass == 2 * ncand - 1) {
      // Both passes done.  Among the candidates within 3% of the fastest --
      // timings closer than that swap places from run to run -- keep the one
      // with the most CTAs: its calls' latency is the shortest, which counts
      // in short streams of calls and before every dump.
      float fastest = 1e30f;
      for (int q = 0; q < ncand; ++q) fastest = cand_ms[q] < fastest ? cand_ms[q] : fastest;
      int best_grid = -1;
      for (int q = 0; q < ncand; ++q) {
        const int g = cands[q].grid > 0 ? cands[q].grid : sms;
        if (cand_ms[q] <= 1.03f * fastest && (g > best_grid || (g == best_grid && cand_ms[q] < best))) {
          best = cand_ms[q];
          best_grid = g;
          best_t.ksplit = cands[q].ksplit;
          best_t.grid = cands[q].grid;
          best_t.wide = cands[q].wide;
          best_t.streamk = cands[q].streamk;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if (rot) cudaFree(rot);
  if (rc != XGPU_OK) return rc;
  in->tune = best_t;
  return check_device_error(in);
}

int xgpuTuning(XGPUContext *context, int *ksplit, int *grid, int *pair) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  if (!ksplit || !grid || !pair) return XGPU_INVALID_ARGUMENT;
  *ksplit = in->tune.ksplit < 1 ? 1 : in->tune.ksplit;
  *grid = in->tune.grid;
  *pair = in->tune.wide ? 1 : (in->tune.streamk ? 2 : 0);
  return XGPU_OK;
}

int xgpuInjectTimeout(XGPUContext *context, int enable) {
  Internal *in = get(context);
  if (!in) return XGPU_NOT_INITIALIZED;
  in->tune.stall = enable ? 1 : 0;
  return XGPU_OK;
}

int xgpuGenerateDevice(void *device_out, size_t nbytes, int kind, unsigned long long seed,
                       double sigma, int device) {
  if (!device_out || kind < 0 || kind > 2 || (kind == 0 && !(sigma > 0))) return XGPU_INVALID_ARGUMENT;
  XGPU_CHECK(cudaSetDevice(device));
  XGPU_CHECK(launch_generate(device_out, nbytes, kind, seed, sigma, 0));
  XGPU_CHECK(cudaStreamSynchronize(0));
  return XGPU_OK;
}

}  // extern "C"
