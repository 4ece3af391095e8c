// internal.h -- state and launcher interfaces shared by the libxgpu.so sources.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/xgpu.h"
#include "tc_job.h"

namespace xgpu {

constexpr int kNpol = 2;

// Samples per launch of an integer engine.  An int32 partial sum of one launch
// holds at most 2 * 128 * 128 * kSegment = 2^30 in magnitude (both products of
// a real or imaginary part at full scale -128), so the int32 accumulators stay
// exact; each launch adds into the int64 integration buffer.
constexpr int kSegment = 32768;

// Device error codes written by kernels into the context's error word.
enum DeviceError : int {
  kErrNone = 0,
  kErrTimeoutProducer = 1,   // TMA producer gave up waiting for a free stage
  kErrTimeoutMma = 2,        // MMA issuer gave up waiting for a loaded stage
  kErrTimeoutDrain = 3,      // epilogue gave up waiting for the accumulator
  kErrTimeoutPanel = 4,      // plain engine gave up waiting for an input panel
  kErrTimeoutConvert = 5,    // packed-input converter gave up waiting for a loaded stage
};

struct Sizes {
  int n;       // stations
  int f;       // channels
  int t;       // samples per call
  int tp;      // samples per transfer chunk
  long long nbaseline;   // n(n+1)/2
  long long vec_length;  // ComplexInput elements per call = t*f*n*2
  long long input_bytes; // bytes of one call's input in its format
  long long mat_length;  // Complex elements of a dump in the context's order
  long long tri_length;  // Complex elements in triangular order
  long long state_elems; // int64 (or float) words of the integration buffer = tri_length*2
  // Input geometry.  The engines' tensor maps step fin channels per sample
  // (fin == f for a compact buffer of this context's channels; the full band
  // when a context of a channel range reads the caller's input in place, from
  // channel fin0 on).
  int fin;               // channels per sample of the input the maps describe
  int fin0;              // first correlated channel of a full-band input
  int fband;             // channels per sample of the caller's input (cfg.input_nfrequency)
  long long band_bytes;  // bytes of one call's full-band input in its format
  long long chan_bytes;  // bytes of one channel in one row of the input (see rows)
  long long rows;        // rows of the input: samples, or 4-sample groups (DP4A swizzle)
};

Sizes make_sizes(const XGPUConfig &cfg);
// 1 if cfg is within the documented ranges of xgpuInitEx (channel range included).
int validate_config(const XGPUConfig &cfg);
// The same sizes with the input read as a compact buffer of this context's
// channels (fin = f, fin0 = 0).
inline Sizes compact_sizes(Sizes s) {
  s.fin = s.f;
  s.fin0 = 0;
  return s;
}

// ---- engines --------------------------------------------------------------
// All engines read int8 input laid out [t][f][s][p][c] (t = 0..t_total) and
// add samples [t0, t0+tcount) into the triangular integration buffer
// state[f][k][p1][p2][re,im], k = i(i+1)/2 + j, i >= j.  overwrite != 0
// stores instead of adding (the buffer is known to be zero).

// The plain engines load their input panels with TMA; err (may be null)
// receives kErrTimeoutPanel if a panel never arrives.  stall (a test switch)
// withholds the loads so that happens.
// overlap: the launch only adds and follows an adding dp4a launch on the
// same stream (programmatic launch: it may run beside it).
cudaError_t launch_plain_dp4a(const int8_t *in, const Sizes &s, int t0, int tcount,
                              int64_t *state, int overwrite, cudaStream_t st, int *err = nullptr,
                              int stall = 0, int f0 = 0, int fcount = -1, int overlap = 0);
cudaError_t launch_plain_fp32(const int8_t *in, const Sizes &s, int t0, int tcount,
                              float *state, int overwrite, cudaStream_t st, int *err = nullptr,
                              int stall = 0, int f0 = 0, int fcount = -1);

// Tensor-core engine.  The tensor map describes `in` (see make_tc_tensor_map).
cudaError_t launch_tc(const CUtensorMap &map, const Sizes &s, int t0, int tcount,
                      int64_t *state, int overwrite, int *err, cudaStream_t st);
// Launched programmatically (PDL): the prologue overlaps the previous kernel of
// the stream.  overlap = 1 promises that the previous kernel of the stream is
// an engine launch of the same integration that does not store (only adds)
// and that nothing this launch reads was written after it was queued: then,
// unless this launch stores, the two run side by side, their reduce-adds
// commuting.  Channels [f0, f0 + fcount) of the input and buffer are
// correlated (fcount < 0: through the last channel); an overwrite stores into,
// or clears, that channel range only.
// packed_in != nullptr: the input is packed 4+4-bit, at packed_in with
// geometry s (the pointer `map` was made from with make_packed_map), and the
// CTA-pair kernel loads and expands it itself; it needs tune.wide.
// words != nullptr (CTA-pair kernel, overwrite = 0): the launch puts its
// sums into the block-major word buffer `words` (words_elems(s) words) instead
// of `state` -- adding them, or storing them with words_store (only with one
// item per tile, tc2_single_item) -- and launch_fold_words later moves them
// into `state`.  At most 65535 samples may go into the words between folds.
cudaError_t launch_tc_tuned(const CUtensorMap &map, const Sizes &s, int t0, int tcount,
                            int64_t *state, int overwrite, int *err, cudaStream_t st,
                            const TcTuning &tune, int overlap, int f0 = 0, int fcount = -1,
                            const void *packed_in = nullptr, uint64_t *words = nullptr,
                            int words_store = 0);
// The CTA-pair (cta_group::2, 256x256 tile) kernel for one job.
cudaError_t launch_tc2(const CUtensorMap &map, const Sizes &s, int t0, int tcount, int64_t *state,
                       int overwrite, int *err, cudaStream_t st, const TcTuning &tune,
                       int overlap, int f0 = 0, int fcount = -1,
                       const void *packed_in = nullptr, uint64_t *words = nullptr,
                       int words_store = 0);
// Word buffer: 64-bit words (im * 2^32 + re of one visibility's sums) in
// 32 x 32-station blocks; its size for sizes s, and the fold that adds the
// words into the int64 buffer (triangular order).  Exact while every sum in
// the words is below 2^31 in magnitude (65535 samples).
long long words_blocks(const Sizes &s);   // 32-station blocks per channel
// Whether a CTA-pair launch of tcount samples with `tune` may use words (its
// items are short enough for the split epilogue), and whether it has one item
// per tile (no time splits: it may store its words).
bool tc2_uses_words(int tcount, const TcTuning &tune);
bool tc2_single_item(int tcount, const TcTuning &tune);
long long words_elems(const Sizes &s);
// overlap: the launch before it on `st` is an engine launch of the same
// context (it may then start while that launch finishes).  store_state: the
// int64 buffer holds nothing yet; the fold stores into it instead of adding.
cudaError_t launch_fold_words(const uint64_t *words, int64_t *state, const Sizes &s,
                              cudaStream_t st, int overlap = 0, int store_state = 0);
constexpr int kWordsMaxSamples = 65535;
// A batch of jobs from a device-resident table (item_begin ascending); with a
// queue (device int) the CTAs take items dynamically, otherwise by stride.
cudaError_t launch_tc_batch(const Job *dev_jobs, int njobs, int total_items, int *queue, int *err,
                            int grid, cudaStream_t st);
// Fill a job for samples [t0, t0+tcount) of dev_in (sizes s).  store=1 asks for
// plain stores (only honoured without time splits); pair=1 cuts it into the
// 256x256 tiles of the CTA-pair kernel.  Returns 0 on success.
int tc_fill_job(Job *job, const void *dev_in, const Sizes &s, int t0, int tcount, int64_t *state,
                int store, int ksplit, int item_begin, int pair);
// The CTA-pair kernel over a device job table filled with pair = 1;
// max_item_steps is the largest steps_per_split in the table (it selects the
// epilogue schedule).
cudaError_t launch_tc2_batch(const Job *dev_jobs, int njobs, int total_items, int *queue, int *err,
                             int grid, cudaStream_t st, int max_item_steps);
// Encodes the 3-D tensor map {x: 4n bytes, y: f, z: t} over a device input
// buffer whose samples are s.fin channels apart (dev_in points at the first
// channel the map covers).  Returns 0 on success.
int make_tc_tensor_map(CUtensorMap *map, const void *dev_in, const Sizes &s);
// The same map with unswizzled boxes of 128 bytes x `rows` samples (the plain
// engines' panels).
int make_panel_map(CUtensorMap *map, const void *dev_in, const Sizes &s, int rows);
// {x: 2n bytes, y: f, z: t} over packed 4+4-bit input [t][f][s][p], unswizzled
// boxes of 64 bytes (32 stations) x 128 samples: the CTA-pair kernel's packed
// loads.  Needs n a multiple of 8.  Returns 0 on success.
int make_packed_map(CUtensorMap *map, const void *dev_in, const Sizes &s);
// 0 if the tensor-core kernel image loads on the current device.
cudaError_t tc_check_device();
// Per-device set-up and facts, cached for devices 0 .. kDeviceCache-1 (others are
// queried or set on every call): the SM count of the current device, and the
// dynamic shared-memory allowance of both tcgen05 kernels on it.
constexpr int kDeviceCache = 64;
int current_device_sms();
cudaError_t tc_configure_device();
cudaError_t tc2_set_smem_attribute();

// ---- input conversion, output formatting, synthetic input -----------------
cudaError_t launch_unpack4(const uint8_t *in, int8_t *out, long long nsamples, cudaStream_t st);
cudaError_t launch_unswizzle_dp4a(const int8_t *in, int8_t *out, const Sizes &s, cudaStream_t st);
cudaError_t launch_unblock32(const int8_t *in, int8_t *out, long long nbytes, cudaStream_t st);
// state (int64 or float) -> Complex words in `order` of type out_type.
// Channels [f0, f0 + fcount) of the buffer into `out` in the requested order
// (fcount < 0: through the last channel); other channels' words are untouched.
cudaError_t launch_format(const void *state, int state_is_float, const Sizes &s, int order,
                          int out_type, void *out, cudaStream_t st, int f0 = 0,
                          int fcount = -1);
cudaError_t launch_generate(void *out, size_t nbytes, int kind, unsigned long long seed,
                            double sigma, cudaStream_t st);

// Host Gaussian table shared with the generator kernel.
void gauss_thresholds(double sigma, uint32_t thr[254]);

}  // namespace xgpu
