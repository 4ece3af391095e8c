/*
 * xgpu.h -- C ABI of the B200 X-engine (libxgpu.so).
 *
 * This header is the drop-in surface for programs written against xGPU's
 * src/xgpu.h.  Every type, macro value, struct layout and prototype that
 * xGPU declares is declared here with the same name, value and layout, so a
 * program that compiled and linked against xGPU compiles and links against
 * this library unchanged.  Citations are to the reference's src/ directory.
 *
 * Names that xGPU does not have are marked "extension".  They add runtime
 * sizing (xGPU fixes every size at library build time), a choice of engine
 * (CUDA-core 2x2 register tile, or tcgen05 int8 tensor cores), exact int64
 * integration dumps, device-resident input and the packed 4+4-bit input.
 */
#ifndef XGPU_H
#define XGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Input samples are 8-bit fixed point (xgpu.h:10-20 hard-codes FIXED_POINT). */
#define FIXED_POINT

#ifndef FIXED_POINT
typedef float ReImInput;
#else
typedef signed char ReImInput;
#endif

/* One complex input sample, real part first (xgpu.h:22-25). */
typedef struct ComplexInputStruct {
  ReImInput real;
  ReImInput imag;
} ComplexInput;

/* One output visibility (xgpu.h:27-37).  Callers that define DP4A receive
 * 32-bit integers; everyone else receives 32-bit floats.  Both are 8 bytes,
 * so buffer sizes do not depend on the choice.  The library writes whichever
 * the context was created for (XGPUConfig.output_type). */
#ifndef DP4A
typedef struct ComplexStruct {
  float real;
  float imag;
} Complex;
#else
typedef struct ComplexStruct {
  int real;
  int imag;
} Complex;
#endif

/* Type codes (xgpu.h:40-42). */
#define XGPU_INT8    (0)
#define XGPU_FLOAT32 (1)
#define XGPU_INT32   (2)

/* Output matrix orders (xgpu.h:45-47). */
#define TRIANGULAR_ORDER 1000
#define REAL_IMAG_TRIANGULAR_ORDER 2000
#define REGISTER_TILE_TRIANGULAR_ORDER 3000

/* xgpuInit flags (xgpu.h:50-54): the low 16 bits select the CUDA device. */
#define XGPU_DEVICE_MASK          ((1<<16)-1)
#define XGPU_DONT_REGISTER_ARRAY  (1<<16)
#define XGPU_DONT_REGISTER_MATRIX (1<<17)
#define XGPU_DONT_REGISTER        (XGPU_DONT_REGISTER_ARRAY | \
                                   XGPU_DONT_REGISTER_MATRIX)

/* Sizing report (xgpu.h:61-92).  Field order and types are unchanged, so the
 * struct is byte-identical to xGPU's. */
typedef struct XGPUInfoStruct {
  unsigned int npol;          /* polarisations per station (always 2) */
  unsigned int nstation;      /* stations */
  unsigned int nbaseline;     /* nstation*(nstation+1)/2, autos included */
  unsigned int nfrequency;    /* channels */
  unsigned int ntime;         /* samples per channel per xgpuCudaXengine call */
  unsigned int ntimepipe;     /* samples per host-to-device transfer chunk */
  unsigned int input_type;    /* XGPU_INT8 */
  unsigned int compute_type;  /* XGPU_INT8 (integer engines) or XGPU_FLOAT32 */
  long long unsigned int vecLength;      /* ComplexInput elements per call */
  long long unsigned int vecLengthPipe;  /* ComplexInput elements per chunk */
  long long unsigned int matLength;      /* Complex elements in the output */
  long long unsigned int triLength;      /* Complex elements in triangular order */
  unsigned int matrix_order;  /* one of the *_ORDER codes */
  size_t shared_atomic_size;  /* kept for layout compatibility; reports 4 */
  size_t complex_block_size;  /* 32 for an XGPU_INPUT_BLOCK32 context, else 1 */
} XGPUInfo;

/* Caller-owned context (xgpu.h:94-113), byte-identical to xGPU's. */
typedef struct XGPUContextStruct {
  ComplexInput *array_h;   /* host input */
  Complex *matrix_h;       /* host output */
  size_t array_len;        /* in ComplexInput units */
  size_t matrix_len;       /* in Complex units */
  size_t input_offset;     /* reset to 0 by xgpuSetHostInputBuffer */
  size_t output_offset;    /* reset to 0 by xgpuSetHostOutputBuffer */
  void *internal;          /* opaque library state */
} XGPUContext;

/* Return codes (xgpu.h:116-121). */
#define XGPU_OK                          (0)
#define XGPU_OUT_OF_MEMORY               (1)
#define XGPU_CUDA_ERROR                  (2)
#define XGPU_INSUFFICIENT_TEXTURE_MEMORY (3)
#define XGPU_NOT_INITIALIZED             (4)
#define XGPU_HOST_BUFFER_NOT_SET         (5)
/* Extension: a size, pointer, offset or option was out of range.  No call
 * that xGPU can make with valid arguments returns it. */
#define XGPU_INVALID_ARGUMENT            (6)

/* syncOp values for xgpuCudaXengine (xgpu.h:124-127). */
#define SYNCOP_NONE           0
#define SYNCOP_DUMP           1
#define SYNCOP_SYNC_TRANSFER  2
#define SYNCOP_SYNC_COMPUTE   3

/* ------------------------------------------------------------------------ */
/* Functions of xGPU's cuda_xengine.cu (xgpu.h:134-219).                    */
/* ------------------------------------------------------------------------ */

/* Library version string (xgpu.h:134); static storage, do not free. */
const char * xgpuVersionString();

/* Default sizes of this build (xgpu.h:140): the sizes xgpuInit uses.  Set at
 * library build time with make NSTATION=... NFREQUENCY=... NTIME=...
 * NTIME_PIPE=... exactly as xGPU's Makefile takes them. */
void xgpuInfo(XGPUInfo *pcxs);

/* Create a context on device (device_flags & XGPU_DEVICE_MASK) with the
 * build's default sizes (xgpu.h:168, cuda_xengine.cu:180-331).  Host buffers
 * follow xGPU's rules: a NULL array_h / matrix_h is allocated pinned by the
 * library; a non-NULL one is registered (page-rounded) unless the matching
 * XGPU_DONT_REGISTER_* flag is set.  Unlike xGPU this never calls exit(): no
 * device gives XGPU_CUDA_ERROR.  The engine is the tcgen05 tensor-core
 * engine unless the environment variable XGPU_ENGINE=plain selects the
 * CUDA-core engine. */
int xgpuInit(XGPUContext *context, int device_flags);

/* Zero the device integration buffer: the next call starts a new
 * integration (xgpu.h:174, cuda_xengine.cu:334-348). */
int xgpuClearDeviceIntegrationBuffer(XGPUContext *context);

/* Replace the host input / output buffer (xgpu.h:188,202;
 * cuda_xengine.cu:354-498).  The previous buffer is freed or unregistered,
 * and input_offset / output_offset are reset to 0. */
int xgpuSetHostInputBuffer(XGPUContext *context);
int xgpuSetHostOutputBuffer(XGPUContext *context);

/* Release everything the context holds (xgpu.h:204, cuda_xengine.cu:501-541).
 * Safe to call twice. */
void xgpuFree(XGPUContext *context);

/* Correlate ntime samples at array_h + input_offset and add them to the
 * device integration buffer (xgpu.h:206-219, cuda_xengine.cu:543-677).
 *   SYNCOP_NONE          return once the work is queued
 *   SYNCOP_DUMP          wait, then write the integration (in the context's
 *                        matrix order and output type) to
 *                        matrix_h + output_offset; the buffer is not cleared
 *   SYNCOP_SYNC_TRANSFER wait until the input has been copied to the device
 *   SYNCOP_SYNC_COMPUTE  wait until the correlation has finished
 * The device buffer holds exact int64 sums for the integer engines, so an
 * integration may span any number of calls without overflow; the int32
 * output of a dump wraps modulo 2^32 exactly as xGPU's int32 buffer does. */
int xgpuCudaXengine(XGPUContext *context, int syncOp);

/* Extension (named after the dump entry point of later xGPU releases):
 * wait for queued work, then write the integration to
 * matrix_h + output_offset exactly as SYNCOP_DUMP does, without correlating
 * new samples. */
int xgpuDumpDeviceIntegrationBuffer(XGPUContext *context);

/* ------------------------------------------------------------------------ */
/* Functions of xGPU's cpu_util.c and omp_xengine.c (xgpu.h:223-235).       */
/* They use the build's default sizes (xgpuInfo), like xGPU's.  They run on  */
/* the host and are never part of the device path.                          */
/* ------------------------------------------------------------------------ */

/* Gaussian noise, sigma 2.5, rounded, saturated to +-7 and scaled by 16, from
 * the C library rand() stream (cpu_util.c:13-55). */
void xgpuRandomComplex(ComplexInput* random_num, long long unsigned int length);

/* In-place conversion of a dumped matrix from the default matrix order to
 * TRIANGULAR_ORDER (cpu_util.c:57-132). */
void xgpuReorderMatrix(Complex *matrix);

/* Compare two triangular-order matrices and print a summary
 * (cpu_util.c:134-232). */
void xgpuCheckResult(Complex *gpu, Complex *cpu, int verbose, ComplexInput *array_h);

/* [t][f][s][p][c] -> [t/4][f][s][p][c][t%4] input swizzle of xGPU's DP4A
 * builds (cpu_util.c:235-255). */
void xgpuSwizzleInput(ComplexInput *out, const ComplexInput *in);

/* Triangular order -> full Hermitian [f][i][j][p1][p2] (cpu_util.c:258-279). */
void xgpuExtractMatrix(Complex *matrix, Complex *packed);

/* Host X-engine in TRIANGULAR_ORDER (omp_xengine.c:36-93), OpenMP over
 * (channel, baseline).  It sums in int64, so it is exact where xGPU's float
 * sums round (above 2^24). */
void xgpuOmpXengine(Complex *matrix_h, ComplexInput *array_h);

/* ------------------------------------------------------------------------ */
/* Extensions: runtime sizing and engine choice.                            */
/* ------------------------------------------------------------------------ */

/* Engines. */
#define XGPU_ENGINE_DEFAULT 0  /* XGPU_ENGINE_TENSOR for integer compute */
#define XGPU_ENGINE_PLAIN   1  /* CUDA-core 2x2 register tile: FP32 or dp4a */
#define XGPU_ENGINE_TENSOR  2  /* tcgen05 int8 tensor cores (compute XGPU_INT8) */

/* Input sample formats. */
#define XGPU_INPUT_INT8     0  /* [t][f][s][p] {re,im} int8 (xGPU's layout) */
#define XGPU_INPUT_PACKED4  1  /* [t][f][s][p] one byte: re in the high nibble,
                                  im in the low nibble, 4-bit two's complement */
#define XGPU_INPUT_DP4A_SWIZZLED 2 /* xgpuSwizzleInput's [t/4][f][s][p][c][t%4] */
#define XGPU_INPUT_BLOCK32  3  /* xGPU built with COMPLEX_BLOCK_SIZE=32: per 16
                                  stations, 32 bytes of {X.re,Y.re} pairs then
                                  32 bytes of {X.im,Y.im} pairs */

typedef struct XGPUConfigStruct {
  unsigned int nstation;     /* multiple of 16 */
  unsigned int nfrequency;   /* >= 1 */
  unsigned int ntime;        /* samples per call, multiple of ntimepipe */
  unsigned int ntimepipe;    /* multiple of 16 */
  unsigned int compute_type; /* XGPU_INT8 (exact) or XGPU_FLOAT32 (plain only) */
  unsigned int output_type;  /* XGPU_FLOAT32 or XGPU_INT32: Complex member type */
  unsigned int matrix_order; /* TRIANGULAR_ORDER, REAL_IMAG_... or REGISTER_TILE_... */
  unsigned int engine;       /* XGPU_ENGINE_* */
  unsigned int input_format; /* XGPU_INPUT_* */
  /* Channel range of a full-band input, for one context per GPU over one
   * shared [t][f][s][p] buffer (xGPU selects the GPU with XGPU_DEVICE_MASK,
   * xgpu.h:50, cuda_xengine.cu:193,225, but every context there reads a
   * buffer of its own NFREQUENCY channels).  The input of one call holds
   * input_nfrequency channels per sample; this context correlates channels
   * [channel_offset, channel_offset + nfrequency) of it, in place, and its
   * integration buffer and dumps hold those nfrequency channels only.
   * input_nfrequency = 0 means nfrequency (the whole input, offset 0).
   * xgpuContextInfo's vecLength is then the full-band input length. */
  unsigned int channel_offset;
  unsigned int input_nfrequency;
} XGPUConfig;

/* Fill cfg with this build's defaults (the sizes xgpuInfo reports). */
void xgpuDefaultConfig(XGPUConfig *cfg);

/* xgpuInit with explicit sizes and options.  Returns XGPU_INVALID_ARGUMENT
 * for sizes or options outside the documented ranges. */
int xgpuInitEx(XGPUContext *context, int device_flags, const XGPUConfig *cfg);

/* Sizes of an initialised context, in xgpuInfo's form. */
int xgpuContextInfo(XGPUContext *context, XGPUInfo *info);

/* xgpuCudaXengine on input that is already in device memory (same layout
 * and size as array_h would hold; 16-byte aligned).  The caller keeps the
 * buffer unchanged until the call's work is done (any syncOp but NONE, or a
 * later synchronising call).  The input must be complete when the call is
 * made, or be produced on the stream given to xgpuSetComputeStream. */
int xgpuCudaXengineDevice(XGPUContext *context, const void *device_input, int syncOp);

/* Exact dump: the integration as int64 in triangular order,
 * [f][baseline][p1][p2][re,im], triLength*2 values, written to host_out.
 * Integer engines only. */
int xgpuDumpDeviceIntegrationBufferInt64(XGPUContext *context, long long *host_out);

/* Complete the integration on the device without reading it.  Accumulating
 * calls of the tensor engine may keep their sums in a short-term buffer that
 * is added into the integration buffer before every dump; this queues that
 * addition on the compute stream now (no host wait), so that work timed or
 * ordered on that stream up to this point includes it.  A no-op when nothing
 * is pending, and for the other engines. */
int xgpuFlushIntegrationBuffer(XGPUContext *context);

/* ---- Test and benchmark hooks (not part of xGPU's API; a correlator
 * pipeline needs none of the three below) ---------------------------------- */

/* Test and benchmark hook.  Fill a device buffer with seeded synthetic
 * samples, identical to the host generator the tests use: kind 0 = Gaussian
 * int8 with the given sigma, rounded and clipped to [-127,127]; kind 1 =
 * uniform integers in [-7,7] packed 4+4-bit (one byte per complex sample);
 * kind 2 = uniform int8 in [-7,7].  nbytes is the buffer size in bytes. */
int xgpuGenerateDevice(void *device_out, size_t nbytes, int kind, unsigned long long seed,
                       double sigma, int device);

/* Benchmark hook.  Measure the device's CUDA-core rate for the plain
 * engines' arithmetic (the denominator of their rooflines) with a
 * register-resident microbenchmark of about 25 ms: kind 0 = dp4a, counted as
 * 8 operations (four int8 products and their sum), kind 1 = FP32 FMA,
 * counted as 2.  *ops_per_second receives the rate, in the X-engine's
 * operations. */
int xgpuMeasureCorePeak(int device, int kind, double *ops_per_second);

/* Run the context's device work (engine launches, dump formatting) on the
 * caller's CUDA stream (a cudaStream_t) instead of the context's own, e.g. to
 * order it with other work or to bracket it with the caller's CUDA events.
 * NULL returns to the context's own stream.  The caller keeps the stream alive
 * until xgpuFree or the next xgpuSetComputeStream. */
int xgpuSetComputeStream(XGPUContext *context, void *stream);

/* The stream (a cudaStream_t) the context queues its device work on: its own
 * unless xgpuSetComputeStream chose another; NULL for an uninitialised
 * context.  On its own stream a context lets an accumulating call over
 * device-resident input start while the previous call's launch finishes (the
 * two only add into the integration), so callers that time or order work
 * should record their events on this stream rather than switch streams. */
void *xgpuComputeStream(XGPUContext *context);

/* Extension with no counterpart in the reference: correlate once without
 * allocating anything, for callers that cannot call cudaMalloc where they
 * correlate (a real-time thread that must not block on an allocation that can
 * synchronise the device, or a plugin whose host framework owns all device
 * memory).  cfg->ntime samples at device_input ([t][f][s][p][c] int8,
 * 16-byte aligned) are correlated by the tensor-core engine into a fresh
 * integration (no accumulation across calls), which is then written to
 * device_output as cfg->matrix_order / cfg->output_type (matLength Complex).
 * The int64 integration buffer lives in a static 32 MiB device array that
 * every GPU loading the library holds until exit, so 64*F*N(N+1)/2 bytes must
 * fit in 32 MiB - 256 (e.g. N=256 with F <= 15); larger sizes return
 * XGPU_INVALID_ARGUMENT, as do the sizes xgpuInitEx rejects and a channel
 * range (channel_offset / input_nfrequency other than the whole input).  Work
 * is queued on `stream` (a cudaStream_t, NULL for the legacy default stream)
 * and the call waits for it and reads its error status back to the host
 * before it returns.  The calling thread's current device is left as it was.
 * All calls share the array: calls that overlap on the GPU race and must be
 * serialised.  The first call on a device looks up the array's device address
 * and keeps it for the process's lifetime, so make that first call before any
 * stream capture begins; after a cudaDeviceReset of that device the address
 * is stale, so make no further call on it. */
int xgpuCorrelateStatic(const void *device_input, void *device_output, const XGPUConfig *cfg,
                        int device, void *stream);

/* Kernel, time splits and grid of the tensor-core engine for this context.
 * pair = 0 runs one CTA per 128x128 tile of the Gram matrix; pair = 1 runs
 * CTA pairs (tcgen05 cta_group::2) on 256x256 tiles; pair = 2 runs single CTAs
 * that each take an equal share of all (tile, 128-sample) steps ("stream-K":
 * tiles cut between CTAs add their parts exactly) when a call adds into
 * existing sums, and 128x128 tiles otherwise.  ksplit >= 1 splits
 * every tile's samples into that many items whose partial sums are added
 * exactly in the integration buffer; grid is the number of CTAs (0 = one per
 * SM).  ksplit = 0 autotunes all three now: the engine is timed on synthetic
 * input and a scratch integration buffer (the context's own is not touched),
 * in chains of calls that overlap as a stream of calls does and read their
 * input from device memory rather than the L2 cache (temporary buffers of up
 * to about 256 MB plus one integration buffer, freed before it returns), and
 * the fastest setting is kept.  With CTA pairs, XGPU_INPUT_PACKED4 input
 * is expanded inside the kernel; the other kernels read an int8 copy that a
 * pre-pass makes. */
int xgpuTune(XGPUContext *context, int ksplit, int grid, int pair);

/* The setting in use (as xgpuTune takes it; ksplit >= 1), e.g. to keep an
 * autotuned choice and pass it to xgpuTune in a later run. */
int xgpuTuning(XGPUContext *context, int *ksplit, int *grid, int *pair);

/* Test hook, for testing a caller's error handling.  While enabled, the
 * engine of this context (tensor-core or plain) issues no input loads, so its
 * bounded device waits expire (about 2 s per launch) instead of completing: the next
 * synchronising call returns XGPU_CUDA_ERROR, the integration in progress is
 * invalid, and once disabled the context works normally (clear it first).
 * Nothing faults or hangs. */
int xgpuInjectTimeout(XGPUContext *context, int enable);

/* ---- Extension: batches of uneven subarrays in one launch ---------------- */
/* One subarray: its own station, channel and sample counts, its input
 * ([t][f][s][p][c] int8, 16-byte aligned) and its int64 integration buffer
 * (triangular order, nfrequency*nstation*(nstation+1)/2*8 values, 16-byte
 * aligned).  accumulate = 0 replaces the buffer's contents with this run's
 * sums; 1 adds to them.  xgpuCudaXengine's limits on sizes apply. */
typedef struct XGPUBatchJobStruct {
  const void *device_input;
  long long *device_state;
  unsigned int nstation;
  unsigned int nfrequency;
  unsigned int ntime;
  int accumulate;
} XGPUBatchJob;

typedef struct XGPUBatchImpl *XGPUBatch;

#define XGPU_BATCH_AUTOTUNE 1  /* time split granularity and grid chosen by timing */
#define XGPU_BATCH_GRAPH    2  /* capture the run once as a CUDA graph and replay it */
#define XGPU_BATCH_PAIR     4  /* CTA-pair kernel, 256x256 tiles (without AUTOTUNE) */

/* Plan a batch on `device`, run on `stream` (a cudaStream_t, NULL = legacy
 * default stream).  The job list is copied; the buffers must stay valid. */
int xgpuBatchCreate(XGPUBatch *batch, const XGPUBatchJob *jobs, int njobs, int device,
                    void *stream, int flags);
/* Queue one run of every job of the batch (one persistent kernel launch). */
int xgpuBatchRun(XGPUBatch batch);
/* Wait for queued runs; XGPU_CUDA_ERROR if a device wait timed out. */
int xgpuBatchSync(XGPUBatch batch);
/* Work items per run, CTAs, and the time split chosen: max_steps >= 0 is the
 * single-CTA kernel with that many 128-sample stages per item (0 = unsplit);
 * max_steps < 0 is the CTA-pair kernel with -1 - max_steps stages per item. */
int xgpuBatchInfo(XGPUBatch batch, int *work_items, int *grid, int *max_steps);
void xgpuBatchDestroy(XGPUBatch batch);

/* ---- Extension: continuous-batching server ------------------------------- */
/* One request: a subarray integrating nblocks blocks of ntime samples per
 * channel.  Block b's samples become available at
 * arrival_s + (b+1) * ntime / sample_rate_hz, already in device memory as a
 * network card would leave them: a slice of a receive pool of seeded
 * Gaussian int8 samples filled before the clock starts (one pool per sigma
 * bucket 4, 8, 16, 32, nearest in log2; the slice starts at byte
 * 256 * (splitmix64(seed * 1000003 + b) mod 2^20) of the generator stream with
 * seed 0x5EED0000 + bucket).  The request is dumped (triangular order, int32
 * Complex) after its last block and, if dump_every > 0, after every
 * dump_every blocks.  Requests must be sorted by arrival_s. */
typedef struct XGPUServeJobStruct {
  unsigned int nstation;
  unsigned int nfrequency;
  unsigned int ntime;        /* <= 32768 */
  unsigned int nblocks;
  unsigned int dump_every;
  unsigned long long seed;
  double sigma;
  double arrival_s;
} XGPUServeJob;

#define XGPU_SERVE_BATCHED      0  /* continuous batching on the tensor-core engine */
#define XGPU_SERVE_PLAIN_SERIAL 1  /* one request at a time, plain dp4a engine */

typedef struct XGPUServeOptionsStruct {
  double sample_rate_hz;            /* per-channel complex sample rate */
  size_t device_budget_bytes;       /* HBM arena for resident state (admission limit) */
  size_t host_budget_bytes;         /* pinned host arena for dumps (0 = 8 GiB) */
  int mode;                         /* XGPU_SERVE_* */
  int device;
} XGPUServeOptions;

typedef struct XGPUServeStatsStruct {
  long long jobs, blocks, dumps;
  double ops;                       /* 16*F*T*N(N+1) summed over blocks */
  double wall_s;                    /* from start to the last dump in host memory */
  double tops;                      /* ops / wall_s / 1e12 */
  double gpu_busy_s;                /* time with device work in flight */
  double dump_p50_ms, dump_p99_ms, dump_max_ms;  /* samples available -> dump in host memory */
  double period_ratio_p99;          /* p99 of dump latency / the request's integration period */
  long long late_dumps;             /* dumps slower than their request's integration period */
  long long admitted_peak;          /* most requests resident at once */
  double device_peak_bytes;         /* peak of the HBM arena */
} XGPUServeStats;

/* Serve the request stream in real time and return when every request has
 * been dumped.  results, if not NULL, holds one host pointer per request
 * (NULL to skip) receiving its final dump: triLength*2 int32 words. */
int xgpuServeRun(const XGPUServeJob *jobs, int njobs, const XGPUServeOptions *options,
                 XGPUServeStats *stats, int **results);

/* Name of the engine a context runs ("tensor-tcgen05-int8", "plain-dp4a",
 * "plain-fp32"). */
const char * xgpuEngineName(XGPUContext *context);

#ifdef __cplusplus
}
#endif

#endif /* XGPU_H */
