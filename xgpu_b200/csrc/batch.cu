// batch.cu -- many uneven subarrays in one persistent tensor-core launch.
//
// A batch is a list of jobs, each its own subarray: station count, channel
// count, sample count, input buffer and int64 integration buffer.  The plan
// cuts every job into work items (channel, time split, 128x128 tile of the
// Gram matrix), writes the job table to device memory once, and runs all
// items in one launch of the persistent tensor-core kernel, whose CTAs take
// items from a global atomic queue so long and short jobs balance across the
// SMs.  Plans are captured once into a CUDA graph (queue reset, buffer clears,
// kernel) and replayed.  An autotuner picks the time-split granularity and the
// grid size by timing the batch on scratch integration buffers.
//
// xGPU has no counterpart: it runs one compile-time shape per library build
// (xgpu_info.h:6-25), so a mixed workload there is a loop of separate
// libraries or processes.
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "internal.h"

using namespace xgpu;

struct XGPUBatchImpl {
  int device = 0;
  cudaStream_t stream = nullptr;
  int flags = 0;
  std::vector<XGPUBatchJob> jobs;
  std::vector<Sizes> sizes;
  Job *d_jobs = nullptr;
  int *d_queue = nullptr;
  int *d_err = nullptr;
  int *h_err = nullptr;
  int total_items = 0;
  int grid = 0;
  int max_steps = 0;          // stages per work item (0: no time split)
  int pair = 0;               // 1: CTA-pair kernel (256x256 tiles)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double tuned_ms = 0.0;
  std::vector<Job> table;    // the uploaded job table
};

namespace {

#define BCHECK(call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "(CUDA) %s (%s:%d)\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return XGPU_CUDA_ERROR;                                                          \
    }                                                                                  \
  } while (0)

int num_sms(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  return v;
}

// Time splits for a job: enough that no item exceeds max_steps stages (and
// none exceeds the int32-exact segment), never more than the job has stages.
int splits_for(int t, int max_steps) {
  const int steps = (t + kTcSamplesPerStage - 1) / kTcSamplesPerStage;
  const int cap = kSegment / kTcSamplesPerStage;
  int lim = max_steps > 0 ? std::min(max_steps, cap) : cap;
  return (steps + lim - 1) / lim;
}

// Build the job table for the given states (the plan's or scratch ones).
int build_table(XGPUBatchImpl *b, const std::vector<int64_t *> &states, int max_steps, int pair,
                std::vector<Job> &table, int &total) {
  table.assign(b->jobs.size(), Job());
  long long begin = 0;
  for (size_t q = 0; q < b->jobs.size(); ++q) {
    const XGPUBatchJob &j = b->jobs[q];
    const Sizes &s = b->sizes[q];
    const int ks = splits_for(s.t, max_steps);
    if (tc_fill_job(&table[q], j.device_input, s, 0, s.t, states[q], j.accumulate ? 0 : 1, ks,
                    (int)begin, pair) != 0)
      return XGPU_INVALID_ARGUMENT;
    begin += table[q].items;
    if (begin > 0x7fffffffLL) return XGPU_INVALID_ARGUMENT;
  }
  total = (int)begin;
  return XGPU_OK;
}

// Queue one run of the batch on the plan's stream (no graph).
int enqueue(XGPUBatchImpl *b, const std::vector<Job> &table, int total, Job *d_jobs, int grid,
            int pair) {
  for (size_t q = 0; q < table.size(); ++q) {
    if (!b->jobs[q].accumulate && !table[q].store)
      BCHECK(cudaMemsetAsync(table[q].state, 0, (size_t)b->sizes[q].state_elems * 8, b->stream));
  }
  int max_steps = 0;
  for (const Job &j : table) max_steps = j.steps_per_split > max_steps ? j.steps_per_split : max_steps;
  if (pair)
    BCHECK(launch_tc2_batch(d_jobs, (int)table.size(), total, b->d_queue, b->d_err, grid, b->stream,
                            max_steps));
  else
    BCHECK(launch_tc_batch(d_jobs, (int)table.size(), total, b->d_queue, b->d_err, grid, b->stream));
  return XGPU_OK;
}

int upload(XGPUBatchImpl *b, const std::vector<Job> &table, Job *d_jobs) {
  BCHECK(cudaMemcpyAsync(d_jobs, table.data(), table.size() * sizeof(Job), cudaMemcpyHostToDevice,
                         b->stream));
  BCHECK(cudaStreamSynchronize(b->stream));
  return XGPU_OK;
}

std::mutex g_tune_mutex;
struct Tuned {
  int max_steps, grid, pair;
};
std::map<std::vector<long long>, Tuned> g_tune_cache;   // shape key -> tuning

std::vector<long long> shape_key(const XGPUBatchImpl *b) {
  std::vector<long long> k;
  for (const Sizes &s : b->sizes) {
    k.push_back(s.n);
    k.push_back(s.f);
    k.push_back(s.t);
  }
  return k;
}

// Time candidate (max_steps, grid) pairs on scratch integration buffers and
// keep the fastest.  The caller's buffers are not touched.
int autotune(XGPUBatchImpl *b) {
  const std::vector<long long> key = shape_key(b);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      b->max_steps = it->second.max_steps;
      b->grid = it->second.grid;
      b->pair = it->second.pair;
      return XGPU_OK;
    }
  }
  const int sms = num_sms(b->device);
  std::vector<int64_t *> scratch(b->jobs.size(), nullptr);
  Job *d_tab = nullptr;
  int rc = XGPU_OK;
  size_t total_bytes = 0;
  for (const Sizes &s : b->sizes) total_bytes += (size_t)s.state_elems * 8;
  char *arena = nullptr;
  if (cudaMalloc(&arena, total_bytes) != cudaSuccess ||
      cudaMalloc(&d_tab, b->jobs.size() * sizeof(Job)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(arena);
    return XGPU_OUT_OF_MEMORY;
  }
  size_t off = 0;
  for (size_t q = 0; q < b->jobs.size(); ++q) {
    scratch[q] = (int64_t *)(arena + off);
    off += (size_t)b->sizes[q].state_elems * 8;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int best_steps = 0, best_grid = sms, best_pair = 0;
  const int steps_cands[] = {0, 64, 32, 16, 8};
  const int grid_cands[] = {sms, (sms * 3 / 4) & ~1};
  std::vector<Job> table;
  for (int cand = 0; cand < 10 && rc == XGPU_OK; ++cand) {
    const int ms = steps_cands[cand % 5], pr = cand / 5;
    int total = 0;
    if ((rc = build_table(b, scratch, ms, pr, table, total)) != XGPU_OK) break;
    if ((rc = upload(b, table, d_tab)) != XGPU_OK) break;
    for (int g : grid_cands) {
      if (g < 2) continue;
      if ((rc = enqueue(b, table, total, d_tab, g, pr)) != XGPU_OK) break;   // warm
      cudaEventRecord(e0, b->stream);
      for (int r = 0; r < 3; ++r)
        if ((rc = enqueue(b, table, total, d_tab, g, pr)) != XGPU_OK) break;
      cudaEventRecord(e1, b->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = XGPU_CUDA_ERROR;
        break;
      }
      float ms_run = 0.f;
      cudaEventElapsedTime(&ms_run, e0, e1);
      if (ms_run < best) {
        best = ms_run;
        best_steps = ms;
        best_grid = g;
        best_pair = pr;
      }
    }
  }
  cudaStreamSynchronize(b->stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_tab);
  cudaFree(arena);
  if (rc != XGPU_OK) return rc;
  b->max_steps = best_steps;
  b->grid = best_grid;
  b->pair = best_pair;
  b->tuned_ms = best / 3.0;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_cache[key] = {best_steps, best_grid, best_pair};
  return XGPU_OK;
}

void destroy(XGPUBatchImpl *b) {
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->d_queue) cudaFree(b->d_queue);
  if (b->d_err) cudaFree(b->d_err);
  if (b->h_err) cudaFreeHost(b->h_err);
  delete b;
}

}  // namespace

extern "C" {

int xgpuBatchCreate(XGPUBatch *out, const XGPUBatchJob *jobs, int njobs, int device, void *stream,
                    int flags) {
  if (!out || !jobs || njobs < 1) return XGPU_INVALID_ARGUMENT;
  *out = nullptr;
  XGPUBatchImpl *b = new (std::nothrow) XGPUBatchImpl();
  if (!b) return XGPU_OUT_OF_MEMORY;
  b->device = device;
  b->stream = (cudaStream_t)stream;
  b->flags = flags;
  b->jobs.assign(jobs, jobs + njobs);
  for (const XGPUBatchJob &j : b->jobs) {
    XGPUConfig c;
    xgpuDefaultConfig(&c);
    c.nstation = j.nstation;
    c.nfrequency = j.nfrequency;
    c.ntime = j.ntime;
    c.ntimepipe = 16;
    c.matrix_order = TRIANGULAR_ORDER;
    // xgpuInitEx's ranges for each job (sample and channel counts included:
    // the planner counts stages and items in int)
    if (!j.device_input || !j.device_state || ((uintptr_t)j.device_input & 15) ||
        ((uintptr_t)j.device_state & 15) || !validate_config(c)) {
      delete b;
      return XGPU_INVALID_ARGUMENT;
    }
    b->sizes.push_back(make_sizes(c));
  }
  auto fail = [&](int code) {
    destroy(b);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail(XGPU_CUDA_ERROR);
  if (tc_check_device() != cudaSuccess) {
    cudaGetLastError();
    return fail(XGPU_CUDA_ERROR);
  }
  if (cudaMalloc(&b->d_jobs, njobs * sizeof(Job)) != cudaSuccess ||
      cudaMalloc(&b->d_queue, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&b->h_err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XGPU_OUT_OF_MEMORY);
  }
  if (cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream) != cudaSuccess)
    return fail(XGPU_CUDA_ERROR);
  b->grid = num_sms(device);
  b->max_steps = 0;
  b->pair = (flags & XGPU_BATCH_PAIR) ? 1 : 0;
  if (flags & XGPU_BATCH_AUTOTUNE) {
    int r = autotune(b);
    if (r != XGPU_OK) return fail(r);
  }
  std::vector<int64_t *> states;
  for (const XGPUBatchJob &j : b->jobs) states.push_back((int64_t *)j.device_state);
  std::vector<Job> &table = b->table;
  int r = build_table(b, states, b->max_steps, b->pair, table, b->total_items);
  if (r != XGPU_OK) return fail(r);
  if ((r = upload(b, table, b->d_jobs)) != XGPU_OK) return fail(r);
  if (flags & XGPU_BATCH_GRAPH) {
    // Capture clears, queue reset and the kernel once; xgpuBatchRun replays.
    cudaStream_t cs;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
      return fail(XGPU_CUDA_ERROR);
    cudaStream_t keep = b->stream;
    b->stream = cs;
    bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) ok = enqueue(b, table, b->total_items, b->d_jobs, b->grid, b->pair) == XGPU_OK;
    cudaGraph_t g = nullptr;
    ok = (cudaStreamEndCapture(cs, &g) == cudaSuccess) && ok;
    b->stream = keep;
    cudaStreamDestroy(cs);
    if (!ok || !g) {
      if (g) cudaGraphDestroy(g);
      return fail(XGPU_CUDA_ERROR);
    }
    b->graph = g;
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) return fail(XGPU_CUDA_ERROR);
  }
  *out = b;
  return XGPU_OK;
}

int xgpuBatchRun(XGPUBatch b) {
  if (!b) return XGPU_NOT_INITIALIZED;
  BCHECK(cudaSetDevice(b->device));
  if (b->exec) {
    BCHECK(cudaGraphLaunch(b->exec, b->stream));
    return XGPU_OK;
  }
  return enqueue(b, b->table, b->total_items, b->d_jobs, b->grid, b->pair);
}

int xgpuBatchSync(XGPUBatch b) {
  if (!b) return XGPU_NOT_INITIALIZED;
  BCHECK(cudaSetDevice(b->device));
  BCHECK(cudaStreamSynchronize(b->stream));
  BCHECK(cudaMemcpyAsync(b->h_err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCHECK(cudaStreamSynchronize(b->stream));
  if (*b->h_err) {
    fprintf(stderr, "xgpu batch: device wait timed out (code %d)\n", *b->h_err);
    BCHECK(cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream));
    BCHECK(cudaStreamSynchronize(b->stream));
    return XGPU_CUDA_ERROR;
  }
  return XGPU_OK;
}

int xgpuBatchInfo(XGPUBatch b, int *work_items, int *grid, int *max_steps) {
  if (!b) return XGPU_NOT_INITIALIZED;
  if (work_items) *work_items = b->total_items;
  if (grid) *grid = b->grid;
  // stages per item, negative when the CTA-pair kernel runs (-1: pairs, unsplit)
  if (max_steps) *max_steps = b->pair ? -1 - b->max_steps : b->max_steps;
  return XGPU_OK;
}

void xgpuBatchDestroy(XGPUBatch b) {
  if (b) destroy(b);
}

}  // extern "C"
