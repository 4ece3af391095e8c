// serve.cpp -- continuous-batching correlation server.
//
// Requests are subarray integrations: (stations, channels, samples per block,
// number of blocks) arriving at given times, whose blocks of input become
// available one block period (samples / sample rate) apart.  The server
//  * admits requests in arrival order as soon as their HBM footprint (int64
//    integration buffer + dump buffer) fits in the device arena, and keeps
//    their integration state resident until their last dump;
//  * every step, takes the available blocks (up to four) of every admitted
//    request -- requests that arrived while others run join the next step --
//    and runs all of them in ONE launch of the persistent CTA-pair tensor-core
//    kernel (engine_tc2.cu, 256x256 tiles)
//    through a device job table, so the work of different requests overlaps
//    on the GPU;  blocks of one request in one step add their partial sums
//    exactly (bulk reduce-add);
//  * after a request's last block (and every `dump_every` blocks) formats its
//    buffer to triangular int32 on the device and copies it to pinned host
//    memory on a separate stream, measuring the dump latency from the moment
//    the block's samples were available to the moment the dump is in host
//    memory.
// Samples reach HBM the way a network card or F-engine would put them there,
// without SM work: every block reads a slice of a receive pool filled once,
// before the clock starts, with seeded Gaussian samples (one pool per sigma
// bucket 4, 8, 16, 32; block b of a request with seed s starts at byte
// 256 * (splitmix64(s * 1000003 + b) mod 2^20) of the stream of seed
// 0x5EED0000 + bucket), so every block is reproducible on the host.
// A second mode runs the same stream one request at a time with the plain
// CUDA-core dp4a engine, the reference-style baseline.
//
// xGPU has no counterpart (one compile-time shape per library, no
// scheduler); the per-request arithmetic is the same X-engine.
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <vector>

#include "internal.h"

using namespace xgpu;

namespace {

// First-fit arena over one big allocation (device or pinned host).
class Arena {
 public:
  bool init(size_t bytes, bool device) {
    device_ = device;
    void *p = nullptr;
    cudaError_t e = device ? cudaMalloc(&p, bytes) : cudaMallocHost(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    base_ = (char *)p;
    size_ = bytes;
    free_[0] = bytes;
    return true;
  }
  ~Arena() {
    if (base_) {
      if (device_) cudaFree(base_); else cudaFreeHost(base_);
    }
  }
  // 256-byte aligned block, or nullptr.
  char *alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > bytes) free_[off + bytes] = len - bytes;
        used_ += bytes;
        peak_ = std::max(peak_, used_);
        sizes_[off] = bytes;
        return base_ + off;
      }
    }
    return nullptr;
  }
  void release(char *p) {
    if (!p) return;
    size_t off = (size_t)(p - base_);
    auto s = sizes_.find(off);
    if (s == sizes_.end()) return;
    size_t len = s->second;
    sizes_.erase(s);
    used_ -= len;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + len == next->first) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    free_[off] = len;
  }
  size_t peak() const { return peak_; }

 private:
  bool device_ = true;
  char *base_ = nullptr;
  size_t size_ = 0, used_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;   // offset -> length
  std::map<size_t, size_t> sizes_;  // offset -> length of live blocks
};

double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

struct Active {
  int id;
  Sizes s;
  const XGPUServeJob *spec;
  char *state = nullptr, *dump = nullptr;  // device
  char *host = nullptr;                    // pinned host dump
  int bucket = 0;            // receive pool
  int next_block = 0;        // next block to correlate
  int in_flight = 0;         // steps queued on the GPU with blocks of this request
  int dumps_pending = 0;
  bool finished = false;     // last block queued
  double period = 0.0;       // seconds per block
  double integration = 0.0;  // seconds per integration (nblocks blocks)
};

constexpr double kSigmas[4] = {4.0, 8.0, 16.0, 32.0};
constexpr size_t kPoolSpan = (size_t)256 << 20;   // offsets span 256 MiB
constexpr int kMaxBlocksPerStep = 4;
// Work per step (X-engine ops): about 2.5 ms of the tensor-core engine, so a
// burst of large blocks cannot hold up the requests queued behind it.
constexpr double kStepOps = 4.0e12;

int sigma_bucket(double sigma) {
  int best = 0;
  for (int q = 1; q < 4; ++q)
    if (std::fabs(std::log2(sigma) - std::log2(kSigmas[q])) <
        std::fabs(std::log2(sigma) - std::log2(kSigmas[best])))
      best = q;
  return best;
}

size_t block_offset(unsigned long long seed, int block) {
  unsigned long long z = seed * 1000003ull + (unsigned long long)block + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (size_t)256 * (size_t)(z % (1ull << 20));
}

struct PendingDump {
  int job;
  cudaEvent_t ev;
  double available;   // when the samples of the dump's last block were available
  double period;      // integration period of the request
  bool final_dump;
};

struct Step {
  cudaEvent_t done;
  std::vector<int> jobs;
};

#define SCHECK(call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "(CUDA) %s (%s:%d)\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      rc = XGPU_CUDA_ERROR;                                                            \
      goto done;                                                                       \
    }                                                                                  \
  } while (0)

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (v.size() - 1);
  const size_t lo = (size_t)std::floor(pos), hi = std::min(v.size() - 1, lo + 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - lo);
}

}  // namespace

extern "C" int xgpuServeRun(const XGPUServeJob *jobs, int njobs, const XGPUServeOptions *opt_in,
                            XGPUServeStats *stats, int **results) {
  if (!jobs || njobs < 1 || !opt_in || !stats) return XGPU_INVALID_ARGUMENT;
  const XGPUServeOptions opt = *opt_in;
  if (!(opt.sample_rate_hz > 0) || opt.device_budget_bytes < (1u << 20)) return XGPU_INVALID_ARGUMENT;
  for (int q = 0; q < njobs; ++q) {
    const XGPUServeJob &j = jobs[q];
    if (j.nstation < 16 || j.nstation % 16 || j.nstation > 8192 || j.nfrequency < 1 ||
        j.nfrequency > 65535 || j.ntime < 16 || j.ntime % 16 || j.ntime > kSegment ||
        j.nblocks < 1 || j.arrival_s < 0 ||
        !(j.sigma > 0) ||
        (q > 0 && j.arrival_s < jobs[q - 1].arrival_s))
      return XGPU_INVALID_ARGUMENT;
  }
  memset(stats, 0, sizeof(*stats));
  const bool plain = opt.mode == XGPU_SERVE_PLAIN_SERIAL;
  int rc = XGPU_OK;
  Arena dev, host;
  cudaStream_t s_step = nullptr, s_dump = nullptr;
  Job *d_tables = nullptr, *h_tables = nullptr;
  int *d_queue = nullptr, *d_err = nullptr, h_err = 0;
  const int kTables = 2;
  int max_table = njobs * kMaxBlocksPerStep;
  std::vector<Active> act;                 // admitted, not retired
  std::deque<int> waiting;                 // arrived, not admitted
  std::deque<Step> steps;                  // in flight
  std::vector<PendingDump> dumps;
  std::vector<double> lat_ms, ratio;
  std::vector<cudaEvent_t> event_pool;
  char *pool[4] = {nullptr, nullptr, nullptr, nullptr};
  int next_arrival = 0, retired = 0, table_slot = 0;
  double t0 = 0, ops_done = 0, last_done = 0, busy_start = -1, busy_s = 0;
  long long blocks_done = 0, admitted_peak = 0, late = 0, dumps_total = 0;
  int sms = 0;
  auto get_event = [&]() {
    cudaEvent_t e;
    if (!event_pool.empty()) {
      e = event_pool.back();
      event_pool.pop_back();
    } else {
      cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
    return e;
  };

  SCHECK(cudaSetDevice(opt.device));
  SCHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt.device));
  if (!plain && tc_check_device() != cudaSuccess) {
    cudaGetLastError();
    return XGPU_CUDA_ERROR;
  }
  if (!dev.init(opt.device_budget_bytes, true)) return XGPU_OUT_OF_MEMORY;
  if (!host.init(opt.host_budget_bytes ? opt.host_budget_bytes : ((size_t)8 << 30), false))
    return XGPU_OUT_OF_MEMORY;
  SCHECK(cudaStreamCreateWithFlags(&s_step, cudaStreamNonBlocking));
  SCHECK(cudaStreamCreateWithFlags(&s_dump, cudaStreamNonBlocking));
  SCHECK(cudaMalloc(&d_tables, sizeof(Job) * max_table * kTables));
  SCHECK(cudaMallocHost(&h_tables, sizeof(Job) * max_table * kTables));
  SCHECK(cudaMalloc(&d_queue, sizeof(int) * kTables));
  SCHECK(cudaMalloc(&d_err, sizeof(int)));
  SCHECK(cudaMemsetAsync(d_err, 0, sizeof(int), s_step));
  {
    size_t need[4] = {0, 0, 0, 0};
    for (int q = 0; q < njobs; ++q) {
      const int b = sigma_bucket(jobs[q].sigma);
      need[b] = std::max(need[b], (size_t)4 * jobs[q].nstation * jobs[q].nfrequency * jobs[q].ntime);
    }
    for (int b = 0; b < 4; ++b) {
      if (!need[b]) continue;
      const size_t bytes = kPoolSpan + ((need[b] + 255) & ~(size_t)255);
      SCHECK(cudaMalloc(&pool[b], bytes));
      SCHECK(launch_generate(pool[b], bytes, 0, 0x5EED0000ull + b, kSigmas[b], s_step));
    }
  }
  SCHECK(cudaStreamSynchronize(s_step));

  t0 = now_s();
  while (retired < njobs) {
    const double t = now_s() - t0;
    // 1. arrivals
    while (next_arrival < njobs && jobs[next_arrival].arrival_s <= t) waiting.push_back(next_arrival++);
    // 2. admission by footprint, in arrival order
    while (!waiting.empty() && (!plain || act.empty())) {
      const int id = waiting.front();
      const XGPUServeJob &j = jobs[id];
      XGPUConfig c;
      xgpuDefaultConfig(&c);
      c.nstation = j.nstation;
      c.nfrequency = j.nfrequency;
      c.ntime = j.ntime;
      c.ntimepipe = 16;
      c.matrix_order = TRIANGULAR_ORDER;
      Active a;
      a.id = id;
      a.spec = &j;
      a.s = make_sizes(c);
      a.state = dev.alloc((size_t)a.s.state_elems * 8);
      a.dump = a.state ? dev.alloc((size_t)a.s.tri_length * 8) : nullptr;
      a.host = a.dump ? host.alloc((size_t)a.s.tri_length * 8) : nullptr;
      if (!a.host) {
        dev.release(a.state);
        dev.release(a.dump);
        break;   // wait until memory frees up
      }
      a.bucket = sigma_bucket(j.sigma);
      a.period = (double)j.ntime / opt.sample_rate_hz;
      a.integration = a.period * j.nblocks;
      act.push_back(a);
      waiting.pop_front();
      admitted_peak = std::max<long long>(admitted_peak, (long long)act.size());
    }
    // 3. completed steps
    while (!steps.empty() && cudaEventQuery(steps.front().done) == cudaSuccess) {
      for (int id : steps.front().jobs)
        for (Active &a : act)
          if (a.id == id) a.in_flight--;
      event_pool.push_back(steps.front().done);
      steps.pop_front();
      if (steps.empty() && busy_start >= 0) {
        busy_s += now_s() - busy_start;
        busy_start = -1;
      }
    }
    // 4. completed dumps
    for (size_t k = 0; k < dumps.size();) {
      if (cudaEventQuery(dumps[k].ev) != cudaSuccess) {
        ++k;
        continue;
      }
      const double tn = now_s() - t0;
      const double l = tn - dumps[k].available;
      lat_ms.push_back(l * 1e3);
      ratio.push_back(l / dumps[k].period);
      if (l > dumps[k].period) late++;
      last_done = tn;
      dumps_total++;
      event_pool.push_back(dumps[k].ev);
      for (size_t q = 0; q < act.size(); ++q) {
        Active &a = act[q];
        if (a.id != dumps[k].job) continue;
        a.dumps_pending--;
        if (dumps[k].final_dump) {
          if (results && results[a.id])
            memcpy(results[a.id], a.host, (size_t)a.s.tri_length * 8);
          dev.release(a.state);
          dev.release(a.dump);
          host.release(a.host);
          act.erase(act.begin() + q);
          retired++;
        }
        break;
      }
      dumps.erase(dumps.begin() + k);
    }
    // 5. next step: the available blocks of every admitted request
    if (steps.size() < (size_t)kTables) {
      std::vector<std::pair<int, int>> ready;   // (request index, blocks this step)
      struct Cand {
        int q, cnt;
        bool completes;   // the step would finish an integration (or a dump period)
        double avail;     // availability of its first block
        double ops;
      };
      std::vector<Cand> cands;
      const double tn = now_s() - t0;
      for (size_t q = 0; q < act.size(); ++q) {
        Active &a = act[q];
        if (a.finished || a.in_flight > 0) continue;
        int cnt = 0;
        const int cap = (plain || a.spec->dump_every) ? 1 : kMaxBlocksPerStep;
        while (cnt < cap && a.next_block + cnt < (int)a.spec->nblocks &&
               a.spec->arrival_s + (a.next_block + cnt + 1) * a.period <= tn)
          ++cnt;
        if (!cnt) continue;
        const int after = a.next_block + cnt;
        Cand c{(int)q, cnt,
               after == (int)a.spec->nblocks || (a.spec->dump_every && after % a.spec->dump_every == 0),
               a.spec->arrival_s + (a.next_block + 1) * a.period,
               cnt * 16.0 * a.s.f * a.s.t * a.s.n * (a.s.n + 1.0)};
        cands.push_back(c);
        if (plain) break;
      }
      // Dumps due first, then oldest samples first, within the step's work cap.
      std::sort(cands.begin(), cands.end(), [](const Cand &x, const Cand &y) {
        if (x.completes != y.completes) return x.completes;
        return x.avail < y.avail;
      });
      double step_ops = 0.0;
      for (const Cand &c : cands) {
        if (!ready.empty() && step_ops + c.ops > kStepOps) break;
        ready.push_back({c.q, c.cnt});
        step_ops += c.ops;
      }
      if (!ready.empty()) {
        Step st;
        st.done = get_event();
        Job *tab = h_tables + (size_t)table_slot * max_table;
        int items = 0, nent = 0;
        for (const auto &rq : ready) {
          Active &a = act[rq.first];
          const XGPUServeJob &j = *a.spec;
          const bool first = a.next_block == 0;
          if (!plain && first && rq.second > 1)
            SCHECK(cudaMemsetAsync(a.state, 0, (size_t)a.s.state_elems * 8, s_step));
          for (int k = 0; k < rq.second; ++k) {
            const int b = a.next_block + k;
            const char *x = pool[a.bucket] + block_offset(j.seed, b);
            if (plain) {
              SCHECK(launch_plain_dp4a((const int8_t *)x, a.s, 0, a.s.t, (int64_t *)a.state,
                                       b == 0, s_step, d_err));
            } else {
              Job &jb = tab[nent++];
              if (tc_fill_job(&jb, x, a.s, 0, a.s.t, (int64_t *)a.state,
                              (first && rq.second == 1) ? 1 : 0, 1, items, 1) != 0) {
                rc = XGPU_CUDA_ERROR;
                goto done;
              }
              items += jb.items;
            }
            ops_done += 16.0 * a.s.f * a.s.t * a.s.n * (a.s.n + 1.0);
            blocks_done++;
          }
        }
        if (!plain) {
          Job *dtab = d_tables + (size_t)table_slot * max_table;
          SCHECK(cudaMemcpyAsync(dtab, tab, sizeof(Job) * nent, cudaMemcpyHostToDevice, s_step));
          int max_steps = 0;
          for (int q = 0; q < nent; ++q)
            max_steps = tab[q].steps_per_split > max_steps ? tab[q].steps_per_split : max_steps;
          SCHECK(launch_tc2_batch(dtab, nent, items, d_queue + table_slot, d_err, sms, s_step,
                                  max_steps));
        }
        table_slot = (table_slot + 1) % kTables;
        for (const auto &rq : ready) {
          Active &a = act[rq.first];
          const XGPUServeJob &j = *a.spec;
          a.next_block += rq.second;
          const int b = a.next_block - 1;   // last block of this step
          a.in_flight++;
          st.jobs.push_back(a.id);
          const bool last = (a.next_block == (int)j.nblocks);
          if (last) a.finished = true;
          if (last || (j.dump_every && (a.next_block % j.dump_every) == 0)) {
            // format on the step stream, copy on the dump stream
            SCHECK(launch_format(a.state, 0, a.s, TRIANGULAR_ORDER, XGPU_INT32, a.dump, s_step));
            cudaEvent_t fe = get_event();
            SCHECK(cudaEventRecord(fe, s_step));
            SCHECK(cudaStreamWaitEvent(s_dump, fe, 0));
            SCHECK(cudaMemcpyAsync(a.host, a.dump, (size_t)a.s.tri_length * 8,
                                   cudaMemcpyDeviceToHost, s_dump));
            PendingDump pd;
            pd.job = a.id;
            pd.ev = get_event();
            SCHECK(cudaEventRecord(pd.ev, s_dump));
            pd.available = j.arrival_s + (b + 1) * a.period;
            pd.period = a.integration;
            pd.final_dump = last;
            a.dumps_pending++;
            dumps.push_back(pd);
            event_pool.push_back(fe);   // reusable once recorded work passes; only waited on
            // A periodic dump's buffer is rewritten by the next dump of this request:
            // the step stream waits for this copy before formatting again.
            if (!last) SCHECK(cudaStreamWaitEvent(s_step, pd.ev, 0));
          }
        }
        SCHECK(cudaEventRecord(st.done, s_step));
        if (busy_start < 0) busy_start = now_s();
        steps.push_back(st);
        continue;
      }
    }
    // nothing to launch: wait briefly
    if (!steps.empty() || !dumps.empty()) usleep(50);
    else if (next_arrival < njobs || !act.empty()) usleep(100);
  }
  SCHECK(cudaStreamSynchronize(s_step));
  SCHECK(cudaStreamSynchronize(s_dump));
  SCHECK(cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h_err) {
    fprintf(stderr, "xgpuServeRun: device wait timed out (code %d)\n", h_err);
    rc = XGPU_CUDA_ERROR;
  }
  stats->jobs = njobs;
  stats->blocks = blocks_done;
  stats->dumps = dumps_total;
  stats->ops = ops_done;
  stats->wall_s = last_done;
  stats->tops = last_done > 0 ? ops_done / last_done / 1e12 : 0.0;
  stats->gpu_busy_s = busy_s;
  stats->dump_p50_ms = percentile(lat_ms, 0.50);
  stats->dump_p99_ms = percentile(lat_ms, 0.99);
  stats->dump_max_ms = lat_ms.empty() ? 0.0 : *std::max_element(lat_ms.begin(), lat_ms.end());
  stats->period_ratio_p99 = percentile(ratio, 0.99);
  stats->late_dumps = late;
  stats->admitted_peak = admitted_peak;
  stats->device_peak_bytes = (double)dev.peak();

done:
  if (s_step) cudaStreamSynchronize(s_step);
  if (s_dump) cudaStreamSynchronize(s_dump);
  for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
  for (PendingDump &d : dumps) cudaEventDestroy(d.ev);
  for (Step &s : steps) cudaEventDestroy(s.done);
  for (int b = 0; b < 4; ++b)
    if (pool[b]) cudaFree(pool[b]);
  if (d_tables) cudaFree(d_tables);
  if (h_tables) cudaFreeHost(h_tables);
  if (d_queue) cudaFree(d_queue);
  if (d_err) cudaFree(d_err);
  if (s_step) cudaStreamDestroy(s_step);
  if (s_dump) cudaStreamDestroy(s_dump);
  return rc;
}
