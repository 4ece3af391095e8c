// tc_job.h -- one unit of work for the tensor-core engine: an input buffer
// (through its TMA tensor map), a sample range and an int64 integration
// buffer.  A launch runs one job (passed as a kernel parameter) or a table of
// jobs in device memory (uneven batches); each job is cut into work items of
// (channel, time split, 128x128 tile).
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace xgpu {

constexpr int kTcSamplesPerStage = 128;

struct Job {
  CUtensorMap map;        // 3-D map {4n bytes, f, t} over the job's int8 input (64-byte aligned)
  int64_t *state;         // triangular int64 integration buffer of the job
  long long nbaseline;    // n(n+1)/2
  int n, f;               // stations; channels of the job's channel range
  int f0;                 // first channel of the range (channel index into the input and buffer)
  int t0;                 // first sample of the range
  int total_steps;        // pipeline stages (of kTcSamplesPerStage samples) in the range
  int steps_per_split;    // stages per time split
  int ksplit;             // time splits (each adds its partial sums into the buffer)
  int npairs;             // lower-triangle tiles per channel
  int items;              // f * npairs * ksplit
  int item_begin;         // first work item of this job in the launch
  int store;              // 1: sole writer of a zero buffer (store); 0: reduce-add
};

struct TcTuning {
  int ksplit = 1;         // time splits per tile (1 = none)
  int grid = 0;           // CTAs (0 = one per SM)
  int wide = 0;           // 1: CTA-pair kernel with 256x256 tiles (cta_group::2)
  int stall = 0;          // test switch: withhold input loads so the bounded waits expire
  int streamk = 0;        // single-CTA kernel: equal shares of all tile steps per CTA
                          // (used for launches that add into existing sums)
};

}  // namespace xgpu
