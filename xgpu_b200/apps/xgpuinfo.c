/* xgpuinfo -- print the build's default sizes of libxgpu.so.
 *
 * The line labels are the ones xGPU's xgpuinfo prints (src/xgpuinfo.c:5-67),
 * because autoconf macros of downstream pipelines scrape them
 * (src/xgpu.m4:57-67: "Number of stations: ", "Number of frequencies: ",
 * "time samples per GPU integration: ").  Two lines are added at the end: the
 * engine xgpuInit selects and the runtime-sizing extension. */
#include <stdio.h>

#include "xgpu.h"

static const char *type_name(unsigned int t) {
  switch (t) {
    case XGPU_INT8: return "8 bit integers";
    case XGPU_FLOAT32: return "32 bit floats";
    case XGPU_INT32: return "32 bit integers";
    default: return "<unknown>";
  }
}

static const char *order_name(unsigned int o) {
  switch (o) {
    case TRIANGULAR_ORDER: return "triangular";
    case REAL_IMAG_TRIANGULAR_ORDER: return "real imaginary triangular";
    case REGISTER_TILE_TRIANGULAR_ORDER: return "register tile triangular";
    default: return "<unknown>";
  }
}

int main(void) {
  XGPUInfo info;
  XGPUConfig cfg;
  xgpuInfo(&info);
  xgpuDefaultConfig(&cfg);
  printf("xGPU library version: %s\n", xgpuVersionString());
  printf("Number of polarizations: %u\n", info.npol);
  printf("Number of stations: %u\n", info.nstation);
  printf("Number of baselines: %u\n", info.nbaseline);
  printf("Number of frequencies: %u\n", info.nfrequency);
  printf("Number of time samples per GPU integration: %u\n", info.ntime);
  printf("Number of time samples per transfer to GPU: %u\n", info.ntimepipe);
  printf("Type of ComplexInput components: %s\n", type_name(info.input_type));
  printf("Type of computation: %s\n", info.compute_type == XGPU_INT8
                                          ? "8 bit multiply, 32-bit accumulate"
                                          : "FP32 multiply, FP32 accumulate");
  printf("Number of ComplexInput elements in GPU input vector: %llu\n", info.vecLength);
  printf("Number of ComplexInput elements per transfer to GPU: %llu\n", info.vecLengthPipe);
  printf("Number of Complex elements in GPU output vector: %llu\n", info.matLength);
  printf("Number of Complex elements in reordered output vector: %llu\n", info.triLength);
  printf("Output matrix order: %s\n", order_name(info.matrix_order));
  printf("Shared atomic transfer size: %lu\n", (unsigned long)info.shared_atomic_size);
  printf("Complex block size: %lu\n", (unsigned long)info.complex_block_size);
  printf("Default engine: %s, %s Complex output, int64 integration buffer\n",
         cfg.engine == XGPU_ENGINE_PLAIN ? "CUDA-core 2x2 register tile"
                                         : "tcgen05 int8 tensor cores",
         cfg.output_type == XGPU_INT32 ? "int32" : "float32");
  printf("Runtime sizing: xgpuInitEx (any NSTATION multiple of 16, NFREQUENCY, NTIME)\n");
  return 0;
}
