/* Prints the ABI-relevant facts of an xgpu.h: struct sizes, field offsets and
 * macro values, one "name value" pair per line.  Compiled once against the
 * reference header (tests/golden/make_golden.py) and once against
 * include/xgpu.h (tests/test_abi.py); the two outputs must agree. */
#include <stddef.h>
#include <stdio.h>
#include "xgpu.h"

#define P(name, v) printf("%s %lld\n", name, (long long)(v))
#define OFF(T, f) P(#T "." #f, offsetof(T, f))

int main(void) {
  P("sizeof.ComplexInput", sizeof(ComplexInput));
  P("sizeof.Complex", sizeof(Complex));
  P("sizeof.XGPUInfo", sizeof(XGPUInfo));
  P("sizeof.XGPUContext", sizeof(XGPUContext));
  OFF(XGPUInfo, npol); OFF(XGPUInfo, nstation); OFF(XGPUInfo, nbaseline);
  OFF(XGPUInfo, nfrequency); OFF(XGPUInfo, ntime); OFF(XGPUInfo, ntimepipe);
  OFF(XGPUInfo, input_type); OFF(XGPUInfo, compute_type); OFF(XGPUInfo, vecLength);
  OFF(XGPUInfo, vecLengthPipe); OFF(XGPUInfo, matLength); OFF(XGPUInfo, triLength);
  OFF(XGPUInfo, matrix_order); OFF(XGPUInfo, shared_atomic_size);
  OFF(XGPUInfo, complex_block_size);
  OFF(XGPUContext, array_h); OFF(XGPUContext, matrix_h); OFF(XGPUContext, array_len);
  OFF(XGPUContext, matrix_len); OFF(XGPUContext, input_offset);
  OFF(XGPUContext, output_offset); OFF(XGPUContext, internal);
  P("XGPU_INT8", XGPU_INT8); P("XGPU_FLOAT32", XGPU_FLOAT32); P("XGPU_INT32", XGPU_INT32);
  P("TRIANGULAR_ORDER", TRIANGULAR_ORDER);
  P("REAL_IMAG_TRIANGULAR_ORDER", REAL_IMAG_TRIANGULAR_ORDER);
  P("REGISTER_TILE_TRIANGULAR_ORDER", REGISTER_TILE_TRIANGULAR_ORDER);
  P("XGPU_DEVICE_MASK", XGPU_DEVICE_MASK);
  P("XGPU_DONT_REGISTER_ARRAY", XGPU_DONT_REGISTER_ARRAY);
  P("XGPU_DONT_REGISTER_MATRIX", XGPU_DONT_REGISTER_MATRIX);
  P("XGPU_DONT_REGISTER", XGPU_DONT_REGISTER);
  P("XGPU_OK", XGPU_OK); P("XGPU_OUT_OF_MEMORY", XGPU_OUT_OF_MEMORY);
  P("XGPU_CUDA_ERROR", XGPU_CUDA_ERROR);
  P("XGPU_INSUFFICIENT_TEXTURE_MEMORY", XGPU_INSUFFICIENT_TEXTURE_MEMORY);
  P("XGPU_NOT_INITIALIZED", XGPU_NOT_INITIALIZED);
  P("XGPU_HOST_BUFFER_NOT_SET", XGPU_HOST_BUFFER_NOT_SET);
  P("SYNCOP_NONE", SYNCOP_NONE); P("SYNCOP_DUMP", SYNCOP_DUMP);
  P("SYNCOP_SYNC_TRANSFER", SYNCOP_SYNC_TRANSFER); P("SYNCOP_SYNC_COMPUTE", SYNCOP_SYNC_COMPUTE);
#ifdef FIXED_POINT
  P("FIXED_POINT", 1);
#endif
  return 0;
}
