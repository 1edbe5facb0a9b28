// FP64 FMA throughput probe: the denominator of the FP64-pipe roofline.  Each thread runs
// `iters` rounds of 8 independent dependent-FMA chains; the result is written so the work
// cannot be removed.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cintx_cuda.h"

__global__ void fp64_fma_probe_kernel(int iters, double seed, double* out) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
  double a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double m = 0.999999999, c = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

extern "C" int cintx_fp64_fma_probe(int blocks, int threads, int iters, double* out_dev, void* stream) {
  fp64_fma_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, 1.0, out_dev);
  return cudaGetLastError() == cudaSuccess ? 0 : CINTX_STATUS_EXECUTION_FAILED;
}
