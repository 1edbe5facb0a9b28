// Device copy of the Rys root table (rys_table.bin, embedded at link time) and its upload.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>
#include "common.h"

extern "C" const unsigned char cintx_rys_table_bin[];
extern "C" const unsigned char cintx_rys_table_bin_end[];
__asm__(
    ".section .rodata\n"
    ".balign 64\n"
    ".global cintx_rys_table_bin\n"
    "cintx_rys_table_bin:\n"
    ".incbin \"" CINTX_RYS_TABLE_PATH "\"\n"
    ".global cintx_rys_table_bin_end\n"
    "cintx_rys_table_bin_end:\n"
    ".previous\n");

namespace cintx {

// Copies the table to the current device and fills *tab with its device pointers.
// Returns 0 on success.
int upload_rys_table(void** dev_buf, RysTable* tab) {
  const unsigned char* p = cintx_rys_table_bin;
  size_t nbytes = (size_t)(cintx_rys_table_bin_end - cintx_rys_table_bin);
  int64_t hdr[16];
  memcpy(hdr, p, sizeof(hdr));
  const int nmax = (int)hdr[0], deg = (int)hdr[1];
  if (nmax < CINTX_NRMAX || deg != CINTX_RYS_DEG || (deg + 1) % 2) return 1;
  // transpose every interval from [degree][function] (file) to [function][degree] (device)
  std::vector<double> host((nbytes - sizeof(hdr)) / sizeof(double));
  memcpy(host.data(), p + sizeof(hdr), nbytes - sizeof(hdr));
  {
    size_t o = 0;
    std::vector<double> tmp;
    for (int n = 1; n <= nmax; ++n) {
      const int nf = 2 * n, nc = deg + 1;
      const int xmax = (int)hdr[1 + n];
      for (int i = 0; i < xmax; ++i, o += (size_t)nf * nc) {
        tmp.assign(host.begin() + o, host.begin() + o + (size_t)nf * nc);
        for (int k = 0; k < nc; ++k)
          for (int f = 0; f < nf; ++f) host[o + (size_t)f * nc + k] = tmp[(size_t)k * nf + f];
      }
    }
  }
  void* d = nullptr;
  if (cudaMalloc(&d, nbytes) != cudaSuccess) return 2;
  if (cudaMemcpy(d, p, sizeof(hdr), cudaMemcpyHostToDevice) != cudaSuccess) return 3;
  if (cudaMemcpy((char*)d + sizeof(hdr), host.data(), nbytes - sizeof(hdr), cudaMemcpyHostToDevice) != cudaSuccess)
    return 3;
  RysTable t;
  memset(&t, 0, sizeof(t));
  const double* base = (const double*)((const char*)d + sizeof(hdr));
  size_t off = 0;
  for (int n = 1; n <= nmax; ++n) {
    int xmax = (int)hdr[1 + n];
    if (n <= CINTX_NRMAX && xmax != cintx_rys_xmax(n)) return 6;
    if (n <= CINTX_NRMAX) {
      t.poly[n] = base + off;
      t.xmax[n] = xmax;
    }
    off += (size_t)xmax * (deg + 1) * 2 * n;
  }
  for (int n = 1; n <= nmax; ++n) {
    if (n <= CINTX_NRMAX) t.asym[n] = base + off;
    off += 2 * n;
  }
  if (sizeof(hdr) + off * sizeof(double) != nbytes) return 4;
  *tab = t;
  *dev_buf = d;
  return 0;
}

int device_sm_count() {
  static int cached[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && cached[dev]) return cached[dev];
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (dev < 64) cached[dev] = n;
  return n;
}

}  // namespace cintx

#include "rys_roots.cuh"

// Evaluates the 2n root/weight functions at nx points: out[i*2n + f].
__global__ void rys_eval_kernel(const __grid_constant__ RysTable t, int n, const double* __restrict__ x,
                                long long nx, double* __restrict__ out) {
  const long long total = nx * 2 * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx / (2 * n);
    const int f = (int)(idx % (2 * n));
    out[idx] = rys_fn(t, n, f, x[i]);
  }
}

namespace cintx {
cudaError_t rys_eval(const RysTable& t, int n, const double* x, long long nx, double* out,
                     cudaStream_t stream) {
  if (nx <= 0) return cudaSuccess;
  long long total = nx * 2 * n;
  long long blocks = (total + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  rys_eval_kernel<<<(unsigned)blocks, 256, 0, stream>>>(t, n, x, nx, out);
  return cudaGetLastError();
}
}  // namespace cintx
