// Device copy of the Rys root table (rys_table.bin, embedded at link time) and its upload.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>
#include "common.h"
#include "host_internal.h"

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

// Reads the embedded table: checks its header against the layout the kernels are compiled for
// (order >= CINTX_NRMAX, degree CINTX_RYS_DEG, the interval counts of cintx_rys_xmax, a payload
// of exactly the size the header implies), and returns the payload transposed from the file's
// [degree][function] order to the [function][degree] order the device reads, with each order's
// polynomial block and asymptotic constants as offsets (doubles) into it.  0 on success.
int rys_table_image(std::vector<double>& payload, RysTableOffsets& offs) {
  const unsigned char* p = cintx_rys_table_bin;
  const size_t nbytes = (size_t)(cintx_rys_table_bin_end - cintx_rys_table_bin);
  int64_t hdr[16];
  if (nbytes < sizeof(hdr)) return 4;
  memcpy(hdr, p, sizeof(hdr));
  const int nmax = (int)hdr[0], deg = (int)hdr[1];
  // hdr[1 + n] holds the interval count of order n: at most 14 orders fit the 16-entry header
  if (nmax < CINTX_NRMAX || nmax > 14 || deg != CINTX_RYS_DEG || (deg + 1) % 2) return 1;
  size_t total = 0;
  for (int n = 1; n <= nmax; ++n) {
    const int xmax = (int)hdr[1 + n];
    if (xmax < 0 || (n <= CINTX_NRMAX && xmax != cintx_rys_xmax(n))) return 6;
    total += (size_t)xmax * (deg + 1) * 2 * n + 2 * n;
  }
  if (sizeof(hdr) + total * sizeof(double) != nbytes) return 4;
  payload.resize(total);
  memcpy(payload.data(), p + sizeof(hdr), total * sizeof(double));
  memset(&offs, 0, sizeof(offs));
  size_t o = 0;
  std::vector<double> tmp;
  const int nc = deg + 1;
  for (int n = 1; n <= nmax; ++n) {
    const int nf = 2 * n, xmax = (int)hdr[1 + n];
    if (n <= CINTX_NRMAX) {
      offs.poly[n] = o;
      offs.xmax[n] = xmax;
    }
    for (int i = 0; i < xmax; ++i, o += (size_t)nf * nc) {
      tmp.assign(payload.begin() + o, payload.begin() + o + (size_t)nf * nc);
      for (int k = 0; k < nc; ++k)
        for (int f = 0; f < nf; ++f) payload[o + (size_t)f * nc + k] = tmp[(size_t)k * nf + f];
    }
  }
  for (int n = 1; n <= nmax; ++n) {
    if (n <= CINTX_NRMAX) offs.asym[n] = o;
    o += 2 * n;
  }
  return o == total ? 0 : 4;
}

// Copies the table to the current device and fills *tab with its device pointers.
// Returns 0 on success.
int upload_rys_table(void** dev_buf, RysTable* tab) {
  std::vector<double> host;
  RysTableOffsets offs;
  const int rc = rys_table_image(host, offs);
  if (rc) return rc;
  void* d = nullptr;
  if (cudaMalloc(&d, host.size() * sizeof(double)) != cudaSuccess) return 2;
  if (cudaMemcpy(d, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return 3;
  }
  RysTable t;
  memset(&t, 0, sizeof(t));
  const double* base = (const double*)d;
  for (int n = 1; n <= CINTX_NRMAX; ++n) {
    t.poly[n] = base + offs.poly[n];
    t.asym[n] = base + offs.asym[n];
    t.xmax[n] = offs.xmax[n];
  }
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
