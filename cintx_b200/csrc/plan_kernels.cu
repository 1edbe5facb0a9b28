// Device-side quartet generation for screened plans.
//
// A tile (A, B) of a screened plan pairs every shell pair p of pair type A (sorted by
// decreasing Schwarz factor) with the first count[p] pairs of type B.  Quartets are numbered
// row-major; row_prefix[r] is the first quartet index of row r.  One thread per quartet finds
// its row by binary search and writes the record; out offsets are consecutive blocks.
#include <cuda_runtime.h>

#include "common.h"

__global__ void gen_tile_quartets(const int* __restrict__ rows, const int* __restrict__ cols,
                                  const long long* __restrict__ row_prefix, int nrows, long long t0,
                                  long long t1, long long nout, long long out_base,
                                  QuartetRec* __restrict__ recs) {
  for (long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < t1;
       t += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nrows - 1;  // last row with row_prefix[row] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (row_prefix[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    QuartetRec r;
    r.pij = rows[lo];
    r.pkl = cols[t - row_prefix[lo]];
    r.out = out_base + (t - t0) * nout;
    recs[t - t0] = r;
  }
}

namespace cintx {
cudaError_t launch_gen_tile(const int* rows, const int* cols, const long long* row_prefix, int nrows,
                            long long t0, long long t1, long long nout, long long out_base, QuartetRec* recs,
                            cudaStream_t stream) {
  const long long n = t1 - t0;
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  gen_tile_quartets<<<(unsigned)blocks, 256, 0, stream>>>(rows, cols, row_prefix, nrows, t0, t1, nout, out_base,
                                                           recs);
  return cudaGetLastError();
}
}  // namespace cintx
