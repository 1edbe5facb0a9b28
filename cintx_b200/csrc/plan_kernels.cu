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

// Multi-range generation: one launch fills the records of every tile range of a kernel class
// within a chunk.  ranges[] are ordered by rec_off; record r belongs to the last range whose
// rec_off <= r.
__global__ void gen_range_quartets(const GenRange* __restrict__ ranges, int nranges, long long nrec,
                                   QuartetRec* __restrict__ recs) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec;
       r += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nranges - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (ranges[mid].rec_off <= r) lo = mid;
      else hi = mid - 1;
    }
    const GenRange g = ranges[lo];
    const long long t = g.t0 + (r - g.rec_off);
    int a = 0, b = g.nrows - 1;
    while (a < b) {
      const int mid = (a + b + 1) >> 1;
      if (g.prefix[mid] <= t) a = mid;
      else b = mid - 1;
    }
    QuartetRec q;
    const int row = g.rows[a], col = g.cols[(g.colstart ? g.colstart[a] : 0) + (t - g.prefix[a])];
    q.pij = g.swap ? col : row;
    q.pkl = g.swap ? row : col;
    q.out = g.out_off + (r - g.rec_off) * g.nout;
    recs[r] = q;
  }
}

// x = a_ij a_kl / (a_ij + a_kl) |P - Q|^2 of every primitive quartet (b over the (kl) pair's
// primitives, a over the (ij) pair's, the ERI kernels' loop order) of nrec records, written at
// xout[pbase[r] + b * npij + a]; the same expression as the kernels, so the roots computed from
// it are the ones those kernels would evaluate.
__global__ void prim_x_kernel(const QuartetRec* __restrict__ recs, long long nrec, const ShellPair* __restrict__ pairs,
                              const PrimPair* __restrict__ prims, const long long* __restrict__ pbase,
                              double* __restrict__ xout) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec;
       r += (long long)gridDim.x * blockDim.x) {
    const QuartetRec rec = recs[r];
    const ShellPair pij = pairs[rec.pij], pkl = pairs[rec.pkl];
    for (int b = 0; b < pkl.nprim; ++b) {
      const PrimPair pk = prims[pkl.prim_off + b];
      for (int a = 0; a < pij.nprim; ++a) {
        const PrimPair pi = prims[pij.prim_off + a];
        const double aijkl = pi.aij + pk.aij;
        const double rs = rsqrt(aijkl);
        const double pqx = pi.px - pk.px, pqy = pi.py - pk.py, pqz = pi.pz - pk.pz;
        xout[pbase[r] + (long long)b * pij.nprim + a] =
            pi.aij * pk.aij * (rs * rs) * (pqx * pqx + pqy * pqy + pqz * pqz);
      }
    }
  }
}

// q[r] = sqrt(max |out[recs[r].out .. + len[r])|): one warp per record.
__global__ void block_absmax_sqrt_kernel(const QuartetRec* __restrict__ recs, long long nrec,
                                         const double* __restrict__ out, const long long* __restrict__ len,
                                         double* __restrict__ q) {
  const int lane = threadIdx.x & 31;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nrec;
       r += ((long long)gridDim.x * blockDim.x) >> 5) {
    const double* o = out + recs[r].out;
    double m = 0.0;
    for (long long e = lane; e < len[r]; e += 32) m = fmax(m, fabs(o[e]));
    for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
    if (lane == 0) q[r] = sqrt(m);
  }
}

namespace cintx {
cudaError_t launch_prim_x(const QuartetRec* recs, long long nrec, const ShellPair* pairs, const PrimPair* prims,
                          const long long* pbase, double* xout, cudaStream_t stream) {
  if (nrec <= 0) return cudaSuccess;
  long long blocks = (nrec + 127) / 128;
  if (blocks > 65535) blocks = 65535;
  prim_x_kernel<<<(unsigned)blocks, 128, 0, stream>>>(recs, nrec, pairs, prims, pbase, xout);
  return cudaGetLastError();
}

cudaError_t launch_block_absmax_sqrt(const QuartetRec* recs, long long nrec, const double* out, const long long* len,
                                     double* q, cudaStream_t stream) {
  if (nrec <= 0) return cudaSuccess;
  long long blocks = (nrec * 32 + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  block_absmax_sqrt_kernel<<<(unsigned)blocks, 256, 0, stream>>>(recs, nrec, out, len, q);
  return cudaGetLastError();
}

cudaError_t launch_gen_ranges(const GenRange* ranges, int nranges, long long nrec, QuartetRec* recs,
                              cudaStream_t stream) {
  if (nrec <= 0) return cudaSuccess;
  long long blocks = (nrec + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  gen_range_quartets<<<(unsigned)blocks, 256, 0, stream>>>(ranges, nranges, nrec, recs);
  return cudaGetLastError();
}
}  // namespace cintx
