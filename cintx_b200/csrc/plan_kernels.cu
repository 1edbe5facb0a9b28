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

// Coulomb/exchange contraction of one chunk of a unique-quartet sweep (a >= b, c >= d, ab >= cd):
// one warp per quartet block v[i + ni*(j + nj*(k + nk*l))] (shells a, b, c, d), with the 8-fold
// permutational symmetry of real integrals and a symmetric density D (row-major nao x nao):
//   A[i,j] += 2 s sum_kl v D[k,l],  A[k,l] += 2 s sum_ij v D[i,j]          (J = A + A^T)
//   B[i,k] += s sum_jl v D[j,l],  B[j,k] += s sum_il v D[i,l],
//   B[i,l] += s sum_jk v D[j,k],  B[j,l] += s sum_ik v D[i,k]               (K = B + B^T)
// with s = 1/2 for each of a == b, c == d, (ab) == (cd) (those blocks hold every element twice).
// Each (row, column) pair of a block reduces its sum first and adds it with one atomic.
__global__ void jk_contract_kernel(const QuartetRec* __restrict__ recs, long long nrec, const int2* __restrict__ psh,
                                   const int* __restrict__ aoloc, const double* __restrict__ out,
                                   const double* __restrict__ dm, int nao, double* __restrict__ A,
                                   double* __restrict__ B) {
  const int lane = threadIdx.x & 31;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nrec;
       r += ((long long)gridDim.x * blockDim.x) >> 5) {
    const QuartetRec rec = recs[r];
    const int2 ab = psh[rec.pij], cd = psh[rec.pkl];
    const int i0 = aoloc[ab.x], j0 = aoloc[ab.y], k0 = aoloc[cd.x], l0 = aoloc[cd.y];
    const int ni = aoloc[ab.x + 1] - i0, nj = aoloc[ab.y + 1] - j0;
    const int nk = aoloc[cd.x + 1] - k0, nl = aoloc[cd.y + 1] - l0;
    const double s = (ab.x == ab.y ? 0.5 : 1.0) * (cd.x == cd.y ? 0.5 : 1.0) * (rec.pij == rec.pkl ? 0.5 : 1.0);
    const double* v = out + rec.out;
    const int sj = ni, sk = ni * nj, sl = ni * nj * nk;
    if (A) {
      for (int e = lane; e < ni * nj; e += 32) {
        const int i = e % ni, j = e / ni;
        double t = 0.0;
        for (int l = 0; l < nl; ++l)
          for (int k = 0; k < nk; ++k) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(k0 + k) * nao + l0 + l];
        atomicAdd(A + (size_t)(i0 + i) * nao + j0 + j, 2.0 * s * t);
      }
      for (int e = lane; e < nk * nl; e += 32) {
        const int k = e % nk, l = e / nk;
        double t = 0.0;
        for (int j = 0; j < nj; ++j)
          for (int i = 0; i < ni; ++i) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(i0 + i) * nao + j0 + j];
        atomicAdd(A + (size_t)(k0 + k) * nao + l0 + l, 2.0 * s * t);
      }
    }
    if (B) {
      for (int e = lane; e < ni * nk; e += 32) {  // B[i,k] += s sum_jl v D[j,l]
        const int i = e % ni, k = e / ni;
        double t = 0.0;
        for (int l = 0; l < nl; ++l)
          for (int j = 0; j < nj; ++j) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(j0 + j) * nao + l0 + l];
        atomicAdd(B + (size_t)(i0 + i) * nao + k0 + k, s * t);
      }
      for (int e = lane; e < nj * nk; e += 32) {  // B[j,k] += s sum_il v D[i,l]
        const int j = e % nj, k = e / nj;
        double t = 0.0;
        for (int l = 0; l < nl; ++l)
          for (int i = 0; i < ni; ++i) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(i0 + i) * nao + l0 + l];
        atomicAdd(B + (size_t)(j0 + j) * nao + k0 + k, s * t);
      }
      for (int e = lane; e < ni * nl; e += 32) {  // B[i,l] += s sum_jk v D[j,k]
        const int i = e % ni, l = e / ni;
        double t = 0.0;
        for (int k = 0; k < nk; ++k)
          for (int j = 0; j < nj; ++j) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(j0 + j) * nao + k0 + k];
        atomicAdd(B + (size_t)(i0 + i) * nao + l0 + l, s * t);
      }
      for (int e = lane; e < nj * nl; e += 32) {  // B[j,l] += s sum_ik v D[i,k]
        const int j = e % nj, l = e / nj;
        double t = 0.0;
        for (int k = 0; k < nk; ++k)
          for (int i = 0; i < ni; ++i) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(i0 + i) * nao + k0 + k];
        atomicAdd(B + (size_t)(j0 + j) * nao + l0 + l, s * t);
      }
    }
  }
}

// Scatters one chunk of a unique-quartet sweep into the 8-fold packed AO tensor
// eri[pq*(pq+1)/2 + rs] (pq = p*(p+1)/2 + q for p >= q, pq >= rs), one warp per quartet block.
// Elements a block holds twice (diagonal shell pairs) map to the same slot and carry equal values.
__global__ void scatter_s8_kernel(const QuartetRec* __restrict__ recs, long long nrec, const int2* __restrict__ psh,
                                  const int* __restrict__ aoloc, const double* __restrict__ out,
                                  double* __restrict__ eri) {
  const int lane = threadIdx.x & 31;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nrec;
       r += ((long long)gridDim.x * blockDim.x) >> 5) {
    const QuartetRec rec = recs[r];
    const int2 ab = psh[rec.pij], cd = psh[rec.pkl];
    const int i0 = aoloc[ab.x], j0 = aoloc[ab.y], k0 = aoloc[cd.x], l0 = aoloc[cd.y];
    const int ni = aoloc[ab.x + 1] - i0, nj = aoloc[ab.y + 1] - j0;
    const int nk = aoloc[cd.x + 1] - k0, nl = aoloc[cd.y + 1] - l0;
    const int n = ni * nj * nk * nl;
    const double* v = out + rec.out;
    for (int e = lane; e < n; e += 32) {
      const int i = e % ni, j = (e / ni) % nj, k = (e / (ni * nj)) % nk, l = e / (ni * nj * nk);
      const long long p = i0 + i, q = j0 + j, u = k0 + k, w = l0 + l;
      const long long pq = p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
      const long long uw = u >= w ? u * (u + 1) / 2 + w : w * (w + 1) / 2 + u;
      eri[pq >= uw ? pq * (pq + 1) / 2 + uw : uw * (uw + 1) / 2 + pq] = v[e];
    }
  }
}

// Scatters one chunk of a unique-quartet sweep into an unpacked AO tensor, one warp per quartet
// block: mode 1 (PySCF ao2mo "s1") eri[((p*nao + q)*nao + r)*nao + s] at all eight index orders
// the quartet stands for; mode 4 ("s4") the pair-pair matrix eri[pq*npair + rs] and its transpose
// slot, pq = p*(p+1)/2 + q over p >= q.  Slots reached twice receive equal elements.
__global__ void scatter_ao_kernel(const QuartetRec* __restrict__ recs, long long nrec, const int2* __restrict__ psh,
                                  const int* __restrict__ aoloc, const double* __restrict__ out,
                                  double* __restrict__ eri, int mode, long long nao) {
  const int lane = threadIdx.x & 31;
  const long long npair = nao * (nao + 1) / 2;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nrec;
       r += ((long long)gridDim.x * blockDim.x) >> 5) {
    const QuartetRec rec = recs[r];
    const int2 ab = psh[rec.pij], cd = psh[rec.pkl];
    const int i0 = aoloc[ab.x], j0 = aoloc[ab.y], k0 = aoloc[cd.x], l0 = aoloc[cd.y];
    const int ni = aoloc[ab.x + 1] - i0, nj = aoloc[ab.y + 1] - j0;
    const int nk = aoloc[cd.x + 1] - k0, nl = aoloc[cd.y + 1] - l0;
    const int n = ni * nj * nk * nl;
    const double* v = out + rec.out;
    for (int e = lane; e < n; e += 32) {
      const int i = e % ni, j = (e / ni) % nj, k = (e / (ni * nj)) % nk, l = e / (ni * nj * nk);
      const long long p = i0 + i, q = j0 + j, u = k0 + k, w = l0 + l;
      const double x = v[e];
      if (mode == 1) {
        const long long pq = p * nao + q, qp = q * nao + p, uw = u * nao + w, wu = w * nao + u;
        const long long n2 = nao * nao;
        eri[pq * n2 + uw] = x;
        eri[qp * n2 + uw] = x;
        eri[pq * n2 + wu] = x;
        eri[qp * n2 + wu] = x;
        eri[uw * n2 + pq] = x;
        eri[wu * n2 + pq] = x;
        eri[uw * n2 + qp] = x;
        eri[wu * n2 + qp] = x;
      } else {
        const long long pq = p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p;
        const long long uw = u >= w ? u * (u + 1) / 2 + w : w * (w + 1) / 2 + u;
        eri[pq * npair + uw] = x;
        eri[uw * npair + pq] = x;
      }
    }
  }
}

// As jk_contract_kernel for small blocks (all of one class, n = ni nj nk nl <= 32 elements): one
// thread per quartet, so the many tiny blocks ((ss|ss), (ps|ss), ...) do not idle a warp each.
__global__ void jk_contract_small_kernel(const QuartetRec* __restrict__ recs, long long nrec,
                                         const int2* __restrict__ psh, const int* __restrict__ aoloc,
                                         const double* __restrict__ out, const double* __restrict__ dm, int nao,
                                         double* __restrict__ A, double* __restrict__ B) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nrec; r += (long long)gridDim.x * blockDim.x) {
    const QuartetRec rec = recs[r];
    const int2 ab = psh[rec.pij], cd = psh[rec.pkl];
    const int i0 = aoloc[ab.x], j0 = aoloc[ab.y], k0 = aoloc[cd.x], l0 = aoloc[cd.y];
    const int ni = aoloc[ab.x + 1] - i0, nj = aoloc[ab.y + 1] - j0;
    const int nk = aoloc[cd.x + 1] - k0, nl = aoloc[cd.y + 1] - l0;
    const double s = (ab.x == ab.y ? 0.5 : 1.0) * (cd.x == cd.y ? 0.5 : 1.0) * (rec.pij == rec.pkl ? 0.5 : 1.0);
    const double* v = out + rec.out;
    const int sj = ni, sk = ni * nj, sl = ni * nj * nk;
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        double tj = 0.0;  // A[i,j]
        for (int l = 0; l < nl; ++l)
          for (int k = 0; k < nk; ++k) tj += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(k0 + k) * nao + l0 + l];
        if (A) atomicAdd(A + (size_t)(i0 + i) * nao + j0 + j, 2.0 * s * tj);
      }
    if (A)
      for (int l = 0; l < nl; ++l)
        for (int k = 0; k < nk; ++k) {
          double t = 0.0;
          for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(i0 + i) * nao + j0 + j];
          atomicAdd(A + (size_t)(k0 + k) * nao + l0 + l, 2.0 * s * t);
        }
    if (B) {
      for (int k = 0; k < nk; ++k) {
        for (int i = 0; i < ni; ++i) {  // B[i,k] += s sum_jl v D[j,l]
          double t = 0.0;
          for (int l = 0; l < nl; ++l)
            for (int j = 0; j < nj; ++j) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(j0 + j) * nao + l0 + l];
          atomicAdd(B + (size_t)(i0 + i) * nao + k0 + k, s * t);
        }
        for (int j = 0; j < nj; ++j) {  // B[j,k] += s sum_il v D[i,l]
          double t = 0.0;
          for (int l = 0; l < nl; ++l)
            for (int i = 0; i < ni; ++i) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(i0 + i) * nao + l0 + l];
          atomicAdd(B + (size_t)(j0 + j) * nao + k0 + k, s * t);
        }
      }
      for (int l = 0; l < nl; ++l) {
        for (int i = 0; i < ni; ++i) {  // B[i,l] += s sum_jk v D[j,k]
          double t = 0.0;
          for (int k = 0; k < nk; ++k)
            for (int j = 0; j < nj; ++j) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(j0 + j) * nao + k0 + k];
          atomicAdd(B + (size_t)(i0 + i) * nao + l0 + l, s * t);
        }
        for (int j = 0; j < nj; ++j) {  // B[j,l] += s sum_ik v D[i,k]
          double t = 0.0;
          for (int k = 0; k < nk; ++k)
            for (int i = 0; i < ni; ++i) t += v[i + j * sj + k * sk + l * sl] * dm[(size_t)(i0 + i) * nao + k0 + k];
          atomicAdd(B + (size_t)(j0 + j) * nao + l0 + l, s * t);
        }
      }
    }
  }
}

// M[p,q] = X[p,q] + X[q,p] (n x n), for J = A + A^T and K = B + B^T.
__global__ void symmetrize_kernel(const double* __restrict__ X, double* __restrict__ M, int n) {
  const long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(e / n), q = (int)(e % n);
    M[e] = X[e] + X[(size_t)q * n + p];
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

cudaError_t launch_jk_contract(const QuartetRec* recs, long long nrec, const int2* psh, const int* aoloc,
                               const double* out, const double* dm, int nao, double* A, double* B, cudaStream_t stream,
                               int block_elems) {
  if (nrec <= 0) return cudaSuccess;
  if (block_elems > 0 && block_elems <= 32) {
    long long blocks = (nrec + 127) / 128;
    if (blocks > 148LL * 64) blocks = 148LL * 64;
    jk_contract_small_kernel<<<(unsigned)blocks, 128, 0, stream>>>(recs, nrec, psh, aoloc, out, dm, nao, A, B);
    return cudaGetLastError();
  }
  long long blocks = (nrec * 32 + 255) / 256;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  jk_contract_kernel<<<(unsigned)blocks, 256, 0, stream>>>(recs, nrec, psh, aoloc, out, dm, nao, A, B);
  return cudaGetLastError();
}

cudaError_t launch_scatter_s8(const QuartetRec* recs, long long nrec, const int2* psh, const int* aoloc,
                              const double* out, double* eri, cudaStream_t stream) {
  if (nrec <= 0) return cudaSuccess;
  long long blocks = (nrec * 32 + 255) / 256;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  scatter_s8_kernel<<<(unsigned)blocks, 256, 0, stream>>>(recs, nrec, psh, aoloc, out, eri);
  return cudaGetLastError();
}

cudaError_t launch_scatter_ao(const QuartetRec* recs, long long nrec, const int2* psh, const int* aoloc,
                              const double* out, double* eri, int mode, long long nao, cudaStream_t stream) {
  if (nrec <= 0) return cudaSuccess;
  long long blocks = (nrec * 32 + 255) / 256;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  scatter_ao_kernel<<<(unsigned)blocks, 256, 0, stream>>>(recs, nrec, psh, aoloc, out, eri, mode, nao);
  return cudaGetLastError();
}

cudaError_t launch_symmetrize(const double* X, double* M, int n, cudaStream_t stream) {
  const long long total = (long long)n * n;
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  if (total > 0) symmetrize_kernel<<<(unsigned)blocks, 256, 0, stream>>>(X, M, n);
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
