// Shared host/device data layout of the B200 two-electron integral engine.
//
// The basis lives in HBM as structure-of-arrays records built once per CINTOpt
// (int2e_optimizer).  Everything the kernels need per primitive pair is precomputed into a
// 64-byte PrimPair record so the inner primitive loop reads one cache line per pair.
#pragma once
#include <stdint.h>

#define CINTX_LMAX 4          // highest angular momentum with compiled kernels (g)
#define CINTX_NRMAX 9         // highest Rys order: (4+4+4+4)/2 + 1
#define CINTX_RYS_DEG 11      // polynomial degree per unit-width x interval

// Table intervals per order (x < xmax uses the table; the file header must match).
__host__ __device__ constexpr int cintx_rys_xmax(int n) {
  return n == 1 ? 40 : n == 2 ? 52 : n == 3 ? 60 : n == 4 ? 64 : n == 5 ? 72 : n == 6 ? 76 : n == 7 ? 84
       : n == 8 ? 92 : 100;
}

// One primitive pair (a, b) of an oriented shell pair (i, j), after exponent screening.
// kab folds exp(-a_i a_j/a_ij |A-B|^2), both contraction coefficients (single contraction)
// and the pair's share of libcint's common factor sqrt(2 pi^2.5) * fac_sp(li) * fac_sp(lj).
// When q is set, a shell pair's primitive pairs are sorted by decreasing q, so a primitive
// quartet loop can stop at the first pair whose bound q_ab * q_cd falls below its threshold.
struct __align__(64) PrimPair {
  double aij;         // a_i + a_j
  double px, py, pz;  // product centre P = (a_i A + a_j B) / a_ij
  double kab;         // prefactor described above
  double cce;         // libcint screening exponent of this pair (CINTset_pairdata)
  double half_inv;    // 0.5 / a_ij
  double q;           // primitive Schwarz factor |c_i c_j| sqrt(max|(ab|ab)|) (0: not computed)
};

// An oriented shell pair (i, j).  Its primitive pairs are prims[prim_off, prim_off+nprim).
struct __align__(16) ShellPair {
  double ax, ay, az;     // centre of shell i
  double abx, aby, abz;  // A - B
  int prim_off;
  int nprim;
  int ish, jsh;          // shell ids
};

// One shell quartet of a launch: pairs (ij) and (kl) and the start of its output block.
struct __align__(16) QuartetRec {
  int pij;
  int pkl;
  long long out;  // offset in doubles
};

// A contiguous run [t0, t1) of one screened tile's row-major quartet numbering, generating
// records rec_off.. of a merged class segment whose blocks start at out_off (doubles).
struct __align__(16) GenRange {
  const int* rows;
  const int* cols;
  const long long* prefix;
  int nrows;
  int swap;  // nonzero: the column pair is the kernel's first pair (pij)
  long long t0, t1;
  long long rec_off;
  long long out_off;
  long long nout;
  const int* colstart;  // per row: first column of the range's tile (nullptr: 0)
};

// Output placement of one launch group: the element (a, b, c, d) of the canonical block
// (a over shell i components fastest) goes to out + rec.out + a*s0 + b*s1 + c*s2 + d*s3.
struct OutStrides {
  long long s0, s1, s2, s3;
};

// Device Rys table (see gen_rys_table.py for the layout).
struct RysTable {
  const double* poly[CINTX_NRMAX + 1];  // [n] -> [xmax][DEG+1][2n]
  const double* asym[CINTX_NRMAX + 1];  // [n] -> h_r^2 (n), W_r (n)
  int xmax[CINTX_NRMAX + 1];
};

// libcint status semantics and cintx C-ABI status codes (cintx-capi errors.rs:9-21)
enum CintxStatus {
  CINTX_SUCCESS = 0,
  CINTX_INVALID_INPUT = 1,
  CINTX_UNSUPPORTED_API = 2,
  CINTX_UNSUPPORTED_REPRESENTATION = 3,
  CINTX_BUFFER_TOO_SMALL = 4,
  CINTX_MEMORY_LIMIT_EXCEEDED = 5,
  CINTX_ALLOCATION_FAILED = 6,
  CINTX_EXECUTION_FAILED = 7,
  CINTX_NULL_POINTER = 8,
  CINTX_PANIC = 9,
  CINTX_BACKEND_NOT_COMPILED = 10,
};
