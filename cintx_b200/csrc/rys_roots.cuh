// Device Rys roots and weights.
//
// For order n and parameter x the n roots t_r^2 (ascending) and weights w_r of
//     int_0^1 exp(-x t^2) P(t^2) dt = sum_r w_r P(t_r^2)
// are the quantities libcint's CINTrys_roots computes (rys_roots.c:57; it returns
// u = t^2/(1-t^2)).  Here they come from a piecewise polynomial table (unit-width intervals
// in x, degree CINTX_RYS_DEG in z = 2(x-i)-1, generated in 50-digit arithmetic by
// gen_rys_table.py) for x < xmax[n], and from the exact large-x limit
// t_r^2 = h_r^2 / x, w_r = W_r / sqrt(x) (positive Gauss-Hermite nodes of order 2n) beyond.
#pragma once
#include "common.h"

// Function f of order n at x: f < n -> t^2 of root f, else weight of root f - n.
__device__ __forceinline__ double rys_fn(const RysTable& c_rys, int n, int f, double x) {
  const int xmax = c_rys.xmax[n];
  if (!(x < (double)xmax)) {  // also routes NaN away from the table index
    const double* a = c_rys.asym[n];
    return f < n ? __ldg(a + f) / x : __ldg(a + f) * rsqrt(x);
  }
  const int i = (int)x;
  const double z = 2.0 * (x - (double)i) - 1.0;
  const double* c = c_rys.poly[n] + (size_t)i * (CINTX_RYS_DEG + 1) * 2 * n + f;
  double acc = __ldg(c + CINTX_RYS_DEG * 2 * n);
#pragma unroll
  for (int k = CINTX_RYS_DEG - 1; k >= 0; --k) acc = fma(acc, z, __ldg(c + k * 2 * n));
  return acc;
}

// All 2n functions at once (one thread).  Coefficient rows are contiguous per degree.
template <int N>
__device__ __forceinline__ void rys_all(const RysTable& c_rys, double x, double* t2, double* w) {
  const int xmax = c_rys.xmax[N];
  if (!(x < (double)xmax)) {  // also routes NaN away from the table index
    const double* a = c_rys.asym[N];
    const double inv = 1.0 / x;
    const double rs = rsqrt(x);
#pragma unroll
    for (int r = 0; r < N; ++r) {
      t2[r] = __ldg(a + r) * inv;
      w[r] = __ldg(a + N + r) * rs;
    }
    return;
  }
  const int i = (int)x;
  const double z = 2.0 * (x - (double)i) - 1.0;
  const double* c = c_rys.poly[N] + (size_t)i * (CINTX_RYS_DEG + 1) * 2 * N;
  double acc[2 * N];
#pragma unroll
  for (int f = 0; f < 2 * N; ++f) acc[f] = __ldg(c + CINTX_RYS_DEG * 2 * N + f);
#pragma unroll
  for (int k = CINTX_RYS_DEG - 1; k >= 0; --k) {
#pragma unroll
    for (int f = 0; f < 2 * N; ++f) acc[f] = fma(acc[f], z, __ldg(c + k * 2 * N + f));
  }
#pragma unroll
  for (int r = 0; r < N; ++r) {
    t2[r] = acc[r];
    w[r] = acc[N + r];
  }
}
