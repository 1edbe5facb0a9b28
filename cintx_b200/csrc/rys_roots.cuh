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

// Device layout (transposed from the file at upload): per order n, interval i, function f the
// DEG+1 monomial coefficients are contiguous (16-byte aligned), so one function costs
// (DEG+1)/2 vector loads.
constexpr int RYS_NC = CINTX_RYS_DEG + 1;  // coefficients per function (even)

// Doubles per interval of an order-n coefficient block staged in shared memory: the 2n*RYS_NC
// coefficients plus 2 of padding, so that the interval stride is an odd number of 16-byte units
// (12n + 1) and the 16-byte loads of lanes reading different intervals spread over the banks
// (unpadded, stride 12n units: lanes 2 intervals apart, n odd, or any two lanes, n even, collide).
__host__ __device__ constexpr int rys_stage_stride(int n) { return 2 * n * RYS_NC + 2; }

__device__ __forceinline__ double rys_horner(const double* __restrict__ c, double z) {
  const double2* c2 = reinterpret_cast<const double2*>(c);
  const double2 hi = __ldg(c2 + RYS_NC / 2 - 1);
  double acc = fma(hi.y, z, hi.x);
#pragma unroll
  for (int k = RYS_NC / 2 - 2; k >= 0; --k) {
    const double2 v = __ldg(c2 + k);
    acc = fma(acc, z, v.y);
    acc = fma(acc, z, v.x);
  }
  return acc;
}

// Function f of order n at x: f < n -> t^2 of root f, else weight of root f - n.
__device__ __forceinline__ double rys_fn(const RysTable& c_rys, int n, int f, double x) {
  const int xmax = c_rys.xmax[n];
  if (!(x < (double)xmax)) {  // also routes NaN away from the table index
    const double* a = c_rys.asym[n];
    return f < n ? __ldg(a + f) / x : __ldg(a + f) * rsqrt(x);
  }
  const int i = (int)x;
  const double z = 2.0 * (x - (double)i) - 1.0;
  return rys_horner(c_rys.poly[n] + ((size_t)i * 2 * n + f) * RYS_NC, z);
}

// Functions [F0, F1) of order N at once (one thread); F0 = N, F1 = 2N gives the weights only.
template <int N, int F0 = 0, int F1 = 2 * N>
__device__ __forceinline__ void rys_all(const RysTable& c_rys, double x, double* t2, double* w) {
  const int xmax = c_rys.xmax[N];
  if (!(x < (double)xmax)) {  // also routes NaN away from the table index
    const double* a = c_rys.asym[N];
    const double rs = rsqrt(x);
    const double inv = rs * rs;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      if (F0 <= r) t2[r] = __ldg(a + r) * inv;
      w[r] = __ldg(a + N + r) * rs;
    }
    return;
  }
  const int i = (int)x;
  const double z = 2.0 * (x - (double)i) - 1.0;
  const double* c = c_rys.poly[N] + (size_t)i * 2 * N * RYS_NC;
#pragma unroll
  for (int f = F0; f < F1; ++f) {
    const double v = rys_horner(c + f * RYS_NC, z);
    if (f < N) t2[f] = v;
    else w[f - N] = v;
  }
}

// As rys_all, with the order-N coefficient block (cintx_rys_xmax(N) intervals, rys_stage_stride(N)
// doubles apart) staged in shared memory at `tab`; only the large-x limit reads global memory.
template <int N, int F0 = 0, int F1 = 2 * N>
__device__ __forceinline__ void rys_all_staged(const double* tab, const RysTable& c_rys, double x, double* t2,
                                               double* w) {
  constexpr int xmax = cintx_rys_xmax(N);
  if (!(x < (double)xmax)) {  // also routes NaN away from the table index
    const double* a = c_rys.asym[N];
    const double rs = rsqrt(x);
    const double inv = rs * rs;
#pragma unroll
    for (int r = 0; r < N; ++r) {
      if (F0 <= r) t2[r] = __ldg(a + r) * inv;
      w[r] = __ldg(a + N + r) * rs;
    }
    return;
  }
  const int i = (int)x;
  const double z = 2.0 * (x - (double)i) - 1.0;
  const double* c = tab + (size_t)i * rys_stage_stride(N);
  auto horner = [&](int f) {
    const double2* c2 = reinterpret_cast<const double2*>(c + f * RYS_NC);
    const double2 hi = c2[RYS_NC / 2 - 1];
    double acc = fma(hi.y, z, hi.x);
#pragma unroll
    for (int k = RYS_NC / 2 - 2; k >= 0; --k) {
      const double2 v = c2[k];
      acc = fma(acc, z, v.y);
      acc = fma(acc, z, v.x);
    }
    return acc;
  };
  // one root (its t^2 and weight polynomials) in flight at a time: the compiler barrier keeps
  // the other roots' coefficient loads from being hoisted into registers ahead of use
#pragma unroll
  for (int r = 0; r < N; ++r) {
    if (F0 <= r) t2[r] = horner(r);
    if (N + r < F1) w[r] = horner(N + r);
    if (r + 1 < N) asm volatile("" ::: "memory");
  }
}

// As rys_fn for order N, with the coefficient block staged in shared memory at `tab`.
template <int N>
__device__ __forceinline__ double rys_fn_staged(const double* tab, const RysTable& c_rys, int f, double x) {
  constexpr int xmax = cintx_rys_xmax(N);
  if (!(x < (double)xmax)) {  // also routes NaN away from the table index
    const double* a = c_rys.asym[N];
    return f < N ? __ldg(a + f) / x : __ldg(a + f) * rsqrt(x);
  }
  const int i = (int)x;
  const double z = 2.0 * (x - (double)i) - 1.0;
  const double2* c2 = reinterpret_cast<const double2*>(tab + (size_t)i * rys_stage_stride(N) + f * RYS_NC);
  const double2 hi = c2[RYS_NC / 2 - 1];
  double acc = fma(hi.y, z, hi.x);
#pragma unroll
  for (int k = RYS_NC / 2 - 2; k >= 0; --k) {
    const double2 v = c2[k];
    acc = fma(acc, z, v.y);
    acc = fma(acc, z, v.x);
  }
  return acc;
}
