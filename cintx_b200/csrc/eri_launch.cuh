// Launch helpers for the per-class ERI kernels.
#pragma once
#include <cuda_runtime.h>
#include <type_traits>
#include "eri_kernel.cuh"

namespace cintx {

struct LaunchArgs {
  const QuartetRec* recs;
  int nrec;
  const ShellPair* pairs;
  const PrimPair* prims;
  double* out;
  OutStrides st;
  double expcutoff;
  RysTable rys;
  cudaStream_t stream;
  int max_blocks;  // grid cap (0: derived from the SM count)
  int query = 0;   // 1: launch nothing; return cudaErrorNotSupported if the class needs scratch
  bool fp32 = false;  // FP32 recurrences and products (spherical output only)
  double prim_eps = 0;  // primitive Schwarz threshold (0: no primitive screening beyond libcint's)
  int variant = 0;      // launch-shape variant (spherical FP64 classes; see variant_acc)
  const double* rootbuf = nullptr;     // precomputed roots [record's base + (b*npij + a)*2*NR]
  const long long* rootbase = nullptr;  // per record of this launch: its base in rootbuf
};

// Device scratch for classes whose transform buffers live in global memory: returns a buffer
// of at least `bytes` owned by the calling host thread (ordered by that thread's launches).
double* class_scratch(size_t bytes);

// A class is compiled when both pairs are oriented (la >= lb) and the first pair is not
// lower than the second in (la, lb) order.
__host__ __device__ constexpr bool class_valid(int li, int lj, int lk, int ll) {
  return li >= lj && lk >= ll && (li > lk || (li == lk && lj >= ll));
}

int device_sm_count();

}  // namespace cintx
#include "eri_splitcoop.cuh"
namespace cintx {

template <int LI, int LJ, int LK, int LL, bool SPH, class R = double, int ACC = 24, int REGS = 128,
          bool SLICE = false, bool ROLL = false, int PASSES = 1>
cudaError_t launch_eri(const LaunchArgs& a) {
  using SH = EriShape<LI, LJ, LK, LL, SPH, R, ACC, REGS, SLICE, ROLL, PASSES>;
  if (a.query) return SH::GLOBAL_BUF ? cudaErrorNotSupported : cudaSuccess;
  auto kern = eri4c_kernel<LI, LJ, LK, LL, SPH, R, ACC, REGS, SLICE, ROLL, PASSES>;
  static int attr_done[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (SH::SMEM_BYTES > 48 * 1024 && dev < 64 && !attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SH::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    attr_done[dev] = 1;
  }
  if (a.nrec <= 0) return cudaSuccess;
  long long blocks = ((long long)a.nrec + SH::Q - 1) / SH::Q;
  long long cap = a.max_blocks > 0 ? a.max_blocks : (long long)device_sm_count() * 32;
  if (blocks > cap) blocks = cap;
  double* scratch = nullptr;
  if constexpr (SH::GLOBAL_BUF) {
    if (blocks > 2LL * device_sm_count()) blocks = 2LL * device_sm_count();
    scratch = class_scratch(sizeof(double) * (size_t)SH::GBUF_PER_BLOCK * (size_t)blocks);
    if (!scratch) return cudaErrorMemoryAllocation;
  }
  kern<<<(unsigned)blocks, SH::BLOCK, SH::SMEM_BYTES, a.stream>>>(a.recs, a.nrec, a.pairs, a.prims, a.out,
                                                                   a.st, a.expcutoff, a.rys, scratch, a.prim_eps,
                                                                   a.rootbuf, a.rootbase);
  return cudaGetLastError();
}

template <int N, class F>
__host__ inline void static_for(F&& f) {
  if constexpr (N > 0) {
    static_for<N - 1>(f);
    f(std::integral_constant<int, N - 1>{});
  }
}

// Dispatch over (lk, ll) for a fixed (li, lj); cudaErrorInvalidValue for classes that are not
// compiled.
template <int LI, int LJ>
cudaError_t dispatch_lij(int lk, int ll, bool sph, const LaunchArgs& a) {
  cudaError_t err = cudaErrorInvalidValue;
  static_for<CINTX_LMAX + 1>([&](auto K) {
    static_for<K.value + 1>([&](auto L) {
      constexpr int k = decltype(K)::value, l = decltype(L)::value;
      if constexpr (class_valid(LI, LJ, k, l)) {
        if (lk == k && ll == l) {
          // variants that give the default shape (lanes, and for multi-lane shapes the register
          // cap) are not compiled separately
          constexpr int s0 = pick_threads(LI, LJ, k, l, variant_acc(0));
          constexpr int s1 = pick_threads(LI, LJ, k, l, variant_acc(1));
          constexpr int s2 = pick_threads(LI, LJ, k, l, variant_acc(2));
          // only shapes that differ from the default are instantiated (if constexpr)
          bool done = false;
          if (a.fp32) {
            err = sph ? launch_eri<LI, LJ, k, l, true, float>(a) : cudaErrorInvalidValue;
            done = true;
          } else if (!sph) {
            err = launch_eri<LI, LJ, k, l, false>(a);
            done = true;
          }
          if constexpr (s1 != s0 || s1 > 1) {
            if (!done && a.variant == 1) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(1), variant_regs(1)>(a);
              done = true;
            }
          }
          if constexpr (s2 != s0) {
            if (!done && a.variant == 2) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(2)>(a);
              done = true;
            }
          }
          if constexpr (s0 > 1) {
            if (!done && a.variant == 3) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(3), variant_regs(3)>(a);
              done = true;
            }
          }
          if constexpr (sliced_ok(LI, LJ, k, l, 4)) {
            if (!done && a.variant == 4) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(4), variant_regs(4), true>(a);
              done = true;
            }
          }
          if constexpr (sliced_ok(LI, LJ, k, l, 5)) {
            if (!done && a.variant == 5) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(5), variant_regs(5), true>(a);
              done = true;
            }
          }
          if constexpr (sliced_ok(LI, LJ, k, l, 6)) {
            if (!done && a.variant == 6) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(6), variant_regs(6), true>(a);
              done = true;
            }
          }
          if constexpr (sliced_ok(LI, LJ, k, l, 7)) {
            if (!done && a.variant == 7) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(7), variant_regs(7), true, true>(a);
              done = true;
            }
          }
          if constexpr (sliced_ok(LI, LJ, k, l, 8)) {
            if (!done && a.variant == 8) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(8), variant_regs(8), true, true>(a);
              done = true;
            }
          }
          if constexpr (sliced_ok(LI, LJ, k, l, 9)) {
            if (!done && a.variant == 9) {
              err = launch_eri<LI, LJ, k, l, true, double, variant_acc(9), variant_regs(9), true, true,
                               variant_passes(9)>(a);
              done = true;
            }
          }
          if constexpr (splitcoop_dims(LI, LJ, k, l, splitcoop_acc(10)).ok) {
            if (!done && a.variant == 10) {
              err = launch_splitcoop<LI, LJ, k, l, splitcoop_acc(10)>(a);
              done = true;
            }
          }
          if constexpr (splitcoop_dims(LI, LJ, k, l, splitcoop_acc(11)).ok) {
            if (!done && a.variant == 11) {
              err = launch_splitcoop<LI, LJ, k, l, splitcoop_acc(11)>(a);
              done = true;
            }
          }
          if (!done) err = launch_eri<LI, LJ, k, l, true>(a);
        }
      }
    });
  });
  return err;
}

#define CINTX_DECL_DISPATCH(I, J) cudaError_t dispatch_l##I##J(int, int, bool, const LaunchArgs&);
CINTX_DECL_DISPATCH(0, 0)
CINTX_DECL_DISPATCH(1, 0) CINTX_DECL_DISPATCH(1, 1)
CINTX_DECL_DISPATCH(2, 0) CINTX_DECL_DISPATCH(2, 1) CINTX_DECL_DISPATCH(2, 2)
CINTX_DECL_DISPATCH(3, 0) CINTX_DECL_DISPATCH(3, 1) CINTX_DECL_DISPATCH(3, 2) CINTX_DECL_DISPATCH(3, 3)
CINTX_DECL_DISPATCH(4, 0) CINTX_DECL_DISPATCH(4, 1) CINTX_DECL_DISPATCH(4, 2) CINTX_DECL_DISPATCH(4, 3)
CINTX_DECL_DISPATCH(4, 4)
#undef CINTX_DECL_DISPATCH

inline cudaError_t dispatch_eri(int li, int lj, int lk, int ll, bool sph, const LaunchArgs& a) {
  if (li > CINTX_LMAX || !class_valid(li, lj, lk, ll)) return cudaErrorInvalidValue;
  switch (li * 10 + lj) {
    case 0: return dispatch_l00(lk, ll, sph, a);
    case 10: return dispatch_l10(lk, ll, sph, a);
    case 11: return dispatch_l11(lk, ll, sph, a);
    case 20: return dispatch_l20(lk, ll, sph, a);
    case 21: return dispatch_l21(lk, ll, sph, a);
    case 22: return dispatch_l22(lk, ll, sph, a);
    case 30: return dispatch_l30(lk, ll, sph, a);
    case 31: return dispatch_l31(lk, ll, sph, a);
    case 32: return dispatch_l32(lk, ll, sph, a);
    case 33: return dispatch_l33(lk, ll, sph, a);
    case 40: return dispatch_l40(lk, ll, sph, a);
    case 41: return dispatch_l41(lk, ll, sph, a);
    case 42: return dispatch_l42(lk, ll, sph, a);
    case 43: return dispatch_l43(lk, ll, sph, a);
    case 44: return dispatch_l44(lk, ll, sph, a);
  }
  return cudaErrorInvalidValue;
}

}  // namespace cintx
