// Host-only enumeration of every launch shape the ERI dispatch compiles (test infrastructure).
//
// For each valid class (li lj | lk ll) and each shape dispatch_lij instantiates (spherical FP64
// variants 0..11 where they apply, cartesian FP64, spherical FP32), prints one line
//   li lj lk ll kind variant S LANES BLOCK Q B_GROUP SMEM_BYTES GLOBAL_BUF violation
// where violation is shape_violation<Shape>() for eri4c_kernel's shapes and splitcoop_violation
// for the split-transfer cooperative shapes (variants 10, 11) (0: every shared-memory, scratch,
// barrier and per-thread index the kernel forms from the shape stays inside its buffer).
// Compiled with nvcc as a host program; it launches nothing.
#include <cstdio>

#include "../cintx_b200/csrc/eri_launch.cuh"

using namespace cintx;

template <class SH>
void row(int li, int lj, int lk, int ll, const char* kind, int v) {
  std::printf("%d %d %d %d %s %d %d %d %d %d %d %d %d %d\n", li, lj, lk, ll, kind, v, SH::S, SH::LANES, SH::BLOCK,
              SH::Q, SH::B_GROUP, SH::SMEM_BYTES, (int)SH::GLOBAL_BUF, shape_violation<SH>());
}

template <int LI, int LJ, int LK, int LL>
void shapes_of_class() {
  row<EriShape<LI, LJ, LK, LL, true>>(LI, LJ, LK, LL, "sph", 0);
  row<EriShape<LI, LJ, LK, LL, false>>(LI, LJ, LK, LL, "cart", 0);
  row<EriShape<LI, LJ, LK, LL, true, float>>(LI, LJ, LK, LL, "fp32", 0);
  row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(1), variant_regs(1)>>(LI, LJ, LK, LL, "sph", 1);
  row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(2)>>(LI, LJ, LK, LL, "sph", 2);
  row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(3), variant_regs(3)>>(LI, LJ, LK, LL, "sph", 3);
  if constexpr (sliced_ok(LI, LJ, LK, LL, 4))
    row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(4), variant_regs(4), true>>(LI, LJ, LK, LL, "sph", 4);
  if constexpr (sliced_ok(LI, LJ, LK, LL, 5))
    row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(5), variant_regs(5), true>>(LI, LJ, LK, LL, "sph", 5);
  if constexpr (sliced_ok(LI, LJ, LK, LL, 6))
    row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(6), variant_regs(6), true>>(LI, LJ, LK, LL, "sph", 6);
  if constexpr (sliced_ok(LI, LJ, LK, LL, 7))
    row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(7), variant_regs(7), true, true>>(LI, LJ, LK, LL, "sph",
                                                                                              7);
  if constexpr (sliced_ok(LI, LJ, LK, LL, 8))
    row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(8), variant_regs(8), true, true>>(LI, LJ, LK, LL, "sph",
                                                                                              8);
  if constexpr (sliced_ok(LI, LJ, LK, LL, 9))
    row<EriShape<LI, LJ, LK, LL, true, double, variant_acc(9), variant_regs(9), true, true, variant_passes(9)>>(
        LI, LJ, LK, LL, "sph", 9);
  static_for<2>([&](auto V) {
    constexpr int v = 10 + decltype(V)::value;
    constexpr int acc = splitcoop_acc(v);
    constexpr SplitCoopDims d = splitcoop_dims(LI, LJ, LK, LL, acc);
    if constexpr (d.ok)
      std::printf("%d %d %d %d %s %d %d %d %d %d %d %d %d %d\n", LI, LJ, LK, LL, "sph", v, d.S, d.S, d.BLOCK, d.Q,
                  d.B_GROUP, d.SMEM_BYTES, 0, splitcoop_violation<LI, LJ, LK, LL, acc>());
  });
}

int main() {
  static_for<CINTX_LMAX + 1>([&](auto I) {
    static_for<I.value + 1>([&](auto J) {
      static_for<CINTX_LMAX + 1>([&](auto K) {
        static_for<K.value + 1>([&](auto L) {
          constexpr int i = decltype(I)::value, j = decltype(J)::value, k = decltype(K)::value,
                        l = decltype(L)::value;
          if constexpr (class_valid(i, j, k, l)) shapes_of_class<i, j, k, l>();
        });
      });
    });
  });
  return 0;
}
