// Class dispatch entry used by the host code (kept in a CUDA translation unit).
#include "eri_launch.cuh"
#include "host_internal.h"

namespace cintx {

cudaError_t launch_class(int li, int lj, int lk, int ll, bool sph, const QuartetRec* recs, int nrec,
                         const ShellPair* pairs, const PrimPair* prims, double* out, OutStrides st,
                         double expcutoff, const RysTable& rys, cudaStream_t stream, bool fp32,
                         double prim_eps, int variant, const double* rootbuf, const long long* rootbase) {
  LaunchArgs a;
  a.recs = recs;
  a.nrec = nrec;
  a.pairs = pairs;
  a.prims = prims;
  a.out = out;
  a.st = st;
  a.expcutoff = expcutoff;
  a.rys = rys;
  a.stream = stream;
  a.max_blocks = 0;
  a.fp32 = fp32;
  a.prim_eps = prim_eps;
  a.variant = variant;
  a.rootbuf = rootbuf;
  a.rootbase = rootbase;
  return dispatch_eri(li, lj, lk, ll, sph, a);
}

static_assert(kNumVariants == kLaunchVariants, "variant count differs between kernel and host headers");

// a split-transfer variant (10, 11) that is not compiled for the class runs the default shape
static bool splitcoop_applies(int li, int lj, int lk, int ll, int variant) {
  return variant_splitcoop(variant) && li <= CINTX_LMAX && splitcoop_dims(li, lj, lk, ll, splitcoop_acc(variant)).ok;
}

int variant_lanes(int li, int lj, int lk, int ll, bool sph, bool fp32, int variant) {
  if (!sph || fp32 || variant <= 0 || variant >= kNumVariants) variant = 0;
  if (variant_splitcoop(variant))
    return splitcoop_applies(li, lj, lk, ll, variant) ? pick_threads(li, lj, lk, ll, splitcoop_acc(variant))
                                                      : pick_threads(li, lj, lk, ll, variant_acc(0));
  if (variant_sliced(variant) && !sliced_ok(li, lj, lk, ll, variant)) variant = 0;
  return pick_threads(li, lj, lk, ll, variant_acc(variant)) / variant_passes(variant);
}

int variant_shape(int li, int lj, int lk, int ll, bool sph, bool fp32, int variant) {
  if (!sph || fp32 || variant <= 0 || variant >= kNumVariants) variant = 0;
  if (variant_splitcoop(variant)) {
    if (!splitcoop_applies(li, lj, lk, ll, variant)) variant = 0;
    else return (1 << 23) + pick_threads(li, lj, lk, ll, splitcoop_acc(variant)) * 1024 + kSplitCoopRegs;
  }
  if (variant_sliced(variant) && !sliced_ok(li, lj, lk, ll, variant)) variant = 0;
  const int s = pick_threads(li, lj, lk, ll, variant_acc(variant));
  if (s == 1) return 1;  // one-lane shapes take no register cap
  return (variant_sliced(variant) ? 1 << 20 : 0) + (variant_roll(variant) ? 1 << 21 : 0) +
         (variant_passes(variant) > 1 ? 1 << 22 : 0) + s * 1024 +
         variant_regs(variant);
}

bool class_needs_scratch(int li, int lj, int lk, int ll, bool sph, int variant) {
  LaunchArgs a{};
  a.query = 1;
  a.variant = variant;
  return dispatch_eri(li, lj, lk, ll, sph, a) == cudaErrorNotSupported;
}

}  // namespace cintx
