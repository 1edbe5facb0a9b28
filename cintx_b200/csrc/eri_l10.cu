// Kernels and dispatch for classes whose first shell pair has angular momenta (1, 0).
#include "eri_launch.cuh"
namespace cintx {
cudaError_t dispatch_l10(int lk, int ll, bool sph, const LaunchArgs& a) {
  return dispatch_lij<1, 0>(lk, ll, sph, a);
}
}  // namespace cintx
