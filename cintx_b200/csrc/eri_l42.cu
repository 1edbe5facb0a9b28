// Kernels and dispatch for classes whose first shell pair has angular momenta (4, 2).
#include "eri_launch.cuh"
namespace cintx {
cudaError_t dispatch_l42(int lk, int ll, bool sph, const LaunchArgs& a) {
  return dispatch_lij<4, 2>(lk, ll, sph, a);
}
}  // namespace cintx
