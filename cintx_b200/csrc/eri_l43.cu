// Kernels and dispatch for classes whose first shell pair has angular momenta (4, 3).
#include "eri_launch.cuh"
namespace cintx {
cudaError_t dispatch_l43(int lk, int ll, bool sph, const LaunchArgs& a) {
  return dispatch_lij<4, 3>(lk, ll, sph, a);
}
}  // namespace cintx
