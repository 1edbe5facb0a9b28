// Kernels and dispatch for classes whose first shell pair has angular momenta (2, 1).
#include "eri_launch.cuh"
namespace cintx {
cudaError_t dispatch_l21(int lk, int ll, bool sph, const LaunchArgs& a) {
  return dispatch_lij<2, 1>(lk, ll, sph, a);
}
}  // namespace cintx
