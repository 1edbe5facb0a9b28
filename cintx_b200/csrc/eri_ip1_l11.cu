// Derivative (int2e_ip1 / int3c2e_ip1) kernels with first pair (l1 l1): one translation unit per
// pair class so nvcc compiles the instances in parallel.
#include "eri_ip1.cuh"
namespace cintx {
cudaError_t dispatch_ip1_l11(int lk, int ll, bool sph, const Ip1Args& a) { return dispatch_ip1_lij<1, 1>(lk, ll, sph, a); }
}  // namespace cintx
