// Learned Rys-root initializer and its FP64 refinement.
//
// RysNet is a small MLP in FP32: inputs (nroots, log x), two hidden layers of 64 SiLU units and
// 18 outputs, read as logit(u_i) (outputs 0..8) and log(w_i) (outputs 9..17) for the n Rys roots
// u_i = t_i^2 and weights w_i of order n.  It is trained on the device by the kernels below
// (sample generation from the table path, a fused forward+backward kernel, Adam) and gives the
// starting point of an FP64 refinement:
//   1. the recurrence coefficients (alpha_k, beta_k), k < n, of the Rys measure
//      e^{-x u} / (2 sqrt(u)) du on [0, 1] are computed by the Stieltjes procedure on its 64-node
//      Gauss-Legendre discretisation (rys_gl64.h), i.e. from the measure's moment
//      (orthogonality) conditions;
//   2. Newton steps with the Aberth correction on the degree-n orthogonal polynomial p_n
//      (evaluated with its derivative by the three-term recurrence) move all n roots together
//      from the network's guess to full accuracy;
//   3. the weights follow from the Christoffel function, w_i = 1 / sum_{k<n} q_k(u_i)^2 with
//      q_k the orthonormal polynomials.
// A point whose refinement does not converge within 8 steps, leaves (0, 1) or yields two equal
// roots takes the table path (rys_roots.cuh) instead and is counted as a fallback (n distinct
// zeros of p_n in (0, 1) are all of them, so passing the checks means the right roots).  x beyond the table range uses the table path's closed-form
// large-x limit, as the plain path does.  The reference's plain path for the same quantities is
// CINTrys_roots (libcint rys_roots.c; cintx-cubecl math/rys.rs, math/rys_wheeler.rs).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/cintx_cuda.h"
#include "common.h"
#include "host_internal.h"
#include "rys_gl64.h"
#include "rys_roots.cuh"

namespace cintx {

constexpr int RN_IN = 2, RN_H = 64, RN_OUT = 18, RN_HALF = 9;
constexpr int RN_W1 = 0;                        // [64][2]
constexpr int RN_B1 = RN_W1 + RN_H * RN_IN;     // [64]
constexpr int RN_W2 = RN_B1 + RN_H;             // [64][64] (out, in)
constexpr int RN_B2 = RN_W2 + RN_H * RN_H;      // [64]
constexpr int RN_W3 = RN_B2 + RN_H;             // [18][64]
constexpr int RN_B3 = RN_W3 + RN_OUT * RN_H;    // [18]
constexpr int RN_NPARAM = RN_B3 + RN_OUT;       // 5522
static_assert(RN_NPARAM == CINTX_RYSNET_NPARAM, "parameter count differs from the header");

constexpr int TRAIN_BS = 128;  // samples (threads) per training block
constexpr int RP = RN_H + 1;   // padded row of the per-sample activation tables
constexpr int DYP = RN_OUT + 1;

__host__ __device__ inline void rysnet_features(int n, double x, float* f) {
  f[0] = (float)(n - 5) * 0.25f;
  const double lx = log(x > 1e-7 ? x : 1e-7);
  f[1] = (float)((lx + 5.75) / 10.35);  // x in [1e-7, 100] -> [-1, 1]
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_double(uint64_t& s) { return (splitmix64(s) >> 11) * 0x1.0p-53; }

// Training samples: n uniform in [n_lo, n_hi]; x log-uniform in [1e-7, 50] with probability 0.7,
// else uniform in [50, 3000]; points at or beyond the table range (where the closed form is used
// and no network is needed) are redrawn log-uniformly below it.  Targets from the table path.
__global__ void rysnet_sample_kernel(const __grid_constant__ RysTable rys, uint64_t seed, long long count, int n_lo,
                                     int n_hi, float* __restrict__ feat, float* __restrict__ tgt,
                                     int* __restrict__ nr, double* __restrict__ xs) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    uint64_t s = seed ^ ((uint64_t)i * 0xD1B54A32D192ED03ull);
    const int n = n_lo + (int)(splitmix64(s) % (uint64_t)(n_hi - n_lo + 1));
    const double r1 = unit_double(s), r2 = unit_double(s);
    double x = r1 < 0.7 ? exp(log(1e-7) + r2 * (log(50.0) - log(1e-7))) : 50.0 + r2 * (3000.0 - 50.0);
    const double xm = (double)rys.xmax[n];
    if (!(x < xm)) x = exp(log(1e-7) + unit_double(s) * (log(xm) - log(1e-7)));
    rysnet_features(n, x, feat + 2 * i);
    for (int k = 0; k < RN_OUT; ++k) tgt[RN_OUT * i + k] = 0.0f;
    for (int r = 0; r < n; ++r) {
      const double u = rys_fn(rys, n, r, x), w = rys_fn(rys, n, n + r, x);
      tgt[RN_OUT * i + r] = (float)(log(u) - log1p(-u));
      tgt[RN_OUT * i + RN_HALF + r] = (float)log(w);
    }
    nr[i] = n;
    if (xs) xs[i] = x;
  }
}

__device__ __forceinline__ float sigmoidf_(float a) { return 1.0f / (1.0f + expf(-a)); }

// One forward + backward pass over `count` samples starting at `first`: loss
// L = (1/B) sum_s (1/(2 n_s)) sum_{valid k} (y_sk - t_sk)^2 with B = `batch`; gradients are
// added to grad (one block of 128 samples reduces its own contribution first) and the loss to
// *loss.
__global__ void __launch_bounds__(TRAIN_BS) rysnet_train_kernel(const float* __restrict__ P, const float* __restrict__ feat,
                                                                const float* __restrict__ tgt, const int* __restrict__ nr,
                                                                long long first, long long count, float inv_batch,
                                                                float* __restrict__ grad, double* __restrict__ loss) {
  extern __shared__ __align__(16) float sm[];
  float* sP = sm;                                // RN_NPARAM
  float* sH1 = sP + ((RN_NPARAM + 3) & ~3);      // [128][RP] silu(a1)
  float* sD1 = sH1 + TRAIN_BS * RP;              // silu'(a1), then dL/da1
  float* sH2 = sD1 + TRAIN_BS * RP;              // silu(a2)
  float* sD2 = sH2 + TRAIN_BS * RP;              // silu'(a2), then dL/da2
  float* sDY = sD2 + TRAIN_BS * RP;              // [128][DYP] dL/dy
  float* sF = sDY + TRAIN_BS * DYP;              // [128][2]
  __shared__ double sLoss[TRAIN_BS / 32];
  const int t = threadIdx.x;
  for (int i = t; i < RN_NPARAM; i += TRAIN_BS) sP[i] = P[i];
  const long long idx = first + blockIdx.x * (long long)TRAIN_BS + t;
  const bool valid = blockIdx.x * (long long)TRAIN_BS + t < count;
  float f0 = 0.0f, f1 = 0.0f;
  int n = 1;
  if (valid) {
    f0 = feat[2 * idx];
    f1 = feat[2 * idx + 1];
    n = nr[idx];
  }
  sF[2 * t] = f0;
  sF[2 * t + 1] = f1;
  __syncthreads();
  float* h1 = sH1 + t * RP;
  float* d1 = sD1 + t * RP;
  float* h2 = sH2 + t * RP;
  float* d2 = sD2 + t * RP;
  float* dy = sDY + t * DYP;
  for (int j = 0; j < RN_H; ++j) {
    const float a = sP[RN_W1 + 2 * j] * f0 + sP[RN_W1 + 2 * j + 1] * f1 + sP[RN_B1 + j];
    const float sg = sigmoidf_(a);
    h1[j] = a * sg;
    d1[j] = sg * (1.0f + a * (1.0f - sg));
  }
  for (int i = 0; i < RN_H; ++i) {
    float a = sP[RN_B2 + i];
    for (int j = 0; j < RN_H; ++j) a = fmaf(sP[RN_W2 + RN_H * i + j], h1[j], a);
    const float sg = sigmoidf_(a);
    h2[i] = a * sg;
    d2[i] = sg * (1.0f + a * (1.0f - sg));
  }
  double ls = 0.0;
  for (int k = 0; k < RN_OUT; ++k) {
    float y = sP[RN_B3 + k];
    for (int j = 0; j < RN_H; ++j) y = fmaf(sP[RN_W3 + RN_H * k + j], h2[j], y);
    const bool used = valid && (k % RN_HALF) < n;
    const float d = used ? y - tgt[RN_OUT * idx + k] : 0.0f;
    ls += (double)d * d;
    dy[k] = d * inv_batch / (float)n;  // d/dy of d^2 / (2 n) / B
  }
  ls = valid ? ls / (2.0 * n) * inv_batch : 0.0;
  for (int o = 16; o > 0; o >>= 1) ls += __shfl_down_sync(0xffffffffu, ls, o);
  if ((t & 31) == 0) sLoss[t >> 5] = ls;
  __syncthreads();
  if (t == 0) {
    double b = 0.0;
    for (int w = 0; w < TRAIN_BS / 32; ++w) b += sLoss[w];
    atomicAdd(loss, b);
  }
  // W3, b3: sum over the block's samples of dy (x) h2
  for (int w = t; w < RN_OUT * RN_H + RN_OUT; w += TRAIN_BS) {
    float g = 0.0f;
    if (w < RN_OUT * RN_H) {
      const int k = w / RN_H, j = w % RN_H;
      for (int s = 0; s < TRAIN_BS; ++s) g = fmaf(sDY[s * DYP + k], sH2[s * RP + j], g);
    } else {
      const int k = w - RN_OUT * RN_H;
      for (int s = 0; s < TRAIN_BS; ++s) g += sDY[s * DYP + k];
    }
    atomicAdd(grad + RN_W3 + w, g);
  }
  // dL/da2 (own row)
  for (int j = 0; j < RN_H; ++j) {
    float g = 0.0f;
    for (int k = 0; k < RN_OUT; ++k) g = fmaf(sP[RN_W3 + RN_H * k + j], dy[k], g);
    d2[j] *= g;
  }
  __syncthreads();
  for (int w = t; w < RN_H * RN_H + RN_H; w += TRAIN_BS) {
    float g = 0.0f;
    if (w < RN_H * RN_H) {
      const int i = w / RN_H, j = w % RN_H;
      for (int s = 0; s < TRAIN_BS; ++s) g = fmaf(sD2[s * RP + i], sH1[s * RP + j], g);
    } else {
      const int i = w - RN_H * RN_H;
      for (int s = 0; s < TRAIN_BS; ++s) g += sD2[s * RP + i];
    }
    atomicAdd(grad + RN_W2 + w, g);
  }
  // dL/da1 (own row)
  for (int j = 0; j < RN_H; ++j) {
    float g = 0.0f;
    for (int i = 0; i < RN_H; ++i) g = fmaf(sP[RN_W2 + RN_H * i + j], d2[i], g);
    d1[j] *= g;
  }
  __syncthreads();
  for (int w = t; w < RN_H * RN_IN + RN_H; w += TRAIN_BS) {
    float g = 0.0f;
    if (w < RN_H * RN_IN) {
      const int j = w / RN_IN, c = w % RN_IN;
      for (int s = 0; s < TRAIN_BS; ++s) g = fmaf(sD1[s * RP + j], sF[2 * s + c], g);
    } else {
      const int j = w - RN_H * RN_IN;
      for (int s = 0; s < TRAIN_BS; ++s) g += sD1[s * RP + j];
    }
    atomicAdd(grad + RN_W1 + w, g);
  }
}

constexpr size_t kTrainSmemBytes =
    sizeof(float) * (((RN_NPARAM + 3) & ~3) + 4 * TRAIN_BS * RP + TRAIN_BS * DYP + 2 * TRAIN_BS);

// Adam step (bias-corrected) on every parameter; clears the gradient.
__global__ void rysnet_adam_kernel(float* __restrict__ P, float* __restrict__ G, float* __restrict__ m,
                                   float* __restrict__ v, int np, float lr, float b1, float b2, float eps,
                                   float bc1, float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const float g = G[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    G[i] = 0.0f;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int EVAL_WARPS = 4;

// One warp per point: network guess (mode 0) or the x = 0 roots (mode 1, the method without the
// network), FP64 refinement, checks, fallback to the table path; mode 2 returns the network's
// guess unrefined.  out[p*2n + f]: t^2 (f < n) then weights; status 0 refined, 1 fallback,
// 2 closed-form large-x limit, 3 unrefined guess; iters = Newton steps of the slowest root.
__global__ void __launch_bounds__(32 * EVAL_WARPS) rys_learned_kernel(const float* __restrict__ P,
                                                                      const __grid_constant__ RysTable rys, int n,
                                                                      const double* __restrict__ xs, long long count,
                                                                      int mode, double* __restrict__ out,
                                                                      int* __restrict__ status, int* __restrict__ iters) {
  __shared__ float sP[RN_NPARAM];
  __shared__ float sAct[EVAL_WARPS][2 * RN_H + RN_OUT];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (mode != 1)
    for (int i = threadIdx.x; i < RN_NPARAM; i += blockDim.x) sP[i] = P[i];
  __syncthreads();
  float* h1 = sAct[wid];
  float* h2 = h1 + RN_H;
  float* y = h2 + RN_H;
  const int xm = rys.xmax[n];
  for (long long p = blockIdx.x * (long long)EVAL_WARPS + wid; p < count; p += (long long)gridDim.x * EVAL_WARPS) {
    const double x = xs[p];
    double* o = out + p * 2 * n;
    if (!(x < (double)xm)) {
      for (int f = lane; f < 2 * n; f += 32) o[f] = rys_fn(rys, n, f, x);
      if (lane == 0) {
        status[p] = 2;
        iters[p] = 0;
      }
      continue;
    }
    // initial guess for root `lane`
    double u = 0.5, wg = 0.0;
    if (mode != 1) {
      float f[2];
      rysnet_features(n, x, f);
      for (int j = lane; j < RN_H; j += 32) {
        const float a = sP[RN_W1 + 2 * j] * f[0] + sP[RN_W1 + 2 * j + 1] * f[1] + sP[RN_B1 + j];
        h1[j] = a * sigmoidf_(a);
      }
      __syncwarp();
      for (int i = lane; i < RN_H; i += 32) {
        float a = sP[RN_B2 + i];
        for (int j = 0; j < RN_H; ++j) a = fmaf(sP[RN_W2 + RN_H * i + j], h1[j], a);
        h2[i] = a * sigmoidf_(a);
      }
      __syncwarp();
      if (lane < RN_OUT) {
        float a = sP[RN_B3 + lane];
        for (int j = 0; j < RN_H; ++j) a = fmaf(sP[RN_W3 + RN_H * lane + j], h2[j], a);
        y[lane] = a;
      }
      __syncwarp();
      if (lane < n) {
        u = 1.0 / (1.0 + exp(-(double)y[lane]));
        wg = exp((double)y[RN_HALF + lane]);
      }
      __syncwarp();
      if (mode == 2) {  // the network's guess itself, for judging it against the table path
        if (lane < n) {
          o[lane] = u;
          o[n + lane] = wg;
        }
        if (lane == 0) {
          status[p] = 3;
          iters[p] = 0;
        }
        continue;
      }
    } else if (lane < n) {
      u = rys_fn(rys, n, lane, 0.0);
    }
    // recurrence coefficients of the discretised measure (Stieltjes), lanes own nodes lane, lane+32
    const double ua = kRysGlU[lane], ub = kRysGlU[lane + 32];
    const double wa = kRysGlW[lane] * exp(-x * ua), wb = kRysGlW[lane + 32] * exp(-x * ub);
    double al[CINTX_NRMAX], be[CINTX_NRMAX];
    double p0a = 0.0, p1a = 1.0, p0b = 0.0, p1b = 1.0;
    double nrm = warp_sum(wa + wb);
    be[0] = nrm;
    for (int k = 0; k < n; ++k) {
      al[k] = warp_sum(wa * ua * p1a * p1a + wb * ub * p1b * p1b) / nrm;
      if (k + 1 == n) break;
      const double bk = k ? be[k] : 0.0;
      const double p2a = (ua - al[k]) * p1a - bk * p0a, p2b = (ub - al[k]) * p1b - bk * p0b;
      const double n2 = warp_sum(wa * p2a * p2a + wb * p2b * p2b);
      be[k + 1] = n2 / nrm;
      p0a = p1a; p1a = p2a; p0b = p1b; p1b = p2b;
      nrm = n2;
    }
    // Newton steps with the Aberth correction on p_n, all roots at once (lane i < n holds root i):
    // u_i -= d_i / (1 - d_i sum_{j != i} 1/(u_i - u_j)), d_i = p_n(u_i) / p_n'(u_i); the
    // repulsion keeps two starts from converging onto the same root
    bool conv = lane >= n;
    int it = 0;
    for (it = 1; it <= 8; ++it) {
      double q0 = 0.0, q1 = 1.0, d0 = 0.0, d1 = 0.0;
      for (int k = 0; k < n; ++k) {
        const double bk = k ? be[k] : 0.0;
        const double q2 = (u - al[k]) * q1 - bk * q0;
        const double d2 = q1 + (u - al[k]) * d1 - bk * d0;
        q0 = q1; q1 = q2; d0 = d1; d1 = d2;
      }
      double rep = 0.0;
      for (int j = 0; j < n; ++j) {
        const double uj = __shfl_sync(0xffffffffu, u, j);
        if (j != lane) rep += 1.0 / (u - uj);
      }
      if (lane < n) {
        const double dl = q1 / d1;
        const double du = dl / (1.0 - dl * rep);
        u -= du;
        conv = fabs(du) <= 1e-14 * fabs(u);
      }
      if (__all_sync(0xffffffffu, conv)) break;
    }
    if (it > 8) it = 8;
    // place root i at its rank among the n roots; distinct roots of p_n in (0, 1) are its zeros
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double uj = __shfl_sync(0xffffffffu, u, j);
      if (j != lane && (uj < u || (uj == u && j < lane))) ++rank;
    }
    double us = u;
    for (int j = 0; j < n; ++j) {
      const double uj = __shfl_sync(0xffffffffu, u, j);
      const int rj = __shfl_sync(0xffffffffu, rank, j);
      if (rj == lane) us = uj;
    }
    bool ok = lane >= n || (conv && us > 0.0 && us < 1.0 && isfinite(us));
    const double unext = __shfl_down_sync(0xffffffffu, us, 1);
    if (lane + 1 < n) ok = ok && unext > us * (1.0 + 1e-12);
    // Christoffel weight of the sorted root
    double wr = 0.0;
    if (lane < n) {
      double sacc = 1.0 / be[0], q0 = 0.0, q1 = 1.0, nn = be[0];
      for (int k = 0; k + 1 < n; ++k) {
        const double bk = k ? be[k] : 0.0;
        const double q2 = (us - al[k]) * q1 - bk * q0;
        nn *= be[k + 1];
        sacc += q2 * q2 / nn;
        q0 = q1; q1 = q2;
      }
      wr = 1.0 / sacc;
      ok = ok && wr > 0.0 && isfinite(wr);
    }
    const int itmax = it;
    if (__all_sync(0xffffffffu, ok)) {
      if (lane < n) {
        o[lane] = us;
        o[n + lane] = wr;
      }
      if (lane == 0) status[p] = 0;
    } else {
      for (int f = lane; f < 2 * n; f += 32) o[f] = rys_fn(rys, n, f, x);
      if (lane == 0) status[p] = 1;
    }
    if (lane == 0) iters[p] = itmax;
  }
}

cudaError_t rys_learned_eval(const float* d_params, const RysTable& rys, int n, const double* d_x, long long count,
                             double* d_out, int* d_status, int* d_iters, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((count + EVAL_WARPS - 1) / EVAL_WARPS, 148LL * 16);
  rys_learned_kernel<<<(unsigned)blocks, 32 * EVAL_WARPS, 0, stream>>>(d_params, rys, n, d_x, count, 0, d_out,
                                                                       d_status, d_iters);
  return cudaGetLastError();
}

}  // namespace cintx

using namespace cintx;

namespace {

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* get() {
    return static_cast<T*>(p);
  }
};

int cuda_fail(const char* what, cudaError_t e) {
  set_error(CINTX_STATUS_EXECUTION_FAILED, std::string(what) + ": " + cudaGetErrorString(e));
  return CINTX_STATUS_EXECUTION_FAILED;
}

int alloc(DevBuf& b, size_t bytes) {
  if (cudaMalloc(&b.p, bytes ? bytes : 1) != cudaSuccess) {
    b.p = nullptr;
    set_error(CINTX_STATUS_ALLOCATION_FAILED, "device allocation failed");
    return CINTX_STATUS_ALLOCATION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

int launch_train_pass(const float* dP, const float* feat, const float* tgt, const int* nr, long long first,
                      long long count, float* grad, double* loss, cudaStream_t st) {
  static bool attr[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr[dev]) {
    cudaError_t e = cudaFuncSetAttribute(rysnet_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTrainSmemBytes);
    if (e != cudaSuccess) return cuda_fail("rysnet training kernel attribute", e);
    if (dev < 64) attr[dev] = true;
  }
  const unsigned blocks = (unsigned)((count + TRAIN_BS - 1) / TRAIN_BS);
  rysnet_train_kernel<<<blocks, TRAIN_BS, kTrainSmemBytes, st>>>(dP, feat, tgt, nr, first, count,
                                                                 1.0f / (float)count, grad, loss);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CINTX_STATUS_SUCCESS : cuda_fail("rysnet training kernel", e);
}

}  // namespace

extern "C" {

int cintx_rysnet_samples(int64_t count, int n_lo, int n_hi, uint64_t seed, float* feat, float* tgt, int* nroots,
                         double* x) {
  clear_error();
  if (count < 0 || n_lo < 1 || n_hi > CINTX_NRMAX || n_lo > n_hi || !feat || !tgt || !nroots) {
    set_error(CINTX_STATUS_INVALID_INPUT, "cintx_rysnet_samples: bad arguments");
    return CINTX_STATUS_INVALID_INPUT;
  }
  DeviceState* ds;
  int rc;
  if ((rc = device_state(&ds))) return rc;
  DevBuf f, t, r, xb;
  if ((rc = alloc(f, sizeof(float) * 2 * count)) || (rc = alloc(t, sizeof(float) * RN_OUT * count)) ||
      (rc = alloc(r, sizeof(int) * count)) || (rc = alloc(xb, sizeof(double) * count)))
    return rc;
  if (count) {
    rysnet_sample_kernel<<<(unsigned)std::min<int64_t>((count + 255) / 256, 4096), 256>>>(
        ds->rys, seed, count, n_lo, n_hi, f.get<float>(), t.get<float>(), r.get<int>(), xb.get<double>());
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail("rysnet sample generation", e);
  }
  cudaMemcpy(feat, f.p, sizeof(float) * 2 * count, cudaMemcpyDeviceToHost);
  cudaMemcpy(tgt, t.p, sizeof(float) * RN_OUT * count, cudaMemcpyDeviceToHost);
  cudaMemcpy(nroots, r.p, sizeof(int) * count, cudaMemcpyDeviceToHost);
  if (x) cudaMemcpy(x, xb.p, sizeof(double) * count, cudaMemcpyDeviceToHost);
  return CINTX_STATUS_SUCCESS;
}

int cintx_rysnet_loss_grad(const float* params, const float* feat, const float* tgt, const int* nroots, int64_t count,
                           float* grad, double* loss) {
  clear_error();
  if (!params || !feat || !tgt || !nroots || !grad || !loss || count <= 0) {
    set_error(CINTX_STATUS_INVALID_INPUT, "cintx_rysnet_loss_grad: bad arguments");
    return CINTX_STATUS_INVALID_INPUT;
  }
  for (int64_t i = 0; i < count; ++i)
    if (nroots[i] < 1 || nroots[i] > RN_HALF) {
      set_error(CINTX_STATUS_INVALID_INPUT, "cintx_rysnet_loss_grad: nroots outside 1..9");
      return CINTX_STATUS_INVALID_INPUT;
    }
  DevBuf P, F, T, R, G, L;
  int rc;
  if ((rc = alloc(P, sizeof(float) * RN_NPARAM)) || (rc = alloc(F, sizeof(float) * 2 * count)) ||
      (rc = alloc(T, sizeof(float) * RN_OUT * count)) || (rc = alloc(R, sizeof(int) * count)) ||
      (rc = alloc(G, sizeof(float) * RN_NPARAM)) || (rc = alloc(L, sizeof(double))))
    return rc;
  cudaMemcpy(P.p, params, sizeof(float) * RN_NPARAM, cudaMemcpyHostToDevice);
  cudaMemcpy(F.p, feat, sizeof(float) * 2 * count, cudaMemcpyHostToDevice);
  cudaMemcpy(T.p, tgt, sizeof(float) * RN_OUT * count, cudaMemcpyHostToDevice);
  cudaMemcpy(R.p, nroots, sizeof(int) * count, cudaMemcpyHostToDevice);
  cudaMemset(G.p, 0, sizeof(float) * RN_NPARAM);
  cudaMemset(L.p, 0, sizeof(double));
  if ((rc = launch_train_pass(P.get<float>(), F.get<float>(), T.get<float>(), R.get<int>(), 0, count, G.get<float>(),
                              L.get<double>(), 0)))
    return rc;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail("rysnet forward/backward", e);
  cudaMemcpy(grad, G.p, sizeof(float) * RN_NPARAM, cudaMemcpyDeviceToHost);
  cudaMemcpy(loss, L.p, sizeof(double), cudaMemcpyDeviceToHost);
  return CINTX_STATUS_SUCCESS;
}

int cintx_rysnet_train(float* params, int64_t nsamples, int n_lo, int n_hi, int epochs, int batch, float lr,
                       uint64_t seed, double* loss_per_epoch) {
  clear_error();
  if (!params || nsamples < batch || batch < TRAIN_BS || epochs < 1 || n_lo < 1 || n_hi > RN_HALF || n_lo > n_hi ||
      !(lr > 0.0f)) {
    set_error(CINTX_STATUS_INVALID_INPUT, "cintx_rysnet_train: bad arguments");
    return CINTX_STATUS_INVALID_INPUT;
  }
  DeviceState* ds;
  int rc;
  if ((rc = device_state(&ds))) return rc;
  DevBuf F, T, R, P, G, M, V, L;
  if ((rc = alloc(F, sizeof(float) * 2 * nsamples)) || (rc = alloc(T, sizeof(float) * RN_OUT * nsamples)) ||
      (rc = alloc(R, sizeof(int) * nsamples)) || (rc = alloc(P, sizeof(float) * RN_NPARAM)) ||
      (rc = alloc(G, sizeof(float) * RN_NPARAM)) || (rc = alloc(M, sizeof(float) * RN_NPARAM)) ||
      (rc = alloc(V, sizeof(float) * RN_NPARAM)) || (rc = alloc(L, sizeof(double) * epochs)))
    return rc;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
    return cuda_fail("cudaStreamCreate", cudaErrorUnknown);
  rysnet_sample_kernel<<<(unsigned)std::min<int64_t>((nsamples + 255) / 256, 8192), 256, 0, st>>>(
      ds->rys, seed, nsamples, n_lo, n_hi, F.get<float>(), T.get<float>(), R.get<int>(), nullptr);
  cudaMemcpyAsync(P.p, params, sizeof(float) * RN_NPARAM, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(G.p, 0, sizeof(float) * RN_NPARAM, st);
  cudaMemsetAsync(M.p, 0, sizeof(float) * RN_NPARAM, st);
  cudaMemsetAsync(V.p, 0, sizeof(float) * RN_NPARAM, st);
  cudaMemsetAsync(L.p, 0, sizeof(double) * epochs, st);
  const int64_t steps_per_epoch = nsamples / batch;
  const int64_t total = steps_per_epoch * epochs;
  const float b1 = 0.9f, b2 = 0.999f;
  float bc1 = 1.0f, bc2 = 1.0f;
  int64_t step = 0;
  for (int ep = 0; ep < epochs && !rc; ++ep) {
    for (int64_t s = 0; s < steps_per_epoch && !rc; ++s, ++step) {
      // cosine decay to 1% of lr over the run
      const float frac = (float)step / (float)std::max<int64_t>(total - 1, 1);
      const float lr_t = lr * (0.01f + 0.99f * 0.5f * (1.0f + cosf(3.14159265f * frac)));
      rc = launch_train_pass(P.get<float>(), F.get<float>(), T.get<float>(), R.get<int>(), s * batch, batch,
                             G.get<float>(), L.get<double>() + ep, st);
      if (rc) break;
      bc1 *= b1;
      bc2 *= b2;
      rysnet_adam_kernel<<<(RN_NPARAM + 255) / 256, 256, 0, st>>>(P.get<float>(), G.get<float>(), M.get<float>(),
                                                                 V.get<float>(), RN_NPARAM, lr_t, b1, b2, 1e-8f,
                                                                 1.0f - bc1, 1.0f - bc2);
    }
  }
  cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail("rysnet training", e);
  cudaMemcpy(params, P.p, sizeof(float) * RN_NPARAM, cudaMemcpyDeviceToHost);
  if (loss_per_epoch) {
    std::vector<double> l(epochs);
    cudaMemcpy(l.data(), L.p, sizeof(double) * epochs, cudaMemcpyDeviceToHost);
    for (int ep = 0; ep < epochs; ++ep) loss_per_epoch[ep] = l[ep] / (double)steps_per_epoch;
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_rys_learned_batch(const float* params, int nroots, const double* x, int64_t count, int mode, double* t2w,
                            int* status, int* iters) {
  clear_error();
  if (nroots < 1 || nroots > RN_HALF || count < 0 || !x || !t2w || !status || !iters || (mode != 1 && !params) ||
      mode < 0 || mode > 2) {
    set_error(CINTX_STATUS_INVALID_INPUT, "cintx_rys_learned_batch: bad arguments");
    return CINTX_STATUS_INVALID_INPUT;
  }
  DeviceState* ds;
  int rc;
  if ((rc = device_state(&ds))) return rc;
  DevBuf P, X, O, S, I;
  if ((rc = alloc(P, sizeof(float) * RN_NPARAM)) || (rc = alloc(X, sizeof(double) * count)) ||
      (rc = alloc(O, sizeof(double) * 2 * nroots * count)) || (rc = alloc(S, sizeof(int) * count)) ||
      (rc = alloc(I, sizeof(int) * count)))
    return rc;
  if (mode != 1) cudaMemcpy(P.p, params, sizeof(float) * RN_NPARAM, cudaMemcpyHostToDevice);
  cudaMemcpy(X.p, x, sizeof(double) * count, cudaMemcpyHostToDevice);
  if (count) {
    const long long blocks = std::min<long long>((count + EVAL_WARPS - 1) / EVAL_WARPS, 148LL * 16);
    rys_learned_kernel<<<(unsigned)blocks, 32 * EVAL_WARPS>>>(P.get<float>(), ds->rys, nroots, X.get<double>(), count,
                                                              mode, O.get<double>(), S.get<int>(), I.get<int>());
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail("learned root evaluation", e);
  }
  cudaMemcpy(t2w, O.p, sizeof(double) * 2 * nroots * count, cudaMemcpyDeviceToHost);
  cudaMemcpy(status, S.p, sizeof(int) * count, cudaMemcpyDeviceToHost);
  cudaMemcpy(iters, I.p, sizeof(int) * count, cudaMemcpyDeviceToHost);
  return CINTX_STATUS_SUCCESS;
}

}  // extern "C"
