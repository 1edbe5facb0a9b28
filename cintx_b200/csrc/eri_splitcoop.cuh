// Cooperative launch shapes with split horizontal transfers (launch-shape variants 10 and 11).
//
// The default cooperative shape of eri4c_kernel (a group of S lanes per quartet) evaluates each
// primitive quartet in three barrier-separated phases: roots on 2*NR lanes, the 3*NR (axis, root)
// recurrences on at most 3*NR lanes (each lane builds a 2D table in shared memory and runs the
// horizontal transfers of its (axis, root) from it), and the cartesian products on all S lanes.
// For the f-shell classes the middle phase is a long serial chain on one warp while the others
// wait at the barrier.  These shapes split it in two:
//   V: 3*NR lanes build the 2D tables G(n, m) of the (axis, root) pairs in registers, one column
//      m at a time (three columns live), and store them to shared memory;
//   H: 3*NR*(LJ+1)*(LL+1) tasks, one per (axis, root, j, l), spread over all S lanes; each writes
//      the (LI+1)*(LK+1) transferred values I(i, j, k, l) of its (j, l).
// The roots, the products into register accumulators, the cartesian-to-spherical stages and the
// strided store are the default cooperative shape's.  Both keep the 128-register cap of the
// default shape (255-register cooperative shapes measured 1.5-2x slower: these classes need
// resident warps); variant 10 keeps 12 accumulators per lane and 11 keeps 24.  They exist for
// spherical FP64 classes up to f shells with 64 or more lanes whose transform buffers are on chip
// (on narrower groups the middle phase is short and the sliced shapes measured faster).
//
// Included by eri_launch.cuh after LaunchArgs, class_valid and device_sm_count.
#pragma once
#include "eri_kernel.cuh"

namespace cintx {

__host__ __device__ constexpr bool variant_splitcoop(int v) { return v == 10 || v == 11; }
__host__ __device__ constexpr int splitcoop_acc(int v) { return v == 11 ? 24 : 12; }
constexpr int kSplitCoopRegs = 128;

// Every size of a split-transfer cooperative shape, from the class and the shape's accumulator
// budget; `ok` says whether the shape is compiled for the class.  The kernel static_asserts that
// these agree with EriShape's.
struct SplitCoopDims {
  int S, NR, GSZ, NIJ, NKL, BLOCK, Q, MINB;
  int loop_doubles;   // roots, I arrays and 2D tables of one group
  int xform_doubles;  // the two transform buffers of one group (alias the loop region)
  int B_GROUP, SMEM_BYTES;
  int ntask_h;        // (axis, root, j, l) transfer tasks
  bool ok;
};

__host__ __device__ constexpr SplitCoopDims splitcoop_dims(int li, int lj, int lk, int ll, int acc) {
  SplitCoopDims d{};
  d.S = pick_threads(li, lj, lk, ll, acc);
  d.NR = (li + lj + lk + ll) / 2 + 1;
  d.GSZ = (li + 1) * (lj + 1) * (lk + 1) * (ll + 1);
  d.NIJ = li + lj + 1;
  d.NKL = lk + ll + 1;
  d.BLOCK = d.S >= 128 ? d.S : 128;
  d.Q = d.BLOCK / d.S;
  d.MINB = 65536 / (d.BLOCK * kSplitCoopRegs) > 0 ? 65536 / (d.BLOCK * kSplitCoopRegs) : 1;
  const int ntup = ncart(lj) * ncart(lk) * ncart(ll);
  const int mi = li >= 2 ? 2 * li + 1 : ncart(li);
  const int mj = lj >= 2 ? 2 * lj + 1 : ncart(lj);
  const int bufa = mi * ntup, bufb = mi * mj * ncart(lk) * ncart(ll);
  const bool global_buf = d.S > 1 && (bufa + bufb) * 8 * (d.S >= 128 ? 1 : 128 / d.S) > 200 * 1024;
  d.loop_doubles = 2 * d.NR + 3 * d.NR * d.GSZ + 3 * d.NR * d.NIJ * d.NKL;
  d.xform_doubles = bufa + bufb;
  d.B_GROUP = ((d.loop_doubles > d.xform_doubles ? d.loop_doubles : d.xform_doubles) * 8 + 15) & ~15;
  d.SMEM_BYTES = d.Q * d.B_GROUP;
  d.ntask_h = 3 * d.NR * (lj + 1) * (ll + 1);
  d.ok = class_valid(li, lj, lk, ll) && li <= 3 && d.S >= 64 && !global_buf && d.SMEM_BYTES <= 200 * 1024;
  return d;
}

// Index bounds of a compiled split-transfer shape (0: all hold; else the failing condition):
// 1 the lanes form whole groups inside the block and own every (j,k,l) tuple, 2 the named-barrier
// ids and counts are valid, 3 the loop region (roots | I arrays | 2D tables) holds every task's
// output and 4 the transform buffers and every transform stage lie inside the group region, 5 the
// block's shared memory is the sum of its group regions.
template <int LI, int LJ, int LK, int LL, int ACC>
__host__ __device__ constexpr int splitcoop_violation() {
  using SH = EriShape<LI, LJ, LK, LL, true, double, ACC, kSplitCoopRegs>;
  constexpr SplitCoopDims d = splitcoop_dims(LI, LJ, LK, LL, ACC);
  if (d.S != SH::S || d.NR != SH::NR || d.GSZ != SH::GSZ || d.BLOCK != SH::BLOCK || d.Q != SH::Q) return 1;
  if (d.S < 1 || d.S > 256 || (d.S & (d.S - 1)) != 0 || d.BLOCK % d.S != 0 || d.BLOCK > 1024) return 1;
  if (SH::TPT * d.S < SH::NTUP) return 1;
  if (d.S > 32 && (d.Q > 15 || d.S % 32 != 0)) return 2;
  if (d.S <= 32 && 32 % d.S != 0) return 2;
  if ((SH::SM_ROOTS + SH::SM_G + 3 * SH::NR * SH::NIJ * SH::NKL) * 8 > d.B_GROUP) return 3;
  if (d.ntask_h != 3 * SH::NR * SH::NJ * SH::NL) return 3;
  if (d.xform_doubles != SH::SM_BUFA + SH::SM_BUFB || d.xform_doubles * 8 > d.B_GROUP || SH::GLOBAL_BUF) return 4;
  if (SH::MI * SH::NTUP > SH::SM_BUFA || SH::MI * SH::MJ * SH::NFK * SH::NFL > SH::SM_BUFB) return 4;
  if (SH::MI * SH::MJ * SH::MK * SH::NFL > (SH::MJ != SH::NFJ ? SH::SM_BUFA : SH::SM_BUFB)) return 4;
  if (d.B_GROUP % 16 != 0 || d.SMEM_BYTES != d.Q * d.B_GROUP || d.SMEM_BYTES > 227 * 1024) return 5;
  return 0;
}

// Horizontal transfers of one (axis, root) for one (j, l):
//   I(i, j, k, l) = sum_a sum_b C(j,a) C(l,b) ab^(j-a) cd^(l-b) G(i+a, k+b)
// for all i <= LI, k <= LK, from the table gt[n * NKL + m] (closed binomial form of g2e.c:428-694),
// written to dst[i + NI*(j + NJ*(k + NK*l))].  j and l are runtime values: the coefficients of
// a > j (b > l) are zero, so the unrolled sums run to LJ (LL).
template <int LI, int LJ, int LK, int LL>
__device__ __forceinline__ void hrr_jl(double* __restrict__ dst, const double* __restrict__ gt, int j, int l,
                                       double ab, double cd) {
  constexpr int NKL = LK + LL + 1;
  constexpr int NI = LI + 1, NJ = LJ + 1, NK = LK + 1;
  // ca[a] = C(j, a) ab^(j - a) for a <= j, else 0: row j of the Pascal table (runtime j: selects)
  double ej[LJ + 1][LJ + 1], el[LL + 1][LL + 1], ca[LJ + 1], cb[LL + 1];
  pascal_powers<LJ, double>(ej, ab);
  pascal_powers<LL, double>(el, cd);
#pragma unroll
  for (int a = 0; a <= LJ; ++a) {
    double v = 0.0;
#pragma unroll
    for (int jj = a; jj <= LJ; ++jj) v = jj == j ? ej[jj][a] : v;
    ca[a] = v;
  }
#pragma unroll
  for (int b = 0; b <= LL; ++b) {
    double v = 0.0;
#pragma unroll
    for (int l2 = b; l2 <= LL; ++l2) v = l2 == l ? el[l2][b] : v;
    cb[b] = v;
  }
#pragma unroll
  for (int i = 0; i <= LI; ++i) {
    double T[NKL];
#pragma unroll
    for (int m = 0; m < NKL; ++m) {
      double v = 0.0;
#pragma unroll
      for (int a = 0; a <= LJ; ++a) v = fma(ca[a], gt[(i + a) * NKL + m], v);
      T[m] = v;
    }
#pragma unroll
    for (int k = 0; k <= LK; ++k) {
      double v = 0.0;
#pragma unroll
      for (int b = 0; b <= LL; ++b) v = fma(cb[b], T[k + b], v);
      dst[i + NI * (j + NJ * (k + NK * l))] = v;
    }
  }
}

template <int LI, int LJ, int LK, int LL, int ACC>
__global__ void __launch_bounds__(splitcoop_dims(LI, LJ, LK, LL, ACC).BLOCK, splitcoop_dims(LI, LJ, LK, LL, ACC).MINB)
    eri_splitcoop_kernel(const QuartetRec* __restrict__ recs, int nrec, const ShellPair* __restrict__ pairs,
                         const PrimPair* __restrict__ prims, double* __restrict__ out, OutStrides st,
                         double expcutoff, const __grid_constant__ RysTable rys, double prim_eps,
                         const double* __restrict__ rootbuf, const long long* __restrict__ rootbase) {
  using SH = EriShape<LI, LJ, LK, LL, true, double, ACC, kSplitCoopRegs>;
  constexpr SplitCoopDims D = splitcoop_dims(LI, LJ, LK, LL, ACC);
  static_assert(D.ok && splitcoop_violation<LI, LJ, LK, LL, ACC>() == 0,
                "an index of this launch shape can leave its buffer");
  static_assert(D.B_GROUP % 16 == 0 && (SH::NI % 2 != 0 || (SH::GSZ % 2 == 0 && (2 * SH::NR) % 2 == 0)),
                "16-byte loads of the I arrays need 16-byte aligned group regions and tables");
  constexpr int S = SH::S, NR = SH::NR, GSZ = SH::GSZ, NFI = SH::NFI, TPT = SH::TPT;
  constexpr int NIJ = SH::NIJ, NKL = SH::NKL, NJ = SH::NJ, NL = SH::NL;
  extern __shared__ __align__(16) double smem[];
  const int group = (int)threadIdx.x / S;
  const int lane = (int)threadIdx.x % S;
  double* sg = smem + (size_t)group * (D.B_GROUP / 8);
  double* s_roots = sg;              // t2[NR], w[NR]
  double* s_g = sg + 2 * NR;         // I arrays [axis][root][GSZ]
  double* s_t = s_g + 3 * NR * GSZ;  // 2D tables [axis][root][NIJ * NKL]

  LaneTuples<SH> lt;
  decode_tuples<SH, LJ, LK, LL>(lt, lane);

  for (int q = (int)blockIdx.x * SH::Q + group; q < nrec; q += (int)gridDim.x * SH::Q) {
    const QuartetRec rec = recs[q];
    const double* rb = rootbuf ? rootbuf + rootbase[q] : nullptr;
    const ShellPair pij = pairs[rec.pij];
    const ShellPair pkl = pairs[rec.pkl];
    double acc[TPT][NFI];
#pragma unroll
    for (int k = 0; k < TPT; ++k)
#pragma unroll
      for (int f = 0; f < NFI; ++f) acc[k][f] = 0.0;
    for (int b = 0; b < pkl.nprim; ++b) {
      const PrimPair pk = prims[pkl.prim_off + b];
      if (b + 1 < pkl.nprim) prefetch_prim(prims + pkl.prim_off + b + 1);
      const double qcx = pk.px - pkl.ax, qcy = pk.py - pkl.ay, qcz = pk.pz - pkl.az;
      const double qthr = prim_eps / pk.q;  // primitive Schwarz screening, as in eri4c_kernel
      for (int a = 0; a < pij.nprim; ++a) {
        const PrimPair pi = prims[pij.prim_off + a];
        if (a + 1 < pij.nprim) prefetch_prim(prims + pij.prim_off + a + 1);
        if (pi.q < qthr) break;
        if (pi.cce + pk.cce > expcutoff) continue;  // CINT2e_loop eijcutoff (cint2e.c:700-712)
        const double aij = pi.aij, akl = pk.aij;
        const double rs = rsqrt(aij + akl);
        const double inv_aijkl = rs * rs;
        const double inv_a1 = 4.0 * pi.half_inv * pk.half_inv;
        const double pqx = pi.px - pk.px, pqy = pi.py - pk.py, pqz = pi.pz - pk.pz;
        const double x = aij * akl * inv_aijkl * (pqx * pqx + pqy * pqy + pqz * pqz);
        const double fac = pi.kab * pk.kab * rs * inv_a1;
        if (rb) {
          const double* r = rb + (size_t)(b * pij.nprim + a) * (2 * NR);
          for (int f = lane; f < 2 * NR; f += S) s_roots[f] = r[f];
        } else {
          for (int f = lane; f < 2 * NR; f += S) s_roots[f] = rys_fn(rys, NR, f, x);
        }
        group_sync<S>(group);
        // V: the 2D tables
        for (int task = lane; task < 3 * NR; task += S) {
          const int axis = task / NR, r = task % NR;
          const double rt_aa = s_roots[r] * inv_aijkl;
          const double b00 = 0.5 * rt_aa;
          const double b10 = pi.half_inv * (1.0 - rt_aa * akl);
          const double b01 = pk.half_inv * (1.0 - rt_aa * aij);
          const double pa = axis == 0 ? pi.px - pij.ax : (axis == 1 ? pi.py - pij.ay : pi.pz - pij.az);
          const double qc = axis == 0 ? qcx : (axis == 1 ? qcy : qcz);
          const double pq = axis == 0 ? pqx : (axis == 1 ? pqy : pqz);
          const double g00 = axis == 2 ? s_roots[NR + r] * fac : 1.0;
          vrr_columns<NIJ, NKL, double>(s_t + task * (NIJ * NKL), g00, pa - rt_aa * akl * pq,
                                        qc + rt_aa * aij * pq, b10, b01, b00);
        }
        group_sync<S>(group);
        // H: the transfers, one (axis, root, j, l) per task
        for (int u = lane; u < D.ntask_h; u += S) {
          const int task = u / (NJ * NL), jl = u % (NJ * NL);
          const int axis = task / NR;
          const double ab = axis == 0 ? pij.abx : (axis == 1 ? pij.aby : pij.abz);
          const double cd = axis == 0 ? pkl.abx : (axis == 1 ? pkl.aby : pkl.abz);
          hrr_jl<LI, LJ, LK, LL>(s_g + task * GSZ, s_t + task * (NIJ * NKL), jl % NJ, jl / NJ, ab, cd);
        }
        group_sync<S>(group);
#pragma unroll 1
        for (int r = 0; r < NR; ++r) {
          const double* gx = s_g + (0 * NR + r) * GSZ;
          const double* gy = s_g + (1 * NR + r) * GSZ;
          const double* gz = s_g + (2 * NR + r) * GSZ;
#pragma unroll
          for (int k = 0; k < TPT; ++k) {
            double ix[SH::NI], iy[SH::NI], iz[SH::NI];
            load_i_column<SH::NI>(ix, gx + lt.ox[k]);
            load_i_column<SH::NI>(iy, gy + lt.oy[k]);
            load_i_column<SH::NI>(iz, gz + lt.oz[k]);
            static_loop(std::make_integer_sequence<int, NFI>{}, [&](auto c) {  // fi constant: ix, iy, iz stay in registers
              constexpr int fi = decltype(c)::value;
              constexpr int cx = cart_x(LI, fi), cy = cart_y(LI, fi), cz = cart_z(LI, fi);
              acc[k][fi] = fma(ix[cx] * iy[cy], iz[cz], acc[k][fi]);
            });
          }
        }
        group_sync<S>(group);
      }
    }
    // ---- transform to spherical and store (the default cooperative shape's stages) ----
    double* const obase = out + rec.out;
    double* bufA = sg;
    double* bufB = bufA + SH::SM_BUFA;
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      const int t = lane + S * k;
      if (t < SH::NTUP) {
#pragma unroll
        for (int mi = 0; mi < SH::MI; ++mi) {
          double v = 0.0;
#pragma unroll
          for (int fi = 0; fi < NFI; ++fi) {
            const double c = LI >= 2 ? c2s_coef(LI, mi, fi) : (mi == fi ? 1.0 : 0.0);
            if (c != 0.0) v += c * acc[k][fi];
          }
          bufA[mi + SH::MI * t] = v;
        }
      }
    }
    group_sync<S>(group);
    const double* cur = bufA;
    if constexpr (LJ >= 2) {
      constexpr int n = SH::MI * SH::MJ * SH::NFK * SH::NFL;
      for (int o = lane; o < n; o += S) {
        const int mi = o % SH::MI;
        const int mj = (o / SH::MI) % SH::MJ;
        const int rest = o / (SH::MI * SH::MJ);
        const C2SRow& row = C2S_ROWS[LJ][mj];
        double v = 0.0;
        for (int z = 0; z < row.nnz; ++z) v += row.c[z] * bufA[mi + SH::MI * (row.f[z] + SH::NFJ * rest)];
        bufB[o] = v;
      }
      group_sync<S>(group);
      cur = bufB;
    }
    if constexpr (LK >= 2) {
      double* nxt = (cur == bufA) ? bufB : bufA;
      constexpr int n = SH::MI * SH::MJ * SH::MK * SH::NFL;
      for (int o = lane; o < n; o += S) {
        const int mij = o % (SH::MI * SH::MJ);
        const int mk = (o / (SH::MI * SH::MJ)) % SH::MK;
        const int fl = o / (SH::MI * SH::MJ * SH::MK);
        const C2SRow& row = C2S_ROWS[LK][mk];
        double v = 0.0;
        for (int z = 0; z < row.nnz; ++z) v += row.c[z] * cur[mij + SH::MI * SH::MJ * (row.f[z] + SH::NFK * fl)];
        nxt[o] = v;
      }
      group_sync<S>(group);
      cur = nxt;
    }
    {
      constexpr int n = SH::NOUT;
      constexpr int MIJK = SH::MI * SH::MJ * SH::MK;
      for (int o = lane; o < n; o += S) {
        const int mi = o % SH::MI;
        const int mj = (o / SH::MI) % SH::MJ;
        const int mk = (o / (SH::MI * SH::MJ)) % SH::MK;
        const int ml = o / MIJK;
        const int mijk = o % MIJK;
        double v;
        if constexpr (LL >= 2) {
          const C2SRow& row = C2S_ROWS[LL][ml];
          v = 0.0;
          for (int z = 0; z < row.nnz; ++z) v += row.c[z] * cur[mijk + MIJK * row.f[z]];
        } else {
          v = cur[mijk + MIJK * ml];
        }
        obase[mi * st.s0 + mj * st.s1 + mk * st.s2 + ml * st.s3] = v;
      }
    }
    group_sync<S>(group);
  }
}

template <int LI, int LJ, int LK, int LL, int ACC>
cudaError_t launch_splitcoop(const LaunchArgs& a) {
  using SH = EriShape<LI, LJ, LK, LL, true, double, ACC, kSplitCoopRegs>;
  constexpr SplitCoopDims D = splitcoop_dims(LI, LJ, LK, LL, ACC);
  if (a.query) return cudaSuccess;  // transform buffers on chip: no scratch
  auto kern = eri_splitcoop_kernel<LI, LJ, LK, LL, ACC>;
  static int attr_done[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (D.SMEM_BYTES > 48 * 1024 && dev < 64 && !attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, D.SMEM_BYTES);
    if (e != cudaSuccess) return e;
    attr_done[dev] = 1;
  }
  if (a.nrec <= 0) return cudaSuccess;
  long long blocks = ((long long)a.nrec + SH::Q - 1) / SH::Q;
  const long long cap = a.max_blocks > 0 ? a.max_blocks : (long long)device_sm_count() * 32;
  if (blocks > cap) blocks = cap;
  kern<<<(unsigned)blocks, SH::BLOCK, D.SMEM_BYTES, a.stream>>>(a.recs, a.nrec, a.pairs, a.prims, a.out, a.st,
                                                                a.expcutoff, a.rys, a.prim_eps, a.rootbuf,
                                                                a.rootbase);
  return cudaGetLastError();
}

}  // namespace cintx
