// First-derivative Rys ERI kernel: (d/dx_i i j|k l) for one class (LI LJ | LK LL), the
// int2e_ip1 / int3c2e_ip1 family of libcint (autocode/grad2.c:19-88, autocode/int3c2e.c:72-88).
//
// The derivative acts on the electron coordinate of shell i.  Per primitive quartet the 2D
// integrals are built with the i ceiling raised to LI + 1 (the recurrence and horizontal transfer
// of the plain kernel, vrr_hrr_smem, on centres i and k) and the derivative of each axis is
//   D_x I(ix, ...) = ix I(ix - 1, ...) - 2 a_i I(ix + 1, ...)
// (libcint's G2E_D_I), a_i the exponent of the quartet's i primitive, which the pair tables of
// derivative launches carry in PrimPair::q as 2 a_i.  The three cartesian components are
// evaluated one after the other (each its own pass over the primitive quartets, so a lane holds
// the accumulators of one component), transformed to spherical form like the plain kernel's
// blocks, and written component-major: component c of element e at out + rec.out + c*scomp + e.
//
// Work unit: one contracted quartet per group of S lanes sharing the (axis, root) tables in
// shared memory.  The kernel's first pair is (i, j) in the requested order (no reorientation: the
// derivative stays on axis i); the second pair is oriented like the plain kernel's.
#pragma once
#include "eri_launch.cuh"

namespace cintx {

template <int LI, int LJ, int LK, int LL, bool SPH>
struct Ip1Shape {
  static constexpr int NR = (LI + 1 + LJ + LK + LL) / 2 + 1;
  static constexpr int NI = LI + 2, NJ = LJ + 1, NK = LK + 1, NL = LL + 1;  // i ceiling LI + 1
  static constexpr int NIJ = LI + LJ + 2, NKL = LK + LL + 1;
  static constexpr int GSZ = NI * NJ * NK * NL;
  static constexpr int NFI = ncart(LI), NFJ = ncart(LJ), NFK = ncart(LK), NFL = ncart(LL);
  static constexpr int NTUP = NFJ * NFK * NFL;
  static constexpr int S = pick_threads(LI, LJ, LK, LL, 24);
  static constexpr int TPT = (NTUP + S - 1) / S;
  static constexpr int MI = SPH && LI >= 2 ? 2 * LI + 1 : NFI;
  static constexpr int MJ = SPH && LJ >= 2 ? 2 * LJ + 1 : NFJ;
  static constexpr int MK = SPH && LK >= 2 ? 2 * LK + 1 : NFK;
  static constexpr int ML = SPH && LL >= 2 ? 2 * LL + 1 : NFL;
  static constexpr int NOUT = MI * MJ * MK * ML;
  static constexpr int SM_ROOTS = 2 * NR;
  static constexpr int SM_G = 3 * NR * GSZ;
  static constexpr int NTASK_CONC = S < 3 * NR ? S : 3 * NR;
  static constexpr int SM_SCR = NTASK_CONC * NIJ * NKL;
  static constexpr int SM_BUFA = MI * NTUP;
  static constexpr int SM_BUFB = MI * MJ * NFK * NFL;
  static constexpr int GROUP_DOUBLES_RAW = cmax(SM_ROOTS + SM_G + SM_SCR, SM_BUFA + SM_BUFB);
  static constexpr int GROUP_DOUBLES = (GROUP_DOUBLES_RAW + 1) & ~1;  // 16-byte groups
  // groups per block: up to 128 threads, as many groups as 200 KB of shared memory holds
  static constexpr int QFIT = (200 * 1024) / (GROUP_DOUBLES * 8);
  static constexpr int QWANT = S >= 128 ? 1 : 128 / S;
  static constexpr int Q = QFIT >= QWANT ? QWANT : (QFIT >= 64 ? 64 : QFIT >= 32 ? 32 : QFIT >= 16 ? 16 : QFIT >= 8 ? 8 : QFIT >= 4 ? 4 : QFIT >= 2 ? 2 : 1);
  static constexpr int BLOCK = Q * S;
  static constexpr int SMEM_BYTES = Q * GROUP_DOUBLES * 8;
};

// Index bounds of an ip1 shape (the kernel static_asserts it): groups fill the block, the
// primitive-loop region and the transform buffers fit the group, stages fit their buffers, the
// block's shared memory fits, and named barriers (S > 32) have ids below 16.
template <class SH>
__host__ __device__ constexpr int ip1_shape_violation() {
  if (SH::S < 1 || SH::S > 256 || (SH::S & (SH::S - 1)) != 0) return 1;
  if (SH::BLOCK != SH::Q * SH::S || SH::BLOCK > 1024 || SH::Q < 1) return 2;
  if (SH::TPT * SH::S < SH::NTUP) return 3;
  if (SH::SM_ROOTS + SH::SM_G + SH::SM_SCR > SH::GROUP_DOUBLES) return 4;
  if (SH::SM_BUFA + SH::SM_BUFB > SH::GROUP_DOUBLES) return 5;
  if (SH::MI * SH::MJ * SH::MK * SH::NFL > (SH::MJ != SH::NFJ ? SH::SM_BUFA : SH::SM_BUFB)) return 6;
  if (SH::SMEM_BYTES > 227 * 1024) return 7;
  if (SH::S > 32 && (SH::Q > 15 || SH::S % 32 != 0)) return 8;
  if (SH::S <= 32 && 32 % SH::S != 0) return 9;
  return 0;
}

template <int LI, int LJ, int LK, int LL, bool SPH>
__global__ void __launch_bounds__(Ip1Shape<LI, LJ, LK, LL, SPH>::BLOCK, 1)
    eri_ip1_kernel(const QuartetRec* __restrict__ recs, int nrec, const ShellPair* __restrict__ pairs,
                   const PrimPair* __restrict__ prims, double* __restrict__ out, OutStrides st, long long scomp,
                   double expcutoff, const __grid_constant__ RysTable rys) {
  using SH = Ip1Shape<LI, LJ, LK, LL, SPH>;
  static_assert(ip1_shape_violation<SH>() == 0, "an index of this ip1 launch shape can leave its buffer");
  constexpr int S = SH::S, NR = SH::NR, GSZ = SH::GSZ, NFI = SH::NFI, TPT = SH::TPT;
  constexpr int NI = SH::NI, NJ = SH::NJ, NK = SH::NK;
  extern __shared__ __align__(16) double smem[];
  const int group = (int)threadIdx.x / S;
  const int lane = (int)threadIdx.x % S;
  double* sg = smem + (size_t)group * SH::GROUP_DOUBLES;
  double* s_roots = sg;
  double* s_g = sg + SH::SM_ROOTS;
  double* s_scr = s_g + SH::SM_G;

  // offsets of this lane's (fj, fk, fl) tuples into the I arrays (i ceiling LI + 1)
  int ox[TPT], oy[TPT], oz[TPT];
#pragma unroll
  for (int k = 0; k < TPT; ++k) {
    int t = lane + S * k;
    if (t >= SH::NTUP) t = 0;
    const int fj = t % SH::NFJ, fk = (t / SH::NFJ) % SH::NFK, fl = t / (SH::NFJ * SH::NFK);
    ox[k] = cart_x(LJ, fj) * NI + cart_x(LK, fk) * NI * NJ + cart_x(LL, fl) * NI * NJ * NK;
    oy[k] = cart_y(LJ, fj) * NI + cart_y(LK, fk) * NI * NJ + cart_y(LL, fl) * NI * NJ * NK;
    oz[k] = cart_z(LJ, fj) * NI + cart_z(LK, fk) * NI * NJ + cart_z(LL, fl) * NI * NJ * NK;
  }

  for (int q = (int)blockIdx.x * SH::Q + group; q < nrec; q += (int)gridDim.x * SH::Q) {
    const QuartetRec rec = recs[q];
    const ShellPair pij = pairs[rec.pij];
    const ShellPair pkl = pairs[rec.pkl];
    for (int comp = 0; comp < 3; ++comp) {
      double acc[TPT][NFI];
#pragma unroll
      for (int k = 0; k < TPT; ++k)
#pragma unroll
        for (int f = 0; f < NFI; ++f) acc[k][f] = 0.0;
      for (int b = 0; b < pkl.nprim; ++b) {
        const PrimPair pk = prims[pkl.prim_off + b];
        const double qcx = pk.px - pkl.ax, qcy = pk.py - pkl.ay, qcz = pk.pz - pkl.az;
        for (int a = 0; a < pij.nprim; ++a) {
          const PrimPair pi = prims[pij.prim_off + a];
          if (pi.cce + pk.cce > expcutoff) continue;  // CINT2e_loop eijcutoff (cint2e.c:700-712)
          const double aij = pi.aij, akl = pk.aij;
          const double rs = rsqrt(aij + akl);
          const double inv_aijkl = rs * rs;
          const double inv_a1 = 4.0 * pi.half_inv * pk.half_inv;
          const double pqx = pi.px - pk.px, pqy = pi.py - pk.py, pqz = pi.pz - pk.pz;
          const double x = aij * akl * inv_aijkl * (pqx * pqx + pqy * pqy + pqz * pqz);
          const double fac = pi.kab * pk.kab * rs * inv_a1;
          const double pax = pi.px - pij.ax, pay = pi.py - pij.ay, paz = pi.pz - pij.az;
          const double ai2 = pi.q;  // 2 a_i of this primitive pair's i primitive
          for (int f = lane; f < 2 * NR; f += S) s_roots[f] = rys_fn(rys, NR, f, x);
          group_sync<S>(group);
          for (int task = lane; task < 3 * NR; task += S) {
            const int axis = task / NR, r = task % NR;
            const double rt_aa = s_roots[r] * inv_aijkl;
            const double b00 = 0.5 * rt_aa;
            const double b10 = pi.half_inv * (1.0 - rt_aa * akl);
            const double b01 = pk.half_inv * (1.0 - rt_aa * aij);
            const double pa = axis == 0 ? pax : (axis == 1 ? pay : paz);
            const double qc = axis == 0 ? qcx : (axis == 1 ? qcy : qcz);
            const double pq = axis == 0 ? pqx : (axis == 1 ? pqy : pqz);
            const double ab = axis == 0 ? pij.abx : (axis == 1 ? pij.aby : pij.abz);
            const double cd = axis == 0 ? pkl.abx : (axis == 1 ? pkl.aby : pkl.abz);
            const double g00 = axis == 2 ? s_roots[NR + r] * fac : 1.0;
            vrr_hrr_smem<LI + 1, LJ, LK, LL, double, 1>(s_g + task * GSZ, s_scr + lane * (SH::NIJ * SH::NKL), g00,
                                                        pa - rt_aa * akl * pq, qc + rt_aa * aij * pq, b10, b01, b00,
                                                        ab, cd, 0);
          }
          group_sync<S>(group);
#pragma unroll 1
          for (int r = 0; r < NR; ++r) {
            const double* gx = s_g + (0 * NR + r) * GSZ;
            const double* gy = s_g + (1 * NR + r) * GSZ;
            const double* gz = s_g + (2 * NR + r) * GSZ;
            // the differentiated axis reads D I(i) = i I(i-1) - 2 a_i I(i+1); the others I(i)
            const double* gd = comp == 0 ? gx : (comp == 1 ? gy : gz);
            const double* ga = comp == 0 ? gy : gx;
            const double* gb = comp == 2 ? gy : gz;
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
              const int od = comp == 0 ? ox[k] : (comp == 1 ? oy[k] : oz[k]);
              const int oa = comp == 0 ? oy[k] : ox[k];
              const int ob = comp == 2 ? oy[k] : oz[k];
              static_loop(std::make_integer_sequence<int, NFI>{}, [&](auto c) {  // fi a compile-time constant
                constexpr int fi = decltype(c)::value;
                constexpr int cx = cart_x(LI, fi), cy = cart_y(LI, fi), cz = cart_z(LI, fi);
                const int nd = comp == 0 ? cx : (comp == 1 ? cy : cz);
                const int na = comp == 0 ? cy : cx;
                const int nb = comp == 2 ? cy : cz;
                double d = -ai2 * gd[nd + 1 + od];
                if (nd > 0) d = fma((double)nd, gd[nd - 1 + od], d);
                acc[k][fi] = fma(d * ga[na + oa], gb[nb + ob], acc[k][fi]);
              });
            }
          }
          group_sync<S>(group);
        }
      }
      // ---- transform this component to spherical and store ----
      double* const obase = out + rec.out + comp * scomp;
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
              const double c = (SPH && LI >= 2) ? c2s_coef(LI, mi, fi) : (mi == fi ? 1.0 : 0.0);
              if (c != 0.0) v += c * acc[k][fi];
            }
            bufA[mi + SH::MI * t] = v;
          }
        }
      }
      group_sync<S>(group);
      const double* cur = bufA;
      if constexpr (SPH && LJ >= 2) {
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
      if constexpr (SPH && LK >= 2) {
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
          if constexpr (SPH && LL >= 2) {
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
}

struct Ip1Args {
  const QuartetRec* recs;
  int nrec;
  const ShellPair* pairs;
  const PrimPair* prims;
  double* out;
  OutStrides st;
  long long scomp;
  double expcutoff;
  RysTable rys;
  cudaStream_t stream;
};

template <int LI, int LJ, int LK, int LL, bool SPH>
cudaError_t launch_ip1(const Ip1Args& a) {
  using SH = Ip1Shape<LI, LJ, LK, LL, SPH>;
  auto kern = eri_ip1_kernel<LI, LJ, LK, LL, SPH>;
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
  const long long cap = (long long)device_sm_count() * 32;
  if (blocks > cap) blocks = cap;
  kern<<<(unsigned)blocks, SH::BLOCK, SH::SMEM_BYTES, a.stream>>>(a.recs, a.nrec, a.pairs, a.prims, a.out, a.st,
                                                                  a.scomp, a.expcutoff, a.rys);
  return cudaGetLastError();
}

// Classes compiled for derivatives: the derivative pair (i, j) with li, lj <= 3 in either order,
// the second pair oriented (lk >= ll) with lk <= 3, or lk = 4 with ll = 0 (3-centre g auxiliaries).
__host__ __device__ constexpr bool ip1_class_valid(int li, int lj, int lk, int ll) {
  return li <= 3 && lj <= 3 && lk >= ll && (lk <= 3 || (lk == 4 && ll == 0));
}

template <int LI, int LJ>
cudaError_t dispatch_ip1_lij(int lk, int ll, bool sph, const Ip1Args& a) {
  cudaError_t err = cudaErrorInvalidValue;
  static_for<CINTX_LMAX + 1>([&](auto K) {
    static_for<K.value + 1>([&](auto L) {
      constexpr int k = decltype(K)::value, l = decltype(L)::value;
      if constexpr (ip1_class_valid(LI, LJ, k, l)) {
        if (lk == k && ll == l) err = sph ? launch_ip1<LI, LJ, k, l, true>(a) : launch_ip1<LI, LJ, k, l, false>(a);
      }
    });
  });
  return err;
}

}  // namespace cintx
