// Fused Rys-quadrature ERI kernel for one angular-momentum class (LI LJ | LK LL).
//
// Work unit: one contracted shell quartet (ij|kl), processed by a group of S threads
// (S = 1 .. 256, a power of two).  Per surviving primitive quartet the group computes
//   1. x = a0 |P-Q|^2 and the prefactor (CINTg0_2e, g2e.c:4425-4475),
//   2. the NR Rys roots/weights (rys_roots.cuh; lanes split the 2*NR table polynomials),
//   3. the 3*NR (axis, root) 2D recurrences (VRR, CINTg0_2e_2d g2e.c:272) built on centres
//      i and k, each followed by the horizontal transfer to j and l (g2e.c:428-694) in closed
//      binomial form I(i,j) = sum_a C(j,a) (A-B)^(j-a) G(i+a), from registers into shared memory,
//   4. the cartesian products sum_r Ix Iy Iz (CINTgout2e, cint2e.c:961) accumulated in
//      registers: each lane owns whole (fj,fk,fl) tuples and all fi of each tuple.
// After the primitive loop the i-axis cart->sph transform (c2s_sph_2e1, cart2sph.c:5324) is
// applied in registers, the j/k axes in shared memory, and the l axis on the way to global
// memory, with consecutive lanes writing consecutive doubles of the libcint-layout block.
//
// Shell pairs are oriented so that LI >= LJ and LK >= LL (the VRR is built on the larger
// angular momentum, libcint's ibase/kbase choice, g2e.c:98-116).  Output strides let a launch
// write any requested index order of the block.
#pragma once
#include <type_traits>
#include <utility>

#include "common.h"
#include "c2s_coef.h"
#include "rys_roots.cuh"

namespace cintx {

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int cart_x(int l, int f) {
  int lx = l;
  while (f >= l - lx + 1) { f -= l - lx + 1; --lx; }
  return lx;
}
__host__ __device__ constexpr int cart_y(int l, int f) {
  int lx = l;
  while (f >= l - lx + 1) { f -= l - lx + 1; --lx; }
  return l - lx - f;
}
__host__ __device__ constexpr int cart_z(int l, int f) { return l - cart_x(l, f) - cart_y(l, f); }
__host__ __device__ constexpr int binom(int n, int k) {
  int r = 1;
  for (int i = 0; i < k; ++i) r = r * (n - i) / (i + 1);
  return r;
}
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }

// Threads per quartet: smallest power of two keeping <= 24 accumulators per lane, capped by
// the tuple count and by 256.
// Lanes per quartet: the fewest (a power of two, at most twice the (j,k,l) tuple count) that
// keep a lane's cartesian accumulators within `acc` doubles.
__host__ __device__ constexpr int pick_threads(int li, int lj, int lk, int ll, int acc = 24) {
  const int ntup = ncart(lj) * ncart(lk) * ncart(ll);
  const int total = ntup * ncart(li);
  int s = 1;
  while (s < 256 && (total + s - 1) / s > acc && s * 2 <= ntup * 2) s *= 2;
  return s;
}

// Launch-shape variants the autotuner chooses between: the accumulator budget per lane and the
// register cap of multi-lane shapes (variant 0 is the default shape, used by plans that are not
// autotuned).  A 255-register cap halves the resident blocks but removes the spills that the
// 128-register cap forces on most d/f/g multi-lane classes.
// Variants 4, 5 and 6 ("sliced") run a multi-lane class without any barrier inside the primitive
// loop: every lane evaluates the roots and all 3*NR recurrences itself in registers and
// accumulates its own slice of (j,k,l) tuples (redundant FP64 work for no shared-memory
// hand-offs); the lanes meet only for the cartesian-to-spherical stages.
// Variants 7 and 8 are variants 5 and 4 with the root loop rolled (a quarter to a fifth of the
// code per slice: the slices' bodies compete for the instruction cache).  Variant 9 runs the eight
// slices of variant 6 on four warps, two slices after one another per warp.  Variants 10 and 11
// are cooperative shapes with the horizontal transfers split over all lanes (eri_splitcoop.cuh).
constexpr int kNumVariants = 12;
__host__ __device__ constexpr int variant_acc(int v) {
  return v == 1 || v == 5 || v == 6 || v == 7 || v == 9 ? 48 : (v == 2 ? 12 : (v == 4 || v == 8 ? 32 : 24));
}
__host__ __device__ constexpr int variant_passes(int v) { return v == 9 ? 2 : 1; }
__host__ __device__ constexpr bool variant_roll(int v) { return v == 7 || v == 8; }
__host__ __device__ constexpr int variant_regs(int v) { return v == 0 || v == 2 ? 128 : 255; }
__host__ __device__ constexpr bool variant_sliced(int v) { return v >= 4 && v <= 9; }
// a sliced shape applies to 2..4 lanes whose three recurrence tables fit in registers (variants
// 4, 5), or to 8 lanes whose tables hold at most 108 values (variant 6: a lane keeps only the
// entries its own tuples read; each lane's slice is a separate compile-time instance of the
// register path)
__host__ __device__ constexpr bool sliced_ok(int li, int lj, int lk, int ll, int v) {
  return v == 6 || v == 9 ? pick_threads(li, lj, lk, ll, variant_acc(v)) == 8 &&
                      3 * (li + 1) * (lj + 1) * (lk + 1) * (ll + 1) <= 108
                : variant_sliced(v) && pick_threads(li, lj, lk, ll, variant_acc(v)) >= 2 &&
                      pick_threads(li, lj, lk, ll, variant_acc(v)) <= 4 &&
                      3 * (li + 1) * (lj + 1) * (lk + 1) * (ll + 1) <= (v == 4 || v == 8 ? 48 : 72);
}

template <int LI, int LJ, int LK, int LL, bool SPH, class R = double, int ACC = 24, int REGS = 128,
          bool SLICE = false, bool ROLL = false, int PASSES = 1>
struct EriShape {
  static constexpr int NR = (LI + LJ + LK + LL) / 2 + 1;
  static constexpr int NI = LI + 1, NJ = LJ + 1, NK = LK + 1, NL = LL + 1;
  static constexpr int NIJ = LI + LJ + 1, NKL = LK + LL + 1;
  static constexpr int GSZ = NI * NJ * NK * NL;
  static constexpr int NFI = ncart(LI), NFJ = ncart(LJ), NFK = ncart(LK), NFL = ncart(LL);
  static constexpr int NTUP = NFJ * NFK * NFL;
  static constexpr int S = pick_threads(LI, LJ, LK, LL, ACC);
  static constexpr int TPT = (NTUP + S - 1) / S;
  static constexpr int MI = SPH && LI >= 2 ? 2 * LI + 1 : NFI;
  static constexpr int MJ = SPH && LJ >= 2 ? 2 * LJ + 1 : NFJ;
  static constexpr int MK = SPH && LK >= 2 ? 2 * LK + 1 : NFK;
  static constexpr int ML = SPH && LL >= 2 ? 2 * LL + 1 : NFL;
  static constexpr int NOUT = MI * MJ * MK * ML;
  // shared memory per group (doubles): roots + g arrays during the primitive loop, two
  // transform buffers afterwards (they alias)
  static constexpr int SM_ROOTS = 2 * NR;
  static constexpr int SM_G = 3 * NR * GSZ;
  static constexpr int SM_BUFA = MI * NTUP;
  static constexpr int SM_BUFB = MI * MJ * NFK * NFL;
  // small classes with few lanes run each (axis, root) recurrence in registers and write only
  // the final I values to shared memory; the others keep the 2D table in shared memory (with
  // 4+ lanes the unrolled form spills under the 128-register cap and measured slower)
  static constexpr bool REG_RECUR = S <= 2 && NIJ * NKL <= 16 && GSZ <= 36;
  // non-default launch shapes with at least twice as many lanes as (axis, root) tasks split each
  // task's horizontal transfers over NPARTS lanes (the default shape keeps one lane per task)
  static constexpr int NPARTS_RAW = (!(ACC == 24 && REGS == 128) && !REG_RECUR && S >= 6 * NR) ? S / (3 * NR) : 1;
  static constexpr int NPARTS = NPARTS_RAW < NI ? NPARTS_RAW : NI;
  static constexpr int NTASK_CONC = S < 3 * NR * NPARTS ? S : 3 * NR * NPARTS;  // tasks running at once
  static constexpr int SM_SCR = REG_RECUR ? 0 : NTASK_CONC * NIJ * NKL;  // per-task 2D tables
  // classes whose transform buffers do not fit on chip keep them in a per-block global scratch
  static constexpr bool GLOBAL_BUF = S > 1 && (SM_BUFA + SM_BUFB) * 8 * (S >= 128 ? 1 : 128 / S) > 200 * 1024;
  static constexpr int GBUF_PER_BLOCK = GLOBAL_BUF ? SM_BUFA + SM_BUFB : 0;
  // group region in bytes: roots (double) | I arrays and 2D tables (R) during the primitive
  // loop; the transform buffers (double) alias it afterwards
  static constexpr int B_ROOTS = SM_ROOTS * 8;
  static constexpr int B_G = SM_G * (int)sizeof(R);
  static constexpr int B_SCR = SM_SCR * (int)sizeof(R);
  static constexpr int B_GROUP_RAW =
      S == 1 ? 0
             : (SLICE ? (GLOBAL_BUF ? 0 : (SM_BUFA + SM_BUFB) * 8)
                      : cmax(B_ROOTS + B_G + B_SCR, GLOBAL_BUF ? 0 : (SM_BUFA + SM_BUFB) * 8));
  // sliced shapes: the 32 lanes of a warp belong to 32 groups and read the same offset of their
  // transform buffers, so the group stride is an odd number of doubles (no bank conflicts within
  // a 16-lane phase of an 8-byte access); other shapes keep 16-byte group alignment
  static constexpr int B_GROUP = SLICE ? ((B_GROUP_RAW + 7) / 8 + ((B_GROUP_RAW + 7) / 8 % 2 == 0 ? 1 : 0)) * 8
                                       : (B_GROUP_RAW + 15) & ~15;
  // threads per quartet: S, or for sliced shapes run in PASSES passes, S / PASSES warps' lanes
  static constexpr int LANES = SLICE ? S / PASSES : S;
  static constexpr int BLOCK = SLICE ? cmax(128, 32 * LANES) : (S >= 128 ? S : 128);
  // 8-lane sliced shapes loop over the roots instead of unrolling them (eight compile-time
  // slices of NR unrolled root bodies made the compile time explode)
  static constexpr bool ROLL_ROOTS = SLICE && (S >= 8 || ROLL);
  // resident blocks requested from the register allocator: <= 128 registers per thread for the
  // multi-lane kernels (their stalls are latency bound and need warps)
  static constexpr int MINB = S == 1 ? 1 : (65536 / (BLOCK * REGS) > 0 ? 65536 / (BLOCK * REGS) : 1);
  static constexpr int Q = BLOCK / LANES;
  // one-lane classes of low order stage their root-table block in shared memory: the lanes'
  // scattered coefficient loads then cost shared-memory wavefronts instead of L1 sectors
  // (multi-lane groups evaluate each root once per group; a per-block copy there costs more
  // occupancy than it saves, measured)
  static constexpr bool STAGE_TABLE = S == 1 && NR <= 3;
  static constexpr int TABLE_DOUBLES = STAGE_TABLE ? cintx_rys_xmax(NR) * rys_stage_stride(NR) : 0;
  static constexpr int SMEM_BYTES = Q * B_GROUP + TABLE_DOUBLES * 8;
  static constexpr bool IS_SLICE = SLICE;
  static constexpr int NPASS = PASSES;
};

// Index bounds of a launch shape.  Every shared-memory, scratch, barrier and per-thread index
// eri4c_kernel forms is a function of the shape's constants and of threadIdx.x < BLOCK, so these
// conditions bound all of them; the kernel static_asserts the result for every compiled shape.
// Returns 0, or the number of the first condition that fails.
template <class SH>
__host__ __device__ constexpr int shape_violation() {
  // 1: S is a power of two in [1, 256]; a sliced shape splits its S slices over PASSES passes
  if (SH::S < 1 || SH::S > 256 || (SH::S & (SH::S - 1)) != 0) return 1;
  if (SH::IS_SLICE ? (SH::S % SH::NPASS != 0 || SH::LANES * SH::NPASS != SH::S) : SH::LANES != SH::S) return 1;
  // 2: the block is a whole number of quartet groups (group = threadIdx.x / S, or for sliced
  //    shapes set * 32 + lane with 32 * LANES threads per set), so group < Q
  if (SH::BLOCK > 1024 || SH::BLOCK % (SH::IS_SLICE ? 32 * SH::LANES : SH::S) != 0) return 2;
  if (SH::Q * SH::LANES != SH::BLOCK) return 2;
  // 3: every (j,k,l) tuple has an owner: lane + S*k over k < TPT covers [0, NTUP)
  if (SH::TPT * SH::S < SH::NTUP) return 3;
  // 4: the primitive-loop region of a cooperative group (roots, 3*NR I arrays, one 2D table per
  //    lane that runs a recurrence task, i.e. lanes < min(S, 3*NR*NPARTS)) lies inside the group
  if (SH::S > 1 && !SH::IS_SLICE) {
    if (SH::B_ROOTS + SH::B_G + SH::B_SCR > SH::B_GROUP) return 4;
    if (!SH::REG_RECUR && SH::SM_SCR < cmin(SH::S, 3 * SH::NR * SH::NPARTS) * SH::NIJ * SH::NKL) return 4;
  }
  // 5: the two transform buffers lie inside the group region (or the per-block global scratch,
  //    which then serves exactly one group per block)
  if (SH::S > 1 && !SH::GLOBAL_BUF && (SH::SM_BUFA + SH::SM_BUFB) * 8 > SH::B_GROUP) return 5;
  if (SH::GLOBAL_BUF && (SH::Q != 1 || SH::GBUF_PER_BLOCK != SH::SM_BUFA + SH::SM_BUFB)) return 5;
  // 6: each transform stage's output fits the buffer it is written to: stage j -> B, stage k ->
  //    A (after stage j) or B, and stage i fills A
  if (SH::MI * SH::NTUP > SH::SM_BUFA) return 6;
  if (SH::MI * SH::MJ * SH::NFK * SH::NFL > SH::SM_BUFB) return 6;
  if (SH::MI * SH::MJ * SH::MK * SH::NFL > (SH::MJ != SH::NFJ ? SH::SM_BUFA : SH::SM_BUFB)) return 6;
  // 7: group regions keep their alignment and the block's dynamic shared memory is the sum
  if (SH::B_GROUP % 8 != 0 || (!SH::IS_SLICE && SH::B_GROUP % 16 != 0)) return 7;
  if (SH::SMEM_BYTES != SH::Q * SH::B_GROUP + SH::TABLE_DOUBLES * 8 || SH::SMEM_BYTES > 227 * 1024) return 7;
  // 8: named barriers: ids 1..15 and thread counts that are multiples of 32
  if (!SH::IS_SLICE && SH::S > 32 && (SH::Q > 15 || SH::S % 32 != 0)) return 8;
  if (SH::IS_SLICE && SH::BLOCK != 32 * SH::LANES && SH::BLOCK / (32 * SH::LANES) > 15) return 8;
  // 9: a warp-level group's lanes lie in one warp
  if (!SH::IS_SLICE && SH::S <= 32 && 32 % SH::S != 0) return 9;
  return 0;
}

// Group barrier: warp-level for S <= 32, a named barrier per group above.
template <int S>
__device__ __forceinline__ void group_sync(int group) {
  if constexpr (S == 1) {
  } else if constexpr (S <= 32) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned base = lane & ~(unsigned)(S - 1);
    const unsigned mask = (S == 32) ? 0xffffffffu : (((1u << S) - 1u) << base);
    __syncwarp(mask);
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(S) : "memory");
  }
}

// Barrier of one quartet's lanes.  Sliced shapes spread a quartet's S lanes over S warps (one
// lane per warp, see eri4c_kernel), so their S warps meet at a named barrier per set of S warps.
template <int S, bool SLICE, int BLOCK>
__device__ __forceinline__ void quartet_sync(int group) {
  if constexpr (SLICE && BLOCK == 32 * S) {
    __syncthreads();
  } else if constexpr (SLICE) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / (32 * S))), "r"(32 * S) : "memory");
  } else {
    group_sync<S>(group);
  }
}

// e[j][a] = C(j, a) x^(j - a) for a <= j <= N (zero above the diagonal), by Pascal's rule
// e[j][a] = e[j-1][a-1] + x e[j-1][a]: the binomial weights of the horizontal transfer come out of
// multiply-adds on registers, with no integer binomial evaluated in the unrolled loops.
template <int N, class R>
__device__ __forceinline__ void pascal_powers(R (&e)[N + 1][N + 1], R x) {
#pragma unroll
  for (int j = 0; j <= N; ++j)
#pragma unroll
    for (int a = 0; a <= N; ++a) e[j][a] = (R)0;
  e[0][0] = (R)1;
#pragma unroll
  for (int j = 1; j <= N; ++j)
#pragma unroll
    for (int a = 0; a <= j; ++a) e[j][a] = (a > 0 ? e[j - 1][a - 1] : (R)0) + (a < j ? x * e[j - 1][a] : (R)0);
}

// 2D recurrence for one (axis, root) followed by the horizontal transfers; writes
// I[i + NI*(j + NJ*(k + NK*l))] to dst (stride 1).
template <int LI, int LJ, int LK, int LL, class R = double>
__device__ __forceinline__ void vrr_hrr(R* __restrict__ dst, R g00, R c00, R c0p, R b10, R b01, R b00, R ab, R cd) {
  constexpr int NIJ = LI + LJ + 1, NKL = LK + LL + 1;
  constexpr int NI = LI + 1, NJ = LJ + 1, NK = LK + 1;
  R G[NIJ][NKL];
  G[0][0] = g00;
#pragma unroll
  for (int n = 1; n < NIJ; ++n)
    G[n][0] = c00 * G[n - 1][0] + (n > 1 ? (R)(n - 1) * b10 * G[n - 2][0] : (R)0);
#pragma unroll
  for (int m = 1; m < NKL; ++m) {
#pragma unroll
    for (int n = 0; n < NIJ; ++n) {
      R v = c0p * G[n][m - 1];
      if (m > 1) v += (R)(m - 1) * b01 * G[n][m - 2];
      if (n > 0) v += (R)n * b00 * G[n - 1][m - 1];
      G[n][m] = v;
    }
  }
  R ej[LJ + 1][LJ + 1], el[LL + 1][LL + 1];
  pascal_powers<LJ, R>(ej, ab);
  pascal_powers<LL, R>(el, cd);
  // two stages: T(i, j, m) = sum_a e_j[a] G(i+a, m), then I(i, j, k, l) = sum_b e_l[b] T(i, j, k+b)
#pragma unroll
  for (int j = 0; j <= LJ; ++j)
#pragma unroll
    for (int i = 0; i <= LI; ++i) {
      R T[NKL];
#pragma unroll
      for (int m = 0; m < NKL; ++m) {
        R v = (R)0;
#pragma unroll
        for (int a = 0; a <= j; ++a) v += ej[j][a] * G[i + a][m];
        T[m] = v;
      }
#pragma unroll
      for (int l = 0; l <= LL; ++l)
#pragma unroll
        for (int k = 0; k <= LK; ++k) {
          R v = (R)0;
#pragma unroll
          for (int b = 0; b <= l; ++b) v += el[l][b] * T[k + b];
          dst[i + NI * (j + NJ * (k + NK * l))] = v;
        }
    }
}

// The 2D table of one (axis, root) (the vertical recurrence of vrr_hrr, CINTg0_2e_2d g2e.c:272),
// built in registers one column m at a time (three columns live, every index a compile-time
// constant) and stored to gt[n * NKL + m].
template <int NIJ, int NKL, class R>
__device__ __forceinline__ void vrr_columns(R* __restrict__ gt, R g00, R c00, R c0p, R b10, R b01, R b00) {
  R c1[NIJ], c2[NIJ];  // columns m - 1 and m - 2
  c1[0] = g00;
#pragma unroll
  for (int n = 1; n < NIJ; ++n) c1[n] = c00 * c1[n - 1] + (n > 1 ? (R)(n - 1) * b10 * c1[n - 2] : (R)0);
#pragma unroll
  for (int n = 0; n < NIJ; ++n) {
    gt[n * NKL] = c1[n];
    c2[n] = (R)0;
  }
#pragma unroll
  for (int m = 1; m < NKL; ++m) {
    R c[NIJ];
#pragma unroll
    for (int n = 0; n < NIJ; ++n) {
      R v = c0p * c1[n];
      if (m > 1) v += (R)(m - 1) * b01 * c2[n];
      if (n > 0) v += (R)n * b00 * c1[n - 1];
      c[n] = v;
    }
#pragma unroll
    for (int n = 0; n < NIJ; ++n) {
      gt[n * NKL + m] = c[n];
      c2[n] = c1[n];
      c1[n] = c[n];
    }
  }
}

// Shared-memory version for the multi-lane path: the 2D table lives in gs[n*NKL + m]; the
// horizontal transfers are unrolled over j and the (k, l) outputs, looped over i.
// NPARTS > 1: this call writes only the i = part, part + NPARTS, ... rows of the transfers (the
// other parts of the same (axis, root) task run on other lanes, each with its own 2D table).
template <int LI, int LJ, int LK, int LL, class R = double, int NPARTS = 1>
__device__ __forceinline__ void vrr_hrr_smem(R* __restrict__ dst, R* __restrict__ gs, R g00, R c00, R c0p, R b10,
                                             R b01, R b00, R ab, R cd, int part = 0) {
  constexpr int NIJ = LI + LJ + 1, NKL = LK + LL + 1;
  constexpr int NI = LI + 1, NJ = LJ + 1, NK = LK + 1;
  vrr_columns<NIJ, NKL, R>(gs, g00, c00, c0p, b10, b01, b00);
  R ej[LJ + 1][LJ + 1], el[LL + 1][LL + 1];
  pascal_powers<LJ, R>(ej, ab);
  pascal_powers<LL, R>(el, cd);
  for (int i = NPARTS > 1 ? part : 0; i <= LI; i += NPARTS) {
#pragma unroll
    for (int j = 0; j <= LJ; ++j) {
      R T[NKL];
#pragma unroll
      for (int m = 0; m < NKL; ++m) {
        R v = (R)0;
#pragma unroll
        for (int a = 0; a <= j; ++a) v += ej[j][a] * gs[(i + a) * NKL + m];
        T[m] = v;
      }
#pragma unroll
      for (int l = 0; l <= LL; ++l)
#pragma unroll
        for (int k = 0; k <= LK; ++k) {
          R v = (R)0;
#pragma unroll
          for (int b = 0; b <= l; ++b) v += el[l][b] * T[k + b];
          dst[i + NI * (j + NJ * (k + NK * l))] = v;
        }
    }
  }
}

// The LI+1 values I(0..LI) of one (axis, root) table at a tuple's offset p (stride 1 in i): 16-byte
// loads when NI = LI+1 is even.  Those loads are aligned: the group regions start on 16 bytes, the
// I arrays follow 2*NR doubles of roots, each (axis, root) table holds GSZ = NI*NJ*NK*NL doubles
// (even) and every tuple offset is a multiple of NI.
template <int NI>
__device__ __forceinline__ void load_i_column(double (&v)[NI], const double* __restrict__ p) {
  if constexpr (NI % 2 == 0) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int h = 0; h < NI / 2; ++h) {
      const double2 t = q[h];
      v[2 * h] = t.x;
      v[2 * h + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int h = 0; h < NI; ++h) v[h] = p[h];
  }
}

// L1 prefetch of the primitive-pair record the next loop iteration reads (one 64-byte line), in the
// cooperative shapes' primitive loops (in the one-lane path its address arithmetic raised the
// register count past an occupancy step: (10|00) 8% slower).  No address past the pair's records
// is prefetched.
__device__ __forceinline__ void prefetch_prim(const PrimPair* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Per-lane handles on the tuples it owns.
template <class SH>
struct LaneTuples {
  int ox[SH::TPT], oy[SH::TPT], oz[SH::TPT];
};

template <class SH, int LJ, int LK, int LL>
__device__ __forceinline__ void decode_tuples(LaneTuples<SH>& lt, int lane) {
#pragma unroll
  for (int k = 0; k < SH::TPT; ++k) {
    int t = lane + SH::S * k;
    if (t >= SH::NTUP) t = 0;
    const int fj = t % SH::NFJ;
    const int fk = (t / SH::NFJ) % SH::NFK;
    const int fl = t / (SH::NFJ * SH::NFK);
    int jx = 0, jy = 0, kx = 0, ky = 0, lx = 0, ly = 0;
    // runtime cartesian decomposition (tiny loops; done once per kernel)
    {
      int f = fj, x = LJ;
      while (f >= LJ - x + 1) { f -= LJ - x + 1; --x; }
      jx = x; jy = LJ - x - f;
    }
    {
      int f = fk, x = LK;
      while (f >= LK - x + 1) { f -= LK - x + 1; --x; }
      kx = x; ky = LK - x - f;
    }
    {
      int f = fl, x = LL;
      while (f >= LL - x + 1) { f -= LL - x + 1; --x; }
      lx = x; ly = LL - x - f;
    }
    const int jz = LJ - jx - jy, kz = LK - kx - ky, lz = LL - lx - ly;
    constexpr int SJ = SH::NI, SK = SH::NI * SH::NJ, SL = SH::NI * SH::NJ * SH::NK;
    lt.ox[k] = jx * SJ + kx * SK + lx * SL;
    lt.oy[k] = jy * SJ + ky * SK + ly * SL;
    lt.oz[k] = jz * SJ + kz * SK + lz * SL;
  }
}

// Calls f(std::integral_constant<int, I>) for I = 0..N-1 in order (compile-time unrolling).
template <class F, int... I>
__device__ __forceinline__ void static_loop(std::integer_sequence<int, I...>, F&& f) {
  (f(std::integral_constant<int, I>{}), ...);
}

// Compile-time offsets of every (fj, fk, fl) tuple into the I arrays, for the one-lane path
// (runtime offsets would force its register arrays into local memory).
template <class SH, int LJ, int LK, int LL>
struct TupleOffsets {
  int ox[SH::NTUP], oy[SH::NTUP], oz[SH::NTUP];
  constexpr TupleOffsets() : ox(), oy(), oz() {
    constexpr int SJ = SH::NI, SK = SH::NI * SH::NJ, SL = SH::NI * SH::NJ * SH::NK;
    for (int t = 0; t < SH::NTUP; ++t) {
      const int fj = t % SH::NFJ, fk = (t / SH::NFJ) % SH::NFK, fl = t / (SH::NFJ * SH::NFK);
      ox[t] = cart_x(LJ, fj) * SJ + cart_x(LK, fk) * SK + cart_x(LL, fl) * SL;
      oy[t] = cart_y(LJ, fj) * SJ + cart_y(LK, fk) * SK + cart_y(LL, fl) * SL;
      oz[t] = cart_z(LJ, fj) * SJ + cart_z(LK, fk) * SK + cart_z(LL, fl) * SL;
    }
  }
};

// Primitive loop of the one-lane classes.  Quartets of a warp share their (ij) pair (row-major
// tiles), so the inner loop's primitive-pair loads are warp-wide broadcasts; the lane's (kl)
// primitive pair is loaded once per outer iteration.  `tab` is the shared-memory copy of the
// order-NR root table when SH::STAGE_TABLE (otherwise the global table is read).
template <int LI, int LJ, int LK, int LL, class SH, class R, int SLICE = 0>
__device__ __forceinline__ void prim_loop_one_lane(const ShellPair& pij, const ShellPair& pkl,
                                                   const PrimPair* __restrict__ prims, const RysTable& rys,
                                                   const double* tab, double expcutoff, double prim_eps,
                                                   const double* __restrict__ rb, const LaneTuples<SH>& lt,
                                                   double (&acc)[SH::TPT][SH::NFI]) {
  constexpr int NR = SH::NR, GSZ = SH::GSZ, NFI = SH::NFI, TPT = SH::TPT;
  constexpr bool SSSS = LI + LJ + LK + LL == 0;
  for (int b = 0; b < pkl.nprim; ++b) {
    const PrimPair pk = prims[pkl.prim_off + b];
    const double qcx = pk.px - pkl.ax, qcy = pk.py - pkl.ay, qcz = pk.pz - pkl.az;
    // primitive Schwarz screening: (ij) pairs are sorted by q, so stop at the first one whose
    // bound q_ij * q_kl < prim_eps (prim_eps == 0 gives NaN or 0 here: never stops)
    const double qthr = prim_eps / pk.q;
    for (int a = 0; a < pij.nprim; ++a) {
      const PrimPair pi = prims[pij.prim_off + a];
      if (pi.q < qthr) break;
      if (pi.cce + pk.cce > expcutoff) continue;  // CINT2e_loop eijcutoff (cint2e.c:700-712)
      const double aij = pi.aij, akl = pk.aij;
      const double aijkl = aij + akl;
      const double rs = rsqrt(aijkl);
      const double inv_aijkl = rs * rs;
      const double a1 = aij * akl;
      const double inv_a1 = 4.0 * pi.half_inv * pk.half_inv;
      const double pqx = pi.px - pk.px, pqy = pi.py - pk.py, pqz = pi.pz - pk.pz;
      const double rr = pqx * pqx + pqy * pqy + pqz * pqz;
      const double x = a1 * inv_aijkl * rr;
      const double fac = pi.kab * pk.kab * rs * inv_a1;
      double t2[NR], w[NR];
      if (rb) {  // roots precomputed for this primitive quartet (learned-root plans)
        const double* r = rb + (size_t)(b * pij.nprim + a) * (2 * NR);
#pragma unroll
        for (int i = 0; i < NR; ++i) {
          t2[i] = r[i];
          w[i] = r[NR + i];
        }
      } else if constexpr (SH::STAGE_TABLE) {
        if constexpr (SSSS) rys_all_staged<NR, NR, 2 * NR>(tab, rys, x, t2, w);
        else rys_all_staged<NR>(tab, rys, x, t2, w);
      } else {
        if constexpr (SSSS) rys_all<NR, NR, 2 * NR>(rys, x, t2, w);
        else rys_all<NR>(rys, x, t2, w);
      }
      if constexpr (SSSS) {
        acc[0][0] = fma(w[0], fac, acc[0][0]);  // (ss|ss) needs the weight only
      } else {
        const double pax = pi.px - pij.ax, pay = pi.py - pij.ay, paz = pi.pz - pij.az;
        // reduced-precision classes sum the roots of one primitive quartet in R and add the sum
        // to the FP64 accumulators (primitive accumulation stays FP64)
        R part[std::is_same<R, double>::value ? 1 : TPT][std::is_same<R, double>::value ? 1 : NFI];
        if constexpr (!std::is_same<R, double>::value) {
#pragma unroll
          for (int k2 = 0; k2 < TPT; ++k2)
#pragma unroll
            for (int f2 = 0; f2 < NFI; ++f2) part[k2][f2] = (R)0;
        }
        auto root_body = [&](const int r) {
          R gg[3 * GSZ];
          const double rt_aa = t2[r] * inv_aijkl;
          const double b00 = 0.5 * rt_aa;
          const double b10 = pi.half_inv * (1.0 - rt_aa * akl);
          const double b01 = pk.half_inv * (1.0 - rt_aa * aij);
          const double ca = rt_aa * akl, cb = rt_aa * aij;
          vrr_hrr<LI, LJ, LK, LL, R>(gg + 0 * GSZ, (R)1, (R)(pax - ca * pqx), (R)(qcx + cb * pqx), (R)b10, (R)b01,
                                     (R)b00, (R)pij.abx, (R)pkl.abx);
          vrr_hrr<LI, LJ, LK, LL, R>(gg + 1 * GSZ, (R)1, (R)(pay - ca * pqy), (R)(qcy + cb * pqy), (R)b10, (R)b01,
                                     (R)b00, (R)pij.aby, (R)pkl.aby);
          vrr_hrr<LI, LJ, LK, LL, R>(gg + 2 * GSZ, (R)(w[r] * fac), (R)(paz - ca * pqz), (R)(qcz + cb * pqz),
                                     (R)b10, (R)b01, (R)b00, (R)pij.abz, (R)pkl.abz);
          // every index below is a constant expression, so gg and acc stay in registers
          static_loop(std::make_integer_sequence<int, TPT * NFI>{}, [&](auto c) {
            constexpr int k = decltype(c)::value / NFI, fi = decltype(c)::value % NFI;
            constexpr int t = SLICE + SH::S * k;  // this lane's k-th (j,k,l) tuple
            if constexpr (t < SH::NTUP) {
              constexpr TupleOffsets<SH, LJ, LK, LL> TO{};
              constexpr int ix = cart_x(LI, fi) + TO.ox[t];
              constexpr int iy = GSZ + cart_y(LI, fi) + TO.oy[t];
              constexpr int iz = 2 * GSZ + cart_z(LI, fi) + TO.oz[t];
              if constexpr (std::is_same<R, double>::value) acc[k][fi] = fma(gg[ix] * gg[iy], gg[iz], acc[k][fi]);
              else part[k][fi] = fmaf(gg[ix] * gg[iy], gg[iz], part[k][fi]);
            }
          });
        };
        if constexpr (SH::ROLL_ROOTS) {  // t2, w then live in local memory: two loads per root
#pragma unroll 1
          for (int r = 0; r < NR; ++r) root_body(r);
        } else {
#pragma unroll
          for (int r = 0; r < NR; ++r) root_body(r);
        }
        if constexpr (!std::is_same<R, double>::value) {
#pragma unroll
          for (int k2 = 0; k2 < TPT; ++k2)
#pragma unroll
            for (int f2 = 0; f2 < NFI; ++f2) acc[k2][f2] += (double)part[k2][f2];
        }
      }
    }
  }
}

template <int LI, int LJ, int LK, int LL, bool SPH, class R = double, int ACC = 24, int REGS = 128,
          bool SLICE = false, bool ROLL = false, int PASSES = 1>
__global__ void __launch_bounds__(EriShape<LI, LJ, LK, LL, SPH, R, ACC, REGS, SLICE, ROLL, PASSES>::BLOCK,
                                  EriShape<LI, LJ, LK, LL, SPH, R, ACC, REGS, SLICE, ROLL, PASSES>::MINB)
    eri4c_kernel(const QuartetRec* __restrict__ recs, int nrec, const ShellPair* __restrict__ pairs,
                 const PrimPair* __restrict__ prims, double* __restrict__ out, OutStrides st,
                 double expcutoff, const __grid_constant__ RysTable rys, double* __restrict__ gscratch,
                 double prim_eps, const double* __restrict__ rootbuf, const long long* __restrict__ rootbase) {
  using SH = EriShape<LI, LJ, LK, LL, SPH, R, ACC, REGS, SLICE, ROLL, PASSES>;
  constexpr int S = SH::S, NR = SH::NR, GSZ = SH::GSZ, NFI = SH::NFI, TPT = SH::TPT;
  constexpr bool FP64 = std::is_same<R, double>::value;
  extern __shared__ __align__(16) double smem[];
  // Sliced shapes run a different compile-time instance of the primitive loop on each of a
  // quartet's S lanes.  Lanes of one quartet therefore sit in S different warps: a set of S warps
  // holds 32 quartets, warp w of the set runs slice w for all of them (no divergence inside a
  // warp), and the set meets at a named barrier for the transform stages.  Other shapes keep a
  // quartet's lanes adjacent within a warp.  With PASSES == 2 a set has S/2 warps and warp w runs
  // slices w and w + S/2 one after the other.
  constexpr int LN = SH::LANES;
  static_assert(!SLICE || (SH::BLOCK % (32 * LN) == 0 && S % PASSES == 0 && !SH::GLOBAL_BUF &&
                           SH::SMEM_BYTES <= 227 * 1024),
                "sliced shape layout");
  static_assert(shape_violation<SH>() == 0, "an index of this launch shape can leave its buffer");
  static_assert(SLICE || S == 1 || (SH::B_GROUP % 16 == 0 && SH::B_ROOTS % 16 == 0 && SH::TABLE_DOUBLES % 2 == 0 &&
                                    (SH::NI % 2 != 0 || SH::GSZ % 2 == 0)),
                "16-byte loads of the I arrays need 16-byte aligned group regions and tables");
  const int group = SLICE ? (int)(threadIdx.x / (32 * LN)) * 32 + (int)(threadIdx.x & 31) : (int)threadIdx.x / S;
  const int lane = SLICE ? (int)(threadIdx.x / 32) % LN : (int)threadIdx.x % S;
  char* sgb = reinterpret_cast<char*>(smem + SH::TABLE_DOUBLES) + group * SH::B_GROUP;
  double* sg = reinterpret_cast<double*>(sgb);  // transform buffers after the primitive loop
  double* s_roots = sg;                         // t2[NR], w[NR]
  R* s_g = reinterpret_cast<R*>(sgb + SH::B_ROOTS);  // [axis][root][GSZ]
  R* s_scr = s_g + SH::SM_G;                    // per-lane 2D tables (lanes < 3*NR)

  if constexpr (SH::STAGE_TABLE) {
    // interval blocks of 2*NR*RYS_NC doubles, each placed rys_stage_stride(NR) doubles apart (the
    // two padding doubles of each interval are never read)
    constexpr int W = NR * RYS_NC, WP = rys_stage_stride(NR) / 2;  // double2 per block, per stride
    const double2* src = reinterpret_cast<const double2*>(rys.poly[NR]);
    double2* dst = reinterpret_cast<double2*>(smem);
    for (int i = threadIdx.x; i < cintx_rys_xmax(NR) * W; i += blockDim.x) dst[(i / W) * WP + i % W] = __ldg(src + i);
    __syncthreads();
  }

  LaneTuples<SH> lt;
  decode_tuples<SH, LJ, LK, LL>(lt, lane);

  // q = blockIdx.x * Q + group; in sliced shapes every thread of a set runs the trip count of the
  // set's first quartet (the set shares barriers) and lanes past the end only take part in them
  const int qfirst = SLICE ? (int)blockIdx.x * SH::Q + (group & ~31) : (int)blockIdx.x * SH::Q + group;
  for (int qb = qfirst; qb < nrec; qb += gridDim.x * SH::Q) {
    const int qv = SLICE ? qb + (group & 31) : qb;
    const bool live = !SLICE || qv < nrec;
    const int q = live ? qv : nrec - 1;
    const QuartetRec rec = recs[q];
    // precomputed roots of this quartet's primitive quartets ([b][a][2*NR]), or table roots
    const double* rb = rootbuf ? rootbuf + rootbase[q] : nullptr;
    const ShellPair pij = pairs[rec.pij];
    const ShellPair pkl = pairs[rec.pkl];
    double acc[TPT][NFI];
#pragma unroll
    for (int k = 0; k < TPT; ++k)
#pragma unroll
      for (int f = 0; f < NFI; ++f) acc[k][f] = 0.0;

    if constexpr (S == 1) {
      prim_loop_one_lane<LI, LJ, LK, LL, SH, R>(pij, pkl, prims, rys, SH::STAGE_TABLE ? smem : nullptr, expcutoff,
                                                prim_eps, rb, lt, acc);
    } else if constexpr (SLICE) {
      // each lane runs the register path for its own tuple slice (lane + S*k)
      static_loop(std::make_integer_sequence<int, S>{}, [&](auto j) {
        constexpr int sl = decltype(j)::value;
        if (live && lane == sl % LN) {
          prim_loop_one_lane<LI, LJ, LK, LL, SH, R, sl>(pij, pkl, prims, rys, nullptr, expcutoff, prim_eps, rb, lt,
                                                        acc);
          if constexpr (PASSES > 1) {
            // stage i of this slice now: the next pass reuses the accumulators
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
              const int t = sl + S * k;
              if (t < SH::NTUP) {
#pragma unroll
                for (int mi = 0; mi < SH::MI; ++mi) {
                  double v = 0.0;
#pragma unroll
                  for (int fi = 0; fi < NFI; ++fi) {
                    const double c = (SPH && LI >= 2) ? c2s_coef(LI, mi, fi) : (mi == fi ? 1.0 : 0.0);
                    if (c != 0.0) v += c * acc[k][fi];
                  }
                  sg[mi + SH::MI * t] = v;
                }
              }
#pragma unroll
              for (int fi = 0; fi < NFI; ++fi) acc[k][fi] = 0.0;
            }
          }
        }
      });
    } else
    for (int b = 0; b < pkl.nprim; ++b) {
      const PrimPair pk = prims[pkl.prim_off + b];
      if (b + 1 < pkl.nprim) prefetch_prim(prims + pkl.prim_off + b + 1);
      const double qcx = pk.px - pkl.ax, qcy = pk.py - pkl.ay, qcz = pk.pz - pkl.az;
      const double qthr = prim_eps / pk.q;  // as in prim_loop_one_lane
      for (int a = 0; a < pij.nprim; ++a) {
        const PrimPair pi = prims[pij.prim_off + a];
        if (a + 1 < pij.nprim) prefetch_prim(prims + pij.prim_off + a + 1);
        if (pi.q < qthr) break;
        if (pi.cce + pk.cce > expcutoff) continue;  // CINT2e_loop eijcutoff (cint2e.c:700-712)
        const double aij = pi.aij, akl = pk.aij;
        const double aijkl = aij + akl;
        const double rs = rsqrt(aijkl);
        const double inv_aijkl = rs * rs;
        const double a1 = aij * akl;
        const double inv_a1 = 4.0 * pi.half_inv * pk.half_inv;
        const double pqx = pi.px - pk.px, pqy = pi.py - pk.py, pqz = pi.pz - pk.pz;
        const double rr = pqx * pqx + pqy * pqy + pqz * pqz;
        const double x = a1 * inv_aijkl * rr;
        const double fac = pi.kab * pk.kab * rs * inv_a1;
        const double pax = pi.px - pij.ax, pay = pi.py - pij.ay, paz = pi.pz - pij.az;

        // roots: the group's lanes split the 2*NR table polynomials (or copy precomputed ones)
        if (rb) {
          const double* r = rb + (size_t)(b * pij.nprim + a) * (2 * NR);
          for (int f = lane; f < 2 * NR; f += S) s_roots[f] = r[f];
        } else if constexpr (SH::STAGE_TABLE) {
          for (int f = lane; f < 2 * NR; f += S) s_roots[f] = rys_fn_staged<NR>(smem, rys, f, x);
        } else {
          for (int f = lane; f < 2 * NR; f += S) s_roots[f] = rys_fn(rys, NR, f, x);
        }
        group_sync<S>(group);
        // (axis, root) recurrences, one per lane; coefficients in FP64, recurrences in R
        for (int tp = lane; tp < 3 * NR * SH::NPARTS; tp += S) {
          const int task = tp / SH::NPARTS, part = tp % SH::NPARTS;
          const int axis = task / NR, r = task % NR;
          const double t2 = s_roots[r];
          const double rt_aa = t2 * inv_aijkl;
          const double b00 = 0.5 * rt_aa;
          const double b10 = pi.half_inv * (1.0 - rt_aa * akl);
          const double b01 = pk.half_inv * (1.0 - rt_aa * aij);
          const double pa = axis == 0 ? pax : (axis == 1 ? pay : paz);
          const double qc = axis == 0 ? qcx : (axis == 1 ? qcy : qcz);
          const double pq = axis == 0 ? pqx : (axis == 1 ? pqy : pqz);
          const double ab = axis == 0 ? pij.abx : (axis == 1 ? pij.aby : pij.abz);
          const double cd = axis == 0 ? pkl.abx : (axis == 1 ? pkl.aby : pkl.abz);
          const double g00 = axis == 2 ? s_roots[NR + r] * fac : 1.0;
          if constexpr (SH::REG_RECUR) {
            vrr_hrr<LI, LJ, LK, LL, R>(s_g + task * GSZ, (R)g00, (R)(pa - rt_aa * akl * pq),
                                       (R)(qc + rt_aa * aij * pq), (R)b10, (R)b01, (R)b00, (R)ab, (R)cd);
          } else {
            vrr_hrr_smem<LI, LJ, LK, LL, R, SH::NPARTS>(s_g + task * GSZ, s_scr + lane * (SH::NIJ * SH::NKL),
                                                        (R)g00, (R)(pa - rt_aa * akl * pq),
                                                        (R)(qc + rt_aa * aij * pq), (R)b10, (R)b01, (R)b00, (R)ab,
                                                        (R)cd, part);
          }
        }
        group_sync<S>(group);
        // cartesian products, summed over roots (R), added to the FP64 accumulators
        R part[FP64 ? 1 : TPT][FP64 ? 1 : NFI];
        if constexpr (!FP64) {
#pragma unroll
          for (int k2 = 0; k2 < TPT; ++k2)
#pragma unroll
            for (int f2 = 0; f2 < NFI; ++f2) part[k2][f2] = (R)0;
        }
#pragma unroll 1
        for (int r = 0; r < NR; ++r) {
          const R* gx = s_g + (0 * NR + r) * GSZ;
          const R* gy = s_g + (1 * NR + r) * GSZ;
          const R* gz = s_g + (2 * NR + r) * GSZ;
#pragma unroll
          for (int k = 0; k < TPT; ++k) {
            if constexpr (FP64) {
              double ix[SH::NI], iy[SH::NI], iz[SH::NI];
              load_i_column<SH::NI>(ix, gx + lt.ox[k]);
              load_i_column<SH::NI>(iy, gy + lt.oy[k]);
              load_i_column<SH::NI>(iz, gz + lt.oz[k]);
              static_loop(std::make_integer_sequence<int, NFI>{}, [&](auto c) {  // fi constant: ix, iy, iz stay in registers
                constexpr int fi = decltype(c)::value;
                constexpr int cx = cart_x(LI, fi), cy = cart_y(LI, fi), cz = cart_z(LI, fi);
                acc[k][fi] = fma(ix[cx] * iy[cy], iz[cz], acc[k][fi]);
              });
            } else {
              static_loop(std::make_integer_sequence<int, NFI>{}, [&](auto c) {
                constexpr int fi = decltype(c)::value;
                constexpr int cx = cart_x(LI, fi), cy = cart_y(LI, fi), cz = cart_z(LI, fi);
                part[k][fi] = fmaf(gx[cx + lt.ox[k]] * gy[cy + lt.oy[k]], gz[cz + lt.oz[k]], part[k][fi]);
              });
            }
          }
        }
        if constexpr (!FP64) {
#pragma unroll
          for (int k2 = 0; k2 < TPT; ++k2)
#pragma unroll
            for (int f2 = 0; f2 < NFI; ++f2) acc[k2][f2] += (double)part[k2][f2];
        }
        group_sync<S>(group);
      }
    }

    // ---- transform to spherical and store ----
    double* const obase = out + rec.out;
    if constexpr (S == 1) {
      // whole block in registers: TPT == NTUP
#pragma unroll
      for (int ml = 0; ml < SH::ML; ++ml)
#pragma unroll
        for (int mk = 0; mk < SH::MK; ++mk)
#pragma unroll
          for (int mj = 0; mj < SH::MJ; ++mj)
#pragma unroll
            for (int mi = 0; mi < SH::MI; ++mi) {
              double v = 0.0;
#pragma unroll
              for (int fl = 0; fl < SH::NFL; ++fl) {
                constexpr bool sl = SPH && LL >= 2;
                const double cl = sl ? c2s_coef(LL, ml, fl) : (ml == fl ? 1.0 : 0.0);
                if (cl == 0.0) continue;
#pragma unroll
                for (int fk = 0; fk < SH::NFK; ++fk) {
                  constexpr bool sk = SPH && LK >= 2;
                  const double ck = sk ? c2s_coef(LK, mk, fk) : (mk == fk ? 1.0 : 0.0);
                  if (ck == 0.0) continue;
#pragma unroll
                  for (int fj = 0; fj < SH::NFJ; ++fj) {
                    constexpr bool sj = SPH && LJ >= 2;
                    const double cj = sj ? c2s_coef(LJ, mj, fj) : (mj == fj ? 1.0 : 0.0);
                    if (cj == 0.0) continue;
#pragma unroll
                    for (int fi = 0; fi < NFI; ++fi) {
                      constexpr bool si = SPH && LI >= 2;
                      const double ci = si ? c2s_coef(LI, mi, fi) : (mi == fi ? 1.0 : 0.0);
                      if (ci == 0.0) continue;
                      v += ci * cj * ck * cl * acc[fj + SH::NFJ * (fk + SH::NFK * fl)][fi];
                    }
                  }
                }
              }
              obase[mi * st.s0 + mj * st.s1 + mk * st.s2 + ml * st.s3] = v;
            }
    } else {
      double* bufA = SH::GLOBAL_BUF ? gscratch + (size_t)blockIdx.x * SH::GBUF_PER_BLOCK : sg;
      double* bufB = bufA + SH::SM_BUFA;
      // stage i in registers -> bufA[mi + MI * t], t = fj + NFJ*(fk + NFK*fl) (two-pass sliced
      // shapes stored it after each pass)
#pragma unroll
      for (int k = 0; k < TPT; ++k) {
        const int t = lane + S * k;
        if (PASSES == 1 && t < SH::NTUP) {
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
      quartet_sync<LN, SLICE, SH::BLOCK>(group);
      // stage j: bufA[mi + MI*(fj + NFJ*(fk + NFK*fl))] -> bufB[mi + MI*(mj + MJ*(fk + NFK*fl))]
      const double* cur = bufA;
      if constexpr (SPH && LJ >= 2) {
        constexpr int n = SH::MI * SH::MJ * SH::NFK * SH::NFL;
        for (int o = lane; o < n; o += LN) {
          const int mi = o % SH::MI;
          const int mj = (o / SH::MI) % SH::MJ;
          const int rest = o / (SH::MI * SH::MJ);
          const C2SRow& row = C2S_ROWS[LJ][mj];
          double v = 0.0;
          for (int z = 0; z < row.nnz; ++z) v += row.c[z] * bufA[mi + SH::MI * (row.f[z] + SH::NFJ * rest)];
          bufB[o] = v;
        }
        quartet_sync<LN, SLICE, SH::BLOCK>(group);
        cur = bufB;
      }
      // stage k: cur[mi + MI*(mj + MJ*(fk + NFK*fl))] -> nxt[mi + MI*(mj + MJ*(mk + MK*fl))]
      if constexpr (SPH && LK >= 2) {
        double* nxt = (cur == bufA) ? bufB : bufA;
        constexpr int n = SH::MI * SH::MJ * SH::MK * SH::NFL;
        for (int o = lane; o < n; o += LN) {
          const int mij = o % (SH::MI * SH::MJ);
          const int mk = (o / (SH::MI * SH::MJ)) % SH::MK;
          const int fl = o / (SH::MI * SH::MJ * SH::MK);
          const C2SRow& row = C2S_ROWS[LK][mk];
          double v = 0.0;
          for (int z = 0; z < row.nnz; ++z)
            v += row.c[z] * cur[mij + SH::MI * SH::MJ * (row.f[z] + SH::NFK * fl)];
          nxt[o] = v;
        }
        quartet_sync<LN, SLICE, SH::BLOCK>(group);
        cur = nxt;
      }
      // stage l + store: cur[mijk + MIJK*fl] -> out
      {
        constexpr int n = SH::NOUT;
        constexpr int MIJK = SH::MI * SH::MJ * SH::MK;
        for (int o = lane; o < n; o += LN) {
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
          if (live) obase[mi * st.s0 + mj * st.s1 + mk * st.s2 + ml * st.s3] = v;
        }
      }
      quartet_sync<LN, SLICE, SH::BLOCK>(group);
    }
  }
}

}  // namespace cintx
