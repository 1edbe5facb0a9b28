// Host-side internals shared by the C-ABI (host_api.cpp) and the planners (host_plan.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.h"

struct CINTOpt;  // the library's optimizer handle (defined below as cintx::Opt)

namespace cintx {

constexpr double kPi = 3.14159265358979323846;
constexpr int ATM_SLOTS = 6, BAS_SLOTS = 8, PTR_COORD = 1;
constexpr int ATOM_OF = 0, ANG_OF = 1, NPRIM_OF = 2, NCTR_OF = 3, PTR_EXP = 5, PTR_COEFF = 6;
constexpr int PTR_EXPCUTOFF = 0, PTR_RANGE_OMEGA = 8;

void set_error(int code, const std::string& msg);
void clear_error();

// Host-phase timer of the optimizer and plan builders: with CINTX_PLAN_LOG=1 in the environment,
// mark() prints the wall time since the previous mark (or construction) to stderr.
struct PhaseLog {
  explicit PhaseLog(const char* what);
  void mark(const char* phase);
  bool on;
  const char* what;
  double t;
};

// One contracted shell of the caller's basis.
struct ShellInfo {
  int l, nprim, nctr, atom;
  int vbase;  // first virtual shell (one per contraction)
  double r[3];
  std::vector<double> exps;
  std::vector<double> coef;      // column-major [ctr][prim] as in env
  std::vector<double> log_maxc;  // log max_ctr |c| per primitive (CINTOpt_log_max_pgto_coeff)
};

struct Basis {
  int natm = 0, nbas = 0, nvirt = 0;
  std::vector<int> atm, bas;
  std::vector<double> env;
  std::vector<ShellInfo> sh;
  std::vector<int> vshell, vctr;  // virtual shell -> (shell, contraction)
};

// Validates and copies a libcint (atm, bas, env); env length is taken from the largest
// pointer used.  Returns a status code.
int load_basis(Basis& b, const int* atm, int natm, const int* bas, int nbas, const double* env);

// Exponent cut-offs of libcint: int2e uses max(40, env[0]) + 1 (g2e.c:57-62), int3c2e and
// int2c2e use max(40, env[0]) (g3c2e.c:55-59, g2c2e.c:46-50); 60 when env[0] == 0.
double expcutoff_2e(const double* env);
double expcutoff_3c(const double* env);

// Host copy of an oriented shell pair (virtual shells a >= b in angular momentum; b < 0 is
// the unit s function used for 3- and 2-centre integrals).
struct PairHost {
  int a = -1, b = -1;
  int la = 0, lb = 0;
  double min_cce = 1e300;
  ShellPair sp{};
  std::vector<PrimPair> prims;
  std::vector<int> pa, pb;  // primitive indices (within shells a and b) of each entry of prims
};

// True when real shell sx is the recurrence centre of the pair (sx, sy): the higher l, and for
// equal l the shell whose recurrence cancels least (host_api.cpp).  Every pair the kernels see is
// oriented this way: its first shell is the centre the vertical recurrence is built on.
bool pair_base_first(const Basis& B, int sx, int sy);

// Builds the screened primitive pairs of virtual shells (a, b), in that order (b < 0: unit).
// lplus raises the pair's angular momentum in libcint's screening estimate (derivative integrals
// screen with the raised ceiling li + 1, cint2e.c CINT2e_loop_nopt -> CINTset_pairdata).
void build_pair(const Basis& B, int a, int b, double expcutoff, PairHost& out, int lplus = 0);

// Device-resident state of one CINTOpt: all unordered virtual-shell pairs (u >= v) oriented by
// angular momentum (larger l first; equal l keeps the larger index first) followed by one unit
// pair per virtual shell.
struct Opt {
  uint64_t magic;
  Basis basis;
  double build_cutoff = 0;
  int device = -1;
  int npairs = 0;             // regular pairs; unit pair of v is npairs + v
  int npv = 0;                // virtual shells u < npv have their pairs (u, v <= u) stored
  std::vector<int> pair_a, pair_b, pair_la, pair_lb, pair_nprim;
  std::vector<double> pair_min_cce;
  ShellPair* d_pairs = nullptr;
  PrimPair* d_prims = nullptr;
  int64_t nprims_total = 0;
  // host copies of the primitive pairs and their primitive indices, for the primitive
  // Schwarz pass; pair_qp[pair] = sum of the pair's q (set once prim_schwarz is true)
  std::vector<PrimPair> h_prims;
  std::vector<int> h_prim_a, h_prim_b;
  std::vector<double> pair_qp;
  // pair_amp[pair] = max over its primitive pairs of (1 + |P - C| sqrt(2 a_ab))^(la + lb), C the
  // farther of the two centres: how far the pair's recurrences can cancel below their terms
  std::vector<double> pair_amp;
  bool prim_schwarz = false;
  std::mutex mu;
  static constexpr uint64_t kMagic = 0x43494e5458423230ull;  // "CINTXB20"
};

inline int pair_index(int u, int v) {  // unordered, u >= v
  return u >= v ? u * (u + 1) / 2 + v : v * (v + 1) / 2 + u;
}

Opt* as_opt(CINTOpt* o);
// Computes every stored primitive pair's Schwarz factor q (cartesian primitive diagonals on the
// device), sorts each shell pair's primitive pairs by decreasing q and re-uploads them.
int compute_prim_schwarz(Opt* o);
// npair_shells < 0: pairs of all shells; otherwise only pairs among the first npair_shells shells
// (unit pairs are built for every shell).
int build_opt(Opt* o, const int* atm, int natm, const int* bas, int nbas, const double* env, int npair_shells = -1);

// Offsets (doubles from the start of the payload) of each order's polynomial block and
// asymptotic constants in the device layout of the Rys table, and its interval counts.
struct RysTableOffsets {
  size_t poly[CINTX_NRMAX + 1];
  size_t asym[CINTX_NRMAX + 1];
  int xmax[CINTX_NRMAX + 1];
};
// The embedded table checked against the compiled layout and transposed to the device layout
// (rys_table.cu).  Returns 0 on success.
int rys_table_image(std::vector<double>& payload, RysTableOffsets& offs);

// Per-device constants (Rys table) and per-thread scratch.
struct DeviceState {
  int dev = -1;
  void* rys_buf = nullptr;
  RysTable rys{};
};
int device_state(DeviceState** out);  // for the current device

struct ThreadScratch {
  int dev = -1;
  cudaStream_t stream = nullptr;
  void* dbuf = nullptr;
  size_t dcap = 0;
  void* hbuf = nullptr;  // pinned
  size_t hcap = 0;
  int64_t launches = 0;
};
int thread_scratch(ThreadScratch** out, size_t dbytes, size_t hbytes);

// Orientation of a requested shell tuple onto a compiled kernel class.
struct Oriented {
  int li, lj, lk, ll;       // kernel class
  int src[4];               // requested axis feeding kernel axis c
  bool swap_ab;             // kernel (ij) pair is the requested second pair
};

// Algorithmic FP64 flop count of the Rys path per primitive quartet and per contracted
// quartet (c2s) for a class.
double flops_per_prim_quartet(int li, int lj, int lk, int ll);
double flops_c2s(int li, int lj, int lk, int ll, bool sph);

bool class_needs_scratch(int li, int lj, int lk, int ll, bool sph, int variant = 0);
cudaError_t launch_class(int li, int lj, int lk, int ll, bool sph, const QuartetRec* recs, int nrec,
                         const ShellPair* pairs, const PrimPair* prims, double* out, OutStrides st,
                         double expcutoff, const RysTable& rys, cudaStream_t stream, bool fp32 = false,
                         double prim_eps = 0.0, int variant = 0, const double* rootbuf = nullptr,
                         const long long* rootbase = nullptr);
// Learned Rys roots (rysnet.cu) of order n at count device points: out[p*2n + f], status[p]
// (0 refined, 1 table fallback, 2 closed form), asynchronous on stream.
cudaError_t rys_learned_eval(const float* d_params, const RysTable& rys, int n, const double* d_x, long long count,
                             double* d_out, int* d_status, int* d_iters, cudaStream_t stream);
// Lanes per quartet of a launch-shape variant (0 = default shape); variants that do not apply
// (cartesian or FP32 classes, unknown ids) report the default shape.
int variant_lanes(int li, int lj, int lk, int ll, bool sph, bool fp32, int variant);
// Distinct launch shape of a variant (lanes and register cap), for telling variants apart.
int variant_shape(int li, int lj, int lk, int ll, bool sph, bool fp32, int variant);
constexpr int kLaunchVariants = 12;

}  // namespace cintx
