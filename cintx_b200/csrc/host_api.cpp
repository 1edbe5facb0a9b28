// libcint-signature C ABI, optimizer handles, pair tables and error state.
//
// The per-call entry points (int2e_sph & co.) follow libcint's CINT2e_drv / CINT3c2e_drv /
// CINT2c2e_drv contract (cint2e.c:794-870): out == NULL returns a cache size, dims places the
// block in a larger array, the return value reports whether any primitive survived the
// exponent screening.  Each call builds the two screened shell pairs on the host, ships them
// with one quartet record to the device in a single copy, runs the class kernel and copies the
// block back.  The batched planners in host_plan.cpp are the throughput path.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cintx_cuda.h"
#include "host_internal.h"

namespace cintx {

int upload_rys_table(void** dev_buf, RysTable* tab);
cudaError_t rys_eval(const RysTable& t, int n, const double* x, long long nx, double* out,
                     cudaStream_t stream);

// ---------------------------------------------------------------- errors
struct ErrState {
  int code = 0;
  std::string msg;
};
static thread_local ErrState g_err;

void set_error(int code, const std::string& msg) {
  g_err.code = code;
  g_err.msg = msg;
}
void clear_error() {
  g_err.code = 0;
  g_err.msg.clear();
}

static double wall_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
PhaseLog::PhaseLog(const char* what_) : what(what_), t(0) {
  const char* e = getenv("CINTX_PLAN_LOG");
  on = e && e[0] && e[0] != '0';
  if (on) t = wall_ms();
}
void PhaseLog::mark(const char* phase) {
  if (!on) return;
  const double now = wall_ms();
  fprintf(stderr, "cintx %s: %s %.2f ms\n", what, phase, now - t);
  t = now;
}

// ---------------------------------------------------------------- basis
static double common_fac_sp(int l) {  // g1e.c:566
  return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
}

double expcutoff_2e(const double* env) {
  return env[PTR_EXPCUTOFF] == 0 ? 60.0 : std::max(40.0, env[PTR_EXPCUTOFF]) + 1.0;
}
double expcutoff_3c(const double* env) {
  return env[PTR_EXPCUTOFF] == 0 ? 60.0 : std::max(40.0, env[PTR_EXPCUTOFF]);
}

int load_basis(Basis& b, const int* atm, int natm, const int* bas, int nbas, const double* env) {
  if (!atm || !bas || !env) {
    set_error(CINTX_STATUS_NULL_POINTER, "atm, bas and env must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (natm <= 0 || nbas <= 0) {
    set_error(CINTX_STATUS_INVALID_INPUT, "natm and nbas must be positive");
    return CINTX_STATUS_INVALID_INPUT;
  }
  size_t env_len = 20;
  for (int a = 0; a < natm; ++a) env_len = std::max(env_len, (size_t)atm[a * ATM_SLOTS + PTR_COORD] + 3);
  for (int s = 0; s < nbas; ++s) {
    const int* r = bas + s * BAS_SLOTS;
    if (r[ATOM_OF] < 0 || r[ATOM_OF] >= natm) {
      set_error(CINTX_STATUS_INVALID_INPUT, "bas[" + std::to_string(s) + "] atom index out of range");
      return CINTX_STATUS_INVALID_INPUT;
    }
    if (r[ANG_OF] < 0 || r[ANG_OF] > CINTX_LMAX) {
      set_error(CINTX_STATUS_INVALID_INPUT,
                "shell " + std::to_string(s) + ": angular momentum " + std::to_string(r[ANG_OF]) +
                    " outside the compiled range 0.." + std::to_string(CINTX_LMAX));
      return CINTX_STATUS_INVALID_INPUT;
    }
    if (r[NPRIM_OF] < 1 || r[NPRIM_OF] > 64 || r[NCTR_OF] < 1 || r[NCTR_OF] > 64) {
      set_error(CINTX_STATUS_INVALID_INPUT, "shell " + std::to_string(s) + ": nprim/nctr outside 1..64");
      return CINTX_STATUS_INVALID_INPUT;
    }
    env_len = std::max(env_len, (size_t)r[PTR_EXP] + r[NPRIM_OF]);
    env_len = std::max(env_len, (size_t)r[PTR_COEFF] + (size_t)r[NPRIM_OF] * r[NCTR_OF]);
  }
  b.natm = natm;
  b.nbas = nbas;
  b.atm.assign(atm, atm + (size_t)natm * ATM_SLOTS);
  b.bas.assign(bas, bas + (size_t)nbas * BAS_SLOTS);
  b.env.assign(env, env + env_len);
  b.sh.resize(nbas);
  b.vshell.clear();
  b.vctr.clear();
  for (int s = 0; s < nbas; ++s) {
    const int* r = bas + s * BAS_SLOTS;
    ShellInfo& si = b.sh[s];
    si.l = r[ANG_OF];
    si.nprim = r[NPRIM_OF];
    si.nctr = r[NCTR_OF];
    si.atom = r[ATOM_OF];
    const double* c = env + atm[si.atom * ATM_SLOTS + PTR_COORD];
    si.r[0] = c[0];
    si.r[1] = c[1];
    si.r[2] = c[2];
    si.exps.assign(env + r[PTR_EXP], env + r[PTR_EXP] + si.nprim);
    si.coef.assign(env + r[PTR_COEFF], env + r[PTR_COEFF] + (size_t)si.nprim * si.nctr);
    si.log_maxc.resize(si.nprim);
    for (int p = 0; p < si.nprim; ++p) {
      double m = 0;
      for (int k = 0; k < si.nctr; ++k) m = std::max(m, fabs(si.coef[(size_t)k * si.nprim + p]));
      si.log_maxc[p] = log(m);
    }
    si.vbase = (int)b.vshell.size();
    for (int k = 0; k < si.nctr; ++k) {
      b.vshell.push_back(s);
      b.vctr.push_back(k);
    }
  }
  b.nvirt = (int)b.vshell.size();
  return CINTX_STATUS_SUCCESS;
}

// Recurrence centre of a shell pair.  The vertical recurrence is built on one centre X and the
// horizontal transfer moves angular momentum to the other, Y; the recurrence's coefficient P - X
// (P the primitive pair's product centre) is a_y/(a_x + a_y) |X - Y| long, and its powers, with
// the transfer's powers of |X - Y|, cancel down to the integral.  Building on the diffuse shell of
// a diffuse/tight pair far apart loses most of the digits: a (ff|ff) block of a 0.17 / 2253
// exponent pair 4 bohr apart is 6% off, while building on the tight shell matches 40-digit
// arithmetic to 1e-19.  libcint takes the shell of higher l and, for equal l, the second one
// (ibase = li > lj, g2e.c:101); this library takes the higher l too and, for equal l, the shell
// with the smaller cancellation measure max over primitive pairs of a_y |X - Y| / sqrt(a_x + a_y)
// (ties, e.g. one centre: the larger shell index).  Returns true when real shell sx is the
// recurrence centre of the pair (sx, sy).
bool pair_base_first(const Basis& B, int sx, int sy) {
  const ShellInfo& X = B.sh[sx];
  const ShellInfo& Y = B.sh[sy];
  if (X.l != Y.l) return X.l > Y.l;
  if (sx == sy) return true;
  const double dx = X.r[0] - Y.r[0], dy = X.r[1] - Y.r[1], dz = X.r[2] - Y.r[2];
  const double d = sqrt(dx * dx + dy * dy + dz * dz);
  double on_x = 0, on_y = 0;
  for (double ax : X.exps)
    for (double ay : Y.exps) {
      const double r = d / sqrt(ax + ay);
      on_x = std::max(on_x, ay * r);
      on_y = std::max(on_y, ax * r);
    }
  if (!(on_x != on_y) || fabs(on_x - on_y) <= 1e-12 * std::max(on_x, on_y)) return sx >= sy;
  return on_x < on_y;
}

// CINTset_pairdata semantics (optimizer.c:288-342) on virtual shells a (first) and b.
void build_pair(const Basis& B, int a, int b, double expcutoff, PairHost& out, int lplus) {
  const ShellInfo& A = B.sh[B.vshell[a]];
  const int ca = B.vctr[a];
  out.a = a;
  out.b = b;
  out.la = A.l;
  out.prims.clear();
  out.pa.clear();
  out.pb.clear();
  out.min_cce = 1e300;
  const double sq_common = sqrt(2.0 * pow(kPi, 2.5));  // sqrt of pi^3 * 2/sqrt(pi)
  ShellPair& sp = out.sp;
  sp.ax = A.r[0];
  sp.ay = A.r[1];
  sp.az = A.r[2];
  if (b < 0) {  // unit s function with exponent 0 at A
    out.lb = 0;
    sp.abx = sp.aby = sp.abz = 0;
    for (int p = 0; p < A.nprim; ++p) {
      PrimPair pp{};
      pp.aij = A.exps[p];
      pp.px = A.r[0];
      pp.py = A.r[1];
      pp.pz = A.r[2];
      pp.kab = A.coef[(size_t)ca * A.nprim + p] * sq_common * common_fac_sp(A.l);
      pp.cce = 0;
      pp.half_inv = 0.5 / A.exps[p];
      out.prims.push_back(pp);
      out.pa.push_back(p);
      out.pb.push_back(0);
      out.min_cce = 0;
    }
  } else {
    const ShellInfo& Bs = B.sh[B.vshell[b]];
    const int cb = B.vctr[b];
    out.lb = Bs.l;
    const double d[3] = {A.r[0] - Bs.r[0], A.r[1] - Bs.r[1], A.r[2] - Bs.r[2]};
    sp.abx = d[0];
    sp.aby = d[1];
    sp.abz = d[2];
    const double rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double log_rr = 1.7 - 1.5 * log(A.exps[A.nprim - 1] + Bs.exps[Bs.nprim - 1]);
    const int lij = A.l + Bs.l + lplus;
    if (lij > 0) log_rr += lij * log(sqrt(rr) + 1.0);
    const double fac = sq_common * common_fac_sp(A.l) * common_fac_sp(Bs.l);
    for (int q = 0; q < Bs.nprim; ++q) {
      for (int p = 0; p < A.nprim; ++p) {
        const double ai = A.exps[p], aj = Bs.exps[q];
        const double inv = 1.0 / (ai + aj);
        const double eij = rr * ai * aj * inv;
        const double cce = eij - log_rr - A.log_maxc[p] - Bs.log_maxc[q];
        if (!(cce < expcutoff)) continue;
        const double cprod = A.coef[(size_t)ca * A.nprim + p] * Bs.coef[(size_t)cb * Bs.nprim + q];
        if (cprod == 0.0) continue;  // zero contraction coefficient contributes nothing
        PrimPair pp{};
        pp.aij = ai + aj;
        const double wj = aj * inv;
        pp.px = A.r[0] - wj * d[0];
        pp.py = A.r[1] - wj * d[1];
        pp.pz = A.r[2] - wj * d[2];
        pp.kab = exp(-eij) * cprod * fac;
        pp.cce = cce;
        pp.half_inv = 0.5 * inv;
        out.prims.push_back(pp);
        out.pa.push_back(p);
        out.pb.push_back(q);
        out.min_cce = std::min(out.min_cce, cce);
      }
    }
  }
  sp.nprim = (int)out.prims.size();
  sp.prim_off = 0;
  sp.ish = a;
  sp.jsh = b;
}

// ---------------------------------------------------------------- device / thread state
static std::mutex g_dev_mu;
static DeviceState g_devs[64];

int device_state(DeviceState** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "no usable CUDA device");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceState& d = g_devs[dev];
  if (d.dev != dev) {
    int rc = upload_rys_table(&d.rys_buf, &d.rys);
    if (rc != 0) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "Rys table upload failed (" + std::to_string(rc) + ")");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
    d.dev = dev;
  }
  *out = &d;
  return CINTX_STATUS_SUCCESS;
}

static thread_local ThreadScratch g_ts;

int thread_scratch(ThreadScratch** out, size_t dbytes, size_t hbytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  ThreadScratch& t = g_ts;
  if (t.dev != dev) {
    // a thread that switches devices gets fresh buffers on the new device
    t = ThreadScratch();
    t.dev = dev;
    if (cudaStreamCreateWithFlags(&t.stream, cudaStreamNonBlocking) != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaStreamCreate failed");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
  }
  if (dbytes > t.dcap) {
    if (t.dbuf) cudaFree(t.dbuf);
    size_t cap = std::max(dbytes, (size_t)1 << 20);
    if (cudaMalloc(&t.dbuf, cap) != cudaSuccess) {
      t.dbuf = nullptr;
      t.dcap = 0;
      set_error(CINTX_STATUS_ALLOCATION_FAILED, "device scratch allocation failed");
      return CINTX_STATUS_ALLOCATION_FAILED;
    }
    t.dcap = cap;
  }
  if (hbytes > t.hcap) {
    if (t.hbuf) cudaFreeHost(t.hbuf);
    size_t cap = std::max(hbytes, (size_t)1 << 20);
    if (cudaMallocHost(&t.hbuf, cap) != cudaSuccess) {
      t.hbuf = nullptr;
      t.hcap = 0;
      set_error(CINTX_STATUS_ALLOCATION_FAILED, "pinned host scratch allocation failed");
      return CINTX_STATUS_ALLOCATION_FAILED;
    }
    t.hcap = cap;
  }
  *out = &t;
  return CINTX_STATUS_SUCCESS;
}

// Transform scratch of the large classes: one growing buffer per host thread and device.
static thread_local int g_cs_dev = -1;
static thread_local double* g_cs_buf = nullptr;
static thread_local size_t g_cs_cap = 0;

double* class_scratch(size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_cs_dev != dev) {
    g_cs_dev = dev;
    g_cs_buf = nullptr;  // a buffer on another device stays with that device's context
    g_cs_cap = 0;
  }
  if (bytes > g_cs_cap) {
    if (g_cs_buf) cudaFree(g_cs_buf);
    g_cs_buf = nullptr;
    g_cs_cap = 0;
    if (cudaMalloc(&g_cs_buf, bytes) != cudaSuccess) return nullptr;
    g_cs_cap = bytes;
  }
  return g_cs_buf;
}

// ---------------------------------------------------------------- flop model
static int ncart_h(int l) { return (l + 1) * (l + 2) / 2; }

double flops_per_prim_quartet(int li, int lj, int lk, int ll) {
  const int n = (li + lj + lk + ll) / 2 + 1;
  const int nij = li + lj + 1, nkl = lk + ll + 1;
  const double vrr = 3.0 * n * 5.0 * nij * nkl;
  double hrr_assign = 0;
  for (int j = 1; j <= lj; ++j) hrr_assign += (double)(nij - j) * nkl;
  for (int l = 1; l <= ll; ++l) hrr_assign += (double)(li + 1) * (lj + 1) * (nkl - l);
  const double hrr = 3.0 * n * 2.0 * hrr_assign;
  const double gout = (double)ncart_h(li) * ncart_h(lj) * ncart_h(lk) * ncart_h(ll) * 3.0 * n;
  return vrr + hrr + gout;
}

double flops_c2s(int li, int lj, int lk, int ll, bool sph) {
  if (!sph) return 0;
  int dims[4] = {ncart_h(li), ncart_h(lj), ncart_h(lk), ncart_h(ll)};
  const int ls[4] = {li, lj, lk, ll};
  double f = 0;
  for (int a = 0; a < 4; ++a) {
    if (ls[a] < 2) continue;
    double rest = 1;
    for (int b = 0; b < 4; ++b)
      if (b != a) rest *= dims[b];
    f += 2.0 * dims[a] * (2 * ls[a] + 1) * rest;
    dims[a] = 2 * ls[a] + 1;
  }
  return f;
}

// ---------------------------------------------------------------- optimizer
Opt* as_opt(CINTOpt* o) {
  Opt* p = reinterpret_cast<Opt*>(o);
  if (p && p->magic != Opt::kMagic) return nullptr;
  return p;
}

static void free_opt_device(Opt* o) {
  if (o->d_pairs) cudaFree(o->d_pairs);
  if (o->d_prims) cudaFree(o->d_prims);
  o->d_pairs = nullptr;
  o->d_prims = nullptr;
}

int build_opt(Opt* o, const int* atm, int natm, const int* bas, int nbas, const double* env, int npair_shells) {
  PhaseLog plog("optimizer");
  int rc = load_basis(o->basis, atm, natm, bas, nbas, env);
  if (rc) return rc;
  if (npair_shells > nbas) {
    set_error(CINTX_STATUS_INVALID_INPUT, "npair_shells exceeds nbas");
    return CINTX_STATUS_INVALID_INPUT;
  }
  DeviceState* ds;
  if ((rc = device_state(&ds))) return rc;
  const Basis& B = o->basis;
  o->build_cutoff = expcutoff_2e(B.env.data());
  const int nv = B.nvirt;
  const int npv = npair_shells < 0 || npair_shells == B.nbas ? nv : B.sh[npair_shells].vbase;
  o->npv = npv;
  o->npairs = npv * (npv + 1) / 2;
  const int ntot = o->npairs + nv;
  std::vector<ShellPair> sps(ntot);
  std::vector<PrimPair> prims;
  o->pair_a.assign(ntot, 0);
  o->pair_b.assign(ntot, 0);
  o->pair_la.assign(ntot, 0);
  o->pair_lb.assign(ntot, 0);
  o->pair_nprim.assign(ntot, 0);
  o->pair_min_cce.assign(ntot, 0);
  o->h_prim_a.clear();
  o->h_prim_b.clear();
  // Pairs of rows u in [u0, u1) have the contiguous ids [pair_index(u0, 0), pair_index(u1, 0)), so
  // host threads fill row ranges of about equal pair counts, each into its own primitive lists,
  // which are then joined in row order (the order of one serial pass).
  {
    const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int nt = npv >= 64 ? nthr : 1;
    std::vector<int> ubound(nt + 1, npv);
    ubound[0] = 0;
    for (int t = 1; t < nt; ++t) {
      const double target = (double)o->npairs * t / nt;  // rows below u hold u(u+1)/2 pairs
      ubound[t] = std::max(ubound[t - 1], std::min(npv, (int)ceil((sqrt(8.0 * target + 1.0) - 1.0) / 2.0)));
    }
    struct Part {
      std::vector<PrimPair> prims;
      std::vector<int> pa, pb;
    };
    std::vector<Part> parts(nt);
    auto work = [&](int t) {
      PairHost ph;
      Part& P = parts[t];
      for (int u = ubound[t]; u < ubound[t + 1]; ++u) {
        for (int v = 0; v <= u; ++v) {
          // recurrence centre first (pair_base_first; contractions of one shell: larger index first)
          const bool uf = pair_base_first(B, B.vshell[u], B.vshell[v]);
          const int a = uf ? u : v, b = uf ? v : u;
          build_pair(B, a, b, o->build_cutoff, ph);
          const int id = pair_index(u, v);
          ph.sp.prim_off = (int)P.prims.size();  // part-relative; shifted below
          sps[id] = ph.sp;
          P.prims.insert(P.prims.end(), ph.prims.begin(), ph.prims.end());
          P.pa.insert(P.pa.end(), ph.pa.begin(), ph.pa.end());
          P.pb.insert(P.pb.end(), ph.pb.begin(), ph.pb.end());
          o->pair_a[id] = a;
          o->pair_b[id] = b;
          o->pair_la[id] = ph.la;
          o->pair_lb[id] = ph.lb;
          o->pair_nprim[id] = ph.sp.nprim;
          o->pair_min_cce[id] = ph.min_cce;
        }
      }
    };
    if (nt == 1) {
      work(0);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < nt; ++t) th.emplace_back(work, t);
      for (auto& x : th) x.join();
    }
    long long base = 0;
    for (int t = 0; t < nt; ++t) {
      const int id0 = pair_index(ubound[t], 0);
      const int id1 = ubound[t + 1] >= npv ? o->npairs : pair_index(ubound[t + 1], 0);
      for (int id = id0; id < id1; ++id) sps[id].prim_off += (int)base;
      base += (long long)parts[t].prims.size();
      prims.insert(prims.end(), parts[t].prims.begin(), parts[t].prims.end());
      o->h_prim_a.insert(o->h_prim_a.end(), parts[t].pa.begin(), parts[t].pa.end());
      o->h_prim_b.insert(o->h_prim_b.end(), parts[t].pb.begin(), parts[t].pb.end());
    }
  }
  PairHost ph;
  for (int v = 0; v < nv; ++v) {
    build_pair(B, v, -1, o->build_cutoff, ph);
    const int id = o->npairs + v;
    ph.sp.prim_off = (int)prims.size();
    sps[id] = ph.sp;
    prims.insert(prims.end(), ph.prims.begin(), ph.prims.end());
    o->h_prim_a.insert(o->h_prim_a.end(), ph.pa.begin(), ph.pa.end());
    o->h_prim_b.insert(o->h_prim_b.end(), ph.pb.begin(), ph.pb.end());
    o->pair_a[id] = v;
    o->pair_b[id] = -1;
    o->pair_la[id] = ph.la;
    o->pair_lb[id] = 0;
    o->pair_nprim[id] = ph.sp.nprim;
    o->pair_min_cce[id] = ph.min_cce;
  }
  plog.mark("basis + pair tables (host)");
  if ((int64_t)prims.size() > 2000000000LL) {
    set_error(CINTX_STATUS_MEMORY_LIMIT_EXCEEDED, "too many primitive pairs");
    return CINTX_STATUS_MEMORY_LIMIT_EXCEEDED;
  }
  o->nprims_total = (int64_t)prims.size();
  o->h_prims = prims;
  o->prim_schwarz = false;
  free_opt_device(o);
  cudaGetDevice(&o->device);
  if (cudaMalloc(&o->d_pairs, sizeof(ShellPair) * sps.size()) != cudaSuccess ||
      cudaMalloc(&o->d_prims, sizeof(PrimPair) * std::max<size_t>(prims.size(), 1)) != cudaSuccess) {
    free_opt_device(o);
    set_error(CINTX_STATUS_ALLOCATION_FAILED, "device allocation of pair tables failed");
    return CINTX_STATUS_ALLOCATION_FAILED;
  }
  cudaMemcpy(o->d_pairs, sps.data(), sizeof(ShellPair) * sps.size(), cudaMemcpyHostToDevice);
  if (!prims.empty())
    cudaMemcpy(o->d_prims, prims.data(), sizeof(PrimPair) * prims.size(), cudaMemcpyHostToDevice);
  if (cudaGetLastError() != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "upload of pair tables failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  plog.mark("upload");
  return CINTX_STATUS_SUCCESS;
}

static void make_optimizer(CINTOpt** opt, const int* atm, int natm, const int* bas, int nbas, const double* env,
                           int npair_shells = -1) {
  if (!opt) return;
  *opt = nullptr;
  clear_error();
  Opt* o = new Opt();
  o->magic = Opt::kMagic;
  if (build_opt(o, atm, natm, bas, nbas, env, npair_shells) != CINTX_STATUS_SUCCESS) {
    free_opt_device(o);
    o->magic = 0;
    delete o;
    return;
  }
  *opt = reinterpret_cast<CINTOpt*>(o);
}

// ---------------------------------------------------------------- orientation
// Requested axes 0..3 with angular momenta l[4] (unit axes have l = 0) of the real shells
// idx0..idx3.  Chooses the kernel class and which requested axis feeds each kernel axis.
static Oriented orient(const Basis& B, const int l[4], bool unit_b1, bool unit_b3, int idx0, int idx1, int idx2,
                       int idx3) {
  Oriented o;
  // pair 1 = axes (0,1), pair 2 = axes (2,3); the recurrence centre of each pair first
  auto pair_first = [&](int ia, int ib, bool unit_b) { return unit_b || pair_base_first(B, ia, ib); };
  const bool f1 = pair_first(idx0, idx1, unit_b1);
  const bool f2 = pair_first(idx2, idx3, unit_b3);
  int p1[2] = {f1 ? 0 : 1, f1 ? 1 : 0};
  int p2[2] = {f2 ? 2 : 3, f2 ? 3 : 2};
  const int l1a = l[p1[0]], l1b = l[p1[1]], l2a = l[p2[0]], l2b = l[p2[1]];
  const bool swap = (l2a > l1a) || (l2a == l1a && l2b > l1b);
  o.swap_ab = swap;
  if (!swap) {
    o.src[0] = p1[0]; o.src[1] = p1[1]; o.src[2] = p2[0]; o.src[3] = p2[1];
  } else {
    o.src[0] = p2[0]; o.src[1] = p2[1]; o.src[2] = p1[0]; o.src[3] = p1[1];
  }
  o.li = l[o.src[0]];
  o.lj = l[o.src[1]];
  o.lk = l[o.src[2]];
  o.ll = l[o.src[3]];
  return o;
}

// ---------------------------------------------------------------- per-call evaluation
enum Family { F2E = 0, F3C = 1, F2C = 2 };

static int cache_size_query(int family, const Basis* B, const int* shls, bool sph, const int* bas) {
  // A size that satisfies callers that size `cache` from the out == NULL query; the device
  // path does not use the cache.  Uses libcint's second term nc*ncomp + nf*4 (cint2e.c:805).
  int nsh = family == F2E ? 4 : (family == F3C ? 3 : 2);
  long long nf = 1, nc = 1;
  for (int a = 0; a < nsh; ++a) {
    const int* r = bas + shls[a] * BAS_SLOTS;
    int l = r[ANG_OF];
    nf *= (l + 1) * (l + 2) / 2;
    nc *= r[NCTR_OF];
  }
  (void)B;
  (void)sph;
  long long n = nf * nc + nf * 4;
  return (int)std::min<long long>(n, 0x7fffffff);
}

static int eval_call(int family, bool sph, double* out, int* dims, int* shls, int* atm, int natm, int* bas,
                     int nbas, double* env, CINTOpt* optp) {
  clear_error();
  const int nsh = family == F2E ? 4 : (family == F3C ? 3 : 2);
  if (!shls || !atm || !bas || !env) {
    set_error(CINTX_STATUS_NULL_POINTER, "shls, atm, bas and env must not be NULL");
    return 0;
  }
  for (int a = 0; a < nsh; ++a) {
    if (shls[a] < 0 || shls[a] >= nbas) {
      set_error(CINTX_STATUS_INVALID_INPUT, "shell index out of range");
      return 0;
    }
  }
  if (!out) return cache_size_query(family, nullptr, shls, sph, bas);
  if (env[PTR_RANGE_OMEGA] != 0.0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "range-separated Coulomb (env[PTR_RANGE_OMEGA] != 0) is not supported");
    return 0;
  }
  // Basis view: the optimizer's copy when given, else a transient copy of the used shells.
  Opt* o = optp ? as_opt(optp) : nullptr;
  if (optp && !o) {
    set_error(CINTX_STATUS_INVALID_INPUT, "opt is not a handle created by this library");
    return 0;
  }
  Basis local;
  const Basis* B;
  if (o) {
    B = &o->basis;
  } else {
    if (load_basis(local, atm, natm, bas, nbas, env)) return 0;
    B = &local;
  }
  const double cutoff = family == F2E ? expcutoff_2e(env) : expcutoff_3c(env);

  // requested axes: shells and unit placeholders
  int rs[4], rl[4];
  bool unit[4] = {false, false, false, false};
  if (family == F2E) {
    for (int a = 0; a < 4; ++a) rs[a] = shls[a];
  } else if (family == F3C) {
    rs[0] = shls[0]; rs[1] = shls[1]; rs[2] = shls[2]; rs[3] = -1; unit[3] = true;
  } else {
    rs[0] = shls[0]; rs[1] = -1; rs[2] = shls[1]; rs[3] = -1; unit[1] = unit[3] = true;
  }
  int next[4], nctr[4];
  for (int a = 0; a < 4; ++a) {
    if (unit[a]) {
      rl[a] = 0;
      next[a] = 1;
      nctr[a] = 1;
    } else {
      const ShellInfo& s = B->sh[rs[a]];
      rl[a] = s.l;
      nctr[a] = s.nctr;
      next[a] = (sph ? 2 * s.l + 1 : (s.l + 1) * (s.l + 2) / 2);
    }
  }
  // output dims of the requested block (libcint counts) and strides
  int counts[4];
  for (int a = 0; a < 4; ++a) counts[a] = next[a] * nctr[a];
  int cdims[4];
  int nd = 0;
  for (int a = 0; a < 4; ++a)
    if (!unit[a]) cdims[nd++] = counts[a];
  int udims[4];
  for (int a = 0; a < nd; ++a) {
    udims[a] = dims ? dims[a] : cdims[a];
    if (udims[a] < cdims[a]) {
      set_error(CINTX_STATUS_BUFFER_TOO_SMALL, "dims smaller than the block extents");
      return 0;
    }
  }
  long long ustride[4];
  {
    long long s = 1;
    for (int a = 0; a < nd; ++a) {
      ustride[a] = s;
      s *= udims[a];
    }
  }
  long long axstride[4];
  {
    int k = 0;
    for (int a = 0; a < 4; ++a) axstride[a] = unit[a] ? 0 : ustride[k++];
  }
  long long block = 1;
  for (int a = 0; a < 4; ++a) block *= counts[a];

  // empty check (screening) and host pair construction per contraction tuple
  const Oriented ori = orient(*B, rl, unit[1], unit[3], rs[0], rs[1], rs[2], rs[3]);
  int rc;
  DeviceState* ds;
  if ((rc = device_state(&ds))) return 0;

  std::vector<PairHost> pairs;
  std::vector<QuartetRec> recs;
  std::vector<PrimPair> allprims;
  bool any = false;
  // enumerate contraction tuples
  int nc0 = nctr[0], nc1 = nctr[1], nc2 = nctr[2], nc3 = nctr[3];
  for (int c3 = 0; c3 < nc3; ++c3)
    for (int c2 = 0; c2 < nc2; ++c2)
      for (int c1 = 0; c1 < nc1; ++c1)
        for (int c0 = 0; c0 < nc0; ++c0) {
          const int cs[4] = {c0, c1, c2, c3};
          int vs[4];
          for (int a = 0; a < 4; ++a) vs[a] = unit[a] ? -1 : B->sh[rs[a]].vbase + cs[a];
          PairHost p1, p2;
          build_pair(*B, vs[ori.src[0]], vs[ori.src[1]], cutoff, p1);
          build_pair(*B, vs[ori.src[2]], vs[ori.src[3]], cutoff, p2);
          const bool pe = p1.prims.empty() || p2.prims.empty() || (p1.min_cce + p2.min_cce > cutoff);
          if (!pe) any = true;
          QuartetRec q;
          q.pij = (int)pairs.size();
          p1.sp.prim_off = (int)allprims.size();
          allprims.insert(allprims.end(), p1.prims.begin(), p1.prims.end());
          pairs.push_back(p1);
          q.pkl = (int)pairs.size();
          p2.sp.prim_off = (int)allprims.size();
          allprims.insert(allprims.end(), p2.prims.begin(), p2.prims.end());
          pairs.push_back(p2);
          long long off = 0;
          for (int a = 0; a < 4; ++a) off += (long long)cs[a] * next[a] * axstride[a];
          q.out = off;
          recs.push_back(q);
        }
  // dims region: libcint writes only the counts region of out (c2s_dset0 for empty blocks)
  long long full = 1;
  for (int a = 0; a < nd; ++a) full *= udims[a];
  if (!any) {
    // zero the counts region
    std::vector<long long> idx(1, 0);
    for (long long e = 0; e < block; ++e) {
      long long r = e, off = 0;
      for (int a = 0; a < 4; ++a) {
        off += (r % counts[a]) * axstride[a];
        r /= counts[a];
      }
      out[off] = 0.0;
    }
    return 0;
  }
  // device buffer layout: [ShellPair * np][PrimPair * nprim][QuartetRec * nq][out full]
  std::vector<ShellPair> sps(pairs.size());
  for (size_t i = 0; i < pairs.size(); ++i) sps[i] = pairs[i].sp;
  size_t off_pairs = 0;
  size_t off_prims = off_pairs + ((sizeof(ShellPair) * sps.size() + 255) & ~(size_t)255);
  size_t off_recs = off_prims + ((sizeof(PrimPair) * std::max<size_t>(allprims.size(), 1) + 255) & ~(size_t)255);
  size_t off_out = off_recs + ((sizeof(QuartetRec) * recs.size() + 255) & ~(size_t)255);
  size_t total = off_out + sizeof(double) * full;
  ThreadScratch* ts;
  if ((rc = thread_scratch(&ts, total, total))) return 0;
  char* h = (char*)ts->hbuf;
  memcpy(h + off_pairs, sps.data(), sizeof(ShellPair) * sps.size());
  if (!allprims.empty()) memcpy(h + off_prims, allprims.data(), sizeof(PrimPair) * allprims.size());
  memcpy(h + off_recs, recs.data(), sizeof(QuartetRec) * recs.size());
  char* d = (char*)ts->dbuf;
  cudaMemcpyAsync(d, h, off_out, cudaMemcpyHostToDevice, ts->stream);
  if (dims) cudaMemsetAsync(d + off_out, 0, sizeof(double) * full, ts->stream);
  OutStrides st;
  long long* sv[4] = {&st.s0, &st.s1, &st.s2, &st.s3};
  for (int c = 0; c < 4; ++c) *sv[c] = axstride[ori.src[c]];
  cudaError_t e = launch_class(ori.li, ori.lj, ori.lk, ori.ll, sph, (const QuartetRec*)(d + off_recs), (int)recs.size(),
                               (const ShellPair*)(d + off_pairs), (const PrimPair*)(d + off_prims),
                               (double*)(d + off_out), st, cutoff, ds->rys, ts->stream);
  if (e != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return 0;
  }
  ts->launches++;
  double* hout = (double*)(h + off_out);
  cudaMemcpyAsync(hout, d + off_out, sizeof(double) * full, cudaMemcpyDeviceToHost, ts->stream);
  e = cudaStreamSynchronize(ts->stream);
  if (e != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("device execution failed: ") + cudaGetErrorString(e));
    return 0;
  }
  if (!dims) {
    memcpy(out, hout, sizeof(double) * full);
  } else {
    for (long long el = 0; el < block; ++el) {
      long long r = el, off = 0;
      for (int a = 0; a < 4; ++a) {
        off += (r % counts[a]) * axstride[a];
        r /= counts[a];
      }
      out[off] = hout[off];
    }
  }
  return 1;
}

}  // namespace cintx

using namespace cintx;

extern "C" {

// Basis bookkeeping of libcint (cint_bas.c:36-155): functions per shell and AO offsets.  As in
// libcint, the offset routines write ao_loc[0..nbas-1] only (the total comes from CINTtot_*).
int CINTcgto_cart(const int bas_id, const int* bas) {
  const int l = bas[bas_id * BAS_SLOTS + ANG_OF];
  return (l + 1) * (l + 2) / 2 * bas[bas_id * BAS_SLOTS + NCTR_OF];
}
int CINTcgto_spheric(const int bas_id, const int* bas) {
  return (2 * bas[bas_id * BAS_SLOTS + ANG_OF] + 1) * bas[bas_id * BAS_SLOTS + NCTR_OF];
}
int CINTtot_cgto_spheric(const int* bas, const int nbas) {
  int n = 0;
  for (int i = 0; i < nbas; ++i) n += CINTcgto_spheric(i, bas);
  return n;
}
int CINTtot_cgto_cart(const int* bas, const int nbas) {
  int n = 0;
  for (int i = 0; i < nbas; ++i) n += CINTcgto_cart(i, bas);
  return n;
}
void CINTshells_spheric_offset(int ao_loc[], const int* bas, const int nbas) {
  if (nbas <= 0) return;
  ao_loc[0] = 0;
  for (int i = 1; i < nbas; ++i) ao_loc[i] = ao_loc[i - 1] + CINTcgto_spheric(i - 1, bas);
}
void CINTshells_cart_offset(int ao_loc[], const int* bas, const int nbas) {
  if (nbas <= 0) return;
  ao_loc[0] = 0;
  for (int i = 1; i < nbas; ++i) ao_loc[i] = ao_loc[i - 1] + CINTcgto_cart(i - 1, bas);
}

int int2e_sph(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
              CINTOpt* opt, double* cache) {
  (void)cache;
  return eval_call(F2E, true, out, dims, shls, atm, natm, bas, nbas, env, opt);
}
int int2e_cart(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
               CINTOpt* opt, double* cache) {
  (void)cache;
  return eval_call(F2E, false, out, dims, shls, atm, natm, bas, nbas, env, opt);
}
int int3c2e_sph(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                CINTOpt* opt, double* cache) {
  (void)cache;
  return eval_call(F3C, true, out, dims, shls, atm, natm, bas, nbas, env, opt);
}
int int3c2e_cart(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                 CINTOpt* opt, double* cache) {
  (void)cache;
  return eval_call(F3C, false, out, dims, shls, atm, natm, bas, nbas, env, opt);
}
int int2c2e_sph(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                CINTOpt* opt, double* cache) {
  (void)cache;
  return eval_call(F2C, true, out, dims, shls, atm, natm, bas, nbas, env, opt);
}
int int2c2e_cart(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                 CINTOpt* opt, double* cache) {
  (void)cache;
  return eval_call(F2C, false, out, dims, shls, atm, natm, bas, nbas, env, opt);
}

// cintx-capi's id-dispatch surface (crates/cintx-capi/src/shim.rs:312-453) for the Coulomb ids this
// library computes: 9 int2e_cart, 10 int2e_sph, 12 int2c2e_cart, 13 int2c2e_sph, and the first
// derivatives 18 int3c2e_ip1_cart, 19 int3c2e_ip1_sph, 35 int2e_ip1_cart, 36 int2e_ip1_sph.
enum { F2E_IP1 = 10, F3C_IP1 = 11 };
static int dispatch_prepare(int api, const int* dims, size_t dims_len, const int* shls, size_t shls_len,
                            const int* atm, size_t atm_len, const int* bas, size_t bas_len, const double* env,
                            size_t env_len, int* family, bool* sph, long long* nout) {
  switch (api) {
    case 9: *family = F2E; *sph = false; break;
    case 10: *family = F2E; *sph = true; break;
    case 12: *family = F2C; *sph = false; break;
    case 13: *family = F2C; *sph = true; break;
    case 18: *family = F3C_IP1; *sph = false; break;
    case 19: *family = F3C_IP1; *sph = true; break;
    case 35: *family = F2E_IP1; *sph = false; break;
    case 36: *family = F2E_IP1; *sph = true; break;
    default:
      set_error(CINTX_STATUS_UNSUPPORTED_API, "api id " + std::to_string(api) +
                                                  " is not a Coulomb integral this library computes "
                                                  "(9, 10, 12, 13, 18, 19, 35, 36)");
      return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (!shls || !atm || !bas || !env) {
    set_error(CINTX_STATUS_NULL_POINTER, "shls, atm, bas and env must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  const int nsh = *family == F2E || *family == F2E_IP1 ? 4 : (*family == F3C_IP1 ? 3 : 2);
  const long long natm = (long long)(atm_len / ATM_SLOTS), nbas = (long long)(bas_len / BAS_SLOTS);
  if ((long long)shls_len < nsh || natm < 1 || nbas < 1) {
    set_error(CINTX_STATUS_INVALID_INPUT, "shls, atm or bas is too short");
    return CINTX_STATUS_INVALID_INPUT;
  }
  // every env slot the basis references must lie inside env_len
  for (long long a = 0; a < natm; ++a)
    if (atm[a * ATM_SLOTS + PTR_COORD] < 0 || (size_t)atm[a * ATM_SLOTS + PTR_COORD] + 3 > env_len) {
      set_error(CINTX_STATUS_INVALID_INPUT, "atm coordinates point outside env");
      return CINTX_STATUS_INVALID_INPUT;
    }
  for (long long b = 0; b < nbas; ++b) {
    const int* r = bas + b * BAS_SLOTS;
    if (r[NPRIM_OF] < 1 || r[NCTR_OF] < 1 || r[PTR_EXP] < 0 || r[PTR_COEFF] < 0 ||
        (size_t)r[PTR_EXP] + r[NPRIM_OF] > env_len || (size_t)r[PTR_COEFF] + (size_t)r[NPRIM_OF] * r[NCTR_OF] > env_len ||
        r[ATOM_OF] < 0 || r[ATOM_OF] >= natm) {
      set_error(CINTX_STATUS_INVALID_INPUT, "bas row " + std::to_string(b) + " points outside env or atm");
      return CINTX_STATUS_INVALID_INPUT;
    }
  }
  long long n = 1;
  std::vector<int> ext;
  for (int a = 0; a < nsh; ++a) {
    const int sh = shls[a];
    if (sh < 0 || sh >= nbas) {
      set_error(CINTX_STATUS_INVALID_INPUT, "shell index out of range");
      return CINTX_STATUS_INVALID_INPUT;
    }
    const int l = bas[sh * BAS_SLOTS + ANG_OF], nc = bas[sh * BAS_SLOTS + NCTR_OF];
    const int e = (*sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2) * nc;
    ext.push_back(e);
    n *= e;
  }
  // cintx-compat accepts dims only equal to the natural extents (compat/src/layout.rs:25-62)
  if (dims) {
    bool same = dims_len == (size_t)nsh;
    for (int a = 0; same && a < nsh; ++a) same = dims[a] == ext[a];
    if (!same) {
      set_error(CINTX_STATUS_INVALID_INPUT, "dims must equal the natural extents of the block");
      return CINTX_STATUS_INVALID_INPUT;
    }
  }
  *nout = n * (*family == F2E_IP1 || *family == F3C_IP1 ? 3 : 1);  // derivatives: 3 components
  return CINTX_STATUS_SUCCESS;
}

int cintrs_query_workspace(int api, const int* dims, size_t dims_len, const int* shls, size_t shls_len, const int* atm,
                           size_t atm_len, const int* bas, size_t bas_len, const double* env, size_t env_len,
                           const CINTOpt* opt, CintxWorkspaceQuery* query_out) {
  clear_error();
  (void)opt;
  if (!query_out) {
    set_error(CINTX_STATUS_NULL_POINTER, "query_out must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  int family;
  bool sph;
  long long nout;
  int rc = dispatch_prepare(api, dims, dims_len, shls, shls_len, atm, atm_len, bas, bas_len, env, env_len, &family,
                            &sph, &nout);
  if (rc) return rc;
  query_out->bytes = 0;  // device working memory is held by the library, not the caller's cache
  query_out->alignment = 8;
  query_out->required_bytes = (size_t)nout * sizeof(double);
  query_out->chunk_count = 1;
  query_out->work_units = 1;
  return CINTX_STATUS_SUCCESS;
}

int cintrs_eval(int api, double* out, size_t out_len, const int* dims, size_t dims_len, const int* shls,
                size_t shls_len, const int* atm, size_t atm_len, const int* bas, size_t bas_len, const double* env,
                size_t env_len, const CINTOpt* opt, double* cache, size_t cache_len, CintxEvalSummary* summary_out) {
  clear_error();
  if (!summary_out) {
    set_error(CINTX_STATUS_NULL_POINTER, "summary_out must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  if ((!out && out_len > 0) || (!cache && cache_len > 0)) {
    set_error(CINTX_STATUS_NULL_POINTER, "out or cache is NULL with a nonzero length");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (out && cache && out == cache) {
    set_error(CINTX_STATUS_INVALID_INPUT, "`out` and `cache` pointers must not alias");
    return CINTX_STATUS_INVALID_INPUT;
  }
  int family;
  bool sph;
  long long nout;
  int rc = dispatch_prepare(api, dims, dims_len, shls, shls_len, atm, atm_len, bas, bas_len, env, env_len, &family,
                            &sph, &nout);
  if (rc) return rc;
  summary_out->not0 = 0;
  summary_out->bytes_written = 0;
  summary_out->workspace_bytes = 0;
  if (!out) return CINTX_STATUS_SUCCESS;  // a workspace-only call
  if ((long long)out_len < nout) {
    set_error(CINTX_STATUS_BUFFER_TOO_SMALL, "out holds " + std::to_string(out_len) + " doubles, the block needs " +
                                                  std::to_string(nout));
    return CINTX_STATUS_BUFFER_TOO_SMALL;
  }
  const int natm = (int)(atm_len / ATM_SLOTS), nbas = (int)(bas_len / BAS_SLOTS);
  int* sh = const_cast<int*>(shls);
  int* at = const_cast<int*>(atm);
  int* ba = const_cast<int*>(bas);
  double* en = const_cast<double*>(env);
  int r;
  if (family == F2E_IP1) {
    r = (sph ? int2e_ip1_sph : int2e_ip1_cart)(out, nullptr, sh, at, natm, ba, nbas, en, nullptr, nullptr);
  } else if (family == F3C_IP1) {
    r = (sph ? int3c2e_ip1_sph : int3c2e_ip1_cart)(out, nullptr, sh, at, natm, ba, nbas, en, nullptr, nullptr);
  } else {
    r = eval_call(family, sph, out, nullptr, sh, at, natm, ba, nbas, en, const_cast<CINTOpt*>(opt));
  }
  if (g_err.code) return g_err.code;
  summary_out->not0 = r;
  summary_out->bytes_written = (size_t)nout * sizeof(double);
  return CINTX_STATUS_SUCCESS;
}

void int2e_optimizer(CINTOpt** opt, int* atm, int natm, int* bas, int nbas, double* env) {
  make_optimizer(opt, atm, natm, bas, nbas, env);
}
void int3c2e_optimizer(CINTOpt** opt, int* atm, int natm, int* bas, int nbas, double* env) {
  make_optimizer(opt, atm, natm, bas, nbas, env);
}
void int2c2e_optimizer(CINTOpt** opt, int* atm, int natm, int* bas, int nbas, double* env) {
  make_optimizer(opt, atm, natm, bas, nbas, env);
}
int cintx_optimizer_pair_shells(CINTOpt** opt, const int* atm, int natm, const int* bas, int nbas, const double* env,
                                int npair_shells) {
  if (!opt || npair_shells < 1 || npair_shells > nbas) {
    set_error(CINTX_STATUS_INVALID_INPUT, "cintx_optimizer_pair_shells: bad arguments");
    return CINTX_STATUS_INVALID_INPUT;
  }
  make_optimizer(opt, atm, natm, bas, nbas, env, npair_shells);
  return *opt ? CINTX_STATUS_SUCCESS : cintx_cuda_last_error_code();
}

void CINTdel_optimizer(CINTOpt** opt) {
  if (!opt || !*opt) return;
  Opt* o = as_opt(*opt);
  if (o) {
    free_opt_device(o);
    o->magic = 0;
    delete o;
  }
  *opt = nullptr;
}

int CINTrys_roots(int nroots, double x, double* u, double* w) {
  clear_error();
  if (nroots < 1 || nroots > CINTX_NRMAX || !u || !w || !(x >= 0)) {
    set_error(CINTX_STATUS_INVALID_INPUT, "CINTrys_roots: nroots must be 1..9, x >= 0");
    return 1;
  }
  DeviceState* ds;
  if (device_state(&ds)) return 1;
  ThreadScratch* ts;
  const size_t nbytes = sizeof(double) * (1 + 2 * nroots);
  if (thread_scratch(&ts, nbytes, nbytes)) return 1;
  double* h = (double*)ts->hbuf;
  h[0] = x;
  double* d = (double*)ts->dbuf;
  cudaMemcpyAsync(d, h, sizeof(double), cudaMemcpyHostToDevice, ts->stream);
  if (rys_eval(ds->rys, nroots, d, 1, d + 1, ts->stream) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "root evaluation launch failed");
    return 1;
  }
  cudaMemcpyAsync(h + 1, d + 1, sizeof(double) * 2 * nroots, cudaMemcpyDeviceToHost, ts->stream);
  if (cudaStreamSynchronize(ts->stream) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "root evaluation failed");
    return 1;
  }
  for (int r = 0; r < nroots; ++r) {
    const double t2 = h[1 + r];
    u[r] = t2 / (1.0 - t2);
    w[r] = h[1 + nroots + r];
  }
  return 0;
}

int cintx_rys_t2_batch(int nroots, const double* x, int64_t nx, double* t2w) {
  clear_error();
  if (nroots < 1 || nroots > CINTX_NRMAX || !x || !t2w || nx < 0) {
    set_error(CINTX_STATUS_INVALID_INPUT, "cintx_rys_t2_batch: bad arguments");
    return CINTX_STATUS_INVALID_INPUT;
  }
  DeviceState* ds;
  int rc;
  if ((rc = device_state(&ds))) return rc;
  ThreadScratch* ts;
  const size_t nb = sizeof(double) * (size_t)nx * (1 + 2 * nroots);
  if ((rc = thread_scratch(&ts, nb, 0))) return rc;
  double* d = (double*)ts->dbuf;
  cudaMemcpyAsync(d, x, sizeof(double) * nx, cudaMemcpyHostToDevice, ts->stream);
  rys_eval(ds->rys, nroots, d, nx, d + nx, ts->stream);
  cudaMemcpyAsync(t2w, d + nx, sizeof(double) * nx * 2 * nroots, cudaMemcpyDeviceToHost, ts->stream);
  if (cudaStreamSynchronize(ts->stream) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "root evaluation failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_cuda_last_error_code(void) { return g_err.code; }
size_t cintx_cuda_last_error_message(char* buf, size_t cap) {
  const std::string& m = g_err.msg;
  if (buf && cap > 0) {
    size_t n = std::min(cap - 1, m.size());
    memcpy(buf, m.data(), n);
    buf[n] = 0;
  }
  return m.size();
}
void cintx_cuda_clear_last_error(void) { clear_error(); }

int64_t cintx_launch_count(void) { return g_ts.launches; }

}  // extern "C"
