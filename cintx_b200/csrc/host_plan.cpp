// Batched plans: explicit shell-tuple lists and Schwarz-screened unique-quartet sweeps.
//
// A plan owns device work descriptions for one CINTOpt.  Its unit of execution is a chunk:
// a list of segments, each one kernel class over a contiguous range of quartet records, with
// the chunk's output blocks back to back (libcint layout per block).  Explicit plans keep
// their records resident; screened plans regenerate each chunk's records on the device from
// per-tile row prefixes (plan_kernels.cu), so no per-quartet host data exists for sweeps of
// 1e10 quartets.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/cintx_cuda.h"
#include "host_internal.h"

namespace cintx {
cudaError_t launch_gen_tile(const int* rows, const int* cols, const long long* row_prefix, int nrows,
                            long long t0, long long t1, long long nout, long long out_base, QuartetRec* recs,
                            cudaStream_t stream);
cudaError_t launch_gen_ranges(const GenRange* ranges, int nranges, long long nrec, QuartetRec* recs,
                              cudaStream_t stream);
cudaError_t launch_prim_x(const QuartetRec* recs, long long nrec, const ShellPair* pairs, const PrimPair* prims,
                          const long long* pbase, double* xout, cudaStream_t stream);
cudaError_t launch_block_absmax_sqrt(const QuartetRec* recs, long long nrec, const double* out, const long long* len,
                                     double* q, cudaStream_t stream);
cudaError_t launch_jk_contract(const QuartetRec* recs, long long nrec, const int2* psh, const int* aoloc,
                               const double* out, const double* dm, int nao, double* A, double* B, cudaStream_t stream,
                               int block_elems);
cudaError_t launch_symmetrize(const double* X, double* M, int n, cudaStream_t stream);
cudaError_t launch_scatter_s8(const QuartetRec* recs, long long nrec, const int2* psh, const int* aoloc,
                              const double* out, double* eri, cudaStream_t stream);
cudaError_t launch_scatter_ao(const QuartetRec* recs, long long nrec, const int2* psh, const int* aoloc,
                              const double* out, double* eri, int mode, long long nao, cudaStream_t stream);
}

using namespace cintx;

namespace {

int nsph_or_cart(int l, bool sph) { return sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }
int ncart(int l) { return (l + 1) * (l + 2) / 2; }

struct Segment {
  int li, lj, lk, ll;
  OutStrides st;
  double expcutoff;
  // explicit: records at d_recs[rec0, rec0+nrec); screened: tile index and quartet range
  long long rec0 = 0;
  long long nrec = 0;
  int tile = -1;
  long long t0 = 0, t1 = 0;
  long long nout = 0;      // doubles per block (screened)
  long long out_off = 0;   // chunk-relative output start of this segment
  double flops = 0;        // algorithmic FP64 flops of the segment
  int range0 = 0;          // merged class segments (tile == -2): GenRange slice
  int nranges = 0;
  bool fp32 = false;       // FP32 recurrences (mixed-precision plans)
  double prim_eps = 0;     // primitive Schwarz threshold (tuned plans)
  int variant = 0;         // launch shape chosen by cintx_plan_autotune (0: default)
  bool swap = false;       // screened: the tile's records are (col, row) pairs
};

struct Chunk {
  std::vector<Segment> segs;     // execution units (one per kernel class for screened plans)
  std::vector<Segment> pieces;   // screened: per-tile ranges in output order
  long long out_size = 0;
  long long nrec = 0;
};

struct Tile {
  int typeA, typeB;
  int li, lj, lk, ll;
  std::vector<int> rows;                // pair ids
  // column pair ids and the prefix of their primitive-pair counts (size cols+1), shared by every
  // tile of one column type
  std::shared_ptr<const std::vector<int>> cols;
  std::shared_ptr<const std::vector<long long>> cum_np;
  std::vector<long long> row_prefix;    // size rows+1
  std::vector<int> colstart;            // per row: first column (empty: 0 for every row)
  long long nprimq = -1;                // primitive quartets of the tile (-1: not yet counted)
  bool fp32 = false;                    // evaluated with FP32 recurrences
  bool swap = false;                    // records take (pij, pkl) = (col, row): the kernel's first pair is the col
  OutStrides st{};                      // output strides of the kernel's axes
  int* d_rows = nullptr;
  int* d_cols = nullptr;
  long long* d_prefix = nullptr;
  int* d_colstart = nullptr;
  int col0(size_t row) const { return colstart.empty() ? 0 : colstart[row]; }
};

// Shells of a stored pair in the order a screened plan reports them and lays its blocks out in.
// The kernels build on the pair's first shell (its recurrence centre, pair_base_first); for equal
// l the pair is reported the other way round, (other, centre), because libcint builds an equal-l
// pair on its second shell (g2e.c:101, g3c2e.c:80): evaluated on a reported tuple, libcint then
// uses the same stable centre.  Unit pairs (3- and 2-centre) report -1 for their missing shell.
int2 reported_shells(const Opt* o, int id) {
  const Basis& B = o->basis;
  const int a = B.vshell[o->pair_a[id]];
  if (o->pair_b[id] < 0) return make_int2(a, -1);
  const int b = B.vshell[o->pair_b[id]];
  return o->pair_la[id] == o->pair_lb[id] ? make_int2(b, a) : make_int2(a, b);
}

}  // namespace

struct CintxPlan {
  Opt* opt = nullptr;
  int family = 0;
  bool sph = true;
  std::vector<Chunk> chunks;
  std::vector<Tile> tiles;
  QuartetRec* d_recs = nullptr;    // explicit: all records; screened: one chunk's records
  long long rec_capacity = 0;
  char* d_tile_pool = nullptr;     // screened: every tile's rows, cols, prefix and colstart arrays
  std::vector<QuartetRec> h_recs;  // explicit plans keep a host copy for chunk_quartets
  std::vector<int> h_tuples;       // explicit: requested tuples (4 per record, -1 for unit)
  CintxPlanStats stats{};
  std::vector<GenRange> ranges;    // screened: all merged-segment ranges
  GenRange* d_ranges = nullptr;
  // captured execution of a chunk list (cintx_plan_graph_build)
  cudaGraphExec_t gexec = nullptr;
  int64_t graph_kernels = 0;
  std::vector<cudaStream_t> branches;
  std::vector<cudaEvent_t> events;
  // end-to-end staging
  double* d_stage = nullptr;
  long long stage_cap = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;
  // explicit plans with learned roots (cintx_plan_use_learned_roots): roots of every primitive
  // quartet, and per record its base (doubles) in d_rootbuf
  double* d_rootbuf = nullptr;
  long long* d_rootbase = nullptr;
  // J/K builds (cintx_plan_jk): shells of each regular pair, AO offsets, accumulators, chunk ring
  int2* d_psh = nullptr;
  int* d_aoloc = nullptr;
  double* d_jkacc = nullptr;
  long long jk_cap = 0;
  cudaEvent_t ev_done[2] = {nullptr, nullptr};
  cudaEvent_t ev_free[2] = {nullptr, nullptr};
};

namespace {

void free_plan_device(CintxPlan* p) {
  if (p->d_recs) cudaFree(p->d_recs);
  p->d_recs = nullptr;
  if (p->d_tile_pool) cudaFree(p->d_tile_pool);  // the tiles' arrays live in it
  p->d_tile_pool = nullptr;
  for (Tile& t : p->tiles) {
    t.d_colstart = nullptr;
    t.d_rows = t.d_cols = nullptr;
    t.d_prefix = nullptr;
  }
  if (p->d_stage) cudaFree(p->d_stage);
  p->d_stage = nullptr;
  if (p->d_ranges) cudaFree(p->d_ranges);
  p->d_ranges = nullptr;
  if (p->gexec) cudaGraphExecDestroy(p->gexec);
  p->gexec = nullptr;
  for (cudaStream_t b : p->branches) cudaStreamDestroy(b);
  p->branches.clear();
  for (cudaEvent_t e : p->events) cudaEventDestroy(e);
  p->events.clear();
  if (p->stream) cudaStreamDestroy(p->stream);
  p->stream = nullptr;
  if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
  p->copy_stream = nullptr;
  if (p->d_rootbuf) cudaFree(p->d_rootbuf);
  if (p->d_rootbase) cudaFree(p->d_rootbase);
  p->d_rootbuf = nullptr;
  p->d_rootbase = nullptr;
  for (int b = 0; b < 2; ++b) {
    if (p->ev_done[b]) cudaEventDestroy(p->ev_done[b]);
    if (p->ev_free[b]) cudaEventDestroy(p->ev_free[b]);
    p->ev_done[b] = p->ev_free[b] = nullptr;
  }
}

// Kernel class and strides for a quartet of oriented pairs (first pair is kernel (ij)).
OutStrides canonical_strides(int li, int lj, int lk, bool sph) {
  OutStrides st;
  const long long n0 = nsph_or_cart(li, sph), n1 = nsph_or_cart(lj, sph), n2 = nsph_or_cart(lk, sph);
  st.s0 = 1;
  st.s1 = n0;
  st.s2 = n0 * n1;
  st.s3 = n0 * n1 * n2;
  return st;
}

}  // namespace

extern "C" {

int cintx_plan_shells(CintxPlan** plan, CINTOpt* optp, int family, const int* shls, int64_t n, int sph,
                      int64_t* offsets_out) {
  clear_error();
  if (!plan || !shls) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan and shls must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  *plan = nullptr;
  Opt* o = as_opt(optp);
  if (!o) {
    set_error(CINTX_STATUS_INVALID_INPUT, "opt is not a handle created by this library");
    return CINTX_STATUS_INVALID_INPUT;
  }
  if (family < CINTX_INT2E || family > CINTX_INT2C2E || n < 0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "unknown integral family");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (o->basis.env[PTR_RANGE_OMEGA] != 0.0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "range-separated Coulomb is not supported");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  const Basis& B = o->basis;
  const int nsh = family == CINTX_INT2E ? 4 : (family == CINTX_INT3C2E ? 3 : 2);
  const double cutoff = family == CINTX_INT2E ? expcutoff_2e(B.env.data()) : expcutoff_3c(B.env.data());
  CintxPlan* p = new CintxPlan();
  p->opt = o;
  p->family = family;
  p->sph = sph != 0;
  // group key -> records
  struct GKey {
    int li, lj, lk, ll;
    long long s0, s1, s2, s3;
    bool operator<(const GKey& o) const {
      return std::tie(li, lj, lk, ll, s0, s1, s2, s3) < std::tie(o.li, o.lj, o.lk, o.ll, o.s0, o.s1, o.s2, o.s3);
    }
  };
  struct Group {
    std::vector<QuartetRec> recs;
    std::vector<int> tuples;
    double flops = 0;
  };
  PhaseLog plog("explicit plan");
  // 1. requested shells and block sizes (serial; the first bad shell index ends the plan)
  auto requested = [&](int64_t q, int (&rs)[4], bool (&unit)[4]) {
    const int* s = shls + q * nsh;
    for (int x = 0; x < 4; ++x) unit[x] = false;
    if (family == CINTX_INT2E) {
      for (int x = 0; x < 4; ++x) rs[x] = s[x];
    } else if (family == CINTX_INT3C2E) {
      rs[0] = s[0]; rs[1] = s[1]; rs[2] = s[2]; rs[3] = -1; unit[3] = true;
    } else {
      rs[0] = s[0]; rs[1] = -1; rs[2] = s[1]; rs[3] = -1; unit[1] = unit[3] = true;
    }
  };
  std::vector<long long> toff((size_t)n + 1, 0);
  int64_t bad_shell = n;  // first tuple with a shell index out of range
  {
    // block sizes into toff[q + 1] on host threads over tuple ranges, then one prefix sum
    const int nb = n >= 65536 ? (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())) : 1;
    std::vector<int64_t> bad(nb, n);
    auto sizes = [&](int t) {
      for (int64_t q = n * t / nb; q < n * (t + 1) / nb; ++q) {
        int rs[4];
        bool unit[4];
        requested(q, rs, unit);
        long long blk = 1;
        for (int x = 0; x < 4; ++x) {
          if (unit[x]) continue;
          if (rs[x] < 0 || rs[x] >= B.nbas) {
            bad[t] = q;
            return;
          }
          blk *= (long long)B.sh[rs[x]].nctr * nsph_or_cart(B.sh[rs[x]].l, p->sph);
        }
        toff[q + 1] = blk;
      }
    };
    if (nb == 1) {
      sizes(0);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < nb; ++t) th.emplace_back(sizes, t);
      for (auto& x : th) x.join();
    }
    for (int t = 0; t < nb; ++t)
      if (bad[t] < n) {
        bad_shell = bad[t];
        break;
      }
    for (int64_t q = 0; q < bad_shell; ++q) toff[q + 1] += toff[q];
  }
  plog.mark("block sizes (host)");
  // 2. records per kernel class: host threads over tuple ranges (each its own groups, joined in
  // tuple order below, so the records of a class keep the order of the list)
  struct Part {
    std::map<GKey, Group> groups;
    double flops = 0;
    long long nprimq = 0;
    int64_t bad_pair = -1;  // first tuple needing a pair the optimizer does not hold
  };
  const int64_t nok = bad_shell;
  const int nthr = nok >= 65536 ? (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())) : 1;
  std::vector<Part> parts(nthr);
  auto work = [&](int t) {
    Part& P = parts[t];
    GKey last_key{};
    Group* last = nullptr;  // consecutive tuples mostly share a group: one map lookup per change
    const int64_t q0 = nok * t / nthr, q1 = nok * (t + 1) / nthr;
    for (int64_t q = q0; q < q1; ++q) {
      int rs[4];
      bool unit[4];
      requested(q, rs, unit);
      int l[4], nc[4], ne[4];
      for (int x = 0; x < 4; ++x) {
        l[x] = unit[x] ? 0 : B.sh[rs[x]].l;
        nc[x] = unit[x] ? 1 : B.sh[rs[x]].nctr;
        ne[x] = unit[x] ? 1 : nsph_or_cart(l[x], p->sph);
      }
      long long ast[4];
      {
        long long st = 1;
        for (int x = 0; x < 4; ++x) {
          ast[x] = unit[x] ? 0 : st;
          if (!unit[x]) st *= (long long)nc[x] * ne[x];
        }
      }
      const long long off = toff[q];
      for (int c3 = 0; c3 < nc[3]; ++c3)
        for (int c2 = 0; c2 < nc[2]; ++c2)
          for (int c1 = 0; c1 < nc[1]; ++c1)
            for (int c0 = 0; c0 < nc[0]; ++c0) {
              const int cs[4] = {c0, c1, c2, c3};
              int v[4];
              for (int x = 0; x < 4; ++x) v[x] = unit[x] ? -1 : B.sh[rs[x]].vbase + cs[x];
              // pair ids with their table orientation
              auto pair_of = [&](int x, int y, int& id, bool& x_first) {
                if (y < 0) {
                  id = o->npairs + x;
                  x_first = true;
                } else if (x < 0) {
                  id = o->npairs + y;
                  x_first = false;
                } else {
                  id = pair_index(x, y);
                  x_first = (o->pair_a[id] == x);
                }
              };
              if ((v[0] >= 0 && v[1] >= 0 && std::max(v[0], v[1]) >= o->npv) ||
                  (v[2] >= 0 && v[3] >= 0 && std::max(v[2], v[3]) >= o->npv)) {
                P.bad_pair = q;
                return;
              }
              int id1, id2;
              bool f1, f2;
              pair_of(v[0], v[1], id1, f1);
              pair_of(v[2], v[3], id2, f2);
              const int l1a = o->pair_la[id1], l1b = o->pair_lb[id1];
              const int l2a = o->pair_la[id2], l2b = o->pair_lb[id2];
              const bool swap = (l2a > l1a) || (l2a == l1a && l2b > l1b);
              int src[4];
              const int p1[2] = {f1 ? 0 : 1, f1 ? 1 : 0};
              const int p2[2] = {f2 ? 2 : 3, f2 ? 3 : 2};
              if (!swap) {
                src[0] = p1[0]; src[1] = p1[1]; src[2] = p2[0]; src[3] = p2[1];
              } else {
                src[0] = p2[0]; src[1] = p2[1]; src[2] = p1[0]; src[3] = p1[1];
              }
              GKey k;
              k.li = l[src[0]];
              k.lj = l[src[1]];
              k.lk = l[src[2]];
              k.ll = l[src[3]];
              k.s0 = ast[src[0]];
              k.s1 = ast[src[1]];
              k.s2 = ast[src[2]];
              k.s3 = ast[src[3]];
              QuartetRec r;
              r.pij = swap ? id2 : id1;
              r.pkl = swap ? id1 : id2;
              long long o2 = off;
              for (int x = 0; x < 4; ++x) o2 += (long long)cs[x] * ne[x] * ast[x];
              r.out = o2;
              if (!last || last_key < k || k < last_key) {
                last = &P.groups[k];
                last_key = k;
              }
              last->recs.push_back(r);
              for (int x = 0; x < 4; ++x) last->tuples.push_back(rs[x]);
              const long long npq = (long long)o->pair_nprim[r.pij] * o->pair_nprim[r.pkl];
              P.nprimq += npq;
              const double fq = npq * flops_per_prim_quartet(k.li, k.lj, k.lk, k.ll) +
                                flops_c2s(k.li, k.lj, k.lk, k.ll, p->sph);
              P.flops += fq;
              last->flops += fq;
            }
    }
  };
  if (nthr == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < nthr; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  plog.mark("records (host threads)");
  int64_t bad_pair = -1;
  for (const Part& P : parts)
    if (P.bad_pair >= 0) {
      bad_pair = P.bad_pair;
      break;
    }
  if (bad_pair >= 0 && bad_pair < bad_shell) {
    delete p;
    set_error(CINTX_STATUS_INVALID_INPUT,
              "tuple " + std::to_string(bad_pair) + " needs a shell pair this optimizer does not hold");
    return CINTX_STATUS_INVALID_INPUT;
  }
  if (bad_shell < n) {
    delete p;
    set_error(CINTX_STATUS_INVALID_INPUT, "shell index out of range in tuple " + std::to_string(bad_shell));
    return CINTX_STATUS_INVALID_INPUT;
  }
  if (offsets_out)
    for (int64_t q = 0; q < n; ++q) offsets_out[q] = toff[q];
  const long long off = toff[n];
  double flops = 0;
  long long nprimq = 0;
  // join: the union of the parts' classes in key order; each class's records are its parts'
  // records in part (= tuple) order, copied once into the plan's host arrays
  std::map<GKey, std::vector<const Group*>> joined;
  size_t nrec_total = 0;
  for (Part& P : parts) {
    flops += P.flops;
    nprimq += P.nprimq;
    for (auto& kv : P.groups) {
      joined[kv.first].push_back(&kv.second);
      nrec_total += kv.second.recs.size();
    }
  }
  p->h_recs.resize(nrec_total);
  p->h_tuples.resize(nrec_total * 4);
  plog.mark("join");
  Chunk ch;
  long long rec0 = 0;
  std::vector<std::pair<const Group*, long long>> copies;  // (part group, first record)
  for (auto& kv : joined) {
    Segment sg;
    sg.li = kv.first.li;
    sg.lj = kv.first.lj;
    sg.lk = kv.first.lk;
    sg.ll = kv.first.ll;
    sg.st.s0 = kv.first.s0;
    sg.st.s1 = kv.first.s1;
    sg.st.s2 = kv.first.s2;
    sg.st.s3 = kv.first.s3;
    sg.expcutoff = cutoff;
    sg.rec0 = rec0;
    sg.nrec = 0;
    sg.out_off = 0;
    sg.flops = 0;
    for (const Group* g : kv.second) {
      copies.emplace_back(g, rec0 + sg.nrec);
      sg.nrec += (long long)g->recs.size();
      sg.flops += g->flops;
    }
    ch.segs.push_back(sg);
    rec0 += sg.nrec;
  }
  {
    // the records and tuples of every part group into place, on host threads
    std::atomic<size_t> next(0);
    auto place = [&]() {
      for (size_t j; (j = next.fetch_add(1)) < copies.size();) {
        const Group* g = copies[j].first;
        const long long r = copies[j].second;
        if (!g->recs.empty()) memcpy(p->h_recs.data() + r, g->recs.data(), sizeof(QuartetRec) * g->recs.size());
        if (!g->tuples.empty()) memcpy(p->h_tuples.data() + 4 * r, g->tuples.data(), sizeof(int) * g->tuples.size());
      }
    };
    const int nc = copies.size() > 16 ? (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency())) : 1;
    std::vector<std::thread> th;
    for (int t = 1; t < nc; ++t) th.emplace_back(place);
    place();
    for (auto& x : th) x.join();
  }
  ch.out_size = off;
  ch.nrec = rec0;
  p->chunks.push_back(ch);
  p->rec_capacity = rec0;
  if (rec0 > 0) {
    if (cudaMalloc(&p->d_recs, sizeof(QuartetRec) * rec0) != cudaSuccess) {
      delete p;
      set_error(CINTX_STATUS_ALLOCATION_FAILED, "device allocation of quartet records failed");
      return CINTX_STATUS_ALLOCATION_FAILED;
    }
    cudaMemcpy(p->d_recs, p->h_recs.data(), sizeof(QuartetRec) * rec0, cudaMemcpyHostToDevice);
  }
  plog.mark("segments, upload");
  p->stats.nquartets = n;
  p->stats.nintegrals = off;
  p->stats.nchunks = 1;
  p->stats.max_chunk_doubles = off;
  p->stats.nprim_quartets = nprimq;
  p->stats.flops = flops;
  p->stats.device_bytes = (int64_t)(sizeof(QuartetRec) * rec0);
  *plan = p;
  return CINTX_STATUS_SUCCESS;
}

static int run_segment(CintxPlan* p, const Segment& sg, double* out_dev, cudaStream_t stream, DeviceState* ds,
                       ThreadScratch* ts) {
  const Opt* o = p->opt;
  const QuartetRec* recs;
  long long nrec;
  if (sg.tile == -2) {
    QuartetRec* dst = p->d_recs + sg.rec0;
    cudaError_t e = launch_gen_ranges(p->d_ranges + sg.range0, sg.nranges, sg.nrec, dst, stream);
    if (e != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("quartet generation failed: ") + cudaGetErrorString(e));
      return CINTX_STATUS_EXECUTION_FAILED;
    }
    ts->launches++;
    recs = dst;
    nrec = sg.nrec;
  } else if (sg.tile < 0) {
    recs = p->d_recs + sg.rec0;
    nrec = sg.nrec;
  } else {
    const Tile& t = p->tiles[sg.tile];
    QuartetRec* dst = p->d_recs + sg.rec0;
    cudaError_t e = launch_gen_tile(t.d_rows, t.d_cols, t.d_prefix, (int)t.rows.size(), sg.t0, sg.t1, sg.nout, 0,
                                    dst, stream);
    if (e != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("quartet generation failed: ") + cudaGetErrorString(e));
      return CINTX_STATUS_EXECUTION_FAILED;
    }
    ts->launches++;
    recs = dst;
    nrec = sg.t1 - sg.t0;
  }
  // the kernels take an int count; split very large segments
  for (long long r0 = 0; r0 < nrec; r0 += 1LL << 30) {
    const int nr = (int)std::min<long long>(nrec - r0, 1LL << 30);
    const bool rb = p->d_rootbuf && sg.tile == -1;  // learned roots: explicit plans only
    cudaError_t e = launch_class(sg.li, sg.lj, sg.lk, sg.ll, p->sph, recs + r0, nr, o->d_pairs, o->d_prims,
                                 out_dev + sg.out_off, sg.st, sg.expcutoff, ds->rys, stream, sg.fp32, sg.prim_eps,
                                 sg.variant, rb ? p->d_rootbuf : nullptr, rb ? p->d_rootbase + sg.rec0 + r0 : nullptr);
    if (e != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("kernel launch failed: ") + cudaGetErrorString(e));
      return CINTX_STATUS_EXECUTION_FAILED;
    }
    ts->launches++;
  }
  return CINTX_STATUS_SUCCESS;
}

static int exec_prepare(CintxPlan* p, double* out_dev, void* stream_, cudaStream_t* stream, DeviceState** ds,
                        ThreadScratch** ts) {
  if (!p || !out_dev) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan and out_dev must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  int rc;
  if ((rc = device_state(ds))) return rc;
  if ((rc = thread_scratch(ts, 0, 0))) return rc;
  *stream = (cudaStream_t)stream_;  // used as given: 0 is the legacy default stream
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_execute(CintxPlan* p, int64_t chunk, double* out_dev, void* stream_) {
  clear_error();
  cudaStream_t stream;
  DeviceState* ds;
  ThreadScratch* ts;
  int rc = exec_prepare(p, out_dev, stream_, &stream, &ds, &ts);
  if (rc) return rc;
  if (chunk >= (int64_t)p->chunks.size()) {
    set_error(CINTX_STATUS_INVALID_INPUT, "chunk index out of range");
    return CINTX_STATUS_INVALID_INPUT;
  }
  const int64_t c0 = chunk < 0 ? 0 : chunk, c1 = chunk < 0 ? (int64_t)p->chunks.size() : chunk + 1;
  for (int64_t c = c0; c < c1; ++c)
    for (const Segment& sg : p->chunks[c].segs)
      if ((rc = run_segment(p, sg, out_dev, stream, ds, ts))) return rc;
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_execute_segment(CintxPlan* p, int64_t chunk, int seg, double* out_dev, void* stream_) {
  clear_error();
  cudaStream_t stream;
  DeviceState* ds;
  ThreadScratch* ts;
  int rc = exec_prepare(p, out_dev, stream_, &stream, &ds, &ts);
  if (rc) return rc;
  if (chunk < 0 || chunk >= (int64_t)p->chunks.size() || seg < 0 || seg >= (int)p->chunks[chunk].segs.size()) {
    set_error(CINTX_STATUS_INVALID_INPUT, "chunk or segment index out of range");
    return CINTX_STATUS_INVALID_INPUT;
  }
  return run_segment(p, p->chunks[chunk].segs[seg], out_dev, stream, ds, ts);
}

int cintx_plan_execute_host(CintxPlan* p, int64_t chunk, double* out_host) {
  clear_error();
  if (!p || !out_host) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan and out_host must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (chunk >= (int64_t)p->chunks.size()) {
    set_error(CINTX_STATUS_INVALID_INPUT, "chunk index out of range");
    return CINTX_STATUS_INVALID_INPUT;
  }
  if (!p->stream && cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaStreamCreate failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  if (!p->copy_stream && cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaStreamCreate failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  for (int b = 0; b < 2; ++b) {
    if ((!p->ev_done[b] && cudaEventCreateWithFlags(&p->ev_done[b], cudaEventDisableTiming) != cudaSuccess) ||
        (!p->ev_free[b] && cudaEventCreateWithFlags(&p->ev_free[b], cudaEventDisableTiming) != cudaSuccess)) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaEventCreate failed");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
  }
  const int64_t c0 = chunk < 0 ? 0 : chunk, c1 = chunk < 0 ? (int64_t)p->chunks.size() : chunk + 1;
  // two staging buffers when several chunks run: chunk c+1 is evaluated into one while chunk c
  // is copied to the host from the other (copy stream), so the copies hide behind the kernels
  const int nbuf = c1 - c0 > 1 ? 2 : 1;
  long long need = 1;
  for (int64_t c = c0; c < c1; ++c) need = std::max(need, p->chunks[c].out_size);
  if (need * nbuf > p->stage_cap) {
    if (p->d_stage) cudaFree(p->d_stage);
    if (cudaMalloc(&p->d_stage, sizeof(double) * need * nbuf) != cudaSuccess) {
      p->d_stage = nullptr;
      p->stage_cap = 0;
      set_error(CINTX_STATUS_ALLOCATION_FAILED, "device output staging allocation failed");
      return CINTX_STATUS_ALLOCATION_FAILED;
    }
    p->stage_cap = need * nbuf;
  }
  long long hoff = 0;
  int rc = CINTX_STATUS_SUCCESS;
  for (int64_t c = c0; c < c1 && !rc; ++c) {
    const int b = (int)((c - c0) % nbuf);
    double* stage = p->d_stage + (size_t)b * need;
    if (c - c0 >= nbuf) cudaStreamWaitEvent(p->stream, p->ev_free[b], 0);  // its previous copy is done
    rc = cintx_plan_execute(p, c, stage, p->stream);
    if (rc) break;
    cudaEventRecord(p->ev_done[b], p->stream);
    cudaStreamWaitEvent(p->copy_stream, p->ev_done[b], 0);
    cudaMemcpyAsync(out_host + hoff, stage, sizeof(double) * p->chunks[c].out_size, cudaMemcpyDeviceToHost,
                    p->copy_stream);
    cudaEventRecord(p->ev_free[b], p->copy_stream);
    hoff += p->chunks[c].out_size;
  }
  // drain both streams even after a failed launch, so no copy is left writing into out_host
  cudaError_t e1 = cudaStreamSynchronize(p->stream);
  cudaError_t e2 = cudaStreamSynchronize(p->copy_stream);
  if (rc) return rc;
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED,
              std::string("device execution failed: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_execute_host_ring(CintxPlan* p, double* ring, int64_t ring_doubles,
                                  void (*on_chunk)(void* user, int64_t chunk, const double* data, int64_t n),
                                  void* user) {
  clear_error();
  if (!p || !ring) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan and ring must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  const int64_t nch = (int64_t)p->chunks.size();
  long long slot = 1;
  for (const Chunk& c : p->chunks) slot = std::max(slot, c.out_size);
  if (ring_doubles < 2 * slot) {
    set_error(CINTX_STATUS_BUFFER_TOO_SMALL, "the host ring must hold two of the plan's largest chunks");
    return CINTX_STATUS_BUFFER_TOO_SMALL;
  }
  if (!p->stream && cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaStreamCreate failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  if (!p->copy_stream && cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaStreamCreate failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  for (int b = 0; b < 2; ++b) {
    if ((!p->ev_done[b] && cudaEventCreateWithFlags(&p->ev_done[b], cudaEventDisableTiming) != cudaSuccess) ||
        (!p->ev_free[b] && cudaEventCreateWithFlags(&p->ev_free[b], cudaEventDisableTiming) != cudaSuccess)) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaEventCreate failed");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
  }
  if (2 * slot > p->stage_cap) {
    if (p->d_stage) cudaFree(p->d_stage);
    if (cudaMalloc(&p->d_stage, sizeof(double) * 2 * slot) != cudaSuccess) {
      p->d_stage = nullptr;
      p->stage_cap = 0;
      set_error(CINTX_STATUS_ALLOCATION_FAILED, "device output staging allocation failed");
      return CINTX_STATUS_ALLOCATION_FAILED;
    }
    p->stage_cap = 2 * slot;
  }
  // chunk c: evaluated into device stage c%2 (stream), copied to ring slot c%2 (copy stream);
  // the host waits for chunk c-1's copy (while chunk c computes) and hands it to on_chunk before
  // slot (c-1)%2 is written again by chunk c+1
  int rc = CINTX_STATUS_SUCCESS;
  auto host_wait = [&](int64_t c) -> bool {
    if (cudaEventSynchronize(p->ev_free[c % 2]) != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "device execution failed");
      return false;
    }
    if (on_chunk) on_chunk(user, c, ring + (size_t)(c % 2) * slot, p->chunks[c].out_size);
    return true;
  };
  for (int64_t c = 0; c < nch; ++c) {
    const int b = (int)(c % 2);
    double* stage = p->d_stage + (size_t)b * slot;
    if (c >= 2) cudaStreamWaitEvent(p->stream, p->ev_free[b], 0);  // chunk c-2's copy left the stage
    if ((rc = cintx_plan_execute(p, c, stage, p->stream))) break;
    cudaEventRecord(p->ev_done[b], p->stream);
    if (c >= 1 && !host_wait(c - 1)) {
      rc = CINTX_STATUS_EXECUTION_FAILED;
      break;
    }
    cudaStreamWaitEvent(p->copy_stream, p->ev_done[b], 0);
    cudaMemcpyAsync(ring + (size_t)b * slot, stage, sizeof(double) * p->chunks[c].out_size, cudaMemcpyDeviceToHost,
                    p->copy_stream);
    cudaEventRecord(p->ev_free[b], p->copy_stream);
  }
  if (!rc && nch > 0 && !host_wait(nch - 1)) rc = CINTX_STATUS_EXECUTION_FAILED;
  cudaError_t e1 = cudaStreamSynchronize(p->stream);
  cudaError_t e2 = cudaStreamSynchronize(p->copy_stream);
  if (rc) return rc;
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED,
              std::string("device execution failed: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_use_learned_roots(CintxPlan* p, const float* params, int64_t* nfallback, int64_t* npoints) {
  clear_error();
  if (!p) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (p->d_rootbuf) cudaFree(p->d_rootbuf);
  if (p->d_rootbase) cudaFree(p->d_rootbase);
  p->d_rootbuf = nullptr;
  p->d_rootbase = nullptr;
  if (p->gexec) {  // the captured graph reads the table roots
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  if (!params) return CINTX_STATUS_SUCCESS;  // back to table roots
  if (!p->tiles.empty() || p->chunks.size() != 1) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "learned roots are available for explicit tuple plans");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  DeviceState* ds;
  int rc;
  if ((rc = device_state(&ds))) return rc;
  const Opt* o = p->opt;
  const Chunk& ch = p->chunks[0];
  // per record: its primitive quartets' base in points (within its segment) and in doubles
  std::vector<long long> pbase(p->rec_capacity), dbase(p->rec_capacity);
  std::vector<long long> seg_pts(ch.segs.size()), seg_dbl(ch.segs.size());
  long long dtot = 0;
  for (size_t si = 0; si < ch.segs.size(); ++si) {
    const Segment& sg = ch.segs[si];
    const int nr = (sg.li + sg.lj + sg.lk + sg.ll) / 2 + 1;
    if (nr > 9) {
      set_error(CINTX_STATUS_UNSUPPORTED_API, "learned roots cover 1..9 roots");
      return CINTX_STATUS_UNSUPPORTED_API;
    }
    long long pts = 0;
    seg_dbl[si] = dtot;
    for (long long r = sg.rec0; r < sg.rec0 + sg.nrec; ++r) {
      const QuartetRec& q = p->h_recs[r];
      pbase[r] = pts;
      dbase[r] = dtot + pts * 2 * nr;
      pts += (long long)o->pair_nprim[q.pij] * o->pair_nprim[q.pkl];
    }
    seg_pts[si] = pts;
    dtot += pts * 2 * nr;
  }
  long long maxpts = 1;
  for (long long v : seg_pts) maxpts = std::max(maxpts, v);
  float* d_params = nullptr;
  long long* d_pbase = nullptr;
  double* d_x = nullptr;
  int *d_status = nullptr, *d_iters = nullptr;
  bool ok = cudaMalloc(&p->d_rootbuf, sizeof(double) * std::max(dtot, 1LL)) == cudaSuccess &&
            cudaMalloc(&p->d_rootbase, sizeof(long long) * std::max<long long>(p->rec_capacity, 1)) == cudaSuccess &&
            cudaMalloc(&d_params, sizeof(float) * CINTX_RYSNET_NPARAM) == cudaSuccess &&
            cudaMalloc(&d_pbase, sizeof(long long) * std::max<long long>(p->rec_capacity, 1)) == cudaSuccess &&
            cudaMalloc(&d_x, sizeof(double) * maxpts) == cudaSuccess &&
            cudaMalloc(&d_status, sizeof(int) * maxpts) == cudaSuccess &&
            cudaMalloc(&d_iters, sizeof(int) * maxpts) == cudaSuccess;
  int64_t fb = 0, total = 0;
  if (ok) {
    cudaMemcpy(p->d_rootbase, dbase.data(), sizeof(long long) * dbase.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_pbase, pbase.data(), sizeof(long long) * pbase.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_params, params, sizeof(float) * CINTX_RYSNET_NPARAM, cudaMemcpyHostToDevice);
    std::vector<int> st;
    for (size_t si = 0; si < ch.segs.size() && ok; ++si) {
      const Segment& sg = ch.segs[si];
      const int nr = (sg.li + sg.lj + sg.lk + sg.ll) / 2 + 1;
      if (!seg_pts[si]) continue;
      ok = launch_prim_x(p->d_recs + sg.rec0, sg.nrec, o->d_pairs, o->d_prims, d_pbase + sg.rec0, d_x, 0) ==
               cudaSuccess &&
           rys_learned_eval(d_params, ds->rys, nr, d_x, seg_pts[si], p->d_rootbuf + seg_dbl[si], d_status, d_iters,
                            0) == cudaSuccess &&
           cudaDeviceSynchronize() == cudaSuccess;
      st.resize(seg_pts[si]);
      if (ok) cudaMemcpy(st.data(), d_status, sizeof(int) * seg_pts[si], cudaMemcpyDeviceToHost);
      for (int v : st) fb += v == 1;
      total += seg_pts[si];
    }
  }
  cudaFree(d_params);
  cudaFree(d_pbase);
  cudaFree(d_x);
  cudaFree(d_status);
  cudaFree(d_iters);
  if (!ok) {
    if (p->d_rootbuf) cudaFree(p->d_rootbuf);
    if (p->d_rootbase) cudaFree(p->d_rootbase);
    p->d_rootbuf = nullptr;
    p->d_rootbase = nullptr;
    set_error(CINTX_STATUS_EXECUTION_FAILED, "learned root evaluation failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  if (nfallback) *nfallback = fb;
  if (npoints) *npoints = total;
  return CINTX_STATUS_SUCCESS;
}

// Device copies of each regular pair's shells and of the AO offsets (cached in the plan).
static bool ao_maps(CintxPlan* p, const std::vector<int>& aoloc) {
  if (p->d_psh) return true;
  const Opt* o = p->opt;
  // block axes 0 and 1 of a pair: its shells in reported order (the layout screened plans write)
  std::vector<int2> psh(o->npairs);
  for (int id = 0; id < o->npairs; ++id) psh[id] = reported_shells(o, id);
  bool ok = cudaMalloc(&p->d_psh, sizeof(int2) * std::max(o->npairs, 1)) == cudaSuccess &&
            cudaMalloc(&p->d_aoloc, sizeof(int) * aoloc.size()) == cudaSuccess;
  if (ok) {
    cudaMemcpy(p->d_psh, psh.data(), sizeof(int2) * psh.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(p->d_aoloc, aoloc.data(), sizeof(int) * aoloc.size(), cudaMemcpyHostToDevice);
  }
  return ok;
}

int cintx_plan_execute_s8(CintxPlan* p, double* eri, int64_t len, void* stream_) {
  return cintx_plan_execute_ao(p, 8, eri, len, stream_);
}

int cintx_plan_execute_ao(CintxPlan* p, int aosym, double* eri, int64_t len, void* stream_) {
  clear_error();
  if (!p || !eri) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan and eri must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (p->tiles.empty() || p->family != CINTX_INT2E) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "the AO tensor is written from an int2e unique-quartet sweep");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (aosym != 1 && aosym != 4 && aosym != 8) {
    set_error(CINTX_STATUS_INVALID_INPUT, "aosym must be 1, 4 or 8");
    return CINTX_STATUS_INVALID_INPUT;
  }
  const Basis& B = p->opt->basis;
  std::vector<int> aoloc(B.nbas + 1, 0);
  for (int sh = 0; sh < B.nbas; ++sh) aoloc[sh + 1] = aoloc[sh] + nsph_or_cart(B.sh[sh].l, p->sph);
  const long long nao = aoloc[B.nbas], npair = nao * (nao + 1) / 2;
  const long long need = aosym == 8 ? npair * (npair + 1) / 2 : (aosym == 4 ? npair * npair : nao * nao * nao * nao);
  if (len < need) {
    set_error(CINTX_STATUS_BUFFER_TOO_SMALL, "the s" + std::to_string(aosym) + " tensor of " + std::to_string(nao) +
                                                 " functions needs " + std::to_string(need) + " doubles");
    return CINTX_STATUS_BUFFER_TOO_SMALL;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  long long slot = 1;
  for (const Chunk& c : p->chunks) slot = std::max(slot, c.out_size);
  bool ok = ao_maps(p, aoloc);
  if (ok && slot > p->stage_cap) {
    if (p->d_stage) cudaFree(p->d_stage);
    ok = cudaMalloc(&p->d_stage, sizeof(double) * slot) == cudaSuccess;
    p->stage_cap = ok ? slot : 0;
    if (!ok) p->d_stage = nullptr;
  }
  if (!ok) {
    set_error(CINTX_STATUS_ALLOCATION_FAILED, "device allocation for the AO tensor failed");
    return CINTX_STATUS_ALLOCATION_FAILED;
  }
  cudaMemsetAsync(eri, 0, sizeof(double) * need, stream);  // quartets below the cutoff stay 0
  for (int64_t c = 0; c < (int64_t)p->chunks.size(); ++c) {
    int rc = cintx_plan_execute(p, c, p->d_stage, stream);
    if (rc) return rc;
    const cudaError_t e = aosym == 8 ? launch_scatter_s8(p->d_recs, p->chunks[c].nrec, p->d_psh, p->d_aoloc,
                                                         p->d_stage, eri, stream)
                                     : launch_scatter_ao(p->d_recs, p->chunks[c].nrec, p->d_psh, p->d_aoloc,
                                                         p->d_stage, eri, aosym, nao, stream);
    if (e != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "scatter launch failed");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_jk(CintxPlan* p, const double* dm, int nao, double* vj, double* vk, void* stream_) {
  clear_error();
  if (!p || !dm || (!vj && !vk)) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan, dm and one of vj / vk must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (p->tiles.empty() || p->family != CINTX_INT2E) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "J/K builds run over an int2e unique-quartet sweep (cintx_plan_int2e_screened)");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  const Opt* o = p->opt;
  const Basis& B = o->basis;
  std::vector<int> aoloc(B.nbas + 1, 0);
  for (int sh = 0; sh < B.nbas; ++sh) aoloc[sh + 1] = aoloc[sh] + nsph_or_cart(B.sh[sh].l, p->sph);
  if (nao != aoloc[B.nbas]) {
    set_error(CINTX_STATUS_INVALID_INPUT, "nao is " + std::to_string(nao) + ", the basis has " +
                                              std::to_string(aoloc[B.nbas]) + " functions");
    return CINTX_STATUS_INVALID_INPUT;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  long long slot = 1;
  for (const Chunk& c : p->chunks) slot = std::max(slot, c.out_size);
  const long long acc = 2LL * nao * nao;
  bool ok = ao_maps(p, aoloc);
  if (ok && acc > p->jk_cap) {
    if (p->d_jkacc) cudaFree(p->d_jkacc);
    ok = cudaMalloc(&p->d_jkacc, sizeof(double) * acc) == cudaSuccess;
    p->jk_cap = ok ? acc : 0;
    if (!ok) p->d_jkacc = nullptr;
  }
  if (ok && slot > p->stage_cap) {
    if (p->d_stage) cudaFree(p->d_stage);
    ok = cudaMalloc(&p->d_stage, sizeof(double) * slot) == cudaSuccess;
    p->stage_cap = ok ? slot : 0;
    if (!ok) p->d_stage = nullptr;
  }
  if (!ok) {
    set_error(CINTX_STATUS_ALLOCATION_FAILED, "device allocation for the J/K build failed");
    return CINTX_STATUS_ALLOCATION_FAILED;
  }
  double* A = vj ? p->d_jkacc : nullptr;
  double* Bk = vk ? p->d_jkacc + (size_t)nao * nao : nullptr;
  cudaMemsetAsync(p->d_jkacc, 0, sizeof(double) * acc, stream);
  // each chunk: the sweep's kernels into the ring, then its contraction (same stream, so the
  // next chunk's record generation waits for the contraction to have read the records)
  for (int64_t c = 0; c < (int64_t)p->chunks.size(); ++c) {
    int rc = cintx_plan_execute(p, c, p->d_stage, stream);
    if (rc) return rc;
    // one contraction launch per class segment: small blocks one thread per quartet, others a warp
    for (const Segment& sg : p->chunks[c].segs) {
      const int n = nsph_or_cart(sg.li, p->sph) * nsph_or_cart(sg.lj, p->sph) * nsph_or_cart(sg.lk, p->sph) *
                    nsph_or_cart(sg.ll, p->sph);
      if (launch_jk_contract(p->d_recs + sg.rec0, sg.nrec, p->d_psh, p->d_aoloc, p->d_stage, dm, nao, A, Bk, stream,
                             n) != cudaSuccess) {
        set_error(CINTX_STATUS_EXECUTION_FAILED, "J/K contraction launch failed");
        return CINTX_STATUS_EXECUTION_FAILED;
      }
    }
  }
  if ((vj && launch_symmetrize(A, vj, nao, stream) != cudaSuccess) ||
      (vk && launch_symmetrize(Bk, vk, nao, stream) != cudaSuccess)) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "J/K symmetrisation launch failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_stats(const CintxPlan* p, CintxPlanStats* s) {
  if (!p || !s) return CINTX_STATUS_NULL_POINTER;
  *s = p->stats;
  return CINTX_STATUS_SUCCESS;
}

int64_t cintx_plan_chunk_size(const CintxPlan* p, int64_t chunk) {
  if (!p || chunk < 0 || chunk >= (int64_t)p->chunks.size()) return -1;
  return p->chunks[chunk].out_size;
}

int64_t cintx_plan_chunk_nquartets(const CintxPlan* p, int64_t chunk) {
  if (!p || chunk < 0 || chunk >= (int64_t)p->chunks.size()) return -1;
  return p->chunks[chunk].nrec;
}

// Shell tuples of a chunk in output order (4 ints each; -1 for unit slots of 3c/2c plans).
int cintx_plan_chunk_quartets(const CintxPlan* p, int64_t chunk, int* quartets, int64_t cap) {
  if (!p || chunk < 0 || chunk >= (int64_t)p->chunks.size()) return CINTX_STATUS_INVALID_INPUT;
  const Chunk& ch = p->chunks[chunk];
  const Opt* o = p->opt;
  int64_t k = 0;
  for (const Segment& sg : (ch.pieces.empty() ? ch.segs : ch.pieces)) {
    if (sg.tile < 0) {
      // explicit plans list tuples per record (group order), as requested
      for (long long r = 0; r < sg.nrec; ++r, ++k) {
        if (k >= cap) return CINTX_STATUS_BUFFER_TOO_SMALL;
        for (int a = 0; a < 4; ++a) quartets[k * 4 + a] = p->h_tuples[(sg.rec0 + r) * 4 + a];
      }
    } else {
      const Tile& t = p->tiles[sg.tile];
      for (long long q = sg.t0; q < sg.t1; ++q, ++k) {
        if (k >= cap) return CINTX_STATUS_BUFFER_TOO_SMALL;
        const long long row = std::upper_bound(t.row_prefix.begin(), t.row_prefix.end(), q) - t.row_prefix.begin() - 1;
        const int pa = t.rows[row], pb = (*t.cols)[t.col0(row) + q - t.row_prefix[row]];
        const int2 ra = reported_shells(o, pa), rb = reported_shells(o, pb);
        quartets[k * 4 + 0] = ra.x;
        quartets[k * 4 + 1] = ra.y;
        quartets[k * 4 + 2] = rb.x;
        quartets[k * 4 + 3] = rb.y;
      }
    }
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_chunk_segments(const CintxPlan* p, int64_t chunk, int* cls, int64_t* nq, double* flops, int cap) {
  if (!p || chunk < 0 || chunk >= (int64_t)p->chunks.size()) return -1;
  const Chunk& ch = p->chunks[chunk];
  const int n = (int)ch.segs.size();
  for (int s = 0; s < n && s < cap; ++s) {
    const Segment& sg = ch.segs[s];
    if (cls) {
      cls[4 * s] = sg.li;
      cls[4 * s + 1] = sg.lj;
      cls[4 * s + 2] = sg.lk;
      cls[4 * s + 3] = sg.ll;
    }
    if (nq) nq[s] = sg.tile < 0 ? sg.nrec : sg.t1 - sg.t0;  // merged (-2) and explicit (-1) use nrec
    if (flops) flops[s] = sg.flops;
  }
  return n;
}

int cintx_plan_sample_quartets(const CintxPlan* p, uint64_t seed, int64_t n, int* quartets) {
  if (!p || !quartets || n < 0) return CINTX_STATUS_NULL_POINTER;
  const Opt* o = p->opt;
  uint64_t st = seed;
  auto next = [&]() {  // splitmix64
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  if (!p->tiles.empty()) {
    std::vector<long long> tp(p->tiles.size() + 1, 0);
    for (size_t t = 0; t < p->tiles.size(); ++t) tp[t + 1] = tp[t] + p->tiles[t].row_prefix.back();
    const long long total = tp.back();
    for (int64_t k = 0; k < n; ++k) {
      const long long g = (long long)(next() % (uint64_t)total);
      const size_t ti = std::upper_bound(tp.begin(), tp.end(), g) - tp.begin() - 1;
      const Tile& t = p->tiles[ti];
      const long long q = g - tp[ti];
      const long long row = std::upper_bound(t.row_prefix.begin(), t.row_prefix.end(), q) - t.row_prefix.begin() - 1;
      const int pa = t.rows[row], pb = (*t.cols)[t.col0(row) + q - t.row_prefix[row]];
      const int2 ra = reported_shells(o, pa), rb = reported_shells(o, pb);
      quartets[k * 4 + 0] = ra.x;
      quartets[k * 4 + 1] = ra.y;
      quartets[k * 4 + 2] = rb.x;
      quartets[k * 4 + 3] = rb.y;
    }
  } else {
    const long long total = (long long)p->h_tuples.size() / 4;
    if (total == 0) return CINTX_STATUS_INVALID_INPUT;
    for (int64_t k = 0; k < n; ++k) {
      const long long g = (long long)(next() % (uint64_t)total);
      for (int a = 0; a < 4; ++a) quartets[k * 4 + a] = p->h_tuples[g * 4 + a];
    }
  }
  return CINTX_STATUS_SUCCESS;
}

// Captures the execution of `chunks` (n entries; all when chunks == NULL) into one CUDA graph
// writing to out_dev.  Inside a chunk the kernel classes are independent (disjoint outputs)
// and are spread over `nbranch` parallel branches by their flop estimate; chunks follow each
// other because they share out_dev.
// Launch shapes chosen by the autotuner, per device and class (li, lj, lk, ll, fp32): kept for
// the life of the process so that later plans can reuse them (cintx_plan_use_tuned_shapes).
static std::mutex g_tuned_mu;
static std::map<std::tuple<int, int, int, int, int, int>, int> g_tuned;

int cintx_plan_autotune(CintxPlan* p, int64_t chunk, double* out_dev, void* stream_, int reps) {
  clear_error();
  cudaStream_t stream;
  DeviceState* ds;
  ThreadScratch* ts;
  int rc = exec_prepare(p, out_dev, stream_, &stream, &ds, &ts);
  if (rc) return rc;
  if (chunk >= (int64_t)p->chunks.size()) {
    set_error(CINTX_STATUS_INVALID_INPUT, "chunk index out of range");
    return CINTX_STATUS_INVALID_INPUT;
  }
  reps = std::max(1, std::min(reps, 100));
  // the segment each class is timed on: its first in `chunk`, or (chunk < 0) its largest in
  // the plan, so that classes living in different chunks are all tuned
  std::map<std::tuple<int, int, int, int, int>, std::pair<int64_t, int>> target;
  for (int64_t c = chunk < 0 ? 0 : chunk; c < (chunk < 0 ? (int64_t)p->chunks.size() : chunk + 1); ++c)
    for (int i = 0; i < (int)p->chunks[c].segs.size(); ++i) {
      const Segment& sg = p->chunks[c].segs[i];
      const auto key = std::make_tuple(sg.li, sg.lj, sg.lk, sg.ll, (int)sg.fp32);
      auto it = target.find(key);
      if (it == target.end() || (chunk < 0 && p->chunks[it->second.first].segs[it->second.second].nrec < sg.nrec))
        target[key] = std::make_pair(c, i);
    }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaEventCreate failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  // time every class segment of the chunk in each launch shape that is distinct (lanes per
  // quartet, register cap) and needs device scratch only if the default shape does, so graphs
  // stay possible
  std::map<std::tuple<int, int, int, int, int>, int> best;
  // CINTX_AUTOTUNE_LOG=1 prints every timing to stderr
  const char* tl = getenv("CINTX_AUTOTUNE_LOG");
  const bool tune_log = tl && tl[0] && tl[0] != '0';
  for (const auto& tg : target) {
    const auto& key = tg.first;
    const Segment& sg0 = p->chunks[tg.second.first].segs[tg.second.second];
    const bool scratch0 = class_needs_scratch(sg0.li, sg0.lj, sg0.lk, sg0.ll, p->sph, 0);
    std::vector<int> lanes_seen;
    double best_ms = 1e300;
    int best_v = 0;
    for (int v = 0; v < kLaunchVariants && !rc; ++v) {
      const int shape = variant_shape(sg0.li, sg0.lj, sg0.lk, sg0.ll, p->sph, sg0.fp32, v);
      if (std::find(lanes_seen.begin(), lanes_seen.end(), shape) != lanes_seen.end()) continue;
      lanes_seen.push_back(shape);
      if (!scratch0 && class_needs_scratch(sg0.li, sg0.lj, sg0.lk, sg0.ll, p->sph, v)) continue;
      Segment sg = sg0;
      sg.variant = v;
      if ((rc = run_segment(p, sg, out_dev, stream, ds, ts))) break;  // warm-up
      cudaEventRecord(e0, stream);
      for (int r = 0; r < reps && !rc; ++r) rc = run_segment(p, sg, out_dev, stream, ds, ts);
      cudaEventRecord(e1, stream);
      if (rc) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        set_error(CINTX_STATUS_EXECUTION_FAILED, "device execution failed during autotuning");
        rc = CINTX_STATUS_EXECUTION_FAILED;
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (tune_log)
        fprintf(stderr, "cintx autotune (%d%d|%d%d)%s variant %d lanes %d: %.4f ms\n", sg0.li, sg0.lj, sg0.lk, sg0.ll,
                sg0.fp32 ? " fp32" : "", v, variant_lanes(sg0.li, sg0.lj, sg0.lk, sg0.ll, p->sph, sg0.fp32, v),
                ms / reps);
      if (ms < best_ms) {
        best_ms = ms;
        best_v = v;
      }
    }
    if (rc) break;
    best[key] = best_v;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    for (const auto& kv : best)
      g_tuned[std::make_tuple(dev, std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
                              std::get<3>(kv.first), std::get<4>(kv.first))] = kv.second;
  }
  for (Chunk& ch : p->chunks)
    for (Segment& sg : ch.segs) {
      auto it = best.find(std::make_tuple(sg.li, sg.lj, sg.lk, sg.ll, (int)sg.fp32));
      if (it != best.end()) sg.variant = it->second;
    }
  if (p->gexec) {  // the captured graph holds the old launch shapes
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_use_tuned_shapes(CintxPlan* p) {
  clear_error();
  if (!p) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan must not be NULL");
    return -1;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  int applied = 0;
  std::lock_guard<std::mutex> lk(g_tuned_mu);
  for (Chunk& ch : p->chunks)
    for (Segment& sg : ch.segs) {
      auto it = g_tuned.find(std::make_tuple(dev, sg.li, sg.lj, sg.lk, sg.ll, (int)sg.fp32));
      if (it != g_tuned.end()) {
        sg.variant = it->second;
        ++applied;
      }
    }
  if (applied && p->gexec) {
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  return applied;
}

int cintx_tuned_shapes_export(int* records, int cap) {
  clear_error();
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tuned_mu);
  int n = 0;
  for (const auto& kv : g_tuned) {
    if (std::get<0>(kv.first) != dev) continue;
    if (records && n < cap) {
      int* r = records + 6 * n;
      r[0] = std::get<1>(kv.first);
      r[1] = std::get<2>(kv.first);
      r[2] = std::get<3>(kv.first);
      r[3] = std::get<4>(kv.first);
      r[4] = std::get<5>(kv.first);
      r[5] = kv.second;
    }
    ++n;
  }
  return n;
}

int cintx_tuned_shapes_import(const int* records, int n) {
  clear_error();
  if (n < 0 || (n > 0 && !records)) {
    set_error(CINTX_STATUS_NULL_POINTER, "records must hold n entries");
    return CINTX_STATUS_NULL_POINTER;
  }
  for (int i = 0; i < n; ++i) {
    const int* r = records + 6 * i;
    if (r[0] < 0 || r[0] > CINTX_LMAX || r[1] < 0 || r[2] < 0 || r[3] < 0 || r[5] < 0 || r[5] >= kLaunchVariants) {
      set_error(CINTX_STATUS_INVALID_INPUT, "tuned-shape record " + std::to_string(i) + " is out of range");
      return CINTX_STATUS_INVALID_INPUT;
    }
  }
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tuned_mu);
  for (int i = 0; i < n; ++i) {
    const int* r = records + 6 * i;
    g_tuned[std::make_tuple(dev, r[0], r[1], r[2], r[3], r[4] ? 1 : 0)] = r[5];
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_set_shape(CintxPlan* p, int variant) {
  clear_error();
  if (!p) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan must not be NULL");
    return -1;
  }
  if (variant < 0 || variant >= kLaunchVariants) {
    set_error(CINTX_STATUS_INVALID_INPUT, "launch-shape variant out of range");
    return -1;
  }
  int changed = 0;
  for (Chunk& ch : p->chunks)
    for (Segment& sg : ch.segs) {
      changed += sg.variant != variant;
      sg.variant = variant;
    }
  if (changed && p->gexec) {
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  return changed;
}

int cintx_plan_segment_lanes(const CintxPlan* p, int64_t chunk, int* lanes, int cap) {
  if (!p || chunk < 0 || chunk >= (int64_t)p->chunks.size()) return -1;
  const std::vector<Segment>& segs = p->chunks[chunk].segs;
  for (int i = 0; i < (int)segs.size() && i < cap && lanes; ++i)
    lanes[i] = variant_lanes(segs[i].li, segs[i].lj, segs[i].lk, segs[i].ll, p->sph, segs[i].fp32, segs[i].variant);
  return (int)segs.size();
}

int cintx_plan_graph_build(CintxPlan* p, const int64_t* chunks, int64_t n, double* out_dev, int nbranch) {
  clear_error();
  if (!p || !out_dev) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan and out_dev must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  std::vector<int64_t> list;
  if (chunks) list.assign(chunks, chunks + n);
  else
    for (int64_t c = 0; c < (int64_t)p->chunks.size(); ++c) list.push_back(c);
  for (int64_t c : list) {
    if (c < 0 || c >= (int64_t)p->chunks.size()) {
      set_error(CINTX_STATUS_INVALID_INPUT, "chunk index out of range");
      return CINTX_STATUS_INVALID_INPUT;
    }
    for (const Segment& sg : p->chunks[c].segs)
      if (class_needs_scratch(sg.li, sg.lj, sg.lk, sg.ll, p->sph, sg.variant)) {
        set_error(CINTX_STATUS_UNSUPPORTED_API, "plan contains classes with device scratch; use cintx_plan_execute");
        return CINTX_STATUS_UNSUPPORTED_API;
      }
  }
  DeviceState* ds;
  ThreadScratch* ts;
  int rc;
  if ((rc = device_state(&ds)) || (rc = thread_scratch(&ts, 0, 0))) return rc;
  nbranch = std::max(1, std::min(nbranch, 16));
  if (p->gexec) {
    cudaGraphExecDestroy(p->gexec);
    p->gexec = nullptr;
  }
  while ((int)p->branches.size() < nbranch) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "cudaStreamCreate failed");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
    p->branches.push_back(s);
  }
  while ((int)p->events.size() < nbranch + 1) {
    cudaEvent_t e;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    p->events.push_back(e);
  }
  cudaStream_t origin = p->branches[0];
  if (cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "stream capture could not start");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  const int64_t l0 = ts->launches;
  for (int64_t c : list) {
    const Chunk& ch = p->chunks[c];
    cudaEventRecord(p->events[0], origin);
    for (int b = 1; b < nbranch; ++b) cudaStreamWaitEvent(p->branches[b], p->events[0], 0);
    // longest-first assignment of class segments to branches
    std::vector<int> idx(ch.segs.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return ch.segs[a].flops > ch.segs[b].flops; });
    std::vector<double> load(nbranch, 0.0);
    for (int i : idx) {
      const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      load[b] += ch.segs[i].flops + 1.0;
      if ((rc = run_segment(p, ch.segs[i], out_dev, p->branches[b], ds, ts))) {
        cudaGraph_t g;
        cudaStreamEndCapture(origin, &g);
        if (g) cudaGraphDestroy(g);
        return rc;
      }
    }
    for (int b = 1; b < nbranch; ++b) {
      cudaEventRecord(p->events[b], p->branches[b]);
      cudaStreamWaitEvent(origin, p->events[b], 0);
    }
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(origin, &graph);
  if (e != cudaSuccess || !graph) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("stream capture failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  e = cudaGraphInstantiate(&p->gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    p->gexec = nullptr;
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("graph instantiation failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  p->graph_kernels = ts->launches - l0;
  ts->launches = l0;  // captured, not launched
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_graph_launch(CintxPlan* p, void* stream) {
  clear_error();
  if (!p || !p->gexec) {
    set_error(CINTX_STATUS_INVALID_INPUT, "plan has no captured graph");
    return CINTX_STATUS_INVALID_INPUT;
  }
  ThreadScratch* ts;
  int rc;
  if ((rc = thread_scratch(&ts, 0, 0))) return rc;
  cudaError_t e = cudaGraphLaunch(p->gexec, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("graph launch failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  ts->launches += p->graph_kernels;
  return CINTX_STATUS_SUCCESS;
}

void cintx_plan_destroy(CintxPlan* p) {
  if (!p) return;
  free_plan_device(p);
  delete p;
}

}  // extern "C"

namespace cintx {

// Primitive Schwarz factors.  A primitive-per-shell copy of the basis (coefficient 1, no
// exponent screening) gives every needed primitive diagonal block (ab|ab) in cartesian form on
// the device; q_ab = |c_a c_b| sqrt(max|(ab|ab)|) then bounds every cartesian primitive integral
// of a quartet, |c_a c_b c_c c_d (ab|cd)| <= q_ab q_cd (Cauchy-Schwarz for the Coulomb metric).
// Pieces of the calling thread's device scratch (grown to fit, kept between calls), one per
// requested byte size, each 256-byte aligned.  Valid until the thread's next scratch request; the
// one-shot passes below use them instead of allocating and freeing device memory on every plan.
static int scratch_pieces(ThreadScratch** ts, const std::vector<size_t>& sizes, std::vector<char*>& out) {
  size_t total = 0;
  for (size_t b : sizes) total += (b + 255) & ~(size_t)255;
  int rc = thread_scratch(ts, std::max<size_t>(total, 256), 0);
  if (rc) return rc;
  out.clear();
  char* p = static_cast<char*>((*ts)->dbuf);
  for (size_t b : sizes) {
    out.push_back(p);
    p += (b + 255) & ~(size_t)255;
  }
  return CINTX_STATUS_SUCCESS;
}

int compute_prim_schwarz(Opt* o) {
  std::lock_guard<std::mutex> lk(o->mu);
  if (o->prim_schwarz) return CINTX_STATUS_SUCCESS;
  PhaseLog plog("primitive Schwarz");
  const Basis& B = o->basis;
  DeviceState* ds;
  ThreadScratch* ts;
  int rc;
  if ((rc = device_state(&ds)) || (rc = thread_scratch(&ts, 0, 0))) return rc;
  std::vector<ShellPair> sps(o->npairs + B.nvirt);
  cudaMemcpy(sps.data(), o->d_pairs, sizeof(ShellPair) * sps.size(), cudaMemcpyDeviceToHost);
  // One single-primitive copy of its shell pair per stored primitive pair k (regular pairs): the
  // diagonal quartet of that copy is (c_a c_b)^2 (ab|ab) of the unit-coefficient primitives, since
  // the pair prefactor holds the coefficients, so sqrt(max |block|) is q_k directly.  Cartesian
  // blocks, no exponent screening; grouped by class (la, lb | la, lb).
  long long nk = 0;
  for (int id = 0; id < o->npairs; ++id) nk += sps[id].nprim;
  std::vector<double> qk(nk, 0.0);
  if (nk > 0) {
    std::vector<ShellPair> tp(nk);
    std::map<std::pair<int, int>, std::vector<QuartetRec>> groups;
    std::vector<long long> blk_off, blk_len;  // per group record, in group order later
    for (int id = 0; id < o->npairs; ++id)
      for (int i = 0; i < sps[id].nprim; ++i) {
        const long long k = sps[id].prim_off + i;
        tp[k] = sps[id];
        tp[k].prim_off = (int)k;
        tp[k].nprim = 1;
        QuartetRec r;
        r.pij = r.pkl = (int)k;
        r.out = 0;
        groups[std::make_pair(o->pair_la[id], o->pair_lb[id])].push_back(r);
      }
    // output offsets, block lengths and the record -> primitive-pair map, group by group
    std::vector<QuartetRec> recs;
    std::vector<long long> len;
    long long tot = 0;
    for (auto& kv : groups) {
      const int la = kv.first.first, lb = kv.first.second;
      const long long n = (long long)ncart(la) * ncart(la) * ncart(lb) * ncart(lb);
      for (QuartetRec& r : kv.second) {
        r.out = tot;
        tot += n;
        recs.push_back(r);
        len.push_back(n);
      }
    }
    plog.mark("records (host)");
    std::vector<char*> pc;
    bool ok = scratch_pieces(&ts, {sizeof(ShellPair) * nk, sizeof(QuartetRec) * recs.size(),
                                   sizeof(double) * std::max(tot, 1LL), sizeof(long long) * len.size(),
                                   sizeof(double) * recs.size()}, pc) == CINTX_STATUS_SUCCESS;
    ShellPair* d_tp = ok ? reinterpret_cast<ShellPair*>(pc[0]) : nullptr;
    QuartetRec* d_recs = ok ? reinterpret_cast<QuartetRec*>(pc[1]) : nullptr;
    double* d_out = ok ? reinterpret_cast<double*>(pc[2]) : nullptr;
    long long* d_len = ok ? reinterpret_cast<long long*>(pc[3]) : nullptr;
    double* d_q = ok ? reinterpret_cast<double*>(pc[4]) : nullptr;
    if (ok) {
      cudaMemcpyAsync(d_tp, tp.data(), sizeof(ShellPair) * nk, cudaMemcpyHostToDevice, ts->stream);
      cudaMemcpyAsync(d_recs, recs.data(), sizeof(QuartetRec) * recs.size(), cudaMemcpyHostToDevice, ts->stream);
      cudaMemcpyAsync(d_len, len.data(), sizeof(long long) * len.size(), cudaMemcpyHostToDevice, ts->stream);
      long long r0 = 0;
      for (auto& kv : groups) {
        const int la = kv.first.first, lb = kv.first.second;
        const long long nrec = (long long)kv.second.size();
        OutStrides st;
        st.s0 = 1;
        st.s1 = ncart(la);
        st.s2 = (long long)ncart(la) * ncart(lb);
        st.s3 = st.s2 * ncart(la);
        for (long long q0 = 0; q0 < nrec && ok; q0 += 1LL << 30) {
          const int nr = (int)std::min<long long>(nrec - q0, 1LL << 30);
          ok = launch_class(la, lb, la, lb, false, d_recs + r0 + q0, nr, d_tp, o->d_prims, d_out, st, 1e6, ds->rys,
                            ts->stream) == cudaSuccess;
          ts->launches++;
        }
        r0 += nrec;
      }
      ok = ok && launch_block_absmax_sqrt(d_recs, (long long)recs.size(), d_out, d_len, d_q, ts->stream) == cudaSuccess;
      std::vector<double> q(recs.size());
      if (ok) ok = cudaMemcpyAsync(q.data(), d_q, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, ts->stream) ==
                       cudaSuccess &&
                   cudaStreamSynchronize(ts->stream) == cudaSuccess;
      if (ok)
        for (size_t i = 0; i < recs.size(); ++i) qk[recs[i].pij] = q[i];
    }
    plog.mark("device pass");
    if (!ok) {
      set_error(CINTX_STATUS_EXECUTION_FAILED, "primitive Schwarz pass failed");
      return CINTX_STATUS_EXECUTION_FAILED;
    }
  }
  // q per stored primitive pair, sorted by decreasing q within each shell pair
  o->pair_qp.assign(o->npairs + B.nvirt, 0.0);
  o->pair_amp.assign(o->npairs + B.nvirt, 1.0);
  // each pair writes only its own primitive range and entries: blocks of pairs run on host threads
  auto sort_pair = [&](int id) {
    const int a = o->pair_a[id], b = o->pair_b[id];
    const ShellInfo& SA = B.sh[B.vshell[a]];
    const ShellInfo& SB = B.sh[B.vshell[b]];
    const int k0 = sps[id].prim_off, n = sps[id].nprim;
    std::vector<int> ord(n);
    std::vector<double> qv(n);
    double sum = 0, amp = 1.0;
    for (int i = 0; i < n; ++i) {
      const int k = k0 + i;
      qv[i] = qk[k];
      ord[i] = i;
      sum += qv[i];
      const PrimPair& pp = o->h_prims[k];
      const double da = sqrt((pp.px - SA.r[0]) * (pp.px - SA.r[0]) + (pp.py - SA.r[1]) * (pp.py - SA.r[1]) +
                             (pp.pz - SA.r[2]) * (pp.pz - SA.r[2]));
      const double db = sqrt((pp.px - SB.r[0]) * (pp.px - SB.r[0]) + (pp.py - SB.r[1]) * (pp.py - SB.r[1]) +
                             (pp.pz - SB.r[2]) * (pp.pz - SB.r[2]));
      amp = std::max(amp, pow(1.0 + std::max(da, db) * sqrt(2.0 * pp.aij), SA.l + SB.l));
    }
    o->pair_amp[id] = amp;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return qv[x] > qv[y]; });
    std::vector<PrimPair> pp(n);
    std::vector<int> pa(n), pb(n);
    for (int i = 0; i < n; ++i) {
      pp[i] = o->h_prims[k0 + ord[i]];
      // scaled by the pair's primitive count P: q'_ab q'_cd < eps bounds a quartet's dropped
      // primitive terms by P_ab P_cd max(q_ab q_cd) < eps whatever the quartet's primitive counts
      pp[i].q = qv[ord[i]] * n;
      pa[i] = o->h_prim_a[k0 + ord[i]];
      pb[i] = o->h_prim_b[k0 + ord[i]];
    }
    for (int i = 0; i < n; ++i) {
      o->h_prims[k0 + i] = pp[i];
      o->h_prim_a[k0 + i] = pa[i];
      o->h_prim_b[k0 + i] = pb[i];
    }
    o->pair_qp[id] = sum;
  };
  {
    const int nblk = (o->npairs + 4095) / 4096;
    std::atomic<int> next(0);
    auto worker = [&]() {
      for (int j; (j = next.fetch_add(1)) < nblk;)
        for (int id = j * 4096; id < std::min(o->npairs, (j + 1) * 4096); ++id) sort_pair(id);
    };
    const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int i = 1; i < std::min(nthr, nblk); ++i) th.emplace_back(worker);
    worker();
    for (auto& x : th) x.join();
  }
  plog.mark("sort primitive pairs (host)");
  if (!o->h_prims.empty() &&
      cudaMemcpy(o->d_prims, o->h_prims.data(), sizeof(PrimPair) * o->h_prims.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "upload of sorted primitive pairs failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  o->prim_schwarz = true;
  plog.mark("upload");
  return CINTX_STATUS_SUCCESS;
}

// Contracted Schwarz factors Q_ij = sqrt(max |(ij|ij)|) of every stored pair, from its spherical
// diagonal block: the class kernels evaluate the blocks into the thread's device scratch (classes
// (la lb|la lb), batches of at most 2^25 doubles), block_absmax_sqrt_kernel reduces each block to
// its factor, and only the factors come back to the host.  Same kernels, launch shapes and records
// as an explicit plan of the tuples (a b a b), so the factors are those of that plan bit for bit.
// np < 0: every stored pair; else the first np.
int diag_schwarz_2e(Opt* o, double ecut, std::vector<double>& Q, int np) {
  if (np < 0 || np > o->npairs) np = o->npairs;  // the first np stored pairs (all by default)
  Q.assign(np, 0.0);
  DeviceState* ds;
  ThreadScratch* ts;
  int rc;
  if ((rc = device_state(&ds)) || (rc = thread_scratch(&ts, 0, 0))) return rc;
  std::map<std::pair<int, int>, std::vector<int>> cls;  // (la, lb) -> pair ids
  for (int id = 0; id < np; ++id)
    if (o->pair_nprim[id] > 0) cls[std::make_pair(o->pair_la[id], o->pair_lb[id])].push_back(id);
  const long long cap = 1LL << 25;  // doubles of diagonal blocks per batch
  std::vector<QuartetRec> recs;
  std::vector<long long> len;
  std::vector<int> ids;
  std::vector<std::pair<int, int>> seg_cls;  // class of each segment of the batch
  std::vector<long long> seg_end;            // record end of each segment
  bool ok = true;
  auto flush = [&](long long tot) {
    const long long n = (long long)recs.size();
    if (n > 0 && ok) {
      std::vector<char*> pc;
      ok = scratch_pieces(&ts, {sizeof(QuartetRec) * n, sizeof(long long) * n, sizeof(double) * n,
                                sizeof(double) * std::max(tot, 1LL)}, pc) == CINTX_STATUS_SUCCESS;
      if (ok) {
        QuartetRec* d_recs = reinterpret_cast<QuartetRec*>(pc[0]);
        long long* d_len = reinterpret_cast<long long*>(pc[1]);
        double* d_q = reinterpret_cast<double*>(pc[2]);
        double* d_out = reinterpret_cast<double*>(pc[3]);
        cudaMemcpyAsync(d_recs, recs.data(), sizeof(QuartetRec) * n, cudaMemcpyHostToDevice, ts->stream);
        cudaMemcpyAsync(d_len, len.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, ts->stream);
        long long r0 = 0;
        for (size_t g = 0; g < seg_cls.size() && ok; ++g) {
          const int la = seg_cls[g].first, lb = seg_cls[g].second;
          const OutStrides st = canonical_strides(la, lb, la, true);
          for (long long q0 = r0; q0 < seg_end[g] && ok; q0 += 1LL << 30) {
            const int nr = (int)std::min<long long>(seg_end[g] - q0, 1LL << 30);
            ok = launch_class(la, lb, la, lb, true, d_recs + q0, nr, o->d_pairs, o->d_prims, d_out, st, ecut,
                              ds->rys, ts->stream, false, 0.0, 0, nullptr, nullptr) == cudaSuccess;
            ts->launches++;
          }
          r0 = seg_end[g];
        }
        ok = ok && launch_block_absmax_sqrt(d_recs, n, d_out, d_len, d_q, ts->stream) == cudaSuccess;
        std::vector<double> q(n);
        ok = ok &&
             cudaMemcpyAsync(q.data(), d_q, sizeof(double) * n, cudaMemcpyDeviceToHost, ts->stream) == cudaSuccess &&
             cudaStreamSynchronize(ts->stream) == cudaSuccess;
        if (ok)
          for (long long i = 0; i < n; ++i) Q[ids[i]] = q[i];
      }
    }
    recs.clear();
    len.clear();
    ids.clear();
    seg_cls.clear();
    seg_end.clear();
  };
  long long tot = 0;
  for (auto& kv : cls) {
    const int la = kv.first.first, lb = kv.first.second;
    const long long n = (long long)nsph_or_cart(la, true) * nsph_or_cart(lb, true) * nsph_or_cart(la, true) *
                        nsph_or_cart(lb, true);
    for (int id : kv.second) {
      if (tot + n > cap && !recs.empty()) {  // close the batch: its last segment is this class so far
        seg_cls.push_back(kv.first);
        seg_end.push_back((long long)recs.size());
        flush(tot);
        tot = 0;
      }
      QuartetRec r;
      r.pij = r.pkl = id;
      r.out = tot;
      recs.push_back(r);
      len.push_back(n);
      ids.push_back(id);
      tot += n;
    }
    seg_cls.push_back(kv.first);
    seg_end.push_back((long long)recs.size());
  }
  flush(tot);
  if (!ok) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "diagonal Schwarz pass failed");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

}  // namespace cintx

extern "C" {

static int build_screened(CintxPlan** plan, CINTOpt* optp, double cutoff, int sph, int64_t max_chunk,
                          double fp32_budget, double prim_budget);

int cintx_plan_int2e_screened(CintxPlan** plan, CINTOpt* optp, double cutoff, int sph, int64_t max_chunk) {
  return build_screened(plan, optp, cutoff, sph, max_chunk, 0.0, 0.0);
}

int cintx_plan_int2e_screened_mixed(CintxPlan** plan, CINTOpt* optp, double cutoff, int sph, int64_t max_chunk,
                                    double fp32_budget, double prim_budget) {
  if (fp32_budget > 0 && !sph) {
    set_error(CINTX_STATUS_UNSUPPORTED_REPRESENTATION, "FP32 quartets are compiled for spherical output only");
    return CINTX_STATUS_UNSUPPORTED_REPRESENTATION;
  }
  return build_screened(plan, optp, cutoff, sph, max_chunk, fp32_budget, prim_budget);
}

// FP32 error model of one quartet: 64 * 2^-24 per unit of bound (a factor 5 above the largest
// error/bound seen in the FP32 emulation of the recurrences)
static constexpr double kFp32ErrScale = 64.0 / 16777216.0;

// Largest row 1-norm of the cartesian -> spherical transform of angular momentum l: an error
// bound on cartesian blocks grows by at most this factor per axis in the spherical block.
static double c2s_amp(int l, bool sph) {
  static const double amp[5] = {1.0, 1.0, 1.26156626101008, 2.985410660720923, 7.569397566060481};
  return sph && l >= 2 ? amp[std::min(l, 4)] : 1.0;
}

// Shared tail of the screened planners: flop model, primitive-screening thresholds, chunking at
// quartet boundaries, per-class merged segments and device upload.  The tiles of p are complete
// (rows, cols, row_prefix, cum_np, kernel class, strides, swap).
static long long tile_prim_quartets(const Tile& t, const Opt* o) {
  const std::vector<long long>& cum = *t.cum_np;
  long long tp = 0;
  for (size_t r = 0; r < t.rows.size(); ++r) {
    const long long cnt = t.row_prefix[r + 1] - t.row_prefix[r];
    tp += (long long)o->pair_nprim[t.rows[r]] * (cum[t.col0(r) + cnt] - cum[t.col0(r)]);
  }
  return tp;
}

static int finish_screened(CintxPlan* p, Opt* o, double ecut, int64_t max_chunk, double prim_budget,
                           long long nq_total, long long nint_total, long long nq_fp32, CintxPlan** plan) {
  // tiles of one kernel class next to each other, so that a chunk holds few classes (few
  // launches when the sweep runs in many small chunks) and a class's records fill large launches
  std::stable_sort(p->tiles.begin(), p->tiles.end(), [](const Tile& x, const Tile& y) {
    return std::make_tuple(x.li, x.lj, x.lk, x.ll, x.fp32, x.swap) <
           std::make_tuple(y.li, y.lj, y.lk, y.ll, y.fp32, y.swap);
  });
  long long nprimq = 0;
  double flops = 0;
  // flops: per tile class
  {
    // recompute nprim-weighted flops per tile
    for (const Tile& t : p->tiles) {
      const long long tp = t.nprimq >= 0 ? t.nprimq : tile_prim_quartets(t, o);
      nprimq += tp;
      const long long nq = t.row_prefix.back();
      flops += tp * flops_per_prim_quartet(t.li, t.lj, t.lk, t.ll) + nq * flops_c2s(t.li, t.lj, t.lk, t.ll, p->sph);
    }
  }
  // primitive screening threshold per kernel class and precision: with the primitive factors
  // scaled by their pair's primitive count (compute_prim_schwarz), the dropped primitive quartets
  // of one contracted quartet sum to at most prim_budget / (c2s amplification) in its cartesian
  // block, hence prim_budget in its spherical block
  std::map<std::tuple<int, int, int, int, int>, double> class_eps;
  if (prim_budget > 0)
    for (const Tile& t : p->tiles) {
      const double amp = c2s_amp(t.li, p->sph) * c2s_amp(t.lj, p->sph) * c2s_amp(t.lk, p->sph) * c2s_amp(t.ll, p->sph);
      class_eps[std::make_tuple(t.li, t.lj, t.lk, t.ll, (int)t.fp32)] = prim_budget / amp;
    }
  // 3. chunks: greedy fill up to max_chunk doubles, splitting tiles at quartet boundaries
  Chunk cur;
  long long max_recs = 0;
  for (int ti = 0; ti < (int)p->tiles.size(); ++ti) {
    const Tile& t = p->tiles[ti];
    const long long nq = t.row_prefix.back();
    const long long nout = (long long)nsph_or_cart(t.li, p->sph) * nsph_or_cart(t.lj, p->sph) *
                           nsph_or_cart(t.lk, p->sph) * nsph_or_cart(t.ll, p->sph);
    long long q = 0;
    while (q < nq) {
      long long room = (max_chunk - cur.out_size) / nout;
      if (room <= 0) {
        if (cur.pieces.empty()) room = 1;  // a single block larger than the chunk limit
        else {
          p->chunks.push_back(cur);
          max_recs = std::max(max_recs, cur.nrec);
          cur = Chunk();
          continue;
        }
      }
      const long long take = std::min(room, nq - q);
      Segment sg;
      sg.li = t.li;
      sg.lj = t.lj;
      sg.lk = t.lk;
      sg.ll = t.ll;
      sg.st = t.st;
      sg.swap = t.swap;
      sg.expcutoff = ecut;
      sg.tile = ti;
      sg.fp32 = t.fp32;
      {
        auto it = class_eps.find(std::make_tuple(t.li, t.lj, t.lk, t.ll, (int)t.fp32));
        sg.prim_eps = it == class_eps.end() ? 0.0 : it->second;
      }
      sg.t0 = q;
      sg.t1 = q + take;
      sg.nout = nout;
      sg.rec0 = cur.nrec;
      sg.out_off = cur.out_size;
      {
        // flops of quartets [q, q + take): rows overlapping the range
        double fl = 0;
        const double fpp = flops_per_prim_quartet(t.li, t.lj, t.lk, t.ll);
        long long r = std::upper_bound(t.row_prefix.begin(), t.row_prefix.end(), q) - t.row_prefix.begin() - 1;
        long long pos = q;
        while (pos < q + take) {
          const long long rend = std::min(t.row_prefix[r + 1], q + take);
          const long long c0 = t.col0(r) + pos - t.row_prefix[r], c1 = t.col0(r) + rend - t.row_prefix[r];
          fl += (double)o->pair_nprim[t.rows[r]] * (double)((*t.cum_np)[c1] - (*t.cum_np)[c0]) * fpp;
          pos = rend;
          ++r;
        }
        sg.flops = fl + take * flops_c2s(t.li, t.lj, t.lk, t.ll, p->sph);
      }
      cur.pieces.push_back(sg);
      cur.nrec += take;
      cur.out_size += take * nout;
      q += take;
    }
  }
  if (!cur.pieces.empty()) {
    p->chunks.push_back(cur);
    max_recs = std::max(max_recs, cur.nrec);
  }
  // 4. device buffers
  p->rec_capacity = max_recs;
  bool ok = true;
  if (max_recs > 0) ok = cudaMalloc(&p->d_recs, sizeof(QuartetRec) * max_recs) == cudaSuccess;
  // every tile's arrays in one device allocation and one copy (256-byte aligned slices); a
  // column list shared by several tiles is stored once
  size_t pool_bytes = 0;
  if (ok && !p->tiles.empty()) {
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    std::map<const std::vector<int>*, size_t> col_at;  // shared column list -> its slice
    size_t total = 0;
    for (const Tile& t : p->tiles) {
      total += align(sizeof(int) * t.rows.size()) + align(sizeof(long long) * t.row_prefix.size()) +
               align(sizeof(int) * t.colstart.size());
      if (col_at.emplace(t.cols.get(), 0).second) total += align(sizeof(int) * t.cols->size());
    }
    pool_bytes = total;
    std::vector<char> img(std::max<size_t>(total, 1));
    std::vector<size_t> at;  // slice offsets: rows, cols, prefix, colstart of each tile
    struct Copy {
      const void* src;
      size_t bytes, pos;
    };
    std::vector<Copy> copies;  // filled in on host threads below
    size_t pos = 0;
    auto put = [&](const void* src, size_t bytes) {
      at.push_back(pos);
      if (bytes) copies.push_back({src, bytes, pos});
      pos += align(bytes);
    };
    col_at.clear();
    for (const Tile& t : p->tiles) {
      put(t.rows.data(), sizeof(int) * t.rows.size());
      auto it = col_at.find(t.cols.get());
      if (it == col_at.end()) {
        put(t.cols->data(), sizeof(int) * t.cols->size());
        col_at.emplace(t.cols.get(), at.back());
      } else {
        at.push_back(it->second);
      }
      put(t.row_prefix.data(), sizeof(long long) * t.row_prefix.size());
      put(t.colstart.data(), sizeof(int) * t.colstart.size());
    }
    {
      std::atomic<size_t> next(0);
      auto worker = [&]() {
        for (size_t j; (j = next.fetch_add(64)) < copies.size();)
          for (size_t k = j; k < std::min(j + 64, copies.size()); ++k)
            memcpy(img.data() + copies[k].pos, copies[k].src, copies[k].bytes);
      };
      const int nthr = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
      std::vector<std::thread> th;
      for (int i = 1; i < nthr && (size_t)i * 64 < copies.size(); ++i) th.emplace_back(worker);
      worker();
      for (auto& x : th) x.join();
    }
    ok = cudaMalloc(&p->d_tile_pool, std::max<size_t>(total, 256)) == cudaSuccess;
    if (ok) ok = cudaMemcpy(p->d_tile_pool, img.data(), total, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok)
      for (size_t i = 0; i < p->tiles.size(); ++i) {
        Tile& t = p->tiles[i];
        t.d_rows = reinterpret_cast<int*>(p->d_tile_pool + at[4 * i]);
        t.d_cols = reinterpret_cast<int*>(p->d_tile_pool + at[4 * i + 1]);
        t.d_prefix = reinterpret_cast<long long*>(p->d_tile_pool + at[4 * i + 2]);
        t.d_colstart = t.colstart.empty() ? nullptr : reinterpret_cast<int*>(p->d_tile_pool + at[4 * i + 3]);
      }
  }
  // merge each chunk's tile pieces into one segment per kernel class (records of a class are
  // contiguous; each record carries its chunk-relative output offset)
  for (Chunk& ch : p->chunks) {
    std::vector<int> order;
    std::map<std::tuple<int, int, int, int, int, int>, int> first;
    std::vector<std::vector<int>> members;
    for (int i = 0; i < (int)ch.pieces.size(); ++i) {
      const Segment& pc = ch.pieces[i];
      auto key = std::make_tuple(pc.li, pc.lj, pc.lk, pc.ll, (int)pc.fp32, (int)pc.swap);
      auto it = first.find(key);
      if (it == first.end()) {
        first[key] = (int)members.size();
        members.push_back({i});
      } else {
        members[it->second].push_back(i);
      }
    }
    ch.segs.clear();
    long long rec = 0;
    for (auto& mem : members) {
      const Segment& p0 = ch.pieces[mem[0]];
      Segment m;
      m.li = p0.li;
      m.lj = p0.lj;
      m.lk = p0.lk;
      m.ll = p0.ll;
      m.st = p0.st;
      m.expcutoff = p0.expcutoff;
      m.tile = -2;
      m.fp32 = p0.fp32;
      m.prim_eps = p0.prim_eps;
      m.swap = p0.swap;
      m.rec0 = rec;
      m.out_off = 0;
      m.range0 = (int)p->ranges.size();
      for (int i : mem) {
        const Segment& pc = ch.pieces[i];
        const Tile& t = p->tiles[pc.tile];
        GenRange g;
        g.rows = t.d_rows;
        g.cols = t.d_cols;
        g.prefix = t.d_prefix;
        g.nrows = (int)t.rows.size();
        g.swap = t.swap ? 1 : 0;
        g.colstart = t.d_colstart;
        g.t0 = pc.t0;
        g.t1 = pc.t1;
        g.rec_off = m.nrec;
        g.out_off = pc.out_off;
        g.nout = pc.nout;
        p->ranges.push_back(g);
        m.nrec += pc.t1 - pc.t0;
        m.flops += pc.flops;
      }
      m.nranges = (int)p->ranges.size() - m.range0;
      rec += m.nrec;
      ch.segs.push_back(m);
    }
  }
  if (ok && !p->ranges.empty()) {
    ok = cudaMalloc(&p->d_ranges, sizeof(GenRange) * p->ranges.size()) == cudaSuccess;
    if (ok) cudaMemcpy(p->d_ranges, p->ranges.data(), sizeof(GenRange) * p->ranges.size(), cudaMemcpyHostToDevice);
  }
  if (!ok) {
    free_plan_device(p);
    delete p;
    set_error(CINTX_STATUS_ALLOCATION_FAILED, "device allocation for the screened plan failed");
    return CINTX_STATUS_ALLOCATION_FAILED;
  }
  long long maxc = 0;
  for (const Chunk& c : p->chunks) maxc = std::max(maxc, c.out_size);
  p->stats.nquartets = nq_total;
  p->stats.nintegrals = nint_total;
  p->stats.nchunks = (int64_t)p->chunks.size();
  p->stats.max_chunk_doubles = maxc;
  p->stats.nprim_quartets = nprimq;
  p->stats.flops = flops;
  p->stats.nquartets_fp32 = nq_fp32;
  {
    p->stats.device_bytes = (long long)sizeof(QuartetRec) * max_recs + (long long)pool_bytes;
  }
  *plan = p;
  return CINTX_STATUS_SUCCESS;
}

static int build_screened(CintxPlan** plan, CINTOpt* optp, double cutoff, int sph, int64_t max_chunk,
                          double fp32_budget, double prim_budget) {
  clear_error();
  if (!plan) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  *plan = nullptr;
  Opt* o = as_opt(optp);
  if (!o) {
    set_error(CINTX_STATUS_INVALID_INPUT, "opt is not a handle created by this library");
    return CINTX_STATUS_INVALID_INPUT;
  }
  const Basis& B = o->basis;
  if (B.nvirt != B.nbas) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "screened plans need single-contraction shells (nctr = 1)");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (o->npv != B.nvirt) {
    set_error(CINTX_STATUS_INVALID_INPUT, "the int2e sweep needs an optimizer holding the pairs of every shell");
    return CINTX_STATUS_INVALID_INPUT;
  }
  if (B.env[PTR_RANGE_OMEGA] != 0.0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "range-separated Coulomb is not supported");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (max_chunk <= 0) max_chunk = 1LL << 28;
  if (fp32_budget > 0 || prim_budget > 0) {
    int rc0 = compute_prim_schwarz(o);
    if (rc0) return rc0;
  }
  PhaseLog plog("int2e plan");
  const int np = o->npairs;
  // 1. Schwarz factors from the diagonal (ij|ij) blocks, spherical, reduced on the device
  std::vector<double> Q;
  int rc = diag_schwarz_2e(o, expcutoff_2e(B.env.data()), Q, -1);
  if (rc) return rc;
  plog.mark("diagonal Schwarz pass");
  // 2. pair types (la, lb, nprim_a, nprim_b, work bucket), sorted pairs by decreasing Q.  The
  // bucket groups pairs by their primitive-pair count after exponent screening (half-octave
  // steps): a (kl) pair's count is the trip count of each lane's outer primitive loop, so
  // columns of one type give the lanes of a warp (consecutive columns of a row) equal trip
  // counts instead of running to the longest lane's.
  auto work_bucket = [](int n) {
    int k = 0;
    while ((2 << k) <= n) ++k;  // 2^k <= n < 2^(k+1)
    return 2 * k + ((long long)n * n >= (2LL << (2 * k)) ? 1 : 0);
  };
  std::map<std::tuple<int, int, int, int, int>, std::vector<int>> types;
  double qmax = 0;
  for (int id = 0; id < np; ++id) qmax = std::max(qmax, Q[id]);
  for (int id = 0; id < np; ++id) {
    if (!(Q[id] * qmax >= cutoff) || o->pair_nprim[id] == 0) continue;
    const int a = o->pair_a[id], b = o->pair_b[id];
    types[std::make_tuple(o->pair_la[id], o->pair_lb[id], B.sh[a].nprim, B.sh[b].nprim, work_bucket(o->pair_nprim[id]))]
        .push_back(id);
  }
  // per type: its pairs, their Q and their primitive-pair prefix, shared by the type's tiles
  std::vector<std::shared_ptr<const std::vector<int>>> tlist;
  std::vector<std::shared_ptr<const std::vector<long long>>> tcum;
  std::vector<std::vector<double>> tq;
  std::vector<std::tuple<int, int, int, int, int>> tkeys;
  for (auto& kv : types) {
    std::vector<int> v = kv.second;
    std::stable_sort(v.begin(), v.end(), [&](int x, int y) { return Q[x] > Q[y]; });
    std::vector<long long> cum(v.size() + 1, 0);
    std::vector<double> q(v.size());
    for (size_t c = 0; c < v.size(); ++c) {
      cum[c + 1] = cum[c] + o->pair_nprim[v[c]];
      q[c] = Q[v[c]];
    }
    tlist.push_back(std::make_shared<const std::vector<int>>(std::move(v)));
    tcum.push_back(std::make_shared<const std::vector<long long>>(std::move(cum)));
    tq.push_back(std::move(q));
    tkeys.push_back(kv.first);
  }
  CintxPlan* p = new CintxPlan();
  p->opt = o;
  p->family = CINTX_INT2E;
  p->sph = sph != 0;
  const double ecut = expcutoff_2e(B.env.data());
  long long nq_total = 0, nint_total = 0, nq_fp32 = 0;
  const int nt = (int)tlist.size();
  // tiles A >= B in type order (types are ordered by (la, lb, ...), so classes are valid); one
  // task per (A, B), run on host threads (each task owns its result), joined in (A, B) order
  struct TileJob {
    std::vector<Tile> tiles;
    long long nq = 0, nint = 0, nq32 = 0;
  };
  auto make_tiles = [&](int A, int Bt, TileJob& R) {
    Tile t;
    t.typeA = A;
    t.typeB = Bt;
    t.li = std::get<0>(tkeys[A]);
    t.lj = std::get<1>(tkeys[A]);
    t.lk = std::get<0>(tkeys[Bt]);
    t.ll = std::get<1>(tkeys[Bt]);
    t.st = canonical_strides(t.li, t.lj, t.lk, p->sph);
    // equal-l pairs are reported (other, centre): their two axes trade strides
    if (t.li == t.lj) std::swap(t.st.s0, t.st.s1);
    if (t.lk == t.ll) std::swap(t.st.s2, t.st.s3);
    const std::vector<int>& rows = *tlist[A];
    const std::vector<int>& cols = *tlist[Bt];
    const std::vector<double>& qcols = tq[Bt];
    // FP32 recurrences only where they replace real work (total l >= 4) and where the estimated
    // FP32 error of the quartet, kFp32ErrScale * (qp amp)_ab * (qp amp)_cd * c2s amplification,
    // stays below fp32_budget.  qp is the primitive-absolute bound sum_ab q_ab; amp bounds the
    // cancellation of the recurrences (checked against an FP32 emulation of the recurrences on
    // random quartets of mixed-exponent molecules: the error stayed below 12 * 2^-24 * bound * amp).
    const bool fp32_class = fp32_budget > 0 && t.li + t.lj + t.lk + t.ll >= 4;
    const double fp32_thr =
        fp32_budget / (kFp32ErrScale * c2s_amp(t.li, p->sph) * c2s_amp(t.lj, p->sph) * c2s_amp(t.lk, p->sph) *
                       c2s_amp(t.ll, p->sph));
    // suffix maxima of qp*amp over the Q-sorted columns: the FP32 tail of a row starts where
    // (qp amp)_row * (largest qp amp still ahead) < fp32_thr
    std::vector<double> qp_sufmax(fp32_class ? cols.size() + 1 : 0, 0.0);
    if (fp32_class)
      for (size_t c = cols.size(); c-- > 0;)
        qp_sufmax[c] = std::max(qp_sufmax[c + 1], o->pair_qp[cols[c]] * o->pair_amp[cols[c]]);
    // each row's partner prefix [0, cnt) splits into FP64 columns [0, c64) and FP32 columns
    // [c64, cnt)
    Tile t32 = t;
    t32.fp32 = true;
    t.row_prefix.push_back(0);
    t32.row_prefix.push_back(0);
    // count of cols with qa * Q >= cutoff (cols sorted decreasing): rows come in decreasing Q, so
    // the count never grows from one row to the next and is found by walking it down
    long long cq = (long long)qcols.size();
    for (size_t r = 0; r < rows.size(); ++r) {
      const double qa = Q[rows[r]];
      while (cq > 0 && !(qa * qcols[cq - 1] >= cutoff)) --cq;
      if (cq == 0) break;  // and for every later row
      long long cnt = cq;
      if (A == Bt) cnt = std::min<long long>(cnt, (long long)r + 1);
      if (cnt <= 0) continue;
      long long c64 = cnt;
      if (fp32_class) {
        const double qpa = o->pair_qp[rows[r]] * o->pair_amp[rows[r]];
        c64 = std::partition_point(qp_sufmax.begin(), qp_sufmax.begin() + cols.size(),
                                   [&](double m) { return qpa * m >= fp32_thr; }) - qp_sufmax.begin();
        c64 = std::min(c64, cnt);
      }
      if (c64 > 0) {
        t.rows.push_back(rows[r]);
        t.row_prefix.push_back(t.row_prefix.back() + c64);
      }
      if (cnt > c64) {
        t32.rows.push_back(rows[r]);
        t32.colstart.push_back((int)c64);
        t32.row_prefix.push_back(t32.row_prefix.back() + (cnt - c64));
      }
    }
    const long long nout = (long long)nsph_or_cart(t.li, p->sph) * nsph_or_cart(t.lj, p->sph) *
                           nsph_or_cart(t.lk, p->sph) * nsph_or_cart(t.ll, p->sph);
    for (Tile* tp : {&t, &t32}) {
      if (tp->rows.empty()) continue;
      tp->cols = tlist[Bt];
      tp->cum_np = tcum[Bt];
      tp->nprimq = tile_prim_quartets(*tp, o);
      const long long nq = tp->row_prefix.back();
      R.nq += nq;
      R.nint += nq * nout;
      if (tp->fp32) R.nq32 += nq;
      R.tiles.push_back(std::move(*tp));
    }
  };
  std::vector<std::pair<int, int>> jobs;
  for (int A = 0; A < nt; ++A)
    for (int Bt = 0; Bt <= A; ++Bt) jobs.emplace_back(A, Bt);
  std::vector<TileJob> res(jobs.size());
  {
    std::atomic<size_t> next(0);
    auto worker = [&]() {
      for (size_t j; (j = next.fetch_add(1)) < jobs.size();) make_tiles(jobs[j].first, jobs[j].second, res[j]);
    };
    const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int i = 1; i < std::min<int>(nthr, (int)jobs.size()); ++i) th.emplace_back(worker);
    worker();
    for (auto& x : th) x.join();
  }
  for (TileJob& R : res) {
    nq_total += R.nq;
    nint_total += R.nint;
    nq_fp32 += R.nq32;
    for (Tile& t : R.tiles) p->tiles.push_back(std::move(t));
  }
  {
    char msg[96];
    snprintf(msg, sizeof msg, "tiles (host; %d pair types, %zu tiles)", nt, p->tiles.size());
    plog.mark(msg);
  }
  const int rcf = finish_screened(p, o, ecut, max_chunk, prim_budget, nq_total, nint_total, nq_fp32, plan);
  plog.mark("chunks, segments, device tables");
  return rcf;
}

// Diagonal Schwarz factors sqrt(max |block|) of a list of tuples of one family (spherical).
static int diag_factors(CINTOpt* optp, int family, const std::vector<int>& tuples, int64_t n, std::vector<double>& q) {
  std::vector<int64_t> off(std::max<int64_t>(n, 1));
  CintxPlan* dp = nullptr;
  int rc = cintx_plan_shells(&dp, optp, family, tuples.data(), n, 1, off.data());
  if (rc) return rc;
  const long long tot = dp->stats.nintegrals;
  std::vector<double> out(std::max<long long>(tot, 1));
  rc = cintx_plan_execute_host(dp, 0, out.data());
  cintx_plan_destroy(dp);
  if (rc) return rc;
  q.assign(n, 0.0);
  for (int64_t t = 0; t < n; ++t) {
    const long long e1 = t + 1 < n ? off[t + 1] : tot;
    double m = 0;
    for (long long e = off[t]; e < e1; ++e) m = std::max(m, fabs(out[e]));
    q[t] = sqrt(m);
  }
  return CINTX_STATUS_SUCCESS;
}

int cintx_plan_int3c2e_screened(CintxPlan** plan, CINTOpt* optp, double cutoff, int sph, int64_t max_chunk,
                                int norb) {
  clear_error();
  if (!plan) {
    set_error(CINTX_STATUS_NULL_POINTER, "plan must not be NULL");
    return CINTX_STATUS_NULL_POINTER;
  }
  *plan = nullptr;
  Opt* o = as_opt(optp);
  if (!o) {
    set_error(CINTX_STATUS_INVALID_INPUT, "opt is not a handle created by this library");
    return CINTX_STATUS_INVALID_INPUT;
  }
  const Basis& B = o->basis;
  const int nb = B.nbas;
  if (B.nvirt != B.nbas) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "screened plans need single-contraction shells (nctr = 1)");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (norb < 1 || norb >= nb || o->npv < norb) {
    set_error(CINTX_STATUS_INVALID_INPUT, "norb must split the basis into orbital shells [0, norb) whose pairs the "
                                          "optimizer holds and auxiliary shells [norb, nbas)");
    return CINTX_STATUS_INVALID_INPUT;
  }
  if (B.env[PTR_RANGE_OMEGA] != 0.0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "range-separated Coulomb is not supported");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  if (max_chunk <= 0) max_chunk = 1LL << 28;
  const int npo = norb * (norb + 1) / 2;  // pair ids of the orbital pairs (u < norb)
  const int naux = nb - norb;
  // 1. Schwarz factors: (ab|ab) for orbital pairs (reduced on the device), (k|k) for auxiliary shells
  PhaseLog plog("int3c2e plan");
  std::vector<int> kt((size_t)naux * 2);
  for (int k = 0; k < naux; ++k) kt[2 * k] = kt[2 * k + 1] = norb + k;
  std::vector<double> Q, Qk;
  int rc = diag_schwarz_2e(o, expcutoff_2e(B.env.data()), Q, npo);
  if (!rc) rc = diag_factors(optp, CINTX_INT2C2E, kt, naux, Qk);
  if (rc) return rc;
  plog.mark("diagonal Schwarz passes");
  double qmax = 0, qkmax = 0;
  for (double v : Q) qmax = std::max(qmax, v);
  for (double v : Qk) qkmax = std::max(qkmax, v);
  // 2. row types (la, lb, nprim_a, nprim_b) of orbital pairs and column types (lk, nprim_k) of
  // auxiliary unit pairs, each sorted by decreasing Schwarz factor
  std::map<std::tuple<int, int, int, int>, std::vector<int>> rtypes;
  std::map<std::pair<int, int>, std::vector<int>> ctypes;
  std::vector<double> qpair(o->npairs + B.nvirt, 0.0);
  for (int id = 0; id < npo; ++id) {
    qpair[id] = Q[id];
    if (!(Q[id] * qkmax >= cutoff) || o->pair_nprim[id] == 0) continue;
    rtypes[std::make_tuple(o->pair_la[id], o->pair_lb[id], B.sh[o->pair_a[id]].nprim, B.sh[o->pair_b[id]].nprim)]
        .push_back(id);
  }
  for (int k = 0; k < naux; ++k) {
    const int id = o->npairs + norb + k;
    qpair[id] = Qk[k];
    if (!(Qk[k] * qmax >= cutoff) || o->pair_nprim[id] == 0) continue;
    ctypes[std::make_pair(B.sh[norb + k].l, B.sh[norb + k].nprim)].push_back(id);
  }
  auto by_q = [&](int x, int y) { return qpair[x] > qpair[y]; };
  CintxPlan* p = new CintxPlan();
  p->opt = o;
  p->family = CINTX_INT3C2E;
  p->sph = sph != 0;
  long long nq_total = 0, nint_total = 0;
  // column types sorted once, shared by their tiles
  std::vector<std::pair<int, std::shared_ptr<const std::vector<int>>>> ccols;
  std::vector<std::shared_ptr<const std::vector<long long>>> ccum;
  for (auto& ck : ctypes) {
    std::vector<int> cols = ck.second;
    std::stable_sort(cols.begin(), cols.end(), by_q);
    std::vector<long long> cum(cols.size() + 1, 0);
    for (size_t c = 0; c < cols.size(); ++c) cum[c + 1] = cum[c] + o->pair_nprim[cols[c]];
    ccols.emplace_back(ck.first.first, std::make_shared<const std::vector<int>>(std::move(cols)));
    ccum.push_back(std::make_shared<const std::vector<long long>>(std::move(cum)));
  }
  for (auto& rk : rtypes) {
    std::vector<int> rows = rk.second;
    std::stable_sort(rows.begin(), rows.end(), by_q);
    const int la = std::get<0>(rk.first), lb = std::get<1>(rk.first);
    for (size_t ci = 0; ci < ccols.size(); ++ci) {
      const std::vector<int>& cols = *ccols[ci].second;
      const int lk = ccols[ci].first;
      const long long ni = nsph_or_cart(la, p->sph), nj = nsph_or_cart(lb, p->sph), nk = nsph_or_cart(lk, p->sph);
      Tile t;
      t.typeA = t.typeB = 0;
      // block layout out[i + ni*(j + nj*k)] for the tuple (a, b, k); the kernel's first pair is
      // the larger in (l, l') order, so an auxiliary shell of higher l than a swaps the pairs
      t.swap = lk > la;
      if (!t.swap) {
        t.li = la; t.lj = lb; t.lk = lk; t.ll = 0;
        t.st.s0 = 1; t.st.s1 = ni; t.st.s2 = ni * nj; t.st.s3 = 0;
        if (la == lb) std::swap(t.st.s0, t.st.s1);  // equal-l pairs are reported (other, centre)
      } else {
        t.li = lk; t.lj = 0; t.lk = la; t.ll = lb;
        t.st.s0 = ni * nj; t.st.s1 = 0; t.st.s2 = 1; t.st.s3 = ni;
        if (la == lb) std::swap(t.st.s2, t.st.s3);
      }
      t.row_prefix.push_back(0);
      for (int r : rows) {
        const double qa = qpair[r];
        const long long cnt = std::partition_point(cols.begin(), cols.end(),
                                                   [&](int c) { return qa * qpair[c] >= cutoff; }) - cols.begin();
        if (cnt <= 0) continue;
        t.rows.push_back(r);
        t.row_prefix.push_back(t.row_prefix.back() + cnt);
      }
      if (t.rows.empty()) continue;
      t.cols = ccols[ci].second;
      t.cum_np = ccum[ci];
      nq_total += t.row_prefix.back();
      nint_total += t.row_prefix.back() * ni * nj * nk;
      p->tiles.push_back(t);
    }
  }
  plog.mark("tiles (host)");
  const int rcf = finish_screened(p, o, expcutoff_3c(B.env.data()), max_chunk, 0.0, nq_total, nint_total, 0, plan);
  plog.mark("chunks, segments, device tables");
  return rcf;
}

int64_t cintx_opt_device_bytes(CINTOpt* optp) {
  Opt* o = as_opt(optp);
  if (!o) return -1;
  return (int64_t)(sizeof(ShellPair) * (o->npairs + o->basis.nvirt) + sizeof(PrimPair) * o->nprims_total);
}

}  // extern "C"
