// Batched int2e evaluation that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they use this library: code that runs inside a
// memory pool or arena owned by a host framework (which forbids stray allocations), code that
// has already claimed nearly all of HBM for its own buffers, and code that must not trigger the
// implicit device synchronisation a cudaMalloc/cudaFree can cause.  cintx_int2e_noalloc serves
// them: the caller passes host inputs and a device output buffer, and every piece of device
// working memory the evaluation needs lives in two file-scope arrays of this translation unit
// that every GPU loading the library holds until the process exits:
//   - g_noalloc_scratch: CINTX_NOALLOC_SCRATCH_BYTES of screened shell pairs, primitive pairs
//     and quartet records, rewritten by every call;
//   - g_noalloc_rys: the Rys root table, copied once per device at set-up.
// Host code must not hand the arrays' names to a kernel (on the host they are stand-ins, not
// device addresses); it uses the addresses cudaGetSymbolAddress returns for each device.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/cintx_cuda.h"
#include "host_internal.h"

namespace {

constexpr size_t kRysTableDoubles = 87040;  // >= doubles in the device layout of the Rys table

static __device__ __align__(256) unsigned char g_noalloc_scratch[CINTX_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) double g_noalloc_rys[kRysTableDoubles];

struct NoallocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  RysTable rys{};
};

std::mutex g_mu;
NoallocDevice g_dev[64];

// Once per device, with that device current: resolve the arrays' device addresses and copy the
// root table, checked and laid out by rys_table_image exactly as the allocating path uploads it,
// into g_noalloc_rys.
int setup_device(int dev, NoallocDevice** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  NoallocDevice& d = g_dev[dev];
  if (d.ready) {
    *out = &d;
    return CINTX_STATUS_SUCCESS;
  }
  void* scratch = nullptr;
  void* table = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
  if (e == cudaSuccess) e = cudaGetSymbolAddress(&table, g_noalloc_rys);
  if (e != cudaSuccess) {
    cintx::set_error(CINTX_STATUS_EXECUTION_FAILED,
                     std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  std::vector<double> host;
  cintx::RysTableOffsets offs;
  if (cintx::rys_table_image(host, offs) || host.size() > kRysTableDoubles) {
    cintx::set_error(CINTX_STATUS_EXECUTION_FAILED, "Rys table does not match the layout of its static device array");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  RysTable t;
  memset(&t, 0, sizeof(t));
  const double* base = (const double*)table;
  for (int n = 1; n <= CINTX_NRMAX; ++n) {
    t.poly[n] = base + offs.poly[n];
    t.asym[n] = base + offs.asym[n];
    t.xmax[n] = offs.xmax[n];
  }
  e = cudaMemcpy(table, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cintx::set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("Rys table copy failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  d.scratch = (unsigned char*)scratch;
  d.rys = t;
  d.ready = true;
  *out = &d;
  return CINTX_STATUS_SUCCESS;
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

extern "C" int cintx_int2e_noalloc(double* out_dev, const int* shls, int64_t n, int sph, const int* atm,
                                   int natm, const int* bas, int nbas, const double* env, void* stream) {
  using namespace cintx;
  clear_error();
  if (!out_dev || !shls || n < 0) {
    set_error(CINTX_STATUS_NULL_POINTER, "out_dev and shls must not be NULL and n must be >= 0");
    return CINTX_STATUS_NULL_POINTER;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, "no usable CUDA device");
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  NoallocDevice* nd;
  int rc = setup_device(dev, &nd);
  if (rc) return rc;
  Basis B;
  if ((rc = load_basis(B, atm, natm, bas, nbas, env))) return rc;
  if (B.env[PTR_RANGE_OMEGA] != 0.0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "range-separated Coulomb is not supported");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  const bool sp = sph != 0;
  const double cutoff = expcutoff_2e(B.env.data());
  auto next = [&](int l) { return sp ? 2 * l + 1 : (l + 1) * (l + 2) / 2; };

  // screened pairs, oriented with their recurrence centre first (pair_base_first; contractions
  // of one shell: larger virtual index first), as the optimizer orients them
  std::map<std::pair<int, int>, int> pair_id;
  std::vector<ShellPair> pairs;
  std::vector<PrimPair> prims;
  std::vector<int> pair_l1, pair_l2;
  PairHost ph;
  auto get_pair = [&](int x, int y, bool& x_first) {
    x_first = B.vshell[x] != B.vshell[y] ? pair_base_first(B, B.vshell[x], B.vshell[y]) : x >= y;
    const int a = x_first ? x : y, b = x_first ? y : x;
    auto key = std::make_pair(a, b);
    auto it = pair_id.find(key);
    if (it != pair_id.end()) return it->second;
    build_pair(B, a, b, cutoff, ph);
    ph.sp.prim_off = (int)prims.size();
    prims.insert(prims.end(), ph.prims.begin(), ph.prims.end());
    const int id = (int)pairs.size();
    pairs.push_back(ph.sp);
    pair_l1.push_back(ph.la);
    pair_l2.push_back(ph.lb);
    pair_id[key] = id;
    return id;
  };
  struct GKey {
    int li, lj, lk, ll;
    long long s0, s1, s2, s3;
    bool operator<(const GKey& o) const {
      return std::tie(li, lj, lk, ll, s0, s1, s2, s3) < std::tie(o.li, o.lj, o.lk, o.ll, o.s0, o.s1, o.s2, o.s3);
    }
  };
  std::map<GKey, std::vector<QuartetRec>> groups;
  long long off = 0;
  for (int64_t q = 0; q < n; ++q) {
    const int* s = shls + 4 * q;
    int l[4], nc[4], ne[4];
    for (int a = 0; a < 4; ++a) {
      if (s[a] < 0 || s[a] >= B.nbas) {
        set_error(CINTX_STATUS_INVALID_INPUT, "shell index out of range in tuple " + std::to_string(q));
        return CINTX_STATUS_INVALID_INPUT;
      }
      l[a] = B.sh[s[a]].l;
      nc[a] = B.sh[s[a]].nctr;
      ne[a] = next(l[a]);
    }
    long long ast[4], st = 1;
    for (int a = 0; a < 4; ++a) {
      ast[a] = st;
      st *= (long long)nc[a] * ne[a];
    }
    for (int c3 = 0; c3 < nc[3]; ++c3)
      for (int c2 = 0; c2 < nc[2]; ++c2)
        for (int c1 = 0; c1 < nc[1]; ++c1)
          for (int c0 = 0; c0 < nc[0]; ++c0) {
            const int cs[4] = {c0, c1, c2, c3};
            int v[4];
            for (int a = 0; a < 4; ++a) v[a] = B.sh[s[a]].vbase + cs[a];
            bool f1, f2;
            const int id1 = get_pair(v[0], v[1], f1);
            const int id2 = get_pair(v[2], v[3], f2);
            const bool swap = (pair_l1[id2] > pair_l1[id1]) || (pair_l1[id2] == pair_l1[id1] && pair_l2[id2] > pair_l2[id1]);
            const int p1[2] = {f1 ? 0 : 1, f1 ? 1 : 0};
            const int p2[2] = {f2 ? 2 : 3, f2 ? 3 : 2};
            int src[4];
            if (!swap) {
              src[0] = p1[0]; src[1] = p1[1]; src[2] = p2[0]; src[3] = p2[1];
            } else {
              src[0] = p2[0]; src[1] = p2[1]; src[2] = p1[0]; src[3] = p1[1];
            }
            GKey k{l[src[0]], l[src[1]], l[src[2]], l[src[3]], ast[src[0]], ast[src[1]], ast[src[2]], ast[src[3]]};
            if (class_needs_scratch(k.li, k.lj, k.lk, k.ll, sp)) {
              set_error(CINTX_STATUS_UNSUPPORTED_API,
                        "this entry point does not evaluate classes with two or more g shells; use the plan API");
              return CINTX_STATUS_UNSUPPORTED_API;
            }
            QuartetRec r;
            r.pij = swap ? id2 : id1;
            r.pkl = swap ? id1 : id2;
            r.out = off;
            for (int a = 0; a < 4; ++a) r.out += (long long)cs[a] * ne[a] * ast[a];
            groups[k].push_back(r);
          }
    off += st;
  }
  // one packed image of [pairs][primitive pairs][records], checked against the array size
  size_t nrec = 0;
  for (auto& kv : groups) nrec += kv.second.size();
  const size_t o_pairs = 0;
  const size_t o_prims = align256(o_pairs + sizeof(ShellPair) * pairs.size());
  const size_t o_recs = align256(o_prims + sizeof(PrimPair) * prims.size());
  const size_t total = o_recs + sizeof(QuartetRec) * nrec;
  if (total > (size_t)CINTX_NOALLOC_SCRATCH_BYTES) {
    set_error(CINTX_STATUS_MEMORY_LIMIT_EXCEEDED,
              "cintx_int2e_noalloc needs " + std::to_string(total) + " bytes of device scratch for this call, more "
              "than its fixed " + std::to_string((size_t)CINTX_NOALLOC_SCRATCH_BYTES) +
              " bytes; split the tuple list into smaller calls");
    return CINTX_STATUS_MEMORY_LIMIT_EXCEEDED;
  }
  if (nrec == 0) return CINTX_STATUS_SUCCESS;
  std::vector<unsigned char> image(total);
  memcpy(image.data() + o_pairs, pairs.data(), sizeof(ShellPair) * pairs.size());
  if (!prims.empty()) memcpy(image.data() + o_prims, prims.data(), sizeof(PrimPair) * prims.size());
  size_t r0 = 0;
  std::vector<std::pair<GKey, std::pair<size_t, size_t>>> launches;
  for (auto& kv : groups) {
    memcpy(image.data() + o_recs + sizeof(QuartetRec) * r0, kv.second.data(), sizeof(QuartetRec) * kv.second.size());
    launches.push_back({kv.first, {r0, kv.second.size()}});
    r0 += kv.second.size();
  }
  cudaStream_t s = (cudaStream_t)stream;
  // The image is host memory of this call.  Earlier work on the stream (a previous call's kernels
  // still reading the shared array) must finish before the array is overwritten, and the copy
  // must have read the image before the call returns: wait for the stream, copy on it, wait for
  // the copy.  CUDA reports a failure of any step as an error, which the call returns.
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(nd->scratch, image.data(), total, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("scratch upload failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  const ShellPair* dpairs = (const ShellPair*)(nd->scratch + o_pairs);
  const PrimPair* dprims = (const PrimPair*)(nd->scratch + o_prims);
  const QuartetRec* drecs = (const QuartetRec*)(nd->scratch + o_recs);
  for (auto& L : launches) {
    const GKey& k = L.first;
    OutStrides st;
    st.s0 = k.s0;
    st.s1 = k.s1;
    st.s2 = k.s2;
    st.s3 = k.s3;
    for (size_t a = 0; a < L.second.second; a += (size_t)1 << 30) {
      const int nr = (int)std::min<size_t>(L.second.second - a, (size_t)1 << 30);
      e = launch_class(k.li, k.lj, k.lk, k.ll, sp, drecs + L.second.first + a, nr, dpairs, dprims, out_dev, st, cutoff,
                       nd->rys, s);
      if (e != cudaSuccess) {
        set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("kernel launch failed: ") + cudaGetErrorString(e));
        return CINTX_STATUS_EXECUTION_FAILED;
      }
    }
  }
  return CINTX_STATUS_SUCCESS;
}
