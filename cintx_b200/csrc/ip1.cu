// First-derivative integrals int2e_ip1 and int3c2e_ip1 (libcint autocode/grad2.c:69-88,
// autocode/int3c2e.c:72-88): libcint-signature per-call entry points and a batched device entry
// point over a tuple list.
//
// A derivative tuple (i, j, k, l) runs the class kernel eri_ip1_kernel<li, lj, lk, ll> with the
// derivative pair (i, j) in the requested order (its primitive pairs carry 2 a_i in PrimPair::q and
// are screened with the raised ceiling li + 1, as libcint's ip1 drivers set li_ceil), the second
// pair oriented with its recurrence centre first (pair_base_first), and blocks written
// component-major in libcint's layout: out[c*blk + i + ni*(j + nj*(k + nk*l))], c = x, y, z.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/cintx_cuda.h"
#include "eri_ip1.cuh"
#include "host_internal.h"

namespace cintx {

#define CINTX_DECL_IP1(I, J) cudaError_t dispatch_ip1_l##I##J(int, int, bool, const Ip1Args&);
CINTX_DECL_IP1(0, 0) CINTX_DECL_IP1(0, 1) CINTX_DECL_IP1(0, 2) CINTX_DECL_IP1(0, 3)
CINTX_DECL_IP1(1, 0) CINTX_DECL_IP1(1, 1) CINTX_DECL_IP1(1, 2) CINTX_DECL_IP1(1, 3)
CINTX_DECL_IP1(2, 0) CINTX_DECL_IP1(2, 1) CINTX_DECL_IP1(2, 2) CINTX_DECL_IP1(2, 3)
CINTX_DECL_IP1(3, 0) CINTX_DECL_IP1(3, 1) CINTX_DECL_IP1(3, 2) CINTX_DECL_IP1(3, 3)
#undef CINTX_DECL_IP1

static cudaError_t dispatch_ip1(int li, int lj, int lk, int ll, bool sph, const Ip1Args& a) {
  if (!ip1_class_valid(li, lj, lk, ll)) return cudaErrorInvalidValue;
  switch (li * 10 + lj) {
    case 0: return dispatch_ip1_l00(lk, ll, sph, a);
    case 1: return dispatch_ip1_l01(lk, ll, sph, a);
    case 2: return dispatch_ip1_l02(lk, ll, sph, a);
    case 3: return dispatch_ip1_l03(lk, ll, sph, a);
    case 10: return dispatch_ip1_l10(lk, ll, sph, a);
    case 11: return dispatch_ip1_l11(lk, ll, sph, a);
    case 12: return dispatch_ip1_l12(lk, ll, sph, a);
    case 13: return dispatch_ip1_l13(lk, ll, sph, a);
    case 20: return dispatch_ip1_l20(lk, ll, sph, a);
    case 21: return dispatch_ip1_l21(lk, ll, sph, a);
    case 22: return dispatch_ip1_l22(lk, ll, sph, a);
    case 23: return dispatch_ip1_l23(lk, ll, sph, a);
    case 30: return dispatch_ip1_l30(lk, ll, sph, a);
    case 31: return dispatch_ip1_l31(lk, ll, sph, a);
    case 32: return dispatch_ip1_l32(lk, ll, sph, a);
    case 33: return dispatch_ip1_l33(lk, ll, sph, a);
  }
  return cudaErrorInvalidValue;
}

namespace {

struct Ip1Work {
  std::vector<ShellPair> pairs;
  std::vector<PrimPair> prims;
  struct Key {  // kernel class, output strides and component stride (the tuple's block size)
    int li, lj, lk, ll;
    long long s0, s1, s2, s3, blk;
    bool operator<(const Key& o) const {
      return std::tie(li, lj, lk, ll, s0, s1, s2, s3, blk) <
             std::tie(o.li, o.lj, o.lk, o.ll, o.s0, o.s1, o.s2, o.s3, o.blk);
    }
  };
  std::map<Key, std::vector<QuartetRec>> groups;
  std::vector<double> pair_min_cce;  // per pair: smallest screening exponent of its primitive pairs
  long long out_doubles = 0;  // all components of all blocks
  bool any = false;           // some primitive survived screening (libcint's return value)
};

// Builds pairs and quartet records of n derivative tuples (nsh = 4: int2e_ip1, 3: int3c2e_ip1),
// blocks back to back, component-major within each block.  offsets (may be NULL) receive each
// tuple's block offset.  Returns a status code.
// Screening follows libcint's two drivers: without an optimizer (CINT2e_loop_nopt) only the
// differentiated pair's estimate takes the raised ceiling li + 1; with one, the optimizer's pair
// table (CINTOpt_setij, optimizer.c:344-420) raises every pair's estimate by the derivative order
// and keeps primitive pairs below the cut-off without its "+1" margin.
int ip1_build(const Basis& B, int nsh, const int* shls, int64_t n, bool sph, bool opt_mode, Ip1Work& W,
              int64_t* offsets) {
  const double cutoff = nsh == 4 ? expcutoff_2e(B.env.data()) : expcutoff_3c(B.env.data());
  const double pair_cutoff = opt_mode ? expcutoff_3c(B.env.data()) : cutoff;
  // (a, b, derivative) -> pair id, packed into one 64-bit key (b may be -1: unit pair)
  std::unordered_map<uint64_t, int> pair_id;
  pair_id.reserve(1024);
  auto get_pair = [&](int a, int b, bool deriv) {
    const uint64_t key = ((uint64_t)(uint32_t)a << 33) | ((uint64_t)(uint32_t)(b + 1) << 1) | (deriv ? 1u : 0u);
    auto it = pair_id.find(key);
    if (it != pair_id.end()) return it->second;
    PairHost ph;
    build_pair(B, a, b, pair_cutoff, ph, deriv || (opt_mode && b >= 0) ? 1 : 0);
    if (deriv) {  // 2 a_i of each primitive pair's i primitive
      const ShellInfo& A = B.sh[B.vshell[a]];
      for (size_t k = 0; k < ph.prims.size(); ++k) ph.prims[k].q = 2.0 * A.exps[ph.pa[k]];
    }
    ph.sp.prim_off = (int)W.prims.size();
    W.prims.insert(W.prims.end(), ph.prims.begin(), ph.prims.end());
    const int id = (int)W.pairs.size();
    W.pairs.push_back(ph.sp);
    W.pair_min_cce.push_back(ph.prims.empty() ? 1e300 : ph.min_cce);
    pair_id[key] = id;
    return id;
  };
  auto ncomp = [&](int l) { return sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2; };
  // recurrence centre of each (k, l) pair, computed once per pair (pair_base_first loops over the
  // primitive exponents)
  std::unordered_map<uint64_t, bool> kfirst;
  auto centre_first = [&](int k, int l2) {
    const uint64_t key = ((uint64_t)(uint32_t)k << 32) | (uint32_t)l2;
    auto it = kfirst.find(key);
    if (it != kfirst.end()) return it->second;
    const bool f = pair_base_first(B, k, l2);
    kfirst.emplace(key, f);
    return f;
  };
  std::vector<QuartetRec>* last = nullptr;  // consecutive tuples mostly share a group
  Ip1Work::Key last_key{};
  long long off = 0;
  for (int64_t q = 0; q < n; ++q) {
    const int* s = shls + q * nsh;
    int rs[4] = {s[0], s[1], s[2], nsh == 4 ? s[3] : -1};
    int l[4], nc[4], ne[4];
    for (int a = 0; a < 4; ++a) {
      if (rs[a] < 0) {
        l[a] = 0;
        nc[a] = 1;
        ne[a] = 1;
        continue;
      }
      if (rs[a] >= B.nbas) {
        set_error(CINTX_STATUS_INVALID_INPUT, "shell index out of range in tuple " + std::to_string(q));
        return CINTX_STATUS_INVALID_INPUT;
      }
      l[a] = B.sh[rs[a]].l;
      nc[a] = B.sh[rs[a]].nctr;
      ne[a] = ncomp(l[a]);
    }
    // kernel axes: (i, j) as requested; (k, l) with the recurrence centre first
    const bool kf = rs[3] < 0 || centre_first(rs[2], rs[3]);
    const int src[4] = {0, 1, kf ? 2 : 3, kf ? 3 : 2};
    if (!ip1_class_valid(l[0], l[1], l[src[2]], l[src[3]])) {
      set_error(CINTX_STATUS_UNSUPPORTED_API, "derivative integrals are compiled for l <= 3 on the differentiated "
                                              "pair and the (k l) pair (l = 4 for a 3-centre auxiliary shell)");
      return CINTX_STATUS_UNSUPPORTED_API;
    }
    long long ast[4], st = 1;
    for (int a = 0; a < 4; ++a) {
      ast[a] = rs[a] < 0 ? 0 : st;
      if (rs[a] >= 0) st *= (long long)nc[a] * ne[a];
    }
    if (offsets) offsets[q] = off;
    for (int c3 = 0; c3 < nc[3]; ++c3)
      for (int c2 = 0; c2 < nc[2]; ++c2)
        for (int c1 = 0; c1 < nc[1]; ++c1)
          for (int c0 = 0; c0 < nc[0]; ++c0) {
            const int cs[4] = {c0, c1, c2, c3};
            int v[4];
            for (int a = 0; a < 4; ++a) v[a] = rs[a] < 0 ? -1 : B.sh[rs[a]].vbase + cs[a];
            QuartetRec r;
            r.pij = get_pair(v[0], v[1], true);
            r.pkl = get_pair(v[src[2]], v[src[3]], false);
            // libcint's emptiness test (CINT2e_loop_nopt): some primitive quartet passes the cut-off
            if (W.pair_min_cce[r.pij] + W.pair_min_cce[r.pkl] <= cutoff) W.any = true;
            r.out = off;
            for (int a = 0; a < 4; ++a) r.out += (long long)cs[a] * ne[a] * ast[a];
            Ip1Work::Key k{l[0], l[1], l[src[2]], l[src[3]], ast[0], ast[1], ast[src[2]], ast[src[3]], st};
            if (!last || last_key < k || k < last_key) {
              last = &W.groups[k];
              last_key = k;
            }
            last->push_back(r);
          }
    off += 3 * st;
  }
  W.out_doubles = off;
  return CINTX_STATUS_SUCCESS;
}

// Device image of the work: [pairs][primitive pairs][records], 256-byte aligned parts.
size_t ip1_image_bytes(const Ip1Work& W, size_t* o_prims, size_t* o_recs) {
  size_t nrec = 0;
  for (auto& kv : W.groups) nrec += kv.second.size();
  *o_prims = (sizeof(ShellPair) * W.pairs.size() + 255) & ~(size_t)255;
  *o_recs = (*o_prims + sizeof(PrimPair) * std::max<size_t>(W.prims.size(), 1) + 255) & ~(size_t)255;
  return *o_recs + sizeof(QuartetRec) * std::max<size_t>(nrec, 1);
}

// Copies the image into `dev` (device memory of ip1_image_bytes) from the host staging buffer
// `host` (kept by the caller until the stream has consumed it) and launches every class group on
// `stream`, writing into out_dev.
int ip1_launch(const Ip1Work& W, bool sph, int nsh, const Basis& B, char* dev, char* host, double* out_dev,
               cudaStream_t stream, const RysTable& rys) {
  size_t o_prims, o_recs;
  const size_t total = ip1_image_bytes(W, &o_prims, &o_recs);
  memcpy(host, W.pairs.data(), sizeof(ShellPair) * W.pairs.size());
  if (!W.prims.empty()) memcpy(host + o_prims, W.prims.data(), sizeof(PrimPair) * W.prims.size());
  size_t r0 = 0;
  std::vector<std::pair<const Ip1Work::Key*, std::pair<size_t, size_t>>> launches;
  for (auto& kv : W.groups) {
    memcpy(host + o_recs + sizeof(QuartetRec) * r0, kv.second.data(), sizeof(QuartetRec) * kv.second.size());
    launches.push_back({&kv.first, {r0, kv.second.size()}});
    r0 += kv.second.size();
  }
  cudaError_t e = cudaMemcpyAsync(dev, host, total, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("upload failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  const double cutoff = nsh == 4 ? expcutoff_2e(B.env.data()) : expcutoff_3c(B.env.data());
  for (auto& L : launches) {
    const Ip1Work::Key& k = *L.first;
    Ip1Args a;
    a.pairs = (const ShellPair*)dev;
    a.prims = (const PrimPair*)(dev + o_prims);
    a.out = out_dev;
    a.st.s0 = k.s0;
    a.st.s1 = k.s1;
    a.st.s2 = k.s2;
    a.st.s3 = k.s3;
    a.scomp = k.blk;
    a.expcutoff = cutoff;
    a.rys = rys;
    a.stream = stream;
    const size_t base = L.second.first, cnt = L.second.second;
    for (size_t s0 = 0; s0 < cnt; s0 += (size_t)1 << 30) {
      a.recs = (const QuartetRec*)(dev + o_recs) + base + s0;
      a.nrec = (int)std::min<size_t>(cnt - s0, (size_t)1 << 30);
      e = dispatch_ip1(k.li, k.lj, k.lk, k.ll, sph, a);
      if (e != cudaSuccess) {
        set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("derivative kernel launch failed: ") +
                                                     cudaGetErrorString(e));
        return CINTX_STATUS_EXECUTION_FAILED;
      }
    }
  }
  return CINTX_STATUS_SUCCESS;
}

}  // namespace

// Evaluates n derivative tuples into out (device memory, or host memory when to_host) with the
// thread's scratch buffers; synchronous.  *any receives libcint's return value semantics over all
// tuples (1 if a primitive survived screening).
int ip1_eval(int nsh, double* out, bool to_host, const int* shls, int64_t n, bool sph, bool opt_mode, const int* atm,
             int natm, const int* bas, int nbas, const double* env, int64_t* offsets, bool* any,
             long long* out_doubles) {
  Basis B;
  int rc = load_basis(B, atm, natm, bas, nbas, env);
  if (rc) return rc;
  if (B.env[PTR_RANGE_OMEGA] != 0.0) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "range-separated Coulomb is not supported");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  Ip1Work W;
  if ((rc = ip1_build(B, nsh, shls, n, sph, opt_mode, W, offsets))) return rc;
  if (any) *any = W.any;
  if (out_doubles) *out_doubles = W.out_doubles;
  if (W.groups.empty()) return CINTX_STATUS_SUCCESS;
  size_t o_prims, o_recs;
  size_t image = ip1_image_bytes(W, &o_prims, &o_recs);
  image = (image + 255) & ~(size_t)255;
  const size_t outb = to_host ? sizeof(double) * (size_t)W.out_doubles : 0;
  DeviceState* ds;
  ThreadScratch* ts;
  if ((rc = device_state(&ds)) || (rc = thread_scratch(&ts, image + outb, image + outb))) return rc;
  char* dev = (char*)ts->dbuf;
  char* host = (char*)ts->hbuf;
  double* dout = to_host ? (double*)(dev + image) : out;
  if (to_host) cudaMemsetAsync(dout, 0, outb, ts->stream);
  if ((rc = ip1_launch(W, sph, nsh, B, dev, host, dout, ts->stream, ds->rys))) return rc;
  if (to_host) cudaMemcpyAsync(out, dout, outb, cudaMemcpyDeviceToHost, ts->stream);
  ts->launches += (int64_t)W.groups.size();
  const cudaError_t e = cudaStreamSynchronize(ts->stream);
  if (e != cudaSuccess) {
    set_error(CINTX_STATUS_EXECUTION_FAILED, std::string("device execution failed: ") + cudaGetErrorString(e));
    return CINTX_STATUS_EXECUTION_FAILED;
  }
  return CINTX_STATUS_SUCCESS;
}

}  // namespace cintx

using namespace cintx;

extern "C" {

int cintx_ip1_eval(int family, double* out_dev, const int* shls, int64_t n, int sph, const int* atm, int natm,
                   const int* bas, int nbas, const double* env, int64_t* offsets_out) {
  clear_error();
  if (!out_dev || !shls || n < 0) {
    set_error(CINTX_STATUS_NULL_POINTER, "out_dev and shls must not be NULL and n must be >= 0");
    return CINTX_STATUS_NULL_POINTER;
  }
  if (family != CINTX_INT2E && family != CINTX_INT3C2E) {
    set_error(CINTX_STATUS_UNSUPPORTED_API, "derivative integrals exist for int2e and int3c2e");
    return CINTX_STATUS_UNSUPPORTED_API;
  }
  return ip1_eval(family == CINTX_INT2E ? 4 : 3, out_dev, false, shls, n, sph != 0, true, atm, natm, bas, nbas, env,
                  offsets_out, nullptr, nullptr);
}

// libcint-signature derivative entry points: out == NULL returns a cache size (as libcint's drivers,
// cint2e.c:801-818), dims places each component's block in an array of those extents, the return
// value is 1 if a primitive survived screening (0 and zeros otherwise), screened as libcint screens
// with or without an optimizer (ip1_build); the optimizer's tables themselves are not needed.
static int ip1_call(int nsh, bool sph, double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas,
                    double* env, bool opt_mode) {
  clear_error();
  if (!shls || !atm || !bas || !env) {
    set_error(CINTX_STATUS_NULL_POINTER, "shls, atm, bas and env must not be NULL");
    return 0;
  }
  long long ext[4] = {1, 1, 1, 1}, nf = 1, blk = 1;
  for (int a = 0; a < nsh; ++a) {
    if (shls[a] < 0 || shls[a] >= nbas) {
      set_error(CINTX_STATUS_INVALID_INPUT, "shell index out of range");
      return 0;
    }
    const int l = bas[shls[a] * BAS_SLOTS + ANG_OF], nc = bas[shls[a] * BAS_SLOTS + NCTR_OF];
    ext[a] = (long long)(sph ? 2 * l + 1 : (l + 1) * (l + 2) / 2) * nc;
    nf *= (long long)(l + 1 + (a == 0)) * (l + 2 + (a == 0)) / 2 * nc;
    blk *= ext[a];
  }
  if (!out) return (int)std::min<long long>(3 * blk + 4 * nf, 0x7fffffff);
  bool any = false;
  long long nd = 0;
  std::vector<double> tmp(3 * blk);
  const int rc = ip1_eval(nsh, tmp.data(), true, shls, 1, sph, opt_mode, atm, natm, bas, nbas, env, nullptr, &any,
                          &nd);
  if (rc) return 0;
  if (!any) std::fill(tmp.begin(), tmp.end(), 0.0);
  if (!dims) {
    std::copy(tmp.begin(), tmp.end(), out);
  } else {
    long long full = 1;
    for (int a = 0; a < nsh; ++a) {
      if (dims[a] < ext[a]) {
        set_error(CINTX_STATUS_BUFFER_TOO_SMALL, "dims smaller than the block extents");
        return 0;
      }
      full *= dims[a];
    }
    for (int c = 0; c < 3; ++c)
      for (long long e = 0; e < blk; ++e) {
        long long r = e, off = 0, st = 1;
        for (int a = 0; a < nsh; ++a) {
          off += (r % ext[a]) * st;
          r /= ext[a];
          st *= dims[a];
        }
        out[c * full + off] = tmp[c * blk + e];
      }
  }
  return any ? 1 : 0;
}

int int2e_ip1_sph(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                  CINTOpt* opt, double* cache) {
  (void)cache;
  return ip1_call(4, true, out, dims, shls, atm, natm, bas, nbas, env, opt != nullptr);
}
int int2e_ip1_cart(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                   CINTOpt* opt, double* cache) {
  (void)cache;
  return ip1_call(4, false, out, dims, shls, atm, natm, bas, nbas, env, opt != nullptr);
}
int int3c2e_ip1_sph(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                    CINTOpt* opt, double* cache) {
  (void)cache;
  return ip1_call(3, true, out, dims, shls, atm, natm, bas, nbas, env, opt != nullptr);
}
int int3c2e_ip1_cart(double* out, int* dims, int* shls, int* atm, int natm, int* bas, int nbas, double* env,
                     CINTOpt* opt, double* cache) {
  (void)cache;
  return ip1_call(3, false, out, dims, shls, atm, natm, bas, nbas, env, opt != nullptr);
}
void int2e_ip1_optimizer(CINTOpt** opt, int* atm, int natm, int* bas, int nbas, double* env) {
  int2e_optimizer(opt, atm, natm, bas, nbas, env);
}
void int3c2e_ip1_optimizer(CINTOpt** opt, int* atm, int natm, int* bas, int nbas, double* env) {
  int3c2e_optimizer(opt, atm, natm, bas, nbas, env);
}

}  // extern "C"
