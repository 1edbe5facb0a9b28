"""ctypes binding of libcintx_cuda.so (declarations in include/cintx_cuda.h)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcintx_cuda.so")

_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


class CintxError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("cintx status %d: %s" % (code, message))
        self.code = code


class PlanStats(ctypes.Structure):
    _fields_ = [("nquartets", _i64), ("nintegrals", _i64), ("nchunks", _i64),
                ("max_chunk_doubles", _i64), ("nprim_quartets", _i64), ("device_bytes", _i64),
                ("nquartets_fp32", _i64), ("flops", _d)]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError("libcintx_cuda.so is not built (run python -m cintx_b200.build or "
                          "__graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    sig = [_dp, _ip, _ip, _ip, _i, _ip, _i, _dp, _vp, _dp]
    for name in ("int2e_sph", "int2e_cart", "int3c2e_sph", "int3c2e_cart", "int2c2e_sph", "int2c2e_cart"):
        f = getattr(L, name)
        f.argtypes = sig
        f.restype = _i
    for name in ("int2e_ip1_sph", "int2e_ip1_cart", "int3c2e_ip1_sph", "int3c2e_ip1_cart"):
        f = getattr(L, name)
        f.argtypes = sig
        f.restype = _i
    L.cintx_ip1_eval.argtypes = [_i, _vp, _ip, _i64, _i, _ip, _i, _ip, _i, _dp, _i64p]
    L.cintx_ip1_eval.restype = _i
    for name in ("int2e_optimizer", "int3c2e_optimizer", "int2c2e_optimizer", "int2e_ip1_optimizer",
                 "int3c2e_ip1_optimizer"):
        f = getattr(L, name)
        f.argtypes = [ctypes.POINTER(_vp), _ip, _i, _ip, _i, _dp]
        f.restype = None
    L.CINTdel_optimizer.argtypes = [ctypes.POINTER(_vp)]
    L.CINTdel_optimizer.restype = None
    L.CINTrys_roots.argtypes = [_i, _d, _dp, _dp]
    L.CINTrys_roots.restype = _i
    L.cintx_rys_t2_batch.argtypes = [_i, _dp, _i64, _dp]
    L.cintx_rys_t2_batch.restype = _i
    L.cintx_cuda_last_error_code.restype = _i
    L.cintx_cuda_last_error_message.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.cintx_cuda_last_error_message.restype = ctypes.c_size_t
    L.cintx_cuda_clear_last_error.restype = None
    L.cintx_plan_shells.argtypes = [ctypes.POINTER(_vp), _vp, _i, _ip, _i64, _i, _i64p]
    L.cintx_plan_shells.restype = _i
    L.cintx_plan_int2e_screened.argtypes = [ctypes.POINTER(_vp), _vp, _d, _i, _i64]
    L.cintx_plan_int2e_screened.restype = _i
    L.cintx_plan_int2e_screened_mixed.argtypes = [ctypes.POINTER(_vp), _vp, _d, _i, _i64, _d, _d]
    L.cintx_plan_int2e_screened_mixed.restype = _i
    _sz = ctypes.c_size_t
    L.cintrs_query_workspace.argtypes = [_i, _ip, _sz, _ip, _sz, _ip, _sz, _ip, _sz, _dp, _sz, _vp, _vp]
    L.cintrs_query_workspace.restype = _i
    L.cintrs_eval.argtypes = [_i, _dp, _sz, _ip, _sz, _ip, _sz, _ip, _sz, _ip, _sz, _dp, _sz, _vp, _dp, _sz, _vp]
    L.cintrs_eval.restype = _i
    L.cintx_optimizer_pair_shells.argtypes = [ctypes.POINTER(_vp), _ip, _i, _ip, _i, _dp, _i]
    L.cintx_optimizer_pair_shells.restype = _i
    L.cintx_plan_int3c2e_screened.argtypes = [ctypes.POINTER(_vp), _vp, _d, _i, _i64, _i]
    L.cintx_plan_int3c2e_screened.restype = _i
    L.cintx_plan_stats.argtypes = [_vp, ctypes.POINTER(PlanStats)]
    L.cintx_plan_stats.restype = _i
    L.cintx_plan_chunk_size.argtypes = [_vp, _i64]
    L.cintx_plan_chunk_size.restype = _i64
    L.cintx_plan_chunk_nquartets.argtypes = [_vp, _i64]
    L.cintx_plan_chunk_nquartets.restype = _i64
    L.cintx_plan_chunk_quartets.argtypes = [_vp, _i64, _ip, _i64]
    L.cintx_plan_chunk_quartets.restype = _i
    L.cintx_plan_execute.argtypes = [_vp, _i64, _vp, _vp]
    L.cintx_plan_execute.restype = _i
    L.cintx_plan_execute_host.argtypes = [_vp, _i64, _dp]
    L.cintx_plan_execute_host.restype = _i
    L.cintx_plan_execute_host_ring.argtypes = [_vp, _dp, _i64, ctypes.c_void_p, ctypes.c_void_p]
    L.cintx_plan_execute_host_ring.restype = _i
    L.cintx_plan_execute_s8.argtypes = [_vp, _vp, _i64, _vp]
    L.cintx_plan_execute_s8.restype = _i
    L.cintx_plan_execute_ao.argtypes = [_vp, _i, _vp, _i64, _vp]
    L.cintx_plan_execute_ao.restype = _i
    for name in ("CINTcgto_cart", "CINTcgto_spheric"):
        getattr(L, name).argtypes = [_i, _ip]
        getattr(L, name).restype = _i
    for name in ("CINTtot_cgto_spheric", "CINTtot_cgto_cart"):
        getattr(L, name).argtypes = [_ip, _i]
        getattr(L, name).restype = _i
    for name in ("CINTshells_spheric_offset", "CINTshells_cart_offset"):
        getattr(L, name).argtypes = [_ip, _ip, _i]
        getattr(L, name).restype = None
    L.cintx_plan_jk.argtypes = [_vp, _vp, _i, _vp, _vp, _vp]
    L.cintx_plan_jk.restype = _i
    L.cintx_plan_autotune.argtypes = [_vp, _i64, ctypes.c_void_p, ctypes.c_void_p, _i]
    L.cintx_plan_autotune.restype = _i
    L.cintx_plan_use_tuned_shapes.argtypes = [_vp]
    L.cintx_plan_use_tuned_shapes.restype = _i
    L.cintx_plan_set_shape.argtypes = [_vp, _i]
    L.cintx_plan_set_shape.restype = _i
    L.cintx_tuned_shapes_export.argtypes = [_ip, _i]
    L.cintx_tuned_shapes_export.restype = _i
    L.cintx_tuned_shapes_import.argtypes = [_ip, _i]
    L.cintx_tuned_shapes_import.restype = _i
    L.cintx_plan_segment_lanes.argtypes = [_vp, _i64, _ip, _i]
    L.cintx_plan_segment_lanes.restype = _i
    L.cintx_plan_destroy.argtypes = [_vp]
    L.cintx_plan_destroy.restype = None
    L.cintx_launch_count.restype = _i64
    L.cintx_plan_chunk_segments.argtypes = [_vp, _i64, _ip, _i64p, _dp, _i]
    L.cintx_plan_chunk_segments.restype = _i
    L.cintx_plan_execute_segment.argtypes = [_vp, _i64, _i, _vp, _vp]
    L.cintx_plan_execute_segment.restype = _i
    L.cintx_plan_sample_quartets.argtypes = [_vp, ctypes.c_uint64, _i64, _ip]
    L.cintx_plan_sample_quartets.restype = _i
    L.cintx_plan_graph_build.argtypes = [_vp, _i64p, _i64, _vp, _i]
    L.cintx_plan_graph_build.restype = _i
    L.cintx_plan_graph_launch.argtypes = [_vp, _vp]
    L.cintx_plan_graph_launch.restype = _i
    L.cintx_opt_device_bytes.argtypes = [_vp]
    L.cintx_opt_device_bytes.restype = _i64
    _fp = ctypes.POINTER(ctypes.c_float)
    L.cintx_rysnet_samples.argtypes = [_i64, _i, _i, ctypes.c_uint64, _fp, _fp, _ip, _dp]
    L.cintx_rysnet_samples.restype = _i
    L.cintx_rysnet_loss_grad.argtypes = [_fp, _fp, _fp, _ip, _i64, _fp, _dp]
    L.cintx_rysnet_loss_grad.restype = _i
    L.cintx_rysnet_train.argtypes = [_fp, _i64, _i, _i, _i, _i, ctypes.c_float, ctypes.c_uint64, _dp]
    L.cintx_rysnet_train.restype = _i
    L.cintx_plan_use_learned_roots.argtypes = [_vp, _fp, _i64p, _i64p]
    L.cintx_plan_use_learned_roots.restype = _i
    L.cintx_rys_learned_batch.argtypes = [_fp, _i, _dp, _i64, _i, _dp, _ip, _ip]
    L.cintx_rys_learned_batch.restype = _i
    L.cintx_fp64_fma_probe.argtypes = [_i, _i, _i, _vp, _vp]
    L.cintx_fp64_fma_probe.restype = _i
    return L


lib = _load()


def last_error() -> tuple[int, str]:
    buf = ctypes.create_string_buffer(1024)
    lib.cintx_cuda_last_error_message(buf, 1024)
    return lib.cintx_cuda_last_error_code(), buf.value.decode()


def _check(code: int):
    if code != 0:
        c, m = last_error()
        raise CintxError(code, m)


def launch_count() -> int:
    return int(lib.cintx_launch_count())


def _arrs(atm, bas, env):
    atm = np.ascontiguousarray(atm, dtype=np.int32)
    bas = np.ascontiguousarray(bas, dtype=np.int32)
    env = np.ascontiguousarray(env, dtype=np.float64)
    return atm, bas, env


def _block_len(bas, shls, sph):
    n = 1
    for s in shls:
        l, nc = int(bas[s, 1]), int(bas[s, 3])
        n *= (2 * l + 1 if sph else (l + 1) * (l + 2) // 2) * nc
    return n


def _call(name, nsh, shls, atm, bas, env, opt=None, dims=None, out=None, sph=True, ncomp=1):
    atm, bas, env = _arrs(atm, bas, env)
    s = np.ascontiguousarray(shls, dtype=np.int32)
    assert s.size == nsh
    if out is None:
        n = _block_len(bas, s, sph) if dims is None else int(np.prod(dims))
        out = np.zeros(n * ncomp)
    d = None if dims is None else np.ascontiguousarray(dims, dtype=np.int32)
    ret = getattr(lib, name)(out.ctypes.data_as(_dp), None if d is None else d.ctypes.data_as(_ip),
                             s.ctypes.data_as(_ip), atm.ctypes.data_as(_ip), atm.shape[0],
                             bas.ctypes.data_as(_ip), bas.shape[0], env.ctypes.data_as(_dp),
                             None if opt is None else opt.handle, None)
    code = lib.cintx_cuda_last_error_code()
    if code:
        raise CintxError(code, last_error()[1])
    return out, ret


def int2e_sph(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int2e_sph", 4, shls, atm, bas, env, opt, dims, out, True)


def int2e_cart(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int2e_cart", 4, shls, atm, bas, env, opt, dims, out, False)


def int3c2e_sph(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int3c2e_sph", 3, shls, atm, bas, env, opt, dims, out, True)


def int3c2e_cart(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int3c2e_cart", 3, shls, atm, bas, env, opt, dims, out, False)


def int2c2e_sph(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int2c2e_sph", 2, shls, atm, bas, env, opt, dims, out, True)


def int2c2e_cart(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int2c2e_cart", 2, shls, atm, bas, env, opt, dims, out, False)


def ao_loc(bas, sph: bool = True) -> np.ndarray:
    """AO offsets of the shells (nbas + 1 entries, the last one the total), from the library's
    CINTshells_spheric_offset / CINTshells_cart_offset and CINTtot_cgto_*."""
    b = np.ascontiguousarray(bas, dtype=np.int32)
    n = b.shape[0]
    loc = np.zeros(n + 1, dtype=np.int32)
    (lib.CINTshells_spheric_offset if sph else lib.CINTshells_cart_offset)(loc.ctypes.data_as(_ip),
                                                                           b.ctypes.data_as(_ip), n)
    loc[n] = (lib.CINTtot_cgto_spheric if sph else lib.CINTtot_cgto_cart)(b.ctypes.data_as(_ip), n)
    return loc


def int2e_ip1_sph(shls, atm, bas, env, opt=None, dims=None, out=None):
    """(nabla i j|k l): three components, each a block in int2e_sph's layout, one after the other."""
    return _call("int2e_ip1_sph", 4, shls, atm, bas, env, opt, dims, out, True, 3)


def int2e_ip1_cart(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int2e_ip1_cart", 4, shls, atm, bas, env, opt, dims, out, False, 3)


def int3c2e_ip1_sph(shls, atm, bas, env, opt=None, dims=None, out=None):
    """(nabla i j|k): three components, each a block in int3c2e_sph's layout."""
    return _call("int3c2e_ip1_sph", 3, shls, atm, bas, env, opt, dims, out, True, 3)


def int3c2e_ip1_cart(shls, atm, bas, env, opt=None, dims=None, out=None):
    return _call("int3c2e_ip1_cart", 3, shls, atm, bas, env, opt, dims, out, False, 3)


def ip1_eval(family: int, tuples, atm, bas, env, out_ptr: int, sph: bool = True) -> np.ndarray:
    """First derivatives of a tuple list (family INT2E: 4 shells each, INT3C2E: 3) into the device
    buffer at out_ptr (cintx_ip1_eval); returns each tuple's block offset."""
    atm, bas, env = _arrs(atm, bas, env)
    t = np.ascontiguousarray(tuples, dtype=np.int32)
    n = t.shape[0]
    offs = np.zeros(n, dtype=np.int64)
    _check(lib.cintx_ip1_eval(family, ctypes.c_void_p(out_ptr), t.ctypes.data_as(_ip), n, int(sph),
                              atm.ctypes.data_as(_ip), atm.shape[0], bas.ctypes.data_as(_ip), bas.shape[0],
                              env.ctypes.data_as(_dp), offs.ctypes.data_as(_i64p)))
    return offs


def ip1_len(family: int, tuples, bas, sph: bool = True) -> int:
    """Doubles a cintx_ip1_eval output of these tuples holds (3 components per block)."""
    b = np.asarray(bas)
    l, nc = b[:, 1].astype(np.int64), b[:, 3].astype(np.int64)
    per = (2 * l + 1 if sph else (l + 1) * (l + 2) // 2) * nc
    t = np.asarray(tuples)
    return int(3 * np.prod(per[t], axis=1).sum())


def tuned_shapes() -> list:
    """The autotuner's launch-shape choices on the current device: [li, lj, lk, ll, fp32, variant]
    records (cintx_tuned_shapes_export), e.g. to save and reload in a later process."""
    n = lib.cintx_tuned_shapes_export(None, 0)
    rec = np.zeros((max(n, 1), 6), dtype=np.int32)
    lib.cintx_tuned_shapes_export(rec.ctypes.data_as(_ip), n)
    return rec[:n].tolist()


def load_tuned_shapes(records) -> None:
    """Adds saved launch-shape choices for the current device (cintx_tuned_shapes_import); plans
    pick them up with Plan.use_tuned_shapes()."""
    rec = np.ascontiguousarray(np.asarray(records, dtype=np.int32).reshape(-1, 6))
    _check(lib.cintx_tuned_shapes_import(rec.ctypes.data_as(_ip), rec.shape[0]))


def rys_roots(n: int, x: float):
    """libcint CINTrys_roots convention: u = t^2/(1-t^2) and weights."""
    u = np.zeros(n)
    w = np.zeros(n)
    _check(lib.CINTrys_roots(n, float(x), u.ctypes.data_as(_dp), w.ctypes.data_as(_dp)))
    return u, w


def rys_t2_batch(n: int, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros((x.size, 2 * n))
    _check(lib.cintx_rys_t2_batch(n, x.ctypes.data_as(_dp), x.size, out.ctypes.data_as(_dp)))
    return out[:, :n], out[:, n:]


class Optimizer:
    """Owns a CINTOpt handle (device-resident basis and primitive-pair tables)."""

    _makers = {0: "int2e_optimizer", 1: "int3c2e_optimizer", 2: "int2c2e_optimizer"}

    def __init__(self, atm, bas, env, family: int = 0, pair_shells: int | None = None):
        """pair_shells: build shell pairs only among the first pair_shells shells (orbital shells
        of a density-fitting basis; cintx_optimizer_pair_shells)."""
        self.atm, self.bas, self.env = _arrs(atm, bas, env)
        self.handle = _vp()
        args = (ctypes.byref(self.handle), self.atm.ctypes.data_as(_ip), self.atm.shape[0],
                self.bas.ctypes.data_as(_ip), self.bas.shape[0], self.env.ctypes.data_as(_dp))
        if pair_shells is None:
            getattr(lib, self._makers[family])(*args)
        else:
            lib.cintx_optimizer_pair_shells(*args, int(pair_shells))
        if not self.handle:
            raise CintxError(*last_error())

    @property
    def device_bytes(self) -> int:
        return int(lib.cintx_opt_device_bytes(self.handle))

    def close(self):
        if self.handle:
            lib.CINTdel_optimizer(ctypes.byref(self.handle))
            self.handle = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A batched device evaluation plan (cintx_plan_* in include/cintx_cuda.h)."""

    def __init__(self, handle, opt: Optimizer, offsets=None):
        self.handle = handle
        self.opt = opt  # keeps the optimizer alive
        self.offsets = offsets

    @classmethod
    def shells(cls, opt: Optimizer, family: int, tuples, sph: bool = True):
        t = np.ascontiguousarray(tuples, dtype=np.int32)
        nsh = 4 if family == 0 else (3 if family == 1 else 2)
        t = t.reshape(-1, nsh)
        offs = np.zeros(t.shape[0], dtype=np.int64)
        h = _vp()
        _check(lib.cintx_plan_shells(ctypes.byref(h), opt.handle, family, t.ctypes.data_as(_ip), t.shape[0],
                                     int(sph), offs.ctypes.data_as(_i64p)))
        return cls(h, opt, offs)

    @classmethod
    def screened(cls, opt: Optimizer, cutoff: float = 1e-12, sph: bool = True, max_chunk_doubles: int = 1 << 28):
        h = _vp()
        _check(lib.cintx_plan_int2e_screened(ctypes.byref(h), opt.handle, float(cutoff), int(sph),
                                             int(max_chunk_doubles)))
        return cls(h, opt)

    @classmethod
    def screened_mixed(cls, opt: Optimizer, cutoff: float = 1e-12, fp32_budget: float = 0.0,
                       prim_budget: float = 5e-11, max_chunk_doubles: int = 1 << 28):
        """Tuned sweep: primitive Schwarz screening within prim_budget per integral and, when
        fp32_budget > 0, FP32 recurrences for quartets whose estimated FP32 error (primitive-
        absolute Schwarz bound times the recurrences' cancellation factor) is below fp32_budget."""
        h = _vp()
        _check(lib.cintx_plan_int2e_screened_mixed(ctypes.byref(h), opt.handle, float(cutoff), 1,
                                                   int(max_chunk_doubles), float(fp32_budget),
                                                   float(prim_budget)))
        return cls(h, opt)

    @classmethod
    def screened_3c(cls, opt: Optimizer, norb: int, cutoff: float = 1e-12, sph: bool = True,
                    max_chunk_doubles: int = 1 << 28):
        """Density-fitting sweep: (ab|k) over orbital pairs a >= b < norb and auxiliary shells
        k >= norb with Schwarz bound >= cutoff (cintx_plan_int3c2e_screened)."""
        h = _vp()
        _check(lib.cintx_plan_int3c2e_screened(ctypes.byref(h), opt.handle, float(cutoff), int(sph),
                                               int(max_chunk_doubles), int(norb)))
        return cls(h, opt)

    @property
    def stats(self) -> PlanStats:
        s = PlanStats()
        _check(lib.cintx_plan_stats(self.handle, ctypes.byref(s)))
        return s

    def chunk_size(self, chunk: int) -> int:
        return int(lib.cintx_plan_chunk_size(self.handle, chunk))

    def chunk_quartets(self, chunk: int) -> np.ndarray:
        n = int(lib.cintx_plan_chunk_nquartets(self.handle, chunk))
        q = np.zeros((max(n, 0), 4), dtype=np.int32)
        _check(lib.cintx_plan_chunk_quartets(self.handle, chunk, q.ctypes.data_as(_ip), n))
        return q

    def segments(self, chunk: int):
        n = lib.cintx_plan_chunk_segments(self.handle, chunk, None, None, None, 0)
        cls = np.zeros((max(n, 0), 4), dtype=np.int32)
        nq = np.zeros(max(n, 0), dtype=np.int64)
        fl = np.zeros(max(n, 0))
        lib.cintx_plan_chunk_segments(self.handle, chunk, cls.ctypes.data_as(_ip), nq.ctypes.data_as(_i64p),
                                      fl.ctypes.data_as(_dp), n)
        return cls, nq, fl

    def execute_segment(self, out_ptr: int, chunk: int, seg: int, stream: int = 0):
        _check(lib.cintx_plan_execute_segment(self.handle, chunk, seg, ctypes.c_void_p(out_ptr),
                                              ctypes.c_void_p(stream)))

    def sample_quartets(self, n: int, seed: int = 0) -> np.ndarray:
        q = np.zeros((n, 4), dtype=np.int32)
        _check(lib.cintx_plan_sample_quartets(self.handle, seed, n, q.ctypes.data_as(_ip)))
        return q

    def use_learned_roots(self, net: "RysNet | None"):
        """Explicit plans: take Rys roots from the learned initializer + FP64 refinement (None:
        the table again).  Returns (fallback count, primitive quartets)."""
        fb = ctypes.c_int64()
        npt = ctypes.c_int64()
        params = None if net is None else net.params.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        _check(lib.cintx_plan_use_learned_roots(self.handle, params, ctypes.byref(fb), ctypes.byref(npt)))
        return fb.value, npt.value

    def execute(self, out_ptr: int, chunk: int = -1, stream: int = 0):
        """Asynchronous device execution into device pointer out_ptr."""
        _check(lib.cintx_plan_execute(self.handle, chunk, ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)))

    def graph_build(self, out_ptr: int, chunks=None, nbranch: int = 4):
        if chunks is None:
            _check(lib.cintx_plan_graph_build(self.handle, None, 0, ctypes.c_void_p(out_ptr), nbranch))
        else:
            c = np.ascontiguousarray(chunks, dtype=np.int64)
            _check(lib.cintx_plan_graph_build(self.handle, c.ctypes.data_as(_i64p), c.size,
                                              ctypes.c_void_p(out_ptr), nbranch))

    def autotune(self, out_ptr: int, chunk: int = -1, stream: int = 0, reps: int = 2):
        """Pick each kernel class's fastest launch shape by timing it on `chunk` (-1: each class
        on its largest segment in the plan).  Synchronous; a captured graph is released and must
        be built again."""
        _check(lib.cintx_plan_autotune(self.handle, chunk, ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream), reps))

    def jk(self, dm_ptr: int, nao: int, vj_ptr: int = 0, vk_ptr: int = 0, stream: int = 0):
        """Coulomb (vj) and exchange (vk) matrices for the symmetric density at dm_ptr (device
        pointers, row-major nao x nao; 0 skips an output).  Asynchronous on stream."""
        _check(lib.cintx_plan_jk(self.handle, ctypes.c_void_p(dm_ptr), int(nao), ctypes.c_void_p(vj_ptr or None),
                                 ctypes.c_void_p(vk_ptr or None), ctypes.c_void_p(stream)))

    def execute_s8(self, eri_ptr: int, length: int, stream: int = 0):
        """The sweep as the 8-fold packed AO tensor at device pointer eri_ptr (length doubles)."""
        _check(lib.cintx_plan_execute_s8(self.handle, ctypes.c_void_p(eri_ptr), int(length), ctypes.c_void_p(stream)))

    def execute_ao(self, eri_ptr: int, length: int, aosym: int = 1, stream: int = 0):
        """The sweep as an AO-indexed tensor at device pointer eri_ptr (length doubles): aosym 1 the
        full nao^4 tensor, 4 the npair x npair pair matrix, 8 the 8-fold packed triangle."""
        _check(lib.cintx_plan_execute_ao(self.handle, int(aosym), ctypes.c_void_p(eri_ptr), int(length),
                                         ctypes.c_void_p(stream)))

    def use_tuned_shapes(self) -> int:
        """Reuse the launch shapes autotuned earlier in this process; returns segments changed."""
        n = lib.cintx_plan_use_tuned_shapes(self.handle)
        if n < 0:
            _check(1)
        return n

    def set_shape(self, variant: int) -> int:
        """Runs every segment in launch-shape variant `variant` (0 = default shape)."""
        n = lib.cintx_plan_set_shape(self.handle, variant)
        if n < 0:
            _check(last_error()[0])
        return n

    def segment_lanes(self, chunk: int) -> np.ndarray:
        n = lib.cintx_plan_segment_lanes(self.handle, chunk, None, 0)
        out = np.zeros(max(n, 0), dtype=np.int32)
        lib.cintx_plan_segment_lanes(self.handle, chunk, out.ctypes.data_as(_ip), n)
        return out

    def graph_launch(self, stream: int = 0):
        _check(lib.cintx_plan_graph_launch(self.handle, ctypes.c_void_p(stream)))

    def execute_host(self, out: np.ndarray, chunk: int = -1):
        """Evaluate one chunk (or all, chunks back to back) into host array `out`."""
        if out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array")
        need = self.stats.nintegrals if chunk < 0 else self.chunk_size(chunk)
        if out.size < need:
            raise ValueError("out holds %d doubles, the output needs %d" % (out.size, need))
        _check(lib.cintx_plan_execute_host(self.handle, chunk, out.ctypes.data_as(_dp)))
        return out

    _CHUNK_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int64, _dp, ctypes.c_int64)

    def execute_host_ring(self, ring: np.ndarray, on_chunk=None):
        """Evaluate every chunk through a two-slot host ring (ring.size >= 2 x max chunk);
        on_chunk(chunk, array_view) is called for each chunk in order before its slot is reused."""
        if ring.dtype != np.float64 or not ring.flags.c_contiguous:
            raise ValueError("ring must be a C-contiguous float64 array")
        cb = None
        if on_chunk is not None:
            def _cb(_user, chunk, data, n):
                on_chunk(int(chunk), np.ctypeslib.as_array(data, shape=(int(n),)))
            cb = self._CHUNK_CB(_cb)
        _check(lib.cintx_plan_execute_host_ring(self.handle, ring.ctypes.data_as(_dp), ring.size,
                                                ctypes.cast(cb, ctypes.c_void_p) if cb else None, None))
        return ring

    def close(self):
        if self.handle:
            lib.cintx_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_fp32p = ctypes.POINTER(ctypes.c_float)


class RysNet:
    """Learned Rys-root initializer (include/cintx_cuda.h, cintx_rysnet_*): an FP32 MLP trained
    on the device from the table path, whose guess an FP64 refinement turns into roots and
    weights at full accuracy (table-path fallback where the refinement fails its checks)."""

    NPARAM = 5522
    SHAPES = [(64, 2), (64,), (64, 64), (64,), (18, 64), (18,)]

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        self.params = np.ascontiguousarray(params if params is not None else self.init(seed), dtype=np.float32)
        assert self.params.size == self.NPARAM

    @classmethod
    def init(cls, seed: int = 0) -> np.ndarray:
        """Glorot-uniform weights, zero biases."""
        rng = np.random.default_rng(seed)
        parts = []
        for shp in cls.SHAPES:
            if len(shp) == 2:
                lim = np.sqrt(6.0 / (shp[0] + shp[1]))
                parts.append(rng.uniform(-lim, lim, size=shp).ravel())
            else:
                parts.append(np.zeros(shp))
        return np.concatenate(parts).astype(np.float32)

    @staticmethod
    def samples(count: int, n_lo: int = 5, n_hi: int = 9, seed: int = 0):
        feat = np.zeros((count, 2), dtype=np.float32)
        tgt = np.zeros((count, 18), dtype=np.float32)
        nr = np.zeros(count, dtype=np.int32)
        x = np.zeros(count)
        _check(lib.cintx_rysnet_samples(count, n_lo, n_hi, seed, feat.ctypes.data_as(_fp32p),
                                        tgt.ctypes.data_as(_fp32p), nr.ctypes.data_as(_ip), x.ctypes.data_as(_dp)))
        return feat, tgt, nr, x

    def loss_grad(self, feat, tgt, nroots):
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        tgt = np.ascontiguousarray(tgt, dtype=np.float32)
        nr = np.ascontiguousarray(nroots, dtype=np.int32)
        grad = np.zeros(self.NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        _check(lib.cintx_rysnet_loss_grad(self.params.ctypes.data_as(_fp32p), feat.ctypes.data_as(_fp32p),
                                          tgt.ctypes.data_as(_fp32p), nr.ctypes.data_as(_ip), nr.size,
                                          grad.ctypes.data_as(_fp32p), ctypes.byref(loss)))
        return loss.value, grad

    def train(self, nsamples: int = 5_000_000, n_lo: int = 5, n_hi: int = 9, epochs: int = 20,
              batch: int = 16384, lr: float = 3e-3, seed: int = 1) -> np.ndarray:
        hist = np.zeros(epochs)
        _check(lib.cintx_rysnet_train(self.params.ctypes.data_as(_fp32p), nsamples, n_lo, n_hi, epochs, batch,
                                      lr, seed, hist.ctypes.data_as(_dp)))
        return hist

    def roots(self, n: int, x, mode: int = 0):
        """(t2, w, status, iters) for order n at points x; mode 0 network + refinement, 1 the
        refinement from the x = 0 roots (no network), 2 the network's guess unrefined."""
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        out = np.zeros((x.size, 2 * n))
        st = np.zeros(x.size, dtype=np.int32)
        it = np.zeros(x.size, dtype=np.int32)
        _check(lib.cintx_rys_learned_batch(self.params.ctypes.data_as(_fp32p), n, x.ctypes.data_as(_dp), x.size,
                                           mode, out.ctypes.data_as(_dp), st.ctypes.data_as(_ip),
                                           it.ctypes.data_as(_ip)))
        return out[:, :n], out[:, n:], st, it
