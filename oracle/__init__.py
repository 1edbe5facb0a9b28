"""CPU oracle for parity tests (TEST INFRASTRUCTURE ONLY).

Two checkers live here and nothing in the product imports them:
  * `Restatement`  - liboracle_cint.so, this folder's own C restatement of libcint's
                     Rys-quadrature integrals (rys_oracle.c, eri_oracle.c, c2s_oracle.c);
  * `RefLibcint`   - _ref/libcint.so, libcint 6.1.3 compiled from the reference sources by
                     this folder's Makefile (present only where the sources were available
                     when the repository was built).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)


def reference_root() -> str:
    """Root of the reference tree whose libcint sources oracle/Makefile compiles: the
    CINTX_REFERENCE_ROOT environment variable, else the Makefile's default mount."""
    return os.environ.get("CINTX_REFERENCE_ROOT", "/root/reference")


def build(ref: bool = True) -> None:
    """Compile the restatement (and libcint from the reference sources when present)."""
    targets = ["liboracle_cint.so"]
    root = reference_root()
    if ref and os.path.isdir(os.path.join(root, "libcint-master")):
        targets += ["ref"]
    subprocess.run(["make", "-s", "-C", HERE, "-j8", "CINTX_REFERENCE_ROOT=" + root] + targets, check=True)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_c_int_p)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_c_dbl_p)


class _Base:
    def _mol(self, mol):
        atm = np.ascontiguousarray(mol.atm, dtype=np.int32)
        bas = np.ascontiguousarray(mol.bas, dtype=np.int32)
        env = np.ascontiguousarray(mol.env, dtype=np.float64)
        return atm, bas, env


class Restatement(_Base):
    def __init__(self):
        path = os.path.join(HERE, "liboracle_cint.so")
        if not os.path.exists(path):
            build(ref=False)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.oracle_rys_t2.argtypes = [ctypes.c_int, ctypes.c_double, _c_dbl_p, _c_dbl_p]
        L.oracle_rys_roots.argtypes = [ctypes.c_int, ctypes.c_double, _c_dbl_p, _c_dbl_p]
        L.oracle_boys.argtypes = [ctypes.c_int, ctypes.c_double, _c_dbl_p]
        L.oracle_c2s_matrix.argtypes = [ctypes.c_int, _c_dbl_p]
        for name in ("oracle_int2e", "oracle_int3c2e", "oracle_int2c2e"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_int, _c_dbl_p, _c_int_p, _c_int_p, ctypes.c_int,
                          _c_int_p, ctypes.c_int, _c_dbl_p]
            f.restype = ctypes.c_int
        L.oracle_int2e_batch.argtypes = [ctypes.c_int, _c_dbl_p, ctypes.POINTER(ctypes.c_longlong),
                                         _c_int_p, ctypes.c_longlong, _c_int_p, ctypes.c_int,
                                         _c_int_p, ctypes.c_int, _c_dbl_p, ctypes.c_int]

    def rys_t2(self, n: int, x: float):
        t2 = np.zeros(n)
        w = np.zeros(n)
        if self.lib.oracle_rys_t2(n, float(x), _dp(t2), _dp(w)):
            raise ValueError("oracle_rys_t2 failed")
        return t2, w

    def rys_roots(self, n: int, x: float):
        u = np.zeros(n)
        w = np.zeros(n)
        if self.lib.oracle_rys_roots(n, float(x), _dp(u), _dp(w)):
            raise ValueError("oracle_rys_roots failed")
        return u, w

    def boys(self, mmax: int, x: float):
        f = np.zeros(mmax + 1)
        self.lib.oracle_boys(mmax, float(x), _dp(f))
        return f

    def c2s(self, l: int):
        nc = (l + 1) * (l + 2) // 2
        m = np.zeros((2 * l + 1, nc))
        self.lib.oracle_c2s_matrix(l, _dp(m))
        return m

    def _call(self, name, sph, shls, mol, size):
        atm, bas, env = self._mol(mol)
        out = np.zeros(size)
        s = np.ascontiguousarray(shls, dtype=np.int32)
        ret = getattr(self.lib, name)(int(sph), _dp(out), _ip(s), _ip(atm), atm.shape[0],
                                      _ip(bas), bas.shape[0], _dp(env))
        return out, ret

    def int2e(self, shls, mol, sph=True):
        n = block_len(mol, shls, sph)
        return self._call("oracle_int2e", sph, shls, mol, n)

    def int3c2e(self, shls, mol, sph=True):
        n = block_len(mol, shls, sph)
        return self._call("oracle_int3c2e", sph, shls, mol, n)

    def int2c2e(self, shls, mol, sph=True):
        n = block_len(mol, shls, sph)
        return self._call("oracle_int2c2e", sph, shls, mol, n)

    def int2e_batch(self, quartets, mol, sph=True, nthreads=0):
        """Blocks of all `quartets` (n x 4 shell ids) concatenated in order."""
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
        sizes = np.array([block_len(mol, r, sph) for r in q], dtype=np.int64)
        offs = np.zeros(len(q), dtype=np.int64)
        offs[1:] = np.cumsum(sizes)[:-1]
        out = np.zeros(int(sizes.sum()))
        atm, bas, env = self._mol(mol)
        self.lib.oracle_int2e_batch(int(sph), _dp(out), offs.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                    _ip(q), len(q), _ip(atm), atm.shape[0], _ip(bas), bas.shape[0],
                                    _dp(env), nthreads)
        return out, offs


class RefLibcint(_Base):
    """libcint 6.1.3 built from the reference sources (oracle/_ref/libcint.so)."""

    path = os.path.join(HERE, "_ref", "libcint.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.path)

    def __init__(self):
        self.lib = ctypes.CDLL(self.path)
        L = self.lib
        for name in ("int2e_sph", "int2e_cart", "int3c2e_sph", "int3c2e_cart",
                     "int2c2e_sph", "int2c2e_cart"):
            f = getattr(L, name)
            f.argtypes = [_c_dbl_p, _c_int_p, _c_int_p, _c_int_p, ctypes.c_int, _c_int_p,
                          ctypes.c_int, _c_dbl_p, ctypes.c_void_p, _c_dbl_p]
            f.restype = ctypes.c_int
        for name in ("int2e_optimizer", "int3c2e_optimizer", "int2c2e_optimizer"):
            f = getattr(L, name)
            f.argtypes = [ctypes.POINTER(ctypes.c_void_p), _c_int_p, ctypes.c_int, _c_int_p,
                          ctypes.c_int, _c_dbl_p]
        L.CINTdel_optimizer.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
        L.CINTrys_roots.argtypes = [ctypes.c_int, ctypes.c_double, _c_dbl_p, _c_dbl_p]
        L.CINTrys_roots.restype = ctypes.c_int

    def rys_roots(self, n: int, x: float):
        u = np.zeros(max(n, 1))
        w = np.zeros(max(n, 1))
        err = self.lib.CINTrys_roots(n, float(x), _dp(u), _dp(w))
        return u, w, err

    def call(self, name, shls, mol, sph=True, opt=None, dims=None):
        atm, bas, env = self._mol(mol)
        n = block_len(mol, shls, sph) if dims is None else int(np.prod(dims))
        out = np.zeros(n)
        s = np.ascontiguousarray(shls, dtype=np.int32)
        d = None if dims is None else np.ascontiguousarray(dims, dtype=np.int32)
        ret = getattr(self.lib, name)(_dp(out), None if d is None else _ip(d), _ip(s), _ip(atm),
                                      atm.shape[0], _ip(bas), bas.shape[0], _dp(env), opt, None)
        return out, ret

    def int2e(self, shls, mol, sph=True):
        return self.call("int2e_sph" if sph else "int2e_cart", shls, mol, sph)

    def int3c2e(self, shls, mol, sph=True):
        return self.call("int3c2e_sph" if sph else "int3c2e_cart", shls, mol, sph)

    def int2c2e(self, shls, mol, sph=True):
        return self.call("int2c2e_sph" if sph else "int2c2e_cart", shls, mol, sph)

    _batch_lib = None

    def batch(self, tuples, mol, sph=True, nthreads=0, ip1=False):
        """Blocks of every tuple (rows of 4, 3 or 2 shell ids: int2e, int3c2e, int2c2e; with ip1
        the first derivatives int2e_ip1 / int3c2e_ip1, three components per block) from libcint,
        concatenated in order (_ref/libcint_batch.so, OpenMP over the tuples).
        Returns (values, offsets[n+1], return values)."""
        if RefLibcint._batch_lib is None:
            L = ctypes.CDLL(os.path.join(HERE, "_ref", "libcint_batch.so"))
            L.ref_batch.argtypes = [ctypes.c_int, ctypes.c_int, _c_dbl_p, ctypes.POINTER(ctypes.c_longlong),
                                    _c_int_p, ctypes.c_longlong, _c_int_p, ctypes.c_int, _c_int_p, ctypes.c_int,
                                    _c_dbl_p, ctypes.c_int, _c_int_p]
            L.ref_batch.restype = ctypes.c_int
            RefLibcint._batch_lib = L
        t = np.ascontiguousarray(tuples, dtype=np.int32)
        fam = t.shape[1] * 10 + 1 if ip1 else t.shape[1]
        atm, bas, env = self._mol(mol)
        l = bas[:, 1].astype(np.int64)
        nc = bas[:, 3].astype(np.int64)
        per = (2 * l + 1 if sph else (l + 1) * (l + 2) // 2) * nc
        sizes = np.prod(per[t], axis=1) * (3 if ip1 else 1) if len(t) else np.zeros(0, dtype=np.int64)
        offs = np.zeros(len(t) + 1, dtype=np.int64)
        offs[1:] = np.cumsum(sizes)
        out = np.zeros(int(offs[-1]))
        rets = np.zeros(len(t), dtype=np.int32)
        if len(t):
            rc = RefLibcint._batch_lib.ref_batch(fam, int(sph), _dp(out),
                                                 offs.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _ip(t),
                                                 len(t), _ip(atm), atm.shape[0], _ip(bas), bas.shape[0], _dp(env),
                                                 int(nthreads), _ip(rets))
            if rc:
                raise MemoryError("ref_batch: cache allocation failed")
        return out, offs, rets


def block_len(mol, shls, sph=True) -> int:
    n = 1
    for s in shls:
        l = int(mol.bas[s, 1])
        nc = int(mol.bas[s, 3])
        n *= (2 * l + 1 if sph else (l + 1) * (l + 2) // 2) * nc
    return n
