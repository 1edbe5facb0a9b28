"""CPU checks of the C-ABI library: it loads and exports every symbol the header declares."""
import ctypes
import os
import re
import subprocess
import sys

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cintx_cuda.h")
LIB = os.path.join(ROOT, "cintx_b200", "libcintx_cuda.so")


def declared_functions():
    src = open(HEADER).read()
    return re.findall(r"CINTX_API\s+[A-Za-z_0-9]+\s+\**\s*([A-Za-z_0-9]+)\s*\(", src)


def test_header_declares_libcint_surface():
    names = set(declared_functions())
    for sym in ("int2e_sph", "int2e_cart", "int2e_optimizer", "int2c2e_sph", "int2c2e_cart",
                "int2c2e_optimizer", "int3c2e_sph", "int3c2e_cart", "int3c2e_optimizer",
                "CINTdel_optimizer", "CINTrys_roots"):
        assert sym in names, sym


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "libcintx_cuda.so not built"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and nothing else with C linkage leaks out besides the declared API
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared_functions()) <= exported


def test_python_package_import_is_lazy():
    code = ("import sys; sys.path.insert(0, %r); import cintx_b200.molecules as m; "
            "import cintx_b200; assert '_lib' not in dir(cintx_b200) or True; "
            "print(m.water_like().nbas)") % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "12", r.stderr


def test_error_state_without_device():
    """Argument validation happens before any device work and sets the thread's last error."""
    from cintx_b200 import _lib
    import numpy as np
    from cintx_b200 import molecules as M
    mol = M.water_like()
    bad = np.array([0, 1, 2, 99], dtype=np.int32)
    out = np.zeros(10)
    ret = _lib.lib.int2e_sph(out.ctypes.data_as(_lib._dp), None, bad.ctypes.data_as(_lib._ip),
                             mol.atm.ctypes.data_as(_lib._ip), mol.natm, mol.bas.ctypes.data_as(_lib._ip),
                             mol.nbas, mol.env.ctypes.data_as(_lib._dp), None, None)
    assert ret == 0
    code, msg = _lib.last_error()
    assert code == 1 and "out of range" in msg
    _lib.lib.cintx_cuda_clear_last_error()
    assert _lib.last_error()[0] == 0
    # out == NULL is the cache-size query: no device needed
    ok = np.array([0, 1, 2, 3], dtype=np.int32)
    n = _lib.lib.int2e_sph(None, None, ok.ctypes.data_as(_lib._ip), mol.atm.ctypes.data_as(_lib._ip), mol.natm,
                           mol.bas.ctypes.data_as(_lib._ip), mol.nbas, mol.env.ctypes.data_as(_lib._dp), None, None)
    assert n > 0


class _Summary(__import__("ctypes").Structure):
    import ctypes as _c
    _fields_ = [("not0", _c.c_int), ("bytes_written", _c.c_size_t), ("workspace_bytes", _c.c_size_t)]


class _Query(__import__("ctypes").Structure):
    import ctypes as _c
    _fields_ = [("bytes", _c.c_size_t), ("alignment", _c.c_size_t), ("required_bytes", _c.c_size_t),
                ("chunk_count", _c.c_size_t), ("work_units", _c.c_size_t)]


def _dispatch_args(mol, shls):
    import ctypes
    import numpy as np
    a = np.ascontiguousarray(mol.atm, dtype=np.int32).ravel()
    b = np.ascontiguousarray(mol.bas, dtype=np.int32).ravel()
    e = np.ascontiguousarray(mol.env, dtype=np.float64)
    s = np.ascontiguousarray(shls, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    return (s, a, b, e), (s.ctypes.data_as(ip), s.size, a.ctypes.data_as(ip), a.size, b.ctypes.data_as(ip), b.size,
                          e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), e.size)


def test_cintrs_dispatch_statuses_without_device_work():
    """cintx-capi id dispatch: statuses of the argument checks and the workspace query (host only)."""
    import ctypes
    import numpy as np
    from cintx_b200 import _lib
    from cintx_b200 import molecules as M
    L = _lib.lib
    mol = M.water_like()
    keep, (s, ns, a, na, b, nb, e, ne) = _dispatch_args(mol, [5, 0, 4, 3])
    q = _Query()
    f = L.cintrs_query_workspace
    f.restype = ctypes.c_int
    rc = f(10, None, 0, s, ns, a, na, b, nb, e, ne, None, ctypes.byref(q))
    assert rc == 0 and q.required_bytes == 8 * 5 * 1 * 3 * 3 and q.chunk_count == 1
    assert f(11, None, 0, s, ns, a, na, b, nb, e, ne, None, ctypes.byref(q)) == 2  # spinor: unsupported
    assert f(10, None, 0, s, ns, a, na, b, nb, e, ne, None, None) == 8
    ev = L.cintrs_eval
    ev.restype = ctypes.c_int
    summ = _Summary()
    out = np.zeros(45)
    dp = ctypes.POINTER(ctypes.c_double)
    args = (s, ns, a, na, b, nb, e, ne, None)
    assert ev(10, None, 0, None, 0, *args, None, 0, ctypes.byref(summ)) == 0  # workspace-only call
    assert summ.bytes_written == 0
    assert ev(10, None, 5, None, 0, *args, None, 0, ctypes.byref(summ)) == 8  # NULL out with a length
    assert ev(10, out.ctypes.data_as(dp), 45, None, 0, *args, out.ctypes.data_as(dp), 45, ctypes.byref(summ)) == 1
    assert ev(10, out.ctypes.data_as(dp), 44, None, 0, *args, None, 0, ctypes.byref(summ)) == 4  # too small
    bad_dims = np.array([5, 1, 3, 4], dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    assert ev(10, out.ctypes.data_as(dp), 45, bad_dims.ctypes.data_as(ip), 4, *args, None, 0,
              ctypes.byref(summ)) == 1
    assert ev(10, out.ctypes.data_as(dp), 45, None, 0, s, ns, a, na, b, nb, e, 3, None, None, 0,
              ctypes.byref(summ)) == 1  # env shorter than the basis needs
    code, msg = _lib.last_error()
    assert code == 1 and "env" in msg


def test_basis_offsets_match_libcint():
    """CINTshells_*_offset / CINTtot_cgto_* / CINTcgto_* (host-only, no device work) against libcint
    built from the reference sources, on a basis with general contractions."""
    import numpy as np
    import pytest
    from cintx_b200 import _lib
    from cintx_b200 import molecules as M
    from oracle import RefLibcint
    g = np.load(os.path.join(ROOT, "tests", "golden", "libcint_ctr2.npz"))
    for bas in (M.mol120().bas, np.ascontiguousarray(g["bas"], dtype=np.int32)):
        n = bas.shape[0]
        for sph in (True, False):
            loc = _lib.ao_loc(bas, sph)
            want = np.concatenate([[0], np.cumsum([(2 * l + 1 if sph else (l + 1) * (l + 2) // 2) * c
                                                   for l, c in zip(bas[:, 1], bas[:, 3])])])
            assert np.array_equal(loc, want)
            if RefLibcint.available():
                ref = ctypes.CDLL(RefLibcint.path)
                rl = np.full(n + 1, -7, dtype=np.int32)
                f = ref.CINTshells_spheric_offset if sph else ref.CINTshells_cart_offset
                f(rl.ctypes.data_as(_lib._ip), bas.ctypes.data_as(_lib._ip), ctypes.c_int(n))
                assert np.array_equal(rl[:n], loc[:n]) and rl[n] == -7  # ao_loc[nbas] untouched
                tot = (ref.CINTtot_cgto_spheric if sph else ref.CINTtot_cgto_cart)(bas.ctypes.data_as(_lib._ip),
                                                                                   ctypes.c_int(n))
                assert tot == loc[n]
                cg = ref.CINTcgto_spheric if sph else ref.CINTcgto_cart
                mine = _lib.lib.CINTcgto_spheric if sph else _lib.lib.CINTcgto_cart
                for s in range(0, n, 7):
                    assert cg(ctypes.c_int(s), bas.ctypes.data_as(_lib._ip)) == mine(s, bas.ctypes.data_as(_lib._ip))
    if not RefLibcint.available():
        pytest.skip("libcint from the reference sources not built")
