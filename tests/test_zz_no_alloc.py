"""GPU test of cintx_int2e_noalloc, the entry point for callers that cannot call cudaMalloc
(code inside a framework's memory pool, code that already holds nearly all of HBM, code that
must avoid an allocation's device-wide synchronisation).  It is called through the C ABI with
a caller-owned device output buffer, twice in a row on different molecules, and each result is
compared with the batched plan entry point (cintx_plan_shells) within the parity tolerance.
This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import close
from cintx_b200 import molecules as M

pytestmark = pytest.mark.gpu


def _noalloc(lib, out, quartets, mol, sph, stream):
    q = np.ascontiguousarray(quartets, dtype=np.int32)
    atm = np.ascontiguousarray(mol.atm, dtype=np.int32)
    bas = np.ascontiguousarray(mol.bas, dtype=np.int32)
    env = np.ascontiguousarray(mol.env, dtype=np.float64)
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    f = lib.cintx_int2e_noalloc
    f.argtypes = [ctypes.c_void_p, ip, ctypes.c_int64, ctypes.c_int, ip, ctypes.c_int, ip, ctypes.c_int, dp,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f(ctypes.c_void_p(out), q.ctypes.data_as(ip), q.shape[0], int(sph), atm.ctypes.data_as(ip),
             atm.shape[0], bas.ctypes.data_as(ip), bas.shape[0], env.ctypes.data_as(dp), ctypes.c_void_p(stream))


def _reference(cx, mol, quartets, sph):
    with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
        plan = cx.Plan.shells(opt, cx.INT2E, quartets, sph=sph)
        out = plan.execute_host(np.zeros(plan.stats.nintegrals))
        plan.close()
    return out


def test_noalloc_matches_plan_on_two_calls_in_a_row():
    import torch

    import cintx_b200 as cx

    rng = np.random.default_rng(2718)
    cases = [(M.water_like(), rng.integers(0, 12, size=(3000, 4)), True),
             (M.mol40(), rng.integers(0, 168, size=(2000, 4)), True)]
    stream = torch.cuda.Stream()
    for mol, quartets, sph in cases:
        ref = _reference(cx, mol, quartets.astype(np.int32), sph)
        out = torch.full((ref.size,), float("nan"), dtype=torch.float64, device="cuda")
        stream.wait_stream(torch.cuda.current_stream())  # the NaN fill lands before the call's kernels
        rc = _noalloc(cx.lib, out.data_ptr(), quartets, mol, sph, stream.cuda_stream)
        assert rc == 0, cx.last_error()
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert close(got, ref), np.abs(got - ref).max()
    # the entry point's promise: a call takes no device memory (the same work again, after the
    # kernels it launches were loaded by the call above, leaves the device's free bytes unchanged)
    mol, quartets, sph = cases[-1]
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = _noalloc(cx.lib, out.data_ptr(), quartets, mol, sph, stream.cuda_stream)
    stream.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert rc == 0, cx.last_error()
    assert free1 == free0, (free0, free1)
    assert close(out.cpu().numpy(), ref)


def test_noalloc_rejects_calls_beyond_its_scratch():
    import torch

    import cintx_b200 as cx

    mol = M.water_like()
    limit = 32 << 20  # CINTX_NOALLOC_SCRATCH_BYTES
    n = limit // 16 + 1  # one 16-byte record per quartet already exceeds the array
    quartets = np.tile(np.array([[0, 1, 2, 3]], dtype=np.int32), (n, 1))
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = _noalloc(cx.lib, out.data_ptr(), quartets, mol, True, 0)
    assert rc == 5
    code, msg = cx.last_error()
    assert code == 5 and "scratch" in msg
