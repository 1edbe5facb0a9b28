"""GPU parity of the first-derivative integrals int2e_ip1 / int3c2e_ip1 (libcint autocode/grad2.c,
autocode/int3c2e.c) against libcint 6.1.3 built from the reference sources: golden blocks of the
3-atom molecule (sph, cart), the 40-atom molecule and the 3-atom molecule with its g-containing
auxiliary basis, through the per-call libcint signatures, the batched device entry point and the
cintx-capi id dispatch; and a live-libcint sample of f-shell derivative quartets of the 120-atom
molecule.  Tolerance: the reference's parity rule, |d| <= 1e-12 or |d| <= 1e-10 |ref|."""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT, close
from cintx_b200 import molecules as M
from oracle import RefLibcint

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden", "libcint_ip1.npz")


@pytest.fixture(scope="module")
def cx():
    import cintx_b200
    return cintx_b200


def _cases():
    w = M.water_like()
    wa = M.with_aux(w)
    return [("water3_int2e_ip1_sph", w, "int2e_ip1_sph"), ("water3_int2e_ip1_cart", w, "int2e_ip1_cart"),
            ("mol40_int2e_ip1_sph", M.mol40(), "int2e_ip1_sph"),
            ("water3aux_int3c2e_ip1_sph", wa, "int3c2e_ip1_sph"),
            ("water3aux_int3c2e_ip1_cart", wa, "int3c2e_ip1_cart")]


def test_per_call_derivatives_match_libcint_goldens(cx):
    """The goldens come from libcint with an optimizer (its screening raises every pair's estimate by
    the derivative order), so the per-call path runs with one too."""
    g = np.load(GOLD)
    for name, mol, fn in _cases():
        tup, offs, vals, rets = (g[name + k] for k in ("_tuples", "_offsets", "_values", "_ret"))
        with cx.Optimizer(mol.atm, mol.bas, mol.env) as opt:
            for q, t in enumerate(tup):
                out, ret = getattr(cx, fn)(t, mol.atm, mol.bas, mol.env, opt=opt)
                ref = vals[offs[q]:offs[q + 1]]
                assert ret == rets[q], (name, t)
                assert out.size == ref.size and close(out, ref), (name, t, np.abs(out - ref).max())


@pytest.mark.skipif(not RefLibcint.available(), reason="libcint from the reference sources not built")
def test_per_call_without_optimizer_screens_like_libcint(cx):
    """Without an optimizer libcint raises only the differentiated pair's screening estimate
    (CINT2e_loop_nopt): return values and blocks against live libcint without one."""
    mol = M.mol40()
    ref = RefLibcint()
    f = ref.lib.int2e_ip1_sph
    rng = np.random.default_rng(77)
    atm, bas, env = (np.ascontiguousarray(a) for a in (mol.atm, mol.bas, mol.env))
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    for t in list(rng.integers(0, mol.nbas, size=(120, 4))) + [np.array([80, 84, 27, 120])]:
        t = np.ascontiguousarray(t, dtype=np.int32)
        out, ret = cx.int2e_ip1_sph(t, mol.atm, mol.bas, mol.env)
        want = np.zeros(out.size)
        r = f(want.ctypes.data_as(dp), None, t.ctypes.data_as(ip), atm.ctypes.data_as(ip), atm.shape[0],
              bas.ctypes.data_as(ip), bas.shape[0], env.ctypes.data_as(dp), None, None)
        assert ret == r and close(out, want), (t, ret, r)


def test_batched_derivatives_match_libcint_goldens(cx):
    import torch
    g = np.load(GOLD)
    for name, mol, fn in _cases():
        tup, offs, vals = g[name + "_tuples"], g[name + "_offsets"], g[name + "_values"]
        fam = cx.INT2E if tup.shape[1] == 4 else cx.INT3C2E
        sph = fn.endswith("sph")
        n = cx.ip1_len(fam, tup, mol.bas, sph)
        assert n == vals.size
        buf = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        got_offs = cx.ip1_eval(fam, tup, mol.atm, mol.bas, mol.env, buf.data_ptr(), sph)
        assert np.array_equal(got_offs, offs[:-1])
        got = buf.cpu().numpy()
        assert np.isfinite(got).all()
        assert close(got, vals), (name, np.abs(got - vals).max())


def test_cintrs_derivative_ids(cx):
    """cintx-capi ids 36/35 (int2e_ip1 sph/cart) and 19/18 (int3c2e_ip1 sph/cart) return the
    per-call blocks and not0."""
    from test_abi import _Summary, _dispatch_args
    dp = ctypes.POINTER(ctypes.c_double)
    w = M.water_like()
    wa = M.with_aux(w)
    for api, mol, shls, fn in [(36, w, [5, 6, 4, 9], cx.int2e_ip1_sph), (35, w, [1, 11, 3, 4], cx.int2e_ip1_cart),
                               (19, wa, [5, 7, 20], cx.int3c2e_ip1_sph), (18, wa, [2, 9, 40], cx.int3c2e_ip1_cart)]:
        ref, ret = fn(shls, mol.atm, mol.bas, mol.env)
        keep, args = _dispatch_args(mol, shls)
        out = np.full(ref.size, np.nan)
        summ = _Summary()
        rc = cx.lib.cintrs_eval(api, out.ctypes.data_as(dp), out.size, None, 0, *args, None, None, 0,
                                ctypes.byref(summ))
        assert rc == 0 and summ.not0 == ret and summ.bytes_written == 8 * ref.size, (api, rc, cx.last_error())
        assert np.array_equal(out, ref)


@pytest.mark.skipif(not RefLibcint.available(), reason="libcint from the reference sources not built")
def test_f_shell_derivatives_match_live_libcint(cx):
    """int2e_ip1_sph on 150 seeded quartets of the 120-atom molecule with an f shell on the
    differentiated pair (derivative ceiling l = 4), batched on the device, against libcint."""
    import torch
    mol = M.mol120()
    rng = np.random.default_rng(31)
    f_sh = np.where(mol.bas[:, 1] == 3)[0]
    xyz = np.array([mol.env[mol.atm[mol.bas[s, 0], 1]:mol.atm[mol.bas[s, 0], 1] + 3] for s in range(mol.nbas)])
    rows = []
    for s in rng.choice(f_sh, 150):
        near = np.where(np.linalg.norm(xyz - xyz[s], axis=1) < 6.0)[0]  # partners within 6 bohr
        rows.append([s] + list(rng.choice(near, 3)))
    tup = np.array(rows, dtype=np.int32)
    ref, offs, rets = RefLibcint().batch(tup, mol, True, ip1=True)
    n = cx.ip1_len(cx.INT2E, tup, mol.bas, True)
    buf = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    cx.ip1_eval(cx.INT2E, tup, mol.atm, mol.bas, mol.env, buf.data_ptr(), True)
    got = buf.cpu().numpy()
    assert np.abs(ref).max() > 0
    assert close(got, ref), np.abs(got - ref).max()
