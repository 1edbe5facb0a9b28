"""CPU checks of the test oracle, the golden fixtures and the shipped root table."""
import hashlib
import os
import struct

import numpy as np
import pytest

from conftest import ROOT, close
from cintx_b200 import molecules as M
from oracle import RefLibcint, Restatement

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def orc():
    return Restatement()


def gold(name):
    return np.load(os.path.join(GOLD, name))


def test_molecule_generator_is_pinned():
    want = {"water3": "28acc6d628d854f6", "mol40_spd": "42cbc709a316a5ed",
            "mol120_spdf": "7a105f2182cdf4ce", "mol20_g": "f319ab378dad6576"}
    for f in (M.water_like, M.mol40, M.mol120, M.mol20_g):
        m = f()
        h = hashlib.sha256(m.env.tobytes() + m.bas.tobytes() + m.atm.tobytes()).hexdigest()[:16]
        assert h == want[m.name], m.name
    w = M.water_like()
    assert w.nbas == 12 and int(w.ao_loc()[-1]) == 24


def test_oracle_roots_vs_mpmath(orc):
    g = gold("roots_mpmath.npz")
    for n in range(1, 10):
        for i, x in enumerate(g["x"]):
            t2, w = orc.rys_t2(n, x)
            np.testing.assert_allclose(t2, g["t2_%d" % n][i], rtol=2e-15, atol=0)
            np.testing.assert_allclose(w, g["w_%d" % n][i], rtol=2e-15, atol=0)


def _check_family(orc, mol, data, fam, call):
    tup = data[fam + "_tuples"]
    offs = data[fam + "_offsets"]
    vals = data[fam + "_values"]
    rets = data[fam + "_ret"]
    for q, t in enumerate(tup):
        out, ret = call(t, mol)
        ref = vals[offs[q]:offs[q + 1]]
        assert ret == rets[q], (fam, t)
        assert close(out, ref), (fam, t, np.abs(out - ref).max())


def test_oracle_vs_golden_water3(orc):
    mol = M.water_like()
    g = gold("libcint_water3.npz")
    _check_family(orc, mol, g, "int2e_sph", lambda t, m: orc.int2e(t, m, True))
    _check_family(orc, mol, g, "int2e_cart", lambda t, m: orc.int2e(t, m, False))
    _check_family(orc, mol, g, "int3c2e_sph", lambda t, m: orc.int3c2e(t, m, True))
    _check_family(orc, mol, g, "int3c2e_cart", lambda t, m: orc.int3c2e(t, m, False))
    _check_family(orc, mol, g, "int2c2e_sph", lambda t, m: orc.int2c2e(t, m, True))
    _check_family(orc, mol, g, "int2c2e_cart", lambda t, m: orc.int2c2e(t, m, False))


def test_oracle_vs_golden_g_shells(orc):
    mol = M.mol20_g()
    _check_family(orc, mol, gold("libcint_mol20g.npz"), "int2e_sph", lambda t, m: orc.int2e(t, m, True))


def test_oracle_vs_golden_general_contraction(orc):
    g = gold("libcint_ctr2.npz")
    mol = M.Molecule("ctr2", g["atm"], g["bas"], g["env"], np.zeros((2, 3)))
    _check_family(orc, mol, g, "int2e_sph", lambda t, m: orc.int2e(t, m, True))
    _check_family(orc, mol, g, "int2e_cart", lambda t, m: orc.int2e(t, m, False))
    _check_family(orc, mol, g, "int3c2e_sph", lambda t, m: orc.int3c2e(t, m, True))


def test_oracle_vs_golden_f_shell_classes(orc):
    """The restatement on 50 quartets of every f-containing class of the 120-atom molecule
    (libcint blocks of the Schwarz-screened set, random index orders)."""
    mol = M.mol120()
    g = gold("libcint_mol120f.npz")
    tup = g["int2e_sph_tuples"]
    offs = g["int2e_sph_offsets"]
    out, o2 = orc.int2e_batch(tup, mol, True)
    assert np.array_equal(o2, offs[:-1])
    assert close(out, g["int2e_sph_values"]), np.abs(out - g["int2e_sph_values"]).max()
    labels = g["class_labels"]
    assert len(labels) == 34 and np.bincount(g["class_index"]).min() == 50


def test_oracle_c2s_is_orthonormal_on_sphere(orc):
    # rows of the l >= 2 transforms, applied to cartesian monomials, give real spherical
    # harmonics; check via the known d(xy) coefficient sqrt(15/(4 pi)) and row count
    for l in range(2, 5):
        m = orc.c2s(l)
        assert m.shape == (2 * l + 1, (l + 1) * (l + 2) // 2)
    np.testing.assert_allclose(orc.c2s(2)[0, 1], np.sqrt(15 / (4 * np.pi)), rtol=1e-15)


@pytest.mark.skipif(not RefLibcint.available(), reason="libcint from the reference sources not built")
def test_oracle_vs_live_libcint(orc):
    ref = RefLibcint()
    rng = np.random.default_rng(7)
    for mol in (M.water_like(), M.mol40()):
        for t in rng.integers(0, mol.nbas, size=(60, 4)):
            a, ra = orc.int2e(t, mol)
            b, rb = ref.int2e(t, mol)
            assert ra == rb and close(a, b), (mol.name, t)
        for t in rng.integers(0, mol.nbas, size=(30, 3)):
            a, ra = orc.int3c2e(t, mol)
            b, rb = ref.int3c2e(t, mol)
            assert ra == rb and close(a, b), (mol.name, t)


def _load_table():
    with open(os.path.join(ROOT, "cintx_b200", "csrc", "rys_table.bin"), "rb") as fh:
        raw = fh.read()
    hdr = struct.unpack("<16q", raw[:128])
    nmax, deg = hdr[0], hdr[1]
    xmax = [0] + list(hdr[2:2 + nmax])
    data = np.frombuffer(raw[128:], dtype="<f8")
    off, poly, asym = 0, {}, {}
    for n in range(1, nmax + 1):
        sz = xmax[n] * (deg + 1) * 2 * n
        poly[n] = data[off:off + sz].reshape(xmax[n], deg + 1, 2 * n)
        off += sz
    for n in range(1, nmax + 1):
        asym[n] = (data[off:off + n], data[off + n:off + 2 * n])
        off += 2 * n
    assert off == data.size
    return deg, xmax, poly, asym


def test_shipped_root_table_vs_mpmath():
    """The table the device evaluates, evaluated the same way on the CPU."""
    deg, xmax, poly, asym = _load_table()
    g = gold("roots_mpmath.npz")
    for n in range(1, 10):
        for i, x in enumerate(g["x"]):
            if x >= xmax[n]:
                t2 = asym[n][0] / x
                w = asym[n][1] / np.sqrt(x)
            else:
                k = int(x)
                z = 2 * (x - k) - 1
                c = poly[n][k]
                acc = c[deg].copy()
                for d in range(deg - 1, -1, -1):
                    acc = acc * z + c[d]
                t2, w = acc[:n], acc[n:]
            np.testing.assert_allclose(t2, g["t2_%d" % n][i], rtol=5e-15, atol=0, err_msg="n=%d x=%g" % (n, x))
            np.testing.assert_allclose(w, g["w_%d" % n][i], rtol=5e-15, atol=0, err_msg="n=%d x=%g" % (n, x))
