"""Regenerate the golden fixtures in this folder.

  roots_mpmath.npz   Rys roots t^2 and weights for n = 1..9 at 48 x values each, computed in
                     50-digit arithmetic (moments -> modified Chebyshev -> Golub-Welsch); this
                     pins root accuracy independently of libcint and of the C oracle.
  libcint_*.npz      Integral blocks and return values from libcint 6.1.3 compiled from the
                     reference sources (oracle/_ref/libcint.so, built by oracle/Makefile) for
                     seeded samples of shell tuples of the synthetic molecules, plus a small
                     generally-contracted basis (nctr = 2) and dims / expcutoff variants.

Run from the repository root: python tests/golden/make_golden.py   (needs oracle/_ref)
"""
from __future__ import annotations

import os
import sys

import mpmath as mp
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cintx_b200 import molecules as M  # noqa: E402
from oracle import RefLibcint  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def boys(k, x):
    if x == 0:
        return mp.mpf(1) / (2 * k + 1)
    return mp.gammainc(k + mp.mpf(1) / 2, 0, x) / (2 * x ** (k + mp.mpf(1) / 2))


def rys_mp(n, x):
    mom = [boys(k, x) for k in range(2 * n)]
    a = [mp.mpf(0)] * n
    b = [mp.mpf(0)] * n
    prev = [mp.mpf(0)] * (2 * n)
    cur = list(mom)
    a[0] = mom[1] / mom[0]
    b[0] = mom[0]
    for k in range(1, n):
        nxt = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            nxt[l] = cur[l + 1] - a[k - 1] * cur[l] - b[k - 1] * prev[l]
        a[k] = nxt[k + 1] / nxt[k] - cur[k] / cur[k - 1]
        b[k] = nxt[k] / cur[k - 1]
        prev, cur = cur, nxt
    J = mp.matrix(n, n)
    for i in range(n):
        J[i, i] = a[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(b[i + 1])
    E, Q = mp.eigsy(J)
    pairs = sorted((E[i], mom[0] * Q[0, i] ** 2) for i in range(n))
    return [float(p[0]) for p in pairs], [float(p[1]) for p in pairs]


def make_roots():
    mp.mp.dps = 50
    rng = np.random.default_rng(12345)
    xs = np.concatenate([[0.0, 1e-9, 1e-4, 0.5, 1.0, 2.999, 7.25, 12.0, 17.5, 24.9, 33.3, 39.999,
                          40.0, 51.5, 63.0, 75.0, 88.0, 99.5, 100.0, 150.0, 1e3, 1e5],
                         rng.uniform(0, 110, 20), 10 ** rng.uniform(-7, 0, 6)])
    out = {"x": xs}
    for n in range(1, 10):
        t = np.zeros((len(xs), n))
        w = np.zeros((len(xs), n))
        for i, x in enumerate(xs):
            t[i], w[i] = rys_mp(n, mp.mpf(float(x)))
        out["t2_%d" % n] = t
        out["w_%d" % n] = w
    np.savez_compressed(os.path.join(HERE, "roots_mpmath.npz"), **out)


def contracted_pair_molecule():
    """Two atoms with general contractions (nctr = 2) for layout checks."""
    rng = M.SplitMix64(77)
    env = [0.0] * M.PTR_ENV_START
    coords = [[0.0, 0.0, 0.0], [0.3, -1.1, 1.4]]
    atm = []
    for c in coords:
        atm.append([1, len(env), 1, 0, 0, 0])
        env.extend(c)
    bas = []
    for ia in range(2):
        for l, nprim, nctr in [(0, 3, 2), (1, 2, 2), (2, 2, 1), (1, 1, 1)]:
            exps = sorted((rng.log_uniform(0.2, 30.0) for _ in range(nprim)), reverse=True)
            pe = len(env)
            env.extend(exps)
            pc = len(env)
            for c in range(nctr):
                env.extend(rng.normal() * M.gto_norm(l, a) for a in exps)
            bas.append([ia, l, nprim, nctr, 0, pe, pc, 0])
    return M.Molecule("ctr2", np.array(atm, dtype=np.int32), np.array(bas, dtype=np.int32),
                      np.array(env), np.array(coords))


def sample_tuples(rng, nbas, k, n):
    return rng.integers(0, nbas, size=(n, k)).astype(np.int32)


def dump_blocks(ref, name, mol, tuples, sph, fam):
    blocks, rets = [], []
    f = {4: ref.int2e, 3: ref.int3c2e, 2: ref.int2c2e}[tuples.shape[1]]
    for t in tuples:
        b, r = f(t, mol, sph)
        blocks.append(b)
        rets.append(r)
    offs = np.zeros(len(blocks) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(b) for b in blocks])
    return {fam + "_tuples": tuples, fam + "_offsets": offs, fam + "_values": np.concatenate(blocks),
            fam + "_ret": np.array(rets, dtype=np.int32)}


def make_integrals():
    ref = RefLibcint()
    rng = np.random.default_rng(2024)
    # water3: all-quartet checks run against the C oracle; here a seeded sample pins both
    mol = M.water_like()
    d = {}
    d.update(dump_blocks(ref, "water3", mol, sample_tuples(rng, mol.nbas, 4, 400), True, "int2e_sph"))
    d.update(dump_blocks(ref, "water3", mol, sample_tuples(rng, mol.nbas, 4, 120), False, "int2e_cart"))
    d.update(dump_blocks(ref, "water3", mol, sample_tuples(rng, mol.nbas, 3, 150), True, "int3c2e_sph"))
    d.update(dump_blocks(ref, "water3", mol, sample_tuples(rng, mol.nbas, 3, 60), False, "int3c2e_cart"))
    d.update(dump_blocks(ref, "water3", mol, sample_tuples(rng, mol.nbas, 2, 100), True, "int2c2e_sph"))
    d.update(dump_blocks(ref, "water3", mol, sample_tuples(rng, mol.nbas, 2, 40), False, "int2c2e_cart"))
    np.savez_compressed(os.path.join(HERE, "libcint_water3.npz"), **d)
    # g shells
    mol = M.mol20_g()
    gsh = [i for i in range(mol.nbas) if mol.bas[i, 1] == 4][:6]
    other = list(range(8))
    t = [(gsh[a % 6], other[b % 8], gsh[(a + b) % 6], other[(a * 3 + b) % 8]) for a in range(6) for b in range(5)]
    t += [(gsh[a % 6], gsh[(a + 1) % 6], gsh[(a + 2) % 6], gsh[(a + 3) % 6]) for a in range(4)]
    d = dump_blocks(ref, "mol20_g", mol, np.array(t, dtype=np.int32), True, "int2e_sph")
    np.savez_compressed(os.path.join(HERE, "libcint_mol20g.npz"), **d)
    # general contractions, all quartets
    mol = contracted_pair_molecule()
    import itertools
    allq = np.array(list(itertools.product(range(mol.nbas), repeat=4)), dtype=np.int32)
    sel = allq[rng.choice(len(allq), size=150, replace=False)]
    d = dump_blocks(ref, "ctr2", mol, sel[:150], True, "int2e_sph")
    d.update(dump_blocks(ref, "ctr2", mol, sel[:80], False, "int2e_cart"))
    d.update(dump_blocks(ref, "ctr2", mol, sample_tuples(rng, mol.nbas, 3, 60), True, "int3c2e_sph"))
    d["atm"], d["bas"], d["env"] = mol.atm, mol.bas, mol.env
    np.savez_compressed(os.path.join(HERE, "libcint_ctr2.npz"), **d)


if __name__ == "__main__":
    make_roots()
    make_integrals()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
