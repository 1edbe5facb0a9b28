"""Regenerate the golden fixtures in this folder.

  roots_mpmath.npz   Rys roots t^2 and weights for n = 1..9 at 48 x values each, computed in
                     50-digit arithmetic (moments -> modified Chebyshev -> Golub-Welsch); this
                     pins root accuracy independently of libcint and of the C oracle.
  libcint_*.npz      Integral blocks and return values from libcint 6.1.3 compiled from the
                     reference sources (oracle/_ref/libcint.so, built by oracle/Makefile) for
                     seeded samples of shell tuples of the synthetic molecules, plus a small
                     generally-contracted basis (nctr = 2) and dims / expcutoff variants.
  libcint_ip1.npz    libcint int2e_ip1 / int3c2e_ip1 blocks (x, y, z components) for seeded tuples
                     of the 3-atom molecule (sph, cart), the 40-atom molecule and the 3-atom
                     molecule with its auxiliary basis (3-centre, auxiliary shells up to g).
  libcint_mol120f.npz  libcint blocks of 50 quartets from every f-containing angular-momentum
                     class of the 120-atom molecule's Schwarz-screened quartet set, each quartet
                     in a random one of its 8 index orders (libcint evaluated with each equal-l
                     pair ordered so that it builds on the pair's stable centre, then transposed
                     to the stored order: libcint_stable).

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


def schwarz_pairs(ref, mol):
    """Every shell pair i >= j with q_ij = sqrt(max |(ij|ij)|) from libcint."""
    ii, jj = np.tril_indices(mol.nbas)
    pairs = np.stack([ii, jj], axis=1).astype(np.int32)
    vals, offs, _ = ref.batch(np.concatenate([pairs, pairs], axis=1), mol)
    q = np.sqrt(np.maximum.reduceat(np.abs(vals), offs[:-1]))
    return pairs, q


def class_stratified_quartets(ref, mol, cutoff, per_class, seed, need_l=3):
    """Seeded sample of per_class quartets (or all, if fewer) from every angular-momentum class
    that contains a shell of l == need_l, drawn uniformly within the class from the 8-fold-unique
    quartets whose Schwarz bound q_ij q_kl reaches cutoff; each quartet is then put in a random
    one of its 8 equivalent index orders.  Returns {class label: tuples}."""
    rng = np.random.default_rng(seed)
    pairs, q = schwarz_pairs(ref, mol)
    order = np.argsort(-q, kind="stable")
    pairs, q = pairs[order], q[order]
    keep = q * q.max() >= cutoff
    pairs, q = pairs[keep], q[keep]
    # partners of pair position i: positions j <= i (q_j >= q_i) with q_i q_j >= cutoff
    count = np.minimum(np.arange(len(q)) + 1, np.searchsorted(-q, -(cutoff / q), side="right"))
    l = mol.bas[:, 1]
    la, lb = l[pairs[:, 0]], l[pairs[:, 1]]
    pc = 10 * np.maximum(la, lb) + np.minimum(la, lb)
    idx = {c: np.where(pc == c)[0] for c in np.unique(pc)}
    out = {}
    for A in sorted(idx):
        for B in sorted(idx):
            if B > A or (A // 10 != need_l and A % 10 != need_l and B // 10 != need_l and B % 10 != need_l):
                continue
            # (i, j) with {pc_i, pc_j} = {A, B}: i of class X, partner j < count[i] of class Y
            cand_i, cand_w, cand_y = [], [], []
            for X, Y in ((A, B), (B, A)) if A != B else ((A, B),):
                ix = idx[X]
                w = np.searchsorted(idx[Y], count[ix])
                cand_i.append(ix)
                cand_w.append(w)
                cand_y.append(np.full(len(ix), Y))
            ci, cw, cy = np.concatenate(cand_i), np.concatenate(cand_w), np.concatenate(cand_y)
            total = int(cw.sum())
            if total == 0:
                continue
            n = min(per_class, total)
            pick = rng.choice(len(ci), size=n, p=cw / total)
            rows = []
            for k in pick:
                j = idx[cy[k]][rng.integers(0, cw[k])]
                a, b = pairs[ci[k]]
                c, d = pairs[j]
                if rng.random() < 0.5:
                    a, b = b, a
                if rng.random() < 0.5:
                    c, d = d, c
                if rng.random() < 0.5:
                    a, b, c, d = c, d, a, b
                rows.append((a, b, c, d))
            out["(%d%d|%d%d)" % (A // 10, A % 10, B // 10, B % 10)] = np.array(rows, dtype=np.int32)
    return out


def base_first(mol, sx, sy):
    """The shell of the pair (sx, sy) a numerically stable recurrence is built on: the higher l,
    and for equal l the smaller cancellation measure max over primitive pairs of
    a_y |X - Y| / sqrt(a_x + a_y) (ties: the larger shell index).  libcint builds on the second
    shell of an equal-l pair (g2e.c:101), so it evaluates a tuple stably when the pair's stable
    centre comes second."""
    lx, ly = int(mol.bas[sx, 1]), int(mol.bas[sy, 1])
    if lx != ly:
        return lx > ly
    if sx == sy:
        return True
    def shell(s):
        b = mol.bas[s]
        return mol.env[b[5]:b[5] + b[2]], mol.env[mol.atm[b[0], 1]:mol.atm[b[0], 1] + 3]
    (ax, rx), (ay, ry) = shell(sx), shell(sy)
    d = float(np.linalg.norm(rx - ry))
    r = d / np.sqrt(ax[:, None] + ay[None, :])
    on_x = float((ay[None, :] * r).max())
    on_y = float((ax[:, None] * r).max())
    if not (on_x != on_y) or abs(on_x - on_y) <= 1e-12 * max(on_x, on_y):
        return sx >= sy
    return on_x < on_y


def libcint_stable(ref, mol, tuples, sph=True):
    """libcint blocks of int2e tuples in the requested index order, each evaluated with every
    equal-l pair ordered (other, stable centre) so that libcint builds its recurrence on the
    stable centre (unequal-l pairs are left as requested: libcint builds on the higher l either
    way), then transposed back.  Returns (values, offsets[n+1], return values)."""
    tuples = np.ascontiguousarray(tuples, dtype=np.int32)
    ords = []
    for t in tuples:
        o = [0, 1, 2, 3]
        for a, b in ((0, 1), (2, 3)):
            la, lb = mol.bas[t[a], 1], mol.bas[t[b], 1]
            # libcint builds on the second shell of an equal-l pair: put the stable centre there
            if la == lb and base_first(mol, t[a], t[b]):
                o[a], o[b] = b, a
        ords.append(o)
    ords = np.array(ords)
    ev = tuples[np.arange(len(tuples))[:, None], ords]
    vals, offs, rets = ref.batch(ev, mol, sph)
    out = np.empty_like(vals)
    l = mol.bas[:, 1]
    nc = mol.bas[:, 3]
    per = (2 * l + 1 if sph else (l + 1) * (l + 2) // 2) * nc
    for q, (t, o) in enumerate(zip(tuples, ords)):
        n = per[t]                                  # requested axis lengths
        blk = vals[offs[q]:offs[q + 1]].reshape([n[o[3]], n[o[2]], n[o[1]], n[o[0]]])
        # blk axes (slowest first) are requested axes o[3], o[2], o[1], o[0]; order them as 3, 2, 1, 0
        pos = {o[3 - k]: k for k in range(4)}
        out[offs[q]:offs[q + 1]] = blk.transpose([pos[3], pos[2], pos[1], pos[0]]).reshape(-1)
    return out, offs, rets


def make_mol120():
    """libcint blocks for a class-stratified sample of the 120-atom f-shell molecule's Schwarz-
    screened (1e-12) quartet set: 50 quartets of every class containing an f shell, evaluated by
    libcint in the index order that makes it build on each pair's stable centre."""
    ref = RefLibcint()
    mol = M.mol120()
    per = class_stratified_quartets(ref, mol, 1e-12, 50, 120)
    labels = sorted(per)
    tuples = np.concatenate([per[k] for k in labels])
    cls = np.concatenate([np.full(len(per[k]), i, dtype=np.int32) for i, k in enumerate(labels)])
    vals, offs, rets = libcint_stable(ref, mol, tuples)
    np.savez_compressed(os.path.join(HERE, "libcint_mol120f.npz"), int2e_sph_tuples=tuples,
                        int2e_sph_offsets=offs, int2e_sph_values=vals, int2e_sph_ret=rets,
                        class_index=cls, class_labels=np.array(labels))


def make_ip1():
    """libcint int2e_ip1 / int3c2e_ip1 blocks (three components each) for seeded tuples of the
    3-atom molecule (sph and cart), the 40-atom molecule (sph) and the 3-atom molecule with its
    auxiliary basis (3-centre, auxiliary shells up to g)."""
    ref = RefLibcint()
    rng = np.random.default_rng(4242)
    d = {}

    def put(name, mol, tuples, sph):
        vals, offs, rets = ref.batch(tuples, mol, sph, ip1=True)
        d[name + "_tuples"], d[name + "_offsets"], d[name + "_values"], d[name + "_ret"] = tuples, offs, vals, rets

    w = M.water_like()
    put("water3_int2e_ip1_sph", w, sample_tuples(rng, w.nbas, 4, 300), True)
    put("water3_int2e_ip1_cart", w, sample_tuples(rng, w.nbas, 4, 100), False)
    m40 = M.mol40()
    put("mol40_int2e_ip1_sph", m40, sample_tuples(rng, m40.nbas, 4, 200), True)
    wa = M.with_aux(w)
    norb = w.nbas
    t3 = np.stack([rng.integers(0, norb, 240), rng.integers(0, norb, 240), rng.integers(norb, wa.nbas, 240)],
                  axis=1).astype(np.int32)
    put("water3aux_int3c2e_ip1_sph", wa, t3[:160], True)
    put("water3aux_int3c2e_ip1_cart", wa, t3[160:], False)
    np.savez_compressed(os.path.join(HERE, "libcint_ip1.npz"), **d)


if __name__ == "__main__":
    make_roots()
    make_integrals()
    make_mol120()
    make_ip1()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
