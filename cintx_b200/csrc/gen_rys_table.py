"""Generate the Rys-root table used by the device root evaluator (rys_roots.cuh).

For each order n = 1..NMAX the roots t_r^2 and weights w_r of the Rys quadrature
    int_0^1 exp(-x t^2) P(t^2) dt = sum_r w_r P(t_r^2)
(the quantity libcint's CINTrys_roots returns as u = t^2/(1-t^2), rys_roots.c:57) are
tabulated on x in [0, XMAX[n]) in unit-width intervals.  Inside interval i the 2n functions
are degree-DEG polynomials in z = 2(x - i) - 1 in the monomial basis, obtained from the
Chebyshev interpolant at DEG+1 Chebyshev points (both computed in 50-digit arithmetic).
For x >= XMAX[n] the device uses the large-x form t_r^2 = h_r^2/x, w_r = W_r/sqrt(x) with
h_r, W_r the positive Gauss-Hermite nodes/weights of order 2n; XMAX[n] is where that form is
exact to double rounding (the truncated tail exp(-x) x^(2n) is below 1e-16 relative).

Roots are computed from the moments F_k(x) = int_0^1 t^2k exp(-x t^2) dt (the Boys function)
by the modified Chebyshev algorithm and the Golub-Welsch eigenproblem in mpmath.

Output: rys_table.bin, little-endian float64, layout
    [header: 16 x int64: NMAX, DEG, XMAX[1..NMAX], pad]
    for n in 1..NMAX: for i in 0..XMAX[n]-1: for k in 0..DEG: for f in 0..2n-1: coef
        (f < n: t_r^2 of root f;  f >= n: w_r of root f-n; roots ascending)
    for n in 1..NMAX: n values h_r^2 then n values W_r
Run: python gen_rys_table.py [--out PATH] [--procs N]
"""
from __future__ import annotations

import argparse
import os
import struct
from multiprocessing import get_context

import mpmath as mp

NMAX = 9
DEG = 11
XMAX = [0, 40, 52, 60, 64, 72, 76, 84, 92, 100]
DPS = 50


def boys(k: int, x):
    if x == 0:
        return mp.mpf(1) / (2 * k + 1)
    half = mp.mpf(1) / 2
    return mp.gammainc(k + half, 0, x) / (2 * x ** (k + half))


def rys_mp(n: int, x):
    """Ascending (t^2, w) of order n by the Chebyshev algorithm + Golub-Welsch."""
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
    return [p[0] for p in pairs], [p[1] for p in pairs]


def interval_coeffs(args):
    n, i = args
    mp.mp.dps = DPS
    npts = DEG + 1
    zs = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / npts) for k in range(npts)]
    vals = []
    for z in zs:
        x = i + (z + 1) / 2
        t, w = rys_mp(n, x)
        vals.append(t + w)
    nf = 2 * n
    # Chebyshev interpolation coefficients c_j = (2/N) sum_k f(z_k) T_j(z_k), c_0 halved
    cheb = [[mp.mpf(0)] * nf for _ in range(npts)]
    for j in range(npts):
        for k, z in enumerate(zs):
            tj = mp.cos(j * mp.acos(z))
            for f in range(nf):
                cheb[j][f] += vals[k][f] * tj
        for f in range(nf):
            cheb[j][f] *= mp.mpf(2) / npts
    for f in range(nf):
        cheb[0][f] /= 2
    # Chebyshev -> monomial: T_j(z) = sum_m tcoef[j][m] z^m
    tco = [[mp.mpf(0)] * npts for _ in range(npts)]
    tco[0][0] = 1
    if npts > 1:
        tco[1][1] = 1
    for j in range(2, npts):
        for m in range(npts):
            v = -tco[j - 2][m]
            if m > 0:
                v += 2 * tco[j - 1][m - 1]
            tco[j][m] = v
    mono = [[mp.mpf(0)] * nf for _ in range(npts)]
    for j in range(npts):
        for m in range(npts):
            if tco[j][m] != 0:
                for f in range(nf):
                    mono[m][f] += cheb[j][f] * tco[j][m]
    return n, i, [[float(mono[m][f]) for f in range(nf)] for m in range(npts)]


def hermite_half(n: int):
    mp.mp.dps = DPS
    m = 2 * n
    J = mp.matrix(m, m)
    for i in range(m - 1):
        J[i, i + 1] = J[i + 1, i] = mp.sqrt(mp.mpf(i + 1) / 2)
    E, Q = mp.eigsy(J)
    pos = sorted((E[i], mp.sqrt(mp.pi) * Q[0, i] ** 2) for i in range(m) if E[i] > 0)
    return [float(p[0] ** 2) for p in pos], [float(p[1]) for p in pos]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "rys_table.bin"))
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    jobs = [(n, i) for n in range(1, NMAX + 1) for i in range(XMAX[n])]
    with get_context("spawn").Pool(args.procs) as pool:
        res = pool.map(interval_coeffs, jobs, chunksize=4)
    table = {(n, i): c for n, i, c in res}
    with open(args.out, "wb") as fh:
        hdr = [NMAX, DEG] + XMAX[1:] + [0] * (16 - 2 - NMAX)
        fh.write(struct.pack("<16q", *hdr))
        for n in range(1, NMAX + 1):
            for i in range(XMAX[n]):
                for row in table[(n, i)]:
                    fh.write(struct.pack("<%dd" % len(row), *row))
        for n in range(1, NMAX + 1):
            h2, W = hermite_half(n)
            fh.write(struct.pack("<%dd" % n, *h2))
            fh.write(struct.pack("<%dd" % n, *W))
    print("wrote", args.out, os.path.getsize(args.out), "bytes")


if __name__ == "__main__":
    main()
