"""Generates rys_gl64.h: the fixed discretisation of the Rys measure used by the learned-root
refinement (rysnet.cu).

The Rys weight e^{-x u} / (2 sqrt(u)) on u in [0, 1] becomes e^{-x t^2} dt with u = t^2, so a
64-point Gauss-Legendre rule on t in [0, 1] (nodes t_m, weights W_m) discretises it as
u_m = t_m^2 with masses W_m e^{-x u_m}; the first 2n moments of that discrete measure match the
Rys measure to double precision for n <= 9 and x below the table's asymptotic switch-over
(x < 100).  Nodes are found by Newton's method on P_64 in 40-digit arithmetic (mpmath) and
rounded once to double.

    python cintx_b200/csrc/gen_rys_gl.py      # rewrites rys_gl64.h next to this script
"""
import os

import mpmath as mp

M = 64


def gauss_legendre(m: int):
    mp.mp.dps = 40
    nodes, weights = [], []
    for k in range(1, m + 1):
        x = mp.cos(mp.pi * (k - mp.mpf(1) / 4) / (m + mp.mpf(1) / 2))
        for _ in range(100):
            p0, p1 = mp.mpf(1), x
            for j in range(2, m + 1):
                p0, p1 = p1, ((2 * j - 1) * x * p1 - (j - 1) * p0) / j
            dp = m * (x * p1 - p0) / (x * x - 1)
            dx = p1 / dp
            x -= dx
            if abs(dx) < mp.mpf(10) ** -38:
                break
        nodes.append(x)
        weights.append(2 / ((1 - x * x) * dp * dp))
    return nodes, weights


def main():
    xs, ws = gauss_legendre(M)
    u = [((x + 1) / 2) ** 2 for x in xs]  # t = (x + 1) / 2 on [0, 1], u = t^2
    w = [v / 2 for v in ws]
    order = sorted(range(M), key=lambda i: u[i])
    out = ["// Generated by gen_rys_gl.py: 64-point Gauss-Legendre discretisation of the Rys measure",
           "// (u_m = t_m^2, W_m for t on [0, 1]).  Do not edit.", "#pragma once", "",
           "namespace cintx {", "constexpr int kRysGlNodes = %d;" % M,
           "__device__ __constant__ const double kRysGlU[%d] = {" % M]
    out += ["    %s," % mp.nstr(u[i], 20, min_fixed=-1, max_fixed=-1) for i in order]
    out += ["};", "__device__ __constant__ const double kRysGlW[%d] = {" % M]
    out += ["    %s," % mp.nstr(w[i], 20, min_fixed=-1, max_fixed=-1) for i in order]
    out += ["};", "}  // namespace cintx", ""]
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rys_gl64.h"), "w") as fh:
        fh.write("\n".join(out))


if __name__ == "__main__":
    main()
