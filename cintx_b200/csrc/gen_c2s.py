"""Generate c2s_coef.h: cartesian -> real spherical coefficients for l = 0..4.

Rows m = -l..l, columns the cartesian monomials in libcint order (x power descending, then
y power descending).  The coefficients are those of the regular real solid harmonics
(Helgaker, Jorgensen & Olsen, Molecular Electronic-Structure Theory, eq. 6.4.47-6.4.50)
scaled by sqrt((2l+1)/(4 pi)), libcint's spherical normalisation for l >= 2
(cart2sph.c g_trans_cart2sph).  For l <= 1 libcint keeps the cartesian functions (p in
x, y, z order) and moves sqrt((2l+1)/(4 pi)) into the common factor (g1e.c:566), so the
table is the identity there.  Values are evaluated in 40-digit arithmetic.

Run: python gen_c2s.py > c2s_coef.h
"""
import mpmath as mp

LMAX = 4
mp.mp.dps = 40


def carts(l):
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def c2s(l):
    cs = carts(l)
    idx = {c: i for i, c in enumerate(cs)}
    M = [[mp.mpf(0)] * len(cs) for _ in range(2 * l + 1)]
    if l <= 1:
        for i in range(len(cs)):
            M[i][i] = mp.mpf(1)
        return M
    scale = mp.sqrt(mp.mpf(2 * l + 1) / (4 * mp.pi))
    for m in range(-l, l + 1):
        am = abs(m)
        nlm = mp.sqrt(2 * mp.factorial(l + am) * mp.factorial(l - am) / (2 if m == 0 else 1)) / (
            2 ** am * mp.factorial(l))
        twovm = 1 if m < 0 else 0
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                for twov in range(twovm, am + 1, 2):
                    sgn = -1 if ((t + (twov - twovm) // 2) & 1) else 1
                    c = sgn * mp.mpf(0.25) ** t * mp.binomial(l, t) * mp.binomial(l - t, am + t) * \
                        mp.binomial(t, u) * mp.binomial(am, twov)
                    ex = 2 * t + am - 2 * u - twov
                    ey = 2 * u + twov
                    M[m + l][idx[(ex, ey, l - ex - ey)]] += scale * nlm * c
    return M


def main():
    print("// Generated by gen_c2s.py: cartesian -> real spherical coefficients, l = 0..%d." % LMAX)
    print("#pragma once")
    print("namespace cintx {")
    print("// c2s_coef(l, m, f): row m (0..2l, i.e. m = -l..l), cartesian column f.")
    print("__host__ __device__ constexpr double c2s_coef(int l, int m, int f) {")
    for l in range(LMAX + 1):
        M = c2s(l)
        print("  if (l == %d) {" % l)
        for m, row in enumerate(M):
            for f, v in enumerate(row):
                if abs(v) > 1e-30:
                    print("    if (m == %d && f == %d) return %s;" % (m, f, mp.nstr(v, 20, strip_zeros=False)))
        print("    return 0.0;")
        print("  }")
    print("  return 0.0;")
    print("}")
    # sparse lists for runtime-indexed transform stages
    maxnnz = 0
    rows = {}
    for l in range(LMAX + 1):
        M = c2s(l)
        for m, row in enumerate(M):
            nz = [(f, v) for f, v in enumerate(row) if abs(v) > 1e-30]
            rows[(l, m)] = nz
            maxnnz = max(maxnnz, len(nz))
    print("constexpr int C2S_MAXNNZ = %d;" % maxnnz)
    print("struct C2SRow { int nnz; int f[C2S_MAXNNZ]; double c[C2S_MAXNNZ]; };")
    print("// C2S_ROWS[l][m] for m < 2l+1 (l >= 2) or m < ncart(l) (l <= 1)")
    print("__device__ __constant__ const C2SRow C2S_ROWS[%d][%d] = {" % (LMAX + 1, 2 * LMAX + 1))
    for l in range(LMAX + 1):
        print("  {")
        nrow = 2 * l + 1 if l >= 2 else (l + 1) * (l + 2) // 2
        for m in range(2 * LMAX + 1):
            nz = rows.get((l, m), []) if m < nrow else []
            fs = [f for f, _ in nz] + [0] * (maxnnz - len(nz))
            cs = [mp.nstr(v, 20, strip_zeros=False) for _, v in nz] + ["0.0"] * (maxnnz - len(nz))
            print("    {%d, {%s}, {%s}}," % (len(nz), ", ".join(map(str, fs)), ", ".join(cs)))
        print("  },")
    print("};")
    print("}  // namespace cintx")


if __name__ == "__main__":
    main()
