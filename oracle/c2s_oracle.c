/*
 * Oracle cartesian -> real spherical transform (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Rows are m = -l..l, columns the cartesian monomials x^a y^b z^c in libcint order
 * (a descending, then b descending; libcint `CINTcart_comp`).  Coefficients are those of the
 * regular real solid harmonics S_lm (Helgaker, Jorgensen & Olsen, "Molecular
 * Electronic-Structure Theory", eq. 6.4.47-6.4.50; Schlegel & Frisch, IJQC 54 (1995) 83)
 * scaled by sqrt((2l+1)/(4 pi)), which is libcint's normalisation of the spherical GTOs for
 * l >= 2 (cart2sph.c g_trans_cart2sph tables).  For l = 0, 1 libcint uses the identity and
 * moves sqrt((2l+1)/(4 pi)) into the common factor (g1e.c:566 CINTcommon_fac_sp); callers
 * of this function get the identity for l <= 1 to match that convention.
 */
#include <math.h>
#include <string.h>
#include "oracle.h"

static double fact(int n)
{
        double r = 1;
        for (int i = 2; i <= n; i++) {
                r *= i;
        }
        return r;
}

static double binom(int n, int k)
{
        if (k < 0 || k > n) {
                return 0;
        }
        return fact(n) / (fact(k) * fact(n - k));
}

static int cart_index(int l, int a, int b)
{
        /* position of x^a y^b z^(l-a-b) in libcint order */
        int idx = 0;
        for (int lx = l; lx > a; lx--) {
                idx += l - lx + 1;
        }
        return idx + (l - a - b);
}

void oracle_c2s_matrix(int l, double *mat)
{
        int nc = (l + 1) * (l + 2) / 2;
        memset(mat, 0, sizeof(double) * (2 * l + 1) * nc);
        if (l <= 1) {
                for (int i = 0; i < nc; i++) {
                        mat[i * nc + i] = 1;
                }
                return;
        }
        const double pi = 3.14159265358979323846;
        double scale = sqrt((2 * l + 1) / (4 * pi));
        for (int m = -l; m <= l; m++) {
                int am = m < 0 ? -m : m;
                double nlm = sqrt(2 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0)) /
                             (pow(2, am) * fact(l));
                /* v runs over integers (m >= 0) or half-integers (m < 0); use 2v */
                int twovm = m < 0 ? 1 : 0;
                for (int t = 0; t <= (l - am) / 2; t++) {
                        for (int u = 0; u <= t; u++) {
                                for (int twov = twovm; twov <= am; twov += 2) {
                                        int sgn_exp = t + (twov - twovm) / 2;
                                        double c = ((sgn_exp & 1) ? -1 : 1) * pow(0.25, t) *
                                                   binom(l, t) * binom(l - t, am + t) *
                                                   binom(t, u) * binom(am, twov);
                                        int ex = 2 * t + am - 2 * u - twov;
                                        int ey = 2 * u + twov;
                                        mat[(m + l) * nc + cart_index(l, ex, ey)] += scale * nlm * c;
                                }
                        }
                }
        }
}
