/*
 * Oracle Rys quadrature (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * The Rys quadrature of order n for parameter x is the n-point Gauss rule for the weight
 * exp(-x t^2) on t in [0,1], written in the variable s = t^2:
 *     int_0^1 exp(-x t^2) P(t^2) dt = sum_r w_r P(s_r)   for deg P <= 2n-1.
 * libcint computes it with per-n polynomial fits (n <= 5) and Jacobi/Wheeler moment methods
 * in 80-bit long double (n >= 6) (rys_roots.c:57-126, rys_wheeler.c:3667-3703).  This oracle
 * uses a different, self-checking route: the discretised Stieltjes procedure (Gautschi,
 * "Orthogonal Polynomials: Computation and Approximation", 2004, sec. 2.2.3) over a 256-point
 * Gauss-Legendre rule on [0, T], followed by the Golub-Welsch eigenproblem solved by cyclic
 * Jacobi rotations, all in long double.  T = min(1, sqrt(L/x)) with L = 200 so the discarded
 * tail exp(-x t^2) < e^-200 of every moment up to degree 2n-1 that matters for n <= 16.
 */
#include <math.h>
#include <string.h>
#include "oracle.h"

#define GL_M 256
#define MAXN 16
static long double gl_x[GL_M], gl_w[GL_M]; /* Gauss-Legendre nodes/weights on [0,1] */

/* Legendre nodes by Newton iteration on P_M with the three-term recurrence. */
__attribute__((constructor)) static void gl_init(void)
{
        const int m = GL_M;
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int i = 0; i < (m + 1) / 2; i++) {
                long double z = cosl(pi * (i + 0.75L) / (m + 0.5L));
                long double dp = 1;
                for (int it = 0; it < 100; it++) {
                        long double p0 = 1, p1 = z;
                        for (int k = 2; k <= m; k++) {
                                long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                                p0 = p1;
                                p1 = p2;
                        }
                        dp = m * (z * p1 - p0) / (z * z - 1);
                        long double dz = p1 / dp;
                        z -= dz;
                        if (fabsl(dz) < 1e-21L) {
                                break;
                        }
                }
                long double w = 2 / ((1 - z * z) * dp * dp);
                /* map [-1,1] -> [0,1] */
                gl_x[i] = 0.5L * (1 - z);
                gl_x[m - 1 - i] = 0.5L * (1 + z);
                gl_w[i] = gl_w[m - 1 - i] = 0.5L * w;
        }
}

/* Eigen-decomposition of a symmetric n x n matrix by cyclic Jacobi rotations.
 * On return a[] holds eigenvalues on its diagonal, v[] the eigenvectors (columns). */
static void jacobi_eig(int n, long double *a, long double *v)
{
        for (int i = 0; i < n; i++) {
                for (int j = 0; j < n; j++) {
                        v[i * n + j] = (i == j);
                }
        }
        for (int sweep = 0; sweep < 100; sweep++) {
                long double off = 0, diag = 0;
                for (int i = 0; i < n; i++) {
                        diag += a[i * n + i] * a[i * n + i];
                        for (int j = i + 1; j < n; j++) {
                                off += a[i * n + j] * a[i * n + j];
                        }
                }
                if (off <= 1e-44L * diag || off == 0) {
                        break;
                }
                for (int p = 0; p < n; p++) {
                        for (int q = p + 1; q < n; q++) {
                                long double apq = a[p * n + q];
                                if (apq == 0) {
                                        continue;
                                }
                                long double theta = (a[q * n + q] - a[p * n + p]) / (2 * apq);
                                long double t = (theta >= 0 ? 1 : -1) /
                                                (fabsl(theta) + sqrtl(theta * theta + 1));
                                long double c = 1 / sqrtl(t * t + 1), s = t * c;
                                for (int k = 0; k < n; k++) { /* columns p, q */
                                        long double akp = a[k * n + p], akq = a[k * n + q];
                                        a[k * n + p] = c * akp - s * akq;
                                        a[k * n + q] = s * akp + c * akq;
                                }
                                for (int k = 0; k < n; k++) { /* rows p, q */
                                        long double apk = a[p * n + k], aqk = a[q * n + k];
                                        a[p * n + k] = c * apk - s * aqk;
                                        a[q * n + k] = s * apk + c * aqk;
                                }
                                for (int k = 0; k < n; k++) {
                                        long double vkp = v[k * n + p], vkq = v[k * n + q];
                                        v[k * n + p] = c * vkp - s * vkq;
                                        v[k * n + q] = s * vkp + c * vkq;
                                }
                        }
                }
        }
}

static int rys_ld(int n, long double x, long double *s_out, long double *w_out)
{
        if (n < 1 || n > MAXN || !(x >= 0)) {
                return 1;
        }
        const long double L = 200.0L;
        long double T = 1;
        if (x > L) {
                T = sqrtl(L / x);
        }
        long double s[GL_M], om[GL_M], p[GL_M], pm[GL_M];
        long double mu0 = 0;
        for (int j = 0; j < GL_M; j++) {
                long double t = T * gl_x[j];
                s[j] = t * t;
                om[j] = T * gl_w[j] * expl(-x * t * t);
                mu0 += om[j];
        }
        long double a[MAXN], b[MAXN + 1];
        long double inv = 1 / sqrtl(mu0);
        for (int j = 0; j < GL_M; j++) {
                p[j] = inv;
                pm[j] = 0;
        }
        b[0] = 0;
        for (int k = 0; k < n; k++) {
                long double alpha = 0;
                for (int j = 0; j < GL_M; j++) {
                        alpha += om[j] * s[j] * p[j] * p[j];
                }
                long double nrm = 0;
                for (int j = 0; j < GL_M; j++) {
                        long double q = (s[j] - alpha) * p[j] - b[k] * pm[j];
                        pm[j] = p[j];
                        p[j] = q;
                        nrm += om[j] * q * q;
                }
                a[k] = alpha;
                b[k + 1] = sqrtl(nrm);
                long double r = 1 / b[k + 1];
                for (int j = 0; j < GL_M; j++) {
                        p[j] *= r;
                }
        }
        long double J[MAXN * MAXN], V[MAXN * MAXN];
        memset(J, 0, sizeof(J));
        for (int k = 0; k < n; k++) {
                J[k * n + k] = a[k];
                if (k + 1 < n) {
                        J[k * n + k + 1] = J[(k + 1) * n + k] = b[k + 1];
                }
        }
        jacobi_eig(n, J, V);
        /* sort ascending */
        int order[MAXN];
        for (int i = 0; i < n; i++) {
                order[i] = i;
        }
        for (int i = 1; i < n; i++) {
                for (int j = i; j > 0 && J[order[j] * n + order[j]] < J[order[j - 1] * n + order[j - 1]]; j--) {
                        int t = order[j];
                        order[j] = order[j - 1];
                        order[j - 1] = t;
                }
        }
        for (int i = 0; i < n; i++) {
                int r = order[i];
                s_out[i] = J[r * n + r];
                w_out[i] = mu0 * V[0 * n + r] * V[0 * n + r];
        }
        return 0;
}

int oracle_rys_t2(int n, double x, double *t2, double *w)
{
        long double s[MAXN], ww[MAXN];
        int err = rys_ld(n, x, s, ww);
        if (err) {
                return err;
        }
        for (int i = 0; i < n; i++) {
                t2[i] = (double)s[i];
                w[i] = (double)ww[i];
        }
        return 0;
}

int oracle_rys_roots(int n, double x, double *u, double *w)
{
        long double s[MAXN], ww[MAXN];
        int err = rys_ld(n, x, s, ww);
        if (err) {
                return err;
        }
        for (int i = 0; i < n; i++) {
                u[i] = (double)(s[i] / (1 - s[i]));
                w[i] = (double)ww[i];
        }
        return 0;
}

/* F_m(x) = int_0^1 t^{2m} exp(-x t^2) dt by the same Gauss-Legendre rule on [0, T]. */
void oracle_boys(int mmax, double x, double *f)
{
        const long double L = 200.0L;
        long double T = 1;
        if (x > L) {
                T = sqrtl(L / (long double)x);
        }
        for (int m = 0; m <= mmax; m++) {
                long double acc = 0;
                for (int j = 0; j < GL_M; j++) {
                        long double t = T * gl_x[j];
                        acc += T * gl_w[j] * powl(t, 2 * m) * expl(-(long double)x * t * t);
                }
                f[m] = (double)acc;
        }
}
