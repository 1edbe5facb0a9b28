/*
 * Oracle electron-repulsion integrals over contracted cartesian/spherical GTOs
 * (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Restates libcint 6.1.3's Rys-quadrature path in a direct form:
 *   - shell data and the exponent screening of CINT2e_loop_nopt (cint2e.c:57-300) and
 *     CINTset_pairdata (optimizer.c:288-342): a primitive pair is dropped when
 *     cceij = ai*aj/(ai+aj)*|Rij|^2 - log_rr - log|c_i|max - log|c_j|max exceeds the cutoff,
 *     with log_rr = 1.7 - 1.5*log(a_i,last + a_j,last) + (li+lj)*log(|Rij|+1);
 *   - the per-primitive prefactor of CINTg0_2e (g2e.c:4425-4475):
 *     fac = common_factor * c_i c_j c_k c_l * exp(-eij) * exp(-ekl) * sqrt(a0 / (aij akl)^3),
 *     common_factor = pi^3 * 2/sqrt(pi) * prod common_fac_sp(l)    (g2e.c:54-56, g1e.c:566);
 *   - the Rys coefficients b00, b10, b01, c00, c0p of g2e.c:4542-4565 written in t^2 form;
 *   - the 2D vertical recurrence (CINTg0_2e_2d, g2e.c:272) built on centres i and k and the
 *     horizontal transfer to j and l (the HRR of g2e.c:428-694), with each pair's shells taken in
 *     the order that puts the recurrence on its stable centre (base_first) and the block
 *     transposed back to the requested order;
 *   - the cartesian product sum of CINTgout2e (cint2e.c:961) and contraction (g1e.c:509);
 *   - the cartesian -> spherical transform of c2s_sph_2e1 (cart2sph.c:5324) / c2s_sph_3c2e1
 *     (cart2sph.c:5884) / c2s_sph_1e (cart2sph.c:4833).
 * 3-centre (ij|k) is (ij|k s0) and 2-centre (i|k) is (i s0|k s0), where s0 is a unit s
 * function with exponent 0, as in CINTinit_int3c2e_EnvVars (g3c2e.c:21, k in the l slot).
 * Roots come from oracle_rys_t2 (rys_oracle.c), not from libcint's tables.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "oracle.h"

#define LMAX 6
#define NRMAX 16
#define PTR_EXPCUTOFF 0
#define PTR_COORD 1
#define ATM_SLOTS 6
#define BAS_SLOTS 8

typedef struct {
        int l, nprim, nctr;
        const double *ai;
        const double *ci; /* column-major [ctr][prim] */
        double r[3];
        double log_maxc[64];
        int unit; /* 1 for the s0 placeholder */
} Shell;

static const double zero_exp = 0.0, unit_coef = 1.0;

static void load_shell(Shell *s, int sh, const int *atm, const int *bas, const double *env)
{
        const int *b = bas + BAS_SLOTS * sh;
        s->l = b[1];
        s->nprim = b[2];
        s->nctr = b[3];
        s->ai = env + b[5];
        s->ci = env + b[6];
        const double *r = env + atm[ATM_SLOTS * b[0] + PTR_COORD];
        s->r[0] = r[0];
        s->r[1] = r[1];
        s->r[2] = r[2];
        s->unit = 0;
        for (int p = 0; p < s->nprim; p++) {
                double m = 0;
                for (int c = 0; c < s->nctr; c++) {
                        double v = fabs(s->ci[c * s->nprim + p]);
                        m = v > m ? v : m;
                }
                s->log_maxc[p] = log(m);
        }
}

static void unit_shell(Shell *s, const double *r)
{
        s->l = 0;
        s->nprim = 1;
        s->nctr = 1;
        s->ai = &zero_exp;
        s->ci = &unit_coef;
        s->r[0] = r[0];
        s->r[1] = r[1];
        s->r[2] = r[2];
        s->log_maxc[0] = 0;
        s->unit = 1;
}

static int ncart(int l)
{
        return (l + 1) * (l + 2) / 2;
}

static double common_fac_sp(int l)
{
        if (l == 0) {
                return 0.282094791773878143;
        } else if (l == 1) {
                return 0.488602511902919921;
        }
        return 1;
}

/* cartesian exponents in libcint order */
static void cart_list(int l, int *lx, int *ly, int *lz)
{
        int n = 0;
        for (int x = l; x >= 0; x--) {
                for (int y = l - x; y >= 0; y--) {
                        lx[n] = x;
                        ly[n] = y;
                        lz[n] = l - x - y;
                        n++;
                }
        }
}

typedef struct {
        int n;                  /* number of surviving primitive pairs */
        int ip[64 * 64], jp[64 * 64];
        double cce[64 * 64];
        double e[64 * 64];      /* exp(-ai aj/aij |Rij|^2) */
        double p[64 * 64][3];   /* product centre */
        int empty;
} PairList;

/* CINTset_pairdata semantics (optimizer.c:288-342); a unit shell contributes log_rr = 0. */
static void pair_list(PairList *pl, const Shell *a, const Shell *b, double cutoff)
{
        double d[3] = {a->r[0] - b->r[0], a->r[1] - b->r[1], a->r[2] - b->r[2]};
        double rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        double log_rr = 0;
        if (!b->unit) {
                double aij = a->ai[a->nprim - 1] + b->ai[b->nprim - 1];
                log_rr = 1.7 - 1.5 * log(aij);
                int lij = a->l + b->l;
                if (lij > 0) {
                        log_rr += lij * log(sqrt(rr) + 1);
                }
        }
        pl->n = 0;
        pl->empty = 1;
        for (int jp = 0; jp < b->nprim; jp++) {
                for (int ip = 0; ip < a->nprim; ip++) {
                        double ai = a->ai[ip], aj = b->ai[jp];
                        double inv = 1 / (ai + aj);
                        double eij = rr * ai * aj * inv;
                        double cce = b->unit ? 0 : eij - log_rr - a->log_maxc[ip] - b->log_maxc[jp];
                        if (cce < cutoff) {
                                int n = pl->n++;
                                pl->ip[n] = ip;
                                pl->jp[n] = jp;
                                pl->cce[n] = cce;
                                pl->e[n] = exp(-eij);
                                double wj = aj * inv;
                                for (int x = 0; x < 3; x++) {
                                        pl->p[n][x] = a->r[x] + wj * (b->r[x] - a->r[x]);
                                }
                                pl->empty = 0;
                        }
                }
        }
}

/*
 * Cartesian block, contracted, layout cart[fi + nfi*(fj + nfj*(fk + nfk*fl))] per
 * contraction tuple (ci,cj,ck,cl) at offset ((cl*nck + ck)*ncj + cj)*nci + ci times nf.
 */
static int eri4c_cart(double *gctr, const Shell *si, const Shell *sj, const Shell *sk,
                      const Shell *sl, double common, double expcutoff, int kl_screen)
{
        const int li = si->l, lj = sj->l, lk = sk->l, ll = sl->l;
        const int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
        const int nf = nfi * nfj * nfk * nfl;
        const int nctr = si->nctr * sj->nctr * sk->nctr * sl->nctr;
        const int nroots = (li + lj + lk + ll) / 2 + 1;
        const int nmax = li + lj, mmax = lk + ll;
        memset(gctr, 0, sizeof(double) * nf * nctr);

        static __thread PairList pij, pkl;
        pair_list(&pij, si, sj, expcutoff);
        if (pij.empty) {
                return 0;
        }
        pair_list(&pkl, sk, sl, expcutoff);

        int ix[4][64], iy[4][64], iz[4][64];
        cart_list(li, ix[0], iy[0], iz[0]);
        cart_list(lj, ix[1], iy[1], iz[1]);
        cart_list(lk, ix[2], iy[2], iz[2]);
        cart_list(ll, ix[3], iy[3], iz[3]);
        const double ab[3] = {si->r[0] - sj->r[0], si->r[1] - sj->r[1], si->r[2] - sj->r[2]};
        const double cd[3] = {sk->r[0] - sl->r[0], sk->r[1] - sl->r[1], sk->r[2] - sl->r[2]};

        /* g2d[axis][root][n][m] then I[axis][root][i][j][k][l] */
        const int dim2 = (nmax + 1) * (mmax + 1);
        const int d_i = LMAX + 1;
        double *g2 = malloc(sizeof(double) * 3 * nroots * dim2);
        double *tmp = malloc(sizeof(double) * (nmax + 1) * (lj + 1) * (mmax + 1));
        size_t isz = (size_t)(li + 1) * (lj + 1) * (lk + 1) * (ll + 1);
        double *I = malloc(sizeof(double) * 3 * nroots * isz);
        double *gprim = malloc(sizeof(double) * nf);
        (void)d_i;
        int any = 0;

        for (int b = 0; b < pkl.n; b++) {
                double ak = sk->ai[pkl.ip[b]], al = sl->ai[pkl.jp[b]];
                double akl = ak + al;
                double cutoff_ij = kl_screen ? expcutoff - pkl.cce[b] : expcutoff;
                if (kl_screen && pkl.cce[b] > expcutoff) {
                        continue;
                }
                for (int a = 0; a < pij.n; a++) {
                        if (pij.cce[a] > cutoff_ij) {
                                continue;
                        }
                        any = 1;
                        double ai = si->ai[pij.ip[a]], aj = sj->ai[pij.jp[a]];
                        double aij = ai + aj;
                        double a1 = aij * akl;
                        double a0 = a1 / (aij + akl);
                        double pq[3], rr = 0;
                        for (int x = 0; x < 3; x++) {
                                pq[x] = pij.p[a][x] - pkl.p[b][x];
                                rr += pq[x] * pq[x];
                        }
                        double fac = common * pij.e[a] * pkl.e[b] * sqrt(a0 / (a1 * a1 * a1));
                        double t2[NRMAX], w[NRMAX];
                        oracle_rys_t2(nroots, a0 * rr, t2, w);
                        for (int r = 0; r < nroots; r++) {
                                double rt_aa = t2[r] / (aij + akl);
                                double b00 = 0.5 * rt_aa;
                                double b10 = 0.5 / aij * (1 - rt_aa * akl);
                                double b01 = 0.5 / akl * (1 - rt_aa * aij);
                                for (int x = 0; x < 3; x++) {
                                        double c00 = pij.p[a][x] - si->r[x] - rt_aa * akl * pq[x];
                                        double c0p = pkl.p[b][x] - sk->r[x] + rt_aa * aij * pq[x];
                                        double *G = g2 + (x * nroots + r) * dim2;
#define G2(n, m) G[(n) * (mmax + 1) + (m)]
                                        G2(0, 0) = (x == 2) ? w[r] * fac : 1.0;
                                        if (nmax > 0) {
                                                G2(1, 0) = c00 * G2(0, 0);
                                        }
                                        for (int n = 1; n < nmax; n++) {
                                                G2(n + 1, 0) = c00 * G2(n, 0) + n * b10 * G2(n - 1, 0);
                                        }
                                        for (int m = 0; m < mmax; m++) {
                                                for (int n = 0; n <= nmax; n++) {
                                                        double v = c0p * G2(n, m);
                                                        if (m > 0) {
                                                                v += m * b01 * G2(n, m - 1);
                                                        }
                                                        if (n > 0) {
                                                                v += n * b00 * G2(n - 1, m);
                                                        }
                                                        G2(n, m + 1) = v;
                                                }
                                        }
                                        /* HRR: (n, m) -> (i, j, m) with j from (A - B) */
                                        for (int m = 0; m <= mmax; m++) {
                                                for (int n = 0; n <= nmax; n++) {
                                                        tmp[(n * (lj + 1) + 0) * (mmax + 1) + m] = G2(n, m);
                                                }
                                                for (int j = 1; j <= lj; j++) {
                                                        for (int n = 0; n + j <= nmax; n++) {
                                                                tmp[(n * (lj + 1) + j) * (mmax + 1) + m] =
                                                                        tmp[((n + 1) * (lj + 1) + j - 1) * (mmax + 1) + m] +
                                                                        ab[x] * tmp[(n * (lj + 1) + j - 1) * (mmax + 1) + m];
                                                        }
                                                }
                                        }
#undef G2
                                        /* (i, j, m) -> (i, j, k, l) with l from (C - D) */
                                        double *Ix = I + (x * nroots + r) * isz;
                                        for (int i = 0; i <= li; i++) {
                                                for (int j = 0; j <= lj; j++) {
                                                        double h[2 * LMAX + 2][LMAX + 1];
                                                        for (int m = 0; m <= mmax; m++) {
                                                                h[m][0] = tmp[(i * (lj + 1) + j) * (mmax + 1) + m];
                                                        }
                                                        for (int l = 1; l <= ll; l++) {
                                                                for (int m = 0; m + l <= mmax; m++) {
                                                                        h[m][l] = h[m + 1][l - 1] + cd[x] * h[m][l - 1];
                                                                }
                                                        }
                                                        for (int k = 0; k <= lk; k++) {
                                                                for (int l = 0; l <= ll; l++) {
                                                                        Ix[((i * (lj + 1) + j) * (lk + 1) + k) * (ll + 1) + l] = h[k][l];
                                                                }
                                                        }
                                                }
                                        }
                                }
                        }
                        /* cartesian products summed over roots */
                        int n = 0;
                        for (int fl = 0; fl < nfl; fl++) {
                                for (int fk = 0; fk < nfk; fk++) {
                                        for (int fj = 0; fj < nfj; fj++) {
                                                for (int fi = 0; fi < nfi; fi++, n++) {
                                                        size_t ox = ((ix[0][fi] * (lj + 1) + ix[1][fj]) * (lk + 1) + ix[2][fk]) * (ll + 1) + ix[3][fl];
                                                        size_t oy = ((iy[0][fi] * (lj + 1) + iy[1][fj]) * (lk + 1) + iy[2][fk]) * (ll + 1) + iy[3][fl];
                                                        size_t oz = ((iz[0][fi] * (lj + 1) + iz[1][fj]) * (lk + 1) + iz[2][fk]) * (ll + 1) + iz[3][fl];
                                                        double s = 0;
                                                        for (int r = 0; r < nroots; r++) {
                                                                s += I[(0 * nroots + r) * isz + ox] *
                                                                     I[(1 * nroots + r) * isz + oy] *
                                                                     I[(2 * nroots + r) * isz + oz];
                                                        }
                                                        gprim[n] = s;
                                                }
                                        }
                                }
                        }
                        /* contraction */
                        int pi = pij.ip[a], pj = pij.jp[a], pk = pkl.ip[b], pl = pkl.jp[b];
                        for (int cl = 0; cl < sl->nctr; cl++) {
                                double c4 = sl->ci[cl * sl->nprim + pl];
                                for (int ck = 0; ck < sk->nctr; ck++) {
                                        double c3 = c4 * sk->ci[ck * sk->nprim + pk];
                                        for (int cj = 0; cj < sj->nctr; cj++) {
                                                double c2 = c3 * sj->ci[cj * sj->nprim + pj];
                                                for (int ci = 0; ci < si->nctr; ci++) {
                                                        double c1 = c2 * si->ci[ci * si->nprim + pi];
                                                        size_t t = ((cl * sk->nctr + ck) * sj->nctr + cj) * si->nctr + ci;
                                                        double *dst = gctr + t * nf;
                                                        for (int f = 0; f < nf; f++) {
                                                                dst[f] += c1 * gprim[f];
                                                        }
                                                }
                                        }
                                }
                        }
                }
        }
        free(g2);
        free(tmp);
        free(I);
        free(gprim);
        return any;
}

/* Write the contracted cartesian block into libcint's output layout, optionally
 * transforming each axis to real spherical harmonics. */
static void write_block(double *out, const double *gctr, const Shell *s[4], int nsh, int sph)
{
        int nf[4], no[4], nc[4], l[4];
        for (int a = 0; a < 4; a++) {
                l[a] = a < nsh ? s[a]->l : 0;
                nc[a] = a < nsh ? s[a]->nctr : 1;
                nf[a] = ncart(l[a]);
                no[a] = sph ? 2 * l[a] + 1 : nf[a];
        }
        double *mats[4];
        for (int a = 0; a < 4; a++) {
                mats[a] = malloc(sizeof(double) * (2 * LMAX + 1) * ncart(LMAX));
                if (sph) {
                        oracle_c2s_matrix(l[a], mats[a]);
                } else {
                        memset(mats[a], 0, sizeof(double) * no[a] * nf[a]);
                        for (int i = 0; i < nf[a]; i++) {
                                mats[a][i * nf[a] + i] = 1;
                        }
                }
        }
        const int ni = no[0] * nc[0], nj = no[1] * nc[1], nk = no[2] * nc[2];
        const int nfall = nf[0] * nf[1] * nf[2] * nf[3];
        for (int c3 = 0; c3 < nc[3]; c3++)
        for (int c2 = 0; c2 < nc[2]; c2++)
        for (int c1 = 0; c1 < nc[1]; c1++)
        for (int c0 = 0; c0 < nc[0]; c0++) {
                size_t t = ((c3 * nc[2] + c2) * nc[1] + c1) * nc[0] + c0;
                const double *g = gctr + t * nfall;
                for (int m3 = 0; m3 < no[3]; m3++)
                for (int m2 = 0; m2 < no[2]; m2++)
                for (int m1 = 0; m1 < no[1]; m1++)
                for (int m0 = 0; m0 < no[0]; m0++) {
                        double v = 0;
                        for (int f3 = 0; f3 < nf[3]; f3++) {
                                double w3 = mats[3][m3 * nf[3] + f3];
                                if (w3 == 0) continue;
                                for (int f2 = 0; f2 < nf[2]; f2++) {
                                        double w2 = w3 * mats[2][m2 * nf[2] + f2];
                                        if (w2 == 0) continue;
                                        for (int f1 = 0; f1 < nf[1]; f1++) {
                                                double w1 = w2 * mats[1][m1 * nf[1] + f1];
                                                if (w1 == 0) continue;
                                                for (int f0 = 0; f0 < nf[0]; f0++) {
                                                        double w0 = w1 * mats[0][m0 * nf[0] + f0];
                                                        if (w0 == 0) continue;
                                                        v += w0 * g[((f3 * nf[2] + f2) * nf[1] + f1) * nf[0] + f0];
                                                }
                                        }
                                }
                        }
                        size_t i0 = c0 * no[0] + m0, i1 = c1 * no[1] + m1;
                        size_t i2 = c2 * no[2] + m2, i3 = c3 * no[3] + m3;
                        out[i0 + ni * (i1 + nj * (i2 + (size_t)nk * i3))] = v;
                }
        }
        for (int a = 0; a < 4; a++) {
                free(mats[a]);
        }
}

static size_t block_size(const Shell *s[4], int nsh, int sph)
{
        size_t n = 1;
        for (int a = 0; a < nsh; a++) {
                n *= (size_t)(sph ? 2 * s[a]->l + 1 : ncart(s[a]->l)) * s[a]->nctr;
        }
        return n;
}

static int run(int sph, double *out, int nsh, const int *shls, const int *atm, const int *bas,
               const double *env)
{
        Shell sh[4];
        for (int a = 0; a < nsh; a++) {
                load_shell(&sh[a], shls[a], atm, bas, env);
        }
        double common = 3.14159265358979323846 * 3.14159265358979323846 * 3.14159265358979323846 *
                        2 / 1.7724538509055160272981674833411451;
        double expcutoff;
        if (nsh == 4) {
                expcutoff = env[PTR_EXPCUTOFF] == 0 ? 60 : fmax(40, env[PTR_EXPCUTOFF]) + 1;
        } else {
                expcutoff = env[PTR_EXPCUTOFF] == 0 ? 60 : fmax(40, env[PTR_EXPCUTOFF]);
        }
        const Shell *s4[4];
        Shell u1, u2;
        if (nsh == 4) {
                s4[0] = &sh[0]; s4[1] = &sh[1]; s4[2] = &sh[2]; s4[3] = &sh[3];
        } else if (nsh == 3) {
                unit_shell(&u1, sh[2].r);
                s4[0] = &sh[0]; s4[1] = &sh[1]; s4[2] = &sh[2]; s4[3] = &u1;
        } else {
                unit_shell(&u1, sh[0].r);
                unit_shell(&u2, sh[1].r);
                s4[0] = &sh[0]; s4[1] = &u1; s4[2] = &sh[1]; s4[3] = &u2;
        }
        for (int a = 0; a < 4; a++) {
                if (!s4[a]->unit) {
                        common *= common_fac_sp(s4[a]->l);
                }
        }
        size_t nf = (size_t)ncart(s4[0]->l) * ncart(s4[1]->l) * ncart(s4[2]->l) * ncart(s4[3]->l);
        size_t nctr = (size_t)s4[0]->nctr * s4[1]->nctr * s4[2]->nctr * s4[3]->nctr;
        double *gctr = malloc(sizeof(double) * nf * nctr);
        int ok = eri4c_cart(gctr, s4[0], s4[1], s4[2], s4[3], common, expcutoff, nsh == 4);
        const Shell *sp[4] = {&sh[0], &sh[1], &sh[2], &sh[3]};
        if (nsh == 2) {
                /* the block is (i|k): reuse the 4-slot writer with ordered shells i, k */
                const Shell *q[4] = {&sh[0], &sh[1], 0, 0};
                Shell e1, e2;
                unit_shell(&e1, sh[0].r);
                unit_shell(&e2, sh[0].r);
                q[2] = &e1;
                q[3] = &e2;
                /* reorder cart block from (i, s0, k, s0) = (i, k) already contiguous */
                if (ok) {
                        write_block(out, gctr, q, 2, sph);
                } else {
                        memset(out, 0, sizeof(double) * block_size(q, 2, sph));
                }
        } else {
                if (nsh == 3) {
                        Shell e;
                        unit_shell(&e, sh[2].r);
                        sp[3] = &e;
                        if (ok) {
                                write_block(out, gctr, sp, 3, sph);
                        } else {
                                memset(out, 0, sizeof(double) * block_size(sp, 3, sph));
                        }
                } else {
                        if (ok) {
                                write_block(out, gctr, sp, 4, sph);
                        } else {
                                memset(out, 0, sizeof(double) * block_size(sp, 4, sph));
                        }
                }
        }
        free(gctr);
        return ok;
}

/*
 * Recurrence centre of the pair (sx, sy): the shell of higher l and, for equal l, the one whose
 * recurrence cancels least, i.e. the smaller max over primitive pairs of a_y |X - Y| /
 * sqrt(a_x + a_y) (ties: the larger shell index).  libcint builds on the higher l and, for equal
 * l, on the second shell (ibase = li > lj, g2e.c:101); on a diffuse/tight pair far apart that
 * choice loses digits to cancellation (a (ff|ff) block of a 0.17 / 2253 exponent pair 4 bohr apart
 * is 6% off), so this restatement takes the stable centre and transposes the block back.
 */
static int base_first(int sx, int sy, const int *atm, const int *bas, const double *env)
{
        Shell x, y;
        load_shell(&x, sx, atm, bas, env);
        load_shell(&y, sy, atm, bas, env);
        if (x.l != y.l) {
                return x.l > y.l;
        }
        if (sx == sy) {
                return 1;
        }
        double d = sqrt((x.r[0] - y.r[0]) * (x.r[0] - y.r[0]) + (x.r[1] - y.r[1]) * (x.r[1] - y.r[1]) +
                        (x.r[2] - y.r[2]) * (x.r[2] - y.r[2]));
        double on_x = 0, on_y = 0;
        for (int p = 0; p < x.nprim; p++) {
                for (int q = 0; q < y.nprim; q++) {
                        double r = d / sqrt(x.ai[p] + y.ai[q]);
                        on_x = fmax(on_x, y.ai[q] * r);
                        on_y = fmax(on_y, x.ai[p] * r);
                }
        }
        if (!(on_x != on_y) || fabs(on_x - on_y) <= 1e-12 * fmax(on_x, on_y)) {
                return sx >= sy;
        }
        return on_x < on_y;
}

static int axis_len(int sh, const int *bas, int sph)
{
        int l = bas[BAS_SLOTS * sh + 1];
        return (sph ? 2 * l + 1 : ncart(l)) * bas[BAS_SLOTS * sh + 3];
}

/* run() on the shells in stable-centre order, with the block written in the requested order */
static int run_oriented(int sph, double *out, int nsh, const int *shls, const int *atm, const int *bas,
                        const double *env)
{
        int ord[4] = {0, 1, 2, 3};
        if (nsh >= 3 && !base_first(shls[0], shls[1], atm, bas, env)) {
                ord[0] = 1;
                ord[1] = 0;
        }
        if (nsh == 4 && !base_first(shls[2], shls[3], atm, bas, env)) {
                ord[2] = 3;
                ord[3] = 2;
        }
        if (ord[0] == 0 && ord[2] == 2) {
                return run(sph, out, nsh, shls, atm, bas, env);
        }
        int s2[4], n[4] = {1, 1, 1, 1};
        for (int a = 0; a < nsh; a++) {
                s2[a] = shls[ord[a]];
                n[a] = axis_len(shls[a], bas, sph);
        }
        size_t tot = (size_t)n[0] * n[1] * n[2] * n[3];
        double *tmp = malloc(sizeof(double) * tot);
        int ok = run(sph, tmp, nsh, s2, atm, bas, env);
        /* tmp axis a is requested axis ord[a] */
        int m[4];
        for (int a = 0; a < 4; a++) {
                m[a] = n[ord[a]];
        }
        for (size_t e = 0; e < tot; e++) {
                size_t r = e, idx[4];
                for (int a = 0; a < 4; a++) {
                        idx[ord[a]] = r % m[a];
                        r /= m[a];
                }
                out[idx[0] + n[0] * (idx[1] + n[1] * (idx[2] + n[2] * idx[3]))] = tmp[e];
        }
        free(tmp);
        return ok;
}

int oracle_int2e(int sph, double *out, const int *shls, const int *atm, int natm,
                 const int *bas, int nbas, const double *env)
{
        (void)natm;
        (void)nbas;
        return run_oriented(sph, out, 4, shls, atm, bas, env);
}

int oracle_int3c2e(int sph, double *out, const int *shls, const int *atm, int natm,
                   const int *bas, int nbas, const double *env)
{
        (void)natm;
        (void)nbas;
        return run_oriented(sph, out, 3, shls, atm, bas, env);
}

int oracle_int2c2e(int sph, double *out, const int *shls, const int *atm, int natm,
                   const int *bas, int nbas, const double *env)
{
        (void)natm;
        (void)nbas;
        int s2[2] = {shls[0], shls[1]};
        return run(sph, out, 2, s2, atm, bas, env);
}

void oracle_int2e_batch(int sph, double *out, const long long *offsets, const int *quartets,
                        long long nq, const int *atm, int natm, const int *bas, int nbas,
                        const double *env, int nthreads)
{
        if (nthreads > 0) {
                omp_set_num_threads(nthreads);
        }
#pragma omp parallel for schedule(dynamic, 4)
        for (long long q = 0; q < nq; q++) {
                oracle_int2e(sph, out + offsets[q], quartets + 4 * q, atm, natm, bas, nbas, env);
        }
}
