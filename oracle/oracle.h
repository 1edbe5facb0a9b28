/*
 * CPU oracle for the two-electron Rys-quadrature integrals (TEST INFRASTRUCTURE ONLY).
 *
 * This is an independent restatement, in plain C with long-double root finding, of the
 * mathematics libcint 6.1.3 implements for int2e / int2c2e / int3c2e.  Only the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it; the product library never
 * links it.  It is pinned against libcint compiled from the reference sources (oracle/_ref)
 * and against golden vectors committed under tests/golden.
 *
 * Output layouts and return values follow libcint with dims == NULL:
 *   int2e:  out[i + ni*(j + nj*(k + nk*l))], axis index = ctr*(2l+1) + m   (cint2e.c:794-870)
 *   int3c2e: out[i + ni*(j + nj*k)]                                          (cint3c2e.c:556)
 *   int2c2e: out[i + ni*k]                                                    (cint2c2e.c:238)
 * Return value: 1 if any primitive survived the exponent screening, else 0 (block zeroed).
 */
#ifndef CINTX_ORACLE_H
#define CINTX_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Rys roots t^2 (ascending) and weights for weight exp(-x t^2) on t in [0,1]
 * (the quantity libcint's CINTrys_roots, rys_roots.c:57, returns as u = t^2/(1-t^2)). */
int oracle_rys_t2(int nroots, double x, double *t2, double *w);
int oracle_rys_roots(int nroots, double x, double *u, double *w);
/* Boys function F_m(x), m = 0..mmax, in long double internally. */
void oracle_boys(int mmax, double x, double *f);

/* Real-solid-harmonic transform, row-major [2l+1][ncart(l)], libcint normalisation. */
void oracle_c2s_matrix(int l, double *mat);

int oracle_int2e(int sph, double *out, const int *shls, const int *atm, int natm,
                 const int *bas, int nbas, const double *env);
int oracle_int3c2e(int sph, double *out, const int *shls, const int *atm, int natm,
                   const int *bas, int nbas, const double *env);
int oracle_int2c2e(int sph, double *out, const int *shls, const int *atm, int natm,
                   const int *bas, int nbas, const double *env);

/* Batch helper for tests: quartets[q*4 .. q*4+3] shell indices; block q written at
 * out + offsets[q] in the dims==NULL layout.  nthreads <= 0 means all cores. */
void oracle_int2e_batch(int sph, double *out, const long long *offsets, const int *quartets,
                        long long nq, const int *atm, int natm, const int *bas, int nbas,
                        const double *env, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
