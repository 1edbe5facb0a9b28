/*
 * Batch evaluation through libcint (TEST/BENCH INFRASTRUCTURE ONLY): evaluates a list of shell
 * tuples with libcint 6.1.3 compiled from the reference sources (_ref/libcint.so) into caller
 * offsets, with one optimizer per call and OpenMP over the tuples (dynamic schedule, one cache
 * buffer per thread sized by libcint's out == NULL query, cint2e.c:801-818).  It is the checker
 * the GPU parity tests and bench.py's error record compare against; nothing in the product
 * loads it.
 *
 * family 4: int2e (4 ints per tuple), 3: int3c2e (3 ints), 2: int2c2e (2 ints), 41: int2e_ip1
 * (4 ints, 3 components), 31: int3c2e_ip1 (3 ints, 3 components); sph != 0 selects the *_sph
 * functions, else *_cart.  Block t is written at out + offs[t]; rets[t] (may be NULL) receives
 * libcint's return value.
 */
#include <omp.h>
#include <stdlib.h>

typedef struct CINTOpt CINTOpt;
typedef int (*intor_t)(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
typedef void (*optor_t)(CINTOpt **, int *, int, int *, int, double *);

int int2e_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int2e_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int3c2e_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int3c2e_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int2c2e_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int2c2e_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
void int2e_optimizer(CINTOpt **, int *, int, int *, int, double *);
void int3c2e_optimizer(CINTOpt **, int *, int, int *, int, double *);
void int2c2e_optimizer(CINTOpt **, int *, int, int *, int, double *);
int int2e_ip1_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int2e_ip1_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int3c2e_ip1_sph(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
int int3c2e_ip1_cart(double *, int *, int *, int *, int, int *, int, double *, CINTOpt *, double *);
void int2e_ip1_optimizer(CINTOpt **, int *, int, int *, int, double *);
void int3c2e_ip1_optimizer(CINTOpt **, int *, int, int *, int, double *);
void CINTdel_optimizer(CINTOpt **);

int ref_batch(int family, int sph, double *out, const long long *offs, const int *tuples, long long n,
              int *atm, int natm, int *bas, int nbas, double *env, int nthreads, int *rets)
{
        intor_t f;
        optor_t mk;
        if (family == 4) {
                f = sph ? int2e_sph : int2e_cart;
                mk = int2e_optimizer;
        } else if (family == 3) {
                f = sph ? int3c2e_sph : int3c2e_cart;
                mk = int3c2e_optimizer;
        } else if (family == 2) {
                f = sph ? int2c2e_sph : int2c2e_cart;
                mk = int2c2e_optimizer;
        } else if (family == 41) {
                f = sph ? int2e_ip1_sph : int2e_ip1_cart;
                mk = int2e_ip1_optimizer;
        } else if (family == 31) {
                f = sph ? int3c2e_ip1_sph : int3c2e_ip1_cart;
                mk = int3c2e_ip1_optimizer;
        } else {
                return 1;
        }
        CINTOpt *opt = NULL;
        mk(&opt, atm, natm, bas, nbas, env);
        if (nthreads > 0) omp_set_num_threads(nthreads);
        int fail = 0;
#pragma omp parallel reduction(| : fail)
        {
                int cap = 0;
                double *cache = NULL;
#pragma omp for schedule(dynamic, 4)
                for (long long t = 0; t < n; t++) {
                        int s[4];
                        const int nsh = family > 10 ? family / 10 : family;
                        for (int a = 0; a < nsh; a++) s[a] = tuples[t * nsh + a];
                        int need = f(NULL, NULL, s, atm, natm, bas, nbas, env, opt, NULL);
                        if (need > cap) {
                                free(cache);
                                cap = need;
                                cache = malloc(sizeof(double) * (size_t)cap);
                                if (!cache) {
                                        cap = 0;
                                        fail = 1;
                                        continue;
                                }
                        }
                        int r = f(out + offs[t], NULL, s, atm, natm, bas, nbas, env, opt, cache);
                        if (rets) rets[t] = r;
                }
                free(cache);
        }
        CINTdel_optimizer(&opt);
        return fail;
}
