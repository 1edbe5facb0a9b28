/*
 * CPU baseline driver (TEST/BENCH INFRASTRUCTURE ONLY): times libcint 6.1.3's int2e_sph,
 * compiled from the reference sources (_ref/libcint.so), over a list of shell quartets with
 * OpenMP (dynamic schedule, one cache buffer per thread sized by the out == NULL query), the
 * way libcint callers parallelise over quartets.  A tuple (a, b, c, -1) runs int3c2e_sph on
 * (a, b, c) and (a, -1, c, -1) runs int2c2e_sph on (a, c), each with its own optimizer.
 *
 * usage: cint_cpu_bench INPUT NTHREADS
 * INPUT (little endian): int32 natm, nbas, nenv, nq; int32 atm[natm*6]; int32 bas[nbas*8];
 *                        double env[nenv]; int32 quartets[nq*4]
 * stdout: {"seconds": S, "nquartets": NQ, "nintegrals": NI, "threads": T, "checksum": C}
 */
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct CINTOpt CINTOpt;
int int2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas, double *env,
              CINTOpt *opt, double *cache);
void int2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);
int int3c2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas, double *env,
                CINTOpt *opt, double *cache);
void int3c2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);
int int2c2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas, double *env,
                CINTOpt *opt, double *cache);
void int2c2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);
void CINTdel_optimizer(CINTOpt **opt);

static int nsph(const int *bas, int s) { return (2 * bas[s * 8 + 1] + 1) * bas[s * 8 + 3]; }

int main(int argc, char **argv)
{
        if (argc < 3) {
                fprintf(stderr, "usage: %s INPUT NTHREADS\n", argv[0]);
                return 2;
        }
        FILE *fh = fopen(argv[1], "rb");
        if (!fh) {
                perror("open");
                return 2;
        }
        int hdr[4];
        if (fread(hdr, sizeof(int), 4, fh) != 4) return 2;
        int natm = hdr[0], nbas = hdr[1], nenv = hdr[2], nq = hdr[3];
        int *atm = malloc(sizeof(int) * natm * 6);
        int *bas = malloc(sizeof(int) * nbas * 8);
        double *env = malloc(sizeof(double) * nenv);
        int *q = malloc(sizeof(int) * (size_t)nq * 4);
        if (fread(atm, sizeof(int), natm * 6, fh) != (size_t)natm * 6 ||
            fread(bas, sizeof(int), nbas * 8, fh) != (size_t)nbas * 8 ||
            fread(env, sizeof(double), nenv, fh) != (size_t)nenv ||
            fread(q, sizeof(int), (size_t)nq * 4, fh) != (size_t)nq * 4) {
                fprintf(stderr, "short read\n");
                return 2;
        }
        fclose(fh);
        int nthreads = atoi(argv[2]);
        if (nthreads > 0) omp_set_num_threads(nthreads);
        CINTOpt *opt = NULL, *opt3 = NULL, *opt2 = NULL;
        int any4 = 0, any3 = 0, any2 = 0;
        for (int i = 0; i < nq; i++) {
                const int *s = q + (size_t)i * 4;
                if (s[3] >= 0) any4 = 1;
                else if (s[1] >= 0) any3 = 1;
                else any2 = 1;
        }
        if (any4) int2e_optimizer(&opt, atm, natm, bas, nbas, env);
        if (any3) int3c2e_optimizer(&opt3, atm, natm, bas, nbas, env);
        if (any2) int2c2e_optimizer(&opt2, atm, natm, bas, nbas, env);
        long long nint = 0;
        double checksum = 0;
        double t0 = omp_get_wtime();
        int used = 1;
#pragma omp parallel reduction(+ : nint, checksum)
        {
#pragma omp single
                used = omp_get_num_threads();
                int cache_n = 0, out_n = 0;
                double *cache = NULL, *out = NULL;
#pragma omp for schedule(dynamic, 8)
                for (int i = 0; i < nq; i++) {
                        int *s = q + (size_t)i * 4;
                        int kind = s[3] >= 0 ? 4 : (s[1] >= 0 ? 3 : 2);
                        int s2[2] = {s[0], s[2]};
                        int n = kind == 4 ? int2e_sph(NULL, NULL, s, atm, natm, bas, nbas, env, opt, NULL)
                              : kind == 3 ? int3c2e_sph(NULL, NULL, s, atm, natm, bas, nbas, env, opt3, NULL)
                                          : int2c2e_sph(NULL, NULL, s2, atm, natm, bas, nbas, env, opt2, NULL);
                        if (n > cache_n) {
                                free(cache);
                                cache_n = n;
                                cache = malloc(sizeof(double) * cache_n);
                        }
                        int blk = nsph(bas, s[0]) * nsph(bas, s[2]);
                        if (kind >= 3) blk *= nsph(bas, s[1]);
                        if (kind == 4) blk *= nsph(bas, s[3]);
                        if (blk > out_n) {
                                free(out);
                                out_n = blk;
                                out = malloc(sizeof(double) * out_n);
                        }
                        if (kind == 4) int2e_sph(out, NULL, s, atm, natm, bas, nbas, env, opt, cache);
                        else if (kind == 3) int3c2e_sph(out, NULL, s, atm, natm, bas, nbas, env, opt3, cache);
                        else int2c2e_sph(out, NULL, s2, atm, natm, bas, nbas, env, opt2, cache);
                        nint += blk;
                        checksum += out[0];
                }
                free(cache);
                free(out);
        }
        double t1 = omp_get_wtime();
        CINTdel_optimizer(&opt);
        CINTdel_optimizer(&opt3);
        CINTdel_optimizer(&opt2);
        printf("{\"seconds\": %.6f, \"nquartets\": %d, \"nintegrals\": %lld, \"threads\": %d, \"checksum\": %.17g}\n",
               t1 - t0, nq, nint, used, checksum);
        return 0;
}
