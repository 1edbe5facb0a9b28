/*
 * CPU baseline driver (TEST/BENCH INFRASTRUCTURE ONLY): times libcint 6.1.3's int2e_sph,
 * compiled from the reference sources (_ref/libcint.so), over a list of shell quartets with
 * OpenMP (dynamic schedule, one cache buffer per thread sized by the out == NULL query), the
 * way libcint callers parallelise over quartets.
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
        CINTOpt *opt = NULL;
        int2e_optimizer(&opt, atm, natm, bas, nbas, env);
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
                        int n = int2e_sph(NULL, NULL, s, atm, natm, bas, nbas, env, opt, NULL);
                        if (n > cache_n) {
                                free(cache);
                                cache_n = n;
                                cache = malloc(sizeof(double) * cache_n);
                        }
                        int blk = nsph(bas, s[0]) * nsph(bas, s[1]) * nsph(bas, s[2]) * nsph(bas, s[3]);
                        if (blk > out_n) {
                                free(out);
                                out_n = blk;
                                out = malloc(sizeof(double) * out_n);
                        }
                        int2e_sph(out, NULL, s, atm, natm, bas, nbas, env, opt, cache);
                        nint += blk;
                        checksum += out[0];
                }
                free(cache);
                free(out);
        }
        double t1 = omp_get_wtime();
        CINTdel_optimizer(&opt);
        printf("{\"seconds\": %.6f, \"nquartets\": %d, \"nintegrals\": %lld, \"threads\": %d, \"checksum\": %.17g}\n",
               t1 - t0, nq, nint, used, checksum);
        return 0;
}
