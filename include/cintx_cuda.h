/*
 * cintx_cuda: B200 (sm_100a) two-electron Gaussian integrals behind libcint's C ABI.
 *
 * libcintx_cuda.so exports libcint 6.1.3's symbols for the Rys-quadrature Coulomb family so a
 * caller that binds libcint (PySCF-style ctypes drivers, the cintx-compat legacy path, the
 * cintx-oracle parity harness) can load this library instead.  Each libcint-signature entry
 * point keeps libcint's argument meaning, output layout and return value:
 *   - out == NULL  -> returns a cache size (in doubles) and computes nothing;
 *   - dims == NULL -> block written as out[i + ni*(j + nj*(k + nk*l))], each axis indexed
 *                     ctr*(2l+1)+m (sph) or ctr*ncart(l)+cart (cart), i.e. the layout of
 *                     c2s_sph_2e1 / c2s_cart_2e1 (cint2e.c:794-870, cart2sph.c:5324);
 *   - dims != NULL -> the same block placed in an array of extents dims[0..3];
 *   - return value -> 1 if any primitive survived libcint's exponent screening
 *                     (CINT2e_loop_nopt, cint2e.c:57), else 0 with the block zeroed.
 * `cache` is accepted and ignored (device memory is managed by the library).  `opt` must be
 * NULL or a handle made by this library's *_optimizer functions.
 * Differences from libcint: range-separated Coulomb (env[PTR_RANGE_OMEGA] != 0) and shells
 * with l > 4 are rejected (last error set, block zeroed, return 0) instead of computed, and
 * Rys-root failures never call exit().
 *
 * FINT is int and CACHE_SIZE_T is int, as in libcint built without I8 (cint.h.in:10-24).
 */
#ifndef CINTX_CUDA_H
#define CINTX_CUDA_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CINTX_API __attribute__((visibility("default")))
#else
#define CINTX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CINTOpt CINTOpt; /* opaque here; libcint's is cint.h.in:136 */

/* ---- libcint-signature entry points ---------------------------------------------------- */

/* Replaces libcint int2e_sph (libcint-master/src/cint2e.c:1186) and, in cintx, the
 * cintx-capi id-dispatch cintrs_eval(api=10) path (crates/cintx-capi/src/shim.rs:371). */
CINTX_API int int2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
              double *env, CINTOpt *opt, double *cache);
/* Replaces libcint int2e_cart (cint2e.c:1202); cintrs_eval api=9. */
CINTX_API int int2e_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
               double *env, CINTOpt *opt, double *cache);
/* Replaces libcint int2e_optimizer (cint2e.c:1195) and cintx-compat int2e_sph_optimizer
 * (crates/cintx-compat/src/optimizer.rs:99).  Builds the device-resident basis and all
 * screened primitive-pair tables once. */
CINTX_API void int2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);

/* Replaces libcint int2c2e_sph / int2c2e_cart / int2c2e_optimizer (cint2c2e.c:351-387);
 * cintrs_eval api=13 / 12. */
CINTX_API int int2c2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                double *env, CINTOpt *opt, double *cache);
CINTX_API int int2c2e_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                 double *env, CINTOpt *opt, double *cache);
CINTX_API void int2c2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);

/* Replaces libcint int3c2e_sph / int3c2e_cart / int3c2e_optimizer (cint3c2e.c:693-718). */
CINTX_API int int3c2e_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                double *env, CINTOpt *opt, double *cache);
CINTX_API int int3c2e_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                 double *env, CINTOpt *opt, double *cache);
CINTX_API void int3c2e_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);

/* First derivatives (nabla i j|k l) and (nabla i j|k), libcint int2e_ip1_sph / int2e_ip1_cart /
 * int2e_ip1_optimizer (autocode/grad2.c:69-88) and int3c2e_ip1_sph / int3c2e_ip1_cart /
 * int3c2e_ip1_optimizer (autocode/int3c2e.c:68-88); cintrs_eval api 36 / 35 and 19 / 18.  The
 * derivative acts on the electron coordinate of the first shell; three components x, y, z, each a
 * block in the plain layout, one after the other: out[c*blk + i + ni*(j + nj*(k + nk*l))] (with
 * dims: out[c*dims[0]*dims[1]*... + ...]).  Return value, out == NULL and screening as int2e_sph.
 * Compiled for l <= 3 on (i, j) and (k, l), and l <= 4 on the 3-centre auxiliary shell k; other
 * shells set CINTX_STATUS_UNSUPPORTED_API.  Primitive screening follows libcint's driver for the
 * call: without an optimizer only the differentiated pair's estimate takes l + 1 (CINT2e_loop_nopt);
 * with one (its tables are not needed) every pair's does (CINTOpt_setij, optimizer.c:344). */
CINTX_API int int2e_ip1_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                            double *env, CINTOpt *opt, double *cache);
CINTX_API int int2e_ip1_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                             double *env, CINTOpt *opt, double *cache);
CINTX_API void int2e_ip1_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);
CINTX_API int int3c2e_ip1_sph(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                              double *env, CINTOpt *opt, double *cache);
CINTX_API int int3c2e_ip1_cart(double *out, int *dims, int *shls, int *atm, int natm, int *bas, int nbas,
                               double *env, CINTOpt *opt, double *cache);
CINTX_API void int3c2e_ip1_optimizer(CINTOpt **opt, int *atm, int natm, int *bas, int nbas, double *env);

/* Replaces libcint CINTdel_optimizer (optimizer.c:69). Sets *opt to NULL. */
CINTX_API void CINTdel_optimizer(CINTOpt **opt);

/* Replaces libcint CINTrys_roots (rys_roots.c:57): u[r] = t_r^2/(1-t_r^2) and w[r] for
 * order nroots (1..9), evaluated by the device root evaluator.  Returns 0 on success. */
CINTX_API int CINTrys_roots(int nroots, double x, double *u, double *w);

/* Basis bookkeeping, as libcint's cint_bas.c (the AO offsets a caller lays AO-indexed tensors out
 * with; cintx-compat helpers.rs:150-200 restates them):
 *   CINTcgto_cart / CINTcgto_spheric (cint_bas.c:36, :49): functions of shell bas_id,
 *     ncart(l) * nctr or (2l+1) * nctr;
 *   CINTtot_cgto_spheric / CINTtot_cgto_cart (cint_bas.c:108, :124): functions of all nbas shells;
 *   CINTshells_spheric_offset / CINTshells_cart_offset (cint_bas.c:149, :141): ao_loc[i] = first
 *     function of shell i, for i < nbas (ao_loc[nbas] is not written, as in libcint). */
CINTX_API int CINTcgto_cart(const int bas_id, const int *bas);
CINTX_API int CINTcgto_spheric(const int bas_id, const int *bas);
CINTX_API int CINTtot_cgto_spheric(const int *bas, const int nbas);
CINTX_API int CINTtot_cgto_cart(const int *bas, const int nbas);
CINTX_API void CINTshells_spheric_offset(int ao_loc[], const int *bas, const int nbas);
CINTX_API void CINTshells_cart_offset(int ao_loc[], const int *bas, const int nbas);

/* Device root evaluator over many points (no libcint counterpart; used to verify the root
 * table): t2w[i*2n + r] = t_r^2 and t2w[i*2n + n + r] = w_r at x[i].  Host arrays. */
CINTX_API int cintx_rys_t2_batch(int nroots, const double *x, int64_t nx, double *t2w);

/* ---- status and last error (cintx-capi errors.rs:9-21, 98-139) ------------------------- */

enum {
  CINTX_STATUS_SUCCESS = 0,
  CINTX_STATUS_INVALID_INPUT = 1,
  CINTX_STATUS_UNSUPPORTED_API = 2,
  CINTX_STATUS_UNSUPPORTED_REPRESENTATION = 3,
  CINTX_STATUS_BUFFER_TOO_SMALL = 4,
  CINTX_STATUS_MEMORY_LIMIT_EXCEEDED = 5,
  CINTX_STATUS_ALLOCATION_FAILED = 6,
  CINTX_STATUS_EXECUTION_FAILED = 7,
  CINTX_STATUS_NULL_POINTER = 8,
  CINTX_STATUS_PANIC = 9,
  CINTX_STATUS_BACKEND_NOT_COMPILED = 10
};

/* Status of the calling thread's most recent failed call (0 if none); cleared by
 * cintx_cuda_clear_last_error.  Mirrors cintrs_last_error_code (cintx-capi errors.rs). */
CINTX_API int cintx_cuda_last_error_code(void);
/* Copies the thread's last error message (NUL-terminated, truncated to cap). Returns the
 * full message length.  Mirrors cintrs_copy_last_error_message. */
CINTX_API size_t cintx_cuda_last_error_message(char *buf, size_t cap);
CINTX_API void cintx_cuda_clear_last_error(void);

/* ---- batched device API (no libcint counterpart; the path the B200 engine is built for) - */

typedef struct CintxPlan CintxPlan;

/* Integral family of a plan. */
enum { CINTX_INT2E = 0, CINTX_INT3C2E = 1, CINTX_INT2C2E = 2 };

/* Plan an explicit list of shell tuples (4 ints per int2e entry, 3 per int3c2e, 2 per
 * int2c2e, host memory).  Output blocks are laid out back to back in list order, each in
 * libcint's dims==NULL layout; offsets_out (host, n entries, may be NULL) receives each
 * block's offset in doubles.  `opt` must come from the matching *_optimizer.  Returns a
 * status code. */
CINTX_API int cintx_plan_shells(CintxPlan **plan, CINTOpt *opt, int family, const int *shls, int64_t n,
                      int sph, int64_t *offsets_out);

/* Plan every 8-fold-unique int2e quartet (i>=j, k>=l, ij>=kl over pairs oriented and ordered
 * by angular momentum) whose Schwarz bound sqrt(max|(ij|ij)| max|(kl|kl)|) reaches cutoff.
 * The work is split into chunks whose outputs fit in max_chunk_doubles; chunk outputs are
 * libcint-layout blocks back to back.  Returns a status code. */
CINTX_API int cintx_plan_int2e_screened(CintxPlan **plan, CINTOpt *opt, double cutoff, int sph,
                              int64_t max_chunk_doubles);

/* ---- cintx-capi id dispatch (crates/cintx-capi/src/shim.rs:312-453) --------------------- */

/* Workspace and result descriptors of cintx-capi (shim.rs:52-68), field for field. */
typedef struct {
  size_t bytes;           /* caller cache bytes needed (0: the library holds its device memory) */
  size_t alignment;
  size_t required_bytes;  /* bytes of the output block */
  size_t chunk_count;
  size_t work_units;
} CintxWorkspaceQuery;
typedef struct {
  int not0;               /* libcint's return value: 1 if any primitive survived screening */
  size_t bytes_written;
  size_t workspace_bytes;
} CintxEvalSummary;

/* cintrs_eval / cintrs_query_workspace for the api ids 9 int2e_cart, 10 int2e_sph, 12 int2c2e_cart,
 * 13 int2c2e_sph, 18 int3c2e_ip1_cart, 19 int3c2e_ip1_sph, 35 int2e_ip1_cart, 36 int2e_ip1_sph
 * (CintxRawApi, shim.rs:8-50; other ids return CINTX_STATUS_UNSUPPORTED_API).
 * natm = atm_len / 6 and nbas = bas_len / 8; every env slot the basis references must lie below
 * env_len; dims, when given, must equal the block's natural extents (cintx-compat layout.rs);
 * out == NULL (out_len 0) is a workspace-only call; out and cache must not alias; opt is NULL or
 * an optimizer of this library.  Statuses and the thread-local last error follow cintx-capi's
 * errors.rs:9-21. */
CINTX_API int cintrs_query_workspace(int api, const int *dims, size_t dims_len, const int *shls, size_t shls_len,
                                     const int *atm, size_t atm_len, const int *bas, size_t bas_len,
                                     const double *env, size_t env_len, const CINTOpt *opt,
                                     CintxWorkspaceQuery *query_out);
CINTX_API int cintrs_eval(int api, double *out, size_t out_len, const int *dims, size_t dims_len, const int *shls,
                          size_t shls_len, const int *atm, size_t atm_len, const int *bas, size_t bas_len,
                          const double *env, size_t env_len, const CINTOpt *opt, double *cache, size_t cache_len,
                          CintxEvalSummary *summary_out);

/* Device bytes held by an optimizer handle (pair and primitive-pair tables). */
CINTX_API int64_t cintx_opt_device_bytes(CINTOpt *opt);

/* The tuned sweep: the same quartet set as cintx_plan_int2e_screened, with two error-budgeted
 * shortcuts built on primitive Schwarz factors q_ab = |c_a c_b| sqrt(max|(ab|ab)|) (computed on
 * the device once per optimizer):
 *   - primitive screening: a primitive quartet with q_ab q_cd below a per-class threshold is
 *     skipped, the threshold chosen so the skipped terms of one block sum to <= prim_budget;
 *   - mixed precision (spherical output only; classes with la+lb+lc+ld >= 4): a quartet runs
 *     its recurrences and cartesian products in FP32 when its estimated FP32 error
 *     64 * 2^-24 * (Qp amp)_ab (Qp amp)_cd * (c2s amplification) is below fp32_budget, where
 *     Qp_ab = sum_ab q_ab and amp_ab = max over primitive pairs of (1 + |P - C| sqrt(2 a_ab))^(la+lb)
 *     bounds the cancellation of the recurrences; roots, prefactors and the sum over primitives
 *     stay FP64.
 * Both are absolute error budgets per integral; fp32_budget <= 0 and prim_budget <= 0 give the
 * FP64 plan. */
CINTX_API int cintx_plan_int2e_screened_mixed(CintxPlan **plan, CINTOpt *opt, double cutoff, int sph,
                                              int64_t max_chunk_doubles, double fp32_budget,
                                              double prim_budget);

/* Optimizer for density-fitting sweeps over a basis whose first npair_shells shells are the
 * orbital shells and the rest auxiliary shells: shell pairs are built only among the orbital
 * shells (the (ij| side of int3c2e), unit pairs for every shell (the |k) side and int2c2e).  The
 * handle works with every entry point; tuples needing a pair it does not hold are rejected.  No
 * counterpart in libcint (CINTall_3c2e_optimizer, optimizer.c:193, builds every pair).  Returns a
 * status code; *opt is NULL on failure. */
CINTX_API int cintx_optimizer_pair_shells(CINTOpt **opt, const int *atm, int natm, const int *bas, int nbas,
                                          const double *env, int npair_shells);

/* Density-fitting 3-centre sweep: every (ab|k) with a >= b orbital shells in [0, norb) and k an
 * auxiliary shell in [norb, nbas) whose Schwarz bound sqrt(max|(ab|ab)|) sqrt(max|(k|k)|) reaches
 * cutoff, as int3c2e_sph/int3c2e_cart blocks (libcint cint3c2e.c:693) out[i + ni*(j + nj*k)] for
 * the tuple (a, b, k) with a the shell of higher l (equal l: higher index), chunked like
 * cintx_plan_int2e_screened; cintx_plan_chunk_quartets reports tuples (a, b, k, -1). */
CINTX_API int cintx_plan_int3c2e_screened(CintxPlan **plan, CINTOpt *opt, double cutoff, int sph,
                                          int64_t max_chunk_doubles, int norb);

/* Coulomb and exchange matrices of a unique-quartet int2e sweep (cintx_plan_int2e_screened or
 * cintx_plan_int2e_screened_mixed) for a symmetric density dm (device, row-major nao x nao in this
 * plan's representation, AOs ordered by shell): vj[p,q] = sum_rs (pq|rs) dm[r,s] and
 * vk[p,r] = sum_qs (pq|rs) dm[q,s] (device, nao x nao; either may be NULL), without writing the
 * integrals anywhere but a device chunk ring.  Each chunk's blocks are contracted right after its
 * kernels with the 8-fold permutational symmetry.  Asynchronous on stream; the plan's device
 * buffers are reused, so calls on one plan must not overlap.  No counterpart in libcint (the
 * direct-SCF consumer of int2e_sph, e.g. PySCF's vhf). */
CINTX_API int cintx_plan_jk(CintxPlan *plan, const double *dm, int nao, double *vj, double *vk, void *stream);
/* The whole sweep as the 8-fold packed AO tensor (PySCF ao2mo's "s8" layout): eri[pq*(pq+1)/2 + rs]
 * with pq = p*(p+1)/2 + q (p >= q, AOs ordered by shell in this plan's representation) and
 * pq >= rs; len >= npair*(npair+1)/2 doubles of device memory, npair = nao*(nao+1)/2.  Quartets
 * below the plan's cutoff are 0.  Asynchronous on stream. */
CINTX_API int cintx_plan_execute_s8(CintxPlan *plan, double *eri, int64_t len, void *stream);

/* The whole sweep as an AO-indexed tensor in one of PySCF ao2mo's layouts (AOs ordered by shell in
 * this plan's representation, offsets as CINTshells_*_offset), quartets below the plan's cutoff 0:
 *   aosym 1 ("s1"): eri[((p*nao + q)*nao + r)*nao + s], nao^4 doubles;
 *   aosym 4 ("s4"): eri[pq*npair + rs], pq = p*(p+1)/2 + q (p >= q), rs likewise, npair^2 doubles;
 *   aosym 8 ("s8"): as cintx_plan_execute_s8.
 * len (doubles of device memory at eri) must hold the layout.  Asynchronous on stream. */
CINTX_API int cintx_plan_execute_ao(CintxPlan *plan, int aosym, double *eri, int64_t len, void *stream);

/* Plan statistics. */
typedef struct {
  int64_t nquartets;        /* shell tuples in the plan */
  int64_t nintegrals;       /* output doubles over all chunks */
  int64_t nchunks;
  int64_t max_chunk_doubles;/* largest chunk output */
  int64_t nprim_quartets;   /* primitive tuples surviving the pair screening */
  int64_t device_bytes;     /* device memory held by the plan (records, tile tables) */
  int64_t nquartets_fp32;   /* quartets evaluated with FP32 recurrences (mixed plans) */
  double flops;             /* FP64 flops of the Rys path: per primitive quartet VRR 15*nroots*
                               (li+lj+1)(lk+ll+1), HRR 6*nroots per transfer step, products
                               3*nroots per cartesian element; per quartet the c2s stages */
} CintxPlanStats;
CINTX_API int cintx_plan_stats(const CintxPlan *plan, CintxPlanStats *stats);
/* Output size (doubles) and tuple list of one chunk; quartets may be NULL. */
CINTX_API int64_t cintx_plan_chunk_size(const CintxPlan *plan, int64_t chunk);
CINTX_API int64_t cintx_plan_chunk_nquartets(const CintxPlan *plan, int64_t chunk);
CINTX_API int cintx_plan_chunk_quartets(const CintxPlan *plan, int64_t chunk, int *quartets, int64_t cap);

/* Segments of a chunk: each is one kernel class over a contiguous run of quartets.  For
 * segment s: cls[4s..4s+3] = (li, lj, lk, ll) of the kernel, nq[s] quartets, flops[s] the
 * algorithmic FP64 flops (model of cintx_plan_stats).  Returns the segment count (or -1). */
CINTX_API int cintx_plan_chunk_segments(const CintxPlan *plan, int64_t chunk, int *cls, int64_t *nq,
                                        double *flops, int cap);
/* Runs one segment of a chunk into out_dev (chunk-relative offsets, as cintx_plan_execute). */
CINTX_API int cintx_plan_execute_segment(CintxPlan *plan, int64_t chunk, int seg, double *out_dev,
                                         void *stream);
/* n shell quartets drawn uniformly (with replacement, seeded) from the whole plan. */
CINTX_API int cintx_plan_sample_quartets(const CintxPlan *plan, uint64_t seed, int64_t n, int *quartets);

/* Run one chunk (or all chunks when chunk < 0, each overwriting out_dev) on `stream`
 * (a cudaStream_t, used as given: NULL is the legacy default stream).  out_dev is device memory of
 * at least the chunk size (all-chunk runs: max_chunk_doubles).  Asynchronous. */
CINTX_API int cintx_plan_execute(CintxPlan *plan, int64_t chunk, double *out_dev, void *stream);
/* Captures the execution of a chunk list (chunks == NULL: every chunk) into one CUDA graph
 * writing to out_dev: within a chunk the kernel classes run on up to nbranch parallel graph
 * branches; chunks run in order.  Replaces any previous capture of this plan. */
CINTX_API int cintx_plan_graph_build(CintxPlan *plan, const int64_t *chunks, int64_t n, double *out_dev,
                                     int nbranch);
/* Launches the captured graph on `stream` (asynchronous). */
CINTX_API int cintx_plan_graph_launch(CintxPlan *plan, void *stream);
/* Autotuner: times every kernel class of chunk `chunk` (chunk < 0: every class of the plan, each
 * on the chunk where it has the most quartets; reps runs after one warm-up, CUDA events on
 * `stream`, output into out_dev of max_chunk_doubles) in each launch shape (lanes per quartet,
 * hence quartets per block) that gives a distinct shape, and keeps the fastest per class for
 * every chunk of the plan.  Synchronous.  A graph captured earlier is released: capture again
 * after tuning. */
CINTX_API int cintx_plan_autotune(CintxPlan *plan, int64_t chunk, double *out_dev, void *stream, int reps);
/* Applies the launch shapes the autotuner chose earlier in this process on the current device
 * (any plan) to this plan's matching classes; returns the number of segments changed (or -1).
 * A graph captured earlier is released when anything changed. */
CINTX_API int cintx_plan_use_tuned_shapes(CintxPlan *plan);
/* The launch shapes the autotuner chose in this process on the current device, as records of six
 * ints (li, lj, lk, ll, fp32, variant): cintx_tuned_shapes_export writes up to cap records and
 * returns how many there are; cintx_tuned_shapes_import adds n records (e.g. saved by an earlier
 * process on the same kind of GPU) to the current device's choices, for cintx_plan_use_tuned_shapes
 * to apply without tuning again.  Import returns a status code. */
CINTX_API int cintx_tuned_shapes_export(int *records, int cap);
CINTX_API int cintx_tuned_shapes_import(const int *records, int n);
/* Sets the launch-shape variant (0..11) of every segment, for tests and tuning scripts; a class
 * that the variant does not apply to runs its default shape.  Returns the number of segments
 * changed (or -1).  A graph captured earlier is released when anything changed. */
CINTX_API int cintx_plan_set_shape(CintxPlan *plan, int variant);
/* Lanes per quartet of each segment of a chunk (as chosen by the autotuner, or the default
 * shape).  Returns the segment count (or -1). */
CINTX_API int cintx_plan_segment_lanes(const CintxPlan *plan, int64_t chunk, int *lanes, int cap);
/* End to end: evaluates one chunk (chunk >= 0) or every chunk (chunk < 0) into device staging
 * buffers and copies the output to host memory out_host, chunks back to back (out_host holds the
 * chunk's size, or the plan's nintegrals for chunk < 0).  With several chunks the copy of chunk c
 * runs on a second stream while chunk c+1 is evaluated (two staging buffers); page-locked
 * out_host lets the copies overlap.  Synchronous. */
CINTX_API int cintx_plan_execute_host(CintxPlan *plan, int64_t chunk, double *out_host);
/* End to end for sweeps larger than host memory: every chunk is evaluated and copied into one of
 * two slots of the host ring (ring_doubles >= 2 x the largest chunk; page-locked memory lets the
 * copies overlap the next chunk's kernels), and on_chunk(user, chunk, data, n) (may be NULL) is
 * called for each chunk in order, on the calling thread, before its slot is reused.
 * Synchronous. */
CINTX_API int cintx_plan_execute_host_ring(CintxPlan *plan, double *ring, int64_t ring_doubles,
                                           void (*on_chunk)(void *user, int64_t chunk, const double *data,
                                                            int64_t n),
                                           void *user);
CINTX_API void cintx_plan_destroy(CintxPlan *plan);

/* Batched first derivatives (no libcint counterpart; the batched form of int2e_ip1 / int3c2e_ip1):
 * family CINTX_INT2E (4 ints per tuple) or CINTX_INT3C2E (3 ints), n tuples (host), blocks back to
 * back in list order, each 3 components of the plain block (layout of int2e_ip1_sph) into out_dev
 * (device memory the caller sized from offsets: offsets_out, host, n entries, may be NULL).
 * Screened as libcint with an optimizer.  Synchronous; blocks of fully screened tuples are zero. */
CINTX_API int cintx_ip1_eval(int family, double *out_dev, const int *shls, int64_t n, int sph, const int *atm,
                             int natm, const int *bas, int nbas, const double *env, int64_t *offsets_out);

/* ---- evaluation without device allocation ------------------------------------------------ */

/* Size of the fixed device scratch array behind cintx_int2e_noalloc (32 MiB per GPU). */
#define CINTX_NOALLOC_SCRATCH_BYTES (32u << 20)

/* Has no counterpart in the reference; it exists for callers that cannot call cudaMalloc while
 * they use this library: code running inside a host framework's memory pool or arena, code that
 * has already claimed almost all HBM, and code that must avoid the device-wide synchronisation an
 * allocation or free may cause.  Evaluates int2e (sph != 0: spherical, else cartesian) for n
 * shell quartets (shls: 4 ints each, host) of the basis (atm, bas, env: host arrays as for
 * int2e_sph) into out_dev, device memory the caller owns, with the blocks back to back in list
 * order in libcint's dims == NULL layout (the offsets cintx_plan_shells reports).  It calls no
 * cudaMalloc/cudaFree: its device working memory is a static array of
 * CINTX_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until the process exits,
 * plus a static copy of the root table.  The first call on each device does a one-time set-up
 * (looks up the arrays' device addresses and copies the root table, synchronously); make that
 * first call before any stream capture.  A call whose screened pairs and quartet records exceed
 * the array returns CINTX_STATUS_MEMORY_LIMIT_EXCEEDED (split the list); classes with two or
 * more g shells return CINTX_STATUS_UNSUPPORTED_API.  Each call builds its tables in host
 * memory that lives only for the call: it waits for earlier work on `stream` (used as given),
 * copies the tables into the array and waits for that copy, then queues its kernels on `stream`
 * and returns without waiting for them.  Every call reuses the same array and rewrites all of it
 * that it reads, so nothing needs clearing between calls, but calls whose work overlaps on the
 * GPU (other streams, other host threads) race on it: serialise them. */
CINTX_API int cintx_int2e_noalloc(double *out_dev, const int *shls, int64_t n, int sph, const int *atm,
                                  int natm, const int *bas, int nbas, const double *env, void *stream);

/* ---- learned Rys-root initializer (RysNet) ------------------------------------------------ */

/* The plain path these replace for a caller that opts in is CINTrys_roots
 * (libcint-master/src/rys_roots.c:57; cintx-cubecl math/rys.rs).  RysNet is an MLP in FP32
 * (inputs: nroots and log x; two hidden layers of 64 SiLU units; 18 outputs read as logit(t_i^2)
 * for outputs 0..8 and log(w_i) for 9..17) whose CINTX_RYSNET_NPARAM parameters are, in order:
 * W1[64][2], b1[64], W2[64][64] (row = output), b2[64], W3[18][64], b3[18]. */
#define CINTX_RYSNET_NPARAM 5522

/* count training samples drawn on the device (seeded): nroots uniform in [n_lo, n_hi], x
 * log-uniform in [1e-7, 50] with probability 0.7 else uniform in [50, 3000], redrawn
 * log-uniformly below the table range where it is reached.  feat[2*count] network inputs,
 * tgt[18*count] targets from the table path (unused outputs 0), nroots[count], x[count] (x may be
 * NULL).  Host arrays; synchronous. */
CINTX_API int cintx_rysnet_samples(int64_t count, int n_lo, int n_hi, uint64_t seed, float *feat, float *tgt,
                                   int *nroots, double *x);
/* One forward and backward pass of the device training kernel over count samples (host arrays
 * as produced by cintx_rysnet_samples): loss = mean over samples of the squared error of the
 * sample's 2*nroots used outputs divided by 2*nroots, and its gradient grad[CINTX_RYSNET_NPARAM]
 * with respect to params.  Synchronous. */
CINTX_API int cintx_rysnet_loss_grad(const float *params, const float *feat, const float *tgt, const int *nroots,
                                     int64_t count, float *grad, double *loss);
/* Trains params (in: initial values, out: trained) on the device: nsamples samples as above,
 * epochs passes of Adam (beta 0.9/0.999, cosine decay of lr to 1%) over minibatches of `batch`
 * (a multiple of 128); loss_per_epoch[epochs] (may be NULL) receives each epoch's mean loss.
 * Synchronous. */
CINTX_API int cintx_rysnet_train(float *params, int64_t nsamples, int n_lo, int n_hi, int epochs, int batch,
                                 float lr, uint64_t seed, double *loss_per_epoch);
/* Rys roots t^2 and weights of order nroots (1..9) at count points x, in cintx_rys_t2_batch's
 * layout t2w[p*2*nroots + f] (roots first), from the network's guess (mode 0; params on the
 * host) or from the x = 0 roots (mode 1: the same refinement without the network), refined in
 * FP64 (Stieltjes recurrence of the measure's 64-node discretisation, at most 8 Newton steps
 * with the Aberth correction on the orthogonal polynomial, roots sorted and checked distinct
 * and inside (0, 1), Christoffel weights); mode 2 returns the network's guess unrefined
 * (status 3), for judging it against the table path.  status[p]: 0 refined, 1 the refinement
 * failed its checks and the table path supplied the values (fallback), 2 x beyond the table range
 * (closed form).  iters[p]: Newton steps of the slowest root.  Synchronous. */
CINTX_API int cintx_rys_learned_batch(const float *params, int nroots, const double *x, int64_t count, int mode,
                                      double *t2w, int *status, int *iters);
/* Makes an explicit plan (cintx_plan_shells) take its Rys roots from RysNet (params on the host)
 * instead of the table: the x of every primitive quartet is enumerated on the device, its roots
 * are computed by the refinement of cintx_rys_learned_batch (mode 0, table fallback per point)
 * into a device buffer the ERI kernels read.  *nfallback / *npoints (may be NULL) receive the
 * fallback count and the number of primitive quartets.  params == NULL restores table roots.
 * Synchronous; a graph captured earlier is released. */
CINTX_API int cintx_plan_use_learned_roots(CintxPlan *plan, const float *params, int64_t *nfallback,
                                           int64_t *npoints);

/* FP64 FMA throughput probe (measurement only): blocks x threads threads each run
 * iters*16*8 FMAs and write one double to out_dev[blocks*threads].  Asynchronous on stream. */
CINTX_API int cintx_fp64_fma_probe(int blocks, int threads, int iters, double *out_dev, void *stream);

/* Kernel launches issued by the calling thread's plan executions so far (for accounting). */
CINTX_API int64_t cintx_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* CINTX_CUDA_H */
