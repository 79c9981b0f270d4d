/*
 * zolo_b200.h -- C-ABI of the B200 (sm_100a) polar-decomposition / SVD path.
 *
 * Drop-in boundary for the reference's Fortran entry points on a 1x1 process
 * grid.  Each reference-named function keeps the reference's argument list
 * and meaning; its comment cites the reference interface it replaces
 * (file:line in shengguolsg/Zolo-SVD).  All matrices are column-major FP64
 * (DOUBLE PRECISION), integers are 32-bit (MKL LP64 INTEGER), CHARACTER
 * arguments are passed as `char` in the C names and as `const char*` plus a
 * trailing hidden `size_t` length in the gfortran-mangled names.
 *
 * Descriptors (DESC(9) = DTYPE_, CTXT_, M_, N_, MB_, NB_, RSRC_, CSRC_, LLD_)
 * must describe a 1x1 grid: DTYPE_ = 1, RSRC_ = CSRC_ = 0, LLD_ >= max(1,M_);
 * CTXT_ is ignored and IA = JA = IQ = JQ = 1.
 *
 * INFO conventions follow the reference: 0 success, -i for a bad scalar
 * argument i, -(i*100+j) for entry j of array argument i, -12 / -16 for a
 * too-small LWORK / LWORK2 (pqdwhfacs.f90:286-294), > 0 from a factorisation.
 * GPU failures are reported as INFO = -1000 - cudaError_t.  Nothing aborts.
 *
 * Threading: every handle owns one CUDA stream; calls on one handle are
 * serialised by a mutex.  The handle's own stream is a blocking stream, so a
 * call is ordered after work already queued on the legacy default stream; with
 * zolo_set_stream the caller's stream is used instead and the caller orders the
 * inputs on it.  The device-pointer solvers return after their results are
 * complete.  The reference-named host-array entry points use a
 * process-wide default handle on device 0 (or ZOLO_DEVICE).
 */
#ifndef ZOLO_B200_H
#define ZOLO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct zolo_handle_s* zolo_handle_t;

typedef struct {
  int iterations;      /* polar iterations executed                       */
  int qr_iterations;   /* of which used the QR form                       */
  int chol_iterations; /* of which used the Cholesky form                 */
  int info;            /* first factorisation INFO seen (0 = none)        */
  double alpha;        /* upper bound used (||A - sigma I||_F)            */
  double beta;         /* lower bound used                                */
  double last_err;     /* last ||X_{k+1} - X_k||_F                        */
  double ms_total;     /* device time of the whole call (CUDA events)     */
  double ms_bounds;
  double ms_iter;
  double ms_h;         /* H (and, for zolo_polar_dev, Q = Q_x Y from the
                          factored iterate) */
  double flops;        /* canonical FP64 flops of the executed steps      */
  int64_t launches;    /* kernels launched                                */
  double con[16];      /* per iteration: CON (Zolo) or c_k (QDWH)         */
  double err[16];      /* per iteration: ||X_{k+1} - X_k||_F              */
  int branch[16];      /* per iteration: 1 = QR form, 2 = Cholesky form,
                          3 = Newton-Schulz step (ZOLO_OPT_NS_FINISH)      */
  double flops_executed; /* FP64 flops actually executed (the shared-QR form
                            does fewer than the canonical count)           */
  int ns_steps;        /* Newton-Schulz steps that ended the iteration     */
  int ns_finish;       /* 1 if Newton-Schulz steps ended the iteration     */
  double ms_step[16];  /* per Zolo-PD / QDWH iteration: device milliseconds */
  double ms_finish;    /* ZOLO_OPT_NS_FINISH: device ms from the check that
                          entered the finish to its end (0 if not entered)   */
  int terms[16];       /* per Zolo-PD iteration: Zolotarev terms used (rk,
                          or the planned count, see ZOLO_OPT_TERM_PLAN)      */
} zolo_stats_t;

/* ---- handles (no reference counterpart: the reference is one MPI job) ---- */
int zolo_create(int device, zolo_handle_t* handle);
int zolo_destroy(zolo_handle_t handle);
int zolo_set_stream(zolo_handle_t handle, void* cuda_stream);
int zolo_get_stats(zolo_handle_t handle, zolo_stats_t* out);
int zolo_default_handle(zolo_handle_t* handle);
int zolo_release_workspace(zolo_handle_t handle);
const char* zolo_version(void);
/* Per-kernel-class device timing with CUDA events on the launching streams
 * (0 = DMMA GEMM general shapes, 1 = Householder panel, 2 = Cholesky leaf,
 * 3 = GEMM M <= 32, 4 = GEMM N <= 64, 5 = GEMM rank-k K <= 64, 6 = GEMM lower
 * triangle, 7 = FP64 product emulated on the INT8 tensor cores (its INT8 kernel), 8 = GEMM
 * with 64 < K <= 256, class 0 then being K > 256, 9 = the emulated products' splitting
 * into digit planes).  While enabled, zolo_profile_read fills out[3*cls + 0..2] =
 * {launches, milliseconds, algorithmic flops} accumulated since the last reset (out holds
 * 30 doubles).  on = 2 times every launch alone (the device is
 * synchronized around it), as a profiler's serialized launch list does; on = 1 leaves the
 * streams overlapping, so a launch's time includes work running beside it. */
int zolo_profile_enable(zolo_handle_t handle, int on);
/* Thread-block-cluster size the Householder panel kernel uses for an m x w panel on the
 * current device (negative when the rows do not fit in shared memory). */
int zolo_panel_cluster_size(int m, int w);
int zolo_profile_read(zolo_handle_t handle, double* out, int reset);
/* Algorithm options of a handle (no reference counterpart).
 * ZOLO_OPT_SHARED_QR: 1 (default) = Zolo-PD QR iterations factor X = Q_x R_x once and
 * run the r structured QRs on the 2n x n stacks [R_x; sqrt(c_j) I]; 0 = one QR of the
 * (m+n) x n stack [X; sqrt(c_j) I] per term, as the reference does (pzolopd1.f90:412,
 * zoloqr.f90:99-111).
 * Both give the same iterate up to rounding.  Returns -1 for an unknown option. */
#define ZOLO_OPT_SHARED_QR 1
/* ZOLO_OPT_NS_FINISH: 0 (default) = the reference's stopping rule
 * (pzolopd1.f90:381-397: iterate until ||X_{k+1} - X_k||_F <= (5 eps)^(1/(2r+1))).
 * 1 = before each Cholesky-form Zolo-PD iteration, measure e = ||X^T X - I||_F/sqrt(n)
 * from the Gram matrix that iteration forms anyway; once e <= 0.1, finish with
 * FP64 Newton-Schulz steps X <- X (3I - X^T X)/2 instead of further Zolo
 * iterations, re-measuring e before each step and stopping at rounding level
 * (max(1e-14, eps sqrt(m)/2), or when a step no longer halves e; at most 12 steps,
 * none when e is already there; the Gram after a step is not formed when the step's bound on
 * the next e, 3/4 e^2 sqrt(n) (1 + e sqrt(n)/3), is below a tenth of that level).  The polar
 * factor of X is that of A, so the result
 * agrees with the reference rule's to rounding.  With this option the loop ends at that
 * measured check rather than on ||X_{k+1} - X_k||.  No reference counterpart. */
#define ZOLO_OPT_NS_FINISH 2
/* ZOLO_OPT_CHOL_INVERSE: 0 (default) = each Cholesky-form term solves
 * X (X^T X + c_j I)^{-1} with two triangular solves (zolochol.f90:87-113); 1 = the
 * terms' inverses L_j^{-T} L_j^{-1} (triangular inverse + one lower-triangle product,
 * 4n^3/3 per term) are summed into S = sum_j w_j (X^T X + c_j I)^{-1} and the iteration
 * takes one Z = X S, about 6n^3 fewer flops per iteration for r = 8.  These matrices
 * are well conditioned in the Cholesky iterations (condition <= CON^2, CON <= 1e3), so
 * both forms agree to rounding.  SYM = 'S' keeps the solves.  No reference counterpart. */
#define ZOLO_OPT_CHOL_INVERSE 3
/* ZOLO_OPT_BETA_FROB: 0 (default) = zolo_polar_dev takes beta = 1/(sqrt(n) ||R^{-1}||_1)
 * (zolo_bounds_dev mode 1, the reference driver's estimate); 1 = beta = 1/||R^{-1}||_F (mode 2),
 * also a lower bound on sigma_min but up to sqrt(n) times tighter.  The Zolotarev
 * coefficients (Auxil_Zolo.f90:165-200, alpha = acos(1/CON)) lose their accuracy once
 * CON = 1/beta passes about 1e15, after which the second iteration no longer converges and
 * one more is needed; the tighter beta keeps CON below that for condition numbers up to
 * about 1e13.  No reference counterpart. */
#define ZOLO_OPT_BETA_FROB 4
/* ZOLO_OPT_TERM_PLAN: 0 (default) = every Zolo-PD iteration takes rk terms; 1 = each
 * iteration takes the r <= rk terms of the cheapest plan to convergence on one GPU.  The
 * reference runs the r terms on r process groups at once; here they run one after another,
 * so an iteration costs a fixed part plus r times a term and fewer terms per iteration can
 * converge sooner.  Before each iteration the CON recursion (pzolopd1.f90:459-472) is
 * searched over the next three iterations and the Newton-Schulz finish with a cost model of
 * this implementation, and the finish is entered from the measured e only when cheaper than
 * the plan; an iteration takes the QR form while CON > 12 (the Cholesky form's error grows
 * with CON).  The coefficients are those of zolo_compute_coeff_kp (exact at any CON, so the
 * recursion predicts the iterate).  Applies with ZOLO_OPT_NS_FINISH and
 * ZOLO_OPT_CHOL_INVERSE (SYM = 'N'); otherwise rk terms.  zolo_stats_t.terms records the
 * counts.  No reference counterpart. */
#define ZOLO_OPT_TERM_PLAN 5
/* ZOLO_OPT_MIXED: 0 (default) = every matrix product on the FP64 tensor path (DMMA);
 * 1 = the mixed form: the large products (K >= 256 and at least two waves of output tiles)
 * of the Cholesky-form iterations, of the Newton-Schulz finish and of forming Q and H run
 * on the INT8 tensor cores with the FP64 product emulated from ZOLO_OPT_MIXED_SLICES digit
 * planes per operand (zolo_ozgemm_dev); the bounds and the QR-form iterations stay on the
 * FP64 tensor path (their graded triangular factors need FP64's elementwise accuracy; the
 * row/column-scaled emulation is accurate normwise).  With 8 planes the emulated product
 * has FP64-level normwise accuracy.  The term plan uses the mixed form's measured costs.
 * No reference counterpart (the reference multiplies with ScaLAPACK PDGEMM in FP64). */
#define ZOLO_OPT_MIXED 6
/* ZOLO_OPT_MIXED_SLICES: digit planes of the emulated products, 6..8 (default 8). */
#define ZOLO_OPT_MIXED_SLICES 7
/* ZOLO_OPT_OWN_BOUNDS: 0 (default) = zolo_pzolopd1 / pzolopd1_ / zolo_pzolopd1_dev scale A
 * by the caller's ALPHA and BETA, as the reference does (pzolopd1.f90:280-291); 1 = they
 * compute ALPHA = ||A||_F and BETA from the QR of A/ALPHA (ZOLO_OPT_BETA_FROB form) and reuse
 * that QR in the first iteration (the zolo_polar_dev flow).  The polar factor does not depend
 * on the scaling of A, so Q is the same to rounding; SYM = 'S' keeps the caller's values.
 * The caller still passes ALPHA, BETA > 0 (checked as before).  No reference counterpart. */
#define ZOLO_OPT_OWN_BOUNDS 8
/* ZOLO_OPT_INJECT_CHOL_FAIL (diagnostic, 0 = off): k + 1 makes the Cholesky-form step of
 * iteration k report a failed factorization (INFO = 1000000 in zolo_stats_t.info) so that
 * the recovery path runs: the step is redone in the QR form, as for a shifted Gram that is
 * not numerically positive definite (the reference ignores PDPOSV's INFO).  Host-side only:
 * no kernel is made to fail. */
#define ZOLO_OPT_INJECT_CHOL_FAIL 9
/* ZOLO_OPT_NORM2_BOUND: 0 (default) = zolo_polar_dev scales by ALPHA = ||A||_F; 1 = ALPHA
 * is lowered to a guaranteed upper bound of ||A||_2 (zolo_bounds_dev mode 3): the power method
 * by repeated squaring of R^T R (R of A/||A||_F), ALPHA = ||A||_F ||(R^T R)^4||_F^(1/8)
 * (1 + 1e-4) = (sum_i sigma_i^16)^(1/16) (1 + 1e-4) >= sigma_max, capped by ||A||_F; BETA is
 * rescaled with it, so the iterate is unchanged and CON = 1/BETA is smaller by ||A||_F/ALPHA.
 * 7n^3/3 extra flops.  The intent of the reference's pdnormest (pdnormest.f90:44-79, a power
 * iteration for ||A||_2).  No reference counterpart as an option. */
#define ZOLO_OPT_NORM2_BOUND 10
/* ZOLO_OPT_BATCH_GRAPH: 1 (default) = zolo_qdwh_batch_dev computes each bucket's iteration
 * schedule on the host from the members' bounds (L_k of a member follows from L_0 alone:
 * the form of every step and its weights) and runs the iterations, H and the unpacking
 * without a host synchronization per step, as one CUDA graph launch: captured the second
 * time a bucket of the same shape and schedule is solved on the handle, replayed afterwards
 * (the first time issues the same launches eagerly and sizes the workspace).  The stopping
 * rule stays PQDWHFACS's (pqdwhfacs.f90:359): a member whose L has converged takes one more
 * step only while its last error is above TOL1^(1/3), which a gate kernel decides on the
 * device from the error just measured; a bucket's final step when it is such a step for all
 * of its members runs only if one of them takes it (one read-back).  Every step's Cholesky
 * INFO and error are read back at the end: a failed Cholesky step reruns the bucket through
 * the synchronized loop (which takes the QR form there), and a member whose error is still
 * above TOL1^(1/3) continues in that loop, so the result is the loop's.  2 = the same
 * schedule, its launches always issued eagerly (no graph).  0 = the host-synchronized loop
 * (pqdwhfacs.f90:359-457 per member, two synchronizations per step). */
#define ZOLO_OPT_BATCH_GRAPH 11
/* ZOLO_OPT_INJECT_BATCH_ERR (diagnostic, 0 = off): 1 = the batched solver's check after a
 * scheduled run sees the first member of each bucket with its last error above TOL1^(1/3), so
 * that member continues in the synchronized loop.  Host-side only. */
#define ZOLO_OPT_INJECT_BATCH_ERR 12
/* ZOLO_OPT_EIG_ZOLO_MIN: the eigensolver (zolo_syev_dev, zolo_svd_dev) splits a node of size
 * n >= this value (default 4096) at its first candidate shift with the polar factor of
 * H - sigma I from Zolo-PD (r = 8 with every cost option: about 0.7x QDWH's time at n = 8192);
 * smaller nodes use QDWH, those of one recursion level as one batched solve; 0 = QDWH for
 * every node (pqdwhsubit.f90's polar factor).  The later candidate shifts always use QDWH. */
#define ZOLO_OPT_EIG_ZOLO_MIN 13
/* The default handle (used by the reference-named host-array entry points) reads its options
 * from the environment when it is created, so an unchanged Fortran driver selects them:
 * ZOLO_FAST=1 sets ZOLO_OPT_SHARED_QR, _NS_FINISH, _CHOL_INVERSE, _BETA_FROB, _TERM_PLAN and
 * _OWN_BOUNDS to 1; ZOLO_OPT_<NAME>=<integer> (e.g. ZOLO_OPT_MIXED=1) sets one option and
 * overrides ZOLO_FAST; ZOLO_DEVICE=<ordinal> picks the GPU.  Invalid values are ignored. */
int zolo_set_option(zolo_handle_t handle, int option, int value);
/* Current value of an option of a handle in *value; -1 for an unknown option. */
int zolo_get_option(zolo_handle_t handle, int option, int* value);

/* ---- host scalar routines (no GPU needed) ---- */
/* Compute_Coeff (Auxil_Zolo.f90:165-200): coeff[0:2rk] = c_i, coeff[2rk:3rk] = -a_i. */
int zolo_compute_coeff(double con, double tol, int rk, double* coeff);
/* The same coefficients computed from the complementary modulus 1/CON directly (the AGM
 * started from (1, 1/CON), and for 1/CON <= 1e-6 the near-unit-modulus expansions of sn, cn),
 * accurate to ~1e-10 relative at any CON > 1, where Compute_Coeff's alpha = acos(1/CON) has a
 * relative error of ~1e-16 CON.  Used by ZOLO_OPT_TERM_PLAN.  No reference counterpart. */
int zolo_compute_coeff_kp(double con, double tol, int rk, double* coeff);
/* The term plan of ZOLO_OPT_TERM_PLAN from CON on (host only, no GPU): terms[k] and
 * qr_form[k] (1 = QR form, 0 = Cholesky form) of each predicted Zolo-PD iteration for an
 * m x n problem with at most rk terms, and *ns_steps, the predicted Newton-Schulz steps of
 * the finish.  prefactored = 1 when the QR of X is at hand for the first iteration (as in
 * zolo_polar_dev).  Returns the number of iterations (at most maxlen), -1 for bad
 * arguments.  The solve itself re-plans before every iteration from the same model and
 * enters the finish from the measured ||X^T X - I||.  No reference counterpart. */
int zolo_plan_terms(double con, int rk, int m, int n, int prefactored, int* terms, int* qr_form, int maxlen,
                    int* ns_steps);
/* mellipke (Auxil_Zolo.f90:36-71) */
void zolo_mellipke(double alpha, double tol, double* k, double* e);
/* MELLIPJ (Auxil_Zolo.f90:73-128) */
void zolo_mellipj(double u, double alpha, double tol, double* sn, double* cn, double* dn);
/* choosem (Auxil_Zolo.f90:130-163) */
int zolo_choosem(double con);
/* hfunc (hfunc.f90:2-42) */
double zolo_hfunc(double x);
/* FONE and next CON of a Zolo iteration (pzolopd1.f90:459-472) */
void zolo_fone_next(double con, const double* coeff, int rk, double* fone, double* next_con);

/* ---- reference-named entry points, host arrays ---- */
/* PQDWHFACS (pqdwhfacs.f90:2-3): QDWH-PD of A - SIGMA*I; Q = polar factor,
 * WORK2 = H = sym(Q^T A) when POLAR = 'T'.  LWORK = -1 or LWORK2 = -1 is a
 * workspace query (WORK(1), WORK(2)).  TAU is not referenced. */
void zolo_pqdwhfacs(char sym, int m, int n, double sigma, const double* a, int ia, int ja, const int* desca,
                    double* q, int iq, int jq, const int* descq, double* work, int lwork, const int* descw,
                    double* tau, double* work2, int lwork2, int* info, char polar);
/* ZOLOPD (zolopd.f90:2-3): older QDWH entry (no SYM, BETA = rcond/sqrt(n), W^{-1} X solve, no IT cap). */
void zolo_zolopd(int m, int n, double sigma, const double* a, int ia, int ja, const int* desca, double* q, int iq,
                 int jq, const int* descq, double* work, int lwork, const int* descw, double* tau, double* work2,
                 int lwork2, int* info, char polar);
/* PZOLOPD1 (pzolopd1.f90:2): Zolo-PD with RK terms from the bounds ALPHA, BETA; Q = polar factor. */
void zolo_pzolopd1(char sym, int rk, int m, int n, double alpha, double beta, const double* as, int ia, int ja,
                   const int* desca, double* q, int iq, int jq, const int* descq, int* info, char polar);
/* PZOLOPD2 (pzolopd2.f90:2): same contract as PZOLOPD1 (the reference's restart variant does not link). */
void zolo_pzolopd2(char sym, int rk, int m, int n, double alpha, double beta, const double* as, int ia, int ja,
                   const int* desca, double* q, int iq, int jq, const int* descq, int* info, char polar);

/* ZoloEig (ZoloEig.f90:2): partial eigendecomposition of the symmetric N x N matrix As
 * from Q = polar factor of As - sigma*I: the Rk = round(||(Q - I)/2||_F^2) eigenpairs
 * below sigma (PQDWHSUBIT subspace iteration, pqdwhsubit.f90:227-312, then an
 * eigensolve of the leading Rk block).  On exit, as in the reference: Q = the subspace
 * basis V (N x N), As = V^T As V, TAU(1:Rk) = eigenvalues (ascending),
 * WORK(1:N*Rk) = eigenvectors (leading dimension N).  CONTXT and MPI_NEWCOMM are
 * ignored (1x1 grid); NBLK is not used.  LWORK >= N*N and LWORK2 >= N*N. */
void zolo_zoloeig(int n, int nblk, double* q, double* as, int contxt, int mpi_newcomm, double* work, int lwork,
                  double* work2, int lwork2, double* tau, int* info);

/* gfortran-mangled aliases: all arguments by reference, hidden CHARACTER lengths last */
void pqdwhfacs_(const char* sym, const int* m, const int* n, const double* sigma, const double* a, const int* ia,
                const int* ja, const int* desca, double* q, const int* iq, const int* jq, const int* descq,
                double* work, const int* lwork, const int* descw, double* tau, double* work2, const int* lwork2,
                int* info, const char* polar, size_t sym_len, size_t polar_len);
void zolopd_(const int* m, const int* n, const double* sigma, const double* a, const int* ia, const int* ja,
             const int* desca, double* q, const int* iq, const int* jq, const int* descq, double* work,
             const int* lwork, const int* descw, double* tau, double* work2, const int* lwork2, int* info,
             const char* polar, size_t polar_len);
void pzolopd1_(const char* sym, const int* rk, const int* m, const int* n, const double* alpha, const double* beta,
               const double* as, const int* ia, const int* ja, const int* desca, double* q, const int* iq,
               const int* jq, const int* descq, int* info, const char* polar, size_t sym_len, size_t polar_len);
void zoloeig_(const int* n, const int* nblk, double* q, double* as, const int* contxt, const int* mpi_newcomm,
              double* work, const int* lwork, double* work2, const int* lwork2, double* tau, int* info);
void pzolopd2_(const char* sym, const int* rk, const int* m, const int* n, const double* alpha, const double* beta,
               const double* as, const int* ia, const int* ja, const int* desca, double* q, const int* iq,
               const int* jq, const int* descq, int* info, const char* polar, size_t sym_len, size_t polar_len);

/* ---- device-pointer entry points (the hot path; no host copies) ---- */
/* QDWH-PD of A - sigma I on device arrays (m >= n).  bounds_mode 0 = PQDWHFACS form,
 * 1 = ZOLOPD form; left_solve != 0 reproduces ZOLOPD's W^{-1} X solve; maxit < 0: no cap.
 * dH may be NULL.  Returns INFO. */
int zolo_qdwh_dev(zolo_handle_t h, char sym, int m, int n, double sigma, const double* dA, int64_t lda, double* dQ,
                  int64_t ldq, double* dH, int64_t ldh, int bounds_mode, int maxit, int left_solve);
/* Batched QDWH-PD of `count` matrices of different sizes on device arrays (no
 * counterpart in the reference, whose drivers factor one matrix per MPI job): member i
 * is the m[i] x n[i] matrix dA[i] (m[i] >= n[i]); dQ[i] receives its polar factor and,
 * when dH is not NULL, dH[i] its H.  Each member follows PQDWHFACS (SYM = 'N',
 * SIGMA = 0, PQDWHFACS bounds on the padded member); members are grouped into buckets
 * of one padded size and each bucket runs as one batched solve with per-member
 * weights and convergence (padding [[A, 0], [0, tau I]] with tau = ||A||_F/sqrt(n)
 * leaves the polar factor and the condition number unchanged).  The pointer and size
 * arrays are host arrays.  info[i] = 0, or > 0 when member i's bounds failed (zero or
 * non-finite input; its outputs are then undefined); iterations[i] (may be NULL)
 * receives member i's iteration count.  Returns 0, or < 0 for a bad argument / GPU
 * failure. */
int zolo_qdwh_batch_dev(zolo_handle_t h, int count, const int* m, const int* n, const double* const* dA,
                        const int64_t* lda, double* const* dQ, const int64_t* ldq, double* const* dH,
                        const int64_t* ldh, int* info, int* iterations);
/* Bucket plan of zolo_qdwh_batch_dev (no reference counterpart).  The members, sorted by n,
 * are split into contiguous runs; each run is one batched solve padded to NB = its largest n
 * and MB = its largest m + NB - n (multiples of 32), and the runs execute concurrently on
 * model[4] worker streams.  The split minimizes the predicted time of the cost model
 *   ms(bucket) = model[0] + model[1] * NB/32 + B * flops(MB, NB) / (model[2] TFLOP/s * NB/(NB + model[3]))
 * (launch-chain latency, shared by the worker streams, plus the members' padded work) by
 * dynamic programming.  zolo_batch_autotune measures the model on the handle's GPU (probe
 * buckets of 1 and 8 members at n = 64, 256, 1024) and stores it in the handle;
 * zolo_batch_set_model sets it (5 values).  zolo_batch_plan (host only, no GPU) returns the
 * number of buckets and fills bucket[i] (member i's bucket), mb[], nb[] (per bucket, count
 * entries suffice) and the predicted ms; model NULL = the defaults; mode 1 = the fixed size
 * ladder instead of the optimized split. */
/* Record of the handle's last zolo_qdwh_batch_dev call: out[0..11] = buckets, largest
 * iteration count, executed FP64 flops (padding included), useful flops (unpadded sizes),
 * device ms, the plan's predicted ms, and the buckets whose iterations ran as a cached graph
 * replayed, a graph captured and launched, the schedule issued eagerly, the synchronized
 * loop, a rerun after a failed Cholesky step, a continuation in the synchronized loop
 * (ZOLO_OPT_BATCH_GRAPH).  Returns 0. */
int zolo_batch_stats(zolo_handle_t h, double* out);
int zolo_batch_autotune(zolo_handle_t h, double* model);
int zolo_batch_set_model(zolo_handle_t h, const double* model);
int zolo_batch_plan(int count, const int* m, const int* n, const double* model, int max_batch, int mode,
                    int* bucket, int* mb, int* nb, double* predicted_ms);
/* Step schedule of one bucket of zolo_qdwh_batch_dev (host only, no GPU): for `count`
 * members with lower bounds l0[b] (PQDWHFACS's L after the bounds; a member with l0 outside
 * (0, 1] takes no step) and IT limit maxit (12 in the solver), *steps receives the number of
 * steps K; when K <= max_steps, qr[k] = 1 for a QR-form step, table[k*5*count + ...] the
 * step's coefficients (count each: c or 1/sqrt(c), cx, cz, an error slot, the conditional
 * flag), ucount[b] member b's unconditional steps, last[b] its last unconditional step and
 * cond[b] its conditional step (-1 = none; see ZOLO_OPT_BATCH_GRAPH).  Output arrays may be
 * NULL.  Returns 0, -2 bad argument, -3 bad maxit, -4 more than max_steps steps. */
int zolo_batch_schedule(int count, const double* l0, int maxit, int max_steps, int* steps, int* qr, double* table,
                        int* ucount, int* last, int* cond);
/* The reference driver's sequence in one call (test_zolodrv1.f90:167-198: the bounds,
 * then PZOLOPD1 with SYM = 'N'), plus H when dH is not NULL: alpha = ||A||_F and
 * beta = 1/(sqrt(n) ||R^{-1}||_1) as zolo_bounds_dev mode 1, then Zolo-PD with rk
 * terms.  The Householder QR of A/alpha that gives beta is reused by the first Zolo-PD
 * iteration when it takes the QR form with ZOLO_OPT_SHARED_QR (X0 = A/(alpha beta) has
 * the same Q), which saves one QR of A.  alpha, beta and the iteration record are in
 * zolo_get_stats.  Returns INFO. */
int zolo_polar_dev(zolo_handle_t h, int rk, int m, int n, const double* dA, int64_t lda, double* dQ, int64_t ldq,
                   double* dH, int64_t ldh);
/* Zolo-PD (PZOLOPD1 semantics) on device arrays; dH may be NULL.  Returns INFO. */
int zolo_pzolopd1_dev(zolo_handle_t h, char sym, int rk, int m, int n, double alpha, double beta, const double* dA,
                      int64_t lda, double* dQ, int64_t ldq, double* dH, int64_t ldh);
/* The driver's bounds (test_zolodrv1.f90:167-189 replaced by a QR + R^{-1} estimate):
 * alpha = ||A||_F, beta = 1/(sqrt(n) ||R^{-1}||_1) for A/alpha = QR (mode 1) or
 * ||A/alpha||_1 / (sqrt(n) ||R^{-1}||_1) (mode 0), or 1/||R^{-1}||_F (mode 2: still a
 * lower bound on sigma_min(A/alpha), and never below mode 1's); mode 3: alpha is the
 * guaranteed ||A||_2 upper bound of ZOLO_OPT_NORM2_BOUND and beta mode 2's bound rescaled to
 * A/alpha (sigma(A/alpha) lies in [beta, 1]).  Returns -7 for another mode. */
int zolo_bounds_dev(zolo_handle_t h, int m, int n, double sigma, const double* dA, int64_t lda, int mode,
                    double* alpha, double* beta);
/* H = (Q^T A + A^T Q)/2 (pqdwhfacs.f90:460-466, ZoloCHK1.f90:80-83). */
int zolo_form_h_dev(zolo_handle_t h, int m, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda,
                    double* dH, int64_t ldh);

/* Symmetric eigendecomposition H = Z diag(w) Z^T (n x n), w ascending: the replacement
 * of ELPA_PDSYEVD2 (elpa_pdsyevd2.F90:199-200) -- spectral divide-and-conquer on the
 * polar decomposition (QDWH of H - sigma I, subspace split as pqdwhsubit.f90:227-312,
 * recursively) with batched Jacobi leaves.  Returns 0, or > 0 if no split point worked.
 * zolo_get_stats afterwards: iterations = splits, qr_iterations = QDWH iterations,
 * chol_iterations = leaves, last_err = largest split residual / ||H||_F, ms_step[l] = device
 * ms of top-down level l, ms_finish = the leaves, ms_h = the back-transformation,
 * ns_steps = subspace passes, terms[0..3] = QDWH solves, Zolo-PD solves, nodes solved in
 * a level's batched QDWH, workspace buffers grown during the call, con[0..3] = host wall ms summed over the levels of reading the
 * diagonals, the batched QDWH solves, the concurrent splits and freeing split nodes. */
int zolo_syev_dev(zolo_handle_t h, int n, const double* dH, int64_t ldh, double* dW, double* dZ, int64_t ldz);
/* Zolo-SVD (test_zolodrv1.f90 + ZoloCHK1.f90:80-91): A = U diag(s) V^T for m >= n via
 * QDWH-PD (algo 0) or Zolo-PD with rk terms (algo 1), H = sym(Q^T A), H = V diag(s) V^T,
 * U = Q V.  s ascending (the order ZoloCHK1 receives from ELPA). */
int zolo_svd_dev(zolo_handle_t h, int algo, int rk, int m, int n, const double* dA, int64_t lda, double* dU,
                 int64_t ldu, double* dS, double* dV, int64_t ldv);
/* ZoloEig on device arrays: *rk eigenpairs of A below the shift used to form Q. */
int zolo_zoloeig_dev(zolo_handle_t h, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, int* rk,
                     double* dW, double* dZ, int64_t ldz);

/* ---- kernel-level entry points (building blocks, used by the parity tests) ---- */
/* C = alpha op(A) op(B) + beta C (PDGEMM on a 1x1 grid); tri = lower-triangle-only output,
 * kfrom_n = 1: op(B) is lower triangular (TRMM-like skip of k < column);
 * kfrom_n = 2: op(A) is upper triangular (skip of k < row); kfrom_n = 3: both (k >= max(row, column)). */
int zolo_dgemm_dev(zolo_handle_t h, char transa, char transb, int m, int n, int k, double alpha, const double* dA,
                   int64_t lda, const double* dB, int64_t ldb, double beta, double* dC, int64_t ldc, int tri,
                   int kfrom_n);
/* C = alpha op(A) op(B) + beta C like zolo_dgemm_dev, with the FP64 products emulated on
 * the INT8 tensor cores (tcgen05.mma kind::i8): each row of op(A) and column of op(B) is
 * scaled by a power of two and split into `slices` (6, 7 or 8) signed 7-bit digit planes,
 * the digit products are accumulated exactly in INT32 and recombined in FP64.  slices = 8
 * gives FP64-level normwise accuracy.  Requires slices * 127^2 * k < 2^31 (k <= 16642 at 8)
 * and finite inputs.  Returns 0, -i for a bad argument i, -1000-cudaError, or -2000-code
 * when a pipeline wait of the kernel timed out (code 901..906).  No reference counterpart:
 * the reference's products are ScaLAPACK PDGEMM in FP64 (zolochol.f90:88-89). */
int zolo_ozgemm_dev(zolo_handle_t h, char transa, char transb, int m, int n, int k, double alpha, const double* dA,
                    int64_t lda, const double* dB, int64_t ldb, double beta, double* dC, int64_t ldc, int tri,
                    int kfrom_n, int slices);
/* Lower Cholesky in place (PDPOTRF 'L'); returns LAPACK INFO. */
int zolo_dpotrf_dev(zolo_handle_t h, int n, double* dA, int64_t lda);
/* Y = X L^{-T} (trans = 'T') or Y = X L^{-1} (trans = 'N'); X is overwritten (workspace). */
int zolo_dtrsm_dev(zolo_handle_t h, char trans, int m, int n, const double* dL, int64_t ldl, double* dX, int64_t ldx,
                   double* dY, int64_t ldy);
/* Y = L^{-1} for lower-triangular L (PDTRTRI 'L','N' on a 1x1 grid; only L's lower triangle
 * is read; Y's upper triangle is set to zero). Returns 0, or -i for a bad argument i. */
int zolo_dtrtri_dev(zolo_handle_t h, int n, const double* dL, int64_t ldl, double* dY, int64_t ldy);
/* Structured Householder QR (MPDGEQRF, mpdgeqrf.f:5-324): mtot x n in place; m_top < 0 = unstructured.
 * dT receives ceil(n/32) blocks of 32x32 compact-WY factors. */
int zolo_dgeqrf_dev(zolo_handle_t h, int mtot, int n, int m_top, double* dW, int64_t ldw, double* dtau, double* dT);
/* Explicit Q (MPDORGQR, mpdorgqr.f:5-348) from zolo_dgeqrf_dev's output. */
int zolo_dorgqr_dev(zolo_handle_t h, int mtot, int n, int m_top, const double* dW, int64_t ldw, const double* dT,
                    double* dQ, int64_t ldq);
/* One Zolotarev term through ZOLOQR (zoloqr.f90:82-112): Z = (a/sqrt(c)) Q1 Q2^T of [X; sqrt(c) I]. */
int zolo_zoloqr_dev(zolo_handle_t h, int m, int n, const double* dX, int64_t ldx, double c, double a, double* dZ,
                    int64_t ldz);
/* One Zolotarev term through ZOLOCHOL (zolochol.f90:87-113): Z = a X (X^T X + c I)^{-1}. */
int zolo_zolochol_dev(zolo_handle_t h, int m, int n, const double* dX, int64_t ldx, double c, double a, double* dZ,
                      int64_t ldz);
/* FormX2 (FormX2.f90:73-89): X <- (X + Z)/fone; returns ||X_new - X_old||_F in *err. */
int zolo_formx2_dev(zolo_handle_t h, int m, int n, double fone, double* dX, int64_t ldx, const double* dZ,
                    int64_t ldz, double* err);

/* ---- MatrixMarket input (prepare_matrix.f90:154-321 prepare_real_GEM, :638-759
 * prepare_real_symm_MM), host only ----
 * Reads the MatrixMarket file `path` (coordinate or array; real, double or integer values)
 * into the column-major m x n host matrix a (leading dimension lda >= m), zero where no entry
 * is given.  A `symmetric` file (one triangle stored) yields the full matrix A + A^T with the
 * diagonal halved, as the reference builds it; a `general` file is used as stored; any other
 * symmetry class is loaded as stored and reported as ZOLO_MM_OTHER.  With a = NULL only the
 * header is read (m, n, kind).  kind may be NULL.  The reference's sigma is 0 (its diagonal
 * shift is commented out, prepare_matrix.f90:260), so no shift is applied.  Returns 0; -1 a
 * null argument, -6 lda < m, -10 the file cannot be opened, -11 not a MatrixMarket matrix
 * banner, -12 neither coordinate nor array, -13 complex or pattern values, -14 a bad size
 * line, -15 too few entries, -16 an index out of range, -17 a non-square symmetric file. */
#define ZOLO_MM_GENERAL 0
#define ZOLO_MM_SYMMETRIC 1
#define ZOLO_MM_OTHER 2
int zolo_read_mm(const char* path, int* m, int* n, int* kind, double* a, int64_t lda);

/* ---- allocation-free entry point (no counterpart in the reference) ----
 * Lower Cholesky in place of an n x n SPD matrix on the caller's stream, with no
 * device allocation and no handle: for callers that cannot let a library call
 * cudaMalloc -- hosts whose device memory is owned entirely by another allocator
 * (a framework's caching pool or an application arena) and latency-sensitive hosts
 * that cannot accept cudaMalloc's device-wide synchronisation.  Same algorithm and
 * result as zolo_dpotrf_dev.  Its scratch is a fixed 2.5 MiB static device array held
 * by every GPU that loads the library, so n <= ZOLO_NOALLOC_MAX_N.  The first call on
 * a device looks the array's address up (cudaGetSymbolAddress) and should be made
 * before any stream capture.  All calls share the scratch: calls that overlap on the
 * GPU race and must be serialised by the caller.  Synchronises `stream` before
 * returning.  Any lda >= max(1,n) is accepted; dA must be 8-byte aligned.  Returns
 * LAPACK INFO (> 0: not positive definite), -1 if n < 0 or n > ZOLO_NOALLOC_MAX_N,
 * -2 if dA is null (n > 0), -3 if lda < max(1,n), -1000 - cudaError on a CUDA error
 * (-1000 - cudaErrorMisalignedAddress for a dA that is not 8-byte aligned). */
#define ZOLO_NOALLOC_MAX_N 1024
int zolo_dpotrf_noalloc(int n, double* dA, int64_t lda, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* ZOLO_B200_H */
