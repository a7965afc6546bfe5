/*
 * fastkpc_b200 — C ABI of the B200 kernel-PC conditional-independence path.
 *
 * Plain C types only: pointers, sizes and PODs.  Every function returns 0 on
 * success and a positive FKPC_STATUS_* code on failure; fkpc_last_error()
 * then holds a message for the calling thread.  Inputs are borrowed (the
 * caller keeps ownership); results returned through fkpc_result** are owned
 * by the library until fkpc_result_free().  Data matrices are column-major
 * n x p binary64 (the layout of an R numeric matrix).  Indices are 0-based.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the wyjistest/fastkpc tree).
 */
#ifndef FASTKPC_B200_H
#define FASTKPC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define FKPC_ABI_VERSION 5

#if defined(__GNUC__)
#define FKPC_API __attribute__((visibility("default")))
#else
#define FKPC_API
#endif

/* status codes */
#define FKPC_OK 0
#define FKPC_STATUS_INVALID_ARGUMENT 1   /* envelope / argument check failed */
#define FKPC_STATUS_CUDA 2               /* CUDA runtime error */
#define FKPC_STATUS_NUMERIC 3            /* non-finite objective / statistic */
#define FKPC_STATUS_NOT_CONVERGED 4      /* optimizer or gamma tail iteration cap */
#define FKPC_STATUS_RANK 5               /* design or augmented system rank deficient */
#define FKPC_STATUS_ALLOCATION 6         /* host or device allocation failed */
#define FKPC_STATUS_NO_DEVICE 7          /* no usable CUDA device */

/* CI methods (kpcalg ic.method) */
#define FKPC_DCC_GAMMA 0
#define FKPC_DCC_PERM 1
#define FKPC_HSIC_GAMMA 2
#define FKPC_HSIC_PERM 3

/* execution forms */
#define FKPC_MODE_BATCHED 0  /* every test of a level in one batched launch set */
#define FKPC_MODE_PLAIN 1    /* one launch set per CI test */

/* smoothing-parameter selection for additive designs (|S| >= 3) */
#define FKPC_SELECT_MAGIC 0      /* mgcv magic's Newton / halving search, as the reference */
#define FKPC_SELECT_GN_NEWTON 1  /* Newton on the Gauss-Newton Hessian of GCV (fkpc_gcv_adjoint's) */

/* per-record flags */
#define FKPC_FLAG_GUARDED 1u       /* dcc.gamma p came from the low-rank refinement */
#define FKPC_FLAG_DIRECT 2u        /* |S| = 0: raw columns, no regression */
#define FKPC_FLAG_RANK_TRUNCATED 4u /* a residual fit dropped a coefficient by magic's rank rule (sqrt(eps)) */

typedef struct fkpc_options {
  double alpha;                 /* significance level; the reference fixes 0.1 */
  double index;                 /* dCov exponent; legacy semantics fix 1 */
  int num_col;                  /* low-rank / inchol rank cap; reference fixes 35 */
  int max_conditioning_size;    /* m.max; negative means Inf (p - 2) */
  int ci_method;                /* FKPC_DCC_GAMMA ... FKPC_HSIC_PERM */
  double hsic_sig;              /* Gaussian kernel width sig (rbfdot sigma = 1/sig) */
  int permutation_replicates;   /* R for the permutation methods, 1..10000 */
  int has_seed;                 /* permutation methods require a seed */
  unsigned int seed;            /* set.seed() value for the R-compatible stream */
  int mode;                     /* FKPC_MODE_BATCHED or FKPC_MODE_PLAIN */
  int collect_trace;            /* keep the per-test logical trace */
  int device;                   /* CUDA device ordinal */
  int strict;                   /* reference envelope: alpha 0.1, index 1, numCol 35 < n, 2 <= p <= 64 */
  int selection;                /* FKPC_SELECT_MAGIC (default) or FKPC_SELECT_GN_NEWTON */
  int level_graph;              /* batched gamma methods: 1 = set each batch up, then run it as one
                                   captured CUDA graph; 0 (default) = the one-shot flow that overlaps
                                   the host set-up with the device work */
} fkpc_options;

/* One CI test result. */
typedef struct fkpc_ci_record {
  double p_value;      /* p used for the decision */
  double p_exact;      /* dcc.gamma exact-screen p (== p_value for other methods) */
  double statistic;    /* nV2, HSIC or the permutation statistic */
  double mean;         /* gamma-approximation mean (NaN for permutation methods) */
  double variance;     /* gamma-approximation variance (NaN for permutation methods) */
  int status;          /* FKPC_OK or a status code */
  unsigned int flags;  /* FKPC_FLAG_* */
} fkpc_ci_record;

/* Per-stage device timings of the last batched call, milliseconds. */
typedef struct fkpc_stage_stats {
  double setup_ms;          /* host design setup (TPRS / additive bases, QR) */
  double upload_ms;         /* host -> device copies */
  double fit_ms;            /* GCV selection + residuals */
  double statistic_ms;      /* dCov / HSIC statistics and p-values */
  double refine_ms;         /* dcc.gamma guard-band low-rank refinement */
  double download_ms;       /* device -> host copies */
  double total_ms;          /* wall time of the call */
  int designs;              /* distinct conditioning sets */
  int targets;              /* distinct (target, S) residual fits */
  int pairs;                /* CI tests evaluated */
  int guarded;              /* tests refined in the guard band */
  int kernel_launches;      /* library kernels launched by the call */
  double h2d_bytes;         /* host -> device bytes copied by the call */
  double d2h_bytes;         /* device -> host bytes copied by the call */
  double fit_evaluations;   /* GCV objective evaluations over all fits */
  double fit_flops;         /* algorithmic FP64 flops of the fit stage */
  double statistic_flops;   /* algorithmic FP64 flops of the statistic stage */
  double fit_iterations;    /* optimizer iterations over all fits */
  int lowrank_components;   /* guarded components given a low-rank eigen-solve */
  int lowrank_steps_max;    /* most Lanczos steps any of them took */
  double lowrank_steps_mean;
  double device_ms;         /* device time of the batch's launch sequence */
  int designs_built;        /* conditioning-set designs the call set up (not found in the cache) */
  int smooths_built;        /* per-variable (univariate) smooth bases the call set up */
  /* timeline of a one-shot call (fkpc_ci_level_batch and the skeleton's levels) */
  double plan_ms;           /* host: components and conditioning sets of the tests */
  double tprs_host_ms;      /* host: unique locations and staging of the thin-plate set-up */
  double design_host_ms;    /* host: design descriptors, initial.sp and penalty roots */
  double smooth_wait_ms;    /* host blocked until the device's univariate smooth bases landed */
  double late_wait_ms;      /* host blocked until the device's bivariate smooth bases landed */
  double prefit_device_ms;  /* device timeline from the call's first launch to the first fit launch */
} fkpc_stage_stats;

typedef struct fkpc_trace_row {
  int level;
  int task_index;      /* position in the canonical level plan */
  int edge_x, edge_y;  /* edge, edge_x < edge_y */
  int x, y;            /* tested orientation */
  int s_offset;        /* into fkpc_result.trace_s_values */
  int s_count;
  double p_value;
  double p_exact;
  int deleted;         /* p_value >= alpha */
  unsigned int flags;
} fkpc_trace_row;

typedef struct fkpc_result {
  int n, p;
  int levels;                /* levels executed */
  int* adjacency;            /* p*p, column-major, 1 = edge kept */
  double* pmax;              /* p*p, column-major; -Inf where untested */
  int* sepset_offsets;       /* p*p+1, CSR over cells i + p*j (column-major) */
  int* sepset_values;        /* conditioning sets of the deleting tests */
  int* n_edgetests;          /* tests per level, length levels */
  int trace_rows;
  fkpc_trace_row* trace;     /* canonical replay order; NULL unless collect_trace */
  int* trace_s_values;
  double elapsed_sec;
  fkpc_stage_stats stats;    /* accumulated over levels */
} fkpc_result;

/*
 * Full default-Inf kernel-PC skeleton (pcalg "stable" level replay).
 * Replaces C_full_cuda_ci_one_call_skeleton / _method
 * (fastkpc/src/r_api_cuda.cpp:9183-9249, driven by
 * fastkpc/src/full_cuda_ci_one_call.cpp:5040) as reached from
 * fastkpc_compatible_cuda_skeleton() (fastkpc/R/fast_kpc.R:56-130).
 */
FKPC_API int fkpc_skeleton_run(const double* data_colmajor, int n, int p,
                      const fkpc_options* options, fkpc_result** out);
FKPC_API void fkpc_result_free(fkpc_result* result);

/* one CI test of the orientation's regrVonPS calls */
typedef struct fkpc_orientation_test {
  int reverse;         /* 0: the tested node's own call; 1: the reverse call for a W in S */
  int target;          /* the regressed node */
  int other;           /* the member of S tested against the residual */
  int s_offset;        /* S, into fkpc_orientation.set_values */
  int s_count;
  int z_offset;        /* S + parents(target), sorted: the residual's conditioning set */
  int z_count;
  double p_value;
  int rejected;        /* p_value < alpha */
} fkpc_orientation_test;

typedef struct fkpc_orientation {
  int p;
  int* pdag;                     /* p*p column-major: pdag[i+p*j] = 1, pdag[j+p*i] = 0 is i -> j; both 1: i - j */
  int collider_orientations;     /* collider triples that changed the graph */
  int rule1_orientations;        /* edges each rule changed */
  int rule2_orientations;
  int rule3_orientations;
  int generalized_orientations;  /* accepted S -> V orientations */
  int regrvonps_calls;
  int residual_fits;             /* residuals fitted on the device */
  int residual_cache_hits;       /* residuals reused for a repeated (target, conditioning set) */
  int tests;
  fkpc_orientation_test* trace;  /* every CI test in call order */
  int* set_values;
  double elapsed_sec;
} fkpc_orientation;

/*
 * WAN-PDAG orientation of a skeleton (kpcalg udag2wanpdag with kpc()'s
 * defaults: colliders, generalised orientations by regrVonPS, rules 1-3 to a
 * fixed point; no unfaithful triples, solve.confl = FALSE).  adjacency is
 * p*p column-major (symmetric, zero diagonal); the sepsets are a CSR over
 * cells i + p*j as fkpc_result holds them.  options supplies alpha, the CI
 * method (gamma methods), numCol, the HSIC sig, the selection and the device.
 * Every residual is fitted and every CI test evaluated on the device.
 * Replaces fastkpc_orient_wanpdag_kpcalg_authority
 * (fastkpc/R/fast_kpc.R:263-330) and C_fast_orient_wanpdag_cuda
 * (fastkpc/R/cuda_native.R:2695, fastkpc/src/wanpdag_engine.hpp:12).
 */
FKPC_API int fkpc_orient_wanpdag(const double* data_colmajor, int n, int p, const int* adjacency,
                                 const int* sepset_offsets, const int* sepset_values,
                                 const fkpc_options* options, fkpc_orientation** out);
FKPC_API void fkpc_orientation_free(fkpc_orientation* orientation);

/*
 * One regrVonPS call for fkpc_orient_wanpdag_custom: fills p_values[k] with
 * the p-value of the test of (residual of ``target`` on ``conditioning``
 * (S + parents(target), sorted), data[:, subset[k]]) for k < subset_count,
 * and returns 0, or a positive FKPC_STATUS_* code.
 */
typedef int (*fkpc_regrvonps_evaluator)(void* user, int target, const int* subset, int subset_count,
                                        const int* conditioning, int conditioning_count, double* p_values);

/*
 * fkpc_orient_wanpdag's graph logic with every regrVonPS call answered by
 * ``evaluator`` (no device use): the hook through which a host supplies its
 * own CI backend.  Replaces orient_wanpdag_native's evaluator argument
 * (fastkpc/src/wanpdag_engine.hpp:12-16).
 */
FKPC_API int fkpc_orient_wanpdag_custom(int p, const int* adjacency, const int* sepset_offsets,
                                        const int* sepset_values, double alpha,
                                        fkpc_regrvonps_evaluator evaluator, void* user,
                                        fkpc_orientation** out);

/*
 * Evaluator of one level's CI tests for fkpc_skeleton_run_custom: fills
 * out[t] for test t = (x[t], y[t], S = s_values[s_offsets[t] ..
 * s_offsets[t+1])) and returns 0, or a positive FKPC_STATUS_* code.
 */
typedef int (*fkpc_level_evaluator)(void* user, int level, const int* x, const int* y, const int* s_offsets,
                                    const int* s_values, int count, fkpc_ci_record* out);

/*
 * fkpc_skeleton_run with every level's batch of tests evaluated by
 * ``evaluator`` (batched gamma methods only): the hook through which a host
 * splits a level's independent tests across GPUs and gathers their records,
 * while the level plan, the canonical replay, pMax and the sepsets stay
 * here.  Uses no device itself.  No reference counterpart (the reference
 * runs one GPU).
 */
FKPC_API int fkpc_skeleton_run_custom(const double* data_colmajor, int n, int p, const fkpc_options* options,
                                      fkpc_level_evaluator evaluator, void* user, fkpc_result** out);

/*
 * One batch of CI tests (x, y, S): residuals of x and y on S by GCV-selected
 * thin-plate / additive smooths, then the statistic and p-value.  Test t uses
 * S = s_values[s_offsets[t] .. s_offsets[t+1]).
 * Replaces execute_group (fastkpc/src/full_cuda_ci_one_call.cpp:4197-5038)
 * and its CUDA calls run_full_cuda_ci_phase35_exact_batch
 * (fastkpc/src/cuda/full_cuda_ci_vertical.cu:2316) and
 * run_full_cuda_ci_method_batch (fastkpc/src/cuda/full_cuda_ci_method_batch.cu:2923).
 * ``stats`` may be NULL.
 */
FKPC_API int fkpc_ci_level_batch(const double* data_colmajor, int n, int p,
                        const int* x, const int* y, const int* s_offsets,
                        const int* s_values, int count,
                        const fkpc_options* options, fkpc_ci_record* out,
                        fkpc_stage_stats* stats);

/*
 * A session: the data matrix stays loaded on one device, with the cache of
 * conditioning-set designs and smooth bases built from it, across calls of
 * fkpc_session_evaluate -- the form a host that evaluates a skeleton level by
 * level (one process per GPU, each taking a share of every level) needs, so
 * that a design is set up once per device and not once per level.
 * fkpc_session_load replaces any earlier session on ``device``.  Any other
 * call that takes a data matrix on the same device (fkpc_ci_level_batch,
 * fkpc_skeleton_run, ...) loads its own data and ends the session; a later
 * fkpc_session_evaluate then fails with FKPC_STATUS_INVALID_ARGUMENT.
 * fkpc_session_evaluate has the arguments and results of fkpc_ci_level_batch
 * without the data; options->device selects the session.
 * Same reference counterpart as fkpc_ci_level_batch (the reference keeps its
 * caches inside one skeleton call, fastkpc/src/full_cuda_ci_one_call.cpp:5040).
 */
FKPC_API int fkpc_session_load(const double* data_colmajor, int n, int p, int device);
FKPC_API int fkpc_session_evaluate(const int* x, const int* y, const int* s_offsets,
                                   const int* s_values, int count,
                                   const fkpc_options* options, fkpc_ci_record* out,
                                   fkpc_stage_stats* stats);

/*
 * The plain per-test form: one CI test, one launch set, synchronised.
 * Replaces the vertical single-pair route
 * (fastkpc/src/cuda/full_cuda_ci_vertical.cu:1240-1339).
 */
FKPC_API int fkpc_ci_plain_one(const double* data_colmajor, int n, int p, int x, int y,
                      const int* s_values, int s_count,
                      const fkpc_options* options, fkpc_ci_record* out);

/*
 * regrXonS residuals for ``count`` (target, S) fits: residuals is n x count
 * column-major; log_sp receives up to ``max_penalties`` selected
 * log smoothing parameters per fit (row-major count x max_penalties, unused
 * entries NaN); status per fit (a failed fit leaves NaN residuals and its
 * FKPC_STATUS_* code; the call itself still returns 0).
 * Replaces single_penalty_gcv_cuda (fastkpc/src/cuda/mgcv_single_penalty_gcv.cu:1863),
 * multi_penalty_gcv_capacity_optimize_batch
 * (fastkpc/src/cuda/mgcv_multi_penalty_gcv_capacity.cpp:233) and
 * solve_fixed_sp_batch (fastkpc/src/cuda/mgcv_fixed_sp_runtime.cu:5668).
 */
FKPC_API int fkpc_regress_batch(const double* data_colmajor, int n, int p,
                       const int* target, const int* s_offsets,
                       const int* s_values, int count,
                       const fkpc_options* options, double* residuals,
                       double* log_sp, int max_penalties, int* status);

/*
 * Statistics and p-values for ``count`` pairs of given residual columns
 * (residuals n x m column-major; pair t uses columns left[t], right[t]).
 * ``permutations`` (count x replicates x n, int32) is required for the
 * permutation methods and ignored otherwise.
 * Replaces the statistic stage of run_full_cuda_ci_phase35_exact_batch,
 * run_full_cuda_ci_phase35_legacy_eig_batch
 * (fastkpc/src/cuda/full_cuda_ci_vertical.cu:2316,2940) and
 * run_full_cuda_ci_method_batch.
 */
FKPC_API int fkpc_stat_batch(const double* residuals, int n, int m, const int* left,
                    const int* right, int count, const int* permutations,
                    const fkpc_options* options, fkpc_ci_record* out);

/*
 * Permutation tables of ``count`` consecutive tests in the R-compatible
 * stream of set.seed(seed) (RNGkind Mersenne-Twister, sample.kind
 * "Rejection"): out is count x replicates x n int32, test after test in
 * stream order -- dcc.perm: energy's dCOVtest swaps (one vector carried
 * across a test's replicates); hsic.perm: sample(n) per replicate.  The
 * tables fkpc_stat_batch's permutation methods take; no device work.
 * Replaces the host table builder of fastkpc/src/full_cuda_ci_one_call.cpp:464-567.
 */
FKPC_API int fkpc_permutation_tables(unsigned int seed, int ci_method, int n, int replicates, int count, int* out);

/*
 * GCV score, gradient and Gauss-Newton Hessian in rho = log(lambda) of the
 * additive-smooth fit of data[:, target] on S (|S| >= 3, m = |S|) at
 * ``count`` given points, plus the exact Hessian for comparison, on CUDA
 * device ``device``.
 * Arrays are count-major: log_lambda and grad are count x m, the Hessians
 * count x m x m (row-major per point); any output may be NULL.  Entry j
 * of a point belongs to the j-th smallest variable of S.  The
 * Gauss-Newton Hessian is 2 J'J of f = sqrt(n) r / (n - EDF), V = |f|^2.
 * Replaces the analytic derivative block of
 * evaluate_multi_penalty_target_device
 * (fastkpc/src/cuda/mgcv_multi_penalty_gcv.cu:1274-1490).
 */
FKPC_API int fkpc_gcv_adjoint(const double* data_colmajor, int n, int p, int target,
                     const int* s_values, int s_count, int count,
                     const double* log_lambda, double* score, double* grad,
                     double* gn_hessian, double* exact_hessian, int device);

/*
 * Q(a[i], x[i]), the regularised upper incomplete gamma function that every
 * gamma-approximation p-value (dcc.gamma, hsic.gamma) takes, evaluated by the
 * statistic kernels' own device routine on CUDA device ``device``; ok[i] = 0
 * where the series or continued fraction did not converge.  Replaces
 * regularized_gamma_q (fastkpc/src/cuda/full_cuda_ci_vertical.cu:334-398)
 * as a testable unit.
 */
FKPC_API int fkpc_gamma_q_eval(int device, const double* a, const double* x, int count,
                               double* q, int* ok);

/*
 * Staged form of fkpc_ci_level_batch on the engine of options->device, for
 * timing the device work with every input already resident in HBM:
 * prepare (host set-up, uploads, graph capture), execute (``repeats`` graph
 * launches; *device_ms = CUDA-event time of all of them on the engine's
 * stream), collect (wait, download, validate).
 * Same reference counterpart as fkpc_ci_level_batch.
 */
FKPC_API int fkpc_batch_prepare(const double* data_colmajor, int n, int p,
                                const int* x, const int* y, const int* s_offsets,
                                const int* s_values, int count,
                                const fkpc_options* options);
FKPC_API int fkpc_batch_execute(int device, int repeats, double* device_ms);
FKPC_API int fkpc_batch_collect(int device, fkpc_ci_record* out,
                                fkpc_stage_stats* stats);
/*
 * Replay one kernel of the prepared batch alone ``repeats`` times and return
 * its mean CUDA-event duration (ms) and its algorithmic FP64 flops per launch.
 * Stages: 0 fit single, 1 fit multi (q <= 40), 2 fit multi (q <= 76),
 * 3 dCov components, 4 dCov pairs, 5 HSIC components, 6 HSIC pairs,
 * 7 low-rank eigen, 8 low-rank pairs, 9 fit multi (q <= 112), 10 fit
 * multi (q <= 560, |S| <= 62).  Run
 * fkpc_batch_execute first.
 * No reference counterpart (measurement utility).
 */
FKPC_API int fkpc_batch_time_stage(int device, int stage, int repeats,
                                   double* avg_ms, double* flops_per_launch);
/*
 * Dense FP64 FMA throughput of the device (TFLOP/s), measured with
 * independent FMA chains in every thread.  No reference counterpart.
 */
FKPC_API int fkpc_measure_fp64_peak(int device, double* tflops);

/*
 * Schedule choices of a device's engine.  No result depends on them: records
 * are bit-identical under every setting (fastkpc_b200/autotune.py checks
 * this while it times the candidates).  No reference counterpart.
 */
typedef struct fkpc_tuning {
  int defer_evaluations;    /* a one-warp GCV search still running after this many evaluations
                               moves to the speculative continuation (0: never); default 25 */
  int split_statistics;     /* 1 (default): the statistics of pairs whose fits are final run
                               beside the continuation; 0: after every fit */
  int lowrank_ctas_per_sm;  /* guard-band Lanczos CTAs per SM, 1..4; default 2 */
  int tprs_ctas_per_sm;     /* single-vector thin-plate Lanczos CTAs per SM, 1..4; default 2 (the block Lanczos runs two per SM, as its shared memory allows) */
} fkpc_tuning;
FKPC_API int fkpc_get_tuning(int device, fkpc_tuning* tuning);
FKPC_API int fkpc_set_tuning(int device, const fkpc_tuning* tuning);

/*
 * Host-only design set-up for one conditioning set S (no device needed):
 * q and m always; when non-NULL, X (n x q column-major), penalties
 * (m blocks, each placed in a full q x q matrix, column-major, m*q*q) and
 * the mgcv initial log smoothing parameters (m).
 * Replaces full_cuda_ci_native_setup
 * (fastkpc/src/full_cuda_ci_native_setup.cpp:1321) with initial.sp
 * (:1019-1127).
 */
FKPC_API int fkpc_design_export(const double* data_colmajor, int n, int p,
                                const int* s_values, int s_count, int* q, int* m,
                                double* X, double* penalties,
                                double* initial_log_sp);

/*
 * The device thin-plate set-up of the bivariate smooth on columns {a, b}
 * (k = 30), for checking the device eigensolvers: n_u (the unique
 * locations), path (2: block Lanczos, taken when 120 <= n_u <= 512; 1:
 * single-vector Lanczos; 0: not taken by the device, values and vectors
 * untouched), ok (1 when the Ritz pairs converged), the 30 Ritz values of
 * the eta matrix of largest magnitude in descending order and their vectors
 * (n_u x 30 column-major, each of unit norm with its largest-magnitude entry
 * positive; ``vectors`` holds at least n x 30 doubles).  The eigen problem of
 * fastkpc/src/full_cuda_ci_native_setup.cpp:114-152 (Lanczos at :303).
 */
FKPC_API int fkpc_tprs_export(const double* data_colmajor, int n, int p, int a, int b, int device, int* n_u,
                              int* path, int* ok, double* values, double* vectors);

/*
 * Exact-screen dcc.gamma records for ``count`` pairs without allocating any
 * device memory, for callers that cannot call cudaMalloc -- code running
 * inside a host framework that owns every device allocation, or that must
 * not allocate once running.  No counterpart in the reference.
 * residuals: device pointer, n x m column-major binary64; pairs: device
 * pointer to 2*count ints (left, right per pair); out: device pointer to
 * count records (p_value = p_exact = the exact-screen p; no guard-band
 * refinement); stream: a cudaStream_t or NULL.  Scratch lives in one fixed
 * 8 MiB device array inside the library: n <= 4096 and
 * n*m + 2.5*m + 2*count + 1 <= 2^20 doubles, otherwise the call fails with
 * FKPC_STATUS_INVALID_ARGUMENT; count == 0 returns FKPC_OK with no device
 * work.  Every call looks the array's address up on the current device; the
 * first call on a device loads the library's device code there (make it
 * before any stream capture).  Calls share the array: calls that overlap on
 * the GPU race.  A pair index outside [0, m) fails the call with
 * FKPC_STATUS_INVALID_ARGUMENT after the kernels ran on clamped indices; the
 * contents of ``out`` are undefined whenever the call fails.  Synchronises
 * ``stream`` before returning.
 */
FKPC_API int fkpc_dcov_gamma_noalloc(const double* residuals, int n, int m,
                                     const int* pairs, int count,
                                     fkpc_ci_record* out, void* stream);

FKPC_API const char* fkpc_last_error(void);
FKPC_API int fkpc_abi_version(void);
FKPC_API void fkpc_default_options(fkpc_options* options);

#ifdef __cplusplus
}
#endif

#endif /* FASTKPC_B200_H */
