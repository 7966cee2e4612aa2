/*
 * cyclops_b200.h -- C ABI of libcyclops_b200.so, the sm_100a engine for the
 * Cyclops cyclic-coordinate-descent (CCD) inner loop.
 *
 * Three layers, all plain C (no C++ or torch types cross this boundary):
 *
 *  1. Datasets: a device-resident copy of the reference's CompressedDataMatrix
 *     plus y / time / stratum vectors (reference: src/cyclops/ModelData.h:178-362,
 *     src/cyclops/CompressedDataMatrix.h:243-452).
 *
 *  2. Engines: one fit's per-coordinate engine, a function-for-function
 *     replacement of the virtual surface of
 *     `bsccs::AbstractModelSpecifics` (src/cyclops/engine/AbstractModelSpecifics.h:36-122).
 *     Each cyc_engine_* call below names the virtual it replaces.  Values
 *     cross as FP64; state stays on the GPU between calls.  This is what
 *     `CyclicCoordinateDescent` drives through the C++ adapter
 *     cyclops_b200/adapter/CudaModelSpecifics.h.
 *
 *  3. Solvers: the whole CCD loop (coordinate step, bounds, convergence test)
 *     kept on the GPU, for one fit or for many fits that share one dataset
 *     (cross-validation folds x prior grid, bootstrap replicates).  The
 *     reference runs this loop on the host in
 *     CyclicCoordinateDescent::update/findMode (src/cyclops/CyclicCoordinateDescent.cpp:586-1216)
 *     and runs independent fits on CPU threads
 *     (src/cyclops/drivers/AbstractCrossValidationDriver.cpp:131-248).
 *
 * Every function returns 0 on success and a nonzero cyc_status otherwise;
 * cyc_last_error() then describes the failure (thread-local).  Nothing
 * throws across this boundary.
 */
#ifndef CYCLOPS_B200_H
#define CYCLOPS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums (values match the reference's enums) ------------------------ */

/* FormatType, src/cyclops/CompressedDataMatrix.h:36-38 */
enum cyc_format { CYC_DENSE = 0, CYC_SPARSE = 1, CYC_INDICATOR = 2, CYC_INTERCEPT = 3 };

/* the model types on this path (ModelType, src/cyclops/Types.h:134-147) */
enum cyc_model { CYC_LR = 0, CYC_PR = 1, CYC_CLR = 2, CYC_CPR = 3, CYC_COX = 4 };

/* PriorType, src/cyclops/Types.h:101-106 */
enum cyc_prior_type { CYC_PRIOR_NONE = 0, CYC_PRIOR_LAPLACE = 1, CYC_PRIOR_NORMAL = 2 };

/* ConvergenceType, src/cyclops/Types.h:110-116 */
enum cyc_convergence {
    CYC_CONV_GRADIENT = 0, CYC_CONV_LANGE = 1, CYC_CONV_MITTAL = 2,
    CYC_CONV_ONE_STEP = 3, CYC_CONV_ZHANG_OLES = 4
};

/* UpdateReturnFlags, src/cyclops/Types.h:124-130 */
enum cyc_return_flag {
    CYC_SUCCESS = 0, CYC_FAIL = 1, CYC_MAX_ITERATIONS = 2, CYC_ILLCONDITIONED = 3
};

enum cyc_status {
    CYC_OK = 0,
    CYC_ERR_ARGUMENT = 1,     /* bad pointer, size or enum */
    CYC_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    CYC_ERR_MEMORY = 3,       /* device allocation failed or over budget */
    CYC_ERR_UNSUPPORTED = 4,  /* path not offered for this model / format */
    CYC_ERR_STATE = 5,        /* call out of order (e.g. gradient before statistics) */
    CYC_ERR_TIMEOUT = 6       /* a device-side wait ran past its bound */
};

/* arithmetic of the device-resident solvers */
enum cyc_precision {
    CYC_FP64 = 0,             /* FP64 state and sums throughout */
    CYC_MIXED = 1             /* FP32 state + compensated sums, then an FP64 polish */
};

/* ---- data --------------------------------------------------------------- */

/* Column store in the reference's ingest order (src/RcppModelData.cpp:751-900):
 * an optional fixed offset column 0, dense columns (intercept first), sparse,
 * indicator.  Rows of survival models sorted by (stratum, -time, y); rows of
 * stratified models by stratum. */
typedef struct {
    int model;                  /* cyc_model */
    int K;                      /* rows */
    int J;                      /* columns */
    const int* pid;             /* K stratum ids (renumbered by runs) or NULL */
    const double* y;            /* K outcomes */
    const double* time;         /* K survival times (cox) or offsets, or NULL */
    const int* col_format;      /* J cyc_format */
    const long long* col_ptr;   /* J+1 offsets into col_idx (SPARSE/INDICATOR) */
    const int* col_idx;         /* ascending row ids per column */
    const long long* val_ptr;   /* J+1 offsets into col_val (SPARSE: nnz, DENSE: K) */
    const double* col_val;      /* values */
    int has_offset;             /* column 0 is an offset with beta fixed at 1 */
    int has_intercept;
} cyc_data_desc;

typedef struct cyc_dataset cyc_dataset;
typedef struct cyc_engine cyc_engine;

const char* cyc_last_error(void);
/* ABI revision: 3 since cyc_run_stats gained batch_cap, batch_shared_rows
 * and batch_levels (2: cyc_control gained use_kkt_swindle, cyc_fit_spec
 * fixed / n_fixed, cyc_run_stats cluster_ctas); fields are appended:
 * zero-initialise these structs, e.g. `cyc_fit_spec s = {0};`. */
#define CYC_ABI_VERSION 3
int cyc_version(void);

/* Copy a dataset to device `device`.  Replaces the host-side ModelData the
 * engine reads by const reference (src/cyclops/engine/ModelSpecifics.h:121-122). */
int cyc_dataset_create(const cyc_data_desc* desc, int device, cyc_dataset** out);
int cyc_dataset_destroy(cyc_dataset* ds);
/* rows, columns, stored indices, device bytes held */
int cyc_dataset_info(const cyc_dataset* ds, int* K, int* J, long long* nnz, size_t* device_bytes);

/* ---- engine: the AbstractModelSpecifics surface ------------------------- */

/* AbstractModelSpecifics::factory + initialize(N,K,J,...)
 * (AbstractModelSpecifics.cpp:128-154, ModelSpecifics.hpp:1899-1952) */
int cyc_engine_create(cyc_dataset* ds, cyc_engine** out);
int cyc_engine_destroy(cyc_engine* e);
/* clone() (ModelSpecifics.hpp:98-101): shares the dataset, own state + stream */
int cyc_engine_clone(const cyc_engine* e, cyc_engine** out);
/* setWeights(double*, double*, bool) (ModelSpecifics.hpp:427-484) */
int cyc_engine_set_weights(cyc_engine* e, const double* weights, int use_cv);
/* computeFixedTermsInLogLikelihood (ModelSpecifics.hpp:570-587) */
int cyc_engine_compute_fixed_terms_ll(cyc_engine* e, int use_cv);
/* computeFixedTermsInGradientAndHessian (ModelSpecifics.hpp:589-603) */
int cyc_engine_compute_fixed_terms_gh(cyc_engine* e, int use_cv);
/* zeroXBeta / axpyXBeta / computeXBeta (ModelSpecifics.hpp:296-423) */
int cyc_engine_zero_xbeta(cyc_engine* e);
int cyc_engine_axpy_xbeta(cyc_engine* e, double beta, int j);
int cyc_engine_compute_xbeta(cyc_engine* e, const double* beta, int use_w);
/* computeRemainingStatistics (ModelSpecifics.hpp:1588-1633) */
int cyc_engine_compute_remaining_statistics(cyc_engine* e, int use_w);
/* computeNumeratorForGradient (ModelSpecifics.hpp:1353-1427) */
int cyc_engine_compute_numerator_for_gradient(cyc_engine* e, int j, int use_w);
/* computeGradientAndHessian (ModelSpecifics.hpp:711-766, 891-1201) */
int cyc_engine_compute_gradient_and_hessian(cyc_engine* e, int j, double* gradient,
                                            double* hessian, int use_w);
/* updateXBeta (ModelSpecifics.hpp:1466-1586) */
int cyc_engine_update_xbeta(cyc_engine* e, double delta, int j, int use_w);
/* getLogLikelihood (ModelSpecifics.hpp:605-650) */
int cyc_engine_get_log_likelihood(cyc_engine* e, int use_cv, double* out);
/* getGradientObjective (ModelSpecifics.hpp:103-120) */
int cyc_engine_get_gradient_objective(cyc_engine* e, int use_cv, double* out);
/* getPredictiveLogLikelihood (ModelSpecifics.hpp:652-690) */
int cyc_engine_get_predictive_log_likelihood(cyc_engine* e, const double* weights, double* out);
/* getPredictiveEstimates (ModelSpecifics.hpp:692-707) */
int cyc_engine_get_predictive_estimates(cyc_engine* e, double* y, const double* weights);
/* getXBeta / saveXBeta / getXBetaSave (ModelSpecifics.hpp:286-308); K doubles */
int cyc_engine_get_xbeta(cyc_engine* e, double* out);
int cyc_engine_save_xbeta(cyc_engine* e);
int cyc_engine_get_xbeta_save(cyc_engine* e, double* out);
/* computeFisherInformation (ModelSpecifics.hpp:1203-1351) for every pair of
 * `columns` at the engine's current coefficients, as
 * CyclicCoordinateDescent::computeFisherInformation
 * (CyclicCoordinateDescent.cpp:1288-1300) assembles it: `out` is the n x n
 * symmetric matrix, row-major.  lr, pr, clr, cpr; unweighted (use_cv != 0 is
 * CYC_ERR_UNSUPPORTED, as the reference throws, :1207-1209). */
int cyc_engine_fisher_information(cyc_engine* e, const int* columns, int n, int use_cv, double* out);
/* number of denominators N (patients / strata / risk-set groups) */
int cyc_engine_get_n(const cyc_engine* e, int* n);

/* ---- device-resident solvers -------------------------------------------- */

/* ModeFindingArguments (src/cyclops/CcdInterface.h:70-94) */
typedef struct {
    double tolerance;           /* default 1e-6 */
    int max_iterations;         /* default 1000 */
    int convergence_type;       /* cyc_convergence, default GRADIENT */
    double initial_bound;       /* default 2.0 */
    int max_bound_count;        /* default 5 */
    int precision;              /* cyc_precision */
    double polish_tolerance;    /* CYC_MIXED: FP32 phase stops at this tolerance */
    int use_kkt_swindle;        /* useKktSwindle (CcdInterface.h:77): the active-set
                                   passes of CyclicCoordinateDescent::kktSwindle
                                   (CyclicCoordinateDescent.cpp:636-814) under a
                                   Laplace prior.  Every fit keeps its own
                                   active set, so cyc_batch_fit and the CV
                                   grids run such fits one by one as cyc_fit;
                                   cyc_cv_auto_search returns
                                   CYC_ERR_UNSUPPORTED */
} cyc_control;

/* the prior: one default prior for every column, a flat prior on `exclude`
 * (MixtureJointPrior, src/cyclops/priors/JointPrior.h:81-160) */
typedef struct {
    int prior_type;             /* cyc_prior_type */
    const int* exclude;         /* column ids with a flat prior (the intercept) */
    int n_exclude;
} cyc_prior;

/* one fit of a batch: its row weights (0/1 CV mask or any nonnegative weights,
 * NULL = unweighted), its prior variance and optional warm start */
typedef struct {
    const double* weights;      /* K, or NULL */
    double variance;            /* prior variance (Laplace lambda = sqrt(2/variance)) */
    const double* start_beta;   /* J, or NULL (zeros; offset column 1) */
    const int* fixed;           /* columns held at their start value (fitCyclopsModel's
                                   fixedCoefficients, R/ModelFit.R:205-214 ->
                                   setFixedBeta), or NULL; the fits of one batched
                                   solve share one set */
    int n_fixed;
} cyc_fit_spec;

typedef struct {
    double* beta;               /* J, caller-owned output */
    double log_likelihood;
    double log_prior;
    int iterations;             /* cycles of the final bound */
    int return_flag;            /* cyc_return_flag */
} cyc_fit_result;

/* One fit with the CCD loop on the GPU, whole-GPU kernels per coordinate and
 * no host round trip inside a cycle (CyclicCoordinateDescent::update,
 * src/cyclops/CyclicCoordinateDescent.cpp:586-615). */
int cyc_fit(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
            const cyc_control* control, cyc_fit_result* out);

/* F fits sharing `ds`, advanced together coordinate by coordinate in one
 * persistent kernel (lr, pr, clr, cpr).  Results in `out[0..F)`.  Cox fits
 * (each with its own risk sets under its weights) and fits under
 * use_kkt_swindle (each with its own active set) run instead as concurrent
 * cyc_fit solves, up to CYC_CONCURRENT_FITS (default 8) at a time on their
 * own streams; each result is the one cyc_fit gives alone.  Run statistics
 * then sum the fits' counts, with kernel_ms the whole section's time. */
int cyc_batch_fit(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* specs, int F,
                  const cyc_control* control, cyc_fit_result* out);

/* Cross-validation grid on the GPU: `n_folds` folds x `n_var` prior
 * variances = n_folds * n_var fits (fit i = variance i / n_folds, fold
 * i % n_folds), each trained on the rows whose fold id differs from its fold
 * (fold_of_row: K ids in 0..n_folds-1, e.g. from cyc_cv_fold_weights) and
 * scored on the held-out rows with the reference's predictive log likelihood
 * (ModelSpecifics.hpp:652-690).  The per-fold, per-grid-point loop of
 * GridSearchCrossValidationDriver / AbstractCrossValidationDriver
 * (src/cyclops/drivers/GridSearchCrossValidationDriver.cpp:96-140,
 * AbstractCrossValidationDriver.cpp:131-261) as one batched solve (cox,
 * and use_kkt_swindle: as cyc_cv_grid_fit_weighted with unit weights).
 * `pred_loglik` (F values, NaN where the fit did not converge) and
 * `grid_mean` (n_var values: mean over folds ignoring NaN) may be NULL. */
int cyc_cv_grid_fit(cyc_dataset* ds, const cyc_prior* prior, const int* fold_of_row, int n_folds,
                    const double* variances, int n_var, const cyc_control* control,
                    cyc_fit_result* out, double* pred_loglik, double* grid_mean);

/* Profile-likelihood confidence bounds (CcdInterface::profileModel with one
 * thread, src/cyclops/CcdInterface.cpp:262-420; R confint.cyclopsFit,
 * R/ModelFit.R:762-800): fits (as cyc_fit), then for each column of
 * `columns` finds where the profile log likelihood (plus the log prior when
 * include_penalty) has dropped by `threshold` (qchisq(level, 1) / 2) above
 * (`upper[i]`) and below (`lower[i]`) the estimate, NaN where no bracket was
 * found; `evaluations[i]` counts the refits of both.  Each refit holds the
 * column fixed and warm-starts from the previous refit's state
 * (OptimizationProfile, :223-260); the bracket grows as RZeroIn's
 * bracketSignChange and the root is Brent's zeroin at tolerance 1e-3
 * (src/utils/RZeroIn.h).  A column with a prior is rejected unless
 * override_no_regularization; the offset column is rejected.  `fit` (may
 * be NULL) receives the fit before profiling. */
int cyc_profile_bounds(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                       const cyc_control* control, const int* columns, int n, double threshold,
                       int include_penalty, int override_no_regularization, double* lower, double* upper,
                       int* evaluations, cyc_fit_result* fit);

/* The profile log likelihood (plus the log prior when include_penalty) of
 * `column` at `points` (CcdInterface::evaluateProfileModel with one thread,
 * src/cyclops/CcdInterface.cpp:527-618; R getCyclopsProfileLogLikelihood,
 * R/ModelFit.R:816-826): fits (as cyc_fit), then refits with the column
 * held at each point in turn, each refit warm-started from the last. */
int cyc_profile_log_likelihood(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                               const cyc_control* control, int column, const double* points, int n,
                               int include_penalty, double* values);

/* The same values as one batched solve (lr, pr, clr, cpr): every point is a
 * fit of the persistent batch kernel with `column` held at the point, all
 * started from the mode (spec->start_beta, or fitted first when NULL), as
 * evaluateProfileModel's per-thread clones start from it
 * (CcdInterface.cpp:545-598).  Values agree with the one-thread order to
 * the fits' convergence tolerance. */
int cyc_profile_log_likelihood_batch(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                                     const cyc_control* control, int column, const double* points, int n,
                                     int include_penalty, double* values);

/* cyc_cv_grid_fit with observation weights (the fit's weights handed to
 * the CV selector, CrossValidationSelector.cpp:72-124): fit (variance v,
 * fold f) trains on the rows outside fold f at their weights and is scored
 * on fold f's rows at their weights (getComplement).  Fits as
 * cyc_batch_fit (cox and use_kkt_swindle: concurrent cyc_fit solves); cold
 * starts; outputs as cyc_cv_grid_fit. */
int cyc_cv_grid_fit_weighted(cyc_dataset* ds, const cyc_prior* prior, const int* fold_of_row, int n_folds,
                             const double* row_weights, const double* variances, int n_var,
                             const cyc_control* control, cyc_fit_result* out, double* pred_loglik,
                             double* grid_mean);

/* Auto-search cross-validation (createControl(cvType = "auto"), R's
 * default: AutoSearchCrossValidationDriver, src/cyclops/drivers/
 * AutoSearchCrossValidationDriver.cpp:63-160, with the UniModalSearch of
 * src/utils/HParSearch.cpp).  From `starting_variance` (<= 0: the
 * normal-based default, ModelData.cpp:716-720) each step refits every fold
 * of every repetition at one variance (one batched solve per repetition,
 * cold starts: the reference's resetCoefficients), takes the mean and
 * standard deviation of the held-out predictive log likelihoods (NaN folds
 * left out) and lets the search propose the next variance; at most 50
 * steps.  fold_of_row: n_reps x K fold ids (e.g. from cyc_cv_fold_weights);
 * row_weights: K observation weights (NULL: all 1), used as
 * cyc_cv_grid_fit_weighted uses them; cox folds and use_kkt_swindle folds
 * run as concurrent cyc_fit solves.
 * Returns the variance the search settles on and its expected value, and
 * the first max_tried points tried (variance, mean, stdev; *n_tried counts
 * all). */
int cyc_cv_auto_search(cyc_dataset* ds, const cyc_prior* prior, const int* fold_of_row, int n_folds, int n_reps,
                       const double* row_weights, double starting_variance, const cyc_control* control,
                       double* best_variance,
                       double* best_value, double* tried_variance, double* tried_mean, double* tried_sd,
                       int max_tried, int* n_tried);

/* Cross-validation fold masks, `n_reps * folds` rows of K weights (0 = held
 * out), exactly as CrossValidationSelector draws them
 * (src/cyclops/drivers/CrossValidationSelector.cpp:21-116): by row
 * (`by_row` = 1) or by stratum id `ids` (0..S-1); seed -1 = no shuffle. */
int cyc_cv_fold_weights(int K, const int* ids, int folds, long seed, int by_row, int n_reps,
                        double* out);

/* Bootstrap replicate weights, `n_replicates` rows of K weights, exactly as
 * BootstrapSelector draws them for BootstrapDriver
 * (src/cyclops/drivers/BootstrapSelector.cpp:15-88,
 * src/cyclops/drivers/BootstrapDriver.cpp:47-64): units are the ids
 * 0..N-1 (`ids` K per-row unit ids, NULL = one unit per row); each replicate
 * draws as many units with replacement from the units whose `unit_exclude`
 * weight is 0 (NULL = all), and weights row k by the draws of its unit.
 * Seed -1 = the engine's default state.  Feed the rows to cyc_batch_fit as
 * per-fit weights. */
int cyc_bootstrap_weights(int K, const int* ids, int n_replicates, long seed, const double* unit_exclude,
                          double* out);

/* Device ingest of a long covariate table (rowId, covariateId,
 * covariateValue): the covariate half of convertToCyclopsData
 * (R/NewDataConversion.R:131-176) and ModelData::loadMultipleX
 * (src/cyclops/ModelData.cpp:148-243) on the GPU.  `outcome_row_id` holds
 * the K outcome rowIds already in the reference's row order (the outcome
 * sort is the caller's: by rowId; stratum, rowId; or stratum, time
 * descending, y, rowId); a covariate row takes the position of the last
 * outcome row with its rowId and is dropped when there is none.  Entries
 * are ordered by (covariateId, position) -- for every model the reference's
 * covariate order when a covariate's stratum is its outcome's -- and each
 * covariateId run becomes a column: INDICATOR unless a value is neither 0
 * nor 1 (then SPARSE), zero values not stored, all entries stored when
 * `value` is NULL; a repeated (row, covariate) fails with
 * "Repeated row-column entry at <rowId> - <covariateId>".  The result stays
 * on the device until copied: cyc_ingest_sizes gives the column count and
 * the row-id and value counts, cyc_ingest_copy fills caller buffers (formats
 * J, col_ptr J+1 and val_ptr J+1 offsets, row positions, values, the
 * columns' covariateIds), cyc_ingest_free releases it.  Offset and intercept
 * columns are the caller's to prepend. */
typedef struct cyc_ingest cyc_ingest;
int cyc_ingest_covariates(int device, long long n, const long long* covariate_id, const long long* row_id,
                          const double* value, int K, const long long* outcome_row_id, cyc_ingest** out);
int cyc_ingest_sizes(const cyc_ingest* h, int* n_columns, long long* n_idx, long long* n_val);
int cyc_ingest_copy(const cyc_ingest* h, int* col_format, long long* col_ptr, int* col_idx, long long* val_ptr,
                    double* col_val, long long* labels);
void cyc_ingest_free(cyc_ingest* h);

/* Statistics of the last cyc_batch_fit / cyc_fit on this thread, for
 * roofline accounting: kernel milliseconds (CUDA events), column entries
 * visited by gradients, entries visited by updates, coordinate steps. */
typedef struct {
    double kernel_ms;           /* solver kernels, CUDA events */
    double algorithmic_bytes;   /* unique bytes the algorithm must move (all phases) */
    double gradient_entries;    /* sum over (fit, coordinate) of nnz_j */
    double update_entries;      /* sum over (fit, coordinate) with delta != 0 of nnz_j */
    double coordinate_steps;    /* (fit, coordinate) steps taken */
    double index_entries;       /* bytes of row ids / values streamed, summed over fit groups */
    double cycles;              /* sum over fits of CCD cycles */
    int launches;               /* solver kernel launches */
    int phases;                 /* 1 (FP64) or 2 (FP32, then FP64 polish) */
    double phase_ms[2];
    double phase_bytes[2];
    int phase_state_bytes[2];   /* bytes per (row, fit) state element of each phase */
    int cluster_ctas;           /* batched solves: CTAs per thread-block cluster (the
                                   tuner's choice, or CYC_BATCH_CLUSTER); 0 otherwise */
    int batch_cap;              /* batched solves of 8-fit groups (lr, pr): the batch shape the
                                   shape tuner chose (or CYC_BATCH_SHAPE): columns with at most
                                   this many entries in every CTA's rows are batched, */
    int batch_shared_rows;      /* a batch shares at most this many rows between its columns, */
    int batch_levels;           /* and replays at most this many levels; 0 otherwise */
} cyc_run_stats;
int cyc_last_run_stats(cyc_run_stats* out);

/* Kernels this library has launched in this process (all entry points). */
long long cyc_launch_count(void);

/* The plain FP64 single-fit GPU CCD: the host runs the coordinate loop and
 * reads each coordinate's (gradient, Hessian) back, as
 * CyclicCoordinateDescent does through AbstractModelSpecifics
 * (src/cyclops/CyclicCoordinateDescent.cpp:1394-1413).  The baseline the
 * device-resident solvers are measured against. */
int cyc_fit_host_loop(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                      const cyc_control* control, cyc_fit_result* out);

/* ---- allocation-free entry point ----------------------------------------- */

/* No counterpart in the reference.  For callers that cannot let this
 * library allocate device memory (they own the GPU's memory through their
 * own pool or caching allocator, or cannot afford the device-wide
 * synchronisation an allocation implies): the gradient and Hessian of one
 * lr / pr column, as cyc_engine_compute_gradient_and_hessian computes them,
 * with every buffer supplied by the caller as a device pointer and the
 * reduction scratch taken from a fixed 64 KiB area compiled into the library
 * (held on every GPU that loads it until the process exits).
 *   rows / values: the column's row ids and values as cyc_data_desc stores
 *   them (dense: K values, no rows; indicator: rows only; intercept: none);
 *   exb = exp(x beta) and, for lr, denom = 1 + exb, K doubles each;
 *   weights: K row weights or NULL (unweighted); xjy: the column's sum x*y*w;
 *   out: 2 doubles on the device receiving (gradient, Hessian);
 *   stream: a cudaStream_t (NULL = the default stream).
 * At most 4,194,304 column entries per call; larger columns are rejected.
 * Runs on the calling thread's current device; the first call on a device
 * looks up the scratch address there, so make it before any stream capture,
 * and during set-up, before the caller's own pool takes the GPU's memory:
 * with lazy module loading that lookup can load the library's device code,
 * which takes device memory.  Later calls allocate nothing.
 * Calls share the scratch: calls that overlap on the GPU race. */
int cyc_gradient_hessian_noalloc(int model, int format, long long n, const int* rows,
                                 const double* values, const double* exb, const double* denom,
                                 const double* weights, double xjy, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CYCLOPS_B200_H */
