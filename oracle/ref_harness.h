/* ref_harness.h -- TEST INFRASTRUCTURE (oracle).
 * C ABI of oracle/_ref/libcyclops_ref.so, the reference Cyclops CPU engine
 * built from its own sources.  Used only by tests/ and bench.py's CPU legs. */
#ifndef CYC_REF_HARNESS_H
#define CYC_REF_HARNESS_H

enum { REF_LR = 0, REF_PR = 1, REF_CLR = 2, REF_CPR = 3, REF_COX = 4 };
enum { REF_DENSE = 0, REF_SPARSE = 1, REF_INDICATOR = 2, REF_INTERCEPT = 3 };
enum { REF_PRIOR_NONE = 0, REF_PRIOR_LAPLACE = 1, REF_PRIOR_NORMAL = 2 };

typedef struct {
    int model;               /* REF_LR ... */
    int K;                   /* rows */
    int J;                   /* columns (incl. offset / intercept) */
    const int* pid;          /* K raw stratum ids, or NULL (one row per stratum) */
    const double* y;         /* K outcomes */
    const double* time;      /* K times / offsets, or NULL */
    const int* col_format;   /* J formats */
    const long long* col_ptr;/* J+1 offsets into col_idx (SPARSE, INDICATOR entries) */
    const int* col_idx;      /* row ids, ascending within a column */
    const long long* val_ptr;/* J+1 offsets into col_val (SPARSE: nnz, DENSE: K, else 0) */
    const double* col_val;   /* values */
    int has_offset;          /* column 0 is a fixed offset (beta = 1) */
    int has_intercept;
    int prior_type;
    double variance;
    const int* exclude;      /* column indices with a flat prior */
    int n_exclude;
    const double* weights;   /* K weights or NULL */
    const int* fixed;        /* columns held at their start (setFixedBeta), or NULL */
    int n_fixed;
} ref_problem;

typedef struct {
    double tolerance;
    int max_iterations;
    int convergence_type;    /* 0 gradient, 1 lange, 2 mittal, 3 one_step, 4 zhang_oles */
    int use_kkt_swindle;
    double initial_bound;
    int max_bound_count;
} ref_control;

typedef struct {
    double* beta;            /* J, caller-owned */
    double log_likelihood;
    double log_prior;
    int iterations;
    int return_flag;
} ref_result;

const char* ref_last_error(void);
int ref_fit(const ref_problem* p, const ref_control* c, const double* start_beta, ref_result* out);
int ref_fit_device(const ref_problem* p, const ref_control* c, const double* start_beta,
                   ref_result* out, int device);
/* The same on ModelData<float> (the reference's floatingPoint = 32 data,
 * RcppModelData.cpp:724-728): device 0 the reference's float CPU engine,
 * device 1 the CUDA engine through the adapter. */
int ref_fit_fp32(const ref_problem* p, const ref_control* c, const double* start_beta, ref_result* out,
                 int device);
int ref_engine_probe(const ref_problem* p, const double* beta, double* gradient, double* hessian,
                     double* xbeta, double* log_likelihood);
int ref_predictive_loglik(const ref_problem* p, const double* beta, const double* held_out,
                          double* out);
int ref_cv_weights(int K, const int* ids, int fold, long seed, int by_row, int n_reps, double* out);
int ref_bootstrap_weights(int K, const int* ids, int n_replicates, long seed, double* out);

/* The reference's own data loader on tables already in the reference's
 * sort order (the R layer sorts, R/NewDataConversion.R:125-176):
 * ModelData::loadY, loadX for the intercept, loadMultipleX, and for Poisson
 * models setOffsetCovariate(-1) + logTransformCovariate(0)
 * (src/cyclops/ModelData.cpp:69-145, 148-243, 246-370, 609-651). */
typedef struct {
    int model;
    long long n_outcomes;
    const long long* stratum_id;      /* n_outcomes or NULL */
    const long long* row_id;          /* n_outcomes */
    const double* y;                  /* n_outcomes */
    const double* time;               /* n_outcomes or NULL */
    long long n_covariates;
    const long long* covariate_id;    /* n_covariates */
    const long long* covariate_row;   /* n_covariates */
    const double* covariate_value;    /* n_covariates or NULL (indicators) */
    int add_intercept;
    int offset_from_time;
} ref_ingest_input;

typedef struct {
    int K, J;
    int* col_format;          /* J */
    long long* col_ptr;       /* J+1 offsets into col_idx */
    int* col_idx;
    long long* val_ptr;       /* J+1 offsets into col_val */
    double* col_val;
    long long* col_label;     /* J numerical labels */
    int* pid;                 /* K strata renumbered by runs */
    double* y;                /* K */
    double* time;             /* K, or NULL */
    int has_offset, has_intercept;
} ref_ingest_output;

int ref_ingest(const ref_ingest_input* in, ref_ingest_output* out);

/* CyclicCoordinateDescent::computeFisherInformation (src/cyclops/
 * CyclicCoordinateDescent.cpp:1288-1300) at `beta` for `n` columns; out is
 * n x n row-major.  device 1 runs it through the CUDA adapter. */
int ref_fisher(const ref_problem* p, const double* beta, const int* columns, int n, double* out, int device);
/* AbstractModelSpecifics::getPredictiveEstimates (src/cyclops/engine/
 * ModelSpecifics.hpp:693-707) at `beta`: y[k] for rows with nonzero weight
 * (all rows when weights is NULL); other entries of y are left as given. */
int ref_predictive_estimates(const ref_problem* p, const double* beta, const double* weights, double* y);
void ref_ingest_free(ref_ingest_output* out);
/* Profile-likelihood bounds (CcdInterface::profileModel, src/cyclops/
 * CcdInterface.cpp:262-420, one thread): fit, then for each column its upper
 * and lower bound where the profile log likelihood drops by `threshold`
 * (NaN when the bracket fails); evaluations[i] counts the refits of both.
 * fit (may be NULL) receives the fit before profiling. */
int ref_profile(const ref_problem* p, const ref_control* c, const double* start_beta, const int* columns, int n,
                double threshold, int include_penalty, int override_no_regularization, double* lower,
                double* upper, int* evaluations, ref_result* fit, int device);
/* The profile log likelihood (plus log prior when include_penalty) at
 * `points` for one column (CcdInterface::evaluateProfileModel, src/cyclops/
 * CcdInterface.cpp:527-618, one thread): fit, makeDirty, one refit at 0,
 * then one refit per point, each warm-started from the last. */
int ref_profile_points(const ref_problem* p, const ref_control* c, const double* start_beta, int column,
                       const double* points, int n, int include_penalty, double* values, int device);
/* Auto-search cross-validation (AutoSearchCrossValidationDriver,
 * src/cyclops/drivers/AutoSearchCrossValidationDriver.cpp:63-160, with the
 * UniModalSearch of src/utils/HParSearch.cpp) as CcdInterface::runCrossValidation
 * runs it with one thread: `fold`-fold CV repeated n_reps times, selector by
 * row or by stratum, seed, starting variance (<= 0: the normal-based
 * default), cold starts when reset_coefficients.  Returns the chosen
 * variance and its predicted value, and the points tried (variance, mean
 * and stdev of the held-out predictive log likelihood; from the driver's
 * log, 6 significant digits). */
int ref_cv_auto(const ref_problem* p, const ref_control* c, int fold, int n_reps, long seed, int by_row,
                double starting_variance, int reset_coefficients, double* best_variance, double* best_value,
                double* tried_variance, double* tried_mean, double* tried_sd, int max_tried, int* n_tried);
/* Grid-search cross-validation (GridSearchCrossValidationDriver,
 * src/cyclops/drivers/GridSearchCrossValidationDriver.cpp:79-103) as
 * CcdInterface::runCrossValidation runs it with one thread: grid_steps
 * variances log-spaced over [lower, upper]; the problem's weights, when
 * given, become the selector's original weights.  points / values: the grid
 * and its mean held-out predictive log likelihood; fold_pred: grid_steps x
 * fold per-fold values from the driver's log (6 significant digits). */
int ref_cv_grid(const ref_problem* p, const ref_control* c, int fold, long seed, int by_row, double lower,
                double upper, int grid_steps, int reset_coefficients, double* points, double* values,
                double* fold_pred);
#endif
