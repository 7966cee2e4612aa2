/* ccd_oracle.h -- TEST INFRASTRUCTURE (oracle).
 * Plain-C restatement of the Cyclops CCD inner loop (see ccd_oracle.c).
 * The problem/control/result structs share their layout with
 * oracle/ref_harness.h so one description drives both oracles. */
#ifndef CCD_ORACLE_H
#define CCD_ORACLE_H
#include "ref_harness.h"

typedef ref_problem ccd_problem;
typedef ref_control ccd_control;
typedef ref_result ccd_result;

const char* ccd_oracle_last_error(void);
int ccd_oracle_fit(const ccd_problem* p, const ccd_control* c, const double* start_beta,
                   ccd_result* out);
int ccd_oracle_probe(const ccd_problem* p, const double* beta, double* gradient, double* hessian,
                     double* xbeta, double* log_likelihood);
int ccd_oracle_profile(const ccd_problem* p, const ccd_control* c, const double* start_beta, const int* columns,
                       int n, double threshold, int include_penalty, int override_no_regularization,
                       double* lower, double* upper, int* evaluations, ccd_result* fit);
int ccd_oracle_profile_points(const ccd_problem* p, const ccd_control* c, const double* start_beta, int column,
                              const double* points, int n, int include_penalty, double* values);
int ccd_oracle_predictive_loglik(const ccd_problem* p, const double* beta, const double* held_out,
                                 double* out);
#endif
