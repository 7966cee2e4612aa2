// solver_common.cuh -- the coordinate step shared by the device-resident
// solvers: prior step, trust region and prior log density.
#pragma once
#include "internal.cuh"

namespace cyc {

struct StepState {
    double* beta;                    // J
    double* hdelta;                  // J trust-region half widths
    double* delta;                   // out: the last step
    const int* prior_type;           // J (flat prior on excluded columns)
    double variance;
    unsigned long long* n_updates;   // steps with delta != 0
    unsigned* col_updates;           // J: steps with delta != 0 per column (null: not counted)
};

__host__ __device__ inline int sgn(double x) { return x == 0 ? 0 : (x < 0 ? -1 : 1); }

// std::max(a, b) semantics: returns a unless a < b (NaN in a propagates)
__host__ __device__ inline double std_max(double a, double b) { return (a < b) ? b : a; }

// getDelta: NoPrior (src/cyclops/priors/CovariatePrior.h:186-188),
// LaplacePrior (:240-273, lambda = sqrt(2/variance), :282-292),
// NormalPrior (:410-415)
// ... with the Laplace rate lambda = sqrt(2 / variance) given by the caller
__host__ __device__ inline double prior_delta_rate(int type, double variance, double lambda, double beta, double g,
                                                   double h) {
    if (type == CYC_PRIOR_NONE) return -(g / h);
    if (type == CYC_PRIOR_NORMAL) return -(g + (beta / variance)) / (h + (1.0 / variance));
    const double neg = -(g - lambda) / h;
    const double pos = -(g + lambda) / h;
    const int s = sgn(beta);
    double delta;
    if (s == 0) {
        if (neg < 0) delta = neg;
        else if (pos > 0) delta = pos;
        else delta = 0;
    } else {
        delta = s < 0 ? neg : pos;
        if (sgn(beta + delta) != s) delta = -beta;
    }
    return delta;
}

__host__ __device__ inline double prior_delta(int type, double variance, double beta, double g, double h) {
    return prior_delta_rate(type, variance, type == CYC_PRIOR_LAPLACE ? sqrt(2.0 / variance) : 0.0, beta, g, h);
}

// applyBounds (src/cyclops/CyclicCoordinateDescent.cpp:1503-1520)
__host__ __device__ inline double apply_bounds(double* hd, double delta) {
    const double b = *hd;
    if (delta < -b) delta = -b;
    else if (delta > b) delta = b;
    double m = std_max(fabs(delta) * 2, b / 2);
    m = std_max(m, 1E-3);
    *hd = m;
    return delta;
}

// logDensity (CovariatePrior.h:221-225, :404-408); the reference's PI macro
// (CovariatePrior.h:20) rounds to the same double as M_PI
__host__ __device__ inline double log_density(int type, double variance, double x) {
    if (type == CYC_PRIOR_LAPLACE) {
        const double lambda = sqrt(2.0 / variance);
        return log(0.5 * lambda) - lambda * fabs(x);
    }
    if (type == CYC_PRIOR_NORMAL) {
        return -0.5 * log(2.0 * 3.14159265358979323846 * variance) - 0.5 * x * x / variance;
    }
    return 0.0;
}

}  // namespace cyc
