/* ccd_oracle.c -- TEST INFRASTRUCTURE (oracle), not product code.
 *
 * A plain-C restatement of the Cyclops cyclic-coordinate-descent inner loop
 * for logistic (lr), Poisson (pr), conditional logistic (clr), conditional
 * Poisson (cpr) and Breslow-tied Cox (cox) regression, with flat, Laplace
 * and normal priors.  Only tests/ and bench.py's CPU legs call it; it is the
 * independent CPU checker for the CUDA engine and is itself pinned against
 * the reference engine compiled from its own sources (oracle/_ref) and the
 * golden fixtures in tests/golden.
 *
 * Every step cites the reference (paths relative to the Cyclops project):
 *   CCD driver        src/cyclops/CyclicCoordinateDescent.cpp
 *   engine            src/cyclops/engine/ModelSpecifics.hpp
 *   model traits      src/cyclops/engine/ModelSpecifics.h
 *   priors            src/cyclops/priors/CovariatePrior.h
 */
#include "ccd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_err[256];
const char* ccd_oracle_last_error(void) { return g_err; }

#define FAIL(...) do { snprintf(g_err, sizeof g_err, __VA_ARGS__); goto fail; } while (0)

enum { CONV_GRADIENT = 0, CONV_LANGE, CONV_MITTAL, CONV_ONE_STEP, CONV_ZHANG_OLES };
enum { FLAG_SUCCESS = 0, FLAG_FAIL, FLAG_MAX_ITERATIONS, FLAG_ILLCONDITIONED };

typedef struct {
    const ccd_problem* p;
    int K, J, N;              /* rows, columns, denominators */
    int model;
    int grouped;              /* clr / cpr: GroupedData (ModelSpecifics.h:329-342) */
    int cumulative;           /* cox: SortedPid (ModelSpecifics.h:406-410) */
    int use_w;                /* useCrossValidation */
    int* strat;               /* K renumbered strata */
    int* group;               /* K denominator index of each row */
    int* acc_reset;           /* cox reset points (stratum starts, then N) */
    int n_reset;
    double* kw;               /* K row weights */
    double* nw;               /* N+1 events per denominator */
    double* xb;               /* K */
    double* xb_save;          /* K (zhang-oles) */
    double* exb;              /* K */
    double* denom;            /* N+1 */
    double* acc_denom;        /* N+1 */
    double* numer;            /* N+1 */
    double* numer2;           /* N+1 */
    double* xjy;              /* J */
    double ll_fixed;
    double* beta;             /* J */
    double* hdelta;           /* J */
    int* fixb;                /* J */
    /* per-column unique denominator lists for cox (setupSparseIndices) */
    int** col_groups;
    int* col_ngroups;
} Ctx;

/* ---- model traits (ModelSpecifics.h) -------------------------------- */

static double denom_null(int model) { return model == REF_LR ? 1.0 : 0.0; } /* :980, :1490 */
static double obs_count(int model, double y) {                              /* :982, :1492, :816 */
    return (model == REF_LR || model == REF_PR) ? 1.0 : y;
}
static int has_fixed_ll(int model) { return model == REF_PR || model == REF_CPR; } /* :1488, :720 */
static double fixed_ll(double y) {                                           /* :1596-1601 */
    double s = 0.0;
    for (int i = 2; i <= (int)y; ++i) s -= log((double)i);
    return s;
}
static double ll_numer(int model, double y, double xb) {                    /* :443-445, :473-475 */
    int yi = (int)y;
    if (model == REF_COX) return yi != 1 ? 0.0 : xb;
    return yi * xb;
}
static double ll_denom(int model, double n, double d) {                     /* :998, :1579, :863 */
    return model == REF_PR ? n * d : n * log(d);
}

/* ---- column access ----------------------------------------------------- */

static int col_fmt(const Ctx* c, int j) { return c->p->col_format[j]; }
static long long col_len(const Ctx* c, int j) {
    int f = col_fmt(c, j);
    if (f == REF_DENSE || f == REF_INTERCEPT) return c->K;
    return c->p->col_ptr[j + 1] - c->p->col_ptr[j];
}
static int col_row(const Ctx* c, int j, long long e) {
    int f = col_fmt(c, j);
    if (f == REF_DENSE || f == REF_INTERCEPT) return (int)e;
    return c->p->col_idx[c->p->col_ptr[j] + e];
}
static double col_val(const Ctx* c, int j, long long e) {
    int f = col_fmt(c, j);
    if (f == REF_INDICATOR || f == REF_INTERCEPT) return 1.0;
    return c->p->col_val[c->p->val_ptr[j] + e];
}
static int is_indicator(const Ctx* c, int j) {       /* Iterators.h:39, :399 */
    int f = col_fmt(c, j);
    return f == REF_INDICATOR || f == REF_INTERCEPT;
}

/* ---- set-up ------------------------------------------------------------- */

static int cmp_int(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* setupSparseIndices (ModelSpecifics.hpp:1870-1892): sorted unique groups < max */
static void setup_sparse_indices(Ctx* c, int max) {
    for (int j = 0; j < c->J; ++j) {
        free(c->col_groups[j]);
        c->col_groups[j] = NULL;
        c->col_ngroups[j] = -1; /* dense / intercept: no list */
        int f = col_fmt(c, j);
        if (f == REF_DENSE || f == REF_INTERCEPT) continue;
        long long n = col_len(c, j);
        int* g = (int*)malloc(sizeof(int) * (n > 0 ? n : 1));
        int m = 0;
        for (long long e = 0; e < n; ++e) {
            int i = c->group[col_row(c, j, e)];
            if (i < max) g[m++] = i;
        }
        qsort(g, m, sizeof(int), cmp_int);
        int u = 0;
        for (int a = 0; a < m; ++a)
            if (u == 0 || g[u - 1] != g[a]) g[u++] = g[a];
        c->col_groups[j] = g;
        c->col_ngroups[j] = u;
    }
}

/* setPidForAccumulation (ModelSpecifics.hpp:1809-1868): Breslow risk-set
 * groups; ties among consecutive events share a group; a stratum change
 * starts a group and a reset; zero-weight rows go to the sentinel N. */
static void set_pid_for_accumulation(Ctx* c, const double* w) {
    const int K = c->K;
    const double* t = c->p->time;
    const double* y = c->p->y;
    int* g = c->group;
    for (int k = 0; k < K; ++k) g[k] = c->strat[k];
    c->n_reset = 0;
    const int ignore = -1;
    int index = 0;
    while (w != NULL && index < K && w[index] == 0.0) { g[index] = ignore; index++; }
    int last_pid = g[index];
    double last_time = t[index];
    double last_event = y[index];
    int pid = g[index] = 0;
    for (int k = index + 1; k < K; ++k) {
        if (w == NULL || w[k] != 0.0) {
            int next = g[k];
            if (next != last_pid) {
                pid++;
                c->acc_reset[c->n_reset++] = pid;
                last_pid = next;
            } else if (last_event == 1.0 && last_time == t[k] && last_event == y[k]) {
                /* tie: same denominator */
            } else {
                pid++;
            }
            last_time = t[k];
            last_event = y[k];
            g[k] = pid;
        } else {
            g[k] = ignore;
        }
    }
    pid++;
    c->acc_reset[c->n_reset++] = pid;
    c->N = pid;
    if (w != NULL)
        for (int k = 0; k < K; ++k)
            if (g[k] == ignore) g[k] = c->N;
    setup_sparse_indices(c, c->N);
}

/* setWeights (ModelSpecifics.hpp:427-484) */
static void set_weights(Ctx* c) {
    const double* w = c->use_w ? c->p->weights : NULL;
    for (int k = 0; k < c->K; ++k) c->kw[k] = w ? w[k] : 1.0;
    if (c->cumulative) set_pid_for_accumulation(c, w);
    for (int i = 0; i <= c->N; ++i) c->nw[i] = 0.0;
    for (int k = 0; k < c->K; ++k) c->nw[c->group[k]] += obs_count(c->model, c->p->y[k]) * c->kw[k];
}

/* computeFixedTermsInLogLikelihood (ModelSpecifics.hpp:570-587) */
static void fixed_terms_ll(Ctx* c) {
    c->ll_fixed = 0.0;
    if (!has_fixed_ll(c->model)) return;
    for (int k = 0; k < c->K; ++k)
        c->ll_fixed += c->use_w ? fixed_ll(c->p->y[k]) * c->kw[k] : fixed_ll(c->p->y[k]);
}

/* computeXjY (ModelSpecifics.hpp:486-524) */
static void compute_xjy(Ctx* c) {
    for (int j = 0; j < c->J; ++j) {
        double s = 0.0;
        long long n = col_len(c, j);
        for (long long e = 0; e < n; ++e) {
            int k = col_row(c, j, e);
            double yk = c->p->y[k];
            if (c->model == REF_COX) yk = obs_count(c->model, yk);
            s += c->use_w ? col_val(c, j, e) * yk * c->kw[k] : col_val(c, j, e) * yk;
        }
        c->xjy[j] = s;
    }
}

/* computeXBeta via zeroXBeta + axpyXBeta (CyclicCoordinateDescent.cpp:1452-1470,
 * ModelSpecifics.hpp:384-423) */
static void compute_xbeta(Ctx* c) {
    memset(c->xb, 0, sizeof(double) * c->K);
    for (int j = 0; j < c->J; ++j) {
        double b = c->beta[j];
        if (b == 0.0) continue;
        long long n = col_len(c, j);
        for (long long e = 0; e < n; ++e) c->xb[col_row(c, j, e)] += b * col_val(c, j, e);
    }
}

/* computeAccumlatedDenominator (ModelSpecifics.hpp:1670-1694) */
static void accumulate_denominator(Ctx* c) {
    if (!c->cumulative) return;
    double total = 0.0;
    int r = 0;
    for (int i = 0; i < c->N; ++i) {
        if (c->acc_reset[r] == i) { total = 0.0; ++r; }
        total += c->denom[i];
        c->acc_denom[i] = total;
    }
}

/* computeRemainingStatistics (ModelSpecifics.hpp:1588-1612) */
static void remaining_statistics(Ctx* c) {
    for (int i = 0; i < c->N; ++i) c->denom[i] = denom_null(c->model);
    c->denom[c->N] = denom_null(c->model);
    for (int k = 0; k < c->K; ++k) {
        c->exb[k] = exp(c->xb[k]);
        double v = c->exb[k];
        if (c->cumulative && c->use_w) v *= c->kw[k];
        c->denom[c->group[k]] += v;
    }
    accumulate_denominator(c);
}

/* computeNumeratorForGradient (ModelSpecifics.hpp:1353-1464), cox only */
static void numerator_for_gradient(Ctx* c, int j) {
    if (!c->cumulative) return;
    int ind = is_indicator(c, j);
    if (c->col_ngroups[j] >= 0) {
        for (int a = 0; a < c->col_ngroups[j]; ++a) {
            c->numer[c->col_groups[j][a]] = 0.0;
            if (!ind) c->numer2[c->col_groups[j][a]] = 0.0;
        }
    } else {
        memset(c->numer, 0, sizeof(double) * c->N);
        memset(c->numer2, 0, sizeof(double) * c->N);
    }
    long long n = col_len(c, j);
    for (long long e = 0; e < n; ++e) {
        int k = col_row(c, j, e);
        double x = col_val(c, j, e);
        double w = c->use_w ? c->kw[k] : 1.0;
        c->numer[c->group[k]] += w * (c->exb[k] * x);
        if (!ind) c->numer2[c->group[k]] += w * (c->exb[k] * x * x);
    }
}

/* computeGradientAndHessian[Impl] (ModelSpecifics.hpp:711-766, 891-1201) */
static void gradient_hessian(Ctx* c, int j, double* og, double* oh) {
    long long n = col_len(c, j);
    if (n == 0) { *og = 0.0; *oh = 0.0; return; }
    const int ind = is_indicator(c, j);
    const int sparse_it = (col_fmt(c, j) == REF_INDICATOR || col_fmt(c, j) == REF_SPARSE);
    double g = 0.0, h = 0.0;

    if (c->cumulative) {                                   /* :904-962 */
        int have = c->col_ngroups[j] < 0 || c->col_ngroups[j] > 0;
        if (have) {
            const int* list = c->col_groups[j];
            int len = c->col_ngroups[j] < 0 ? c->N : c->col_ngroups[j];
            int pos = 0;
            double acc = 0.0, acc2 = 0.0;
            int r = 0;
            int first = list ? list[0] : 0;
            while (c->acc_reset[r] < first) ++r;
            while (pos < len) {
                int i = list ? list[pos] : pos;
                if (c->acc_reset[r] <= i) { acc = 0.0; acc2 = 0.0; ++r; }
                acc += c->numer[i];
                acc2 += c->numer2[i];
                {
                    double t = acc / c->acc_denom[i];
                    double gg = c->nw[i] * t;
                    g += gg;
                    h += ind ? gg * (1.0 - t) : c->nw[i] * (acc2 / c->acc_denom[i] - t * t);
                }
                ++pos;
                if (sparse_it) {
                    int next = pos < len ? list[pos] : c->N;
                    for (++i; i < next; ++i) {
                        if (c->acc_reset[r] <= i) { acc = 0.0; acc2 = 0.0; ++r; }
                        double t = acc / c->acc_denom[i];
                        double gg = c->nw[i] * t;
                        g += gg;
                        h += ind ? gg * (1.0 - t) : c->nw[i] * (acc2 / c->acc_denom[i] - t * t);
                    }
                }
            }
        }
    } else if (!c->grouped) {                              /* :1022-1038 */
        for (long long e = 0; e < n; ++e) {
            int k = col_row(c, j, e);
            double x = col_val(c, j, e);
            double n1 = c->exb[k] * x;
            double n2 = ind ? 0.0 : c->exb[k] * x * x;
            double w = c->nw[k];
            if (c->model == REF_LR) {                      /* ModelSpecifics.h:540-568 */
                double gi = n1 / c->denom[k];
                g += c->use_w ? w * gi : gi;
                double hi = ind ? gi * (1.0 - gi) : (n2 / c->denom[k] - gi * gi);
                h += c->use_w ? w * hi : hi;
            } else {                                       /* ModelSpecifics.h:1508-1543 */
                g += c->use_w ? w * n1 : n1;
                h += c->use_w ? w * (ind ? n1 : n2) : (ind ? n1 : n2);
            }
        }
    } else {                                               /* :1127-1178 */
        double n1 = 0.0, n2 = 0.0;
        int key = c->strat[col_row(c, j, 0)];
        for (long long e = 0; e < n; ++e) {
            int k = col_row(c, j, e);
            double x = col_val(c, j, e);
            n1 += c->exb[k] * x;
            n2 += ind ? 0.0 : c->exb[k] * x * x;
            int last = (e == n - 1);
            int next_key = last ? -1 : c->strat[col_row(c, j, e + 1)];
            if (last || next_key != key) {                 /* ModelSpecifics.h:820-837 */
                double t = n1 / c->denom[key];
                double gg = c->nw[key] * t;
                g += gg;
                h += ind ? gg * (1.0 - t) : c->nw[key] * (n2 / c->denom[key] - t * t);
                n1 = n2 = 0.0;
                key = next_key;
            }
        }
    }
    g -= c->xjy[j];                                        /* :1181-1183 */
    *og = g;
    *oh = h;
}

/* updateXBeta[Impl] (ModelSpecifics.hpp:1466-1586) */
static void update_xbeta(Ctx* c, int j, double delta) {
    long long n = col_len(c, j);
    for (long long e = 0; e < n; ++e) {
        int k = col_row(c, j, e);
        c->xb[k] += delta * col_val(c, j, e);
        double w = (c->cumulative && c->use_w) ? c->kw[k] : 1.0;
        double old = w * c->exb[k];
        c->exb[k] = exp(c->xb[k]);
        double nw_ = w * c->exb[k];
        c->denom[c->group[k]] += nw_ - old;
    }
    accumulate_denominator(c);
}

/* getLogLikelihood (ModelSpecifics.hpp:605-650) */
static double log_likelihood(Ctx* c) {
    double ll = 0.0;
    for (int k = 0; k < c->K; ++k) {
        double v = ll_numer(c->model, c->p->y[k], c->xb[k]);
        ll += c->use_w ? v * c->kw[k] : v;
    }
    const double* d = c->cumulative ? c->acc_denom : c->denom;
    for (int i = 0; i < c->N; ++i) ll -= ll_denom(c->model, c->nw[i], d[i]);
    if (has_fixed_ll(c->model)) ll += c->ll_fixed;
    return ll;
}

/* getGradientObjective (ModelSpecifics.hpp:103-120) */
static double gradient_objective(Ctx* c) {
    double s = 0.0;
    for (int k = 0; k < c->K; ++k)
        s += c->use_w ? c->xb[k] * c->p->y[k] * c->kw[k] : c->xb[k] * c->p->y[k];
    return s;
}

/* ---- priors (CovariatePrior.h) ------------------------------------------ */

static int prior_of(const Ctx* c, int j) {
    for (int a = 0; a < c->p->n_exclude; ++a)
        if (c->p->exclude[a] == j) return REF_PRIOR_NONE;
    return c->p->prior_type;
}
static int sgn(double x) { return x == 0 ? 0 : (x < 0 ? -1 : 1); }

static double prior_delta(const Ctx* c, int j, double g, double h) {
    int type = prior_of(c, j);
    double beta = c->beta[j];
    if (type == REF_PRIOR_NONE) return -(g / h);                       /* :186-188 */
    if (type == REF_PRIOR_NORMAL) {                                    /* :410-415 */
        double s2 = c->p->variance;
        return -(g + beta / s2) / (h + 1.0 / s2);
    }
    double lambda = sqrt(2.0 / c->p->variance);                         /* :240-273 */
    double neg = -(g - lambda) / h;
    double pos = -(g + lambda) / h;
    int s = sgn(beta);
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

static double log_prior(const Ctx* c) {                                /* JointPrior.h:123-131 */
    double s = 0.0;
    for (int j = 0; j < c->J; ++j) {
        int type = prior_of(c, j);
        double x = c->beta[j];
        if (type == REF_PRIOR_LAPLACE) {
            double lambda = sqrt(2.0 / c->p->variance);
            s += log(0.5 * lambda) - lambda * fabs(x);
        } else if (type == REF_PRIOR_NORMAL) {
            double s2 = c->p->variance;
            s += -0.5 * log(2.0 * 3.14159265358979323846 * s2) - 0.5 * x * x / s2;
        }
    }
    return s;
}

static double cmax(double a, double b) { return (a < b) ? b : a; }     /* std::max semantics */

/* applyBounds (CyclicCoordinateDescent.cpp:1503-1520) */
static double apply_bounds(Ctx* c, int j, double delta) {
    if (delta < -c->hdelta[j]) delta = -c->hdelta[j];
    else if (delta > c->hdelta[j]) delta = c->hdelta[j];
    double m = cmax(fabs(delta) * 2, c->hdelta[j] / 2);
    m = cmax(m, 1E-3);
    c->hdelta[j] = m;
    return delta;
}

static double objective(Ctx* c, int conv) {                            /* :541-558 */
    if (conv == CONV_GRADIENT) return gradient_objective(c);
    if (conv == CONV_MITTAL) return log_likelihood(c);
    if (conv == CONV_LANGE) return log_likelihood(c) + log_prior(c);
    return 0.0;
}

static double zhang_oles(Ctx* c) {                                      /* :560-579 */
    double d = 0.0, r = 0.0;
    for (int k = 0; k < c->K; ++k) {
        double w = c->use_w ? c->kw[k] : 1.0;
        d += fabs(c->xb[k] - c->xb_save[k]) * w;
        r += fabs(c->xb[k]) * w;
    }
    return d / (1.0 + r);
}

/* findMode, cyclic CCD branch (CyclicCoordinateDescent.cpp:909-1216) */
static int find_mode(Ctx* c, const ccd_control* ctl, double initial_bound, int* iterations) {
    for (int j = 0; j < c->J; ++j) c->hdelta[j] = initial_bound;      /* resetBounds */
    int conv_type = ctl->convergence_type;
    double last = 0.0;
    if (conv_type < CONV_ZHANG_OLES) last = objective(c, conv_type);
    else memcpy(c->xb_save, c->xb, sizeof(double) * c->K);
    int it = 0;
    int flag = FLAG_SUCCESS;
    for (;;) {
        for (int j = 0; j < c->J; ++j) {                               /* cycle */
            if (c->fixb[j]) continue;
            double g, h;
            numerator_for_gradient(c, j);
            gradient_hessian(c, j, &g, &h);
            if (h < 0.0) { g = 0.0; h = 0.0; }                         /* ccdUpdateBeta :1407-1410 */
            double delta = prior_delta(c, j, g, h);
            delta = apply_bounds(c, j, delta);
            if (delta != 0.0) {
                c->beta[j] += delta;
                update_xbeta(c, j, delta);
            }
        }
        it++;
        /* performCheckConvergence (:839-906) */
        double conv;
        int ill = 0;
        if (conv_type < CONV_ZHANG_OLES) {
            double o = objective(c, conv_type);
            if (o != o) { conv = 0.0; ill = 1; }
            else conv = fabs(o - last) / (fabs(o) + 1.0);
            last = o;
        } else {
            conv = zhang_oles(c);
            memcpy(c->xb_save, c->xb, sizeof(double) * c->K);
        }
        if (ctl->tolerance > 0 && conv < ctl->tolerance) {
            flag = ill ? FLAG_ILLCONDITIONED : FLAG_SUCCESS;
            break;
        } else if (it == ctl->max_iterations) {
            flag = FLAG_MAX_ITERATIONS;
            break;
        }
    }
    *iterations = it;
    return flag;
}

/* kktSwindle (CyclicCoordinateDescent.cpp:636-814): the intercept and
 * columns whose prior has no KKT boundary (flat, normal) start active, the
 * Laplace columns inactive with beta 0 (zeroed through updateXBeta, as
 * setBeta does, :473-486); each pass runs findMode over the active set
 * (:617-634), stops when nothing is inactive or the fit failed, else moves
 * every inactive column whose |gradient| exceeds lambda into the active set
 * (computeKktConditions :817-837; the sorted list's violators are exactly
 * those); MAX_ITERATIONS after max_iterations passes.  An empty active set
 * skips findMode and keeps the last iteration count. */
static int kkt_swindle(Ctx* c, const ccd_control* ctl, double bound, int* iterations) {
    const int J = c->J;
    int intercept = -1;
    if (c->p->has_intercept) intercept = c->p->has_offset ? 1 : 0;
    int* excluded = (int*)malloc(sizeof(int) * J);
    int* active = (int*)malloc(sizeof(int) * J);
    int n_active = 0, n_inactive = 0;
    for (int j = 0; j < J; ++j) {
        excluded[j] = c->fixb[j];
        active[j] = !excluded[j] && (j == intercept || prior_of(c, j) != REF_PRIOR_LAPLACE);
        if (excluded[j]) continue;
        if (active[j]) ++n_active;
        else ++n_inactive;
    }
    const double lambda = sqrt(2.0 / c->p->variance);                 /* getKktBoundary, CovariatePrior.h:235-238 */
    int flag = FLAG_SUCCESS;
    for (int pass = 1;; ++pass) {
        for (int j = 0; j < J; ++j) {
            if (excluded[j] || active[j] || c->beta[j] == 0.0) continue;
            const double delta = 0.0 - c->beta[j];
            c->beta[j] += delta;
            update_xbeta(c, j, delta);
        }
        flag = FLAG_SUCCESS;
        if (n_active > 0) {
            for (int j = 0; j < J; ++j) c->fixb[j] = !active[j];
            flag = find_mode(c, ctl, bound, iterations);
        }
        if (n_inactive == 0 || flag != FLAG_SUCCESS) break;
        if (pass == ctl->max_iterations) { flag = FLAG_MAX_ITERATIONS; break; }
        int moved = 0;
        for (int j = 0; j < J; ++j) {
            if (excluded[j] || active[j]) continue;
            double g, h;
            numerator_for_gradient(c, j);
            gradient_hessian(c, j, &g, &h);
            if (!(fabs(g) <= lambda)) { active[j] = 1; ++moved; }
        }
        if (moved == 0) break;
        n_active += moved;
        n_inactive -= moved;
    }
    for (int j = 0; j < J; ++j) c->fixb[j] = excluded[j];
    free(excluded);
    free(active);
    return flag;
}

/* ---- context lifetime --------------------------------------------------- */

static void ctx_free(Ctx* c) {
    if (c->col_groups) for (int j = 0; j < c->J; ++j) free(c->col_groups[j]);
    free(c->col_groups); free(c->col_ngroups);
    free(c->strat); free(c->group); free(c->acc_reset); free(c->kw); free(c->nw);
    free(c->xb); free(c->xb_save); free(c->exb); free(c->denom); free(c->acc_denom);
    free(c->numer); free(c->numer2); free(c->xjy); free(c->beta); free(c->hdelta); free(c->fixb);
}

static int ctx_init(Ctx* c, const ccd_problem* p) {
    memset(c, 0, sizeof *c);
    c->p = p; c->K = p->K; c->J = p->J; c->model = p->model;
    if (p->K <= 0 || p->J <= 0) { snprintf(g_err, sizeof g_err, "empty problem"); return 1; }
    if (p->model < REF_LR || p->model > REF_COX) { snprintf(g_err, sizeof g_err, "Invalid model type."); return 1; }
    if (p->model == REF_COX && !p->time) { snprintf(g_err, sizeof g_err, "cox needs times"); return 1; }
    c->grouped = (p->model == REF_CLR || p->model == REF_CPR);
    c->cumulative = (p->model == REF_COX);
    c->use_w = p->weights != NULL;
    const int K = p->K, J = p->J;
    c->strat = (int*)malloc(sizeof(int) * K);
    /* pid renumbering by runs (RcppModelData.cpp:878-900) */
    if (p->pid) {
        int cur = 0, last = p->pid[0];
        for (int k = 0; k < K; ++k) {
            if (p->pid[k] != last) { ++cur; last = p->pid[k]; }
            c->strat[k] = cur;
        }
        c->N = cur + 1;
    } else {
        for (int k = 0; k < K; ++k) c->strat[k] = k;
        c->N = K;
    }
    c->group = (int*)malloc(sizeof(int) * K);
    for (int k = 0; k < K; ++k) c->group[k] = (c->grouped) ? c->strat[k] : k;
    if (!c->grouped && !c->cumulative) c->N = K;
    c->acc_reset = (int*)malloc(sizeof(int) * (K + 2));
    const int M = K + 2;
    c->kw = (double*)calloc(K, sizeof(double));
    c->nw = (double*)calloc(M, sizeof(double));
    c->xb = (double*)calloc(K, sizeof(double));
    c->xb_save = (double*)calloc(K, sizeof(double));
    c->exb = (double*)calloc(K, sizeof(double));
    c->denom = (double*)calloc(M, sizeof(double));
    c->acc_denom = (double*)calloc(M, sizeof(double));
    c->numer = (double*)calloc(M, sizeof(double));
    c->numer2 = (double*)calloc(M, sizeof(double));
    c->xjy = (double*)calloc(J, sizeof(double));
    c->beta = (double*)calloc(J, sizeof(double));
    c->hdelta = (double*)calloc(J, sizeof(double));
    c->fixb = (int*)calloc(J, sizeof(int));
    c->col_groups = (int**)calloc(J, sizeof(int*));
    c->col_ngroups = (int*)calloc(J, sizeof(int));
    if (p->has_offset) { c->beta[0] = 1.0; c->fixb[0] = 1; }           /* CCD init :218-221 */
    for (int i = 0; i < p->n_fixed; ++i) c->fixb[p->fixed[i]] = 1;     /* setFixedBeta (R/ModelFit.R:205-214) */
    if (c->cumulative) {
        set_pid_for_accumulation(c, NULL);                             /* initialize :1931-1932 */
    } else {
        setup_sparse_indices(c, c->N);
    }
    return 0;
}

static void prepare(Ctx* c) {
    set_weights(c);
    fixed_terms_ll(c);
    compute_xjy(c);
    compute_xbeta(c);
    remaining_statistics(c);
}

/* update (CyclicCoordinateDescent.cpp:586-615): restart with a smaller
 * bounding box while ill-conditioned; the swindle runs when some prior has
 * a KKT boundary (JointPrior.h:149-157) */
static int update(Ctx* c, const ccd_control* ctl, int* iters) {
    double bound = ctl->initial_bound;
    int count = 0, flag = FLAG_SUCCESS;
    const int swindle = ctl->use_kkt_swindle && c->p->prior_type == REF_PRIOR_LAPLACE;
    for (;;) {
        flag = swindle ? kkt_swindle(c, ctl, bound, iters) : find_mode(c, ctl, bound, iters);
        ++count;
        if (flag == FLAG_ILLCONDITIONED && count < ctl->max_bound_count) {
            bound /= 10.0;
            for (int j = c->p->has_offset ? 1 : 0; j < c->J; ++j) c->beta[j] = 0.0;  /* resetBeta :256-264 */
            compute_xbeta(c);
            remaining_statistics(c);
        } else {
            break;
        }
    }
    return flag;
}

int ccd_oracle_fit(const ccd_problem* p, const ccd_control* ctl, const double* start,
                   ccd_result* out) {
    Ctx c;
    if (ctx_init(&c, p)) return 1;
    if (start) for (int j = 0; j < p->J; ++j) c.beta[j] = start[j];
    prepare(&c);
    int iters = 0;
    const int flag = update(&c, ctl, &iters);
    for (int j = 0; j < p->J; ++j) out->beta[j] = c.beta[j];
    out->log_likelihood = log_likelihood(&c);
    out->log_prior = log_prior(&c);
    out->iterations = iters;
    out->return_flag = flag;
    ctx_free(&c);
    return 0;
}

/* ---- profile likelihood (CcdInterface.cpp:223-420) ----------------------- */

typedef struct {
    Ctx* c;
    const ccd_control* ctl;
    int index;
    double mode, threshold;
    int penalty;
    int evals;
} Profile;

/* OptimizationProfile::objective (CcdInterface.cpp:238-249): beta[index] set
 * to x through updateXBeta (setBeta, CyclicCoordinateDescent.cpp:473-486),
 * held fixed while update refits the rest from the current state, then the
 * log likelihood (+ log prior) + threshold - mode */
static double profile_objective(Profile* f, double x) {
    Ctx* c = f->c;
    f->evals++;
    const double delta = x - c->beta[f->index];
    c->beta[f->index] += delta;
    update_xbeta(c, f->index, delta);
    c->fixb[f->index] = 1;
    int iters = 0;
    update(c, f->ctl, &iters);
    c->fixb[f->index] = 0;
    double y = log_likelihood(c) + f->threshold - f->mode;
    if (f->penalty) y += log_prior(c);
    return y;
}

/* bracketSignChange (src/utils/RZeroIn.h): steps of 0.1, 0.2, 0.4, ... times
 * max(|x0|, 0.01) from x0 in `direction` until the objective is no longer
 * positive; NaN objective when it turns NaN or after 22 steps */
static double profile_bracket(Profile* f, double x0, double f0, double direction, double* f1) {
    const double displacement = cmax(fabs(x0), 0.01);
    double multiplier = 0.1;
    double x1 = x0, y1 = f0;
    for (int steps = 0; y1 > 0; ++steps) {
        x1 = x0 + direction * displacement * multiplier;
        y1 = profile_objective(f, x1);
        if (isnan(y1)) break;
        if (steps > 20) { y1 = NAN; break; }
        multiplier *= 2.0;
    }
    *f1 = y1;
    return x1;
}

/* Brent's root finder as Forsythe, Malcolm & Moler give it (Computer Methods
 * for Mathematical Computations, 1977, zeroin), the variant RZeroIn::getRoot
 * runs (src/utils/RZeroIn.h): f(a), f(b) of opposite signs known; each step
 * takes inverse quadratic (or secant) interpolation when it falls well inside
 * [b, c] and shrinks fast enough, else bisection; stops when half the
 * bracket is within 2 eps |b| + tol / 2, or after max_it + 1 steps. */
static double profile_root(Profile* f, double a, double b, double fa, double fb, double tol, int max_it) {
    if (b < a) {
        double t = a; a = b; b = t;
        t = fa; fa = fb; fb = t;
    }
    if (fa == 0.0) return a;
    if (fb == 0.0) return b;
    double c = a, fc = fa;
    for (int k = 0; k <= max_it; ++k) {
        const double prev_step = b - a;
        if (fabs(fc) < fabs(fb)) {                       /* b: the best point so far */
            a = b; b = c; c = a;
            fa = fb; fb = fc; fc = fa;
        }
        const double tol_act = 2 * DBL_EPSILON * fabs(b) + tol / 2;
        double step = (c - b) / 2;
        if (fabs(step) <= tol_act || fb == 0.0) return b;
        if (fabs(prev_step) >= tol_act && fabs(fa) > fabs(fb)) {
            const double cb = c - b;
            double p, q;
            if (a == c) {                                /* secant */
                const double t1 = fb / fa;
                p = cb * t1;
                q = 1.0 - t1;
            } else {                                     /* inverse quadratic */
                const double r = fa / fc, t1 = fb / fc, t2 = fb / fa;
                p = t2 * (cb * r * (r - t1) - (b - a) * (t1 - 1.0));
                q = (r - 1.0) * (t1 - 1.0) * (t2 - 1.0);
            }
            if (p > 0) q = -q;
            else p = -p;
            if (p < (0.75 * cb * q - fabs(tol_act * q) / 2) && p < fabs(prev_step * q / 2)) step = p / q;
        }
        if (fabs(step) < tol_act) step = step > 0 ? tol_act : -tol_act;
        a = b; fa = fb;
        b += step;
        fb = profile_objective(f, b);
        if ((fb > 0 && fc > 0) || (fb < 0 && fc < 0)) { c = a; fc = fa; }
    }
    return b;
}

/* evaluateProfileModel with one thread (CcdInterface.cpp:527-618): fit;
 * makeDirty (CyclicCoordinateDescent.cpp:448-452), so the first refit's
 * findMode recomputes the fixed terms, xbeta and the statistics from beta;
 * one refit at 0; then values[i] = the refit objective at points[i]
 * (threshold 0, mode 0), each refit warm-started from the last */
int ccd_oracle_profile_points(const ccd_problem* p, const ccd_control* ctl, const double* start, int column,
                              const double* points, int n, int include_penalty, double* values) {
    Ctx c;
    if (ctx_init(&c, p)) return 1;
    if (column < 0 || column >= p->J || (p->has_offset && column == 0)) {
        snprintf(g_err, sizeof g_err, "profile column %d out of range", column);
        ctx_free(&c);
        return 1;
    }
    if (start) for (int j = 0; j < p->J; ++j) c.beta[j] = start[j];
    prepare(&c);
    int iters = 0;
    update(&c, ctl, &iters);
    Profile f = {&c, ctl, column, 0.0, 0.0, include_penalty, 0};
    /* the first refit: setBeta through updateXBeta, then the dirty state is rebuilt from beta */
    const double delta = 0.0 - c.beta[column];
    c.beta[column] += delta;
    update_xbeta(&c, column, delta);
    prepare(&c);
    c.fixb[column] = 1;
    update(&c, ctl, &iters);
    c.fixb[column] = 0;
    for (int i = 0; i < n; ++i) values[i] = profile_objective(&f, points[i]);
    ctx_free(&c);
    return 0;
}

int ccd_oracle_profile(const ccd_problem* p, const ccd_control* ctl, const double* start, const int* cols, int n,
                       double threshold, int include_penalty, int override_no_regularization, double* lower,
                       double* upper, int* evaluations, ccd_result* fit) {
    Ctx c;
    if (ctx_init(&c, p)) return 1;
    for (int i = 0; i < n; ++i) {
        if (cols[i] < 0 || cols[i] >= p->J || (p->has_offset && cols[i] == 0)) {
            snprintf(g_err, sizeof g_err, "profile column %d out of range", cols[i]);
            ctx_free(&c);
            return 1;
        }
        if (!override_no_regularization && prior_of(&c, cols[i]) != REF_PRIOR_NONE) {
            snprintf(g_err, sizeof g_err, "Variable %d is regularized.", cols[i]);
            ctx_free(&c);
            return 1;
        }
    }
    if (start) for (int j = 0; j < p->J; ++j) c.beta[j] = start[j];
    prepare(&c);
    int iters = 0;
    const int flag = update(&c, ctl, &iters);
    if (fit) {
        for (int j = 0; j < p->J; ++j) fit->beta[j] = c.beta[j];
        fit->log_likelihood = log_likelihood(&c);
        fit->log_prior = log_prior(&c);
        fit->iterations = iters;
        fit->return_flag = flag;
    }
    double mode = log_likelihood(&c);
    if (include_penalty) mode += log_prior(&c);
    double* x0s = (double*)malloc(sizeof(double) * p->J);
    memcpy(x0s, c.beta, sizeof(double) * p->J);
    for (int i = 0; i < n; ++i) {              /* (column, +1) then (column, -1), one state throughout */
        int count = 0;
        for (int d = 0; d < 2; ++d) {
            const double direction = d == 0 ? 1.0 : -1.0;
            Profile f = {&c, ctl, cols[i], mode, threshold, include_penalty, 0};
            const double x0 = x0s[cols[i]];
            double f1;
            const double x1 = profile_bracket(&f, x0, threshold, direction, &f1);
            const double pt = isnan(f1) ? NAN : profile_root(&f, x0, x1, threshold, f1, 1e-3, 1000);
            (d == 0 ? upper : lower)[i] = pt;
            count += f.evals;
        }
        evaluations[i] = count;
    }
    free(x0s);
    ctx_free(&c);
    return 0;
}

int ccd_oracle_probe(const ccd_problem* p, const double* beta, double* gradient, double* hessian,
                     double* xbeta, double* loglik) {
    Ctx c;
    if (ctx_init(&c, p)) return 1;
    for (int j = 0; j < p->J; ++j) c.beta[j] = beta[j];
    prepare(&c);
    *loglik = log_likelihood(&c);
    for (int j = 0; j < p->J; ++j) {
        numerator_for_gradient(&c, j);
        gradient_hessian(&c, j, gradient + j, hessian + j);
    }
    if (xbeta) memcpy(xbeta, c.xb, sizeof(double) * p->K);
    ctx_free(&c);
    return 0;
}

/* getPredictiveLogLikelihood (ModelSpecifics.hpp:652-690) for the
 * independent and grouped models (cox is re-grouped under the held-out
 * weights). */
int ccd_oracle_predictive_loglik(const ccd_problem* p, const double* beta, const double* held,
                                 double* out) {
    Ctx c;
    if (ctx_init(&c, p)) return 1;
    for (int j = 0; j < p->J; ++j) c.beta[j] = beta[j];
    prepare(&c);
    if (c.cumulative) {
        set_pid_for_accumulation(&c, held);
        for (int k = 0; k < c.K; ++k) c.kw[k] = held[k];
        for (int i = 0; i <= c.N; ++i) c.nw[i] = 0.0;
        for (int k = 0; k < c.K; ++k) c.nw[c.group[k]] += c.p->y[k] * c.kw[k];
        int save = c.use_w; c.use_w = 1;
        remaining_statistics(&c);
        c.use_w = save;
    }
    double ll = 0.0;
    for (int k = 0; k < c.K; ++k) {
        double y = p->y[k], w = held[k], xb = c.xb[k];
        double v;
        if (p->model == REF_PR) v = (y * xb - exp(xb)) * w;                         /* h:1587-1590 */
        else if (p->model == REF_COX) v = w == 0.0 ? 0.0 : y * w * (xb - log(c.acc_denom[c.group[k]]));
        else v = y * w * (xb - log(c.denom[c.group[k]]));                           /* h:1006-1009 */
        ll += v;
    }
    *out = ll;
    ctx_free(&c);
    return 0;
}
