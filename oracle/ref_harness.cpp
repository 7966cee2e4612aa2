// ref_harness.cpp -- TEST INFRASTRUCTURE (oracle).
//
// A C-ABI driver around the reference Cyclops C++ engine, compiled from the
// reference's own sources (oracle/Makefile) into oracle/_ref/libcyclops_ref.so.
// It is the parity checker for the CUDA path and the "reference" CPU
// baseline; it is never linked into the product library.
//
// What it mirrors:
//   * data ingest       RcppModelData ctor      src/RcppModelData.cpp:751-900
//                       (offset column first, dense, sparse, indicator; pid
//                       renumbered by runs, :878-900)
//   * prior set-up      .cyclopsSetPrior with the intercept excluded
//                       R/ModelFit.R:120-144 -> MixtureJointPrior::changePrior
//                       src/cyclops/priors/JointPrior.h:81-90
//   * fit               CcdInterface::fitModel -> CyclicCoordinateDescent::update
//                       src/cyclops/CcdInterface.cpp:654-672,
//                       src/cyclops/CyclicCoordinateDescent.cpp:586-615
//   * CV fold masks     CrossValidationSelector  src/cyclops/drivers/CrossValidationSelector.cpp:21-116
//   * engine probes     AbstractModelSpecifics virtuals, called directly on the
//                       same engine object the CCD uses.
//   * auto-search CV    AutoSearchCrossValidationDriver (drivers/, with
//                       utils/HParSearch.cpp) as CcdInterface::runCrossValidation
//                       drives it, src/cyclops/CcdInterface.cpp:731-790
//   * profile points    CcdInterface::evaluateProfileModel with one thread
//                       src/cyclops/CcdInterface.cpp:527-618
//   * profile bounds    CcdInterface::profileModel with one thread
//                       src/cyclops/CcdInterface.cpp:262-420: the reference's
//                       own RZeroIn (src/utils/RZeroIn.h, header-only) over
//                       OptimizationProfile (:223-260, restated below since
//                       CcdInterface.cpp needs the R runtime).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "CyclicCoordinateDescent.h"
#include "ModelData.h"
#include "engine/AbstractModelSpecifics.h"
#include "priors/JointPrior.h"
#include "priors/CovariatePrior.h"
#include "drivers/CrossValidationSelector.h"
#include "drivers/BootstrapSelector.h"
#include "drivers/AutoSearchCrossValidationDriver.h"
#include "drivers/GridSearchCrossValidationDriver.h"
#include "CcdInterface.h"
#include "io/ProgressLogger.h"

#include "utils/RZeroIn.h"

#ifdef CYC_REF_WITH_CUDA_ADAPTER
#include "CudaModelSpecifics.h"
#endif

extern "C" {
#include "ref_harness.h"
}

using namespace bsccs;

namespace {

thread_local std::string g_error;

class QuietLogger : public loggers::ProgressLogger {
public:
    void writeLine(const std::ostringstream&) override {}
    void yield() override {}
};

// keeps every line the drivers log (the auto search logs each point it tries)
class RecordingLogger : public loggers::ProgressLogger {
public:
    std::vector<std::string> lines;
    void writeLine(const std::ostringstream& s) override { lines.push_back(s.str()); }
    void yield() override {}
};

class ThrowingErrorHandler : public loggers::ErrorHandler {
public:
    void throwError(const std::ostringstream& stream) override {
        throw std::runtime_error(stream.str());
    }
};

// ModelData subclass that takes plain arrays, in the ingest order of
// RcppModelData (src/RcppModelData.cpp:751-900); RealType float is the
// reference's floatingPoint = 32 data (RcppModelData.cpp:724-728), the
// arrays rounded to float as they are copied in.
template <class RealType>
class HarnessModelDataT : public ModelData<RealType> {
public:
    HarnessModelDataT(ModelType type, const ref_problem* p,
                      std::vector<int> pid, std::vector<double> y, std::vector<double> time)
        : ModelData<RealType>(type, pid, y, std::vector<double>(), time,
                            bsccs::make_shared<QuietLogger>(),
                            bsccs::make_shared<ThrowingErrorHandler>()) {
        const int K = p->K;
        for (int j = 0; j < p->J; ++j) {
            const long long b = p->col_ptr[j];
            const long long e = p->col_ptr[j + 1];
            const long long vb = p->val_ptr[j];
            switch (p->col_format[j]) {
            case REF_DENSE:
                this->X.push_back((int*)nullptr, (int*)nullptr, p->col_val + vb, p->col_val + vb + K, DENSE);
                break;
            case REF_SPARSE:
                this->X.push_back(p->col_idx + b, p->col_idx + e, p->col_val + vb, p->col_val + vb + (e - b), SPARSE);
                break;
            case REF_INDICATOR:
                this->X.push_back(p->col_idx + b, p->col_idx + e, (double*)nullptr, (double*)nullptr, INDICATOR);
                break;
            case REF_INTERCEPT:
                this->X.push_back((int*)nullptr, (int*)nullptr, (double*)nullptr, (double*)nullptr, INTERCEPT);
                break;
            default:
                throw std::runtime_error("unknown column format");
            }
            this->X.getColumn(this->X.getNumberOfColumns() - 1).add_label(j);
        }
        this->X.nRows = K;
        if (p->has_offset) this->setHasOffsetCovariate(true);
        if (p->has_intercept) this->setHasInterceptCovariate(true);
        // pid renumbering by runs (RcppModelData.cpp:878-900)
        std::vector<int>& cpid = this->getPidVectorRef();
        if (cpid.empty()) {
            for (int i = 0; i < K; ++i) cpid.push_back(i);
            this->nPatients = K;
        } else {
            int current = 0;
            int last = cpid[0];
            cpid[0] = 0;
            for (size_t i = 1; i < cpid.size(); ++i) {
                if (cpid[i] != last) { ++current; last = cpid[i]; }
                cpid[i] = current;
            }
            this->nPatients = current + 1;
        }
    }
};

using HarnessModelData = HarnessModelDataT<double>;

ModelType toModelType(int m) {
    switch (m) {
    case REF_LR: return ModelType::LOGISTIC;
    case REF_PR: return ModelType::POISSON;
    case REF_CLR: return ModelType::CONDITIONAL_LOGISTIC;
    case REF_CPR: return ModelType::CONDITIONAL_POISSON;
    case REF_COX: return ModelType::COX;
    default: throw std::runtime_error("unknown model type");
    }
}

priors::PriorPtr makeCovariatePrior(int type, double variance) {
    switch (type) {
    case REF_PRIOR_NONE: return bsccs::make_shared<priors::NoPrior>();
    case REF_PRIOR_LAPLACE: return bsccs::make_shared<priors::LaplacePrior>(variance);
    case REF_PRIOR_NORMAL: return bsccs::make_shared<priors::NormalPrior>(variance);
    default: throw std::runtime_error("unknown prior type");
    }
}

struct Instance {
    std::unique_ptr<AbstractModelData> data;
    std::unique_ptr<AbstractModelSpecifics> engine;
    std::unique_ptr<CyclicCoordinateDescent> ccd;
    bool useWeights = false;
};

std::unique_ptr<Instance> build(const ref_problem* p, int device, bool fp32 = false) {
    std::vector<int> pid;
    if (p->pid) pid.assign(p->pid, p->pid + p->K);
    std::vector<double> y(p->y, p->y + p->K);
    std::vector<double> time;
    if (p->time) time.assign(p->time, p->time + p->K);

    auto inst = std::unique_ptr<Instance>(new Instance());
    if (fp32) inst->data.reset(new HarnessModelDataT<float>(toModelType(p->model), p, pid, y, time));
    else inst->data.reset(new HarnessModelData(toModelType(p->model), p, pid, y, time));
    if (device == 0) {
        inst->engine.reset(AbstractModelSpecifics::factory(
            toModelType(p->model), *inst->data, DeviceType::CPU, ""));
    } else {
#ifdef CYC_REF_WITH_CUDA_ADAPTER
        inst->engine.reset(cyclops_b200::makeCudaModelSpecifics(
            toModelType(p->model), *inst->data));
#else
        throw std::runtime_error("harness built without the CUDA adapter");
#endif
    }
    if (!inst->engine) throw std::runtime_error("Invalid model type.");

    auto defaultPrior = makeCovariatePrior(p->prior_type, p->variance);
    auto joint = bsccs::make_shared<priors::MixtureJointPrior>(defaultPrior, p->J);
    for (int i = 0; i < p->n_exclude; ++i) {
        joint->changePrior(bsccs::make_shared<priors::NoPrior>(), p->exclude[i]);
    }
    inst->ccd.reset(new CyclicCoordinateDescent(
        *inst->data, *inst->engine, joint,
        bsccs::make_shared<QuietLogger>(), bsccs::make_shared<ThrowingErrorHandler>()));
    inst->ccd->setNoiseLevel(SILENT);
    for (int i = 0; i < p->n_fixed; ++i) inst->ccd->setFixedBeta(p->fixed[i], true);   // R/ModelFit.R:205-214
    if (p->weights) {
        std::vector<double> w(p->weights, p->weights + p->K);
        inst->ccd->setWeights(w.data());
        inst->useWeights = true;
    }
    return inst;
}

ModeFindingArguments toArguments(const ref_control* c) {
    ModeFindingArguments a;
    a.tolerance = c->tolerance;
    a.maxIterations = c->max_iterations;
    a.convergenceType = c->convergence_type;
    a.useKktSwindle = c->use_kkt_swindle != 0;
    a.initialBound = c->initial_bound;
    a.maxBoundCount = c->max_bound_count;
    return a;
}

template <class F>
int guarded(F f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    } catch (const std::exception* e) {  // the engine throws pointers (ModelSpecifics.h:417)
        g_error = e->what();
        return 1;
    } catch (...) {
        g_error = "unknown exception";
        return 1;
    }
}

void fillResult(Instance& inst, int J, ref_result* out) {
    for (int j = 0; j < J; ++j) out->beta[j] = inst.ccd->getBeta(j);
    out->log_likelihood = inst.ccd->getLogLikelihood();
    out->log_prior = inst.ccd->getLogPrior();
    out->iterations = inst.ccd->getIterationCount();
    out->return_flag = (int)inst.ccd->getUpdateReturnFlag();
}

int fitWithDevice(const ref_problem* p, const ref_control* c, const double* start, ref_result* out,
                  int device, bool fp32 = false) {
    return guarded([&] {
        auto inst = build(p, device, fp32);
        if (start) {
            std::vector<double> b(start, start + p->J);
            inst->ccd->setBeta(b);
        }
        inst->ccd->update(toArguments(c));
        fillResult(*inst, p->J, out);
    });
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_fit(const ref_problem* p, const ref_control* c, const double* start_beta, ref_result* out) {
    return fitWithDevice(p, c, start_beta, out, 0);
}

int ref_fit_device(const ref_problem* p, const ref_control* c, const double* start_beta,
                   ref_result* out, int device) {
    return fitWithDevice(p, c, start_beta, out, device);
}

int ref_fit_fp32(const ref_problem* p, const ref_control* c, const double* start_beta, ref_result* out,
                 int device) {
    return fitWithDevice(p, c, start_beta, out, device, true);
}

int ref_engine_probe(const ref_problem* p, const double* beta, double* gradient, double* hessian,
                     double* xbeta, double* log_likelihood) {
    return guarded([&] {
        auto inst = build(p, 0);
        std::vector<double> b(beta, beta + p->J);
        inst->ccd->setBeta(b);
        *log_likelihood = inst->ccd->getLogLikelihood();  // runs the lazy set-up
        const bool w = inst->useWeights;
        for (int j = 0; j < p->J; ++j) {
            inst->engine->computeNumeratorForGradient(j, w);
            inst->engine->computeGradientAndHessian(j, gradient + j, hessian + j, w);
        }
        if (xbeta) {
            auto xb = inst->engine->getXBeta();
            std::memcpy(xbeta, xb.data(), sizeof(double) * p->K);
        }
    });
}

int ref_predictive_loglik(const ref_problem* p, const double* beta, const double* held_out,
                          double* out) {
    return guarded([&] {
        auto inst = build(p, 0);
        std::vector<double> b(beta, beta + p->J);
        inst->ccd->setBeta(b);
        inst->ccd->getLogLikelihood();
        std::vector<double> w(held_out, held_out + p->K);
        *out = inst->ccd->getNewPredictiveLogLikelihood(w.data());
    });
}

int ref_cv_weights(int K, const int* ids, int fold, long seed, int by_row, int n_reps,
                   double* out /* n_reps*fold x K */) {
    return guarded([&] {
        std::vector<int> idv(ids, ids + K);
        auto logger = bsccs::make_shared<QuietLogger>();
        auto err = bsccs::make_shared<ThrowingErrorHandler>();
        CrossValidationSelector sel(fold, idv, by_row ? SelectorType::BY_ROW : SelectorType::BY_PID,
                                    seed, logger, err, nullptr, nullptr);
        sel.reseed();
        std::vector<double> w;
        for (int task = 0; task < n_reps * fold; ++task) {
            const int f = task % fold;
            if (f == 0) sel.permute();
            sel.getWeights(f, w);
            std::memcpy(out + (size_t)task * K, w.data(), sizeof(double) * K);
        }
    });
}

// BootstrapSelector (by unit id) as BootstrapDriver::drive uses it: one
// permute per replicate, then the weights of batch 0.
int ref_bootstrap_weights(int K, const int* ids, int n_replicates, long seed, double* out /* n_replicates x K */) {
    return guarded([&] {
        std::vector<int> idv(ids, ids + K);
        auto logger = bsccs::make_shared<QuietLogger>();
        auto err = bsccs::make_shared<ThrowingErrorHandler>();
        BootstrapSelector sel(n_replicates, idv, SelectorType::BY_PID, seed, logger, err, nullptr);
        std::vector<double> w;
        for (int r = 0; r < n_replicates; ++r) {
            sel.permute();
            sel.getWeights(0, w);
            std::memcpy(out + (size_t)r * K, w.data(), sizeof(double) * K);
        }
    });
}

int ref_predictive_estimates(const ref_problem* p, const double* beta, const double* weights, double* y) {
    return guarded([&] {
        auto inst = build(p, 0);
        std::vector<double> b(beta, beta + p->J);
        inst->ccd->setBeta(b);
        inst->ccd->getLogLikelihood();          // runs the lazy set-up (xbeta)
        std::vector<double> w;
        if (weights) w.assign(weights, weights + p->K);
        inst->engine->getPredictiveEstimates(y, weights ? w.data() : nullptr);
    });
}

int ref_fisher(const ref_problem* p, const double* beta, const int* columns, int n, double* out, int device) {
    return guarded([&] {
        auto inst = build(p, device);
        std::vector<double> b(beta, beta + p->J);
        inst->ccd->setBeta(b);
        inst->ccd->getLogLikelihood();          // runs the lazy set-up (exp(xb), denominators)
        std::vector<size_t> idx(columns, columns + n);
        const auto m = inst->ccd->computeFisherInformation(idx);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) out[(size_t)i * n + j] = m(i, j);
    });
}

}  // extern "C"

namespace {
// OptimizationProfile (src/cyclops/CcdInterface.cpp:223-260): the profile
// objective at beta[index] = x, the other coefficients refitted
struct ProfileObjective {
    CyclicCoordinateDescent& ccd;
    ModeFindingArguments args;
    int index;
    double max, threshold;
    bool includePenalty;
    int nEvals = 0;
    double objective(double x) {
        ++nEvals;
        ccd.setBeta(index, x);
        ccd.setFixedBeta(index, true);
        ccd.update(args);
        ccd.setFixedBeta(index, false);
        double y = ccd.getLogLikelihood() + threshold - max;
        if (includePenalty) y += ccd.getLogPrior();
        return y;
    }
    double getMaximum() { return threshold; }
};
}  // namespace

extern "C" {

int ref_profile(const ref_problem* p, const ref_control* c, const double* start_beta, const int* columns, int n,
                double threshold, int include_penalty, int override_no_regularization, double* lower,
                double* upper, int* evaluations, ref_result* fit, int device) {
    return guarded([&] {
        auto inst = build(p, device);
        if (start_beta) {
            std::vector<double> b(start_beta, start_beta + p->J);
            inst->ccd->setBeta(b);
        }
        const ModeFindingArguments args = toArguments(c);
        CyclicCoordinateDescent& ccd = *inst->ccd;
        ccd.update(args);
        if (fit) fillResult(*inst, p->J, fit);
        double mode = ccd.getLogLikelihood();
        if (include_penalty) mode += ccd.getLogPrior();
        std::vector<double> x0s(p->J);
        for (int j = 0; j < p->J; ++j) x0s[j] = ccd.getBeta(j);
        for (int i = 0; i < n; ++i) {
            if (!override_no_regularization && ccd.getIsRegularized(columns[i])) {
                std::ostringstream m;
                m << "Variable " << columns[i] << " is regularized.";
                throw std::runtime_error(m.str());
            }
        }
        for (int i = 0; i < n; ++i) {                     // bounds (id, +1), (id, -1) in order, one CCD
            int count = 0;
            for (double direction : {+1.0, -1.0}) {
                const int index = columns[i];
                ProfileObjective eval{ccd, args, index, mode, threshold, include_penalty != 0};
                bsccs::RZeroIn<ProfileObjective> zeroIn(eval, 1E-3);
                const double obj0 = eval.getMaximum();
                auto bracket = zeroIn.bracketSignChange(x0s[index], obj0, direction);
                const double pt = std::isnan(bracket.second)
                                      ? NAN : zeroIn.getRoot(x0s[index], bracket.first, obj0, bracket.second);
                (direction > 0 ? upper : lower)[i] = pt;
                count += eval.nEvals;
            }
            evaluations[i] = count;
        }
    });
}

int ref_profile_points(const ref_problem* p, const ref_control* c, const double* start_beta, int column,
                       const double* points, int n, int include_penalty, double* values, int device) {
    return guarded([&] {
        auto inst = build(p, device);
        if (start_beta) {
            std::vector<double> b(start_beta, start_beta + p->J);
            inst->ccd->setBeta(b);
        }
        const ModeFindingArguments args = toArguments(c);
        CyclicCoordinateDescent& ccd = *inst->ccd;
        ccd.update(args);
        for (int j = 0; j < p->J; ++j) ccd.getBeta(j);    // x0s (CcdInterface.cpp:555-559)
        // evaluateProfileModel with one thread (CcdInterface.cpp:527-618)
        ccd.makeDirty();
        {
            ProfileObjective eval{ccd, args, column, 0.0, 0.0, include_penalty != 0};
            eval.objective(0.0);
        }
        for (int i = 0; i < n; ++i) {
            ProfileObjective eval{ccd, args, column, 0.0, 0.0, include_penalty != 0};
            values[i] = eval.objective(points[i]);
        }
    });
}

}  // extern "C"

namespace {
// the auto-search driver with its result readable (maxPoint is protected)
class AutoSearchProbe : public AutoSearchCrossValidationDriver {
public:
    using AutoSearchCrossValidationDriver::AutoSearchCrossValidationDriver;
    MaxPoint best() const { return maxPoint; }
};

// the grid-search driver with its grid readable (protected members)
class GridSearchProbe : public GridSearchCrossValidationDriver {
public:
    using GridSearchCrossValidationDriver::GridSearchCrossValidationDriver;
    const std::vector<double>& points() const { return gridPoint; }
    const std::vector<double>& values() const { return gridValue; }
};
}  // namespace

extern "C" {

int ref_cv_auto(const ref_problem* p, const ref_control* c, int fold, int n_reps, long seed, int by_row,
                double starting_variance, int reset_coefficients, double* best_variance, double* best_value,
                double* tried_variance, double* tried_mean, double* tried_sd, int max_tried, int* n_tried) {
    return guarded([&] {
        auto inst = build(p, 0);
        CCDArguments args = CCDArguments();   // value-initialised: the flags it leaves unset read as false / 0
        args.modeFinding = toArguments(c);
        args.threads = 1;
        args.seed = seed;
        args.resetCoefficients = reset_coefficients != 0;
        args.useNormalPrior = p->prior_type == REF_PRIOR_NORMAL;
        args.crossValidation.doCrossValidation = true;
        args.crossValidation.useAutoSearchCV = true;
        args.crossValidation.fold = fold;
        args.crossValidation.foldToCompute = fold * n_reps;
        args.crossValidation.startingVariance = starting_variance;
        args.crossValidation.selectorType = by_row ? SelectorType::BY_ROW : SelectorType::BY_PID;
        auto logger = bsccs::make_shared<RecordingLogger>();
        auto err = bsccs::make_shared<ThrowingErrorHandler>();
        std::vector<int> ids = inst->data->getPidVectorSTL();
        CrossValidationSelector selector(fold, ids, args.crossValidation.selectorType, seed, logger, err,
                                         nullptr, nullptr);
        AutoSearchProbe driver(*inst->data, args, logger, err, nullptr);
        driver.drive(*inst->ccd, selector, args);
        const MaxPoint mp = driver.best();
        *best_variance = mp.point[0];
        *best_value = mp.value;
        // the points tried, from the driver's log (6 significant digits)
        int n = 0;
        double m = 0, sd = 0;
        for (const auto& line : logger->lines) {
            const auto a = line.find("AvgPred = ");
            if (a != std::string::npos) std::sscanf(line.c_str() + a, "AvgPred = %lf with stdev = %lf", &m, &sd);
            const auto b = line.find("Completed at ");
            if (b != std::string::npos && n < max_tried) {
                double v = 0;
                std::sscanf(line.c_str() + b, "Completed at %lf", &v);
                tried_variance[n] = v;
                tried_mean[n] = m;
                tried_sd[n] = sd;
                ++n;
            }
        }
        *n_tried = n;
    });
}

int ref_cv_grid(const ref_problem* p, const ref_control* c, int fold, long seed, int by_row, double lower,
                double upper, int grid_steps, int reset_coefficients, double* points, double* values,
                double* fold_pred) {
    return guarded([&] {
        auto inst = build(p, 0);
        CCDArguments args = CCDArguments();
        args.modeFinding = toArguments(c);
        args.threads = 1;
        args.seed = seed;
        args.resetCoefficients = reset_coefficients != 0;
        args.useNormalPrior = p->prior_type == REF_PRIOR_NORMAL;
        args.crossValidation.doCrossValidation = true;
        args.crossValidation.useAutoSearchCV = false;
        args.crossValidation.fold = fold;
        args.crossValidation.foldToCompute = fold;
        args.crossValidation.lowerLimit = lower;
        args.crossValidation.upperLimit = upper;
        args.crossValidation.gridSteps = grid_steps;
        args.crossValidation.selectorType = by_row ? SelectorType::BY_ROW : SelectorType::BY_PID;
        auto logger = bsccs::make_shared<RecordingLogger>();
        auto err = bsccs::make_shared<ThrowingErrorHandler>();
        // the fit's weights become the selector's original weights
        // (CcdInterface::runCrossValidation, CcdInterface.cpp:738-754)
        std::vector<double> original;
        if (p->weights) original.assign(p->weights, p->weights + p->K);
        std::vector<int> ids = inst->data->getPidVectorSTL();
        CrossValidationSelector selector(fold, ids, args.crossValidation.selectorType, seed, logger, err, nullptr,
                                         p->weights ? &original : nullptr);
        GridSearchProbe driver(args, logger, err, nullptr);
        driver.drive(*inst->ccd, selector, args);
        for (int i = 0; i < grid_steps; ++i) {
            points[i] = driver.points()[i];
            values[i] = driver.values()[i];
        }
        // per-fold held-out log likelihoods from the driver's log (6 digits), NaN if not computed
        int n = 0;
        for (const auto& line : logger->lines) {
            const auto a = line.find("pred log like = ");
            if (a == std::string::npos || n >= grid_steps * fold) continue;
            double v = NAN;
            if (std::sscanf(line.c_str() + a, "pred log like = %lf", &v) != 1) v = NAN;
            fold_pred[n++] = v;
        }
    });
}

int ref_ingest(const ref_ingest_input* in, ref_ingest_output* out) {
    return guarded([&] {
        std::memset(out, 0, sizeof(*out));
        ModelData<double> md(toModelType(in->model), bsccs::make_shared<QuietLogger>(),
                             bsccs::make_shared<ThrowingErrorHandler>());
        const size_t n = (size_t)in->n_outcomes;
        std::vector<IdType> strata, rows(in->row_id, in->row_id + n);
        if (in->stratum_id) strata.assign(in->stratum_id, in->stratum_id + n);
        std::vector<double> y(in->y, in->y + n), time;
        if (in->time) time.assign(in->time, in->time + n);
        md.loadY(strata, rows, y, time);
        if (in->add_intercept) md.loadX(0, std::vector<IdType>(), std::vector<double>(), false, false, false);
        const size_t m = (size_t)in->n_covariates;
        if (m) {
            std::vector<int64_t> cid(in->covariate_id, in->covariate_id + m), crow(in->covariate_row, in->covariate_row + m);
            std::vector<double> cval;
            if (in->covariate_value) cval.assign(in->covariate_value, in->covariate_value + m);
            md.loadMultipleX(cid, crow, cval, false, false, false, false);
        }
        if (in->offset_from_time) {
            md.setOffsetCovariate(-1);
            md.logTransformCovariate(0);
        }
        const auto& X = md.getX();
        const int J = (int)X.getNumberOfColumns(), K = (int)X.getNumberOfRows();
        out->K = K;
        out->J = J;
        out->col_format = (int*)std::malloc(sizeof(int) * (J + 1));
        out->col_ptr = (long long*)std::malloc(sizeof(long long) * (J + 1));
        out->val_ptr = (long long*)std::malloc(sizeof(long long) * (J + 1));
        out->col_label = (long long*)std::malloc(sizeof(long long) * (J + 1));
        std::vector<int> idx;
        std::vector<double> val;
        out->col_ptr[0] = out->val_ptr[0] = 0;
        for (int j = 0; j < J; ++j) {
            const auto& c = X.getColumn(j);
            const FormatType f = c.getFormatType();
            out->col_format[j] = f == DENSE ? REF_DENSE : f == SPARSE ? REF_SPARSE : f == INDICATOR ? REF_INDICATOR : REF_INTERCEPT;
            out->col_label[j] = (long long)c.getNumericalLabel();
            if (f == SPARSE || f == INDICATOR) {
                const auto& r = c.getColumnsVector();
                idx.insert(idx.end(), r.begin(), r.end());
            }
            if (f == SPARSE || f == DENSE) {
                const auto& v = c.getDataVector();
                val.insert(val.end(), v.begin(), v.end());
            }
            out->col_ptr[j + 1] = (long long)idx.size();
            out->val_ptr[j + 1] = (long long)val.size();
        }
        out->col_idx = (int*)std::malloc(sizeof(int) * (idx.size() + 1));
        out->col_val = (double*)std::malloc(sizeof(double) * (val.size() + 1));
        std::memcpy(out->col_idx, idx.data(), sizeof(int) * idx.size());
        std::memcpy(out->col_val, val.data(), sizeof(double) * val.size());
        const auto pid = md.getPidVectorSTL();
        out->pid = (int*)std::malloc(sizeof(int) * (K + 1));
        for (int k = 0; k < K; ++k) out->pid[k] = pid.empty() ? k : pid[k];
        out->y = (double*)std::malloc(sizeof(double) * (K + 1));
        const auto& yy = md.getYVectorRef();
        for (int k = 0; k < K; ++k) out->y[k] = yy[k];
        if (!time.empty()) {
            out->time = (double*)std::malloc(sizeof(double) * (K + 1));
            const auto& tt = md.getTimeVectorRef();
            for (int k = 0; k < K; ++k) out->time[k] = tt[k];
        }
        out->has_offset = md.getHasOffsetCovariate() ? 1 : 0;
        out->has_intercept = md.getHasInterceptCovariate() ? 1 : 0;
    });
}

void ref_ingest_free(ref_ingest_output* out) {
    if (!out) return;
    std::free(out->col_format); std::free(out->col_ptr); std::free(out->col_idx); std::free(out->val_ptr);
    std::free(out->col_val); std::free(out->col_label); std::free(out->pid); std::free(out->y); std::free(out->time);
    std::memset(out, 0, sizeof(*out));
}

}  // extern "C"
