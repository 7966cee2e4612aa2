// CudaModelSpecifics.h -- drop-in GPU engine for Cyclops.
//
// A subclass of the reference's bsccs::AbstractModelSpecifics
// (src/cyclops/engine/AbstractModelSpecifics.h:36-229) whose virtuals forward
// to the C ABI of libcyclops_b200.so (include/cyclops_b200.h).  It is the
// object `AbstractModelSpecifics::deviceFactory` returns for DeviceType::GPU
// (src/cyclops/engine/AbstractModelSpecifics.cpp:21-41), so
// CyclicCoordinateDescent and, above it, fitCyclopsModel(computeDevice = ...)
// (src/RcppCyclopsInterface.cpp:884-892) drive the CUDA engine unchanged.
//
// Header-only; compile it inside the reference tree (it needs the reference's
// ModelData.h and AbstractModelSpecifics.h) and link libcyclops_b200.so.
#ifndef CYCLOPS_B200_CUDA_MODEL_SPECIFICS_H
#define CYCLOPS_B200_CUDA_MODEL_SPECIFICS_H

#include <stdexcept>
#include <string>
#include <vector>

#include "ModelData.h"
#include "engine/AbstractModelSpecifics.h"
#include "cyclops_b200.h"

namespace cyclops_b200 {

inline void check(int status) {
    if (status != CYC_OK) throw std::runtime_error(std::string("cyclops_b200: ") + cyc_last_error());
}

inline int toCycModel(bsccs::ModelType t) {
    switch (t) {
    case bsccs::ModelType::LOGISTIC: return CYC_LR;
    case bsccs::ModelType::POISSON: return CYC_PR;
    case bsccs::ModelType::CONDITIONAL_LOGISTIC: return CYC_CLR;
    case bsccs::ModelType::CONDITIONAL_POISSON: return CYC_CPR;
    case bsccs::ModelType::COX: return CYC_COX;
    default: return -1;
    }
}

// Shares one device dataset between an engine and its clones.
struct SharedDataset {
    cyc_dataset* ds = nullptr;
    ~SharedDataset() { if (ds) cyc_dataset_destroy(ds); }
};

// RealType is the ModelData's: double, or float for the reference's
// floatingPoint = 32 data (src/RcppModelData.cpp:724-728), whose values,
// outcomes and times are widened to double at upload; the engine computes
// in FP64 on those values either way.
template <class RealType>
class CudaModelSpecificsT : public bsccs::AbstractModelSpecifics {
public:
    CudaModelSpecificsT(const bsccs::ModelData<RealType>& data, int cycModel, int device = 0)
        : bsccs::AbstractModelSpecifics(data), data_(data), model_(cycModel), device_(device),
          shared_(std::make_shared<SharedDataset>()) {
        upload();
    }

    ~CudaModelSpecificsT() override {
        if (engine_) cyc_engine_destroy(engine_);
    }

    // initialize (ModelSpecifics.hpp:1899-1952): the CCD passes all-null pointers
    void initialize(int iN, int iK, int iJ, const void*, double*, double*, double*, double*,
                    std::vector<std::vector<int>*>*, const int*, double*, double*, double*, double*,
                    const double*) override {
        N = iN; K = iK; J = iJ;
        if (!engine_) check(cyc_engine_create(shared_->ds, &engine_));
        int n = 0;
        check(cyc_engine_get_n(engine_, &n));
        N = n;
    }

    void setWeights(double* w, double* /*cenWeights*/, bool useCV) override {
        check(cyc_engine_set_weights(engine_, w, useCV ? 1 : 0));
    }
    void computeGradientAndHessian(int index, double* g, double* h, bool useWeights) override {
        check(cyc_engine_compute_gradient_and_hessian(engine_, index, g, h, useWeights ? 1 : 0));
    }
    void computeMMGradientAndHessian(std::vector<bsccs::GradientHessian>&, const std::vector<bool>&,
                                     bool) override {
        throw std::logic_error("cyclops_b200: the MM algorithm is not offered on the GPU engine");
    }
    void computeNumeratorForGradient(int index, bool useWeights) override {
        check(cyc_engine_compute_numerator_for_gradient(engine_, index, useWeights ? 1 : 0));
    }
    // computeFisherInformation (ModelSpecifics.hpp:1203-1351) for one pair
    void computeFisherInformation(int indexOne, int indexTwo, double* oinfo, bool useWeights) override {
        if (indexOne == indexTwo) {
            check(cyc_engine_fisher_information(engine_, &indexOne, 1, useWeights ? 1 : 0, oinfo));
        } else {
            const int cols[2] = {indexOne, indexTwo};
            double m[4];
            check(cyc_engine_fisher_information(engine_, cols, 2, useWeights ? 1 : 0, m));
            *oinfo = m[1];
        }
    }
    void updateXBeta(double delta, int index, bool useWeights) override {
        check(cyc_engine_update_xbeta(engine_, delta, index, useWeights ? 1 : 0));
    }
    void computeXBeta(double* beta, bool useWeights) override {
        check(cyc_engine_compute_xbeta(engine_, beta, useWeights ? 1 : 0));
    }
    void computeRemainingStatistics(bool useWeights) override {
        check(cyc_engine_compute_remaining_statistics(engine_, useWeights ? 1 : 0));
    }
    void computeFixedTermsInLogLikelihood(bool useCV) override {
        check(cyc_engine_compute_fixed_terms_ll(engine_, useCV ? 1 : 0));
    }
    void computeFixedTermsInGradientAndHessian(bool useCV) override {
        check(cyc_engine_compute_fixed_terms_gh(engine_, useCV ? 1 : 0));
    }
    double getLogLikelihood(bool useCV) override {
        double v = 0.0;
        check(cyc_engine_get_log_likelihood(engine_, useCV ? 1 : 0, &v));
        return v;
    }
    double getPredictiveLogLikelihood(double* weights) override {
        double v = 0.0;
        check(cyc_engine_get_predictive_log_likelihood(engine_, weights, &v));
        return v;
    }
    void getPredictiveEstimates(double* y, double* weights) override {
        check(cyc_engine_get_predictive_estimates(engine_, y, weights));
    }
    double getGradientObjective(bool useCV) override {
        double v = 0.0;
        check(cyc_engine_get_gradient_objective(engine_, useCV ? 1 : 0, &v));
        return v;
    }
    void printTiming() override {}

    bsccs::AbstractModelSpecifics* clone() const override {
        return new CudaModelSpecificsT(*this, CloneTag());
    }

    const std::vector<double> getXBeta() override {
        std::vector<double> v(K);
        check(cyc_engine_get_xbeta(engine_, v.data()));
        return v;
    }
    const std::vector<double> getXBetaSave() override {
        std::vector<double> v(K);
        check(cyc_engine_get_xbeta_save(engine_, v.data()));
        return v;
    }
    void saveXBeta() override { check(cyc_engine_save_xbeta(engine_)); }
    void zeroXBeta() override { check(cyc_engine_zero_xbeta(engine_)); }
    void axpyXBeta(const double beta, const int j) override {
        check(cyc_engine_axpy_xbeta(engine_, beta, j));
    }

protected:
    void deviceInitialization() override {}
    bool allocateXjY() override { return true; }
    bool allocateXjX() override { return false; }
    bool initializeAccumulationVectors() override { return model_ == CYC_COX; }
    bool hasResetableAccumulators() override { return false; }

private:
    struct CloneTag {};
    CudaModelSpecificsT(const CudaModelSpecificsT& other, CloneTag)
        : bsccs::AbstractModelSpecifics(other.data_), data_(other.data_), model_(other.model_),
          device_(other.device_), shared_(other.shared_) {}

    // ModelData -> cyc_data_desc (the column store in ingest order)
    void upload() {
        const auto& X = data_.getX();
        const int K0 = (int)data_.getNumberOfRows();
        const int J0 = (int)data_.getNumberOfColumns();
        std::vector<int> fmt(J0);
        std::vector<long long> cp(J0 + 1, 0), vp(J0 + 1, 0);
        std::vector<int> idx;
        std::vector<double> val;
        for (int j = 0; j < J0; ++j) {
            const auto f = X.getFormatType(j);
            fmt[j] = (int)f;
            if (f == bsccs::SPARSE || f == bsccs::INDICATOR) {
                const int* r = X.getCompressedColumnVector(j);
                const size_t n = X.getNumberOfEntries(j);
                idx.insert(idx.end(), r, r + n);
                if (f == bsccs::SPARSE) {
                    const RealType* v = X.getDataVector(j);
                    val.insert(val.end(), v, v + n);
                }
            } else if (f == bsccs::DENSE) {
                const RealType* v = X.getDataVector(j);
                val.insert(val.end(), v, v + K0);
            }
            cp[j + 1] = (long long)idx.size();
            vp[j + 1] = (long long)val.size();
        }
        const auto& pid = data_.getPidVectorRef();
        const std::vector<double> y(data_.getYVectorRef().begin(), data_.getYVectorRef().end());
        const std::vector<double> t(data_.getTimeVectorRef().begin(), data_.getTimeVectorRef().end());
        cyc_data_desc d{};
        d.model = model_;
        d.K = K0;
        d.J = J0;
        d.pid = pid.empty() ? nullptr : pid.data();
        d.y = y.data();
        d.time = t.empty() ? nullptr : t.data();
        d.col_format = fmt.data();
        d.col_ptr = cp.data();
        d.col_idx = idx.empty() ? nullptr : idx.data();
        d.val_ptr = vp.data();
        d.col_val = val.empty() ? nullptr : val.data();
        d.has_offset = data_.getHasOffsetCovariate() ? 1 : 0;
        d.has_intercept = data_.getHasInterceptCovariate() ? 1 : 0;
        check(cyc_dataset_create(&d, device_, &shared_->ds));
    }

    const bsccs::ModelData<RealType>& data_;
    int model_;
    int device_;
    std::shared_ptr<SharedDataset> shared_;
    cyc_engine* engine_ = nullptr;
};

// The body of the GPU case of deviceFactory
// (src/cyclops/engine/AbstractModelSpecifics.cpp:32-35): nullptr for model
// types this engine does not offer, which the caller reports as
// "Invalid model type." (src/RcppCyclopsInterface.cpp:890-892).
using CudaModelSpecifics = CudaModelSpecificsT<double>;

inline bsccs::AbstractModelSpecifics* makeCudaModelSpecifics(bsccs::ModelType type,
                                                             const bsccs::AbstractModelData& data,
                                                             int device = 0) {
    const int m = toCycModel(type);
    if (m < 0) return nullptr;
    if (data.getPrecisionType() == bsccs::PrecisionType::FP64)
        return new CudaModelSpecificsT<double>(static_cast<const bsccs::ModelData<double>&>(data), m, device);
    if (data.getPrecisionType() == bsccs::PrecisionType::FP32)
        return new CudaModelSpecificsT<float>(static_cast<const bsccs::ModelData<float>&>(data), m, device);
    return nullptr;
}

}  // namespace cyclops_b200

#endif
