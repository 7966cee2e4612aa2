// cv.cu -- cross-validation fold masks (host code).
//
// Restates CrossValidationSelector (src/cyclops/drivers/CrossValidationSelector.cpp:21-116,
// 138-143) and its use in AbstractCrossValidationDriver::doCrossValidationStep
// (src/cyclops/drivers/AbstractCrossValidationDriver.cpp:160-190): a
// std::mt19937 seeded once, a std::shuffle of the exchangeable units at the
// first fold of every repetition, and fold f holding out the f-th interval
// of the permutation (interval sizes differ by at most one).  Using the same
// standard-library engine and shuffle gives the reference's masks exactly.
#include "internal.cuh"

#include <algorithm>
#include <random>
#include <set>

using namespace cyc;

extern "C" int cyc_cv_fold_weights(int K, const int* ids, int folds, long seed, int by_row, int n_reps,
                                   double* out) {
    return guarded([&] {
        CYC_REQUIRE(K > 0 && folds > 0 && n_reps > 0 && out, CYC_ERR_ARGUMENT, "bad argument");
        CYC_REQUIRE(by_row || ids, CYC_ERR_ARGUMENT, "by-stratum folds need ids");
        size_t N = (size_t)K;
        if (!by_row) N = (size_t)(*std::max_element(ids, ids + K)) + 1;
        CYC_REQUIRE(N >= (size_t)folds, CYC_ERR_ARGUMENT, "fewer units than folds");
        std::vector<int> start;
        int index = 0;
        const int fraction = (int)(N / folds);
        const int extra = (int)N - fraction * folds;
        for (int i = 0; i < folds; ++i) {
            start.push_back(index);
            index += fraction;
            if (i < extra) index++;
        }
        start.push_back((int)N);
        const bool deterministic = (seed == -1);
        std::mt19937 prng;
        if (!deterministic) prng.seed(seed);
        std::vector<int> perm(N);
        for (size_t i = 0; i < N; ++i) perm[i] = (int)i;
        for (int task = 0; task < n_reps * folds; ++task) {
            const int f = task % folds;
            if (f == 0 && !deterministic) std::shuffle(perm.begin(), perm.end(), prng);
            double* w = out + (size_t)task * K;
            std::fill(w, w + K, 1.0);
            if (by_row) {
                for (int i = start[f]; i < start[f + 1]; ++i) w[perm[i]] = 0.0;
            } else {
                std::set<int> ex(perm.begin() + start[f], perm.begin() + start[f + 1]);
                for (int k = 0; k < K; ++k)
                    if (ex.count(ids[k])) w[k] = 0.0;
            }
        }
    });
}

// Bootstrap replicate weights: restates BootstrapSelector
// (src/cyclops/drivers/BootstrapSelector.cpp:15-88) as BootstrapDriver::drive
// uses it (src/cyclops/drivers/BootstrapDriver.cpp:47-64).  The exchangeable
// units are the ids 0..N-1 (BY_PID, N = max id + 1); the units whose
// exclusion weight is 0 (all of them without one) are the ones drawn from.
// One std::mt19937, seeded as AbstractSelector seeds it
// (AbstractSelector.cpp:18-37), draws N_included units with replacement by
// std::uniform_int_distribution per permute(); the selector's constructor
// permutes once, then every replicate permutes again and weights row k by
// the number of times its unit was drawn.  The same standard-library engine
// and distribution give the reference's weights exactly.
extern "C" int cyc_bootstrap_weights(int K, const int* ids, int n_replicates, long seed,
                                     const double* unit_exclude, double* out) {
    return guarded([&] {
        CYC_REQUIRE(K > 0 && n_replicates > 0 && out, CYC_ERR_ARGUMENT, "bad argument");
        CYC_REQUIRE(seed != -99, CYC_ERR_ARGUMENT, "seed -99 (the clock) is not reproducible; pass a seed");
        std::vector<int> idv(K);
        for (int k = 0; k < K; ++k) idv[k] = ids ? ids[k] : k;
        for (int k = 0; k < K; ++k) CYC_REQUIRE(idv[k] >= 0, CYC_ERR_ARGUMENT, "negative unit id");
        const int N = *std::max_element(idv.begin(), idv.end()) + 1;
        std::vector<int> included;
        for (int i = 0; i < N; ++i)
            if (!unit_exclude || unit_exclude[i] == 0) included.push_back(i);
        CYC_REQUIRE(!included.empty(), CYC_ERR_ARGUMENT, "every unit is excluded");
        std::mt19937 prng;
        if (seed != -1) prng.seed(seed);
        const int n_inc = (int)included.size();
        std::vector<int> count(N);
        auto permute = [&] {
            std::fill(count.begin(), count.end(), 0);
            std::uniform_int_distribution<int> uniform(0, n_inc - 1);
            for (int i = 0; i < n_inc; ++i) ++count[included[uniform(prng)]];
        };
        permute();                                      // the selector's constructor
        for (int r = 0; r < n_replicates; ++r) {
            permute();
            double* w = out + (size_t)r * K;
            for (int k = 0; k < K; ++k) w[k] = (double)count[idv[k]];
        }
    });
}
