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
