// variance_search.h -- the one-dimensional search over a prior variance that
// auto-search cross-validation runs (host code, no CUDA).
//
// UniModalSearch (src/utils/HParSearch.h:28-60, src/utils/HParSearch.cpp)
// with the settings AutoSearchCrossValidationDriver gives it
// (src/cyclops/drivers/AutoSearchCrossValidationDriver.cpp:104).
#pragma once
#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <utility>

namespace cyc {

// UniModalSearch with the driver's settings: steps of x10 until the best
// point is bracketed, then the argmax of a quadratic in log(variance)
// fitted with weights 1 / stdev; stops when that argmax is within log(1.5)
// of the best point or promises less than 1 % over it
struct VarianceSearch {
    static constexpr double kStep = 10.0, kStopY = 0.01, kFirstCut = 1.0;
    std::map<double, std::pair<double, double>> pts;     // x -> (mean, stdev)
    double best = 0.0;

    void tried(double x, double m, double sd) {
        pts[x] = {m, sd};
        if (pts.size() == 1 || m > pts[best].first) best = x;
    }

    // weighted least squares for c0 + c1 log x + c2 log^2 x (QuadrLogFit),
    // the 3x3 normal equations solved by Gaussian elimination with full pivoting
    void fit(double c[3]) const {
        double minsd = std::numeric_limits<double>::max();
        for (const auto& p : pts)
            if (p.second.second > 0 && p.second.second < minsd) minsd = p.second.second;
        const double zero = minsd < std::numeric_limits<double>::max() ? 100.0 / minsd : 1.0;
        double A[3][4] = {};
        for (const auto& p : pts) {
            const double w = p.second.second > 0 ? 1.0 / p.second.second : zero;
            const double l = std::log(p.first);
            const double row[3] = {1.0, l, l * l};
            for (int i = 0; i < 3; ++i) {
                for (int j = 0; j < 3; ++j) A[i][j] += row[i] * w * row[j];
                A[i][3] += row[i] * w * p.second.first;
            }
        }
        int col[3] = {0, 1, 2};
        for (int k = 0; k < 3; ++k) {
            int pi = k, pj = k;
            for (int i = k; i < 3; ++i)
                for (int j = k; j < 3; ++j)
                    if (std::fabs(A[i][j]) > std::fabs(A[pi][pj])) { pi = i; pj = j; }
            std::swap(A[k], A[pi]);
            for (int i = 0; i < 3; ++i) std::swap(A[i][k], A[i][pj]);
            std::swap(col[k], col[pj]);
            for (int i = k + 1; i < 3; ++i) {
                const double f = A[i][k] / A[k][k];
                for (int j = k; j < 4; ++j) A[i][j] -= f * A[k][j];
            }
        }
        double x[3];
        for (int k = 2; k >= 0; --k) {
            double sum = A[k][3];
            for (int j = k + 1; j < 3; ++j) sum -= A[k][j] * x[j];
            x[k] = sum / A[k][k];
        }
        for (int k = 0; k < 3; ++k) c[col[k]] = x[k];
    }

    // (continue, next x, expected value there)
    void step(bool* go, double* next, double* expected) const {
        *go = true;
        *expected = 0.0;
        const double lo = pts.begin()->first, hi = pts.rbegin()->first;
        if (pts.size() == 1) {
            *next = lo < kFirstCut ? lo * kStep : lo / kStep;
        } else if (pts.size() == 2) {
            *next = pts.begin()->second.first > pts.rbegin()->second.first ? lo / kStep : hi * kStep;
        } else if (lo == best) {
            *next = best / kStep;
            if (!(best > std::numeric_limits<double>::denorm_min())) { *go = false; *expected = pts.at(best).first; }
        } else if (hi == best) {
            *next = best * kStep;
            if (!(best < std::numeric_limits<double>::infinity())) { *go = false; *expected = pts.at(best).first; }
        } else {
            double c[3];
            fit(c);
            const double log_argmax = -c[1] / c[2] / 2;
            const double expected_max = -c[1] * c[1] / c[2] / 4 + c[0];
            const double maxval = pts.at(best).first;
            if (maxval == 0) *go = false;
            else if ((expected_max - maxval) / std::fabs(maxval) < kStopY) *go = false;
            else if (std::fabs(log_argmax - std::log(best)) < std::log(1.5)) *go = false;
            *next = std::exp(log_argmax);
            *expected = expected_max;
        }
    }
};

}  // namespace cyc
