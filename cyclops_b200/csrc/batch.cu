// batch.cu -- cyc_batch_fit: many fits sharing one dataset, advanced
// coordinate by coordinate in one persistent kernel (lr, pr, clr, cpr).
//
// The reference runs such fits (CV folds x prior grid, bootstrap replicates)
// as independent CyclicCoordinateDescent clones on CPU threads
// (src/cyclops/drivers/AbstractCrossValidationDriver.cpp:131-248); each clone
// runs the serial coordinate loop of findMode
// (src/cyclops/CyclicCoordinateDescent.cpp:1008-1021).
//
// Layout and schedule (B200):
//  * fits are packed G to a group; a group is one thread-block cluster of C
//    CTAs; the cluster's CTAs split the rows into C contiguous ranges
//    (aligned to strata for clr/cpr), so the per-row state a CTA touches is
//    its own and only the per-fit (gradient, Hessian) partials cross CTAs,
//    through distributed shared memory, once per coordinate;
//  * per-(row, fit) state is the linear predictor only, stored
//    xb[group][row][G] so the G fits of one row share one 32-byte sector
//    (FP32) -- exp(xb) is recomputed where needed instead of stored;
//  * every CTA of a cluster computes the coordinate step for all G fits from
//    the same partials in the same order, so all CTAs agree on delta without
//    a second barrier; rank 0 alone writes beta and the trust region;
//  * the convergence test (performCheckConvergence, :839-906) runs in the
//    kernel after every cycle; a fit that has converged stops stepping, and
//    the cluster exits when all its fits are done.
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "engine.cuh"
#include "solver_common.cuh"
#include "variance_search.h"

namespace cg = cooperative_groups;

namespace cyc {

namespace {

constexpr int kBT = 256;          // threads per CTA
constexpr int kMaxC = 8;          // CTAs per cluster (portable limit)
// shared memory per CTA for rows arriving by cp.async (8-fit groups)
constexpr int kAsyncBytes = 32768;

struct BatchArgs {
    int model, K, J, S, C;
    const int* fmt;
    const long long* col_ptr;
    const long long* val_ptr;
    const int* idx;
    const double* val;
    const int* split;             // J x (C+1): first entry of rank r's rows, relative to the column
    const int* rpart;             // C+1 row boundaries
    const double* y;
    const int* strat;             // K (grouped)
    const int* strat_ptr;         // S+1 (grouped)
    const int* fixb;              // J
    const unsigned char* lane_fix; // [groups][J]: fits (bit f) holding column j at its value in this
                                  // launch (the inactive columns of the KKT swindle), or null
    const int* ptype;             // J
    void* xb;                     // [groups][K][G] T
    int xb_smem;                  // one-fit groups: a CTA keeps its rows' linear predictors in shared
                                  // memory when they fit (the capacity in rows), 0 = global memory
    const void* w;                // [groups][K][G] T
    double* denom;                // grouped: [groups][S][G]
    const double* nw;             // grouped: [groups][S][G]
    const double* xjy;            // [F][J]
    double* beta;                 // [F][J]
    double* hdelta;               // [F][J]
    const double* variance;       // [F]
    const double* llfixed;        // [F]
    const int* active;            // [F] 0 for padding fits
    const signed char* fold;      // K fold id per row (CV grid) or null
    const int* fitfold;           // [F] held-out fold of each fit (CV grid)
    const int* run_len;           // J: columns in the batch starting here (1 = alone), 0 inside a batch
    const int* run_lvl;           // J: level of the column within its batch
    const int* run_dr0;           // J: first shared row of the batch starting here (into drow)
    const int* run_nd;            // J: shared rows of that batch
    const int* drow;              // shared row ids
    const int* de_ptr;            // J+1: entries of column j on shared rows
    const int* de_d;              // shared-row slot | (column within the batch << 8)
    const double* de_x;           // the entry's value (1 for indicator columns)
    int conv;
    double tol;
    int max_iter;
    int* out_iter;                // [F]
    int* out_flag;                // [F]
    double* out_obj;              // [F]
    unsigned long long* counters; // [3 + groups]: grad fit-entries, update fit-entries, steps, then
                                  // per group the bytes of row ids / values it streamed
};

template <class T>
struct Kahan {
    T s = 0, c = 0;
    __device__ __forceinline__ void add(T v) {
        const T yv = v - c;
        const T t = s + yv;
        c = (t - s) - yv;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

template <>
struct Kahan<double> {
    double s = 0;
    __device__ __forceinline__ void add(double v) { s += v; }
    __device__ __forceinline__ double value() const { return s; }
};

__device__ __forceinline__ float fexp(float x) { return __expf(x); }
__device__ __forceinline__ double fexp(double x) { return exp(x); }
__device__ __forceinline__ float flog(float x) { return __logf(x); }
__device__ __forceinline__ double flog(double x) { return log(x); }

// sum (a, b) over the CTA's slots that share this thread's fit lane; result
// for lane f lands in out[f] (threads < G then read it)
template <int G>
__device__ __forceinline__ void block_reduce_lanes(double a, double b, double2* out, double2 (*scratch)[G]) {
    for (int o = G; o < 32; o <<= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane < G) scratch[wid][lane] = make_double2(a, b);
    __syncthreads();
    if (threadIdx.x < G) {
        double sa = 0.0, sb = 0.0;
        for (int q = 0; q < kBT / 32; ++q) {
            sa += scratch[q][threadIdx.x].x;
            sb += scratch[q][threadIdx.x].y;
        }
        out[threadIdx.x] = make_double2(sa, sb);
    }
    __syncthreads();
}

// weight of (row k, fit lane) for one group: from the per-fit weight array,
// or, for a CV grid, 1 when the row's fold is not the fit's held-out fold
template <class T, int WM>
__device__ __forceinline__ T row_weight(const T* wg, const signed char* fold, int fitfold, int k, int G, int fl) {
    if (WM == 1) return (fitfold >= -1 && (int)__ldg(fold + k) != fitfold) ? T(1) : T(0);
    return wg[(size_t)k * G + fl];
}

template <class T, int MODEL, int G, int WM>
__device__ __forceinline__ double objective_partial(const BatchArgs& A, int grp, int r0, int r1, int s0, int s1,
                                                    const T* xbg, const T* wg, int fitfold, int fl, bool use_ll) {
    Kahan<double> acc;
    const int slot = threadIdx.x / G, nslots = kBT / G;
    for (int k = r0 + slot; k < r1; k += nslots) {
        const double v = (double)xbg[(size_t)k * G + fl];
        const double wt = (double)row_weight<T, WM>(wg, A.fold, fitfold, k, G, fl);
        const double yk = A.y[k];
        if (!use_ll) {
            acc.add(v * yk * wt);                                       // getGradientObjective
        } else {
            const int yi = (int)yk;                                     // logLikeNumeratorContrib
            double c = yi * v * wt;
            if (MODEL == CYC_LR) c -= wt * log(1.0 + exp(v));          // nw * log(denom), denom = 1 + exb
            if (MODEL == CYC_PR) c -= wt * exp(v);                      // nw * denom
            acc.add(c);
        }
    }
    if (use_ll && (MODEL == CYC_CLR || MODEL == CYC_CPR)) {
        const double* dg = A.denom + (size_t)grp * A.S * G;
        const double* ng = A.nw + (size_t)grp * A.S * G;
        for (int s = s0 + slot; s < s1; s += nslots) acc.add(-ng[(size_t)s * G + fl] * log(dg[(size_t)s * G + fl]));
    }
    return acc.value();
}

// per-row contribution to (gradient, Hessian) of an independent-rows model
// (Logistic / PoissonRegression::incrementGradientAndHessian,
// ModelSpecifics.h:540-568, 1508-1543); the logistic probability is formed as
// 1 / (1 + exp(-xb)), which equals exb / (1 + exb) without overflowing
// the row's mean under the model: the logistic probability, or exp(xb)
template <class T, int MODEL>
__device__ __forceinline__ T row_mean(T v) {
    if (MODEL == CYC_LR) return T(1) / (T(1) + fexp(-v));
    return fexp(v);
}

// (gradient, Hessian) terms of one entry from its row's mean
template <class T, int MODEL>
__device__ __forceinline__ void mean_terms(T m, T x, T wt, bool ind, T& gi, T& hi) {
    if (MODEL == CYC_LR) {
        const T g1 = m * x;
        gi = wt * g1;
        hi = wt * (ind ? g1 * (T(1) - g1) : x * x * m * (T(1) - m));
    } else {
        const T n1 = m * x;
        gi = wt * n1;
        hi = wt * (ind ? n1 : n1 * x);
    }
}

template <class T, int MODEL>
__device__ __forceinline__ void row_terms(T v, T x, T wt, bool ind, T& gi, T& hi) {
    mean_terms<T, MODEL>(row_mean<T, MODEL>(v), x, wt, ind, gi, hi);
}

// (callers skip rows of weight zero: their terms are exactly zero, and the
// exp() they would cost is the FP64 pipe's largest load)
template <class T, int MODEL>
__device__ __forceinline__ void row_gh(T v, T x, T wt, bool ind, Kahan<T>& ag, Kahan<T>& ah) {
    T gi, hi;
    row_terms<T, MODEL>(v, x, wt, ind, gi, hi);
    ag.add(gi);
    ah.add(hi);
}

// xb + delta * x as one fused multiply-add, the same wherever a batch
// replays an update (the owning CTA and every CTA's copy of a shared row)
__device__ __forceinline__ float upd_fma(float d, float x, float v) { return __fmaf_rn(d, x, v); }
__device__ __forceinline__ double upd_fma(double d, double x, double v) { return __fma_rn(d, x, v); }

// N consecutive values of one row of the [K][G] layout (16-byte aligned
// when N * sizeof(T) is a multiple of 16)
template <class T, int N>
__device__ __forceinline__ void load_row(const T* p, T (&v)[N]) {
    if constexpr (sizeof(T) == 4 && N % 4 == 0) {
        #pragma unroll
        for (int i = 0; i < N / 4; ++i) {
            const float4 q = reinterpret_cast<const float4*>(p)[i];
            v[4 * i] = q.x; v[4 * i + 1] = q.y; v[4 * i + 2] = q.z; v[4 * i + 3] = q.w;
        }
    } else if constexpr (sizeof(T) == 8 && N % 2 == 0) {
        #pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            const double2 q = reinterpret_cast<const double2*>(p)[i];
            v[2 * i] = q.x; v[2 * i + 1] = q.y;
        }
    } else {
        #pragma unroll
        for (int i = 0; i < N; ++i) v[i] = p[i];
    }
}

template <class T, int N>
__device__ __forceinline__ void store_row(T* p, const T (&v)[N]) {
    if constexpr (sizeof(T) == 4 && N % 4 == 0) {
        #pragma unroll
        for (int i = 0; i < N / 4; ++i)
            reinterpret_cast<float4*>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    } else if constexpr (sizeof(T) == 8 && N % 2 == 0) {
        #pragma unroll
        for (int i = 0; i < N / 2; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
    } else {
        #pragma unroll
        for (int i = 0; i < N; ++i) p[i] = v[i];
    }
}

// Thread-per-row layout of one group's G fits: a row's linear predictors
// are split into TPR parts of FPT = 4 fits (16 bytes in FP32, one 32-byte
// sector in FP64), and each thread holds R = 2 rows' parts at a time.  The
// layout is a parameter of the caller (a CTA streaming one long column,
// BLOCK, or a warp taking one short column of a batch); wider parts or more
// rows per thread measured slower on B200 here: the registers they take make
// the rest of the persistent kernel spill.
template <class T, int G, bool BLOCK>
struct RowLayout {
    static constexpr int FPT = (G % 4 != 0) ? G : 4;
    static constexpr int TPR = G / FPT;
    static constexpr int R = 2;
    // row parts in flight per thread when rows arrive by cp.async (their
    // slots fit in kAsyncBytes per CTA)
    static constexpr int D = 4;
    static_assert(kBT * D * FPT * sizeof(T) <= kAsyncBytes, "cp.async slots exceed their shared memory");
};

// 16-byte asynchronous copies global -> shared (L2 only), one group per row
// slot; a thread waits for its own copies only.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// one row part (FPT values, a multiple of 16 bytes) into a slot
template <class T, int FPT>
__device__ __forceinline__ void issue_part(T* slot, const T* src) {
    static_assert((FPT * sizeof(T)) % 16 == 0, "row parts are whole 16-byte pieces");
    #pragma unroll
    for (int i = 0; i < (int)(FPT * sizeof(T)) / 16; ++i)
        cp_async16(reinterpret_cast<char*>(slot) + 16 * i, reinterpret_cast<const char*>(src) + 16 * i);
}

// Warp sum of per-lane (g[f], h[f]), f < FPT (the lane's part lane % TPR of
// the fits), by a butterfly reduce-scatter: each level halves the values a
// lane carries (2 FPT values: FPT + FPT/2 + ... + 1 shuffles per lane, then
// one more).  Returns the sum of this lane's value and sets `fit` (within the
// group) and `is_h`; `holder` marks one of the two lanes that hold it.
// Fixed order: deterministic.
template <int FPT, int TPR>
__device__ __forceinline__ double warp_reduce_rows(const double (&g)[FPT], const double (&h)[FPT], int& fit,
                                                   bool& is_h, bool& holder) {
    constexpr unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double v[2 * FPT];
    #pragma unroll
    for (int f = 0; f < FPT; ++f) { v[f] = g[f]; v[FPT + f] = h[f]; }
    int vi = 0;
    #pragma unroll
    for (int half = FPT, off = 16; half >= 1; half >>= 1, off >>= 1) {
        const bool up = (lane & off) != 0;
        #pragma unroll
        for (int i = 0; i < half; ++i) {
            const double send = up ? v[i] : v[i + half];
            const double keep = up ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(full, send, off);
        }
        vi += up ? half : 0;
    }
    v[0] += __shfl_xor_sync(full, v[0], TPR);
    fit = (lane % TPR) * FPT + (vi % FPT);
    is_h = vi >= FPT;
    holder = (lane & TPR) == 0;
    return v[0];
}

// Block sum of per-thread (g, h) parts into out[f] = (g, h): warp sums, then
// the warps' sums in warp order.  Deterministic.
template <int G, int FPT, int TPR>
__device__ __forceinline__ void block_reduce_rows(const double (&g)[FPT], const double (&h)[FPT], double2* out,
                                                  double* scr /* [kBT/32][2G] */) {
    const int wid = threadIdx.x >> 5;
    int fit;
    bool is_h, holder;
    const double v = warp_reduce_rows<FPT, TPR>(g, h, fit, is_h, holder);
    if (holder) scr[wid * 2 * G + (is_h ? G : 0) + fit] = v;
    __syncthreads();
    if (threadIdx.x < 2 * G) {
        double s = 0.0;
        for (int q = 0; q < kBT / 32; ++q) s += scr[q * 2 * G + threadIdx.x];
        if (threadIdx.x < G) out[threadIdx.x].x = s;
        else out[threadIdx.x - G].y = s;
    }
    __syncthreads();
}

// Where the entries of one column in this CTA's rows come from: positions
// [e0, e1) of the column (row ids `cidx`, values `cval`), or, when staged in
// shared memory, sidx / sx [0, e1 - e0) (values from `cval` when sx is null).
template <class T>
struct ColRows {
    const int* cidx;
    const double* cval;
    const int* sidx;
    const T* sx;
    int e0, e1;
    bool dense, ind;
    __device__ __forceinline__ void get(int e, int& k, T& x) const {
        if (e >= e1) { k = -1; x = T(1); return; }
        if (sidx) {
            k = sidx[e - e0];
            x = ind ? T(1) : (sx ? sx[e - e0] : (T)__ldg(cval + e));
        } else {
            k = dense ? e : __ldg(cidx + e);
            x = ind ? T(1) : (T)__ldg(cval + e);
        }
    }
};

// Gradient and Hessian terms of the group's fits over the entries of a column
// (an independent-rows model), by the STRIDE threads t0 = 0 .. STRIDE-1:
// thread t takes rows t / TPR, t / TPR + STRIDE / TPR, ... and fits part
// t % TPR of each.  Two-stage pipeline per thread: a row's id (and value,
// fold id) loads 2D rows ahead; its part of the linear predictors arrives by
// cp.async into the thread's D slots (`abuf`) D rows ahead of the one being
// summed.  `wmask[fold]` holds the fits that train on rows of that fold (CV
// grid); `done` the fits that have converged (skipped).
template <class T, int MODEL, int G, int WM, int STRIDE>
__device__ __forceinline__ void rows_gh(const ColRows<T>& c, int t0, const T* xbg, const T* wg,
                                        const signed char* fold, const unsigned char* wmask, unsigned done, T* abuf,
                                        double (&g)[RowLayout<T, G, STRIDE == kBT>::FPT],
                                        double (&h)[RowLayout<T, G, STRIDE == kBT>::FPT]) {
    using Lay = RowLayout<T, G, STRIDE == kBT>;
    constexpr int FPT = Lay::FPT, TPR = Lay::TPR, D = Lay::D, RS = STRIDE / TPR;
    const int f0 = (t0 % TPR) * FPT;
    const unsigned dn = done >> f0;
    Kahan<T> ag[FPT], ah[FPT];
    int base = c.e0 + t0 / TPR;
    int k[D], kn[D], fd[D];                  // rows in the slots, and the rows after them
    T x[D], xn[D];
    T w[D][FPT];
    auto fetch = [&](int s, int e) { c.get(e, kn[s], xn[s]); };   // stage 1: id and value
    auto issue = [&](int s) {                // stage 2: the row part into slot s, its fold id
        k[s] = kn[s];
        x[s] = xn[s];
        fd[s] = 0;
        if (k[s] >= 0) {
            issue_part<T, FPT>(abuf + s * FPT, xbg + (size_t)k[s] * G + f0);
            if (WM == 0) load_row<T, FPT>(wg + (size_t)k[s] * G + f0, w[s]);
            else fd[s] = (int)__ldg(fold + k[s]);
        }
        cp_async_commit();
    };
    #pragma unroll
    for (int s = 0; s < D; ++s) fetch(s, base + s * RS);
    #pragma unroll
    for (int s = 0; s < D; ++s) {
        issue(s);
        fetch(s, base + (D + s) * RS);
    }
    for (; base < c.e1; base += D * RS) {
        #pragma unroll
        for (int s = 0; s < D; ++s) {
            cp_async_wait<D - 1>();
            if (k[s] >= 0) {
                T v[FPT];
                load_row<T, FPT>(abuf + s * FPT, v);
                const unsigned wm = (WM == 1) ? (unsigned)wmask[fd[s]] >> f0 : 0u;
                #pragma unroll
                for (int f = 0; f < FPT; ++f) {
                    if ((dn >> f) & 1u) continue;
                    const T wt = (WM == 1) ? (((wm >> f) & 1u) ? T(1) : T(0)) : w[s][f];
                    if (wt != T(0)) row_gh<T, MODEL>(v[f], x[s], wt, c.ind, ag[f], ah[f]);
                }
            }
            issue(s);
            fetch(s, base + (2 * D + s) * RS);
        }
    }
    cp_async_wait<0>();
    #pragma unroll
    for (int f = 0; f < FPT; ++f) { g[f] = ag[f].value(); h[f] = ah[f].value(); }
}

// updateXBeta over the entries of a column by the STRIDE threads t0 (same
// split and the same two-stage pipeline as rows_gh; the new values are stored
// from registers)
template <class T, int G, int STRIDE>
__device__ __forceinline__ void rows_update(const ColRows<T>& c, int t0, T* xbg, const T (&d)[G], T* abuf) {
    using Lay = RowLayout<T, G, STRIDE == kBT>;
    constexpr int FPT = Lay::FPT, TPR = Lay::TPR, D = Lay::D, RS = STRIDE / TPR;
    const int f0 = (t0 % TPR) * FPT;
    bool moved = false;                     // a part whose fits all kept their coefficients stays
    #pragma unroll
    for (int f = 0; f < FPT; ++f) moved |= (d[f0 + f] != T(0));
    if (!moved) return;
    int base = c.e0 + t0 / TPR;
    int k[D], kn[D];
    T x[D], xn[D];
    auto fetch = [&](int s, int e) { c.get(e, kn[s], xn[s]); };
    auto issue = [&](int s) {
        k[s] = kn[s];
        x[s] = xn[s];
        if (k[s] >= 0) issue_part<T, FPT>(abuf + s * FPT, xbg + (size_t)k[s] * G + f0);
        cp_async_commit();
    };
    #pragma unroll
    for (int s = 0; s < D; ++s) fetch(s, base + s * RS);
    #pragma unroll
    for (int s = 0; s < D; ++s) {
        issue(s);
        fetch(s, base + (D + s) * RS);
    }
    for (; base < c.e1; base += D * RS) {
        #pragma unroll
        for (int s = 0; s < D; ++s) {
            cp_async_wait<D - 1>();
            if (k[s] >= 0) {
                T v[FPT];
                load_row<T, FPT>(abuf + s * FPT, v);
                #pragma unroll
                for (int f = 0; f < FPT; ++f) v[f] = upd_fma(d[f0 + f], x[s], v[f]);
                store_row<T, FPT>(xbg + (size_t)k[s] * G + f0, v);
            }
            issue(s);
            fetch(s, base + (2 * D + s) * RS);
        }
    }
    cp_async_wait<0>();
}

// updateXBeta of a batch's columns over this CTA's rows, flat: item i is part
// i % TPR of entry i / TPR of the concatenated columns (offsets `boff`, empty
// for columns without a step), U items per thread in flight.  Entries on the
// batch's shared rows (`drow`, nd of them) are left to their owner.  No two
// items touch the same (row, part): a row outside `drow` is in one column.
template <class T, int G>
__device__ __forceinline__ void batch_update(T* xbg, const int* idx, const double* val, const int* sidx, const T* sx,
                                             const long long* cp, const long long* vp, const int* e0, const int* off,
                                             const int* fmt, int q, int L, const int* boff,
                                             const double (*dr)[G], const int* drow, int nd) {
    using Lay = RowLayout<T, G, false>;
    constexpr int FPT = Lay::FPT, TPR = Lay::TPR, U = 4;
    unsigned bloom = 0;
    for (int d = 0; d < nd; ++d) bloom |= 1u << (drow[d] & 31);
    const int items = boff[L] * TPR;
    for (int i0 = threadIdx.x; i0 < items; i0 += U * kBT) {
        int k[U], w[U];
        T x[U];
        #pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * kBT;
            k[u] = -1;
            w[u] = 0;
            x[u] = T(1);
            if (i >= items) continue;
            const int it = i / TPR;
            int c = 0;
            while (it >= boff[c + 1]) ++c;
            const int qq = q + c, e = it - boff[c];
            w[u] = c;
            if (off[qq] >= 0) {
                k[u] = sidx[off[qq] + e];
                if (fmt[qq] == CYC_SPARSE) x[u] = sx ? sx[off[qq] + e] : (T)__ldg(val + vp[qq] + e0[qq] + e);
            } else {
                k[u] = __ldg(idx + cp[qq] + e0[qq] + e);
                if (fmt[qq] == CYC_SPARSE) x[u] = (T)__ldg(val + vp[qq] + e0[qq] + e);
            }
            if ((bloom >> (k[u] & 31)) & 1u) {
                bool sh = false;
                for (int d = 0; d < nd; ++d) sh |= (drow[d] == k[u]);
                if (sh) k[u] = -1;
            }
            bool moved = false;             // a part whose fits all kept their coefficients stays
            const int f0 = (i % TPR) * FPT;
            #pragma unroll
            for (int f = 0; f < FPT; ++f) moved |= (dr[c][f0 + f] != 0.0);
            if (!moved) k[u] = -1;
        }
        T v[U][FPT];
        #pragma unroll
        for (int u = 0; u < U; ++u)
            if (k[u] >= 0) load_row<T, FPT>(xbg + (size_t)k[u] * G + ((i0 + u * kBT) % TPR) * FPT, v[u]);
        #pragma unroll
        for (int u = 0; u < U; ++u) {
            if (k[u] < 0) continue;
            const int f0 = ((i0 + u * kBT) % TPR) * FPT;
            #pragma unroll
            for (int f = 0; f < FPT; ++f) v[u][f] = upd_fma((T)dr[w[u]][f0 + f], x[u], v[u][f]);
            store_row<T, FPT>(xbg + (size_t)k[u] * G + f0, v[u]);
        }
    }
}

// The batch cache: a batch of short columns whose entries in this CTA's rows
// number at most kRows (the planner caps batches so) is gathered once into
// shared memory -- every entry's row of linear predictors (all G fits, by
// 16-byte cp.async), its row id, value and fold id -- with all copies in
// flight at once, so the batch pays one memory round trip; the gradient
// partials then read shared memory and the update writes the new values from
// it without reading global memory again.  It occupies the bytes the
// cp.async row slots of the single-column path use (kAsyncBytes).
template <class T, int G>
struct BatchCache {
    static constexpr int kPieces = (int)(G * sizeof(T)) / 16;          // 16-byte pieces of a row
    static constexpr int kEntryBytes = (int)(G * sizeof(T) + sizeof(int) + sizeof(T) + 1);
    static constexpr int kRows = (kAsyncBytes / kEntryBytes) / 32 * 32;
    static_assert(kPieces >= 1 && (G * sizeof(T)) % 16 == 0, "rows are whole 16-byte pieces");
    static_assert(kRows * kEntryBytes <= kAsyncBytes, "the batch cache exceeds its shared memory");
    T* v;                  // [kRows][G] linear predictors at the batch's start
    int* row;              // [kRows] row ids
    T* x;                  // [kRows] values (1 for indicators)
    unsigned char* fold;   // [kRows] fold ids (CV grid)
    __device__ explicit BatchCache(void* base) {
        unsigned char* b = static_cast<unsigned char*>(base);
        v = reinterpret_cast<T*>(b);
        row = reinterpret_cast<int*>(b + (size_t)kRows * G * sizeof(T));
        x = reinterpret_cast<T*>(b + (size_t)kRows * (G * sizeof(T) + sizeof(int)));
        fold = b + (size_t)kRows * (G * sizeof(T) + sizeof(int) + sizeof(T));
    }
};

// Gather the batch's entries in this CTA's rows (columns q .. q+L-1, entry
// offsets boff[0..L]) into the cache; returns after every copy has landed
// and the CTA has synchronised.
template <class T, int G, int WM>
__device__ __forceinline__ void batch_gather(const BatchCache<T, G>& bc, const T* xbg, const int* idx,
                                             const double* val, const signed char* fold, const int* sidx,
                                             const long long* cp, const long long* vp, const int* e0,
                                             const int* off, const int* fmt, int q, const int* boff, int L) {
    constexpr int P = BatchCache<T, G>::kPieces;
    constexpr int PV = 16 / (int)sizeof(T);
    const int E = boff[L];
    for (int i = threadIdx.x; i < E * P; i += kBT) {
        const int e = i / P, p = i % P;
        int w = 0;
        while (e >= boff[w + 1]) ++w;
        const int qq = q + w, el = e - boff[w];
        const int k = off[qq] >= 0 ? sidx[off[qq] + el] : __ldg(idx + cp[qq] + e0[qq] + el);
        cp_async16(bc.v + (size_t)e * G + p * PV, xbg + (size_t)k * G + p * PV);
    }
    cp_async_commit();
    for (int e = threadIdx.x; e < E; e += kBT) {
        int w = 0;
        while (e >= boff[w + 1]) ++w;
        const int qq = q + w, el = e - boff[w];
        const int k = off[qq] >= 0 ? sidx[off[qq] + el] : __ldg(idx + cp[qq] + e0[qq] + el);
        bc.row[e] = k;
        bc.x[e] = fmt[qq] == CYC_SPARSE ? (T)__ldg(val + vp[qq] + e0[qq] + el) : T(1);
        if (WM == 1) bc.fold[e] = (unsigned char)__ldg(fold + k);
    }
    cp_async_wait<0>();
    __syncthreads();
}

// Gradient and Hessian terms of the group's fits over cache entries
// [b0, b1) (one column) by STRIDE threads (a warp taking one column of a
// batch, or the CTA taking a column alone): thread t takes entries
// b0 + t / TPR, b0 + t / TPR + STRIDE / TPR, ... and fits part t % TPR of
// each -- the entries and order rows_gh gives them, so the sums are the
// same.
template <class T, int MODEL, int G, int WM, int STRIDE = 32>
__device__ __forceinline__ void cache_gh(const BatchCache<T, G>& bc, int b0, int b1, bool ind, const T* wg,
                                         const unsigned char* wmask, unsigned done,
                                         double (&g)[RowLayout<T, G, STRIDE == kBT>::FPT],
                                         double (&h)[RowLayout<T, G, STRIDE == kBT>::FPT]) {
    using Lay = RowLayout<T, G, STRIDE == kBT>;
    constexpr int FPT = Lay::FPT, TPR = Lay::TPR, RS = STRIDE / TPR;
    const int lane = STRIDE == kBT ? (int)threadIdx.x : (int)(threadIdx.x & 31);
    const int f0 = (lane % TPR) * FPT;
    const unsigned dn = done >> f0;
    Kahan<T> ag[FPT], ah[FPT];
    for (int e = b0 + lane / TPR; e < b1; e += RS) {
        T v[FPT];
        load_row<T, FPT>(bc.v + (size_t)e * G + f0, v);
        const T x = bc.x[e];
        T w[FPT];
        if (WM == 0) load_row<T, FPT>(wg + (size_t)bc.row[e] * G + f0, w);
        const unsigned wm = (WM == 1) ? (unsigned)wmask[bc.fold[e]] >> f0 : 0u;
        #pragma unroll
        for (int f = 0; f < FPT; ++f) {
            if ((dn >> f) & 1u) continue;
            const T wt = (WM == 1) ? (((wm >> f) & 1u) ? T(1) : T(0)) : w[f];
            if (wt != T(0)) row_gh<T, MODEL>(v[f], x, wt, ind, ag[f], ah[f]);
        }
    }
    #pragma unroll
    for (int f = 0; f < FPT; ++f) { g[f] = ag[f].value(); h[f] = ah[f].value(); }
}

// updateXBeta of a cached batch over this CTA's rows: each (entry, part) of a
// column with a step writes its new values from the cache; entries on the
// batch's shared rows (`drow`, nd of them) are left to their owner.  No two
// items touch the same (row, part): a row outside `drow` is in one column.
template <class T, int G>
__device__ __forceinline__ void cache_update(const BatchCache<T, G>& bc, T* xbg, const int* boff, int L,
                                             const double (*dr)[G], const int* drow, int nd) {
    using Lay = RowLayout<T, G, false>;
    constexpr int FPT = Lay::FPT, TPR = Lay::TPR;
    unsigned bloom = 0;
    for (int d = 0; d < nd; ++d) bloom |= 1u << (drow[d] & 31);
    const int items = boff[L] * TPR;
    for (int i = threadIdx.x; i < items; i += kBT) {
        const int e = i / TPR, f0 = (i % TPR) * FPT;
        int w = 0;
        while (e >= boff[w + 1]) ++w;
        bool moved = false;                 // a part whose fits all kept their coefficients stays
        #pragma unroll
        for (int f = 0; f < FPT; ++f) moved |= (dr[w][f0 + f] != 0.0);
        if (!moved) continue;
        const int k = bc.row[e];
        if ((bloom >> (k & 31)) & 1u) {
            bool sh = false;
            for (int d = 0; d < nd; ++d) sh |= (drow[d] == k);
            if (sh) continue;
        }
        T v[FPT];
        load_row<T, FPT>(bc.v + (size_t)e * G + f0, v);
        const T x = bc.x[e];
        #pragma unroll
        for (int f = 0; f < FPT; ++f) v[f] = upd_fma((T)dr[w][f0 + f], x, v[f]);
        store_row<T, FPT>(xbg + (size_t)k * G + f0, v);
    }
}

// Items of one coordinate a thread keeps in registers between the gradient
// and the update: columns with at most kRegItems * (kBT / G) entries in this
// CTA's rows take this path (one load round trip, no reload for the update);
// longer ones stream through twice.
constexpr int kRegItems = 8;
// coordinates staged in shared memory at a time
constexpr int kChunk = 128;
// row ids of short columns staged per chunk (dynamic shared memory)
constexpr int kStage = 4096;

// Columns processed together: consecutive short columns whose rows are
// pairwise disjoint (planned on the host, ConflictFreeRuns) form a run of at
// most kRunMax columns.  For independent-rows models the gradient of a column
// depends only on the linear predictor of its own rows, so the columns of a
// run see exactly the state the serial coordinate loop would show them, and
// their updates touch disjoint rows: the run gives the serial CCD result while
// paying for one load round trip and one cluster barrier.  Warp w of every
// CTA takes column w of the run.
constexpr int kRunMax = kBT / 32;
// entries per slot of a run column (a warp has 32/G slots)
constexpr int kRunItems = 8;
// With G = 8 fits per group (independent-rows models) a batch may share rows
// between its columns: at most kDirtyMax such rows, replayed serially (see
// k_batch).  Columns of at most kBatchCap entries in every CTA's rows join.
constexpr int kDirtyMax = 32;
constexpr int kBatchCap = 256;

// The batch shape of an 8-fit group's plan: columns with at most `cap`
// entries in every CTA's rows are short (batched, a warp per column; the
// rest stream through the whole CTA), a batch shares at most `dmax` rows
// between its columns and replays at most `lvl` levels.  The defaults are
// the largest the kernel's shared memory allows; the shape tuner
// (tuned_shape) may pick smaller ones for a problem.
struct BatchShape {
    int cap = 256, dmax = 32, lvl = 8;
    bool operator==(const BatchShape& o) const { return cap == o.cap && dmax == o.dmax && lvl == o.lvl; }
};
// levels of the serial replay a batch may have (each costs a step chain)
constexpr int kLevelMax = kRunMax;

// 8-fit groups of independent-rows models take the thread-per-row paths
template <int MODEL, int G>
constexpr bool row_stream() { return G == 8 && MODEL != CYC_CLR && MODEL != CYC_CPR; }

// bytes after the staged row ids: staged values, or the cp.async row slots
template <class T, int MODEL, int G>
constexpr size_t staged_value_bytes() { return row_stream<MODEL, G>() ? (size_t)kAsyncBytes : kStage * sizeof(T); }

template <class T, int MODEL, int G, int WM>
__global__ void __launch_bounds__(kBT, 2) k_batch(const BatchArgs A) {
    cg::cluster_group cluster = cg::this_cluster();
    const int C = A.C;
    const int rank = (int)cluster.block_rank();
    const int grp = blockIdx.x / C;
    const int r0 = A.rpart[rank], r1 = A.rpart[rank + 1];
    const bool grouped = (MODEL == CYC_CLR || MODEL == CYC_CPR);
    // independent rows, 8 fits per group: columns stream thread per row (all
    // fits of a row by vector loads) and short columns go in batches
    constexpr bool kRowStream = row_stream<MODEL, G>();
    using LayW = RowLayout<T, G, false>;   // a warp per column (batches)
    using LayB = RowLayout<T, G, true>;    // the CTA per column (single columns)
    // strata of my rows (partition boundaries are stratum starts); none if my range is empty
    const int s0 = (grouped && r0 < r1) ? A.strat[r0] : 0;
    const int s1 = (grouped && r0 < r1) ? (r1 >= A.K ? A.S : A.strat[r1]) : 0;
    T* xbg = (T*)A.xb + (size_t)grp * A.K * G;
    const T* wg = (WM == 0) ? (const T*)A.w + (size_t)grp * A.K * G : nullptr;
    double* dg = grouped ? A.denom + (size_t)grp * A.S * G : nullptr;
    const double* ng = grouped ? A.nw + (size_t)grp * A.S * G : nullptr;
    const int fl = threadIdx.x % G;
    const int slot = threadIdx.x / G;
    constexpr int NS = kBT / G;
    constexpr int WS = 32 / G;                // slots per warp
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wslot = lane / G;
    const int fg = grp * G;                   // first fit of the group
    const int fitfold = (WM == 1) ? A.fitfold[fg + fl] : 0;

    // every CTA's (g, h) partials, pushed into each CTA of the cluster before
    // the barrier (double buffered by parity; one slot per column of a run)
    __shared__ double2 s_part[2][kMaxC][kRunMax][G];
    __shared__ double2 s_scr[kBT / 32][G];
    __shared__ double2 s_red[G];
    __shared__ double s_obj[2][kMaxC][G];
    __shared__ double s_delta[G];
    __shared__ double s_dr[kRunMax][G];
    __shared__ double s_last[G];
    __shared__ int s_done[G];
    __shared__ int s_flag[G];
    __shared__ int s_iter[G];
    __shared__ int s_all_done;
    // CV grid: the fits of the group that train on rows of fold v (bit f)
    __shared__ unsigned char s_wmask[128];
    // the open batch: its entries on shared rows (slot, value) per column, and
    // the shared rows' fold masks
    __shared__ int s_bde_ptr[kRunMax + 1];
    __shared__ int s_bde_d[kRunMax * kDirtyMax];
    __shared__ double s_bde_x[kRunMax * kDirtyMax];
    __shared__ unsigned char s_dwm[kDirtyMax];
    __shared__ int s_drow[kDirtyMax];
    __shared__ int s_boff[kRunMax + 1];
    __shared__ int s_cbo[kRunMax + 1];     // the open batch's columns in the batch cache
    // the current chunk of coordinates
    __shared__ int c_fmt[kChunk], c_fix[kChunk], c_pt[kChunk], c_e0[kChunk], c_e1[kChunk], c_run[kChunk];
    __shared__ unsigned char c_lfix[kChunk];   // fits holding the coordinate fixed (active-set passes)
    __shared__ int c_lvl[kChunk], c_nd[kChunk], c_dr0[kChunk], c_de0[kChunk + 1];
    __shared__ long long c_cp[kChunk], c_vp[kChunk];
    __shared__ int c_off[kChunk];          // staged offset of coordinate q, -1 if not staged
    __shared__ int c_sq[kChunk + 1];       // staged coordinates in order
    __shared__ int c_soff[kChunk + 1];     // their offsets (prefix sums)
    __shared__ int c_ns;
    // dynamic: this group's beta / trust region / XjY for the chunk (kept
    // identical in every CTA of the cluster), then the staged row ids / values
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    double (*c_beta)[G] = reinterpret_cast<double (*)[G]>(dyn_smem);
    double (*c_hd)[G] = reinterpret_cast<double (*)[G]>(dyn_smem + kChunk * G * sizeof(double));
    double (*c_xjy)[G] = reinterpret_cast<double (*)[G]>(dyn_smem + 2 * kChunk * G * sizeof(double));
    int* s_sidx = reinterpret_cast<int*>(dyn_smem + 3 * kChunk * G * sizeof(double));
    // staged values of short sparse columns (per-lane paths), or, for 8-fit
    // groups of independent-rows models, each thread's cp.async row slots
    T* s_sx = reinterpret_cast<T*>(dyn_smem + 3 * kChunk * G * sizeof(double) + kStage * sizeof(int));
    T* s_abuf = s_sx + (size_t)threadIdx.x * LayB::D * LayB::FPT;
    // the batch cache (8-fit groups of independent-rows models) shares those bytes
    const BatchCache<T, kRowStream ? G : 8> bcache(s_sx);
    // shared rows of the open batch: as pushed by their owners (by parity; the
    // replay then moves this CTA's copy of the current parity in place), their
    // model means at the batch's start and now, and their weights
    T* s_dirty = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(s_sx) + staged_value_bytes<T, MODEL, G>());
    T (*s_dst)[kDirtyMax][G] = reinterpret_cast<T (*)[kDirtyMax][G]>(s_dirty);
    T (*s_m0)[G] = reinterpret_cast<T (*)[G]>(s_dirty + 2 * kDirtyMax * G);
    T (*s_mc)[G] = reinterpret_cast<T (*)[G]>(s_dirty + 3 * kDirtyMax * G);
    T (*s_dw)[G] = reinterpret_cast<T (*)[G]>(s_dirty + 4 * kDirtyMax * G);
    // one-fit groups whose rows fit: the CTA's linear predictors live in
    // shared memory for the launch (every access to them is of the CTA's own
    // rows), loaded here and written back at the end; xbg then addresses
    // them by absolute row
    T* const xb_global = xbg;
    T* const s_xb = s_dirty + 5 * kDirtyMax * G;
    const bool xb_local = (G == 1) && A.xb_smem > 0 && (r1 - r0) <= A.xb_smem;
    if (xb_local) {
        for (int i = threadIdx.x; i < r1 - r0; i += kBT) s_xb[i] = xb_global[r0 + i];
        xbg = s_xb - r0;                 // rows r0 .. r1 - 1 only
    }

    const bool use_ll = (A.conv == CYC_CONV_MITTAL || A.conv == CYC_CONV_LANGE);
    if (threadIdx.x < G) {
        const int f = fg + threadIdx.x;
        s_done[threadIdx.x] = A.active[f] ? 0 : 1;
        s_flag[threadIdx.x] = CYC_SUCCESS;
        s_iter[threadIdx.x] = 0;
    }
    if (WM == 1 && threadIdx.x < 128) {
        unsigned m = 0;
        for (int f = 0; f < G; ++f) {
            const int ff = A.fitfold[fg + f];
            if (ff >= -1 && ff != (int)threadIdx.x) m |= 1u << f;
        }
        s_wmask[threadIdx.x] = (unsigned char)m;
    }
    __syncthreads();

    // initial objective (findMode :949-953)
    int opar = 0;
    {
        const double p = objective_partial<T, MODEL, G, WM>(A, grp, r0, r1, s0, s1, xbg, wg, fitfold, fl, use_ll);
        block_reduce_lanes<G>(p, 0.0, s_red, s_scr);
        if (threadIdx.x < G)
            for (int r = 0; r < C; ++r) *cluster.map_shared_rank(&s_obj[opar][rank][threadIdx.x], r) = s_red[threadIdx.x].x;
        if (C > 1) cluster.sync(); else __syncthreads();
        if (threadIdx.x < G) {
            const int f = fg + threadIdx.x;
            double o = 0.0;
            for (int r = 0; r < C; ++r) o += s_obj[opar][r][threadIdx.x];
            if (use_ll && (MODEL == CYC_PR || MODEL == CYC_CPR)) o += A.llfixed[f];
            if (A.conv == CYC_CONV_LANGE) {
                const double* bf = A.beta + (size_t)f * A.J;
                for (int j = 0; j < A.J; ++j) o += log_density(A.ptype[j], A.variance[f], bf[j]);
            }
            s_last[threadIdx.x] = o;
        }
        opar ^= 1;
    }
    __syncthreads();
    bool done_l = s_done[fl] != 0;   // this thread's fit lane has converged
    unsigned done_m = 0;             // all converged fits of the group (bit f)
    for (int f = 0; f < G; ++f) done_m |= (s_done[f] ? 1u : 0u) << f;
    const double var_l = A.variance[fg + fl];
    const double lam_l = sqrt(2.0 / var_l);      // LaplacePrior rate, :282-292

    unsigned long long n_grad = 0, n_upd = 0, n_steps = 0, n_idx = 0;
    int par = 0;
    for (int it = 1; it <= A.max_iter; ++it) {
      for (int j0 = 0; j0 < A.J; j0 += kChunk) {
        const int jn = min(kChunk, A.J - j0);
        // ccdUpdateBeta for fit f of chunk coordinate qq from its (g, h) summed
        // over the cluster; called by the thread whose fit lane is f
        auto coord_step = [&](int qq, int f, double g, double h) -> double {
            g -= c_xjy[qq][f];                             // :1181-1183
            if (s_done[f] || ((c_lfix[qq] >> f) & 1u)) return 0.0;
            if (h < 0.0) { g = 0.0; h = 0.0; }             // :1407-1410
            const double b = c_beta[qq][f];
            double hd = c_hd[qq][f];
            double dl = prior_delta_rate(c_pt[qq], var_l, lam_l, b, g, h);
            dl = apply_bounds(&hd, dl);
            c_hd[qq][f] = hd;
            if (dl != 0.0) c_beta[qq][f] = b + dl;
            return dl;
        };
        // work counters of L columns from chunk coordinate q0 (deltas in s_dr),
        // kept by thread 0 of every CTA over the CTA's own entries of each
        // column (shared memory only: the counters stay off the loads); the
        // CTAs' counts add up to the group's, the steps are counted by rank 0
        auto count_run = [&](int q0, int L) {
            int act = 0;
            for (int f = 0; f < G; ++f) act += !s_done[f];
            for (int w = 0; w < L; ++w) {
                int upd = 0;
                for (int f = 0; f < G; ++f) upd += (s_dr[w][f] != 0.0);
                const int fm = c_fmt[q0 + w];
                const bool dn = (fm == CYC_DENSE || fm == CYC_INTERCEPT);
                const bool in = (fm == CYC_INDICATOR || fm == CYC_INTERCEPT);
                const long long nn = c_e1[q0 + w] - c_e0[q0 + w];
                n_grad += (unsigned long long)(act * nn);
                n_upd += (unsigned long long)(upd * nn);
                if (rank == 0) n_steps += act;
                n_idx += (unsigned long long)(nn * ((dn ? 0 : 4) + (in ? 0 : 8)) * (1 + (upd ? 1 : 0)));
            }
        };
        // ---- stage the chunk (coalesced)
        for (int q = threadIdx.x; q < jn; q += kBT) {
            const int j = j0 + q;
            const int f0 = A.fmt[j];
            c_fmt[q] = f0;
            c_fix[q] = A.fixb[j];
            c_lfix[q] = A.lane_fix ? A.lane_fix[(size_t)grp * A.J + j] : 0;
            c_pt[q] = A.ptype[j];
            c_run[q] = A.run_len[j];
            c_lvl[q] = A.run_lvl[j];
            c_nd[q] = A.run_nd[j];
            c_dr0[q] = A.run_dr0[j];
            c_de0[q] = A.de_ptr[j];
            if (q == jn - 1) c_de0[jn] = A.de_ptr[j + 1];
            c_cp[q] = A.col_ptr[j];
            c_vp[q] = A.val_ptr[j];
            const bool dn = (f0 == CYC_DENSE || f0 == CYC_INTERCEPT);
            c_e0[q] = dn ? r0 : A.split[j * (C + 1) + rank];
            c_e1[q] = dn ? r1 : A.split[j * (C + 1) + rank + 1];
        }
        for (int q = threadIdx.x; q < jn * G; q += kBT) {
            const int ff = q / jn, jj = q % jn;
            const size_t o = (size_t)(fg + ff) * A.J + j0 + jj;
            c_beta[jj][ff] = A.beta[o];
            c_hd[jj][ff] = A.hdelta[o];
            c_xjy[jj][ff] = A.xjy[o];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int off = 0, ns = 0;
            for (int qq = 0; qq < jn; ++qq) {
                const int n = c_e1[qq] - c_e0[qq];
                const bool dn = (c_fmt[qq] == CYC_DENSE || c_fmt[qq] == CYC_INTERCEPT);
                // a column every running fit holds fixed (an active-set
                // pass) is not staged: it is skipped, or read in place
                const bool held = A.lane_fix && ((~(unsigned)c_lfix[qq] & ~done_m & ((1u << G) - 1u)) == 0);
                if (!grouped && !c_fix[qq] && !held && !dn && n > 0 && n <= kRegItems * NS && off + n <= kStage) {
                    c_off[qq] = off;
                    c_sq[ns] = qq;
                    c_soff[ns] = off;
                    ++ns;
                    off += n;
                } else {
                    c_off[qq] = -1;
                }
            }
            c_soff[ns] = off;
            c_ns = ns;
        }
        __syncthreads();
        {
            const int ns = c_ns, total = c_soff[ns];
            for (int t = threadIdx.x; t < total; t += kBT) {
                int lo = 0, hi = ns - 1;                 // last staged column with offset <= t
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (c_soff[mid] <= t) lo = mid;
                    else hi = mid - 1;
                }
                const int qq = c_sq[lo];
                const long long e = c_e0[qq] + (t - c_soff[lo]);
                s_sidx[t] = __ldg(A.idx + c_cp[qq] + e);
                if constexpr (!kRowStream) s_sx[t] = (c_fmt[qq] == CYC_SPARSE) ? (T)__ldg(A.val + c_vp[qq] + e) : T(1);
            }
        }
        __syncthreads();
        int q = 0;
        while (q < jn) {
            const int L = c_run[q];
            if (c_fix[q] || L <= 0) { ++q; continue; }
            if (A.lane_fix) {
                // a batch (or column) that every running fit holds fixed is
                // skipped: its steps would all be zero
                unsigned moving = 0;
                for (int w = 0; w < L; ++w) moving |= ~(unsigned)c_lfix[q + w];
                if ((moving & ~done_m & ((1u << G) - 1u)) == 0) { q += L; continue; }
            }
            if constexpr (kRowStream) {
            if (L > 1) {
                // ---- a batch of L short columns (planned: plan_runs); warp w takes column q + w
                const int nd = c_nd[q], dr0 = c_dr0[q];
                const int de0 = c_de0[q], nde = c_de0[q + L] - de0;
                // rows shared inside the batch: their owners push them (all G fits)
                // into every CTA; the weights of those rows are kept locally
                for (int t = threadIdx.x; t < nd * G; t += kBT) {
                    const int d = t / G, f = t % G;
                    const int k = __ldg(A.drow + dr0 + d);
                    if (k >= r0 && k < r1) {
                        const T v = xbg[(size_t)k * G + f];
                        for (int r = 0; r < C; ++r) *cluster.map_shared_rank(&s_dst[par][d][f], r) = v;
                    }
                    if (f == 0) s_drow[d] = k;
                    if (WM == 1) {
                        if (f == 0) s_dwm[d] = s_wmask[(int)__ldg(A.fold + k)];
                    } else {
                        s_dw[d][f] = wg[(size_t)k * G + f];
                    }
                }
                if (threadIdx.x <= L) s_bde_ptr[threadIdx.x] = c_de0[q + threadIdx.x] - de0;
                for (int t = threadIdx.x; t < nde; t += kBT) {
                    s_bde_d[t] = __ldg(A.de_d + de0 + t) & 0xff;
                    s_bde_x[t] = __ldg(A.de_x + de0 + t);
                }
                // the batch's entries in my rows, column by column (cache offsets)
                if (threadIdx.x <= L) {
                    int o = 0;
                    for (int w = 0; w < (int)threadIdx.x; ++w) o += c_e1[q + w] - c_e0[q + w];
                    s_cbo[threadIdx.x] = o;
                }
                __syncthreads();
                const bool cached = s_cbo[L] <= BatchCache<T, G>::kRows;
                if (cached)
                    batch_gather<T, G, WM>(bcache, xbg, A.idx, A.val, A.fold, s_sidx, c_cp, c_vp, c_e0, c_off, c_fmt,
                                           q, s_cbo, L);
                // gradient partials of every column from the state at the batch's start
                if (cached) {
                    if (warp < L) {
                        double g[LayW::FPT], h[LayW::FPT];
                        cache_gh<T, MODEL, G, WM>(bcache, s_cbo[warp], s_cbo[warp + 1], c_fmt[q + warp] == CYC_INDICATOR,
                                                  wg, s_wmask, done_m, g, h);
                        int fit;
                        bool is_h, holder;
                        const double v = warp_reduce_rows<LayW::FPT, LayW::TPR>(g, h, fit, is_h, holder);
                        if (holder) {
                            double* dst = is_h ? &s_part[par][rank][warp][fit].y : &s_part[par][rank][warp][fit].x;
                            for (int r = 0; r < C; ++r) *cluster.map_shared_rank(dst, r) = v;
                        }
                    }
                } else if (warp < L) {
                    const int qq = q + warp, so = c_off[qq];
                    double g[LayW::FPT], h[LayW::FPT];
                    const ColRows<T> cr{A.idx + c_cp[qq], A.val + c_vp[qq], so >= 0 ? s_sidx + so : nullptr,
                                        nullptr, c_e0[qq], c_e1[qq], false, c_fmt[qq] == CYC_INDICATOR};
                    rows_gh<T, MODEL, G, WM, 32>(cr, lane, xbg, wg, A.fold, s_wmask, done_m, s_abuf, g, h);
                    int fit;
                    bool is_h, holder;
                    const double v = warp_reduce_rows<LayW::FPT, LayW::TPR>(g, h, fit, is_h, holder);
                    if (holder) {
                        double* dst = is_h ? &s_part[par][rank][warp][fit].y : &s_part[par][rank][warp][fit].x;
                        for (int r = 0; r < C; ++r) *cluster.map_shared_rank(dst, r) = v;
                    }
                }
                if (C > 1) cluster.sync(); else __syncthreads();
                // the serial steps, replayed identically in every CTA: level by
                // level, a column's (g, h) is its partials plus, for each of its
                // entries on a shared row, the change of that row's terms since
                // the batch's start (zero unless an earlier column moved it).
                // The shared rows move in place in s_dst[par]; their means at the
                // start (s_m0) and now (s_mc) make a correction exp-free.
                if (nd > 0) {
                    for (int t = threadIdx.x; t < nd * G; t += kBT) {
                        const T m = row_mean<T, MODEL>(s_dst[par][t / G][t % G]);
                        s_m0[t / G][t % G] = m;
                        s_mc[t / G][t % G] = m;
                    }
                    __syncthreads();
                }
                int nlev = 1;
                for (int w = 0; w < L; ++w) nlev = max(nlev, c_lvl[q + w]);
                const int fw = lane % G, sl = lane / G;    // (fit, entry slot) inside a warp
                for (int lv = 1; lv <= nlev; ++lv) {
                    if (warp < L && c_lvl[q + warp] == lv) {
                        const int qq = q + warp;
                        const bool ind = c_fmt[qq] == CYC_INDICATOR;
                        const int i0 = s_bde_ptr[warp], i1 = s_bde_ptr[warp + 1];
                        double gc = 0.0, hc = 0.0;
                        if (!((done_m >> fw) & 1u))
                            for (int i = i0 + sl; i < i1; i += 32 / G) {
                                const int d = s_bde_d[i];
                                const T mc = s_mc[d][fw], m0 = s_m0[d][fw];
                                if (mc == m0) continue;        // not moved yet: the change is exactly zero
                                const T x = (T)s_bde_x[i];
                                const T wt = (WM == 1) ? (((s_dwm[d] >> fw) & 1u) ? T(1) : T(0)) : s_dw[d][fw];
                                T g1, h1, g0, h0;
                                mean_terms<T, MODEL>(mc, x, wt, ind, g1, h1);
                                mean_terms<T, MODEL>(m0, x, wt, ind, g0, h0);
                                gc += (double)g1 - (double)g0;
                                hc += (double)h1 - (double)h0;
                            }
                        for (int o = G; o < 32; o <<= 1) {
                            gc += __shfl_xor_sync(0xffffffffu, gc, o);
                            hc += __shfl_xor_sync(0xffffffffu, hc, o);
                        }
                        double dl = 0.0;
                        if (lane < G) {
                            // the CTAs' partials summed as a tree (the same order in every CTA)
                            double gv[kMaxC], hv[kMaxC];
                            #pragma unroll
                            for (int r = 0; r < kMaxC; ++r) {
                                const double2 pp = r < C ? s_part[par][r][warp][lane] : make_double2(0.0, 0.0);
                                gv[r] = pp.x;
                                hv[r] = pp.y;
                            }
                            #pragma unroll
                            for (int st = 1; st < kMaxC; st <<= 1) {
                                #pragma unroll
                                for (int r = 0; r + st < kMaxC; r += 2 * st) {
                                    gv[r] += gv[r + st];
                                    hv[r] += hv[r + st];
                                }
                            }
                            const double g = gv[0] + gc, h = hv[0] + hc;
                            dl = coord_step(qq, lane, g, h);
                            s_dr[warp][lane] = dl;
                        }
                        dl = __shfl_sync(0xffffffffu, dl, fw);
                        if (dl != 0.0)
                            for (int i = i0 + sl; i < i1; i += 32 / G) {
                                const int d = s_bde_d[i];
                                const T v = upd_fma((T)dl, (T)s_bde_x[i], s_dst[par][d][fw]);
                                s_dst[par][d][fw] = v;
                                s_mc[d][fw] = row_mean<T, MODEL>(v);
                            }
                    }
                    __syncthreads();
                }
                // updateXBeta of my rows in one pass over the batch's entries (all
                // threads, flat): a row that one column of the batch touches gets
                // that column's step; a row the batch shares gets its replayed
                // value, written by its owner.  Columns whose fits all kept their
                // coefficients are skipped.  A cached batch writes the new values
                // from the cache.
                if (cached) {
                    cache_update<T, G>(bcache, xbg, s_cbo, L, s_dr, s_drow, nd);
                } else {
                    if (threadIdx.x == 0) {
                        int o = 0;
                        for (int w = 0; w < L; ++w) {
                            s_boff[w] = o;
                            bool any = false;
                            for (int f = 0; f < G; ++f) any |= (s_dr[w][f] != 0.0);
                            if (any) o += c_e1[q + w] - c_e0[q + w];
                        }
                        s_boff[L] = o;
                    }
                    __syncthreads();
                    batch_update<T, G>(xbg, A.idx, A.val, s_sidx, nullptr, c_cp, c_vp, c_e0, c_off, c_fmt, q, L,
                                       s_boff, s_dr, s_drow, nd);
                }
                for (int t = threadIdx.x; t < nd * G; t += kBT) {
                    const int d = t / G, k = s_drow[d];
                    if (k >= r0 && k < r1) xbg[(size_t)k * G + t % G] = s_dst[par][d][t % G];
                }
                __syncthreads();
                if (threadIdx.x == 0) count_run(q, L);
                par ^= 1;
                q += L;
                continue;
            }
            // ---- a single column, thread per row (all G fits)
            {
                const int fmt = c_fmt[q], so = c_off[q];
                const bool dense = (fmt == CYC_DENSE || fmt == CYC_INTERCEPT);
                const ColRows<T> cr{A.idx + c_cp[q], A.val + c_vp[q], so >= 0 ? s_sidx + so : nullptr, nullptr,
                                    c_e0[q], c_e1[q], dense, fmt == CYC_INDICATOR || fmt == CYC_INTERCEPT};
                double g[LayB::FPT], h[LayB::FPT];
                // a column whose entries in my rows fit the batch cache is
                // gathered once and updated from the cache
                const int n1 = c_e1[q] - c_e0[q];
                const bool cached1 = !dense && n1 <= BatchCache<T, G>::kRows;
                if (cached1) {
                    if (threadIdx.x <= 1) s_cbo[threadIdx.x] = threadIdx.x ? n1 : 0;
                    __syncthreads();
                    batch_gather<T, G, WM>(bcache, xbg, A.idx, A.val, A.fold, s_sidx, c_cp, c_vp, c_e0, c_off,
                                           c_fmt, q, s_cbo, 1);
                    cache_gh<T, MODEL, G, WM, kBT>(bcache, 0, n1, cr.ind, wg, s_wmask, done_m, g, h);
                } else {
                    rows_gh<T, MODEL, G, WM, kBT>(cr, threadIdx.x, xbg, wg, A.fold, s_wmask, done_m, s_abuf, g, h);
                }
                block_reduce_rows<G, LayB::FPT, LayB::TPR>(g, h, s_red, reinterpret_cast<double*>(s_scr));
                if (threadIdx.x < G)
                    for (int r = 0; r < C; ++r) *cluster.map_shared_rank(&s_part[par][rank][0][threadIdx.x], r) = s_red[threadIdx.x];
                if (C > 1) cluster.sync(); else __syncthreads();
                if (threadIdx.x < G) {
                    double gs = 0.0, hs = 0.0;
                    for (int r = 0; r < C; ++r) {
                        const double2 pp = s_part[par][r][0][threadIdx.x];
                        gs += pp.x;
                        hs += pp.y;
                    }
                    s_dr[0][threadIdx.x] = coord_step(q, threadIdx.x, gs, hs);
                }
                __syncthreads();
                T dd[G];
                bool any = false;
                #pragma unroll
                for (int f = 0; f < G; ++f) { dd[f] = (T)s_dr[0][f]; any |= (s_dr[0][f] != 0.0); }
                if (threadIdx.x == 0) count_run(q, 1);
                if (any) {
                    if (cached1) cache_update<T, G>(bcache, xbg, s_cbo, 1, s_dr, s_drow, 0);
                    else rows_update<T, G, kBT>(cr, threadIdx.x, xbg, dd, s_abuf);
                }
                __syncthreads();
                par ^= 1;
                ++q;
            }
            } else {
              if (L > 1) {
                  // ---- a run of L conflict-free short columns: warp w takes column q + w
                  const int qq = q + warp;
                  int kk[kRunItems];
                  T vv[kRunItems], xx[kRunItems];
                  bool ind = true;
                  if (warp < L) {
                      const int fmt = c_fmt[qq];
                      ind = (fmt == CYC_INDICATOR || fmt == CYC_INTERCEPT);
                      const int e0 = c_e0[qq], n = c_e1[qq] - e0, so = c_off[qq];
                      const int* cidx = A.idx + c_cp[qq];
                      const double* cval = A.val + c_vp[qq];
                      #pragma unroll
                      for (int r = 0; r < kRunItems; ++r) {
                          const int e = wslot + r * WS;
                          const bool ok = e < n && !done_l;
                          kk[r] = !ok ? -1 : (so >= 0 ? s_sidx[so + e] : __ldg(cidx + e0 + e));
                          xx[r] = (!ok || ind) ? T(1) : (so >= 0 ? s_sx[so + e] : (T)__ldg(cval + e0 + e));
                      }
                      T ww[kRunItems];
                      #pragma unroll
                      for (int r = 0; r < kRunItems; ++r) {
                          vv[r] = kk[r] >= 0 ? xbg[(size_t)kk[r] * G + fl] : T(0);
                          ww[r] = kk[r] >= 0 ? row_weight<T, WM>(wg, A.fold, fitfold, kk[r], G, fl) : T(0);
                      }
                      Kahan<T> ag, ah;
                      #pragma unroll
                      for (int r = 0; r < kRunItems; ++r)
                          if (kk[r] >= 0 && ww[r] != T(0)) row_gh<T, MODEL>(vv[r], xx[r], ww[r], ind, ag, ah);
                      double g = ag.value(), h = ah.value();
                      for (int o = G; o < 32; o <<= 1) {
                          g += __shfl_xor_sync(0xffffffffu, g, o);
                          h += __shfl_xor_sync(0xffffffffu, h, o);
                      }
                      if (lane < G)
                          for (int r = 0; r < C; ++r)
                              *cluster.map_shared_rank(&s_part[par][rank][warp][lane], r) = make_double2(g, h);
                  }
                  if (C > 1) cluster.sync(); else __syncthreads();
                  double dl = 0.0;
                  if (warp < L) {
                      if (lane < G) {
                          double g = 0.0, h = 0.0;
                          for (int r = 0; r < C; ++r) {
                              const double2 pp = s_part[par][r][warp][lane];
                              g += pp.x;
                              h += pp.y;
                          }
                          g -= c_xjy[qq][lane];                     // :1181-1183
                          if (!s_done[lane] && !((c_lfix[qq] >> lane) & 1u)) {
                              if (h < 0.0) { g = 0.0; h = 0.0; }    // ccdUpdateBeta :1407-1410
                              const double b = c_beta[qq][lane];
                              double hd = c_hd[qq][lane];
                              dl = prior_delta(c_pt[qq], var_l, b, g, h);
                              dl = apply_bounds(&hd, dl);
                              c_hd[qq][lane] = hd;
                              if (dl != 0.0) c_beta[qq][lane] = b + dl;
                          }
                          s_dr[warp][lane] = dl;
                      }
                      dl = __shfl_sync(0xffffffffu, dl, fl);
                      if (dl != 0.0) {
                          const T d = (T)dl;
                          #pragma unroll
                          for (int r = 0; r < kRunItems; ++r)
                              if (kk[r] >= 0) xbg[(size_t)kk[r] * G + fl] = vv[r] + d * xx[r];
                      }
                  }
                  __syncthreads();
                  if (threadIdx.x == 0) count_run(q, L);
                  par ^= 1;
                  q += L;
                  continue;
              }
              // ---- a single column
              const int fmt = c_fmt[q];
              const bool dense = (fmt == CYC_DENSE || fmt == CYC_INTERCEPT);
              const bool ind = (fmt == CYC_INDICATOR || fmt == CYC_INTERCEPT);
              const int* cidx = A.idx + c_cp[q];
              const double* cval = A.val + c_vp[q];
              const int e0 = c_e0[q], e1 = c_e1[q];
              const bool regpath = !grouped && (e1 - e0) <= kRegItems * NS;
              Kahan<T> ag, ah;
              int kk[kRegItems];
              T vv[kRegItems], xx[kRegItems];
              if (regpath) {
                  const int so = c_off[q];
                  #pragma unroll
                  for (int r = 0; r < kRegItems; ++r) {
                      const int e = slot + r * NS;                 // relative to e0
                      const bool ok = e < e1 - e0 && !done_l;
                      kk[r] = !ok ? -1 : (so >= 0 ? s_sidx[so + e] : (dense ? e0 + e : __ldg(cidx + e0 + e)));
                      xx[r] = (!ok || ind) ? T(1) : (so >= 0 ? s_sx[so + e] : (T)__ldg(cval + e0 + e));
                  }
                  T ww[kRegItems];
                  #pragma unroll
                  for (int r = 0; r < kRegItems; ++r) {
                      vv[r] = kk[r] >= 0 ? xbg[(size_t)kk[r] * G + fl] : T(0);
                      ww[r] = kk[r] >= 0 ? row_weight<T, WM>(wg, A.fold, fitfold, kk[r], G, fl) : T(0);
                  }
                  #pragma unroll
                  for (int r = 0; r < kRegItems; ++r)
                      if (kk[r] >= 0 && ww[r] != T(0)) row_gh<T, MODEL>(vv[r], xx[r], ww[r], ind, ag, ah);
              } else if (!grouped) {
                  if (!done_l) {
                      // long column: batches of kRegItems entries per thread, loads first
                      for (int base = e0 + slot; base < e1; base += kRegItems * NS) {
                          int k2[kRegItems];
                          T x2[kRegItems], v2[kRegItems], w2[kRegItems];
                          #pragma unroll
                          for (int r = 0; r < kRegItems; ++r) {
                              const int e = base + r * NS;
                              k2[r] = (e < e1) ? (dense ? e : __ldg(cidx + e)) : -1;
                              x2[r] = (e < e1 && !ind) ? (T)__ldg(cval + e) : T(1);
                          }
                          #pragma unroll
                          for (int r = 0; r < kRegItems; ++r) {
                              v2[r] = k2[r] >= 0 ? xbg[(size_t)k2[r] * G + fl] : T(0);
                              w2[r] = k2[r] >= 0 ? row_weight<T, WM>(wg, A.fold, fitfold, k2[r], G, fl) : T(0);
                          }
                          #pragma unroll
                          for (int r = 0; r < kRegItems; ++r)
                              if (k2[r] >= 0 && w2[r] != T(0)) row_gh<T, MODEL>(v2[r], x2[r], w2[r], ind, ag, ah);
                      }
                  }
              } else {
                  for (int e = e0 + slot; e < e1; e += NS) {
                      const int k = dense ? e : __ldg(cidx + e);
                      const int s = A.strat[k];
                      if (e > e0) {
                          const int kp = dense ? e - 1 : __ldg(cidx + e - 1);
                          if (A.strat[kp] == s) continue;
                      }
                      T n1 = 0, n2 = 0;
                      int qe = e;
                      int kq = k;
                      do {                                  // the run of stratum s in this column
                          const T x = ind ? T(1) : (T)__ldg(cval + qe);
                          const T ex = fexp(xbg[(size_t)kq * G + fl]);
                          n1 += ex * x;
                          if (!ind) n2 += ex * x * x;
                          ++qe;
                          if (qe >= e1) break;
                          kq = dense ? qe : __ldg(cidx + qe);
                      } while (A.strat[kq] == s);
                      const double d = dg[(size_t)s * G + fl];
                      const double nwv = ng[(size_t)s * G + fl];
                      const double t = (double)n1 / d;        // ConditionalLogisticRegression::incrementGradientAndHessian
                      const double gg = nwv * t;
                      ag.add((T)gg);
                      ah.add((T)(ind ? gg * (1.0 - t) : nwv * ((double)n2 / d - t * t)));
                  }
              }
              block_reduce_lanes<G>(ag.value(), ah.value(), s_red, s_scr);
              if (threadIdx.x < G)
                  for (int r = 0; r < C; ++r) *cluster.map_shared_rank(&s_part[par][rank][0][threadIdx.x], r) = s_red[threadIdx.x];
              if (C > 1) cluster.sync(); else __syncthreads();
              // ---- coordinate step, identical in every CTA of the cluster
              if (threadIdx.x < G) {
                  double g = 0.0, h = 0.0;
                  for (int r = 0; r < C; ++r) {
                      const double2 pp = s_part[par][r][0][threadIdx.x];
                      g += pp.x;
                      h += pp.y;
                  }
                  g -= c_xjy[q][threadIdx.x];                    // :1181-1183
                  double delta = 0.0;
                  if (!s_done[threadIdx.x] && !((c_lfix[q] >> threadIdx.x) & 1u)) {
                      if (h < 0.0) { g = 0.0; h = 0.0; }          // ccdUpdateBeta :1407-1410
                      const double b = c_beta[q][threadIdx.x];
                      double hd = c_hd[q][threadIdx.x];
                      delta = prior_delta(c_pt[q], var_l, b, g, h);
                      delta = apply_bounds(&hd, delta);
                      c_hd[q][threadIdx.x] = hd;
                      if (delta != 0.0) c_beta[q][threadIdx.x] = b + delta;
                  }
                  s_delta[threadIdx.x] = delta;
              }
              __syncthreads();
              const double dl = s_delta[fl];
              if (threadIdx.x == 0) {
                  // as count_run, over this CTA's entries of the column
                  int act = 0, upd = 0;
                  for (int f = 0; f < G; ++f) { act += !s_done[f]; upd += (s_delta[f] != 0.0); }
                  const long long nnc = e1 - e0;
                  n_grad += (unsigned long long)(act * nnc);
                  n_upd += (unsigned long long)(upd * nnc);
                  if (rank == 0) n_steps += act;
                  // the column streamed by this group: row ids (not for dense) and
                  // values (sparse, dense), once for the gradient, again for an update
                  const long long cb = nnc * ((dense ? 0 : 4) + (ind ? 0 : 8));
                  n_idx += (unsigned long long)(cb * (1 + (upd ? 1 : 0)));
              }
              // ---- updateXBeta for my rows
              if (dl != 0.0) {
                  const T d = (T)dl;
                  if (regpath) {
                      #pragma unroll
                      for (int r = 0; r < kRegItems; ++r)
                          if (kk[r] >= 0) xbg[(size_t)kk[r] * G + fl] = vv[r] + d * xx[r];
                  } else if (!grouped) {
                      for (int base = e0 + slot; base < e1; base += kRegItems * NS) {
                          int k2[kRegItems];
                          T x2[kRegItems], v2[kRegItems];
                          #pragma unroll
                          for (int r = 0; r < kRegItems; ++r) {
                              const int e = base + r * NS;
                              k2[r] = (e < e1) ? (dense ? e : __ldg(cidx + e)) : -1;
                              x2[r] = (e < e1 && !ind) ? (T)__ldg(cval + e) : T(1);
                          }
                          #pragma unroll
                          for (int r = 0; r < kRegItems; ++r) v2[r] = k2[r] >= 0 ? xbg[(size_t)k2[r] * G + fl] : T(0);
                          #pragma unroll
                          for (int r = 0; r < kRegItems; ++r)
                              if (k2[r] >= 0) xbg[(size_t)k2[r] * G + fl] = v2[r] + d * x2[r];
                      }
                  } else {
                      for (int e = e0 + slot; e < e1; e += NS) {
                          const int k = dense ? e : __ldg(cidx + e);
                          const int s = A.strat[k];
                          if (e > e0) {
                              const int kp = dense ? e - 1 : __ldg(cidx + e - 1);
                              if (A.strat[kp] == s) continue;
                          }
                          double acc = dg[(size_t)s * G + fl];
                          int qe = e;
                          int kq = k;
                          do {
                              const T x = ind ? T(1) : (T)__ldg(cval + qe);
                              T* pp = xbg + (size_t)kq * G + fl;
                              const T old = *pp;
                              const T nv = old + d * x;
                              *pp = nv;
                              acc += (double)fexp(nv) - (double)fexp(old);
                              ++qe;
                              if (qe >= e1) break;
                              kq = dense ? qe : __ldg(cidx + qe);
                          } while (A.strat[kq] == s);
                          dg[(size_t)s * G + fl] = acc;
                      }
                  }
              }
              __syncthreads();
              par ^= 1;
              ++q;
            }
        }
        // chunk done: rank 0 writes the group's beta and trust regions back
        if (rank == 0)
            for (int qq = threadIdx.x; qq < jn * G; qq += kBT) {
                const int ff = qq / jn, jj = qq % jn;
                const size_t o = (size_t)(fg + ff) * A.J + j0 + jj;
                A.beta[o] = c_beta[jj][ff];
                A.hdelta[o] = c_hd[jj][ff];
            }
        __syncthreads();
      }
        // ---- convergence test (performCheckConvergence)
        const double p = objective_partial<T, MODEL, G, WM>(A, grp, r0, r1, s0, s1, xbg, wg, fitfold, fl, use_ll);
        block_reduce_lanes<G>(p, 0.0, s_red, s_scr);
        if (threadIdx.x < G)
            for (int r = 0; r < C; ++r) *cluster.map_shared_rank(&s_obj[opar][rank][threadIdx.x], r) = s_red[threadIdx.x].x;
        if (C > 1) cluster.sync(); else __syncthreads();
        if (threadIdx.x < G) {
            const int f = fg + threadIdx.x;
            double o = 0.0;
            for (int r = 0; r < C; ++r) o += s_obj[opar][r][threadIdx.x];
            if (use_ll && (MODEL == CYC_PR || MODEL == CYC_CPR)) o += A.llfixed[f];
            if (A.conv == CYC_CONV_LANGE) {
                const double* bf = A.beta + (size_t)f * A.J;
                for (int j = 0; j < A.J; ++j) o += log_density(A.ptype[j], A.variance[f], bf[j]);
            }
            if (!s_done[threadIdx.x]) {
                double convv;
                int ill = 0;
                if (o != o) { convv = 0.0; ill = 1; }
                else convv = fabs(o - s_last[threadIdx.x]) / (fabs(o) + 1.0);
                s_iter[threadIdx.x] = it;
                if (A.tol > 0 && convv < A.tol) {
                    s_done[threadIdx.x] = 1;
                    s_flag[threadIdx.x] = ill ? CYC_ILLCONDITIONED : CYC_SUCCESS;
                } else if (it == A.max_iter) {
                    s_done[threadIdx.x] = 1;
                    s_flag[threadIdx.x] = CYC_MAX_ITERATIONS;
                }
                s_last[threadIdx.x] = o;
            }
        }
        opar ^= 1;
        __syncthreads();
        if (threadIdx.x == 0) {
            int all = 1;
            for (int f = 0; f < G; ++f) all &= s_done[f];
            s_all_done = all;
        }
        __syncthreads();
        done_l = s_done[fl] != 0;
        done_m = 0;
        for (int f = 0; f < G; ++f) done_m |= (s_done[f] ? 1u : 0u) << f;
        if (s_all_done) break;
    }
    if (xb_local) {
        __syncthreads();
        for (int i = threadIdx.x; i < r1 - r0; i += kBT) xb_global[r0 + i] = s_xb[i];
    }
    if (C > 1) cluster.sync();   // no CTA leaves while others may still read its shared memory
    if (rank == 0 && threadIdx.x < G) {
        const int f = fg + threadIdx.x;
        A.out_iter[f] = s_iter[threadIdx.x];
        A.out_flag[f] = s_flag[threadIdx.x];
        A.out_obj[f] = s_last[threadIdx.x];
    }
    if (threadIdx.x == 0) {
        atomicAdd(A.counters + 0, n_grad);
        atomicAdd(A.counters + 1, n_upd);
        if (rank == 0) atomicAdd(A.counters + 2, n_steps);
        atomicAdd(A.counters + 3 + grp, n_idx);
    }
}

// ---- set-up kernels ----------------------------------------------------------

// first entry of column j whose row is >= rpart[r]
__global__ void k_splits(int J, int C, const int* fmt, const long long* col_ptr, const int* idx,
                         const int* rpart, int* split) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= J * (C + 1)) return;
    const int j = t / (C + 1), r = t % (C + 1);
    const int f = fmt[j];
    if (f == CYC_DENSE || f == CYC_INTERCEPT) { split[t] = rpart[r]; return; }
    const int* c = idx + col_ptr[j];
    int lo = 0, hi = (int)(col_ptr[j + 1] - col_ptr[j]);
    const int key = rpart[r];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (c[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    split[t] = lo;
}

// one fit's weights (K doubles, or all ones) into the [group][K][G] layout
template <class T>
__global__ void k_scatter_weights(int K, int G, int f, const double* __restrict__ src, T* __restrict__ w) {
    const int grp = f / G, lane = f % G;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        w[((size_t)grp * K + k) * G + lane] = src ? (T)src[k] : T(1);
}

// values of the entries a batch shares (index into the value array, -1 for 1)
__global__ void k_gather_values(int n, const int* __restrict__ vi, const double* __restrict__ val,
                                double* __restrict__ out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        out[t] = vi[t] >= 0 ? val[vi[t]] : 1.0;
}

__global__ void k_fold_to_i8(int K, const int* __restrict__ fold, signed char* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) out[k] = (signed char)fold[k];
}

// per fit: log likelihood under its training weights (getLogLikelihood,
// ModelSpecifics.hpp:605-650) and, for a CV grid, the predictive log
// likelihood of its held-out rows (getPredictiveLogLikelihood, :652-690 with
// logPredLikeContrib, ModelSpecifics.h:1002-1009, 1583-1590, 871-874)
__global__ void k_batch_final(int model, int K, int S, int G, int F, const double* __restrict__ y,
                              const double* __restrict__ xb, const double* __restrict__ w,
                              const double* __restrict__ denom, const double* __restrict__ nw,
                              const int* __restrict__ strat, const int* __restrict__ fold,
                              const int* __restrict__ fitfold, const double* __restrict__ llfixed,
                              double* __restrict__ ll, double* __restrict__ pll) {
    const int f = blockIdx.x;
    if (f >= F) return;
    const int grp = f / G, lane = f % G;
    const bool grouped = (model == CYC_CLR || model == CYC_CPR);
    double a = 0.0, p = 0.0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const size_t o = ((size_t)grp * K + k) * G + lane;
        const double v = xb[o], yk = y[k];
        const double wt = w ? w[o] : ((fitfold[f] >= -1 && fold[k] != fitfold[f]) ? 1.0 : 0.0);
        const int yi = (int)yk;
        a += yi * v * wt;
        if (model == CYC_LR) a -= wt * log(1.0 + exp(v));
        if (model == CYC_PR) a -= wt * exp(v);
        if (fold) {
            const double h = (fold[k] == fitfold[f]) ? 1.0 : 0.0;
            if (model == CYC_LR) p += yk * h * (v - log(1.0 + exp(v)));
            else if (model == CYC_PR) p += (yk * v - exp(v)) * h;
            else p += yk * h * (v - log(denom[((size_t)grp * S + strat[k]) * G + lane]));
        }
    }
    if (grouped)
        for (int s = threadIdx.x; s < S; s += blockDim.x) {
            const size_t o = ((size_t)grp * S + s) * G + lane;
            a -= nw[o] * log(denom[o]);
        }
    block_sum2(a, p);
    if (threadIdx.x == 0) {
        ll[f] = a + ((model == CYC_PR || model == CYC_CPR) ? llfixed[f] : 0.0);
        pll[f] = p;
    }
}

// KKT scores of an active-set pass (computeKktConditions,
// CyclicCoordinateDescent.cpp:817-837): |gradient| of column j for the fits
// of group blockIdx.y that hold it inactive (bit f of `need`), at their
// current linear predictors (independent-rows models, FP64 state); one CTA
// per (column, group), entries strided over the threads, fixed-order sums.
template <int G>
__global__ void __launch_bounds__(kBT) k_batch_kkt(int model, int K, int J, const int* __restrict__ fmt,
                                                   const long long* __restrict__ col_ptr,
                                                   const long long* __restrict__ val_ptr, const int* __restrict__ idx,
                                                   const double* __restrict__ val, const double* __restrict__ xb,
                                                   const double* __restrict__ w, const signed char* __restrict__ fold,
                                                   const int* __restrict__ fitfold, const double* __restrict__ xjy,
                                                   const unsigned char* __restrict__ need, double* __restrict__ score) {
    const int j = blockIdx.x, grp = blockIdx.y;
    const unsigned nm = need[(size_t)grp * J + j];
    if (nm == 0) return;
    __shared__ unsigned char s_wm[128];
    __shared__ double s_g[kBT / 32][G];
    if (fold)
        for (int v = threadIdx.x; v < 128; v += blockDim.x) {
            unsigned m = 0;
            for (int f = 0; f < G; ++f) {
                const int ff = fitfold[grp * G + f];
                if (ff >= -1 && ff != v) m |= 1u << f;
            }
            s_wm[v] = (unsigned char)m;
        }
    __syncthreads();
    const int fm = fmt[j];
    const bool dense = (fm == CYC_DENSE || fm == CYC_INTERCEPT);
    const bool ind = (fm == CYC_INDICATOR || fm == CYC_INTERCEPT);
    const long long n = dense ? (long long)K : col_ptr[j + 1] - col_ptr[j];
    double g[G];
    #pragma unroll
    for (int f = 0; f < G; ++f) g[f] = 0.0;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        const int k = dense ? (int)e : idx[col_ptr[j] + e];
        const double x = ind ? 1.0 : val[val_ptr[j] + e];
        const size_t o = ((size_t)grp * K + k) * G;
        const unsigned wm = fold ? (unsigned)s_wm[fold[k]] : 0u;
        #pragma unroll
        for (int f = 0; f < G; ++f) {
            const double wt = fold ? (double)((wm >> f) & 1u) : w[o + f];
            if (wt == 0.0) continue;
            const double v = xb[o + f];
            const double m = model == CYC_LR ? 1.0 / (1.0 + exp(-v)) : exp(v);
            g[f] += wt * m * x;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    #pragma unroll
    for (int f = 0; f < G; ++f) {
        double v = g[f];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_g[wid][f] = v;
    }
    __syncthreads();
    if (threadIdx.x < G && ((nm >> threadIdx.x) & 1u)) {
        double t = 0.0;
        for (int q = 0; q < kBT / 32; ++q) t += s_g[q][threadIdx.x];
        const size_t o = (size_t)(grp * G + threadIdx.x) * J + j;
        score[o] = fabs(t - xjy[o]);
    }
}

// initial linear predictor of every fit from its starting coefficients
// (zeroXBeta + axpyXBeta in column order, FP64 sums)
template <class T>
__global__ void k_init_xb(int K, int G, int F, const long long* __restrict__ row_ptr, const int* __restrict__ row_col,
                          const double* __restrict__ row_val, const double* __restrict__ beta, int J,
                          T* __restrict__ xb) {
    const long long total = (long long)K * F;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t % F);
        const int k = (int)(t / F);
        const double* bf = beta + (size_t)f * J;
        double s = 0.0;
        for (long long p = row_ptr[k]; p < row_ptr[k + 1]; ++p) {
            const double b = bf[row_col[p]];
            if (b != 0.0) s = add_mul_rn(s, b, row_val[p]);
        }
        xb[((size_t)(f / G) * K + k) * G + (f % G)] = (T)s;
    }
}

// per-fit XjY (computeXjY, ModelSpecifics.hpp:486-524): one block per column
template <class T>
__global__ void k_batch_xjy(int J, int K, int G, int ngroups, const int* fmt, const long long* col_ptr,
                            const long long* val_ptr, const int* idx, const double* val, const double* y,
                            const T* w, double* xjy) {
    __shared__ double s_scr[kBT / 32][32];
    for (int j = blockIdx.x; j < J; j += gridDim.x) {
        const int f = fmt[j];
        const bool dense = (f == CYC_DENSE || f == CYC_INTERCEPT);
        const long long n = dense ? K : col_ptr[j + 1] - col_ptr[j];
        const int* c = idx + col_ptr[j];
        const double* v = val + val_ptr[j];
        for (int grp = 0; grp < ngroups; ++grp) {
            // thread = (lane, slot) over G lanes
            const int lane = threadIdx.x % G, slot = threadIdx.x / G, ns = kBT / G;
            double acc = 0.0;
            for (long long e = slot; e < n; e += ns) {
                const int k = dense ? (int)e : c[e];
                const double x = (f == CYC_SPARSE || f == CYC_DENSE) ? v[e] : 1.0;
                acc += x * y[k] * (double)w[((size_t)grp * K + k) * G + lane];
            }
            for (int o = G; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            const int l = threadIdx.x & 31, wid = threadIdx.x >> 5;
            if (l < G) s_scr[wid][l] = acc;
            __syncthreads();
            if (threadIdx.x < G) {
                double s = 0.0;
                for (int q = 0; q < kBT / 32; ++q) s += s_scr[q][threadIdx.x];
                xjy[(size_t)(grp * G + threadIdx.x) * J + j] = s;
            }
            __syncthreads();
        }
    }
}

// CV grid XjY (computeXjY, ModelSpecifics.hpp:486-524, with 0/1 fold
// weights): per column, the sums of x*y over its entries in each fold, 16
// folds per pass, each thread summing its own entries, then the threads'
// sums in thread order (deterministic).  out[j][v], v < n_folds.
__global__ void k_fold_xy(int J, int K, int n_folds, const int* fmt, const long long* col_ptr,
                          const long long* val_ptr, const int* idx, const double* val, const double* y,
                          const signed char* fold, double* out) {
    __shared__ double part[16][kBT];
    for (int j = blockIdx.x; j < J; j += gridDim.x) {
        const int f = fmt[j];
        const bool dense = (f == CYC_DENSE || f == CYC_INTERCEPT);
        const bool hasx = (f == CYC_SPARSE || f == CYC_DENSE);
        const long long n = dense ? K : col_ptr[j + 1] - col_ptr[j];
        const int* c = idx + col_ptr[j];
        const double* v = val + val_ptr[j];
        for (int v0 = 0; v0 < n_folds; v0 += 16) {
            for (int q = 0; q < 16; ++q) part[q][threadIdx.x] = 0.0;
            for (long long e = threadIdx.x; e < n; e += kBT) {
                const int k = dense ? (int)e : c[e];
                const int q = (int)fold[k] - v0;
                if (q >= 0 && q < 16) part[q][threadIdx.x] += (hasx ? v[e] : 1.0) * y[k];
            }
            __syncthreads();
            if (threadIdx.x < 16 && v0 + (int)threadIdx.x < n_folds) {
                double sum = 0.0;
                for (int t = 0; t < kBT; ++t) sum += part[threadIdx.x][t];
                out[(size_t)j * n_folds + v0 + threadIdx.x] = sum;
            }
            __syncthreads();
        }
    }
}

// every fit's XjY from the fold sums: fit f trains on the folds other than
// fitfold[f] (all of them for -1, none for padding fits)
__global__ void k_cv_xjy(int J, int Fp, int n_folds, const double* __restrict__ fs, const int* __restrict__ fitfold,
                         double* __restrict__ xjy) {
    const long long total = (long long)Fp * J;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / J), j = (int)(t % J);
        const int ff = fitfold[f];
        double sum = 0.0;
        if (ff >= -1)
            for (int v = 0; v < n_folds; ++v)
                if (v != ff) sum += fs[(size_t)j * n_folds + v];
        xjy[(size_t)f * J + j] = sum;
    }
}

// grouped models: per (stratum, fit) events sum(y*w) and denominator sum(exp(xb))
template <class T>
__global__ void k_batch_strata(int S, int K, int G, int ngroups, const int* strat_ptr, const double* y, const T* w,
                               const signed char* fold, const int* fitfold, const T* xb, double* nw, double* denom) {
    const long long total = (long long)S * G * ngroups;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int lane = (int)(t % G);
        const int s = (int)((t / G) % S);
        const int grp = (int)(t / ((long long)G * S));
        double a = 0.0, d = 0.0;
        for (int k = strat_ptr[s]; k < strat_ptr[s + 1]; ++k) {
            const size_t o = ((size_t)grp * K + k) * G + lane;
            const int ff = w ? 0 : fitfold[grp * G + lane];
            a += y[k] * (w ? (double)w[o] : ((ff >= -1 && fold[k] != ff) ? 1.0 : 0.0));
            d += exp((double)xb[o]);
        }
        nw[((size_t)grp * S + s) * G + lane] = a;
        denom[((size_t)grp * S + s) * G + lane] = d;
    }
}

// fixed likelihood terms per fit: sum_k w_fk * c_k with c_k = -log(y_k!)
template <class T>
__global__ void k_batch_llfixed(int K, int G, int F, const double* c, const T* w, const signed char* fold,
                                const int* fitfold, double* out) {
    const int f = blockIdx.x;
    if (f >= F) return;
    const int grp = f / G, lane = f % G;
    const int ff = w ? 0 : fitfold[f];
    double a = 0.0, dummy = 0.0;
    for (int k = threadIdx.x; k < K; k += blockDim.x)
        a += c[k] * (w ? (double)w[((size_t)grp * K + k) * G + lane] : ((ff >= -1 && fold[k] != ff) ? 1.0 : 0.0));
    block_sum2(a, dummy);
    if (threadIdx.x == 0) out[f] = a;
}

}  // namespace


// Column batches (see k_batch): walk the columns in order and extend the open
// batch with the next short column (sparse or indicator, not fixed, at most
// `cap` entries in every CTA's rows) while it holds fewer than kRunMax
// columns, the chunk of kChunk coordinates goes on, and the rows shared
// between its columns number at most `dmax`; otherwise close it and open a new
// one.  A column's level is 1 + the highest level of the earlier columns of
// its batch it shares a row with, so columns of one level touch disjoint
// rows.  Each shared row gets a slot, and every entry on a shared row is
// listed with (slot, column within the batch, position in the column).
// dmax = 0 gives the conflict-free runs used with one fit per group.
// `batch_rows` > 0 also closes a batch before its entries in any one CTA's
// rows would exceed that many (the batch cache holds them all).
static RunPlan plan_runs(const Dataset& ds, const std::vector<int>& rpart, const std::vector<int>& fixb, int cap,
                         bool allow, int dmax, int batch_rows = 0, int lvl_max = kLevelMax) {
    const int J = ds.J, K = ds.K, C = (int)rpart.size() - 1;
    RunPlan P;
    P.len.assign(J, 1);
    P.lvl.assign(J, 1);
    P.dr0.assign(J, 0);
    P.nd.assign(J, 0);
    P.de_ptr.assign(J + 1, 0);
    // per row: the batch that last touched it, its level, its shared-row slot
    // and its first (column, entry) in that batch -- one struct per row, so
    // the random row lookups of a column touch one cache line each
    struct RowState { int stamp = -1, rlvl = 0, dslot = -1, first_w = 0, first_e = 0; };
    std::vector<RowState> rs(K);
    struct Ent { int w, d, e; };
    std::vector<Ent> ents;
    std::vector<int> shared;            // row ids in order of their slots
    int run_id = -1, start = -1, len = 0;
    std::vector<int> bsum(C, 0);        // the open batch's entries per CTA
    auto close = [&] {
        std::fill(bsum.begin(), bsum.end(), 0);
        if (start < 0) return;
        P.len[start] = len;
        P.dr0[start] = (int)P.drow.size();
        P.nd[start] = (int)shared.size();
        P.drow.insert(P.drow.end(), shared.begin(), shared.end());
        std::stable_sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) { return a.w < b.w; });
        size_t i = 0;
        for (int w = 0; w < len; ++w) {
            P.de_ptr[start + w] = (int)P.de_d.size();
            for (; i < ents.size() && ents[i].w == w; ++i) {
                P.de_d.push_back(ents[i].d | (w << 8));
                P.de_e.push_back(ds.fmt[start + w] == CYC_SPARSE ? (int)(ds.val_ptr[start + w] + ents[i].e) : -1);
            }
        }
        ents.clear();
        shared.clear();
        start = -1;
        len = 0;
    };
    std::vector<int> cnt(C);
    for (int j = 0; j < J; ++j) {
        if (j % kChunk == 0) close();
        const int f = ds.fmt[j];
        bool small = allow && (f == CYC_SPARSE || f == CYC_INDICATOR) && !fixb[j];
        const int* rows = ds.h_idx.data() + ds.col_ptr[j];
        const int n = (int)(ds.col_ptr[j + 1] - ds.col_ptr[j]);
        if (small) {
            std::fill(cnt.begin(), cnt.end(), 0);
            int r = 0;
            for (int e = 0; e < n && small; ++e) {
                while (r < C - 1 && rows[e] >= rpart[r + 1]) ++r;
                if (++cnt[r] > cap) small = false;
            }
        }
        if (!small) {
            close();
            P.de_ptr[j] = (int)P.de_d.size();
            continue;
        }
        // rows shared with the open batch: how many become shared, and the level
        int fresh = 0, level = 1;
        if (start >= 0)
            for (int e = 0; e < n; ++e)
                if (rs[rows[e]].stamp == run_id) {
                    fresh += rs[rows[e]].dslot < 0;
                    level = std::max(level, rs[rows[e]].rlvl + 1);
                }
        bool full = false;
        if (batch_rows > 0)
            for (int r = 0; r < C; ++r) full |= bsum[r] + cnt[r] > batch_rows;
        if (start >= 0 && (len == kRunMax || (int)shared.size() + fresh > dmax || level > lvl_max || full)) {
            close();
            level = 1;
        }
        for (int r = 0; r < C; ++r) bsum[r] += cnt[r];
        if (start < 0) {
            start = j;
            ++run_id;
        }
        const int w = len;
        for (int e = 0; e < n; ++e) {
            const int r = rows[e];
            if (rs[r].stamp == run_id) {
                if (rs[r].dslot < 0) {
                    rs[r].dslot = (int)shared.size();
                    shared.push_back(r);
                    ents.push_back({rs[r].first_w, rs[r].dslot, rs[r].first_e});
                }
                ents.push_back({w, rs[r].dslot, e});
            } else {
                rs[r].stamp = run_id;
                rs[r].dslot = -1;
                rs[r].first_w = w;
                rs[r].first_e = e;
            }
            rs[r].rlvl = level;
        }
        P.len[j] = 0;
        P.lvl[j] = level;
        ++len;
    }
    close();
    P.de_ptr[J] = (int)P.de_d.size();
    return P;
}

template <class T, int MODEL, int G, int WM>
static void launch_batch(const BatchArgs& a, int ngroups, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ngroups * a.C);
    cfg.blockDim = dim3(kBT);
    const size_t dyn = 3 * kChunk * G * sizeof(double) + kStage * sizeof(int) + staged_value_bytes<T, MODEL, G>() +
                       5 * kDirtyMax * G * sizeof(T) + (G == 1 ? (size_t)a.xb_smem * sizeof(T) : 0);
    CYC_CHECK_CUDA(cudaFuncSetAttribute(k_batch<T, MODEL, G, WM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CYC_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_batch<T, MODEL, G, WM>, a));
    count_launch();
}

template <class T, int G>
static void launch_model(const BatchArgs& a, int ngroups, cudaStream_t stream) {
    const bool cv = a.fold != nullptr;
    switch (a.model) {
    case CYC_LR: cv ? launch_batch<T, CYC_LR, G, 1>(a, ngroups, stream) : launch_batch<T, CYC_LR, G, 0>(a, ngroups, stream); break;
    case CYC_PR: cv ? launch_batch<T, CYC_PR, G, 1>(a, ngroups, stream) : launch_batch<T, CYC_PR, G, 0>(a, ngroups, stream); break;
    case CYC_CLR: cv ? launch_batch<T, CYC_CLR, G, 1>(a, ngroups, stream) : launch_batch<T, CYC_CLR, G, 0>(a, ngroups, stream); break;
    case CYC_CPR: cv ? launch_batch<T, CYC_CPR, G, 1>(a, ngroups, stream) : launch_batch<T, CYC_CPR, G, 0>(a, ngroups, stream); break;
    default: throw Error{CYC_ERR_UNSUPPORTED, "batched fits support lr, pr, clr, cpr"};
    }
}

// One batched solve at precision T over fits [0, F) with starting
// coefficients `h_beta` (F x J, updated in place) and trust regions.
// CTAs per cluster when nothing is tuned: one per 8k rows, at most 8 (single
// fits measured here: 61k rows 12.7 ms a cycle at 8 CTAs against 14.2 at 4,
// 24k-35k rows 2-3 % faster at 8; up to ~8k rows one CTA is fastest, the
// cluster barrier costing more than the rows save); CYC_BATCH_CLUSTER (1..8)
// forces a size
static int default_cluster(int K) {
    if (const char* e = std::getenv("CYC_BATCH_CLUSTER")) return std::max(1, std::min(kMaxC, std::atoi(e)));
    return std::max(1, std::min(kMaxC, (K + 8191) / 8192));
}

template <class T>
struct BatchRunner {
    Dataset& ds;
    cudaStream_t stream;
    int F, G, ngroups, Fp, C;
    BatchShape shape;
    std::vector<int> rpart;
    DevBuf<int> d_rpart, d_split, d_fixb, d_ptype, d_active, d_iter, d_flag;
    DevBuf<int> d_runlen, d_runlvl, d_rundr0, d_runnd, d_drow, d_deptr, d_ded, d_dee;
    DevBuf<T> d_xb, d_w;
    DevBuf<double> d_dex;
    DevBuf<double> d_denom, d_nw, d_xjy, d_beta, d_hdelta, d_var, d_llfixed, d_obj, d_stage, d_fixedc;
    DevBuf<unsigned long long> d_counters;
    DevBuf<unsigned char> d_lfix;

    BatchRunner(Dataset& d, cudaStream_t s, int F_, int G_, int C_ = 0, BatchShape sh = BatchShape{})
        : ds(d), stream(s), F(F_), G(G_), shape(sh) {
        ngroups = (F + G - 1) / G;
        Fp = ngroups * G;
        const int K = ds.K;
        C = C_ > 0 ? std::min(kMaxC, C_) : default_cluster(K);
        // row partition, aligned to strata for grouped models
        rpart.assign(C + 1, K);
        for (int r = 0; r < C; ++r) {
            int b = (int)((long long)K * r / C);
            if (model_grouped(ds.model)) {
                auto it = std::lower_bound(ds.strat_ptr.begin(), ds.strat_ptr.end(), b);
                b = (it == ds.strat_ptr.end()) ? K : *it;
            }
            rpart[r] = b;
        }
        rpart[C] = K;
        for (int r = 1; r <= C; ++r) rpart[r] = std::max(rpart[r], rpart[r - 1]);
    }

    // weights come either from per-fit host vectors (`specs`) or, for a CV
    // grid, from fold ids on the device: fit f trains on fold_of_row != fold[f]
    const int* d_fold = nullptr;
    DevBuf<int> d_fitfold;

    DevBuf<signed char> d_fold8;

    int n_folds = 0;

    void set_folds(const int* d_fold_of_row, int folds, const std::vector<int>& fit_fold) {
        d_fold = d_fold_of_row;
        n_folds = folds;
        d_fold8.alloc(ds.K);
        launch(k_fold_to_i8, grid_for(ds.K, 1), 256, 0, stream, ds.K, d_fold, d_fold8.get());
        std::vector<int> ff(Fp, -2);
        std::copy(fit_fold.begin(), fit_fold.end(), ff.begin());
        d_fitfold.alloc(Fp);
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_fitfold.get(), ff.data(), Fp * sizeof(int), cudaMemcpyHostToDevice, stream));
    }

    void setup(const cyc_prior& prior, const cyc_fit_spec* specs, const std::vector<double>& h_beta,
               const std::vector<double>& h_hdelta, const std::vector<int>& fixed_cols) {
        const int K = ds.K, J = ds.J;
        d_rpart.alloc(C + 1);
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_rpart.get(), rpart.data(), (C + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
        d_split.alloc((size_t)J * (C + 1));
        launch(k_splits, (J * (C + 1) + 255) / 256, 256, 0, stream, J, C, ds.d_fmt.get(), ds.d_col_ptr.get(), ds.d_idx.get(),
                                                                  d_rpart.get(), d_split.get());
        CYC_CHECK_LAUNCH();
        std::vector<int> fixb(J, 0), pt(J, prior.prior_type), act(Fp, 0);
        if (ds.has_offset) fixb[0] = 1;
        for (int j : fixed_cols) fixb[j] = 1;
        for (int i = 0; i < prior.n_exclude; ++i) pt[prior.exclude[i]] = CYC_PRIOR_NONE;
        for (int f = 0; f < F; ++f) act[f] = 1;
        std::vector<double> var(Fp, 1.0);
        for (int f = 0; f < F; ++f) var[f] = specs[f].variance;
        d_fixb.alloc(J); d_ptype.alloc(J); d_active.alloc(Fp); d_var.alloc(Fp);
        {
            const RunPlan* plan = nullptr;
            const bool rows8 = (G == 8) && model_independent(ds.model);
            // batches are planned without regard to the cache: those whose
            // entries fit it in every CTA take the cached path, the rest stream
            const int brows = 0;
            const int cap = rows8 ? shape.cap : (32 / G) * kRunItems;
            const int dmax = rows8 ? shape.dmax : 0;
            const int lvl = rows8 ? shape.lvl : kLevelMax;
            for (auto& pl : ds.run_plans)
                if (pl.C == C && pl.G == G && pl.batch_rows == brows && pl.cap == cap && pl.dmax == dmax &&
                    pl.max_levels == lvl && pl.fixed == fixed_cols)
                    plan = &pl;
            if (!plan) {
                RunPlan pl = plan_runs(ds, rpart, fixb, cap, model_independent(ds.model), dmax, brows, lvl);
                pl.C = C;
                pl.G = G;
                pl.batch_rows = brows;
                pl.cap = cap;
                pl.dmax = dmax;
                pl.max_levels = lvl;
                pl.fixed = fixed_cols;
                ds.run_plans.push_back(std::move(pl));
                plan = &ds.run_plans.back();
            }
            auto up = [&](DevBuf<int>& d, const std::vector<int>& h) {
                d.alloc(std::max<size_t>(1, h.size()));
                if (!h.empty())
                    CYC_CHECK_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
            };
            up(d_runlen, plan->len);
            up(d_runlvl, plan->lvl);
            up(d_rundr0, plan->dr0);
            up(d_runnd, plan->nd);
            up(d_drow, plan->drow);
            up(d_deptr, plan->de_ptr);
            up(d_ded, plan->de_d);
            up(d_dee, plan->de_e);
            d_dex.alloc(std::max<size_t>(1, plan->de_e.size()));
            if (!plan->de_e.empty())
                launch(k_gather_values, grid_for((long long)plan->de_e.size(), 4), 256, 0, stream,
                       (int)plan->de_e.size(), (const int*)d_dee.get(), (const double*)ds.d_val.get(), d_dex.get());
            CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
        }
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_fixb.get(), fixb.data(), J * sizeof(int), cudaMemcpyHostToDevice, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_ptype.get(), pt.data(), J * sizeof(int), cudaMemcpyHostToDevice, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_active.get(), act.data(), Fp * sizeof(int), cudaMemcpyHostToDevice, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_var.get(), var.data(), Fp * sizeof(double), cudaMemcpyHostToDevice, stream));
        // weights: per-fit vectors in the [group][K][G] layout; a CV grid's
        // weights are its fold ids (no array)
        if (!d_fold) {
          d_w.alloc((size_t)ngroups * K * G);
          d_stage.alloc(K);
          for (int f = 0; f < Fp; ++f) {
            const double* src = nullptr;
            if (f < F && specs[f].weights) {
                CYC_CHECK_CUDA(cudaMemcpyAsync(d_stage.get(), specs[f].weights, K * sizeof(double), cudaMemcpyHostToDevice, stream));
                src = d_stage.get();
            }
            launch(k_scatter_weights<T>, grid_for(K, 4), 256, 0, stream, K, G, f, src, d_w.get());
            if (src) CYC_CHECK_CUDA(cudaStreamSynchronize(stream));  // staging buffer reuse
          }
        }
        // coefficients and trust regions
        d_beta.alloc((size_t)Fp * J);
        d_hdelta.alloc((size_t)Fp * J);
        std::vector<double> b((size_t)Fp * J, 0.0), hd((size_t)Fp * J, 2.0);
        std::copy(h_beta.begin(), h_beta.end(), b.begin());
        std::copy(h_hdelta.begin(), h_hdelta.end(), hd.begin());
        if (ds.has_offset) for (int f = F; f < Fp; ++f) b[(size_t)f * J] = 1.0;
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_beta.get(), b.data(), b.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_hdelta.get(), hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        // linear predictors: zero when every coefficient is zero (a cold
        // start without an offset), else sum_j beta_j x_kj over the row-major copy
        d_xb.alloc((size_t)ngroups * K * G);
        const bool all_zero = std::all_of(b.begin(), b.end(), [](double v) { return v == 0.0; });
        if (all_zero) {
            CYC_CHECK_CUDA(cudaMemsetAsync(d_xb.get(), 0, (size_t)ngroups * K * G * sizeof(T), stream));
        } else {
            ds.ensure_csr();
            launch(k_init_xb<T>, grid_for((long long)K * Fp, 1), 256, 0, stream, K, G, Fp, ds.d_row_ptr.get(),
                   ds.d_row_col.get(), ds.d_row_val.get(), d_beta.get(), J, d_xb.get());
            CYC_CHECK_LAUNCH();
        }
        // fixed gradient terms
        d_xjy.alloc((size_t)Fp * J);
        if (d_fold) {
            DevBuf<double> fs;
            fs.alloc((size_t)J * n_folds);
            launch(k_fold_xy, std::min(J, 148 * 8), kBT, 0, stream, J, K, n_folds, ds.d_fmt.get(), ds.d_col_ptr.get(),
                   ds.d_val_ptr.get(), ds.d_idx.get(), ds.d_val.get(), ds.d_y.get(), (const signed char*)d_fold8.get(),
                   fs.get());
            launch(k_cv_xjy, grid_for((long long)Fp * J, 4), 256, 0, stream, J, Fp, n_folds, (const double*)fs.get(),
                   (const int*)d_fitfold.get(), d_xjy.get());
            CYC_CHECK_CUDA(cudaStreamSynchronize(stream));   // before fs is freed
        } else {
            launch(k_batch_xjy<T>, std::min(J, 148 * 8), kBT, 0, stream, J, K, G, ngroups, ds.d_fmt.get(),
                   ds.d_col_ptr.get(), ds.d_val_ptr.get(), ds.d_idx.get(), ds.d_val.get(), ds.d_y.get(),
                   (const T*)d_w.get(), d_xjy.get());
        }
        if (model_grouped(ds.model)) {
            d_nw.alloc((size_t)ngroups * ds.S * G);
            d_denom.alloc((size_t)ngroups * ds.S * G);
            launch(k_batch_strata<T>, grid_for((long long)ds.S * Fp, 1), 256, 0, stream, 
                ds.S, K, G, ngroups, ds.d_strat_ptr.get(), ds.d_y.get(), (const T*)d_w.get(),
                (const signed char*)d_fold8.get(), (const int*)d_fitfold.get(), (const T*)d_xb.get(), d_nw.get(),
                d_denom.get());
            CYC_CHECK_LAUNCH();
        }
        d_llfixed.alloc(Fp);
        CYC_CHECK_CUDA(cudaMemsetAsync(d_llfixed.get(), 0, Fp * sizeof(double), stream));
        if (has_fixed_ll(ds.model)) {
            std::vector<double> c(K, 0.0);
            for (int k = 0; k < K; ++k)
                for (int i = 2; i <= (int)ds.y[k]; ++i) c[k] -= std::log((double)i);
            d_fixedc.alloc(K);
            CYC_CHECK_CUDA(cudaMemcpyAsync(d_fixedc.get(), c.data(), K * sizeof(double), cudaMemcpyHostToDevice, stream));
            launch(k_batch_llfixed<T>, Fp, 256, 0, stream, K, G, Fp, (const double*)d_fixedc.get(), (const T*)d_w.get(),
                   (const signed char*)d_fold8.get(), (const int*)d_fitfold.get(), d_llfixed.get());
            CYC_CHECK_LAUNCH();
            CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
        }
        d_iter.alloc(Fp); d_flag.alloc(Fp); d_obj.alloc(Fp); d_counters.alloc(3 + ngroups);
        CYC_CHECK_CUDA(cudaMemsetAsync(d_counters.get(), 0, (3 + ngroups) * sizeof(unsigned long long), stream));
    }

    void run(const cyc_control& ctl, double tol, float* ms) {
        BatchArgs a{};
        a.model = ds.model; a.K = ds.K; a.J = ds.J; a.S = ds.S; a.C = C;
        a.fmt = ds.d_fmt.get(); a.col_ptr = ds.d_col_ptr.get(); a.val_ptr = ds.d_val_ptr.get();
        a.idx = ds.d_idx.get(); a.val = ds.d_val.get(); a.split = d_split.get(); a.rpart = d_rpart.get();
        a.y = ds.d_y.get(); a.strat = ds.d_strat.get(); a.strat_ptr = ds.d_strat_ptr.get();
        a.fixb = d_fixb.get(); a.lane_fix = d_lfix.get(); a.ptype = d_ptype.get(); a.xb = d_xb.get(); a.w = d_w.get();
        // one-fit groups keep a CTA's linear predictors in shared memory when
        // its rows fit in 128 KB (CYC_BATCH_XB_SMEM=0 keeps them in global memory)
        a.xb_smem = 0;
        const char* xs = std::getenv("CYC_BATCH_XB_SMEM");
        if (G == 1 && !(xs && std::atoi(xs) == 0)) {
            int rows = 0;
            for (int r = 0; r < C; ++r) rows = std::max(rows, rpart[r + 1] - rpart[r]);
            if ((size_t)rows * sizeof(T) <= (size_t)128 * 1024) a.xb_smem = rows;
        }
        a.denom = d_denom.get(); a.nw = d_nw.get(); a.xjy = d_xjy.get(); a.beta = d_beta.get();
        a.hdelta = d_hdelta.get(); a.variance = d_var.get(); a.llfixed = d_llfixed.get(); a.active = d_active.get();
        a.fold = d_fold ? d_fold8.get() : nullptr;
        a.fitfold = d_fold ? d_fitfold.get() : nullptr;
        a.run_len = d_runlen.get();
        a.run_lvl = d_runlvl.get();
        a.run_dr0 = d_rundr0.get();
        a.run_nd = d_runnd.get();
        a.drow = d_drow.get();
        a.de_ptr = d_deptr.get();
        a.de_d = d_ded.get();
        a.de_x = d_dex.get();
        a.conv = ctl.convergence_type; a.tol = tol; a.max_iter = ctl.max_iterations;
        a.out_iter = d_iter.get(); a.out_flag = d_flag.get(); a.out_obj = d_obj.get(); a.counters = d_counters.get();
        cudaEvent_t e0, e1;
        CYC_CHECK_CUDA(cudaEventCreate(&e0));
        CYC_CHECK_CUDA(cudaEventCreate(&e1));
        CYC_CHECK_CUDA(cudaEventRecord(e0, stream));
        if (G == 1) launch_model<T, 1>(a, ngroups, stream);
        else launch_model<T, 8>(a, ngroups, stream);
        CYC_CHECK_CUDA(cudaEventRecord(e1, stream));
        CYC_CHECK_CUDA(cudaEventSynchronize(e1));
        CYC_CHECK_CUDA(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        CYC_CHECK_LAUNCH();
    }

    // active-set passes: the fits (bit f of [group][J]) holding each column
    // fixed, the fits that run the next launch, and fresh trust regions
    // (findMode's resetBounds, CyclicCoordinateDescent.cpp:943)
    void set_pass(const std::vector<unsigned char>& lane_fix, const std::vector<int>& running, double bound) {
        const int J = ds.J;
        d_lfix.alloc(lane_fix.size());
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_lfix.get(), lane_fix.data(), lane_fix.size(), cudaMemcpyHostToDevice, stream));
        std::vector<int> act(Fp, 0);
        std::copy(running.begin(), running.end(), act.begin());
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_active.get(), act.data(), Fp * sizeof(int), cudaMemcpyHostToDevice, stream));
        std::vector<double> hd((size_t)Fp * J, bound);
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_hdelta.get(), hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice,
                                       stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
    }

    // |gradient| of the columns `need` marks (bit f of [group][J]) for those
    // fits, into score[F][J] (FP64 state of an independent-rows model)
    void kkt_scores(const std::vector<unsigned char>& need, std::vector<double>& score) {
        const int J = ds.J;
        DevBuf<unsigned char> d_need;
        DevBuf<double> d_score;
        d_need.alloc(need.size());
        d_score.alloc((size_t)Fp * J);
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_need.get(), need.data(), need.size(), cudaMemcpyHostToDevice, stream));
        CYC_CHECK_CUDA(cudaMemsetAsync(d_score.get(), 0, (size_t)Fp * J * sizeof(double), stream));
        const dim3 grid(J, ngroups);
        const double* w = d_fold ? nullptr : (const double*)d_w.get();
        const signed char* fd = d_fold ? d_fold8.get() : nullptr;
        const int* ff = d_fold ? d_fitfold.get() : nullptr;
        if (G == 1)
            launch(k_batch_kkt<1>, grid, kBT, 0, stream, ds.model, ds.K, J, ds.d_fmt.get(), ds.d_col_ptr.get(),
                   ds.d_val_ptr.get(), ds.d_idx.get(), ds.d_val.get(), (const double*)d_xb.get(), w, fd, ff,
                   d_xjy.get(), d_need.get(), d_score.get());
        else
            launch(k_batch_kkt<8>, grid, kBT, 0, stream, ds.model, ds.K, J, ds.d_fmt.get(), ds.d_col_ptr.get(),
                   ds.d_val_ptr.get(), ds.d_idx.get(), ds.d_val.get(), (const double*)d_xb.get(), w, fd, ff,
                   d_xjy.get(), d_need.get(), d_score.get());
        CYC_CHECK_LAUNCH();
        score.resize((size_t)F * J);
        CYC_CHECK_CUDA(cudaMemcpyAsync(score.data(), d_score.get(), score.size() * sizeof(double),
                                       cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
    }

    // log likelihood (and held-out predictive log likelihood for CV) per fit
    void finalize(std::vector<double>& ll, std::vector<double>& pll) {
        DevBuf<double> d_ll, d_pll;
        d_ll.alloc(Fp);
        d_pll.alloc(Fp);
        const bool grouped = model_grouped(ds.model);
        launch(k_batch_final, Fp, kBT, 0, stream, ds.model, ds.K, ds.S, G, Fp, (const double*)ds.d_y.get(),
               (const double*)d_xb.get(), (const double*)d_w.get(), grouped ? (const double*)d_denom.get() : nullptr,
               grouped ? (const double*)d_nw.get() : nullptr, (const int*)ds.d_strat.get(), d_fold,
               (const int*)d_fitfold.get(), (const double*)d_llfixed.get(), d_ll.get(), d_pll.get());
        ll.resize(Fp);
        pll.resize(Fp);
        CYC_CHECK_CUDA(cudaMemcpyAsync(ll.data(), d_ll.get(), Fp * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(pll.data(), d_pll.get(), Fp * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
    }

    void results(std::vector<double>& beta, std::vector<double>& hd, std::vector<int>& iters, std::vector<int>& flags,
                 std::vector<unsigned long long>& counters) {
        const int J = ds.J;
        beta.resize((size_t)F * J);
        hd.resize((size_t)F * J);
        iters.resize(F);
        flags.resize(F);
        CYC_CHECK_CUDA(cudaMemcpyAsync(beta.data(), d_beta.get(), beta.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(hd.data(), d_hdelta.get(), hd.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(iters.data(), d_iter.get(), F * sizeof(int), cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(flags.data(), d_flag.get(), F * sizeof(int), cudaMemcpyDeviceToHost, stream));
        counters.assign(3 + ngroups, 0ull);
        CYC_CHECK_CUDA(cudaMemcpyAsync(counters.data(), d_counters.get(), counters.size() * sizeof(unsigned long long),
                                       cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
    }
};

}  // namespace cyc

using namespace cyc;

namespace {

// ---- cluster-size tuner ------------------------------------------------------
// How many CTAs share a group's rows trades per-step work (fewer rows per
// CTA) against cluster barrier cost and against how many clusters are
// resident at once (G fits per cluster, F / G clusters).  A solve large
// enough to amortise it (16 fits or more, 1e8 fit-entries or more per cycle)
// times one cycle of the real problem at the default size and at its halves
// (8, 4, 2 CTAs for large K) and keeps the fastest; the choice is cached for
// the process per problem shape, so repeated solves of one shape (a CV grid
// per step, a dataset uploaded again) probe once.  CYC_BATCH_CLUSTER skips
// the tuner.
struct TuneKey {
    int model, K, J, F, G, precision, folds;
    std::vector<int> fixed;
    long long nnz;
    bool operator<(const TuneKey& o) const {
        return std::tie(model, K, J, F, G, precision, folds, fixed, nnz) <
               std::tie(o.model, o.K, o.J, o.F, o.G, o.precision, o.folds, o.fixed, o.nnz);
    }
};
std::mutex g_tune_mutex;
std::map<TuneKey, int>& tuned_sizes() {
    static auto* m = new std::map<TuneKey, int>();   // lives to process exit
    return *m;
}

template <class T>
float probe_cycle(Dataset& ds, cudaStream_t stream, int F, int G, int C, const cyc_prior& prior,
                  const cyc_fit_spec* specs, const std::vector<double>& beta, const std::vector<double>& hd,
                  const int* d_fold, int n_folds, const std::vector<int>* fit_fold, const cyc_control& ctl,
                  const std::vector<int>& fixed_cols, BatchShape shape = BatchShape{}) {
    BatchRunner<T> r(ds, stream, F, G, C, shape);
    if (d_fold) r.set_folds(d_fold, n_folds, *fit_fold);
    r.setup(prior, specs, beta, hd, fixed_cols);
    cyc_control one = ctl;
    one.max_iterations = 1;
    float ms = 0.f;
    r.run(one, ctl.tolerance, &ms);
    return ms;
}

int tuned_cluster(Dataset& ds, cudaStream_t stream, int F, int G, const cyc_prior& prior, const cyc_fit_spec* specs,
                  const std::vector<double>& beta, const std::vector<double>& hd, const int* d_fold, int n_folds,
                  const std::vector<int>* fit_fold, const cyc_control& ctl, const std::vector<int>& fixed_cols) {
    const int base = default_cluster(ds.K);
    const double work = (double)F * (double)(ds.nnz_idx + ds.nnz_val);
    if (std::getenv("CYC_BATCH_CLUSTER") || base <= 1 || F < 16 || work < 1e8) return base;
    const TuneKey key{ds.model, ds.K, ds.J, F, G, ctl.precision, d_fold ? n_folds : 0, fixed_cols, ds.nnz_idx};
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = tuned_sizes().find(key);
        if (it != tuned_sizes().end()) return it->second;
    }
    int best = base;
    float best_ms = 0.f;
    for (int c = base; c >= 1 && c >= base / 4; c /= 2) {
        const float ms = ctl.precision == CYC_MIXED
                             ? probe_cycle<float>(ds, stream, F, G, c, prior, specs, beta, hd, d_fold, n_folds,
                                                  fit_fold, ctl, fixed_cols)
                             : probe_cycle<double>(ds, stream, F, G, c, prior, specs, beta, hd, d_fold, n_folds,
                                                   fit_fold, ctl, fixed_cols);
        if (c == base || ms < best_ms) {
            best = c;
            best_ms = ms;
        }
    }
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    tuned_sizes()[key] = best;
    return best;
}

// ---- batch-shape tuner -------------------------------------------------------
// Which columns are short (batched, a warp per column) and which stream
// through the whole CTA is a question of the columns' densities: the bound
// `cap` on a short column's entries per CTA splits the columns into the two
// buckets.  With it go the rows a batch may share (`dmax`) and the replay
// levels it may take (`lvl`).  For an 8-fit group of an independent-rows
// model large enough to amortise it (the cluster tuner's criteria), the
// tuner times one cycle of the real problem at the chosen cluster size for
// the default shape and then, one parameter at a time, for smaller
// settings (cap 128, 64; dmax 16; lvl 2), keeping each change that is
// faster; the choice is cached per problem shape for the process.
// CYC_BATCH_SHAPE="cap,dmax,lvl" sets it without probing.
std::map<std::pair<TuneKey, int>, BatchShape>& tuned_shapes() {
    static auto* m = new std::map<std::pair<TuneKey, int>, BatchShape>();   // lives to process exit
    return *m;
}

BatchShape tuned_shape(Dataset& ds, cudaStream_t stream, int F, int G, int C, const cyc_prior& prior,
                       const cyc_fit_spec* specs, const std::vector<double>& beta, const std::vector<double>& hd,
                       const int* d_fold, int n_folds, const std::vector<int>* fit_fold, const cyc_control& ctl,
                       const std::vector<int>& fixed_cols) {
    BatchShape best;
    if (const char* e = std::getenv("CYC_BATCH_SHAPE")) {
        int a = best.cap, b = best.dmax, c = best.lvl;
        if (std::sscanf(e, "%d,%d,%d", &a, &b, &c) == 3) {
            best.cap = std::max(1, std::min(kBatchCap, a));
            best.dmax = std::max(0, std::min(kDirtyMax, b));
            best.lvl = std::max(1, std::min(kLevelMax, c));
        }
        return best;
    }
    const double work = (double)F * (double)(ds.nnz_idx + ds.nnz_val);
    if (G != 8 || !model_independent(ds.model) || F < 16 || work < 1e8) return best;
    const TuneKey key{ds.model, ds.K, ds.J, F, G, ctl.precision, d_fold ? n_folds : 0, fixed_cols, ds.nnz_idx};
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = tuned_shapes().find({key, C});
        if (it != tuned_shapes().end()) return it->second;
    }
    auto time = [&](const BatchShape& sh) {
        return ctl.precision == CYC_MIXED
                   ? probe_cycle<float>(ds, stream, F, G, C, prior, specs, beta, hd, d_fold, n_folds, fit_fold, ctl,
                                        fixed_cols, sh)
                   : probe_cycle<double>(ds, stream, F, G, C, prior, specs, beta, hd, d_fold, n_folds, fit_fold,
                                         ctl, fixed_cols, sh);
    };
    float best_ms = time(best);
    auto consider = [&](BatchShape sh) {
        const float ms = time(sh);
        if (ms < best_ms) { best = sh; best_ms = ms; }
    };
    for (int cap : {128, 64}) { BatchShape sh = best; sh.cap = cap; consider(sh); }
    { BatchShape sh = best; sh.dmax = 16; consider(sh); }
    { BatchShape sh = best; sh.lvl = 2; consider(sh); }
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    tuned_shapes()[{key, C}] = best;
    return best;
}

// Fits the persistent kernel does not take -- Cox, whose risk sets follow
// each fit's weights and are rescanned after every moving coordinate, and
// fits under the KKT swindle, each with its own active set -- run
// concurrently: one device-resident single-fit CCD (cyc_fit: its own engine,
// stream and CUDA graphs) per host thread, up to CYC_CONCURRENT_FITS (default
// 8) at a time, so their kernels overlap on the device.  Each fit is the one
// cyc_fit computes alone.
void run_fits_concurrently(cyc_dataset* dsh, const cyc_prior* prior, const cyc_fit_spec* specs, int F,
                           const cyc_control* ctl, cyc_fit_result* out) {
    int slots = 8;
    if (const char* e = std::getenv("CYC_CONCURRENT_FITS")) slots = std::max(1, std::atoi(e));
    slots = std::min(slots, F);
    for (int f = 0; f < F; ++f)
        if (specs[f].start_beta) { dsh->ds.ensure_csr(); break; }     // built once, before the threads
    std::atomic<int> next{0};
    std::mutex mutex;                  // guards the error and the summed statistics
    int err_status = CYC_OK;
    std::string err_text;
    cyc_run_stats sum{};
    auto worker = [&] {
        for (;;) {
            const int f = next.fetch_add(1);
            if (f >= F) return;
            {
                std::lock_guard<std::mutex> lk(mutex);
                if (err_status != CYC_OK) return;
            }
            const int rc = cyc_fit(dsh, prior, &specs[f], ctl, &out[f]);
            std::lock_guard<std::mutex> lk(mutex);
            if (rc != CYC_OK) {
                if (err_status == CYC_OK) { err_status = rc; err_text = cyc_last_error(); }
                return;
            }
            cyc_run_stats st{};
            cyc_last_run_stats(&st);   // this worker thread's fit
            sum.algorithmic_bytes += st.algorithmic_bytes;
            sum.gradient_entries += st.gradient_entries;
            sum.update_entries += st.update_entries;
            sum.coordinate_steps += st.coordinate_steps;
            sum.index_entries += st.index_entries;
            sum.cycles += st.cycles;
            sum.phase_bytes[0] += st.phase_bytes[0];
            sum.phase_state_bytes[0] = st.phase_state_bytes[0];
        }
    };
    const long long launches0 = cyc_launch_count();
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < slots; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    CYC_REQUIRE(err_status == CYC_OK, err_status, err_text);
    // the fits overlap: the time is the whole concurrent section's (every
    // fit has synchronised its stream when cyc_fit returns)
    sum.kernel_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    sum.launches = (int)(cyc_launch_count() - launches0);
    sum.phases = 1;
    sum.phase_ms[0] = sum.kernel_ms;
    set_last_stats(sum);
}

// Whether the batch kernel runs a solve's KKT-swindle passes itself: the
// active sets are per-fit masks in the kernel and the inactive columns'
// scores one launch (independent-rows models, FP64 state).  Other swindle
// fits run as concurrent cyc_fit solves.
bool batch_swindle(const Dataset& ds, const cyc_control* ctl) {
    return model_independent(ds.model) && ctl->precision != CYC_MIXED;
}

// The shared driver of cyc_batch_fit and cyc_cv_grid_fit.  `d_fold` (fold id
// per row, `n_folds` of them) and `fit_fold` (the held-out fold of each fit)
// select the CV-grid weights; otherwise `specs[f].weights`.
void run_batch(Dataset& ds, const cyc_prior* prior, const cyc_fit_spec* specs, int F, const cyc_control* ctl,
               cyc_fit_result* out, const int* d_fold, int n_folds, const std::vector<int>* fit_fold,
               std::vector<double>* pll, int fixed_col = -1) {
    CYC_REQUIRE(!model_cumulative(ds.model), CYC_ERR_UNSUPPORTED,
                "batched fits support lr, pr, clr, cpr (use cyc_fit for cox)");
    CYC_REQUIRE(!ctl->use_kkt_swindle || batch_swindle(ds, ctl), CYC_ERR_UNSUPPORTED,
                "batched KKT-swindle fits support lr and pr at FP64");
    CYC_REQUIRE(ctl->convergence_type == CYC_CONV_GRADIENT || ctl->convergence_type == CYC_CONV_MITTAL ||
                    ctl->convergence_type == CYC_CONV_LANGE,
                CYC_ERR_UNSUPPORTED, "batched fits support gradient, mittal and lange convergence");
    CYC_REQUIRE(prior->prior_type >= CYC_PRIOR_NONE && prior->prior_type <= CYC_PRIOR_NORMAL, CYC_ERR_ARGUMENT,
                "Unknown prior type");
    for (int i = 0; i < prior->n_exclude; ++i)
        CYC_REQUIRE(prior->exclude[i] >= 0 && prior->exclude[i] < ds.J, CYC_ERR_ARGUMENT, "exclude index out of range");
    for (int f = 0; f < F; ++f) {
        CYC_REQUIRE(out[f].beta, CYC_ERR_ARGUMENT, "null result buffer");
        CYC_REQUIRE(specs[f].n_fixed >= 0 && (specs[f].n_fixed == 0 || specs[f].fixed), CYC_ERR_ARGUMENT,
                    "bad fixed-column list");
        CYC_REQUIRE(prior->prior_type == CYC_PRIOR_NONE || specs[f].variance > 0, CYC_ERR_ARGUMENT,
                    "prior variance must be positive");
    }
    // columns held fixed (besides the offset): the fits' shared fixed set and
    // the profiled column
    std::vector<int> fixed_cols(specs[0].fixed, specs[0].fixed + (specs[0].fixed ? specs[0].n_fixed : 0));
    for (int j : fixed_cols) CYC_REQUIRE(j >= 0 && j < ds.J, CYC_ERR_ARGUMENT, "fixed column out of range");
    std::sort(fixed_cols.begin(), fixed_cols.end());
    for (int f = 1; f < F; ++f) {
        std::vector<int> o(specs[f].fixed, specs[f].fixed + (specs[f].fixed ? specs[f].n_fixed : 0));
        std::sort(o.begin(), o.end());
        CYC_REQUIRE(o == fixed_cols, CYC_ERR_UNSUPPORTED, "the fits of one batched solve share their fixed columns");
    }
    if (fixed_col >= 0) fixed_cols.push_back(fixed_col);
    std::sort(fixed_cols.begin(), fixed_cols.end());
    fixed_cols.erase(std::unique(fixed_cols.begin(), fixed_cols.end()), fixed_cols.end());
    if (ds.has_offset) fixed_cols.erase(std::remove(fixed_cols.begin(), fixed_cols.end(), 0), fixed_cols.end());
    CYC_CHECK_CUDA(cudaSetDevice(ds.device));
    cudaStream_t stream;
    CYC_CHECK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamDestroy(s); } } sg{stream};
    StreamScope scope(stream);   // every buffer of this solve lives on `stream`
    const int J = ds.J;
    std::vector<double> beta((size_t)F * J, 0.0), hd((size_t)F * J, ctl->initial_bound);
    for (int f = 0; f < F; ++f) {
        if (specs[f].start_beta) std::copy(specs[f].start_beta, specs[f].start_beta + J, beta.begin() + (size_t)f * J);
        if (ds.has_offset) beta[(size_t)f * J] = 1.0;
    }
    const int G = F >= 4 ? 8 : 1;
    // the swindle runs when some column has a Laplace prior (a KKT boundary,
    // JointPrior.h:149-157); otherwise it is findMode itself
    std::vector<int> ptype(J, prior->prior_type);
    for (int i = 0; i < prior->n_exclude; ++i) ptype[prior->exclude[i]] = CYC_PRIOR_NONE;
    const bool swindle = ctl->use_kkt_swindle && std::count(ptype.begin(), ptype.end(), (int)CYC_PRIOR_LAPLACE) > 0;
    std::vector<int> iters, flags;
    std::vector<unsigned long long> ctr;
    cyc_run_stats st{};
    // Algorithmic bytes of one phase (the bytes the algorithm must move, not
    // what this kernel's layout re-reads): per cycle and column, the column's
    // row ids and values once (every group streams them, the fits share
    // them: the slowest group's count stands for all), per gradient visit of
    // a fit its linear predictor and weight (a CV grid's weight is one fold
    // byte per row shared by the group's G fits: 1/G B), per updated entry of
    // a fit its linear predictor read and written, and per convergence check
    // (linear predictor, weight) per fit plus y once.
    auto account = [&](int phase, float ms, const std::vector<int>& it, int s) {
        const double K = ds.K;
        const double wb = d_fold ? 1.0 / G : (double)s;
        double conv = 0.0;
        int mx = 0;
        for (int f = 0; f < F; ++f) {
            conv += (it[f] + 1) * K * (s + wb);
            mx = std::max(mx, it[f]);
        }
        conv += (mx + 1) * K * 8.0;
        double idx_once = 0.0, idx_all = 0.0;
        for (size_t g = 3; g < ctr.size(); ++g) {
            idx_once = std::max(idx_once, (double)ctr[g]);
            idx_all += (double)ctr[g];
        }
        const double bytes = idx_once + (double)ctr[0] * (s + wb) + (double)ctr[1] * 2.0 * s + conv;
        st.phase_ms[phase] = ms;
        st.phase_bytes[phase] = bytes;
        st.phase_state_bytes[phase] = s;
        st.kernel_ms += ms;
        st.algorithmic_bytes += bytes;
        st.gradient_entries += (double)ctr[0];
        st.update_entries += (double)ctr[1];
        st.coordinate_steps += (double)ctr[2];
        st.index_entries += idx_all;
        for (int f = 0; f < F; ++f) st.cycles += it[f];
        st.launches += 1;
        st.phases = phase + 1;
    };
    // the tuners time whole cycles over every column, which an active-set
    // pass does not run: swindle solves keep the defaults
    int C = default_cluster(ds.K);
    if (!swindle) {
        NvtxRange range("cyclops batch: cluster tuner");
        C = tuned_cluster(ds, stream, F, G, *prior, specs, beta, hd, d_fold, n_folds, fit_fold, *ctl, fixed_cols);
    }
    BatchShape shape;
    if (!swindle) {
        NvtxRange range("cyclops batch: shape tuner");
        shape = tuned_shape(ds, stream, F, G, C, *prior, specs, beta, hd, d_fold, n_folds, fit_fold, *ctl,
                            fixed_cols);
    }
    int phase = 0;
    if (ctl->precision == CYC_MIXED) {
        // FP32 state + compensated sums to the looser tolerance, then the FP64 polish below
        NvtxRange range("cyclops batch: fp32 phase");
        BatchRunner<float> r32(ds, stream, F, G, C, shape);
        if (d_fold) r32.set_folds(d_fold, n_folds, *fit_fold);
        r32.setup(*prior, specs, beta, hd, fixed_cols);
        float ms = 0.f;
        r32.run(*ctl, std::max(ctl->polish_tolerance, ctl->tolerance), &ms);
        r32.results(beta, hd, iters, flags, ctr);
        account(phase++, ms, iters, (int)sizeof(float));
        // the FP64 phase restarts the trust regions (resetBounds, :943)
        std::fill(hd.begin(), hd.end(), ctl->initial_bound);
    }
    NvtxRange range64("cyclops batch: fp64 phase");
    BatchRunner<double> r64(ds, stream, F, G, C, shape);
    if (d_fold) r64.set_folds(d_fold, n_folds, *fit_fold);
    float ms = 0.f;
    std::vector<int> it64;
    if (!swindle) {
        r64.setup(*prior, specs, beta, hd, fixed_cols);
        r64.run(*ctl, ctl->tolerance, &ms);
        r64.results(beta, hd, it64, flags, ctr);
        account(phase, ms, it64, (int)sizeof(double));
    } else {
        // kktSwindle (CyclicCoordinateDescent.cpp:636-814) for every fit at
        // once.  The intercept and the columns whose prior has no KKT
        // boundary start active, the Laplace columns inactive at beta 0.
        // Each pass is one launch: a fit holds its inactive columns fixed
        // (findMode over the active set, :617-634, with fresh trust regions),
        // and a batch every running fit holds fixed is skipped.  Then one
        // launch scores every running fit's inactive columns (|gradient|)
        // and each fit moves the columns above its lambda into its active
        // set.  A fit stops when nothing is inactive, its pass failed, no
        // column violates, or after max_iterations passes (MAX_ITERATIONS);
        // an empty active set skips the pass's findMode.  Reported cycles
        // are the last pass's, as lastIterationCount.
        const int intercept = ds.has_intercept ? (ds.has_offset ? 1 : 0) : -1;
        std::vector<char> fixc(J, 0);
        for (int j : fixed_cols) fixc[j] = 1;
        if (ds.has_offset) fixc[0] = 1;
        std::vector<unsigned char> lfix((size_t)r64.ngroups * J, 0);
        std::vector<int> n_act(F, 0), n_inact(F, 0);
        for (int f = 0; f < F; ++f)
            for (int j = 0; j < J; ++j) {
                if (fixc[j]) continue;
                if (j == intercept || ptype[j] != CYC_PRIOR_LAPLACE) {
                    ++n_act[f];
                } else {
                    ++n_inact[f];
                    lfix[(size_t)(f / G) * J + j] |= (unsigned char)(1u << (f % G));
                    beta[(size_t)f * J + j] = 0.0;          // setBeta(0) of a nonzero start
                }
            }
        r64.setup(*prior, specs, beta, hd, fixed_cols);
        std::vector<int> running(F, 1), run_k(F, 0), it_last(F, 0), total_it(F, 0), itp, flp;
        flags.assign(F, CYC_SUCCESS);
        std::vector<double> score;
        for (int pass = 1;; ++pass) {
            bool any = false;
            for (int f = 0; f < F; ++f) {
                run_k[f] = running[f] && n_act[f] > 0;
                any |= run_k[f] != 0;
                if (running[f]) flags[f] = CYC_SUCCESS;
            }
            if (any) {
                r64.set_pass(lfix, run_k, ctl->initial_bound);
                float pm = 0.f;
                r64.run(*ctl, ctl->tolerance, &pm);
                ms += pm;
                r64.results(beta, hd, itp, flp, ctr);
                for (int f = 0; f < F; ++f)
                    if (run_k[f]) {
                        it_last[f] = itp[f];
                        total_it[f] += itp[f];
                        flags[f] = flp[f];
                    }
            }
            std::vector<unsigned char> need((size_t)r64.ngroups * J, 0);
            bool any_need = false;
            for (int f = 0; f < F; ++f) {
                if (!running[f]) continue;
                if (n_inact[f] == 0 || flags[f] != CYC_SUCCESS) { running[f] = 0; continue; }
                if (pass == ctl->max_iterations) { flags[f] = CYC_MAX_ITERATIONS; running[f] = 0; continue; }
                const unsigned char bit = (unsigned char)(1u << (f % G));
                const size_t g0 = (size_t)(f / G) * J;
                for (int j = 0; j < J; ++j)
                    if (lfix[g0 + j] & bit) need[g0 + j] |= bit;
                any_need = true;
            }
            if (!any_need) break;
            r64.kkt_scores(need, score);
            for (int f = 0; f < F; ++f) {
                if (!running[f]) continue;
                const double lambda = std::sqrt(2.0 / specs[f].variance);   // getKktBoundary, CovariatePrior.h:235-238
                const unsigned char bit = (unsigned char)(1u << (f % G));
                const size_t g0 = (size_t)(f / G) * J;
                int moved = 0;
                for (int j = 0; j < J; ++j)
                    if ((need[g0 + j] & bit) && !(score[(size_t)f * J + j] <= lambda)) {
                        lfix[g0 + j] &= (unsigned char)~bit;
                        ++moved;
                    }
                if (moved == 0) running[f] = 0;
                n_act[f] += moved;
                n_inact[f] -= moved;
            }
        }
        it64 = it_last;
        account(phase, ms, total_it, (int)sizeof(double));
    }
    std::vector<double> ll, p;
    r64.finalize(ll, p);
    std::vector<int> pt(J, prior->prior_type);
    for (int i = 0; i < prior->n_exclude; ++i) pt[prior->exclude[i]] = CYC_PRIOR_NONE;
    for (int f = 0; f < F; ++f) {
        std::copy(beta.begin() + (size_t)f * J, beta.begin() + (size_t)(f + 1) * J, out[f].beta);
        out[f].iterations = it64[f];
        out[f].return_flag = flags[f];
        out[f].log_likelihood = ll[f];
        double lp = 0.0;
        for (int j = 0; j < J; ++j) lp += log_density(pt[j], specs[f].variance, out[f].beta[j]);
        out[f].log_prior = lp;
    }
    if (pll) pll->assign(p.begin(), p.begin() + F);
    st.cluster_ctas = C;
    if (G == 8 && model_independent(ds.model)) {
        st.batch_cap = shape.cap;
        st.batch_shared_rows = shape.dmax;
        st.batch_levels = shape.lvl;
    }
    set_last_stats(st);
}

}  // namespace

extern "C" int cyc_batch_fit(cyc_dataset* dsh, const cyc_prior* prior, const cyc_fit_spec* specs, int F,
                             const cyc_control* ctl, cyc_fit_result* out) {
    return guarded([&] {
        NvtxRange range("cyc_batch_fit");
        CYC_REQUIRE(dsh && prior && specs && ctl && out && F > 0, CYC_ERR_ARGUMENT, "null argument");
        if (model_cumulative(dsh->ds.model) || (ctl->use_kkt_swindle && !batch_swindle(dsh->ds, ctl))) {
            // cox fits carry their own risk sets, and swindle fits of grouped
            // models or mixed precision their own active sets, which one
            // batch kernel does not share: they run as concurrent cyc_fit calls
            run_fits_concurrently(dsh, prior, specs, F, ctl, out);
            return;
        }
        run_batch(dsh->ds, prior, specs, F, ctl, out, nullptr, 0, nullptr, nullptr);
    });
}

extern "C" int cyc_cv_grid_fit(cyc_dataset* dsh, const cyc_prior* prior, const int* fold_of_row, int n_folds,
                               const double* variances, int n_var, const cyc_control* ctl, cyc_fit_result* out,
                               double* pred_loglik, double* grid_mean) {
    return guarded([&] {
        NvtxRange range("cyc_cv_grid_fit");
        CYC_REQUIRE(dsh && prior && fold_of_row && variances && ctl && out && n_folds > 1 && n_var > 0,
                    CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(n_folds <= 127, CYC_ERR_ARGUMENT, "at most 127 folds");
        Dataset& ds = dsh->ds;
        for (int k = 0; k < ds.K; ++k)
            CYC_REQUIRE(fold_of_row[k] >= 0 && fold_of_row[k] < n_folds, CYC_ERR_ARGUMENT, "fold id out of range");
        if (model_cumulative(ds.model) || (ctl->use_kkt_swindle && !batch_swindle(ds, ctl))) {
            // per-fit risk sets (cox) or active sets the kernel does not run: the per-fit path, unit weights
            std::vector<double> ones(ds.K, 1.0);
            const int rc = cyc_cv_grid_fit_weighted(dsh, prior, fold_of_row, n_folds, ones.data(), variances, n_var,
                                                    ctl, out, pred_loglik, grid_mean);
            CYC_REQUIRE(rc == CYC_OK, rc, cyc_last_error());
            return;
        }
        CYC_CHECK_CUDA(cudaSetDevice(ds.device));
        const int F = n_folds * n_var;
        std::vector<cyc_fit_spec> specs(F);
        std::vector<int> fit_fold(F);
        for (int i = 0; i < F; ++i) {
            specs[i].weights = nullptr;
            specs[i].variance = variances[i / n_folds];
            specs[i].start_beta = nullptr;
            fit_fold[i] = i % n_folds;
        }
        StreamScope scope(ds.stream);
        DevBuf<int> d_fold;
        d_fold.alloc(ds.K);
        CYC_CHECK_CUDA(cudaMemcpyAsync(d_fold.get(), fold_of_row, ds.K * sizeof(int), cudaMemcpyHostToDevice, ds.stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(ds.stream));
        std::vector<double> pll;
        run_batch(ds, prior, specs.data(), F, ctl, out, d_fold.get(), n_folds, &fit_fold, &pll);
        // AbstractCrossValidationDriver: NaN for fits that did not converge;
        // the grid point's estimate is the mean over folds ignoring NaN
        // (computePointEstimate, AbstractCrossValidationDriver.cpp:252-264)
        for (int i = 0; i < F; ++i)
            if (out[i].return_flag != CYC_SUCCESS) pll[i] = std::nan("");
        if (pred_loglik) std::copy(pll.begin(), pll.end(), pred_loglik);
        if (grid_mean)
            for (int v = 0; v < n_var; ++v) {
                double tot = 0.0;
                int cnt = 0;
                for (int f = 0; f < n_folds; ++f) {
                    const double x = pll[v * n_folds + f];
                    if (x == x) { tot += x; ++cnt; }
                }
                grid_mean[v] = tot / cnt;
            }
    });
}

// getCyclopsProfileLogLikelihood as one batched solve: every point is a fit
// of the persistent kernel, started from the mode with the column moved to
// the point and held there (the column joins the offset as a fixed column),
// so all points refit together instead of one after another.  Each fit
// starts from the mode, as evaluateProfileModel's per-thread clones do
// (CcdInterface.cpp:545-598); the one-thread, warm-start-chained order is
// cyc_profile_log_likelihood.
extern "C" int cyc_profile_log_likelihood_batch(cyc_dataset* dsh, const cyc_prior* prior, const cyc_fit_spec* spec,
                                                const cyc_control* ctl, int column, const double* points, int n,
                                                int include_penalty, double* values) {
    return guarded([&] {
        NvtxRange range("cyc_profile_log_likelihood_batch");
        CYC_REQUIRE(dsh && prior && spec && ctl && n >= 0 && (n == 0 || (points && values)), CYC_ERR_ARGUMENT,
                    "null argument");
        Dataset& ds = dsh->ds;
        const int J = ds.J;
        CYC_REQUIRE(column >= 0 && column < J && !(ds.has_offset && column == 0), CYC_ERR_ARGUMENT,
                    "profile column out of range (or the offset)");
        if (n == 0) return;
        std::vector<double> mode(J, 0.0);
        if (spec->start_beta) {
            std::copy(spec->start_beta, spec->start_beta + J, mode.begin());
        } else {                                          // fit the mode first
            cyc_fit_result r{};
            r.beta = mode.data();
            cyc_fit_spec s0 = *spec;
            run_batch(ds, prior, &s0, 1, ctl, &r, nullptr, 0, nullptr, nullptr);
        }
        std::vector<double> starts((size_t)n * J), outb((size_t)n * J);
        std::vector<cyc_fit_spec> specs(n, *spec);
        std::vector<cyc_fit_result> out(n);
        for (int i = 0; i < n; ++i) {
            std::copy(mode.begin(), mode.end(), starts.begin() + (size_t)i * J);
            starts[(size_t)i * J + column] = points[i];
            specs[i].start_beta = starts.data() + (size_t)i * J;
            out[i].beta = outb.data() + (size_t)i * J;
        }
        run_batch(ds, prior, specs.data(), n, ctl, out.data(), nullptr, 0, nullptr, nullptr, column);
        for (int i = 0; i < n; ++i)
            values[i] = out[i].log_likelihood + (include_penalty ? out[i].log_prior : 0.0);
    });
}

// ---- auto-search cross-validation ---------------------------------------------
//
// AutoSearchCrossValidationDriver::doCrossValidationLoop
// (src/cyclops/drivers/AutoSearchCrossValidationDriver.cpp:63-160): one
// variance at a time, every fold (of every repetition) refit at it, the
// held-out predictive log likelihoods' mean and standard deviation
// (computePointEstimate / computeStDev, AbstractCrossValidationDriver.cpp:
// 252-276) handed to UniModalSearch (src/utils/HParSearch.cpp), which
// proposes the next variance.  Each step's folds are one batched solve here.
// Every fit cold-starts (the reference's resetCoefficients).
namespace {

// getNormalBasedDefaultVar (ModelData.cpp:680-728): the summed squares of
// the variable columns (those after the offset and intercept) / their
// count / K
double normal_based_default_variance(Dataset& ds) {
    const int start = (ds.has_intercept ? 1 : 0) + (ds.has_offset ? 1 : 0);
    CYC_REQUIRE(ds.J > start, CYC_ERR_ARGUMENT, "no variable columns");
    std::vector<double> val(ds.nnz_val);
    if (ds.nnz_val) {
        CYC_CHECK_CUDA(cudaMemcpyAsync(val.data(), ds.d_val.get(), ds.nnz_val * sizeof(double),
                                       cudaMemcpyDeviceToHost, ds.stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(ds.stream));
    }
    double total = 0.0;
    for (int j = start; j < ds.J; ++j) {
        const int f = ds.fmt[j];
        if (f == CYC_INDICATOR) {
            total += (double)(ds.col_ptr[j + 1] - ds.col_ptr[j]);
        } else if (f == CYC_INTERCEPT) {
            total += (double)ds.K;
        } else {
            double s = 0.0;
            for (long long e = ds.val_ptr[j]; e < ds.val_ptr[j + 1]; ++e) s += val[e] * val[e];
            total += s;
        }
    }
    return total / (ds.J - start) / ds.K;
}

}  // namespace

extern "C" int cyc_cv_auto_search(cyc_dataset* dsh, const cyc_prior* prior, const int* fold_of_row, int n_folds,
                                  int n_reps, const double* row_weights, double starting_variance,
                                  const cyc_control* ctl,
                                  double* best_variance, double* best_value, double* tried_variance,
                                  double* tried_mean, double* tried_sd, int max_tried, int* n_tried) {
    return guarded([&] {
        NvtxRange range("cyc_cv_auto_search");
        CYC_REQUIRE(dsh && prior && fold_of_row && ctl && best_variance && best_value && n_folds > 1 && n_reps > 0,
                    CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(n_folds <= 127, CYC_ERR_ARGUMENT, "at most 127 folds");
        CYC_REQUIRE(max_tried <= 0 || (tried_variance && tried_mean && tried_sd), CYC_ERR_ARGUMENT, "null argument");
        Dataset& ds = dsh->ds;
        for (long long k = 0; k < (long long)ds.K * n_reps; ++k)
            CYC_REQUIRE(fold_of_row[k] >= 0 && fold_of_row[k] < n_folds, CYC_ERR_ARGUMENT, "fold id out of range");
        CYC_CHECK_CUDA(cudaSetDevice(ds.device));
        StreamScope scope(ds.stream);
        const int J = ds.J;
        double x = starting_variance > 0 ? starting_variance : normal_based_default_variance(ds);
        std::vector<DevBuf<int>> d_folds(n_reps);
        for (int r = 0; r < n_reps; ++r) {
            d_folds[r].alloc(ds.K);
            CYC_CHECK_CUDA(cudaMemcpyAsync(d_folds[r].get(), fold_of_row + (size_t)r * ds.K, ds.K * sizeof(int),
                                           cudaMemcpyHostToDevice, ds.stream));
        }
        CYC_CHECK_CUDA(cudaStreamSynchronize(ds.stream));
        std::vector<int> fit_fold(n_folds);
        for (int f = 0; f < n_folds; ++f) fit_fold[f] = f;
        std::vector<double> betas((size_t)n_folds * J);
        std::vector<cyc_fit_result> out(n_folds);
        std::vector<double> ones(row_weights ? 0 : ds.K, 1.0);
        cyc::VarianceSearch search;
        double value = 0.0;
        int tried = 0;
        for (int step = 0; step < 50; ++step) {            // MAX_STEPS, AutoSearchCrossValidationDriver.cpp:28
            std::vector<double> pll_all;
            for (int r = 0; r < n_reps; ++r) {
                if (row_weights || ctl->use_kkt_swindle || model_cumulative(ds.model)) {
                    // observation weights, per-fit active sets or risk sets: the weighted grid path
                    std::vector<double> w(row_weights ? row_weights : ones.data(),
                                          (row_weights ? row_weights : ones.data()) + ds.K);
                    std::vector<double> pll(n_folds);
                    for (int f = 0; f < n_folds; ++f) {
                        out[f] = cyc_fit_result{};
                        out[f].beta = betas.data() + (size_t)f * J;
                    }
                    const int rc = cyc_cv_grid_fit_weighted(dsh, prior, fold_of_row + (size_t)r * ds.K, n_folds,
                                                            w.data(), &x, 1, ctl, out.data(), pll.data(), nullptr);
                    CYC_REQUIRE(rc == CYC_OK, rc, cyc_last_error());
                    pll_all.insert(pll_all.end(), pll.begin(), pll.end());
                    continue;
                }
                std::vector<cyc_fit_spec> specs(n_folds);
                for (int f = 0; f < n_folds; ++f) {
                    specs[f] = cyc_fit_spec{};
                    specs[f].variance = x;
                    out[f] = cyc_fit_result{};
                    out[f].beta = betas.data() + (size_t)f * J;
                }
                std::vector<double> pll;
                run_batch(ds, prior, specs.data(), n_folds, ctl, out.data(), d_folds[r].get(), n_folds, &fit_fold,
                          &pll);
                for (int f = 0; f < n_folds; ++f)
                    pll_all.push_back(out[f].return_flag == CYC_SUCCESS ? pll[f] : std::nan(""));
            }
            double total = 0.0, inner = 0.0;
            int count = 0;
            for (double v : pll_all)
                if (v == v) { total += v; ++count; }
            const double mean = total / count;
            for (double v : pll_all)
                if (v == v) inner += v * v;
            const double sd = std::sqrt(inner / count - mean * mean);
            if (tried < max_tried) {
                tried_variance[tried] = x;
                tried_mean[tried] = mean;
                tried_sd[tried] = sd;
            }
            ++tried;
            search.tried(x, mean, sd);
            bool go;
            search.step(&go, &x, &value);
            if (!go) break;
        }
        *best_variance = x;
        *best_value = value;
        if (n_tried) *n_tried = tried;
    });
}

// Cross-validation with observation weights (CrossValidationSelector with
// wtsOriginal, src/cyclops/drivers/CrossValidationSelector.cpp:72-124, as
// CcdInterface::runCrossValidation passes the fit's weights, :738-754): fit
// (variance v, fold f) trains with the original weight on rows outside fold
// f and 0 on it, and is scored on fold f's rows at their original weights
// (getComplement).  The fits run as one batched solve with per-fit weights;
// each held-out predictive log likelihood is one engine evaluation at the
// fit's coefficients (getNewPredictiveLogLikelihood, CyclicCoordinateDescent
// .cpp:319-353).  Cold starts, as cyc_cv_grid_fit.
extern "C" int cyc_cv_grid_fit_weighted(cyc_dataset* dsh, const cyc_prior* prior, const int* fold_of_row,
                                        int n_folds, const double* row_weights, const double* variances, int n_var,
                                        const cyc_control* ctl, cyc_fit_result* out, double* pred_loglik,
                                        double* grid_mean) {
    return guarded([&] {
        NvtxRange range("cyc_cv_grid_fit_weighted");
        CYC_REQUIRE(dsh && prior && fold_of_row && row_weights && variances && ctl && out && n_folds > 1 && n_var > 0,
                    CYC_ERR_ARGUMENT, "null argument");
        Dataset& ds = dsh->ds;
        const int K = ds.K;
        for (int k = 0; k < K; ++k) {
            CYC_REQUIRE(fold_of_row[k] >= 0 && fold_of_row[k] < n_folds, CYC_ERR_ARGUMENT, "fold id out of range");
            CYC_REQUIRE(std::isfinite(row_weights[k]) && row_weights[k] >= 0, CYC_ERR_ARGUMENT,
                        "weights must be finite and nonnegative");
        }
        CYC_CHECK_CUDA(cudaSetDevice(ds.device));
        const int F = n_folds * n_var;
        std::vector<double> train((size_t)n_folds * K), held((size_t)n_folds * K);
        for (int f = 0; f < n_folds; ++f)
            for (int k = 0; k < K; ++k) {
                const bool out_f = fold_of_row[k] == f;
                train[(size_t)f * K + k] = out_f ? 0.0 : row_weights[k];
                held[(size_t)f * K + k] = out_f ? row_weights[k] : 0.0;
            }
        std::vector<cyc_fit_spec> specs(F);
        for (int i = 0; i < F; ++i) {
            specs[i] = cyc_fit_spec{};
            specs[i].weights = train.data() + (size_t)(i % n_folds) * K;
            specs[i].variance = variances[i / n_folds];
        }
        if (model_cumulative(ds.model) || (ctl->use_kkt_swindle && !batch_swindle(ds, ctl))) {
            run_fits_concurrently(dsh, prior, specs.data(), F, ctl, out);
        } else {
            run_batch(ds, prior, specs.data(), F, ctl, out, nullptr, 0, nullptr, nullptr);
        }
        std::vector<double> pll(F);
        {
            Engine eng(&ds);
            StreamScope scope(eng.stream);
            for (int i = 0; i < F; ++i) {
                if (out[i].return_flag != CYC_SUCCESS) {       // AbstractCrossValidationDriver.cpp:236-240
                    pll[i] = std::nan("");
                    continue;
                }
                const int f = i % n_folds;
                eng.set_weights(train.data() + (size_t)f * K, true);
                eng.compute_xbeta(out[i].beta);
                eng.remaining_statistics(true);
                pll[i] = eng.predictive_log_likelihood(held.data() + (size_t)f * K);
            }
        }
        if (pred_loglik) std::copy(pll.begin(), pll.end(), pred_loglik);
        if (grid_mean)
            for (int v = 0; v < n_var; ++v) {
                double tot = 0.0;
                int cnt = 0;
                for (int f = 0; f < n_folds; ++f) {
                    const double x = pll[v * n_folds + f];
                    if (x == x) { tot += x; ++cnt; }
                }
                grid_mean[v] = tot / cnt;
            }
    });
}
