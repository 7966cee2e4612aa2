// engine_kernels.cuh -- FP64 kernels of the per-coordinate engine.
//
// Each kernel restates one piece of the reference engine
// (src/cyclops/engine/ModelSpecifics.hpp) for the GPU; the reference
// function is named above each kernel.  Reductions are deterministic:
// per-block partials are combined in block order by the last block
// (grid_sum2_finalize), so a result does not depend on scheduling.
#pragma once
#include "internal.cuh"

namespace cyc {

// ---- weights ---------------------------------------------------------------

// setWeights, hKWeight (ModelSpecifics.hpp:428-440)
__global__ void k_set_kw(int K, const double* __restrict__ w, double* __restrict__ kw) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        kw[k] = w ? w[k] : 1.0;
}

// setWeights, hNWeight for independent rows: 0 + observationCount(y)*w (:451-455)
__global__ void k_nw_independent(int K, const double* __restrict__ kw, double* __restrict__ nw) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        nw[k] = 0.0 + 1.0 * kw[k];
}

// setWeights, hNWeight for grouped rows: per-group sequential sum of y*w in row
// order (same order as the reference's incrementByGroup loop, :451-455)
__global__ void k_nw_grouped(int G, const int* __restrict__ grow_ptr, const double* __restrict__ y,
                             const double* __restrict__ kw, double* __restrict__ nw) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = grow_ptr[g]; k < grow_ptr[g + 1]; ++k) s += y[k] * kw[k];
        nw[g] = s;
    }
}

// computeXjY (ModelSpecifics.hpp:486-524): one block per column
__global__ void k_xjy(int J, const int* __restrict__ fmt, const long long* __restrict__ col_ptr,
                      const long long* __restrict__ val_ptr, const int* __restrict__ idx,
                      const double* __restrict__ val, int K, const double* __restrict__ y,
                      const double* __restrict__ kw, int use_w, double* __restrict__ xjy) {
    for (int j = blockIdx.x; j < J; j += gridDim.x) {
        ColView c;
        c.fmt = fmt[j];
        c.n = (c.fmt == CYC_DENSE || c.fmt == CYC_INTERCEPT) ? K : col_ptr[j + 1] - col_ptr[j];
        c.idx = idx + col_ptr[j];
        c.val = val + val_ptr[j];
        double s = 0.0, dummy = 0.0;
        for (long long e = threadIdx.x; e < c.n; e += blockDim.x) {
            const int k = c.row(e);
            s += use_w ? c.x(e) * y[k] * kw[k] : c.x(e) * y[k];
        }
        block_sum2(s, dummy);
        if (threadIdx.x == 0) xjy[j] = s;
        __syncthreads();
    }
}

// computeFixedTermsInLogLikelihood (ModelSpecifics.hpp:570-587): -sum log(y!)
__global__ void k_fixed_ll(int K, const double* __restrict__ y, const double* __restrict__ kw,
                           int use_w, double2* partial, unsigned* ticket, double* out) {
    double s = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        double f = 0.0;
        for (int i = 2; i <= (int)y[k]; ++i) f -= log((double)i);
        s += use_w ? f * kw[k] : f;
    }
    grid_sum2_finalize(s, 0.0, partial, ticket, [&](double a, double) { *out = a; });
}

// ---- linear predictor ------------------------------------------------------

// zeroXBeta + axpyXBeta over all columns in order (CyclicCoordinateDescent.cpp:1452-1470)
__global__ void k_xbeta_rows(int K, const long long* __restrict__ row_ptr, const int* __restrict__ row_col,
                             const double* __restrict__ row_val, const double* __restrict__ beta,
                             double* __restrict__ xb) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (long long p = row_ptr[k]; p < row_ptr[k + 1]; ++p) {
            const double b = beta[row_col[p]];
            if (b != 0.0) s = add_mul_rn(s, b, row_val[p]);
        }
        xb[k] = s;
    }
}

// axpy (ModelSpecifics.hpp:384-391)
__global__ void k_axpy(ColView c, double beta, double* __restrict__ xb) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = c.row(e);
        xb[k] = add_mul_rn(xb[k], beta, c.x(e));
    }
}

// ---- remaining statistics (ModelSpecifics.hpp:1588-1612) --------------------

__global__ void k_rs_independent(int K, int model, const double* __restrict__ xb,
                                 double* __restrict__ exb, double* __restrict__ denom) {
    const double nul = denom_null(model);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        const double e = exp(xb[k]);
        exb[k] = e;
        denom[k] = nul + e;
    }
}

// grouped / cumulative: exp per row and a per-group sum in row order
__global__ void k_rs_grouped(int G, const int* __restrict__ grow_ptr, const double* __restrict__ xb,
                             const double* __restrict__ kw, int weighted, double* __restrict__ exb,
                             double* __restrict__ denom) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = grow_ptr[g]; k < grow_ptr[g + 1]; ++k) {
            const double e = exp(xb[k]);
            exb[k] = e;
            if (!weighted) s += e;
            else if (kw[k] != 0.0) s += kw[k] * e;
        }
        denom[g] = s;
    }
}

// ---- Fisher information (ModelSpecifics.hpp:1203-1351) ------------------------

// per row, the factor of x_i * x_j in incrementFisherInformation: Logistic
// (ModelSpecifics.h:524-538) p - p^2 with p = exb / denom; PoissonRegression
// (:1497-1506) exb; the grouped models' Survival (:488-497) exb / denom of
// the row's stratum.  Unweighted, as the reference (:1207-1209).
__global__ void k_fisher_row(int K, int model, const double* __restrict__ exb, const double* __restrict__ denom,
                             const int* __restrict__ strat, double* __restrict__ v) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        if (model == CYC_LR) {
            const double g = exb[k] / denom[k];
            v[k] = exb[k] / denom[k] - g * g;
        } else if (model == CYC_PR) {
            v[k] = exb[k];
        } else {
            v[k] = exb[k] / denom[strat[k]];
        }
    }
}

__device__ __forceinline__ ColView fisher_view(int j, int K, const int* fmt, const long long* col_ptr,
                                               const long long* val_ptr, const int* idx, const double* val) {
    ColView c;
    c.fmt = fmt[j];
    c.n = (c.fmt == CYC_DENSE || c.fmt == CYC_INTERCEPT) ? K : col_ptr[j + 1] - col_ptr[j];
    c.idx = idx + col_ptr[j];
    c.val = val + val_ptr[j];
    return c;
}

// row k in column c (binary search of its ascending row ids): its value, or false
__device__ __forceinline__ bool fisher_lookup(const ColView& c, int k, double& x) {
    if (c.fmt == CYC_DENSE) { x = __ldg(c.val + k); return true; }
    if (c.fmt == CYC_INTERCEPT) { x = 1.0; return true; }
    long long lo = 0, hi = c.n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (__ldg(c.idx + mid) < k) lo = mid + 1;
        else hi = mid;
    }
    if (lo < c.n && __ldg(c.idx + lo) == k) {
        x = c.fmt == CYC_SPARSE ? __ldg(c.val + lo) : 1.0;
        return true;
    }
    return false;
}

// grouped models: per column of the set, its per-stratum sums of x * exb
// (getSubjectSpecificHessianIterator, ModelSpecifics.hpp:1247-1270), dense
// over strata (t[c * S + s], zero where the column has no row); the first
// entry of each run of one stratum walks the run
__global__ void k_fisher_strata(int n_cols, const int* __restrict__ cols, int K, int S, const int* fmt,
                                const long long* col_ptr, const long long* val_ptr, const int* idx,
                                const double* val, const int* __restrict__ strat, const double* __restrict__ exb,
                                double* __restrict__ t) {
    for (int c = blockIdx.x; c < n_cols; c += gridDim.x) {
        const ColView a = fisher_view(cols[c], K, fmt, col_ptr, val_ptr, idx, val);
        for (long long e = threadIdx.x; e < a.n; e += blockDim.x) {
            const int k = a.row(e), s = strat[k];
            if (e > 0 && strat[a.row(e - 1)] == s) continue;
            double sum = 0.0;
            long long q = e;
            do {
                const int kq = a.row(q);
                sum += exb[kq] * a.x(q);
                ++q;
            } while (q < a.n && strat[a.row(q)] == s);
            t[(size_t)c * S + s] = sum;
        }
    }
}

// one block per pair (a, b) of the set: the sum over the rows of both columns
// of v_k * x_a * x_b (PairProductIterator, :1276-1289), walking the shorter
// column and looking its rows up in the other; grouped models subtract
// sum_s t_a(s) t_b(s) / denom_s^2 (:1296-1347).  Fixed order: deterministic.
__global__ void k_fisher_pairs(int n_pairs, const int* __restrict__ pa, const int* __restrict__ pb,
                               const int* __restrict__ cols, int K, int S, int grouped, const int* fmt,
                               const long long* col_ptr, const long long* val_ptr, const int* idx,
                               const double* val, const double* __restrict__ v, const int* __restrict__ strat,
                               const double* __restrict__ denom, const double* __restrict__ t,
                               double* __restrict__ out) {
    for (int p = blockIdx.x; p < n_pairs; p += gridDim.x) {
        ColView a = fisher_view(cols[pa[p]], K, fmt, col_ptr, val_ptr, idx, val);
        ColView b = fisher_view(cols[pb[p]], K, fmt, col_ptr, val_ptr, idx, val);
        if (b.n < a.n) { const ColView tmp = a; a = b; b = tmp; }
        double info = 0.0, cross = 0.0;
        for (long long e = threadIdx.x; e < a.n; e += blockDim.x) {
            const int k = a.row(e);
            double xb;
            if (fisher_lookup(b, k, xb)) info += v[k] * (a.x(e) * xb);
        }
        if (grouped) {
            const double* ta = t + (size_t)pa[p] * S;
            const double* tb = t + (size_t)pb[p] * S;
            const ColView c = fisher_view(cols[pa[p]], K, fmt, col_ptr, val_ptr, idx, val);
            for (long long e = threadIdx.x; e < c.n; e += blockDim.x) {
                const int s = strat[c.row(e)];
                if (e > 0 && strat[c.row(e - 1)] == s) continue;
                cross += (ta[s] * tb[s]) / (denom[s] * denom[s]);
            }
        }
        block_sum2(info, cross);
        if (threadIdx.x == 0) out[p] = info - cross;
        __syncthreads();
    }
}

// ---- gradient and Hessian ---------------------------------------------------

// independent rows (ModelSpecifics.hpp:1022-1038 with LogisticRegression /
// PoissonRegression::incrementGradientAndHessian, ModelSpecifics.h:540-568, 1508-1543)
template <int MODEL, bool IND>
__global__ void k_gh_independent(ColView c, const double* __restrict__ exb, const double* __restrict__ denom,
                                 const double* __restrict__ nw, int use_w, const double* __restrict__ xjy, int j,
                                 double2* partial, unsigned* ticket, double* out) {
    double g = 0.0, h = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = c.row(e);
        const double x = c.x(e);
        const double ex = exb[k];
        const double n1 = ex * x;
        const double w = use_w ? nw[k] : 1.0;
        if (MODEL == CYC_LR) {
            const double d = denom[k];
            const double gi = n1 / d;
            g += w * gi;
            h += w * (IND ? gi * (1.0 - gi) : (n1 * x / d - gi * gi));
        } else {
            g += w * n1;
            h += w * (IND ? n1 : n1 * x);
        }
    }
    grid_sum2_finalize(g, h, partial, ticket, [&](double G, double H) {
        out[0] = G - xjy[j];
        out[1] = H;
    });
}

// grouped rows (ModelSpecifics.hpp:1127-1178 with
// ConditionalLogisticRegression::incrementGradientAndHessian, ModelSpecifics.h:820-837):
// the first entry of each run of equal stratum walks the run.
template <bool IND>
__global__ void k_gh_grouped(ColView c, const int* __restrict__ group, const double* __restrict__ exb,
                             const double* __restrict__ denom, const double* __restrict__ nw,
                             const double* __restrict__ xjy, int j, double2* partial, unsigned* ticket,
                             double* out) {
    double g = 0.0, h = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int key = group[c.row(e)];
        if (e > 0 && group[c.row(e - 1)] == key) continue;
        double n1 = 0.0, n2 = 0.0;
        long long f = e;
        do {
            const int k = c.row(f);
            const double x = c.x(f);
            n1 += exb[k] * x;
            if (!IND) n2 += exb[k] * x * x;
            ++f;
        } while (f < c.n && group[c.row(f)] == key);
        const double d = denom[key];
        const double t = n1 / d;
        const double gg = nw[key] * t;
        g += gg;
        h += IND ? gg * (1.0 - t) : nw[key] * (n2 / d - t * t);
    }
    grid_sum2_finalize(g, h, partial, ticket, [&](double G, double H) {
        out[0] = G - xjy[j];
        out[1] = H;
    });
}

// computeNumeratorForGradient for cox (ModelSpecifics.hpp:1353-1464):
// numer[g] = sum of w*exb*x over the column's rows in risk-set group g
template <bool IND>
__global__ void k_cox_numerator(ColView c, const int* __restrict__ group, const double* __restrict__ exb,
                                const double* __restrict__ kw, int use_w, double* __restrict__ numer,
                                double* __restrict__ numer2) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int key = group[c.row(e)];
        if (e > 0 && group[c.row(e - 1)] == key) continue;
        double n1 = 0.0, n2 = 0.0;
        long long f = e;
        do {
            const int k = c.row(f);
            const double x = c.x(f);
            const double w = use_w ? kw[k] : 1.0;
            if (w != 0.0) {
                n1 += w * (exb[k] * x);
                if (!IND) n2 += w * (exb[k] * x * x);
            }
            ++f;
        } while (f < c.n && group[c.row(f)] == key);
        numer[key] = n1;
        if (!IND) numer2[key] = n2;
    }
}

// cumulative gradient for Breslow cox (ModelSpecifics.hpp:904-962).
//
// The reference walks every risk-set group i from the column's first group
// to N, with A_i / B_i the stratum-segmented running sums of the column's
// numerators, adding n_i*A_i/D_i (and the Hessian terms).  Between two
// consecutive column groups A and B are constant, so the walk over a gap
// [g_a, e_a) collapses to A*(P1(e_a-1) - P1(g_a-1)) and A^2*(P2(..)-P2(..)),
// where P1 / P2 are stratum-segmented prefix sums of n/D and n/D^2 kept
// (in double-double) by the denominator scan.  One block walks the column's
// group list in tiles, carrying the segmented running sums across tiles.
struct SegAB {
    int f;          // a segment (stratum) starts in the span
    double a, b;
};
__device__ __forceinline__ SegAB seg_combine(SegAB l, SegAB r) { return r.f ? r : SegAB{l.f, l.a + r.a, l.b + r.b}; }

template <bool IND>
__global__ void k_cox_gradient(const int* __restrict__ list, int L, const int* __restrict__ gstart,
                               const int* __restrict__ gend, const double* __restrict__ numer,
                               const double* __restrict__ numer2, const double* __restrict__ P1h,
                               const double* __restrict__ P1l, const double* __restrict__ P2h,
                               const double* __restrict__ P2l, const double* __restrict__ xjy, int j,
                               double* out) {
    // Each thread takes kItems consecutive groups of the list per tile; the
    // running sums A (and B) restart at every stratum change and carry
    // across tiles; threads' spans are combined by warp shuffles and then
    // across the warps' totals.
    constexpr int kItems = 4;
    constexpr int kTile = kThreads * kItems;
    __shared__ SegAB s_w[kThreads / 32];
    __shared__ SegAB s_carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = SegAB{0, 0.0, 0.0};
    double g = 0.0, h = 0.0;
    for (int base = 0; base < L; base += kTile) {
        const int a0 = base + threadIdx.x * kItems;
        int ga[kItems], key[kItems], fl[kItems];
        double A[kItems], B[kItems];
        #pragma unroll
        for (int q = 0; q < kItems; ++q) {
            const int a = a0 + q;
            ga[q] = 0; key[q] = -2; fl[q] = 0; A[q] = 0.0; B[q] = 0.0;
            if (a < L) {
                ga[q] = list[a];
                key[q] = gstart[ga[q]];
                fl[q] = (a == 0) || gstart[list[a - 1]] != key[q];
                A[q] = numer[ga[q]];
                B[q] = IND ? 0.0 : numer2[ga[q]];
            }
        }
        // inclusive within the thread's span
        SegAB run{0, 0.0, 0.0};
        #pragma unroll
        for (int q = 0; q < kItems; ++q) run = seg_combine(run, SegAB{fl[q], A[q], B[q]});
        // exclusive prefix of the span: warp shuffles, then the warps' totals
        int f = run.f;
        double va = run.a, vb = run.b;
        #pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int uf = __shfl_up_sync(0xffffffffu, f, off);
            const double ua = __shfl_up_sync(0xffffffffu, va, off);
            const double ub = __shfl_up_sync(0xffffffffu, vb, off);
            if (lane >= off) {
                if (!f) { va = ua + va; vb = ub + vb; }
                f |= uf;
            }
        }
        int ef = __shfl_up_sync(0xffffffffu, f, 1);
        double ea = __shfl_up_sync(0xffffffffu, va, 1), eb = __shfl_up_sync(0xffffffffu, vb, 1);
        if (lane == 0) { ef = 0; ea = 0.0; eb = 0.0; }
        if (lane == 31) s_w[w] = SegAB{f, va, vb};
        __syncthreads();
        SegAB pre = s_carry;
        for (int q = 0; q < w; ++q) pre = seg_combine(pre, s_w[q]);
        SegAB cur = seg_combine(pre, SegAB{ef, ea, eb});
        #pragma unroll
        for (int q = 0; q < kItems; ++q) {
            const int a = a0 + q;
            if (a >= L) break;
            cur = seg_combine(cur, SegAB{fl[q], A[q], B[q]});
            // interval end: next column group in the same stratum, else the stratum end
            int e_a;
            if (a + 1 < L && gstart[list[a + 1]] == key[q]) e_a = list[a + 1];
            else e_a = gend[ga[q]];
            const DD p1e{P1h[e_a - 1], P1l[e_a - 1]};
            const DD p2e{P2h[e_a - 1], P2l[e_a - 1]};
            const DD p1s = (ga[q] == key[q]) ? DD{0.0, 0.0} : DD{P1h[ga[q] - 1], P1l[ga[q] - 1]};
            const DD p2s = (ga[q] == key[q]) ? DD{0.0, 0.0} : DD{P2h[ga[q] - 1], P2l[ga[q] - 1]};
            const DD d1 = dd_sub(p1e, p1s);
            const DD d2 = dd_sub(p2e, p2s);
            const double s1 = d1.hi + d1.lo;
            const double s2 = d2.hi + d2.lo;
            g += cur.a * s1;
            h += IND ? (cur.a * s1 - cur.a * cur.a * s2) : (cur.b * s1 - cur.a * cur.a * s2);
        }
        __syncthreads();
        if (threadIdx.x == 0) {                     // the carry into the next tile
            SegAB t = s_carry;
            for (int q = 0; q < kThreads / 32; ++q) t = seg_combine(t, s_w[q]);
            s_carry = SegAB{0, t.a, t.b};
        }
        __syncthreads();
    }
    block_sum2(g, h);
    if (threadIdx.x == 0) {
        out[0] = g - xjy[j];
        out[1] = h;
    }
}

// a column whose group list is empty: gradient -XjY, Hessian 0 (ModelSpecifics.hpp:906)
__global__ void k_copy_neg_xjy(const double* __restrict__ xjy, int j, double* out) {
    out[0] = 0.0 - xjy[j];
    out[1] = 0.0;
}

// ---- KKT conditions (CyclicCoordinateDescent.cpp:817-837) ---------------------

// |gradient| of every listed column at the current state, one warp per
// column: the gradient halves of k_gh_independent / k_gh_grouped, so one
// launch scores the whole inactive set of the KKT swindle.  Empty columns
// score 0 (ModelSpecifics.hpp:720-723).
template <int MODEL>
__global__ void k_kkt_independent(int n_cols, const int* __restrict__ cols, int K, const int* fmt,
                                  const long long* col_ptr, const long long* val_ptr, const int* idx,
                                  const double* val, const double* __restrict__ exb,
                                  const double* __restrict__ denom, const double* __restrict__ nw, int use_w,
                                  const double* __restrict__ xjy, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n_cols; c += nwarps) {
        const int j = cols[c];
        const ColView v = fisher_view(j, K, fmt, col_ptr, val_ptr, idx, val);
        double g = 0.0;
        for (long long e = lane; e < v.n; e += 32) {
            const int k = v.row(e);
            const double n1 = exb[k] * v.x(e);
            const double w = use_w ? nw[k] : 1.0;
            g += w * (MODEL == CYC_LR ? n1 / denom[k] : n1);
        }
        for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) out[c] = v.n == 0 ? 0.0 : fabs(g - xjy[j]);
    }
}

// grouped rows: the first entry of each run of one stratum walks the run
__global__ void k_kkt_grouped(int n_cols, const int* __restrict__ cols, int K, const int* fmt,
                              const long long* col_ptr, const long long* val_ptr, const int* idx,
                              const double* val, const int* __restrict__ group, const double* __restrict__ exb,
                              const double* __restrict__ denom, const double* __restrict__ nw,
                              const double* __restrict__ xjy, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n_cols; c += nwarps) {
        const int j = cols[c];
        const ColView v = fisher_view(j, K, fmt, col_ptr, val_ptr, idx, val);
        double g = 0.0;
        for (long long e = lane; e < v.n; e += 32) {
            const int key = group[v.row(e)];
            if (e > 0 && group[v.row(e - 1)] == key) continue;
            double n1 = 0.0;
            long long f = e;
            do {
                n1 += exb[v.row(f)] * v.x(f);
                ++f;
            } while (f < v.n && group[v.row(f)] == key);
            g += nw[key] * (n1 / denom[key]);
        }
        for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) out[c] = v.n == 0 ? 0.0 : fabs(g - xjy[j]);
    }
}

// |gh[2i]| -> out[i]
__global__ void k_abs_gradients(int n, const double* __restrict__ gh, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = fabs(gh[2 * i]);
}

// ---- updateXBeta (ModelSpecifics.hpp:1524-1586) -----------------------------

// independent rows: each row is its own denominator
__global__ void k_update_independent(ColView c, const double* delta_ptr, double delta_val,
                                     double* __restrict__ xb, double* __restrict__ exb,
                                     double* __restrict__ denom) {
    const double delta = delta_ptr ? *delta_ptr : delta_val;
    if (delta == 0.0) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = c.row(e);
        const double v = add_mul_rn(xb[k], delta, c.x(e));
        xb[k] = v;
        const double old = exb[k];
        const double nw_ = exp(v);
        exb[k] = nw_;
        denom[k] += nw_ - old;
    }
}

// grouped / cumulative rows: the first entry of each run updates the run and
// adds its denominator change (weighted for cox when use_w)
__global__ void k_update_grouped(ColView c, const double* delta_ptr, double delta_val,
                                 const int* __restrict__ group, const double* __restrict__ kw,
                                 int weighted, double* __restrict__ xb, double* __restrict__ exb,
                                 double* __restrict__ denom) {
    const double delta = delta_ptr ? *delta_ptr : delta_val;
    if (delta == 0.0) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int key = group[c.row(e)];
        if (e > 0 && group[c.row(e - 1)] == key) continue;
        double d = denom[key];
        long long f = e;
        do {
            const int k = c.row(f);
            const double v = add_mul_rn(xb[k], delta, c.x(f));
            xb[k] = v;
            const double w = weighted ? kw[k] : 1.0;
            const double old = w * exb[k];
            const double ne = exp(v);
            exb[k] = ne;
            if (w != 0.0) d += w * ne - old;
            ++f;
        } while (f < c.n && group[c.row(f)] == key);
        denom[key] = d;
    }
}

// ---- cox denominator scan (computeAccumlatedDenominator, ModelSpecifics.hpp:1670-1694)
//
// D_i  = stratum-segmented inclusive prefix of denom
// P1_i = stratum-segmented inclusive prefix of n_i / D_i      (double-double)
// P2_i = stratum-segmented inclusive prefix of n_i / D_i^2    (double-double)
// computed over [lo, N) in tiles of kScanTile groups: a pass of tile
// aggregates for D, then a rewrite pass for D (which also forms the P terms
// and their tile aggregates) and one for P.  A rewrite CTA folds the
// aggregates of the tiles before its own into its carry itself (a few
// thousand L2-resident values), so no carry-scan launch sits between the
// passes.

constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;

__device__ __forceinline__ SegD seg_combine(SegD l, SegD r) { return r.f ? r : SegD{l.f, l.v + r.v}; }
__device__ __forceinline__ SegP seg_combine(SegP l, SegP r) {
    return r.f ? r : SegP{l.f, dd_add(l.a, r.a), dd_add(l.b, r.b)};
}

// The tile kernels: thread t of a tile holds kScanItems consecutive groups
// (tiles start at multiples of kScanItems, so those loads are aligned vectors; groups
// below `lo` or at or above `hi` are the identity), sums them in order, and
// the threads' sums are scanned by warp shuffles and then across the warps'
// totals -- no block-wide barrier rounds.  Segment starts (a group whose
// stratum starts there, gstart[i] == i) reset the sums.

// warp-inclusive segmented scan of (f, v), lane order
__device__ __forceinline__ void warp_seg_scan(int& f, double& v) {
    const int lane = threadIdx.x & 31;
    #pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int uf = __shfl_up_sync(0xffffffffu, f, off);
        const double uv = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) {
            if (!f) v = uv + v;
            f |= uf;
        }
    }
}
__device__ __forceinline__ void warp_seg_scan(int& f, DD& a, DD& b) {
    const int lane = threadIdx.x & 31;
    #pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int uf = __shfl_up_sync(0xffffffffu, f, off);
        const DD ua{__shfl_up_sync(0xffffffffu, a.hi, off), __shfl_up_sync(0xffffffffu, a.lo, off)};
        const DD ub{__shfl_up_sync(0xffffffffu, b.hi, off), __shfl_up_sync(0xffffffffu, b.lo, off)};
        if (lane >= off) {
            if (!f) { a = dd_add(ua, a); b = dd_add(ub, b); }
            f |= uf;
        }
    }
}

// exclusive prefix of this thread's aggregate within the block (identity
// for thread 0), and the block's total; `s_w` holds the warps' totals
__device__ __forceinline__ SegD block_seg_excl(SegD mine, SegD* s_w, SegD* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int f = mine.f;
    double v = mine.v;
    warp_seg_scan(f, v);
    int ef = __shfl_up_sync(0xffffffffu, f, 1);
    double ev = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane == 0) { ef = 0; ev = 0.0; }
    if (lane == 31) s_w[w] = SegD{f, v};
    __syncthreads();
    SegD pre{0, 0.0};
    for (int q = 0; q < w; ++q) pre = seg_combine(pre, s_w[q]);
    if (total) {
        SegD t{0, 0.0};
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = seg_combine(t, s_w[q]);
        *total = t;
    }
    __syncthreads();
    return seg_combine(pre, SegD{ef, ev});
}
__device__ __forceinline__ SegP block_seg_excl(SegP mine, SegP* s_w, SegP* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int f = mine.f;
    DD a = mine.a, b = mine.b;
    warp_seg_scan(f, a, b);
    int ef = __shfl_up_sync(0xffffffffu, f, 1);
    DD ea{__shfl_up_sync(0xffffffffu, a.hi, 1), __shfl_up_sync(0xffffffffu, a.lo, 1)};
    DD eb{__shfl_up_sync(0xffffffffu, b.hi, 1), __shfl_up_sync(0xffffffffu, b.lo, 1)};
    if (lane == 0) { ef = 0; ea = DD{0.0, 0.0}; eb = DD{0.0, 0.0}; }
    if (lane == 31) s_w[w] = SegP{f, a, b};
    __syncthreads();
    SegP pre{0, {0.0, 0.0}, {0.0, 0.0}};
    for (int q = 0; q < w; ++q) pre = seg_combine(pre, s_w[q]);
    if (total) {
        SegP t{0, {0.0, 0.0}, {0.0, 0.0}};
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = seg_combine(t, s_w[q]);
        *total = t;
    }
    __syncthreads();
    return seg_combine(pre, SegP{ef, ea, eb});
}

// the thread's kScanItems groups from i0 (a multiple of kScanItems): segment flags and values
// of `a` (and `b`), groups outside [lo, hi) as identity (flag 0, value 0)
__device__ __forceinline__ void load_items(int i0, int lo, int hi, const int* __restrict__ gstart,
                                      const double* __restrict__ a, const double* __restrict__ b, int (&f)[kScanItems],
                                      double (&va)[kScanItems], double (&vb)[kScanItems]) {
    if (i0 >= lo && i0 + kScanItems <= hi) {
        const int4* g4 = reinterpret_cast<const int4*>(gstart + i0);
        const double2* a2 = reinterpret_cast<const double2*>(a + i0);
        #pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const int4 g = __ldg(g4 + q);
            f[4 * q] = g.x == i0 + 4 * q;
            f[4 * q + 1] = g.y == i0 + 4 * q + 1;
            f[4 * q + 2] = g.z == i0 + 4 * q + 2;
            f[4 * q + 3] = g.w == i0 + 4 * q + 3;
        }
        #pragma unroll
        for (int q = 0; q < kScanItems / 2; ++q) {
            const double2 x = __ldg(a2 + q);
            va[2 * q] = x.x;
            va[2 * q + 1] = x.y;
        }
        if (b) {
            const double2* b2 = reinterpret_cast<const double2*>(b + i0);
            #pragma unroll
            for (int q = 0; q < kScanItems / 2; ++q) {
                const double2 x = __ldg(b2 + q);
                vb[2 * q] = x.x;
                vb[2 * q + 1] = x.y;
            }
        }
    } else {
        #pragma unroll
        for (int q = 0; q < kScanItems; ++q) {
            const int i = i0 + q;
            const bool in = i >= lo && i < hi;
            f[q] = in && gstart[i] == i;
            va[q] = in ? a[i] : 0.0;
            vb[q] = (in && b) ? b[i] : 0.0;
        }
    }
}

// first group of the tiling: lo rounded down to a multiple of 8
__host__ __device__ __forceinline__ int scan_base(int lo) { return lo & ~(kScanItems - 1); }

// `gate`: when non-null and *gate == 0 (a zero coordinate step), nothing changed
__global__ void __launch_bounds__(kThreads, 4) k_scanD_tiles(const double* gate, int lo, int hi, const int* __restrict__ gstart,
                              const double* __restrict__ denom, SegD* __restrict__ agg) {
    if (gate && *gate == 0.0) return;
    __shared__ SegD s_w[kThreads / 32];
    const int i0 = scan_base(lo) + blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int f[kScanItems];
    double v[kScanItems], unused[kScanItems];
    load_items(i0, lo, hi, gstart, denom, nullptr, f, v, unused);
    SegD a{0, 0.0};
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q) a = seg_combine(a, SegD{f[q], v[q]});
    SegD tot;
    block_seg_excl(a, s_w, &tot);
    if (threadIdx.x == 0) agg[blockIdx.x] = tot;
}

// the carry into tile `b`: `init` combined with the aggregates of tiles
// [0, b) in order (each thread folds a contiguous run, then the runs are
// combined across the block); every thread gets it
template <class T>
__device__ __forceinline__ T tile_carry(const T* __restrict__ agg, int b, T init, T* s_w) {
    const int per = (b + (int)blockDim.x - 1) / (int)blockDim.x;
    const int s0 = threadIdx.x * per, s1 = min(b, s0 + per);
    T acc{};                                       // the identity: no segment start, zero sums
    // several loads in flight at a time (eight D aggregates, four P ones; a
    // run is a few tiles: 2M groups are ~1,000 tiles of 2,048)
    constexpr int U = sizeof(T) > 16 ? 4 : 8;
    for (int i = s0; i < s1; i += U) {
        T v[U];
        #pragma unroll
        for (int k = 0; k < U; ++k) v[k] = (i + k < s1) ? agg[i + k] : T{};
        #pragma unroll
        for (int k = 0; k < U; ++k) acc = seg_combine(acc, v[k]);
    }
    T tot;
    block_seg_excl(acc, s_w, &tot);
    return seg_combine(init, tot);
}

// the carry's starting value: the prefix at lo - 1 when lo continues its stratum
__device__ __forceinline__ SegD carry_init_D(int lo, const int* __restrict__ gstart, const double* __restrict__ D) {
    return SegD{0, (lo > 0 && gstart[lo] != lo) ? D[lo - 1] : 0.0};
}
__device__ __forceinline__ SegP carry_init_P(int lo, const int* __restrict__ gstart, const double* __restrict__ P1h,
                                             const double* __restrict__ P1l, const double* __restrict__ P2h,
                                             const double* __restrict__ P2l) {
    SegP init{0, {0.0, 0.0}, {0.0, 0.0}};
    if (lo > 0 && gstart[lo] != lo) {
        init.a = DD{P1h[lo - 1], P1l[lo - 1]};
        init.b = DD{P2h[lo - 1], P2l[lo - 1]};
    }
    return init;
}

// writes D and the P terms r1 = n/D, r2 = n/D^2 (R1, R2) for the P pass
__global__ void __launch_bounds__(kThreads, 3) k_scanD_write(const double* gate, int lo, int hi, const int* __restrict__ gstart,
                              const double* __restrict__ denom, const double* __restrict__ nw,
                              const SegD* __restrict__ aggD, double* __restrict__ D, double* __restrict__ R1,
                              double* __restrict__ R2, SegP* __restrict__ aggP) {
    if (gate && *gate == 0.0) return;
    __shared__ SegD s_w[kThreads / 32];
    __shared__ SegP s_wp[kThreads / 32];
    const SegD carry = tile_carry(aggD, (int)blockIdx.x, carry_init_D(lo, gstart, D), s_w);
    const int i0 = scan_base(lo) + blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int f[kScanItems];
    double v[kScanItems], n[kScanItems];
    load_items(i0, lo, hi, gstart, denom, nw, f, v, n);
    SegD a{0, 0.0};
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q) a = seg_combine(a, SegD{f[q], v[q]});
    const SegD ex = block_seg_excl(a, s_w, nullptr);
    SegD run = seg_combine(carry, ex);
    SegP p{0, {0.0, 0.0}, {0.0, 0.0}};
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const int i = i0 + q;
        if (i >= lo && i < hi) {
            run = seg_combine(run, SegD{f[q], v[q]});
            D[i] = run.v;
            const double inv = 1.0 / run.v;            // one division for both terms
            const double r1 = n[q] * inv;
            const double r2 = r1 * inv;
            R1[i] = r1;
            R2[i] = r2;
            p = seg_combine(p, SegP{f[q], {r1, 0.0}, {r2, 0.0}});
        }
    }
    SegP totp;
    block_seg_excl(p, s_wp, &totp);
    if (threadIdx.x == 0) aggP[blockIdx.x] = totp;
}

__global__ void __launch_bounds__(kThreads, 3) k_scanP_write(const double* gate, int lo, int hi, const int* __restrict__ gstart,
                              const double* __restrict__ R1, const double* __restrict__ R2,
                              const SegP* __restrict__ aggP, double* __restrict__ P1h, double* __restrict__ P1l,
                              double* __restrict__ P2h, double* __restrict__ P2l) {
    if (gate && *gate == 0.0) return;
    __shared__ SegP s_wp[kThreads / 32];
    const SegP carry = tile_carry(aggP, (int)blockIdx.x, carry_init_P(lo, gstart, P1h, P1l, P2h, P2l), s_wp);
    const int i0 = scan_base(lo) + blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int f[kScanItems];
    double r1[kScanItems], r2[kScanItems];
    load_items(i0, lo, hi, gstart, R1, R2, f, r1, r2);          // identity (0) outside [lo, hi)
    SegP p{0, {0.0, 0.0}, {0.0, 0.0}};
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q) p = seg_combine(p, SegP{f[q], {r1[q], 0.0}, {r2[q], 0.0}});
    const SegP ex = block_seg_excl(p, s_wp, nullptr);
    SegP run = seg_combine(carry, ex);
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const int i = i0 + q;
        if (i >= lo && i < hi) {
            run = seg_combine(run, SegP{f[q], {r1[q], 0.0}, {r2[q], 0.0}});
            P1h[i] = run.a.hi; P1l[i] = run.a.lo;
            P2h[i] = run.b.hi; P2l[i] = run.b.lo;
        }
    }
}

// ---- log likelihood (ModelSpecifics.hpp:605-650) -----------------------------

__device__ __forceinline__ double ll_numer(int model, double y, double xb) {
    const int yi = (int)y;                      // logLikeNumeratorContrib(int, RealType)
    if (model == CYC_COX) return yi != 1 ? 0.0 : xb;
    return yi * xb;
}
__device__ __forceinline__ double ll_denom(int model, double n, double d) {
    return model == CYC_PR ? n * d : n * log(d);
}

__global__ void k_loglik(int model, int K, int N, const double* __restrict__ y, const double* __restrict__ xb,
                         const double* __restrict__ kw, int use_cv, const double* __restrict__ nw,
                         const double* __restrict__ den, const double* __restrict__ fixed,
                         double2* partial, unsigned* ticket, double* out) {
    double a = 0.0, b = 0.0;
    const int M = K > N ? K : N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
        if (i < K) {
            const double v = ll_numer(model, y[i], xb[i]);
            a += use_cv ? v * kw[i] : v;
        }
        if (i < N) b += ll_denom(model, nw[i], den[i]);
    }
    grid_sum2_finalize(a, b, partial, ticket, [&](double A, double B) {
        double ll = A - B;
        if (has_fixed_ll(model)) ll += *fixed;
        *out = ll;
    });
}

// getGradientObjective (ModelSpecifics.hpp:103-120)
__global__ void k_grad_objective(int K, const double* __restrict__ y, const double* __restrict__ xb,
                                 const double* __restrict__ kw, int use_cv, double2* partial,
                                 unsigned* ticket, double* out) {
    double a = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        a += use_cv ? xb[k] * y[k] * kw[k] : xb[k] * y[k];
    grid_sum2_finalize(a, 0.0, partial, ticket, [&](double A, double) { *out = A; });
}

// getPredictiveLogLikelihood (ModelSpecifics.hpp:652-690 and logPredLikeContrib,
// ModelSpecifics.h:1002-1009, 1137-1146, 1583-1590)
__global__ void k_pred_loglik(int model, int K, const double* __restrict__ y, const double* __restrict__ xb,
                              const double* __restrict__ w, const int* __restrict__ group,
                              const double* __restrict__ den, double2* partial, unsigned* ticket,
                              double* out) {
    double a = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        const double yk = y[k], wk = w[k], x = xb[k];
        double v;
        if (model == CYC_PR) {
            v = (yk * x - exp(x)) * wk;
        } else {
            const int g = group ? group[k] : k;
            if (model == CYC_COX) v = wk == 0.0 ? 0.0 : yk * wk * (x - log(den[g]));
            else v = yk * wk * (x - log(den[g]));
        }
        a += v;
    }
    grid_sum2_finalize(a, 0.0, partial, ticket, [&](double A, double) { *out = A; });
}

// getPredictiveEstimates (ModelSpecifics.hpp:692-707, predictEstimate)
__global__ void k_pred_estimates(int model, int K, const double* __restrict__ xb, const double* __restrict__ w,
                                 double* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        if (w && w[k] == 0.0) continue;
        const double x = xb[k];
        if (model == CYC_LR) {
            const double t = exp(x);
            out[k] = t / (t + 1.0);
        } else if (model == CYC_PR) {
            out[k] = exp(x);
        } else {
            out[k] = x;
        }
    }
}

}  // namespace cyc
