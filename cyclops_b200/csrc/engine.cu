// engine.cu -- the per-coordinate engine behind the AbstractModelSpecifics
// surface (src/cyclops/engine/AbstractModelSpecifics.h:36-122), FP64.
//
// Per-fit HBM state (one engine):
//   xb, xb_save, exb, kw          K doubles   (hXBeta, hXBetaSave, offsExpXBeta, hKWeight)
//   denom, nw, numer, numer2      N+1 doubles (denomPid, hNWeight, numerPid, numerPid2)
//   xjy                           J doubles   (hXjY)
// cox adds the risk-set grouping of the current weights and its scans:
//   group[K], grow_ptr[N+1], gstart[N], gend[N], per-column group lists,
//   D (accDenomPid), P1/P2 (double-double prefix sums of n/D and n/D^2).
#include "engine.cuh"
#include "engine_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <memory>

namespace cyc {

Engine::Engine(Dataset* d) : ds(d), device(d->device) {
    CYC_CHECK_CUDA(cudaSetDevice(ds->device));
    CYC_CHECK_CUDA(cudaStreamCreateWithFlags(&own.s, cudaStreamNonBlocking));
    stream = own.s;
    StreamScope scope(stream);
    model = ds->model;
    const int K = ds->K;
    // initialize (ModelSpecifics.hpp:1899-1952)
    xb.alloc(K);
    exb.alloc(K);
    kw.alloc(K);
    xjy.alloc(ds->J);
    partial.alloc(148 * 8);
    ticket.alloc(1);
    result.alloc(8);
    ll_fixed.alloc(1);
    CYC_CHECK_CUDA(cudaMemsetAsync(ticket.get(), 0, sizeof(unsigned), stream));
    CYC_CHECK_CUDA(cudaMemsetAsync(xb.get(), 0, K * sizeof(double), stream));
    CYC_CHECK_CUDA(cudaMemsetAsync(ll_fixed.get(), 0, sizeof(double), stream));
    if (model_cumulative(model)) {
        regroup(nullptr);                                // setPidForAccumulation(nullptr)
    } else {
        N = model_grouped(model) ? ds->S : K;
        alloc_denominators();
    }
    set_weights(nullptr, false);
    sync();
}

Engine::~Engine() {
    // the buffers are freed on the stream after its work; `own` then releases it
    cudaSetDevice(device);
}

void Engine::sync() { CYC_CHECK_CUDA(cudaStreamSynchronize(stream)); }

void Engine::alloc_denominators() {
    denom.alloc(N + 1);
    nw.alloc(N + 1);
    numer.alloc(N + 1);
    numer2.alloc(N + 1);
    CYC_CHECK_CUDA(cudaMemsetAsync(denom.get(), 0, (N + 1) * sizeof(double), stream));
    CYC_CHECK_CUDA(cudaMemsetAsync(numer.get(), 0, (N + 1) * sizeof(double), stream));
    CYC_CHECK_CUDA(cudaMemsetAsync(numer2.get(), 0, (N + 1) * sizeof(double), stream));
}

const int* Engine::groups() const {
    if (model_grouped(model)) return ds->d_strat.get();
    if (model_cumulative(model)) return group.get();
    return nullptr;
}

const int* Engine::group_rows() const {
    if (model_grouped(model)) return ds->d_strat_ptr.get();
    return grow_ptr.get();
}

// setPidForAccumulation (ModelSpecifics.hpp:1809-1868) and setupSparseIndices
// (:1870-1892) for Breslow cox.  Rows with zero weight are given the group of
// the preceding weighted row instead of the reference's sentinel N; their
// contributions are exactly zero in every sum, and group ids stay
// non-decreasing in row order so every group is a contiguous row range.
void Engine::regroup(const double* w) {
    const int K = ds->K;
    const std::vector<int>& strat = ds->strat;
    const std::vector<double>& t = ds->time;
    const std::vector<double>& y = ds->y;
    std::vector<int> g(K, -1);
    std::vector<int> resets;  // stratum starts (group ids), first is 0
    int index = 0;
    while (w != nullptr && index < K && w[index] == 0.0) index++;
    CYC_REQUIRE(index < K, CYC_ERR_ARGUMENT, "all weights are zero");
    int last_pid = strat[index];
    double last_time = t[index];
    double last_event = y[index];
    int pid = 0;
    g[index] = 0;
    resets.push_back(0);
    for (int k = index + 1; k < K; ++k) {
        if (w == nullptr || w[k] != 0.0) {
            const int next = strat[k];
            if (next != last_pid) {
                pid++;
                resets.push_back(pid);
                last_pid = next;
            } else if (last_event == 1.0 && last_time == t[k] && last_event == y[k]) {
                // tie: same denominator
            } else {
                pid++;
            }
            last_time = t[k];
            last_event = y[k];
            g[k] = pid;
        }
    }
    N = pid + 1;
    int prev = 0;
    for (int k = 0; k < K; ++k) {
        if (g[k] < 0) g[k] = prev;
        prev = g[k];
    }
    std::vector<int> gs(N), ge(N), rp(N + 1, 0);
    resets.push_back(N);
    for (size_t r = 0; r + 1 < resets.size(); ++r)
        for (int i = resets[r]; i < resets[r + 1]; ++i) {
            gs[i] = resets[r];
            ge[i] = resets[r + 1];
        }
    for (int k = 0; k < K; ++k) rp[g[k] + 1]++;
    for (int i = 0; i < N; ++i) rp[i + 1] += rp[i];
    // per-column group lists
    const int J = ds->J;
    std::vector<long long> lp(J + 1, 0);
    std::vector<int> lst;
    lst.reserve(ds->nnz_idx);
    for (int j = 0; j < J; ++j) {
        const int f = ds->fmt[j];
        if (f == CYC_DENSE || f == CYC_INTERCEPT) {
            for (int i = 0; i < N; ++i) lst.push_back(i);
        } else {
            int lastg = -1;
            for (long long e = ds->col_ptr[j]; e < ds->col_ptr[j + 1]; ++e) {
                const int gg = g[ds->h_idx[e]];
                if (gg != lastg) { lst.push_back(gg); lastg = gg; }
            }
        }
        lp[j + 1] = (long long)lst.size();
    }
    h_glist_ptr = lp;
    h_first_group.assign(J, N);
    for (int j = 0; j < J; ++j)
        if (lp[j + 1] > lp[j]) h_first_group[j] = lst[lp[j]];
    alloc_denominators();
    group.alloc(K);
    grow_ptr.alloc(N + 1);
    gstart.alloc(N);
    gend.alloc(N);
    glist_ptr.alloc(J + 1);
    glist.alloc(std::max<size_t>(lst.size(), 1));
    D.alloc(N + 1);
    P1h.alloc(N + 1); P1l.alloc(N + 1); P2h.alloc(N + 1); P2l.alloc(N + 1);
    R1.alloc(N + 1); R2.alloc(N + 1);
    const int ntiles = (N + kScanTile - 1) / kScanTile;
    aggD.alloc(ntiles + 1);
    aggP.alloc(ntiles + 1);
    CYC_CHECK_CUDA(cudaMemcpyAsync(group.get(), g.data(), K * sizeof(int), cudaMemcpyHostToDevice, stream));
    CYC_CHECK_CUDA(cudaMemcpyAsync(grow_ptr.get(), rp.data(), (N + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
    CYC_CHECK_CUDA(cudaMemcpyAsync(gstart.get(), gs.data(), N * sizeof(int), cudaMemcpyHostToDevice, stream));
    CYC_CHECK_CUDA(cudaMemcpyAsync(gend.get(), ge.data(), N * sizeof(int), cudaMemcpyHostToDevice, stream));
    CYC_CHECK_CUDA(cudaMemcpyAsync(glist_ptr.get(), lp.data(), (J + 1) * sizeof(long long), cudaMemcpyHostToDevice, stream));
    if (!lst.empty())
        CYC_CHECK_CUDA(cudaMemcpyAsync(glist.get(), lst.data(), lst.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    // host copies must outlive the async copies
    sync();
}

// setWeights (ModelSpecifics.hpp:427-484).  As in the reference, the
// statistics (exb, denominators) stay usable: lr / pr / clr / cpr
// denominators do not depend on the weights, and cox, whose risk-set groups
// are rebuilt here, gets its weighted denominators recomputed from the
// unchanged xbeta when they were current before.  (The reference's CCD calls
// setWeights again at the start of findMode while it holds its statistics
// current, e.g. inside kktSwindle.)
void Engine::set_weights(const double* w, bool use_cv) {
    const int K = ds->K;
    const bool had_stats = stats_known;
    use_w = use_cv && w != nullptr;
    const double* wp = use_w ? w : nullptr;
    if (model_cumulative(model)) regroup(wp);
    if (wp) {
        weights_buf.alloc(K);
        CYC_CHECK_CUDA(cudaMemcpyAsync(weights_buf.get(), wp, K * sizeof(double), cudaMemcpyHostToDevice, stream));
        launch(k_set_kw, grid_for(K, 1), kThreads, 0, stream, K, weights_buf.get(), kw.get());
        sync();  // the caller's host buffer may go away after return
    } else {
        launch(k_set_kw, grid_for(K, 1), kThreads, 0, stream, K, nullptr, kw.get());
    }
    CYC_CHECK_CUDA(cudaMemsetAsync(nw.get(), 0, (N + 1) * sizeof(double), stream));
    if (model_independent(model)) {
        launch(k_nw_independent, grid_for(K, 1), kThreads, 0, stream, K, kw.get(), nw.get());
    } else {
        launch(k_nw_grouped, grid_for(N, 1), kThreads, 0, stream, N, group_rows(), ds->d_y.get(), kw.get(), nw.get());
    }
    CYC_CHECK_LAUNCH();
    if (model_cumulative(model)) {
        if (had_stats) remaining_statistics(true);
        else stats_known = false;
    }
}

void Engine::fixed_terms_ll(bool use_cv) {
    if (!has_fixed_ll(model)) return;
    const int K = ds->K;
    const int blocks = grid_for(K, 4);
    launch(k_fixed_ll, blocks, kThreads, 0, stream, K, ds->d_y.get(), kw.get(), use_cv && use_w,
                                                partial.get(), ticket.get(), ll_fixed.get());
    CYC_CHECK_LAUNCH();
}

void Engine::fixed_terms_gh(bool use_cv) {
    const int J = ds->J;
    launch(k_xjy, std::min(J, 148 * 16), 128, 0, stream, J, ds->d_fmt.get(), ds->d_col_ptr.get(),
                                                     ds->d_val_ptr.get(), ds->d_idx.get(), ds->d_val.get(),
                                                     ds->K, ds->d_y.get(), kw.get(), use_cv && use_w, xjy.get());
    CYC_CHECK_LAUNCH();
}

void Engine::zero_xbeta() {
    CYC_CHECK_CUDA(cudaMemsetAsync(xb.get(), 0, ds->K * sizeof(double), stream));
    stats_known = false;
}

void Engine::axpy_xbeta(double beta, int j) {
    if (beta == 0.0) return;
    ColView c = ds->view(j);
    launch(k_axpy, grid_for(c.n, 4), kThreads, 0, stream, c, beta, xb.get());
    CYC_CHECK_LAUNCH();
    stats_known = false;
}

void Engine::compute_xbeta(const double* beta_host) {
    const int J = ds->J;
    bool any = false;
    for (int j = 0; j < J; ++j) any |= beta_host[j] != 0.0;
    if (!any) { zero_xbeta(); return; }
    ds->ensure_csr();
    beta_buf.alloc(J);
    CYC_CHECK_CUDA(cudaMemcpyAsync(beta_buf.get(), beta_host, J * sizeof(double), cudaMemcpyHostToDevice, stream));
    compute_xbeta_device(beta_buf.get());
    sync();
}

void Engine::compute_xbeta_device(const double* d_beta) {
    ds->ensure_csr();
    const int K = ds->K;
    launch(k_xbeta_rows, grid_for(K, 1), kThreads, 0, stream, K, ds->d_row_ptr.get(), ds->d_row_col.get(),
                                                          ds->d_row_val.get(), d_beta, xb.get());
    CYC_CHECK_LAUNCH();
    stats_known = false;
}

void Engine::cox_rescan(int lo) {
    if (lo >= N) return;
    cox_rescan_gated(nullptr, lo);
}

// computeRemainingStatistics (ModelSpecifics.hpp:1588-1633)
void Engine::remaining_statistics(bool use_weights) {
    const int K = ds->K;
    if (model_independent(model)) {
        launch(k_rs_independent, grid_for(K, 1), kThreads, 0, stream, K, model, xb.get(), exb.get(), denom.get());
    } else {
        launch(k_rs_grouped, grid_for(N, 1), kThreads, 0, stream, 
            N, group_rows(), xb.get(), kw.get(), model_cumulative(model) && use_weights && use_w,
            exb.get(), denom.get());
        if (model_cumulative(model)) cox_rescan(0);
    }
    CYC_CHECK_LAUNCH();
    stats_known = true;
}

void Engine::numerator_for_gradient(int j, bool use_weights) {
    if (!model_cumulative(model)) return;
    ColView c = ds->view(j);
    if (c.n == 0) return;
    const int blocks = grid_for(c.n, 4);
    if (c.indicator())
        launch(k_cox_numerator<true>, blocks, kThreads, 0, stream, c, group.get(), exb.get(), kw.get(),
                                                              use_weights && use_w, numer.get(), numer2.get());
    else
        launch(k_cox_numerator<false>, blocks, kThreads, 0, stream, c, group.get(), exb.get(), kw.get(),
                                                               use_weights && use_w, numer.get(), numer2.get());
    CYC_CHECK_LAUNCH();
}

// launches the gradient/Hessian of column j into out[0..1] (device)
void Engine::launch_gradient(int j, bool use_weights, double* out) {
    ColView c = ds->view(j);
    if (c.n == 0) {                                   // ModelSpecifics.hpp:720-723
        CYC_CHECK_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(double), stream));
        return;
    }
    const int blocks = grid_for(c.n, 4);
    const bool uw = use_weights && use_w;
    if (model_independent(model)) {
        if (model == CYC_LR) {
            if (c.indicator())
                launch(k_gh_independent<CYC_LR, true>, blocks, kThreads, 0, stream, c, exb.get(), denom.get(), nw.get(), uw, xjy.get(), j, partial.get(), ticket.get(), out);
            else
                launch(k_gh_independent<CYC_LR, false>, blocks, kThreads, 0, stream, c, exb.get(), denom.get(), nw.get(), uw, xjy.get(), j, partial.get(), ticket.get(), out);
        } else {
            if (c.indicator())
                launch(k_gh_independent<CYC_PR, true>, blocks, kThreads, 0, stream, c, exb.get(), denom.get(), nw.get(), uw, xjy.get(), j, partial.get(), ticket.get(), out);
            else
                launch(k_gh_independent<CYC_PR, false>, blocks, kThreads, 0, stream, c, exb.get(), denom.get(), nw.get(), uw, xjy.get(), j, partial.get(), ticket.get(), out);
        }
    } else if (model_grouped(model)) {
        if (c.indicator())
            launch(k_gh_grouped<true>, blocks, kThreads, 0, stream, c, groups(), exb.get(), denom.get(), nw.get(), xjy.get(), j, partial.get(), ticket.get(), out);
        else
            launch(k_gh_grouped<false>, blocks, kThreads, 0, stream, c, groups(), exb.get(), denom.get(), nw.get(), xjy.get(), j, partial.get(), ticket.get(), out);
    } else {
        const long long b = h_glist_ptr[j], e = h_glist_ptr[j + 1];
        const int L = (int)(e - b);
        if (L == 0) {
            launch(k_copy_neg_xjy, 1, 1, 0, stream, xjy.get(), j, out);
        } else if (c.indicator()) {
            launch(k_cox_gradient<true>, 1, kThreads, 0, stream, glist.get() + b, L, gstart.get(), gend.get(), numer.get(), numer2.get(), P1h.get(), P1l.get(), P2h.get(), P2l.get(), xjy.get(), j, out);
        } else {
            launch(k_cox_gradient<false>, 1, kThreads, 0, stream, glist.get() + b, L, gstart.get(), gend.get(), numer.get(), numer2.get(), P1h.get(), P1l.get(), P2h.get(), P2l.get(), xjy.get(), j, out);
        }
    }
    CYC_CHECK_LAUNCH();
}

void Engine::gradient_hessian(int j, bool use_weights, double* g, double* h) {
    CYC_REQUIRE(stats_known, CYC_ERR_STATE, "Error in state synchronization.");
    launch_gradient(j, use_weights, result.get());
    CYC_CHECK_CUDA(cudaMemcpyAsync(h_result, result.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    *g = h_result[0];
    *h = h_result[1];
}

// updateXBeta (ModelSpecifics.hpp:1466-1586); delta either a host value or a
// device pointer (the device-resident solver)
void Engine::launch_update(int j, bool use_weights, const double* d_delta, double delta) {
    ColView c = ds->view(j);
    if (c.n == 0) return;
    const int blocks = grid_for(c.n, 4);
    if (model_independent(model)) {
        launch(k_update_independent, blocks, kThreads, 0, stream, c, d_delta, delta, xb.get(), exb.get(), denom.get());
    } else {
        launch(k_update_grouped, blocks, kThreads, 0, stream, c, d_delta, delta, groups(), kw.get(),
                                                          model_cumulative(model) && use_weights && use_w,
                                                          xb.get(), exb.get(), denom.get());
        if (model_cumulative(model)) cox_rescan_gated(d_delta, first_group(j));
    }
    CYC_CHECK_LAUNCH();
}

int Engine::first_group(int j) const { return h_first_group[j]; }

// D / P1 / P2 over groups [lo, N); `gate` (device) skips the work when the
// coordinate step it points at is zero
void Engine::cox_rescan_gated(const double* gate, int lo) {
    if (lo >= N) return;
    const int hi = N;
    // tiles start at lo rounded down to a multiple of kScanItems (aligned loads)
    const int ntiles = (hi - scan_base(lo) + kScanTile - 1) / kScanTile;
    launch(k_scanD_tiles, ntiles, kThreads, 0, stream, gate, lo, hi, gstart.get(), denom.get(), aggD.get());
    launch(k_scanD_write, ntiles, kThreads, 0, stream, gate, lo, hi, gstart.get(), denom.get(), nw.get(),
                                                   (const SegD*)aggD.get(), D.get(), R1.get(), R2.get(), aggP.get());
    launch(k_scanP_write, ntiles, kThreads, 0, stream, gate, lo, hi, gstart.get(), (const double*)R1.get(),
                                                   (const double*)R2.get(), (const SegP*)aggP.get(),
                                                   P1h.get(), P1l.get(), P2h.get(), P2l.get());
    CYC_CHECK_LAUNCH();
}

void Engine::update_xbeta(double delta, int j, bool use_weights) {
    launch_update(j, use_weights, nullptr, delta);
    sync();
}

void Engine::launch_loglik(bool use_cv, double* out) {
    const int K = ds->K;
    const int M = std::max(K, N);
    const double* den = model_cumulative(model) ? D.get() : denom.get();
    launch(k_loglik, grid_for(M, 4), kThreads, 0, stream, model, K, N, ds->d_y.get(), xb.get(), kw.get(),
                                                      use_cv && use_w, nw.get(), den, ll_fixed.get(),
                                                      partial.get(), ticket.get(), out);
    CYC_CHECK_LAUNCH();
}

double Engine::log_likelihood(bool use_cv) {
    launch_loglik(use_cv, result.get());
    CYC_CHECK_CUDA(cudaMemcpyAsync(h_result, result.get(), sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    return h_result[0];
}

void Engine::launch_gradient_objective(bool use_cv, double* out) {
    const int K = ds->K;
    launch(k_grad_objective, grid_for(K, 4), kThreads, 0, stream, K, ds->d_y.get(), xb.get(), kw.get(),
                                                              use_cv && use_w, partial.get(), ticket.get(), out);
    CYC_CHECK_LAUNCH();
}

double Engine::gradient_objective(bool use_cv) {
    launch_gradient_objective(use_cv, result.get());
    CYC_CHECK_CUDA(cudaMemcpyAsync(h_result, result.get(), sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    return h_result[0];
}

// getPredictiveLogLikelihood (ModelSpecifics.hpp:652-690)
double Engine::predictive_log_likelihood(const double* w) {
    const int K = ds->K;
    std::vector<double> saved;
    if (model_cumulative(model)) {
        saved.resize(K);
        CYC_CHECK_CUDA(cudaMemcpyAsync(saved.data(), kw.get(), K * sizeof(double), cudaMemcpyDeviceToHost, stream));
        sync();
        set_weights(w, true);
        remaining_statistics(true);
    }
    weights_buf.alloc(K);
    CYC_CHECK_CUDA(cudaMemcpyAsync(weights_buf.get(), w, K * sizeof(double), cudaMemcpyHostToDevice, stream));
    const double* den = model_cumulative(model) ? D.get() : denom.get();
    launch(k_pred_loglik, grid_for(K, 4), kThreads, 0, stream, model, K, ds->d_y.get(), xb.get(), weights_buf.get(),
                                                           groups(), den, partial.get(), ticket.get(),
                                                           result.get());
    CYC_CHECK_LAUNCH();
    CYC_CHECK_CUDA(cudaMemcpyAsync(h_result, result.get(), sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    const double out = h_result[0];
    if (model_cumulative(model)) {
        set_weights(saved.data(), true);
        remaining_statistics(true);
        sync();
    }
    return out;
}

void Engine::predictive_estimates(double* y, const double* w) {
    const int K = ds->K;
    DevBuf<double> out;
    out.alloc(K);
    CYC_CHECK_CUDA(cudaMemcpyAsync(out.get(), y, K * sizeof(double), cudaMemcpyHostToDevice, stream));
    const double* dw = nullptr;
    if (w) {
        weights_buf.alloc(K);
        CYC_CHECK_CUDA(cudaMemcpyAsync(weights_buf.get(), w, K * sizeof(double), cudaMemcpyHostToDevice, stream));
        dw = weights_buf.get();
    }
    launch(k_pred_estimates, grid_for(K, 1), kThreads, 0, stream, model, K, xb.get(), dw, out.get());
    CYC_CHECK_LAUNCH();
    CYC_CHECK_CUDA(cudaMemcpyAsync(y, out.get(), K * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
}

// computeFisherInformation over every pair of `cols` (CyclicCoordinateDescent
// computeFisherInformation, src/cyclops/CyclicCoordinateDescent.cpp:1288-1300):
// out is the n x n symmetric matrix, row-major
void Engine::fisher_information(const int* cols, int n, double* out) {
    CYC_REQUIRE(model_independent(model) || model_grouped(model), CYC_ERR_UNSUPPORTED,
                "Fisher information is offered for lr, pr, clr and cpr");
    const int K = ds->K, S = ds->S, J = ds->J;
    for (int i = 0; i < n; ++i)
        CYC_REQUIRE(cols[i] >= 0 && cols[i] < J, CYC_ERR_ARGUMENT, "column index out of range");
    if (n == 0) return;
    remaining_statistics(false);
    const bool grouped = model_grouped(model);
    if (grouped)
        CYC_REQUIRE((double)n * S <= (double)(1u << 27), CYC_ERR_MEMORY,
                    "too many columns x strata for one Fisher information call");
    std::vector<int> pa, pb;
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) { pa.push_back(i); pb.push_back(j); }
    const int np = (int)pa.size();
    DevBuf<int> d_cols, d_pa, d_pb;
    DevBuf<double> d_v, d_t, d_out;
    d_cols.alloc(n); d_pa.alloc(np); d_pb.alloc(np); d_v.alloc(K); d_out.alloc(np);
    CYC_CHECK_CUDA(cudaMemcpyAsync(d_cols.get(), cols, n * sizeof(int), cudaMemcpyHostToDevice, stream));
    CYC_CHECK_CUDA(cudaMemcpyAsync(d_pa.get(), pa.data(), np * sizeof(int), cudaMemcpyHostToDevice, stream));
    CYC_CHECK_CUDA(cudaMemcpyAsync(d_pb.get(), pb.data(), np * sizeof(int), cudaMemcpyHostToDevice, stream));
    launch(k_fisher_row, grid_for(K, 4), kThreads, 0, stream, K, model, (const double*)exb.get(),
           (const double*)denom.get(), (const int*)ds->d_strat.get(), d_v.get());
    if (grouped) {
        d_t.alloc((size_t)n * S);
        CYC_CHECK_CUDA(cudaMemsetAsync(d_t.get(), 0, (size_t)n * S * sizeof(double), stream));
        launch(k_fisher_strata, std::min(n, 148 * 8), kThreads, 0, stream, n, (const int*)d_cols.get(), K, S,
               (const int*)ds->d_fmt.get(), (const long long*)ds->d_col_ptr.get(), (const long long*)ds->d_val_ptr.get(),
               (const int*)ds->d_idx.get(), (const double*)ds->d_val.get(), (const int*)ds->d_strat.get(),
               (const double*)exb.get(), d_t.get());
    }
    launch(k_fisher_pairs, std::min(np, 148 * 8), kThreads, 0, stream, np, (const int*)d_pa.get(),
           (const int*)d_pb.get(), (const int*)d_cols.get(), K, S, grouped ? 1 : 0, (const int*)ds->d_fmt.get(),
           (const long long*)ds->d_col_ptr.get(), (const long long*)ds->d_val_ptr.get(), (const int*)ds->d_idx.get(),
           (const double*)ds->d_val.get(), (const double*)d_v.get(), (const int*)ds->d_strat.get(),
           (const double*)denom.get(), (const double*)d_t.get(), d_out.get());
    std::vector<double> h(np);
    CYC_CHECK_CUDA(cudaMemcpyAsync(h.data(), d_out.get(), np * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
    for (int p = 0; p < np; ++p) out[(size_t)pa[p] * n + pb[p]] = out[(size_t)pb[p] * n + pa[p]] = h[p];
}

// computeKktConditions (CyclicCoordinateDescent.cpp:817-837): |gradient| of
// columns cols[0..n) (host ids; d_cols the same ids on the device) into
// d_out[0..n) at the current state.  lr / pr / clr / cpr score every column
// in one launch; cox walks its risk sets column by column.
void Engine::kkt_scores(const int* cols, const int* d_cols, int n, bool use_weights, double* d_out) {
    if (n == 0) return;
    const bool uw = use_weights && use_w;
    const int K = ds->K;
    const int blocks = std::min((n + kThreads / 32 - 1) / (kThreads / 32), 148 * 16);
    const int* fmt = ds->d_fmt.get();
    const long long* cp = ds->d_col_ptr.get();
    const long long* vp = ds->d_val_ptr.get();
    const int* ix = ds->d_idx.get();
    const double* vl = ds->d_val.get();
    if (model_independent(model)) {
        if (model == CYC_LR)
            launch(k_kkt_independent<CYC_LR>, blocks, kThreads, 0, stream, n, d_cols, K, fmt, cp, vp, ix, vl,
                   (const double*)exb.get(), (const double*)denom.get(), (const double*)nw.get(), uw ? 1 : 0,
                   (const double*)xjy.get(), d_out);
        else
            launch(k_kkt_independent<CYC_PR>, blocks, kThreads, 0, stream, n, d_cols, K, fmt, cp, vp, ix, vl,
                   (const double*)exb.get(), (const double*)denom.get(), (const double*)nw.get(), uw ? 1 : 0,
                   (const double*)xjy.get(), d_out);
    } else if (model_grouped(model)) {
        launch(k_kkt_grouped, blocks, kThreads, 0, stream, n, d_cols, K, fmt, cp, vp, ix, vl, groups(),
               (const double*)exb.get(), (const double*)denom.get(), (const double*)nw.get(),
               (const double*)xjy.get(), d_out);
    } else {
        DevBuf<double> gh;
        gh.alloc(2 * (size_t)n);
        for (int i = 0; i < n; ++i) {
            numerator_for_gradient(cols[i], use_weights);
            launch_gradient(cols[i], use_weights, gh.get() + 2 * (size_t)i);
        }
        launch(k_abs_gradients, grid_for(n, 1), kThreads, 0, stream, n, (const double*)gh.get(), d_out);
    }
    CYC_CHECK_LAUNCH();
}

void Engine::get_xbeta(double* out) {
    CYC_CHECK_CUDA(cudaMemcpyAsync(out, xb.get(), ds->K * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
}

void Engine::save_xbeta() {
    xb_save.alloc(ds->K);
    CYC_CHECK_CUDA(cudaMemcpyAsync(xb_save.get(), xb.get(), ds->K * sizeof(double), cudaMemcpyDeviceToDevice, stream));
}

void Engine::get_xbeta_save(double* out) {
    if (xb_save.n == 0) return;
    CYC_CHECK_CUDA(cudaMemcpyAsync(out, xb_save.get(), ds->K * sizeof(double), cudaMemcpyDeviceToHost, stream));
    sync();
}

}  // namespace cyc

using namespace cyc;

#define CYC_REQUIRE_C(cond)                                                    \
    do {                                                                       \
        if (!(cond)) { set_error("null argument"); return CYC_ERR_ARGUMENT; }  \
    } while (0)

#define ENGINE_CALL(e, body)                                                   \
    guarded([&] {                                                              \
        CYC_REQUIRE((e) != nullptr, CYC_ERR_ARGUMENT, "null engine");          \
        CYC_CHECK_CUDA(cudaSetDevice((e)->eng->ds->device));                   \
        StreamScope scope_((e)->eng->stream);                                  \
        body;                                                                  \
    })

extern "C" int cyc_engine_create(cyc_dataset* ds, cyc_engine** out) {
    return guarded([&] {
        CYC_REQUIRE(ds && out, CYC_ERR_ARGUMENT, "null argument");
        *out = nullptr;
        CYC_CHECK_CUDA(cudaSetDevice(ds->ds.device));
        auto* e = new cyc_engine();
        std::unique_ptr<cyc_engine> g(e);
        e->owner = ds;
        e->eng.reset(new Engine(&ds->ds));
        *out = g.release();
    });
}

extern "C" int cyc_engine_destroy(cyc_engine* e) {
    return guarded([&] { delete e; });
}

// clone() (ModelSpecifics.hpp:98-101) builds a fresh engine on the same data
extern "C" int cyc_engine_clone(const cyc_engine* e, cyc_engine** out) {
    CYC_REQUIRE_C(e && out);
    return cyc_engine_create(e->owner, out);
}

extern "C" int cyc_engine_set_weights(cyc_engine* e, const double* w, int use_cv) {
    return ENGINE_CALL(e, e->eng->set_weights(w, use_cv != 0); e->eng->sync());
}
extern "C" int cyc_engine_compute_fixed_terms_ll(cyc_engine* e, int use_cv) {
    return ENGINE_CALL(e, e->eng->fixed_terms_ll(use_cv != 0); e->eng->sync());
}
extern "C" int cyc_engine_compute_fixed_terms_gh(cyc_engine* e, int use_cv) {
    return ENGINE_CALL(e, e->eng->fixed_terms_gh(use_cv != 0); e->eng->sync());
}
extern "C" int cyc_engine_zero_xbeta(cyc_engine* e) {
    return ENGINE_CALL(e, e->eng->zero_xbeta(); e->eng->sync());
}
extern "C" int cyc_engine_axpy_xbeta(cyc_engine* e, double beta, int j) {
    return ENGINE_CALL(e, CYC_REQUIRE(j >= 0 && j < e->eng->ds->J, CYC_ERR_ARGUMENT, "column out of range");
                       e->eng->axpy_xbeta(beta, j); e->eng->sync());
}
extern "C" int cyc_engine_compute_xbeta(cyc_engine* e, const double* beta, int use_w) {
    (void)use_w;
    return ENGINE_CALL(e, CYC_REQUIRE(beta, CYC_ERR_ARGUMENT, "null beta"); e->eng->compute_xbeta(beta));
}
extern "C" int cyc_engine_compute_remaining_statistics(cyc_engine* e, int use_w) {
    return ENGINE_CALL(e, e->eng->remaining_statistics(use_w != 0); e->eng->sync());
}
extern "C" int cyc_engine_compute_numerator_for_gradient(cyc_engine* e, int j, int use_w) {
    return ENGINE_CALL(e, CYC_REQUIRE(j >= 0 && j < e->eng->ds->J, CYC_ERR_ARGUMENT, "column out of range");
                       e->eng->numerator_for_gradient(j, use_w != 0));
}
extern "C" int cyc_engine_compute_gradient_and_hessian(cyc_engine* e, int j, double* g, double* h, int use_w) {
    return ENGINE_CALL(e, CYC_REQUIRE(j >= 0 && j < e->eng->ds->J, CYC_ERR_ARGUMENT, "column out of range");
                       CYC_REQUIRE(g && h, CYC_ERR_ARGUMENT, "null output");
                       e->eng->gradient_hessian(j, use_w != 0, g, h));
}
extern "C" int cyc_engine_update_xbeta(cyc_engine* e, double delta, int j, int use_w) {
    return ENGINE_CALL(e, CYC_REQUIRE(j >= 0 && j < e->eng->ds->J, CYC_ERR_ARGUMENT, "column out of range");
                       e->eng->update_xbeta(delta, j, use_w != 0));
}
extern "C" int cyc_engine_get_log_likelihood(cyc_engine* e, int use_cv, double* out) {
    return ENGINE_CALL(e, CYC_REQUIRE(out, CYC_ERR_ARGUMENT, "null output");
                       *out = e->eng->log_likelihood(use_cv != 0));
}
extern "C" int cyc_engine_get_gradient_objective(cyc_engine* e, int use_cv, double* out) {
    return ENGINE_CALL(e, CYC_REQUIRE(out, CYC_ERR_ARGUMENT, "null output");
                       *out = e->eng->gradient_objective(use_cv != 0));
}
extern "C" int cyc_engine_get_predictive_log_likelihood(cyc_engine* e, const double* w, double* out) {
    return ENGINE_CALL(e, CYC_REQUIRE(w && out, CYC_ERR_ARGUMENT, "null argument");
                       *out = e->eng->predictive_log_likelihood(w));
}
extern "C" int cyc_engine_get_predictive_estimates(cyc_engine* e, double* y, const double* w) {
    return ENGINE_CALL(e, CYC_REQUIRE(y, CYC_ERR_ARGUMENT, "null output"); e->eng->predictive_estimates(y, w));
}
extern "C" int cyc_engine_get_xbeta(cyc_engine* e, double* out) {
    return ENGINE_CALL(e, CYC_REQUIRE(out, CYC_ERR_ARGUMENT, "null output"); e->eng->get_xbeta(out));
}
extern "C" int cyc_engine_save_xbeta(cyc_engine* e) {
    return ENGINE_CALL(e, e->eng->save_xbeta(); e->eng->sync());
}
extern "C" int cyc_engine_get_xbeta_save(cyc_engine* e, double* out) {
    return ENGINE_CALL(e, CYC_REQUIRE(out, CYC_ERR_ARGUMENT, "null output"); e->eng->get_xbeta_save(out));
}
extern "C" int cyc_engine_fisher_information(cyc_engine* e, const int* columns, int n, int use_cv, double* out) {
    return ENGINE_CALL(e, {
        CYC_REQUIRE((columns && out) || n == 0, CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(n >= 0, CYC_ERR_ARGUMENT, "negative column count");
        CYC_REQUIRE(!use_cv, CYC_ERR_UNSUPPORTED, "Weights are not yet implemented in Fisher Information calculations");
        e->eng->fisher_information(columns, n, out);
    });
}

extern "C" int cyc_engine_get_n(const cyc_engine* e, int* n) {
    return guarded([&] {
        CYC_REQUIRE(e && n, CYC_ERR_ARGUMENT, "null argument");
        *n = e->eng->N;
    });
}
