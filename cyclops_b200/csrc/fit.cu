// fit.cu -- cyc_fit: one fit with the whole CCD loop on the GPU.
//
// The reference runs the loop on the host (CyclicCoordinateDescent::findMode,
// src/cyclops/CyclicCoordinateDescent.cpp:909-1216) and crosses into the
// engine three times per coordinate.  Here the coordinate step
// (ccdUpdateBeta + prior getDelta + applyBounds, :1394-1413, :1503-1520,
// src/cyclops/priors/CovariatePrior.h:186-188, 240-273, 410-415) runs in a
// one-thread kernel between the gradient and update kernels, beta / the trust
// region / delta stay in device memory, and one cycle is replayed as CUDA
// graphs.  The host reads two flags per cycle (the convergence test).
#include "engine.cuh"
#include "solver_common.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <memory>
#include <string>

namespace cyc {

static thread_local cyc_run_stats g_stats{};

namespace {

__global__ void k_step(int j, const double* __restrict__ gh, StepState st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double g = gh[0], h = gh[1];
    if (h < 0.0) { g = 0.0; h = 0.0; }                     // ccdUpdateBeta :1407-1410
    const double beta = st.beta[j];
    double delta = prior_delta(st.prior_type[j], st.variance, beta, g, h);
    delta = apply_bounds(st.hdelta + j, delta);
    if (delta != 0.0) st.beta[j] = beta + delta;
    *st.delta = delta;
    if (delta != 0.0) {
        atomicAdd(st.n_updates, 1ull);
        if (st.col_updates) st.col_updates[j] += 1u;
    }
}

// performCheckConvergence (CyclicCoordinateDescent.cpp:839-906) for the
// objective-based criteria; flags[0] = done, flags[1] = ill-conditioned
__global__ void k_check(const double* __restrict__ obj, double* __restrict__ last, double tol,
                        int iteration, int max_iter, int zhang_oles, int* __restrict__ flags) {
    if (threadIdx.x != 0) return;
    double conv;
    int ill = 0;
    const double o = *obj;
    if (!zhang_oles) {
        if (o != o) { conv = 0.0; ill = 1; }
        else conv = fabs(o - *last) / (fabs(o) + 1.0);
        *last = o;
    } else {
        conv = o;
    }
    int done = 0;
    if (tol > 0 && conv < tol) done = 1;
    else if (iteration == max_iter) done = 2;
    flags[0] = done;
    flags[1] = ill;
}

// computeZhangOlesConvergenceCriterion (CyclicCoordinateDescent.cpp:560-579), then saveXBeta
__global__ void k_zhang_oles(int K, const double* __restrict__ xb, double* __restrict__ xb_save,
                             const double* __restrict__ kw, int use_w, double2* partial,
                             unsigned* ticket, double* out) {
    double a = 0.0, b = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        const double w = use_w ? kw[k] : 1.0;
        a += fabs(xb[k] - xb_save[k]) * w;
        b += fabs(xb[k]) * w;
    }
    grid_sum2_finalize(a, b, partial, ticket, [&](double A, double B) { *out = A / (1.0 + B); });
}

__global__ void k_copy(int K, const double* __restrict__ src, double* __restrict__ dst) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) dst[k] = src[k];
}

// LANGE objective: log likelihood + log prior
__global__ void k_add_logprior(int J, const double* __restrict__ beta, const int* __restrict__ ptype,
                               double variance, const double* __restrict__ ll, double* __restrict__ out) {
    __shared__ double s[kThreads];
    double a = 0.0;
    for (int j = threadIdx.x; j < J; j += blockDim.x) a += log_density(ptype[j], variance, beta[j]);
    double dummy = 0.0;
    block_sum2(a, dummy);
    (void)s;
    if (threadIdx.x == 0) out[0] = (ll ? *ll : 0.0) + a;
}

}  // namespace

struct FitRunner {
    Engine& e;
    const cyc_control& ctl;
    int J;
    std::vector<int> fixb, base_fix, pt, graphs_fix;
    DevBuf<double> beta, hdelta, gh, delta, obj, last;
    DevBuf<int> ptype, flags;
    DevBuf<unsigned long long> n_updates;
    DevBuf<unsigned> col_updates;        // per column: coordinate steps that moved beta
    double variance;
    PinnedBlock h_block;                 // two flags read back per cycle (pinned, pooled)
    int* h_flags = h_block.as<int>();
    std::vector<cudaGraphExec_t> graphs;
    std::vector<double> h_start;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    FitRunner(Engine& eng, const cyc_prior& prior, const cyc_fit_spec& spec, const cyc_control& c)
        : e(eng), ctl(c), J(eng.ds->J), variance(spec.variance) {
        fixb.assign(J, 0);
        h_start.assign(J, 0.0);
        if (spec.start_beta) std::copy(spec.start_beta, spec.start_beta + J, h_start.begin());
        if (e.ds->has_offset) { fixb[0] = 1; h_start[0] = 1.0; }   // CCD init :218-221
        CYC_REQUIRE(spec.n_fixed >= 0 && (spec.n_fixed == 0 || spec.fixed), CYC_ERR_ARGUMENT, "bad fixed-column list");
        for (int i = 0; i < spec.n_fixed; ++i) {                 // setFixedBeta (fixedCoefficients)
            CYC_REQUIRE(spec.fixed[i] >= 0 && spec.fixed[i] < J, CYC_ERR_ARGUMENT, "fixed column out of range");
            fixb[spec.fixed[i]] = 1;
        }
        base_fix = fixb;
        pt.assign(J, prior.prior_type);
        for (int i = 0; i < prior.n_exclude; ++i) {
            CYC_REQUIRE(prior.exclude[i] >= 0 && prior.exclude[i] < J, CYC_ERR_ARGUMENT, "exclude index out of range");
            pt[prior.exclude[i]] = CYC_PRIOR_NONE;
        }
        beta.alloc(J); hdelta.alloc(J); gh.alloc(2); delta.alloc(1); obj.alloc(1); last.alloc(1);
        ptype.alloc(J); flags.alloc(2); n_updates.alloc(1); col_updates.alloc(J);
        CYC_CHECK_CUDA(cudaMemcpyAsync(ptype.get(), pt.data(), J * sizeof(int), cudaMemcpyHostToDevice, e.stream));
        CYC_CHECK_CUDA(cudaMemsetAsync(n_updates.get(), 0, sizeof(unsigned long long), e.stream));
        CYC_CHECK_CUDA(cudaMemsetAsync(col_updates.get(), 0, J * sizeof(unsigned), e.stream));
        CYC_CHECK_CUDA(cudaEventCreate(&ev0));
        CYC_CHECK_CUDA(cudaEventCreate(&ev1));
        e.sync();
    }
    ~FitRunner() {
        for (auto g : graphs) cudaGraphExecDestroy(g);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }

    StepState step_state() {
        StepState s;
        s.beta = beta.get();
        s.hdelta = hdelta.get();
        s.delta = delta.get();
        s.prior_type = ptype.get();
        s.variance = variance;
        s.n_updates = n_updates.get();
        s.col_updates = col_updates.get();
        return s;
    }

    void set_beta(const std::vector<double>& b) {
        CYC_CHECK_CUDA(cudaMemcpyAsync(beta.get(), b.data(), J * sizeof(double), cudaMemcpyHostToDevice, e.stream));
        // all zero (a cold start without an offset): xbeta is zero, and the
        // row-major copy the general case reads need not be built
        if (std::all_of(b.begin(), b.end(), [](double v) { return v == 0.0; })) e.zero_xbeta();
        else e.compute_xbeta_device(beta.get());
        e.sync();
    }

    void launch_coordinate(int j) {
        e.numerator_for_gradient(j, true);
        e.launch_gradient(j, true, gh.get());
        launch(k_step, 1, 32, 0, e.stream, j, gh.get(), step_state());
        CYC_CHECK_LAUNCH();
        e.launch_update(j, true, delta.get(), 0.0);
    }

    // one cycle as a list of graphs of at most `chunk` coordinates each
    void build_graphs() {
        for (auto g : graphs) CYC_CHECK_CUDA(cudaGraphExecDestroy(g));
        graphs.clear();
        graphs_fix = fixb;
        const int chunk = 4096;
        for (int b = 0; b < J; b += chunk) {
            cudaGraph_t g;
            CYC_CHECK_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
            for (int j = b; j < std::min(J, b + chunk); ++j)
                if (!fixb[j]) launch_coordinate(j);
            CYC_CHECK_CUDA(cudaStreamEndCapture(e.stream, &g));
            cudaGraphExec_t x;
            CYC_CHECK_CUDA(cudaGraphInstantiate(&x, g, 0));
            CYC_CHECK_CUDA(cudaGraphDestroy(g));
            graphs.push_back(x);
        }
    }

    void launch_objective(int conv) {
        if (conv == CYC_CONV_GRADIENT) {
            e.launch_gradient_objective(true, obj.get());
        } else if (conv == CYC_CONV_MITTAL) {
            e.launch_loglik(true, obj.get());
        } else if (conv == CYC_CONV_LANGE) {
            e.launch_loglik(true, obj.get());
            launch(k_add_logprior, 1, kThreads, 0, e.stream, J, beta.get(), ptype.get(), variance, obj.get(), obj.get());
        } else if (conv == CYC_CONV_ONE_STEP) {
            CYC_CHECK_CUDA(cudaMemsetAsync(obj.get(), 0, sizeof(double), e.stream));
        }
        CYC_CHECK_LAUNCH();
    }

    // findMode (CyclicCoordinateDescent.cpp:909-1216), cyclic branch
    int find_mode(double bound, int* iterations) {
        std::vector<double> hd(J, bound);                       // resetBounds
        CYC_CHECK_CUDA(cudaMemcpyAsync(hdelta.get(), hd.data(), J * sizeof(double), cudaMemcpyHostToDevice, e.stream));
        const int conv = ctl.convergence_type;
        CYC_REQUIRE(conv >= CYC_CONV_GRADIENT && conv <= CYC_CONV_ZHANG_OLES, CYC_ERR_ARGUMENT,
                    "Unknown convergence criterion");
        const int K = e.ds->K;
        if (conv < CYC_CONV_ZHANG_OLES) {
            launch_objective(conv);
            launch(k_copy, 1, 1, 0, e.stream, 1, obj.get(), last.get());
            CYC_CHECK_LAUNCH();
        } else {
            e.xb_save.alloc(K);
            launch(k_copy, grid_for(K, 1), kThreads, 0, e.stream, K, e.xb.get(), e.xb_save.get());
        }
        e.sync();
        int it = 0;
        for (;;) {
            for (auto g : graphs) CYC_CHECK_CUDA(cudaGraphLaunch(g, e.stream));
            it++;
            if (conv < CYC_CONV_ZHANG_OLES) {
                launch_objective(conv);
                launch(k_check, 1, 32, 0, e.stream, obj.get(), last.get(), ctl.tolerance, it, ctl.max_iterations, 0, flags.get());
                CYC_CHECK_LAUNCH();
            } else {
                launch(k_zhang_oles, grid_for(K, 4), kThreads, 0, e.stream, K, e.xb.get(), e.xb_save.get(), e.kw.get(),
                                                                        e.use_w, e.partial.get(), e.ticket.get(), obj.get());
                launch(k_copy, grid_for(K, 1), kThreads, 0, e.stream, K, e.xb.get(), e.xb_save.get());
                launch(k_check, 1, 32, 0, e.stream, obj.get(), last.get(), ctl.tolerance, it, ctl.max_iterations, 1, flags.get());
            }
            CYC_CHECK_CUDA(cudaMemcpyAsync(h_flags, flags.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, e.stream));
            e.sync();
            if (h_flags[0]) break;
        }
        *iterations = it;
        if (h_flags[0] == 1) return h_flags[1] ? CYC_ILLCONDITIONED : CYC_SUCCESS;
        return CYC_MAX_ITERATIONS;
    }

    // kktSwindle (CyclicCoordinateDescent.cpp:636-814).  The intercept and
    // the columns whose prior has no KKT boundary (flat, normal) start
    // active, the Laplace columns inactive at beta 0 (a nonzero start is
    // zeroed through updateXBeta, as setBeta does, :473-486).  Each pass runs
    // findMode over the active set (:617-634: every other column fixed), then
    // scores the inactive columns' |gradient| in one launch and moves every
    // column above lambda into the active set (the violators at the front of
    // the reference's sorted list, :739-792); it ends when nothing is
    // inactive, the fit failed, no column violates, or after max_iterations
    // passes (MAX_ITERATIONS).  An empty active set skips findMode.
    int kkt_swindle(double bound, int* iterations) {
        const int intercept = e.ds->has_intercept ? (e.ds->has_offset ? 1 : 0) : -1;
        std::vector<char> active(J, 0);
        int n_active = 0, n_inactive = 0;
        for (int j = 0; j < J; ++j) {
            if (base_fix[j]) continue;
            active[j] = (j == intercept || pt[j] != CYC_PRIOR_LAPLACE);
            if (active[j]) ++n_active;
            else ++n_inactive;
        }
        const double lambda = std::sqrt(2.0 / variance);      // getKktBoundary, CovariatePrior.h:235-238
        std::vector<double> hb(J);
        CYC_CHECK_CUDA(cudaMemcpyAsync(hb.data(), beta.get(), J * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        e.sync();
        for (int j = 0; j < J; ++j) {
            if (base_fix[j] || active[j] || hb[j] == 0.0) continue;
            CYC_CHECK_CUDA(cudaMemsetAsync(beta.get() + j, 0, sizeof(double), e.stream));
            e.launch_update(j, true, nullptr, 0.0 - hb[j]);
        }
        std::vector<int> inactive;
        DevBuf<int> d_inactive;
        DevBuf<double> d_score;
        std::vector<double> score;
        int flag = CYC_SUCCESS;
        for (int pass = 1;; ++pass) {
            flag = CYC_SUCCESS;
            if (n_active > 0) {
                for (int j = 0; j < J; ++j) fixb[j] = !active[j];
                build_graphs();
                flag = find_mode(bound, iterations);
            }
            if (n_inactive == 0 || flag != CYC_SUCCESS) break;
            if (pass == ctl.max_iterations) { flag = CYC_MAX_ITERATIONS; break; }
            inactive.clear();
            for (int j = 0; j < J; ++j)
                if (!base_fix[j] && !active[j]) inactive.push_back(j);
            const int n = (int)inactive.size();
            d_inactive.alloc(n);
            d_score.alloc(n);
            score.resize(n);
            CYC_CHECK_CUDA(cudaMemcpyAsync(d_inactive.get(), inactive.data(), n * sizeof(int), cudaMemcpyHostToDevice, e.stream));
            e.kkt_scores(inactive.data(), d_inactive.get(), n, true, d_score.get());
            CYC_CHECK_CUDA(cudaMemcpyAsync(score.data(), d_score.get(), n * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
            e.sync();
            int moved = 0;
            for (int i = 0; i < n; ++i)
                if (!(score[i] <= lambda)) { active[inactive[i]] = 1; ++moved; }
            if (moved == 0) break;
            n_active += moved;
            n_inactive -= moved;
        }
        fixb = base_fix;
        return flag;
    }

    bool swindle = false;

    // the graphs replay one cycle over the columns not fixed now
    void ensure_graphs() {
        if (graphs.empty() || graphs_fix != fixb) build_graphs();
    }

    // update (CyclicCoordinateDescent.cpp:586-615): findMode (or the
    // swindle), restarted from beta 0 with a tenfold smaller trust region
    // while ill-conditioned, at most max_bound_count times
    int update(int* iters) {
        double bound = ctl.initial_bound;
        int count = 0, flag = CYC_SUCCESS;
        for (;;) {
            if (!swindle) ensure_graphs();
            flag = swindle ? kkt_swindle(bound, iters) : find_mode(bound, iters);
            ++count;
            if (flag == CYC_ILLCONDITIONED && count < ctl.max_bound_count) {
                bound /= 10.0;
                std::vector<double> b(J, 0.0);                   // resetBeta :256-264
                if (e.ds->has_offset) b[0] = 1.0;
                set_beta(b);
                e.remaining_statistics(true);
            } else {
                break;
            }
        }
        return flag;
    }

    void prepare() {
        e.fixed_terms_ll(true);
        e.fixed_terms_gh(true);
        set_beta(h_start);
        e.remaining_statistics(true);
        // the swindle runs when some prior has a KKT boundary (JointPrior.h:149-157)
        swindle = ctl.use_kkt_swindle && std::count(pt.begin(), pt.end(), (int)CYC_PRIOR_LAPLACE) > 0;
        if (!swindle) ensure_graphs();
    }

    // getLogLikelihood and getLogPrior at the current state
    void objective_terms(double* ll, double* lp) {
        e.launch_loglik(true, obj.get());
        launch(k_add_logprior, 1, kThreads, 0, e.stream, J, beta.get(), ptype.get(), variance, nullptr, last.get());
        CYC_CHECK_LAUNCH();
        CYC_CHECK_CUDA(cudaMemcpyAsync(&h_block.as<double>()[1], obj.get(), sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(&h_block.as<double>()[2], last.get(), sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        e.sync();
        *ll = h_block.as<double>()[1];
        *lp = h_block.as<double>()[2];
    }

    void results(cyc_fit_result* out, int flag, int iters) {
        CYC_CHECK_CUDA(cudaMemcpyAsync(out->beta, beta.get(), J * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        objective_terms(&out->log_likelihood, &out->log_prior);
        out->iterations = iters;
        out->return_flag = flag;
    }

    // Algorithmic bytes of the coordinate loop (the bytes the algorithm must
    // move; FP64 state s = 8, s_x = 8 for real-valued columns and 0 for
    // indicators, w = 8 with row weights), per column j with nnz_j entries:
    //   lr / pr   gradient nnz_j (4 + s_x + s + w), update nnz_j (4 + s_x + 3 s);
    //   clr / cpr the same plus 16 B per stratum the column touches (at most
    //             one per entry) for the gradient and for an update;
    //   cox       numerator scatter nnz_j (4 + s_x + s + w) + 16 g_j, gradient
    //             32 g_j (the two double-double prefix sums at the g_j groups
    //             the column touches), update nnz_j (4 + s_x + 3 s + w)
    //             + 16 g_j and the rescan of the groups from the column's first
    //             to N at 56 B a group (denominator and group weight read; the
    //             accumulated denominator and two double-double prefix sums
    //             written).
    // Gradients count once per cycle for every column not fixed, updates once
    // per step that moved beta; each convergence check reads K (2 s + 8).
    double algorithmic_bytes(int iters, const std::vector<unsigned>& upd) const {
        const Dataset& ds = *e.ds;
        const int K = ds.K;
        const double w = e.use_w ? 8.0 : 0.0;
        double bytes = (double)(iters + 1) * K * (2 * 8.0 + 8.0);
        for (int j = 0; j < J; ++j) {
            if (fixb[j]) continue;
            const int f = ds.fmt[j];
            const bool dense = (f == CYC_DENSE || f == CYC_INTERCEPT);
            const double n = dense ? (double)K : (double)(ds.col_ptr[j + 1] - ds.col_ptr[j]);
            const double sx = (f == CYC_INDICATOR || f == CYC_INTERCEPT) ? 0.0 : 8.0;
            const double si = dense ? 0.0 : 4.0;
            double grad, upd_b;
            if (model_cumulative(ds.model)) {
                const double g = (double)(e.h_glist_ptr[j + 1] - e.h_glist_ptr[j]);
                grad = n * (si + sx + 8.0 + w) + 16.0 * g + 32.0 * g;
                upd_b = n * (si + sx + 24.0 + w) + 16.0 * g + 56.0 * (double)std::max(0, e.N - e.first_group(j));
            } else if (model_grouped(ds.model)) {
                grad = n * (si + sx + 8.0 + w) + 16.0 * n;
                upd_b = n * (si + sx + 24.0) + 16.0 * n;
            } else {
                grad = n * (si + sx + 8.0 + w);
                upd_b = n * (si + sx + 24.0);
            }
            bytes += (double)iters * grad + (double)upd[j] * upd_b;
        }
        return bytes;
    }

    void run(cyc_fit_result* out) {
        prepare();
        CYC_CHECK_CUDA(cudaEventRecord(ev0, e.stream));
        int iters = 0;
        const int flag = update(&iters);
        CYC_CHECK_CUDA(cudaEventRecord(ev1, e.stream));
        results(out, flag, iters);
        float ms = 0.f;
        CYC_CHECK_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        std::vector<unsigned> upd(J);
        CYC_CHECK_CUDA(cudaMemcpyAsync(upd.data(), col_updates.get(), J * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                       e.stream));
        e.sync();
        cyc_run_stats st{};
        st.kernel_ms = ms;
        st.coordinate_steps = (double)iters * J;
        st.cycles = iters;
        st.phases = 1;
        st.phase_ms[0] = ms;
        st.phase_state_bytes[0] = 8;
        // the swindle's passes run findMode over changing active sets: not counted
        st.algorithmic_bytes = swindle ? 0.0 : algorithmic_bytes(iters, upd);
        st.phase_bytes[0] = st.algorithmic_bytes;
        for (int j = 0; j < J; ++j) {
            if (fixb[j]) continue;
            const int f = e.ds->fmt[j];
            const double n = (f == CYC_DENSE || f == CYC_INTERCEPT) ? (double)e.ds->K
                                                                    : (double)(e.ds->col_ptr[j + 1] - e.ds->col_ptr[j]);
            st.gradient_entries += (double)iters * n;
            st.update_entries += (double)upd[j] * n;
        }
        set_last_stats(st);
    }

    // ---- profile likelihood (CcdInterface.cpp:223-420) ----------------------

    // setBeta(j, x) (CyclicCoordinateDescent.cpp:473-486): beta_j += x - beta_j
    // through updateXBeta, so the statistics stay current
    void set_coordinate(int j, double x) {
        double* hb = h_block.as<double>() + 3;
        CYC_CHECK_CUDA(cudaMemcpyAsync(hb, beta.get() + j, sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        e.sync();
        const double delta = x - hb[0];
        hb[0] += delta;
        CYC_CHECK_CUDA(cudaMemcpyAsync(beta.get() + j, hb, sizeof(double), cudaMemcpyHostToDevice, e.stream));
        e.launch_update(j, true, nullptr, delta);
        e.sync();
    }

    // OptimizationProfile::objective (CcdInterface.cpp:238-249): beta_j = x
    // held fixed while update refits the rest from the current state
    double profile_objective(int j, double x, double mode, double threshold, bool penalty, int* evals) {
        ++*evals;
        set_coordinate(j, x);
        fixb[j] = base_fix[j] = 1;
        int iters = 0;
        update(&iters);
        fixb[j] = base_fix[j] = 0;
        double ll, lp;
        objective_terms(&ll, &lp);
        double y = ll + threshold - mode;
        if (penalty) y += lp;
        return y;
    }

    // RZeroIn::bracketSignChange (src/utils/RZeroIn.h): steps of 0.1, 0.2,
    // 0.4, ... times max(|x0|, 0.01) from x0 until the objective is no
    // longer positive; a NaN objective when it turns NaN or after 22 steps
    double bracket(int j, double x0, double f0, double direction, double* f1, double mode, double threshold,
                   bool penalty, int* evals) {
        const double displacement = std::max(std::fabs(x0), 0.01);
        double multiplier = 0.1;
        double x1 = x0, y1 = f0;
        for (int steps = 0; y1 > 0; ++steps) {
            x1 = x0 + direction * displacement * multiplier;
            y1 = profile_objective(j, x1, mode, threshold, penalty, evals);
            if (std::isnan(y1)) break;
            if (steps > 20) { y1 = NAN; break; }
            multiplier *= 2.0;
        }
        *f1 = y1;
        return x1;
    }

    // Brent's root finder in the form of Forsythe, Malcolm & Moler
    // (Computer Methods for Mathematical Computations, 1977, zeroin), the
    // variant RZeroIn::getRoot runs: given f(a), f(b) of opposite signs, each
    // step takes inverse quadratic (or secant) interpolation when it lands
    // well inside [b, c] and shrinks the bracket fast enough, bisection
    // otherwise; it stops when half the bracket is within 2 eps |b| + tol / 2
    // or after max_it + 1 steps
    double root(int j, double a, double b, double fa, double fb, double tol, int max_it, double mode,
                double threshold, bool penalty, int* evals) {
        if (b < a) {
            std::swap(a, b);
            std::swap(fa, fb);
        }
        if (fa == 0.0) return a;
        if (fb == 0.0) return b;
        double c = a, fc = fa;
        for (int k = 0; k <= max_it; ++k) {
            const double prev_step = b - a;
            if (std::fabs(fc) < std::fabs(fb)) {                 // b: the best point so far
                a = b; b = c; c = a;
                fa = fb; fb = fc; fc = fa;
            }
            const double tol_act = 2 * DBL_EPSILON * std::fabs(b) + tol / 2;
            double step = (c - b) / 2;
            if (std::fabs(step) <= tol_act || fb == 0.0) return b;
            if (std::fabs(prev_step) >= tol_act && std::fabs(fa) > std::fabs(fb)) {
                const double cb = c - b;
                double p, q;
                if (a == c) {                                    // secant
                    const double t1 = fb / fa;
                    p = cb * t1;
                    q = 1.0 - t1;
                } else {                                         // inverse quadratic
                    const double r = fa / fc, t1 = fb / fc, t2 = fb / fa;
                    p = t2 * (cb * r * (r - t1) - (b - a) * (t1 - 1.0));
                    q = (r - 1.0) * (t1 - 1.0) * (t2 - 1.0);
                }
                if (p > 0) q = -q;
                else p = -p;
                if (p < (0.75 * cb * q - std::fabs(tol_act * q) / 2) && p < std::fabs(prev_step * q / 2)) step = p / q;
            }
            if (std::fabs(step) < tol_act) step = step > 0 ? tol_act : -tol_act;
            a = b;
            fa = fb;
            b += step;
            fb = profile_objective(j, b, mode, threshold, penalty, evals);
            if ((fb > 0 && fc > 0) || (fb < 0 && fc < 0)) {
                c = a;
                fc = fa;
            }
        }
        return b;
    }

    // evaluateProfileModel with one thread (CcdInterface.cpp:527-618): fit;
    // makeDirty (CyclicCoordinateDescent.cpp:448-452), so the first refit
    // rebuilds the fixed terms, xbeta and the statistics from beta; one
    // refit at 0; then the objective (threshold 0, mode 0) at each point,
    // each refit warm-started from the last
    void profile_points(int j, const double* points, int n, bool penalty, double* values) {
        prepare();
        int iters = 0;
        update(&iters);
        set_coordinate(j, 0.0);
        e.fixed_terms_ll(true);
        e.fixed_terms_gh(true);
        e.compute_xbeta_device(beta.get());
        e.remaining_statistics(true);
        fixb[j] = base_fix[j] = 1;
        update(&iters);
        fixb[j] = base_fix[j] = 0;
        int evals = 0;
        for (int i = 0; i < n; ++i) values[i] = profile_objective(j, points[i], 0.0, 0.0, penalty, &evals);
    }

    // profileModel with one thread (CcdInterface.cpp:262-420): fit, then for
    // each column its upper and then its lower bound, all on one state
    void profile(const int* cols, int n, double threshold, bool penalty, double* lower, double* upper,
                 int* evaluations, cyc_fit_result* out) {
        prepare();
        int iters = 0;
        const int flag = update(&iters);
        std::vector<double> x0s(J);
        CYC_CHECK_CUDA(cudaMemcpyAsync(x0s.data(), beta.get(), J * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        double ll, lp;
        objective_terms(&ll, &lp);
        if (out) {
            std::copy(x0s.begin(), x0s.end(), out->beta);
            out->log_likelihood = ll;
            out->log_prior = lp;
            out->iterations = iters;
            out->return_flag = flag;
        }
        const double mode = penalty ? ll + lp : ll;
        for (int i = 0; i < n; ++i) {
            const int j = cols[i];
            int count = 0;
            for (double direction : {1.0, -1.0}) {
                int evals = 0;
                double f1;
                const double x1 = bracket(j, x0s[j], threshold, direction, &f1, mode, threshold, penalty, &evals);
                const double pt = std::isnan(f1) ? NAN
                                                 : root(j, x0s[j], x1, threshold, f1, 1e-3, 1000, mode, threshold,
                                                        penalty, &evals);
                (direction > 0 ? upper : lower)[i] = pt;
                count += evals;
            }
            evaluations[i] = count;
        }
    }
};

void set_last_stats(const cyc_run_stats& s) { g_stats = s; }

// CyclicCoordinateDescent::findMode / update with the host driving the
// engine one call at a time (src/cyclops/CyclicCoordinateDescent.cpp:586-615,
// 909-1216): every coordinate reads (gradient, Hessian) back, takes the
// step on the host and launches the update.  The plain FP64 single-fit GPU
// CCD, kept as the measured baseline of the device-resident solvers.
static void host_loop_fit(Engine& e, const cyc_prior& prior, const cyc_fit_spec& spec, const cyc_control& ctl,
                          cyc_fit_result* out) {
    const int J = e.ds->J;
    const int K = e.ds->K;
    std::vector<int> fixb(J, 0), pt(J, prior.prior_type);
    for (int i = 0; i < prior.n_exclude; ++i) {
        CYC_REQUIRE(prior.exclude[i] >= 0 && prior.exclude[i] < J, CYC_ERR_ARGUMENT, "exclude index out of range");
        pt[prior.exclude[i]] = CYC_PRIOR_NONE;
    }
    std::vector<double> beta(J, 0.0);
    if (spec.start_beta) std::copy(spec.start_beta, spec.start_beta + J, beta.begin());
    if (e.ds->has_offset) { fixb[0] = 1; beta[0] = 1.0; }
    CYC_REQUIRE(spec.n_fixed >= 0 && (spec.n_fixed == 0 || spec.fixed), CYC_ERR_ARGUMENT, "bad fixed-column list");
    for (int i = 0; i < spec.n_fixed; ++i) {
        CYC_REQUIRE(spec.fixed[i] >= 0 && spec.fixed[i] < J, CYC_ERR_ARGUMENT, "fixed column out of range");
        fixb[spec.fixed[i]] = 1;
    }
    const int conv = ctl.convergence_type;
    CYC_REQUIRE(conv >= CYC_CONV_GRADIENT && conv <= CYC_CONV_ZHANG_OLES, CYC_ERR_ARGUMENT,
                "Unknown convergence criterion");
    auto log_prior = [&]() {
        double s = 0.0;
        for (int j = 0; j < J; ++j) s += log_density(pt[j], spec.variance, beta[j]);
        return s;
    };
    auto objective = [&]() {
        if (conv == CYC_CONV_GRADIENT) return e.gradient_objective(true);
        if (conv == CYC_CONV_MITTAL) return e.log_likelihood(true);
        if (conv == CYC_CONV_LANGE) return e.log_likelihood(true) + log_prior();
        return 0.0;
    };
    std::vector<double> xb(K), xs(K), kw(K, 1.0);
    if (spec.weights) std::copy(spec.weights, spec.weights + K, kw.begin());
    auto zhang_oles = [&]() {
        e.get_xbeta(xb.data());
        double d = 0.0, r = 0.0;
        for (int k = 0; k < K; ++k) {
            const double w = spec.weights ? kw[k] : 1.0;
            d += std::fabs(xb[k] - xs[k]) * w;
            r += std::fabs(xb[k]) * w;
        }
        xs = xb;
        return d / (1.0 + r);
    };
    e.fixed_terms_ll(true);
    e.fixed_terms_gh(true);
    e.compute_xbeta(beta.data());
    e.remaining_statistics(true);
    std::vector<double> hd(J);
    double bound = ctl.initial_bound;
    int count = 0, flag = CYC_SUCCESS, it = 0;
    for (;;) {
        std::fill(hd.begin(), hd.end(), bound);
        double last = 0.0;
        if (conv < CYC_CONV_ZHANG_OLES) last = objective();
        else e.get_xbeta(xs.data());
        it = 0;
        bool done = false;
        while (!done) {
            for (int j = 0; j < J; ++j) {
                if (fixb[j]) continue;
                double g, h;
                e.numerator_for_gradient(j, true);
                e.gradient_hessian(j, true, &g, &h);
                if (h < 0.0) { g = 0.0; h = 0.0; }
                double delta = prior_delta(pt[j], spec.variance, beta[j], g, h);
                delta = apply_bounds(&hd[j], delta);
                if (delta != 0.0) {
                    beta[j] += delta;
                    e.update_xbeta(delta, j, true);
                }
            }
            ++it;
            double c;
            bool ill = false;
            if (conv < CYC_CONV_ZHANG_OLES) {
                const double o = objective();
                if (o != o) { c = 0.0; ill = true; }
                else c = std::fabs(o - last) / (std::fabs(o) + 1.0);
                last = o;
            } else {
                c = zhang_oles();
            }
            if (ctl.tolerance > 0 && c < ctl.tolerance) { flag = ill ? CYC_ILLCONDITIONED : CYC_SUCCESS; done = true; }
            else if (it == ctl.max_iterations) { flag = CYC_MAX_ITERATIONS; done = true; }
        }
        ++count;
        if (flag == CYC_ILLCONDITIONED && count < ctl.max_bound_count) {
            bound /= 10.0;
            for (int j = e.ds->has_offset ? 1 : 0; j < J; ++j) beta[j] = 0.0;
            e.compute_xbeta(beta.data());
            e.remaining_statistics(true);
        } else {
            break;
        }
    }
    std::copy(beta.begin(), beta.end(), out->beta);
    out->log_likelihood = e.log_likelihood(true);
    out->log_prior = log_prior();
    out->iterations = it;
    out->return_flag = flag;
}

}  // namespace cyc

using namespace cyc;

extern "C" int cyc_fit(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                       const cyc_control* control, cyc_fit_result* out) {
    return guarded([&] {
        NvtxRange range("cyc_fit");
        CYC_REQUIRE(ds && prior && spec && control && out && out->beta, CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(prior->prior_type >= CYC_PRIOR_NONE && prior->prior_type <= CYC_PRIOR_NORMAL,
                    CYC_ERR_ARGUMENT, "Unknown prior type");
        CYC_REQUIRE(prior->prior_type == CYC_PRIOR_NONE || spec->variance > 0, CYC_ERR_ARGUMENT,
                    "prior variance must be positive");
        CYC_CHECK_CUDA(cudaSetDevice(ds->ds.device));
        Engine eng(&ds->ds);
        StreamScope scope(eng.stream);
        eng.set_weights(spec->weights, spec->weights != nullptr);
        FitRunner r(eng, *prior, *spec, *control);
        r.run(out);
    });
}

extern "C" int cyc_profile_bounds(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                                  const cyc_control* control, const int* columns, int n, double threshold,
                                  int include_penalty, int override_no_regularization, double* lower,
                                  double* upper, int* evaluations, cyc_fit_result* fit) {
    return guarded([&] {
        NvtxRange range("cyc_profile_bounds");
        CYC_REQUIRE(ds && prior && spec && control && n >= 0, CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(n == 0 || (columns && lower && upper && evaluations), CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(!fit || fit->beta, CYC_ERR_ARGUMENT, "null result buffer");
        CYC_REQUIRE(prior->prior_type >= CYC_PRIOR_NONE && prior->prior_type <= CYC_PRIOR_NORMAL,
                    CYC_ERR_ARGUMENT, "Unknown prior type");
        CYC_REQUIRE(prior->prior_type == CYC_PRIOR_NONE || spec->variance > 0, CYC_ERR_ARGUMENT,
                    "prior variance must be positive");
        const Dataset& d = ds->ds;
        for (int i = 0; i < n; ++i)
            CYC_REQUIRE(columns[i] >= 0 && columns[i] < d.J && !(d.has_offset && columns[i] == 0), CYC_ERR_ARGUMENT,
                        "profile column out of range (or the offset)");
        CYC_CHECK_CUDA(cudaSetDevice(d.device));
        Engine eng(&ds->ds);
        StreamScope scope(eng.stream);
        eng.set_weights(spec->weights, spec->weights != nullptr);
        FitRunner r(eng, *prior, *spec, *control);
        for (int i = 0; i < n; ++i) {                     // CcdInterface.cpp:297-302, R/ModelFit.R:774-778
            CYC_REQUIRE(override_no_regularization || r.pt[columns[i]] == CYC_PRIOR_NONE, CYC_ERR_ARGUMENT,
                        "Variable " + std::to_string(columns[i]) + " is regularized.");
            CYC_REQUIRE(!r.base_fix[columns[i]], CYC_ERR_ARGUMENT,
                        "Cannot estimate confidence interval for a fixed coefficient");
        }
        r.profile(columns, n, threshold, include_penalty != 0, lower, upper, evaluations, fit);
    });
}

extern "C" int cyc_profile_log_likelihood(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                                          const cyc_control* control, int column, const double* points, int n,
                                          int include_penalty, double* values) {
    return guarded([&] {
        NvtxRange range("cyc_profile_log_likelihood");
        CYC_REQUIRE(ds && prior && spec && control && n >= 0 && (n == 0 || (points && values)), CYC_ERR_ARGUMENT,
                    "null argument");
        CYC_REQUIRE(prior->prior_type >= CYC_PRIOR_NONE && prior->prior_type <= CYC_PRIOR_NORMAL,
                    CYC_ERR_ARGUMENT, "Unknown prior type");
        CYC_REQUIRE(prior->prior_type == CYC_PRIOR_NONE || spec->variance > 0, CYC_ERR_ARGUMENT,
                    "prior variance must be positive");
        const Dataset& d = ds->ds;
        CYC_REQUIRE(column >= 0 && column < d.J && !(d.has_offset && column == 0), CYC_ERR_ARGUMENT,
                    "profile column out of range (or the offset)");
        CYC_CHECK_CUDA(cudaSetDevice(d.device));
        Engine eng(&ds->ds);
        StreamScope scope(eng.stream);
        eng.set_weights(spec->weights, spec->weights != nullptr);
        FitRunner r(eng, *prior, *spec, *control);
        CYC_REQUIRE(!r.base_fix[column], CYC_ERR_ARGUMENT, "cannot profile a fixed coefficient");
        r.profile_points(column, points, n, include_penalty != 0, values);
    });
}

extern "C" int cyc_fit_host_loop(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                                 const cyc_control* control, cyc_fit_result* out) {
    return guarded([&] {
        NvtxRange range("cyc_fit_host_loop");
        CYC_REQUIRE(ds && prior && spec && control && out && out->beta, CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(prior->prior_type >= CYC_PRIOR_NONE && prior->prior_type <= CYC_PRIOR_NORMAL,
                    CYC_ERR_ARGUMENT, "Unknown prior type");
        CYC_REQUIRE(!control->use_kkt_swindle, CYC_ERR_UNSUPPORTED, "the KKT swindle is offered by cyc_fit only");
        CYC_CHECK_CUDA(cudaSetDevice(ds->ds.device));
        Engine eng(&ds->ds);
        StreamScope scope(eng.stream);
        eng.set_weights(spec->weights, spec->weights != nullptr);
        cudaEvent_t e0, e1;
        CYC_CHECK_CUDA(cudaEventCreate(&e0));
        CYC_CHECK_CUDA(cudaEventCreate(&e1));
        CYC_CHECK_CUDA(cudaEventRecord(e0, eng.stream));
        host_loop_fit(eng, *prior, *spec, *control, out);
        CYC_CHECK_CUDA(cudaEventRecord(e1, eng.stream));
        CYC_CHECK_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cyc_run_stats st{};
        st.kernel_ms = ms;
        st.cycles = out->iterations;
        st.phases = 1;
        st.phase_ms[0] = ms;
        st.phase_state_bytes[0] = 8;
        set_last_stats(st);
    });
}

extern "C" int cyc_last_run_stats(cyc_run_stats* out) {
    return guarded([&] {
        CYC_REQUIRE(out, CYC_ERR_ARGUMENT, "null argument");
        *out = g_stats;
    });
}
