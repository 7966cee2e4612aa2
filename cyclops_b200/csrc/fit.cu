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
#include <cmath>
#include <memory>

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
    if (delta != 0.0) atomicAdd(st.n_updates, 1ull);
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
    std::vector<int> fixb;
    DevBuf<double> beta, hdelta, gh, delta, obj, last;
    DevBuf<int> ptype, flags;
    DevBuf<unsigned long long> n_updates;
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
        std::vector<int> pt(J, prior.prior_type);
        for (int i = 0; i < prior.n_exclude; ++i) {
            CYC_REQUIRE(prior.exclude[i] >= 0 && prior.exclude[i] < J, CYC_ERR_ARGUMENT, "exclude index out of range");
            pt[prior.exclude[i]] = CYC_PRIOR_NONE;
        }
        beta.alloc(J); hdelta.alloc(J); gh.alloc(2); delta.alloc(1); obj.alloc(1); last.alloc(1);
        ptype.alloc(J); flags.alloc(2); n_updates.alloc(1);
        CYC_CHECK_CUDA(cudaMemcpyAsync(ptype.get(), pt.data(), J * sizeof(int), cudaMemcpyHostToDevice, e.stream));
        CYC_CHECK_CUDA(cudaMemsetAsync(n_updates.get(), 0, sizeof(unsigned long long), e.stream));
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
        return s;
    }

    void set_beta(const std::vector<double>& b) {
        CYC_CHECK_CUDA(cudaMemcpyAsync(beta.get(), b.data(), J * sizeof(double), cudaMemcpyHostToDevice, e.stream));
        e.compute_xbeta_device(beta.get());
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

    void run(cyc_fit_result* out) {
        const double* w = nullptr;
        (void)w;
        e.fixed_terms_ll(true);
        e.fixed_terms_gh(true);
        set_beta(h_start);
        e.remaining_statistics(true);
        build_graphs();
        CYC_CHECK_CUDA(cudaEventRecord(ev0, e.stream));
        double bound = ctl.initial_bound;
        int count = 0, flag = CYC_SUCCESS, iters = 0;
        for (;;) {                                               // update :586-615
            flag = find_mode(bound, &iters);
            ++count;
            if (flag == CYC_ILLCONDITIONED && count < ctl.max_bound_count) {
                bound /= 10.0;
                std::vector<double> b(J, 0.0);                   // resetBeta
                if (e.ds->has_offset) b[0] = 1.0;
                set_beta(b);
                e.remaining_statistics(true);
            } else {
                break;
            }
        }
        CYC_CHECK_CUDA(cudaEventRecord(ev1, e.stream));
        // results
        CYC_CHECK_CUDA(cudaMemcpyAsync(out->beta, beta.get(), J * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        e.launch_loglik(true, obj.get());
        launch(k_add_logprior, 1, kThreads, 0, e.stream, J, beta.get(), ptype.get(), variance, nullptr, last.get());
        double h2[2];
        CYC_CHECK_CUDA(cudaMemcpyAsync(&h2[0], obj.get(), sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        CYC_CHECK_CUDA(cudaMemcpyAsync(&h2[1], last.get(), sizeof(double), cudaMemcpyDeviceToHost, e.stream));
        unsigned long long nup = 0;
        CYC_CHECK_CUDA(cudaMemcpyAsync(&nup, n_updates.get(), sizeof(nup), cudaMemcpyDeviceToHost, e.stream));
        e.sync();
        out->log_likelihood = h2[0];
        out->log_prior = h2[1];
        out->iterations = iters;
        out->return_flag = flag;
        float ms = 0.f;
        CYC_CHECK_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        cyc_run_stats st{};
        st.kernel_ms = ms;
        st.coordinate_steps = (double)iters * J;
        st.cycles = iters;
        st.phases = 1;
        st.phase_ms[0] = ms;
        st.phase_state_bytes[0] = 8;
        set_last_stats(st);
        (void)nup;
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

extern "C" int cyc_fit_host_loop(cyc_dataset* ds, const cyc_prior* prior, const cyc_fit_spec* spec,
                                 const cyc_control* control, cyc_fit_result* out) {
    return guarded([&] {
        CYC_REQUIRE(ds && prior && spec && control && out && out->beta, CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(prior->prior_type >= CYC_PRIOR_NONE && prior->prior_type <= CYC_PRIOR_NORMAL,
                    CYC_ERR_ARGUMENT, "Unknown prior type");
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
