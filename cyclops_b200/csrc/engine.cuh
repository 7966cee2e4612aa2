// engine.cuh -- the per-coordinate engine (one fit's device state + stream).
#pragma once
#include <memory>

#include "internal.cuh"

namespace cyc {

struct Engine {
    explicit Engine(Dataset* d);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    OwnedStream own;              // the engine's stream (declared first: destroyed last)
    Dataset* ds;                  // borrowed: the caller keeps the dataset alive
    int device = 0;
    cudaStream_t stream = nullptr;
    int model = 0;
    int N = 0;              // denominators: K (lr/pr), strata (clr/cpr), risk-set groups (cox)
    bool use_w = false;     // weights set with useCrossValidation
    bool stats_known = false;

    DevBuf<double> xb, xb_save, exb, kw, denom, nw, numer, numer2, xjy;
    DevBuf<double> weights_buf, beta_buf;
    DevBuf<double2> partial;
    DevBuf<unsigned> ticket;
    DevBuf<double> result, ll_fixed;
    PinnedBlock h_block;          // results read back (pinned, from the process-wide pool)
    double* h_result = h_block.as<double>();

    // cox
    DevBuf<int> group, grow_ptr, gstart, gend, glist;
    DevBuf<long long> glist_ptr;
    DevBuf<double> D, P1h, P1l, P2h, P2l;
    DevBuf<double> R1, R2;             // scan scratch: n/D and n/D^2 per group
    DevBuf<SegD> aggD;
    DevBuf<SegP> aggP;
    std::vector<long long> h_glist_ptr;
    std::vector<int> h_first_group;

    void sync();
    void alloc_denominators();
    const int* groups() const;
    const int* group_rows() const;
    void regroup(const double* w);
    int first_group(int j) const;

    void set_weights(const double* w, bool use_cv);
    void fixed_terms_ll(bool use_cv);
    void fixed_terms_gh(bool use_cv);
    void zero_xbeta();
    void axpy_xbeta(double beta, int j);
    void compute_xbeta(const double* beta_host);
    void compute_xbeta_device(const double* d_beta);
    void remaining_statistics(bool use_weights);
    void numerator_for_gradient(int j, bool use_weights);
    void launch_gradient(int j, bool use_weights, double* out);
    void gradient_hessian(int j, bool use_weights, double* g, double* h);
    void launch_update(int j, bool use_weights, const double* d_delta, double delta);
    void update_xbeta(double delta, int j, bool use_weights);
    void cox_rescan(int lo);
    void cox_rescan_gated(const double* gate, int lo);
    void launch_loglik(bool use_cv, double* out);
    double log_likelihood(bool use_cv);
    void launch_gradient_objective(bool use_cv, double* out);
    double gradient_objective(bool use_cv);
    double predictive_log_likelihood(const double* w);
    void predictive_estimates(double* y, const double* w);
    void get_xbeta(double* out);
    void fisher_information(const int* cols, int n, double* out);
    void kkt_scores(const int* cols, const int* d_cols, int n, bool use_weights, double* d_out);
    void save_xbeta();
    void get_xbeta_save(double* out);
};

}  // namespace cyc

struct cyc_engine {
    cyc_dataset* owner = nullptr;
    std::unique_ptr<cyc::Engine> eng;
};
