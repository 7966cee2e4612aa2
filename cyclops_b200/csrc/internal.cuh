// internal.cuh -- shared internals of libcyclops_b200.so (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "cyclops_b200.h"

namespace cyc {

// ---------------------------------------------------------------------------
// status handling: every C-ABI entry point returns a cyc_status and records a
// message in a thread-local string.
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);

struct Error {
    int status;
    std::string msg;
};

#define CYC_CHECK_CUDA(call)                                                            \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            throw ::cyc::Error{(e_ == cudaErrorMemoryAllocation) ? CYC_ERR_MEMORY       \
                                                                 : CYC_ERR_CUDA,        \
                               std::string(#call) + ": " + cudaGetErrorString(e_)};     \
        }                                                                               \
    } while (0)

// kernels launched by this library (counted by launch() below)
void count_launch();
// statistics reported by cyc_last_run_stats for the calling thread
void set_last_stats(const cyc_run_stats& s);

// reports a failed (or pending) launch with the call site
#define CYC_CHECK_LAUNCH()                                                              \
    do {                                                                                \
        cudaError_t e_ = cudaGetLastError();                                            \
        if (e_ != cudaSuccess)                                                          \
            throw ::cyc::Error{CYC_ERR_CUDA, std::string(__FILE__ ":") +                \
                               std::to_string(__LINE__) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define CYC_REQUIRE(cond, status, msg)                                                  \
    do {                                                                                \
        if (!(cond)) throw ::cyc::Error{(status), (msg)};                               \
    } while (0)

// every kernel of the library is launched through here: counted and checked
template <class Kern, class... Args>
inline void launch(Kern kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args... args) {
    kernel<<<grid, block, smem, stream>>>(args...);
    count_launch();
    CYC_CHECK_LAUNCH();
}

template <class F>
int guarded(F&& f) {
    // a non-sticky error left by an earlier, unrelated runtime call must not
    // be reported against this call's launches
    (void)cudaGetLastError();
    try {
        f();
        return CYC_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return CYC_ERR_MEMORY;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CYC_ERR_ARGUMENT;
    } catch (...) {
        set_error("unknown error");
        return CYC_ERR_ARGUMENT;
    }
}

// Device memory is stream-ordered: a buffer is allocated (cudaMallocAsync) on
// the stream its owner set for the calling thread (StreamScope) and freed
// (cudaFreeAsync) on that same stream, after the owner's work on it.  Neither
// waits for other streams, so fits running side by side on one device never
// stall one another the way cudaMalloc / cudaFree (device-wide waits) would.
// Without a scope a buffer falls back to cudaMalloc / cudaFree.
cudaStream_t& alloc_stream();          // per thread
void prepare_pool(int device);         // keeps freed memory cached in the device's pool

struct StreamScope {
    cudaStream_t prev;
    explicit StreamScope(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~StreamScope() { alloc_stream() = prev; }
    StreamScope(const StreamScope&) = delete;
    StreamScope& operator=(const StreamScope&) = delete;
};

// a named NVTX range for the object's lifetime: profilers (nsys, ncu --nvtx)
// see the library's entry points and solver phases by name; with no tool
// attached the calls return at once
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// a stream owned by an object; declared first among the owner's members so
// that it is destroyed last, after every buffer freed on it
struct OwnedStream {
    cudaStream_t s = nullptr;
    OwnedStream() = default;
    OwnedStream(const OwnedStream&) = delete;
    OwnedStream& operator=(const OwnedStream&) = delete;
    ~OwnedStream() { if (s) cudaStreamDestroy(s); }
};

// 64 pinned host bytes from a process-wide pool (allocated in chunks, never
// freed: cudaFreeHost would wait for the whole device)
void* pinned_block();
void release_pinned_block(void* p);

struct PinnedBlock {
    void* p = nullptr;
    PinnedBlock() : p(pinned_block()) {}
    ~PinnedBlock() { release_pinned_block(p); }
    PinnedBlock(const PinnedBlock&) = delete;
    PinnedBlock& operator=(const PinnedBlock&) = delete;
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// device buffer with RAII
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    bool ordered = false;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            if (ordered) cudaFreeAsync(p, s);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        s = alloc_stream();
        ordered = (s != nullptr);
        if (ordered) CYC_CHECK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), s));
        else CYC_CHECK_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    size_t bytes() const { return n * sizeof(T); }
    T* get() const { return p; }
};

// ---------------------------------------------------------------------------
// model traits (reference: src/cyclops/engine/ModelSpecifics.h)
// ---------------------------------------------------------------------------
__host__ __device__ inline bool model_grouped(int m) { return m == CYC_CLR || m == CYC_CPR; }
__host__ __device__ inline bool model_cumulative(int m) { return m == CYC_COX; }
__host__ __device__ inline bool model_independent(int m) { return m == CYC_LR || m == CYC_PR; }
// getDenomNullValue: 1 for logistic, 0 otherwise (:980, :1490, :814)
__host__ __device__ inline double denom_null(int m) { return m == CYC_LR ? 1.0 : 0.0; }
// observationCount: 1 for independent models, y otherwise (:982, :1492, :816, :1179)
__host__ __device__ inline double obs_count(int m, double y) { return model_independent(m) ? 1.0 : y; }
// likelihoodHasFixedTerms (:1488, :720)
__host__ __device__ inline bool has_fixed_ll(int m) { return m == CYC_PR || m == CYC_CPR; }

// ---------------------------------------------------------------------------
// column view (Iterators.h: IndicatorIterator / SparseIterator / DenseIterator
// / InterceptIterator)
// ---------------------------------------------------------------------------
struct ColView {
    int fmt;
    long long n;         // entries visited by the column's iterator
    const int* idx;      // SPARSE / INDICATOR row ids
    const double* val;   // SPARSE / DENSE values
    __device__ __forceinline__ int row(long long e) const {
        return (fmt == CYC_DENSE || fmt == CYC_INTERCEPT) ? (int)e : __ldg(idx + e);
    }
    __device__ __forceinline__ double x(long long e) const {
        return (fmt == CYC_SPARSE || fmt == CYC_DENSE) ? __ldg(val + e) : 1.0;
    }
    // isIndicator (Iterators.h:39, :399)
    __host__ __device__ bool indicator() const { return fmt == CYC_INDICATOR || fmt == CYC_INTERCEPT; }
};

// ---------------------------------------------------------------------------
// column batches of the batched solver (planned on the host, batch.cu)
// ---------------------------------------------------------------------------
struct RunPlan {
    int C = 0, G = 0;
    int batch_rows = 0;         // cap on a batch's entries in any one CTA's rows (0: none)
    int cap = 0, dmax = 0, max_levels = 0;   // the batch shape it was planned with (short-column
                                             // bound, shared rows, replay levels)
    std::vector<int> fixed;     // columns held fixed besides the offset (ascending)
    std::vector<int> len;       // J: columns in the batch starting here (1 = alone), 0 inside a batch
    std::vector<int> lvl;       // J: level of the column in its batch (1 + max level of earlier sharers)
    std::vector<int> dr0, nd;   // J (batch starts): its shared rows are drow[dr0, dr0 + nd)
    std::vector<int> drow;      // row ids shared by two or more columns of a batch
    std::vector<int> de_ptr;    // J+1: entries of column j on shared rows are de_*[de_ptr[j], de_ptr[j+1])
    std::vector<int> de_d;      // shared-row slot | (column within the batch << 8)
    std::vector<int> de_e;      // index of the entry's value (sparse columns), -1 for indicators
};

// ---------------------------------------------------------------------------
// dataset
// ---------------------------------------------------------------------------
struct Dataset {
    OwnedStream own;                // uploads and the dataset's buffers (declared first: destroyed last)
    cudaStream_t stream = nullptr;
    int device = 0;
    int model = 0;
    int K = 0, J = 0;
    int S = 0;                      // strata (renumbered by runs)
    bool has_offset = false, has_intercept = false;
    std::vector<int> fmt;
    std::vector<long long> col_ptr, val_ptr;
    std::vector<int> strat;         // K
    std::vector<int> strat_ptr;     // S+1 row offsets (rows sorted by stratum)
    std::vector<double> y, time;
    std::vector<int> h_idx;         // host copy of the indices (cox grouping)
    long long nnz_idx = 0, nnz_val = 0;

    DevBuf<int> d_fmt;
    DevBuf<long long> d_col_ptr, d_val_ptr;
    DevBuf<int> d_idx;
    DevBuf<double> d_val;
    DevBuf<double> d_y, d_time;
    DevBuf<int> d_strat, d_strat_ptr;

    // row-major copy for computeXBeta (built on first use, once: fits that run
    // concurrently on one dataset may ask for it together)
    std::mutex csr_mutex;
    bool have_csr = false;
    DevBuf<long long> d_row_ptr;
    DevBuf<int> d_row_col;
    DevBuf<double> d_row_val;

    // column batches of the batched solver, cached per (cluster size, fits per group)
    std::vector<RunPlan> run_plans;

    long long col_len(int j) const {
        return (fmt[j] == CYC_DENSE || fmt[j] == CYC_INTERCEPT) ? K : col_ptr[j + 1] - col_ptr[j];
    }
    ColView view(int j) const {
        ColView c;
        c.fmt = fmt[j];
        c.n = col_len(j);
        c.idx = d_idx.get() + col_ptr[j];
        c.val = d_val.get() + val_ptr[j];
        return c;
    }
    size_t device_bytes() const;
    void ensure_csr();
};

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum of two doubles; result valid in thread 0.  Fixed order.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sa[32], sb[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    __syncthreads();
    if (lane == 0) { sa[wid] = a; sb[wid] = b; }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (wid == 0) {
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
}

// Two-level deterministic reduction: every block writes its partial; the
// last block to finish (ticket) sums the partials in block order and calls
// `fin(total_a, total_b)` from thread 0.  `ticket` must be zero on entry and
// is left at zero.
template <class Fin>
__device__ __forceinline__ void grid_sum2_finalize(double a, double b, double2* partial,
                                                   unsigned* ticket, Fin fin) {
    block_sum2(a, b);
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = make_double2(a, b);
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        double sa = 0.0, sb = 0.0;
        for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
            const double2 p = __ldcg(partial + i);
            sa += p.x;
            sb += p.y;
        }
        block_sum2(sa, sb);
        if (threadIdx.x == 0) {
            fin(sa, sb);
            *ticket = 0u;
        }
    }
}

inline int grid_for(long long n, int items_per_thread = 4, int max_blocks = 148 * 8) {
    long long b = (n + (long long)kThreads * items_per_thread - 1) / ((long long)kThreads * items_per_thread);
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

// x*y then +, without contraction into an FMA (matches a non-FMA host build
// of the reference's `xBeta[k] += delta * x`).
__device__ __forceinline__ double add_mul_rn(double s, double a, double b) {
    return __dadd_rn(s, __dmul_rn(a, b));
}

// double-double helpers (Knuth two-sum)
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_add(DD a, DD b) {
    const double s = a.hi + b.hi;
    const double bb = s - a.hi;
    const double err = (a.hi - (s - bb)) + (b.hi - bb);
    const double lo = err + a.lo + b.lo;
    const double hi = s + lo;
    return DD{hi, lo - (hi - s)};
}
__device__ __forceinline__ DD dd_sub(DD a, DD b) { return dd_add(a, DD{-b.hi, -b.lo}); }


struct SegD {
    int f;        // segment start seen
    double v;
};
struct SegP {
    int f;
    DD a, b;
};
}  // namespace cyc

struct cyc_dataset {
    cyc::Dataset ds;
};
