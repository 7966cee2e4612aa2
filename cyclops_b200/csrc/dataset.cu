// dataset.cu -- device-resident column store (the engine's view of the
// reference's ModelData / CompressedDataMatrix).
//
// HBM layout (one dataset, shared read-only by every engine and fit):
//   d_fmt[J]          int32 column formats
//   d_col_ptr[J+1]    int64 offsets into d_idx
//   d_idx[nnz]        int32 row ids, ascending within a column; one flat
//                     array so a column is one contiguous, coalesced range
//   d_val_ptr[J+1]    int64 offsets into d_val
//   d_val[...]        float64 SPARSE values (parallel to d_idx) and DENSE
//                     columns (K values each)
//   d_y, d_time[K]    float64
//   d_strat[K]        int32 stratum of each row, renumbered by runs
//   d_strat_ptr[S+1]  int32 first row of each stratum
// plus, on first computeXBeta with a nonzero coefficient, a row-major copy
// (d_row_ptr / d_row_col / d_row_val) whose per-row column order equals the
// reference's column-by-column axpy order.
#include "internal.cuh"

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <atomic>

namespace cyc {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {
std::mutex g_pinned_mutex;
std::vector<void*>& pinned_free() {
    static std::vector<void*>* v = new std::vector<void*>();   // lives to process exit
    return *v;
}
}  // namespace

void* pinned_block() {
    std::lock_guard<std::mutex> lk(g_pinned_mutex);
    auto& fl = pinned_free();
    if (fl.empty()) {
        char* chunk = nullptr;
        CYC_CHECK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&chunk), 64 * 512));
        for (int i = 511; i >= 0; --i) fl.push_back(chunk + 64 * i);
    }
    void* p = fl.back();
    fl.pop_back();
    return p;
}

void release_pinned_block(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pinned_mutex);
    pinned_free().push_back(p);
}

cudaStream_t& alloc_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}

// freed memory stays in the device's default pool for the next allocation
// instead of going back to the driver at every synchronisation (a setting of
// this process's pool, not of the GPU)
void prepare_pool(int device) {
    static std::mutex m;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(m);
    for (int d : done)
        if (d == device) return;
    cudaMemPool_t pool;
    CYC_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    unsigned long long keep = ~0ull;
    CYC_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    done.push_back(device);
}

size_t Dataset::device_bytes() const {
    return d_fmt.bytes() + d_col_ptr.bytes() + d_val_ptr.bytes() + d_idx.bytes() + d_val.bytes() +
           d_y.bytes() + d_time.bytes() + d_strat.bytes() + d_strat_ptr.bytes() + d_row_ptr.bytes() +
           d_row_col.bytes() + d_row_val.bytes();
}

// on the calling thread's allocation stream (the dataset's, during uploads)
template <class T>
static void upload(DevBuf<T>& buf, const T* src, size_t n) {
    buf.alloc(n);
    if (n) CYC_CHECK_CUDA(cudaMemcpyAsync(buf.get(), src, n * sizeof(T), cudaMemcpyHostToDevice, alloc_stream()));
}

void Dataset::ensure_csr() {
    std::lock_guard<std::mutex> lock(csr_mutex);
    if (have_csr) return;
    StreamScope scope(stream);
    // counting sort by row; columns visited in ascending order, so each row
    // lists its columns ascending (the order of zeroXBeta + axpyXBeta per j,
    // CyclicCoordinateDescent.cpp:1452-1470)
    std::vector<long long> rp(K + 1, 0);
    for (int j = 0; j < J; ++j) {
        const long long n = col_len(j);
        if (fmt[j] == CYC_DENSE || fmt[j] == CYC_INTERCEPT) {
            for (int k = 0; k < K; ++k) rp[k + 1]++;
        } else {
            for (long long e = 0; e < n; ++e) rp[h_idx[col_ptr[j] + e] + 1]++;
        }
    }
    for (int k = 0; k < K; ++k) rp[k + 1] += rp[k];
    std::vector<long long> cur(rp.begin(), rp.end() - 1);
    std::vector<int> rc(rp[K]);
    std::vector<double> rv(rp[K]);
    std::vector<double> hval(nnz_val);
    if (nnz_val) {
        CYC_CHECK_CUDA(cudaMemcpyAsync(hval.data(), d_val.get(), nnz_val * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CYC_CHECK_CUDA(cudaStreamSynchronize(stream));
    }
    for (int j = 0; j < J; ++j) {
        const int f = fmt[j];
        const long long n = col_len(j);
        for (long long e = 0; e < n; ++e) {
            const int k = (f == CYC_DENSE || f == CYC_INTERCEPT) ? (int)e : h_idx[col_ptr[j] + e];
            const double x = (f == CYC_DENSE || f == CYC_SPARSE) ? hval[val_ptr[j] + e] : 1.0;
            const long long p = cur[k]++;
            rc[p] = j;
            rv[p] = x;
        }
    }
    upload(d_row_ptr, rp.data(), rp.size());
    upload(d_row_col, rc.data(), rc.size());
    upload(d_row_val, rv.data(), rv.size());
    CYC_CHECK_CUDA(cudaStreamSynchronize(stream));   // usable from every stream
    have_csr = true;
}

}  // namespace cyc

using namespace cyc;

extern "C" const char* cyc_last_error(void) { return g_last_error.c_str(); }
extern "C" int cyc_version(void) { return CYC_ABI_VERSION; }
extern "C" long long cyc_launch_count(void) { return g_launches.load(); }

extern "C" int cyc_dataset_create(const cyc_data_desc* d, int device, cyc_dataset** out) {
    return guarded([&] {
        NvtxRange range("cyc_dataset_create");
        CYC_REQUIRE(d && out, CYC_ERR_ARGUMENT, "null argument");
        *out = nullptr;
        CYC_REQUIRE(d->K > 0 && d->J > 0, CYC_ERR_ARGUMENT, "K and J must be positive");
        CYC_REQUIRE(d->model >= CYC_LR && d->model <= CYC_COX, CYC_ERR_ARGUMENT, "Invalid model type.");
        CYC_REQUIRE(d->y && d->col_format && d->col_ptr && d->val_ptr, CYC_ERR_ARGUMENT, "missing arrays");
        CYC_REQUIRE(d->model != CYC_COX || d->time, CYC_ERR_ARGUMENT, "cox needs survival times");
        // a NaN or an infinity among the outcomes, times or covariate values
        // leaves every fit undefined (the reference's fit on such data comes
        // back ILLCONDITIONED with NaN coefficients), so such data is refused
        // before any device work
        auto finite = [](const double* a, long long n) {
            for (long long i = 0; i < n; ++i)
                if (!std::isfinite(a[i])) return false;
            return true;
        };
        CYC_REQUIRE(finite(d->y, d->K), CYC_ERR_ARGUMENT, "non-finite outcome (y)");
        CYC_REQUIRE(!d->time || finite(d->time, d->K), CYC_ERR_ARGUMENT, "non-finite time");
        CYC_REQUIRE(d->val_ptr[d->J] >= 0, CYC_ERR_ARGUMENT, "offsets must not decrease");
        CYC_REQUIRE(!d->col_val || finite(d->col_val, d->val_ptr[d->J]), CYC_ERR_ARGUMENT,
                    "non-finite covariate value");
        int ndev = 0;
        CYC_CHECK_CUDA(cudaGetDeviceCount(&ndev));
        CYC_REQUIRE(device >= 0 && device < ndev, CYC_ERR_ARGUMENT, "no such CUDA device");
        CYC_CHECK_CUDA(cudaSetDevice(device));

        auto* h = new cyc_dataset();
        std::unique_ptr<cyc_dataset> guard(h);
        Dataset& s = h->ds;
        s.device = device;
        prepare_pool(device);
        CYC_CHECK_CUDA(cudaStreamCreateWithFlags(&s.own.s, cudaStreamNonBlocking));
        s.stream = s.own.s;
        StreamScope scope(s.stream);
        s.model = d->model;
        s.K = d->K;
        s.J = d->J;
        s.has_offset = d->has_offset != 0;
        s.has_intercept = d->has_intercept != 0;
        s.fmt.assign(d->col_format, d->col_format + d->J);
        s.col_ptr.assign(d->col_ptr, d->col_ptr + d->J + 1);
        s.val_ptr.assign(d->val_ptr, d->val_ptr + d->J + 1);
        s.nnz_idx = s.col_ptr[d->J];
        s.nnz_val = s.val_ptr[d->J];
        CYC_REQUIRE(s.col_ptr[0] == 0 && s.val_ptr[0] == 0, CYC_ERR_ARGUMENT, "offsets must start at 0");
        CYC_REQUIRE(s.nnz_idx == 0 || d->col_idx, CYC_ERR_ARGUMENT, "missing col_idx");
        CYC_REQUIRE(s.nnz_val == 0 || d->col_val, CYC_ERR_ARGUMENT, "missing col_val");
        for (int j = 0; j < d->J; ++j) {
            const int f = s.fmt[j];
            CYC_REQUIRE(f >= CYC_DENSE && f <= CYC_INTERCEPT, CYC_ERR_ARGUMENT, "bad column format");
            const long long ni = s.col_ptr[j + 1] - s.col_ptr[j];
            const long long nv = s.val_ptr[j + 1] - s.val_ptr[j];
            CYC_REQUIRE(ni >= 0 && nv >= 0, CYC_ERR_ARGUMENT, "offsets must not decrease");
            if (f == CYC_DENSE) CYC_REQUIRE(nv == d->K && ni == 0, CYC_ERR_ARGUMENT, "dense column needs K values");
            if (f == CYC_SPARSE) CYC_REQUIRE(nv == ni, CYC_ERR_ARGUMENT, "sparse column values/indices mismatch");
            if (f == CYC_INDICATOR) CYC_REQUIRE(nv == 0, CYC_ERR_ARGUMENT, "indicator column holds no values");
            if (f == CYC_INTERCEPT) CYC_REQUIRE(nv == 0 && ni == 0, CYC_ERR_ARGUMENT, "intercept column holds nothing");
            if (f == CYC_SPARSE || f == CYC_INDICATOR) {
                const int* r = d->col_idx + s.col_ptr[j];
                for (long long e = 0; e < ni; ++e) {
                    CYC_REQUIRE(r[e] >= 0 && r[e] < d->K, CYC_ERR_ARGUMENT, "row index out of range");
                    CYC_REQUIRE(e == 0 || r[e] > r[e - 1], CYC_ERR_ARGUMENT, "row ids must ascend within a column");
                }
            }
        }
        if (d->has_offset) CYC_REQUIRE(s.fmt[0] == CYC_DENSE, CYC_ERR_ARGUMENT, "offset column must be dense");
        s.y.assign(d->y, d->y + d->K);
        if (d->time) s.time.assign(d->time, d->time + d->K);
        s.h_idx.assign(d->col_idx ? d->col_idx : (const int*)nullptr,
                       d->col_idx ? d->col_idx + s.nnz_idx : (const int*)nullptr);

        // strata renumbered by runs (src/RcppModelData.cpp:878-900)
        s.strat.resize(d->K);
        if (d->pid) {
            int cur = 0, last = d->pid[0];
            for (int k = 0; k < d->K; ++k) {
                if (d->pid[k] != last) { ++cur; last = d->pid[k]; }
                s.strat[k] = cur;
            }
            s.S = cur + 1;
        } else {
            for (int k = 0; k < d->K; ++k) s.strat[k] = k;
            s.S = d->K;
        }
        s.strat_ptr.assign(s.S + 1, 0);
        for (int k = 0; k < d->K; ++k) s.strat_ptr[s.strat[k] + 1]++;
        for (int i = 0; i < s.S; ++i) s.strat_ptr[i + 1] += s.strat_ptr[i];

        upload(s.d_fmt, s.fmt.data(), s.fmt.size());
        upload(s.d_col_ptr, s.col_ptr.data(), s.col_ptr.size());
        upload(s.d_val_ptr, s.val_ptr.data(), s.val_ptr.size());
        upload(s.d_idx, d->col_idx, (size_t)s.nnz_idx);
        upload(s.d_val, d->col_val, (size_t)s.nnz_val);
        upload(s.d_y, d->y, (size_t)d->K);
        if (d->time) upload(s.d_time, d->time, (size_t)d->K);
        upload(s.d_strat, s.strat.data(), s.strat.size());
        upload(s.d_strat_ptr, s.strat_ptr.data(), s.strat_ptr.size());
        CYC_CHECK_CUDA(cudaStreamSynchronize(s.stream));   // usable from every stream
        *out = guard.release();
    });
}

extern "C" int cyc_dataset_destroy(cyc_dataset* ds) {
    return guarded([&] {
        if (!ds) return;
        cudaSetDevice(ds->ds.device);
        delete ds;
    });
}

extern "C" int cyc_dataset_info(const cyc_dataset* ds, int* K, int* J, long long* nnz, size_t* bytes) {
    return guarded([&] {
        CYC_REQUIRE(ds, CYC_ERR_ARGUMENT, "null dataset");
        if (K) *K = ds->ds.K;
        if (J) *J = ds->ds.J;
        if (nnz) *nnz = ds->ds.nnz_idx;
        if (bytes) *bytes = ds->ds.device_bytes();
    });
}
