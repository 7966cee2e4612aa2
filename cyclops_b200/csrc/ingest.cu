// Device ingest of a long covariate table: the covariate half of
// convertToCyclopsData (R/NewDataConversion.R:131-176: rows without an
// outcome dropped, the rest ordered like their outcome rows within each
// covariate) and of ModelData::loadMultipleX (src/cyclops/ModelData.cpp:
// 148-243: one column per covariateId run, INDICATOR unless some value is
// neither 0 nor 1, zero values not stored, a repeated (row, covariate) an
// error), on the GPU.
//
// The outcome table arrives already in the reference's row order (sorted on
// the host; K rows), so a covariate entry's place in that order is its
// outcome position, and the covariate order of every model (lr/pr: covariate,
// row; clr/cpr: covariate, stratum, row; cox: covariate, stratum, time
// descending, y, row) is (covariate, outcome position).  The pipeline:
//   1. outcome rowIds sorted (stable radix sort, positions as values): a
//      covariate row's position is the last outcome row with its rowId
//      (the reference's rowId map keeps the last assignment);
//   2. entries without an outcome dropped (stream compaction);
//   3. two stable radix sorts -- by position, then by covariateId -- give the
//      (covariate, position) order;
//   4. flags per entry (a column starts, a repeated row, a value stored, a
//      value outside {0, 1}), segment ids by a scan, a column's format by an
//      OR over its entries, and the stored entries' places by exclusive scans;
//   5. one scatter writes row ids and values in column order.
// Every step is a CUB primitive or a one-pass kernel over the entries: the
// work is sorting-bound, a few passes over 24 bytes an entry.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <cstdint>
#include <string>
#include <vector>

#include "internal.cuh"

struct cyc_ingest {
    int device = 0;
    int J = 0;                      // covariate columns
    long long n_idx = 0, n_val = 0;
    cyc::DevBuf<int> fmt, col_idx;
    cyc::DevBuf<long long> col_ptr, val_ptr, labels;
    cyc::DevBuf<double> col_val;
};

namespace cyc {
namespace {

__global__ void k_iota(long long n, int* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (int)i;
}

// position of each covariate row's outcome: the last of the outcome rows
// with its rowId (okey sorted, opos their positions, ascending within a
// run of equal keys), -1 when there is none
__global__ void k_outcome_position(long long n, const long long* __restrict__ row, int K,
                                   const long long* __restrict__ okey, const int* __restrict__ opos,
                                   int* __restrict__ pos, unsigned char* __restrict__ keep) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = row[i];
        int lo = 0, hi = K;                 // first key > r
        while (lo < hi) {
            const int mid = (int)(((unsigned)lo + (unsigned)hi) >> 1);
            if (okey[mid] <= r) lo = mid + 1;
            else hi = mid;
        }
        const bool found = lo > 0 && okey[lo - 1] == r;
        pos[i] = found ? opos[lo - 1] : -1;
        keep[i] = found ? 1 : 0;
    }
}

template <class A, class B>
__global__ void k_gather(long long n, const int* __restrict__ perm, const A* __restrict__ src, B* __restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (B)src[perm[i]];
}

// perm2[i] = perm1[perm0[i]]: composes the compaction and sort permutations
__global__ void k_compose(long long n, const int* __restrict__ outer, const int* __restrict__ inner, int* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = inner[outer[i]];
}

// per entry of the (covariate, position) order: a column starts here; the
// entry repeats the previous one's row (first such index into *dup); its
// value is stored (nonzero, or no values at all); its value is outside {0, 1}
__global__ void k_entry_flags(long long n, const long long* __restrict__ cid, const int* __restrict__ pos,
                              const double* __restrict__ val, int* __restrict__ start,
                              unsigned char* __restrict__ nz, unsigned char* __restrict__ not01,
                              unsigned long long* __restrict__ dup) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const bool s = (i == 0) || cid[i] != cid[i - 1];
        start[i] = s ? 1 : 0;
        if (!s && pos[i] == pos[i - 1]) atomicMin(dup, (unsigned long long)i);
        if (val) {
            const double v = val[i];
            nz[i] = (v != 0.0) ? 1 : 0;
            not01[i] = !(v == 0.0 || v == 1.0) ? 1 : 0;
        } else {
            nz[i] = 1;
            not01[i] = 0;
        }
    }
}

// seg = inclusive scan of the start flags, so entry i is in column seg[i] - 1
__global__ void k_segment_marks(long long n, const int* __restrict__ seg, const int* __restrict__ start,
                                const unsigned char* __restrict__ not01, int* __restrict__ seg_start,
                                int* __restrict__ sparse) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = seg[i] - 1;
        if (start[i]) seg_start[s] = (int)i;
        if (not01[i]) sparse[s] = 1;        // benign race: every writer stores 1
    }
}

__global__ void k_value_flags(long long n, const int* __restrict__ seg, const int* __restrict__ sparse,
                              const unsigned char* __restrict__ nz, int* __restrict__ keep_idx,
                              int* __restrict__ keep_val) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        keep_idx[i] = nz[i];
        keep_val[i] = (nz[i] && sparse[seg[i] - 1]) ? 1 : 0;
    }
}

// the stored entries in column order, and each column's format, pointers
// and label
__global__ void k_scatter(long long n, const int* __restrict__ pos, const double* __restrict__ val,
                          const int* __restrict__ keep_idx, const int* __restrict__ keep_val,
                          const int* __restrict__ at_idx, const int* __restrict__ at_val, int* __restrict__ col_idx,
                          double* __restrict__ col_val) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (keep_idx[i]) col_idx[at_idx[i]] = pos[i];
        if (keep_val[i]) col_val[at_val[i]] = val[i];
    }
}

__global__ void k_columns(int J, long long n, const int* __restrict__ seg_start, const int* __restrict__ sparse,
                          const int* __restrict__ at_idx, const int* __restrict__ at_val, long long n_idx,
                          long long n_val, const long long* __restrict__ cid, int* __restrict__ fmt,
                          long long* __restrict__ col_ptr, long long* __restrict__ val_ptr,
                          long long* __restrict__ labels) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= J; s += gridDim.x * blockDim.x) {
        if (s == J) {
            col_ptr[J] = n_idx;
            val_ptr[J] = n_val;
            continue;
        }
        const int i = seg_start[s];
        fmt[s] = sparse[s] ? CYC_SPARSE : CYC_INDICATOR;
        col_ptr[s] = at_idx[i];
        val_ptr[s] = at_val[i];
        labels[s] = cid[i];
    }
}

inline int blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

// temporary storage for one CUB call: query, allocate, run
template <class F>
void cub_call(DevBuf<unsigned char>& tmp, F&& f) {
    size_t bytes = 0;
    CYC_CHECK_CUDA(f(nullptr, bytes));
    if (bytes > tmp.n) tmp.alloc(bytes);
    CYC_CHECK_CUDA(f(tmp.get(), bytes));
}

}  // namespace
}  // namespace cyc

using namespace cyc;

extern "C" int cyc_ingest_covariates(int device, long long n, const long long* covariate_id, const long long* row_id,
                                     const double* value, int K, const long long* outcome_row_id, cyc_ingest** out) {
    return guarded([&] {
        NvtxRange range("cyc_ingest_covariates");
        CYC_REQUIRE(out && K >= 0 && n >= 0 && (n == 0 || (covariate_id && row_id)) && (K == 0 || outcome_row_id),
                    CYC_ERR_ARGUMENT, "null argument");
        CYC_REQUIRE(n < (1ll << 31) - 1 && K < (1 << 30), CYC_ERR_ARGUMENT, "at most 2^31 - 2 entries");
        *out = nullptr;
        CYC_CHECK_CUDA(cudaSetDevice(device));
        prepare_pool(device);
        OwnedStream own;
        CYC_CHECK_CUDA(cudaStreamCreateWithFlags(&own.s, cudaStreamNonBlocking));
        const cudaStream_t st = own.s;
        StreamScope scope(st);
        auto h = std::make_unique<cyc_ingest>();
        h->device = device;
        DevBuf<unsigned char> tmp;
        // 1. outcome rowIds, sorted with their positions
        DevBuf<long long> orow, okey;
        DevBuf<int> opos0, opos;
        orow.alloc(K); okey.alloc(K); opos0.alloc(K); opos.alloc(K);
        if (K) {
            CYC_CHECK_CUDA(cudaMemcpyAsync(orow.get(), outcome_row_id, K * sizeof(long long), cudaMemcpyHostToDevice, st));
            launch(k_iota, blocks(K), 256, 0, st, (long long)K, opos0.get());
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceRadixSort::SortPairs(t, b, orow.get(), okey.get(), opos0.get(), opos.get(), K, 0, 64, st);
            });
        }
        // 2. positions of the covariate rows; entries without an outcome dropped
        DevBuf<long long> cid, row;
        DevBuf<double> val;
        DevBuf<int> pos, idx0, kept, n_sel;
        DevBuf<unsigned char> keep;
        cid.alloc(n); row.alloc(n); pos.alloc(n); keep.alloc(n); idx0.alloc(n); kept.alloc(n); n_sel.alloc(1);
        if (value) val.alloc(n);
        int nk = 0;
        if (n) {
            CYC_CHECK_CUDA(cudaMemcpyAsync(cid.get(), covariate_id, n * sizeof(long long), cudaMemcpyHostToDevice, st));
            CYC_CHECK_CUDA(cudaMemcpyAsync(row.get(), row_id, n * sizeof(long long), cudaMemcpyHostToDevice, st));
            if (value) CYC_CHECK_CUDA(cudaMemcpyAsync(val.get(), value, n * sizeof(double), cudaMemcpyHostToDevice, st));
            launch(k_outcome_position, blocks(n), 256, 0, st, n, row.get(), K, okey.get(), opos.get(), pos.get(), keep.get());
            launch(k_iota, blocks(n), 256, 0, st, n, idx0.get());
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceSelect::Flagged(t, b, idx0.get(), keep.get(), kept.get(), n_sel.get(), (int)n, st);
            });
            CYC_CHECK_CUDA(cudaMemcpyAsync(&nk, n_sel.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
            CYC_CHECK_CUDA(cudaStreamSynchronize(st));
        }
        // 3. (covariate, position) order: stable sorts by position, then covariate
        DevBuf<int> kpos, spos, sidx0, sidx1, perm;
        DevBuf<long long> kcid, scid;
        kpos.alloc(nk); spos.alloc(nk); sidx0.alloc(nk); sidx1.alloc(nk); perm.alloc(nk); kcid.alloc(nk); scid.alloc(nk);
        if (nk) {
            launch(k_gather<int, int>, blocks(nk), 256, 0, st, (long long)nk, kept.get(), pos.get(), kpos.get());
            launch(k_iota, blocks(nk), 256, 0, st, (long long)nk, sidx0.get());
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceRadixSort::SortPairs(t, b, kpos.get(), spos.get(), sidx0.get(), sidx1.get(), nk, 0, 31, st);
            });
            // covariate ids in that order, then sorted with the order as values
            launch(k_compose, blocks(nk), 256, 0, st, (long long)nk, sidx1.get(), kept.get(), sidx0.get());
            launch(k_gather<long long, long long>, blocks(nk), 256, 0, st, (long long)nk, sidx0.get(), cid.get(), kcid.get());
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceRadixSort::SortPairs(t, b, kcid.get(), scid.get(), sidx0.get(), perm.get(), nk, 0, 64, st);
            });
        }
        // perm[i]: the input entry at place i of the order
        DevBuf<int> opos_s, start, seg, seg_start, sparse, keep_idx, keep_val, at_idx, at_val;
        DevBuf<double> sval;
        DevBuf<unsigned char> nz, not01;
        DevBuf<unsigned long long> dup;
        opos_s.alloc(nk); start.alloc(nk); seg.alloc(nk); nz.alloc(nk); not01.alloc(nk); dup.alloc(1);
        keep_idx.alloc(nk); keep_val.alloc(nk); at_idx.alloc(nk); at_val.alloc(nk);
        if (value) sval.alloc(nk);
        int J = 0;
        long long n_idx = 0, n_val = 0;
        if (nk) {
            launch(k_gather<int, int>, blocks(nk), 256, 0, st, (long long)nk, perm.get(), pos.get(), opos_s.get());
            if (value) launch(k_gather<double, double>, blocks(nk), 256, 0, st, (long long)nk, perm.get(), val.get(), sval.get());
            const unsigned long long none = ~0ull;
            CYC_CHECK_CUDA(cudaMemcpyAsync(dup.get(), &none, sizeof(none), cudaMemcpyHostToDevice, st));
            // 4. flags, columns, formats
            launch(k_entry_flags, blocks(nk), 256, 0, st, (long long)nk, scid.get(), opos_s.get(),
                   value ? sval.get() : nullptr, start.get(), nz.get(), not01.get(), dup.get());
            unsigned long long first_dup = none;
            CYC_CHECK_CUDA(cudaMemcpyAsync(&first_dup, dup.get(), sizeof(first_dup), cudaMemcpyDeviceToHost, st));
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceScan::InclusiveSum(t, b, start.get(), seg.get(), nk, st);
            });
            CYC_CHECK_CUDA(cudaMemcpyAsync(&J, seg.get() + nk - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            CYC_CHECK_CUDA(cudaStreamSynchronize(st));
            if (first_dup != none) {
                // the reference's message names the rowId and covariateId of the repeat
                int at = 0;
                CYC_CHECK_CUDA(cudaMemcpyAsync(&at, perm.get() + first_dup, sizeof(int), cudaMemcpyDeviceToHost, st));
                CYC_CHECK_CUDA(cudaStreamSynchronize(st));
                throw Error{CYC_ERR_ARGUMENT, "Repeated row-column entry at " + std::to_string(row_id[at]) + " - " +
                                                  std::to_string(covariate_id[at])};
            }
            seg_start.alloc(J);
            sparse.alloc(J);
            CYC_CHECK_CUDA(cudaMemsetAsync(sparse.get(), 0, J * sizeof(int), st));
            launch(k_segment_marks, blocks(nk), 256, 0, st, (long long)nk, seg.get(), start.get(), not01.get(),
                   seg_start.get(), sparse.get());
            launch(k_value_flags, blocks(nk), 256, 0, st, (long long)nk, seg.get(), sparse.get(), nz.get(),
                   keep_idx.get(), keep_val.get());
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceScan::ExclusiveSum(t, b, keep_idx.get(), at_idx.get(), nk, st);
            });
            cub_call(tmp, [&](void* t, size_t& b) {
                return cub::DeviceScan::ExclusiveSum(t, b, keep_val.get(), at_val.get(), nk, st);
            });
            int last[4];
            CYC_CHECK_CUDA(cudaMemcpyAsync(&last[0], at_idx.get() + nk - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            CYC_CHECK_CUDA(cudaMemcpyAsync(&last[1], keep_idx.get() + nk - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            CYC_CHECK_CUDA(cudaMemcpyAsync(&last[2], at_val.get() + nk - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            CYC_CHECK_CUDA(cudaMemcpyAsync(&last[3], keep_val.get() + nk - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            CYC_CHECK_CUDA(cudaStreamSynchronize(st));
            n_idx = (long long)last[0] + last[1];
            n_val = (long long)last[2] + last[3];
        }
        // 5. the column store (outliving this call's stream: plain allocations)
        h->J = J;
        h->n_idx = n_idx;
        h->n_val = n_val;
        {
            StreamScope unordered(nullptr);
            h->fmt.alloc(J);
            h->col_ptr.alloc(J + 1);
            h->val_ptr.alloc(J + 1);
            h->labels.alloc(J);
            h->col_idx.alloc(n_idx);
            h->col_val.alloc(n_val);
        }
        if (nk) {
            launch(k_scatter, blocks(nk), 256, 0, st, (long long)nk, opos_s.get(), value ? sval.get() : nullptr,
                   keep_idx.get(), keep_val.get(), at_idx.get(), at_val.get(), h->col_idx.get(), h->col_val.get());
            launch(k_columns, blocks(J + 1), 256, 0, st, J, (long long)nk, seg_start.get(), sparse.get(), at_idx.get(),
                   at_val.get(), n_idx, n_val, scid.get(), h->fmt.get(), h->col_ptr.get(), h->val_ptr.get(),
                   h->labels.get());
        } else {
            const long long zero[2] = {0, 0};
            CYC_CHECK_CUDA(cudaMemcpyAsync(h->col_ptr.get(), zero, sizeof(long long), cudaMemcpyHostToDevice, st));
            CYC_CHECK_CUDA(cudaMemcpyAsync(h->val_ptr.get(), zero + 1, sizeof(long long), cudaMemcpyHostToDevice, st));
        }
        CYC_CHECK_LAUNCH();
        CYC_CHECK_CUDA(cudaStreamSynchronize(st));
        *out = h.release();
    });
}

extern "C" int cyc_ingest_sizes(const cyc_ingest* h, int* n_columns, long long* n_idx, long long* n_val) {
    return guarded([&] {
        CYC_REQUIRE(h && n_columns && n_idx && n_val, CYC_ERR_ARGUMENT, "null argument");
        *n_columns = h->J;
        *n_idx = h->n_idx;
        *n_val = h->n_val;
    });
}

extern "C" int cyc_ingest_copy(const cyc_ingest* h, int* col_format, long long* col_ptr, int* col_idx,
                               long long* val_ptr, double* col_val, long long* labels) {
    return guarded([&] {
        CYC_REQUIRE(h && col_format && col_ptr && val_ptr && labels && (h->n_idx == 0 || col_idx) &&
                        (h->n_val == 0 || col_val),
                    CYC_ERR_ARGUMENT, "null argument");
        CYC_CHECK_CUDA(cudaSetDevice(h->device));
        const int J = h->J;
        CYC_CHECK_CUDA(cudaMemcpy(col_format, h->fmt.get(), J * sizeof(int), cudaMemcpyDeviceToHost));
        CYC_CHECK_CUDA(cudaMemcpy(col_ptr, h->col_ptr.get(), (J + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
        CYC_CHECK_CUDA(cudaMemcpy(val_ptr, h->val_ptr.get(), (J + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
        CYC_CHECK_CUDA(cudaMemcpy(labels, h->labels.get(), J * sizeof(long long), cudaMemcpyDeviceToHost));
        if (h->n_idx)
            CYC_CHECK_CUDA(cudaMemcpy(col_idx, h->col_idx.get(), h->n_idx * sizeof(int), cudaMemcpyDeviceToHost));
        if (h->n_val)
            CYC_CHECK_CUDA(cudaMemcpy(col_val, h->col_val.get(), h->n_val * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

extern "C" void cyc_ingest_free(cyc_ingest* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    delete h;
}
