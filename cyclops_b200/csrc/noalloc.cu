// noalloc.cu -- gradient/Hessian of one column without any device allocation.
//
// Who needs this: callers that own all device memory themselves -- a host
// application that hands the GPU's memory to its own pool or caching
// allocator up front, or a loop where an allocation's implicit device
// synchronisation is not acceptable -- cannot let this library call
// cudaMalloc.  The ordinary engine keeps per-engine scratch buffers that it
// allocates when the engine is created; this entry point instead uses one
// fixed scratch area compiled into the library, so a call allocates nothing.
//
// The scratch (per-block partial sums plus one completion counter) is a
// file-scope __device__ array of kNoAllocMaxBlocks entries (64 KiB); every
// GPU that loads this library holds it until the process exits.  Host code
// cannot use the array's name as a device address, so the first call on each
// device looks the address up with cudaGetSymbolAddress (with that device
// current) and caches it; make that first call before any stream capture.
// All calls share the one scratch area: calls that overlap on the GPU (other
// streams, other host threads) race and must be serialised by the caller.
#include <mutex>

#include "internal.cuh"

namespace cyc {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocItems = 4;
constexpr int kNoAllocMaxBlocks = 4096;          // 4096 x 16 B partials = 64 KiB
constexpr long long kNoAllocMaxEntries = (long long)kNoAllocMaxBlocks * kNoAllocThreads * kNoAllocItems;

// layout of the scratch bytes: per-block partials, then the completion counter
struct NoAllocScratch {
    double2 partial[kNoAllocMaxBlocks];
    unsigned ticket;
};
constexpr size_t kNoAllocScratchBytes = (sizeof(NoAllocScratch) + 255) / 256 * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
NoAllocScratch* g_noalloc_addr[kMaxDevices] = {};

// The variant of the engine's independent-rows gradient kernel
// (computeGradientAndHessianImpl, ModelSpecifics.hpp:1022-1038) whose
// partials and ticket live in the fixed scratch area and whose XjY arrives
// by value.
template <int MODEL, bool IND>
__global__ void k_gh_independent_noalloc(ColView c, const double* __restrict__ exb, const double* __restrict__ denom,
                                         const double* __restrict__ w, double xjy, NoAllocScratch* scratch,
                                         double* out) {
    double g = 0.0, h = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.n;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = c.row(e);
        const double x = c.x(e);
        const double ex = exb[k];
        const double n1 = ex * x;
        const double wk = w ? w[k] : 1.0;
        if (MODEL == CYC_LR) {
            const double d = denom[k];
            const double gi = n1 / d;
            g += wk * gi;
            h += wk * (IND ? gi * (1.0 - gi) : (n1 * x / d - gi * gi));
        } else {
            g += wk * n1;
            h += wk * (IND ? n1 : n1 * x);
        }
    }
    grid_sum2_finalize(g, h, scratch->partial, &scratch->ticket, [&](double G, double H) {
        out[0] = G - xjy;
        out[1] = H;
    });
}

NoAllocScratch* scratch_for_current_device() {
    int dev = 0;
    CYC_CHECK_CUDA(cudaGetDevice(&dev));
    CYC_REQUIRE(dev >= 0 && dev < kMaxDevices, CYC_ERR_UNSUPPORTED, "device ordinal beyond the no-alloc table");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        CYC_CHECK_CUDA(cudaGetSymbolAddress((void**)&p, g_noalloc_scratch));
        CYC_REQUIRE(p != nullptr, CYC_ERR_CUDA, "cudaGetSymbolAddress returned no address");
        g_noalloc_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    return g_noalloc_addr[dev];
}

}  // namespace
}  // namespace cyc

using namespace cyc;

extern "C" int cyc_gradient_hessian_noalloc(int model, int format, long long n, const int* rows,
                                            const double* values, const double* exb, const double* denom,
                                            const double* weights, double xjy, double* out, void* stream) {
    return guarded([&] {
        CYC_REQUIRE(model == CYC_LR || model == CYC_PR, CYC_ERR_UNSUPPORTED,
                    "cyc_gradient_hessian_noalloc covers lr and pr");
        CYC_REQUIRE(format >= CYC_DENSE && format <= CYC_INTERCEPT, CYC_ERR_ARGUMENT, "bad column format");
        CYC_REQUIRE(n >= 0, CYC_ERR_ARGUMENT, "negative entry count");
        CYC_REQUIRE(n <= kNoAllocMaxEntries, CYC_ERR_ARGUMENT,
                    "column has more entries than the fixed scratch covers (4,194,304)");
        CYC_REQUIRE(out && exb, CYC_ERR_ARGUMENT, "null output or exp(xbeta)");
        CYC_REQUIRE(model != CYC_LR || denom, CYC_ERR_ARGUMENT, "logistic needs the denominators");
        CYC_REQUIRE((format != CYC_SPARSE && format != CYC_INDICATOR) || n == 0 || rows, CYC_ERR_ARGUMENT,
                    "null row ids");
        CYC_REQUIRE((format != CYC_SPARSE && format != CYC_DENSE) || n == 0 || values, CYC_ERR_ARGUMENT,
                    "null values");
        NoAllocScratch* scratch = scratch_for_current_device();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (n == 0) {                                    // ModelSpecifics.hpp:720-723
            CYC_CHECK_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(double), s));
            return;
        }
        // the completion counter must start at zero; a previous call that
        // failed part-way may have left it otherwise
        CYC_CHECK_CUDA(cudaMemsetAsync(&scratch->ticket, 0, sizeof(unsigned), s));
        ColView c;
        c.fmt = format;
        c.n = n;
        c.idx = rows;
        c.val = values;
        const long long per = (long long)kNoAllocThreads * kNoAllocItems;
        const int blocks = (int)((n + per - 1) / per);
        const bool ind = c.indicator();
        if (model == CYC_LR) {
            if (ind) launch(k_gh_independent_noalloc<CYC_LR, true>, blocks, kNoAllocThreads, 0, s, c, exb, denom, weights, xjy, scratch, out);
            else launch(k_gh_independent_noalloc<CYC_LR, false>, blocks, kNoAllocThreads, 0, s, c, exb, denom, weights, xjy, scratch, out);
        } else {
            if (ind) launch(k_gh_independent_noalloc<CYC_PR, true>, blocks, kNoAllocThreads, 0, s, c, exb, denom, weights, xjy, scratch, out);
            else launch(k_gh_independent_noalloc<CYC_PR, false>, blocks, kNoAllocThreads, 0, s, c, exb, denom, weights, xjy, scratch, out);
        }
    });
}
