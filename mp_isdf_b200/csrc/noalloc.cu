// Pair-space error reduction that allocates no memory.
//
// Some callers cannot allocate device memory on the call path: code running
// under a host-side memory budget that forbids cudaMalloc after start-up,
// callers that hand every byte of device memory to their own pool or arena,
// and code that must not synchronise the device the way cudaFree does.  For
// them this file provides a variant of isdf_pair_error_terms whose only
// scratch is a file-scope device array of fixed size (every GPU that loads the
// library keeps it for the life of the process).
//
// Limits and behaviour:
//   * k (anchors) <= kNoAllocMaxAnchors; larger k is rejected with
//     ISDF_ERR_INVALID.  Any number of grid points.
//   * All calls share the one array.  Calls whose GPU work overlaps (two
//     streams, or two host threads) race on it; serialise them.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     that first call before any stream capture.  The address is kept for the
//     life of the process: after cudaDeviceReset on a device the library's
//     module is loaded again and the kept address is stale, so do not call
//     this entry point on a device after resetting it.
//   * Each call copies the two sums to host memory and waits for its stream
//     to finish before returning.
#include "../../include/isdf_b200.h"
#include "isdf_internal.h"
#include "isdf_reduce.cuh"

#include <cmath>
#include <mutex>

namespace isdf {
namespace {

constexpr int kNoAllocMaxAnchors = 64;
constexpr int kNoAllocBlocks = 1024;
constexpr int kNoAllocThreads = 256;

// [0, 2*kNoAllocBlocks): per-block partial sums; [2*kNoAllocBlocks, +2): totals.
__device__ __align__(256) double g_pair_error_scratch[2 * kNoAllocBlocks + 2];

// err_g = |w| (q^2 - 2 x.h + x^T M x), exact_g = |w| q^2; per-block partials.
__global__ void __launch_bounds__(kNoAllocThreads)
pair_error_partials_kernel(int64_t n, int k, const double* __restrict__ q,
                           const double* __restrict__ H, const double* __restrict__ X,
                           const double* __restrict__ M, const double* __restrict__ w,
                           double* __restrict__ scratch) {
    __shared__ double Ms[kNoAllocMaxAnchors * kNoAllocMaxAnchors];
    __shared__ double red[kNoAllocThreads / 32];
    for (int i = threadIdx.x; i < k * k; i += blockDim.x) Ms[i] = M[i];
    __syncthreads();
    double e = 0, ex = 0;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < n;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double* h = H + g * k;
        const double* x = X + g * k;
        double xh = 0, xmx = 0;
        for (int a = 0; a < k; ++a) {
            xh += x[a] * h[a];
            double t = 0;
            for (int b = 0; b < k; ++b) t += Ms[a * k + b] * x[b];
            xmx += x[a] * t;
        }
        const double aw = fabs(w[g]);
        e += aw * (q[g] * q[g] - 2.0 * xh + xmx);
        ex += aw * q[g] * q[g];
    }
    e = block_sum<kNoAllocThreads>(e, red);
    ex = block_sum<kNoAllocThreads>(ex, red);
    if (threadIdx.x == 0) {
        scratch[2 * blockIdx.x] = e;
        scratch[2 * blockIdx.x + 1] = ex;
    }
}

// Fixed-order sum of the partials (deterministic), totals at the end of scratch.
__global__ void __launch_bounds__(kNoAllocThreads)
pair_error_total_kernel(int nblocks, double* __restrict__ scratch) {
    __shared__ double red[kNoAllocThreads / 32];
    double e = 0, ex = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        e += scratch[2 * b];
        ex += scratch[2 * b + 1];
    }
    e = block_sum<kNoAllocThreads>(e, red);
    ex = block_sum<kNoAllocThreads>(ex, red);
    if (threadIdx.x == 0) {
        scratch[2 * kNoAllocBlocks] = e;
        scratch[2 * kNoAllocBlocks + 1] = ex;
    }
}

std::mutex g_addr_mu;
double* g_addr[64] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device with that device current).
double* scratch_address() {
    int dev = 0;
    ISDF_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        ISDF_CUDA(cudaGetSymbolAddress(&p, g_pair_error_scratch));
        g_addr[dev] = static_cast<double*>(p);
    }
    return g_addr[dev];
}

}  // namespace
}  // namespace isdf

extern "C" int isdf_pair_error_terms_noalloc(int64_t n, int64_t k, const double* q, const double* H,
                                             const double* X, const double* M, const double* w,
                                             double* out, void* stream) {
    try {
        if (n < 0 || k < 0 || !out) isdf::fail(isdf::kInvalid, "invalid pair error terms");
        if (k > isdf::kNoAllocMaxAnchors)
            isdf::fail(isdf::kInvalid, "isdf_pair_error_terms_noalloc supports at most 64 anchors");
        if (n > 0 && (!q || !w || (k > 0 && (!H || !X || !M))))
            isdf::fail(isdf::kInvalid, "null pair error term array");
        double acc[2] = {0, 0};
        if (n > 0) {
            cudaStream_t s = static_cast<cudaStream_t>(stream);
            double* scratch = isdf::scratch_address();
            const int64_t want = (n + isdf::kNoAllocThreads - 1) / isdf::kNoAllocThreads;
            const int nb = static_cast<int>(std::min<int64_t>(want, isdf::kNoAllocBlocks));
            isdf::pair_error_partials_kernel<<<nb, isdf::kNoAllocThreads, 0, s>>>(
                n, static_cast<int>(k), q, H, X, M, w, scratch);
            ISDF_LAUNCH_CHECK();
            isdf::pair_error_total_kernel<<<1, isdf::kNoAllocThreads, 0, s>>>(nb, scratch);
            ISDF_LAUNCH_CHECK();
            ISDF_CUDA(cudaMemcpyAsync(acc, scratch + 2 * isdf::kNoAllocBlocks, 2 * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
            ISDF_CUDA(cudaStreamSynchronize(s));
        }
        const double a = std::sqrt(std::max(acc[0], 0.0));
        out[0] = a;
        out[1] = acc[1] ? a / std::sqrt(acc[1]) : (a == 0 ? 0.0 : INFINITY);
        return ISDF_OK;
    } catch (const isdf::Error& e) {
        isdf::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        isdf::set_last_error(e.what());
        return ISDF_ERR_RUNTIME;
    }
}
