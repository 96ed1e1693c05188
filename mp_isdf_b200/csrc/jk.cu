// ISDF Coulomb (J) and exchange (K) matrices of a density matrix
// (evaluate_isdf_jk, python/isdf.py:130-151, mikovtun/mp_isdf):
//   (mu nu|lam sig) ~ sum_pq X[p,mu] X[p,nu] Z[p,q] X[q,lam] X[q,sig],
//   P = X D X^T (k x k),  d_p = P_pp,
//   J = X^T diag(Z d) X,  K = X^T (Z o P) X,
// both returned symmetrised, (A + A^T) / 2.  X is the anchors' AO values
// (k x nao), Z the anchor-weighted Coulomb metric (k x k), D the AO density
// (nao x nao).  Every contraction is an FP64 tensor-core GEMM (gemm_f64); the
// O(k^2) steps are small elementwise kernels.
#include "isdf_internal.h"

#include <cmath>

namespace isdf {
namespace {

unsigned blocks(int64_t n) { return static_cast<unsigned>((n + 255) / 256); }

__global__ void transpose_kernel(const double* __restrict__ a, int64_t rows, int64_t cols, double* __restrict__ at) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const int64_t r = i / cols, c = i % cols;
    at[c * rows + r] = a[i];
}

// u = Z diag(P) (k), then Xu[p][mu] = u_p X[p][mu] and W = Z o P
__global__ void jk_anchor_kernel(const double* __restrict__ Z, const double* __restrict__ P, int k,
                                 double* __restrict__ u, double* __restrict__ W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) {
        double s = 0.0;
        for (int q = 0; q < k; ++q) s += Z[i * k + q] * P[q * k + q];
        u[i] = s;
    }
    if (i < k * k) W[i] = Z[i] * P[i];
}

__global__ void scale_rows_kernel(const double* __restrict__ X, const double* __restrict__ u, int k, int64_t nao,
                                  double* __restrict__ Y) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= k * nao) return;
    Y[i] = u[i / nao] * X[i];
}

// A = (A + A^T) / 2 in place (n x n)
__global__ void symmetrise_kernel(double* A, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n * n) return;
    const int64_t r = i / n, c = i % n;
    if (c <= r) return;
    const double v = 0.5 * (A[r * n + c] + A[c * n + r]);
    A[r * n + c] = v;
    A[c * n + r] = v;
}

}  // namespace

void isdf_jk_device(int64_t nao, int64_t k, const double* X, const double* Z, const double* D, double* J,
                    double* K, cudaStream_t s) {
    if (nao == 0) return;
    if (k == 0) {
        if (J) ISDF_CUDA(cudaMemsetAsync(J, 0, nao * nao * sizeof(double), s));
        if (K) ISDF_CUDA(cudaMemsetAsync(K, 0, nao * nao * sizeof(double), s));
        return;
    }
    DeviceBuffer<double> XT(static_cast<size_t>(nao * k), s), XD(static_cast<size_t>(k * nao), s),
        P(static_cast<size_t>(k * k), s), u(k, s), W(static_cast<size_t>(k * k), s),
        Y(static_cast<size_t>(k * nao), s);
    transpose_kernel<<<blocks(k * nao), 256, 0, s>>>(X, k, nao, XT.get());
    ISDF_LAUNCH_CHECK();
    // P = X D X^T
    gemm_f64(k, nao, nao, X, nao, 0, D, nao, 0, XD.get(), nao, 0, 1, false, s);
    gemm_f64(k, k, nao, XD.get(), nao, 0, XT.get(), k, 0, P.get(), k, 0, 1, false, s);
    jk_anchor_kernel<<<blocks(k * k), 256, 0, s>>>(Z, P.get(), static_cast<int>(k), u.get(), W.get());
    ISDF_LAUNCH_CHECK();
    if (J) {
        // J = X^T (u o X)
        scale_rows_kernel<<<blocks(k * nao), 256, 0, s>>>(X, u.get(), static_cast<int>(k), nao, Y.get());
        ISDF_LAUNCH_CHECK();
        gemm_f64(nao, nao, k, XT.get(), k, 0, Y.get(), nao, 0, J, nao, 0, 1, false, s);
        symmetrise_kernel<<<blocks(nao * nao), 256, 0, s>>>(J, nao);
        ISDF_LAUNCH_CHECK();
    }
    if (K) {
        // K = X^T (W X)
        gemm_f64(k, nao, k, W.get(), k, 0, X, nao, 0, Y.get(), nao, 0, 1, false, s);
        gemm_f64(nao, nao, k, XT.get(), k, 0, Y.get(), nao, 0, K, nao, 0, 1, false, s);
        symmetrise_kernel<<<blocks(nao * nao), 256, 0, s>>>(K, nao);
        ISDF_LAUNCH_CHECK();
    }
}

}  // namespace isdf
