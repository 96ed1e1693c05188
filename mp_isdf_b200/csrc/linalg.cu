// Small FP64 dense building blocks shared by the selection and fit stages.
#include "isdf_internal.h"
#include "isdf_reduce.cuh"

#include <algorithm>

namespace isdf {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, TM = 4, TN = 4;

// C[z] = A[z] (M x K, row-major, lda) * B[z] (K x N, row-major, ldb) (+ C[z]).
__global__ void __launch_bounds__(256)
gemm_f64_kernel(int64_t M, int64_t N, int64_t K, const double* __restrict__ A, int64_t lda,
                int64_t sA, const double* __restrict__ B, int64_t ldb, int64_t sB,
                double* __restrict__ C, int64_t ldc, int64_t sC, bool acc) {
    __shared__ double As[BK][BM + 1];
    __shared__ double Bs[BK][BN];
    const int z = blockIdx.z;
    A += z * sA;
    B += z * sB;
    C += z * sC;
    const int64_t m0 = static_cast<int64_t>(blockIdx.x) * BM;
    const int64_t n0 = static_cast<int64_t>(blockIdx.y) * BN;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double r[TM][TN] = {};
    for (int64_t k0 = 0; k0 < K; k0 += BK) {
        for (int i = threadIdx.x; i < BM * BK; i += 256) {
            const int mm = i / BK, kk = i % BK;
            const int64_t gm = m0 + mm, gk = k0 + kk;
            As[kk][mm] = (gm < M && gk < K) ? A[gm * lda + gk] : 0.0;
        }
        for (int i = threadIdx.x; i < BN * BK; i += 256) {
            const int kk = i / BN, nn = i % BN;
            const int64_t gn = n0 + nn, gk = k0 + kk;
            Bs[kk][nn] = (gn < N && gk < K) ? B[gk * ldb + gn] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[kk][ty * TM + i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) r[i][j] = fma(a[i], b[j], r[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int64_t gm = m0 + ty * TM + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int64_t gn = n0 + tx + 16 * j;
            if (gn < N) C[gm * ldc + gn] = acc ? C[gm * ldc + gn] + r[i][j] : r[i][j];
        }
    }
}

// warp per row: out[g] = F[g,:] . x   (and nf[g] = |F[g,:]|^2 when x == nullptr)
__global__ void row_dot_kernel(const double* __restrict__ F, int64_t n, int64_t d,
                               const double* __restrict__ x, double* __restrict__ out) {
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (g >= n) return;
    const double* row = F + g * d;
    double acc = 0;
    if (x)
        for (int64_t k = lane; k < d; k += 32) acc += row[k] * x[k];
    else
        for (int64_t k = lane; k < d; k += 32) acc += row[k] * row[k];
    acc = warp_sum(acc);
    if (lane == 0) out[g] = acc;
}

// a[i*d + k] = s f[i] f[k]
__global__ void pair_vector_kernel(const double* __restrict__ f, int64_t d, double s,
                                   double* __restrict__ a) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= d * d) return;
    a[i] = s * f[i / d] * f[i % d];
}

// out[r] += Q[r,:] . x over a chunk (split-K), r < rows
__global__ void __launch_bounds__(256)
rows_dot_kernel(const double* __restrict__ Q, int rows, int64_t m, const double* __restrict__ x,
                double* __restrict__ out) {
    __shared__ double sh[256 / 32];
    const int64_t chunk = (m + gridDim.x - 1) / gridDim.x;
    const int64_t k0 = blockIdx.x * chunk, k1 = min(m, k0 + chunk);
    for (int r = 0; r < rows; ++r) {
        double acc = 0;
        const double* q = Q + static_cast<int64_t>(r) * m;
        for (int64_t k = k0 + threadIdx.x; k < k1; k += 256) acc += q[k] * x[k];
        acc = block_sum<256>(acc, sh);
        if (threadIdx.x == 0) atomicAdd(&out[r], acc);
    }
}

// y = x - Q^T t ; norm2 += |y|^2
__global__ void __launch_bounds__(256)
rows_axpy_kernel(const double* __restrict__ Q, int rows, int64_t m, const double* __restrict__ t,
                 const double* x, double* y, double* norm2) {
    __shared__ double sh[256 / 32];
    __shared__ double ts[64];
    double acc = 0;
    const int64_t k = static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x;
    double v = 0;
    if (k < m) v = x[k];
    for (int r0 = 0; r0 < rows; r0 += 64) {
        const int nr = min(64, rows - r0);
        __syncthreads();
        if (threadIdx.x < nr) ts[threadIdx.x] = t[r0 + threadIdx.x];
        __syncthreads();
        if (k < m)
            for (int r = 0; r < nr; ++r) v -= Q[static_cast<int64_t>(r0 + r) * m + k] * ts[r];
    }
    if (k < m) { y[k] = v; acc = v * v; }
    acc = block_sum<256>(acc, sh);
    if (threadIdx.x == 0 && norm2) atomicAdd(norm2, acc);
}

__global__ void scale_copy_kernel(const double* __restrict__ x, double s, int64_t m,
                                  double* __restrict__ y) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < m) y[k] = x[k] * s;
}

__global__ void iota_kernel(int64_t* out, int64_t n) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

}  // namespace

namespace {
__global__ void widen_kernel(const float* __restrict__ x, int64_t n, double* __restrict__ y) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) y[i] = static_cast<double>(x[i]);
}
}  // namespace

void widen_f32(const float* x, int64_t n, double* y, cudaStream_t s) {
    if (n <= 0) return;
    widen_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(x, n, y);
    ISDF_LAUNCH_CHECK();
}

void iota_i64(int64_t* out, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    iota_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(out, n);
    ISDF_LAUNCH_CHECK();
}

void row_dot(const double* F, int64_t n, int64_t d, const double* x, double* out, cudaStream_t s) {
    if (n <= 0) return;
    ISDF_PROFILE("row_dot_f64", s);
    row_dot_kernel<<<static_cast<unsigned>((n * 32 + 255) / 256), 256, 0, s>>>(F, n, d, x, out);
    ISDF_LAUNCH_CHECK();
}

void pair_vector(const double* f, int64_t d, double scale, double* a, cudaStream_t s) {
    const int64_t m = d * d;
    if (m <= 0) return;
    pair_vector_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, s>>>(f, d, scale, a);
    ISDF_LAUNCH_CHECK();
}

void rows_dot(const double* Q, int rows, int64_t m, const double* x, double* out, cudaStream_t s) {
    if (rows <= 0 || m <= 0) return;
    const unsigned sk = static_cast<unsigned>(std::min<int64_t>(592, (m + 4095) / 4096));
    rows_dot_kernel<<<sk, 256, 0, s>>>(Q, rows, m, x, out);
    ISDF_LAUNCH_CHECK();
}

void rows_axpy(const double* Q, int rows, int64_t m, const double* t, const double* x, double* y,
               double* norm2, cudaStream_t s) {
    if (m <= 0) return;
    rows_axpy_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, s>>>(Q, rows, m, t, x, y, norm2);
    ISDF_LAUNCH_CHECK();
}

void scale_copy(const double* x, double scale, int64_t m, double* y, cudaStream_t s) {
    if (m <= 0) return;
    scale_copy_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, s>>>(x, scale, m, y);
    ISDF_LAUNCH_CHECK();
}

void gemm_f64(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, int64_t strideA,
              const double* B, int64_t ldb, int64_t strideB, double* C, int64_t ldc,
              int64_t strideC, int batch, bool accumulate, cudaStream_t s) {
    if (M == 0 || N == 0 || batch == 0) return;
    dim3 grid(static_cast<unsigned>((M + BM - 1) / BM), static_cast<unsigned>((N + BN - 1) / BN),
              batch);
    require(grid.x < (1u << 31) && grid.y < 65536, "GEMM shape exceeds the launch limits");
    ISDF_PROFILE("gemm_f64", s);
    gemm_f64_kernel<<<grid, 256, 0, s>>>(M, N, K, A, lda, strideA, B, ldb, strideB, C, ldc,
                                         strideC, accumulate);
    ISDF_LAUNCH_CHECK();
}

}  // namespace isdf
