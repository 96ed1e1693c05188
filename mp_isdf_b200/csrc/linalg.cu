// Small FP64 dense building blocks shared by the selection and fit stages.
#include "isdf_internal.h"
#include "isdf_reduce.cuh"

#include <algorithm>

namespace isdf {
namespace {

// ---- FP64 GEMM on the FP64 tensor cores (DMMA) ------------------------------------
// C[z] (+)= A[z] (M x K, row-major, lda) * B[z] (K x N, row-major, ldb).
// A block of 128 threads computes a 128 x (8 NT) tile of C: each warp owns 32
// rows (two m16 tiles) and all 8 NT columns (NT n8 tiles), so one k4 step is
// 2 NT mma.sync.m16n8k4.f64.  A and B tiles of BK = 16 go through shared
// memory (padded so that the fragment loads take the minimum two wavefronts);
// the next tile is prefetched into registers while the current one is
// multiplied.  Split-K (atomic FP64 adds into a zeroed C) spreads small M x N
// over the SMs when K is long.
constexpr int kGemmThreads = 128;
constexpr int kGemmBM = 128, kGemmBK = 16;
constexpr int kAStride = kGemmBK + 4;   // A[m][k] rows: 20 doubles (fragment loads conflict-free)

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b));
}

template <int NT>
__global__ void __launch_bounds__(kGemmThreads)
gemm_dmma_kernel(int64_t M, int64_t N, int64_t K, const double* __restrict__ A, int64_t lda, int64_t sA,
                 const double* __restrict__ B, int64_t ldb, int64_t sB, double* __restrict__ C, int64_t ldc,
                 int64_t sC, bool acc, int64_t kslice, int nz) {
    constexpr int BN = 8 * NT;
    // B[k][n] rows: a stride of 8 mod 16 doubles makes the fragment loads conflict-free
    constexpr int kBStride = BN + ((BN % 16 == 0) ? 8 : 16);
    constexpr int kALoads = kGemmBM * kGemmBK / kGemmThreads;               // 16
    constexpr int kBLoads = (kGemmBK * BN + kGemmThreads - 1) / kGemmThreads;
    __shared__ double As[kGemmBM * kAStride];
    __shared__ double Bs[kGemmBK * kBStride];
    const int z = blockIdx.z % nz;           // batch entry
    const int split = blockIdx.z / nz;       // K slice
    A += z * sA;
    B += z * sB;
    C += z * sC;
    const int64_t m0 = static_cast<int64_t>(blockIdx.x) * kGemmBM;
    const int64_t n0 = static_cast<int64_t>(blockIdx.y) * BN;
    const int64_t kb = split * kslice, ke = min(K, kb + kslice);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    double c[2][NT][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) c[i][j][q] = 0.0;
    double ra[kALoads], rb[kBLoads];
    auto load = [&](int64_t k0) {
#pragma unroll
        for (int j = 0; j < kALoads; ++j) {
            const int i = t + kGemmThreads * j;
            const int64_t gm = m0 + i / kGemmBK, gk = k0 + i % kGemmBK;
            ra[j] = (gm < M && gk < ke) ? __ldg(A + gm * lda + gk) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < kBLoads; ++j) {
            const int i = t + kGemmThreads * j;
            const int64_t gk = k0 + i / BN, gn = n0 + i % BN;
            rb[j] = (i < kGemmBK * BN && gk < ke && gn < N) ? __ldg(B + gk * ldb + gn) : 0.0;
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int j = 0; j < kALoads; ++j) {
            const int i = t + kGemmThreads * j;
            As[(i / kGemmBK) * kAStride + i % kGemmBK] = ra[j];
        }
#pragma unroll
        for (int j = 0; j < kBLoads; ++j) {
            const int i = t + kGemmThreads * j;
            if (i < kGemmBK * BN) Bs[(i / BN) * kBStride + i % BN] = rb[j];
        }
    };
    if (kb < ke) {
        load(kb);
        store();
        __syncthreads();
    }
    const int wm = warp * 32;
    for (int64_t k0 = kb; k0 < ke; k0 += kGemmBK) {
        const bool more = k0 + kGemmBK < ke;
        if (more) load(k0 + kGemmBK);
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk += 4) {
            double a[2][2], b[NT];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                a[i][0] = As[(wm + i * 16 + g) * kAStride + kk + t4];
                a[i][1] = As[(wm + i * 16 + g + 8) * kAStride + kk + t4];
            }
#pragma unroll
            for (int j = 0; j < NT; ++j) b[j] = Bs[(kk + t4) * kBStride + j * 8 + g];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j) dmma_16x8x4(c[i][j], a[i][0], a[i][1], b[j]);
        }
        __syncthreads();
        if (more) {
            store();
            __syncthreads();
        }
    }
    const bool atomic = gridDim.z > static_cast<unsigned>(nz);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t gm = m0 + wm + i * 16 + g + 8 * h;
            if (gm >= M) continue;
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int64_t gn = n0 + j * 8 + 2 * t4 + e;
                    if (gn >= N) continue;
                    double* dst = C + gm * ldc + gn;
                    const double v = c[i][j][2 * h + e];
                    if (atomic) atomicAdd(dst, v);
                    else *dst = acc ? *dst + v : v;
                }
        }
}

// C[z][m][n] = 0 (split-K target)
__global__ void zero_matrix_kernel(double* C, int64_t M, int64_t N, int64_t ldc, int64_t sC, int nz) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= M * N * nz) return;
    const int64_t z = i / (M * N), r = (i / N) % M, col = i % N;
    C[z * sC + r * ldc + col] = 0.0;
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
    // column tile: the narrowest of 16, 32, 56, 64 that covers N (or 64 columns per tile)
    const int nt = N <= 16 ? 2 : N <= 32 ? 4 : N <= 56 ? 7 : 8;
    const int64_t bn = 8 * nt;
    const int64_t tiles_m = (M + kGemmBM - 1) / kGemmBM, tiles_n = (N + bn - 1) / bn;
    // split K when the output tiles cannot fill the GPU and K is long
    int64_t splits = 1;
    const int64_t tiles = tiles_m * tiles_n * batch;
    if (K >= 4096 && tiles < 296) splits = std::min<int64_t>((K + 2047) / 2048, (592 + tiles - 1) / tiles);
    splits = std::max<int64_t>(1, std::min<int64_t>(splits, 65535 / std::max(batch, 1)));
    int64_t kslice = (K + splits - 1) / splits;
    kslice = (kslice + kGemmBK - 1) / kGemmBK * kGemmBK;
    splits = std::max<int64_t>(1, (K + kslice - 1) / kslice);
    if (K == 0) {
        kslice = 0;
        splits = 1;
    }
    dim3 grid(static_cast<unsigned>(tiles_m), static_cast<unsigned>(tiles_n),
              static_cast<unsigned>(batch * splits));
    require(grid.x < (1u << 31) && grid.y < 65536 && grid.z < 65536, "GEMM shape exceeds the launch limits");
    ISDF_PROFILE("gemm_f64", s);
    if (splits > 1 && !accumulate) {
        const int64_t total = M * N * batch;
        zero_matrix_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(C, M, N, ldc, strideC, batch);
        ISDF_LAUNCH_CHECK();
    }
#define ISDF_GEMM_CASE(NT_)                                                                              \
    if (nt == NT_) {                                                                                     \
        gemm_dmma_kernel<NT_><<<grid, kGemmThreads, 0, s>>>(M, N, K, A, lda, strideA, B, ldb, strideB, C, \
                                                            ldc, strideC, accumulate, kslice, batch);    \
    }
    ISDF_GEMM_CASE(2) ISDF_GEMM_CASE(4) ISDF_GEMM_CASE(7) ISDF_GEMM_CASE(8)
#undef ISDF_GEMM_CASE
    ISDF_LAUNCH_CHECK();
}

}  // namespace isdf
