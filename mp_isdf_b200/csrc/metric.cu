// Spherical-cell grid Coulomb metric of interpolation vectors
// (grid_coulomb_metric and grid_cross_metric, python/isdf.py:48-97,
// mikovtun/mp_isdf):
//   L[a][g] = Left[a][g] w_g,  R[b][g] = Right[b][g] w_g,
//   V = L K R^T,  K_gh = 1 / |r_g - r_h| for g != h (0 for coincident points),
//                 K_gg = c |w_g|^(-1/3),  c = (32/15) pi^2 (3 / (4 pi))^(5/3),
// and for the metric of one set (Left = Right) symmetrised, (V + V^T) / 2.
// The reference forms K block by block on the host (O(Ngrid^2) work and
// memory traffic).  Here the potential P = K R^T is an FP64 all-pairs sum on
// the device: K's entries are formed in registers as the A fragments of FP64
// tensor-core MMAs (16 grid points per warp), the source points h staged
// through shared memory in tiles of their coordinates and their k values of X
// (zero-padded to the column blocks of 8, so the inner loop has no
// predicates); the self term is added once per point after the sweep (the
// sweep's own h = g pair has r = 0 and contributes 0).  Then V = L P by the
// FP64 GEMM.
#include "isdf_metric.h"

#include <algorithm>
#include <cmath>

namespace isdf {
namespace {

constexpr int kMetricThreads = 256;

// X[j][g] = Theta[j][g] w_g (row-major k x n, leading dimension n).
__global__ void scale_theta_kernel(const double* __restrict__ theta, int64_t ldt, int k, int64_t n,
                                   const double* __restrict__ w, double* __restrict__ X) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<int64_t>(k) * n) return;
    const int64_t j = i / n, g = i % n;
    X[i] = theta[j * ldt + g] * w[g];
}

// One DMMA step (FP64 tensor cores): the 16 x 8 block c += a (16 x 4) b (4 x 8),
// a in rows (lane / 4, lane / 4 + 8) and column lane % 4, b in row lane % 4
// and column lane / 4, c in rows (lane / 4, lane / 4 + 8) and columns
// 2 (lane % 4) + {0, 1} (PTX mma.m16n8k4 .f64 fragment layout).
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b));
}

__device__ __forceinline__ double inverse_distance(double gx, double gy, double gz, double4 h) {
    const double dx = gx - h.x, dy = gy - h.y, dz = gz - h.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    return r2 > 0.0 ? rsqrt(r2) : 0.0;
}

// Source points per shared-memory tile for NT column blocks of 8: about 32 KB
// of X fragments plus 32 B of coordinates per point.
template <int NT>
__host__ __device__ constexpr int metric_tile() { return NT <= 2 ? 256 : NT <= 4 ? 128 : 64; }

// P[g][j] = sum_h K_gh X[j][h] for the n grid points (row-major n x k),
// k <= 8 NT.  Each warp owns 16 grid points (rows of K) and walks the source
// points four at a time: every lane forms the two kernel entries of its A
// fragment (FP64 rsqrt) and the tensor cores accumulate the 16 x 8 blocks of
// P, NT per step.  The source tile's X values are stored in shared memory in
// B-fragment order (one double per lane per step and column block, so the
// loads are conflict-free); padded rows and columns hold zeros and contribute
// exactly nothing.  The FP64 DMMA adds its four products into the accumulator
// one after the other in order, so the sums are those of a sequential loop
// over the source points.
//
// upper: the symmetric form.  With the points cut into tiles of kTile, a warp
// (16 points inside one tile S) takes only the source tiles T > S and, with
// weight 1/2, its own tile S (and half the self term): P_up.  Every ordered
// pair (g, h) is then counted exactly once in P_up or in the transposed
// product, so X K X^T = W + W^T with W = X P_up, for half the pairs.  A block
// starts at its first warp's tile and walks the tiles in order, so the blocks
// with the longest rows are the first ones launched.
template <int NT>
__global__ void __launch_bounds__(kMetricThreads)
grid_potential_kernel(const double* __restrict__ xyz, const double* __restrict__ w,
                      const double* __restrict__ X, int k, int64_t n, double c_sphere, bool upper,
                      double* __restrict__ P) {
    constexpr int kTile = metric_tile<NT>();
    constexpr int kSteps = kTile / 4;
    constexpr int kRowsPerBlock = kMetricThreads / 32 * 16;
    __shared__ double4 sh_xyz[kTile];
    __shared__ double sh_b[kSteps * NT * 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int gq = lane >> 2, t4 = lane & 3;
    const int64_t row0 = static_cast<int64_t>(blockIdx.x) * kRowsPerBlock + warp * 16;
    double rx[2], ry[2], rz[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int64_t g = row0 + gq + 8 * r;
        rx[r] = ry[r] = rz[r] = 0.0;
        if (g < n) { rx[r] = xyz[3 * g]; ry[r] = xyz[3 * g + 1]; rz[r] = xyz[3 * g + 2]; }
    }
    double c[NT][4];
#pragma unroll
    for (int q = 0; q < NT; ++q)
#pragma unroll
        for (int i = 0; i < 4; ++i) c[q][i] = 0.0;
    const int64_t block_row0 = static_cast<int64_t>(blockIdx.x) * kRowsPerBlock;
    const int64_t own_tile = row0 / kTile;   // the warp's 16 points lie in one tile
    for (int64_t h0 = upper ? block_row0 / kTile * kTile : 0; h0 < n; h0 += kTile) {
        for (int i = t; i < kTile; i += kMetricThreads) {
            const int64_t h = h0 + i;
            sh_xyz[i] = h < n ? make_double4(xyz[3 * h], xyz[3 * h + 1], xyz[3 * h + 2], 0.0)
                              : make_double4(0.0, 0.0, 0.0, 0.0);
        }
        // X[j][h0 + hh] -> step hh / 4, column block j / 8, lane (j % 8) * 4 + hh % 4
        for (int i = t; i < kTile * NT * 8; i += kMetricThreads) {
            const int j = i / kTile, hh = i % kTile;
            const int64_t h = h0 + hh;
            const double v = (j < k && h < n) ? X[static_cast<int64_t>(j) * n + h] : 0.0;
            sh_b[((hh >> 2) * NT + (j >> 3)) * 32 + (j & 7) * 4 + (hh & 3)] = v;
        }
        __syncthreads();
        const int64_t tile = h0 / kTile;
        if (!upper || tile > own_tile) {
#pragma unroll 4
            for (int st = 0; st < kSteps; ++st) {
                const double4 hc = sh_xyz[st * 4 + t4];
                const double a0 = inverse_distance(rx[0], ry[0], rz[0], hc);
                const double a1 = inverse_distance(rx[1], ry[1], rz[1], hc);
#pragma unroll
                for (int q = 0; q < NT; ++q) dmma_16x8x4(c[q], a0, a1, sh_b[(st * NT + q) * 32 + lane]);
            }
        } else if (tile == own_tile) {
#pragma unroll 4
            for (int st = 0; st < kSteps; ++st) {
                const double4 hc = sh_xyz[st * 4 + t4];
                const double a0 = 0.5 * inverse_distance(rx[0], ry[0], rz[0], hc);
                const double a1 = 0.5 * inverse_distance(rx[1], ry[1], rz[1], hc);
#pragma unroll
                for (int q = 0; q < NT; ++q) dmma_16x8x4(c[q], a0, a1, sh_b[(st * NT + q) * 32 + lane]);
            }
        }
        __syncthreads();
    }
    // self term: P[g][j] += c |w_g|^(-1/3) X[j][g]
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int64_t g = row0 + gq + 8 * r;
        if (g >= n) continue;
        const double self = (upper ? 0.5 : 1.0) * c_sphere * pow(fabs(w[g]), -1.0 / 3.0);
#pragma unroll
        for (int q = 0; q < NT; ++q)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int j = q * 8 + 2 * t4 + e;
                if (j < k) P[g * k + j] = c[q][2 * r + e] + self * X[static_cast<int64_t>(j) * n + g];
            }
    }
}

template <int NT>
void launch_potential(const double* xyz, const double* w, const double* X, int k, int64_t n, double c,
                      bool upper, double* P, cudaStream_t s) {
    constexpr int64_t rows = kMetricThreads / 32 * 16;
    const int64_t blocks = (n + rows - 1) / rows;
    require(blocks < (1ll << 31), "too many grid points for one launch");
    grid_potential_kernel<NT><<<static_cast<unsigned>(blocks), kMetricThreads, 0, s>>>(xyz, w, X, k, n, c, upper,
                                                                                        P);
    ISDF_LAUNCH_CHECK();
}

}  // namespace

void grid_metric(const double* left, int64_t ldl, int kl, const double* right, int64_t ldr, int kr,
                 const double* xyz, const double* w, int64_t n, bool symmetrize, double* metric_host,
                 cudaStream_t s) {
    require(kl >= 0 && kr >= 0 && n >= 0 && ldl >= n && ldr >= n, "invalid grid metric sizes");
    require(kr <= kMaxMetricAnchors, "the grid metric supports at most 64 interpolation vectors per set");
    require(!symmetrize || kl == kr, "a symmetrised metric needs one set of interpolation vectors");
    std::fill(metric_host, metric_host + static_cast<size_t>(kl) * kr, 0.0);
    if (kl == 0 || kr == 0 || n == 0) return;
    const double pi = 3.14159265358979323846;
    const double c_sphere = (32.0 / 15.0) * pi * pi * std::pow(3.0 / (4.0 * pi), 5.0 / 3.0);
    // one set (the same rows on both sides): the half-pairs form, V = W + W^T
    const bool one_set = symmetrize && left == right && ldl == ldr;
    DeviceBuffer<double> L(static_cast<size_t>(kl) * n, s), R(one_set ? 0 : static_cast<size_t>(kr) * n, s),
        P(static_cast<size_t>(kr) * n, s), V(static_cast<size_t>(kl) * kr, s);
    scale_theta_kernel<<<static_cast<unsigned>((static_cast<int64_t>(kl) * n + 255) / 256), 256, 0, s>>>(
        left, ldl, kl, n, w, L.get());
    ISDF_LAUNCH_CHECK();
    if (!one_set) {
        scale_theta_kernel<<<static_cast<unsigned>((static_cast<int64_t>(kr) * n + 255) / 256), 256, 0, s>>>(
            right, ldr, kr, n, w, R.get());
        ISDF_LAUNCH_CHECK();
    }
    {
        ISDF_PROFILE("grid_potential", s);
        const double* X = one_set ? L.get() : R.get();
        const int k = kr;
        switch ((k + 7) / 8) {
            case 1: launch_potential<1>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            case 2: launch_potential<2>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            case 3: launch_potential<3>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            case 4: launch_potential<4>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            case 5: launch_potential<5>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            case 6: launch_potential<6>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            case 7: launch_potential<7>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
            default: launch_potential<8>(xyz, w, X, k, n, c_sphere, one_set, P.get(), s); break;
        }
    }
    // V = L (kl x n) P (n x kr); for one set P holds P_up and V = W + W^T
    gemm_f64(kl, kr, n, L.get(), n, 0, P.get(), kr, 0, V.get(), kr, 0, 1, false, s);
    std::vector<double> h(static_cast<size_t>(kl) * kr);
    ISDF_CUDA(cudaMemcpyAsync(h.data(), V.get(), h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    for (int a = 0; a < kl; ++a)
        for (int b = 0; b < kr; ++b)
            metric_host[a * kr + b] = one_set      ? h[a * kr + b] + h[b * kr + a]
                                      : symmetrize ? 0.5 * (h[a * kr + b] + h[b * kr + a])
                                                   : h[a * kr + b];
}

}  // namespace isdf
