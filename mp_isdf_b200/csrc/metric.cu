// Spherical-cell grid Coulomb metric of interpolation vectors
// (grid_coulomb_metric and grid_cross_metric, python/isdf.py:48-97,
// mikovtun/mp_isdf):
//   L[a][g] = Left[a][g] w_g,  R[b][g] = Right[b][g] w_g,
//   V = L K R^T,  K_gh = 1 / |r_g - r_h| for g != h (0 for coincident points),
//                 K_gg = c |w_g|^(-1/3),  c = (32/15) pi^2 (3 / (4 pi))^(5/3),
// and for the metric of one set (Left = Right) symmetrised, (V + V^T) / 2.
// The reference forms K block by block on the host (O(Ngrid^2) work and
// memory traffic).  Here the potential P = K R^T is an FP64 all-pairs sum on
// the device: one thread per grid point g, the
// source points h staged through shared memory in tiles of their coordinates
// and their k values of X (padded to the instantiated width with zeros, so
// the inner loop has no predicates); the self term is added once per point
// after the sweep (the sweep's own h = g pair has r = 0 and contributes 0).
// Then V = L P by the FP64 GEMM.
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

// Source points per shared-memory tile: about 40 KB of coordinates and X.
template <int KM>
constexpr int metric_tile() { return KM <= 16 ? 256 : KM <= 32 ? 128 : 64; }

// P[g][j] = sum_h K_gh X[j][h] for the n grid points (row-major n x k).
template <int KM>
__global__ void __launch_bounds__(kMetricThreads)
grid_potential_kernel(const double* __restrict__ xyz, const double* __restrict__ w,
                      const double* __restrict__ X, int k, int64_t n, double c_sphere,
                      double* __restrict__ P) {
    constexpr int kTile = metric_tile<KM>();
    __shared__ double sx[kTile][3];
    __shared__ double sX[kTile][KM];
    const int t = threadIdx.x;
    const int64_t g = static_cast<int64_t>(blockIdx.x) * kMetricThreads + t;
    const bool valid = g < n;
    double gx = 0, gy = 0, gz = 0;
    if (valid) { gx = xyz[3 * g]; gy = xyz[3 * g + 1]; gz = xyz[3 * g + 2]; }
    double acc[KM];
#pragma unroll
    for (int j = 0; j < KM; ++j) acc[j] = 0.0;
    for (int64_t h0 = 0; h0 < n; h0 += kTile) {
        if (t < kTile) {
            const int64_t h = h0 + t;
            if (h < n) {
                sx[t][0] = xyz[3 * h];
                sx[t][1] = xyz[3 * h + 1];
                sx[t][2] = xyz[3 * h + 2];
            }
#pragma unroll
            for (int j = 0; j < KM; ++j) sX[t][j] = (h < n && j < k) ? X[j * n + h] : 0.0;
        }
        __syncthreads();
        const int cnt = n - h0 < kTile ? static_cast<int>(n - h0) : kTile;
        if (valid) {
            for (int s = 0; s < cnt; ++s) {
                const double dx = gx - sx[s][0], dy = gy - sx[s][1], dz = gz - sx[s][2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                const double kern = r2 > 0.0 ? rsqrt(r2) : 0.0;
#pragma unroll
                for (int j = 0; j < KM; ++j) acc[j] += kern * sX[s][j];
            }
        }
        __syncthreads();
    }
    if (!valid) return;
    const double self = c_sphere * pow(fabs(w[g]), -1.0 / 3.0);
#pragma unroll
    for (int j = 0; j < KM; ++j)
        if (j < k) P[g * k + j] = acc[j] + self * X[j * n + g];
}

template <int KM>
void launch_potential(const double* xyz, const double* w, const double* X, int k, int64_t n, double c,
                      double* P, cudaStream_t s) {
    const int64_t blocks = (n + kMetricThreads - 1) / kMetricThreads;
    require(blocks < (1ll << 31), "too many grid points for one launch");
    grid_potential_kernel<KM><<<static_cast<unsigned>(blocks), kMetricThreads, 0, s>>>(xyz, w, X, k, n, c, P);
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
    DeviceBuffer<double> L(static_cast<size_t>(kl) * n, s), R(static_cast<size_t>(kr) * n, s),
        P(static_cast<size_t>(kr) * n, s), V(static_cast<size_t>(kl) * kr, s);
    scale_theta_kernel<<<static_cast<unsigned>((static_cast<int64_t>(kl) * n + 255) / 256), 256, 0, s>>>(
        left, ldl, kl, n, w, L.get());
    ISDF_LAUNCH_CHECK();
    scale_theta_kernel<<<static_cast<unsigned>((static_cast<int64_t>(kr) * n + 255) / 256), 256, 0, s>>>(
        right, ldr, kr, n, w, R.get());
    ISDF_LAUNCH_CHECK();
    {
        ISDF_PROFILE("grid_potential", s);
        const double* X = R.get();
        const int k = kr;
        if (k <= 4) launch_potential<4>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else if (k <= 8) launch_potential<8>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else if (k <= 12) launch_potential<12>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else if (k <= 16) launch_potential<16>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else if (k <= 24) launch_potential<24>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else if (k <= 32) launch_potential<32>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else if (k <= 48) launch_potential<48>(xyz, w, X, k, n, c_sphere, P.get(), s);
        else launch_potential<64>(xyz, w, X, k, n, c_sphere, P.get(), s);
    }
    // V = L (kl x n) P (n x kr)
    gemm_f64(kl, kr, n, L.get(), n, 0, P.get(), kr, 0, V.get(), kr, 0, 1, false, s);
    std::vector<double> h(static_cast<size_t>(kl) * kr);
    ISDF_CUDA(cudaMemcpyAsync(h.data(), V.get(), h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    for (int a = 0; a < kl; ++a)
        for (int b = 0; b < kr; ++b)
            metric_host[a * kr + b] = symmetrize ? 0.5 * (h[a * kr + b] + h[b * kr + a]) : h[a * kr + b];
}

}  // namespace isdf
