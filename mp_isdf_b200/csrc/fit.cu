// Interpolation-vector fit and pair-space error.
//
// Reference (mikovtun/mp_isdf python/isdf.py:238-263, _physical_pair_refit):
//   C = anchor AO pairs (k x nao^2), U S V^T = svd(C^T), keep s > 1e-12 s_0,
//   X = V S^-1 U^T p_g for every grid pair column p_g = phi_g (x) phi_g,
//   Theta[:, g] = X / w_anchor.
// Without forming any grid pair column: C p_g = (Phi_a phi_g)^2 =: h_g and
// C C^T = (Phi_a Phi_a^T)^2 =: M (Hadamard squares), so
//   X_g = V_r S_r^-2 V_r^T h_g = T h_g,
// with V, S the SVD of C^T computed accurately from the R factor of an
// explicit CGS2 QR of C^T (C^T = Q R, svd(R) = U_r S V^T).
// Pair-space error (python/isdf.py:154-191), per grid point:
//   |p_g - C^T X_g|^2 = q_g^2 - 2 X_g.h_g + X_g^T M X_g,  q_g = |phi_g|^2.
#include "isdf_fit.h"
#include "isdf_project.h"
#include "isdf_reduce.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <string>

namespace isdf {
namespace {

__global__ void transpose_kernel(const double* __restrict__ a, int64_t rows, int64_t cols,
                                 double* __restrict__ at) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const int64_t r = i / cols, c = i % cols;
    at[c * rows + r] = a[i];
}

__global__ void hadamard_square_kernel(const double* __restrict__ a, int64_t n, double* __restrict__ b) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i] * a[i];
}

__global__ void gather_points_kernel(const double* __restrict__ pts, const double* __restrict__ w,
                                     const int64_t* __restrict__ idx, int64_t n,
                                     double* __restrict__ out_pts, double* __restrict__ out_w,
                                     int64_t npts_total, int* __restrict__ bad) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t g = idx[i];
    if (g < 0 || g >= npts_total) { atomicOr(bad, 1); return; }
    out_pts[3 * i] = pts[3 * g];
    out_pts[3 * i + 1] = pts[3 * g + 1];
    out_pts[3 * i + 2] = pts[3 * g + 2];
    if (out_w) out_w[i] = w[g];
}

// One-sided Jacobi SVD of the k x k column-major matrix A (overwritten by
// U*S), accumulating the right singular vectors in V (column-major).  One CTA,
// round-robin (circle method) pair ordering, warps own pairs.
__global__ void __launch_bounds__(1024)
jacobi_svd_kernel(double* A, double* V, int k, int max_sweeps, int* sweeps_out) {
    const int kp = k + (k & 1);
    const int lane = threadIdx.x % 32, wid = threadIdx.x / 32, nw = blockDim.x / 32;
    for (int i = threadIdx.x; i < k * k; i += blockDim.x) V[i] = (i % k == i / k) ? 1.0 : 0.0;
    __shared__ int rotated;
    const double eps = 2.220446049250313e-16;
    int sweep = 0;
    for (; sweep < max_sweeps; ++sweep) {
        if (threadIdx.x == 0) rotated = 0;
        __syncthreads();
        for (int round = 0; round < kp - 1; ++round) {
            for (int pr = wid; pr < kp / 2; pr += nw) {
                // circle method: player 0 fixed, others rotate
                int a = pr == 0 ? 0 : 1 + (pr - 1 + round) % (kp - 1);
                int b = 1 + (kp - 2 - pr + round) % (kp - 1);
                if (pr == 0) b = 1 + (kp - 2 + round) % (kp - 1);
                if (a >= k || b >= k || a == b) continue;
                if (a > b) { int t = a; a = b; b = t; }
                double alpha = 0, beta = 0, gamma = 0;
                for (int r = lane; r < k; r += 32) {
                    const double x = A[a * k + r], y = A[b * k + r];
                    alpha += x * x; beta += y * y; gamma += x * y;
                }
                alpha = warp_sum(alpha); beta = warp_sum(beta); gamma = warp_sum(gamma);
                alpha = __shfl_sync(0xffffffffu, alpha, 0);
                beta = __shfl_sync(0xffffffffu, beta, 0);
                gamma = __shfl_sync(0xffffffffu, gamma, 0);
                if (gamma == 0.0 || fabs(gamma) <= eps * sqrt(alpha * beta)) continue;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                for (int r = lane; r < k; r += 32) {
                    const double x = A[a * k + r], y = A[b * k + r];
                    A[a * k + r] = cs * x - sn * y;
                    A[b * k + r] = sn * x + cs * y;
                    const double vx = V[a * k + r], vy = V[b * k + r];
                    V[a * k + r] = cs * vx - sn * vy;
                    V[b * k + r] = sn * vx + cs * vy;
                }
                if (lane == 0) rotated = 1;
            }
            __syncthreads();
        }
        __syncthreads();
        if (!rotated) break;
        __syncthreads();
    }
    if (threadIdx.x == 0) sweeps_out[0] = sweep;
}

// s[j] = |A[:, j]|
// S[a][b] = phi_a . phi_b for rows a, b of A (k x n), one warp per entry.
__global__ void gram_rows_kernel(const double* __restrict__ A, int k, int n, double* __restrict__ S) {
    const int a = blockIdx.x / k, b = blockIdx.x % k;
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += 32) acc += A[static_cast<int64_t>(a) * n + i] * A[static_cast<int64_t>(b) * n + i];
    acc = warp_allsum(acc);
    if (threadIdx.x == 0) S[blockIdx.x] = acc;
}

__global__ void column_norms_kernel(const double* __restrict__ A, int k, double* __restrict__ s) {
    const int j = blockIdx.x;
    double acc = 0;
    for (int r = threadIdx.x; r < k; r += 32) acc += A[j * k + r] * A[j * k + r];
    acc = warp_sum(acc);
    if (threadIdx.x == 0) s[j] = sqrt(acc);
}

// T[a][b] = sum_j V[a,j] V[b,j] / s_j^2 over retained j  (V column-major)
__global__ void pinv_from_svd_kernel(const double* __restrict__ V, const double* __restrict__ s,
                                     int k, double cutoff, double power, double* __restrict__ T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k * k) return;
    const int a = i / k, b = i % k;
    double acc = 0;
    for (int j = 0; j < k; ++j)
        if (s[j] > cutoff) acc += V[j * k + a] * V[j * k + b] / pow(s[j], power);
    T[i] = acc;
}

// Per point: Theta, pair-error terms, Theta.w and max |X|.
template <bool HAVE_THETA>
__global__ void fit_point_kernel(const double* __restrict__ H, const double* __restrict__ X,
                                 const double* __restrict__ Y, const double* __restrict__ q,
                                 const double* __restrict__ w, int64_t b, int k,
                                 const double* __restrict__ wa, double* __restrict__ theta,
                                 int64_t ldt, int64_t g0, double* __restrict__ acc) {
    __shared__ double sh[8];
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double e = 0, ex = 0, mx = 0;
    if (g < b) {
        const double* h = H + g * k;
        const double* x = X + g * k;
        const double* y = Y + g * k;
        double xh = 0, xy = 0;
        for (int a = 0; a < k; ++a) {
            xh += x[a] * h[a];
            xy += x[a] * y[a];
            mx = fmax(mx, fabs(x[a]));
            if (!HAVE_THETA) theta[a * ldt + g0 + g] = x[a] / wa[a];
        }
        const double aw = fabs(w[g]);
        e = aw * (q[g] * q[g] - 2.0 * xh + xy);
        ex = aw * q[g] * q[g];
    }
    e = block_sum<256>(e, sh);
    ex = block_sum<256>(ex, sh);
    double m = mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double msh[8];
    if (threadIdx.x % 32 == 0) msh[threadIdx.x / 32] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < 8; ++i) m = fmax(m, msh[i]);
        atomicAdd(&acc[0], e);
        atomicAdd(&acc[1], ex);
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long*>(&acc[2]),
                  static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// tw[a] += sum_g Theta[a, g] w_g over the chunk (one block per anchor row)
__global__ void theta_dot_w_kernel(const double* __restrict__ theta, int64_t ldt, int64_t g0,
                                   int64_t b, const double* __restrict__ w, double* __restrict__ tw) {
    __shared__ double sh[8];
    const int a = blockIdx.y;
    double acc = 0;
    for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < b;
         g += static_cast<int64_t>(gridDim.x) * blockDim.x)
        acc += theta[a * ldt + g0 + g] * w[g];
    acc = block_sum<256>(acc, sh);
    if (threadIdx.x == 0) atomicAdd(&tw[a], acc);
}

// X[g][a] = Theta[a, g0+g] * wa[a]
__global__ void theta_to_x_kernel(const double* __restrict__ theta, int64_t ldt, int64_t g0,
                                  int64_t b, int k, const double* __restrict__ wa,
                                  double* __restrict__ X) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= b * k) return;
    const int64_t g = i / k;
    const int a = static_cast<int>(i % k);
    X[i] = theta[a * ldt + g0 + g] * wa[a];
}

unsigned blocks_for(int64_t n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

AnchorFactor factor_anchors(const Context& c, const double* anchor_pts, const double* anchor_w,
                            int64_t k, cudaStream_t s) {
    AnchorFactor f;
    f.k = k;
    const int64_t nao = c.nao;
    if (k == 0) return f;
    require(k <= 4096, "more than 4096 anchors are not supported by the fit");
    f.phi_a.reset(static_cast<size_t>(k * nao), s);
    f.phi_aT.reset(static_cast<size_t>(k * nao), s);
    f.M.reset(static_cast<size_t>(k * k), s);
    f.T.reset(static_cast<size_t>(k * k), s);
    f.wa.reset(k, s);
    ISDF_CUDA(cudaMemcpyAsync(f.wa.get(), anchor_w, k * sizeof(double), cudaMemcpyDeviceToDevice, s));
    f.anchor_pts.reset(static_cast<size_t>(3 * k), s);
    ISDF_CUDA(cudaMemcpyAsync(f.anchor_pts.get(), anchor_pts, 3 * k * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
    eval_ao<double>(c, anchor_pts, k, f.phi_a.get(), nullptr, nao, s);
    transpose_kernel<<<blocks_for(k * nao), 256, 0, s>>>(f.phi_a.get(), k, nao, f.phi_aT.get());
    ISDF_LAUNCH_CHECK();
    DeviceBuffer<double> S(static_cast<size_t>(k * k), s);
    if (k <= 64) {
        // a few anchors: one warp per entry of the symmetric k x k Gram
        gram_rows_kernel<<<static_cast<unsigned>(k * k), 32, 0, s>>>(f.phi_a.get(), static_cast<int>(k),
                                                                     static_cast<int>(nao), S.get());
        ISDF_LAUNCH_CHECK();
    } else {
        gemm_f64(k, k, nao, f.phi_a.get(), nao, 0, f.phi_aT.get(), k, 0, S.get(), k, 0, 1, false, s);
    }
    hadamard_square_kernel<<<blocks_for(k * k), 256, 0, s>>>(S.get(), k * k, f.M.get());
    ISDF_LAUNCH_CHECK();

    // Singular values of C^T and T = pinv(C C^T) on the retained ones.  First
    // from the eigen-decomposition of M = C C^T (the route of the FP64 oracle);
    // when an eigenvalue of M falls below 1e-10 of the largest, a singular
    // value of C is within ~1e-5 of the cutoff's scale and M's roundoff could
    // decide it, so the R factor of an explicit CGS2 QR of C^T (nao^2 x k) is
    // used instead.
    const int64_t m = nao * nao;
    double power = 1.0;                 // singular values of M are s^2
    DeviceBuffer<double> A(static_cast<size_t>(k * k), s), V(static_cast<size_t>(k * k), s), sv(k, s);
    DeviceBuffer<int> sweeps(1, s);
    std::vector<double> hs(k);
    auto svd = [&]() {
        jacobi_svd_kernel<<<1, 1024, 0, s>>>(A.get(), V.get(), static_cast<int>(k), 60, sweeps.get());
        ISDF_LAUNCH_CHECK();
        column_norms_kernel<<<static_cast<unsigned>(k), 32, 0, s>>>(A.get(), static_cast<int>(k), sv.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaMemcpyAsync(hs.data(), sv.get(), k * sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
    };
    ISDF_CUDA(cudaMemcpyAsync(A.get(), f.M.get(), k * k * sizeof(double), cudaMemcpyDeviceToDevice, s));
    svd();
    const double lam_max = *std::max_element(hs.begin(), hs.end());
    const double lam_min = *std::min_element(hs.begin(), hs.end());
    f.gram_fallback = true;
    if (!(lam_min >= 1e-10 * lam_max) && m * k <= (int64_t(1) << 30)) {
        std::vector<double> R(static_cast<size_t>(k * k), 0.0);   // column-major
        DeviceBuffer<double> Q(static_cast<size_t>(m * k), s), a(m, s), r(m, s), t(k, s), nrm(1, s);
        std::vector<double> ht(k);
        for (int64_t j = 0; j < k; ++j) {
            pair_vector(f.phi_a.get() + j * nao, nao, 1.0, a.get(), s);
            const double* src = a.get();
            for (int pass = 0; pass < 2; ++pass) {
                t.zero(s);
                nrm.zero(s);
                rows_dot(Q.get(), static_cast<int>(j), m, src, t.get(), s);
                rows_axpy(Q.get(), static_cast<int>(j), m, t.get(), src, r.get(), nrm.get(), s);
                if (j) {
                    ISDF_CUDA(cudaMemcpyAsync(ht.data(), t.get(), j * sizeof(double), cudaMemcpyDeviceToHost, s));
                    ISDF_CUDA(cudaStreamSynchronize(s));
                    for (int64_t i = 0; i < j; ++i) R[j * k + i] += ht[i];
                }
                src = r.get();
            }
            double n2 = 0;
            ISDF_CUDA(cudaMemcpyAsync(&n2, nrm.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
            ISDF_CUDA(cudaStreamSynchronize(s));
            const double rjj = std::sqrt(n2);
            R[j * k + j] = rjj;
            scale_copy(r.get(), rjj > 0 ? 1.0 / rjj : 0.0, m, Q.get() + j * m, s);
        }
        ISDF_CUDA(cudaMemcpyAsync(A.get(), R.data(), R.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        svd();
        power = 2.0;   // T = V S^-2 V^T from the SVD of R
        f.gram_fallback = false;
    }
    if (f.gram_fallback)
        for (auto& x : hs) x = std::sqrt(std::max(x, 0.0));
    f.sv = hs;
    std::sort(f.sv.begin(), f.sv.end(), std::greater<double>());
    const double s0 = f.sv.empty() ? 0.0 : f.sv.front();
    const double cutoff = 1e-12 * s0;
    f.retained = 0;
    for (double x : f.sv) f.retained += x > cutoff;
    f.condition = (!f.sv.empty() && f.sv.back() > 0) ? s0 / f.sv.back() : std::numeric_limits<double>::infinity();
    // singular values in A's column order (power 1 for the Gram fallback)
    const double dev_cut = f.gram_fallback ? cutoff * cutoff : cutoff;
    pinv_from_svd_kernel<<<blocks_for(k * k), 256, 0, s>>>(V.get(), sv.get(), static_cast<int>(k),
                                                           dev_cut, power, f.T.get());
    ISDF_LAUNCH_CHECK();
    ISDF_CUDA(cudaStreamSynchronize(s));
    return f;
}

FitOutput fit_grid(const Context& c, const double* pts, const double* w, const KeptPoints& kp,
                   const AnchorFactor& f, double* theta, int64_t ldt, bool have_theta,
                   cudaStream_t s) {
    FitOutput out;
    const int64_t n = kp.n, k = f.k, nao = c.nao;
    out.theta_w.assign(k, 0.0);
    if (n == 0 || k == 0) return out;
    const int64_t chunk = std::max<int64_t>(256, std::min<int64_t>(n, (int64_t(1) << 26) / nao));
    DeviceBuffer<double> phi(static_cast<size_t>(chunk * nao), s), q(chunk, s), G(chunk * k, s),
        H(chunk * k, s), X(chunk * k, s), Y(chunk * k, s), cpts(chunk * 3, s), cw(chunk, s),
        acc(3, s), tw(k, s);
    DeviceBuffer<int> bad(1, s);
    acc.zero(s);
    tw.zero(s);
    bad.zero(s);
    for (int64_t g0 = 0; g0 < n; g0 += chunk) {
        const int64_t b = std::min(chunk, n - g0);
        gather_points_kernel<<<blocks_for(b), 256, 0, s>>>(pts, w, kp.index.get() + g0, b, cpts.get(),
                                                           cw.get(), INT64_MAX, bad.get());
        ISDF_LAUNCH_CHECK();
        eval_ao<double>(c, cpts.get(), b, phi.get(), nullptr, nao, s);
        row_dot(phi.get(), b, nao, nullptr, q.get(), s);
        gemm_f64(b, k, nao, phi.get(), nao, 0, f.phi_aT.get(), k, 0, G.get(), k, 0, 1, false, s);
        hadamard_square_kernel<<<blocks_for(b * k), 256, 0, s>>>(G.get(), b * k, H.get());
        ISDF_LAUNCH_CHECK();
        if (have_theta) {
            theta_to_x_kernel<<<blocks_for(b * k), 256, 0, s>>>(theta, ldt, g0, b, static_cast<int>(k),
                                                                f.wa.get(), X.get());
            ISDF_LAUNCH_CHECK();
        } else {
            gemm_f64(b, k, k, H.get(), k, 0, f.T.get(), k, 0, X.get(), k, 0, 1, false, s);
        }
        gemm_f64(b, k, k, X.get(), k, 0, f.M.get(), k, 0, Y.get(), k, 0, 1, false, s);
        ISDF_PROFILE("fit_point", s);
        if (have_theta)
            fit_point_kernel<true><<<blocks_for(b), 256, 0, s>>>(H.get(), X.get(), Y.get(), q.get(), cw.get(), b,
                                                                 static_cast<int>(k), f.wa.get(), theta, ldt, g0, acc.get());
        else
            fit_point_kernel<false><<<blocks_for(b), 256, 0, s>>>(H.get(), X.get(), Y.get(), q.get(), cw.get(), b,
                                                                  static_cast<int>(k), f.wa.get(), theta, ldt, g0, acc.get());
        ISDF_LAUNCH_CHECK();
        dim3 tg(static_cast<unsigned>(std::min<int64_t>(64, (b + 255) / 256)), static_cast<unsigned>(k));
        theta_dot_w_kernel<<<tg, 256, 0, s>>>(theta, ldt, g0, b, cw.get(), tw.get());
        ISDF_LAUNCH_CHECK();
    }
    double h[3];
    ISDF_CUDA(cudaMemcpyAsync(h, acc.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(out.theta_w.data(), tw.get(), k * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    out.err2 = std::max(h[0], 0.0);
    out.exact2 = h[1];
    out.max_abs_coeff = h[2];
    out.n = n;
    return out;
}

namespace {

// Mixed-precision fit epilogue, the first iterate: G (FP32, from the
// tensor-core projection) -> h = G o G, X0 = T h, Theta0 = X0 / w_anchor in
// FP64; also Theta.w, max |X|, and the terms of an a-posteriori bound on how far
// the pair error of Theta0 can lie from the FP64 fit's:
//   excess <= lambda_max(T) * sum_g |w_g| |dh_g|^2,
//   |dG_ga| <= (kFitGramBound |phi_g| + trunc) |phi_a|  (dh = 2 G dG + dG^2),
// trunc = kScreenFp32 sqrt(nao) covering the pieces the fused kernel screened.
// When the bound exceeds the tolerance (ill-conditioned anchors amplify the
// split-BF16 error of the anchors' side of G by cond(C)^2), the FP64
// refinement step below follows.
constexpr double kFitGramBound = 2e-5;

// KMAX >= k: the per-point vectors stay in registers (loops unrolled to KMAX).
template <int KMAX>
__global__ void __launch_bounds__(256)
fit_mixed_kernel(const float* __restrict__ G, const float* __restrict__ psq, int64_t n, int k,
                 const double* __restrict__ T, const double* __restrict__ M,
                 const double* __restrict__ anorm, const double* __restrict__ wa,
                 const double* __restrict__ w, const int64_t* __restrict__ index,
                 double* __restrict__ theta, int64_t ldt, double* __restrict__ tw,
                 double* __restrict__ acc, double trunc) {
    extern __shared__ double sm[];
    double* Ts = sm;                // k*k
    double* Ms = sm + k * k;        // k*k
    double* tws = sm + 2 * k * k;   // k partial sums
    __shared__ double red[8];
    for (int i = threadIdx.x; i < k * k; i += blockDim.x) { Ts[i] = T[i]; Ms[i] = M[i]; }
    for (int i = threadIdx.x; i < k; i += blockDim.x) tws[i] = 0.0;
    __syncthreads();
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double mx = 0, dh2 = 0, e2 = 0, q2 = 0;
    double h[KMAX], x[KMAX], twl[KMAX];
#pragma unroll
    for (int a = 0; a < KMAX; ++a) { h[a] = 0.0; x[a] = 0.0; twl[a] = 0.0; }
    if (g < n) {
        const double qg = static_cast<double>(psq[g * 4]);   // |phi_g|^2
        const double fn = sqrt(qg);
        const int64_t gi = index[g];
        const double wg = w[gi], aw = fabs(wg);
#pragma unroll
        for (int a = 0; a < KMAX; ++a)
            if (a < k) {
                const double gv = static_cast<double>(G[g * k + a]);
                h[a] = gv * gv;
                const double dG = (kFitGramBound * fn + trunc) * anorm[a];
                const double dh = 2.0 * fabs(gv) * dG + dG * dG;
                dh2 += dh * dh;
            }
        double xh = 0;
#pragma unroll
        for (int a = 0; a < KMAX; ++a)
            if (a < k) {
                double xa = 0;
#pragma unroll
                for (int b = 0; b < KMAX; ++b)
                    if (b < k) xa += Ts[a * k + b] * h[b];
                x[a] = xa;
                xh += xa * h[a];
                mx = fmax(mx, fabs(xa));
                const double th = xa / wa[a];
                theta[a * ldt + g] = th;
                twl[a] = th * wg;
            }
        double xmx = 0;
#pragma unroll
        for (int a = 0; a < KMAX; ++a)
            if (a < k) {
                double t = 0;
#pragma unroll
                for (int b = 0; b < KMAX; ++b)
                    if (b < k) t += Ms[a * k + b] * x[b];
                xmx += x[a] * t;
            }
        dh2 *= aw;
        e2 = aw * (qg * qg - 2.0 * xh + xmx);
        q2 = aw * qg * qg;
    }
    // Theta.w partial sums: warp reduction, one shared-memory add per warp
#pragma unroll
    for (int a = 0; a < KMAX; ++a)
        if (a < k) {
            const double v = warp_sum(twl[a]);
            if (threadIdx.x % 32 == 0) atomicAdd(&tws[a], v);
        }
    dh2 = block_sum<256>(dh2, red);
    e2 = block_sum<256>(e2, red);
    q2 = block_sum<256>(q2, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[3], dh2);
        atomicAdd(&acc[4], e2);
        atomicAdd(&acc[5], q2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if (threadIdx.x % 32 == 0)
        atomicMax(reinterpret_cast<unsigned long long*>(&acc[2]),
                  static_cast<unsigned long long>(__double_as_longlong(mx)));
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += blockDim.x) atomicAdd(&tw[i], tws[i]);
}

__global__ void row_norms_kernel(const double* __restrict__ a, int rows, int cols, double* __restrict__ out) {
    const int r = blockIdx.x;
    double s = 0;
    for (int c = threadIdx.x; c < cols; c += 32) s += a[static_cast<int64_t>(r) * cols + c] * a[static_cast<int64_t>(r) * cols + c];
    s = warp_sum(s);
    if (threadIdx.x == 0) out[r] = sqrt(s);
}

}  // namespace

// ---- one FP64 iterative-refinement step of Theta over the stored tiles ----------
// The tensor-core fit X0 = T h~ carries the split-BF16 error of BOTH operands
// of G = Phi_g Phi_a^T; an error in the anchors' values perturbs C and is
// amplified by cond(C)^2 in X.  The refinement recomputes
//     G64[g][a] = sum_mu x[g][mu] phi_a(mu)     (FP64 FMAs, FP64 anchors)
// from the stored tiles, where x = hi + lo + r is the FP32 AO value exactly
// (the fused kernel stores the BF16 remainder r next to the (hi, lo) tiles),
// then h = G64 o G64, the FP64 residual r = h - M X0 and X1 = X0 + T r,
// Theta = X1 / w_a.  Only the grid-side error dp_g = p~_g - p_g of the FP32
// evaluation remains, and it is projected, not amplified: the pair-error
// excess is
//     sum_g |w_g| |P_C dp_g|^2 <= sum_g |w_g| |dp_g|^2,  |dp_g| <= 2 |x_g| d_g + d_g^2,
// with d_g = 2^-19 |x_g| + trunc bounding |x_g - phi_g| (2^-19: twice the
// largest 2-norm error of the FP32 AO values measured against FP64 ones;
// trunc = kScreenFp32 sqrt(nao): the pieces the fused kernel screened).
namespace {

constexpr double kFp32EvalError = 1.0 / 524288.0;   // 2^-19

// PhiS[c][j][a] = phi_a[a][ao0[c] + j] for the used slots j < fill[c], else 0
// (row stride k).
__global__ void anchor_slot_image_kernel(const double* __restrict__ phi_a, int k, int nao, int nchunks,
                                         const int* __restrict__ chunk_ao0, const int* __restrict__ fill,
                                         double* __restrict__ img) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t total = static_cast<int64_t>(nchunks) * 32 * k;
    if (i >= total) return;
    const int a = static_cast<int>(i % k);
    const int j = static_cast<int>((i / k) % 32);
    const int c = static_cast<int>(i / (32 * k));
    const int ao = chunk_ao0[c] + j;
    img[i] = (j < fill[c] && ao < nao) ? phi_a[static_cast<int64_t>(a) * nao + ao] : 0.0;
}

// H[g][a0 + a] = (sum_mu x[g][mu] phi_{a0+a}(mu))^2 for a < KMAX, a0 + a < k, with
// x = hi + lo + r from the stored tiles (FP64 FMAs); q[g] = sum_mu x^2 when a0 == 0.
// One 128-point tile per block of 64 threads: thread t takes rows t and t + 64,
// so every anchor value read from shared memory (two per 16-byte load) feeds
// two FMAs.  hi + lo is exact in FP32 and so is (hi + lo) + r, whose exact
// value is the FP32 AO value itself: one conversion to FP64 per entry.
constexpr int kRefineThreads = 64;

template <int KMAX>
__global__ void __launch_bounds__(kRefineThreads)
refine_gram_kernel(const uint8_t* __restrict__ tiles, const uint8_t* __restrict__ tiles_r, int nchunks,
                   int64_t n, int k, int a0, const double* __restrict__ img, double* __restrict__ H,
                   double* __restrict__ q_out) {
    constexpr int KP = (KMAX + 1) & ~1;        // even row length: 16-byte loads of anchor pairs
    __shared__ __align__(16) double S[32 * KP];
    const int t = threadIdx.x;
    const int64_t tile = blockIdx.x;
    const int na = min(KMAX, k - a0);
    // rows t and t + 64 of a K-major interleaved 128 x 32 BF16 tile: core
    // matrices of 8 rows x 8 K (16 B rows), K-adjacent ones 2048 B apart,
    // M-adjacent ones 128 B apart
    uint32_t row_off[2];
    bool valid[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int r = t + 64 * h;
        row_off[h] = static_cast<uint32_t>(r >> 3) * 128u + static_cast<uint32_t>(r & 7) * 16u;
        valid[h] = tile * 128 + r < n;
    }
    double G[2][KP];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int a = 0; a < KP; ++a) G[h][a] = 0.0;
    double q[2] = {0.0, 0.0};
    for (int c = 0; c < nchunks; ++c) {
        __syncthreads();
        for (int i = t; i < 32 * KP; i += kRefineThreads) {
            const int j = i / KP, a = i % KP;
            S[i] = a < na ? img[(static_cast<int64_t>(c) * 32 + j) * k + a0 + a] : 0.0;
        }
        __syncthreads();
        const size_t blk = static_cast<size_t>(tile) * nchunks + c;
        const uint8_t* hi = tiles + blk * 16384u;
        const uint8_t* lo = hi + 8192u;
        const uint8_t* rm = tiles_r + blk * 8192u;
#pragma unroll
        for (int kg = 0; kg < 4; ++kg) {
            float x[2][8];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint4 vh = make_uint4(0, 0, 0, 0), vl = vh, vr = vh;
                if (valid[h]) {
                    vh = __ldcs(reinterpret_cast<const uint4*>(hi + kg * 2048u + row_off[h]));
                    vl = __ldcs(reinterpret_cast<const uint4*>(lo + kg * 2048u + row_off[h]));
                    vr = __ldcs(reinterpret_cast<const uint4*>(rm + kg * 2048u + row_off[h]));
                }
                const uint32_t h4[4] = {vh.x, vh.y, vh.z, vh.w}, l4[4] = {vl.x, vl.y, vl.z, vl.w},
                               r4[4] = {vr.x, vr.y, vr.z, vr.w};
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const uint32_t sel = (e & 1) ? 0xffff0000u : 0x0000ffffu;
                    const int shl = (e & 1) ? 0 : 16;
                    const float fh = __uint_as_float((h4[e >> 1] & sel) << shl);
                    const float fl = __uint_as_float((l4[e >> 1] & sel) << shl);
                    const float fr = __uint_as_float((r4[e >> 1] & sel) << shl);
                    x[h][e] = __fadd_rn(__fadd_rn(fh, fl), fr);   // the FP32 value, exactly
                }
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const double x0 = static_cast<double>(x[0][e]), x1 = static_cast<double>(x[1][e]);
                q[0] = fma(x0, x0, q[0]);
                q[1] = fma(x1, x1, q[1]);
                const double2* srow = reinterpret_cast<const double2*>(S + (kg * 8 + e) * KP);
#pragma unroll
                for (int a = 0; a < KP / 2; ++a) {
                    const double2 s2 = srow[a];
                    G[0][2 * a] = fma(x0, s2.x, G[0][2 * a]);
                    G[0][2 * a + 1] = fma(x0, s2.y, G[0][2 * a + 1]);
                    G[1][2 * a] = fma(x1, s2.x, G[1][2 * a]);
                    G[1][2 * a + 1] = fma(x1, s2.y, G[1][2 * a + 1]);
                }
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (!valid[h]) continue;
        const int64_t g = tile * 128 + t + 64 * h;
#pragma unroll
        for (int a = 0; a < KMAX; ++a)
            if (a < na) H[g * k + a0 + a] = G[h][a] * G[h][a];
        if (a0 == 0) q_out[g] = q[h];
    }
}

// Per point: X0 = Theta0 w_a, r = H - M X0 (FP64 residual), X1 = X0 + T r,
// Theta = X1 / w_a; with Theta.w per anchor and acc = {sum |w| e_g (pair error
// of the refined fit over the tile values), sum |w| q_g^2, max |X1|,
// sum |w| (2 |x_g| d_g + d_g^2)^2 (the excess bound)}.
__global__ void __launch_bounds__(256)
refine_update_kernel(const double* __restrict__ H, const double* __restrict__ qv, int64_t n, int k,
                     const double* __restrict__ T, const double* __restrict__ M, const double* __restrict__ wa,
                     const double* __restrict__ w, const int64_t* __restrict__ index, double* __restrict__ theta,
                     int64_t ldt, double* __restrict__ tw, double* __restrict__ acc, double trunc) {
    __shared__ double red[8];
    __shared__ double tws[64];
    for (int i = threadIdx.x; i < k; i += blockDim.x) tws[i] = 0.0;
    __syncthreads();
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double e2 = 0.0, q2 = 0.0, mx = 0.0, b2 = 0.0;
    if (g < n) {
        const double* h = H + g * k;
        double x0[64], r[64], x1[64];
        for (int a = 0; a < k; ++a) x0[a] = theta[a * ldt + g] * wa[a];
        for (int a = 0; a < k; ++a) {
            double v = h[a];
            for (int b = 0; b < k; ++b) v -= __ldg(M + a * k + b) * x0[b];
            r[a] = v;
        }
        double xh = 0.0;
        for (int a = 0; a < k; ++a) {
            double d = 0.0;
            for (int b = 0; b < k; ++b) d += __ldg(T + a * k + b) * r[b];
            x1[a] = x0[a] + d;
        }
        for (int a = 0; a < k; ++a) x0[a] = x1[a];
        double xmx = 0.0;
        const double wg = w[index[g]], aw = fabs(wg);
        for (int a = 0; a < k; ++a) {
            xh += x0[a] * h[a];
            double t = 0.0;
            for (int b = 0; b < k; ++b) t += __ldg(M + a * k + b) * x0[b];
            xmx += x0[a] * t;
            const double th = x0[a] / wa[a];
            theta[a * ldt + g] = th;
            atomicAdd(&tws[a], th * wg);
            mx = fmax(mx, fabs(x0[a]));
        }
        const double q = qv[g];
        e2 = aw * (q * q - 2.0 * xh + xmx);
        q2 = aw * q * q;
        const double xn = sqrt(q);
        const double d = kFp32EvalError * xn + trunc;
        const double dp = 2.0 * xn * d + d * d;
        b2 = aw * dp * dp;
    }
    e2 = block_sum<256>(e2, red);
    q2 = block_sum<256>(q2, red);
    b2 = block_sum<256>(b2, red);
    if (threadIdx.x == 0) {
        atomicAdd(&acc[0], e2);
        atomicAdd(&acc[1], q2);
        atomicAdd(&acc[3], b2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(reinterpret_cast<unsigned long long*>(&acc[2]),
                  static_cast<unsigned long long>(__double_as_longlong(mx)));
    __syncthreads();
    for (int i = threadIdx.x; i < k; i += blockDim.x) atomicAdd(&tw[i], tws[i]);
}

}  // namespace

bool fit_mixed_supported(int64_t k) { return k >= 1 && k <= 64 && project_tc_supported(1, static_cast<int>(k)); }

namespace {

// Register width (anchors per pass) of the refinement's Gram kernel.
int refine_kmax(int64_t k) { return k <= 4 ? 4 : k <= 8 ? 8 : k <= 10 ? 10 : k <= 12 ? 12 : k <= 16 ? 16 : 32; }

template <int K>
void launch_refine_gram(const uint8_t* tiles, const uint8_t* tiles_r, int nchunks, int64_t n, int k,
                        const double* img, double* H, double* q, cudaStream_t s) {
    const unsigned grid = static_cast<unsigned>((n + 127) / 128);
    for (int a0 = 0; a0 < k; a0 += K) {
        refine_gram_kernel<K><<<grid, kRefineThreads, 0, s>>>(tiles, tiles_r, nchunks, n, k, a0, img, H, q);
        ISDF_LAUNCH_CHECK();
    }
}

// One FP64 refinement step of the Theta columns of n points whose AO tiles
// start at `tiles`.
void refine_theta(int kmax, const uint8_t* tiles, const uint8_t* tiles_r, int nchunks, int64_t n, int k,
                  const double* img,
                  const AnchorFactor& f, const double* w, const int64_t* index, double* theta, int64_t ldt,
                  double* H, double* q, double* tw, double* acc, double trunc, cudaStream_t s) {
    switch (kmax) {
    case 4: launch_refine_gram<4>(tiles, tiles_r, nchunks, n, k, img, H, q, s); break;
    case 8: launch_refine_gram<8>(tiles, tiles_r, nchunks, n, k, img, H, q, s); break;
    case 10: launch_refine_gram<10>(tiles, tiles_r, nchunks, n, k, img, H, q, s); break;
    case 12: launch_refine_gram<12>(tiles, tiles_r, nchunks, n, k, img, H, q, s); break;
    case 16: launch_refine_gram<16>(tiles, tiles_r, nchunks, n, k, img, H, q, s); break;
    default: launch_refine_gram<32>(tiles, tiles_r, nchunks, n, k, img, H, q, s); break;
    }
    refine_update_kernel<<<blocks_for(n), 256, 0, s>>>(H, q, n, k, f.T.get(), f.M.get(), f.wa.get(), w, index,
                                                     theta, ldt, tw, acc, trunc);
    ISDF_LAUNCH_CHECK();
}

}  // namespace

FitOutput fit_grid_mixed(const Context& c, const double* pts, const double* w, const KeptPoints& kp,
                         const AnchorFactor& f, double* theta, int64_t ldt, cudaStream_t s,
                         const uint8_t* ao_tiles, const uint8_t* ao_tiles_r, const float* ao_psq,
                         const FitChunkHook* on_chunk, const uint8_t* ao_chunk_zero) {
    FitOutput out;
    const int64_t n = kp.n, k = f.k, nao = c.nao;
    out.theta_w.assign(k, 0.0);
    if (n == 0 || k == 0) return out;
    ProjectPlan plan;
    {
        ISDF_PROFILE("phase:fit_plan", s);
        // W[mu][a] = phi_a[a*nao + mu]
        const WSource src{f.phi_a.get(), 0, 1, nao, static_cast<int>(k), 0};
        plan = make_project_plan(c, {0}, static_cast<int>(k), &src, 1, s);
    }
    DeviceBuffer<float> G(static_cast<size_t>(n * k), s), psq;
    DeviceBuffer<int> err(1, s);
    DeviceBuffer<double> acc(6, s), tw(k, s), anorm(k, s);
    err.zero(s);
    acc.zero(s);
    tw.zero(s);
    row_norms_kernel<<<static_cast<unsigned>(k), 32, 0, s>>>(f.phi_a.get(), static_cast<int>(k),
                                                            static_cast<int>(nao), anorm.get());
    ISDF_LAUNCH_CHECK();
    const float* point_sq = ao_psq;
    const uint8_t* tiles = ao_tiles;
    const uint8_t* tiles_r = ao_tiles_r;
    DeviceBuffer<uint8_t> own_tiles;
    if (!ao_tiles || !ao_tiles_r || !ao_psq) {
        // no tiles from a preceding sketch: the projection computes G and
        // stores the tiles (hi, lo and remainder) for a refinement step
        psq.reset(static_cast<size_t>(n * 4), s);
        psq.zero(s);
        own_tiles.reset(stored_tile_bytes(c, n) + stored_remainder_bytes(c, n), s);
        project_tc(c, plan, pts, kp.index.get(), n, nullptr, G.get(), k, 1, nullptr, psq.get(), err.get(), s,
                   own_tiles.get(), 0, own_tiles.get() + stored_tile_bytes(c, n));
        point_sq = psq.get();
        tiles = own_tiles.get();
        tiles_r = own_tiles.get() + stored_tile_bytes(c, n);
        ao_tiles = nullptr;
    }
    // With stored tiles and a hook, the points go in a few chunks of whole
    // 128-point tiles, each at least two waves of the stored-tile GEMM.
    const int64_t ntiles = (n + 127) / 128;
    const int64_t nchunk = (ao_tiles && on_chunk) ? std::max<int64_t>(1, std::min<int64_t>(8, ntiles / 296)) : 1;
    int64_t per = (ntiles + nchunk - 1) / nchunk * 128;
    // chunks of whole windows of a spatial order, so that each chunk's Theta
    // columns can be put back in ascending order on their own
    if (kp.spatial()) per = (per + kSpatialWindow - 1) / kSpatialWindow * kSpatialWindow;
    const size_t smem = static_cast<size_t>(2 * k * k + k) * sizeof(double);
    auto kern = k <= 16 ? fit_mixed_kernel<16> : k <= 32 ? fit_mixed_kernel<32> : fit_mixed_kernel<64>;
    const double trunc = kScreenFp32 * std::sqrt(static_cast<double>(c.nao));
    // 1. the tensor-core first iterate Theta0 and its a-posteriori bound
    for (int64_t g0 = 0; g0 < n; g0 += per) {
        const int64_t m = std::min(per, n - g0);
        if (ao_tiles)
            // AO values of these points already sit in HBM as split-BF16 tiles
            gram_from_tiles(c, plan, ao_tiles + stored_tile_bytes(c, g0), m, G.get() + g0 * k, k, err.get(), s,
                            ao_chunk_zero ? ao_chunk_zero + (g0 / 128) * c.nchunks : nullptr);
        {
            ISDF_PROFILE("fit_mixed", s);
            kern<<<blocks_for(m), 256, smem, s>>>(G.get() + g0 * k, point_sq + g0 * 4, m, static_cast<int>(k),
                                                  f.T.get(), f.M.get(), anorm.get(), f.wa.get(), w,
                                                  kp.index.get() + g0, theta + g0, ldt, tw.get(), acc.get(),
                                                  trunc);
            ISDF_LAUNCH_CHECK();
        }
        if (on_chunk && ao_tiles) (*on_chunk)(g0, m);
    }
    double h[6];
    int herr = 0;
    ISDF_CUDA(cudaMemcpyAsync(h, acc.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(out.theta_w.data(), tw.get(), k * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (herr) fail(kRuntime, "tensor-core fit pipeline timed out (error flags " + std::to_string(herr) + ")");
    // lambda_max(T) = 1 / s_min^2 over the retained singular values of C^T
    double smin = 0;
    for (double x : f.sv)
        if (x > 1e-12 * (f.sv.empty() ? 0.0 : f.sv.front())) smin = x;
    const double lam = smin > 0 ? 1.0 / (smin * smin) : std::numeric_limits<double>::infinity();
    out.mixed_bound = (h[4] > 0) ? lam * h[3] / (2.0 * h[4]) : std::numeric_limits<double>::infinity();
    out.max_abs_coeff = h[2];
    out.n = n;
    out.err2 = std::numeric_limits<double>::quiet_NaN();
    out.exact2 = std::numeric_limits<double>::quiet_NaN();
    out.path = 1;
    if (out.mixed_bound <= kMixedFitTolerance) return out;

    // 2. one FP64 iterative-refinement step over the stored tiles
    const int kmax = refine_kmax(k);
    DeviceBuffer<double> img(static_cast<size_t>(c.nchunks) * 32 * k, s), racc(4, s), rtw(k, s);
    racc.zero(s);
    rtw.zero(s);
    {
        const int64_t total = static_cast<int64_t>(c.nchunks) * 32 * k;
        anchor_slot_image_kernel<<<blocks_for(total), 256, 0, s>>>(f.phi_a.get(), static_cast<int>(k),
                                                                   static_cast<int>(nao), c.nchunks, c.d_chunk_ao0,
                                                                   c.d_fill, img.get());
        ISDF_LAUNCH_CHECK();
    }
    DeviceBuffer<double> H64(static_cast<size_t>(std::min(per, n) * k), s), q64(std::min(per, n), s);
    for (int64_t g0 = 0; g0 < n; g0 += per) {
        const int64_t m = std::min(per, n - g0);
        ISDF_PROFILE("fit_refine", s);
        refine_theta(kmax, tiles + stored_tile_bytes(c, g0), tiles_r + stored_remainder_bytes(c, g0), c.nchunks, m,
                     static_cast<int>(k), img.get(), f, w, kp.index.get() + g0, theta + g0, ldt, H64.get(),
                     q64.get(), rtw.get(), racc.get(), trunc, s);
    }
    double r[4];
    ISDF_CUDA(cudaMemcpyAsync(r, racc.get(), sizeof(r), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(out.theta_w.data(), rtw.get(), k * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    // relative pair-error excess of the refined Theta over the FP64 fit:
    // (err^2 + excess)^(1/2) / err - 1 <= excess / (2 err^2)
    out.mixed_bound = (r[0] > 0) ? r[3] / (2.0 * r[0]) : std::numeric_limits<double>::infinity();
    out.max_abs_coeff = r[2];
    out.path = 3;
    return out;
}

void gather_points(const double* pts, const double* w, const int64_t* idx, int64_t n,
                   int64_t npts_total, double* out_pts, double* out_w, cudaStream_t s) {
    if (n == 0) return;
    DeviceBuffer<int> bad(1, s);
    bad.zero(s);
    gather_points_kernel<<<blocks_for(n), 256, 0, s>>>(pts, w, idx, n, out_pts, out_w, npts_total,
                                                       bad.get());
    ISDF_LAUNCH_CHECK();
    int hb = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hb) fail(kInvalid, "anchor index outside the grid");
}

void pair_error_terms(int64_t n, int64_t k, const double* q, const double* H, const double* X,
                      const double* M, const double* w, double* out2, cudaStream_t s) {
    DeviceBuffer<double> Y(std::max<int64_t>(1, n * k), s), acc(3, s);
    acc.zero(s);
    gemm_f64(n, k, k, X, k, 0, M, k, 0, Y.get(), k, 0, 1, false, s);
    fit_point_kernel<true><<<blocks_for(n), 256, 0, s>>>(H, X, Y.get(), q, w, n, static_cast<int>(k),
                                                         nullptr, nullptr, 0, 0, acc.get());
    ISDF_LAUNCH_CHECK();
    ISDF_CUDA(cudaMemcpyAsync(out2, acc.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
}

}  // namespace isdf
