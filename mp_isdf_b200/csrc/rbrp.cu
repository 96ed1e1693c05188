// AO-only robust blockwise random pivoting (RBRP) and its interpolative
// decomposition (rbrp_ao_cpu, cpp/src/anchor_select_rbrp.cpp:195-320,
// mikovtun/mp_isdf).
//
// The columns are the weighted AO pair rows of the grid points,
//   row_g[(mu, nu)] = sqrt|w_g| phi_mu(g) phi_nu(g) c_mu_nu,  mu <= nu,
//   c = 1 on the diagonal and sqrt(2) off it (p = nao (nao + 1) / 2 entries).
// Each iteration draws a block of points with probability proportional to
// their residual norms (std::discrete_distribution over std::mt19937_64, the
// reference's own sampler, on the host), orthogonalises their pair rows against
// the basis Q (two classical Gram-Schmidt passes), runs a column-pivoted QR of
// the block, keeps the columns above the block and rank cutoffs, and extends Q
// and the coefficients L (L[g][t] = row_g . q_t) of every point.
//
// Device work: the AO values stay on the GPU; the coefficients of a new basis
// vector q_t for all points are sqrt|w_g| phi_g^T S_t phi_g with S_t the
// symmetric nao x nao matrix of q_t (an FP64 GEMM over point chunks and a row
// dot); the residual refresh forms each point's pair row on the fly (one warp
// per point) and subtracts L Q.  Host work: sampling, the block QR (b <= block
// size columns), the re-orthogonalisation and the small ID (k x k SVD).
#include "isdf_rbrp.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <random>

namespace isdf {
namespace {

constexpr double kSqrt2 = 1.41421356237309504880;

// d[g] = |w_g| (sum_j phi_gj^2)^2 (the squared norm of the pair row); flags
// non-finite AO values (1) and zero or non-finite weights (2).
__global__ void rbrp_norm_kernel(const double* __restrict__ ao, const double* __restrict__ w, int64_t n,
                                 int nao, double* __restrict__ d, double* __restrict__ sw, int* bad) {
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (g >= n) return;
    double s = 0;
    bool finite = true;
    for (int j = lane; j < nao; j += 32) {
        const double x = ao[g * nao + j];
        finite = finite && isfinite(x);
        s += x * x;
    }
    s = warp_allsum(s);
    finite = __all_sync(0xffffffffu, finite);
    if (lane == 0) {
        const double wg = w[g];
        if (!finite) atomicOr(bad, 1);
        if (!isfinite(wg) || wg == 0.0) atomicOr(bad, 2);
        d[g] = fabs(wg) * s * s;
        sw[g] = sqrt(fabs(wg));
    }
}

// d[g] = |row_g - sum_t L[g][t] q_t|^2 for unchosen points (0 for chosen);
// one warp per point, lanes over the packed pair entries of each row mu.
__global__ void rbrp_residual_kernel(const double* __restrict__ ao, const double* __restrict__ sw,
                                     const double* __restrict__ L, int64_t ldl, int k,
                                     const double* __restrict__ Q, int64_t p, const char* __restrict__ chosen,
                                     int64_t n, int nao, double* __restrict__ d) {
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (g >= n) return;
    if (chosen[g]) {
        if (lane == 0) d[g] = 0.0;
        return;
    }
    const double* phi = ao + g * nao;
    const double* lg = L + g * ldl;
    const double s = sw[g];
    double acc = 0;
    int64_t base = 0;
    for (int mu = 0; mu < nao; ++mu) {
        const double a = s * phi[mu];
        for (int nu = mu + lane; nu < nao; nu += 32) {
            const int64_t i = base + (nu - mu);
            double e = a * phi[nu] * (nu == mu ? 1.0 : kSqrt2);
            for (int t = 0; t < k; ++t) e -= lg[t] * Q[t * p + i];
            acc += e * e;
        }
        base += nao - mu;
    }
    acc = warp_allsum(acc);
    if (lane == 0) d[g] = acc;
}

// S[t][mu][nu] = S[t][nu][mu] = q_t[(mu, nu)] (mu = nu) or q_t[(mu, nu)] / sqrt 2.
__global__ void rbrp_unpack_kernel(const double* __restrict__ Q, int64_t p, int nt, int nao,
                                   double* __restrict__ S) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<int64_t>(nt) * nao * nao) return;
    const int t = static_cast<int>(i / (static_cast<int64_t>(nao) * nao));
    const int r = static_cast<int>(i % (static_cast<int64_t>(nao) * nao));
    const int mu = min(r / nao, r % nao), nu = max(r / nao, r % nao);
    // packed index of (mu, nu), mu <= nu: rows 0..mu-1 hold nao + (nao-1) + ... entries
    const int64_t base = static_cast<int64_t>(mu) * nao - static_cast<int64_t>(mu) * (mu - 1) / 2;
    const double q = Q[t * p + base + (nu - mu)];
    S[i] = mu == nu ? q : q / kSqrt2;
}

// L[g][col] = sqrt|w_g| sum_mu T[g][mu] phi_g[mu] (0 for points chosen before
// this block), g in [g0, g0 + b).
__global__ void rbrp_rowdot_kernel(const double* __restrict__ T, const double* __restrict__ ao,
                                   const double* __restrict__ sw, const char* __restrict__ previously,
                                   int64_t g0, int64_t b, int nao, double* __restrict__ L, int64_t ldl,
                                   int col) {
    const int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (r >= b) return;
    const int64_t g = g0 + r;
    double s = 0;
    if (!previously[g])
        for (int j = lane; j < nao; j += 32) s += T[r * nao + j] * ao[g * nao + j];
    s = warp_allsum(s);
    if (lane == 0) L[g * ldl + col] = previously[g] ? 0.0 : sw[g] * s;
}

// d[g] = previously chosen ? 0 : max(0, d[g] - sum_{t in [old, old+keep)} L[g][t]^2).
__global__ void rbrp_decrease_kernel(const double* __restrict__ L, int64_t ldl, int old, int keep,
                                     const char* __restrict__ previously, int64_t n, double* __restrict__ d) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    double dec = 0;
    for (int t = old; t < old + keep; ++t) dec += L[g * ldl + t] * L[g * ldl + t];
    d[g] = previously[g] ? 0.0 : fmax(0.0, d[g] - dec);
}

// interp[a][g] = (sum_t L[g][t] inv[t][a]) sqrt|w_a| / (w_a sqrt|w_g|).
__global__ void rbrp_interp_kernel(const double* __restrict__ L, int64_t ldl, int k,
                                   const double* __restrict__ inv, const double* __restrict__ fac_a,
                                   const double* __restrict__ sw, int64_t n, double* __restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<int64_t>(k) * n) return;
    const int a = static_cast<int>(i / n);
    const int64_t g = i % n;
    double h = 0;
    for (int t = 0; t < k; ++t) h += L[g * ldl + t] * inv[t * k + a];
    out[i] = h * fac_a[a] / sw[g];
}

double sum_of(const std::vector<double>& a) { return std::accumulate(a.begin(), a.end(), 0.0); }

// Column-pivoted Householder QR of the p x b column-major block v (dgeqp3's
// pivot rule: the largest trailing column norm, the first in the current column
// order on ties, the pivot swapped into place).  Norms are recomputed at every
// step.  jpvt: original column of each position.
void block_qrcp(std::vector<double>& v, int64_t p, int b, std::vector<int>& jpvt, std::vector<double>& tau) {
    jpvt.resize(b);
    tau.assign(b, 0.0);
    std::iota(jpvt.begin(), jpvt.end(), 0);
    for (int s = 0; s < b && s < p; ++s) {
        int best = s;
        double bestn = -1.0;
        for (int j = s; j < b; ++j) {
            double nrm = 0;
            for (int64_t i = s; i < p; ++i) nrm += v[j * p + i] * v[j * p + i];
            if (nrm > bestn) { bestn = nrm; best = j; }
        }
        if (best != s) {
            for (int64_t i = 0; i < p; ++i) std::swap(v[s * p + i], v[best * p + i]);
            std::swap(jpvt[s], jpvt[best]);
        }
        double* col = v.data() + s * p;
        const double alpha = col[s];
        double xnorm = 0;
        for (int64_t i = s + 1; i < p; ++i) xnorm = std::hypot(xnorm, col[i]);
        if (xnorm == 0.0) { tau[s] = 0.0; continue; }
        const double beta = -std::copysign(std::hypot(alpha, xnorm), alpha);
        tau[s] = (beta - alpha) / beta;
        const double scale = 1.0 / (alpha - beta);
        for (int64_t i = s + 1; i < p; ++i) col[i] *= scale;
        col[s] = beta;
        for (int j = s + 1; j < b; ++j) {
            double* cj = v.data() + j * p;
            double dot = cj[s];
            for (int64_t i = s + 1; i < p; ++i) dot += col[i] * cj[i];
            dot *= tau[s];
            cj[s] -= dot;
            for (int64_t i = s + 1; i < p; ++i) cj[i] -= dot * col[i];
        }
    }
}

// The first `keep` columns of the orthogonal factor (dorg2r): Q = H_0 ... H_{keep-1} [I; 0].
std::vector<double> block_orgqr(const std::vector<double>& v, int64_t p, int keep, const std::vector<double>& tau) {
    std::vector<double> q(static_cast<size_t>(p) * keep, 0.0);
    for (int j = 0; j < keep; ++j) q[j * p + j] = 1.0;
    for (int s = keep - 1; s >= 0; --s) {
        const double* u = v.data() + s * p;   // u[s] = 1, u[s+1:] stored
        for (int j = s; j < keep; ++j) {
            double* qj = q.data() + j * p;
            double dot = qj[s];
            for (int64_t i = s + 1; i < p; ++i) dot += u[i] * qj[i];
            dot *= tau[s];
            qj[s] -= dot;
            for (int64_t i = s + 1; i < p; ++i) qj[i] -= dot * u[i];
        }
    }
    return q;
}

// One-sided Jacobi SVD of the k x k column-major a: a = U diag(s) V^T with s
// descending (U, Vt column-major k x k).
void small_svd(std::vector<double> a, int k, std::vector<double>& u, std::vector<double>& s,
               std::vector<double>& vt) {
    std::vector<double> v(static_cast<size_t>(k) * k, 0.0);
    for (int i = 0; i < k; ++i) v[i * k + i] = 1.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0;
        for (int i = 0; i < k; ++i)
            for (int j = i + 1; j < k; ++j) {
                double aii = 0, ajj = 0, aij = 0;
                for (int r = 0; r < k; ++r) {
                    aii += a[i * k + r] * a[i * k + r];
                    ajj += a[j * k + r] * a[j * k + r];
                    aij += a[i * k + r] * a[j * k + r];
                }
                if (aij == 0.0) continue;
                off = std::max(off, std::fabs(aij) / std::sqrt(aii * ajj));
                const double zeta = (ajj - aii) / (2 * aij);
                const double t = std::copysign(1.0, zeta) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
                const double c = 1 / std::sqrt(1 + t * t), sn = c * t;
                for (int r = 0; r < k; ++r) {
                    const double x = a[i * k + r], y = a[j * k + r];
                    a[i * k + r] = c * x - sn * y;
                    a[j * k + r] = sn * x + c * y;
                    const double vx = v[i * k + r], vy = v[j * k + r];
                    v[i * k + r] = c * vx - sn * vy;
                    v[j * k + r] = sn * vx + c * vy;
                }
            }
        if (off < 1e-15) break;
    }
    std::vector<double> sv(k);
    for (int i = 0; i < k; ++i) {
        double nrm = 0;
        for (int r = 0; r < k; ++r) nrm += a[i * k + r] * a[i * k + r];
        sv[i] = std::sqrt(nrm);
    }
    std::vector<int> order(k);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return sv[x] > sv[y]; });
    u.assign(static_cast<size_t>(k) * k, 0.0);
    vt.assign(static_cast<size_t>(k) * k, 0.0);
    s.assign(k, 0.0);
    for (int c = 0; c < k; ++c) {
        const int o = order[c];
        s[c] = sv[o];
        for (int r = 0; r < k; ++r) {
            u[c * k + r] = sv[o] > 0 ? a[o * k + r] / sv[o] : (r == c ? 1.0 : 0.0);
            vt[r * k + c] = v[o * k + r];   // Vt(c, r) = V(r, c)
        }
    }
}

}  // namespace

RbrpResult rbrp_ao(const double* ao, const double* w, int64_t n, int nao, const RbrpParams& prm,
                   cudaStream_t s) {
    const double tau_in = prm.tau_block;
    if (n <= 0 || nao <= 0 || prm.batch_size <= 0 || prm.block_size <= 0 || !std::isfinite(prm.tolerance) ||
        prm.tolerance < 0 || !std::isfinite(prm.rank_rtol) || prm.rank_rtol <= 0 ||
        !std::isfinite(prm.svd_rtol) || prm.svd_rtol < 0 ||
        (std::isfinite(tau_in) && (tau_in < 0 || tau_in >= 1)) || (!std::isfinite(tau_in) && !std::isnan(tau_in)))
        fail(kInvalid, "invalid RBRP dimensions, batch size or tolerances");
    const int64_t p = static_cast<int64_t>(nao) * (nao + 1) / 2;
    const int64_t cap = std::min({p, n, prm.max_rank ? prm.max_rank : std::min(n, p)});
    require(cap <= (int64_t(1) << 20), "RBRP rank cap exceeds the supported range");
    const double tau_block = std::isnan(tau_in) ? (prm.block_size > 1 ? 1.0 / prm.block_size : 0.0) : tau_in;
    DeviceBuffer<double> d_d(n, s), sw(n, s), L(static_cast<size_t>(n) * std::max<int64_t>(cap, 1), s),
        Q(static_cast<size_t>(p) * std::max<int64_t>(cap, 1), s);
    DeviceBuffer<char> chosen_d(n, s), prev_d(n, s);
    DeviceBuffer<int> bad(1, s);
    bad.zero(s);
    chosen_d.zero(s);
    const unsigned warps_blocks = static_cast<unsigned>((n * 32 + 255) / 256);
    rbrp_norm_kernel<<<warps_blocks, 256, 0, s>>>(ao, w, n, nao, d_d.get(), sw.get(), bad.get());
    ISDF_LAUNCH_CHECK();
    int hbad = 0;
    std::vector<double> d(n);
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(d.data(), d_d.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad & 2) fail(kInvalid, "RBRP requires finite nonzero weights");
    if (hbad & 1) fail(kInvalid, "RBRP requires finite real AOs");
    for (double x : d)
        if (!std::isfinite(x)) fail(kOverflow, "non-finite RBRP AO pair norm");
    const double total = sum_of(d), target = prm.tolerance * prm.tolerance * total;
    if (!std::isfinite(total)) fail(kOverflow, "non-finite RBRP total norm");

    std::vector<double> q;                 // host copy of the basis, k x p (row t = q_t)
    std::vector<char> chosen(n, 0);
    std::mt19937_64 rng(prm.seed);
    RbrpResult out;
    out.status = "rank_cap";
    int64_t iteration = 0;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n, (int64_t(1) << 26) / nao));
    DeviceBuffer<double> T(static_cast<size_t>(chunk) * nao, s);
    auto refresh = [&](int64_t k) {
        ISDF_CUDA(cudaMemcpyAsync(chosen_d.get(), chosen.data(), n, cudaMemcpyHostToDevice, s));
        rbrp_residual_kernel<<<warps_blocks, 256, 0, s>>>(ao, sw.get(), L.get(), std::max<int64_t>(cap, 1),
                                                          static_cast<int>(k), Q.get(), p, chosen_d.get(), n, nao,
                                                          d_d.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaMemcpyAsync(d.data(), d_d.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
    };
    std::vector<double> ao_row(nao);
    while (true) {
        const int64_t old = static_cast<int64_t>(out.indices.size());
        if (old && (sum_of(d) <= target || (prm.refresh_every && iteration % prm.refresh_every == 0))) refresh(old);
        if (sum_of(d) <= target) { out.status = "tolerance"; break; }
        if (old >= cap) break;
        std::vector<int64_t> active;
        for (int64_t i = 0; i < n; ++i)
            if (d[i] > 0 && !chosen[i]) active.push_back(i);
        if (active.empty()) { out.status = "no_candidates"; break; }
        const int b = static_cast<int>(std::min<int64_t>({prm.block_size, cap - old, static_cast<int64_t>(active.size())}));
        std::vector<int64_t> sample;
        for (int j = 0; j < b; ++j) {
            std::vector<double> left;
            left.reserve(active.size());
            for (int64_t id : active) left.push_back(d[id]);
            std::discrete_distribution<std::size_t> dist(left.begin(), left.end());
            const std::size_t pos = dist(rng);
            sample.push_back(active[pos]);
            active.erase(active.begin() + static_cast<std::ptrdiff_t>(pos));
        }
        // pair rows of the sampled points (column-major p x b)
        std::vector<double> v(static_cast<size_t>(p) * b);
        double original2 = 0;
        for (int j = 0; j < b; ++j) {
            ISDF_CUDA(cudaMemcpyAsync(ao_row.data(), ao + sample[j] * nao, nao * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
            double wj = 0;
            ISDF_CUDA(cudaMemcpyAsync(&wj, sw.get() + sample[j], sizeof(double), cudaMemcpyDeviceToHost, s));
            ISDF_CUDA(cudaStreamSynchronize(s));
            int64_t t = 0;
            for (int mu = 0; mu < nao; ++mu)
                for (int nu = mu; nu < nao; ++nu, ++t) {
                    const double x = wj * ao_row[mu] * ao_row[nu] * (mu == nu ? 1.0 : kSqrt2);
                    v[j * p + t] = x;
                    original2 += x * x;
                }
        }
        // two projection passes against the basis
        for (int pass = 0; pass < 2; ++pass)
            for (int j = 0; j < b; ++j)
                for (int64_t t = 0; t < old; ++t) {
                    double dot = 0;
                    for (int64_t i = 0; i < p; ++i) dot += v[j * p + i] * q[t * p + i];
                    for (int64_t i = 0; i < p; ++i) v[j * p + i] -= dot * q[t * p + i];
                }
        std::vector<int> piv;
        std::vector<double> tau;
        block_qrcp(v, p, b, piv, tau);
        std::vector<double> tails(b, 0.0);
        for (int row = b; row-- > 0;) {
            tails[row] = row + 1 < b ? tails[row + 1] : 0.0;
            for (int col = row; col < b; ++col) tails[row] += v[col * p + row] * v[col * p + row];
        }
        if (!(tails[0] > 0) || !std::isfinite(tails[0])) { out.status = "numerical_rank"; break; }
        int keep = 0;
        for (int i = 0; i < b; ++i)
            if (tails[i] >= tau_block * tails[0]) keep = i + 1;
        const double cutoff = prm.rank_rtol * std::sqrt(original2);
        for (int i = 0; i < keep; ++i)
            if (std::fabs(v[i * p + i]) <= cutoff) { keep = i; break; }
        if (!keep) { out.status = "numerical_rank"; break; }
        std::vector<double> qb = block_orgqr(v, p, keep, tau);
        // re-orthogonalise against the basis and the block's earlier columns
        for (int j = 0; j < keep; ++j) {
            double* col = qb.data() + static_cast<int64_t>(j) * p;
            for (int pass = 0; pass < 2; ++pass) {
                for (int64_t t = 0; t < old; ++t) {
                    double dot = 0;
                    for (int64_t i = 0; i < p; ++i) dot += q[t * p + i] * col[i];
                    for (int64_t i = 0; i < p; ++i) col[i] -= dot * q[t * p + i];
                }
                for (int t = 0; t < j; ++t) {
                    double dot = 0;
                    for (int64_t i = 0; i < p; ++i) dot += qb[t * p + i] * col[i];
                    for (int64_t i = 0; i < p; ++i) col[i] -= dot * qb[t * p + i];
                }
            }
            double nrm = 0;
            for (int64_t i = 0; i < p; ++i) nrm = std::hypot(nrm, col[i]);
            if (!(nrm > 0) || !std::isfinite(nrm)) fail(kRuntime, "RBRP block lost orthogonality");
            for (int64_t i = 0; i < p; ++i) col[i] /= nrm;
        }
        // coefficients of the new vectors for every point, and the residual decrease
        ISDF_CUDA(cudaMemcpyAsync(prev_d.get(), chosen.data(), n, cudaMemcpyHostToDevice, s));
        ISDF_CUDA(cudaMemcpyAsync(Q.get() + old * p, qb.data(), qb.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        DeviceBuffer<double> S(static_cast<size_t>(keep) * nao * nao, s);
        rbrp_unpack_kernel<<<static_cast<unsigned>((static_cast<int64_t>(keep) * nao * nao + 255) / 256), 256, 0, s>>>(
            Q.get() + old * p, p, keep, nao, S.get());
        ISDF_LAUNCH_CHECK();
        for (int t = 0; t < keep; ++t)
            for (int64_t g0 = 0; g0 < n; g0 += chunk) {
                const int64_t bb = std::min(chunk, n - g0);
                gemm_f64(bb, nao, nao, ao + g0 * nao, nao, 0, S.get() + static_cast<int64_t>(t) * nao * nao, nao, 0,
                         T.get(), nao, 0, 1, false, s);
                rbrp_rowdot_kernel<<<static_cast<unsigned>((bb * 32 + 255) / 256), 256, 0, s>>>(
                    T.get(), ao, sw.get(), prev_d.get(), g0, bb, nao, L.get(), std::max<int64_t>(cap, 1),
                    static_cast<int>(old + t));
                ISDF_LAUNCH_CHECK();
            }
        rbrp_decrease_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
            L.get(), std::max<int64_t>(cap, 1), static_cast<int>(old), keep, prev_d.get(), n, d_d.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaMemcpyAsync(d.data(), d_d.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        q.insert(q.end(), qb.begin(), qb.end());
        for (int j = 0; j < keep; ++j) {
            if (piv[j] < 0 || piv[j] >= b) fail(kRuntime, "RBRP block returned invalid pivot");
            const int64_t id = sample[piv[j]];
            out.indices.push_back(id);
            chosen[id] = 1;
            d[id] = 0.0;
        }
        ISDF_CUDA(cudaMemcpyAsync(d_d.get(), d.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
        out.history.insert(out.history.end(), {static_cast<double>(out.indices.size()), static_cast<double>(b),
                                               static_cast<double>(keep), total ? std::sqrt(sum_of(d) / total) : 0.0});
        ++iteration;
    }
    const int64_t k = static_cast<int64_t>(out.indices.size());
    refresh(k);
    out.relative_residual = total ? std::sqrt(sum_of(d) / total) : 0.0;
    if (out.relative_residual <= prm.tolerance) out.status = "tolerance";
    else if (out.status == "tolerance") out.status = "roundoff_limited";
    if (!prm.compute_id || k == 0) return out;

    // ---- interpolative decomposition (cpp/src/anchor_select_rbrp.cpp:136-186) ----
    std::vector<double> Lh(static_cast<size_t>(k) * k), swh(n);
    const int64_t ldl = std::max<int64_t>(cap, 1);
    for (int64_t r = 0; r < k; ++r)
        ISDF_CUDA(cudaMemcpyAsync(Lh.data() + r * k, L.get() + out.indices[r] * ldl, k * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(swh.data(), sw.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
    std::vector<double> wa(k);
    for (int64_t a = 0; a < k; ++a)
        ISDF_CUDA(cudaMemcpyAsync(&wa[a], w + out.indices[a], sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    std::vector<double> a(static_cast<size_t>(k) * k), u, sv, vt;
    for (int64_t col = 0; col < k; ++col)
        for (int64_t row = 0; row < k; ++row) a[row + col * k] = Lh[row * k + col];
    small_svd(a, static_cast<int>(k), u, sv, vt);
    out.condition = sv.back() ? sv.front() / sv.back() : std::numeric_limits<double>::infinity();
    for (double x : sv)
        if (x > prm.svd_rtol * sv.front()) ++out.retained_rank;
    if (!out.retained_rank) fail(kRuntime, "RBRP anchor block has zero numerical rank");
    std::vector<double> inv(static_cast<size_t>(k) * k, 0.0);
    for (int64_t i = 0; i < k; ++i)
        for (int64_t j = 0; j < k; ++j)
            for (int64_t t = 0; t < out.retained_rank; ++t) inv[i * k + j] += vt[t + i * k] * u[j + t * k] / sv[t];
    std::vector<double> fac(k);
    for (int64_t aa = 0; aa < k; ++aa) fac[aa] = swh[out.indices[aa]] / wa[aa];
    DeviceBuffer<double> dinv(inv.size(), s), dfac(k, s), dout(static_cast<size_t>(k) * n, s);
    ISDF_CUDA(cudaMemcpyAsync(dinv.get(), inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaMemcpyAsync(dfac.get(), fac.data(), k * sizeof(double), cudaMemcpyHostToDevice, s));
    rbrp_interp_kernel<<<static_cast<unsigned>((k * n + 255) / 256), 256, 0, s>>>(
        L.get(), ldl, static_cast<int>(k), dinv.get(), dfac.get(), sw.get(), n, dout.get());
    ISDF_LAUNCH_CHECK();
    out.interp_vecs.resize(static_cast<size_t>(k) * n);
    ISDF_CUDA(cudaMemcpyAsync(out.interp_vecs.data(), dout.get(), out.interp_vecs.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    // the cardinality condition, imposed after any SVD clipping
    for (int64_t aa = 0; aa < k; ++aa)
        for (int64_t bb = 0; bb < k; ++bb)
            out.interp_vecs[aa * n + out.indices[bb]] = aa == bb ? 1.0 / wa[bb] : 0.0;
    out.transform.assign(static_cast<size_t>(k) * nao * nao, 0.0);
    int64_t packed = 0;
    for (int mu = 0; mu < nao; ++mu)
        for (int nu = mu; nu < nao; ++nu, ++packed)
            for (int64_t aa = 0; aa < k; ++aa) {
                double value = 0;
                for (int64_t t = 0; t < k; ++t) value += inv[t * k + aa] * q[t * p + packed];
                value *= fac[aa];
                if (mu != nu) value /= kSqrt2;
                out.transform[aa * nao * nao + mu * nao + nu] = value;
                out.transform[aa * nao * nao + nu * nao + mu] = value;
            }
    return out;
}

}  // namespace isdf
