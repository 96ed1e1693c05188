// qrcp_dense / qrcp_online anchor selection on the weighted AO-pair columns
// a_g = sqrt|w_g| f_g (x) f_g without materialising the d^2 x n pair matrix.
//
// The greedy rule of column-pivoted QR (dgeqp3 for qrcp_dense,
// cpp/src/anchor_select_qrcp.cpp:275-306; the multipass selector of
// cpp/src/anchor_select_online_qr.cpp:200-358 for qrcp_online) selects at
// each step the column with the largest residual norm after projection onto
// the span of the previous pivots.  Here:
//   * residual estimates e_g = K_gg - sum_i L_gi^2 use the pair Gram
//     K_pg = sqrt|w_p w_g| (f_p . f_g)^2: one GEMV over the feature matrix per
//     pivot, L_gj = (K_pg - sum_{i<j} R_ij L_gi) / R_jj;
//   * the leading candidate is always re-verified exactly: its explicit pair
//     vector is orthogonalised twice (CGS2) against the explicit orthonormal
//     pivot basis, giving R[:, j] with Householder-level accuracy.  If the
//     exact value loses the lead, the next candidate is verified (the online
//     reference's reselection loop, online_qr.cpp:238-254);
//   * a stop decided on an estimate is confirmed by an exact scan of every
//     column whose estimate, within its rounding bound, could still exceed
//     the threshold ("no optimistic estimate may terminate", online_qr.cpp:233).
// Tie-breaking: qrcp_dense emulates dgeqp3's column swaps (first maximum in
// the current column order); qrcp_online takes the first maximum in grid order.
#include "isdf_reduce.cuh"
#include "isdf_select.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace isdf {
namespace {

constexpr int kNT = 256;

__global__ void gather_weights_kernel(const double* __restrict__ w, const int64_t* __restrict__ idx,
                                      int64_t n, double* __restrict__ sw) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g < n) sw[g] = sqrt(fabs(w[idx[g]]));
}

// The multi-axis scales are applied where F is read instead of in F itself
// (a pass over n x d values saved): cs[j] = scale of column j's axis entry.
__global__ void column_scales_kernel(AxisSpec ax, const double* __restrict__ scales, int64_t d,
                                     double* __restrict__ cs) {
    const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= d) return;
    int a = 0;
    while (a + 1 < ax.naxes && j >= ax.offset[a + 1]) ++a;
    cs[j] = scales[a];
}

// warp per row: nf[g] = sum_k (cs[k] F[g,k])^2
__global__ void scaled_row_norms_kernel(const double* __restrict__ F, int64_t n, int64_t d,
                                        const double* __restrict__ cs, double* __restrict__ nf) {
    const int64_t g = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x % 32;
    if (g >= n) return;
    const double* row = F + g * d;
    double acc = 0;
    for (int64_t k = lane; k < d; k += 32) {
        const double v = cs[k] * row[k];
        acc += v * v;
    }
    acc = warp_sum(acc);
    if (lane == 0) nf[g] = acc;
}

// x[k] = cs[k]^2 F[p,k]: with it, F x is the Gram row of the scaled features
__global__ void scaled_pivot_row_kernel(const double* __restrict__ fp, const double* __restrict__ cs, int64_t d,
                                        double* __restrict__ x) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < d) x[k] = cs[k] * cs[k] * fp[k];
}

__global__ void init_est_kernel(const double* __restrict__ sw, const double* __restrict__ nf,
                                int64_t n, double* __restrict__ est, double* __restrict__ kdiag) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double a = sw[g] * nf[g];
    est[g] = a * a;
    kdiag[g] = a * a;
}

// est argmax over unselected columns -> per-block keys (value = estimate of the
// squared residual norm).
__global__ void __launch_bounds__(kNT)
argmax_kernel(const double* __restrict__ est, const char* __restrict__ selected,
              const int64_t* __restrict__ pos, int64_t n, ArgKey* __restrict__ partial) {
    __shared__ ArgKey sh[kNT / 32];
    const int64_t g = static_cast<int64_t>(blockIdx.x) * kNT + threadIdx.x;
    ArgKey k = key_none();
    if (g < n && !selected[g]) k = ArgKey{est[g], pos ? pos[g] : g, g};
    k = block_best<kNT>(k, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = k;
}

__global__ void __launch_bounds__(1024)
argmax_final_kernel(const ArgKey* __restrict__ partial, int nblocks, ArgKey* __restrict__ out) {
    __shared__ ArgKey sh[32];
    ArgKey k = key_none();
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        if (key_better(partial[b], k)) k = partial[b];
    k = block_best<1024>(k, sh);
    if (threadIdx.x == 0) out[0] = k;
}

// L[g, j] = (sw_p sw_g D_g^2 - sum_{i<j} R_ij L_gi) / R_jj ; est_g -= L_gj^2
__global__ void update_residual_kernel(const double* __restrict__ D, const double* __restrict__ sw,
                                       int64_t p, int64_t n, double* __restrict__ L,
                                       int64_t ldl, int j, const double* __restrict__ Rcol,
                                       double rjj, double* __restrict__ est,
                                       const char* __restrict__ selected) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    double v = sw[p] * sw[g] * D[g] * D[g];
    const double* lg = L + g * ldl;
    for (int i = 0; i < j; ++i) v -= Rcol[i] * lg[i];
    v /= rjj;
    L[g * ldl + j] = v;
    if (!selected[g]) est[g] = fmax(est[g] - v * v, 0.0);
}

// a[i*d + k] = sw[p] f[i] f[k]: the weighted pair vector of column p (f
// scaled by cs where the axis entries carry scales)
__global__ void pair_vector_sw_kernel(const double* __restrict__ f, int64_t d, const double* __restrict__ sw,
                                      int64_t p, const double* __restrict__ cs, double* __restrict__ a) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= d * d) return;
    const int64_t r = i / d, c = i % d;
    a[i] = cs ? sw[p] * (cs[r] * f[r]) * (cs[c] * f[c]) : sw[p] * f[r] * f[c];
}

// est[p] = the exact squared residual just computed
__global__ void set_est_kernel(double* __restrict__ est, int64_t p, const double* __restrict__ scal) {
    est[p] = scal[0];
}

// column j of R: the two CGS passes' coefficients and R_jj = |r|
__global__ void rcol_kernel(const double* __restrict__ t0, const double* __restrict__ t1, int j,
                            const double* __restrict__ scal, double* __restrict__ Rcol) {
    for (int i = threadIdx.x; i <= j; i += blockDim.x) Rcol[i] = i < j ? t0[i] + t1[i] : sqrt(scal[0]);
}

// per-block sums of K_gg and a non-finite flag (fixed order: deterministic)
__global__ void __launch_bounds__(256) kdiag_partial_kernel(const double* __restrict__ kd, int64_t n,
                                                            double* __restrict__ part, int* __restrict__ bad) {
    __shared__ double sh[256 / 32];
    const int64_t g = static_cast<int64_t>(blockIdx.x) * 256 + threadIdx.x;
    double v = 0.0;
    if (g < n) {
        v = kd[g];
        if (!isfinite(v)) atomicOr(bad, 1);
    }
    v = block_sum<256>(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void __launch_bounds__(256) sum_partials_kernel(const double* __restrict__ part, int nb,
                                                           double* __restrict__ out) {
    __shared__ double sh[256 / 32];
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += 256) v += part[b];
    v = block_sum<256>(v, sh);
    if (threadIdx.x == 0) out[0] = v;
}

__global__ void gather_index_kernel(const int64_t* __restrict__ index, const int64_t* __restrict__ pos, int k,
                                    int64_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) out[i] = index[pos[i]];
}

// ---- fixed-order reductions (the sharded QR needs bit-identical results on
// every rank): per-block partials, then one block per output in block order
constexpr int kDetBlocks = 256;

// part[r * kDetBlocks + b] = sum over block b's slice of Q[r, :] . x
__global__ void __launch_bounds__(256) rows_dot_part_kernel(const double* __restrict__ Q, int rows, int64_t m,
                                                            const double* __restrict__ x, double* __restrict__ part) {
    __shared__ double sh[256 / 32];
    const int64_t chunk = (m + gridDim.x - 1) / gridDim.x;
    const int64_t k0 = blockIdx.x * chunk, k1 = min(m, k0 + chunk);
    for (int r = 0; r < rows; ++r) {
        double acc = 0;
        const double* q = Q + static_cast<int64_t>(r) * m;
        for (int64_t k = k0 + threadIdx.x; k < k1; k += 256) acc += q[k] * x[k];
        acc = block_sum<256>(acc, sh);
        if (threadIdx.x == 0) part[r * kDetBlocks + blockIdx.x] = acc;
    }
}

// y = x - Q^T t (elementwise); part[b] = block b's sum of y^2
__global__ void __launch_bounds__(256) rows_axpy_part_kernel(const double* __restrict__ Q, int rows, int64_t m,
                                                             const double* __restrict__ t, const double* x, double* y,
                                                             double* __restrict__ part) {
    __shared__ double sh[256 / 32];
    double acc = 0;
    const int64_t chunk = (m + gridDim.x - 1) / gridDim.x;
    const int64_t k0 = blockIdx.x * chunk, k1 = min(m, k0 + chunk);
    for (int64_t k = k0 + threadIdx.x; k < k1; k += 256) {
        double v = x[k];
        for (int r = 0; r < rows; ++r) v -= Q[static_cast<int64_t>(r) * m + k] * t[r];
        y[k] = v;
        acc += v * v;
    }
    acc = block_sum<256>(acc, sh);
    if (threadIdx.x == 0 && part) part[blockIdx.x] = acc;
}

// out[r] = sum_b part[r * kDetBlocks + b], in block order per thread, then a fixed tree
__global__ void __launch_bounds__(256) reduce_parts_kernel(const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sh[256 / 32];
    double v = 0;
    for (int b = threadIdx.x; b < kDetBlocks; b += 256) v += part[blockIdx.x * kDetBlocks + b];
    v = block_sum<256>(v, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
}

// L[g, j] and the downdate, with the pivot's weight from a device scalar
__global__ void update_residual_swp_kernel(const double* __restrict__ D, const double* __restrict__ sw,
                                           const double* __restrict__ swp, int64_t n, double* __restrict__ L,
                                           int64_t ldl, int j, const double* __restrict__ Rcol, double rjj,
                                           double* __restrict__ est, const char* __restrict__ selected) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    double v = swp[0] * sw[g] * D[g] * D[g];
    const double* lg = L + g * ldl;
    for (int i = 0; i < j; ++i) v -= Rcol[i] * lg[i];
    v /= rjj;
    L[g * ldl + j] = v;
    if (!selected[g]) est[g] = fmax(est[g] - v * v, 0.0);
}

// dgeqp3's swap over shards: the local column at position j takes the winner's
// old position, the winner (if local) takes j
__global__ void shard_swap_pos_kernel(int64_t* __restrict__ pos, int64_t n, int64_t j, int64_t winner_pos,
                                      int64_t winner_local) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    if (g == winner_local) pos[g] = j;
    else if (pos[g] == j) pos[g] = winner_pos;
}

__global__ void pos_iota_kernel(int64_t* __restrict__ pos, int64_t n, int64_t offset) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g < n) pos[g] = offset + g;
}

// row buffer of column p: its d features and sqrt|w_p|
__global__ void export_row_kernel(const double* __restrict__ F, int64_t d, const double* __restrict__ sw, int64_t p,
                                  double* __restrict__ row) {
    for (int64_t k = threadIdx.x; k <= d; k += blockDim.x) row[k] = k < d ? F[p * d + k] : sw[p];
}

}  // namespace

namespace {

struct PairQr {
    const Context& c;
    cudaStream_t s;
    int64_t n = 0, d = 0, m = 0;
    DeviceBuffer<double> F, sw, nf, est, kdiag, D, L, Q, a, r, t0, t1, scal, Rcol, cs, xp;
    DeviceBuffer<char> selected;
    DeviceBuffer<int64_t> pos;
    DeviceBuffer<ArgKey> partial, best;
    int64_t capL = 0;
    int nblocks = 0;
    PairQr(const Context& ctx, cudaStream_t st) : c(ctx), s(st) {}

    void argmax_launch(bool use_pos) {
        argmax_kernel<<<nblocks, kNT, 0, s>>>(est.get(), selected.get(),
                                              use_pos ? pos.get() : nullptr, n, partial.get());
        ISDF_LAUNCH_CHECK();
        argmax_final_kernel<<<1, 1024, 0, s>>>(partial.get(), nblocks, best.get());
        ISDF_LAUNCH_CHECK();
    }
    ArgKey argmax(bool use_pos) {
        argmax_launch(use_pos);
        ArgKey h;
        ISDF_CUDA(cudaMemcpyAsync(&h, best.get(), sizeof(ArgKey), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        return h;
    }

    // Exact residual of column p against the j current basis vectors, on the
    // device: the residual in r, the two CGS passes' coefficients in t0 and
    // t1, |r|^2 in scal, and est[p] = |r|^2.
    void exact_residual_launch(int64_t p, int j) {
        pair_vector_sw_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, s>>>(
            F.get() + p * d, d, sw.get(), p, cs.get(), a.get());
        ISDF_LAUNCH_CHECK();
        scal.zero(s);
        if (j == 0) {
            rows_axpy(Q.get(), 0, m, t0.get(), a.get(), r.get(), scal.get(), s);
        } else {
            t0.zero(s);
            rows_dot(Q.get(), j, m, a.get(), t0.get(), s);
            rows_axpy(Q.get(), j, m, t0.get(), a.get(), r.get(), nullptr, s);
            t1.zero(s);
            rows_dot(Q.get(), j, m, r.get(), t1.get(), s);
            rows_axpy(Q.get(), j, m, t1.get(), r.get(), r.get(), scal.get(), s);
        }
        set_est_kernel<<<1, 1, 0, s>>>(est.get(), p, scal.get());
        ISDF_LAUNCH_CHECK();
    }
    double exact_residual(int64_t p, int j) {
        exact_residual_launch(p, j);
        double nr2 = 0;
        ISDF_CUDA(cudaMemcpyAsync(&nr2, scal.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        return nr2;
    }
    // exact residual of p, then the argmax over the updated estimates: one
    // host round trip for both
    ArgKey verify(int64_t p, int j, bool use_pos, double& exact2) {
        exact_residual_launch(p, j);
        argmax_launch(use_pos);
        ArgKey h;
        ISDF_CUDA(cudaMemcpyAsync(&h, best.get(), sizeof(ArgKey), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaMemcpyAsync(&exact2, scal.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        return h;
    }

    void grow(int64_t need) {
        if (need <= capL) return;
        const int64_t cap2 = std::max<int64_t>(need, std::max<int64_t>(8, 2 * capL));
        DeviceBuffer<double> L2(static_cast<size_t>(n * cap2), s), Q2(static_cast<size_t>(cap2 * m), s),
            t02(cap2, s), t12(cap2, s);
        if (capL) {
            if (n > 0)   // a shard may hold no kept point
                ISDF_CUDA(cudaMemcpy2DAsync(L2.get(), cap2 * sizeof(double), L.get(), capL * sizeof(double),
                                            capL * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
            ISDF_CUDA(cudaMemcpyAsync(Q2.get(), Q.get(), capL * m * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s));
            // the coefficients of the column being accepted
            ISDF_CUDA(cudaMemcpyAsync(t02.get(), t0.get(), capL * sizeof(double), cudaMemcpyDeviceToDevice, s));
            ISDF_CUDA(cudaMemcpyAsync(t12.get(), t1.get(), capL * sizeof(double), cudaMemcpyDeviceToDevice, s));
        }
        L = std::move(L2);
        Q = std::move(Q2);
        t0 = std::move(t02);
        t1 = std::move(t12);
        capL = cap2;
        Rcol.reset(capL, s);
    }
};

__global__ void swap_positions_kernel(int64_t* pos, int64_t* col_at, int64_t p, int64_t j) {
    const int64_t pp = pos[p];
    const int64_t cj = col_at[j];
    col_at[pp] = cj;
    pos[cj] = pp;
    col_at[j] = p;
    pos[p] = j;
}

__global__ void mark_selected_kernel(char* selected, double* est, int64_t p) {
    selected[p] = 1;
    est[p] = 0.0;
}

// exact-scan candidates: unselected g with est_g + bound_g > thr2
__global__ void flag_uncertain_kernel(const double* __restrict__ est, const double* __restrict__ kdiag,
                                      const char* __restrict__ selected, int64_t n, double rel,
                                      double thr2, char* __restrict__ flag) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    flag[g] = !selected[g] && est[g] + rel * kdiag[g] > thr2;
}

}  // namespace

std::vector<int64_t> select_pair_qr(const Context& c, const double* pts, const double* w,
                                    int64_t ng, const SelectOptions& o, cudaStream_t s,
                                    PairQrDiagnostics* diag) {
    const bool online = o.algorithm == 1;
    if (!std::isfinite(o.tolerance) || o.tolerance < 0 || (online && o.batch_size <= 0))
        fail(kInvalid, online ? "invalid online QR weights, tolerance or batch size"
                              : "invalid weights, axis list, or tolerance");
    validate_axis_weights(o.axis_weights.empty() ? nullptr : o.axis_weights.data(),
                          static_cast<int>(o.axes.size()));
    AxisSetup axs = make_axis_setup(c, o, s);
    const AxisSpec& ax = axs.ax;
    const int64_t d = ax.d;
    if (d > 46340)
        fail(kOverflow, online ? "AO pair dimension is too large" : "pair-product matrix is too large");
    KeptPoints kp = compact_points(pts, w, ng, s);
    const int64_t n = kp.n;
    if (n == 0) return {};

    PairQr q(c, s);
    q.n = n; q.d = d; q.m = d * d;
    const int64_t m = q.m;
    q.nblocks = static_cast<int>((n + kNT - 1) / kNT);
    q.F.reset(static_cast<size_t>(n * d), s);
    DeviceBuffer<double> sumsq(5, s);
    sumsq.zero(s);
    eval_axis_features<double>(c, pts, kp.index.get(), n, ax, q.F.get(), d,
                               ax.naxes > 1 ? sumsq.get() : nullptr, nullptr, s);
    if (ax.naxes > 1) {
        double h[5];
        ISDF_CUDA(cudaMemcpyAsync(h, sumsq.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        auto sc = axis_scales_from_sumsq(ax, h, o.axis_weights.empty() ? nullptr : o.axis_weights.data(), true);
        DeviceBuffer<double> dsc(sc.size(), s);
        ISDF_CUDA(cudaMemcpyAsync(dsc.get(), sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        q.cs.reset(d, s);
        q.xp.reset(d, s);
        column_scales_kernel<<<static_cast<unsigned>((d + 255) / 256), 256, 0, s>>>(ax, dsc.get(), d, q.cs.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaStreamSynchronize(s));   // host scales go out of scope
    }
    const unsigned nb = static_cast<unsigned>((n + 255) / 256);
    q.sw.reset(n, s); q.nf.reset(n, s); q.est.reset(n, s); q.kdiag.reset(n, s); q.D.reset(n, s);
    q.selected.reset(n, s); q.selected.zero(s);
    q.pos.reset(n, s);
    DeviceBuffer<int64_t> col_at(n, s);
    iota_i64(q.pos.get(), n, s);
    iota_i64(col_at.get(), n, s);
    q.partial.reset(q.nblocks, s);
    q.best.reset(1, s);
    q.a.reset(m, s); q.r.reset(m, s); q.scal.reset(1, s);
    DeviceBuffer<double> kpart(q.nblocks, s), ksum(1, s);
    DeviceBuffer<int> kbad(1, s);
    kbad.zero(s);
    gather_weights_kernel<<<nb, 256, 0, s>>>(w, kp.index.get(), n, q.sw.get());
    ISDF_LAUNCH_CHECK();
    if (q.cs.get()) {
        scaled_row_norms_kernel<<<static_cast<unsigned>((n * 32 + 255) / 256), 256, 0, s>>>(q.F.get(), n, d,
                                                                                          q.cs.get(), q.nf.get());
        ISDF_LAUNCH_CHECK();
    } else {
        row_dot(q.F.get(), n, d, nullptr, q.nf.get(), s);
    }
    init_est_kernel<<<nb, 256, 0, s>>>(q.sw.get(), q.nf.get(), n, q.est.get(), q.kdiag.get());
    ISDF_LAUNCH_CHECK();
    {
        // sum of K_gg (the squared Frobenius norm of the pair matrix) and its finiteness
        kdiag_partial_kernel<<<q.nblocks, 256, 0, s>>>(q.kdiag.get(), n, kpart.get(), kbad.get());
        ISDF_LAUNCH_CHECK();
        sum_partials_kernel<<<1, 256, 0, s>>>(kpart.get(), q.nblocks, ksum.get());
        ISDF_LAUNCH_CHECK();
        double frob2 = 0;
        int hbad = 0;
        ISDF_CUDA(cudaMemcpyAsync(&frob2, ksum.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaMemcpyAsync(&hbad, kbad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        if (hbad || !std::isfinite(frob2))
            fail(kOverflow, online ? "non-finite online AO pair column" : "non-finite weighted pair product");
        if (diag) diag->floor = 32 * std::numeric_limits<double>::epsilon() * std::sqrt(frob2);
        q.grow(8);
        const int64_t cap = std::min({m, n, o.max_rank ? o.max_rank : std::min(m, n)});
        const double eps = std::numeric_limits<double>::epsilon();
        const double floor = online ? 32 * eps * std::sqrt(frob2) : 0.0;
        std::vector<int64_t> result;
        double first = -1;
        int64_t verifications = 0, reselections = 0, exact_scans = 0;
        DeviceBuffer<char> flags(n, s);
        std::vector<char> hflags;
        bool exact_mode = false;   // every estimate in `est` is exact (after a scan)
        while (true) {
            const int j = static_cast<int>(result.size());
            if (j == cap) break;
            ArgKey k = q.argmax(!online);
            if (k.col < 0) break;
            // verification loop: the leader's exact residual, then the argmax
            // over the updated estimates (one host round trip per candidate)
            double exact2 = 0;
            while (true) {
                const ArgKey k2 = q.verify(k.col, j, !online, exact2);
                ++verifications;
                if (k2.col == k.col) break;
                ++reselections;
                k = k2;
            }
            const double rjj = std::sqrt(exact2);
            if (first < 0) first = rjj;   // R_00: the largest column norm
            const double thr = std::max(o.tolerance * first, floor);
            const bool stop = first == 0 || rjj <= thr || (online && rjj <= floor);
            if (stop) {
                if (exact_mode) break;
                // confirm on exact values: scan every column that could still exceed thr
                const double rel = 64.0 * eps * static_cast<double>(j + 1);
                flag_uncertain_kernel<<<nb, 256, 0, s>>>(q.est.get(), q.kdiag.get(), q.selected.get(),
                                                          n, rel, thr * thr, flags.get());
                ISDF_LAUNCH_CHECK();
                hflags.resize(n);
                ISDF_CUDA(cudaMemcpyAsync(hflags.data(), flags.get(), n, cudaMemcpyDeviceToHost, s));
                ISDF_CUDA(cudaStreamSynchronize(s));
                ++exact_scans;
                for (int64_t g = 0; g < n; ++g)
                    if (hflags[g]) q.exact_residual_launch(g, j);   // also sets est[g]
                exact_mode = true;
                k = q.argmax(!online);
                if (k.col < 0) break;
                exact2 = q.exact_residual(k.col, j);
                const double r2 = std::sqrt(exact2);
                if (first == 0 || r2 <= thr) break;
            }
            // accept pivot k.col
            const int64_t p = k.col;
            const double rj = std::sqrt(exact2);
            q.grow(j + 1);
            rcol_kernel<<<1, 64, 0, s>>>(q.t0.get(), q.t1.get(), j, q.scal.get(), q.Rcol.get());
            ISDF_LAUNCH_CHECK();
            scale_copy(q.r.get(), 1.0 / rj, m, q.Q.get() + static_cast<int64_t>(j) * m, s);
            mark_selected_kernel<<<1, 1, 0, s>>>(q.selected.get(), q.est.get(), p);
            ISDF_LAUNCH_CHECK();
            if (!online) {
                swap_positions_kernel<<<1, 1, 0, s>>>(q.pos.get(), col_at.get(), p, j);
                ISDF_LAUNCH_CHECK();
            }
            // new column of L and downdated estimates
            const double* xrow = q.F.get() + p * d;
            if (q.cs.get()) {
                scaled_pivot_row_kernel<<<static_cast<unsigned>((d + 255) / 256), 256, 0, s>>>(xrow, q.cs.get(), d,
                                                                                             q.xp.get());
                ISDF_LAUNCH_CHECK();
                xrow = q.xp.get();
            }
            row_dot(q.F.get(), n, d, xrow, q.D.get(), s);
            update_residual_kernel<<<nb, 256, 0, s>>>(q.D.get(), q.sw.get(), p, n, q.L.get(), q.capL,
                                                      j, q.Rcol.get(), rj, q.est.get(), q.selected.get());
            ISDF_LAUNCH_CHECK();
            exact_mode = false;   // downdated estimates carry rounding again
            result.push_back(p);
            if (diag) diag->rdiag.push_back(rj);
        }
        // grid indices of the pivots
        std::vector<int64_t> out(result.size());
        if (!result.empty()) {
            DeviceBuffer<int64_t> dres(result.size(), s), dout(result.size(), s);
            ISDF_CUDA(cudaMemcpyAsync(dres.get(), result.data(), result.size() * sizeof(int64_t),
                                      cudaMemcpyHostToDevice, s));
            gather_index_kernel<<<static_cast<unsigned>((result.size() + 255) / 256), 256, 0, s>>>(
                kp.index.get(), dres.get(), static_cast<int>(result.size()), dout.get());
            ISDF_LAUNCH_CHECK();
            ISDF_CUDA(cudaMemcpyAsync(out.data(), dout.get(), out.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                                      s));
        }
        ISDF_CUDA(cudaStreamSynchronize(s));
        if (diag) {
            diag->rank = static_cast<int64_t>(out.size());
            diag->verifications = verifications;
            diag->reselections = reselections;
            diag->exact_scans = exact_scans;
            diag->first = first;
        }
        return out;
    }
}

// ---- the pair QR over grid shards -------------------------------------------------
struct PairQrShard::Impl {
    const Context& c;
    cudaStream_t s;
    SelectOptions o;
    AxisSetup axs;
    KeptPoints kp;
    PairQr q;
    const double* pts = nullptr;
    const double* w = nullptr;
    int64_t grid_offset = 0, pos_offset = 0;
    double sumsq[5] = {0, 0, 0, 0, 0};
    DeviceBuffer<double> rowbuf, part;
    Impl(const Context& ctx, const SelectOptions& opt, cudaStream_t st) : c(ctx), s(st), o(opt), q(ctx, st) {}

    void ensure(int64_t rows) {
        q.grow(rows);
        if (part.size() < static_cast<size_t>(kDetBlocks) * q.capL) part.reset(static_cast<size_t>(kDetBlocks) * q.capL, s);
    }
    // CGS2 of the pair vector of the row in rowbuf against the j basis vectors,
    // in fixed reduction order: r, t0, t1 and scal = |r|^2
    void exact_residual(int j) {
        const int64_t m = q.m, d = q.d;
        pair_vector_sw_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, s>>>(rowbuf.get(), d,
                                                                                    rowbuf.get() + d, 0,
                                                                                    q.cs.get(), q.a.get());
        ISDF_LAUNCH_CHECK();
        if (j == 0) {
            rows_axpy_part_kernel<<<kDetBlocks, 256, 0, s>>>(q.Q.get(), 0, m, q.t0.get(), q.a.get(), q.r.get(),
                                                             part.get());
            ISDF_LAUNCH_CHECK();
        } else {
            rows_dot_part_kernel<<<kDetBlocks, 256, 0, s>>>(q.Q.get(), j, m, q.a.get(), part.get());
            ISDF_LAUNCH_CHECK();
            reduce_parts_kernel<<<j, 256, 0, s>>>(part.get(), q.t0.get());
            ISDF_LAUNCH_CHECK();
            rows_axpy_part_kernel<<<kDetBlocks, 256, 0, s>>>(q.Q.get(), j, m, q.t0.get(), q.a.get(), q.r.get(),
                                                             nullptr);
            ISDF_LAUNCH_CHECK();
            rows_dot_part_kernel<<<kDetBlocks, 256, 0, s>>>(q.Q.get(), j, m, q.r.get(), part.get());
            ISDF_LAUNCH_CHECK();
            reduce_parts_kernel<<<j, 256, 0, s>>>(part.get(), q.t1.get());
            ISDF_LAUNCH_CHECK();
            rows_axpy_part_kernel<<<kDetBlocks, 256, 0, s>>>(q.Q.get(), j, m, q.t1.get(), q.r.get(), q.r.get(),
                                                             part.get());
            ISDF_LAUNCH_CHECK();
        }
        reduce_parts_kernel<<<1, 256, 0, s>>>(part.get(), q.scal.get());
        ISDF_LAUNCH_CHECK();
    }
    int64_t local(int64_t gcol) const {
        const int64_t l = gcol - pos_offset;
        return (gcol >= 0 && l >= 0 && l < q.n) ? l : -1;
    }
    void upload_row(const double* row_host) {
        ISDF_CUDA(cudaMemcpyAsync(rowbuf.get(), row_host, (q.d + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
    }
};

PairQrShard::PairQrShard(const Context& c, const SelectOptions& o, const double* pts, const double* w, int64_t ng,
                         int64_t grid_offset, cudaStream_t s)
    : p_(new Impl(c, o, s)) {
    Impl& I = *p_;
    const bool online = o.algorithm == 1;
    if (!std::isfinite(o.tolerance) || o.tolerance < 0 || (online && o.batch_size <= 0))
        fail(kInvalid, online ? "invalid online QR weights, tolerance or batch size"
                              : "invalid weights, axis list, or tolerance");
    validate_axis_weights(o.axis_weights.empty() ? nullptr : o.axis_weights.data(), static_cast<int>(o.axes.size()));
    I.axs = make_axis_setup(c, o, s);
    const int64_t d = I.axs.ax.d;
    if (d > 46340) fail(kOverflow, online ? "AO pair dimension is too large" : "pair-product matrix is too large");
    I.pts = pts;
    I.w = w;
    I.grid_offset = grid_offset;
    I.kp = compact_points(pts, w, ng, s);
    PairQr& q = I.q;
    q.n = I.kp.n; q.d = d; q.m = d * d;
    q.nblocks = static_cast<int>(std::max<int64_t>(1, (q.n + kNT - 1) / kNT));
    q.F.reset(static_cast<size_t>(std::max<int64_t>(q.n, 1) * d), s);
    DeviceBuffer<double> sq(5, s);
    sq.zero(s);
    if (q.n > 0)
        eval_axis_features<double>(c, pts, I.kp.index.get(), q.n, I.axs.ax, q.F.get(), d,
                                   I.axs.ax.naxes > 1 ? sq.get() : nullptr, nullptr, s);
    ISDF_CUDA(cudaMemcpyAsync(I.sumsq, sq.get(), sizeof(I.sumsq), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
}

PairQrShard::~PairQrShard() { delete p_; }
int64_t PairQrShard::n_kept() const { return p_->q.n; }
int64_t PairQrShard::features() const { return p_->q.d; }
void PairQrShard::local_sumsq(double out[5]) const { std::memcpy(out, p_->sumsq, sizeof(p_->sumsq)); }

void PairQrShard::init(const double* sumsq_global, int64_t pos_offset, double out[2]) {
    Impl& I = *p_;
    PairQr& q = I.q;
    cudaStream_t s = I.s;
    const int64_t n = q.n, d = q.d;
    I.pos_offset = pos_offset;
    const AxisSpec& ax = I.axs.ax;
    if (ax.naxes > 1) {
        // every rank derives the same scales from the same global sums
        auto sc = axis_scales_from_sumsq(ax, sumsq_global,
                                         I.o.axis_weights.empty() ? nullptr : I.o.axis_weights.data(), true);
        DeviceBuffer<double> dsc(sc.size(), s);
        ISDF_CUDA(cudaMemcpyAsync(dsc.get(), sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        q.cs.reset(d, s);
        q.xp.reset(d, s);
        column_scales_kernel<<<static_cast<unsigned>((d + 255) / 256), 256, 0, s>>>(ax, dsc.get(), d, q.cs.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaStreamSynchronize(s));
    }
    const int64_t nn = std::max<int64_t>(n, 1);
    q.sw.reset(nn, s); q.nf.reset(nn, s); q.est.reset(nn, s); q.kdiag.reset(nn, s); q.D.reset(nn, s);
    q.selected.reset(nn, s); q.selected.zero(s);
    q.pos.reset(nn, s);
    q.partial.reset(q.nblocks, s);
    q.best.reset(1, s);
    q.a.reset(q.m, s); q.r.reset(q.m, s); q.scal.reset(1, s);
    I.rowbuf.reset(d + 1, s);
    I.ensure(8);
    out[0] = 0.0;
    out[1] = 0.0;
    if (n > 0) {
        const unsigned nb = static_cast<unsigned>((n + 255) / 256);
        pos_iota_kernel<<<nb, 256, 0, s>>>(q.pos.get(), n, pos_offset);
        ISDF_LAUNCH_CHECK();
        gather_weights_kernel<<<nb, 256, 0, s>>>(I.w, I.kp.index.get(), n, q.sw.get());
        ISDF_LAUNCH_CHECK();
        if (q.cs.get()) {
            scaled_row_norms_kernel<<<static_cast<unsigned>((n * 32 + 255) / 256), 256, 0, s>>>(q.F.get(), n, d,
                                                                                              q.cs.get(), q.nf.get());
            ISDF_LAUNCH_CHECK();
        } else {
            row_dot(q.F.get(), n, d, nullptr, q.nf.get(), s);
        }
        init_est_kernel<<<nb, 256, 0, s>>>(q.sw.get(), q.nf.get(), n, q.est.get(), q.kdiag.get());
        ISDF_LAUNCH_CHECK();
        DeviceBuffer<double> kpart(q.nblocks, s), ksum(1, s);
        DeviceBuffer<int> kbad(1, s);
        kbad.zero(s);
        kdiag_partial_kernel<<<q.nblocks, 256, 0, s>>>(q.kdiag.get(), n, kpart.get(), kbad.get());
        ISDF_LAUNCH_CHECK();
        sum_partials_kernel<<<1, 256, 0, s>>>(kpart.get(), q.nblocks, ksum.get());
        ISDF_LAUNCH_CHECK();
        int hbad = 0;
        ISDF_CUDA(cudaMemcpyAsync(&out[0], ksum.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaMemcpyAsync(&hbad, kbad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        out[1] = hbad ? 1.0 : 0.0;
    }
}

void PairQrShard::argmax(double key[3]) {
    Impl& I = *p_;
    PairQr& q = I.q;
    key[0] = -1.0; key[1] = -1.0; key[2] = -1.0;
    if (q.n == 0) return;
    const ArgKey k = q.argmax(true);
    if (k.col < 0) return;
    key[0] = k.v;
    key[1] = static_cast<double>(k.pos);
    key[2] = static_cast<double>(I.pos_offset + k.col);
}

void PairQrShard::row(int64_t gcol, double* out) const {
    const Impl& I = *p_;
    const PairQr& q = I.q;
    const int64_t l = I.local(gcol);
    require(l >= 0, "the column is not on this shard");
    DeviceBuffer<double> buf(q.d + 1, I.s);
    export_row_kernel<<<1, 256, 0, I.s>>>(q.F.get(), q.d, q.sw.get(), l, buf.get());
    ISDF_LAUNCH_CHECK();
    int64_t gi = 0;
    ISDF_CUDA(cudaMemcpyAsync(out, buf.get(), (q.d + 1) * sizeof(double), cudaMemcpyDeviceToHost, I.s));
    ISDF_CUDA(cudaMemcpyAsync(&gi, I.kp.index.get() + l, sizeof(int64_t), cudaMemcpyDeviceToHost, I.s));
    ISDF_CUDA(cudaStreamSynchronize(I.s));
    double xyzw[4];
    ISDF_CUDA(cudaMemcpyAsync(xyzw, I.pts + 3 * gi, 3 * sizeof(double), cudaMemcpyDeviceToHost, I.s));
    ISDF_CUDA(cudaMemcpyAsync(xyzw + 3, I.w + gi, sizeof(double), cudaMemcpyDeviceToHost, I.s));
    ISDF_CUDA(cudaStreamSynchronize(I.s));
    out[q.d + 1] = static_cast<double>(I.grid_offset + gi);
    for (int i = 0; i < 4; ++i) out[q.d + 2 + i] = xyzw[i];
}

double PairQrShard::verify(const double* row_host, int j, int64_t gcol) {
    Impl& I = *p_;
    PairQr& q = I.q;
    I.ensure(j + 1);
    I.upload_row(row_host);
    I.exact_residual(j);
    const int64_t l = I.local(gcol);
    if (l >= 0) {
        set_est_kernel<<<1, 1, 0, I.s>>>(q.est.get(), l, q.scal.get());
        ISDF_LAUNCH_CHECK();
    }
    double exact2 = 0;
    ISDF_CUDA(cudaMemcpyAsync(&exact2, q.scal.get(), sizeof(double), cudaMemcpyDeviceToHost, I.s));
    ISDF_CUDA(cudaStreamSynchronize(I.s));
    return exact2;
}

void PairQrShard::accept(const double* row_host, int j, int64_t gcol, double exact2, int64_t winner_pos, bool dense) {
    Impl& I = *p_;
    PairQr& q = I.q;
    cudaStream_t s = I.s;
    const int64_t n = q.n, d = q.d, m = q.m;
    I.ensure(j + 1);
    I.upload_row(row_host);   // the same row as the last verify (r, t0, t1 are its)
    const double rj = std::sqrt(exact2);
    rcol_kernel<<<1, 64, 0, s>>>(q.t0.get(), q.t1.get(), j, q.scal.get(), q.Rcol.get());
    ISDF_LAUNCH_CHECK();
    scale_copy(q.r.get(), 1.0 / rj, m, q.Q.get() + static_cast<int64_t>(j) * m, s);
    const int64_t l = I.local(gcol);
    if (l >= 0) {
        mark_selected_kernel<<<1, 1, 0, s>>>(q.selected.get(), q.est.get(), l);
        ISDF_LAUNCH_CHECK();
    }
    if (n > 0) {
        const unsigned nb = static_cast<unsigned>((n + 255) / 256);
        if (dense) {
            shard_swap_pos_kernel<<<nb, 256, 0, s>>>(q.pos.get(), n, j, winner_pos, l);
            ISDF_LAUNCH_CHECK();
        }
        const double* xrow = I.rowbuf.get();
        if (q.cs.get()) {
            scaled_pivot_row_kernel<<<static_cast<unsigned>((d + 255) / 256), 256, 0, s>>>(I.rowbuf.get(), q.cs.get(),
                                                                                         d, q.xp.get());
            ISDF_LAUNCH_CHECK();
            xrow = q.xp.get();
        }
        row_dot(q.F.get(), n, d, xrow, q.D.get(), s);
        update_residual_swp_kernel<<<nb, 256, 0, s>>>(q.D.get(), q.sw.get(), I.rowbuf.get() + d, n, q.L.get(), q.capL,
                                                      j, q.Rcol.get(), rj, q.est.get(), q.selected.get());
        ISDF_LAUNCH_CHECK();
    }
    ISDF_CUDA(cudaStreamSynchronize(s));   // the host row may go out of scope
}

int64_t PairQrShard::scan(int j, double thr2) {
    Impl& I = *p_;
    PairQr& q = I.q;
    cudaStream_t s = I.s;
    const int64_t n = q.n;
    if (n == 0) return 0;
    I.ensure(j + 1);
    const double rel = 64.0 * std::numeric_limits<double>::epsilon() * static_cast<double>(j + 1);
    DeviceBuffer<char> flags(n, s);
    flag_uncertain_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(q.est.get(), q.kdiag.get(),
                                                                                q.selected.get(), n, rel, thr2,
                                                                                flags.get());
    ISDF_LAUNCH_CHECK();
    std::vector<char> h(n);
    ISDF_CUDA(cudaMemcpyAsync(h.data(), flags.get(), n, cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    int64_t cnt = 0;
    for (int64_t g = 0; g < n; ++g)
        if (h[g]) {
            export_row_kernel<<<1, 256, 0, s>>>(q.F.get(), q.d, q.sw.get(), g, I.rowbuf.get());
            ISDF_LAUNCH_CHECK();
            I.exact_residual(j);
            set_est_kernel<<<1, 1, 0, s>>>(q.est.get(), g, q.scal.get());
            ISDF_LAUNCH_CHECK();
            ++cnt;
        }
    ISDF_CUDA(cudaStreamSynchronize(s));
    return cnt;
}

}  // namespace isdf
