// Grid-point compaction, multi-axis Frobenius scales, the quadrature
// Khatri-Rao pair sketch and the column-pivoted QR of the sketch.
//
// Reference behaviour restated (mikovtun/mp_isdf):
//   eligibility (weights finite, zero weights skipped, kept coordinates finite)
//       cpp/src/anchor_select_randomized_id.cpp:131-146
//   multi-axis global Frobenius scales      cpp/src/anchor_select.cpp:437-480
//   sketch rows, caps and validation        cpp/src/anchor_select_randomized_id.cpp:116-191
//   U/V streams (mt19937_64, normal_distribution, u[a*ell+s])
//                                           cpp/src/anchor_select_randomized_id.cpp:269-279
//   Y[s,g] = sqrt|w_g|/sqrt(ell) (f_g.u_s)(f_g.v_s)   :297-309
//   dgeqp3 of Y, row energies -> tails, numerical rank, exact-rank / tolerance
//   rank selection                          cpp/src/anchor_select_randomized_id.cpp:320-374
#include "isdf_select.h"
#include "isdf_reduce.cuh"

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <random>

namespace isdf {

// ------------------------------------------------------------------------------
// eligibility + compaction
// ------------------------------------------------------------------------------
namespace {

__global__ void flag_points_kernel(const double* __restrict__ pts, const double* __restrict__ w,
                                   int64_t n, char* __restrict__ keep, int* __restrict__ bad) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double wg = w[g];
    if (!isfinite(wg)) { atomicOr(bad, 1); keep[g] = 0; return; }
    const bool k = wg != 0.0;
    keep[g] = k;
    if (k && !(isfinite(pts[3 * g]) && isfinite(pts[3 * g + 1]) && isfinite(pts[3 * g + 2])))
        atomicOr(bad, 2);
}

}  // namespace

KeptPoints compact_points(const double* pts, const double* w, int64_t n, cudaStream_t s) {
    KeptPoints kp;
    kp.index.reset(std::max<int64_t>(n, 1), s);
    if (n == 0) return kp;
    DeviceBuffer<char> keep(n, s);
    DeviceBuffer<int> bad(1, s);
    DeviceBuffer<int64_t> count(1, s);
    bad.zero(s);
    flag_points_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(pts, w, n, keep.get(),
                                                                              bad.get());
    ISDF_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    thrust::counting_iterator<int64_t> it(0);
    ISDF_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, keep.get(), kp.index.get(),
                                         count.get(), n, s));
    DeviceBuffer<char> tmp(tmp_bytes, s);
    ISDF_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tmp_bytes, it, keep.get(), kp.index.get(),
                                         count.get(), n, s));
    int hbad = 0;
    int64_t hcount = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(&hcount, count.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad & 1) fail(kInvalid, "grid weights must be finite");
    if (hbad & 2) fail(kInvalid, "grid coordinates must be finite");
    kp.n = hcount;
    return kp;
}

// ------------------------------------------------------------------------------
// axis bookkeeping
// ------------------------------------------------------------------------------
AxisSpec make_axis_spec(const Context& c, const int32_t* axes, int naxes) {
    require(naxes > 0, "axis list must not be empty");
    if (naxes > 16) fail(kNotImplemented, "more than 16 axis entries are not supported");
    AxisSpec ax{};
    ax.naxes = naxes;
    for (int a = 0; a < naxes; ++a) {
        const int t = axes[a];
        if (t == 4) fail(kNotImplemented, "the OccupiedOrbital axis is not implemented on the B200 path");
        require(t >= 0 && t <= 3, "unknown AxisType");
        ax.comp[a] = t;
        ax.scale[a] = 1.0;
        ax.need_mask |= 1 << t;
    }
    require(c.nao > 0, "no orbital features available");
    return ax;
}

std::vector<double> axis_scales_from_sumsq(const AxisSpec& ax, const double* sumsq4,
                                           const double* axis_weights, bool any_eligible) {
    std::vector<double> scales;
    if (!any_eligible) return scales;
    for (int a = 0; a < ax.naxes; ++a) {
        const double norm = std::sqrt(sumsq4[ax.comp[a]]);
        if (!(norm > 0) || !std::isfinite(norm))
            fail(kInvalid, "axis Frobenius norm must be finite and positive");
        const double scale = (axis_weights ? axis_weights[a] : 1.0) / norm;
        if (!(scale > 0) || !std::isfinite(scale))
            fail(kInvalid, "normalized axis scale must be finite and positive");
        scales.push_back(scale);
    }
    return scales;
}

void validate_axis_weights(const double* axis_weights, int naxes) {
    if (!axis_weights) return;
    for (int a = 0; a < naxes; ++a)
        if (!std::isfinite(axis_weights[a]) || axis_weights[a] <= 0)
            fail(kInvalid, "axis weights must be finite and positive");
}

// ------------------------------------------------------------------------------
// sketch
// ------------------------------------------------------------------------------
void sketch_factors(int64_t d, int64_t ell, uint64_t seed, std::vector<double>& u,
                    std::vector<double>& v) {
    // Two independent streams; fill order i = a*ell + s.
    std::mt19937_64 gen_u(seed), gen_v(seed ^ 0x9e3779b97f4a7c15ULL);
    std::normal_distribution<double> normal_u(0, 1), normal_v(0, 1);
    u.resize(static_cast<size_t>(d * ell));
    v.resize(static_cast<size_t>(d * ell));
    for (int64_t i = 0; i < d * ell; ++i) {
        u[i] = normal_u(gen_u);
        v[i] = normal_v(gen_v);
    }
}

namespace {

// Yt[s*ldy + g] = sqrt|w|/sqrt(ell) * (sum_a sc_a P[g][a][s]) * (sum_a sc_a P[g][a][ell+s])
__global__ void combine_sketch_kernel(const double* __restrict__ P, int naxes, int64_t ell,
                                      const double* __restrict__ scales,
                                      const double* __restrict__ w,
                                      const int64_t* __restrict__ index, int64_t n,
                                      double* __restrict__ Yt, int64_t ldy, int* __restrict__ bad) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const double sw = sqrt(fabs(w[index[g]])) / sqrt(static_cast<double>(ell));
    const double* pg = P + g * naxes * 2 * ell;
    bool ok = true;
    for (int64_t s = 0; s < ell; ++s) {
        double left = 0, right = 0;
        for (int a = 0; a < naxes; ++a) {
            const double sc = scales ? scales[a] : 1.0;
            left += sc * pg[a * 2 * ell + s];
            right += sc * pg[a * 2 * ell + ell + s];
        }
        const double y = sw * left * right;
        ok = ok && isfinite(y);
        Yt[s * ldy + g] = y;
    }
    if (!ok) atomicOr(bad, 1);
}

}  // namespace

void sketch_fp64(const Context& c, const double* pts, const KeptPoints& kp, const double* w,
                 const AxisSpec& ax, const double* axis_weights, int64_t ell,
                 const std::vector<double>& u, const std::vector<double>& v, double* Yt,
                 int64_t ldy, int64_t chunk, cudaStream_t s) {
    const int nao = c.nao;
    const int naxes = ax.naxes;
    const int64_t d = static_cast<int64_t>(naxes) * nao;
    const int64_t n = kp.n;
    // W[j][0..ell) = U row j, W[j][ell..2ell) = V row j
    std::vector<double> hw(static_cast<size_t>(d * 2 * ell));
    for (int64_t j = 0; j < d; ++j)
        for (int64_t t = 0; t < ell; ++t) {
            hw[j * 2 * ell + t] = u[j * ell + t];
            hw[j * 2 * ell + ell + t] = v[j * ell + t];
        }
    DeviceBuffer<double> W(hw.size(), s);
    ISDF_CUDA(cudaMemcpyAsync(W.get(), hw.data(), hw.size() * sizeof(double),
                              cudaMemcpyHostToDevice, s));
    DeviceBuffer<double> P(static_cast<size_t>(n * naxes * 2 * ell), s);
    DeviceBuffer<double> sumsq(4, s);
    sumsq.zero(s);
    chunk = std::max<int64_t>(1, std::min(chunk, n));
    DeviceBuffer<double> F(static_cast<size_t>(chunk * d), s);
    for (int64_t g0 = 0; g0 < n; g0 += chunk) {
        const int64_t b = std::min(chunk, n - g0);
        eval_axis_features<double>(c, pts, kp.index.get() + g0, b, ax, F.get(), d,
                                   naxes > 1 ? sumsq.get() : nullptr, nullptr, s);
        // per-axis partial projections P[g][a][0..2ell)
        gemm_f64(b, 2 * ell, nao, F.get(), d, nao, W.get(), 2 * ell, nao * 2 * ell,
                 P.get() + g0 * naxes * 2 * ell, naxes * 2 * ell, 2 * ell, naxes, false, s);
    }
    DeviceBuffer<double> dscales;
    if (naxes > 1) {
        double h[4];
        ISDF_CUDA(cudaMemcpyAsync(h, sumsq.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        auto sc = axis_scales_from_sumsq(ax, h, axis_weights, n > 0);
        dscales.reset(sc.size(), s);
        ISDF_CUDA(cudaMemcpyAsync(dscales.get(), sc.data(), sc.size() * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    }
    DeviceBuffer<int> bad(1, s);
    bad.zero(s);
    ISDF_PROFILE("sketch_combine", s);
    combine_sketch_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
        P.get(), naxes, ell, naxes > 1 ? dscales.get() : nullptr, w, kp.index.get(), n, Yt, ldy,
        bad.get());
    ISDF_LAUNCH_CHECK();
    int hbad = 0;
    ISDF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    if (hbad) fail(kOverflow, "non-finite randomized ID sketch");
}

// ------------------------------------------------------------------------------
// column-pivoted Householder QR of the (ell x n) sketch, dgeqp3 pivot rule:
// at step j the column with the largest trailing norm wins, ties broken by the
// smallest current (swapped) column position.
// ------------------------------------------------------------------------------
namespace {

constexpr int kQrThreads = 256;

struct QrState {
    double* Yt; int64_t ldy; int64_t m; int64_t n;
    int64_t* pos;        // current position of each column
    int64_t* col_at;     // column at each position (inverse of pos)
    char* selected;
    double* v;           // current reflector (m)
    double* tau;         // per step
    double* diag;        // |R_jj| per step
    double* energy;      // row energies of R per step
    int64_t* jpvt;       // pivot columns per step
    ArgKey* partial;     // per block
};

// Apply reflector j-1 (if j > 0) to every unselected column, accumulate the
// final row-(j-1) energy and produce per-block argmax keys of the rows j..m-1
// norms.
__global__ void __launch_bounds__(kQrThreads) qr_update_kernel(QrState st, int64_t j) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * kQrThreads + threadIdx.x;
    __shared__ ArgKey ksh[kQrThreads / 32];
    ArgKey key = key_none();
    double e = 0.0;
    if (g < st.n && !st.selected[g]) {
        double* col = st.Yt + g;
        const int64_t ld = st.ldy;
        if (j > 0) {
            const double t = st.tau[j - 1];
            if (t != 0.0) {
                double dot = 0;
                for (int64_t i = j - 1; i < st.m; ++i) dot += st.v[i] * col[i * ld];
                dot *= t;
                for (int64_t i = j - 1; i < st.m; ++i) col[i * ld] -= st.v[i] * dot;
            }
            const double r = col[(j - 1) * ld];
            e = r * r;
        }
        if (j < st.m) {
            double nrm = 0;
            for (int64_t i = j; i < st.m; ++i) { const double x = col[i * ld]; nrm += x * x; }
            key = ArgKey{nrm, st.pos[g], g};
        }
    }
    // block reductions
    __shared__ double esh[kQrThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if (threadIdx.x % 32 == 0) esh[threadIdx.x / 32] = e;
    ArgKey best = block_best<kQrThreads>(key, ksh);
    if (threadIdx.x == 0) {
        double et = 0;
        for (int i = 0; i < kQrThreads / 32; ++i) et += esh[i];
        if (j > 0 && et != 0.0) atomicAdd(&st.energy[j - 1], et);
        st.partial[blockIdx.x] = best;
    }
}

// Reduce the block keys, record the pivot, swap positions, build reflector j.
__global__ void __launch_bounds__(1024) qr_pivot_kernel(QrState st, int64_t j, int nblocks) {
    __shared__ ArgKey ksh[32];
    ArgKey k = key_none();
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        if (key_better(st.partial[b], k)) k = st.partial[b];
    k = block_best<1024>(k, ksh);
    __shared__ int64_t piv;
    __shared__ double sh_scale;
    if (threadIdx.x == 0) piv = k.col;
    __syncthreads();
    if (piv < 0) return;   // every column already pivoted (cannot happen for j < min(m, n))
    if (threadIdx.x == 0) {
        const int64_t p = piv;
        st.jpvt[j] = p;
        st.selected[p] = 1;
        // dgeqp3 swaps the pivot column into position j
        const int64_t pp = st.pos[p];
        const int64_t cj = st.col_at[j];
        st.col_at[pp] = cj;
        st.pos[cj] = pp;
        st.col_at[j] = p;
        st.pos[p] = j;
        const double* col = st.Yt + p;
        const double alpha = col[j * st.ldy];
        double xnorm = 0;
        for (int64_t i = j + 1; i < st.m; ++i) xnorm = hypot(xnorm, col[i * st.ldy]);
        double beta, tau, scale;
        if (xnorm == 0.0) {
            beta = alpha; tau = 0.0; scale = 0.0;
        } else {
            beta = -copysign(hypot(alpha, xnorm), alpha);
            tau = (beta - alpha) / beta;
            scale = 1.0 / (alpha - beta);
        }
        st.tau[j] = tau;
        st.diag[j] = fabs(beta);
        atomicAdd(&st.energy[j], beta * beta);
        sh_scale = scale;
    }
    __syncthreads();
    const int64_t p = piv;
    for (int64_t i = threadIdx.x; i < st.m; i += blockDim.x) {
        double vi;
        if (i < j) vi = 0.0;
        else if (i == j) vi = 1.0;
        else vi = st.Yt[i * st.ldy + p] * sh_scale;
        st.v[i] = vi;
    }
}

}  // namespace

SketchQR qrcp_sketch(double* Yt, int64_t ldy, int64_t m, int64_t n, cudaStream_t s) {
    SketchQR out;
    const int64_t steps = std::min(m, n);
    if (steps == 0) return out;
    const int nblocks = static_cast<int>((n + kQrThreads - 1) / kQrThreads);
    DeviceBuffer<int64_t> pos(n, s), col_at(n, s), jpvt(steps, s);
    DeviceBuffer<char> selected(n, s);
    DeviceBuffer<double> v(m, s), tau(steps, s), diag(steps, s), energy(steps, s);
    DeviceBuffer<ArgKey> partial(nblocks, s);
    selected.zero(s);
    energy.zero(s);
    iota_i64(pos.get(), n, s);
    iota_i64(col_at.get(), n, s);
    QrState st{Yt, ldy, m, n, pos.get(), col_at.get(), selected.get(), v.get(), tau.get(),
               diag.get(), energy.get(), jpvt.get(), partial.get()};
    for (int64_t j = 0; j <= steps; ++j) {
        {
            ISDF_PROFILE("qrcp_sketch_update", s);
            qr_update_kernel<<<nblocks, kQrThreads, 0, s>>>(st, j);
            ISDF_LAUNCH_CHECK();
        }
        if (j < steps) {
            ISDF_PROFILE("qrcp_sketch_pivot", s);
            qr_pivot_kernel<<<1, 1024, 0, s>>>(st, j, nblocks);
            ISDF_LAUNCH_CHECK();
        }
    }
    out.jpvt.resize(steps);
    out.diag.resize(steps);
    out.energy.resize(steps);
    ISDF_CUDA(cudaMemcpyAsync(out.jpvt.data(), jpvt.get(), steps * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(out.diag.data(), diag.get(), steps * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(out.energy.data(), energy.get(), steps * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    return out;
}

// ------------------------------------------------------------------------------
// rand_sketch (quadrature) driver
// ------------------------------------------------------------------------------
std::vector<int64_t> select_rand_sketch(const Context& c, const double* pts, const double* w,
                                        int64_t ng, const SelectOptions& o, cudaStream_t s,
                                        SketchDiagnostics* diag_out) {
    if (!std::isfinite(o.tolerance) || o.tolerance < 0 || o.batch_size <= 0 ||
        o.oversampling <= 0 || (!o.max_rank && o.sketch_size <= o.oversampling))
        fail(kInvalid, "invalid randomized ID grid, tolerance, batch, sketch or rank/oversampling");
    AxisSpec ax = make_axis_spec(c, o.axes.data(), static_cast<int>(o.axes.size()));
    const int64_t d = static_cast<int64_t>(ax.naxes) * c.nao;
    if (o.max_rank > std::numeric_limits<int64_t>::max() - o.oversampling)
        fail(kOverflow, "randomized ID rank + oversampling overflows size_t");
    const int64_t requested = o.max_rank ? o.max_rank + o.oversampling : o.sketch_size;
    KeptPoints kp = compact_points(pts, w, ng, s);
    const int64_t n = kp.n;
    if (n == 0) return {};
    const int64_t physical_rank = d * (d + 1) / 2;
    const int64_t physical_limit = physical_rank + o.oversampling;
    const int64_t backend_limit = std::numeric_limits<int64_t>::max() / n;
    const int64_t ell = requested <= backend_limit
                            ? requested
                            : std::min({requested, physical_limit, backend_limit});
    if (ell <= o.oversampling ||
        (o.max_rank && std::min(o.max_rank, physical_rank) > ell - o.oversampling))
        fail(kInvalid, "randomized ID sketch/rank exceeds the ILP64 QRCP backend limit for this "
                       "grid; reduce the sketch/rank or use a tiled QRCP backend");
    if (o.max_rank > std::min(n, physical_rank))
        fail(kInvalid, "requested anchor_rank exceeds eligible candidates or physical pair rank");
    std::vector<double> u, v;
    sketch_factors(d, ell, o.seed, u, v);
    const int64_t ldy = n;
    DeviceBuffer<double> Yt(static_cast<size_t>(ell * n), s);
    const int64_t chunk = std::max<int64_t>(1024, std::min<int64_t>(n, (int64_t(1) << 28) / d));
    sketch_fp64(c, pts, kp, w, ax, o.axis_weights.empty() ? nullptr : o.axis_weights.data(), ell,
                u, v, Yt.get(), ldy, chunk, s);
    SketchQR qr = qrcp_sketch(Yt.get(), ldy, ell, n, s);
    const int64_t steps = std::min(ell, n);
    std::vector<double> tails(steps + 1, 0.0);
    double diag_max = 0;
    for (int64_t i = steps; i-- > 0;) {
        tails[i] = std::hypot(tails[i + 1], std::sqrt(qr.energy[i]));
        diag_max = std::max(diag_max, qr.diag[i]);
    }
    if (!std::isfinite(tails[0]) || !std::isfinite(diag_max))
        fail(kOverflow, "non-finite randomized ID QR residual");
    const double norm = tails[0];
    const double floor = std::numeric_limits<double>::epsilon() *
                         static_cast<double>(std::max(ell, n)) * diag_max;
    int64_t numerical_rank = steps;
    for (int64_t i = 0; i < steps; ++i)
        if (qr.diag[i] <= floor) { numerical_rank = i; break; }
    const int64_t cap = std::min({o.max_rank ? o.max_rank : ell - o.oversampling,
                                  ell - o.oversampling, steps, physical_rank, numerical_rank});
    if (o.max_rank && numerical_rank < o.max_rank)
        fail(kInvalid, "requested anchor_rank exceeds the numerical rank of the randomized sketch");
    int64_t rank = o.max_rank ? o.max_rank : cap;
    if (!o.max_rank)
        for (int64_t i = 0; i <= cap; ++i)
            if (tails[i] <= o.tolerance * norm) { rank = i; break; }
    std::vector<int64_t> kept_host(n);
    ISDF_CUDA(cudaMemcpyAsync(kept_host.data(), kp.index.get(), n * sizeof(int64_t),
                              cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> selected;
    for (int64_t i = 0; i < rank; ++i) {
        const int64_t pv = qr.jpvt[i];
        if (pv < 0 || pv >= n) fail(kRuntime, "randomized ID QRCP returned invalid pivot");
        selected.push_back(kept_host[pv]);
    }
    if (diag_out) {
        diag_out->ell = ell;
        diag_out->numerical_rank = numerical_rank;
        diag_out->cap = cap;
        diag_out->rank = rank;
        diag_out->relative_tail = norm ? tails[rank] / norm : 0.0;
        diag_out->diag = qr.diag;
        diag_out->tails = tails;
    }
    return selected;
}

}  // namespace isdf
