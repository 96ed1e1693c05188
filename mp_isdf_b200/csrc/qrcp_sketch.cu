// Column-pivoted Householder QR of the ell x n Khatri-Rao sketch (FP64).
//
// Pivot rule of LAPACK dgeqp3 (used by the reference through LAPACK++ /
// MAGMA, cpp/src/anchor_select_qrcp.cpp:36-90): at step j the column with the
// largest norm of rows j..ell-1 wins; ties go to the first column in the
// current (swapped) column order.  The trailing norms are recomputed exactly
// at every step (one pass over the sketch, fused with the reflector update and
// a warp-shuffle argmax), so no norm-downdating error enters the decision.
// Outputs per step: pivot, |R_jj| and the energy of row j of R (for the
// reference's tail / numerical-rank logic, cpp/src/anchor_select_randomized_id.cpp:327-374).
//
// Verified mode (mixed-precision sketch): every column carries an absolute
// error bound delta_g of its residual norm.  Before each pivot choice, every
// column whose interval [r_g - delta_g, r_g + delta_g] overlaps the best lower
// bound is recomputed exactly in FP64 (AO values and gradients, projection,
// all previous reflectors) and its bound set to zero, so the chosen pivot is
// the FP64 sketch's pivot whenever the FP64 values are not tied.
#include "ao_device.cuh"
#include "isdf_reduce.cuh"
#include "isdf_select.h"

#include <algorithm>
#include <cmath>

namespace isdf {
namespace {

constexpr int kQrThreads = 256;
constexpr int kExactBlocks = 148;   // fixed grid of the candidate re-verification

struct QrState {
    double* Yt; int64_t ldy; int64_t m; int64_t n;
    int64_t* pos;        // current position of each column
    int64_t* col_at;     // column at each position (inverse of pos)
    char* selected;
    double* vhist;       // reflectors of all steps (m each)
    double* tau;         // per step
    double* diag;        // |R_jj| per step
    double* energy;      // row energies of R per step
    int64_t* jpvt;       // pivot columns per step
    ArgKey* partial;     // per block
    double* est;         // verified mode: squared trailing norms
    double* delta;       // verified mode: error bounds (0 = exact)
    double* lb_partial;  // verified mode: per-block best lower bound
};

// Apply reflector j-1 (if j > 0) to every unselected column, accumulate the
// final row-(j-1) energy and produce per-block argmax keys of the rows j..m-1
// norms (and, in verified mode, the squared norms and best lower bound).
__global__ void __launch_bounds__(kQrThreads) qr_update_kernel(QrState st, int64_t j) {
    __shared__ ArgKey ksh[kQrThreads / 32];
    __shared__ double esh[kQrThreads / 32];
    __shared__ double lsh[kQrThreads / 32];
    const int64_t g = static_cast<int64_t>(blockIdx.x) * kQrThreads + threadIdx.x;
    ArgKey key = key_none();
    double e = 0.0, lb = -1.0;
    if (g < st.n && !st.selected[g]) {
        double* col = st.Yt + g;
        const int64_t ld = st.ldy;
        if (j > 0) {
            const double t = st.tau[j - 1];
            const double* v = st.vhist + (j - 1) * st.m;
            if (t != 0.0) {
                double dot = 0;
                for (int64_t i = j - 1; i < st.m; ++i) dot += v[i] * col[i * ld];
                dot *= t;
                for (int64_t i = j - 1; i < st.m; ++i) col[i * ld] -= v[i] * dot;
            }
            const double r = col[(j - 1) * ld];
            e = r * r;
        }
        if (j < st.m) {
            double nrm = 0;
            for (int64_t i = j; i < st.m; ++i) { const double x = col[i * ld]; nrm += x * x; }
            key = ArgKey{nrm, st.pos[g], g};
            if (st.est) {
                st.est[g] = nrm;
                lb = sqrt(nrm) - st.delta[g];
            }
        }
    }
    e = warp_sum(e);
    double lw = lb;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lw = fmax(lw, __shfl_down_sync(0xffffffffu, lw, o));
    if (threadIdx.x % 32 == 0) { esh[threadIdx.x / 32] = e; lsh[threadIdx.x / 32] = lw; }
    ArgKey best = block_best<kQrThreads>(key, ksh);
    if (threadIdx.x == 0) {
        double et = 0, lt = -1.0;
        for (int i = 0; i < kQrThreads / 32; ++i) { et += esh[i]; lt = fmax(lt, lsh[i]); }
        if (j > 0 && et != 0.0) atomicAdd(&st.energy[j - 1], et);
        st.partial[blockIdx.x] = best;
        if (st.lb_partial) st.lb_partial[blockIdx.x] = lt;
    }
}

// Verified mode: argmax keys from the (partly re-verified) squared norms.
__global__ void __launch_bounds__(kQrThreads) est_argmax_kernel(QrState st) {
    __shared__ ArgKey ksh[kQrThreads / 32];
    const int64_t g = static_cast<int64_t>(blockIdx.x) * kQrThreads + threadIdx.x;
    ArgKey key = key_none();
    if (g < st.n && !st.selected[g]) key = ArgKey{st.est[g], st.pos[g], g};
    ArgKey best = block_best<kQrThreads>(key, ksh);
    if (threadIdx.x == 0) st.partial[blockIdx.x] = best;
}

// Verified mode: best lower bound, then the list of columns to recompute.
__global__ void __launch_bounds__(1024) lb_reduce_kernel(const double* lb_partial, int nblocks,
                                                         double* lb_out) {
    __shared__ double sh[32];
    double v = -1.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = fmax(v, lb_partial[b]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (threadIdx.x % 32 == 0) sh[threadIdx.x / 32] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < 32; ++i) v = fmax(v, sh[i]);
        lb_out[0] = v;
    }
}

__global__ void candidates_kernel(QrState st, const double* lb, int64_t* cand, int64_t* count) {
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= st.n || st.selected[g]) return;
    const double d = st.delta[g];
    if (d > 0.0 && sqrt(st.est[g]) + d >= lb[0]) {
        const int64_t i = static_cast<int64_t>(atomicAdd(reinterpret_cast<unsigned long long*>(count), 1ull));
        cand[i] = g;
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
    double* v = st.vhist + j * st.m;
    for (int64_t i = threadIdx.x; i < st.m; i += blockDim.x) {
        double vi;
        if (i < j) vi = 0.0;
        else if (i == j) vi = 1.0;
        else vi = st.Yt[i * st.ldy + p] * sh_scale;
        v[i] = vi;
    }
}

// ---- exact FP64 sketch columns -----------------------------------------------------
// Component-major AO values of one point: feat[C*nao + ao].
struct CompSink {
    double* feat; int nao;
    template <int C> __device__ __forceinline__ void put(int ao, double v) { feat[C * nao + ao] = v; }
};

struct ExactArgs {
    const ShellDesc* shells; int nshell; const double* exps; const double* coefs;
    int nao; int naxes; int comp[16]; int grad;
    const double* scales;       // naxes (device)
    const double* WT;           // (2 ell) x d, row-major
    const double* pts; const int64_t* index; const double* w;
    int64_t ell;
};

// FP64 recomputation of sketch column g (block-wide; feat holds kNComp*nao
// AO values, 2*ell projections and m sketch rows).
template <bool GRAD, int LMAX>
__device__ void exact_column(const ExactArgs& ea, const QrState& st, int64_t g, int64_t j, double* feat) {
    constexpr int kNComp = GRAD ? 4 : 1;
    const int64_t gi = ea.index[g];
    const int nao = ea.nao;
    const int64_t d = static_cast<int64_t>(ea.naxes) * nao;
    double* lr = feat + kNComp * nao;
    const double px = ea.pts[3 * gi], py = ea.pts[3 * gi + 1], pz = ea.pts[3 * gi + 2];
    CompSink sink{feat, nao};
    for (int sh = threadIdx.x; sh < ea.nshell; sh += blockDim.x) {
        const ShellDesc b = ea.shells[sh];
        eval_shell_any<double, GRAD, LMAX>(b, px - b.x, py - b.y, pz - b.z, ea.exps, ea.coefs, sink);
    }
    __syncthreads();
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    // projections lr[s2] = sum_a scale_a comp_a(g) . WT[s2][a]
    for (int64_t s2 = warp; s2 < 2 * ea.ell; s2 += blockDim.x / 32) {
        const double* wt = ea.WT + s2 * d;
        double acc = 0;
        for (int a = 0; a < ea.naxes; ++a) {
            const double* f = feat + (GRAD ? ea.comp[a] : 0) * nao;
            const double* wa = wt + static_cast<int64_t>(a) * nao;
            double pa = 0;
            for (int i = lane; i < nao; i += 32) pa += f[i] * wa[i];
            acc += ea.scales[a] * pa;
        }
        acc = warp_sum(acc);
        if (lane == 0) lr[s2] = acc;
    }
    __syncthreads();
    // apply the j previous reflectors to the sketch column (warp 0, lanes over rows)
    if (warp == 0) {
        const int64_t m = st.m;
        double* y = lr + 2 * ea.ell;
        const double sw = sqrt(fabs(ea.w[gi])) / sqrt(static_cast<double>(ea.ell));
        for (int64_t s = lane; s < m; s += 32) y[s] = sw * lr[s] * lr[ea.ell + s];
        __syncwarp();
        for (int64_t i = 0; i < j; ++i) {
            const double t = st.tau[i];
            if (t == 0.0) continue;
            const double* v = st.vhist + i * m;
            double dot = 0;
            for (int64_t r = i + lane; r < m; r += 32) dot += v[r] * y[r];
            dot = warp_allsum(dot) * t;
            for (int64_t r = i + lane; r < m; r += 32) y[r] -= v[r] * dot;
            __syncwarp();
        }
        double nrm = 0;
        for (int64_t s = lane; s < m; s += 32) {
            st.Yt[s * st.ldy + g] = y[s];
            if (s >= j) nrm += y[s] * y[s];
        }
        nrm = warp_sum(nrm);
        if (lane == 0) {
            st.est[g] = nrm;
            st.delta[g] = 0.0;
        }
    }
}

// Re-verifies the candidates cand[0 .. *count) chosen on the device this step;
// the grid is fixed, so the host needs no count before the launch.
template <bool GRAD, int LMAX, int NTHR>
__global__ void __launch_bounds__(NTHR)
exact_columns_kernel(ExactArgs ea, QrState st, const int64_t* cand, const int64_t* count, int64_t j,
                     unsigned long long* total) {
    extern __shared__ double feat[];
    const int64_t nc = *count;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(total, static_cast<unsigned long long>(nc));
    for (int64_t ci = blockIdx.x; ci < nc; ci += gridDim.x) {
        exact_column<GRAD, LMAX>(ea, st, cand[ci], j, feat);
        __syncthreads();   // feat is reused by the next candidate
    }
}

using ExactKernelFn = void (*)(ExactArgs, QrState, const int64_t*, const int64_t*, int64_t, unsigned long long*);
struct ExactKernel {
    ExactKernelFn fn = nullptr;
    int threads = 0;
};

// Specialisation on the basis' largest angular momentum keeps the FP64
// evaluation within registers; small l leaves room for about one shell per
// thread of a 1024-thread block.
ExactKernel pick_exact_kernel(bool grad, int lmax) {
    if (grad) {
        if (lmax <= 2) return {exact_columns_kernel<true, 2, 1024>, 1024};
        if (lmax <= 4) return {exact_columns_kernel<true, 4, 256>, 256};
        return {exact_columns_kernel<true, kMaxL, 256>, 256};
    }
    if (lmax <= 2) return {exact_columns_kernel<false, 2, 1024>, 1024};
    if (lmax <= 4) return {exact_columns_kernel<false, 4, 256>, 256};
    return {exact_columns_kernel<false, kMaxL, 256>, 256};
}

}  // namespace

SketchQR qrcp_sketch(double* Yt, int64_t ldy, int64_t m, int64_t n, cudaStream_t s,
                     const ExactSketchSource* exact) {
    SketchQR out;
    const int64_t steps = std::min(m, n);
    if (steps == 0) return out;
    if (exact) require(m <= 128, "verified sketch QR supports at most 128 sketch rows");
    const int nblocks = static_cast<int>((n + kQrThreads - 1) / kQrThreads);
    DeviceBuffer<int64_t> pos(n, s), col_at(n, s), jpvt(steps, s);
    DeviceBuffer<char> selected(n, s);
    DeviceBuffer<double> vhist(static_cast<size_t>(m * steps), s), tau(steps, s), diag(steps, s),
        energy(steps, s);
    DeviceBuffer<ArgKey> partial(nblocks, s);
    DeviceBuffer<double> est, lbp, lb;
    DeviceBuffer<int64_t> cand, count;
    selected.zero(s);
    energy.zero(s);
    iota_i64(pos.get(), n, s);
    iota_i64(col_at.get(), n, s);
    QrState st{Yt, ldy, m, n, pos.get(), col_at.get(), selected.get(), vhist.get(), tau.get(),
               diag.get(), energy.get(), jpvt.get(), partial.get(), nullptr, nullptr, nullptr};
    ExactArgs ea{};
    size_t exact_smem = 0;
    ExactKernel exact_kernel;
    if (exact) {
        est.reset(n, s);
        lbp.reset(nblocks, s);
        lb.reset(1, s);
        cand.reset(n, s);
        count.reset(1, s);
        st.est = est.get();
        st.delta = exact->delta;
        st.lb_partial = lbp.get();
        const Context& c = *exact->ctx;
        ea.shells = c.d_shells; ea.nshell = c.nshell; ea.exps = c.d_exp; ea.coefs = c.d_coef;
        ea.nao = c.nao; ea.naxes = exact->naxes; ea.grad = 0;
        for (int a = 0; a < exact->naxes; ++a) { ea.comp[a] = exact->comp[a]; ea.grad |= exact->comp[a] > 0; }
        ea.scales = exact->scales; ea.WT = exact->WT; ea.pts = exact->pts; ea.index = exact->index;
        ea.w = exact->w; ea.ell = exact->ell;
        exact_smem = (static_cast<size_t>(ea.grad ? 4 : 1) * c.nao + 2 * exact->ell + m) * sizeof(double);
        exact_kernel = pick_exact_kernel(ea.grad != 0, c.lmax);
        ISDF_CUDA(cudaFuncSetAttribute(exact_kernel.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(exact_smem)));
    }
    DeviceBuffer<unsigned long long> reverified_d(1, s);
    reverified_d.zero(s);
    for (int64_t j = 0; j <= steps; ++j) {
        {
            ISDF_PROFILE("qrcp_sketch_update", s);
            qr_update_kernel<<<nblocks, kQrThreads, 0, s>>>(st, j);
            ISDF_LAUNCH_CHECK();
        }
        if (j == steps) break;
        if (exact) {
            ISDF_PROFILE("qrcp_sketch_verify", s);
            lb_reduce_kernel<<<1, 1024, 0, s>>>(lbp.get(), nblocks, lb.get());
            ISDF_LAUNCH_CHECK();
            count.zero(s);
            candidates_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(st, lb.get(), cand.get(),
                                                                                      count.get());
            ISDF_LAUNCH_CHECK();
            exact_kernel.fn<<<kExactBlocks, exact_kernel.threads, exact_smem, s>>>(ea, st, cand.get(), count.get(), j,
                                                                reverified_d.get());
            ISDF_LAUNCH_CHECK();
            est_argmax_kernel<<<nblocks, kQrThreads, 0, s>>>(st);
            ISDF_LAUNCH_CHECK();
        }
        {
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
    unsigned long long reverified = 0;
    if (exact)
        ISDF_CUDA(cudaMemcpyAsync(&reverified, reverified_d.get(), sizeof(reverified), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    out.reverified = static_cast<int64_t>(reverified);
    return out;
}

}  // namespace isdf
