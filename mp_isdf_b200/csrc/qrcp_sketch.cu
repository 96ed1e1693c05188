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
#include <cstdint>
#include <cmath>
#include <cstring>

namespace isdf {
namespace {

constexpr int kQrThreads = 256;
constexpr int kExactBlocks = 148;   // fixed grid of the candidate re-verification
constexpr int kRegRows = 32;        // trailing rows the update stages in shared memory
constexpr int kSplitCands = 16;     // up to this many candidates are split over blocks
constexpr int kMaxSketchRows = 128;

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
    ArgKey* partial;     // per block of the column sweep
    // verified mode
    double* est;                  // squared trailing norms
    double* delta;                // error bounds (0 = exact)
    unsigned long long* lb_bits;  // best lower bound max(sqrt(est) - delta, 0), as its bits
    int64_t* count;               // candidates of this step
    ArgKey* xpartial;             // per re-verification block
    // per update block (kQrThreads columns), verified mode: the largest upper
    // bound sqrt(est) + delta of its inexact columns (-1 if none) and the best
    // argmax key of its exact columns, so the candidate scan can pass over a
    // block that holds no candidate without reading its columns
    double* seg_ub;
    ArgKey* seg_key;
};

// Update blocks that one block of the candidate scan covers.
constexpr int kCandSegs = 16;

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Apply reflector j-1 (if j > 0) to every unselected column, accumulate the
// final row-(j-1) energy and form the squared norms of rows j..m-1: as
// per-block argmax keys, or in verified mode as est[] plus the best lower
// bound, kept by an atomic max on its bits (non-negative doubles order like
// their bit patterns).  Row j-1 of an unselected column is final there
// (R[j-1][g]) and nothing reads it again, so only rows j..m-1 are stored.
// STAGED: the touched rows (at most kRegRows) are copied once into shared
// memory (xs[row][thread], cp.async: no registers held while they are in
// flight) and read from there by the dot product and the update.
template <bool STAGED>
__global__ void __launch_bounds__(kQrThreads) qr_update_kernel(QrState st, int64_t j) {
    __shared__ ArgKey ksh[kQrThreads / 32];
    __shared__ double esh[kQrThreads / 32];
    __shared__ double lsh[kQrThreads / 32];
    __shared__ double ush[kQrThreads / 32];
    __shared__ double vsh[kRegRows];
    extern __shared__ double xs[];   // STAGED: [kRegRows][kQrThreads]
    const int tid = threadIdx.x;
    const int64_t g = static_cast<int64_t>(blockIdx.x) * kQrThreads + tid;
    const bool verified = st.est != nullptr;
    const int64_t m = st.m, ld = st.ldy;
    const int64_t r0 = j > 0 ? j - 1 : 0;   // first row touched
    const bool active = g < st.n && !st.selected[g];
    double* col = st.Yt + g;
    if constexpr (STAGED) {
        const int cnt = static_cast<int>(m - r0);
        if (active) {
            const double* src = col + r0 * ld;
            for (int i = 0; i < cnt; ++i, src += ld) {
                const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(&xs[i * kQrThreads + tid]));
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        // the reflector's touched entries, read by every thread
        if (j > 0 && tid < cnt) vsh[tid] = st.vhist[(j - 1) * m + r0 + tid];
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
    }
    ArgKey key = key_none();
    double e = 0.0, lb = 0.0, ub = -1.0;
    if (active) {
        const double t = j > 0 ? st.tau[j - 1] : 0.0;
        double nrm = 0;
        if constexpr (STAGED) {
            const int cnt = static_cast<int>(m - r0);
            const double* x = xs + tid;
            double dot = 0;
            if (t != 0.0) {
                for (int i = 0; i < cnt; ++i) dot += vsh[i] * x[i * kQrThreads];
                dot *= t;
            }
            if (j > 0) {
                const double x0 = x[0] - vsh[0] * dot;
                e = x0 * x0;
            }
            double* dst = col + j * ld;
            for (int i = j > 0 ? 1 : 0; i < cnt; ++i, dst += ld) {
                double xi = x[i * kQrThreads];
                if (t != 0.0) {
                    xi -= vsh[i] * dot;
                    *dst = xi;
                }
                nrm += xi * xi;
            }
        } else {
            const double* v = st.vhist + (j > 0 ? (j - 1) * m : 0);
            double dot = 0;
            if (t != 0.0) {
                for (int64_t i = r0; i < m; ++i) dot += v[i] * col[i * ld];
                dot *= t;
            }
            if (j > 0) {
                const double x0 = col[r0 * ld] - v[r0] * dot;
                e = x0 * x0;
            }
            for (int64_t i = j; i < m; ++i) {
                double x = col[i * ld];
                if (t != 0.0) {
                    x -= v[i] * dot;
                    col[i * ld] = x;
                }
                nrm += x * x;
            }
        }
        if (j < m) {
            if (verified) {
                st.est[g] = nrm;
                const double d = st.delta[g], r = sqrt(nrm);
                lb = fmax(r - d, 0.0);
                if (d > 0.0) ub = r + d;
                else key = ArgKey{nrm, st.pos[g], g};   // exact column
            } else {
                key = ArgKey{nrm, st.pos[g], g};
            }
        }
    }
    e = warp_sum(e);
    lb = warp_max(lb);
    ub = warp_max(ub);
    if (tid % 32 == 0) { esh[tid / 32] = e; lsh[tid / 32] = lb; ush[tid / 32] = ub; }
    // verified: a block key only where the block holds an exact column (rare)
    ArgKey best = key_none();
    if (!verified || __syncthreads_or(key.col >= 0)) best = block_best<kQrThreads>(key, ksh);
    if (tid == 0) {
        double et = 0, lt = 0.0, ut = -1.0;
        for (int i = 0; i < kQrThreads / 32; ++i) { et += esh[i]; lt = fmax(lt, lsh[i]); ut = fmax(ut, ush[i]); }
        if (j > 0 && et != 0.0) atomicAdd(&st.energy[j - 1], et);
        if (!verified) {
            st.partial[blockIdx.x] = best;
        } else {
            st.seg_ub[blockIdx.x] = ut;
            st.seg_key[blockIdx.x] = best;
            if (lt > 0.0) atomicMax(st.lb_bits, static_cast<unsigned long long>(__double_as_longlong(lt)));
        }
    }
}

// Paired form of the staged update, for an even leading dimension and 16-byte
// aligned rows: a thread takes two adjacent columns, copies each touched row
// pair with one 16-byte cp.async and stores an updated pair with one 16-byte
// store, halving the copy and store instructions; each column's arithmetic is
// that of qr_update_kernel<true>, and a block still covers kQrThreads columns
// (one argmax key per block, as the pivot kernel expects).
constexpr int kPairThreads = kQrThreads / 2;
__global__ void __launch_bounds__(kPairThreads) qr_update_pairs_kernel(QrState st, int64_t j) {
    __shared__ ArgKey ksh[kPairThreads / 32];
    __shared__ double esh[kPairThreads / 32];
    __shared__ double lsh[kPairThreads / 32];
    __shared__ double ush[kPairThreads / 32];
    __shared__ double vsh[kRegRows];
    extern __shared__ __align__(16) double xs[];   // [rows][kQrThreads], columns 2 tid and 2 tid + 1
    const int tid = threadIdx.x;
    const int64_t g0 = static_cast<int64_t>(blockIdx.x) * kQrThreads + 2 * tid;
    const bool verified = st.est != nullptr;
    const int64_t m = st.m, ld = st.ldy;
    const int64_t r0 = j > 0 ? j - 1 : 0;   // first row touched
    const int cnt = static_cast<int>(m - r0);
    bool act[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) act[c] = g0 + c < st.n && !st.selected[g0 + c];
    if (act[0] || act[1]) {
        const bool both = g0 + 1 < st.n;
        const double* src = st.Yt + r0 * ld + g0;
        for (int i = 0; i < cnt; ++i, src += ld) {
            const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(&xs[i * kQrThreads + 2 * tid]));
            if (both) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
            else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    if (j > 0 && tid < cnt) vsh[tid] = st.vhist[(j - 1) * m + r0 + tid];
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    ArgKey key = key_none();
    double e = 0.0, lb = 0.0, ub = -1.0;
    if (act[0] || act[1]) {
        const double t = j > 0 ? st.tau[j - 1] : 0.0;
        const double* x = xs + 2 * tid;
        double dot[2] = {0.0, 0.0}, nrm[2] = {0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 2; ++c)
            if (act[c] && t != 0.0) {
                double d = 0;
                for (int i = 0; i < cnt; ++i) d += vsh[i] * x[i * kQrThreads + c];
                dot[c] = d * t;
            }
        if (j > 0) {
#pragma unroll
            for (int c = 0; c < 2; ++c)
                if (act[c]) {
                    const double x0 = x[c] - vsh[0] * dot[c];
                    e += x0 * x0;
                }
        }
        double* dst = st.Yt + j * ld + g0;
        for (int i = j > 0 ? 1 : 0; i < cnt; ++i, dst += ld) {
            double x0 = x[i * kQrThreads], x1 = x[i * kQrThreads + 1];
            if (t != 0.0) {
                x0 -= vsh[i] * dot[0];
                x1 -= vsh[i] * dot[1];
                if (act[0] && act[1]) {
                    *reinterpret_cast<double2*>(dst) = make_double2(x0, x1);
                } else {
                    if (act[0]) dst[0] = x0;
                    if (act[1]) dst[1] = x1;
                }
            }
            nrm[0] += x0 * x0;
            nrm[1] += x1 * x1;
        }
        if (j < m) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                if (!act[c]) continue;
                const int64_t g = g0 + c;
                if (verified) {
                    st.est[g] = nrm[c];
                    const double d = st.delta[g], r = sqrt(nrm[c]);
                    lb = fmax(lb, fmax(r - d, 0.0));
                    if (d > 0.0) {
                        ub = fmax(ub, r + d);
                    } else {   // exact column
                        const ArgKey k{nrm[c], st.pos[g], g};
                        if (key_better(k, key)) key = k;
                    }
                } else {
                    const ArgKey k{nrm[c], st.pos[g], g};
                    if (key_better(k, key)) key = k;
                }
            }
        }
    }
    e = warp_sum(e);
    lb = warp_max(lb);
    ub = warp_max(ub);
    if (tid % 32 == 0) { esh[tid / 32] = e; lsh[tid / 32] = lb; ush[tid / 32] = ub; }
    // verified: a block key only where the block holds an exact column (rare)
    ArgKey best = key_none();
    if (!verified || __syncthreads_or(key.col >= 0)) best = block_best<kPairThreads>(key, ksh);
    if (tid == 0) {
        double et = 0, lt = 0.0, ut = -1.0;
        for (int i = 0; i < kPairThreads / 32; ++i) { et += esh[i]; lt = fmax(lt, lsh[i]); ut = fmax(ut, ush[i]); }
        if (j > 0 && et != 0.0) atomicAdd(&st.energy[j - 1], et);
        if (!verified) {
            st.partial[blockIdx.x] = best;
        } else {
            st.seg_ub[blockIdx.x] = ut;
            st.seg_key[blockIdx.x] = best;
            if (lt > 0.0) atomicMax(st.lb_bits, static_cast<unsigned long long>(__double_as_longlong(lt)));
        }
    }
}

// Verified mode: every unselected column whose interval reaches the best
// lower bound (and is not exact yet) is listed for recomputation; the exact
// columns enter the per-block argmax keys directly.  A column that is neither
// cannot win: its estimate is below (sqrt(e) + delta)^2 < lb^2, and the column
// that sets lb is a candidate or exact with a norm of at least lb.
// A block covers kCandSegs update blocks; one whose largest upper bound is
// below lb holds no candidate, and its exact columns' best key is the one the
// update left, so its columns are not read.
__global__ void __launch_bounds__(kQrThreads) candidates_kernel(QrState st, int64_t* cand, int nseg) {
    __shared__ ArgKey ksh[kQrThreads / 32];
    const double lb = __longlong_as_double(static_cast<long long>(*st.lb_bits));
    ArgKey key = key_none();
    const int s0 = blockIdx.x * kCandSegs, s1 = min(nseg, s0 + kCandSegs);
    for (int sg = s0; sg < s1; ++sg) {
        if (st.seg_ub[sg] < lb) {
            if (threadIdx.x == 0 && key_better(st.seg_key[sg], key)) key = st.seg_key[sg];
            continue;
        }
        const int64_t g = static_cast<int64_t>(sg) * kQrThreads + threadIdx.x;
        if (g < st.n && !st.selected[g]) {
            const double d = st.delta[g], e = st.est[g];
            if (d > 0.0 && sqrt(e) + d >= lb) {
                const int64_t i = static_cast<int64_t>(
                    atomicAdd(reinterpret_cast<unsigned long long*>(st.count), 1ull));
                cand[i] = g;
            } else if (!(d > 0.0)) {
                const ArgKey k{e, st.pos[g], g};
                if (key_better(k, key)) key = k;
            }
        }
    }
    const ArgKey best = block_best<kQrThreads>(key, ksh);
    if (threadIdx.x == 0) st.partial[blockIdx.x] = best;
}

inline int cand_blocks(int nblocks) { return (nblocks + kCandSegs - 1) / kCandSegs; }

// Reduce the block keys (and, verified, the re-verification blocks' keys),
// record the pivot, swap positions, build reflector j; then clear the
// verified-mode step state for step j+1.
__global__ void __launch_bounds__(1024) qr_pivot_kernel(QrState st, int64_t j, int nblocks, int nxblocks) {
    __shared__ ArgKey ksh[32];
    ArgKey k = key_none();
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        if (key_better(st.partial[b], k)) k = st.partial[b];
    for (int b = threadIdx.x; b < nxblocks; b += blockDim.x)
        if (key_better(st.xpartial[b], k)) k = st.xpartial[b];
    k = block_best<1024>(k, ksh);
    __shared__ int64_t piv;
    __shared__ double sh_scale;
    if (threadIdx.x == 0) {
        piv = k.col;
        if (st.count) {
            *st.count = 0;
            *st.lb_bits = 0ull;
        }
    }
    __syncthreads();
    if (piv < 0) return;   // every column already pivoted (cannot happen for j < min(m, n))
    // the pivot column's rows, loaded in parallel (strided by the leading
    // dimension) when they fit; otherwise read in place
    __shared__ double colsh[kMaxSketchRows];
    const bool staged = st.m <= kMaxSketchRows;
    const double* colg = st.Yt + piv;
    auto row = [&](int64_t i) { return staged ? colsh[i] : colg[i * st.ldy]; };
    if (staged)
        for (int64_t i = threadIdx.x; i < st.m; i += blockDim.x) colsh[i] = colg[i * st.ldy];
    __syncthreads();
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
        const double alpha = row(j);
        double xnorm = 0;
        for (int64_t i = j + 1; i < st.m; ++i) xnorm = hypot(xnorm, row(i));
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
    double* v = st.vhist + j * st.m;
    for (int64_t i = threadIdx.x; i < st.m; i += blockDim.x) {
        double vi;
        if (i < j) vi = 0.0;
        else if (i == j) vi = 1.0;
        else vi = row(i) * sh_scale;
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

// FP64 AO values (and gradients) of grid point gi, component-major in feat.
template <bool GRAD, int LMAX>
__device__ void exact_features(const ExactArgs& ea, int64_t gi, double* feat) {
    const double px = ea.pts[3 * gi], py = ea.pts[3 * gi + 1], pz = ea.pts[3 * gi + 2];
    CompSink sink{feat, ea.nao};
    for (int sh = threadIdx.x; sh < ea.nshell; sh += blockDim.x) {
        const ShellDesc b = ea.shells[sh];
        eval_shell_any<double, GRAD, LMAX>(b, px - b.x, py - b.y, pz - b.z, ea.exps, ea.coefs, sink);
    }
    __syncthreads();
}

// Projections lr[s2] = sum_a scale_a comp_a(g) . WT[s2][a] for s2 in
// [s2a, s2b): one warp per s2 when the range is wide, otherwise the warps
// split each s2's AO range and add their partial sums (part: >= 256 doubles).
template <bool GRAD>
__device__ void exact_projections(const ExactArgs& ea, const double* feat, double* lr, int s2a, int s2b,
                                  double* part) {
    const int nao = ea.nao;
    const int64_t d = static_cast<int64_t>(ea.naxes) * nao;
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32, nw = blockDim.x / 32;
    const int cnt = s2b - s2a;
    const int nseg = max(1, nw / cnt);
    for (int item = warp; item < cnt * nseg; item += nw) {
        const int si = item / nseg, seg = item % nseg;
        const double* wt = ea.WT + (s2a + si) * d;
        double acc = 0;
        int a = 0;
        // four axis entries per pass, so their weight loads are in flight
        // together; each entry's sum and the order of acc are unchanged
        for (; a + 4 <= ea.naxes; a += 4) {
            const double* f0 = feat + (GRAD ? ea.comp[a] : 0) * nao;
            const double* f1 = feat + (GRAD ? ea.comp[a + 1] : 0) * nao;
            const double* f2 = feat + (GRAD ? ea.comp[a + 2] : 0) * nao;
            const double* f3 = feat + (GRAD ? ea.comp[a + 3] : 0) * nao;
            const double* w0 = wt + static_cast<int64_t>(a) * nao;
            double p0 = 0, p1 = 0, p2 = 0, p3 = 0;
            for (int i = seg * 32 + lane; i < nao; i += 32 * nseg) {
                const double x0 = w0[i], x1 = w0[nao + i], x2 = w0[2 * nao + i], x3 = w0[3 * nao + i];
                p0 += f0[i] * x0;
                p1 += f1[i] * x1;
                p2 += f2[i] * x2;
                p3 += f3[i] * x3;
            }
            acc += ea.scales[a] * p0;
            acc += ea.scales[a + 1] * p1;
            acc += ea.scales[a + 2] * p2;
            acc += ea.scales[a + 3] * p3;
        }
        for (; a < ea.naxes; ++a) {
            const double* f = feat + (GRAD ? ea.comp[a] : 0) * nao;
            const double* wa = wt + static_cast<int64_t>(a) * nao;
            double pa = 0;
            for (int i = seg * 32 + lane; i < nao; i += 32 * nseg) pa += f[i] * wa[i];
            acc += ea.scales[a] * pa;
        }
        acc = warp_sum(acc);
        if (lane == 0) part[item] = acc;
    }
    __syncthreads();
    for (int si = threadIdx.x; si < cnt; si += blockDim.x) {
        double sum = 0;
        for (int seg = 0; seg < nseg; ++seg) sum += part[si * nseg + seg];
        lr[s2a + si] = sum;
    }
    __syncthreads();
}

// Sketch column g from its projections (warp 0): y_s = sw lr[s] lr[ell+s],
// the j previous reflectors, rows stored, squared trailing norm into est[g]
// with a zero bound.  Returns the column's argmax key (lane 0).
__device__ ArgKey exact_finish(const ExactArgs& ea, const QrState& st, int64_t g, int64_t j, const double* lr,
                               double* y, const double* vhist, const double* tau) {
    const int lane = threadIdx.x % 32;
    const int64_t m = st.m;
    const int64_t gi = ea.index[g];
    const double sw = sqrt(fabs(ea.w[gi])) / sqrt(static_cast<double>(ea.ell));
    for (int64_t s = lane; s < m; s += 32) y[s] = sw * lr[s] * lr[ea.ell + s];
    __syncwarp();
    for (int64_t i = 0; i < j; ++i) {
        const double t = tau[i];
        if (t == 0.0) continue;
        const double* v = vhist + i * m;
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
    ArgKey k = key_none();
    if (lane == 0) {
        st.est[g] = nrm;
        st.delta[g] = 0.0;
        k = ArgKey{nrm, st.pos[g], g};
    }
    return k;
}

// Re-verifies the candidates cand[0 .. *count) listed on the device this step
// (fixed grid, so the host needs no count before the launch) and leaves one
// argmax key per block.  Few candidates: each column's projections are split
// over several blocks (each evaluates the point's AOs itself); the block that
// completes a column last, seen by an atomic counter, finishes it.  Many:
// one block per column.
template <bool GRAD, int LMAX, int NTHR>
__global__ void __launch_bounds__(NTHR)
exact_columns_kernel(ExactArgs ea, QrState st, const int64_t* cand, int64_t j, unsigned long long* total,
                     double* lr_split, unsigned* done) {
    constexpr int kNComp = GRAD ? 4 : 1;
    extern __shared__ double feat[];
    __shared__ double part[256];
    __shared__ int last_sh;
    double* lr = feat + kNComp * ea.nao;
    double* y = lr + 2 * ea.ell;
    const int64_t nc = *st.count;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(total, static_cast<unsigned long long>(nc));
    const int ell2 = static_cast<int>(2 * ea.ell);
    int nsl = 1;
    if (nc > 0 && nc <= kSplitCands) nsl = max(1, min(ell2, static_cast<int>(gridDim.x / nc)));
    const int per = (ell2 + nsl - 1) / nsl;
    nsl = (ell2 + per - 1) / per;
    ArgKey best = key_none();
    for (int64_t it = blockIdx.x; it < nc * nsl; it += gridDim.x) {
        const int64_t ci = it / nsl;
        const int sl = static_cast<int>(it % nsl);
        const int64_t g = cand[ci];
        const int s2a = sl * per, s2b = min(ell2, s2a + per);
        exact_features<GRAD, LMAX>(ea, ea.index[g], feat);
        exact_projections<GRAD>(ea, feat, lr, s2a, s2b, part);
        if (nsl > 1) {
            for (int s2 = s2a + threadIdx.x; s2 < s2b; s2 += blockDim.x) lr_split[ci * ell2 + s2] = lr[s2];
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) last_sh = atomicAdd(&done[ci], 1u) == static_cast<unsigned>(nsl - 1);
            __syncthreads();
            if (!last_sh) continue;
            __threadfence();
            for (int s2 = threadIdx.x; s2 < ell2; s2 += blockDim.x) lr[s2] = __ldcg(&lr_split[ci * ell2 + s2]);
            if (threadIdx.x == 0) done[ci] = 0u;   // ready for the next step
            __syncthreads();
        }
        // the j reflectors and their tau, staged by the whole block into the
        // feature area (no longer read) when they fit, so the one warp that
        // applies them in sequence reads shared memory
        const double* vh = st.vhist;
        const double* tau = st.tau;
        if ((j + 1) * st.m <= static_cast<int64_t>(kNComp) * ea.nao) {
            for (int64_t i = threadIdx.x; i < j * st.m; i += blockDim.x) feat[i] = st.vhist[i];
            for (int64_t i = threadIdx.x; i < j; i += blockDim.x) feat[j * st.m + i] = st.tau[i];
            __syncthreads();
            vh = feat;
            tau = feat + j * st.m;
        }
        if (threadIdx.x < 32) {
            const ArgKey k = exact_finish(ea, st, g, j, lr, y, vh, tau);
            if (threadIdx.x == 0 && key_better(k, best)) best = k;
        }
        __syncthreads();   // feat is reused by the next item
    }
    if (threadIdx.x == 0) st.xpartial[blockIdx.x] = best;
}

using ExactKernelFn = void (*)(ExactArgs, QrState, const int64_t*, int64_t, unsigned long long*, double*,
                               unsigned*);
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

// ---- one rank's share of a distributed pivoted QR ----------------------------------
// pos[g] = offset + g (global positions of this rank's columns)
__global__ void iota_offset_kernel(int64_t* pos, int64_t n, int64_t offset) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) pos[i] = offset + i;
}

// Best of the per-block keys (and re-verification keys) of this rank.
__global__ void __launch_bounds__(1024) reduce_keys_kernel(const ArgKey* partial, int nblocks, const ArgKey* xpartial,
                                                           int nx, ArgKey* out) {
    __shared__ ArgKey ksh[32];
    ArgKey k = key_none();
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        if (key_better(partial[b], k)) k = partial[b];
    for (int b = threadIdx.x; b < nx; b += blockDim.x)
        if (key_better(xpartial[b], k)) k = xpartial[b];
    k = block_best<1024>(k, ksh);
    if (threadIdx.x == 0) *out = k;
}

// Pivot step j of a distributed QR, identical on every rank: the owner marks
// its pivot column selected (position j); the rank holding the column at
// position j moves it to the pivot's former position (dgeqp3's swap); every
// rank builds reflector j from the pivot column's rows (the arithmetic of
// qr_pivot_kernel) and clears the verified-mode step state.
__global__ void shard_pivot_kernel(QrState st, int64_t j, const double* __restrict__ rows, int64_t pivot_col,
                                   int64_t pivot_pos, int64_t moved_col, double* beta_out) {
    __shared__ double sh_scale;
    if (threadIdx.x == 0) {
        if (pivot_col >= 0) {
            st.selected[pivot_col] = 1;
            st.pos[pivot_col] = j;
        }
        if (moved_col >= 0) st.pos[moved_col] = pivot_pos;
        if (st.count) {
            *st.count = 0;
            *st.lb_bits = 0ull;
        }
        const double alpha = rows[j];
        double xnorm = 0;
        for (int64_t i = j + 1; i < st.m; ++i) xnorm = hypot(xnorm, rows[i]);
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
        *beta_out = beta;
        sh_scale = scale;
    }
    __syncthreads();
    double* v = st.vhist + j * st.m;
    for (int64_t i = threadIdx.x; i < st.m; i += blockDim.x)
        v[i] = i < j ? 0.0 : i == j ? 1.0 : rows[i] * sh_scale;
}

ExactArgs make_exact_args(const ExactSketchSource& ex) {
    ExactArgs ea{};
    const Context& c = *ex.ctx;
    ea.shells = c.d_shells; ea.nshell = c.nshell; ea.exps = c.d_exp; ea.coefs = c.d_coef;
    ea.nao = c.nao; ea.naxes = ex.naxes; ea.grad = 0;
    for (int a = 0; a < ex.naxes; ++a) { ea.comp[a] = ex.comp[a]; ea.grad |= ex.comp[a] > 0; }
    ea.scales = ex.scales; ea.WT = ex.WT; ea.pts = ex.pts; ea.index = ex.index;
    ea.w = ex.w; ea.ell = ex.ell;
    return ea;
}

}  // namespace

struct QrShard::Impl {
    cudaStream_t s;
    int64_t m, n, steps, ldy;
    int nblocks;
    bool pairs;
    QrState st;
    DeviceBuffer<int64_t> pos, col_at, jpvt, cand, count;
    DeviceBuffer<char> selected;
    DeviceBuffer<double> vhist, tau, diag, energy, est, lr_split, rows, beta, seg_ub;
    DeviceBuffer<ArgKey> partial, xpartial, key, seg_key;
    DeviceBuffer<unsigned long long> lb_bits, reverified;
    DeviceBuffer<unsigned> done;
    bool verified = false;
    ExactArgs ea{};
    size_t exact_smem = 0;
    ExactKernel exact_kernel;
};

QrShard::QrShard(double* Yt, int64_t ldy, int64_t m, int64_t n, int64_t pos_offset, const ExactSketchSource* exact,
                 cudaStream_t s)
    : d_(new Impl) {
    Impl& d = *d_;
    d.s = s;
    d.m = m;
    d.n = n;
    d.ldy = ldy;
    d.steps = m;
    require(m >= 1 && m <= kMaxSketchRows, "distributed sketch QR supports 1 to 128 sketch rows");
    d.nblocks = static_cast<int>((n + kQrThreads - 1) / kQrThreads);
    const size_t nn = static_cast<size_t>(std::max<int64_t>(n, 1));
    d.pos.reset(nn, s);
    d.col_at.reset(nn, s);
    d.jpvt.reset(m, s);
    d.selected.reset(nn, s);
    d.vhist.reset(static_cast<size_t>(m * m), s);
    d.tau.reset(m, s);
    d.diag.reset(m, s);
    d.energy.reset(m + 1, s);
    d.partial.reset(std::max(d.nblocks, 1), s);
    d.key.reset(1, s);
    d.rows.reset(m, s);
    d.beta.reset(1, s);
    d.selected.zero(s);
    d.energy.zero(s);
    d.tau.zero(s);
    if (n > 0) {
        iota_offset_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(d.pos.get(), n, pos_offset);
        ISDF_LAUNCH_CHECK();
    }
    d.st = QrState{Yt, ldy, m, n, d.pos.get(), d.col_at.get(), d.selected.get(), d.vhist.get(), d.tau.get(),
                   d.diag.get(), d.energy.get(), d.jpvt.get(), d.partial.get(), nullptr, nullptr, nullptr,
                   nullptr, nullptr};
    d.reverified.reset(1, s);
    d.reverified.zero(s);
    if (exact) {
        d.verified = true;
        d.est.reset(nn, s);
        d.lb_bits.reset(1, s);
        d.cand.reset(nn, s);
        d.count.reset(1, s);
        d.xpartial.reset(kExactBlocks, s);
        d.seg_ub.reset(std::max(d.nblocks, 1), s);
        d.seg_key.reset(std::max(d.nblocks, 1), s);
        d.lr_split.reset(static_cast<size_t>(kSplitCands) * 2 * exact->ell, s);
        d.done.reset(kSplitCands, s);
        d.lb_bits.zero(s);
        d.count.zero(s);
        d.done.zero(s);
        d.st.est = d.est.get();
        d.st.seg_ub = d.seg_ub.get();
        d.st.seg_key = d.seg_key.get();
        d.st.delta = exact->delta;
        d.st.lb_bits = d.lb_bits.get();
        d.st.count = d.count.get();
        d.st.xpartial = d.xpartial.get();
        d.ea = make_exact_args(*exact);
        d.exact_smem = (static_cast<size_t>(d.ea.grad ? 4 : 1) * exact->ctx->nao + 2 * exact->ell + m) * sizeof(double);
        d.exact_kernel = pick_exact_kernel(d.ea.grad != 0, exact->ctx->lmax);
        ISDF_CUDA(cudaFuncSetAttribute(d.exact_kernel.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(d.exact_smem)));
    }
    constexpr size_t kStagedBytes = static_cast<size_t>(kRegRows) * kQrThreads * sizeof(double);
    ISDF_CUDA(cudaFuncSetAttribute(qr_update_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kStagedBytes)));
    ISDF_CUDA(cudaFuncSetAttribute(qr_update_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kStagedBytes)));
    d.pairs = ldy % 2 == 0 && reinterpret_cast<uintptr_t>(Yt) % 16 == 0;
}

QrShard::~QrShard() = default;

QrShardKey QrShard::update(int64_t j, double* energy_part, double* lower_bound) {
    Impl& d = *d_;
    QrShardKey out{-1.0, INT64_MAX, -1};
    *energy_part = 0.0;
    *lower_bound = 0.0;
    if (d.n == 0) return out;
    {
        ISDF_PROFILE("qrcp_sketch_update", d.s);
        const int64_t touched = d.m - (j > 0 ? j - 1 : 0);
        const size_t staged = static_cast<size_t>(touched) * kQrThreads * sizeof(double);
        if (touched <= kRegRows && d.pairs)
            qr_update_pairs_kernel<<<d.nblocks, kPairThreads, staged, d.s>>>(d.st, j);
        else if (touched <= kRegRows)
            qr_update_kernel<true><<<d.nblocks, kQrThreads, staged, d.s>>>(d.st, j);
        else
            qr_update_kernel<false><<<d.nblocks, kQrThreads, 0, d.s>>>(d.st, j);
        ISDF_LAUNCH_CHECK();
    }
    if (j > 0)
        ISDF_CUDA(cudaMemcpyAsync(energy_part, d.energy.get() + (j - 1), sizeof(double), cudaMemcpyDeviceToHost, d.s));
    if (j < d.m) {
        if (d.verified) {
            unsigned long long bits = 0;
            ISDF_CUDA(cudaMemcpyAsync(&bits, d.lb_bits.get(), sizeof(bits), cudaMemcpyDeviceToHost, d.s));
            ISDF_CUDA(cudaStreamSynchronize(d.s));
            std::memcpy(lower_bound, &bits, sizeof(double));
            return out;
        }
        reduce_keys_kernel<<<1, 1024, 0, d.s>>>(d.partial.get(), d.nblocks, nullptr, 0, d.key.get());
        ISDF_LAUNCH_CHECK();
        ISDF_CUDA(cudaMemcpyAsync(&out, d.key.get(), sizeof(out), cudaMemcpyDeviceToHost, d.s));
    }
    ISDF_CUDA(cudaStreamSynchronize(d.s));
    return out;
}

QrShardKey QrShard::verify(int64_t j, double lower_bound) {
    Impl& d = *d_;
    QrShardKey out{-1.0, INT64_MAX, -1};
    if (d.n == 0) return out;
    require(d.verified, "verify() needs error bounds");
    unsigned long long bits = 0;
    std::memcpy(&bits, &lower_bound, sizeof(bits));
    ISDF_CUDA(cudaMemcpyAsync(d.lb_bits.get(), &bits, sizeof(bits), cudaMemcpyHostToDevice, d.s));
    {
        ISDF_PROFILE("qrcp_sketch_verify", d.s);
        candidates_kernel<<<cand_blocks(d.nblocks), kQrThreads, 0, d.s>>>(d.st, d.cand.get(), d.nblocks);
        ISDF_LAUNCH_CHECK();
        d.exact_kernel.fn<<<kExactBlocks, d.exact_kernel.threads, d.exact_smem, d.s>>>(
            d.ea, d.st, d.cand.get(), j, d.reverified.get(), d.lr_split.get(), d.done.get());
        ISDF_LAUNCH_CHECK();
    }
    reduce_keys_kernel<<<1, 1024, 0, d.s>>>(d.partial.get(), cand_blocks(d.nblocks), d.xpartial.get(), kExactBlocks,
                                            d.key.get());
    ISDF_LAUNCH_CHECK();
    ISDF_CUDA(cudaMemcpyAsync(&out, d.key.get(), sizeof(out), cudaMemcpyDeviceToHost, d.s));
    ISDF_CUDA(cudaStreamSynchronize(d.s));
    return out;
}

void QrShard::column(int64_t col, double* rows_host) {
    Impl& d = *d_;
    require(col >= 0 && col < d.n, "pivot column outside this rank's columns");
    ISDF_CUDA(cudaMemcpy2DAsync(rows_host, sizeof(double), d.st.Yt + col, d.ldy * sizeof(double), sizeof(double),
                                d.m, cudaMemcpyDeviceToHost, d.s));
    ISDF_CUDA(cudaStreamSynchronize(d.s));
}

double QrShard::pivot(int64_t j, const double* rows_host, int64_t pivot_col, int64_t pivot_pos, int64_t moved_col) {
    Impl& d = *d_;
    require(j >= 0 && j < d.m, "pivot step outside the sketch rows");
    require(pivot_col < d.n && moved_col < d.n, "pivot or moved column outside this rank's columns");
    ISDF_CUDA(cudaMemcpyAsync(d.rows.get(), rows_host, d.m * sizeof(double), cudaMemcpyHostToDevice, d.s));
    {
        ISDF_PROFILE("qrcp_sketch_pivot", d.s);
        shard_pivot_kernel<<<1, 128, 0, d.s>>>(d.st, j, d.rows.get(), pivot_col, pivot_pos, moved_col, d.beta.get());
        ISDF_LAUNCH_CHECK();
    }
    double beta = 0;
    ISDF_CUDA(cudaMemcpyAsync(&beta, d.beta.get(), sizeof(beta), cudaMemcpyDeviceToHost, d.s));
    ISDF_CUDA(cudaStreamSynchronize(d.s));
    return beta;
}

int64_t QrShard::reverified() const {
    unsigned long long r = 0;
    ISDF_CUDA(cudaMemcpyAsync(&r, d_->reverified.get(), sizeof(r), cudaMemcpyDeviceToHost, d_->s));
    ISDF_CUDA(cudaStreamSynchronize(d_->s));
    return static_cast<int64_t>(r);
}

SketchQR qrcp_sketch(double* Yt, int64_t ldy, int64_t m, int64_t n, cudaStream_t s,
                     const ExactSketchSource* exact) {
    SketchQR out;
    const int64_t steps = std::min(m, n);
    if (steps == 0) return out;
    if (exact) require(m <= kMaxSketchRows, "verified sketch QR supports at most 128 sketch rows");
    const int nblocks = static_cast<int>((n + kQrThreads - 1) / kQrThreads);
    DeviceBuffer<int64_t> pos(n, s), col_at(n, s), jpvt(steps, s);
    DeviceBuffer<char> selected(n, s);
    DeviceBuffer<double> vhist(static_cast<size_t>(m * steps), s), tau(steps, s), diag(steps, s),
        energy(steps, s);
    DeviceBuffer<ArgKey> partial(nblocks, s), xpartial, seg_key;
    DeviceBuffer<double> est, lr_split, seg_ub;
    DeviceBuffer<unsigned long long> lb_bits;
    DeviceBuffer<unsigned> done;
    DeviceBuffer<int64_t> cand, count;
    selected.zero(s);
    energy.zero(s);
    iota_i64(pos.get(), n, s);
    iota_i64(col_at.get(), n, s);
    QrState st{Yt, ldy, m, n, pos.get(), col_at.get(), selected.get(), vhist.get(), tau.get(),
               diag.get(), energy.get(), jpvt.get(), partial.get(), nullptr, nullptr, nullptr, nullptr,
               nullptr};
    ExactArgs ea{};
    size_t exact_smem = 0;
    ExactKernel exact_kernel;
    if (exact) {
        est.reset(n, s);
        lb_bits.reset(1, s);
        cand.reset(n, s);
        count.reset(1, s);
        xpartial.reset(kExactBlocks, s);
        seg_ub.reset(nblocks, s);
        seg_key.reset(nblocks, s);
        lr_split.reset(static_cast<size_t>(kSplitCands) * 2 * exact->ell, s);
        done.reset(kSplitCands, s);
        lb_bits.zero(s);
        count.zero(s);
        done.zero(s);
        st.est = est.get();
        st.seg_ub = seg_ub.get();
        st.seg_key = seg_key.get();
        st.delta = exact->delta;
        st.lb_bits = lb_bits.get();
        st.count = count.get();
        st.xpartial = xpartial.get();
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
    constexpr size_t kStagedBytes = static_cast<size_t>(kRegRows) * kQrThreads * sizeof(double);
    ISDF_CUDA(cudaFuncSetAttribute(qr_update_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kStagedBytes)));
    ISDF_CUDA(cudaFuncSetAttribute(qr_update_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kStagedBytes)));
    // two columns per thread where every row of the pairs is 16-byte aligned
    const bool pairs = st.ldy % 2 == 0 && reinterpret_cast<uintptr_t>(st.Yt) % 16 == 0;
    for (int64_t j = 0; j <= steps; ++j) {
        {
            ISDF_PROFILE("qrcp_sketch_update", s);
            const int64_t touched = m - (j > 0 ? j - 1 : 0);
            // shared memory for the rows this step stages only: later steps
            // (fewer rows) keep more blocks, and more copies in flight, per SM
            const size_t staged = static_cast<size_t>(touched) * kQrThreads * sizeof(double);
            if (touched <= kRegRows && pairs)
                qr_update_pairs_kernel<<<nblocks, kPairThreads, staged, s>>>(st, j);
            else if (touched <= kRegRows)
                qr_update_kernel<true><<<nblocks, kQrThreads, staged, s>>>(st, j);
            else
                qr_update_kernel<false><<<nblocks, kQrThreads, 0, s>>>(st, j);
            ISDF_LAUNCH_CHECK();
        }
        if (j == steps) break;
        if (exact) {
            ISDF_PROFILE("qrcp_sketch_verify", s);
            candidates_kernel<<<cand_blocks(nblocks), kQrThreads, 0, s>>>(st, cand.get(), nblocks);
            ISDF_LAUNCH_CHECK();
            exact_kernel.fn<<<kExactBlocks, exact_kernel.threads, exact_smem, s>>>(
                ea, st, cand.get(), j, reverified_d.get(), lr_split.get(), done.get());
            ISDF_LAUNCH_CHECK();
        }
        {
            ISDF_PROFILE("qrcp_sketch_pivot", s);
            // verified: one key per candidate-scan block, else one per update block
            qr_pivot_kernel<<<1, 1024, 0, s>>>(st, j, exact ? cand_blocks(nblocks) : nblocks,
                                               exact ? kExactBlocks : 0);
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
