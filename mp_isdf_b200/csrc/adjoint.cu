// Nuclear gradient of the ISDF density functional (not in the reference).
//
//   E = sum_g w_g rho(g)^2,   rho(g) = sum_k Theta_kg w_k rho_a(k) = h_g . z,
//   h_g = (Phi_a phi_g)^2,  z = M^+ rho_a,  M = (Phi_a Phi_a^T)^2,
//   rho_a(k) = phi(a_k)^T D phi(a_k),
// with grid points, anchors and weights fixed and d phi_mu / d R_A = -grad_r phi_mu
// for AOs mu on atom A (the AO gradient formula of cpp/src/ao_eval.cpp:240-244).
// With u_g = 2 w_g rho_g and alpha_gk = 2 u_g z_k G_gk (G = Phi_g Phi_a^T):
//   grid terms    dE/dR_A -= sum_g sum_{mu in A} (alpha_g Phi_a)_mu grad phi_mu(g)
//   anchor terms  dE/dR_A -= sum_k sum_{mu in A} c_k,mu grad phi_mu(a_k),
//                 c = alpha^T Phi_g + 2 y o (Phi_a D) - (W + W^T) Phi_a,
//                 y = M^+ v, v = sum_g u_g h_g, W = 2 S o (y z^T), S = Phi_a Phi_a^T.
// The grid pass is one fused kernel (adjoint_grid_kernel): per tile of 128
// points it evaluates the FP64 AO values (sweep 1: G, rho, u, alpha, E, v),
// then values and gradients again (sweep 2) and folds both the grid terms and
// the alpha^T Phi_g part of the anchor coefficients,
//   sum_g phi_mu(g) sum_k alpha_gk grad phi_mu(a_k),
// straight into per-atom sums; Phi and grad Phi never reach HBM.  Bases or
// anchor counts beyond its limits take a chunked path (AO chunks in HBM and
// GEMMs).
#include "ao_device.cuh"
#include "isdf_adjoint.h"
#include "isdf_reduce.cuh"

#include <algorithm>
#include <cmath>

namespace isdf {
namespace {

unsigned nblk(int64_t n) { return static_cast<unsigned>((n + 255) / 256); }

// per point: h = G^2, rho = h.z, u = 2 w rho; E += w rho^2; v += u h;
// alpha[g][k] = 2 u z_k G_gk (row-major) and alphaT[k][g] (for B += alpha^T Phi)
__global__ void __launch_bounds__(256)
adjoint_point_kernel(const double* __restrict__ G, const double* __restrict__ w, int64_t b, int k,
                     const double* __restrict__ z, double* __restrict__ alpha,
                     double* __restrict__ alphaT, double* __restrict__ v, double* __restrict__ energy) {
    __shared__ double sh[8];
    __shared__ double vs[64];
    for (int i = threadIdx.x; i < k && i < 64; i += blockDim.x) vs[i] = 0.0;
    __syncthreads();
    const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double e = 0;
    if (g < b) {
        const double* Gg = G + g * k;
        double rho = 0;
        for (int a = 0; a < k; ++a) rho += Gg[a] * Gg[a] * z[a];
        const double u = 2.0 * w[g] * rho;
        e = w[g] * rho * rho;
        for (int a = 0; a < k; ++a) {
            const double al = 2.0 * u * z[a] * Gg[a];
            alpha[g * k + a] = al;
            alphaT[a * b + g] = al;
            if (a < 64) atomicAdd(&vs[a], u * Gg[a] * Gg[a]);
            else atomicAdd(&v[a], u * Gg[a] * Gg[a]);
        }
    }
    e = block_sum<256>(e, sh);
    if (threadIdx.x == 0) atomicAdd(energy, e);
    for (int i = threadIdx.x; i < k && i < 64; i += blockDim.x) atomicAdd(&v[i], vs[i]);
}

// acc[c][mu] += sum_g beta[g][mu] * grad[c][g][mu] over the chunk
__global__ void __launch_bounds__(256)
column_dot_kernel(const double* __restrict__ beta, const double* __restrict__ grad, int64_t b,
                  int nao, double* __restrict__ acc) {
    const int mu = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (mu >= nao) return;
    const double* gr = grad + static_cast<int64_t>(c) * b * nao;
    double s = 0;
    for (int64_t g = 0; g < b; ++g) s += beta[g * nao + mu] * gr[g * nao + mu];
    acc[c * nao + mu] += s;
}

__global__ void gather_kernel(const double* __restrict__ pts, const double* __restrict__ w,
                              const int64_t* __restrict__ idx, int64_t n, double* __restrict__ op,
                              double* __restrict__ ow) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t g = idx[i];
    op[3 * i] = pts[3 * g]; op[3 * i + 1] = pts[3 * g + 1]; op[3 * i + 2] = pts[3 * g + 2];
    ow[i] = w[g];
}

// Small anchor-side algebra, one block: see the header comment.
__global__ void anchor_terms_kernel(int k, int nao, const double* __restrict__ phia,
                                    const double* __restrict__ S, const double* __restrict__ T,
                                    const double* __restrict__ DphiT, const double* __restrict__ z,
                                    const double* __restrict__ v, double* __restrict__ y,
                                    double* __restrict__ W) {
    // y = T v
    for (int a = threadIdx.x; a < k; a += blockDim.x) {
        double s = 0;
        for (int b = 0; b < k; ++b) s += T[a * k + b] * v[b];
        y[a] = s;
    }
    __syncthreads();
    // W = 2 S o (y z^T) + its transpose (symmetrised coefficient of dS)
    for (int i = threadIdx.x; i < k * k; i += blockDim.x) {
        const int a = i / k, b = i % k;
        W[i] = 2.0 * S[i] * (y[a] * z[b] + y[b] * z[a]);
    }
    (void)phia; (void)DphiT; (void)nao;
}

// coef[k][mu] = B[k][mu] + 2 y_k (Phi_a D)[k][mu] - (W Phi_a)[k][mu]
__global__ void anchor_coef_kernel(int k, int nao, const double* __restrict__ B,
                                   const double* __restrict__ PhiD, const double* __restrict__ WPhi,
                                   const double* __restrict__ y, double* __restrict__ coef) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k * nao) return;
    const int a = i / nao;
    coef[i] = B[i] + 2.0 * y[a] * PhiD[i] - WPhi[i];
}

// acc[c][mu] += sum_k coef[k][mu] dphi_a[c][k][mu]
__global__ void anchor_contrib_kernel(int k, int nao, const double* __restrict__ coef,
                                      const double* __restrict__ dphia, double* __restrict__ acc) {
    const int mu = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (mu >= nao) return;
    double s = 0;
    for (int a = 0; a < k; ++a) s += coef[a * nao + mu] * dphia[(static_cast<int64_t>(c) * k + a) * nao + mu];
    acc[c * nao + mu] += s;
}

// rho_a(k) = (Phi_a D)[k] . Phi_a[k]
__global__ void rho_anchor_kernel(int k, int nao, const double* __restrict__ PhiD,
                                  const double* __restrict__ phia, double* __restrict__ rho) {
    const int a = blockIdx.x;
    double s = 0;
    for (int mu = threadIdx.x; mu < nao; mu += 32) s += PhiD[a * nao + mu] * phia[a * nao + mu];
    s = warp_sum(s);
    if (threadIdx.x == 0) rho[a] = s;
}

__global__ void matvec_kernel(int k, const double* __restrict__ T, const double* __restrict__ x,
                              double* __restrict__ y) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= k) return;
    double s = 0;
    for (int b = 0; b < k; ++b) s += T[a * k + b] * x[b];
    y[a] = s;
}

// ---- fused grid pass -----------------------------------------------------------
constexpr int kAdjPts = 128;      // points per tile
constexpr int kAdjLanes = 2;      // shell lanes per point
constexpr int kAdjMaxAtoms = 1024;
constexpr double kAdjCut = kExpCut * 1.0001;   // margin for the FP32 screening exponent

struct AdjGridArgs {
    const ShellDesc* shells;
    int nshell, nao, natm;
    const double* exps;
    const double* coefs;
    const double* pts;
    const double* w;
    const int64_t* index;      // kept points
    int64_t n;
    const double* pk;          // [nao][4][KMAX]: Phi_a and its d/dx, d/dy, d/dz per AO, anchors >= k zero
    const double* z;           // [KMAX], zero padded
    double* gacc;              // [natm][3] += sum_g sum_{mu in atom} (beta grad phi + phi t)
    double* v;                 // [KMAX] += sum_g u_g G_gk^2
    double* energy;            // += sum_g w_g rho_g^2
};

// sweep 1: G[a] += phi_mu(g) Phi_a[a][mu]; an AO's anchor values are
// contiguous, read as 16-byte pairs
template <int KMAX>
struct GramSink {
    const double* pk;
    double G[KMAX];
    template <int C>
    __device__ __forceinline__ void put(int ao, double v) {
        if constexpr (C == 0) {
            const double2* q = reinterpret_cast<const double2*>(pk + static_cast<int64_t>(ao) * 4 * KMAX);
#pragma unroll
            for (int a = 0; a < KMAX / 2; ++a) {
                const double2 x = __ldg(q + a);
                G[2 * a] += v * x.x;
                G[2 * a + 1] += v * x.y;
            }
        }
    }
};

// sweep 2: per AO, beta = alpha . Phi_a[:, mu] and t = alpha . grad phi_mu(a_:);
// acc += beta grad phi_mu(g) + phi_mu(g) t
template <int KMAX>
struct GradSink {
    const double* pk;
    double al[KMAX];
    double beta, acc[3];
    template <int C>
    __device__ __forceinline__ void put(int ao, double v) {
        if constexpr (C == 0) {
            double b = 0, t0 = 0, t1 = 0, t2 = 0;
            const double2* q = reinterpret_cast<const double2*>(pk + static_cast<int64_t>(ao) * 4 * KMAX);
#pragma unroll
            for (int a = 0; a < KMAX / 2; ++a) {
                const double2 x = __ldg(q + a), x0 = __ldg(q + KMAX / 2 + a), x1 = __ldg(q + KMAX + a),
                              x2 = __ldg(q + 3 * KMAX / 2 + a);
                b += al[2 * a] * x.x;
                t0 += al[2 * a] * x0.x;
                t1 += al[2 * a] * x1.x;
                t2 += al[2 * a] * x2.x;
                b += al[2 * a + 1] * x.y;
                t0 += al[2 * a + 1] * x0.y;
                t1 += al[2 * a + 1] * x1.y;
                t2 += al[2 * a + 1] * x2.y;
            }
            beta = b;
            acc[0] += v * t0;
            acc[1] += v * t1;
            acc[2] += v * t2;
        } else {
            acc[C - 1] += beta * v;
        }
    }
};

// GRAD = false: the energy alone (sweep 1 only).
template <int LMAX, int KMAX, bool GRAD>
__global__ void __launch_bounds__(kAdjPts * kAdjLanes, 1) adjoint_grid_kernel(AdjGridArgs args) {
    extern __shared__ double adj_smem[];
    double* Gs = adj_smem;                                   // [lanes][pts][KMAX]
    double* As = Gs + kAdjLanes * kAdjPts * KMAX;            // [pts][KMAX]
    double* grad_s = As + kAdjPts * KMAX;                    // [natm][3]
    double* v_s = grad_s + 3 * args.natm;                    // [KMAX]
    double* e_s = v_s + KMAX;                                // [1]
    const int tid = threadIdx.x, lane = tid % 32;
    const int p = tid % kAdjPts, sl = tid / kAdjPts;         // point, shell lane (warp-uniform)
    for (int i = tid; i < 3 * args.natm + KMAX + 1; i += blockDim.x) grad_s[i] = 0.0;
    __syncthreads();
    const int64_t ntiles = (args.n + kAdjPts - 1) / kAdjPts;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t g = tile * kAdjPts + p;
        const bool valid = g < args.n;
        double px = 0, py = 0, pz = 0, wg = 0;
        if (valid) {
            const int64_t gi = args.index[g];
            px = args.pts[3 * gi]; py = args.pts[3 * gi + 1]; pz = args.pts[3 * gi + 2];
            wg = args.w[gi];
        }
        // sweep 1: G = Phi_a phi_g, partial over this lane's shells
        GramSink<KMAX> gs{args.pk, {}};
#pragma unroll
        for (int a = 0; a < KMAX; ++a) gs.G[a] = 0.0;
        // a shell whose FP64 screening exponent puts all 32 points of the warp
        // beyond kExpCut is skipped (no value or gradient above kScreenFp64);
        // the shell loop is uniform over the warp (sl is)
        for (int sh = sl; sh < args.nshell; sh += kAdjLanes) {
            const ShellDesc b = args.shells[sh];
            const double dx = px - b.x, dy = py - b.y, dz = pz - b.z;
            if (__all_sync(0xffffffffu, !valid || b.scr64 * (dx * dx + dy * dy + dz * dz) > kAdjCut)) continue;
            if (valid) eval_shell_any<double, false, LMAX>(b, dx, dy, dz, args.exps, args.coefs, gs);
        }
#pragma unroll
        for (int a = 0; a < KMAX; ++a) Gs[(sl * kAdjPts + p) * KMAX + a] = gs.G[a];
        __syncthreads();
        if (sl == 0) {
            double G[KMAX], rho = 0;
#pragma unroll
            for (int a = 0; a < KMAX; ++a) {
                G[a] = 0;
                for (int l = 0; l < kAdjLanes; ++l) G[a] += Gs[(l * kAdjPts + p) * KMAX + a];
                rho += G[a] * G[a] * args.z[a];
            }
            const double u = 2.0 * wg * rho;
            double e = wg * rho * rho;
#pragma unroll
            for (int a = 0; a < KMAX; ++a) {
                As[p * KMAX + a] = 2.0 * u * args.z[a] * G[a];
                const double va = warp_allsum(u * G[a] * G[a]);
                if (lane == 0) atomicAdd(&v_s[a], va);
            }
            e = warp_allsum(e);
            if (lane == 0) atomicAdd(e_s, e);
        }
        __syncthreads();
        if constexpr (!GRAD) continue;
        // sweep 2: values and gradients; per shell, the warp's 32 points are
        // reduced before one shared-memory add per component
        GradSink<KMAX> gr{args.pk, {}, 0.0, {0.0, 0.0, 0.0}};
#pragma unroll
        for (int a = 0; a < KMAX; ++a) gr.al[a] = As[p * KMAX + a];
        for (int sh = sl; sh < args.nshell; sh += kAdjLanes) {
            const ShellDesc b = args.shells[sh];
            const double dx = px - b.x, dy = py - b.y, dz = pz - b.z;
            if (__all_sync(0xffffffffu, !valid || b.scr64 * (dx * dx + dy * dy + dz * dz) > kAdjCut)) continue;
            gr.acc[0] = gr.acc[1] = gr.acc[2] = 0.0;
            if (valid) eval_shell_any<double, true, LMAX>(b, dx, dy, dz, args.exps, args.coefs, gr);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double r = warp_allsum(gr.acc[c]);
                if (lane == 0) atomicAdd(&grad_s[3 * b.atom + c], r);
            }
        }
        __syncthreads();   // Gs and As are rewritten by the next tile
    }
    for (int i = tid; i < 3 * args.natm; i += blockDim.x) atomicAdd(&args.gacc[i], grad_s[i]);
    for (int i = tid; i < KMAX; i += blockDim.x) atomicAdd(&args.v[i], v_s[i]);
    if (tid == 0) atomicAdd(args.energy, *e_s);
}

template <int LMAX, int KMAX>
void launch_adjoint_grid(const AdjGridArgs& a, bool grad, cudaStream_t s) {
    const size_t smem = (static_cast<size_t>(kAdjLanes + 1) * kAdjPts * KMAX + 3 * a.natm + KMAX + 1) * sizeof(double);
    auto kern = grad ? adjoint_grid_kernel<LMAX, KMAX, true> : adjoint_grid_kernel<LMAX, KMAX, false>;
    ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    int dev = 0, nsm = 148;
    ISDF_CUDA(cudaGetDevice(&dev));
    ISDF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t ntiles = (a.n + kAdjPts - 1) / kAdjPts;
    kern<<<static_cast<unsigned>(std::min<int64_t>(ntiles, nsm)), kAdjPts * kAdjLanes, smem, s>>>(a);
    ISDF_LAUNCH_CHECK();
}

// rows [0, k) of a [rows_in][nao] matrix into a zero-padded [kmax][nao] one, per component
__global__ void pad_rows_kernel(const double* __restrict__ src, int ncomp, int k, int kmax, int nao,
                                double* __restrict__ dst) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t total = static_cast<int64_t>(ncomp) * kmax * nao;
    if (i >= total) return;
    const int mu = static_cast<int>(i % nao);
    const int a = static_cast<int>((i / nao) % kmax);
    const int c = static_cast<int>(i / (static_cast<int64_t>(nao) * kmax));
    dst[i] = a < k ? src[(static_cast<int64_t>(c) * k + a) * nao + mu] : 0.0;
}

// out[mu][c][a] = (c == 0 ? phi_a : dphi_a[c - 1])[a][mu] for a < k, 0 for k <= a < kmax
__global__ void pack_anchor_rows_kernel(const double* __restrict__ phia, const double* __restrict__ dphia, int k,
                                        int kmax, int nao, double* __restrict__ out) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<int64_t>(nao) * 4 * kmax) return;
    const int a = static_cast<int>(i % kmax);
    const int c = static_cast<int>((i / kmax) % 4);
    const int64_t mu = i / (4 * kmax);
    double v = 0.0;
    if (a < k && (c == 0 || dphia))
        v = c == 0 ? phia[static_cast<int64_t>(a) * nao + mu] : dphia[(static_cast<int64_t>(c - 1) * k + a) * nao + mu];
    out[i] = v;
}

}  // namespace

void set_atom_coords(Context& c, const double* coords) {
    for (int a = 0; a < c.natm; ++a)
        for (int x = 0; x < 3; ++x) {
            if (!std::isfinite(coords[3 * a + x])) fail(kInvalid, "atom coordinates must be finite");
            c.atom_xyz[3 * a + x] = coords[3 * a + x];
        }
    for (auto& sh : c.shells) {
        sh.x = c.atom_xyz[3 * sh.atom];
        sh.y = c.atom_xyz[3 * sh.atom + 1];
        sh.z = c.atom_xyz[3 * sh.atom + 2];
    }
    if (!c.shells.empty())
        ISDF_CUDA(cudaMemcpy(c.d_shells, c.shells.data(), c.shells.size() * sizeof(ShellDesc),
                             cudaMemcpyHostToDevice));
    upload_shell_centres(c);
}

namespace {

// Anchor-side quantities of both passes: Phi_a D, rho_a, z = T rho_a, S and
// (with gradients) the anchors' AO gradients.
struct AnchorSide {
    DeviceBuffer<double> dphia, Dd, PhiD, S, rhoa, z;
};
AnchorSide anchor_side(const Context& c, const AnchorFactor& f, const double* dm, bool want_grad, cudaStream_t s) {
    const int64_t k = f.k, nao = c.nao;
    AnchorSide a;
    a.dphia.reset(static_cast<size_t>(3 * k * nao), s);
    a.Dd.reset(static_cast<size_t>(nao * nao), s);
    a.PhiD.reset(static_cast<size_t>(k * nao), s);
    a.S.reset(static_cast<size_t>(k * k), s);
    a.rhoa.reset(k, s);
    a.z.reset(k, s);
    ISDF_CUDA(cudaMemcpyAsync(a.Dd.get(), dm, nao * nao * sizeof(double), cudaMemcpyHostToDevice, s));
    if (want_grad)   // anchor AO gradients (anchor coordinates gathered by the caller into f)
        eval_ao<double>(c, f.anchor_pts.get(), k, nullptr, a.dphia.get(), nao, s);
    gemm_f64(k, nao, nao, f.phi_a.get(), nao, 0, a.Dd.get(), nao, 0, a.PhiD.get(), nao, 0, 1, false, s);
    rho_anchor_kernel<<<static_cast<unsigned>(k), 32, 0, s>>>(static_cast<int>(k), static_cast<int>(nao),
                                                                a.PhiD.get(), f.phi_a.get(), a.rhoa.get());
    ISDF_LAUNCH_CHECK();
    matvec_kernel<<<nblk(k), 256, 0, s>>>(static_cast<int>(k), f.T.get(), a.rhoa.get(), a.z.get());
    ISDF_LAUNCH_CHECK();
    gemm_f64(k, k, nao, f.phi_a.get(), nao, 0, f.phi_aT.get(), k, 0, a.S.get(), k, 0, 1, false, s);
    return a;
}

}  // namespace

size_t adjoint_partial_size(const Context& c, int64_t k) {
    return static_cast<size_t>(1 + k + 3 * c.natm + k * c.nao + 3 * c.nao);
}

std::vector<double> energy_gradient_partial(const Context& c, const double* pts, const double* w,
                                            const KeptPoints& kp, const AnchorFactor& f, const double* dm,
                                            bool want_grad, cudaStream_t s) {
    const int64_t n = kp.n, k = f.k, nao = c.nao;
    std::vector<double> out(adjoint_partial_size(c, k), 0.0);
    if (k == 0 || n == 0) return out;
    require(k <= 4096, "too many anchors for the adjoint");
    AnchorSide as = anchor_side(c, f, dm, want_grad, s);
    const DeviceBuffer<double>& dphia = as.dphia;
    const DeviceBuffer<double>& z = as.z;
    DeviceBuffer<double> v(k, s), B(static_cast<size_t>(k * nao), s), acc(static_cast<size_t>(3 * nao), s),
        energy(1, s);
    v.zero(s); B.zero(s); acc.zero(s); energy.zero(s);

    const int kmax = k <= 4 ? 4 : k <= 8 ? 8 : k <= 12 ? 12 : k <= 16 ? 16 : 32;
    const size_t fused_smem =
        (static_cast<size_t>(kAdjLanes + 1) * kAdjPts * kmax + 3 * c.natm + kmax + 1) * sizeof(double);
    const bool fused = k <= 32 && c.natm <= kAdjMaxAtoms && fused_smem <= 200 * 1024;
    DeviceBuffer<double> gacc(static_cast<size_t>(3 * c.natm), s);
    gacc.zero(s);
    if (fused) {
        ISDF_PROFILE("adjoint_grid", s);
        // anchor values and gradients per AO, contiguous (16-byte pair loads)
        DeviceBuffer<double> pk(static_cast<size_t>(4 * kmax * nao), s), z_pad(kmax, s);
        pack_anchor_rows_kernel<<<nblk(4 * kmax * nao), 256, 0, s>>>(f.phi_a.get(), want_grad ? dphia.get() : nullptr,
                                                                    static_cast<int>(k), kmax, static_cast<int>(nao),
                                                                    pk.get());
        ISDF_LAUNCH_CHECK();
        pad_rows_kernel<<<1, 256, 0, s>>>(z.get(), 1, static_cast<int>(k), kmax, 1, z_pad.get());
        ISDF_LAUNCH_CHECK();
        AdjGridArgs a{c.d_shells, c.nshell, static_cast<int>(nao), c.natm, c.d_exp, c.d_coef, pts, w,
                      kp.index.get(), n, pk.get(), z_pad.get(), gacc.get(), v.get(), energy.get()};
        if (c.lmax <= 2) {
            if (kmax == 4) launch_adjoint_grid<2, 4>(a, want_grad, s);
            else if (kmax == 8) launch_adjoint_grid<2, 8>(a, want_grad, s);
            else if (kmax == 12) launch_adjoint_grid<2, 12>(a, want_grad, s);
            else if (kmax == 16) launch_adjoint_grid<2, 16>(a, want_grad, s);
            else launch_adjoint_grid<2, 32>(a, want_grad, s);
        } else {
            if (kmax == 4) launch_adjoint_grid<kMaxL, 4>(a, want_grad, s);
            else if (kmax == 8) launch_adjoint_grid<kMaxL, 8>(a, want_grad, s);
            else if (kmax == 12) launch_adjoint_grid<kMaxL, 12>(a, want_grad, s);
            else if (kmax == 16) launch_adjoint_grid<kMaxL, 16>(a, want_grad, s);
            else launch_adjoint_grid<kMaxL, 32>(a, want_grad, s);
        }
    }
    // otherwise the grid pass in chunks: AO values + gradients recomputed per chunk
    const int64_t chunk = fused ? 1 : std::max<int64_t>(256, std::min<int64_t>(n, (int64_t(1) << 25) / nao));
    DeviceBuffer<double> cp(static_cast<size_t>(3 * chunk), s), cw(chunk, s),
        phi(static_cast<size_t>(chunk * nao), s), dphi(static_cast<size_t>(3 * chunk * nao), s),
        G(static_cast<size_t>(chunk * k), s), alpha(static_cast<size_t>(chunk * k), s),
        alphaT(static_cast<size_t>(chunk * k), s), beta(static_cast<size_t>(chunk * nao), s);
    for (int64_t g0 = 0; !fused && g0 < n; g0 += chunk) {
        const int64_t b = std::min(chunk, n - g0);
        ISDF_PROFILE("adjoint_grid", s);
        gather_kernel<<<nblk(b), 256, 0, s>>>(pts, w, kp.index.get() + g0, b, cp.get(), cw.get());
        ISDF_LAUNCH_CHECK();
        eval_ao<double>(c, cp.get(), b, phi.get(), want_grad ? dphi.get() : nullptr, nao, s);
        gemm_f64(b, k, nao, phi.get(), nao, 0, f.phi_aT.get(), k, 0, G.get(), k, 0, 1, false, s);
        adjoint_point_kernel<<<nblk(b), 256, 0, s>>>(G.get(), cw.get(), b, static_cast<int>(k), z.get(),
                                                     alpha.get(), alphaT.get(), v.get(), energy.get());
        ISDF_LAUNCH_CHECK();
        if (!want_grad) continue;
        // B += alpha^T Phi_chunk ; beta = alpha Phi_a
        gemm_f64(k, nao, b, alphaT.get(), b, 0, phi.get(), nao, 0, B.get(), nao, 0, 1, true, s);
        gemm_f64(b, nao, k, alpha.get(), k, 0, f.phi_a.get(), nao, 0, beta.get(), nao, 0, 1, false, s);
        dim3 cg(static_cast<unsigned>((nao + 255) / 256), 3);
        column_dot_kernel<<<cg, 256, 0, s>>>(beta.get(), dphi.get(), b, static_cast<int>(nao), acc.get());
        ISDF_LAUNCH_CHECK();
    }
    // [E, v (k), per-atom grid terms (natm x 3), B (k x nao), acc (3 x nao)]
    double* o = out.data();
    ISDF_CUDA(cudaMemcpyAsync(o, energy.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(o + 1, v.get(), k * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(o + 1 + k, gacc.get(), 3 * c.natm * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(o + 1 + k + 3 * c.natm, B.get(), k * nao * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaMemcpyAsync(o + 1 + k + 3 * c.natm + k * nao, acc.get(), 3 * nao * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    return out;
}

AdjointResult energy_gradient_finish(const Context& c, const AnchorFactor& f, const double* dm,
                                     const double* sums, bool want_grad, cudaStream_t s) {
    AdjointResult r;
    const int64_t k = f.k, nao = c.nao;
    r.grad.assign(static_cast<size_t>(c.natm) * 3, 0.0);
    r.energy = sums[0];
    if (k == 0 || !want_grad) return r;
    AnchorSide as = anchor_side(c, f, dm, true, s);
    DeviceBuffer<double> v(k, s), y(k, s), W(static_cast<size_t>(k * k), s), B(static_cast<size_t>(k * nao), s),
        WPhi(static_cast<size_t>(k * nao), s), coef(static_cast<size_t>(k * nao), s),
        acc(static_cast<size_t>(3 * nao), s);
    const double* hB = sums + 1 + k + 3 * c.natm;
    ISDF_CUDA(cudaMemcpyAsync(v.get(), sums + 1, k * sizeof(double), cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaMemcpyAsync(B.get(), hB, k * nao * sizeof(double), cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaMemcpyAsync(acc.get(), hB + k * nao, 3 * nao * sizeof(double), cudaMemcpyHostToDevice, s));
    // anchor terms
    anchor_terms_kernel<<<1, 256, 0, s>>>(static_cast<int>(k), static_cast<int>(nao), f.phi_a.get(), as.S.get(),
                                          f.T.get(), as.PhiD.get(), as.z.get(), v.get(), y.get(), W.get());
    ISDF_LAUNCH_CHECK();
    gemm_f64(k, nao, k, W.get(), k, 0, f.phi_a.get(), nao, 0, WPhi.get(), nao, 0, 1, false, s);
    anchor_coef_kernel<<<nblk(k * nao), 256, 0, s>>>(static_cast<int>(k), static_cast<int>(nao), B.get(),
                                                     as.PhiD.get(), WPhi.get(), y.get(), coef.get());
    ISDF_LAUNCH_CHECK();
    dim3 cg(static_cast<unsigned>((nao + 255) / 256), 3);
    anchor_contrib_kernel<<<cg, 256, 0, s>>>(static_cast<int>(k), static_cast<int>(nao), coef.get(),
                                             as.dphia.get(), acc.get());
    ISDF_LAUNCH_CHECK();
    std::vector<double> hacc(3 * nao);
    ISDF_CUDA(cudaMemcpyAsync(hacc.data(), acc.get(), hacc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    ISDF_CUDA(cudaStreamSynchronize(s));
    // d phi / d R_A = -grad_r phi for AOs on atom A
    for (int64_t mu = 0; mu < nao; ++mu) {
        const int a = c.ao_atom[mu];
        for (int cc = 0; cc < 3; ++cc) r.grad[a * 3 + cc] -= hacc[cc * nao + mu];
    }
    const double* hg = sums + 1 + k;
    for (int i = 0; i < 3 * c.natm; ++i) r.grad[i] -= hg[i];   // fused grid pass (per atom)
    return r;
}

AdjointResult energy_gradient(const Context& c, const double* pts, const double* w, const KeptPoints& kp,
                              const AnchorFactor& f, const double* dm, bool want_grad, cudaStream_t s) {
    const std::vector<double> part = energy_gradient_partial(c, pts, w, kp, f, dm, want_grad, s);
    return energy_gradient_finish(c, f, dm, part.data(), want_grad, s);
}

}  // namespace isdf
