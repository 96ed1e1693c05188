// extern "C" boundary of libisdf_b200.so (declared in include/isdf_b200.h).
#include "../../include/isdf_b200.h"
#include "isdf_adjoint.h"
#include "isdf_fit.h"
#include "isdf_metric.h"
#include "isdf_project.h"
#include "isdf_rbrp.h"
#include "isdf_select.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

struct isdf_ctx {
    std::unique_ptr<isdf::Context> c;
    cudaStream_t stream = nullptr;   // private stream of the host-buffer entry points
};

namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return ISDF_OK;
    } catch (const isdf::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return ISDF_ERR_RUNTIME;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return ISDF_ERR_RUNTIME;
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        ISDF_CUDA(cudaGetDevice(&prev));
        if (prev != dev) ISDF_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

isdf::Context& ctx_of(isdf_ctx* ctx) {
    if (!ctx || !ctx->c) isdf::fail(isdf::kInvalid, "null isdf context");
    return *ctx->c;
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

template <class T>
void upload(isdf::DeviceBuffer<T>& d, const T* h, size_t n, cudaStream_t s) {
    d.reset(n, s);
    if (n) ISDF_CUDA(cudaMemcpyAsync(d.get(), h, n * sizeof(T), cudaMemcpyHostToDevice, s));
}

isdf::SelectOptions options_of(const isdf_select_args* a) {
    if (!a) isdf::fail(isdf::kInvalid, "null selection arguments");
    isdf::SelectOptions o;
    o.algorithm = a->algorithm;
    if (a->naxes <= 0 || !a->axes) isdf::fail(isdf::kInvalid, "axis list must not be empty");
    o.axes.assign(a->axes, a->axes + a->naxes);
    if (a->axis_weights) o.axis_weights.assign(a->axis_weights, a->axis_weights + a->naxes);
    o.tolerance = a->tolerance;
    o.max_rank = a->max_rank;
    o.batch_size = a->batch_size;
    o.sketch_size = a->sketch_size;
    o.oversampling = a->oversampling;
    o.seed = a->seed;
    o.precision = a->precision;
    o.debug = a->debug != 0;
    o.importance = a->point_importance;
    o.ao_threshold = a->ao_screening_threshold;
    o.mo_host = a->mo_coeff;
    o.nocc = a->nocc;
    if (o.max_rank < 0 || o.batch_size < 0 || o.sketch_size < 0 || o.oversampling < 0)
        isdf::fail(isdf::kInvalid, "sizes must be nonnegative");
    return o;
}

// The host-buffer entry points take the importance vector in host memory: a
// copy of the arguments pointing at a device copy of it.
isdf_select_args device_importance(const isdf_select_args* a, isdf::DeviceBuffer<double>& dm, int64_t ng,
                                   cudaStream_t s) {
    if (!a) isdf::fail(isdf::kInvalid, "null selection arguments");
    isdf_select_args out = *a;
    if (a->point_importance && ng > 0) {
        upload(dm, a->point_importance, static_cast<size_t>(ng), s);
        out.point_importance = dm.get();
    }
    return out;
}

}  // namespace

namespace isdf {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace isdf

extern "C" {

const char* isdf_status_string(int status) {
    switch (status) {
    case ISDF_OK: return "ok";
    case ISDF_ERR_INVALID: return "invalid argument";
    case ISDF_ERR_OVERFLOW: return "overflow";
    case ISDF_ERR_RUNTIME: return "runtime error";
    case ISDF_ERR_CUDA: return "CUDA error";
    case ISDF_ERR_NOT_IMPLEMENTED: return "not implemented";
    case ISDF_ERR_LOGIC: return "logic error";
    default: return "unknown status";
    }
}

const char* isdf_last_error(void) { return g_last_error.c_str(); }

int isdf_cuda_available(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0 ? 1 : 0;
}

int isdf_ctx_create(const int32_t* atm, int32_t natm, const int32_t* bas, int32_t nbas,
                    const double* env, int64_t nenv, isdf_ctx** out) {
    return guarded([&] {
        if (!out) isdf::fail(isdf::kInvalid, "null output pointer");
        *out = nullptr;
        if ((natm && !atm) || (nbas && !bas) || !env)
            isdf::fail(isdf::kInvalid, "expected atm[natm,6], bas[nbas,8], env[nenv]");
        auto h = std::make_unique<isdf_ctx>();
        h->c.reset(isdf::create_context(atm, natm, bas, nbas, env, nenv));
        ISDF_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        *out = h.release();
    });
}

int isdf_ctx_destroy(isdf_ctx* ctx) {
    return guarded([&] {
        if (!ctx) return;
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
    });
}

int isdf_ctx_info(const isdf_ctx* ctx, int64_t* nao, int32_t* natm, int32_t* nshell) {
    return guarded([&] {
        auto& c = ctx_of(const_cast<isdf_ctx*>(ctx));
        if (nao) *nao = c.nao;
        if (natm) *natm = c.natm;
        if (nshell) *nshell = c.nshell;
    });
}

int isdf_ctx_ao_atoms(const isdf_ctx* ctx, int32_t* out) {
    return guarded([&] {
        auto& c = ctx_of(const_cast<isdf_ctx*>(ctx));
        std::memcpy(out, c.ao_atom.data(), c.ao_atom.size() * sizeof(int32_t));
    });
}

int isdf_eval_ao(isdf_ctx* ctx, const double* xyz, int64_t ng, int32_t dtype, void* values,
                 void* grad, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        if (ng < 0) isdf::fail(isdf::kInvalid, "expected coords[ngrid,3] in Bohr");
        if (dtype == 0)
            isdf::eval_ao<double>(c, xyz, ng, static_cast<double*>(values), static_cast<double*>(grad),
                                  c.nao, as_stream(stream));
        else if (dtype == 1)
            isdf::eval_ao<float>(c, xyz, ng, static_cast<float*>(values), static_cast<float*>(grad),
                                 c.nao, as_stream(stream));
        else
            isdf::fail(isdf::kInvalid, "dtype must be 0 (float64) or 1 (float32)");
    });
}

int isdf_eval_ao_host(isdf_ctx* ctx, const double* xyz, int64_t ng, double* values, double* grad) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = ctx->stream;
        if (ng < 0) isdf::fail(isdf::kInvalid, "expected coords[ngrid,3] in Bohr");
        if (ng == 0 || c.nao == 0) return;
        isdf::DeviceBuffer<double> dx, dv, dg2;
        upload(dx, xyz, static_cast<size_t>(3 * ng), s);
        const size_t nv = static_cast<size_t>(ng) * c.nao;
        if (values) dv.reset(nv, s);
        if (grad) dg2.reset(3 * nv, s);
        isdf::eval_ao<double>(c, dx.get(), ng, values ? dv.get() : nullptr, grad ? dg2.get() : nullptr,
                              c.nao, s);
        if (values) ISDF_CUDA(cudaMemcpyAsync(values, dv.get(), nv * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (grad) ISDF_CUDA(cudaMemcpyAsync(grad, dg2.get(), 3 * nv * sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
    });
}

int isdf_evaluate_axis_mo(isdf_ctx* ctx, const double* xyz, int64_t ng, const int32_t* axes, int32_t naxes,
                          const double* mo_host, int64_t nocc, double* out, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = as_stream(stream);
        if (!axes) isdf::fail(isdf::kInvalid, "axis list must not be empty");
        isdf::DeviceBuffer<double> dmo;
        if (mo_host) upload(dmo, mo_host, static_cast<size_t>(c.nao) * c.nao, s);
        isdf::AxisSpec ax = isdf::make_axis_spec(c, axes, naxes, dmo.get(), nocc);
        isdf::eval_axis_features<double>(c, xyz, nullptr, ng, ax, out, ax.d, nullptr, nullptr, s);
        ISDF_CUDA(cudaStreamSynchronize(s));   // the MO copy outlives its use
    });
}

int isdf_evaluate_axis_mo_host(isdf_ctx* ctx, const double* xyz, int64_t ng, const int32_t* axes,
                               int32_t naxes, const double* mo_host, int64_t nocc, double* out) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = ctx->stream;
        if (!axes) isdf::fail(isdf::kInvalid, "axis list must not be empty");
        isdf::DeviceBuffer<double> dmo;
        if (mo_host) upload(dmo, mo_host, static_cast<size_t>(c.nao) * c.nao, s);
        isdf::AxisSpec ax = isdf::make_axis_spec(c, axes, naxes, dmo.get(), nocc);
        if (ng <= 0) return;
        const int64_t d = ax.d;
        isdf::DeviceBuffer<double> dx, dout(static_cast<size_t>(ng * d), s);
        upload(dx, xyz, static_cast<size_t>(3 * ng), s);
        isdf::eval_axis_features<double>(c, dx.get(), nullptr, ng, ax, dout.get(), d, nullptr, nullptr, s);
        ISDF_CUDA(cudaMemcpyAsync(out, dout.get(), ng * d * sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
    });
}

int isdf_evaluate_axis(isdf_ctx* ctx, const double* xyz, int64_t ng, const int32_t* axes,
                       int32_t naxes, double* out, void* stream) {
    return isdf_evaluate_axis_mo(ctx, xyz, ng, axes, naxes, nullptr, 0, out, stream);
}

int isdf_evaluate_axis_host(isdf_ctx* ctx, const double* xyz, int64_t ng, const int32_t* axes,
                            int32_t naxes, double* out) {
    return isdf_evaluate_axis_mo_host(ctx, xyz, ng, axes, naxes, nullptr, 0, out);
}

void isdf_select_args_default(isdf_select_args* a) {
    if (!a) return;
    std::memset(a, 0, sizeof(*a));
    a->algorithm = ISDF_QRCP_DENSE;
    a->tolerance = 1e-10;
    a->max_rank = 0;
    a->batch_size = 128;
    a->sketch_size = 128;
    a->oversampling = 16;
    a->seed = 7;
    a->precision = ISDF_FP64;
    a->point_importance = nullptr;
    a->ao_screening_threshold = 1e-24;
}

namespace {

std::vector<int64_t> select_impl(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz,
                                 const double* w, int64_t ng, isdf_select_info* info, cudaStream_t s,
                                 isdf::RetainedAo* keep) {
    auto& c = ctx_of(ctx);
    DeviceGuard dg(c.device);
    isdf::SelectOptions o = options_of(args);
    if (ng < 0) isdf::fail(isdf::kInvalid, "expected points[ngrid,3]");
    const bool density = o.algorithm == ISDF_RAND_SKETCH_DENSITY || o.algorithm == ISDF_RAND_SKETCH_DENSITY_NORM;
    if (density && (o.axes.size() != 1 || o.axes[0] != ISDF_AXIS_AO))
        isdf::fail(isdf::kInvalid, "density Khatri-Rao sketches with non-AO axis features are NYI");
    isdf::validate_axis_weights(o.axis_weights.empty() ? nullptr : o.axis_weights.data(),
                                static_cast<int>(o.axes.size()));
    std::vector<int64_t> out;
    if (info) std::memset(info, 0, sizeof(*info));
    switch (o.algorithm) {
    case ISDF_QRCP_DENSE:
    case ISDF_QRCP_ONLINE: {
        isdf::PairQrDiagnostics d;
        out = isdf::select_pair_qr(c, xyz, w, ng, o, s, &d);
        if (info) {
            info->verifications = d.verifications;
            info->reselections = d.reselections;
            info->relative_residual = (d.first > 0 && !d.rdiag.empty()) ? d.rdiag.back() / d.first : 0.0;
        }
        if (o.debug)
            std::fprintf(stderr,
                         "[%s qrcp] rank=%lld max_initial_norm=%.6e relative_residual=%.6e "
                         "candidate_checks=%lld candidate_reselections=%lld exact_scans=%lld\n",
                         o.algorithm == ISDF_QRCP_ONLINE ? "online" : "dense",
                         static_cast<long long>(out.size()), d.first,
                         info ? info->relative_residual : 0.0,
                         static_cast<long long>(d.verifications),
                         static_cast<long long>(d.reselections), static_cast<long long>(d.exact_scans));
        break;
    }
    case ISDF_RAND_SKETCH_QUADRATURE:
    case ISDF_RAND_SKETCH_DENSITY:
    case ISDF_RAND_SKETCH_DENSITY_NORM: {
        isdf::SketchDiagnostics d;
        out = isdf::select_rand_sketch(c, xyz, w, ng, o, s, &d, keep);
        if (info) {
            info->sketch_rows = d.ell;
            info->numerical_rank = d.numerical_rank;
            info->relative_residual = d.relative_tail;
            info->verifications = d.reverified;
            info->precision_used = d.precision_used;
        }
        if (o.debug)
            std::fprintf(stderr,
                         "[rand_sketch:%s] rank=%lld sketch_size=%lld oversampling=%lld "
                         "sketch_relative_frobenius=%.6e numerical_rank=%lld rank_cap=%lld "
                         "seed=%llu precision=%s space=device\n",
                         o.algorithm == ISDF_RAND_SKETCH_DENSITY_NORM ? "density_col_norm"
                         : o.algorithm == ISDF_RAND_SKETCH_DENSITY   ? "density"
                                                                     : "quadrature",
                         static_cast<long long>(d.rank), static_cast<long long>(d.ell),
                         static_cast<long long>(o.oversampling), d.relative_tail,
                         static_cast<long long>(d.numerical_rank), static_cast<long long>(d.cap),
                         static_cast<unsigned long long>(o.seed), o.precision ? "mixed" : "fp64");
        break;
    }
    case ISDF_CVT:
        isdf::fail(isdf::kNotImplemented,
                   "this anchor selection algorithm is outside the B200 hot path (NYI)");
    default:
        isdf::fail(isdf::kInvalid, "unknown anchor selection algorithm");
    }
    return out;
}

}  // namespace

int isdf_select(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz, const double* w,
                int64_t ng, int64_t* pivots, int64_t capacity, int64_t* npivots,
                isdf_select_info* info, void* stream) {
    return guarded([&] {
        if (npivots) *npivots = 0;
        std::vector<int64_t> out = select_impl(ctx, args, xyz, w, ng, info, as_stream(stream), nullptr);
        if (static_cast<int64_t>(out.size()) > capacity)
            isdf::fail(isdf::kInvalid, "pivot buffer is too small");
        if (!out.empty()) std::memcpy(pivots, out.data(), out.size() * sizeof(int64_t));
        if (npivots) *npivots = static_cast<int64_t>(out.size());
    });
}

int isdf_select_host(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz,
                     const double* w, int64_t ng, int64_t* pivots, int64_t capacity,
                     int64_t* npivots, isdf_select_info* info) {
    int rc = guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = ctx->stream;
        isdf::DeviceBuffer<double> dx, dw, dm;
        upload(dx, xyz, static_cast<size_t>(3 * std::max<int64_t>(ng, 0)), s);
        upload(dw, w, static_cast<size_t>(std::max<int64_t>(ng, 0)), s);
        isdf_select_args a = device_importance(args, dm, ng, s);
        const int r = isdf_select(ctx, &a, dx.get(), dw.get(), ng, pivots, capacity, npivots, info, s);
        if (r != ISDF_OK) throw isdf::Error(r, g_last_error);
    });
    return rc;
}

namespace {

// Anchors given by host coordinates and weights instead of grid indices.
struct AnchorCoords {
    const double* xyz = nullptr;   // k x 3
    const double* w = nullptr;     // k
};

// Fit form of the fused selection + fit.  A mixed request whose selection left
// no AO tiles (the FP64 selections, or no plain value axis) would have to run
// its own fused AO pass plus the bound's host round trips; below 2^28 AO values
// that costs more than the FP64 fit (about 0.5 ms at C1 and C4), so those fits
// run in FP64 (fit_path 0).
int32_t fused_fit_precision(isdf_ctx* ctx, int32_t precision, const isdf::RetainedAo& keep, int64_t ng) {
    if (precision != ISDF_MIXED || keep.valid) return precision;
    const double values = static_cast<double>(ng) * ctx_of(ctx).nao;
    return values < 268435456.0 ? ISDF_FP64 : precision;
}

void fit_impl(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng, const int64_t* anchors,
              int64_t k, int32_t precision, const double* theta_in, double* theta_out,
              isdf_fit_info* info, double* l2, double* rel, cudaStream_t s, bool want_error = true,
              const isdf::RetainedAo* ra = nullptr, const AnchorCoords* ac = nullptr,
              double* sums = nullptr, const isdf::FitChunkHook* on_chunk = nullptr) {
    auto& c = ctx_of(ctx);
    DeviceGuard dg(c.device);
    if (ng < 0 || k < 0) isdf::fail(isdf::kInvalid, "sizes must be nonnegative");
    if (precision != ISDF_FP64 && precision != ISDF_MIXED)
        isdf::fail(isdf::kInvalid, "precision must be fp64 or mixed");
    ISDF_PROFILE("phase:fit", s);
    // the kept points (and AO tiles) of a preceding mixed selection on these points
    const bool reuse = ra && ra->valid;
    isdf::KeptPoints kp_own;
    if (!reuse) {
        ISDF_PROFILE("phase:compact", s);
        kp_own = isdf::compact_points(xyz, w, ng, s);
    }
    const isdf::KeptPoints& kp = reuse ? ra->kp : kp_own;
    isdf::DeviceBuffer<double> apts(static_cast<size_t>(3 * std::max<int64_t>(k, 1)), s),
        aw(std::max<int64_t>(k, 1), s);
    if (ac) {
        if (k && (!ac->xyz || !ac->w)) isdf::fail(isdf::kInvalid, "anchor coordinates and weights are required");
        for (int64_t i = 0; i < 3 * k; ++i)
            if (!std::isfinite(ac->xyz[i])) isdf::fail(isdf::kInvalid, "anchor coordinates must be finite");
        if (k) {
            ISDF_CUDA(cudaMemcpyAsync(apts.get(), ac->xyz, 3 * k * sizeof(double), cudaMemcpyHostToDevice, s));
            ISDF_CUDA(cudaMemcpyAsync(aw.get(), ac->w, k * sizeof(double), cudaMemcpyHostToDevice, s));
        }
    } else {
        isdf::DeviceBuffer<int64_t> didx;
        upload(didx, anchors, static_cast<size_t>(k), s);
        isdf::gather_points(xyz, w, didx.get(), k, ng, apts.get(), aw.get(), s);
    }
    isdf::AnchorFactor f;
    {
        ISDF_PROFILE("phase:factor_anchors", s);
        f = isdf::factor_anchors(c, apts.get(), aw.get(), k, s);
    }
    const bool have = theta_in != nullptr;
    double* theta = have ? const_cast<double*>(theta_in) : theta_out;
    isdf::FitOutput o;
    if (!have && precision == ISDF_MIXED && isdf::fit_mixed_supported(k)) {
        o = isdf::fit_grid_mixed(c, xyz, w, kp, f, theta, kp.n, s, reuse ? ra->tiles : nullptr,
                                 reuse ? ra->tiles_r : nullptr,
                                 reuse ? ra->psq.get() : nullptr, on_chunk, reuse ? ra->chunk_zero : nullptr);
        if (!(o.mixed_bound <= isdf::kMixedFitTolerance)) {
            // a fit whose pair error is very small cannot absorb the stored
            // tiles' representation error: recompute Theta with FP64 AO values
            const double bound = o.mixed_bound;
            o = isdf::fit_grid(c, xyz, w, kp, f, theta, kp.n, false, s);
            o.mixed_bound = bound;
            o.path = 2;
        } else if (want_error) {
            // pair-space error of the mixed Theta, evaluated with FP64 AO values
            isdf::FitOutput e = isdf::fit_grid(c, xyz, w, kp, f, theta, kp.n, true, s);
            o.err2 = e.err2;
            o.exact2 = e.exact2;
        }
    } else {
        o = isdf::fit_grid(c, xyz, w, kp, f, theta, kp.n, have, s);
    }
    if (!have && theta && k > 0 && kp.n > 0 && kp.spatial()) {
        // the selection's spatial point order: Theta's columns back to the
        // ascending kept order of the interface
        isdf::DeviceBuffer<double> tmp(static_cast<size_t>(k * kp.n), s);
        isdf::unpermute_columns(theta, tmp.get(), kp.n, k, kp.rank.get(), 0, kp.n, s);
        ISDF_CUDA(cudaMemcpyAsync(theta, tmp.get(), static_cast<size_t>(k * kp.n) * sizeof(double),
                                  cudaMemcpyDeviceToDevice, s));
    }
    const double el2 = std::sqrt(o.err2);
    const double erel = o.exact2 ? el2 / std::sqrt(o.exact2) : (el2 == 0 ? 0.0 : INFINITY);
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->n_kept = kp.n;
        info->retained_rank = f.retained;
        info->condition = f.condition;
        info->max_abs_physical_coefficient = o.max_abs_coeff;
        info->pair_l2 = el2;
        info->pair_relative = erel;
        info->fit_path = o.path;
        info->mixed_bound = o.mixed_bound;
        for (int64_t a = 0; a < k && a < 64; ++a) info->theta_w[a] = o.theta_w[a];
    }
    if (l2) *l2 = el2;
    if (rel) *rel = erel;
    if (sums) {
        sums[0] = o.err2;
        sums[1] = o.exact2;
    }
}

}  // namespace

int isdf_fit(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng, const int64_t* anchors,
             int64_t k, int32_t precision, int32_t want_error, double* theta, isdf_fit_info* info,
             void* stream) {
    return guarded([&] {
        fit_impl(ctx, xyz, w, ng, anchors, k, precision, nullptr, theta, info, nullptr, nullptr,
                 as_stream(stream), want_error != 0);
    });
}

int isdf_fit_host(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng,
                  const int64_t* anchors, int64_t k, int32_t precision, int32_t want_error,
                  double* theta_host, isdf_fit_info* info) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = ctx->stream;
        isdf::DeviceBuffer<double> dx, dw, dt(static_cast<size_t>(std::max<int64_t>(1, k * ng)), s);
        upload(dx, xyz, static_cast<size_t>(3 * std::max<int64_t>(ng, 0)), s);
        upload(dw, w, static_cast<size_t>(std::max<int64_t>(ng, 0)), s);
        isdf_fit_info local{};
        fit_impl(ctx, dx.get(), dw.get(), ng, anchors, k, precision, nullptr, dt.get(), &local,
                 nullptr, nullptr, s, want_error != 0);
        if (theta_host && k * local.n_kept)
            ISDF_CUDA(cudaMemcpyAsync(theta_host, dt.get(), k * local.n_kept * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        if (info) *info = local;
    });
}

int isdf_select_fit(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz, const double* w,
                    int64_t ng, int64_t* pivots, int64_t capacity, int64_t* npivots,
                    isdf_select_info* select_info, int32_t want_error, double* theta,
                    isdf_fit_info* fit_info, void* stream) {
    return guarded([&] {
        if (npivots) *npivots = 0;
        if (!args) isdf::fail(isdf::kInvalid, "selection arguments are required");
        cudaStream_t s = as_stream(stream);
        std::lock_guard<std::mutex> lock(ctx_of(ctx).ws_mu);   // workspace held to the end of the fit
        isdf::RetainedAo keep;
        std::vector<int64_t> out = select_impl(ctx, args, xyz, w, ng, select_info, s, &keep);
        if (static_cast<int64_t>(out.size()) > capacity)
            isdf::fail(isdf::kInvalid, "pivot buffer is too small");
        if (!out.empty()) std::memcpy(pivots, out.data(), out.size() * sizeof(int64_t));
        if (npivots) *npivots = static_cast<int64_t>(out.size());
        fit_impl(ctx, xyz, w, ng, out.data(), static_cast<int64_t>(out.size()),
                 fused_fit_precision(ctx, args->precision, keep, ng), nullptr, theta, fit_info, nullptr, nullptr,
                 s, want_error != 0, &keep);
    });
}

namespace {

// A copy stream and its events for streaming results out while the compute
// stream runs; finish() (or the destructor, on an error path) waits for the
// copies and releases them.
struct ChunkCopies {
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> events;
    void begin() {
        if (!stream) ISDF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    }
    cudaEvent_t event() {
        cudaEvent_t e = nullptr;
        ISDF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        events.push_back(e);
        return e;
    }
    bool used() const { return stream != nullptr; }
    void finish() {
        if (stream) {
            const cudaError_t r = cudaStreamSynchronize(stream);
            release();
            ISDF_CUDA(r);
        }
    }
    void release() {
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        events.clear();
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        stream = nullptr;
    }
    ~ChunkCopies() { release(); }
};

}  // namespace

int isdf_select_fit_host(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz,
                         const double* w, int64_t ng, int64_t* pivots, int64_t capacity,
                         int64_t* npivots, isdf_select_info* select_info, int32_t want_error,
                         double* theta_host, isdf_fit_info* fit_info) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = ctx->stream;
        if (npivots) *npivots = 0;
        if (!args) isdf::fail(isdf::kInvalid, "selection arguments are required");
        isdf::DeviceBuffer<double> dx, dw, dm;
        upload(dx, xyz, static_cast<size_t>(3 * std::max<int64_t>(ng, 0)), s);
        upload(dw, w, static_cast<size_t>(std::max<int64_t>(ng, 0)), s);
        isdf_select_args a = device_importance(args, dm, ng, s);
        std::lock_guard<std::mutex> lock(c.ws_mu);   // workspace held to the end of the fit
        isdf::RetainedAo keep;
        std::vector<int64_t> out = select_impl(ctx, &a, dx.get(), dw.get(), ng, select_info, s, &keep);
        if (static_cast<int64_t>(out.size()) > capacity)
            isdf::fail(isdf::kInvalid, "pivot buffer is too small");
        if (!out.empty()) std::memcpy(pivots, out.data(), out.size() * sizeof(int64_t));
        const int64_t np = static_cast<int64_t>(out.size());
        isdf::DeviceBuffer<double> dt(static_cast<size_t>(std::max<int64_t>(1, np * ng)), s);
        isdf_fit_info local{};
        // In the mixed fit over the stored AO tiles, each chunk's Theta columns
        // are copied out on a second stream while the next chunk is fitted; if
        // the mixed Theta is then rejected (FP64 recompute), it is copied again.
        ChunkCopies cp;
        // a spatial kept order (whole windows per chunk): each chunk's columns
        // go back to ascending order in a staging copy before they leave
        isdf::DeviceBuffer<double> dt_asc;
        if (keep.valid && keep.kp.spatial() && np > 0)
            dt_asc.reset(static_cast<size_t>(np * keep.kp.n), s);
        isdf::FitChunkHook hook = [&](int64_t g0, int64_t m) {
            const int64_t n = keep.kp.n;
            const double* src = dt.get();
            if (dt_asc.get()) {
                isdf::unpermute_columns(dt.get(), dt_asc.get(), n, np, keep.kp.rank.get(), g0, m, s);
                src = dt_asc.get();
            }
            cp.begin();
            cudaEvent_t ev = cp.event();
            ISDF_CUDA(cudaEventRecord(ev, s));
            ISDF_CUDA(cudaStreamWaitEvent(cp.stream, ev, 0));
            ISDF_CUDA(cudaMemcpy2DAsync(theta_host + g0, n * sizeof(double), src + g0, n * sizeof(double),
                                        m * sizeof(double), np, cudaMemcpyDeviceToHost, cp.stream));
        };
        const bool stream_out = theta_host && np > 0 && keep.valid;
        fit_impl(ctx, dx.get(), dw.get(), ng, out.data(), np, fused_fit_precision(ctx, args->precision, keep, ng),
                 nullptr, dt.get(), &local,
                 nullptr, nullptr, s, want_error != 0, &keep, nullptr, nullptr, stream_out ? &hook : nullptr);
        const bool copied = cp.used() && local.fit_path == 1;
        cp.finish();
        if (theta_host && np * local.n_kept && !copied)
            ISDF_CUDA(cudaMemcpyAsync(theta_host, dt.get(), np * local.n_kept * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
        if (npivots) *npivots = np;
        if (fit_info) *fit_info = local;
    });
}

int isdf_pair_error(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng,
                    const int64_t* anchors, int64_t k, const double* theta, double* l2,
                    double* relative, void* stream) {
    return guarded([&] {
        if (!theta) isdf::fail(isdf::kInvalid, "theta is required");
        fit_impl(ctx, xyz, w, ng, anchors, k, ISDF_FP64, theta, nullptr, nullptr, l2, relative,
                 as_stream(stream));
    });
}

int isdf_energy_gradient(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng,
                         const int64_t* anchors, int64_t k, const double* dm, double* energy,
                         double* grad, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = as_stream(stream);
        if (ng < 0 || k <= 0 || !anchors || !dm) isdf::fail(isdf::kInvalid, "invalid adjoint arguments");
        isdf::KeptPoints kp = isdf::compact_points(xyz, w, ng, s);
        isdf::DeviceBuffer<int64_t> didx;
        upload(didx, anchors, static_cast<size_t>(k), s);
        isdf::DeviceBuffer<double> apts(static_cast<size_t>(3 * k), s), aw(k, s);
        isdf::gather_points(xyz, w, didx.get(), k, ng, apts.get(), aw.get(), s);
        isdf::AnchorFactor f;
    {
        ISDF_PROFILE("phase:factor_anchors", s);
        f = isdf::factor_anchors(c, apts.get(), aw.get(), k, s);
    }
        isdf::AdjointResult r = isdf::energy_gradient(c, xyz, w, kp, f, dm, grad != nullptr, s);
        if (energy) *energy = r.energy;
        if (grad) std::memcpy(grad, r.grad.data(), r.grad.size() * sizeof(double));
    });
}

namespace {
// Anchors given by coordinates and weights (host), factored on the device.
isdf::AnchorFactor factor_anchor_coords(isdf::Context& c, const double* axyz, const double* aw, int64_t k,
                                        cudaStream_t s) {
    if (k <= 0 || !axyz || !aw) isdf::fail(isdf::kInvalid, "anchor coordinates and weights are required");
    for (int64_t i = 0; i < 3 * k; ++i)
        if (!std::isfinite(axyz[i])) isdf::fail(isdf::kInvalid, "anchor coordinates must be finite");
    isdf::DeviceBuffer<double> apts(static_cast<size_t>(3 * k), s), dw(k, s);
    ISDF_CUDA(cudaMemcpyAsync(apts.get(), axyz, 3 * k * sizeof(double), cudaMemcpyHostToDevice, s));
    ISDF_CUDA(cudaMemcpyAsync(dw.get(), aw, k * sizeof(double), cudaMemcpyHostToDevice, s));
    ISDF_PROFILE("phase:factor_anchors", s);
    isdf::AnchorFactor f = isdf::factor_anchors(c, apts.get(), dw.get(), k, s);
    ISDF_CUDA(cudaStreamSynchronize(s));   // the host arrays may go out of scope
    return f;
}
}  // namespace

int isdf_adjoint_partial_size(isdf_ctx* ctx, int64_t k, int64_t* size) {
    return guarded([&] {
        if (k < 0 || !size) isdf::fail(isdf::kInvalid, "invalid adjoint partial size arguments");
        *size = static_cast<int64_t>(isdf::adjoint_partial_size(ctx_of(ctx), k));
    });
}

int isdf_energy_gradient_shard(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng,
                               const double* anchor_xyz, const double* anchor_w, int64_t k, const double* dm,
                               int32_t want_grad, double* partial, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = as_stream(stream);
        if (ng < 0 || k <= 0 || !dm || !partial) isdf::fail(isdf::kInvalid, "invalid adjoint arguments");
        isdf::AnchorFactor f = factor_anchor_coords(c, anchor_xyz, anchor_w, k, s);
        isdf::KeptPoints kp = isdf::compact_points(xyz, w, ng, s);
        const std::vector<double> part = isdf::energy_gradient_partial(c, xyz, w, kp, f, dm, want_grad != 0, s);
        std::memcpy(partial, part.data(), part.size() * sizeof(double));
    });
}

int isdf_energy_gradient_finish(isdf_ctx* ctx, const double* anchor_xyz, const double* anchor_w, int64_t k,
                                const double* dm, const double* sums, double* energy, double* grad, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = as_stream(stream);
        if (k <= 0 || !dm || !sums) isdf::fail(isdf::kInvalid, "invalid adjoint arguments");
        isdf::AnchorFactor f = factor_anchor_coords(c, anchor_xyz, anchor_w, k, s);
        isdf::AdjointResult r = isdf::energy_gradient_finish(c, f, dm, sums, grad != nullptr, s);
        if (energy) *energy = r.energy;
        if (grad) std::memcpy(grad, r.grad.data(), r.grad.size() * sizeof(double));
    });
}

int isdf_ctx_set_coords(isdf_ctx* ctx, const double* coords) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        if (!coords) isdf::fail(isdf::kInvalid, "null coordinates");
        ISDF_CUDA(cudaDeviceSynchronize());
        isdf::set_atom_coords(c, coords);
    });
}

int isdf_grid_metric(isdf_ctx* ctx, const double* left, int64_t ldl, int64_t kl, const double* right,
                     int64_t ldr, int64_t kr, const double* xyz, const double* w, int64_t n,
                     int32_t symmetrize, double* metric_host, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        if (kl < 0 || kr < 0 || n < 0 || kl > INT32_MAX || kr > INT32_MAX)
            isdf::fail(isdf::kInvalid, "invalid grid metric sizes");
        if (!metric_host || (n > 0 && (!xyz || !w)) || (n > 0 && kl > 0 && !left) || (n > 0 && kr > 0 && !right))
            isdf::fail(isdf::kInvalid, "null grid metric buffer");
        isdf::grid_metric(left, ldl, static_cast<int>(kl), right, ldr, static_cast<int>(kr), xyz, w, n,
                          symmetrize != 0, metric_host, as_stream(stream));
    });
}

int isdf_grid_metric_host(isdf_ctx* ctx, const double* left, int64_t kl, const double* right, int64_t kr,
                          const double* xyz, const double* w, int64_t n, int32_t symmetrize,
                          double* metric_host) {
    return guarded([&] {
        int dev = 0;
        if (ctx) dev = ctx_of(ctx).device;
        else ISDF_CUDA(cudaGetDevice(&dev));
        DeviceGuard dg(dev);
        if (kl < 0 || kr < 0 || n < 0 || kl > INT32_MAX || kr > INT32_MAX)
            isdf::fail(isdf::kInvalid, "invalid grid metric sizes");
        if (!metric_host || (n > 0 && (!xyz || !w)) || (n > 0 && kl > 0 && !left) || (n > 0 && kr > 0 && !right))
            isdf::fail(isdf::kInvalid, "null grid metric buffer");
        cudaStream_t s = ctx ? ctx->stream : nullptr;
        // one set given on both sides: one upload, so the device sees one set
        const bool same = left == right && kl == kr;
        isdf::DeviceBuffer<double> dl, dr, dx, dw;
        upload(dl, left, static_cast<size_t>(kl * n), s);
        if (!same) upload(dr, right, static_cast<size_t>(kr * n), s);
        upload(dx, xyz, static_cast<size_t>(3 * n), s);
        upload(dw, w, static_cast<size_t>(n), s);
        isdf::grid_metric(dl.get(), n, static_cast<int>(kl), same ? dl.get() : dr.get(), n, static_cast<int>(kr),
                          dx.get(), dw.get(), n, symmetrize != 0, metric_host, s);
    });
}

int isdf_jk(isdf_ctx* ctx, const double* x, int64_t k, const double* z, const double* dm, double* j,
            double* kout, void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        if (k < 0) isdf::fail(isdf::kInvalid, "invalid anchor count");
        if ((k > 0 && (!x || !z)) || (c.nao > 0 && !dm)) isdf::fail(isdf::kInvalid, "null J/K input");
        isdf::isdf_jk_device(c.nao, k, x, z, dm, j, kout, as_stream(stream));
    });
}

int isdf_jk_host(isdf_ctx* ctx, const double* x, int64_t k, const double* z, const double* dm, double* j,
                 double* kout) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        if (k < 0) isdf::fail(isdf::kInvalid, "invalid anchor count");
        if ((k > 0 && (!x || !z)) || (c.nao > 0 && !dm)) isdf::fail(isdf::kInvalid, "null J/K input");
        cudaStream_t s = ctx->stream;
        const int64_t nao = c.nao;
        isdf::DeviceBuffer<double> dx, dz, dd, dj(static_cast<size_t>(j ? nao * nao : 0), s),
            dk(static_cast<size_t>(kout ? nao * nao : 0), s);
        upload(dx, x, static_cast<size_t>(k * nao), s);
        upload(dz, z, static_cast<size_t>(k * k), s);
        upload(dd, dm, static_cast<size_t>(nao * nao), s);
        isdf::isdf_jk_device(nao, k, dx.get(), dz.get(), dd.get(), j ? dj.get() : nullptr,
                             kout ? dk.get() : nullptr, s);
        if (j) ISDF_CUDA(cudaMemcpyAsync(j, dj.get(), nao * nao * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (kout) ISDF_CUDA(cudaMemcpyAsync(kout, dk.get(), nao * nao * sizeof(double), cudaMemcpyDeviceToHost, s));
        ISDF_CUDA(cudaStreamSynchronize(s));
    });
}

struct isdf_rbrp_result {
    isdf::RbrpResult r;
    int64_t n = 0, nao = 0;
};

void isdf_rbrp_args_default(isdf_rbrp_args* a) {
    if (!a) return;
    isdf::RbrpParams d;
    a->batch_size = d.batch_size;
    a->block_size = d.block_size;
    a->tolerance = d.tolerance;
    a->max_rank = d.max_rank;
    a->seed = d.seed;
    a->tau_block = d.tau_block;
    a->rank_rtol = d.rank_rtol;
    a->refresh_every = d.refresh_every;
    a->svd_rtol = d.svd_rtol;
    a->compute_id = 0;
}

namespace {

isdf::RbrpParams rbrp_params(const isdf_rbrp_args* a) {
    if (!a) isdf::fail(isdf::kInvalid, "RBRP arguments are required");
    if (a->batch_size < 0 || a->block_size < 0 || a->max_rank < 0 || a->refresh_every < 0)
        isdf::fail(isdf::kInvalid, "invalid RBRP dimensions, batch size or tolerances");
    isdf::RbrpParams p;
    p.batch_size = a->batch_size;
    p.block_size = a->block_size;
    p.tolerance = a->tolerance;
    p.max_rank = a->max_rank;
    p.seed = a->seed;
    p.tau_block = a->tau_block;
    p.rank_rtol = a->rank_rtol;
    p.refresh_every = a->refresh_every;
    p.svd_rtol = a->svd_rtol;
    p.compute_id = a->compute_id != 0;
    return p;
}

}  // namespace

int isdf_rbrp_ao(isdf_ctx* ctx, const double* ao, const double* w, int64_t n, int64_t nao,
                 const isdf_rbrp_args* args, isdf_rbrp_result** out) {
    return guarded([&] {
        if (!out) isdf::fail(isdf::kInvalid, "null result handle");
        *out = nullptr;
        int dev = 0;
        if (ctx) dev = ctx_of(ctx).device;
        else ISDF_CUDA(cudaGetDevice(&dev));
        DeviceGuard dg(dev);
        const isdf::RbrpParams p = rbrp_params(args);
        if (n < 0 || nao < 0 || nao > INT32_MAX || (n > 0 && nao > 0 && (!ao || !w)))
            isdf::fail(isdf::kInvalid, "expected ao[grid,nao] and weights[grid]");
        cudaStream_t s = ctx ? ctx->stream : nullptr;
        isdf::DeviceBuffer<double> dao, dw;
        upload(dao, ao, static_cast<size_t>(n * nao), s);
        upload(dw, w, static_cast<size_t>(n), s);
        auto h = std::make_unique<isdf_rbrp_result>();
        h->r = isdf::rbrp_ao(dao.get(), dw.get(), n, static_cast<int>(nao), p, s);
        h->n = n;
        h->nao = nao;
        *out = h.release();
    });
}

int isdf_rbrp_points(isdf_ctx* ctx, const double* xyz, const double* w, int64_t n, const isdf_rbrp_args* args,
                     isdf_rbrp_result** out) {
    return guarded([&] {
        if (!out) isdf::fail(isdf::kInvalid, "null result handle");
        *out = nullptr;
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        const isdf::RbrpParams p = rbrp_params(args);
        if (n < 0 || (n > 0 && (!xyz || !w))) isdf::fail(isdf::kInvalid, "expected weights[ngrid]");
        cudaStream_t s = ctx->stream;
        isdf::DeviceBuffer<double> dx, dw, dao(static_cast<size_t>(std::max<int64_t>(n, 1)) * c.nao, s);
        upload(dx, xyz, static_cast<size_t>(3 * n), s);
        upload(dw, w, static_cast<size_t>(n), s);
        isdf::eval_ao<double>(c, dx.get(), n, dao.get(), nullptr, c.nao, s);
        auto h = std::make_unique<isdf_rbrp_result>();
        h->r = isdf::rbrp_ao(dao.get(), dw.get(), n, c.nao, p, s);
        h->n = n;
        h->nao = c.nao;
        *out = h.release();
    });
}

int isdf_rbrp_result_info(const isdf_rbrp_result* r, int64_t* rank, int64_t* nblocks, int64_t* n, int64_t* nao,
                          double* relres, double* condition, int64_t* retained, char* status, int64_t cap) {
    return guarded([&] {
        if (!r) isdf::fail(isdf::kInvalid, "null result handle");
        if (rank) *rank = static_cast<int64_t>(r->r.indices.size());
        if (nblocks) *nblocks = static_cast<int64_t>(r->r.history.size() / 4);
        if (n) *n = r->n;
        if (nao) *nao = r->nao;
        if (relres) *relres = r->r.relative_residual;
        if (condition) *condition = r->r.condition;
        if (retained) *retained = r->r.retained_rank;
        if (status && cap > 0) {
            const size_t m = std::min<size_t>(r->r.status.size(), static_cast<size_t>(cap - 1));
            std::memcpy(status, r->r.status.data(), m);
            status[m] = '\0';
        }
    });
}

int isdf_rbrp_result_copy(const isdf_rbrp_result* r, int64_t* indices, double* history, double* interp,
                          double* transform) {
    return guarded([&] {
        if (!r) isdf::fail(isdf::kInvalid, "null result handle");
        if (indices) std::copy(r->r.indices.begin(), r->r.indices.end(), indices);
        if (history) std::copy(r->r.history.begin(), r->r.history.end(), history);
        if (interp) std::copy(r->r.interp_vecs.begin(), r->r.interp_vecs.end(), interp);
        if (transform) std::copy(r->r.transform.begin(), r->r.transform.end(), transform);
    });
}

void isdf_rbrp_result_free(isdf_rbrp_result* r) { delete r; }

int isdf_sketch_factors(int64_t d, int64_t ell, uint64_t seed, double* u_host, double* v_host) {
    return guarded([&] {
        isdf::require(d >= 0 && ell >= 0, "sketch factor sizes must be non-negative");
        isdf::require(d * ell == 0 || (u_host && v_host), "null output buffer");
        isdf::sketch_factors(d, ell, seed, u_host, v_host);
    });
}

int isdf_project_axes(isdf_ctx* ctx, const double* xyz, int64_t ng, const int32_t* axes,
                      int32_t naxes, const double* W, int32_t nout, int32_t precision, double* out,
                      void* stream) {
    return guarded([&] {
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        cudaStream_t s = as_stream(stream);
        if (!axes || !W || nout <= 0 || ng < 0) isdf::fail(isdf::kInvalid, "invalid projection arguments");
        isdf::AxisSpec ax = isdf::make_axis_spec(c, axes, naxes);
        const int64_t d = static_cast<int64_t>(naxes) * c.nao;
        if (ng == 0) return;
        if (precision == ISDF_MIXED) {
            if (!isdf::project_tc_supported(naxes, nout))
                isdf::fail(isdf::kNotImplemented, "tensor-core projection needs naxes <= 4 and nout <= 64");
            std::vector<int> comps(ax.comp, ax.comp + naxes);
            isdf::DeviceBuffer<double> dW(static_cast<size_t>(d * nout), s);
            ISDF_CUDA(cudaMemcpyAsync(dW.get(), W, d * nout * sizeof(double), cudaMemcpyHostToDevice, s));
            // W row-major [a*nao + mu][j]
            const isdf::WSource src{dW.get(), static_cast<int64_t>(c.nao) * nout, nout, 1, nout, 0};
            isdf::ProjectPlan plan = isdf::make_project_plan(c, comps, nout, &src, 1, s);
            isdf::DeviceBuffer<float> P(static_cast<size_t>(ng * naxes * nout), s);
            isdf::DeviceBuffer<int> err(1, s);
            err.zero(s);
            isdf::project_tc(c, plan, xyz, nullptr, ng, nullptr, P.get(), naxes * nout, 1, nullptr,
                             nullptr, err.get(), s);
            isdf::widen_f32(P.get(), ng * naxes * nout, out, s);
            int herr = 0;
            ISDF_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
            ISDF_CUDA(cudaStreamSynchronize(s));
            if (herr) isdf::fail(isdf::kRuntime, "tensor-core projection timed out");
        } else if (precision == ISDF_FP64) {
            isdf::DeviceBuffer<double> F(static_cast<size_t>(ng * d), s), dW(static_cast<size_t>(d * nout), s);
            ISDF_CUDA(cudaMemcpyAsync(dW.get(), W, d * nout * sizeof(double), cudaMemcpyHostToDevice, s));
            isdf::eval_axis_features<double>(c, xyz, nullptr, ng, ax, F.get(), d, nullptr, nullptr, s);
            isdf::gemm_f64(ng, nout, c.nao, F.get(), d, c.nao, dW.get(), nout,
                           static_cast<int64_t>(c.nao) * nout, out, static_cast<int64_t>(naxes) * nout,
                           nout, naxes, false, s);
            ISDF_CUDA(cudaStreamSynchronize(s));
        } else {
            isdf::fail(isdf::kInvalid, "precision must be fp64 or mixed");
        }
    });
}

int isdf_pair_error_terms(int64_t n, int64_t k, const double* q, const double* H, const double* X,
                          const double* M, const double* w, double* out, void* stream) {
    return guarded([&] {
        if (n < 0 || k < 0 || !out) isdf::fail(isdf::kInvalid, "invalid pair error terms");
        if (n > 0 && (!q || !w || (k > 0 && (!H || !X || !M))))
            isdf::fail(isdf::kInvalid, "null pair error term array");
        double acc[2] = {0, 0};
        if (n > 0) isdf::pair_error_terms(n, k, q, H, X, M, w, acc, as_stream(stream));
        const double a = std::sqrt(std::max(acc[0], 0.0));
        out[0] = a;
        out[1] = acc[1] ? a / std::sqrt(acc[1]) : (a == 0 ? 0.0 : INFINITY);
    });
}

// ---- grid-sharded selection phases -----------------------------------------------
struct isdf_sketch_shard {
    isdf_ctx* ctx = nullptr;
    isdf::SketchShard st;
};

int isdf_sketch_shard_project(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz,
                              const double* w, int64_t ng, int64_t ng_total, isdf_sketch_shard** out,
                              int64_t* n_kept, int64_t* ell, double* sumsq_host, void* stream) {
    return guarded([&] {
        if (!out) isdf::fail(isdf::kInvalid, "null shard handle");
        *out = nullptr;
        if (!args) isdf::fail(isdf::kInvalid, "selection arguments are required");
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        isdf::SelectOptions o = options_of(args);
        if (o.algorithm != ISDF_RAND_SKETCH_QUADRATURE)
            isdf::fail(isdf::kInvalid, "grid-sharded selection supports rand_sketch (quadrature)");
        if (ng < 0 || ng_total < ng) isdf::fail(isdf::kInvalid, "invalid shard or total grid size");
        isdf::validate_axis_weights(o.axis_weights.empty() ? nullptr : o.axis_weights.data(),
                                    static_cast<int>(o.axes.size()));
        auto h = std::make_unique<isdf_sketch_shard>();
        h->ctx = ctx;
        isdf::sketch_shard_project(c, xyz, w, ng, o, ng_total, h->st, as_stream(stream));
        if (n_kept) *n_kept = h->st.kp.n;
        if (ell) *ell = h->st.su.ell;
        if (sumsq_host) std::memcpy(sumsq_host, h->st.sumsq, 4 * sizeof(double));
        *out = h.release();
    });
}

int isdf_sketch_shard_combine(isdf_sketch_shard* h, const double* sumsq_global, double* yt, double* delta,
                              int64_t* kept, double* kept_xyz, double* kept_w, double* scales_host,
                              void* stream) {
    return guarded([&] {
        if (!h || !sumsq_global || (!yt && h->st.kp.n)) isdf::fail(isdf::kInvalid, "invalid shard combine arguments");
        auto& c = ctx_of(h->ctx);
        DeviceGuard dg(c.device);
        std::vector<double> scales;
        isdf::sketch_shard_combine(c, h->st, sumsq_global, yt, delta, kept, kept_xyz, kept_w, scales,
                                   as_stream(stream));
        if (scales_host) std::memcpy(scales_host, scales.data(), scales.size() * sizeof(double));
    });
}

void isdf_sketch_shard_free(isdf_sketch_shard* h) { delete h; }

struct isdf_qr_shard {
    isdf_ctx* ctx = nullptr;
    std::unique_ptr<isdf::SketchQrShard> sh;
    bool verified = false;
};

int isdf_qr_shard_create(isdf_ctx* ctx, const isdf_select_args* args, double* yt, int64_t n_local, int64_t n_total,
                         int64_t pos_offset, const double* kept_xyz, const double* kept_w, double* delta,
                         const double* scales_host, isdf_qr_shard** out, int64_t* ell, int32_t* verified,
                         void* stream) {
    return guarded([&] {
        if (!out) isdf::fail(isdf::kInvalid, "null QR shard handle");
        *out = nullptr;
        if (!args || !scales_host) isdf::fail(isdf::kInvalid, "invalid distributed QR arguments");
        if (n_local > 0 && (!yt || !kept_xyz || !kept_w)) isdf::fail(isdf::kInvalid, "null distributed QR input");
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        isdf::SelectOptions o = options_of(args);
        if (o.algorithm != ISDF_RAND_SKETCH_QUADRATURE)
            isdf::fail(isdf::kInvalid, "grid-sharded selection supports rand_sketch (quadrature)");
        const std::vector<double> scales(scales_host, scales_host + o.axes.size());
        auto h = std::make_unique<isdf_qr_shard>();
        h->ctx = ctx;
        h->sh = isdf::make_sketch_qr_shard(c, o, yt, n_local, n_total, kept_xyz, kept_w, delta, scales, pos_offset,
                                           as_stream(stream));
        h->verified = delta != nullptr && h->sh->su.mixed;
        if (ell) *ell = h->sh->su.ell;
        if (verified) *verified = h->verified ? 1 : 0;
        *out = h.release();
    });
}

int isdf_qr_shard_update(isdf_qr_shard* h, int64_t j, double* key_value, int64_t* key_pos, int64_t* key_col,
                         double* energy_part, double* lower_bound) {
    return guarded([&] {
        if (!h || !key_value || !key_pos || !key_col || !energy_part || !lower_bound)
            isdf::fail(isdf::kInvalid, "null distributed QR argument");
        DeviceGuard dg(ctx_of(h->ctx).device);
        const isdf::QrShardKey k = h->sh->qr->update(j, energy_part, lower_bound);
        *key_value = k.v;
        *key_pos = k.pos;
        *key_col = k.col;
    });
}

int isdf_qr_shard_verify(isdf_qr_shard* h, int64_t j, double lower_bound, double* key_value, int64_t* key_pos,
                         int64_t* key_col) {
    return guarded([&] {
        if (!h || !key_value || !key_pos || !key_col) isdf::fail(isdf::kInvalid, "null distributed QR argument");
        DeviceGuard dg(ctx_of(h->ctx).device);
        const isdf::QrShardKey k = h->sh->qr->verify(j, lower_bound);
        *key_value = k.v;
        *key_pos = k.pos;
        *key_col = k.col;
    });
}

int isdf_qr_shard_column(isdf_qr_shard* h, int64_t col, double* rows_host) {
    return guarded([&] {
        if (!h || !rows_host) isdf::fail(isdf::kInvalid, "null distributed QR argument");
        DeviceGuard dg(ctx_of(h->ctx).device);
        h->sh->qr->column(col, rows_host);
    });
}

int isdf_qr_shard_pivot(isdf_qr_shard* h, int64_t j, const double* rows_host, int64_t pivot_col, int64_t pivot_pos,
                        int64_t moved_col, double* r_jj) {
    return guarded([&] {
        if (!h || !rows_host || !r_jj) isdf::fail(isdf::kInvalid, "null distributed QR argument");
        DeviceGuard dg(ctx_of(h->ctx).device);
        *r_jj = h->sh->qr->pivot(j, rows_host, pivot_col, pivot_pos, moved_col);
    });
}

int isdf_qr_shard_reverified(isdf_qr_shard* h, int64_t* count) {
    return guarded([&] {
        if (!h || !count) isdf::fail(isdf::kInvalid, "null distributed QR argument");
        DeviceGuard dg(ctx_of(h->ctx).device);
        *count = h->sh->qr->reverified();
    });
}

void isdf_qr_shard_free(isdf_qr_shard* h) { delete h; }

int isdf_sketch_rank(isdf_ctx* ctx, const isdf_select_args* args, int64_t n_total, const double* diag,
                     const double* energy, int64_t steps, int64_t* rank, int64_t* numerical_rank,
                     double* relative_tail) {
    return guarded([&] {
        if (!args || !rank || steps < 0 || (steps > 0 && (!diag || !energy)))
            isdf::fail(isdf::kInvalid, "invalid sketch rank arguments");
        auto& c = ctx_of(ctx);
        isdf::SelectOptions o = options_of(args);
        const isdf::SketchSetup su = isdf::sketch_setup(c, o, std::max<int64_t>(n_total, 1));
        isdf::SketchQR qr;
        qr.diag.assign(diag, diag + steps);
        qr.energy.assign(energy, energy + steps);
        qr.jpvt.assign(steps, 0);   // the pivots themselves are the caller's
        const isdf::SketchRank r = isdf::sketch_rank(qr, su.ell, n_total, o, su.physical_rank);
        *rank = r.rank;
        if (numerical_rank) *numerical_rank = r.numerical_rank;
        if (relative_tail) *relative_tail = r.relative_tail;
    });
}

int isdf_sketch_select_gathered(isdf_ctx* ctx, const isdf_select_args* args, double* yt, int64_t n,
                                const double* kept_xyz, const double* kept_w, double* delta,
                                const double* scales_host, int64_t* pivots, int64_t capacity,
                                int64_t* npivots, isdf_select_info* info, void* stream) {
    return guarded([&] {
        if (npivots) *npivots = 0;
        if (!args || !scales_host || n < 0) isdf::fail(isdf::kInvalid, "invalid gathered selection arguments");
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        isdf::SelectOptions o = options_of(args);
        if (o.algorithm != ISDF_RAND_SKETCH_QUADRATURE)
            isdf::fail(isdf::kInvalid, "grid-sharded selection supports rand_sketch (quadrature)");
        if (info) std::memset(info, 0, sizeof(*info));
        const std::vector<double> scales(scales_host, scales_host + o.axes.size());
        isdf::SketchDiagnostics d;
        std::vector<int64_t> out =
            isdf::select_sketch_gathered(c, o, yt, n, kept_xyz, kept_w, delta, scales, &d, as_stream(stream));
        if (info) {
            info->sketch_rows = d.ell;
            info->numerical_rank = d.numerical_rank;
            info->relative_residual = d.relative_tail;
            info->verifications = d.reverified;
            info->precision_used = d.precision_used;
        }
        if (static_cast<int64_t>(out.size()) > capacity) isdf::fail(isdf::kInvalid, "pivot buffer is too small");
        if (!out.empty()) std::memcpy(pivots, out.data(), out.size() * sizeof(int64_t));
        if (npivots) *npivots = static_cast<int64_t>(out.size());
    });
}

int isdf_fit_at(isdf_ctx* ctx, const double* xyz, const double* w, int64_t ng, const double* anchor_xyz,
                const double* anchor_w, int64_t k, int32_t precision, int32_t want_error, double* theta,
                isdf_fit_info* info, double* sums_host, void* stream) {
    return guarded([&] {
        const AnchorCoords ac{anchor_xyz, anchor_w};
        fit_impl(ctx, xyz, w, ng, nullptr, k, precision, nullptr, theta, info, nullptr, nullptr,
                 as_stream(stream), want_error != 0, nullptr, &ac, sums_host);
    });
}

struct isdf_pairqr_shard {
    isdf_ctx* ctx = nullptr;
    std::unique_ptr<isdf::PairQrShard> sh;
};

int isdf_pairqr_shard_create(isdf_ctx* ctx, const isdf_select_args* args, const double* xyz, const double* w,
                             int64_t ng, int64_t grid_offset, isdf_pairqr_shard** out, int64_t* n_kept,
                             int64_t* features, double* sumsq_host, void* stream) {
    return guarded([&] {
        if (!out) isdf::fail(isdf::kInvalid, "null shard handle");
        *out = nullptr;
        if (!args) isdf::fail(isdf::kInvalid, "selection arguments are required");
        auto& c = ctx_of(ctx);
        DeviceGuard dg(c.device);
        isdf::SelectOptions o = options_of(args);
        if (o.algorithm != ISDF_QRCP_DENSE && o.algorithm != ISDF_QRCP_ONLINE)
            isdf::fail(isdf::kInvalid, "the sharded pair QR takes qrcp_dense or qrcp_online");
        if (ng < 0 || grid_offset < 0) isdf::fail(isdf::kInvalid, "invalid shard size or offset");
        auto h = std::make_unique<isdf_pairqr_shard>();
        h->ctx = ctx;
        h->sh = std::make_unique<isdf::PairQrShard>(c, o, xyz, w, ng, grid_offset, as_stream(stream));
        if (n_kept) *n_kept = h->sh->n_kept();
        if (features) *features = h->sh->features();
        if (sumsq_host) h->sh->local_sumsq(sumsq_host);
        *out = h.release();
    });
}

int isdf_pairqr_shard_init(isdf_pairqr_shard* h, const double* sumsq_global, int64_t pos_offset, double* out2) {
    return guarded([&] {
        if (!h || !sumsq_global || !out2 || pos_offset < 0) isdf::fail(isdf::kInvalid, "invalid shard init arguments");
        DeviceGuard dg(ctx_of(h->ctx).device);
        h->sh->init(sumsq_global, pos_offset, out2);
    });
}

int isdf_pairqr_shard_argmax(isdf_pairqr_shard* h, double* key3) {
    return guarded([&] {
        if (!h || !key3) isdf::fail(isdf::kInvalid, "invalid shard argmax arguments");
        DeviceGuard dg(ctx_of(h->ctx).device);
        h->sh->argmax(key3);
    });
}

int isdf_pairqr_shard_row(isdf_pairqr_shard* h, int64_t col, double* row_host) {
    return guarded([&] {
        if (!h || !row_host) isdf::fail(isdf::kInvalid, "invalid shard row arguments");
        DeviceGuard dg(ctx_of(h->ctx).device);
        h->sh->row(col, row_host);
    });
}

int isdf_pairqr_shard_verify(isdf_pairqr_shard* h, const double* row_host, int64_t j, int64_t col, double* exact2) {
    return guarded([&] {
        if (!h || !row_host || !exact2 || j < 0) isdf::fail(isdf::kInvalid, "invalid shard verify arguments");
        DeviceGuard dg(ctx_of(h->ctx).device);
        *exact2 = h->sh->verify(row_host, static_cast<int>(j), col);
    });
}

int isdf_pairqr_shard_accept(isdf_pairqr_shard* h, const double* row_host, int64_t j, int64_t col, double exact2,
                             int64_t winner_pos, int32_t dense) {
    return guarded([&] {
        if (!h || !row_host || j < 0 || !(exact2 > 0)) isdf::fail(isdf::kInvalid, "invalid shard accept arguments");
        DeviceGuard dg(ctx_of(h->ctx).device);
        h->sh->accept(row_host, static_cast<int>(j), col, exact2, winner_pos, dense != 0);
    });
}

int isdf_pairqr_shard_scan(isdf_pairqr_shard* h, int64_t j, double thr2, int64_t* count) {
    return guarded([&] {
        if (!h || j < 0) isdf::fail(isdf::kInvalid, "invalid shard scan arguments");
        DeviceGuard dg(ctx_of(h->ctx).device);
        const int64_t c = h->sh->scan(static_cast<int>(j), thr2);
        if (count) *count = c;
    });
}

void isdf_pairqr_shard_free(isdf_pairqr_shard* h) {
    if (!h) return;
    DeviceGuard dg(ctx_of(h->ctx).device);
    delete h;
}

}  // extern "C"
