// Drop-in `mp_isdf` Python module over the C-ABI of libisdf_b200.so.
//
// Mirrors the reference module's names, argument meanings and error types
// (mikovtun/mp_isdf cpp/src/ao_eval_pybind.cpp:70-120,
// cpp/src/anchor_select_pybind.cpp:142-222, cpp/src/evaluation_space_pybind.hpp).
// Every computation runs on the GPU; the `space` argument is validated as in
// the reference and "host" only means the result is returned in host memory.
#include "isdf_b200.h"

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace py = pybind11;

namespace {

using IntArray = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;
using FloatArray = py::array_t<double, py::array::c_style | py::array::forcecast>;

enum class AxisType : int { AtomicOrbital = 0, AtomicOrbitalGradX, AtomicOrbitalGradY,
                            AtomicOrbitalGradZ, OccupiedOrbital };
enum class LocalAlgo : int { QRColumnPivoting = 0, OnlineQRColumnPivoting, RandomizedQuadratureKhatriRao,
                             CentroidalVoronoi, RandomizedAODensityKhatriRao,
                             RandomizedAODensityNormalizedKhatriRao };
enum class DistAlgo : int { SVD = 0, RandomizedQRColumnPivoting };

struct NotImplemented : std::runtime_error { using std::runtime_error::runtime_error; };

void check(int status) {
    if (status == ISDF_OK) return;
    const std::string msg = isdf_last_error();
    switch (status) {
    case ISDF_ERR_INVALID: throw std::invalid_argument(msg);
    case ISDF_ERR_OVERFLOW: throw std::overflow_error(msg);
    case ISDF_ERR_NOT_IMPLEMENTED: throw NotImplemented(msg);
    case ISDF_ERR_LOGIC: throw std::logic_error(msg);
    default: throw std::runtime_error(msg);
    }
}

void parse_space(const std::string& space) {
    if (space == "auto" || space == "default" || space == "host" || space == "device") return;
    throw std::invalid_argument("space must be 'auto', 'host', or 'device'");
}

FloatArray points_of(const FloatArray& coords, const char* what) {
    if (coords.ndim() != 2 || coords.shape(1) != 3) throw std::invalid_argument(what);
    return coords;
}

struct Context {
    isdf_ctx* h = nullptr;
    int64_t nao = 0;
    int32_t natm = 0, nshell = 0;
    Context(const IntArray& atm, const IntArray& bas, const FloatArray& env) {
        if (atm.ndim() != 2 || atm.shape(1) != 6 || bas.ndim() != 2 || bas.shape(1) != 8 || env.ndim() != 1)
            throw std::invalid_argument("expected atm[natm,6], bas[nbas,8], env[nenv]");
        check(isdf_ctx_create(atm.data(), static_cast<int32_t>(atm.shape(0)), bas.data(),
                              static_cast<int32_t>(bas.shape(0)), env.data(), env.shape(0), &h));
        check(isdf_ctx_info(h, &nao, &natm, &nshell));
    }
    ~Context() { if (h) isdf_ctx_destroy(h); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;

    py::array_t<double> evaluate(const FloatArray& coords, bool gradient, const std::string& space) {
        parse_space(space);
        auto pts = points_of(coords, "expected coords[ngrid,3] in Bohr");
        const py::ssize_t ng = pts.shape(0);
        std::vector<py::ssize_t> shape = gradient ? std::vector<py::ssize_t>{3, ng, static_cast<py::ssize_t>(nao)}
                                                  : std::vector<py::ssize_t>{ng, static_cast<py::ssize_t>(nao)};
        py::array_t<double> out(shape);
        double* o = out.mutable_data();
        const double* p = pts.data();
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_eval_ao_host(h, p, ng, gradient ? nullptr : o, gradient ? o : nullptr);
        }
        check(rc);
        return out;
    }

    py::array_t<int32_t> ao_atoms() const {
        py::array_t<int32_t> out(nao);
        check(isdf_ctx_ao_atoms(h, out.mutable_data()));
        return out;
    }
};

std::vector<int32_t> read_axes(py::object axes) {
    std::vector<int32_t> out;
    if (py::isinstance<py::list>(axes) || py::isinstance<py::tuple>(axes)) {
        for (auto a : axes) out.push_back(static_cast<int32_t>(a.cast<AxisType>()));
    } else {
        out.push_back(static_cast<int32_t>(axes.cast<AxisType>()));
    }
    return out;
}

// The MO coefficients of an OccupiedOrbital axis (cpp/src/anchor_select_pybind.cpp:43-53,
// cpp/src/anchor_select.cpp:43-49); an empty array when no entry needs them.
FloatArray check_occupied(const std::vector<int32_t>& axes, py::object mo_coeff, std::size_t nocc, int64_t nao) {
    bool occ = false;
    for (auto a : axes) occ |= a == ISDF_AXIS_OCC;
    if (!occ) return FloatArray();
    if (mo_coeff.is_none() || nocc == 0 || static_cast<int64_t>(nocc) > nao)
        throw std::invalid_argument(
            "OccupiedOrbital requires row-major (nao,nao) RHF mo_coeff and 1 <= nocc <= nao");
    auto c = mo_coeff.cast<FloatArray>();
    if (c.ndim() != 2 || c.shape(0) != nao || c.shape(1) != nao)
        throw std::invalid_argument("mo_coeff must have shape (nao,nao)");
    return c;
}

int64_t feature_width(const std::vector<int32_t>& axes, std::size_t nocc, int64_t nao) {
    int64_t d = 0;
    for (auto a : axes) d += a == ISDF_AXIS_OCC ? static_cast<int64_t>(nocc) : nao;
    return d;
}

struct Selector {
    std::shared_ptr<Context> ctx;
    explicit Selector(std::shared_ptr<Context> c) : ctx(std::move(c)) {}

    std::vector<int64_t> select(const FloatArray& points, const FloatArray& weights, py::object axes,
                                double tolerance, std::size_t max_rank, LocalAlgo algorithm,
                                py::object mo_coeff, std::size_t nocc, const std::string& space,
                                std::size_t batch_size, bool debug, std::size_t sketch_size,
                                std::size_t oversampling, std::uint64_t seed, bool audit,
                                py::object cvt_weights, std::size_t cvt_max_iter, double cvt_tol,
                                const std::vector<double>& axis_weights, py::object point_importance,
                                double ao_screening_threshold, const std::string& precision) {
        (void)audit; (void)cvt_max_iter; (void)cvt_tol;
        auto pts = points_of(points, "expected points[ngrid,3]");
        if (weights.ndim() != 1 || weights.shape(0) != pts.shape(0))
            throw std::invalid_argument("expected weights[ngrid]");
        auto ax = read_axes(axes);
        const bool density = algorithm == LocalAlgo::RandomizedAODensityKhatriRao ||
                             algorithm == LocalAlgo::RandomizedAODensityNormalizedKhatriRao;
        if (!cvt_weights.is_none() || algorithm == LocalAlgo::CentroidalVoronoi)
            throw NotImplemented("CVT is outside the B200 hot path (NYI)");
        // density sketches (cpp/src/anchor_select_randomized_id.cpp:104-118)
        FloatArray importance;
        if (density) {
            if (point_importance.is_none())
                throw std::invalid_argument("point_importance must have shape (ngrid,)");
            importance = FloatArray::ensure(point_importance);
            if (!importance || importance.ndim() != 1 || importance.shape(0) != pts.shape(0))
                throw std::invalid_argument("point_importance must have shape (ngrid,)");
            for (py::ssize_t i = 0; i < importance.shape(0); ++i) {
                const double m = importance.data()[i];
                if (!std::isfinite(m) || m < 0)
                    throw std::invalid_argument("point_importance must be finite and nonnegative");
            }
            if (!std::isfinite(ao_screening_threshold) || ao_screening_threshold < 0)
                throw std::invalid_argument("AO screening threshold must be finite and nonnegative");
            if (ax.size() != 1 || ax[0] != ISDF_AXIS_AO)
                throw std::invalid_argument("density Khatri-Rao sketches with non-AO axis features are NYI");
        }
        FloatArray mo = check_occupied(ax, mo_coeff, nocc, ctx->nao);
        parse_space(space);
        if (!axis_weights.empty() && axis_weights.size() != ax.size())
            throw std::invalid_argument("axis weights must match axes");
        if (precision != "fp64" && precision != "mixed")
            throw std::invalid_argument("precision must be 'fp64' or 'mixed'");
        isdf_select_args a;
        isdf_select_args_default(&a);
        a.algorithm = static_cast<int32_t>(algorithm);
        a.naxes = static_cast<int32_t>(ax.size());
        a.axes = ax.data();
        a.axis_weights = axis_weights.empty() ? nullptr : axis_weights.data();
        a.tolerance = tolerance;
        a.max_rank = static_cast<int64_t>(max_rank);
        a.batch_size = static_cast<int64_t>(batch_size);
        a.sketch_size = static_cast<int64_t>(sketch_size);
        a.oversampling = static_cast<int64_t>(oversampling);
        a.seed = seed;
        a.precision = precision == "mixed" ? ISDF_MIXED : ISDF_FP64;
        a.debug = debug;
        if (density) {
            a.point_importance = importance.data();
            a.ao_screening_threshold = ao_screening_threshold;
        }
        if (mo) {
            a.mo_coeff = mo.data();
            a.nocc = static_cast<int64_t>(nocc);
        }
        const int64_t ng = pts.shape(0);
        std::vector<int64_t> piv(static_cast<size_t>(std::max<int64_t>(ng, 1)));
        int64_t np = 0;
        isdf_select_info info{};
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_select_host(ctx->h, &a, pts.data(), weights.data(), ng, piv.data(),
                                  static_cast<int64_t>(piv.size()), &np, &info);
        }
        check(rc);
        piv.resize(np);
        return piv;
    }

    py::array_t<double> evaluate_axis(const FloatArray& points, py::object axes, py::object mo_coeff,
                                      std::size_t nocc, const std::string& space) {
        auto ax = read_axes(axes);
        FloatArray mo = check_occupied(ax, mo_coeff, nocc, ctx->nao);
        parse_space(space);
        auto pts = points_of(points, "expected points[ngrid,3]");
        const py::ssize_t ng = pts.shape(0);
        py::array_t<double> out({ng, static_cast<py::ssize_t>(feature_width(ax, nocc, ctx->nao))});
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_evaluate_axis_mo_host(ctx->h, pts.data(), ng, ax.data(), static_cast<int32_t>(ax.size()),
                                            mo ? mo.data() : nullptr, static_cast<int64_t>(nocc),
                                            out.mutable_data());
        }
        check(rc);
        return out;
    }
};

py::dict fit(const std::shared_ptr<Context>& ctx, const FloatArray& coords, const FloatArray& weights,
             py::array_t<int64_t, py::array::c_style | py::array::forcecast> anchors,
             const std::string& precision, bool pair_space_error) {
    auto pts = points_of(coords, "expected coords[ngrid,3]");
    if (weights.ndim() != 1 || weights.shape(0) != pts.shape(0))
        throw std::invalid_argument("expected weights[ngrid]");
    if (precision != "fp64" && precision != "mixed")
        throw std::invalid_argument("precision must be 'fp64' or 'mixed'");
    const int64_t ng = pts.shape(0), k = anchors.size();
    std::vector<double> theta(static_cast<size_t>(std::max<int64_t>(1, k * ng)));
    isdf_fit_info info{};
    int rc;
    {
        py::gil_scoped_release release;
        rc = isdf_fit_host(ctx->h, pts.data(), weights.data(), ng, anchors.data(), k,
                           precision == "mixed" ? ISDF_MIXED : ISDF_FP64, pair_space_error, theta.data(), &info);
    }
    check(rc);
    py::array_t<double> th({static_cast<py::ssize_t>(k), static_cast<py::ssize_t>(info.n_kept)});
    std::memcpy(th.mutable_data(), theta.data(), sizeof(double) * k * info.n_kept);
    py::dict d;
    d["interp_vecs"] = th;
    d["retained_rank"] = info.retained_rank;
    d["condition"] = info.condition;
    d["max_abs_physical_coefficient"] = info.max_abs_physical_coefficient;
    d["pair_l2"] = info.pair_l2;
    d["pair_relative"] = info.pair_relative;
    std::vector<double> tw(info.theta_w, info.theta_w + std::min<int64_t>(k, 64));
    d["theta_w"] = tw;
    d["fit_path"] = info.fit_path == 0   ? "fp64"
                    : info.fit_path == 1 ? "mixed"
                    : info.fit_path == 3 ? "mixed-refined"
                                         : "fp64-fallback";
    d["mixed_bound"] = info.mixed_bound;
    return d;
}

}  // namespace

PYBIND11_MODULE(mp_isdf, m) {
    m.doc() = "B200 (sm_100a) ISDF hot path: spherical AO values/gradients, anchor selection and fit";
    m.attr("cuda_enabled") = true;
    m.attr("backend") = "b200";
    py::register_exception<NotImplemented>(m, "NotImplementedError", PyExc_NotImplementedError);

    py::class_<Context, std::shared_ptr<Context>>(m, "LibcintContext",
        "Own a private copy of libcint tables and cache the shell table on the B200.")
        .def(py::init<const IntArray&, const IntArray&, const FloatArray&>(), py::arg("atm"),
             py::arg("bas"), py::arg("env"))
        .def_property_readonly("nao", [](const Context& c) { return c.nao; })
        .def_property_readonly("natm", [](const Context& c) { return c.natm; })
        .def_property_readonly("ao_atoms", &Context::ao_atoms)
        .def("eval_ao", [](Context& c, const FloatArray& coords, const std::string& space) {
            return c.evaluate(coords, false, space);
        }, py::arg("coords"), py::arg("space") = "auto", "Return real spherical AOs with shape (ngrid, nao).")
        .def("eval_ao_gradient", [](Context& c, const FloatArray& coords, const std::string& space) {
            return c.evaluate(coords, true, space);
        }, py::arg("coords"), py::arg("space") = "auto", "Return x,y,z AO gradients with shape (3, ngrid, nao).");

    // grid Coulomb metric (python/isdf.py:48-97): interpolation vectors k x n
    auto metric = [](const FloatArray& left, py::object right, const FloatArray& coords, const FloatArray& weights) {
        if (left.ndim() != 2) throw std::invalid_argument("interpolation vectors must have shape (k, ngrid)");
        auto pts = points_of(coords, "expected coords[ngrid,3]");
        const int64_t n = pts.shape(0);
        if (weights.ndim() != 1 || weights.shape(0) != n || left.shape(1) != n)
            throw std::invalid_argument("interpolation vectors, coords and weights disagree on ngrid");
        const bool sym = right.is_none();
        FloatArray r = sym ? left : right.cast<FloatArray>();
        if (r.ndim() != 2 || r.shape(1) != n)
            throw std::invalid_argument("interpolation vectors, coords and weights disagree on ngrid");
        py::array_t<double> out({left.shape(0), r.shape(0)});
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_grid_metric_host(nullptr, left.data(), left.shape(0), r.data(), r.shape(0), pts.data(),
                                       weights.data(), n, sym ? 1 : 0, out.mutable_data());
        }
        check(rc);
        return out;
    };
    m.def("grid_coulomb_metric", [metric](const FloatArray& interp_vecs, const FloatArray& coords,
                                          const FloatArray& weights) {
        return metric(interp_vecs, py::none(), coords, weights);
    }, py::arg("interp_vecs"), py::arg("coords"), py::arg("weights"));
    m.def("grid_cross_metric", [metric](const FloatArray& left, const FloatArray& right, const FloatArray& coords,
                                        const FloatArray& weights) {
        return metric(left, right, coords, weights);
    }, py::arg("left"), py::arg("right"), py::arg("coords"), py::arg("weights"));
    // ISDF J and K (python/isdf.py:130-151) on the device: x k x nao anchor AO
    // values, z k x k metric, dm nao x nao (symmetric)
    m.def("isdf_jk", [](Context& c, const FloatArray& x, const FloatArray& z, const FloatArray& dm) {
        if (x.ndim() != 2 || x.shape(1) != c.nao) throw std::invalid_argument("X must have shape (k, nao)");
        const int64_t k = x.shape(0);
        if (z.ndim() != 2 || z.shape(0) != k || z.shape(1) != k)
            throw std::invalid_argument("Coulomb metric has the wrong anchor dimensions");
        if (dm.ndim() != 2 || dm.shape(0) != c.nao || dm.shape(1) != c.nao)
            throw std::invalid_argument("dm must be a finite AO density matrix of shape (nao,nao)");
        py::array_t<double> j({c.nao, c.nao}), kk({c.nao, c.nao});
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_jk_host(c.h, x.data(), k, z.data(), dm.data(), j.mutable_data(), kk.mutable_data());
        }
        check(rc);
        return py::make_tuple(j, kk);
    }, py::arg("context"), py::arg("x"), py::arg("z"), py::arg("dm"));
    // RBRP (cpp/src/anchor_select_pybind.cpp:68-140): result dict in the reference's layout
    auto rbrp_dict = [](isdf_rbrp_result* h, bool compute_id) {
        struct Free { isdf_rbrp_result* h; ~Free() { isdf_rbrp_result_free(h); } } guard{h};
        int64_t rank = 0, nb = 0, n = 0, nao = 0, ret = 0;
        double rel = 0, cond = 0;
        char status[64];
        check(isdf_rbrp_result_info(h, &rank, &nb, &n, &nao, &rel, &cond, &ret, status, sizeof(status)));
        py::array_t<int64_t> idx(rank);
        py::array_t<double> hist({static_cast<py::ssize_t>(nb), py::ssize_t(4)});
        py::array_t<double> theta({static_cast<py::ssize_t>(rank), static_cast<py::ssize_t>(compute_id ? n : 0)});
        py::array_t<double> transform({static_cast<py::ssize_t>(rank), static_cast<py::ssize_t>(compute_id ? nao * nao : 0)});
        check(isdf_rbrp_result_copy(h, idx.mutable_data(), hist.mutable_data(),
                                    compute_id ? theta.mutable_data() : nullptr,
                                    compute_id ? transform.mutable_data() : nullptr));
        py::dict out;
        py::list indices;
        for (int64_t i = 0; i < rank; ++i) indices.append(idx.data()[i]);
        out["indices"] = indices;
        out["relative_residual"] = rel;
        out["status"] = std::string(status);
        out["condition"] = cond;
        out["retained_rank"] = ret;
        out["history"] = hist;
        if (compute_id) {
            out["interp_vecs"] = theta;
            out["transform"] = transform;
        }
        return out;
    };
    auto rbrp_args_of = [](std::size_t batch_size, std::size_t block_size, double tolerance, std::size_t max_rank,
                           std::uint64_t seed, py::object tau_block, double rank_rtol, std::size_t refresh_every,
                           double svd_rtol, bool compute_id) {
        isdf_rbrp_args a;
        isdf_rbrp_args_default(&a);
        a.batch_size = static_cast<int64_t>(batch_size);
        a.block_size = static_cast<int64_t>(block_size);
        a.tolerance = tolerance;
        a.max_rank = static_cast<int64_t>(max_rank);
        a.seed = seed;
        a.tau_block = tau_block.is_none() ? std::numeric_limits<double>::quiet_NaN() : tau_block.cast<double>();
        a.rank_rtol = rank_rtol;
        a.refresh_every = static_cast<int64_t>(refresh_every);
        a.svd_rtol = svd_rtol;
        a.compute_id = compute_id ? 1 : 0;
        return a;
    };
    m.def("rbrp_ao_cpu", [rbrp_dict, rbrp_args_of](const FloatArray& ao, const FloatArray& weights, std::size_t batch_size,
                                                  std::size_t block_size, double tolerance, std::size_t max_rank,
                                                  std::uint64_t seed, py::object tau_block, double rank_rtol,
                                                  std::size_t refresh_every, double svd_rtol, bool compute_id) {
        if (ao.ndim() != 2 || weights.ndim() != 1 || weights.shape(0) != ao.shape(0))
            throw std::invalid_argument("expected ao[grid,nao] and weights[grid]");
        isdf_rbrp_args a = rbrp_args_of(batch_size, block_size, tolerance, max_rank, seed, tau_block, rank_rtol,
                                        refresh_every, svd_rtol, compute_id);
        isdf_rbrp_result* h = nullptr;
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_rbrp_ao(nullptr, ao.data(), weights.data(), ao.shape(0), ao.shape(1), &a, &h);
        }
        check(rc);
        return rbrp_dict(h, compute_id);
    }, py::arg("ao"), py::arg("weights"), py::arg("batch_size") = 128, py::arg("block_size") = 16,
       py::arg("tolerance") = 1e-10, py::arg("max_rank") = 0, py::arg("seed") = 7, py::arg("tau_block") = py::none(),
       py::arg("rank_rtol") = 1e-12, py::arg("refresh_every") = 8, py::arg("svd_rtol") = 1e-12,
       py::arg("compute_id") = false,
       "AO-only RBRP on nonzero grid rows (computed on the GPU); optional ID.");
    m.def("rbrp_ao_device", [rbrp_dict, rbrp_args_of](const Selector& selector, const FloatArray& points,
                                                     const FloatArray& weights, std::size_t batch_size,
                                                     std::size_t block_size, double tolerance, std::size_t max_rank,
                                                     std::uint64_t seed, py::object tau_block, double rank_rtol,
                                                     std::size_t refresh_every, double svd_rtol, bool compute_id) {
        auto pts = points_of(points, "expected points[ngrid,3]");
        if (weights.ndim() != 1 || weights.shape(0) != pts.shape(0))
            throw std::invalid_argument("expected weights[ngrid]");
        isdf_rbrp_args a = rbrp_args_of(batch_size, block_size, tolerance, max_rank, seed, tau_block, rank_rtol,
                                        refresh_every, svd_rtol, compute_id);
        isdf_rbrp_result* h = nullptr;
        int rc;
        {
            py::gil_scoped_release release;
            rc = isdf_rbrp_points(selector.ctx->h, pts.data(), weights.data(), pts.shape(0), &a, &h);
        }
        check(rc);
        return rbrp_dict(h, compute_id);
    }, py::arg("selector"), py::arg("points"), py::arg("weights"), py::arg("batch_size") = 128,
       py::arg("block_size") = 16, py::arg("tolerance") = 1e-10, py::arg("max_rank") = 0, py::arg("seed") = 7,
       py::arg("tau_block") = py::none(), py::arg("rank_rtol") = 1e-12, py::arg("refresh_every") = 8,
       py::arg("svd_rtol") = 1e-12, py::arg("compute_id") = false,
       "AO-only RBRP with the AOs evaluated on the device; optional ID.");
    m.def("eval_ao", [](const IntArray& atm, const IntArray& bas, const FloatArray& env,
                        const FloatArray& coords, const std::string& space) {
        Context c(atm, bas, env);
        return c.evaluate(coords, false, space);
    }, py::arg("atm"), py::arg("bas"), py::arg("env"), py::arg("coords"), py::arg("space") = "auto");
    m.def("eval_ao_gradient", [](const IntArray& atm, const IntArray& bas, const FloatArray& env,
                                 const FloatArray& coords, const std::string& space) {
        Context c(atm, bas, env);
        return c.evaluate(coords, true, space);
    }, py::arg("atm"), py::arg("bas"), py::arg("env"), py::arg("coords"), py::arg("space") = "auto");

    py::enum_<AxisType>(m, "AxisType")
        .value("AtomicOrbital", AxisType::AtomicOrbital)
        .value("AtomicOrbitalGradX", AxisType::AtomicOrbitalGradX)
        .value("AtomicOrbitalGradY", AxisType::AtomicOrbitalGradY)
        .value("AtomicOrbitalGradZ", AxisType::AtomicOrbitalGradZ)
        .value("OccupiedOrbital", AxisType::OccupiedOrbital);
    py::enum_<LocalAlgo>(m, "LocalAnchorSelectionAlgorithm")
        .value("QRColumnPivoting", LocalAlgo::QRColumnPivoting)
        .value("OnlineQRColumnPivoting", LocalAlgo::OnlineQRColumnPivoting)
        .value("RandomizedQuadratureKhatriRao", LocalAlgo::RandomizedQuadratureKhatriRao)
        .value("CentroidalVoronoi", LocalAlgo::CentroidalVoronoi)
        .value("RandomizedAODensityKhatriRao", LocalAlgo::RandomizedAODensityKhatriRao)
        .value("RandomizedAODensityNormalizedKhatriRao", LocalAlgo::RandomizedAODensityNormalizedKhatriRao);
    py::enum_<DistAlgo>(m, "DistributedAnchorSelectionAlgorithm")
        .value("SVD", DistAlgo::SVD)
        .value("RandomizedQRColumnPivoting", DistAlgo::RandomizedQRColumnPivoting);

    py::class_<Selector>(m, "AnchorSelection")
        .def(py::init<std::shared_ptr<Context>>(), py::arg("context"), py::keep_alive<1, 2>())
        .def_property_readonly("nao", [](const Selector& s) { return s.ctx->nao; })
        .def("select", &Selector::select, py::arg("points"), py::arg("weights"), py::arg("axes"),
             py::arg("tolerance") = 1e-10, py::arg("max_rank") = 0,
             py::arg("algorithm") = LocalAlgo::QRColumnPivoting, py::arg("mo_coeff") = py::none(),
             py::arg("nocc") = 0, py::arg("space") = "auto", py::arg("batch_size") = 128,
             py::arg("debug") = false, py::arg("sketch_size") = 128, py::arg("oversampling") = 16,
             py::arg("seed") = 7, py::arg("audit") = false, py::arg("cvt_weights") = py::none(),
             py::arg("cvt_max_iter") = 100, py::arg("cvt_tol") = 1e-5,
             py::arg("axis_weights") = std::vector<double>{}, py::arg("point_importance") = py::none(),
             py::arg("ao_screening_threshold") = 1e-24, py::arg("precision") = "fp64",
             "Select original grid indices in pivot order (QRCP / online QRCP / quadrature sketch).")
        .def("evaluate_axis", &Selector::evaluate_axis, py::arg("points"), py::arg("axes"),
             py::arg("mo_coeff") = py::none(), py::arg("nocc") = 0, py::arg("space") = "auto",
             "Evaluate concatenated axis functions (ngrid, naxes*nao).");

    py::class_<Context>* unused = nullptr;
    (void)unused;
    struct Distributed { std::shared_ptr<Context> ctx; };
    py::class_<Distributed>(m, "DistributedAnchorSelection")
        .def(py::init([](std::shared_ptr<Context> c) { return Distributed{std::move(c)}; }),
             py::arg("context"), py::keep_alive<1, 2>())
        .def("select", [](const Distributed&, py::object, py::object, py::object, DistAlgo) {
            throw std::logic_error("distributed SLATE SVD anchor selection is not implemented");
        }, py::arg("points"), py::arg("weights"), py::arg("axes"), py::arg("algorithm") = DistAlgo::SVD);

    m.def("fit", &fit, py::arg("context"), py::arg("coords"), py::arg("weights"),
          py::arg("anchor_indices"), py::arg("precision") = "fp64", py::arg("pair_space_error") = true,
          "Interpolation vectors Theta (k, n_nonzero_weight) for the given anchors, with the "
          "pair-space error evaluated in FP64.");
}
