// CPU oracle for the ISDF hot path -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++ (OpenMP for the timed CPU baseline), the
// reference algorithm of mikovtun/mp_isdf for the hot path.  It is linked
// only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
// the checker; the product library never includes or calls it.
//
// Parity pinning: the reference cannot be built in this environment (its
// CMake configure fetches Kokkos, LAPACK++, SLATE, libcint and MAGMA over the
// network), so this restatement is pinned against the known answers held by
// the reference's own tests (three unit-coefficient s shells -> 6 pivots and
// scipy QRCP pivot equality, the signed-weight pair error sqrt(24), the
// Khatri-Rao identity, Theta == lstsq / w_anchor); see tests/test_oracle.py.
// The cartesian->spherical matrices are passed in from oracle/oracle.py,
// which derives them independently of the product code.
//
// Citations are to files of the reference project.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_error;

struct OShell {
    int atom, l, nprim, nctr, ncart, nsph;
    int exp_off, coeff_off, tr_off, ao_off;
    double x, y, z;
};

struct OContext {
    std::vector<OShell> shells;
    std::vector<double> env;
    std::vector<double> tr;     // per shell: nsph x ncart, row-major
    std::vector<int> ao_atom;   // atom owning each AO
    int nao = 0;
    int natm = 0;
};

// cpp/src/ao_eval.cpp:22-28
inline double integer_power(double x, int n)
{
    double v = 1.0;
    for (int i = 0; i < n; ++i) v *= x;
    return v;
}

// cpp/src/ao_eval.cpp:30-44 -- libcint cartesian order x^l, x^(l-1)y, ...
inline void cartesian_powers(int l, int index, int& lx, int& ly, int& lz)
{
    for (lx = l; lx >= 0; --lx) {
        const int count = l - lx + 1;
        if (index < count) {
            ly = l - lx - index;
            lz = index;
            return;
        }
        index -= count;
    }
    lx = ly = lz = 0;
}

// One (point, shell) work item of cpp/src/ao_eval.cpp:207-249.
inline void eval_shell(const OContext& c, const OShell& b, const double* p,
                       bool gradient, std::size_t point, std::size_t npoints,
                       double* out)
{
    const int nao = c.nao;
    const double x = p[0] - b.x, y = p[1] - b.y, z = p[2] - b.z;
    const double r2 = x * x + y * y + z * z;
    for (int ctr = 0; ctr < b.nctr; ++ctr) {
        double radial = 0.0, radial_prime = 0.0;
        for (int prim = 0; prim < b.nprim; ++prim) {
            const double alpha = c.env[b.exp_off + prim];
            const double term = c.env[b.coeff_off + ctr * b.nprim + prim] * std::exp(-alpha * r2);
            radial += term;
            if (gradient) radial_prime -= alpha * term;
        }
        for (int s = 0; s < b.nsph; ++s) {
            double value = 0, dx = 0, dy = 0, dz = 0;
            for (int cc = 0; cc < b.ncart; ++cc) {
                int lx, ly, lz;
                cartesian_powers(b.l, cc, lx, ly, lz);
                const double px = integer_power(x, lx), py = integer_power(y, ly),
                             pz = integer_power(z, lz);
                const double t = c.tr[b.tr_off + s * b.ncart + cc];
                value += t * px * py * pz;
                if (gradient) {
                    if (lx) dx += t * lx * integer_power(x, lx - 1) * py * pz;
                    if (ly) dy += t * ly * px * integer_power(y, ly - 1) * pz;
                    if (lz) dz += t * lz * px * py * integer_power(z, lz - 1);
                }
            }
            const std::size_t index = point * nao + b.ao_off + ctr * b.nsph + s;
            if (gradient) {
                const std::size_t stride = npoints * static_cast<std::size_t>(nao);
                out[index] = radial * dx + 2.0 * x * radial_prime * value;
                out[stride + index] = radial * dy + 2.0 * y * radial_prime * value;
                out[2 * stride + index] = radial * dz + 2.0 * z * radial_prime * value;
            } else {
                out[index] = radial * value;
            }
        }
    }
}

void eval_points(const OContext& c, const double* pts, std::size_t n, bool gradient, double* out)
{
#pragma omp parallel for schedule(static)
    for (long long p = 0; p < static_cast<long long>(n); ++p)
        for (const auto& b : c.shells)
            eval_shell(c, b, pts + 3 * p, gradient, static_cast<std::size_t>(p), n, out);
}

// Axis codes: 0 ao, 1 dx, 2 dy, 3 dz (cpp/include/enums.hpp:4-10).
// Concatenated scaled features (cpp/include/anchor_select_impl.hpp:51-79).
void axis_features(const OContext& c, const double* pts, std::size_t n, const int* axes,
                   int naxes, const double* scales, double* out)
{
    const int nao = c.nao;
    const std::size_t width = static_cast<std::size_t>(naxes) * nao;
#pragma omp parallel
    {
        std::vector<double> val(nao), grad(3 * static_cast<std::size_t>(nao));
#pragma omp for schedule(static)
        for (long long g = 0; g < static_cast<long long>(n); ++g) {
            for (const auto& b : c.shells) eval_shell(c, b, pts + 3 * g, false, 0, 1, val.data());
            for (const auto& b : c.shells) eval_shell(c, b, pts + 3 * g, true, 0, 1, grad.data());
            for (int a = 0; a < naxes; ++a) {
                const double* src = axes[a] == 0 ? val.data() : grad.data() + (axes[a] - 1) * nao;
                const double s = scales ? scales[a] : 1.0;
                for (int j = 0; j < nao; ++j) out[g * width + a * nao + j] = s * src[j];
            }
        }
    }
}

} // namespace

extern "C" {

const char* oracle_last_error() { return g_error.c_str(); }

int oracle_num_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Shell table as in cpp/src/ao_eval.cpp:94-142; `c2s` holds, for l = 0..lmax,
// the nsph x ncart spherical transform (including the s/p scaling of
// ao_eval.cpp:135-137) concatenated in order of l.
void* oracle_ctx_create(const int32_t* atm, int natm, const int32_t* bas, int nbas,
                        const double* env, long long nenv, const double* c2s, int lmax)
{
    try {
        auto* c = new OContext;
        c->env.assign(env, env + nenv);
        c->natm = natm;
        std::vector<int> c2s_off(lmax + 2, 0);
        for (int l = 0; l <= lmax; ++l)
            c2s_off[l + 1] = c2s_off[l] + (2 * l + 1) * (l + 1) * (l + 2) / 2;
        for (int i = 0; i < nbas; ++i) {
            const int32_t* b = bas + 8 * i;
            const int atom = b[0], l = b[1], np = b[2], nc = b[3];
            if (atom < 0 || atom >= natm || l < 0 || l > lmax || np <= 0 || nc <= 0)
                throw std::invalid_argument("invalid basis shell");
            OShell s{};
            s.atom = atom; s.l = l; s.nprim = np; s.nctr = nc;
            s.ncart = (l + 1) * (l + 2) / 2; s.nsph = 2 * l + 1;
            s.exp_off = b[5]; s.coeff_off = b[6];
            s.tr_off = static_cast<int>(c->tr.size());
            s.ao_off = c->nao;
            const int pc = atm[6 * atom + 1];
            s.x = env[pc]; s.y = env[pc + 1]; s.z = env[pc + 2];
            c->tr.insert(c->tr.end(), c2s + c2s_off[l], c2s + c2s_off[l + 1]);
            c->shells.push_back(s);
            for (int k = 0; k < s.nsph * nc; ++k) c->ao_atom.push_back(atom);
            c->nao += s.nsph * nc;
        }
        return c;
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void oracle_ctx_destroy(void* ctx) { delete static_cast<OContext*>(ctx); }
int oracle_ctx_nao(void* ctx) { return static_cast<OContext*>(ctx)->nao; }

void oracle_ao_atoms(void* ctx, int32_t* out)
{
    auto* c = static_cast<OContext*>(ctx);
    std::copy(c->ao_atom.begin(), c->ao_atom.end(), out);
}

// values (n, nao) or gradients (3, n, nao): cpp/src/ao_eval.cpp:164-252
void oracle_eval_ao(void* ctx, const double* pts, long long n, int gradient, double* out)
{
    eval_points(*static_cast<OContext*>(ctx), pts, static_cast<std::size_t>(n), gradient != 0, out);
}

void oracle_axis_features(void* ctx, const double* pts, long long n, const int* axes,
                          int naxes, const double* scales, double* out)
{
    axis_features(*static_cast<OContext*>(ctx), pts, static_cast<std::size_t>(n), axes,
                  naxes, scales, out);
}

// Multi-axis Frobenius norms over nonzero-weight points, std::hypot
// accumulation in the reference order (cpp/src/anchor_select.cpp:441-470).
// Sequential by construction; use for small grids.
int oracle_axis_norms_hypot(void* ctx, const double* pts, const double* w, long long n,
                            const int* axes, int naxes, double* norms)
{
    auto* c = static_cast<OContext*>(ctx);
    const int nao = c->nao;
    std::vector<double> f(static_cast<std::size_t>(naxes) * nao);
    for (int a = 0; a < naxes; ++a) norms[a] = 0.0;
    int any = 0;
    for (long long g = 0; g < n; ++g) {
        if (!std::isfinite(w[g])) { g_error = "grid weights must be finite"; return -1; }
        if (w[g] == 0) continue;
        any = 1;
        axis_features(*c, pts + 3 * g, 1, axes, naxes, nullptr, f.data());
        for (int a = 0; a < naxes; ++a)
            for (int j = 0; j < nao; ++j)
                norms[a] = std::hypot(norms[a], f[static_cast<std::size_t>(a) * nao + j]);
    }
    return any;
}

// Same norms with OpenMP sum-of-squares (CPU baseline; identical to within
// rounding).
void oracle_axis_norms_sq(void* ctx, const double* pts, const double* w, long long n,
                          const int* axes, int naxes, double* norms)
{
    auto* c = static_cast<OContext*>(ctx);
    const int nao = c->nao;
    std::vector<double> acc(naxes, 0.0);
#pragma omp parallel
    {
        std::vector<double> f(static_cast<std::size_t>(naxes) * nao), loc(naxes, 0.0);
#pragma omp for schedule(static)
        for (long long g = 0; g < n; ++g) {
            if (w[g] == 0) continue;
            axis_features(*c, pts + 3 * g, 1, axes, naxes, nullptr, f.data());
            for (int a = 0; a < naxes; ++a)
                for (int j = 0; j < nao; ++j) {
                    const double v = f[static_cast<std::size_t>(a) * nao + j];
                    loc[a] += v * v;
                }
        }
#pragma omp critical
        for (int a = 0; a < naxes; ++a) acc[a] += loc[a];
    }
    for (int a = 0; a < naxes; ++a) norms[a] = std::sqrt(acc[a]);
}

// Gaussian factors U, V (d x ell, row-major u[a*ell+s]) from two
// independent std::mt19937_64 streams through std::normal_distribution
// (cpp/src/anchor_select_randomized_id.cpp:269-277).
void oracle_sketch_factors(long long d, long long ell, uint64_t seed, double* u, double* v)
{
    std::mt19937_64 gen_u(seed), gen_v(seed ^ 0x9e3779b97f4a7c15ULL);
    std::normal_distribution<double> normal_u(0, 1), normal_v(0, 1);
    for (long long i = 0; i < d * ell; ++i) {
        u[i] = normal_u(gen_u);
        v[i] = normal_v(gen_v);
    }
}

// Khatri-Rao quadrature sketch Y[g*ell+s] = sqrt|w_g|/sqrt(ell) (f_g.u_s)(f_g.v_s)
// over the given (already weight-filtered) points
// (cpp/src/anchor_select_randomized_id.cpp:281-309).
void oracle_sketch(void* ctx, const double* pts, const double* w, long long n,
                   const int* axes, int naxes, const double* scales,
                   const double* u, const double* v, long long ell, double* y)
{
    auto* c = static_cast<OContext*>(ctx);
    const std::size_t d = static_cast<std::size_t>(naxes) * c->nao;
    const double scaling = 1 / std::sqrt(static_cast<double>(ell));
#pragma omp parallel
    {
        std::vector<double> f(d);
#pragma omp for schedule(static)
        for (long long g = 0; g < n; ++g) {
            axis_features(*c, pts + 3 * g, 1, axes, naxes, scales, f.data());
            const double sw = std::sqrt(std::abs(w[g]));
            for (long long s = 0; s < ell; ++s) {
                double left = 0, right = 0;
                for (std::size_t a = 0; a < d; ++a) {
                    left += f[a] * u[a * ell + s];
                    right += f[a] * v[a * ell + s];
                }
                y[g * ell + s] = scaling * sw * left * right;
            }
        }
    }
}

// Per-point Gram quantities of the fit for AO values phi_g:
//   G[g,k] = phi_g . phi_a(k),  q[g] = phi_g . phi_g.
void oracle_grid_gram(void* ctx, const double* pts, long long n, const double* anchor_ao,
                      long long k, double* G, double* q)
{
    auto* c = static_cast<OContext*>(ctx);
    const int nao = c->nao;
#pragma omp parallel
    {
        std::vector<double> f(nao);
#pragma omp for schedule(static)
        for (long long g = 0; g < n; ++g) {
            for (const auto& b : c->shells) eval_shell(*c, b, pts + 3 * g, false, 0, 1, f.data());
            double qq = 0;
            for (int m = 0; m < nao; ++m) qq += f[m] * f[m];
            q[g] = qq;
            for (long long a = 0; a < k; ++a) {
                double s = 0;
                for (int m = 0; m < nao; ++m) s += f[m] * anchor_ao[a * nao + m];
                G[g * k + a] = s;
            }
        }
    }
}

// Fit + pair error in the Gram form for CPU timing:
//   X_g = T (G_g o G_g), theta[k,g] = X_g[k]/w_anchor[k]  (python/isdf.py:238-263)
//   err^2 = sum |w_g| (q_g^2 - 2 X_g.h_g + X_g^T M X_g)     (python/isdf.py:154-191)
void oracle_fit_apply(long long n, long long k, const double* G, const double* q,
                      const double* w, const double* T, const double* M,
                      const double* anchor_w, double* theta, double* err2, double* exact2)
{
    double e_acc = 0, x_acc = 0;
#pragma omp parallel reduction(+ : e_acc, x_acc)
    {
        std::vector<double> h(k), x(k);
#pragma omp for schedule(static)
        for (long long g = 0; g < n; ++g) {
            for (long long a = 0; a < k; ++a) h[a] = G[g * k + a] * G[g * k + a];
            double xh = 0, xmx = 0;
            for (long long a = 0; a < k; ++a) {
                double s = 0;
                for (long long b = 0; b < k; ++b) s += T[a * k + b] * h[b];
                x[a] = s;
                theta[a * n + g] = s / anchor_w[a];
                xh += s * h[a];
            }
            for (long long a = 0; a < k; ++a) {
                double s = 0;
                for (long long b = 0; b < k; ++b) s += M[a * k + b] * x[b];
                xmx += x[a] * s;
            }
            const double aw = std::abs(w[g]);
            e_acc += aw * (q[g] * q[g] - 2 * xh + xmx);
            x_acc += aw * q[g] * q[g];
        }
    }
    *err2 = e_acc;
    *exact2 = x_acc;
}

// Weighted draws of RBRP (cpp/src/anchor_select_rbrp.cpp:249-258): one
// std::mt19937_64(seed) for the whole run and a fresh
// std::discrete_distribution over the remaining candidates' weights per draw.
void* oracle_rng_new(uint64_t seed) { return new std::mt19937_64(seed); }
void oracle_rng_free(void* rng) { delete static_cast<std::mt19937_64*>(rng); }
long long oracle_rng_discrete(void* rng, const double* w, long long n)
{
    std::discrete_distribution<std::size_t> dist(w, w + n);
    return static_cast<long long>(dist(*static_cast<std::mt19937_64*>(rng)));
}

} // extern "C"
