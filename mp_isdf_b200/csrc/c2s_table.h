// Compile-time cartesian -> real-spherical coefficients (l <= 6).
//
// Rows m = -l..l of r^l Y_lm (unit-sphere normalised real harmonics without
// the Condon-Shortley phase) expanded in the libcint cartesian order, from the
// closed-form expansion of real regular solid harmonics (Helgaker, Jorgensen &
// Olsen, "Molecular Electronic-Structure Theory", eqs. 6.4.47-6.4.50) times
// sqrt((2l+1)/4pi).  l = 0 is 1/sqrt(4pi) and l = 1 keeps the (x, y, z) order
// scaled by sqrt(3/4pi), as the reference does for libcint's s/p path
// (cpp/src/ao_eval.cpp:132-138).  Everything is constexpr so that unrolled
// shell code multiplies only by the nonzero coefficients, as compile-time
// constants.
#pragma once

#ifndef __CUDACC__
#define ISDF_HD
#else
#define ISDF_HD __host__ __device__
#endif

namespace isdf {
namespace c2s_detail {

ISDF_HD constexpr double cfact(int n) {
    double r = 1;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}
ISDF_HD constexpr double cbinom(int n, int k) {
    return (k < 0 || k > n) ? 0.0 : cfact(n) / (cfact(k) * cfact(n - k));
}
ISDF_HD constexpr double cpow(double x, int n) {
    double r = 1;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}
// Newton iteration to a fixed point (the arguments here are small rationals).
ISDF_HD constexpr double csqrt(double x) {
    if (x <= 0) return 0;
    double r = x < 1 ? 1.0 : x;
    for (int i = 0; i < 200; ++i) {
        const double next = 0.5 * (r + x / r);
        if (next == r) break;
        r = next;
    }
    return r;
}
ISDF_HD constexpr int cabs(int x) { return x < 0 ? -x : x; }
constexpr double kPi = 3.14159265358979323846;

// Cartesian index c of angular momentum l in libcint order -> (lx, lz).
ISDF_HD constexpr int cart_lx(int l, int c) {
    int x = l;
    while (c >= l - x + 1) { c -= l - x + 1; --x; }
    return x;
}
ISDF_HD constexpr int cart_lz(int l, int c) {
    int x = l;
    while (c >= l - x + 1) { c -= l - x + 1; --x; }
    return c;
}

}  // namespace c2s_detail

// Coefficient of cartesian monomial c in spherical component s (m = s - l).
ISDF_HD constexpr double c2s_coef(int l, int s, int c) {
    using namespace c2s_detail;
    if (l == 0) return 1.0 / csqrt(4 * kPi);
    if (l == 1) return s == c ? csqrt(3.0 / (4 * kPi)) : 0.0;
    const int m = s - l, am = cabs(m);
    const int lx = cart_lx(l, c), lz = cart_lz(l, c), ly = l - lx - lz;
    const double pref = csqrt((2 * l + 1) / (4 * kPi));
    const double norm = 1.0 / (cpow(2.0, am) * cfact(l)) *
                        csqrt(2.0 * cfact(l + am) * cfact(l - am) / (m == 0 ? 2.0 : 1.0));
    const int wm = m < 0 ? 1 : 0;
    double sum = 0;
    for (int t = 0; t <= (l - am) / 2; ++t)
        for (int u = 0; u <= t; ++u)
            for (int w = wm; w <= am; w += 2) {
                if (2 * t + am - 2 * u - w != lx || 2 * u + w != ly || l - 2 * t - am != lz) continue;
                const int sgn = t + (w - wm) / 2;
                sum += ((sgn & 1) ? -1.0 : 1.0) * cpow(0.25, t) * cbinom(l, t) * cbinom(l - t, am + t) *
                       cbinom(t, u) * cbinom(am, w);
            }
    return pref * norm * sum;
}

template <int L, int S, int C>
struct C2s {
    static constexpr double value = c2s_coef(L, S, C);
};

}  // namespace isdf
