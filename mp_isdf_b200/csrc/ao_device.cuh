// Device-side evaluation of one contracted spherical shell at one point.
//
// Restates cpp/src/ao_eval.cpp:207-249 (mikovtun/mp_isdf): radial sum over
// primitives, its derivative with respect to r^2, cartesian monomials in
// libcint order (cpp/src/ao_eval.cpp:30-44) contracted with the cartesian ->
// spherical coefficients, gradient = R * d(poly) + 2 x R' * poly.  The
// coefficients are compile-time constants (c2s_table.h): the unrolled code
// multiplies only by the nonzero ones.
#pragma once

#include "c2s_table.h"
#include "isdf_internal.h"

#include <type_traits>

namespace isdf {

template <int B, int E, class F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

__device__ __forceinline__ double ao_exp(double x) { return exp(x); }
__device__ __forceinline__ float ao_exp(float x) { return __expf(x); }

// Spherical polynomial values (and cartesian derivatives) of angular
// momentum L at the offset (x, y, z).
template <class T, int L, bool GRAD>
struct SphPoly {
    static constexpr int NS = 2 * L + 1;
    T v[NS], vx[GRAD ? NS : 1], vy[GRAD ? NS : 1], vz[GRAD ? NS : 1];
    __device__ __forceinline__ SphPoly(T x, T y, T z) {
        constexpr int NC = (L + 1) * (L + 2) / 2;
        T px[L + 1], py[L + 1], pz[L + 1];
        px[0] = py[0] = pz[0] = T(1);
#pragma unroll
        for (int i = 1; i <= L; ++i) { px[i] = px[i - 1] * x; py[i] = py[i - 1] * y; pz[i] = pz[i - 1] * z; }
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            v[s] = T(0);
            if constexpr (GRAD) { vx[s] = T(0); vy[s] = T(0); vz[s] = T(0); }
        }
        static_for<0, NC>([&](auto ci) {
            constexpr int c = decltype(ci)::value;
            constexpr int ax = c2s_detail::cart_lx(L, c), az = c2s_detail::cart_lz(L, c);
            constexpr int ay = L - ax - az;
            const T m = px[ax] * py[ay] * pz[az];
            [[maybe_unused]] T mx = T(0), my = T(0), mz = T(0);
            if constexpr (GRAD) {
                if constexpr (ax > 0) mx = T(ax) * px[ax > 0 ? ax - 1 : 0] * py[ay] * pz[az];
                if constexpr (ay > 0) my = T(ay) * px[ax] * py[ay > 0 ? ay - 1 : 0] * pz[az];
                if constexpr (az > 0) mz = T(az) * px[ax] * py[ay] * pz[az > 0 ? az - 1 : 0];
            }
            static_for<0, NS>([&](auto si) {
                constexpr int s = decltype(si)::value;
                constexpr double t = C2s<L, s, c>::value;
                if constexpr (t != 0.0) {
                    v[s] += T(t) * m;
                    if constexpr (GRAD) {
                        if constexpr (ax > 0) vx[s] += T(t) * mx;
                        if constexpr (ay > 0) vy[s] += T(t) * my;
                        if constexpr (az > 0) vz[s] += T(t) * mz;
                    }
                }
            });
        });
    }
};

// Contractions [g0, g0 + ng) of shell b (ng <= NG): radial sums over the
// primitives, then every component of every spherical function.
template <class T, int L, bool GRAD, int NG, class Sink>
__device__ __forceinline__ void eval_shell_group(const ShellDesc& b, const SphPoly<T, L, GRAD>& poly, T x, T y,
                                                 T z, T r2, const T* __restrict__ exps,
                                                 const T* __restrict__ coefs, Sink& sink, int g0, int ng) {
    constexpr int NS = 2 * L + 1;
    T R[NG], Rp[NG];
#pragma unroll
    for (int j = 0; j < NG; ++j) { R[j] = T(0); Rp[j] = T(0); }
    for (int p = 0; p < b.nprim; ++p) {
        const T a = exps[b.prim_off + p];
        const T arg = a * r2;
        if (arg > T(kExpCut)) continue;
        const T e = ao_exp(-arg);
#pragma unroll
        for (int j = 0; j < NG; ++j)
            if (NG == 1 || j < ng) {
                const T cc = coefs[b.coef_off + (g0 + j) * b.nprim + p] * e;
                R[j] += cc;
                if constexpr (GRAD) Rp[j] -= a * cc;
            }
    }
#pragma unroll
    for (int j = 0; j < NG; ++j)
        if (NG == 1 || j < ng) {
            const int ao0 = b.ao_off + (g0 + j) * NS;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                sink.template put<0>(ao0 + s, R[j] * poly.v[s]);
                if constexpr (GRAD) {
                    const T two_rp = T(2) * Rp[j] * poly.v[s];
                    sink.template put<1>(ao0 + s, R[j] * poly.vx[s] + x * two_rp);
                    sink.template put<2>(ao0 + s, R[j] * poly.vy[s] + y * two_rp);
                    sink.template put<3>(ao0 + s, R[j] * poly.vz[s] + z * two_rp);
                }
            }
        }
}

// `sink.put<C>(ao, v)` receives component C (0 value, 1..3 d/dx, d/dy, d/dz)
// of AO index `ao` for the contractions [ctr0, ctr1) of shell b, given the
// offset (x, y, z) from the shell centre and r2 = |offset|^2.  A single
// contraction (the common case) takes a path without a group's unused lanes.
template <class T, int L, bool GRAD, class Sink>
__device__ __forceinline__ void eval_shell_core(const ShellDesc& b, T x, T y, T z, T r2,
                                                const T* __restrict__ exps, const T* __restrict__ coefs,
                                                Sink& sink, int ctr0, int ctr1) {
    const SphPoly<T, L, GRAD> poly(x, y, z);
    const int cend = min(b.nctr, ctr1);
    if (cend - ctr0 == 1) {
        eval_shell_group<T, L, GRAD, 1>(b, poly, x, y, z, r2, exps, coefs, sink, ctr0, 1);
        return;
    }
    for (int g0 = ctr0; g0 < cend; g0 += kMaxCtrGroup)
        eval_shell_group<T, L, GRAD, kMaxCtrGroup>(b, poly, x, y, z, r2, exps, coefs, sink, g0,
                                                   min(kMaxCtrGroup, cend - g0));
}

// Runtime dispatch on l up to LMAX (at least the context's largest angular
// momentum; shells above LMAX are not evaluated), offset and r2 in T.
template <class T, bool GRAD, int LMAX = kMaxL, class Sink>
__device__ __forceinline__ void eval_shell_rel(const ShellDesc& b, T x, T y, T z, T r2, const T* exps,
                                               const T* coefs, Sink& sink, int ctr0 = 0,
                                               int ctr1 = 1 << 30) {
    switch (b.l) {
    case 0: eval_shell_core<T, 0, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    case 1: if constexpr (LMAX >= 1) eval_shell_core<T, 1, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    case 2: if constexpr (LMAX >= 2) eval_shell_core<T, 2, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    case 3: if constexpr (LMAX >= 3) eval_shell_core<T, 3, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    case 4: if constexpr (LMAX >= 4) eval_shell_core<T, 4, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    case 5: if constexpr (LMAX >= 5) eval_shell_core<T, 5, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    default: if constexpr (LMAX >= 6) eval_shell_core<T, 6, GRAD>(b, x, y, z, r2, exps, coefs, sink, ctr0, ctr1); break;
    }
}

// ---- packed pieces -------------------------------------------------------------------
// A piece's primitives come as one record (alpha, c_j, c_j+1, c_j+2) per
// primitive and group of three contractions -- one float4 (FP32 table) or two
// double2 (FP64 table) -- so one or two 16-byte loads feed the exponential
// and up to three radial sums.  `sink.put<C>(ao, v)` receives the AO index
// relative to the piece's first AO.
template <class T> struct PackedPrim;
template <> struct PackedPrim<float> {
    using rec = float4;
    static __device__ __forceinline__ void load(const float4* __restrict__ pr, int p, float& a, float (&c)[3]) {
        const float4 q = __ldg(pr + p);
        a = q.x; c[0] = q.y; c[1] = q.z; c[2] = q.w;
    }
};
template <> struct PackedPrim<double> {
    using rec = double2;   // two per primitive
    static __device__ __forceinline__ void load(const double2* __restrict__ pr, int p, double& a, double (&c)[3]) {
        const double2 u = __ldg(pr + 2 * p), v = __ldg(pr + 2 * p + 1);
        a = u.x; c[0] = u.y; c[1] = v.x; c[2] = v.y;
    }
};

template <class T, int L, bool GRAD, int NG, class Sink>
__device__ __forceinline__ void eval_piece_group(const SphPoly<T, L, GRAD>& poly, T x, T y, T z, T r2,
                                                 const typename PackedPrim<T>::rec* __restrict__ pr, int nprim,
                                                 int ng, int ao_rel0, Sink& sink) {
    constexpr int NS = 2 * L + 1;
    T R[NG], Rp[NG];
#pragma unroll
    for (int j = 0; j < NG; ++j) { R[j] = T(0); Rp[j] = T(0); }
    // several primitives' loads and exponentials in flight (FP64 exp is a
    // long dependent chain)
#pragma unroll(sizeof(T) == 8 ? 4 : 2)
    for (int p = 0; p < nprim; ++p) {
        T a, cc[3];
        PackedPrim<T>::load(pr, p, a, cc);
        const T arg = a * r2;
        if (arg > static_cast<T>(kExpCut)) continue;
        const T e = ao_exp(-arg);
#pragma unroll
        for (int j = 0; j < NG; ++j) {
            const T c = cc[j] * e;
            R[j] += c;
            if constexpr (GRAD) Rp[j] -= a * c;
        }
    }
#pragma unroll
    for (int j = 0; j < NG; ++j)
        if (NG == 1 || j < ng) {
            const int ao0 = ao_rel0 + j * NS;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                sink.template put<0>(ao0 + s, R[j] * poly.v[s]);
                if constexpr (GRAD) {
                    const T two_rp = T(2) * Rp[j] * poly.v[s];
                    sink.template put<1>(ao0 + s, R[j] * poly.vx[s] + x * two_rp);
                    sink.template put<2>(ao0 + s, R[j] * poly.vy[s] + y * two_rp);
                    sink.template put<3>(ao0 + s, R[j] * poly.vz[s] + z * two_rp);
                }
            }
        }
}

template <class T, int L, bool GRAD, class Sink>
__device__ __forceinline__ void eval_piece_core(T x, T y, T z, T r2, const typename PackedPrim<T>::rec* __restrict__ pr,
                                                int nprim, int nc, Sink& sink) {
    const SphPoly<T, L, GRAD> poly(x, y, z);
    if (nc == 1) {
        eval_piece_group<T, L, GRAD, 1>(poly, x, y, z, r2, pr, nprim, 1, 0, sink);
        return;
    }
    constexpr int kRecs = sizeof(T) == 8 ? 2 : 1;   // records per primitive
    for (int g0 = 0; g0 < nc; g0 += 3, pr += kRecs * nprim)
        eval_piece_group<T, L, GRAD, 3>(poly, x, y, z, r2, pr, nprim, min(3, nc - g0), g0 * (2 * L + 1), sink);
}

template <class T, bool GRAD, int LMAX, class Sink>
__device__ __forceinline__ void eval_piece(int l, T x, T y, T z, T r2, const typename PackedPrim<T>::rec* pr,
                                           int nprim, int nc, Sink& sink) {
    switch (l) {
    case 0: eval_piece_core<T, 0, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    case 1: if constexpr (LMAX >= 1) eval_piece_core<T, 1, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    case 2: if constexpr (LMAX >= 2) eval_piece_core<T, 2, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    case 3: if constexpr (LMAX >= 3) eval_piece_core<T, 3, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    case 4: if constexpr (LMAX >= 4) eval_piece_core<T, 4, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    case 5: if constexpr (LMAX >= 5) eval_piece_core<T, 5, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    default: if constexpr (LMAX >= 6) eval_piece_core<T, 6, GRAD>(x, y, z, r2, pr, nprim, nc, sink); break;
    }
}

// Same, from FP64 offsets: r2 is formed in FP64 and rounded once to T.
template <class T, bool GRAD, int LMAX = kMaxL, class Sink>
__device__ __forceinline__ void eval_shell_any(const ShellDesc& b, double dx, double dy, double dz,
                                               const T* exps, const T* coefs, Sink& sink,
                                               int ctr0 = 0, int ctr1 = 1 << 30) {
    eval_shell_rel<T, GRAD, LMAX>(b, static_cast<T>(dx), static_cast<T>(dy), static_cast<T>(dz),
                                  static_cast<T>(dx * dx + dy * dy + dz * dz), exps, coefs, sink, ctr0, ctr1);
}

}  // namespace isdf
