// Device-side evaluation of one contracted spherical shell at one point.
//
// Restates cpp/src/ao_eval.cpp:207-249 (mikovtun/mp_isdf): radial sum over
// primitives, its derivative with respect to r^2, cartesian monomials in
// libcint order (cpp/src/ao_eval.cpp:30-44) contracted with the cartesian ->
// spherical table, gradient = R * d(poly) + 2 x R' * poly.
#pragma once

#include "isdf_internal.h"

namespace isdf {

__host__ __device__ constexpr int c2s_table_offset(int l) {
    int off = 0;
    for (int i = 0; i < l; ++i) off += (2 * i + 1) * (i + 1) * (i + 2) / 2;
    return off;
}
constexpr int kC2sTableSize = c2s_table_offset(kMaxL + 1);

template <int L>
struct CartOrder {
    static constexpr int nc = (L + 1) * (L + 2) / 2;
    static __host__ __device__ constexpr int lx(int c) {
        int x = L;
        while (c >= L - x + 1) { c -= L - x + 1; --x; }
        return x;
    }
    static __host__ __device__ constexpr int lz(int c) {
        int x = L;
        while (c >= L - x + 1) { c -= L - x + 1; --x; }
        return c;
    }
};

__device__ __forceinline__ double ao_exp(double x) { return exp(x); }
__device__ __forceinline__ float ao_exp(float x) { return __expf(x); }

// `sink.put<C>(ao, v)` receives component C (0 value, 1..3 d/dx, d/dy, d/dz)
// of AO index `ao`; `sink.wants(ao_first, ao_last)` may skip whole
// contraction groups.
template <class T, int L, bool GRAD, class Sink>
__device__ __forceinline__ void eval_shell_t(const ShellDesc& b, double dxd, double dyd, double dzd,
                                             const T* __restrict__ exps, const T* __restrict__ coefs,
                                             const T* __restrict__ c2s, Sink& sink) {
    constexpr int NC = CartOrder<L>::nc;
    constexpr int NS = 2 * L + 1;
    constexpr int OFF = c2s_table_offset(L);
    const T x = static_cast<T>(dxd), y = static_cast<T>(dyd), z = static_cast<T>(dzd);
    const T r2 = static_cast<T>(dxd * dxd + dyd * dyd + dzd * dzd);
    T px[L + 1], py[L + 1], pz[L + 1];
    px[0] = py[0] = pz[0] = T(1);
#pragma unroll
    for (int i = 1; i <= L; ++i) { px[i] = px[i - 1] * x; py[i] = py[i - 1] * y; pz[i] = pz[i - 1] * z; }
    T v[NS], vx[NS], vy[NS], vz[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) { v[s] = vx[s] = vy[s] = vz[s] = T(0); }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const int ax = CartOrder<L>::lx(c), az = CartOrder<L>::lz(c), ay = L - ax - az;
        const T m = px[ax] * py[ay] * pz[az];
        T mx = T(0), my = T(0), mz = T(0);
        if (GRAD) {
            if (ax) mx = T(ax) * px[ax - 1] * py[ay] * pz[az];
            if (ay) my = T(ay) * px[ax] * py[ay - 1] * pz[az];
            if (az) mz = T(az) * px[ax] * py[ay] * pz[az - 1];
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const T t = c2s[OFF + s * NC + c];
            v[s] += t * m;
            if (GRAD) { vx[s] += t * mx; vy[s] += t * my; vz[s] += t * mz; }
        }
    }
    for (int g0 = 0; g0 < b.nctr; g0 += kMaxCtrGroup) {
        const int ng = min(kMaxCtrGroup, b.nctr - g0);
        if (!sink.wants(b.ao_off + g0 * NS, b.ao_off + (g0 + ng) * NS)) continue;
        T R[kMaxCtrGroup], Rp[kMaxCtrGroup];
#pragma unroll
        for (int j = 0; j < kMaxCtrGroup; ++j) { R[j] = T(0); Rp[j] = T(0); }
        for (int p = 0; p < b.nprim; ++p) {
            const T a = exps[b.prim_off + p];
            const T arg = a * r2;
            if (arg > T(kExpCut)) continue;
            const T e = ao_exp(-arg);
#pragma unroll
            for (int j = 0; j < kMaxCtrGroup; ++j)
                if (j < ng) {
                    const T cc = coefs[b.coef_off + (g0 + j) * b.nprim + p] * e;
                    R[j] += cc;
                    if (GRAD) Rp[j] -= a * cc;
                }
        }
#pragma unroll
        for (int j = 0; j < kMaxCtrGroup; ++j)
            if (j < ng) {
                const int ao0 = b.ao_off + (g0 + j) * NS;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    sink.template put<0>(ao0 + s, R[j] * v[s]);
                    if (GRAD) {
                        const T two_rp = T(2) * Rp[j] * v[s];
                        sink.template put<1>(ao0 + s, R[j] * vx[s] + x * two_rp);
                        sink.template put<2>(ao0 + s, R[j] * vy[s] + y * two_rp);
                        sink.template put<3>(ao0 + s, R[j] * vz[s] + z * two_rp);
                    }
                }
            }
    }
}

template <class T, bool GRAD, class Sink>
__device__ __forceinline__ void eval_shell_any(const ShellDesc& b, double dx, double dy, double dz,
                                               const T* exps, const T* coefs, const T* c2s,
                                               Sink& sink) {
    switch (b.l) {
    case 0: eval_shell_t<T, 0, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    case 1: eval_shell_t<T, 1, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    case 2: eval_shell_t<T, 2, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    case 3: eval_shell_t<T, 3, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    case 4: eval_shell_t<T, 4, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    case 5: eval_shell_t<T, 5, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    default: eval_shell_t<T, 6, GRAD>(b, dx, dy, dz, exps, coefs, c2s, sink); break;
    }
}

}  // namespace isdf
