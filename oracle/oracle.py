"""CPU oracle for the ISDF hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker.  The product package (``mp_isdf_b200``) never
imports it and has no CPU fallback.

It restates the reference (mikovtun/mp_isdf) algorithm for the path:

* AO values / gradients and axis features: the C++ restatement in
  ``oracle/isdf_oracle.cpp`` (``cpp/src/ao_eval.cpp:205-250``,
  ``cpp/include/anchor_select_impl.hpp:51-79``);
* cartesian -> real-spherical matrices: derived here by least squares against
  real spherical harmonics built from scipy's associated Legendre functions
  (independently of the product's closed-form derivation); libcint's
  ``CINTc2s_bra_sph`` is not vendored, so its convention is restated as: p in
  (x, y, z) order scaled by sqrt(3/4pi), s by 1/sqrt(4pi)
  (``cpp/src/ao_eval.cpp:132-138``), l >= 2 as r^l Y_lm, m = -l..l, unit-sphere
  normalised, without the Condon-Shortley phase;
* qrcp_dense: explicit weighted pair matrix + LAPACK ``dgeqp3`` via scipy
  (``cpp/src/anchor_select_qrcp.cpp:248-307``);
* rand_sketch quadrature: U/V from ``std::mt19937_64`` +
  ``std::normal_distribution`` (C++), ``dgeqp3`` of the sketch, tail / rank
  logic (``cpp/src/anchor_select_randomized_id.cpp:92-374``);
* multi-axis scaling (``cpp/src/anchor_select.cpp:426-480``);
* the fit ``_physical_pair_refit`` and the pair-space error functions
  (``python/isdf.py:154-191, 238-263``), literally for small grids and in
  Gram form for large ones;
* the FP64 nuclear gradient of E = sum_g w_g rho_ISDF(g)^2 assembled from AO
  values and their dx/dy/dz derivatives.

Parity pinning: see tests/test_oracle.py (known answers of the reference's
own tests).  The reference itself cannot be built here, and PySCF is absent,
so AO values are pinned by orthonormality and derivative consistency only.
"""
from __future__ import annotations

import ctypes
import os
from math import factorial, pi, sqrt
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libisdf_oracle.so"
LMAX = 6

_lib = None


def build(force=False):
    """Compile the C++ restatement (g++ -O2 -fopenmp)."""
    src = HERE / "isdf_oracle.cpp"
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    import subprocess
    tmp = LIB_PATH.with_suffix(".so.tmp")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
                           str(src), "-o", str(tmp)])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        L.oracle_ctx_create.restype = P
        L.oracle_ctx_create.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P,
                                        ctypes.c_longlong, P, ctypes.c_int]
        L.oracle_ctx_destroy.argtypes = [P]
        L.oracle_ctx_nao.argtypes = [P]
        L.oracle_ctx_nao.restype = ctypes.c_int
        L.oracle_ao_atoms.argtypes = [P, P]
        L.oracle_eval_ao.argtypes = [P, P, ctypes.c_longlong, ctypes.c_int, P]
        L.oracle_axis_features.argtypes = [P, P, ctypes.c_longlong, P, ctypes.c_int, P, P]
        L.oracle_axis_norms_hypot.argtypes = [P, P, P, ctypes.c_longlong, P, ctypes.c_int, P]
        L.oracle_axis_norms_hypot.restype = ctypes.c_int
        L.oracle_axis_norms_sq.argtypes = [P, P, P, ctypes.c_longlong, P, ctypes.c_int, P]
        L.oracle_sketch_factors.argtypes = [ctypes.c_longlong, ctypes.c_longlong,
                                            ctypes.c_uint64, P, P]
        L.oracle_sketch.argtypes = [P, P, P, ctypes.c_longlong, P, ctypes.c_int, P, P, P,
                                    ctypes.c_longlong, P]
        L.oracle_grid_gram.argtypes = [P, P, ctypes.c_longlong, P, ctypes.c_longlong, P, P]
        L.oracle_fit_apply.argtypes = [ctypes.c_longlong, ctypes.c_longlong] + [P] * 9
        L.oracle_rng_new.restype = P
        L.oracle_rng_new.argtypes = [ctypes.c_uint64]
        L.oracle_rng_free.argtypes = [P]
        L.oracle_rng_discrete.restype = ctypes.c_longlong
        L.oracle_rng_discrete.argtypes = [P, P, ctypes.c_longlong]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------
# cartesian -> spherical
# ---------------------------------------------------------------------------
def cart_powers(l):
    """libcint cartesian order (``cpp/src/ao_eval.cpp:30-44``)."""
    out = []
    for lx in range(l, -1, -1):
        for lz in range(0, l - lx + 1):
            out.append((lx, l - lx - lz, lz))
    return out


def real_harmonics(l, pts):
    """Real unit-sphere-normalised Y_lm (m=-l..l), no Condon-Shortley phase."""
    from scipy.special import lpmv
    x, y, z = pts.T
    theta = np.arccos(np.clip(z, -1, 1))
    phi = np.arctan2(y, x)
    out = []
    for m in range(-l, l + 1):
        am = abs(m)
        norm = sqrt((2 * l + 1) / (4 * pi) * factorial(l - am) / factorial(l + am))
        leg = lpmv(am, l, np.cos(theta)) * (-1) ** am      # drop the CS phase
        if m == 0:
            out.append(norm * leg)
        elif m > 0:
            out.append(sqrt(2) * norm * leg * np.cos(am * phi))
        else:
            out.append(sqrt(2) * norm * leg * np.sin(am * phi))
    return np.array(out)


def c2s_matrix(l):
    """nsph x ncart matrix T with sum_c T[s,c] x^lx y^ly z^lz = r^l Y_ls."""
    if l == 0:
        return np.array([[1.0 / sqrt(4 * pi)]])
    if l == 1:
        return np.eye(3) * sqrt(3.0 / (4 * pi))
    rng = np.random.default_rng(1000 + l)
    pts = rng.normal(size=(8 * (l + 1) ** 2 + 64, 3))
    pts /= np.linalg.norm(pts, axis=1)[:, None]
    mono = np.array([pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c
                     for a, b, c in cart_powers(l)])            # [ncart, npts]
    target = real_harmonics(l, pts)                            # [nsph, npts]
    t, *_ = np.linalg.lstsq(mono.T, target.T, rcond=None)
    t = t.T
    t[np.abs(t) < 1e-13] = 0.0
    return t


def c2s_table(lmax=LMAX):
    return np.concatenate([c2s_matrix(l).ravel() for l in range(lmax + 1)])


_C2S = None


# ---------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------
class OracleContext:
    def __init__(self, atm, bas, env):
        global _C2S
        if _C2S is None:
            _C2S = np.ascontiguousarray(c2s_table(LMAX))
        self.atm = np.ascontiguousarray(atm, dtype=np.int32)
        self.bas = np.ascontiguousarray(bas, dtype=np.int32)
        self.env = np.ascontiguousarray(env, dtype=np.float64)
        L = lib()
        self.h = L.oracle_ctx_create(_p(self.atm), len(self.atm), _p(self.bas), len(self.bas),
                                     _p(self.env), len(self.env), _p(_C2S), LMAX)
        if not self.h:
            raise ValueError(L.oracle_last_error().decode())
        self.nao = L.oracle_ctx_nao(self.h)
        self.natm = len(self.atm)
        self.ao_atom = np.empty(self.nao, dtype=np.int32)
        L.oracle_ao_atoms(self.h, _p(self.ao_atom))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_ctx_destroy(self.h)
            self.h = None

    def eval_ao(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        out = np.empty((len(pts), self.nao))
        lib().oracle_eval_ao(self.h, _p(pts), len(pts), 0, _p(out))
        return out

    def eval_ao_gradient(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        out = np.empty((3, len(pts), self.nao))
        lib().oracle_eval_ao(self.h, _p(pts), len(pts), 1, _p(out))
        return out

    def axis_features(self, pts, axes, scales=None):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        ax = np.ascontiguousarray(axes, dtype=np.int32)
        sc = None if scales is None else np.ascontiguousarray(scales, dtype=np.float64)
        out = np.empty((len(pts), len(ax) * self.nao))
        lib().oracle_axis_features(self.h, _p(pts), len(pts), _p(ax), len(ax),
                                   None if sc is None else _p(sc), _p(out))
        return out

    def axis_norms(self, pts, w, axes, exact_order=True):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, dtype=np.float64)
        ax = np.ascontiguousarray(axes, dtype=np.int32)
        out = np.zeros(len(ax))
        if exact_order:
            rc = lib().oracle_axis_norms_hypot(self.h, _p(pts), _p(w), len(pts), _p(ax),
                                               len(ax), _p(out))
            if rc < 0:
                raise ValueError(lib().oracle_last_error().decode())
            return out, bool(rc)
        lib().oracle_axis_norms_sq(self.h, _p(pts), _p(w), len(pts), _p(ax), len(ax), _p(out))
        return out, bool(np.any(w != 0))

    def sketch(self, pts, w, axes, scales, u, v, ell):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, dtype=np.float64)
        ax = np.ascontiguousarray(axes, dtype=np.int32)
        sc = np.ascontiguousarray(scales if scales is not None else np.ones(len(ax)))
        y = np.empty((len(pts), ell))
        lib().oracle_sketch(self.h, _p(pts), _p(w), len(pts), _p(ax), len(ax), _p(sc),
                            _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)), ell, _p(y))
        return y

    def grid_gram(self, pts, anchor_ao):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        a = np.ascontiguousarray(anchor_ao, dtype=np.float64)
        G = np.empty((len(pts), len(a)))
        q = np.empty(len(pts))
        lib().oracle_grid_gram(self.h, _p(pts), len(pts), _p(a), len(a), _p(G), _p(q))
        return G, q


AXIS_CODES = {"ao": 0, "dx": 1, "dy": 2, "dz": 3}


def sketch_factors(d, ell, seed):
    u = np.empty(d * ell)
    v = np.empty(d * ell)
    lib().oracle_sketch_factors(d, ell, np.uint64(seed), _p(u), _p(v))
    return u.reshape(d, ell), v.reshape(d, ell)


# ---------------------------------------------------------------------------
# selection (cpp/src/anchor_select.cpp:426-505)
# ---------------------------------------------------------------------------
def axis_scales(ctx, pts, w, axes, axis_weights=None, exact_order=True):
    """Global Frobenius scales for >1 axes (``cpp/src/anchor_select.cpp:437-480``)."""
    if len(axes) <= 1:
        return None
    norms, any_eligible = ctx.axis_norms(pts, w, axes, exact_order=exact_order)
    if not any_eligible:
        return np.array([])
    if np.any(~(norms > 0)) or not np.all(np.isfinite(norms)):
        raise ValueError("axis Frobenius norm must be finite and positive")
    factors = np.ones(len(axes)) if not axis_weights else np.asarray(axis_weights, float)
    return factors / norms


def occ_features(ctx, pts, axes, mo_coeff=None, nocc=0, scales=None):
    """Concatenated axis features with OccupiedOrbital entries (code 4)
    (``cpp/src/anchor_select.cpp:18-52``, ``anchor_select_impl.hpp:55-77``):
    AO values (0), gradients (1..3), and psi_j = sum_mu phi_mu C[mu][j],
    j < nocc (4), each block times its scale."""
    if 4 in list(axes) and (mo_coeff is None or not 1 <= nocc <= ctx.nao):
        raise ValueError("OccupiedOrbital requires row-major (nao,nao) RHF mo_coeff and 1 <= nocc <= nao")
    ao = ctx.eval_ao(pts)
    grad = ctx.eval_ao_gradient(pts) if any(a in (1, 2, 3) for a in axes) else None
    blocks = []
    for i, a in enumerate(axes):
        if a == 0:
            b = ao
        elif a == 4:
            b = ao @ np.asarray(mo_coeff, float)[:, :nocc]
        else:
            b = grad[a - 1]
        blocks.append(b * (1.0 if scales is None else scales[i]))
    return np.hstack(blocks)


def occ_axis_scales(ctx, pts, w, axes, mo_coeff, nocc, axis_weights=None):
    """Global Frobenius scales (``cpp/src/anchor_select.cpp:437-480``) over the
    nonzero-weight points, with occupied-orbital entries."""
    if len(axes) <= 1:
        return None
    keep = np.asarray(w, float) != 0
    f = occ_features(ctx, pts[keep], axes, mo_coeff, nocc)
    widths = [nocc if a == 4 else ctx.nao for a in axes]
    edges = np.cumsum([0] + widths)
    norms = np.array([np.linalg.norm(f[:, edges[i]:edges[i + 1]]) for i in range(len(axes))])
    factors = np.ones(len(axes)) if not axis_weights else np.asarray(axis_weights, float)
    return factors / norms


def select_qrcp_dense_features(f, keep, tolerance=1e-10, max_rank=0, w=None):
    """qrcp_dense (dgeqp3 of the explicit pair matrix) over given features of the
    kept points; returns original indices."""
    from scipy.linalg import qr
    A = pair_matrix(f, w)
    m, n = A.shape
    _, r, piv = qr(A, pivoting=True, mode="economic")
    cap = min(m, n, max_rank if max_rank else min(m, n))
    diag = np.abs(np.diag(r))
    first = diag[0] if cap else 0.0
    out = []
    for i in range(cap):
        if first == 0 or diag[i] <= tolerance * first:
            break
        out.append(int(keep[piv[i]]))
    return out


def select_rand_sketch_features(f, keep, w, ell, oversampling, seed, tolerance=1e-10, max_rank=0):
    """Quadrature sketch + dgeqp3 + rank rule over given (scaled) features."""
    d = f.shape[1]
    u, v = sketch_factors(d, ell, seed)
    y = (np.sqrt(np.abs(w)) / np.sqrt(ell))[:, None] * (f @ u) * (f @ v)
    pos, _ = sketch_qr_rank(y, ell, oversampling, tolerance, max_rank, d * (d + 1) // 2)
    return [int(keep[p]) for p in pos]


def pair_matrix(features, w):
    """A[:, g] = sqrt|w_g| f_g (x) f_g (``cpp/src/anchor_select_qrcp.cpp:253-267``)."""
    outer = np.einsum("gi,gj->gij", features, features).reshape(len(features), -1)
    return (outer * np.sqrt(np.abs(w))[:, None]).T


def select_qrcp_dense(ctx, pts, w, axes, tolerance=1e-10, max_rank=0, scales=None):
    """qrcp_dense via scipy/LAPACK dgeqp3 (``anchor_select_qrcp.cpp:178-307``)."""
    from scipy.linalg import qr
    w = np.asarray(w, float)
    keep = np.flatnonzero(w != 0)
    if len(keep) == 0:
        return []
    f = ctx.axis_features(pts[keep], axes, scales)
    A = pair_matrix(f, w[keep])
    m, n = A.shape
    _, r, piv = qr(A, pivoting=True, mode="economic")
    cap = min(m, n, max_rank if max_rank else min(m, n))
    diag = np.abs(np.diag(r))
    first = diag[0] if cap else 0.0
    out = []
    for i in range(cap):
        if first == 0 or diag[i] <= tolerance * first:
            break
        out.append(int(keep[piv[i]]))
    return out


def _top_two(res, chosen):
    """First index of the largest residual norm among unchosen columns, its
    norm, and the relative gap to the runner-up: (p, r_top, gap)."""
    r = np.where(chosen, -np.inf, res)
    p = int(np.argmax(r))                      # first maximum, as idamax
    top = np.sqrt(max(r[p], 0.0))
    r[p] = -np.inf
    second = np.sqrt(max(np.max(r), 0.0)) if np.isfinite(np.max(r)) else 0.0
    return p, top, ((top - second) / top) if top > 0 else 0.0


def pair_qrcp_exact(features, w, steps, chunk=16384):
    """Truncated column-pivoted QR of the weighted pair columns
    a_g = sqrt|w_g| f_g (x) f_g with EXACT residual norms at every step.

    This is the greedy rule of LAPACK ``dgeqp3`` that qrcp_dense applies to the
    explicit d^2 x n pair matrix (``cpp/src/anchor_select_qrcp.cpp:172-223,
    248-307``) and the max-norm rule of the online selector
    (``cpp/src/anchor_select_online_qr.cpp:200-358``), for grids whose pair
    matrix is too large to form.  The orthonormal pair basis is kept as
    symmetric d x d matrices Q_j (Gram-Schmidt with one re-orthogonalisation),
    so q_j . a_g = sqrt|w_g| f_g^T Q_j f_g and the squared residual of column g
    after j steps is |a_g|^2 - sum_i (q_i . a_g)^2.

    Returns (positions, |R_jj|, gaps): gaps[j] is the relative difference of
    the two largest residual norms at step j -- the quantity that decides
    whether an implementation's pivot at that step is forced (gap > 1e-10) or
    a near tie.
    """
    F = np.ascontiguousarray(features, dtype=np.float64)
    n, d = F.shape
    sw = np.sqrt(np.abs(np.asarray(w, float)))
    norm2 = (sw * np.einsum("gi,gi->g", F, F)) ** 2
    coef = np.zeros((n, steps))
    chosen = np.zeros(n, bool)
    basis, pos, diag, gaps = [], [], [], []
    for j in range(min(steps, n)):
        res = norm2 - np.einsum("gj,gj->g", coef[:, :j], coef[:, :j])
        p, top, gap = _top_two(res, chosen)
        if top == 0:
            break
        pos.append(p)
        diag.append(top)
        gaps.append(gap)
        v = sw[p] * np.outer(F[p], F[p])
        for i, Q in enumerate(basis):
            v -= coef[p, i] * Q
        for Q in basis:                          # second Gram-Schmidt pass
            v -= np.sum(Q * v) * Q
        v /= np.linalg.norm(v)
        v = 0.5 * (v + v.T)
        basis.append(v)
        for s0 in range(0, n, chunk):
            Fc = F[s0:s0 + chunk]
            coef[s0:s0 + chunk, j] = sw[s0:s0 + chunk] * np.einsum("gi,gi->g", Fc @ v, Fc)
        chosen[p] = True
    return pos, np.array(diag), np.array(gaps)


def sketch_qrcp_exact(yt, steps):
    """Column-pivoted Householder QR of the sketch Y (``yt``: ell x n) with
    exact trailing column norms at every step: the pivot rule of ``dgeqp3``
    in ``cpp/src/anchor_select_randomized_id.cpp:320-374`` without its norm
    downdating.  Returns (positions, |R_jj|, gaps) as ``pair_qrcp_exact``."""
    A = np.array(yt, dtype=np.float64, copy=True)
    ell, n = A.shape
    chosen = np.zeros(n, bool)
    pos, diag, gaps = [], [], []
    for j in range(min(steps, ell, n)):
        sub = A[j:]
        p, top, gap = _top_two(np.einsum("ij,ij->j", sub, sub), chosen)
        if top == 0:
            break
        pos.append(p)
        diag.append(top)
        gaps.append(gap)
        x = sub[:, p].copy()
        alpha = -np.copysign(np.linalg.norm(x), x[0])
        x[0] -= alpha
        x /= np.linalg.norm(x)
        sub -= 2.0 * np.outer(x, x @ sub)
        chosen[p] = True
    return pos, np.array(diag), np.array(gaps)


def physical_fit_svd(phi_a):
    """SVD of the transposed anchor pair matrix C^T (nao^2 x k),
    C[k] = phi_a(k) (x) phi_a(k), with the cutoff s > 1e-12 s_0 of
    ``_physical_pair_refit`` (``python/isdf.py:238-263``): (U, s, Vt) of the
    retained singular triplets, and the condition number s_0 / s_last."""
    k, nao = phi_a.shape
    C = np.einsum("ki,kj->kij", phi_a, phi_a).reshape(k, nao * nao)
    u, s, vt = np.linalg.svd(C.T, full_matrices=False)
    keep = s > (1e-12 * s[0] if len(s) else 0)
    cond = float(s[0] / s[-1]) if len(s) and s[-1] > 0 else float("inf")
    return u[:, keep], s[keep], vt[keep], cond


def physical_fit_columns(u, s, vt, anchor_weights, phi_cols, chunk=512):
    """Theta columns of ``_physical_pair_refit`` (``python/isdf.py:238-263``),
    Theta_g = (V S^-1 U^T p_g) / w_anchor with p_g = phi_g (x) phi_g, for the
    given points' AO values; U^T p_g is formed as phi_g^T U_j phi_g per
    retained singular vector so that no nao^2-long pair vector is stored."""
    nao = phi_cols.shape[1]
    r = u.shape[1]
    ut_p = np.empty((r, len(phi_cols)))
    for j in range(r):
        Uj = u[:, j].reshape(nao, nao)
        for s0 in range(0, len(phi_cols), chunk):
            P = phi_cols[s0:s0 + chunk]
            ut_p[j, s0:s0 + chunk] = np.einsum("gi,gi->g", P @ Uj, P)
    return (vt.T @ (ut_p / s[:, None])) / np.asarray(anchor_weights, float)[:, None]


def physical_pair_error(ctx, coords, weights, phi_a, s, vt):
    """Pair-space error (``python/isdf.py:154-191``) of the SVD fit in Gram
    form over all given points: err^2 = sum_g |w_g| (q_g^2 - 2 X_g.h_g +
    X_g^T M X_g) with h_g = (Phi_a phi_g)^2, q_g = |phi_g|^2,
    X_g = V S^-2 V^T h_g (= Theta_g * w_anchor), M = (Phi_a Phi_a^T)^2.
    Returns {"l2", "relative", "err2", "exact2"}."""
    G, q = ctx.grid_gram(coords, phi_a)
    H = G * G
    T = (vt.T / s ** 2) @ vt
    M = (phi_a @ phi_a.T) ** 2
    X = H @ T
    aw = np.abs(np.asarray(weights, float))
    per = q * q - 2.0 * np.einsum("gk,gk->g", X, H) + np.einsum("gk,gk->g", X @ M, X)
    err2 = max(float(np.dot(aw, per)), 0.0)
    exact2 = float(np.dot(aw, q * q))
    return {"l2": np.sqrt(err2), "relative": np.sqrt(err2 / exact2) if exact2 else 0.0,
            "err2": err2, "exact2": exact2}


def sketch_qr_rank(y, ell, oversampling, tolerance, max_rank, physical_rank):
    """dgeqp3 of the sketch Y (y: [n, ell]) and the rank rule of
    ``anchor_select_randomized_id.cpp:320-374``: (positions 0..n-1, details)."""
    from scipy.linalg.lapack import dgeqp3
    n = len(y)
    ymat = np.asfortranarray(np.asarray(y, float).T)              # ell x n column-major
    qr_, jpvt, tau, work, info = dgeqp3(ymat)
    if info != 0:
        raise RuntimeError("dgeqp3 failed")
    steps = min(ell, n)
    energy = np.array([np.sum(qr_[i, i:] ** 2) for i in range(steps)])
    diag = np.abs(np.diag(qr_)[:steps])
    rank, tails, numerical_rank = sketch_rank_rules(diag, energy, ell, n, oversampling, tolerance, max_rank,
                                                    physical_rank)
    pos = [int(jpvt[i] - 1) for i in range(rank)]
    return pos, dict(jpvt=jpvt - 1, diag=diag, tails=tails, numerical_rank=numerical_rank)


def sketch_rank_rules(diag, energy, ell, n, oversampling, tolerance, max_rank, physical_rank):
    """Tails, numerical rank, cap and selected rank from the per-step |R_ii|
    and row energies of the sketch QR (``anchor_select_randomized_id.cpp:320-374``):
    (rank, tails, numerical_rank)."""
    steps = min(ell, n)
    diag = np.asarray(diag, float)[:steps]
    energy = np.asarray(energy, float)[:steps]
    tails = np.zeros(steps + 1)
    for i in range(steps - 1, -1, -1):
        tails[i] = np.hypot(tails[i + 1], np.sqrt(energy[i]))
    diag_max = diag.max() if steps else 0.0
    norm = tails[0]
    floor = np.finfo(float).eps * max(ell, n) * diag_max
    numerical_rank = steps
    for i in range(steps):
        if diag[i] <= floor:
            numerical_rank = i
            break
    cap = min(max_rank if max_rank else ell - oversampling, ell - oversampling, steps,
              physical_rank, numerical_rank)
    if max_rank and numerical_rank < max_rank:
        raise ValueError("requested anchor_rank exceeds the numerical rank of the randomized sketch")
    rank = max_rank if max_rank else cap
    if not max_rank:
        for i in range(cap + 1):
            if tails[i] <= tolerance * norm:
                rank = i
                break
    return rank, tails, numerical_rank


def select_rand_sketch(ctx, pts, w, axes, tolerance=1e-10, max_rank=0, sketch_size=128,
                       oversampling=16, seed=7, scales=None, return_details=False):
    """Quadrature Khatri-Rao sketch + dgeqp3 (``anchor_select_randomized_id.cpp``)."""
    if oversampling == 0 or (not max_rank and sketch_size <= oversampling):
        raise ValueError("invalid randomized ID grid, tolerance, batch, sketch or rank/oversampling")
    w = np.asarray(w, float)
    keep = np.flatnonzero(w != 0)
    d = len(axes) * ctx.nao
    ell = max_rank + oversampling if max_rank else sketch_size
    n = len(keep)
    if n == 0:
        return ([], {}) if return_details else []
    physical_rank = d * (d + 1) // 2
    if max_rank > min(n, physical_rank):
        raise ValueError("requested anchor_rank exceeds eligible candidates or physical pair rank")
    u, v = sketch_factors(d, ell, seed)
    y = ctx.sketch(pts[keep], w[keep], axes, scales, u, v, ell)   # [n, ell]
    pos, det = sketch_qr_rank(y, ell, oversampling, tolerance, max_rank, physical_rank)
    jpvt, diag, tails, numerical_rank = det["jpvt"] + 1, det["diag"], det["tails"], det["numerical_rank"]
    rank = len(pos)
    piv = [int(keep[jpvt[i] - 1]) for i in range(rank)]
    if return_details:
        return piv, dict(y=y, diag=diag, tails=tails, numerical_rank=numerical_rank,
                         jpvt=jpvt - 1, u=u, v=v, keep=keep)
    return piv


def select_density_sketch(ctx, pts, w, importance, normalized=False, tolerance=1e-10, max_rank=0,
                          sketch_size=128, oversampling=16, seed=7, ao_screening_threshold=1e-24,
                          return_details=False):
    """AO-density Khatri-Rao sketch + dgeqp3 (``anchor_select_randomized_id.cpp:104-118,
    131-146, 231-309``): candidates are the points with w != 0 and importance m != 0
    whose squared AO norm q exceeds the screening threshold; column g of the
    sketch is sqrt(m_g)/sqrt(ell) (f.u_s)(f.v_s) with f = phi_g, or phi_g/sqrt(q_g)
    in the normalized (``density_col_norm``) form.  Only the AO axis."""
    w = np.asarray(w, float)
    importance = np.asarray(importance, float)
    if importance.shape != (len(pts),):
        raise ValueError("point_importance must have shape (ngrid,)")
    if not np.isfinite(importance).all() or np.any(importance < 0):
        raise ValueError("point_importance must be finite and nonnegative")
    if not np.isfinite(ao_screening_threshold) or ao_screening_threshold < 0:
        raise ValueError("AO screening threshold must be finite and nonnegative")
    if oversampling == 0 or (not max_rank and sketch_size <= oversampling):
        raise ValueError("invalid randomized ID grid, tolerance, batch, sketch or rank/oversampling")
    keep = np.flatnonzero((w != 0) & (importance != 0))
    if len(keep) == 0:
        if max_rank:
            raise ValueError("requested anchor_rank exceeds eligible candidates")
        return ([], {}) if return_details else []
    d = ctx.nao
    ell = max_rank + oversampling if max_rank else sketch_size
    ao = ctx.eval_ao(pts[keep])
    q = np.einsum("ga,ga->g", ao, ao)
    if not np.isfinite(q).all():
        raise OverflowError("non-finite AO squared norm")
    elig = q > ao_screening_threshold
    keep, ao, q = keep[elig], ao[elig], q[elig]
    n = len(keep)
    physical_rank = d * (d + 1) // 2
    if max_rank > min(n, physical_rank):
        raise ValueError("requested anchor_rank exceeds eligible candidates or physical pair rank")
    if n == 0:
        return ([], {}) if return_details else []
    u, v = sketch_factors(d, ell, seed)
    f = ao / np.sqrt(q)[:, None] if normalized else ao
    y = (np.sqrt(importance[keep]) / np.sqrt(ell))[:, None] * (f @ u) * (f @ v)
    pos, det = sketch_qr_rank(y, ell, oversampling, tolerance, max_rank, physical_rank)
    piv = [int(keep[p]) for p in pos]
    if return_details:
        return piv, dict(y=y, keep=keep, q=q, **det)
    return piv


# ---------------------------------------------------------------------------
# RBRP (cpp/src/anchor_select_rbrp.cpp:195-320), explicit pair rows
# ---------------------------------------------------------------------------
def rbrp_pair_rows(ao, w):
    """row_g[(mu, nu)] = sqrt|w_g| phi_mu phi_nu (x sqrt 2 off the diagonal), mu <= nu."""
    n, nao = ao.shape
    iu, ju = np.triu_indices(nao)
    c = np.where(iu == ju, 1.0, np.sqrt(2.0))
    return np.sqrt(np.abs(w))[:, None] * ao[:, iu] * ao[:, ju] * c[None, :]


def rbrp_ao(ao, w, batch_size=128, block_size=16, tolerance=1e-10, max_rank=0, seed=7, tau_block=None,
            rank_rtol=1e-12, refresh_every=8, svd_rtol=1e-12, compute_id=False):
    """Robust blockwise random pivoting over the AO pair rows and its ID
    (``cpp/src/anchor_select_rbrp.cpp:136-320``), with LAPACK dgeqp3 / dorgqr
    (scipy) for the block QR and gesdd (numpy) for the small SVD."""
    from scipy.linalg.lapack import dgeqp3, dorgqr
    ao = np.asarray(ao, float)
    w = np.asarray(w, float)
    n, nao = ao.shape
    if (not n or not nao or batch_size <= 0 or block_size <= 0 or not np.isfinite(tolerance) or tolerance < 0
            or not np.isfinite(rank_rtol) or rank_rtol <= 0 or not np.isfinite(svd_rtol) or svd_rtol < 0
            or (tau_block is not None and (not np.isfinite(tau_block) or not 0 <= tau_block < 1))):
        raise ValueError("invalid RBRP dimensions, batch size or tolerances")
    p = nao * (nao + 1) // 2
    cap = min(p, n, max_rank if max_rank else min(n, p))
    tau_block = (1.0 / block_size if block_size > 1 else 0.0) if tau_block is None else tau_block
    if not np.all(np.isfinite(w)) or np.any(w == 0):
        raise ValueError("RBRP requires finite nonzero weights")
    if not np.all(np.isfinite(ao)):
        raise ValueError("RBRP requires finite real AOs")
    rows = rbrp_pair_rows(ao, w)
    d = np.abs(w) * np.einsum("gi,gi->g", ao, ao) ** 2
    total = float(np.sum(d))
    target = tolerance * tolerance * total
    q = np.zeros((0, p))
    L = np.zeros((n, 0))
    chosen = np.zeros(n, bool)
    rng = lib().oracle_rng_new(np.uint64(seed))
    indices, history, status, it = [], [], "rank_cap", 0

    def residual():
        e = rows - L @ q
        r = np.einsum("gi,gi->g", e, e)
        r[chosen] = 0.0
        return r

    try:
        while True:
            old = len(indices)
            if old and (sum(d) <= target or (refresh_every and it % refresh_every == 0)):
                d = residual()
            if sum(d) <= target:
                status = "tolerance"
                break
            if old >= cap:
                break
            active = [i for i in range(n) if d[i] > 0 and not chosen[i]]
            if not active:
                status = "no_candidates"
                break
            b = min(block_size, cap - old, len(active))
            sample = []
            for _ in range(b):
                left = np.ascontiguousarray([d[i] for i in active])
                pos = lib().oracle_rng_discrete(rng, _p(left), len(left))
                sample.append(active.pop(pos))
            v = rows[sample].T.copy()                          # p x b
            original2 = float(np.sum(v * v))
            for _ in range(2):
                for j in range(b):
                    for t in range(old):
                        v[:, j] -= (v[:, j] @ q[t]) * q[t]
            qr_, jpvt, tau_, _, info = dgeqp3(np.asfortranarray(v))
            if info != 0:
                raise RuntimeError("RBRP block geqp3 failed")
            tails = np.zeros(b)
            for row in range(b - 1, -1, -1):
                tails[row] = (tails[row + 1] if row + 1 < b else 0.0) + np.sum(qr_[row, row:b] ** 2)
            if not (tails[0] > 0) or not np.isfinite(tails[0]):
                status = "numerical_rank"
                break
            keep = 0
            for i in range(b):
                if tails[i] >= tau_block * tails[0]:
                    keep = i + 1
            cutoff = rank_rtol * np.sqrt(original2)
            for i in range(keep):
                if abs(qr_[i, i]) <= cutoff:
                    keep = i
                    break
            if not keep:
                status = "numerical_rank"
                break
            qb, _, info = dorgqr(qr_[:, :keep], tau_[:keep])
            if info != 0:
                raise RuntimeError("RBRP block orgqr failed")
            qb = np.array(qb)
            for j in range(keep):
                col = qb[:, j]
                for _ in range(2):
                    for t in range(old):
                        col -= (q[t] @ col) * q[t]
                    for t in range(j):
                        col -= (qb[:, t] @ col) * qb[:, t]
                nrm = np.linalg.norm(col)
                if not (nrm > 0) or not np.isfinite(nrm):
                    raise RuntimeError("RBRP block lost orthogonality")
                qb[:, j] = col / nrm
            prev = chosen.copy()
            lnew = rows @ qb
            lnew[prev] = 0.0
            d = np.where(prev, 0.0, np.maximum(0.0, d - np.sum(lnew ** 2, axis=1)))
            L = np.hstack([L, lnew])
            q = np.vstack([q, qb.T])
            for j in range(keep):
                idx = sample[jpvt[j] - 1]
                indices.append(idx)
                chosen[idx] = True
                d[idx] = 0.0
            history.append([len(indices), b, keep, np.sqrt(sum(d) / total) if total else 0.0])
            it += 1
    finally:
        lib().oracle_rng_free(rng)
    d = residual()
    rel = np.sqrt(sum(d) / total) if total else 0.0
    if rel <= tolerance:
        status = "tolerance"
    elif status == "tolerance":
        status = "roundoff_limited"
    out = {"indices": indices, "relative_residual": rel, "status": status, "history": np.array(history),
           "condition": 0.0, "retained_rank": 0}
    if not compute_id or not indices:
        return out
    k = len(indices)
    A = L[indices, :k]
    u, s, vt = np.linalg.svd(A)
    out["condition"] = s[0] / s[-1] if s[-1] else np.inf
    retained = int(np.sum(s > svd_rtol * s[0]))
    if not retained:
        raise RuntimeError("RBRP anchor block has zero numerical rank")
    out["retained_rank"] = retained
    inv = vt[:retained].T @ np.diag(1.0 / s[:retained]) @ u[:, :retained].T
    idx = np.array(indices)
    sw = np.sqrt(np.abs(w))
    fac = sw[idx] / w[idx]
    theta = (L[:, :k] @ inv).T * fac[:, None] / sw[None, :]
    theta[:, idx] = np.diag(1.0 / w[idx])
    iu, ju = np.triu_indices(nao)
    packed = (inv.T @ q[:k]) * fac[:, None]
    packed = packed / np.where(iu == ju, 1.0, np.sqrt(2.0))[None, :]
    transform = np.zeros((k, nao, nao))
    transform[:, iu, ju] = packed
    transform[:, ju, iu] = packed
    out["interp_vecs"] = theta
    out["transform"] = transform.reshape(k, nao * nao)
    return out


# ---------------------------------------------------------------------------
# grid Coulomb metric (python/isdf.py:48-97)
# ---------------------------------------------------------------------------
C_SPHERE = (32.0 / 15.0) * np.pi ** 2 * (3.0 / (4.0 * np.pi)) ** (5.0 / 3.0)


def grid_cross_metric(left, right, coords, weights, block=256):
    """sum_{g,h} left[a,g] w_g K_gh w_h right[b,h] with K_gh = 1/|r_g - r_h|
    off the diagonal (0 for coincident points) and K_gg = c |w_g|^(-1/3)
    (``python/isdf.py:80-97``), accumulated over row blocks of K."""
    coords = np.asarray(coords, float)
    weights = np.asarray(weights, float)
    lw = np.asarray(left, float).T * weights[:, None]
    rw = np.asarray(right, float).T * weights[:, None]
    out = np.zeros((lw.shape[1], rw.shape[1]))
    for g0 in range(0, len(weights), block):
        g1 = min(g0 + block, len(weights))
        r = np.linalg.norm(coords[g0:g1, None, :] - coords[None, :, :], axis=-1)
        kern = np.divide(1.0, r, out=np.zeros_like(r), where=r > 0)
        rows = np.arange(g0, g1)
        kern[rows - g0, rows] = C_SPHERE * np.abs(weights[rows]) ** (-1.0 / 3.0)
        out += lw[g0:g1].T @ (kern @ rw)
    return out


def grid_coulomb_metric(interp_vecs, coords, weights):
    """Symmetrised metric of one set (``python/isdf.py:48-68``)."""
    v = grid_cross_metric(interp_vecs, interp_vecs, coords, weights)
    return 0.5 * (v + v.T)


def isdf_jk(x, z, dm):
    """ISDF J and K of a symmetric density matrix (``python/isdf.py:130-151``):
    (mu nu|lam sig) ~ sum_pq X[p,mu] X[p,nu] Z[p,q] X[q,lam] X[q,sig]."""
    x = np.asarray(x, float)
    d = x @ dm @ x.T
    j = x.T @ ((z @ np.diag(d))[:, None] * x)
    k = x.T @ (z * d) @ x
    return 0.5 * (j + j.T), 0.5 * (k + k.T)


# ---------------------------------------------------------------------------
# fit and pair error (python/isdf.py)
# ---------------------------------------------------------------------------
def physical_pair_refit(anchor_pairs, anchor_weights, ao, batch_size=2048):
    """``_physical_pair_refit`` (``python/isdf.py:238-263``) restated."""
    u, s, vh = np.linalg.svd(anchor_pairs.T, full_matrices=False)
    retained = s > (1e-12 * s[0] if len(s) else 0)
    physical_transform = (vh[retained].T / s[retained]) @ u[:, retained].T
    theta = np.empty((len(anchor_weights), len(ao)))
    for first in range(0, len(ao), batch_size):
        block = ao[first:first + batch_size]
        pairs = (block[:, :, None] * block[:, None, :]).reshape(len(block), -1)
        theta[:, first:first + len(block)] = (physical_transform @ pairs.T) / anchor_weights[:, None]
    diag = {"retained_rank": int(np.count_nonzero(retained)),
            "condition": float(s[0] / s[-1]) if len(s) and s[-1] > 0 else float("inf"),
            "singular_values": s}
    return theta, diag


def pair_space_error_norms(pair_grid, pair_anchor, anchor_weights, theta, grid_weights,
                           block_size=256):
    """``pair_space_error_norms`` (``python/isdf.py:154-173``) restated."""
    weighted_anchor = pair_anchor * anchor_weights[:, None]
    residual_sq = exact_sq = 0.0
    for first in range(0, len(grid_weights), block_size):
        last = min(first + block_size, len(grid_weights))
        exact = pair_grid[first:last]
        rec = theta[:, first:last].T @ weighted_anchor
        weight = np.abs(grid_weights[first:last])
        residual_sq += np.einsum("g,gi,gi->", weight, exact - rec, exact - rec)
        exact_sq += np.einsum("g,gi,gi->", weight, exact, exact)
    absolute = np.sqrt(residual_sq)
    relative = absolute / np.sqrt(exact_sq) if exact_sq else (0.0 if absolute == 0 else np.inf)
    return {"l2": absolute, "relative": relative}


def gram_fit(ctx, coords, weights, anchor_coords, anchor_weights):
    """Theta and pair error in Gram form (large grids), FP64.

    X_g = pinv((Phi_a Phi_a^T)o2) (G_g o G_g) equals pinv(C^T) p_g of the
    literal SVD fit when the anchor pair matrix C has full rank; the cutoff
    is applied to singular values of C (sqrt of eigenvalues of M).
    """
    phi_a = ctx.eval_ao(anchor_coords)
    S = phi_a @ phi_a.T
    M = S * S
    lam, vec = np.linalg.eigh(M)
    s = np.sqrt(np.clip(lam, 0, None))
    keep = s > 1e-12 * s.max()
    T = (vec[:, keep] / lam[keep]) @ vec[:, keep].T
    G, q = ctx.grid_gram(coords, phi_a)
    n, k = G.shape
    theta = np.empty((k, n))
    err2 = np.zeros(1)
    ex2 = np.zeros(1)
    w = np.ascontiguousarray(weights, float)
    lib().oracle_fit_apply(n, k, _p(G), _p(q), _p(w), _p(np.ascontiguousarray(T)),
                           _p(np.ascontiguousarray(M)),
                           _p(np.ascontiguousarray(anchor_weights, float)), _p(theta),
                           _p(err2), _p(ex2))
    err2 = max(err2[0], 0.0)
    return theta, {"l2": np.sqrt(err2), "relative": np.sqrt(err2 / ex2[0]) if ex2[0] else 0.0,
                   "err2": err2, "exact2": float(ex2[0])}


# ---------------------------------------------------------------------------
# nuclear-gradient reference (not in the reference project)
# ---------------------------------------------------------------------------
def isdf_energy(ctx, coords, weights, anchor_coords, anchor_weights, dm):
    """E = sum_g w_g rho_ISDF(g)^2 with rho_ISDF(g) = sum_k Theta_kg w_k rho_a(k)."""
    phi_a = ctx.eval_ao(anchor_coords)
    M = (phi_a @ phi_a.T) ** 2
    rho_a = np.einsum("ki,ij,kj->k", phi_a, dm, phi_a)
    z = np.linalg.solve(M, rho_a)
    G, _ = ctx.grid_gram(coords, phi_a)
    rho = (G * G) @ z
    return float(np.sum(weights * rho * rho))


def isdf_energy_gradient(ctx, coords, weights, anchor_coords, anchor_weights, dm,
                         chunk=65536):
    """Analytic dE/dR[natm,3] from AO values and dx/dy/dz (d phi/dR_A = -grad_r phi)."""
    natm = ctx.natm
    own = ctx.ao_atom
    phi_a = ctx.eval_ao(anchor_coords)              # [k, nao]
    dphi_a = ctx.eval_ao_gradient(anchor_coords)    # [3, k, nao]
    S = phi_a @ phi_a.T
    M = S * S
    rho_a = np.einsum("ki,ij,kj->k", phi_a, dm, phi_a)
    z = np.linalg.solve(M, rho_a)
    k, nao = phi_a.shape
    grad = np.zeros((natm, 3))
    B = np.zeros((k, nao))
    v = np.zeros(k)
    for s in range(0, len(coords), chunk):
        pts = coords[s:s + chunk]
        w = weights[s:s + chunk]
        phi = ctx.eval_ao(pts)                      # [b, nao]
        dphi = ctx.eval_ao_gradient(pts)            # [3, b, nao]
        G = phi @ phi_a.T                           # [b, k]
        h = G * G
        rho = h @ z
        u = 2 * w * rho
        v += u @ h
        alpha = 2 * u[:, None] * z[None, :] * G     # [b, k]
        B += alpha.T @ phi
        beta = alpha @ phi_a                        # [b, nao]
        contrib = np.einsum("gm,cgm->cm", beta, dphi)   # [3, nao]
        for c in range(3):
            np.add.at(grad[:, c], own, -contrib[c])
    # anchor-side terms: B (grid reduction) and the M / rho_a dependence
    y = np.linalg.solve(M, v)
    # d rho_a(k) = 2 phi_a(k)^T D dphi_a(k)
    Dphi = phi_a @ dm                               # [k, nao]
    anchor_coef = B + 2 * y[:, None] * Dphi         # coefficient of dphi_a[k, mu]
    # -y^T dM z, dM_kl = 2 S_kl dS_kl, dS_kl = dphi_k.phi_l + phi_k.dphi_l
    W = 2 * S * (y[:, None] * z[None, :])           # coefficient of dS_kl
    anchor_coef -= (W + W.T) @ phi_a
    contrib = np.einsum("km,ckm->cm", anchor_coef, dphi_a)
    for c in range(3):
        np.add.at(grad[:, c], own, -contrib[c])
    return grad
