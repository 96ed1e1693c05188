"""The allocation-free pair-error reduction (isdf_pair_error_terms_noalloc)
against the allocating one (isdf_pair_error_terms), through the C-ABI.

Callers that may not allocate device memory on the call path (fixed memory
budgets, their own pools, no cudaFree synchronisation) use the no-alloc entry
point; its only scratch is a fixed device array inside the library.  Two
consecutive calls on different inputs check that the shared scratch left by
the previous call does not leak into the next result.  Runs alone in a fresh
process or after the other tests; collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _terms(rng, n, k):
    import torch
    phi_g = rng.normal(size=(n, 12))
    phi_a = rng.normal(size=(k, 12))
    G = phi_g @ phi_a.T
    H = G * G
    M = (phi_a @ phi_a.T) ** 2
    X = np.linalg.solve(M, H.T).T * (1 + 1e-3 * rng.normal(size=(n, k)))
    q = np.sum(phi_g * phi_g, axis=1)
    w = rng.uniform(-1, 2, size=n)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    return t(q), t(H), t(X), t(M), t(w)


def _noalloc(q, H, X, M, w):
    import torch
    from mp_isdf_b200 import capi
    n, k = H.shape
    out = np.zeros(2)
    P = ctypes.c_void_p
    s = P(torch.cuda.current_stream().cuda_stream)
    capi.check(capi.lib().isdf_pair_error_terms_noalloc(
        n, k, P(q.data_ptr()), P(H.data_ptr()), P(X.data_ptr()), P(M.data_ptr()),
        P(w.data_ptr()), out.ctypes.data_as(P), s))
    return out


def test_noalloc_matches_allocating_entry_point_twice():
    from mp_isdf_b200 import capi
    rng = np.random.default_rng(5)
    for n, k in ((300001, 10), (777, 64)):
        q, H, X, M, w = _terms(rng, n, k)
        ref = capi.pair_error_terms(q, H, X, M, w)
        got = _noalloc(q, H, X, M, w)
        np.testing.assert_allclose(got[0], ref["l2"], rtol=1e-12)
        np.testing.assert_allclose(got[1], ref["relative"], rtol=1e-12)


def test_noalloc_rejects_too_many_anchors():
    from mp_isdf_b200 import capi
    rng = np.random.default_rng(6)
    q, H, X, M, w = _terms(rng, 100, 65)
    with pytest.raises(capi.IsdfError) as exc:
        _noalloc(q, H, X, M, w)
    assert exc.value.status == 1
