"""Pins the CPU oracle against the known answers held by the reference's own
tests (mikovtun/mp_isdf python/test/*.py) and against independent checks.

The reference cannot be built in this environment and PySCF is absent, so:
selection pivots are pinned to LAPACK dgeqp3 (scipy) exactly as the
reference tests do; fit/error to the reference's literal NumPy functions and
to their hand-computed answers; AO values by normalisation and derivative
consistency (PySCF parity is unpinned here).
"""
import numpy as np
import pytest
from scipy.linalg import qr

from oracle import oracle as O


@pytest.fixture(scope="module")
def sctx(s_shells):
    return O.OracleContext(*s_shells)


def test_c2s_orthonormal_on_sphere():
    from scipy.integrate import lebedev_rule
    x, w = lebedev_rule(41)
    pts = x.T
    w = w / w.sum() * 4 * np.pi
    for l in range(0, O.LMAX + 1):
        t = O.c2s_matrix(l)
        mono = np.array([pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c
                         for a, b, c in O.cart_powers(l)])
        y = t @ mono
        np.testing.assert_allclose((y * w) @ y.T, np.eye(2 * l + 1), atol=1e-12)


def test_ao_normalised_and_gradient_consistent(small_water):
    mol, pts, w = small_water
    ctx = O.OracleContext(mol.atm, mol.bas, mol.env)
    # each synthetic AO integrates to one (PySCF normalisation convention)
    from mp_isdf_b200 import inputs
    sym, xyz = mol.symbols[:3], mol.coords[:3]
    gp, gw = inputs.becke_grid(sym, xyz, level=3)
    single = inputs.build_tables(sym, xyz)
    c1 = O.OracleContext(single.atm, single.bas, single.env)
    phi = c1.eval_ao(gp)
    np.testing.assert_allclose(np.einsum("g,gi,gi->i", gw, phi, phi), 1.0, atol=2e-5)
    # analytic gradient vs central differences
    rng = np.random.default_rng(3)
    p = rng.normal(size=(7, 3)) + mol.coords[0]
    g = ctx.eval_ao_gradient(p)
    h = 1e-5
    for c in range(3):
        e = np.zeros(3); e[c] = h
        fd = (ctx.eval_ao(p + e) - ctx.eval_ao(p - e)) / (2 * h)
        np.testing.assert_allclose(g[c], fd, rtol=1e-6, atol=1e-8)


def test_three_s_shells_qrcp_known_answers(sctx):
    """python/test/test_online_anchor_select.py:44-69, 85-96."""
    points = np.random.default_rng(23).normal(size=(17, 3))
    weights = np.linspace(0.5, 2, 17)
    weights[2] = 0
    weights[4] *= -1
    mask = weights != 0
    features = sctx.axis_features(points[mask], [0])
    matrix = O.pair_matrix(features, weights[mask])
    expected = np.flatnonzero(mask)[qr(matrix, pivoting=True)[2]]
    actual = O.select_qrcp_dense(sctx, points, weights, [0])
    assert len(actual) == 6                      # symmetric AO pairs
    np.testing.assert_array_equal(actual, expected[:6])
    np.testing.assert_array_equal(O.select_qrcp_dense(sctx, points, weights, [0], max_rank=3),
                                  expected[:3])
    assert O.select_qrcp_dense(sctx, points, weights, [0], tolerance=1) == []
    assert O.select_qrcp_dense(sctx, points, np.zeros(17), [0]) == []
    # greedy residual property at every rank
    pos = np.searchsorted(np.flatnonzero(mask), actual)
    for k, pv in enumerate(pos):
        if k:
            q = qr(matrix[:, pos[:k]], mode="economic")[0]
            res = matrix - q @ (q.T @ matrix)
        else:
            res = matrix
        assert abs(np.linalg.norm(res[:, pv]) - np.linalg.norm(res, axis=0).max()) < 1e-9


def test_three_s_shells_rand_sketch_known_answers(sctx):
    """python/test/test_randomized_anchor_select.py:151-172."""
    points = np.random.default_rng(23).normal(size=(19, 3))
    weights = np.linspace(.4, 1.5, 19)
    weights[2] = 0
    weights[4] = -1
    opts = dict(sketch_size=12, oversampling=3, seed=31)
    piv = O.select_rand_sketch(sctx, points, weights, [0], max_rank=3, **opts)
    assert len(piv) == 3 and 2 not in piv
    mask = weights != 0
    a = O.pair_matrix(sctx.axis_features(points[mask], [0]), weights[mask])
    q = qr(a[:, np.searchsorted(np.flatnonzero(mask), piv)], mode="economic")[0]
    assert np.linalg.norm(a - q @ (q.T @ a)) / np.linalg.norm(a) < 0.4
    assert len(O.select_rand_sketch(sctx, points, weights, [0], **opts)) == 6
    assert O.select_rand_sketch(sctx, points, weights, [0], tolerance=1, **opts) == []
    assert len(O.select_rand_sketch(sctx, points, weights, [0], tolerance=1, max_rank=2,
                                    **opts)) == 2
    assert len(O.select_rand_sketch(sctx, points, weights, [0], tolerance=0, max_rank=2,
                                    **opts)) == 2
    # explicit rank fixes the sketch rows independently of sketch_size
    assert (O.select_rand_sketch(sctx, points, weights, [0], max_rank=3, sketch_size=2,
                                 oversampling=3, seed=31) == piv)
    with pytest.raises(ValueError):
        O.select_rand_sketch(sctx, points, weights, [0], sketch_size=12, oversampling=0)


def test_khatri_rao_identity():
    """python/test/test_randomized_anchor_select.py:215-224."""
    rng = np.random.default_rng(7)
    phi = rng.normal(size=(4, 9))
    w = rng.uniform(.1, 2., size=9)
    g = rng.normal(size=(6, 4))
    h = rng.normal(size=(6, 4))
    structured = (g @ phi) * (h @ phi) * (np.sqrt(w) / np.sqrt(6))[None, :]
    pairs = np.einsum("ig,jg->ijg", phi, phi).reshape(16, 9)
    projection = np.einsum("si,sj->sij", g, h).reshape(6, 16) / np.sqrt(6)
    np.testing.assert_allclose(structured, projection @ (pairs * np.sqrt(w)))


def test_sketch_matches_explicit_khatri_rao(sctx):
    points = np.random.default_rng(5).normal(size=(11, 3))
    w = np.linspace(0.3, 1.2, 11)
    f = sctx.axis_features(points, [0])
    u, v = O.sketch_factors(3, 5, 9)
    y = sctx.sketch(points, w, [0], None, u, v, 5)
    expected = np.sqrt(w)[:, None] / np.sqrt(5) * (f @ u) * (f @ v)
    np.testing.assert_allclose(y, expected, rtol=1e-14)


def test_pair_error_signed_weights_known_answer():
    """python/test/test_isdf.py:157-164."""
    exact = np.array([[1., 2.], [3., 4.]])
    anchor = np.array([[1., 0.]])
    theta = np.array([[1., 3.]])
    e = O.pair_space_error_norms(exact, anchor, np.array([1.]), theta, np.array([2., -1.]),
                                 block_size=1)
    np.testing.assert_allclose(e["l2"], np.sqrt(24.))
    np.testing.assert_allclose(e["relative"], np.sqrt(24. / 35.))


def test_fit_matches_lstsq_and_gram_form(small_water):
    """python/test/test_isdf.py:43-49: Theta == lstsq(pairs^T, products^T)/w_anchor."""
    mol, pts, w = small_water
    ctx = O.OracleContext(mol.atm, mol.bas, mol.env)
    keep = w != 0
    coords, weights = pts[keep][::7], w[keep][::7]
    piv = O.select_qrcp_dense(ctx, coords, weights, [0], max_rank=6)
    ao = ctx.eval_ao(coords)
    anchor_ao = ctx.eval_ao(coords[piv])
    pairs = (anchor_ao[:, :, None] * anchor_ao[:, None, :]).reshape(len(piv), -1)
    theta, _ = O.physical_pair_refit(pairs, weights[piv], ao, batch_size=7)
    products = (ao[:, :, None] * ao[:, None, :]).reshape(len(ao), -1)
    ref = np.linalg.lstsq(pairs.T, products.T, rcond=1e-12)[0] / weights[piv][:, None]
    np.testing.assert_allclose(theta, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    err = O.pair_space_error_norms(products, pairs, weights[piv], theta, weights)
    theta_g, err_g = O.gram_fit(ctx, coords, weights, coords[piv], weights[piv])
    np.testing.assert_allclose(theta_g, theta, rtol=1e-7, atol=1e-7 * np.abs(theta).max())
    np.testing.assert_allclose(err_g["relative"], err["relative"], rtol=1e-9)
    np.testing.assert_allclose(err_g["l2"], err["l2"], rtol=1e-9)


def test_multi_axis_scales_follow_reference_rule(small_water):
    mol, pts, w = small_water
    ctx = O.OracleContext(mol.atm, mol.bas, mol.env)
    sub = slice(0, 400)
    s_exact = O.axis_scales(ctx, pts[sub], w[sub], [0, 1, 3], [1.0, 0.5, 2.0])
    s_fast = O.axis_scales(ctx, pts[sub], w[sub], [0, 1, 3], [1.0, 0.5, 2.0],
                           exact_order=False)
    np.testing.assert_allclose(s_exact, s_fast, rtol=1e-12)
    keep = w[sub] != 0
    f = ctx.axis_features(pts[sub][keep], [0, 1, 3])
    nao = ctx.nao
    norms = [np.linalg.norm(f[:, i * nao:(i + 1) * nao]) for i in range(3)]
    np.testing.assert_allclose(s_exact, np.array([1.0, 0.5, 2.0]) / norms, rtol=1e-12)


def test_adjoint_reference_matches_finite_differences(small_water):
    mol, pts, w = small_water
    keep = w != 0
    coords, weights = pts[keep][::5], w[keep][::5]
    ctx = O.OracleContext(mol.atm, mol.bas, mol.env)
    piv = O.select_qrcp_dense(ctx, coords, weights, [0], max_rank=5)
    phi = ctx.eval_ao(coords)
    S = phi.T @ (weights[:, None] * phi)
    from mp_isdf_b200.inputs import random_density
    dm = random_density(mol, S, 20.0, seed=3)
    grad = O.isdf_energy_gradient(ctx, coords, weights, coords[piv], weights[piv], dm)
    # Central differences at h = 1e-4 bohr, Richardson-extrapolated with h/2:
    # the synthetic O core exponent (~1e4) makes the plain h^2 error ~1e-4
    # relative for grid points a few 1e-3 bohr from the oxygen nucleus.
    def energy(atom, c, step):
        xyz = mol.coords.copy()
        xyz[atom, c] += step
        m2 = mol.with_coords(xyz)
        c2 = O.OracleContext(m2.atm, m2.bas, m2.env)
        return O.isdf_energy(c2, coords, weights, coords[piv], weights[piv], dm)

    h = 1e-4
    for atom, c in [(0, 0), (1, 2), (4, 1)]:
        fd1 = (energy(atom, c, h) - energy(atom, c, -h)) / (2 * h)
        fd2 = (energy(atom, c, h / 2) - energy(atom, c, -h / 2)) / h
        fd = (4 * fd2 - fd1) / 3
        np.testing.assert_allclose(grad[atom, c], fd, rtol=1e-6,
                                   atol=1e-6 * np.abs(grad).max())


def test_exact_norm_qrcps_match_lapack_dgeqp3(small_water):
    """The exact-norm truncated QRCPs that write the golden fixtures pick the
    same pivots as LAPACK dgeqp3 (scipy) on the explicit pair matrix
    (qrcp_dense, cpp/src/anchor_select_qrcp.cpp:248-307) and on the sketch
    (cpp/src/anchor_select_randomized_id.cpp:320-374), with the same |R_jj|."""
    mol, pts, w = small_water
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    keep = np.flatnonzero(w != 0)
    f = oc.axis_features(pts[keep], [0])
    ref = O.select_qrcp_dense(oc, pts, w, [0], max_rank=12)
    pos, diag, gaps = O.pair_qrcp_exact(f, w[keep], 12)
    assert [int(keep[p]) for p in pos] == ref
    assert np.all(gaps > 1e-10)
    piv, det = O.select_rand_sketch(oc, pts, w, [0], max_rank=10, oversampling=16, seed=7,
                                    return_details=True)
    pos, diag, gaps = O.sketch_qrcp_exact(det["y"].T, 26)
    assert pos == [int(j) for j in det["jpvt"][:26]]
    np.testing.assert_allclose(diag, det["diag"][:26], rtol=1e-12)


def test_golden_fixtures_are_consistent():
    """Each committed golden fixture (tests/golden/*.npz) holds one anchor per
    rank, positive step gaps, Theta on the sampled columns, and -- for the
    randomized sketch -- anchors equal to LAPACK dgeqp3's pivots wherever the
    exact-norm gap exceeds 1e-10."""
    from pathlib import Path
    files = sorted((Path(__file__).resolve().parent / "golden").glob("*.npz"))
    assert {p.stem for p in files} >= {"c1", "c2", "c2o", "c3", "c4"}
    for p in files:
        g = np.load(p)
        k = int(g["rank"])
        assert len(g["anchors"]) == k and len(g["step_gap"]) == k
        assert np.all(g["step_gap"] >= 0) and np.all(g["step_diag"] > 0)
        assert g["theta_sample"].shape == (k, len(g["theta_pos"]))
        assert 0 < float(g["pair_relative"]) < 1
        if "dgeqp3_pivots" in g:
            for j, (a, b) in enumerate(zip(g["anchors"], g["dgeqp3_pivots"])):
                if a != b:
                    assert g["step_gap"][j] <= 1e-10
                    break
