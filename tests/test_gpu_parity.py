"""GPU parity of the B200 library against the CPU oracle, through the drop-in
module and the C-ABI.  Tolerances: AO values/gradients rtol 1e-11, atol 1e-12
(the reference's own test tolerance, python/test/test_ao_eval.py:207);
pivots exact except where the oracle's top-two residual gap is below 1e-10
relative; Theta rtol 1e-9 x cond^2 scale; pair error rtol 1e-9."""
import numpy as np
import pytest
from scipy.linalg import qr

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mpi():
    import mp_isdf
    return mp_isdf


@pytest.fixture(scope="module")
def s_ctx(mpi, s_shells):
    c = mpi.LibcintContext(*s_shells)
    return c, mpi.AnchorSelection(c), O.OracleContext(*s_shells)


@pytest.fixture(scope="module")
def water(mpi, small_water):
    mol, pts, w = small_water
    c = mpi.LibcintContext(mol.atm, mol.bas, mol.env)
    return mol, pts, w, c, mpi.AnchorSelection(c), O.OracleContext(mol.atm, mol.bas, mol.env)


# ---------------------------------------------------------------------------
# AO evaluation
# ---------------------------------------------------------------------------
def test_ao_values_gradients_match_oracle(water):
    mol, pts, w, c, sel, oc = water
    rng = np.random.default_rng(42)
    p = np.vstack([mol.coords[:2], rng.normal(size=(37, 3)) * 2 + mol.coords[0], pts[::97]])
    np.testing.assert_allclose(c.eval_ao(p), oc.eval_ao(p), rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(c.eval_ao_gradient(p), oc.eval_ao_gradient(p), rtol=1e-11, atol=1e-12)
    assert c.eval_ao(p).shape == (len(p), mol.nao)
    assert c.eval_ao_gradient(p).shape == (3, len(p), mol.nao)


def test_ao_empty_grid_and_owned_tables(mpi, small_water):
    mol, _, _ = small_water
    atm, bas, env = mol.atm.copy(), mol.bas.copy(), mol.env.copy()
    c = mpi.LibcintContext(atm, bas, env)
    assert c.nao == mol.nao
    assert c.eval_ao(np.empty((0, 3))).shape == (0, mol.nao)
    assert c.eval_ao_gradient(np.empty((0, 3))).shape == (3, 0, mol.nao)
    p = np.random.default_rng(7).normal(size=(9, 3))
    ref = c.eval_ao(p)
    atm.fill(0); bas.fill(0); env.fill(0)   # the context owns private copies
    for _ in range(2):
        np.testing.assert_array_equal(c.eval_ao(p), ref)
    with pytest.raises(ValueError):
        c.eval_ao(p, space="invalid")
    for space in ("auto", "host", "device"):
        np.testing.assert_array_equal(c.eval_ao(p, space=space), ref)
    np.testing.assert_array_equal(mpi.eval_ao(mol.atm, mol.bas, mol.env, p), ref)


def test_ao_float32_and_device_tensor_path(small_water):
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    p = pts[::13]
    xyz = torch.tensor(p, device="cuda")
    v64 = torch.empty(len(p), mol.nao, dtype=torch.float64, device="cuda")
    g64 = torch.empty(3, len(p), mol.nao, dtype=torch.float64, device="cuda")
    ctx.eval_ao(xyz, v64, g64)
    v32 = torch.empty(len(p), mol.nao, dtype=torch.float32, device="cuda")
    g32 = torch.empty(3, len(p), mol.nao, dtype=torch.float32, device="cuda")
    ctx.eval_ao(xyz, v32, g32)
    torch.cuda.synchronize()
    ref, gref = oc.eval_ao(p), oc.eval_ao_gradient(p)
    np.testing.assert_allclose(v64.cpu().numpy(), ref, rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(g64.cpu().numpy(), gref, rtol=1e-11, atol=1e-12)
    # FP32 storage form: relative to each point's largest value
    scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-30
    assert np.max(np.abs(v32.cpu().numpy() - ref) / scale) < 2e-6
    gscale = np.abs(gref).max(axis=2, keepdims=True) + 1e-30
    assert np.max(np.abs(g32.cpu().numpy() - gref) / gscale) < 4e-6


@pytest.mark.parametrize("extra_l", [None, 4, 6])
def test_ao_tiled_path_matches_point_path_and_oracle(small_water, extra_l):
    """Grids above 2048 points take the tiled evaluator (64 points per block,
    aligned 32-AO window rows); fewer take one point per block.  Both
    give the same values (up to the contraction of a product into an FMA,
    which may differ between kernels, and the tiled kernel's screening, which
    writes zeros for a piece whose values and gradients stay below 1e-15 at
    all 32 points of a warp), over a ragged point count, a block of points far
    from every atom (every piece screened) and, with an added l = 4 or l = 6
    shell, the two-lane layouts; FP64 also against the oracle."""
    import torch
    from mp_isdf_b200 import capi, inputs
    mol, pts, w = small_water
    if extra_l is None:
        tables = mol
    else:
        def shells_of(sym):
            sh = inputs.element_shells(sym)
            if sym == "O":
                sh = sh + [inputs.Shell(extra_l, np.array([2.1, 0.6]), np.array([[0.7, 0.4], [0.0, 1.0]]))]
            return sh
        tables = inputs.build_tables(mol.symbols, mol.coords, shells_of)
    ctx = capi.Context(tables.atm, tables.bas, tables.env)
    oc = O.OracleContext(tables.atm, tables.bas, tables.env)
    rng = np.random.default_rng(3)
    far = mol.coords[0] + np.array([40.0, 0.0, 0.0]) + rng.normal(size=(64, 3))
    p = np.vstack([pts[: 2000], far, mol.coords, rng.normal(size=(1000, 3)) * 3 + mol.coords[1]])
    n, nao = len(p), tables.nao
    assert n > 2048 and n % 32 != 0
    xyz = torch.tensor(p, device="cuda")
    sub = torch.arange(0, n, 3, device="cuda")   # 1023 points: the one-point-per-block path
    with pytest.raises(capi.IsdfError, match="needs a values or a gradient output"):
        ctx.eval_ao(xyz, None, None, dtype=torch.float64)   # nothing to write
    for dt, tol in ((torch.float64, 1e-14), (torch.float32, 1e-6)):
        v = torch.empty(n, nao, dtype=dt, device="cuda")
        g = torch.empty(3, n, nao, dtype=dt, device="cuda")
        ctx.eval_ao(xyz, v, g)
        vo = torch.empty(n, nao, dtype=dt, device="cuda")
        ctx.eval_ao(xyz, vo)
        go = torch.empty(3, n, nao, dtype=dt, device="cuda")
        ctx.eval_ao(xyz, None, go, dtype=dt)
        vs = torch.empty(len(sub), nao, dtype=dt, device="cuda")
        gs = torch.empty(3, len(sub), nao, dtype=dt, device="cuda")
        ctx.eval_ao(xyz[sub].contiguous(), vs, gs)
        torch.cuda.synchronize()
        assert torch.equal(g, go)   # the same kernel with and without the values written
        vt, gt = v[sub].double().cpu().numpy(), g[:, sub].double().cpu().numpy()
        vp, gp = vs.double().cpu().numpy(), gs.double().cpu().numpy()
        vscale = np.abs(vp).max(axis=1, keepdims=True) + 1e-300
        gscale = np.abs(gp).max(axis=2, keepdims=True) + 1e-300
        # values alone come from the kernel without gradients (its own FMA contraction)
        vv = vo[sub].double().cpu().numpy()
        screen = 1e-15   # kScreenFp64: the most a screened value or gradient can be
        assert np.all(np.abs(vv - vp) <= tol * vscale + screen)
        assert np.all(np.abs(vt - vp) <= tol * vscale + screen)
        assert np.all(np.abs(gt - gp) <= tol * gscale + screen)
        assert not v[2000:2064].any() and not g[:, 2000:2064].any()   # far block: exact zeros
        if dt == torch.float64:
            np.testing.assert_allclose(v.cpu().numpy(), oc.eval_ao(p), rtol=1e-11, atol=1e-12)
            np.testing.assert_allclose(g.cpu().numpy(), oc.eval_ao_gradient(p), rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("extra_l", [None, 4, 6])
def test_ao_value_warp_form_matches_block_form_and_oracle(small_water, extra_l):
    """Value-only launches of at least two waves (SMs x 1536 points) take the
    warp form of the tiled evaluator (one warp per 32 points, its own bounding
    box, no block barriers); smaller ones the block form.  Over a ragged count
    just above that size, with a block of points far from every atom, the
    values equal the block form's (the same points in slices below the
    threshold: the same per-piece arithmetic, up to FMA contraction) and, in
    FP64, the oracle's on a sample."""
    import torch
    from mp_isdf_b200 import capi, inputs
    mol, pts, w = small_water
    if extra_l is None:
        tables = mol
    else:
        def shells_of(sym):
            sh = inputs.element_shells(sym)
            if sym == "O":
                sh = sh + [inputs.Shell(extra_l, np.array([2.1, 0.6]), np.array([[0.7, 0.4], [0.0, 1.0]]))]
            return sh
        tables = inputs.build_tables(mol.symbols, mol.coords, shells_of)
    ctx = capi.Context(tables.atm, tables.bas, tables.env)
    oc = O.OracleContext(tables.atm, tables.bas, tables.env)
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    threshold = nsm * 1536
    rng = np.random.default_rng(11)
    n = threshold + 1000 + 13
    reps = -(-n // len(pts))
    p = (np.tile(pts, (reps, 1)) + rng.normal(scale=0.05, size=(reps * len(pts), 3)))[:n]
    far0 = 4096
    p[far0:far0 + 64] = mol.coords[0] + np.array([40.0, 0.0, 0.0]) + rng.normal(size=(64, 3))
    nao = tables.nao
    xyz = torch.tensor(p, device="cuda")
    slab = threshold // 2   # block form
    for dt, tol in ((torch.float64, 1e-14), (torch.float32, 1e-6)):
        v = torch.empty(n, nao, dtype=dt, device="cuda")
        ctx.eval_ao(xyz, v)
        vb = torch.empty(n, nao, dtype=dt, device="cuda")
        for s0 in range(0, n, slab):
            part = torch.empty(min(slab, n - s0), nao, dtype=dt, device="cuda")
            ctx.eval_ao(xyz[s0:s0 + slab].contiguous(), part)
            vb[s0:s0 + len(part)] = part
        torch.cuda.synchronize()
        a, b = v.double().cpu().numpy(), vb.double().cpu().numpy()
        scale = np.abs(b).max(axis=1, keepdims=True) + 1e-300
        assert np.all(np.abs(a - b) <= tol * scale + 1e-15)
        assert not v[far0:far0 + 64].any()   # far block: exact zeros
        if dt == torch.float64:
            sample = np.sort(rng.choice(n, 600, replace=False))
            np.testing.assert_allclose(a[sample], oc.eval_ao(p[sample]), rtol=1e-11, atol=1e-12)


def test_evaluate_axis_matches_oracle(water, mpi):
    mol, pts, w, c, sel, oc = water
    p = pts[::211]
    axes = [mpi.AxisType.AtomicOrbitalGradZ, mpi.AxisType.AtomicOrbital,
            mpi.AxisType.AtomicOrbitalGradZ, mpi.AxisType.AtomicOrbitalGradX]
    np.testing.assert_allclose(sel.evaluate_axis(p, axes), oc.axis_features(p, [3, 0, 3, 1]),
                               rtol=1e-11, atol=1e-12)
    with pytest.raises(ValueError):
        sel.evaluate_axis(p, mpi.AxisType.OccupiedOrbital)


# ---------------------------------------------------------------------------
# selection: known answers of the reference's tests
# ---------------------------------------------------------------------------
def test_three_s_shell_dense_and_online(s_ctx, mpi):
    """python/test/test_online_anchor_select.py:44-101."""
    c, sel, oc = s_ctx
    points = np.random.default_rng(23).normal(size=(17, 3))
    weights = np.linspace(0.5, 2, 17)
    weights[2] = 0
    weights[4] *= -1
    mask = weights != 0
    matrix = O.pair_matrix(oc.axis_features(points[mask], [0]), weights[mask])
    expected = np.flatnonzero(mask)[qr(matrix, pivoting=True)[2]]
    axis = mpi.AxisType.AtomicOrbital
    online = mpi.LocalAnchorSelectionAlgorithm.OnlineQRColumnPivoting
    dense = sel.select(points, weights, axis)
    assert len(dense) == 6
    np.testing.assert_array_equal(dense, expected[:6])
    for space in ("host", "device"):
        for batch in (1, 3, 17):
            got = sel.select(points, weights, axis, algorithm=online, space=space, batch_size=batch)
            np.testing.assert_array_equal(got, expected[:6])
            np.testing.assert_array_equal(
                sel.select(points, weights, axis, algorithm=online, batch_size=batch, max_rank=3),
                expected[:3])
    assert sel.select(points, weights, axis, algorithm=online, tolerance=1) == []
    for cutoff in (0.1, 0.5):
        assert (sel.select(points, weights, axis, algorithm=online, tolerance=cutoff, batch_size=2)
                == sel.select(points, weights, axis, tolerance=cutoff))
    assert sel.select(points, np.zeros_like(weights), axis, algorithm=online) == []
    with pytest.raises(ValueError):
        sel.select(points, weights, axis, algorithm=online, batch_size=0)


def test_three_s_shell_rand_sketch(s_ctx, mpi):
    """python/test/test_randomized_anchor_select.py:151-172, 283-307."""
    c, sel, oc = s_ctx
    points = np.random.default_rng(23).normal(size=(19, 3))
    weights = np.linspace(.4, 1.5, 19)
    weights[2] = 0
    weights[4] = -1
    algo = mpi.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao
    axis = mpi.AxisType.AtomicOrbital

    def select(**kw):
        return sel.select(points, weights, axis, algorithm=algo, sketch_size=12, oversampling=3,
                          seed=31, **kw)
    ref = O.select_rand_sketch(oc, points, weights, [0], max_rank=3, sketch_size=12,
                               oversampling=3, seed=31)
    for batch in (1, 4, 19):
        piv = select(batch_size=batch, max_rank=3)
        assert piv == ref
        assert len(piv) == 3 and 2 not in piv
    assert len(select(batch_size=4)) == 6
    assert select(tolerance=1, max_rank=0) == []
    assert len(select(tolerance=1, max_rank=2)) == 2
    assert len(select(tolerance=0, max_rank=2)) == 2
    assert sel.select(points, weights, axis, algorithm=algo, sketch_size=2, oversampling=3,
                      max_rank=3, seed=31) == ref
    with pytest.raises(ValueError):
        sel.select(points, weights, axis, algorithm=algo, sketch_size=12, oversampling=0)
    with pytest.raises(ValueError):
        select(batch_size=0)
    assert sel.select(points, np.zeros_like(weights), axis, algorithm=algo, sketch_size=12,
                      oversampling=3) == []
    # signed weights enter as |w|
    assert sel.select(points, np.abs(weights), axis, algorithm=algo, max_rank=3, oversampling=4,
                      sketch_size=1, seed=31) == \
        sel.select(points, weights, axis, algorithm=algo, max_rank=3, oversampling=4,
                   sketch_size=1, seed=31)


def _greedy_gaps(matrix, pivots_local):
    """Relative gap between the best and runner-up residual norm at each step."""
    gaps = []
    for k in range(len(pivots_local)):
        if k:
            q = qr(matrix[:, pivots_local[:k]], mode="economic")[0]
            res = matrix - q @ (q.T @ matrix)
        else:
            res = matrix
        nrm = np.linalg.norm(res, axis=0)
        nrm[pivots_local[:k]] = -1
        top = np.sort(nrm)[::-1]
        gaps.append((top[0] - top[1]) / top[0])
    return np.array(gaps)


@pytest.mark.parametrize("axes,weights_", [([0], None), ([0, 1, 3], [1.0, 0.5, 2.0])])
def test_dense_pivots_match_lapack_small_water(water, mpi, axes, weights_):
    mol, pts, w, c, sel, oc = water
    pts_s, w_s = pts[::40], w[::40].copy()
    w_s[5] = -abs(w_s[5])
    scales = O.axis_scales(oc, pts_s, w_s, axes, weights_)
    expected = O.select_qrcp_dense(oc, pts_s, w_s, axes, max_rank=12, scales=scales)
    axt = [mpi.AxisType(a) for a in axes]
    got = sel.select(pts_s, w_s, axt, max_rank=12, axis_weights=weights_ or [])
    mask = w_s != 0
    keep = np.flatnonzero(mask)
    matrix = O.pair_matrix(oc.axis_features(pts_s[mask], axes, scales), w_s[mask])
    gaps = _greedy_gaps(matrix, np.searchsorted(keep, expected))
    for i, (a, b) in enumerate(zip(got, expected)):
        if a != b:
            assert gaps[i] <= 1e-10, (i, a, b, gaps[i])
            break
    online = sel.select(pts_s, w_s, axt, max_rank=12, axis_weights=weights_ or [],
                        algorithm=mpi.LocalAnchorSelectionAlgorithm.OnlineQRColumnPivoting,
                        batch_size=64)
    assert online == got


def test_rand_sketch_matches_oracle_small_water(water, mpi):
    mol, pts, w, c, sel, oc = water
    algo = mpi.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao
    for axes, aw in (([0], None), ([0, 1, 2, 3], [1.0, 0.5, 0.5, 0.5])):
        scales = O.axis_scales(oc, pts, w, axes, aw)
        ref, det = O.select_rand_sketch(oc, pts, w, axes, max_rank=8, oversampling=4, seed=2,
                                        scales=scales, return_details=True)
        got = sel.select(pts, w, [mpi.AxisType(a) for a in axes], algorithm=algo, max_rank=8,
                         oversampling=4, seed=2, axis_weights=aw or [])
        assert got == ref, (got, ref)


# ---------------------------------------------------------------------------
# fit and pair error
# ---------------------------------------------------------------------------
def test_fit_matches_literal_refit_and_error(water, mpi):
    mol, pts, w, c, sel, oc = water
    pts_s, w_s = pts[::11], w[::11]
    piv = sel.select(pts_s, w_s, mpi.AxisType.AtomicOrbital, max_rank=8)
    res = mpi.fit(c, pts_s, w_s, np.array(piv))
    keep = w_s != 0
    ao = oc.eval_ao(pts_s[keep])
    anchor_ao = oc.eval_ao(pts_s[piv])
    pairs = (anchor_ao[:, :, None] * anchor_ao[:, None, :]).reshape(len(piv), -1)
    theta, diag = O.physical_pair_refit(pairs, w_s[piv], ao)
    cond = diag["condition"]
    tol = max(1e-10, 1e-15 * cond ** 2)
    th = res["interp_vecs"]
    assert th.shape == theta.shape
    np.testing.assert_allclose(th, theta, rtol=tol, atol=tol * np.abs(theta).max())
    assert res["retained_rank"] == diag["retained_rank"]
    np.testing.assert_allclose(res["condition"], cond, rtol=1e-6)
    products = (ao[:, :, None] * ao[:, None, :]).reshape(len(ao), -1)
    err = O.pair_space_error_norms(products, pairs, w_s[piv], theta, w_s[keep])
    np.testing.assert_allclose(res["pair_l2"], err["l2"], rtol=1e-9)
    np.testing.assert_allclose(res["pair_relative"], err["relative"], rtol=1e-9)
    np.testing.assert_allclose(res["theta_w"], theta @ w_s[keep], rtol=1e-9,
                               atol=1e-9 * np.abs(theta @ w_s[keep]).max())


def test_pair_error_terms_known_answer():
    """python/test/test_isdf.py:157-164 through the C-ABI reduction kernel."""
    import torch
    from mp_isdf_b200 import capi
    exact = np.array([[1., 2.], [3., 4.]])
    anchor = np.array([[1., 0.]])
    theta = np.array([[1., 3.]])
    aw = np.array([1.])
    wg = np.array([2., -1.])
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    q = t(np.linalg.norm(exact, axis=1))
    H = t(exact @ anchor.T)
    X = t((theta * aw[:, None]).T)
    M = t(anchor @ anchor.T)
    e = capi.pair_error_terms(q, H, X, M, t(wg))
    np.testing.assert_allclose(e["l2"], np.sqrt(24.), rtol=1e-14)
    np.testing.assert_allclose(e["relative"], np.sqrt(24. / 35.), rtol=1e-14)


# ---------------------------------------------------------------------------
# error paths
# ---------------------------------------------------------------------------
def test_error_paths(water, mpi):
    mol, pts, w, c, sel, oc = water
    axis = mpi.AxisType.AtomicOrbital
    p, ww = pts[:50].copy(), w[:50].copy()
    bad = ww.copy(); bad[3] = np.nan
    with pytest.raises(ValueError):
        sel.select(p, bad, axis)
    badp = p.copy(); badp[np.flatnonzero(ww)[0], 1] = np.inf
    with pytest.raises(ValueError):
        sel.select(badp, ww, axis)
    with pytest.raises(ValueError):
        sel.select(p, ww, axis, space="invalid")
    with pytest.raises(ValueError):
        sel.select(p, ww, [axis, mpi.AxisType.AtomicOrbitalGradX], axis_weights=[1.0])
    for f in ([0., 1.], [np.nan, 1.], [np.inf, 1.]):
        with pytest.raises(ValueError):
            sel.select(p, ww, [axis, mpi.AxisType.AtomicOrbitalGradX], axis_weights=f)
    with pytest.raises(ValueError):
        sel.select(p, ww, axis, algorithm=mpi.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao,
                   max_rank=10 ** 6, oversampling=4)
    with pytest.raises(ValueError):
        sel.select(np.empty((0, 3)), np.empty(0), mpi.AxisType.OccupiedOrbital)
    with pytest.raises(RuntimeError):
        mpi.DistributedAnchorSelection(c).select(p, ww, axis)
    with pytest.raises(NotImplementedError):
        sel.select(p, ww, axis, algorithm=mpi.LocalAnchorSelectionAlgorithm.CentroidalVoronoi,
                   max_rank=2)
    assert sel.select(p, np.zeros(50), axis) == []
