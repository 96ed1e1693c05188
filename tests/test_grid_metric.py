"""Grid Coulomb metric of the interpolation vectors (grid_coulomb_metric and
grid_cross_metric, python/isdf.py:48-97) and the ISDF J/K build that consumes
it (:130-151).

CPU: the oracle restatement against a literal double loop over grid pairs.
GPU: the library's FP64 all-pairs kernel through the C-ABI (host and device
buffers) and the drop-in module against the oracle, within rtol 1e-11 of the
largest entry (FP64 summation order); one-set and cross forms, coincident
points, every instantiated width; the driver's metric and J/K."""
import numpy as np
import pytest

from oracle import oracle as O


def _literal_metric(left, right, c, w):
    out = np.zeros((len(left), len(right)))
    for g in range(len(w)):
        for h in range(len(w)):
            if g == h:
                kern = O.C_SPHERE * abs(w[g]) ** (-1.0 / 3.0)
            else:
                r = np.linalg.norm(c[g] - c[h])
                kern = 0.0 if r == 0 else 1.0 / r
            out += np.outer(left[:, g] * w[g], right[:, h] * w[h]) * kern
    return out


def test_oracle_metric_matches_literal_pairs():
    rng = np.random.default_rng(0)
    n = 40
    c = rng.normal(size=(n, 3))
    c[5] = c[7]                         # coincident points contribute nothing
    w = rng.uniform(-1.0, 1.0, n)
    left, right = rng.normal(size=(3, n)), rng.normal(size=(4, n))
    lit = _literal_metric(left, right, c, w)
    np.testing.assert_allclose(O.grid_cross_metric(left, right, c, w, block=7), lit, rtol=1e-12, atol=1e-12)
    sym = _literal_metric(left, left, c, w)
    np.testing.assert_allclose(O.grid_coulomb_metric(left, c, w), 0.5 * (sym + sym.T), rtol=1e-12, atol=1e-12)


def test_oracle_jk_symmetric():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(6, 9))
    z = rng.normal(size=(6, 6))
    z = z @ z.T
    dm = rng.normal(size=(9, 9))
    dm = dm + dm.T
    j, k = O.isdf_jk(x, z, dm)
    assert np.allclose(j, j.T) and np.allclose(k, k.T)
    # J from the factorised integrals (mu nu|lam sig) ~ sum_pq X X Z X X
    eri = np.einsum("pm,pn,pq,ql,qs->mnls", x, x, z, x, x)
    np.testing.assert_allclose(j, np.einsum("mnls,ls->mn", eri, dm), rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(k, 0.5 * (np.einsum("mlns,ls->mn", eri, dm) + np.einsum("mlns,ls->mn", eri, dm).T),
                               rtol=1e-10, atol=1e-10)


@pytest.fixture(scope="module")
def grid():
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((2, 1, 1), seed=2)
    pts, w = inputs.becke_grid(symbols, xyz, level=0)
    keep = w != 0
    pts, w = pts[keep][::2].copy(), w[keep][::2].copy()
    pts[11] = pts[10]                   # a coincident pair
    return pts, w


def _close(got, ref):
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("k", [3, 7, 10, 13, 20, 30, 40, 64])
def test_grid_metric_matches_oracle(grid, k):
    from mp_isdf_b200 import capi
    pts, w = grid
    theta = np.random.default_rng(k).normal(size=(k, len(w)))
    ref = O.grid_coulomb_metric(theta, pts, w)
    got = capi.grid_metric_host(theta, pts, w)
    _close(got, ref)
    assert np.array_equal(got, got.T)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [37, 129, 1000, 4097])
@pytest.mark.parametrize("k", [5, 17, 40])
def test_one_set_half_pairs_form(grid, n, k):
    """One set on both sides sums half the pairs (tiles above the diagonal, the
    diagonal tile at weight 1/2); the same values in two buffers take the full
    sum and (V + V^T)/2.  Both equal the oracle: grids smaller than a row block,
    ragged tile edges, k across the column-block widths."""
    import torch
    from mp_isdf_b200 import capi
    from mp_isdf_b200 import inputs
    pts, w = grid
    rng = np.random.default_rng(n + k)
    sel = np.sort(rng.choice(len(w), size=min(n, len(w)), replace=False))
    sel[1] = sel[0]                     # a coincident pair
    p, ww = pts[sel].copy(), w[sel].copy()
    theta = rng.normal(size=(k, len(ww)))
    ref = O.grid_coulomb_metric(theta, p, ww)
    symbols, xyz = inputs.water_cluster((1, 1, 1), seed=0)
    mol = inputs.build_tables(symbols, xyz)
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(p, device="cuda")
    wt = torch.tensor(ww, device="cuda")
    lt = torch.tensor(theta, device="cuda")
    half = ctx.grid_metric(x, wt, lt)
    _close(half, ref)
    assert np.array_equal(half, half.T)
    copy = lt.clone()
    full = np.empty((k, k))
    capi.check(capi.lib().isdf_grid_metric(ctx.h, capi._ptr(lt), lt.stride(0), k, capi._ptr(copy), copy.stride(0),
                                           k, capi._ptr(x), capi._ptr(wt), len(ww), 1, capi._ptr(full),
                                           capi._stream(x)))
    _close(full, ref)
    np.testing.assert_allclose(half, full, rtol=1e-12, atol=1e-12 * np.abs(full).max())


@pytest.mark.gpu
def test_grid_cross_metric_device_and_module(grid):
    import torch
    import mp_isdf
    from mp_isdf_b200 import capi
    from mp_isdf_b200 import inputs
    pts, w = grid
    rng = np.random.default_rng(3)
    left, right = rng.normal(size=(5, len(w))), rng.normal(size=(9, len(w)))
    ref = O.grid_cross_metric(left, right, pts, w)
    _close(capi.grid_metric_host(left, pts, w, right=right), ref)
    _close(mp_isdf.grid_cross_metric(left, right, pts, w), ref)
    _close(mp_isdf.grid_coulomb_metric(left, pts, w), O.grid_coulomb_metric(left, pts, w))
    # device buffers with a leading dimension larger than the grid
    symbols, xyz = inputs.water_cluster((1, 1, 1), seed=0)
    mol = inputs.build_tables(symbols, xyz)
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    wide = torch.zeros((9, len(w) + 5), dtype=torch.float64, device="cuda")
    wide[:, :len(w)] = torch.tensor(right, device="cuda")
    lt = torch.tensor(left, device="cuda")
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    _close(ctx.grid_metric(x, wt, lt, wide[:, :len(w)]), ref)
    with pytest.raises(ValueError):
        mp_isdf.grid_coulomb_metric(rng.normal(size=(65, len(w))), pts, w)
    with pytest.raises(ValueError):
        mp_isdf.grid_coulomb_metric(left[:, :-1], pts, w)


@pytest.mark.gpu
def test_driver_metric_and_jk(grid):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "python"))
    import isdf
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((2, 1, 1), seed=2)
    t = inputs.build_tables(symbols, xyz)
    M = isdf.Molecule(t.atm, t.bas, t.env, t.coords, t.symbols)
    pts, w = grid
    res = isdf.build_isdf(M, anchor_rank=8, anchor_algorithm="qrcp_dense", grid=(pts, w), compute_metric=True)
    raw = O.grid_coulomb_metric(res["interp_vecs"], res["coordinates"], res["weights"])
    ref = res["anchor_weights"][:, None] * raw * res["anchor_weights"][None, :]
    _close(res["coulomb_metric"], ref)
    dm = np.random.default_rng(4).normal(size=(t.nao, t.nao))
    dm = dm + dm.T
    j, k = isdf.evaluate_isdf_jk(res, dm)
    jr, kr = O.isdf_jk(res["X1"], ref, dm)
    np.testing.assert_allclose(j, jr, rtol=1e-9, atol=1e-9 * np.abs(jr).max())
    np.testing.assert_allclose(k, kr, rtol=1e-9, atol=1e-9 * np.abs(kr).max())
    with pytest.raises(NotImplementedError):
        isdf.build_isdf(M, anchor_rank=8, grid=(pts, w), compute_metric=True, metric_algorithm="unblocked_greedy")
    with pytest.raises(ValueError, match="symmetric"):
        isdf.evaluate_isdf_jk(res, dm + np.triu(np.ones_like(dm), 1))


@pytest.mark.gpu
def test_isdf_jk_device_matches_oracle():
    """mp_isdf.isdf_jk (FP64 tensor-core GEMMs on the device) against the
    oracle's NumPy restatement of evaluate_isdf_jk (python/isdf.py:130-151),
    for anchor counts 1, 8, 37 (ragged GEMM tiles) and the device C-ABI."""
    import ctypes
    import mp_isdf
    import torch
    from mp_isdf_b200 import capi, inputs
    symbols, xyz = inputs.water_cluster((2, 1, 1), seed=2)
    t = inputs.build_tables(symbols, xyz)
    c = mp_isdf.LibcintContext(t.atm, t.bas, t.env)
    rng = np.random.default_rng(9)
    for k in (1, 8, 37):
        x = rng.normal(size=(k, t.nao))
        z = rng.normal(size=(k, k))
        z = z + z.T
        dm = rng.normal(size=(t.nao, t.nao))
        dm = dm + dm.T
        j, kk = mp_isdf.isdf_jk(c, x, z, dm)
        jr, kr = O.isdf_jk(x, z, dm)
        np.testing.assert_allclose(j, jr, rtol=1e-12, atol=1e-12 * np.abs(jr).max())
        np.testing.assert_allclose(kk, kr, rtol=1e-12, atol=1e-12 * np.abs(kr).max())
        assert np.array_equal(j, j.T) and np.array_equal(kk, kk.T)
    # device pointers through the C-ABI, K only
    ctx = capi.Context(t.atm, t.bas, t.env)
    dx, dz, dd = (torch.tensor(a, device="cuda") for a in (x, z, dm))
    kd = torch.empty(t.nao, t.nao, dtype=torch.float64, device="cuda")
    P = ctypes.c_void_p
    capi.check(capi.lib().isdf_jk(ctx.h, P(dx.data_ptr()), len(x), P(dz.data_ptr()), P(dd.data_ptr()), None,
                                  P(kd.data_ptr()), P(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    np.testing.assert_allclose(kd.cpu().numpy(), kr, rtol=1e-12, atol=1e-12 * np.abs(kr).max())
    with pytest.raises(ValueError):
        mp_isdf.isdf_jk(c, x[:, :-1], z, dm)
