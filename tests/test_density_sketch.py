"""AO-density Khatri-Rao sketches (RandomizedAODensityKhatriRao and its
column-normalized form, cpp/src/anchor_select_randomized_id.cpp:104-118,
131-146, 231-309): candidates are the points with nonzero weight and nonzero
importance whose squared AO norm exceeds the screening threshold; the sketch
column of point g is sqrt(m_g)/sqrt(ell) (f.u_s)(f.v_s), f = phi_g or
phi_g/|phi_g|.

CPU: the oracle against its own quadrature sketch (importance = |w| makes the
two sketches identical) and its validation.  GPU: anchors through the C-ABI
(device and host buffers) and the drop-in module equal to the oracle's,
exactly, as for the quadrature sketch; screening and zero importances; the
reference's error behaviour."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def cluster():
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((2, 1, 1), seed=11)
    mol = inputs.build_tables(symbols, xyz)
    pts, w = inputs.becke_grid(symbols, xyz, level=0)
    rng = np.random.default_rng(5)
    importance = np.abs(w) * rng.uniform(0.0, 2.0, len(w))
    importance[rng.uniform(size=len(w)) < 0.2] = 0.0          # zero-importance points
    return mol, pts, w, importance, O.OracleContext(mol.atm, mol.bas, mol.env)


def test_oracle_density_with_weight_importance_is_the_quadrature_sketch(cluster):
    mol, pts, w, _, oc = cluster
    dens = O.select_density_sketch(oc, pts, w, np.abs(w), max_rank=8, oversampling=6, seed=3,
                                   ao_screening_threshold=0.0)
    quad = O.select_rand_sketch(oc, pts, w, [0], max_rank=8, oversampling=6, seed=3)
    assert dens == quad


def test_oracle_density_validation(cluster):
    mol, pts, w, m, oc = cluster
    with pytest.raises(ValueError, match="shape"):
        O.select_density_sketch(oc, pts, w, m[:-1], max_rank=4)
    bad = m.copy()
    bad[3] = -1.0
    with pytest.raises(ValueError, match="finite and nonnegative"):
        O.select_density_sketch(oc, pts, w, bad, max_rank=4)
    with pytest.raises(ValueError, match="threshold"):
        O.select_density_sketch(oc, pts, w, m, max_rank=4, ao_screening_threshold=-1.0)
    with pytest.raises(ValueError, match="eligible candidates"):
        O.select_density_sketch(oc, pts, w, np.zeros_like(m), max_rank=4)
    assert O.select_density_sketch(oc, pts, w, np.zeros_like(m)) == []


ALGOS = {False: "rand_sketch_density", True: "rand_sketch_density_col_norm"}


def _screen_threshold(oc, pts, w, m, fraction):
    """A threshold that screens about `fraction` of the candidates."""
    keep = (w != 0) & (m != 0)
    ao = oc.eval_ao(pts[keep])
    q = np.einsum("ga,ga->g", ao, ao)
    return float(np.quantile(q, fraction))


@pytest.mark.gpu
@pytest.mark.parametrize("normalized", [False, True])
@pytest.mark.parametrize("fraction", [0.0, 0.3])
def test_density_sketch_matches_oracle(cluster, normalized, fraction):
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w, m, oc = cluster
    thr = 1e-24 if fraction == 0.0 else _screen_threshold(oc, pts, w, m, fraction)
    ref = O.select_density_sketch(oc, pts, w, m, normalized=normalized, max_rank=8, oversampling=6,
                                  seed=3, ao_screening_threshold=thr)
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    kw = dict(algorithm=ALGOS[normalized], axes=("ao",), max_rank=8, oversampling=6, seed=3,
              ao_screening_threshold=thr)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    mt = torch.tensor(m, device="cuda")
    piv, info = ctx.select(x, wt, point_importance=mt, **kw)
    assert piv.tolist() == ref
    assert np.all(m[piv] > 0) and np.all(w[piv] != 0)
    piv_h, _ = ctx.select_host(pts, w, point_importance=m, **kw)
    assert piv_h.tolist() == ref
    # tolerance mode (rank from the sketch tails)
    ref_t = O.select_density_sketch(oc, pts, w, m, normalized=normalized, tolerance=1e-3, sketch_size=24,
                                    oversampling=6, seed=3, ao_screening_threshold=thr)
    kt = dict(kw, max_rank=0, sketch_size=24, tolerance=1e-3)
    assert ctx.select_host(pts, w, point_importance=m, **kt)[0].tolist() == ref_t


@pytest.mark.gpu
def test_density_sketch_dropin_module(cluster):
    import mp_isdf
    mol, pts, w, m, oc = cluster
    c = mp_isdf.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mp_isdf.AnchorSelection(c)
    for normalized, algo in ((False, mp_isdf.LocalAnchorSelectionAlgorithm.RandomizedAODensityKhatriRao),
                             (True, mp_isdf.LocalAnchorSelectionAlgorithm.RandomizedAODensityNormalizedKhatriRao)):
        ref = O.select_density_sketch(oc, pts, w, m, normalized=normalized, max_rank=6, oversampling=6, seed=9)
        got = sel.select(pts, w, mp_isdf.AxisType.AtomicOrbital, max_rank=6, oversampling=6, seed=9,
                         algorithm=algo, point_importance=m)
        assert got == ref


@pytest.mark.gpu
def test_density_sketch_errors(cluster):
    import mp_isdf
    from mp_isdf_b200 import capi
    mol, pts, w, m, oc = cluster
    c = mp_isdf.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mp_isdf.AnchorSelection(c)
    algo = mp_isdf.LocalAnchorSelectionAlgorithm.RandomizedAODensityKhatriRao
    ao = mp_isdf.AxisType.AtomicOrbital
    with pytest.raises(ValueError, match="shape"):
        sel.select(pts, w, ao, max_rank=4, algorithm=algo)
    with pytest.raises(ValueError, match="shape"):
        sel.select(pts, w, ao, max_rank=4, algorithm=algo, point_importance=m[:-1])
    bad = m.copy()
    bad[0] = np.nan
    with pytest.raises(ValueError, match="finite and nonnegative"):
        sel.select(pts, w, ao, max_rank=4, algorithm=algo, point_importance=bad)
    with pytest.raises(ValueError, match="non-AO"):
        sel.select(pts, w, [ao, mp_isdf.AxisType.AtomicOrbitalGradX], max_rank=4, algorithm=algo,
                   point_importance=m)
    with pytest.raises(ValueError, match="threshold"):
        sel.select(pts, w, ao, max_rank=4, algorithm=algo, point_importance=m, ao_screening_threshold=-1.0)
    with pytest.raises(ValueError, match="eligible candidates"):
        sel.select(pts, w, ao, max_rank=4, algorithm=algo, point_importance=np.zeros_like(m))
    assert sel.select(pts, w, ao, algorithm=algo, point_importance=np.zeros_like(m)) == []
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    with pytest.raises(capi.IsdfError, match="FP64 form"):
        ctx.select_host(pts, w, algorithm="rand_sketch_density", max_rank=4, point_importance=m,
                        precision="mixed")


@pytest.mark.gpu
def test_build_isdf_density_col_norm_and_normalized_pair_error(cluster):
    """The driver's density path: anchors equal to the oracle's, and its
    density-normalized pair error (Gram form) equal to the reference's literal
    per-point pair formation (python/isdf.py:266-287)."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "python"))
    import isdf
    mol, pts, w, m, oc = cluster
    M = isdf.Molecule(mol.atm, mol.bas, mol.env, mol.coords, mol.symbols)
    thr = _screen_threshold(oc, pts, w, m, 0.1)
    res = isdf.build_isdf(M, anchor_rank=6, anchor_algorithm="rand_sketch", sketch="density_col_norm",
                          anchor_oversampling=6, anchor_seed=9, grid=(pts, w), point_importance=m,
                          ao_screening_threshold=thr, pair_space_error=True)
    ref = O.select_density_sketch(oc, pts, w, m, normalized=True, max_rank=6, oversampling=6, seed=9,
                                  ao_screening_threshold=thr)
    assert list(res["anchor_indices"]) == ref
    keep = w != 0
    ao = oc.eval_ao(pts[keep])
    a_ao = oc.eval_ao(pts[ref])
    pairs_a = np.einsum("ka,kb->kab", a_ao, a_ao).reshape(len(ref), -1)
    coeff = (w[ref][:, None] * res["interp_vecs"]).T
    mm = m[keep]
    residual = total = screened = 0.0
    for row, mg, c in zip(ao, mm, coeff):
        q = row @ row
        if q <= thr:
            screened += mg
            continue
        if mg == 0:
            continue
        exact = np.outer(row, row).ravel()
        residual += mg * np.sum(((exact - c @ pairs_a) / q) ** 2)
        total += mg
    got = res["pair_space_errors"]["density_normalized"]
    np.testing.assert_allclose(got["relative"], np.sqrt(residual / total), rtol=1e-8)
    np.testing.assert_allclose(got["l2"], np.sqrt(residual), rtol=1e-8)
    np.testing.assert_allclose(got["included_mass"], total, rtol=1e-12)
    np.testing.assert_allclose(got["screened_mass"], screened, rtol=1e-12)
    with pytest.raises(NotImplementedError, match="point_importance"):
        isdf.build_isdf(M, anchor_rank=6, anchor_algorithm="rand_sketch", sketch="density", grid=(pts, w))
    with pytest.raises(ValueError, match="requires CVT or a density sketch"):
        isdf.build_isdf(M, anchor_rank=6, anchor_algorithm="rand_sketch", grid=(pts, w), point_importance=m)
