"""The OccupiedOrbital axis (cpp/src/anchor_select.cpp:18-52,
cpp/include/anchor_select_impl.hpp:55-77): features psi_j = sum_mu phi_mu C[mu][j]
for j < nocc with row-major (nao, nao) MO coefficients C, alone or beside the AO
and gradient axes, in evaluate_axis, qrcp_dense / qrcp_online and the quadrature
sketch (FP64; a mixed rand_sketch request with an occupied entry runs in FP64).

CPU: the oracle's occupied features against the AO axis (C = I, nocc = nao).
GPU: features within the AO tolerance (rtol 1e-11, atol 1e-12) and anchors
equal to the oracle's over the same features."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def water():
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((1, 1, 1), seed=3)
    mol = inputs.build_tables(symbols, xyz)
    pts, w = inputs.becke_grid(symbols, xyz, level=0)
    rng = np.random.default_rng(8)
    q, _ = np.linalg.qr(rng.normal(size=(mol.nao, mol.nao)))
    return mol, pts, w, np.ascontiguousarray(q), 5, O.OracleContext(mol.atm, mol.bas, mol.env)


def test_oracle_occupied_identity_is_the_ao_axis(water):
    mol, pts, w, _, _, oc = water
    eye = np.eye(mol.nao)
    np.testing.assert_array_equal(O.occ_features(oc, pts[:40], [4], eye, mol.nao), oc.eval_ao(pts[:40]))
    np.testing.assert_allclose(O.occ_axis_scales(oc, pts, w, [0, 4], eye, mol.nao),
                               O.axis_scales(oc, pts, w, [0, 0]), rtol=1e-12)
    with pytest.raises(ValueError, match="OccupiedOrbital"):
        O.occ_features(oc, pts[:4], [4], None, 0)


@pytest.mark.gpu
def test_occupied_features_match_oracle(water):
    import mp_isdf
    from mp_isdf_b200 import capi
    mol, pts, w, mo, nocc, oc = water
    p = pts[::7]
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    for axes in ([4], [0, 4, 1], [4, 3, 4]):
        got = ctx.evaluate_axis_host(p, axes, mo, nocc)
        ref = O.occ_features(oc, p, axes, mo, nocc)
        np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-12)
    c = mp_isdf.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mp_isdf.AnchorSelection(c)
    T = mp_isdf.AxisType
    got = sel.evaluate_axis(p, [T.AtomicOrbital, T.OccupiedOrbital], mo_coeff=mo, nocc=nocc)
    np.testing.assert_allclose(got, O.occ_features(oc, p, [0, 4], mo, nocc), rtol=1e-11, atol=1e-12)
    with pytest.raises(ValueError, match="OccupiedOrbital"):
        sel.evaluate_axis(p, T.OccupiedOrbital)
    with pytest.raises(ValueError, match="OccupiedOrbital"):
        sel.evaluate_axis(p, T.OccupiedOrbital, mo_coeff=mo, nocc=mol.nao + 1)


@pytest.mark.gpu
@pytest.mark.parametrize("axes", [[4], [0, 4]])
def test_occupied_rand_sketch_matches_oracle(water, axes):
    import mp_isdf
    mol, pts, w, mo, nocc, oc = water
    keep = np.flatnonzero(w != 0)
    scales = O.occ_axis_scales(oc, pts, w, axes, mo, nocc)
    f = O.occ_features(oc, pts[keep], axes, mo, nocc, scales)
    ref = O.select_rand_sketch_features(f, keep, w[keep], ell=6 + 6, oversampling=6, seed=5, max_rank=6)
    c = mp_isdf.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mp_isdf.AnchorSelection(c)
    T = mp_isdf.AxisType
    ax = [T(a) for a in axes]
    algo = mp_isdf.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao
    got = sel.select(pts, w, ax, algorithm=algo, max_rank=6, oversampling=6, seed=5, mo_coeff=mo, nocc=nocc)
    assert got == ref
    # a mixed request with an occupied entry runs the FP64 form
    assert sel.select(pts, w, ax, algorithm=algo, max_rank=6, oversampling=6, seed=5, mo_coeff=mo, nocc=nocc,
                      precision="mixed") == ref


@pytest.mark.gpu
def test_occupied_dense_and_online_qrcp(water):
    import mp_isdf
    mol, pts, w, mo, nocc, oc = water
    pts_s, w_s = pts[::13], w[::13]
    axes = [0, 4]
    keep = np.flatnonzero(w_s != 0)
    scales = O.occ_axis_scales(oc, pts_s, w_s, axes, mo, nocc)
    f = O.occ_features(oc, pts_s[keep], axes, mo, nocc, scales)
    ref = O.select_qrcp_dense_features(f, keep, max_rank=8, w=w_s[keep])
    c = mp_isdf.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mp_isdf.AnchorSelection(c)
    T = mp_isdf.AxisType
    ax = [T.AtomicOrbital, T.OccupiedOrbital]
    got = sel.select(pts_s, w_s, ax, max_rank=8, mo_coeff=mo, nocc=nocc)
    assert got == ref
    online = sel.select(pts_s, w_s, ax, max_rank=8, mo_coeff=mo, nocc=nocc, batch_size=64,
                        algorithm=mp_isdf.LocalAnchorSelectionAlgorithm.OnlineQRColumnPivoting)
    assert online == got
    with pytest.raises(ValueError, match="OccupiedOrbital"):
        sel.select(pts_s, w_s, ax, max_rank=8)
