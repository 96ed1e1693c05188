"""RBRP (robust blockwise random pivoting over AO pair rows) and its ID
(rbrp_ao_cpu / rbrp_ao_device, cpp/src/anchor_select_rbrp.cpp:136-320).

The oracle restates the reference with explicit pair rows, LAPACK dgeqp3 /
dorgqr (scipy) and the reference's sampler (std::discrete_distribution over
std::mt19937_64, from the oracle's C++).  GPU: the library's run over the same
AO rows gives the same anchors, stopping status and block history, and the ID
(interpolation vectors and pair transform) within 1e-8 relative."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def rows():
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((1, 1, 1), seed=3)
    mol = inputs.build_tables(symbols, xyz)
    pts, w = inputs.becke_grid(symbols, xyz, level=0)
    keep = w != 0
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    p, ww = pts[keep][::3].copy(), w[keep][::3].copy()
    return mol, p, ww, oc.eval_ao(p)


def test_oracle_rbrp_id_reconstructs_the_chosen_rows(rows):
    mol, p, w, ao = rows
    r = O.rbrp_ao(ao, w, max_rank=12, block_size=6, compute_id=True)
    idx = np.array(r["indices"])
    assert len(idx) == 12 and len(set(idx)) == 12
    th = r["interp_vecs"]
    np.testing.assert_allclose(th[:, idx], np.diag(1.0 / w[idx]), rtol=0, atol=0)   # cardinality
    assert r["history"][-1][0] == 12
    with pytest.raises(ValueError, match="nonzero weights"):
        O.rbrp_ao(ao, np.where(np.arange(len(w)) == 3, 0.0, w))


CASES = [dict(max_rank=20, block_size=8), dict(tolerance=0.08, block_size=16),
         dict(max_rank=15, block_size=4, refresh_every=0), dict(max_rank=10, block_size=5, tau_block=0.0, seed=11)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_rbrp_matches_oracle(rows, case):
    from mp_isdf_b200 import capi
    mol, p, w, ao = rows
    kw = CASES[case]
    ref = O.rbrp_ao(ao, w, compute_id=True, **kw)
    got = capi.rbrp_ao(ao, w, compute_id=True, **kw)
    assert got["indices"].tolist() == ref["indices"]
    assert got["status"] == ref["status"]
    np.testing.assert_allclose(got["relative_residual"], ref["relative_residual"], rtol=1e-8)
    np.testing.assert_allclose(got["history"], ref["history"], rtol=1e-8, atol=1e-12)
    assert got["retained_rank"] == ref["retained_rank"]
    np.testing.assert_allclose(got["condition"], ref["condition"], rtol=1e-6)
    scale = max(1.0, ref["condition"])
    for key in ("interp_vecs", "transform"):
        r = ref[key]
        np.testing.assert_allclose(got[key], r, rtol=0, atol=1e-9 * scale * np.abs(r).max())


@pytest.mark.gpu
def test_rbrp_dropin_module(rows):
    import mp_isdf
    mol, p, w, ao = rows
    ref = O.rbrp_ao(ao, w, max_rank=12, block_size=6, compute_id=True)
    got = mp_isdf.rbrp_ao_cpu(ao, w, max_rank=12, block_size=6, compute_id=True)
    assert got["indices"] == ref["indices"]
    assert set(got) == {"indices", "relative_residual", "status", "condition", "retained_rank", "history",
                        "interp_vecs", "transform"}
    c = mp_isdf.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mp_isdf.AnchorSelection(c)
    dev = mp_isdf.rbrp_ao_device(sel, p, w, max_rank=12, block_size=6)
    assert dev["indices"] == ref["indices"] and "interp_vecs" not in dev
    with pytest.raises(ValueError, match="nonzero weights"):
        mp_isdf.rbrp_ao_cpu(ao, np.where(np.arange(len(w)) == 3, 0.0, w))
    with pytest.raises(ValueError, match="tolerances"):
        mp_isdf.rbrp_ao_cpu(ao, w, tolerance=-1.0)
    with pytest.raises(ValueError):
        mp_isdf.rbrp_ao_cpu(ao[:, :3], w[:-1])


@pytest.mark.gpu
def test_driver_rbrp_and_rbrp_id(rows):
    """The driver's rbrp (anchors, then the usual fit) and rbrp_id (the ID is the
    fit) against the oracle; the ID's pair error in the Gram form equals the
    literal one of its Theta."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "python"))
    import isdf
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((1, 1, 1), seed=3)
    t = inputs.build_tables(symbols, xyz)
    M = isdf.Molecule(t.atm, t.bas, t.env, t.coords, t.symbols)
    mol, p, w, ao = rows
    ref = O.rbrp_ao(ao, w, max_rank=10, block_size=5, compute_id=True)
    res = isdf.build_isdf(M, anchor_rank=10, anchor_algorithm="rbrp", rbrp_block_size=5, grid=(p, w))
    assert res["anchor_indices"].tolist() == ref["indices"]
    rid = isdf.build_isdf(M, anchor_rank=10, anchor_algorithm="rbrp_id", rbrp_block_size=5, grid=(p, w),
                          pair_space_error=True)
    assert rid["anchor_indices"].tolist() == ref["indices"]
    th = rid["interp_vecs"]
    np.testing.assert_allclose(th, ref["interp_vecs"], rtol=0,
                               atol=1e-9 * max(1.0, ref["condition"]) * np.abs(ref["interp_vecs"]).max())
    idx = np.array(ref["indices"])
    pa = np.einsum("ka,kb->kab", ao[idx], ao[idx]).reshape(len(idx), -1)
    pg = np.einsum("ga,gb->gab", ao, ao).reshape(len(ao), -1)
    resid = pg - (th * w[idx][:, None]).T @ pa
    lit = np.sqrt(np.sum(np.abs(w)[:, None] * resid ** 2))
    got = rid["pair_space_errors"]["scalar"]["l2"]
    np.testing.assert_allclose(got, lit, rtol=1e-6)
    with pytest.raises(ValueError, match="axes"):
        isdf.build_isdf(M, anchor_rank=10, anchor_algorithm="rbrp", axes=("ao", "dx"), grid=(p, w))
