"""Mixed-precision form (FP32 AO values, split-BF16 tcgen05 projections, FP64
QRCP with exact re-verification of near-tie columns, FP64 solve) against the
FP64 form and the oracle.  Criteria: anchors identical to the FP64 path's;
pair-space error of the mixed Theta (evaluated with FP64 AO values) within
1e-8 relative of the FP64 fit's; Theta within 1e-4 relative."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mpi():
    import mp_isdf
    return mp_isdf


@pytest.fixture(scope="module")
def c1(mpi):
    from mp_isdf_b200 import inputs
    mol, pts, w, cfg = inputs.make_config("c1")
    c = mpi.LibcintContext(mol.atm, mol.bas, mol.env)
    return mol, pts, w, c, mpi.AnchorSelection(c)


@pytest.mark.parametrize("axes,aw,rank,ovs", [
    ([0], None, 8, 4),
    ([0, 1, 2, 3], [1.0, 0.5, 0.5, 0.5], 8, 4),
    ([0, 1, 2, 3], None, 10, 16),
    ([0, 3], [1.0, 2.0], 6, 10),
])
def test_mixed_sketch_pivots_equal_fp64_small(mpi, small_water, axes, aw, rank, ovs):
    mol, pts, w = small_water
    c = mpi.LibcintContext(mol.atm, mol.bas, mol.env)
    sel = mpi.AnchorSelection(c)
    algo = mpi.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao
    axt = [mpi.AxisType(a) for a in axes]
    kw = dict(algorithm=algo, max_rank=rank, oversampling=ovs, seed=2, axis_weights=aw or [])
    fp64 = sel.select(pts, w, axt, precision="fp64", **kw)
    mixed = sel.select(pts, w, axt, precision="mixed", **kw)
    assert mixed == fp64
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    scales = O.axis_scales(oc, pts, w, axes, aw)
    ref = O.select_rand_sketch(oc, pts, w, axes, max_rank=rank, oversampling=ovs, seed=2,
                               scales=scales)
    assert mixed == ref


def test_mixed_sketch_and_fit_c1(mpi, c1):
    mol, pts, w, c, sel = c1
    algo = mpi.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao
    for axes in ([mpi.AxisType.AtomicOrbital],
                 [mpi.AxisType.AtomicOrbital, mpi.AxisType.AtomicOrbitalGradX,
                  mpi.AxisType.AtomicOrbitalGradY, mpi.AxisType.AtomicOrbitalGradZ]):
        kw = dict(algorithm=algo, max_rank=8, oversampling=16, seed=7)
        fp64 = sel.select(pts, w, axes, precision="fp64", **kw)
        mixed = sel.select(pts, w, axes, precision="mixed", **kw)
        assert mixed == fp64
    piv = np.array(fp64)
    f64 = mpi.fit(c, pts, w, piv, precision="fp64")
    mx = mpi.fit(c, pts, w, piv, precision="mixed")
    th64, thm = f64["interp_vecs"], mx["interp_vecs"]
    assert thm.shape == th64.shape
    rel = np.abs(thm - th64).max() / np.abs(th64).max()
    cond = f64["condition"]
    info = (f"theta rel {rel:.3e} cond(C) {cond:.3e} pair {f64['pair_relative']:.12e} "
            f"{mx['pair_relative']:.12e} path {mx['fit_path']} bound {mx['mixed_bound']:.3e}")
    print(info)
    # Theta errors are amplified by cond(C)^2 (the solve with (Phi_a Phi_a^T)^2);
    # the pair error is stationary in Theta and is the acceptance criterion.
    assert rel < 1e-5 * max(1.0, cond) ** 2, info
    assert abs(mx["pair_relative"] - f64["pair_relative"]) <= 1e-8 * f64["pair_relative"], info
    assert abs(mx["pair_l2"] - f64["pair_l2"]) <= 1e-8 * f64["pair_l2"], info


def test_tensor_core_projection_accuracy(small_water):
    """Split-BF16 tcgen05 projection of FP32 AO features vs the FP64 path and
    the oracle: error bounded by 1.5e-4 * |f_g| * |w_j| per entry (the bound
    the verified QR relies on), typically ~1e-5 of it."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    p = pts[::3]
    x = torch.tensor(p, device="cuda")
    rng = np.random.default_rng(0)
    for axes, nout in ((("ao",), 10), (("ao", "dx", "dy", "dz"), 52), (("dz", "ao"), 24)):
        d = len(axes) * mol.nao
        W = rng.normal(size=(d, nout))
        p64 = ctx.project_axes(x, axes, W, "fp64").cpu().numpy()
        pm = ctx.project_axes(x, axes, W, "mixed").cpu().numpy()
        codes = [O.AXIS_CODES[a] for a in axes]
        f = oc.axis_features(p, codes)
        nao = mol.nao
        ref = np.stack([f[:, a * nao:(a + 1) * nao] @ W[a * nao:(a + 1) * nao] for a in range(len(axes))],
                       axis=1)
        np.testing.assert_allclose(p64, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
        fn = np.stack([np.linalg.norm(f[:, a * nao:(a + 1) * nao], axis=1) for a in range(len(axes))], axis=1)
        wn = np.stack([np.linalg.norm(W[a * nao:(a + 1) * nao], axis=0) for a in range(len(axes))])
        bound = fn[:, :, None] * wn[None, :, :] + 1e-300
        ratio = np.abs(pm - ref) / bound
        print(axes, "max err/(|f||w|) =", ratio.max(), "median", np.median(ratio))
        assert ratio.max() < 1.5e-4, ratio.max()


def test_mixed_dense_device_api(small_water):
    """C-ABI device path with torch tensors, mixed precision."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    p64, i64 = ctx.select(x, wt, axes=("ao", "dx", "dy", "dz"), max_rank=8, oversampling=16,
                          precision="fp64")
    pm, im = ctx.select(x, wt, axes=("ao", "dx", "dy", "dz"), max_rank=8, oversampling=16,
                        precision="mixed")
    np.testing.assert_array_equal(pm, p64)
    assert im.verifications >= 1          # the winner of every step is recomputed exactly
    theta = torch.empty(len(pm) * len(pts), dtype=torch.float64, device="cuda")
    info = ctx.fit(x, wt, pm, theta, precision="mixed", want_error=True)
    theta64 = torch.empty_like(theta)
    info64 = ctx.fit(x, wt, pm, theta64, precision="fp64")
    torch.cuda.synchronize()
    print("small water mixed fit path", info.fit_path, "bound", info.mixed_bound)
    assert info.fit_path in (1, 3) and info.mixed_bound <= 1e-8
    assert abs(info.pair_relative - info64.pair_relative) <= 1e-8 * info64.pair_relative


@pytest.mark.parametrize("axes", [("ao",), ("ao", "dx", "dy", "dz"), ("dx", "ao"), ("dz",)])
def test_select_fit_matches_select_then_fit(small_water, axes):
    """isdf_select_fit (selection and fit in one call; in the mixed form the fit
    contracts the AO value tiles the sketch left in HBM) against isdf_select
    followed by isdf_fit on the same device points: identical anchors, the
    same fit path, Theta and the error bound to FP32-evaluation level, and the
    pair-space error within 1e-8 relative of the FP64 fit's.  Without a plain
    AO value axis the sketch keeps no AO tiles, and below 2^28 AO values the
    fused call then fits in FP64 (fit path 0), as isdf_fit in FP64 does."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    kw = dict(axes=axes, max_rank=8, oversampling=16, seed=3)
    for precision in ("mixed", "fp64"):
        piv, _ = ctx.select(x, wt, precision=precision, **kw)
        theta = torch.zeros(len(piv) * len(pts), dtype=torch.float64, device="cuda")
        fit_precision = "fp64" if "ao" not in axes else precision
        info = ctx.fit(x, wt, piv, theta, precision=fit_precision, want_error=True)
        theta2 = torch.zeros(8 * len(pts), dtype=torch.float64, device="cuda")
        piv2, sinfo, info2 = ctx.select_fit(x, wt, theta2, want_error=True, precision=precision, **kw)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(piv2, piv)
        assert info2.n_kept == info.n_kept and info2.fit_path == info.fit_path
        n = len(piv) * info.n_kept
        t1, t2 = theta[:n].cpu().numpy(), theta2[:n].cpu().numpy()
        rel = np.abs(t1 - t2).max() / np.abs(t1).max()
        print(axes, precision, "path", info.fit_path, "bound", info.mixed_bound, info2.mixed_bound,
              "theta rel", rel)
        # FP64 fits differ only by the order of atomic reductions, amplified by
        # cond(C)^2 in the solve; mixed fits also by FP32 AO rounding
        scale = max(1.0, info.condition) ** 2
        assert rel <= (1e-12 * scale if info.fit_path in (0, 2) else 1e-5 * scale), rel
        if fit_precision == "mixed":
            assert abs(info2.mixed_bound - info.mixed_bound) <= 1e-3 * info.mixed_bound
        assert abs(info2.pair_relative - info.pair_relative) <= 1e-8 * info.pair_relative


def test_select_fit_host_buffers(small_water):
    """Host-buffer twin of the fused call returns what the device call does."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    kw = dict(axes=("ao", "dx", "dy", "dz"), max_rank=6, oversampling=10, seed=5, precision="mixed")
    piv_h, th_h, si, fi = ctx.select_fit_host(pts, w, want_error=False, **kw)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    theta = torch.zeros(6 * len(pts), dtype=torch.float64, device="cuda")
    piv_d, _, fd = ctx.select_fit(x, wt, theta, want_error=False, **kw)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(piv_h, piv_d)
    th_d = theta[:len(piv_d) * fd.n_kept].cpu().numpy().reshape(len(piv_d), fd.n_kept)
    assert fi.fit_path == fd.fit_path and fi.n_kept == fd.n_kept
    # equal up to the order of atomic FP64 reductions, amplified by cond(C)^2
    rel = np.abs(th_h - th_d).max() / np.abs(th_d).max()
    assert rel <= 1e-12 * max(1.0, fd.condition) ** 2, rel


def test_select_fit_host_streams_theta_by_chunks():
    """(H2O)32 at grid level 3: the mixed Theta is accepted (fit path 1), so the
    host-buffer call fits the kept points in chunks and copies each chunk's
    Theta columns out while the next is fitted.  Its Theta equals the device
    call's bit for bit (per point the same tile GEMM and FP64 epilogue), into a
    pinned and into a pageable host buffer."""
    import torch
    from mp_isdf_b200 import capi, inputs
    mol, pts, w, cfg = inputs.make_config("c3")
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    kw = dict(algorithm="rand_sketch", axes=("ao",), max_rank=cfg["rank"], oversampling=cfg["oversampling"],
              seed=cfg["sketch_seed"], precision="mixed")
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    theta = torch.zeros(cfg["rank"] * len(pts), dtype=torch.float64, device="cuda")
    piv_d, _, fd = ctx.select_fit(x, wt, theta, want_error=False, **kw)
    torch.cuda.synchronize()
    assert fd.fit_path == 1 and fd.n_kept > 4 * 296 * 128
    th_d = theta[:len(piv_d) * fd.n_kept].cpu().numpy().reshape(len(piv_d), fd.n_kept)
    pinned = torch.empty(cfg["rank"] * len(pts), dtype=torch.float64).pin_memory().numpy()
    for out in (pinned, None):
        piv_h, th_h, si, fi = ctx.select_fit_host(pts, w, want_error=False, out=out, **kw)
        np.testing.assert_array_equal(piv_h, piv_d)
        assert fi.fit_path == 1 and fi.n_kept == fd.n_kept
        np.testing.assert_array_equal(th_h, th_d)


def test_mixed_projection_follows_moved_atoms(small_water):
    """After isdf_ctx_set_coords the tensor-core path evaluates AOs at the new
    centres: mixed and FP64 projections agree to the split-BF16 bound."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    moved = mol.coords + np.random.default_rng(1).normal(scale=0.2, size=mol.coords.shape)
    ctx.set_coords(moved)
    x = torch.tensor(pts[::5], device="cuda")
    W = np.random.default_rng(2).normal(size=(4 * mol.nao, 16))
    p64 = ctx.project_axes(x, ("ao", "dx", "dy", "dz"), W, "fp64").cpu().numpy()
    pm = ctx.project_axes(x, ("ao", "dx", "dy", "dz"), W, "mixed").cpu().numpy()
    scale = np.abs(p64).max()
    assert np.abs(pm - p64).max() <= 1e-4 * scale
    ctx.set_coords(mol.coords)


@pytest.mark.parametrize("axes,expect_mixed", [
    (("ao",), True),                    # 1 x 128-column accumulator
    (("ao", "dz"), True),               # 2 x 128
    (("ao", "dx", "dy"), True),         # 3 x 128
    (("ao", "dx", "dy", "dz"), False),  # 4 x 128 columns exceed the shared-memory plan: FP64 form
])
def test_wide_sketch_reports_form_and_matches_fp64(small_water, axes, expect_mixed):
    """rank 24 + oversampling 16 (ell = 40, 80 projection columns per axis):
    the mixed form runs with 128-column accumulators for up to three axis
    entries and reports the FP64 form otherwise; pivots equal the FP64 form's
    and the oracle's either way."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = small_water
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    kw = dict(axes=axes, max_rank=24, oversampling=16, seed=3)
    p64, i64 = ctx.select(x, wt, precision="fp64", **kw)
    pm, im = ctx.select(x, wt, precision="mixed", **kw)
    assert i64.precision_used == 0
    assert im.precision_used == (1 if expect_mixed else 0)
    assert im.sketch_rows == 40
    assert list(pm) == list(p64)
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    codes = [O.AXIS_CODES[a] for a in axes]
    scales = O.axis_scales(oc, pts, w, codes)
    ref = O.select_rand_sketch(oc, pts, w, codes, max_rank=24, oversampling=16, seed=3, scales=scales)
    assert list(pm) == ref
