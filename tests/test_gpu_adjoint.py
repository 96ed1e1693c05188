"""Nuclear-gradient adjoint on the B200 against the FP64 oracle gradient
(assembled from AO values and dx/dy/dz) and against Richardson-extrapolated
central differences at h = 1e-4 bohr; tolerance 1e-6 relative."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system(small_water):
    import torch
    from mp_isdf_b200 import capi, inputs
    mol, pts, w = small_water
    keep = w != 0
    coords, weights = pts[keep][::3], w[keep][::3]
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    piv = O.select_qrcp_dense(oc, coords, weights, [0], max_rank=6)
    phi = oc.eval_ao(coords)
    S = phi.T @ (weights[:, None] * phi)
    dm = inputs.random_density(mol, S, 20.0, seed=3)
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(coords, device="cuda")
    wt = torch.tensor(weights, device="cuda")
    return mol, coords, weights, piv, dm, ctx, x, wt, oc


def test_gradient_matches_oracle(system):
    mol, coords, weights, piv, dm, ctx, x, wt, oc = system
    e, g = ctx.energy_gradient(x, wt, piv, dm)
    e_ref = O.isdf_energy(oc, coords, weights, coords[piv], weights[piv], dm)
    g_ref = O.isdf_energy_gradient(oc, coords, weights, coords[piv], weights[piv], dm)
    np.testing.assert_allclose(e, e_ref, rtol=1e-10)
    np.testing.assert_allclose(g, g_ref, rtol=1e-8, atol=1e-9 * np.abs(g_ref).max())


def test_gradient_matches_finite_differences(system):
    mol, coords, weights, piv, dm, ctx, x, wt, oc = system
    ctx.set_coords(mol.coords)
    _, g = ctx.energy_gradient(x, wt, piv, dm)

    def energy(atom, c, step):
        xyz = mol.coords.copy()
        xyz[atom, c] += step
        ctx.set_coords(xyz)
        return ctx.energy_gradient(x, wt, piv, dm)[0]

    h = 1e-4
    for atom, c in [(0, 0), (1, 2), (4, 1), (3, 0)]:
        fd1 = (energy(atom, c, h) - energy(atom, c, -h)) / (2 * h)
        fd2 = (energy(atom, c, h / 2) - energy(atom, c, -h / 2)) / h
        fd = (4 * fd2 - fd1) / 3
        np.testing.assert_allclose(g[atom, c], fd, rtol=1e-6, atol=1e-6 * np.abs(g).max())
    ctx.set_coords(mol.coords)


def test_autograd_function(system):
    import torch
    from mp_isdf_b200.autograd import isdf_energy
    mol, coords, weights, piv, dm, ctx, x, wt, oc = system
    R = torch.tensor(mol.coords, dtype=torch.float64, requires_grad=True)
    E = isdf_energy(R, ctx, x, wt, piv, dm)
    (2.0 * E).backward()
    g_ref = O.isdf_energy_gradient(oc, coords, weights, coords[piv], weights[piv], dm)
    np.testing.assert_allclose(R.grad.numpy(), 2.0 * g_ref, rtol=1e-8,
                               atol=1e-9 * np.abs(g_ref).max())


# ---- benchmark configurations C4 ((H2O)8) and C5 ((H2O)64) ------------------
GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def _golden_system(key):
    import torch
    from mp_isdf_b200 import capi, inputs
    path = GOLDEN / f"{key}.npz"
    if not path.exists():
        pytest.fail(f"missing golden fixture {path.name}; run tests/golden/make_goldens.py {key}")
    gold = dict(np.load(path))
    mol, pts, w, cfg = inputs.make_config(key)
    c = np.random.default_rng(int(gold["dm_seed"])).normal(size=(mol.nao, int(gold["dm_nocc"])))
    dm = float(gold["dm_scale"]) * (c @ c.T)
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    return gold, mol, dm, ctx, x, wt


@pytest.mark.parametrize("key", ["c4", "c5"])
def test_gradient_at_config_matches_oracle_and_differences(key):
    """dE/dR for every atom at the configuration's frozen FP64 anchors (the
    oracle's qrcp_dense / rand_sketch anchors of the golden fixture) against
    the oracle's FP64 gradient from AO dx/dy/dz values (1e-8 of max |g|) and
    against central differences of the oracle energy at h = 1e-4 bohr (1e-6
    of max |g|).  Where the plain h = 1e-4 difference carries an O(h^2)
    truncation error above 1e-6 of max |g| -- estimated from the h/2
    difference as 4/3 |fd_h - fd_h/2| -- the check uses the Richardson
    extrapolation (4 fd_h/2 - fd_h)/3 and reports the coordinate."""
    gold, mol, dm, ctx, x, wt = _golden_system(key)
    anchors = gold["anchors"]
    e, g = ctx.energy_gradient(x, wt, anchors, dm)
    e_only = ctx.energy(x, wt, anchors, dm)
    g_ref = gold["gradient"]
    scale = np.abs(g_ref).max()
    np.testing.assert_allclose(e, float(gold["energy"]), rtol=1e-10)
    np.testing.assert_allclose(e_only, e, rtol=1e-12)
    np.testing.assert_allclose(g, g_ref, rtol=0, atol=1e-8 * scale)
    richardson = []
    for (a, c), fh, fh2 in zip(gold["fd_coords"], gold["fd_h"], gold["fd_h2"]):
        trunc = 4.0 / 3.0 * abs(fh - fh2)
        if abs(g[a, c] - fh) <= 1e-6 * scale:
            continue
        assert trunc > 1e-6 * scale, (key, a, c, g[a, c], fh, trunc)
        rich = (4.0 * fh2 - fh) / 3.0
        assert abs(g[a, c] - rich) <= 1e-6 * scale, (key, a, c, g[a, c], rich)
        richardson.append((int(a), int(c), float(abs(g[a, c] - fh) / scale)))
    print(f"{key}: E {e:.12e}, max |g| {scale:.6e}, {len(gold['fd_coords'])} coordinates checked, "
          f"h^2-limited (atom, axis, |g - fd_h| / max|g|): {richardson}")
