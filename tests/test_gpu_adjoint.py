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
