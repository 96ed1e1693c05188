"""Generate the per-configuration golden fixtures from the CPU oracle.

Run on a CPU machine (no GPU needed):  ``python tests/golden/make_goldens.py [c1 c2 ...]``.
Each configuration of the benchmark suite (the five seeded water clusters,
plus C2's qrcp_online run ``c2o``) gets ``tests/golden/<key>.npz`` with

* ``anchors``         original grid indices of the oracle's anchors (pivot order);
* ``step_gap``        relative gap between the two largest residual norms at
                      each pivot step (exact norms); an implementation may pick
                      a different pivot only at a step whose gap is <= 1e-10;
* ``step_diag``       |R_jj| of each step;
* ``theta_pos`` / ``theta_sample``  Theta (k x S) of ``_physical_pair_refit``
                      (python/isdf.py:238-263) at a seeded sample of kept-point
                      positions (plus the anchors' own positions);
* ``pair_l2`` / ``pair_relative`` / ``exact2``  the pair-space error
                      (python/isdf.py:154-191) of that fit over all kept points;
* ``condition`` / ``retained_rank`` of the anchor pair matrix;
* for the randomized sketch: ``ell`` and LAPACK dgeqp3's pivots, |R_ii|,
  tails and numerical rank of the oracle's sketch (``dgeqp3_*``);
* for C4 and C5 (the differentiation configs): the seeded density's
  ``dm_seed``/``dm_nocc``/``dm_scale`` (D = dm_scale * c c^T with c from
  numpy's default_rng(dm_seed).normal((nao, nocc))), the ISDF energy and its
  FP64 nuclear gradient assembled from AO values and dx/dy/dz, and plain
  central differences at h = 1e-4 and h/2 bohr on listed coordinates (all 72
  of C4, six of C5).

The grid and basis come from ``mp_isdf_b200.inputs`` (seeded, deterministic);
``grid_checksum`` records sum(coords), sum(weights) and sum(|weights|) so that
a test can tell a regenerated grid from a different one.
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from mp_isdf_b200 import inputs  # noqa: E402
from oracle import oracle as O  # noqa: E402

AXIS = {"ao": 0, "dx": 1, "dy": 2, "dz": 3}
SAMPLE = 2048


def density_matrix(nao, nocc, seed, scale):
    """D = scale * c c^T, c ~ N(0,1) (nao x nocc) from numpy's default_rng(seed)."""
    c = np.random.default_rng(seed).normal(size=(nao, nocc))
    return scale * (c @ c.T)


def grid_checksum(pts, w):
    return np.array([pts.sum(), w.sum(), np.abs(w).sum()])


def make(key, log=print):
    t0 = time.time()
    mol, pts, w, cfg = inputs.make_config(key)
    names, factors = inputs.parse_axes(cfg["axes"])
    axes = [AXIS[a] for a in names]
    aw = factors if any(f != 1.0 for f in factors) else None
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    keep = np.flatnonzero(w != 0)
    n = len(keep)
    rank = cfg["rank"]
    out = dict(key=key, nao=mol.nao, n_grid=len(pts), n_kept=n, axes=np.array(axes),
               grid_checksum=grid_checksum(pts, w), rank=rank)
    # Multi-axis Frobenius scales: reference-order std::hypot accumulation
    # where it is affordable, else the OpenMP sum of squares (equal to rounding).
    exact_order = len(axes) * mol.nao * n < 2e9
    scales = O.axis_scales(oc, pts, w, axes, aw, exact_order=exact_order)
    out["scales"] = np.array([] if scales is None else scales)
    out["scales_exact_order"] = exact_order
    log(f"[{key}] nao {mol.nao} kept {n} axes {axes} scales {scales} ({time.time() - t0:.1f}s)")
    if cfg["algorithm"] == "rand_sketch":
        ell = rank + cfg["oversampling"]
        d = len(axes) * mol.nao
        u, v = O.sketch_factors(d, ell, cfg["sketch_seed"])
        y = oc.sketch(pts[keep], w[keep], axes, scales, u, v, ell)          # [n, ell]
        log(f"[{key}] sketch {y.shape} ({time.time() - t0:.1f}s)")
        pos_lapack, det = O.sketch_qr_rank(y, ell, cfg["oversampling"], 1e-10, rank,
                                           d * (d + 1) // 2)
        pos, diag, gaps = O.sketch_qrcp_exact(y.T, rank)
        out.update(ell=ell, dgeqp3_pivots=np.array([keep[p] for p in pos_lapack]),
                   dgeqp3_diag=det["diag"], dgeqp3_tails=det["tails"],
                   numerical_rank=det["numerical_rank"])
    else:
        f = oc.axis_features(pts[keep], axes, scales)
        pos, diag, gaps = O.pair_qrcp_exact(f, w[keep], rank)
        del f
    anchors = np.array([keep[p] for p in pos], dtype=np.int64)
    if cfg["algorithm"] == "rand_sketch":
        agree = [a == b for a, b in zip(anchors, out["dgeqp3_pivots"])]
        first_diff = agree.index(False) if False in agree else len(agree)
        if first_diff < len(agree):
            assert gaps[first_diff] <= 1e-10, (key, first_diff, gaps[first_diff])
    out.update(anchors=anchors, anchor_pos=np.array(pos, dtype=np.int64), step_gap=gaps,
               step_diag=diag)
    log(f"[{key}] anchors {anchors.tolist()} min gap {gaps.min():.3e} ({time.time() - t0:.1f}s)")
    # literal SVD fit at a sample of columns, pair error over all kept points
    phi_a = oc.eval_ao(pts[anchors])
    u_, s_, vt_, cond = O.physical_fit_svd(phi_a)
    rng = np.random.default_rng(1234)
    sample = np.union1d(rng.choice(n, size=min(SAMPLE, n), replace=False), np.array(pos))
    theta = O.physical_fit_columns(u_, s_, vt_, w[anchors], oc.eval_ao(pts[keep[sample]]))
    err = O.physical_pair_error(oc, pts[keep], w[keep], phi_a, s_, vt_)
    out.update(theta_pos=sample.astype(np.int64), theta_sample=theta, pair_l2=err["l2"],
               pair_relative=err["relative"], exact2=err["exact2"], condition=cond,
               retained_rank=len(s_))
    log(f"[{key}] cond {cond:.3e} pair rel {err['relative']:.15e} ({time.time() - t0:.1f}s)")
    if cfg.get("electrons"):
        out.update(adjoint(key, mol, pts[keep], w[keep], anchors, pts[anchors], w[anchors], oc, cfg,
                           log, t0))
    np.savez_compressed(HERE / f"{key}.npz", **out)
    log(f"[{key}] written ({time.time() - t0:.1f}s)")


def adjoint(key, mol, coords, weights, anchors, anchor_xyz, anchor_w, oc, cfg, log, t0):
    """Seeded density, ISDF energy, oracle gradient and central differences."""
    nao = mol.nao
    electrons = float(cfg["electrons"])
    nocc = max(1, int(round(electrons / 2)))
    seed = cfg["seed"]
    S = np.zeros((nao, nao))
    for s0 in range(0, len(coords), 65536):
        phi = oc.eval_ao(coords[s0:s0 + 65536])
        S += phi.T @ (weights[s0:s0 + 65536, None] * phi)
    base = density_matrix(nao, nocc, seed, 1.0)
    scale = electrons / np.trace(base @ S)
    dm = scale * base
    e = O.isdf_energy(oc, coords, weights, anchor_xyz, anchor_w, dm)
    g = O.isdf_energy_gradient(oc, coords, weights, anchor_xyz, anchor_w, dm)
    log(f"[{key}] energy {e:.12e} |grad| {np.linalg.norm(g):.6e} ({time.time() - t0:.1f}s)")

    def energy(atom, c, step):
        xyz = mol.coords.copy()
        xyz[atom, c] += step
        m2 = mol.with_coords(xyz)
        o2 = O.OracleContext(m2.atm, m2.bas, m2.env)
        return O.isdf_energy(o2, coords, weights, anchor_xyz, anchor_w, dm)

    h = 1e-4
    if key == "c4":
        fd_coords = [(a, c) for a in range(mol.coords.shape[0]) for c in range(3)]
    else:
        fd_coords = [(0, 0), (1, 1), (2, 2), (96, 0), (130, 1), (191, 2)]
    fd_h, fd_h2 = [], []
    for a, c in fd_coords:
        fd_h.append((energy(a, c, h) - energy(a, c, -h)) / (2 * h))
        fd_h2.append((energy(a, c, h / 2) - energy(a, c, -h / 2)) / h)
    log(f"[{key}] finite differences on {len(fd_coords)} coordinates ({time.time() - t0:.1f}s)")
    out = dict(dm_seed=seed, dm_nocc=nocc, dm_scale=scale, electrons=electrons, energy=e,
               gradient=g, fd_coords=np.array(fd_coords, dtype=np.int64), fd_h=np.array(fd_h), fd_step=h)
    if fd_h2:
        out["fd_h2"] = np.array(fd_h2)
    return out


if __name__ == "__main__":
    keys = sys.argv[1:] or ["c1", "c4", "c2", "c2o", "c3", "c5"]
    for k in keys:
        make(k)
