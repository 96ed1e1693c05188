#!/usr/bin/env python3
"""ISDF hot-path driver on the B200: grid -> anchor selection -> Theta fit.

Mirrors the selection-to-fit slice of mikovtun/mp_isdf ``python/isdf.py``
(``build_isdf`` :287-672 and the CLI :825-1004) over the drop-in ``mp_isdf``
module of this repository.  PySCF is not required: molecules are either
synthetic water clusters (``--molecule water:4x4x4[:seed]``, the seeded
cc-pVDZ-shaped basis of ``mp_isdf_b200.inputs``) or libcint tables loaded from
an ``.npz`` file with arrays atm, bas, env (and optionally coords, weights).
The Coulomb metric is available in its grid form (``--metric-algorithm grid``,
computed on the GPU; without ``--no-metric``); the integral-direct Cholesky
metrics and derivative targets are outside this path.

Example:
  python python/isdf.py --molecule water:2x2x1 --level 2 --axes ao \
      --anchor-algorithm qrcp_dense --anchor-rank 8 --pair-space-error
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, os.environ.get("ISDF_BUILD_DIR", str(ROOT / "mp_isdf_b200")))
import mp_isdf  # noqa: E402

from mp_isdf_b200 import inputs  # noqa: E402

KHATRIRAO_SKETCH_TECHNIQUES = ("quadrature", "density", "density_col_norm")
DENSITY_SKETCHES = ("density", "density_col_norm")
SKETCH_ENUM = {"quadrature": "RandomizedQuadratureKhatriRao", "density": "RandomizedAODensityKhatriRao",
               "density_col_norm": "RandomizedAODensityNormalizedKhatriRao"}
SKETCH_ALGORITHMS = ("rand_sketch",)
AXES = {
    "ao": mp_isdf.AxisType.AtomicOrbital,
    "dx": mp_isdf.AxisType.AtomicOrbitalGradX,
    "dy": mp_isdf.AxisType.AtomicOrbitalGradY,
    "dz": mp_isdf.AxisType.AtomicOrbitalGradZ,
    "occ": mp_isdf.AxisType.OccupiedOrbital,
}


def pair_space_error_norms(pair_grid, pair_anchor, anchor_weights, theta, grid_weights,
                           block_size=256):
    """Absolute and relative |w|-weighted L2 error of explicit pair columns
    (``python/isdf.py:154-173``); for small grids."""
    weighted_anchor = pair_anchor * anchor_weights[:, None]
    residual_sq = exact_sq = 0.0
    for first in range(0, len(grid_weights), block_size):
        last = min(first + block_size, len(grid_weights))
        exact = pair_grid[first:last]
        rec = theta[:, first:last].T @ weighted_anchor
        weight = np.abs(grid_weights[first:last])
        residual_sq += np.einsum("g,gi,gi->", weight, exact - rec, exact - rec, optimize=True)
        exact_sq += np.einsum("g,gi,gi->", weight, exact, exact, optimize=True)
    absolute = np.sqrt(residual_sq)
    relative = absolute / np.sqrt(exact_sq) if exact_sq else (0.0 if absolute == 0 else np.inf)
    return {"l2": absolute, "relative": relative}


class Molecule:
    """Minimal stand-in for the PySCF molecule: libcint tables + helpers."""

    def __init__(self, atm, bas, env, coords=None, symbols=None):
        self._atm, self._bas, self._env = atm, bas, env
        self.coords = coords
        self.symbols = symbols

    @classmethod
    def from_spec(cls, spec: str):
        if spec.startswith("water:"):
            parts = spec.split(":")
            lat = tuple(int(v) for v in parts[1].split("x"))
            seed = int(parts[2]) if len(parts) > 2 else 0
            sym, xyz = inputs.water_cluster(lat, seed=seed)
            t = inputs.build_tables(sym, xyz)
            return cls(t.atm, t.bas, t.env, t.coords, t.symbols)
        d = np.load(spec)
        return cls(d["atm"], d["bas"], d["env"])


def grid_coulomb_metric(interp_vecs, coords, weights):
    """Spherical-cell grid Coulomb metric (``python/isdf.py:48-68``), computed
    on the GPU by the library's FP64 all-pairs kernel.  interp_vecs has shape
    (Nanchor, Ngrid) and is NOT weight-scaled."""
    return mp_isdf.grid_coulomb_metric(np.ascontiguousarray(interp_vecs, dtype=np.float64),
                                       np.ascontiguousarray(coords, dtype=np.float64),
                                       np.ascontiguousarray(weights, dtype=np.float64))


def grid_cross_metric(left, right, coords, weights):
    """Grid Coulomb metric between two independently fitted channel sets
    (``python/isdf.py:80-97``), on the GPU."""
    return mp_isdf.grid_cross_metric(np.ascontiguousarray(left, dtype=np.float64),
                                     np.ascontiguousarray(right, dtype=np.float64),
                                     np.ascontiguousarray(coords, dtype=np.float64),
                                     np.ascontiguousarray(weights, dtype=np.float64))


def evaluate_isdf_jk(result, dm):
    """Return (J, K) for a real symmetric AO density matrix
    (``python/isdf.py:130-151``).  The metric in `result` already includes both
    anchor quadrature weights; (mu nu|lam sig) is approximated by
    sum_pq X[p,mu] X[p,nu] Z[p,q] X[q,lam] X[q,sig] with X[p,mu] = AO_mu(anchor_p); J and K
    are built on the B200 (mp_isdf.isdf_jk: FP64 tensor-core GEMMs)."""
    x = np.asarray(result["X1"])
    z = result["coulomb_metric"]
    if z is None:
        raise ValueError("a Coulomb metric is required to evaluate J and K")
    density = np.asarray(dm, dtype=np.float64)
    if density.shape != (x.shape[1], x.shape[1]) or not np.isfinite(density).all():
        raise ValueError("dm must be a finite AO density matrix of shape (nao,nao)")
    if not np.allclose(density, density.T, rtol=1e-12, atol=1e-12):
        raise ValueError("dm must be symmetric")
    if np.shape(z) != (len(x), len(x)):
        raise ValueError("Coulomb metric has the wrong anchor dimensions")
    context = result.get("context")
    if context is None:
        raise ValueError("the ISDF result carries no AO context")
    return mp_isdf.isdf_jk(context, np.ascontiguousarray(x), np.ascontiguousarray(z, dtype=np.float64),
                           np.ascontiguousarray(density))


def _validate_point_importance(importance, ngrid):
    """``python/isdf.py:231-235``."""
    importance = np.asarray(importance, dtype=np.float64)
    if importance.shape != (ngrid,) or not np.isfinite(importance).all() or np.any(importance < 0):
        raise ValueError("point_importance must be a finite nonnegative array of shape (ngrid,)")
    return np.ascontiguousarray(importance)


def _normalized_pair_error(context, coords, anchor_ao, anchor_weights, theta, importance, threshold,
                           space, batch=65536):
    """Density-weighted relative-column error (``python/isdf.py:266-287``):
    sum_g m_g |p_g - sum_k c_k p_k|^2 / q_g^2 over points with q_g = |phi_g|^2 >
    threshold, relative to sum_g m_g; by the Gram expansion |p_g - C^T c|^2 =
    q^2 - 2 c.h + c^T M c (h = (Phi_a phi_g)^2, M = (Phi_a Phi_a^T)^2), so no pair
    vector is formed."""
    M = (anchor_ao @ anchor_ao.T) ** 2
    residual_sq = total = screened = 0.0
    for g0 in range(0, len(coords), batch):
        ao = context.eval_ao(coords[g0:g0 + batch], space=space)
        m = importance[g0:g0 + batch]
        q = np.einsum("ga,ga->g", ao, ao)
        c = (np.asarray(theta)[:, g0:g0 + batch] * anchor_weights[:, None]).T
        h = (ao @ anchor_ao.T) ** 2
        r2 = q * q - 2 * np.einsum("gk,gk->g", c, h) + np.einsum("gk,kl,gl->g", c, M, c)
        inc = (q > threshold) & (m != 0)
        screened += float(m[q <= threshold].sum())
        residual_sq += float(np.sum(m[inc] * np.maximum(r2[inc], 0.0) / q[inc] ** 2))
        total += float(m[inc].sum())
    return {"l2": float(np.sqrt(residual_sq)),
            "relative": float(np.sqrt(residual_sq / total)) if total else 0.0,
            "included_mass": float(total), "screened_mass": float(screened)}


def _pair_error(context, coords, weights, anchor_ao, anchor_weights, theta, space, batch=65536):
    """Pair-space error of a given Theta (``python/isdf.py:154-191``):
    sum_g |w_g| |p_g - sum_k Theta_kg w_k p_k|^2 in the Gram form
    q^2 - 2 c.h + c^T M c (c = Theta_g w_a, h = (Phi_a phi_g)^2, M = (Phi_a Phi_a^T)^2),
    relative to sum_g |w_g| q_g^2."""
    M = (anchor_ao @ anchor_ao.T) ** 2
    err2 = exact2 = 0.0
    for g0 in range(0, len(coords), batch):
        ao = context.eval_ao(coords[g0:g0 + batch], space=space)
        aw = np.abs(weights[g0:g0 + batch])
        q = np.einsum("ga,ga->g", ao, ao)
        c = (np.asarray(theta)[:, g0:g0 + batch] * anchor_weights[:, None]).T
        h = (ao @ anchor_ao.T) ** 2
        r2 = q * q - 2 * np.einsum("gk,gk->g", c, h) + np.einsum("gk,kl,gl->g", c, M, c)
        err2 += float(np.sum(aw * r2))
        exact2 += float(np.sum(aw * q * q))
    err2 = max(err2, 0.0)
    return {"l2": float(np.sqrt(err2)), "relative": float(np.sqrt(err2 / exact2)) if exact2 else 0.0}


def build_isdf(mol, *, level=0, anchor_rank=0, anchor_tol=None, axes=("ao",), axis_weights=None,
               space="auto", anchor_algorithm="qrcp_dense", sketch="quadrature",
               anchor_batch_size=128, fit_batch_size=2048, anchor_sketch_size=128,
               anchor_oversampling=16, anchor_seed=7, selection_only=False, debug=False,
               pair_space_error=False, report_timings=False, report_dimensions=False, grid=None,
               precision="fp64", point_importance=None, density_weight="electron_density",
               ao_screening_threshold=1e-24, compute_metric=False, metric_algorithm="grid",
               mo_coeff=None, nocc=0, rbrp_block_size=16, rbrp_tau_block=None, rbrp_rank_rtol=1e-12,
               rbrp_refresh_every=8, rbrp_svd_rtol=1e-12):
    """Selection-to-fit slice of ``build_isdf`` (``python/isdf.py:287-672``).

    `grid` is an optional (coords, weights) pair; otherwise a Becke-partitioned
    atom-centred grid of the requested level is generated for the synthetic
    waters.  `precision` selects the FP64 or mixed (FP32 AO / split-BF16
    tensor-core / FP64 QR and solve) form on the B200.

    Density sketches (`sketch="density"` / `"density_col_norm"`, rand_sketch,
    AO axis only, FP64 form) weight pair columns by sqrt(point_importance) and
    screen points whose squared AO norm is <= `ao_screening_threshold`
    (``python/isdf.py:322-340``).  `point_importance` is the complete m on the
    grid; generating it needs an RKS B3LYP density (PySCF), which this
    package does not provide, so it must be given.

    The occupied-orbital axis (`"occ"`) takes the row-major (nao, nao) RHF
    `mo_coeff` and `nocc` (the reference takes them from a PySCF RHF,
    ``python/isdf.py:505-511``).

    `compute_metric=True` with `metric_algorithm="grid"` adds the anchor-
    weighted grid Coulomb metric (``python/isdf.py:674-683``) as
    `coulomb_metric`; the integral-direct Cholesky metrics need ERIs that are
    outside this path.
    """
    started = time.perf_counter()
    last = started
    timings = {}

    def record(stage):
        nonlocal last
        now = time.perf_counter()
        timings[stage] = now - last
        last = now
        if report_timings and not debug:
            print(f"  {stage:18s} {timings[stage]:10.6f} s  (elapsed {last - started:.6f} s)", flush=True)

    if isinstance(axes, str):
        axes = (axes,)
    try:
        axis_types = [AXES[a] if isinstance(a, str) else a for a in axes]
    except KeyError as exc:
        raise ValueError(f"unknown axis: {exc.args[0]!r}; choose from {list(AXES)}") from exc
    if axis_weights is not None:
        axis_weights = tuple(float(w) for w in axis_weights)
        if len(axis_weights) != len(axis_types) or not all(np.isfinite(w) and w > 0 for w in axis_weights):
            raise ValueError("axis_weights must contain one finite positive factor per axis")
    sketch_algorithm = anchor_algorithm == "rand_sketch"
    if sketch_algorithm:
        if sketch not in KHATRIRAO_SKETCH_TECHNIQUES:
            raise ValueError(f"sketch must be one of {KHATRIRAO_SKETCH_TECHNIQUES} for rand_sketch")
    elif sketch != "quadrature":
        raise ValueError("non-default sketch requires anchor_algorithm='rand_sketch'")
    density_sketch = sketch_algorithm and sketch in DENSITY_SKETCHES
    if density_sketch and axis_types != [mp_isdf.AxisType.AtomicOrbital]:
        raise NotImplementedError("density Khatri--Rao sketches with non-AO axis features are NYI")
    if density_weight not in ("electron_density", "quadrature_density"):
        raise ValueError("density_weight must be electron_density or quadrature_density")
    if not np.isfinite(ao_screening_threshold) or ao_screening_threshold < 0:
        raise ValueError("ao_screening_threshold must be finite and nonnegative")
    if point_importance is not None and not density_sketch:
        raise ValueError("point_importance requires CVT or a density sketch")
    if metric_algorithm not in ("grid", "unblocked_greedy", "unblocked_uniform"):
        raise ValueError(f"unknown metric algorithm: {metric_algorithm!r}")
    if selection_only and compute_metric:
        raise ValueError("selection_only requires compute_metric=False")
    if compute_metric and metric_algorithm != "grid":
        raise NotImplementedError("the integral-direct Cholesky metrics are outside the B200 hot path (NYI)")
    rbrp_mode = anchor_algorithm in ("rbrp", "rbrp_id")
    if anchor_algorithm not in ("qrcp_dense", "qrcp_online", "rbrp", "rbrp_id", *SKETCH_ALGORITHMS):
        if anchor_algorithm == "cvt":
            raise NotImplementedError("cvt is outside the B200 hot path (NYI)")
        raise ValueError(f"unknown anchor algorithm: {anchor_algorithm!r}")
    if rbrp_mode:
        # python/isdf.py:427-436
        if axis_types != [mp_isdf.AxisType.AtomicOrbital]:
            raise ValueError("RBRP currently requires axes=('ao',)")
        if (not isinstance(rbrp_block_size, (int, np.integer)) or rbrp_block_size < 1 or
                not isinstance(rbrp_refresh_every, (int, np.integer)) or rbrp_refresh_every < 0 or
                not np.isfinite(rbrp_rank_rtol) or rbrp_rank_rtol <= 0 or
                not np.isfinite(rbrp_svd_rtol) or rbrp_svd_rtol < 0 or
                (rbrp_tau_block is not None and
                 (not np.isfinite(rbrp_tau_block) or not 0 <= rbrp_tau_block < 1))):
            raise ValueError("invalid RBRP block size, refresh interval or tolerances")
    if not isinstance(anchor_batch_size, (int, np.integer)) or anchor_batch_size <= 0:
        raise ValueError("anchor_batch_size must be a positive integer")
    if not isinstance(fit_batch_size, (int, np.integer)) or fit_batch_size <= 0:
        raise ValueError("fit_batch_size must be a positive integer")
    if anchor_rank != 0 and anchor_tol is not None:
        raise ValueError("anchor_rank and anchor_tol are mutually exclusive")
    if anchor_tol is None:
        anchor_tol = 1e-10
    if not np.isfinite(anchor_tol) or anchor_tol < 0:
        raise ValueError("anchor_tol must be finite and nonnegative")
    if (not isinstance(anchor_sketch_size, (int, np.integer)) or
            not isinstance(anchor_oversampling, (int, np.integer)) or
            anchor_oversampling < 1 or anchor_sketch_size < 1 or
            (sketch_algorithm and anchor_rank == 0 and anchor_sketch_size <= anchor_oversampling)):
        raise ValueError("randomized anchor sketch_size must exceed oversampling when anchor_rank=0")
    if not isinstance(anchor_seed, (int, np.integer)) or not 0 <= anchor_seed < 2 ** 64:
        raise ValueError("anchor_seed must be an unsigned 64-bit integer")
    if selection_only and pair_space_error:
        raise ValueError("pair_space_error requires fitting; disable selection_only")
    needs_occ = mp_isdf.AxisType.OccupiedOrbital in axis_types
    if needs_occ and mo_coeff is None:
        raise NotImplementedError("the occupied-orbital axis needs RHF MO coefficients (PySCF is not "
                                  "available here); pass mo_coeff and nocc")

    if grid is None:
        if mol.symbols is None:
            raise ValueError("a grid is required for molecules loaded from tables")
        all_coords, all_weights = inputs.becke_grid(mol.symbols, mol.coords, level=level)
    else:
        all_coords, all_weights = grid
    all_coords = np.ascontiguousarray(all_coords, dtype=np.float64)
    all_weights = np.ascontiguousarray(all_weights, dtype=np.float64)
    keep = all_weights != 0
    if not np.any(keep):
        raise ValueError("grid has no nonzero weights")
    record("grid")

    context = mp_isdf.LibcintContext(mol._atm, mol._bas, mol._env)
    selector = mp_isdf.AnchorSelection(context)
    record("context")
    nao = context.nao
    axis_width = sum(nocc if a == mp_isdf.AxisType.OccupiedOrbital else nao for a in axis_types)
    pair_rank_ceiling = axis_width * (axis_width + 1) // 2
    if report_dimensions:
        dims = (f"[ISDF dimensions] AOs={nao} axis_features={axis_width} "
                f"symmetric_pair_rank_ceiling={pair_rank_ceiling} "
                f"grid_points={len(all_coords)} nonzero_weight_points={int(np.count_nonzero(keep))}")
        if sketch_algorithm:
            ell = anchor_rank + anchor_oversampling if anchor_rank > 0 else anchor_sketch_size
            cap = min(ell - anchor_oversampling, pair_rank_ceiling, int(np.count_nonzero(keep)))
            dims += (f" sketch_rows={ell} oversampling={anchor_oversampling}"
                     f" sketch_rank_cap={cap} sketch_matrix={ell}x{int(np.count_nonzero(keep))}"
                     f" sketch_storage={ell * int(np.count_nonzero(keep)) * 8 / 2**20:.1f}MiB")
            if anchor_rank > 0:
                dims += f" requested_rank={anchor_rank} (anchor_sketch_size ignored)"
        print(dims, flush=True)
    importance = None
    if density_sketch:
        if point_importance is None:
            raise NotImplementedError("the selection density needs an RKS B3LYP calculation (PySCF), "
                                      "which is not available here; pass point_importance")
        importance = _validate_point_importance(point_importance, len(all_coords))
        record("point_importance")
    rbrp_result = None
    if rbrp_mode:
        # python/isdf.py:564-589: RBRP on the nonzero-weight points, AOs on the device
        settings = dict(batch_size=anchor_batch_size, block_size=rbrp_block_size,
                        tolerance=anchor_tol, max_rank=anchor_rank, seed=anchor_seed,
                        tau_block=rbrp_tau_block, rank_rtol=rbrp_rank_rtol,
                        refresh_every=rbrp_refresh_every, svd_rtol=rbrp_svd_rtol,
                        compute_id=(anchor_algorithm == "rbrp_id" and not selection_only))
        rbrp_result = mp_isdf.rbrp_ao_device(selector, all_coords[keep], all_weights[keep], **settings)
        anchor_indices = np.flatnonzero(keep)[np.asarray(rbrp_result["indices"], dtype=np.intp)]
        if debug:
            print(f"[rbrp] rank={len(anchor_indices)} residual={rbrp_result['relative_residual']:.6e} "
                  f"status={rbrp_result['status']} blocks={len(rbrp_result['history'])}", flush=True)
    algo = {"qrcp_dense": mp_isdf.LocalAnchorSelectionAlgorithm.QRColumnPivoting,
            "qrcp_online": mp_isdf.LocalAnchorSelectionAlgorithm.OnlineQRColumnPivoting,
            "rand_sketch": mp_isdf.LocalAnchorSelectionAlgorithm.RandomizedQuadratureKhatriRao,
            "rbrp": None, "rbrp_id": None}[anchor_algorithm]
    if density_sketch:
        algo = getattr(mp_isdf.LocalAnchorSelectionAlgorithm, SKETCH_ENUM[sketch])
    if not rbrp_mode:
        anchor_indices = np.asarray(selector.select(
            all_coords, all_weights, axis_types, tolerance=anchor_tol, max_rank=anchor_rank,
            algorithm=algo, space=space, batch_size=anchor_batch_size, debug=debug,
            sketch_size=anchor_sketch_size, oversampling=anchor_oversampling, seed=anchor_seed,
            axis_weights=list(axis_weights) if axis_weights is not None else [],
            point_importance=importance, ao_screening_threshold=ao_screening_threshold,
            mo_coeff=np.ascontiguousarray(mo_coeff) if needs_occ else None, nocc=nocc if needs_occ else 0,
            precision=precision), dtype=np.intp)
    if len(anchor_indices) == 0:
        raise ValueError("anchor selection found no anchors; adjust settings or grid")
    record("anchor_selection")
    if selection_only:
        return {"anchor_indices": anchor_indices, "anchor_coords": all_coords[anchor_indices],
                "anchor_weights": all_weights[anchor_indices], "coordinates": all_coords[keep],
                "weights": all_weights[keep], "interp_vecs": None, "pair_space_errors": None,
                "coulomb_metric": None,
                "fit_diagnostics": None, "elapsed": last - started, "timings": timings}

    coords = all_coords[keep]
    weights = all_weights[keep]
    anchor_coords = all_coords[anchor_indices]
    anchor_weights = all_weights[anchor_indices]
    anchor_ao = context.eval_ao(anchor_coords, space=space)
    record("ao_evaluation")
    id_info = None
    if anchor_algorithm == "rbrp_id":
        # python/isdf.py:640-647: the RBRP interpolative decomposition is the fit
        interp_vecs = np.asarray(rbrp_result["interp_vecs"])
        id_info = {key: rbrp_result[key] for key in ("retained_rank", "condition", "relative_residual", "status")}
        fit_diagnostics = None
        theta_w = interp_vecs @ weights
    else:
        fit = mp_isdf.fit(context, all_coords, all_weights, anchor_indices, precision=precision,
                          pair_space_error=pair_space_error)
        interp_vecs = fit["interp_vecs"]
        fit_diagnostics = {key: fit[key] for key in ("retained_rank", "condition",
                                                     "max_abs_physical_coefficient")}
        theta_w = np.asarray(fit["theta_w"][:len(anchor_weights)])
    record("isdf_fit")
    pair_space_errors = None
    if pair_space_error:
        if anchor_algorithm == "rbrp_id":
            pair_space_errors = {"scalar": _pair_error(context, coords, weights, anchor_ao, anchor_weights,
                                                       interp_vecs, space)}
        else:
            pair_space_errors = {"scalar": {"l2": fit["pair_l2"], "relative": fit["pair_relative"]}}
        if importance is not None:
            pair_space_errors["density_normalized"] = _normalized_pair_error(
                context, coords, anchor_ao, anchor_weights, interp_vecs, importance[keep],
                ao_screening_threshold, space)
        record("pair_space_check")
    # Overlap reconstruction (python/isdf.py:665-671); without int1e_ovlp the
    # reference overlap is the grid quadrature Phi^T diag(w) Phi (small systems).
    overlap_approx = np.einsum("ku,kv,k->uv", anchor_ao, anchor_ao,
                               anchor_weights * theta_w,
                               optimize=True) if len(anchor_weights) <= 64 else None
    overlap_relative_error = None
    if overlap_approx is not None and nao <= 400 and len(coords) <= 400000:
        ao = context.eval_ao(coords, space=space)
        overlap = ao.T @ (weights[:, None] * ao)
        overlap_relative_error = (np.linalg.norm(overlap_approx - overlap) /
                                  max(np.linalg.norm(overlap), 1e-30))
    record("overlap_check")
    metric = None
    if compute_metric:
        raw = grid_coulomb_metric(interp_vecs, coords, weights)
        metric = anchor_weights[:, None] * raw * anchor_weights[None, :]
        record("coulomb_metric")
    return {"anchor_indices": anchor_indices, "fit_diagnostics": fit_diagnostics, "coulomb_metric": metric,
            "rbrp_diagnostics": ({key: rbrp_result[key] for key in ("relative_residual", "status", "history")}
                                 if rbrp_result is not None else None),
            "id_diagnostics": id_info,
            "anchor_coords": anchor_coords, "anchor_weights": anchor_weights,
            "coordinates": coords, "weights": weights, "interp_vecs": interp_vecs,
            "overlap_reconstruction": overlap_approx,
            "overlap_relative_error": overlap_relative_error,
            "pair_space_errors": pair_space_errors, "X1": anchor_ao, "context": context,
            "elapsed": last - started, "timings": timings}


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--molecule", default="water:1x1x1",
                        help="water:AxBxC[:seed] synthetic cluster, or an .npz with atm/bas/env")
    parser.add_argument("--basis", default="synthetic-cc-pvdz",
                        help="basis label (only the synthetic cc-pVDZ-shaped basis is available)")
    parser.add_argument("--level", type=int, default=0)
    parser.add_argument("--anchor-rank", type=int, default=0)
    parser.add_argument("--anchor-tol", type=float, default=None)
    parser.add_argument("--anchor-algorithm", choices=("qrcp_dense", "qrcp_online", *SKETCH_ALGORITHMS,
                                                       "cvt", "rbrp", "rbrp_id"), default="qrcp_dense")
    parser.add_argument("--sketch", choices=KHATRIRAO_SKETCH_TECHNIQUES, default=None)
    parser.add_argument("--rbrp-block-size", type=int, default=16)
    parser.add_argument("--rbrp-tau-block", type=float, default=None,
                        help="local QR trailing-energy threshold (default: 1/block_size)")
    parser.add_argument("--rbrp-rank-rtol", type=float, default=1e-12)
    parser.add_argument("--rbrp-refresh-every", type=int, default=8)
    parser.add_argument("--rbrp-svd-rtol", type=float, default=1e-12)
    parser.add_argument("--anchor-batch-size", type=int, default=128)
    parser.add_argument("--fit-batch-size", type=int, default=2048)
    parser.add_argument("--anchor-sketch-size", type=int, default=128)
    parser.add_argument("--anchor-oversampling", type=int, default=16)
    parser.add_argument("--anchor-seed", type=int, default=7)
    parser.add_argument("--density-weight", choices=("electron_density", "quadrature_density"),
                        default="electron_density", help="density sketch importance: rho or abs(w)*rho")
    parser.add_argument("--ao-screening-threshold", type=float, default=1e-24,
                        help="density sketch squared AO norm cutoff (selection only)")
    parser.add_argument("--importance-file", default=None,
                        help=".npy with the density sketch importance m over the grid (no RKS here)")
    parser.add_argument("--axes", default="ao")
    parser.add_argument("--space", choices=("auto", "host", "device"), default="auto")
    parser.add_argument("--pair-space-error", action="store_true")
    parser.add_argument("--no-metric", action="store_true", help="skip the Coulomb metric")
    parser.add_argument("--metric-algorithm", choices=("grid", "unblocked_greedy", "unblocked_uniform"),
                        default=None, help="grid: spherical-cell grid metric on the GPU (the "
                        "Cholesky metrics are outside this path); without it no metric is computed")
    parser.add_argument("--debug", action="store_true")
    parser.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    parser.add_argument("--grid-file", default=None, help=".npz with coords and weights")
    parser.add_argument("--json", default=None, help="write a JSON record of the run")
    args = parser.parse_args(argv)
    if args.anchor_rank < 0:
        parser.error("--anchor-rank must be nonnegative")
    if args.anchor_algorithm not in SKETCH_ALGORITHMS and args.sketch is not None:
        parser.error("--sketch requires --anchor-algorithm rand_sketch")
    if not np.isfinite(args.ao_screening_threshold) or args.ao_screening_threshold < 0:
        parser.error("--ao-screening-threshold must be finite and nonnegative")
    if args.anchor_batch_size <= 0:
        parser.error("--anchor-batch-size must be positive")
    if args.fit_batch_size <= 0:
        parser.error("--fit-batch-size must be positive")
    if args.anchor_sketch_size < 1 or args.anchor_oversampling < 1 or (
            args.anchor_algorithm in SKETCH_ALGORITHMS and args.anchor_rank == 0 and
            args.anchor_sketch_size <= args.anchor_oversampling):
        parser.error("randomized sketch size must exceed oversampling when --anchor-rank=0")
    if not 0 <= args.anchor_seed < 2 ** 64:
        parser.error("--anchor-seed must be an unsigned 64-bit integer")
    if args.anchor_rank != 0 and args.anchor_tol is not None:
        parser.error("--anchor-rank and --anchor-tol are mutually exclusive")
    if args.anchor_tol is not None and (not np.isfinite(args.anchor_tol) or args.anchor_tol < 0):
        parser.error("--anchor-tol must be finite and nonnegative")
    if args.level < 0:
        parser.error("--level must be nonnegative")
    axes, axis_weights = [], []
    for entry in args.axes.split(","):
        fields = entry.strip().lower().split(":")
        if len(fields) > 2 or fields[0] not in AXES:
            parser.error(f"invalid --axes entry: {entry!r}")
        try:
            factor = float(fields[1]) if len(fields) == 2 else 1.0
        except ValueError:
            parser.error(f"invalid --axes factor: {entry!r}")
        if not np.isfinite(factor) or factor <= 0:
            parser.error(f"--axes factor must be finite and positive: {entry!r}")
        axes.append(fields[0])
        axis_weights.append(factor)
    mol = Molecule.from_spec(args.molecule)
    grid = None
    if args.grid_file:
        g = np.load(args.grid_file)
        grid = (g["coords"], g["weights"])
    result = build_isdf(mol, level=args.level, anchor_rank=args.anchor_rank,
                        anchor_tol=args.anchor_tol, axes=axes, axis_weights=axis_weights,
                        space=args.space, anchor_algorithm=args.anchor_algorithm,
                        sketch=args.sketch or "quadrature",
                        anchor_batch_size=args.anchor_batch_size,
                        fit_batch_size=args.fit_batch_size,
                        anchor_sketch_size=args.anchor_sketch_size,
                        anchor_oversampling=args.anchor_oversampling, anchor_seed=args.anchor_seed,
                        pair_space_error=args.pair_space_error, report_timings=not args.debug,
                        debug=args.debug, report_dimensions=True, grid=grid,
                        precision=args.precision,
                        point_importance=np.load(args.importance_file) if args.importance_file else None,
                        density_weight=args.density_weight,
                        ao_screening_threshold=args.ao_screening_threshold,
                        compute_metric=bool(args.metric_algorithm) and not args.no_metric,
                        metric_algorithm=args.metric_algorithm or "grid",
                        rbrp_block_size=args.rbrp_block_size, rbrp_tau_block=args.rbrp_tau_block,
                        rbrp_rank_rtol=args.rbrp_rank_rtol, rbrp_refresh_every=args.rbrp_refresh_every,
                        rbrp_svd_rtol=args.rbrp_svd_rtol)
    print(f"Grid points: {len(result['coordinates'])}; AOs: {result['X1'].shape[1]}; "
          f"anchors: {len(result['anchor_indices'])}")
    if args.anchor_rank and len(result["anchor_indices"]) == args.anchor_rank:
        print(f"Anchor count equals --anchor-rank {args.anchor_rank}; use --anchor-rank 0 "
              "for tolerance-only selection or a larger value for a higher cap.")
    if result["overlap_relative_error"] is not None:
        print(f"Overlap reconstruction relative error: {result['overlap_relative_error']:.3e}")
    if result["pair_space_errors"] is not None:
        for label, error in result["pair_space_errors"].items():
            print(f"Pair-space {label} grid L2 error: {error['l2']:.3e}; "
                  f"relative error: {error['relative']:.3e}")
    if result["coulomb_metric"] is not None:
        z = result["coulomb_metric"]
        print(f"Coulomb metric (grid): {z.shape[0]}x{z.shape[1]}; "
              f"diagonal range [{np.min(np.diag(z)):.6e}, {np.max(np.diag(z)):.6e}]")
    if not args.debug:
        print(f"ISDF build time: {result['elapsed']:.6f} s")
    else:
        print("Timing report:")
        for stage, seconds in result["timings"].items():
            frac = 100 * seconds / result["elapsed"] if result["elapsed"] else 0.0
            print(f"  {stage:22s} {seconds:10.6f} s  ({frac:5.1f}% of build)")
        print(f"  ISDF build total       {result['elapsed']:10.6f} s")
    if args.json:
        rec = {"anchor_indices": [int(i) for i in result["anchor_indices"]],
               "timings": result["timings"], "elapsed": result["elapsed"],
               "pair_space_errors": result["pair_space_errors"],
               "fit_diagnostics": ({k: float(v) for k, v in result["fit_diagnostics"].items()}
                                   if result["fit_diagnostics"] is not None else None),
               "id_diagnostics": ({k: (v if isinstance(v, str) else float(v))
                                   for k, v in result["id_diagnostics"].items()}
                                  if result.get("id_diagnostics") else None),
               "precision": args.precision, "axes": args.axes}
        Path(args.json).write_text(json.dumps(rec, indent=1))
    return result


if __name__ == "__main__":
    main()
