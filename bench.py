#!/usr/bin/env python3
"""Anchor selection + interpolation-vector fit, seconds per water cluster.

One step = rand_sketch (quadrature) anchor selection + Theta fit for one
cluster, grid and weights resident in HBM (`value`), and the same through the
host-buffer C-ABI entry points with host<->device copies inside the timed
region (`e2e`).  Default workload: (H2O)64, synthetic cc-pVDZ-shaped basis
(1536 AOs), level-3 stand-in grid (~2e6 points), axes ao,dx,dy,dz, rank 10.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--config c5] [--precision fp64|mixed]
Under torchrun (N > 1) every rank runs its own cluster (replicas, weak scaling);
`value` is the max-over-ranks time divided by the number of clusters.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "anchor-select+fit s per cluster (mixed vs FP64 GPU) at fixed pair error; GB/s, TC util"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="c5")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ao-eval", action="store_true",
                    help="skip the standalone eval_ao timing over the whole grid")
    ap.add_argument("--widened", action="store_true",
                    help="also time the widened rows on this workload: the grid Coulomb metric of the "
                         "fitted Theta, the FP64 density (column-normalized) sketch and the FP64 "
                         "quadrature sketch with an occupied-orbital axis")
    ap.add_argument("--mode", choices=("auto", "sharded", "replicas"), default="auto",
                    help="N > 1: shard one cluster's grid over the ranks (auto) or run one cluster "
                         "per rank")
    ap.add_argument("--ao-eval-points", type=int, default=0,
                    help="time eval_ao on a contiguous slice of this many points from the middle of "
                         "the grid instead of the whole grid (small cases for profiling; 0 = whole grid)")
    ap.add_argument("--ao-eval-only", action="store_true",
                    help="print only the eval_ao timings (profiling the standalone evaluator)")
    ap.add_argument("--max-points", type=int, default=0,
                    help="keep every k-th grid point so that at most this many remain "
                         "(small cases for profiling; 0 = full grid)")
    return ap.parse_args()


MAX_POINTS = 0


def workload(cfg_key):
    from mp_isdf_b200 import inputs
    mol, pts, w, cfg = inputs.make_config(cfg_key)
    if MAX_POINTS and len(pts) > MAX_POINTS:
        stride = -(-len(pts) // MAX_POINTS)
        pts, w = pts[::stride].copy(), w[::stride].copy()
    names, factors = inputs.parse_axes(cfg["axes"])
    return mol, pts, w, cfg, names, factors


def workload_desc(cfg_key, cfg, mol, pts, w, names, precision):
    if cfg["algorithm"] == "rand_sketch":
        algo = f"rand_sketch quadrature rank {cfg['rank']} oversampling {cfg['oversampling']}"
    else:
        algo = f"{cfg['algorithm']} rank {cfg['rank']}"
    return {
        "workload": f"{cfg_key} {cfg['name']}: synthetic cc-pVDZ-shaped basis ({mol.nao} AOs), "
                    f"level-{cfg['level']} stand-in grid ({len(pts)} points, "
                    f"{int(np.count_nonzero(w))} nonzero-weight), axes {cfg['axes']}, {algo}",
        "nao": mol.nao, "grid_points": int(len(pts)), "axes": cfg["axes"], "algorithm": cfg["algorithm"],
        "anchor_rank": cfg["rank"],
        "sketch_rows": cfg["rank"] + cfg["oversampling"] if cfg["algorithm"] == "rand_sketch" else None,
        "precision": precision, "l2_policy": "working set >> L2 (126 MB); 256 MB L2 flush before every timed step",
    }


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i - 5] for r in self.rows for i in range(5, 9)
                          if r[i].lower() in ("active", "1")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# roofline bookkeeping
# ---------------------------------------------------------------------------
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


# DRAM bytes per kept grid point of one launch, from an ncu capture of the
# (H2O)64 case cut to 397312 grid points / 363237 kept points
# (dram__bytes_read.sum + dram__bytes_write.sum = 28.1 MB + 3737.3 MB); the
# kernel streams per-point data, so the traffic scales with the points.
MEASURED_TRAFFIC_PER_POINT = {"project_tc_grad": 10366.0}
TRAFFIC_SOURCE = "ncu dram bytes of a 363237-kept-point capture, scaled by kept points"

# ncu figures of the adjoint's fused grid kernel (one launch, --set full) on
# the (H2O)64 basis with the C5 anchors, grid cut to 60000 points
ADJOINT_PROFILE = {
    "kernel": "adjoint_grid_kernel<2, 12, 1>",
    "workload": "(H2O)64, 1536 AOs, 10 anchors, 60000 grid points",
    "issue_active_frac": 0.251, "fp64_pipe_frac": 0.132, "warps_active_frac": 0.125,
    "registers_per_thread": 255, "summary": "profiles/adjoint_grid_kernel_c5_fp64.md",
}


def inputs_axis_comp(name):
    return {"ao": 0, "dx": 1, "dy": 2, "dz": 3}[name]


def k_chunks(mol):
    """K-chunks of 32 AO slots of the fused kernel: whole contractions of one
    shell, packed in shell order (the library's chunk layout rule)."""
    chunks, used = 0, 0
    for b in mol.bas:
        ns, nctr = 2 * int(b[1]) + 1, int(b[3])
        j = 0
        while j < nctr:
            room = (32 - used) // ns
            if room == 0:
                chunks, used = chunks + 1, 0
                continue
            take = min(room, nctr - j)
            used += take * ns
            j += take
    return chunks + (1 if used or not chunks else 0)


def algorithmic(family, cfg, mol, n_kept, naxes, ell, k, precision="fp64"):
    """(bound, units per kernel family over one step, unit).  Bytes are the
    minimal HBM traffic of the family's outputs/inputs; flops are 2*M*N*K."""
    nao = mol.nao
    d = naxes * nao
    if family.startswith("ao_axis"):
        s = 8 if family.endswith("f64") else 4
        return "hbm", n_kept * d * s + n_kept * 24, "bytes"
    if family.startswith("ao_eval"):
        s = 8 if family.endswith("f64") else 4
        if precision == "mixed":
            # the mixed step evaluates FP64 AO values at the k anchors only
            return "hbm", k * nao * s + k * 24, "bytes"
        # FP64 step: the fit's AO values of every kept point and the anchors'
        return "hbm", (n_kept + k) * nao * s + (n_kept + k) * 24, "bytes"
    if family == "gemm_f64":
        # sketch projection (reads F once) + fit Gram (reads Phi once)
        return "hbm", n_kept * d * 8 + n_kept * nao * 8, "bytes"
    if family.startswith("sketch_tc") or family.startswith("fit_tc"):
        return "tensor", 2.0 * n_kept * d * 2 * ell * 3, "flop"
    if family.startswith("qrcp_sketch_update"):
        return "hbm", sum(2 * (ell - j + 1) * n_kept * 8 for j in range(ell + 1)), "bytes"
    if family == "sketch_combine":
        if precision == "mixed":
            # FP32 projections + 4 FP32 squared norms in, FP64 sketch column
            # and its error bound out
            return "hbm", n_kept * (naxes * 2 * ell * 4 + 16 + ell * 8 + 8), "bytes"
        return "hbm", n_kept * (naxes * 2 * ell + ell) * 8, "bytes"
    if family == "gram_tiles":
        # stored split-BF16 AO tiles read once, G written once
        return "hbm", -(-n_kept // 128) * k_chunks(mol) * 16384 + n_kept * k * 4, "bytes"
    if family == "fit_point":
        return "hbm", n_kept * k * 8 * 4, "bytes"
    return "hbm", 0, "bytes"


# ---------------------------------------------------------------------------
# CPU baseline (oracle restatement, bounded sample)
# ---------------------------------------------------------------------------
def time_adjoint(ctx, mol, x, wt, anchors, cfg, steps=3):
    """Nuclear gradient of E = sum_g w_g rho_ISDF(g)^2 for the config's seeded
    density (tr(DS) = electrons, S by grid quadrature), timed with CUDA events."""
    import torch
    from mp_isdf_b200 import inputs
    nao = mol.nao
    S = torch.zeros(nao, nao, dtype=torch.float64, device=x.device)
    for i in range(0, x.shape[0], 65536):
        xb = x[i:i + 65536].contiguous()
        phi = torch.empty(xb.shape[0], nao, dtype=torch.float64, device=x.device)
        ctx.eval_ao(xb, phi)
        S += phi.T @ (phi * wt[i:i + 65536, None])
    dm = inputs.random_density(mol, S.cpu().numpy(), cfg["electrons"], cfg["seed"])
    ctx.energy_gradient(x, wt, anchors, dm)
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        e, g = ctx.energy_gradient(x, wt, anchors, dm)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) / 1e3)
    return {"s": statistics.mean(times), "step_times_s": times, "energy": e,
            "grad_norm": float(np.linalg.norm(g)), "form": "FP64, fused grid pass: AO values and gradients recomputed per 128-point tile, never stored",
            "electrons": cfg["electrons"], "ncu": ADJOINT_PROFILE}


def _event_time(fn, reps=2):
    """Seconds of the last of `reps` calls, CUDA events around each."""
    import torch
    out, t = None, 0.0
    for _ in range(reps):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / 1e3
    return out, t


def time_ao_eval(ctx, mol, x, hbm, points=0):
    """Standalone AO evaluation (the eval_ao / eval_ao_gradient boundary) over
    every grid point of the workload (or a contiguous slice of `points` from
    the middle of the grid): FP64 values (Ng, nao) and FP32 values plus
    gradients (Ng, nao) + (3, Ng, nao), CUDA events around the last of three
    calls.  Algorithmic bytes: the output written plus 24 B of coordinates
    read per point; the roofline is HBM."""
    import torch
    if 0 < points < x.shape[0]:
        lo = (x.shape[0] - points) // 2
        x = x[lo:lo + points].contiguous()
    n, nao = x.shape[0], mol.nao
    out = {}
    for name, dt, grad in (("fp64_values", torch.float64, False), ("fp32_values_gradients", torch.float32, True)):
        es = 8 if dt == torch.float64 else 4
        v = torch.empty(n, nao, dtype=dt, device=x.device)
        g = torch.empty(3, n, nao, dtype=dt, device=x.device) if grad else None
        _, t = _event_time(lambda: ctx.eval_ao(x, v, g), reps=3)
        units = n * nao * es * (4 if grad else 1) + n * 24
        out[name] = {"ms": t * 1e3, "points": int(n), "algorithmic_bytes": int(units),
                     "achieved_gbs": units / t / 1e9, "peak_gbs": hbm, "frac": units / t / 1e9 / hbm}
        del v, g
        torch.cuda.empty_cache()
    return out


def time_widened(ctx, mol, x, wt, w, theta, k, n_kept, cfg):
    """The rows widened beyond the selection + fit path, on the bench workload:
    the grid Coulomb metric of the fitted Theta (python/isdf.py:48-68), the FP64
    density_col_norm sketch (importance = |w| times a seeded factor in
    [0.5, 1.5]), the FP64 quadrature sketch over the ao + occ axes (a seeded
    orthogonal nao x nao MO matrix, nocc = electrons / 2) and, for bases of at
    most 256 AOs, RBRP-ID over the kept points."""
    import torch
    from mp_isdf_b200 import capi
    keep = torch.as_tensor(w != 0, device=x.device)
    xk, wk = x[keep].contiguous(), wt[keep].contiguous()
    th = theta[:k * n_kept].view(k, n_kept)
    _, t_metric = _event_time(lambda: ctx.grid_metric(xk, wk, th), reps=1)
    rng = np.random.default_rng(cfg["seed"])
    imp = torch.as_tensor(np.abs(w) * rng.uniform(0.5, 1.5, len(w)), device=x.device)
    ov = cfg.get("oversampling", 16)
    (piv_d, _), t_dens = _event_time(lambda: ctx.select(
        x, wt, algorithm="rand_sketch_density_col_norm", axes=("ao",), max_rank=k, oversampling=ov,
        seed=cfg.get("sketch_seed", 7), point_importance=imp))
    nocc = max(1, int(cfg.get("electrons", 2 * k)) // 2)
    mo, _ = np.linalg.qr(rng.normal(size=(mol.nao, mol.nao)))
    (piv_o, _), t_occ = _event_time(lambda: ctx.select(
        x, wt, algorithm="rand_sketch", axes=("ao", "occ"), max_rank=k, oversampling=ov,
        seed=cfg.get("sketch_seed", 7), mo_coeff=np.ascontiguousarray(mo), nocc=nocc))
    # FP64 roofline denominator: a cuBLAS DGEMM burst on this GPU (the measured
    # peaks file holds HBM and BF16 only)
    A = torch.randn(8192, 8192, dtype=torch.float64, device=x.device)
    _, t_gemm = _event_time(lambda: A @ A, reps=3)
    fp64_peak = 2.0 * 8192 ** 3 / t_gemm / 1e12
    pairs = float(n_kept) * n_kept
    # the metric of one set sums each unordered pair once: the upper tiles and,
    # at weight 1/2, the diagonal tiles (256 points for k <= 16, 128 for k <= 32,
    # else 64), so the work counted is the pairs actually formed
    tile = 256 if k <= 16 else 128 if k <= 32 else 64
    pairs_summed = pairs / 2 + float(n_kept) * tile / 2
    flops_pair = 8 + 2 * k      # 3 differences, r^2 (1 mul + 2 FMA), k FMAs; rsqrt counted once
    achieved = pairs_summed * flops_pair / t_metric / 1e12
    # CPU beside it: the oracle's restatements on bounded samples, scaled
    from oracle import oracle as O
    keep_idx = np.flatnonzero(w != 0)
    rs = np.random.default_rng(1)
    sub = np.sort(rs.choice(keep_idx, size=min(12000, len(keep_idx)), replace=False))
    th_h = th.cpu().numpy()
    pos = np.searchsorted(keep_idx, sub)
    t0 = time.perf_counter()
    O.grid_coulomb_metric(th_h[:, pos], np.asarray(x[keep].cpu())[pos], w[sub])
    cpu_metric = (time.perf_counter() - t0) * (len(keep_idx) / len(sub)) ** 2
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    sub2 = np.sort(rs.choice(keep_idx, size=min(3000, len(keep_idx)), replace=False))
    pts_h = np.asarray(x.cpu())
    t0 = time.perf_counter()
    O.select_density_sketch(oc, pts_h[sub2], w[sub2], imp.cpu().numpy()[sub2], normalized=True, max_rank=k,
                            oversampling=ov, seed=cfg.get("sketch_seed", 7))
    cpu_dens = (time.perf_counter() - t0) * len(keep_idx) / len(sub2)
    t0 = time.perf_counter()
    sc = O.occ_axis_scales(oc, pts_h[sub2], w[sub2], [0, 4], mo, nocc)
    f = O.occ_features(oc, pts_h[sub2], [0, 4], mo, nocc, sc)
    O.select_rand_sketch_features(f, sub2, w[sub2], k + ov, ov, cfg.get("sketch_seed", 7), max_rank=k)
    cpu_occ = (time.perf_counter() - t0) * len(keep_idx) / len(sub2)
    cores = O.lib().oracle_num_threads()
    rbrp = None
    if mol.nao <= 256:
        # RBRP-ID over the kept points (AO pair rows nao (nao + 1) / 2 long)
        pk, wk_h = pts_h[keep_idx], w[keep_idx]
        r, t_rbrp = _event_time(lambda: capi.rbrp_points(ctx, pk, wk_h, max_rank=k, block_size=16,
                                                         compute_id=True), reps=2)
        aos = oc.eval_ao(pts_h[sub2])
        t0 = time.perf_counter()
        O.rbrp_ao(aos, w[sub2], max_rank=k, block_size=16, compute_id=True)
        cpu_rbrp = (time.perf_counter() - t0) * len(keep_idx) / len(sub2)
        rbrp = {"s": t_rbrp, "points": int(len(keep_idx)), "rank": len(r["indices"]), "status": r["status"],
                "relative_residual": r["relative_residual"],
                "cpu_baseline": {"value": cpu_rbrp, "unit": "s", "cores": cores, "kind": "port",
                                 "sample": f"oracle (explicit pair rows) on {len(sub2)} points, linear in points"}}
    return {
        "rbrp_id": rbrp,
        "grid_metric": {"s": t_metric, "points": n_kept, "anchors": k, "metric_pairs_per_s": pairs / t_metric,
                        "pairs_summed": pairs_summed, "pairs_summed_per_s": pairs_summed / t_metric,
                        "form": "FP64 all-pairs potential over the upper tiles (K symmetric) on the FP64 "
                                "tensor cores (DMMA) + FP64 GEMM",
                        "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                                     "frac": achieved / fp64_peak, "flops_per_pair": flops_pair,
                                     "peak_source": "cuBLAS DGEMM 8192^3 burst, measured here"},
                        "cpu_baseline": {"value": cpu_metric, "unit": "s", "cores": 1, "kind": "port",
                                         "sample": f"oracle NumPy restatement on {len(sub)} points, time x "
                                                   f"(n/{len(sub)})^2"}},
        "density_col_norm_sketch_fp64": {"s": t_dens, "anchors": [int(a) for a in piv_d],
                                         "cpu_baseline": {"value": cpu_dens, "unit": "s", "cores": cores,
                                                          "kind": "port", "sample": f"oracle on {len(sub2)} "
                                                          "points, linear in points"}},
        "occ_axis_sketch_fp64": {"s": t_occ, "axes": "ao,occ", "nocc": nocc, "anchors": [int(a) for a in piv_o],
                                 "cpu_baseline": {"value": cpu_occ, "unit": "s", "cores": cores, "kind": "port",
                                                  "sample": f"oracle on {len(sub2)} points, linear in points"}},
    }


def golden_compare(cfg_key, piv, theta, n_kept, k, pair_rel):
    """This form's anchors, Theta and pair error against the FP64 oracle's
    golden fixture of the configuration (tests/golden/<key>.npz, written by
    tests/golden/make_goldens.py): Theta at the fixture's sample of columns,
    relative to its largest entry, and the pair error relative to the
    oracle's.  None for reduced grids or configurations without a fixture."""
    path = ROOT / "tests" / "golden" / f"{cfg_key}.npz"
    if MAX_POINTS or not path.exists():
        return None
    g = np.load(path)
    ref = [int(a) for a in g["anchors"]]
    gold = float(g["pair_relative"])
    out = {"fixture": f"tests/golden/{cfg_key}.npz", "oracle_pair_relative": gold,
           "oracle_condition": float(g["condition"]), "oracle_min_step_gap": float(np.min(g["step_gap"]))}
    div = next((j for j, (a, b) in enumerate(zip(piv, ref)) if a != b), None)
    if div is None and len(piv) != len(ref):
        div = min(len(piv), len(ref))
    out["anchors_equal_oracle"] = div is None
    if div is not None:
        out["first_divergent_pivot"] = div
        out["oracle_gap_at_divergence"] = float(g["step_gap"][div]) if div < len(g["step_gap"]) else None
        out["theta_rel_err_vs_oracle"] = None
        out["pair_rel_err_vs_oracle"] = None
        return out
    import torch
    pos = torch.as_tensor(g["theta_pos"], device=theta.device)
    th = theta[: k * n_kept].view(k, n_kept)[:, pos].cpu().numpy()
    sample = g["theta_sample"]
    out["theta_rel_err_vs_oracle"] = float(np.abs(th - sample).max() / np.abs(sample).max())
    out["theta_columns_compared"] = int(sample.shape[1])
    out["pair_rel_err_vs_oracle"] = abs(pair_rel - gold) / gold
    return out


def selection_kwargs(cfg, names, factors, precision):
    """isdf_select arguments of a config (algorithm, axes, rank, sketch)."""
    return dict(algorithm=cfg["algorithm"], axes=names, axis_weights=factors, max_rank=cfg["rank"],
                oversampling=cfg.get("oversampling", 16), seed=cfg.get("sketch_seed", 7),
                batch_size=cfg.get("online_batch", 128), precision=precision)


def cpu_sample_size(cfg, mol, names):
    """Sample size of the CPU restatement run and whether it fits the host:
    dense pair QR materialises d^2 x n doubles as the reference does."""
    if cfg["algorithm"] == "rand_sketch":
        return 32768, True
    d2 = (len(names) * mol.nao) ** 2
    n = 1000
    return n, d2 * n * 8 <= 2e9


def cpu_sample(mol, pts, w, names, factors, cfg, n_sample=4000, seed=0):
    """Time the oracle's restatement of the same path on `n_sample` nonzero
    points, scaled to the full kept-point count: axis norms, Khatri-Rao sketch,
    dgeqp3 of the sketch, AO values + Gram fit.  Returns (seconds/cluster, cores, sample)."""
    from oracle import oracle as O
    axes = [O.AXIS_CODES[a] for a in names]
    keep = np.flatnonzero(w != 0)
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(keep, size=min(n_sample, len(keep)), replace=False))
    p, ww = pts[idx], w[idx]
    ctx = O.OracleContext(mol.atm, mol.bas, mol.env)
    t0 = time.perf_counter()
    scales = O.axis_scales(ctx, p, ww, axes, factors, exact_order=False) if len(axes) > 1 else None
    if cfg["algorithm"] == "rand_sketch":
        piv = O.select_rand_sketch(ctx, p, ww, axes, max_rank=cfg["rank"],
                                   oversampling=cfg["oversampling"], seed=cfg.get("sketch_seed", 7),
                                   scales=scales)
        scale = len(keep) / len(idx)
        how = "linear in points"
    else:
        # dgeqp3 of the explicit d^2 x n pair matrix, as the reference: its
        # cost grows as n * min(d^2, n)
        piv = O.select_qrcp_dense(ctx, p, ww, axes, max_rank=cfg["rank"], scales=scales)
        d2 = (len(axes) * mol.nao) ** 2
        scale = len(keep) / len(idx) * min(d2, len(keep)) / min(d2, len(idx))
        how = "scaled by n*min(d^2, n)"
    O.gram_fit(ctx, p, ww, p[piv], ww[piv])
    dt = time.perf_counter() - t0
    return dt * scale, O.lib().oracle_num_threads(), \
        f"{len(idx)} of {len(keep)} nonzero-weight points (uniform random), time x{scale:.1f} ({how})"


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    mol, pts, w, cfg, names, factors = workload(args.config)
    precision = args.precision or "fp64"
    vals = []
    cores = 1
    sample = ""
    n_sample, feasible = cpu_sample_size(cfg, mol, names)
    if not feasible:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's qrcp on this config "
                          "materialises a d^2 x n pair matrix that exceeds host memory"}), flush=True)
        return
    # the timed steps cycle through the point samples that the default run's cpu_baseline
    # leg times (seeds 0..2), so both legs time the same work
    for i in range(args.warmup + args.steps):
        seed = (i - args.warmup) % 3 if i >= args.warmup else i % 3
        v, cores, sample = cpu_sample(mol, pts, w, names, factors, cfg, n_sample=n_sample, seed=seed)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": workload_desc(args.config, cfg, mol, pts, w, names, precision),
        "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                         "sample": sample + f"; median of {len(vals)} samples (seeds 0..2 in turn)",
                         "min": min(vals), "max": max(vals),
                         "spread": (max(vals) - min(vals)) / value},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CMake build needs network FetchContent (Kokkos, LAPACK++, SLATE, "
                "libcint, MAGMA); timed is the C++/OpenMP restatement of its algorithm in oracle/",
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    from mp_isdf_b200 import capi
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    mol, pts, w, cfg, names, factors = workload(args.config)
    forms = [args.precision] if args.precision else ["mixed", "fp64"]
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device=dev)
    if args.ao_eval_only:
        if rank == 0:
            print(json.dumps({"config": args.config,
                              "ao_eval": time_ao_eval(ctx, mol, x, peaks()[0], args.ao_eval_points)}), flush=True)
        return
    wt = torch.tensor(w, device=dev)
    n = len(pts)
    n_kept = int(np.count_nonzero(w))
    k = cfg["rank"]
    ell = k + cfg.get("oversampling", 16)
    theta = torch.empty(k * n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def sel_kw(precision):
        return selection_kwargs(cfg, names, factors, precision)

    # every selection algorithm shards (the sketch QR, the pair-space QR)
    sharded = args.mode == "sharded" or (args.mode == "auto" and world > 1)
    if sharded:
        # one cluster per step, its grid split into contiguous per-rank shards
        from mp_isdf_b200.sharded import CudaBackend, LocalComm, TorchComm, select_fit_sharded
        edges = np.linspace(0, n, world + 1).astype(np.int64)
        lo, hi = int(edges[rank]), int(edges[rank + 1])
        xs, ws = x[lo:hi].contiguous(), wt[lo:hi].contiguous()
        comm = TorchComm() if world > 1 else LocalComm()
        backend = CudaBackend(ctx)

        def step(precision, want_error=False):
            r = select_fit_sharded(backend, comm, xs, ws, lo, n, want_error=want_error, **sel_kw(precision))
            return r.anchors, r.select_info, r.fit_info, r
    else:
        def step(precision, want_error=False):
            # selection + fit in one library call (isdf_select_fit)
            piv, sinfo, finfo = ctx.select_fit(x, wt, theta, want_error=want_error, **sel_kw(precision))
            return piv, sinfo, finfo, None

    results = {}
    for precision in forms:
        for _ in range(args.warmup):
            step(precision)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        capi.profile_enable(True)
        capi.profile_read()
        sampler = ClockSampler(local_rank)
        sampler.start()
        times = []
        prof_all, step_phases = {}, []
        launches0 = capi.launch_count()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            piv, sinfo, finfo, _ = step(precision)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
            # per-step profile (read after the timed region)
            p = capi.profile_read()
            step_phases.append({nm[6:]: round(v[0], 3) for nm, v in p.items() if nm.startswith("phase:")})
            for name, (ms, cnt) in p.items():
                acc = prof_all.setdefault(name, [0.0, 0])
                acc[0] += ms
                acc[1] += cnt
        launched = capi.launch_count() - launches0
        clocks = sampler.stop()
        capi.profile_enable(False)
        prof_all = {k: tuple(v) for k, v in prof_all.items()}
        # "phase:" scopes time host+device phases of the call on the stream;
        # the rest are kernel families
        prof = {k: v for k, v in prof_all.items() if not k.startswith("phase:")}
        phases = {k[6:]: v for k, v in prof_all.items() if k.startswith("phase:")}
        total = sum(times)
        if world > 1:
            t = torch.tensor([total], device=dev, dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            total = float(t.item())
        # pair-space error of this form's Theta, evaluated with FP64 AO values (untimed)
        if sharded:
            _, _, finfo, r = step(precision, want_error=True)
            pl2, prel = r.pair_l2, r.pair_relative
        else:
            pl2, prel = ctx.pair_error(x, wt, piv, theta)
        einfo = {"pair_l2": pl2, "pair_relative": prel, "fit_path": finfo.fit_path,
                 "mixed_bound": finfo.mixed_bound,
                 "vs_oracle": golden_compare(args.config, [int(p) for p in piv], theta, n_kept, k, prel)
                 if not sharded else None}
        torch.cuda.synchronize()
        results[precision] = dict(total=total, times=times, prof=prof, phases=phases, step_phases=step_phases,
                                  launches=launched / max(args.steps, 1),
                                  clocks=clocks,
                                  piv=[int(p) for p in piv], sinfo=sinfo, einfo=einfo)

    head = forms[0]
    res = results[head]
    # replicas: each rank times its own cluster; sharded: all ranks one cluster
    per_cluster = res["total"] / args.steps / (1 if sharded else world)
    launches = int(round(res["launches"]))   # this library's kernel launches per timed step

    # e2e through the host-buffer C-ABI (headline form)
    e2e = None
    if not args.no_e2e and sharded:
        # each rank uploads its shard from pinned memory and downloads its Theta columns
        pts_h = torch.from_numpy(np.ascontiguousarray(pts[lo:hi])).pin_memory()
        w_h = torch.from_numpy(np.ascontiguousarray(w[lo:hi])).pin_memory()
        e2e_times = []
        for i in range(max(1, min(3, args.steps)) + 1):
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            t0 = time.perf_counter()
            xd = pts_h.to(dev, non_blocking=True)
            wd = w_h.to(dev, non_blocking=True)
            r = select_fit_sharded(backend, comm, xd, wd, lo, n, want_error=False, **sel_kw(head))
            th = r.theta.cpu()
            dt = time.perf_counter() - t0
            if i:
                e2e_times.append(dt)
        t = torch.tensor([statistics.mean(e2e_times)], device=dev, dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e = {"value": float(t.item()), "unit": "s",
               "h2d_bytes_per_step": int(pts_h.numel() * 8 + w_h.numel() * 8),
               "d2h_bytes_per_step": int(th.numel() * 8 + 8 * len(r.anchors)),
               "path": "grid-sharded select+fit (shard from pinned memory, Theta columns back; max over ranks)"}
    elif not args.no_e2e:
        # pinned host buffers: inputs copied in by each call, Theta copied out
        pts_h = torch.from_numpy(np.ascontiguousarray(pts)).pin_memory().numpy()
        w_h = torch.from_numpy(np.ascontiguousarray(w)).pin_memory().numpy()
        th_h = torch.empty(k * n, dtype=torch.float64).pin_memory().numpy()
        e2e_times = []
        for i in range(max(1, min(3, args.steps)) + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            piv_h, th, _, _ = ctx.select_fit_host(pts_h, w_h, want_error=False, out=th_h, **sel_kw(head))
            dt = time.perf_counter() - t0
            if i:
                e2e_times.append(dt)
        h2d = pts_h.nbytes + w_h.nbytes
        d2h = th.nbytes + 8 * len(piv_h)
        e2e = {"value": statistics.mean(e2e_times) / world, "unit": "s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "isdf_select_fit_host (pinned host buffers, wall clock)"}

    adjoint = None
    if cfg.get("electrons") and not args.no_adjoint and world == 1:
        adjoint = time_adjoint(ctx, mol, x, wt, results[head]["piv"], cfg)

    ao_eval = None
    if world == 1 and not args.no_ao_eval:
        ao_eval = time_ao_eval(ctx, mol, x, peaks()[0], args.ao_eval_points)

    widened = None
    if args.widened and world == 1:
        widened = time_widened(ctx, mol, x, wt, w, theta, k, n_kept, cfg)

    if rank != 0:
        return
    hbm, bf16, peak_kind = peaks()
    fams = sorted(res["prof"].items(), key=lambda kv: -kv[1][0])
    tot_ms = sum(v[0] for v in res["prof"].values())
    kernels = {}
    nao_pad = k_chunks(mol) * 32   # K slots of the fused kernel
    ncomp = len({inputs_axis_comp(a) for a in names})
    for name, (ms, cnt) in fams:
        t_launch = ms / cnt / 1e3
        entry = {"ms_per_step": ms / args.steps, "launches_per_step": cnt / args.steps,
                 "share": ms / tot_ms, "per_launch_ms": ms / cnt}
        if name == "project_tc_grad":
            # Fused AO evaluation + projection: its roofline is that of the AO
            # evaluation it replaces, the minimal HBM output of the unfused
            # evaluator (n * nao * components * 4 B FP32).
            units = n_kept * mol.nao * ncomp * 4 + n_kept * 24
            nt = 16 if 2 * ell <= 16 else 32 if 2 * ell <= 32 else 64
            useful = 2.0 * n_kept * len(names) * mol.nao * 2 * ell
            issued = 2.0 * n_kept * len(names) * nao_pad * nt * 3
            entry["roofline"] = {
                "bound": "hbm", "limiter": "instruction issue (ncu: ALU/FMA/LSU pipes, long-scoreboard and "
                                          "barrier stalls), not DRAM or the tensor pipe",
                "achieved": units / t_launch / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": units / t_launch / 1e9 / hbm, "algorithmic_bytes_per_launch": units,
                "algorithmic_model": f"n_kept*nao*{ncomp} components*4 B (unfused AO output) + n_kept*24 B",
                "traffic": MEASURED_TRAFFIC_PER_POINT[name] * n_kept,
                "traffic_source": TRAFFIC_SOURCE,
                "tensor": {"useful_tflops": useful / t_launch / 1e12,
                           "issued_tflops": issued / t_launch / 1e12,
                           "issued_frac_of_bf16": issued / t_launch / 1e12 / bf16,
                           "issued_model": "3 split-BF16 products x 2*n*(naxes*K_slots)*N_tile"}}
        else:
            bound, units, unit = algorithmic(name, cfg, mol, n_kept, len(names), ell, k, head)
            if units:
                ach, pk, u = ((units / t_launch / 1e9, hbm, "GB/s") if bound == "hbm"
                              else (units / t_launch / 1e12, bf16, "TFLOP/s"))
                per_launch = units / max(cnt / args.steps, 1)
                entry["roofline"] = {"bound": bound, "achieved": ach * (per_launch / units), "peak": pk,
                                     "unit": u, "frac": ach * (per_launch / units) / pk,
                                     "algorithmic_per_launch": per_launch,
                                     "traffic": (MEASURED_TRAFFIC_PER_POINT[name] * n_kept
                                                 if name in MEASURED_TRAFFIC_PER_POINT else None)}
        kernels[name] = entry
    top = fams[0][0]
    rl = kernels[top].get("roofline") or {}
    roofline = dict(rl, kernel=top, peak_source=f"{peak_kind} (MEASURED_PEAKS.json)") if rl else None
    cpu = None
    if not args.no_cpu and world == 1:
        n_sample, feasible = cpu_sample_size(cfg, mol, names)
        if feasible:
            vals = []
            for seed in range(3):
                v, cores, sample = cpu_sample(mol, pts, w, names, factors, cfg, n_sample=n_sample, seed=seed)
                vals.append(v)
            med = statistics.median(vals)
            cpu = {"value": med, "unit": "s", "cores": cores, "kind": "port",
                   "sample": sample + "; median of 3 samples (seeds 0..2)",
                   "min": min(vals), "max": max(vals), "spread": (max(vals) - min(vals)) / med}
        else:
            cpu = {"value": None, "unit": "s", "cores": None, "kind": "port",
                   "sample": "infeasible: the reference's explicit d^2 x n pair matrix does not fit host memory"}
    forms_out = {}
    for p, r in results.items():
        forms_out[p] = {"s_per_cluster": r["total"] / args.steps / world,
                        "step_times_s": r["times"], "anchors": r["piv"],
                        "pair_relative": r["einfo"]["pair_relative"], "pair_l2": r["einfo"]["pair_l2"],
                        "fit_path": r["einfo"]["fit_path"], "mixed_fit_bound": r["einfo"]["mixed_bound"],
                        "vs_oracle": r["einfo"]["vs_oracle"],
                        "sketch_columns_reverified": r["sinfo"].verifications,
                        "precision_used": "mixed" if r["sinfo"].precision_used else "fp64",
                        "phases_ms_per_step": {k: v[0] / args.steps for k, v in r["phases"].items()},
                        "phases_ms_each_step": r["step_phases"],
                        "clocks": r["clocks"]}
    extra = {}
    if "mixed" in results and "fp64" in results:
        m, f = results["mixed"], results["fp64"]
        extra = {"speedup_mixed_vs_fp64": f["total"] / m["total"],
                 "anchors_identical": m["piv"] == f["piv"],
                 "pair_relative_rel_diff": abs(m["einfo"]["pair_relative"] - f["einfo"]["pair_relative"])
                 / f["einfo"]["pair_relative"]}
    line = {
        "metric": METRIC, "value": per_cluster, "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["total"] / args.steps * 1e3,
        "higher_is_better": False, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
        "dtype": "f64" if head == "fp64" else "bf16x3+f32+f64", "data": "synthetic",
        "config": workload_desc(args.config, cfg, mol, pts, w, names, head)
        | {"parallelism": (f"grid shards x{world} (one cluster)" if sharded else f"replicas x{world}")},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
        "clocks": res["clocks"], "kernels": kernels, "forms": forms_out, **extra,
        "theta_rel_err_vs_oracle": (res["einfo"]["vs_oracle"] or {}).get("theta_rel_err_vs_oracle"),
        "pair_rel_err_vs_oracle": (res["einfo"]["vs_oracle"] or {}).get("pair_rel_err_vs_oracle"),
        "adjoint": adjoint, "ao_eval": ao_eval,
    }
    if widened is not None:
        line["widened"] = widened
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    global MAX_POINTS
    MAX_POINTS = args.max_points
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
