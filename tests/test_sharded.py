"""Grid-sharded selection + fit (mp_isdf_b200.sharded).

CPU: two or three gloo ranks (one of them possibly without grid points) run the
protocol -- the distributed pivoted QR or the gathered one -- with the oracle
backend and must give
the single-process oracle's anchors, Theta columns and pair error.  GPU: the
library's sharded phases with two shards in one process (threads standing in
for ranks, no collectives between kernels) against isdf_select_fit on the
whole grid.
"""
import json
import os
import socket
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

KW = dict(axes=("ao", "dx", "dy", "dz"), axis_weights=[1.0, 0.5, 0.5, 0.5], max_rank=6, oversampling=8,
          seed=4)


def _system():
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((2, 1, 1), seed=11)
    mol = inputs.build_tables(symbols, xyz)
    pts, w = inputs.becke_grid(symbols, xyz, level=0)
    return mol, pts, w


def _split(ng, size):
    edges = np.linspace(0, ng, size + 1).astype(int)
    return [(edges[r], edges[r + 1]) for r in range(size)]


def _gloo_rank(rank, size, port, out_dir, qr="distributed", empty_rank=-1):
    import datetime
    import torch
    import torch.distributed as dist
    from mp_isdf_b200.sharded import TorchComm, select_fit_sharded
    from sharded_helpers import OracleBackend
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=120))
    try:
        mol, pts, w = _system()
        bounds = _split(len(pts), size - (empty_rank >= 0))
        if empty_rank >= 0:   # this rank's shard holds no grid point at all
            bounds.insert(empty_rank, (bounds[empty_rank - 1][1], bounds[empty_rank - 1][1]) if empty_rank
                          else (0, 0))
        lo, hi = bounds[rank]
        res = select_fit_sharded(OracleBackend(mol), TorchComm(), torch.as_tensor(pts[lo:hi]),
                                 torch.as_tensor(w[lo:hi]), lo, len(pts), qr=qr, **KW)
        np.save(os.path.join(out_dir, f"theta{rank}.npy"), res.theta.numpy())
        with open(os.path.join(out_dir, f"res{rank}.json"), "w") as f:
            json.dump({"anchors": res.anchors.tolist(), "pair_relative": res.pair_relative,
                       "kept_offset": res.kept_offset, "counts": res.counts}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("size,qr,empty_rank", [
    (2, "distributed", -1),   # pivoted QR with the columns left on their ranks
    (2, "gathered", -1),      # the whole sketch gathered, the QR replicated
    (3, "distributed", 1),    # the middle rank owns no kept point
    (2, "distributed", 0),    # rank 0 owns no kept point
])
def test_gloo_ranks_match_single_process(size, qr, empty_rank):
    """The sharded protocol on gloo CPU ranks with the oracle backend gives
    the single-process oracle's anchors, Theta columns and pair error."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    mol, pts, w = _system()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_rank, args=(size, _free_port(), d, qr, empty_rank), nprocs=size, join=True,
                           start_method="spawn")
        res = [json.load(open(os.path.join(d, f"res{r}.json"))) for r in range(size)]
        thetas = [np.load(os.path.join(d, f"theta{r}.npy")) for r in range(size)]
    for r in range(1, size):
        assert res[r]["anchors"] == res[0]["anchors"]
    counts = res[0]["counts"]
    assert all((c == 0) == (r == empty_rank) for r, c in enumerate(counts)), counts
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    codes = [O.AXIS_CODES[a] for a in KW["axes"]]
    scales = O.axis_scales(oc, pts, w, codes, KW["axis_weights"])
    ref = O.select_rand_sketch(oc, pts, w, codes, max_rank=KW["max_rank"], oversampling=KW["oversampling"],
                               seed=KW["seed"], scales=scales)
    assert res[0]["anchors"] == ref
    keep = w != 0
    theta_ref, err = O.gram_fit(oc, pts[keep], w[keep], pts[ref], w[ref])
    theta = np.concatenate(thetas, axis=1)
    np.testing.assert_allclose(theta, theta_ref, rtol=1e-9, atol=1e-9 * np.abs(theta_ref).max())
    for r in range(size):
        np.testing.assert_allclose(res[r]["pair_relative"], err["relative"], rtol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,qr", [("mixed", "distributed"), ("fp64", "distributed"),
                                          ("mixed", "gathered"), ("fp64", "gathered")])
def test_cuda_phases_two_shards_match_select_fit(precision, qr):
    import threading
    import torch
    from mp_isdf_b200 import capi
    from mp_isdf_b200.sharded import CudaBackend, select_fit_sharded
    from sharded_helpers import ThreadComm
    mol, pts, w = _system()
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    theta = torch.zeros(KW["max_rank"] * len(pts), dtype=torch.float64, device="cuda")
    piv, _, finfo = ctx.select_fit(x, wt, theta, want_error=True, precision=precision, **KW)
    torch.cuda.synchronize()
    size = 2
    shared = ThreadComm.Shared(size)
    results, errors = [None] * size, []

    def run(rank):
        try:
            torch.cuda.set_device(0)
            c = capi.Context(mol.atm, mol.bas, mol.env)
            lo, hi = _split(len(pts), size)[rank]
            results[rank] = select_fit_sharded(CudaBackend(c), ThreadComm(rank, size, shared),
                                               x[lo:hi].contiguous(), wt[lo:hi].contiguous(), lo, len(pts),
                                               precision=precision, qr=qr, **KW)
            torch.cuda.synchronize()
        except Exception as e:  # surfaced below
            errors.append(e)
            shared.barrier.abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    np.testing.assert_array_equal(results[0].anchors, piv)
    np.testing.assert_array_equal(results[1].anchors, piv)
    th_sharded = torch.cat([r.theta for r in results], dim=1).cpu().numpy()
    k, n = len(piv), finfo.n_kept
    th_ref = theta[:k * n].view(k, n).cpu().numpy()
    scale = max(1.0, finfo.condition) ** 2
    rel = np.abs(th_sharded - th_ref).max() / np.abs(th_ref).max()
    assert rel <= (1e-5 if precision == "mixed" else 1e-12) * scale, rel
    assert abs(results[0].pair_relative - finfo.pair_relative) <= 1e-8 * finfo.pair_relative


@pytest.mark.gpu
def test_cuda_single_rank_local_comm():
    import torch
    from mp_isdf_b200 import capi
    from mp_isdf_b200.sharded import CudaBackend, LocalComm, select_fit_sharded
    mol, pts, w = _system()
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    res = select_fit_sharded(CudaBackend(ctx), LocalComm(), x, wt, 0, len(pts), precision="mixed", **KW)
    piv, _ = ctx.select(x, wt, precision="mixed", **KW)
    np.testing.assert_array_equal(res.anchors, piv)


# ---- the adjoint over grid shards -------------------------------------------------
ADJ_ANCHORS = [3, 40, 77, 120, 161, 205]   # kept-point positions used as anchors


def _adjoint_inputs():
    mol, pts, w = _system()
    keep = np.flatnonzero(w != 0)
    anchors = keep[ADJ_ANCHORS]
    c = np.random.default_rng(8).normal(size=(mol.nao, 4))
    dm = 0.05 * (c @ c.T)
    return mol, pts, w, anchors, dm


def _gloo_adjoint_rank(rank, size, port, out_dir, empty_rank):
    import datetime
    import torch
    import torch.distributed as dist
    from mp_isdf_b200.sharded import TorchComm, energy_gradient_sharded
    from sharded_helpers import OracleBackend
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=120))
    try:
        mol, pts, w, anchors, dm = _adjoint_inputs()
        bounds = _split(len(pts), size - (empty_rank >= 0))
        if empty_rank >= 0:
            bounds.insert(empty_rank, (0, 0))
        lo, hi = bounds[rank]
        e, g = energy_gradient_sharded(OracleBackend(mol), TorchComm(), torch.as_tensor(pts[lo:hi]),
                                       torch.as_tensor(w[lo:hi]), pts[anchors], w[anchors], dm)
        np.save(os.path.join(out_dir, f"grad{rank}.npy"), np.concatenate([[e], g.ravel()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size,empty_rank", [(2, -1), (3, 0)])
def test_gloo_adjoint_matches_oracle(size, empty_rank):
    """The sharded adjoint (per-rank partial sums, one all-reduce, the same
    anchor-side finish on every rank) on gloo CPU ranks with the oracle backend
    gives the single-process oracle's energy and nuclear gradient, also with a
    rank that holds no grid point."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    mol, pts, w, anchors, dm = _adjoint_inputs()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_adjoint_rank, args=(size, _free_port(), d, empty_rank), nprocs=size, join=True,
                           start_method="spawn")
        out = [np.load(os.path.join(d, f"grad{r}.npy")) for r in range(size)]
    for r in range(1, size):
        np.testing.assert_array_equal(out[r], out[0])
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    keep = w != 0
    e_ref = O.isdf_energy(oc, pts[keep], w[keep], pts[anchors], w[anchors], dm)
    g_ref = O.isdf_energy_gradient(oc, pts[keep], w[keep], pts[anchors], w[anchors], dm)
    np.testing.assert_allclose(out[0][0], e_ref, rtol=1e-11)
    np.testing.assert_allclose(out[0][1:].reshape(-1, 3), g_ref, rtol=0, atol=1e-10 * np.abs(g_ref).max())


@pytest.mark.gpu
def test_cuda_adjoint_two_shards_match_single_call():
    """The library's sharded adjoint entry points with two shards in one
    process (threads standing in for ranks) against isdf_energy_gradient on
    the whole grid, gradient and energy-only."""
    import threading
    import torch
    from mp_isdf_b200 import capi
    from mp_isdf_b200.sharded import CudaBackend, energy_gradient_sharded
    from sharded_helpers import ThreadComm
    mol, pts, w, anchors, dm = _adjoint_inputs()
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    e_ref, g_ref = ctx.energy_gradient(x, wt, anchors, dm)
    size = 2
    for want_grad in (True, False):
        shared = ThreadComm.Shared(size)
        results, errors = [None] * size, []

        def run(rank):
            try:
                torch.cuda.set_device(0)
                c = capi.Context(mol.atm, mol.bas, mol.env)
                lo, hi = _split(len(pts), size)[rank]
                results[rank] = energy_gradient_sharded(CudaBackend(c), ThreadComm(rank, size, shared),
                                                        x[lo:hi].contiguous(), wt[lo:hi].contiguous(),
                                                        pts[anchors], w[anchors], dm, want_grad)
                torch.cuda.synchronize()
            except Exception as e:  # surfaced below
                errors.append(e)
                shared.barrier.abort()

        threads = [threading.Thread(target=run, args=(r,)) for r in range(size)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors, errors
        for e, g in results:
            np.testing.assert_allclose(e, e_ref, rtol=1e-12)
            if want_grad:
                # the per-atom terms are FP64 atomic sums in an order that
                # varies between runs, and the gradient is a small difference
                # of large terms: 1e-10 of the largest component, as above
                np.testing.assert_allclose(g, g_ref, rtol=0, atol=1e-10 * np.abs(g_ref).max())
            else:
                assert not g.any()


# ---- the pair-space QR over grid shards -------------------------------------------
PQ_KW = dict(axes=("ao", "dx", "dy", "dz"), axis_weights=[1.0, 0.5, 0.5, 0.5], max_rank=6)


def _gloo_pairqr_rank(rank, size, port, out_dir, algorithm, empty_rank):
    import datetime
    import torch
    import torch.distributed as dist
    from mp_isdf_b200.sharded import TorchComm, select_fit_sharded
    from sharded_helpers import OracleBackend
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=120))
    try:
        mol, pts, w = _system()
        bounds = _split(len(pts), size - (empty_rank >= 0))
        if empty_rank >= 0:
            bounds.insert(empty_rank, (bounds[empty_rank - 1][1], bounds[empty_rank - 1][1]) if empty_rank
                          else (0, 0))
        lo, hi = bounds[rank]
        res = select_fit_sharded(OracleBackend(mol), TorchComm(), torch.as_tensor(pts[lo:hi]),
                                 torch.as_tensor(w[lo:hi]), lo, len(pts), algorithm=algorithm, **PQ_KW)
        np.save(os.path.join(out_dir, f"theta{rank}.npy"), res.theta.numpy())
        with open(os.path.join(out_dir, f"res{rank}.json"), "w") as f:
            json.dump({"anchors": res.anchors.tolist(), "pair_relative": res.pair_relative}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size,algorithm,empty_rank", [(2, "qrcp_dense", -1), (3, "qrcp_online", 1)])
def test_gloo_pair_qr_matches_oracle(size, algorithm, empty_rank):
    """The pair-space QR over gloo CPU ranks (per-step key all-gather, the
    leader's row by all-reduce, the same exact residual on every rank) with
    the oracle backend gives the single-process oracle's exact-norm pivots,
    Theta and pair error, also with a rank that owns no kept point."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    mol, pts, w = _system()
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_pairqr_rank, args=(size, _free_port(), d, algorithm, empty_rank), nprocs=size,
                           join=True, start_method="spawn")
        res = [json.load(open(os.path.join(d, f"res{r}.json"))) for r in range(size)]
        thetas = [np.load(os.path.join(d, f"theta{r}.npy")) for r in range(size)]
    for r in range(1, size):
        assert res[r]["anchors"] == res[0]["anchors"]
    oc = O.OracleContext(mol.atm, mol.bas, mol.env)
    codes = [O.AXIS_CODES[a] for a in PQ_KW["axes"]]
    keep = np.flatnonzero(w != 0)
    scales = O.axis_scales(oc, pts, w, codes, PQ_KW["axis_weights"])
    pos, _, gaps = O.pair_qrcp_exact(oc.axis_features(pts[keep], codes, scales), w[keep], PQ_KW["max_rank"])
    ref = [int(keep[p]) for p in pos]
    for j, (a, b) in enumerate(zip(res[0]["anchors"], ref)):
        if a != b:
            assert gaps[j] <= 1e-10, (j, a, b, gaps[j])
            return
    assert res[0]["anchors"] == ref
    theta_ref, err = O.gram_fit(oc, pts[keep], w[keep], pts[ref], w[ref])
    theta = np.concatenate([t for t in thetas if t.size], axis=1)
    np.testing.assert_allclose(theta, theta_ref, rtol=1e-9, atol=1e-9 * np.abs(theta_ref).max())
    for r in range(size):
        np.testing.assert_allclose(res[r]["pair_relative"], err["relative"], rtol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("algorithm,empty", [("qrcp_dense", False), ("qrcp_online", False), ("qrcp_dense", True)])
def test_cuda_pair_qr_two_shards_match_select_fit(algorithm, empty):
    """The library's sharded pair-space QR (isdf_pairqr_shard_*) with two
    shards in one process (threads standing in for ranks; with `empty` a third
    shard between them holds no grid point) against isdf_select_fit on the
    whole grid: the same anchors, Theta and pair error."""
    import threading
    import torch
    from mp_isdf_b200 import capi
    from mp_isdf_b200.sharded import CudaBackend, select_fit_sharded
    from sharded_helpers import ThreadComm
    mol, pts, w = _system()
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    theta = torch.zeros(PQ_KW["max_rank"] * len(pts), dtype=torch.float64, device="cuda")
    piv, _, finfo = ctx.select_fit(x, wt, theta, want_error=True, precision="fp64", algorithm=algorithm, **PQ_KW)
    torch.cuda.synchronize()
    bounds = _split(len(pts), 2)
    if empty:
        bounds.insert(1, (bounds[0][1], bounds[0][1]))
    size = len(bounds)
    shared = ThreadComm.Shared(size)
    results, errors = [None] * size, []

    def run(rank):
        try:
            torch.cuda.set_device(0)
            c = capi.Context(mol.atm, mol.bas, mol.env)
            lo, hi = bounds[rank]
            results[rank] = select_fit_sharded(CudaBackend(c), ThreadComm(rank, size, shared),
                                               x[lo:hi].contiguous(), wt[lo:hi].contiguous(), lo, len(pts),
                                               precision="fp64", algorithm=algorithm, **PQ_KW)
            torch.cuda.synchronize()
        except Exception as e:  # surfaced below
            errors.append(e)
            shared.barrier.abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for r in results:
        np.testing.assert_array_equal(r.anchors, piv)
    th_sharded = torch.cat([r.theta for r in results if r.theta.shape[1]], dim=1).cpu().numpy()
    k, n = len(piv), finfo.n_kept
    th_ref = theta[:k * n].view(k, n).cpu().numpy()
    rel = np.abs(th_sharded - th_ref).max() / np.abs(th_ref).max()
    assert rel <= 1e-12 * max(1.0, finfo.condition) ** 2, rel
    assert abs(results[0].pair_relative - finfo.pair_relative) <= 1e-10 * finfo.pair_relative


@pytest.mark.gpu
def test_verified_sketch_qr_every_column_a_candidate():
    """Error bounds inflated to 1e30 make every column of the mixed sketch a
    re-verification candidate at the first step (one block per column, several
    columns per block, a candidate scan that reads every block) and exact from
    then on (the scan takes every block's key from the update).  The pivots
    equal those of the sketch's own bounds: a pivot is always an exact column."""
    import torch
    from mp_isdf_b200 import capi
    mol, pts, w = _system()
    ctx = capi.Context(mol.atm, mol.bas, mol.env)
    x = torch.tensor(pts, device="cuda")
    wt = torch.tensor(w, device="cuda")
    shard, n_kept, ell, sumsq = ctx.sketch_shard_project(x, wt, len(pts), precision="mixed", **KW)
    yt, delta, _, kxyz, kw_, scales = ctx.sketch_shard_combine(shard, sumsq, ell, n_kept, len(KW["axes"]))
    assert n_kept > 16 * 148
    piv, info = ctx.sketch_select_gathered(yt.clone(), kxyz, kw_, delta.clone(), scales, precision="mixed", **KW)
    big = torch.full_like(delta, 1e30)
    piv_all, info_all = ctx.sketch_select_gathered(yt.clone(), kxyz, kw_, big, scales, precision="mixed", **KW)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(piv_all, piv)
    assert info_all.verifications >= n_kept > info.verifications
    assert info_all.numerical_rank == info.numerical_rank
