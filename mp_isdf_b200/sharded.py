"""Grid-sharded anchor selection + fit: one rank per GPU, one cluster.

The distributed form of ``AnchorSelection.select`` (RandomizedQuadratureKhatriRao,
``cpp/src/anchor_select_randomized_id.cpp:92-374``) followed by the fit
(``python/isdf.py:238-263``); the reference's ``DistributedAnchorSelection`` is
a stub that throws (``cpp/src/anchor_select.cpp:175-181``).  Every rank holds a
contiguous shard of the grid, in grid order, and runs::

    1. project its shard                  -> per-component sums of squares
       all-reduce(sum) of 4 doubles       -> global multi-axis scales
    2. its shard's sketch columns          (ell x n_r, + error bounds)
       all-gather of the columns, bounds, kept coordinates and weights
    3. the pivoted QR of the gathered sketch (identical inputs on every rank,
       hence identical anchors; this is the single-GPU QR of the whole grid)
    4. the fit on its shard with the anchors' coordinates
       all-reduce(sum) of the pair-error sums

The AO evaluation and projections (the dominant cost) are split over the
ranks; the exchanged data is O(ell * n) doubles, which NVLink moves in well
under a millisecond at (H2O)64.  Collectives go through ``torch.distributed``
(NCCL for CUDA tensors; gloo works for CPU tensors), or ``LocalComm`` for one
process.  The compute backend is pluggable; ``CudaBackend`` drives the
library's C-ABI phases.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


class LocalComm:
    """A single rank (no process group)."""

    rank, size = 0, 1

    def allreduce_sum(self, t):
        return t

    def allgather(self, t):
        return [t]


class TorchComm:
    """Collectives of a torch.distributed process group."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def allreduce_sum(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t

    def allgather(self, t):
        out = [t.new_empty(t.shape) for _ in range(self.size)]
        self.dist.all_gather(out, t.contiguous(), group=self.group)
        return out


def _gather_ragged(comm, t, n_local, counts):
    """Concatenate per-rank tensors along dim 0 (their first n_r rows)."""
    import torch
    nmax = max(counts)
    pad = t.new_zeros((nmax,) + tuple(t.shape[1:]))
    pad[:n_local] = t[:n_local]
    parts = comm.allgather(pad)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)


@dataclass
class ShardedResult:
    anchors: np.ndarray            # global grid indices, pivot order
    theta: object                  # this rank's Theta columns [k, n_kept_local]
    n_kept_local: int
    kept_offset: int               # first global kept-point column of this rank
    pair_l2: float
    pair_relative: float
    select_info: object = None
    fit_info: object = None
    counts: list = field(default_factory=list)


def select_fit_sharded(backend, comm, xyz, w, grid_offset, ng_total, want_error=True, **select_kw):
    """Selection + fit of one cluster whose grid is split over the ranks.

    ``xyz``/``w``: this rank's contiguous shard (device tensors for the CUDA
    backend), starting at global grid index ``grid_offset``; ``ng_total``: the
    whole grid's size.  ``select_kw``: the arguments of ``Context.select``
    (rand_sketch).  Returns a ``ShardedResult`` with global anchor indices
    (identical on every rank) and this rank's Theta columns.
    """
    import torch
    precision = select_kw.get("precision", "fp64")
    naxes = len(select_kw.get("axes", ("ao",)))
    # 1. projection of the shard and the global per-component sums of squares
    shard, n_kept, ell, sumsq = backend.project(xyz, w, ng_total, **select_kw)
    sums = comm.allreduce_sum(backend.tensor(np.asarray(sumsq, np.float64)))
    # 2. this shard's sketch columns with the global scales
    yt, delta, kept, kxyz, kw, scales = backend.combine(shard, backend.to_numpy(sums), ell, n_kept, naxes)
    # 3. gather everything the pivoted QR needs, in grid order
    counts = [int(backend.to_numpy(c)[0]) for c in comm.allgather(backend.tensor(np.array([n_kept], np.int64)))]
    offsets = [int(backend.to_numpy(o)[0])
               for o in comm.allgather(backend.tensor(np.array([grid_offset], np.int64)))]
    yt_all = _gather_ragged(comm, yt.t().contiguous(), n_kept, counts).t().contiguous()
    delta_all = _gather_ragged(comm, delta, n_kept, counts)
    kxyz_all = _gather_ragged(comm, kxyz, n_kept, counts)
    kw_all = _gather_ragged(comm, kw, n_kept, counts)
    kept_all = torch.cat([p[:c] + o for p, c, o in
                          zip(comm.allgather(_pad(kept, max(counts))), counts, offsets)])
    pos, sinfo = backend.select_gathered(yt_all, kxyz_all, kw_all, delta_all, scales, **select_kw)
    pos_t = torch.as_tensor(pos, dtype=torch.int64, device=yt_all.device)
    anchors = backend.to_numpy(kept_all[pos_t])
    a_xyz = backend.to_numpy(kxyz_all[pos_t])
    a_w = backend.to_numpy(kw_all[pos_t])
    # 4. the fit on this shard; the pair-error sums add up over ranks
    theta, finfo, fsums = backend.fit_at(xyz, w, a_xyz, a_w, precision, want_error)
    tot = backend.to_numpy(comm.allreduce_sum(backend.tensor(np.asarray(fsums, np.float64))))
    err2, exact2 = max(float(tot[0]), 0.0), float(tot[1])
    shard_free = getattr(shard, "free", None)
    if shard_free:
        shard_free()
    return ShardedResult(anchors=np.asarray(anchors, np.int64), theta=theta, n_kept_local=n_kept,
                         kept_offset=int(sum(counts[:comm.rank])),
                         pair_l2=float(np.sqrt(err2)),
                         pair_relative=float(np.sqrt(err2 / exact2)) if exact2 else 0.0,
                         select_info=sinfo, fit_info=finfo, counts=counts)


def _pad(t, n):
    out = t.new_zeros((n,) + tuple(t.shape[1:]))
    out[:t.shape[0]] = t
    return out


class CudaBackend:
    """The library's sharded phases on this rank's GPU (mp_isdf_b200.capi)."""

    def __init__(self, ctx):
        import torch
        self.ctx = ctx
        self.device = torch.device("cuda", torch.cuda.current_device())

    def tensor(self, a):
        import torch
        return torch.as_tensor(a, device=self.device)

    @staticmethod
    def to_numpy(t):
        return t.detach().cpu().numpy()

    def project(self, xyz, w, ng_total, **kw):
        return self.ctx.sketch_shard_project(xyz, w, ng_total, **kw)

    def combine(self, shard, sumsq, ell, n_kept, naxes):
        return self.ctx.sketch_shard_combine(shard, sumsq, ell, n_kept, naxes)

    def select_gathered(self, yt, kxyz, kw, delta, scales, **kw_sel):
        return self.ctx.sketch_select_gathered(yt, kxyz, kw, delta, scales, **kw_sel)

    def fit_at(self, xyz, w, a_xyz, a_w, precision, want_error):
        import torch
        n = xyz.shape[0]
        theta = torch.empty(max(1, len(a_w) * n), dtype=torch.float64, device=self.device)
        info, sums = self.ctx.fit_at(xyz, w, a_xyz, a_w, theta, precision, want_error)
        k = len(a_w)
        return theta[:k * info.n_kept].view(k, info.n_kept), info, sums
