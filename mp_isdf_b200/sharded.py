"""Grid-sharded anchor selection + fit: one rank per GPU, one cluster.

The distributed form of ``AnchorSelection.select`` (RandomizedQuadratureKhatriRao,
``cpp/src/anchor_select_randomized_id.cpp:92-374``) followed by the fit
(``python/isdf.py:238-263``); the reference's ``DistributedAnchorSelection`` is
a stub that throws (``cpp/src/anchor_select.cpp:175-181``).  Every rank holds a
contiguous shard of the grid, in grid order, and runs::

    1. project its shard                  -> per-component sums of squares
       all-reduce(sum) of 4 doubles       -> global multi-axis scales
    2. its shard's sketch columns          (ell x n_r, + error bounds)
    3. the pivoted QR of the whole sketch with the columns left where they
       are (``distributed_sketch_qr``).  Per pivot step j:
         - every rank applies reflector j-1 to its columns and forms its best
           key (squared trailing norm, global position); in the mixed form its
           best lower bound first, all-reduce(max), then the exact
           re-verification of its candidates;
         - all-gather of one key per rank (4 doubles): the global winner
           (ties to the smaller position, dgeqp3's order) and row j-1's energy;
         - the winner's ell rows and its grid index, coordinates and weight
           from its owner (all-reduce(sum) of a vector that is zero elsewhere);
         - every rank builds reflector j from those rows and moves the column
           at position j to the winner's position (dgeqp3's swap);
       then the tail / numerical-rank rules on the per-step |R_jj| and
       energies (identical on every rank, hence identical anchors: those of
       the single-GPU QR of the whole grid);
    4. the fit on its shard with the anchors' coordinates
       all-reduce(sum) of the pair-error sums

qrcp_dense and qrcp_online go through ``select_pair_qr_sharded``: the ranks keep
their points' features and residual estimates, the pair basis is replicated,
and per pivot one key per rank is all-gathered and the leader's row
all-reduced; every rank verifies it exactly with the same result.

``energy_gradient_sharded`` runs the nuclear-gradient adjoint the same way:
per-rank partial sums, one all-reduce(sum), the anchor-side algebra on every
rank.

The AO evaluation, the projections and the QR updates are split over the
ranks; per pivot step the ranks exchange O(ell + ranks) doubles, so the
exchange is latency-bound (2-3 small collectives per step, ell steps).
``qr="gathered"`` keeps the earlier form: all-gather of the whole sketch and
the same QR replicated on every rank.  Collectives go through
``torch.distributed`` (NCCL for CUDA tensors; gloo works for CPU tensors), or
``LocalComm`` for one process.  The compute backend is pluggable;
``CudaBackend`` drives the library's C-ABI phases.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from types import SimpleNamespace

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


def _allreduce_max(comm, backend, value):
    return max(float(backend.to_numpy(t)[0]) for t in comm.allgather(backend.tensor(np.array([value], np.float64))))


def distributed_sketch_qr(backend, comm, qr, steps, verified, offsets, counts, record):
    """Column-pivoted QR of a sketch whose columns stay on their ranks.

    ``qr``: this rank's QR state (``backend.qr_begin``); ``offsets``/``counts``:
    every rank's first global position and column count; ``record(col)``:
    this rank's (grid index, x, y, z, weight) of a local column.  Returns the
    per-step pivots as (grid index, xyz, weight) records, |R_jj| and the row
    energies of R, identical on every rank.
    """
    moved = {}   # global position -> (rank, local column), for positions a swap changed

    def holder(pos):
        if pos in moved:
            return moved[pos]
        for r in range(len(offsets)):
            if offsets[r] <= pos < offsets[r] + counts[r]:
                return r, pos - offsets[r]
        raise RuntimeError("position outside the sketch")

    diag, energy, pivots = [], np.zeros(steps), []
    ell = qr.ell
    for j in range(steps + 1):
        val, pos, col, e_part, lb = backend.qr_update(qr, j)
        if j == steps:
            tot = backend.to_numpy(comm.allreduce_sum(backend.tensor(np.array([e_part], np.float64))))
            if j > 0:
                energy[j - 1] += float(tot[0])
            break
        if verified:
            val, pos, col = backend.qr_verify(qr, j, _allreduce_max(comm, backend, lb))
        keys = [backend.to_numpy(k) for k in
                comm.allgather(backend.tensor(np.array([val, pos, col, e_part], np.float64)))]
        if j > 0:
            energy[j - 1] += float(sum(k[3] for k in keys))
        best = None
        for r, k in enumerate(keys):
            if k[0] < 0:
                continue
            if best is None or k[0] > keys[best][0] or (k[0] == keys[best][0] and k[1] < keys[best][1]):
                best = r
        if best is None:
            raise RuntimeError("no column left for the pivoted QR")
        p, lc = int(keys[best][1]), int(keys[best][2])
        buf = np.zeros(ell + 5)
        if comm.rank == best:
            buf[:ell] = backend.qr_column(qr, lc)
            buf[ell:] = record(lc)
        buf = backend.to_numpy(comm.allreduce_sum(backend.tensor(buf)))
        hr, hc = holder(j)
        moved[p] = (hr, hc)
        moved[j] = (best, lc)
        r_jj = backend.qr_pivot(qr, j, buf[:ell], lc if comm.rank == best else -1, p,
                                hc if comm.rank == hr else -1)
        diag.append(abs(r_jj))
        energy[j] += r_jj * r_jj
        pivots.append(buf[ell:].copy())
    return pivots, np.array(diag), energy


_EPS = np.finfo(np.float64).eps


def _better(a, b):
    """Key order of the pivot choice: larger value, then smaller position."""
    if b is None or b[2] < 0:
        return a[2] >= 0
    if a[2] < 0:
        return False
    return a[0] > b[0] or (a[0] == b[0] and a[1] < b[1])


def select_pair_qr_sharded(backend, comm, xyz, w, grid_offset, algorithm="qrcp_dense", tolerance=1e-10,
                           max_rank=0, **kw):
    """The pair-space QR of qrcp_dense / qrcp_online over grid shards
    (``cpp/src/anchor_select_qrcp.cpp:95-225``, ``anchor_select_online_qr.cpp:176-375``;
    the single-GPU form is ``select_pairqr.cu``).  Every rank holds its kept
    points' features and residual estimates; the explicit pair basis is
    replicated.  Per pivot: all-gather of one key per rank (estimate, position,
    global kept index), the owner's row of the leader (d + 6 doubles) by
    all-reduce(sum), its exact residual on every rank (the same value
    everywhere) and, while the leader changes, again; the same stop rules and
    stop-confirming scan as the single-GPU selection.  Returns (anchor grid
    indices, anchor coordinates [k, 3], anchor weights [k], kept count)."""
    online = algorithm in ("qrcp_online", 1)
    dense = not online
    sel = dict(kw, algorithm=algorithm, tolerance=tolerance, max_rank=max_rank)
    st = backend.pq_begin(xyz, w, grid_offset, **sel)
    counts = [int(backend.to_numpy(c)[0]) for c in comm.allgather(backend.tensor(np.array([st.n_kept], np.int64)))]
    n_total = int(sum(counts))
    pos_offset = int(sum(counts[:comm.rank]))
    sums = backend.to_numpy(comm.allreduce_sum(backend.tensor(np.asarray(st.sumsq, np.float64))))
    kd = backend.to_numpy(comm.allreduce_sum(backend.tensor(backend.pq_init(st, sums, pos_offset))))
    if kd[1] != 0 or not np.isfinite(kd[0]):
        raise OverflowError("non-finite online AO pair column" if online else "non-finite weighted pair product")
    frob2 = float(kd[0])
    d = st.d
    m = d * d
    cap = min(m, n_total, max_rank if max_rank else min(m, n_total))
    floor = 32 * _EPS * np.sqrt(frob2) if online else 0.0
    rows_width = d + 6
    starts = [int(sum(counts[:r])) for r in range(len(counts))]

    def global_argmax():
        keys = [backend.to_numpy(k) for k in comm.allgather(backend.tensor(np.asarray(backend.pq_argmax(st),
                                                                                      np.float64)))]
        best = None
        for k in keys:
            if _better(k, best):
                best = k
        return best if best is not None and best[2] >= 0 else None

    def fetch_row(key):
        col = int(key[2])
        own = starts[comm.rank] <= col < starts[comm.rank] + counts[comm.rank]
        row = backend.pq_row(st, col) if own else np.zeros(rows_width)
        return backend.to_numpy(comm.allreduce_sum(backend.tensor(np.asarray(row, np.float64))))

    result, first, exact_mode = [], -1.0, False
    while True:
        j = len(result)
        if j == cap:
            break
        k = global_argmax()
        if k is None:
            break
        # verification loop: the leader's exact residual, then the argmax again
        while True:
            row = fetch_row(k)
            exact2 = backend.pq_verify(st, row, j, int(k[2]))
            k2 = global_argmax()
            if k2 is not None and int(k2[2]) == int(k[2]):
                break
            if k2 is None:
                break
            k = k2
        rjj = float(np.sqrt(exact2))
        if first < 0:
            first = rjj
        thr = max(tolerance * first, floor)
        stop = first == 0 or rjj <= thr or (online and rjj <= floor)
        if stop:
            if exact_mode:
                break
            # confirm on exact values: every rank rescans its uncertain columns
            backend.pq_scan(st, j, thr * thr)
            exact_mode = True
            k = global_argmax()
            if k is None:
                break
            row = fetch_row(k)
            exact2 = backend.pq_verify(st, row, j, int(k[2]))
            if first == 0 or np.sqrt(exact2) <= thr:
                break
        backend.pq_accept(st, row, j, int(k[2]), exact2, int(k[1]), dense)
        exact_mode = False
        result.append(row[d + 1:d + 6].copy())
    backend.pq_end(st)
    rec = np.array(result).reshape(-1, 5)
    return rec[:, 0].round().astype(np.int64), rec[:, 1:4], rec[:, 4], n_total


def select_fit_sharded(backend, comm, xyz, w, grid_offset, ng_total, want_error=True, qr="distributed",
                       **select_kw):
    """Selection + fit of one cluster whose grid is split over the ranks.

    ``xyz``/``w``: this rank's contiguous shard (device tensors for the CUDA
    backend), starting at global grid index ``grid_offset``; ``ng_total``: the
    whole grid's size.  ``select_kw``: the arguments of ``Context.select``
    (rand_sketch, qrcp_dense or qrcp_online).  Returns a ``ShardedResult`` with
    global anchor indices (identical on every rank) and this rank's Theta
    columns.
    """
    import torch
    precision = select_kw.get("precision", "fp64")
    naxes = len(select_kw.get("axes", ("ao",)))
    if select_kw.get("algorithm", "rand_sketch") in ("qrcp_dense", "qrcp_online", 0, 1):
        # pair-space QR over the shards, then the fit on each shard
        sel = {kk: v for kk, v in select_kw.items() if kk != "precision"}
        anchors, a_xyz, a_w, n_total = select_pair_qr_sharded(backend, comm, xyz, w, grid_offset, **sel)
        theta, finfo, fsums = backend.fit_at(xyz, w, a_xyz, a_w, precision, want_error)
        tot = backend.to_numpy(comm.allreduce_sum(backend.tensor(np.asarray(fsums, np.float64))))
        err2, exact2 = max(float(tot[0]), 0.0), float(tot[1])
        counts = [int(backend.to_numpy(c)[0]) for c in
                  comm.allgather(backend.tensor(np.array([theta.shape[1]], np.int64)))]
        sinfo = SimpleNamespace(n_kept=n_total, sketch_rows=0, numerical_rank=0, relative_residual=0.0,
                                verifications=0, reselections=0, precision_used=0)
        return ShardedResult(anchors=anchors, theta=theta, n_kept_local=int(theta.shape[1]),
                             kept_offset=int(sum(counts[:comm.rank])), pair_l2=float(np.sqrt(err2)),
                             pair_relative=float(np.sqrt(err2 / exact2)) if exact2 else 0.0,
                             select_info=sinfo, fit_info=finfo, counts=counts)
    # 1. projection of the shard and the global per-component sums of squares
    shard, n_kept, ell, sumsq = backend.project(xyz, w, ng_total, **select_kw)
    sums = comm.allreduce_sum(backend.tensor(np.asarray(sumsq, np.float64)))
    # 2. this shard's sketch columns with the global scales
    yt, delta, kept, kxyz, kw, scales = backend.combine(shard, backend.to_numpy(sums), ell, n_kept, naxes)
    counts = [int(backend.to_numpy(c)[0]) for c in comm.allgather(backend.tensor(np.array([n_kept], np.int64)))]
    offsets = [int(backend.to_numpy(o)[0])
               for o in comm.allgather(backend.tensor(np.array([grid_offset], np.int64)))]
    if qr == "distributed":
        # 3. the pivoted QR with the columns left on their ranks
        n_total = int(sum(counts))
        pos_offset = int(sum(counts[:comm.rank]))
        state = backend.qr_begin(yt, n_total, pos_offset, kxyz, kw, delta, scales, **select_kw)
        kept_np = backend.to_numpy(kept) if n_kept else np.zeros(0, np.int64)
        kxyz_np = backend.to_numpy(kxyz) if n_kept else np.zeros((0, 3))
        kw_np = backend.to_numpy(kw) if n_kept else np.zeros(0)

        def record(col):
            return np.array([kept_np[col] + grid_offset, *kxyz_np[col], kw_np[col]], np.float64)

        steps = min(state.ell, n_total)
        pivots, diag, energy = distributed_sketch_qr(backend, comm, state, steps, state.verified,
                                                     [int(sum(counts[:r])) for r in range(len(counts))],
                                                     counts, record)
        rank_k, numerical_rank, rel_tail = backend.sketch_rank(n_total, diag, energy, **select_kw)
        sinfo = SimpleNamespace(n_kept=n_total, sketch_rows=state.ell, numerical_rank=numerical_rank,
                                relative_residual=rel_tail, verifications=backend.qr_reverified(state),
                                reselections=0, precision_used=int(state.verified))
        backend.qr_end(state)
        chosen = pivots[:rank_k]
        anchors = np.array([int(round(r[0])) for r in chosen], np.int64)
        a_xyz = np.array([r[1:4] for r in chosen], np.float64).reshape(-1, 3)
        a_w = np.array([r[4] for r in chosen], np.float64)
        theta, finfo, fsums = backend.fit_at(xyz, w, a_xyz, a_w, precision, want_error)
        tot = backend.to_numpy(comm.allreduce_sum(backend.tensor(np.asarray(fsums, np.float64))))
        err2, exact2 = max(float(tot[0]), 0.0), float(tot[1])
        shard_free = getattr(shard, "free", None)
        if shard_free:
            shard_free()
        return ShardedResult(anchors=anchors, theta=theta, n_kept_local=n_kept, kept_offset=pos_offset,
                             pair_l2=float(np.sqrt(err2)),
                             pair_relative=float(np.sqrt(err2 / exact2)) if exact2 else 0.0,
                             select_info=sinfo, fit_info=finfo, counts=counts)
    # 3. (gathered form) everything the pivoted QR needs, in grid order
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


def energy_gradient_sharded(backend, comm, xyz, w, anchor_xyz, anchor_w, dm, want_grad=True):
    """The adjoint (E = sum_g w_g rho_ISDF(g)^2 and dE/dR) over grid shards:
    every rank sums over its own points (``backend.adjoint_partial``: E, v,
    the per-atom grid terms and the anchor-coefficient sums), one
    all-reduce(sum) adds the partials, and every rank finishes the same
    anchor-side algebra (``backend.adjoint_finish``).  Anchors are given by
    coordinates (k x 3) and weights, as from select_fit_sharded.  Returns
    (E, dE/dR[natm, 3]), the same on every rank."""
    part = backend.adjoint_partial(xyz, w, anchor_xyz, anchor_w, dm, want_grad)
    tot = backend.to_numpy(comm.allreduce_sum(backend.tensor(np.asarray(part, np.float64))))
    return backend.adjoint_finish(anchor_xyz, anchor_w, dm, tot, want_grad)


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

    # distributed QR (isdf_qr_shard_*)
    def qr_begin(self, yt, n_total, pos_offset, kxyz, kw, delta, scales, **kw_sel):
        return self.ctx.qr_shard(yt.contiguous(), n_total, pos_offset, kxyz, kw, delta, scales, **kw_sel)

    @staticmethod
    def qr_update(qr, j):
        return qr.update(j)

    @staticmethod
    def qr_verify(qr, j, bound):
        return qr.verify(j, bound)

    @staticmethod
    def qr_column(qr, col):
        return qr.column(col)

    @staticmethod
    def qr_pivot(qr, j, rows, pivot_col, pivot_pos, moved_col):
        return qr.pivot(j, rows, pivot_col, pivot_pos, moved_col)

    @staticmethod
    def qr_reverified(qr):
        return qr.reverified()

    @staticmethod
    def qr_end(qr):
        qr.free()

    def sketch_rank(self, n_total, diag, energy, **kw_sel):
        return self.ctx.sketch_rank(n_total, diag, energy, **kw_sel)

    def adjoint_partial(self, xyz, w, a_xyz, a_w, dm, want_grad):
        return self.ctx.energy_gradient_shard(xyz, w, a_xyz, a_w, dm, want_grad)

    # the sharded pair-space QR (isdf_pairqr_shard_*)
    def pq_begin(self, xyz, w, grid_offset, **kw_sel):
        return self.ctx.pairqr_shard(xyz, w, grid_offset, **kw_sel)

    @staticmethod
    def pq_init(st, sums, pos_offset):
        return st.init(sums, pos_offset)

    @staticmethod
    def pq_argmax(st):
        return st.argmax()

    @staticmethod
    def pq_row(st, col):
        return st.row(col)

    @staticmethod
    def pq_verify(st, row, j, col):
        return st.verify(row, j, col)

    @staticmethod
    def pq_accept(st, row, j, col, exact2, winner_pos, dense):
        st.accept(row, j, col, exact2, winner_pos, dense)

    @staticmethod
    def pq_scan(st, j, thr2):
        return st.scan(j, thr2)

    @staticmethod
    def pq_end(st):
        st.free()

    def adjoint_finish(self, a_xyz, a_w, dm, sums, want_grad):
        return self.ctx.energy_gradient_finish(a_xyz, a_w, dm, sums, want_grad)

    def fit_at(self, xyz, w, a_xyz, a_w, precision, want_error):
        import torch
        n = xyz.shape[0]
        theta = torch.empty(max(1, len(a_w) * n), dtype=torch.float64, device=self.device)
        info, sums = self.ctx.fit_at(xyz, w, a_xyz, a_w, theta, precision, want_error)
        k = len(a_w)
        return theta[:k * info.n_kept].view(k, info.n_kept), info, sums
