"""Test-side pieces of the grid-sharded protocol (mp_isdf_b200.sharded): a
CPU backend built on the oracle (so that the protocol runs on gloo ranks
without a GPU) and a thread-based communicator (so that several shards can
run in one process on one GPU).  Test infrastructure only."""
import threading

import numpy as np
import torch

from oracle import oracle as O


class OracleBackend:
    """The sharded phases restated on the CPU with the oracle (FP64)."""

    def __init__(self, mol):
        self.oc = O.OracleContext(mol.atm, mol.bas, mol.env)
        self.nao = mol.nao

    @staticmethod
    def tensor(a):
        return torch.as_tensor(a)

    @staticmethod
    def to_numpy(t):
        return t.detach().cpu().numpy()

    def project(self, xyz, w, ng_total, axes=("ao",), axis_weights=None, max_rank=0, oversampling=16,
                seed=7, **_):
        xyz, w = self.to_numpy(xyz), self.to_numpy(w)
        keep = np.flatnonzero(w != 0)
        codes = [O.AXIS_CODES[a] for a in axes]
        f = self.oc.axis_features(xyz[keep], codes, None)
        sumsq = np.zeros(4)
        for a, c in enumerate(codes):
            sumsq[c] = np.sum(f[:, a * self.nao:(a + 1) * self.nao] ** 2)
        shard = dict(xyz=xyz, w=w, keep=keep, codes=codes, seed=seed, aw=axis_weights)
        return shard, len(keep), max_rank + oversampling, sumsq

    def combine(self, shard, sumsq, ell, n_kept, naxes):
        codes, keep = shard["codes"], shard["keep"]
        factors = np.ones(naxes) if not shard["aw"] else np.asarray(shard["aw"], float)
        scales = factors / np.sqrt(sumsq[codes]) if naxes > 1 else np.ones(1)
        u, v = O.sketch_factors(naxes * self.nao, ell, shard["seed"])
        y = self.oc.sketch(shard["xyz"][keep], shard["w"][keep], codes, scales if naxes > 1 else None, u, v, ell)
        return (torch.as_tensor(np.ascontiguousarray(y.T)), torch.zeros(len(keep), dtype=torch.float64),
                torch.as_tensor(keep.astype(np.int64)), torch.as_tensor(shard["xyz"][keep]),
                torch.as_tensor(shard["w"][keep]), scales)

    def select_gathered(self, yt, kxyz, kw, delta, scales, axes=("ao",), max_rank=0, oversampling=16,
                        tolerance=1e-10, **_):
        d = len(axes) * self.nao
        y = self.to_numpy(yt).T
        pos, _ = O.sketch_qr_rank(y, y.shape[1], oversampling, tolerance, max_rank, d * (d + 1) // 2)
        return pos, None

    def fit_at(self, xyz, w, a_xyz, a_w, precision, want_error):
        xyz, w = self.to_numpy(xyz), self.to_numpy(w)
        keep = w != 0
        theta, err = O.gram_fit(self.oc, xyz[keep], w[keep], a_xyz, a_w)
        return torch.as_tensor(theta), None, np.array([err["err2"], err["exact2"]])


class ThreadComm:
    """Collectives among threads of one process (one thread per shard)."""

    class Shared:
        def __init__(self, size):
            self.barrier = threading.Barrier(size, timeout=120)
            self.slots = [None] * size

    def __init__(self, rank, size, shared):
        self.rank, self.size, self.shared = rank, size, shared

    def allgather(self, t):
        self.shared.slots[self.rank] = t
        self.shared.barrier.wait()
        out = list(self.shared.slots)
        self.shared.barrier.wait()
        return out

    def allreduce_sum(self, t):
        parts = self.allgather(t.clone())
        total = parts[0].clone()
        for p in parts[1:]:
            total += p.to(total.device)
        return total
