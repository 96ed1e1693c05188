"""Test-side pieces of the grid-sharded protocol (mp_isdf_b200.sharded): a
CPU backend built on the oracle (so that the protocol runs on gloo ranks
without a GPU) and a thread-based communicator (so that several shards can
run in one process on one GPU).  Test infrastructure only."""
import threading
from types import SimpleNamespace

import numpy as np
import torch

from oracle import oracle as O


class _State(dict):
    """A dict whose entries also read as attributes (state.ell, state.verified)."""
    __getattr__ = dict.__getitem__


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
        xyz, w = self.to_numpy(xyz).reshape(-1, 3), self.to_numpy(w)
        keep = np.flatnonzero(w != 0)
        codes = [O.AXIS_CODES[a] for a in axes]
        f = self.oc.axis_features(xyz[keep], codes, None) if len(keep) else np.zeros((0, len(codes) * self.nao))
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
        y = (self.oc.sketch(shard["xyz"][keep], shard["w"][keep], codes, scales if naxes > 1 else None, u, v, ell)
             if len(keep) else np.zeros((0, ell)))
        return (torch.as_tensor(np.ascontiguousarray(y.T)), torch.zeros(len(keep), dtype=torch.float64),
                torch.as_tensor(keep.astype(np.int64)), torch.as_tensor(shard["xyz"][keep]),
                torch.as_tensor(shard["w"][keep]), scales)

    def select_gathered(self, yt, kxyz, kw, delta, scales, axes=("ao",), max_rank=0, oversampling=16,
                        tolerance=1e-10, **_):
        d = len(axes) * self.nao
        y = self.to_numpy(yt).T
        pos, _ = O.sketch_qr_rank(y, y.shape[1], oversampling, tolerance, max_rank, d * (d + 1) // 2)
        return pos, None

    # the distributed QR of the sketch columns of this rank, restated in NumPy
    # with the arithmetic of the library's per-rank steps (exact trailing
    # norms, dgeqp3's pivot order through global positions)
    def qr_begin(self, yt, n_total, pos_offset, kxyz, kw, delta, scales, **_):
        a = self.to_numpy(yt).copy()
        n = a.shape[1] if a.ndim == 2 else 0
        ell = a.shape[0]
        return _State(A=a.reshape(ell, n), ell=ell, pos=pos_offset + np.arange(n), sel=np.zeros(n, bool),
                      v=np.zeros((ell, ell)), tau=np.zeros(ell), verified=False)

    @staticmethod
    def qr_update(st, j):
        A, act = st["A"], ~st["sel"]
        ell = st["ell"]
        e = 0.0
        if j > 0 and st["tau"][j - 1] != 0.0 and act.any():
            v = st["v"][j - 1][j - 1:]
            sub = A[j - 1:, act]
            A[j - 1:, act] = sub - np.outer(v, st["tau"][j - 1] * (v @ sub))
        if j > 0:
            e = float(np.sum(A[j - 1, act] ** 2))
        if j < ell and act.any():
            cols = np.flatnonzero(act)
            nrm = np.sum(A[j:, cols] ** 2, axis=0)
            top = nrm.max()
            tied = cols[nrm == top]
            c = int(tied[np.argmin(st["pos"][tied])])
            return float(top), int(st["pos"][c]), c, e, 0.0
        return -1.0, 2 ** 62, -1, e, 0.0

    @staticmethod
    def qr_column(st, col):
        return st["A"][:, col].copy()

    @staticmethod
    def qr_pivot(st, j, rows, pivot_col, pivot_pos, moved_col):
        if pivot_col >= 0:
            st["sel"][pivot_col] = True
            st["pos"][pivot_col] = j
        if moved_col >= 0:
            st["pos"][moved_col] = pivot_pos
        alpha = rows[j]
        xnorm = 0.0
        for x in rows[j + 1:]:
            xnorm = float(np.hypot(xnorm, x))
        if xnorm == 0.0:
            beta, tau, scale = alpha, 0.0, 0.0
        else:
            beta = -np.copysign(np.hypot(alpha, xnorm), alpha)
            tau = (beta - alpha) / beta
            scale = 1.0 / (alpha - beta)
        v = np.zeros(st["ell"])
        v[j] = 1.0
        v[j + 1:] = rows[j + 1:] * scale
        st["v"][j], st["tau"][j] = v, tau
        return float(beta)

    @staticmethod
    def qr_reverified(st):
        return 0

    @staticmethod
    def qr_end(st):
        pass

    def sketch_rank(self, n_total, diag, energy, axes=("ao",), max_rank=0, oversampling=16, sketch_size=128,
                    tolerance=1e-10, **_):
        d = len(axes) * self.nao
        ell = max_rank + oversampling if max_rank else sketch_size
        rank, tails, nrank = O.sketch_rank_rules(diag, energy, ell, n_total, oversampling, tolerance, max_rank,
                                                 d * (d + 1) // 2)
        return rank, nrank, float(tails[rank] / tails[0]) if tails[0] else 0.0

    # ---- the sharded pair-space QR, restated with exact residuals (the
    # arithmetic of oracle.pair_qrcp_exact: basis as symmetric d x d matrices)
    def pq_begin(self, xyz, w, grid_offset, axes=("ao",), axis_weights=None, algorithm="qrcp_dense", **_):
        xyz, w = self.to_numpy(xyz).reshape(-1, 3), self.to_numpy(w)
        keep = np.flatnonzero(w != 0)
        codes = [O.AXIS_CODES[a] for a in axes]
        nao = self.nao
        F = self.oc.axis_features(xyz[keep], codes) if len(keep) else np.zeros((0, len(codes) * nao))
        sumsq = np.zeros(5)
        for i in range(len(codes)):
            sumsq[i] = np.sum(F[:, i * nao:(i + 1) * nao] ** 2)
        return SimpleNamespace(n_kept=len(keep), d=F.shape[1], sumsq=sumsq, F=F, sw=np.sqrt(np.abs(w[keep])),
                               keep=keep, xyz=xyz, w=w, grid_offset=grid_offset, codes=codes,
                               aw=axis_weights, basis=[], coef=[], est={}, last=None)

    def pq_init(self, st, sums, pos_offset):
        ne = len(st.codes)
        st.colscale = np.ones(st.d)
        if ne > 1:   # every rank derives the same scales from the same global sums
            factors = np.ones(ne) if not st.aw else np.asarray(st.aw, float)
            st.colscale = np.repeat(factors / np.sqrt(sums[:ne]), self.nao)
        st.Fs = st.F * st.colscale[None, :]
        st.pos = pos_offset + np.arange(st.n_kept)
        st.pos_offset = pos_offset
        st.selected = np.zeros(st.n_kept, bool)
        st.norm2 = (st.sw * np.einsum("gi,gi->g", st.Fs, st.Fs)) ** 2
        return np.array([st.norm2.sum(), 0.0 if np.all(np.isfinite(st.norm2)) else 1.0])

    @staticmethod
    def pq_argmax(st):
        if st.n_kept == 0 or st.selected.all():
            return np.array([-1.0, -1.0, -1.0])
        res = st.norm2 - sum((c ** 2 for c in st.coef), np.zeros(st.n_kept))
        for g, v in st.est.items():
            res[g] = v
        res[st.selected] = -np.inf
        best = max(np.flatnonzero(~st.selected), key=lambda g: (res[g], -st.pos[g]))
        return np.array([res[best], st.pos[best], st.pos_offset + best])

    @staticmethod
    def pq_row(st, col):
        g = col - st.pos_offset
        gi = st.keep[g]
        return np.concatenate([st.F[g], [st.sw[g], st.grid_offset + gi], st.xyz[gi], [st.w[gi]]])

    def pq_verify(self, st, row, j, col):
        d = st.d
        f = row[:d] * st.colscale
        v = row[d] * np.outer(f, f)
        t0 = [np.sum(Q * v) for Q in st.basis]
        for t, Q in zip(t0, st.basis):
            v = v - t * Q
        for Q in st.basis:                      # second Gram-Schmidt pass
            v = v - np.sum(Q * v) * Q
        exact2 = float(np.sum(v * v))
        st.last = (col, v)
        g = col - st.pos_offset
        if 0 <= g < st.n_kept:
            st.est[g] = exact2
        return exact2

    def pq_accept(self, st, row, j, col, exact2, winner_pos, dense):
        v = st.last[1] / np.sqrt(exact2)
        v = 0.5 * (v + v.T)
        st.basis.append(v)
        st.coef.append(st.sw * np.einsum("gi,gi->g", st.Fs @ v, st.Fs) if st.n_kept else np.zeros(0))
        st.est = {}
        g = col - st.pos_offset
        if dense and st.n_kept:
            at_j = np.flatnonzero(st.pos == j)
            if len(at_j):
                st.pos[at_j] = winner_pos
        if 0 <= g < st.n_kept:
            st.selected[g] = True
            if dense:
                st.pos[g] = j

    @staticmethod
    def pq_scan(st, j, thr2):
        return 0

    @staticmethod
    def pq_end(st):
        pass

    def adjoint_partial(self, xyz, w, a_xyz, a_w, dm, want_grad):
        return oracle_adjoint_partial(self.oc, self.to_numpy(xyz).reshape(-1, 3), self.to_numpy(w),
                                      np.asarray(a_xyz).reshape(-1, 3), np.asarray(dm), want_grad)

    def adjoint_finish(self, a_xyz, a_w, dm, sums, want_grad):
        return oracle_adjoint_finish(self.oc, np.asarray(a_xyz).reshape(-1, 3), np.asarray(dm), np.asarray(sums),
                                     want_grad)

    def fit_at(self, xyz, w, a_xyz, a_w, precision, want_error):
        xyz, w = self.to_numpy(xyz).reshape(-1, 3), self.to_numpy(w)
        keep = w != 0
        if not keep.any():
            return torch.zeros((len(a_w), 0), dtype=torch.float64), None, np.zeros(2)
        theta, err = O.gram_fit(self.oc, xyz[keep], w[keep], a_xyz, a_w)
        return torch.as_tensor(theta), None, np.array([err["err2"], err["exact2"]])


def _anchor_side(oc, a_xyz, dm):
    phi_a = oc.eval_ao(a_xyz)
    S = phi_a @ phi_a.T
    M = S * S
    rho_a = np.einsum("ki,ij,kj->k", phi_a, dm, phi_a)
    return phi_a, S, M, np.linalg.solve(M, rho_a)


def oracle_adjoint_partial(oc, xyz, w, a_xyz, dm, want_grad):
    """One shard's sums of the oracle adjoint (oracle.isdf_energy_gradient split
    at its grid loop): [E, v, per-atom grid terms, alpha^T Phi_g, zeros(3 nao)]."""
    keep = w != 0
    xyz, w = xyz[keep], w[keep]
    phi_a, S, M, z = _anchor_side(oc, a_xyz, dm)
    k, nao = phi_a.shape
    E, v, gacc, B = 0.0, np.zeros(k), np.zeros((oc.natm, 3)), np.zeros((k, nao))
    if len(w):
        phi = oc.eval_ao(xyz)
        G = phi @ phi_a.T
        h = G * G
        rho = h @ z
        E = float(np.sum(w * rho * rho))
        u = 2 * w * rho
        v = u @ h
        if want_grad:
            dphi = oc.eval_ao_gradient(xyz)
            alpha = 2 * u[:, None] * z[None, :] * G
            B = alpha.T @ phi
            contrib = np.einsum("gm,cgm->cm", alpha @ phi_a, dphi)
            for c in range(3):
                np.add.at(gacc[:, c], oc.ao_atom, contrib[c])
    return np.concatenate([[E], v, gacc.ravel(), B.ravel(), np.zeros(3 * nao)])


def oracle_adjoint_finish(oc, a_xyz, dm, sums, want_grad):
    phi_a, S, M, z = _anchor_side(oc, a_xyz, dm)
    k, nao = phi_a.shape
    grad = np.zeros((oc.natm, 3))
    if not want_grad:
        return float(sums[0]), grad
    v = sums[1:1 + k]
    gacc = sums[1 + k:1 + k + 3 * oc.natm].reshape(oc.natm, 3)
    B = sums[1 + k + 3 * oc.natm:1 + k + 3 * oc.natm + k * nao].reshape(k, nao)
    y = np.linalg.solve(M, v)
    coef = B + 2 * y[:, None] * (phi_a @ dm)
    W = 2 * S * (y[:, None] * z[None, :])
    coef -= (W + W.T) @ phi_a
    contrib = np.einsum("km,ckm->cm", coef, oc.eval_ao_gradient(a_xyz))
    for c in range(3):
        np.add.at(grad[:, c], oc.ao_atom, -contrib[c])
    return float(sums[0]), grad - gacc


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
