"""ctypes binding of the C-ABI in ``include/isdf_b200.h`` (libisdf_b200.so).

Device-pointer entry points take torch CUDA tensors; the stream is torch's
current stream on the tensor's device.  Host-buffer entry points take numpy
arrays.  There is no CPU implementation behind any of these calls: without a
CUDA device they raise.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libisdf_b200.so"

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
F64 = ctypes.c_double

SYMBOLS = [
    "isdf_status_string", "isdf_last_error", "isdf_cuda_available",
    "isdf_ctx_create", "isdf_ctx_destroy", "isdf_ctx_info", "isdf_ctx_ao_atoms",
    "isdf_eval_ao", "isdf_eval_ao_host", "isdf_evaluate_axis", "isdf_evaluate_axis_host",
    "isdf_select_args_default", "isdf_select", "isdf_select_host",
    "isdf_fit", "isdf_fit_host", "isdf_pair_error", "isdf_pair_error_terms",
    "isdf_profile_enable", "isdf_profile_read", "isdf_project_axes",
    "isdf_energy_gradient", "isdf_ctx_set_coords", "isdf_pair_error_terms_noalloc",
    "isdf_adjoint_partial_size", "isdf_energy_gradient_shard", "isdf_energy_gradient_finish",
    "isdf_select_fit", "isdf_select_fit_host", "isdf_launch_count", "isdf_sketch_factors",
    "isdf_grid_metric", "isdf_grid_metric_host", "isdf_evaluate_axis_mo", "isdf_evaluate_axis_mo_host",
    "isdf_rbrp_args_default", "isdf_rbrp_ao", "isdf_rbrp_points", "isdf_rbrp_result_info",
    "isdf_rbrp_result_copy", "isdf_rbrp_result_free",
    "isdf_sketch_shard_project", "isdf_sketch_shard_combine", "isdf_sketch_shard_free",
    "isdf_sketch_select_gathered", "isdf_fit_at", "isdf_jk", "isdf_jk_host",
    "isdf_pairqr_shard_create", "isdf_pairqr_shard_init", "isdf_pairqr_shard_argmax", "isdf_pairqr_shard_row",
    "isdf_pairqr_shard_verify", "isdf_pairqr_shard_accept", "isdf_pairqr_shard_scan", "isdf_pairqr_shard_free",
    "isdf_qr_shard_create", "isdf_qr_shard_update", "isdf_qr_shard_verify", "isdf_qr_shard_column",
    "isdf_qr_shard_pivot", "isdf_qr_shard_reverified", "isdf_qr_shard_free", "isdf_sketch_rank",
]

ALGORITHMS = {"qrcp_dense": 0, "qrcp_online": 1, "rand_sketch": 2, "rand_sketch_density": 4,
              "rand_sketch_density_col_norm": 5}
AXES = {"ao": 0, "dx": 1, "dy": 2, "dz": 3, "occ": 4}


class SelectArgs(ctypes.Structure):
    _fields_ = [("algorithm", I32), ("naxes", I32), ("axes", P), ("axis_weights", P),
                ("tolerance", F64), ("max_rank", I64), ("batch_size", I64),
                ("sketch_size", I64), ("oversampling", I64), ("seed", ctypes.c_uint64),
                ("precision", I32), ("debug", I32), ("point_importance", P),
                ("ao_screening_threshold", F64), ("mo_coeff", P), ("nocc", I64)]


class RbrpArgs(ctypes.Structure):
    _fields_ = [("batch_size", I64), ("block_size", I64), ("tolerance", F64), ("max_rank", I64),
                ("seed", ctypes.c_uint64), ("tau_block", F64), ("rank_rtol", F64),
                ("refresh_every", I64), ("svd_rtol", F64), ("compute_id", I32)]


class SelectInfo(ctypes.Structure):
    _fields_ = [("n_kept", I64), ("sketch_rows", I64), ("numerical_rank", I64),
                ("verifications", I64), ("reselections", I64), ("relative_residual", F64),
                ("precision_used", I64)]


class FitInfo(ctypes.Structure):
    _fields_ = [("n_kept", I64), ("retained_rank", I64), ("condition", F64),
                ("max_abs_physical_coefficient", F64), ("pair_l2", F64),
                ("pair_relative", F64), ("theta_w", F64 * 64), ("fit_path", I64),
                ("mixed_bound", F64)]


class IsdfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing; run `python -m mp_isdf_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        L.isdf_status_string.restype = ctypes.c_char_p
        L.isdf_last_error.restype = ctypes.c_char_p
        L.isdf_ctx_create.argtypes = [P, I32, P, I32, P, I64, ctypes.POINTER(P)]
        L.isdf_ctx_destroy.argtypes = [P]
        L.isdf_ctx_info.argtypes = [P, ctypes.POINTER(I64), ctypes.POINTER(I32), ctypes.POINTER(I32)]
        L.isdf_ctx_ao_atoms.argtypes = [P, P]
        L.isdf_eval_ao.argtypes = [P, P, I64, I32, P, P, P]
        L.isdf_eval_ao_host.argtypes = [P, P, I64, P, P]
        L.isdf_evaluate_axis.argtypes = [P, P, I64, P, I32, P, P]
        L.isdf_evaluate_axis_host.argtypes = [P, P, I64, P, I32, P]
        L.isdf_evaluate_axis_mo.argtypes = [P, P, I64, P, I32, P, I64, P, P]
        L.isdf_rbrp_args_default.argtypes = [ctypes.POINTER(RbrpArgs)]
        L.isdf_rbrp_args_default.restype = None
        L.isdf_rbrp_ao.argtypes = [P, P, P, I64, I64, ctypes.POINTER(RbrpArgs), ctypes.POINTER(P)]
        L.isdf_rbrp_points.argtypes = [P, P, P, I64, ctypes.POINTER(RbrpArgs), ctypes.POINTER(P)]
        L.isdf_rbrp_result_info.argtypes = [P, P, P, P, P, P, P, P, ctypes.c_char_p, I64]
        L.isdf_rbrp_result_copy.argtypes = [P, P, P, P, P]
        L.isdf_rbrp_result_free.argtypes = [P]
        L.isdf_rbrp_result_free.restype = None
        L.isdf_evaluate_axis_mo_host.argtypes = [P, P, I64, P, I32, P, I64, P]
        L.isdf_select_args_default.argtypes = [ctypes.POINTER(SelectArgs)]
        L.isdf_select.argtypes = [P, ctypes.POINTER(SelectArgs), P, P, I64, P, I64,
                                  ctypes.POINTER(I64), ctypes.POINTER(SelectInfo), P]
        L.isdf_select_host.argtypes = [P, ctypes.POINTER(SelectArgs), P, P, I64, P, I64,
                                       ctypes.POINTER(I64), ctypes.POINTER(SelectInfo)]
        L.isdf_fit.argtypes = [P, P, P, I64, P, I64, I32, I32, P, ctypes.POINTER(FitInfo), P]
        L.isdf_fit_host.argtypes = [P, P, P, I64, P, I64, I32, I32, P, ctypes.POINTER(FitInfo)]
        L.isdf_select_fit.argtypes = [P, ctypes.POINTER(SelectArgs), P, P, I64, P, I64,
                                      ctypes.POINTER(I64), ctypes.POINTER(SelectInfo), I32, P,
                                      ctypes.POINTER(FitInfo), P]
        L.isdf_select_fit_host.argtypes = [P, ctypes.POINTER(SelectArgs), P, P, I64, P, I64,
                                           ctypes.POINTER(I64), ctypes.POINTER(SelectInfo), I32, P,
                                           ctypes.POINTER(FitInfo)]
        L.isdf_sketch_shard_project.argtypes = [P, ctypes.POINTER(SelectArgs), P, P, I64, I64,
                                                ctypes.POINTER(P), ctypes.POINTER(I64),
                                                ctypes.POINTER(I64), P, P]
        L.isdf_sketch_shard_combine.argtypes = [P, P, P, P, P, P, P, P, P]
        L.isdf_sketch_shard_free.argtypes = [P]
        L.isdf_sketch_shard_free.restype = None
        L.isdf_sketch_select_gathered.argtypes = [P, ctypes.POINTER(SelectArgs), P, I64, P, P, P, P, P,
                                                  I64, ctypes.POINTER(I64), ctypes.POINTER(SelectInfo), P]
        L.isdf_fit_at.argtypes = [P, P, P, I64, P, P, I64, I32, I32, P, ctypes.POINTER(FitInfo), P, P]
        L.isdf_qr_shard_create.argtypes = [P, ctypes.POINTER(SelectArgs), P, I64, I64, I64, P, P, P, P,
                                           ctypes.POINTER(P), ctypes.POINTER(I64), ctypes.POINTER(I32), P]
        L.isdf_qr_shard_update.argtypes = [P, I64, ctypes.POINTER(F64), ctypes.POINTER(I64), ctypes.POINTER(I64),
                                           ctypes.POINTER(F64), ctypes.POINTER(F64)]
        L.isdf_qr_shard_verify.argtypes = [P, I64, F64, ctypes.POINTER(F64), ctypes.POINTER(I64),
                                           ctypes.POINTER(I64)]
        L.isdf_qr_shard_column.argtypes = [P, I64, P]
        L.isdf_qr_shard_pivot.argtypes = [P, I64, P, I64, I64, I64, ctypes.POINTER(F64)]
        L.isdf_qr_shard_reverified.argtypes = [P, ctypes.POINTER(I64)]
        L.isdf_qr_shard_free.argtypes = [P]
        L.isdf_pairqr_shard_create.argtypes = [P, ctypes.POINTER(SelectArgs), P, P, I64, I64, ctypes.POINTER(P),
                                               ctypes.POINTER(I64), ctypes.POINTER(I64), P, P]
        L.isdf_pairqr_shard_init.argtypes = [P, P, I64, P]
        L.isdf_pairqr_shard_argmax.argtypes = [P, P]
        L.isdf_pairqr_shard_row.argtypes = [P, I64, P]
        L.isdf_pairqr_shard_verify.argtypes = [P, P, I64, I64, ctypes.POINTER(F64)]
        L.isdf_pairqr_shard_accept.argtypes = [P, P, I64, I64, F64, I64, I32]
        L.isdf_pairqr_shard_scan.argtypes = [P, I64, F64, ctypes.POINTER(I64)]
        L.isdf_pairqr_shard_free.argtypes = [P]
        L.isdf_pairqr_shard_free.restype = None
        L.isdf_qr_shard_free.restype = None
        L.isdf_sketch_rank.argtypes = [P, ctypes.POINTER(SelectArgs), I64, P, P, I64, ctypes.POINTER(I64),
                                       ctypes.POINTER(I64), ctypes.POINTER(F64)]
        L.isdf_pair_error.argtypes = [P, P, P, I64, P, I64, P, ctypes.POINTER(F64),
                                      ctypes.POINTER(F64), P]
        L.isdf_pair_error_terms.argtypes = [I64, I64, P, P, P, P, P, P, P]
        L.isdf_pair_error_terms_noalloc.argtypes = [I64, I64, P, P, P, P, P, P, P]
        L.isdf_project_axes.argtypes = [P, P, I64, P, I32, P, I32, I32, P, P]
        L.isdf_energy_gradient.argtypes = [P, P, P, I64, P, I64, P, ctypes.POINTER(F64), P, P]
        L.isdf_adjoint_partial_size.argtypes = [P, I64, ctypes.POINTER(I64)]
        L.isdf_energy_gradient_shard.argtypes = [P, P, P, I64, P, P, I64, P, I32, P, P]
        L.isdf_energy_gradient_finish.argtypes = [P, P, P, I64, P, P, ctypes.POINTER(F64), P, P]
        L.isdf_ctx_set_coords.argtypes = [P, P]
        L.isdf_profile_enable.argtypes = [I32]
        L.isdf_launch_count.argtypes = []
        L.isdf_launch_count.restype = I64
        L.isdf_sketch_factors.argtypes = [I64, I64, ctypes.c_uint64, P, P]
        L.isdf_grid_metric.argtypes = [P, P, I64, I64, P, I64, I64, P, P, I64, I32, P, P]
        L.isdf_grid_metric_host.argtypes = [P, P, I64, P, I64, P, P, I64, I32, P]
        L.isdf_jk.argtypes = [P, P, I64, P, P, P, P, P]
        L.isdf_jk_host.argtypes = [P, P, I64, P, P, P, P]
        L.isdf_profile_read.argtypes = [I32, P, P, P, ctypes.POINTER(I32)]
        _lib = L
    return _lib


def check(status: int):
    if status != 0:
        raise IsdfError(status, lib().isdf_last_error().decode())


def _np(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr(a):
    """Data pointer of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(P)
    return P(a.data_ptr())


def _stream(t):
    import torch
    return P(torch.cuda.current_stream(t.device).cuda_stream)


class Context:
    """Device context over libcint-layout tables (C-ABI ``isdf_ctx``)."""

    def __init__(self, atm, bas, env):
        self._atm = _np(atm, np.int32)
        self._bas = _np(bas, np.int32)
        self._env = _np(env, np.float64)
        h = P()
        check(lib().isdf_ctx_create(_ptr(self._atm), len(self._atm), _ptr(self._bas),
                                    len(self._bas), _ptr(self._env), len(self._env),
                                    ctypes.byref(h)))
        self.h = h
        nao, natm, nsh = I64(), I32(), I32()
        check(lib().isdf_ctx_info(self.h, ctypes.byref(nao), ctypes.byref(natm), ctypes.byref(nsh)))
        self.nao, self.natm, self.nshell = nao.value, natm.value, nsh.value
        self.ao_atoms = np.empty(self.nao, dtype=np.int32)
        check(lib().isdf_ctx_ao_atoms(self.h, _ptr(self.ao_atoms)))

    def close(self):
        if getattr(self, "h", None):
            lib().isdf_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter exit the module's globals may already be gone; the
        # process teardown releases the device context then
        try:
            self.close()
        except Exception:
            pass

    # ---- device tensors ------------------------------------------------------
    def eval_ao(self, xyz, values=None, grad=None, dtype=None):
        """xyz: CUDA float64 tensor [ng,3]; fills/returns values [ng,nao] and/or grad [3,ng,nao]."""
        import torch
        ng = xyz.shape[0]
        dt = dtype or (values.dtype if values is not None else torch.float64)
        code = 0 if dt == torch.float64 else 1
        check(lib().isdf_eval_ao(self.h, _ptr(xyz), ng, code, _ptr(values), _ptr(grad),
                                 _stream(xyz)))
        return values, grad

    def select(self, xyz, w, algorithm="rand_sketch", axes=("ao",), axis_weights=None,
               tolerance=1e-10, max_rank=0, batch_size=128, sketch_size=128, oversampling=16,
               seed=7, precision="fp64", debug=False, point_importance=None, ao_screening_threshold=1e-24,
               mo_coeff=None, nocc=0):
        """Anchor selection on device-resident points/weights; returns (pivots, info)."""
        args, keep = make_select_args(algorithm, axes, axis_weights, tolerance, max_rank,
                                      batch_size, sketch_size, oversampling, seed, precision, debug,
                                      point_importance, ao_screening_threshold, mo_coeff, nocc)
        ng = xyz.shape[0]
        piv = np.empty(max(ng, 1), dtype=np.int64)
        n = I64()
        info = SelectInfo()
        check(lib().isdf_select(self.h, ctypes.byref(args), _ptr(xyz), _ptr(w), ng, _ptr(piv),
                                len(piv), ctypes.byref(n), ctypes.byref(info), _stream(xyz)))
        del keep
        return piv[:n.value].copy(), info

    def fit(self, xyz, w, anchors, theta, precision="fp64", want_error=True):
        """Theta into the CUDA float64 tensor `theta` (capacity k*ng); returns FitInfo."""
        a = _np(anchors, np.int64)
        info = FitInfo()
        check(lib().isdf_fit(self.h, _ptr(xyz), _ptr(w), xyz.shape[0], _ptr(a), len(a),
                             1 if precision == "mixed" else 0, int(want_error), _ptr(theta),
                             ctypes.byref(info), _stream(xyz)))
        return info

    def select_fit(self, xyz, w, theta, want_error=True, **kw):
        """Selection then fit on the same device points in one call (keyword
        arguments as select()); Theta into `theta` (capacity max_rank * ng).
        Returns (pivots, select info, fit info)."""
        args, keep = make_select_args(**kw)
        ng = xyz.shape[0]
        cap = max(1, min(ng, theta.numel() // max(ng, 1)))
        piv = np.empty(cap, dtype=np.int64)
        n = I64()
        sinfo, finfo = SelectInfo(), FitInfo()
        check(lib().isdf_select_fit(self.h, ctypes.byref(args), _ptr(xyz), _ptr(w), ng, _ptr(piv),
                                    len(piv), ctypes.byref(n), ctypes.byref(sinfo), int(want_error),
                                    _ptr(theta), ctypes.byref(finfo), _stream(xyz)))
        del keep
        return piv[:n.value].copy(), sinfo, finfo

    # ---- grid-sharded selection phases (see mp_isdf_b200.sharded) ----------------
    def sketch_shard_project(self, xyz, w, ng_total, **kw):
        """Project this rank's grid shard (device tensors).  Returns (shard
        handle, kept points, sketch rows, per-component sums of squares [4])."""
        args, keep = make_select_args(**kw)
        h, n, ell = P(), I64(), I64()
        sumsq = np.zeros(4)
        check(lib().isdf_sketch_shard_project(self.h, ctypes.byref(args), _ptr(xyz), _ptr(w), xyz.shape[0],
                                              int(ng_total), ctypes.byref(h), ctypes.byref(n),
                                              ctypes.byref(ell), _ptr(sumsq), _stream(xyz)))
        del keep
        return SketchShard(h.value, xyz), n.value, ell.value, sumsq

    def sketch_shard_combine(self, shard, sumsq_global, ell, n_kept, naxes):
        """The shard's sketch columns with the global scales: (yt [ell, n_kept],
        delta [n_kept], kept grid indices, kept xyz [n_kept, 3], kept w, scales)."""
        import torch
        dev = shard.xyz.device
        yt = torch.empty(ell, max(n_kept, 1), dtype=torch.float64, device=dev)
        delta = torch.zeros(max(n_kept, 1), dtype=torch.float64, device=dev)
        kept = torch.empty(max(n_kept, 1), dtype=torch.int64, device=dev)
        kxyz = torch.empty(max(n_kept, 1), 3, dtype=torch.float64, device=dev)
        kw_ = torch.empty(max(n_kept, 1), dtype=torch.float64, device=dev)
        scales = np.ones(naxes)
        sg = _np(sumsq_global, np.float64)
        check(lib().isdf_sketch_shard_combine(shard.h, _ptr(sg), _ptr(yt), _ptr(delta), _ptr(kept), _ptr(kxyz),
                                              _ptr(kw_), _ptr(scales), _stream(shard.xyz)))
        return (yt[:, :n_kept], delta[:n_kept], kept[:n_kept], kxyz[:n_kept], kw_[:n_kept], scales)

    def sketch_select_gathered(self, yt, kept_xyz, kept_w, delta, scales, **kw):
        """Pivoted QR of a gathered sketch (device tensors; yt contiguous
        [ell, n]); returns (positions in the gathered order, SelectInfo)."""
        args, keep = make_select_args(**kw)
        n = yt.shape[1]
        piv = np.empty(max(n, 1), dtype=np.int64)
        npiv = I64()
        info = SelectInfo()
        sc = _np(scales, np.float64)
        check(lib().isdf_sketch_select_gathered(self.h, ctypes.byref(args), _ptr(yt), n, _ptr(kept_xyz),
                                                _ptr(kept_w), _ptr(delta), _ptr(sc), _ptr(piv), len(piv),
                                                ctypes.byref(npiv), ctypes.byref(info), _stream(yt)))
        del keep
        return piv[:npiv.value].copy(), info

    def pairqr_shard(self, xyz, w, grid_offset, **kw):
        """This rank's share of the sharded pair-space QR (qrcp_dense /
        qrcp_online) over its grid shard (device tensors)."""
        args, keep = make_select_args(**kw)
        h, n, d = P(), I64(), I64()
        sumsq = np.zeros(5)
        check(lib().isdf_pairqr_shard_create(self.h, ctypes.byref(args), _ptr(xyz), _ptr(w), xyz.shape[0],
                                             int(grid_offset), ctypes.byref(h), ctypes.byref(n), ctypes.byref(d),
                                             _ptr(sumsq), _stream(xyz)))
        del keep
        return PairQrShard(h.value, n.value, d.value, sumsq, (xyz, w))

    def qr_shard(self, yt, n_total, pos_offset, kept_xyz, kept_w, delta, scales, **kw):
        """This rank's share of the distributed sketch QR over its columns yt
        ([ell, n_local] device tensor)."""
        args, keep = make_select_args(**kw)
        h, ell, ver = P(), I64(), I32()
        sc = _np(scales, np.float64)
        n_local = yt.shape[1] if yt.dim() == 2 else 0
        check(lib().isdf_qr_shard_create(self.h, ctypes.byref(args), _ptr(yt), n_local, n_total, pos_offset,
                                         _ptr(kept_xyz), _ptr(kept_w), _ptr(delta), _ptr(sc), ctypes.byref(h),
                                         ctypes.byref(ell), ctypes.byref(ver), _stream(yt)))
        del keep
        return QrShard(h.value, ell.value, bool(ver.value), (yt, kept_xyz, kept_w, delta))

    def sketch_rank(self, n_total, diag, energy, **kw):
        """(rank, numerical rank, relative tail) of a sketch QR's |R_jj| and row energies."""
        args, keep = make_select_args(**kw)
        d, e = _np(diag, np.float64), _np(energy, np.float64)
        r, nr, t = I64(), I64(), F64()
        check(lib().isdf_sketch_rank(self.h, ctypes.byref(args), n_total, _ptr(d), _ptr(e), len(d),
                                     ctypes.byref(r), ctypes.byref(nr), ctypes.byref(t)))
        del keep
        return r.value, nr.value, t.value

    def fit_at(self, xyz, w, anchor_xyz, anchor_w, theta, precision="fp64", want_error=True):
        """Fit on device points with anchors given by coordinates; returns
        (FitInfo, [err2, exact2] of these points)."""
        axyz = _np(anchor_xyz, np.float64).reshape(-1, 3)
        aw = _np(anchor_w, np.float64)
        info = FitInfo()
        sums = np.zeros(2)
        check(lib().isdf_fit_at(self.h, _ptr(xyz), _ptr(w), xyz.shape[0], _ptr(axyz), _ptr(aw), len(aw),
                                1 if precision == "mixed" else 0, int(want_error), _ptr(theta),
                                ctypes.byref(info), _ptr(sums), _stream(xyz)))
        return info, sums

    def pair_error(self, xyz, w, anchors, theta):
        a = _np(anchors, np.int64)
        l2, rel = F64(), F64()
        check(lib().isdf_pair_error(self.h, _ptr(xyz), _ptr(w), xyz.shape[0], _ptr(a), len(a),
                                    _ptr(theta), ctypes.byref(l2), ctypes.byref(rel),
                                    _stream(xyz)))
        return l2.value, rel.value

    def project_axes(self, xyz, axes, W, precision="fp64"):
        """out[g][a][j] = sum_mu comp_a(g, mu) W[a*nao+mu][j] (CUDA float64 tensor)."""
        import torch
        ax = np.array([AXES[a] if isinstance(a, str) else int(a) for a in axes], dtype=np.int32)
        W = _np(W, np.float64)
        nout = W.shape[1]
        out = torch.empty(xyz.shape[0], len(ax), nout, dtype=torch.float64, device=xyz.device)
        check(lib().isdf_project_axes(self.h, _ptr(xyz), xyz.shape[0], _ptr(ax), len(ax), _ptr(W),
                                      nout, 1 if precision == "mixed" else 0, _ptr(out),
                                      _stream(xyz)))
        return out

    def grid_metric(self, xyz, w, left, right=None):
        """Grid Coulomb metric of device tensors (left/right: k x n float64,
        not weight-scaled); right=None gives the symmetrised metric of `left`."""
        sym = right is None
        right = left if sym else right
        out = np.empty((left.shape[0], right.shape[0]), dtype=np.float64)
        check(lib().isdf_grid_metric(self.h, _ptr(left), left.stride(0), left.shape[0], _ptr(right),
                                     right.stride(0), right.shape[0], _ptr(xyz), _ptr(w), xyz.shape[0],
                                     int(sym), _ptr(out), _stream(xyz)))
        return out

    def evaluate_axis_host(self, xyz, axes, mo_coeff=None, nocc=0):
        """Concatenated axis features (host arrays; occupied-orbital entries
        nocc wide from the row-major nao x nao `mo_coeff`)."""
        ax = np.array([AXES[a] if isinstance(a, str) else int(a) for a in axes], dtype=np.int32)
        xyz = _np(xyz, np.float64).reshape(-1, 3)
        mo = None if mo_coeff is None else _np(mo_coeff, np.float64)
        d = sum(nocc if a == 4 else self.nao for a in ax)
        out = np.empty((len(xyz), d), dtype=np.float64)
        check(lib().isdf_evaluate_axis_mo_host(self.h, _ptr(xyz), len(xyz), _ptr(ax), len(ax), _ptr(mo),
                                               int(nocc), _ptr(out)))
        return out

    def set_coords(self, coords):
        """Move the atoms (natm x 3, bohr)."""
        c = _np(coords, np.float64).reshape(self.natm, 3)
        check(lib().isdf_ctx_set_coords(self.h, _ptr(c)))

    def energy_gradient(self, xyz, w, anchors, dm):
        """(E, dE/dR[natm,3]) of E = sum_g w_g rho_ISDF(g)^2 on device tensors."""
        a = _np(anchors, np.int64)
        d = _np(dm, np.float64)
        e = F64()
        g = np.zeros((self.natm, 3))
        check(lib().isdf_energy_gradient(self.h, _ptr(xyz), _ptr(w), xyz.shape[0], _ptr(a), len(a),
                                         _ptr(d), ctypes.byref(e), _ptr(g), _stream(xyz)))
        return e.value, g

    def energy_gradient_shard(self, xyz, w, anchor_xyz, anchor_w, dm, want_grad=True):
        """A grid shard's partial sums (numpy float64) of the adjoint for anchors
        given by coordinates (k x 3) and weights; device tensors xyz, w."""
        axyz = _np(anchor_xyz, np.float64).reshape(-1, 3)
        aw = _np(anchor_w, np.float64)
        d = _np(dm, np.float64)
        n = I64()
        check(lib().isdf_adjoint_partial_size(self.h, len(aw), ctypes.byref(n)))
        out = np.zeros(n.value)
        check(lib().isdf_energy_gradient_shard(self.h, _ptr(xyz), _ptr(w), xyz.shape[0], _ptr(axyz), _ptr(aw),
                                               len(aw), _ptr(d), 1 if want_grad else 0, _ptr(out),
                                               _stream(xyz)))
        return out

    def energy_gradient_finish(self, anchor_xyz, anchor_w, dm, sums, want_grad=True):
        """(E, dE/dR[natm,3]) from the partial sums added over all shards."""
        axyz = _np(anchor_xyz, np.float64).reshape(-1, 3)
        aw = _np(anchor_w, np.float64)
        d = _np(dm, np.float64)
        sm = _np(sums, np.float64)
        e = F64()
        g = np.zeros((self.natm, 3))
        check(lib().isdf_energy_gradient_finish(self.h, _ptr(axyz), _ptr(aw), len(aw), _ptr(d), _ptr(sm),
                                                ctypes.byref(e), _ptr(g) if want_grad else None, None))
        return e.value, g

    def energy(self, xyz, w, anchors, dm):
        """E = sum_g w_g rho_ISDF(g)^2 alone (no gradient sweep), device tensors."""
        a = _np(anchors, np.int64)
        d = _np(dm, np.float64)
        e = F64()
        check(lib().isdf_energy_gradient(self.h, _ptr(xyz), _ptr(w), xyz.shape[0], _ptr(a), len(a),
                                         _ptr(d), ctypes.byref(e), None, _stream(xyz)))
        return e.value

    # ---- host arrays -----------------------------------------------------------
    def eval_ao_host(self, xyz, gradient=False):
        xyz = _np(xyz, np.float64).reshape(-1, 3)
        out = np.empty((3, len(xyz), self.nao) if gradient else (len(xyz), self.nao))
        check(lib().isdf_eval_ao_host(self.h, _ptr(xyz), len(xyz),
                                      None if gradient else _ptr(out),
                                      _ptr(out) if gradient else None))
        return out

    def select_host(self, xyz, w, **kw):
        args, keep = make_select_args(**kw)
        xyz = _np(xyz, np.float64).reshape(-1, 3)
        w = _np(w, np.float64)
        piv = np.empty(max(len(xyz), 1), dtype=np.int64)
        n = I64()
        info = SelectInfo()
        check(lib().isdf_select_host(self.h, ctypes.byref(args), _ptr(xyz), _ptr(w), len(xyz),
                                     _ptr(piv), len(piv), ctypes.byref(n), ctypes.byref(info)))
        del keep
        return piv[:n.value].copy(), info

    def select_fit_host(self, xyz, w, want_error=True, out=None, **kw):
        """Selection then fit from host buffers in one call.  Returns (pivots,
        Theta [k, n_kept], select info, fit info); `out` may supply the float64
        host buffer for Theta (capacity ng * ng, or max_rank * ng when max_rank
        is given)."""
        args, keep = make_select_args(**kw)
        xyz = _np(xyz, np.float64).reshape(-1, 3)
        w = _np(w, np.float64)
        ng = len(xyz)
        cap = max(1, kw.get("max_rank") or ng)
        theta = out if out is not None else np.empty(max(1, cap * ng))
        if theta.dtype != np.float64 or not theta.flags.c_contiguous or theta.size < min(cap, ng) * ng:
            raise ValueError("out must be a contiguous float64 buffer of at least max_rank*ng entries")
        piv = np.empty(cap, dtype=np.int64)
        n = I64()
        sinfo, finfo = SelectInfo(), FitInfo()
        check(lib().isdf_select_fit_host(self.h, ctypes.byref(args), _ptr(xyz), _ptr(w), ng, _ptr(piv),
                                         len(piv), ctypes.byref(n), ctypes.byref(sinfo), int(want_error),
                                         _ptr(theta), ctypes.byref(finfo)))
        del keep
        k = n.value
        return piv[:k].copy(), theta[:k * finfo.n_kept].reshape(k, finfo.n_kept), sinfo, finfo

    def fit_host(self, xyz, w, anchors, precision="fp64", want_error=True, out=None):
        """Theta (k x n_kept) from host buffers.  `out` may supply the float64
        host buffer (capacity k*ng, e.g. pinned memory) that Theta lands in."""
        xyz = _np(xyz, np.float64).reshape(-1, 3)
        w = _np(w, np.float64)
        a = _np(anchors, np.int64)
        if out is None:
            theta = np.empty(max(1, len(a) * len(xyz)))
        else:
            theta = out
            if theta.dtype != np.float64 or not theta.flags.c_contiguous or theta.size < len(a) * len(xyz):
                raise ValueError("out must be a contiguous float64 buffer of at least k*ng entries")
        info = FitInfo()
        check(lib().isdf_fit_host(self.h, _ptr(xyz), _ptr(w), len(xyz), _ptr(a), len(a),
                                  1 if precision == "mixed" else 0, int(want_error), _ptr(theta),
                                  ctypes.byref(info)))
        return theta[:len(a) * info.n_kept].reshape(len(a), info.n_kept), info


class PairQrShard:
    """One rank's share of the sharded pair-space QR (isdf_pairqr_shard_*)."""

    def __init__(self, h, n_kept, d, sumsq, keep):
        self.h, self.n_kept, self.d, self.sumsq = h, n_kept, d, sumsq
        self._keep = keep   # the device arrays the handle points at

    def init(self, sumsq_global, pos_offset):
        out = np.zeros(2)
        check(lib().isdf_pairqr_shard_init(self.h, _ptr(_np(sumsq_global, np.float64)), int(pos_offset), _ptr(out)))
        return out

    def argmax(self):
        key = np.zeros(3)
        check(lib().isdf_pairqr_shard_argmax(self.h, _ptr(key)))
        return key

    def row(self, col):
        out = np.zeros(self.d + 6)
        check(lib().isdf_pairqr_shard_row(self.h, int(col), _ptr(out)))
        return out

    def verify(self, row, j, col):
        e = F64()
        check(lib().isdf_pairqr_shard_verify(self.h, _ptr(_np(row, np.float64)), int(j), int(col), ctypes.byref(e)))
        return e.value

    def accept(self, row, j, col, exact2, winner_pos, dense):
        check(lib().isdf_pairqr_shard_accept(self.h, _ptr(_np(row, np.float64)), int(j), int(col), float(exact2),
                                             int(winner_pos), 1 if dense else 0))

    def scan(self, j, thr2):
        n = I64()
        check(lib().isdf_pairqr_shard_scan(self.h, int(j), float(thr2), ctypes.byref(n)))
        return n.value

    def free(self):
        if self.h:
            lib().isdf_pairqr_shard_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class QrShard:
    """One rank's share of the distributed sketch QR (isdf_qr_shard_*)."""

    def __init__(self, h, ell, verified, keep):
        self.h, self.ell, self.verified = h, ell, verified
        self._keep = keep   # the device arrays the handle points at

    def update(self, j):
        v, e, lb = F64(), F64(), F64()
        p, c = I64(), I64()
        check(lib().isdf_qr_shard_update(self.h, j, ctypes.byref(v), ctypes.byref(p), ctypes.byref(c),
                                         ctypes.byref(e), ctypes.byref(lb)))
        return v.value, p.value, c.value, e.value, lb.value

    def verify(self, j, bound):
        v, p, c = F64(), I64(), I64()
        check(lib().isdf_qr_shard_verify(self.h, j, bound, ctypes.byref(v), ctypes.byref(p), ctypes.byref(c)))
        return v.value, p.value, c.value

    def column(self, col):
        rows = np.empty(self.ell)
        check(lib().isdf_qr_shard_column(self.h, col, _ptr(rows)))
        return rows

    def pivot(self, j, rows, pivot_col, pivot_pos, moved_col):
        rows = _np(rows, np.float64)
        r = F64()
        check(lib().isdf_qr_shard_pivot(self.h, j, _ptr(rows), pivot_col, pivot_pos, moved_col, ctypes.byref(r)))
        return r.value

    def reverified(self):
        n = I64()
        check(lib().isdf_qr_shard_reverified(self.h, ctypes.byref(n)))
        return n.value

    def free(self):
        if self.h:
            lib().isdf_qr_shard_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class SketchShard:
    """Owns a projected grid shard (isdf_sketch_shard) until it is freed."""

    def __init__(self, h, xyz):
        self.h = h
        self.xyz = xyz     # keeps the shard's grid alive for the combine step

    def free(self):
        if self.h:
            lib().isdf_sketch_shard_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def make_select_args(algorithm="rand_sketch", axes=("ao",), axis_weights=None, tolerance=1e-10,
                     max_rank=0, batch_size=128, sketch_size=128, oversampling=16, seed=7,
                     precision="fp64", debug=False, point_importance=None, ao_screening_threshold=1e-24,
                     mo_coeff=None, nocc=0):
    """isdf_select_args (and the arrays it points at, to keep alive).  For the
    density sketches `point_importance` is a float64 vector over the grid: a
    CUDA tensor for the device entry points, host memory for the _host ones."""
    args = SelectArgs()
    lib().isdf_select_args_default(ctypes.byref(args))
    ax = np.array([AXES[a] if isinstance(a, str) else int(a) for a in axes], dtype=np.int32)
    aw = None if axis_weights is None else _np(axis_weights, np.float64)
    args.algorithm = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
    args.naxes = len(ax)
    args.axes = _ptr(ax)
    args.axis_weights = _ptr(aw) if aw is not None else None
    args.tolerance = tolerance
    args.max_rank = max_rank
    args.batch_size = batch_size
    args.sketch_size = sketch_size
    args.oversampling = oversampling
    args.seed = seed
    args.precision = 1 if precision == "mixed" else 0
    args.debug = int(debug)
    imp = None
    if point_importance is not None:
        imp = point_importance if hasattr(point_importance, "data_ptr") else _np(point_importance, np.float64)
        args.point_importance = _ptr(imp)
    args.ao_screening_threshold = ao_screening_threshold
    mo = None
    if mo_coeff is not None:
        mo = _np(mo_coeff, np.float64)
        args.mo_coeff = _ptr(mo)
        args.nocc = int(nocc)
    return args, (ax, aw, imp, mo)


def _rbrp_collect(h):
    """Result dict of an isdf_rbrp_result handle (freed here), in the
    reference's layout (cpp/src/anchor_select_pybind.cpp:68-91)."""
    try:
        rank, nb, n, nao, ret = I64(), I64(), I64(), I64(), I64()
        rel, cond = F64(), F64()
        status = ctypes.create_string_buffer(64)
        check(lib().isdf_rbrp_result_info(h, ctypes.byref(rank), ctypes.byref(nb), ctypes.byref(n),
                                          ctypes.byref(nao), ctypes.byref(rel), ctypes.byref(cond),
                                          ctypes.byref(ret), status, 64))
        idx = np.empty(rank.value, dtype=np.int64)
        hist = np.empty((nb.value, 4))
        interp = np.empty((rank.value, n.value))
        transform = np.empty((rank.value, nao.value * nao.value))
        check(lib().isdf_rbrp_result_copy(h, _ptr(idx), _ptr(hist), _ptr(interp), _ptr(transform)))
        return {"indices": idx, "relative_residual": rel.value, "status": status.value.decode(),
                "condition": cond.value, "retained_rank": ret.value, "history": hist,
                "interp_vecs": interp, "transform": transform}
    finally:
        lib().isdf_rbrp_result_free(h)


def rbrp_args(batch_size=128, block_size=16, tolerance=1e-10, max_rank=0, seed=7, tau_block=None,
              rank_rtol=1e-12, refresh_every=8, svd_rtol=1e-12, compute_id=False):
    a = RbrpArgs()
    lib().isdf_rbrp_args_default(ctypes.byref(a))
    a.batch_size, a.block_size, a.tolerance, a.max_rank, a.seed = batch_size, block_size, tolerance, max_rank, seed
    a.tau_block = float("nan") if tau_block is None else tau_block
    a.rank_rtol, a.refresh_every, a.svd_rtol, a.compute_id = rank_rtol, refresh_every, svd_rtol, int(compute_id)
    return a


def rbrp_ao(ao, weights, ctx=None, **kw):
    """RBRP over host AO rows (n x nao) and weights; returns the result dict
    (interp_vecs / transform are meaningful with compute_id=True)."""
    ao = _np(ao, np.float64)
    w = _np(weights, np.float64)
    a = rbrp_args(**kw)
    h = P()
    check(lib().isdf_rbrp_ao(ctx.h if ctx is not None else None, _ptr(ao), _ptr(w), ao.shape[0], ao.shape[1],
                             ctypes.byref(a), ctypes.byref(h)))
    return _rbrp_collect(h)


def rbrp_points(ctx, xyz, weights, **kw):
    """RBRP with the AOs of the host points evaluated on the device."""
    xyz = _np(xyz, np.float64).reshape(-1, 3)
    w = _np(weights, np.float64)
    a = rbrp_args(**kw)
    h = P()
    check(lib().isdf_rbrp_points(ctx.h, _ptr(xyz), _ptr(w), len(w), ctypes.byref(a), ctypes.byref(h)))
    return _rbrp_collect(h)


def grid_metric_host(left, xyz, w, right=None, ctx=None):
    """Grid Coulomb metric between interpolation-vector sets (host arrays;
    left/right: k x n, not weight-scaled).  right=None: the symmetrised metric
    of `left` with itself."""
    left = _np(left, np.float64)
    sym = right is None
    right = left if sym else _np(right, np.float64)
    xyz = _np(xyz, np.float64).reshape(-1, 3)
    w = _np(w, np.float64)
    out = np.empty((left.shape[0], right.shape[0]), dtype=np.float64)
    check(lib().isdf_grid_metric_host(ctx.h if ctx is not None else None, _ptr(left), left.shape[0],
                                      _ptr(right), right.shape[0], _ptr(xyz), _ptr(w), len(w), int(sym),
                                      _ptr(out)))
    return out


def sketch_factors(d, ell, seed):
    """The rand_sketch Gaussian factors U, V (d x ell each), computed on the host."""
    u = np.empty((d, ell), dtype=np.float64)
    v = np.empty((d, ell), dtype=np.float64)
    check(lib().isdf_sketch_factors(d, ell, seed, u.ctypes.data, v.ctypes.data))
    return u, v


def launch_count():
    """Kernels launched by the library so far in this process."""
    return int(lib().isdf_launch_count())


def profile_enable(on=True):
    check(lib().isdf_profile_enable(1 if on else 0))


def profile_read(max_entries=64):
    """{family: (total_ms, launches)} since the last read, sorted by time."""
    names = ctypes.create_string_buffer(48 * max_entries)
    ms = np.zeros(max_entries)
    cnt = np.zeros(max_entries, dtype=np.int64)
    n = I32()
    check(lib().isdf_profile_read(max_entries, names, _ptr(ms), _ptr(cnt), ctypes.byref(n)))
    out = {}
    for i in range(n.value):
        name = names.raw[48 * i:48 * (i + 1)].split(b"\0", 1)[0].decode()
        out[name] = (float(ms[i]), int(cnt[i]))
    return out


def pair_error_terms(q, H, X, M, w):
    """{l2, relative} from device tensors (see isdf_pair_error_terms)."""
    n, k = H.shape
    out = np.zeros(2)
    check(lib().isdf_pair_error_terms(n, k, _ptr(q), _ptr(H), _ptr(X), _ptr(M), _ptr(w),
                                      _ptr(out), _stream(q)))
    return {"l2": out[0], "relative": out[1]}
