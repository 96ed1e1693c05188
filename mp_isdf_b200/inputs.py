"""Seeded synthetic inputs for the ISDF hot path: water clusters, a
cc-pVDZ-shaped Gaussian basis in libcint ATM/BAS/ENV layout, and an
atom-centred Becke-partitioned molecular grid.

PySCF (which builds the molecule tables and the Becke grid in the reference
driver, ``python/isdf.py:488-501``) is not available, so this module stands
in for it:

* ``water_cluster`` places waters (O-H 0.9572 A, H-O-H 104.52 deg, random
  rotation) on a cubic lattice of 3.0 A with +-0.2 A uniform jitter.
* ``synthetic_basis`` builds the cc-pVDZ *shell structure* (O [3s2p1d] from a
  9-primitive general s contraction, H [2s1p]; 24 AOs per water) with seeded
  even-tempered exponents.  Coefficients are normalised exactly as PySCF
  stores them in ``mol._env`` (primitive ``gto_norm`` times a per-contraction
  normalisation), so every spherical AO integrates to one.  The numbers are
  synthetic, not the published cc-pVDZ values.
* ``becke_grid`` builds Gauss-Chebyshev radial x Lebedev angular atomic grids
  with Becke fuzzy-cell weights restricted to the nearest atoms.  Point counts
  are tuned to the reference's level-2 / level-3 grid sizes (about 2e4 and
  3.1e4 points per water).

libcint slot layout (``cpp/include/libcint_wrapper.hpp:32-51``; slots as used
by ``cpp/src/ao_eval.cpp:94-119``): ATM row = [charge, ptr_coord, nuc_mod,
ptr_zeta, ptr_frac_charge, reserved]; BAS row = [atom, l, nprim, nctr, kappa,
ptr_exp, ptr_coeff, reserved]; ENV payload starts at offset 20.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from math import gamma, pi, sqrt

import numpy as np

ANGSTROM_TO_BOHR = 1.8897261246257702
PTR_ENV_START = 20
ATM_SLOTS = 6
BAS_SLOTS = 8


# --------------------------------------------------------------------------
# geometry
# --------------------------------------------------------------------------
def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a*a + b*b - c*c - d*d, 2*(b*c - a*d), 2*(b*d + a*c)],
        [2*(b*c + a*d), a*a - b*b + c*c - d*d, 2*(c*d - a*b)],
        [2*(b*d - a*c), 2*(c*d + a*b), a*a - b*b - c*c + d*d],
    ])


def water_cluster(lattice=(2, 2, 1), seed=0, spacing=3.0, jitter=0.2):
    """Return (symbols, coords_bohr[natm,3]) for len(lattice) product waters."""
    rng = np.random.default_rng(seed)
    r_oh, angle = 0.9572, np.deg2rad(104.52)
    local = np.array([
        [0.0, 0.0, 0.0],
        [r_oh * np.sin(angle / 2), 0.0, r_oh * np.cos(angle / 2)],
        [-r_oh * np.sin(angle / 2), 0.0, r_oh * np.cos(angle / 2)],
    ])
    symbols, coords = [], []
    for i in range(lattice[0]):
        for j in range(lattice[1]):
            for k in range(lattice[2]):
                rot = _random_rotation(rng)
                origin = np.array([i, j, k], dtype=float) * spacing
                origin += rng.uniform(-jitter, jitter, size=3)
                for sym, pos in zip("OHH", local @ rot.T + origin):
                    symbols.append(sym)
                    coords.append(pos)
    return symbols, np.asarray(coords) * ANGSTROM_TO_BOHR


# --------------------------------------------------------------------------
# basis
# --------------------------------------------------------------------------
def gto_norm(l: int, alpha: np.ndarray) -> np.ndarray:
    """Radial normalisation of r^l exp(-alpha r^2) (PySCF ``gto_norm``)."""
    alpha = np.asarray(alpha, dtype=float)
    return np.sqrt(2.0 ** (2 * l + 3) * gamma(l + 2) * (2 * alpha) ** (l + 1.5)
                   / (gamma(2 * l + 3) * sqrt(pi)))


def normalise_contraction(l: int, exps: np.ndarray, coeffs: np.ndarray) -> np.ndarray:
    """Return env-ready coefficients [nctr, nprim]: c * gto_norm scaled so each
    contracted radial function satisfies int R^2 r^(2l+2) dr = 1."""
    exps = np.asarray(exps, dtype=float)
    cs = np.asarray(coeffs, dtype=float).reshape(-1, len(exps))
    cs = cs * gto_norm(l, exps)[None, :]
    ee = exps[:, None] + exps[None, :]
    s = gamma(l + 1.5) / (2.0 * ee ** (l + 1.5))
    norms = np.einsum("ip,pq,iq->i", cs, s, cs)
    return cs / np.sqrt(norms)[:, None]


@dataclass
class Shell:
    l: int
    exps: np.ndarray
    coeffs: np.ndarray          # [nctr, nprim], raw contraction coefficients


def _even_tempered(hi: float, lo: float, n: int, rng) -> np.ndarray:
    if n == 1:
        return np.array([hi * np.exp(rng.uniform(-0.05, 0.05))])
    base = np.geomspace(hi, lo, n)
    return base * np.exp(rng.uniform(-0.05, 0.05, size=n))


def element_shells(symbol: str, seed: int = 1234) -> list[Shell]:
    """cc-pVDZ-shaped shells with synthetic seeded exponents/coefficients."""
    rng = np.random.default_rng(seed + (0 if symbol == "O" else 1))
    if symbol == "O":
        s_exp = _even_tempered(1.2e4, 0.30, 9, rng)
        core = np.exp(-0.5 * ((np.arange(9) - 3.0) / 1.6) ** 2) * rng.uniform(0.8, 1.2, 9)
        valence = np.exp(-0.5 * ((np.arange(9) - 7.0) / 1.2) ** 2) * rng.uniform(0.8, 1.2, 9)
        valence[:5] -= 0.15 * core[:5]
        p_exp = _even_tempered(17.0, 0.35, 4, rng)
        p_c = np.exp(-0.5 * ((np.arange(4) - 2.0) / 1.3) ** 2) * rng.uniform(0.8, 1.2, 4)
        return [
            Shell(0, s_exp, np.vstack([core, valence])),
            Shell(0, _even_tempered(0.30, 0.30, 1, rng), np.ones((1, 1))),
            Shell(1, p_exp, p_c[None, :]),
            Shell(1, _even_tempered(0.27, 0.27, 1, rng), np.ones((1, 1))),
            Shell(2, _even_tempered(1.18, 1.18, 1, rng), np.ones((1, 1))),
        ]
    if symbol == "H":
        s_exp = _even_tempered(13.0, 0.45, 3, rng)
        s_c = np.array([0.2, 0.5, 0.6]) * rng.uniform(0.9, 1.1, 3)
        return [
            Shell(0, s_exp, s_c[None, :]),
            Shell(0, _even_tempered(0.122, 0.122, 1, rng), np.ones((1, 1))),
            Shell(1, _even_tempered(0.727, 0.727, 1, rng), np.ones((1, 1))),
        ]
    raise ValueError(f"synthetic basis has no element {symbol!r}")


CHARGES = {"H": 1, "O": 8}


@dataclass
class Molecule:
    symbols: list
    coords: np.ndarray          # bohr
    atm: np.ndarray             # int32 [natm, 6]
    bas: np.ndarray             # int32 [nbas, 8]
    env: np.ndarray             # float64
    nao: int
    basis_label: str = "synthetic-cc-pVDZ-shaped"
    meta: dict = field(default_factory=dict)

    def with_coords(self, coords: np.ndarray) -> "Molecule":
        env = self.env.copy()
        for a in range(len(self.symbols)):
            p = self.atm[a, 1]
            env[p:p + 3] = coords[a]
        return Molecule(self.symbols, np.asarray(coords, dtype=float).copy(),
                        self.atm.copy(), self.bas.copy(), env, self.nao,
                        self.basis_label, dict(self.meta))


def build_tables(symbols, coords_bohr, shells_of=element_shells) -> Molecule:
    """libcint tables for the given atoms and per-element shells."""
    env = [0.0] * PTR_ENV_START
    atm, bas = [], []
    for sym, xyz in zip(symbols, coords_bohr):
        ptr = len(env)
        env.extend(float(v) for v in xyz)
        env.append(0.0)                       # zeta slot
        atm.append([CHARGES.get(sym, 0), ptr, 1, ptr + 3, 0, 0])
    cache = {}
    nao = 0
    for ia, sym in enumerate(symbols):
        if sym not in cache:
            entries = []
            for sh in shells_of(sym):
                pe = len(env)
                env.extend(sh.exps.tolist())
                pc = len(env)
                env.extend(normalise_contraction(sh.l, sh.exps, sh.coeffs).ravel().tolist())
                entries.append((sh.l, len(sh.exps), sh.coeffs.shape[0], pe, pc))
            cache[sym] = entries
        for l, nprim, nctr, pe, pc in cache[sym]:
            bas.append([ia, l, nprim, nctr, 0, pe, pc, 0])
            nao += (2 * l + 1) * nctr
    return Molecule(list(symbols), np.asarray(coords_bohr, dtype=float),
                    np.asarray(atm, dtype=np.int32), np.asarray(bas, dtype=np.int32),
                    np.asarray(env, dtype=np.float64), nao)


# --------------------------------------------------------------------------
# grid
# --------------------------------------------------------------------------
# (radial points, Lebedev degree) per element and level; degree 17 -> 110,
# 19 -> 146, 23 -> 194 angular points.
GRID_LEVELS = {
    2: {"O": (60, 19), "H": (50, 17)},
    3: {"O": (70, 23), "H": (45, 23)},
    0: {"O": (20, 11), "H": (15, 9)},
    1: {"O": (40, 15), "H": (30, 13)},
}
RADIAL_XI = {"H": 0.8, "O": 0.9}          # bohr; radial map scale
_LEBEDEV_CACHE: dict = {}


def _lebedev(degree: int):
    if degree not in _LEBEDEV_CACHE:
        from scipy.integrate import lebedev_rule
        x, w = lebedev_rule(degree)
        _LEBEDEV_CACHE[degree] = (x.T.copy(), w / w.sum() * 4.0 * pi)
    return _LEBEDEV_CACHE[degree]


def _radial(n: int, xi: float):
    """Gauss-Chebyshev (second kind) nodes mapped by the Treutler-Ahlrichs M4
    map r = xi/ln2 (1+x)^0.6 ln(2/(1-x)); weights include r^2 dr/dx."""
    i = np.arange(1, n + 1)
    x = np.cos(i * pi / (n + 1))
    w_cheb = pi / (n + 1) * np.sin(i * pi / (n + 1)) ** 2 / np.sqrt(1 - x ** 2)
    c = xi / np.log(2.0)
    r = c * (1 + x) ** 0.6 * np.log(2 / (1 - x))
    drdx = c * (0.6 * (1 + x) ** -0.4 * np.log(2 / (1 - x)) + (1 + x) ** 0.6 / (1 - x))
    return r, w_cheb * r ** 2 * drdx


def becke_grid(symbols, coords, level=3, neighbours=8, chunk=32768,
               zero_below=1e-14):
    """Atom-centred grid; returns (coords[Ng,3], weights[Ng]) in bohr.

    Becke cell functions (three iterations of p(mu) = 1.5 mu - 0.5 mu^3) are
    evaluated against the ``neighbours`` nearest nuclei of each point; weights
    whose magnitude falls below ``zero_below`` are set to exactly zero and the
    point is kept (the selection code skips zero-weight points).
    """
    from scipy.spatial import cKDTree
    coords = np.asarray(coords, dtype=float)
    natm = len(symbols)
    pts, wts, owner = [], [], []
    for a, sym in enumerate(symbols):
        nrad, deg = GRID_LEVELS[level][sym]
        r, wr = _radial(nrad, RADIAL_XI[sym])
        ang, wa = _lebedev(deg)
        p = (r[:, None, None] * ang[None, :, :]).reshape(-1, 3) + coords[a]
        pts.append(p)
        wts.append((wr[:, None] * wa[None, :]).ravel())
        owner.append(np.full(len(p), a, dtype=np.int64))
    pts = np.concatenate(pts)
    wts = np.concatenate(wts)
    owner = np.concatenate(owner)
    k = min(neighbours, natm)
    tree = cKDTree(coords)
    rab = np.linalg.norm(coords[:, None] - coords[None], axis=-1)
    out = np.empty_like(wts)

    def partition(s):
        p = pts[s:s + chunk]
        own = owner[s:s + chunk]
        _, nb = tree.query(p, k=k)
        nb = nb.reshape(len(p), k)
        # make sure the owning atom is among the partition atoms
        has = (nb == own[:, None]).any(axis=1)
        nb[~has, -1] = own[~has]
        d = np.linalg.norm(p[:, None, :] - coords[nb], axis=-1)        # [b,k]
        mu = (d[:, :, None] - d[:, None, :]) / np.maximum(
            rab[nb[:, :, None], nb[:, None, :]], 1e-12)
        f = mu
        for _ in range(3):
            f = 1.5 * f - 0.5 * f ** 3
        s_ab = 0.5 * (1 - f)
        idx = np.arange(k)
        s_ab[:, idx, idx] = 1.0
        cell = s_ab.prod(axis=2)                                         # [b,k]
        mine = cell[nb == own[:, None]].reshape(len(p))
        out[s:s + chunk] = wts[s:s + chunk] * mine / cell.sum(axis=1)

    import concurrent.futures as cf
    import os
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        list(ex.map(partition, range(0, len(pts), chunk)))
    out[np.abs(out) < zero_below] = 0.0
    return pts, out


# --------------------------------------------------------------------------
# configurations (the five water-cluster workloads)
# --------------------------------------------------------------------------
CONFIGS = {
    "c1": dict(name="(H2O)4", lattice=(2, 2, 1), seed=0, level=2, axes="ao",
               algorithm="qrcp_dense", rank=8),
    "c2": dict(name="(H2O)16", lattice=(4, 2, 2), seed=1, level=3,
               axes="ao:1,dx:0.5,dy:0.5,dz:0.5", algorithm="rand_sketch", rank=8,
               oversampling=4, sketch_seed=2, online_batch=65536),
    "c2o": dict(name="(H2O)16", lattice=(4, 2, 2), seed=1, level=3,
                axes="ao:1,dx:0.5,dy:0.5,dz:0.5", algorithm="qrcp_online", rank=8,
                online_batch=65536),
    "c3": dict(name="(H2O)32", lattice=(4, 4, 2), seed=3, level=3, axes="ao",
               algorithm="rand_sketch", rank=10, oversampling=16, sketch_seed=7),
    "c4": dict(name="(H2O)8", lattice=(2, 2, 2), seed=4, level=3, axes="ao",
               algorithm="qrcp_dense", rank=8, electrons=80),
    "c5": dict(name="(H2O)64", lattice=(4, 4, 4), seed=5, level=3,
               axes="ao,dx,dy,dz", algorithm="rand_sketch", rank=10,
               oversampling=16, sketch_seed=7, electrons=640),
}


def parse_axes(spec: str):
    """'ao:1,dx:0.5' -> (['ao','dx'], [1.0, 0.5]) as in ``python/isdf.py:938-951``."""
    names, factors = [], []
    for entry in spec.split(","):
        fields = entry.strip().lower().split(":")
        if len(fields) > 2 or fields[0] not in ("ao", "dx", "dy", "dz", "occ"):
            raise ValueError(f"invalid --axes entry: {entry!r}")
        factor = float(fields[1]) if len(fields) == 2 else 1.0
        if not np.isfinite(factor) or factor <= 0:
            raise ValueError(f"--axes factor must be finite and positive: {entry!r}")
        names.append(fields[0])
        factors.append(factor)
    return names, factors


def make_config(key: str, level=None):
    """Return (Molecule, grid_coords, grid_weights, config dict)."""
    cfg = dict(CONFIGS[key])
    if level is not None:
        cfg["level"] = level
    symbols, xyz = water_cluster(cfg["lattice"], seed=cfg["seed"])
    mol = build_tables(symbols, xyz)
    pts, w = becke_grid(symbols, xyz, level=cfg["level"])
    mol.meta.update(cfg)
    return mol, pts, w, cfg


def random_density(mol: Molecule, overlap: np.ndarray, electrons: float, seed: int):
    """Seeded symmetric PSD density matrix scaled so that tr(D S) = electrons."""
    rng = np.random.default_rng(seed)
    nao = mol.nao
    nocc = max(1, int(round(electrons / 2)))
    c = rng.normal(size=(nao, min(nocc, nao)))
    d = c @ c.T
    d *= electrons / np.trace(d @ overlap)
    return d
