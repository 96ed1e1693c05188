import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "mp_isdf_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: larger CPU-only cases")


def three_s_shells():
    """Three unit-coefficient s shells on different atoms: the hand-built
    libcint tables of the reference's selector tests
    (python/test/test_online_anchor_select.py:19-30)."""
    atm = np.zeros((3, 6), dtype=np.int32)
    atm[:, 1] = [20, 23, 26]
    bas = np.zeros((3, 8), dtype=np.int32)
    bas[:, 0] = [0, 1, 2]
    bas[:, 2:4] = 1
    bas[:, 5] = [29, 31, 33]
    bas[:, 6] = [30, 32, 34]
    env = np.zeros(35)
    env[20:29] = [0, 0, 0, 0, 0, 1.0, 0, 1.0, 0]
    env[29:35] = [0.8, 1, 1.1, 1, 1.3, 1]
    return atm, bas, env


@pytest.fixture(scope="session")
def s_shells():
    return three_s_shells()


@pytest.fixture(scope="session")
def small_water():
    """(H2O)2 with the synthetic cc-pVDZ-shaped basis (48 AOs) and a
    level-0 grid: small enough for explicit pair matrices on the CPU."""
    from mp_isdf_b200 import inputs
    symbols, xyz = inputs.water_cluster((2, 1, 1), seed=11)
    mol = inputs.build_tables(symbols, xyz)
    pts, w = inputs.becke_grid(symbols, xyz, level=0)
    return mol, pts, w
