"""The drop-in driver python/isdf.py run as a program (its CLI,
python/isdf.py:825-1004 of the reference): every anchor algorithm of this
package, the axes parser, the pair-space error, the grid metric and the JSON
record; refusals for what is outside its scope."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu


def _run(args, tmp_path, ok=True):
    out = tmp_path / "rec.json"
    cmd = [sys.executable, str(ROOT / "python" / "isdf.py"), "--molecule", "water:1x1x1:3", "--level", "0",
           *args, "--json", str(out)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if ok:
        assert p.returncode == 0, p.stdout + p.stderr
        return p.stdout, json.loads(out.read_text())
    assert p.returncode != 0
    return p.stdout + p.stderr, None


@pytest.mark.parametrize("algo,extra", [
    ("qrcp_dense", []),
    ("qrcp_online", ["--anchor-batch-size", "64"]),
    ("rand_sketch", ["--axes", "ao:1,dx:0.5,dy:0.5,dz:0.5", "--anchor-oversampling", "8"]),
    ("rand_sketch", ["--precision", "mixed", "--anchor-oversampling", "8"]),
    ("rbrp", ["--rbrp-block-size", "4"]),
    ("rbrp_id", ["--rbrp-block-size", "4"]),
])
def test_cli_algorithms(tmp_path, algo, extra):
    out, rec = _run(["--anchor-algorithm", algo, "--anchor-rank", "6", "--pair-space-error", *extra], tmp_path)
    assert "anchors: 6" in out
    assert "Pair-space scalar grid L2 error" in out
    assert len(rec["anchor_indices"]) == 6
    assert 0 <= rec["pair_space_errors"]["scalar"]["relative"] < 1.5
    if algo == "rbrp_id":
        assert rec["id_diagnostics"]["retained_rank"] == 6 and rec["fit_diagnostics"] is None


def test_cli_grid_metric(tmp_path):
    out, rec = _run(["--anchor-algorithm", "qrcp_dense", "--anchor-rank", "5", "--metric-algorithm", "grid"],
                    tmp_path)
    assert "Coulomb metric (grid): 5x5" in out


def test_cli_refusals(tmp_path):
    msg, _ = _run(["--anchor-algorithm", "cvt", "--anchor-rank", "4"], tmp_path, ok=False)
    assert "NotImplementedError" in msg
    msg, _ = _run(["--anchor-algorithm", "rand_sketch", "--sketch", "density", "--anchor-rank", "4"], tmp_path,
                  ok=False)
    assert "point_importance" in msg
    msg, _ = _run(["--anchor-algorithm", "qrcp_dense", "--sketch", "density"], tmp_path, ok=False)
    assert "--sketch requires" in msg
