"""CPU-side checks of the C-ABI library and the drop-in module (no GPU compute)."""
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "isdf_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(isdf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    from mp_isdf_b200 import capi
    lib = ctypes.CDLL(str(capi.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(capi.SYMBOLS)


def test_status_strings_and_cuda_probe():
    from mp_isdf_b200 import capi
    L = capi.lib()
    assert L.isdf_status_string(0) == b"ok"
    assert L.isdf_status_string(1) == b"invalid argument"
    assert L.isdf_cuda_available() in (0, 1)


def test_dropin_module_surface():
    import mp_isdf
    assert mp_isdf.cuda_enabled is True
    for name in ("AtomicOrbital", "AtomicOrbitalGradX", "AtomicOrbitalGradY",
                 "AtomicOrbitalGradZ", "OccupiedOrbital"):
        assert hasattr(mp_isdf.AxisType, name)
    for name in ("QRColumnPivoting", "OnlineQRColumnPivoting", "RandomizedQuadratureKhatriRao",
                 "CentroidalVoronoi", "RandomizedAODensityKhatriRao",
                 "RandomizedAODensityNormalizedKhatriRao"):
        assert hasattr(mp_isdf.LocalAnchorSelectionAlgorithm, name)
    assert hasattr(mp_isdf.DistributedAnchorSelectionAlgorithm, "SVD")
    for name in ("LibcintContext", "AnchorSelection", "DistributedAnchorSelection",
                 "eval_ao", "eval_ao_gradient", "fit"):
        assert hasattr(mp_isdf, name)


def test_context_without_gpu_fails_loudly(s_shells):
    """No CPU fallback: without a CUDA device the context constructor raises."""
    from mp_isdf_b200 import capi
    if capi.lib().isdf_cuda_available():
        pytest.skip("a CUDA device is present")
    import mp_isdf
    with pytest.raises(RuntimeError):
        mp_isdf.LibcintContext(*s_shells)


def test_c2s_compile_time_table_matches_oracle_least_squares():
    """The product's compile-time solid-harmonic table (c2s_table.h, the
    coefficients the device AO code multiplies by) and the oracle's
    least-squares derivation agree; the header is compiled host-only."""
    import subprocess, tempfile
    from oracle import oracle as O
    hdr = ROOT / "mp_isdf_b200" / "csrc" / "c2s_table.h"
    snippet = (f'#include "{hdr}"\n#include <cstdio>\n'
               "int main(){for(int l=0;l<=6;++l)for(int s=0;s<2*l+1;++s)"
               "for(int c=0;c<(l+1)*(l+2)/2;++c)std::printf(\"%.17g\\n\", isdf::c2s_coef(l,s,c));}\n")
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "c2s.cpp"
        c.write_text(snippet)
        exe = Path(d) / "c2s"
        subprocess.check_call(["g++", "-O1", "-std=c++17", str(c), "-o", str(exe)])
        vals = np.array([float(x) for x in subprocess.check_output([str(exe)]).split()])
    ref = O.c2s_table(6)
    np.testing.assert_allclose(vals, ref, atol=1e-12)


def test_inputs_generator_shapes():
    from mp_isdf_b200 import inputs
    mol, pts, w, cfg = inputs.make_config("c1", level=0)
    assert mol.nao == 96 and len(mol.symbols) == 12
    assert pts.shape[1] == 3 and len(w) == len(pts)
    assert np.all(np.isfinite(w)) and np.any(w == 0)
    sym, xyz = inputs.water_cluster((4, 4, 4), seed=5)
    assert len(sym) == 192
    tables = inputs.build_tables(sym, xyz)
    assert tables.nao == 1536


@pytest.mark.parametrize("d,ell,seed", [(1, 1, 0), (7, 3, 11), (96, 12, 2), (6144, 26, 7), (12288, 41, 13)])
def test_sketch_factors_match_standard_library_streams(d, ell, seed):
    """U/V of rand_sketch (threaded polar-method draws) equal the oracle's
    std::normal_distribution streams bit for bit, odd counts included."""
    from mp_isdf_b200 import capi
    from oracle import oracle as O
    u, v = capi.sketch_factors(d, ell, seed)
    ou, ov = O.sketch_factors(d, ell, seed)
    assert np.array_equal(u, ou)
    assert np.array_equal(v, ov)


def test_sketch_factors_concurrent_calls():
    """The draw's process-wide worker pool serves one call at a time: calls
    from several host threads at once (different seeds and sizes) each return
    their own standard-library streams."""
    import threading
    from mp_isdf_b200 import capi
    from oracle import oracle as O
    cases = [(96, 12, 2), (384, 26, 5), (1536, 26, 9), (7, 3, 11)] * 2
    got = [None] * len(cases)

    def draw(i):
        got[i] = capi.sketch_factors(*cases[i])

    threads = [threading.Thread(target=draw, args=(i,)) for i in range(len(cases))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for (d, ell, seed), (u, v) in zip(cases, got):
        ou, ov = O.sketch_factors(d, ell, seed)
        assert np.array_equal(u, ou) and np.array_equal(v, ov)


def test_pair_error_terms_reject_null_arrays_without_gpu():
    """Both pair-error reductions reject null device arrays with
    ISDF_ERR_INVALID before any CUDA call (so this runs without a GPU)."""
    import ctypes
    from mp_isdf_b200 import capi
    L = capi.lib()
    out = np.zeros(2)
    P = ctypes.c_void_p
    dummy = np.zeros(16)
    d = P(dummy.ctypes.data)
    for fn in (L.isdf_pair_error_terms, L.isdf_pair_error_terms_noalloc):
        # null q / w with n > 0
        assert fn(10, 2, None, d, d, d, d, out.ctypes.data_as(P), None) == 1
        assert fn(10, 2, d, d, d, d, None, out.ctypes.data_as(P), None) == 1
        # null H / X / M with n > 0 and k > 0
        assert fn(10, 2, d, None, d, d, d, out.ctypes.data_as(P), None) == 1
        assert fn(10, 2, d, d, None, d, d, out.ctypes.data_as(P), None) == 1
        assert fn(10, 2, d, d, d, None, d, out.ctypes.data_as(P), None) == 1
        # null output
        assert fn(10, 2, d, d, d, d, d, None, None) == 1
