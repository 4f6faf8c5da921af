"""The C-ABI library loads and exports every symbol include/rcpg.h declares;
compute entry points fail loudly (RCPG_ECUDA) without a GPU instead of
falling back to a CPU path."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (REPO / "include" / "rcpg.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rcpg_\w+)\s*\(", src)) - {"rcpg_observer_fn"})


def test_exports_every_declared_symbol(native):
    names = declared_functions()
    assert names, "no declarations parsed"
    assert set(names) == set(native.EXPORTED_SYMBOLS)
    lib = C.CDLL(str(native.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_abi(native):
    assert native.lib.rcpg_abi_version() == 3
    assert b"sm_100a" in native.lib.rcpg_version()


def test_no_cpu_fallback_without_gpu(native):
    if native.lib.rcpg_device_count() > 0:
        return  # only meaningful on a machine without a GPU
    import rcpgenerator_b200 as rb
    inp = {"positions": [[0.1, 0.1], [0.5, 0.5]], "diameters": [0.1, 0.1]}
    try:
        rb.run_packing(inp, {"box": [1.0, 1.0]})
    except native.NativeError as e:
        assert e.code == native.RCPG_ECUDA
        assert "no CUDA device" in str(e)
    else:
        raise AssertionError("run_packing succeeded without a GPU")


def test_scale_diameters_host(native):
    D = np.array([1.0, 1.4, 1.0, 1.4])
    out = np.zeros(4)
    dp = C.POINTER(C.c_double)
    box = np.array([1.0, 1.0])
    f = native.lib.rcpg_scale_diameters_nd(D.ctypes.data_as(dp), 4, 0.5, box.ctypes.data_as(dp), 2, 0,
                                           out.ctypes.data_as(dp))
    vol = (np.pi / 4 * out ** 2).sum()
    assert abs(vol - 0.5) < 1e-12
    assert np.allclose(out, D * f, rtol=0, atol=0)


def test_scale_diameters_host_large_is_the_sequential_result(native):
    """Above 65,536 particles the per-particle volumes are computed on several
    host threads; they are summed in index order, so the result equals the
    one-thread restatement bit for bit."""
    import math
    rng = np.random.default_rng(9)
    n, nd = 100_000, 3
    D = rng.uniform(0.5, 1.5, n)
    out = np.zeros(n)
    dp = C.POINTER(C.c_double)
    box = np.array([1.0, 1.3, 0.9])
    f = native.lib.rcpg_scale_diameters_nd(D.ctypes.data_as(dp), n, 0.33, box.ctypes.data_as(dp), nd, 0,
                                           out.ctypes.data_as(dp))
    c_pi, c_gamma = math.pow(math.pi, nd / 2.0), math.gamma(nd / 2.0 + 1.0)
    s = 0.0
    for d in D.tolist():
        s += c_pi * math.pow(d * 0.5, float(nd)) / c_gamma
    v_box = 1.0 * 1.3 * 0.9
    factor = math.pow(0.33 * v_box / s, 1.0 / nd)
    assert f == factor
    np.testing.assert_array_equal(out, D * factor)
