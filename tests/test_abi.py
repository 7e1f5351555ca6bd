"""The C-ABI library loads, exports every symbol include/ppm.h declares, and
reports errors as status codes (no GPU needed)."""
import ctypes
import os
import re

import numpy as np

from gpu_ppm_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "ppm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ppm_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    L = _abi.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_abi.SIGNATURES), "ctypes mirror out of sync with include/ppm.h"
    assert L.missing_symbols == []


def test_version_and_error_strings():
    L = _abi.lib()
    assert b"sm_100a" in L.ppm_version()
    rc = L.ppm_write_counts(None, 1, 1, None, 10)
    assert rc == _abi.PPM_E_INVALID
    assert b"bad argument" in L.ppm_last_error_string()


def test_null_engine_is_an_error():
    L = _abi.lib()
    p = _abi.Params()
    assert L.ppm_profile(None, ctypes.byref(p), None, None, None) == _abi.PPM_E_INVALID


def test_write_counts_format(tmp_path):
    L = _abi.lib()
    c = np.arange(6, dtype=np.float64).reshape(2, 3) + 0.5
    path = tmp_path / "x_counts_gpu.txt"
    assert L.ppm_write_counts(str(path).encode(), 2, 3, _abi.dptr(c), 16) == 0
    lines = path.read_text().splitlines()
    assert len(lines) == 2
    assert np.allclose(np.array([list(map(float, ln.split())) for ln in lines]), c)
