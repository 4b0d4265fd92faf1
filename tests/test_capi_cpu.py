"""C ABI checks that need no GPU: the library loads, exports every function
include/psc.h declares, and its host-side spline construction matches the
oracle (and hence the reference) bit for bit."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from parsec_python_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "psc.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(psc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.exported_symbols())
    assert lib.psc_version() == 1


def test_spline_coefficients_match_oracle_bitwise():
    tables = O.load_tables()
    lib = _lib.load()
    for el in ("H", "C", "O", "Si"):
        d = tables[el]
        for col in (d[:, 1], d[:, 2], d[:, 4], d[:, 5], d[:, 3] - d[:, 4]):
            x = np.ascontiguousarray(d[:, 0])
            y = np.ascontiguousarray(col)
            n = len(x)
            xk, z, c, dd = (np.zeros(n) for _ in range(4))
            nk = ctypes.c_int()
            p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
            assert lib.psc_spline_coeffs(n, p(x), p(y), ctypes.byref(nk), p(xk), p(z), p(c), p(dd)) == 0
            keep = O.prune_knots(y)
            s = O.Spline(x[keep], y[keep])
            m = nk.value
            assert m == len(keep)
            np.testing.assert_array_equal(xk[:m], x[keep])
            np.testing.assert_array_equal(z[:m], s.z)
            np.testing.assert_array_equal(c[:m - 1], s.c)
            np.testing.assert_array_equal(dd[:m - 1], s.d)


def test_invalid_arguments_are_rejected_with_a_message():
    lib = _lib.load()
    ptr = ctypes.c_void_p()
    assert lib.psc_ctx_create(0, 4, 4, 0.5, 8, ctypes.byref(ptr)) == 2
    assert b"grid dimensions" in lib.psc_last_error(None)
    assert lib.psc_ctx_create(4, 4, 4, -1.0, 8, ctypes.byref(ptr)) == 2


def test_gpu_entry_points_fail_loudly_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from parsec_python_b200 import gpu
    with pytest.raises(_lib.PscError):
        gpu.require_cuda()
