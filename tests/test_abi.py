"""The C ABI library builds, loads and exports every entry point declared in include/amrclaw_b200.h."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "amrclaw_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(amrgpu_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "amrgpu_init" in syms and "amrgpu_level_advance" in syms and "amrgpu_destroy" in syms


def test_library_exports_all_declared_symbols():
    from amrclaw_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from amrclaw_b200 import _lib
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_init_reports_errors_without_crashing(tmp_path):
    from amrclaw_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.amrgpu_init(str(tmp_path).encode(), str(tmp_path).encode(), 0, ctypes.byref(h))
    assert rc != 0
    assert lib.amrgpu_last_error()
    assert lib.amrgpu_init(None, None, 0, ctypes.byref(h)) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_values_size_query_full_and_partial_buffers(tmp_path, dim):
    """amrgpu_values: a NULL buffer returns the count, a full buffer receives every value
    straight from the device, and a short one the first cap values, in both dimensions."""
    import numpy as np
    import configs
    from amrclaw_b200 import Solver, _lib
    rd = configs.euler_quadrants(n=32, levels=3, tfinal=0.05) if dim == 2 else \
        configs.euler_blast(n=16, levels=2, tfinal=0.05, seed=0)
    rd.write(str(tmp_path))
    with Solver(str(tmp_path)) as s:
        s.run(3)
        lib = _lib.load()
        n = ctypes.c_longlong()
        assert lib.amrgpu_values(s._h, None, 0, ctypes.byref(n)) == 0
        full = s.values()
        assert n.value == full.size > 0
        cap = n.value // 3
        part = np.full(cap, np.nan)
        m = ctypes.c_longlong()
        assert lib.amrgpu_values(s._h, part.ctypes.data_as(_lib.c_double_p), cap, ctypes.byref(m)) == 0
        assert m.value == n.value
        assert np.array_equal(part, full[:cap])
        again = s.values()
        assert np.array_equal(again, full)
