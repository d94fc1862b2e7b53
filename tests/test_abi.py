"""CPU tests of the C ABI: the library loads, exports every entry point that
include/ljcell.h declares, and its host-only functions behave."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ljcell.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^LJ_API\s+[\w\s\*]+?\b(lj_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("lj_create", "lj_bin", "lj_exclusive_scan", "lj_compute", "lj_compute_compat", "lj_simulate_host"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import ljcell

    out = subprocess.run(["nm", "-D", "--defined-only", ljcell.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s(lj_\w+)$", out, flags=re.M))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    lib = C.CDLL(ljcell.LIB_PATH)
    for s in declared_symbols():
        assert getattr(lib, s) is not None
    assert set(ljcell.ABI_SYMBOLS) == set(declared_symbols())


def test_checked_build_exports_the_same_symbols():
    """The bounds-checked debug build (-DLJ_CHECKS, libljcell_checks.so) is the same ABI."""
    import ljcell

    path = os.path.join(os.path.dirname(ljcell.LIB_PATH), "libljcell_checks.so")
    assert os.path.exists(path), "make builds libljcell_checks.so beside libljcell.so"
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(lj_\w+)$", out, flags=re.M))
    assert set(declared_symbols()) <= exported


def test_abi_version_and_status_strings():
    import ljcell

    assert ljcell.lib().lj_abi_version() == 1
    assert ljcell.status_str(ljcell.LJ_OK) == "ok"
    assert "timed out" in ljcell.status_str(ljcell.LJ_ETIMEOUT)
    assert "LJ_CHECKS" in ljcell.status_str(ljcell.LJ_ECHECK)


def test_grid_from_box_matches_oracle():
    import ljcell
    import ljoracle as O

    for lo, hi, rc in [((0, 0, 0), (1, 1, 1), 0.01), ((-0.5,) * 3, (1.5,) * 3, 0.005), ((0, 0, 0), (1, 2, 3), 0.03)]:
        g = ljcell.grid_from_box(lo, hi, rc)
        og = O.grid_from_box(lo, hi, rc)
        assert tuple(g.dim) == tuple(og.dim)
        assert g.width == og.width and tuple(g.origin) == tuple(og.origin)


def test_grid_compat_is_reference_formula():
    import ljcell

    g = ljcell.grid_compat(1.0, 1.0 / 32)
    assert tuple(g.dim) == (int(np.float32(1.0) / np.float32(1.0 / 32)),) * 3
    assert tuple(g.origin) == (0.0, 0.0, 0.0)


def test_bad_arguments_are_errors_not_crashes():
    import ljcell

    lib = ljcell.lib()
    g = ljcell.Grid()
    f3 = (C.c_float * 3)(0, 0, 0)
    assert lib.lj_grid_from_box(f3, f3, 0.1, C.byref(g)) == ljcell.LJ_EINVAL       # empty box
    hi = (C.c_float * 3)(1, 1, 1)
    assert lib.lj_grid_from_box(f3, hi, -1.0, C.byref(g)) == ljcell.LJ_EINVAL      # negative cutoff
    assert lib.lj_create(None, 0, None) == ljcell.LJ_EINVAL
    assert lib.lj_bin(None, None, 0, None, None, None, 1, 0, None, None, None, None, None, None) == ljcell.LJ_EINVAL
    assert lib.lj_compute(None, None, None, 0, None, None, None, 0, None, None, None) == ljcell.LJ_EINVAL
    assert lib.lj_sync(None) == ljcell.LJ_EINVAL


def test_create_without_gpu_reports_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import ljcell

    h = C.c_void_p()
    assert ljcell.lib().lj_create(C.byref(h), 0, None) in (ljcell.LJ_ECUDA, ljcell.LJ_EINVAL)
