"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/nrgpu.h, and its pure-host parameter default agrees with
the Python mirror."""
import ctypes as C
import os
import re

import pytest

from baum_b200 import abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "nrgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nrgpu_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return abi.lib()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(lib):
    assert lib.nrgpu_abi_version() == 1


def test_params_default_matches_python_mirror(lib):
    a = abi.BssnParams()
    lib.nrgpu_bssn_params_default(C.byref(a))
    b = abi.bssn_params()
    for name, _ in abi.BssnParams._fields_:
        va, vb = getattr(a, name), getattr(b, name)
        if hasattr(va, "__len__"):
            assert list(va) == pytest.approx(list(vb)), name
        else:
            assert va == pytest.approx(vb), name


def test_level_create_rejects_bad_descriptions(lib):
    """Host-side validation runs before any device call."""
    h = C.c_void_p()
    assert lib.nrgpu_level_create(None, C.byref(h)) == -1
    lev = abi.Level.single_box(6, 0.5)
    lev.desc.npoints = lev.npoints + 1
    assert lib.nrgpu_level_create(C.byref(lev.desc), C.byref(h)) == -1
    assert b"npoints" in lib.nrgpu_last_error()


def test_symmetry_flags_are_refused(lib):
    import numpy as np
    lev = abi.Level.single_box(6, 0.5)
    b = lev.boundary.copy()
    b[0] = 3  # SYMBOUND
    lev2 = abi.Level([(6, 6, 6, lev.boxes[0].x0, lev.boxes[0].y0, lev.boxes[0].z0)], 0.5, b)
    h = C.c_void_p()
    assert lib.nrgpu_level_create(C.byref(lev2.desc), C.byref(h)) == -5
