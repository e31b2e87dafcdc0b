"""CPU checks of the C-ABI library: it loads, exports every symbol that
include/smac_b200.h declares, and refuses bad arguments without a GPU."""
import ctypes
import os
import re

import pytest

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "smac_b200.h")).read()
    return sorted(set(re.findall(r"^(?:smac_status|const char\*|void)\s+(smac_\w+)\s*\(", txt, re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return nat.load()


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(nat.EXPORTS) == names


def test_default_options(lib):
    o = nat.default_options()
    assert o.solver_type == nat.PURENEUMANN_GMG_PCG
    assert o.precision == nat.PRECISION_FP64
    assert o.tol == 1e-8 and o.max_iter == 2000 and o.nu1 == 2 and o.nu2 == 2


def test_null_arguments_are_refused(lib):
    assert lib.smac_create(None, None, None, None) == nat.BAD_ARG
    assert "null" in nat.last_error()
    assert lib.smac_solve(None, None, None) == nat.BAD_ARG
    assert lib.smac_destroy(None) == nat.OK
    assert lib.smac_async_create(None, None) == nat.BAD_ARG
    assert lib.smac_async_submit(None, None, None, None, 1.0, None, None, None, None, None) == nat.BAD_ARG
    assert lib.smac_async_wait(None, 0, None) == nat.BAD_ARG
    lib.smac_async_destroy(None)


def test_bad_options_are_refused(lib):
    d = nat.GridDesc(16, 16, 16, 1 / 16, 1 / 16, 1 / 16)
    h = ctypes.c_void_p()
    for bad in (dict(tol=0.0), dict(solver_type=9), dict(nu1=0), dict(max_iter=0), dict(reliable_delta=1.5)):
        o = nat.default_options(**bad)
        assert lib.smac_create(ctypes.byref(d), ctypes.byref(o), None, ctypes.byref(h)) == nat.BAD_ARG
    bad = nat.GridDesc(1, 16, 16, 1.0, 1.0, 1.0)
    assert lib.smac_create(ctypes.byref(bad), None, None, ctypes.byref(h)) == nat.BAD_SHAPE


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="needs a machine without a GPU")
def test_no_device_is_reported(lib):
    d = nat.GridDesc(16, 16, 16, 1 / 16, 1 / 16, 1 / 16)
    h = ctypes.c_void_p()
    rc = lib.smac_create(ctypes.byref(d), None, None, ctypes.byref(h))
    assert rc == nat.NO_DEVICE
    assert h.value is None
