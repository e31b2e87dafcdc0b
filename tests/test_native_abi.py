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
    return sorted(set(re.findall(r"^(?:smac_status|const char\*|void|size_t)\s+(smac_\w+)\s*\(", txt, re.M)))


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


def test_post_pass_arguments_are_checked_before_any_device_work(lib):
    fake = ctypes.c_void_p(256)  # never dereferenced: every call below fails its argument checks
    d = nat.GridDesc(8, 8, 8, 0.125, 0.125, 0.125)
    assert lib.smac_update_pressure_ghost(ctypes.byref(d), None, None, 0.0, 0.0, -9.8, fake, None) == nat.BAD_ARG
    flat = nat.GridDesc(8, 0, 8, 0.125, 0.125, 0.125)
    assert lib.smac_update_pressure_ghost(ctypes.byref(flat), fake, None, 0.0, 0.0, -9.8, fake, None) == nat.BAD_SHAPE
    assert lib.smac_face_gradp(ctypes.byref(flat), fake, fake, fake, fake, None) == nat.BAD_SHAPE
    assert lib.smac_face_gradp(ctypes.byref(d), fake, None, fake, fake, None) == nat.BAD_ARG
    import numpy as np
    types = np.zeros(1, np.uint8)
    vel = np.zeros(1)
    empty = nat.BoundaryTable(0, types.ctypes.data, vel.ctypes.data, vel.ctypes.data, vel.ctypes.data)
    args = (fake,) * 3 + (None,) * 3 + (None,) * 3 + (None,) * 6 + (None, 1.0) + (fake,) * 3 + (None,)
    assert lib.smac_update_velocity_ghost(ctypes.byref(d), ctypes.byref(empty), *args) == nat.BAD_ARG
    one = nat.BoundaryTable(1, types.ctypes.data, vel.ctypes.data, vel.ctypes.data, vel.ctypes.data)
    thin = nat.GridDesc(8, 1, 8, 0.125, 0.125, 0.125)
    assert lib.smac_update_velocity_ghost(ctypes.byref(thin), ctypes.byref(one), *args) == nat.BAD_SHAPE
    # outlet marks without p_delta
    bad = (fake,) * 3 + (fake,) * 3 + (None,) * 3 + (fake,) * 6 + (None, 1.0) + (fake,) * 3 + (None,)
    assert lib.smac_update_velocity_ghost(ctypes.byref(d), ctypes.byref(one), *bad) == nat.BAD_ARG
