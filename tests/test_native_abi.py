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
    assert o.sweep_kernel == nat.SWEEP_AUTO and o.coarse_kernel == nat.COARSE_AUTO


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
    for bad in (dict(tol=0.0), dict(solver_type=9), dict(nu1=0), dict(max_iter=0), dict(reliable_delta=1.5),
                dict(sweep_kernel=4), dict(coarse_kernel=2)):
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


def test_step_call_arguments_are_checked_before_any_device_work(lib):
    """The property update, both predictors, the mass flux and the two-way
    coefficients refuse null and mis-shaped arguments before any CUDA call
    (so this runs without a GPU)."""
    import numpy as np
    fake = ctypes.c_void_p(256)  # never dereferenced
    d = nat.GridDesc(8, 8, 8, 0.125, 0.125, 0.125)
    flat = nat.GridDesc(8, 0, 8, 0.125, 0.125, 0.125)
    thin = nat.GridDesc(8, 1, 8, 0.125, 0.125, 0.125)
    neg = nat.GridDesc(8, 8, 8, 0.125, -0.125, 0.125)
    vp = nat.VofParams(1.0, 1000.0, 1e-3, 1e-1)
    out = nat.PropertyFields(*(256,) * 15)
    assert lib.smac_update_properties(ctypes.byref(d), ctypes.byref(vp), None, fake, fake, fake, fake,
                                      ctypes.byref(out), None) == nat.BAD_ARG
    assert lib.smac_update_properties(ctypes.byref(flat), ctypes.byref(vp), fake, fake, fake, fake, fake,
                                      ctypes.byref(out), None) == nat.BAD_SHAPE
    no_mu = nat.PropertyFields(*(256,) * 12, None, 256, 256)   # f_mux missing
    assert lib.smac_update_properties(ctypes.byref(d), ctypes.byref(vp), fake, fake, fake, fake, fake,
                                      ctypes.byref(no_mu), None) == nat.BAD_ARG
    optional = nat.PropertyFields(256, None, 256, 256, 256, 256, None, None, None, None, None, None, 256, 256, 256)
    assert lib.smac_update_properties(ctypes.byref(neg), ctypes.byref(vp), fake, fake, fake, fake, fake,
                                      ctypes.byref(optional), None) == nat.BAD_SHAPE

    types = np.zeros(1, np.uint8)
    vel = np.zeros(1)
    one = nat.BoundaryTable(1, types.ctypes.data, vel.ctypes.data, vel.ctypes.data, vel.ctypes.data)
    empty = nat.BoundaryTable(0, types.ctypes.data, vel.ctypes.data, vel.ctypes.data, vel.ctypes.data)
    mf = nat.MomentumFields(*(256,) * 30)
    tw = nat.TwoWayFields(*(256,) * 5)
    vs = (fake,) * 3
    assert lib.smac_predict_vstar(ctypes.byref(thin), ctypes.byref(one), ctypes.byref(mf), 0.01, 0.0, 0.0, -9.8,
                                  *vs, None) == nat.BAD_SHAPE
    assert lib.smac_predict_vstar(ctypes.byref(d), ctypes.byref(empty), ctypes.byref(mf), 0.01, 0.0, 0.0, -9.8,
                                  *vs, None) == nat.BAD_ARG
    assert lib.smac_predict_vstar_two_way(ctypes.byref(d), ctypes.byref(one), ctypes.byref(mf), None, 0.01, 0.0,
                                          0.0, -9.8, *vs, None) == nat.BAD_ARG
    no_eps = nat.TwoWayFields(256, None, 256, 256, 256)
    assert lib.smac_predict_vstar_two_way(ctypes.byref(d), ctypes.byref(one), ctypes.byref(mf), ctypes.byref(no_eps),
                                          0.01, 0.0, 0.0, -9.8, *vs, None) == nat.BAD_ARG
    # the two-way form reads f_inv_rho from tw, so mf's f_b may be null there, not in the one-way form
    mf_no_fb = nat.MomentumFields(*(256,) * 21, None, None, None, *(256,) * 6)
    assert lib.smac_predict_vstar(ctypes.byref(d), ctypes.byref(one), ctypes.byref(mf_no_fb), 0.01, 0.0, 0.0, -9.8,
                                  *vs, None) == nat.BAD_ARG
    assert lib.smac_predict_vstar_two_way(ctypes.byref(thin), ctypes.byref(one), ctypes.byref(mf_no_fb),
                                          ctypes.byref(tw), 0.01, 0.0, 0.0, -9.8, *vs, None) == nat.BAD_SHAPE

    ff = nat.MassFluxFields(*(256,) * 15)
    ff_no_F = nat.MassFluxFields(*(256,) * 12, None, 256, 256)
    mfo = (fake,) * 3
    assert lib.smac_mass_flux_from_alpha_flux(ctypes.byref(d), ctypes.byref(one), ctypes.byref(ff_no_F), 1.0, 1000.0,
                                              0.01, None, *mfo, None) == nat.BAD_ARG
    assert lib.smac_mass_flux_from_alpha_flux(ctypes.byref(flat), ctypes.byref(one), ctypes.byref(ff), 1.0, 1000.0,
                                              0.01, None, *mfo, None) == nat.BAD_SHAPE
    assert lib.smac_mass_flux_from_alpha_flux(ctypes.byref(d), ctypes.byref(empty), ctypes.byref(ff), 1.0, 1000.0,
                                              0.01, fake, *mfo, None) == nat.BAD_ARG

    assert lib.smac_poisson_beta_two_way(ctypes.byref(d), fake, fake, None, fake, fake, fake, fake, None) == nat.BAD_ARG
    assert lib.smac_poisson_beta_two_way(ctypes.byref(flat), fake, fake, fake, fake, fake, fake, fake,
                                         None) == nat.BAD_SHAPE


def test_predictor_and_mass_flux_refuse_grids_beyond_32_bit_offsets(lib):
    """The predictor, the mass flux and the property update index their
    arrays with 32-bit offsets: a grid with a face array of 2^31 entries or
    more is refused before any device work."""
    import numpy as np
    fake = ctypes.c_void_p(256)
    big = nat.GridDesc(1300, 1300, 1300, 1e-3, 1e-3, 1e-3)
    types = np.zeros(1, np.uint8)
    vel = np.zeros(1)
    one = nat.BoundaryTable(1, types.ctypes.data, vel.ctypes.data, vel.ctypes.data, vel.ctypes.data)
    mf = nat.MomentumFields(*(256,) * 30)
    assert lib.smac_predict_vstar(ctypes.byref(big), ctypes.byref(one), ctypes.byref(mf), 0.01, 0.0, 0.0, -9.8,
                                  fake, fake, fake, None) == nat.BAD_SHAPE
    assert "2^31" in nat.last_error()
    ff = nat.MassFluxFields(*(256,) * 15)
    assert lib.smac_mass_flux_from_alpha_flux(ctypes.byref(big), ctypes.byref(one), ctypes.byref(ff), 1.0, 1000.0,
                                              0.01, None, fake, fake, fake, None) == nat.BAD_SHAPE
    vp = nat.VofParams(1.0, 1000.0, 1e-3, 1e-1)
    out = nat.PropertyFields(*(256,) * 15)
    assert lib.smac_update_properties(ctypes.byref(big), ctypes.byref(vp), fake, fake, fake, fake, fake,
                                      ctypes.byref(out), None) == nat.BAD_SHAPE
