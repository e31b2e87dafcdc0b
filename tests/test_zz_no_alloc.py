"""The allocation-free operator entry point, smac_apply_A_dot_noalloc.

It exists for callers that cannot allocate device memory (a step loop being
recorded into a CUDA graph, or a host code whose pool allocator already owns
the device memory): it uses a static device array as its only scratch.  This
file is collected last, so a run that stops at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid, _ptr

pytestmark = pytest.mark.gpu


def _noalloc(case, g, x, y, xAx):
    d = nat.GridDesc(*case.N, *case.h)
    s = torch.cuda.current_stream().cuda_stream
    return nat.load().smac_apply_A_dot_noalloc(
        ctypes.byref(d), _ptr(g.f_bx_), _ptr(g.f_by_), _ptr(g.f_bz_), _ptr(g.celltype_), _ptr(g.f_xtype_),
        _ptr(g.f_ytype_), _ptr(g.f_ztype_), _ptr(x), _ptr(y), _ptr(xAx), ctypes.c_void_p(s))


@pytest.mark.parametrize("kind", ["vof", "ibm"])
def test_noalloc_matches_apply_A_twice(kind):
    if kind == "vof":
        case = W.vof_case(40, seed=21, ratio=1000.0)
    else:
        from _cases import oracle_solid_fraction
        case = W.ibm_case(48, seed=22, nsph=6, solid_fraction=oracle_solid_fraction, rmin_cells=3.0,
                          rmax_cells=6.0)
    g = DeviceGrid.from_case(case)
    solver = B200PressureSolver(case.N, case.h)
    solver.set_coefficients(g)
    sh = W.shapes(case.N)
    for call in range(2):  # two calls in a row share the static scratch
        x = torch.from_numpy(W.uniform_pm1(900 + call, int(np.prod(sh["cell"]))).reshape(sh["cell"])).cuda()
        y_ref = torch.zeros_like(x)
        solver.apply_A(x, y_ref)  # the existing entry point (handle-owned scratch)
        y = torch.zeros_like(x)
        xAx = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert _noalloc(case, g, x, y, xAx) == nat.OK, nat.last_error()
        torch.cuda.synchronize()
        yi, yri = W.interior(y.cpu().numpy()), W.interior(y_ref.cpu().numpy())
        scale = np.abs(yri).max()
        assert np.abs(yi - yri).max() <= 1e-13 * scale
        ref_dot = float((W.interior(x.cpu().numpy()) * yri).sum())
        assert abs(float(xAx.item()) - ref_dot) <= 1e-12 * abs(ref_dot)
        # ghost entries of y are not written
        assert float(y[0].abs().max()) == 0.0 and float(y[:, :, -1].abs().max()) == 0.0
    solver.close()


def test_noalloc_refuses_grids_beyond_its_scratch():
    d = nat.GridDesc(4096, 4096, 8, 1.0, 1.0, 1.0)
    dummy = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = nat.load().smac_apply_A_dot_noalloc(ctypes.byref(d), *([dummy] * 10), None)
    assert rc == nat.BAD_SHAPE
    assert "static scratch" in nat.last_error()
