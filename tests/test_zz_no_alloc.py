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


def _oracle_y(case, x):
    """The reference's operator (k_build_vof_poisson_A + Ap) from the oracle."""
    from oracle import oracle as O
    from _cases import ref_grid
    return O.apply_A(case.N, O.build_A(ref_grid(case)), x)


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
        xh = W.uniform_pm1(900 + call, int(np.prod(sh["cell"]))).reshape(sh["cell"])
        x = torch.from_numpy(xh).cuda()
        y_ref = torch.zeros_like(x)
        solver.apply_A(x, y_ref)  # the existing entry point (handle-owned scratch)
        y = torch.zeros_like(x)
        xAx = torch.zeros(1, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        alloc0 = torch.cuda.memory_allocated()
        assert _noalloc(case, g, x, y, xAx) == nat.OK, nat.last_error()
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the library's module (and its static array)
            assert torch.cuda.mem_get_info()[0] == free0, "the call allocated device memory"
            assert torch.cuda.memory_allocated() == alloc0
        yi, yri = W.interior(y.cpu().numpy()), W.interior(y_ref.cpu().numpy())
        scale = np.abs(yri).max()
        assert np.abs(yi - yri).max() <= 1e-13 * scale
        # and against the oracle's restatement of the reference's operator
        y_o = W.interior(_oracle_y(case, xh))
        assert np.abs(yi - y_o).max() <= 1e-13 * np.abs(y_o).max()
        ref_dot = float((W.interior(xh) * y_o).sum())
        assert abs(float(xAx.item()) - ref_dot) <= 1e-12 * abs(ref_dot)
        # ghost entries of y are not written
        assert float(y[0].abs().max()) == 0.0 and float(y[:, :, -1].abs().max()) == 0.0
    solver.close()


def test_noalloc_recorded_in_a_cuda_graph():
    """The use the entry point exists for: one eager call (which may load the
    module), then the call recorded in a stream capture (its memset node and
    kernel) and replayed on new x."""
    case = W.vof_case(40, seed=23, ratio=1000.0)
    g = DeviceGrid.from_case(case)
    solver = B200PressureSolver(case.N, case.h)
    solver.set_coefficients(g)
    sh = W.shapes(case.N)
    n = int(np.prod(sh["cell"]))
    x = torch.from_numpy(W.uniform_pm1(930, n).reshape(sh["cell"])).cuda()
    y = torch.zeros_like(x)
    xAx = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _noalloc(case, g, x, y, xAx) == nat.OK, nat.last_error()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        rc = _noalloc(case, g, x, y, xAx)
    assert rc == nat.OK, nat.last_error()
    for rep in range(2):
        xh = W.uniform_pm1(931 + rep, n).reshape(sh["cell"])
        x.copy_(torch.from_numpy(xh))
        y.zero_()
        xAx.fill_(12345.0)
        graph.replay()
        y_ref = torch.zeros_like(x)
        solver.apply_A(x, y_ref)
        torch.cuda.synchronize()
        yi, yri = W.interior(y.cpu().numpy()), W.interior(y_ref.cpu().numpy())
        assert np.abs(yi - yri).max() <= 1e-13 * np.abs(yri).max()
        ref_dot = float((W.interior(xh) * yri).sum())
        assert abs(float(xAx.item()) - ref_dot) <= 1e-12 * abs(ref_dot)
    del graph
    solver.close()


def test_noalloc_at_the_scratch_limit():
    """32 x 32768 x 2 cells: ceil(32/32) * ceil(32768/4) = 8192 blocks, every
    partial-sum slot of the static array in use (one z-chunk)."""
    N = (32, 32768, 2)
    h = (1.0 / 32, 1.0 / 32768, 0.5)
    ct, fxt, fyt, fzt = W.box_types(N)
    sh = W.shapes(N)
    fb = [np.where(t == W.F_INTERIOR, 0.5 + 0.5 * W.uniform01(700 + i, t.size).reshape(t.shape), 0.0)
          for i, t in enumerate((fxt, fyt, fzt))]
    xh = W.uniform_pm1(711, int(np.prod(sh["cell"]))).reshape(sh["cell"])
    from oracle import oracle as O
    rg = O.RefGrid(N, h, 1.0, *(np.zeros(sh[k]) for k in "xyz"), np.ones(sh["cell"]), np.ones(sh["cell"]), *fb,
                   *(np.zeros(sh[k]) for k in "xyz"), *fb, ct, fxt, fyt, fzt)
    y_o = W.interior(O.apply_A(N, O.build_A(rg), xh))
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    x, y = dev(xh), torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")
    xAx = torch.zeros(1, dtype=torch.float64, device="cuda")
    d = nat.GridDesc(*N, *h)
    args = [dev(a) for a in (*fb, ct, fxt, fyt, fzt)]
    for _ in range(2):
        y.zero_()
        rc = nat.load().smac_apply_A_dot_noalloc(ctypes.byref(d), *(_ptr(a) for a in args), _ptr(x), _ptr(y),
                                                 _ptr(xAx), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == nat.OK, nat.last_error()
        torch.cuda.synchronize()
        yi = W.interior(y.cpu().numpy())
        assert np.abs(yi - y_o).max() <= 1e-13 * np.abs(y_o).max()
        ref_dot = float((W.interior(xh) * y_o).sum())
        assert abs(float(xAx.item()) - ref_dot) <= 1e-12 * abs(ref_dot)


@pytest.mark.parametrize("nx,ny", [(4096, 4096), (32, 32769), (33, 32768)])
def test_noalloc_refuses_grids_beyond_its_scratch(nx, ny):
    """8193 blocks or more are refused before any pointer is touched."""
    d = nat.GridDesc(nx, ny, 2, 1.0, 1.0, 1.0)
    dummy = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = nat.load().smac_apply_A_dot_noalloc(ctypes.byref(d), *([dummy] * 10), None)
    assert rc == nat.BAD_SHAPE
    assert "static scratch" in nat.last_error()
