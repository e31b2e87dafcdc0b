"""Queued projections with host buffers (smac_async_*) against smac_project.

Three projections of different inputs are submitted back to back, so that
the copies of one overlap the solves of the others and a staging slot is
reused; each one's outputs must equal, bit for bit, those of a synchronous
smac_project of the same input on device arrays (the solve is deterministic).
"""
import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import AsyncProjector, B200PressureSolver, DeviceGrid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [nat.PRECISION_FP64, nat.PRECISION_MIXED])
def test_async_projections_equal_synchronous(precision):
    case = W.vof_case(48, seed=11, ratio=100.0)
    g = DeviceGrid.from_case(case)
    sh = W.shapes(case.N)
    s = B200PressureSolver(case.N, case.h, precision=precision, tol=1e-10)
    s.set_coefficients(g)
    inputs = []
    for q in range(3):
        u = [torch.from_numpy(np.ascontiguousarray(a) * (1.0 + q)).pin_memory()
             for a in (case.vxs, case.vys, case.vzs)]
        inputs.append(u)
    # synchronous reference on device arrays
    expected = []
    for u in inputs:
        dev = [t.cuda() for t in u]
        out = [torch.zeros(sh[k], dtype=torch.float64, device="cuda") for k in "xyz"]
        pd = torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")
        st = s.project(*dev, case.dt, pd, *out)
        torch.cuda.synchronize()
        expected.append(([t.cpu() for t in out] + [pd.cpu()], st["iterations"]))
    # queued, host buffers
    proj = AsyncProjector(s)
    outs = [[torch.full(sh[k], np.nan, dtype=torch.float64).pin_memory() for k in ("x", "y", "z", "cell")]
            for _ in inputs]
    tickets = [proj.submit(*u, case.dt, o[3], o[0], o[1], o[2]) for u, o in zip(inputs, outs)]
    stats = [proj.wait(t) for t in tickets]
    proj.close()
    for (exp, it), o, st in zip(expected, outs, stats):
        assert st["iterations"] == it
        for a, b in zip(o, exp):
            assert torch.equal(a, b)
    s.close()


def test_async_wait_refuses_unknown_ticket():
    case = W.plain_case(16, seed=1)
    g = DeviceGrid.from_case(case)
    s = B200PressureSolver(case.N, case.h)
    s.set_coefficients(g)
    proj = AsyncProjector(s)
    with pytest.raises(nat.SmacError):
        proj.wait(5)
    proj.close()
    s.close()
