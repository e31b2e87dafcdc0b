"""This build against the reference's own GPU pressure solve, on one B200.

The reference's solve_poisson (RHS, GMG-preconditioned PCG) is built from its
sources (oracle/_ref, test infrastructure).  Both run the 256³ plain input to
a 1e-8 true relative residual:
- the reference stops on its own rule, max|r|·dt < tol checked every 5
  iterations, so its tol is lowered until its output meets 1e-8 (measured
  with this library's operator, which matches the reference's to 1e-13);
- this library is called the way the reference's driver calls its solver
  (coefficients, RHS, solve: G_PressureSolverBase::solve).
Both are timed with CUDA events around the call, host waits included (the
reference copies its residual to the host every 5 iterations; this library
reads its convergence flag once per two iterations).
"""
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid, SMACStep

from oracle import ref as REF

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")]


def _rel_residual(s, p_delta, rhs, fluid):
    """||b - A x|| / ||b|| over the fluid cells, b and r with their fluid means removed."""
    x = torch.from_numpy(p_delta).cuda()
    y = torch.zeros_like(x)
    s.apply_A(x, y)
    torch.cuda.synchronize()
    b = torch.from_numpy(rhs).cuda()[1:-1, 1:-1, 1:-1][fluid]
    ax = y[1:-1, 1:-1, 1:-1][fluid]
    b = b - b.mean()
    r = b - ax
    r = r - r.mean()
    return float(torch.linalg.norm(r) / torch.linalg.norm(b))


def _time(fn, reps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        e0.record()
        st = fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best, st


def test_faster_than_reference_gpu_solve_256():
    case = W.plain_case(256, seed=2)
    g = DeviceGrid.from_case(case)
    fluid = torch.from_numpy(W.interior(case.ct) == W.C_INTERIOR).cuda()
    probe = B200PressureSolver(case.N, case.h, precision=nat.PRECISION_FP64, tol=1e-8)
    probe.set_coefficients(g)

    # the reference, at the loosest of its tolerances that reaches 1e-8
    tol, ref = 1e-2, None
    for _ in range(12):
        out = REF.solve(case, solver_type=nat.PURENEUMANN_GMG_PCG, tol=tol, levels=6, do_correct=False)
        rel = _rel_residual(probe, out["p_delta"], out["rhs"], fluid)
        if rel <= 1e-8:
            ref = (tol, out, rel)
            break
        tol *= 0.25
    assert ref is not None
    tol, out, rel = ref
    ref_ms = min([out["solve_ms"]] + [REF.solve(case, solver_type=nat.PURENEUMANN_GMG_PCG, tol=tol, levels=6,
                                                do_correct=False)["solve_ms"] for _ in range(2)])

    res = {}
    for name, prec in (("fp64", nat.PRECISION_FP64), ("mixed", nat.PRECISION_MIXED)):
        s = B200PressureSolver(case.N, case.h, precision=prec, tol=1e-8)
        step = SMACStep(g, case.dt)
        step.pressure_solver_ = s
        ms, st = _time(step.solve_poisson, 5)
        mine = _rel_residual(probe, g.p_delta_.cpu().numpy(), g.rhs_.cpu().numpy(), fluid)
        assert mine <= 1e-8, (name, mine)
        res[name] = (ms, st["iterations"], mine)
        s.close()
    probe.close()
    print(f"reference GPU solve 256^3: tol {tol:.3g} (max|r|*dt), {out['iterations']} iterations, "
          f"rel residual {rel:.2e}, {ref_ms:.2f} ms")
    for name, (ms, it, mine) in res.items():
        print(f"this library {name}: {it} iterations, rel residual {mine:.2e}, {ms:.2f} ms, "
              f"{ref_ms / ms:.1f}x the reference")
    assert res["fp64"][0] < ref_ms
    assert res["mixed"][0] < ref_ms
