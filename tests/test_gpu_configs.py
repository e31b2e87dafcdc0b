"""The named validation workloads at their full sizes, on the GPU.

- plain 256³: mixed and FP64 reach the 1e-8 FP64 true relative residual;
  each pressure is compared with an FP64 solve to 1e-12;
- VoF 192³, 1000:1, seeded sphere (radius 0.25, 1.5-cell interface): same;
- IBM 256³, 200 seeded spheres (radii 4-12 cells): same, and the solid cells
  keep p = 0;
- differentiable projection at 128³, 100:1, eight unrolled steps (a seeded
  sphere per step): the mixed-precision adjoint gradient against FP64
  central differences on 16 seeded directions and against the FP64 adjoint
  gradient, both within 1e-6 relative.

Pressure errors are relative 2-norms over the fluid cells after removing the
fluid mean (the pure-Neumann null space).  The bound for a solve stopped at
relative residual 1e-8 is 1e-6: the error is at most the residual times the
condition of the low modes, which these grids keep below 1e2.
"""
import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid, SMACStep, ibm_solid_fraction_device

pytestmark = pytest.mark.gpu

ERR_BOUND = 1e-6


def _fluid_err(p, p_ref, fluid):
    a = p[fluid] - p[fluid].mean()
    b = p_ref[fluid] - p_ref[fluid].mean()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _solve(case, g, precision, tol):
    s = B200PressureSolver(case.N, case.h, precision=precision, tol=tol)
    step = SMACStep(g, case.dt)
    step.pressure_solver_ = s
    g.p_delta_.zero_()
    st = step.solve_poisson()
    torch.cuda.synchronize()
    p = g.p_delta_[1:-1, 1:-1, 1:-1].clone()
    s.close()
    return p, st


def _check_case(case):
    g = DeviceGrid.from_case(case)
    fluid = torch.from_numpy(W.interior(case.ct) == W.C_INTERIOR).cuda()
    p_ref, st_ref = _solve(case, g, nat.PRECISION_FP64, 1e-12)
    assert st_ref["rel_residual"] <= 1e-12
    out = {}
    for name, prec in (("fp64", nat.PRECISION_FP64), ("mixed", nat.PRECISION_MIXED)):
        p, st = _solve(case, g, prec, 1e-8)
        assert st["rel_residual"] <= 1e-8, (name, st)
        err = _fluid_err(p, p_ref, fluid)
        print(f"{case.name} {name}: {st['iterations']} iterations, rel residual {st['rel_residual']:.2e}, "
              f"error vs FP64 1e-12 solve {err:.2e}")
        assert err <= ERR_BOUND, (name, err)
        out[name] = (p, st, err)
    return g, p_ref, out


def test_plain_256_mixed_and_fp64_against_tight_fp64():
    _check_case(W.plain_case(256, seed=2))


def test_vof_192_ratio_1000_mixed_and_fp64_against_tight_fp64():
    _check_case(W.vof_case(192, seed=3, ratio=1000.0))


def test_ibm_256_200_spheres_mixed_and_fp64_against_tight_fp64():
    case = W.ibm_case(256, seed=4, nsph=200,
                      solid_fraction=lambda N, h, o, s: ibm_solid_fraction_device(N, h, o, s).cpu().numpy())
    g, p_ref, out = _check_case(case)
    solid = torch.from_numpy(W.interior(case.ct) == W.C_SOLID).cuda()
    assert int(solid.sum()) > 0
    for name, (p, _, _) in out.items():
        assert float(p[solid].abs().max()) == 0.0, name


def test_adjoint_128_eight_steps_mixed_against_fd_and_fp64_gradient():
    from mydemcfd_b200.autograd import StepOperator, project, unrolled
    n, steps = 128, 8
    base = W.vof_case(n, seed=3, ratio=100.0)
    ct, fxt, fyt, fzt = (torch.from_numpy(a).cuda() for a in (base.ct, base.fxt, base.fyt, base.fzt))
    ops = [StepOperator(torch.from_numpy(W.vof_case(n, seed=3 + k, ratio=100.0).meta["alpha"]).cuda(), 1.0, 100.0,
                        ct, fxt, fyt, fzt) for k in range(steps)]
    sh = W.shapes(base.N)
    rand = lambda seed: [torch.from_numpy(W.uniform_pm1(seed + i, int(np.prod(sh[k]))).reshape(sh[k])).cuda()
                         for i, k in enumerate("xyz")]
    s64 = B200PressureSolver(base.N, base.h, precision=nat.PRECISION_FP64, tol=1e-11)
    smx = B200PressureSolver(base.N, base.h, precision=nat.PRECISION_MIXED, tol=1e-10)
    u0 = rand(400)
    with torch.no_grad():  # an independent divergence-free target
        tgt = [t.clone() for t in project(rand(500), s64, ops[0])]

    def loss(u, s):
        out = unrolled(u, s, ops)
        return sum(((a - b) ** 2).sum() for a, b in zip(out, tgt))

    def grad(s):
        u = [t.clone().requires_grad_(True) for t in u0]
        checkpoints = []
        out = u
        for op in ops:
            out = project(out, s, op, 1.0, checkpoints)
        L = sum(((a - b) ** 2).sum() for a, b in zip(out, tgt))
        L.backward()
        assert len(checkpoints) == steps
        return [t.grad for t in u]

    g_mixed = grad(smx)
    g_fp64 = grad(s64)
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(g_mixed, g_fp64)) ** 0.5
    den = sum(float((b ** 2).sum()) for b in g_fp64) ** 0.5
    print(f"adjoint 128^3 x {steps}: mixed vs FP64 gradient {num / den:.2e}")
    assert num / den <= 1e-6
    # The unrolled projections are linear in u and the loss is quadratic, so
    # a central difference is exact for any step; 1e-3 of |u| keeps the solve
    # tolerance's share of the difference far below the 1e-6 check.
    worst = 0.0
    for d in range(16):
        dirs = rand(600 + 10 * d)
        eps = 1e-3 * float(torch.sqrt(sum((t ** 2).sum() for t in u0)) / torch.sqrt(sum((t ** 2).sum() for t in dirs)))
        with torch.no_grad():
            lp = loss([a + eps * b for a, b in zip(u0, dirs)], s64)
            lm = loss([a - eps * b for a, b in zip(u0, dirs)], s64)
        fd = float(lp - lm) / (2 * eps)
        an = sum(float((gg * dd).sum()) for gg, dd in zip(g_mixed, dirs))
        rel = abs(fd - an) / max(abs(fd), 1e-30)
        worst = max(worst, rel)
        assert rel <= 1e-6, (d, fd, an)
    print(f"adjoint 128^3 x {steps}: worst of 16 central differences {worst:.2e}")
    s64.close()
    smx.close()
