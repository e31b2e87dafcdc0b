"""Differentiable SMAC projection over the C ABI.

Forward: u = P(u*) = u* + B G A^+ D u* on F_INTERIOR faces (u* elsewhere),
i.e. divergence -> pressure solve -> correction (smac_project).
Backward: dL/du* = P^T g = g + G A^+ D_int(B g) (smac_project_adjoint): one
more MG-PCG solve with the same symmetric operator plus the transposed
divergence and gradient kernels.

Checkpointing across unrolled steps: the projection is linear in u*, so the
backward of a step needs only that step's operator.  Each step keeps its
volume fraction (one cell field) and its pressure increment (the pressure
checkpoint, one cell field) instead of the three face-coefficient arrays;
the backward recomputes the face coefficients from the volume fraction
(smac_assemble_vof, FP64) before the adjoint solve.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from .solver import B200PressureSolver, assemble_vof_device
from .workloads import shapes


@dataclass
class StepOperator:
    """What defines one step's operator: a VoF volume fraction (cells) with
    densities rho0 (alpha = 0) and rho1 (alpha = 1), and the cell/face types."""
    alpha: torch.Tensor
    rho0: float
    rho1: float
    ct: torch.Tensor
    fxt: torch.Tensor
    fyt: torch.Tensor
    fzt: torch.Tensor

    def install(self, solver: B200PressureSolver):
        """Assemble the face coefficients (FP64) and hand them to the solver."""
        _, fb, _ = assemble_vof_device(solver.N, solver.h, self.alpha, self.rho0, self.rho1, self.ct, self.fxt,
                                       self.fyt, self.fzt)
        self._fb = fb  # kept alive until the solver has imported them
        from .solver import _ptr
        from . import _native as nat
        nat.check(solver._lib.smac_set_coefficients(solver._h, _ptr(fb[0]), _ptr(fb[1]), _ptr(fb[2]),
                                                    _ptr(self.ct), _ptr(self.fxt), _ptr(self.fyt), _ptr(self.fzt)))
        torch.cuda.current_stream().synchronize()
        self._fb = None


class ProjectionFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ux, uy, uz, solver: B200PressureSolver, op: StepOperator, dt: float, checkpoints):
        op.install(solver)
        ox, oy, oz = torch.empty_like(ux), torch.empty_like(uy), torch.empty_like(uz)
        p_delta = torch.zeros(shapes(solver.N)["cell"], dtype=torch.float64, device=ux.device)
        solver.project(ux.contiguous(), uy.contiguous(), uz.contiguous(), dt, p_delta, ox, oy, oz)
        if checkpoints is not None:
            checkpoints.append(p_delta)
        ctx.solver = solver
        ctx.op = op
        return ox, oy, oz

    @staticmethod
    def backward(ctx, gx, gy, gz):
        solver, op = ctx.solver, ctx.op
        op.install(solver)  # recompute this step's coefficients
        ox, oy, oz = torch.empty_like(gx), torch.empty_like(gy), torch.empty_like(gz)
        solver.project_adjoint(gx.contiguous(), gy.contiguous(), gz.contiguous(), ox, oy, oz)
        return ox, oy, oz, None, None, None, None


def project(u, solver: B200PressureSolver, op: StepOperator, dt: float = 1.0, checkpoints=None):
    """u = (ux, uy, uz) face tensors (reference layout, float64, CUDA)."""
    return ProjectionFunction.apply(u[0], u[1], u[2], solver, op, dt, checkpoints)


def unrolled(u, solver: B200PressureSolver, ops, dt: float = 1.0, checkpoints=None):
    """Apply one projection per step operator in `ops` (the unrolled steps)."""
    for op in ops:
        u = project(u, solver, op, dt, checkpoints)
    return u
