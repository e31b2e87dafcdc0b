"""The drop-in at the reference's own seam.

The reference's step calls, compiled from its sources (oracle/_ref), run with
this library's G_B200PressureSolver (mydemcfd_b200/seam/G_B200PressureSolver.h)
installed at G_SMACSolver::pressure_solver_ in place of G_PCGSolver, the one
line a maintainer changes in CFD/main.cu:225-227 (driver: oracle/ref_seam.cu).
G_SMACSolver::solve_poisson() (CFD/G_SMACSolver.cu:1499-1501) then reaches
this library through the C ABI, and the reference's correct_vof_velocity()
(:1269-1275) runs unchanged on the p_delta_ it wrote.

Checked against the same calls with the reference's own G_PCGSolver:
- the RHS the solver leaves in rhs_ is bit for bit the reference's;
- p_delta agrees to 1e-10 relative on the fluid cells (mean removed), both
  solved tight;
- the reference's correction of our p_delta is bit for bit the oracle's
  correction of it;
- tol_ keeps the reference's meaning (max|r| dt < tol_): a looser tol_ stops
  earlier.
"""
import numpy as np
import pytest

from mydemcfd_b200 import workloads as W
from oracle import ref as REF

from _cases import fluid_demeaned, oracle_solid_fraction, ref_grid, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (REF.available() and REF.seam_available()),
                                 reason="reference builds oracle/_ref not present")]


def _cases():
    return [W.plain_case(64, seed=1), W.vof_case(32, seed=3, ratio=1000.0),
            W.ibm_case(48, seed=4, nsph=6, solid_fraction=oracle_solid_fraction, rmin_cells=3.0, rmax_cells=6.0)]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c.name)
def test_reference_step_with_b200_solver_installed(oracle_lib, case):
    O = oracle_lib
    rg = ref_grid(case)
    rhs_max = float(np.abs(W.interior(O.make_rhs(rg))).max())
    ref = REF.solve(case, tol=1e-11 / (10 ** (case.N[0] // 32)), do_correct=True)
    tight = 3e-13 * rhs_max * case.dt  # max|r| dt < tol_: 3e-13 of the largest RHS entry
    seam = REF.solve_seam(case, tol=tight, do_correct=True)
    assert seam["iterations"] > 0
    # the divergence our solver wrote into rhs_ is the reference's
    assert np.array_equal(W.interior(seam["rhs"]), W.interior(ref["rhs"]))
    # the pressure increment
    err = rel_err(fluid_demeaned(W.interior(seam["p_delta"]), case.ct),
                  fluid_demeaned(W.interior(ref["p_delta"]), case.ct))
    print(f"{case.name}: seam {seam['iterations']} iterations, reference {ref['iterations']}; p_delta {err:.2e}")
    assert err <= 1e-10
    # the reference's correction of our p_delta is the oracle's, bit for bit
    vx, vy, vz, p = O.correct(rg, seam["p_delta"])
    for got, want, t in ((seam["vx"], vx, case.fxt), (seam["vy"], vy, case.fyt), (seam["vz"], vz, case.fzt)):
        m = t == W.F_INTERIOR
        assert np.array_equal(got[m], want[m])
    assert np.array_equal(W.interior(seam["p"]), W.interior(p))
    # tol_ is the reference's max|r| dt test: a looser one stops earlier
    loose = REF.solve_seam(case, tol=1e-6 * rhs_max * case.dt, do_correct=False)
    assert 0 < loose["iterations"] < seam["iterations"]
    assert rel_err(fluid_demeaned(W.interior(loose["p_delta"]), case.ct),
                   fluid_demeaned(W.interior(ref["p_delta"]), case.ct)) <= 1e-3


def test_reference_step_with_mixed_precision_solver():
    case = W.plain_case(64, seed=1)
    ref = REF.solve(case, tol=1e-13, do_correct=True)
    from oracle import oracle as O
    rhs_max = float(np.abs(W.interior(O.make_rhs(ref_grid(case)))).max())
    seam = REF.solve_seam(case, tol=1e-10 * rhs_max * case.dt, precision=1, do_correct=True)
    err = rel_err(fluid_demeaned(W.interior(seam["p_delta"]), case.ct),
                  fluid_demeaned(W.interior(ref["p_delta"]), case.ct))
    print(f"mixed through the seam: {seam['iterations']} iterations, p_delta {err:.2e}")
    assert err <= 1e-7
