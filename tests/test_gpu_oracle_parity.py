"""GPU parity of every PCG variant and of the golden vectors, against the
oracle and the reference's own solve.

- Each of the four PCG_TYPES (CFD/Enums.h:25-30; the reference's
  solve_pcg, solve_pureneumann_pcg, solve_gmgpcg and solve_pureneumann_gmgpcg,
  CFD/pressure_solver/G_PCGSolver.cu:307-922) runs on the GPU and in the
  oracle with the same solver type, both to a relative true residual of
  1e-13; the converged pressures agree to 1e-10 relative on the fluid cells
  after removing their mean (the pure-Neumann null space).  The grids are a
  plain 32^3 box, a VoF sphere at 1000:1, IBM spheres and a ragged
  40 x 24 x 22 VoF grid.
- Every golden vector of the reference's own GPU solve (tests/golden/,
  made by tests/golden/make_golden.py) is solved on the GPU with the
  vector's solver type.  The GPU result agrees with the oracle's tight solve
  to 1e-10, and with the vector to within the vector's own distance from
  that tight solve plus 1e-10 (the vectors stop at the reference's
  max|r|*dt test, tol 1e-9 .. 1e-11, so each supports its own precision).
- Full-size configurations: VoF 192^3 at 1000:1 and IBM 256^3 with 200
  spheres, FP64 on the GPU and in the oracle, both to 1e-13, agree to 1e-10.
"""
import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import B200PressureSolver, DeviceGrid, SMACStep, ibm_solid_fraction_device

from _cases import (build_case, fluid_demeaned, golden_names, load_golden, oracle_solid_fraction, ref_grid,
                    rel_err)

pytestmark = pytest.mark.gpu

TIGHT = 1e-13
VALUE_TOL = 1e-10


def _gpu_solve(case, solver_type, tol=TIGHT, max_iter=5000):
    g = DeviceGrid.from_case(case)
    s = B200PressureSolver(case.N, case.h, tol=tol, solver_type=solver_type, max_iter=max_iter)
    step = SMACStep(g, case.dt)
    step.pressure_solver_ = s
    st = step.solve_poisson()
    torch.cuda.synchronize()
    pd = W.interior(g.p_delta_.cpu().numpy()).copy()
    rhs = W.interior(g.rhs_.cpu().numpy()).copy()
    s.close()
    return pd, st, rhs


def _oracle_solve(O, case, solver_type, tol=TIGHT):
    pd, _, st = O.solve(ref_grid(case), solver_type=solver_type, tol=tol, stop_rule=O.STOP_REL_TRUE, max_iter=5000)
    assert st["converged"] and st["true_res_rel"] <= tol, st
    return W.interior(pd)


def _cases():
    return {
        "plain32": lambda: W.plain_case(32, seed=8),
        "vof32_r1000": lambda: W.vof_case(32, seed=3, ratio=1000.0),
        "ibm48": lambda: W.ibm_case(48, seed=4, nsph=6, solid_fraction=oracle_solid_fraction, rmin_cells=3.0,
                                    rmax_cells=6.0),
        # ragged: depths and widths that fill no kernel's tiles or plane groups
        "vof_40x24x22": lambda: W.vof_case(40, seed=5, ratio=100.0, N=(40, 24, 22)),
    }


VARIANTS = [nat.STANDARD_PCG, nat.PURENEUMANN_STANDARD_PCG, nat.GMG_PCG, nat.PURENEUMANN_GMG_PCG]


@pytest.mark.parametrize("case_name", list(_cases()))
@pytest.mark.parametrize("solver_type", VARIANTS)
def test_pcg_variant_matches_oracle_variant(oracle_lib, solver_type, case_name):
    """The GPU's solver_type against the oracle's restatement of the same
    reference variant, both to 1e-13: 1e-10 on the fluid cells."""
    O = oracle_lib
    case = _cases()[case_name]()
    pd, st, _ = _gpu_solve(case, solver_type)
    assert st["status"] == 0 and st["rel_residual"] <= TIGHT, st
    pd_o = _oracle_solve(O, case, solver_type)
    err = rel_err(fluid_demeaned(pd, case.ct), fluid_demeaned(pd_o, case.ct))
    print(f"{case_name} solver_type {solver_type}: {st['iterations']} iterations, error vs oracle {err:.2e}")
    assert err <= VALUE_TOL
    # cells without an unknown keep p_delta = 0
    assert np.all(pd[W.interior(case.ct) != W.C_INTERIOR] == 0.0)


def _golden_distance(case, arr, p):
    """Relative distance of the fluid-demeaned interior pressure p from the
    golden vector: whole fields compare after removing the fluid mean;
    sampled fields compare on their fluid samples after the best constant
    shift (the null space)."""
    if "p_delta" in arr:
        return rel_err(fluid_demeaned(p, case.ct), fluid_demeaned(arr["p_delta"], case.ct))
    idx = arr["p_delta_idx"]
    fl = (W.interior(case.ct) == W.C_INTERIOR).reshape(-1)[idx]
    ours = fluid_demeaned(p, case.ct).reshape(-1)[idx][fl]
    ref = arr["p_delta_val"][fl]
    return rel_err(ours + (ref - ours).mean(), ref)


GOLDEN = golden_names()


@pytest.mark.skipif(not GOLDEN, reason="no golden vectors")
@pytest.mark.parametrize("name", GOLDEN)
def test_gpu_matches_reference_golden(oracle_lib, name):
    O = oracle_lib
    meta, arr = load_golden(name)
    case = build_case(meta["spec"])
    pd, st, rhs = _gpu_solve(case, meta["solver_type"])
    assert st["status"] == 0 and st["rel_residual"] <= TIGHT, st
    # the divergence is element-wise: bit exact against the reference's
    if "rhs" in arr:
        assert np.array_equal(rhs, arr["rhs"])
    else:
        assert np.array_equal(rhs.reshape(-1)[arr["rhs_idx"]], arr["rhs_val"])
    pd_o = _oracle_solve(O, case, O.PURENEUMANN_GMG_PCG)
    err_oracle = rel_err(fluid_demeaned(pd, case.ct), fluid_demeaned(pd_o, case.ct))
    support = _golden_distance(case, arr, pd_o)  # how close the vector itself is to the tight solution
    err_golden = _golden_distance(case, arr, pd)
    print(f"{name}: GPU vs oracle {err_oracle:.2e}, GPU vs golden {err_golden:.2e} (vector's own {support:.2e})")
    assert err_oracle <= VALUE_TOL
    assert err_golden <= support + VALUE_TOL


def _full_size(case):
    pd, st, _ = _gpu_solve(case, nat.PURENEUMANN_GMG_PCG, max_iter=400)
    assert st["status"] == 0 and st["rel_residual"] <= TIGHT, st
    from oracle import oracle as O
    pd_o = _oracle_solve(O, case, O.PURENEUMANN_GMG_PCG)
    err = rel_err(fluid_demeaned(pd, case.ct), fluid_demeaned(pd_o, case.ct))
    print(f"{case.name}: {st['iterations']} iterations, GPU FP64 vs oracle (both 1e-13) {err:.2e}")
    assert err <= VALUE_TOL
    return pd


def test_vof_192_ratio_1000_fp64_matches_oracle(oracle_lib):
    _full_size(W.vof_case(192, seed=3, ratio=1000.0))


def test_ibm_256_200_spheres_fp64_matches_oracle(oracle_lib):
    case = W.ibm_case(256, seed=4, nsph=200,
                      solid_fraction=lambda N, h, o, s: ibm_solid_fraction_device(N, h, o, s).cpu().numpy())
    pd = _full_size(case)
    assert np.all(pd[W.interior(case.ct) == W.C_SOLID] == 0.0)
