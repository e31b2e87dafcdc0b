"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle and,
where it was built, the reference's own GPU solve (oracle/_ref).

Tolerances: element-wise kernels (divergence, correction, VoF and IBM set-up)
are bit exact; the operator agrees to 1e-13 relative (summation order);
converged FP64 solutions agree with the oracle to 1e-10 relative after
removing the fluid mean (both solved to <= 1e-13 relative residual); mixed
precision meets the 1e-8 FP64 true relative residual.
"""
import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import (B200PressureSolver, DeviceGrid, SMACStep, assemble_vof_device,
                                  box_types_device, ibm_set_solid_device, ibm_solid_fraction_device,
                                  update_boundary_faces_device)

from _cases import fluid_demeaned, load_golden, golden_names, oracle_solid_fraction, ref_grid, rel_err

pytestmark = pytest.mark.gpu


def cpu(t):
    return t.detach().cpu().numpy()


def make_solver(case, **kw):
    s = B200PressureSolver(case.N, case.h, **kw)
    return s


def solve_gpu(case, tol=1e-13, **kw):
    g = DeviceGrid.from_case(case)
    s = make_solver(case, tol=tol, **kw)
    step = SMACStep(g, case.dt)
    step.pressure_solver_ = s
    st = step.solve_poisson()
    torch.cuda.synchronize()
    return g, s, st


# ---------------------------------------------------------------------------
# element-wise kernels: bit exact
def test_box_types_device():
    N = (12, 10, 8)
    ct, fxt, fyt, fzt = box_types_device(N)
    ct2, fxt2, fyt2, fzt2 = W.box_types(N)
    for a, b in ((ct, ct2), (fxt, fxt2), (fyt, fyt2), (fzt, fzt2)):
        assert np.array_equal(cpu(a), b)


@pytest.mark.parametrize("N", [(24, 24, 24), (37, 11, 18), (20, 9, 5)])
def test_divergence_bit_exact(oracle_lib, N):
    """The RHS is bit for bit the reference's; the grids' depths 18 and 5
    leave the kernel's last group of four planes part full."""
    O = oracle_lib
    case = W.vof_case(N[0], seed=3, ratio=10.0, N=N, dt=0.37) if N[1] != N[0] else W.plain_case(24, seed=3, dt=0.37)
    g = DeviceGrid.from_case(case)
    s = make_solver(case)
    s.set_coefficients(g)
    s.divergence(g, case.dt)
    torch.cuda.synchronize()
    ref = O.make_rhs(ref_grid(case))
    assert np.array_equal(W.interior(cpu(g.rhs_)), W.interior(ref))


def test_divergence_with_void_fraction_and_surface_tension_bit_exact(oracle_lib):
    O = oracle_lib
    case = W.vof_case(24, seed=9, ratio=50.0)
    sh = W.shapes(case.N)
    eps = 0.5 + 0.5 * W.uniform01(101, int(np.prod(sh["cell"]))).reshape(sh["cell"])
    eps_old = 0.5 + 0.5 * W.uniform01(102, int(np.prod(sh["cell"]))).reshape(sh["cell"])
    fs = tuple(W.uniform_pm1(103 + i, int(np.prod(sh[k]))).reshape(sh[k]) for i, k in enumerate("xyz"))
    g = DeviceGrid.from_case(case)
    g.void_fraction_ = torch.from_numpy(eps).cuda()
    g.void_fraction_old_ = torch.from_numpy(eps_old).cuda()
    g.f_sx_, g.f_sy_, g.f_sz_ = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in fs)
    s = make_solver(case)
    s.set_coefficients(g)
    s.divergence(g, 0.5)
    torch.cuda.synchronize()
    case.dt = 0.5
    ref = O.make_rhs(ref_grid(case, eps=eps, eps_old=eps_old, fs=fs))
    assert np.array_equal(W.interior(cpu(g.rhs_)), W.interior(ref))


def test_correction_bit_exact(oracle_lib):
    O = oracle_lib
    case = W.vof_case(24, seed=2, ratio=10.0)
    g = DeviceGrid.from_case(case)
    rg = ref_grid(case)
    pd, _, _ = O.solve(rg, tol=1e-12, stop_rule=O.STOP_REL_TRUE)
    g.p_delta_.copy_(torch.from_numpy(pd))
    g.p_.copy_(torch.from_numpy(np.full_like(pd, 0.25)))
    s = make_solver(case)
    s.set_coefficients(g)
    s.correct(g, case.dt, zero_p_delta=True)
    torch.cuda.synchronize()
    vx, vy, vz, p = O.correct(rg, pd, p=np.full_like(pd, 0.25))
    for dv, hv, t in ((g.f_vx_, vx, case.fxt), (g.f_vy_, vy, case.fyt), (g.f_vz_, vz, case.fzt)):
        m = t == W.F_INTERIOR
        assert np.array_equal(cpu(dv)[m], hv[m])
        assert np.all(cpu(dv)[~m] == 0.0)  # untouched
    assert np.array_equal(cpu(g.p_), p)
    assert float(g.p_delta_.abs().max()) == 0.0  # correct_vof_velocity zeroes p_delta_


@pytest.mark.parametrize("N", [(24, 24, 24), (37, 11, 18)])
def test_project_correction_bit_exact(oracle_lib, N):
    """smac_project's correction is the reference's k_correct_vof_velocity of
    the p_delta it exports, bit for bit, and every other face carries u*."""
    O = oracle_lib
    case = W.vof_case(N[0], seed=2, ratio=10.0, N=N)
    g = DeviceGrid.from_case(case)
    s = make_solver(case, tol=1e-10)
    s.set_coefficients(g)
    sh = W.shapes(case.N)
    out = [torch.zeros(sh[k], dtype=torch.float64, device="cuda") for k in "xyz"]
    pd = torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")
    s.project(g.f_vx_star_, g.f_vy_star_, g.f_vz_star_, case.dt, pd, *out)
    torch.cuda.synchronize()
    vx, vy, vz, _ = O.correct(ref_grid(case), cpu(pd))
    for got, want, t, star in zip(out, (vx, vy, vz), (case.fxt, case.fyt, case.fzt), (case.vxs, case.vys, case.vzs)):
        got = cpu(got)
        m = t == W.F_INTERIOR
        assert np.array_equal(got[m], want[m])
        assert np.array_equal(got[~m], star[~m])


def test_vof_assembly_bit_exact(oracle_lib):
    O = oracle_lib
    case = W.vof_case(20, seed=4, ratio=1000.0)
    alpha = torch.from_numpy(case.meta["alpha"]).cuda()
    ct, fxt, fyt, fzt = (torch.from_numpy(a).cuda() for a in (case.ct, case.fxt, case.fyt, case.fzt))
    rho, fb, fir = assemble_vof_device(case.N, case.h, alpha, 1.0, 1000.0, ct, fxt, fyt, fzt)
    rho_o, fb_o, fir_o = O.face_coeffs_vof(case.N, case.meta["alpha"], 1.0, 1000.0, case.ct, case.fxt, case.fyt,
                                           case.fzt)
    for a, b in zip(fb + fir, fb_o + fir_o):
        assert np.array_equal(cpu(a), b)
    assert np.array_equal(W.interior(cpu(rho)), W.interior(rho_o))


def test_ibm_solid_fraction_and_mask_bit_exact(oracle_lib):
    O = oracle_lib
    N = (40, 40, 40)
    h = (1 / 40,) * 3
    sph = W.random_spheres(N, h, seed=12, nsph=8, rmin_cells=3, rmax_cells=7)
    assert len(sph) >= 4
    sf = ibm_solid_fraction_device(N, h, (0.0, 0.0, 0.0), sph)
    sf_o = O.solid_fraction_spheres(N, h, (0.0, 0.0, 0.0), sph)
    assert np.array_equal(W.interior(cpu(sf)), W.interior(sf_o))
    ct, fxt, fyt, fzt = box_types_device(N)
    ibm_set_solid_device(N, sf, ct, fxt, fyt, fzt)
    ct2, fxt2, fyt2, fzt2 = W.box_types(N)
    O.set_solid_cells(N, sf_o, ct2, fxt2, fyt2, fzt2)
    for a, b in ((ct, ct2), (fxt, fxt2), (fyt, fyt2), (fzt, fzt2)):
        assert np.array_equal(cpu(a), b)
    assert (ct2 == W.C_SOLID).sum() > 100


def test_apply_A_matches_reference_operator(oracle_lib):
    O = oracle_lib
    case = W.vof_case(24, seed=6, ratio=1000.0)
    rg = ref_grid(case)
    A = O.build_A(rg)
    x = np.zeros(W.shapes(case.N)["cell"])
    W.interior(x)[...] = W.uniform_pm1(55, 24 ** 3).reshape(24, 24, 24)
    y_o = O.apply_A(case.N, A, x)
    g = DeviceGrid.from_case(case)
    s = make_solver(case)
    s.set_coefficients(g)
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros_like(xd)
    s.apply_A(xd, yd)
    torch.cuda.synchronize()
    scale = np.abs(A[6] * x).max()
    assert np.abs(W.interior(cpu(yd)) - W.interior(y_o)).max() <= 1e-13 * scale


@pytest.mark.parametrize("sweep", [nat.SWEEP_TMA, nat.SWEEP_ZMARCH, nat.SWEEP_SHARED])
@pytest.mark.parametrize("precision", [nat.PRECISION_FP64, nat.PRECISION_MIXED])
@pytest.mark.parametrize("N", [(64, 64, 64), (40, 40, 40), (200, 30, 18), (100, 22, 36), (256, 16, 12), (64, 6, 40)])
def test_fused_sweep_equals_half_sweeps(precision, N, sweep):
    """Each fused one-pass red-black sweep kernel is bitwise the two half-sweep
    launches: the TMA ring, the register z-march (whole rows of 64 to 256
    cells in one to four warps, tile heights of 2, 6 and 14 rows, rows and
    planes that do not fill the last tile) and the shared-memory tiles."""
    case = W.vof_case(N[0], seed=3, ratio=1000.0, N=N)
    g, s, st = solve_gpu(case, tol=1e-6, precision=precision, sweep_kernel=sweep)
    for mode in (0, 1, 2):
        assert s.selftest_sweep(precision, mode) == 0, (mode, precision, sweep)


def test_bounded_wait_expires_and_is_reported():
    """A device-side wait that nothing ends gives up after its limit (about a
    second of SM clock, the limit of every wait in the sweeps), the status
    the host reads is SMAC_CUDA_ERROR, and the handle solves afterwards."""
    case = W.plain_case(16, seed=1)
    g = DeviceGrid.from_case(case)
    s = make_solver(case, tol=1e-10)
    s.set_coefficients(g)
    status, cycles = s.selftest_wait()
    assert status == nat.CUDA_ERROR
    assert cycles >= 1_000_000_000
    step = SMACStep(g, case.dt)
    step.pressure_solver_ = s
    st = step.solve_poisson()
    assert st["status"] == nat.OK and st["rel_residual"] <= 1e-10, st
    s.close()


def _coarse_cases():
    from _cases import oracle_solid_fraction
    return {
        "plain64": lambda: W.plain_case(64, seed=1),
        "plain128": lambda: W.plain_case(128, seed=2),
        "vof40_r1000": lambda: W.vof_case(40, seed=3, ratio=1000.0),
        "ibm48": lambda: W.ibm_case(48, seed=4, nsph=6, solid_fraction=oracle_solid_fraction, rmin_cells=3.0,
                                    rmax_cells=6.0),
        "vof_256x16x12": lambda: W.vof_case(256, seed=3, ratio=1000.0, N=(256, 16, 12)),
        "vof_64x6x40": lambda: W.vof_case(64, seed=3, ratio=1000.0, N=(64, 6, 40)),
    }


@pytest.mark.parametrize("precision", [nat.PRECISION_FP64, nat.PRECISION_MIXED])
@pytest.mark.parametrize("name", list(_coarse_cases()))
def test_cluster_coarse_grids_equal_single_cta(name, precision):
    """The lower V-cycle in one cluster (grids in distributed shared memory,
    SMAC_COARSE_AUTO) gives the solve of the separately launched sweeps plus
    the single-CTA kernel (SMAC_COARSE_CTA) bit for bit: the same iterations
    and the same p_delta.  Cases: cubic grids whose cluster set starts at 32^3
    or 20^3, a thin grid spread over six ranks one plane each, and one whose
    set holds grids of five planes."""
    case = _coarse_cases()[name]()
    out = []
    for ck in (nat.COARSE_AUTO, nat.COARSE_CTA):
        g, s, st = solve_gpu(case, tol=1e-12, precision=precision, coarse_kernel=ck)
        assert st["status"] == 0, st
        out.append((st["iterations"], cpu(g.p_delta_).copy(), st["kernel_launches"]))
        s.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    print(f"{name}: {out[0][0]} iterations, {out[0][2]} launches with the cluster, {out[1][2]} without")


# ---------------------------------------------------------------------------
# solves
def test_fp64_solve_matches_oracle_64(oracle_lib):
    """Config 1: 64^3, plain FP64 MG-PCG, 1e-10 relative in value."""
    O = oracle_lib
    case = W.plain_case(64, seed=1)
    g, s, st = solve_gpu(case, tol=1e-13)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-13
    pd_o, _, st_o = O.solve(ref_grid(case), tol=1e-14, stop_rule=O.STOP_REL_TRUE, max_iter=400)
    a = fluid_demeaned(W.interior(cpu(g.p_delta_)), case.ct)
    b = fluid_demeaned(W.interior(pd_o), case.ct)
    assert rel_err(a, b) <= 1e-10
    # layout: ghost entries of p_delta_ are never written
    full = cpu(g.p_delta_)
    assert full[0].max() == 0 and full[-1].max() == 0 and full[:, 0].max() == 0 and full[:, :, -1].max() == 0


@pytest.mark.skipif("plain64_s1_gmg" not in golden_names(), reason="no golden vector")
def test_fp64_solve_matches_reference_golden_64():
    meta, arr = load_golden("plain64_s1_gmg")
    case = W.plain_case(64, seed=1)
    g, s, st = solve_gpu(case, tol=1e-13)
    ours = W.interior(cpu(g.p_delta_)).reshape(-1)[arr["p_delta_idx"]]
    ref = arr["p_delta_val"] - float(arr["p_delta_mean"])
    assert rel_err(ours, ref) <= 1e-10


def test_fp64_solve_matches_reference_build():
    from oracle import ref as REF
    if not REF.available():
        pytest.skip("oracle/_ref not built")
    ibm = W.ibm_case(48, seed=4, nsph=6, solid_fraction=oracle_solid_fraction, rmin_cells=3.0, rmax_cells=6.0)
    for case in (W.plain_case(64, seed=1), W.vof_case(32, seed=3, ratio=1000.0), ibm):
        # the reference's own stop test, max|r| dt < tol every 5 iterations
        r = REF.solve(case, tol=1e-11 / (10 ** (case.N[0] // 32)), do_correct=True)
        g, s, st = solve_gpu(case, tol=1e-13)
        a = fluid_demeaned(W.interior(cpu(g.p_delta_)), case.ct)
        b = fluid_demeaned(W.interior(r["p_delta"]), case.ct)
        assert rel_err(a, b) <= 1e-10, case.name


def test_mixed_precision_reaches_fp64_tolerance():
    case = W.plain_case(64, seed=2)
    g64, s64, st64 = solve_gpu(case, tol=1e-12)
    gm, sm, stm = solve_gpu(case, tol=1e-8, precision=nat.PRECISION_MIXED)
    assert stm["status"] == 0
    assert stm["rel_residual"] <= 1e-8
    assert stm["reliable_updates"] >= 1
    err = rel_err(fluid_demeaned(W.interior(cpu(gm.p_delta_)), case.ct),
                  fluid_demeaned(W.interior(cpu(g64.p_delta_)), case.ct))
    assert err < 1e-5


def test_vof_1000_to_1(oracle_lib):
    """VoF 48^3 at 1000:1: FP64 to 1e-13 against the oracle's tight solve at
    1e-10; mixed precision to the 1e-8 FP64 true residual, whose error bound
    is the residual times the conditioning of the low modes (1e-6)."""
    O = oracle_lib
    case = W.vof_case(48, seed=3, ratio=1000.0)
    pd_o, _, st_o = O.solve(ref_grid(case), tol=1e-13, stop_rule=O.STOP_REL_TRUE, max_iter=1000)
    assert st_o["converged"] and st_o["true_res_rel"] <= 1e-13
    ref = fluid_demeaned(W.interior(pd_o), case.ct)
    g, s, st = solve_gpu(case, tol=1e-13)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-13
    assert rel_err(fluid_demeaned(W.interior(cpu(g.p_delta_)), case.ct), ref) <= 1e-10
    g, s, st = solve_gpu(case, tol=1e-8, precision=nat.PRECISION_MIXED)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-8
    assert rel_err(fluid_demeaned(W.interior(cpu(g.p_delta_)), case.ct), ref) <= 1e-6


def test_outlet_faces_bit_exact_and_outlet_solve(oracle_lib):
    """Outlets on two sides (p = 0 there): the face rule is bit exact against
    the oracle, and the non-singular GMG-PCG solve matches the oracle's."""
    import dataclasses
    O = oracle_lib
    case = W.vof_case(32, seed=21, ratio=100.0)
    marks = W.outlet_marks(case.N, ("x+", "y-"))
    fb_o = O.update_boundary_faces(case.N, *marks, case.fbx, case.fby, case.fbz)
    fb_d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (case.fbx, case.fby, case.fbz)]
    update_boundary_faces_device(case.N, case.h, [torch.from_numpy(m).cuda() for m in marks], fb_d)
    torch.cuda.synchronize()
    for a, b in zip(fb_d, fb_o):
        assert np.array_equal(cpu(a), b)
    oc = dataclasses.replace(case, fbx=fb_o[0], fby=fb_o[1], fbz=fb_o[2])
    g, s, st = solve_gpu(oc, tol=1e-12, solver_type=nat.GMG_PCG)
    assert st["status"] == 0
    pd_o, _, st_o = O.solve(ref_grid(oc), solver_type=O.GMG_PCG, tol=1e-13, stop_rule=O.STOP_REL_TRUE, max_iter=1000)
    assert st_o["converged"]
    assert rel_err(W.interior(cpu(g.p_delta_)), W.interior(pd_o)) < 1e-9


def test_ibm_solids_stay_zero_and_match_oracle(oracle_lib):
    O = oracle_lib
    case = W.ibm_case(48, seed=4, nsph=6, solid_fraction=oracle_solid_fraction, rmin_cells=3.0, rmax_cells=6.0)
    assert case.meta["solid_cells"] > 0
    g, s, st = solve_gpu(case, tol=1e-13)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-13
    pd = W.interior(cpu(g.p_delta_))
    solid = W.interior(case.ct) == W.C_SOLID
    assert np.all(pd[solid] == 0.0)
    pd_o, _, st_o = O.solve(ref_grid(case), tol=1e-13, stop_rule=O.STOP_REL_TRUE, max_iter=1000)
    assert st_o["converged"] and st_o["true_res_rel"] <= 1e-13
    assert rel_err(fluid_demeaned(pd, case.ct), fluid_demeaned(W.interior(pd_o), case.ct)) <= 1e-10


@pytest.mark.parametrize("solver_type", [nat.PURENEUMANN_STANDARD_PCG, nat.GMG_PCG, nat.STANDARD_PCG])
def test_solver_variants_agree(solver_type):
    case = W.plain_case(32, seed=8)
    g0, _, st0 = solve_gpu(case, tol=1e-12)
    g1, _, st1 = solve_gpu(case, tol=1e-11, solver_type=solver_type)
    assert st1["status"] == 0
    assert rel_err(fluid_demeaned(W.interior(cpu(g1.p_delta_)), case.ct),
                   fluid_demeaned(W.interior(cpu(g0.p_delta_)), case.ct)) < 1e-8


def test_reference_stop_rule():
    case = W.plain_case(32, seed=5, dt=0.1)
    g, s, st = solve_gpu(case, tol=1e-7, stop_rule=nat.STOP_REFERENCE)
    assert st["status"] == 0
    assert st["max_residual"] * 0.1 < 1e-7


def test_non_cubic_and_odd_sizes():
    case = W.plain_case(N=(40, 24, 26), seed=9)
    g, s, st = solve_gpu(case, tol=1e-10)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-10
    assert s.num_levels() >= 2


def test_deterministic_replay():
    case = W.plain_case(48, seed=10)
    g1, s, _ = solve_gpu(case, tol=1e-10, precision=nat.PRECISION_MIXED)
    a = cpu(g1.p_delta_).copy()
    step = SMACStep(g1, case.dt)
    step.pressure_solver_ = s
    step.solve_poisson()
    torch.cuda.synchronize()
    assert np.array_equal(a, cpu(g1.p_delta_))


# ---------------------------------------------------------------------------
# failures are reported, never faulted
def test_nan_input_reports_status():
    case = W.plain_case(24, seed=1)
    case.vxs[5, 5, 5] = np.nan
    g = DeviceGrid.from_case(case)
    s = make_solver(case)
    step = SMACStep(g, 1.0)
    step.pressure_solver_ = s
    st = s.solve(step, raise_on_fail=False)
    assert st["status"] == nat.NAN


def test_iteration_cap_reports_not_converged():
    case = W.plain_case(32, seed=1)
    g = DeviceGrid.from_case(case)
    s = make_solver(case, tol=1e-14, max_iter=2)
    step = SMACStep(g, 1.0)
    step.pressure_solver_ = s
    with pytest.raises(nat.SmacError) as ei:
        step.solve_poisson()
    assert ei.value.status == nat.NOT_CONVERGED


def test_reference_call_sequence():
    """solve_poisson -> correct_vof_velocity, as CFD/main.cu:313-315 calls them."""
    case = W.plain_case(32, seed=3)
    g = DeviceGrid.from_case(case)
    step = SMACStep(g, case.dt)
    step.pressure_solver_ = B200PressureSolver(case.N, case.h)
    step.pressure_solver_.set_solver(nat.PURENEUMANN_GMG_PCG)
    step.pressure_solver_.tol_ = 1e-12
    step.solve_poisson()
    pd = cpu(g.p_delta_).copy()
    step.correct_vof_velocity()
    torch.cuda.synchronize()
    assert np.array_equal(W.interior(cpu(g.p_)), np.where(W.interior(case.ct) == 0, W.interior(pd), 0.0))
    assert float(g.p_delta_.abs().max()) == 0.0
    # the corrected field is divergence free
    s2 = B200PressureSolver(case.N, case.h)
    g2 = DeviceGrid.from_case(case)
    g2.f_vx_star_.copy_(g.f_vx_); g2.f_vy_star_.copy_(g.f_vy_); g2.f_vz_star_.copy_(g.f_vz_)
    s2.set_coefficients(g2)
    s2.divergence(g2, case.dt)
    torch.cuda.synchronize()
    assert float(g2.rhs_.abs().max()) < 1e-8 * float(g.rhs_.abs().max())


# ---------------------------------------------------------------------------
# adjoint
def _project(s, case, u):
    sh = W.shapes(case.N)
    out = [torch.zeros(sh[k], dtype=torch.float64, device="cuda") for k in "xyz"]
    pd = torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")
    s.project(*u, case.dt, pd, *out)
    return out


def _adjoint(s, case, gvec):
    out = [torch.zeros_like(t) for t in gvec]
    s.project_adjoint(*gvec, *out)
    return out


def test_adjoint_dot_product():
    case = W.vof_case(32, seed=7, ratio=100.0)
    g = DeviceGrid.from_case(case)
    s = make_solver(case, tol=1e-13)
    s.set_coefficients(g)
    sh = W.shapes(case.N)
    u = [torch.from_numpy(W.uniform_pm1(200 + i, int(np.prod(sh[k]))).reshape(sh[k])).cuda() for i, k in enumerate("xyz")]
    v = [torch.from_numpy(W.uniform_pm1(300 + i, int(np.prod(sh[k]))).reshape(sh[k])).cuda() for i, k in enumerate("xyz")]
    Pu = _project(s, case, u)
    PTv = _adjoint(s, case, v)
    lhs = sum(float((a * b).sum()) for a, b in zip(Pu, v))
    rhs = sum(float((a * b).sum()) for a, b in zip(u, PTv))
    assert abs(lhs - rhs) <= 1e-9 * max(abs(lhs), 1.0)


def test_autograd_matches_finite_differences():
    # The unrolled projections are linear in u and the loss is quadratic, so a
    # central difference has no truncation error for any step: a large step
    # (1e-3 of |u|) keeps the solve tolerance's share of the difference near
    # 1e-11 / 1e-3 = 1e-8, well inside the 1e-6 check.
    from mydemcfd_b200.autograd import StepOperator, unrolled
    case = W.vof_case(24, seed=5, ratio=100.0)
    s = make_solver(case, tol=1e-11)
    ct, fxt, fyt, fzt = (torch.from_numpy(a).cuda() for a in (case.ct, case.fxt, case.fyt, case.fzt))
    ops = []
    for k in range(3):
        c = W.vof_case(24, seed=5 + k, ratio=100.0)
        ops.append(StepOperator(torch.from_numpy(c.meta["alpha"]).cuda(), 1.0, 100.0, ct, fxt, fyt, fzt))
    sh = W.shapes(case.N)
    u0 = [torch.from_numpy(W.uniform_pm1(400 + i, int(np.prod(sh[k]))).reshape(sh[k])).cuda() for i, k in enumerate("xyz")]
    tgt = [torch.from_numpy(W.uniform_pm1(500 + i, int(np.prod(sh[k]))).reshape(sh[k])).cuda() for i, k in enumerate("xyz")]

    def loss(u):
        out = unrolled(u, s, ops)
        return sum(((a - b) ** 2).sum() for a, b in zip(out, tgt))

    u = [t.clone().requires_grad_(True) for t in u0]
    L = loss(u)
    L.backward()
    grads = [t.grad for t in u]
    for d in range(16):
        dirs = [torch.from_numpy(W.uniform_pm1(600 + 10 * d + i, int(np.prod(sh[k]))).reshape(sh[k])).cuda()
                for i, k in enumerate("xyz")]
        eps = 1e-3 * float(torch.sqrt(sum((t ** 2).sum() for t in u0)) / torch.sqrt(sum((t ** 2).sum() for t in dirs)))
        with torch.no_grad():
            lp = loss([a + eps * b for a, b in zip(u0, dirs)])
            lm = loss([a - eps * b for a, b in zip(u0, dirs)])
        fd = float(lp - lm) / (2 * eps)
        an = sum(float((gg * dd).sum()) for gg, dd in zip(grads, dirs))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-30), (fd, an)
