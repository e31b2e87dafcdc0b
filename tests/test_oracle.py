"""CPU tests of the oracle: known answers of the discrete operator, the
reference's quirks, and agreement with the golden vectors that the
reference's own GPU solve produced (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from mydemcfd_b200 import workloads as W

from _cases import build_case, fluid_demeaned, golden_names, load_golden, ref_grid, rel_err


def test_box_types_match_reference_setup(oracle_lib):
    O = oracle_lib
    for N in ((8, 8, 8), (6, 10, 12)):
        fxt, fyt, fzt = O.set_face_type(N)
        ct = O.set_cell_type(N)
        ct2, fxt2, fyt2, fzt2 = W.box_types(N)
        for a, b in ((fxt, fxt2), (fyt, fyt2), (fzt, fzt2), (ct, ct2)):
            assert np.array_equal(a, b)


def test_vof_coefficients_numpy_equals_oracle(oracle_lib):
    O = oracle_lib
    c = W.vof_case(16, seed=3, ratio=1000.0)
    alpha = c.meta["alpha"]
    rho, (fbx, fby, fbz), (irx, iry, irz) = O.face_coeffs_vof(c.N, alpha, 1.0, 1000.0, c.ct, c.fxt, c.fyt, c.fzt)
    for a, b in ((fbx, c.fbx), (fby, c.fby), (fbz, c.fbz), (irx, c.fbx)):
        assert np.array_equal(a, b)  # bit-exact: the same IEEE operations
    # 1000:1 spans three decades of coefficients
    nz = fbx[fbx > 0]
    assert nz.max() / nz.min() > 900


def test_rhs_is_minus_divergence(oracle_lib):
    O = oracle_lib
    c = W.plain_case(12, seed=3)
    g = ref_grid(c)
    rhs = O.make_rhs(g)
    nx = c.N[0]
    h = c.h[0]
    div = np.zeros_like(W.interior(rhs))
    div += (c.vxs[1:-1, 1:-1, 2:nx + 2] - c.vxs[1:-1, 1:-1, 1:nx + 1]) * (1 / h)
    div += (c.vys[1:-1, 2:nx + 2, 1:-1] - c.vys[1:-1, 1:nx + 1, 1:-1]) * (1 / h)
    div += (c.vzs[2:nx + 2, 1:-1, 1:-1] - c.vzs[1:nx + 1, 1:-1, 1:-1]) * (1 / h)
    assert np.allclose(W.interior(rhs), -div, rtol=0, atol=1e-12)
    # compatible: walls carry u* = 0, so the sum vanishes
    assert abs(W.interior(rhs).sum()) < 1e-9


def test_operator_symmetric_and_neumann(oracle_lib):
    O = oracle_lib
    c = W.vof_case(12, seed=5, ratio=100.0)
    g = ref_grid(c)
    A = O.build_A(g)
    rng = np.random.default_rng(0)
    x = np.zeros(W.shapes(c.N)["cell"]); y = np.zeros_like(x)
    W.interior(x)[...] = rng.standard_normal(W.interior(x).shape)
    W.interior(y)[...] = rng.standard_normal(W.interior(y).shape)
    Ax, Ay = O.apply_A(c.N, A, x), O.apply_A(c.N, A, y)
    lhs = (W.interior(Ax) * W.interior(y)).sum()
    rhs = (W.interior(x) * W.interior(Ay)).sum()
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # pure Neumann: constants are in the null space
    one = np.zeros_like(x); W.interior(one)[...] = 1.0
    assert np.abs(W.interior(O.apply_A(c.N, A, one))).max() < 1e-9 * A[6].max()


def test_cosine_eigenmode_known_answer(oracle_lib):
    """cos(pi k (i+1/2)/N) is an exact eigenvector of the Neumann 7-point
    Laplacian with eigenvalue (4/h^2) sin^2(pi k/(2N)) per direction."""
    O = oracle_lib
    N = (16, 16, 16)
    c = W.plain_case(16, seed=1)
    g = ref_grid(c)
    A = O.build_A(g)
    h = c.h[0]
    k = (1, 2, 3)
    i = np.arange(16) + 0.5
    ex, ey, ez = (np.cos(np.pi * k[d] * i / 16) for d in range(3))
    mode = ez[:, None, None] * ey[None, :, None] * ex[None, None, :]
    x = np.zeros(W.shapes(N)["cell"]); W.interior(x)[...] = mode
    lam = sum(4 / h ** 2 * np.sin(np.pi * kk / 32) ** 2 for kk in k)
    Ax = O.apply_A(N, A, x)
    assert np.abs(W.interior(Ax) - lam * mode).max() < 1e-9 * lam


def test_projection_divergence_free_and_idempotent(oracle_lib):
    O = oracle_lib
    c = W.plain_case(24, seed=11)
    g = ref_grid(c)
    pd, rhs, st = O.solve(g, tol=1e-13, stop_rule=O.STOP_REL_TRUE)
    vx, vy, vz, p = O.correct(g, pd)
    # walls keep u* (=0); the corrected field is discretely divergence free
    c2 = W.Case("p", c.N, c.h, c.dt, vx, vy, vz, c.fbx, c.fby, c.fbz, c.ct, c.fxt, c.fyt, c.fzt)
    g2 = ref_grid(c2)
    rhs2 = O.make_rhs(g2)
    assert np.abs(W.interior(rhs2)).max() < 1e-9 * np.abs(W.interior(rhs)).max()
    # P(Pu) = Pu
    pd2, _, st2 = O.solve(g2, tol=1e-13, stop_rule=O.STOP_REL_TRUE)
    vx2, vy2, vz2, _ = O.correct(g2, pd2)
    assert rel_err(vx2, vx) < 1e-9 and rel_err(vy2, vy) < 1e-9 and rel_err(vz2, vz) < 1e-9


def test_single_level_shape_refused(oracle_lib):
    """The reference indexes levels_[-1] when only one level exists
    (G_GMGSolver.cu:977); the oracle refuses such shapes."""
    O = oracle_lib
    c = W.plain_case(16, seed=1)
    _, _, st = O.solve(ref_grid(c), tol=1e-8)
    assert st["rc"] == -2
    c = W.plain_case(N=(26, 24, 24), seed=1)  # 13 is odd and still coarsens -> reference abort()
    _, _, st = O.solve(ref_grid(c), tol=1e-8)
    assert st["rc"] == -1


def test_reference_stop_rule(oracle_lib):
    O = oracle_lib
    c = W.plain_case(24, seed=2)
    g = ref_grid(c)
    pd, rhs, st = O.solve(g, tol=1e-6, stop_rule=O.STOP_REFERENCE)
    assert st["converged"] and st["res_max"] * c.dt < 1e-6
    # checked only every 5 iterations (G_PCGSolver.cu:884): count is 5k+1
    assert (st["iterations"] - 1) % 5 == 0


def test_oracle_thread_count_does_not_change_results(oracle_lib):
    O = oracle_lib
    c = W.plain_case(32, seed=4)
    n0 = O.num_threads()
    try:
        O.set_num_threads(1)
        a, _, s1 = O.solve(ref_grid(c), tol=1e-10)
        O.set_num_threads(max(2, n0))
        b, _, s2 = O.solve(ref_grid(c), tol=1e-10)
    finally:
        O.set_num_threads(n0)
    assert s1["iterations"] == s2["iterations"]
    assert np.array_equal(a, b)


# ---------------------------------------------------------------------------
# golden vectors from the reference's own GPU solve
GOLDEN = golden_names()


@pytest.mark.skipif(not GOLDEN, reason="no golden vectors")
@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_golden(oracle_lib, name):
    O = oracle_lib
    meta, arr = load_golden(name)
    case = build_case(meta["spec"])
    g = ref_grid(case)
    pd, rhs, st = O.solve(g, solver_type=meta["solver_type"], tol=meta["tol"], levels=meta["levels"])
    assert st["rc"] == 0
    assert st["num_levels"] == (meta["num_levels"] if meta["solver_type"] in (2, 3) else 0)
    # the reference prints the iteration count; the checks land on the same
    # multiple of the check frequency
    assert st["iterations"] == meta["iterations"]
    rhs_i, pd_i = W.interior(rhs), W.interior(pd)
    if "rhs" in arr:
        assert np.array_equal(rhs_i, arr["rhs"])  # element-wise, bit exact
        ref_pd = arr["p_delta"]
        assert rel_err(pd_i, ref_pd) < 1e-9
        assert rel_err(fluid_demeaned(pd_i, case.ct), fluid_demeaned(ref_pd, case.ct)) < 1e-9
    else:
        assert np.array_equal(rhs_i.reshape(-1)[arr["rhs_idx"]], arr["rhs_val"])
        got = pd_i.reshape(-1)[arr["p_delta_idx"]]
        assert rel_err(got, arr["p_delta_val"]) < 1e-9
        assert abs(np.linalg.norm(pd_i) - float(arr["p_delta_norm"])) < 1e-9 * float(arr["p_delta_norm"])
    if "vx" in arr:
        # the correction is element-wise: given the reference's p_delta it is bit exact
        full = np.zeros(W.shapes(case.N)["cell"])
        W.interior(full)[...] = arr["p_delta"]
        vx, vy, vz, p = O.correct(g, full)
        m = case.fxt == W.F_INTERIOR
        assert np.array_equal(vx[m], arr["vx"][m])
        assert np.array_equal(vy[case.fyt == W.F_INTERIOR], arr["vy"][case.fyt == W.F_INTERIOR])
        assert np.array_equal(vz[case.fzt == W.F_INTERIOR], arr["vz"][case.fzt == W.F_INTERIOR])
        assert np.array_equal(W.interior(p), W.interior(arr["p"]))


def test_outlet_faces_twice_the_interior_neighbour(oracle_lib):
    O = oracle_lib
    N = (6, 5, 4)
    ct, fxt, fyt, fzt = W.box_types(N)
    rng = np.random.default_rng(3)
    fb = [np.where(t == W.F_INTERIOR, rng.uniform(0.1, 1.0, t.shape), 0.0) for t in (fxt, fyt, fzt)]
    marks = W.outlet_marks(N, ("x+", "z-"))
    out = O.update_boundary_faces(N, *marks, *fb)
    nx, ny, nz = N
    mx, _, mz = marks
    assert int((mx == 2).sum()) == ny * nz and int((mz == 1).sum()) == nx * ny
    np.testing.assert_array_equal(out[0][:, :, nx + 1][mx[:, :, nx + 1] == 2],
                                  2.0 * fb[0][:, :, nx][mx[:, :, nx + 1] == 2])
    np.testing.assert_array_equal(out[2][1][mz[1] == 1], 2.0 * fb[2][2][mz[1] == 1])
    for o, f, m in zip(out, fb, marks):
        np.testing.assert_array_equal(o[m == 0], f[m == 0])
