"""CPU tests of the oracle: known answers of the discrete operator, the
reference's quirks, and agreement with the golden vectors that the
reference's own GPU solve produced (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from mydemcfd_b200 import workloads as W

from _cases import (build_case, fluid_demeaned, golden_names, load_golden, post_case_from_spec, post_golden_names,
                    ref_grid, rel_err, surface_case_from_spec, surface_golden_names, vstar_golden_names,
                    momentum_case_from_spec, momentum_golden_names, property_case_from_spec,
                    property_golden_names, beta_case_from_spec, beta_golden_names, flux_case_from_spec,
                    flux_golden_names)


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


# ---------------------------------------------------------------------------
# the pass after the projection (update_boundary_ghost + make_face_gradp)

def _post_loops(c):
    """A second restatement in plain loops, written from the reference's
    kernels (CFD/G_SMACSolver.cu:1144-1343, CFD/G_BoundaryFunctions.cu:143-560),
    with the reference's evaluation order."""
    nx, ny, nz = c.N
    dx, dy, dz = c.h
    gx, gy, gz = c.g
    p = c.p.copy()
    ct, rho = c.ct, c.rho
    for iz in range(1, nz + 1):
        for iy in range(1, ny + 1):
            for ix in range(1, nx + 1):
                if ct[iz, iy, ix] != W.C_SOLID:
                    continue
                v = 0.0
                for (jx, jy, jz, s, gg, hh) in ((ix - 1, iy, iz, 1, gx, dx), (ix + 1, iy, iz, -1, gx, dx),
                                                 (ix, iy - 1, iz, 1, gy, dy), (ix, iy + 1, iz, -1, gy, dy),
                                                 (ix, iy, iz - 1, 1, gz, dz), (ix, iy, iz + 1, -1, gz, dz)):
                    if ct[jz, jy, jx] == W.C_INTERIOR:
                        t = rho[jz, jy, jx] * gg * hh
                        v = p[jz, jy, jx] + t if s > 0 else p[jz, jy, jx] - t
                        break
                p[iz, iy, ix] = v
    for iz in range(nz + 2):
        for iy in range(ny + 2):
            for ix in range(nx + 2):
                if 0 < ix <= nx and 0 < iy <= ny and 0 < iz <= nz:
                    continue
                sx, sy, sz = min(max(ix, 1), nx), min(max(iy, 1), ny), min(max(iz, 1), nz)
                r = (ix - sx) * dx * gx + (iy - sy) * dy * gy + (iz - sz) * dz * gz
                p[iz, iy, ix] = p[sz, sy, sx] + rho[sz, sy, sx] * r
    v = [a.copy() for a in c.v]
    inv = (1.0 / dx, 1.0 / dy, 1.0 / dz)
    for a in range(3):
        m = c.marks[a]
        for (iz, iy, ix) in zip(*np.nonzero(m)):
            if not (1 <= ix <= nx + 1 and 1 <= iy <= ny + 1 and 1 <= iz <= nz + 1):
                continue
            s = 1 if m[iz, iy, ix] == 1 else -1
            cidx = [ix, iy, iz]
            cidx[a] += s
            sign = 1.0 if s < 0 else -1.0
            v[a][iz, iy, ix] = c.vs[a][iz, iy, ix] + sign * c.fb[a][iz, iy, ix] * c.dt * \
                c.p_delta[cidx[2], cidx[1], cidx[0]] * inv[a]

    def rule(t, vb, lam, bnd, inner):
        return {2: 2.0 * (1.0 - lam) * vb - inner, 0: -inner, 4: 2.0 * bnd - inner, 1: inner}.get(int(t), bnd)

    N = (nx, ny, nz)
    for a in range(3):
        b, cc = [k for k in range(3) if k != a]
        arr, ids = v[a], c.bcid[a]
        lam = c.lam[a] if c.lam is not None else np.zeros(arr.shape)
        get = lambda A, i: A[i[2], i[1], i[0]]  # noqa: E731

        def ghost(i, gax):
            low = i[gax] == 0
            ib, inn = list(i), list(i)
            ib[gax] = 1 if low else N[gax]
            inn[gax] = 2 if low else N[gax] - 1
            t = get(ids, ib)
            return rule(c.bc_type[t], c.bc_v[a][t], get(lam, ib), get(arr, ib), get(arr, inn))

        for ia in range(1, N[a] + 2):
            for gax, oax in ((b, cc), (cc, b)):
                for side in (0, N[gax] + 1):
                    for io in range(1, N[oax] + 1):
                        i = [0, 0, 0]
                        i[a], i[gax], i[oax] = ia, side, io
                        arr[i[2], i[1], i[0]] = ghost(i, gax)
            for sb in (0, N[b] + 1):
                for sc in (0, N[cc] + 1):
                    i = [0, 0, 0]
                    i[a], i[b], i[cc] = ia, sb, sc
                    j1, j2 = list(i), list(i)
                    j1[cc] = 1 if sc == 0 else N[cc]
                    j2[b] = 1 if sb == 0 else N[b]
                    arr[i[2], i[1], i[0]] = 0.5 * (get(arr, j1) + get(arr, j2))
    gp = [np.zeros(a.shape) for a in c.v]
    for iz in range(1, nz + 2):
        for iy in range(1, ny + 2):
            for ix in range(1, nx + 2):
                gp[0][iz, iy, ix] = (p[iz, iy, ix] - p[iz, iy, ix - 1]) * inv[0]
                gp[1][iz, iy, ix] = (p[iz, iy, ix] - p[iz, iy - 1, ix]) * inv[1]
                gp[2][iz, iy, ix] = (p[iz, iy, ix] - p[iz - 1, iy, ix]) * inv[2]
    return p, tuple(v), tuple(gp)


@pytest.mark.parametrize("spec", [
    dict(N=(7, 6, 5), seed=1, sides=("x+", "z-")),
    dict(N=(8, 8, 6), seed=2, sides=("x-", "y+", "z+"), solid_fraction=0.4),
    dict(N=(5, 7, 4), seed=3, sides=(), lam=False, g=(0.3, 0.0, -9.8)),
])
def test_post_pass_oracle_equals_loop_restatement(oracle_lib, spec):
    c = W.post_case(**spec)
    if spec.get("solid_fraction"):
        assert int((c.ct == W.C_SOLID).sum()) > 0
    p, v, gp = oracle_lib.post_pass(c)
    p2, v2, gp2 = _post_loops(c)
    assert np.array_equal(p, p2)
    for a, b in zip(v + gp, v2 + gp2):
        assert np.array_equal(a, b)
    # only solid and ghost cells change
    changed = p != c.p
    assert not np.any(changed & (c.ct == W.C_INTERIOR))


def test_post_pass_solid_cell_without_fluid_neighbour_gets_zero(oracle_lib):
    c = W.post_case((8, 8, 8), seed=5, sides=(), solid_fraction=0.0)
    c.ct[3:6, 3:6, 3:6] = W.C_SOLID  # the centre (4,4,4) has only solid neighbours
    p, _, _ = oracle_lib.post_pass(c)
    assert p[4, 4, 4] == 0.0
    # a face cell of the block takes its fluid neighbour's value, shifted
    assert p[4, 4, 3] == c.p[4, 4, 2] + c.rho[4, 4, 2] * c.g[0] * c.h[0]


POST_GOLDEN = post_golden_names()


@pytest.mark.skipif(not POST_GOLDEN, reason="no post-projection golden vectors")
@pytest.mark.parametrize("name", POST_GOLDEN)
def test_post_pass_oracle_matches_reference_golden(oracle_lib, name):
    """The oracle against the reference's own update_boundary_ghost +
    make_face_gradp run on the same seeded inputs: every entry bit exact."""
    meta, arr = load_golden(name)
    c = post_case_from_spec(meta)
    p, v, gp = oracle_lib.post_pass(c)
    assert np.array_equal(p, arr["p"])
    for k, a in zip(("vx", "vy", "vz", "gpx", "gpy", "gpz"), v + gp):
        assert np.array_equal(a, arr[k]), k


# ---------------------------------------------------------------------------
# the wall u* rule before the projection (update_vstar_boundary)

def _vstar_loops(c):
    """A second restatement in loops of d_get_v*star_*face
    (CFD/G_BoundaryFunctions.h:369-470)."""
    vs = [a.copy() for a in c.vs]
    N = c.N
    for a in range(3):
        t, ids, m = c.ft[a], c.bcid[a], c.marks[a]
        lam = c.lam[a] if c.lam is not None else np.zeros(t.shape)
        for iz in range(1, N[2] + 2):
            for iy in range(1, N[1] + 2):
                for ix in range(1, N[0] + 2):
                    if t[iz, iy, ix] != W.F_BOUNDARY:
                        continue
                    b = ids[iz, iy, ix]
                    typ = c.bc_type[b]
                    val = 0.0
                    if typ == W.BC_INFLOW:
                        val = (1.0 - lam[iz, iy, ix]) * c.bc_v[a][b]
                    elif typ == W.BC_OUTLET:
                        j = [ix, iy, iz]
                        j[a] += -1 if m[iz, iy, ix] == 2 else 1
                        val = vs[a][j[2], j[1], j[0]]
                    vs[a][iz, iy, ix] = val
    return tuple(vs)


@pytest.mark.parametrize("spec", [
    dict(N=(7, 6, 5), seed=1, sides=("x+", "z-")),
    dict(N=(9, 8, 8), seed=2, sides=("x-", "y+", "z+"), solid_fraction=0.4, solid_margin=3),
    dict(N=(5, 7, 4), seed=3, sides=("y-",), lam=False),
])
def test_vstar_boundary_oracle_equals_loop_restatement(oracle_lib, spec):
    c = W.post_case(**spec)
    got = oracle_lib.vstar_boundary(c.N, c.bc_type, c.bc_v, c.ft, c.bcid, c.marks, c.lam, c.vs)
    want = _vstar_loops(c)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    # interior faces keep u*
    for a, t, v in zip(got, c.ft, c.vs):
        assert np.array_equal(a[t == W.F_INTERIOR], v[t == W.F_INTERIOR])


def test_vstar_boundary_noslip_walls_make_the_neumann_system_compatible(oracle_lib):
    """With no-slip walls the wall u* is 0, so the divergence of u* sums to 0
    over the box (the pure-Neumann system's compatibility condition)."""
    c = W.post_case((10, 9, 8), seed=4, sides=())
    only_noslip = np.zeros(5, np.uint8)
    vs = oracle_lib.vstar_boundary(c.N, only_noslip, c.bc_v, c.ft, c.bcid, None, None, c.vs)
    nx, ny, nz = c.N
    for a, t in zip(vs, c.ft):
        assert np.all(a[t == W.F_BOUNDARY] == 0.0)
    net = (vs[0][1:nz + 1, 1:ny + 1, nx + 1].sum() - vs[0][1:nz + 1, 1:ny + 1, 1].sum()
           + vs[1][1:nz + 1, ny + 1, 1:nx + 1].sum() - vs[1][1:nz + 1, 1, 1:nx + 1].sum()
           + vs[2][nz + 1, 1:ny + 1, 1:nx + 1].sum() - vs[2][1, 1:ny + 1, 1:nx + 1].sum())
    assert net == 0.0


VSTAR_GOLDEN = vstar_golden_names()


@pytest.mark.skipif(not VSTAR_GOLDEN, reason="no update_vstar_boundary golden vectors")
@pytest.mark.parametrize("name", VSTAR_GOLDEN)
def test_vstar_boundary_oracle_matches_reference_golden(oracle_lib, name):
    meta, arr = load_golden(name)
    c = post_case_from_spec(meta)
    got = oracle_lib.vstar_boundary(c.N, c.bc_type, c.bc_v, c.ft, c.bcid, c.marks, c.lam, c.vs)
    for k, a in zip(("vxs", "vys", "vzs"), got):
        assert np.array_equal(a, arr[k]), k


# ---------------------------------------------------------------------------
# the surface-tension force (calc_surface_tension)

def _surface_loops(N, h, alpha, ct, sigma):
    """A second restatement in loops of k_calc_interface_normal,
    k_calc_curvature and k_calc_surface_tension_face
    (CFD/G_SMACSolver_VoF.cu:87-433), from zeroed work arrays."""
    import math
    nx_, ny_, nz_ = N
    sh = W.shapes(N)
    n = [np.zeros(sh["cell"]) for _ in range(3)]
    gm = np.zeros(sh["cell"])
    kap = np.zeros(sh["cell"])
    ih = [1.0 / x for x in h]
    i2h = [1.0 / (2.0 * x) for x in h]
    I = W.C_INTERIOR

    def d(p, m, fp, f0, fm, a):
        if p and m:
            return (fp - fm) * i2h[a]
        if p:
            return (fp - f0) * ih[a]
        if m:
            return (f0 - fm) * ih[a]
        return 0.0

    off = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    for z in range(1, nz_ + 1):
        for y in range(1, ny_ + 1):
            for x in range(1, nx_ + 1):
                if ct[z, y, x] != I:
                    continue
                g = []
                for a, (ox, oy, oz) in enumerate(off):
                    g.append(d(ct[z + oz, y + oy, x + ox] == I, ct[z - oz, y - oy, x - ox] == I,
                               alpha[z + oz, y + oy, x + ox], alpha[z, y, x], alpha[z - oz, y - oy, x - ox], a))
                m2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2]
                m = math.sqrt(m2)
                gm[z, y, x] = m
                for a in range(3):
                    n[a][z, y, x] = g[a] * (1.0 / m) if m2 > 1e-12 else 0.0
    for z in range(1, nz_ + 1):
        for y in range(1, ny_ + 1):
            for x in range(1, nx_ + 1):
                a0 = alpha[z, y, x]
                if a0 > 0.99 or a0 < 0.01:
                    kap[z, y, x] = 0.0
                    continue
                s = []
                for a, (ox, oy, oz) in enumerate(off):
                    okp = ct[z + oz, y + oy, x + ox] == I and gm[z + oz, y + oy, x + ox] > 1e-6
                    okm = ct[z - oz, y - oy, x - ox] == I and gm[z - oz, y - oy, x - ox] > 1e-6
                    s.append(d(okp, okm, n[a][z + oz, y + oy, x + ox], n[a][z, y, x], n[a][z - oz, y - oy, x - ox], a))
                kap[z, y, x] = -1.0 * (s[0] + s[1] + s[2])
    fs = [np.zeros(sh[k]) for k in "xyz"]

    def valid(v):
        return 1e-2 < v < 1 - 1e-2

    for a, (ox, oy, oz) in enumerate(off):
        for z in range(1 + oz, nz_ + 1):
            for y in range(1 + oy, ny_ + 1):
                for x in range(1 + ox, nx_ + 1):
                    if not (ct[z, y, x] == I and ct[z - oz, y - oy, x - ox] == I):
                        continue
                    ap, am = alpha[z, y, x], alpha[z - oz, y - oy, x - ox]
                    kp, km = kap[z, y, x], kap[z - oz, y - oy, x - ox]
                    kf = 0.5 * (kp + km) if valid(ap) and valid(am) else kp if valid(ap) else km if valid(am) else 0.0
                    fs[a][z, y, x] = sigma * kf * (ap - am) * ih[a]
    return (*fs, *n, kap, gm)


@pytest.mark.parametrize("spec", [
    dict(N=(10, 9, 8), seed=3, kind="sphere"),
    dict(N=(9, 8, 7), seed=5, kind="random", solid_fraction=0.15),
])
def test_surface_tension_oracle_equals_loop_restatement(oracle_lib, spec):
    N, h, alpha, ct, sigma = W.surface_case(**spec)
    got = oracle_lib.surface_tension(N, h, alpha, ct, sigma)
    want = _surface_loops(N, h, alpha, ct, sigma)
    for k, a, b in zip(("fsx", "fsy", "fsz", "nx", "ny", "nz", "kappa", "gm"), got, want):
        assert np.array_equal(a, b), k


def test_surface_tension_sphere_curvature_is_two_over_radius(oracle_lib):
    """Known answer: on a resolved sphere the curvature -div n of the cells
    well inside the interface band is 2/R (n points from the outside in, alpha
    being 1 inside), within the discretisation error."""
    n = 48
    N, h = (n, n, n), (1.0 / 32,) * 3
    ext = n * h[0]
    centre, R = (0.5 * ext,) * 3, 0.3 * ext
    alpha = np.ascontiguousarray(W.sphere_alpha(N, h, centre, R, 3.0))
    ct = W.box_types(N)[0]
    _, _, _, _, _, _, kappa, _ = oracle_lib.surface_tension(N, h, alpha, ct, 1.0)
    band = (alpha > 0.3) & (alpha < 0.7)
    k = kappa[band]
    assert abs(np.median(k) - 2.0 / R) < 0.05 * (2.0 / R)


SURFACE_GOLDEN = surface_golden_names()


@pytest.mark.skipif(not SURFACE_GOLDEN, reason="no calc_surface_tension golden vectors")
@pytest.mark.parametrize("name", SURFACE_GOLDEN)
def test_surface_tension_oracle_matches_reference_golden(oracle_lib, name):
    meta, arr = load_golden(name)
    N, h, alpha, ct, sigma = surface_case_from_spec(meta)
    got = oracle_lib.surface_tension(N, h, alpha, ct, sigma)
    for k, a in zip(("fsx", "fsy", "fsz", "nx", "ny", "nz", "kappa", "gm"), got):
        assert np.array_equal(a, arr[k]), k


# ---------------------------------------------------------------------------
# the momentum predictor (get_vof_vstar_rhouu_consistent)

def test_predict_vstar_fluid_at_rest_is_pressure_and_gravity(oracle_lib):
    """Known answer: with u = 0, no advecting flux and zero boundary
    velocities every stress and flux term is 0, so on each F_INTERIOR face
    u* = (1 - s)(f_b (0 + I/V) + dt (f_b (-(p - p_m)/h) + g))."""
    import dataclasses
    m = W.momentum_case((8, 7, 6), seed=4, solid_fraction=0.3)
    zero = lambda arrs: tuple(np.zeros_like(a) for a in arrs)  # noqa: E731
    m = dataclasses.replace(m, v=zero(m.v), mf=zero(m.mf), bc_v=zero(m.bc_v))
    got = oracle_lib.predict_vstar(m)
    inv_vol = (1.0 / m.h[0]) * (1.0 / m.h[1]) * (1.0 / m.h[2])
    for a in range(3):
        t = m.ft[a]
        z, y, x = np.nonzero(t == W.F_INTERIOR)
        cz, cy, cx = z.copy(), y.copy(), x.copy()
        (cx, cy, cz)[a][...] -= 1
        dp = (m.p[z, y, x] - m.p[cz, cy, cx]) * (1.0 / m.h[a])
        tmp = 0.0 - dp
        fb = m.fb[a][z, y, x]
        coup = m.imp[a][z, y, x] * inv_vol
        want = fb * (0.0 * (0.5 * (m.rho_old[z, y, x] + m.rho_old[cz, cy, cx])) + coup) + m.dt * (fb * tmp + m.g[a])
        want = (1.0 - m.sf[a][z, y, x]) * want
        np.testing.assert_array_equal(got[a][z, y, x], want)
        # other faces keep their u*
        np.testing.assert_array_equal(got[a][t != W.F_INTERIOR], m.vs[a][t != W.F_INTERIOR])


MOMENTUM_GOLDEN = momentum_golden_names()


@pytest.mark.skipif(not MOMENTUM_GOLDEN, reason="no momentum-predictor golden vectors")
@pytest.mark.parametrize("name", MOMENTUM_GOLDEN)
def test_predict_vstar_oracle_matches_reference_golden(oracle_lib, name):
    meta, arr = load_golden(name)
    got = oracle_lib.predict_vstar(momentum_case_from_spec(meta))
    for k, a in zip(("vxs", "vys", "vzs"), got):
        assert np.array_equal(a, arr[k]), k


# ---------------------------------------------------------------------------
# the property update (update_properties_by_alpha)

def _oracle_props(O, N, prm, alpha, ct, ft, init):
    """The oracle on the arrays as the call sees them: rho is the array the
    reference's swap makes rho (the former rho_old)."""
    src = dict(init)
    src["rho"] = init["rho_old"]
    return O.update_properties(N, *prm, alpha, ct, ft, src)


def test_update_properties_single_phase_known_answer(oracle_lib):
    """alpha = 0: rho = rho0 and mu = mu0 in every interior, solid-with-fluid
    and ghost cell, f_b = 1/rho0 on F_INTERIOR faces and 0 on the others."""
    N, h, prm, alpha, ct, ft, init = W.property_case((9, 8, 7), seed=3, solid_fraction=0.3)
    out = _oracle_props(oracle_lib, N, prm, np.zeros_like(alpha), ct, ft, init)
    rho0, _, mu0, _ = prm
    fluid_or_ghost = (ct == W.C_INTERIOR) | (ct == W.C_GHOST)
    assert np.all(out["rho"][fluid_or_ghost] == rho0) and np.all(out["mu"][fluid_or_ghost] == mu0)
    for k, t in zip(("fbx", "fby", "fbz"), ft):
        inner = t == W.F_INTERIOR
        assert np.all(out[k][inner] == 1.0 / rho0)
    # a face outside the written range keeps its value
    assert out["fbx"][0, 0, 0] == init["fbx"][0, 0, 0]


PROPERTY_GOLDEN = property_golden_names()


@pytest.mark.skipif(not PROPERTY_GOLDEN, reason="no property-update golden vectors")
@pytest.mark.parametrize("name", PROPERTY_GOLDEN)
def test_update_properties_oracle_matches_reference_golden(oracle_lib, name):
    meta, arr = load_golden(name)
    N, h, prm, alpha, ct, ft, init = property_case_from_spec(meta)
    out = _oracle_props(oracle_lib, N, prm, alpha, ct, ft, init)
    for k in out:
        assert np.array_equal(out[k], arr[k]), k
    assert np.array_equal(arr["rho_old"], init["rho"])  # the swap keeps the previous rho


def test_predict_vstar_two_way_with_unit_void_fraction_is_one_way(oracle_lib):
    """eps_old = eps_new = 1 and f_inv_rho = f_b: every eps weight is exactly
    1, so the two-way u* is the one-way u* up to the association of the last
    update (inv_rho (eps rho u + dt tmp + imp/V) + dt g against
    inv_rho (rho u + imp/V) + dt (inv_rho tmp + g))."""
    import dataclasses
    m = W.momentum_case((10, 9, 8), seed=7, sides=("x+", "y-"), solid_fraction=0.2)
    ones = np.ones(W.shapes(m.N)["cell"])
    m2 = dataclasses.replace(m, eps_old=ones, eps_new=ones, fir=m.fb)
    for a, b in zip(oracle_lib.predict_vstar(m), oracle_lib.predict_vstar(m2)):
        np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-12 * np.abs(a).max())
    # and the weights do act: eps_new = 1/2 changes every predicted face
    m3 = dataclasses.replace(m2, eps_new=0.5 * ones)
    one, half = oracle_lib.predict_vstar(m2), oracle_lib.predict_vstar(m3)
    inner = m.ft[0] == W.F_INTERIOR
    assert np.all(one[0][inner] != half[0][inner])


# ---------------------------------------------------------------------------
# the two-way Poisson coefficients (update_poisson_beta_two_way)

def test_poisson_beta_two_way_known_answer(oracle_lib):
    """eps = 1: f_b = f_inv_rho on the interior box faces, untouched elsewhere;
    eps = 1/2 on one side of a face: f_b = 3/4 f_inv_rho there."""
    N, h, eps, fir, fb = W.beta_two_way_case((6, 5, 4), seed=3)
    ones = np.ones_like(eps)
    out = oracle_lib.poisson_beta_two_way(N, ones, fir, fb)
    nx, ny, nz = N
    box = [(slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 2)), (slice(1, nz + 1), slice(1, ny + 2), slice(1, nx + 1)),
           (slice(1, nz + 2), slice(1, ny + 1), slice(1, nx + 1))]
    for a in range(3):
        assert np.array_equal(out[a][box[a]], fir[a][box[a]])
        keep = np.ones(out[a].shape, bool)
        keep[box[a]] = False
        assert np.array_equal(out[a][keep], fb[a][keep])
    half = ones.copy()
    half[2, 2, 2] = 0.5   # cell (x, y, z) = (2, 2, 2)
    out = oracle_lib.poisson_beta_two_way(N, half, fir, fb)
    assert out[0][2, 2, 2] == 0.75 * fir[0][2, 2, 2] and out[0][2, 2, 3] == 0.75 * fir[0][2, 2, 3]


@pytest.mark.skipif(not beta_golden_names(), reason="no two-way coefficient golden vectors")
@pytest.mark.parametrize("name", beta_golden_names())
def test_poisson_beta_two_way_oracle_matches_reference_golden(oracle_lib, name):
    meta, arr = load_golden(name)
    N, h, eps, fir, fb = beta_case_from_spec(meta)
    for k, a in zip(("fbx", "fby", "fbz"), oracle_lib.poisson_beta_two_way(N, eps, fir, fb)):
        assert np.array_equal(a, arr[k]), k


# ---------------------------------------------------------------------------
# the mass-flux update (compute_mass_flux_from_alpha_flux)

def test_mass_flux_known_answers(oracle_lib):
    """rho0 = rho1 = 1: mf is the face velocity (F drops out), equal to u on
    F_INTERIOR faces; the two-way form with eps_half = 1 equals the one-way
    form on faces 1..N+1 along each axis and is 0 on faces 0 and N+2."""
    import dataclasses
    c = W.mass_flux_case((7, 6, 5), seed=4, sides=("x+", "y-"), solid_fraction=0.2, rho=(1.0, 1.0))
    mf = oracle_lib.mass_flux(c)
    for a in range(3):
        inner = c.mom.ft[a] == W.F_INTERIOR
        assert np.array_equal(mf[a][inner], c.mom.v[a][inner])
    c = W.mass_flux_case((7, 6, 5), seed=4, sides=("x+", "y-"), solid_fraction=0.2)
    one = oracle_lib.mass_flux(c)
    two = oracle_lib.mass_flux(dataclasses.replace(c, eps_half=np.ones(W.shapes(c.mom.N)["cell"])))
    for a in range(3):
        sl = [slice(None)] * 3
        sl[2 - a] = slice(1, c.mom.N[a] + 2)
        assert np.array_equal(two[a][tuple(sl)], one[a][tuple(sl)])
        for edge in (0, c.mom.N[a] + 2):
            sl[2 - a] = edge
            assert np.all(two[a][tuple(sl)] == 0.0)


@pytest.mark.skipif(not flux_golden_names(), reason="no mass-flux golden vectors")
@pytest.mark.parametrize("name", flux_golden_names())
def test_mass_flux_oracle_matches_reference_golden(oracle_lib, name):
    meta, arr = load_golden(name)
    for k, a in zip(("mfx", "mfy", "mfz"), oracle_lib.mass_flux(flux_case_from_spec(meta))):
        assert np.array_equal(a, arr[k]), k


def test_predict_vstar_two_way_fluid_at_rest_known_answer(oracle_lib):
    """Known answer of the two-way form: with u = 0, no advecting flux and
    zero boundary velocities every stress and flux term is 0, so on each
    F_INTERIOR face u* = (1 - s)((f_inv_rho / eps_new_f)(eps_old_f rho_old_f 0
    + dt (0 - eps_old_f (p - p_m) / h) + I/V) + dt g), with the operations in
    the reference's order (CFD/G_SMACSolver.cu:1734-1757)."""
    import dataclasses
    m = W.momentum_case((8, 7, 6), seed=14, solid_fraction=0.3, two_way=True)
    zero = lambda arrs: tuple(np.zeros_like(a) for a in arrs)  # noqa: E731
    m = dataclasses.replace(m, v=zero(m.v), mf=zero(m.mf), bc_v=zero(m.bc_v))
    got = oracle_lib.predict_vstar(m)
    inv_vol = (1.0 / m.h[0]) * (1.0 / m.h[1]) * (1.0 / m.h[2])
    for a in range(3):
        t = m.ft[a]
        z, y, x = np.nonzero(t == W.F_INTERIOR)
        cz, cy, cx = z.copy(), y.copy(), x.copy()
        (cx, cy, cz)[a][...] -= 1
        eo = 0.5 * (m.eps_old[cz, cy, cx] + m.eps_old[z, y, x])
        en = 0.5 * (m.eps_new[cz, cy, cx] + m.eps_new[z, y, x])
        tmp = 0.0 - (eo * (m.p[z, y, x] - m.p[cz, cy, cx])) * (1.0 / m.h[a])
        rho_f = 0.5 * (m.rho_old[z, y, x] + m.rho_old[cz, cy, cx])
        coup = m.imp[a][z, y, x] * inv_vol
        want = (m.fir[a][z, y, x] / en) * ((eo * rho_f) * 0.0 + m.dt * tmp + coup) + m.dt * m.g[a]
        want = (1.0 - m.sf[a][z, y, x]) * want
        np.testing.assert_array_equal(got[a][z, y, x], want)
        np.testing.assert_array_equal(got[a][t != W.F_INTERIOR], m.vs[a][t != W.F_INTERIOR])


def _props_passes_numpy(N, rho0, rho1, mu0, mu1, alpha, ct, ft, init):
    """The reference's property passes one after another, in numpy
    (CFD/G_SMACSolver_VoF.cu:1244-1535): mixing on C_INTERIOR /
    C_NEAR_BOUNDARY cells 1..N+1, the solid rule on interior C_SOLID cells
    (first C_INTERIOR neighbour x-, x+, y-, y+, z-, z+, else 0), ghost cells
    from the nearest interior cell, then the faces."""
    nx, ny, nz = N
    out = {k: np.array(v, copy=True) for k, v in init.items()}
    rho, inv, mu = out["rho"], out["inv_rho"], out["mu"]
    box = (slice(1, nz + 2), slice(1, ny + 2), slice(1, nx + 2))
    mix = (ct[box] == 0) | (ct[box] == 1)
    a = alpha[box]
    r = (1.0 - a) * rho0 + a * rho1
    rho[box] = np.where(mix, r, rho[box])
    inv[box] = np.where(mix, 1.0 / r, inv[box])
    mu[box] = np.where(mix, (1.0 - a) * mu0 + a * mu1, mu[box])
    r1, m1 = rho.copy(), mu.copy()
    for z in range(1, nz + 1):
        for y in range(1, ny + 1):
            for x in range(1, nx + 1):
                if ct[z, y, x] != 3:
                    continue
                rho[z, y, x] = mu[z, y, x] = 0.0
                for dz, dy, dx in ((0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)):
                    if ct[z + dz, y + dy, x + dx] == 0:
                        rho[z, y, x], mu[z, y, x] = r1[z + dz, y + dy, x + dx], m1[z + dz, y + dy, x + dx]
                        break
    for z in range(nz + 2):
        for y in range(ny + 2):
            for x in range(nx + 2):
                if 0 < x <= nx and 0 < y <= ny and 0 < z <= nz:
                    continue
                s = (min(max(z, 1), nz), min(max(y, 1), ny), min(max(x, 1), nx))
                rho[z, y, x], mu[z, y, x] = rho[s], mu[s]
    for k, ax in enumerate("xyz"):
        t = ft[k]
        lo = [slice(1, nz + 2), slice(1, ny + 2), slice(1, nx + 2)]
        lo[2 - k] = slice(1, (nz, ny, nx)[2 - k] + 3)
        lo = tuple(lo)
        hi = [slice(1, nz + 2), slice(1, ny + 2), slice(1, nx + 2)]
        mlo = [slice(1, nz + 2), slice(1, ny + 2), slice(1, nx + 2)]
        mlo[2 - k] = slice(0, (nz, ny, nx)[2 - k] + 1)
        inner = t[tuple(hi)] == 0
        fr = 0.5 * (rho[tuple(hi)] + rho[tuple(mlo)])
        fm = 0.5 * (mu[tuple(hi)] + mu[tuple(mlo)])
        for key in ("fb", "fir"):
            out[key + ax][lo] = 0.0
        out["fb" + ax][tuple(hi)] = np.where(inner, 1.0 / fr, 0.0)
        out["fir" + ax][tuple(hi)] = np.where(inner, 1.0 / fr, 0.0)
        out["rho" + ax][tuple(hi)] = np.where(inner, fr, out["rho" + ax][tuple(hi)])
        out["mu" + ax][tuple(hi)] = np.where(inner, fm, out["mu" + ax][tuple(hi)])
    return out


def test_update_properties_oracle_matches_passes_with_near_boundary_cells(oracle_lib):
    """Cells of all four types (C_NEAR_BOUNDARY and isolated C_SOLID cells
    included): the oracle equals the reference's passes run in order."""
    N, h, prm, alpha, ct, ft, init = W.property_case((7, 6, 5), seed=31, solid_fraction=0.25, mixed_types=True)
    inside = ct[1:-1, 1:-1, 1:-1]
    assert (inside == 1).sum() > 20 and (inside == W.C_SOLID).sum() > 20
    src = dict(init)
    src["rho"] = init["rho_old"]
    got = oracle_lib.update_properties(N, *prm, alpha, ct, ft, src)
    want = _props_passes_numpy(N, *prm, alpha, ct, ft, {k: src[k] for k in got})
    for k in got:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
