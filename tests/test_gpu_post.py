"""The calls either side of the projection on the GPU: before it the
momentum predictor (smac_predict_vstar), the wall u* rule
(smac_update_vstar_boundary) and the surface-tension force
(smac_surface_tension), after it the pass over p
(smac_update_pressure_ghost, smac_update_velocity_ghost, smac_face_gradp),
against the oracle and the reference.

Every output is element-wise arithmetic of the inputs, so the bar is bit
equality: with the oracle on seeded inputs (small and 256^3), with the
golden vectors of the reference's own update_boundary_ghost +
make_face_gradp, and with the reference library itself where it is built.
"""
import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.solver import (BoundaryConditions, DeviceGrid, SMACStep, face_gradp_device, predict_vstar_device,
                                  mass_flux_device, poisson_beta_two_way_device, surface_tension_device,
                                  update_pressure_ghost_device, update_properties_device,
                                  update_velocity_ghost_device, update_vstar_boundary_device)
from oracle import oracle as O
from oracle import ref as REF

from _cases import (beta_case_from_spec, beta_golden_names, flux_case_from_spec, flux_golden_names, load_golden, momentum_case_from_spec, momentum_golden_names, post_case_from_spec,
                    post_golden_names, property_case_from_spec, property_golden_names, surface_case_from_spec,
                    surface_golden_names, vstar_golden_names)

pytestmark = pytest.mark.gpu


def _cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _misaligned(a, offset=3):
    """A contiguous CUDA copy of uint8 array a whose data pointer is not 16-byte aligned."""
    buf = torch.zeros(a.size + 32, dtype=torch.uint8, device="cuda")
    t = buf[offset:offset + a.size].view(a.shape)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
    assert t.data_ptr() % 16 != 0
    return t


def run_post(c, misaligned=False):
    """The three calls on device copies of a workloads.PostCase."""
    u8 = _misaligned if misaligned else _cuda
    p = _cuda(c.p)
    v = [_cuda(a) for a in c.v]
    gp = [torch.zeros(a.shape, dtype=torch.float64, device="cuda") for a in c.v]
    update_pressure_ghost_device(c.N, c.h, u8(c.ct), _cuda(c.rho), c.g, p)
    bc = BoundaryConditions(c.bc_type, *c.bc_v)
    update_velocity_ghost_device(c.N, c.h, bc, [u8(a) for a in c.bcid], [u8(a) for a in c.marks],
                                 None if c.lam is None else [_cuda(a) for a in c.lam], [_cuda(a) for a in c.vs],
                                 [_cuda(a) for a in c.fb], _cuda(c.p_delta), c.dt, v)
    face_gradp_device(c.N, c.h, p, gp)
    torch.cuda.synchronize()
    return p.cpu().numpy(), tuple(a.cpu().numpy() for a in v), tuple(a.cpu().numpy() for a in gp)


def _assert_equal(got, want):
    p, v, gp = got
    p2, v2, gp2 = want
    assert np.array_equal(p, p2)
    for k, a, b in zip(("vx", "vy", "vz", "gpx", "gpy", "gpz"), v + gp, v2 + gp2):
        assert np.array_equal(a, b), k


@pytest.mark.parametrize("spec,misaligned", [
    (dict(N=(12, 10, 8), seed=1, sides=("x+", "z-")), False),
    (dict(N=(16, 16, 16), seed=2, sides=("x-", "y+"), solid_fraction=0.35), False),
    (dict(N=(9, 7, 11), seed=3, sides=("x+", "y-", "z+"), lam=False, g=(0.3, 0.0, -9.8)), True),
    (dict(N=(33, 17, 2), seed=4, sides=("z+",), solid_fraction=0.2), True),
])
def test_post_pass_bit_exact_against_oracle(spec, misaligned):
    c = W.post_case(**spec)
    _assert_equal(run_post(c, misaligned), O.post_pass(c))


@pytest.mark.parametrize("name", post_golden_names())
def test_post_pass_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    c = post_case_from_spec(meta)
    want = (arr["p"], (arr["vx"], arr["vy"], arr["vz"]), (arr["gpx"], arr["gpy"], arr["gpz"]))
    _assert_equal(run_post(c), want)


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_post_pass_bit_exact_against_reference_library():
    c = W.post_case((24, 20, 16), seed=9, sides=("x+", "y-", "z-"), solid_fraction=0.3, g=(0.5, -1.0, -9.8))
    r = REF.post(c)
    _assert_equal(run_post(c), (r["p"], (r["vx"], r["vy"], r["vz"]), (r["gpx"], r["gpy"], r["gpz"])))


def test_post_pass_256_bit_exact_and_gradp_bandwidth():
    c = W.post_case((256, 256, 256), seed=6, sides=("x+", "z-"), solid_fraction=0.05)
    _assert_equal(run_post(c), O.post_pass(c))
    # face gradient: p read once, three face arrays written
    p = _cuda(c.p)
    gp = [torch.empty(a.shape, dtype=torch.float64, device="cuda") for a in c.v]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(8):
        flush.fill_(1)
        torch.cuda._sleep(400000)  # the host's call overhead stays outside the events
        e0.record()
        face_gradp_device(c.N, c.h, p, gp)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = sorted(times)[len(times) // 2]
    n = 257 ** 3
    alg = 8.0 * (258 ** 3 + 3 * n)
    print(f"face_gradp 256^3: {ms * 1e3:.1f} us, {alg / ms / 1e6:.0f} GB/s algorithmic")
    assert ms < 1.0


def _device_ms(fn, reps=8):
    """Median device time of fn's launches, replayed from a CUDA graph so
    that no host time falls between them (CUDA events, L2 flushed before
    each replay)."""
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        fn()
    ts = []
    for _ in range(reps):
        flush.fill_(1)
        torch.cuda._sleep(400000)
        e0.record()
        graph.replay()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return sorted(ts)[len(ts) // 2]


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_post_pass_against_reference_time_256():
    """update_boundary_ghost and make_face_gradp: this library's calls against
    the reference's own kernels on the same 256^3 inputs, device time."""
    c = W.post_case((256, 256, 256), seed=7, sides=("x+",), solid_fraction=0.05)
    REF.post(c)  # loads the reference's kernels
    r = REF.post(c)
    p = _cuda(c.p)
    v = [_cuda(a) for a in c.v]
    gp = [torch.zeros(a.shape, dtype=torch.float64, device="cuda") for a in c.v]
    ct, rho = _cuda(c.ct), _cuda(c.rho)
    bcid, marks = [_cuda(a) for a in c.bcid], [_cuda(a) for a in c.marks]
    lam, vs, fb, pd = [_cuda(a) for a in c.lam], [_cuda(a) for a in c.vs], [_cuda(a) for a in c.fb], _cuda(c.p_delta)
    bc = BoundaryConditions(c.bc_type, *c.bc_v)

    def ghost():
        update_pressure_ghost_device(c.N, c.h, ct, rho, c.g, p)
        update_velocity_ghost_device(c.N, c.h, bc, bcid, marks, lam, vs, fb, pd, c.dt, v)

    ms_ghost = _device_ms(ghost)
    ms_gradp = _device_ms(lambda: face_gradp_device(c.N, c.h, p, gp))
    print(f"update_boundary_ghost 256^3: {ms_ghost * 1e3:.1f} us (reference {r['ghost_ms'] * 1e3:.1f} us); "
          f"make_face_gradp: {ms_gradp * 1e3:.1f} us (reference {r['gradp_ms'] * 1e3:.1f} us)")
    assert ms_ghost + ms_gradp < r["ghost_ms"] + r["gradp_ms"]


def test_smac_step_post_calls_match_oracle():
    """SMACStep.update_boundary_ghost + make_face_gradp on a DeviceGrid."""
    c = W.post_case((20, 16, 12), seed=8, sides=("y+",), solid_fraction=0.2, g=(0.0, 0.0, -9.8))
    sh = W.shapes(c.N)
    g = DeviceGrid(*c.N, *c.h, *(_cuda(a) for a in c.vs), *(_cuda(a) for a in c.fb), *(_cuda(a) for a in c.fb),
                   _cuda(c.ct), *(_cuda(a) for a in c.ft), _cuda(c.p), _cuda(c.p_delta),
                   torch.zeros(sh["cell"], dtype=torch.float64, device="cuda"), *(_cuda(a) for a in c.v))
    g.rho_ = _cuda(c.rho)
    g.f_xbcid_, g.f_ybcid_, g.f_zbcid_ = (_cuda(a) for a in c.bcid)
    g.f_xoutlet_, g.f_youtlet_, g.f_zoutlet_ = (_cuda(a) for a in c.marks)
    g.f_ibm_area_solid_fraction_x_, g.f_ibm_area_solid_fraction_y_, g.f_ibm_area_solid_fraction_z_ = (
        _cuda(a) for a in c.lam)
    step = SMACStep(g, c.dt, g=c.g, bc=BoundaryConditions(c.bc_type, *c.bc_v))
    step.update_boundary_ghost()
    step.make_face_gradp()
    torch.cuda.synchronize()
    got = (g.p_.cpu().numpy(), tuple(a.cpu().numpy() for a in (g.f_vx_, g.f_vy_, g.f_vz_)),
           tuple(a.cpu().numpy() for a in (g.f_gradp_x_, g.f_gradp_y_, g.f_gradp_z_)))
    _assert_equal(got, O.post_pass(c))


def test_velocity_ghost_refuses_single_cell_extent():
    c = W.post_case((4, 4, 4), seed=1)
    bc = BoundaryConditions(c.bc_type, *c.bc_v)
    v = [_cuda(a) for a in c.v]
    with pytest.raises(nat.SmacError):
        update_velocity_ghost_device((4, 1, 4), c.h, bc, [_cuda(a) for a in c.bcid], None, None, (None,) * 3,
                                     (None,) * 3, None, c.dt, v)


def run_vstar(c, misaligned=False):
    u8 = _misaligned if misaligned else _cuda
    vs = [_cuda(a) for a in c.vs]
    update_vstar_boundary_device(c.N, c.h, BoundaryConditions(c.bc_type, *c.bc_v), [u8(a) for a in c.ft],
                                 [u8(a) for a in c.bcid], [u8(a) for a in c.marks],
                                 None if c.lam is None else [_cuda(a) for a in c.lam], vs)
    torch.cuda.synchronize()
    return tuple(a.cpu().numpy() for a in vs)


@pytest.mark.parametrize("spec,misaligned", [
    (dict(N=(12, 10, 8), seed=1, sides=("x+", "z-")), False),
    (dict(N=(16, 16, 16), seed=2, sides=("x-", "y+"), solid_fraction=0.35, solid_margin=3), True),
    (dict(N=(33, 17, 5), seed=4, sides=("z+", "x-"), lam=False, solid_fraction=0.2, solid_margin=3), True),
])
def test_vstar_boundary_bit_exact_against_oracle(spec, misaligned):
    c = W.post_case(**spec)
    want = O.vstar_boundary(c.N, c.bc_type, c.bc_v, c.ft, c.bcid, c.marks, c.lam, c.vs)
    for a, b in zip(run_vstar(c, misaligned), want):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", vstar_golden_names())
def test_vstar_boundary_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    c = post_case_from_spec(meta)
    for k, a in zip(("vxs", "vys", "vzs"), run_vstar(c)):
        assert np.array_equal(a, arr[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_vstar_boundary_against_reference_library_and_time_256():
    c = W.post_case((256, 256, 256), seed=5, sides=("x+", "z-"), solid_fraction=0.05, solid_margin=3)
    REF.vstar(c)  # loads the reference's kernels
    *ref, ref_ms = REF.vstar(c)
    for a, b in zip(run_vstar(c), ref):
        assert np.array_equal(a, b)
    vs = [_cuda(a) for a in c.vs]
    args = (c.N, c.h, BoundaryConditions(c.bc_type, *c.bc_v), [_cuda(a) for a in c.ft], [_cuda(a) for a in c.bcid],
            [_cuda(a) for a in c.marks], [_cuda(a) for a in c.lam], vs)
    ms = _device_ms(lambda: update_vstar_boundary_device(*args))
    print(f"update_vstar_boundary 256^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


ST_KEYS = ("fsx", "fsy", "fsz", "nx", "ny", "nz", "kappa", "gm")


def run_surface(N, h, alpha, ct, sigma, work=None):
    sh = W.shapes(N)
    work = [torch.zeros(sh["cell"], dtype=torch.float64, device="cuda") for _ in range(5)] if work is None else \
        [_cuda(a) for a in work]
    fs = [torch.full(sh[k], np.nan, dtype=torch.float64, device="cuda") for k in "xyz"]
    surface_tension_device(N, h, _cuda(alpha), _cuda(ct), sigma, work, fs)
    torch.cuda.synchronize()
    return tuple(a.cpu().numpy() for a in fs + work)


@pytest.mark.parametrize("spec", [
    dict(N=(24, 24, 24), seed=3, kind="sphere"),
    dict(N=(20, 16, 12), seed=5, kind="random", solid_fraction=0.15),
    dict(N=(37, 19, 23), seed=7, kind="sphere", solid_fraction=0.1),
])
def test_surface_tension_bit_exact_against_oracle(spec):
    N, h, alpha, ct, sigma = W.surface_case(**spec)
    # work arrays with prior contents: cells the reference does not write keep them
    sh = W.shapes(N)
    work = [W.uniform_pm1(900 + k, int(np.prod(sh["cell"]))).reshape(sh["cell"]) for k in range(5)]
    got = run_surface(N, h, alpha, ct, sigma, work)
    want = O.surface_tension(N, h, alpha, ct, sigma, *work)
    for k, a, b in zip(ST_KEYS, got, want):
        assert np.array_equal(a, b), k


@pytest.mark.parametrize("name", surface_golden_names())
def test_surface_tension_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    got = run_surface(*surface_case_from_spec(meta))
    for k, a in zip(ST_KEYS, got):
        assert np.array_equal(a, arr[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_surface_tension_against_reference_library_and_time_192():
    N, h, alpha, ct, sigma = W.surface_case((192, 192, 192), seed=4, kind="sphere", solid_fraction=0.02)
    REF.surface_tension(N, h, alpha, ct, sigma)  # loads the reference's kernels
    *ref, ref_ms = REF.surface_tension(N, h, alpha, ct, sigma)
    got = run_surface(N, h, alpha, ct, sigma)
    for k, a, b in zip(ST_KEYS, got, ref):
        assert np.array_equal(a, b), k
    sh = W.shapes(N)
    work = [torch.zeros(sh["cell"], dtype=torch.float64, device="cuda") for _ in range(5)]
    fs = [torch.zeros(sh[k], dtype=torch.float64, device="cuda") for k in "xyz"]
    a_d, ct_d = _cuda(alpha), _cuda(ct)
    ms = _device_ms(lambda: surface_tension_device(N, h, a_d, ct_d, sigma, work, fs))
    print(f"calc_surface_tension 192^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


def _momentum_fields(m):
    f = {}
    for k, ax in enumerate("xyz"):
        f["f" + ax + "t"] = _cuda(m.ft[k])
        f["f" + ax + "bcid"] = _cuda(m.bcid[k])
        f["v" + ax] = _cuda(m.v[k])
        f["mf" + ax] = _cuda(m.mf[k])
        f["mu" + ax] = _cuda(m.muf[k])
        f["fb" + ax] = _cuda(m.fb[k])
        if m.lam is not None:
            f["lam" + ax] = _cuda(m.lam[k])
        if m.imp is not None:
            f["imp" + ax] = _cuda(m.imp[k])
        if m.sf is not None:
            f["sf" + ax] = _cuda(m.sf[k])
    f["mu"], f["rho_old"], f["p"] = _cuda(m.mu), _cuda(m.rho_old), _cuda(m.p)
    return f


def _two_way_fields(m):
    if m.eps_old is None:
        return None
    f = {"eps_old": _cuda(m.eps_old), "eps_new": _cuda(m.eps_new)}
    for k, ax in enumerate("xyz"):
        f["inv_rho" + ax] = _cuda(m.fir[k])
    return f


def run_predict(m):
    vs = [_cuda(a) for a in m.vs]
    predict_vstar_device(m.N, m.h, BoundaryConditions(m.bc_type, *m.bc_v), _momentum_fields(m), m.dt, m.g, vs,
                         two_way=_two_way_fields(m))
    torch.cuda.synchronize()
    return tuple(a.cpu().numpy() for a in vs)


@pytest.mark.parametrize("spec", [
    dict(N=(12, 10, 8), seed=1, sides=("x+", "z-")),
    dict(N=(16, 16, 16), seed=2, sides=("x-", "y+"), solid_fraction=0.3),
    dict(N=(9, 7, 11), seed=3, sides=("y-",), extras=False),
    dict(N=(33, 18, 20), seed=5, sides=("x-", "x+", "z+"), solid_fraction=0.2),
    dict(N=(12, 10, 8), seed=4, sides=("x+", "z-"), two_way=True),
    dict(N=(17, 14, 19), seed=6, sides=("y-", "z+"), solid_fraction=0.25, two_way=True),
    dict(N=(9, 7, 11), seed=8, sides=("x-",), extras=False, two_way=True),
])
def test_predict_vstar_bit_exact_against_oracle(spec):
    m = W.momentum_case(**spec)
    for k, a, b in zip(("vxs", "vys", "vzs"), run_predict(m), O.predict_vstar(m)):
        assert np.array_equal(a, b), k


@pytest.mark.parametrize("name", momentum_golden_names())
def test_predict_vstar_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    for k, a in zip(("vxs", "vys", "vzs"), run_predict(momentum_case_from_spec(meta))):
        assert np.array_equal(a, arr[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_predict_vstar_against_reference_library_128_and_time_256():
    m = W.momentum_case((128, 128, 128), seed=6, sides=("x+", "z-"), solid_fraction=0.05)
    *ref, _ = REF.predict_vstar(m)
    for k, a, b in zip(("vxs", "vys", "vzs"), run_predict(m), ref):
        assert np.array_equal(a, b), k
    m = W.momentum_case((256, 256, 256), seed=7, sides=("x+",), solid_fraction=0.02)
    REF.predict_vstar(m)  # loads the reference's kernels
    *_, ref_ms = REF.predict_vstar(m)
    fields = _momentum_fields(m)
    vs = [_cuda(a) for a in m.vs]
    bc = BoundaryConditions(m.bc_type, *m.bc_v)
    ms = _device_ms(lambda: predict_vstar_device(m.N, m.h, bc, fields, m.dt, m.g, vs))
    print(f"get_vof_vstar_rhouu_consistent 256^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


def test_smac_step_predictor_and_surface_tension_match_oracle():
    """SMACStep.get_vof_vstar_rhouu_consistent and calc_surface_tension on a
    DeviceGrid, against the oracle."""
    m = W.momentum_case((14, 12, 10), seed=9, sides=("x+",), solid_fraction=0.2)
    sh = W.shapes(m.N)
    zc = lambda: torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")  # noqa: E731
    g = DeviceGrid(*m.N, *m.h, *(_cuda(a) for a in m.vs), *(_cuda(a) for a in m.fb), *(_cuda(a) for a in m.fb),
                   _cuda(m.ct), *(_cuda(a) for a in m.ft), _cuda(m.p), zc(), zc(), *(_cuda(a) for a in m.v))
    g.f_xbcid_, g.f_ybcid_, g.f_zbcid_ = (_cuda(a) for a in m.bcid)
    g.f_ibm_area_solid_fraction_x_, g.f_ibm_area_solid_fraction_y_, g.f_ibm_area_solid_fraction_z_ = (
        _cuda(a) for a in m.lam)
    g.f_mfx_, g.f_mfy_, g.f_mfz_ = (_cuda(a) for a in m.mf)
    g.f_mux_, g.f_muy_, g.f_muz_ = (_cuda(a) for a in m.muf)
    g.mu_, g.rho_old_ = _cuda(m.mu), _cuda(m.rho_old)
    g.f_coupling_impulse_x_, g.f_coupling_impulse_y_, g.f_coupling_impulse_z_ = (_cuda(a) for a in m.imp)
    g.f_ibm_solid_fraction_x_, g.f_ibm_solid_fraction_y_, g.f_ibm_solid_fraction_z_ = (_cuda(a) for a in m.sf)
    step = SMACStep(g, m.dt, g=m.g, bc=BoundaryConditions(m.bc_type, *m.bc_v))
    step.get_vof_vstar_rhouu_consistent()
    torch.cuda.synchronize()
    for a, b in zip((g.f_vx_star_, g.f_vy_star_, g.f_vz_star_), O.predict_vstar(m)):
        assert np.array_equal(a.cpu().numpy(), b)
    N, h, alpha, ct, sigma = W.surface_case(m.N, seed=9, kind="sphere", h=m.h[0])
    g.alpha_ = _cuda(alpha)
    g.celltype_ = _cuda(ct)
    step.calc_surface_tension(sigma)
    torch.cuda.synchronize()
    want = O.surface_tension(N, h, alpha, ct, sigma)
    got = (g.f_sx_, g.f_sy_, g.f_sz_, g.nx_, g.ny_, g.nz_, g.kappa_, g.p_tmp_)
    for k, a, b in zip(("fsx", "fsy", "fsz", "nx", "ny", "nz", "kappa", "gm"), got, want):
        assert np.array_equal(a.cpu().numpy(), b), k


ANISO = (0.03125, 0.0625, 0.015625)  # powers of two: the reference's (N h) / N is exact


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_anisotropic_spacing_bit_exact_against_reference_library():
    """The calls around the projection with hx != hy != hz, against the
    reference's kernels directly: predictor, surface tension, wall u* rule,
    ghost/gradient pass."""
    m = W.momentum_case((24, 20, 16), seed=11, sides=("x-", "z+"), solid_fraction=0.2, h=ANISO)
    *ref, _ = REF.predict_vstar(m)
    for k, a, b in zip(("vxs", "vys", "vzs"), run_predict(m), ref):
        assert np.array_equal(a, b), k
    N, h, alpha, ct, sigma = W.surface_case((20, 16, 24), seed=12, kind="sphere", solid_fraction=0.05, h=ANISO)
    *ref, _ = REF.surface_tension(N, h, alpha, ct, sigma)
    for k, a, b in zip(ST_KEYS, run_surface(N, h, alpha, ct, sigma), ref):
        assert np.array_equal(a, b), k
    c = W.post_case((18, 22, 14), seed=13, h=ANISO, sides=("y+", "z-"), solid_fraction=0.2, solid_margin=3)
    r = REF.post(c)
    _assert_equal(run_post(c), (r["p"], (r["vx"], r["vy"], r["vz"]), (r["gpx"], r["gpy"], r["gpz"])))
    *ref, _ = REF.vstar(c)
    for k, a, b in zip(("vxs", "vys", "vzs"), run_vstar(c), ref):
        assert np.array_equal(a, b), k


# ---------------------------------------------------------------------------
# the property update (update_properties_by_alpha)

def _prop_tensors(init):
    """CUDA copies of the arrays before the call, after the reference's
    swap: the array written as rho is the former rho_old."""
    t = {k: _cuda(v) for k, v in init.items() if k not in ("rho", "rho_old")}
    t["rho"] = _cuda(init["rho_old"])
    return t


def run_props(N, h, prm, alpha, ct, ft, init):
    t = _prop_tensors(init)
    update_properties_device(N, h, *prm, _cuda(alpha), _cuda(ct), tuple(_cuda(a) for a in ft), t)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in t.items()}


def _oracle_props(N, prm, alpha, ct, ft, init):
    src = dict(init)
    src["rho"] = init["rho_old"]
    return O.update_properties(N, *prm, alpha, ct, ft, src)


@pytest.mark.parametrize("spec", [
    dict(N=(12, 10, 8), seed=1),
    dict(N=(16, 16, 16), seed=2, solid_fraction=0.35),
    dict(N=(33, 18, 20), seed=5, solid_fraction=0.2),
    dict(N=(1, 7, 5), seed=8, solid_fraction=0.1),
    dict(N=(19, 14, 11), seed=31, solid_fraction=0.25, mixed_types=True),
])
def test_update_properties_bit_exact_against_oracle(spec):
    N, h, prm, alpha, ct, ft, init = W.property_case(**spec)
    got = run_props(N, h, prm, alpha, ct, ft, init)
    want = _oracle_props(N, prm, alpha, ct, ft, init)
    for k in want:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.parametrize("name", property_golden_names())
def test_update_properties_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    N, h, prm, alpha, ct, ft, init = property_case_from_spec(meta)
    got = run_props(N, h, prm, alpha, ct, ft, init)
    for k in got:
        assert np.array_equal(got[k], arr[k]), k


def test_update_properties_optional_outputs_left_alone():
    """inv_rho, f_inv_rho* and f_rho* may be absent: the others are written as before."""
    N, h, prm, alpha, ct, ft, init = W.property_case((14, 9, 11), seed=9, solid_fraction=0.2)
    t = _prop_tensors(init)
    for k in ("inv_rho", "firx", "firy", "firz", "rhox", "rhoy", "rhoz"):
        del t[k]
    update_properties_device(N, h, *prm, _cuda(alpha), _cuda(ct), tuple(_cuda(a) for a in ft), t)
    want = _oracle_props(N, prm, alpha, ct, ft, init)
    for k, v in t.items():
        assert np.array_equal(v.cpu().numpy(), want[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_update_properties_against_reference_library_and_time_256():
    case = W.property_case((96, 80, 72), seed=11, solid_fraction=0.1)
    N, h, prm, alpha, ct, ft, init = case
    ref, _ = REF.update_properties(N, h, *prm, alpha, ct, ft, init)
    got = run_props(*case)
    for k in got:
        assert np.array_equal(got[k], ref[k]), k
    N, h, prm, alpha, ct, ft, init = W.property_case((256, 256, 256), seed=12, solid_fraction=0.02)
    REF.update_properties(N, h, *prm, alpha, ct, ft, init)  # loads the reference's kernels
    _, ref_ms = REF.update_properties(N, h, *prm, alpha, ct, ft, init)
    t = _prop_tensors(init)
    a, c, f = _cuda(alpha), _cuda(ct), tuple(_cuda(x) for x in ft)
    ms = _device_ms(lambda: update_properties_device(N, h, *prm, a, c, f, t))
    print(f"update_properties_by_alpha 256^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


def test_smac_step_update_properties_swaps_and_matches_oracle():
    N, h, prm, alpha, ct, ft, init = W.property_case((20, 12, 16), seed=13, solid_fraction=0.25)
    c = W.post_case(N, 13, sides=())
    sh = W.shapes(N)
    zc = lambda: torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")  # noqa: E731
    g = DeviceGrid(*N, *h, *(_cuda(a) for a in c.vs), *(_cuda(a) for a in c.fb), *(_cuda(a) for a in c.fb),
                   _cuda(ct), *(_cuda(a) for a in ft), _cuda(c.p), zc(), zc(), *(_cuda(a) for a in c.v))
    g.alpha_ = _cuda(alpha)
    g.rho_, g.rho_old_, g.inv_rho_, g.mu_ = (_cuda(init[k]) for k in ("rho", "rho_old", "inv_rho", "mu"))
    for ax in "xyz":
        setattr(g, f"f_b{ax}_", _cuda(init["fb" + ax]))
        setattr(g, f"f_inv_rho{ax}_", _cuda(init["fir" + ax]))
        setattr(g, f"f_rho{ax}_", _cuda(init["rho" + ax]))
        setattr(g, f"f_mu{ax}_", _cuda(init["mu" + ax]))
    prev_rho = g.rho_
    SMACStep(g).update_properties_by_alpha(*prm)
    torch.cuda.synchronize()
    assert g.rho_old_ is prev_rho and np.array_equal(g.rho_old_.cpu().numpy(), init["rho"])
    want = _oracle_props(N, prm, alpha, ct, ft, init)
    got = {"rho": g.rho_, "inv_rho": g.inv_rho_, "mu": g.mu_}
    for ax in "xyz":
        got.update({"fb" + ax: getattr(g, f"f_b{ax}_"), "fir" + ax: getattr(g, f"f_inv_rho{ax}_"),
                    "rho" + ax: getattr(g, f"f_rho{ax}_"), "mu" + ax: getattr(g, f"f_mu{ax}_")})
    for k, v in got.items():
        assert np.array_equal(v.cpu().numpy(), want[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_predict_vstar_two_way_against_reference_library_128_and_time_256():
    """The two-way-coupled predictor (get_vof_vstar_rhouu_consistent_two_way)
    against the reference's own three kernels: bit for bit at 128^3, faster at
    256^3."""
    m = W.momentum_case((128, 128, 128), seed=16, sides=("x+", "z-"), solid_fraction=0.05, two_way=True)
    *ref, _ = REF.predict_vstar(m)
    for k, a, b in zip(("vxs", "vys", "vzs"), run_predict(m), ref):
        assert np.array_equal(a, b), k
    m = W.momentum_case((256, 256, 256), seed=17, sides=("x+",), solid_fraction=0.02, two_way=True)
    REF.predict_vstar(m)  # loads the reference's kernels
    *_, ref_ms = REF.predict_vstar(m)
    fields, tw = _momentum_fields(m), _two_way_fields(m)
    vs = [_cuda(a) for a in m.vs]
    bc = BoundaryConditions(m.bc_type, *m.bc_v)
    ms = _device_ms(lambda: predict_vstar_device(m.N, m.h, bc, fields, m.dt, m.g, vs, two_way=tw))
    print(f"get_vof_vstar_rhouu_consistent_two_way 256^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


def test_smac_step_two_way_predictor_matches_oracle():
    """SMACStep.get_vof_vstar_rhouu_consistent_two_way on a DeviceGrid."""
    m = W.momentum_case((14, 12, 10), seed=19, sides=("x+",), solid_fraction=0.2, two_way=True)
    sh = W.shapes(m.N)
    zc = lambda: torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")  # noqa: E731
    g = DeviceGrid(*m.N, *m.h, *(_cuda(a) for a in m.vs), *(_cuda(a) for a in m.fb), *(_cuda(a) for a in m.fir),
                   _cuda(m.ct), *(_cuda(a) for a in m.ft), _cuda(m.p), zc(), zc(), *(_cuda(a) for a in m.v))
    g.void_fraction_old_, g.void_fraction_ = _cuda(m.eps_old), _cuda(m.eps_new)
    g.f_xbcid_, g.f_ybcid_, g.f_zbcid_ = (_cuda(a) for a in m.bcid)
    g.f_ibm_area_solid_fraction_x_, g.f_ibm_area_solid_fraction_y_, g.f_ibm_area_solid_fraction_z_ = (
        _cuda(a) for a in m.lam)
    g.f_mfx_, g.f_mfy_, g.f_mfz_ = (_cuda(a) for a in m.mf)
    g.f_mux_, g.f_muy_, g.f_muz_ = (_cuda(a) for a in m.muf)
    g.mu_, g.rho_old_ = _cuda(m.mu), _cuda(m.rho_old)
    g.f_coupling_impulse_x_, g.f_coupling_impulse_y_, g.f_coupling_impulse_z_ = (_cuda(a) for a in m.imp)
    g.f_ibm_solid_fraction_x_, g.f_ibm_solid_fraction_y_, g.f_ibm_solid_fraction_z_ = (_cuda(a) for a in m.sf)
    SMACStep(g, m.dt, g=m.g, bc=BoundaryConditions(m.bc_type, *m.bc_v)).get_vof_vstar_rhouu_consistent_two_way()
    torch.cuda.synchronize()
    for a, b in zip((g.f_vx_star_, g.f_vy_star_, g.f_vz_star_), O.predict_vstar(m)):
        assert np.array_equal(a.cpu().numpy(), b)


# ---------------------------------------------------------------------------
# the two-way Poisson coefficients (update_poisson_beta_two_way)

def run_beta(N, h, eps, fir, fb):
    out = [_cuda(a) for a in fb]
    poisson_beta_two_way_device(N, h, _cuda(eps), [_cuda(a) for a in fir], out)
    torch.cuda.synchronize()
    return tuple(a.cpu().numpy() for a in out)


@pytest.mark.parametrize("N", [(12, 10, 8), (1, 6, 3), (33, 17, 9)])
def test_poisson_beta_two_way_bit_exact_against_oracle(N):
    N, h, eps, fir, fb = W.beta_two_way_case(N, seed=5)
    for a, b in zip(run_beta(N, h, eps, fir, fb), O.poisson_beta_two_way(N, eps, fir, fb)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", beta_golden_names())
def test_poisson_beta_two_way_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    for k, a in zip(("fbx", "fby", "fbz"), run_beta(*beta_case_from_spec(meta))):
        assert np.array_equal(a, arr[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
def test_poisson_beta_two_way_against_reference_library_and_time_256():
    case = W.beta_two_way_case((64, 48, 40), seed=6)
    *ref, _ = REF.poisson_beta_two_way(*case)
    for a, b in zip(run_beta(*case), ref):
        assert np.array_equal(a, b)
    N, h, eps, fir, fb = W.beta_two_way_case((256, 256, 256), seed=7)
    REF.poisson_beta_two_way(N, h, eps, fir, fb)  # loads the reference's kernel
    *_, ref_ms = REF.poisson_beta_two_way(N, h, eps, fir, fb)
    e, fi, out = _cuda(eps), [_cuda(a) for a in fir], [_cuda(a) for a in fb]
    ms = _device_ms(lambda: poisson_beta_two_way_device(N, h, e, fi, out))
    print(f"update_poisson_beta_two_way 256^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


# ---------------------------------------------------------------------------
# the mass-flux update (compute_mass_flux_from_alpha_flux)

def _flux_fields(c):
    m = c.mom
    f = {}
    for k, ax in enumerate("xyz"):
        f["f" + ax + "t"] = _cuda(m.ft[k])
        f["f" + ax + "bcid"] = _cuda(m.bcid[k])
        f["v" + ax] = _cuda(m.v[k])
        f["F" + ax] = _cuda(c.F[k])
        if m.lam is not None:
            f["lam" + ax] = _cuda(m.lam[k])
    return f


def run_flux(c):
    out = [_cuda(a) for a in c.mf]
    m = c.mom
    mass_flux_device(m.N, m.h, BoundaryConditions(m.bc_type, *m.bc_v), _flux_fields(c), c.rho0, c.rho1, m.dt, out,
                     eps_half=None if c.eps_half is None else _cuda(c.eps_half))
    torch.cuda.synchronize()
    return tuple(a.cpu().numpy() for a in out)


@pytest.mark.parametrize("spec", [
    dict(N=(12, 10, 8), seed=1, sides=("x+", "z-")),
    dict(N=(17, 9, 13), seed=2, sides=("y-",), solid_fraction=0.3),
    dict(N=(9, 7, 11), seed=3, sides=("x-",), extras=False),
    dict(N=(12, 10, 8), seed=4, sides=("x-", "y+"), two_way=True),
    dict(N=(1, 6, 4), seed=5, sides=(), two_way=True),
])
def test_mass_flux_bit_exact_against_oracle(spec):
    c = W.mass_flux_case(**spec)
    for k, a, b in zip(("mfx", "mfy", "mfz"), run_flux(c), O.mass_flux(c)):
        assert np.array_equal(a, b), k


@pytest.mark.parametrize("name", flux_golden_names())
def test_mass_flux_bit_exact_against_reference_golden(name):
    meta, arr = load_golden(name)
    for k, a in zip(("mfx", "mfy", "mfz"), run_flux(flux_case_from_spec(meta))):
        assert np.array_equal(a, arr[k]), k


@pytest.mark.skipif(not REF.available(), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("two_way", [False, True])
def test_mass_flux_against_reference_library_and_time_256(two_way):
    c = W.mass_flux_case((64, 48, 40), seed=6, sides=("x+", "z-"), solid_fraction=0.05, two_way=two_way)
    *ref, _ = REF.mass_flux(c)
    for k, a, b in zip(("mfx", "mfy", "mfz"), run_flux(c), ref):
        assert np.array_equal(a, b), k
    c = W.mass_flux_case((256, 256, 256), seed=7, sides=("x+",), solid_fraction=0.02, two_way=two_way)
    REF.mass_flux(c)  # loads the reference's kernel
    *_, ref_ms = REF.mass_flux(c)
    m = c.mom
    fields, out = _flux_fields(c), [_cuda(a) for a in c.mf]
    eh = None if c.eps_half is None else _cuda(c.eps_half)
    bc = BoundaryConditions(m.bc_type, *m.bc_v)
    ms = _device_ms(lambda: mass_flux_device(m.N, m.h, bc, fields, c.rho0, c.rho1, m.dt, out, eps_half=eh))
    name = "compute_mass_flux_from_alpha_flux" + ("_two_way" if two_way else "")
    print(f"{name} 256^3: {ms * 1e3:.1f} us (reference {ref_ms * 1e3:.1f} us)")
    assert ms < ref_ms


def test_smac_step_mass_flux_matches_oracle():
    """SMACStep.compute_mass_flux_from_alpha_flux, one-way and two-way, on a DeviceGrid."""
    c = W.mass_flux_case((14, 12, 10), seed=9, sides=("x+",), solid_fraction=0.2, two_way=True)
    m = c.mom
    sh = W.shapes(m.N)
    zc = lambda: torch.zeros(sh["cell"], dtype=torch.float64, device="cuda")  # noqa: E731
    g = DeviceGrid(*m.N, *m.h, *(_cuda(a) for a in m.vs), *(_cuda(a) for a in m.fb), *(_cuda(a) for a in m.fb),
                   _cuda(m.ct), *(_cuda(a) for a in m.ft), _cuda(m.p), zc(), zc(), *(_cuda(a) for a in m.v))
    g.f_xbcid_, g.f_ybcid_, g.f_zbcid_ = (_cuda(a) for a in m.bcid)
    g.f_ibm_area_solid_fraction_x_, g.f_ibm_area_solid_fraction_y_, g.f_ibm_area_solid_fraction_z_ = (
        _cuda(a) for a in m.lam)
    g.f_Fx_accum_, g.f_Fy_accum_, g.f_Fz_accum_ = (_cuda(a) for a in c.F)
    g.void_fraction_half_ = _cuda(c.eps_half)
    g.f_mfx_, g.f_mfy_, g.f_mfz_ = (_cuda(a) for a in c.mf)
    step = SMACStep(g, m.dt, g=m.g, bc=BoundaryConditions(m.bc_type, *m.bc_v))
    import dataclasses
    for two_way, case in ((True, c), (False, dataclasses.replace(c, eps_half=None))):
        step.compute_mass_flux_from_alpha_flux(c.rho0, c.rho1, two_way=two_way)
        torch.cuda.synchronize()
        for a, b in zip((g.f_mfx_, g.f_mfy_, g.f_mfz_), O.mass_flux(case)):
            assert np.array_equal(a.cpu().numpy(), b)


def test_smac_step_boundary_faces_and_two_way_coefficients_match_oracle():
    """SMACStep.update_boundary_faces (outlet f_b) and, on the same grid,
    SMACStep.update_poisson_beta_two_way (f_b = eps_f f_inv_rho)."""
    c = W.post_case((16, 12, 10), seed=23, sides=("x+", "y-"), solid_fraction=0.1)
    sh = W.shapes(c.N)
    g = DeviceGrid(*c.N, *c.h, *(_cuda(a) for a in c.vs), *(_cuda(a) for a in c.fb), *(_cuda(a) for a in c.fb),
                   _cuda(c.ct), *(_cuda(a) for a in c.ft), _cuda(c.p), _cuda(c.p_delta),
                   torch.zeros(sh["cell"], dtype=torch.float64, device="cuda"), *(_cuda(a) for a in c.v))
    g.f_xoutlet_, g.f_youtlet_, g.f_zoutlet_ = (_cuda(a) for a in c.marks)
    step = SMACStep(g, c.dt, g=c.g, bc=BoundaryConditions(c.bc_type, *c.bc_v))
    step.update_boundary_faces()
    torch.cuda.synchronize()
    want = O.update_boundary_faces(c.N, *c.marks, *c.fb)
    for a, b in zip((g.f_bx_, g.f_by_, g.f_bz_), want):
        assert np.array_equal(a.cpu().numpy(), b)
    N, h, eps, fir, fb = W.beta_two_way_case(c.N, seed=23)
    g.void_fraction_ = _cuda(eps)
    g.f_inv_rhox_, g.f_inv_rhoy_, g.f_inv_rhoz_ = (_cuda(a) for a in fir)
    g.f_bx_, g.f_by_, g.f_bz_ = (_cuda(a) for a in fb)
    step.update_poisson_beta_two_way()
    torch.cuda.synchronize()
    for a, b in zip((g.f_bx_, g.f_by_, g.f_bz_), O.poisson_beta_two_way(N, eps, fir, fb)):
        assert np.array_equal(a.cpu().numpy(), b)
