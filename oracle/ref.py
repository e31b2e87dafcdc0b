"""ctypes binding of oracle/_ref/libref_smac.so: the REFERENCE's own GPU
pressure solve built from its sources (oracle/Makefile target `ref`,
driver oracle/ref_harness.cu).  TEST INFRASTRUCTURE ONLY.

It runs only on a CUDA device; the library is built where the reference
sources are available and travels with the repository as a built file.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_smac.so")
_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class RefInputs(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double), ("dt", ctypes.c_double),
        ("solver_type", ctypes.c_int), ("tol", ctypes.c_double), ("levels", ctypes.c_int),
        ("do_correct", ctypes.c_int),
        ("vxs", _dp), ("vys", _dp), ("vzs", _dp), ("eps", _dp), ("eps_old", _dp),
        ("fbx", _dp), ("fby", _dp), ("fbz", _dp), ("fsx", _dp), ("fsy", _dp), ("fsz", _dp),
        ("firx", _dp), ("firy", _dp), ("firz", _dp),
        ("ct", _u8p), ("fxt", _u8p), ("fyt", _u8p), ("fzt", _u8p),
    ]


class RefOutputs(ctypes.Structure):
    _fields_ = [("p_delta", _dp), ("rhs", _dp), ("vx", _dp), ("vy", _dp), ("vz", _dp), ("p", _dp),
                ("iterations", ctypes.c_int), ("num_levels", ctypes.c_int),
                ("solve_ms", ctypes.c_double), ("correct_ms", ctypes.c_double)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise ImportError(f"{LIB_PATH} is not built (make -C oracle ref, where the reference sources exist)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.ref_solve.restype = ctypes.c_int
        _lib.ref_solve.argtypes = [ctypes.POINTER(RefInputs), ctypes.POINTER(RefOutputs)]
    return _lib


def _p(a, t=ctypes.c_double):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(t))


SEAM_PATH = os.path.join(_HERE, "_ref", "libref_seam.so")
_seam = None


def seam_available() -> bool:
    return os.path.exists(SEAM_PATH)


def _seam_lib():
    global _seam
    if _seam is None:
        if not seam_available():
            raise ImportError(f"{SEAM_PATH} is not built (make -C oracle ref, where the reference sources exist)")
        _seam = ctypes.CDLL(SEAM_PATH)
        _seam.ref_solve_seam.restype = ctypes.c_int
        _seam.ref_solve_seam.argtypes = [ctypes.POINTER(RefInputs), ctypes.POINTER(RefOutputs), ctypes.c_int]
    return _seam


def solve_seam(case, solver_type=3, tol=1e-11, precision=0, do_correct=True, eps=None, eps_old=None, fs=None):
    """The reference's G_SMACSolver::solve_poisson() + correct_vof_velocity()
    with this library's G_B200PressureSolver installed at its seam
    (oracle/ref_seam.cu): the drop-in as a maintainer would install it.
    tol is the reference's tol_ (max|r| dt); returns the same dict as solve."""
    return _run(_seam_lib().ref_solve_seam, case, solver_type, tol, 4, do_correct, eps, eps_old, fs,
                extra=(ctypes.c_int(precision),))


def solve(case, solver_type=3, tol=1e-11, levels=4, do_correct=True, eps=None, eps_old=None, fs=None):
    """Run the reference's solve_poisson (+ correct_vof_velocity) on a
    mydemcfd_b200.workloads.Case.  eps defaults to 1 (the reference's
    standalone driver leaves it at 0, which zeroes the divergence term)."""
    return _run(lib().ref_solve, case, solver_type, tol, levels, do_correct, eps, eps_old, fs)


def _run(fn, case, solver_type, tol, levels, do_correct, eps, eps_old, fs, extra=()):
    N = case.N
    nx, ny, nz = N
    cell = (nz + 2, ny + 2, nx + 2)
    xs, ys, zs = (nz + 2, ny + 2, nx + 3), (nz + 2, ny + 3, nx + 2), (nz + 3, ny + 2, nx + 2)
    eps = np.ones(cell) if eps is None else eps
    eps_old = np.ones(cell) if eps_old is None else eps_old
    fsx, fsy, fsz = fs if fs is not None else (np.zeros(xs), np.zeros(ys), np.zeros(zs))
    out = {k: np.zeros(cell) for k in ("p_delta", "rhs", "p")}
    out["vx"], out["vy"], out["vz"] = np.zeros(xs), np.zeros(ys), np.zeros(zs)
    i = RefInputs()
    i.Nx, i.Ny, i.Nz = N
    i.Lx, i.Ly, i.Lz = nx * case.h[0], ny * case.h[1], nz * case.h[2]
    i.dt = case.dt
    i.solver_type = solver_type
    i.tol = tol
    i.levels = levels
    i.do_correct = 1 if do_correct else 0
    keep = [eps, eps_old, fsx, fsy, fsz]
    for name, arr in (("vxs", case.vxs), ("vys", case.vys), ("vzs", case.vzs), ("eps", eps), ("eps_old", eps_old),
                      ("fbx", case.fbx), ("fby", case.fby), ("fbz", case.fbz), ("fsx", fsx), ("fsy", fsy),
                      ("fsz", fsz), ("firx", case.fbx), ("firy", case.fby), ("firz", case.fbz)):
        arr = np.ascontiguousarray(arr, np.float64)
        keep.append(arr)
        setattr(i, name, _p(arr))
    for name, arr in (("ct", case.ct), ("fxt", case.fxt), ("fyt", case.fyt), ("fzt", case.fzt)):
        arr = np.ascontiguousarray(arr, np.uint8)
        keep.append(arr)
        setattr(i, name, _p(arr, ctypes.c_uint8))
    o = RefOutputs()
    for k in ("p_delta", "rhs", "p", "vx", "vy", "vz"):
        setattr(o, k, _p(out[k]))
    rc = fn(ctypes.byref(i), ctypes.byref(o), *extra)
    if rc != 0:
        raise RuntimeError(f"{fn.__name__} returned {rc} (iterations field {o.iterations})")
    out["iterations"] = o.iterations
    out["num_levels"] = o.num_levels
    out["solve_ms"] = o.solve_ms
    out["correct_ms"] = o.correct_ms
    return out


class RefPostInputs(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double), ("dt", ctypes.c_double),
        ("gx", ctypes.c_double), ("gy", ctypes.c_double), ("gz", ctypes.c_double),
        ("num_ids", ctypes.c_int), ("bc_type", _u8p), ("bc_vx", _dp), ("bc_vy", _dp), ("bc_vz", _dp),
        ("p", _dp), ("p_delta", _dp), ("rho", _dp),
        ("ct", _u8p), ("fxt", _u8p), ("fyt", _u8p), ("fzt", _u8p), ("fxbcid", _u8p), ("fybcid", _u8p),
        ("fzbcid", _u8p),
        ("fxid", ctypes.POINTER(ctypes.c_int)), ("fyid", ctypes.POINTER(ctypes.c_int)),
        ("fzid", ctypes.POINTER(ctypes.c_int)),
        ("lamx", _dp), ("lamy", _dp), ("lamz", _dp),
        ("vxs", _dp), ("vys", _dp), ("vzs", _dp), ("fbx", _dp), ("fby", _dp), ("fbz", _dp),
        ("vx", _dp), ("vy", _dp), ("vz", _dp),
    ]


class RefPostOutputs(ctypes.Structure):
    _fields_ = [(k, _dp) for k in ("p", "vx", "vy", "vz", "gpx", "gpy", "gpz")] + \
        [("ghost_ms", ctypes.c_double), ("gradp_ms", ctypes.c_double)]


def grid_spacing(N, h):
    """The spacing the reference computes from the domain size: (N h) / N."""
    return tuple(float(np.float64(n * hh) / np.float64(n)) for n, hh in zip(N, h))


def _post_inputs(case, keep):
    nx, ny, nz = case.N
    ghost = np.ones(case.ct.shape, bool)
    ghost[1:nz + 1, 1:ny + 1, 1:nx + 1] = False
    # a C_SOLID ghost cell would make the reference read the cell type one
    # entry past its own index range
    assert not np.any(case.ct[ghost] == 3), "solid ghost cells are not passed to the reference"
    i = RefPostInputs()
    i.Nx, i.Ny, i.Nz = case.N
    i.Lx, i.Ly, i.Lz = (n * hh for n, hh in zip(case.N, case.h))
    i.dt = case.dt
    i.gx, i.gy, i.gz = case.g

    def d(a):
        a = np.ascontiguousarray(a, np.float64)
        keep.append(a)
        return _p(a)

    def u8(a):
        a = np.ascontiguousarray(a, np.uint8)
        keep.append(a)
        return _p(a, ctypes.c_uint8)

    def i32(a):
        a = np.ascontiguousarray(a, np.int32)
        keep.append(a)
        return _p(a, ctypes.c_int)

    i.num_ids = len(case.bc_type)
    i.bc_type = u8(case.bc_type)
    i.bc_vx, i.bc_vy, i.bc_vz = (d(a) for a in case.bc_v)
    i.p, i.p_delta, i.rho = d(case.p), d(case.p_delta), d(case.rho)
    i.ct = u8(case.ct)
    i.fxt, i.fyt, i.fzt = (u8(a) for a in case.ft)
    i.fxbcid, i.fybcid, i.fzbcid = (u8(a) for a in case.bcid)
    i.fxid, i.fyid, i.fzid = (i32(a) for a in case.internal_id)
    lam = case.lam if case.lam is not None else tuple(np.zeros(a.shape) for a in case.v)
    i.lamx, i.lamy, i.lamz = (d(a) for a in lam)
    i.vxs, i.vys, i.vzs = (d(a) for a in case.vs)
    i.fbx, i.fby, i.fbz = (d(a) for a in case.fb)
    i.vx, i.vy, i.vz = (d(a) for a in case.v)
    return i


def _post_lib():
    L = lib()
    if not hasattr(L, "_post_set"):
        L.ref_post.restype = ctypes.c_int
        L.ref_post.argtypes = [ctypes.POINTER(RefPostInputs), ctypes.POINTER(RefPostOutputs)]
        L.ref_vstar.restype = ctypes.c_int
        L.ref_vstar.argtypes = [ctypes.POINTER(RefPostInputs), _dp, _dp, _dp, _dp]
        L._post_set = True
    return L


def vstar(case):
    """Run the reference's update_vstar_boundary on the u* of a
    mydemcfd_b200.workloads.PostCase: returns (vxs, vys, vzs, ms)."""
    keep = []
    i = _post_inputs(case, keep)
    out = [np.zeros(a.shape) for a in case.vs]
    ms = ctypes.c_double(0.0)
    rc = _post_lib().ref_vstar(ctypes.byref(i), *(_p(a) for a in out), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_vstar returned {rc}")
    return (*out, ms.value)


def post(case):
    """Run the reference's update_boundary_ghost + make_face_gradp on a
    mydemcfd_b200.workloads.PostCase (lam None -> zeros); also returns the
    device time of each call (ghost_ms, gradp_ms)."""
    keep = []
    i = _post_inputs(case, keep)
    L = _post_lib()
    out = {"p": np.zeros(case.p.shape), "vx": np.zeros(case.v[0].shape), "vy": np.zeros(case.v[1].shape),
           "vz": np.zeros(case.v[2].shape), "gpx": np.zeros(case.v[0].shape), "gpy": np.zeros(case.v[1].shape),
           "gpz": np.zeros(case.v[2].shape)}
    o = RefPostOutputs()
    for k, a in out.items():
        setattr(o, k, _p(a))
    rc = L.ref_post(ctypes.byref(i), ctypes.byref(o))
    if rc != 0:
        raise RuntimeError(f"ref_post returned {rc}")
    out["ghost_ms"], out["gradp_ms"] = o.ghost_ms, o.gradp_ms
    return out


class RefStIO(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
                ("sigma", ctypes.c_double), ("alpha", _dp), ("ct", _u8p)] + \
        [(k, _dp) for k in ("nx", "ny", "nz", "kappa", "gm", "fsx", "fsy", "fsz")] + [("ms", ctypes.c_double)]


def surface_tension(N, h, alpha, ct, sigma):
    """Run the reference's calc_surface_tension on zeroed work arrays:
    returns (fsx, fsy, fsz, nx, ny, nz, kappa, gm, ms)."""
    L = lib()
    if not hasattr(L, "_st_set"):
        L.ref_surface_tension.restype = ctypes.c_int
        L.ref_surface_tension.argtypes = [ctypes.POINTER(RefStIO)]
        L._st_set = True
    nx_, ny_, nz_ = N
    cell = (nz_ + 2, ny_ + 2, nx_ + 2)
    shapes = [(nz_ + 2, ny_ + 2, nx_ + 3), (nz_ + 2, ny_ + 3, nx_ + 2), (nz_ + 3, ny_ + 2, nx_ + 2)]
    alpha = np.ascontiguousarray(alpha, np.float64)
    ct = np.ascontiguousarray(ct, np.uint8)
    work = [np.zeros(cell) for _ in range(5)]
    fs = [np.zeros(s) for s in shapes]
    io = RefStIO()
    io.Nx, io.Ny, io.Nz = N
    io.Lx, io.Ly, io.Lz = (n * hh for n, hh in zip(N, h))
    io.sigma = sigma
    io.alpha, io.ct = _p(alpha), _p(ct, ctypes.c_uint8)
    io.nx, io.ny, io.nz, io.kappa, io.gm = (_p(a) for a in work)
    io.fsx, io.fsy, io.fsz = (_p(a) for a in fs)
    rc = L.ref_surface_tension(ctypes.byref(io))
    if rc != 0:
        raise RuntimeError(f"ref_surface_tension returned {rc}")
    return (*fs, *work, io.ms)


class RefMomIO(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int)] + \
        [(k, ctypes.c_double) for k in ("Lx", "Ly", "Lz", "dt", "gx", "gy", "gz")] + \
        [("num_ids", ctypes.c_int), ("bc_type", _u8p), ("bc_vx", _dp), ("bc_vy", _dp), ("bc_vz", _dp)] + \
        [(k, ctypes.c_void_p * 3) for k in ("ft", "bcid", "lam", "v", "mf", "muf", "fb", "imp", "sf")] + \
        [("mu", _dp), ("rho_old", _dp), ("p", _dp), ("vs", ctypes.c_void_p * 3), ("ms", ctypes.c_double),
         ("eps_old", _dp), ("eps_new", _dp), ("fir", ctypes.c_void_p * 3)]


def predict_vstar(m):
    """Run the reference's get_vof_vstar_rhouu_consistent (or, for a case
    with eps_old set, get_vof_vstar_rhouu_consistent_two_way) on a
    mydemcfd_b200.workloads.MomentumCase (None fields as zeros): returns
    (vxs, vys, vzs, ms)."""
    L = lib()
    if not hasattr(L, "_mom_set"):
        L.ref_predict_vstar.restype = ctypes.c_int
        L.ref_predict_vstar.argtypes = [ctypes.POINTER(RefMomIO)]
        L._mom_set = True
    keep = []

    def arr(a, dtype=np.float64):
        a = np.ascontiguousarray(a, dtype)
        keep.append(a)
        return a

    def three(arrs, dtype=np.float64, like=None):
        if arrs is None:
            arrs = tuple(np.zeros(x.shape) for x in like)
        return (ctypes.c_void_p * 3)(*(arr(a, dtype).ctypes.data for a in arrs))

    io = RefMomIO()
    io.Nx, io.Ny, io.Nz = m.N
    io.Lx, io.Ly, io.Lz = (n * hh for n, hh in zip(m.N, m.h))
    io.dt = m.dt
    io.gx, io.gy, io.gz = m.g
    io.num_ids = len(m.bc_type)
    io.bc_type = _p(arr(m.bc_type, np.uint8), ctypes.c_uint8)
    io.bc_vx, io.bc_vy, io.bc_vz = (_p(arr(a)) for a in m.bc_v)
    io.ft, io.bcid = three(m.ft, np.uint8), three(m.bcid, np.uint8)
    io.lam, io.imp, io.sf = three(m.lam, like=m.v), three(m.imp, like=m.v), three(m.sf, like=m.v)
    io.v, io.mf, io.muf, io.fb = three(m.v), three(m.mf), three(m.muf), three(m.fb)
    io.mu, io.rho_old, io.p = _p(arr(m.mu)), _p(arr(m.rho_old)), _p(arr(m.p))
    if m.eps_old is not None:
        io.eps_old, io.eps_new = _p(arr(m.eps_old)), _p(arr(m.eps_new))
        io.fir = three(m.fir)
    out = [np.array(a, dtype=np.float64, order="C", copy=True) for a in m.vs]
    io.vs = (ctypes.c_void_p * 3)(*(a.ctypes.data for a in out))
    rc = L.ref_predict_vstar(ctypes.byref(io))
    if rc != 0:
        raise RuntimeError(f"ref_predict_vstar returned {rc}")
    return (*out, io.ms)


IO_LIB_PATH = os.path.join(_HERE, "_ref", "libref_io.so")
_io_lib = None


def io_available() -> bool:
    return os.path.exists(IO_LIB_PATH)


def write_vti(N, h, origin, p, alpha, vx, vy, vz, ibm_sf, outdir, step):
    """Run the reference's FileInOut::output_vti_binary_cellData (host code,
    oracle/_ref/libref_io.so) on the given reference-layout arrays; returns
    the path of the file it wrote (<outdir>/result_<step:06d>.vti)."""
    global _io_lib
    if _io_lib is None:
        _io_lib = ctypes.CDLL(IO_LIB_PATH)
        _io_lib.ref_write_vti.restype = ctypes.c_int
        _io_lib.ref_write_vti.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 6 + [_dp] * 6 + \
            [ctypes.c_char_p, ctypes.c_int]
    arrs = [np.ascontiguousarray(a, np.float64) for a in (p, alpha, vx, vy, vz, ibm_sf)]
    rc = _io_lib.ref_write_vti(*N, *h, *origin, *(_p(a) for a in arrs), str(outdir).encode(), int(step))
    if rc != 0:
        raise RuntimeError(f"ref_write_vti returned {rc}")
    return os.path.join(str(outdir), f"result_{int(step):06d}.vti")


class RefPropsIO(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int)] + \
        [(k, ctypes.c_double) for k in ("Lx", "Ly", "Lz", "rho0", "rho1", "mu0", "mu1")] + \
        [("alpha", _dp), ("ct", _u8p), ("ft", ctypes.c_void_p * 3)] + \
        [(k, _dp) for k in ("rho", "rho_old", "inv_rho", "mu")] + \
        [(k, ctypes.c_void_p * 3) for k in ("fb", "fir", "frho", "fmu")] + [("ms", ctypes.c_double)]


def update_properties(N, h, rho0, rho1, mu0, mu1, alpha, ct, ft, init):
    """Run the reference's update_properties_by_alpha.  init: dict with the
    arrays before the call (keys of oracle.PROP_KEYS plus rho_old, which the
    reference's swap turns into rho); returns the dict after it (rho_old
    holds the previous rho) and the device time."""
    L = lib()
    if not hasattr(L, "_props_set"):
        L.ref_update_properties.restype = ctypes.c_int
        L.ref_update_properties.argtypes = [ctypes.POINTER(RefPropsIO)]
        L._props_set = True
    keys = ("rho", "rho_old", "inv_rho", "mu", "fbx", "fby", "fbz", "firx", "firy", "firz", "rhox", "rhoy", "rhoz",
            "mux", "muy", "muz")
    out = {k: np.array(init[k], dtype=np.float64, order="C", copy=True) for k in keys}
    keep = [np.ascontiguousarray(alpha, np.float64), np.ascontiguousarray(ct, np.uint8)] + \
        [np.ascontiguousarray(t, np.uint8) for t in ft]
    io = RefPropsIO()
    io.Nx, io.Ny, io.Nz = N
    io.Lx, io.Ly, io.Lz = (n * hh for n, hh in zip(N, h))
    io.rho0, io.rho1, io.mu0, io.mu1 = rho0, rho1, mu0, mu1
    io.alpha, io.ct = _p(keep[0]), _p(keep[1], ctypes.c_uint8)
    io.ft = (ctypes.c_void_p * 3)(*(t.ctypes.data for t in keep[2:]))
    for k in ("rho", "rho_old", "inv_rho", "mu"):
        setattr(io, k, _p(out[k]))
    for name, ks in (("fb", ("fbx", "fby", "fbz")), ("fir", ("firx", "firy", "firz")),
                     ("frho", ("rhox", "rhoy", "rhoz")), ("fmu", ("mux", "muy", "muz"))):
        setattr(io, name, (ctypes.c_void_p * 3)(*(out[k].ctypes.data for k in ks)))
    rc = L.ref_update_properties(ctypes.byref(io))
    if rc != 0:
        raise RuntimeError(f"ref_update_properties returned {rc}")
    return out, io.ms


class RefBetaIO(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int)] + \
        [(k, ctypes.c_double) for k in ("Lx", "Ly", "Lz")] + \
        [("eps", _dp), ("fir", ctypes.c_void_p * 3), ("fb", ctypes.c_void_p * 3), ("ms", ctypes.c_double)]


def poisson_beta_two_way(N, h, eps, fir, fb):
    """Run the reference's G_CFDDEMCoupling::update_poisson_beta_two_way:
    returns (fbx, fby, fbz, ms), fb after the call."""
    L = lib()
    if not hasattr(L, "_beta_set"):
        L.ref_poisson_beta_two_way.restype = ctypes.c_int
        L.ref_poisson_beta_two_way.argtypes = [ctypes.POINTER(RefBetaIO)]
        L._beta_set = True
    e = np.ascontiguousarray(eps, np.float64)
    firs = [np.ascontiguousarray(a, np.float64) for a in fir]
    out = [np.array(a, dtype=np.float64, order="C", copy=True) for a in fb]
    io = RefBetaIO()
    io.Nx, io.Ny, io.Nz = N
    io.Lx, io.Ly, io.Lz = (n * hh for n, hh in zip(N, h))
    io.eps = _p(e)
    io.fir = (ctypes.c_void_p * 3)(*(a.ctypes.data for a in firs))
    io.fb = (ctypes.c_void_p * 3)(*(a.ctypes.data for a in out))
    rc = L.ref_poisson_beta_two_way(ctypes.byref(io))
    if rc != 0:
        raise RuntimeError(f"ref_poisson_beta_two_way returned {rc}")
    return (*out, io.ms)


class RefFluxIO(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int)] + \
        [(k, ctypes.c_double) for k in ("Lx", "Ly", "Lz", "dt", "rho0", "rho1")] + \
        [("num_ids", ctypes.c_int), ("bc_type", _u8p), ("bc_vx", _dp), ("bc_vy", _dp), ("bc_vz", _dp)] + \
        [(k, ctypes.c_void_p * 3) for k in ("ft", "bcid", "lam", "v", "F")] + \
        [("eps_half", _dp), ("mf", ctypes.c_void_p * 3), ("ms", ctypes.c_double)]


def mass_flux(c):
    """Run the reference's compute_mass_flux_from_alpha_flux (two-way form
    when c.eps_half is set) on a mydemcfd_b200.workloads.MassFluxCase:
    returns (mfx, mfy, mfz, ms)."""
    L = lib()
    if not hasattr(L, "_flux_set"):
        L.ref_mass_flux.restype = ctypes.c_int
        L.ref_mass_flux.argtypes = [ctypes.POINTER(RefFluxIO)]
        L._flux_set = True
    keep = []

    def arr(a, dtype=np.float64):
        a = np.ascontiguousarray(a, dtype)
        keep.append(a)
        return a

    def three(arrs, dtype=np.float64, like=None):
        if arrs is None:
            arrs = tuple(np.zeros(x.shape) for x in like)
        return (ctypes.c_void_p * 3)(*(arr(a, dtype).ctypes.data for a in arrs))

    m = c.mom
    io = RefFluxIO()
    io.Nx, io.Ny, io.Nz = m.N
    io.Lx, io.Ly, io.Lz = (n * hh for n, hh in zip(m.N, m.h))
    io.dt, io.rho0, io.rho1 = m.dt, c.rho0, c.rho1
    io.num_ids = len(m.bc_type)
    io.bc_type = _p(arr(m.bc_type, np.uint8), ctypes.c_uint8)
    io.bc_vx, io.bc_vy, io.bc_vz = (_p(arr(a)) for a in m.bc_v)
    io.ft, io.bcid = three(m.ft, np.uint8), three(m.bcid, np.uint8)
    io.lam, io.v, io.F = three(m.lam, like=m.v), three(m.v), three(c.F)
    if c.eps_half is not None:
        io.eps_half = _p(arr(c.eps_half))
    out = [np.array(a, dtype=np.float64, order="C", copy=True) for a in c.mf]
    io.mf = (ctypes.c_void_p * 3)(*(a.ctypes.data for a in out))
    rc = L.ref_mass_flux(ctypes.byref(io))
    if rc != 0:
        raise RuntimeError(f"ref_mass_flux returned {rc}")
    return (*out, io.ms)
