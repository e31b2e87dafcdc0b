"""ctypes binding of ``libsmac_oracle.so`` (see ``smac_oracle.cpp``).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.
All arrays are numpy arrays in the reference layout: shape (sz, sy, sx),
C order, so that flat index = (z*sy + y)*sx + x (CFD/MyArray.h:43-51).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsmac_oracle.so")
_lib = None

# CFD/Enums.h:25-30
STANDARD_PCG = 0
PURENEUMANN_STANDARD_PCG = 1
GMG_PCG = 2
PURENEUMANN_GMG_PCG = 3

STOP_REFERENCE = 0      # max|r|*dt < tol every check_freq iterations (G_PCGSolver.cu:884-903)
STOP_REL_RECURSIVE = 1  # ||r||/||b|| < tol on the recursive residual, same frequency
STOP_REL_TRUE = 2       # ||b - A p||/||b|| < tol, every iteration


class OrcStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("norm_b", ctypes.c_double),
        ("res_max", ctypes.c_double),
        ("res_rel", ctypes.c_double),
        ("true_res_rel", ctypes.c_double),
        ("num_levels", ctypes.c_int),
        ("status", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class OrcProblem(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("vxs", _dp), ("vys", _dp), ("vzs", _dp),
        ("eps", _dp), ("eps_old", _dp),
        ("fbx", _dp), ("fby", _dp), ("fbz", _dp),
        ("fsx", _dp), ("fsy", _dp), ("fsz", _dp),
        ("ct", _u8p), ("fxt", _u8p), ("fyt", _u8p), ("fzt", _u8p),
    ]


def build(force: bool = False) -> str:
    """Compile libsmac_oracle.so with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "smac_oracle.cpp"))
    ):
        subprocess.run(["make", "-C", _HERE, "libsmac_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_solve.restype = ctypes.c_int
        _lib.orc_num_threads.restype = ctypes.c_int
    return _lib


def _p(a, ctype=ctypes.c_double):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C contiguous"
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _u8(a):
    return _p(a, ctypes.c_uint8)


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


# ---------------------------------------------------------------------------
# shapes (CFD/memberList/gridMembers.def)
def cell_shape(N):
    nx, ny, nz = N
    return (nz + 2, ny + 2, nx + 2)


def xface_shape(N):
    nx, ny, nz = N
    return (nz + 2, ny + 2, nx + 3)


def yface_shape(N):
    nx, ny, nz = N
    return (nz + 2, ny + 3, nx + 2)


def zface_shape(N):
    nx, ny, nz = N
    return (nz + 3, ny + 2, nx + 2)


def set_face_type(N):
    fxt = np.empty(xface_shape(N), np.uint8)
    fyt = np.empty(yface_shape(N), np.uint8)
    fzt = np.empty(zface_shape(N), np.uint8)
    lib().orc_set_face_type(*N, _u8(fxt), _u8(fyt), _u8(fzt))
    return fxt, fyt, fzt


def set_cell_type(N):
    ct = np.empty(cell_shape(N), np.uint8)
    lib().orc_set_cell_type(*N, _u8(ct))
    return ct


def solid_fraction_spheres(N, h, origin, spheres):
    sf = np.zeros(cell_shape(N), np.float64)
    sph = np.ascontiguousarray(np.asarray(spheres, np.float64).reshape(-1, 4))
    c = ctypes.c_double
    lib().orc_solid_fraction_spheres(*N, c(h[0]), c(h[1]), c(h[2]), c(origin[0]), c(origin[1]), c(origin[2]),
                                     _p(sph), ctypes.c_int(sph.shape[0]), _p(sf))
    return sf


def set_solid_cells(N, sf, ct, fxt, fyt, fzt):
    lib().orc_set_solid_cells(*N, _p(sf), _u8(ct), _u8(fxt), _u8(fyt), _u8(fzt))


def update_boundary_faces(N, fxo, fyo, fzo, fbx, fby, fbz):
    """Outlet rule of G_SMACSolver::update_boundary_faces
    (CFD/G_SMACSolver_VoF.cu:1798-1950) on copies of the face coefficients;
    marks 1 / 2 give the interior side +1 / -1."""
    fbx, fby, fbz = (np.array(a, dtype=np.float64, order="C", copy=True) for a in (fbx, fby, fbz))
    lib().orc_update_boundary_faces(*N, _u8(fxo), _u8(fyo), _u8(fzo), _p(fbx), _p(fby), _p(fbz))
    return fbx, fby, fbz


def pressure_ghost(N, h, g, ct, rho, p):
    """Pressure part of G_SMACSolver::update_boundary_ghost
    (CFD/G_SMACSolver.cu:1144-1267) on a copy of p: C_SOLID cells from their
    first C_INTERIOR neighbour, ghost cells from the nearest interior cell,
    both shifted hydrostatically by rho g."""
    p = np.array(p, dtype=np.float64, order="C", copy=True)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    c = ctypes.c_double
    lib().orc_pressure_ghost(*N, c(h[0]), c(h[1]), c(h[2]), c(g[0]), c(g[1]), c(g[2]), _u8(ct), _p(rho), _p(p))
    return p


def face_gradp(N, h, p):
    """G_SMACSolver::make_face_gradp (CFD/G_SMACSolver.cu:1277-1343): face
    pressure gradients on faces 1..N+1 of each family; other entries 0."""
    p = np.ascontiguousarray(p, dtype=np.float64)
    gx = np.zeros(xface_shape(N)); gy = np.zeros(yface_shape(N)); gz = np.zeros(zface_shape(N))
    c = ctypes.c_double
    lib().orc_face_gradp(*N, c(h[0]), c(h[1]), c(h[2]), _p(p), _p(gx), _p(gy), _p(gz))
    return gx, gy, gz


def velocity_outlet(N, h, dt, marks, vs, fb, p_delta, v):
    """k_update_v{x,y,z}_outlet (CFD/G_BoundaryFunctions.cu:143-255) on copies
    of the velocities v."""
    v = [np.array(a, dtype=np.float64, order="C", copy=True) for a in v]
    c = ctypes.c_double
    lib().orc_velocity_outlet(*N, c(h[0]), c(h[1]), c(h[2]), c(dt), *(_u8(m) for m in marks),
                              *(_p(np.ascontiguousarray(a)) for a in vs), *(_p(np.ascontiguousarray(a)) for a in fb),
                              _p(np.ascontiguousarray(p_delta)), *(_p(a) for a in v))
    return tuple(v)


def velocity_ghost(N, bc_type, bc_v, bcid, lam, v):
    """k_update_v*_ghost + k_update_v*_ghost_corner
    (CFD/G_BoundaryFunctions.cu:277-560) on copies of the velocities v."""
    v = [np.array(a, dtype=np.float64, order="C", copy=True) for a in v]
    bct = np.ascontiguousarray(bc_type, np.uint8)
    bv = [np.ascontiguousarray(a, np.float64) for a in bc_v]
    lam = (None, None, None) if lam is None else tuple(np.ascontiguousarray(a) for a in lam)
    lib().orc_velocity_ghost(*N, _u8(bct), *(_p(a) for a in bv), *(_u8(np.ascontiguousarray(b)) for b in bcid),
                             *(_p(a) for a in lam), *(_p(a) for a in v))
    return tuple(v)


def vstar_boundary(N, bc_type, bc_v, ft, bcid, marks, lam, vs):
    """G_SMACSolver::update_vstar_boundary (k_update_v*star_boundary,
    CFD/G_BoundaryFunctions.cu:3-71) on copies of u*; marks/lam may be None."""
    vs = [np.array(a, dtype=np.float64, order="C", copy=True) for a in vs]
    bct = np.ascontiguousarray(bc_type, np.uint8)
    bv = [np.ascontiguousarray(a, np.float64) for a in bc_v]
    marks = (None, None, None) if marks is None else tuple(np.ascontiguousarray(m, np.uint8) for m in marks)
    lam = (None, None, None) if lam is None else tuple(np.ascontiguousarray(a) for a in lam)
    lib().orc_vstar_boundary(*N, _u8(bct), *(_p(a) for a in bv), *(_u8(np.ascontiguousarray(t)) for t in ft),
                             *(_u8(np.ascontiguousarray(b)) for b in bcid), *(_u8(m) for m in marks),
                             *(_p(a) for a in lam), *(_p(a) for a in vs))
    return tuple(vs)


def surface_tension(N, h, alpha, ct, sigma, nx=None, ny=None, nz=None, kappa=None, gm=None):
    """G_SMACSolver::calc_surface_tension (CFD/G_SMACSolver_VoF.cu:435-445):
    returns (fsx, fsy, fsz, nx, ny, nz, kappa, gm); the work arrays start from
    the given ones (zeros by default), as the reference's keep their values
    where it does not write them."""
    sh = cell_shape(N)
    work = [np.zeros(sh) if a is None else np.array(a, dtype=np.float64, order="C", copy=True)
            for a in (nx, ny, nz, kappa, gm)]
    fs = [np.zeros(xface_shape(N)), np.zeros(yface_shape(N)), np.zeros(zface_shape(N))]
    c = ctypes.c_double
    lib().orc_surface_tension(*N, c(h[0]), c(h[1]), c(h[2]), _p(np.ascontiguousarray(alpha, np.float64)),
                              _u8(np.ascontiguousarray(ct, np.uint8)), c(sigma), *(_p(a) for a in work),
                              *(_p(a) for a in fs))
    return (*fs, *work)


def predict_vstar(m):
    """G_SMACSolver::get_vof_vstar_rhouu_consistent (CFD/G_SMACSolver.cu:90-1070)
    on a workloads.MomentumCase: returns (vxs, vys, vzs), copies of m.vs with
    every F_INTERIOR face predicted.  A case with m.eps_old set takes the
    two-way form, get_vof_vstar_rhouu_consistent_two_way (:1538-2203), with
    m.fir in place of m.fb."""
    vs = [np.array(a, dtype=np.float64, order="C", copy=True) for a in m.vs]
    keep = []

    def arr3(arrs, dtype):
        if arrs is None:
            return (ctypes.c_void_p * 3)(None, None, None)
        out = []
        for a in arrs:
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            out.append(a.ctypes.data)
        return (ctypes.c_void_p * 3)(*out)

    def one(a):
        a = np.ascontiguousarray(a, np.float64)
        keep.append(a)
        return _p(a)

    c = ctypes.c_double
    bct = np.ascontiguousarray(m.bc_type, np.uint8)
    bv = [np.ascontiguousarray(a, np.float64) for a in m.bc_v]
    vsp = (ctypes.c_void_p * 3)(*(a.ctypes.data for a in vs))
    tw = m.eps_old is not None
    lib().orc_predict_vstar2(*m.N, c(m.h[0]), c(m.h[1]), c(m.h[2]), c(m.dt), c(m.g[0]), c(m.g[1]), c(m.g[2]),
                             _u8(bct), *(_p(a) for a in bv), arr3(m.ft, np.uint8), arr3(m.bcid, np.uint8),
                             arr3(m.lam, np.float64), arr3(m.v, np.float64), arr3(m.mf, np.float64),
                             arr3(m.muf, np.float64), one(m.mu), one(m.rho_old), one(m.p),
                             arr3(m.fir if tw else m.fb, np.float64), arr3(m.imp, np.float64),
                             arr3(m.sf, np.float64), one(m.eps_old) if tw else None, one(m.eps_new) if tw else None,
                             vsp)
    return tuple(vs)


def post_pass(case):
    """G_SMACSolver::update_boundary_ghost then make_face_gradp
    (CFD/G_SMACSolver.cu:1277-1363) on a workloads.PostCase: returns
    (p, (vx, vy, vz), (gpx, gpy, gpz))."""
    p = pressure_ghost(case.N, case.h, case.g, case.ct, case.rho, case.p)
    v = velocity_outlet(case.N, case.h, case.dt, case.marks, case.vs, case.fb, case.p_delta, case.v)
    v = velocity_ghost(case.N, case.bc_type, case.bc_v, case.bcid, case.lam, v)
    return p, v, face_gradp(case.N, case.h, p)


def face_coeffs_vof(N, alpha, rho0, rho1, ct, fxt, fyt, fzt):
    rho = np.ones(cell_shape(N), np.float64)
    fbx = np.zeros(xface_shape(N)); fby = np.zeros(yface_shape(N)); fbz = np.zeros(zface_shape(N))
    irx = np.zeros(xface_shape(N)); iry = np.zeros(yface_shape(N)); irz = np.zeros(zface_shape(N))
    c = ctypes.c_double
    lib().orc_face_coeffs_vof(*N, _p(alpha), c(rho0), c(rho1), _u8(ct), _u8(fxt), _u8(fyt), _u8(fzt), _p(rho),
                              _p(fbx), _p(fby), _p(fbz), _p(irx), _p(iry), _p(irz))
    return rho, (fbx, fby, fbz), (irx, iry, irz)


def make_rhs(g: "RefGrid"):
    rhs = np.zeros(cell_shape(g.N))
    c = ctypes.c_double
    lib().orc_make_rhs(*g.N, c(1.0 / g.h[0]), c(1.0 / g.h[1]), c(1.0 / g.h[2]), c(1.0 / g.dt),
                       _p(g.vxs), _p(g.vys), _p(g.vzs), _p(g.eps), _p(g.eps_old),
                       _p(g.fbx), _p(g.fby), _p(g.fbz), _p(g.fsx), _p(g.fsy), _p(g.fsz), _u8(g.ct), _p(rhs))
    return rhs


def build_A(g: "RefGrid"):
    """The 8 stencil arrays of k_build_vof_poisson_A, shape (8,)+cell_shape."""
    A = np.zeros((8,) + cell_shape(g.N))
    c = ctypes.c_double
    lib().orc_build_A(*g.N, c(1.0 / g.h[0] ** 2), c(1.0 / g.h[1] ** 2), c(1.0 / g.h[2] ** 2),
                      _p(g.fbx), _p(g.fby), _p(g.fbz), _u8(g.ct), _u8(g.fxt), _u8(g.fyt), _u8(g.fzt), _p(A))
    return A


def apply_A(N, A, p):
    out = np.zeros(cell_shape(N))
    lib().orc_apply_A(*N, _p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(p)), _p(out))
    return out


def solve(g: "RefGrid", solver_type=PURENEUMANN_GMG_PCG, tol=1e-11, levels=4, max_iter=0,
          stop_rule=STOP_REFERENCE, check_freq=0, p_delta=None):
    """Run the reference PCG solver restatement; returns (p_delta, rhs, stats dict)."""
    pd = np.zeros(cell_shape(g.N)) if p_delta is None else np.ascontiguousarray(p_delta).copy()
    rhs = np.zeros(cell_shape(g.N))
    prob = g.problem()
    st = OrcStats()
    rc = lib().orc_solve(ctypes.byref(prob), ctypes.c_int(solver_type), ctypes.c_double(tol),
                         ctypes.c_int(levels), ctypes.c_int(max_iter), ctypes.c_int(stop_rule),
                         ctypes.c_int(check_freq), _p(pd), _p(rhs), ctypes.byref(st))
    d = st.as_dict()
    d["rc"] = rc
    return pd, rhs, d


def correct(g: "RefGrid", p_delta, p=None, v=None):
    """k_correct_vof_velocity: returns (vx, vy, vz, p) after the correction."""
    N = g.N
    p = np.zeros(cell_shape(N)) if p is None else p.copy()
    if v is None:
        vx, vy, vz = np.zeros(xface_shape(N)), np.zeros(yface_shape(N)), np.zeros(zface_shape(N))
    else:
        vx, vy, vz = (a.copy() for a in v)
    c = ctypes.c_double
    lib().orc_correct(*N, c(1.0 / g.h[0]), c(1.0 / g.h[1]), c(1.0 / g.h[2]), c(g.dt),
                      _u8(g.ct), _u8(g.fxt), _u8(g.fyt), _u8(g.fzt), _p(np.ascontiguousarray(p_delta)), _p(p),
                      _p(g.vxs), _p(g.vys), _p(g.vzs), _p(g.firx), _p(g.firy), _p(g.firz),
                      _p(g.fsx), _p(g.fsy), _p(g.fsz), _p(vx), _p(vy), _p(vz))
    return vx, vy, vz, p


@dataclass
class RefGrid:
    """The grid fields the pressure path reads, in the reference layout."""
    N: tuple
    h: tuple
    dt: float
    vxs: np.ndarray
    vys: np.ndarray
    vzs: np.ndarray
    eps: np.ndarray
    eps_old: np.ndarray
    fbx: np.ndarray
    fby: np.ndarray
    fbz: np.ndarray
    fsx: np.ndarray
    fsy: np.ndarray
    fsz: np.ndarray
    firx: np.ndarray
    firy: np.ndarray
    firz: np.ndarray
    ct: np.ndarray
    fxt: np.ndarray
    fyt: np.ndarray
    fzt: np.ndarray

    def problem(self) -> OrcProblem:
        pr = OrcProblem()
        pr.Nx, pr.Ny, pr.Nz = self.N
        pr.dx, pr.dy, pr.dz = self.h
        pr.dt = self.dt
        for name in ("vxs", "vys", "vzs", "eps", "eps_old", "fbx", "fby", "fbz", "fsx", "fsy", "fsz"):
            setattr(pr, name, _p(getattr(self, name)))
        for name in ("ct", "fxt", "fyt", "fzt"):
            setattr(pr, name, _u8(getattr(self, name)))
        self._keep = pr  # arrays are owned by self
        return pr


def vti_block(N, p, alpha, vx, vy, vz, ibm_sf):
    """The appended-data block of FileInOut::output_vti_binary_cellData
    (CFD/FileInOut.cpp:208-254) in numpy: four Float32 cell arrays of the
    interior cells, x fastest, each after its UInt32 byte count; the velocity
    is the mean of each cell's two faces in FP64, then rounded to Float32.
    alpha / ibm_sf None mean zeros."""
    nx, ny, nz = N
    inner = (slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1))
    n = nx * ny * nz
    zeros = np.zeros((nz + 2, ny + 2, nx + 2))
    ux = 0.5 * (vx[1:nz + 1, 1:ny + 1, 1:nx + 1] + vx[1:nz + 1, 1:ny + 1, 2:nx + 2])
    uy = 0.5 * (vy[1:nz + 1, 1:ny + 1, 1:nx + 1] + vy[1:nz + 1, 2:ny + 2, 1:nx + 1])
    uz = 0.5 * (vz[1:nz + 1, 1:ny + 1, 1:nx + 1] + vz[2:nz + 2, 1:ny + 1, 1:nx + 1])
    vel = np.stack([ux, uy, uz], axis=-1).astype(np.float32).reshape(-1)
    parts = []
    for arr, cnt in ((p, n), (alpha if alpha is not None else zeros, n), (None, 3 * n),
                     (ibm_sf if ibm_sf is not None else zeros, n)):
        parts.append(np.array([4 * cnt], np.uint32).tobytes())
        parts.append(vel.tobytes() if arr is None else arr[inner].astype(np.float32).reshape(-1).tobytes())
    return b"".join(parts)


PROP_KEYS = ("rho", "inv_rho", "mu", "fbx", "fby", "fbz", "firx", "firy", "firz", "rhox", "rhoy", "rhoz",
             "mux", "muy", "muz")


def update_properties(N, rho0, rho1, mu0, mu1, alpha, ct, ft, init):
    """G_SMACSolver::update_properties_by_alpha (CFD/G_SMACSolver_VoF.cu:1543-1566)
    after its rho/rho_old swap, on copies of the arrays in `init` (a dict
    with every PROP_KEYS entry); returns the updated dict."""
    out = {k: np.array(init[k], dtype=np.float64, order="C", copy=True) for k in PROP_KEYS}
    p3 = lambda ks: (ctypes.c_void_p * 3)(*(out[k].ctypes.data for k in ks))  # noqa: E731
    fts = [np.ascontiguousarray(t, np.uint8) for t in ft]
    c = ctypes.c_double
    lib().orc_update_properties(*N, c(rho0), c(rho1), c(mu0), c(mu1), _p(np.ascontiguousarray(alpha, np.float64)),
                                _u8(np.ascontiguousarray(ct, np.uint8)),
                                (ctypes.c_void_p * 3)(*(t.ctypes.data for t in fts)), _p(out["rho"]),
                                _p(out["inv_rho"]), _p(out["mu"]), p3(("fbx", "fby", "fbz")),
                                p3(("firx", "firy", "firz")), p3(("rhox", "rhoy", "rhoz")), p3(("mux", "muy", "muz")))
    return out


def poisson_beta_two_way(N, eps, fir, fb):
    """G_CFDDEMCoupling::update_poisson_beta_two_way (Coupling/G_CFDDEMCoupling.cu:
    419-460) on copies of fb: returns (fbx, fby, fbz) with f_b = eps_f f_inv_rho
    on the interior box faces."""
    out = [np.array(a, dtype=np.float64, order="C", copy=True) for a in fb]
    firs = [np.ascontiguousarray(a, np.float64) for a in fir]
    e = np.ascontiguousarray(eps, np.float64)
    lib().orc_poisson_beta_two_way(*N, _p(e), (ctypes.c_void_p * 3)(*(a.ctypes.data for a in firs)),
                                   (ctypes.c_void_p * 3)(*(a.ctypes.data for a in out)))
    return tuple(out)


def mass_flux(c):
    """G_SMACSolver::compute_mass_flux_from_alpha_flux (CFD/G_SMACSolver_VoF.cu:
    1708-1795), or its two-way form (:2472-2687) when c.eps_half is set, on a
    workloads.MassFluxCase: returns (mfx, mfy, mfz), copies of c.mf after the call."""
    keep = []

    def arr3(arrs, dtype=np.float64):
        if arrs is None:
            return (ctypes.c_void_p * 3)(None, None, None)
        out = []
        for a in arrs:
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            out.append(a.ctypes.data)
        return (ctypes.c_void_p * 3)(*out)

    m = c.mom
    mf = [np.array(a, dtype=np.float64, order="C", copy=True) for a in c.mf]
    bv = [np.ascontiguousarray(a, np.float64) for a in m.bc_v]
    bct = np.ascontiguousarray(m.bc_type, np.uint8)
    eh = None if c.eps_half is None else np.ascontiguousarray(c.eps_half, np.float64)
    d = ctypes.c_double
    lib().orc_mass_flux(*m.N, d(m.h[0]), d(m.h[1]), d(m.h[2]), d(m.dt), d(c.rho0), d(c.rho1), _u8(bct),
                        *(_p(a) for a in bv), arr3(m.ft, np.uint8), arr3(m.bcid, np.uint8), arr3(m.lam), arr3(m.v),
                        arr3(c.F), None if eh is None else _p(eh),
                        (ctypes.c_void_p * 3)(*(a.ctypes.data for a in mf)))
    return tuple(mf)
