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


def solve(case, solver_type=3, tol=1e-11, levels=4, do_correct=True, eps=None, eps_old=None, fs=None):
    """Run the reference's solve_poisson (+ correct_vof_velocity) on a
    mydemcfd_b200.workloads.Case.  eps defaults to 1 (the reference's
    standalone driver leaves it at 0, which zeroes the divergence term)."""
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
    rc = lib().ref_solve(ctypes.byref(i), ctypes.byref(o))
    if rc != 0:
        raise RuntimeError(f"ref_solve returned {rc}")
    out["iterations"] = o.iterations
    out["num_levels"] = o.num_levels
    out["solve_ms"] = o.solve_ms
    out["correct_ms"] = o.correct_ms
    return out
