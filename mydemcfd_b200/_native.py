"""ctypes binding of libsmac_b200.so (the C ABI in include/smac_b200.h).

The library is the only compute path: if it is missing or cannot be loaded
every entry point raises; there is no fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsmac_b200.so")

# smac_status
OK, NOT_CONVERGED, BREAKDOWN, NAN, BAD_ARG, BAD_SHAPE, CUDA_ERROR, NO_DEVICE = range(8)
STATUS_NAMES = {
    OK: "OK", NOT_CONVERGED: "NOT_CONVERGED", BREAKDOWN: "BREAKDOWN", NAN: "NAN", BAD_ARG: "BAD_ARG",
    BAD_SHAPE: "BAD_SHAPE", CUDA_ERROR: "CUDA_ERROR", NO_DEVICE: "NO_DEVICE",
}
# smac_solver_type == the reference's PCG_TYPES (CFD/Enums.h:25-30)
STANDARD_PCG, PURENEUMANN_STANDARD_PCG, GMG_PCG, PURENEUMANN_GMG_PCG = range(4)
PRECISION_FP64, PRECISION_MIXED = 0, 1
STOP_RELATIVE, STOP_REFERENCE = 0, 1
SWEEP_AUTO, SWEEP_TMA, SWEEP_ZMARCH, SWEEP_SHARED = range(4)
COARSE_AUTO, COARSE_CTA = range(2)


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [
        ("solver_type", ctypes.c_int), ("precision", ctypes.c_int), ("stop_rule", ctypes.c_int),
        ("tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("min_coarse", ctypes.c_int),
        ("max_levels", ctypes.c_int), ("nu1", ctypes.c_int), ("nu2", ctypes.c_int),
        ("coarse_sweeps", ctypes.c_int), ("check_every", ctypes.c_int), ("reliable_delta", ctypes.c_double),
        ("bf16_coarse_cells", ctypes.c_int), ("sweep_kernel", ctypes.c_int), ("coarse_kernel", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("iterations", ctypes.c_int), ("reliable_updates", ctypes.c_int),
        ("num_levels", ctypes.c_int), ("norm_b", ctypes.c_double), ("rel_residual", ctypes.c_double),
        ("max_residual", ctypes.c_double), ("alg_bytes", ctypes.c_double), ("kernel_launches", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BoundaryTable(ctypes.Structure):
    """smac_boundary_table: the bc_ table (HOST arrays)."""
    _fields_ = [("num_ids", ctypes.c_int), ("type", ctypes.c_void_p), ("vx", ctypes.c_void_p),
                ("vy", ctypes.c_void_p), ("vz", ctypes.c_void_p)]


class MomentumFields(ctypes.Structure):
    """smac_momentum_fields: the device arrays the momentum predictor reads."""
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "fxt", "fyt", "fzt", "fxbcid", "fybcid", "fzbcid", "lamx", "lamy", "lamz", "vx", "vy", "vz",
        "mfx", "mfy", "mfz", "mux", "muy", "muz", "mu", "rho_old", "p", "fbx", "fby", "fbz",
        "impx", "impy", "impz", "sfx", "sfy", "sfz")]


class TwoWayFields(ctypes.Structure):
    """smac_two_way_fields: the void fractions and f_inv_rho of the two-way predictor."""
    _fields_ = [(k, ctypes.c_void_p) for k in ("eps_old", "eps_new", "inv_rhox", "inv_rhoy", "inv_rhoz")]


class MassFluxFields(ctypes.Structure):
    """smac_mass_flux_fields: the inputs of the mass-flux update."""
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "fxt", "fyt", "fzt", "fxbcid", "fybcid", "fzbcid", "lamx", "lamy", "lamz", "vx", "vy", "vz",
        "Fx", "Fy", "Fz")]


class VofParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("rho0", "rho1", "mu0", "mu1")]


class PropertyFields(ctypes.Structure):
    """smac_property_fields: the outputs of the property update."""
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "rho", "inv_rho", "mu", "fbx", "fby", "fbz", "firx", "firy", "firz", "rhox", "rhoy", "rhoz",
        "mux", "muy", "muz")]


class SmacError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None

# every symbol include/smac_b200.h declares
EXPORTS = [
    "smac_default_options", "smac_create", "smac_destroy", "smac_set_options", "smac_last_error_string",
    "smac_level_shape", "smac_set_coefficients", "smac_box_types", "smac_assemble_vof",
    "smac_ibm_solid_fraction_spheres", "smac_ibm_set_solid_cells", "smac_divergence", "smac_solve",
    "smac_set_rhs", "smac_correct", "smac_project", "smac_project_adjoint", "smac_apply_A", "smac_time_kernel",
    "smac_selftest_sweep", "smac_selftest_wait", "smac_apply_A_dot_noalloc", "smac_async_create", "smac_async_submit",
    "smac_async_wait", "smac_async_destroy", "smac_update_boundary_faces", "smac_update_pressure_ghost",
    "smac_update_velocity_ghost", "smac_face_gradp", "smac_update_vstar_boundary", "smac_surface_tension",
    "smac_predict_vstar", "smac_predict_vstar_two_way", "smac_poisson_beta_two_way", "smac_mass_flux_from_alpha_flux",
    "smac_vti_block_bytes", "smac_vti_pack", "smac_vti_write", "smac_update_properties",
]


def load(path: str = LIB_PATH):
    """Load the native library (build it first with mydemcfd_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"native library {path} is missing: run `python -m mydemcfd_b200.build`")
    lib = ctypes.CDLL(path)
    vp, dp, u8p, ip = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int
    d = ctypes.c_double
    sig = {
        "smac_default_options": [ctypes.POINTER(Options)],
        "smac_create": [ctypes.POINTER(GridDesc), ctypes.POINTER(Options), vp, ctypes.POINTER(vp)],
        "smac_destroy": [vp],
        "smac_set_options": [vp, ctypes.POINTER(Options)],
        "smac_level_shape": [vp, ip, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)],
        "smac_set_coefficients": [vp, dp, dp, dp, u8p, u8p, u8p, u8p],
        "smac_box_types": [ctypes.POINTER(GridDesc), u8p, u8p, u8p, u8p, vp],
        "smac_assemble_vof": [ctypes.POINTER(GridDesc), dp, d, d, u8p, u8p, u8p, u8p, dp, dp, dp, dp, dp, dp, dp, vp],
        "smac_ibm_solid_fraction_spheres": [ctypes.POINTER(GridDesc), ctypes.POINTER(d), ctypes.POINTER(d), ip, dp,
                                            vp],
        "smac_ibm_set_solid_cells": [ctypes.POINTER(GridDesc), dp, u8p, u8p, u8p, u8p, vp],
        "smac_divergence": [vp, dp, dp, dp, dp, dp, dp, dp, dp, d, dp],
        "smac_solve": [vp, dp, ctypes.POINTER(Stats)],
        "smac_set_rhs": [vp, dp],
        "smac_correct": [vp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, d, dp, dp, dp, ip],
        "smac_project": [vp, dp, dp, dp, d, dp, dp, dp, dp, ctypes.POINTER(Stats)],
        "smac_project_adjoint": [vp, dp, dp, dp, dp, dp, dp, dp, ctypes.POINTER(Stats)],
        "smac_apply_A": [vp, dp, dp],
        "smac_time_kernel": [vp, ip, ip, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(d)],
        "smac_selftest_sweep": [vp, ip, ip, ctypes.POINTER(ctypes.c_longlong)],
        "smac_selftest_wait": [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)],
        "smac_apply_A_dot_noalloc": [ctypes.POINTER(GridDesc), dp, dp, dp, u8p, u8p, u8p, u8p, dp, dp, dp, vp],
        "smac_async_create": [vp, ctypes.POINTER(vp)],
        "smac_async_submit": [vp, dp, dp, dp, d, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_ulonglong)],
        "smac_async_wait": [vp, ctypes.c_ulonglong, ctypes.POINTER(Stats)],
        "smac_async_destroy": [vp],
        "smac_update_boundary_faces": [ctypes.POINTER(GridDesc), u8p, u8p, u8p, dp, dp, dp, vp],
        "smac_update_pressure_ghost": [ctypes.POINTER(GridDesc), u8p, dp, d, d, d, dp, vp],
        "smac_update_velocity_ghost": [ctypes.POINTER(GridDesc), ctypes.POINTER(BoundaryTable), u8p, u8p, u8p,
                                       u8p, u8p, u8p, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, d, dp, dp, dp, vp],
        "smac_face_gradp": [ctypes.POINTER(GridDesc), dp, dp, dp, dp, vp],
        "smac_surface_tension": [ctypes.POINTER(GridDesc), dp, u8p, d, dp, dp, dp, dp, dp, dp, dp, dp, vp],
        "smac_predict_vstar": [ctypes.POINTER(GridDesc), ctypes.POINTER(BoundaryTable), ctypes.POINTER(MomentumFields),
                               d, d, d, d, dp, dp, dp, vp],
        "smac_poisson_beta_two_way": [ctypes.POINTER(GridDesc), dp, dp, dp, dp, dp, dp, dp, vp],
        "smac_mass_flux_from_alpha_flux": [ctypes.POINTER(GridDesc), ctypes.POINTER(BoundaryTable),
                                           ctypes.POINTER(MassFluxFields), d, d, d, dp, dp, dp, dp, vp],
        "smac_predict_vstar_two_way": [ctypes.POINTER(GridDesc), ctypes.POINTER(BoundaryTable),
                                       ctypes.POINTER(MomentumFields), ctypes.POINTER(TwoWayFields), d, d, d, d, dp,
                                       dp, dp, vp],
        "smac_vti_pack": [ctypes.POINTER(GridDesc), dp, dp, dp, dp, dp, dp, vp, vp],
        "smac_update_properties": [ctypes.POINTER(GridDesc), ctypes.POINTER(VofParams), dp, u8p, u8p, u8p, u8p,
                                   ctypes.POINTER(PropertyFields), vp],
        "smac_vti_write": [ctypes.POINTER(GridDesc), ctypes.POINTER(d), vp, ctypes.c_char_p],
        "smac_update_vstar_boundary": [ctypes.POINTER(GridDesc), ctypes.POINTER(BoundaryTable), u8p, u8p, u8p, u8p,
                                       u8p, u8p, u8p, u8p, u8p, dp, dp, dp, dp, dp, dp, vp],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.smac_vti_block_bytes.restype = ctypes.c_size_t
    lib.smac_vti_block_bytes.argtypes = [ctypes.POINTER(GridDesc)]
    lib.smac_last_error_string.restype = ctypes.c_char_p
    lib.smac_last_error_string.argtypes = []
    _lib = lib
    return lib


def last_error() -> str:
    return load().smac_last_error_string().decode(errors="replace")


def check(status: int, allow=()):
    if status != OK and status not in allow:
        raise SmacError(status, last_error())
    return status


def default_options(**kw) -> Options:
    o = Options()
    check(load().smac_default_options(ctypes.byref(o)))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o
