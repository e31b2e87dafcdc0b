"""Shared builders for the tests: workload Case -> oracle RefGrid, golden I/O."""
from __future__ import annotations

import json
import os

import numpy as np

from mydemcfd_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def ref_grid(case, eps=None, eps_old=None, fs=None):
    from oracle import oracle as O
    sh = W.shapes(case.N)
    eps = np.ones(sh["cell"]) if eps is None else eps
    eps_old = np.ones(sh["cell"]) if eps_old is None else eps_old
    fsx, fsy, fsz = fs if fs is not None else (np.zeros(sh["x"]), np.zeros(sh["y"]), np.zeros(sh["z"]))
    return O.RefGrid(case.N, case.h, case.dt, case.vxs, case.vys, case.vzs, eps, eps_old,
                     case.fbx, case.fby, case.fbz, fsx, fsy, fsz, case.fbx, case.fby, case.fbz,
                     case.ct, case.fxt, case.fyt, case.fzt)


def oracle_solid_fraction(N, h, origin, spheres):
    from oracle import oracle as O
    return O.solid_fraction_spheres(N, h, origin, spheres)


def build_case(spec):
    spec = dict(spec)
    kind = spec.pop("kind")
    if kind == "plain":
        if "N" in spec:
            spec["N"] = tuple(spec["N"])
        return W.plain_case(**spec)
    if kind == "vof":
        return W.vof_case(**spec)
    if kind == "ibm":
        return W.ibm_case(solid_fraction=oracle_solid_fraction, rmin_cells=3.0, rmax_cells=6.0, **spec)
    raise ValueError(kind)


def golden_names():
    """Fixtures of the reference's solve (those of the calls around it excluded)."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and not f.startswith(("post", "vstar", "surface", "mom", "props", "beta", "flux")))


def surface_golden_names():
    """Fixtures of the reference's calc_surface_tension."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("surface"))


def surface_case_from_spec(spec):
    spec = dict(spec)
    spec["N"] = tuple(spec["N"])
    return W.surface_case(**spec)


def vstar_golden_names():
    """Fixtures of the reference's update_vstar_boundary."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("vstar"))


def post_golden_names():
    """Fixtures of the reference's update_boundary_ghost + make_face_gradp."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("post"))


def post_case_from_spec(spec):
    """workloads.post_case from a fixture's JSON spec (lists back to tuples)."""
    spec = dict(spec)
    for k in ("N", "sides", "g", "h"):
        if k in spec:
            spec[k] = tuple(spec[k])
    return W.post_case(**spec)


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(d["meta"]))
    return meta, {k: d[k] for k in d.files if k != "meta"}


def fluid_demeaned(p_interior, ct):
    m = W.interior(ct) == W.C_INTERIOR
    out = np.where(m, p_interior, 0.0)
    out[m] -= out[m].mean()
    return out


def rel_err(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def momentum_golden_names():
    """Fixtures of the reference's get_vof_vstar_rhouu_consistent."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("mom"))


def momentum_case_from_spec(spec):
    spec = dict(spec)
    for k in ("N", "sides", "g"):
        if k in spec:
            spec[k] = tuple(spec[k])
    return W.momentum_case(**spec)


def property_golden_names():
    """Fixtures of the reference's update_properties_by_alpha."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("props"))


def property_case_from_spec(spec):
    spec = dict(spec)
    spec["N"] = tuple(spec["N"])
    return W.property_case(**spec)


def beta_golden_names():
    """Fixtures of the reference's update_poisson_beta_two_way."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("beta"))


def beta_case_from_spec(spec):
    spec = dict(spec)
    spec["N"] = tuple(spec["N"])
    return W.beta_two_way_case(**spec)


def flux_golden_names():
    """Fixtures of the reference's compute_mass_flux_from_alpha_flux (one-way and two-way)."""
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("flux"))


def flux_case_from_spec(spec):
    spec = dict(spec)
    for k in ("N", "sides"):
        if k in spec:
            spec[k] = tuple(spec[k])
    return W.mass_flux_case(**spec)
