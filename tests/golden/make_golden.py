"""Generate the golden vectors of tests/golden/ by running the REFERENCE's own
GPU pressure path (oracle/_ref/libref_smac.so, built from the reference
sources by `make -C oracle ref`) on seeded inputs.

Needs a CUDA device.  Inputs are NOT stored: they are regenerated from the
seeds by mydemcfd_b200.workloads (SplitMix64), so a fixture holds only the
reference's outputs and the parameters that produced them.

    python tests/golden/make_golden.py --out tests/golden
    python tests/golden/make_golden.py --out tests/golden --post-only
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mydemcfd_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import ref as REF  # noqa: E402

# (name, builder kwargs, solver_type, tol, levels, store velocities)
CASES = [
    ("plain24_s7_gmg", dict(kind="plain", n=24, seed=7), 3, 1e-11, 4, True),
    ("plain32_s1_gmg", dict(kind="plain", n=32, seed=1), 3, 1e-11, 4, False),
    ("plain48_s2_gmg", dict(kind="plain", n=48, seed=2), 3, 1e-9, 4, False),
    ("plain24_s5_jacobi", dict(kind="plain", n=24, seed=5), 1, 1e-10, 4, False),
    ("plain24_s6_gmg_nomean", dict(kind="plain", n=24, seed=6), 2, 1e-10, 4, False),
    ("plain32x24x48_s8_gmg", dict(kind="plain", N=(32, 24, 48), seed=8), 3, 1e-10, 4, False),
    ("vof32_s3_r1000", dict(kind="vof", n=32, seed=3, ratio=1000.0), 3, 1e-9, 4, False),
    ("ibm48_s4", dict(kind="ibm", n=48, seed=4, nsph=6), 3, 1e-9, 4, False),
    ("plain64_s1_gmg", dict(kind="plain", n=64, seed=1), 3, 1e-11, 4, False),  # config 1, stored sparsely
]


# The pass after the projection (update_boundary_ghost + make_face_gradp):
# (name, workloads.post_case kwargs); every output array is stored.
POST_CASES = [
    ("post12x10x8_s1", dict(N=(12, 10, 8), seed=1, sides=("x+", "z-"))),
    ("post16_s2_solid", dict(N=(16, 16, 16), seed=2, sides=("x-", "y+"), solid_fraction=0.35)),
    ("post9x7x11_s3_nolam", dict(N=(9, 7, 11), seed=3, sides=("x+", "y-", "z+"), lam=False, g=(0.3, 0.0, -9.8))),
]

# The wall u* rule before the projection (update_vstar_boundary); solids keep
# off the outlets' neighbours (an outlet face reading an F_BOUNDARY face is a
# race in the reference).
VSTAR_CASES = [
    ("vstar12x10x8_s1", dict(N=(12, 10, 8), seed=1, sides=("x+", "z-"))),
    ("vstar16_s2_solid", dict(N=(16, 16, 16), seed=2, sides=("x-", "y+"), solid_fraction=0.35, solid_margin=3)),
    ("vstar9x7x11_s3_nolam", dict(N=(9, 7, 11), seed=3, sides=("x+", "y-", "z+"), lam=False)),
]

# The surface-tension force (calc_surface_tension): workloads.surface_case
# kwargs; the work arrays start at zero as the reference driver's do.
SURFACE_CASES = [
    ("surface24_s3_sphere", dict(N=(24, 24, 24), seed=3, kind="sphere")),
    ("surface20x16x12_s5_random", dict(N=(20, 16, 12), seed=5, kind="random", solid_fraction=0.15)),
    ("surface18x20x16_s6_sphere_solid", dict(N=(18, 20, 16), seed=6, kind="sphere", solid_fraction=0.1)),
]

# The momentum predictor (get_vof_vstar_rhouu_consistent): workloads.momentum_case kwargs.
MOMENTUM_CASES = [
    ("mom12x10x8_s1", dict(N=(12, 10, 8), seed=1, sides=("x+", "z-"))),
    ("mom16_s2_solid", dict(N=(16, 16, 16), seed=2, sides=("x-", "y+"), solid_fraction=0.3)),
    ("mom9x7x11_s3_noextras", dict(N=(9, 7, 11), seed=3, sides=("y-",), extras=False)),
    # the two-way-coupled form (get_vof_vstar_rhouu_consistent_two_way)
    ("mom2w12x10x8_s4", dict(N=(12, 10, 8), seed=4, sides=("x+", "z-"), two_way=True)),
    ("mom2w16_s5_solid", dict(N=(16, 16, 16), seed=5, sides=("x-", "y+"), solid_fraction=0.3, two_way=True)),
]

# The mass-flux update (compute_mass_flux_from_alpha_flux, one-way and two-way):
# workloads.mass_flux_case kwargs.
FLUX_CASES = [
    ("flux12x10x8_s1", dict(N=(12, 10, 8), seed=1, sides=("x+", "z-"))),
    ("flux9x7x11_s2_solid", dict(N=(9, 7, 11), seed=2, sides=("y-",), solid_fraction=0.3)),
    ("flux2w12x10x8_s3", dict(N=(12, 10, 8), seed=3, sides=("x-", "y+"), two_way=True)),
]

# The two-way Poisson coefficients (update_poisson_beta_two_way): workloads.beta_two_way_case kwargs.
BETA_CASES = [
    ("beta2w12x10x8_s1", dict(N=(12, 10, 8), seed=1)),
    ("beta2w7x9x5_s2", dict(N=(7, 9, 5), seed=2)),
]

# The property update (update_properties_by_alpha): workloads.property_case kwargs.
PROPERTY_CASES = [
    ("props12x10x8_s1", dict(N=(12, 10, 8), seed=1)),
    ("props16_s2_solid", dict(N=(16, 16, 16), seed=2, solid_fraction=0.35)),
]


def oracle_solid_fraction(N, h, origin, spheres):
    return O.solid_fraction_spheres(N, h, origin, spheres)


def build_case(spec):
    spec = dict(spec)
    kind = spec.pop("kind")
    if kind == "plain":
        return W.plain_case(**spec)
    if kind == "vof":
        return W.vof_case(**spec)
    if kind == "ibm":
        return W.ibm_case(solid_fraction=oracle_solid_fraction, rmin_cells=3.0, rmax_cells=6.0, **spec)
    raise ValueError(kind)


def sparse_sample(a, stride=97):
    flat = a.reshape(-1)
    idx = np.arange(0, flat.size, stride)
    return idx, flat[idx]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--post-only", action="store_true",
                    help="only the fixtures of the calls either side of the projection")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    post_index = {}
    for name, spec in POST_CASES:
        r = REF.post(W.post_case(**spec))
        arrays = {k: v for k, v in r.items() if isinstance(v, np.ndarray)}  # outputs, not the timings
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), **arrays)
        post_index[name] = spec
        print(name, spec, flush=True)
    for name, spec in VSTAR_CASES:
        vxs, vys, vzs, _ = REF.vstar(W.post_case(**spec))
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), vxs=vxs,
                            vys=vys, vzs=vzs)
        post_index[name] = spec
        print(name, spec, flush=True)
    for name, spec in SURFACE_CASES:
        N, h, alpha, ct, sigma = W.surface_case(**spec)
        fsx, fsy, fsz, nx, ny, nz, kappa, gm, _ = REF.surface_tension(N, h, alpha, ct, sigma)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), fsx=fsx, fsy=fsy,
                            fsz=fsz, nx=nx, ny=ny, nz=nz, kappa=kappa, gm=gm)
        post_index[name] = spec
        print(name, spec, flush=True)
    for name, spec in MOMENTUM_CASES:
        vxs, vys, vzs, _ = REF.predict_vstar(W.momentum_case(**spec))
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), vxs=vxs,
                            vys=vys, vzs=vzs)
        post_index[name] = spec
        print(name, spec, flush=True)
    for name, spec in PROPERTY_CASES:
        N, h, (r0, r1, m0, m1), alpha, ct, ft, init = W.property_case(**spec)
        out, _ = REF.update_properties(N, h, r0, r1, m0, m1, alpha, ct, ft, init)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), **out)
        post_index[name] = spec
        print(name, spec, flush=True)
    for name, spec in FLUX_CASES:
        mfx, mfy, mfz, _ = REF.mass_flux(W.mass_flux_case(**spec))
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), mfx=mfx, mfy=mfy,
                            mfz=mfz)
        post_index[name] = spec
        print(name, spec, flush=True)
    for name, spec in BETA_CASES:
        N, h, eps, fir, fb = W.beta_two_way_case(**spec)
        fbx, fby, fbz, _ = REF.poisson_beta_two_way(N, h, eps, fir, fb)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), meta=np.array(json.dumps(spec)), fbx=fbx, fby=fby,
                            fbz=fbz)
        post_index[name] = spec
        print(name, spec, flush=True)
    with open(os.path.join(args.out, "post_index.json"), "w") as f:
        json.dump(post_index, f, indent=1, sort_keys=True)
    if args.post_only:
        return
    index = {}
    for name, spec, st, tol, levels, store_v in CASES:
        case = build_case(spec)
        r = REF.solve(case, solver_type=st, tol=tol, levels=levels, do_correct=True)
        meta = {"spec": spec, "solver_type": st, "tol": tol, "levels": levels, "iterations": r["iterations"],
                "num_levels": r["num_levels"], "N": list(case.N), "dt": case.dt}
        pd = W.interior(r["p_delta"])
        rhs = W.interior(r["rhs"])
        arrays = {"meta": np.array(json.dumps(meta))}
        if case.N[0] * case.N[1] * case.N[2] <= 32 ** 3:
            arrays["p_delta"] = pd
            arrays["rhs"] = rhs
        else:
            idx, val = sparse_sample(pd)
            arrays["p_delta_idx"], arrays["p_delta_val"] = idx, val
            idx, val = sparse_sample(rhs)
            arrays["rhs_idx"], arrays["rhs_val"] = idx, val
            arrays["p_delta_norm"] = np.array(np.linalg.norm(pd))
            arrays["p_delta_mean"] = np.array(pd.mean())
        if store_v:
            arrays["vx"], arrays["vy"], arrays["vz"] = r["vx"], r["vy"], r["vz"]
            arrays["p"] = r["p"]
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **arrays)
        index[name] = meta
        print(name, meta, flush=True)
    with open(os.path.join(args.out, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
