"""Seeded synthetic inputs for the projection, in the reference layout.

Arrays are numpy, shape (sz, sy, sx), x fastest (CFD/MyArray.h:43-51);
cells (N+2)^3, x-faces (Nx+3)(Ny+2)(Nz+2) and so on (gridMembers.def).

Random numbers: SplitMix64(seed) -> u = (bits >> 11) * 2^-53 -> 2u - 1,
uniform in [-1, 1); the i-th draw of a stream depends only on (seed, i), so
the same arrays come out on any host.

Workloads (the benchmark configurations; seeded synthetic fields with the stated
shapes stand in for simulation state):
  plain   - single phase, rho = 1 (f_b = 1 on interior faces), dt = 1,
            u* i.i.d. U[-1,1) on F_INTERIOR faces, 0 on the others
  vof     - a sphere of radius 0.25 L centred U[0.3,0.7]^3, alpha ramped
            linearly over 1.5 cells across the interface, density ratio
            rho1/rho0 (alpha = 1 inside), f_b = 1/(0.5(rho_L+rho_R))
  ibm     - `nsph` non-overlapping spheres, radii U[4,12] cells, centres
            uniform in the interior with rejection sampling; cells >= 99%
            solid (8^3 sub-samples) become C_SOLID with zero-flux faces
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

F_INTERIOR, F_BOUNDARY, F_GHOST = 0, 1, 2
C_INTERIOR, C_GHOST, C_SOLID = 0, 2, 3

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """Draws offset+1 .. offset+n of SplitMix64 seeded with `seed`."""
    i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int, offset: int = 0) -> np.ndarray:
    return (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def uniform_pm1(seed: int, n: int, offset: int = 0) -> np.ndarray:
    return 2.0 * uniform01(seed, n, offset) - 1.0


def substream(seed: int, tag: int) -> int:
    """Seed of an independent stream derived from (seed, tag)."""
    return int(splitmix64((seed * 0x100000001B3 + tag) & 0xFFFFFFFFFFFFFFFF, 1)[0])


# ---------------------------------------------------------------------------
def shapes(N):
    nx, ny, nz = N
    return {
        "cell": (nz + 2, ny + 2, nx + 2),
        "x": (nz + 2, ny + 2, nx + 3),
        "y": (nz + 2, ny + 3, nx + 2),
        "z": (nz + 3, ny + 2, nx + 2),
    }


def box_types(N):
    """SMACSolver::set_face_type / set_cell_type (CFD/SMACSolver.cpp:104-248)."""
    nx, ny, nz = N
    sh = shapes(N)
    fxt = np.full(sh["x"], F_GHOST, np.uint8)
    fyt = np.full(sh["y"], F_GHOST, np.uint8)
    fzt = np.full(sh["z"], F_GHOST, np.uint8)
    fxt[1:nz + 1, 1:ny + 1, 1:nx + 2] = F_INTERIOR
    fxt[1:nz + 1, 1:ny + 1, 1] = F_BOUNDARY
    fxt[1:nz + 1, 1:ny + 1, nx + 1] = F_BOUNDARY
    fyt[1:nz + 1, 1:ny + 2, 1:nx + 1] = F_INTERIOR
    fyt[1:nz + 1, 1, 1:nx + 1] = F_BOUNDARY
    fyt[1:nz + 1, ny + 1, 1:nx + 1] = F_BOUNDARY
    fzt[1:nz + 2, 1:ny + 1, 1:nx + 1] = F_INTERIOR
    fzt[1, 1:ny + 1, 1:nx + 1] = F_BOUNDARY
    fzt[nz + 1, 1:ny + 1, 1:nx + 1] = F_BOUNDARY
    ct = np.full(sh["cell"], C_GHOST, np.uint8)
    ct[1:nz + 1, 1:ny + 1, 1:nx + 1] = C_INTERIOR
    return ct, fxt, fyt, fzt


def set_solid_cells(sf, ct, fxt, fyt, fzt):
    """k_set_solid_cell_from_ibm (CFD/G_SMACSolver_IBM.cu:763-792), in place."""
    solid = np.zeros(sf.shape, bool)
    solid[1:, 1:, 1:] = sf[1:, 1:, 1:] > 1.0 - 1e-12
    ct[solid] = C_SOLID
    z, y, x = np.nonzero(solid)
    fxt[z, y, x] = F_BOUNDARY
    fxt[z, y, x + 1] = F_BOUNDARY
    fyt[z, y, x] = F_BOUNDARY
    fyt[z, y + 1, x] = F_BOUNDARY
    fzt[z, y, x] = F_BOUNDARY
    fzt[z + 1, y, x] = F_BOUNDARY


def seeded_faces(N, seed, fxt, fyt, fzt):
    """Face field i.i.d. U[-1,1) on F_INTERIOR faces and 0 elsewhere (the
    wall rule of G_BoundaryFunctions.h:388-389: no-slip u* = 0)."""
    sh = shapes(N)
    out = []
    for tag, (key, t) in enumerate((("x", fxt), ("y", fyt), ("z", fzt))):
        n = int(np.prod(sh[key]))
        v = uniform_pm1(substream(seed, tag + 1), n).reshape(sh[key])
        v[t != F_INTERIOR] = 0.0
        out.append(np.ascontiguousarray(v))
    return tuple(out)


def face_coeffs_vof(N, alpha, rho0, rho1, ct, fxt, fyt, fzt):
    """k_update_cell_properties_by_alpha + k_update_*_face_properties_by_alpha
    (CFD/G_SMACSolver_VoF.cu:1374-1535) in numpy: same operations."""
    nx, ny, nz = N
    sh = shapes(N)
    rho = np.ones(sh["cell"])
    fluid = (ct == C_INTERIOR) | (ct == 1)
    fluid[0, :, :] = False
    fluid[:, 0, :] = False
    fluid[:, :, 0] = False
    rho[fluid] = (1.0 - alpha[fluid]) * rho0 + alpha[fluid] * rho1
    fbx = np.zeros(sh["x"])
    fby = np.zeros(sh["y"])
    fbz = np.zeros(sh["z"])
    m = fxt[:, :, 1:nx + 2] == F_INTERIOR
    fr = 0.5 * (rho[:, :, 1:nx + 2] + rho[:, :, 0:nx + 1])
    fbx[:, :, 1:nx + 2] = np.where(m, 1.0 / np.where(m, fr, 1.0), 0.0)
    m = fyt[:, 1:ny + 2, :] == F_INTERIOR
    fr = 0.5 * (rho[:, 1:ny + 2, :] + rho[:, 0:ny + 1, :])
    fby[:, 1:ny + 2, :] = np.where(m, 1.0 / np.where(m, fr, 1.0), 0.0)
    m = fzt[1:nz + 2, :, :] == F_INTERIOR
    fr = 0.5 * (rho[1:nz + 2, :, :] + rho[0:nz + 1, :, :])
    fbz[1:nz + 2, :, :] = np.where(m, 1.0 / np.where(m, fr, 1.0), 0.0)
    return rho, (fbx, fby, fbz)


def outlet_marks(N, sides):
    """Face marks for outlets on domain sides ("x-", "x+", "y-", ...): the
    boundary faces of that side get 1 (interior on the +1 side, low sides)
    or 2 (interior on the -1 side, high sides), the reference's
    f_*internal_id_ convention (CFD/G_SMACSolver_VoF.cu:1818-1833)."""
    nx, ny, nz = N
    sh = shapes(N)
    marks = {k: np.zeros(sh[k], dtype=np.uint8) for k in "xyz"}
    for s in sides:
        a, side = s[0], s[1]
        m = marks[a]
        if a == "x":
            m[1:nz + 1, 1:ny + 1, 1 if side == "-" else nx + 1] = 1 if side == "-" else 2
        elif a == "y":
            m[1:nz + 1, 1 if side == "-" else ny + 1, 1:nx + 1] = 1 if side == "-" else 2
        else:
            m[1 if side == "-" else nz + 1, 1:ny + 1, 1:nx + 1] = 1 if side == "-" else 2
    return marks["x"], marks["y"], marks["z"]


def constant_coeffs(N, fxt, fyt, fzt, value=1.0):
    """rho = 1 everywhere: f_b = 1 on F_INTERIOR faces, 0 on the others."""
    return tuple(np.where(t == F_INTERIOR, value, 0.0) for t in (fxt, fyt, fzt))


def cell_centres(N, h, origin=(0.0, 0.0, 0.0)):
    """StaggeredGrid::get_cell_coord (CFD/StaggeredGrid.h:121-142)."""
    nx, ny, nz = N
    x = h[0] * np.arange(nx + 2) - 0.5 * h[0] + origin[0]
    y = h[1] * np.arange(ny + 2) - 0.5 * h[1] + origin[1]
    z = h[2] * np.arange(nz + 2) - 0.5 * h[2] + origin[2]
    return x, y, z


def sphere_alpha(N, h, centre, radius, width_cells=1.5):
    """Volume fraction of a sphere: 1 inside, 0 outside, linear across a band
    of width_cells cells centred on the interface."""
    x, y, z = cell_centres(N, h)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    w = width_cells * min(h)
    return np.clip(0.5 - (r - radius) / w, 0.0, 1.0)


def random_spheres(N, h, seed, nsph=200, rmin_cells=4.0, rmax_cells=12.0, gap_cells=2.0, margin_cells=2.0,
                   max_tries=200000):
    """Non-overlapping spheres (x, y, z, r) in physical units, rejection sampled."""
    nx, ny, nz = N
    hmin = min(h)
    L = np.array([nx * h[0], ny * h[1], nz * h[2]])
    st = substream(seed, 77)
    spheres = []
    k = 0
    tries = 0
    while len(spheres) < nsph and tries < max_tries:
        u = uniform01(st, 4, offset=4 * k)
        k += 1
        tries += 1
        r = (rmin_cells + (rmax_cells - rmin_cells) * u[3]) * hmin
        lo = r + margin_cells * hmin
        c = lo + (L - 2 * lo) * u[:3]
        if np.any(L - 2 * lo <= 0):
            continue
        ok = True
        for s in spheres:
            if np.linalg.norm(c - s[:3]) < r + s[3] + gap_cells * hmin:
                ok = False
                break
        if ok:
            spheres.append(np.array([c[0], c[1], c[2], r]))
    return np.array(spheres).reshape(-1, 4)


@dataclass
class Case:
    """Inputs of one projection in the reference layout (host numpy)."""
    name: str
    N: tuple
    h: tuple
    dt: float
    vxs: np.ndarray
    vys: np.ndarray
    vzs: np.ndarray
    fbx: np.ndarray
    fby: np.ndarray
    fbz: np.ndarray
    ct: np.ndarray
    fxt: np.ndarray
    fyt: np.ndarray
    fzt: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def fir(self):
        return (self.fbx, self.fby, self.fbz)


def plain_case(n=64, seed=1, dt=1.0, N=None):
    N = tuple(N) if N is not None else (n, n, n)
    h = tuple(1.0 / N[0] for _ in range(3))
    ct, fxt, fyt, fzt = box_types(N)
    vxs, vys, vzs = seeded_faces(N, seed, fxt, fyt, fzt)
    fbx, fby, fbz = constant_coeffs(N, fxt, fyt, fzt)
    return Case(f"plain{N[0]}", N, h, dt, vxs, vys, vzs, fbx, fby, fbz, ct, fxt, fyt, fzt,
                {"seed": seed})


def vof_case(n=192, seed=3, ratio=1000.0, dt=1.0, width_cells=1.5, N=None):
    """The VoF sphere on the unit cube of n^3 cells, or of N = (nx, ny, nz)
    cells (spacing 1/nx, 1/ny, 1/nz) when N is given."""
    N = (n, n, n) if N is None else tuple(N)
    h = tuple(1.0 / m for m in N)
    ct, fxt, fyt, fzt = box_types(N)
    u = uniform01(substream(seed, 11), 3)
    centre = 0.3 + 0.4 * u
    alpha = sphere_alpha(N, h, centre, 0.25, width_cells)
    rho, (fbx, fby, fbz) = face_coeffs_vof(N, alpha, 1.0, ratio, ct, fxt, fyt, fzt)
    vxs, vys, vzs = seeded_faces(N, seed, fxt, fyt, fzt)
    name = f"vof{n}" if N == (n, n, n) else "vof{}x{}x{}".format(*N)
    return Case(name, N, h, dt, vxs, vys, vzs, fbx, fby, fbz, ct, fxt, fyt, fzt,
                {"seed": seed, "alpha": alpha, "rho": rho, "centre": centre, "ratio": ratio})


def ibm_case(n=256, seed=4, nsph=200, dt=1.0, solid_fraction=None, rmin_cells=4.0, rmax_cells=12.0):
    """`solid_fraction(N, h, origin, spheres)` computes the 8^3-sampled solid
    fraction (the GPU kernel or the oracle); it is required."""
    N = (n, n, n)
    h = (1.0 / n,) * 3
    spheres = random_spheres(N, h, seed, nsph=nsph, rmin_cells=rmin_cells, rmax_cells=rmax_cells)
    sf = solid_fraction(N, h, (0.0, 0.0, 0.0), spheres)
    ct, fxt, fyt, fzt = box_types(N)
    set_solid_cells(sf, ct, fxt, fyt, fzt)
    fbx, fby, fbz = constant_coeffs(N, fxt, fyt, fzt)
    vxs, vys, vzs = seeded_faces(N, seed, fxt, fyt, fzt)
    return Case(f"ibm{n}", N, h, dt, vxs, vys, vzs, fbx, fby, fbz, ct, fxt, fyt, fzt,
                {"seed": seed, "spheres": spheres, "sf": sf, "solid_cells": int((ct == C_SOLID).sum())})


def interior(a):
    """Interior block of a reference-layout cell array."""
    return a[1:-1, 1:-1, 1:-1]


def demean_fluid(p, ct):
    """p minus its mean over C_INTERIOR cells (interior block returned)."""
    pi = interior(p).copy()
    m = interior(ct) == C_INTERIOR
    pi[m] -= pi[m].mean()
    pi[~m] = 0.0
    return pi


# Boundary types, CFD/Enums.h:10-16
BC_NOSLIP, BC_SLIP, BC_INFLOW, BC_OUTFLOW, BC_OUTLET = 0, 1, 2, 3, 4


@dataclass
class PostCase:
    """Inputs of the pass after the projection (update_boundary_ghost and
    make_face_gradp), all in the reference layout."""
    N: tuple
    h: tuple
    dt: float
    g: tuple
    bc_type: np.ndarray   # bc_.bcType_ per boundary id (uint8)
    bc_v: tuple           # bc_.vx_, vy_, vz_ per boundary id
    ct: np.ndarray
    ft: tuple             # f_xtype_, f_ytype_, f_ztype_
    bcid: tuple           # f_*bcid_ (uint8)
    marks: tuple          # outlet marks: 1 interior side +1, 2 interior side -1
    internal_id: tuple    # f_*internal_id_ (int32): +1 / -1 on outlet faces, 0 elsewhere
    lam: tuple            # f_ibm_area_solid_fraction_* (or None)
    p: np.ndarray
    p_delta: np.ndarray
    rho: np.ndarray
    vs: tuple             # v*
    fb: tuple
    v: tuple              # velocity after the correction


def post_case(N, seed, h=(0.03125, 0.03125, 0.03125), dt=0.5, g=(0.0, -1.5, -9.8), sides=("x+", "z-"),
              solid_fraction=0.0, lam=True, solid_margin=2):
    """Seeded inputs for the post-projection pass.  Boundary ids 0..4 carry
    the types NOSLIP, SLIP, INFLOW, OUTFLOW, OUTLET with U[-1,1) boundary
    velocities; every face gets a U{0..3} id except the outlet faces of
    `sides`, which get id 4 (so the marks and the ids agree).  With
    solid_fraction > 0 that share of the cells m..N+1-m, m = solid_margin
    (in clusters, so some have no interior neighbour) become C_SOLID.  Fields are U[-1,1) (rho in
    [1, 1000), f_b in [0.1, 1) on F_INTERIOR faces, lam in [0, 1))."""
    N = tuple(int(n) for n in N)
    sh = shapes(N)
    rnd = lambda tag, key, lo=-1.0, hi=1.0: (lo + (hi - lo) * uniform01(substream(seed, tag),  # noqa: E731
                                                                         int(np.prod(sh[key])))).reshape(sh[key])
    ct, fxt, fyt, fzt = box_types(N)
    if solid_fraction > 0.0:
        nx, ny, nz = N
        # clusters: coarse blocks of 2^3 cells switched on together, then thinned
        blk = (uniform01(substream(seed, 90), int(np.prod(sh["cell"]))).reshape(sh["cell"]) < solid_fraction)
        coarse = blk[::2, ::2, ::2]
        dense = np.repeat(np.repeat(np.repeat(coarse, 2, 0), 2, 1), 2, 2)[:sh["cell"][0], :sh["cell"][1],
                                                                           :sh["cell"][2]]
        thin = uniform01(substream(seed, 91), int(np.prod(sh["cell"]))).reshape(sh["cell"]) < 0.85
        sf = np.zeros(sh["cell"])
        inner = np.zeros(sh["cell"], bool)
        m = solid_margin
        inner[m:nz + 2 - m, m:ny + 2 - m, m:nx + 2 - m] = True
        sf[inner & dense & thin] = 1.0
        set_solid_cells(sf, ct, fxt, fyt, fzt)
    marks = outlet_marks(N, sides)
    bcid = []
    for tag, (key, m) in enumerate(zip("xyz", marks)):
        ids = np.minimum((uniform01(substream(seed, 10 + tag), int(np.prod(sh[key]))) * 4).astype(np.uint8),
                         3).reshape(sh[key])
        ids[m != 0] = BC_OUTLET
        bcid.append(np.ascontiguousarray(ids))
    internal_id = tuple(np.where(m == 1, 1, np.where(m == 2, -1, 0)).astype(np.int32) for m in marks)
    bc_type = np.array([BC_NOSLIP, BC_SLIP, BC_INFLOW, BC_OUTFLOW, BC_OUTLET], np.uint8)
    bc_v = tuple(uniform_pm1(substream(seed, 20 + k), 5) for k in range(3))
    lam_t = tuple(np.ascontiguousarray(rnd(30 + k, key, 0.0, 1.0)) for k, key in enumerate("xyz")) if lam else None
    fb = tuple(np.where(t == F_INTERIOR, rnd(40 + k, key, 0.1, 1.0), 0.0) for k, (key, t) in
               enumerate(zip("xyz", (fxt, fyt, fzt))))
    return PostCase(N=N, h=tuple(float(x) for x in h), dt=float(dt), g=tuple(float(x) for x in g),
                    bc_type=bc_type, bc_v=bc_v, ct=ct, ft=(fxt, fyt, fzt), bcid=tuple(bcid), marks=marks,
                    internal_id=internal_id, lam=lam_t, p=rnd(50, "cell"), p_delta=rnd(51, "cell"),
                    rho=rnd(52, "cell", 1.0, 1000.0),
                    vs=tuple(np.ascontiguousarray(rnd(60 + k, key)) for k, key in enumerate("xyz")),
                    fb=tuple(np.ascontiguousarray(a) for a in fb),
                    v=tuple(np.ascontiguousarray(rnd(70 + k, key)) for k, key in enumerate("xyz")))


def surface_case(N, seed, kind="sphere", solid_fraction=0.0, sigma=0.07, h=0.03125):
    # h: one spacing, or three (powers of two keep the reference's (N h) / N exact)
    """Inputs of the surface-tension force: (N, h, alpha, ct, sigma).
    kind "sphere": a sphere of radius 0.3 of the smallest extent, centred
    U[0.35, 0.65] of the box, alpha ramped over 1.5 cells; kind "random":
    alpha U[0,1) with 30% set to 0, 20% to 1 and 10% within 1e-3 of the
    0.01 / 0.99 thresholds.  solid_fraction > 0 turns that share of the cells
    2..N-1 C_SOLID (single cells).  h is a power of two, so the reference's
    spacing (N h) / N equals it."""
    N = tuple(int(n) for n in N)
    hh = tuple(float(x) for x in h) if np.ndim(h) else (float(h),) * 3
    sh = shapes(N)
    ncell = int(np.prod(sh["cell"]))
    ct, fxt, fyt, fzt = box_types(N)
    if kind == "sphere":
        u = uniform01(substream(seed, 80), 3)
        ext = np.array(N, np.float64) * np.array(hh)
        centre = (0.35 + 0.3 * u) * ext
        alpha = sphere_alpha(N, hh, centre, 0.3 * ext.min(), 1.5)
    else:
        u = uniform01(substream(seed, 81), ncell)
        v = uniform01(substream(seed, 82), ncell)
        alpha = u.copy()
        alpha[v < 0.3] = 0.0
        alpha[(v >= 0.3) & (v < 0.5)] = 1.0
        near = (v >= 0.5) & (v < 0.6)
        alpha[near] = np.where(u[near] < 0.5, 0.01, 0.99) + (u[near] - 0.5) * 2e-3
        alpha = alpha.reshape(sh["cell"])
    if solid_fraction > 0.0:
        nx, ny, nz = N
        w = uniform01(substream(seed, 83), ncell).reshape(sh["cell"])
        inner = np.zeros(sh["cell"], bool)
        inner[2:nz, 2:ny, 2:nx] = True
        sf = np.where(inner & (w < solid_fraction), 1.0, 0.0)
        set_solid_cells(sf, ct, fxt, fyt, fzt)
    return N, hh, np.ascontiguousarray(alpha), ct, float(sigma)


@dataclass
class MomentumCase:
    """Inputs of the momentum predictor u* (get_vof_vstar_rhouu_consistent),
    reference layout; lam / imp / sf may be None (zero)."""
    N: tuple
    h: tuple
    dt: float
    g: tuple
    bc_type: np.ndarray
    bc_v: tuple
    ct: np.ndarray
    ft: tuple
    bcid: tuple
    lam: tuple
    v: tuple       # f_v*_ at time n
    mf: tuple      # f_mf*_: advecting face velocities
    muf: tuple     # f_mu*_: face viscosities
    mu: np.ndarray
    rho_old: np.ndarray
    p: np.ndarray
    fb: tuple      # f_b*: 1/rho on faces
    imp: tuple     # f_coupling_impulse_*
    sf: tuple      # f_ibm_solid_fraction_*
    vs: tuple      # f_v*_star_ before the call (faces it does not write keep these)
    # the two-way-coupled predictor only (None: the one-way form)
    eps_old: np.ndarray | None = None  # void_fraction_old_
    eps_new: np.ndarray | None = None  # void_fraction_
    fir: tuple | None = None           # f_inv_rho*_


def momentum_case(N, seed, sides=("x+", "z-"), solid_fraction=0.0, extras=True, dt=0.01, g=(0.0, 0.0, -9.8),
                  h=(0.03125, 0.03125, 0.03125), two_way=False):
    """Seeded momentum-predictor inputs on the boundary set-up of post_case
    (all five boundary types, outlets on `sides`, clustered solids).  Fields:
    v, v* U[-1,1); mf U[-1,1) with 10% exact zeros (the flux-sign ties);
    face and cell viscosities U[1e-3, 1e-2); rho_old U[1, 1000); p U[-1,1);
    f_b U[1e-3, 1); with extras the coupling impulse U[-1e-6, 1e-6), the IBM
    area and solid fractions U[0,1) with half of them 0.  two_way adds the
    void fractions eps_old, eps_new U[0.4, 1) and f_inv_rho U[1e-3, 1)."""
    base = post_case(N, seed, h=h, dt=dt, g=g, sides=sides, solid_fraction=solid_fraction, lam=extras,
                     solid_margin=3)
    sh = shapes(base.N)

    def rnd(tag, key, lo=-1.0, hi=1.0):
        n = int(np.prod(sh[key]))
        return np.ascontiguousarray((lo + (hi - lo) * uniform01(substream(seed, tag), n)).reshape(sh[key]))

    def half_zero(a, tag):
        return np.where(uniform01(substream(seed, tag), a.size).reshape(a.shape) < 0.5, 0.0, a)

    def extra(t0, lo, hi):
        if not extras:
            return None
        return tuple(np.ascontiguousarray(half_zero(rnd(t0 + k, key, lo, hi), t0 + 10 + k))
                     for k, key in enumerate("xyz"))

    mf = []
    for k, key in enumerate("xyz"):
        a = rnd(100 + k, key)
        a[uniform01(substream(seed, 110 + k), a.size).reshape(a.shape) < 0.1] = 0.0
        mf.append(a)
    return MomentumCase(
        N=base.N, h=base.h, dt=base.dt, g=base.g, bc_type=base.bc_type, bc_v=base.bc_v, ct=base.ct, ft=base.ft,
        bcid=base.bcid, lam=base.lam,
        v=tuple(rnd(120 + k, key) for k, key in enumerate("xyz")), mf=tuple(mf),
        muf=tuple(rnd(130 + k, key, 1e-3, 1e-2) for k, key in enumerate("xyz")),
        mu=rnd(140, "cell", 1e-3, 1e-2), rho_old=rnd(141, "cell", 1.0, 1000.0), p=rnd(142, "cell"),
        fb=tuple(rnd(150 + k, key, 1e-3, 1.0) for k, key in enumerate("xyz")),
        imp=extra(160, -1e-6, 1e-6), sf=extra(180, 0.0, 1.0),
        vs=tuple(rnd(200 + k, key) for k, key in enumerate("xyz")),
        eps_old=rnd(210, "cell", 0.4, 1.0) if two_way else None,
        eps_new=rnd(211, "cell", 0.4, 1.0) if two_way else None,
        fir=tuple(rnd(212 + k, key, 1e-3, 1.0) for k, key in enumerate("xyz")) if two_way else None)


PROPERTY_KEYS = ("rho", "rho_old", "inv_rho", "mu", "fbx", "fby", "fbz", "firx", "firy", "firz", "rhox", "rhoy",
                 "rhoz", "mux", "muy", "muz")


def property_case(N, seed, solid_fraction=0.0, rho=(1.0, 1000.0), mu=(1e-3, 1e-1), mixed_types=False):
    """Inputs of the property update: alpha of a seeded sphere (1.5-cell
    ramp) plus 20% of the cells U[0,1); box types with clustered solids
    (post_case's rule); every output array filled with U[-1,1) beforehand,
    so that entries the update must not write are checked too.  mixed_types:
    30% of the C_INTERIOR cells become C_NEAR_BOUNDARY and 7% isolated
    C_SOLID cells (faces unchanged).  Returns
    (N, h, (rho0, rho1, mu0, mu1), alpha, ct, ft, init)."""
    base = post_case(N, seed, sides=(), solid_fraction=solid_fraction)
    if mixed_types:
        ct = base.ct.copy()
        inside = ct[1:-1, 1:-1, 1:-1]
        u = uniform01(substream(seed, 900), inside.size).reshape(inside.shape)
        inside[(inside == C_INTERIOR) & (u < 0.3)] = 1   # C_NEAR_BOUNDARY
        inside[(inside == C_INTERIOR) & (u > 0.93)] = C_SOLID
        base = PostCase(**{**base.__dict__, "ct": ct})
    N = base.N
    sh = shapes(N)
    n = int(np.prod(sh["cell"]))
    u = uniform01(substream(seed, 300), 3)
    ext = np.array(N, np.float64) * np.array(base.h)
    alpha = sphere_alpha(N, base.h, (0.3 + 0.4 * u) * ext, 0.25 * ext.min(), 1.5)
    mix = uniform01(substream(seed, 301), n).reshape(sh["cell"]) < 0.2
    alpha = np.where(mix, uniform01(substream(seed, 302), n).reshape(sh["cell"]), alpha)
    init = {}
    for k, key in enumerate(PROPERTY_KEYS):
        kind = "cell" if key in ("rho", "rho_old", "inv_rho", "mu") else key[-1]
        init[key] = uniform_pm1(substream(seed, 310 + k), int(np.prod(sh[kind]))).reshape(sh[kind])
    return N, base.h, (rho[0], rho[1], mu[0], mu[1]), np.ascontiguousarray(alpha), base.ct, base.ft, init


def beta_two_way_case(N, seed, h=(0.03125, 0.03125, 0.03125)):
    """Inputs of the two-way Poisson coefficients: void fraction U[0.4, 1) on
    the cells, f_inv_rho U[1e-3, 1) and f_b U[-1, 1) (its value before the
    call) on the faces.  Returns (N, h, eps, fir, fb)."""
    N = tuple(int(n) for n in N)
    sh = shapes(N)

    def rnd(tag, key, lo, hi):
        n = int(np.prod(sh[key]))
        return np.ascontiguousarray((lo + (hi - lo) * uniform01(substream(seed, tag), n)).reshape(sh[key]))

    eps = rnd(400, "cell", 0.4, 1.0)
    fir = tuple(rnd(401 + k, key, 1e-3, 1.0) for k, key in enumerate("xyz"))
    fb = tuple(rnd(404 + k, key, -1.0, 1.0) for k, key in enumerate("xyz"))
    return N, tuple(h), eps, fir, fb


@dataclass
class MassFluxCase:
    """Inputs of the mass-flux update (compute_mass_flux_from_alpha_flux):
    the face rule's fields and dt of a MomentumCase, the accumulated
    volume-fraction flux F, rho0 / rho1, the mass flux before the call, and
    (two-way) void_fraction_half_."""
    mom: MomentumCase
    F: tuple
    rho0: float
    rho1: float
    mf: tuple
    eps_half: np.ndarray | None = None


def mass_flux_case(N, seed, sides=("x+", "z-"), solid_fraction=0.0, extras=True, two_way=False, rho=(1.0, 1000.0)):
    """Seeded mass-flux inputs: momentum_case's faces and velocities, F
    U[-0.5, 0.5) on every face, the previous mf U[-1, 1), void_fraction_half_
    U[0.4, 1) for the two-way form."""
    m = momentum_case(N, seed, sides=sides, solid_fraction=solid_fraction, extras=extras)
    sh = shapes(m.N)

    def rnd(tag, key, lo, hi):
        n = int(np.prod(sh[key]))
        return np.ascontiguousarray((lo + (hi - lo) * uniform01(substream(seed, tag), n)).reshape(sh[key]))

    return MassFluxCase(mom=m, F=tuple(rnd(500 + k, key, -0.5, 0.5) for k, key in enumerate("xyz")),
                        rho0=rho[0], rho1=rho[1], mf=tuple(rnd(510 + k, key, -1.0, 1.0) for k, key in enumerate("xyz")),
                        eps_half=rnd(520, "cell", 0.4, 1.0) if two_way else None)
