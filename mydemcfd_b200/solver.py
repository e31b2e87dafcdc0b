"""Host-side mirror of the reference's pressure-solver seam over the C ABI.

Reference interface (CFD/pressure_solver/G_PressureSolverBase.h:24-42,
CFD/pressure_solver/G_PCGSolver.h:17-38, CFD/G_SMACSolver.h:9-125):

    struct G_PressureSolverBase { virtual void solve(G_SMACSolver&) = 0; double tol_; ... };
    struct G_PCGSolver : G_PressureSolverBase { void set_solver(PCG_TYPES); ... };
    G_SMACSolver::solve_poisson()          -> pressure_solver_->solve(*this)   (G_SMACSolver.cu:1499-1501)
    G_SMACSolver::correct_vof_velocity()   -> k_correct_vof_velocity; p_delta_ = 0 (G_SMACSolver.cu:1269-1275)

Here `DeviceGrid` holds the G_StaggeredGrid members the path reads or writes
as CUDA tensors in the reference layout, `B200PressureSolver` is the
G_PressureSolverBase replacement (same `tol_`, `set_solver`, `solve`), and
`SMACStep` carries the two G_SMACSolver calls.  All compute goes through
libsmac_b200.so; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat
from .workloads import Case, shapes


def _ptr(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "device tensors must be contiguous CUDA tensors"
    return ctypes.c_void_p(t.data_ptr())


def _dev(a, dtype, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


@dataclass
class DeviceGrid:
    """The G_StaggeredGrid members of the projection (CFD/memberList/gridMembers.def)."""
    Nx_: int
    Ny_: int
    Nz_: int
    dx_: float
    dy_: float
    dz_: float
    f_vx_star_: torch.Tensor
    f_vy_star_: torch.Tensor
    f_vz_star_: torch.Tensor
    f_bx_: torch.Tensor
    f_by_: torch.Tensor
    f_bz_: torch.Tensor
    f_inv_rhox_: torch.Tensor
    f_inv_rhoy_: torch.Tensor
    f_inv_rhoz_: torch.Tensor
    celltype_: torch.Tensor
    f_xtype_: torch.Tensor
    f_ytype_: torch.Tensor
    f_ztype_: torch.Tensor
    p_: torch.Tensor
    p_delta_: torch.Tensor
    rhs_: torch.Tensor
    f_vx_: torch.Tensor
    f_vy_: torch.Tensor
    f_vz_: torch.Tensor
    void_fraction_: torch.Tensor | None = None
    void_fraction_old_: torch.Tensor | None = None
    f_sx_: torch.Tensor | None = None
    f_sy_: torch.Tensor | None = None
    f_sz_: torch.Tensor | None = None
    # read or written only by the pass after the projection
    rho_: torch.Tensor | None = None
    f_xbcid_: torch.Tensor | None = None
    f_ybcid_: torch.Tensor | None = None
    f_zbcid_: torch.Tensor | None = None
    f_xoutlet_: torch.Tensor | None = None      # outlet marks (1 / 2: interior side +1 / -1)
    f_youtlet_: torch.Tensor | None = None
    f_zoutlet_: torch.Tensor | None = None
    f_ibm_area_solid_fraction_x_: torch.Tensor | None = None
    f_ibm_area_solid_fraction_y_: torch.Tensor | None = None
    f_ibm_area_solid_fraction_z_: torch.Tensor | None = None
    f_gradp_x_: torch.Tensor | None = None
    f_gradp_y_: torch.Tensor | None = None
    f_gradp_z_: torch.Tensor | None = None
    # read by the momentum predictor
    f_mfx_: torch.Tensor | None = None
    f_mfy_: torch.Tensor | None = None
    f_mfz_: torch.Tensor | None = None
    f_mux_: torch.Tensor | None = None
    f_muy_: torch.Tensor | None = None
    f_muz_: torch.Tensor | None = None
    mu_: torch.Tensor | None = None
    rho_old_: torch.Tensor | None = None
    # read by the mass-flux update (it writes f_mf*_)
    f_Fx_accum_: torch.Tensor | None = None
    f_Fy_accum_: torch.Tensor | None = None
    f_Fz_accum_: torch.Tensor | None = None
    void_fraction_half_: torch.Tensor | None = None
    # written by the property update (besides rho_, mu_, f_b*_, f_inv_rho*_, f_mu*_)
    inv_rho_: torch.Tensor | None = None
    f_rhox_: torch.Tensor | None = None
    f_rhoy_: torch.Tensor | None = None
    f_rhoz_: torch.Tensor | None = None
    f_coupling_impulse_x_: torch.Tensor | None = None
    f_coupling_impulse_y_: torch.Tensor | None = None
    f_coupling_impulse_z_: torch.Tensor | None = None
    f_ibm_solid_fraction_x_: torch.Tensor | None = None
    f_ibm_solid_fraction_y_: torch.Tensor | None = None
    f_ibm_solid_fraction_z_: torch.Tensor | None = None
    # read and written by the surface-tension force
    alpha_: torch.Tensor | None = None
    nx_: torch.Tensor | None = None
    ny_: torch.Tensor | None = None
    nz_: torch.Tensor | None = None
    kappa_: torch.Tensor | None = None
    p_tmp_: torch.Tensor | None = None

    @property
    def N(self):
        return (self.Nx_, self.Ny_, self.Nz_)

    @staticmethod
    def from_case(case: Case, device="cuda") -> "DeviceGrid":
        sh = shapes(case.N)
        f64, u8 = torch.float64, torch.uint8
        z = lambda k: torch.zeros(sh[k], dtype=f64, device=device)  # noqa: E731
        return DeviceGrid(
            *case.N, *case.h,
            f_vx_star_=_dev(case.vxs, f64, device), f_vy_star_=_dev(case.vys, f64, device),
            f_vz_star_=_dev(case.vzs, f64, device),
            f_bx_=_dev(case.fbx, f64, device), f_by_=_dev(case.fby, f64, device), f_bz_=_dev(case.fbz, f64, device),
            f_inv_rhox_=_dev(case.fbx, f64, device), f_inv_rhoy_=_dev(case.fby, f64, device),
            f_inv_rhoz_=_dev(case.fbz, f64, device),
            celltype_=_dev(case.ct, u8, device), f_xtype_=_dev(case.fxt, u8, device),
            f_ytype_=_dev(case.fyt, u8, device), f_ztype_=_dev(case.fzt, u8, device),
            p_=z("cell"), p_delta_=z("cell"), rhs_=z("cell"), f_vx_=z("x"), f_vy_=z("y"), f_vz_=z("z"),
        )


class B200PressureSolver:
    """Drop-in for G_PressureSolverBase / G_PCGSolver over libsmac_b200.so.

    `tol_` has the meaning of the chosen stop rule: by default the relative
    FP64 true residual ||b - A x|| / ||b||; with stop_rule=STOP_REFERENCE the
    reference's test max|r| * dt < tol_ (G_PCGSolver.cu:884-903).
    """

    def __init__(self, N, h, precision=nat.PRECISION_FP64, tol=1e-8, stream=None, **options):
        self._lib = nat.load()
        self.N = tuple(N)
        self.h = tuple(h)
        self.opts = nat.default_options(precision=precision, tol=tol, **options)
        self.desc = nat.GridDesc(*self.N, *self.h)
        self._stream = stream if stream is not None else torch.cuda.current_stream()
        handle = ctypes.c_void_p()
        nat.check(self._lib.smac_create(ctypes.byref(self.desc), ctypes.byref(self.opts),
                                        ctypes.c_void_p(self._stream.cuda_stream), ctypes.byref(handle)))
        self._h = handle
        self.last_stats: dict | None = None

    # -- G_PressureSolverBase surface -------------------------------------
    @property
    def tol_(self) -> float:
        return self.opts.tol

    @tol_.setter
    def tol_(self, v: float):
        self.opts.tol = float(v)
        self._apply()

    def set_solver(self, pcg_type: int):
        """G_PCGSolver::set_solver(PCG_TYPES) (G_PCGSolver.cu:592-613)."""
        self.opts.solver_type = int(pcg_type)
        self._apply()

    def set_options(self, **kw):
        for k, v in kw.items():
            setattr(self.opts, k, v)
        self._apply()

    def _apply(self):
        if getattr(self, "_h", None):
            nat.check(self._lib.smac_set_options(self._h, ctypes.byref(self.opts)))

    def solve(self, solv: "SMACStep", raise_on_fail=True) -> dict:
        """G_PressureSolverBase::solve(G_SMACSolver&): RHS from the grid, then
        the Poisson solve into grid.p_delta_."""
        g = solv.grid_
        self.set_coefficients(g)
        self.divergence(g, solv.dt_)
        return self.solve_rhs(g.p_delta_, raise_on_fail=raise_on_fail)

    # -- finer-grained calls ----------------------------------------------
    def set_coefficients(self, g: DeviceGrid):
        nat.check(self._lib.smac_set_coefficients(
            self._h, _ptr(g.f_bx_), _ptr(g.f_by_), _ptr(g.f_bz_), _ptr(g.celltype_), _ptr(g.f_xtype_),
            _ptr(g.f_ytype_), _ptr(g.f_ztype_)))

    def divergence(self, g: DeviceGrid, dt: float):
        nat.check(self._lib.smac_divergence(
            self._h, _ptr(g.f_vx_star_), _ptr(g.f_vy_star_), _ptr(g.f_vz_star_), _ptr(g.void_fraction_),
            _ptr(g.void_fraction_old_), _ptr(g.f_sx_), _ptr(g.f_sy_), _ptr(g.f_sz_), ctypes.c_double(dt),
            _ptr(g.rhs_)))

    def set_rhs(self, rhs: torch.Tensor):
        nat.check(self._lib.smac_set_rhs(self._h, _ptr(rhs)))

    def solve_rhs(self, p_delta: torch.Tensor, raise_on_fail=True) -> dict:
        st = nat.Stats()
        rc = self._lib.smac_solve(self._h, _ptr(p_delta), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if raise_on_fail:
            nat.check(rc)
        elif rc not in (nat.OK, nat.NOT_CONVERGED, nat.BREAKDOWN, nat.NAN):
            nat.check(rc)
        return self.last_stats

    def correct(self, g: DeviceGrid, dt: float, zero_p_delta=True):
        nat.check(self._lib.smac_correct(
            self._h, _ptr(g.p_delta_), _ptr(g.p_), _ptr(g.f_vx_star_), _ptr(g.f_vy_star_), _ptr(g.f_vz_star_),
            _ptr(g.f_inv_rhox_), _ptr(g.f_inv_rhoy_), _ptr(g.f_inv_rhoz_), _ptr(g.f_sx_), _ptr(g.f_sy_),
            _ptr(g.f_sz_), ctypes.c_double(dt), _ptr(g.f_vx_), _ptr(g.f_vy_), _ptr(g.f_vz_),
            ctypes.c_int(1 if zero_p_delta else 0)))

    def project(self, vxs, vys, vzs, dt, p_delta, vx, vy, vz, raise_on_fail=True) -> dict:
        st = nat.Stats()
        rc = self._lib.smac_project(self._h, _ptr(vxs), _ptr(vys), _ptr(vzs), ctypes.c_double(dt), _ptr(p_delta),
                                    _ptr(vx), _ptr(vy), _ptr(vz), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if raise_on_fail:
            nat.check(rc)
        return self.last_stats

    def project_adjoint(self, gvx, gvy, gvz, ox, oy, oz, phi=None, raise_on_fail=True) -> dict:
        st = nat.Stats()
        rc = self._lib.smac_project_adjoint(self._h, _ptr(gvx), _ptr(gvy), _ptr(gvz), _ptr(ox), _ptr(oy), _ptr(oz),
                                            _ptr(phi), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if raise_on_fail:
            nat.check(rc)
        return self.last_stats

    def apply_A(self, x: torch.Tensor, y: torch.Tensor):
        nat.check(self._lib.smac_apply_A(self._h, _ptr(x), _ptr(y)))

    def time_kernel(self, kernel_id: int, reps: int = 20):
        ms = ctypes.c_float()
        b = ctypes.c_double()
        nat.check(self._lib.smac_time_kernel(self._h, kernel_id, reps, ctypes.byref(ms), ctypes.byref(b)))
        return ms.value, b.value

    def selftest_wait(self):
        """(status the device recorded, SM cycles waited) of a bounded wait that
        nothing ends (smac_selftest_wait)."""
        st = ctypes.c_int()
        cyc = ctypes.c_longlong()
        nat.check(self._lib.smac_selftest_wait(self._h, ctypes.byref(st), ctypes.byref(cyc)))
        return st.value, cyc.value

    def selftest_sweep(self, precision: int, mode: int) -> int:
        n = ctypes.c_longlong()
        nat.check(self._lib.smac_selftest_sweep(self._h, precision, mode, ctypes.byref(n)))
        return n.value

    def num_levels(self) -> int:
        n = ctypes.c_int()
        nat.check(self._lib.smac_level_shape(self._h, 0, None, None, None, ctypes.byref(n)))
        return n.value

    def level_shape(self, level: int):
        a, b, c, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nat.check(self._lib.smac_level_shape(self._h, level, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                             ctypes.byref(n)))
        return (a.value, b.value, c.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.smac_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AsyncProjector:
    """Queued projections with host buffers (smac_async_*): submit() copies
    u* in and returns a ticket, wait(ticket) returns once u and p_delta are in
    the host buffers, with the projection's statistics.  The next
    projection's input copy and the previous one's output copy overlap the
    current solve.  Host tensors should be pinned (tensor.pin_memory()) and
    stay alive until their wait returns; the solver must not be used directly
    while the projector is open."""

    def __init__(self, solver: "B200PressureSolver"):
        self._lib = solver._lib
        self._solver = solver
        a = ctypes.c_void_p()
        nat.check(self._lib.smac_async_create(solver._h, ctypes.byref(a)))
        self._a = a

    def submit(self, vxs, vys, vzs, dt, p_delta, vx, vy, vz) -> int:
        for t in (vxs, vys, vzs, p_delta, vx, vy, vz):
            if t.device.type != "cpu" or t.dtype != torch.float64 or not t.is_contiguous():
                raise ValueError("AsyncProjector: host float64 contiguous tensors expected")
        ticket = ctypes.c_ulonglong()
        hp = lambda t: ctypes.c_void_p(t.data_ptr())
        nat.check(self._lib.smac_async_submit(self._a, hp(vxs), hp(vys), hp(vzs), ctypes.c_double(dt), hp(p_delta),
                                              hp(vx), hp(vy), hp(vz), ctypes.byref(ticket)))
        return ticket.value

    def wait(self, ticket: int, raise_on_fail=True) -> dict:
        st = nat.Stats()
        rc = self._lib.smac_async_wait(self._a, ctypes.c_ulonglong(ticket), ctypes.byref(st))
        if raise_on_fail:
            nat.check(rc)
        return st.as_dict()

    def close(self):
        if getattr(self, "_a", None):
            self._lib.smac_async_destroy(self._a)
            self._a = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class BoundaryConditions:
    """bc_ (CFD/memberList/boundaryConditionMembers.def): per boundary id its
    BoundaryType (CFD/Enums.h:10-16) and boundary velocity, host arrays."""
    bcType_: np.ndarray
    vx_: np.ndarray
    vy_: np.ndarray
    vz_: np.ndarray

    def table(self):
        """(smac_boundary_table, the arrays it points into)."""
        keep = [np.ascontiguousarray(self.bcType_, np.uint8)] + \
            [np.ascontiguousarray(a, np.float64) for a in (self.vx_, self.vy_, self.vz_)]
        t = nat.BoundaryTable(len(keep[0]), *(a.ctypes.data for a in keep))
        return t, keep


class SMACStep:
    """The G_SMACSolver calls of a time step, in the reference's order
    (CFD/main.cu:298-317): calc_surface_tension(sigma),
    get_vof_vstar_rhouu_consistent(), update_vstar_boundary(),
    solve_poisson(), correct_vof_velocity(), update_boundary_ghost(),
    make_face_gradp()."""

    def __init__(self, grid: DeviceGrid, dt: float = 1.0, g=(0.0, 0.0, 0.0), bc: BoundaryConditions | None = None):
        self.grid_ = grid
        self.dt_ = float(dt)
        self.inv_dt_ = 1.0 / self.dt_
        self.gx_, self.gy_, self.gz_ = (float(x) for x in g)
        self.bc_ = bc
        self.pressure_solver_: B200PressureSolver | None = None

    def get_vof_vstar_rhouu_consistent(self, two_way: dict | None = None):
        """G_SMACSolver::get_vof_vstar_rhouu_consistent (CFD/G_SMACSolver.cu:1062-1070):
        u* into f_v*_star_ from the grid's time-n fields (smac_predict_vstar)."""
        g = self.grid_
        need = ("f_mfx_", "f_mfy_", "f_mfz_", "f_mux_", "f_muy_", "f_muz_", "mu_", "rho_old_", "f_xbcid_")
        if self.bc_ is None or any(getattr(g, k) is None for k in need):
            raise ValueError("get_vof_vstar_rhouu_consistent needs bc_ and the grid's " + ", ".join(need))
        f = {"mu": g.mu_, "rho_old": g.rho_old_, "p": g.p_}
        for ax in "xyz":
            f["f" + ax + "t"] = getattr(g, f"f_{ax}type_")
            f["f" + ax + "bcid"] = getattr(g, f"f_{ax}bcid_")
            f["lam" + ax] = getattr(g, f"f_ibm_area_solid_fraction_{ax}_")
            f["v" + ax] = getattr(g, f"f_v{ax}_")
            f["mf" + ax] = getattr(g, f"f_mf{ax}_")
            f["mu" + ax] = getattr(g, f"f_mu{ax}_")
            f["fb" + ax] = getattr(g, f"f_b{ax}_")
            f["imp" + ax] = getattr(g, f"f_coupling_impulse_{ax}_")
            f["sf" + ax] = getattr(g, f"f_ibm_solid_fraction_{ax}_")
        predict_vstar_device(g.N, (g.dx_, g.dy_, g.dz_), self.bc_, f, self.dt_, (self.gx_, self.gy_, self.gz_),
                             (g.f_vx_star_, g.f_vy_star_, g.f_vz_star_), two_way=two_way)

    def get_vof_vstar_rhouu_consistent_two_way(self):
        """G_SMACSolver::get_vof_vstar_rhouu_consistent_two_way
        (CFD/G_SMACSolver.cu:2196-2203): the two-way-coupled u* into
        f_v*_star_, from the same fields as get_vof_vstar_rhouu_consistent
        plus void_fraction_old_, void_fraction_ and f_inv_rho*_
        (smac_predict_vstar_two_way)."""
        g = self.grid_
        need = ("void_fraction_old_", "void_fraction_")
        if any(getattr(g, k) is None for k in need):
            raise ValueError("get_vof_vstar_rhouu_consistent_two_way needs the grid's " + ", ".join(need))
        self.get_vof_vstar_rhouu_consistent(two_way={
            "eps_old": g.void_fraction_old_, "eps_new": g.void_fraction_, "inv_rhox": g.f_inv_rhox_,
            "inv_rhoy": g.f_inv_rhoy_, "inv_rhoz": g.f_inv_rhoz_})

    def compute_mass_flux_from_alpha_flux(self, rho0: float, rho1: float, two_way: bool = False):
        """G_SMACSolver::compute_mass_flux_from_alpha_flux (CFD/G_SMACSolver_VoF.cu:
        1792-1795), or with two_way compute_mass_flux_from_alpha_flux_two_way
        (:2685-2687, reading void_fraction_half_): f_mf*_ from f_v*_ and
        f_F*_accum_ (smac_mass_flux_from_alpha_flux).  Missing f_mf*_ are
        allocated."""
        g = self.grid_
        need = ("f_Fx_accum_", "f_Fy_accum_", "f_Fz_accum_", "f_xbcid_") + (("void_fraction_half_",) if two_way else ())
        if self.bc_ is None or any(getattr(g, k) is None for k in need):
            raise ValueError("compute_mass_flux_from_alpha_flux needs bc_ and the grid's " + ", ".join(need))
        sh = shapes(g.N)
        for ax in "xyz":
            if getattr(g, f"f_mf{ax}_") is None:
                setattr(g, f"f_mf{ax}_", torch.zeros(sh[ax], dtype=torch.float64, device=g.p_.device))
        f = {}
        for ax in "xyz":
            f["f" + ax + "t"] = getattr(g, f"f_{ax}type_")
            f["f" + ax + "bcid"] = getattr(g, f"f_{ax}bcid_")
            f["lam" + ax] = getattr(g, f"f_ibm_area_solid_fraction_{ax}_")
            f["v" + ax] = getattr(g, f"f_v{ax}_")
            f["F" + ax] = getattr(g, f"f_F{ax}_accum_")
        mass_flux_device(g.N, (g.dx_, g.dy_, g.dz_), self.bc_, f, rho0, rho1, self.dt_,
                         (g.f_mfx_, g.f_mfy_, g.f_mfz_), eps_half=g.void_fraction_half_ if two_way else None)

    def update_boundary_faces(self):
        """G_SMACSolver::update_boundary_faces (CFD/G_SMACSolver_VoF.cu:1798-1950):
        f_b*_ of the outlet faces marked in f_*outlet_ become twice the f_b of
        their interior neighbour (smac_update_boundary_faces)."""
        g = self.grid_
        if g.f_xoutlet_ is None:
            raise ValueError("update_boundary_faces needs the grid's f_*outlet_ marks")
        update_boundary_faces_device(g.N, (g.dx_, g.dy_, g.dz_), (g.f_xoutlet_, g.f_youtlet_, g.f_zoutlet_),
                                     (g.f_bx_, g.f_by_, g.f_bz_))

    def update_poisson_beta_two_way(self):
        """G_CFDDEMCoupling::update_poisson_beta_two_way
        (Coupling/G_CFDDEMCoupling.cu:419-460): f_b*_ = eps_f f_inv_rho*_ from
        void_fraction_ (smac_poisson_beta_two_way)."""
        g = self.grid_
        if g.void_fraction_ is None:
            raise ValueError("update_poisson_beta_two_way needs the grid's void_fraction_")
        poisson_beta_two_way_device(g.N, (g.dx_, g.dy_, g.dz_), g.void_fraction_,
                                    (g.f_inv_rhox_, g.f_inv_rhoy_, g.f_inv_rhoz_), (g.f_bx_, g.f_by_, g.f_bz_))

    def update_properties_by_alpha(self, rho0: float, rho1: float, mu0: float, mu1: float):
        """G_SMACSolver::update_properties_by_alpha (CFD/G_SMACSolver_VoF.cu:1544-1566):
        rho_ and rho_old_ swap (the previous rho is kept as rho_old_), then
        rho, 1/rho, mu of the cells and 1/rho (f_b and f_inv_rho), rho, mu of
        the faces from alpha_ (smac_update_properties).  Missing outputs are
        allocated."""
        g = self.grid_
        if g.alpha_ is None:
            raise ValueError("update_properties_by_alpha needs the grid's alpha_")
        sh = shapes(g.N)
        dev = g.p_.device
        for k in ("rho_", "rho_old_", "inv_rho_", "mu_"):
            if getattr(g, k) is None:
                setattr(g, k, torch.zeros(sh["cell"], dtype=torch.float64, device=dev))
        for ax in "xyz":
            for k in (f"f_b{ax}_", f"f_inv_rho{ax}_", f"f_rho{ax}_", f"f_mu{ax}_"):
                if getattr(g, k) is None:
                    setattr(g, k, torch.zeros(sh[ax], dtype=torch.float64, device=dev))
        g.rho_, g.rho_old_ = g.rho_old_, g.rho_
        out = {"rho": g.rho_, "inv_rho": g.inv_rho_, "mu": g.mu_}
        for ax in "xyz":
            out["fb" + ax] = getattr(g, f"f_b{ax}_")
            out["fir" + ax] = getattr(g, f"f_inv_rho{ax}_")
            out["rho" + ax] = getattr(g, f"f_rho{ax}_")
            out["mu" + ax] = getattr(g, f"f_mu{ax}_")
        update_properties_device(g.N, (g.dx_, g.dy_, g.dz_), rho0, rho1, mu0, mu1, g.alpha_, g.celltype_,
                                 (g.f_xtype_, g.f_ytype_, g.f_ztype_), out)

    def calc_surface_tension(self, sigma: float):
        """G_SMACSolver::calc_surface_tension (CFD/G_SMACSolver_VoF.cu:435-445):
        normals, curvature and the face force into f_s*_ (smac_surface_tension);
        sigma is the grid's sigma_."""
        g = self.grid_
        sh = shapes(g.N)
        dev = g.p_.device
        for k in ("nx_", "ny_", "nz_", "kappa_", "p_tmp_"):
            if getattr(g, k) is None:
                setattr(g, k, torch.zeros(sh["cell"], dtype=torch.float64, device=dev))
        for ax in "xyz":
            if getattr(g, f"f_s{ax}_") is None:
                setattr(g, f"f_s{ax}_", torch.zeros(sh[ax], dtype=torch.float64, device=dev))
        surface_tension_device(g.N, (g.dx_, g.dy_, g.dz_), g.alpha_, g.celltype_, sigma,
                               (g.nx_, g.ny_, g.nz_, g.kappa_, g.p_tmp_), (g.f_sx_, g.f_sy_, g.f_sz_))

    def update_vstar_boundary(self):
        """G_SMACSolver::update_vstar_boundary (CFD/G_SMACSolver.cu:1044-1052):
        wall u* before the projection."""
        g = self.grid_
        if self.bc_ is None or g.f_xbcid_ is None:
            raise ValueError("update_vstar_boundary needs the boundary table bc_ and the grid's f_*bcid_")
        marks = None if g.f_xoutlet_ is None else (g.f_xoutlet_, g.f_youtlet_, g.f_zoutlet_)
        lam = None if g.f_ibm_area_solid_fraction_x_ is None else (
            g.f_ibm_area_solid_fraction_x_, g.f_ibm_area_solid_fraction_y_, g.f_ibm_area_solid_fraction_z_)
        update_vstar_boundary_device(g.N, (g.dx_, g.dy_, g.dz_), self.bc_, (g.f_xtype_, g.f_ytype_, g.f_ztype_),
                                     (g.f_xbcid_, g.f_ybcid_, g.f_zbcid_), marks, lam,
                                     (g.f_vx_star_, g.f_vy_star_, g.f_vz_star_))

    def solve_poisson(self):
        return self.pressure_solver_.solve(self)

    def correct_vof_velocity(self):
        self.pressure_solver_.correct(self.grid_, self.dt_, zero_p_delta=True)

    def update_boundary_ghost(self):
        """G_SMACSolver::update_boundary_ghost (CFD/G_SMACSolver.cu:1345-1363):
        p in solid and ghost cells, then outlet and ghost velocities."""
        g = self.grid_
        update_pressure_ghost_device(g.N, (g.dx_, g.dy_, g.dz_), g.celltype_, g.rho_, (self.gx_, self.gy_, self.gz_),
                                     g.p_)
        if self.bc_ is None or g.f_xbcid_ is None:
            raise ValueError("update_boundary_ghost needs the boundary table bc_ and the grid's f_*bcid_")
        marks = None if g.f_xoutlet_ is None else (g.f_xoutlet_, g.f_youtlet_, g.f_zoutlet_)
        lam = None if g.f_ibm_area_solid_fraction_x_ is None else (
            g.f_ibm_area_solid_fraction_x_, g.f_ibm_area_solid_fraction_y_, g.f_ibm_area_solid_fraction_z_)
        update_velocity_ghost_device(g.N, (g.dx_, g.dy_, g.dz_), self.bc_, (g.f_xbcid_, g.f_ybcid_, g.f_zbcid_),
                                     marks, lam, (g.f_vx_star_, g.f_vy_star_, g.f_vz_star_), (g.f_bx_, g.f_by_, g.f_bz_),
                                     g.p_delta_, self.dt_, (g.f_vx_, g.f_vy_, g.f_vz_))

    def make_face_gradp(self):
        """G_SMACSolver::make_face_gradp (CFD/G_SMACSolver.cu:1336-1343)."""
        g = self.grid_
        if g.f_gradp_x_ is None:
            sh = shapes(g.N)
            g.f_gradp_x_, g.f_gradp_y_, g.f_gradp_z_ = (torch.zeros(sh[k], dtype=torch.float64, device=g.p_.device)
                                                        for k in "xyz")
        face_gradp_device(g.N, (g.dx_, g.dy_, g.dz_), g.p_, (g.f_gradp_x_, g.f_gradp_y_, g.f_gradp_z_))


# -- set-up helpers on the device (reference layout) --------------------------
def box_types_device(N, device="cuda"):
    sh = shapes(N)
    ct = torch.empty(sh["cell"], dtype=torch.uint8, device=device)
    fxt = torch.empty(sh["x"], dtype=torch.uint8, device=device)
    fyt = torch.empty(sh["y"], dtype=torch.uint8, device=device)
    fzt = torch.empty(sh["z"], dtype=torch.uint8, device=device)
    d = nat.GridDesc(*N, 1.0, 1.0, 1.0)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_box_types(ctypes.byref(d), _ptr(ct), _ptr(fxt), _ptr(fyt), _ptr(fzt),
                                        ctypes.c_void_p(s)))
    return ct, fxt, fyt, fzt


def assemble_vof_device(N, h, alpha, rho0, rho1, ct, fxt, fyt, fzt):
    sh = shapes(N)
    dev = alpha.device
    rho = torch.ones(sh["cell"], dtype=torch.float64, device=dev)
    fb = [torch.zeros(sh[k], dtype=torch.float64, device=dev) for k in "xyz"]
    fir = [torch.zeros(sh[k], dtype=torch.float64, device=dev) for k in "xyz"]
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_assemble_vof(ctypes.byref(d), _ptr(alpha), ctypes.c_double(rho0), ctypes.c_double(rho1),
                                           _ptr(ct), _ptr(fxt), _ptr(fyt), _ptr(fzt), _ptr(rho), *map(_ptr, fb),
                                           *map(_ptr, fir), ctypes.c_void_p(s)))
    return rho, fb, fir


def update_boundary_faces_device(N, h, marks, fb):
    """Outlet faces in place on the device face coefficients fb = (fbx, fby,
    fbz): smac_update_boundary_faces (G_SMACSolver::update_boundary_faces).
    marks: uint8 face tensors, 1 / 2 = interior side +1 / -1, 0 = untouched."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_update_boundary_faces(ctypes.byref(d), *map(_ptr, marks), *map(_ptr, fb),
                                                    ctypes.c_void_p(s)))


def ibm_solid_fraction_device(N, h, origin, spheres, device="cuda"):
    sh = shapes(N)
    sf = torch.zeros(sh["cell"], dtype=torch.float64, device=device)
    sph = np.ascontiguousarray(np.asarray(spheres, np.float64).reshape(-1))
    org = (ctypes.c_double * 3)(*origin)
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_ibm_solid_fraction_spheres(
        ctypes.byref(d), org, sph.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.c_int(len(sph) // 4),
        _ptr(sf), ctypes.c_void_p(s)))
    return sf


def ibm_set_solid_device(N, sf, ct, fxt, fyt, fzt):
    d = nat.GridDesc(*N, 1.0, 1.0, 1.0)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_ibm_set_solid_cells(ctypes.byref(d), _ptr(sf), _ptr(ct), _ptr(fxt), _ptr(fyt),
                                                  _ptr(fzt), ctypes.c_void_p(s)))


# -- the pass after the projection (update_boundary_ghost, make_face_gradp) --
def update_pressure_ghost_device(N, h, ct, rho, g, p):
    """smac_update_pressure_ghost in place on p (cells); rho None means 1."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    dd = ctypes.c_double
    nat.check(nat.load().smac_update_pressure_ghost(ctypes.byref(d), _ptr(ct), _ptr(rho), dd(g[0]), dd(g[1]),
                                                    dd(g[2]), _ptr(p), ctypes.c_void_p(s)))


def update_velocity_ghost_device(N, h, bc: BoundaryConditions, bcid, marks, lam, vs, fb, p_delta, dt, v):
    """smac_update_velocity_ghost in place on v = (vx, vy, vz): outlet faces
    (marks None: none), then ghost faces and corners; lam None means 0."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    table, keep = bc.table()
    marks = marks if marks is not None else (None, None, None)
    lam = lam if lam is not None else (None, None, None)
    if marks[0] is None:
        vs, fb, p_delta = (None, None, None), (None, None, None), None
    nat.check(nat.load().smac_update_velocity_ghost(
        ctypes.byref(d), ctypes.byref(table), *map(_ptr, bcid), *map(_ptr, marks), *map(_ptr, lam), *map(_ptr, vs),
        *map(_ptr, fb), _ptr(p_delta), ctypes.c_double(dt), *map(_ptr, v), ctypes.c_void_p(s)))
    del keep


def update_vstar_boundary_device(N, h, bc: BoundaryConditions, ft, bcid, marks, lam, vs):
    """smac_update_vstar_boundary in place on vs = (vxs, vys, vzs): the wall
    u* of every F_BOUNDARY face; marks / lam None mean none / 0."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    table, keep = bc.table()
    marks = marks if marks is not None else (None, None, None)
    lam = lam if lam is not None else (None, None, None)
    nat.check(nat.load().smac_update_vstar_boundary(
        ctypes.byref(d), ctypes.byref(table), *map(_ptr, ft), *map(_ptr, bcid), *map(_ptr, marks), *map(_ptr, lam),
        *map(_ptr, vs), ctypes.c_void_p(s)))
    del keep


def surface_tension_device(N, h, alpha, ct, sigma, work, fs):
    """smac_surface_tension: work = (nx, ny, nz, kappa, grad_mag) cell tensors
    (the grid's nx_, ny_, nz_, kappa_, p_tmp_), fs = (fsx, fsy, fsz) face
    tensors, all written as G_SMACSolver::calc_surface_tension writes them."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_surface_tension(ctypes.byref(d), _ptr(alpha), _ptr(ct), ctypes.c_double(sigma),
                                              *map(_ptr, work), *map(_ptr, fs), ctypes.c_void_p(s)))


def predict_vstar_device(N, h, bc: BoundaryConditions, fields: dict, dt, g, vs, two_way: dict | None = None):
    """smac_predict_vstar: u* of every F_INTERIOR face into vs = (vxs, vys,
    vzs).  fields maps the smac_momentum_fields names (fxt .. sfz) to CUDA
    tensors; lam*/imp*/sf* may be missing (0).  With two_way (the
    smac_two_way_fields names eps_old, eps_new, inv_rhox.. to CUDA tensors)
    the two-way-coupled form, smac_predict_vstar_two_way."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    table, keep = bc.table()
    mf = nat.MomentumFields()
    for name, _ in nat.MomentumFields._fields_:
        t = fields.get(name)
        setattr(mf, name, None if t is None else _ptr(t).value)
    dd = ctypes.c_double
    if two_way is None:
        nat.check(nat.load().smac_predict_vstar(ctypes.byref(d), ctypes.byref(table), ctypes.byref(mf), dd(dt),
                                                dd(g[0]), dd(g[1]), dd(g[2]), *map(_ptr, vs), ctypes.c_void_p(s)))
    else:
        tw = nat.TwoWayFields()
        for name, _ in nat.TwoWayFields._fields_:
            t = two_way.get(name)
            setattr(tw, name, None if t is None else _ptr(t).value)
        nat.check(nat.load().smac_predict_vstar_two_way(ctypes.byref(d), ctypes.byref(table), ctypes.byref(mf),
                                                        ctypes.byref(tw), dd(dt), dd(g[0]), dd(g[1]), dd(g[2]),
                                                        *map(_ptr, vs), ctypes.c_void_p(s)))
    del keep


def mass_flux_device(N, h, bc: BoundaryConditions, fields: dict, rho0, rho1, dt, mf, eps_half=None):
    """smac_mass_flux_from_alpha_flux: mf = (mfx, mfy, mfz) <- rho0 q + (rho1 -
    rho0) F h / dt on every face.  fields maps the smac_mass_flux_fields names
    to CUDA tensors (lam* may be missing); eps_half selects the two-way form."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    table, keep = bc.table()
    f = nat.MassFluxFields()
    for name, _ in nat.MassFluxFields._fields_:
        t = fields.get(name)
        setattr(f, name, None if t is None else _ptr(t).value)
    dd = ctypes.c_double
    nat.check(nat.load().smac_mass_flux_from_alpha_flux(ctypes.byref(d), ctypes.byref(table), ctypes.byref(f),
                                                        dd(rho0), dd(rho1), dd(dt), _ptr(eps_half), *map(_ptr, mf),
                                                        ctypes.c_void_p(s)))
    del keep


def poisson_beta_two_way_device(N, h, eps, fir, fb):
    """smac_poisson_beta_two_way: fb = (fbx, fby, fbz) <- eps_f * fir on the
    interior box faces (CUDA tensors, written in place)."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_poisson_beta_two_way(ctypes.byref(d), _ptr(eps), *map(_ptr, fir), *map(_ptr, fb),
                                                   ctypes.c_void_p(s)))


def update_properties_device(N, h, rho0, rho1, mu0, mu1, alpha, ct, ft, out: dict):
    """smac_update_properties: out maps the smac_property_fields names (rho,
    inv_rho, mu, fbx.., firx.., rhox.., mux..) to CUDA tensors written in place;
    inv_rho, fir*, rho{x,y,z} may be missing."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    f = nat.PropertyFields()
    for name, _ in nat.PropertyFields._fields_:
        t = out.get(name)
        setattr(f, name, None if t is None else _ptr(t).value)
    vp = nat.VofParams(rho0, rho1, mu0, mu1)
    nat.check(nat.load().smac_update_properties(ctypes.byref(d), ctypes.byref(vp), _ptr(alpha), _ptr(ct),
                                                *map(_ptr, ft), ctypes.byref(f), ctypes.c_void_p(s)))


def face_gradp_device(N, h, p, gp):
    """smac_face_gradp: gp = (gpx, gpy, gpz) face tensors, faces 1..N+1 written."""
    d = nat.GridDesc(*N, *h)
    s = torch.cuda.current_stream().cuda_stream
    nat.check(nat.load().smac_face_gradp(ctypes.byref(d), _ptr(p), *map(_ptr, gp), ctypes.c_void_p(s)))
