/*
 * smac_b200.h -- C ABI of the B200-native SMAC pressure projection.
 *
 * A drop-in for the reference's pressure-solver seam
 *   struct G_PressureSolverBase { virtual void solve(G_SMACSolver&) = 0; ... }
 *   (CFD/pressure_solver/G_PressureSolverBase.h:24-42)
 * and for the calls on either side of it: the Poisson right-hand side
 * (G_PressureSolverBase.cu:49-118), the velocity correction
 * (CFD/G_SMACSolver.cu:1072-1142,1269-1275), the VoF face-coefficient update
 * (CFD/G_SMACSolver_VoF.cu:1374-1535) and the IBM solid mask
 * (CFD/G_SMACSolver_IBM.cu:94-147,763-792).
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer in the reference layout
 *    (MyArray<T,3>, x fastest, index (z*sy + y)*sx + x, CFD/MyArray.h:43-51):
 *      cells   (Nx+2)(Ny+2)(Nz+2)   x-faces (Nx+3)(Ny+2)(Nz+2)
 *      y-faces (Nx+2)(Ny+3)(Nz+2)   z-faces (Nx+2)(Ny+2)(Nz+3)
 *    (CFD/memberList/gridMembers.def), doubles and unsigned chars exactly as
 *    G_StaggeredGrid holds them.  Type codes are CFD/Enums.h:3-23.
 *  - Every call returns an smac_status; 0 is success.  Nothing aborts.
 *    smac_last_error_string() describes the last failure of this thread.
 *  - A handle owns its stream (given at creation), its multigrid hierarchy,
 *    its coefficients and all scratch; caller arrays are only borrowed for
 *    the duration of a call.  One handle must not be used from two threads
 *    at once.  Calls are asynchronous on the handle's stream except where a
 *    smac_stats is requested, which ends with one stream synchronisation.
 */
#ifndef SMAC_B200_H
#define SMAC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct smac_handle smac_handle;

typedef enum {
  SMAC_OK = 0,
  SMAC_NOT_CONVERGED = 1, /* tolerance not met within max_iter (reference: silent stop, G_PCGSolver.cu:788) */
  SMAC_BREAKDOWN = 2,     /* p.Ap <= 0 or r.z <= 0 inside PCG */
  SMAC_NAN = 3,           /* a non-finite value reached a reduction */
  SMAC_BAD_ARG = 4,       /* null pointer, bad option value */
  SMAC_BAD_SHAPE = 5,     /* grid sizes the hierarchy cannot use (reference: abort(), G_GMGSolver.cu:38-51) */
  SMAC_CUDA_ERROR = 6,    /* a CUDA runtime call failed */
  SMAC_NO_DEVICE = 7      /* no usable sm_100 device */
} smac_status;

/* Solver variants: the same four the reference selects with
 * G_PCGSolver::set_solver(PCG_TYPES) (G_PCGSolver.cu:592-613, CFD/Enums.h:25-30). */
typedef enum {
  SMAC_STANDARD_PCG = 0,             /* Jacobi-preconditioned CG                (solve_pcg :448-586) */
  SMAC_PURENEUMANN_STANDARD_PCG = 1, /* ... with zero-mean projection          (solve_pureneumann_pcg :307-445) */
  SMAC_GMG_PCG = 2,                  /* multigrid-preconditioned CG            (solve_gmgpcg :619-770) */
  SMAC_PURENEUMANN_GMG_PCG = 3       /* ... with zero-mean projection          (solve_pureneumann_gmgpcg :772-922) */
} smac_solver_type;

typedef enum {
  SMAC_PRECISION_FP64 = 0,  /* every vector, coefficient and reduction in FP64 */
  SMAC_PRECISION_MIXED = 1  /* FP32 Krylov vectors, matvec and V-cycle (BF16 coefficients on the
                               coarsest grids), FP64 true residual, solution, reductions,
                               zero-mean projection and coefficient assembly */
} smac_precision;

typedef enum {
  SMAC_STOP_RELATIVE = 0,  /* ||b - A x||_2 / ||b||_2 < tol (b de-meaned for pure Neumann) */
  SMAC_STOP_REFERENCE = 1  /* max|b - A x| * dt < tol: the reference's test (G_PCGSolver.cu:884-903),
                              dt being the one passed to smac_divergence */
} smac_stop_rule;

typedef struct {
  int nx, ny, nz;     /* interior cells: G_StaggeredGrid::Nx_, Ny_, Nz_ */
  double dx, dy, dz;  /* spacing: G_StaggeredGrid::dx_, dy_, dz_ */
} smac_grid_desc;

typedef struct {
  int solver_type;        /* smac_solver_type, default SMAC_PURENEUMANN_GMG_PCG */
  int precision;          /* smac_precision, default SMAC_PRECISION_FP64 */
  int stop_rule;          /* smac_stop_rule, default SMAC_STOP_RELATIVE */
  double tol;             /* default 1e-8; the reference's tol_ (G_PressureSolverBase.h:40) */
  int max_iter;           /* PCG iteration cap, default 2000 (G_PCGSolver.cu:788) */
  int min_coarse;         /* a direction is halved while the result stays >= min_coarse and even
                             (default 4; the reference's min_size_ is 6, G_GMGSolver.h:22) */
  int max_levels;         /* grids in the hierarchy including the finest, default 16 (MAX_LEVELS) */
  int nu1, nu2;           /* red-black Gauss-Seidel pre/post sweeps per level, default 2/2 */
  int coarse_sweeps;      /* symmetric sweep pairs on the coarsest grid, default 8 */
  int check_every;        /* residual tests every check_every iterations (device side), default 1 */
  double reliable_delta;  /* MIXED: recompute the FP64 true residual when the FP32 residual has
                             fallen by this factor since the last recomputation, default 1e-4 */
  int bf16_coarse_cells;  /* MIXED: grids with at most this many cells store BF16 coefficients
                             (default 4096, i.e. 16^3 and below); 0 disables BF16 */
  int sweep_kernel;       /* smac_sweep_kernel: which kernel runs the fused red-black sweeps of the
                             separately launched grids, default SMAC_SWEEP_AUTO; every choice gives
                             the same result bit for bit */
  int coarse_kernel;      /* smac_coarse_kernel: how the lower part of the V-cycle runs, default
                             SMAC_COARSE_AUTO; both choices give the same result bit for bit */
} smac_options;

typedef enum {
  SMAC_SWEEP_AUTO = 0,     /* the z-march where the grid allows it and it measured faster, else the
                              TMA ring */
  SMAC_SWEEP_TMA = 1,      /* tiles staged in a shared-memory ring by the Tensor Memory Accelerator */
  SMAC_SWEEP_ZMARCH = 2,   /* whole x-rows per warp, a register z-march (x extent <= 256 cells FP64,
                              512 FP32); other grids fall back to the TMA ring */
  SMAC_SWEEP_SHARED = 3    /* tiles staged in shared memory by plain loads */
} smac_sweep_kernel;

typedef enum {
  SMAC_COARSE_AUTO = 0,    /* from the first grid of <= 32768 cells down, one cluster of 8 CTAs that
                              holds the grids in distributed shared memory, where they fit (else as
                              SMAC_COARSE_CTA) */
  SMAC_COARSE_CTA = 1      /* the grids of <= 4096 cells in one CTA on global memory, the grids
                              above them launched sweep by sweep */
} smac_coarse_kernel;

typedef struct {
  int status;              /* smac_status of the solve */
  int iterations;          /* PCG iterations (preconditioner applications) */
  int reliable_updates;    /* MIXED: FP64 true-residual recomputations */
  int num_levels;          /* grids in the multigrid hierarchy */
  double norm_b;           /* ||b||_2 after the zero-mean projection */
  double rel_residual;     /* ||b - A x||_2 / ||b||_2 at exit, FP64 operator */
  double max_residual;     /* max |b - A x| at exit */
  double alg_bytes;        /* algorithmic HBM bytes of the kernels launched (byte model) */
  int kernel_launches;     /* kernels launched by the call */
} smac_stats;

/* ---- lifetime ----------------------------------------------------------- */

/* Fill *opts with the defaults listed above. */
smac_status smac_default_options(smac_options* opts);

/* Allocate a solver for the grid on the current CUDA device.  stream may be
 * NULL (legacy default stream).  Replaces the set-up in CFD/main.cu:225-243
 * (G_PCGSolver + G_GMGSolver::initialize, G_GMGSolver.cu:10-147). */
smac_status smac_create(const smac_grid_desc* desc, const smac_options* opts, void* cuda_stream,
                        smac_handle** out);
smac_status smac_destroy(smac_handle* h);
/* Change solver options between solves (hierarchy options are fixed at creation). */
smac_status smac_set_options(smac_handle* h, const smac_options* opts);
const char* smac_last_error_string(void);
/* Number of grids in the hierarchy and the interior size of grid `level`. */
smac_status smac_level_shape(const smac_handle* h, int level, int* nx, int* ny, int* nz, int* num_levels);

/* ---- coefficients --------------------------------------------------------- */

/* Import the Poisson face coefficients f_b and the cell/face types.
 * Replaces k_build_vof_poisson_A (G_PCGSolver.cu:126-212) and
 * G_GMGSolver::create_coeffs (G_GMGSolver.cu:913-922): the fine operator is
 * A_c = sum_faces f_b/h^2 (diagonal) minus f_b/h^2 per F_INTERIOR face; rows of
 * cells that are not C_INTERIOR are zero; coarse grids are built in FP64.
 * fbx/fby/fbz: x/y/z-face doubles; celltype: cell bytes; fxt/fyt/fzt: face bytes. */
smac_status smac_set_coefficients(smac_handle* h, const double* fbx, const double* fby, const double* fbz,
                                  const uint8_t* celltype, const uint8_t* fxt, const uint8_t* fyt,
                                  const uint8_t* fzt);

/* Cell and face types of an all-wall box: SMACSolver::set_face_type and
 * set_cell_type (CFD/SMACSolver.cpp:104-248). */
smac_status smac_box_types(const smac_grid_desc* desc, uint8_t* celltype, uint8_t* fxt, uint8_t* fyt,
                           uint8_t* fzt, void* cuda_stream);

/* VoF density and face coefficients from the volume fraction alpha:
 * k_update_cell_properties_by_alpha + k_update_{x,y,z}_face_properties_by_alpha
 * (CFD/G_SMACSolver_VoF.cu:1374-1535), FP64.  rho: cells (written on
 * C_INTERIOR / C_NEAR_BOUNDARY cells); fb*: f_b; fir*: f_inv_rho (may be NULL). */
smac_status smac_assemble_vof(const smac_grid_desc* desc, const double* alpha, double rho0, double rho1,
                              const uint8_t* celltype, const uint8_t* fxt, const uint8_t* fyt,
                              const uint8_t* fzt, double* rho, double* fbx, double* fby, double* fbz,
                              double* firx, double* firy, double* firz, void* cuda_stream);

/* The two phases' densities and viscosities (G_SMACSolver::rho0_, rho1_,
 * mu0_, mu1_; alpha = 1 is phase 1). */
typedef struct {
  double rho0, rho1, mu0, mu1;
} smac_vof_params;

/* Outputs of the property update (device pointers, reference layout); the
 * marked ones may be NULL (not written). */
typedef struct {
  double *rho, *inv_rho, *mu;       /* cells: rho_, inv_rho_ (NULL ok), mu_ */
  double *fbx, *fby, *fbz;          /* f_b*_ */
  double *firx, *firy, *firz;       /* f_inv_rho*_ (NULL ok) */
  double *rhox, *rhoy, *rhoz;       /* f_rho*_ (NULL ok) */
  double *mux, *muy, *muz;          /* f_mu*_: the face viscosities the momentum predictor reads */
} smac_property_fields;

/* The whole property update, G_SMACSolver::update_properties_by_alpha
 * (CFD/G_SMACSolver_VoF.cu:1543-1566), after its swap of rho_ and rho_old_
 * (the caller swaps its two arrays):
 *  - C_INTERIOR / C_NEAR_BOUNDARY cells 1..N+1: rho and mu linear in alpha,
 *    inv_rho = 1/rho (:1374-1407);
 *  - C_SOLID interior cells: rho and mu of the first C_INTERIOR neighbour
 *    (x-, x+, y-, y+, z-, z+; 0 without one); ghost cells: those of the
 *    nearest interior cell (:1241-1372, their final state);
 *  - F_INTERIOR faces: rho_f = the two cells' mean, f_b = f_inv_rho =
 *    1/rho_f, mu_f = the mean viscosity; other faces with indices 1..N+2
 *    along, 1..N+1 across: f_b = f_inv_rho = 0 (:1409-1535).
 * One launch computes every final value from alpha and the types; every
 * face array must have fewer than 2^31 entries (SMAC_BAD_SHAPE otherwise).  The ghost
 * layer must not hold C_INTERIOR cells next to C_SOLID interior cells (the
 * reference's set-up types it C_GHOST, CFD/SMACSolver.cpp:220; there the
 * reference's own passes would race).
 * smac_assemble_vof is the subset that feeds the pressure operator. */
smac_status smac_update_properties(const smac_grid_desc* d, const smac_vof_params* vp, const double* alpha,
                                   const uint8_t* celltype, const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt,
                                   const smac_property_fields* out, void* stream);

/* Poisson coefficients of the two-way-coupled step,
 * G_CFDDEMCoupling::update_poisson_beta_two_way (Coupling/G_CFDDEMCoupling.cu:
 * 419-460, called at Coupling/main.cu:533 after the property update):
 * f_b = eps_f f_inv_rho, eps_f = (eps_L + eps_R)/2 of the face's two cells,
 * on x-faces 1..Nx+1 x 1..Ny x 1..Nz (y and z alike); other faces keep their
 * values.  eps: void_fraction_ (cells). */
smac_status smac_poisson_beta_two_way(const smac_grid_desc* d, const double* eps, const double* firx,
                                      const double* firy, const double* firz, double* fbx, double* fby, double* fbz,
                                      void* stream);

/* Outlet boundary faces: f_b = 2 f_b of the neighbouring face on the interior
 * side, where p = 0 is imposed.  G_SMACSolver::update_boundary_faces
 * (CFD/G_SMACSolver_VoF.cu:1798-1950), run after smac_assemble_vof.  The
 * marks (face arrays, uint8) give the interior side of an outlet face:
 * 1 -> +1, 2 -> -1 (the reference's f_*internal_id_); 0 leaves a face as it
 * is (walls keep f_b = 0).  Marked faces must have unmarked neighbours on the
 * interior side (outlets on domain sides). */
smac_status smac_update_boundary_faces(const smac_grid_desc* d, const uint8_t* fxo, const uint8_t* fyo,
                                       const uint8_t* fzo, double* fbx, double* fby, double* fbz, void* stream);

/* IBM solid fraction of cells 1..N+1 by 8^3 sub-sampling
 * (k_get_solid_fraction, CFD/G_SMACSolver_IBM.cu:94-147, clip >= 0.99 -> 1)
 * for a union of non-overlapping spheres (x, y, z, r per sphere, HOST array
 * of 4*num_spheres doubles) in place of the reference's cylinder. */
smac_status smac_ibm_solid_fraction_spheres(const smac_grid_desc* desc, const double origin[3],
                                            const double* spheres_host, int num_spheres, double* solid_fraction,
                                            void* cuda_stream);
/* k_set_solid_cell_from_ibm (CFD/G_SMACSolver_IBM.cu:763-792): cells with
 * solid fraction > 1-1e-12 become C_SOLID and their six faces F_BOUNDARY. */
smac_status smac_ibm_set_solid_cells(const smac_grid_desc* desc, const double* solid_fraction, uint8_t* celltype,
                                     uint8_t* fxt, uint8_t* fyt, uint8_t* fzt, void* cuda_stream);

/* ---- the projection ------------------------------------------------------- */

/* Right-hand side, base_k_make_poisson_rhs (G_PressureSolverBase.cu:49-118):
 *   rhs = -(1/dt) div(eps u*) - (eps - eps_old)/dt^2 - div(f_b f_s)   on C_INTERIOR cells, 0 elsewhere.
 * eps/eps_old NULL means eps == 1 (so the second term vanishes); fsx/fsy/fsz
 * NULL means no surface-tension force.  Uses the coefficients of the last
 * smac_set_coefficients.  rhs_out (cells, may be NULL) receives the RHS in the
 * reference layout (interior entries).  dt is also the dt of SMAC_STOP_REFERENCE. */
smac_status smac_divergence(smac_handle* h, const double* vxs, const double* vys, const double* vzs,
                            const double* eps, const double* eps_old, const double* fsx, const double* fsy,
                            const double* fsz, double dt, double* rhs_out);

/* Solve A p_delta = rhs for the RHS of the last smac_divergence (or
 * smac_set_rhs).  Replaces G_PressureSolverBase::solve -> G_PCGSolver::solve
 * (G_SMACSolver.cu:1499-1501, G_PCGSolver.cu:615-617).  Pure-Neumann variants
 * project b and the result onto zero mean over the fluid (C_INTERIOR) cells.
 * p_delta: cells, interior entries written (ghosts untouched).  stats may be
 * NULL (then the call does not synchronise). */
smac_status smac_solve(smac_handle* h, double* p_delta, smac_stats* stats);

/* Supply the RHS directly (cells, reference layout, interior entries read). */
smac_status smac_set_rhs(smac_handle* h, const double* rhs);

/* Velocity correction, k_correct_vof_velocity + correct_vof_velocity
 * (G_SMACSolver.cu:1072-1142,1269-1275): on F_INTERIOR faces
 *   u = u* + f_inv_rho dt (f_s - grad p_delta),
 * p += p_delta on C_INTERIOR cells (p may be NULL), then p_delta is zeroed
 * when zero_p_delta != 0 (the reference always zeroes it).  Faces that are
 * not F_INTERIOR are not written.  fs* may be NULL; fir* NULL means use f_b. */
smac_status smac_correct(smac_handle* h, double* p_delta, double* p, const double* vxs, const double* vys,
                         const double* vzs, const double* firx, const double* firy, const double* firz,
                         const double* fsx, const double* fsy, const double* fsz, double dt, double* vx,
                         double* vy, double* vz, int zero_p_delta);

/* divergence -> solve -> correction in one call (eps == 1, no f_s, f_inv_rho = f_b).
 * p_delta receives the pressure increment (not zeroed); faces that are not
 * F_INTERIOR receive u* so that (vx,vy,vz) is the projected field everywhere. */
smac_status smac_project(smac_handle* h, const double* vxs, const double* vys, const double* vzs, double dt,
                         double* p_delta, double* vx, double* vy, double* vz, smac_stats* stats);

/* Adjoint of smac_project with respect to u*: given g = dL/du (faces) returns
 * dL/du* = g + G A^+ D(B g) on F_INTERIOR faces (g elsewhere), one more MG-PCG
 * solve with the same operator (A is symmetric).  phi (cells, may be NULL)
 * receives the adjoint pressure. */
smac_status smac_project_adjoint(smac_handle* h, const double* gvx, const double* gvy, const double* gvz,
                                 double* gvxs, double* gvys, double* gvzs, double* phi, smac_stats* stats);

/* ---- after the projection ------------------------------------------------
 * The reference's G_SMACSolver::update_boundary_ghost and make_face_gradp
 * (CFD/G_SMACSolver.cu:1144-1363, CFD/G_BoundaryFunctions.cu:143-560), the
 * consumers of p.  Grid-only calls (no handle), asynchronous on `stream`. */

/* Pressure in solid and ghost cells (k_update_cell_boundary_pressure +
 * k_update_cell_ghost_pressure, CFD/G_SMACSolver.cu:1144-1267), in place:
 * a C_SOLID cell takes p of its first C_INTERIOR neighbour (x-, x+, y-, y+,
 * z-, z+) shifted by rho g h (0 without one); every ghost cell then takes p
 * of the nearest interior cell plus rho(src) g.r.  rho (cells) may be NULL
 * (rho = 1); (gx, gy, gz) is SMACSolver::gx_, gy_, gz_. */
smac_status smac_update_pressure_ghost(const smac_grid_desc* d, const uint8_t* celltype, const double* rho,
                                       double gx, double gy, double gz, double* p, void* stream);

/* The boundary-condition table bc_ (CFD/memberList/boundaryConditionMembers.def),
 * HOST arrays of num_ids entries (1..256): BoundaryType codes (CFD/Enums.h:10-16:
 * 0 no-slip, 1 slip, 2 inflow, 3 outflow, 4 outlet) and boundary velocities. */
typedef struct {
  int num_ids;
  const uint8_t* type;
  const double *vx, *vy, *vz;
} smac_boundary_table;

/* The fields the momentum predictor reads (G_StaggeredGrid members, device
 * pointers in the reference layout; the marked ones may be NULL, read as 0). */
typedef struct {
  const uint8_t *fxt, *fyt, *fzt;           /* f_*type_ */
  const uint8_t *fxbcid, *fybcid, *fzbcid;  /* f_*bcid_ */
  const double *lamx, *lamy, *lamz;         /* f_ibm_area_solid_fraction_*_ (NULL: 0) */
  const double *vx, *vy, *vz;               /* f_v*_: the velocity at time n */
  const double *mfx, *mfy, *mfz;            /* f_mf*_: advecting face velocities */
  const double *mux, *muy, *muz;            /* f_mu*_: face viscosities */
  const double *mu, *rho_old, *p;           /* mu_, rho_old_, p_ (cells) */
  const double *fbx, *fby, *fbz;            /* f_b*_: 1/rho on faces */
  const double *impx, *impy, *impz;         /* f_coupling_impulse_*_ (NULL: 0) */
  const double *sfx, *sfy, *sfz;            /* f_ibm_solid_fraction_*_ (NULL: 0) */
} smac_momentum_fields;

/* The momentum predictor, G_SMACSolver::get_vof_vstar_rhouu_consistent
 * (CFD/G_SMACSolver.cu:1062-1070; k_get_vof_vstar_rhouu_consistent_{x,y,z}
 * :90-1012, boundary rules CFD/G_BoundaryFunctions.h:9-367): on every
 * F_INTERIOR face with indices 1..N+1,
 *   u* = (1/rho)(rho_old u + impulse/V) + dt((1/rho)(div tau - div(mf u) - grad p) + g),
 * times (1 - IBM solid fraction); tau the Newtonian stress with the cell and
 * face viscosities, convection MUSCL with the minmod limiter, neighbours past
 * a wall mirrored about it (slip and outlet walls copied).  Other faces of
 * (vxs, vys, vzs) are not written.  Every grid extent must be >= 2, and
 * every face array below 2^31 entries (SMAC_BAD_SHAPE otherwise). */
smac_status smac_predict_vstar(const smac_grid_desc* d, const smac_boundary_table* bc, const smac_momentum_fields* mf,
                               double dt, double gx, double gy, double gz, double* vxs, double* vys, double* vzs,
                               void* stream);

/* The extra cell and face fields of the two-way-coupled predictor (device
 * pointers, reference layout). */
typedef struct {
  const double *eps_old, *eps_new;            /* void_fraction_old_, void_fraction_ (cells) */
  const double *inv_rhox, *inv_rhoy, *inv_rhoz; /* f_inv_rho*_ (read in place of mf's f_b*) */
} smac_two_way_fields;

/* The two-way-coupled momentum predictor,
 * G_SMACSolver::get_vof_vstar_rhouu_consistent_two_way (CFD/G_SMACSolver.cu:
 * 2196-2203; k_get_vof_vstar_rhouu_consistent_{x,y,z}_two_way :1538-2194),
 * the step the CFD-DEM coupled solver takes (Coupling/main.cu:540): as
 * smac_predict_vstar with each stress times the void fraction eps_old of its
 * cell or edge (the mean of the four cells around an edge), the pressure
 * gradient times the face's eps_old, and
 *   u* = (f_inv_rho / eps_new_f)(eps_old_f rho_old_f u + dt (...) + impulse/V) + dt g,
 * times (1 - IBM solid fraction).  mf's fbx..fbz are not read. */
smac_status smac_predict_vstar_two_way(const smac_grid_desc* d, const smac_boundary_table* bc,
                                       const smac_momentum_fields* mf, const smac_two_way_fields* tw, double dt,
                                       double gx, double gy, double gz, double* vxs, double* vys, double* vzs,
                                       void* stream);

/* Inputs of the mass-flux update (device pointers, reference layout). */
typedef struct {
  const uint8_t *fxt, *fyt, *fzt;           /* f_*type_ */
  const uint8_t *fxbcid, *fybcid, *fzbcid;  /* f_*bcid_ */
  const double *lamx, *lamy, *lamz;         /* f_ibm_area_solid_fraction_*_ (NULL: 0) */
  const double *vx, *vy, *vz;               /* f_v*_ */
  const double *Fx, *Fy, *Fz;               /* f_F*_accum_: the accumulated volume-fraction flux */
} smac_mass_flux_fields;

/* The advecting mass flux the momentum predictor reads,
 * G_SMACSolver::compute_mass_flux_from_alpha_flux (CFD/G_SMACSolver_VoF.cu:
 * 1708-1795, called at CFD/main.cu:298): on every face of the three families
 * mf = rho0 q + (rho1 - rho0) F_accum h / dt, q the face velocity by the
 * boundary face rule (as smac_predict_vstar reads it).  With eps_half (the
 * grid's void_fraction_half_, cells) the two-way form
 * compute_mass_flux_from_alpha_flux_two_way (:2472-2687, Coupling/main.cu:531):
 * q = eps_f u_f on faces 1..N+1 along their axis (eps_f the mean of the two
 * cells, the one interior cell's at faces 1 and N+1), mf = 0 on faces 0 and
 * N+2.  Every face array must have fewer than 2^31 entries. */
smac_status smac_mass_flux_from_alpha_flux(const smac_grid_desc* d, const smac_boundary_table* bc,
                                           const smac_mass_flux_fields* in, double rho0, double rho1, double dt,
                                           const double* eps_half, double* mfx, double* mfy, double* mfz,
                                           void* stream);

/* Wall-face u* before the projection, G_SMACSolver::update_vstar_boundary
 * (CFD/G_SMACSolver.cu:1044-1052, k_update_v*star_boundary,
 * CFD/G_BoundaryFunctions.cu:3-71, CFD/G_BoundaryFunctions.h:369-470), in
 * place on (vxs, vys, vzs): every F_BOUNDARY face with indices 1..N+1 gets,
 * by the type of its id in f_*bcid_: inflow (1 - lam) v_b, no-slip 0,
 * outlet the u* of the next face on its interior side (outlet mark 2: -1,
 * otherwise +1), slip and outflow 0.  With no-slip walls this makes the
 * pure-Neumann system compatible (sum of D u* = 0).  Marks and lam may be
 * NULL.  An outlet face whose neighbour is also F_BOUNDARY reads a value
 * that another thread may be writing, as in the reference. */
smac_status smac_update_vstar_boundary(const smac_grid_desc* d, const smac_boundary_table* bc, const uint8_t* fxt,
                                      const uint8_t* fyt, const uint8_t* fzt, const uint8_t* fxbcid,
                                      const uint8_t* fybcid, const uint8_t* fzbcid, const uint8_t* fxo,
                                      const uint8_t* fyo, const uint8_t* fzo, const double* lamx, const double* lamy,
                                      const double* lamz, double* vxs, double* vys, double* vzs, void* stream);

/* Surface-tension face force f_s from the volume fraction,
 * G_SMACSolver::calc_surface_tension (CFD/G_SMACSolver_VoF.cu:435-445):
 *  1. on C_INTERIOR cells: grad alpha (central differences, one-sided next to
 *     non-interior cells), |grad alpha| into grad_mag, the unit normal into
 *     nx/ny/nz (0 where |grad|^2 <= 1e-12); other cells keep their values
 *     (k_calc_interface_normal :87-182);
 *  2. on cells 1..N: kappa = -div n, 0 outside 0.01 <= alpha <= 0.99, a
 *     neighbour counting only if C_INTERIOR with |grad alpha| > 1e-6
 *     (k_calc_curvature :184-290);
 *  3. every entry of fsx/fsy/fsz: sigma kappa_f (alpha_R - alpha_L) / h on
 *     faces 2..N along their axis and 1..N across between two C_INTERIOR
 *     cells (kappa_f the mean of the cells' kappa where 0.01 < alpha < 0.99),
 *     0 elsewhere (k_calc_surface_tension_face :292-433).
 * nx, ny, nz, kappa, grad_mag are cell arrays: the grid's nx_, ny_, nz_,
 * kappa_ and p_tmp_, read and written as the reference does. */
smac_status smac_surface_tension(const smac_grid_desc* d, const double* alpha, const uint8_t* celltype, double sigma,
                                 double* nx, double* ny, double* nz, double* kappa, double* grad_mag, double* fsx,
                                 double* fsy, double* fsz, void* stream);

/* Velocity part of update_boundary_ghost, in place on (vx, vy, vz):
 *  1. outlet faces (k_update_v*_outlet, CFD/G_BoundaryFunctions.cu:143-255):
 *     a face with outlet mark 1 (interior side +1) or 2 (side -1) -- the marks
 *     of smac_update_boundary_faces -- gets v = v* + sign f_b dt p_delta(face
 *     index + side) / h, sign = -side; skipped when fxo/fyo/fzo are NULL;
 *  2. ghost faces across each family's two tangential axes
 *     (k_update_v*_ghost, :277-520) by the type of the id in f_*bcid_ of the
 *     first face inside: inflow 2(1-lam)v_b - v2, no-slip -v2, outlet
 *     2 v1 - v2, slip v2, outflow v1 (v1, v2 the first and second faces
 *     inside, lam the f_ibm_area_solid_fraction_* entry of the first; lam*
 *     may be NULL: 0); edge corners the mean of their two ghost neighbours
 *     (k_update_v*_ghost_corner).
 * Every grid extent must be >= 2.  bcid entries >= num_ids read as no-slip
 * with velocity 0. */
smac_status smac_update_velocity_ghost(const smac_grid_desc* d, const smac_boundary_table* bc, const uint8_t* fxbcid,
                                       const uint8_t* fybcid, const uint8_t* fzbcid, const uint8_t* fxo,
                                       const uint8_t* fyo, const uint8_t* fzo, const double* lamx, const double* lamy,
                                       const double* lamz, const double* vxs, const double* vys, const double* vzs,
                                       const double* fbx, const double* fby, const double* fbz, const double* p_delta,
                                       double dt, double* vx, double* vy, double* vz, void* stream);

/* Face pressure gradient, G_SMACSolver::make_face_gradp
 * (CFD/G_SMACSolver.cu:1277-1343): gp_x(i) = (p(i) - p(i-x)) / dx and so on,
 * on face indices 1..N+1 of every axis of each family (other entries are not
 * written). */
smac_status smac_face_gradp(const smac_grid_desc* d, const double* p, double* gpx, double* gpy, double* gpz,
                            void* stream);

/* ---- output ----------------------------------------------------------------
 * FileInOut::output_vti_binary_cellData (CFD/FileInOut.cpp:144-262): a VTK
 * ImageData file of the interior cells with four Float32 cell arrays in raw
 * appended data, pressure, alpha, velocity (the mean of each cell's two faces,
 * 3 components) and ibm_solid_fraction, each after its UInt32 byte count.
 * Pack the appended block on the device, copy it to the host, write the file:
 * the file equals the reference's byte for byte. */

/* Bytes of the appended block: 16 + 24 Nx Ny Nz (0 for a bad grid). */
size_t smac_vti_block_bytes(const smac_grid_desc* d);
/* Build the appended block in device memory `block` (4-byte aligned,
 * smac_vti_block_bytes long) from the cell arrays p, alpha, ibm_sf and the
 * face arrays vx, vy, vz; alpha and ibm_sf may be NULL (written as 0).
 * Grids whose velocity block would pass 2^32 bytes are refused (the file's
 * size fields are UInt32). */
smac_status smac_vti_pack(const smac_grid_desc* d, const double* p, const double* alpha, const double* vx,
                          const double* vy, const double* vz, const double* ibm_sf, void* block, void* stream);
/* Write the .vti file `path` around a packed block in HOST memory; origin is
 * StaggeredGrid::origin_x_, y_, z_.  Host code only: it needs no GPU. */
smac_status smac_vti_write(const smac_grid_desc* d, const double origin[3], const void* block_host, const char* path);

/* y = A x with the FP64 fine operator (cells, reference layout, interior
 * entries); the reference's k_build_vof_poisson_Ap (G_PCGSolver.cu:214-245). */
smac_status smac_apply_A(smac_handle* h, const double* x, double* y);

/* Time `reps` launches of one kernel of the solve on the handle's stream with
 * CUDA events, on the finest grid (kernel ids: 0 FP64 matvec+dot, 1 FP32
 * matvec+dot, 2 FP64 fused red-black sweep, 3 FP32 fused red-black sweep,
 * 4 FP64 true residual, 5 FP64 sweep as two half-sweep launches, 6 FP32 sweep
 * as two half-sweep launches, 7 FP32 direction update + matvec, 8 FP64
 * direction update + matvec, 9 FP32 x/r update, 10 FP64 x/r update).  Writes the
 * mean milliseconds per launch (per sweep for 5 and 6) and the algorithmic
 * bytes of one launch. */
smac_status smac_time_kernel(smac_handle* h, int kernel_id, int reps, float* ms_per_launch,
                             double* alg_bytes_per_launch);

/* y = A x (interior cells, reference layout) and *xAx = x.Ax (one device
 * double) with the FP64 operator of smac_set_coefficients, built directly
 * from the reference-layout f_b and types, WITHOUT a handle and without
 * allocating any device memory.  No counterpart in the reference.
 * It is for callers that cannot allocate: a step loop being recorded into a
 * CUDA graph (cudaMalloc is not allowed while the stream captures) or a host
 * code whose pool allocator already owns the device memory.  Its scratch (the
 * reduction's per-block partials and arrival counter) is a static device array
 * of 64 KB that every GPU loading this library keeps until the process exits;
 * grids need ceil(nx/32)*ceil(ny/4) <= 8192 (x-y planes up to 1024 x 1024),
 * larger ones are refused with SMAC_BAD_SHAPE.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress), so make that
 * first call before any stream capture; a call after the device's context
 * has changed (cudaDeviceReset) looks it up again.  All calls share the one array:
 * calls that overlap on the GPU (other streams, other threads) race; order
 * them on one stream.  All pointers are device pointers; x's ghost entries are
 * not read. */
smac_status smac_apply_A_dot_noalloc(const smac_grid_desc* desc, const double* fbx, const double* fby,
                                     const double* fbz, const uint8_t* celltype, const uint8_t* fxt,
                                     const uint8_t* fyt, const uint8_t* fzt, const double* x, double* y,
                                     double* xAx, void* cuda_stream);

/* Self-test of the fused red-black sweep: runs one fused out-of-place sweep
 * (mode 0 plain, 1 from zero, 2 with the coarse-grid correction of grid 1
 * added to the input) and the same sweep as two in-place half-sweep launches
 * on the handle's current finest-grid iterate and residual (left by the last
 * solve; the call overwrites scratch vectors), and writes the number of cells
 * whose results differ bitwise.  precision: smac_precision of the vectors.
 * No counterpart in the reference (it has no Gauss-Seidel smoother). */
smac_status smac_selftest_sweep(smac_handle* h, int precision, int mode, long long* mismatches);

/* Self-test of the kernels' bounded waits: one warp waits on a shared-memory
 * mbarrier that nothing arrives on, with the limit every device-side wait of
 * this library uses (about one second of SM clock), and records the expiry
 * as the kernels do (solver status SMAC_CUDA_ERROR).  Writes the status the
 * device recorded (SMAC_CUDA_ERROR when the wait gave up) and the SM cycles it
 * waited; the handle stays usable (the status is cleared after the read).
 * No counterpart in the reference (its kernels do not wait on the device). */
smac_status smac_selftest_wait(smac_handle* h, int* status, long long* cycles);

/* ---------------------------------------------------------------------------
 * Projections with host buffers, queued.  A queue on a handle runs
 * smac_project on inputs and outputs in host memory (the reference layout, as
 * for smac_project), and overlaps each projection's copies with the solves of
 * its neighbours: the input of the next projection is copied in and the
 * outputs of the previous one are copied out while this one is solved.  Two
 * device staging slots and a worker thread belong to the queue.  New: the
 * reference solves one step at a time on device-resident arrays
 * (G_SMACSolver::solve_poisson, CFD/G_SMACSolver.cu:1499-1501).
 *
 * smac_async_submit copies the input in (asynchronously) and returns a
 * ticket; smac_async_wait(ticket) returns once that projection's outputs are
 * in host memory, with its status and statistics.  Host buffers should be
 * page-locked for the copies to overlap, and stay valid until the wait
 * returns.  While a queue exists, the handle must not be used directly. */
typedef struct smac_async smac_async;
smac_status smac_async_create(smac_handle* h, smac_async** out);
smac_status smac_async_submit(smac_async* a, const double* vxs, const double* vys, const double* vzs, double dt,
                              double* p_delta, double* vx, double* vy, double* vz, unsigned long long* ticket);
smac_status smac_async_wait(smac_async* a, unsigned long long ticket, smac_stats* stats);
void smac_async_destroy(smac_async* a);

#ifdef __cplusplus
}
#endif
#endif /* SMAC_B200_H */
