// G_B200PressureSolver.h -- the drop-in for the reference's pressure-solver
// seam: a G_PressureSolverBase (CFD/pressure_solver/G_PressureSolverBase.h:24-42)
// whose solve() runs this library's projection solve through the C ABI of
// include/smac_b200.h.  It is compiled with the reference's sources (it
// needs G_SMACSolver and G_StaggeredGrid) and links libsmac_b200.so.
//
// Installed in place of G_PCGSolver, one line in the driver
// (CFD/main.cu:225-227):
//
//     G_B200PressureSolver b200(isPureNeumann ? PURENEUMANN_GMG_PCG : GMG_PCG);
//     b200.copyData(g_solv);              // the base class's bookkeeping, unchanged
//     g_solv.pressure_solver_ = &b200;    // was: &pcgSolver
//
// G_SMACSolver::solve_poisson() (CFD/G_SMACSolver.cu:1499-1501) then calls
// solve() below, which reads the grid's device arrays in the reference
// layout and writes p_delta_ (and rhs_) where the reference's solver does;
// correct_vof_velocity() runs unchanged after it.  tol_ keeps its meaning:
// the reference's test max|r| * dt < tol_ (G_PCGSolver.cu:884-903), set per
// step by the driver (CFD/main.cu:260-268).
#pragma once

#include <cstdio>

#include "G_PressureSolverBase.h"
#include "smac_b200.h"

struct G_B200PressureSolver : G_PressureSolverBase {
  smac_handle* h_ = nullptr;
  smac_options opts_;
  smac_stats stats_{};
  int last_status_ = SMAC_OK;

  // pcg_type: the PCG_TYPES value (CFD/Enums.h:25-30; smac_solver_type has the
  // same values); precision: smac_precision.
  explicit G_B200PressureSolver(int pcg_type = PURENEUMANN_GMG_PCG, int precision = SMAC_PRECISION_FP64) {
    smac_default_options(&opts_);
    opts_.solver_type = pcg_type;
    opts_.precision = precision;
    opts_.stop_rule = SMAC_STOP_REFERENCE;  // the reference's test: max|r| * dt < tol_
    tol_ = opts_.tol;
  }
  ~G_B200PressureSolver() override {
    if (h_) smac_destroy(h_);
  }

  void solve(G_SMACSolver& solv) override {
    G_StaggeredGrid& g = solv.grid_;
    if (!h_) {
      smac_grid_desc d{g.Nx_, g.Ny_, g.Nz_, g.dx_, g.dy_, g.dz_};
      // a null stream: the handle's own blocking stream, ordered with the
      // legacy default stream on which the reference launches
      if ((last_status_ = smac_create(&d, &opts_, nullptr, &h_)) != SMAC_OK) {
        fprintf(stderr, "smac_create: %s\n", smac_last_error_string());
        h_ = nullptr;
        return;
      }
    }
    opts_.tol = tol_;
    smac_set_options(h_, &opts_);
    // the coefficients change with rho every step (update_properties_by_alpha)
    last_status_ = smac_set_coefficients(h_, g.f_bx_.data_, g.f_by_.data_, g.f_bz_.data_, g.celltype_.data_,
                                         g.f_xtype_.data_, g.f_ytype_.data_, g.f_ztype_.data_);
    if (last_status_ == SMAC_OK)
      last_status_ = smac_divergence(h_, g.f_vx_star_.data_, g.f_vy_star_.data_, g.f_vz_star_.data_,
                                     g.void_fraction_.data_, g.void_fraction_old_.data_, g.f_sx_.data_, g.f_sy_.data_,
                                     g.f_sz_.data_, solv.dt_, g.rhs_.data_);
    if (last_status_ == SMAC_OK) last_status_ = smac_solve(h_, g.p_delta_.data_, &stats_);
    if (last_status_ != SMAC_OK) fprintf(stderr, "G_B200PressureSolver: %s\n", smac_last_error_string());
    printf("PCG iter = %d\n", stats_.iterations);  // the reference's log line (G_PCGSolver.cu:921)
  }
};
