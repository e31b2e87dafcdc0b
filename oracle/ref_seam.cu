// ref_seam.cu -- the reference's own step calls with this library's solver
// installed at the reference's pressure-solver seam.  TEST INFRASTRUCTURE
// ONLY (oracle/Makefile, target `seam`): it proves the drop-in.
//
// The set-up is the reference driver's (CFD/main.cu:183-243), as in
// ref_harness.cu, except for the one line a maintainer changes: the solver
// installed at g.pressure_solver_ is G_B200PressureSolver
// (mydemcfd_b200/seam/G_B200PressureSolver.h) instead of G_PCGSolver.  Then
// the reference's G_SMACSolver::solve_poisson() and correct_vof_velocity()
// run unchanged.
#include <cstdio>

#include "G_SMACSolver.h"
#include "SMACSolver.h"
#include "G_B200PressureSolver.h"
#include "ref_harness.h"

extern "C" {

// Returns 0 on success, -2 on a CUDA error, -3 when the solver reported a
// status other than SMAC_OK (out->iterations then holds -status).
int ref_solve_seam(const ref_inputs* in, ref_outputs* out, int precision) {
  const int Nx = in->Nx, Ny = in->Ny, Nz = in->Nz;
  SMACSolver solv;
  solv.set_calc_properties(0., 0., 0., in->Lx, in->Ly, in->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = 1;
  solv.solver_malloc();
  StaggeredGrid& hg = solv.grid_;
  put(hg.f_vx_star_, in->vxs); put(hg.f_vy_star_, in->vys); put(hg.f_vz_star_, in->vzs);
  put(hg.void_fraction_, in->eps); put(hg.void_fraction_old_, in->eps_old);
  put(hg.f_bx_, in->fbx); put(hg.f_by_, in->fby); put(hg.f_bz_, in->fbz);
  put(hg.f_sx_, in->fsx); put(hg.f_sy_, in->fsy); put(hg.f_sz_, in->fsz);
  put(hg.f_inv_rhox_, in->firx); put(hg.f_inv_rhoy_, in->firy); put(hg.f_inv_rhoz_, in->firz);
  put(hg.celltype_, in->ct); put(hg.f_xtype_, in->fxt); put(hg.f_ytype_, in->fyt); put(hg.f_ztype_, in->fzt);
  solv.dt_ = in->dt;
  solv.inv_dt_ = 1. / in->dt;

  G_SMACSolver g;
  g.set_calc_properties(0., 0., 0., in->Lx, in->Ly, in->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = 1;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  g.dt_ = in->dt;
  g.inv_dt_ = 1. / in->dt;

  // the drop-in: the one line of CFD/main.cu:225-227 that changes
  G_B200PressureSolver b200(in->solver_type, precision);
  b200.copyData(g);
  g.pressure_solver_ = &b200;
  b200.tol_ = in->tol;
  cudaDeviceSynchronize();

  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0, 0);
  g.solve_poisson();
  cudaEventRecord(ev1, 0);
  cudaDeviceSynchronize();
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0, ev1);
  out->solve_ms = ms;
  out->iterations = b200.stats_.iterations;
  out->num_levels = b200.stats_.num_levels;
  int rc = 0;
  if (b200.last_status_ != SMAC_OK) {
    out->iterations = -b200.last_status_;
    rc = -3;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_solve_seam: %s\n", cudaGetErrorString(e));
    return -2;
  }
  g.gpuTocpu(solv.grid_);
  get(hg.p_delta_, out->p_delta);
  get(hg.rhs_, out->rhs);
  out->correct_ms = 0.0;
  if (in->do_correct && rc == 0) {
    cudaEventRecord(ev0, 0);
    g.correct_vof_velocity(solv);
    cudaEventRecord(ev1, 0);
    cudaDeviceSynchronize();
    cudaEventElapsedTime(&ms, ev0, ev1);
    out->correct_ms = ms;
    g.gpuTocpu(solv.grid_);
    get(hg.f_vx_, out->vx); get(hg.f_vy_, out->vy); get(hg.f_vz_, out->vz);
    get(hg.p_, out->p);
  }
  e = cudaGetLastError();
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_solve_seam: %s\n", cudaGetErrorString(e));
    return -2;
  }
  return rc;
}

}  // extern "C"
