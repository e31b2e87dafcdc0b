// ref_harness.cu -- a small driver of ours that runs the REFERENCE's own GPU
// pressure path, compiled unmodified from its sources (oracle/Makefile, target
// `ref`), on host arrays.  TEST INFRASTRUCTURE ONLY: it pins the CPU oracle
// (oracle/smac_oracle.cpp) to the reference and produces the golden vectors in
// tests/golden/.  The product never links it.
//
// It follows the reference driver's set-up (CFD/main.cu:183-243): a host
// SMACSolver with calloc'ed members, G_SMACSolver::solver_malloc + cpuTogpu,
// G_PCGSolver + G_GMGSolver::initialize, set_solver, tol_, then
// G_SMACSolver::solve_poisson() and correct_vof_velocity().  More entries
// run the calls either side of it on given arrays: ref_predict_vstar
// (get_vof_vstar_rhouu_consistent), ref_update_properties
// (update_properties_by_alpha), ref_vstar (update_vstar_boundary),
// ref_surface_tension (calc_surface_tension) and ref_post
// (update_boundary_ghost and make_face_gradp).
//
// Two things the reference leaves to chance are pinned here: every multigrid
// level array is zeroed after G_GMGSolver::initialize (the reference reads
// never-written ghost entries of q_tmp_ and of the coarse f_b arrays), and
// shapes for which the reference would abort() or index levels_[-1] are
// refused before any reference code runs.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>

#include "G_SMACSolver.h"
#include "SMACSolver.h"
#include "../Coupling/G_CFDDEMCoupling.h"
#include "pressure_solver/G_GMGSolver.h"
#include "pressure_solver/G_PCGSolver.h"
#include "ref_harness.h"

namespace {

// G_GMGSolver::initialize's level count and abort conditions
// (CFD/pressure_solver/G_GMGSolver.cu:10-147), evaluated without running it.
int count_levels(int Nx, int Ny, int Nz, int levels, int min_size) {
  bool cx = Nx / 2 >= min_size, cy = Ny / 2 >= min_size, cz = Nz / 2 >= min_size;
  if ((Nx % 2 == 1 && cx) || (Ny % 2 == 1 && cy) || (Nz % 2 == 1 && cz)) return -1;
  int sx = cx ? Nx / 2 : Nx, sy = cy ? Ny / 2 : Ny, sz = cz ? Nz / 2 : Nz;
  int n = 1;
  for (int i = 1; i < levels; ++i) {
    cx = sx / 2 >= min_size; cy = sy / 2 >= min_size; cz = sz / 2 >= min_size;
    if (!cx && !cy && !cz) break;
    if ((sx % 2 == 1 && cx) || (sy % 2 == 1 && cy) || (sz % 2 == 1 && cz)) return -1;
    if (cx) sx /= 2;
    if (cy) sy /= 2;
    if (cz) sz /= 2;
    ++n;
  }
  return n;
}

}  // namespace

extern "C" {

// Returns 0 on success, -1 refused shape, -2 CUDA error.
int ref_solve(const ref_inputs* in, ref_outputs* out) {
  const int Nx = in->Nx, Ny = in->Ny, Nz = in->Nz;
  const bool gmg = in->solver_type == GMG_PCG || in->solver_type == PURENEUMANN_GMG_PCG;
  if (gmg) {
    const int nl = count_levels(Nx, Ny, Nz, in->levels, 6);
    if (nl < 2) return -1;
    out->num_levels = nl;
  }
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

  G_PCGSolver pcg;
  pcg.copyData(g);
  g.pressure_solver_ = &pcg;
  G_GMGSolver gmgs;
  if (gmg) {
    gmgs.initialize(g, in->levels);
    gmgs.copyData(g);
    for (int i = 0; i < gmgs.num_levels_; ++i) {
#define MEMBER(type, name, xs, ys, zs, save) \
      cudaMemset(gmgs.levels_[i].name.data_, 0, sizeof(type) * (size_t)gmgs.levels_[i].name.size_);
#include "memberList/levelMembers.def"
#undef MEMBER
    }
    pcg.set_gmg(gmgs);
  }
  pcg.set_solver((PCG_TYPES)in->solver_type);
  pcg.tol_ = in->tol;
  cudaDeviceSynchronize();

  // capture the reference's stdout to read its iteration count
  fflush(stdout);
  char path[] = "/tmp/ref_harness_XXXXXX";
  const int fd = mkstemp(path);
  const int saved = dup(1);
  if (fd >= 0) dup2(fd, 1);
  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0, 0);
  g.solve_poisson();
  cudaEventRecord(ev1, 0);
  cudaDeviceSynchronize();
  {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    out->solve_ms = ms;
  }
  fflush(stdout);
  if (fd >= 0) {
    dup2(saved, 1);
    close(saved);
    FILE* f = fopen(path, "r");
    char line[512];
    out->iterations = -1;
    while (f && fgets(line, sizeof(line), f)) {
      int it;
      if (sscanf(line, "PCG iter = %d", &it) == 1) out->iterations = it;
    }
    if (f) fclose(f);
    close(fd);
    unlink(path);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_solve: %s\n", cudaGetErrorString(e));
    return -2;
  }
  g.gpuTocpu(solv.grid_);
  get(hg.p_delta_, out->p_delta);
  get(hg.rhs_, out->rhs);
  out->correct_ms = 0.0;
  if (in->do_correct) {
    cudaEventRecord(ev0, 0);
    g.correct_vof_velocity(solv);
    cudaEventRecord(ev1, 0);
    cudaDeviceSynchronize();
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    out->correct_ms = ms;
    g.gpuTocpu(solv.grid_);
    get(hg.f_vx_, out->vx); get(hg.f_vy_, out->vy); get(hg.f_vz_, out->vz);
    get(hg.p_, out->p);
  }
  e = cudaGetLastError();
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (gmg) gmgs.free_levels();
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

struct ref_post_inputs {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz, dt, gx, gy, gz;
  int num_ids;                         // bc_.num_boundary_id_
  const uint8_t* bc_type;              // bc_.bcType_
  const double *bc_vx, *bc_vy, *bc_vz; // bc_.vx_, vy_, vz_
  const double *p, *p_delta, *rho;
  const uint8_t *ct, *fxt, *fyt, *fzt, *fxbcid, *fybcid, *fzbcid;
  const int *fxid, *fyid, *fzid;       // f_*internal_id_
  const double *lamx, *lamy, *lamz;    // f_ibm_area_solid_fraction_*
  const double *vxs, *vys, *vzs, *fbx, *fby, *fbz, *vx, *vy, *vz;
};

struct ref_post_outputs {
  double *p, *vx, *vy, *vz, *gpx, *gpy, *gpz;
  double ghost_ms;  // device time of update_boundary_ghost (CUDA events, legacy stream)
  double gradp_ms;  // device time of make_face_gradp
};

// The grid of a ref_post_inputs on host and device, as the reference's
// driver sets it up (CFD/main.cu:183-243).
static void post_setup(const ref_post_inputs* in, SMACSolver& solv, G_SMACSolver& g) {
  const int Nx = in->Nx, Ny = in->Ny, Nz = in->Nz;
  solv.set_calc_properties(0., 0., 0., in->Lx, in->Ly, in->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = in->num_ids;
  solv.solver_malloc();
  solv.gx_ = in->gx; solv.gy_ = in->gy; solv.gz_ = in->gz;
  solv.dt_ = in->dt;
  solv.inv_dt_ = 1. / in->dt;
  StaggeredGrid& hg = solv.grid_;
  put(hg.p_, in->p); put(hg.p_delta_, in->p_delta); put(hg.rho_, in->rho);
  put(hg.celltype_, in->ct); put(hg.f_xtype_, in->fxt); put(hg.f_ytype_, in->fyt); put(hg.f_ztype_, in->fzt);
  put(hg.f_xbcid_, in->fxbcid); put(hg.f_ybcid_, in->fybcid); put(hg.f_zbcid_, in->fzbcid);
  put(hg.f_xinternal_id_, in->fxid); put(hg.f_yinternal_id_, in->fyid); put(hg.f_zinternal_id_, in->fzid);
  put(hg.f_ibm_area_solid_fraction_x_, in->lamx); put(hg.f_ibm_area_solid_fraction_y_, in->lamy);
  put(hg.f_ibm_area_solid_fraction_z_, in->lamz);
  put(hg.f_vx_star_, in->vxs); put(hg.f_vy_star_, in->vys); put(hg.f_vz_star_, in->vzs);
  put(hg.f_bx_, in->fbx); put(hg.f_by_, in->fby); put(hg.f_bz_, in->fbz);
  put(hg.f_vx_, in->vx); put(hg.f_vy_, in->vy); put(hg.f_vz_, in->vz);
  std::memcpy(hg.bc_.bcType_.data_, in->bc_type, (size_t)in->num_ids);
  std::memcpy(hg.bc_.vx_.data_, in->bc_vx, sizeof(double) * (size_t)in->num_ids);
  std::memcpy(hg.bc_.vy_.data_, in->bc_vy, sizeof(double) * (size_t)in->num_ids);
  std::memcpy(hg.bc_.vz_.data_, in->bc_vz, sizeof(double) * (size_t)in->num_ids);

  g.set_calc_properties(0., 0., 0., in->Lx, in->Ly, in->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = in->num_ids;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  g.dt_ = in->dt;
  g.inv_dt_ = 1. / in->dt;
  cudaDeviceSynchronize();
}

// G_SMACSolver::update_boundary_ghost then make_face_gradp
// (CFD/G_SMACSolver.cu:1277-1363), the reference's pass after the projection,
// on host arrays.  Returns 0 on success, -2 on a CUDA error.
int ref_post(const ref_post_inputs* in, ref_post_outputs* out) {
  SMACSolver solv;
  G_SMACSolver g;
  post_setup(in, solv, g);
  StaggeredGrid& hg = solv.grid_;
  cudaEvent_t ev[3];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  g.update_boundary_ghost(solv);
  cudaEventRecord(ev[1], 0);
  g.make_face_gradp();
  cudaEventRecord(ev[2], 0);
  cudaDeviceSynchronize();
  float ms0 = 0.f, ms1 = 0.f;
  cudaEventElapsedTime(&ms0, ev[0], ev[1]);
  cudaEventElapsedTime(&ms1, ev[1], ev[2]);
  out->ghost_ms = ms0;
  out->gradp_ms = ms1;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    g.gpuTocpu(solv.grid_);
    get(hg.p_, out->p);
    get(hg.f_vx_, out->vx); get(hg.f_vy_, out->vy); get(hg.f_vz_, out->vz);
    get(hg.f_gradp_x_, out->gpx); get(hg.f_gradp_y_, out->gpy); get(hg.f_gradp_z_, out->gpz);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

// G_SMACSolver::update_vstar_boundary (CFD/G_SMACSolver.cu:1044-1052) on the
// u* of a ref_post_inputs; *ms receives its device time.
int ref_vstar(const ref_post_inputs* in, double* vxs, double* vys, double* vzs, double* ms) {
  SMACSolver solv;
  G_SMACSolver g;
  post_setup(in, solv, g);
  StaggeredGrid& hg = solv.grid_;
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  g.update_vstar_boundary();
  cudaEventRecord(ev[1], 0);
  cudaDeviceSynchronize();
  float t = 0.f;
  cudaEventElapsedTime(&t, ev[0], ev[1]);
  *ms = t;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    g.gpuTocpu(solv.grid_);
    get(hg.f_vx_star_, vxs); get(hg.f_vy_star_, vys); get(hg.f_vz_star_, vzs);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

struct ref_st_io {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz, sigma;
  const double* alpha;
  const uint8_t* ct;
  double *nx, *ny, *nz, *kappa, *gm;  // in: initial contents (nx_, ny_, nz_, kappa_, p_tmp_); out: final
  double *fsx, *fsy, *fsz;            // out
  double ms;                          // out: device time of calc_surface_tension
};

// G_SMACSolver::calc_surface_tension (CFD/G_SMACSolver_VoF.cu:435-445) on
// host arrays.  Returns 0 on success, -2 on a CUDA error.
int ref_surface_tension(ref_st_io* io) {
  const int Nx = io->Nx, Ny = io->Ny, Nz = io->Nz;
  SMACSolver solv;
  solv.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = 1;
  solv.solver_malloc();
  StaggeredGrid& hg = solv.grid_;
  put(hg.alpha_, io->alpha); put(hg.celltype_, io->ct);
  put(hg.nx_, io->nx); put(hg.ny_, io->ny); put(hg.nz_, io->nz); put(hg.kappa_, io->kappa); put(hg.p_tmp_, io->gm);
  hg.sigma_.data_[0] = io->sigma;
  G_SMACSolver g;
  g.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = 1;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  cudaDeviceSynchronize();
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  g.calc_surface_tension();
  cudaEventRecord(ev[1], 0);
  cudaDeviceSynchronize();
  float t = 0.f;
  cudaEventElapsedTime(&t, ev[0], ev[1]);
  io->ms = t;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    g.gpuTocpu(solv.grid_);
    get(hg.nx_, io->nx); get(hg.ny_, io->ny); get(hg.nz_, io->nz); get(hg.kappa_, io->kappa); get(hg.p_tmp_, io->gm);
    get(hg.f_sx_, io->fsx); get(hg.f_sy_, io->fsy); get(hg.f_sz_, io->fsz);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

struct ref_mom_io {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz, dt, gx, gy, gz;
  int num_ids;
  const uint8_t* bc_type;
  const double *bc_vx, *bc_vy, *bc_vz;
  const uint8_t *ft[3], *bcid[3];
  const double *lam[3], *v[3], *mf[3], *muf[3], *fb[3], *imp[3], *sf[3];
  const double *mu, *rho_old, *p;
  double* vs[3];  // in: u* before the call; out: after it
  double ms;      // out: device time
  // set: the two-way form (void fractions and f_inv_rho); NULL: the one-way form
  const double *eps_old, *eps_new, *fir[3];
};

// G_SMACSolver::get_vof_vstar_rhouu_consistent (CFD/G_SMACSolver.cu:1062-1070),
// or with io->eps_old set get_vof_vstar_rhouu_consistent_two_way (:2196-2203),
// on host arrays.  Returns 0 on success, -2 on a CUDA error.
int ref_predict_vstar(ref_mom_io* io) {
  const int Nx = io->Nx, Ny = io->Ny, Nz = io->Nz;
  SMACSolver solv;
  solv.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = io->num_ids;
  solv.solver_malloc();
  solv.dt_ = io->dt;
  solv.inv_dt_ = 1. / io->dt;
  solv.gx_ = io->gx; solv.gy_ = io->gy; solv.gz_ = io->gz;
  StaggeredGrid& hg = solv.grid_;
  put(hg.f_xtype_, io->ft[0]); put(hg.f_ytype_, io->ft[1]); put(hg.f_ztype_, io->ft[2]);
  put(hg.f_xbcid_, io->bcid[0]); put(hg.f_ybcid_, io->bcid[1]); put(hg.f_zbcid_, io->bcid[2]);
  put(hg.f_ibm_area_solid_fraction_x_, io->lam[0]); put(hg.f_ibm_area_solid_fraction_y_, io->lam[1]);
  put(hg.f_ibm_area_solid_fraction_z_, io->lam[2]);
  put(hg.f_vx_, io->v[0]); put(hg.f_vy_, io->v[1]); put(hg.f_vz_, io->v[2]);
  put(hg.f_mfx_, io->mf[0]); put(hg.f_mfy_, io->mf[1]); put(hg.f_mfz_, io->mf[2]);
  put(hg.f_mux_, io->muf[0]); put(hg.f_muy_, io->muf[1]); put(hg.f_muz_, io->muf[2]);
  put(hg.f_bx_, io->fb[0]); put(hg.f_by_, io->fb[1]); put(hg.f_bz_, io->fb[2]);
  put(hg.f_coupling_impulse_x_, io->imp[0]); put(hg.f_coupling_impulse_y_, io->imp[1]);
  put(hg.f_coupling_impulse_z_, io->imp[2]);
  put(hg.f_ibm_solid_fraction_x_, io->sf[0]); put(hg.f_ibm_solid_fraction_y_, io->sf[1]);
  put(hg.f_ibm_solid_fraction_z_, io->sf[2]);
  put(hg.mu_, io->mu); put(hg.rho_old_, io->rho_old); put(hg.p_, io->p);
  put(hg.void_fraction_old_, io->eps_old); put(hg.void_fraction_, io->eps_new);
  put(hg.f_inv_rhox_, io->fir[0]); put(hg.f_inv_rhoy_, io->fir[1]); put(hg.f_inv_rhoz_, io->fir[2]);
  put(hg.f_vx_star_, io->vs[0]); put(hg.f_vy_star_, io->vs[1]); put(hg.f_vz_star_, io->vs[2]);
  std::memcpy(hg.bc_.bcType_.data_, io->bc_type, (size_t)io->num_ids);
  std::memcpy(hg.bc_.vx_.data_, io->bc_vx, sizeof(double) * (size_t)io->num_ids);
  std::memcpy(hg.bc_.vy_.data_, io->bc_vy, sizeof(double) * (size_t)io->num_ids);
  std::memcpy(hg.bc_.vz_.data_, io->bc_vz, sizeof(double) * (size_t)io->num_ids);
  G_SMACSolver g;
  g.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = io->num_ids;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  g.dt_ = io->dt;
  g.inv_dt_ = 1. / io->dt;
  cudaDeviceSynchronize();
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  if (io->eps_old)
    g.get_vof_vstar_rhouu_consistent_two_way(solv);
  else
    g.get_vof_vstar_rhouu_consistent(solv);
  cudaEventRecord(ev[1], 0);
  cudaDeviceSynchronize();
  float t = 0.f;
  cudaEventElapsedTime(&t, ev[0], ev[1]);
  io->ms = t;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    g.gpuTocpu(solv.grid_);
    get(hg.f_vx_star_, io->vs[0]); get(hg.f_vy_star_, io->vs[1]); get(hg.f_vz_star_, io->vs[2]);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

struct ref_props_io {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz, rho0, rho1, mu0, mu1;
  const double* alpha;
  const uint8_t *ct, *ft[3];
  // in: contents before the call, rho_old the array that becomes rho after
  // the reference's swap; out: after it
  double *rho, *rho_old, *inv_rho, *mu, *fb[3], *fir[3], *frho[3], *fmu[3];
  double ms;
};

// G_SMACSolver::update_properties_by_alpha (CFD/G_SMACSolver_VoF.cu:1543-1566)
// on host arrays.  Returns 0 on success, -2 on a CUDA error.
int ref_update_properties(ref_props_io* io) {
  const int Nx = io->Nx, Ny = io->Ny, Nz = io->Nz;
  SMACSolver solv;
  solv.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = 1;
  solv.solver_malloc();
  StaggeredGrid& hg = solv.grid_;
  put(hg.alpha_, io->alpha); put(hg.celltype_, io->ct);
  put(hg.f_xtype_, io->ft[0]); put(hg.f_ytype_, io->ft[1]); put(hg.f_ztype_, io->ft[2]);
  put(hg.rho_, io->rho); put(hg.rho_old_, io->rho_old); put(hg.inv_rho_, io->inv_rho); put(hg.mu_, io->mu);
  put(hg.f_bx_, io->fb[0]); put(hg.f_by_, io->fb[1]); put(hg.f_bz_, io->fb[2]);
  put(hg.f_inv_rhox_, io->fir[0]); put(hg.f_inv_rhoy_, io->fir[1]); put(hg.f_inv_rhoz_, io->fir[2]);
  put(hg.f_rhox_, io->frho[0]); put(hg.f_rhoy_, io->frho[1]); put(hg.f_rhoz_, io->frho[2]);
  put(hg.f_mux_, io->fmu[0]); put(hg.f_muy_, io->fmu[1]); put(hg.f_muz_, io->fmu[2]);
  G_SMACSolver g;
  g.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = 1;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  g.rho0_ = io->rho0; g.rho1_ = io->rho1; g.mu0_ = io->mu0; g.mu1_ = io->mu1;
  cudaDeviceSynchronize();
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  g.update_properties_by_alpha();
  cudaEventRecord(ev[1], 0);
  cudaDeviceSynchronize();
  float t = 0.f;
  cudaEventElapsedTime(&t, ev[0], ev[1]);
  io->ms = t;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    // the device grid's rho_/rho_old_ pointers were swapped; copy back by member
    g.gpuTocpu(solv.grid_);
    get(hg.rho_, io->rho); get(hg.rho_old_, io->rho_old); get(hg.inv_rho_, io->inv_rho); get(hg.mu_, io->mu);
    get(hg.f_bx_, io->fb[0]); get(hg.f_by_, io->fb[1]); get(hg.f_bz_, io->fb[2]);
    get(hg.f_inv_rhox_, io->fir[0]); get(hg.f_inv_rhoy_, io->fir[1]); get(hg.f_inv_rhoz_, io->fir[2]);
    get(hg.f_rhox_, io->frho[0]); get(hg.f_rhoy_, io->frho[1]); get(hg.f_rhoz_, io->frho[2]);
    get(hg.f_mux_, io->fmu[0]); get(hg.f_muy_, io->fmu[1]); get(hg.f_muz_, io->fmu[2]);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

}  // extern "C"

struct ref_beta_io {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz;
  const double* eps;       // void_fraction_
  const double* fir[3];    // f_inv_rho*_
  double* fb[3];           // in: f_b*_ before the call; out: after it
  double ms;               // out: device time
};

// G_CFDDEMCoupling::update_poisson_beta_two_way (Coupling/G_CFDDEMCoupling.cu:
// 419-460) on host arrays, launched with the dimensions the coupled driver
// gives it (those of G_SMACSolver::set_block_grid, Coupling/main.cu:484-485).
// Returns 0 on success, -2 on a CUDA error.
extern "C" int ref_poisson_beta_two_way(ref_beta_io* io) {
  const int Nx = io->Nx, Ny = io->Ny, Nz = io->Nz;
  SMACSolver solv;
  solv.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = 1;  // sizes the boundary table solver_malloc allocates
  solv.solver_malloc();
  StaggeredGrid& hg = solv.grid_;
  put(hg.void_fraction_, io->eps);
  put(hg.f_inv_rhox_, io->fir[0]); put(hg.f_inv_rhoy_, io->fir[1]); put(hg.f_inv_rhoz_, io->fir[2]);
  put(hg.f_bx_, (const double*)io->fb[0]); put(hg.f_by_, (const double*)io->fb[1]);
  put(hg.f_bz_, (const double*)io->fb[2]);
  G_SMACSolver g;
  g.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = 1;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  G_CFDDEMCoupling cpl;
  cpl.block_dim_ = g.block_dim_;
  cpl.grid_dim_ = g.grid_dim_;
  cudaDeviceSynchronize();
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  cpl.update_poisson_beta_two_way(g.grid_);
  cudaEventRecord(ev[1], 0);
  cudaDeviceSynchronize();
  float t = 0.f;
  cudaEventElapsedTime(&t, ev[0], ev[1]);
  io->ms = t;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    g.gpuTocpu(solv.grid_);
    get(hg.f_bx_, io->fb[0]); get(hg.f_by_, io->fb[1]); get(hg.f_bz_, io->fb[2]);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}

struct ref_flux_io {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz, dt, rho0, rho1;
  int num_ids;
  const uint8_t* bc_type;
  const double *bc_vx, *bc_vy, *bc_vz;
  const uint8_t *ft[3], *bcid[3];
  const double *lam[3], *v[3], *F[3];
  const double* eps_half;  // set: the two-way form; NULL: the one-way form
  double* mf[3];           // in: f_mf*_ before the call; out: after it
  double ms;               // out: device time
};

// G_SMACSolver::compute_mass_flux_from_alpha_flux (CFD/G_SMACSolver_VoF.cu:
// 1792-1795), or with io->eps_half set compute_mass_flux_from_alpha_flux_two_way
// (:2685-2687), on host arrays.  Returns 0 on success, -2 on a CUDA error.
extern "C" int ref_mass_flux(ref_flux_io* io) {
  const int Nx = io->Nx, Ny = io->Ny, Nz = io->Nz;
  SMACSolver solv;
  solv.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  solv.grid_.bc_.num_boundary_id_ = io->num_ids;
  solv.solver_malloc();
  solv.dt_ = io->dt;
  solv.inv_dt_ = 1. / io->dt;
  solv.rho0_ = io->rho0;
  solv.rho1_ = io->rho1;
  StaggeredGrid& hg = solv.grid_;
  put(hg.f_xtype_, io->ft[0]); put(hg.f_ytype_, io->ft[1]); put(hg.f_ztype_, io->ft[2]);
  put(hg.f_xbcid_, io->bcid[0]); put(hg.f_ybcid_, io->bcid[1]); put(hg.f_zbcid_, io->bcid[2]);
  put(hg.f_ibm_area_solid_fraction_x_, io->lam[0]); put(hg.f_ibm_area_solid_fraction_y_, io->lam[1]);
  put(hg.f_ibm_area_solid_fraction_z_, io->lam[2]);
  put(hg.f_vx_, io->v[0]); put(hg.f_vy_, io->v[1]); put(hg.f_vz_, io->v[2]);
  put(hg.f_Fx_accum_, io->F[0]); put(hg.f_Fy_accum_, io->F[1]); put(hg.f_Fz_accum_, io->F[2]);
  put(hg.void_fraction_half_, io->eps_half);
  put(hg.f_mfx_, (const double*)io->mf[0]); put(hg.f_mfy_, (const double*)io->mf[1]);
  put(hg.f_mfz_, (const double*)io->mf[2]);
  std::memcpy(hg.bc_.bcType_.data_, io->bc_type, (size_t)io->num_ids);
  std::memcpy(hg.bc_.vx_.data_, io->bc_vx, sizeof(double) * (size_t)io->num_ids);
  std::memcpy(hg.bc_.vy_.data_, io->bc_vy, sizeof(double) * (size_t)io->num_ids);
  std::memcpy(hg.bc_.vz_.data_, io->bc_vz, sizeof(double) * (size_t)io->num_ids);
  G_SMACSolver g;
  g.set_calc_properties(0., 0., 0., io->Lx, io->Ly, io->Lz, Nx, Ny, Nz);
  g.grid_.bc_.num_boundary_id_ = io->num_ids;
  g.solver_malloc();
  g.cpuTogpu(solv.grid_);
  g.set_block_grid(Nx, Ny, Nz);
  g.dt_ = io->dt;
  g.inv_dt_ = 1. / io->dt;
  cudaDeviceSynchronize();
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], 0);
  if (io->eps_half)
    g.compute_mass_flux_from_alpha_flux_two_way(solv);
  else
    g.compute_mass_flux_from_alpha_flux(solv);
  cudaEventRecord(ev[1], 0);
  cudaDeviceSynchronize();
  float t = 0.f;
  cudaEventElapsedTime(&t, ev[0], ev[1]);
  io->ms = t;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    g.gpuTocpu(solv.grid_);
    get(hg.f_mfx_, io->mf[0]); get(hg.f_mfy_, io->mf[1]); get(hg.f_mfz_, io->mf[2]);
    e = cudaGetLastError();
  }
  g.solver_free();
  solv.solver_free();
  return e == cudaSuccess ? 0 : -2;
}
