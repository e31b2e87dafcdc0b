// smac_oracle.cpp -- CPU restatement of the reference SMAC pressure projection.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// path in mydemcfd_b200/csrc; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py may load it.  The product
// never links it and never falls back to it.
//
// It restates, operation for operation, the reference's GPU algorithm for the
// pressure path (the reference has no CPU pressure solve: CFD/main.cu:60-69
// refuses to run on the CPU and CFD/SMACSolver.cpp declares but never defines
// solve_poisson).  Arrays use the reference layout: MyArray<T,3> with x
// fastest, index (z*sy + y)*sx + x (CFD/MyArray.h:43-51); cells are
// (Nx+2)(Ny+2)(Nz+2), x-faces (Nx+3)(Ny+2)(Nz+2), y-faces (Nx+2)(Ny+3)(Nz+2),
// z-faces (Nx+2)(Ny+2)(Nz+3) (CFD/memberList/gridMembers.def).
//
// Build with -ffp-contract=off: the reference is compiled with -fmad=false
// (makefile_CFD:5), so every elementwise kernel here rounds exactly like the
// reference's.  Reductions (the reference calls cub::DeviceReduce::Sum/Max)
// use a fixed-chunk pairwise order that does not depend on the thread count.
//
// Memory the reference reads without ever writing (the ghost entries of the
// multigrid q_tmp_ buffers and of the coarse-level face coefficients,
// CFD/pressure_solver/G_GMGSolver.cu:499-644,692-717) is taken to be zero.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// CFD/Enums.h:3-23
enum : uint8_t { F_INTERIOR = 0, F_BOUNDARY = 1, F_GHOST = 2, F_NEAR_BOUNDARY = 3 };
enum : uint8_t { C_INTERIOR = 0, C_NEAR_BOUNDARY = 1, C_GHOST = 2, C_SOLID = 3 };
// CFD/Enums.h:25-30
enum : int { STANDARD_PCG = 0, PURENEUMANN_STANDARD_PCG = 1, GMG_PCG = 2, PURENEUMANN_GMG_PCG = 3 };

constexpr double kEPS = 1.e-12;  // CFD/hardCodedParameters.h:7

struct Arr {
  double* d = nullptr;
  int sx = 0, sy = 0, sz = 0;
  inline double& operator()(int x, int y, int z) const {
    return d[((size_t)z * sy + y) * sx + x];
  }
  size_t size() const { return (size_t)sx * sy * sz; }
};

struct Buf {
  std::vector<double> v;
  Arr a;
  void alloc(int sx, int sy, int sz) {
    v.assign((size_t)sx * sy * sz, 0.0);
    a.d = v.data();
    a.sx = sx; a.sy = sy; a.sz = sz;
  }
};

template <class T>
struct View {
  T* d = nullptr;
  int sx = 0, sy = 0, sz = 0;
  inline T& operator()(int x, int y, int z) const {
    return d[((size_t)z * sy + y) * sx + x];
  }
};

// Deterministic sum: fixed chunks of whole (y,z) rows, each chunk summed
// sequentially, chunk partials combined pairwise.  Independent of threads.
template <class F>
double det_sum_rows(int nrows, F&& rowsum) {
  const int chunk = 16;
  const int nchunks = (nrows + chunk - 1) / chunk;
  std::vector<double> part(nchunks, 0.0);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nchunks; ++c) {
    double s = 0.0;
    const int r1 = std::min(nrows, (c + 1) * chunk);
    for (int r = c * chunk; r < r1; ++r) s += rowsum(r);
    part[c] = s;
  }
  // pairwise combine
  int n = nchunks;
  while (n > 1) {
    const int h = n / 2;
    for (int i = 0; i < h; ++i) part[i] = part[2 * i] + part[2 * i + 1];
    if (n & 1) part[h] = part[n - 1];
    n = h + (n & 1);
  }
  return nchunks ? part[0] : 0.0;
}

template <class F>
double det_max_rows(int nrows, F&& rowmax) {
  double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (int r = 0; r < nrows; ++r) m = std::max(m, rowmax(r));
  return m;
}

// ---------------------------------------------------------------------------
// Grid state for one solve (the subset of G_StaggeredGrid the path touches).
struct Grid {
  int Nx, Ny, Nz;
  double inv_dx, inv_dy, inv_dz, inv_dx2, inv_dy2, inv_dz2;
  View<const uint8_t> ct, fxt, fyt, fzt;
  Arr fbx, fby, fbz;            // face coefficients (inputs, read only)
  Buf rhs, r, z, dir, Ap, ptmp, res; // cell work arrays, (N+2)^3
  Buf Axp, Axm, Ayp, Aym, Azp, Azm, Adiag, invAdiag;
  Arr pd;                       // p_delta_ (caller owned, in/out)
};

// ---------------------------------------------------------------------------
// Multigrid hierarchy: CFD/pressure_solver/G_GMGSolver.{h,cu}, G_Levels.h,
// CFD/memberList/levelMembers.def.
struct Level {
  bool cx = true, cy = true, cz = true;
  double idx2, idy2, idz2;
  Buf q, qtmp, fbx, fby, fbz, rhs, res, Axp, Axm, Ayp, Aym, Azp, Azm, invAdiag, Adiag;
  int sx() const { return q.a.sx; }
  int sy() const { return q.a.sy; }
  int sz() const { return q.a.sz; }
};

struct GMG {
  int num_levels = 0;
  int min_size = 6;         // G_GMGSolver.h:22
  int num_iter_coarse = 30; // G_GMGSolver.h:23
  int num_iter_fine = 4;    // G_GMGSolver.h:24
  double omega = 0.6;       // G_GMGSolver.cu:697,724
  std::vector<Level> lv;
};

// G_GMGSolver::initialize (G_GMGSolver.cu:10-147).  Returns 0, or -1 where
// the reference would abort() (odd size in a direction that coarsens).
int gmg_initialize(GMG& g, const Grid& grid, int num_levels) {
  if (num_levels > 16 || num_levels < 1) return -1;
  g.lv.clear();
  g.lv.reserve(num_levels);
  g.num_levels = 0;
  const int Nx = grid.Nx, Ny = grid.Ny, Nz = grid.Nz;
  {
    Level L;
    if (Nx / 2 < g.min_size) L.cx = false;
    if (Ny / 2 < g.min_size) L.cy = false;
    if (Nz / 2 < g.min_size) L.cz = false;
    if ((Nx % 2 == 1 && L.cx) || (Ny % 2 == 1 && L.cy) || (Nz % 2 == 1 && L.cz)) return -1;
    const int nx = L.cx ? Nx / 2 : Nx, ny = L.cy ? Ny / 2 : Ny, nz = L.cz ? Nz / 2 : Nz;
    for (Buf* b : {&L.q, &L.qtmp, &L.rhs, &L.res, &L.Axp, &L.Axm, &L.Ayp, &L.Aym, &L.Azp, &L.Azm,
                   &L.invAdiag, &L.Adiag})
      b->alloc(nx + 2, ny + 2, nz + 2);
    L.fbx.alloc(nx + 3, ny + 2, nz + 2);
    L.fby.alloc(nx + 2, ny + 3, nz + 2);
    L.fbz.alloc(nx + 2, ny + 2, nz + 3);
    L.idx2 = L.cx ? grid.inv_dx2 * 0.25 : grid.inv_dx2;
    L.idy2 = L.cy ? grid.inv_dy2 * 0.25 : grid.inv_dy2;
    L.idz2 = L.cz ? grid.inv_dz2 * 0.25 : grid.inv_dz2;
    g.lv.push_back(std::move(L));
    g.num_levels = 1;
  }
  for (int i = 1; i < num_levels; ++i) {
    const Level& O = g.lv[i - 1];
    Level L;
    if ((O.sx() - 2) / 2 < g.min_size) L.cx = false;
    if ((O.sy() - 2) / 2 < g.min_size) L.cy = false;
    if ((O.sz() - 2) / 2 < g.min_size) L.cz = false;
    if (!L.cx && !L.cy && !L.cz) break;
    if (((O.sx() - 2) % 2 == 1 && L.cx) || ((O.sy() - 2) % 2 == 1 && L.cy) ||
        ((O.sz() - 2) % 2 == 1 && L.cz))
      return -1;
    const int nx = L.cx ? (O.sx() - 2) / 2 : O.sx() - 2;
    const int ny = L.cy ? (O.sy() - 2) / 2 : O.sy() - 2;
    const int nz = L.cz ? (O.sz() - 2) / 2 : O.sz() - 2;
    for (Buf* b : {&L.q, &L.qtmp, &L.rhs, &L.res, &L.Axp, &L.Axm, &L.Ayp, &L.Aym, &L.Azp, &L.Azm,
                   &L.invAdiag, &L.Adiag})
      b->alloc(nx + 2, ny + 2, nz + 2);
    L.fbx.alloc(nx + 3, ny + 2, nz + 2);
    L.fby.alloc(nx + 2, ny + 3, nz + 2);
    L.fbz.alloc(nx + 2, ny + 2, nz + 3);
    L.idx2 = L.cx ? O.idx2 * 0.25 : O.idx2;
    L.idy2 = L.cy ? O.idy2 * 0.25 : O.idy2;
    L.idz2 = L.cz ? O.idz2 * 0.25 : O.idz2;
    g.lv.push_back(std::move(L));
    g.num_levels += 1;
  }
  // With a single level the reference's v_cycle_as_preconditioner launches
  // k_propagate_level_to_level on levels_[num_levels-2] = levels_[-1]
  // (G_GMGSolver.cu:977): undefined behaviour, so such shapes are refused.
  if (g.num_levels < 2) return -2;
  return 0;
}

// k_create_level0_coeffs / k_create_level_coeffs (G_GMGSolver.cu:499-644):
// coarse f_b(ix,iy,iz) = mean over the fine faces (2ix-1..2ix) x (2iy-1..2iy)
// x (2iz-1..2iz) of a coarsened direction (quirk: includes the mid-cell face).
void coarsen_face(const Arr& fine, Arr& coarse, bool cx, bool cy, bool cz) {
  const int rx = cx ? 2 : 1, ry = cy ? 2 : 1, rz = cz ? 2 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < coarse.sz - 1; ++iz)
    for (int iy = 1; iy < coarse.sy - 1; ++iy)
      for (int ix = 1; ix < coarse.sx - 1; ++ix) {
        const int IX = cx ? 2 * ix - 1 : ix, IY = cy ? 2 * iy - 1 : iy, IZ = cz ? 2 * iz - 1 : iz;
        double count = 0., tmp = 0.;
        for (int kz = 0; kz < rz; ++kz)
          for (int ky = 0; ky < ry; ++ky)
            for (int kx = 0; kx < rx; ++kx) {
              tmp += fine(IX + kx, IY + ky, IZ + kz);
              count += 1.0;
            }
        coarse(ix, iy, iz) = tmp / count;
      }
}

// k_create_level_A (G_GMGSolver.cu:646-685)
void level_build_A(Level& L) {
  const Arr &fbx = L.fbx.a, &fby = L.fby.a, &fbz = L.fbz.a;
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < L.sz() - 1; ++iz)
    for (int iy = 1; iy < L.sy() - 1; ++iy)
      for (int ix = 1; ix < L.sx() - 1; ++ix) {
        const double axp = fbx(ix + 1, iy, iz) * L.idx2;
        const double axm = fbx(ix, iy, iz) * L.idx2;
        const double ayp = fby(ix, iy + 1, iz) * L.idy2;
        const double aym = fby(ix, iy, iz) * L.idy2;
        const double azp = fbz(ix, iy, iz + 1) * L.idz2;
        const double azm = fbz(ix, iy, iz) * L.idz2;
        L.Axp.a(ix, iy, iz) = axp; L.Axm.a(ix, iy, iz) = axm;
        L.Ayp.a(ix, iy, iz) = ayp; L.Aym.a(ix, iy, iz) = aym;
        L.Azp.a(ix, iy, iz) = azp; L.Azm.a(ix, iy, iz) = azm;
        const double ad = (axp + axm + ayp + aym + azp + azm);
        L.Adiag.a(ix, iy, iz) = ad;
        L.invAdiag.a(ix, iy, iz) = (std::fabs(ad) < kEPS) ? 0. : 1. / ad;
      }
}

// G_GMGSolver::create_coeffs (G_GMGSolver.cu:913-922)
void gmg_create_coeffs(GMG& g, const Grid& grid) {
  Level& L0 = g.lv[0];
  coarsen_face(grid.fbx, L0.fbx.a, L0.cx, L0.cy, L0.cz);
  coarsen_face(grid.fby, L0.fby.a, L0.cx, L0.cy, L0.cz);
  coarsen_face(grid.fbz, L0.fbz.a, L0.cx, L0.cy, L0.cz);
  level_build_A(L0);
  for (int l = 1; l < g.num_levels; ++l) {
    Level& L = g.lv[l];
    coarsen_face(g.lv[l - 1].fbx.a, L.fbx.a, L.cx, L.cy, L.cz);
    coarsen_face(g.lv[l - 1].fby.a, L.fby.a, L.cx, L.cy, L.cz);
    coarsen_face(g.lv[l - 1].fbz.a, L.fbz.a, L.cx, L.cy, L.cz);
    level_build_A(L);
  }
}

// One omega-Jacobi sweep over the interior of an (sx,sy,sz) array
// (k_jacobi_iteration_general / k_jacobi_level_iteration, G_GMGSolver.cu:692-746).
void jacobi_sweep(const Arr& Axp, const Arr& Axm, const Arr& Ayp, const Arr& Aym, const Arr& Azp,
                  const Arr& Azm, const Arr& invAdiag, const Arr& p, const Arr& rhs, Arr& ptmp,
                  double omega) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < p.sz - 1; ++iz)
    for (int iy = 1; iy < p.sy - 1; ++iy)
      for (int ix = 1; ix < p.sx - 1; ++ix) {
        const double tmp_p = Axp(ix, iy, iz) * p(ix + 1, iy, iz) + Axm(ix, iy, iz) * p(ix - 1, iy, iz) +
                             Ayp(ix, iy, iz) * p(ix, iy + 1, iz) + Aym(ix, iy, iz) * p(ix, iy - 1, iz) +
                             Azp(ix, iy, iz) * p(ix, iy, iz + 1) + Azm(ix, iy, iz) * p(ix, iy, iz - 1);
        ptmp(ix, iy, iz) = (1.0 - omega) * p(ix, iy, iz) + omega * (tmp_p + rhs(ix, iy, iz)) * invAdiag(ix, iy, iz);
      }
}

// residue = rhs - A q on the interior (k_get_res_general / k_get_res_levels,
// G_GMGSolver.cu:152-226)
void residual(const Arr& Axp, const Arr& Axm, const Arr& Ayp, const Arr& Aym, const Arr& Azp,
              const Arr& Azm, const Arr& Adiag, const Arr& q, const Arr& rhs, Arr& res) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < q.sz - 1; ++iz)
    for (int iy = 1; iy < q.sy - 1; ++iy)
      for (int ix = 1; ix < q.sx - 1; ++ix) {
        const double Ap = q(ix, iy, iz) * Adiag(ix, iy, iz) -
                          (Axp(ix, iy, iz) * q(ix + 1, iy, iz) + Axm(ix, iy, iz) * q(ix - 1, iy, iz) +
                           Ayp(ix, iy, iz) * q(ix, iy + 1, iz) + Aym(ix, iy, iz) * q(ix, iy - 1, iz) +
                           Azp(ix, iy, iz) * q(ix, iy, iz + 1) + Azm(ix, iy, iz) * q(ix, iy, iz - 1));
        res(ix, iy, iz) = rhs(ix, iy, iz) - Ap;
      }
}

// coarse_rhs = mean of children (k_restrict_grid_to_level0 /
// k_restrict_level_to_level, G_GMGSolver.cu:416-493)
void restrict_avg(const Arr& res, Arr& crhs, bool cx, bool cy, bool cz) {
  const int rx = cx ? 2 : 1, ry = cy ? 2 : 1, rz = cz ? 2 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < crhs.sz - 1; ++iz)
    for (int iy = 1; iy < crhs.sy - 1; ++iy)
      for (int ix = 1; ix < crhs.sx - 1; ++ix) {
        const int IX = cx ? 2 * ix - 1 : ix, IY = cy ? 2 * iy - 1 : iy, IZ = cz ? 2 * iz - 1 : iz;
        double count = 0., tmp = 0.;
        for (int kz = 0; kz < rz; ++kz)
          for (int ky = 0; ky < ry; ++ky)
            for (int kx = 0; kx < rx; ++kx) {
              tmp += res(IX + kx, IY + ky, IZ + kz);
              count += 1.0;
            }
        crhs(ix, iy, iz) = tmp / count;
      }
}

// fine += coarse on the children (k_propagate_*, G_GMGSolver.cu:285-389)
void prolong_inject(const Arr& cq, Arr& fq, bool cx, bool cy, bool cz) {
  const int rx = cx ? 2 : 1, ry = cy ? 2 : 1, rz = cz ? 2 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < cq.sz - 1; ++iz)
    for (int iy = 1; iy < cq.sy - 1; ++iy)
      for (int ix = 1; ix < cq.sx - 1; ++ix) {
        const int IX = cx ? 2 * ix - 1 : ix, IY = cy ? 2 * iy - 1 : iy, IZ = cz ? 2 * iz - 1 : iz;
        const double prop = cq(ix, iy, iz);
        for (int kz = 0; kz < rz; ++kz)
          for (int ky = 0; ky < ry; ++ky)
            for (int kx = 0; kx < rx; ++kx) fq(IX + kx, IY + ky, IZ + kz) += prop;
      }
}

void zero(Arr& a) { std::fill(a.d, a.d + a.size(), 0.0); }

// G_GMGSolver::v_cycle_as_preconditioner (G_GMGSolver.cu:925-998).
// q is overwritten with V(rhs), x0 = 0.  The host-side pointer swaps of the
// reference are reproduced with local buffer swaps (even sweep counts).
void gmg_vcycle(GMG& g, Grid& grid, Arr& q, const Arr& rhs) {
  const int nf = g.num_iter_fine, nc = g.num_iter_coarse, NL = g.num_levels;
  zero(q);
  for (int l = 0; l < NL; ++l) zero(g.lv[l].q.a);
  Arr a = q, b = grid.ptmp.a;  // ptmp ghosts stay 0
  for (int it = 0; it < nf; ++it) {
    jacobi_sweep(grid.Axp.a, grid.Axm.a, grid.Ayp.a, grid.Aym.a, grid.Azp.a, grid.Azm.a, grid.invAdiag.a,
                 a, rhs, b, g.omega);
    std::swap(a, b);
  }
  // after an even number of sweeps the current iterate lives in q again;
  // grid.res plays the role of grid.residue_
  residual(grid.Axp.a, grid.Axm.a, grid.Ayp.a, grid.Aym.a, grid.Azp.a, grid.Azm.a, grid.Adiag.a, a, rhs,
           grid.res.a);
  restrict_avg(grid.res.a, g.lv[0].rhs.a, g.lv[0].cx, g.lv[0].cy, g.lv[0].cz);

  auto level_sweeps = [&](Level& L, int n) {
    Arr x = L.q.a, y = L.qtmp.a;
    for (int it = 0; it < n; ++it) {
      jacobi_sweep(L.Axp.a, L.Axm.a, L.Ayp.a, L.Aym.a, L.Azp.a, L.Azm.a, L.invAdiag.a, x, L.rhs.a, y, g.omega);
      std::swap(x, y);
    }
    if (n % 2) {  // keep the iterate in L.q (reference sweep counts are even)
      std::swap(L.q.v, L.qtmp.v);
      L.q.a.d = L.q.v.data();
      L.qtmp.a.d = L.qtmp.v.data();
    }
  };

  for (int l = 0; l < NL - 1; ++l) {
    Level& L = g.lv[l];
    level_sweeps(L, nf);
    residual(L.Axp.a, L.Axm.a, L.Ayp.a, L.Aym.a, L.Azp.a, L.Azm.a, L.Adiag.a, L.q.a, L.rhs.a, L.res.a);
    Level& C = g.lv[l + 1];
    restrict_avg(L.res.a, C.rhs.a, C.cx, C.cy, C.cz);
  }
  level_sweeps(g.lv[NL - 1], nc);
  if (NL >= 2) {
    Level& C = g.lv[NL - 1];
    prolong_inject(C.q.a, g.lv[NL - 2].q.a, C.cx, C.cy, C.cz);
  }
  for (int l = NL - 2; l >= 0; --l) {
    Level& L = g.lv[l];
    level_sweeps(L, nf);
    if (l != 0) {
      prolong_inject(L.q.a, g.lv[l - 1].q.a, L.cx, L.cy, L.cz);
    } else {
      prolong_inject(L.q.a, a, L.cx, L.cy, L.cz);
    }
  }
  for (int it = 0; it < nf; ++it) {
    jacobi_sweep(grid.Axp.a, grid.Axm.a, grid.Ayp.a, grid.Aym.a, grid.Azp.a, grid.Azm.a, grid.invAdiag.a,
                 a, rhs, b, g.omega);
    std::swap(a, b);
  }
  if (a.d != q.d) std::memcpy(q.d, a.d, q.size() * sizeof(double));
}

// ---------------------------------------------------------------------------
// Interior reductions over a cell array: the reference copies the N^3
// interior to pcg_tmp_ and calls cub::DeviceReduce::Sum / Max.
double interior_sum(const Grid& g, const Arr& a) {
  const int Ny = g.Ny, Nz = g.Nz, Nx = g.Nx;
  return det_sum_rows(Ny * Nz, [&](int r) {
    const int iy = r % Ny + 1, iz = r / Ny + 1;
    double s = 0.0;
    for (int ix = 1; ix <= Nx; ++ix) s += a(ix, iy, iz);
    return s;
  });
}
double interior_dot(const Grid& g, const Arr& a, const Arr& b) {
  const int Ny = g.Ny, Nz = g.Nz, Nx = g.Nx;
  return det_sum_rows(Ny * Nz, [&](int r) {
    const int iy = r % Ny + 1, iz = r / Ny + 1;
    double s = 0.0;
    for (int ix = 1; ix <= Nx; ++ix) s += a(ix, iy, iz) * b(ix, iy, iz);
    return s;
  });
}
double interior_maxabs(const Grid& g, const Arr& a) {
  const int Ny = g.Ny, Nz = g.Nz, Nx = g.Nx;
  return det_max_rows(Ny * Nz, [&](int r) {
    const int iy = r % Ny + 1, iz = r / Ny + 1;
    double m = 0.0;
    for (int ix = 1; ix <= Nx; ++ix) m = std::max(m, std::fabs(a(ix, iy, iz)));
    return m;
  });
}

// G_PressureSolverBase::subtract_cell_mean (G_PressureSolverBase.cu:142-155):
// mean over the N^3 interior, subtracted from every (N+2)^3 entry.
void subtract_cell_mean(const Grid& g, Arr& p) {
  const double sum = interior_sum(g, p);
  const double size_inv = 1. / (double)((size_t)g.Nx * g.Ny * g.Nz);
  const double a = -1. * size_inv;
  const size_t n = p.size();
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) p.d[i] += a * sum;
}

// k_build_vof_poisson_A (G_PCGSolver.cu:126-212)
void build_A(Grid& g) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz <= g.Nz; ++iz)
    for (int iy = 1; iy <= g.Ny; ++iy)
      for (int ix = 1; ix <= g.Nx; ++ix) {
        if (g.ct(ix, iy, iz) != C_INTERIOR) {
          g.Axp.a(ix, iy, iz) = 0.; g.Axm.a(ix, iy, iz) = 0.;
          g.Ayp.a(ix, iy, iz) = 0.; g.Aym.a(ix, iy, iz) = 0.;
          g.Azp.a(ix, iy, iz) = 0.; g.Azm.a(ix, iy, iz) = 0.;
          g.Adiag.a(ix, iy, iz) = 0.; g.invAdiag.a(ix, iy, iz) = 0.;
          continue;
        }
        double axp = g.fbx(ix + 1, iy, iz) * g.inv_dx2;
        double axm = g.fbx(ix, iy, iz) * g.inv_dx2;
        double ayp = g.fby(ix, iy + 1, iz) * g.inv_dy2;
        double aym = g.fby(ix, iy, iz) * g.inv_dy2;
        double azp = g.fbz(ix, iy, iz + 1) * g.inv_dz2;
        double azm = g.fbz(ix, iy, iz) * g.inv_dz2;
        const double ad = (axp + axm + ayp + aym + azp + azm);
        g.Adiag.a(ix, iy, iz) = ad;
        g.invAdiag.a(ix, iy, iz) = 1. / ad;
        if (g.fxt(ix + 1, iy, iz) == F_BOUNDARY) axp = 0.;
        if (g.fxt(ix, iy, iz) == F_BOUNDARY) axm = 0.;
        if (g.fyt(ix, iy + 1, iz) == F_BOUNDARY) ayp = 0.;
        if (g.fyt(ix, iy, iz) == F_BOUNDARY) aym = 0.;
        if (g.fzt(ix, iy, iz + 1) == F_BOUNDARY) azp = 0.;
        if (g.fzt(ix, iy, iz) == F_BOUNDARY) azm = 0.;
        g.Axp.a(ix, iy, iz) = axp; g.Axm.a(ix, iy, iz) = axm;
        g.Ayp.a(ix, iy, iz) = ayp; g.Aym.a(ix, iy, iz) = aym;
        g.Azp.a(ix, iy, iz) = azp; g.Azm.a(ix, iy, iz) = azm;
      }
}

// Ap = A p on the interior (k_build_vof_poisson_Ap, G_PCGSolver.cu:214-245;
// the same expression as k_make_pAp :87-124).
void apply_A(const Grid& g, const Arr& p, Arr& out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz <= g.Nz; ++iz)
    for (int iy = 1; iy <= g.Ny; ++iy)
      for (int ix = 1; ix <= g.Nx; ++ix) {
        out(ix, iy, iz) =
            g.Adiag.a(ix, iy, iz) * p(ix, iy, iz) -
            (g.Axp.a(ix, iy, iz) * p(ix + 1, iy, iz) + g.Axm.a(ix, iy, iz) * p(ix - 1, iy, iz) +
             g.Ayp.a(ix, iy, iz) * p(ix, iy + 1, iz) + g.Aym.a(ix, iy, iz) * p(ix, iy - 1, iz) +
             g.Azp.a(ix, iy, iz) * p(ix, iy, iz + 1) + g.Azm.a(ix, iy, iz) * p(ix, iy, iz - 1));
      }
}

}  // namespace

// ===========================================================================
// C ABI (ctypes).  All arrays are in the reference layout described above.
extern "C" {

struct orc_stats {
  int iterations;        // PCG iterations, counted like the reference's print (G_PCGSolver.cu:921)
  int converged;         // 1 if the stopping test passed before max_iter
  double norm_b;         // sqrt(sum b^2) of the de-meaned rhs (guarded like :814-817)
  double res_max;        // max |r| (recursive residual) at exit
  double res_rel;        // ||r||_2 / norm_b (recursive) at exit
  double true_res_rel;   // ||b - A p||_2 / norm_b at exit (b de-meaned for pure Neumann)
  int num_levels;        // multigrid levels built (0 for Jacobi PCG)
  int status;            // 0 ok, -1 odd size (reference abort()), -2 single level (reference UB)
};

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// SMACSolver::set_face_type (CFD/SMACSolver.cpp:104-202): all-wall box.
void orc_set_face_type(int Nx, int Ny, int Nz, uint8_t* fxt, uint8_t* fyt, uint8_t* fzt) {
  View<uint8_t> X{fxt, Nx + 3, Ny + 2, Nz + 2}, Y{fyt, Nx + 2, Ny + 3, Nz + 2}, Z{fzt, Nx + 2, Ny + 2, Nz + 3};
  std::memset(fxt, F_GHOST, (size_t)(Nx + 3) * (Ny + 2) * (Nz + 2));
  std::memset(fyt, F_GHOST, (size_t)(Nx + 2) * (Ny + 3) * (Nz + 2));
  std::memset(fzt, F_GHOST, (size_t)(Nx + 2) * (Ny + 2) * (Nz + 3));
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx + 1; ++ix) X(ix, iy, iz) = F_INTERIOR;
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy) { X(1, iy, iz) = F_BOUNDARY; X(Nx + 1, iy, iz) = F_BOUNDARY; }
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny + 1; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) Y(ix, iy, iz) = F_INTERIOR;
  for (int iz = 1; iz <= Nz; ++iz)
    for (int ix = 1; ix <= Nx; ++ix) { Y(ix, 1, iz) = F_BOUNDARY; Y(ix, Ny + 1, iz) = F_BOUNDARY; }
  for (int iz = 1; iz <= Nz + 1; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) Z(ix, iy, iz) = F_INTERIOR;
  for (int iy = 1; iy <= Ny; ++iy)
    for (int ix = 1; ix <= Nx; ++ix) { Z(ix, iy, 1) = F_BOUNDARY; Z(ix, iy, Nz + 1) = F_BOUNDARY; }
}

// SMACSolver::set_cell_type (CFD/SMACSolver.cpp:206-248): ghosts C_GHOST,
// every real cell C_INTERIOR (the near-boundary tag is disabled at :240-241).
void orc_set_cell_type(int Nx, int Ny, int Nz, uint8_t* ct) {
  View<uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  std::memset(ct, C_GHOST, (size_t)(Nx + 2) * (Ny + 2) * (Nz + 2));
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) C(ix, iy, iz) = C_INTERIOR;
}

// Solid fraction by 8^3 sub-sampling (k_get_solid_fraction,
// CFD/G_SMACSolver_IBM.cu:94-147, constants :13-17) with a sphere predicate in
// place of the reference's z-aligned cylinder (:28-37).  spheres: n x 4
// (xc, yc, zc, r).  Cells ix,iy,iz in 1..N+1 like the reference kernel.
// Cells entirely inside or outside every sphere (by a margin far above the
// rounding of the sample coordinates) are classified without sampling; all
// others are sampled exactly as the reference does.
void orc_solid_fraction_spheres(int Nx, int Ny, int Nz, double dx, double dy, double dz, double ox,
                                double oy, double oz, const double* sph, int nsph, double* sf) {
  Arr S{sf, Nx + 2, Ny + 2, Nz + 2};
  const int N8 = 8;
  const double fact = 1. / (double)N8;
  const double inv_total = 1. / (double)(N8 * N8 * N8);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy)
      for (int ix = 1; ix < Nx + 2; ++ix) {
        const double xc = dx * (double)(ix)-0.5 * dx + ox;  // StaggeredGrid::get_cell_coord :136-138
        const double yc = dy * (double)(iy)-0.5 * dy + oy;
        const double zc = dz * (double)(iz)-0.5 * dz + oz;
        const double xini = xc - dx * 0.5, yini = yc - dy * 0.5, zini = zc - dz * 0.5;
        const double sdx = dx * fact, sdy = dy * fact, sdz = dz * fact;
        int numpts = 0;
        for (int s = 0; s < nsph; ++s) {
          const double cx = sph[4 * s], cy = sph[4 * s + 1], cz = sph[4 * s + 2], r = sph[4 * s + 3];
          const double rsq = r * r;
          // nearest / farthest distance from the sphere centre to the cell box
          const double lx = xini, hx = xini + dx, ly = yini, hy = yini + dy, lz = zini, hz = zini + dz;
          const double nx_ = std::max(0.0, std::max(lx - cx, cx - hx));
          const double ny_ = std::max(0.0, std::max(ly - cy, cy - hy));
          const double nz_ = std::max(0.0, std::max(lz - cz, cz - hz));
          const double fx = std::max(std::fabs(lx - cx), std::fabs(hx - cx));
          const double fy = std::max(std::fabs(ly - cy), std::fabs(hy - cy));
          const double fz = std::max(std::fabs(lz - cz), std::fabs(hz - cz));
          const double near2 = nx_ * nx_ + ny_ * ny_ + nz_ * nz_;
          const double far2 = fx * fx + fy * fy + fz * fz;
          const double margin = 1e-6 * (dx * dx + dy * dy + dz * dz);
          if (near2 > rsq + margin) continue;
          if (far2 < rsq - margin) { numpts += N8 * N8 * N8; continue; }
          for (int kz = 0; kz < N8; ++kz)
            for (int ky = 0; ky < N8; ++ky)
              for (int kx = 0; kx < N8; ++kx) {
                const double x_pt = xini + sdx * (kx + 0.5);
                const double y_pt = yini + sdy * (ky + 0.5);
                const double z_pt = zini + sdz * (kz + 0.5);
                const double ddx = x_pt - cx, ddy = y_pt - cy, ddz = z_pt - cz;
                if (ddx * ddx + ddy * ddy + ddz * ddz <= rsq) numpts += 1;
              }
        }
        double solidfraction = (double)numpts * inv_total;
        if (solidfraction > 1. - 1.e-2) solidfraction = 1.0;  // clip, :137-139
        S(ix, iy, iz) = solidfraction;
      }
}

// k_set_solid_cell_from_ibm (CFD/G_SMACSolver_IBM.cu:763-792).
void orc_set_solid_cells(int Nx, int Ny, int Nz, const double* sf, uint8_t* ct, uint8_t* fxt, uint8_t* fyt,
                         uint8_t* fzt) {
  View<const double> S{sf, Nx + 2, Ny + 2, Nz + 2};
  View<uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  View<uint8_t> X{fxt, Nx + 3, Ny + 2, Nz + 2}, Y{fyt, Nx + 2, Ny + 3, Nz + 2}, Z{fzt, Nx + 2, Ny + 2, Nz + 3};
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy)
      for (int ix = 1; ix < Nx + 2; ++ix)
        if (S(ix, iy, iz) > 1. - kEPS) {
          C(ix, iy, iz) = C_SOLID;
          X(ix, iy, iz) = F_BOUNDARY; X(ix + 1, iy, iz) = F_BOUNDARY;
          Y(ix, iy, iz) = F_BOUNDARY; Y(ix, iy + 1, iz) = F_BOUNDARY;
          Z(ix, iy, iz) = F_BOUNDARY; Z(ix, iy, iz + 1) = F_BOUNDARY;
        }
}

// Face coefficients from the volume fraction:
// k_update_cell_properties_by_alpha (CFD/G_SMACSolver_VoF.cu:1374-1407) then
// k_update_{x,y,z}_face_properties_by_alpha (:1409-1535):
// rho = (1-a) rho0 + a rho1 on C_INTERIOR/C_NEAR_BOUNDARY cells;
// f_b = f_inv_rho = 1/(0.5(rho_L+rho_R)) on F_INTERIOR faces, 0 elsewhere.
// rho must hold valid values on non-fluid cells on entry (only F_INTERIOR
// faces read it, and those touch fluid cells only).
// Pressure in solid and ghost cells after a projection, the pressure part of
// G_SMACSolver::update_boundary_ghost (CFD/G_SMACSolver.cu:1144-1267):
//  1. a C_SOLID cell takes p of its first C_INTERIOR neighbour in the order
//     x-, x+, y-, y+, z-, z+, shifted hydrostatically by rho g h (0 without
//     such a neighbour);
//  2. every ghost cell (an index 0 or N+1) takes p of the nearest interior
//     cell (indices clamped to 1..N), shifted by rho(src) g.r.
// The reference's first kernel also writes the ghost cells, racing at edges
// and corners; its second kernel overwrites all of them, so this final
// state is the reference's.
void orc_pressure_ghost(int Nx, int Ny, int Nz, double dx, double dy, double dz, double gx, double gy, double gz,
                        const uint8_t* ct, const double* rho, double* p) {
  View<const uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  View<const double> R{rho, Nx + 2, Ny + 2, Nz + 2};
  Arr P{p, Nx + 2, Ny + 2, Nz + 2};
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        if (C(ix, iy, iz) != C_SOLID) continue;
        double v;
        if (C(ix - 1, iy, iz) == C_INTERIOR) v = P(ix - 1, iy, iz) + R(ix - 1, iy, iz) * gx * dx;
        else if (C(ix + 1, iy, iz) == C_INTERIOR) v = P(ix + 1, iy, iz) - R(ix + 1, iy, iz) * gx * dx;
        else if (C(ix, iy - 1, iz) == C_INTERIOR) v = P(ix, iy - 1, iz) + R(ix, iy - 1, iz) * gy * dy;
        else if (C(ix, iy + 1, iz) == C_INTERIOR) v = P(ix, iy + 1, iz) - R(ix, iy + 1, iz) * gy * dy;
        else if (C(ix, iy, iz - 1) == C_INTERIOR) v = P(ix, iy, iz - 1) + R(ix, iy, iz - 1) * gz * dz;
        else if (C(ix, iy, iz + 1) == C_INTERIOR) v = P(ix, iy, iz + 1) - R(ix, iy, iz + 1) * gz * dz;
        else v = 0.;
        P(ix, iy, iz) = v;
      }
  for (int iz = 0; iz < Nz + 2; ++iz)
    for (int iy = 0; iy < Ny + 2; ++iy)
      for (int ix = 0; ix < Nx + 2; ++ix) {
        const bool ghost = ix == 0 || ix == Nx + 1 || iy == 0 || iy == Ny + 1 || iz == 0 || iz == Nz + 1;
        if (!ghost) continue;
        const int sx = ix == 0 ? 1 : ix == Nx + 1 ? Nx : ix;
        const int sy = iy == 0 ? 1 : iy == Ny + 1 ? Ny : iy;
        const int sz = iz == 0 ? 1 : iz == Nz + 1 ? Nz : iz;
        const double rx = (double)(ix - sx) * dx, ry = (double)(iy - sy) * dy, rz = (double)(iz - sz) * dz;
        P(ix, iy, iz) = P(sx, sy, sz) + R(sx, sy, sz) * (rx * gx + ry * gy + rz * gz);
      }
}

// Face pressure gradient, G_SMACSolver::make_face_gradp
// (CFD/G_SMACSolver.cu:1277-1343): g_x(ix) = (p(ix) - p(ix-1)) / dx on faces
// 1..N+1 of each family (rows and planes 1..N+1 as the reference's threads).
void orc_face_gradp(int Nx, int Ny, int Nz, double dx, double dy, double dz, const double* p, double* gpx,
                    double* gpy, double* gpz) {
  View<const double> P{p, Nx + 2, Ny + 2, Nz + 2};
  Arr GX{gpx, Nx + 3, Ny + 2, Nz + 2}, GY{gpy, Nx + 2, Ny + 3, Nz + 2}, GZ{gpz, Nx + 2, Ny + 2, Nz + 3};
  const double ix_ = 1. / dx, iy_ = 1. / dy, iz_ = 1. / dz;
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy)
      for (int ix = 1; ix < Nx + 2; ++ix) {
        GX(ix, iy, iz) = (P(ix, iy, iz) - P(ix - 1, iy, iz)) * ix_;
        GY(ix, iy, iz) = (P(ix, iy, iz) - P(ix, iy - 1, iz)) * iy_;
        GZ(ix, iy, iz) = (P(ix, iy, iz) - P(ix, iy, iz - 1)) * iz_;
      }
}

// Velocity on outlet faces, k_update_v{x,y,z}_outlet
// (CFD/G_BoundaryFunctions.cu:143-255), run by update_boundary_ghost: a face
// with the outlet mark m (1: interior side +1, 2: interior side -1) gets
//   v = v* + sign f_b dt p_delta(interior cell) / h,  sign = +1 for m = 2, -1 for m = 1,
// for face indices 1..N+1 on all three axes (the reference's thread range).
// Other mark values, and marks whose interior cell index would pass N+1
// (where the reference reads the next row), are left alone.
void orc_velocity_outlet(int Nx, int Ny, int Nz, double dx, double dy, double dz, double dt, const uint8_t* fxo,
                         const uint8_t* fyo, const uint8_t* fzo, const double* vxs, const double* vys,
                         const double* vzs, const double* fbx, const double* fby, const double* fbz,
                         const double* pd, double* vx, double* vy, double* vz) {
  View<const uint8_t> MX{fxo, Nx + 3, Ny + 2, Nz + 2}, MY{fyo, Nx + 2, Ny + 3, Nz + 2}, MZ{fzo, Nx + 2, Ny + 2, Nz + 3};
  View<const double> SX{vxs, Nx + 3, Ny + 2, Nz + 2}, SY{vys, Nx + 2, Ny + 3, Nz + 2}, SZ{vzs, Nx + 2, Ny + 2, Nz + 3};
  View<const double> BX{fbx, Nx + 3, Ny + 2, Nz + 2}, BY{fby, Nx + 2, Ny + 3, Nz + 2}, BZ{fbz, Nx + 2, Ny + 2, Nz + 3};
  View<const double> P{pd, Nx + 2, Ny + 2, Nz + 2};
  Arr VX{vx, Nx + 3, Ny + 2, Nz + 2}, VY{vy, Nx + 2, Ny + 3, Nz + 2}, VZ{vz, Nx + 2, Ny + 2, Nz + 3};
  const double ix_ = 1. / dx, iy_ = 1. / dy, iz_ = 1. / dz;
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy)
      for (int ix = 1; ix < Nx + 2; ++ix) {
        if (const uint8_t m = MX(ix, iy, iz); (m == 1 || m == 2) && ix + (m == 1) <= Nx + 1) {
          const int s = m == 1 ? 1 : -1;
          const double sign = s < 0 ? 1. : -1.;
          VX(ix, iy, iz) = SX(ix, iy, iz) + sign * BX(ix, iy, iz) * dt * P(ix + s, iy, iz) * ix_;
        }
        if (const uint8_t m = MY(ix, iy, iz); (m == 1 || m == 2) && iy + (m == 1) <= Ny + 1) {
          const int s = m == 1 ? 1 : -1;
          const double sign = s < 0 ? 1. : -1.;
          VY(ix, iy, iz) = SY(ix, iy, iz) + sign * BY(ix, iy, iz) * dt * P(ix, iy + s, iz) * iy_;
        }
        if (const uint8_t m = MZ(ix, iy, iz); (m == 1 || m == 2) && iz + (m == 1) <= Nz + 1) {
          const int s = m == 1 ? 1 : -1;
          const double sign = s < 0 ? 1. : -1.;
          VZ(ix, iy, iz) = SZ(ix, iy, iz) + sign * BZ(ix, iy, iz) * dt * P(ix, iy, iz + s) * iz_;
        }
      }
}

}  // extern "C"

namespace {

// d_get_velocity_ghost_value (CFD/G_BoundaryFunctions.cu:258-275); boundary
// types from CFD/Enums.h:10-16.
double ghost_value(uint8_t type, double vb, double lam, double bnd, double inner) {
  if (type == 2) return 2.0 * (1.0 - lam) * vb - inner;  // BC_INFLOW
  if (type == 0) return -inner;                          // BC_NOSLIP
  if (type == 4) return 2.0 * bnd - inner;               // BC_OUTLET
  if (type == 1) return inner;                           // BC_SLIP
  return bnd;                                            // BC_OUTFLOW
}

// One face family: normal axis a, ghosts across the two other axes b < c.
// k_update_v*_ghost then k_update_v*_ghost_corner
// (CFD/G_BoundaryFunctions.cu:277-560).
void velocity_ghost_family(const int N[3], int a, const uint8_t* bct, const double* bvel, const uint8_t* bcid,
                           const double* lam, double* v) {
  int S[3] = {N[0] + 2, N[1] + 2, N[2] + 2};
  S[a] += 1;
  auto at = [&](const int i[3]) { return ((size_t)i[2] * S[1] + i[1]) * S[0] + i[0]; };
  const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
  int i[3];
  for (int ia = 1; ia < N[a] + 2; ++ia) {
    i[a] = ia;
    // edges of the b-c ring, corners excluded
    for (int side = 0; side < 4; ++side) {
      const int g = side < 2 ? b : c, o = side < 2 ? c : b;  // ghost axis, other axis
      const bool low = (side & 1) == 0;
      for (int io = 1; io <= N[o]; ++io) {
        i[o] = io;
        int ib[3] = {i[0], i[1], i[2]}, in[3] = {i[0], i[1], i[2]};
        ib[g] = low ? 1 : N[g];
        in[g] = low ? 2 : N[g] - 1;
        i[g] = low ? 0 : N[g] + 1;
        const int id = bcid[at(ib)];
        v[at(i)] = ghost_value(bct[id], bvel[id], lam ? lam[at(ib)] : 0., v[at(ib)], v[at(in)]);
      }
    }
    // corners: the mean of the two neighbouring ghost values
    for (int cb = 0; cb < 2; ++cb)
      for (int cc = 0; cc < 2; ++cc) {
        i[b] = cb ? N[b] + 1 : 0;
        i[c] = cc ? N[c] + 1 : 0;
        int j1[3] = {i[0], i[1], i[2]}, j2[3] = {i[0], i[1], i[2]};
        j1[c] = cc ? N[c] : 1;  // ghost across b, inner along c
        j2[b] = cb ? N[b] : 1;  // ghost across c, inner along b
        v[at(i)] = 0.5 * (v[at(j1)] + v[at(j2)]);
      }
  }
}

}  // namespace

extern "C" {

// Ghost velocities of update_boundary_ghost (k_update_v*_ghost and
// k_update_v*_ghost_corner, CFD/G_BoundaryFunctions.cu:277-560): ghost faces
// across the two tangential axes take the boundary rule of the bc id of the
// first face inside; corners take the mean of their two ghost neighbours.
// bct/bvx/bvy/bvz: the boundary table (bc_.bcType_, bc_.v*_); lam* may be
// NULL (no IBM area fractions).
void orc_velocity_ghost(int Nx, int Ny, int Nz, const uint8_t* bct, const double* bvx, const double* bvy,
                        const double* bvz, const uint8_t* fxbcid, const uint8_t* fybcid, const uint8_t* fzbcid,
                        const double* lamx, const double* lamy, const double* lamz, double* vx, double* vy,
                        double* vz) {
  const int N[3] = {Nx, Ny, Nz};
  velocity_ghost_family(N, 0, bct, bvx, fxbcid, lamx, vx);
  velocity_ghost_family(N, 1, bct, bvy, fybcid, lamy, vy);
  velocity_ghost_family(N, 2, bct, bvz, fzbcid, lamz, vz);
}

// Wall-face u*, G_SMACSolver::update_vstar_boundary
// (CFD/G_SMACSolver.cu:1044-1052 -> k_update_v{x,y,z}star_boundary,
// CFD/G_BoundaryFunctions.cu:3-71, rules d_get_v*star_*face,
// CFD/G_BoundaryFunctions.h:369-470): on every F_BOUNDARY face with indices
// 1..N+1, by the type of its boundary id: inflow (1 - lam) v_b, no-slip 0,
// outlet the u* of the next face on the side given by the outlet mark
// (2: -1, otherwise +1, the reference's f_*internal_id_ < 0 test), others 0.
// Families in the order x, y, z, faces in index order (an outlet face whose
// neighbour is itself F_BOUNDARY is a race in the reference).
void orc_vstar_boundary(int Nx, int Ny, int Nz, const uint8_t* bct, const double* bvx, const double* bvy,
                        const double* bvz, const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt,
                        const uint8_t* fxbcid, const uint8_t* fybcid, const uint8_t* fzbcid, const uint8_t* fxo,
                        const uint8_t* fyo, const uint8_t* fzo, const double* lamx, const double* lamy,
                        const double* lamz, double* vxs, double* vys, double* vzs) {
  const int N[3] = {Nx, Ny, Nz};
  const uint8_t* ft[3] = {fxt, fyt, fzt};
  const uint8_t* id[3] = {fxbcid, fybcid, fzbcid};
  const uint8_t* mk[3] = {fxo, fyo, fzo};
  const double* lam[3] = {lamx, lamy, lamz};
  const double* bv[3] = {bvx, bvy, bvz};
  double* vs[3] = {vxs, vys, vzs};
  for (int a = 0; a < 3; ++a) {
    int S[3] = {Nx + 2, Ny + 2, Nz + 2};
    S[a] += 1;
    const size_t stride = a == 0 ? 1 : a == 1 ? (size_t)S[0] : (size_t)S[0] * S[1];
    for (int iz = 1; iz < N[2] + 2; ++iz)
      for (int iy = 1; iy < N[1] + 2; ++iy)
        for (int ix = 1; ix < N[0] + 2; ++ix) {
          const size_t f = ((size_t)iz * S[1] + iy) * S[0] + ix;
          if (ft[a][f] != F_BOUNDARY) continue;
          const int b = id[a][f];
          const uint8_t t = bct[b];
          double v = 0.;
          if (t == 2) {  // BC_INFLOW
            v = (1. - (lam[a] ? lam[a][f] : 0.)) * bv[a][b];
          } else if (t == 4) {  // BC_OUTLET
            const bool low = mk[a] && mk[a][f] == 2;
            v = low ? vs[a][f - stride] : vs[a][f + stride];
          }
          vs[a][f] = v;
        }
  }
}

// Surface-tension face force, G_SMACSolver::calc_surface_tension
// (CFD/G_SMACSolver_VoF.cu:435-445): the three reference kernels in order.
//  1. k_calc_interface_normal (:87-182): on C_INTERIOR cells, grad alpha by
//     central differences (one-sided next to non-interior cells, 0 with no
//     interior neighbour on either side), |grad| into gm, n = grad / |grad|
//     (0 when |grad|^2 <= 1e-12).  Other cells keep n and gm.
//  2. k_calc_curvature (:184-290): on cells 1..N, kappa = 0 where alpha >
//     0.99 or < 0.01, else -div n by the same differences, a neighbour
//     counting only if C_INTERIOR with gm > 1e-6.
//  3. k_calc_surface_tension_face (:292-433): f_s = 0 everywhere, then on
//     faces 2..N along their axis (1..N across) between two C_INTERIOR cells
//     f_s = sigma kappa_f (alpha_R - alpha_L) / h, kappa_f the mean of the
//     two cells' kappa where both have 0.01 < alpha < 0.99, the one that
//     has, or 0.
// nx/ny/nz/gm/kappa are in-out cell arrays (the grid's nx_, ny_, nz_, p_tmp_
// and kappa_), f_s three face arrays.
void orc_surface_tension(int Nx, int Ny, int Nz, double dx, double dy, double dz, const double* alpha,
                         const uint8_t* ct, double sigma, double* nx, double* ny, double* nz, double* kappa,
                         double* gm, double* fsx, double* fsy, double* fsz) {
  View<const double> A{alpha, Nx + 2, Ny + 2, Nz + 2};
  View<const uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  Arr NX{nx, Nx + 2, Ny + 2, Nz + 2}, NY{ny, Nx + 2, Ny + 2, Nz + 2}, NZ{nz, Nx + 2, Ny + 2, Nz + 2};
  Arr K{kappa, Nx + 2, Ny + 2, Nz + 2}, G{gm, Nx + 2, Ny + 2, Nz + 2};
  Arr FX{fsx, Nx + 3, Ny + 2, Nz + 2}, FY{fsy, Nx + 2, Ny + 3, Nz + 2}, FZ{fsz, Nx + 2, Ny + 2, Nz + 3};
  const double idx = 1. / dx, idy = 1. / dy, idz = 1. / dz;
  const double i2dx = 1. / (2. * dx), i2dy = 1. / (2. * dy), i2dz = 1. / (2. * dz);
  // difference of f along one axis from the two neighbours' flags
  auto diff = [](bool p, bool m, double fp, double f0, double fm, double i2h, double ih) {
    if (p && m) return (fp - fm) * i2h;
    if (p) return (fp - f0) * ih;
    if (m) return (f0 - fm) * ih;
    return 0.0;
  };
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        if (C(ix, iy, iz) != C_INTERIOR) continue;
        const double gx = diff(C(ix + 1, iy, iz) == C_INTERIOR, C(ix - 1, iy, iz) == C_INTERIOR, A(ix + 1, iy, iz),
                               A(ix, iy, iz), A(ix - 1, iy, iz), i2dx, idx);
        const double gy = diff(C(ix, iy + 1, iz) == C_INTERIOR, C(ix, iy - 1, iz) == C_INTERIOR, A(ix, iy + 1, iz),
                               A(ix, iy, iz), A(ix, iy - 1, iz), i2dy, idy);
        const double gz = diff(C(ix, iy, iz + 1) == C_INTERIOR, C(ix, iy, iz - 1) == C_INTERIOR, A(ix, iy, iz + 1),
                               A(ix, iy, iz), A(ix, iy, iz - 1), i2dz, idz);
        const double mag2 = gx * gx + gy * gy + gz * gz;
        const double mag = std::sqrt(mag2);
        G(ix, iy, iz) = mag;
        if (mag2 > 1e-12) {
          const double inv = 1. / mag;
          NX(ix, iy, iz) = gx * inv;
          NY(ix, iy, iz) = gy * inv;
          NZ(ix, iy, iz) = gz * inv;
        } else {
          NX(ix, iy, iz) = 0.;
          NY(ix, iy, iz) = 0.;
          NZ(ix, iy, iz) = 0.;
        }
      }
  const double th = 1e-6;
  auto ok = [&](int x, int y, int z) { return C(x, y, z) == C_INTERIOR && G(x, y, z) > th; };
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        const double a = A(ix, iy, iz);
        if (a > 0.99 || a < 0.01) {
          K(ix, iy, iz) = 0.;
          continue;
        }
        const double dnx = diff(ok(ix + 1, iy, iz), ok(ix - 1, iy, iz), NX(ix + 1, iy, iz), NX(ix, iy, iz),
                                NX(ix - 1, iy, iz), i2dx, idx);
        const double dny = diff(ok(ix, iy + 1, iz), ok(ix, iy - 1, iz), NY(ix, iy + 1, iz), NY(ix, iy, iz),
                                NY(ix, iy - 1, iz), i2dy, idy);
        const double dnz = diff(ok(ix, iy, iz + 1), ok(ix, iy, iz - 1), NZ(ix, iy, iz + 1), NZ(ix, iy, iz),
                                NZ(ix, iy, iz - 1), i2dz, idz);
        K(ix, iy, iz) = -1.0 * (dnx + dny + dnz);
      }
  std::fill(fsx, fsx + FX.size(), 0.0);
  std::fill(fsy, fsy + FY.size(), 0.0);
  std::fill(fsz, fsz + FZ.size(), 0.0);
  auto valid = [&](int x, int y, int z) { return A(x, y, z) > 1e-2 && A(x, y, z) < 1 - 1e-2; };
  auto kface = [&](int x, int y, int z, int xm, int ym, int zm) {
    const bool vp = valid(x, y, z), vm = valid(xm, ym, zm);
    if (vp && vm) return 0.5 * (K(x, y, z) + K(xm, ym, zm));
    if (vp) return K(x, y, z);
    if (vm) return K(xm, ym, zm);
    return 0.0;
  };
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        const bool c0 = C(ix, iy, iz) == C_INTERIOR;
        if (ix >= 2)
          FX(ix, iy, iz) = c0 && C(ix - 1, iy, iz) == C_INTERIOR
                               ? sigma * kface(ix, iy, iz, ix - 1, iy, iz) * (A(ix, iy, iz) - A(ix - 1, iy, iz)) * idx
                               : 0.0;
        if (iy >= 2)
          FY(ix, iy, iz) = c0 && C(ix, iy - 1, iz) == C_INTERIOR
                               ? sigma * kface(ix, iy, iz, ix, iy - 1, iz) * (A(ix, iy, iz) - A(ix, iy - 1, iz)) * idy
                               : 0.0;
        if (iz >= 2)
          FZ(ix, iy, iz) = c0 && C(ix, iy, iz - 1) == C_INTERIOR
                               ? sigma * kface(ix, iy, iz, ix, iy, iz - 1) * (A(ix, iy, iz) - A(ix, iy, iz - 1)) * idz
                               : 0.0;
      }
}

}  // extern "C"

namespace {

// The fields of the momentum predictor, per family a = x, y, z where a field
// lives on faces.  Cells are (Nx+2)(Ny+2)(Nz+2), family-a faces have one
// more entry along a.
struct MomFields {
  int N[3];
  const uint8_t* bct;      // boundary types per id
  const double* bv[3];     // boundary velocity components per id
  const uint8_t* ft[3];    // face types
  const uint8_t* id[3];    // boundary ids
  const double* lam[3];    // IBM area fractions (nullptr: 0)
  const double* v[3];      // velocity at time n
  const double* mf[3];     // advecting face velocities
  const double* muf[3];    // face viscosities
  const double* mu;        // cell viscosity
  const double* rho_old;   // cell density at time n
  const double* p;         // cell pressure
  const double* fb[3];     // 1/rho on faces
  const double* imp[3];    // coupling impulse (nullptr: 0)
  const double* sf[3];     // IBM solid fraction of the face (nullptr: 0)
  const double* eps_old;   // two-way form only (nullptr: the one-way form)
  const double* eps_new;
};

struct Idx3 {
  int i[3];
};

inline size_t face_off(const MomFields& F, int a, const Idx3& q) {
  const size_t S0 = F.N[0] + 2 + (a == 0), S1 = F.N[1] + 2 + (a == 1);
  return ((size_t)q.i[2] * S1 + q.i[1]) * S0 + q.i[0];
}
inline size_t cell_off(const MomFields& F, const Idx3& q) {
  return ((size_t)q.i[2] * (F.N[1] + 2) + q.i[1]) * (F.N[0] + 2) + q.i[0];
}
inline Idx3 shifted(Idx3 q, int axis, int s) {
  q.i[axis] += s;
  return q;
}

// d_get_v{b}_{b}face (CFD/G_BoundaryFunctions.h:9-98): velocity of family b
// at face q, boundary faces by their type.  The x-face rule passes the
// stored value through for outlets only, the y and z rules also for slip.
double face_val(const MomFields& F, int b, const Idx3& q) {
  const size_t f = face_off(F, b, q);
  const uint8_t t = F.ft[b][f];
  if (t == F_INTERIOR) return F.v[b][f];
  if (t == F_BOUNDARY) {
    const int bid = F.id[b][f];
    const uint8_t bt = F.bct[bid];
    if (bt == 2) return (1. - (F.lam[b] ? F.lam[b][f] : 0.)) * F.bv[b][bid];  // BC_INFLOW
    if (bt == 0) return 0.;                                                  // BC_NOSLIP
    if (bt == 4 || (b != 0 && bt == 1)) return F.v[b][f];                    // BC_OUTLET (and BC_SLIP for y, z)
  }
  return 0.;
}

// d_get_v{a}_{d}dir (CFD/G_BoundaryFunctions.h:100-367): velocity of family
// a next to face q along axis d != a on side s; a non-interior neighbour is
// mirrored about the wall (the mean velocity of the one or two family-d
// boundary faces there), or copied for slip and outlet walls.
double dir_val(const MomFields& F, int a, int d, const Idx3& q, int s) {
  const double inside = F.v[a][face_off(F, a, q)];
  const Idx3 q2 = shifted(q, d, s);
  if (F.ft[a][face_off(F, a, q2)] == F_INTERIOR) return F.v[a][face_off(F, a, q2)];
  const Idx3 qf = s > 0 ? shifted(q, d, 1) : q;
  const Idx3 qg = shifted(qf, a, -1);
  double wall = 0.;
  int count = 0;
  const size_t ff = face_off(F, d, qf), fg = face_off(F, d, qg);
  if (F.ft[d][ff] == F_BOUNDARY) {
    wall += F.bv[a][F.id[d][ff]];
    count++;
  }
  if (F.ft[d][fg] == F_BOUNDARY) {
    wall += F.bv[a][F.id[d][fg]];
    count++;
  }
  if (count > 0) wall /= (double)count;
  const uint8_t bt = F.bct[F.id[d][ff]];
  if (bt == 1 || bt == 4) return inside;  // BC_SLIP, BC_OUTLET
  return 2.0 * wall - inside;
}

double minmod(double dp, double dm) {  // d_minmod, CFD/G_SMACSolver.cu:67-88
  if (dp * dm > 0.) return std::fabs(dp) < std::fabs(dm) ? dp : dm;
  return 0.;
}
double sgn1(double x) { return x < 0 ? -1. : 1.; }  // sgn, CFD/G_SMACSolver.h:130-139

// Two-way form: eps_old averaged over the four cells around the edge on side
// s along axis d of the family-a face q (its cells cm, c and their
// neighbours along d), added in ascending index order as the reference
// writes them (CFD/G_SMACSolver.cu:1610-1622, 1832-1844, 2050-2062).
double eps_edge(const MomFields& F, int a, int d, const Idx3& q, int s) {
  const Idx3 lc = s > 0 ? q : shifted(q, d, -1), lcm = shifted(lc, a, -1);
  const Idx3 hc = shifted(lc, d, 1), hcm = shifted(lcm, d, 1);
  const double* e = F.eps_old;
  const double sum = d > a ? e[cell_off(F, lcm)] + e[cell_off(F, lc)] + e[cell_off(F, hcm)] + e[cell_off(F, hc)]
                           : e[cell_off(F, lcm)] + e[cell_off(F, hcm)] + e[cell_off(F, lc)] + e[cell_off(F, hc)];
  return 0.25 * sum;
}

// u* of the F_INTERIOR face q of family a: k_get_vof_vstar_rhouu_consistent_{x,y,z}
// (CFD/G_SMACSolver.cu:90-1012) with the family's axis as a parameter, or
// with F.eps_old set the two-way form k_get_vof_vstar_rhouu_consistent_*_two_way
// (:1538-2194).
double vstar_face(const MomFields& F, int a, const Idx3& q, const double ih[3], const double ih2[3], double dt,
                  double g) {
  const double v0 = F.v[a][face_off(F, a, q)];
  const double vp = face_val(F, a, shifted(q, a, 1)), vm = face_val(F, a, shifted(q, a, -1));
  double vdp[3] = {0, 0, 0}, vdm[3] = {0, 0, 0};
  for (int d = 0; d < 3; ++d)
    if (d != a) {
      vdp[d] = dir_val(F, a, d, q, +1);
      vdm[d] = dir_val(F, a, d, q, -1);
    }
  // viscous: the own axis, then the other two in axis order
  const Idx3 cm = shifted(q, a, -1);
  const double tau_p = F.mu[cell_off(F, q)] * (vp - v0);
  const double tau_m = F.mu[cell_off(F, cm)] * (v0 - vm);
  const bool tw = F.eps_old != nullptr;
  double tmp = tw ? 2. * (F.eps_old[cell_off(F, q)] * tau_p - F.eps_old[cell_off(F, cm)] * tau_m) * ih2[a]
                  : 2. * (tau_p - tau_m) * ih2[a];
  for (int d = 0; d < 3; ++d) {
    if (d == a) continue;
    const Idx3 qd = shifted(q, d, 1), qda = shifted(qd, a, -1);
    const double wp0 = face_val(F, d, qd), wpm = face_val(F, d, qda);
    const double w0 = face_val(F, d, q), wm = face_val(F, d, cm);
    const double mup = 0.5 * (F.muf[d][face_off(F, d, qd)] + F.muf[d][face_off(F, d, qda)]);
    const double tp = mup * ((wp0 - wpm) * ih[a] + (vdp[d] - v0) * ih[d]);
    const double mum = 0.5 * (F.muf[d][face_off(F, d, q)] + F.muf[d][face_off(F, d, cm)]);
    const double tm = mum * ((w0 - wm) * ih[a] + (v0 - vdm[d]) * ih[d]);
    if (tw)
      tmp += (eps_edge(F, a, d, q, +1) * tp - eps_edge(F, a, d, q, -1) * tm) * ih[d];
    else
      tmp += (tp - tm) * ih[d];
  }
  // convection, MUSCL with minmod, in axis order
  for (int d = 0; d < 3; ++d) {
    double fp, fm;
    if (d == a) {
      fp = 0.5 * (F.mf[a][face_off(F, a, q)] + F.mf[a][face_off(F, a, shifted(q, a, 1))]);
      fm = 0.5 * (F.mf[a][face_off(F, a, cm)] + F.mf[a][face_off(F, a, q)]);
    } else {
      const Idx3 qd = shifted(q, d, 1);
      fp = 0.5 * (F.mf[d][face_off(F, d, shifted(qd, a, -1))] + F.mf[d][face_off(F, d, qd)]);
      fm = 0.5 * (F.mf[d][face_off(F, d, q)] + F.mf[d][face_off(F, d, cm)]);
    }
    const double nplus = d == a ? vp : vdp[d], nminus = d == a ? vm : vdm[d];
    auto reconstruct = [&](double flux, const Idx3& up, double upwind_v) {
      if (F.ft[a][face_off(F, a, up)] != F_INTERIOR) return upwind_v;
      const double vu = F.v[a][face_off(F, a, up)];
      const double np = d == a ? face_val(F, a, shifted(up, a, 1)) : dir_val(F, a, d, up, +1);
      const double nm = d == a ? face_val(F, a, shifted(up, a, -1)) : dir_val(F, a, d, up, -1);
      const double su = minmod(np - vu, vu - nm);
      const int dir = (int)sgn1(flux);
      return upwind_v + dir * 0.5 * su;
    };
    const double up_p = reconstruct(fp, fp > 0. ? q : shifted(q, d, 1), fp > 0. ? v0 : nplus);
    const double up_m = reconstruct(fm, fm > 0. ? shifted(q, d, -1) : q, fm > 0. ? nminus : v0);
    const double Mp = fp * up_p, Mm = fm * up_m;
    tmp -= (Mp - Mm) * ih[d];
  }
  const size_t f = face_off(F, a, q);
  const double inv_rho = F.fb[a][f];
  const double rho_old_f = 0.5 * (F.rho_old[cell_off(F, q)] + F.rho_old[cell_off(F, cm)]);
  const double inv_volume = ih[0] * ih[1] * ih[2];
  const double coupling = (F.imp[a] ? F.imp[a][f] : 0.) * inv_volume;
  double vs;
  if (tw) {
    const double eo = 0.5 * (F.eps_old[cell_off(F, cm)] + F.eps_old[cell_off(F, q)]);
    const double en = 0.5 * (F.eps_new[cell_off(F, cm)] + F.eps_new[cell_off(F, q)]);
    tmp -= eo * (F.p[cell_off(F, q)] - F.p[cell_off(F, cm)]) * ih[a];
    const double inv_eps_rho = inv_rho / en;
    vs = inv_eps_rho * (eo * rho_old_f * v0 + dt * tmp + coupling) + dt * g;
  } else {
    tmp -= (F.p[cell_off(F, q)] - F.p[cell_off(F, cm)]) * ih[a];
    vs = inv_rho * (v0 * rho_old_f + coupling) + dt * (inv_rho * tmp + g);
  }
  vs = (1.0 - (F.sf[a] ? F.sf[a][f] : 0.)) * vs;
  return vs;
}

}  // namespace

extern "C" {

// The momentum predictor u*, G_SMACSolver::get_vof_vstar_rhouu_consistent
// (CFD/G_SMACSolver.cu:1062-1070): on every F_INTERIOR face with indices
// 1..N+1, u* = (1/rho)(rho_old u + impulse/V) + dt((1/rho)(viscous -
// convection - grad p) + g), scaled by 1 - IBM solid fraction.  Families in
// the order x, y, z (independent: each reads only time-n fields).  Arrays
// per family in the argument triples; lam/imp/sf may be NULL (0).
// The advecting mass flux, G_SMACSolver::compute_mass_flux_from_alpha_flux
// (CFD/G_SMACSolver_VoF.cu:1708-1795): on every face of family a,
// mf = rho0 q + (rho1 - rho0) F_accum (h_a / dt), q = face_val.  With
// eps_half given, the two-way form (:2472-2687): q = eps_f q on faces
// 1..N+1 along a (eps_f the mean of eps_half of the face's two cells; at
// faces 1 and N+1 the one interior cell's), mf = 0 at faces 0 and N+2.
void orc_mass_flux(int Nx, int Ny, int Nz, double dx, double dy, double dz, double dt, double rho0, double rho1,
                   const uint8_t* bct, const double* bvx, const double* bvy, const double* bvz,
                   const uint8_t* const* ft, const uint8_t* const* id, const double* const* lam,
                   const double* const* v, const double* const* Fa, const double* eps_half, double* const* mf) {
  MomFields F{};
  F.N[0] = Nx; F.N[1] = Ny; F.N[2] = Nz;
  F.bct = bct;
  F.bv[0] = bvx; F.bv[1] = bvy; F.bv[2] = bvz;
  for (int a = 0; a < 3; ++a) {
    F.ft[a] = ft[a]; F.id[a] = id[a]; F.lam[a] = lam[a]; F.v[a] = v[a];
  }
  const double inv_dt = 1. / dt, h[3] = {dx, dy, dz}, drho = rho1 - rho0;
  for (int a = 0; a < 3; ++a) {
    const double hdt = h[a] * inv_dt;
    const int ex = Nx + 1 + (a == 0), ey = Ny + 1 + (a == 1), ez = Nz + 1 + (a == 2);
    for (int z = 0; z <= ez; ++z)
      for (int y = 0; y <= ey; ++y)
        for (int x = 0; x <= ex; ++x) {
          const Idx3 q{{x, y, z}};
          const size_t f = face_off(F, a, q);
          double u = face_val(F, a, q);
          if (eps_half) {
            const int along = q.i[a], n = F.N[a];
            if (along < 1 || along > n + 1) {
              mf[a][f] = 0.0;
              continue;
            }
            const double e = along == 1       ? eps_half[cell_off(F, q)]
                             : along == n + 1 ? eps_half[cell_off(F, shifted(q, a, -1))]
                                              : 0.5 * (eps_half[cell_off(F, shifted(q, a, -1))] + eps_half[cell_off(F, q)]);
            u = e * u;
          }
          mf[a][f] = rho0 * u + drho * (Fa[a][f] * hdt);
        }
  }
}

// With eps_old and eps_new given (not NULL): the two-way form,
// G_SMACSolver::get_vof_vstar_rhouu_consistent_two_way (:2196-2203), with fb
// the faces' f_inv_rho.
void orc_predict_vstar2(int Nx, int Ny, int Nz, double dx, double dy, double dz, double dt, double gx, double gy,
                        double gz, const uint8_t* bct, const double* bvx, const double* bvy, const double* bvz,
                        const uint8_t* const* ft, const uint8_t* const* id, const double* const* lam,
                        const double* const* v, const double* const* mf, const double* const* muf, const double* mu,
                        const double* rho_old, const double* p, const double* const* fb, const double* const* imp,
                        const double* const* sf, const double* eps_old, const double* eps_new, double* const* vs) {
  MomFields F;
  F.eps_old = eps_old;
  F.eps_new = eps_new;
  F.N[0] = Nx; F.N[1] = Ny; F.N[2] = Nz;
  F.bct = bct;
  F.bv[0] = bvx; F.bv[1] = bvy; F.bv[2] = bvz;
  for (int a = 0; a < 3; ++a) {
    F.ft[a] = ft[a]; F.id[a] = id[a]; F.lam[a] = lam[a]; F.v[a] = v[a]; F.mf[a] = mf[a]; F.muf[a] = muf[a];
    F.fb[a] = fb[a]; F.imp[a] = imp[a]; F.sf[a] = sf[a];
  }
  F.mu = mu; F.rho_old = rho_old; F.p = p;
  const double h[3] = {dx, dy, dz};
  double ih[3], ih2[3];
  for (int a = 0; a < 3; ++a) {
    ih[a] = 1. / h[a];
    ih2[a] = 1. / (h[a] * h[a]);
  }
  const double g[3] = {gx, gy, gz};
  for (int a = 0; a < 3; ++a)
    for (int iz = 1; iz <= Nz + 1; ++iz)
      for (int iy = 1; iy <= Ny + 1; ++iy)
        for (int ix = 1; ix <= Nx + 1; ++ix) {
          const Idx3 q{{ix, iy, iz}};
          const size_t f = face_off(F, a, q);
          if (F.ft[a][f] != F_INTERIOR) continue;
          vs[a][f] = vstar_face(F, a, q, ih, ih2, dt, g[a]);
        }
}

void orc_predict_vstar(int Nx, int Ny, int Nz, double dx, double dy, double dz, double dt, double gx, double gy,
                       double gz, const uint8_t* bct, const double* bvx, const double* bvy, const double* bvz,
                       const uint8_t* const* ft, const uint8_t* const* id, const double* const* lam,
                       const double* const* v, const double* const* mf, const double* const* muf, const double* mu,
                       const double* rho_old, const double* p, const double* const* fb, const double* const* imp,
                       const double* const* sf, double* const* vs) {
  orc_predict_vstar2(Nx, Ny, Nz, dx, dy, dz, dt, gx, gy, gz, bct, bvx, bvy, bvz, ft, id, lam, v, mf, muf, mu, rho_old,
                     p, fb, imp, sf, nullptr, nullptr, vs);
}

// The two-way Poisson coefficients, G_CFDDEMCoupling::update_poisson_beta_two_way
// (Coupling/G_CFDDEMCoupling.cu:419-460): f_b = (eps_L + eps_R)/2 * f_inv_rho
// on x-faces 1..Nx+1 x 1..Ny x 1..Nz, y-faces 1..Nx x 1..Ny+1 x 1..Nz, z-faces
// 1..Nx x 1..Ny x 1..Nz+1.
void orc_poisson_beta_two_way(int Nx, int Ny, int Nz, const double* eps, const double* const* fir,
                              double* const* fb) {
  const long long sx = Nx + 2, sxy = sx * (Ny + 2);
  for (int a = 0; a < 3; ++a) {
    const long long S0 = Nx + 2 + (a == 0), S1 = Ny + 2 + (a == 1);
    const long long step = a == 0 ? 1 : a == 1 ? sx : sxy;
    const int ex = Nx + (a == 0), ey = Ny + (a == 1), ez = Nz + (a == 2);
    for (int z = 1; z <= ez; ++z)
      for (int y = 1; y <= ey; ++y)
        for (int x = 1; x <= ex; ++x) {
          const long long c = z * sxy + y * sx + x, f = ((long long)z * S1 + y) * S0 + x;
          const double epsf = 0.5 * (eps[c - step] + eps[c]);
          fb[a][f] = epsf * fir[a][f];
        }
  }
}

// The property update, G_SMACSolver::update_properties_by_alpha
// (CFD/G_SMACSolver_VoF.cu:1543-1566), after its swap of rho_ and rho_old_
// (which the caller does by swapping arrays):
//  1. k_update_cell_properties_by_alpha (:1374-1407): on C_INTERIOR and
//     C_NEAR_BOUNDARY cells with indices 1..N+1, rho = (1-a) rho0 + a rho1,
//     inv_rho = 1/rho, mu = (1-a) mu0 + a mu1;
//  2. k_update_cell_boundary_properties_by_alpha + k_update_cell_ghost_properties
//     (:1241-1372), final state: a C_SOLID interior cell takes rho and mu of
//     its first C_INTERIOR neighbour (x-, x+, y-, y+, z-, z+; 0 without
//     one), every ghost cell those of the nearest interior cell;
//  3. k_update_{x,y,z}_face_properties_by_alpha (:1409-1535): on F_INTERIOR
//     faces rho_f = (rho_L + rho_R)/2, f_b = f_inv_rho = 1/rho_f,
//     mu_f = (mu_L + mu_R)/2; on the other faces (indices 1..N+2 along, 1..N+1
//     across) f_b = f_inv_rho = 0, rho_f and mu_f untouched.
// inv_rho, fir*, frho* may be NULL (not written).
void orc_update_properties(int Nx, int Ny, int Nz, double rho0, double rho1, double mu0, double mu1,
                           const double* alpha, const uint8_t* ct, const uint8_t* const* ft, double* rho,
                           double* inv_rho, double* mu, double* const* fb, double* const* fir, double* const* frho,
                           double* const* fmu) {
  View<const double> A{alpha, Nx + 2, Ny + 2, Nz + 2};
  View<const uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  Arr R{rho, Nx + 2, Ny + 2, Nz + 2}, M{mu, Nx + 2, Ny + 2, Nz + 2};
  for (int iz = 1; iz <= Nz + 1; ++iz)
    for (int iy = 1; iy <= Ny + 1; ++iy)
      for (int ix = 1; ix <= Nx + 1; ++ix) {
        const uint8_t t = C(ix, iy, iz);
        if (t != C_INTERIOR && t != C_NEAR_BOUNDARY) continue;
        const double a = A(ix, iy, iz);
        R(ix, iy, iz) = (1. - a) * rho0 + a * rho1;
        if (inv_rho) inv_rho[((size_t)iz * (Ny + 2) + iy) * (Nx + 2) + ix] = 1. / R(ix, iy, iz);
        M(ix, iy, iz) = (1. - a) * mu0 + a * mu1;
      }
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        if (C(ix, iy, iz) != C_SOLID) continue;
        const int nb[6][3] = {{ix - 1, iy, iz}, {ix + 1, iy, iz}, {ix, iy - 1, iz},
                              {ix, iy + 1, iz}, {ix, iy, iz - 1}, {ix, iy, iz + 1}};
        double r = 0., m = 0.;
        for (const auto& q : nb)
          if (C(q[0], q[1], q[2]) == C_INTERIOR) {
            r = R(q[0], q[1], q[2]);
            m = M(q[0], q[1], q[2]);
            break;
          }
        R(ix, iy, iz) = r;
        M(ix, iy, iz) = m;
      }
  for (int iz = 0; iz < Nz + 2; ++iz)
    for (int iy = 0; iy < Ny + 2; ++iy)
      for (int ix = 0; ix < Nx + 2; ++ix) {
        if (!(ix == 0 || ix == Nx + 1 || iy == 0 || iy == Ny + 1 || iz == 0 || iz == Nz + 1)) continue;
        const int sx = ix == 0 ? 1 : ix == Nx + 1 ? Nx : ix;
        const int sy = iy == 0 ? 1 : iy == Ny + 1 ? Ny : iy;
        const int sz = iz == 0 ? 1 : iz == Nz + 1 ? Nz : iz;
        R(ix, iy, iz) = R(sx, sy, sz);
        M(ix, iy, iz) = M(sx, sy, sz);
      }
  const int N[3] = {Nx, Ny, Nz};
  for (int a = 0; a < 3; ++a) {
    int S[3] = {Nx + 2, Ny + 2, Nz + 2};
    S[a] += 1;
    for (int iz = 1; iz <= Nz + 1 + (a == 2); ++iz)
      for (int iy = 1; iy <= Ny + 1 + (a == 1); ++iy)
        for (int ix = 1; ix <= Nx + 1 + (a == 0); ++ix) {
          const size_t f = ((size_t)iz * S[1] + iy) * S[0] + ix;
          if (ft[a][f] != F_INTERIOR) {
            fb[a][f] = 0.;
            if (fir[a]) fir[a][f] = 0.;
            continue;
          }
          int q[3] = {ix, iy, iz};
          q[a] -= 1;
          const double fr = 0.5 * (R(ix, iy, iz) + R(q[0], q[1], q[2]));
          if (frho[a]) frho[a][f] = fr;
          fb[a][f] = 1. / fr;
          if (fir[a]) fir[a][f] = fb[a][f];
          fmu[a][f] = 0.5 * (M(ix, iy, iz) + M(q[0], q[1], q[2]));
        }
  }
  (void)N;
}

// Outlet boundary faces (G_SMACSolver::update_boundary_faces,
// CFD/G_SMACSolver_VoF.cu:1798-1950): f_b of an outlet face is twice the f_b
// of the face next to it on the interior side (p = 0 on the outlet).  The
// mark of a face gives that side: 1 -> +1 (f_xinternal_id_ >= 0), 2 -> -1;
// 0 leaves the face alone (walls are already 0 from the face assembly).
// Marked faces must have unmarked interior neighbours (outlets on domain
// sides), so the result does not depend on the update order.
void orc_update_boundary_faces(int Nx, int Ny, int Nz, const uint8_t* fxo, const uint8_t* fyo, const uint8_t* fzo,
                               double* fbx, double* fby, double* fbz) {
  View<const uint8_t> OX{fxo, Nx + 3, Ny + 2, Nz + 2}, OY{fyo, Nx + 2, Ny + 3, Nz + 2}, OZ{fzo, Nx + 2, Ny + 2, Nz + 3};
  Arr BX{fbx, Nx + 3, Ny + 2, Nz + 2}, BY{fby, Nx + 2, Ny + 3, Nz + 2}, BZ{fbz, Nx + 2, Ny + 2, Nz + 3};
  for (int iz = 0; iz < Nz + 2; ++iz)
    for (int iy = 0; iy < Ny + 2; ++iy)
      for (int ix = 0; ix < Nx + 3; ++ix) {
        const uint8_t m = OX(ix, iy, iz);
        if (m == 1 && ix + 1 < Nx + 3) BX(ix, iy, iz) = 2.0 * BX(ix + 1, iy, iz);
        if (m == 2 && ix >= 1) BX(ix, iy, iz) = 2.0 * BX(ix - 1, iy, iz);
      }
  for (int iz = 0; iz < Nz + 2; ++iz)
    for (int iy = 0; iy < Ny + 3; ++iy)
      for (int ix = 0; ix < Nx + 2; ++ix) {
        const uint8_t m = OY(ix, iy, iz);
        if (m == 1 && iy + 1 < Ny + 3) BY(ix, iy, iz) = 2.0 * BY(ix, iy + 1, iz);
        if (m == 2 && iy >= 1) BY(ix, iy, iz) = 2.0 * BY(ix, iy - 1, iz);
      }
  for (int iz = 0; iz < Nz + 3; ++iz)
    for (int iy = 0; iy < Ny + 2; ++iy)
      for (int ix = 0; ix < Nx + 2; ++ix) {
        const uint8_t m = OZ(ix, iy, iz);
        if (m == 1 && iz + 1 < Nz + 3) BZ(ix, iy, iz) = 2.0 * BZ(ix, iy, iz + 1);
        if (m == 2 && iz >= 1) BZ(ix, iy, iz) = 2.0 * BZ(ix, iy, iz - 1);
      }
}

void orc_face_coeffs_vof(int Nx, int Ny, int Nz, const double* alpha, double rho0, double rho1,
                         const uint8_t* ct, const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt,
                         double* rho, double* fbx, double* fby, double* fbz, double* firx, double* firy,
                         double* firz) {
  View<const double> A{alpha, Nx + 2, Ny + 2, Nz + 2};
  View<const uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  View<const uint8_t> X{fxt, Nx + 3, Ny + 2, Nz + 2}, Y{fyt, Nx + 2, Ny + 3, Nz + 2}, Z{fzt, Nx + 2, Ny + 2, Nz + 3};
  Arr R{rho, Nx + 2, Ny + 2, Nz + 2};
  Arr BX{fbx, Nx + 3, Ny + 2, Nz + 2}, BY{fby, Nx + 2, Ny + 3, Nz + 2}, BZ{fbz, Nx + 2, Ny + 2, Nz + 3};
  Arr IX{firx, Nx + 3, Ny + 2, Nz + 2}, IY{firy, Nx + 2, Ny + 3, Nz + 2}, IZ{firz, Nx + 2, Ny + 2, Nz + 3};
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy)
      for (int ix = 1; ix < Nx + 2; ++ix) {
        const uint8_t c = C(ix, iy, iz);
        if (c == C_INTERIOR || c == C_NEAR_BOUNDARY) {
          const double a = A(ix, iy, iz);
          R(ix, iy, iz) = (1. - a) * rho0 + a * rho1;
        }
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy) {
      for (int ix = 1; ix < Nx + 3; ++ix) {
        if (X(ix, iy, iz) != F_INTERIOR) { BX(ix, iy, iz) = 0.; IX(ix, iy, iz) = 0.; continue; }
        const double fr = 0.5 * (R(ix, iy, iz) + R(ix - 1, iy, iz));
        BX(ix, iy, iz) = 1. / fr; IX(ix, iy, iz) = BX(ix, iy, iz);
      }
    }
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < Nz + 2; ++iz)
    for (int iy = 1; iy < Ny + 3; ++iy) {
      for (int ix = 1; ix < Nx + 2; ++ix) {
        if (Y(ix, iy, iz) != F_INTERIOR) { BY(ix, iy, iz) = 0.; IY(ix, iy, iz) = 0.; continue; }
        const double fr = 0.5 * (R(ix, iy, iz) + R(ix, iy - 1, iz));
        BY(ix, iy, iz) = 1. / fr; IY(ix, iy, iz) = BY(ix, iy, iz);
      }
    }
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < Nz + 3; ++iz)
    for (int iy = 1; iy < Ny + 2; ++iy) {
      for (int ix = 1; ix < Nx + 2; ++ix) {
        if (Z(ix, iy, iz) != F_INTERIOR) { BZ(ix, iy, iz) = 0.; IZ(ix, iy, iz) = 0.; continue; }
        const double fr = 0.5 * (R(ix, iy, iz) + R(ix, iy, iz - 1));
        BZ(ix, iy, iz) = 1. / fr; IZ(ix, iy, iz) = BZ(ix, iy, iz);
      }
    }
}

// base_k_make_poisson_rhs (CFD/pressure_solver/G_PressureSolverBase.cu:49-118)
void orc_make_rhs(int Nx, int Ny, int Nz, double inv_dx, double inv_dy, double inv_dz, double inv_dt,
                  const double* vxs, const double* vys, const double* vzs, const double* eps,
                  const double* eps_old, const double* fbx, const double* fby, const double* fbz,
                  const double* fsx, const double* fsy, const double* fsz, const uint8_t* ct, double* rhs) {
  View<const double> VX{vxs, Nx + 3, Ny + 2, Nz + 2}, VY{vys, Nx + 2, Ny + 3, Nz + 2}, VZ{vzs, Nx + 2, Ny + 2, Nz + 3};
  View<const double> E{eps, Nx + 2, Ny + 2, Nz + 2}, EO{eps_old, Nx + 2, Ny + 2, Nz + 2};
  View<const double> BX{fbx, Nx + 3, Ny + 2, Nz + 2}, BY{fby, Nx + 2, Ny + 3, Nz + 2}, BZ{fbz, Nx + 2, Ny + 2, Nz + 3};
  View<const double> SX{fsx, Nx + 3, Ny + 2, Nz + 2}, SY{fsy, Nx + 2, Ny + 3, Nz + 2}, SZ{fsz, Nx + 2, Ny + 2, Nz + 3};
  View<const uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  Arr R{rhs, Nx + 2, Ny + 2, Nz + 2};
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        if (C(ix, iy, iz) != C_INTERIOR) { R(ix, iy, iz) = 0.0; continue; }
        const double exp_ = 0.5 * (E(ix, iy, iz) + E(ix + 1, iy, iz));
        const double exm = 0.5 * (E(ix - 1, iy, iz) + E(ix, iy, iz));
        const double eyp = 0.5 * (E(ix, iy, iz) + E(ix, iy + 1, iz));
        const double eym = 0.5 * (E(ix, iy - 1, iz) + E(ix, iy, iz));
        const double ezp = 0.5 * (E(ix, iy, iz) + E(ix, iy, iz + 1));
        const double ezm = 0.5 * (E(ix, iy, iz - 1) + E(ix, iy, iz));
        const double div_eps = (exp_ * VX(ix + 1, iy, iz) - exm * VX(ix, iy, iz)) * inv_dx +
                               (eyp * VY(ix, iy + 1, iz) - eym * VY(ix, iy, iz)) * inv_dy +
                               (ezp * VZ(ix, iy, iz + 1) - ezm * VZ(ix, iy, iz)) * inv_dz;
        const double deps = E(ix, iy, iz) - EO(ix, iy, iz);
        const double f_st = (BX(ix + 1, iy, iz) * SX(ix + 1, iy, iz) - BX(ix, iy, iz) * SX(ix, iy, iz)) * inv_dx +
                            (BY(ix, iy + 1, iz) * SY(ix, iy + 1, iz) - BY(ix, iy, iz) * SY(ix, iy, iz)) * inv_dy +
                            (BZ(ix, iy, iz + 1) * SZ(ix, iy, iz + 1) - BZ(ix, iy, iz) * SZ(ix, iy, iz)) * inv_dz;
        R(ix, iy, iz) = -inv_dt * div_eps - deps * inv_dt * inv_dt - f_st;
      }
}

// k_build_vof_poisson_A exported for kernel-level parity: writes the 8
// stencil arrays (Axp,Axm,Ayp,Aym,Azp,Azm,Adiag,invAdiag), each (N+2)^3,
// interior only (entries outside the interior are left untouched).
void orc_build_A(int Nx, int Ny, int Nz, double inv_dx2, double inv_dy2, double inv_dz2, const double* fbx,
                 const double* fby, const double* fbz, const uint8_t* ct, const uint8_t* fxt, const uint8_t* fyt,
                 const uint8_t* fzt, double* A8) {
  Grid g;
  g.Nx = Nx; g.Ny = Ny; g.Nz = Nz;
  g.inv_dx2 = inv_dx2; g.inv_dy2 = inv_dy2; g.inv_dz2 = inv_dz2;
  g.ct = {ct, Nx + 2, Ny + 2, Nz + 2};
  g.fxt = {fxt, Nx + 3, Ny + 2, Nz + 2}; g.fyt = {fyt, Nx + 2, Ny + 3, Nz + 2}; g.fzt = {fzt, Nx + 2, Ny + 2, Nz + 3};
  g.fbx = {const_cast<double*>(fbx), Nx + 3, Ny + 2, Nz + 2};
  g.fby = {const_cast<double*>(fby), Nx + 2, Ny + 3, Nz + 2};
  g.fbz = {const_cast<double*>(fbz), Nx + 2, Ny + 2, Nz + 3};
  const size_t nc = (size_t)(Nx + 2) * (Ny + 2) * (Nz + 2);
  Buf* bufs[8] = {&g.Axp, &g.Axm, &g.Ayp, &g.Aym, &g.Azp, &g.Azm, &g.Adiag, &g.invAdiag};
  for (int k = 0; k < 8; ++k) {
    bufs[k]->a = {A8 + k * nc, Nx + 2, Ny + 2, Nz + 2};
  }
  build_A(g);
}

// (A p) on the interior from the 7 stencil arrays written by orc_build_A.
void orc_apply_A(int Nx, int Ny, int Nz, const double* A8, const double* p, double* out) {
  Grid g;
  g.Nx = Nx; g.Ny = Ny; g.Nz = Nz;
  const size_t nc = (size_t)(Nx + 2) * (Ny + 2) * (Nz + 2);
  Buf* bufs[8] = {&g.Axp, &g.Axm, &g.Ayp, &g.Aym, &g.Azp, &g.Azm, &g.Adiag, &g.invAdiag};
  for (int k = 0; k < 8; ++k) bufs[k]->a = {const_cast<double*>(A8) + k * nc, Nx + 2, Ny + 2, Nz + 2};
  Arr P{const_cast<double*>(p), Nx + 2, Ny + 2, Nz + 2}, O{out, Nx + 2, Ny + 2, Nz + 2};
  apply_A(g, P, O);
}

// The PCG solvers of CFD/pressure_solver/G_PCGSolver.cu, selected like
// G_PCGSolver::set_solver (:592-613):
//   PURENEUMANN_GMG_PCG  solve_pureneumann_gmgpcg  :772-922
//   GMG_PCG              solve_gmgpcg              :619-770
//   PURENEUMANN_STANDARD_PCG solve_pureneumann_pcg :307-445
//   STANDARD_PCG         solve_pcg                 :448-586
// The solve builds its own RHS (base_k_make_poisson_rhs) and operator from the
// grid fields, exactly like the reference, and updates p_delta in place.
//
// stop_rule 0: the reference's test, max|r|*dt < tol every check_freq
//              iterations (:884-903); check_freq <= 0 selects the reference's
//              frequency (5 for GMG, 10 for Jacobi PCG).
// stop_rule 1: ||r||_2 / norm_b < tol on the recursive residual, same
//              checking frequency (a relative-residual form of the same loop).
// stop_rule 2: true residual ||b - A p||_2 / norm_b < tol, every iteration.
// max_iter <= 0 selects the reference's 2000.
struct orc_problem {
  int Nx, Ny, Nz;
  double dx, dy, dz, dt;
  const double *vxs, *vys, *vzs;         // u* faces
  const double *eps, *eps_old;           // void fraction (new, old) cells
  const double *fbx, *fby, *fbz;         // face coefficients
  const double *fsx, *fsy, *fsz;         // surface-tension face force
  const uint8_t *ct, *fxt, *fyt, *fzt;   // cell and face types
};

int orc_solve(const orc_problem* P, int solver_type, double tol, int levels, int max_iter, int stop_rule,
              int check_freq, double* p_delta, double* rhs_out, orc_stats* st) {
  const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz;
  Grid g;
  g.Nx = Nx; g.Ny = Ny; g.Nz = Nz;
  g.inv_dx = 1. / P->dx; g.inv_dy = 1. / P->dy; g.inv_dz = 1. / P->dz;
  g.inv_dx2 = 1. / (P->dx * P->dx); g.inv_dy2 = 1. / (P->dy * P->dy); g.inv_dz2 = 1. / (P->dz * P->dz);
  g.ct = {P->ct, Nx + 2, Ny + 2, Nz + 2};
  g.fxt = {P->fxt, Nx + 3, Ny + 2, Nz + 2}; g.fyt = {P->fyt, Nx + 2, Ny + 3, Nz + 2}; g.fzt = {P->fzt, Nx + 2, Ny + 2, Nz + 3};
  g.fbx = {const_cast<double*>(P->fbx), Nx + 3, Ny + 2, Nz + 2};
  g.fby = {const_cast<double*>(P->fby), Nx + 2, Ny + 3, Nz + 2};
  g.fbz = {const_cast<double*>(P->fbz), Nx + 2, Ny + 2, Nz + 3};
  for (Buf* b : {&g.rhs, &g.r, &g.z, &g.dir, &g.Ap, &g.ptmp, &g.res, &g.Axp, &g.Axm, &g.Ayp, &g.Aym, &g.Azp, &g.Azm,
                 &g.Adiag, &g.invAdiag})
    b->alloc(Nx + 2, Ny + 2, Nz + 2);
  g.pd = {p_delta, Nx + 2, Ny + 2, Nz + 2};

  const bool use_gmg = (solver_type == GMG_PCG || solver_type == PURENEUMANN_GMG_PCG);
  const bool pure = (solver_type == PURENEUMANN_GMG_PCG || solver_type == PURENEUMANN_STANDARD_PCG);
  if (check_freq <= 0) check_freq = use_gmg ? 5 : 10;
  if (max_iter <= 0) max_iter = 2000;
  const double dt = P->dt;

  std::memset(st, 0, sizeof(*st));
  GMG gmg;
  if (use_gmg) {
    const int rc = gmg_initialize(gmg, g, levels);
    if (rc != 0) { st->status = rc; return rc; }
    st->num_levels = gmg.num_levels;
  }

  orc_make_rhs(Nx, Ny, Nz, g.inv_dx, g.inv_dy, g.inv_dz, 1. / dt, P->vxs, P->vys, P->vzs, P->eps, P->eps_old,
               P->fbx, P->fby, P->fbz, P->fsx, P->fsy, P->fsz, P->ct, g.rhs.a.d);
  if (rhs_out) std::memcpy(rhs_out, g.rhs.a.d, g.rhs.a.size() * sizeof(double));
  build_A(g);
  apply_A(g, g.pd, g.Ap.a);

  // mean of b over the interior (:800-804), then r = (b - mean) - Ap and the
  // norm of b (:807-817).  The non-Neumann variants skip the mean (:655).
  const double mean_b = interior_sum(g, g.rhs.a) / (double)((size_t)Nx * Ny * Nz);
  Buf bhat;  // b as the loop sees it (de-meaned for pure Neumann)
  bhat.alloc(Nx + 2, Ny + 2, Nz + 2);
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz <= Nz; ++iz)
    for (int iy = 1; iy <= Ny; ++iy)
      for (int ix = 1; ix <= Nx; ++ix) {
        const double b = pure ? g.rhs.a(ix, iy, iz) - mean_b : g.rhs.a(ix, iy, iz);
        bhat.a(ix, iy, iz) = b;
        g.r.a(ix, iy, iz) = b - g.Ap.a(ix, iy, iz);
      }
  double norm_b = interior_dot(g, bhat.a, bhat.a);
  if (norm_b < 1.0e-16) norm_b = 1.0;
  norm_b = std::sqrt(norm_b);
  st->norm_b = norm_b;

  if (pure) subtract_cell_mean(g, g.r.a);

  if (use_gmg) {
    gmg_create_coeffs(gmg, g);
    gmg_vcycle(gmg, g, g.z.a, g.r.a);
  } else {
    // z = invAdiag * r over all (N+2)^3 entries (base_k_mult_elementwise_array, :359)
    const size_t n = g.z.a.size();
    for (size_t i = 0; i < n; ++i) g.z.a.d[i] = g.invAdiag.a.d[i] * g.r.a.d[i];
  }
  if (pure) subtract_cell_mean(g, g.z.a);
  std::memcpy(g.dir.a.d, g.z.a.d, g.z.a.size() * sizeof(double));

  double rz[2];
  int rz_old = 0, rz_new = 1;
  rz[rz_old] = interior_dot(g, g.r.a, g.z.a);

  auto true_rel = [&]() {
    Buf t;
    t.alloc(Nx + 2, Ny + 2, Nz + 2);
    apply_A(g, g.pd, t.a);
    const double s = det_sum_rows(Ny * Nz, [&](int rr) {
      const int iy = rr % Ny + 1, iz = rr / Ny + 1;
      double acc = 0.0;
      for (int ix = 1; ix <= Nx; ++ix) {
        const double d = bhat.a(ix, iy, iz) - t.a(ix, iy, iz);
        acc += d * d;
      }
      return acc;
    });
    return std::sqrt(s) / norm_b;
  };

  int iter = 0;
  bool conv = false;
  for (iter = 0; iter < max_iter; ++iter) {
    apply_A(g, g.dir.a, g.Ap.a);  // k_make_pAp
    const double pAp = interior_dot(g, g.dir.a, g.Ap.a);
    const double alpha = rz[rz_old] / pAp;
    if (use_gmg) {
      // k_update_p_r (:66-85)
#pragma omp parallel for collapse(2) schedule(static)
      for (int iz = 1; iz <= Nz; ++iz)
        for (int iy = 1; iy <= Ny; ++iy)
          for (int ix = 1; ix <= Nx; ++ix) {
            g.pd(ix, iy, iz) += alpha * g.dir.a(ix, iy, iz);
            g.r.a(ix, iy, iz) -= alpha * g.Ap.a(ix, iy, iz);
          }
      if (pure) subtract_cell_mean(g, g.r.a);
      gmg_vcycle(gmg, g, g.z.a, g.r.a);
      rz[rz_new] = interior_dot(g, g.r.a, g.z.a);
    } else {
      // k_update_p_r_z_make_rz_tmp (:248-273)
#pragma omp parallel for collapse(2) schedule(static)
      for (int iz = 1; iz <= Nz; ++iz)
        for (int iy = 1; iy <= Ny; ++iy)
          for (int ix = 1; ix <= Nx; ++ix) {
            const double r_new = g.r.a(ix, iy, iz) - alpha * g.Ap.a(ix, iy, iz);
            g.pd(ix, iy, iz) += alpha * g.dir.a(ix, iy, iz);
            g.r.a(ix, iy, iz) = r_new;
            g.z.a(ix, iy, iz) = g.invAdiag.a(ix, iy, iz) * r_new;
          }
      rz[rz_new] = interior_dot(g, g.r.a, g.z.a);
    }
    bool stop = false;
    if (stop_rule == 2) {
      stop = true_rel() < tol;
    } else if (iter % check_freq == 0) {
      if (stop_rule == 0) {
        const double max_divu = interior_maxabs(g, g.r.a) * dt;
        stop = max_divu < tol;
      } else {
        stop = std::sqrt(interior_dot(g, g.r.a, g.r.a)) / norm_b < tol;
      }
    }
    if (stop) { iter++; conv = true; break; }
    // k_update_dir (:276-288)
    const double beta = rz[rz_new] / rz[rz_old];
#pragma omp parallel for collapse(2) schedule(static)
    for (int iz = 1; iz <= Nz; ++iz)
      for (int iy = 1; iy <= Ny; ++iy)
        for (int ix = 1; ix <= Nx; ++ix)
          g.dir.a(ix, iy, iz) = g.z.a(ix, iy, iz) + beta * g.dir.a(ix, iy, iz);
    std::swap(rz_old, rz_new);
  }
  st->iterations = iter;
  st->converged = conv ? 1 : 0;
  st->res_max = interior_maxabs(g, g.r.a);
  st->res_rel = std::sqrt(interior_dot(g, g.r.a, g.r.a)) / norm_b;
  st->true_res_rel = true_rel();
  return 0;
}

// k_correct_vof_velocity (CFD/G_SMACSolver.cu:1072-1142): on F_INTERIOR
// faces u = u* + f_inv_rho*dt*(f_s - grad p_delta); p += p_delta on
// C_INTERIOR cells.  Faces of other types are left untouched.
void orc_correct(int Nx, int Ny, int Nz, double inv_dx, double inv_dy, double inv_dz, double dt,
                 const uint8_t* ct, const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt,
                 const double* pd, double* p, const double* vxs, const double* vys, const double* vzs,
                 const double* firx, const double* firy, const double* firz, const double* fsx,
                 const double* fsy, const double* fsz, double* vx, double* vy, double* vz) {
  View<const uint8_t> C{ct, Nx + 2, Ny + 2, Nz + 2};
  View<const uint8_t> X{fxt, Nx + 3, Ny + 2, Nz + 2}, Y{fyt, Nx + 2, Ny + 3, Nz + 2}, Z{fzt, Nx + 2, Ny + 2, Nz + 3};
  View<const double> PD{pd, Nx + 2, Ny + 2, Nz + 2};
  Arr PN{p, Nx + 2, Ny + 2, Nz + 2};
  View<const double> VXS{vxs, Nx + 3, Ny + 2, Nz + 2}, VYS{vys, Nx + 2, Ny + 3, Nz + 2}, VZS{vzs, Nx + 2, Ny + 2, Nz + 3};
  View<const double> IRX{firx, Nx + 3, Ny + 2, Nz + 2}, IRY{firy, Nx + 2, Ny + 3, Nz + 2}, IRZ{firz, Nx + 2, Ny + 2, Nz + 3};
  View<const double> SX{fsx, Nx + 3, Ny + 2, Nz + 2}, SY{fsy, Nx + 2, Ny + 3, Nz + 2}, SZ{fsz, Nx + 2, Ny + 2, Nz + 3};
  Arr VX{vx, Nx + 3, Ny + 2, Nz + 2}, VY{vy, Nx + 2, Ny + 3, Nz + 2}, VZ{vz, Nx + 2, Ny + 2, Nz + 3};
  // the reference's thread range: ix,iy,iz from 1, bounded per face kind
#pragma omp parallel for collapse(2) schedule(static)
  for (int iz = 1; iz < Nz + 3; ++iz)
    for (int iy = 1; iy < Ny + 3; ++iy)
      for (int ix = 1; ix < Nx + 3; ++ix) {
        if (!(iy >= Ny + 2 || ix >= Nx + 3 || iz >= Nz + 2))
          if (X(ix, iy, iz) == F_INTERIOR)
            VX(ix, iy, iz) = VXS(ix, iy, iz) + IRX(ix, iy, iz) * dt *
                                                   (SX(ix, iy, iz) - (PD(ix, iy, iz) - PD(ix - 1, iy, iz)) * inv_dx);
        if (!(iy >= Ny + 3 || ix >= Nx + 2 || iz >= Nz + 2))
          if (Y(ix, iy, iz) == F_INTERIOR)
            VY(ix, iy, iz) = VYS(ix, iy, iz) + IRY(ix, iy, iz) * dt *
                                                   (SY(ix, iy, iz) - (PD(ix, iy, iz) - PD(ix, iy - 1, iz)) * inv_dy);
        if (!(iy >= Ny + 2 || ix >= Nx + 2 || iz >= Nz + 3))
          if (Z(ix, iy, iz) == F_INTERIOR)
            VZ(ix, iy, iz) = VZS(ix, iy, iz) + IRZ(ix, iy, iz) * dt *
                                                   (SZ(ix, iy, iz) - (PD(ix, iy, iz) - PD(ix, iy, iz - 1)) * inv_dz);
        if (ix < Nx + 1 && iy < Ny + 1 && iz < Nz + 1)
          if (C(ix, iy, iz) == C_INTERIOR) PN(ix, iy, iz) += PD(ix, iy, iz);
      }
}

}  // extern "C"
