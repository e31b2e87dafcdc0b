// ref_io.cpp -- a small driver of ours that runs the REFERENCE's own VTI
// writer, FileInOut::output_vti_binary_cellData (CFD/FileInOut.cpp:144-262),
// compiled unmodified from its source for the host (oracle/Makefile, target
// `ref`).  TEST INFRASTRUCTURE ONLY: the file it writes is the byte-for-byte
// target of this repository's VTI output.  Host code: it runs without a GPU.
#include <cstring>

#include "FileInOut.h"

namespace {

void view(MyArray<double, 3>& a, double* data, int sx, int sy, int sz) {
  a.data_ = data;
  a.sizex_ = sx;
  a.sizey_ = sy;
  a.sizez_ = sz;
  a.size_ = sx * sy * sz;
}

}  // namespace

extern "C" {

// Writes <outdir>/result_<step>.vti from cell arrays p, alpha, ibm_sf
// ((Nx+2)(Ny+2)(Nz+2)) and face arrays vx, vy, vz (reference layout).
// Returns 0, or -1 if the output directory cannot be used.
int ref_write_vti(int Nx, int Ny, int Nz, double dx, double dy, double dz, double ox, double oy, double oz,
                  double* p, double* alpha, double* vx, double* vy, double* vz, double* ibm_sf, const char* outdir,
                  int step) {
  FileInOut io;
  if (io.solver_output_init(outdir) != 0) return -1;
  StaggeredGrid g;
  g.Nx_ = Nx; g.Ny_ = Ny; g.Nz_ = Nz;
  g.dx_ = dx; g.dy_ = dy; g.dz_ = dz;
  g.origin_x_ = ox; g.origin_y_ = oy; g.origin_z_ = oz;
  view(g.p_, p, Nx + 2, Ny + 2, Nz + 2);
  view(g.alpha_, alpha, Nx + 2, Ny + 2, Nz + 2);
  view(g.ibm_solid_fraction_, ibm_sf, Nx + 2, Ny + 2, Nz + 2);
  view(g.f_vx_, vx, Nx + 3, Ny + 2, Nz + 2);
  view(g.f_vy_, vy, Nx + 2, Ny + 3, Nz + 2);
  view(g.f_vz_, vz, Nx + 2, Ny + 2, Nz + 3);
  io.output_vti_binary_cellData(g, step);
  return 0;
}

}  // extern "C"
