// ref_harness.h -- the inputs and outputs of the drivers in ref_harness.cu
// and ref_seam.cu (TEST INFRASTRUCTURE ONLY), mirrored by oracle/ref.py.
#pragma once

#include <cstdint>
#include <cstring>

#include "MyArray.h"

template <class T>
inline void put(MyArray<T, 3>& a, const T* src) {
  if (src) std::memcpy(a.data_, src, sizeof(T) * (size_t)a.size_);
}
template <class T>
inline void get(const MyArray<T, 3>& a, T* dst) {
  if (dst) std::memcpy(dst, a.data_, sizeof(T) * (size_t)a.size_);
}

extern "C" {

struct ref_inputs {
  int Nx, Ny, Nz;
  double Lx, Ly, Lz, dt;
  int solver_type;   // PCG_TYPES
  double tol;        // tol_ (max|r|*dt)
  int levels;        // gmg_levels
  int do_correct;
  const double *vxs, *vys, *vzs, *eps, *eps_old, *fbx, *fby, *fbz, *fsx, *fsy, *fsz, *firx, *firy, *firz;
  const uint8_t *ct, *fxt, *fyt, *fzt;
};

struct ref_outputs {
  double *p_delta, *rhs, *vx, *vy, *vz, *p;
  int iterations;     // parsed from the reference's "PCG iter = %d" line
  int num_levels;
  double solve_ms;    // device time of solve_poisson (CUDA events on the legacy stream)
  double correct_ms;  // device time of correct_vof_velocity (0 without do_correct)
};

}  // extern "C"
