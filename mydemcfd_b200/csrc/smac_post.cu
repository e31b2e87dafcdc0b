// smac_post.cu -- the pass after the projection: pressure in solid and ghost
// cells, outlet and ghost velocities, face pressure gradient.
//
// The reference runs it as G_SMACSolver::update_boundary_ghost followed by
// make_face_gradp (CFD/G_SMACSolver.cu:1144-1363, CFD/G_BoundaryFunctions.cu:
// 143-560): eleven kernels over the whole (N+3)^3 thread box each, most of
// whose threads find nothing to do.  Here:
//
//   k_pressure_ghost   one launch: a 16-byte-vector scan of the cell types
//                      for C_SOLID cells (the only interior cells written),
//                      plus one thread per ghost cell (O(N^2) threads);
//   k_velocity_outlet  one launch: a 16-byte-vector scan of the three outlet
//                      mark arrays, writing only marked faces;
//   k_velocity_ghost   one launch over the ghost faces and edge corners of
//                      the three face families (O(N^2) threads);
//   k_face_gradp       a z-march over the (N+1)^3 box writing the three
//                      gradient arrays: the one HBM-bound kernel of the pass
//                      (reads p once, writes 3 face arrays).
//
// Every product and sum is an explicit round-to-nearest intrinsic, the
// reference being compiled with -fmad=false (makefile_CFD:5), so every value
// equals the reference's bit for bit.
//
// Where the reference's launches race (its first pressure kernel writes ghost
// cells that its second overwrites; its corner kernels read the ghost values
// of the kernel before), the final state is reproduced without the race:
// a ghost cell whose source cell is C_SOLID computes that cell's new value
// itself (from interior neighbours that nothing writes), and a corner face
// computes its two ghost neighbours' values itself.
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "smac_b200.h"
#include "smac_common.cuh"

namespace smac {
void set_error_text(const char* fmt, ...);
}

using smac::RefDims;

namespace {

#define DADD __dadd_rn
#define DSUB __dsub_rn
#define DMUL __dmul_rn

constexpr uint8_t kInterior = 0;  // C_INTERIOR (CFD/Enums.h:18-23)
constexpr uint8_t kSolid = 3;     // C_SOLID
constexpr int kPostThreads = 256;
constexpr int kMaxIds = 256;      // f_*bcid_ is unsigned char

// Bytes of a 16-byte word that are non-zero / equal to 3.  SWAR zero-byte test:
// (v - 0x01..) & ~v & 0x80.. is non-zero iff some byte of v is zero.
__device__ __forceinline__ bool any_zero_byte(uint32_t v) { return ((v - 0x01010101u) & ~v & 0x80808080u) != 0u; }

template <bool EQ3>
__device__ __forceinline__ bool word_hits(uint32_t w) {
  if (EQ3) return any_zero_byte(w ^ 0x03030303u);
  return w != 0u;
}
template <bool EQ3>
__device__ __forceinline__ bool byte_hits(uint8_t b) {
  return EQ3 ? b == 3 : b != 0;
}

// Calls f(i, byte) for every byte i of a[0, n) that is non-zero (EQ3 false)
// or equals 3 (EQ3 true).  The aligned body is read in 16-byte vectors; the
// unaligned head and the tail byte by byte, so nothing outside a[0, n) is read.
template <bool EQ3, class F>
__device__ __forceinline__ void scan_bytes(const uint8_t* __restrict__ a, long long n, long long tid, long long nth,
                                           F&& f) {
  const long long mis = (long long)(reinterpret_cast<uintptr_t>(a) & 15u);
  const long long head = mis ? (16 - mis < n ? 16 - mis : n) : 0;
  const long long nvec = (n - head) / 16;
  const long long tail0 = head + 16 * nvec;
  const uint4* v = reinterpret_cast<const uint4*>(a + head);
  for (long long u = tid; u < nvec; u += nth) {
    const uint4 w = __ldg(v + u);
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (!word_hits<EQ3>(ws[q])) continue;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint8_t b = (uint8_t)(ws[q] >> (8 * k));
        if (byte_hits<EQ3>(b)) f(head + 16 * u + 4 * q + k, b);
      }
    }
  }
  const long long extra = head + (n - tail0);
  for (long long u = tid; u < extra; u += nth) {
    const long long i = u < head ? u : tail0 + (u - head);
    const uint8_t b = a[i];
    if (byte_hits<EQ3>(b)) f(i, b);
  }
}

// ---------------------------------------------------------------------------
// Pressure (k_update_cell_boundary_pressure + k_update_cell_ghost_pressure)

struct PressureArgs {
  RefDims R;
  const uint8_t* ct;
  const double* rho;  // nullptr: rho = 1
  double* p;
  double gx, gy, gz, dx, dy, dz;
  long long ncell;
  long long nghost;
  int scan_blocks;
};

__device__ __forceinline__ double rho_at(const PressureArgs& A, long long c) { return A.rho ? A.rho[c] : 1.0; }

// New pressure of the C_SOLID interior cell (ix,iy,iz): that of its first
// C_INTERIOR neighbour in the order x-, x+, y-, y+, z-, z+, hydrostatically
// shifted, else 0 (CFD/G_SMACSolver.cu:1209-1226).  Reads only interior
// cells, which this pass never writes.
__device__ double solid_pressure(const PressureArgs& A, int ix, int iy, int iz) {
  const RefDims& R = A.R;
  long long n;
  if (A.ct[n = R.cell(ix - 1, iy, iz)] == kInterior) return DADD(A.p[n], DMUL(DMUL(rho_at(A, n), A.gx), A.dx));
  if (A.ct[n = R.cell(ix + 1, iy, iz)] == kInterior) return DSUB(A.p[n], DMUL(DMUL(rho_at(A, n), A.gx), A.dx));
  if (A.ct[n = R.cell(ix, iy - 1, iz)] == kInterior) return DADD(A.p[n], DMUL(DMUL(rho_at(A, n), A.gy), A.dy));
  if (A.ct[n = R.cell(ix, iy + 1, iz)] == kInterior) return DSUB(A.p[n], DMUL(DMUL(rho_at(A, n), A.gy), A.dy));
  if (A.ct[n = R.cell(ix, iy, iz - 1)] == kInterior) return DADD(A.p[n], DMUL(DMUL(rho_at(A, n), A.gz), A.dz));
  if (A.ct[n = R.cell(ix, iy, iz + 1)] == kInterior) return DSUB(A.p[n], DMUL(DMUL(rho_at(A, n), A.gz), A.dz));
  return 0.0;
}

// Ghost cell number k: the planes z = 0 and z = Nz+1 whole, then the rows
// y = 0 and y = Ny+1 of planes 1..Nz, then the cells x = 0 and x = Nx+1 of
// rows 1..Ny of planes 1..Nz.
__device__ __forceinline__ void ghost_cell(const RefDims& R, long long k, int& ix, int& iy, int& iz) {
  const long long sx = R.Nx + 2, P = sx * (R.Ny + 2), Q = sx * R.Nz;
  if (k < 2 * P) {
    iz = k < P ? 0 : R.Nz + 1;
    const long long r = k % P;
    iy = (int)(r / sx);
    ix = (int)(r % sx);
    return;
  }
  k -= 2 * P;
  if (k < 2 * Q) {
    iy = k < Q ? 0 : R.Ny + 1;
    const long long r = k % Q;
    iz = 1 + (int)(r / sx);
    ix = (int)(r % sx);
    return;
  }
  k -= 2 * Q;
  const long long S = (long long)R.Ny * R.Nz;
  ix = k < S ? 0 : R.Nx + 1;
  const long long r = k % S;
  iz = 1 + (int)(r / R.Ny);
  iy = 1 + (int)(r % R.Ny);
}

__global__ void __launch_bounds__(kPostThreads) k_pressure_ghost(PressureArgs A) {
  const RefDims& R = A.R;
  if ((int)blockIdx.x < A.scan_blocks) {
    // interior C_SOLID cells
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nth = (long long)A.scan_blocks * blockDim.x;
    const long long sx = R.Nx + 2, sxy = sx * (R.Ny + 2);
    scan_bytes<true>(A.ct, A.ncell, tid, nth, [&](long long i, uint8_t) {
      const int iz = (int)(i / sxy), iy = (int)((i % sxy) / sx), ix = (int)(i % sx);
      if (ix < 1 || ix > R.Nx || iy < 1 || iy > R.Ny || iz < 1 || iz > R.Nz) return;
      A.p[i] = solid_pressure(A, ix, iy, iz);
    });
    return;
  }
  // ghost cells (CFD/G_SMACSolver.cu:1229-1267)
  const long long k = (long long)(blockIdx.x - A.scan_blocks) * blockDim.x + threadIdx.x;
  if (k >= A.nghost) return;
  int ix, iy, iz;
  ghost_cell(R, k, ix, iy, iz);
  const int sx_ = ix == 0 ? 1 : ix == R.Nx + 1 ? R.Nx : ix;
  const int sy_ = iy == 0 ? 1 : iy == R.Ny + 1 ? R.Ny : iy;
  const int sz_ = iz == 0 ? 1 : iz == R.Nz + 1 ? R.Nz : iz;
  const long long s = R.cell(sx_, sy_, sz_);
  const double ps = A.ct[s] == kSolid ? solid_pressure(A, sx_, sy_, sz_) : A.p[s];
  const double rx = DMUL((double)(ix - sx_), A.dx), ry = DMUL((double)(iy - sy_), A.dy),
               rz = DMUL((double)(iz - sz_), A.dz);
  const double gr = DADD(DADD(DMUL(rx, A.gx), DMUL(ry, A.gy)), DMUL(rz, A.gz));
  A.p[R.cell(ix, iy, iz)] = DADD(ps, DMUL(rho_at(A, s), gr));
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Outlet velocities (k_update_v{x,y,z}_outlet, CFD/G_BoundaryFunctions.cu:143-255)

struct OutletArgs {
  RefDims R;
  const uint8_t* mark[3];  // 1: interior side +1, 2: interior side -1
  const double* vs[3];
  const double* fb[3];
  const double* pd;
  double* v[3];
  double dt;
  double inv_h[3];
  long long n[3];
};

// blockIdx.y is the face family.  Faces outside the reference's thread range
// (indices 1..N+1 on all axes) and marks whose interior cell lies outside the
// cell array are left alone.
__global__ void __launch_bounds__(kPostThreads) k_velocity_outlet(OutletArgs A) {
  const int f = blockIdx.y;
  const RefDims& R = A.R;
  const long long sx = R.Nx + 2 + (f == 0), sy = R.Ny + 2 + (f == 1);
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  scan_bytes<false>(A.mark[f], A.n[f], tid, nth, [&](long long i, uint8_t m) {
    if (m != 1 && m != 2) return;
    int c[3] = {(int)(i % sx), (int)((i / sx) % sy), (int)(i / (sx * sy))};
    if (c[0] < 1 || c[0] > R.Nx + 1 || c[1] < 1 || c[1] > R.Ny + 1 || c[2] < 1 || c[2] > R.Nz + 1) return;
    const int s = m == 1 ? 1 : -1;
    c[f] += s;
    if (c[0] > R.Nx + 1 || c[1] > R.Ny + 1 || c[2] > R.Nz + 1) return;
    const double sign = s < 0 ? 1.0 : -1.0;
    const double dp = A.pd[R.cell(c[0], c[1], c[2])];
    A.v[f][i] = DADD(A.vs[f][i], DMUL(DMUL(DMUL(DMUL(sign, A.fb[f][i]), A.dt), dp), A.inv_h[f]));
  });
}

// ---------------------------------------------------------------------------
// Ghost velocities (k_update_v*_ghost + k_update_v*_ghost_corner,
// CFD/G_BoundaryFunctions.cu:258-560)

struct GhostArgs {
  int N[3];
  const uint8_t* bcid[3];
  const double* lam[3];  // nullptr: 0
  double* v[3];
  uint8_t type[kMaxIds];  // bc_.bcType_; ids past num_ids read as BC_NOSLIP, velocity 0
  double bv[3][kMaxIds];  // bc_.vx_, vy_, vz_
};

// d_get_velocity_ghost_value (CFD/G_BoundaryFunctions.cu:258-275)
__device__ __forceinline__ double ghost_rule(uint8_t type, double vb, double lam, double bnd, double inner) {
  if (type == 2) return DSUB(DMUL(DMUL(2.0, DSUB(1.0, lam)), vb), inner);  // BC_INFLOW
  if (type == 0) return -inner;                                            // BC_NOSLIP
  if (type == 4) return DSUB(DMUL(2.0, bnd), inner);                       // BC_OUTLET
  if (type == 1) return inner;                                             // BC_SLIP
  return bnd;                                                              // BC_OUTFLOW
}

struct FaceLayout {
  long long S0, S1;
  __device__ __forceinline__ long long at(const int i[3]) const { return ((long long)i[2] * S1 + i[1]) * S0 + i[0]; }
};

// Value of the ghost face at i (i[g] = 0 or N[g]+1) of family a: the rule of
// the boundary id of the first face inside, from the first two faces inside.
__device__ __forceinline__ double ghost_face(const GhostArgs& A, int a, const FaceLayout& L, const int i[3], int g) {
  const bool low = i[g] == 0;
  int ib[3] = {i[0], i[1], i[2]}, in[3] = {i[0], i[1], i[2]};
  ib[g] = low ? 1 : A.N[g];
  in[g] = low ? 2 : A.N[g] - 1;
  const long long fbnd = L.at(ib);
  const uint8_t id = A.bcid[a][fbnd];
  const double lam = A.lam[a] ? A.lam[a][fbnd] : 0.0;
  return ghost_rule(A.type[id], A.bv[a][id], lam, A.v[a][fbnd], A.v[a][L.at(in)]);
}

// blockIdx.z: face family a; blockIdx.y: 0-3 the ghost slabs (low/high across
// the first tangential axis b, then low/high across the second c), 4 the
// four corner lines.  Threads run along the lower-numbered free axis so that
// x-contiguous slabs are read and written coalesced.  Ghost faces read only
// faces 1..N across their ghost axis, which this kernel never writes (N >= 2);
// corner faces evaluate their two ghost neighbours themselves.
__global__ void __launch_bounds__(kPostThreads) k_velocity_ghost(GhostArgs A) {
  const int a = blockIdx.z, part = blockIdx.y;
  const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
  FaceLayout L;
  L.S0 = A.N[0] + 2 + (a == 0);
  L.S1 = A.N[1] + 2 + (a == 1);
  const int na = A.N[a] + 1;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  double* __restrict__ v = A.v[a];
  int i[3];
  if (part < 4) {
    const int g = part < 2 ? b : c, o = part < 2 ? c : b;
    const bool low = (part & 1) == 0;
    const int no = A.N[o];
    const long long total = (long long)na * no;
    for (long long t = tid; t < total; t += nth) {
      if (a < o) {
        i[a] = 1 + (int)(t % na);
        i[o] = 1 + (int)(t / na);
      } else {
        i[o] = 1 + (int)(t % no);
        i[a] = 1 + (int)(t / no);
      }
      i[g] = low ? 0 : A.N[g] + 1;
      v[L.at(i)] = ghost_face(A, a, L, i, g);
    }
    return;
  }
  const long long total = 4LL * na;
  for (long long t = tid; t < total; t += nth) {
    const int corner = (int)(t / na);
    i[a] = 1 + (int)(t % na);
    const bool hb = corner & 1, hc = corner >> 1;
    i[b] = hb ? A.N[b] + 1 : 0;
    i[c] = hc ? A.N[c] + 1 : 0;
    int j1[3] = {i[0], i[1], i[2]}, j2[3] = {i[0], i[1], i[2]};
    j1[c] = hc ? A.N[c] : 1;  // ghost across b, first face inside along c
    j2[b] = hb ? A.N[b] : 1;  // ghost across c, first face inside along b
    v[L.at(i)] = DMUL(0.5, DADD(ghost_face(A, a, L, j1, b), ghost_face(A, a, L, j2, c)));
  }
}

// ---------------------------------------------------------------------------
// Face pressure gradient (k_make_face_gradp_{x,y,z}, CFD/G_SMACSolver.cu:1277-1343)

constexpr int GP_TX = 32, GP_TY = 8;

// One thread per (x, y) column of the (N+1)^3 box of faces 1..N+1, marching
// in z over a chunk of planes: p(z-1) stays in a register, p(x-1) and p(y-1)
// come from the lines that neighbouring threads of the block just loaded.
__global__ void __launch_bounds__(GP_TX* GP_TY) k_face_gradp(RefDims R, const double* __restrict__ p,
                                                             double* __restrict__ gx, double* __restrict__ gy,
                                                             double* __restrict__ gz, double idx, double idy,
                                                             double idz, int zchunk) {
  const int ix = blockIdx.x * GP_TX + threadIdx.x + 1;
  const int iy = blockIdx.y * GP_TY + threadIdx.y + 1;
  if (ix > R.Nx + 1 || iy > R.Ny + 1) return;
  const int z0 = 1 + blockIdx.z * zchunk;
  const int z1 = min(R.Nz + 1, z0 + zchunk - 1);
  const long long sx = R.Nx + 2, sxy = sx * (R.Ny + 2);
  long long c = R.cell(ix, iy, z0);
  double below = __ldg(p + c - sxy);
  for (int iz = z0; iz <= z1; ++iz, c += sxy) {
    const double pc = __ldg(p + c), pxm = __ldg(p + c - 1), pym = __ldg(p + c - sx);
    gx[R.xf(ix, iy, iz)] = DMUL(DSUB(pc, pxm), idx);
    gy[R.yf(ix, iy, iz)] = DMUL(DSUB(pc, pym), idy);
    gz[R.zf(ix, iy, iz)] = DMUL(DSUB(pc, below), idz);
    below = pc;
  }
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

bool bad_desc(const smac_grid_desc* d, const char* fn, int min_n) {
  if (d->nx < min_n || d->ny < min_n || d->nz < min_n) {
    smac::set_error_text("%s: grid %d x %d x %d (each at least %d)", fn, d->nx, d->ny, d->nz, min_n);
    return true;
  }
  if (!(d->dx > 0.0) || !(d->dy > 0.0) || !(d->dz > 0.0)) {
    smac::set_error_text("%s: spacing must be > 0", fn);
    return true;
  }
  return false;
}

smac_status launch_status(const char* fn) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    smac::set_error_text("%s: %s", fn, cudaGetErrorString(e));
    return SMAC_CUDA_ERROR;
  }
  return SMAC_OK;
}

}  // namespace

extern "C" {

smac_status smac_update_pressure_ghost(const smac_grid_desc* d, const uint8_t* celltype, const double* rho, double gx,
                                       double gy, double gz, double* p, void* stream) {
  static const char* fn = "smac_update_pressure_ghost";
  if (!d || !celltype || !p) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bad_desc(d, fn, 1)) return SMAC_BAD_SHAPE;
  PressureArgs A;
  A.R = RefDims{d->nx, d->ny, d->nz};
  A.ct = celltype;
  A.rho = rho;
  A.p = p;
  A.gx = gx; A.gy = gy; A.gz = gz;
  A.dx = d->dx; A.dy = d->dy; A.dz = d->dz;
  const long long sx = d->nx + 2, sy = d->ny + 2, sz = d->nz + 2;
  A.ncell = sx * sy * sz;
  A.nghost = A.ncell - (long long)d->nx * d->ny * d->nz;
  const long long vec_units = A.ncell / 16 + 16;
  const long long want = (vec_units + kPostThreads - 1) / kPostThreads;
  A.scan_blocks = (int)(want < 4LL * sm_count() ? want : 4LL * sm_count());
  const long long ghost_blocks = (A.nghost + kPostThreads - 1) / kPostThreads;
  k_pressure_ghost<<<(unsigned)(A.scan_blocks + ghost_blocks), kPostThreads, 0, (cudaStream_t)stream>>>(A);
  return launch_status(fn);
}

smac_status smac_update_velocity_ghost(const smac_grid_desc* d, const smac_boundary_table* bc, const uint8_t* fxbcid,
                                       const uint8_t* fybcid, const uint8_t* fzbcid, const uint8_t* fxo,
                                       const uint8_t* fyo, const uint8_t* fzo, const double* lamx, const double* lamy,
                                       const double* lamz, const double* vxs, const double* vys, const double* vzs,
                                       const double* fbx, const double* fby, const double* fbz, const double* p_delta,
                                       double dt, double* vx, double* vy, double* vz, void* stream) {
  static const char* fn = "smac_update_velocity_ghost";
  if (!d || !bc || !fxbcid || !fybcid || !fzbcid || !vx || !vy || !vz) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bc->num_ids < 1 || bc->num_ids > kMaxIds || !bc->type || !bc->vx || !bc->vy || !bc->vz) {
    smac::set_error_text("%s: boundary table needs 1..%d ids and its four arrays", fn, kMaxIds);
    return SMAC_BAD_ARG;
  }
  const bool outlets = fxo || fyo || fzo;
  if (outlets && (!fxo || !fyo || !fzo || !vxs || !vys || !vzs || !fbx || !fby || !fbz || !p_delta)) {
    smac::set_error_text("%s: outlet marks need all three mark arrays, v*, f_b and p_delta", fn);
    return SMAC_BAD_ARG;
  }
  // the ghost rule reads the second face inside, which must not be a ghost face
  if (bad_desc(d, fn, 2)) return SMAC_BAD_SHAPE;
  cudaStream_t s = (cudaStream_t)stream;
  const long long X = d->nx, Y = d->ny, Z = d->nz;
  if (outlets) {
    OutletArgs O;
    O.R = RefDims{d->nx, d->ny, d->nz};
    O.mark[0] = fxo; O.mark[1] = fyo; O.mark[2] = fzo;
    O.vs[0] = vxs; O.vs[1] = vys; O.vs[2] = vzs;
    O.fb[0] = fbx; O.fb[1] = fby; O.fb[2] = fbz;
    O.pd = p_delta;
    O.v[0] = vx; O.v[1] = vy; O.v[2] = vz;
    O.dt = dt;
    O.inv_h[0] = 1. / d->dx; O.inv_h[1] = 1. / d->dy; O.inv_h[2] = 1. / d->dz;
    O.n[0] = (X + 3) * (Y + 2) * (Z + 2);
    O.n[1] = (X + 2) * (Y + 3) * (Z + 2);
    O.n[2] = (X + 2) * (Y + 2) * (Z + 3);
    const long long want = (O.n[0] / 16 + 16 + kPostThreads - 1) / kPostThreads;
    const int blocks = (int)(want < 2LL * sm_count() ? want : 2LL * sm_count());
    k_velocity_outlet<<<dim3(blocks, 3), kPostThreads, 0, s>>>(O);
    const smac_status st = launch_status(fn);
    if (st != SMAC_OK) return st;
  }
  GhostArgs G;
  std::memset(&G, 0, sizeof(G));
  G.N[0] = d->nx; G.N[1] = d->ny; G.N[2] = d->nz;
  G.bcid[0] = fxbcid; G.bcid[1] = fybcid; G.bcid[2] = fzbcid;
  G.lam[0] = lamx; G.lam[1] = lamy; G.lam[2] = lamz;
  G.v[0] = vx; G.v[1] = vy; G.v[2] = vz;
  std::memcpy(G.type, bc->type, (size_t)bc->num_ids);
  for (int k = 0; k < bc->num_ids; ++k) {
    G.bv[0][k] = bc->vx[k];
    G.bv[1][k] = bc->vy[k];
    G.bv[2][k] = bc->vz[k];
  }
  const long long longest = (X > Y ? (X > Z ? X : Z) : (Y > Z ? Y : Z)) + 1;
  const long long per_slab = longest * longest;
  const long long want = (per_slab + kPostThreads - 1) / kPostThreads;
  const int blocks = (int)(want < 64 ? want : 64);
  k_velocity_ghost<<<dim3(blocks, 5, 3), kPostThreads, 0, s>>>(G);
  return launch_status(fn);
}

smac_status smac_face_gradp(const smac_grid_desc* d, const double* p, double* gpx, double* gpy, double* gpz,
                            void* stream) {
  static const char* fn = "smac_face_gradp";
  if (!d || !p || !gpx || !gpy || !gpz) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bad_desc(d, fn, 1)) return SMAC_BAD_SHAPE;
  const RefDims R{d->nx, d->ny, d->nz};
  const unsigned bx = (unsigned)((d->nx + 1 + GP_TX - 1) / GP_TX), by = (unsigned)((d->ny + 1 + GP_TY - 1) / GP_TY);
  // about 8 blocks of 256 threads per SM, each marching over a z-chunk
  const long long target = 8LL * sm_count();
  long long nzc = (target + (long long)bx * by - 1) / ((long long)bx * by);
  if (nzc < 1) nzc = 1;
  if (nzc > d->nz + 1) nzc = d->nz + 1;
  const int zchunk = (int)((d->nz + 1 + nzc - 1) / nzc);
  const unsigned bz = (unsigned)((d->nz + 1 + zchunk - 1) / zchunk);
  k_face_gradp<<<dim3(bx, by, bz), dim3(GP_TX, GP_TY), 0, (cudaStream_t)stream>>>(
      R, p, gpx, gpy, gpz, 1. / d->dx, 1. / d->dy, 1. / d->dz, zchunk);
  return launch_status(fn);
}

}  // extern "C"
