// smac_post.cu -- the calls either side of the projection: before it the
// momentum predictor u*, the wall u* rule and the surface-tension force;
// after it the pressure in solid and ghost cells, outlet and ghost
// velocities, and the face pressure gradient.
//
// The reference runs it as G_SMACSolver::update_boundary_ghost followed by
// make_face_gradp (CFD/G_SMACSolver.cu:1144-1363, CFD/G_BoundaryFunctions.cu:
// 143-560): eleven kernels over the whole (N+3)^3 thread box each, most of
// whose threads find nothing to do.  Here:
//
//   k_pressure_ghost   one launch: a word-wise scan of the cell types for
//                      C_SOLID cells (the only interior cells written),
//                      plus one thread per ghost cell (O(N^2) threads);
//   k_velocity_outlet  one launch: a word-wise scan of the three outlet mark
//                      arrays, writing only marked faces;
//   k_velocity_ghost   one launch over the ghost faces and edge corners of
//                      the three face families (O(N^2) threads);
//   k_face_gradp       one thread per face index of the (N+1)^3 box writing
//                      the three gradient arrays: the one HBM-bound kernel
//                      of the pass (reads p once, writes 3 face arrays).
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

// Byte matches: MATCH < 0 means "non-zero", otherwise "equal to MATCH".
// SWAR zero-byte test: (v - 0x01..) & ~v & 0x80.. is non-zero iff some byte
// of v is zero.
__device__ __forceinline__ bool any_zero_byte(uint32_t v) { return ((v - 0x01010101u) & ~v & 0x80808080u) != 0u; }

template <int MATCH>
__device__ __forceinline__ bool word_hits(uint32_t w) {
  if (MATCH < 0) return w != 0u;
  return any_zero_byte(w ^ (0x01010101u * (uint32_t)MATCH));
}
template <int MATCH>
__device__ __forceinline__ bool byte_hits(uint32_t b) {
  return MATCH < 0 ? b != 0u : b == (uint32_t)MATCH;
}

// Unsigned 32-bit division by an invariant divisor d >= 1 as a multiply-high
// and two shifts (Granlund and Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994, fig. 4.1): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1,  n / d = (t + ((n - t) >> min(l,1))) >> max(l-1,0)
// where t = mulhi(m, n), exact for every 32-bit n.
struct FastDiv {
  uint32_t d, m;
  int s1, s2;
};
inline FastDiv make_fastdiv(uint32_t d) {
  int l = 0;
  while ((1ull << l) < d) ++l;
  const uint64_t m = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
  return FastDiv{d, (uint32_t)m, l < 1 ? l : 1, l > 1 ? l - 1 : 0};
}
__device__ __forceinline__ uint32_t fdiv(const FastDiv& f, uint32_t n) {
  const uint32_t t = __umulhi(f.m, n);
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

// Row and plane lengths of an array: the divisors of its flat index.
struct Shape2 {
  FastDiv sx, sy;
  bool small;  // every flat index < 2^32: the fast division applies
};
inline Shape2 make_shape2(long long sx, long long sy, long long n) {
  return Shape2{make_fastdiv((uint32_t)sx), make_fastdiv((uint32_t)sy), n <= 0xffffffffLL};
}

// Position of a flat index in an array of rows of sx entries and planes of
// sy rows.
struct Pos {
  int x, y, z;
};
__device__ __forceinline__ Pos decode(long long i, const Shape2& S) {
  if (S.small) {
    const uint32_t r = fdiv(S.sx, (uint32_t)i), z = fdiv(S.sy, r);
    return Pos{(int)((uint32_t)i - r * S.sx.d), (int)(r - z * S.sy.d), (int)z};
  }
  const long long sx = S.sx.d, sy = S.sy.d, r = i / sx;
  return Pos{(int)(i - r * sx), (int)(r % sy), (int)(r / sy)};
}
constexpr int SCAN_U = 4;                   // 4-byte loads in flight per lane
constexpr int SCAN_QUEUE = 32 * SCAN_U * 4;  // a warp's hits of one pass (every byte)
constexpr int kPostWarps = kPostThreads / 32;

// Calls hit(i) for every byte i of a[0, n) that matches (byte_hits<MATCH>),
// with whole warps doing the work.  Each lane reads SCAN_U 4-byte words of
// the aligned body (all issued before any is tested); the lanes' matching
// bytes go to the warp's queue in shared memory (ballot + prefix count), and
// then the warp's 32 lanes take the queue's entries in turn.  Matches are
// rare or come in runs (solid regions, boundary planes): either way a
// warp's lanes stay busy, where handling a match in the lane that found it
// leaves most lanes idle.  The unaligned head and the tail are tested byte
// by byte by single lanes, so nothing outside a[0, n) is read.  The loop
// bounds are the same for all lanes of a warp (nth and tid - lane are
// multiples of 32).
template <int MATCH, class F>
__device__ __forceinline__ void scan_compact(const uint8_t* __restrict__ a, long long n, long long tid, long long nth,
                                             long long* __restrict__ queue, F&& hit) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const long long mis = (long long)(reinterpret_cast<uintptr_t>(a) & 3u);
  const long long head = mis ? (4 - mis < n ? 4 - mis : n) : 0;
  const long long nw = (n - head) / 4;
  const long long tail0 = head + 4 * nw;
  const uint32_t* v = reinterpret_cast<const uint32_t*>(a + head);
  for (long long u0 = tid - lane; u0 < nw; u0 += SCAN_U * nth) {
    const long long u = u0 + lane;
    uint32_t w[SCAN_U];
#pragma unroll
    for (int k = 0; k < SCAN_U; ++k) w[k] = u + k * nth < nw ? __ldg(v + u + k * nth) : 0u;
    bool any = false;
#pragma unroll
    for (int k = 0; k < SCAN_U; ++k) any |= word_hits<MATCH>(w[k]) && u + k * nth < nw;
    if (!__any_sync(0xffffffffu, any)) continue;
    int count = 0;
#pragma unroll
    for (int k = 0; k < SCAN_U; ++k) {
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const bool h = u + k * nth < nw && byte_hits<MATCH>((w[k] >> (8 * b)) & 0xffu);
        const unsigned m = __ballot_sync(0xffffffffu, h);
        if (h) queue[count + __popc(m & below)] = head + 4 * (u + k * nth) + b;
        count += __popc(m);
      }
    }
    __syncwarp();
    for (int q = lane; q < count; q += 32) hit(queue[q]);
    __syncwarp();
  }
  const long long extra = head + (n - tail0);
  for (long long u = tid; u < extra; u += nth) {
    const long long i = u < head ? u : tail0 + (u - head);
    if (byte_hits<MATCH>(a[i])) hit(i);
  }
}

// Blocks for a scan of n bytes: one pass of SCAN_U words per thread, at
// most 16 blocks per SM.  (Each block also holds kPostWarps queues of
// SCAN_QUEUE flat indices in shared memory.)
inline int scan_blocks_for(long long n, int sms) {
  const long long want = (n / 4 + SCAN_U * kPostThreads - 1) / (SCAN_U * kPostThreads) + 1;
  return (int)(want < 16LL * sms ? want : 16LL * sms);
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
  Shape2 shape;  // of the cell array
  int scan_blocks;
  int gz_bx, gz_by;  // blocks of the z-ghost planes (32 x 8 threads, x by y)
  int gy_bx, gy_bz;  // blocks of the y-ghost rows (x by z)
  int gx_by, gx_bz;  // blocks of the x-ghost cells (y by z)
};

__device__ __forceinline__ double rho_at(const PressureArgs& A, long long c) { return A.rho ? A.rho[c] : 1.0; }

// The neighbour that sets the new pressure of the C_SOLID interior cell c:
// its first C_INTERIOR neighbour in the order x-, x+, y-, y+, z-, z+
// (CFD/G_SMACSolver.cu:1209-1226).  Returns -1 without one (p = 0); axis
// and side of the chosen neighbour go to *axis and *up.  The six types are
// loaded together.
__device__ __forceinline__ long long solid_source(const PressureArgs& A, long long c, int* axis, bool* up) {
  const long long sx = A.R.Nx + 2, sxy = sx * (A.R.Ny + 2);
  const uint8_t t0 = A.ct[c - 1], t1 = A.ct[c + 1], t2 = A.ct[c - sx], t3 = A.ct[c + sx], t4 = A.ct[c - sxy],
                t5 = A.ct[c + sxy];
  *up = false;
  if (t0 == kInterior) { *axis = 0; return c - 1; }
  *up = true;
  if (t1 == kInterior) { *axis = 0; return c + 1; }
  *up = false;
  if (t2 == kInterior) { *axis = 1; return c - sx; }
  *up = true;
  if (t3 == kInterior) { *axis = 1; return c + sx; }
  *up = false;
  if (t4 == kInterior) { *axis = 2; return c - sxy; }
  *up = true;
  if (t5 == kInterior) { *axis = 2; return c + sxy; }
  *axis = 0;
  return -1;
}

// p(n) shifted by rho(n) g h along axis, subtracted for an up-side neighbour.
__device__ __forceinline__ double solid_value(const PressureArgs& A, double pn, double rn, int axis, bool up) {
  const double g = axis == 0 ? A.gx : axis == 1 ? A.gy : A.gz;
  const double h = axis == 0 ? A.dx : axis == 1 ? A.dy : A.dz;
  const double shift = DMUL(DMUL(rn, g), h);
  return up ? DSUB(pn, shift) : DADD(pn, shift);
}

__device__ double solid_pressure(const PressureArgs& A, long long c) {
  int axis;
  bool up;
  const long long n = solid_source(A, c, &axis, &up);
  return n < 0 ? 0.0 : solid_value(A, A.p[n], rho_at(A, n), axis, up);
}

// Ghost cell (ix,iy,iz) takes p of the nearest interior cell plus
// rho(src) g.r (CFD/G_SMACSolver.cu:1229-1267); a C_SOLID source's new value
// is computed here rather than read.
__device__ __forceinline__ void ghost_pressure(const PressureArgs& A, int ix, int iy, int iz) {
  const RefDims& R = A.R;
  const int sx_ = ix == 0 ? 1 : ix == R.Nx + 1 ? R.Nx : ix;
  const int sy_ = iy == 0 ? 1 : iy == R.Ny + 1 ? R.Ny : iy;
  const int sz_ = iz == 0 ? 1 : iz == R.Nz + 1 ? R.Nz : iz;
  const long long s = R.cell(sx_, sy_, sz_);
  const uint8_t ts = A.ct[s];
  const double ps_read = A.p[s], rs = rho_at(A, s);
  const double ps = ts == kSolid ? solid_pressure(A, s) : ps_read;
  const double rx = DMUL((double)(ix - sx_), A.dx), ry = DMUL((double)(iy - sy_), A.dy),
               rz = DMUL((double)(iz - sz_), A.dz);
  const double gr = DADD(DADD(DMUL(rx, A.gx), DMUL(ry, A.gy)), DMUL(rz, A.gz));
  A.p[R.cell(ix, iy, iz)] = DADD(ps, DMUL(rs, gr));
}

// Blocks [0, scan_blocks): the cell types are scanned for interior C_SOLID
// cells.  The blocks after them cover the ghost cells as three 2-D groups of
// 32 x 8 threads: the planes z = 0 and Nz+1 (x by y), the rows y = 0 and
// Ny+1 of planes 1..Nz (x by z), the cells x = 0 and Nx+1 of rows 1..Ny of
// planes 1..Nz (y by z).
__global__ void __launch_bounds__(kPostThreads) k_pressure_ghost(PressureArgs A) {
  const RefDims& R = A.R;
  if ((int)blockIdx.x < A.scan_blocks) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nth = (long long)A.scan_blocks * blockDim.x;
    __shared__ long long queue[kPostWarps * SCAN_QUEUE];
    scan_compact<kSolid>(A.ct, A.ncell, tid, nth, queue + (threadIdx.x >> 5) * SCAN_QUEUE, [&](long long i) {
      const Pos q = decode(i, A.shape);
      if (q.x >= 1 && q.x <= R.Nx && q.y >= 1 && q.y <= R.Ny && q.z >= 1 && q.z <= R.Nz)
        A.p[i] = solid_pressure(A, i);
    });
    return;
  }
  int b = (int)blockIdx.x - A.scan_blocks;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int nz_blocks = 2 * A.gz_bx * A.gz_by, ny_blocks = 2 * A.gy_bx * A.gy_bz;
  if (b < nz_blocks) {
    const int side = b / (A.gz_bx * A.gz_by);
    b -= side * A.gz_bx * A.gz_by;
    const int ix = (b % A.gz_bx) * 32 + tx, iy = (b / A.gz_bx) * 8 + ty;
    if (ix < R.Nx + 2 && iy < R.Ny + 2) ghost_pressure(A, ix, iy, side ? R.Nz + 1 : 0);
    return;
  }
  b -= nz_blocks;
  if (b < ny_blocks) {
    const int side = b / (A.gy_bx * A.gy_bz);
    b -= side * A.gy_bx * A.gy_bz;
    const int ix = (b % A.gy_bx) * 32 + tx, iz = 1 + (b / A.gy_bx) * 8 + ty;
    if (ix < R.Nx + 2 && iz <= R.Nz) ghost_pressure(A, ix, side ? R.Ny + 1 : 0, iz);
    return;
  }
  b -= ny_blocks;
  const int side = b / (A.gx_by * A.gx_bz);
  b -= side * A.gx_by * A.gx_bz;
  const int iy = 1 + (b % A.gx_by) * 32 + tx, iz = 1 + (b / A.gx_by) * 8 + ty;
  if (iy <= R.Ny && iz <= R.Nz) ghost_pressure(A, side ? R.Nx + 1 : 0, iy, iz);
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
  Shape2 shape[3];  // of each family's face arrays
};

// Outlet faces of family FAM.  Faces outside the reference's thread range
// (indices 1..N+1 on all axes) and marks whose interior cell lies outside
// the cell array are left alone.
template <int FAM>
__device__ __forceinline__ void outlet_family(const OutletArgs& A, long long tid, long long nth, long long* queue) {
  const RefDims& R = A.R;
  const int nmax = (FAM == 0 ? R.Nx : FAM == 1 ? R.Ny : R.Nz) + 1;
  const uint8_t* __restrict__ mark = A.mark[FAM];
  const double* __restrict__ vs = A.vs[FAM];
  const double* __restrict__ fb = A.fb[FAM];
  double* __restrict__ v = A.v[FAM];
  const double inv_h = A.inv_h[FAM];
  scan_compact<-1>(mark, A.n[FAM], tid, nth, queue, [&](long long i) {
    const uint8_t m = mark[i];
    const Pos q = decode(i, A.shape[FAM]);
    const int s = m == 1 ? 1 : -1;
    int c[3] = {q.x, q.y, q.z};
    c[FAM] += s;
    if ((m != 1 && m != 2) || q.x < 1 || q.x > R.Nx + 1 || q.y < 1 || q.y > R.Ny + 1 || q.z < 1 || q.z > R.Nz + 1 ||
        c[FAM] > nmax)
      return;
    const double sign = s < 0 ? 1.0 : -1.0;
    const double dp = A.pd[R.cell(c[0], c[1], c[2])];
    v[i] = DADD(vs[i], DMUL(DMUL(DMUL(DMUL(sign, fb[i]), A.dt), dp), inv_h));
  });
}

// blockIdx.y is the face family.
__global__ void __launch_bounds__(kPostThreads) k_velocity_outlet(OutletArgs A) {
  __shared__ long long queue[kPostWarps * SCAN_QUEUE];
  long long* q = queue + (threadIdx.x >> 5) * SCAN_QUEUE;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  switch (blockIdx.y) {
    case 0: outlet_family<0>(A, tid, nth, q); break;
    case 1: outlet_family<1>(A, tid, nth, q); break;
    default: outlet_family<2>(A, tid, nth, q); break;
  }
}

// ---------------------------------------------------------------------------
// Ghost velocities (k_update_v*_ghost + k_update_v*_ghost_corner,
// CFD/G_BoundaryFunctions.cu:258-560)

// The boundary table, passed by value in the kernel parameters.
struct BcTable {
  uint8_t type[kMaxIds];  // bc_.bcType_; ids past num_ids read as BC_NOSLIP, velocity 0
  double bv[3][kMaxIds];  // bc_.vx_, vy_, vz_
};

struct GhostArgs {
  int N[3];
  const uint8_t* bcid[3];
  const double* lam[3];  // nullptr: 0
  double* v[3];
  BcTable bc;
};

// d_get_velocity_ghost_value (CFD/G_BoundaryFunctions.cu:258-275)
__device__ __forceinline__ double ghost_rule(uint8_t type, double vb, double lam, double bnd, double inner) {
  if (type == 2) return DSUB(DMUL(DMUL(2.0, DSUB(1.0, lam)), vb), inner);  // BC_INFLOW
  if (type == 0) return -inner;                                            // BC_NOSLIP
  if (type == 4) return DSUB(DMUL(2.0, bnd), inner);                       // BC_OUTLET
  if (type == 1) return inner;                                             // BC_SLIP
  return bnd;                                                              // BC_OUTFLOW
}

// Face index (i0, i1, i2) of family FAM in the reference layout.
template <int FAM>
__device__ __forceinline__ long long face_at(const int N[3], int i0, int i1, int i2) {
  const long long S0 = N[0] + 2 + (FAM == 0), S1 = N[1] + 2 + (FAM == 1);
  return ((long long)i2 * S1 + i1) * S0 + i0;
}

// Value of the ghost face i (i[G] = 0 or N[G]+1) of family FAM: the rule of
// the boundary id of the first face inside, from the first two faces inside.
template <int FAM, int G>
__device__ __forceinline__ double ghost_face(const GhostArgs& A, int i0, int i1, int i2) {
  int ib[3] = {i0, i1, i2}, in[3] = {i0, i1, i2};
  const bool low = (G == 0 ? i0 : G == 1 ? i1 : i2) == 0;
  ib[G] = low ? 1 : A.N[G];
  in[G] = low ? 2 : A.N[G] - 1;
  const long long fbnd = face_at<FAM>(A.N, ib[0], ib[1], ib[2]);
  const uint8_t id = A.bcid[FAM][fbnd];
  const double lam = A.lam[FAM] ? A.lam[FAM][fbnd] : 0.0;
  return ghost_rule(A.bc.type[id], A.bc.bv[FAM][id], lam, A.v[FAM][fbnd],
                    A.v[FAM][face_at<FAM>(A.N, in[0], in[1], in[2])]);
}

// One part of family FAM: PART 0-3 the ghost slabs (low/high across the first
// tangential axis B, then low/high across the second C), PART 4 the four
// corner lines.  Threads run along the lower-numbered free axis, so that
// x-contiguous slabs are read and written coalesced.
template <int FAM, int PART>
__device__ __forceinline__ void ghost_part(const GhostArgs& A, long long tid, long long nth) {
  constexpr int B = FAM == 0 ? 1 : 0, C = FAM == 2 ? 1 : 2;
  const int na = A.N[FAM] + 1;
  double* __restrict__ v = A.v[FAM];
  if (PART < 4) {
    constexpr int G = PART < 2 ? B : C, O = PART < 2 ? C : B;
    constexpr bool LOW = (PART & 1) == 0;
    const int no = A.N[O];
    // 32-bit index arithmetic: a slab has (N+1) N < 2^32 faces
    const uint32_t total = (uint32_t)na * (uint32_t)no, fast = FAM < O ? na : no;
    for (uint32_t t = (uint32_t)tid; t < total; t += (uint32_t)nth) {
      const uint32_t slow = t / fast, f = t - slow * fast;
      int i[3];
      if (FAM < O) {
        i[FAM] = 1 + (int)f;
        i[O] = 1 + (int)slow;
      } else {
        i[O] = 1 + (int)f;
        i[FAM] = 1 + (int)slow;
      }
      i[G] = LOW ? 0 : A.N[G] + 1;
      v[face_at<FAM>(A.N, i[0], i[1], i[2])] = ghost_face<FAM, G>(A, i[0], i[1], i[2]);
    }
    return;
  }
  const uint32_t total = 4u * (uint32_t)na;
  for (uint32_t t = (uint32_t)tid; t < total; t += (uint32_t)nth) {
    const int corner = (int)(t / (uint32_t)na);
    const bool hb = corner & 1, hc = corner >> 1;
    int i[3];
    i[FAM] = 1 + (int)(t - (uint32_t)corner * (uint32_t)na);
    i[B] = hb ? A.N[B] + 1 : 0;
    i[C] = hc ? A.N[C] + 1 : 0;
    int j1[3] = {i[0], i[1], i[2]}, j2[3] = {i[0], i[1], i[2]};
    j1[C] = hc ? A.N[C] : 1;  // ghost across B, first face inside along C
    j2[B] = hb ? A.N[B] : 1;  // ghost across C, first face inside along B
    v[face_at<FAM>(A.N, i[0], i[1], i[2])] =
        DMUL(0.5, DADD(ghost_face<FAM, B>(A, j1[0], j1[1], j1[2]), ghost_face<FAM, C>(A, j2[0], j2[1], j2[2])));
  }
}

template <int FAM>
__device__ __forceinline__ void ghost_family(const GhostArgs& A, int part, long long tid, long long nth) {
  switch (part) {
    case 0: ghost_part<FAM, 0>(A, tid, nth); break;
    case 1: ghost_part<FAM, 1>(A, tid, nth); break;
    case 2: ghost_part<FAM, 2>(A, tid, nth); break;
    case 3: ghost_part<FAM, 3>(A, tid, nth); break;
    default: ghost_part<FAM, 4>(A, tid, nth); break;
  }
}

// blockIdx.z: face family; blockIdx.y: part (ghost_part).  Ghost faces read
// only faces 1..N across their ghost axis, which this kernel never writes
// (N >= 2); corner faces evaluate their two ghost neighbours themselves.
__global__ void __launch_bounds__(kPostThreads) k_velocity_ghost(GhostArgs A) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  switch (blockIdx.z) {
    case 0: ghost_family<0>(A, blockIdx.y, tid, nth); break;
    case 1: ghost_family<1>(A, blockIdx.y, tid, nth); break;
    default: ghost_family<2>(A, blockIdx.y, tid, nth); break;
  }
}

// ---------------------------------------------------------------------------
// Wall-face u* (k_update_v{x,y,z}star_boundary, CFD/G_BoundaryFunctions.cu:3-71)

struct VstarArgs {
  RefDims R;
  const uint8_t* ft[3];
  const uint8_t* bcid[3];
  const uint8_t* mark[3];  // nullptr: no marks (outlet side +1)
  const double* lam[3];    // nullptr: 0
  double* vs[3];
  long long n[3];
  Shape2 shape[3];
  BcTable bc;
};

// F_BOUNDARY faces of family FAM with indices 1..N+1 (the reference's thread
// range), by the type of their boundary id (d_get_v*star_*face,
// CFD/G_BoundaryFunctions.h:369-470): inflow (1 - lam) v_b, no-slip 0,
// outlet the u* of the next face on the marked side, others 0.
template <int FAM>
__device__ __forceinline__ void vstar_family(const VstarArgs& A, long long tid, long long nth, long long* queue) {
  const RefDims& R = A.R;
  const long long stride = FAM == 0 ? 1 : FAM == 1 ? (long long)(R.Nx + 2) : (long long)(R.Nx + 2) * (R.Ny + 2);
  double* __restrict__ vs = A.vs[FAM];
  scan_compact<1>(A.ft[FAM], A.n[FAM], tid, nth, queue, [&](long long i) {
    const Pos q = decode(i, A.shape[FAM]);
    if (q.x < 1 || q.x > R.Nx + 1 || q.y < 1 || q.y > R.Ny + 1 || q.z < 1 || q.z > R.Nz + 1) return;
    const uint8_t id = A.bcid[FAM][i];
    const uint8_t t = A.bc.type[id];
    double v = 0.0;
    if (t == 2) {  // BC_INFLOW
      v = DMUL(DSUB(1.0, A.lam[FAM] ? A.lam[FAM][i] : 0.0), A.bc.bv[FAM][id]);
    } else if (t == 4) {  // BC_OUTLET
      const bool low = A.mark[FAM] && A.mark[FAM][i] == 2;
      v = vs[low ? i - stride : i + stride];
    }
    vs[i] = v;
  });
}

// blockIdx.y is the face family (the reference's three launches touch
// disjoint arrays, so one launch does them all).
__global__ void __launch_bounds__(kPostThreads) k_vstar_boundary(VstarArgs A) {
  __shared__ long long queue[kPostWarps * SCAN_QUEUE];
  long long* q = queue + (threadIdx.x >> 5) * SCAN_QUEUE;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  switch (blockIdx.y) {
    case 0: vstar_family<0>(A, tid, nth, q); break;
    case 1: vstar_family<1>(A, tid, nth, q); break;
    default: vstar_family<2>(A, tid, nth, q); break;
  }
}

// ---------------------------------------------------------------------------
// Face pressure gradient (k_make_face_gradp_{x,y,z}, CFD/G_SMACSolver.cu:1277-1343)

constexpr int GP_TX = 32, GP_TY = 8;

// One thread per face index (x, y) of plane z of the (N+1)^3 box of faces
// 1..N+1, writing the three families' gradients there.  p(x-1), p(y-1) and
// p(z-1) are lines that neighbouring threads and the previous plane's blocks
// load, so they come from L1 / L2: p is read from HBM about once.  (Marching
// each thread in z, with p(z-1) kept in a register, measured slower at
// 256^3: 3.5-4.2 TB/s against 4.5 TB/s.)
__global__ void __launch_bounds__(GP_TX* GP_TY) k_face_gradp(RefDims R, const double* __restrict__ p,
                                                             double* __restrict__ gx, double* __restrict__ gy,
                                                             double* __restrict__ gz, double idx, double idy,
                                                             double idz) {
  const int ix = blockIdx.x * GP_TX + threadIdx.x + 1;
  const int iy = blockIdx.y * GP_TY + threadIdx.y + 1;
  const int iz = blockIdx.z + 1;
  if (ix > R.Nx + 1 || iy > R.Ny + 1) return;
  const long long sx = R.Nx + 2, sxy = sx * (R.Ny + 2);
  const long long c = R.cell(ix, iy, iz);
  const double pc = __ldg(p + c);
  gx[R.xf(ix, iy, iz)] = DMUL(DSUB(pc, __ldg(p + c - 1)), idx);
  gy[R.yf(ix, iy, iz)] = DMUL(DSUB(pc, __ldg(p + c - sx)), idy);
  gz[R.zf(ix, iy, iz)] = DMUL(DSUB(pc, __ldg(p + c - sxy)), idz);
}

// ---------------------------------------------------------------------------
// Surface tension (G_SMACSolver::calc_surface_tension,
// CFD/G_SMACSolver_VoF.cu:87-445): normals, curvature, face force

struct StArgs {
  RefDims R;
  const double* alpha;
  const uint8_t* ct;
  double* nx;
  double* ny;
  double* nz;
  double* kappa;
  double* gm;  // |grad alpha| (the reference's p_tmp_)
  double* fs[3];
  double sigma;
  double ih[3], i2h[3];  // 1/h and 1/(2h), computed as the reference does
};

// One-sided or central difference along an axis from the two neighbours'
// flags (the branches of k_calc_interface_normal / k_calc_curvature).
__device__ __forceinline__ double st_diff(bool p, bool m, double fp, double f0, double fm, double i2h, double ih) {
  if (p && m) return DMUL(DSUB(fp, fm), i2h);
  if (p) return DMUL(DSUB(fp, f0), ih);
  if (m) return DMUL(DSUB(f0, fm), ih);
  return 0.0;
}

// Pass 1, k_calc_interface_normal (:87-182): grad alpha, |grad alpha| and the
// unit normal of every C_INTERIOR cell; other cells are left as they are.
__global__ void __launch_bounds__(256) k_st_normal(StArgs A) {
  const RefDims& R = A.R;
  const int ix = blockIdx.x * 32 + threadIdx.x + 1, iy = blockIdx.y * 8 + threadIdx.y + 1, iz = blockIdx.z + 1;
  if (ix > R.Nx || iy > R.Ny) return;
  const long long sx = R.Nx + 2, sxy = sx * (R.Ny + 2), c = R.cell(ix, iy, iz);
  if (A.ct[c] != kInterior) return;
  const double* a = A.alpha;
  const double gx = st_diff(A.ct[c + 1] == kInterior, A.ct[c - 1] == kInterior, a[c + 1], a[c], a[c - 1], A.i2h[0],
                            A.ih[0]);
  const double gy = st_diff(A.ct[c + sx] == kInterior, A.ct[c - sx] == kInterior, a[c + sx], a[c], a[c - sx],
                            A.i2h[1], A.ih[1]);
  const double gz = st_diff(A.ct[c + sxy] == kInterior, A.ct[c - sxy] == kInterior, a[c + sxy], a[c], a[c - sxy],
                            A.i2h[2], A.ih[2]);
  const double mag2 = DADD(DADD(DMUL(gx, gx), DMUL(gy, gy)), DMUL(gz, gz));
  const double mag = __dsqrt_rn(mag2);
  A.gm[c] = mag;
  if (mag2 > 1e-12) {
    const double inv = __ddiv_rn(1.0, mag);
    A.nx[c] = DMUL(gx, inv);
    A.ny[c] = DMUL(gy, inv);
    A.nz[c] = DMUL(gz, inv);
  } else {
    A.nx[c] = 0.0;
    A.ny[c] = 0.0;
    A.nz[c] = 0.0;
  }
}

// Curvature of cell (ix,iy,iz) in 1..N, k_calc_curvature (:184-290):
// 0 outside 0.01 <= alpha <= 0.99, else -div n, a neighbour counting where
// it is C_INTERIOR with |grad alpha| > 1e-6.
__device__ double st_kappa(const StArgs& A, int ix, int iy, int iz) {
  const RefDims& R = A.R;
  const long long sx = R.Nx + 2, sxy = sx * (R.Ny + 2), c = R.cell(ix, iy, iz);
  const double a = A.alpha[c];
  if (a > 0.99 || a < 0.01) return 0.0;
  auto ok = [&](long long n) { return A.ct[n] == kInterior && A.gm[n] > 1e-6; };
  const double dnx = st_diff(ok(c + 1), ok(c - 1), A.nx[c + 1], A.nx[c], A.nx[c - 1], A.i2h[0], A.ih[0]);
  const double dny = st_diff(ok(c + sx), ok(c - sx), A.ny[c + sx], A.ny[c], A.ny[c - sx], A.i2h[1], A.ih[1]);
  const double dnz = st_diff(ok(c + sxy), ok(c - sxy), A.nz[c + sxy], A.nz[c], A.nz[c - sxy], A.i2h[2], A.ih[2]);
  return -DADD(DADD(dnx, dny), dnz);
}

// Face force between cells m (low) and p (high), k_calc_surface_tension_face
// (:292-433): sigma kappa_f (alpha_p - alpha_m) / h.
__device__ __forceinline__ double st_force(double sigma, double ap, double am, double kp, double km, double ih) {
  const bool vp = ap > 1e-2 && ap < 1 - 1e-2, vm = am > 1e-2 && am < 1 - 1e-2;
  const double kf = vp && vm ? DMUL(0.5, DADD(kp, km)) : vp ? kp : vm ? km : 0.0;
  return DMUL(DMUL(DMUL(sigma, kf), DSUB(ap, am)), ih);
}

constexpr int ST_TX = 32, ST_TY = 8;

// Pass 2: curvature and face force fused.  A block owns a 32 x 8 tile of one
// plane: each thread computes its cell's curvature (stored) and the one
// below it, 40 threads also the tile's low-x column and low-y row (into a
// shared tile), and after one barrier every thread writes the three faces on
// the low side of its cell.  Cells with alpha outside [0.01, 0.99], most of
// them, cost one load per curvature, so the recomputation is cheap; a
// z-march that carried the curvature below in a register ran at a quarter of
// the occupancy (one barrier per plane, serial planes) and took 2.5x as long.
// Faces 1..N of every family are written (0 where the reference's memset
// leaves 0); the rest is k_st_rim's.
__global__ void __launch_bounds__(ST_TX* ST_TY, 4) k_st_force(StArgs A) {
  __shared__ double ks[ST_TY + 1][ST_TX + 1];
  const RefDims& R = A.R;
  const int tx = threadIdx.x, ty = threadIdx.y, t = ty * ST_TX + tx;
  const int x0 = blockIdx.x * ST_TX, y0 = blockIdx.y * ST_TY, iz = blockIdx.z + 1;
  const int ix = x0 + tx + 1, iy = y0 + ty + 1;
  const bool in = ix <= R.Nx && iy <= R.Ny;
  // the extra cell: column x0 (rows y0+1..y0+8) or row y0 (columns x0+1..x0+32)
  const bool hcol = t < ST_TY, hrow = t >= ST_TY && t < ST_TY + ST_TX;
  const int hx = hcol ? x0 : x0 + 1 + (t - ST_TY), hy = hcol ? y0 + 1 + t : y0;
  const bool hin = (hcol || hrow) && hx >= 1 && hx <= R.Nx && hy >= 1 && hy <= R.Ny;
  const long long sx = R.Nx + 2, sxy = sx * (R.Ny + 2);
  double k = 0.0, kb = 0.0, a0 = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
  bool fx = false, fy = false, fz = false;
  long long c = 0;
  if (in) {
    // everything the faces need but the shared tile, before the barrier
    c = R.cell(ix, iy, iz);
    const bool c0 = A.ct[c] == kInterior;
    fx = ix >= 2 && c0 && A.ct[c - 1] == kInterior;
    fy = iy >= 2 && c0 && A.ct[c - sx] == kInterior;
    fz = iz >= 2 && c0 && A.ct[c - sxy] == kInterior;
    a0 = A.alpha[c];
    ax = A.alpha[c - 1];
    ay = A.alpha[c - sx];
    az = A.alpha[c - sxy];
    k = st_kappa(A, ix, iy, iz);
    if (fz) kb = st_kappa(A, ix, iy, iz - 1);
    A.kappa[c] = k;
  }
  ks[ty + 1][tx + 1] = k;
  if (hcol || hrow) {
    const double kh = hin ? st_kappa(A, hx, hy, iz) : 0.0;
    if (hcol) ks[t + 1][0] = kh;
    else ks[0][t - ST_TY + 1] = kh;
  }
  __syncthreads();
  if (!in) return;
  A.fs[0][R.xf(ix, iy, iz)] = fx ? st_force(A.sigma, a0, ax, k, ks[ty + 1][tx], A.ih[0]) : 0.0;
  A.fs[1][R.yf(ix, iy, iz)] = fy ? st_force(A.sigma, a0, ay, k, ks[ty][tx + 1], A.ih[1]) : 0.0;
  A.fs[2][R.zf(ix, iy, iz)] = fz ? st_force(A.sigma, a0, az, k, kb, A.ih[2]) : 0.0;
}

// Zero of every face outside the box 1..N of each family (the part of the
// reference's memset that k_st_force does not overwrite).  blockIdx.y:
// family * 3 + group; group 0 the planes z outside 1..Nz, group 1 the rows y
// outside 1..Ny of planes 1..Nz, group 2 the entries x outside 1..Nx of the
// remaining rows.  An axis of S entries has S - N outside indices: 0 and
// N+1 .. S-1.
__global__ void __launch_bounds__(256) k_st_rim(StArgs A) {
  const RefDims& R = A.R;
  const int f = blockIdx.y / 3, grp = blockIdx.y % 3;
  const uint32_t B0 = R.Nx, B1 = R.Ny, B2 = R.Nz;
  const uint32_t S0 = B0 + 2 + (f == 0), S1 = B1 + 2 + (f == 1), S2 = B2 + 2 + (f == 2);
  const uint32_t o0 = S0 - B0, o1 = S1 - B1, o2 = S2 - B2;
  const uint32_t total = grp == 0 ? o2 * S0 * S1 : grp == 1 ? B2 * o1 * S0 : B2 * B1 * o0;
  double* fs = A.fs[f];
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < total; u += gridDim.x * blockDim.x) {
    uint32_t x, y, z;
    if (grp == 0) {
      const uint32_t zi = u / (S0 * S1), r = u - zi * (S0 * S1);
      z = zi == 0 ? 0 : B2 + zi;
      y = r / S0;
      x = r - y * S0;
    } else if (grp == 1) {
      const uint32_t zi = u / (o1 * S0), r = u - zi * (o1 * S0), yi = r / S0;
      z = 1 + zi;
      y = yi == 0 ? 0 : B1 + yi;
      x = r - yi * S0;
    } else {
      const uint32_t zi = u / (B1 * o0), r = u - zi * (B1 * o0), yi = r / o0, xi = r - yi * o0;
      z = 1 + zi;
      y = 1 + yi;
      x = xi == 0 ? 0 : B0 + xi;
    }
    fs[((long long)z * S1 + y) * S0 + x] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// Momentum predictor u* (G_SMACSolver::get_vof_vstar_rhouu_consistent,
// k_get_vof_vstar_rhouu_consistent_{x,y,z}, CFD/G_SMACSolver.cu:90-1070,
// boundary rules CFD/G_BoundaryFunctions.h:9-367)

// Offsets into the predictor's and the mass flux's arrays are 32-bit: a grid
// must keep every array below 2^31 entries (index_fits).  That bound is not a
// practical limit here: the predictor's two dozen FP64 input arrays of a grid
// that large would need more than 400 GB.  32-bit offsets cut the kernel's
// registers and spills (80 instead of 164 bytes of spill stores) and its time
// at 256^3 from 3.31 to 3.14 ms.
struct MomArgs {
  int N[3];
  const uint8_t* ft[3];
  const uint8_t* id[3];
  const double* lam[3];  // nullptr: 0
  const double* v[3];
  const double* mf[3];
  const double* muf[3];
  const double* mu;
  const double* rho_old;
  const double* p;
  const double* fb[3];   // f_b (one-way) or f_inv_rho (two-way)
  const double* imp[3];  // nullptr: 0
  const double* sf[3];   // nullptr: 0
  const double* eps_old;  // two-way only: void_fraction_old_, void_fraction_
  const double* eps_new;
  double* vs[3];
  double dt, g[3], ih[3], ih2[3], inv_volume;
  int st[4][3];  // index strides along x, y, z of the three face families and (3) the cells
  BcTable bc;
};

// d_get_v{B}_{B}face (G_BoundaryFunctions.h:9-98): family-B velocity at
// face f, boundary faces by their type; the x rule passes the stored value
// through for outlets only, the y and z rules for slip too.
// The value is loaded with the type, not after it: every face index of the
// family holds one, and the common case (F_INTERIOR) then costs one round
// trip instead of two dependent ones.
template <int B>
__device__ __forceinline__ double m_face_val(const MomArgs& A, int f) {
  const uint8_t t = A.ft[B][f];
  const double v = A.v[B][f];
  if (t == 0) return v;  // F_INTERIOR
  if (t == 1) {          // F_BOUNDARY
    const int bid = A.id[B][f];
    const uint8_t bt = A.bc.type[bid];
    if (bt == 2) return DMUL(DSUB(1.0, A.lam[B] ? A.lam[B][f] : 0.0), A.bc.bv[B][bid]);
    if (bt == 0) return 0.0;
    if (bt == 4 || (B != 0 && bt == 1)) return v;
  }
  return 0.0;
}

// d_get_v{AF}_{D}dir (G_BoundaryFunctions.h:100-367): family-AF velocity
// next to a face along D != AF on side s, mirrored about a wall.  fa, fd:
// the face's index in the family-AF and family-D layouts.
template <int AF, int D>
__device__ __forceinline__ double m_dir_val(const MomArgs& A, int fa, int fd, int s) {
  const int f2 = s > 0 ? fa + A.st[AF][D] : fa - A.st[AF][D];
  const double v2 = A.v[AF][f2];  // loaded with its type (see m_face_val)
  if (A.ft[AF][f2] == 0) return v2;
  const double inside = A.v[AF][fa];
  const int ff = s > 0 ? fd + A.st[D][D] : fd, fg = ff - A.st[D][AF];
  double wall = 0.0;
  int count = 0;
  if (A.ft[D][ff] == 1) {
    wall = DADD(wall, A.bc.bv[AF][A.id[D][ff]]);
    ++count;
  }
  if (A.ft[D][fg] == 1) {
    wall = DADD(wall, A.bc.bv[AF][A.id[D][fg]]);
    ++count;
  }
  if (count > 0) wall = __ddiv_rn(wall, (double)count);
  const uint8_t bt = A.bc.type[A.id[D][ff]];
  if (bt == 1 || bt == 4) return inside;
  return DSUB(DMUL(2.0, wall), inside);
}

__device__ __forceinline__ double m_minmod(double dp, double dm) {
  if (DMUL(dp, dm) > 0.0) return fabs(dp) < fabs(dm) ? dp : dm;
  return 0.0;
}

// The two other axes of AF in ascending order, as compile-time values.
template <int AF> struct Others { static constexpr int D0 = AF == 0 ? 1 : 0, D1 = AF == 2 ? 1 : 2; };

// Two-way form: eps_old averaged over the four cells around the edge on
// side s along D of the family-AF face with high cell c: its two cells (cm,
// c) and their neighbours along D, added in ascending index order as the
// reference writes them (k_get_vof_vstar_rhouu_consistent_*_two_way,
// CFD/G_SMACSolver.cu:1610-1622, 1832-1844, 2050-2062).
template <int AF, int D>
__device__ __forceinline__ double m_eps4(const MomArgs& A, int c, int s) {
  const int sa = A.st[3][AF], sd = A.st[3][D];
  const int lc = s > 0 ? c : c - sd, lcm = lc - sa, hc = lc + sd, hcm = lcm + sd;
  const double* e = A.eps_old;
  const double sum = D > AF ? DADD(DADD(DADD(e[lcm], e[lc]), e[hcm]), e[hc]) : DADD(DADD(DADD(e[lcm], e[hcm]), e[lc]), e[hc]);
  return DMUL(0.25, sum);
}

// Viscous cross term of axis D: (tau_D+ - tau_D-) / h_D, each stress times
// its edge's eps_old in the two-way form.  b: the face's indices in the
// three family layouts and (b[3]) its high cell; vdp, vdm: its mirrored
// neighbours along D.
template <int AF, int D, bool TW>
__device__ __forceinline__ double m_cross(const MomArgs& A, const int* b, double v0, double vdp, double vdm) {
  const int qd = b[D] + A.st[D][D], qda = qd - A.st[D][AF], q = b[D], qm = b[D] - A.st[D][AF];
  const double wp0 = m_face_val<D>(A, qd), wpm = m_face_val<D>(A, qda);
  const double w0 = m_face_val<D>(A, q), wm = m_face_val<D>(A, qm);
  const double mup = DMUL(0.5, DADD(A.muf[D][qd], A.muf[D][qda]));
  const double tp = DMUL(mup, DADD(DMUL(DSUB(wp0, wpm), A.ih[AF]), DMUL(DSUB(vdp, v0), A.ih[D])));
  const double mum = DMUL(0.5, DADD(A.muf[D][q], A.muf[D][qm]));
  const double tm = DMUL(mum, DADD(DMUL(DSUB(w0, wm), A.ih[AF]), DMUL(DSUB(v0, vdm), A.ih[D])));
  if (TW) return DMUL(DSUB(DMUL(m_eps4<AF, D>(A, b[3], +1), tp), DMUL(m_eps4<AF, D>(A, b[3], -1), tm)), A.ih[D]);
  return DMUL(DSUB(tp, tm), A.ih[D]);
}

// The neighbour two faces away along D on side s (the one value the MUSCL
// reconstruction at an upwind neighbour needs that the face's own
// stencil does not hold): the face rule along AF, the mirrored rule across.
template <int AF, int D>
__device__ __forceinline__ double m_far(const MomArgs& A, const int* b, int s) {
  if (D == AF) return m_face_val<AF>(A, b[AF] + 2 * s * A.st[AF][AF]);
  const int fa = b[AF] + s * A.st[AF][D], fd = b[D] + s * A.st[D][D];
  return m_dir_val<AF, D == AF ? Others<AF>::D0 : D>(A, fa, fd, s);
}

__device__ __forceinline__ double m_muscl(double upwind_v, double flux, double su) {
  const double dir = flux < 0.0 ? -1.0 : 1.0;
  return DADD(upwind_v, DMUL(DMUL(dir, 0.5), su));
}

// Convection through the two D-sides of the control volume, (M+ - M-)/h_D,
// with MUSCL (minmod) values at the upwind faces (k_get_vof_vstar_* :150-290).
// np, nm: the face's neighbours along D.  At the face itself the limiter
// uses np and nm; at an F_INTERIOR upwind neighbour its value is np (or nm),
// its inner neighbour the face itself, its outer one m_far; a neighbour
// that is not F_INTERIOR gives its value unlimited.
template <int AF, int D>
__device__ __forceinline__ double m_conv(const MomArgs& A, const int* b, double v0, double np, double nm) {
  double fp, fm;
  if (D == AF) {
    const int f = b[AF], s = A.st[AF][AF];
    fp = DMUL(0.5, DADD(A.mf[AF][f], A.mf[AF][f + s]));
    fm = DMUL(0.5, DADD(A.mf[AF][f - s], A.mf[AF][f]));
  } else {
    const int qd = b[D] + A.st[D][D], qda = qd - A.st[D][AF];
    fp = DMUL(0.5, DADD(A.mf[D][qda], A.mf[D][qd]));
    fm = DMUL(0.5, DADD(A.mf[D][b[D]], A.mf[D][b[D] - A.st[D][AF]]));
  }
  const double su0 = (fp > 0.0 || !(fm > 0.0)) ? m_minmod(DSUB(np, v0), DSUB(v0, nm)) : 0.0;
  double up, um;
  if (fp > 0.0) {
    up = m_muscl(v0, fp, su0);
  } else if (A.ft[AF][b[AF] + A.st[AF][D]] == 0) {
    up = m_muscl(np, fp, m_minmod(DSUB(m_far<AF, D>(A, b, +1), np), DSUB(np, v0)));
  } else {
    up = np;
  }
  if (!(fm > 0.0)) {
    um = m_muscl(v0, fm, su0);
  } else if (A.ft[AF][b[AF] - A.st[AF][D]] == 0) {
    um = m_muscl(nm, fm, m_minmod(DSUB(v0, nm), DSUB(nm, m_far<AF, D>(A, b, -1))));
  } else {
    um = nm;
  }
  return DMUL(DSUB(DMUL(fp, up), DMUL(fm, um)), A.ih[D]);
}

// u* of the F_INTERIOR family-AF face with indices b[0..2] in the family
// layouts and b[3] in the cells.  TW: the two-way-coupled form
// (k_get_vof_vstar_rhouu_consistent_{x,y,z}_two_way, CFD/G_SMACSolver.cu:
// 1538-2194): the stresses and the pressure gradient weighted by eps_old,
// u* = (f_inv_rho / eps_new_f)(eps_old_f rho_old_f u + dt (...) + impulse/V) + dt g.
template <int AF, bool TW>
__device__ __forceinline__ double m_vstar(const MomArgs& A, const int* b) {
  constexpr int D0 = Others<AF>::D0, D1 = Others<AF>::D1;
  const int f = b[AF], c = b[3], cm = b[3] - A.st[3][AF];
  const double v0 = A.v[AF][f];
  const double vp = m_face_val<AF>(A, f + A.st[AF][AF]), vm = m_face_val<AF>(A, f - A.st[AF][AF]);
  const double p0 = m_dir_val<AF, D0>(A, f, b[D0], +1), m0 = m_dir_val<AF, D0>(A, f, b[D0], -1);
  const double p1 = m_dir_val<AF, D1>(A, f, b[D1], +1), m1 = m_dir_val<AF, D1>(A, f, b[D1], -1);
  // viscous: the own axis, then the other two in axis order
  const double tau_p = DMUL(A.mu[c], DSUB(vp, v0));
  const double tau_m = DMUL(A.mu[cm], DSUB(v0, vm));
  double tmp = TW ? DMUL(DMUL(2.0, DSUB(DMUL(A.eps_old[c], tau_p), DMUL(A.eps_old[cm], tau_m))), A.ih2[AF])
                  : DMUL(DMUL(2.0, DSUB(tau_p, tau_m)), A.ih2[AF]);
  tmp = DADD(tmp, m_cross<AF, D0, TW>(A, b, v0, p0, m0));
  tmp = DADD(tmp, m_cross<AF, D1, TW>(A, b, v0, p1, m1));
  // convection in axis order
  const double npx = AF == 0 ? vp : (D0 == 0 ? p0 : p1), nmx = AF == 0 ? vm : (D0 == 0 ? m0 : m1);
  const double npy = AF == 1 ? vp : (D0 == 1 ? p0 : p1), nmy = AF == 1 ? vm : (D0 == 1 ? m0 : m1);
  const double npz = AF == 2 ? vp : p1, nmz = AF == 2 ? vm : m1;
  tmp = DSUB(tmp, m_conv<AF, 0>(A, b, v0, npx, nmx));
  tmp = DSUB(tmp, m_conv<AF, 1>(A, b, v0, npy, nmy));
  tmp = DSUB(tmp, m_conv<AF, 2>(A, b, v0, npz, nmz));
  const double inv_rho = A.fb[AF][f];
  const double rho_old_f = DMUL(0.5, DADD(A.rho_old[c], A.rho_old[cm]));
  const double coupling = DMUL(A.imp[AF] ? A.imp[AF][f] : 0.0, A.inv_volume);
  double vs;
  if (TW) {
    const double eo = DMUL(0.5, DADD(A.eps_old[cm], A.eps_old[c]));
    const double en = DMUL(0.5, DADD(A.eps_new[cm], A.eps_new[c]));
    tmp = DSUB(tmp, DMUL(DMUL(eo, DSUB(A.p[c], A.p[cm])), A.ih[AF]));
    const double ier = __ddiv_rn(inv_rho, en);
    vs = DADD(DMUL(ier, DADD(DADD(DMUL(DMUL(eo, rho_old_f), v0), DMUL(A.dt, tmp)), coupling)), DMUL(A.dt, A.g[AF]));
  } else {
    tmp = DSUB(tmp, DMUL(DSUB(A.p[c], A.p[cm]), A.ih[AF]));
    vs = DADD(DMUL(inv_rho, DADD(DMUL(v0, rho_old_f), coupling)), DMUL(A.dt, DADD(DMUL(inv_rho, tmp), A.g[AF])));
  }
  return DMUL(DSUB(1.0, A.sf[AF] ? A.sf[AF][f] : 0.0), vs);
}

// One thread per face index (x, y) of plane z of the box 1..N+1;
// blockIdx.z takes SMAC_PV_ZG planes of family 0, the same planes of
// family 1, then of family 2, so that the three families of a few planes run
// together and share the arrays they all read (velocities, fluxes, cell
// fields) through L2, while an SM mostly runs one family's code at a time.
// At 256^3, groups of 1, 2, 4, 8 and 16 planes: 2.268, 2.239, 2.244, 2.307
// and 2.523 ms (two-way 2.540, 2.497, 2.507, 2.608, 2.839).  Only
// F_INTERIOR faces are written.  The kernel waits on chains of dependent
// loads (a face type, then the value it selects), so resident warps matter
// more than registers: 5 blocks per SM (48 registers,
// a few spills to L1) measured 3.32 ms at 256^3 with 64-bit offsets (3.14 ms
// with the 32-bit ones now used), against 3.60 ms with 4 blocks, 4.27 ms
// with 3 and 3.43 ms with 6.  Family-major block order (all
// planes of one family, then the next, so that resident warps share one
// family's code) took 3.64 ms: the interleaved families' shared reads
// through L2 are worth more than the instruction-cache locality.  Block
// shapes of 256 faces at 256^3: 32 x 8 2.28 ms, 64 x 4 2.32, 16 x 16 2.37,
// 128 x 2 2.50 (two-way 2.56, 2.62, 2.65, 2.85).
#ifndef SMAC_PV_BX
#define SMAC_PV_BX 32  // predictor block: SMAC_PV_BX x (256 / SMAC_PV_BX) faces of one plane
#endif
#ifndef SMAC_PV_ZG
#define SMAC_PV_ZG 2  // planes per family group: blockIdx.z runs G planes of family 0, then of 1, then of 2
#endif
constexpr int kPvBx = SMAC_PV_BX, kPvBy = 256 / SMAC_PV_BX, kPvZg = SMAC_PV_ZG;
static_assert(kPvBx * kPvBy == 256, "the predictor's block has 256 threads");
template <bool TW>
__global__ void __launch_bounds__(256, 5) k_predict_vstar(MomArgs A) {
  const int q = blockIdx.z % (3 * kPvZg);
  const int fam = q / kPvZg;
  const int z = blockIdx.z / (3 * kPvZg) * kPvZg + q % kPvZg + 1;
  const int x = blockIdx.x * kPvBx + threadIdx.x + 1, y = blockIdx.y * kPvBy + threadIdx.y + 1;
  if (x > A.N[0] + 1 || y > A.N[1] + 1 || z > A.N[2] + 1) return;
  int b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) b[k] = x * A.st[k][0] + y * A.st[k][1] + z * A.st[k][2];
  if (fam == 0) {
    if (A.ft[0][b[0]] == 0) A.vs[0][b[0]] = m_vstar<0, TW>(A, b);
  } else if (fam == 1) {
    if (A.ft[1][b[1]] == 0) A.vs[1][b[1]] = m_vstar<1, TW>(A, b);
  } else {
    if (A.ft[2][b[2]] == 0) A.vs[2][b[2]] = m_vstar<2, TW>(A, b);
  }
}

// ---------------------------------------------------------------------------
// Property update (G_SMACSolver::update_properties_by_alpha,
// CFD/G_SMACSolver_VoF.cu:1241-1566)

struct PropArgs {
  RefDims R;
  const double* alpha;
  const uint8_t* ct;
  const uint8_t* ft[3];
  double* rho;
  double* inv_rho;  // nullptr: not written
  double* mu;
  double* fb[3];
  double* fir[3];   // nullptr: not written
  double* frho[3];  // nullptr: not written
  double* fmu[3];
  double rho0, rho1, mu0, mu1;
};

struct RhoMu {
  double r, m;
};

// rho = (1 - a) rho0 + a rho1, mu = (1 - a) mu0 + a mu1 (:1397-1405)
__device__ __forceinline__ RhoMu props_mix(const PropArgs& A, double a) {
  return {DADD(DMUL(DSUB(1.0, a), A.rho0), DMUL(a, A.rho1)), DADD(DMUL(DSUB(1.0, a), A.mu0), DMUL(a, A.mu1))};
}

// rho and mu of the C_SOLID interior cell s: those of its first C_INTERIOR
// neighbour (x-, x+, y-, y+, z-, z+), 0 without one (:1313-1340).  The
// neighbour's value is the one the mixing pass gave it.  The six alphas are
// loaded with the six types, so the rule costs one round trip.
__device__ __forceinline__ RhoMu props_solid(const PropArgs& A, int s) {
  const int sx = A.R.Nx + 2, sxy = sx * (A.R.Ny + 2);
  const uint8_t t0 = __ldg(A.ct + s - 1), t1 = __ldg(A.ct + s + 1), t2 = __ldg(A.ct + s - sx),
                t3 = __ldg(A.ct + s + sx), t4 = __ldg(A.ct + s - sxy), t5 = __ldg(A.ct + s + sxy);
  const double a0 = __ldg(A.alpha + s - 1), a1 = __ldg(A.alpha + s + 1), a2 = __ldg(A.alpha + s - sx),
               a3 = __ldg(A.alpha + s + sx), a4 = __ldg(A.alpha + s - sxy), a5 = __ldg(A.alpha + s + sxy);
  if (t0 == kInterior) return props_mix(A, a0);
  if (t1 == kInterior) return props_mix(A, a1);
  if (t2 == kInterior) return props_mix(A, a2);
  if (t3 == kInterior) return props_mix(A, a3);
  if (t4 == kInterior) return props_mix(A, a4);
  if (t5 == kInterior) return props_mix(A, a5);
  return {0.0, 0.0};
}

// The final rho, mu of interior cell s (1..N in each direction) with type t
// and alpha a: mixed for C_INTERIOR / C_NEAR_BOUNDARY, the solid rule for
// C_SOLID, and unchanged for any other type (no pass writes such a cell, so
// its entries may be read while the kernel runs).
__device__ __forceinline__ RhoMu props_interior(const PropArgs& A, int s, uint8_t t, double a) {
  if (t == 0 || t == 1) return props_mix(A, a);
  if (t == kSolid) return props_solid(A, s);
  return {A.rho[s], A.mu[s]};
}

// The final rho, mu of any cell (0..N+1 in each direction): a ghost cell
// takes those of the nearest interior cell (:1345-1372; the copies of
// :1260-1311 before it are all overwritten there).
__device__ __forceinline__ RhoMu props_final(const PropArgs& A, int x, int y, int z) {
  const RefDims& R = A.R;
  const int sx_ = x == 0 ? 1 : x == R.Nx + 1 ? R.Nx : x;
  const int sy_ = y == 0 ? 1 : y == R.Ny + 1 ? R.Ny : y;
  const int sz_ = z == 0 ? 1 : z == R.Nz + 1 ? R.Nz : z;
  const int s = R.cell(sx_, sy_, sz_);
  return props_interior(A, s, __ldg(A.ct + s), __ldg(A.alpha + s));
}

// update_properties_by_alpha (:1544-1566) in one launch.  The reference runs
// five passes over the whole box, each reading what the previous one wrote:
// mix rho and mu from alpha (:1374-1407), the solid-cell rule and ghost
// copies (:1244-1343), ghost copies again (:1345-1372), then the face values
// of the three families (:1409-1535).  Every final value is a function of
// alpha and the types alone, so here one thread per index (x, y, z) of the
// box 0..N+2 computes it directly:
//   - the cell (x, y, z) if it exists (0..N+1): rho, mu (and 1/rho where the
//     mixing pass writes it) with the rules above, written once;
//   - the x-, y- and z-face at (x, y, z) (1..N+2 along the face's axis,
//     1..N+1 across): an F_INTERIOR face gets rho_f = (rho_c + rho_cm) / 2,
//     f_b = f_inv_rho = 1 / rho_f and mu_f = (mu_c + mu_cm) / 2 from its high
//     cell c = (x, y, z) and low cell cm; any other face f_b = f_inv_rho = 0.
// The low cell in x comes from the neighbouring lane (a shuffle; lane 0
// recomputes it).  The low cells in y and z are recomputed: their type and
// alpha are loaded with the thread's own, before anything else is known, so
// that in the common case (an interior cell of a mixed type) every value the
// thread needs arrives in one round trip; those loads hit L1 / L2 (the row
// and the plane before).  Nothing in rho or mu is read that the launch
// writes, so threads need no order among themselves and no barrier; alpha,
// the types and each output are touched once per element in DRAM.
// Measured at 256^3 (CUDA events, L2 flushed): 553 us against 594 us with the
// neighbours exchanged through shared memory behind a barrier, and 604 us
// with each thread marching over 8 planes with the next plane prefetched.
// 32-bit offsets (40 registers instead of 48, 6 blocks per SM instead of 5)
// then brought it to 530 us; arrays must stay below 2^31 entries.
constexpr int PR_TX = 32, PR_TY = 8;

__global__ void __launch_bounds__(PR_TX* PR_TY) k_props(PropArgs A) {
  const RefDims& R = A.R;
  const int tx = threadIdx.x;
  const int x = blockIdx.x * PR_TX + tx, y = blockIdx.y * PR_TY + threadIdx.y, z = blockIdx.z;
  const int sx = R.Nx + 2, sxy = sx * (R.Ny + 2);
  const bool cin = x <= R.Nx + 1 && y <= R.Ny + 1 && z <= R.Nz + 1;
  const bool ghost = x == 0 || y == 0 || z == 0 || x == R.Nx + 1 || y == R.Ny + 1 || z == R.Nz + 1;
  // faces at this index, and their types (loaded with the cell's own)
  const bool lo = x >= 1 && y >= 1 && z >= 1;
  const bool has[3] = {lo && x <= R.Nx + 2 && y <= R.Ny + 1 && z <= R.Nz + 1,
                       lo && x <= R.Nx + 1 && y <= R.Ny + 2 && z <= R.Nz + 1,
                       lo && x <= R.Nx + 1 && y <= R.Ny + 1 && z <= R.Nz + 2};
  const int f[3] = {((int)z * (R.Ny + 2) + y) * (sx + 1) + x, ((int)z * (R.Ny + 3) + y) * sx + x,
                          (int)z * sxy + (int)y * sx + x};
  const int c = f[2];
  uint8_t t[3];
#pragma unroll
  for (int F = 0; F < 3; ++F) t[F] = has[F] ? __ldg(A.ft[F] + f[F]) : (uint8_t)1;
  uint8_t tc = 0, ty_ = 2, tz_ = 2;
  double ac = 0.0, ay_ = 0.0, az_ = 0.0;
  if (cin) {
    tc = __ldg(A.ct + c);
    ac = __ldg(A.alpha + c);
    // the cells below in y and z, loaded now: when they are interior cells
    // of a mixed type (the common case) their values need no second trip
    if (y >= 1 && x >= 1 && z >= 1) {
      ty_ = __ldg(A.ct + c - sx);
      ay_ = __ldg(A.alpha + c - sx);
      tz_ = __ldg(A.ct + c - sxy);
      az_ = __ldg(A.alpha + c - sxy);
    }
  }
  RhoMu v = {0.0, 0.0};
  if (cin) v = ghost ? props_final(A, x, y, z) : props_interior(A, c, tc, ac);

  const double xr = __shfl_up_sync(0xffffffffu, v.r, 1), xm = __shfl_up_sync(0xffffffffu, v.m, 1);

  if (cin) {
    if (ghost) {
      A.rho[c] = v.r;
      A.mu[c] = v.m;
      // the mixing pass covers 1..N+1: its 1/rho of a cell on the high ghost
      // layers stays (the ghost passes copy rho and mu only)
      if (A.inv_rho && lo && (tc == 0 || tc == 1)) A.inv_rho[c] = __ddiv_rn(1.0, props_mix(A, ac).r);
    } else if (tc == 0 || tc == 1) {
      A.rho[c] = v.r;
      if (A.inv_rho) A.inv_rho[c] = __ddiv_rn(1.0, v.r);
      A.mu[c] = v.m;
    } else if (tc == kSolid) {
      A.rho[c] = v.r;
      A.mu[c] = v.m;
    }
  }
#pragma unroll
  for (int F = 0; F < 3; ++F) {
    if (!has[F]) continue;
    // (a face at N+2 has no cell on its high side: typed F_INTERIOR it would
    // be invalid input, and it is treated as a wall face)
    if (t[F] != 0 || !cin) {
      A.fb[F][f[F]] = 0.0;
      if (A.fir[F]) A.fir[F][f[F]] = 0.0;
      continue;
    }
    RhoMu w;
    if (F == 0)
      w = tx > 0 ? RhoMu{xr, xm} : props_final(A, x - 1, y, z);
    else if (F == 1)
      w = (y >= 2 && y - 1 <= R.Ny && x <= R.Nx && z <= R.Nz && (ty_ == 0 || ty_ == 1)) ? props_mix(A, ay_)
                                                                                        : props_final(A, x, y - 1, z);
    else
      w = (z >= 2 && z - 1 <= R.Nz && x <= R.Nx && y <= R.Ny && (tz_ == 0 || tz_ == 1)) ? props_mix(A, az_)
                                                                                        : props_final(A, x, y, z - 1);
    const double fr = DMUL(0.5, DADD(v.r, w.r));
    if (A.frho[F]) A.frho[F][f[F]] = fr;
    const double b = __ddiv_rn(1.0, fr);
    A.fb[F][f[F]] = b;
    if (A.fir[F]) A.fir[F][f[F]] = b;
    A.fmu[F][f[F]] = DMUL(0.5, DADD(v.m, w.m));
  }
}

// ---------------------------------------------------------------------------
// Advecting mass flux from the accumulated volume-fraction flux
// (G_SMACSolver::compute_mass_flux_from_alpha_flux, k_compute_mass_flux_from_alpha_flux,
// CFD/G_SMACSolver_VoF.cu:1708-1795; two-way form
// k_compute_mass_flux_from_alpha_flux_two_way :2472-2687): on every face of
// the three families mf = rho0 q + (rho1 - rho0) F_accum h / dt with q the
// face velocity by the boundary face rule (m_face_val).  Two-way: q = eps_f
// u_f with eps_f the mean void_fraction_half_ of the face's cells (the first
// and last faces along the axis take their one interior cell's), and the
// faces at 0 and N+2 along the axis get 0.

struct FluxArgs {
  MomArgs M;            // ft, id, lam, v and the boundary table of the face rule
  const double* Fa[3];  // f_F*_accum_
  const double* epsh;   // void_fraction_half_ (two-way); nullptr: the one-way form
  double* mf[3];
  double rho0, drho, hdt[3];  // h_d / dt as the reference forms it: h_d * (1 / dt)
};

template <int F, bool TW>
__device__ __forceinline__ void flux_face(const FluxArgs& A, int x, int y, int z) {
  const MomArgs& M = A.M;
  const int f = x * M.st[F][0] + y * M.st[F][1] + z * M.st[F][2];
  const double aq = DMUL(A.Fa[F][f], A.hdt[F]);
  double q = m_face_val<F>(M, f);
  if (TW) {
    const int along = F == 0 ? x : F == 1 ? y : z, n = M.N[F];
    if (along < 1 || along > n + 1) {
      A.mf[F][f] = 0.0;
      return;
    }
    const int c = x * M.st[3][0] + y * M.st[3][1] + z * M.st[3][2], s = M.st[3][F];
    const double e = along == 1 ? A.epsh[c] : along == n + 1 ? A.epsh[c - s] : DMUL(0.5, DADD(A.epsh[c - s], A.epsh[c]));
    q = DMUL(e, q);
  }
  A.mf[F][f] = DADD(DMUL(A.rho0, q), DMUL(A.drho, aq));
}

// One thread per index (x, y, z) of the box 0..N+2 writes the x-, y- and
// z-face there (each family over its own extent).
template <bool TW>
__global__ void __launch_bounds__(256) k_mass_flux(FluxArgs A) {
  const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  const int nx = A.M.N[0], ny = A.M.N[1], nz = A.M.N[2];
  if (x <= nx + 2 && y <= ny + 1 && z <= nz + 1) flux_face<0, TW>(A, x, y, z);
  if (x <= nx + 1 && y <= ny + 2 && z <= nz + 1) flux_face<1, TW>(A, x, y, z);
  if (x <= nx + 1 && y <= ny + 1 && z <= nz + 2) flux_face<2, TW>(A, x, y, z);
}

// ---------------------------------------------------------------------------
// Two-way Poisson coefficients (G_CFDDEMCoupling::update_poisson_beta_two_way,
// k_update_poisson_beta_two_way, Coupling/G_CFDDEMCoupling.cu:419-460):
// f_b = eps_f f_inv_rho with eps_f the mean void fraction of the face's two
// cells, on x-faces 1..Nx+1 x 1..Ny x 1..Nz and likewise for y and z.  One
// thread per index (x, y, z) of the box 1..N+1 writes the faces there; the
// void fractions of the cell and its three low neighbours come through L1.
__global__ void __launch_bounds__(256) k_beta_two_way(RefDims R, const double* __restrict__ eps, const double* firx,
                                                      const double* firy, const double* firz, double* fbx, double* fby,
                                                      double* fbz) {
  const int x = blockIdx.x * 32 + threadIdx.x + 1, y = blockIdx.y * 8 + threadIdx.y + 1, z = blockIdx.z + 1;
  if (x > R.Nx + 1 || y > R.Ny + 1) return;
  const long long c = R.cell(x, y, z), sx = R.Nx + 2, sxy = sx * (R.Ny + 2);
  const double e = __ldg(eps + c);
  if (y <= R.Ny && z <= R.Nz) {
    const long long f = R.xf(x, y, z);
    fbx[f] = DMUL(DMUL(0.5, DADD(__ldg(eps + c - 1), e)), firx[f]);
  }
  if (x <= R.Nx && z <= R.Nz) {
    const long long f = R.yf(x, y, z);
    fby[f] = DMUL(DMUL(0.5, DADD(__ldg(eps + c - sx), e)), firy[f]);
  }
  if (x <= R.Nx && y <= R.Ny) {
    const long long f = R.zf(x, y, z);
    fbz[f] = DMUL(DMUL(0.5, DADD(__ldg(eps + c - sxy), e)), firz[f]);
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

void fill_table(BcTable* t, const smac_boundary_table* bc) {
  std::memset(t, 0, sizeof(*t));
  std::memcpy(t->type, bc->type, (size_t)bc->num_ids);
  for (int k = 0; k < bc->num_ids; ++k) {
    t->bv[0][k] = bc->vx[k];
    t->bv[1][k] = bc->vy[k];
    t->bv[2][k] = bc->vz[k];
  }
}

bool bad_table(const smac_boundary_table* bc, const char* fn) {
  if (bc->num_ids < 1 || bc->num_ids > kMaxIds || !bc->type || !bc->vx || !bc->vy || !bc->vz) {
    smac::set_error_text("%s: boundary table needs 1..%d ids and its four arrays", fn, kMaxIds);
    return true;
  }
  return false;
}

// Every face and cell array of the grid has fewer than 2^31 entries (the
// predictor and the mass flux index them with 32-bit offsets).
bool index_fits(const smac_grid_desc* d, const char* fn) {
  for (int k = 0; k < 3; ++k) {
    const long long n = (long long)(d->nx + 2 + (k == 0)) * (d->ny + 2 + (k == 1)) * (d->nz + 2 + (k == 2));
    if (n > 0x7fffffffLL) {
      smac::set_error_text("%s: grid %d x %d x %d: a face array would exceed 2^31 - 1 entries", fn, d->nx, d->ny,
                           d->nz);
      return false;
    }
  }
  return true;
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
  A.shape = make_shape2(sx, sy, A.ncell);
  A.scan_blocks = scan_blocks_for(A.ncell, sm_count());
  A.gz_bx = (int)((sx + 31) / 32); A.gz_by = (int)((sy + 7) / 8);
  A.gy_bx = (int)((sx + 31) / 32); A.gy_bz = (d->nz + 7) / 8;
  A.gx_by = (d->ny + 31) / 32;     A.gx_bz = (d->nz + 7) / 8;
  const long long ghost_blocks = 2LL * (A.gz_bx * A.gz_by + A.gy_bx * A.gy_bz + A.gx_by * A.gx_bz);
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
  if (bad_table(bc, fn)) return SMAC_BAD_ARG;
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
    O.shape[0] = make_shape2(X + 3, Y + 2, O.n[0]);
    O.shape[1] = make_shape2(X + 2, Y + 3, O.n[1]);
    O.shape[2] = make_shape2(X + 2, Y + 2, O.n[2]);
    const long long nmax = O.n[0] > O.n[1] ? (O.n[0] > O.n[2] ? O.n[0] : O.n[2]) : (O.n[1] > O.n[2] ? O.n[1] : O.n[2]);
    k_velocity_outlet<<<dim3(scan_blocks_for(nmax, sm_count()), 3), kPostThreads, 0, s>>>(O);
    const smac_status st = launch_status(fn);
    if (st != SMAC_OK) return st;
  }
  GhostArgs G;
  std::memset(&G, 0, sizeof(G));
  G.N[0] = d->nx; G.N[1] = d->ny; G.N[2] = d->nz;
  G.bcid[0] = fxbcid; G.bcid[1] = fybcid; G.bcid[2] = fzbcid;
  G.lam[0] = lamx; G.lam[1] = lamy; G.lam[2] = lamz;
  G.v[0] = vx; G.v[1] = vy; G.v[2] = vz;
  fill_table(&G.bc, bc);
  const long long longest = (X > Y ? (X > Z ? X : Z) : (Y > Z ? Y : Z)) + 1;
  const long long per_slab = longest * longest;
  const long long want = (per_slab + kPostThreads - 1) / kPostThreads;
  const int blocks = (int)(want < 1024 ? want : 1024);
  k_velocity_ghost<<<dim3(blocks, 5, 3), kPostThreads, 0, s>>>(G);
  return launch_status(fn);
}

smac_status smac_update_vstar_boundary(const smac_grid_desc* d, const smac_boundary_table* bc, const uint8_t* fxt,
                                      const uint8_t* fyt, const uint8_t* fzt, const uint8_t* fxbcid,
                                      const uint8_t* fybcid, const uint8_t* fzbcid, const uint8_t* fxo,
                                      const uint8_t* fyo, const uint8_t* fzo, const double* lamx, const double* lamy,
                                      const double* lamz, double* vxs, double* vys, double* vzs, void* stream) {
  static const char* fn = "smac_update_vstar_boundary";
  if (!d || !bc || !fxt || !fyt || !fzt || !fxbcid || !fybcid || !fzbcid || !vxs || !vys || !vzs) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bad_table(bc, fn)) return SMAC_BAD_ARG;
  if (bad_desc(d, fn, 1)) return SMAC_BAD_SHAPE;
  const long long X = d->nx, Y = d->ny, Z = d->nz;
  VstarArgs V;
  V.R = RefDims{d->nx, d->ny, d->nz};
  V.ft[0] = fxt; V.ft[1] = fyt; V.ft[2] = fzt;
  V.bcid[0] = fxbcid; V.bcid[1] = fybcid; V.bcid[2] = fzbcid;
  V.mark[0] = fxo; V.mark[1] = fyo; V.mark[2] = fzo;
  V.lam[0] = lamx; V.lam[1] = lamy; V.lam[2] = lamz;
  V.vs[0] = vxs; V.vs[1] = vys; V.vs[2] = vzs;
  V.n[0] = (X + 3) * (Y + 2) * (Z + 2);
  V.n[1] = (X + 2) * (Y + 3) * (Z + 2);
  V.n[2] = (X + 2) * (Y + 2) * (Z + 3);
  V.shape[0] = make_shape2(X + 3, Y + 2, V.n[0]);
  V.shape[1] = make_shape2(X + 2, Y + 3, V.n[1]);
  V.shape[2] = make_shape2(X + 2, Y + 2, V.n[2]);
  fill_table(&V.bc, bc);
  const long long nmax = V.n[0] > V.n[1] ? (V.n[0] > V.n[2] ? V.n[0] : V.n[2]) : (V.n[1] > V.n[2] ? V.n[1] : V.n[2]);
  k_vstar_boundary<<<dim3(scan_blocks_for(nmax, sm_count()), 3), kPostThreads, 0, (cudaStream_t)stream>>>(V);
  return launch_status(fn);
}

smac_status smac_surface_tension(const smac_grid_desc* d, const double* alpha, const uint8_t* celltype, double sigma,
                                 double* nx, double* ny, double* nz, double* kappa, double* grad_mag, double* fsx,
                                 double* fsy, double* fsz, void* stream) {
  static const char* fn = "smac_surface_tension";
  if (!d || !alpha || !celltype || !nx || !ny || !nz || !kappa || !grad_mag || !fsx || !fsy || !fsz) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bad_desc(d, fn, 1)) return SMAC_BAD_SHAPE;
  StArgs A;
  A.R = RefDims{d->nx, d->ny, d->nz};
  A.alpha = alpha;
  A.ct = celltype;
  A.nx = nx; A.ny = ny; A.nz = nz;
  A.kappa = kappa;
  A.gm = grad_mag;
  A.fs[0] = fsx; A.fs[1] = fsy; A.fs[2] = fsz;
  A.sigma = sigma;
  const double h[3] = {d->dx, d->dy, d->dz};
  for (int k = 0; k < 3; ++k) {
    A.ih[k] = 1. / h[k];
    A.i2h[k] = 1. / (2. * h[k]);
  }
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned bx = (unsigned)((d->nx + ST_TX - 1) / ST_TX), by = (unsigned)((d->ny + ST_TY - 1) / ST_TY);
  k_st_rim<<<dim3(64, 9), 256, 0, s>>>(A);
  k_st_normal<<<dim3(bx, by, (unsigned)d->nz), dim3(32, 8), 0, s>>>(A);
  k_st_force<<<dim3(bx, by, (unsigned)d->nz), dim3(ST_TX, ST_TY), 0, s>>>(A);
  return launch_status(fn);
}

}  // extern "C"

namespace {

// The two predictor entries: tw == nullptr the one-way form with mf's f_b,
// otherwise the two-way form with tw's eps and f_inv_rho.
smac_status predict_vstar(const char* fn, const smac_grid_desc* d, const smac_boundary_table* bc,
                          const smac_momentum_fields* mf, const smac_two_way_fields* tw, double dt, double gx,
                          double gy, double gz, double* vxs, double* vys, double* vzs, void* stream) {
  if (!d || !bc || !mf || !vxs || !vys || !vzs) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  const double* const* inv_rho = tw ? &tw->inv_rhox : &mf->fbx;
  const void* need[] = {mf->fxt, mf->fyt, mf->fzt, mf->fxbcid, mf->fybcid, mf->fzbcid, mf->vx, mf->vy, mf->vz,
                        mf->mfx, mf->mfy, mf->mfz, mf->mux, mf->muy, mf->muz, mf->mu, mf->rho_old, mf->p,
                        inv_rho[0], inv_rho[1], inv_rho[2], tw ? tw->eps_old : mf->p, tw ? tw->eps_new : mf->p};
  for (const void* q : need)
    if (!q) {
      smac::set_error_text("%s: a required field is null", fn);
      return SMAC_BAD_ARG;
    }
  if (bad_table(bc, fn)) return SMAC_BAD_ARG;
  // the mirrored neighbours read two faces inside across every axis
  if (bad_desc(d, fn, 2) || !index_fits(d, fn)) return SMAC_BAD_SHAPE;
  MomArgs A;
  std::memset(&A, 0, sizeof(A));
  A.N[0] = d->nx; A.N[1] = d->ny; A.N[2] = d->nz;
  A.ft[0] = mf->fxt; A.ft[1] = mf->fyt; A.ft[2] = mf->fzt;
  A.id[0] = mf->fxbcid; A.id[1] = mf->fybcid; A.id[2] = mf->fzbcid;
  A.lam[0] = mf->lamx; A.lam[1] = mf->lamy; A.lam[2] = mf->lamz;
  A.v[0] = mf->vx; A.v[1] = mf->vy; A.v[2] = mf->vz;
  A.mf[0] = mf->mfx; A.mf[1] = mf->mfy; A.mf[2] = mf->mfz;
  A.muf[0] = mf->mux; A.muf[1] = mf->muy; A.muf[2] = mf->muz;
  A.mu = mf->mu; A.rho_old = mf->rho_old; A.p = mf->p;
  A.fb[0] = inv_rho[0]; A.fb[1] = inv_rho[1]; A.fb[2] = inv_rho[2];
  if (tw) {
    A.eps_old = tw->eps_old;
    A.eps_new = tw->eps_new;
  }
  A.imp[0] = mf->impx; A.imp[1] = mf->impy; A.imp[2] = mf->impz;
  A.sf[0] = mf->sfx; A.sf[1] = mf->sfy; A.sf[2] = mf->sfz;
  A.vs[0] = vxs; A.vs[1] = vys; A.vs[2] = vzs;
  A.dt = dt;
  A.g[0] = gx; A.g[1] = gy; A.g[2] = gz;
  const double h[3] = {d->dx, d->dy, d->dz};
  for (int k = 0; k < 3; ++k) {
    A.ih[k] = 1. / h[k];
    A.ih2[k] = 1. / (h[k] * h[k]);
  }
  A.inv_volume = A.ih[0] * A.ih[1] * A.ih[2];
  for (int k = 0; k < 4; ++k) {  // families 0..2, cells 3
    const long long S0 = d->nx + 2 + (k == 0), S1 = d->ny + 2 + (k == 1);
    A.st[k][0] = 1;
    A.st[k][1] = (int)S0;
    A.st[k][2] = (int)(S0 * S1);
  }
  fill_table(&A.bc, bc);
  const dim3 grid((unsigned)((d->nx + 1 + kPvBx - 1) / kPvBx), (unsigned)((d->ny + 1 + kPvBy - 1) / kPvBy),
                  3u * (unsigned)((d->nz + 1 + kPvZg - 1) / kPvZg * kPvZg));
  if (tw)
    k_predict_vstar<true><<<grid, dim3(kPvBx, kPvBy), 0, (cudaStream_t)stream>>>(A);
  else
    k_predict_vstar<false><<<grid, dim3(kPvBx, kPvBy), 0, (cudaStream_t)stream>>>(A);
  return launch_status(fn);
}

}  // namespace

extern "C" {

smac_status smac_predict_vstar(const smac_grid_desc* d, const smac_boundary_table* bc, const smac_momentum_fields* mf,
                               double dt, double gx, double gy, double gz, double* vxs, double* vys, double* vzs,
                               void* stream) {
  return predict_vstar("smac_predict_vstar", d, bc, mf, nullptr, dt, gx, gy, gz, vxs, vys, vzs, stream);
}

smac_status smac_predict_vstar_two_way(const smac_grid_desc* d, const smac_boundary_table* bc,
                                       const smac_momentum_fields* mf, const smac_two_way_fields* tw, double dt,
                                       double gx, double gy, double gz, double* vxs, double* vys, double* vzs,
                                       void* stream) {
  if (!tw) {
    smac::set_error_text("smac_predict_vstar_two_way: null argument");
    return SMAC_BAD_ARG;
  }
  return predict_vstar("smac_predict_vstar_two_way", d, bc, mf, tw, dt, gx, gy, gz, vxs, vys, vzs, stream);
}

smac_status smac_update_properties(const smac_grid_desc* d, const smac_vof_params* vp, const double* alpha,
                                   const uint8_t* celltype, const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt,
                                   const smac_property_fields* out, void* stream) {
  static const char* fn = "smac_update_properties";
  if (!d || !vp || !alpha || !celltype || !fxt || !fyt || !fzt || !out || !out->rho || !out->mu || !out->fbx ||
      !out->fby || !out->fbz || !out->mux || !out->muy || !out->muz) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bad_desc(d, fn, 1) || !index_fits(d, fn)) return SMAC_BAD_SHAPE;
  PropArgs A;
  std::memset(&A, 0, sizeof(A));
  A.R = RefDims{d->nx, d->ny, d->nz};
  A.alpha = alpha;
  A.ct = celltype;
  A.ft[0] = fxt; A.ft[1] = fyt; A.ft[2] = fzt;
  A.rho = out->rho; A.inv_rho = out->inv_rho; A.mu = out->mu;
  A.fb[0] = out->fbx; A.fb[1] = out->fby; A.fb[2] = out->fbz;
  A.fir[0] = out->firx; A.fir[1] = out->firy; A.fir[2] = out->firz;
  A.frho[0] = out->rhox; A.frho[1] = out->rhoy; A.frho[2] = out->rhoz;
  A.fmu[0] = out->mux; A.fmu[1] = out->muy; A.fmu[2] = out->muz;
  A.rho0 = vp->rho0; A.rho1 = vp->rho1; A.mu0 = vp->mu0; A.mu1 = vp->mu1;
  const dim3 grid((unsigned)((d->nx + 3 + PR_TX - 1) / PR_TX), (unsigned)((d->ny + 3 + PR_TY - 1) / PR_TY),
                  (unsigned)(d->nz + 3));
  k_props<<<grid, dim3(PR_TX, PR_TY), 0, (cudaStream_t)stream>>>(A);
  return launch_status(fn);
}

smac_status smac_mass_flux_from_alpha_flux(const smac_grid_desc* d, const smac_boundary_table* bc,
                                           const smac_mass_flux_fields* in, double rho0, double rho1, double dt,
                                           const double* eps_half, double* mfx, double* mfy, double* mfz,
                                           void* stream) {
  static const char* fn = "smac_mass_flux_from_alpha_flux";
  if (!d || !bc || !in || !mfx || !mfy || !mfz) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  const void* need[] = {in->fxt, in->fyt, in->fzt, in->fxbcid, in->fybcid, in->fzbcid,
                        in->vx, in->vy, in->vz, in->Fx, in->Fy, in->Fz};
  for (const void* q : need)
    if (!q) {
      smac::set_error_text("%s: a required field is null", fn);
      return SMAC_BAD_ARG;
    }
  if (bad_table(bc, fn)) return SMAC_BAD_ARG;
  if (bad_desc(d, fn, 1) || !index_fits(d, fn)) return SMAC_BAD_SHAPE;
  FluxArgs A;
  std::memset(&A, 0, sizeof(A));
  MomArgs& M = A.M;
  M.N[0] = d->nx; M.N[1] = d->ny; M.N[2] = d->nz;
  M.ft[0] = in->fxt; M.ft[1] = in->fyt; M.ft[2] = in->fzt;
  M.id[0] = in->fxbcid; M.id[1] = in->fybcid; M.id[2] = in->fzbcid;
  M.lam[0] = in->lamx; M.lam[1] = in->lamy; M.lam[2] = in->lamz;
  M.v[0] = in->vx; M.v[1] = in->vy; M.v[2] = in->vz;
  for (int k = 0; k < 4; ++k) {
    const long long S0 = d->nx + 2 + (k == 0), S1 = d->ny + 2 + (k == 1);
    M.st[k][0] = 1;
    M.st[k][1] = (int)S0;
    M.st[k][2] = (int)(S0 * S1);
  }
  fill_table(&M.bc, bc);
  A.Fa[0] = in->Fx; A.Fa[1] = in->Fy; A.Fa[2] = in->Fz;
  A.epsh = eps_half;
  A.mf[0] = mfx; A.mf[1] = mfy; A.mf[2] = mfz;
  A.rho0 = rho0;
  A.drho = rho1 - rho0;
  const double inv_dt = 1. / dt;
  A.hdt[0] = d->dx * inv_dt; A.hdt[1] = d->dy * inv_dt; A.hdt[2] = d->dz * inv_dt;
  const dim3 grid((unsigned)((d->nx + 3 + 31) / 32), (unsigned)((d->ny + 3 + 7) / 8), (unsigned)(d->nz + 3));
  if (eps_half)
    k_mass_flux<true><<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(A);
  else
    k_mass_flux<false><<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(A);
  return launch_status(fn);
}

smac_status smac_poisson_beta_two_way(const smac_grid_desc* d, const double* eps, const double* firx,
                                      const double* firy, const double* firz, double* fbx, double* fby, double* fbz,
                                      void* stream) {
  static const char* fn = "smac_poisson_beta_two_way";
  if (!d || !eps || !firx || !firy || !firz || !fbx || !fby || !fbz) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (bad_desc(d, fn, 1)) return SMAC_BAD_SHAPE;
  const RefDims R{d->nx, d->ny, d->nz};
  const dim3 grid((unsigned)((d->nx + 1 + 31) / 32), (unsigned)((d->ny + 1 + 7) / 8), (unsigned)(d->nz + 1));
  k_beta_two_way<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(R, eps, firx, firy, firz, fbx, fby, fbz);
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
  const dim3 grid((unsigned)((d->nx + 1 + GP_TX - 1) / GP_TX), (unsigned)((d->ny + 1 + GP_TY - 1) / GP_TY),
                  (unsigned)(d->nz + 1));
  k_face_gradp<<<grid, dim3(GP_TX, GP_TY), 0, (cudaStream_t)stream>>>(R, p, gpx, gpy, gpz, 1. / d->dx, 1. / d->dy,
                                                                      1. / d->dz);
  return launch_status(fn);
}

}  // extern "C"
