// smac_common.cuh -- layout, numeric helpers and deterministic reductions
// shared by the SMAC projection kernels (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace smac {

// Reference type codes (CFD/Enums.h:3-23).
enum : uint8_t { F_INTERIOR = 0, F_BOUNDARY = 1, F_GHOST = 2, F_NEAR_BOUNDARY = 3 };
enum : uint8_t { C_INTERIOR = 0, C_NEAR_BOUNDARY = 1, C_GHOST = 2, C_SOLID = 3 };

// ---------------------------------------------------------------------------
// Padded SoA layout of one grid level.
//
// Cells (i,j,k), 0 <= i < nx etc., and the three face families share ONE
// index map idx(i,j,k) = k*ps + j*px + i with px = roundup(nx+1, 8) and
// ps = px*(ny+1), over (nz+1) planes:
//   x-face i (low face of cell i, i = 0..nx),  y-face j (j = 0..ny),
//   z-face k (k = 0..nz) all fit in the same box.
// Every entry outside the interior (pad column i >= nx, pad row j = ny, pad
// plane k = nz) and a guard of `guard` elements in front of the origin hold
// zeros for cell arrays, so a 7-point neighbour outside the domain reads
// 0.0: exactly the reference's zero ghost (its wall coefficients are 0 for
// pure Neumann walls, and q_tmp_ ghosts are 0 on the coarse grids).
// Rows are 32-byte aligned for both float and double (px multiple of 8).
struct Geom {
  int nx, ny, nz;
  int px;        // row pitch in elements
  int py;        // rows per plane (ny + 1)
  int ps;        // plane stride px*py
  int guard;     // zero elements in front of idx(0,0,0)
  long long alloc;  // elements to allocate per array
  double ihx2, ihy2, ihz2;  // 1/h^2 of this level
  __host__ __device__ __forceinline__ int idx(int i, int j, int k) const { return k * ps + j * px + i; }
  __host__ __device__ __forceinline__ long long cells() const { return (long long)nx * ny * nz; }
};

inline Geom make_geom(int nx, int ny, int nz, double ihx2, double ihy2, double ihz2) {
  Geom g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.px = ((nx + 1) + 7) / 8 * 8;
  g.py = ny + 1;
  g.ps = g.px * g.py;
  g.guard = (g.ps + g.px + 31) / 32 * 32;
  g.alloc = (long long)g.guard + (long long)(nz + 1) * g.ps + 64;
  g.ihx2 = ihx2; g.ihy2 = ihy2; g.ihz2 = ihz2;
  return g;
}

// Coefficient storage types.
template <class C> struct CoefLoad;
template <> struct CoefLoad<double> {
  static __device__ __forceinline__ double get(const double* p, int c) { return __ldg(p + c); }
};
template <> struct CoefLoad<float> {
  static __device__ __forceinline__ float get(const float* p, int c) { return __ldg(p + c); }
};
template <> struct CoefLoad<__nv_bfloat16> {
  static __device__ __forceinline__ float get(const __nv_bfloat16* p, int c) {
    return __bfloat162float(__ldg(p + c));
  }
};
template <class C> __device__ __forceinline__ C coef_from_double(double v);
template <> __device__ __forceinline__ double coef_from_double<double>(double v) { return v; }
template <> __device__ __forceinline__ float coef_from_double<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ __nv_bfloat16 coef_from_double<__nv_bfloat16>(double v) {
  return __float2bfloat16_rn((float)v);
}

// ---------------------------------------------------------------------------
// Device-resident solver state.  Kernels read alpha/beta/shift from here and
// the last block of each reducing kernel writes the next values, so an
// iteration needs no host round trip.  `done` makes every later kernel of
// the iteration return at once.
struct Scalars {
  double rz;         // r.z of the current direction
  double pAp;        // d.A d
  double alpha;      // rz / pAp
  double beta;       // rz_new / rz
  double rr;         // ||r - mean(r)||^2 (recursive)
  double rmax;       // max |r| (recursive)
  double rshift;     // mean of r over fluid cells, removed on the fly
  double rr_anchor;  // ||r||^2 at the last FP64 residual recomputation (mixed)
  double bb;         // ||b||^2 after the zero-mean projection
  double tol2bb;     // tol^2 * bb
  double tol_max;    // tol / dt for the reference's max-norm test
  double true_rr;    // last FP64 true-residual ||r||^2
  double true_rmax;  // last FP64 true-residual max |r|
  double reliable_delta2;
  double inv_nfluid; // 1 / number of fluid cells (0 when not pure Neumann)
  double sum_tmp;    // scratch for one-off sums
  double zshift;     // mean of z = M r over fluid cells, removed in the direction update
  int iter;          // matvecs done
  int max_iter;
  int done;          // 1: converged or failed
  int status;        // smac_status
  int first;         // 1 before the first direction update
  int stop_rule;     // 0 relative L2, 1 reference max-norm
  int do_reliable;   // mixed: recompute the FP64 residual in this iteration
  int e_reset;       // mixed: the next update starts the FP32 increment from 0
  int xbuf;          // mixed: which FP64 solution buffer is current
  int reliable_count;
  int mixed;
  int pad;
};

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  The iteration's kernels are launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, so the next kernel's
// CTAs may become resident while this one drains.  Every such kernel calls
// pdl_enter() before its first global access: griddepcontrol.wait blocks
// until the preceding grid has completed and its writes are visible, so the
// ordering is that of a plain stream; launch_dependents then lets the next
// grid be scheduled as soon as every CTA of this one has started.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// L2 prefetch of `bytes` (a multiple of 16) from a 16-byte aligned address
// (a hint: nothing waits for it)
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// ---------------------------------------------------------------------------
// Deterministic grid reduction: every block reduces NV doubles in a fixed
// tree, writes them to partials[block*NV + v], and the last block to arrive
// (atomic ticket) sums the partials in a fixed order.  The result does not
// depend on block scheduling.  Returns true in the threads of the last block;
// `out` then holds the totals in every thread of that block.
struct RedBuf {
  double* partials;   // >= max_blocks * 4
  unsigned* ticket;   // one counter per reducing kernel slot, reset by the last block
};

enum class Op { Sum, Max };

template <int NV, int NT>
__device__ __forceinline__ void block_reduce(double (&v)[NV], const Op (&ops)[NV], double* sm) {
  // warp level
#pragma unroll
  for (int q = 0; q < NV; ++q) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, v[q], off);
      v[q] = (ops[q] == Op::Sum) ? v[q] + o : fmax(v[q], o);
    }
  }
  const int lane = threadIdx.x & 31;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int warp = tid >> 5;
  constexpr int NW = NT / 32;
  if ((tid & 31) == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) sm[q * NW + warp] = v[q];
  }
  (void)lane;
  __syncthreads();
  if (tid < 32) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = (tid < NW) ? sm[q * NW + tid] : (ops[q] == Op::Sum ? 0.0 : -INFINITY);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, x, off);
        x = (ops[q] == Op::Sum) ? x + o : fmax(x, o);
      }
      v[q] = x;  // valid in thread 0
    }
  }
}

template <int NV, int NT>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], const Op (&ops)[NV], RedBuf red, int slot,
                                            double (&out)[NV]) {
  __shared__ double sm[NV * (NT / 32)];
  __shared__ bool am_last;
  __shared__ double res[NV];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nblocks = gridDim.x * gridDim.y * gridDim.z;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  block_reduce<NV, NT>(v, ops, sm);
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) red.partials[(size_t)bid * NV + q] = v[q];
    __threadfence();
    const unsigned t = atomicAdd(red.ticket + slot, 1u);
    am_last = (t == (unsigned)nblocks - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  // fixed-order sum over partials: thread t takes blocks t, t+NT, ...
  double w[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) w[q] = (ops[q] == Op::Sum) ? 0.0 : -INFINITY;
  for (int b = tid; b < nblocks; b += NT) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double x = __ldcg(red.partials + (size_t)b * NV + q);
      w[q] = (ops[q] == Op::Sum) ? w[q] + x : fmax(w[q], x);
    }
  }
  __syncthreads();
  block_reduce<NV, NT>(w, ops, sm);
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) res[q] = w[q];
    red.ticket[slot] = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) out[q] = res[q];
  return true;
}

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

template <class T> struct Acc { typedef T type; };
template <class T> using acc_t = typename Acc<T>::type;


// ------------------------------------------------------------------------
// Reference-layout index helpers (MyArray<T,3>: (z*sy + y)*sx + x).
struct RefDims {
  int Nx, Ny, Nz;
  __host__ __device__ __forceinline__ long long cell(int x, int y, int z) const {
    return ((long long)z * (Ny + 2) + y) * (Nx + 2) + x;
  }
  __host__ __device__ __forceinline__ long long xf(int x, int y, int z) const {
    return ((long long)z * (Ny + 2) + y) * (Nx + 3) + x;
  }
  __host__ __device__ __forceinline__ long long yf(int x, int y, int z) const {
    return ((long long)z * (Ny + 3) + y) * (Nx + 2) + x;
  }
  __host__ __device__ __forceinline__ long long zf(int x, int y, int z) const {
    return ((long long)z * (Ny + 2) + y) * (Nx + 2) + x;
  }
};

// ------------------------------------------------------------------------
// Stencil pieces.  Every product and sum is an explicit round-to-nearest
// intrinsic, so the compiler contracts nothing on its own: every kernel that
// evaluates the same cell update rounds identically (the fused sweep equals
// the half-sweep kernels bit for bit) whatever the code around it.
template <class A> struct Ar;
// rcp(d): 1/d from the hardware's approximate reciprocal refined by
// Newton-Raphson steps y <- y + y (1 - d y) (two for FP64, one for FP32),
// for the Gauss-Seidel update, where a last-bit difference from the IEEE
// quotient only perturbs the smoother, identically in every kernel.
template <> struct Ar<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double rcp(double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = __fma_rn(-d, y, 1.0);
    y = __fma_rn(y, e, y);
    e = __fma_rn(-d, y, 1.0);
    return __fma_rn(y, e, y);
  }
};
template <> struct Ar<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float rcp(float d) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
    const float e = __fmaf_rn(-d, y, 1.0f);
    return __fmaf_rn(y, e, y);
  }
};

// The coefficient arrays hold the stencil weights w = f_b / h^2 of their
// grid (the reference's Axp/Axm/... values, G_PCGSolver.cu:168-173), so a
// cell update only loads them.
template <class T, class C>
struct Stencil {
  typedef acc_t<T> A;
  typedef Ar<A> R;
  const C* __restrict__ bx;
  const C* __restrict__ by;
  const C* __restrict__ bz;
  // face weights of cell c: x-, x+, y-, y+, z-, z+
  __device__ __forceinline__ void coeffs(int c, int px, int ps, A& wxm, A& wxp, A& wym, A& wyp, A& wzm,
                                         A& wzp) const {
    wxm = (A)CoefLoad<C>::get(bx, c);
    wxp = (A)CoefLoad<C>::get(bx, c + 1);
    wym = (A)CoefLoad<C>::get(by, c);
    wyp = (A)CoefLoad<C>::get(by, c + px);
    wzm = (A)CoefLoad<C>::get(bz, c);
    wzp = (A)CoefLoad<C>::get(bz, c + ps);
  }
  static __device__ __forceinline__ A diag(A wxm, A wxp, A wym, A wyp, A wzm, A wzp) {
    return R::add(R::add(R::add(wxm, wxp), R::add(wym, wyp)), R::add(wzm, wzp));
  }
  // bv + sum w * n (neighbours in the order x-, x+, y-, y+, z-, z+)
  static __device__ __forceinline__ A offsum(A bv, A wxm, A wxp, A wym, A wyp, A wzm, A wzp, A n0, A n1, A n2,
                                             A n3, A n4, A n5) {
    A acc = R::fma(wxm, n0, bv);
    acc = R::fma(wxp, n1, acc);
    acc = R::fma(wym, n2, acc);
    acc = R::fma(wyp, n3, acc);
    acc = R::fma(wzm, n4, acc);
    return R::fma(wzp, n5, acc);
  }
  // (A x)_c = diag x_c - sum w * n
  static __device__ __forceinline__ A apply(A xc, A wxm, A wxp, A wym, A wyp, A wzm, A wzp, A n0, A n1, A n2,
                                            A n3, A n4, A n5) {
    const A d = diag(wxm, wxp, wym, wyp, wzm, wzp);
    return offsum(R::mul(d, xc), -wxm, -wxp, -wym, -wyp, -wzm, -wzp, n0, n1, n2, n3, n4, n5);
  }
  // Gauss-Seidel value (bv + sum w * n) / diag, 0 where the diagonal is 0
  static __device__ __forceinline__ A gs(A bv, A wxm, A wxp, A wym, A wyp, A wzm, A wzp, A n0, A n1, A n2, A n3,
                                         A n4, A n5) {
    const A d = diag(wxm, wxp, wym, wyp, wzm, wzp);
    if (!(d > (A)0)) return (A)0;
    return R::mul(offsum(bv, wxm, wxp, wym, wyp, wzm, wzp, n0, n1, n2, n3, n4, n5), R::rcp(d));
  }
};

}  // namespace smac
