// smac_coarse_cluster.cuh -- the coarse grids of the V-cycle in one thread-block
// cluster, held in distributed shared memory.
//
// Below about 64^3 cells a separately launched sweep is bound by latency, not
// bytes: every grid of the V-cycle's lower half costs its launches' ramp and
// the z-march's dependent steps (about 7 us per sweep at 32^3 and at 16^3
// alike), and the single-CTA kernel for the grids of <= 4096 cells waits on L2
// at every one of its ~50 steps.  This kernel runs the whole lower part of
// the V-cycle -- from the first grid of <= 32768 cells down to the coarsest --
// in one cluster of KCL CTAs:
//   - every grid's cells, right-hand side and face weights live in shared
//     memory, the planes of a grid spread over the ranks in chunks (plane k in
//     rank k / chunk); a rank reads the x of a neighbour's plane through
//     distributed shared memory (the only remote reads) and the restriction
//     writes a coarse right-hand side into the rank that owns it;
//   - the steps of the spread grids are separated by cluster barriers, the
//     steps of the grids of <= KCL_SOLO cells, held whole by rank 0, by
//     __syncthreads in rank 0 while the other ranks wait at the next cluster
//     barrier;
//   - the chunks halve with the grids (a coarse plane is in the rank of its
//     two children), so a rank's residual and its cells' weights are local.
// The operation sequence and every operation are those of the single-CTA
// kernel (k_coarse_vcycle) and of the separately launched sweeps they
// replace (each of those equal to two half-sweeps, bit for bit), so the
// V-cycle's result is the same bit for bit.
#pragma once

#include <cooperative_groups.h>
#include <cuda_pipeline.h>

#include "smac_kernels.cuh"

namespace smac {

constexpr int KCL = 8;           // CTAs in the cluster (the portable maximum)
// threads per CTA: 512, 128 registers a thread (at 1024 the phases' state
// spills at 64 registers)
#ifndef SMAC_KCL_NT32
#define SMAC_KCL_NT32 512
#endif
template <class T> __host__ __device__ constexpr int kcl_threads() { return sizeof(T) == 8 ? 512 : SMAC_KCL_NT32; }
constexpr int KCL_SOLO = 512;    // grids of at most this many cells are held and swept by rank 0
constexpr int KCL_TOP = 32768;   // the set starts at the first grid of at most this many cells
constexpr int MAX_CLL = 12;

// One grid of the set.  Every rank lays out the same arrays at the same
// shared-memory offsets (in elements of T), sized for one chunk of planes:
//   x, rhs  chunk planes of nx*ny cells;
//   bx      chunk planes of ny rows of nx+1 x-faces;
//   by      chunk planes of ny+1 rows of nx y-faces;
//   bz      chunk+1 planes of nx*ny z-faces (also the top face of the last plane).
struct ClusterLevel {
  Geom g;             // the grid's padded layout in global memory
  int cx, cy, cz;     // how this grid was coarsened from the one above
  int chunk;          // planes per rank (nz for a grid held by rank 0)
  int ox, orhs, obx, oby, obz;
  int ctype;          // global coefficient storage: 0 FP64, 1 FP32, 2 BF16
  const void* bx;
  const void* by;
  const void* bz;
};
struct ClusterSet {
  ClusterLevel L[MAX_CLL];
  int n;        // grids in the set
  int nd;       // the first nd are spread over the ranks, the rest held by rank 0
  const void* rhs0;  // right-hand side of L[0] (global, padded layout)
  void* x0;          // its result (global, padded layout; the pads are not written)
};

// A grid of the set as the phases use it, passed by value (registers): its
// dimensions, chunk and shared-memory offsets.
struct ClGrid {
  int nx, ny, nz, chunk, ox, orhs, obx, oby, obz, cx, cy, cz;
};
__device__ __forceinline__ ClGrid cl_grid(const ClusterLevel& L) {
  return ClGrid{L.g.nx, L.g.ny, L.g.nz, L.chunk, L.ox, L.orhs, L.obx, L.oby, L.obz, L.cx, L.cy, L.cz};
}

template <class T>
struct ClusterView {
  T* local;  // this rank's shared memory
  int me;
  // element `off` of rank r's shared memory (a distributed-shared-memory
  // address for another rank)
  __device__ __forceinline__ T* at(int r, int off) const {
    T* p = local + off;
    return r == me ? p : cooperative_groups::this_cluster().map_shared_rank(p, r);
  }
  __device__ __forceinline__ int p0(const ClGrid& L) const { return min(L.nz, me * L.chunk); }
  __device__ __forceinline__ int p1(const ClGrid& L) const { return min(L.nz, (me + 1) * L.chunk); }
  // x of cell (i, j, k) of grid L, in whichever rank holds plane k; 0 outside the grid
  __device__ __forceinline__ T x(const ClGrid& L, int i, int j, int k) const {
    if (i < 0 || j < 0 || k < 0 || i >= L.nx || j >= L.ny || k >= L.nz) return (T)0;
    const int r = k / L.chunk;
    return *at(r, L.ox + ((k - r * L.chunk) * L.ny + j) * L.nx + i);
  }
  __device__ __forceinline__ T* rhsp(const ClGrid& L, int i, int j, int k) const {  // any rank
    const int r = k / L.chunk;
    return at(r, L.orhs + ((k - r * L.chunk) * L.ny + j) * L.nx + i);
  }
};

// Copies nrows rows of rl elements (global row r at src + base + (r / rpp) *
// ps + (r % rpp) * px, for rpp rows per plane) into dst, row after row.  The
// warps take rows in turn and the lanes a row's elements: one division per
// row.  Arrays stored as T are copied by asynchronous element copies (all of
// a thread's copies in flight; the caller waits), others through registers
// (converted exactly to T).
template <class T>
__device__ __forceinline__ void cl_copy_rows(T* dst, const void* src, int ctype, int base, int nrows, int rl,
                                             int rpp, int px, int ps) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool same = ctype == (sizeof(T) == 8 ? 0 : 1);
  for (int r = w; r < nrows; r += nw) {
    const int g0 = base + (r / rpp) * ps + (r % rpp) * px;
    T* d = dst + r * rl;
    if (same) {
      const T* sp = reinterpret_cast<const T*>(src) + g0;
      for (int i = lane; i < rl; i += 32) __pipeline_memcpy_async(d + i, sp + i, sizeof(T));
    } else {
      for (int i = lane; i < rl; i += 32) {
        if (ctype == 0) d[i] = (T)reinterpret_cast<const double*>(src)[g0 + i];
        else if (ctype == 1) d[i] = (T)reinterpret_cast<const float*>(src)[g0 + i];
        else d[i] = (T)__bfloat162float(reinterpret_cast<const __nv_bfloat16*>(src)[g0 + i]);
      }
    }
  }
}

// The weights of this rank's planes of grid L and, for the set's first grid,
// its right-hand side, into shared memory.
template <class T>
__device__ __noinline__ void cl_stage(ClusterView<T> V, const ClusterLevel& Lp, const T* rhs0) {
  const ClGrid L = cl_grid(Lp);
  const Geom& g = Lp.g;
  const int k0 = V.p0(L), np = V.p1(L) - k0;
  if (np <= 0) return;
  const int b = g.idx(0, 0, k0);
  cl_copy_rows<T>(V.local + L.obx, Lp.bx, Lp.ctype, b, np * L.ny, L.nx + 1, L.ny, g.px, g.ps);
  cl_copy_rows<T>(V.local + L.oby, Lp.by, Lp.ctype, b, np * (L.ny + 1), L.nx, L.ny + 1, g.px, g.ps);
  cl_copy_rows<T>(V.local + L.obz, Lp.bz, Lp.ctype, b, (np + 1) * L.ny, L.nx, L.ny, g.px, g.ps);  // z-faces k0..k0+np
  if (rhs0) cl_copy_rows<T>(V.local + L.orhs, rhs0, sizeof(T) == 8 ? 0 : 1, b, np * L.ny, L.nx, L.ny, g.px, g.ps);
}
template <class T>
__device__ __noinline__ void cl_stage_rhs(ClusterView<T> V, const ClusterLevel& Lp, const T* rhs0) {
  const ClGrid L = cl_grid(Lp);
  const Geom& g = Lp.g;
  const int k0 = V.p0(L), np = V.p1(L) - k0;
  if (np <= 0) return;
  cl_copy_rows<T>(V.local + L.orhs, rhs0, sizeof(T) == 8 ? 0 : 1, g.idx(0, 0, k0), np * L.ny, L.nx, L.ny, g.px, g.ps);
}

// The six neighbours (x-, x+, y-, y+, z-, z+) of the own cell (i, j, k) of
// grid L at local offset c (plane kk of the rank's np planes); 0 outside the
// grid.  Only the planes below the first and above the last own plane come
// from another rank: the last plane of rank me-1 and the first of rank me+1
// (every spread grid has the same chunk in every rank; a grid of rank 0 has
// all its planes).
template <class T>
__device__ __forceinline__ void cl_nb(const ClusterView<T>& V, const ClGrid& L, int i, int j, int k, int kk, int np,
                                      int c, T (&n)[6]) {
  const int nx = L.nx, ny = L.ny, pl = nx * ny;
  const T* x = V.local + L.ox;
  n[0] = i > 0 ? x[c - 1] : (T)0;
  n[1] = i + 1 < nx ? x[c + 1] : (T)0;
  n[2] = j > 0 ? x[c - nx] : (T)0;
  n[3] = j + 1 < ny ? x[c + nx] : (T)0;
  n[4] = (T)0;
  if (k > 0) n[4] = kk > 0 ? x[c - pl] : *V.at(V.me - 1, L.ox + (L.chunk - 1) * pl + j * nx + i);
  n[5] = (T)0;
  if (k + 1 < L.nz) n[5] = kk + 1 < np ? x[c + pl] : *V.at(V.me + 1, L.ox + j * nx + i);
}

template <class T>
__device__ __forceinline__ void cl_weights(const ClusterView<T>& V, const ClGrid& L, int i, int j, int kk, int c,
                                           T& wxm, T& wxp, T& wym, T& wyp, T& wzm, T& wzp) {
  const int nx = L.nx, ny = L.ny;
  const T* bx = V.local + L.obx + (kk * ny + j) * (nx + 1) + i;
  const T* by = V.local + L.oby + (kk * (ny + 1) + j) * nx + i;
  const T* bz = V.local + L.obz + c;
  wxm = bx[0];
  wxp = bx[1];
  wym = by[0];
  wyp = by[nx];
  wzm = bz[0];
  wzp = bz[nx * ny];
}

// Half-sweep of colour `colour` over this rank's planes of grid L: the
// operations of cta_half_sweep.  pro: with the prolongation of the coarse
// grid Lc's x added to every neighbour inside the grid.  A thread's items are
// t, t + blockDim, ... of the (pair, row, plane) box; their coordinates
// advance by carries, with no division inside the loop.
template <class T>
__device__ __noinline__ void cl_half_sweep(ClusterView<T> V, ClGrid L, int colour, bool zero_init, bool pro,
                                           ClGrid Lc) {
  typedef acc_t<T> A;
  const int nx = L.nx, ny = L.ny, k0 = V.p0(L), np = V.p1(L) - k0;
  const int half = (nx + 1) / 2;
  const int total = half * ny * max(0, np);
  int t = threadIdx.x;
  if (t >= total) return;
  int tx = t % half, j = (t / half) % ny, kk = t / (half * ny);
  const int st = blockDim.x, sx = st % half, sj = (st / half) % ny, sk = st / (half * ny);
  for (; t < total; t += st) {
    const int k = k0 + kk;
    const int i = 2 * tx + ((2 * tx + j + k + colour) & 1);
    if (i < nx) {
      const int c = (kk * ny + j) * nx + i;
      T wxm, wxp, wym, wyp, wzm, wzp;
      cl_weights(V, L, i, j, kk, c, wxm, wxp, wym, wyp, wzm, wzp);
      const A bv = (A)V.local[L.orhs + c];  // (no mean shift below the finest grid)
      A n[6] = {(A)0, (A)0, (A)0, (A)0, (A)0, (A)0};
      if (!zero_init) {
        T xn[6];
        cl_nb(V, L, i, j, k, kk, np, c, xn);
#pragma unroll
        for (int q = 0; q < 6; ++q) n[q] = (A)xn[q];
        if (pro) {
          const int ci[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1},
                                {i, j, k + 1}};
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            const int a = ci[q][0], b = ci[q][1], d = ci[q][2];
            if (a >= 0 && b >= 0 && d >= 0 && a < nx && b < ny && d < L.nz)
              n[q] = Ar<A>::add(n[q], (A)V.x(Lc, Lc.cx ? a >> 1 : a, Lc.cy ? b >> 1 : b, Lc.cz ? d >> 1 : d));
          }
        }
      }
      V.local[L.ox + c] = (T)Stencil<T, T>::gs(bv, (A)wxm, (A)wxp, (A)wym, (A)wyp, (A)wzm, (A)wzp, n[0], n[1], n[2],
                                               n[3], n[4], n[5]);
    }
    tx += sx;
    int cy = tx >= half;
    tx -= cy ? half : 0;
    j += sj + cy;
    cy = j >= ny;
    j -= cy ? ny : 0;
    kk += sk + cy;
  }
}

// Residual of fine cell (i, j, k) (plane kk of the rank's np) added to acc:
// the operations of cta_resid_restrict.
template <class T>
__device__ __forceinline__ void cl_resid_add(const ClusterView<T>& V, const ClGrid& L, int i, int j, int k, int kk,
                                             int np, acc_t<T>& acc) {
  typedef acc_t<T> A;
  const int c = (kk * L.ny + j) * L.nx + i;
  T wxm, wxp, wym, wyp, wzm, wzp, xn[6];
  cl_weights(V, L, i, j, kk, c, wxm, wxp, wym, wyp, wzm, wzp);
  cl_nb(V, L, i, j, k, kk, np, c, xn);
  const A bv = (A)V.local[L.orhs + c];  // (no mean shift below the finest grid)
  const A ax = Stencil<T, T>::apply((A)V.local[L.ox + c], (A)wxm, (A)wxp, (A)wym, (A)wyp, (A)wzm, (A)wzp, (A)xn[0],
                                    (A)xn[1], (A)xn[2], (A)xn[3], (A)xn[4], (A)xn[5]);
  acc = Ar<A>::add(acc, Ar<A>::add(bv, -ax));
}

// Residual of grid L restricted to grid Lc (the operations of
// cta_resid_restrict): each rank takes the coarse cells whose children lie in
// its planes and writes them into the rank that holds their plane.
template <class T>
__device__ __noinline__ void cl_resid_restrict(ClusterView<T> V, ClGrid L, ClGrid Lc) {
  typedef acc_t<T> A;
  const int rx = Lc.cx ? 2 : 1, ry = Lc.cy ? 2 : 1, rz = Lc.cz ? 2 : 1;
  // coarse planes whose first child plane is in [k0, k1)
  const int k0 = V.p0(L), k1 = V.p1(L), np = k1 - k0;
  const int K0 = (k0 + rz - 1) / rz, K1 = min(Lc.nz, (k1 + rz - 1) / rz);
  const int total = Lc.nx * Lc.ny * max(0, K1 - K0);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int I = t % Lc.nx, J = (t / Lc.nx) % Lc.ny, K = K0 + t / (Lc.nx * Lc.ny);
    A acc = (A)0;
    for (int dk = 0; dk < rz; ++dk)
      for (int dj = 0; dj < ry; ++dj)
        for (int di = 0; di < rx; ++di) {
          const int k = (Lc.cz ? 2 * K : K) + dk;
          cl_resid_add(V, L, (Lc.cx ? 2 * I : I) + di, (Lc.cy ? 2 * J : J) + dj, k, k - k0, np, acc);
        }
    *V.rhsp(Lc, I, J, K) = (T)Ar<A>::div(acc, (A)(rx * ry * rz));
  }
}

// nhalf half-sweeps of a grid held whole by rank 0 (nx*ny*nz <= KCL_SOLO <=
// blockDim.x): thread t keeps cell t's weights and rhs in registers across
// the half-sweeps, which read the neighbours' x from shared memory and end
// at a CTA barrier.  Half-sweep h has colour c0 ^ (h & 1) before swap_at and
// (1 - c0) ^ ((h - swap_at) & 1) from there (the coarsest grid's backward
// pairs); the first starts from zero (zero_first) or adds the prolongation
// of Lc's x to the neighbours (pro_first).  The operations are those of
// cl_half_sweep.  Called by every thread of rank 0.
template <class T>
__device__ __noinline__ void cl_solo_run(ClusterView<T> V, ClGrid L, int nhalf, int c0, int swap_at, bool zero_first,
                                         bool pro_first, ClGrid Lc) {
  typedef acc_t<T> A;
  const int nx = L.nx, ny = L.ny, nz = L.nz, pc = nx, pl = nx * ny;
  const int t = threadIdx.x;
  const bool own = t < nx * ny * nz;
  int i = 0, j = 0, k = 0, c = 0;
  T wxm = (T)0, wxp = (T)0, wym = (T)0, wyp = (T)0, wzm = (T)0, wzp = (T)0;
  A bv = (A)0;
  if (own) {
    i = t % nx;
    j = (t / nx) % ny;
    k = t / pl;
    c = (k * ny + j) * pc + i;
    cl_weights(V, L, i, j, k, c, wxm, wxp, wym, wyp, wzm, wzp);
    bv = (A)V.local[L.orhs + c];  // (no mean shift below the finest grid)
  }
  T* x = V.local + L.ox;
  for (int h = 0; h < nhalf; ++h) {
    const int colour = h < swap_at ? (c0 ^ (h & 1)) : ((1 - c0) ^ ((h - swap_at) & 1));
    if (own && ((i + j + k + colour) & 1) == 0) {
      A n[6] = {(A)0, (A)0, (A)0, (A)0, (A)0, (A)0};
      if (!(h == 0 && zero_first)) {
        n[0] = (A)(i > 0 ? x[c - 1] : (T)0);
        n[1] = (A)(i + 1 < nx ? x[c + 1] : (T)0);
        n[2] = (A)(j > 0 ? x[c - pc] : (T)0);
        n[3] = (A)(j + 1 < ny ? x[c + pc] : (T)0);
        n[4] = (A)(k > 0 ? x[c - pl] : (T)0);
        n[5] = (A)(k + 1 < nz ? x[c + pl] : (T)0);
        if (h == 0 && pro_first) {
          const int ci[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1},
                                {i, j, k + 1}};
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            const int a = ci[q][0], b = ci[q][1], d = ci[q][2];
            if (a >= 0 && b >= 0 && d >= 0 && a < nx && b < ny && d < nz)
              n[q] = Ar<A>::add(n[q], (A)V.x(Lc, Lc.cx ? a >> 1 : a, Lc.cy ? b >> 1 : b, Lc.cz ? d >> 1 : d));
          }
        }
      }
      x[c] = (T)Stencil<T, T>::gs(bv, (A)wxm, (A)wxp, (A)wym, (A)wyp, (A)wzm, (A)wzp, n[0], n[1], n[2], n[3], n[4],
                                  n[5]);
    }
    __syncthreads();
  }
}

// Smoothing step helpers: the spread grids end each step at a cluster
// barrier, the grids of rank 0 at a CTA barrier (rank 0 only).
template <class T, class F>
__device__ __forceinline__ void cl_step(const ClusterView<T>& V, bool spread, F&& f) {
  if (spread || V.me == 0) f();
  if (spread) cooperative_groups::this_cluster().sync();
  else if (V.me == 0) __syncthreads();
}

// The lower part of the V-cycle: pre-smoothing (nu1 sweeps from zero) and
// restriction down the set, coarse_pairs symmetric sweep pairs on the
// coarsest grid, prolongation and post-smoothing (nu2 sweeps) back up; the
// sequence of k_coarse_vcycle.  The set's first grid is not the finest
// (no mean shift is applied).
template <class T>
__global__ void __cluster_dims__(KCL, 1, 1) __launch_bounds__(kcl_threads<T>())
    k_coarse_cluster(const __grid_constant__ ClusterSet set, int nu1, int nu2, int coarse_pairs, const Scalars* s) {
  static_assert(KCL_SOLO <= kcl_threads<T>(), "a rank-0 grid needs a thread per cell");
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char cl_smem[];
  cg::cluster_group cl = cg::this_cluster();
  ClusterView<T> V;
  V.me = (int)cl.block_rank();
  V.local = reinterpret_cast<T*>(cl_smem);
  const int n = set.n, nd = set.nd;
  // The weights, which no kernel of the solve writes, are staged while the
  // previous kernel drains; the first grid's rhs, its output, after the wait.
  for (int q = 0; q < n; ++q) cl_stage<T>(V, set.L[q], nullptr);
  pdl_enter();
  if (s && s->done) {  // the same flag for every rank: all return, or none
    __pipeline_commit();
    __pipeline_wait_prior(0);  // no copy into this CTA's shared memory outlives it
    return;
  }
  cl_stage_rhs<T>(V, set.L[0], (const T*)set.rhs0);
  __pipeline_commit();
  __pipeline_wait_prior(0);
  cl.sync();
  // down the spread grids
  for (int q = 0; q < nd; ++q) {
    const ClGrid L = cl_grid(set.L[q]);
    for (int it = 0; it < nu1; ++it) {
      cl_step(V, true, [&] { cl_half_sweep<T>(V, L, 0, it == 0, false, L); });
      cl_step(V, true, [&] { cl_half_sweep<T>(V, L, 1, false, false, L); });
    }
    cl_step(V, true, [&] { cl_resid_restrict<T>(V, L, cl_grid(set.L[q + 1])); });
  }
  // the grids of rank 0: down, the coarsest, up
  if (V.me == 0) {
    for (int q = nd; q < n - 1; ++q) {
      const ClGrid L = cl_grid(set.L[q]);
      cl_solo_run<T>(V, L, 2 * nu1, 0, 2 * nu1, true, false, L);
      cl_step(V, false, [&] { cl_resid_restrict<T>(V, L, cl_grid(set.L[q + 1])); });
    }
    const ClGrid C = cl_grid(set.L[n - 1]);
    cl_solo_run<T>(V, C, 4 * coarse_pairs, 0, 2 * coarse_pairs, true, false, C);
    for (int q = n - 2; q >= nd; --q) {
      const ClGrid L = cl_grid(set.L[q]);
      cl_solo_run<T>(V, L, 2 * nu2, 1, 2 * nu2, false, true, cl_grid(set.L[q + 1]));
    }
  }
  cl.sync();
  // up the spread grids
  for (int q = nd - 1; q >= 0; --q) {
    const ClGrid L = cl_grid(set.L[q]);
    for (int it = 0; it < nu2; ++it) {
      cl_step(V, true, [&] { cl_half_sweep<T>(V, L, 1, false, it == 0, cl_grid(set.L[q + 1])); });
      cl_step(V, true, [&] { cl_half_sweep<T>(V, L, 0, false, false, L); });
    }
  }
  // the first grid's x back to global memory (own planes; after the last
  // barrier no rank reads another's shared memory)
  {
    const ClusterLevel& Lp = set.L[0];
    const ClGrid L = cl_grid(Lp);
    const Geom& g = Lp.g;
    const int k0 = V.p0(L), np = V.p1(L) - k0;
    T* x0 = reinterpret_cast<T*>(set.x0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = w; r < max(0, np) * L.ny; r += nw) {
      const int j = r % L.ny, k = k0 + r / L.ny;
      const T* src = V.local + L.ox + r * L.nx;
      T* dst = x0 + g.idx(0, j, k);
      for (int i = lane; i < L.nx; i += 32) dst[i] = src[i];
    }
  }
}

}  // namespace smac
