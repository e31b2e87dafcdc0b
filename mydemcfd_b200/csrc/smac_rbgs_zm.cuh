// smac_rbgs_zm.cuh -- the fused red-black Gauss-Seidel sweep as a register
// z-march over whole x-rows.
//
// Same mathematics and rounding as k_rbgs_sweep, k_rbgs_tma and the two
// half-sweep kernels (k_rbgs): xout = S(xin), colour c0 from xin, then colour
// 1-c0 from the new c0 values.  The data movement is different:
//
//   - a warp owns 32 x NV consecutive cells of one row (NV = 4 or 2 FP32, 2
//     FP64: one 16- or 8-byte vector per lane and array), WX warps side by side cover the
//     whole x extent, so the tile needs no ring in x;
//   - a CTA stacks TY rows of such warps plus one ring row above and below
//     (j0-1 and j0+TY), which compute colour c0 only: their values are the
//     y-neighbours of the tile's edge rows in the colour-(1-c0) pass, and
//     recomputing them keeps every CTA independent of the others;
//   - the CTA marches z through its chunk.  A lane keeps in registers the
//     values of its own column that the stencil reads across planes: the
//     colour-(1-c0) inputs of planes k-1..k+1 and the colour-c0 results of
//     planes k-2..k.  x-neighbours across the vector edge come from the next
//     lane (shuffle), across the warp edge from shared memory;
//   - shared memory carries each row to the rows above and below: the input
//     vector of plane k+1 whole, and the c0 results of plane k packed H per
//     lane (so that both stores are conflict-free); four planes of each
//     rotate (a plane is written at steps k-1 and k and last read at step
//     k+1, by the slowest warp before the barrier of step k+2);
//   - the loads of step k+1 (input, rhs, weights) are issued at the start of
//     step k, so one step of global latency is hidden behind the arithmetic
//     of the step.
// Step k computes colour c0 on plane k, then (after the step's one barrier)
// colour 1-c0 on plane k-1, whose finished vector is stored.
//
// Algorithmic HBM bytes per cell: xin, rhs, bx, by, bz read, xout written
// (6 values); the ring rows and the by row above are re-read from L1/L2.
#pragma once

#include <type_traits>

#include "smac_rbgs.cuh"
#include "smac_rbgs_tma.cuh"

namespace smac {

// x += P(xc) on the cells of the fine grid, in place: the prolongation of
// the coarse-grid correction (the parent (i>>1, j>>1, k>>1) on the halved
// directions), run ahead of the first post-smoothing sweep of the z-march,
// which then takes its plain form.  Each cell's sum is the one the fused
// forms compute, so the sweep's result is the same bit for bit.  (Fused into
// the z-march, the coarse loads and sums cost 60% more than the sweep.)
template <class T>
__global__ void __launch_bounds__(256) k_prolong_add(Geom g, T* __restrict__ x, const T* __restrict__ xc, Geom gc,
                                                     int cx, int cy, int cz, const Scalars* s) {
  pdl_enter();
  if (s && s->done) return;
  typedef typename Vec16<T>::type V;
  constexpr int NV = Vec16<T>::n;
  const int nvr = (g.nx + NV - 1) / NV;  // vectors per row; the last one may reach into the zero pad
  const long long total = (long long)nvr * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(t % nvr);
    const long long r = t / nvr;
    const int j = (int)(r % g.ny), k = (int)(r / g.ny);
    const int ib = v * NV;
    V* p = reinterpret_cast<V*>(x + g.idx(ib, j, k));
    V a = *p;
    T* pa = reinterpret_cast<T*>(&a);
    const int jc = cy ? j >> 1 : j, kc = cz ? k >> 1 : k;
#pragma unroll
    for (int e = 0; e < NV; ++e) {
      const int i = ib + e;
      if (i < g.nx) pa[e] = (T)Ar<T>::add((T)pa[e], (T)xc[gc.idx(cx ? i >> 1 : i, jc, kc)]);
    }
    *p = a;
  }
}

// Planes ahead of the one a step loads that one thread of the CTA asks the
// L2 to fetch (one bulk prefetch per array and plane over the rows the tile
// reads), on grids whose arrays do not fit in L2; 0 leaves the loads to find
// their data in DRAM.
#ifndef SMAC_ZM_PF
#define SMAC_ZM_PF 2
#endif

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// A bounded wait on an mbarrier that nothing arrives on (the self-test of the
// kernels' wait limit): lane 0 records the expiry the way the sweeps do and
// the cycles it waited.
__global__ void k_wait_probe(Scalars* s, long long* cycles) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const long long t0 = clock64();
  const bool ok = mbar_wait_bounded(&bar, 0u);
  if (threadIdx.x == 0) {
    cycles[0] = clock64() - t0;
    if (!ok) s->status = 6;
  }
}

// NV consecutive cells of one row as one register vector (8 or 16 bytes)
template <class T, int N> struct VecN;
template <> struct VecN<float, 2> { typedef float2 type; };
template <> struct VecN<float, 4> { typedef float4 type; };
template <> struct VecN<double, 2> { typedef double2 type; };

template <class T, int NV_, int WX, int TY, int MODE>
struct ZmTile {
  static constexpr int NV = NV_;                  // cells per lane
  static constexpr int H = NV / 2;                // cells of one colour per lane and plane
  static constexpr int TW = 32 * NV * WX;         // cells per row: the whole x extent
  static constexpr int ROWS = TY + 2;             // tile rows plus the two ring rows
  static constexpr int NT = 32 * WX * ROWS;       // threads per CTA
  // CTAs per SM the registers must allow: a 256-thread tile runs two (three
  // with float2 lanes) per SM at 128 (85) registers a thread
  static constexpr int MINB = NT <= 256 ? (NV == 2 && sizeof(T) == 4 ? 3 : 2) : 1;
  static constexpr int NB = 4;                    // shared planes in rotation
  static constexpr int M_BYTES = NB * ROWS * TW * (int)sizeof(T);           // inputs, whole vectors
  static constexpr int R_BYTES = NB * ROWS * 32 * WX * H * (int)sizeof(T);  // c0 results, H per lane
  static constexpr int SMEM = M_BYTES + R_BYTES;
};

// Operands of the colour-c0 pass on plane m, loaded one step ahead: the rhs,
// the x-faces (and the one past the lane's vector), the y-faces of rows j and
// j+1, the z-faces m+1, the input of plane m+1 and, for the ring rows, the
// input of the row beyond on plane m.
template <class T, int NV>
struct ZmOps {
  typename VecN<T, NV>::type rh, bx, by, byu, bzu, x1, xo;
  T bxe;
  T c1[2];  // with the prolongation on a grid halved in every direction: the parents of x1
};
// Operands of the colour-(1-c0) pass on plane m, carried to the next step:
// per cell of that colour its rhs and six weights.
template <class T, int H>
struct ZmBlk {
  T rh[H], bxm[H], bxp[H], by[H], byu[H], bz[H], bzu[H];
};

template <class T, int NV_, int WX, int TY, int MODE, bool DOT>
__global__ void __launch_bounds__(ZmTile<T, NV_, WX, TY, MODE>::NT, ZmTile<T, NV_, WX, TY, MODE>::MINB)
    k_rbgs_zm(Geom g, const T* __restrict__ xin, T* __restrict__ xout, const T* __restrict__ rhs, const double* shift,
              Stencil<T, T> S, int c0, const T* __restrict__ xc, Geom gc, int cx, int cy, int cz, Scalars* s,
              RedBuf red, int zchunk, int pf) {
  pdl_enter();
  typedef ZmTile<T, NV_, WX, TY, MODE> L;
  typedef typename VecN<T, NV_>::type V;
  typedef T A;
  typedef ZmOps<T, NV_> Ops;
  constexpr int NV = L::NV, H = L::H, TW = L::TW, ROWS = L::ROWS, NT = L::NT;
  typedef ZmBlk<T, H> Blk;
  extern __shared__ __align__(16) unsigned char zm_smem[];
  T* M = reinterpret_cast<T*>(zm_smem);                  // inputs [NB][ROWS][TW]
  T* R = reinterpret_cast<T*>(zm_smem + L::M_BYTES);     // c0 results [NB][ROWS][32 WX][H]
  if (s && s->done) return;
  // One barrier phase per step, split: a warp arrives once its shared writes
  // of step k are done and waits for the phase only before the first shared
  // read of step k+1, so the colour-(1-c0) pass of step k (which reads step
  // k-1's results) and the next step's loads overlap the slower warps.
  // Waits are bounded; on expiry the status records the failure and the
  // kernel runs on without waiting.
  __shared__ uint64_t zm_bar;
  if (threadIdx.x == 0) mbar_init(&zm_bar, ZmTile<T, NV_, WX, TY, MODE>::NT / 32);
  __syncthreads();
  uint32_t zm_phase = 0;
  bool zm_bad = false;
  auto zm_arrive = [&]() {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&zm_bar);
  };
  auto zm_wait = [&]() {
    if (!zm_bad && !mbar_wait_bounded(&zm_bar, zm_phase & 1u)) {
      zm_bad = true;
      if (s) s->status = 6;
    }
    ++zm_phase;
  };
  const int tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5;
  const int wx = w % WX, wr = w / WX;
  const bool ring = (wr == 0 || wr == ROWS - 1);
  const int ib = (wx * 32 + lane) * NV;  // first cell of this lane's vector
  const bool col_ok = ib < g.px;         // the vector lies inside the padded row
  const double shd = shift ? *shift : 0.0;
  const A sh = (A)shd;
  const int nty = (g.ny + TY - 1) / TY;
  const int items = nty * ((g.nz + zchunk - 1) / zchunk);
  auto Mrow = [&](int k, int r) -> T* { return M + ((k & 3) * ROWS + r) * TW; };
  // the c0 results of lane t of row r on plane k: H consecutive values (one 8-byte access)
  auto Rlane = [&](int k, int r, int t) -> T* { return R + (((k & 3) * ROWS + r) * 32 * WX + t) * H; };
  typedef typename std::conditional<H == 2, typename Vec2<T>::type, T>::type RV;  // H values as one access
  double dv[2] = {0.0, 0.0};

  auto zero = []() {
    V v;
    T* p = reinterpret_cast<T*>(&v);
#pragma unroll
    for (int e = 0; e < NV; ++e) p[e] = (T)0;
    return v;
  };
  auto el = [](const V& v, int e) -> T { return reinterpret_cast<const T*>(&v)[e]; };

  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int ty = item % nty, zi = item / nty;
    const int j0 = ty * TY;
    const int j = j0 - 1 + wr;  // this warp's row
    const bool row_ok = j >= 0 && j < g.ny;
    const int z0 = zi * zchunk, z1 = min(z0 + zchunk, g.nz);
    const int jo = wr == 0 ? j - 1 : j + 1;  // ring warps: the row beyond the ring
    const bool jo_ok = ring && jo >= 0 && jo < g.ny;

    // the input vector of plane m, row jj (the coarse correction added in MODE 2); 0 outside the grid
    auto load_x = [&](int m, int jj, bool ok) -> V {
      if constexpr (MODE == 1) return zero();
      if (!ok || !col_ok || m < 0 || m >= g.nz) return zero();
      V v = *reinterpret_cast<const V*>(xin + g.idx(ib, jj, m));
      if constexpr (MODE == 2) {
        T* pv = reinterpret_cast<T*>(&v);
#pragma unroll
        for (int e = 0; e < NV; ++e) {
          const int i = ib + e;
          if (i < g.nx) pv[e] = (T)Ar<A>::add((A)pv[e], (A)xc[gc.idx(cx ? i >> 1 : i, cy ? jj >> 1 : jj, cz ? m >> 1 : m)]);
        }
      }
      return v;
    };
    auto load_v = [&](const T* a, int m, int jj, bool ok) -> V {
      if (!ok || !col_ok) return zero();
      return *reinterpret_cast<const V*>(a + g.idx(ib, jj, m));
    };
    // With the prolongation on a grid halved in every direction, the input
    // vector of the lane's row is loaded as it is and its cells' parents
    // (NV/2 coarse values) beside it; the sum is formed when the vector is
    // used, a step later, so that no load is waited for where it is issued.
    // (The ring rows' row beyond takes the immediate path: those warps wait
    // at the step's barrier anyway.)
    const bool pro4 = MODE == 2 && cx && cy && cz;
    auto load_parents = [&](int m, int jj, bool ok, T (&c)[2]) {
      c[0] = c[1] = (T)0;
      if (!ok || !col_ok || m < 0 || m >= g.nz || ib >= g.nx) return;
      const T* p = xc + gc.idx(ib >> 1, jj >> 1, m >> 1);
      if constexpr (NV == 4) {
        const typename Vec2<T>::type v = *reinterpret_cast<const typename Vec2<T>::type*>(p);
        c[0] = v.x;
        c[1] = v.y;
      } else {
        c[0] = p[0];
      }
    };
    auto add_parents = [&](V v, const T (&c)[2]) -> V {
      T* pv = reinterpret_cast<T*>(&v);
#pragma unroll
      for (int e = 0; e < NV; ++e)
        if (ib + e < g.nx) pv[e] = (T)Ar<A>::add((A)pv[e], (A)c[e >> 1]);
      return v;
    };
    auto load_ops = [&](int m, Ops& o) {
      const bool ok = row_ok && m >= 0 && m < g.nz;
      o.rh = load_v(rhs, m, j, ok);
      o.bx = load_v(S.bx, m, j, ok);
      o.bxe = (ok && col_ok && ib + NV <= g.nx) ? S.bx[g.idx(ib + NV, j, m)] : (T)0;
      o.by = load_v(S.by, m, j, ok);
      o.byu = load_v(S.by, m, j + 1, ok);
      o.bzu = load_v(S.bz, m + 1, j, row_ok && m + 1 >= 0 && m + 1 <= g.nz);  // z-face m+1 (0..nz)
      if (pro4) {
        o.x1 = (row_ok && col_ok && m + 1 >= 0 && m + 1 < g.nz) ? *reinterpret_cast<const V*>(xin + g.idx(ib, j, m + 1))
                                                                : zero();
        o.xo = load_x(m, jo, jo_ok);
        load_parents(m + 1, j, row_ok, o.c1);
      } else {
        o.x1 = load_x(m + 1, j, row_ok);
        o.xo = load_x(m, jo, jo_ok);
      }
    };

    // The rows the tile reads on one plane (j0-2 .. j0+TY+1, clipped to the
    // grid's ny+1 allocated rows) lie at consecutive addresses: one prefetch
    // per array covers them.  Planes 0..nz are allocated in every array, and
    // the host passes pf = 0 unless every array is 16-byte aligned.  Thread 0
    // (row j0-1) issues them from the kernel's parameters and its own row, so
    // that no other thread keeps a value live for them.
    auto prefetch = [&](int m) {  // the operands of plane m (its z-faces m+1 and input m+1 with them)
      if (threadIdx.x != 0 || m < 0 || m + 1 > g.nz) return;
      const int ja = max(0, j - 1);
      const uint32_t bytes = (uint32_t)((min(g.ny, j + TY + 2) - ja + 1) * g.px * (int)sizeof(T));
      const int o = g.idx(0, ja, m), o1 = o + g.ps;
      bulk_prefetch_l2(rhs + o, bytes);
      bulk_prefetch_l2(S.bx + o, bytes);
      bulk_prefetch_l2(S.by + o, bytes);
      bulk_prefetch_l2(S.bz + o1, bytes);
      if (MODE != 1) bulk_prefetch_l2(xin + o1, bytes);
    };

    // prologue: the inputs of planes kb-1 and kb, the shared plane kb, the
    // operands of the first c0 plane kb = z0 - 1
    const int kb = z0 - 1;
    for (int d = 1; d <= pf; ++d) prefetch(kb + 1 + d);
    const int pk = (c0 + j + kb) & 1;  // parity of the c0 cells of plane kb in this row (warp-uniform)
    Ops opA, opB;
    load_ops(kb, opA);
    opB.bzu = (row_ok && col_ok && kb >= 0 && kb < g.nz) ? *reinterpret_cast<const V*>(S.bz + g.idx(ib, j, kb))
                                                         : zero();  // the z-faces kb, read as "the step before"
    const V xv_m = load_x(kb - 1, j, row_ok);
    const V xv_0 = load_x(kb, j, row_ok);
    *reinterpret_cast<V*>(Mrow(kb, wr) + ib) = xv_0;
    // colour-(1-c0) inputs of planes kb-1 and kb at the c0 positions of plane kb
    T xh_m[H], xh_0[H];
#pragma unroll
    for (int q = 0; q < H; ++q) {
      xh_m[q] = pk ? el(xv_m, 2 * q + 1) : el(xv_m, 2 * q);
      xh_0[q] = pk ? el(xv_0, 2 * q) : el(xv_0, 2 * q + 1);
    }
    // c0 results kept for the colour-(1-c0) pass
    T red_m2[H], red_m1[H];
    Blk blA, blB;
#pragma unroll
    for (int q = 0; q < H; ++q) red_m2[q] = red_m1[q] = (T)0;
    zm_arrive();  // the prologue's shared writes (waited for by the first step)

    // Step k with P = parity of plane k's c0 cells (a compile-time constant):
    // colour c0 on plane k from `cur`, the operands of plane k+1 loaded into
    // `nxt`, the colour-(1-c0) operands of plane k saved to `bout`; after the
    // barrier colour 1-c0 on plane k-1 from `bin`.
    auto step = [&](auto Pc, int k, Ops& cur, Ops& nxt, const Blk& bin, Blk& bout) {
      constexpr int P = decltype(Pc)::value;
      const V bz_c = nxt.bzu;  // z-faces k (the previous step's faces k-1+1), read before nxt is reloaded
      if (k + 1 <= z1) load_ops(k + 1, nxt);
      if (pf > 0 && k + 1 + pf <= z1) prefetch(k + 1 + pf);
      if (pro4) cur.x1 = add_parents(cur.x1, cur.c1);  // the deferred prolongation of this step's input
      // --- the input of plane k+1 becomes visible to the rows above and below
      *reinterpret_cast<V*>(Mrow(k + 1, wr) + ib) = cur.x1;
      T xh_p[H];
#pragma unroll
      for (int q = 0; q < H; ++q) xh_p[q] = el(cur.x1, 2 * q + P);  // colour 1-c0 of plane k+1
      // --- colour c0 on plane k: cells 2q + P
      T red_k[H];
      const bool plane_ok = k >= 0 && k < g.nz;
      zm_wait();  // every warp's shared writes of the previous step
      {
        const T* Mk = Mrow(k, 0);
        // x-neighbours across the vector edge: colour-(1-c0) inputs of plane k
        T left = __shfl_up_sync(0xffffffffu, xh_0[H - 1], 1);
        T right = __shfl_down_sync(0xffffffffu, xh_0[0], 1);
        if (lane == 0) left = wx > 0 ? Mk[wr * TW + ib - 1] : (T)0;
        if (lane == 31) right = wx < WX - 1 ? Mk[wr * TW + ib + NV] : (T)0;
        V ym, yp;
        if (wr == 0) ym = cur.xo; else ym = *reinterpret_cast<const V*>(Mk + (wr - 1) * TW + ib);
        if (wr == ROWS - 1) yp = cur.xo; else yp = *reinterpret_cast<const V*>(Mk + (wr + 1) * TW + ib);
#pragma unroll
        for (int q = 0; q < H; ++q) {
          const int e = 2 * q + P;
          A v = (A)0;
          if (row_ok && plane_ok && ib + e < g.nx) {
            const A bv = Ar<A>::add((A)el(cur.rh, 2 * q + P), -sh);
            const A wxm = (A)el(cur.bx, 2 * q + P);
            const A wxp = (A)(2 * q + P + 1 < NV ? el(cur.bx, (2 * q + P + 1) % NV) : cur.bxe);
            const A wym = (A)el(cur.by, 2 * q + P), wyp = (A)el(cur.byu, 2 * q + P);
            const A wzm = (A)el(bz_c, 2 * q + P), wzp = (A)el(cur.bzu, 2 * q + P);
            if constexpr (MODE == 1) {
              v = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, (A)0, (A)0, (A)0, (A)0, (A)0, (A)0);
            } else {
              // colour-(1-c0) positions of plane k: e-1 and e+1
              const A n0 = (A)(P == 0 ? (q > 0 ? xh_0[q > 0 ? q - 1 : 0] : left) : xh_0[q]);
              const A n1 = (A)(P == 0 ? xh_0[q] : (q + 1 < H ? xh_0[q + 1 < H ? q + 1 : q] : right));
              v = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, n0, n1, (A)el(ym, 2 * q + P),
                                    (A)el(yp, 2 * q + P), (A)xh_m[q], (A)xh_p[q]);
            }
          }
          red_k[q] = (T)v;
          if constexpr (DOT) {
            // r.z: the c0 cells of the chunk's planes (not the ring rows' nor the extra planes)
            if (!ring && k >= z0 && k < z1 && row_ok && ib + e < g.nx) {
              const double z = (double)red_k[q];
              dv[0] += ((double)el(cur.rh, 2 * q + P) - shd) * z;
              dv[1] += z;
            }
          }
        }
        // c0 results of plane k, H per lane side by side (0 outside the grid)
        {
          RV rv;
          T* pr = reinterpret_cast<T*>(&rv);
#pragma unroll
          for (int q = 0; q < H; ++q) pr[q] = red_k[q];
          *reinterpret_cast<RV*>(Rlane(k, wr, wx * 32 + lane)) = rv;
        }
      }
      // operands of the colour-(1-c0) pass on plane k (next step): cells 2q + (1-P)
#pragma unroll
      for (int q = 0; q < H; ++q) {
        constexpr int Q = 1 - P;
        bout.rh[q] = el(cur.rh, 2 * q + Q);
        bout.bxm[q] = el(cur.bx, 2 * q + Q);
        bout.bxp[q] = 2 * q + Q + 1 < NV ? el(cur.bx, (2 * q + Q + 1) % NV) : cur.bxe;
        bout.by[q] = el(cur.by, 2 * q + Q);
        bout.byu[q] = el(cur.byu, 2 * q + Q);
        bout.bz[q] = el(bz_c, 2 * q + Q);
        bout.bzu[q] = el(cur.bzu, 2 * q + Q);
      }
      zm_arrive();
      // --- colour 1-c0 on plane k-1 (tile rows only): cells 2q + P
      const int kk = k - 1;
      if (!ring && kk >= z0 && kk < z1) {
        // c0 results of plane k-1 sit at positions 2q + (1-P) of this row and
        // at 2q + P of the rows above and below: there they are the y-neighbours
        const int t = wx * 32 + lane;
        T left = __shfl_up_sync(0xffffffffu, red_m1[H - 1], 1);
        T right = __shfl_down_sync(0xffffffffu, red_m1[0], 1);
        if (lane == 0) left = wx > 0 ? Rlane(kk, wr, t - 1)[H - 1] : (T)0;
        if (lane == 31) right = wx < WX - 1 ? Rlane(kk, wr, t + 1)[0] : (T)0;
        const RV ymv = *reinterpret_cast<const RV*>(Rlane(kk, wr - 1, t));
        const RV ypv = *reinterpret_cast<const RV*>(Rlane(kk, wr + 1, t));
        const T* ym = reinterpret_cast<const T*>(&ymv);
        const T* yp = reinterpret_cast<const T*>(&ypv);
        T blk[H];
#pragma unroll
        for (int q = 0; q < H; ++q) {
          const int e = 2 * q + P;
          A v = (A)0;
          if (row_ok && ib + e < g.nx) {
            const A bv = Ar<A>::add((A)bin.rh[q], -sh);
            const A n0 = (A)(P == 0 ? (q > 0 ? red_m1[q > 0 ? q - 1 : 0] : left) : red_m1[q]);
            const A n1 = (A)(P == 0 ? red_m1[q] : (q + 1 < H ? red_m1[q + 1 < H ? q + 1 : q] : right));
            v = Stencil<T, T>::gs(bv, (A)bin.bxm[q], (A)bin.bxp[q], (A)bin.by[q], (A)bin.byu[q], (A)bin.bz[q],
                                  (A)bin.bzu[q], n0, n1, (A)ym[q], (A)yp[q], (A)red_m2[q], (A)red_k[q]);
          }
          blk[q] = (T)v;
        }
        if (row_ok && col_ok) {
          V out;
          T* o = reinterpret_cast<T*>(&out);
#pragma unroll
          for (int q = 0; q < H; ++q) {
            o[2 * q + P] = blk[q];
            o[2 * q + 1 - P] = red_m1[q];
          }
          *reinterpret_cast<V*>(xout + g.idx(ib, j, kk)) = out;
          if constexpr (DOT) {
            // r.z: the colour-(1-c0) cells of plane k-1
#pragma unroll
            for (int q = 0; q < H; ++q) {
              if (ib + 2 * q + P < g.nx) {
                const double z = (double)blk[q];
                dv[0] += ((double)bin.rh[q] - shd) * z;
                dv[1] += z;
              }
            }
          }
        }
      }
      // --- the march state moves one plane up
#pragma unroll
      for (int q = 0; q < H; ++q) {
        red_m2[q] = red_m1[q];
        red_m1[q] = red_k[q];
        xh_m[q] = xh_0[q];
        xh_0[q] = xh_p[q];
      }
    };

    // the steps in pairs, so that the parity and the roles of the two
    // operand sets are compile-time constants
    auto march = [&](auto P0c) {
      constexpr int P0 = decltype(P0c)::value;
      for (int k = kb; k <= z1; k += 2) {
        step(std::integral_constant<int, P0>{}, k, opA, opB, blB, blA);
        if (k + 1 <= z1) step(std::integral_constant<int, 1 - P0>{}, k + 1, opB, opA, blA, blB);
      }
    };
    if (pk) march(std::integral_constant<int, 1>{});
    else march(std::integral_constant<int, 0>{});
    zm_wait();        // the last step's phase
    __syncthreads();  // the shared planes are reused by the next item
  }

  if constexpr (DOT) {
    const Op ops[2] = {Op::Sum, Op::Sum};
    double out[2];
    if (grid_reduce<2, NT>(dv, ops, red, 0, out)) {
      if (tid == 0 && !(s->done)) {
        const double rz_new = out[0];
        if (!isfinite(rz_new)) { s->status = 3; s->done = 1; }
        else if (!(rz_new > 0.0)) { s->status = 2; s->done = 1; }
        else {
          s->beta = s->first ? 0.0 : rz_new / s->rz;
          s->rz = rz_new;
          s->zshift = out[1] * s->inv_nfluid;
          s->first = 0;
        }
      }
    }
  }
}

}  // namespace smac
