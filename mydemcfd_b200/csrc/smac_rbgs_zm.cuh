// smac_rbgs_zm.cuh -- the fused red-black Gauss-Seidel sweep as a register
// z-march over whole x-rows.
//
// Same mathematics and rounding as k_rbgs_sweep, k_rbgs_tma and the two
// half-sweep kernels (k_rbgs): xout = S(xin), colour c0 from xin, then colour
// 1-c0 from the new c0 values.  The data movement is different:
//
//   - a warp owns 32 x NV consecutive cells of one row (NV = 4 FP32, 2 FP64,
//     one 16-byte vector per lane and array), WX warps side by side cover the
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
//   - one shared-memory plane per step carries each row to the rows above
//     and below: the input vector of plane k+1 is stored whole, the c0
//     results of plane k over it; four planes rotate (a plane is written at
//     step k-1 and k and last read at step k+1, by the slowest warp before
//     the barrier of step k+2);
//   - the loads of step k+1 (input, rhs, weights) are issued at the start of
//     step k, so one step of global latency is hidden behind the arithmetic
//     of the step.
// Step k computes colour c0 on plane k, then (after the step's one barrier)
// colour 1-c0 on plane k-1, whose finished vector is stored.
//
// Algorithmic HBM bytes per cell: xin, rhs, bx, by, bz read, xout written
// (6 values); the ring rows and the by row above are re-read from L1/L2.
#pragma once

#include "smac_rbgs.cuh"

namespace smac {

template <class T, int WX, int TY>
struct ZmTile {
  static constexpr int NV = Vec16<T>::n;          // cells per lane
  static constexpr int H = NV / 2;                // cells of one colour per lane and plane
  static constexpr int TW = 32 * NV * WX;         // cells per row: the whole x extent
  static constexpr int ROWS = TY + 2;             // tile rows plus the two ring rows
  static constexpr int NT = 32 * WX * ROWS;       // threads per CTA
  static constexpr int NB = 4;                    // shared planes in rotation
  static constexpr int SMEM = NB * ROWS * TW * (int)sizeof(T);
};

template <class T, int WX, int TY, int MODE, bool DOT>
__global__ void __launch_bounds__(ZmTile<T, WX, TY>::NT)
    k_rbgs_zm(Geom g, const T* __restrict__ xin, T* __restrict__ xout, const T* __restrict__ rhs, const double* shift,
              Stencil<T, T> S, int c0, const T* __restrict__ xc, Geom gc, int cx, int cy, int cz, Scalars* s,
              RedBuf red, int zchunk) {
  typedef ZmTile<T, WX, TY> L;
  typedef typename Vec16<T>::type V;
  typedef T A;
  constexpr int NV = L::NV, H = L::H, TW = L::TW, ROWS = L::ROWS, NT = L::NT;
  extern __shared__ __align__(16) unsigned char zm_smem[];
  T* M = reinterpret_cast<T*>(zm_smem);  // [NB][ROWS][TW]
  if (s && s->done) return;
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
  double dv[2] = {0.0, 0.0};

  auto zero = []() {
    V v;
    T* p = reinterpret_cast<T*>(&v);
#pragma unroll
    for (int e = 0; e < NV; ++e) p[e] = (T)0;
    return v;
  };
  auto el = [](const V& v, int e) -> T { return reinterpret_cast<const T*>(&v)[e]; };
  // element 2q + p of v, and the x+ face of cell 2q + p (element 2q + p + 1,
  // or `edge` past the vector); q is a compile-time constant of the unrolled
  // loops and p a warp-uniform parity, so both are register selects
  auto at = [&](const V& v, int q, int p) -> T { return p ? el(v, 2 * q + 1) : el(v, 2 * q); };
  auto at_next = [&](const V& v, T edge, int q, int p) -> T {
    return p ? (2 * q + 2 < NV ? el(v, 2 * q + 2) : edge) : el(v, 2 * q + 1);
  };

  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int ty = item % nty, zi = item / nty;
    const int j0 = ty * TY;
    const int j = j0 - 1 + wr;  // this warp's row
    const bool row_ok = j >= 0 && j < g.ny;
    const int z0 = zi * zchunk, z1 = min(z0 + zchunk, g.nz);
    const int jo = wr == 0 ? j - 1 : j + 1;  // ring warps: the row beyond the ring
    const bool jo_ok = ring && jo >= 0 && jo < g.ny;
    const bool col_any = col_ok;

    // the input vector of plane m, row jj (the coarse correction added in MODE 2); 0 outside the grid
    auto load_x = [&](int m, int jj, bool ok) -> V {
      if constexpr (MODE == 1) return zero();
      if (!ok || !col_any || m < 0 || m >= g.nz) return zero();
      V v = *reinterpret_cast<const V*>(xin + g.idx(ib, jj, m));
      if constexpr (MODE == 2) {
        T* p = reinterpret_cast<T*>(&v);
#pragma unroll
        for (int e = 0; e < NV; ++e) {
          const int i = ib + e;
          if (i < g.nx) p[e] = (T)Ar<A>::add((A)p[e], (A)xc[gc.idx(cx ? i >> 1 : i, cy ? jj >> 1 : jj, cz ? m >> 1 : m)]);
        }
      }
      return v;
    };
    auto load_v = [&](const T* a, int m, int jj, bool ok) -> V {
      if (!ok || !col_any) return zero();
      return *reinterpret_cast<const V*>(a + g.idx(ib, jj, m));
    };
    auto load_s = [&](const T* a, int idx, bool ok) -> T { return ok ? a[idx] : (T)0; };

    // operands of the colour-c0 pass on plane m (loaded one step ahead)
    struct Ops {
      V rh, bx, by, byu, bzu;  // rhs, x-faces, y-faces j and j+1, z-faces m+1
      T bxe;                   // x-face ib+NV
    };
    auto load_ops = [&](int m) -> Ops {
      Ops o;
      const bool ok = row_ok && m >= 0 && m < g.nz;
      o.rh = load_v(rhs, m, j, ok);
      o.bx = load_v(S.bx, m, j, ok);
      o.bxe = load_s(S.bx, g.idx(ib + NV, j, m), ok && col_ok && ib + NV <= g.nx);
      o.by = load_v(S.by, m, j, ok);
      o.byu = load_v(S.by, m, j + 1, ok);
      o.bzu = load_v(S.bz, m + 1, j, row_ok && m + 1 >= 0 && m + 1 <= g.nz);  // z-face m+1 (0..nz)
      return o;
    };

    // prologue: the inputs of the first c0 plane (z0 - 1) and the shared plane z0 - 1
    const int kb = z0 - 1;
    V xv_m = load_x(kb - 1, j, row_ok);  // plane kb-1
    V xv_0 = load_x(kb, j, row_ok);      // plane kb
    V xv_p = load_x(kb + 1, j, row_ok);  // plane kb+1
    V xo_0 = load_x(kb, jo, jo_ok);      // ring warps: the row beyond, plane kb
    V xo_p = load_x(kb + 1, jo, jo_ok);
    V bz_c = load_v(S.bz, kb, j, row_ok && kb >= 0 && kb < g.nz);  // z-faces of plane kb
    Ops cur = load_ops(kb);
    *reinterpret_cast<V*>(Mrow(kb, wr) + ib) = xv_0;
    // colour-(1-c0) inputs of planes kb-1 and kb at the c0 positions of plane kb
    const int pk = (c0 + j + kb) & 1;  // parity of the c0 cells of plane kb in this row
    T xh_m[H], xh_0[H];
#pragma unroll
    for (int q = 0; q < H; ++q) {
      xh_m[q] = at(xv_m, q, pk);
      xh_0[q] = at(xv_0, q, pk ^ 1);
    }
    // c0 results kept for the colour-(1-c0) pass, and its operands
    T red_m2[H], red_m1[H];
    T b_rh[H], b_bxm[H], b_bxp[H], b_by[H], b_byu[H], b_bz[H], b_bzu[H];
    V b_rhs_full;
#pragma unroll
    for (int q = 0; q < H; ++q)
      red_m2[q] = red_m1[q] = b_rh[q] = b_bxm[q] = b_bxp[q] = b_by[q] = b_byu[q] = b_bz[q] = b_bzu[q] = (T)0;
    b_rhs_full = zero();
    __syncthreads();

    for (int k = kb; k <= z1; ++k) {
      const int p = (c0 + j + k) & 1;  // c0 cells of plane k sit at e = p, p+2, ...; colour-(1-c0) cells of k-1 too
      // --- issue the loads of step k+1
      const bool more = k + 1 <= z1;
      V nx_p = zero(), no_p = zero();
      Ops nxt{};
      if (more) {
        nx_p = load_x(k + 2, j, row_ok);
        no_p = load_x(k + 2, jo, jo_ok);
        nxt = load_ops(k + 1);
      }
      // --- the input of plane k+1 becomes visible to the rows above and below
      *reinterpret_cast<V*>(Mrow(k + 1, wr) + ib) = xv_p;
      T xh_p[H];
#pragma unroll
      for (int q = 0; q < H; ++q) xh_p[q] = at(xv_p, q, p);  // colour 1-c0 of plane k+1 at positions p + 2q
      // --- colour c0 on plane k
      T red_k[H];
      const bool plane_ok = k >= 0 && k < g.nz;
      {
        const T* Mk = Mrow(k, 0);
        // x-neighbours across the vector edge: colour-(1-c0) inputs of plane k
        T left = __shfl_up_sync(0xffffffffu, xh_0[H - 1], 1);
        T right = __shfl_down_sync(0xffffffffu, xh_0[0], 1);
        if (lane == 0) left = wx > 0 ? Mk[wr * TW + ib - 1] : (T)0;
        if (lane == 31) right = wx < WX - 1 ? Mk[wr * TW + ib + NV] : (T)0;
        V ym, yp;
        if (wr == 0) ym = xo_0; else ym = *reinterpret_cast<const V*>(Mk + (wr - 1) * TW + ib);
        if (wr == ROWS - 1) yp = xo_0; else yp = *reinterpret_cast<const V*>(Mk + (wr + 1) * TW + ib);
#pragma unroll
        for (int q = 0; q < H; ++q) {
          const int e = 2 * q + p;
          A v = (A)0;
          if (row_ok && plane_ok && ib + e < g.nx) {
            const A bv = Ar<A>::add((A)at(cur.rh, q, p), -sh);
            const A wxm = (A)at(cur.bx, q, p);
            const A wxp = (A)at_next(cur.bx, cur.bxe, q, p);
            const A wym = (A)at(cur.by, q, p), wyp = (A)at(cur.byu, q, p);
            const A wzm = (A)at(bz_c, q, p), wzp = (A)at(cur.bzu, q, p);
            if constexpr (MODE == 1) {
              v = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, (A)0, (A)0, (A)0, (A)0, (A)0, (A)0);
            } else {
              // colour-(1-c0) positions of plane k: e-1 and e+1
              const A n0 = (A)(p == 0 ? (q > 0 ? xh_0[q - 1] : left) : xh_0[q]);
              const A n1 = (A)(p == 0 ? xh_0[q] : (q + 1 < H ? xh_0[q + 1] : right));
              v = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, n0, n1, (A)at(ym, q, p), (A)at(yp, q, p),
                                    (A)xh_m[q], (A)xh_p[q]);
            }
          }
          red_k[q] = (T)v;
        }
        // c0 results of plane k over the input in the shared plane
        T* Mw = Mrow(k, wr) + ib;
        if (row_ok && plane_ok && col_ok) {
#pragma unroll
          for (int q = 0; q < H; ++q) Mw[2 * q + p] = red_k[q];
        }
      }
      // operands of the colour-(1-c0) pass on plane k (next step), at positions (p^1) + 2q
      T n_rh[H], n_bxm[H], n_bxp[H], n_by[H], n_byu[H], n_bz[H], n_bzu[H];
      {
        const int pb = p ^ 1;
#pragma unroll
        for (int q = 0; q < H; ++q) {
          n_rh[q] = at(cur.rh, q, pb);
          n_bxm[q] = at(cur.bx, q, pb);
          n_bxp[q] = at_next(cur.bx, cur.bxe, q, pb);
          n_by[q] = at(cur.by, q, pb);
          n_byu[q] = at(cur.byu, q, pb);
          n_bz[q] = at(bz_c, q, pb);
          n_bzu[q] = at(cur.bzu, q, pb);
        }
      }
      const V n_rhs_full = cur.rh;
      __syncthreads();
      // --- colour 1-c0 on plane k-1 (tile rows only)
      const int kk = k - 1;
      if (!ring && kk >= z0 && kk < z1) {
        const T* Mp = Mrow(kk, 0);
        // c0 results of plane k-1 sit at positions (p^1) + 2q; the cells updated now at p + 2q
        T left = __shfl_up_sync(0xffffffffu, red_m1[H - 1], 1);
        T right = __shfl_down_sync(0xffffffffu, red_m1[0], 1);
        if (lane == 0) left = wx > 0 ? Mp[wr * TW + ib - 1] : (T)0;
        if (lane == 31) right = wx < WX - 1 ? Mp[wr * TW + ib + NV] : (T)0;
        const V ym = *reinterpret_cast<const V*>(Mp + (wr - 1) * TW + ib);
        const V yp = *reinterpret_cast<const V*>(Mp + (wr + 1) * TW + ib);
        T blk[H];
#pragma unroll
        for (int q = 0; q < H; ++q) {
          const int e = 2 * q + p;
          A v = (A)0;
          if (row_ok && ib + e < g.nx) {
            const A bv = Ar<A>::add((A)b_rh[q], -sh);
            const A n0 = (A)(p == 0 ? (q > 0 ? red_m1[q - 1] : left) : red_m1[q]);
            const A n1 = (A)(p == 0 ? red_m1[q] : (q + 1 < H ? red_m1[q + 1] : right));
            v = Stencil<T, T>::gs(bv, (A)b_bxm[q], (A)b_bxp[q], (A)b_by[q], (A)b_byu[q], (A)b_bz[q], (A)b_bzu[q], n0,
                                  n1, (A)at(ym, q, p), (A)at(yp, q, p), (A)red_m2[q], (A)red_k[q]);
          }
          blk[q] = (T)v;
        }
        if (row_ok && col_ok) {
          V out;
          T* o = reinterpret_cast<T*>(&out);
#pragma unroll
          for (int q = 0; q < H; ++q) {
            o[2 * q] = p ? red_m1[q] : blk[q];
            o[2 * q + 1] = p ? blk[q] : red_m1[q];
          }
          *reinterpret_cast<V*>(xout + g.idx(ib, j, kk)) = out;
          if constexpr (DOT) {
#pragma unroll
            for (int e = 0; e < NV; ++e) {
              if (ib + e < g.nx) {
                const double z = (double)o[e];
                dv[0] += ((double)el(b_rhs_full, e) - shd) * z;
                dv[1] += z;
              }
            }
          }
        }
      }
      // --- rotate the march state
#pragma unroll
      for (int q = 0; q < H; ++q) {
        red_m2[q] = red_m1[q];
        red_m1[q] = red_k[q];
        xh_m[q] = xh_0[q];
        b_rh[q] = n_rh[q];
        b_bxm[q] = n_bxm[q];
        b_bxp[q] = n_bxp[q];
        b_by[q] = n_by[q];
        b_byu[q] = n_byu[q];
        b_bz[q] = n_bz[q];
        b_bzu[q] = n_bzu[q];
      }
      b_rhs_full = n_rhs_full;
      // colour-(1-c0) inputs of plane k+1 (its cells at parity p)
#pragma unroll
      for (int q = 0; q < H; ++q) xh_0[q] = xh_p[q];
      xv_p = nx_p;
      xo_0 = xo_p;
      xo_p = no_p;
      bz_c = cur.bzu;
      cur = nxt;
    }
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
