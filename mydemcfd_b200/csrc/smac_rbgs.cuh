// smac_rbgs.cuh -- fused red-black Gauss-Seidel sweep (both colours in one
// pass over HBM), out of place: xout = S(xin).
//
// S updates colour c0 from xin, then colour c1 = 1 - c0 from the new c0
// values (pre-smoothing c0 = red, post-smoothing c0 = black, which keeps the
// V-cycle symmetric).  A CTA owns a TX x TY column of cells and marches z
// through its chunk [z0, z1):
//   - plane k+1 of xin (tile + 2-cell ring) is staged in shared memory,
//   - colour c0 is computed on plane k over the tile + 1-cell ring (the ring
//     values are recomputed here, so the c1 update at the tile edge never
//     reads another CTA's output and the result is independent of block
//     scheduling),
//   - colour c1 is computed on plane k-1 and the finished row pairs of
//     plane k-1 are written with one vector store per pair.
// HBM traffic per cell: xin, rhs and three face coefficients read once and
// xout written once (6 values), the algorithmic minimum of a full sweep;
// the ring re-reads hit L2.  Arithmetic is the same expression, in the same
// order, as the two half-sweep kernels (k_rbgs), so the result is bitwise
// identical to them.
//
// MODE 0: plain sweep.  MODE 1: xin == 0 (first pre-smoothing sweep), not
// read.  MODE 2: xin + coarse correction xc[parent] (prolongation fused into
// the first post-smoothing sweep).
// DOT: also accumulate sum((rhs - shift) * xout) and sum(xout) and finish
// r.z / beta in the last block (the PCG dot product of the preconditioned
// residual, fused into the last sweep of the fine grid).
#pragma once

#include <type_traits>

#include "smac_kernels.cuh"

namespace smac {

constexpr int RB_TX = 64;
constexpr int RB_NT = 256;
// tile height: 16 rows for FP32, 8 for FP64 (static shared memory < 48 KB)
template <class T> struct RbTile { static constexpr int TY = sizeof(T) == 8 ? 8 : 16; };


template <class T, class C, int MODE, bool DOT>
__global__ void __launch_bounds__(RB_NT) k_rbgs_sweep(Geom g, const T* __restrict__ xin, T* __restrict__ xout,
                                                      const T* __restrict__ rhs, const double* shift, Stencil<T, C> S,
                                                      int c0, const T* __restrict__ xc, Geom gc, int cx, int cy, int cz,
                                                      Scalars* s, RedBuf red, int zchunk) {
  pdl_enter();
  typedef acc_t<T> A;
  constexpr int TX = RB_TX, TY = RbTile<T>::TY;
  constexpr int XW = TX + 8;  // staged xin columns i0-4 .. i0+TX+3
  constexpr int XH = TY + 4;  // staged xin rows    j0-2 .. j0+TY+1
  constexpr int RW = TX + 2;  // c0 region columns  i0-1 .. i0+TX
  constexpr int RH = TY + 2;  // c0 region rows     j0-1 .. j0+TY
  __shared__ A Xs[MODE == 1 ? 1 : 3][XH][XW];
  __shared__ A Rs[3][RH][RW];
  if (s && s->done) return;
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int z0 = blockIdx.z * zchunk;
  const int z1 = min(z0 + zchunk, g.nz);
  const double shd = shift ? *shift : 0.0;
  const A sh = (A)shd;
  auto slot = [](int k) { return (k + 3) % 3; };

  auto load_plane = [&](int k) {
    if constexpr (MODE != 1) {
      const int sl = slot(k);
      const bool kin = (k >= 0 && k < g.nz);
      for (int p = tid; p < XH * XW; p += RB_NT) {
        const int jj = p / XW, ii = p - jj * XW;
        const int i = i0 - 4 + ii, j = j0 - 2 + jj;
        A v = (A)0;
        if (kin && i >= 0 && i < g.nx && j >= 0 && j < g.ny) {
          v = (A)xin[g.idx(i, j, k)];
          if constexpr (MODE == 2)
            v = Ar<A>::add(v, (A)xc[gc.idx(cx ? i >> 1 : i, cy ? j >> 1 : j, cz ? k >> 1 : k)]);
        }
        Xs[sl][jj][ii] = v;
      }
    }
  };

  // colour c0 on plane k over the tile and its one-cell ring
  auto c0_plane = [&](int k) {
    const int rs = slot(k);
    const bool kin = (k >= 0 && k < g.nz);
    for (int q = tid; q < RH * (RW / 2); q += RB_NT) {
      const int jj = q / (RW / 2), m = q - jj * (RW / 2);
      const int j = j0 - 1 + jj;
      const int ibase = i0 - 1;
      const int ii = ((c0 - j - k - ibase) & 1) + 2 * m;
      const int i = ibase + ii;
      A out = (A)0;
      if (kin && i >= 0 && i < g.nx && j >= 0 && j < g.ny) {
        const int c = g.idx(i, j, k);
        A wxm, wxp, wym, wyp, wzm, wzp;
        S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
        const A bv = Ar<A>::add((A)rhs[c], -sh);
        if constexpr (MODE != 1) {
          const int xi = ii + 3, yj = jj + 1;  // position in Xs
          out = Stencil<T, C>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, Xs[rs][yj][xi - 1], Xs[rs][yj][xi + 1],
                                  Xs[rs][yj - 1][xi], Xs[rs][yj + 1][xi], Xs[slot(k - 1)][yj][xi],
                                  Xs[slot(k + 1)][yj][xi]);
        } else {
          out = Stencil<T, C>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, (A)0, (A)0, (A)0, (A)0, (A)0, (A)0);
        }
      }
      Rs[rs][jj][ii] = out;
    }
  };

  double dv[2] = {0.0, 0.0};
  // colour c1 on plane k over the tile; store both colours of plane k
  auto c1_plane = [&](int k) {
    const int rs = slot(k);
    for (int q = tid; q < TY * (TX / 2); q += RB_NT) {
      const int jj = q / (TX / 2), m = q - jj * (TX / 2);
      const int j = j0 + jj, i = i0 + 2 * m;
      if (j >= g.ny || i >= g.nx) continue;
      A val[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int ie = i + e;
        const int ri = ie - (i0 - 1), rj = jj + 1;  // position in Rs
        if (ie >= g.nx) { val[e] = (A)0; continue; }
        if (((ie + j + k) & 1) == c0) {
          val[e] = Rs[rs][rj][ri];
          continue;
        }
        const int c = g.idx(ie, j, k);
        A wxm, wxp, wym, wyp, wzm, wzp;
        S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
        const A bv = Ar<A>::add((A)rhs[c], -sh);
        val[e] = Stencil<T, C>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, Rs[rs][rj][ri - 1], Rs[rs][rj][ri + 1],
                                   Rs[rs][rj - 1][ri], Rs[rs][rj + 1][ri], Rs[slot(k - 1)][rj][ri],
                                   Rs[slot(k + 1)][rj][ri]);
      }
      const int c = g.idx(i, j, k);
      if (i + 1 < g.nx) {
        typename Vec2<T>::type v2;
        v2.x = (T)val[0];
        v2.y = (T)val[1];
        *reinterpret_cast<typename Vec2<T>::type*>(xout + c) = v2;
      } else {
        xout[c] = (T)val[0];
      }
      if constexpr (DOT) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (i + e < g.nx) {
            const double zv = (double)(T)val[e];
            dv[0] += ((double)rhs[c + e] - shd) * zv;
            dv[1] += zv;
          }
        }
      }
    }
  };

  load_plane(z0 - 2);
  load_plane(z0 - 1);
  load_plane(z0);
  __syncthreads();
  c0_plane(z0 - 1);
  __syncthreads();  // c0_plane read the slot that load_plane(z0 + 1) refills
  for (int k = z0; k <= z1; ++k) {
    load_plane(k + 1);
    __syncthreads();
    c0_plane(k);
    __syncthreads();
    if (k - 1 >= z0) c1_plane(k - 1);
  }

  if constexpr (DOT) {
    const Op ops[2] = {Op::Sum, Op::Sum};
    double out[2];
    if (grid_reduce<2, RB_NT>(dv, ops, red, 0, out)) {
      if (tid == 0) {
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

// d = (z - zshift) + beta d fused with q = A d and p.Ap (the direction
// update of the next iteration is folded into the matvec that needs it):
// reads z and the old d at the stencil points, writes the new d and q.
// zshift (the fluid mean of z) keeps d free of the constant null-space
// component of the pure-Neumann operator, which would otherwise make p.Ap a
// cancellation near the rounding floor; cells without unknowns keep d = 0.
// Each thread takes 16 bytes of consecutive cells of one row (4 FP32 or 2
// FP64) and marches kz planes: rows and planes move as 16-byte vectors, and
// x-neighbours across the vector edge come from the adjacent lanes (lanes 0
// and 31 load them).
constexpr int DMV_TX = 32, DMV_TY = 4;
template <class T>
__global__ void __launch_bounds__(DMV_TX * DMV_TY) k_dir_matvec_vec(Geom g, const T* __restrict__ z,
                                                                    const T* __restrict__ d_old, T* __restrict__ d_new,
                                                                    Stencil<T, T> S, T* __restrict__ q,
                                                                    const uint8_t* __restrict__ fluid, RedBuf red,
                                                                    Scalars* s, int kz) {
  pdl_enter();
  if (s->done) return;
  typedef acc_t<T> A;
  typedef typename Vec16<T>::type V;
  constexpr int NV = Vec16<T>::n;
  const int lane = threadIdx.x;
  const int i0 = (blockIdx.x * DMV_TX + lane) * NV;
  const int j = blockIdx.y * DMV_TY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  const A beta = (A)s->beta;
  const A zs = (A)s->zshift;
  double v[1] = {0.0};
  // rows of this warp are uniform: the whole warp is in or out of the grid in j
  const bool row_in = j < g.ny;
  const bool any_in = i0 < g.nx;
  if (row_in && __any_sync(0xffffffffu, any_in)) {
    const int k1 = min(k0 + kz, g.nz);
    // lanes past the padded row read a valid vector of it and store nothing
    // (the lane after the last one in the grid still reads its own vector:
    // its first element is the neighbour of cell nx-1)
    int c = g.idx(i0 < g.px ? i0 : g.px - NV, j, k0);
    auto Dv = [&](int cc, A (&o)[NV]) {
      const V zz = *reinterpret_cast<const V*>(z + cc);
      const V dd = *reinterpret_cast<const V*>(d_old + cc);
      const T* zp = reinterpret_cast<const T*>(&zz);
      const T* dp = reinterpret_cast<const T*>(&dd);
#pragma unroll
      for (int e = 0; e < NV; ++e) o[e] = Ar<A>::fma(beta, (A)dp[e], Ar<A>::add((A)zp[e], -zs));
    };
    auto Ds = [&](int cc) -> A { return Ar<A>::fma(beta, (A)d_old[cc], Ar<A>::add((A)z[cc], -zs)); };
    A xm[NV], xc[NV], xp[NV];
    Dv(c - g.ps, xm);
    Dv(c, xc);
    V bzc = *reinterpret_cast<const V*>(S.bz + c);
    for (int k = k0; k < k1; ++k, c += g.ps) {
      Dv(c + g.ps, xp);
      A ym[NV], yp[NV];
      Dv(c - g.px, ym);
      Dv(c + g.px, yp);
      const V bxv = *reinterpret_cast<const V*>(S.bx + c);
      const V byv = *reinterpret_cast<const V*>(S.by + c);
      const V byu = *reinterpret_cast<const V*>(S.by + c + g.px);
      const V bzu = *reinterpret_cast<const V*>(S.bz + c + g.ps);
      const T* bxs = reinterpret_cast<const T*>(&bxv);
      const T* bys = reinterpret_cast<const T*>(&byv);
      const T* byus = reinterpret_cast<const T*>(&byu);
      const T* bzs = reinterpret_cast<const T*>(&bzc);
      const T* bzus = reinterpret_cast<const T*>(&bzu);
      // the vector's mask bytes in one load (c is a multiple of NV)
      uint8_t fl[NV];
      {
        typedef typename std::conditional<NV == 4, uint32_t, uint16_t>::type MW;
        const MW mw = *reinterpret_cast<const MW*>(fluid + c);
#pragma unroll
        for (int e = 0; e < NV; ++e) fl[e] = (uint8_t)(mw >> (8 * e));
      }
      // centre values with the fluid mask applied, as stored in d_new
      A xcm[NV];
#pragma unroll
      for (int e = 0; e < NV; ++e) xcm[e] = (fl[e] & 2) ? xc[e] : (A)0;
      // x-neighbours across the vector edge (the unmasked D, as k_dir_matvec reads them)
      A left = __shfl_up_sync(0xffffffffu, xc[NV - 1], 1);
      A right = __shfl_down_sync(0xffffffffu, xc[0], 1);
      T bxr = __shfl_down_sync(0xffffffffu, bxs[0], 1);
      if (lane == 0) left = Ds(c - 1);
      if (lane == DMV_TX - 1) {
        right = Ds(c + NV);
        bxr = S.bx[c + NV];
      }
      A y[NV];
#pragma unroll
      for (int e = 0; e < NV; ++e) {
        const A wxm = (A)bxs[e], wxp = (A)(e + 1 < NV ? bxs[e + 1] : bxr);
        const A nl = e > 0 ? xc[e - 1] : left, nr = e + 1 < NV ? xc[e + 1] : right;
        y[e] = Stencil<T, T>::apply(xcm[e], wxm, wxp, (A)bys[e], (A)byus[e], (A)bzs[e], (A)bzus[e], nl, nr, ym[e], yp[e],
                                    xm[e], xp[e]);
      }
      if (any_in) {
        V dn, qn;
        T* dns = reinterpret_cast<T*>(&dn);
        T* qns = reinterpret_cast<T*>(&qn);
#pragma unroll
        for (int e = 0; e < NV; ++e) {
          const bool in = i0 + e < g.nx;
          dns[e] = in ? (T)xcm[e] : (T)0;
          qns[e] = in ? (T)y[e] : (T)0;
          if (in) v[0] += (double)dns[e] * (double)qns[e];
        }
        *reinterpret_cast<V*>(d_new + c) = dn;
        *reinterpret_cast<V*>(q + c) = qn;
      }
#pragma unroll
      for (int e = 0; e < NV; ++e) {
        xm[e] = xcm[e];
        xc[e] = xp[e];
      }
      bzc = bzu;
    }
  }
  const Op ops[1] = {Op::Sum};
  double out[1];
  if (grid_reduce<1, DMV_TX * DMV_TY>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      const double pAp = out[0];
      s->pAp = pAp;
      if (!isfinite(pAp)) { s->status = 3; s->done = 1; }
      else if (!(pAp > 0.0)) { s->status = 2; s->done = 1; }
      else s->alpha = s->rz / pAp;
    }
  }
}

// Number of interior cells where a and b differ bitwise (self-test).
template <class T>
__global__ void k_count_mismatch(Geom g, const T* __restrict__ a, const T* __restrict__ b, unsigned long long* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = g.idx(i, j, k);
  if (!(a[c] == b[c]) && !(a[c] != a[c] && b[c] != b[c])) atomicAdd(cnt, 1ull);
}

}  // namespace smac
