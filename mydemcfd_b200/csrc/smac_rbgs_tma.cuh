// smac_rbgs_tma.cuh -- the fused red-black Gauss-Seidel sweep with its input
// tiles staged by the Tensor Memory Accelerator.
//
// Same mathematics and the same rounding as k_rbgs_sweep (and therefore as the
// two half-sweep kernels): xout = S(xin), colour c0 from xin, then colour
// 1-c0 from the new c0 values.  What changes is how the data arrive:
//
//   - persistent CTAs (two per SM) walk (z-chunk, column tile) items in
//     z-chunk-major order, each item a z-march over its chunk;
//   - plane p of the five inputs (xin tile + 2-cell ring; rhs, bx, by, bz tiles
//     + 1-cell ring) forms one stage, loaded by five cp.async.bulk.tensor 3-D
//     tile copies issued by one thread and completing on one mbarrier;
//   - NS stages live in a shared-memory ring fed as one stream across the
//     CTA's items: while plane k is computed, planes k+2 and k+3 (or the next
//     item's first planes) are in flight;
//   - step k computes colour c0 on plane k (tile + ring, from the staged
//     xin) and, after the step's one barrier, colour 1-c0 on plane k-1 from
//     the c0 results of planes k-2 .. k, which stay in shared memory;
//   - out-of-bounds boxes are zero-filled by the copy engine, which is the
//     zero ghost of the layout; cells outside the domain are masked to zero.
// Every mbarrier wait is bounded: on expiry the CTA records SMAC_CUDA_ERROR in
// the solver state, drains its own copies (again bounded) and returns.
#pragma once

#include <cuda.h>

#include "smac_rbgs.cuh"

namespace smac {

#ifndef SMAC_TMA_NS
#define SMAC_TMA_NS 5
#endif
constexpr int TMA_NS = SMAC_TMA_NS;  // stages in the ring
constexpr long long TMA_WAIT_CYCLES = 2000000000LL;  // ~1 s of SM clock before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (clock64() - t0 < TMA_WAIT_CYCLES)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// 3-D tile copy global -> shared, completing on `bar` (no multicast).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Tile geometry of one stage for vector type T: 64 x 8 cells (FP32) or
// 32 x 8 (FP64), so that a 5-stage ring fits twice in an SM's shared memory.
// One thread per pair of cells (i0+2m, i0+2m+1) of one row: each pair holds
// one cell of either colour on every plane.
template <class T>
struct TmaTile {
  static constexpr int TX = sizeof(T) == 8 ? 32 : 64;
  static constexpr int TY = 8;
  static constexpr int NT = TX / 2 * TY;           // threads per CTA
  static constexpr int NRING = TX + 2 + TY;        // colour-c0 cells of the 1-cell ring, per plane
  static constexpr int NRS = 4;                    // planes of colour-c0 results kept
  static constexpr int XW = TX + 8;                // box width: columns i0-4 .. i0+TX+3 (16 B aligned start)
  static constexpr int XH = TY + 4;                // xin rows j0-2 .. j0+TY+1
  static constexpr int RH = TY + 2;                // rhs/bx/bz rows j0-1 .. j0+TY
  static constexpr int YH = TY + 3;                // by rows j0-1 .. j0+TY+1
  static constexpr int RW = TX + 2;                // c0 region columns i0-1 .. i0+TX
  static constexpr int pad128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int X_BYTES = XH * XW * (int)sizeof(T);
  static constexpr int R_BYTES = RH * XW * (int)sizeof(T);
  static constexpr int Y_BYTES = YH * XW * (int)sizeof(T);
  static constexpr int X_OFF = 0;
  static constexpr int R_OFF = pad128(X_OFF + X_BYTES);
  static constexpr int BX_OFF = pad128(R_OFF + R_BYTES);
  static constexpr int BY_OFF = pad128(BX_OFF + R_BYTES);
  static constexpr int BZ_OFF = pad128(BY_OFF + Y_BYTES);
  static constexpr int STAGE_BYTES = pad128(BZ_OFF + R_BYTES);
  static constexpr int TX_BYTES = X_BYTES + 3 * R_BYTES + Y_BYTES;  // bytes the copies deliver per stage
  static constexpr int RS_BYTES = pad128(NRS * RH * RW * (int)sizeof(T));
  static constexpr int SMEM_BYTES = TMA_NS * STAGE_BYTES + RS_BYTES + 128;  // + mbarriers
};

struct SweepMaps {
  CUtensorMap xin, rhs, bx, by, bz;
};

// The coarse-grid values the prolongation adds to the six neighbours of one
// fine cell on a grid halved in every direction: the cell's parent, and the
// parent's neighbour in x, y and z on the side the cell's parity selects.
template <class A>
struct Coarse4 {
  A c, x, y, z;
};

template <class T, int MODE, bool DOT>
__global__ void __launch_bounds__(TmaTile<T>::NT, 2)
    k_rbgs_tma(const __grid_constant__ SweepMaps maps, Geom g, T* __restrict__ xout, const double* shift, int c0,
               const T* __restrict__ xc, Geom gc, int cx, int cy, int cz, Scalars* s, RedBuf red, int zchunk) {
  pdl_enter();
  typedef acc_t<T> A;
  typedef TmaTile<T> L;
  constexpr int TX = L::TX, TY = L::TY, XW = L::XW, RW = L::RW, RH = L::RH, NT = L::NT, HP = TX / 2;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TMA_NS * L::STAGE_BYTES + L::RS_BYTES);
  A (*Rs)[RH][RW] = reinterpret_cast<A (*)[RH][RW]>(smem + TMA_NS * L::STAGE_BYTES);
  if (s && s->done) return;
  const int tid = threadIdx.x;
  const double shd = shift ? *shift : 0.0;
  const A sh = (A)shd;

  if (tid == 0) {
    for (int q = 0; q < TMA_NS; ++q) mbar_init(&bars[q], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // Work items are (z-chunk, column tile) in z-chunk-major order, taken with
  // a stride of the grid size: all column tiles of a z-slab are in flight
  // together, so the ring rows and columns one CTA reads from its
  // neighbours' tiles come from L2 rather than DRAM.
  const int ncx = (g.nx + TX - 1) / TX, ncy = (g.ny + TY - 1) / TY;
  const int ncol = ncx * ncy;
  const int items = ncol * ((g.nz + zchunk - 1) / zchunk);
  const int nmine = (int)blockIdx.x < items ? (items - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto item_of = [&](int n) { return (int)blockIdx.x + n * (int)gridDim.x; };
  auto first_plane = [&](int n) { return (item_of(n) / ncol) * zchunk - 2; };
  auto last_plane = [&](int n) { return min(g.nz, (item_of(n) / ncol) * zchunk + zchunk) + 1; };

  // Producer (thread 0): issues the CTA's stage stream in order, one stage
  // per slot released by the consumers.
  int pn = 0, pp = nmine > 0 ? first_plane(0) : 0, ppe = nmine > 0 ? last_plane(0) : 0;
  unsigned pgi = 0;
  auto issue_next = [&]() {
    if (pn >= nmine) return;
    const int col = item_of(pn) % ncol;
    const int i0 = (col % ncx) * TX, j0 = (col / ncx) * TY;
    unsigned char* st = smem + (pgi % TMA_NS) * L::STAGE_BYTES;
    uint64_t* bar = &bars[pgi % TMA_NS];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, (uint32_t)(MODE == 1 ? L::TX_BYTES - L::X_BYTES : L::TX_BYTES));
    if constexpr (MODE != 1) tma_load_3d(st + L::X_OFF, &maps.xin, i0 - 4, j0 - 2, pp, bar);
    tma_load_3d(st + L::R_OFF, &maps.rhs, i0 - 4, j0 - 1, pp, bar);
    tma_load_3d(st + L::BX_OFF, &maps.bx, i0 - 4, j0 - 1, pp, bar);
    tma_load_3d(st + L::BY_OFF, &maps.by, i0 - 4, j0 - 1, pp, bar);
    tma_load_3d(st + L::BZ_OFF, &maps.bz, i0 - 4, j0 - 1, pp, bar);
    ++pgi;
    if (++pp > ppe && ++pn < nmine) { pp = first_plane(pn); ppe = last_plane(pn); }
  };
  if (tid == 0)
    for (int q = 0; q < TMA_NS; ++q) issue_next();

  // this thread's pair: cells (i0 + 2m, i0 + 2m + 1) of row j0 + jr
  // A warp takes 16 pairs of each of two adjacent rows.  The colour-c0 cells
  // of the two rows sit at opposite parities and every tile row has an even
  // length, so the two half-warps read disjoint shared-memory banks.
  static_assert(HP % 16 == 0 && TY % 2 == 0, "tile shape");
  const int lane = tid & 31, wv = tid >> 5;
  const int m = (wv % (HP / 16)) * 16 + (lane & 15);
  const int jr = 2 * (wv / (HP / 16)) + (lane >> 4);
  unsigned cgi = 0;  // consumer: global index of the item's first stage
  bool failed = false;
  double dv[2] = {0.0, 0.0};

  for (int n = 0; n < nmine && !failed; ++n) {
    const int col = item_of(n) % ncol;
    const int i0 = (col % ncx) * TX, j0 = (col / ncx) * TY;
    const int kb = first_plane(n) + 2, ke = last_plane(n) - 1;
    const unsigned gbase = cgi;
    cgi += (unsigned)(ke - kb + 4);
    auto stage = [&](int p) { return smem + ((gbase + (unsigned)(p - kb + 2)) % TMA_NS) * L::STAGE_BYTES; };
    auto wait = [&](int p) -> bool {
      const unsigned gi = gbase + (unsigned)(p - kb + 2);
      return mbar_wait_bounded(&bars[gi % TMA_NS], (gi / TMA_NS) & 1u);
    };
    const int j = j0 + jr, ip = i0 + 2 * m;

    // Colour c0 at tile column xcol (xin tile coordinates: cell i = i0 - 4 + xcol)
    // and tile row jt (cell j = j0 - 1 + jt) of plane k; zero outside the domain.
    auto red_at = [&](int xcol, int jt, int k, const unsigned char* sm, const unsigned char* s0,
                      const unsigned char* sp, const Coarse4<A>& cv) -> A {
      const int ia = i0 - 4 + xcol, ja = j0 - 1 + jt;
      if (ia < 0 || ia >= g.nx || ja < 0 || ja >= g.ny || k < 0 || k >= g.nz) return (A)0;
      const T* Rh = reinterpret_cast<const T*>(s0 + L::R_OFF);
      const T* Bx = reinterpret_cast<const T*>(s0 + L::BX_OFF);
      const T* By = reinterpret_cast<const T*>(s0 + L::BY_OFF);
      const T* Bz0 = reinterpret_cast<const T*>(s0 + L::BZ_OFF);
      const T* Bz1 = reinterpret_cast<const T*>(sp + L::BZ_OFF);
      const int cr = jt * XW + xcol;
      const A bv = Ar<A>::add((A)Rh[cr], -sh);
      const A wxm = (A)Bx[cr], wxp = (A)Bx[cr + 1], wym = (A)By[cr], wyp = (A)By[cr + XW];
      const A wzm = (A)Bz0[cr], wzp = (A)Bz1[cr];
      if constexpr (MODE == 1) {
        return Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, (A)0, (A)0, (A)0, (A)0, (A)0, (A)0);
      } else {
        const T* Xm = reinterpret_cast<const T*>(sm + L::X_OFF);
        const T* X0 = reinterpret_cast<const T*>(s0 + L::X_OFF);
        const T* Xp = reinterpret_cast<const T*>(sp + L::X_OFF);
        const int cp = cr + XW;  // xin rows start one row lower
        A n0 = (A)X0[cp - 1], n1 = (A)X0[cp + 1], n2 = (A)X0[cp - XW], n3 = (A)X0[cp + XW];
        A n4 = (A)Xm[cp], n5 = (A)Xp[cp];
        if constexpr (MODE == 2) {
          // prolongation of the coarse correction, added to each neighbour
          if (cx && cy && cz) {
            // Halved in every direction: three neighbours share the cell's
            // coarse parent, the other three are the parent's neighbours
            // on the side the cell's parity selects.  A neighbour outside
            // the domain maps to a coarse ghost, which holds 0, like the
            // neighbour itself: no bounds test is needed.
            // (the values were loaded one step ahead, coarse4 below)
            const A c0v = cv.c, cxv = cv.x, cyv = cv.y, czv = cv.z;
            n0 = Ar<A>::add(n0, (ia & 1) ? c0v : cxv);
            n1 = Ar<A>::add(n1, (ia & 1) ? cxv : c0v);
            n2 = Ar<A>::add(n2, (ja & 1) ? c0v : cyv);
            n3 = Ar<A>::add(n3, (ja & 1) ? cyv : c0v);
            n4 = Ar<A>::add(n4, (k & 1) ? c0v : czv);
            n5 = Ar<A>::add(n5, (k & 1) ? czv : c0v);
          } else {
            auto P = [&](A v, int ib, int jb, int kc) -> A {
              if (ib < 0 || ib >= g.nx || jb < 0 || jb >= g.ny || kc < 0 || kc >= g.nz) return v;
              return Ar<A>::add(v, (A)xc[gc.idx(cx ? ib >> 1 : ib, cy ? jb >> 1 : jb, cz ? kc >> 1 : kc)]);
            };
            n0 = P(n0, ia - 1, ja, k); n1 = P(n1, ia + 1, ja, k);
            n2 = P(n2, ia, ja - 1, k); n3 = P(n3, ia, ja + 1, k);
            n4 = P(n4, ia, ja, k - 1); n5 = P(n5, ia, ja, k + 1);
          }
        }
        return Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, n0, n1, n2, n3, n4, n5);
      }
    };

    // Coarse values of a fine cell (MODE 2 on a grid halved in every
    // direction), loaded from L2 one step before the cell's update so that
    // the loads overlap the barrier and the colour-(1-c0) pass.
    const bool pro4 = MODE == 2 && cx && cy && cz;
    auto coarse4 = [&](int ia, int ja, int k) -> Coarse4<A> {
      Coarse4<A> q{(A)0, (A)0, (A)0, (A)0};
      if (pro4 && (unsigned)ia < (unsigned)g.nx && (unsigned)ja < (unsigned)g.ny && (unsigned)k < (unsigned)g.nz) {
        const T* C = xc + gc.idx(ia >> 1, ja >> 1, k >> 1);
        q.c = (A)C[0];
        q.x = (A)C[(ia & 1) ? 1 : -1];
        q.y = (A)C[(ja & 1) ? gc.px : -gc.px];
        q.z = (A)C[(k & 1) ? gc.ps : -gc.ps];
      }
      return q;
    };
    // the ring cell (tile coordinates) of this thread on plane k
    auto ring_cell = [&](int k, int& rc, int& rr) {
      if (tid < 2 * (HP + 1)) {
        rr = tid < HP + 1 ? 0 : TY + 1;
        const int t = tid < HP + 1 ? tid : tid - (HP + 1);
        rc = ((c0 + 1 + j0 - 1 + rr + k) & 1) + 2 * t;
      } else {
        const int t = tid - 2 * (HP + 1);
        const bool left = t < TY / 2;
        rc = left ? 0 : TX + 1;
        const int tt = left ? t : t - TY / 2;
        rr = 1 + (((left ? c0 + 1 : c0) + j0 + k) & 1) + 2 * tt;
      }
    };
    Coarse4<A> cm{}, cr4{};
    if (pro4) {
      cm = coarse4(ip + ((c0 + j + kb - 1) & 1), j, kb - 1);
      if (tid < L::NRING) {
        int rc, rr;
        ring_cell(kb - 1, rc, rr);
        cr4 = coarse4(i0 - 1 + rc, j0 - 1 + rr, kb - 1);
      }
    }

    A red_prev = (A)0;
    for (int k = kb - 1; k <= ke; ++k) {
      bool ok = true;
      if (k == kb - 1) ok = wait(k - 1) && wait(k);
      ok = ok && wait(k + 1);
      const unsigned char* sm = stage(k - 1);
      const unsigned char* s0 = stage(k);
      const unsigned char* sp = stage(k + 1);
      A (*Rk)[RW] = Rs[(k + 4) & 3];
      // main: the colour-c0 cell of this thread's pair
      const int e = (c0 + j + k) & 1;
      const A rk = red_at(2 * m + e + 4, jr + 1, k, sm, s0, sp, cm);
      Rk[jr + 1][2 * m + e + 1] = rk;
      // ring: rows j0-1 and j0+TY (HP+1 cells each), columns i0-1 and i0+TX (TY/2 each)
      if (tid < L::NRING) {
        int rc, rr;  // ring cell in result coordinates (column i - (i0-1), row j - (j0-1))
        ring_cell(k, rc, rr);
        Rk[rr][rc] = red_at(rc + 3, rr, k, sm, s0, sp, cr4);
      }
      if (pro4 && k + 1 <= ke) {  // next plane's coarse values
        cm = coarse4(ip + ((c0 + j + k + 1) & 1), j, k + 1);
        if (tid < L::NRING) {
          int rc, rr;
          ring_cell(k + 1, rc, rr);
          cr4 = coarse4(i0 - 1 + rc, j0 - 1 + rr, k + 1);
        }
      }
      if (__syncthreads_or(!ok)) { failed = true; break; }
      if (tid == 0 && k >= kb) issue_next();  // stage k-2 is free
      if (k - 1 >= kb) {
        // colour 1-c0 on plane kk = k-1 for this thread's pair
        const int kk = k - 1;
        const int eb = 1 - ((c0 + j + kk) & 1);
        const int rcb = 2 * m + eb + 1;  // result coordinates of the cell
        A (*Rm)[RW] = Rs[(kk + 3) & 3];
        A (*R0)[RW] = Rs[(kk + 4) & 3];
        const unsigned char* t0 = sm;  // stage kk
        const T* Rh = reinterpret_cast<const T*>(t0 + L::R_OFF);
        const T* Bx = reinterpret_cast<const T*>(t0 + L::BX_OFF);
        const T* By = reinterpret_cast<const T*>(t0 + L::BY_OFF);
        const T* Bz0 = reinterpret_cast<const T*>(t0 + L::BZ_OFF);
        const T* Bz1 = reinterpret_cast<const T*>(s0 + L::BZ_OFF);
        const int cr = (jr + 1) * XW + rcb + 3;
        A blk = (A)0;
        if (ip + eb < g.nx && j < g.ny) {
          const A bv = Ar<A>::add((A)Rh[cr], -sh);
          blk = Stencil<T, T>::gs(bv, (A)Bx[cr], (A)Bx[cr + 1], (A)By[cr], (A)By[cr + XW], (A)Bz0[cr], (A)Bz1[cr],
                                  R0[jr + 1][rcb - 1], R0[jr + 1][rcb + 1], R0[jr][rcb], R0[jr + 2][rcb],
                                  Rm[jr + 1][rcb], Rk[jr + 1][rcb]);
        }
        if (j < g.ny && ip < g.nx) {
          A v0 = eb ? red_prev : blk, v1 = eb ? blk : red_prev;
          const int c = g.idx(ip, j, kk);
          if (ip + 1 < g.nx) {
            typename Vec2<T>::type v2;
            v2.x = (T)v0;
            v2.y = (T)v1;
            *reinterpret_cast<typename Vec2<T>::type*>(xout + c) = v2;
          } else {
            xout[c] = (T)v0;
          }
          if constexpr (DOT) {
            const int crp = (jr + 1) * XW + 2 * m + 4;  // cell ip in tile coordinates
            const double z0 = (double)(T)v0;
            dv[0] += ((double)Rh[crp] - shd) * z0;
            dv[1] += z0;
            if (ip + 1 < g.nx) {
              const double z1 = (double)(T)v1;
              dv[0] += ((double)Rh[crp + 1] - shd) * z1;
              dv[1] += z1;
            }
          }
        }
      }
      red_prev = rk;
    }
    if (failed) {
      // Record the failure (the update kernel stops the solve on it; `done` is
      // not set here so that every CTA still joins the reduction below), then
      // wait, bounded, for every copy this CTA has issued and not consumed.
      if (tid == 0) {
        if (s) s->status = 6;
        for (unsigned gi = gbase; gi < pgi; ++gi) (void)mbar_wait_bounded(&bars[gi % TMA_NS], (gi / TMA_NS) & 1u);
      }
      __syncthreads();
      break;
    }
    __syncthreads();  // stages ke-1 .. ke+1 and the result planes are free
    if (tid == 0)
      for (int q = 0; q < 3; ++q) issue_next();
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
