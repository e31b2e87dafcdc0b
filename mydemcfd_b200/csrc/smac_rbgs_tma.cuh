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
//   - NS stages live in a shared-memory ring: while plane k is computed,
//     planes k+2 .. k+NS-2 are in flight, which hides the DRAM latency that
//     bounded the register-staged kernel;
//   - out-of-bounds boxes are zero-filled by the copy engine, which is the
//     zero ghost of the layout; cells outside the domain are masked to zero.
// Every mbarrier wait is bounded: on expiry the CTA records SMAC_CUDA_ERROR in
// the solver state, drains its own copies (again bounded) and returns.
#pragma once

#include <cuda.h>

#include "smac_rbgs.cuh"

namespace smac {

constexpr int TMA_NS = 5;        // stages in the ring
constexpr int TMA_NT = 256;      // threads per CTA
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
template <class T>
struct TmaTile {
  static constexpr int TX = sizeof(T) == 8 ? 32 : 64;
  static constexpr int TY = 8;
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
  static constexpr int RS_BYTES = pad128(3 * RH * RW * (int)sizeof(T));
  static constexpr int SMEM_BYTES = TMA_NS * STAGE_BYTES + RS_BYTES + 128;  // + mbarriers
};

struct SweepMaps {
  CUtensorMap xin, rhs, bx, by, bz;
};

template <class T, int MODE, bool DOT>
__global__ void __launch_bounds__(TMA_NT, 2)
    k_rbgs_tma(const __grid_constant__ SweepMaps maps, Geom g, T* __restrict__ xout, const double* shift, double ihx2,
               double ihy2, double ihz2, int c0, const T* __restrict__ xc, Geom gc, int cx, int cy, int cz, Scalars* s,
               RedBuf red, int zchunk) {
  typedef acc_t<T> A;
  typedef TmaTile<T> L;
  constexpr int TX = L::TX, TY = L::TY, XW = L::XW, RW = L::RW, RH = L::RH;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TMA_NS * L::STAGE_BYTES + L::RS_BYTES);
  A (*Rs)[RH][RW] = reinterpret_cast<A (*)[RH][RW]>(smem + TMA_NS * L::STAGE_BYTES);
  if (s && s->done) return;
  const int tid = threadIdx.x;
  const A sh = shift ? (A)(*shift) : (A)0;
  const A hx = (A)ihx2, hy = (A)ihy2, hz = (A)ihz2;

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
  const int nzc = (g.nz + zchunk - 1) / zchunk;
  const int items = ncol * nzc;
  long long gstage = 0;  // stages issued by this CTA so far (mbarrier phase bookkeeping)
  bool failed = false;
  double dv[2] = {0.0, 0.0};

  auto stage_ptr = [&](long long gi) { return smem + (gi % TMA_NS) * L::STAGE_BYTES; };
  auto tileX = [&](long long gi) { return reinterpret_cast<const T*>(stage_ptr(gi) + L::X_OFF); };
  auto tileR = [&](long long gi) { return reinterpret_cast<const T*>(stage_ptr(gi) + L::R_OFF); };
  auto tileBX = [&](long long gi) { return reinterpret_cast<const T*>(stage_ptr(gi) + L::BX_OFF); };
  auto tileBY = [&](long long gi) { return reinterpret_cast<const T*>(stage_ptr(gi) + L::BY_OFF); };
  auto tileBZ = [&](long long gi) { return reinterpret_cast<const T*>(stage_ptr(gi) + L::BZ_OFF); };

  for (int item = blockIdx.x; item < items && !failed; item += gridDim.x) {
    const int col = item % ncol;
    const int kb = (item / ncol) * zchunk;
    const int ke = min(g.nz, kb + zchunk);
    const int i0 = (col % ncx) * TX, j0 = (col / ncx) * TY;
    const int pb = kb - 2, pe = ke + 1;  // stages (planes) of this piece
    const long long gbase = gstage;      // global index of stage pb
    const int nst = pe - pb + 1;
    gstage += nst;
    auto gidx = [&](int p) { return gbase + (p - pb); };
    auto issue = [&](int p) {  // thread 0 only
      const long long gi = gidx(p);
      unsigned char* st = stage_ptr(gi);
      uint64_t* bar = &bars[gi % TMA_NS];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(bar, (uint32_t)(MODE == 1 ? L::TX_BYTES - L::X_BYTES : L::TX_BYTES));
      if constexpr (MODE != 1) tma_load_3d(st + L::X_OFF, &maps.xin, i0 - 4, j0 - 2, p, bar);
      tma_load_3d(st + L::R_OFF, &maps.rhs, i0 - 4, j0 - 1, p, bar);
      tma_load_3d(st + L::BX_OFF, &maps.bx, i0 - 4, j0 - 1, p, bar);
      tma_load_3d(st + L::BY_OFF, &maps.by, i0 - 4, j0 - 1, p, bar);
      tma_load_3d(st + L::BZ_OFF, &maps.bz, i0 - 4, j0 - 1, p, bar);
    };
    auto wait = [&](int p) -> bool {
      const long long gi = gidx(p);
      return mbar_wait_bounded(&bars[gi % TMA_NS], (uint32_t)((gi / TMA_NS) & 1));
    };
    if (tid == 0)
      for (int p = pb; p <= min(pe, pb + TMA_NS - 1); ++p) issue(p);

    // colour c0 on plane k over the tile + ring; stages k-1, k, k+1 resident
    auto c0_plane = [&](int k) {
      const int rs = (k + 3) % 3;
      const bool kin = (k >= 0 && k < g.nz);
      const T* Xm = tileX(gidx(k - 1));
      const T* X0 = tileX(gidx(k));
      const T* Xp = tileX(gidx(k + 1));
      const T* Rh = tileR(gidx(k));
      const T* Bx = tileBX(gidx(k));
      const T* By = tileBY(gidx(k));
      const T* Bz0 = tileBZ(gidx(k));
      const T* Bz1 = tileBZ(gidx(k + 1));
      for (int q = tid; q < RH * (RW / 2); q += TMA_NT) {
        const int jj = q / (RW / 2), m = q - jj * (RW / 2);
        const int j = j0 - 1 + jj;
        const int ibase = i0 - 1;
        const int ii = ((c0 - j - k - ibase) & 1) + 2 * m;
        const int i = ibase + ii;
        A out = (A)0;
        if (kin && i >= 0 && i < g.nx && j >= 0 && j < g.ny) {
          const int cr = jj * XW + ii + 3;        // rhs / bx / by / bz position
          const int cxp = (jj + 1) * XW + ii + 3;  // xin position
          const A wxm = Ar<A>::mul((A)Bx[cr], hx), wxp = Ar<A>::mul((A)Bx[cr + 1], hx);
          const A wym = Ar<A>::mul((A)By[cr], hy), wyp = Ar<A>::mul((A)By[cr + XW], hy);
          const A wzm = Ar<A>::mul((A)Bz0[cr], hz), wzp = Ar<A>::mul((A)Bz1[cr], hz);
          const A bv = Ar<A>::add((A)Rh[cr], -sh);
          if constexpr (MODE == 1) {
            out = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, (A)0, (A)0, (A)0, (A)0, (A)0, (A)0);
          } else {
            auto XV = [&](const T* t, int pos, int ia, int ja, int ka) -> A {
              A v = (A)t[pos];
              if constexpr (MODE == 2) {
                if (ia >= 0 && ia < g.nx && ja >= 0 && ja < g.ny && ka >= 0 && ka < g.nz)
                  v = Ar<A>::add(v, (A)xc[gc.idx(cx ? ia >> 1 : ia, cy ? ja >> 1 : ja, cz ? ka >> 1 : ka)]);
              }
              return v;
            };
            out = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, XV(X0, cxp - 1, i - 1, j, k),
                                    XV(X0, cxp + 1, i + 1, j, k), XV(X0, cxp - XW, i, j - 1, k),
                                    XV(X0, cxp + XW, i, j + 1, k), XV(Xm, cxp, i, j, k - 1), XV(Xp, cxp, i, j, k + 1));
          }
        }
        Rs[rs][jj][ii] = out;
      }
    };

    // the march: c0 on planes kb-1 .. ke, c1 on kb .. ke-1
    int kfail = 0;
    for (int k = kb - 1; k <= ke && !failed; ++k) {
      // stages k-1, k, k+1 must have landed (k-1 and k were waited before)
      const int need_lo = (k == kb - 1) ? k - 1 : k + 1;
      for (int p = need_lo; p <= k + 1; ++p)
        if (!wait(p)) failed = true;
      if (failed) { kfail = k; break; }
      c0_plane(k);
      __syncthreads();
      if (k - 1 >= kb) {
        // inline c1 (needs the DOT accumulation on rhs values)
        const int kk = k - 1;
        const int rs = (kk + 3) % 3;
        const T* Rh = tileR(gidx(kk));
        const T* Bx = tileBX(gidx(kk));
        const T* By = tileBY(gidx(kk));
        const T* Bz0 = tileBZ(gidx(kk));
        const T* Bz1 = tileBZ(gidx(kk + 1));
        for (int q = tid; q < TY * (TX / 2); q += TMA_NT) {
          const int jj = q / (TX / 2), m = q - jj * (TX / 2);
          const int j = j0 + jj, i = i0 + 2 * m;
          if (j >= g.ny || i >= g.nx) continue;
          A val[2];
          A rv[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int ie = i + e;
            const int ri = ie - (i0 - 1), rj = jj + 1;
            const int cr = rj * XW + (ie - i0) + 4;
            rv[e] = (A)Rh[cr];
            if (ie >= g.nx) { val[e] = (A)0; continue; }
            if (((ie + j + kk) & 1) == c0) { val[e] = Rs[rs][rj][ri]; continue; }
            const A wxm = Ar<A>::mul((A)Bx[cr], hx), wxp = Ar<A>::mul((A)Bx[cr + 1], hx);
            const A wym = Ar<A>::mul((A)By[cr], hy), wyp = Ar<A>::mul((A)By[cr + XW], hy);
            const A wzm = Ar<A>::mul((A)Bz0[cr], hz), wzp = Ar<A>::mul((A)Bz1[cr], hz);
            const A bv = Ar<A>::add(rv[e], -sh);
            val[e] = Stencil<T, T>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, Rs[rs][rj][ri - 1], Rs[rs][rj][ri + 1],
                                       Rs[rs][rj - 1][ri], Rs[rs][rj + 1][ri], Rs[(kk + 2) % 3][rj][ri],
                                       Rs[(kk + 4) % 3][rj][ri]);
          }
          const int c = g.idx(i, j, kk);
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
                dv[0] += (double)(T)rv[e] * zv;
                dv[1] += zv;
              }
            }
          }
        }
      }
      __syncthreads();  // every thread is done with stage k-1 (and with Rs of plane k-2)
      if (tid == 0 && k - 1 >= pb && k - 1 + TMA_NS <= pe) issue(k - 1 + TMA_NS);
    }
    if (failed) {
      // record the failure (the update kernel stops the solve on it; `done` is
      // not set here so that every CTA still joins the reduction below), then
      // wait, bounded, for this piece's copies in flight
      if (tid == 0 && s) s->status = 6;
      // only stages k-1 .. k-2+NS can have been issued and not yet consumed
      for (int p = max(pb, kfail - 1); p <= min(pe, kfail - 2 + TMA_NS); ++p) (void)wait(p);
    }
    __syncthreads();
  }

  if constexpr (DOT) {
    const Op ops[2] = {Op::Sum, Op::Sum};
    double out[2];
    if (grid_reduce<2, TMA_NT>(dv, ops, red, 0, out)) {
      if (tid == 0 && !(s->done)) {
        const double rz_new = out[0] - s->rshift * out[1];
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
