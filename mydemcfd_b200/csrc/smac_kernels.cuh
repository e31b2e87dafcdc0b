// smac_kernels.cuh -- sm_100a kernels of the SMAC pressure projection.
//
// Operator.  For cell c with face coefficients b (x: bx[c] low, bx[c+1] high;
// y: by[c], by[c+px]; z: bz[c], bz[c+ps]) and h-scales ih2:
//   diag = sum of the six b*ih2,  off = sum of b*ih2*x_nb,  (A x)_c = diag x_c - off
// which is the reference's k_build_vof_poisson_A / k_build_vof_poisson_Ap
// (CFD/pressure_solver/G_PCGSolver.cu:126-245) without the seven stored
// stencil arrays: the diagonal is recomputed from the three face arrays.
//
// Parity-critical element-wise kernels (divergence, correction, VoF and IBM
// set-up) use __dadd_rn/__dmul_rn so that no multiply-add is contracted and
// each result rounds exactly like the reference built with -fmad=false.
#pragma once

#include "smac_common.cuh"

namespace smac {

constexpr int TBX = 32;   // threads along x
constexpr int TBY = 4;    // threads along y
constexpr int TNT = TBX * TBY;

#define DADD __dadd_rn
#define DMUL __dmul_rn
#define DDIV __ddiv_rn

// ------------------------------------------------------------------------
// Import of the reference-layout f_b into the padded fine arrays (FP64).
// Face between cells a (low) and b (high): coefficient = f_b unless an
// in-domain neighbour cell is not C_INTERIOR (the reference zeroes such rows,
// G_PCGSolver.cu:156-166) or the face lies inside the domain and is not
// F_INTERIOR (the reference's f_b is 0 there, CFD/G_SMACSolver_VoF.cu:1432-1436).
// Domain-boundary faces keep f_b: with the zero ghost it enters only the
// diagonal, as the reference's Adiag does (G_PCGSolver.cu:168-175).
// Writes the masked f_b (b*) and the stencil weights w = f_b / h^2 (w*),
// rounded as the reference's Axp = f_bx * inv_dx2 (G_PCGSolver.cu:168-173).
__global__ void k_import_coeffs(Geom g, RefDims R, const double* __restrict__ fbx, const double* __restrict__ fby,
                                const double* __restrict__ fbz, const uint8_t* __restrict__ ct,
                                const uint8_t* __restrict__ fxt, const uint8_t* __restrict__ fyt,
                                const uint8_t* __restrict__ fzt, double* bx, double* by, double* bz,
                                double* wx, double* wy, double* wz, uint8_t* fluid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const int c = g.idx(i, j, k);
  auto interior_cell = [&](int ii, int jj, int kk) -> int {  // 1 C_INTERIOR, 0 other, -1 outside
    if (ii < 0 || jj < 0 || kk < 0 || ii >= g.nx || jj >= g.ny || kk >= g.nz) return -1;
    return ct[R.cell(ii + 1, jj + 1, kk + 1)] == C_INTERIOR ? 1 : 0;
  };
  // x-face i between cells i-1 and i
  if (i <= g.nx && j < g.ny && k < g.nz) {
    const int a = interior_cell(i - 1, j, k), b = interior_cell(i, j, k);
    double v = fbx[R.xf(i + 1, j + 1, k + 1)];
    if (a == 0 || b == 0) v = 0.0;
    if (a == 1 && b == 1 && fxt[R.xf(i + 1, j + 1, k + 1)] != F_INTERIOR) v = 0.0;
    bx[c] = v;
    wx[c] = __dmul_rn(v, g.ihx2);
  }
  if (i < g.nx && j <= g.ny && k < g.nz) {
    const int a = interior_cell(i, j - 1, k), b = interior_cell(i, j, k);
    double v = fby[R.yf(i + 1, j + 1, k + 1)];
    if (a == 0 || b == 0) v = 0.0;
    if (a == 1 && b == 1 && fyt[R.yf(i + 1, j + 1, k + 1)] != F_INTERIOR) v = 0.0;
    by[c] = v;
    wy[c] = __dmul_rn(v, g.ihy2);
  }
  if (i < g.nx && j < g.ny && k <= g.nz) {
    const int a = interior_cell(i, j, k - 1), b = interior_cell(i, j, k);
    double v = fbz[R.zf(i + 1, j + 1, k + 1)];
    if (a == 0 || b == 0) v = 0.0;
    if (a == 1 && b == 1 && fzt[R.zf(i + 1, j + 1, k + 1)] != F_INTERIOR) v = 0.0;
    bz[c] = v;
    wz[c] = __dmul_rn(v, g.ihz2);
  }
  if (i < g.nx && j < g.ny && k < g.nz) fluid[c] = (interior_cell(i, j, k) == 1) ? 1 : 0;
}

// Cell bits: bit 0 C_INTERIOR, bit 1 fluid (C_INTERIOR with a non-zero
// diagonal: the cells that carry unknowns).  Counts the fluid cells.

__global__ void __launch_bounds__(TNT) k_fluid_finalize(Geom g, const double* __restrict__ bx,
                                                        const double* __restrict__ by, const double* __restrict__ bz,
                                                        uint8_t* fluid, RedBuf red, Scalars* s, int kz) {
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[1] = {0.0};
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    for (int k = k0; k < k1; ++k) {
      const int c = g.idx(i, j, k);
      const double d = bx[c] + bx[c + 1] + by[c] + by[c + g.px] + bz[c] + bz[c + g.ps];
      const uint8_t in = fluid[c] & 1;
      const uint8_t f = (in && d > 0.0) ? 1 : 0;
      fluid[c] = (uint8_t)(in | (f << 1));
      v[0] += f;
    }
  }
  const Op ops[1] = {Op::Sum};
  double out[1];
  if (grid_reduce<1, TNT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) s->sum_tmp = out[0];
  }
}

// Coarse stencil weights: mean of the fine weights of the faces that tile the
// coarse face (2x2 in 3-D), times 1/4 when the face-normal direction is
// coarsened (1/H^2 = (1/h^2)/4, G_GMGSolver.cu:71-73,135-137); computed in
// FP64 and stored as C.  Both scalings are powers of two, so they are exact.
template <class C>
__global__ void k_coarsen_coeffs(Geom gf, Geom gc, int cx, int cy, int cz, const double* __restrict__ fbx,
                                 const double* __restrict__ fby, const double* __restrict__ fbz, C* bx, C* by,
                                 C* bz, double* bx64, double* by64, double* bz64) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  const int K = blockIdx.z;
  if (I > gc.nx || J > gc.ny || K > gc.nz) return;
  const int c = gc.idx(I, J, K);
  const int ry = cy ? 2 : 1, rz = cz ? 2 : 1, rx = cx ? 2 : 1;
  if (J < gc.ny && K < gc.nz) {  // x-face I
    const int i = cx ? 2 * I : I;
    double s = 0.0;
    for (int dk = 0; dk < rz; ++dk)
      for (int dj = 0; dj < ry; ++dj) s += fbx[gf.idx(i, (cy ? 2 * J : J) + dj, (cz ? 2 * K : K) + dk)];
    s *= (cx ? 0.25 : 1.0) / (double)(ry * rz);
    bx[c] = coef_from_double<C>(s);
    if (bx64) bx64[c] = s;
  }
  if (I < gc.nx && K < gc.nz) {  // y-face J
    const int jj = cy ? 2 * J : J;
    double s = 0.0;
    for (int dk = 0; dk < rz; ++dk)
      for (int di = 0; di < rx; ++di) s += fby[gf.idx((cx ? 2 * I : I) + di, jj, (cz ? 2 * K : K) + dk)];
    s *= (cy ? 0.25 : 1.0) / (double)(rx * rz);
    by[c] = coef_from_double<C>(s);
    if (by64) by64[c] = s;
  }
  if (I < gc.nx && J < gc.ny) {  // z-face K
    const int kk = cz ? 2 * K : K;
    double s = 0.0;
    for (int dj = 0; dj < ry; ++dj)
      for (int di = 0; di < rx; ++di) s += fbz[gf.idx((cx ? 2 * I : I) + di, (cy ? 2 * J : J) + dj, kk)];
    s *= (cz ? 0.25 : 1.0) / (double)(rx * ry);
    bz[c] = coef_from_double<C>(s);
    if (bz64) bz64[c] = s;
  }
}

// Word copy of a small struct (the solver scalars to and from their mapped
// host mirror) and a 16-byte clearing loop.
static_assert(sizeof(Scalars) % 4 == 0, "scalar block in words");
__global__ void k_copy_words(const unsigned* __restrict__ src, unsigned* __restrict__ dst, int n) {
  for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
}
__global__ void k_zero16(int4* p, long long n16) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n16; t += (long long)gridDim.x * blockDim.x)
    p[t] = make_int4(0, 0, 0, 0);
}

// FP64 -> C copy of a whole padded array (fine-level FP32 / BF16 coefficients).
template <class C>
__global__ void k_convert(const double* __restrict__ a, C* b, long long n) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; t < n; t += (long long)gridDim.x * blockDim.x) b[t] = coef_from_double<C>(a[t]);
}

// BF16 -> FP32 copy of a whole padded array (exact): the cluster kernel's
// copy of the BF16 coefficients, which it stages without conversion.
__global__ void k_widen_bf16(const __nv_bfloat16* __restrict__ a, float* b, long long n) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; t < n; t += (long long)gridDim.x * blockDim.x) b[t] = __bfloat162float(a[t]);
}

// ------------------------------------------------------------------------
// Right-hand side: base_k_make_poisson_rhs (G_PressureSolverBase.cu:49-118),
// same operation order; eps == nullptr means eps == 1, fs == nullptr means
// f_s == 0.  The f_b of the surface-tension term is read from the padded
// coefficients (equal to the reference's f_b on every face of a C_INTERIOR
// cell: the masked faces carry f_b = 0 in the reference as well).
// `cellbits` bit 0 marks C_INTERIOR cells.  Writes the padded rhs and
// optionally the reference-layout rhs.
__global__ void k_divergence(Geom g, RefDims R, double inv_dx, double inv_dy, double inv_dz, double inv_dt,
                             const double* __restrict__ vx, const double* __restrict__ vy,
                             const double* __restrict__ vz, const double* __restrict__ eps,
                             const double* __restrict__ eps_old, const double* __restrict__ bx,
                             const double* __restrict__ by, const double* __restrict__ bz,
                             const double* __restrict__ fsx, const double* __restrict__ fsy,
                             const double* __restrict__ fsz, const uint8_t* __restrict__ cellbits, double* rhs,
                             double* rhs_ref) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int ix = i + 1, iy = j + 1, iz = k + 1;
  const int c = g.idx(i, j, k);
  double out = 0.0;
  if (cellbits[c] & 1) {
    double exp_ = 1.0, exm = 1.0, eyp = 1.0, eym = 1.0, ezp = 1.0, ezm = 1.0, deps = 0.0;
    if (eps) {
      const double e0 = eps[R.cell(ix, iy, iz)];
      exp_ = DMUL(0.5, DADD(e0, eps[R.cell(ix + 1, iy, iz)]));
      exm = DMUL(0.5, DADD(eps[R.cell(ix - 1, iy, iz)], e0));
      eyp = DMUL(0.5, DADD(e0, eps[R.cell(ix, iy + 1, iz)]));
      eym = DMUL(0.5, DADD(eps[R.cell(ix, iy - 1, iz)], e0));
      ezp = DMUL(0.5, DADD(e0, eps[R.cell(ix, iy, iz + 1)]));
      ezm = DMUL(0.5, DADD(eps[R.cell(ix, iy, iz - 1)], e0));
      deps = DADD(e0, -eps_old[R.cell(ix, iy, iz)]);
    }
    const double tx = DMUL(DADD(DMUL(exp_, vx[R.xf(ix + 1, iy, iz)]), -DMUL(exm, vx[R.xf(ix, iy, iz)])), inv_dx);
    const double ty = DMUL(DADD(DMUL(eyp, vy[R.yf(ix, iy + 1, iz)]), -DMUL(eym, vy[R.yf(ix, iy, iz)])), inv_dy);
    const double tz = DMUL(DADD(DMUL(ezp, vz[R.zf(ix, iy, iz + 1)]), -DMUL(ezm, vz[R.zf(ix, iy, iz)])), inv_dz);
    const double div_eps = DADD(DADD(tx, ty), tz);
    double f_st = 0.0;
    if (fsx) {
      const double sx = DMUL(DADD(DMUL(bx[c + 1], fsx[R.xf(ix + 1, iy, iz)]), -DMUL(bx[c], fsx[R.xf(ix, iy, iz)])), inv_dx);
      const double sy = DMUL(DADD(DMUL(by[c + g.px], fsy[R.yf(ix, iy + 1, iz)]), -DMUL(by[c], fsy[R.yf(ix, iy, iz)])), inv_dy);
      const double sz = DMUL(DADD(DMUL(bz[c + g.ps], fsz[R.zf(ix, iy, iz + 1)]), -DMUL(bz[c], fsz[R.zf(ix, iy, iz)])), inv_dz);
      f_st = DADD(DADD(sx, sy), sz);
    }
    out = DADD(DADD(DMUL(-inv_dt, div_eps), -DMUL(DMUL(deps, inv_dt), inv_dt)), -f_st);
  }
  rhs[c] = out;
  if (rhs_ref) rhs_ref[R.cell(ix, iy, iz)] = out;
}

// The same RHS without ε and f_s (ε = 1, f_s = 0: the same operations with
// those constants), KZ planes per thread with every plane's loads issued
// before the first result is formed; a z-face between two of the planes is
// read once.
template <int KZ>
__global__ void __launch_bounds__(TNT) k_divergence_z(Geom g, RefDims R, double inv_dx, double inv_dy, double inv_dz,
                                                      double inv_dt, const double* __restrict__ vx,
                                                      const double* __restrict__ vy, const double* __restrict__ vz,
                                                      const uint8_t* __restrict__ cellbits, double* rhs,
                                                      double* rhs_ref) {
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * KZ;
  if (i >= g.nx || j >= g.ny) return;
  const int ix = i + 1, iy = j + 1;
  double xp[KZ], xm[KZ], yp[KZ], ym[KZ], zf[KZ + 1];
  uint8_t bits[KZ];
#pragma unroll
  for (int q = 0; q < KZ; ++q) {
    const int k = k0 + q, iz = k + 1;
    bits[q] = 0;
    xp[q] = xm[q] = yp[q] = ym[q] = 0.0;
    if (k < g.nz) {
      bits[q] = cellbits[g.idx(i, j, k)];
      xp[q] = vx[R.xf(ix + 1, iy, iz)];
      xm[q] = vx[R.xf(ix, iy, iz)];
      yp[q] = vy[R.yf(ix, iy + 1, iz)];
      ym[q] = vy[R.yf(ix, iy, iz)];
    }
    zf[q] = k <= g.nz ? vz[R.zf(ix, iy, iz)] : 0.0;  // the low face of plane k, the top face of plane k-1
  }
  zf[KZ] = k0 + KZ <= g.nz ? vz[R.zf(ix, iy, k0 + KZ + 1)] : 0.0;
#pragma unroll
  for (int q = 0; q < KZ; ++q) {
    const int k = k0 + q;
    if (k >= g.nz) break;
    const double ztop = zf[q + 1];
    double out = 0.0;
    if (bits[q] & 1) {
      const double one = 1.0, deps = 0.0, f_st = 0.0;
      const double tx = DMUL(DADD(DMUL(one, xp[q]), -DMUL(one, xm[q])), inv_dx);
      const double ty = DMUL(DADD(DMUL(one, yp[q]), -DMUL(one, ym[q])), inv_dy);
      const double tz = DMUL(DADD(DMUL(one, ztop), -DMUL(one, zf[q])), inv_dz);
      const double div_eps = DADD(DADD(tx, ty), tz);
      out = DADD(DADD(DMUL(-inv_dt, div_eps), -DMUL(DMUL(deps, inv_dt), inv_dt)), -f_st);
    }
    rhs[g.idx(i, j, k)] = out;
    if (rhs_ref) rhs_ref[R.cell(ix, iy, k + 1)] = out;
  }
}

// Reference-layout cell array (interior) -> padded array.
template <class T>
__global__ void k_import_cells(Geom g, RefDims R, const double* __restrict__ src, T* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  dst[g.idx(i, j, k)] = (T)src[R.cell(i + 1, j + 1, k + 1)];
}

// Padded FP64 array -> reference-layout interior, minus `shift` on fluid cells
// (the zero-mean projection of the solution).
// KZ planes per thread, every plane's loads issued before the first store.
template <int KZ>
__global__ void __launch_bounds__(TNT) k_export_cells_z(Geom g, RefDims R, const double* __restrict__ src,
                                                        const uint8_t* __restrict__ fluid, const double* shift,
                                                        double* dst) {
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * KZ;
  if (i >= g.nx || j >= g.ny) return;
  const double sh = shift ? *shift : 0.0;
  double v[KZ];
  uint8_t f[KZ];
#pragma unroll
  for (int q = 0; q < KZ; ++q) {
    v[q] = 0.0;
    f[q] = 0;
    if (k0 + q < g.nz) {
      const int c = g.idx(i, j, k0 + q);
      v[q] = src[c];
      f[q] = fluid[c];
    }
  }
#pragma unroll
  for (int q = 0; q < KZ; ++q) {
    if (k0 + q >= g.nz) break;
    double w = v[q];
    if (shift && (f[q] & 2)) w -= sh;
    dst[R.cell(i + 1, j + 1, k0 + q + 1)] = w;
  }
}
__global__ void k_export_cells(Geom g, RefDims R, const double* __restrict__ src, const uint8_t* __restrict__ fluid,
                               const double* shift, double* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = g.idx(i, j, k);
  double v = src[c];
  if (shift && (fluid[c] & 2)) v -= *shift;
  dst[R.cell(i + 1, j + 1, k + 1)] = v;
}

// ------------------------------------------------------------------------
// Set-up of a solve: b -= mean_fluid(b) (pure Neumann), r = b (FP64 or
// FP32), x = 0, ||b||^2.  Two passes: sum, then project + norm.
template <class TR>
__global__ void __launch_bounds__(TNT) k_setup_sum(Geom g, const double* __restrict__ b, RedBuf red, Scalars* s,
                                                   int kz) {
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[1] = {0.0};
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    // four planes' loads at once, summed in plane order
    for (int kb = k0; kb < k1; kb += 4) {
      double bq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) bq[q] = kb + q < k1 ? b[g.idx(i, j, kb + q)] : 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (kb + q < k1) v[0] += bq[q];
    }
  }
  const Op ops[1] = {Op::Sum};
  double out[1];
  if (grid_reduce<1, TNT>(v, ops, red, 0, out))
    if (threadIdx.x == 0 && threadIdx.y == 0) s->sum_tmp = out[0] * s->inv_nfluid;
}

template <class TR>
__global__ void __launch_bounds__(TNT) k_setup_project(Geom g, double* b, const uint8_t* __restrict__ fluid, TR* r,
                                                       RedBuf red, Scalars* s, double tol, int kz) {
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[2] = {0.0, 0.0};
  const double m = s->sum_tmp;
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    // four planes' loads ahead of their stores, the planes taken in order
    for (int kb = k0; kb < k1; kb += 4) {
      double bq[4];
      uint8_t fq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        bq[q] = 0.0;
        fq[q] = 0;
        if (kb + q < k1) {
          const int c = g.idx(i, j, kb + q);
          bq[q] = b[c];
          fq[q] = fluid[c];
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (kb + q >= k1) break;
        const int c = g.idx(i, j, kb + q);
        double bv = bq[q];
        if (fq[q] & 2) bv -= m;
        else bv = 0.0;
        b[c] = bv;
        r[c] = (TR)bv;
        v[0] += bv * bv;
        v[1] = fmax(v[1], fabs(bv));
      }
    }
  }
  const Op ops[2] = {Op::Sum, Op::Max};
  double out[2];
  if (grid_reduce<2, TNT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      s->bb = out[0];
      s->tol2bb = tol * tol * out[0];
      s->rr = out[0];
      s->rr_anchor = out[0];
      s->rmax = out[1];
      s->rshift = 0.0;
      s->true_rr = out[0];
      s->true_rmax = out[1];
      s->iter = 0;
      s->first = 1;
      s->e_reset = s->mixed;
      s->xbuf = 0;
      s->reliable_count = 0;
      s->do_reliable = 0;
      s->status = 0;
      s->done = 0;
      if (!isfinite(out[0])) { s->status = 3; s->done = 1; }
      else if (out[0] == 0.0) { s->done = 1; }  // b == 0: x = 0 is exact
      else if (s->stop_rule == 1 && out[1] < s->tol_max) { s->done = 1; }
    }
  }
}

// ------------------------------------------------------------------------
// PCG: q = A d, pAp = d.q, alpha = rz/pAp.
template <class T, class C>
__global__ void __launch_bounds__(TNT) k_matvec_pap(Geom g, const T* __restrict__ d, Stencil<T, C> S, T* q,
                                                    RedBuf red, Scalars* s, int kz) {
  pdl_enter();
  if (s->done) return;
  typedef acc_t<T> A;
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[1] = {0.0};
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    int c = g.idx(i, j, k0);
    A xm = (A)d[c - g.ps], xc = (A)d[c];
    for (int k = k0; k < k1; ++k, c += g.ps) {
      const A xp = (A)d[c + g.ps];
      A wxm, wxp, wym, wyp, wzm, wzp;
      S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
      const A y = Stencil<T, C>::apply(xc, wxm, wxp, wym, wyp, wzm, wzp, (A)d[c - 1], (A)d[c + 1], (A)d[c - g.px],
                                       (A)d[c + g.px], xm, xp);
      q[c] = (T)y;
      v[0] += (double)xc * (double)y;
      xm = xc;
      xc = xp;
    }
  }
  const Op ops[1] = {Op::Sum};
  double out[1];
  if (grid_reduce<1, TNT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      const double pAp = out[0];
      s->pAp = pAp;
      if (!isfinite(pAp)) { s->status = 3; s->done = 1; }
      else if (!(pAp > 0.0)) { s->status = 2; s->done = 1; }
      else s->alpha = s->rz / pAp;
    }
  }
}

// PCG: x += alpha d, r -= alpha q, recursive residual statistics and the
// stopping test.  In mixed precision x is the FP32 increment since the last
// FP64 recomputation (reset to alpha d after one) and a small enough
// residual requests an FP64 recomputation instead of stopping.
// The scalar bookkeeping of the update, run by one thread of the last block:
// iteration count, the running mean of r (subtracted on the fly by the
// V-cycle), ||r||^2 of the de-meaned residual, max|r| and the stopping test.
__device__ __forceinline__ void update_finish(Scalars* s, const double (&out)[3]) {
  if (s->status == 6) { s->done = 1; return; }  // a copy-engine wait expired in a sweep
  s->iter += 1;
  s->e_reset = 0;
  const double m = out[0] * s->inv_nfluid;
  s->rshift = m;
  const double rr = fmax(out[1] - out[0] * m, 0.0);
  s->rr = rr;
  s->rmax = out[2];
  if (!isfinite(out[1])) { s->status = 3; s->done = 1; return; }
  const bool small = (s->stop_rule == 1) ? (out[2] < s->tol_max) : (rr <= s->tol2bb);
  if (s->mixed) {
    if (small || rr < s->reliable_delta2 * s->rr_anchor || s->iter >= s->max_iter) s->do_reliable = 1;
  } else if (small) {
    s->status = 0; s->done = 1;
  } else if (s->iter >= s->max_iter) {
    s->status = 1; s->done = 1;
  }
}

template <class T> struct Vec2;
template <> struct Vec2<double> { typedef double2 type; };
template <> struct Vec2<float> { typedef float2 type; };
template <class T> struct Vec16;
template <> struct Vec16<float> { typedef float4 type; static constexpr int n = 4; };
template <> struct Vec16<double> { typedef double2 type; static constexpr int n = 2; };

// PCG: x += alpha d, r -= alpha q, recursive residual statistics and the
// stopping test.  In mixed precision x is the FP32 increment since the last
// FP64 recomputation (reset to alpha d after one) and a small enough
// residual requests an FP64 recomputation instead of stopping.
// The update is element-wise, and d, q and r are 0 in every padding cell, so
// the kernel streams whole padded arrays (`n` elements from the allocation
// base) as 16-byte vectors, grid-stride, with a fixed grid for a fixed
// reduction order.
constexpr int UPD_NT = 256;
template <class T>
__global__ void __launch_bounds__(UPD_NT) k_update_flat(T* x, const T* __restrict__ d, T* r,
                                                        const T* __restrict__ q, long long n, RedBuf red,
                                                        Scalars* s) {
  pdl_enter();
  if (s->done) return;
  typedef typename Vec16<T>::type V;
  constexpr int NV = Vec16<T>::n;
  const T alpha = (T)s->alpha;
  const bool reset = s->e_reset;
  double v[3] = {0.0, 0.0, 0.0};
  const long long nvec = n / NV;
  const long long stride = (long long)gridDim.x * UPD_NT;
  V* xv = reinterpret_cast<V*>(x);
  V* rv = reinterpret_cast<V*>(r);
  const V* dv = reinterpret_cast<const V*>(d);
  const V* qv = reinterpret_cast<const V*>(q);
  for (long long t = blockIdx.x * (long long)UPD_NT + threadIdx.x; t < nvec; t += stride) {
    const V dd = dv[t], qq = qv[t];
    V rr = rv[t];
    V xx;
    if (!reset) xx = xv[t];
    T* xs = reinterpret_cast<T*>(&xx);
    T* rs = reinterpret_cast<T*>(&rr);
    const T* ds = reinterpret_cast<const T*>(&dd);
    const T* qs = reinterpret_cast<const T*>(&qq);
#pragma unroll
    for (int e = 0; e < NV; ++e) {
      xs[e] = reset ? alpha * ds[e] : xs[e] + alpha * ds[e];
      rs[e] = rs[e] - alpha * qs[e];
      v[0] += (double)rs[e];
      v[1] += (double)rs[e] * (double)rs[e];
      v[2] = fmax(v[2], fabs((double)rs[e]));
    }
    xv[t] = xx;
    rv[t] = rr;
  }
  const Op ops[3] = {Op::Sum, Op::Sum, Op::Max};
  double out[3];
  if (grid_reduce<3, UPD_NT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0) update_finish(s, out);
  }
}

// Mixed precision: FP64 true residual.  x_new = x64[xbuf] + e (FP64 sum at
// every stencil point), r = b - A64 x_new written as FP32, x_new stored in
// the other FP64 buffer; the stopping test runs on this true residual.
// Each thread takes 2 consecutive cells of one row and marches kz planes:
// FP64 rows move as 16-byte vectors, and x-neighbours across the pair come
// from the adjacent lanes (lanes 0 and 31 load them).
constexpr int REL_TX = 32, REL_TY = 4;
template <class T>
__global__ void __launch_bounds__(REL_TX * REL_TY) k_reliable_vec(Geom g, double* x64a, double* x64b,
                                                                  const T* __restrict__ e,
                                                                  const double* __restrict__ b,
                                                                  Stencil<double, double> S, T* r, RedBuf red,
                                                                  Scalars* s, int kz) {
  pdl_enter();
  if (s->done || !s->do_reliable) return;
  typedef typename Vec2<T>::type ET;
  const int lane = threadIdx.x;
  const int i0 = (blockIdx.x * REL_TX + lane) * 2;
  const int j = blockIdx.y * REL_TY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  const double* __restrict__ xs = s->xbuf ? x64b : x64a;
  double* xd = s->xbuf ? x64a : x64b;
  double v[3] = {0.0, 0.0, 0.0};
  const bool any_in = i0 < g.nx;
  if (j < g.ny && __any_sync(0xffffffffu, any_in)) {
    const int k1 = min(k0 + kz, g.nz);
    // lanes past the padded row read a valid pair of it and store nothing
    int c = g.idx(i0 < g.px ? i0 : g.px - 2, j, k0);
    auto X2 = [&](int cc, double& a, double& bb) {
      const double2 xv = *reinterpret_cast<const double2*>(xs + cc);
      const ET ev = *reinterpret_cast<const ET*>(e + cc);
      a = xv.x + (double)ev.x;
      bb = xv.y + (double)ev.y;
    };
    auto X = [&](int cc) { return xs[cc] + (double)e[cc]; };
    double xm[2], xc[2], xp[2];
    X2(c - g.ps, xm[0], xm[1]);
    X2(c, xc[0], xc[1]);
    double2 bzc = *reinterpret_cast<const double2*>(S.bz + c);
    for (int k = k0; k < k1; ++k, c += g.ps) {
      X2(c + g.ps, xp[0], xp[1]);
      double ym[2], yp[2];
      X2(c - g.px, ym[0], ym[1]);
      X2(c + g.px, yp[0], yp[1]);
      const double2 bxv = *reinterpret_cast<const double2*>(S.bx + c);
      const double2 byv = *reinterpret_cast<const double2*>(S.by + c);
      const double2 byu = *reinterpret_cast<const double2*>(S.by + c + g.px);
      const double2 bzu = *reinterpret_cast<const double2*>(S.bz + c + g.ps);
      const double2 bv = *reinterpret_cast<const double2*>(b + c);
      double left = __shfl_up_sync(0xffffffffu, xc[1], 1);
      double right = __shfl_down_sync(0xffffffffu, xc[0], 1);
      double bxr = __shfl_down_sync(0xffffffffu, bxv.x, 1);
      if (lane == 0) left = X(c - 1);
      if (lane == REL_TX - 1) {
        right = X(c + 2);
        bxr = S.bx[c + 2];
      }
      const double rv0 = bv.x - Stencil<double, double>::apply(xc[0], bxv.x, bxv.y, byv.x, byu.x, bzc.x, bzu.x, left,
                                                               xc[1], ym[0], yp[0], xm[0], xp[0]);
      const double rv1 = bv.y - Stencil<double, double>::apply(xc[1], bxv.y, bxr, byv.y, byu.y, bzc.y, bzu.y, xc[0],
                                                               right, ym[1], yp[1], xm[1], xp[1]);
      if (any_in) {
        const bool in1 = i0 + 1 < g.nx;
        double2 xo;
        xo.x = xc[0];
        xo.y = in1 ? xc[1] : 0.0;
        *reinterpret_cast<double2*>(xd + c) = xo;
        ET ro;
        ro.x = (T)rv0;
        ro.y = in1 ? (T)rv1 : (T)0;
        *reinterpret_cast<ET*>(r + c) = ro;
        v[0] += rv0;
        v[1] += rv0 * rv0;
        v[2] = fmax(v[2], fabs(rv0));
        if (in1) {
          v[0] += rv1;
          v[1] += rv1 * rv1;
          v[2] = fmax(v[2], fabs(rv1));
        }
      }
      xm[0] = xc[0];
      xm[1] = xc[1];
      xc[0] = xp[0];
      xc[1] = xp[1];
      bzc = bzu;
    }
  }
  const Op ops[3] = {Op::Sum, Op::Sum, Op::Max};
  double out[3];
  if (grid_reduce<3, REL_TX * REL_TY>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      s->xbuf ^= 1;
      s->e_reset = 1;
      s->do_reliable = 0;
      s->reliable_count += 1;
      const double m = out[0] * s->inv_nfluid;
      s->rshift = m;
      const double rr = fmax(out[1] - out[0] * m, 0.0);
      s->rr = rr;
      s->rr_anchor = rr;
      s->rmax = out[2];
      s->true_rr = rr;
      s->true_rmax = out[2];
      if (!isfinite(out[1])) { s->status = 3; s->done = 1; return; }
      const bool ok = (s->stop_rule == 1) ? (out[2] < s->tol_max) : (rr <= s->tol2bb);
      if (ok) { s->status = 0; s->done = 1; }
      else if (s->iter >= s->max_iter) { s->status = 1; s->done = 1; }
    }
  }
}

// rz_new = (r - shift).z over all cells (z is 0 where the diagonal is 0, so
// the shift needs no mask), beta = rz_new / rz.
template <class T>
__global__ void __launch_bounds__(TNT) k_dot_rz(Geom g, const T* __restrict__ r, const T* __restrict__ z, RedBuf red,
                                                Scalars* s, int kz) {
  pdl_enter();
  if (s->done) return;
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[2] = {0.0, 0.0};
  const double sh = s->rshift;
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    int c = g.idx(i, j, k0);
    for (int k = k0; k < k1; ++k, c += g.ps) {
      const double zv = (double)z[c];
      v[0] += ((double)r[c] - sh) * zv;  // z is 0 off the fluid cells
      v[1] += zv;
    }
  }
  const Op ops[2] = {Op::Sum, Op::Sum};
  double out[2];
  if (grid_reduce<2, TNT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      const double rz_new = out[0];
      if (!isfinite(rz_new)) { s->status = 3; s->done = 1; return; }
      if (!(rz_new > 0.0)) {
        // r.z <= 0 with r != 0 means the preconditioner lost definiteness
        s->status = 2; s->done = 1; return;
      }
      s->beta = s->first ? 0.0 : rz_new / s->rz;
      s->rz = rz_new;
      s->zshift = out[1] * s->inv_nfluid;
      s->first = 0;
    }
  }
}

// d = z + beta d
template <class T>
__global__ void __launch_bounds__(TNT) k_dir(Geom g, const T* __restrict__ z, T* d, const Scalars* s, int kz) {
  if (s->done) return;
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  const T beta = (T)s->beta;
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    int c = g.idx(i, j, k0);
    for (int k = k0; k < k1; ++k, c += g.ps) d[c] = z[c] + beta * d[c];
  }
}

// FP64 true residual r = b - A x with statistics (final check, plain mode).
// When `restart` is set and the test fails, r is overwritten with the true
// residual and PCG restarts from it.
__global__ void __launch_bounds__(TNT) k_true_residual(Geom g, const double* __restrict__ x, const double* __restrict__ b,
                                                       Stencil<double, double> S, double* r, int write_r, RedBuf red,
                                                       Scalars* s, int kz) {
  pdl_enter();
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[3] = {0.0, 0.0, 0.0};
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    int c = g.idx(i, j, k0);
    double xm = x[c - g.ps], xc = x[c];
    for (int k = k0; k < k1; ++k, c += g.ps) {
      const double xp = x[c + g.ps];
      double wxm, wxp, wym, wyp, wzm, wzp;
      S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
      const double rv = b[c] - Stencil<double, double>::apply(xc, wxm, wxp, wym, wyp, wzm, wzp, x[c - 1], x[c + 1],
                                                              x[c - g.px], x[c + g.px], xm, xp);
      if (write_r) r[c] = rv;
      v[0] += rv;
      v[1] += rv * rv;
      v[2] = fmax(v[2], fabs(rv));
      xm = xc;
      xc = xp;
    }
  }
  const Op ops[3] = {Op::Sum, Op::Sum, Op::Max};
  double out[3];
  if (grid_reduce<3, TNT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      const double m = out[0] * s->inv_nfluid;
      s->true_rr = fmax(out[1] - out[0] * m, 0.0);
      s->true_rmax = out[2];
      if (write_r) { s->rshift = m; s->rr = s->true_rr; s->rmax = out[2]; }
    }
  }
}

// y = A x (FP64), plain operator application for testing.
__global__ void k_apply(Geom g, const double* __restrict__ x, Stencil<double, double> S, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = g.idx(i, j, k);
  double wxm, wxp, wym, wyp, wzm, wzp;
  S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
  y[c] = Stencil<double, double>::apply(x[c], wxm, wxp, wym, wyp, wzm, wzp, x[c - 1], x[c + 1], x[c - g.px],
                                        x[c + g.px], x[c - g.ps], x[c + g.ps]);
}

// Sum of x over fluid cells (the zero-mean projection of the solution).
__global__ void __launch_bounds__(TNT) k_sum_fluid(Geom g, const double* __restrict__ x,
                                                   const uint8_t* __restrict__ fluid, RedBuf red, Scalars* s, int kz) {
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  double v[1] = {0.0};
  if (i < g.nx && j < g.ny) {
    const int k1 = min(k0 + kz, g.nz);
    // four planes' values and masks loaded at once, summed in plane order
    for (int kb = k0; kb < k1; kb += 4) {
      double xq[4];
      uint8_t fq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        xq[q] = 0.0;
        fq[q] = 0;
        if (kb + q < k1) {
          const int c = g.idx(i, j, kb + q);
          xq[q] = x[c];
          fq[q] = fluid[c];
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (kb + q < k1 && (fq[q] & 2)) v[0] += xq[q];
    }
  }
  const Op ops[1] = {Op::Sum};
  double out[1];
  if (grid_reduce<1, TNT>(v, ops, red, 0, out))
    if (threadIdx.x == 0 && threadIdx.y == 0) s->sum_tmp = out[0] * s->inv_nfluid;
}

// ------------------------------------------------------------------------
// Multigrid V-cycle pieces (red-black Gauss-Seidel).  Colour of (i,j,k) is
// (i+j+k)&1.  A thread owns the x-pair (2t, 2t+1) of a row and updates the
// member of the requested colour in every plane of its z-chunk.
//   rhs_eff = rhs - shift on cells with a non-zero diagonal (shift: the
//             running mean of the PCG residual, fine grid only)
//   zero_init: the iterate is 0 before this half-sweep (first pre-smoothing
//             sweep): neighbours are not read.
//   xc != nullptr: add the coarse-grid correction xc[parent] to every
//             neighbour read (prolongation fused into the first
//             post-smoothing half-sweep; the updated cell needs no old value).
template <class T, class C>
__global__ void __launch_bounds__(TNT) k_rbgs(Geom g, T* x, const T* __restrict__ rhs, const double* shift,
                                              Stencil<T, C> S, int colour, int zero_init, const T* __restrict__ xc,
                                              Geom gc, int cx, int cy, int cz, const Scalars* s, int kz) {
  if (s && s->done) return;
  typedef acc_t<T> A;
  const int t = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  const int i0 = 2 * t;
  if (i0 >= g.nx || j >= g.ny) return;
  const A sh = shift ? (A)(*shift) : (A)0;
  const int k1 = min(k0 + kz, g.nz);
  for (int k = k0; k < k1; ++k) {
    const int i = i0 + ((i0 + j + k + colour) & 1);
    if (i >= g.nx) continue;
    const int c = g.idx(i, j, k);
    A wxm, wxp, wym, wyp, wzm, wzp;
    S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
    const A bv = Ar<A>::add((A)rhs[c], -sh);
    A n[6] = {(A)0, (A)0, (A)0, (A)0, (A)0, (A)0};
    if (!zero_init) {
      n[0] = (A)x[c - 1]; n[1] = (A)x[c + 1]; n[2] = (A)x[c - g.px]; n[3] = (A)x[c + g.px];
      n[4] = (A)x[c - g.ps]; n[5] = (A)x[c + g.ps];
      if (xc) {
        const int ci[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const int a = ci[q][0], b = ci[q][1], d = ci[q][2];
          if (a >= 0 && b >= 0 && d >= 0 && a < g.nx && b < g.ny && d < g.nz)
            n[q] = Ar<A>::add(n[q], (A)xc[gc.idx(cx ? a >> 1 : a, cy ? b >> 1 : b, cz ? d >> 1 : d)]);
        }
      }
    }
    x[c] = (T)Stencil<T, C>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, n[0], n[1], n[2], n[3], n[4], n[5]);
  }
}

// Residual of the fine grid restricted to the coarse grid:
// rhs_c = mean over the children of (rhs_eff - A x)  (the reference's
// k_get_res_* followed by k_restrict_* averaging, G_GMGSolver.cu:152-226,416-493).
template <class T, class C>
__global__ void __launch_bounds__(TNT) k_resid_restrict(Geom g, const T* __restrict__ x, const T* __restrict__ rhs,
                                                        const double* shift, Stencil<T, C> S, Geom gc, int cx, int cy,
                                                        int cz, T* rhs_c, const Scalars* s) {
  pdl_enter();
  if (s && s->done) return;
  typedef acc_t<T> A;
  const int I = blockIdx.x * TBX + threadIdx.x;
  const int J = blockIdx.y * TBY + threadIdx.y;
  const int K = blockIdx.z;
  if (I >= gc.nx || J >= gc.ny || K >= gc.nz) return;
  const A sh = shift ? (A)(*shift) : (A)0;
  A acc = (A)0;
  const int rx = cx ? 2 : 1, ry = cy ? 2 : 1, rz = cz ? 2 : 1;
  for (int dk = 0; dk < rz; ++dk)
    for (int dj = 0; dj < ry; ++dj)
      for (int di = 0; di < rx; ++di) {
        const int i = (cx ? 2 * I : I) + di, j = (cy ? 2 * J : J) + dj, k = (cz ? 2 * K : K) + dk;
        const int c = g.idx(i, j, k);
        A wxm, wxp, wym, wyp, wzm, wzp;
        S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
        const A diag = Stencil<T, C>::diag(wxm, wxp, wym, wyp, wzm, wzp);
        A bv = (A)rhs[c];
        if (diag > (A)0) bv = Ar<A>::add(bv, -sh);
        const A ax = Stencil<T, C>::apply((A)x[c], wxm, wxp, wym, wyp, wzm, wzp, (A)x[c - 1], (A)x[c + 1],
                                          (A)x[c - g.px], (A)x[c + g.px], (A)x[c - g.ps], (A)x[c + g.ps]);
        acc = Ar<A>::add(acc, Ar<A>::add(bv, -ax));
      }
  rhs_c[gc.idx(I, J, K)] = (T)Ar<A>::div(acc, (A)(rx * ry * rz));
}

// The same for a coarse grid halved in every direction: each thread reads its
// 2x2x2 block's rows, the rows and planes around it and the faces once, as
// 2-vectors of cells (i = 2I, 2I+1), and sums the eight residuals in the
// order of k_resid_restrict.
template <class T>
__global__ void __launch_bounds__(TNT) k_resid_restrict2(Geom g, const T* __restrict__ x, const T* __restrict__ rhs,
                                                         const double* shift, Stencil<T, T> S, Geom gc, T* rhs_c,
                                                         const Scalars* s) {
  pdl_enter();
  if (s && s->done) return;
  typedef acc_t<T> A;
  typedef typename Vec2<T>::type V2;
  const int I = blockIdx.x * TBX + threadIdx.x;
  const int J = blockIdx.y * TBY + threadIdx.y;
  const int K = blockIdx.z;
  if (I >= gc.nx || J >= gc.ny || K >= gc.nz) return;
  const A sh = shift ? (A)(*shift) : (A)0;
  const int i = 2 * I, j = 2 * J, k = 2 * K;
  auto ld2 = [&](const T* p, int c, A& a, A& b) {
    const V2 v = *reinterpret_cast<const V2*>(p + c);
    a = (A)v.x;
    b = (A)v.y;
  };
  // x: rows j-1 .. j+2 on planes k, k+1; planes k-1, k+2 on rows j, j+1
  A xr[2][4][2], xz[2][2][2], xl[2][2], xh[2][2];
#pragma unroll
  for (int dk = 0; dk < 2; ++dk) {
#pragma unroll
    for (int r = 0; r < 4; ++r) ld2(x, g.idx(i, j - 1 + r, k + dk), xr[dk][r][0], xr[dk][r][1]);
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int c = g.idx(i, j + dj, k + dk);
      xl[dk][dj] = (A)x[c - 1];
      xh[dk][dj] = (A)x[c + 2];
    }
  }
#pragma unroll
  for (int dj = 0; dj < 2; ++dj) {
    ld2(x, g.idx(i, j + dj, k - 1), xz[0][dj][0], xz[0][dj][1]);
    ld2(x, g.idx(i, j + dj, k + 2), xz[1][dj][0], xz[1][dj][1]);
  }
  A acc = (A)0;
#pragma unroll
  for (int dk = 0; dk < 2; ++dk) {
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const int c = g.idx(i, j + dj, k + dk);
      A b0, b1, bx0, bx1, by0, by1, bu0, bu1, bz0, bz1, bw0, bw1;
      ld2(rhs, c, b0, b1);
      ld2(S.bx, c, bx0, bx1);
      const A bx2 = (A)S.bx[c + 2];
      ld2(S.by, c, by0, by1);
      ld2(S.by, c + g.px, bu0, bu1);
      ld2(S.bz, c, bz0, bz1);
      ld2(S.bz, c + g.ps, bw0, bw1);
      // z-neighbours of this row: plane below and above
      const A* zm = dk == 0 ? xz[0][dj] : xr[0][1 + dj];
      const A* zp = dk == 0 ? xr[1][1 + dj] : xz[1][dj];
      const A* row = xr[dk][1 + dj];
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        const A wxm = di ? bx1 : bx0, wxp = di ? bx2 : bx1;
        const A wym = di ? by1 : by0, wyp = di ? bu1 : bu0;
        const A wzm = di ? bz1 : bz0, wzp = di ? bw1 : bw0;
        const A diag = Stencil<T, T>::diag(wxm, wxp, wym, wyp, wzm, wzp);
        A bv = di ? b1 : b0;
        if (diag > (A)0) bv = Ar<A>::add(bv, -sh);
        const A xw = di ? row[0] : xl[dk][dj];
        const A xe = di ? xh[dk][dj] : row[1];
        const A ax = Stencil<T, T>::apply(row[di], wxm, wxp, wym, wyp, wzm, wzp, xw, xe, xr[dk][dj][di],
                                          xr[dk][2 + dj][di], zm[di], zp[di]);
        acc = Ar<A>::add(acc, Ar<A>::add(bv, -ax));
      }
    }
  }
  rhs_c[gc.idx(I, J, K)] = (T)Ar<A>::div(acc, (A)8);
}

// ------------------------------------------------------------------------
// Coarse grids in one persistent single-CTA kernel: pre-smoothing,
// residual/restriction, the coarsest solve (symmetric sweep pairs),
// prolongation and post-smoothing of every grid at or below the first
// grid with <= 4096 cells, with __syncthreads between the steps.
struct CoarseLevel {
  Geom g;
  int cx, cy, cz;          // how this grid was coarsened from the one above
  const void* bx;
  const void* by;
  const void* bz;
  void* x;
  void* rhs;
};
constexpr int MAX_COARSE = 8;
struct CoarseSet {
  CoarseLevel L[MAX_COARSE];
  int n;  // grids in the set; L[0] receives rhs and returns x
};

template <class T, class C>
__device__ __forceinline__ void cta_half_sweep(const CoarseLevel& L, int colour, bool zero_init, const T* xc,
                                               const CoarseLevel* Lc, const double* shift) {
  typedef acc_t<T> A;
  const Geom& g = L.g;
  T* x = (T*)L.x;
  const T* rhs = (const T*)L.rhs;
  Stencil<T, C> S{(const C*)L.bx, (const C*)L.by, (const C*)L.bz};
  const A sh = shift ? (A)(*shift) : (A)0;
  const int half = (g.nx + 1) / 2;
  const int total = half * g.ny * g.nz;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int tx = t % half;
    const int j = (t / half) % g.ny;
    const int k = t / (half * g.ny);
    const int i0 = 2 * tx;
    const int i = i0 + ((i0 + j + k + colour) & 1);
    if (i >= g.nx) continue;
    const int c = g.idx(i, j, k);
    A wxm, wxp, wym, wyp, wzm, wzp;
    S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
    const A bv = Ar<A>::add((A)rhs[c], -sh);
    A n[6] = {(A)0, (A)0, (A)0, (A)0, (A)0, (A)0};
    if (!zero_init) {
      n[0] = (A)x[c - 1]; n[1] = (A)x[c + 1]; n[2] = (A)x[c - g.px]; n[3] = (A)x[c + g.px];
      n[4] = (A)x[c - g.ps]; n[5] = (A)x[c + g.ps];
      if (xc) {
        const Geom& gc = Lc->g;
        const int ci[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const int a = ci[q][0], b = ci[q][1], d = ci[q][2];
          if (a >= 0 && b >= 0 && d >= 0 && a < g.nx && b < g.ny && d < g.nz)
            n[q] = Ar<A>::add(n[q], (A)xc[gc.idx(Lc->cx ? a >> 1 : a, Lc->cy ? b >> 1 : b, Lc->cz ? d >> 1 : d)]);
        }
      }
    }
    x[c] = (T)Stencil<T, C>::gs(bv, wxm, wxp, wym, wyp, wzm, wzp, n[0], n[1], n[2], n[3], n[4], n[5]);
  }
}

template <class T, class C>
__device__ __forceinline__ void cta_resid_restrict(const CoarseLevel& L, const CoarseLevel& Lc, const double* shift) {
  typedef acc_t<T> A;
  const Geom& g = L.g;
  const Geom& gc = Lc.g;
  const T* x = (const T*)L.x;
  const T* rhs = (const T*)L.rhs;
  T* rhs_c = (T*)Lc.rhs;
  Stencil<T, C> S{(const C*)L.bx, (const C*)L.by, (const C*)L.bz};
  const A sh = shift ? (A)(*shift) : (A)0;
  const int total = gc.nx * gc.ny * gc.nz;
  const int rx = Lc.cx ? 2 : 1, ry = Lc.cy ? 2 : 1, rz = Lc.cz ? 2 : 1;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int I = t % gc.nx, J = (t / gc.nx) % gc.ny, K = t / (gc.nx * gc.ny);
    A acc = (A)0;
    for (int dk = 0; dk < rz; ++dk)
      for (int dj = 0; dj < ry; ++dj)
        for (int di = 0; di < rx; ++di) {
          const int i = (Lc.cx ? 2 * I : I) + di, j = (Lc.cy ? 2 * J : J) + dj, k = (Lc.cz ? 2 * K : K) + dk;
          const int c = g.idx(i, j, k);
          A wxm, wxp, wym, wyp, wzm, wzp;
          S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
          const A diag = Stencil<T, C>::diag(wxm, wxp, wym, wyp, wzm, wzp);
          A bv = (A)rhs[c];
          if (diag > (A)0) bv = Ar<A>::add(bv, -sh);
          const A ax = Stencil<T, C>::apply((A)x[c], wxm, wxp, wym, wyp, wzm, wzp, (A)x[c - 1], (A)x[c + 1],
                                            (A)x[c - g.px], (A)x[c + g.px], (A)x[c - g.ps], (A)x[c + g.ps]);
          acc = Ar<A>::add(acc, Ar<A>::add(bv, -ax));
        }
    rhs_c[gc.idx(I, J, K)] = (T)Ar<A>::div(acc, (A)(rx * ry * rz));
  }
}

template <class T, class C>
__global__ void __launch_bounds__(1024) k_coarse_vcycle(CoarseSet set, int nu1, int nu2, int coarse_pairs,
                                                        const double* shift0, const Scalars* s) {
  pdl_enter();
  if (s && s->done) return;
  const int n = set.n;
  // down
  for (int l = 0; l < n - 1; ++l) {
    const double* sh = (l == 0) ? shift0 : nullptr;
    for (int it = 0; it < nu1; ++it) {
      cta_half_sweep<T, C>(set.L[l], 0, it == 0, nullptr, nullptr, sh);
      __syncthreads();
      cta_half_sweep<T, C>(set.L[l], 1, false, nullptr, nullptr, sh);
      __syncthreads();
    }
    cta_resid_restrict<T, C>(set.L[l], set.L[l + 1], sh);
    __syncthreads();
  }
  // coarsest: symmetric sweep pairs from zero
  {
    const CoarseLevel& L = set.L[n - 1];
    const double* sh = (n == 1) ? shift0 : nullptr;
    for (int it = 0; it < coarse_pairs; ++it) {
      cta_half_sweep<T, C>(L, 0, it == 0, nullptr, nullptr, sh);
      __syncthreads();
      cta_half_sweep<T, C>(L, 1, false, nullptr, nullptr, sh);
      __syncthreads();
    }
    for (int it = 0; it < coarse_pairs; ++it) {
      cta_half_sweep<T, C>(L, 1, false, nullptr, nullptr, sh);
      __syncthreads();
      cta_half_sweep<T, C>(L, 0, false, nullptr, nullptr, sh);
      __syncthreads();
    }
  }
  // up
  for (int l = n - 2; l >= 0; --l) {
    const double* sh = (l == 0) ? shift0 : nullptr;
    for (int it = 0; it < nu2; ++it) {
      const bool fuse = (it == 0);
      cta_half_sweep<T, C>(set.L[l], 1, false, fuse ? (const T*)set.L[l + 1].x : nullptr, &set.L[l + 1], sh);
      __syncthreads();
      cta_half_sweep<T, C>(set.L[l], 0, false, nullptr, nullptr, sh);
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------------
// Velocity correction: k_correct_vof_velocity (CFD/G_SMACSolver.cu:1072-1142),
// same thread ranges and operation order.  fs == nullptr: f_s = 0;
// fir == nullptr: f_inv_rho taken from the padded f_b.  write_all: faces that
// are not F_INTERIOR receive u* (used by smac_project).
__global__ void k_correct(RefDims R, Geom g, double inv_dx, double inv_dy, double inv_dz, double dt,
                          const uint8_t* __restrict__ ct, const uint8_t* __restrict__ fxt,
                          const uint8_t* __restrict__ fyt, const uint8_t* __restrict__ fzt,
                          const double* __restrict__ pd, double* p, const double* __restrict__ vxs,
                          const double* __restrict__ vys, const double* __restrict__ vzs,
                          const double* __restrict__ firx, const double* __restrict__ firy,
                          const double* __restrict__ firz, const double* __restrict__ fbx,
                          const double* __restrict__ fby, const double* __restrict__ fbz,
                          const double* __restrict__ fsx, const double* __restrict__ fsy,
                          const double* __restrict__ fsz, double* vx, double* vy, double* vz, int write_all) {
  // every face index from 0 (the reference's threads start at 1; index-0
  // faces are ghost faces that only write_all touches)
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  const int Nx = R.Nx, Ny = R.Ny, Nz = R.Nz;
  // padded f_b of the face, used when f_inv_rho is not supplied
  auto padded = [&](const double* b, int i, int j, int k) -> double {
    if (i < 0 || j < 0 || k < 0 || i > g.nx || j > g.ny || k > g.nz) return 0.0;
    return b[g.idx(i, j, k)];
  };
  // a face is corrected only when both of its cells exist (F_INTERIOR faces
  // always satisfy this; the bound keeps mislabelled ghost faces harmless)
  if (!(iy >= Ny + 2 || ix >= Nx + 3 || iz >= Nz + 2)) {
    const long long f = R.xf(ix, iy, iz);
    if (fxt[f] == F_INTERIOR && ix >= 1 && ix <= Nx + 1) {
      const double ir = firx ? firx[f] : padded(fbx, ix - 1, iy - 1, iz - 1);
      const double fs = fsx ? fsx[f] : 0.0;
      const double gp = DMUL(DADD(pd[R.cell(ix, iy, iz)], -pd[R.cell(ix - 1, iy, iz)]), inv_dx);
      vx[f] = DADD(vxs[f], DMUL(DMUL(ir, dt), DADD(fs, -gp)));
    } else if (write_all) {
      vx[f] = vxs[f];
    }
  }
  if (!(iy >= Ny + 3 || ix >= Nx + 2 || iz >= Nz + 2)) {
    const long long f = R.yf(ix, iy, iz);
    if (fyt[f] == F_INTERIOR && iy >= 1 && iy <= Ny + 1) {
      const double ir = firy ? firy[f] : padded(fby, ix - 1, iy - 1, iz - 1);
      const double fs = fsy ? fsy[f] : 0.0;
      const double gp = DMUL(DADD(pd[R.cell(ix, iy, iz)], -pd[R.cell(ix, iy - 1, iz)]), inv_dy);
      vy[f] = DADD(vys[f], DMUL(DMUL(ir, dt), DADD(fs, -gp)));
    } else if (write_all) {
      vy[f] = vys[f];
    }
  }
  if (!(iy >= Ny + 2 || ix >= Nx + 2 || iz >= Nz + 3)) {
    const long long f = R.zf(ix, iy, iz);
    if (fzt[f] == F_INTERIOR && iz >= 1 && iz <= Nz + 1) {
      const double ir = firz ? firz[f] : padded(fbz, ix - 1, iy - 1, iz - 1);
      const double fs = fsz ? fsz[f] : 0.0;
      const double gp = DMUL(DADD(pd[R.cell(ix, iy, iz)], -pd[R.cell(ix, iy, iz - 1)]), inv_dz);
      vz[f] = DADD(vzs[f], DMUL(DMUL(ir, dt), DADD(fs, -gp)));
    } else if (write_all) {
      vz[f] = vzs[f];
    }
  }
  if (p && ix >= 1 && iy >= 1 && iz >= 1 && ix < Nx + 1 && iy < Ny + 1 && iz < Nz + 1) {
    if (ct[R.cell(ix, iy, iz)] == C_INTERIOR) p[R.cell(ix, iy, iz)] = DADD(p[R.cell(ix, iy, iz)], pd[R.cell(ix, iy, iz)]);
  }
}

// The correction as smac_project runs it (f_s = 0, f_inv_rho from the padded
// f_b, p untouched, faces that are not F_INTERIOR receive u*): the
// operations of k_correct, with every value a face may need loaded together
// with its type (the indices are valid for every face in the reference's
// range), so an F_INTERIOR face costs one round trip instead of two.
__global__ void k_correct_project(RefDims R, Geom g, double inv_dx, double inv_dy, double inv_dz, double dt,
                                  const uint8_t* __restrict__ fxt, const uint8_t* __restrict__ fyt,
                                  const uint8_t* __restrict__ fzt, const double* __restrict__ pd,
                                  const double* __restrict__ vxs, const double* __restrict__ vys,
                                  const double* __restrict__ vzs, const double* __restrict__ fbx,
                                  const double* __restrict__ fby, const double* __restrict__ fbz, double* vx,
                                  double* vy, double* vz) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  const int Nx = R.Nx, Ny = R.Ny, Nz = R.Nz;
  auto padded = [&](const double* b, int i, int j, int k) -> double {
    if (i < 0 || j < 0 || k < 0 || i > g.nx || j > g.ny || k > g.nz) return 0.0;
    return b[g.idx(i, j, k)];
  };
  const bool cin = ix < Nx + 2 && iy < Ny + 2 && iz < Nz + 2;
  const double p0 = cin ? pd[R.cell(ix, iy, iz)] : 0.0;
  // x-faces
  const bool xin = iy < Ny + 2 && ix < Nx + 3 && iz < Nz + 2, xr = ix >= 1 && ix <= Nx + 1;
  uint8_t tx = 0;
  double ux = 0.0, pxm = 0.0, irx = 0.0;
  long long fx = 0;
  if (xin) {
    fx = R.xf(ix, iy, iz);
    tx = fxt[fx];
    ux = vxs[fx];
    if (xr) {
      pxm = pd[R.cell(ix - 1, iy, iz)];
      irx = padded(fbx, ix - 1, iy - 1, iz - 1);
    }
  }
  // y-faces
  const bool yin = iy < Ny + 3 && ix < Nx + 2 && iz < Nz + 2, yr = iy >= 1 && iy <= Ny + 1;
  uint8_t ty = 0;
  double uy = 0.0, pym = 0.0, iry = 0.0;
  long long fy = 0;
  if (yin) {
    fy = R.yf(ix, iy, iz);
    ty = fyt[fy];
    uy = vys[fy];
    if (yr) {
      pym = pd[R.cell(ix, iy - 1, iz)];
      iry = padded(fby, ix - 1, iy - 1, iz - 1);
    }
  }
  // z-faces
  const bool zin = iy < Ny + 2 && ix < Nx + 2 && iz < Nz + 3, zr = iz >= 1 && iz <= Nz + 1;
  uint8_t tz = 0;
  double uz = 0.0, pzm = 0.0, irz = 0.0;
  long long fz = 0;
  if (zin) {
    fz = R.zf(ix, iy, iz);
    tz = fzt[fz];
    uz = vzs[fz];
    if (zr) {
      pzm = pd[R.cell(ix, iy, iz - 1)];
      irz = padded(fbz, ix - 1, iy - 1, iz - 1);
    }
  }
  // (a face with xr, yr or zr has both of its cells, so p0 was loaded)
  const double fs = 0.0;
  if (xin) {
    if (tx == F_INTERIOR && xr) {
      const double gp = DMUL(DADD(p0, -pxm), inv_dx);
      vx[fx] = DADD(ux, DMUL(DMUL(irx, dt), DADD(fs, -gp)));
    } else {
      vx[fx] = ux;
    }
  }
  if (yin) {
    if (ty == F_INTERIOR && yr) {
      const double gp = DMUL(DADD(p0, -pym), inv_dy);
      vy[fy] = DADD(uy, DMUL(DMUL(iry, dt), DADD(fs, -gp)));
    } else {
      vy[fy] = uy;
    }
  }
  if (zin) {
    if (tz == F_INTERIOR && zr) {
      const double gp = DMUL(DADD(p0, -pzm), inv_dz);
      vz[fz] = DADD(uz, DMUL(DMUL(irz, dt), DADD(fs, -gp)));
    } else {
      vz[fz] = uz;
    }
  }
}

// ------------------------------------------------------------------------
// Adjoint pieces.  The projection on F_INTERIOR faces is
//   u = u* + B G A^+ D u*     (B = diag f_b, G = face gradient, D = divergence)
// with the zero-mean projection Pi of the pure-Neumann solve, so
//   dL/du* = g + D^T Pi A^+ G^T B g = g + G psi,  psi = Pi A^+ D_int(B g)
// using D^T = -G and G^T = -D_int (D_int: divergence over F_INTERIOR faces).
// rhs_adj = D_int(B g) on fluid cells, written to the padded rhs.
__global__ void k_adj_divergence(Geom g, RefDims R, double inv_dx, double inv_dy, double inv_dz,
                                 const double* __restrict__ gx, const double* __restrict__ gy,
                                 const double* __restrict__ gz, const double* __restrict__ bx,
                                 const double* __restrict__ by, const double* __restrict__ bz,
                                 const uint8_t* __restrict__ fluid, double* rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = g.idx(i, j, k);
  double out = 0.0;
  if (fluid[c] & 2) {
    // only faces between two cells carry the projection; wall faces have
    // f_b = 0 for pure Neumann walls and are excluded explicitly otherwise
    const double wxm = (i > 0) ? bx[c] : 0.0, wxp = (i < g.nx - 1) ? bx[c + 1] : 0.0;
    const double wym = (j > 0) ? by[c] : 0.0, wyp = (j < g.ny - 1) ? by[c + g.px] : 0.0;
    const double wzm = (k > 0) ? bz[c] : 0.0, wzp = (k < g.nz - 1) ? bz[c + g.ps] : 0.0;
    const int ix = i + 1, iy = j + 1, iz = k + 1;
    out = (wxp * gx[R.xf(ix + 1, iy, iz)] - wxm * gx[R.xf(ix, iy, iz)]) * inv_dx +
          (wyp * gy[R.yf(ix, iy + 1, iz)] - wym * gy[R.yf(ix, iy, iz)]) * inv_dy +
          (wzp * gz[R.zf(ix, iy, iz + 1)] - wzm * gz[R.zf(ix, iy, iz)]) * inv_dz;
  }
  rhs[c] = out;
}

// dL/du* = g + G psi on every face, psi = A^+ D_int(B g) on fluid cells and 0
// elsewhere (also beyond the walls).  The forward map reads u* on every face
// of a fluid cell through the divergence, wall faces included, so the
// gradient term reaches those faces too.  psi = x - shift on fluid cells
// (shift: the fluid mean of the solve's solution).
__global__ void k_adj_gradient(Geom g, RefDims R, double inv_dx, double inv_dy, double inv_dz,
                               const double* __restrict__ x, const uint8_t* __restrict__ fluid, const double* shift,
                               const double* __restrict__ gx, const double* __restrict__ gy,
                               const double* __restrict__ gz, double* ox, double* oy, double* oz) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  const int Nx = R.Nx, Ny = R.Ny, Nz = R.Nz;
  const double sh = *shift;
  // psi at reference cell (cx, cy, cz)
  auto P = [&](int cx, int cy, int cz) -> double {
    const int i = cx - 1, j = cy - 1, k = cz - 1;
    if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return 0.0;
    const int c = g.idx(i, j, k);
    return (fluid[c] & 2) ? x[c] - sh : 0.0;
  };
  if (ix < Nx + 3 && iy < Ny + 2 && iz < Nz + 2) {
    const long long f = R.xf(ix, iy, iz);
    double v = gx[f];
    if (ix >= 1 && ix <= Nx + 1) v += (P(ix, iy, iz) - P(ix - 1, iy, iz)) * inv_dx;
    ox[f] = v;
  }
  if (ix < Nx + 2 && iy < Ny + 3 && iz < Nz + 2) {
    const long long f = R.yf(ix, iy, iz);
    double v = gy[f];
    if (iy >= 1 && iy <= Ny + 1) v += (P(ix, iy, iz) - P(ix, iy - 1, iz)) * inv_dy;
    oy[f] = v;
  }
  if (ix < Nx + 2 && iy < Ny + 2 && iz < Nz + 3) {
    const long long f = R.zf(ix, iy, iz);
    double v = gz[f];
    if (iz >= 1 && iz <= Nz + 1) v += (P(ix, iy, iz) - P(ix, iy, iz - 1)) * inv_dz;
    oz[f] = v;
  }
}

// Jacobi preconditioner z = (r - shift)/diag on cells with a non-zero
// diagonal (the reference's z = invAdiag r, G_PCGSolver.cu:248-273).
template <class T, class C>
__global__ void __launch_bounds__(TNT) k_jacobi_precond(Geom g, const T* __restrict__ r, const double* shift,
                                                        Stencil<T, C> S, T* z, const Scalars* s, int kz) {
  pdl_enter();
  if (s->done) return;
  typedef acc_t<T> A;
  const int i = blockIdx.x * TBX + threadIdx.x;
  const int j = blockIdx.y * TBY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  if (i >= g.nx || j >= g.ny) return;
  const A sh = shift ? (A)(*shift) : (A)0;
  const int k1 = min(k0 + kz, g.nz);
  int c = g.idx(i, j, k0);
  for (int k = k0; k < k1; ++k, c += g.ps) {
    A wxm, wxp, wym, wyp, wzm, wzp;
    S.coeffs(c, g.px, g.ps, wxm, wxp, wym, wyp, wzm, wzp);
    const A diag = Stencil<T, C>::diag(wxm, wxp, wym, wyp, wzm, wzp);
    z[c] = (T)((diag > (A)0) ? Ar<A>::div(Ar<A>::add((A)r[c], -sh), diag) : (A)0);
  }
}

// ------------------------------------------------------------------------
// Set-up kernels in the reference layout.
// SMACSolver::set_face_type / set_cell_type (CFD/SMACSolver.cpp:104-248).
__global__ void k_box_types(RefDims R, uint8_t* ct, uint8_t* fxt, uint8_t* fyt, uint8_t* fzt) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  const int Nx = R.Nx, Ny = R.Ny, Nz = R.Nz;
  if (ix < Nx + 3 && iy < Ny + 2 && iz < Nz + 2) {
    uint8_t t = F_GHOST;
    if (iz >= 1 && iz <= Nz && iy >= 1 && iy <= Ny && ix >= 1 && ix <= Nx + 1)
      t = (ix == 1 || ix == Nx + 1) ? F_BOUNDARY : F_INTERIOR;
    fxt[R.xf(ix, iy, iz)] = t;
  }
  if (ix < Nx + 2 && iy < Ny + 3 && iz < Nz + 2) {
    uint8_t t = F_GHOST;
    if (iz >= 1 && iz <= Nz && iy >= 1 && iy <= Ny + 1 && ix >= 1 && ix <= Nx)
      t = (iy == 1 || iy == Ny + 1) ? F_BOUNDARY : F_INTERIOR;
    fyt[R.yf(ix, iy, iz)] = t;
  }
  if (ix < Nx + 2 && iy < Ny + 2 && iz < Nz + 3) {
    uint8_t t = F_GHOST;
    if (iz >= 1 && iz <= Nz + 1 && iy >= 1 && iy <= Ny && ix >= 1 && ix <= Nx)
      t = (iz == 1 || iz == Nz + 1) ? F_BOUNDARY : F_INTERIOR;
    fzt[R.zf(ix, iy, iz)] = t;
  }
  if (ix < Nx + 2 && iy < Ny + 2 && iz < Nz + 2) {
    const bool in = ix >= 1 && ix <= Nx && iy >= 1 && iy <= Ny && iz >= 1 && iz <= Nz;
    ct[R.cell(ix, iy, iz)] = in ? C_INTERIOR : C_GHOST;
  }
}

// k_update_cell_properties_by_alpha (CFD/G_SMACSolver_VoF.cu:1374-1407)
__global__ void k_vof_rho(RefDims R, const double* __restrict__ alpha, double rho0, double rho1,
                          const uint8_t* __restrict__ ct, double* rho) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int iz = blockIdx.z + 1;
  if (ix >= R.Nx + 2 || iy >= R.Ny + 2 || iz >= R.Nz + 2) return;
  const long long c = R.cell(ix, iy, iz);
  const uint8_t t = ct[c];
  if (t == C_INTERIOR || t == C_NEAR_BOUNDARY) {
    const double a = alpha[c];
    rho[c] = DADD(DMUL(DADD(1., -a), rho0), DMUL(a, rho1));
  }
}

// k_update_{x,y,z}_face_properties_by_alpha (CFD/G_SMACSolver_VoF.cu:1409-1535)
__global__ void k_vof_faces(RefDims R, const double* __restrict__ rho, const uint8_t* __restrict__ fxt,
                            const uint8_t* __restrict__ fyt, const uint8_t* __restrict__ fzt, double* fbx, double* fby,
                            double* fbz, double* firx, double* firy, double* firz) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int iz = blockIdx.z + 1;
  const int Nx = R.Nx, Ny = R.Ny, Nz = R.Nz;
  if (!(ix >= Nx + 3 || iy >= Ny + 2 || iz >= Nz + 2)) {
    const long long f = R.xf(ix, iy, iz);
    double b = 0.0;
    if (fxt[f] == F_INTERIOR && ix <= Nx + 1) b = DDIV(1., DMUL(0.5, DADD(rho[R.cell(ix, iy, iz)], rho[R.cell(ix - 1, iy, iz)])));
    fbx[f] = b;
    if (firx) firx[f] = b;
  }
  if (!(ix >= Nx + 2 || iy >= Ny + 3 || iz >= Nz + 2)) {
    const long long f = R.yf(ix, iy, iz);
    double b = 0.0;
    if (fyt[f] == F_INTERIOR && iy <= Ny + 1) b = DDIV(1., DMUL(0.5, DADD(rho[R.cell(ix, iy, iz)], rho[R.cell(ix, iy - 1, iz)])));
    fby[f] = b;
    if (firy) firy[f] = b;
  }
  if (!(ix >= Nx + 2 || iy >= Ny + 2 || iz >= Nz + 3)) {
    const long long f = R.zf(ix, iy, iz);
    double b = 0.0;
    if (fzt[f] == F_INTERIOR && iz <= Nz + 1) b = DDIV(1., DMUL(0.5, DADD(rho[R.cell(ix, iy, iz)], rho[R.cell(ix, iy, iz - 1)])));
    fbz[f] = b;
    if (firz) firz[f] = b;
  }
}

// Outlet boundary faces (G_SMACSolver::update_boundary_faces,
// CFD/G_SMACSolver_VoF.cu:1798-1950): f_b = 2 f_b of the neighbouring face on
// the interior side (p = 0 on the outlet); mark 1: side +1, 2: side -1, 0:
// untouched.  Marked faces have unmarked neighbours, so no face is read after
// it is written.
__global__ void k_outlet_faces(RefDims R, const uint8_t* __restrict__ fxo, const uint8_t* __restrict__ fyo,
                               const uint8_t* __restrict__ fzo, double* fbx, double* fby, double* fbz) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int iz = blockIdx.z;
  const int Nx = R.Nx, Ny = R.Ny, Nz = R.Nz;
  if (ix < Nx + 3 && iy < Ny + 2 && iz < Nz + 2) {
    const long long f = R.xf(ix, iy, iz);
    const uint8_t m = fxo[f];
    if (m == 1 && ix + 1 < Nx + 3) fbx[f] = DMUL(2.0, fbx[R.xf(ix + 1, iy, iz)]);
    if (m == 2 && ix >= 1) fbx[f] = DMUL(2.0, fbx[R.xf(ix - 1, iy, iz)]);
  }
  if (ix < Nx + 2 && iy < Ny + 3 && iz < Nz + 2) {
    const long long f = R.yf(ix, iy, iz);
    const uint8_t m = fyo[f];
    if (m == 1 && iy + 1 < Ny + 3) fby[f] = DMUL(2.0, fby[R.yf(ix, iy + 1, iz)]);
    if (m == 2 && iy >= 1) fby[f] = DMUL(2.0, fby[R.yf(ix, iy - 1, iz)]);
  }
  if (ix < Nx + 2 && iy < Ny + 2 && iz < Nz + 3) {
    const long long f = R.zf(ix, iy, iz);
    const uint8_t m = fzo[f];
    if (m == 1 && iz + 1 < Nz + 3) fbz[f] = DMUL(2.0, fbz[R.zf(ix, iy, iz + 1)]);
    if (m == 2 && iz >= 1) fbz[f] = DMUL(2.0, fbz[R.zf(ix, iy, iz - 1)]);
  }
}

// Solid fraction by 8^3 sub-sampling (k_get_solid_fraction,
// CFD/G_SMACSolver_IBM.cu:94-147) for a union of non-overlapping spheres.
// Cells entirely inside or outside a sphere by a margin far above the
// rounding of the sample coordinates skip the sampling; the count is the same.
__global__ void k_ibm_spheres(RefDims R, double dx, double dy, double dz, double ox, double oy, double oz,
                              const double* __restrict__ sph, int nsph, double* sf) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int iz = blockIdx.z + 1;
  if (ix >= R.Nx + 2 || iy >= R.Ny + 2 || iz >= R.Nz + 2) return;
  const double xc = DADD(DADD(DMUL(dx, (double)ix), -DMUL(0.5, dx)), ox);
  const double yc = DADD(DADD(DMUL(dy, (double)iy), -DMUL(0.5, dy)), oy);
  const double zc = DADD(DADD(DMUL(dz, (double)iz), -DMUL(0.5, dz)), oz);
  const double xini = DADD(xc, -DMUL(dx, 0.5)), yini = DADD(yc, -DMUL(dy, 0.5)), zini = DADD(zc, -DMUL(dz, 0.5));
  const double fact = 1. / 8.;
  const double sdx = DMUL(dx, fact), sdy = DMUL(dy, fact), sdz = DMUL(dz, fact);
  const double margin = DMUL(1e-6, DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz)));
  int numpts = 0;
  for (int s = 0; s < nsph; ++s) {
    const double cx = sph[4 * s], cy = sph[4 * s + 1], cz = sph[4 * s + 2], r = sph[4 * s + 3];
    const double rsq = DMUL(r, r);
    const double lx = xini, hx = DADD(xini, dx), ly = yini, hy = DADD(yini, dy), lz = zini, hz = DADD(zini, dz);
    const double nx_ = fmax(0.0, fmax(DADD(lx, -cx), DADD(cx, -hx)));
    const double ny_ = fmax(0.0, fmax(DADD(ly, -cy), DADD(cy, -hy)));
    const double nz_ = fmax(0.0, fmax(DADD(lz, -cz), DADD(cz, -hz)));
    const double fx = fmax(fabs(DADD(lx, -cx)), fabs(DADD(hx, -cx)));
    const double fy = fmax(fabs(DADD(ly, -cy)), fabs(DADD(hy, -cy)));
    const double fz = fmax(fabs(DADD(lz, -cz)), fabs(DADD(hz, -cz)));
    const double near2 = DADD(DADD(DMUL(nx_, nx_), DMUL(ny_, ny_)), DMUL(nz_, nz_));
    const double far2 = DADD(DADD(DMUL(fx, fx), DMUL(fy, fy)), DMUL(fz, fz));
    if (near2 > DADD(rsq, margin)) continue;
    if (far2 < DADD(rsq, -margin)) { numpts += 512; continue; }
    for (int kz = 0; kz < 8; ++kz)
      for (int ky = 0; ky < 8; ++ky)
        for (int kx = 0; kx < 8; ++kx) {
          const double x_pt = DADD(xini, DMUL(sdx, kx + 0.5));
          const double y_pt = DADD(yini, DMUL(sdy, ky + 0.5));
          const double z_pt = DADD(zini, DMUL(sdz, kz + 0.5));
          const double ddx = DADD(x_pt, -cx), ddy = DADD(y_pt, -cy), ddz = DADD(z_pt, -cz);
          if (DADD(DADD(DMUL(ddx, ddx), DMUL(ddy, ddy)), DMUL(ddz, ddz)) <= rsq) numpts += 1;
        }
  }
  double frac = DMUL((double)numpts, 1. / 512.);
  if (frac > 1. - 1.e-2) frac = 1.0;
  sf[R.cell(ix, iy, iz)] = frac;
}

// k_set_solid_cell_from_ibm (CFD/G_SMACSolver_IBM.cu:763-792)
__global__ void k_ibm_set_solid(RefDims R, const double* __restrict__ sf, uint8_t* ct, uint8_t* fxt, uint8_t* fyt,
                                uint8_t* fzt) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int iz = blockIdx.z + 1;
  if (ix >= R.Nx + 2 || iy >= R.Ny + 2 || iz >= R.Nz + 2) return;
  if (sf[R.cell(ix, iy, iz)] > 1. - 1.e-12) {
    ct[R.cell(ix, iy, iz)] = C_SOLID;
    fxt[R.xf(ix, iy, iz)] = F_BOUNDARY;
    fxt[R.xf(ix + 1, iy, iz)] = F_BOUNDARY;
    fyt[R.yf(ix, iy, iz)] = F_BOUNDARY;
    fyt[R.yf(ix, iy + 1, iz)] = F_BOUNDARY;
    fzt[R.zf(ix, iy, iz)] = F_BOUNDARY;
    fzt[R.zf(ix, iy, iz + 1)] = F_BOUNDARY;
  }
}

}  // namespace smac
