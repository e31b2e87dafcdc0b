// smac_api.cu -- host side of the B200-native SMAC pressure projection:
// handle, multigrid hierarchy, CUDA-graph PCG iterations and the C ABI
// declared in include/smac_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "smac_b200.h"
#include "smac_kernels.cuh"
#include "smac_rbgs.cuh"
#include "smac_rbgs_tma.cuh"
#include "smac_rbgs_zm.cuh"
#include "smac_coarse_cluster.cuh"

#include <cudaTypedefs.h>
#include <type_traits>

using namespace smac;

namespace {

thread_local char g_err[512] = "";

void set_err(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

}  // namespace

namespace smac {
// error text for smac_last_error_string() from the other translation units
void set_error_text(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
}  // namespace smac

namespace {

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      set_err("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));        \
      return SMAC_CUDA_ERROR;                                                             \
    }                                                                                     \
  } while (0)

#define CKL()                                                                             \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      set_err("%s:%d: kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_));    \
      return SMAC_CUDA_ERROR;                                                             \
    }                                                                                     \
  } while (0)

#define TRY(expr)                       \
  do {                                  \
    smac_status st_ = (expr);           \
    if (st_ != SMAC_OK) return st_;     \
  } while (0)

// Launch of an iteration kernel (one that starts with pdl_enter()) with
// programmatic stream serialisation: its CTAs may be scheduled while the
// previous kernel drains, and wait on the device for that kernel's writes.
// SMAC_PDL=0 builds the plain stream order.  A launch error is left for
// CKL() to report.
#ifndef SMAC_PDL
#define SMAC_PDL 1
#endif
template <class... KArgs, class... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = SMAC_PDL;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr int MAXL = 16;
constexpr int COARSE_CELLS = 4096;  // grids at or below this size run in the single-CTA kernel

enum CoefType { CT_F64 = 0, CT_F32 = 1, CT_BF16 = 2 };

struct Level {
  Geom g{};
  int cx = 0, cy = 0, cz = 0;  // coarsened from the grid above
  double *bx64 = nullptr, *by64 = nullptr, *bz64 = nullptr;  // stencil weights f_b / h^2 of this grid
  double *x64 = nullptr, *x64b = nullptr, *rhs64 = nullptr;  // levels >= 1 (two iterates: out-of-place sweeps)
  void *bxm = nullptr, *bym = nullptr, *bzm = nullptr;  // mixed-precision weights
  int ctm = CT_F32;
  float *bxw = nullptr, *byw = nullptr, *bzw = nullptr;  // BF16 weights widened to FP32 (the cluster kernel's)
  float *x32 = nullptr, *x32b = nullptr, *rhs32 = nullptr;   // levels >= 1
  // TMA tensor maps of the fused sweep, indexed by the iterate buffer read
  SweepMaps mp64[2], mp32[2];
  bool tma64 = false, tma32 = false;
};

}  // namespace

struct smac_handle {
  smac_grid_desc desc{};
  smac_options opts{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  RefDims R{};
  int nlev = 0;
  int lc = 0;  // first grid of the single-CTA coarse set
  // the cluster set (k_coarse_cluster): its first grid (-1: not used), grids
  // spread over the ranks, and per grid its chunk and shared-memory offsets
  int lk = -1, kc_nd = 0;
  int kc_chunk[MAXL] = {}, kc_off[MAXL][5] = {};
  int kc_elems = 0;
  bool kc_ok[2] = {false, false};  // [FP32, FP64]: launchable
  Level lv[MAXL];
  uint8_t* fluid = nullptr;   // padded cell bits: 1 C_INTERIOR, 2 fluid unknown
  double *fbx = nullptr, *fby = nullptr, *fbz = nullptr;  // masked f_b, padded (divergence, correction, adjoint)
  double nfluid = 0.0;
  // copies of the reference-layout types (the correction and the adjoint read them)
  uint8_t *ct = nullptr, *fxt = nullptr, *fyt = nullptr, *fzt = nullptr;
  // fine FP64 vectors
  double *b64 = nullptr, *x64a = nullptr, *x64b = nullptr, *r64 = nullptr, *z64 = nullptr, *z64b = nullptr,
         *d64 = nullptr, *d64b = nullptr, *q64 = nullptr, *tmp64 = nullptr;
  // fine FP32 vectors (mixed)
  float *r32 = nullptr, *z32 = nullptr, *z32b = nullptr, *d32 = nullptr, *d32b = nullptr, *q32 = nullptr,
        *e32 = nullptr;
  RedBuf red{};
  long long red_blocks = 0;  // blocks a reducing launch may have (4 partials each)
  int num_sms = 148;
  long long l2_bytes = 126LL << 20;
  bool use_tma = true;     // fused sweeps stage their tiles with the copy engine
  int tma_ctas[2] = {1, 1};  // resident CTAs per SM of the TMA sweep: [0] FP32, [1] FP64
  int zm_ctas[2][6] = {};  // resident CTAs per SM of the z-march: [FP32, FP64][shape]
  Scalars* s = nullptr;    // device
  Scalars* hs = nullptr;   // pinned, mapped host mirror of the device scalars
  Scalars* hs_dev = nullptr;  // the mirror's device-side address
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [precision][gmg]
  bool have_coeffs = false, have_rhs = false;
  double dt = 1.0;
  double alg_bytes = 0.0;
  int launches = 0;
  std::vector<void*> allocs;
};

namespace {

template <class T>
smac_status dalloc(smac_handle* h, T** p, long long n) {
  void* q = nullptr;
  CK(cudaMalloc(&q, sizeof(T) * (size_t)n));
  CK(cudaMemsetAsync(q, 0, sizeof(T) * (size_t)n, h->stream));
  h->allocs.push_back(q);
  *p = (T*)q;
  return SMAC_OK;
}

// Padded array: returns the pointer to idx(0,0,0) (guard zeros in front).
template <class T>
smac_status palloc(smac_handle* h, const Geom& g, T** p) {
  T* base = nullptr;
  TRY(dalloc(h, &base, g.alloc));
  *p = base + g.guard;
  return SMAC_OK;
}

template <class T>
T* base_of(const Geom& g, T* p) {
  return p - g.guard;
}

inline int kz_for(const Geom& g) { return g.nz >= 64 ? 16 : (g.nz >= 16 ? 8 : 4); }
inline dim3 grid_cells(const Geom& g, int kz) {
  return dim3((g.nx + TBX - 1) / TBX, (g.ny + TBY - 1) / TBY, (g.nz + kz - 1) / kz);
}
inline dim3 grid_pairs(const Geom& g, int kz) {
  return dim3(((g.nx + 1) / 2 + TBX - 1) / TBX, (g.ny + TBY - 1) / TBY, (g.nz + kz - 1) / kz);
}
inline dim3 grid_planes(int nx, int ny, int nz) { return dim3((nx + TBX - 1) / TBX, (ny + TBY - 1) / TBY, nz); }
const dim3 kBlock(TBX, TBY, 1);

// Scalars between the device and the mapped host mirror, and clearing of
// solver buffers, by kernels on the handle's stream: copy engines would queue
// these small operations behind bulk copies of other streams (smac_async).
smac_status scalars_to_host(smac_handle* h) {
  k_copy_words<<<1, 64, 0, h->stream>>>(reinterpret_cast<const unsigned*>(h->s), reinterpret_cast<unsigned*>(h->hs_dev),
                                        (int)(sizeof(Scalars) / 4));
  CKL();
  return SMAC_OK;
}
smac_status scalars_to_device(smac_handle* h) {
  k_copy_words<<<1, 64, 0, h->stream>>>(reinterpret_cast<const unsigned*>(h->hs_dev), reinterpret_cast<unsigned*>(h->s),
                                        (int)(sizeof(Scalars) / 4));
  CKL();
  return SMAC_OK;
}
smac_status zero_async(smac_handle* h, void* p, size_t bytes) {
  const long long n16 = (long long)(bytes / 16);
  const int G = (int)std::max(1LL, std::min(4LL * h->num_sms, (n16 + 255) / 256));
  k_zero16<<<G, 256, 0, h->stream>>>(reinterpret_cast<int4*>(p), n16);
  CKL();
  return SMAC_OK;
}

template <class T, class C>
Stencil<T, C> stencil(const Geom&, const void* bx, const void* by, const void* bz) {
  return Stencil<T, C>{(const C*)bx, (const C*)by, (const C*)bz};
}

smac_status validate_options(const smac_options* o) {
  if (!o) { set_err("options: null"); return SMAC_BAD_ARG; }
  if (o->solver_type < 0 || o->solver_type > 3) { set_err("options: solver_type %d", o->solver_type); return SMAC_BAD_ARG; }
  if (o->precision < 0 || o->precision > 1) { set_err("options: precision %d", o->precision); return SMAC_BAD_ARG; }
  if (o->stop_rule < 0 || o->stop_rule > 1) { set_err("options: stop_rule %d", o->stop_rule); return SMAC_BAD_ARG; }
  if (!(o->tol > 0.0) || !std::isfinite(o->tol)) { set_err("options: tol must be > 0"); return SMAC_BAD_ARG; }
  if (o->max_iter < 1) { set_err("options: max_iter must be >= 1"); return SMAC_BAD_ARG; }
  if (o->min_coarse < 2) { set_err("options: min_coarse must be >= 2"); return SMAC_BAD_ARG; }
  if (o->max_levels < 1 || o->max_levels > MAXL) { set_err("options: max_levels in [1,16]"); return SMAC_BAD_ARG; }
  if (o->nu1 < 1 || o->nu2 < 1 || o->nu1 > 16 || o->nu2 > 16) { set_err("options: nu1, nu2 in [1,16]"); return SMAC_BAD_ARG; }
  if (o->coarse_sweeps < 1 || o->coarse_sweeps > 1024) { set_err("options: coarse_sweeps in [1,1024]"); return SMAC_BAD_ARG; }
  if (o->check_every < 1) { set_err("options: check_every >= 1"); return SMAC_BAD_ARG; }
  if (o->sweep_kernel < 0 || o->sweep_kernel > 3) { set_err("options: sweep_kernel %d", o->sweep_kernel); return SMAC_BAD_ARG; }
  if (o->coarse_kernel < 0 || o->coarse_kernel > 1) { set_err("options: coarse_kernel %d", o->coarse_kernel); return SMAC_BAD_ARG; }
  if (!(o->reliable_delta > 0.0 && o->reliable_delta < 1.0)) { set_err("options: reliable_delta in (0,1)"); return SMAC_BAD_ARG; }
  return SMAC_OK;
}

bool is_gmg(const smac_options& o) { return o.solver_type == SMAC_GMG_PCG || o.solver_type == SMAC_PURENEUMANN_GMG_PCG; }
bool is_pure(const smac_options& o) {
  return o.solver_type == SMAC_PURENEUMANN_GMG_PCG || o.solver_type == SMAC_PURENEUMANN_STANDARD_PCG;
}

// BF16 coefficients on the single-CTA grids when they are small enough and
// do not include the finest grid (whose mixed copy is FP32).
bool use_bf16(const smac_handle* h, const smac_options& o) {
  return h->lc >= 1 && o.bf16_coarse_cells > 0 && h->lv[h->lc].g.cells() <= o.bf16_coarse_cells;
}

void account(smac_handle* h, const Geom& g, double bytes_per_cell, int n = 1) {
  h->alg_bytes += bytes_per_cell * (double)g.cells() * n;
  h->launches += n;
}

// ---------------------------------------------------------------------------
// V-cycle launch sequence.  T: vector type, CS: coefficient type of the
// separately launched grids, CC: coefficient type of the single-CTA set.
// Grids above the single-CTA set use the fused out-of-place sweep
// (k_rbgs_sweep): pre-smoothing red first from x = 0, residual + restriction,
// post-smoothing black first with the prolongation fused into its first
// sweep; `dot` folds r.z into the last sweep of the finest grid.  Returns the
// buffer that holds z.
template <class T>
int sweep_zchunk(const Geom& g) {
  return g.nz >= 128 ? 16 : (g.nz >= 32 ? 8 : 4);
}
template <class T>
inline dim3 grid_sweep(const Geom& g, int zc) {
  constexpr int TY = RbTile<T>::TY;
  return dim3((g.nx + RB_TX - 1) / RB_TX, (g.ny + TY - 1) / TY, (g.nz + zc - 1) / zc);
}

template <class T, int MODE, bool DOT>
void launch_tma_sweep(smac_handle* h, int l, const SweepMaps& maps, T* xout, const double* sh, int c0, const T* xc) {
  typedef TmaTile<T> Lt;
  const Level& L = h->lv[l];
  const Geom& g = L.g;
  const Level& Lc = h->lv[l + 1 < h->nlev ? l + 1 : l];
  // z-chunk: fewest planes per CTA, counting the 4 staged halo planes of each item
  const long long ncol = (long long)((g.nx + Lt::TX - 1) / Lt::TX) * ((g.ny + Lt::TY - 1) / Lt::TY);
  const long long slots = (long long)h->tma_ctas[sizeof(T) == 8 ? 1 : 0] * h->num_sms;
  int zc = g.nz;
  long long best = -1;
  for (int cand = std::min(64, g.nz); cand >= std::min(4, g.nz); --cand) {
    const long long items = ncol * ((g.nz + cand - 1) / cand);
    const long long cost = ((items + slots - 1) / slots) * (cand + 4);
    if (best < 0 || cost < best) { best = cost; zc = cand; }
  }
  const long long items = ncol * ((g.nz + zc - 1) / zc);
  const int G = (int)std::max(1LL, std::min(std::min(slots, items), h->red_blocks));
  launch_pdl(k_rbgs_tma<T, MODE, DOT>, G, Lt::NT, Lt::SMEM_BYTES, h->stream, maps, g, xout, sh, c0, xc, Lc.g, Lc.cx,
      Lc.cy, Lc.cz, h->s, h->red, zc);
}

// z-march shapes: the whole x extent in WX warps of 32 x NV cells, TY tile
// rows.  FP64 (NV = 2): shape 0 one warp per row (x extent <= 64), 14 rows;
// shape 1 two warps (<= 128), 6 rows; shape 2 four warps (<= 256), 2 rows;
// shape 4 one warp, 6 rows (256 threads, two or more CTAs per SM).  FP32:
// shapes 0-2 and 4 the same with NV = 4 (extents 128, 256, 512 and 128),
// shape 3 four warps of float2 lanes (<= 256), 6 rows, 1024 threads, shape 5
// one warp of float2 lanes (<= 64), 6 rows.
template <class T> constexpr int zm_nv(int shape) {
  return sizeof(T) == 8 ? 2 : (shape == 3 || shape == 5) ? 2 : 4;
}
template <class T> constexpr int zm_wx(int shape) {
  return (shape == 0 || shape == 4 || shape == 5) ? 1 : shape == 1 ? 2 : 4;
}
template <class T> constexpr int zm_ty(int shape) { return shape == 0 ? 14 : shape == 2 ? 2 : 6; }
constexpr int ZM_SHAPES = 6;
// Rows of at most 128 (FP32) or 64 cells (FP64): SMAC_ZM_SMALL32 = 5 (the
// default) takes shape 5 for FP32 rows of at most 64 cells and shape 4 up to
// 128, 4 shape 4 for both, 0 the 14-row shape 0; SMAC_ZM_SMALL64 = 4 takes
// shape 4 for FP64 rows of at most 64 cells.  Measured (FP32 sweep): 64^3
// 5.6 us with shape 5, 7.0 with shape 4, 7.8 with shape 0; 128^3 12.4 with
// shape 4, 13.6 with shape 0; FP64 64^3 shape 4 7.25, shape 0 7.31 (not
// taken: the FP64 projection measured no faster).
#ifndef SMAC_ZM_SMALL32
#define SMAC_ZM_SMALL32 5
#endif
#ifndef SMAC_ZM_SMALL64
#define SMAC_ZM_SMALL64 0
#endif
#ifndef SMAC_ZM_F32_ORDER
#define SMAC_ZM_F32_ORDER 0, 1, 2, 3, -1, -1
#endif
// The narrowest shape that covers the x extent, or -1.  With `automatic`,
// -1 also where the TMA ring measured faster: a two-row tile (four warps per
// row) whose lanes are less than 80% busy.
template <class T>
int zm_shape(const smac_handle* h, const Geom& g, bool automatic) {
  const int pt = sizeof(T) == 8 ? 1 : 0;
  if (sizeof(T) == 4) {
    if (SMAC_ZM_SMALL32 == 5 && g.nx <= 64 && h->zm_ctas[0][5] > 0) return 5;
    if (SMAC_ZM_SMALL32 >= 4 && g.nx <= 128 && h->zm_ctas[0][4] > 0) return 4;
  } else if (SMAC_ZM_SMALL64 == 4 && g.nx <= 64 && h->zm_ctas[1][4] > 0) {
    return 4;
  }
  const int order32[ZM_SHAPES] = {SMAC_ZM_F32_ORDER};
  const int order64[ZM_SHAPES] = {0, 1, 2, -1, -1, -1};
  for (int q = 0; q < ZM_SHAPES; ++q) {
    const int sh = sizeof(T) == 8 ? order64[q] : order32[q];
    if (sh < 0) continue;
    const int tw = 32 * zm_nv<T>(sh) * zm_wx<T>(sh);
    if (g.nx <= tw && h->zm_ctas[pt][sh] > 0) {
      if (automatic && zm_ty<T>(sh) < 6 && 5 * g.nx < 4 * tw) return -1;
      return sh;
    }
  }
  return -1;
}

template <class T, int NV, int WX, int TY, int MODE, bool DOT>
void launch_zm_shape(smac_handle* h, int l, const T* xin, T* xout, const T* rhs, const double* sh, const void* bx,
                     const void* by, const void* bz, int c0, const T* xc, int ctas) {
  constexpr int NT = ZmTile<T, NV, WX, TY, MODE>::NT;
  const Geom& g = h->lv[l].g;
  const Level& Lc = h->lv[l + 1 < h->nlev ? l + 1 : l];
  // z-chunk: the fewest planes per CTA, counting the two extra c0 planes of each item
  const long long nty = (g.ny + TY - 1) / TY;
  const long long slots = (long long)ctas * h->num_sms;
  int zc = g.nz;
  long long best = -1;
  // (an item costs about six steps beyond its planes: two extra c0 planes and
  // the exposed latency of its first loads; measured at 192^3 and 256^3)
  for (int cand = std::min(64, g.nz); cand >= std::min(4, g.nz); --cand) {
    const long long items = nty * ((g.nz + cand - 1) / cand);
    const long long cost = ((items + slots - 1) / slots) * (cand + 6);
    if (best < 0 || cost < best) { best = cost; zc = cand; }
  }
  const long long items = nty * ((g.nz + zc - 1) / zc);
  // persistent CTAs; one partial sum each in the reduction buffer
  const int G = (int)std::max(1LL, std::min(std::min(slots, items), h->red_blocks));
  Stencil<T, T> S{(const T*)bx, (const T*)by, (const T*)bz};
  // the L2 prefetch pays only where the sweep's five arrays do not stay in
  // L2; its bulk copies need 16-byte aligned arrays (rows and planes are
  // multiples of 32 bytes)
  const uintptr_t al = (uintptr_t)xin | (uintptr_t)rhs | (uintptr_t)bx | (uintptr_t)by | (uintptr_t)bz;
  const int pf = ((al & 15u) == 0 && 5.0 * (double)g.alloc * sizeof(T) > (double)h->l2_bytes) ? SMAC_ZM_PF : 0;
  launch_pdl(k_rbgs_zm<T, NV, WX, TY, MODE, DOT>, G, NT, ZmTile<T, NV, WX, TY, MODE>::SMEM, h->stream, g, xin, xout,
      rhs, sh, S, c0, xc, Lc.g, Lc.cx, Lc.cy, Lc.cz, h->s, h->red, zc, pf);
}

template <class T, int MODE, bool DOT>
void launch_zm(smac_handle* h, int l, int shape, const T* xin, T* xout, const T* rhs, const double* sh,
               const void* bx, const void* by, const void* bz, int c0, const T* xc) {
  const int n = h->zm_ctas[sizeof(T) == 8 ? 1 : 0][shape];
#define ZM_SHAPE(S) launch_zm_shape<T, zm_nv<T>(S), zm_wx<T>(S), zm_ty<T>(S), MODE, DOT>(h, l, xin, xout, rhs, sh, bx, by, bz, c0, xc, n)
  if (shape == 0) ZM_SHAPE(0);
  else if (shape == 1) ZM_SHAPE(1);
  else if (shape == 2) ZM_SHAPE(2);
  else if (shape == 4) ZM_SHAPE(4);
  else if constexpr (sizeof(T) == 4) {
    if (shape == 3) ZM_SHAPE(3);
    else if (shape == 5) ZM_SHAPE(5);
  }
#undef ZM_SHAPE
}

template <class T>
void launch_zm_any(smac_handle* h, int l, int zs, int mode, bool dot, const T* xin, T* xout, const T* rhs,
                   const double* sh, const void* bx, const void* by, const void* bz, int c0, const T* xc) {
  if (mode == 0) { if (dot) launch_zm<T, 0, true>(h, l, zs, xin, xout, rhs, sh, bx, by, bz, c0, xc); else launch_zm<T, 0, false>(h, l, zs, xin, xout, rhs, sh, bx, by, bz, c0, xc); }
  else if (mode == 1) { if (dot) launch_zm<T, 1, true>(h, l, zs, xin, xout, rhs, sh, bx, by, bz, c0, xc); else launch_zm<T, 1, false>(h, l, zs, xin, xout, rhs, sh, bx, by, bz, c0, xc); }
  else { if (dot) launch_zm<T, 2, true>(h, l, zs, xin, xout, rhs, sh, bx, by, bz, c0, xc); else launch_zm<T, 2, false>(h, l, zs, xin, xout, rhs, sh, bx, by, bz, c0, xc); }
}

// One fused red-black sweep of grid l (mode 0 plain, 1 from zero, 2 with the
// prolongation of the coarse correction xc added to the input).  Returns true
// when mode 2 ran as a separate prolongation pass over xin (in place: the
// input of that sweep is consumed) followed by the plain sweep.
template <class T, class CS>
bool launch_sweep(smac_handle* h, int l, int mode, bool dot, const T* xin, T* xout, const T* rhs, const double* sh,
                  const void* bx, const void* by, const void* bz, int c0, const T* xc) {
  const Level& L = h->lv[l];
  const Geom& g = L.g;
  const Level& Lc = h->lv[l + 1 < h->nlev ? l + 1 : l];
  const int sk = h->opts.sweep_kernel;
  // FP64 sweeps from zero on rows wider than 128 cells take the shared-memory
  // tiles, which stage no input then: measured 173 against 226 us (z-march)
  // and 244 us (TMA ring) at 256^3, 68 against 119 and 104 us at 192^3.
  const bool zero_shared = sk == SMAC_SWEEP_AUTO && sizeof(T) == 8 && mode == 1 && g.nx > 128;
  if constexpr (std::is_same<T, CS>::value) {
    const int zs = (!zero_shared && (sk == SMAC_SWEEP_ZMARCH || sk == SMAC_SWEEP_AUTO))
                       ? zm_shape<T>(h, g, sk == SMAC_SWEEP_AUTO) : -1;
    if (zs >= 0) {
      if (mode == 2) {
        constexpr int NV = Vec16<T>::n;
        const long long vecs = (long long)((g.nx + NV - 1) / NV) * g.ny * g.nz;
        const int G = (int)std::max(1LL, std::min(8LL * h->num_sms, (vecs + 255) / 256));
        launch_pdl(k_prolong_add<T>, G, 256, 0, h->stream, g, const_cast<T*>(xin), xc, Lc.g, Lc.cx, Lc.cy, Lc.cz,
            h->s);
        launch_zm_any<T>(h, l, zs, 0, dot, xin, xout, rhs, sh, bx, by, bz, c0, nullptr);
        return true;
      }
      launch_zm_any<T>(h, l, zs, mode, dot, xin, xout, rhs, sh, bx, by, bz, c0, xc);
      return false;
    }
    const bool ok = sizeof(T) == 8 ? L.tma64 : L.tma32;
    if (h->use_tma && ok && sk != SMAC_SWEEP_SHARED && !zero_shared) {
      // the maps bind the level's two iterate buffers, its rhs and coefficients
      const SweepMaps* mp = sizeof(T) == 8 ? L.mp64 : L.mp32;
      const void* xb = (l == 0) ? (sizeof(T) == 8 ? (const void*)h->z64b : (const void*)h->z32b)
                                : (sizeof(T) == 8 ? (const void*)L.x64b : (const void*)L.x32b);
      const SweepMaps& M = mp[(xin != nullptr && (const void*)xin == xb) ? 1 : 0];
      if (mode == 0) { if (dot) launch_tma_sweep<T, 0, true>(h, l, M, xout, sh, c0, xc); else launch_tma_sweep<T, 0, false>(h, l, M, xout, sh, c0, xc); }
      else if (mode == 1) { if (dot) launch_tma_sweep<T, 1, true>(h, l, M, xout, sh, c0, xc); else launch_tma_sweep<T, 1, false>(h, l, M, xout, sh, c0, xc); }
      else { if (dot) launch_tma_sweep<T, 2, true>(h, l, M, xout, sh, c0, xc); else launch_tma_sweep<T, 2, false>(h, l, M, xout, sh, c0, xc); }
      (void)rhs; (void)bx; (void)by; (void)bz;
      return false;
    }
  }
  auto S = stencil<T, CS>(g, bx, by, bz);
  const int zc = sweep_zchunk<T>(g);
  const dim3 gr = grid_sweep<T>(g, zc);
  const dim3 bl(RB_NT, 1, 1);
#define SW(M, D)                                                                                           \
  launch_pdl(k_rbgs_sweep<T, CS, M, D>, gr, bl, 0, h->stream, g, xin, xout, rhs, sh, S, c0, xc, Lc.g, Lc.cx, Lc.cy, \
             Lc.cz, h->s, h->red, zc)
  if (mode == 0) { if (dot) SW(0, true); else SW(0, false); }
  else if (mode == 1) { if (dot) SW(1, true); else SW(1, false); }
  else { if (dot) SW(2, true); else SW(2, false); }
#undef SW
  return false;
}

// Mixed precision: the FP64 true residual and reliable update (k_reliable_vec).
void launch_reliable(smac_handle* h, const Geom& g, const Stencil<double, double>& S64, int kz) {
  const dim3 gr((g.nx + 2 * REL_TX - 1) / (2 * REL_TX), (g.ny + REL_TY - 1) / REL_TY, (g.nz + kz - 1) / kz);
  launch_pdl(k_reliable_vec<float>, gr, dim3(REL_TX, REL_TY, 1), 0, h->stream, g, h->x64a, h->x64b, h->e32, h->b64, S64,
      h->r32, h->red, h->s, kz);
}

// d = z - zshift + beta d, q = A d, p.Ap (k_dir_matvec_vec).
template <class T>
void launch_dir_matvec(smac_handle* h, const Geom& g, const T* z, const T* dold, T* dnew, const Stencil<T, T>& S,
                       T* q, int kz) {
  constexpr int NV = Vec16<T>::n;
  const dim3 gr((g.nx + DMV_TX * NV - 1) / (DMV_TX * NV), (g.ny + DMV_TY - 1) / DMV_TY, (g.nz + kz - 1) / kz);
  launch_pdl(k_dir_matvec_vec<T>, gr, dim3(DMV_TX, DMV_TY, 1), 0, h->stream, g, z, dold, dnew, S, q, h->fluid, h->red,
      h->s, kz);
}

// x += alpha d, r -= alpha q over whole padded arrays (k_update_flat).
template <class T>
void launch_update(smac_handle* h, const Geom& g, T* x, const T* d, T* r, const T* q) {
  const long long nvec = g.alloc / Vec16<T>::n;
  const long long blocks = (nvec + UPD_NT - 1) / UPD_NT;
  const int G = (int)std::max(1LL, std::min(4LL * h->num_sms, blocks));
  launch_pdl(k_update_flat<T>, G, UPD_NT, 0, h->stream, base_of(g, x), base_of(g, d), base_of(g, r), base_of(g, q),
      g.alloc, h->red, h->s);
}

// Whether the lower part of the V-cycle runs in the cluster kernel, and the
// first grid of the part that does not run sweep by sweep.
bool use_cluster(const smac_handle* h, bool mixed) {
  return h->lk >= 1 && h->opts.coarse_kernel == SMAC_COARSE_AUTO && h->kc_ok[mixed ? 0 : 1];
}
int coarse_start(const smac_handle* h, bool mixed) { return use_cluster(h, mixed) ? h->lk : h->lc; }

// Global bytes of the cluster kernel per launch: the first grid's rhs in and
// x out, every grid's three weight arrays in.
double cluster_bytes(const smac_handle* h, bool mixed) {
  const double s = mixed ? 4.0 : 8.0;
  double b = 2.0 * s * (double)h->lv[h->lk].g.cells();
  for (int l = h->lk; l < h->nlev; ++l) {
    const double sc = mixed ? 4.0 : 8.0;  // (BF16 weights through their FP32 copies)
    b += 3.0 * sc * (double)h->lv[l].g.cells();
  }
  return b;
}

template <class T>
void launch_cluster(smac_handle* h, bool mixed, const T* rhs, T* x) {
  ClusterSet set{};
  set.n = h->nlev - h->lk;
  set.nd = h->kc_nd;
  for (int q = 0; q < set.n; ++q) {
    const Level& L = h->lv[h->lk + q];
    ClusterLevel& C = set.L[q];
    C.g = L.g;
    C.cx = L.cx; C.cy = L.cy; C.cz = L.cz;
    C.chunk = h->kc_chunk[q];
    C.ox = h->kc_off[q][0]; C.orhs = h->kc_off[q][1];
    C.obx = h->kc_off[q][2]; C.oby = h->kc_off[q][3]; C.obz = h->kc_off[q][4];
    // every array staged as T: BF16 weights through their exact FP32 copies
    const bool wide = mixed && L.ctm == CT_BF16;
    C.ctype = mixed ? CT_F32 : CT_F64;
    C.bx = wide ? (const void*)L.bxw : mixed ? L.bxm : (const void*)L.bx64;
    C.by = wide ? (const void*)L.byw : mixed ? L.bym : (const void*)L.by64;
    C.bz = wide ? (const void*)L.bzw : mixed ? L.bzm : (const void*)L.bz64;
  }
  set.rhs0 = rhs;
  set.x0 = x;
  launch_pdl(k_coarse_cluster<T>, KCL, kcl_threads<T>(), (size_t)h->kc_elems * sizeof(T), h->stream, set, h->opts.nu1,
      h->opts.nu2, h->opts.coarse_sweeps, (const Scalars*)h->s);
  h->alg_bytes += cluster_bytes(h, mixed);
  h->launches += 1;
}

template <class T, class CS, class CC>
smac_status launch_vcycle(smac_handle* h, T* r0, T* z0a, T* z0b, bool mixed, bool dot, T** z_out) {
  const smac_options& o = h->opts;
  const bool clu = use_cluster(h, mixed);
  const int lc = coarse_start(h, mixed);
  const double* shift0 = &h->s->rshift;
  const double s = sizeof(T);
  const double sc = mixed ? (double)sizeof(CS) : 8.0;
  auto XA = [&](int l) -> T* { return l == 0 ? z0a : (mixed ? (T*)h->lv[l].x32 : (T*)h->lv[l].x64); };
  auto XB = [&](int l) -> T* { return l == 0 ? z0b : (mixed ? (T*)h->lv[l].x32b : (T*)h->lv[l].x64b); };
  auto B = [&](int l) -> T* { return l == 0 ? r0 : (mixed ? (T*)h->lv[l].rhs32 : (T*)h->lv[l].rhs64); };
  auto CF = [&](int l, int which) -> const void* {
    const Level& L = h->lv[l];
    if (!mixed) return which == 0 ? (const void*)L.bx64 : which == 1 ? (const void*)L.by64 : (const void*)L.bz64;
    return which == 0 ? L.bxm : which == 1 ? L.bym : L.bzm;
  };
  T* cur[MAXL] = {};
  T* fin[MAXL] = {};
  auto other = [&](int l, T* p) { return p == XA(l) ? XB(l) : XA(l); };
  for (int l = 0; l < lc; ++l) {
    const Geom& g = h->lv[l].g;
    const double* sh = (l == 0) ? shift0 : nullptr;
    T* in = nullptr;
    T* out = XA(l);
    launch_sweep<T, CS>(h, l, 1, false, in, out, B(l), sh, CF(l, 0), CF(l, 1), CF(l, 2), 0, nullptr);
    account(h, g, 4.0 * s + 3 * sc, 1);
    in = out;
    for (int it = 1; it < o.nu1; ++it) {
      out = other(l, in);
      launch_sweep<T, CS>(h, l, 0, false, in, out, B(l), sh, CF(l, 0), CF(l, 1), CF(l, 2), 0, nullptr);
      account(h, g, 3.0 * s + 3 * sc, 1);
      in = out;
    }
    cur[l] = in;
    CKL();
    const Level& Lc = h->lv[l + 1];
    auto S = stencil<T, CS>(g, CF(l, 0), CF(l, 1), CF(l, 2));
    if (std::is_same<T, CS>::value && Lc.cx && Lc.cy && Lc.cz)
      launch_pdl(k_resid_restrict2<T>, grid_planes(Lc.g.nx, Lc.g.ny, Lc.g.nz), kBlock, 0, h->stream, g, cur[l], B(l),
          sh, stencil<T, T>(g, CF(l, 0), CF(l, 1), CF(l, 2)), Lc.g, B(l + 1), h->s);
    else
      launch_pdl(k_resid_restrict<T, CS>, grid_planes(Lc.g.nx, Lc.g.ny, Lc.g.nz), kBlock, 0, h->stream, g, cur[l], B(l),
          sh, S, Lc.g, Lc.cx, Lc.cy, Lc.cz, B(l + 1), h->s);
    account(h, g, 2 * s + 3 * sc + s / 8, 1);
    CKL();
  }
  if (clu) {
    launch_cluster<T>(h, mixed, B(lc), XA(lc));
    CKL();
    fin[lc] = XA(lc);
  } else {
    // single-CTA coarse set, in place on XA
    CoarseSet set{};
    set.n = h->nlev - lc;
    for (int q = 0; q < set.n; ++q) {
      const int l = lc + q;
      CoarseLevel& C = set.L[q];
      C.g = h->lv[l].g;
      C.cx = h->lv[l].cx; C.cy = h->lv[l].cy; C.cz = h->lv[l].cz;
      C.bx = CF(l, 0); C.by = CF(l, 1); C.bz = CF(l, 2);
      C.x = XA(l);
      C.rhs = B(l);
    }
    launch_pdl(k_coarse_vcycle<T, CC>, 1, 1024, 0, h->stream, set, o.nu1, o.nu2, o.coarse_sweeps,
        lc == 0 ? shift0 : nullptr, h->s);
    h->launches += 1;
    CKL();
    fin[lc] = XA(lc);
  }
  for (int l = lc - 1; l >= 0; --l) {
    const Geom& g = h->lv[l].g;
    const double* sh = (l == 0) ? shift0 : nullptr;
    T* in = cur[l];
    for (int it = 0; it < o.nu2; ++it) {
      T* out = other(l, in);
      const bool last_dot = dot && l == 0 && it == o.nu2 - 1;
      const bool split = launch_sweep<T, CS>(h, l, it == 0 ? 2 : 0, last_dot, in, out, B(l), sh, CF(l, 0), CF(l, 1),
                                             CF(l, 2), 1, it == 0 ? fin[l + 1] : nullptr);
      if (split) {  // the prolongation pass (x read and written, coarse read), then the plain sweep
        account(h, g, 2.0 * s + s / 8, 1);
        account(h, g, 3.0 * s + 3 * sc, 1);
      } else {
        account(h, g, 3.0 * s + 3 * sc + (it == 0 ? s / 8 : 0.0), 1);
      }
      in = out;
    }
    fin[l] = in;
    CKL();
  }
  *z_out = fin[0];
  return SMAC_OK;
}

// One PCG iteration: preconditioner (+ r.z, beta), direction update fused
// with the matvec (+ p.Ap, alpha), update of x and r (+ stopping test), and
// in mixed precision the FP64 residual recomputation when requested.
// `parity` selects which direction buffer is the old one.
smac_status launch_iteration(smac_handle* h, bool mixed, bool gmg, int parity) {
  const Geom& g = h->lv[0].g;
  const int kz = kz_for(g);
  const dim3 gr = grid_cells(g, kz);
  const bool fused_dot = gmg && h->lc > 0;
  if (!mixed) {
    double* z = h->z64;
    if (gmg) {
      TRY((launch_vcycle<double, double, double>(h, h->r64, h->z64, h->z64b, false, fused_dot, &z)));
    } else {
      auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
      launch_pdl(k_jacobi_precond<double, double>, gr, kBlock, 0, h->stream, g, h->r64, &h->s->rshift, S, h->z64, h->s,
          kz);
      account(h, g, 2 * 8 + 3 * 8);
    }
    if (!fused_dot) {
      launch_pdl(k_dot_rz<double>, gr, kBlock, 0, h->stream, g, h->r64, z, h->red, h->s, kz);
      account(h, g, 16, 1);
    }
    double* dold = parity ? h->d64b : h->d64;
    double* dnew = parity ? h->d64 : h->d64b;
    auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
    launch_dir_matvec<double>(h, g, z, dold, dnew, S, h->q64, kz);
    launch_update<double>(h, g, h->x64a, dnew, h->r64, h->q64);
    account(h, g, 7 * 8, 1);
    account(h, g, 6 * 8, 1);
    CKL();
  } else {
    const bool bf16 = use_bf16(h, h->opts);
    float* z = h->z32;
    if (gmg) {
      if (bf16) {
        TRY((launch_vcycle<float, float, __nv_bfloat16>(h, h->r32, h->z32, h->z32b, true, fused_dot, &z)));
      } else {
        TRY((launch_vcycle<float, float, float>(h, h->r32, h->z32, h->z32b, true, fused_dot, &z)));
      }
    } else {
      auto S = stencil<float, float>(g, h->lv[0].bxm, h->lv[0].bym, h->lv[0].bzm);
      launch_pdl(k_jacobi_precond<float, float>, gr, kBlock, 0, h->stream, g, h->r32, &h->s->rshift, S, h->z32, h->s,
          kz);
      account(h, g, 2 * 4 + 3 * 4);
    }
    if (!fused_dot) {
      launch_pdl(k_dot_rz<float>, gr, kBlock, 0, h->stream, g, h->r32, z, h->red, h->s, kz);
      account(h, g, 8, 1);
    }
    float* dold = parity ? h->d32b : h->d32;
    float* dnew = parity ? h->d32 : h->d32b;
    auto S = stencil<float, float>(g, h->lv[0].bxm, h->lv[0].bym, h->lv[0].bzm);
    launch_dir_matvec<float>(h, g, z, dold, dnew, S, h->q32, kz);
    launch_update<float>(h, g, h->e32, dnew, h->r32, h->q32);
    auto S64 = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
    launch_reliable(h, g, S64, kz);
    account(h, g, 7 * 4, 1);
    account(h, g, 6 * 4, 1);
    h->launches += 1;  // the FP64 residual kernel (its bytes are counted when it runs)
    CKL();
  }
  return SMAC_OK;
}

smac_status get_graph(smac_handle* h, bool mixed, bool gmg, cudaGraphExec_t* out) {
  cudaGraphExec_t& ex = h->graph[mixed ? 1 : 0][gmg ? 1 : 0];
  if (!ex) {
    cudaGraph_t graph = nullptr;
    const double saved_bytes = h->alg_bytes;
    const int saved_launches = h->launches;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    smac_status st = launch_iteration(h, mixed, gmg, 0);
    if (st == SMAC_OK) st = launch_iteration(h, mixed, gmg, 1);
    cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
    h->alg_bytes = saved_bytes;
    h->launches = saved_launches;
    if (st != SMAC_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (ec != cudaSuccess) {
      set_err("stream capture: %s", cudaGetErrorString(ec));
      return SMAC_CUDA_ERROR;
    }
    cudaError_t ei = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      ex = nullptr;
      set_err("graph instantiate: %s", cudaGetErrorString(ei));
      return SMAC_CUDA_ERROR;
    }
  }
  *out = ex;
  return SMAC_OK;
}

void drop_graphs(smac_handle* h) {
  for (auto& a : h->graph)
    for (auto& e : a)
      if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

// Algorithmic bytes of one PCG iteration (the byte model: every array a
// kernel must touch, read or written once; s = vector element size, sc =
// coefficient element size): fused sweeps 5s+... per cell as accounted in
// launch_vcycle, direction+matvec 7s, update 6s.
double iteration_bytes(smac_handle* h, bool mixed, bool gmg, int* launches) {
  const Geom& g = h->lv[0].g;
  double bytes = 0.0;
  int n = 0;
  const double s = mixed ? 4.0 : 8.0;
  if (gmg) {
    const int lc = coarse_start(h, mixed);
    for (int l = 0; l < lc; ++l) {
      const double cells = (double)h->lv[l].g.cells();
      const double sc = mixed ? 4.0 : 8.0;
      bytes += (4.0 * s + 3 * sc) * cells;
      n += 1;
      for (int it = 1; it < h->opts.nu1; ++it) { bytes += (3.0 * s + 3 * sc) * cells; n += 1; }
      bytes += (2 * s + 3 * sc + s / 8) * cells;
      n += 1;
      // the first post-smoothing sweep: fused with the prolongation, or (the
      // z-march) a prolongation pass followed by the plain sweep
      const int sk = h->opts.sweep_kernel;
      const bool zm_ok = sk == SMAC_SWEEP_ZMARCH || sk == SMAC_SWEEP_AUTO;
      const bool split = zm_ok && (mixed ? zm_shape<float>(h, h->lv[l].g, sk == SMAC_SWEEP_AUTO)
                                         : zm_shape<double>(h, h->lv[l].g, sk == SMAC_SWEEP_AUTO)) >= 0;
      if (split) { bytes += (2.0 * s + s / 8) * cells; n += 1; }
      for (int it = 0; it < h->opts.nu2; ++it) {
        bytes += (3.0 * s + 3 * sc + (it == 0 && !split ? s / 8 : 0.0)) * cells;
        n += 1;
      }
    }
    n += 1;  // the coarse grids' kernel (the single-CTA one's bytes are negligible)
    if (use_cluster(h, mixed)) bytes += cluster_bytes(h, mixed);
    if (lc == 0) { bytes += 2 * s * (double)g.cells(); n += 1; }
  } else {
    bytes += (2 * s + 3 * s) * (double)g.cells() + 2 * s * (double)g.cells();
    n += 2;
  }
  bytes += (7 * s + 6 * s) * (double)g.cells();
  n += 2;
  if (mixed) n += 1;
  if (launches) *launches = n;
  return bytes;
}


// ---------------------------------------------------------------------------
// TMA tensor maps.  cuTensorMapEncodeTiled is reached through the runtime's
// driver entry point (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

bool tma_encoder() {
  if (g_encode) return true;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return false;
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return true;
}

// 3-D map of a padded array: extents (e0, e1, e2) elements, row/plane strides
// of the layout, box (b0, b1, 1); out-of-bounds elements read as zero.
bool encode_map(CUtensorMap* m, const void* base, bool f64, const Geom& g, int e0, int e1, int e2, int b0, int b1) {
  const size_t es = f64 ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)e0, (cuuint64_t)e1, (cuuint64_t)e2};
  cuuint64_t strides[2] = {(cuuint64_t)g.px * es, (cuuint64_t)g.ps * es};
  cuuint32_t box[3] = {(cuuint32_t)b0, (cuuint32_t)b1, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = g_encode(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                              const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <class T>
bool build_level_maps(SweepMaps (&mp)[2], const Geom& g, const void* xa, const void* xb, const void* rhs,
                      const void* bx, const void* by, const void* bz) {
  typedef TmaTile<T> Lt;
  const bool f64 = sizeof(T) == 8;
  for (int q = 0; q < 2; ++q) {
    SweepMaps& M = mp[q];
    if (!encode_map(&M.xin, q == 0 ? xa : xb, f64, g, g.nx, g.ny, g.nz, Lt::XW, Lt::XH)) return false;
    if (!encode_map(&M.rhs, rhs, f64, g, g.nx, g.ny, g.nz, Lt::XW, Lt::RH)) return false;
    if (!encode_map(&M.bx, bx, f64, g, g.nx + 1, g.ny, g.nz, Lt::XW, Lt::RH)) return false;
    if (!encode_map(&M.by, by, f64, g, g.nx, g.ny + 1, g.nz, Lt::XW, Lt::YH)) return false;
    if (!encode_map(&M.bz, bz, f64, g, g.nx, g.ny, g.nz + 1, Lt::XW, Lt::RH)) return false;
  }
  return true;
}

template <class T, int MODE, bool DOT>
cudaError_t tma_attr() {
  return cudaFuncSetAttribute(k_rbgs_tma<T, MODE, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              TmaTile<T>::SMEM_BYTES);
}

// Resident CTAs per SM of each z-march shape (0: not usable): the kernels'
// shared-memory limit raised to their needs, then the fewest resident CTAs
// of the six forms.
template <class T, int SH, int MODE, bool DOT>
int zm_occupancy_one() {
  constexpr int NV = zm_nv<T>(SH), WX = zm_wx<T>(SH), TY = zm_ty<T>(SH);
  constexpr int NT = ZmTile<T, NV, WX, TY, MODE>::NT;
  constexpr int SM = ZmTile<T, NV, WX, TY, MODE>::SMEM;
  auto fn = k_rbgs_zm<T, NV, WX, TY, MODE, DOT>;
  int n = 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, SM) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, NT, SM) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
template <class T, int SH>
int zm_occupancy() {
  const int n[6] = {zm_occupancy_one<T, SH, 0, false>(), zm_occupancy_one<T, SH, 0, true>(),
                    zm_occupancy_one<T, SH, 1, false>(), zm_occupancy_one<T, SH, 1, true>(),
                    zm_occupancy_one<T, SH, 2, false>(), zm_occupancy_one<T, SH, 2, true>()};
  int m = n[0];
  for (int v : n) m = std::min(m, v);
  return m;
}
void setup_zm(smac_handle* h) {
  h->zm_ctas[0][0] = zm_occupancy<float, 0>();
  h->zm_ctas[0][1] = zm_occupancy<float, 1>();
  h->zm_ctas[0][2] = zm_occupancy<float, 2>();
  h->zm_ctas[0][3] = zm_occupancy<float, 3>();
  h->zm_ctas[0][4] = zm_occupancy<float, 4>();
  h->zm_ctas[0][5] = zm_occupancy<float, 5>();
  h->zm_ctas[1][0] = zm_occupancy<double, 0>();
  h->zm_ctas[1][1] = zm_occupancy<double, 1>();
  h->zm_ctas[1][2] = zm_occupancy<double, 2>();
  h->zm_ctas[1][3] = 0;
  h->zm_ctas[1][4] = zm_occupancy<double, 4>();
  h->zm_ctas[1][5] = 0;
}

// The cluster set: from the first grid below the finest with <= KCL_TOP
// cells down, where the coarsest grid has <= KCL_SOLO cells (rank 0 holds
// those) and one rank's share fits in shared memory.  The spread grids'
// chunks halve with every z-coarsening, so that a coarse plane is in the
// rank of its two children: the first chunk is the planes per rank rounded
// up to a multiple of 2^(z-coarsenings below it within the spread grids and
// into the first held one).
template <class T>
bool cluster_attr(int bytes) {
  if (cudaFuncSetAttribute(k_coarse_cluster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(KCL, 1, 1);
  cfg.blockDim = dim3(kcl_threads<T>(), 1, 1);
  cfg.dynamicSmemBytes = (size_t)bytes;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_coarse_cluster<T>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n >= 1;
}

void setup_cluster(smac_handle* h, int smem_optin) {
  h->lk = -1;
  int lk = -1;
  for (int l = 1; l < h->nlev; ++l)
    if (h->lv[l].g.cells() <= KCL_TOP) { lk = l; break; }
  if (lk < 1 || h->lv[h->nlev - 1].g.cells() > KCL_SOLO || h->nlev - lk > MAX_CLL) return;
  const int n = h->nlev - lk;
  int nd = 0;
  while (nd < n && h->lv[lk + nd].g.cells() > KCL_SOLO) ++nd;
  int pow2 = 1;
  for (int q = 1; q <= nd && q < n; ++q)
    if (h->lv[lk + q].cz) pow2 *= 2;
  const int nz0 = h->lv[lk].g.nz;
  int chunk = (nz0 + KCL - 1) / KCL;
  chunk = (chunk + pow2 - 1) / pow2 * pow2;
  long long tot = 0;
  auto take = [&](long long e) { const long long o = tot; tot += (e + 3) / 4 * 4; return (int)o; };
  for (int q = 0; q < n; ++q) {
    const Geom& g = h->lv[lk + q].g;
    if (q > 0 && q < nd && h->lv[lk + q].cz) chunk /= 2;
    const int c = q < nd ? chunk : g.nz;
    if (c < 1) return;
    h->kc_chunk[q] = c;
    const long long nx = g.nx, ny = g.ny;
    h->kc_off[q][0] = take(c * nx * ny);            // x
    h->kc_off[q][1] = take(c * nx * ny);            // rhs
    h->kc_off[q][2] = take(c * ny * (nx + 1));      // bx
    h->kc_off[q][3] = take(c * (ny + 1) * nx);      // by
    h->kc_off[q][4] = take((c + 1) * ny * nx);      // bz
  }
  if (tot * 8 > (1LL << 30)) return;
  h->kc_elems = (int)tot;
  h->kc_nd = nd;
  h->kc_ok[0] = tot * 4 <= smem_optin && cluster_attr<float>((int)(tot * 4));
  h->kc_ok[1] = tot * 8 <= smem_optin && cluster_attr<double>((int)(tot * 8));
  if (h->kc_ok[0] || h->kc_ok[1]) h->lk = lk;
}

// Tensor maps for every separately launched grid, or use_tma = false.
void setup_tma(smac_handle* h) {
  h->use_tma = false;
  if (!tma_encoder()) return;
  cudaError_t e = cudaSuccess;
  cudaError_t es[12] = {tma_attr<double, 0, false>(), tma_attr<double, 0, true>(), tma_attr<double, 1, false>(),
                        tma_attr<double, 1, true>(),  tma_attr<double, 2, false>(), tma_attr<double, 2, true>(),
                        tma_attr<float, 0, false>(),  tma_attr<float, 0, true>(),  tma_attr<float, 1, false>(),
                        tma_attr<float, 1, true>(),   tma_attr<float, 2, false>(), tma_attr<float, 2, true>()};
  for (cudaError_t x : es)
    if (x != cudaSuccess) e = x;
  if (e != cudaSuccess) { cudaGetLastError(); return; }
  {
    int n32 = 0, n64 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n32, k_rbgs_tma<float, 0, true>, TmaTile<float>::NT,
                                                      TmaTile<float>::SMEM_BYTES) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n64, k_rbgs_tma<double, 0, true>, TmaTile<double>::NT,
                                                      TmaTile<double>::SMEM_BYTES) != cudaSuccess ||
        n32 < 1 || n64 < 1) {
      cudaGetLastError();
      return;
    }
    h->tma_ctas[0] = n32;
    h->tma_ctas[1] = n64;
  }
  for (int l = 0; l < h->nlev; ++l) {
    Level& L = h->lv[l];
    const void* xa64 = l == 0 ? (const void*)h->z64 : (const void*)L.x64;
    const void* xb64 = l == 0 ? (const void*)h->z64b : (const void*)L.x64b;
    const void* r64 = l == 0 ? (const void*)h->r64 : (const void*)L.rhs64;
    const void* xa32 = l == 0 ? (const void*)h->z32 : (const void*)L.x32;
    const void* xb32 = l == 0 ? (const void*)h->z32b : (const void*)L.x32b;
    const void* r32 = l == 0 ? (const void*)h->r32 : (const void*)L.rhs32;
    L.tma64 = build_level_maps<double>(L.mp64, L.g, xa64, xb64, r64, L.bx64, L.by64, L.bz64);
    L.tma32 = L.ctm == CT_F32 && build_level_maps<float>(L.mp32, L.g, xa32, xb32, r32, L.bxm, L.bym, L.bzm);
  }
  h->use_tma = true;
}

}  // namespace

// Internal accessors for smac_async.cu.
namespace smac {
cudaStream_t handle_stream(const smac_handle* h) { return h->stream; }
void handle_shape(const smac_handle* h, int* nx, int* ny, int* nz) {
  *nx = h->desc.nx;
  *ny = h->desc.ny;
  *nz = h->desc.nz;
}
}  // namespace smac

// ===========================================================================
extern "C" {

const char* smac_last_error_string(void) { return g_err; }

smac_status smac_default_options(smac_options* o) {
  if (!o) { set_err("null options"); return SMAC_BAD_ARG; }
  o->solver_type = SMAC_PURENEUMANN_GMG_PCG;
  o->precision = SMAC_PRECISION_FP64;
  o->stop_rule = SMAC_STOP_RELATIVE;
  o->tol = 1e-8;
  o->max_iter = 2000;
  o->min_coarse = 4;
  o->max_levels = 16;
  o->nu1 = 2;
  o->nu2 = 2;
  o->coarse_sweeps = 8;
  o->check_every = 1;
  o->reliable_delta = 1e-4;
  o->bf16_coarse_cells = COARSE_CELLS;
  o->sweep_kernel = SMAC_SWEEP_AUTO;
  o->coarse_kernel = SMAC_COARSE_AUTO;
  return SMAC_OK;
}

smac_status smac_create(const smac_grid_desc* desc, const smac_options* opts, void* cuda_stream, smac_handle** out) {
  if (!desc || !out) { set_err("smac_create: null argument"); return SMAC_BAD_ARG; }
  *out = nullptr;
  smac_options o;
  if (opts) o = *opts; else smac_default_options(&o);
  TRY(validate_options(&o));
  if (desc->nx < 2 || desc->ny < 2 || desc->nz < 2 || !(desc->dx > 0) || !(desc->dy > 0) || !(desc->dz > 0)) {
    set_err("smac_create: grid %dx%dx%d, spacing must be > 0", desc->nx, desc->ny, desc->nz);
    return SMAC_BAD_SHAPE;
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_err("smac_create: no CUDA device: %s", cudaGetErrorString(e)); return SMAC_NO_DEVICE; }
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major != 10) {
    set_err("smac_create: device %s is sm_%d%d; this library is built for sm_100a", prop.name, prop.major, prop.minor);
    return SMAC_NO_DEVICE;
  }
  smac_handle* h = new (std::nothrow) smac_handle();
  if (!h) { set_err("smac_create: out of host memory"); return SMAC_BAD_ARG; }
  h->desc = *desc;
  h->opts = o;
  h->R = RefDims{desc->nx, desc->ny, desc->nz};
  if (cuda_stream) {
    h->stream = (cudaStream_t)cuda_stream;
  } else {
    // a blocking stream: ordered with work on the legacy default stream, and capturable
    cudaError_t es = cudaStreamCreate(&h->stream);
    if (es != cudaSuccess) { set_err("cudaStreamCreate: %s", cudaGetErrorString(es)); delete h; return SMAC_CUDA_ERROR; }
    h->own_stream = true;
  }
  auto fail = [&](smac_status st) {
    char keep[512];
    memcpy(keep, g_err, sizeof(keep));
    smac_destroy(h);
    memcpy(g_err, keep, sizeof(keep));
    return st;
  };
  // hierarchy: halve a direction while it stays even and >= min_coarse
  {
    int nx = desc->nx, ny = desc->ny, nz = desc->nz;
    double ix2 = 1.0 / (desc->dx * desc->dx), iy2 = 1.0 / (desc->dy * desc->dy), iz2 = 1.0 / (desc->dz * desc->dz);
    h->lv[0].g = make_geom(nx, ny, nz, ix2, iy2, iz2);
    h->nlev = 1;
    while (h->nlev < o.max_levels && is_gmg(o)) {
      const int cx = (nx % 2 == 0 && nx / 2 >= o.min_coarse), cy = (ny % 2 == 0 && ny / 2 >= o.min_coarse),
                cz = (nz % 2 == 0 && nz / 2 >= o.min_coarse);
      if (!cx && !cy && !cz) break;
      if (cx) { nx /= 2; ix2 *= 0.25; }
      if (cy) { ny /= 2; iy2 *= 0.25; }
      if (cz) { nz /= 2; iz2 *= 0.25; }
      Level& L = h->lv[h->nlev];
      L.g = make_geom(nx, ny, nz, ix2, iy2, iz2);
      L.cx = cx; L.cy = cy; L.cz = cz;
      h->nlev += 1;
    }
    h->lc = h->nlev - 1;
    for (int l = 0; l < h->nlev; ++l)
      if (h->lv[l].g.cells() <= COARSE_CELLS) { h->lc = l; break; }
    if (h->lv[0].g.alloc >= (1LL << 31)) { set_err("smac_create: grid too large for 32-bit indexing"); return fail(SMAC_BAD_SHAPE); }
  }
  // storage
  const Geom& g0 = h->lv[0].g;
  smac_status st;
#define PA(ptr) do { st = palloc(h, g0, &(ptr)); if (st != SMAC_OK) return fail(st); } while (0)
  PA(h->lv[0].bx64); PA(h->lv[0].by64); PA(h->lv[0].bz64);
  PA(h->fbx); PA(h->fby); PA(h->fbz);
  PA(h->b64); PA(h->x64a); PA(h->x64b); PA(h->r64); PA(h->z64); PA(h->z64b); PA(h->d64); PA(h->d64b); PA(h->q64);
  PA(h->tmp64);
  {
    float* p;
    st = palloc(h, g0, &p); if (st != SMAC_OK) return fail(st); h->lv[0].bxm = p;
    st = palloc(h, g0, &p); if (st != SMAC_OK) return fail(st); h->lv[0].bym = p;
    st = palloc(h, g0, &p); if (st != SMAC_OK) return fail(st); h->lv[0].bzm = p;
    h->lv[0].ctm = CT_F32;
  }
  PA(h->r32); PA(h->z32); PA(h->z32b); PA(h->d32); PA(h->d32b); PA(h->q32); PA(h->e32);
  PA(h->fluid);
#undef PA
  {
    const long long nc = (long long)(desc->nx + 2) * (desc->ny + 2) * (desc->nz + 2);
    const long long nxf = (long long)(desc->nx + 3) * (desc->ny + 2) * (desc->nz + 2);
    const long long nyf = (long long)(desc->nx + 2) * (desc->ny + 3) * (desc->nz + 2);
    const long long nzf = (long long)(desc->nx + 2) * (desc->ny + 2) * (desc->nz + 3);
    if ((st = dalloc(h, &h->ct, nc)) || (st = dalloc(h, &h->fxt, nxf)) || (st = dalloc(h, &h->fyt, nyf)) ||
        (st = dalloc(h, &h->fzt, nzf)))
      return fail(st);
  }
  for (int l = 1; l < h->nlev; ++l) {
    Level& L = h->lv[l];
    const Geom& g = L.g;
    if ((st = palloc(h, g, &L.bx64)) || (st = palloc(h, g, &L.by64)) || (st = palloc(h, g, &L.bz64)) ||
        (st = palloc(h, g, &L.x64)) || (st = palloc(h, g, &L.x64b)) || (st = palloc(h, g, &L.rhs64)) ||
        (st = palloc(h, g, &L.x32)) || (st = palloc(h, g, &L.x32b)) || (st = palloc(h, g, &L.rhs32)))
      return fail(st);
    const bool bf16 = use_bf16(h, o) && l >= h->lc;
    if (bf16) {
      __nv_bfloat16* p;
      if ((st = palloc(h, g, &p))) return fail(st); L.bxm = p;
      if ((st = palloc(h, g, &p))) return fail(st); L.bym = p;
      if ((st = palloc(h, g, &p))) return fail(st); L.bzm = p;
      L.ctm = CT_BF16;
      if ((st = palloc(h, g, &L.bxw)) || (st = palloc(h, g, &L.byw)) || (st = palloc(h, g, &L.bzw))) return fail(st);
    } else {
      float* p;
      if ((st = palloc(h, g, &p))) return fail(st); L.bxm = p;
      if ((st = palloc(h, g, &p))) return fail(st); L.bym = p;
      if ((st = palloc(h, g, &p))) return fail(st); L.bzm = p;
      L.ctm = CT_F32;
    }
  }
  // reductions: the largest reducing launch is a fine-grid cell launch
  {
    long long maxb = 0;
    for (int l = 0; l < h->nlev; ++l) {
      const dim3 gr = grid_cells(h->lv[l].g, kz_for(h->lv[l].g));
      maxb = std::max(maxb, (long long)gr.x * gr.y * gr.z);
      const dim3 gp = grid_planes(h->lv[l].g.nx, h->lv[l].g.ny, h->lv[l].g.nz);
      maxb = std::max(maxb, (long long)gp.x * gp.y * gp.z);
    }
    if ((st = dalloc(h, &h->red.partials, maxb * 4 + 64))) return fail(st);
    h->red_blocks = maxb;
    if ((st = dalloc(h, &h->red.ticket, 64))) return fail(st);
  }
  if ((st = dalloc(h, &h->s, 1))) return fail(st);
  {
    // mapped, so that kernels move the scalars over PCIe without a copy
    // engine: a copy would queue behind bulk copies of other streams
    cudaError_t eh = cudaHostAlloc((void**)&h->hs, sizeof(Scalars), cudaHostAllocMapped);
    if (eh == cudaSuccess) eh = cudaHostGetDevicePointer((void**)&h->hs_dev, h->hs, 0);
    if (eh != cudaSuccess) { set_err("cudaHostAlloc: %s", cudaGetErrorString(eh)); return fail(SMAC_CUDA_ERROR); }
    memset(h->hs, 0, sizeof(Scalars));
  }
  h->num_sms = prop.multiProcessorCount;
  h->l2_bytes = prop.l2CacheSize;
  setup_tma(h);
  setup_zm(h);
  setup_cluster(h, prop.sharedMemPerBlockOptin);
  cudaError_t es = cudaStreamSynchronize(h->stream);
  if (es != cudaSuccess) { set_err("smac_create: %s", cudaGetErrorString(es)); return fail(SMAC_CUDA_ERROR); }
  *out = h;
  return SMAC_OK;
}

smac_status smac_destroy(smac_handle* h) {
  if (!h) return SMAC_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  for (void* p : h->allocs) cudaFree(p);
  if (h->hs) cudaFreeHost(h->hs);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return SMAC_OK;
}

smac_status smac_set_options(smac_handle* h, const smac_options* opts) {
  if (!h || !opts) { set_err("smac_set_options: null argument"); return SMAC_BAD_ARG; }
  TRY(validate_options(opts));
  if (opts->min_coarse != h->opts.min_coarse || opts->max_levels != h->opts.max_levels ||
      opts->bf16_coarse_cells != h->opts.bf16_coarse_cells || is_gmg(*opts) != is_gmg(h->opts)) {
    set_err("smac_set_options: min_coarse, max_levels, bf16_coarse_cells and the GMG/Jacobi choice are fixed at creation");
    return SMAC_BAD_ARG;
  }
  if (opts->nu1 != h->opts.nu1 || opts->nu2 != h->opts.nu2 || opts->coarse_sweeps != h->opts.coarse_sweeps ||
      opts->sweep_kernel != h->opts.sweep_kernel || opts->coarse_kernel != h->opts.coarse_kernel)
    drop_graphs(h);  // the captured iterations launch the old sweeps
  h->opts = *opts;
  return SMAC_OK;
}

smac_status smac_level_shape(const smac_handle* h, int level, int* nx, int* ny, int* nz, int* num_levels) {
  if (!h) { set_err("null handle"); return SMAC_BAD_ARG; }
  if (num_levels) *num_levels = h->nlev;
  if (level < 0 || level >= h->nlev) { set_err("level %d out of range", level); return SMAC_BAD_ARG; }
  if (nx) *nx = h->lv[level].g.nx;
  if (ny) *ny = h->lv[level].g.ny;
  if (nz) *nz = h->lv[level].g.nz;
  return SMAC_OK;
}

smac_status smac_set_coefficients(smac_handle* h, const double* fbx, const double* fby, const double* fbz,
                                  const uint8_t* ct, const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt) {
  if (!h || !fbx || !fby || !fbz || !ct || !fxt || !fyt || !fzt) {
    set_err("smac_set_coefficients: null argument");
    return SMAC_BAD_ARG;
  }
  const Geom& g = h->lv[0].g;
  {
    const RefDims& R = h->R;
    const size_t nc = (size_t)(R.Nx + 2) * (R.Ny + 2) * (R.Nz + 2);
    const size_t nxf = (size_t)(R.Nx + 3) * (R.Ny + 2) * (R.Nz + 2);
    const size_t nyf = (size_t)(R.Nx + 2) * (R.Ny + 3) * (R.Nz + 2);
    const size_t nzf = (size_t)(R.Nx + 2) * (R.Ny + 2) * (R.Nz + 3);
    CK(cudaMemcpyAsync(h->ct, ct, nc, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->fxt, fxt, nxf, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->fyt, fyt, nyf, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->fzt, fzt, nzf, cudaMemcpyDeviceToDevice, h->stream));
  }
  k_import_coeffs<<<grid_planes(g.nx + 1, g.ny + 1, g.nz + 1), kBlock, 0, h->stream>>>(
      g, h->R, fbx, fby, fbz, ct, fxt, fyt, fzt, h->fbx, h->fby, h->fbz, h->lv[0].bx64, h->lv[0].by64,
      h->lv[0].bz64, h->fluid);
  CKL();
  k_fluid_finalize<<<grid_cells(g, kz_for(g)), kBlock, 0, h->stream>>>(g, h->fbx, h->fby, h->fbz, h->fluid, h->red,
                                                                       h->s, kz_for(g));
  CKL();
  // FP32 fine copy for the mixed-precision Krylov operator
  {
    const long long n = g.alloc;
    k_convert<float><<<1184, 256, 0, h->stream>>>(base_of(g, h->lv[0].bx64), base_of(g, (float*)h->lv[0].bxm), n);
    k_convert<float><<<1184, 256, 0, h->stream>>>(base_of(g, h->lv[0].by64), base_of(g, (float*)h->lv[0].bym), n);
    k_convert<float><<<1184, 256, 0, h->stream>>>(base_of(g, h->lv[0].bz64), base_of(g, (float*)h->lv[0].bzm), n);
    CKL();
  }
  for (int l = 1; l < h->nlev; ++l) {
    Level& F = h->lv[l - 1];
    Level& L = h->lv[l];
    const dim3 gr = grid_planes(L.g.nx + 1, L.g.ny + 1, L.g.nz + 1);
    k_coarsen_coeffs<double><<<gr, kBlock, 0, h->stream>>>(F.g, L.g, L.cx, L.cy, L.cz, F.bx64, F.by64, F.bz64, L.bx64,
                                                           L.by64, L.bz64, nullptr, nullptr, nullptr);
    CKL();
    const long long n = L.g.alloc;
    if (L.ctm == CT_BF16) {
      k_convert<__nv_bfloat16><<<256, 256, 0, h->stream>>>(base_of(L.g, L.bx64), base_of(L.g, (__nv_bfloat16*)L.bxm), n);
      k_convert<__nv_bfloat16><<<256, 256, 0, h->stream>>>(base_of(L.g, L.by64), base_of(L.g, (__nv_bfloat16*)L.bym), n);
      k_convert<__nv_bfloat16><<<256, 256, 0, h->stream>>>(base_of(L.g, L.bz64), base_of(L.g, (__nv_bfloat16*)L.bzm), n);
      k_widen_bf16<<<256, 256, 0, h->stream>>>(base_of(L.g, (const __nv_bfloat16*)L.bxm), base_of(L.g, L.bxw), n);
      k_widen_bf16<<<256, 256, 0, h->stream>>>(base_of(L.g, (const __nv_bfloat16*)L.bym), base_of(L.g, L.byw), n);
      k_widen_bf16<<<256, 256, 0, h->stream>>>(base_of(L.g, (const __nv_bfloat16*)L.bzm), base_of(L.g, L.bzw), n);
    } else {
      k_convert<float><<<256, 256, 0, h->stream>>>(base_of(L.g, L.bx64), base_of(L.g, (float*)L.bxm), n);
      k_convert<float><<<256, 256, 0, h->stream>>>(base_of(L.g, L.by64), base_of(L.g, (float*)L.bym), n);
      k_convert<float><<<256, 256, 0, h->stream>>>(base_of(L.g, L.bz64), base_of(L.g, (float*)L.bzm), n);
    }
    CKL();
  }
  TRY(scalars_to_host(h));
  CK(cudaStreamSynchronize(h->stream));
  h->nfluid = h->hs->sum_tmp;
  h->have_coeffs = true;
  return SMAC_OK;
}

smac_status smac_box_types(const smac_grid_desc* d, uint8_t* ct, uint8_t* fxt, uint8_t* fyt, uint8_t* fzt,
                           void* stream) {
  if (!d || !ct || !fxt || !fyt || !fzt) { set_err("smac_box_types: null argument"); return SMAC_BAD_ARG; }
  RefDims R{d->nx, d->ny, d->nz};
  k_box_types<<<grid_planes(d->nx + 3, d->ny + 3, d->nz + 3), kBlock, 0, (cudaStream_t)stream>>>(R, ct, fxt, fyt, fzt);
  CKL();
  return SMAC_OK;
}

smac_status smac_assemble_vof(const smac_grid_desc* d, const double* alpha, double rho0, double rho1, const uint8_t* ct,
                              const uint8_t* fxt, const uint8_t* fyt, const uint8_t* fzt, double* rho, double* fbx,
                              double* fby, double* fbz, double* firx, double* firy, double* firz, void* stream) {
  if (!d || !alpha || !ct || !fxt || !fyt || !fzt || !rho || !fbx || !fby || !fbz) {
    set_err("smac_assemble_vof: null argument");
    return SMAC_BAD_ARG;
  }
  RefDims R{d->nx, d->ny, d->nz};
  cudaStream_t s = (cudaStream_t)stream;
  k_vof_rho<<<grid_planes(d->nx + 1, d->ny + 1, d->nz + 1), kBlock, 0, s>>>(R, alpha, rho0, rho1, ct, rho);
  CKL();
  k_vof_faces<<<grid_planes(d->nx + 2, d->ny + 2, d->nz + 2), kBlock, 0, s>>>(R, rho, fxt, fyt, fzt, fbx, fby, fbz,
                                                                                firx, firy, firz);
  CKL();
  return SMAC_OK;
}

smac_status smac_update_boundary_faces(const smac_grid_desc* d, const uint8_t* fxo, const uint8_t* fyo,
                                       const uint8_t* fzo, double* fbx, double* fby, double* fbz, void* stream) {
  if (!d || !fxo || !fyo || !fzo || !fbx || !fby || !fbz) {
    set_err("smac_update_boundary_faces: null argument");
    return SMAC_BAD_ARG;
  }
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) {
    set_err("smac_update_boundary_faces: bad grid %d x %d x %d", d->nx, d->ny, d->nz);
    return SMAC_BAD_SHAPE;
  }
  RefDims R{d->nx, d->ny, d->nz};
  k_outlet_faces<<<grid_planes(d->nx + 3, d->ny + 3, d->nz + 3), kBlock, 0, (cudaStream_t)stream>>>(R, fxo, fyo, fzo,
                                                                                                    fbx, fby, fbz);
  CKL();
  return SMAC_OK;
}

smac_status smac_ibm_solid_fraction_spheres(const smac_grid_desc* d, const double origin[3], const double* spheres,
                                            int nsph, double* sf, void* stream) {
  if (!d || !origin || (!spheres && nsph > 0) || nsph < 0 || !sf) {
    set_err("smac_ibm_solid_fraction_spheres: bad argument");
    return SMAC_BAD_ARG;
  }
  RefDims R{d->nx, d->ny, d->nz};
  cudaStream_t s = (cudaStream_t)stream;
  double* dsph = nullptr;
  if (nsph > 0) {
    CK(cudaMallocAsync((void**)&dsph, sizeof(double) * 4 * nsph, s));
    CK(cudaMemcpyAsync(dsph, spheres, sizeof(double) * 4 * nsph, cudaMemcpyHostToDevice, s));
  }
  k_ibm_spheres<<<grid_planes(d->nx + 1, d->ny + 1, d->nz + 1), kBlock, 0, s>>>(R, d->dx, d->dy, d->dz, origin[0],
                                                                                  origin[1], origin[2], dsph, nsph, sf);
  CKL();
  if (dsph) CK(cudaFreeAsync(dsph, s));
  CK(cudaStreamSynchronize(s));
  return SMAC_OK;
}

smac_status smac_ibm_set_solid_cells(const smac_grid_desc* d, const double* sf, uint8_t* ct, uint8_t* fxt, uint8_t* fyt,
                                     uint8_t* fzt, void* stream) {
  if (!d || !sf || !ct || !fxt || !fyt || !fzt) { set_err("smac_ibm_set_solid_cells: null argument"); return SMAC_BAD_ARG; }
  RefDims R{d->nx, d->ny, d->nz};
  k_ibm_set_solid<<<grid_planes(d->nx + 1, d->ny + 1, d->nz + 1), kBlock, 0, (cudaStream_t)stream>>>(R, sf, ct, fxt, fyt,
                                                                                                       fzt);
  CKL();
  return SMAC_OK;
}

smac_status smac_divergence(smac_handle* h, const double* vxs, const double* vys, const double* vzs, const double* eps,
                            const double* eps_old, const double* fsx, const double* fsy, const double* fsz, double dt,
                            double* rhs_out) {
  if (!h || !vxs || !vys || !vzs) { set_err("smac_divergence: null argument"); return SMAC_BAD_ARG; }
  if (!h->have_coeffs) { set_err("smac_divergence: call smac_set_coefficients first"); return SMAC_BAD_ARG; }
  if ((eps == nullptr) != (eps_old == nullptr)) { set_err("smac_divergence: eps and eps_old go together"); return SMAC_BAD_ARG; }
  if (!((fsx && fsy && fsz) || (!fsx && !fsy && !fsz))) { set_err("smac_divergence: fsx/fsy/fsz go together"); return SMAC_BAD_ARG; }
  if (!(dt > 0) || !std::isfinite(dt)) { set_err("smac_divergence: dt must be > 0"); return SMAC_BAD_ARG; }
  const Geom& g = h->lv[0].g;
  if (!eps && !fsx) {
    constexpr int KZ = 4;
    k_divergence_z<KZ><<<dim3((g.nx + TBX - 1) / TBX, (g.ny + TBY - 1) / TBY, (g.nz + KZ - 1) / KZ), kBlock, 0,
                         h->stream>>>(g, h->R, 1.0 / h->desc.dx, 1.0 / h->desc.dy, 1.0 / h->desc.dz, 1.0 / dt, vxs,
                                      vys, vzs, h->fluid, h->b64, rhs_out);
  } else {
    k_divergence<<<grid_planes(g.nx, g.ny, g.nz), kBlock, 0, h->stream>>>(
        g, h->R, 1.0 / h->desc.dx, 1.0 / h->desc.dy, 1.0 / h->desc.dz, 1.0 / dt, vxs, vys, vzs, eps, eps_old,
        h->fbx, h->fby, h->fbz, fsx, fsy, fsz, h->fluid, h->b64, rhs_out);
  }
  CKL();
  h->dt = dt;
  h->have_rhs = true;
  return SMAC_OK;
}

smac_status smac_set_rhs(smac_handle* h, const double* rhs) {
  if (!h || !rhs) { set_err("smac_set_rhs: null argument"); return SMAC_BAD_ARG; }
  const Geom& g = h->lv[0].g;
  k_import_cells<double><<<grid_planes(g.nx, g.ny, g.nz), kBlock, 0, h->stream>>>(g, h->R, rhs, h->b64);
  CKL();
  h->have_rhs = true;
  return SMAC_OK;
}

namespace {

// Solve A x = b for the padded b64; leaves the solution (not yet de-meaned)
// in *xout and the scalars on the host mirror.
smac_status run_solve(smac_handle* h, const double** xout) {
  const smac_options& o = h->opts;
  const bool mixed = o.precision == SMAC_PRECISION_MIXED;
  const bool gmg = is_gmg(o);
  const bool pure = is_pure(o);
  const Geom& g = h->lv[0].g;
  const int kz = kz_for(g);
  const size_t bytes = sizeof(double) * (size_t)g.alloc;
  h->alg_bytes = 0.0;
  h->launches = 0;
  // device scalars that the set-up kernel does not write
  Scalars init{};
  init.max_iter = o.max_iter;
  init.stop_rule = o.stop_rule;
  init.tol_max = o.tol / h->dt;
  init.reliable_delta2 = o.reliable_delta * o.reliable_delta;
  init.inv_nfluid = (pure && h->nfluid > 0) ? 1.0 / h->nfluid : 0.0;
  init.mixed = mixed ? 1 : 0;
  *h->hs = init;
  TRY(scalars_to_device(h));
  TRY(zero_async(h, base_of(g, h->x64a), bytes));
  if (mixed) {
    // x64b and e32 need no clearing: a reliable update writes every cell of
    // x64b, and the first x/r update sets e = alpha d (e_reset)
    TRY(zero_async(h, base_of(g, h->d32), sizeof(float) * (size_t)g.alloc));
  } else {
    TRY(zero_async(h, base_of(g, h->d64), bytes));
  }
  const dim3 gr = grid_cells(g, kz);
  k_setup_sum<double><<<gr, kBlock, 0, h->stream>>>(g, h->b64, h->red, h->s, kz);
  if (mixed)
    k_setup_project<float><<<gr, kBlock, 0, h->stream>>>(g, h->b64, h->fluid, h->r32, h->red, h->s, o.tol, kz);
  else
    k_setup_project<double><<<gr, kBlock, 0, h->stream>>>(g, h->b64, h->fluid, h->r64, h->red, h->s, o.tol, kz);
  CKL();
  account(h, g, 8, 1);
  account(h, g, 8 + 8 + (mixed ? 4 : 8) + 1, 1);
  cudaGraphExec_t ex = nullptr;
  TRY(get_graph(h, mixed, gmg, &ex));
  int per_launch = 0;
  const double per_bytes = iteration_bytes(h, mixed, gmg, &per_launch);
  int restarts = 0;
  int launched = 0;
  const int max_launches = o.max_iter + 8;
  for (;;) {
    if (launched > max_launches) {  // the device sets done by max_iter; this is a second bound
      set_err("run_solve: iteration bound exceeded without a device decision");
      return SMAC_NOT_CONVERGED;
    }
    // launch a batch of iterations (one graph = two iterations); kernels after
    // convergence return at once
    int batch = 1;
    for (int q = 0; q < batch; ++q) CK(cudaGraphLaunch(ex, h->stream));
    launched += 2 * batch;
    TRY(scalars_to_host(h));
    CK(cudaStreamSynchronize(h->stream));
    if (h->hs->done) {
      if (h->hs->status == 2 && restarts < 3) {
        // Breakdown (p.Ap or r.z <= 0).  Near the rounding floor of a tight
        // tolerance it means the Krylov space is exhausted, not failure:
        // decide by the FP64 true residual and restart PCG from it.
        const Scalars& hs0 = *h->hs;
        const int it_now = hs0.iter;
        auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
        if (mixed) {
          // fold the FP32 increment into x64 and recompute r (k_reliable
          // decides convergence on the true residual)
          h->hs->done = 0;
          h->hs->status = 0;
          h->hs->do_reliable = 1;
          TRY(scalars_to_device(h));
          launch_reliable(h, g, S, kz);
          CKL();
        } else {
          launch_pdl(k_true_residual, grid_cells(g, kz), kBlock, 0, h->stream, g, h->x64a, h->b64, S, h->r64, 1, h->red,
              h->s, kz);
          CKL();
        }
        account(h, g, 6 * 8, 1);
        TRY(scalars_to_host(h));
        CK(cudaStreamSynchronize(h->stream));
        const Scalars& hs = *h->hs;
        const bool ok = (o.stop_rule == 1) ? (hs.true_rmax < hs.tol_max) : (hs.true_rr <= hs.tol2bb);
        if (ok) {
          h->hs->status = 0;
          h->hs->done = 1;
          break;
        }
        if (it_now >= o.max_iter) {
          h->hs->status = 1;
          break;
        }
        ++restarts;
        if (mixed)
          TRY(zero_async(h, base_of(g, h->d32), sizeof(float) * (size_t)g.alloc));
        else
          TRY(zero_async(h, base_of(g, h->d64), sizeof(double) * (size_t)g.alloc));
        h->hs->done = 0;
        h->hs->first = 1;
        h->hs->status = 0;
        TRY(scalars_to_device(h));
        continue;
      }
      if (!mixed && h->hs->status == 0) {
        // verify the recursive residual with the FP64 true residual
        auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
        launch_pdl(k_true_residual, grid_cells(g, kz), kBlock, 0, h->stream, g, h->x64a, h->b64, S, h->r64, 0, h->red,
            h->s, kz);
        CKL();
        account(h, g, 5 * 8, 1);
        TRY(scalars_to_host(h));
        CK(cudaStreamSynchronize(h->stream));
        const Scalars& hs = *h->hs;
        const bool ok = (o.stop_rule == 1) ? (hs.true_rmax < hs.tol_max) : (hs.true_rr <= hs.tol2bb);
        if (!ok && hs.iter < o.max_iter && restarts < 3) {
          // restart PCG from the true residual
          ++restarts;
          launch_pdl(k_true_residual, grid_cells(g, kz), kBlock, 0, h->stream, g, h->x64a, h->b64, S, h->r64, 1, h->red,
              h->s, kz);
          CKL();
          account(h, g, 6 * 8, 1);
          TRY(zero_async(h, base_of(g, h->d64), bytes));
          TRY(scalars_to_host(h));
          CK(cudaStreamSynchronize(h->stream));
          h->hs->done = 0;
          h->hs->first = 1;
          h->hs->status = 0;
          TRY(scalars_to_device(h));
          continue;
        }
      }
      break;
    }
  }
  // accounting: iterations actually executed (early-exited launches move no data)
  {
    const int it = h->hs->iter;
    h->alg_bytes += per_bytes * it;
    h->launches += per_launch * launched;
    if (mixed) {
      h->alg_bytes += (double)h->hs->reliable_count * (8 + 4 + 3 * 8 + 8 + 8 + 4) * (double)g.cells();
    }
  }
  if (!mixed) {
    *xout = h->x64a;
  } else {
    *xout = h->hs->xbuf ? h->x64b : h->x64a;
  }
  if (h->hs->status != 0) {
    // true residual of the final iterate of a solve that did not converge
    // (a converged solve has just computed it: the FP64 check of the plain
    // form, the last reliable update of the mixed form)
    auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
    launch_pdl(k_true_residual, grid_cells(g, kz), kBlock, 0, h->stream, g, *xout, h->b64, S, h->r64, 0, h->red, h->s,
        kz);
    CKL();
    account(h, g, 5 * 8, 1);
    TRY(scalars_to_host(h));
    CK(cudaStreamSynchronize(h->stream));
  }
  return SMAC_OK;
}

void fill_stats(smac_handle* h, smac_stats* st) {
  if (!st) return;
  const Scalars& hs = *h->hs;
  st->status = hs.status;
  st->iterations = hs.iter;
  st->reliable_updates = hs.reliable_count;
  st->num_levels = is_gmg(h->opts) ? h->nlev : 0;
  st->norm_b = std::sqrt(hs.bb);
  st->rel_residual = hs.bb > 0 ? std::sqrt(hs.true_rr / hs.bb) : 0.0;
  st->max_residual = hs.true_rmax;
  st->alg_bytes = h->alg_bytes;
  st->kernel_launches = h->launches;
}

// x -> reference-layout p_delta, zero-mean over fluid cells for pure Neumann.
smac_status export_solution(smac_handle* h, const double* x, double* p_delta) {
  const Geom& g = h->lv[0].g;
  const dim3 gp = grid_planes(g.nx, g.ny, g.nz);
  const bool pure = is_pure(h->opts);
  if (pure) {
    k_sum_fluid<<<grid_cells(g, kz_for(g)), kBlock, 0, h->stream>>>(g, x, h->fluid, h->red, h->s, kz_for(g));
    CKL();
  }
  constexpr int KZ = 4;
  k_export_cells_z<KZ><<<dim3(gp.x, gp.y, (g.nz + KZ - 1) / KZ), kBlock, 0, h->stream>>>(
      g, h->R, x, h->fluid, pure ? &h->s->sum_tmp : nullptr, p_delta);
  CKL();
  account(h, g, pure ? 8 + 1 + 8 + 1 + 8 : 16, pure ? 2 : 1);
  return SMAC_OK;
}

}  // namespace

smac_status smac_solve(smac_handle* h, double* p_delta, smac_stats* stats) {
  if (!h || !p_delta) { set_err("smac_solve: null argument"); return SMAC_BAD_ARG; }
  if (!h->have_coeffs || !h->have_rhs) { set_err("smac_solve: coefficients and rhs are required first"); return SMAC_BAD_ARG; }
  const double* x = nullptr;
  TRY(run_solve(h, &x));
  TRY(export_solution(h, x, p_delta));
  if (stats) {
    TRY(scalars_to_host(h));
    CK(cudaStreamSynchronize(h->stream));
    fill_stats(h, stats);
  }
  const int status = h->hs->status;
  if (status != 0) {
    set_err("smac_solve: %s after %d iterations (relative residual %.3e)",
            status == 1 ? "not converged" : status == 2 ? "breakdown" : "non-finite value", h->hs->iter,
            h->hs->bb > 0 ? std::sqrt(h->hs->true_rr / h->hs->bb) : 0.0);
  }
  return (smac_status)status;
}

smac_status smac_correct(smac_handle* h, double* p_delta, double* p, const double* vxs, const double* vys,
                         const double* vzs, const double* firx, const double* firy, const double* firz,
                         const double* fsx, const double* fsy, const double* fsz, double dt, double* vx, double* vy,
                         double* vz, int zero_p_delta) {
  if (!h || !p_delta || !vxs || !vys || !vzs || !vx || !vy || !vz) { set_err("smac_correct: null argument"); return SMAC_BAD_ARG; }
  if (!h->have_coeffs) { set_err("smac_correct: coefficients required"); return SMAC_BAD_ARG; }
  if (!((firx && firy && firz) || (!firx && !firy && !firz))) { set_err("smac_correct: fir* go together"); return SMAC_BAD_ARG; }
  if (!((fsx && fsy && fsz) || (!fsx && !fsy && !fsz))) { set_err("smac_correct: fs* go together"); return SMAC_BAD_ARG; }
  const Geom& g = h->lv[0].g;
  const RefDims& R = h->R;
  k_correct<<<grid_planes(R.Nx + 3, R.Ny + 3, R.Nz + 3), kBlock, 0, h->stream>>>(
      R, g, 1.0 / h->desc.dx, 1.0 / h->desc.dy, 1.0 / h->desc.dz, dt, h->ct, h->fxt, h->fyt, h->fzt, p_delta, p, vxs,
      vys, vzs, firx, firy, firz, h->fbx, h->fby, h->fbz, fsx, fsy, fsz, vx, vy, vz, 0);
  CKL();
  account(h, g, 3 * 8 + 8 + 3 * 8 + 3 * 8 + 3, 1);
  if (zero_p_delta) {
    const long long n = (long long)(R.Nx + 2) * (R.Ny + 2) * (R.Nz + 2);
    CK(cudaMemsetAsync(p_delta, 0, sizeof(double) * (size_t)n, h->stream));
  }
  return SMAC_OK;
}


smac_status smac_project(smac_handle* h, const double* vxs, const double* vys, const double* vzs, double dt,
                         double* p_delta, double* vx, double* vy, double* vz, smac_stats* stats) {
  if (!h || !vxs || !vys || !vzs || !p_delta || !vx || !vy || !vz) { set_err("smac_project: null argument"); return SMAC_BAD_ARG; }
  TRY(smac_divergence(h, vxs, vys, vzs, nullptr, nullptr, nullptr, nullptr, nullptr, dt, nullptr));
  const double* x = nullptr;
  TRY(run_solve(h, &x));
  TRY(export_solution(h, x, p_delta));
  const Geom& g = h->lv[0].g;
  const RefDims& R = h->R;
  k_correct_project<<<grid_planes(R.Nx + 3, R.Ny + 3, R.Nz + 3), kBlock, 0, h->stream>>>(
      R, g, 1.0 / h->desc.dx, 1.0 / h->desc.dy, 1.0 / h->desc.dz, dt, h->fxt, h->fyt, h->fzt, p_delta, vxs, vys, vzs,
      h->fbx, h->fby, h->fbz, vx, vy, vz);
  CKL();
  account(h, g, 3 * 8 + 8 + 3 * 8 + 3 * 8 + 3, 1);
  if (stats) {
    CK(cudaStreamSynchronize(h->stream));
    fill_stats(h, stats);
  }
  const int status = h->hs->status;
  if (status != 0) set_err("smac_project: solve status %d after %d iterations", status, h->hs->iter);
  return (smac_status)status;
}

smac_status smac_project_adjoint(smac_handle* h, const double* gvx, const double* gvy, const double* gvz, double* gvxs,
                                 double* gvys, double* gvzs, double* phi, smac_stats* stats) {
  if (!h || !gvx || !gvy || !gvz || !gvxs || !gvys || !gvzs) { set_err("smac_project_adjoint: null argument"); return SMAC_BAD_ARG; }
  if (!h->have_coeffs) { set_err("smac_project_adjoint: coefficients required"); return SMAC_BAD_ARG; }
  const Geom& g = h->lv[0].g;
  const RefDims& R = h->R;
  k_adj_divergence<<<grid_planes(g.nx, g.ny, g.nz), kBlock, 0, h->stream>>>(
      g, R, 1.0 / h->desc.dx, 1.0 / h->desc.dy, 1.0 / h->desc.dz, gvx, gvy, gvz, h->fbx, h->fby, h->fbz,
      h->fluid, h->b64);
  CKL();
  h->have_rhs = true;
  const double* x = nullptr;
  TRY(run_solve(h, &x));
  account(h, g, 3 * 8 + 3 * 8 + 1 + 8, 1);
  const dim3 gp = grid_planes(g.nx, g.ny, g.nz);
  k_sum_fluid<<<grid_cells(g, kz_for(g)), kBlock, 0, h->stream>>>(g, x, h->fluid, h->red, h->s, kz_for(g));
  CKL();
  if (!is_pure(h->opts)) {
    // no null space: psi is the solution itself
    CK(cudaMemsetAsync(&h->s->sum_tmp, 0, sizeof(double), h->stream));
  }
  k_adj_gradient<<<grid_planes(R.Nx + 3, R.Ny + 3, R.Nz + 3), kBlock, 0, h->stream>>>(
      g, R, 1.0 / h->desc.dx, 1.0 / h->desc.dy, 1.0 / h->desc.dz, x, h->fluid, &h->s->sum_tmp, gvx, gvy, gvz, gvxs,
      gvys, gvzs);
  CKL();
  account(h, g, 8 + 1 + 6 * 8, 2);
  if (phi) {
    k_export_cells<<<gp, kBlock, 0, h->stream>>>(g, R, x, h->fluid, is_pure(h->opts) ? &h->s->sum_tmp : nullptr, phi);
    CKL();
  }
  if (stats) {
    CK(cudaStreamSynchronize(h->stream));
    fill_stats(h, stats);
  }
  const int status = h->hs->status;
  if (status != 0) set_err("smac_project_adjoint: solve status %d after %d iterations", status, h->hs->iter);
  return (smac_status)status;
}

smac_status smac_apply_A(smac_handle* h, const double* x, double* y) {
  if (!h || !x || !y) { set_err("smac_apply_A: null argument"); return SMAC_BAD_ARG; }
  if (!h->have_coeffs) { set_err("smac_apply_A: coefficients required"); return SMAC_BAD_ARG; }
  const Geom& g = h->lv[0].g;
  const dim3 gp = grid_planes(g.nx, g.ny, g.nz);
  k_import_cells<double><<<gp, kBlock, 0, h->stream>>>(g, h->R, x, h->tmp64);
  auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
  k_apply<<<gp, kBlock, 0, h->stream>>>(g, h->tmp64, S, h->q64);
  k_export_cells<<<gp, kBlock, 0, h->stream>>>(g, h->R, h->q64, h->fluid, nullptr, y);
  CKL();
  return SMAC_OK;
}

smac_status smac_time_kernel(smac_handle* h, int kernel_id, int reps, float* ms, double* bytes) {
  if (!h || !ms || !bytes || reps < 1) { set_err("smac_time_kernel: bad argument"); return SMAC_BAD_ARG; }
  if (!h->have_coeffs) { set_err("smac_time_kernel: coefficients required"); return SMAC_BAD_ARG; }
  const Geom& g = h->lv[0].g;
  const int kz = kz_for(g);
  // a state in which no kernel early-exits and the updates are no-ops
  Scalars st{};
  st.max_iter = 1 << 30;
  st.inv_nfluid = 0.0;
  st.rz = 1.0;
  st.alpha = 0.0;
  st.beta = 0.0;
  st.tol2bb = -1.0;
  st.tol_max = -1.0;
  *h->hs = st;
  TRY(scalars_to_device(h));
  // non-zero operands: d = z = b (FP64), d32 = r32 = z32 = b, so that p.Ap > 0
  CK(cudaMemcpyAsync(base_of(g, h->d64), base_of(g, h->b64), sizeof(double) * (size_t)g.alloc, cudaMemcpyDeviceToDevice,
                     h->stream));
  CK(cudaMemcpyAsync(base_of(g, h->z64), base_of(g, h->b64), sizeof(double) * (size_t)g.alloc, cudaMemcpyDeviceToDevice,
                     h->stream));
  k_convert<float><<<1184, 256, 0, h->stream>>>(base_of(g, h->b64), base_of(g, h->d32), g.alloc);
  k_convert<float><<<1184, 256, 0, h->stream>>>(base_of(g, h->b64), base_of(g, h->r32), g.alloc);
  k_convert<float><<<1184, 256, 0, h->stream>>>(base_of(g, h->b64), base_of(g, h->z32), g.alloc);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double per = 0.0;
  auto launch = [&]() -> smac_status {
    switch (kernel_id) {
      case 0: {
        auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
        launch_pdl(k_matvec_pap<double, double>, grid_cells(g, kz), kBlock, 0, h->stream, g, h->d64, S, h->q64, h->red,
            h->s, kz);
        per = 5 * 8.0;
        break;
      }
      case 1: {
        auto S = stencil<float, float>(g, h->lv[0].bxm, h->lv[0].bym, h->lv[0].bzm);
        launch_pdl(k_matvec_pap<float, float>, grid_cells(g, kz), kBlock, 0, h->stream, g, h->d32, S, h->q32, h->red,
            h->s, kz);
        per = 5 * 4.0;
        break;
      }
      case 2: {
        launch_sweep<double, double>(h, 0, 0, false, h->z64, h->z64b, h->r64, nullptr, h->lv[0].bx64, h->lv[0].by64,
                                     h->lv[0].bz64, 0, nullptr);
        per = 6 * 8.0;
        break;
      }
      case 3: {
        launch_sweep<float, float>(h, 0, 0, false, h->z32, h->z32b, h->r32, nullptr, h->lv[0].bxm, h->lv[0].bym,
                                   h->lv[0].bzm, 0, nullptr);
        per = 6 * 4.0;
        break;
      }
      case 5: {
        auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
        k_rbgs<double, double><<<grid_pairs(g, kz), kBlock, 0, h->stream>>>(g, h->z64, h->r64, nullptr, S, 0, 0, nullptr, g, 0, 0, 0, h->s, kz);
        k_rbgs<double, double><<<grid_pairs(g, kz), kBlock, 0, h->stream>>>(g, h->z64, h->r64, nullptr, S, 1, 0, nullptr, g, 0, 0, 0, h->s, kz);
        per = 6 * 8.0;
        break;
      }
      case 6: {
        auto S = stencil<float, float>(g, h->lv[0].bxm, h->lv[0].bym, h->lv[0].bzm);
        k_rbgs<float, float><<<grid_pairs(g, kz), kBlock, 0, h->stream>>>(g, h->z32, h->r32, nullptr, S, 0, 0, nullptr, g, 0, 0, 0, h->s, kz);
        k_rbgs<float, float><<<grid_pairs(g, kz), kBlock, 0, h->stream>>>(g, h->z32, h->r32, nullptr, S, 1, 0, nullptr, g, 0, 0, 0, h->s, kz);
        per = 6 * 4.0;
        break;
      }
      case 7: {
        auto S = stencil<float, float>(g, h->lv[0].bxm, h->lv[0].bym, h->lv[0].bzm);
        launch_dir_matvec<float>(h, g, h->z32, h->d32, h->d32b, S, h->q32, kz);
        per = 7 * 4.0;
        break;
      }
      case 8: {
        auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
        launch_dir_matvec<double>(h, g, h->z64, h->d64, h->d64b, S, h->q64, kz);
        per = 7 * 8.0;
        break;
      }
      case 9: {
        launch_update<float>(h, g, h->e32, h->d32, h->r32, h->q32);
        per = 6 * 4.0;
        break;
      }
      case 10: {
        launch_update<double>(h, g, h->tmp64, h->d64, h->r64, h->q64);
        per = 6 * 8.0;
        break;
      }
      case 11: case 12: case 13: {  // FP32 sweep from zero / with the prolongation / with r.z
        const int mode = kernel_id == 11 ? 1 : kernel_id == 12 ? 2 : 0;
        launch_sweep<float, float>(h, 0, mode, kernel_id == 13, mode == 1 ? nullptr : h->z32, h->z32b, h->r32, nullptr,
                                   h->lv[0].bxm, h->lv[0].bym, h->lv[0].bzm, mode == 2 ? 1 : 0,
                                   mode == 2 ? h->lv[1].x32 : nullptr);
        per = (mode == 1 ? 5 : 6) * 4.0 + (mode == 2 ? 4.0 / 8 : 0.0);
        break;
      }
      case 14: case 15: case 16: {  // FP64 sweep from zero / with the prolongation / with r.z
        const int mode = kernel_id == 14 ? 1 : kernel_id == 15 ? 2 : 0;
        launch_sweep<double, double>(h, 0, mode, kernel_id == 16, mode == 1 ? nullptr : h->z64, h->z64b, h->r64,
                                     nullptr, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64, mode == 2 ? 1 : 0,
                                     mode == 2 ? h->lv[1].x64 : nullptr);
        per = (mode == 1 ? 5 : 6) * 8.0 + (mode == 2 ? 8.0 / 8 : 0.0);
        break;
      }
      case 4: {
        auto S = stencil<double, double>(g, h->lv[0].bx64, h->lv[0].by64, h->lv[0].bz64);
        launch_pdl(k_true_residual, grid_cells(g, kz), kBlock, 0, h->stream, g, h->x64a, h->b64, S, h->r64, 0, h->red,
            h->s, kz);
        per = 5 * 8.0;
        break;
      }
      default:
        set_err("smac_time_kernel: unknown kernel id %d", kernel_id);
        return SMAC_BAD_ARG;
    }
    CKL();
    return SMAC_OK;
  };
  TRY(launch());  // warm-up
  CK(cudaEventRecord(e0, h->stream));
  for (int q = 0; q < reps; ++q) TRY(launch());
  CK(cudaEventRecord(e1, h->stream));
  CK(cudaEventSynchronize(e1));
  float tot = 0.f;
  CK(cudaEventElapsedTime(&tot, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = tot / reps;
  *bytes = per * (double)g.cells();
  return SMAC_OK;
}


}  // extern "C"

namespace {
template <class T, class C>
smac_status sweep_selftest(smac_handle* h, int mode, T* x, T* xa, T* xb, T* rhs, const void* bx, const void* by,
                           const void* bz, const T* xc, long long* mismatches) {
  const Geom& g = h->lv[0].g;
  const int kz = kz_for(g);
  const Level& Lc = h->lv[1];
  const int c0 = (mode == 2) ? 1 : 0;
  // reference: two in-place half-sweeps on a copy of x
  CK(cudaMemcpyAsync(base_of(g, xa), base_of(g, x), sizeof(T) * (size_t)g.alloc, cudaMemcpyDeviceToDevice, h->stream));
  auto S = stencil<T, C>(g, bx, by, bz);
  k_rbgs<T, C><<<grid_pairs(g, kz), kBlock, 0, h->stream>>>(g, xa, rhs, &h->s->rshift, S, c0, mode == 1,
                                                            mode == 2 ? xc : (const T*)nullptr, Lc.g, Lc.cx, Lc.cy,
                                                            Lc.cz, nullptr, kz);
  k_rbgs<T, C><<<grid_pairs(g, kz), kBlock, 0, h->stream>>>(g, xa, rhs, &h->s->rshift, S, 1 - c0, 0, (const T*)nullptr,
                                                            g, 0, 0, 0, nullptr, kz);
  CKL();
  // fused sweep, out of place
  launch_sweep<T, C>(h, 0, mode, false, x, xb, rhs, &h->s->rshift, bx, by, bz, c0, xc);
  CKL();
  unsigned long long* cnt = nullptr;
  CK(cudaMallocAsync((void**)&cnt, sizeof(unsigned long long), h->stream));
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), h->stream));
  k_count_mismatch<T><<<grid_planes(g.nx, g.ny, g.nz), kBlock, 0, h->stream>>>(g, xa, xb, cnt);
  CKL();
  unsigned long long hc = 0;
  CK(cudaMemcpyAsync(&hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaFreeAsync(cnt, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *mismatches = (long long)hc;
  return SMAC_OK;
}
}  // namespace

extern "C" {

smac_status smac_selftest_wait(smac_handle* h, int* status, long long* cycles) {
  if (!h || !status || !cycles) { set_err("smac_selftest_wait: null argument"); return SMAC_BAD_ARG; }
  long long* dcyc = nullptr;
  CK(cudaMalloc(&dcyc, sizeof(long long)));
  h->hs->status = 0;
  TRY(scalars_to_device(h));
  k_wait_probe<<<1, 32, 0, h->stream>>>(h->s, dcyc);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(cycles, dcyc, sizeof(long long), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dcyc);
  if (e != cudaSuccess) { set_err("smac_selftest_wait: %s", cudaGetErrorString(e)); return SMAC_CUDA_ERROR; }
  TRY(scalars_to_host(h));
  CK(cudaStreamSynchronize(h->stream));
  *status = h->hs->status;
  h->hs->status = 0;  // the handle stays usable
  TRY(scalars_to_device(h));
  CK(cudaStreamSynchronize(h->stream));
  return SMAC_OK;
}

smac_status smac_selftest_sweep(smac_handle* h, int precision, int mode, long long* mismatches) {
  if (!h || !mismatches || mode < 0 || mode > 2 || precision < 0 || precision > 1) {
    set_err("smac_selftest_sweep: bad argument");
    return SMAC_BAD_ARG;
  }
  if (!h->have_coeffs || h->nlev < 2) { set_err("smac_selftest_sweep: needs coefficients and >= 2 grids"); return SMAC_BAD_ARG; }
  // the V-cycle's shift must be finite; a state with shift 0 is used
  Scalars st{};
  *h->hs = st;
  TRY(scalars_to_device(h));
  if (precision == SMAC_PRECISION_FP64)
    return sweep_selftest<double, double>(h, mode, h->z64, h->tmp64, h->z64b, h->r64, h->lv[0].bx64, h->lv[0].by64,
                                          h->lv[0].bz64, h->lv[1].x64, mismatches);
  return sweep_selftest<float, float>(h, mode, h->z32, h->q32, h->z32b, h->r32, h->lv[0].bxm, h->lv[0].bym,
                                      h->lv[0].bzm, h->lv[1].x32, mismatches);
}

}  // extern "C"
