// smac_noalloc.cu -- y = A x and x.Ax without allocating device memory.
//
// Some callers cannot allocate: a time-step loop that is being recorded into a
// CUDA graph may not call cudaMalloc while its stream is capturing, and a host
// code that hands all device memory to its own pool allocator leaves
// cudaMalloc nothing to give.  smac_apply_A_dot_noalloc serves them: it needs
// no handle, reads the reference-layout coefficients, types and x directly,
// and keeps the only scratch it needs (the per-block partial sums of x.Ax and
// the arrival counter of the final reduction) in the file-scope device array
// below, which every GPU that loads this library holds until the process
// exits.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "smac_b200.h"
#include "smac_common.cuh"

#include <cudaTypedefs.h>

using namespace smac;

namespace smac {
void set_error_text(const char* fmt, ...);  // smac_last_error_string() reports it (smac_api.cu)
}

namespace {

constexpr int NA_BX = 32, NA_BY = 4, NA_NT = NA_BX * NA_BY;

// Largest number of thread blocks one call may use; each block owns one
// partial sum.  A call covers its grid with ceil(nx/32) x ceil(ny/4) blocks per
// z-chunk and at least one z-chunk, so x-y planes up to 1024 x 1024 cells fit.
constexpr int NA_MAX_BLOCKS = 8192;

struct NoAllocScratch {
  double partials[NA_MAX_BLOCKS];  // one partial sum per block
  unsigned int ticket[32];         // arrival counter of the last-block reduction (slot 0)
};

// The scratch itself (64 KB + 128 B per device).
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch, per device ordinal.  In host code the
// symbol is a host-side stand-in, not a device address, so it is looked up
// once per device with cudaGetSymbolAddress while that device is current.
// The address belongs to the device's current context: it is looked up again
// when that context has changed (after cudaDeviceReset, for instance, the
// module and its array are loaded anew).
constexpr int NA_MAX_DEVICES = 128;
std::mutex g_na_mutex;
NoAllocScratch* g_na_addr[NA_MAX_DEVICES] = {};
CUcontext g_na_ctx[NA_MAX_DEVICES] = {};
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;

// The calling thread's current context (the driver's cuCtxGetCurrent, reached
// through the runtime's entry-point query so the library needs no libcuda link).
bool current_context(CUcontext* ctx) {
  if (!g_ctx_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
  }
  return g_ctx_current(ctx) == CUDA_SUCCESS;
}

// Coefficient of the face between cells a (low) and b (high), reference
// layout indices: the same masking as smac_set_coefficients.
__device__ __forceinline__ double face_coef(double fb, int a_in, int b_in, uint8_t ftype) {
  if (a_in == 0 || b_in == 0) return 0.0;                       // next to a non-C_INTERIOR cell
  if (a_in == 1 && b_in == 1 && ftype != F_INTERIOR) return 0.0;  // inside the domain, not F_INTERIOR
  return fb;
}

__global__ void __launch_bounds__(NA_NT)
    k_apply_dot_noalloc(RefDims R, double ihx2, double ihy2, double ihz2, const double* __restrict__ fbx,
                        const double* __restrict__ fby, const double* __restrict__ fbz, const uint8_t* __restrict__ ct,
                        const uint8_t* __restrict__ fxt, const uint8_t* __restrict__ fyt,
                        const uint8_t* __restrict__ fzt, const double* __restrict__ x, double* y, double* xAx,
                        NoAllocScratch* scratch, int kz) {
  const int nx = R.Nx, ny = R.Ny, nz = R.Nz;
  const int i = blockIdx.x * NA_BX + threadIdx.x;
  const int j = blockIdx.y * NA_BY + threadIdx.y;
  const int k0 = blockIdx.z * kz;
  // 1 C_INTERIOR cell, 0 other cell, -1 outside the domain (interior indices)
  auto cin = [&](int ii, int jj, int kk) -> int {
    if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) return -1;
    return ct[R.cell(ii + 1, jj + 1, kk + 1)] == C_INTERIOR ? 1 : 0;
  };
  // x at an interior cell, 0 outside the domain (the zero ghost)
  auto X = [&](int ii, int jj, int kk) -> double {
    if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) return 0.0;
    return x[R.cell(ii + 1, jj + 1, kk + 1)];
  };
  typedef Ar<double> Rd;
  double v[1] = {0.0};
  if (i < nx && j < ny) {
    const int k1 = min(k0 + kz, nz);
    for (int k = k0; k < k1; ++k) {
      const int ix = i + 1, iy = j + 1, iz = k + 1;
      const int me = cin(i, j, k);
      const double wxm = Rd::mul(face_coef(fbx[R.xf(ix, iy, iz)], cin(i - 1, j, k), me, fxt[R.xf(ix, iy, iz)]), ihx2);
      const double wxp = Rd::mul(face_coef(fbx[R.xf(ix + 1, iy, iz)], me, cin(i + 1, j, k), fxt[R.xf(ix + 1, iy, iz)]), ihx2);
      const double wym = Rd::mul(face_coef(fby[R.yf(ix, iy, iz)], cin(i, j - 1, k), me, fyt[R.yf(ix, iy, iz)]), ihy2);
      const double wyp = Rd::mul(face_coef(fby[R.yf(ix, iy + 1, iz)], me, cin(i, j + 1, k), fyt[R.yf(ix, iy + 1, iz)]), ihy2);
      const double wzm = Rd::mul(face_coef(fbz[R.zf(ix, iy, iz)], cin(i, j, k - 1), me, fzt[R.zf(ix, iy, iz)]), ihz2);
      const double wzp = Rd::mul(face_coef(fbz[R.zf(ix, iy, iz + 1)], me, cin(i, j, k + 1), fzt[R.zf(ix, iy, iz + 1)]), ihz2);
      const double xc = X(i, j, k);
      const double yv = Stencil<double, double>::apply(xc, wxm, wxp, wym, wyp, wzm, wzp, X(i - 1, j, k), X(i + 1, j, k),
                                                       X(i, j - 1, k), X(i, j + 1, k), X(i, j, k - 1), X(i, j, k + 1));
      y[R.cell(ix, iy, iz)] = yv;
      v[0] += xc * yv;
    }
  }
  const Op ops[1] = {Op::Sum};
  double out[1];
  RedBuf red{scratch->partials, scratch->ticket};
  if (grid_reduce<1, NA_NT>(v, ops, red, 0, out)) {
    if (threadIdx.x == 0 && threadIdx.y == 0) *xAx = out[0];
  }
}

}  // namespace

extern "C" smac_status smac_apply_A_dot_noalloc(const smac_grid_desc* d, const double* fbx, const double* fby,
                                                const double* fbz, const uint8_t* celltype, const uint8_t* fxt,
                                                const uint8_t* fyt, const uint8_t* fzt, const double* x, double* y,
                                                double* xAx, void* cuda_stream) {
  if (!d || !fbx || !fby || !fbz || !celltype || !fxt || !fyt || !fzt || !x || !y || !xAx) {
    smac::set_error_text("smac_apply_A_dot_noalloc: null argument");
    return SMAC_BAD_ARG;
  }
  if (d->nx < 1 || d->ny < 1 || d->nz < 1 || !(d->dx > 0) || !(d->dy > 0) || !(d->dz > 0)) {
    smac::set_error_text("smac_apply_A_dot_noalloc: bad grid %dx%dx%d", d->nx, d->ny, d->nz);
    return SMAC_BAD_SHAPE;
  }
  const long long bxy = (long long)((d->nx + NA_BX - 1) / NA_BX) * ((d->ny + NA_BY - 1) / NA_BY);
  if (bxy > NA_MAX_BLOCKS) {
    smac::set_error_text("smac_apply_A_dot_noalloc: a %dx%d x-y plane needs %lld blocks; the static scratch holds %d "
             "(ceil(nx/32)*ceil(ny/4) must be <= %d)", d->nx, d->ny, bxy, NA_MAX_BLOCKS, NA_MAX_BLOCKS);
    return SMAC_BAD_SHAPE;
  }
  // z-chunk: as many chunks as the scratch allows, at most one per plane
  const int zmax = (int)(NA_MAX_BLOCKS / bxy);
  const int nzc = std::min(d->nz, std::max(1, std::min(zmax, (d->nz + 15) / 16)));
  const int kz = (d->nz + nzc - 1) / nzc;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) {
    smac::set_error_text("smac_apply_A_dot_noalloc: no usable device (%s)", cudaGetErrorString(e));
    return SMAC_NO_DEVICE;
  }
  NoAllocScratch* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    CUcontext ctx = nullptr;
    // cudaGetDevice does not create the context; the first runtime call that
    // needs it does, so a missing context just means "look the address up"
    const bool have_ctx = current_context(&ctx) && ctx != nullptr;
    if (!g_na_addr[dev] || !have_ctx || ctx != g_na_ctx[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        smac::set_error_text("smac_apply_A_dot_noalloc: cudaGetSymbolAddress: %s",
                 cudaGetErrorString(e));
        return SMAC_CUDA_ERROR;
      }
      g_na_addr[dev] = (NoAllocScratch*)p;
      CUcontext now = nullptr;
      g_na_ctx[dev] = current_context(&now) ? now : nullptr;
    }
    scratch = g_na_addr[dev];
  }
  cudaStream_t s = (cudaStream_t)cuda_stream;
  // the arrival counter must start at zero (the previous call's last block
  // reset it, but a call that failed mid-way may not have)
  e = cudaMemsetAsync(scratch->ticket, 0, sizeof(scratch->ticket), s);
  if (e != cudaSuccess) {
    smac::set_error_text("smac_apply_A_dot_noalloc: %s", cudaGetErrorString(e));
    return SMAC_CUDA_ERROR;
  }
  RefDims R{d->nx, d->ny, d->nz};
  const dim3 grid((d->nx + NA_BX - 1) / NA_BX, (d->ny + NA_BY - 1) / NA_BY, (d->nz + kz - 1) / kz);
  k_apply_dot_noalloc<<<grid, dim3(NA_BX, NA_BY, 1), 0, s>>>(R, 1.0 / (d->dx * d->dx), 1.0 / (d->dy * d->dy),
                                                            1.0 / (d->dz * d->dz), fbx, fby, fbz, celltype, fxt, fyt,
                                                            fzt, x, y, xAx, scratch, kz);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    smac::set_error_text("smac_apply_A_dot_noalloc: launch: %s", cudaGetErrorString(e));
    return SMAC_CUDA_ERROR;
  }
  return SMAC_OK;
}
