// smac_vti.cu -- VTK ImageData (.vti) output of the cell fields: the
// reference's FileInOut::output_vti_binary_cellData (CFD/FileInOut.cpp:
// 144-262), file for file the same bytes.
//
// The reference copies every grid member to the host (gpuTocpu,
// CFD/G_SMACSolver.cu:1524-1535; some 60 arrays) and then converts four of
// them to Float32 in host loops.  Here one kernel builds the file's
// appended-data block in device memory, converted and in file order:
//
//   UInt32 bytes | Float32 p[n] | UInt32 | Float32 alpha[n] | UInt32 |
//   Float32 (ux,uy,uz)[n] | UInt32 | Float32 ibm_solid_fraction[n]
//
// with n = Nx Ny Nz interior cells, x fastest, u the mean of the cell's two
// faces in FP64 rounded to Float32.  So 24 bytes per cell cross to the host
// in one copy, and the host only writes the XML text around the block.  The
// caller owns both buffers; the copy and the file write can overlap the next
// time step (mydemcfd_b200.vti.VtiWriter does that).
#include <cstdint>
#include <cstdio>

#include <cuda_runtime.h>

#include "smac_b200.h"

namespace smac {
void set_error_text(const char* fmt, ...);
}

namespace {

constexpr int VTI_TX = 32, VTI_TY = 8;

// One thread per cell (x, y) of plane z.  The block is addressed in 4-byte
// units: header h_k at unit u_k, the k-th array right after it.
__global__ void __launch_bounds__(VTI_TX* VTI_TY)
    k_vti_pack(int nx, int ny, int nz, const double* __restrict__ p, const double* __restrict__ alpha,
               const double* __restrict__ vx, const double* __restrict__ vy, const double* __restrict__ vz,
               const double* __restrict__ sf, uint32_t* __restrict__ block) {
  const long long n = (long long)nx * ny * nz;
  const int x = blockIdx.x * VTI_TX + threadIdx.x + 1, y = blockIdx.y * VTI_TY + threadIdx.y + 1,
            z = blockIdx.z + 1;
  float* f = reinterpret_cast<float*>(block);
  if (x == 1 && y == 1 && z == 1) {
    block[0] = (uint32_t)(4 * n);
    block[n + 1] = (uint32_t)(4 * n);
    block[2 * n + 2] = (uint32_t)(12 * n);
    block[5 * n + 3] = (uint32_t)(4 * n);
  }
  if (x > nx || y > ny) return;
  const long long sx = nx + 2, sxy = sx * (ny + 2);
  const long long c = (long long)z * sxy + (long long)y * sx + x;
  const long long i = ((long long)(z - 1) * ny + (y - 1)) * nx + (x - 1);  // the cell's place in file order
  f[1 + i] = __double2float_rn(p[c]);
  f[n + 2 + i] = alpha ? __double2float_rn(alpha[c]) : 0.0f;
  // faces: x-faces (Nx+3) per row, y-faces (Ny+3) rows per plane
  const long long fx = (long long)z * (ny + 2) * (nx + 3) + (long long)y * (nx + 3) + x;
  const long long fy = (long long)z * (ny + 3) * sx + (long long)y * sx + x;
  const long long fz = c;
  const double ux = __dmul_rn(0.5, __dadd_rn(vx[fx], vx[fx + 1]));
  const double uy = __dmul_rn(0.5, __dadd_rn(vy[fy], vy[fy + sx]));
  const double uz = __dmul_rn(0.5, __dadd_rn(vz[fz], vz[fz + sxy]));
  float* fv = f + 2 * n + 3 + 3 * i;
  fv[0] = __double2float_rn(ux);
  fv[1] = __double2float_rn(uy);
  fv[2] = __double2float_rn(uz);
  f[5 * n + 4 + i] = sf ? __double2float_rn(sf[c]) : 0.0f;
}

bool vti_shape_ok(const smac_grid_desc* d, const char* fn) {
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) {
    smac::set_error_text("%s: grid %d x %d x %d", fn, d->nx, d->ny, d->nz);
    return false;
  }
  // each block's byte count is a UInt32 in the file (header_type="UInt32")
  const long long n = (long long)d->nx * d->ny * d->nz;
  if (12 * n > 0xffffffffLL) {
    smac::set_error_text("%s: %lld cells: the velocity block exceeds the UInt32 size field", fn, n);
    return false;
  }
  return true;
}

}  // namespace

extern "C" {

size_t smac_vti_block_bytes(const smac_grid_desc* d) {
  if (!d || d->nx < 1 || d->ny < 1 || d->nz < 1) return 0;
  const size_t n = (size_t)d->nx * d->ny * d->nz;
  return 16 + 24 * n;
}

smac_status smac_vti_pack(const smac_grid_desc* d, const double* p, const double* alpha, const double* vx,
                          const double* vy, const double* vz, const double* ibm_sf, void* block, void* stream) {
  static const char* fn = "smac_vti_pack";
  if (!d || !p || !vx || !vy || !vz || !block) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (!vti_shape_ok(d, fn)) return SMAC_BAD_SHAPE;
  if (reinterpret_cast<uintptr_t>(block) & 3u) {
    smac::set_error_text("%s: the block must be 4-byte aligned", fn);
    return SMAC_BAD_ARG;
  }
  const dim3 grid((unsigned)((d->nx + VTI_TX - 1) / VTI_TX), (unsigned)((d->ny + VTI_TY - 1) / VTI_TY),
                  (unsigned)d->nz);
  k_vti_pack<<<grid, dim3(VTI_TX, VTI_TY), 0, (cudaStream_t)stream>>>(d->nx, d->ny, d->nz, p, alpha, vx, vy, vz,
                                                                      ibm_sf, static_cast<uint32_t*>(block));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    smac::set_error_text("%s: %s", fn, cudaGetErrorString(e));
    return SMAC_CUDA_ERROR;
  }
  return SMAC_OK;
}

smac_status smac_vti_write(const smac_grid_desc* d, const double origin[3], const void* block_host, const char* path) {
  static const char* fn = "smac_vti_write";
  if (!d || !origin || !block_host || !path) {
    smac::set_error_text("%s: null argument", fn);
    return SMAC_BAD_ARG;
  }
  if (!vti_shape_ok(d, fn)) return SMAC_BAD_SHAPE;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) {
    smac::set_error_text("%s: cannot open %s", fn, path);
    return SMAC_BAD_ARG;
  }
  const size_t n = (size_t)d->nx * d->ny * d->nz;
  // offsets of the four arrays in the appended block: each is preceded by
  // its UInt32 byte count
  const size_t off_p = 0, off_a = off_p + 4 + 4 * n, off_v = off_a + 4 + 4 * n, off_s = off_v + 4 + 12 * n;
  // The XML text of the reference's file (CFD/FileInOut.cpp:185-204), kept
  // character for character so that the files compare equal.
  std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
  std::fprintf(fp, "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt32\">\n");
  std::fprintf(fp,
               "  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\" Origin=\"%.15e %.15e %.15e\" "
               "Spacing=\"%.15e %.15e %.15e\">\n",
               d->nx, d->ny, d->nz, origin[0], origin[1], origin[2], d->dx, d->dy, d->dz);
  std::fprintf(fp, "    <Piece Extent=\"0 %d 0 %d 0 %d\">\n", d->nx, d->ny, d->nz);
  std::fprintf(fp, "      <PointData></PointData>\n");
  std::fprintf(fp, "      <CellData Scalars=\"alpha\" Vectors=\"velocity\">\n");
  std::fprintf(fp, "        <DataArray type=\"Float32\" Name=\"pressure\" format=\"appended\" offset=\"%zu\"/>\n",
               off_p);
  std::fprintf(fp, "        <DataArray type=\"Float32\" Name=\"alpha\" format=\"appended\" offset=\"%zu\"/>\n", off_a);
  std::fprintf(fp,
               "        <DataArray type=\"Float32\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"appended\" "
               "offset=\"%zu\"/>\n",
               off_v);
  std::fprintf(fp,
               "        <DataArray type=\"Float32\" Name=\"ibm_solid_fraction\" format=\"appended\" offset=\"%zu\"/>\n",
               off_s);
  std::fprintf(fp, "      </CellData>\n");
  std::fprintf(fp, "    </Piece>\n");
  std::fprintf(fp, "  </ImageData>\n");
  std::fprintf(fp, "  <AppendedData encoding=\"raw\">\n_");
  const size_t bytes = 16 + 24 * n;
  const size_t wrote = std::fwrite(block_host, 1, bytes, fp);
  std::fprintf(fp, "\n  </AppendedData>\n");
  std::fprintf(fp, "</VTKFile>\n");
  const int closed = std::fclose(fp);
  if (wrote != bytes || closed != 0) {
    smac::set_error_text("%s: short write to %s", fn, path);
    return SMAC_BAD_ARG;
  }
  return SMAC_OK;
}

}  // extern "C"
