// bfvm_output.cu -- density output in the reference's MATLAB v4 format.
//
// Reference: Microenvironment::write_to_matlab(filename)
// (BioFVM/BioFVM_microenvironment.cpp:1222-1249) with write_matlab4_header
// (BioFVM/BioFVM_matlab.cpp:536-578): a 20-byte header (type 0, rows 4+S,
// columns = voxels, imag 0, name length), the variable name
// "multiscale_microenvironment" without a terminator, then one column per
// voxel in reference order: centre x, y, z, volume, the S densities.  Voxel
// centres are start + (i + 0.5)*dx, which the reference's build evaluates as
// one fma (BioFVM/BioFVM_mesh.cpp:1436-1560, one rank), and the volume is
// dx*dy*dz; the file is byte-identical to the reference's for an FP64 solve.
//
// The columns are assembled on the device in chunks (centres computed there,
// densities from the reference-layout copy of the field) and streamed to the
// file through a pinned host buffer.
#include <cstdio>
#include <cstring>

#include "bfvm_ctx.h"

namespace {

__global__ void matlab_columns_kernel(const double* __restrict__ aos, long long v0, long long count, int ny, int nz,
                                      int S, double xs, double ys, double zs, double dx, double dv,
                                      double* __restrict__ out) {
  const int w = 4 + S;
  const long long total = count * w;
  for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long vl = e / w;
    const int c = static_cast<int>(e - vl * w);
    const long long v = v0 + vl;
    double val;
    if (c < 3) {
      const long long ij = v / nz;
      const int idx = c == 0 ? static_cast<int>(ij / ny) : (c == 1 ? static_cast<int>(ij % ny) : static_cast<int>(v % nz));
      const double start = c == 0 ? xs : (c == 1 ? ys : zs);
      val = __fma_rn(static_cast<double>(idx) + 0.5, dx, start);
    } else if (c == 3) {
      val = dv;
    } else {
      val = aos[v * S + (c - 4)];
    }
    out[e] = val;
  }
}

}  // namespace

namespace bfvm {

// One MATLAB v4 matrix of 4 + S rows (S = c->S with densities, else 0) and
// one column per voxel, assembled on the device in chunks: the
// microenvironment file (name "multiscale_microenvironment", with the
// densities) or General_Mesh::write_to_matlab's mesh file
// (BioFVM/BioFVM_mesh.cpp:425-447: name "mesh", centre and volume only).
int write_matlab_columns(bfvm_ctx* c, const char* path, const char* name, bool densities, double x_start,
                         double y_start, double z_start) {
  if (!c || !path) return BFVM_ERR_ARG;
  bfvm::DeviceGuard g(c->device);
  int rc = BFVM_OK;
  if (densities) {
    rc = bfvm::ensure_staging(c);
    if (rc != BFVM_OK) return rc;
    if ((rc = bfvm::unpack_to_device_aos(c, c->d_staging)) != BFVM_OK) return rc;
  }
  const int S = densities ? c->S : 0;
  const long long nv = static_cast<long long>(c->nx) * c->ny * c->nz;
  const int w = 4 + S;
  const long long chunk = nv < (1LL << 20) ? nv : (1LL << 20);  // voxels per transfer
  const size_t chunk_bytes = sizeof(double) * static_cast<size_t>(chunk) * w;
  double* d_cols = nullptr;
  double* h_cols = nullptr;
  FILE* fp = nullptr;
  auto finish = [&](int status) {
    if (d_cols) cudaFree(d_cols);
    if (h_cols) cudaFreeHost(h_cols);
    if (fp) {
      if (std::fclose(fp) != 0 && status == BFVM_OK) status = BFVM_ERR_ARG;
    }
    return status;
  };
  if (cudaMalloc(&d_cols, chunk_bytes) != cudaSuccess || cudaMallocHost(&h_cols, chunk_bytes) != cudaSuccess) {
    cudaGetLastError();
    return finish(BFVM_ERR_OOM);
  }
  fp = std::fopen(path, "wb");
  if (!fp) {
    std::fprintf(stderr, "biofvm_b200: cannot open %s for writing\n", path);
    return finish(BFVM_ERR_ARG);
  }
  const size_t name_len = std::strlen(name);
  const unsigned int hdr[5] = {0u, static_cast<unsigned int>(w), static_cast<unsigned int>(nv), 0u,
                               static_cast<unsigned int>(name_len)};
  bool ok = std::fwrite(hdr, sizeof(unsigned int), 5, fp) == 5 && std::fwrite(name, 1, name_len, fp) == name_len;
  double dv = c->dx * c->dx;
  dv *= c->dx;
  const double xs = x_start + 0.0, ys = y_start + 0.0, zs = z_start + 0.0;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  for (long long v0 = 0; ok && v0 < nv; v0 += chunk) {
    const long long cnt = nv - v0 < chunk ? nv - v0 : chunk;
    const long long total = cnt * w;
    long long blocks = (total + 255) / 256;
    if (blocks > 8LL * sms) blocks = 8LL * sms;
    matlab_columns_kernel<<<static_cast<unsigned>(blocks), 256, 0, c->stream>>>(
        c->d_staging, v0, cnt, c->ny, c->nz, S, xs, ys, zs, c->dx, dv, d_cols);
    if (cudaGetLastError() != cudaSuccess) return finish(BFVM_ERR_CUDA);
    bfvm::note_launches(1);
    const size_t bytes = sizeof(double) * static_cast<size_t>(total);
    if (cudaMemcpyAsync(h_cols, d_cols, bytes, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
      return finish(BFVM_ERR_CUDA);
    ok = std::fwrite(h_cols, 1, bytes, fp) == bytes;
  }
  if (!ok) std::fprintf(stderr, "biofvm_b200: writing %s failed\n", path);
  return finish(ok ? BFVM_OK : BFVM_ERR_ARG);
}

}  // namespace bfvm

extern "C" int bfvm_write_matlab(bfvm_ctx* c, const char* path, double x_start, double y_start, double z_start) {
  return bfvm::write_matlab_columns(c, path, "multiscale_microenvironment", true, x_start, y_start, z_start);
}

extern "C" int bfvm_write_mesh_matlab(bfvm_ctx* c, const char* path, double x_start, double y_start,
                                      double z_start) {
  return bfvm::write_matlab_columns(c, path, "mesh", false, x_start, y_start, z_start);
}
