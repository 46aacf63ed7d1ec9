// bfvm_layout.cu -- conversion between the reference field layout and the
// device layout.
//
// Reference: one flat array, index ((i*ny + j)*nz + k)*S + d, z fastest with
// substrates interleaved (Cartesian_Mesh::voxel_index,
// BioFVM/BioFVM_mesh.cpp:1149-1158; Microenvironment::density_vector,
// BioFVM/BioFVM_microenvironment.cpp:1123-1130).
// Device:    f[d][k][j][i] with rows padded to nxp, x fastest.
// For each y-plane j the conversion is an (x,z) transpose per substrate,
// staged through a 32x33 shared-memory tile.
#include "bfvm_internal.h"

namespace bfvm {

namespace {

// FP32 fields hold rho - off[s] (off null for FP64, where values are exact).
template <typename T>
__global__ void pack_kernel(const double* __restrict__ aos, T* __restrict__ f, int nx, int ny, int nz, int S,
                            int nxp, const double* __restrict__ off) {
  __shared__ double tile[32][33];
  const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32, j = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int s = 0; s < S; ++s) {
    const double o = off ? off[s] : 0.0;
    for (int r = ty; r < 32; r += 8) {
      const int i = i0 + r, k = k0 + tx;
      if (i < nx && k < nz) {
        const double v = aos[((static_cast<size_t>(i) * ny + j) * nz + k) * S + s];
        tile[r][tx] = off ? v - o : v;
      }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int k = k0 + r, i = i0 + tx;
      if (i < nx && k < nz) f[((static_cast<size_t>(s) * nz + k) * ny + j) * nxp + i] = static_cast<T>(tile[tx][r]);
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void unpack_kernel(const T* __restrict__ f, double* __restrict__ aos, int nx, int ny, int nz, int S,
                              int nxp, const double* __restrict__ off) {
  __shared__ double tile[32][33];
  const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32, j = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int s = 0; s < S; ++s) {
    const double o = off ? off[s] : 0.0;
    for (int r = ty; r < 32; r += 8) {
      const int k = k0 + r, i = i0 + tx;
      if (i < nx && k < nz) {
        const double v = static_cast<double>(f[((static_cast<size_t>(s) * nz + k) * ny + j) * nxp + i]);
        tile[r][tx] = off ? v + o : v;
      }
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int i = i0 + r, k = k0 + tx;
      if (i < nx && k < nz) aos[((static_cast<size_t>(i) * ny + j) * nz + k) * S + s] = tile[tx][r];
    }
    __syncthreads();
  }
}

}  // namespace

template <typename T>
cudaError_t launch_pack(const double* aos, T* f, int nx, int ny, int nz, int S, int nxp, const double* off,
                        cudaStream_t st) {
  dim3 grid((nz + 31) / 32, (nx + 31) / 32, ny), block(32, 8);
  pack_kernel<T><<<grid, block, 0, st>>>(aos, f, nx, ny, nz, S, nxp, off);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_unpack(const T* f, double* aos, int nx, int ny, int nz, int S, int nxp, const double* off,
                          cudaStream_t st) {
  dim3 grid((nz + 31) / 32, (nx + 31) / 32, ny), block(32, 8);
  unpack_kernel<T><<<grid, block, 0, st>>>(f, aos, nx, ny, nz, S, nxp, off);
  return cudaGetLastError();
}

template cudaError_t launch_pack<double>(const double*, double*, int, int, int, int, int, const double*,
                                         cudaStream_t);
template cudaError_t launch_pack<float>(const double*, float*, int, int, int, int, int, const double*, cudaStream_t);
template cudaError_t launch_unpack<double>(const double*, double*, int, int, int, int, int, const double*,
                                           cudaStream_t);
template cudaError_t launch_unpack<float>(const float*, double*, int, int, int, int, int, const double*,
                                          cudaStream_t);

}  // namespace bfvm
