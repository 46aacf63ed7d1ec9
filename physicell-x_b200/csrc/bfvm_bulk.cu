// bfvm_bulk.cu -- bulk (per-voxel) sources and sinks.
//
// Reference: Microenvironment::simulate_bulk_sources_and_sinks
// (BioFVM/BioFVM_microenvironment.cpp:1327-1368).  The reference asks three
// host callbacks for every voxel's supply rate S, target density T and
// uptake rate U; here they are device arrays in the field's device layout,
// uploaded once (bfvm_set_bulk_rates), and one elementwise pass applies
//     temp2 = T * S;  rho = fma(dt, temp2, rho);     (the reference's g++
//     temp3 = ((U + S) * dt) + 1;  rho /= temp3;      build contracts the
//                                                     first update, not temp3)
// so FP64 results equal the reference's bit for bit.  The pass reads the
// field, the three rate arrays and writes the field: 40 bytes per
// voxel-substrate in FP64 (36 in FP32).
#include "bfvm_internal.h"

namespace bfvm {

namespace {

template <typename T>
__global__ void bulk_kernel(T* __restrict__ f, const double* __restrict__ rates, size_t plane, int nx, int nxp,
                            long long rows, int rows_per_s, double dt, const double* __restrict__ off) {
  const long long total = rows * nx;
  for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long r = e / nx;
    const int i = static_cast<int>(e - r * nx);
    const size_t q = static_cast<size_t>(r) * nxp + i;
    const double s_rate = rates[q];
    const double target = rates[plane + q];
    const double u_rate = rates[2 * plane + q];
    const double o = off ? off[r / rows_per_s] : 0.0;
    double rho = static_cast<double>(f[q]) + o;
    double t2 = target;
    t2 *= s_rate;
    rho = __fma_rn(dt, t2, rho);
    double t3 = u_rate;
    t3 += s_rate;
    t3 *= dt;
    t3 += 1.0;
    rho /= t3;
    f[q] = static_cast<T>(rho - o);
  }
}

}  // namespace

template <typename T>
cudaError_t launch_bulk(T* f, const double* rates, int nx, int ny, int nz, int S, int nxp, double dt,
                        const double* off, int sm_count, cudaStream_t st) {
  const long long rows = static_cast<long long>(S) * nz * ny;
  const size_t plane = static_cast<size_t>(rows) * nxp;
  const long long total = rows * nx;
  long long blocks = (total + 255) / 256;
  const long long cap = static_cast<long long>(sm_count) * 8;
  if (blocks > cap) blocks = cap;
  bulk_kernel<T><<<static_cast<unsigned>(blocks), 256, 0, st>>>(f, rates, plane, nx, nxp, rows, nz * ny, dt, off);
  return cudaGetLastError();
}

template cudaError_t launch_bulk<double>(double*, const double*, int, int, int, int, int, double, const double*, int,
                                         cudaStream_t);
template cudaError_t launch_bulk<float>(float*, const double*, int, int, int, int, int, double, const double*, int,
                                        cudaStream_t);

}  // namespace bfvm
