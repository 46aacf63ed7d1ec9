// bfvm_gradients.cu -- substrate gradients at every voxel.
//
// Reference: Microenvironment::compute_all_gradient_vectors
// (BioFVM/BioFVM_microenvironment.cpp:1454-1616): per substrate and axis, a
// one-sided difference (a - b) / dx at the two ends of each line and a
// central difference (a - b) / (2 dx) inside, evaluated as
// `g = a; g -= b; g /= h` -- one subtraction and one IEEE division, which the
// kernel repeats, so FP64 results equal the reference's bit for bit.  An axis
// of length 1 gets 0 (the reference reads outside its array there, and skips
// the z component when nz == 1).  The reference caches 2*dx in function
// statics on its first call; here each solve uses its own dx.
//
// Output layout is the reference's gradient_vectors: out[(v*S + d)*3 + axis]
// with v = (i*ny + j)*nz + k, z fastest, while the device field is x
// fastest.  A CTA owns 32 consecutive z by 8 consecutive x of one y-plane:
// per substrate it stages that block with a one-voxel halo in x and z, and
// the block's two y neighbours, in shared memory (rows of x read from the
// field), computes the gradients of its 256 voxels into a shared-memory
// output block, and then each warp writes one x row's 32 voxels -- a
// contiguous run of the output -- for up to kGroup substrates at a time.
#include "bfvm_ctx.h"

namespace {

constexpr int kGroup = 4;  // substrates staged per output block (keeps static shared memory under 48 KB)

template <typename T>
__global__ void __launch_bounds__(256) gradient_kernel(const T* __restrict__ f, int nx, int ny, int nz, int S,
                                                       int nxp, const double* __restrict__ off, double dx,
                                                       double* __restrict__ out) {
  __shared__ double c[34][10];     // this plane: (k - k0 + 1, i - i0 + 1)
  __shared__ double ym[32][9];     // plane j - 1: (k - k0, i - i0)
  __shared__ double yp[32][9];     // plane j + 1
  __shared__ double og[8][32][3 * kGroup + 1];  // output: (i - i0, k - k0, 3*(s - s0) + axis)
  const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 8, j = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const double two_dx = dx * 2.0;
  auto at = [&](int s, int k, int jj, int i) {
    return static_cast<double>(f[((static_cast<size_t>(s) * nz + k) * ny + jj) * nxp + i]);
  };
  // g = a; g -= b; g /= h  (BioFVM_microenvironment.cpp:1480-1482 and the
  // matching lines of every end cap and interior loop)
  auto grad = [](double a, double b, double h) {
    double g = a;
    g -= b;
    return g / h;
  };
  const int i = i0 + ty, k = k0 + tx;
  const int nk = min(32, nz - k0);
  for (int s0 = 0; s0 < S; s0 += kGroup) {
    const int ns = min(kGroup, S - s0);
    for (int sl = 0; sl < ns; ++sl) {
      const int s = s0 + sl;
      const double o = off ? off[s] : 0.0;
      for (int q = tid; q < 34 * 10; q += 256) {
        const int kk = q / 10, ii = q - kk * 10;
        const int gk = k0 - 1 + kk, gi = i0 - 1 + ii;
        if (gk >= 0 && gk < nz && gi >= 0 && gi < nx) c[kk][ii] = at(s, gk, j, gi) + o;
      }
      {
        const int kk = tid >> 3, ii = tid & 7;
        const int gk = k0 + kk, gi = i0 + ii;
        if (gk < nz && gi < nx) {
          if (j > 0) ym[kk][ii] = at(s, gk, j - 1, gi) + o;
          if (j < ny - 1) yp[kk][ii] = at(s, gk, j + 1, gi) + o;
        }
      }
      __syncthreads();
      if (i < nx && k < nz) {
        const int kk = tx + 1, ii = ty + 1;
        const double ctr = c[kk][ii];
        double gx = 0.0, gy = 0.0, gz = 0.0;
        if (nx > 1) {
          if (i == 0)
            gx = grad(c[kk][ii + 1], ctr, dx);
          else if (i == nx - 1)
            gx = grad(ctr, c[kk][ii - 1], dx);
          else
            gx = grad(c[kk][ii + 1], c[kk][ii - 1], two_dx);
        }
        if (ny > 1) {
          if (j == 0)
            gy = grad(yp[tx][ty], ctr, dx);
          else if (j == ny - 1)
            gy = grad(ctr, ym[tx][ty], dx);
          else
            gy = grad(yp[tx][ty], ym[tx][ty], two_dx);
        }
        if (nz > 1) {
          if (k == 0)
            gz = grad(c[kk + 1][ii], ctr, dx);
          else if (k == nz - 1)
            gz = grad(ctr, c[kk - 1][ii], dx);
          else
            gz = grad(c[kk + 1][ii], c[kk - 1][ii], two_dx);
        }
        og[ty][tx][3 * sl + 0] = gx;
        og[ty][tx][3 * sl + 1] = gy;
        og[ty][tx][3 * sl + 2] = gz;
      }
      __syncthreads();
    }
    // warp ty writes x row i: nk voxels, each 3*ns values at column 3*s0
    if (i < nx) {
      const int w = 3 * ns;
      double* row = out + (((static_cast<size_t>(i) * ny + j) * nz + k0) * S + s0) * 3;
      for (int q = tx; q < nk * w; q += 32) {
        const int kk = q / w, e = q - kk * w;
        row[static_cast<size_t>(kk) * 3 * S + e] = og[ty][kk][e];
      }
    }
    __syncthreads();
  }
}

int launch_gradients(bfvm_ctx* c, double* d_out) {
  const dim3 block(32, 8);
  const dim3 grid((c->nz + 31) / 32, (c->nx + 7) / 8, c->ny);
  if (c->prec == BFVM_FP64)
    gradient_kernel<double><<<grid, block, 0, c->stream>>>(static_cast<const double*>(c->f), c->nx, c->ny, c->nz,
                                                           c->S, c->nxp, nullptr, c->dx, d_out);
  else
    gradient_kernel<float><<<grid, block, 0, c->stream>>>(static_cast<const float*>(c->f), c->nx, c->ny, c->nz,
                                                          c->S, c->nxp, c->d_off, c->dx, d_out);
  BFVM_CUDA(cudaGetLastError());
  bfvm::note_launches(1);
  return BFVM_OK;
}

}  // namespace

extern "C" int bfvm_compute_gradients_device(bfvm_ctx* c, double* d_out) {
  if (!c || !d_out) return BFVM_ERR_ARG;
  bfvm::DeviceGuard g(c->device);
  return launch_gradients(c, d_out);
}

extern "C" int bfvm_compute_gradients(bfvm_ctx* c, double* out) {
  if (!c || !out) return BFVM_ERR_ARG;
  bfvm::DeviceGuard g(c->device);
  const size_t bytes = sizeof(double) * 3 * static_cast<size_t>(c->nx) * c->ny * c->nz * c->S;
  if (!c->d_grad) {
    const int rc = bfvm::dalloc(c, reinterpret_cast<void**>(&c->d_grad), bytes);
    if (rc != BFVM_OK) return rc;
  }
  int rc = launch_gradients(c, c->d_grad);
  if (rc != BFVM_OK) return rc;
  BFVM_CUDA(cudaMemcpyAsync(out, c->d_grad, bytes, cudaMemcpyDeviceToHost, c->stream));
  return bfvm_synchronize(c);
}
