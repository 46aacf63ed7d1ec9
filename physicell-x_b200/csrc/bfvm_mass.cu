// bfvm_mass.cu -- the periodic FP64 mass-balance record of a solve
// (bfvm_set_mass_log / bfvm_read_mass_log).
//
// Every `every` LOD steps bfvm_step appends one record: for each substrate
// the sum of the densities over all voxels, accumulated in FP64 on the
// device (for an FP32 solve, of the stored FP32 values plus the substrate's
// offset times the voxel count).  The sum is deterministic -- fixed
// per-block partials over whole rows, then one thread per substrate adds
// them in order -- so an FP64 solve's records are the same bits run after
// run, and an FP32 solve's records can be compared with them step for step:
// the check of the FP32 form against the FP64 path.  Records go into a ring
// of `capacity` entries on the device; a device counter places them, so the
// records are also right when the steps replay from a CUDA graph.  The
// reference has no counterpart (it has one precision); its own conservation
// printout is unit_test_conservation.cpp.
#include "bfvm_ctx.h"

namespace {

constexpr int kMassParts = 512;

// Partial sums of whole rows: block (b, s) adds rows b, b + G, ... of
// substrate s (rows of nx values at pitch nxp), threads across x.
template <typename T>
__global__ void __launch_bounds__(256) mass_partial_kernel(const T* __restrict__ f, int nx, int rows, int nxp,
                                                           double* __restrict__ partial) {
  __shared__ double red[256];
  const int s = blockIdx.y;
  double acc = 0.0;
  for (int r = blockIdx.x; r < rows; r += gridDim.x) {
    const T* row = f + (static_cast<size_t>(s) * rows + r) * nxp;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) acc += static_cast<double>(row[i]);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[static_cast<size_t>(s) * gridDim.x + blockIdx.x] = red[0];
}

// One record: partials added in order (plus the FP32 offset term), written
// at ring slot count % capacity; then the count advances.
__global__ void mass_record_kernel(const double* __restrict__ partial, int nparts, int S, const double* __restrict__ off,
                                   double nvox, double* __restrict__ ring, int capacity,
                                   unsigned long long* __restrict__ count) {
  const unsigned long long k = *count;
  const int s = threadIdx.x;
  if (s < S) {
    double acc = 0.0;
    for (int b = 0; b < nparts; ++b) acc += partial[static_cast<size_t>(s) * nparts + b];
    if (off != nullptr) acc += off[s] * nvox;
    ring[static_cast<size_t>(k % static_cast<unsigned long long>(capacity)) * S + s] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) *count = k + 1;
}

}  // namespace

namespace bfvm {

int enqueue_mass_record(bfvm_ctx* c) {
  const int rows = c->ny * c->nz;
  const int parts = rows < kMassParts ? rows : kMassParts;
  const dim3 grid(parts, c->S);
  double* partial = c->d_mass;
  double* ring = c->d_mass + static_cast<size_t>(c->S) * kMassParts;
  unsigned long long* count = reinterpret_cast<unsigned long long*>(ring + static_cast<size_t>(c->mass_capacity) * c->S);
  if (c->prec == BFVM_FP64)
    mass_partial_kernel<double><<<grid, 256, 0, c->stream>>>(static_cast<const double*>(c->f), c->nx, rows, c->nxp,
                                                             partial);
  else
    mass_partial_kernel<float><<<grid, 256, 0, c->stream>>>(static_cast<const float*>(c->f), c->nx, rows, c->nxp,
                                                            partial);
  BFVM_CUDA(cudaGetLastError());
  const double nvox = static_cast<double>(c->nx) * c->ny * c->nz;
  mass_record_kernel<<<1, 32 * ((c->S + 31) / 32), 0, c->stream>>>(
      partial, parts, c->S, c->prec == BFVM_FP32 ? c->d_off : nullptr, nvox, ring, c->mass_capacity, count);
  BFVM_CUDA(cudaGetLastError());
  note_launches(2);
  return BFVM_OK;
}

}  // namespace bfvm

extern "C" int bfvm_set_mass_log(bfvm_ctx* c, int every, int capacity) {
  if (!c || every < 0 || (every > 0 && (capacity < 1 || capacity > (1 << 24)))) return BFVM_ERR_ARG;
  bfvm::DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  bfvm::dfree(c, c->d_mass);
  c->d_mass = nullptr;
  c->mass_every = 0;
  c->mass_capacity = 0;
  c->mass_steps = 0;
  if (every == 0) return BFVM_OK;
  const size_t doubles = static_cast<size_t>(c->S) * kMassParts + static_cast<size_t>(capacity) * c->S;
  int rc = bfvm::dalloc(c, reinterpret_cast<void**>(&c->d_mass), doubles * sizeof(double) + 16);
  if (rc != BFVM_OK) return rc;
  BFVM_CUDA(cudaMemset(c->d_mass, 0, doubles * sizeof(double) + 16));
  c->mass_every = every;
  c->mass_capacity = capacity;
  return BFVM_OK;
}

extern "C" int bfvm_read_mass_log(bfvm_ctx* c, double* out, int max_records, int* n_total) {
  if (!c || max_records < 0 || (max_records > 0 && !out)) return BFVM_ERR_ARG;
  if (c->mass_every == 0) return BFVM_ERR_STATE;
  bfvm::DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  const size_t S = c->S;
  const double* ring = c->d_mass + S * kMassParts;
  unsigned long long count = 0;
  BFVM_CUDA(cudaMemcpy(&count, ring + static_cast<size_t>(c->mass_capacity) * S, sizeof(count),
                       cudaMemcpyDeviceToHost));
  const unsigned long long cap = static_cast<unsigned long long>(c->mass_capacity);
  const unsigned long long kept = count < cap ? count : cap;
  const unsigned long long first = count - kept;  // oldest record still in the ring
  const unsigned long long want = kept < static_cast<unsigned long long>(max_records) ? kept : max_records;
  for (unsigned long long q = 0; q < want; ++q) {
    const size_t slot = static_cast<size_t>((first + q) % cap);
    BFVM_CUDA(cudaMemcpy(out + q * S, ring + slot * S, sizeof(double) * S, cudaMemcpyDeviceToHost));
  }
  if (n_total) *n_total = static_cast<int>(count);
  return BFVM_OK;
}
