// bfvm_agents.cu -- device side of the cell sources/sinks.
//
// Reference: Microenvironment::simulate_cell_sources_and_sinks
// (BioFVM/BioFVM_microenvironment.cpp:1370-1384) loops over all agents and
// each agent updates the densities of its voxel,
// Basic_Agent::simulate_secretion_and_uptake (BioFVM/BioFVM_basic_agent.cpp:509-559):
//     rho += c1;  rho /= c2;  rho += e2          (per substrate)
// with the constants of Basic_Agent::set_internal_uptake_constants (:224-274).
// Updates of agents in different voxels commute; agents sharing a voxel must
// be applied in agent-list order (the single-threaded reference order; its
// OpenMP loop races there).  So the device keeps the agents stably sorted by
// voxel: a stable LSD radix sort on the device voxel id keeps agent-list order
// inside each voxel, and a CSR over x-lines lets the x sweep apply a line's
// agents as it walks the line.
#include <climits>

#include "bfvm_agents.h"

namespace bfvm {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

// Reference voxel index ((i*ny + j)*nz + k) -> device voxel id ((k*ny + j)*nx + i).
__device__ __forceinline__ unsigned ref_to_dev(int v, int nx, int ny, int nz) {
  const int k = v % nz;
  const int ij = v / nz;
  const int j = ij % ny;
  const int i = ij / ny;
  return (static_cast<unsigned>(k) * ny + j) * nx + i;
}

__global__ void agent_keys_kernel(int n, const int* __restrict__ voxel, const unsigned char* __restrict__ active,
                                  int nx, int ny, int nz, unsigned sentinel, unsigned* __restrict__ keys,
                                  int* __restrict__ vals, unsigned* __restrict__ dev_voxel) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int v = voxel[a];
  const bool ok = v >= 0 && v < nx * ny * nz && (active == nullptr || active[a] != 0);
  const unsigned key = ok ? ref_to_dev(v, nx, ny, nz) : sentinel;
  keys[a] = key;
  vals[a] = a;
  dev_voxel[a] = key;
}

// Basic_Agent::set_internal_uptake_constants (BioFVM_basic_agent.cpp:224-274),
// operation by operation; the two axpy calls are fused multiply-adds as in the
// reference's g++ build.  e1 (optional) receives net_export_rate * dt, the
// export an agent with internalized-substrate tracking subtracts from its own
// amounts each step (cell_source_sink_solver_temp_export1).
__global__ void agent_constants_kernel(int n, int S, double dt, double voxel_volume, const double* __restrict__ volume,
                                       const double* __restrict__ sec, const double* __restrict__ upt,
                                       const double* __restrict__ sat, const double* __restrict__ exp_,
                                       double* __restrict__ c1, double* __restrict__ c2, double* __restrict__ e2,
                                       double* __restrict__ e1) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * S) return;
  const int a = idx / S;
  const double k = dt * volume[a] / voxel_volume;
  double t1 = 0.0;
  t1 += sec[idx];
  t1 *= sat[idx];
  t1 *= k;
  double t2 = 1.0;
  t2 = __fma_rn(k, sec[idx], t2);
  t2 = __fma_rn(k, upt[idx], t2);
  double x1 = exp_[idx];
  x1 *= dt;
  c1[idx] = t1;
  c2[idx] = t2;
  e2[idx] = x1 / voxel_volume;
  if (e1) e1[idx] = x1;
}

__global__ void radix_hist_kernel(int n, const unsigned* __restrict__ keys, int shift, int nblocks,
                                  unsigned* __restrict__ hist) {
  __shared__ unsigned cnt[kRadix];
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) cnt[d] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortItems; ++r) {
    const int e = base + r * kSortThreads + threadIdx.x;
    if (e < n) atomicAdd(&cnt[(keys[e] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[static_cast<size_t>(d) * nblocks + blockIdx.x] = cnt[d];
}

// Exclusive scan of m entries in place, one block of 1024 threads.
__global__ void scan_kernel(unsigned* __restrict__ x, int m) {
  __shared__ unsigned part[1024];
  const int t = threadIdx.x;
  const int per = (m + blockDim.x - 1) / blockDim.x;
  const int lo = min(m, t * per), hi = min(m, lo + per);
  unsigned s = 0;
  for (int e = lo; e < hi; ++e) s += x[e];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const unsigned v = (t >= off) ? part[t - off] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  unsigned run = (t == 0) ? 0u : part[t - 1];
  for (int e = lo; e < hi; ++e) {
    const unsigned v = x[e];
    x[e] = run;
    run += v;
  }
}

// Stable scatter of one radix pass.  Within a block the tile is walked in
// steps of 256 consecutive elements; an element's rank among equal digits
// is (earlier steps) + (earlier warps of this step) + (lower lanes of its warp),
// so the output keeps the input order of equal digits.
__global__ void radix_scatter_kernel(int n, const unsigned* __restrict__ kin, const int* __restrict__ vin, int shift,
                                     int nblocks, const unsigned* __restrict__ offsets, unsigned* __restrict__ kout,
                                     int* __restrict__ vout) {
  __shared__ unsigned warp_cnt[kSortThreads / 32][kRadix];
  __shared__ unsigned running[kRadix];
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  for (int d = t; d < kRadix; d += blockDim.x) running[d] = offsets[static_cast<size_t>(d) * nblocks + blockIdx.x];
  const int base = blockIdx.x * kSortTile;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int r = 0; r < kSortItems; ++r) {
    for (int q = t; q < (kSortThreads / 32) * kRadix; q += blockDim.x) (&warp_cnt[0][0])[q] = 0;
    __syncthreads();
    const int e = base + r * kSortThreads + t;
    const bool in = e < n;
    unsigned key = 0;
    int val = 0;
    unsigned digit = kRadix;  // out-of-range lanes group among themselves
    if (in) {
      key = kin[e];
      val = vin[e];
      digit = (key >> shift) & (kRadix - 1);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const unsigned below = __popc(peers & lt_mask);
    if (in && below == 0) warp_cnt[w][digit] = __popc(peers);
    __syncthreads();
    if (in) {
      unsigned rank = running[digit] + below;
      for (int w2 = 0; w2 < w; ++w2) rank += warp_cnt[w2][digit];
      kout[rank] = key;
      vout[rank] = val;
    }
    __syncthreads();
    for (int d = t; d < kRadix; d += blockDim.x) {
      unsigned tot = 0;
      for (int w2 = 0; w2 < kSortThreads / 32; ++w2) tot += warp_cnt[w2][d];
      running[d] += tot;
    }
    __syncthreads();
  }
}

// CSR over x-lines from the sorted keys, plus the per-agent x index and the
// coefficients gathered into [S][n] in sorted order.
__global__ void agent_csr_kernel(int n, const unsigned* __restrict__ sk, const int* __restrict__ sv, unsigned sentinel,
                                 int nx, int n_lines, int S, const double* __restrict__ c1, const double* __restrict__ c2,
                                 const double* __restrict__ e2, int* __restrict__ line_off, int* __restrict__ a_i,
                                 double* __restrict__ ac1, double* __restrict__ ac2, double* __restrict__ ae2,
                                 int* __restrict__ n_valid_out, int* __restrict__ agent_pos) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && (n == 0 || sk[0] >= sentinel)) {
    *n_valid_out = 0;
    for (int l = 0; l <= n_lines; ++l) line_off[l] = 0;
  }
  if (p >= n) return;
  if (agent_pos != nullptr) agent_pos[sv[p]] = p;
  const unsigned key = sk[p];
  if (key >= sentinel) return;
  const int line = static_cast<int>(key / nx);
  const int lprev = (p == 0) ? -1 : static_cast<int>(sk[p - 1] / nx);
  for (int l = lprev + 1; l <= line; ++l) line_off[l] = p;
  const bool last = (p + 1 == n) || (sk[p + 1] >= sentinel);
  if (last) {
    for (int l = line + 1; l <= n_lines; ++l) line_off[l] = p + 1;
    *n_valid_out = p + 1;
  }
  a_i[p] = static_cast<int>(key % nx);
  const int a = sv[p];
  for (int s = 0; s < S; ++s) {
    ac1[static_cast<size_t>(s) * n + p] = c1[static_cast<size_t>(a) * S + s];
    ac2[static_cast<size_t>(s) * n + p] = c2[static_cast<size_t>(a) * S + s];
    ae2[static_cast<size_t>(s) * n + p] = e2[static_cast<size_t>(a) * S + s];
  }
}

// Standalone (unfused) source/sink stage: one thread per (voxel run, substrate).
template <typename T>
__global__ void agent_sources_kernel(int n, const unsigned* __restrict__ sk, unsigned sentinel, int S, int nx, int ny,
                                     int nz, int nxp, const double* __restrict__ ac1, const double* __restrict__ ac2,
                                     const double* __restrict__ ae2, const double* __restrict__ off,
                                     T* __restrict__ f, const AgentTrack tr, int s_lo, int s_hi) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long long>(n) * (s_hi - s_lo)) return;
  const int s = s_lo + static_cast<int>(idx / n);
  const int p = static_cast<int>(idx % n);
  const unsigned key = sk[p];
  if (key >= sentinel) return;
  if (p > 0 && sk[p - 1] == key) return;
  const int i = key % nx;
  const int jk = key / nx;
  T* rho = f + (static_cast<size_t>(s) * nz * ny + jk) * nxp + i;
  double r = static_cast<double>(*rho);
  if (off) r += off[s];
  for (int q = p; q < n && sk[q] == key; ++q) {
    const size_t c = static_cast<size_t>(s) * n + q;
    r = agent_update(r, ac1[c], ac2[c], ae2[c], q, s, tr);
  }
  if (off) r -= off[s];
  *rho = static_cast<T>(r);
  (void)ny;
}

// The same stage with the constants read through the sorted order from the
// agent-list layout c1/c2/e2[a*S + s], so no gathered copy is needed; the
// operations and their order per voxel are those of agent_sources_kernel.
template <typename T>
__global__ void agent_sources_by_order_kernel(int n, const unsigned* __restrict__ sk, const int* __restrict__ order,
                                              unsigned sentinel, int S, int nx, int nz_ny, int nxp,
                                              const double* __restrict__ c1, const double* __restrict__ c2,
                                              const double* __restrict__ e2, const double* __restrict__ off,
                                              T* __restrict__ f) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long long>(n) * S) return;
  const int s = static_cast<int>(idx / n);
  const int p = static_cast<int>(idx % n);
  const unsigned key = sk[p];
  if (key >= sentinel) return;
  if (p > 0 && sk[p - 1] == key) return;
  const int i = key % nx;
  const int jk = key / nx;
  T* rho = f + (static_cast<size_t>(s) * nz_ny + jk) * nxp + i;
  double r = static_cast<double>(*rho);
  if (off) r += off[s];
  for (int q = p; q < n && sk[q] == key; ++q) {
    const size_t a = static_cast<size_t>(order[q]) * S + s;
    r += c1[a];
    r /= c2[a];
    r += e2[a];
  }
  if (off) r -= off[s];
  *rho = static_cast<T>(r);
}

// Densities at each agent's voxel, in agent-list order, [n][S] FP64
// (what Basic_Agent::nearest_density_vector exposes to the agent).
template <typename T>
__global__ void agent_sample_kernel(int n, const unsigned* __restrict__ dev_voxel, unsigned sentinel, int S, int nx,
                                    int ny, int nz, int nxp, const T* __restrict__ f, const double* __restrict__ off,
                                    double* __restrict__ out) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long long>(n) * S) return;
  const int a = static_cast<int>(idx / S), s = static_cast<int>(idx % S);
  const unsigned key = dev_voxel[a];
  double v = 0.0;
  if (key < sentinel) {
    const int i = key % nx;
    const int jk = key / nx;
    v = static_cast<double>(f[(static_cast<size_t>(s) * nz * ny + jk) * nxp + i]);
    if (off) v += off[s];
  }
  out[idx] = v;
  (void)ny;
}

}  // namespace

size_t agent_scratch_bytes(int n) {
  const int nblocks = (n + kSortTile - 1) / kSortTile;
  return sizeof(unsigned) * (4 * static_cast<size_t>(n) + static_cast<size_t>(kRadix) * (nblocks + 1)) + 256;
}

cudaError_t agents_compute_constants(int n, int S, double dt, double voxel_volume, const double* volume,
                                     const double* sec, const double* upt, const double* sat, const double* exp_,
                                     double* c1, double* c2, double* e2, cudaStream_t st, double* e1) {
  if (n == 0) return cudaSuccess;
  const int total = n * S;
  agent_constants_kernel<<<(total + 255) / 256, 256, 0, st>>>(n, S, dt, voxel_volume, volume, sec, upt, sat, exp_, c1,
                                                              c2, e2, e1);
  return cudaGetLastError();
}

cudaError_t agents_build(const AgentBuild& b, cudaStream_t st, int* launches) {
  const int n = b.n;
  const unsigned sentinel = static_cast<unsigned>(b.nx) * b.ny * b.nz;
  if (n == 0) {
    agent_csr_kernel<<<1, 1, 0, st>>>(0, b.sorted_keys, b.sorted_vals, sentinel, b.nx, b.ny * b.nz, b.S, b.c1, b.c2,
                                      b.e2, b.line_off, b.a_i, b.ac1, b.ac2, b.ae2, b.n_valid, nullptr);
    *launches = 1;
    return cudaGetLastError();
  }
  // scratch: keys0 | vals0 | keys1 | vals1 | hist
  unsigned* k0 = reinterpret_cast<unsigned*>(b.scratch);
  int* v0 = reinterpret_cast<int*>(k0 + n);
  unsigned* k1 = reinterpret_cast<unsigned*>(v0 + n);
  int* v1 = reinterpret_cast<int*>(k1 + n);
  unsigned* hist = reinterpret_cast<unsigned*>(v1 + n);
  agent_keys_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, b.voxel, b.active, b.nx, b.ny, b.nz, sentinel, k0, v0,
                                                     b.dev_voxel);
  int bits = 1;
  while (bits < 32 && (static_cast<unsigned long long>(1) << bits) <= sentinel) ++bits;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  const int nblocks = (n + kSortTile - 1) / kSortTile;
  unsigned* kin = k0;
  int* vin = v0;
  for (int pass = 0; pass < passes; ++pass) {
    // The last pass writes straight into the sorted arrays.
    unsigned* kout = (pass == passes - 1) ? b.sorted_keys : (kin == k0 ? k1 : k0);
    int* vout = (pass == passes - 1) ? b.sorted_vals : (vin == v0 ? v1 : v0);
    const int shift = pass * kRadixBits;
    radix_hist_kernel<<<nblocks, kSortThreads, 0, st>>>(n, kin, shift, nblocks, hist);
    scan_kernel<<<1, 1024, 0, st>>>(hist, kRadix * nblocks);
    radix_scatter_kernel<<<nblocks, kSortThreads, 0, st>>>(n, kin, vin, shift, nblocks, hist, kout, vout);
    kin = kout;
    vin = vout;
  }
  // the sort needs only the voxel ids; the constants are first read here
  if (b.constants_ready) {
    const cudaError_t e = cudaStreamWaitEvent(st, b.constants_ready, 0);
    if (e != cudaSuccess) return e;
  }
  agent_csr_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, b.sorted_keys, b.sorted_vals, sentinel, b.nx, b.ny * b.nz, b.S,
                                                    b.c1, b.c2, b.e2, b.line_off, b.a_i, b.ac1, b.ac2, b.ae2,
                                                    b.n_valid, b.agent_pos);
  *launches = 2 + 3 * passes;
  return cudaGetLastError();
}

cudaError_t agents_sort(int n, const int* voxel, const unsigned char* active, int nx, int ny, int nz, void* scratch,
                        cudaStream_t st, const unsigned** sorted_keys, const int** sorted_order, int* launches) {
  *launches = 0;
  if (n == 0) return cudaSuccess;
  const unsigned sentinel = static_cast<unsigned>(nx) * ny * nz;
  // scratch: keys0 | vals0 | keys1 | vals1 | hist; the passes ping-pong
  // between the two key/value pairs.
  unsigned* k0 = reinterpret_cast<unsigned*>(scratch);
  int* v0 = reinterpret_cast<int*>(k0 + n);
  unsigned* k1 = reinterpret_cast<unsigned*>(v0 + n);
  int* v1 = reinterpret_cast<int*>(k1 + n);
  unsigned* hist = reinterpret_cast<unsigned*>(v1 + n);
  // The per-agent device voxel ids go to keys1, which the first pass then
  // overwrites: this variant keeps no list-order copy.
  agent_keys_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, voxel, active, nx, ny, nz, sentinel, k0, v0, k1);
  int bits = 1;
  while (bits < 32 && (static_cast<unsigned long long>(1) << bits) <= sentinel) ++bits;
  const int passes = (bits + kRadixBits - 1) / kRadixBits;
  const int nblocks = (n + kSortTile - 1) / kSortTile;
  unsigned* kin = k0;
  int* vin = v0;
  for (int pass = 0; pass < passes; ++pass) {
    unsigned* kout = (kin == k0) ? k1 : k0;
    int* vout = (vin == v0) ? v1 : v0;
    const int shift = pass * kRadixBits;
    radix_hist_kernel<<<nblocks, kSortThreads, 0, st>>>(n, kin, shift, nblocks, hist);
    scan_kernel<<<1, 1024, 0, st>>>(hist, kRadix * nblocks);
    radix_scatter_kernel<<<nblocks, kSortThreads, 0, st>>>(n, kin, vin, shift, nblocks, hist, kout, vout);
    kin = kout;
    vin = vout;
  }
  *sorted_keys = kin;
  *sorted_order = vin;
  *launches = 1 + 3 * passes;
  return cudaGetLastError();
}

// New constants for m listed agents (agent-list indices idx[m], rows v1/v2/v3
// [m][S]) of a built list: written to the list-order arrays c1/c2/e2 [n][S]
// and, through agent_pos (list index -> sorted position), to the sorted,
// substrate-major arrays ac1/ac2/ae2 [S][n] the source stage reads.
__global__ void agent_update_kernel(int m, int S, int n, const int* __restrict__ idx, const double* __restrict__ v1,
                                    const double* __restrict__ v2, const double* __restrict__ v3,
                                    const int* __restrict__ agent_pos, double* __restrict__ c1,
                                    double* __restrict__ c2, double* __restrict__ e2, double* __restrict__ ac1,
                                    double* __restrict__ ac2, double* __restrict__ ae2) {
  const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= static_cast<long long>(m) * S) return;
  const int r = static_cast<int>(q / S), s = static_cast<int>(q % S);
  const int a = idx[r];
  const int p = agent_pos[a];
  const size_t src = static_cast<size_t>(r) * S + s, lst = static_cast<size_t>(a) * S + s;
  const size_t srt = static_cast<size_t>(s) * n + p;
  const double x1 = v1[src], x2 = v2[src], x3 = v3[src];
  c1[lst] = x1;
  c2[lst] = x2;
  e2[lst] = x3;
  ac1[srt] = x1;
  ac2[srt] = x2;
  ae2[srt] = x3;
}

cudaError_t agents_update_constants(int m, int S, int n, const int* idx, const double* v1, const double* v2,
                                    const double* v3, const int* agent_pos, double* c1, double* c2, double* e2,
                                    double* ac1, double* ac2, double* ae2, cudaStream_t st) {
  if (m == 0) return cudaSuccess;
  const long long total = static_cast<long long>(m) * S;
  agent_update_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(m, S, n, idx, v1, v2, v3, agent_pos,
                                                                                  c1, c2, e2, ac1, ac2, ae2);
  return cudaGetLastError();
}

// Loads (under CUDA's lazy module loading) every kernel agents_sort and
// agents_apply_sources_by_order launch, so their first launch on the current
// device allocates nothing for code.
cudaError_t agents_preload_sort_kernels() {
  const void* kernels[] = {reinterpret_cast<const void*>(agent_keys_kernel),
                           reinterpret_cast<const void*>(radix_hist_kernel),
                           reinterpret_cast<const void*>(scan_kernel),
                           reinterpret_cast<const void*>(radix_scatter_kernel),
                           reinterpret_cast<const void*>(agent_sources_by_order_kernel<double>),
                           reinterpret_cast<const void*>(agent_sources_by_order_kernel<float>)};
  for (const void* k : kernels) {
    cudaFuncAttributes a;
    const cudaError_t e = cudaFuncGetAttributes(&a, k);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T>
cudaError_t agents_apply_sources_by_order(int n, const unsigned* sorted_keys, const int* sorted_order, int S, int nx,
                                          int ny, int nz, int nxp, const double* c1, const double* c2,
                                          const double* e2, const double* off, T* f, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned sentinel = static_cast<unsigned>(nx) * ny * nz;
  const long long total = static_cast<long long>(n) * S;
  agent_sources_by_order_kernel<T><<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(
      n, sorted_keys, sorted_order, sentinel, S, nx, ny * nz, nxp, c1, c2, e2, off, f);
  return cudaGetLastError();
}

template cudaError_t agents_apply_sources_by_order<double>(int, const unsigned*, const int*, int, int, int, int, int,
                                                           const double*, const double*, const double*,
                                                           const double*, double*, cudaStream_t);
template cudaError_t agents_apply_sources_by_order<float>(int, const unsigned*, const int*, int, int, int, int, int,
                                                          const double*, const double*, const double*, const double*,
                                                          float*, cudaStream_t);

template <typename T>
cudaError_t agents_apply_sources(int n, const unsigned* sorted_keys, int S, int nx, int ny, int nz, int nxp,
                                 const double* ac1, const double* ac2, const double* ae2, const double* off, T* f,
                                 const AgentTrack& track, cudaStream_t st, int s_lo, int s_hi) {
  if (n == 0) return cudaSuccess;
  if (s_hi < 0) s_hi = S;
  if (s_lo < 0 || s_lo >= s_hi || s_hi > S) return cudaErrorInvalidValue;
  const unsigned sentinel = static_cast<unsigned>(nx) * ny * nz;
  const long long total = static_cast<long long>(n) * (s_hi - s_lo);
  agent_sources_kernel<T><<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(
      n, sorted_keys, sentinel, S, nx, ny, nz, nxp, ac1, ac2, ae2, off, f, track, s_lo, s_hi);
  return cudaGetLastError();
}

namespace {
// dst[s*n + p] = src[order[p]*S + s]: a per-agent [n][S] array gathered into
// sorted order, substrate-major.
__global__ void gather_sorted_kernel(int n, int S, const int* __restrict__ order, const double* __restrict__ src,
                                     double* __restrict__ dst) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long long>(n) * S) return;
  const int s = static_cast<int>(idx / n);
  const int p = static_cast<int>(idx % n);
  dst[idx] = src[static_cast<size_t>(order[p]) * S + s];
}
}  // namespace

cudaError_t agents_gather_sorted(int n, int S, const int* order, const double* src, double* dst, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const long long total = static_cast<long long>(n) * S;
  gather_sorted_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(n, S, order, src, dst);
  return cudaGetLastError();
}

template <typename T>
cudaError_t agents_sample(int n, const unsigned* dev_voxel, int S, int nx, int ny, int nz, int nxp, const T* f,
                          const double* off, double* out, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned sentinel = static_cast<unsigned>(nx) * ny * nz;
  const long long total = static_cast<long long>(n) * S;
  agent_sample_kernel<T><<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(n, dev_voxel, sentinel, S, nx,
                                                                                      ny, nz, nxp, f, off, out);
  return cudaGetLastError();
}

template cudaError_t agents_apply_sources<double>(int, const unsigned*, int, int, int, int, int, const double*,
                                                  const double*, const double*, const double*, double*,
                                                  const AgentTrack&, cudaStream_t, int, int);
template cudaError_t agents_apply_sources<float>(int, const unsigned*, int, int, int, int, int, const double*,
                                                 const double*, const double*, const double*, float*,
                                                 const AgentTrack&, cudaStream_t, int, int);
template cudaError_t agents_sample<double>(int, const unsigned*, int, int, int, int, int, const double*,
                                           const double*, double*, cudaStream_t);
template cudaError_t agents_sample<float>(int, const unsigned*, int, int, int, int, int, const float*, const double*,
                                          double*, cudaStream_t);

}  // namespace bfvm
