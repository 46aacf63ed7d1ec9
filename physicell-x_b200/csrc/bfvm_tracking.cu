// bfvm_tracking.cu -- the substrates each agent internalizes.
//
// Reference: with Microenvironment_Options::track_internalized_substrates_in_each_agent
// (BioFVM/BioFVM_microenvironment.h:477) on, Basic_Agent::simulate_secretion_and_uptake
// (BioFVM/BioFVM_basic_agent.cpp:520-532, 553-556) keeps, per agent and
// substrate, the opposite of the net change it made to its voxel:
//     internal -= (((1 - c2) * rho + c1) / c2) * V_voxel    before the update
//     internal -= export1                                   after it
// with export1 = net_export_rate * dt (:261-262).  The bookkeeping itself runs
// inside the source/sink stage (agent_update, used by the fused x sweep and
// by the standalone stage); this file holds the per-solve buffers and the
// C-ABI entry points: switching it on, the per-step exports of a list given
// as constants, reading and writing the amounts, and
// Basic_Agent::release_internalized_substrates (:310-333).
//
// The amounts are one [n][S] array in agent-list order.  A new agent list
// keeps the amounts of the list positions it shares with the previous one
// and starts new positions at zero, as the reference's per-agent vectors
// start at zero (:301) and survive while the agent lives.
#include "bfvm_agents.h"
#include "bfvm_ctx.h"

using namespace bfvm;

namespace {

// e1[a*S + s] = net_export[a*S + s] * dt (BioFVM_basic_agent.cpp:261-262).
__global__ void export_kernel(long long total, double dt, const double* __restrict__ net_export,
                              double* __restrict__ e1) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  double x = net_export[idx];
  x *= dt;
  e1[idx] = x;
}

// Basic_Agent::release_internalized_substrates (BioFVM_basic_agent.cpp:
// 310-333) for `count` agents in the order given: internal /= V_voxel;
// internal *= fraction; rho += internal; internal = 0.  One thread per
// substrate walks the agents in order, so agents sharing a voxel add in the
// reference's order.  The reference releases whether or not the agent is
// active, so the voxel comes from the list's voxel index (reference layout
// (i*ny + j)*nz + k); an agent outside the mesh keeps its amounts.
template <typename T>
__global__ void release_kernel(int count, const int* __restrict__ agents, const double* __restrict__ fraction, int n,
                               const int* __restrict__ voxel, int S, int nx, int ny, int nz, int nxp, double vvox,
                               const double* __restrict__ off, double* __restrict__ internal, T* __restrict__ f) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const long long nvox = static_cast<long long>(nx) * ny * nz;
  for (int q = 0; q < count; ++q) {
    const int a = agents[q];
    if (a < 0 || a >= n) continue;
    const int v = voxel[a];
    if (v < 0 || v >= nvox) continue;
    double* in = internal + static_cast<size_t>(a) * S + s;
    double x = *in;
    x /= vvox;
    x *= fraction[static_cast<size_t>(q) * S + s];
    const int k = v % nz;
    const int j = (v / nz) % ny;
    const int i = v / (nz * ny);
    T* rho = f + ((static_cast<size_t>(s) * nz + k) * ny + j) * nxp + i;
    double r = static_cast<double>(*rho);
    if (off) r += off[s];
    r += x;
    if (off) r -= off[s];
    *rho = static_cast<T>(r);
    *in = 0.0;
  }
}

// The amounts array sized for n agents, contents of the first
// min(n, previous n) positions kept, the rest zero.
int resize_internal(bfvm_ctx* c, int n) {
  const size_t row = sizeof(double) * c->S;
  if (n > c->cap_internal) {
    const int cap = n < 1024 ? 1024 : n;
    double* fresh = nullptr;
    const int rc = dalloc(c, reinterpret_cast<void**>(&fresh), row * cap);
    if (rc != BFVM_OK) return rc;
    BFVM_CUDA(cudaMemsetAsync(fresh, 0, row * cap, c->stream));
    if (c->d_internal && c->n_internal > 0)
      BFVM_CUDA(cudaMemcpyAsync(fresh, c->d_internal, row * c->n_internal, cudaMemcpyDeviceToDevice, c->stream));
    if (c->d_internal) {
      BFVM_CUDA(cudaStreamSynchronize(c->stream));
      dfree(c, c->d_internal);
    }
    c->d_internal = fresh;
    c->cap_internal = cap;
    ++c->version;
  } else if (n > c->n_internal) {
    BFVM_CUDA(cudaMemsetAsync(c->d_internal + static_cast<size_t>(c->S) * c->n_internal, 0,
                              row * (n - c->n_internal), c->stream));
  }
  c->n_internal = n;
  return BFVM_OK;
}

// Sorted per-step exports: from the list's net export rates when it came from
// rates, else zero (bfvm_set_agent_exports sets them).
int refresh_exports(bfvm_ctx* c) {
  const int n = c->n_agents;
  const size_t SN = static_cast<size_t>(c->S) * n;
  if (!c->d_ae1) {
    const int rc = dalloc(c, reinterpret_cast<void**>(&c->d_ae1), sizeof(double) * c->S * c->cap_agents);
    if (rc != BFVM_OK) return rc;
    ++c->version;
  }
  if (n == 0) return BFVM_OK;
  if (c->agents_from_rates) {
    const double* net_export = c->d_rates + n + 3 * SN;  // volume [n] | sec | upt | sat | exp
    export_kernel<<<static_cast<unsigned>((SN + 255) / 256), 256, 0, c->stream>>>(static_cast<long long>(SN), c->dt,
                                                                                  net_export, c->d_sample);
    BFVM_CUDA(cudaGetLastError());
    BFVM_CUDA(agents_gather_sorted(n, c->S, c->d_sorted_vals, c->d_sample, c->d_ae1, c->stream));
    note_launches(2);
  } else {
    BFVM_CUDA(cudaMemsetAsync(c->d_ae1, 0, sizeof(double) * SN, c->stream));
  }
  return BFVM_OK;
}

}  // namespace

namespace bfvm {

int tracking_after_agents(bfvm_ctx* c) {
  if (!c->track) return BFVM_OK;
  int rc = resize_internal(c, c->n_agents);
  if (rc == BFVM_OK) rc = refresh_exports(c);
  return rc;
}

}  // namespace bfvm

extern "C" {

int bfvm_set_agent_tracking(bfvm_ctx* c, int on) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  const int want = on ? 1 : 0;
  if (want == c->track) return BFVM_OK;
  c->track = want;
  ++c->version;
  if (!want) {
    c->n_internal = 0;  // turning it on again starts from zero
    return BFVM_OK;
  }
  if (c->d_voxel == nullptr) {  // no list yet: the buffers come with the first one
    c->n_internal = 0;
    return BFVM_OK;
  }
  return tracking_after_agents(c);
}

int bfvm_set_agent_exports(bfvm_ctx* c, const double* export1) {
  if (!c || (!export1 && c->n_agents > 0)) return BFVM_ERR_ARG;
  if (!c->track) return BFVM_ERR_STATE;
  DeviceGuard g(c->device);
  const int n = c->n_agents;
  if (n == 0) return BFVM_OK;
  const size_t SN = static_cast<size_t>(c->S) * n;
  BFVM_CUDA(cudaMemcpyAsync(c->d_sample, export1, sizeof(double) * SN, cudaMemcpyHostToDevice, c->stream));
  BFVM_CUDA(agents_gather_sorted(n, c->S, c->d_sorted_vals, c->d_sample, c->d_ae1, c->stream));
  note_launches(1);
  return bfvm_synchronize(c);
}

int bfvm_get_internalized(bfvm_ctx* c, double* out) {
  if (!c || (!out && c->n_internal > 0)) return BFVM_ERR_ARG;
  if (!c->track) return BFVM_ERR_STATE;
  DeviceGuard g(c->device);
  if (c->n_internal == 0) return BFVM_OK;
  BFVM_CUDA(cudaMemcpyAsync(out, c->d_internal, sizeof(double) * c->S * static_cast<size_t>(c->n_internal),
                            cudaMemcpyDeviceToHost, c->stream));
  return bfvm_synchronize(c);
}

int bfvm_set_internalized(bfvm_ctx* c, const double* in) {
  if (!c) return BFVM_ERR_ARG;
  if (!c->track) return BFVM_ERR_STATE;
  DeviceGuard g(c->device);
  if (c->n_internal == 0) return BFVM_OK;
  const size_t bytes = sizeof(double) * c->S * static_cast<size_t>(c->n_internal);
  if (in)
    BFVM_CUDA(cudaMemcpyAsync(c->d_internal, in, bytes, cudaMemcpyHostToDevice, c->stream));
  else
    BFVM_CUDA(cudaMemsetAsync(c->d_internal, 0, bytes, c->stream));
  return bfvm_synchronize(c);
}

int bfvm_release_internalized(bfvm_ctx* c, int count, const int* agents, const double* fraction) {
  if (!c || count < 0 || (count > 0 && (!agents || !fraction))) return BFVM_ERR_ARG;
  if (!c->track) return BFVM_ERR_STATE;
  DeviceGuard g(c->device);
  if (count == 0 || c->n_internal == 0) return BFVM_OK;
  for (int q = 0; q < count; ++q)
    if (agents[q] < 0 || agents[q] >= c->n_internal) return BFVM_ERR_ARG;
  // Host arrays staged through one small device buffer: agents | fraction.
  const size_t abytes = (sizeof(int) * count + 15) / 16 * 16;
  const size_t fbytes = sizeof(double) * c->S * static_cast<size_t>(count);
  void* buf = nullptr;
  int rc = dalloc(c, &buf, abytes + fbytes);
  if (rc != BFVM_OK) return rc;
  int* d_agents = static_cast<int*>(buf);
  double* d_fraction = reinterpret_cast<double*>(static_cast<char*>(buf) + abytes);
  cudaError_t e = cudaMemcpyAsync(d_agents, agents, sizeof(int) * count, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_fraction, fraction, fbytes, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    const double vvox = c->dx * c->dx * c->dx;
    const unsigned blocks = static_cast<unsigned>((c->S + 63) / 64);
    if (c->prec == BFVM_FP64)
      release_kernel<double><<<blocks, 64, 0, c->stream>>>(count, d_agents, d_fraction, c->n_agents, c->d_voxel, c->S,
                                                            c->nx, c->ny, c->nz, c->nxp, vvox, nullptr, c->d_internal,
                                                            static_cast<double*>(c->f));
    else
      release_kernel<float><<<blocks, 64, 0, c->stream>>>(count, d_agents, d_fraction, c->n_agents, c->d_voxel, c->S,
                                                           c->nx, c->ny, c->nz, c->nxp, vvox, c->d_off, c->d_internal,
                                                           static_cast<float*>(c->f));
    e = cudaGetLastError();
    note_launches(1);
  }
  rc = bfvm_synchronize(c);
  dfree(c, buf);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "biofvm_b200: bfvm_release_internalized failed: %s\n", cudaGetErrorString(e));
    return BFVM_ERR_CUDA;
  }
  return rc;
}

}  // extern "C"
