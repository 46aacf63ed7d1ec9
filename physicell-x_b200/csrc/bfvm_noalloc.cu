// bfvm_noalloc.cu -- bfvm_apply_sources_noalloc: one source/sink stage from
// agent arrays that are already in device memory, with no device allocation.
//
// Who needs it.  bfvm_set_agents + bfvm_apply_sources copy the agent list
// into per-solve buffers that grow (cudaMalloc) whenever a larger list
// arrives, and the voxel sort needs scratch of its own.  Some callers must
// not allocate at the point where they apply sources: a GPU-resident agent
// model that rebuilds its agent arrays every step inside a loop whose device
// memory was reserved up front (a fixed HBM budget with no headroom, where an
// allocation can fail mid-run or wait for the device to go idle), or code
// that runs where cudaMalloc is not allowed at all.  This entry point reads
// the caller's device arrays directly and keeps the sort scratch in one fixed
// array in the library's device image, so it calls no allocating routine.
//
// Rules for callers.
//   * At most kNoAllocMaxAgents agents per call; a longer list is rejected
//     with BFVM_ERR_ARG before any work is queued.
//   * There is one scratch array per device.  Calls on the same device must
//     not overlap in time: two host threads, or two streams whose work may run
//     concurrently, would race on the scratch and corrupt each other's sort.
//     Calls on different devices are independent.
//   * The first call on a device (n = 0 is enough) is its set-up: it looks up
//     the array's device address (cudaGetSymbolAddress, which loads this
//     module's device image and so places the array in device memory) and
//     loads the kernels later calls launch.  Make it at set-up time, before
//     the loop that must not allocate and before any stream capture begins.
//   * The looked-up address is kept per device for the life of the process.
//     After cudaDeviceReset on a device it is stale: do not call this entry
//     point again on that device after a reset.
//   * Nothing in the scratch has to start at zero: every word a call reads
//     was written earlier in the same call (keys and histograms are rebuilt
//     from the inputs), so the scratch is never cleared.
#include <cstddef>
#include <mutex>

#include "bfvm_agents.h"
#include "bfvm_ctx.h"

namespace {

constexpr int kNoAllocMaxAgents = 1 << 18;  // 262,144 agents per call
// Sort scratch for kNoAllocMaxAgents agents: four [n] key/value arrays plus
// the per-block digit histograms, 4.25 MiB.
constexpr size_t kNoAllocScratchBytes = (static_cast<size_t>(4) << 20) + (static_cast<size_t>(256) << 10);
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_sources_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on `device`, which must be the current
// device; looked up once per device.
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return BFVM_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (g_scratch_addr[device] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sources_scratch);
    if (e != cudaSuccess || p == nullptr) {
      std::fprintf(stderr, "biofvm_b200: cudaGetSymbolAddress of the sources scratch failed: %s\n",
                   cudaGetErrorString(e));
      return BFVM_ERR_CUDA;
    }
    // Load the sort and source kernels now too, so that later calls on this
    // device allocate nothing for code either.
    const cudaError_t e2 = bfvm::agents_preload_sort_kernels();
    if (e2 != cudaSuccess) {
      std::fprintf(stderr, "biofvm_b200: loading the sources kernels failed: %s\n", cudaGetErrorString(e2));
      return BFVM_ERR_CUDA;
    }
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return BFVM_OK;
}

}  // namespace

extern "C" int bfvm_apply_sources_noalloc(bfvm_ctx* c, int n, const int* voxel, const unsigned char* active,
                                          const double* c1, const double* c2, const double* e2) {
  if (!c || n < 0 || (n > 0 && (!voxel || !c1 || !c2 || !e2))) return BFVM_ERR_ARG;
  if (n > kNoAllocMaxAgents || bfvm::agent_scratch_bytes(n) > kNoAllocScratchBytes) {
    std::fprintf(stderr, "biofvm_b200: bfvm_apply_sources_noalloc takes at most %d agents (got %d)\n",
                 kNoAllocMaxAgents, n);
    return BFVM_ERR_ARG;
  }
  bfvm::DeviceGuard g(c->device);
  void* scratch = nullptr;
  const int rc = scratch_address(c->device, &scratch);
  if (rc != BFVM_OK) return rc;
  if (n == 0) return BFVM_OK;
  const unsigned* keys = nullptr;
  const int* order = nullptr;
  int launches = 0;
  BFVM_CUDA(bfvm::agents_sort(n, voxel, active, c->nx, c->ny, c->nz, scratch, c->stream, &keys, &order, &launches));
  bfvm::note_launches(launches);
  if (c->prec == BFVM_FP64)
    BFVM_CUDA(bfvm::agents_apply_sources_by_order<double>(n, keys, order, c->S, c->nx, c->ny, c->nz, c->nxp, c1, c2,
                                                          e2, nullptr, static_cast<double*>(c->f), c->stream));
  else
    BFVM_CUDA(bfvm::agents_apply_sources_by_order<float>(n, keys, order, c->S, c->nx, c->ny, c->nz, c->nxp, c1, c2,
                                                         e2, c->d_off, static_cast<float*>(c->f), c->stream));
  bfvm::note_launches(1);
  return BFVM_OK;
}
