// bfvm_ctx.h -- the state of one resident solve (the opaque bfvm_ctx of the
// C ABI) and the host helpers shared by the translation units that launch
// its kernels (single-solve steps and the batched engine).
#pragma once

#include <cstdio>
#include <unordered_map>
#include <vector>

#include "../../include/biofvm_b200.h"
#include "bfvm_internal.h"

struct bfvm_ctx {
  int device = 0;
  int nx = 0, ny = 0, nz = 0, S = 0, nxp = 0, prec = BFVM_FP64, eb = 8;
  double dx = 0, dt = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // agent lists: the constants cross to the device on copy_stream while the
  // voxel ids are sorted on stream (fork: stream -> copy_stream, join back)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // substrate groups (bfvm_set_substrate_streams): with 2, runs of steps
  // sweep the second half of the substrates on group_stream, forked from
  // stream and joined back (measured slower at cube200: default 1)
  int sub_streams = 1;
  cudaStream_t group_stream = nullptr;
  cudaEvent_t ev_gfork = nullptr, ev_gjoin = nullptr;
  void* f = nullptr;           // field, device layout
  size_t field_bytes = 0;
  // coefficients: per axis a, DR rows [S][npad_a] at dr_off[a] and CU rows
  // [S][npad_a] at cu_off[a] (bytes into d_coef); c1 as Coef<T>::C1 [S]
  void* d_coef = nullptr;
  size_t dr_off[3] = {0, 0, 0}, cu_off[3] = {0, 0, 0};
  size_t conv_off[3] = {0, 0, 0};  // int [S] per axis: AxisCoefs::conv
  void* d_c1 = nullptr;
  int screen = 0;              // SweepParams::screen of the 3-D sweeps (kScreenFast: short FP64 chain)
  int screen_exact = 0;        // 1 when no diffusion or decay rate is negative (the exactness screen applies)
  int fp64_chain = 0;          // bfvm_set_fp64_chain: 0 reference-exact, 1 short chain, 2 partitioned
  int part_min_line = -1;      // bfvm_set_partition_min_line (-1: the default of the precision)
  void* d_part = nullptr;      // partitioned-sweep coefficient rows of the three axes (chain 2)
  bfvm::PartAxis part[3] = {};
  double* d_off = nullptr;      // FP32: per-substrate field offsets [S]
  void* d_shift = nullptr;      // FP32: RN32(c2 * off) [S]
  int* d_active = nullptr;
  double* d_faces = nullptr;   // xface | yface | zface
  int* d_status = nullptr;
  int* h_status = nullptr;     // pinned host copy of d_status, read back in the same stream wait
  unsigned long long* d_tile_counter = nullptr;  // [2] per substrate group: persistent sweeps' work counter
  double* d_sums = nullptr;    // partial sums + result
  bfvm::FieldMaps maps{};
  bfvm::SweepConfig cfg{};
  // agents
  int n_agents = 0, cap_agents = 0;
  int* d_voxel = nullptr;
  unsigned char* d_agent_active = nullptr;
  double* d_c = nullptr;       // c1 | c2 | e2, [n][S] each
  double* d_rates = nullptr;   // volume [n] | sec | upt | sat | exp [n][S]
  unsigned* d_dev_voxel = nullptr;
  unsigned* d_sorted_keys = nullptr;
  int* d_sorted_vals = nullptr;
  int* d_line_off = nullptr;
  int* d_a_i = nullptr;
  double* d_ac = nullptr;      // ac1 | ac2 | ae2, [S][n] each
  int* d_nvalid = nullptr;
  int* d_agent_pos = nullptr;  // [n] sorted position of each list index
  void* d_delta = nullptr;     // bfvm_update_agents staging: idx [m] | c1, c2, e2 [m][S]
  size_t cap_delta = 0;        // bytes of d_delta
  void* d_agent_scratch = nullptr;
  double* d_sample = nullptr;
  // internalized-substrate tracking (bfvm_set_agent_tracking)
  int track = 0;
  double* d_ae1 = nullptr;      // [S][cap_agents] export per step, sorted order
  double* d_internal = nullptr; // [cap_internal][S] amounts per agent, list order
  int n_internal = 0, cap_internal = 0;
  int agents_from_rates = 0;    // the list came from bfvm_set_agents_from_rates (rates kept in d_rates)
  // 2-D LOD (bfvm_step_2d) and Dirichlet nodes (bfvm_set_dirichlet_nodes)
  std::vector<double> D, decay; // the solve's rates (host copies)
  void* d_coef2d = nullptr;     // x and y coefficient rows of the 2-D solver, laid out as d_coef
  size_t dr2_off[2] = {0, 0}, cu2_off[2] = {0, 0};
  std::vector<double> c2_2d;    // dt*decay/2 per substrate
  double* d_shift2d = nullptr;  // FP32: c2_2d * off [S]
  int* d_zero_active = nullptr; // [S] zeros: the 2-D sweeps pin no faces
  int n_nodes = 0;
  void* d_nodes = nullptr;      // long long offset [n] | double value [n][S] | uchar activation [n][S]
  // host-side mirrors
  std::vector<unsigned char> active;
  std::vector<double> faces;    // same layout as d_faces
  std::vector<double> c2;       // dt*decay/3 per substrate (thomas_constant2)
  std::vector<double> off;      // FP32 offsets currently applied to the field
  size_t device_bytes = 0;     // bytes currently allocated by dalloc
  std::unordered_map<void*, size_t> alloc_bytes;
  int version = 0;             // bumped whenever device pointers in SweepParams change
  double* d_staging = nullptr; // reference-layout field, for host uploads/downloads
  double* d_grad = nullptr;    // gradients for host reads (bfvm_compute_gradients)
  double* d_bulk = nullptr;    // bulk supply | target | uptake rates, device layout (bfvm_set_bulk_rates)
  // periodic FP64 mass-balance record (bfvm_set_mass_log): partials
  // [S][512] | ring [capacity][S] | record count (u64)
  double* d_mass = nullptr;
  int mass_every = 0, mass_capacity = 0;
  long long mass_steps = 0;    // steps since the log was enabled
  // bfvm_step's CUDA graph: kGraphSteps LOD steps captured once and replayed
  // while nothing it captured by value changes (graph_key)
  cudaGraphExec_t step_graph = nullptr;
  std::vector<long long> graph_key;
  // per-kernel timing: 4 events per recorded step
  bool timing = false;
  int timed_steps = 0;
  std::vector<cudaEvent_t> events;
};


namespace bfvm {

#define BFVM_CUDA(call)                                                                                      \
  do {                                                                                                       \
    cudaError_t e__ = (call);                                                                                \
    if (e__ != cudaSuccess) {                                                                                \
      std::fprintf(stderr, "biofvm_b200: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e__), __FILE__, \
                   __LINE__);                                                                                \
      return e__ == cudaErrorMemoryAllocation ? BFVM_ERR_OOM : BFVM_ERR_CUDA;                                \
    }                                                                                                        \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Host-transfer helpers of bfvm_capi.cu: the reference-layout staging buffer
// (allocated on first use) and the device-layout -> reference-layout copy.
int ensure_staging(bfvm_ctx* c);
int unpack_to_device_aos(bfvm_ctx* c, double* d_aos);

// bfvm_lod2d.cu: the FP32 right-hand-side shift of the 2-D solver, brought
// in line with the field offsets (no-op until the 2-D solver is set up).
int update_shift_2d(bfvm_ctx* c);

// bfvm_mass.cu: one mass-balance record of the current field, enqueued on
// the solve's stream.
int enqueue_mass_record(bfvm_ctx* c);
// The standalone source kernel of the solve's agents on stream st
// (bfvm_apply_sources on the solve's own stream), substrates [s_lo, s_hi)
// (s_hi < 0: all from s_lo).
int apply_sources_on(bfvm_ctx* c, cudaStream_t st, int s_lo = 0, int s_hi = -1);
// One LOD step of the solve (sources when asked, then the x, y and z sweeps,
// with the solve's own kernels and settings) enqueued on stream st, as
// bfvm_step launches it; used by the batched engine for members it steps
// with their own kernels.
int enqueue_step_on(bfvm_ctx* c, bool sources, cudaStream_t st);

// bfvm_capi.cu: Thomas factorization of one axis (half: 2-D constants).
void thomas_axis_host(int n, int S, const double* D, const double* decay, double dt, double dx, double* denom,
                      double* cup, double* c1, bool half);

// bfvm_tracking.cu: after a new agent list is built, bring the tracking
// buffers to its size (amounts of surviving list positions kept, new ones
// zeroed) and set the per-step exports (from the rates, else zero).
int tracking_after_agents(bfvm_ctx* c);

inline int dalloc(bfvm_ctx* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return e == cudaErrorMemoryAllocation ? BFVM_ERR_OOM : BFVM_ERR_CUDA;
  }
  c->device_bytes += bytes;
  c->alloc_bytes[*p] = bytes;
  return BFVM_OK;
}

// Free a dalloc'ed buffer (null is a no-op) and take it off the account.
inline void dfree(bfvm_ctx* c, void* p) {
  if (!p) return;
  auto it = c->alloc_bytes.find(p);
  if (it != c->alloc_bytes.end()) {
    c->device_bytes -= it->second;
    c->alloc_bytes.erase(it);
  }
  cudaFree(p);
}

inline AgentTrack track_params(const bfvm_ctx* c) {
  AgentTrack t{};
  if (!c->track || c->n_agents == 0) return t;
  t.internal = c->d_internal;
  t.order = c->d_sorted_vals;
  t.ae1 = c->d_ae1;
  t.vvox = c->dx * c->dx * c->dx;
  t.S = c->S;
  t.n = c->n_agents;
  return t;
}

template <typename T>
inline SweepParams<T> make_params(bfvm_ctx* c, bool sources) {
  SweepParams<T> p{};
  p.f = static_cast<T*>(c->f);
  p.nx = c->nx;
  p.ny = c->ny;
  p.nz = c->nz;
  p.S = c->S;
  p.nxp = c->nxp;
  const size_t S = c->S;
  const bool f32 = sizeof(T) == 4;
  using DR = typename Coef<T>::DR;
  using CU = typename Coef<T>::CU;
  p.c1 = static_cast<const typename Coef<T>::C1*>(c->d_c1);
  p.off = f32 ? c->d_off : nullptr;
  p.shift = f32 ? static_cast<const double*>(c->d_shift) : nullptr;
  p.active = c->d_active;
  p.xface = c->d_faces;
  p.yface = p.xface + 2 * S * c->nz * c->ny;
  p.zface = p.yface + 2 * S * c->nz * c->nx;
  const unsigned char* cb = static_cast<const unsigned char*>(c->d_coef);
  const int n_axis[3] = {c->nx, c->ny, c->nz};
  AxisCoefs<T>* axes[3] = {&p.ax, &p.ay, &p.az};
  for (int a = 0; a < 3; ++a) {
    axes[a]->dr = reinterpret_cast<const DR*>(cb + c->dr_off[a]);
    axes[a]->cu = reinterpret_cast<const CU*>(cb + c->cu_off[a]);
    axes[a]->npad = coef_pad(n_axis[a]);
    axes[a]->conv = reinterpret_cast<const int*>(cb + c->conv_off[a]);
  }
  if (sources && c->n_agents > 0) {
    p.line_off = c->d_line_off;
    p.a_key = c->d_sorted_keys;
    p.ac1 = c->d_ac;
    p.ac2 = c->d_ac + S * c->n_agents;
    p.ae2 = c->d_ac + 2 * S * c->n_agents;
    p.n_sorted = c->n_agents;
    if (c->track) p.track = track_params(c);
  }
  p.screen = c->screen;
  p.status = c->d_status;
  p.tile_counter = c->d_tile_counter;
  p.s_lo = 0;
  p.s_hi = c->S;
  return p;
}

}  // namespace bfvm
