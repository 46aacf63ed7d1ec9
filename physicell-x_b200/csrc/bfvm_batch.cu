// bfvm_batch.cu -- the batched engine: many resident solves of different
// shapes advanced together, one fused launch (batch_step_kernel) per LOD
// step, with the per-step sequence captured in a CUDA graph.
//
// The reference has no batched form: PhysiCell parameter sweeps run one
// process per parameter set (beta/params_run.py).  Each member here is an
// ordinary solve (bfvm_ctx) and gives the same result, bit for bit, as when
// it is stepped alone -- the fused kernel runs the same per-tile code.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "bfvm_ctx.h"

using namespace bfvm;

struct bfvm_batch {
  int prec = BFVM_FP64;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<bfvm_ctx*> members;
  // device tables (capacity `cap` members)
  int cap = 0;
  void* d_envs = nullptr;
  int* d_pre = nullptr;
  int* d_counters = nullptr;
  BatchHeader* d_hdr = nullptr;
  int* d_status = nullptr;
  std::vector<unsigned char> h_envs;
  // schedule
  int mode = 0;         // 0: one fused persistent launch per step; 1: three launches (x, y, z) per step;
                        // 2: as 1 for the members under direct_min values, the others stepped with
                        // their own kernels (enqueue_step_on) on the batch stream
  long long direct_min = 2097152;  // mode 2: N*S (voxel-substrate values) from which a member steps directly
  std::vector<bfvm_ctx*> direct;  // mode 2: the members stepped directly (set with the tables)
  int direct_launches = 0;        // their kernels per step
  // mode 2: the direct members run on up to kSideStreams side streams, forked
  // from the batch stream and joined back around each run of steps, so that
  // the members' own persistent kernels share the GPU; direct_lane[i] is the
  // side stream of direct[i] (members balanced by size)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
  cudaEvent_t fork_ev = nullptr;
  std::vector<int> direct_lane;
  int yz_chunk = 32;
  int order = 0;        // 0: members in insertion order; 1: largest first
  int ctas_per_sm = 0;  // 0: as many as fit
  int graph_steps = 16;
  // launch shape of the current tables
  size_t smem = 0;
  int grid = 0;
  int items[3] = {0, 0, 0};
  size_t axis_smem[3] = {0, 0, 0};
  bool built_sources = false;
  // The device tables are rebuilt only when the membership, the schedule, the
  // sources flag or a member's device pointers (bfvm_ctx::version) changed.
  bool dirty = true;
  std::vector<int> versions;
  // captured graph of graph_steps steps
  cudaGraphExec_t gexec = nullptr;
  size_t g_smem = 0;
  int g_grid = 0, g_cap = 0, g_steps = 0, g_mode = -1;
  int g_items[3] = {0, 0, 0};
  long long launches = 0;
  std::vector<int> env_of;  // member index -> position in the device tables
  bfvm_ctx* stall = nullptr;  // bfvm_batch_inject_stall: member whose next step's x tiles never count
};

namespace {

constexpr int kSideStreams = 8;

int sm_count_dev(int dev) {
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  return n;
}

void drop_graph(bfvm_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->g_steps = 0;
}

int ensure_capacity(bfvm_batch* b, int n) {
  if (n <= b->cap && b->d_envs) return BFVM_OK;
  const int cap = std::max(n, std::max(16, 2 * b->cap));
  const size_t env_sz = b->prec == BFVM_FP64 ? sizeof(BatchEnv<double>) : sizeof(BatchEnv<float>);
  void *envs = nullptr, *pre = nullptr, *cnt = nullptr;
  if (cudaMalloc(&envs, env_sz * cap) != cudaSuccess || cudaMalloc(&pre, sizeof(int) * 3 * (cap + 1)) != cudaSuccess ||
      cudaMalloc(&cnt, sizeof(int) * (1 + 3 * cap)) != cudaSuccess) {
    cudaGetLastError();
    if (envs) cudaFree(envs);
    if (pre) cudaFree(pre);
    if (cnt) cudaFree(cnt);
    return BFVM_ERR_OOM;
  }
  if (b->d_envs) cudaFree(b->d_envs);
  if (b->d_pre) cudaFree(b->d_pre);
  if (b->d_counters) cudaFree(b->d_counters);
  b->d_envs = envs;
  b->d_pre = static_cast<int*>(pre);
  b->d_counters = static_cast<int*>(cnt);
  b->cap = cap;
  drop_graph(b);
  return BFVM_OK;
}

template <typename T>
int build_tables(bfvm_batch* b, bool sources) {
  const int n = static_cast<int>(b->members.size());
  int rc = ensure_capacity(b, std::max(n, 1));
  if (rc != BFVM_OK) return rc;
  // mode 2: the large members step with their own kernels, outside the tables
  std::vector<int> idx;
  b->direct.clear();
  b->direct_launches = 0;
  for (int q = 0; q < n; ++q) {
    bfvm_ctx* c = b->members[q];
    if (b->mode == 2 && 1LL * c->nx * c->ny * c->nz * c->S >= b->direct_min) {
      b->direct.push_back(c);
      b->direct_launches += 3 + ((sources && c->n_agents > 0 && !c->cfg.fuse_sources) ? 1 : 0);
    } else {
      idx.push_back(q);
    }
  }
  // the direct members' side streams: the largest member first onto the
  // least loaded stream
  {
    const int K = std::min(static_cast<int>(b->direct.size()), kSideStreams);
    while (static_cast<int>(b->side.size()) < K) {
      cudaStream_t st = nullptr;
      cudaEvent_t ev = nullptr;
      BFVM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaStreamDestroy(st);
        return BFVM_ERR_CUDA;
      }
      b->side.push_back(st);
      b->side_ev.push_back(ev);
    }
    if (K > 0 && !b->fork_ev) BFVM_CUDA(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
    std::vector<int> order(b->direct.size());
    for (size_t q = 0; q < order.size(); ++q) order[q] = static_cast<int>(q);
    auto work = [&](int q) {
      const bfvm_ctx* c = b->direct[q];
      return 1LL * c->nx * c->ny * c->nz * c->S;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return work(a) > work(c); });
    std::vector<long long> load(K, 0);
    b->direct_lane.assign(b->direct.size(), 0);
    for (int q : order) {
      const int k = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
      b->direct_lane[q] = k;
      load[k] += work(q);
    }
  }
  const int nb = static_cast<int>(idx.size());
  if (b->order == 1) {
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) {
      const bfvm_ctx* x = b->members[a];
      const bfvm_ctx* y = b->members[c];
      return 1LL * x->nx * x->ny * x->nz * x->S > 1LL * y->nx * y->ny * y->nz * y->S;
    });
  }
  std::vector<BatchEnv<T>> envs(nb);
  std::vector<int> pre(3 * (b->cap + 1), 0);
  size_t smem = 1024 + 1024;
  size_t axis_smem[3] = {2048, 2048, 2048};
  int items[3] = {0, 0, 0};
  SweepConfig cfg;
  cfg.x_lines = kBatchTile;
  cfg.yz_tile = kBatchTile;
  cfg.yz_chunk = b->yz_chunk;
  for (int q = 0; q < nb; ++q) {
    bfvm_ctx* c = b->members[idx[q]];
    BatchEnv<T>& E = envs[q];
    std::memset(static_cast<void*>(&E), 0, sizeof(E));
    FieldMaps maps;
    if (encode_field_maps(&maps, c->f, c->eb, c->nx, c->ny, c->nz, c->S, c->nxp, cfg) != 0) return BFVM_ERR_CUDA;
    E.mx = maps.x;
    E.my = maps.y;
    E.mz = maps.z;
    E.p = make_params<T>(c, sources);
    const int chy_target = b->yz_chunk;
    auto rows = [chy_target](int n_line) {
      const int C = (n_line + chy_target - 1) / chy_target;
      return (n_line + C - 1) / C;
    };
    E.chy = rows(c->ny);
    E.chz = rows(c->nz);
    E.nty = (c->ny + kBatchTile - 1) / kBatchTile;
    E.ntx = (c->nx + kBatchTile - 1) / kBatchTile;
    const int tiles[3] = {E.nty * c->nz * c->S, E.ntx * c->nz * c->S, E.ntx * c->ny * c->S};
    for (int a = 0; a < 3; ++a) {
      pre[a * (b->cap + 1) + q] = items[a];
      items[a] += tiles[a];
    }
    const size_t need = batch_member_smem(c->eb, c->nx, c->ny, c->nz, b->yz_chunk);
    if (need > 227 * 1024) return BFVM_ERR_SHAPE;
    smem = std::max(smem, need);
    const int n_line[3] = {c->nx, c->ny, c->nz};
    for (int a = 0; a < 3; ++a)
      axis_smem[a] = std::max(axis_smem[a], batch_axis_smem(c->eb, a, n_line[a], b->yz_chunk));
  }
  for (int a = 0; a < 3; ++a) pre[a * (b->cap + 1) + nb] = items[a];
  b->env_of.assign(n, -1);
  for (int q = 0; q < nb; ++q) b->env_of[idx[q]] = q;
  BatchHeader hdr;
  hdr.n_env = nb;
  for (int a = 0; a < 3; ++a) hdr.n_items[a] = items[a];
  if (nb > 0)
    BFVM_CUDA(cudaMemcpyAsync(b->d_envs, envs.data(), sizeof(BatchEnv<T>) * nb, cudaMemcpyHostToDevice, b->stream));
  BFVM_CUDA(cudaMemcpyAsync(b->d_pre, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, b->stream));
  BFVM_CUDA(cudaMemcpyAsync(b->d_hdr, &hdr, sizeof(hdr), cudaMemcpyHostToDevice, b->stream));
  // the host copies above must stay alive until the copies ran
  BFVM_CUDA(cudaStreamSynchronize(b->stream));
  int occ = 0;
  BFVM_CUDA(batch_occupancy<T>(smem, &occ));
  if (occ <= 0) return BFVM_ERR_SHAPE;
  if (b->ctas_per_sm > 0 && b->ctas_per_sm < occ) occ = b->ctas_per_sm;
  const int total = items[0] + items[1] + items[2];
  const int grid = std::max(1, std::min(total, occ * sm_count_dev(b->device)));
  if (smem != b->smem || grid != b->grid) drop_graph(b);
  for (int a = 0; a < 3; ++a) {
    if (items[a] != b->items[a] || axis_smem[a] != b->axis_smem[a]) drop_graph(b);
    b->items[a] = items[a];
    b->axis_smem[a] = axis_smem[a];
  }
  b->smem = smem;
  b->grid = grid;
  b->built_sources = sources;
  drop_graph(b);  // the direct members' launches live in the graph too
  return BFVM_OK;
}

// One step of the fused schedule (schedule 0) on the batch stream.
template <typename T>
cudaError_t enqueue_fused_step(bfvm_batch* b, int stall_env) {
  cudaError_t e = cudaMemsetAsync(b->d_counters, 0, sizeof(int) * (1 + 3 * b->cap), b->stream);
  if (e != cudaSuccess) return e;
  if (stall_env >= 0) {
    e = cudaMemsetAsync(b->d_counters + 1 + stall_env, 0xC0, sizeof(int), b->stream);  // 0xC0C0C0C0 < 0
    if (e != cudaSuccess) return e;
  }
  return launch_batch_step<T>(b->d_hdr, static_cast<const BatchEnv<T>*>(b->d_envs), b->d_pre, b->cap, b->d_counters,
                              b->d_status, b->grid, b->smem, b->stream);
}

// Launches of nsteps steps on the batch stream (also used while capturing).
// Schedules 1 and 2: the batched sweeps on the batch stream; the direct
// members (schedule 2), each with all of its steps in order, on their side
// streams, forked from the batch stream before the first step and joined
// back after the last (the members are independent solves).
// stall_env >= 0 (fault injection, fused schedule only): that table entry's
// finished-x-tile counter starts far below zero, so its y tiles wait on x
// tiles that never count up and their bounded waits run out.
template <typename T>
cudaError_t enqueue_steps(bfvm_batch* b, int nsteps, int stall_env = -1) {
  if (b->mode >= 1) {
    const int K = std::min(static_cast<int>(b->direct.size()), static_cast<int>(b->side.size()));
    cudaError_t e = cudaSuccess;
    if (K > 0) {
      if ((e = cudaEventRecord(b->fork_ev, b->stream)) != cudaSuccess) return e;
      for (int k = 0; k < K; ++k)
        if ((e = cudaStreamWaitEvent(b->side[k], b->fork_ev, 0)) != cudaSuccess) return e;
    }
    for (int s = 0; s < nsteps && e == cudaSuccess; ++s)
      e = launch_batch_sweeps<T>(b->d_hdr, static_cast<const BatchEnv<T>*>(b->d_envs), b->d_pre, b->cap, b->items,
                                 b->axis_smem, b->stream);
    for (size_t q = 0; q < b->direct.size() && e == cudaSuccess; ++q) {
      cudaStream_t st = K > 0 ? b->side[b->direct_lane[q] % K] : b->stream;
      for (int s = 0; s < nsteps && e == cudaSuccess; ++s)
        if (enqueue_step_on(b->direct[q], b->built_sources, st) != BFVM_OK) e = cudaErrorLaunchFailure;
    }
    // joined even after a failed launch, so that a capture can end
    for (int k = 0; k < K; ++k) {
      cudaError_t e2 = cudaEventRecord(b->side_ev[k], b->side[k]);
      if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(b->stream, b->side_ev[k], 0);
      if (e == cudaSuccess) e = e2;
    }
    return e;
  }
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < nsteps && e == cudaSuccess; ++s) e = enqueue_fused_step<T>(b, s == 0 ? stall_env : -1);
  return e;
}

// The batched kernels of one step (the directly stepped members count their
// own launches as they enqueue them).
int kernels_per_step(const bfvm_batch* b) {
  if (b->mode == 0) return 1;
  return (b->items[0] > 0) + (b->items[1] > 0) + (b->items[2] > 0);
}

template <typename T>
int launch_one(bfvm_batch* b, int stall_env = -1) {
  BFVM_CUDA(enqueue_steps<T>(b, 1, stall_env));
  note_launches(kernels_per_step(b));
  b->launches += kernels_per_step(b) + b->direct_launches;
  return BFVM_OK;
}

template <typename T>
int capture_graph(bfvm_batch* b) {
  drop_graph(b);
  cudaGraph_t g = nullptr;
  BFVM_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  set_launch_capture(true);  // the replays count the launches
  {
    const cudaError_t e2 = enqueue_steps<T>(b, b->graph_steps);
    if (e2 != cudaSuccess) {
      set_launch_capture(false);
      cudaStreamEndCapture(b->stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return BFVM_ERR_CUDA;
    }
  }
  set_launch_capture(false);
  BFVM_CUDA(cudaStreamEndCapture(b->stream, &g));
  cudaError_t e = cudaGraphInstantiate(&b->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->gexec = nullptr;
    return BFVM_ERR_CUDA;
  }
  b->g_steps = b->graph_steps;
  b->g_smem = b->smem;
  b->g_grid = b->grid;
  b->g_cap = b->cap;
  b->g_mode = b->mode;
  for (int a = 0; a < 3; ++a) b->g_items[a] = b->items[a];
  return BFVM_OK;
}

// Order the batch stream after every member's pending work, and every
// member's later work after the batch.
int join_members(bfvm_batch* b) {
  for (bfvm_ctx* c : b->members) {
    if (c->stream == b->stream) continue;
    BFVM_CUDA(cudaEventRecord(b->ev, c->stream));
    BFVM_CUDA(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  return BFVM_OK;
}

int release_members(bfvm_batch* b) {
  BFVM_CUDA(cudaEventRecord(b->ev, b->stream));
  for (bfvm_ctx* c : b->members)
    if (c->stream != b->stream) BFVM_CUDA(cudaStreamWaitEvent(c->stream, b->ev, 0));
  return BFVM_OK;
}

template <typename T>
int step_impl(bfvm_batch* b, int nsteps, bool sources) {
  if (b->members.empty() || nsteps == 0) return BFVM_OK;
  int rc = join_members(b);
  if (rc != BFVM_OK) return rc;
  bool rebuild = b->dirty || sources != b->built_sources || b->versions.size() != b->members.size();
  for (size_t q = 0; !rebuild && q < b->members.size(); ++q) rebuild = b->versions[q] != b->members[q]->version;
  if (rebuild) {
    if ((rc = build_tables<T>(b, sources)) != BFVM_OK) return rc;
    b->versions.resize(b->members.size());
    for (size_t q = 0; q < b->members.size(); ++q) b->versions[q] = b->members[q]->version;
    b->dirty = false;
  }
  int left = nsteps;
  if (b->stall != nullptr) {
    // an injected stall applies to the first step of this call, launched alone
    const auto it = std::find(b->members.begin(), b->members.end(), b->stall);
    b->stall = nullptr;
    if (it != b->members.end() && b->mode == 0) {
      if ((rc = launch_one<T>(b, b->env_of[it - b->members.begin()])) != BFVM_OK) return rc;
      --left;
    }
  }
  if (b->graph_steps > 1 && left >= b->graph_steps) {
    if (!b->gexec || b->g_steps != b->graph_steps || b->g_smem != b->smem || b->g_grid != b->grid ||
        b->g_cap != b->cap || b->g_mode != b->mode || b->g_items[0] != b->items[0] ||
        b->g_items[1] != b->items[1] || b->g_items[2] != b->items[2]) {
      if ((rc = capture_graph<T>(b)) != BFVM_OK) return rc;
    }
    while (left >= b->g_steps) {
      BFVM_CUDA(cudaGraphLaunch(b->gexec, b->stream));
      note_launches(b->g_steps * (kernels_per_step(b) + b->direct_launches));
      b->launches += b->g_steps * (kernels_per_step(b) + b->direct_launches);
      left -= b->g_steps;
    }
  }
  for (; left > 0; --left)
    if ((rc = launch_one<T>(b)) != BFVM_OK) return rc;
  return release_members(b);
}

}  // namespace

extern "C" {

int bfvm_batch_create(int precision, int device, bfvm_batch** out) {
  if (!out || (precision != BFVM_FP64 && precision != BFVM_FP32)) return BFVM_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return BFVM_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return BFVM_ERR_NODEVICE;
  DeviceGuard g(device);
  bfvm_batch* b = new (std::nothrow) bfvm_batch();
  if (!b) return BFVM_ERR_OOM;
  b->prec = precision;
  b->device = device;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&b->d_hdr), sizeof(BatchHeader)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&b->d_status), sizeof(int)) != cudaSuccess ||
      cudaMemset(b->d_status, 0, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    bfvm_batch_destroy(b);
    return BFVM_ERR_CUDA;
  }
  *out = b;
  return BFVM_OK;
}

int bfvm_batch_destroy(bfvm_batch* b) {
  if (!b) return BFVM_ERR_ARG;
  DeviceGuard g(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  if (b->d_envs) cudaFree(b->d_envs);
  if (b->d_pre) cudaFree(b->d_pre);
  if (b->d_counters) cudaFree(b->d_counters);
  if (b->d_hdr) cudaFree(b->d_hdr);
  if (b->d_status) cudaFree(b->d_status);
  if (b->ev) cudaEventDestroy(b->ev);
  for (size_t k = 0; k < b->side.size(); ++k) {
    cudaStreamSynchronize(b->side[k]);
    cudaStreamDestroy(b->side[k]);
    cudaEventDestroy(b->side_ev[k]);
  }
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return BFVM_OK;
}

int bfvm_batch_add(bfvm_batch* b, bfvm_ctx* c) {
  if (!b || !c) return BFVM_ERR_ARG;
  if (c->prec != b->prec || c->device != b->device) return BFVM_ERR_ARG;
  if (std::find(b->members.begin(), b->members.end(), c) != b->members.end()) return BFVM_ERR_STATE;
  if (batch_member_smem(c->eb, c->nx, c->ny, c->nz, b->yz_chunk) > 227 * 1024) return BFVM_ERR_SHAPE;
  b->members.push_back(c);
  b->dirty = true;
  return BFVM_OK;
}

int bfvm_batch_remove(bfvm_batch* b, bfvm_ctx* c) {
  if (!b || !c) return BFVM_ERR_ARG;
  auto it = std::find(b->members.begin(), b->members.end(), c);
  if (it == b->members.end()) return BFVM_ERR_STATE;
  DeviceGuard g(b->device);
  // the member's next work must follow whatever the batch already queued
  BFVM_CUDA(cudaEventRecord(b->ev, b->stream));
  BFVM_CUDA(cudaStreamWaitEvent(c->stream, b->ev, 0));
  b->members.erase(it);
  b->dirty = true;
  return BFVM_OK;
}

int bfvm_batch_size(bfvm_batch* b) { return b ? static_cast<int>(b->members.size()) : 0; }

int bfvm_batch_step(bfvm_batch* b, int nsteps, int flags) {
  if (!b || nsteps < 0) return BFVM_ERR_ARG;
  DeviceGuard g(b->device);
  const bool sources = (flags & BFVM_STEP_SOURCES) != 0;
  return b->prec == BFVM_FP64 ? step_impl<double>(b, nsteps, sources) : step_impl<float>(b, nsteps, sources);
}

int bfvm_batch_synchronize(bfvm_batch* b) {
  if (!b) return BFVM_ERR_ARG;
  DeviceGuard g(b->device);
  BFVM_CUDA(cudaStreamSynchronize(b->stream));
  int st = 0;
  BFVM_CUDA(cudaMemcpy(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  int member_rc = BFVM_OK;
  for (bfvm_ctx* c : b->members) {
    const int rc = bfvm_synchronize(c);
    if (rc != BFVM_OK) member_rc = rc;
  }
  if (st != 0) {
    cudaMemset(b->d_status, 0, sizeof(int));
    return BFVM_ERR_TIMEOUT;
  }
  return member_rc;
}

void* bfvm_batch_stream(bfvm_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

int bfvm_batch_inject_stall(bfvm_batch* b, bfvm_ctx* c) {
  if (!b || !c) return BFVM_ERR_ARG;
  if (std::find(b->members.begin(), b->members.end(), c) == b->members.end()) return BFVM_ERR_STATE;
  if (b->mode != 0) return BFVM_ERR_STATE;
  b->stall = c;
  return BFVM_OK;
}

int bfvm_batch_set_schedule(bfvm_batch* b, int mode, int yz_chunk, int order, int ctas_per_sm, int graph_steps) {
  if (!b || mode < 0 || mode > 2 || yz_chunk < 1 || yz_chunk > 256 || order < 0 || order > 1 || ctas_per_sm < 0 ||
      graph_steps < 1 || graph_steps > 1024)
    return BFVM_ERR_ARG;
  for (bfvm_ctx* c : b->members)
    if (batch_member_smem(c->eb, c->nx, c->ny, c->nz, yz_chunk) > 227 * 1024) return BFVM_ERR_SHAPE;
  b->mode = mode;
  b->yz_chunk = yz_chunk;
  b->order = order;
  b->ctas_per_sm = ctas_per_sm;
  b->graph_steps = graph_steps;
  b->dirty = true;
  drop_graph(b);
  return BFVM_OK;
}

int bfvm_batch_set_direct_threshold(bfvm_batch* b, long long values) {
  if (!b || values < 1) return BFVM_ERR_ARG;
  if (values != b->direct_min) {
    b->direct_min = values;
    b->dirty = true;
    drop_graph(b);
  }
  return BFVM_OK;
}

int bfvm_batch_get_direct_threshold(bfvm_batch* b, long long* values) {
  if (!b || !values) return BFVM_ERR_ARG;
  *values = b->direct_min;
  return BFVM_OK;
}

int bfvm_batch_get_schedule(bfvm_batch* b, int* mode, int* yz_chunk, int* order, int* ctas_per_sm,
                            int* graph_steps) {
  if (!b) return BFVM_ERR_ARG;
  if (mode) *mode = b->mode;
  if (yz_chunk) *yz_chunk = b->yz_chunk;
  if (order) *order = b->order;
  if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
  if (graph_steps) *graph_steps = b->graph_steps;
  return BFVM_OK;
}

// Time `trial_steps` fused steps under each candidate schedule and keep the
// fastest.  The fields (and the agents' internalized amounts of tracking
// solves) are saved before and restored after the trials, so tuning leaves
// the solves exactly as it found them (and every schedule computes the same
// bits anyway).
int bfvm_batch_autotune(bfvm_batch* b, int flags, int trial_steps, double* best_ms_per_step) {
  if (!b || trial_steps < 1) return BFVM_ERR_ARG;
  if (b->members.empty()) return BFVM_OK;
  DeviceGuard g(b->device);
  int rc = bfvm_batch_synchronize(b);
  if (rc != BFVM_OK) return rc;
  std::vector<void*> saved(b->members.size(), nullptr);
  auto internal_bytes = [](const bfvm_ctx* c) {
    return c->track && c->d_internal ? sizeof(double) * c->S * static_cast<size_t>(c->n_internal) : size_t{0};
  };
  for (size_t q = 0; q < b->members.size(); ++q) {
    bfvm_ctx* c = b->members[q];
    if (cudaMalloc(&saved[q], c->field_bytes + internal_bytes(c)) != cudaSuccess) {
      cudaGetLastError();
      for (void* p : saved)
        if (p) cudaFree(p);
      return BFVM_ERR_OOM;
    }
    BFVM_CUDA(cudaMemcpyAsync(saved[q], c->f, c->field_bytes, cudaMemcpyDeviceToDevice, b->stream));
    if (internal_bytes(c))
      BFVM_CUDA(cudaMemcpyAsync(static_cast<char*>(saved[q]) + c->field_bytes, c->d_internal, internal_bytes(c),
                                cudaMemcpyDeviceToDevice, b->stream));
  }
  struct Cand {
    int mode, yz_chunk, order, ctas;
    long long direct_min;
  };
  std::vector<Cand> cands;
  for (int ch : {16, 32, 64}) {
    cands.push_back({1, ch, 0, 0, b->direct_min});
    for (int ord : {0, 1})
      for (int ctas : {0, 8, 4}) cands.push_back({0, ch, ord, ctas, b->direct_min});
  }
  // mode 2: every member, or members from 32^3, 64^3 or 128^3 voxel-substrate
  // values, step directly (their own kernels on the side streams)
  for (long long dm : {1LL, 32768LL, 262144LL, 2097152LL})
    for (int ch : {32, 64}) cands.push_back({2, ch, 0, 0, dm});
  const int keep_graph = b->graph_steps;
  const long long keep_direct = b->direct_min;
  double best = 1e30;
  Cand best_c{b->mode, b->yz_chunk, b->order, b->ctas_per_sm, b->direct_min};
  cudaEvent_t e0, e1;
  BFVM_CUDA(cudaEventCreate(&e0));
  BFVM_CUDA(cudaEventCreate(&e1));
  for (const Cand& cd : cands) {
    b->direct_min = cd.direct_min;
    if (bfvm_batch_set_schedule(b, cd.mode, cd.yz_chunk, cd.order, cd.ctas, 1) != BFVM_OK) continue;
    if ((rc = bfvm_batch_step(b, 1, flags)) != BFVM_OK) break;  // warm-up (also builds the tables)
    cudaEventRecord(e0, b->stream);
    if ((rc = bfvm_batch_step(b, trial_steps, flags)) != BFVM_OK) break;
    cudaEventRecord(e1, b->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double per = ms / trial_steps;
    if (per < best) {
      best = per;
      best_c = cd;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (size_t q = 0; q < b->members.size(); ++q) {
    bfvm_ctx* c = b->members[q];
    cudaMemcpyAsync(c->f, saved[q], c->field_bytes, cudaMemcpyDeviceToDevice, b->stream);
    if (internal_bytes(c))
      cudaMemcpyAsync(c->d_internal, static_cast<char*>(saved[q]) + c->field_bytes, internal_bytes(c),
                      cudaMemcpyDeviceToDevice, b->stream);
  }
  cudaStreamSynchronize(b->stream);
  for (void* p : saved) cudaFree(p);
  release_members(b);
  if (rc != BFVM_OK) {
    b->direct_min = keep_direct;
    return rc;
  }
  b->direct_min = best_c.direct_min;
  bfvm_batch_set_schedule(b, best_c.mode, best_c.yz_chunk, best_c.order, best_c.ctas, keep_graph);
  if (best_ms_per_step) *best_ms_per_step = best;
  return BFVM_OK;
}

}  // extern "C"
