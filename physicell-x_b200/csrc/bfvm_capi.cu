// bfvm_capi.cu -- the C ABI (include/biofvm_b200.h): one resident
// microenvironment solve per handle.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/biofvm_b200.h"
#include "bfvm_agents.h"
#include "bfvm_ctx.h"
#include "bfvm_internal.h"

using namespace bfvm;

namespace bfvm {

static std::atomic<long long> g_launches{0};
// Set while this thread captures a CUDA graph: captured launches are counted
// when the graph is launched, not when they are recorded.
static thread_local bool t_capturing = false;
void set_launch_capture(bool on) { t_capturing = on; }
void note_launches(int n) {
  if (!t_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}

// Thomas factorization of one axis, FP64, operation by operation as in
// diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING
// (BioFVM/BioFVM_solvers.cpp:196-329, one rank): outputs [n][S] like the
// reference's thomas_denom*/thomas_c* and c1[S] = thomas_constant1.
// Contractions are written out with std::fma (this file is compiled with
// -ffp-contract=off), matching the reference's g++ FMA contraction of axpy.
// half: the 2-D solver's constants (diffusion_decay_solver__constant_coefficients_LOD_2D,
// :1696-1707: constant2 = decay; *= dt; *= 0.5), otherwise the same steps.
void thomas_axis_host(int n, int S, const double* D, const double* decay, double dt, double dx, double* denom,
                      double* cup, double* c1, bool half) {
  for (int d = 0; d < S; ++d) {
    double k1 = D[d];
    k1 *= dt;
    k1 /= dx;
    k1 /= dx;
    const double k1a = k1 * -1.0;
    double k2 = decay[d];
    k2 *= dt;
    if (half)
      k2 *= 0.5;
    else
      k2 /= 3.0;
    double k3 = 1.0;
    k3 += k1;
    k3 += k1;
    k3 += k2;
    double k3a = 1.0;
    k3a += k1;
    k3a += k2;
    c1[d] = k1;
    for (int i = 0; i < n; ++i) {
      cup[static_cast<size_t>(i) * S + d] = k1a;
      denom[static_cast<size_t>(i) * S + d] = k3;
    }
    denom[d] = k3a;
    denom[static_cast<size_t>(n - 1) * S + d] = k3a;
    if (n == 1) {
      double v = 1.0;
      v += k2;
      denom[d] = v;
    }
    cup[d] /= denom[d];
    for (int i = 1; i < n; ++i) {
      const size_t a = static_cast<size_t>(i) * S + d, b = static_cast<size_t>(i - 1) * S + d;
      denom[a] = std::fma(k1, cup[b], denom[a]);
      cup[a] /= denom[a];
    }
  }
}

}  // namespace bfvm


namespace {

constexpr int kMaxTimedSteps = 4096;
constexpr int kStepEvents = 5;  // timing events per recorded step (enqueue_step)
// LOD steps per captured CUDA graph of bfvm_step (four launches each).
constexpr int kGraphSteps = 16;

int part_min_line(const bfvm_ctx* c) {
  return c->part_min_line >= 0 ? c->part_min_line : (c->eb == 8 ? kPartMinLine64 : kPartMinLine32);
}

// Everything a captured step holds by value: the kernels' parameters are
// built from these (device pointers change only with c->version), the
// launch shapes from the sweep configuration.
std::vector<long long> step_key(const bfvm_ctx* c, bool sources) {
  const SweepConfig& g = c->cfg;
  return {c->version, sources ? 1 : 0, c->n_agents, c->track, c->sub_streams, g.x_lines, g.yz_tile, g.yz_chunk, g.persistent,
          g.fuse_sources, g.tmem, part_min_line(c), static_cast<long long>(reinterpret_cast<uintptr_t>(c->d_internal)),
          static_cast<long long>(reinterpret_cast<uintptr_t>(c->d_ae1))};
}

void drop_step_graph(bfvm_ctx* c) {
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
  c->graph_key.clear();
}

// Whether the y (axis 1) or z (axis 2) sweep runs partitioned: chain 2, a
// line of at least part_min_line voxels, and a tile that fits one CTA.
bool use_part(const bfvm_ctx* c, int axis) {
  const int n = axis == 1 ? c->ny : c->nz;
  return c->fp64_chain == 2 && n >= part_min_line(c) && (n + kRingRows - 1) / kRingRows <= kPartMaxChunks &&
         part_smem_bytes(c->eb, n) <= 227 * 1024;
}

// The launches of one LOD step on c->stream (also while capturing): the
// standalone source kernel (unless fused or without agents), then the x, y
// and z sweeps, over the substrates [p.s_lo, p.s_hi); per-step timing events
// when ev is given (kStepEvents: before the sources, before the x sweep,
// after it, after y, after z).
template <typename T>
int enqueue_step(bfvm_ctx* c, const SweepParams<T>& p, bool standalone, cudaEvent_t* ev,
                 cudaStream_t st = nullptr) {
  if (st == nullptr) st = c->stream;
  if (ev) BFVM_CUDA(cudaEventRecord(ev[0], st));
  if (standalone) {
    const int rc = apply_sources_on(c, st, p.s_lo, p.s_hi);
    if (rc != BFVM_OK) return rc;
  }
  if (ev) BFVM_CUDA(cudaEventRecord(ev[1], st));
  BFVM_CUDA(launch_sweep_x<T>(c->maps, p, c->cfg, st));
  if (ev) BFVM_CUDA(cudaEventRecord(ev[2], st));
  if (use_part(c, 1))
    BFVM_CUDA((launch_part<T, 1>(c->maps.ry, p, c->part[1], st)));
  else
    BFVM_CUDA(launch_sweep_y<T>(c->maps, p, c->cfg, st));
  if (ev) BFVM_CUDA(cudaEventRecord(ev[3], st));
  if (use_part(c, 2))
    BFVM_CUDA((launch_part<T, 2>(c->maps.rz, p, c->part[2], st)));
  else
    BFVM_CUDA(launch_sweep_z<T>(c->maps, p, c->cfg, st));
  if (ev) BFVM_CUDA(cudaEventRecord(ev[4], st));
  note_launches(3);
  return BFVM_OK;
}

// Whether runs of steps split the substrates into two groups on two streams.
// Every launch of a step touches only its own substrates (the sources, the
// sweeps, their pins), so the two groups are independent problems; each
// persistent sweep leaves SMs idle while its last tiles finish, and the
// other group's kernels take them.  Not while timing single kernels.
bool use_groups(const bfvm_ctx* c) { return c->sub_streams == 2 && c->S >= 2 && !c->timing; }

// nsteps LOD steps on c->stream: one group, or the substrates [0, h) on
// c->stream and [h, S) on c->group_stream (its own tile counter), forked and
// joined around the whole run so that neither group waits on the other.
template <typename T>
int enqueue_steps(bfvm_ctx* c, const SweepParams<T>& p, bool standalone, int nsteps) {
  if (nsteps <= 0) return BFVM_OK;
  if (!use_groups(c)) {
    for (int s = 0; s < nsteps; ++s) {
      const int rc = enqueue_step<T>(c, p, standalone, nullptr);
      if (rc != BFVM_OK) return rc;
    }
    return BFVM_OK;
  }
  const int h = (c->S + 1) / 2;
  SweepParams<T> pa = p, pb = p;
  pa.s_lo = 0;
  pa.s_hi = h;
  pb.s_lo = h;
  pb.s_hi = c->S;
  pb.tile_counter = c->d_tile_counter + 2;
  BFVM_CUDA(cudaEventRecord(c->ev_gfork, c->stream));
  BFVM_CUDA(cudaStreamWaitEvent(c->group_stream, c->ev_gfork, 0));
  int rc = BFVM_OK;
  for (int s = 0; s < nsteps && rc == BFVM_OK; ++s) rc = enqueue_step<T>(c, pa, standalone, nullptr, c->stream);
  for (int s = 0; s < nsteps && rc == BFVM_OK; ++s) rc = enqueue_step<T>(c, pb, standalone, nullptr, c->group_stream);
  // joined even after a failed launch, so that a capture can end
  BFVM_CUDA(cudaEventRecord(c->ev_gjoin, c->group_stream));
  BFVM_CUDA(cudaStreamWaitEvent(c->stream, c->ev_gjoin, 0));
  return rc;
}

// Capture kGraphSteps steps into c->step_graph.  The caller has run at least
// one step uncaptured since the key last changed, so every host-side set-up
// of the launches (kernel attributes, occupancy lookups) is cached already.
template <typename T>
int capture_step_graph(bfvm_ctx* c, const SweepParams<T>& p, bool standalone, const std::vector<long long>& key) {
  drop_step_graph(c);
  cudaGraph_t g = nullptr;
  BFVM_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  t_capturing = true;
  {
    const int rc = enqueue_steps<T>(c, p, standalone, kGraphSteps);
    if (rc != BFVM_OK) {
      t_capturing = false;
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc;
    }
  }
  t_capturing = false;
  BFVM_CUDA(cudaStreamEndCapture(c->stream, &g));
  const cudaError_t e = cudaGraphInstantiate(&c->step_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->step_graph = nullptr;
    return BFVM_ERR_CUDA;
  }
  c->graph_key = key;
  return BFVM_OK;
}

template <typename T>
int run_steps_plain(bfvm_ctx* c, int nsteps, bool sources) {
  const bool standalone = sources && c->n_agents > 0 && !c->cfg.fuse_sources;
  const SweepParams<T> p = make_params<T>(c, sources && !standalone);
  // Runs of steps replay a captured graph of kGraphSteps steps (the same
  // launches, so the same bits), which removes most of the per-launch host
  // cost on small grids.  Not while timing per step, nor on a stream the
  // caller is capturing already (the steps then go into the caller's graph).
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BFVM_CUDA(cudaStreamIsCapturing(c->stream, &cap));
  if (!c->timing && cap == cudaStreamCaptureStatusNone && nsteps > kGraphSteps) {
    const std::vector<long long> key = step_key(c, sources);
    int left = nsteps;
    if (c->step_graph == nullptr || c->graph_key != key) {
      int rc = enqueue_steps<T>(c, p, standalone, 1);  // the uncaptured warm step
      if (rc != BFVM_OK) return rc;
      --left;
      if ((rc = capture_step_graph<T>(c, p, standalone, key)) != BFVM_OK) return rc;
    }
    const int per_step = (3 + (standalone ? 1 : 0)) * (use_groups(c) ? 2 : 1);
    for (; left >= kGraphSteps; left -= kGraphSteps) {
      BFVM_CUDA(cudaGraphLaunch(c->step_graph, c->stream));
      note_launches(kGraphSteps * per_step);
    }
    return enqueue_steps<T>(c, p, standalone, left);
  }
  if (!c->timing) return enqueue_steps<T>(c, p, standalone, nsteps);
  for (int s = 0; s < nsteps; ++s) {
    cudaEvent_t* ev = nullptr;
    if (c->timing && c->timed_steps < kMaxTimedSteps) {
      const size_t need = kStepEvents * static_cast<size_t>(c->timed_steps + 1);
      while (c->events.size() < need) {
        cudaEvent_t e;
        BFVM_CUDA(cudaEventCreate(&e));
        c->events.push_back(e);
      }
      ev = &c->events[kStepEvents * static_cast<size_t>(c->timed_steps)];
      ++c->timed_steps;
    }
    const int rc = enqueue_step<T>(c, p, standalone, ev);
    if (rc != BFVM_OK) return rc;
  }
  return BFVM_OK;
}

// nsteps LOD steps; with the mass-balance log on, a record after every
// mass_every-th step since the log was enabled.
template <typename T>
int run_steps(bfvm_ctx* c, int nsteps, bool sources) {
  if (c->mass_every <= 0) return run_steps_plain<T>(c, nsteps, sources);
  int left = nsteps;
  while (left > 0) {
    const int to_record = static_cast<int>(c->mass_every - c->mass_steps % c->mass_every);
    const int seg = left < to_record ? left : to_record;
    int rc = run_steps_plain<T>(c, seg, sources);
    if (rc != BFVM_OK) return rc;
    c->mass_steps += seg;
    left -= seg;
    if (c->mass_steps % c->mass_every == 0 && (rc = enqueue_mass_record(c)) != BFVM_OK) return rc;
  }
  return BFVM_OK;
}

bool config_fits(int eb, int nx, int ny, int nz, const SweepConfig& cfg) {
  const size_t lim = 227 * 1024;
  return sweep_x_smem(eb, nx, cfg) <= lim && sweep_yz_smem(eb, ny, cfg) <= lim && sweep_yz_smem(eb, nz, cfg) <= lim;
}

// Default launch shape: 32-line tiles, shrunk (keeping whole 128-byte rows)
// until a CTA's staged tile fits in shared memory.
bool pick_config(int eb, int nx, int ny, int nz, SweepConfig* cfg) {
  SweepConfig c;
  const int min_tile = 128 / eb;
  const size_t lim = 227 * 1024;
  while (!config_fits(eb, nx, ny, nz, c)) {
    bool changed = false;
    if (sweep_x_smem(eb, nx, c) > lim && c.x_lines > 8) {
      c.x_lines /= 2;
      changed = true;
    }
    if ((sweep_yz_smem(eb, ny, c) > lim || sweep_yz_smem(eb, nz, c) > lim) &&
        c.yz_tile > min_tile) {
      c.yz_tile /= 2;
      changed = true;
    }
    if (!changed) return false;
  }
  *cfg = c;
  return true;
}

// Coefficient storage of one precision: sizes of the DR/CU rows and the
// host-side packing (padding entries are neutral: a unit denominator and a
// -0 upper diagonal).
size_t coef_bytes(const bfvm_ctx* c, size_t* dr_off, size_t* cu_off, size_t* conv_off = nullptr) {
  const size_t S = c->S;
  const size_t dr_sz = c->prec == BFVM_FP64 ? sizeof(double2) : sizeof(double);
  const size_t cu_sz = sizeof(double);
  const int n_axis[3] = {c->nx, c->ny, c->nz};
  size_t o = 0;
  for (int a = 0; a < 3; ++a) {
    const size_t rows = S * coef_pad(n_axis[a]);
    dr_off[a] = o;
    o += rows * dr_sz;
    o = (o + 255) & ~size_t(255);
    cu_off[a] = o;
    o += rows * cu_sz;
    o = (o + 255) & ~size_t(255);
  }
  // each axis's first converged index per substrate (AxisCoefs::conv)
  for (int a = 0; a < 3; ++a) {
    if (conv_off) conv_off[a] = o;
    o += S * sizeof(int);
  }
  return (o + 255) & ~size_t(255);
}

// The first index from which a factorized row is constant: the constant-
// coefficient factorization d_i = fma(c1, c_{i-1}, k3), c_i = -c1 / d_i is a
// contraction that reaches a fixed point in FP64 after a few to a few dozen
// entries (4 for D dt/dx^2 = 0.01, 57 for 10), after which every entry up to
// the line's second-to-last is bit-identical.  Returns the smallest i such
// that entries i .. n-2 of both rows (as uploaded) equal entry n-2; n when
// the line is shorter than 3.
template <typename DR>
static int converged_from(const DR* dr, const double* cu, int n) {
  if (n < 3) return n;
  const int e = n - 2;
  int i = e;
  while (i > 0 && std::memcmp(&dr[i - 1], &dr[e], sizeof(DR)) == 0 &&
         std::memcmp(&cu[i - 1], &cu[e], sizeof(double)) == 0)
    --i;
  return i;
}

int upload_coefficients(bfvm_ctx* c, const double* D, const double* decay) {
  const int S = c->S;
  c->D.assign(D, D + S);
  c->decay.assign(decay, decay + S);
  c->screen_exact = 1;
  for (int s = 0; s < S; ++s)
    if (!(D[s] >= 0.0) || !(decay[s] >= 0.0)) c->screen_exact = 0;
  const bool fast = c->prec == BFVM_FP64 && c->fp64_chain >= 1;
  // 2: the short chain (kScreenFast); under chain 2 the other kernels that
  // step this solve (the batched engine) run the short chain too
  c->screen = c->fp64_chain >= 1 ? 2 : c->screen_exact;
  const int n_axis[3] = {c->nx, c->ny, c->nz};
  size_t dr_off[3], cu_off[3], conv_off[3];
  const size_t bytes = coef_bytes(c, dr_off, cu_off, conv_off);
  std::vector<unsigned char> host(bytes, 0);
  std::vector<double> c1(S);
  for (int ax = 0; ax < 3; ++ax) {
    const int n = n_axis[ax];
    const int np = coef_pad(n);
    std::vector<double> dn(static_cast<size_t>(n) * S), cu(static_cast<size_t>(n) * S);
    thomas_axis_host(n, S, D, decay, c->dt, c->dx, dn.data(), cu.data(), c1.data(), false);
    for (int s = 0; s < S; ++s)
      for (int i = 0; i < np; ++i) {
        const size_t q = static_cast<size_t>(s) * np + i;
        const bool in = i < n;
        const double d = in ? dn[static_cast<size_t>(i) * S + s] : 1.0;
        const double r = 1.0 / d;  // RN(1/d), IEEE double division
        const double u = in ? cu[static_cast<size_t>(i) * S + s] : -0.0;
        if (c->prec == BFVM_FP64) {
          // reference-exact chain: {d, RN(1/d)}; short chain: {RN(c1 * RN(1/d)), RN(1/d)}
          const double first = fast ? c1[s] * r : d;
          reinterpret_cast<double2*>(host.data() + dr_off[ax])[q] = make_double2(first, r);
        } else {
          reinterpret_cast<double*>(host.data() + dr_off[ax])[q] = r;
        }
        reinterpret_cast<double*>(host.data() + cu_off[ax])[q] = u;
      }
    int* conv = reinterpret_cast<int*>(host.data() + conv_off[ax]);
    for (int s = 0; s < S; ++s) {
      const size_t r0 = static_cast<size_t>(s) * np;
      const double* cur = reinterpret_cast<const double*>(host.data() + cu_off[ax]) + r0;
      conv[s] = c->prec == BFVM_FP64
                    ? converged_from(reinterpret_cast<const double2*>(host.data() + dr_off[ax]) + r0, cur, n)
                    : converged_from(reinterpret_cast<const double*>(host.data() + dr_off[ax]) + r0, cur, n);
    }
  }
  BFVM_CUDA(cudaMemcpy(c->d_coef, host.data(), bytes, cudaMemcpyHostToDevice));
  for (int a = 0; a < 3; ++a) {
    c->dr_off[a] = dr_off[a];
    c->cu_off[a] = cu_off[a];
    c->conv_off[a] = conv_off[a];
  }
  BFVM_CUDA(cudaMemcpy(c->d_c1, c1.data(), S * sizeof(double), cudaMemcpyHostToDevice));
  // thomas_constant2 = decay; *= dt; /= 3 (BioFVM_solvers.cpp:208-209)
  c->c2.assign(S, 0.0);
  for (int s = 0; s < S; ++s) {
    double k2 = decay[s];
    k2 *= c->dt;
    k2 /= 3.0;
    c->c2[s] = k2;
  }
  return BFVM_OK;
}

// The partitioned sweeps' coefficient rows of the three axes (see PartAxis):
// products formed in long double from the FP64 factors and rounded once.
int upload_part_coefficients(bfvm_ctx* c) {
  const int S = c->S;
  const int n_axis[3] = {c->nx, c->ny, c->nz};
  size_t off[3][4];
  size_t bytes = 0;
  for (int a = 0; a < 3; ++a) {
    const size_t rows = static_cast<size_t>(S) * coef_pad(n_axis[a]);
    off[a][0] = bytes;
    bytes += rows * 16;  // ra
    off[a][1] = bytes;
    bytes += rows * 16;  // pg
    off[a][2] = bytes;
    bytes += rows * 8;   // q
    off[a][3] = bytes;
    bytes += static_cast<size_t>(S) * kPartWarps * 16;  // ag
    bytes = (bytes + 255) & ~size_t(255);
  }
  std::vector<unsigned char> host(bytes, 0);
  std::vector<double> c1(S);
  for (int a = 0; a < 3; ++a) {
    const int n = n_axis[a];
    const int np = coef_pad(n);
    const int mseg = (n + kPartWarps - 1) / kPartWarps;
    std::vector<double> dn(static_cast<size_t>(n) * S), cu(static_cast<size_t>(n) * S);
    thomas_axis_host(n, S, c->D.data(), c->decay.data(), c->dt, c->dx, dn.data(), cu.data(), c1.data(), false);
    double2* ra = reinterpret_cast<double2*>(host.data() + off[a][0]);
    double2* pg = reinterpret_cast<double2*>(host.data() + off[a][1]);
    double* q = reinterpret_cast<double*>(host.data() + off[a][2]);
    double2* ag = reinterpret_cast<double2*>(host.data() + off[a][3]);
    for (int s = 0; s < S; ++s) {
      std::vector<double> av(n), gv(n);
      for (int i = 0; i < n; ++i) {
        const double r = 1.0 / dn[static_cast<size_t>(i) * S + s];
        av[i] = i == 0 ? 0.0 : c1[s] * r;
        gv[i] = i < n - 1 ? -cu[static_cast<size_t>(i) * S + s] : 0.0;
        ra[static_cast<size_t>(s) * np + i] = make_double2(r, av[i]);
      }
      for (int w = 0; w < kPartWarps; ++w) {
        const int lo = w * mseg, hi = std::min(n, lo + mseg);
        long double pa = 1.0L, pq = 1.0L;
        for (int i = lo; i < hi; ++i) {
          pa *= static_cast<long double>(av[i]);
          pg[static_cast<size_t>(s) * np + i] = make_double2(static_cast<double>(pa), gv[i]);
        }
        for (int i = hi - 1; i >= lo; --i) {
          pq *= static_cast<long double>(gv[i]);
          q[static_cast<size_t>(s) * np + i] = static_cast<double>(pq);
        }
        ag[static_cast<size_t>(s) * kPartWarps + w] = make_double2(static_cast<double>(pa), static_cast<double>(pq));
      }
    }
  }
  if (c->d_part) dfree(c, c->d_part);
  c->d_part = nullptr;
  int rc = dalloc(c, &c->d_part, bytes);
  if (rc != BFVM_OK) return rc;
  BFVM_CUDA(cudaMemcpy(c->d_part, host.data(), bytes, cudaMemcpyHostToDevice));
  const unsigned char* b = static_cast<const unsigned char*>(c->d_part);
  for (int a = 0; a < 3; ++a) {
    c->part[a].ra = reinterpret_cast<const double2*>(b + off[a][0]);
    c->part[a].pg = reinterpret_cast<const double2*>(b + off[a][1]);
    c->part[a].q = reinterpret_cast<const double*>(b + off[a][2]);
    c->part[a].ag = reinterpret_cast<const double2*>(b + off[a][3]);
    c->part[a].mseg = (n_axis[a] + kPartWarps - 1) / kPartWarps;
    c->part[a].npad = coef_pad(n_axis[a]);
  }
  return BFVM_OK;
}

size_t face_elems(const bfvm_ctx* c) {
  return 2ull * c->S * (static_cast<size_t>(c->nz) * c->ny + static_cast<size_t>(c->nz) * c->nx +
                        static_cast<size_t>(c->ny) * c->nx);
}

int free_agents(bfvm_ctx* c) {
  dfree(c, c->d_voxel);
  dfree(c, c->d_agent_active);
  dfree(c, c->d_c);
  dfree(c, c->d_rates);
  dfree(c, c->d_dev_voxel);
  dfree(c, c->d_sorted_keys);
  dfree(c, c->d_sorted_vals);
  dfree(c, c->d_a_i);
  dfree(c, c->d_ac);
  dfree(c, c->d_agent_scratch);
  dfree(c, c->d_sample);
  dfree(c, c->d_agent_pos);
  c->d_agent_pos = nullptr;
  dfree(c, c->d_ae1);
  c->d_ae1 = nullptr;
  c->d_voxel = nullptr;
  c->d_agent_active = nullptr;
  c->d_c = c->d_rates = c->d_ac = c->d_sample = nullptr;
  c->d_dev_voxel = c->d_sorted_keys = nullptr;
  c->d_sorted_vals = c->d_a_i = nullptr;
  c->d_agent_scratch = nullptr;
  c->cap_agents = 0;
  ++c->version;
  return BFVM_OK;
}

int ensure_agent_capacity(bfvm_ctx* c, int n) {
  if (n <= c->cap_agents && c->d_voxel != nullptr) return BFVM_OK;
  free_agents(c);
  const int cap = n < 1024 ? 1024 : n;
  const size_t S = c->S;
  int rc = BFVM_OK;
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_voxel), sizeof(int) * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_agent_active), cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_c), sizeof(double) * 3 * S * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_rates), sizeof(double) * (1 + 4 * S) * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_dev_voxel), sizeof(unsigned) * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_sorted_keys), sizeof(unsigned) * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_sorted_vals), sizeof(int) * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_a_i), sizeof(int) * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_ac), sizeof(double) * 3 * S * cap);
  if (rc == BFVM_OK) rc = dalloc(c, &c->d_agent_scratch, agent_scratch_bytes(cap));
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_sample), sizeof(double) * S * cap);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_agent_pos), sizeof(int) * cap);
  if (rc != BFVM_OK) {
    free_agents(c);
    return rc;
  }
  c->cap_agents = cap;
  return BFVM_OK;
}

int build_agents(bfvm_ctx* c, int n, cudaEvent_t constants_ready = nullptr) {
  AgentBuild b{};
  b.constants_ready = constants_ready;
  b.n = n;
  b.S = c->S;
  b.nx = c->nx;
  b.ny = c->ny;
  b.nz = c->nz;
  b.voxel = c->d_voxel;
  b.active = c->d_agent_active;
  const size_t S = c->S;
  b.c1 = c->d_c;
  b.c2 = c->d_c + S * n;
  b.e2 = c->d_c + 2 * S * n;
  b.scratch = c->d_agent_scratch;
  b.dev_voxel = c->d_dev_voxel;
  b.sorted_keys = c->d_sorted_keys;
  b.sorted_vals = c->d_sorted_vals;
  b.line_off = c->d_line_off;
  b.a_i = c->d_a_i;
  b.ac1 = c->d_ac;
  b.ac2 = c->d_ac + S * n;
  b.ae2 = c->d_ac + 2 * S * n;
  b.n_valid = c->d_nvalid;
  b.agent_pos = c->d_agent_pos;
  int launches = 0;
  BFVM_CUDA(agents_build(b, c->stream, &launches));
  note_launches(launches);
  c->n_agents = n;
  ++c->version;
  return BFVM_OK;
}

}  // namespace

extern "C" {

const char* bfvm_status_string(int s) {
  switch (s) {
    case BFVM_OK: return "ok";
    case BFVM_ERR_ARG: return "invalid argument";
    case BFVM_ERR_CUDA: return "CUDA error";
    case BFVM_ERR_OOM: return "out of device memory";
    case BFVM_ERR_SHAPE: return "unsupported grid shape";
    case BFVM_ERR_NODEVICE: return "no CUDA device";
    case BFVM_ERR_TIMEOUT: return "device wait timed out";
    case BFVM_ERR_STATE: return "invalid state";
    default: return "unknown status";
  }
}

long long bfvm_kernel_launches(void) { return g_launches.load(); }

int bfvm_create(const bfvm_config* cfg, bfvm_ctx** out) {
  if (!cfg || !out || !cfg->diffusion_coefficients || !cfg->decay_rates) return BFVM_ERR_ARG;
  *out = nullptr;
  if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || cfg->n_substrates < 1 || cfg->n_substrates > kMaxSubstrates ||
      !(cfg->dx > 0) || !(cfg->dt > 0) || (cfg->precision != BFVM_FP64 && cfg->precision != BFVM_FP32))
    return BFVM_ERR_ARG;
  const long long nvox = 1LL * cfg->nx * cfg->ny * cfg->nz;
  if (nvox >= (1LL << 31) || cfg->nx > 65535 || cfg->ny > 65535 || cfg->nz > 65535) return BFVM_ERR_SHAPE;
  for (int s = 0; s < cfg->n_substrates; ++s)
    if (!(cfg->diffusion_coefficients[s] >= 0) || !(cfg->decay_rates[s] >= 0)) return BFVM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return BFVM_ERR_NODEVICE;
  }
  if (cfg->device < 0 || cfg->device >= ndev) return BFVM_ERR_NODEVICE;
  DeviceGuard g(cfg->device);
  bfvm_ctx* c = new (std::nothrow) bfvm_ctx();
  if (!c) return BFVM_ERR_OOM;
  c->device = cfg->device;
  c->nx = cfg->nx;
  c->ny = cfg->ny;
  c->nz = cfg->nz;
  c->S = cfg->n_substrates;
  c->prec = cfg->precision;
  c->eb = c->prec == BFVM_FP64 ? 8 : 4;
  c->dx = cfg->dx;
  c->dt = cfg->dt;
  const int row_align = 128 / c->eb;
  c->nxp = (c->nx + row_align - 1) / row_align * row_align;
  if (!pick_config(c->eb, c->nx, c->ny, c->nz, &c->cfg)) {
    delete c;
    return BFVM_ERR_SHAPE;
  }
  auto fail = [&](int rc) {
    bfvm_destroy(c);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) return fail(BFVM_ERR_CUDA);
  c->stream = c->own_stream;
  const size_t S = c->S;
  c->field_bytes = static_cast<size_t>(c->nxp) * c->ny * c->nz * S * c->eb;
  int rc = BFVM_OK;
  if (rc == BFVM_OK) rc = dalloc(c, &c->f, c->field_bytes);
  size_t dr_tmp[3], cu_tmp[3];
  if (rc == BFVM_OK) rc = dalloc(c, &c->d_coef, coef_bytes(c, dr_tmp, cu_tmp));
  if (rc == BFVM_OK) rc = dalloc(c, &c->d_c1, S * 16);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_off), S * sizeof(double));
  if (rc == BFVM_OK) rc = dalloc(c, &c->d_shift, S * sizeof(double));
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_active), S * sizeof(int));
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_faces), face_elems(c) * 8);
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_status), sizeof(int));
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_tile_counter), 4 * sizeof(unsigned long long));
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_nvalid), sizeof(int));
  if (rc == BFVM_OK)
    rc = dalloc(c, reinterpret_cast<void**>(&c->d_line_off), sizeof(int) * (static_cast<size_t>(c->ny) * c->nz + 1));
  if (rc == BFVM_OK) rc = dalloc(c, reinterpret_cast<void**>(&c->d_sums), sizeof(double) * (S * 1024 + S));
  if (rc != BFVM_OK) return fail(rc);
  if (cudaMallocHost(reinterpret_cast<void**>(&c->h_status), sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    c->h_status = nullptr;
    return fail(BFVM_ERR_OOM);
  }
  if (cudaMemset(c->f, 0, c->field_bytes) != cudaSuccess || cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess ||
      cudaMemset(c->d_tile_counter, 0, 4 * sizeof(unsigned long long)) != cudaSuccess)
    return fail(BFVM_ERR_CUDA);
  // made here, not on first use, so that steps may run inside a caller's
  // stream capture of any mode
  if (cudaStreamCreateWithFlags(&c->group_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_gfork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_gjoin, cudaEventDisableTiming) != cudaSuccess)
    return fail(BFVM_ERR_CUDA);
  if ((rc = upload_coefficients(c, cfg->diffusion_coefficients, cfg->decay_rates)) != BFVM_OK) return fail(rc);
  // Reference defaults: activation on, value 1.0 on every face voxel.
  c->active.assign(S, 1);
  std::vector<int> act(S, 1);
  c->faces.assign(face_elems(c), 1.0);
  c->off.assign(S, 0.0);
  if (cudaMemcpy(c->d_active, act.data(), S * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_faces, c->faces.data(), c->faces.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_off, c->off.data(), S * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_shift, c->off.data(), S * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(BFVM_ERR_CUDA);
  if (encode_field_maps(&c->maps, c->f, c->eb, c->nx, c->ny, c->nz, c->S, c->nxp, c->cfg) != 0)
    return fail(BFVM_ERR_CUDA);
  *out = c;
  return BFVM_OK;
}

int bfvm_destroy(bfvm_ctx* c) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_agents(c);
  dfree(c, c->f);
  dfree(c, c->d_coef);
  dfree(c, c->d_c1);
  dfree(c, c->d_off);
  dfree(c, c->d_shift);
  dfree(c, c->d_active);
  dfree(c, c->d_faces);
  dfree(c, c->d_status);
  if (c->h_status) cudaFreeHost(c->h_status);
  dfree(c, c->d_tile_counter);
  dfree(c, c->d_nvalid);
  dfree(c, c->d_line_off);
  dfree(c, c->d_sums);
  dfree(c, c->d_staging);
  dfree(c, c->d_grad);
  dfree(c, c->d_bulk);
  dfree(c, c->d_internal);
  dfree(c, c->d_coef2d);
  dfree(c, c->d_shift2d);
  dfree(c, c->d_zero_active);
  dfree(c, c->d_nodes);
  dfree(c, c->d_delta);
  dfree(c, c->d_mass);
  dfree(c, c->d_part);
  for (cudaEvent_t e : c->events) cudaEventDestroy(e);
  drop_step_graph(c);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->group_stream) {
    cudaStreamSynchronize(c->group_stream);
    cudaStreamDestroy(c->group_stream);
  }
  if (c->ev_gfork) cudaEventDestroy(c->ev_gfork);
  if (c->ev_gjoin) cudaEventDestroy(c->ev_gjoin);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return BFVM_OK;
}

int bfvm_set_dirichlet_activation(bfvm_ctx* c, const unsigned char* active) {
  if (!c || !active) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  std::vector<int> act(c->S);
  for (int s = 0; s < c->S; ++s) act[s] = active[s] ? 1 : 0;
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  BFVM_CUDA(cudaMemcpy(c->d_active, act.data(), c->S * sizeof(int), cudaMemcpyHostToDevice));
  c->active.assign(active, active + c->S);
  return BFVM_OK;
}

int bfvm_set_dirichlet_face(bfvm_ctx* c, int face, const double* values) {
  if (!c || !values || face < 0 || face > 5) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  const int S = c->S, nx = c->nx, ny = c->ny, nz = c->nz;
  const int side = face & 1;
  // Transpose the reference-oriented plane into the device face layout.
  std::vector<double> plane;
  size_t dst_off = 0;
  if (face < 2) {  // [ny][nz][S] -> xface[side][s][k][j]
    plane.resize(static_cast<size_t>(S) * nz * ny);
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k)
        for (int s = 0; s < S; ++s)
          plane[(static_cast<size_t>(s) * nz + k) * ny + j] = values[(static_cast<size_t>(j) * nz + k) * S + s];
    dst_off = static_cast<size_t>(side) * S * nz * ny;
  } else if (face < 4) {  // [nx][nz][S] -> yface[side][s][k][i]
    plane.resize(static_cast<size_t>(S) * nz * nx);
    for (int i = 0; i < nx; ++i)
      for (int k = 0; k < nz; ++k)
        for (int s = 0; s < S; ++s)
          plane[(static_cast<size_t>(s) * nz + k) * nx + i] = values[(static_cast<size_t>(i) * nz + k) * S + s];
    dst_off = 2ull * S * nz * ny + static_cast<size_t>(side) * S * nz * nx;
  } else {  // [nx][ny][S] -> zface[side][s][j][i]
    plane.resize(static_cast<size_t>(S) * ny * nx);
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int s = 0; s < S; ++s)
          plane[(static_cast<size_t>(s) * ny + j) * nx + i] = values[(static_cast<size_t>(i) * ny + j) * S + s];
    dst_off = 2ull * S * nz * ny + 2ull * S * nz * nx + static_cast<size_t>(side) * S * ny * nx;
  }
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  BFVM_CUDA(cudaMemcpy(c->d_faces + dst_off, plane.data(), plane.size() * 8, cudaMemcpyHostToDevice));
  std::copy(plane.begin(), plane.end(), c->faces.begin() + dst_off);
  return BFVM_OK;
}

int bfvm_set_dirichlet_uniform(bfvm_ctx* c, const double* values) {
  if (!c || !values) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  const int S = c->S, nx = c->nx, ny = c->ny, nz = c->nz;
  std::vector<double> all(face_elems(c));
  size_t o = 0;
  for (int side = 0; side < 2; ++side)
    for (int s = 0; s < S; ++s)
      for (size_t q = 0; q < static_cast<size_t>(nz) * ny; ++q) all[o++] = values[s];
  for (int side = 0; side < 2; ++side)
    for (int s = 0; s < S; ++s)
      for (size_t q = 0; q < static_cast<size_t>(nz) * nx; ++q) all[o++] = values[s];
  for (int side = 0; side < 2; ++side)
    for (int s = 0; s < S; ++s)
      for (size_t q = 0; q < static_cast<size_t>(ny) * nx; ++q) all[o++] = values[s];
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  BFVM_CUDA(cudaMemcpy(c->d_faces, all.data(), all.size() * 8, cudaMemcpyHostToDevice));
  c->faces = all;
  return BFVM_OK;
}

}  // extern "C"

int bfvm::ensure_staging(bfvm_ctx* c) {
  if (c->d_staging) return BFVM_OK;
  return dalloc(c, reinterpret_cast<void**>(&c->d_staging),
                sizeof(double) * static_cast<size_t>(c->nx) * c->ny * c->nz * c->S);
}

// FP32 solves store each substrate as a deviation from an FP64 offset: the
// mean Dirichlet face value of an activated substrate, else 0.  Values near
// the boundary value then keep more significant bits, and the sweeps stay
// exact in structure (a constant solves the zero-flux system up to the
// factor 1 + c2, which the right-hand-side shift accounts for).  The offsets
// are chosen when a field is uploaded.
static int choose_offsets(bfvm_ctx* c) {
  if (c->prec != BFVM_FP32) return BFVM_OK;
  const int S = c->S, nx = c->nx, ny = c->ny, nz = c->nz;
  std::vector<double> off(S, 0.0);
  std::vector<double> shift(S, 0.0);
  const size_t px = static_cast<size_t>(nz) * ny, py = static_cast<size_t>(nz) * nx,
               pz = static_cast<size_t>(ny) * nx;
  for (int s = 0; s < S; ++s) {
    if (!c->active[s]) continue;
    double acc = 0.0;
    size_t cnt = 0;
    for (int side = 0; side < 2; ++side) {
      const double* a = c->faces.data() + (static_cast<size_t>(side) * S + s) * px;
      for (size_t q = 0; q < px; ++q) acc += a[q];
      const double* b = c->faces.data() + 2 * S * px + (static_cast<size_t>(side) * S + s) * py;
      for (size_t q = 0; q < py; ++q) acc += b[q];
      const double* z = c->faces.data() + 2 * S * px + 2 * S * py + (static_cast<size_t>(side) * S + s) * pz;
      for (size_t q = 0; q < pz; ++q) acc += z[q];
      cnt += px + py + pz;
    }
    off[s] = acc / static_cast<double>(cnt);
    shift[s] = c->c2[s] * off[s];
  }
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  BFVM_CUDA(cudaMemcpy(c->d_off, off.data(), S * sizeof(double), cudaMemcpyHostToDevice));
  BFVM_CUDA(cudaMemcpy(c->d_shift, shift.data(), S * sizeof(double), cudaMemcpyHostToDevice));
  c->off = off;
  return update_shift_2d(c);
}

static int pack_from_device_aos(bfvm_ctx* c, const double* d_aos) {
  if (c->prec == BFVM_FP64) {
    BFVM_CUDA(launch_pack<double>(d_aos, static_cast<double*>(c->f), c->nx, c->ny, c->nz, c->S, c->nxp, nullptr,
                                  c->stream));
  } else {
    const int rc = choose_offsets(c);
    if (rc != BFVM_OK) return rc;
    BFVM_CUDA(launch_pack<float>(d_aos, static_cast<float*>(c->f), c->nx, c->ny, c->nz, c->S, c->nxp, c->d_off,
                                 c->stream));
  }
  note_launches(1);
  return BFVM_OK;
}

int bfvm::unpack_to_device_aos(bfvm_ctx* c, double* d_aos) {
  if (c->prec == BFVM_FP64)
    BFVM_CUDA(launch_unpack<double>(static_cast<const double*>(c->f), d_aos, c->nx, c->ny, c->nz, c->S, c->nxp,
                                    nullptr, c->stream));
  else
    BFVM_CUDA(launch_unpack<float>(static_cast<const float*>(c->f), d_aos, c->nx, c->ny, c->nz, c->S, c->nxp,
                                   c->d_off, c->stream));
  note_launches(1);
  return BFVM_OK;
}

extern "C" {

int bfvm_upload_field(bfvm_ctx* c, const double* field) {
  if (!c || !field) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  int rc = ensure_staging(c);
  if (rc != BFVM_OK) return rc;
  const size_t bytes = sizeof(double) * static_cast<size_t>(c->nx) * c->ny * c->nz * c->S;
  BFVM_CUDA(cudaMemcpyAsync(c->d_staging, field, bytes, cudaMemcpyHostToDevice, c->stream));
  return pack_from_device_aos(c, c->d_staging);
}

int bfvm_download_field(bfvm_ctx* c, double* field) {
  if (!c || !field) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  int rc = ensure_staging(c);
  if (rc != BFVM_OK) return rc;
  if ((rc = unpack_to_device_aos(c, c->d_staging)) != BFVM_OK) return rc;
  const size_t bytes = sizeof(double) * static_cast<size_t>(c->nx) * c->ny * c->nz * c->S;
  BFVM_CUDA(cudaMemcpyAsync(field, c->d_staging, bytes, cudaMemcpyDeviceToHost, c->stream));
  return bfvm_synchronize(c);
}

int bfvm_upload_field_device(bfvm_ctx* c, const double* d_field) {
  if (!c || !d_field) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  return pack_from_device_aos(c, d_field);
}

int bfvm_download_field_device(bfvm_ctx* c, double* d_field) {
  if (!c || !d_field) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  return unpack_to_device_aos(c, d_field);
}

// The side stream that carries an agent list's constants (or rates) to the
// device while the voxel ids, copied first on the solve's stream, are sorted.
// Returns with copy_stream ordered after everything enqueued on the stream
// so far (the previous list's readers of the constants included).
static int fork_copy_stream(bfvm_ctx* c) {
  if (!c->copy_stream) {
    BFVM_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    BFVM_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    BFVM_CUDA(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  }
  BFVM_CUDA(cudaEventRecord(c->ev_fork, c->stream));
  BFVM_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_fork, 0));
  return BFVM_OK;
}

static int set_agents_common(bfvm_ctx* c, int n, const int* voxel, const unsigned char* active) {
  int rc = ensure_agent_capacity(c, n);
  if (rc != BFVM_OK) return rc;
  if (n > 0) {
    BFVM_CUDA(cudaMemcpyAsync(c->d_voxel, voxel, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
    if (active) {
      BFVM_CUDA(cudaMemcpyAsync(c->d_agent_active, active, n, cudaMemcpyHostToDevice, c->stream));
    } else {
      BFVM_CUDA(cudaMemsetAsync(c->d_agent_active, 1, n, c->stream));
    }
  }
  return BFVM_OK;
}

int bfvm_set_agents(bfvm_ctx* c, int n, const int* voxel, const unsigned char* active, const double* c1,
                    const double* c2, const double* e2) {
  if (!c || n < 0 || (n > 0 && (!voxel || !c1 || !c2 || !e2))) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  int rc = set_agents_common(c, n, voxel, active);
  if (rc != BFVM_OK) return rc;
  const size_t row = sizeof(double) * c->S * static_cast<size_t>(n);
  cudaEvent_t ready = nullptr;
  if (n > 0) {
    if ((rc = fork_copy_stream(c)) != BFVM_OK) return rc;
    BFVM_CUDA(cudaMemcpyAsync(c->d_c, c1, row, cudaMemcpyHostToDevice, c->copy_stream));
    BFVM_CUDA(cudaMemcpyAsync(c->d_c + static_cast<size_t>(c->S) * n, c2, row, cudaMemcpyHostToDevice,
                              c->copy_stream));
    BFVM_CUDA(cudaMemcpyAsync(c->d_c + 2ull * c->S * n, e2, row, cudaMemcpyHostToDevice, c->copy_stream));
    BFVM_CUDA(cudaEventRecord(c->ev_join, c->copy_stream));
    ready = c->ev_join;
  }
  c->agents_from_rates = 0;
  rc = build_agents(c, n, ready);
  return rc == BFVM_OK ? tracking_after_agents(c) : rc;
}

int bfvm_set_agents_from_rates(bfvm_ctx* c, int n, const int* voxel, const unsigned char* active, const double* volume,
                               const double* sec, const double* upt, const double* sat, const double* exp_) {
  if (!c || n < 0 || (n > 0 && (!voxel || !volume || !sec || !upt || !sat || !exp_))) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  int rc = set_agents_common(c, n, voxel, active);
  if (rc != BFVM_OK) return rc;
  cudaEvent_t ready = nullptr;
  if (n > 0) {
    const size_t row = sizeof(double) * c->S * static_cast<size_t>(n);
    double* vol = c->d_rates;
    double* r = c->d_rates + n;
    const size_t SN = static_cast<size_t>(c->S) * n;
    if ((rc = fork_copy_stream(c)) != BFVM_OK) return rc;
    cudaStream_t cs = c->copy_stream;
    BFVM_CUDA(cudaMemcpyAsync(vol, volume, sizeof(double) * n, cudaMemcpyHostToDevice, cs));
    BFVM_CUDA(cudaMemcpyAsync(r, sec, row, cudaMemcpyHostToDevice, cs));
    BFVM_CUDA(cudaMemcpyAsync(r + SN, upt, row, cudaMemcpyHostToDevice, cs));
    BFVM_CUDA(cudaMemcpyAsync(r + 2 * SN, sat, row, cudaMemcpyHostToDevice, cs));
    BFVM_CUDA(cudaMemcpyAsync(r + 3 * SN, exp_, row, cudaMemcpyHostToDevice, cs));
    const double vvox = c->dx * c->dx * c->dx;
    BFVM_CUDA(agents_compute_constants(n, c->S, c->dt, vvox, vol, r, r + SN, r + 2 * SN, r + 3 * SN, c->d_c,
                                       c->d_c + SN, c->d_c + 2 * SN, cs));
    note_launches(1);
    BFVM_CUDA(cudaEventRecord(c->ev_join, cs));
    ready = c->ev_join;
  }
  c->agents_from_rates = 1;
  rc = build_agents(c, n, ready);
  return rc == BFVM_OK ? tracking_after_agents(c) : rc;
}

int bfvm_update_agents(bfvm_ctx* c, int n_changed, const int* idx, const double* c1, const double* c2,
                       const double* e2) {
  if (!c || n_changed < 0 || (n_changed > 0 && (!idx || !c1 || !c2 || !e2))) return BFVM_ERR_ARG;
  if (n_changed == 0) return BFVM_OK;
  if (n_changed > c->n_agents) return BFVM_ERR_ARG;
  // Distinct indices of the current list: the update kernel writes each
  // listed agent's constants from one thread per substrate, in parallel.
  std::vector<unsigned char> seen(static_cast<size_t>(c->n_agents), 0);
  for (int q = 0; q < n_changed; ++q) {
    const int a = idx[q];
    if (a < 0 || a >= c->n_agents || seen[a]) return BFVM_ERR_ARG;
    seen[a] = 1;
  }
  DeviceGuard g(c->device);
  const size_t S = c->S, m = static_cast<size_t>(n_changed);
  const size_t idx_bytes = (sizeof(int) * m + 255) & ~size_t(255);
  const size_t row = sizeof(double) * S * m;
  const size_t need = idx_bytes + 3 * row;
  if (need > c->cap_delta) {
    dfree(c, c->d_delta);
    c->d_delta = nullptr;
    c->cap_delta = 0;
    const int rc = dalloc(c, &c->d_delta, need);
    if (rc != BFVM_OK) return rc;
    c->cap_delta = need;
  }
  unsigned char* base = static_cast<unsigned char*>(c->d_delta);
  int* d_idx = reinterpret_cast<int*>(base);
  double* v = reinterpret_cast<double*>(base + idx_bytes);
  BFVM_CUDA(cudaMemcpyAsync(d_idx, idx, sizeof(int) * m, cudaMemcpyHostToDevice, c->stream));
  BFVM_CUDA(cudaMemcpyAsync(v, c1, row, cudaMemcpyHostToDevice, c->stream));
  BFVM_CUDA(cudaMemcpyAsync(v + S * m, c2, row, cudaMemcpyHostToDevice, c->stream));
  BFVM_CUDA(cudaMemcpyAsync(v + 2 * S * m, e2, row, cudaMemcpyHostToDevice, c->stream));
  const size_t SN = S * c->n_agents;
  BFVM_CUDA(agents_update_constants(n_changed, c->S, c->n_agents, d_idx, v, v + S * m, v + 2 * S * m, c->d_agent_pos,
                                    c->d_c, c->d_c + SN, c->d_c + 2 * SN, c->d_ac, c->d_ac + SN, c->d_ac + 2 * SN,
                                    c->stream));
  note_launches(1);
  return BFVM_OK;
}

int bfvm_agent_constants_device(int n, int S, double dt, double voxel_volume, const double* volume,
                                const double* sec, const double* upt, const double* sat, const double* exp_,
                                double* c1, double* c2, double* e2, void* stream) {
  if (n < 0 || S < 1 || S > kMaxSubstrates || !(dt > 0) || !(voxel_volume > 0)) return BFVM_ERR_ARG;
  if (n > 0 && (!volume || !sec || !upt || !sat || !exp_ || !c1 || !c2 || !e2)) return BFVM_ERR_ARG;
  BFVM_CUDA(agents_compute_constants(n, S, dt, voxel_volume, volume, sec, upt, sat, exp_, c1, c2, e2,
                                     static_cast<cudaStream_t>(stream)));
  if (n > 0) note_launches(1);
  return BFVM_OK;
}

int bfvm_step(bfvm_ctx* c, int nsteps, int flags) {
  if (!c || nsteps < 0) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  const bool src = (flags & BFVM_STEP_SOURCES) != 0;
  return c->prec == BFVM_FP64 ? run_steps<double>(c, nsteps, src) : run_steps<float>(c, nsteps, src);
}

int bfvm_apply_sources(bfvm_ctx* c) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  return bfvm::apply_sources_on(c, c->stream);
}


int bfvm_sample_agents(bfvm_ctx* c, double* out) {
  if (!c || (!out && c->n_agents > 0)) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  if (c->n_agents == 0) return BFVM_OK;
  if (c->prec == BFVM_FP64)
    BFVM_CUDA(agents_sample<double>(c->n_agents, c->d_dev_voxel, c->S, c->nx, c->ny, c->nz, c->nxp,
                                    static_cast<const double*>(c->f), nullptr, c->d_sample, c->stream));
  else
    BFVM_CUDA(agents_sample<float>(c->n_agents, c->d_dev_voxel, c->S, c->nx, c->ny, c->nz, c->nxp,
                                   static_cast<const float*>(c->f), c->d_off, c->d_sample, c->stream));
  note_launches(1);
  BFVM_CUDA(cudaMemcpyAsync(out, c->d_sample, sizeof(double) * c->S * static_cast<size_t>(c->n_agents),
                            cudaMemcpyDeviceToHost, c->stream));
  return bfvm_synchronize(c);
}

}  // extern "C"

namespace {

// Deterministic per-substrate sums: fixed block partials, then one block adds
// the partials in order.
template <typename T>
__global__ void field_partial_sums(const T* __restrict__ f, int nx, int rows_per_s, int nxp, double* partial) {
  __shared__ double red[256];
  const int s = blockIdx.y;
  const long long n = static_cast<long long>(rows_per_s) * nx;
  double acc = 0.0;
  for (long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long r = q / nx, i = q % nx;
    acc += static_cast<double>(f[(static_cast<size_t>(s) * rows_per_s + r) * nxp + i]);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[static_cast<size_t>(s) * gridDim.x + blockIdx.x] = red[0];
}

__global__ void field_final_sums(const double* partial, int nparts, int S, double* out) {
  const int s = threadIdx.x;
  if (s >= S) return;
  double acc = 0.0;
  for (int b = 0; b < nparts; ++b) acc += partial[static_cast<size_t>(s) * nparts + b];
  out[s] = acc;
}

}  // namespace

extern "C" int bfvm_field_sums(bfvm_ctx* c, double* out) {
  if (!c || !out) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  const int nparts = 1024;
  dim3 grid(nparts, c->S);
  double* partial = c->d_sums;
  double* res = c->d_sums + static_cast<size_t>(c->S) * nparts;
  if (c->prec == BFVM_FP64)
    field_partial_sums<double><<<grid, 256, 0, c->stream>>>(static_cast<const double*>(c->f), c->nx, c->ny * c->nz,
                                                            c->nxp, partial);
  else
    field_partial_sums<float><<<grid, 256, 0, c->stream>>>(static_cast<const float*>(c->f), c->nx, c->ny * c->nz,
                                                           c->nxp, partial);
  BFVM_CUDA(cudaGetLastError());
  field_final_sums<<<1, 64, 0, c->stream>>>(partial, nparts, c->S, res);
  BFVM_CUDA(cudaGetLastError());
  note_launches(2);
  BFVM_CUDA(cudaMemcpyAsync(out, res, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->stream));
  const int rc = bfvm_synchronize(c);
  if (rc == BFVM_OK && c->prec == BFVM_FP32) {
    const double nv = static_cast<double>(c->nx) * c->ny * c->nz;
    for (int s = 0; s < c->S; ++s) out[s] += c->off[s] * nv;
  }
  return rc;
}

extern "C" int bfvm_field_offsets(bfvm_ctx* c, double* out) {
  if (!c || !out) return BFVM_ERR_ARG;
  for (int s = 0; s < c->S; ++s) out[s] = c->off[s];
  return BFVM_OK;
}

extern "C" int bfvm_synchronize(bfvm_ctx* c) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  // the status word comes back behind the stream's work, in the same wait
  BFVM_CUDA(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  if (*c->h_status != 0) {
    cudaMemset(c->d_status, 0, sizeof(int));
    return BFVM_ERR_TIMEOUT;
  }
  return BFVM_OK;
}

extern "C" int bfvm_set_wait_limit_ns(int device, unsigned long long ns) {
  if (ns < 1000ull || ns > 60000000000ull) return BFVM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return BFVM_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return BFVM_ERR_NODEVICE;
  DeviceGuard g(device);
  BFVM_CUDA(sweeps_set_wait_limit(ns));
  BFVM_CUDA(tmem_sweeps_set_wait_limit(ns));
  return BFVM_OK;
}

extern "C" int bfvm_timing_enable(bfvm_ctx* c, int on) {
  if (!c) return BFVM_ERR_ARG;
  c->timing = on != 0;
  return BFVM_OK;
}

extern "C" int bfvm_timing_read_kernels(bfvm_ctx* c, double* ms_sxyz, int* steps) {
  if (!c || !ms_sxyz) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  double acc[kStepEvents - 1] = {0, 0, 0, 0};
  for (int s = 0; s < c->timed_steps; ++s) {
    const cudaEvent_t* ev = &c->events[kStepEvents * static_cast<size_t>(s)];
    for (int k = 0; k + 1 < kStepEvents; ++k) {
      float ms = 0.f;
      BFVM_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      acc[k] += ms;
    }
  }
  for (int k = 0; k + 1 < kStepEvents; ++k) ms_sxyz[k] = acc[k];
  if (steps) *steps = c->timed_steps;
  c->timed_steps = 0;
  return BFVM_OK;
}

extern "C" int bfvm_timing_read(bfvm_ctx* c, double* ms_xyz, int* steps) {
  if (!c || !ms_xyz) return BFVM_ERR_ARG;
  double ms[4];
  const int rc = bfvm_timing_read_kernels(c, ms, steps);
  if (rc != BFVM_OK) return rc;
  ms_xyz[0] = ms[0] + ms[1];  // the sources with the x sweep
  ms_xyz[1] = ms[2];
  ms_xyz[2] = ms[3];
  return BFVM_OK;
}

extern "C" void* bfvm_stream(bfvm_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

extern "C" int bfvm_set_stream(bfvm_ctx* c, void* stream) {
  if (!c) return BFVM_ERR_ARG;
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return BFVM_OK;
}

extern "C" int bfvm_device_field(bfvm_ctx* c, void** ptr, int* pitch, int* elem_bytes) {
  if (!c) return BFVM_ERR_ARG;
  if (ptr) *ptr = c->f;
  if (pitch) *pitch = c->nxp;
  if (elem_bytes) *elem_bytes = c->eb;
  return BFVM_OK;
}

extern "C" size_t bfvm_device_bytes(bfvm_ctx* c) { return c ? c->device_bytes : 0; }

// Bytes bfvm_create + one host field upload + bfvm_set_agents(n_agents) would
// request, computed from the same sizes those calls allocate.
extern "C" size_t bfvm_estimate_bytes(const bfvm_config* cfg, int n_agents) {
  if (!cfg || cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || cfg->n_substrates < 1 || n_agents < 0 ||
      (cfg->precision != BFVM_FP64 && cfg->precision != BFVM_FP32))
    return 0;
  bfvm_ctx c;
  c.nx = cfg->nx;
  c.ny = cfg->ny;
  c.nz = cfg->nz;
  c.S = cfg->n_substrates;
  c.prec = cfg->precision;
  c.eb = c.prec == BFVM_FP64 ? 8 : 4;
  const int row_align = 128 / c.eb;
  c.nxp = (c.nx + row_align - 1) / row_align * row_align;
  const size_t S = c.S;
  const size_t nvox = static_cast<size_t>(c.nx) * c.ny * c.nz;
  size_t dr[3], cu[3];
  size_t b = static_cast<size_t>(c.nxp) * c.ny * c.nz * S * c.eb;  // field
  b += coef_bytes(&c, dr, cu);
  b += S * 16 + S * sizeof(double) + S * sizeof(float) + S * sizeof(int);
  b += face_elems(&c) * 8 + 2 * sizeof(int);
  b += sizeof(int) * (static_cast<size_t>(c.ny) * c.nz + 1);
  b += sizeof(double) * (S * 1024 + S);
  b += sizeof(double) * nvox * S;  // host-transfer staging (bfvm_release_staging frees it)
  if (n_agents > 0) {
    const size_t cap = n_agents < 1024 ? 1024 : static_cast<size_t>(n_agents);
    b += cap * (sizeof(int) + 1 + 4 * sizeof(unsigned));
    b += sizeof(double) * cap * (3 * S + (1 + 4 * S) + 3 * S + S);
    b += agent_scratch_bytes(static_cast<int>(cap));
  }
  return b;
}

extern "C" int bfvm_set_bulk_rates(bfvm_ctx* c, const double* supply, const double* target, const double* uptake) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  if (!supply && !target && !uptake) {
    BFVM_CUDA(cudaStreamSynchronize(c->stream));
    dfree(c, c->d_bulk);
    c->d_bulk = nullptr;
    return BFVM_OK;
  }
  if (!supply || !target || !uptake) return BFVM_ERR_ARG;
  const size_t plane = static_cast<size_t>(c->nxp) * c->ny * c->nz * c->S;
  if (!c->d_bulk) {
    const int rc = dalloc(c, reinterpret_cast<void**>(&c->d_bulk), 3 * plane * sizeof(double));
    if (rc != BFVM_OK) return rc;
  }
  int rc = ensure_staging(c);
  if (rc != BFVM_OK) return rc;
  const size_t bytes = sizeof(double) * static_cast<size_t>(c->nx) * c->ny * c->nz * c->S;
  const double* src[3] = {supply, target, uptake};
  for (int a = 0; a < 3; ++a) {
    BFVM_CUDA(cudaMemcpyAsync(c->d_staging, src[a], bytes, cudaMemcpyHostToDevice, c->stream));
    BFVM_CUDA(launch_pack<double>(c->d_staging, c->d_bulk + a * plane, c->nx, c->ny, c->nz, c->S, c->nxp, nullptr,
                                  c->stream));
    note_launches(1);
  }
  return bfvm_synchronize(c);
}

extern "C" int bfvm_apply_bulk_sources(bfvm_ctx* c) {
  if (!c) return BFVM_ERR_ARG;
  if (!c->d_bulk) return BFVM_ERR_STATE;
  DeviceGuard g(c->device);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  if (c->prec == BFVM_FP64)
    BFVM_CUDA(launch_bulk<double>(static_cast<double*>(c->f), c->d_bulk, c->nx, c->ny, c->nz, c->S, c->nxp, c->dt,
                                  nullptr, sms, c->stream));
  else
    BFVM_CUDA(launch_bulk<float>(static_cast<float*>(c->f), c->d_bulk, c->nx, c->ny, c->nz, c->S, c->nxp, c->dt,
                                 c->d_off, sms, c->stream));
  note_launches(1);
  return BFVM_OK;
}

extern "C" int bfvm_release_staging(bfvm_ctx* c) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  dfree(c, c->d_staging);
  c->d_staging = nullptr;
  dfree(c, c->d_grad);
  c->d_grad = nullptr;
  return BFVM_OK;
}

extern "C" int bfvm_set_sweep_schedule(bfvm_ctx* c, int persistent) {
  if (!c || persistent < 0 || persistent > 2) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  c->cfg.persistent = persistent;
  return BFVM_OK;
}

extern "C" int bfvm_set_substrate_streams(bfvm_ctx* c, int streams) {
  if (!c || (streams != 1 && streams != 2)) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  c->sub_streams = streams;  // part of the step graph's key: recaptured on the next run
  return BFVM_OK;
}

extern "C" int bfvm_get_substrate_streams(const bfvm_ctx* c, int* streams) {
  if (!c || !streams) return BFVM_ERR_ARG;
  *streams = c->sub_streams;
  return BFVM_OK;
}

extern "C" int bfvm_set_fused_sources(bfvm_ctx* c, int fused) {
  if (!c || (fused != 0 && fused != 1)) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  c->cfg.fuse_sources = fused;
  return BFVM_OK;
}

extern "C" int bfvm_set_fp64_chain(bfvm_ctx* c, int chain) {
  if (!c || chain < 0 || chain > 2) return BFVM_ERR_ARG;
  if (chain == c->fp64_chain) return BFVM_OK;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  const int prev = c->fp64_chain;
  c->fp64_chain = chain;
  const std::vector<double> D = c->D, decay = c->decay;
  int rc = upload_coefficients(c, D.data(), decay.data());
  if (rc == BFVM_OK && chain == 2) rc = upload_part_coefficients(c);
  if (rc != BFVM_OK) {
    c->fp64_chain = prev;
    upload_coefficients(c, D.data(), decay.data());
    return rc;
  }
  ++c->version;  // the sweeps' parameters (screen) changed: graphs and batch tables are rebuilt
  return BFVM_OK;
}

extern "C" int bfvm_get_fp64_chain(bfvm_ctx* c, int* chain) {
  if (!c || !chain) return BFVM_ERR_ARG;
  *chain = c->fp64_chain;
  return BFVM_OK;
}

extern "C" int bfvm_set_partition_min_line(bfvm_ctx* c, int n_line) {
  if (!c || n_line < -1 || n_line == 0) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  c->part_min_line = n_line;
  return BFVM_OK;
}

extern "C" int bfvm_get_partition_min_line(bfvm_ctx* c, int* n_line) {
  if (!c || !n_line) return BFVM_ERR_ARG;
  *n_line = part_min_line(c);
  return BFVM_OK;
}

extern "C" int bfvm_set_sweep_tmem(bfvm_ctx* c, int on) {
  if (!c || on < 0 || on > 2) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  c->cfg.tmem = on;
  return BFVM_OK;
}

extern "C" int bfvm_get_sweep_schedule(bfvm_ctx* c, int* persistent) {
  if (!c || !persistent) return BFVM_ERR_ARG;
  *persistent = c->cfg.persistent;
  return BFVM_OK;
}

extern "C" int bfvm_get_launch(bfvm_ctx* c, int* x_lines, int* yz_tile, int* yz_chunk) {
  if (!c) return BFVM_ERR_ARG;
  if (x_lines) *x_lines = c->cfg.x_lines;
  if (yz_tile) *yz_tile = c->cfg.yz_tile;
  if (yz_chunk) *yz_chunk = c->cfg.yz_chunk;
  return BFVM_OK;
}

extern "C" int bfvm_set_launch(bfvm_ctx* c, int x_lines, int yz_tile, int yz_chunk) {
  if (!c) return BFVM_ERR_ARG;
  SweepConfig cfg;
  cfg.x_lines = x_lines;
  cfg.yz_tile = yz_tile;
  cfg.yz_chunk = yz_chunk;
  cfg.persistent = c->cfg.persistent;
  cfg.fuse_sources = c->cfg.fuse_sources;
  cfg.tmem = c->cfg.tmem;
  // x_lines: multiple of 8 (1024-byte swizzle atoms), at most 256 (box
  // limit); yz_tile: 16 (FP64 only), 32 or 64 consecutive x -- whole 128-byte
  // rows, so every TMA chunk starts 128-byte aligned in shared memory and
  // every box's x coordinate is 16-byte aligned.
  if (x_lines < 8 || x_lines > 256 || x_lines % 8 != 0) return BFVM_ERR_ARG;
  if ((yz_tile != 16 && yz_tile != 32 && yz_tile != 64) || (yz_tile * c->eb) % 128 != 0) return BFVM_ERR_ARG;
  if (yz_chunk < 1 || yz_chunk > 256) return BFVM_ERR_ARG;
  if (!config_fits(c->eb, c->nx, c->ny, c->nz, cfg)) return BFVM_ERR_SHAPE;
  DeviceGuard g(c->device);
  FieldMaps maps;
  if (encode_field_maps(&maps, c->f, c->eb, c->nx, c->ny, c->nz, c->S, c->nxp, cfg) != 0) return BFVM_ERR_CUDA;
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  c->maps = maps;
  c->cfg = cfg;
  return BFVM_OK;
}

namespace bfvm {

int apply_sources_on(bfvm_ctx* c, cudaStream_t st, int s_lo, int s_hi) {
  if (c->n_agents == 0) return BFVM_OK;
  const size_t SN = static_cast<size_t>(c->S) * c->n_agents;
  if (c->prec == BFVM_FP64)
    BFVM_CUDA(agents_apply_sources<double>(c->n_agents, c->d_sorted_keys, c->S, c->nx, c->ny, c->nz, c->nxp, c->d_ac,
                                           c->d_ac + SN, c->d_ac + 2 * SN, nullptr, static_cast<double*>(c->f),
                                           track_params(c), st, s_lo, s_hi));
  else
    BFVM_CUDA(agents_apply_sources<float>(c->n_agents, c->d_sorted_keys, c->S, c->nx, c->ny, c->nz, c->nxp, c->d_ac,
                                          c->d_ac + SN, c->d_ac + 2 * SN, c->d_off, static_cast<float*>(c->f),
                                          track_params(c), st, s_lo, s_hi));
  note_launches(1);
  return BFVM_OK;
}

int enqueue_step_on(bfvm_ctx* c, bool sources, cudaStream_t st) {
  const bool standalone = sources && c->n_agents > 0 && !c->cfg.fuse_sources;
  if (c->prec == BFVM_FP64)
    return enqueue_step<double>(c, make_params<double>(c, sources && !standalone), standalone, nullptr, st);
  return enqueue_step<float>(c, make_params<float>(c, sources && !standalone), standalone, nullptr, st);
}

}  // namespace bfvm
