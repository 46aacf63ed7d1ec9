// bfvm_lod2d.cu -- Dirichlet nodes and the 2-D LOD step.
//
// Dirichlet nodes.  Microenvironment::add_dirichlet_node / update_dirichlet_node
// (BioFVM/BioFVM_microenvironment.cpp:218-243) mark any voxel -- interior or
// on a face -- as a Dirichlet node with its own values, and
// set_substrate_dirichlet_activation(substrate, voxel, on) (:288-292) its own
// per-substrate activation; Microenvironment::apply_dirichlet_conditions
// (:303-323) sets every activated density of every node to its value.  Here a
// solve holds one node list (voxel, values [S], activation [S]); a voxel
// given twice keeps its last entry, as a later update_dirichlet_node
// overwrites an earlier one.  The 3-D step (bfvm_step) pins the six faces
// only, as the reference's _BLOCKING solver does; nodes are applied by
// bfvm_apply_dirichlet_nodes and by the 2-D step.
//
// 2-D LOD.  diffusion_decay_solver__constant_coefficients_LOD_2D
// (BioFVM/BioFVM_solvers.cpp:1668-1832) on an nx x ny x 1 grid: nodes pinned;
// x sweep; nodes pinned; y sweep; nodes pinned, with the factorization of the
// 3-D solver except constant2 = decay * dt * 0.5 (:1696-1707).  The sweeps are
// the 3-D sweep kernels, given 2-D coefficient rows and no activated faces.
// The recurrence is the one the reference's commented-out vector forms state
// (axpy forward, naxpy back); its scalar loops in this tree step through the
// array by S and by nx values (a y line, then a stride past the array for
// most shapes), loop over substrates up to n_subs, which only the 3-D setup
// sets, and add the y upper-diagonal term where naxpy subtracts it.  For one
// substrate and ny == 1 the two agree bit for bit (the oracle is checked
// against the reference build there); elsewhere the reference has no
// defined result to compare with.
#include <cstring>

#include "bfvm_ctx.h"

using namespace bfvm;

namespace {

// nodes: device offset of the voxel within a substrate plane, value [n][S],
// activation [n][S]; off [S] (FP32: the field holds rho - off) or null.
template <typename T>
__global__ void dirichlet_nodes_kernel(int n, int S, const long long* __restrict__ node_off,
                                       const double* __restrict__ val, const unsigned char* __restrict__ act,
                                       const double* __restrict__ off, size_t plane, T* __restrict__ f) {
  const long long idx = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long long>(n) * S) return;
  const int q = static_cast<int>(idx / S), s = static_cast<int>(idx % S);
  if (!act[idx]) return;
  double v = val[idx];
  if (off) v -= off[s];
  f[static_cast<size_t>(s) * plane + node_off[q]] = static_cast<T>(v);
}

size_t nodes_bytes(int n, int S) {
  const size_t a = ((sizeof(long long) * n + 255) / 256) * 256;
  const size_t b = ((sizeof(double) * static_cast<size_t>(n) * S + 255) / 256) * 256;
  return a + b + static_cast<size_t>(n) * S;
}

int launch_nodes(bfvm_ctx* c) {
  if (c->n_nodes == 0) return BFVM_OK;
  const int n = c->n_nodes, S = c->S;
  const unsigned char* base = static_cast<const unsigned char*>(c->d_nodes);
  const long long* node_off = reinterpret_cast<const long long*>(base);
  const size_t a = ((sizeof(long long) * n + 255) / 256) * 256;
  const double* val = reinterpret_cast<const double*>(base + a);
  const unsigned char* act = base + a + ((sizeof(double) * static_cast<size_t>(n) * S + 255) / 256) * 256;
  const size_t plane = static_cast<size_t>(c->nxp) * c->ny * c->nz;
  const long long total = static_cast<long long>(n) * S;
  const unsigned blocks = static_cast<unsigned>((total + 255) / 256);
  if (c->prec == BFVM_FP64)
    dirichlet_nodes_kernel<double><<<blocks, 256, 0, c->stream>>>(n, S, node_off, val, act, nullptr, plane,
                                                                   static_cast<double*>(c->f));
  else
    dirichlet_nodes_kernel<float><<<blocks, 256, 0, c->stream>>>(n, S, node_off, val, act, c->d_off, plane,
                                                                  static_cast<float*>(c->f));
  BFVM_CUDA(cudaGetLastError());
  note_launches(1);
  return BFVM_OK;
}

// 2-D coefficient rows for the x and y axes (same packing as the 3-D rows),
// the no-face activation array and, for FP32, the 2-D right-hand-side shift.
int ensure_2d(bfvm_ctx* c) {
  if (c->d_coef2d) return BFVM_OK;
  const int S = c->S;
  const size_t dr_sz = c->prec == BFVM_FP64 ? sizeof(double2) : sizeof(double);
  const int n_axis[2] = {c->nx, c->ny};
  size_t dr_off[2], cu_off[2], o = 0;
  for (int a = 0; a < 2; ++a) {
    const size_t rows = static_cast<size_t>(S) * coef_pad(n_axis[a]);
    dr_off[a] = o;
    o = (o + rows * dr_sz + 255) & ~size_t(255);
    cu_off[a] = o;
    o = (o + rows * sizeof(double) + 255) & ~size_t(255);
  }
  std::vector<unsigned char> host(o, 0);
  std::vector<double> c1(S);
  for (int a = 0; a < 2; ++a) {
    const int n = n_axis[a], np = coef_pad(n);
    std::vector<double> dn(static_cast<size_t>(n) * S), cu(static_cast<size_t>(n) * S);
    thomas_axis_host(n, S, c->D.data(), c->decay.data(), c->dt, c->dx, dn.data(), cu.data(), c1.data(), true);
    for (int s = 0; s < S; ++s)
      for (int i = 0; i < np; ++i) {
        const size_t q = static_cast<size_t>(s) * np + i;
        const bool in = i < n;
        const double d = in ? dn[static_cast<size_t>(i) * S + s] : 1.0;
        const double r = 1.0 / d;  // RN(1/d)
        const double u = in ? cu[static_cast<size_t>(i) * S + s] : -0.0;
        if (c->prec == BFVM_FP64)
          reinterpret_cast<double2*>(host.data() + dr_off[a])[q] = make_double2(d, r);
        else
          reinterpret_cast<double*>(host.data() + dr_off[a])[q] = r;
        reinterpret_cast<double*>(host.data() + cu_off[a])[q] = u;
      }
  }
  void* coef = nullptr;
  int rc = dalloc(c, &coef, o);
  if (rc != BFVM_OK) return rc;
  int* zero = nullptr;
  rc = dalloc(c, reinterpret_cast<void**>(&zero), sizeof(int) * S);
  if (rc != BFVM_OK) {
    dfree(c, coef);
    return rc;
  }
  double* shift = nullptr;
  rc = dalloc(c, reinterpret_cast<void**>(&shift), sizeof(double) * S);
  if (rc != BFVM_OK) {
    dfree(c, coef);
    dfree(c, zero);
    return rc;
  }
  BFVM_CUDA(cudaMemcpy(coef, host.data(), o, cudaMemcpyHostToDevice));
  BFVM_CUDA(cudaMemset(zero, 0, sizeof(int) * S));
  c->d_coef2d = coef;
  c->d_zero_active = zero;
  c->d_shift2d = shift;
  for (int a = 0; a < 2; ++a) {
    c->dr2_off[a] = dr_off[a];
    c->cu2_off[a] = cu_off[a];
  }
  c->c2_2d.assign(S, 0.0);
  for (int s = 0; s < S; ++s) {
    double k2 = c->decay[s];
    k2 *= c->dt;
    k2 *= 0.5;
    c->c2_2d[s] = k2;
  }
  return update_shift_2d(c);
}

template <typename T>
SweepParams<T> make_params_2d(bfvm_ctx* c) {
  SweepParams<T> p = make_params<T>(c, false);
  using DR = typename Coef<T>::DR;
  using CU = typename Coef<T>::CU;
  const unsigned char* cb = static_cast<const unsigned char*>(c->d_coef2d);
  const int n_axis[2] = {c->nx, c->ny};
  AxisCoefs<T>* axes[2] = {&p.ax, &p.ay};
  for (int a = 0; a < 2; ++a) {
    axes[a]->dr = reinterpret_cast<const DR*>(cb + c->dr2_off[a]);
    axes[a]->cu = reinterpret_cast<const CU*>(cb + c->cu2_off[a]);
    axes[a]->npad = coef_pad(n_axis[a]);
    axes[a]->conv = nullptr;  // every chunk reads its coefficients
  }
  p.active = c->d_zero_active;
  p.shift = sizeof(T) == 4 ? c->d_shift2d : nullptr;
  p.screen = c->screen_exact;  // the 2-D rows are {d, 1/d}: the reference-exact chain
  return p;
}

template <typename T>
int run_steps_2d(bfvm_ctx* c, int nsteps, bool sources) {
  const SweepParams<T> p = make_params_2d<T>(c);
  for (int st = 0; st < nsteps; ++st) {
    if (sources) {
      const int rc = bfvm_apply_sources(c);
      if (rc != BFVM_OK) return rc;
    }
    int rc = launch_nodes(c);
    if (rc != BFVM_OK) return rc;
    BFVM_CUDA(launch_sweep_x<T>(c->maps, p, c->cfg, c->stream));
    if ((rc = launch_nodes(c)) != BFVM_OK) return rc;
    BFVM_CUDA(launch_sweep_y<T>(c->maps, p, c->cfg, c->stream));
    if ((rc = launch_nodes(c)) != BFVM_OK) return rc;
    note_launches(2);
  }
  return BFVM_OK;
}

}  // namespace

namespace bfvm {

int update_shift_2d(bfvm_ctx* c) {
  if (!c->d_shift2d || c->prec != BFVM_FP32) return BFVM_OK;
  std::vector<double> shift(c->S, 0.0);
  for (int s = 0; s < c->S; ++s) shift[s] = c->c2_2d[s] * (s < static_cast<int>(c->off.size()) ? c->off[s] : 0.0);
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  BFVM_CUDA(cudaMemcpy(c->d_shift2d, shift.data(), sizeof(double) * c->S, cudaMemcpyHostToDevice));
  return BFVM_OK;
}

}  // namespace bfvm

extern "C" {

int bfvm_set_dirichlet_nodes(bfvm_ctx* c, int count, const int* voxel, const double* values,
                             const unsigned char* activation) {
  if (!c || count < 0 || (count > 0 && (!voxel || !values))) return BFVM_ERR_ARG;
  const int S = c->S;
  const long long nvox = static_cast<long long>(c->nx) * c->ny * c->nz;
  for (int q = 0; q < count; ++q)
    if (voxel[q] < 0 || voxel[q] >= nvox) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  // the last entry of each voxel, in order of first appearance
  std::vector<int> last(count, 1);
  {
    std::unordered_map<int, int> seen;
    for (int q = count - 1; q >= 0; --q) {
      if (seen.count(voxel[q])) last[q] = 0;
      else seen[voxel[q]] = q;
    }
  }
  std::vector<long long> off;
  std::vector<double> val;
  std::vector<unsigned char> act;
  for (int q = 0; q < count; ++q) {
    if (!last[q]) continue;
    const int v = voxel[q];
    const int k = v % c->nz, j = (v / c->nz) % c->ny, i = v / (c->nz * c->ny);
    off.push_back((static_cast<long long>(k) * c->ny + j) * c->nxp + i);
    for (int s = 0; s < S; ++s) {
      val.push_back(values[static_cast<size_t>(q) * S + s]);
      act.push_back(activation ? (activation[static_cast<size_t>(q) * S + s] ? 1 : 0) : (c->active[s] ? 1 : 0));
    }
  }
  const int n = static_cast<int>(off.size());
  BFVM_CUDA(cudaStreamSynchronize(c->stream));
  dfree(c, c->d_nodes);
  c->d_nodes = nullptr;
  c->n_nodes = 0;
  if (n == 0) return BFVM_OK;
  const size_t bytes = nodes_bytes(n, S);
  const int rc = dalloc(c, &c->d_nodes, bytes);
  if (rc != BFVM_OK) return rc;
  std::vector<unsigned char> host(bytes, 0);
  const size_t a = ((sizeof(long long) * n + 255) / 256) * 256;
  const size_t b = ((sizeof(double) * static_cast<size_t>(n) * S + 255) / 256) * 256;
  std::memcpy(host.data(), off.data(), sizeof(long long) * n);
  std::memcpy(host.data() + a, val.data(), sizeof(double) * val.size());
  std::memcpy(host.data() + a + b, act.data(), act.size());
  BFVM_CUDA(cudaMemcpy(c->d_nodes, host.data(), bytes, cudaMemcpyHostToDevice));
  c->n_nodes = n;
  return BFVM_OK;
}

int bfvm_apply_dirichlet_nodes(bfvm_ctx* c) {
  if (!c) return BFVM_ERR_ARG;
  DeviceGuard g(c->device);
  return launch_nodes(c);
}

int bfvm_step_2d(bfvm_ctx* c, int nsteps, int flags) {
  if (!c || nsteps < 0) return BFVM_ERR_ARG;
  if (c->nz != 1) return BFVM_ERR_SHAPE;
  DeviceGuard g(c->device);
  int rc = ensure_2d(c);
  if (rc != BFVM_OK) return rc;
  const bool src = (flags & BFVM_STEP_SOURCES) != 0;
  return c->prec == BFVM_FP64 ? run_steps_2d<double>(c, nsteps, src) : run_steps_2d<float>(c, nsteps, src);
}

}  // extern "C"
