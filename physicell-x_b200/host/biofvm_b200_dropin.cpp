// biofvm_b200_dropin.cpp -- definition of the reference's declared-but-never-
// defined entry point
//     void BioFVM::diffusion_decay_solver__constant_coefficients_LOD_3D(
//         Microenvironment&, double, mpi_Environment&, mpi_Cartesian&)
// (BioFVM/BioFVM_solvers.h:66; friend of Microenvironment at
// BioFVM/BioFVM_microenvironment.h:349), on top of the C ABI in
// include/biofvm_b200.h.  Being the friend, it reads the Microenvironment's
// private Dirichlet tables (dirichlet_value_vectors,
// dirichlet_activation_vector, BioFVM_microenvironment.h:145-146) without any
// change to the reference sources.
//
// Behaviour matches diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING
// (BioFVM/BioFVM_solvers.cpp:102-780) run with one rank: same mesh checks and
// messages, same Dirichlet semantics, and the same FP64 result bit for bit.
// The whole domain lives in one GPU's memory, so the MPI world must have one
// rank.  On any failure the solver prints a message and returns with the
// densities unchanged, as the reference does (:116-121).
//
// bfvm_b200_lod2d_serial is the GPU form of the serial 2-D solver
// diffusion_decay_solver__constant_coefficients_LOD_2D(M, dt)
// (BioFVM/BioFVM_solvers.cpp:1668-1832) for meshes one voxel deep in z.  The
// reference already defines that name, so this is a new function for the
// same slot (Microenvironment::diffusion_decay_solver).  It reaches the
// Dirichlet nodes through public members only: like the reference solver it
// calls M.apply_dirichlet_conditions() on the host densities and takes each
// node (is_dirichlet_node) with the values that call wrote and its
// per-substrate activation (get_substrate_dirichlet_activation(d, voxel)).
#include "biofvm_b200_dropin.h"

#include <cstdlib>
#include <iostream>
#include <map>
#include <mutex>
#include <vector>

#include "BioFVM_basic_agent.h"
#include "BioFVM_solvers.h"
#include "biofvm_b200.h"

namespace BioFVM {

namespace {

struct DropinState {
  bfvm_ctx* ctx = nullptr;
  int nx = 0, ny = 0, nz = 0, S = 0;
  double dx = 0, dt = 0;
  std::vector<Basic_Agent*>* agents = nullptr;
  bool resident = false;
  bool uploaded = false;
  std::vector<int> voxel;
  std::vector<unsigned char> active;
  std::vector<double> c1, c2, e2, plane;
  std::vector<double> e1, internal;  // internalized-substrate tracking
  std::vector<int> node_voxel;       // 2-D solver: Dirichlet nodes
  std::vector<double> node_value;
  std::vector<unsigned char> node_active;
};

std::mutex g_mu;

std::map<const Microenvironment*, DropinState>& table() {
  static std::map<const Microenvironment*, DropinState> t;
  return t;
}

int device_from_env() {
  const char* s = std::getenv("BFVM_DEVICE");
  return s ? std::atoi(s) : 0;
}

bool failed(const char* what, int rc) {
  if (rc == BFVM_OK) return false;
  std::cout << "B200 LOD solver: " << what << " failed: " << bfvm_status_string(rc) << std::endl;
  return true;
}

// M's state, its context (re)created when the mesh, substrate count or dx
// changed.  A new dt alone keeps the context: the reference factors its
// Thomas systems on the first call only (diffusion_solver_setup_done,
// BioFVM/BioFVM_solvers.cpp:125,335) and steps every later call with the
// first call's dt, diffusion coefficients and decay rates, and so does this
// solver.  nullptr (after a message) when the context cannot be made.
DropinState* state_for(Microenvironment& M, double dt) {
  DropinState& st = table()[&M];
  const int nx = static_cast<int>(M.mesh.x_coordinates.size());
  const int ny = static_cast<int>(M.mesh.y_coordinates.size());
  const int nz = static_cast<int>(M.mesh.z_coordinates.size());
  const int S = static_cast<int>(M.number_of_densities());
  if (st.ctx == nullptr || st.nx != nx || st.ny != ny || st.nz != nz || st.S != S || st.dx != M.mesh.dx) {
    if (st.ctx) bfvm_destroy(st.ctx);
    st.ctx = nullptr;
    st.uploaded = false;
    bfvm_config cfg;
    cfg.nx = nx;
    cfg.ny = ny;
    cfg.nz = nz;
    cfg.n_substrates = S;
    cfg.dx = M.mesh.dx;
    cfg.dt = dt;
    cfg.diffusion_coefficients = M.diffusion_coefficients.data();
    cfg.decay_rates = M.decay_rates.data();
    cfg.precision = BFVM_FP64;
    cfg.device = device_from_env();
    bfvm_ctx* ctx = nullptr;
    if (failed("bfvm_create", bfvm_create(&cfg, &ctx))) return nullptr;
    st.ctx = ctx;
    st.nx = nx;
    st.ny = ny;
    st.nz = nz;
    st.S = S;
    st.dt = dt;
    st.dx = M.mesh.dx;
  }
  return &st;
}

// Gather the agents as Basic_Agent::simulate_secretion_and_uptake sees them
// (BioFVM_basic_agent.cpp:509-518): constants refreshed when the volume
// changed.  With Microenvironment_Options::track_internalized_substrates_in_each_agent
// on (BioFVM_microenvironment.h:477), each agent's internalized_substrates go
// to the GPU with it (BioFVM_basic_agent.cpp:520-532, 553-556).  Sets the
// step flags; false after a failure message.
bool send_agents(DropinState& st, double dt, int* flags) {
  *flags = 0;
  if (st.agents == nullptr) return true;
  const int S = st.S;
  const bool track = default_microenvironment_options.track_internalized_substrates_in_each_agent;
  const std::vector<Basic_Agent*>& list = *st.agents;
  const size_t n = list.size();
  st.voxel.resize(n);
  st.active.resize(n);
  st.c1.resize(n * S);
  st.c2.resize(n * S);
  st.e2.resize(n * S);
  if (track) {
    st.e1.resize(n * S);
    st.internal.resize(n * S);
  }
  for (size_t a = 0; a < n; ++a) {
    Basic_Agent* ag = list[a];
    st.active[a] = ag->is_active ? 1 : 0;
    st.voxel[a] = ag->get_current_voxel_index();
    if (ag->is_active && ag->get_is_volume_changed()) ag->set_internal_uptake_constants(dt);
    const std::vector<double>& t1 = ag->get_cell_source_sink_solver_temp1();
    const std::vector<double>& t2 = ag->get_cell_source_sink_solver_temp2();
    const std::vector<double>& x2 = ag->get_cell_source_sink_solver_temp_export2();
    for (int d = 0; d < S; ++d) {
      st.c1[a * S + d] = t1[d];
      st.c2[a * S + d] = t2[d];
      st.e2[a * S + d] = x2[d];
    }
    if (track) {
      const std::vector<double>& x1 = ag->get_cell_source_sink_solver_temp_export1();
      const std::vector<double>& in = *ag->internalized_substrates;
      for (int d = 0; d < S; ++d) {
        st.e1[a * S + d] = d < static_cast<int>(x1.size()) ? x1[d] : 0.0;
        st.internal[a * S + d] = d < static_cast<int>(in.size()) ? in[d] : 0.0;
      }
    }
  }
  bfvm_ctx* ctx = st.ctx;
  if (failed("bfvm_set_agent_tracking", bfvm_set_agent_tracking(ctx, track ? 1 : 0))) return false;
  if (failed("bfvm_set_agents", bfvm_set_agents(ctx, static_cast<int>(n), st.voxel.data(), st.active.data(),
                                                st.c1.data(), st.c2.data(), st.e2.data())))
    return false;
  if (track && n > 0) {
    if (failed("bfvm_set_agent_exports", bfvm_set_agent_exports(ctx, st.e1.data()))) return false;
    if (failed("bfvm_set_internalized", bfvm_set_internalized(ctx, st.internal.data()))) return false;
  }
  *flags = BFVM_STEP_SOURCES;
  return true;
}

// After a step: the agents' internalized amounts written back (when tracked)
// and, unless resident, the densities downloaded into M.
void finish_step(Microenvironment& M, DropinState& st, int flags) {
  const int S = st.S;
  if ((flags & BFVM_STEP_SOURCES) && default_microenvironment_options.track_internalized_substrates_in_each_agent &&
      !st.agents->empty()) {
    const std::vector<Basic_Agent*>& list = *st.agents;
    if (failed("bfvm_get_internalized", bfvm_get_internalized(st.ctx, st.internal.data()))) return;
    for (size_t a = 0; a < list.size(); ++a) {
      std::vector<double>& in = *list[a]->internalized_substrates;
      if (static_cast<int>(in.size()) < S) in.resize(S, 0.0);
      for (int d = 0; d < S; ++d) in[d] = st.internal[a * S + d];
    }
  }
  if (!st.resident) {
    if (failed("bfvm_download_field", bfvm_download_field(st.ctx, M.p_density_vectors->data()))) return;
  }
}

}  // namespace

void diffusion_decay_solver__constant_coefficients_LOD_3D(Microenvironment& M, double dt, mpi_Environment& world,
                                                          mpi_Cartesian& cart_topo) {
  (void)cart_topo;
  if (M.mesh.uniform_mesh == false || M.mesh.Cartesian_mesh == false) {
    std::cout << "Error: This algorithm is written for uniform Cartesian meshes. Try: other solvers!" << std::endl
              << std::endl;
    return;
  }
  if (world.size != 1) {
    std::cout << "Error: the B200 LOD solver keeps the whole domain on one GPU; run it with one MPI rank."
              << std::endl;
    return;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState* sp = state_for(M, dt);
  if (sp == nullptr) return;
  DropinState& st = *sp;
  bfvm_ctx* ctx = st.ctx;
  const int nx = st.nx, ny = st.ny, nz = st.nz, S = st.S;

  // Dirichlet tables, re-read every call: callers may change them at any time
  // (update_dirichlet_node, set_substrate_dirichlet_activation).
  st.active.assign(S, 0);
  for (int d = 0; d < S; ++d) st.active[d] = M.dirichlet_activation_vector[d] ? 1 : 0;
  if (failed("bfvm_set_dirichlet_activation", bfvm_set_dirichlet_activation(ctx, st.active.data()))) return;
  for (int face = 0; face < 6; ++face) {
    const int axis = face / 2, side = face % 2;
    const int na = axis == 0 ? ny : nx;
    const int nb = axis == 2 ? ny : nz;
    st.plane.resize(static_cast<size_t>(na) * nb * S);
    for (int a = 0; a < na; ++a)
      for (int b = 0; b < nb; ++b) {
        int i, j, k;
        if (axis == 0) {
          i = side ? nx - 1 : 0;
          j = a;
          k = b;
        } else if (axis == 1) {
          i = a;
          j = side ? ny - 1 : 0;
          k = b;
        } else {
          i = a;
          j = b;
          k = side ? nz - 1 : 0;
        }
        const std::vector<double>& v = M.dirichlet_value_vectors[M.voxel_index(i, j, k)];
        for (int d = 0; d < S; ++d) st.plane[(static_cast<size_t>(a) * nb + b) * S + d] = v[d];
      }
    if (failed("bfvm_set_dirichlet_face", bfvm_set_dirichlet_face(ctx, face, st.plane.data()))) return;
  }

  if (!st.resident || !st.uploaded) {
    if (failed("bfvm_upload_field", bfvm_upload_field(ctx, M.p_density_vectors->data()))) return;
    st.uploaded = true;
  }

  int flags = 0;
  if (!send_agents(st, dt, &flags)) return;
  if (failed("bfvm_step", bfvm_step(ctx, 1, flags))) return;
  finish_step(M, st, flags);
}

void bfvm_b200_lod3d_serial(Microenvironment& M, double dt) {
  static mpi_Environment world;
  static mpi_Cartesian cart;
  world.size = 1;
  world.rank = 0;
  diffusion_decay_solver__constant_coefficients_LOD_3D(M, dt, world, cart);
}

void bfvm_b200_lod2d_serial(Microenvironment& M, double dt) {
  if (M.mesh.regular_mesh == false) {
    std::cout << "Error: This algorithm is written for regular Cartesian meshes. Try: something else." << std::endl
              << std::endl;
    return;
  }
  if (M.mesh.z_coordinates.size() != 1) {
    std::cout << "Error: the B200 2-D LOD solver needs a mesh one voxel deep in z." << std::endl;
    return;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState* sp = state_for(M, dt);
  if (sp == nullptr) return;
  DropinState& st = *sp;
  bfvm_ctx* ctx = st.ctx;
  const int S = st.S;
  const int n_vox = st.nx * st.ny;

  // The nodes as the reference solver meets them: its first act is
  // apply_dirichlet_conditions() (BioFVM_solvers.cpp:1751), which writes each
  // active node value into the densities.  Node values and activations may
  // change between calls, so they are read again every call: the node
  // densities are saved, apply_dirichlet_conditions() writes the values, they
  // are read and the saved densities put back, so that fused sources see the
  // densities the reference's agent loop (run before the solver) would.
  std::vector<double>& rho = *M.p_density_vectors;
  st.node_voxel.clear();
  for (int v = 0; v < n_vox; ++v)
    if (M.is_dirichlet_node(v)) st.node_voxel.push_back(v);
  const size_t n_nodes = st.node_voxel.size();
  st.node_value.resize(n_nodes * S);
  st.node_active.resize(n_nodes * S);
  for (size_t q = 0; q < n_nodes; ++q)
    for (int d = 0; d < S; ++d) st.node_value[q * S + d] = rho[static_cast<size_t>(st.node_voxel[q]) * S + d];
  M.apply_dirichlet_conditions();
  for (size_t q = 0; q < n_nodes; ++q)
    for (int d = 0; d < S; ++d) {
      const size_t at = static_cast<size_t>(st.node_voxel[q]) * S + d;
      const double saved = st.node_value[q * S + d];
      st.node_value[q * S + d] = rho[at];
      st.node_active[q * S + d] = M.get_substrate_dirichlet_activation(d, st.node_voxel[q]) ? 1 : 0;
      rho[at] = saved;
    }
  if (failed("bfvm_set_dirichlet_nodes",
             bfvm_set_dirichlet_nodes(ctx, static_cast<int>(n_nodes), st.node_voxel.data(),
                                      st.node_value.data(), st.node_active.data())))
    return;

  if (!st.resident || !st.uploaded) {
    if (failed("bfvm_upload_field", bfvm_upload_field(ctx, M.p_density_vectors->data()))) return;
    st.uploaded = true;
  }

  int flags = 0;
  if (!send_agents(st, dt, &flags)) return;
  if (failed("bfvm_step_2d", bfvm_step_2d(ctx, 1, flags))) return;
  finish_step(M, st, flags);
}

void bfvm_b200_install(Microenvironment& M) {
  M.diffusion_decay_solver_mpi = diffusion_decay_solver__constant_coefficients_LOD_3D;
  M.diffusion_decay_solver = bfvm_b200_lod3d_serial;
}

void bfvm_b200_install_2d(Microenvironment& M) { M.diffusion_decay_solver = bfvm_b200_lod2d_serial; }

int bfvm_b200_set_fused_sources(Microenvironment& M, std::vector<Basic_Agent*>* agents, double dt) {
  (void)dt;
  std::lock_guard<std::mutex> lock(g_mu);
  table()[&M].agents = agents;
  return BFVM_OK;
}

int bfvm_b200_set_resident(Microenvironment& M, bool resident) {
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState& st = table()[&M];
  st.resident = resident;
  st.uploaded = false;
  return BFVM_OK;
}

int bfvm_b200_sync_to_host(Microenvironment& M) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = table().find(&M);
  if (it == table().end() || it->second.ctx == nullptr) return BFVM_ERR_STATE;
  return bfvm_download_field(it->second.ctx, M.p_density_vectors->data());
}

void bfvm_b200_release(Microenvironment& M) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = table().find(&M);
  if (it == table().end()) return;
  if (it->second.ctx) bfvm_destroy(it->second.ctx);
  table().erase(it);
}

}  // namespace BioFVM
