/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE (part of the oracle).
 *
 * A small extern "C" driver around the reference BioFVM public API, compiled
 * together with the unmodified reference sources (BioFVM/*.cpp, DistPhy/*.cpp)
 * and the single-rank MPI shim (oracle/mpi_shim/mpi.h) into
 * oracle/_ref/libbiofvm_ref.so by oracle/Makefile.  Only the tests, smoke()
 * and bench.py's CPU-baseline leg load that library, as the test oracle.
 *
 * What it drives (all reference code, nothing re-implemented here):
 *   - Microenvironment::resize_space(..., world, cart)   BioFVM_microenvironment.cpp:584-607
 *   - set_density / add_density                           BioFVM_microenvironment.cpp
 *   - update_dirichlet_node / set_substrate_dirichlet_activation  :224-282
 *   - apply_dirichlet_boundaries_conditions(rank,size)    :348-446
 *   - diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING  BioFVM_solvers.cpp:102-780
 *   - diffusion_decay_solver__constant_coefficients_LOD_3D_AVX256D   BioFVM_solvers.cpp:796-1665
 *   - Microenvironment::simulate_cell_sources_and_sinks(list, dt)     :1370-1379
 *       -> Basic_Agent::simulate_secretion_and_uptake      BioFVM_basic_agent.cpp:509-559
 *       -> Basic_Agent::set_internal_uptake_constants      BioFVM_basic_agent.cpp:224-274
 *   - Basic_Agent::assign_position / update_voxel_index    BioFVM_basic_agent.cpp:159-186
 *
 * With -DBFVM_WITH_DROPIN the same driver can also route a step through the
 * project's drop-in definition of the 4-argument
 * diffusion_decay_solver__constant_coefficients_LOD_3D (declared at
 * BioFVM_solvers.h:66, friend at BioFVM_microenvironment.h:349), which is how
 * the drop-in is tested inside the reference's own Microenvironment.
 */
#include <omp.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>
#include <vector>

#include "BioFVM.h"
#include "BioFVM_agent_container.h"
#include "BioFVM_MultiCellDS.h"
#include "BioFVM_solvers.h"
#include "DistPhy/DistPhy_Cartesian.h"
#include "DistPhy/DistPhy_Environment.h"

using namespace BioFVM;
using DistPhy::mpi::mpi_Cartesian;
using DistPhy::mpi::mpi_Environment;

#ifdef BFVM_WITH_DROPIN
namespace BioFVM {
/* Provided by physicell-x_b200/host/biofvm_b200_dropin.cpp. */
void bfvm_b200_release(Microenvironment& M);
int bfvm_b200_set_fused_sources(Microenvironment& M, std::vector<Basic_Agent*>* agents, double dt);
void bfvm_b200_install_2d(Microenvironment& M);
}
#endif

namespace {

mpi_Environment g_world;
mpi_Cartesian g_cart;
bool g_mpi_ready = false;

void ensure_world() {
  if (g_mpi_ready) return;
  g_world.Initialize();
  g_cart.Build_Cartesian_Topology(g_world);
  g_cart.Find_Cartesian_Coordinates(g_world);
  g_cart.Find_Left_Right_Neighbours(g_world);
  g_mpi_ready = true;
}

struct RefEnv {
  Microenvironment* M = nullptr;
  std::vector<Basic_Agent*> agents;
  int nx = 0, ny = 0, nz = 0, S = 0;
};

}  // namespace

extern "C" {

/* Create a uniform nx*ny*nz grid of edge dx starting at (x0,y0,z0), with S
 * substrates of the given diffusion coefficients and decay rates.  Returns
 * NULL if the reference mesh does not come out with the requested shape. */
void* ref_env_create(int nx, int ny, int nz, double dx, double x0, double y0, double z0, int S,
                     const double* D, const double* decay) {
  ensure_world();
  RefEnv* e = new RefEnv();
  e->M = new Microenvironment("oracle");
  e->M->agent_container = new Agent_Container();
  Microenvironment& M = *e->M;
  M.set_density(0, "s0", "none", D[0], decay[0]);
  for (int d = 1; d < S; ++d) {
    char name[32];
    std::snprintf(name, sizeof(name), "s%d", d);
    M.add_density(name, "none", D[d], decay[d]);
  }
  M.resize_space(x0, x0 + nx * dx, y0, y0 + ny * dx, z0, z0 + nz * dx, dx, dx, dx, g_world, g_cart);
  M.diffusion_decay_solver_mpi = diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING;
  if ((int)M.mesh.x_coordinates.size() != nx || (int)M.mesh.y_coordinates.size() != ny ||
      (int)M.mesh.z_coordinates.size() != nz || (int)M.number_of_densities() != S) {
    std::fprintf(stderr, "ref_env_create: mesh came out %zu x %zu x %zu (S=%u)\n",
                 M.mesh.x_coordinates.size(), M.mesh.y_coordinates.size(),
                 M.mesh.z_coordinates.size(), M.number_of_densities());
    delete e->M;
    delete e;
    return nullptr;
  }
  e->nx = nx;
  e->ny = ny;
  e->nz = nz;
  e->S = S;
  return e;
}

void ref_env_destroy(void* h) {
  RefEnv* e = static_cast<RefEnv*>(h);
  if (!e) return;
#ifdef BFVM_WITH_DROPIN
  bfvm_b200_release(*e->M);
#endif
  for (Basic_Agent* a : e->agents) delete a;
  delete e->M->agent_container;
  delete e->M;
  delete e;
}

long long ref_env_num_values(void* h) {
  RefEnv* e = static_cast<RefEnv*>(h);
  return (long long)e->nx * e->ny * e->nz * e->S;
}

/* Field in the reference layout: flat [x][y][z][substrate]. */
void ref_env_set_field(void* h, const double* aos) {
  RefEnv* e = static_cast<RefEnv*>(h);
  std::memcpy(e->M->p_density_vectors->data(), aos, sizeof(double) * ref_env_num_values(h));
}

void ref_env_get_field(void* h, double* aos) {
  RefEnv* e = static_cast<RefEnv*>(h);
  std::memcpy(aos, e->M->p_density_vectors->data(), sizeof(double) * ref_env_num_values(h));
}

void ref_env_set_dirichlet_activation(void* h, int substrate, int on) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->set_substrate_dirichlet_activation(substrate, on != 0);
}

/* Dirichlet values for every voxel on the six outer faces, read from a full
 * grid in the reference layout (interior entries are ignored). */
void ref_env_set_dirichlet_face_values(void* h, const double* aos) {
  RefEnv* e = static_cast<RefEnv*>(h);
  const int nx = e->nx, ny = e->ny, nz = e->nz, S = e->S;
  std::vector<double> v(S);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        if (!(i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1)) continue;
        int vox = e->M->voxel_index(i, j, k);
        for (int d = 0; d < S; ++d) v[d] = aos[(long long)vox * S + d];
        e->M->update_dirichlet_node(vox, v);
      }
}

void ref_env_apply_dirichlet(void* h) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->apply_dirichlet_boundaries_conditions(0, 1);
}

/* The Microenvironment's names and units: name, mesh.units, spatial_units,
 * time_units, and substrate d's density_names[d] / density_units[d]. */
void ref_env_set_names(void* h, const char* domain, const char* mesh_units, const char* spatial_units,
                       const char* time_units) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->name = domain;
  e->M->mesh.units = mesh_units;
  e->M->spatial_units = spatial_units;
  e->M->time_units = time_units;
}

void ref_env_set_density_name(void* h, int d, const char* name, const char* units) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->density_names[d] = name;
  e->M->density_units[d] = units;
}

/* mesh.bounding_box [6]. */
void ref_env_bounding_box(void* h, double* out) {
  RefEnv* e = static_cast<RefEnv*>(h);
  for (int q = 0; q < 6; ++q) out[q] = e->M->mesh.bounding_box[q];
}

/* add_BioFVM_substrates_to_open_xml_pugi(biofvm_doc, base, M)
 * (BioFVM_MultiCellDS.cpp:518-823) -- its first call in a process builds the
 * <microenvironment> element and writes base_mesh0.mat and
 * base_microenvironment0.mat -- then the global document as pugixml saves
 * it (save_BioFVM_to_MultiCellDS_xml_pugi, :1880-1890) copied into out.
 * Returns the text's length, or -1 if it does not fit in cap bytes. */
long ref_env_multicellds_substrates(void* h, const char* base, char* out, long cap) {
  RefEnv* e = static_cast<RefEnv*>(h);
  add_BioFVM_substrates_to_open_xml_pugi(biofvm_doc, base, *e->M);
  std::ostringstream ss;
  biofvm_doc.save(ss);
  const std::string t = ss.str();
  if (static_cast<long>(t.size()) + 1 > cap) return -1;
  std::memcpy(out, t.c_str(), t.size() + 1);
  return static_cast<long>(t.size());
}

/* Microenvironment::add_dirichlet_node(voxel, values [S])
 * (BioFVM_microenvironment.cpp:218-225). */
void ref_env_add_dirichlet_node(void* h, int voxel, const double* values) {
  RefEnv* e = static_cast<RefEnv*>(h);
  std::vector<double> v(values, values + e->S);
  e->M->add_dirichlet_node(voxel, v);
}

/* Microenvironment::remove_dirichlet_node (BioFVM_microenvironment.cpp:247-252). */
void ref_env_remove_dirichlet_node(void* h, int voxel) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->remove_dirichlet_node(voxel);
}

/* Microenvironment::set_substrate_dirichlet_activation(substrate, voxel, on)
 * (BioFVM_microenvironment.cpp:288-292): one voxel's activation. */
void ref_env_set_node_activation(void* h, int voxel, int substrate, int on) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->set_substrate_dirichlet_activation(substrate, voxel, on != 0);
}

/* Microenvironment::apply_dirichlet_conditions (BioFVM_microenvironment.cpp:303-323). */
void ref_env_apply_dirichlet_conditions(void* h) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->apply_dirichlet_conditions();
}

/* One call of diffusion_decay_solver__constant_coefficients_LOD_2D(M, dt)
 * (BioFVM_solvers.cpp:1668-1832).  Callers keep to shapes where its loops
 * stay inside the density array (ny == 1). */
void ref_env_lod2d(void* h, double dt) {
  RefEnv* e = static_cast<RefEnv*>(h);
  diffusion_decay_solver__constant_coefficients_LOD_2D(*e->M, dt);
}

/* Add one agent through the reference API.  Rates are [S] arrays.  Returns
 * the agent's index in this environment's list, or -1 if the reference
 * rejects the position. */
int ref_env_add_agent(void* h, double x, double y, double z, double volume, const double* secretion,
                      const double* uptake, const double* saturation, const double* net_export) {
  RefEnv* e = static_cast<RefEnv*>(h);
  Basic_Agent* a = new Basic_Agent();
  a->register_microenvironment(e->M);
  if (!a->assign_position(x, y, z)) {
    delete a;
    return -1;
  }
  for (int d = 0; d < e->S; ++d) {
    (*a->secretion_rates)[d] = secretion[d];
    (*a->uptake_rates)[d] = uptake[d];
    (*a->saturation_densities)[d] = saturation[d];
    (*a->net_export_rates)[d] = net_export[d];
  }
  a->set_total_volume(volume);
  e->agents.push_back(a);
  return (int)e->agents.size() - 1;
}

int ref_env_num_agents(void* h) { return (int)static_cast<RefEnv*>(h)->agents.size(); }

int ref_env_agent_voxel(void* h, int a) {
  return static_cast<RefEnv*>(h)->agents[a]->get_current_voxel_index();
}

/* The agent's implicit source/sink constants for time step dt, as the
 * reference computes them (set_internal_uptake_constants). */
void ref_env_agent_constants(void* h, int a, double dt, double* c1, double* c2, double* e2) {
  RefEnv* e = static_cast<RefEnv*>(h);
  Basic_Agent* ag = e->agents[a];
  ag->set_internal_uptake_constants(dt);
  for (int d = 0; d < e->S; ++d) {
    c1[d] = ag->get_cell_source_sink_solver_temp1()[d];
    c2[d] = ag->get_cell_source_sink_solver_temp2()[d];
    e2[d] = ag->get_cell_source_sink_solver_temp_export2()[d];
  }
}

/* simulate_cell_sources_and_sinks over this environment's agents with the
 * given OpenMP thread count (1 = the deterministic oracle mode). */
void ref_env_sources(void* h, double dt, int threads) {
  RefEnv* e = static_cast<RefEnv*>(h);
  omp_set_num_threads(threads > 0 ? threads : 1);
  e->M->simulate_cell_sources_and_sinks(e->agents, dt);
}

/* One diffusion-decay step.  solver: 0 = _BLOCKING (what
 * initialize_microenvironment(world,cart) installs), 1 = _AVX256D (constructor
 * default; it has no final Dirichlet pin), 2 = the project's drop-in (only in
 * the drop-in build).  Returns 0, or -1 for an unknown solver. */
int ref_env_diffusion(void* h, double dt, int solver, int threads) {
  RefEnv* e = static_cast<RefEnv*>(h);
  omp_set_num_threads(threads > 0 ? threads : 1);
  switch (solver) {
    case 0:
      e->M->diffusion_decay_solver_mpi = diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING;
      break;
    case 1:
      e->M->diffusion_decay_solver_mpi = diffusion_decay_solver__constant_coefficients_LOD_3D_AVX256D;
      break;
#ifdef BFVM_WITH_DROPIN
    case 2:
      e->M->diffusion_decay_solver_mpi = diffusion_decay_solver__constant_coefficients_LOD_3D;
      break;
#endif
    default:
      return -1;
  }
  e->M->simulate_diffusion_decay(dt, g_world, g_cart);
  return 0;
}

/* nsteps of [sources (sources_threads) ; diffusion (solver, threads)]. */
int ref_env_run(void* h, double dt, int nsteps, int solver, int threads, int sources_threads) {
  RefEnv* e = static_cast<RefEnv*>(h);
  for (int s = 0; s < nsteps; ++s) {
    if (!e->agents.empty()) ref_env_sources(h, dt, sources_threads);
    if (ref_env_diffusion(h, dt, solver, threads) != 0) return -1;
  }
  return 0;
}

int ref_has_dropin(void) {
#ifdef BFVM_WITH_DROPIN
  return 1;
#else
  return 0;
#endif
}

#ifdef BFVM_WITH_DROPIN
/* Route this environment's agents through the drop-in's fused GPU source
 * stage on every following drop-in step (pass enable=0 to turn it off). */
int ref_env_dropin_fuse_sources(void* h, int enable, double dt) {
  RefEnv* e = static_cast<RefEnv*>(h);
  return bfvm_b200_set_fused_sources(*e->M, enable ? &e->agents : nullptr, dt);
}

/* One step of the drop-in's 2-D solver, installed in the serial slot and run
 * through Microenvironment::simulate_diffusion_decay(dt) as a caller of the
 * reference's 2-D solver would. */
void ref_env_dropin_lod2d(void* h, double dt) {
  RefEnv* e = static_cast<RefEnv*>(h);
  bfvm_b200_install_2d(*e->M);
  e->M->simulate_diffusion_decay(dt);
}
#endif

int ref_max_threads(void) { return omp_get_max_threads(); }

/* Bulk sources and sinks: per-voxel supply rate S, target density T and
 * uptake rate U [voxel][S] served to Microenvironment's three callback
 * pointers (BioFVM_microenvironment.h:210-212) from arrays the caller owns,
 * then one Microenvironment::simulate_bulk_sources_and_sinks(dt)
 * (BioFVM_microenvironment.cpp:1327-1368). */
namespace {
struct BulkRates {
  const double *S = nullptr, *T = nullptr, *U = nullptr;
  int n = 0;
};
std::map<const Microenvironment*, BulkRates>& bulk_table() {
  static std::map<const Microenvironment*, BulkRates> t;
  return t;
}
void bulk_copy(const double* src, Microenvironment* M, int voxel, double* dst) {
  const int n = bulk_table()[M].n;
  std::memcpy(dst, src + (size_t)voxel * n, sizeof(double) * n);
}
void bulk_supply(Microenvironment* M, int v, double* w) { bulk_copy(bulk_table()[M].S, M, v, w); }
void bulk_target(Microenvironment* M, int v, double* w) { bulk_copy(bulk_table()[M].T, M, v, w); }
void bulk_uptake(Microenvironment* M, int v, double* w) { bulk_copy(bulk_table()[M].U, M, v, w); }
}  // namespace

void ref_env_bulk(void* h, double dt, const double* supply, const double* target, const double* uptake,
                  int threads) {
  RefEnv* e = static_cast<RefEnv*>(h);
  Microenvironment& M = *e->M;
  BulkRates& r = bulk_table()[&M];
  r.S = supply;
  r.T = target;
  r.U = uptake;
  r.n = e->S;
  M.bulk_supply_rate_function = bulk_supply;
  M.bulk_supply_target_densities_function = bulk_target;
  M.bulk_uptake_rate_function = bulk_uptake;
  omp_set_num_threads(threads > 0 ? threads : 1);
  M.simulate_bulk_sources_and_sinks(dt);
}

/* Microenvironment_Options::track_internalized_substrates_in_each_agent
 * (BioFVM_microenvironment.h:477), read by every agent's
 * simulate_secretion_and_uptake (BioFVM_basic_agent.cpp:520-532, 553-556). */
void ref_set_tracking(int on) { default_microenvironment_options.track_internalized_substrates_in_each_agent = on != 0; }

/* Agent a's internalized_substrates [S] (BioFVM_basic_agent.h:134). */
void ref_env_agent_internalized(void* h, int a, double* out) {
  RefEnv* e = static_cast<RefEnv*>(h);
  const std::vector<double>& v = *e->agents[a]->internalized_substrates;
  for (int d = 0; d < e->S; ++d) out[d] = d < (int)v.size() ? v[d] : 0.0;
}

/* Overwrite agent a's internalized_substrates [S]. */
void ref_env_agent_set_internalized(void* h, int a, const double* in) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->agents[a]->internalized_substrates->assign(in, in + e->S);
}

/* Basic_Agent::release_internalized_substrates (BioFVM_basic_agent.cpp:
 * 310-333) for agent a with fraction_released_at_death = fraction [S]; the
 * reference reads the default microenvironment, which is set to this one. */
void ref_env_agent_release(void* h, int a, const double* fraction) {
  RefEnv* e = static_cast<RefEnv*>(h);
  set_default_microenvironment(e->M);
  e->agents[a]->fraction_released_at_death->assign(fraction, fraction + e->S);
  e->agents[a]->release_internalized_substrates();
}

/* Microenvironment::write_to_matlab(filename) (BioFVM_microenvironment.cpp:
 * 1222-1249): MATLAB v4 header, then one column [cx, cy, cz, volume,
 * densities...] per voxel. */
void ref_env_write_matlab(void* h, const char* path) {
  RefEnv* e = static_cast<RefEnv*>(h);
  e->M->write_to_matlab(std::string(path));
}

/* Microenvironment::compute_all_gradient_vectors
 * (BioFVM/BioFVM_microenvironment.cpp:1454-1616), read back through the
 * public gradient_vector(n) accessor (:1431-1441) as out[(n*S + d)*3 + axis].
 * The reference caches 2*dx in function statics on its first call, so every
 * environment of one process must share dx for its results to be valid. */
void ref_env_gradients(void* h, double* out) {
  RefEnv* e = static_cast<RefEnv*>(h);
  Microenvironment& M = *e->M;
  M.compute_all_gradient_vectors();
  const long nv = (long)e->nx * e->ny * e->nz;
  for (long n = 0; n < nv; ++n) {
    std::vector<gradient>& g = M.gradient_vector((int)n);
    for (int d = 0; d < e->S; ++d)
      for (int a = 0; a < 3; ++a) out[(n * e->S + d) * 3 + a] = g[d][a];
  }
}

}  // extern "C"
