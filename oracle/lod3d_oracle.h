/*
 * lod3d_oracle.h -- TEST INFRASTRUCTURE: the CPU oracle (plain C restatement)
 * of PhysiCell-X's BioFVM 3-D LOD diffusion-decay step and cell
 * sources/sinks.  Only tests, smoke() and bench.py's CPU-baseline leg may
 * call it; it is the test oracle, never the product.
 *
 * Layout is the reference's: one flat array, index ((i*ny + j)*nz + k)*S + d
 * (Cartesian_Mesh::voxel_index, BioFVM/BioFVM_mesh.cpp:1149-1158, times the
 * substrate count as in Microenvironment::density_vector,
 * BioFVM/BioFVM_microenvironment.cpp:1123-1130).
 *
 * Parity status: pinned against the reference itself.  The reference ships
 * no golden vectors for this path, so tests/test_oracle.py compares this
 * restatement bit for bit with the reference's own solver built from its
 * sources (oracle/_ref/libbiofvm_ref.so), and tests/golden/ holds fixtures
 * generated from that build.
 */
#ifndef BFVM_LOD3D_ORACLE_H
#define BFVM_LOD3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Thomas coefficients of one axis with n voxels, for S substrates.
 * Outputs denom[n*S], cupper[n*S] (index i*S+d) and c1[S].
 * Restates BioFVM/BioFVM_solvers.cpp:196-329 (one rank). */
void orc_thomas_axis(int n, int S, const double* D, const double* decay, double dt, double dx,
                     double* denom, double* cupper, double* c1);

/* The Dirichlet pin: every voxel on the six outer faces takes its value from
 * dirichlet_values (same layout as the field) for each substrate d with
 * active[d] != 0.  Restates Microenvironment::apply_dirichlet_boundaries_conditions
 * BioFVM/BioFVM_microenvironment.cpp:348-446 (rank 0 of 1). */
void orc_apply_dirichlet(double* field, int nx, int ny, int nz, int S, const unsigned char* active,
                         const double* dirichlet_values);

/* One diffusion-decay LOD step: pin; x sweep; pin; y sweep; pin; z sweep; pin.
 * Restates diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING,
 * BioFVM/BioFVM_solvers.cpp:102-780 with one rank.  threads<=0 uses the
 * OpenMP default; the result does not depend on the thread count. */
void orc_lod3d_step(double* field, int nx, int ny, int nz, int S, const double* D,
                    const double* decay, double dt, double dx, const unsigned char* active,
                    const double* dirichlet_values, int threads);

/* Per-agent implicit source/sink constants for one time step.
 * Restates Basic_Agent::set_internal_uptake_constants,
 * BioFVM/BioFVM_basic_agent.cpp:224-274.  Outputs c1,c2,e2 [S]. */
void orc_agent_constants(int S, double dt, double agent_volume, double voxel_volume,
                         const double* secretion, const double* uptake, const double* saturation,
                         const double* net_export, double* c1, double* c2, double* e2);

/* Apply agents in list order to their voxels (one thread, the reference's
 * deterministic order).  voxel[a] is the reference linear voxel index; agents
 * with active[a]==0 or voxel[a]<0 are skipped.  c1,c2,e2 are [n][S].
 * Restates Basic_Agent::simulate_secretion_and_uptake,
 * BioFVM/BioFVM_basic_agent.cpp:509-559, driven as in
 * Microenvironment::simulate_cell_sources_and_sinks (:1370-1379). */
void orc_sources(double* field, int S, int n_agents, const int* voxel, const unsigned char* active,
                 const double* c1, const double* c2, const double* e2);

/* Cartesian_Mesh::nearest_voxel_index for a one-rank mesh whose box starts
 * at (x0,y0,z0) (BioFVM/BioFVM_mesh.cpp:1825-1843): floor((p-x0)/dx), clamped
 * to [0,n-1].  Returns the reference linear index. */
int orc_nearest_voxel(double x, double y, double z, double x0, double y0, double z0, double dx,
                      int nx, int ny, int nz);

/* Gradients of every substrate at every voxel, out[(v*S + d)*3 + axis]:
 * one-sided differences (a - b) / dx at the two ends of each line and
 * central differences (a - b) / (2 dx) inside, each as one subtraction and
 * one division.  Restates Microenvironment::compute_all_gradient_vectors,
 * BioFVM/BioFVM_microenvironment.cpp:1454-1616.  An axis of length 1 gets 0
 * (the reference reads outside the array there; with nz == 1 it skips the z
 * component). */
void orc_gradients(const double* field, int nx, int ny, int nz, int S, double dx, double* out);

/* Bulk sources and sinks with per-voxel supply rate S, target density T and
 * uptake rate U (arrays like the field): rho = fma(dt, S*T, rho) -- the
 * reference's g++ build contracts `rho += dt * temp2` -- then
 * rho /= ((U + S) * dt) + 1.  Restates
 * Microenvironment::simulate_bulk_sources_and_sinks,
 * BioFVM/BioFVM_microenvironment.cpp:1327-1368. */
void orc_bulk_sources(double* field, long n_values, double dt, const double* supply, const double* target,
                      const double* uptake);

/* Microenvironment::write_to_matlab(filename), one rank
 * (BioFVM/BioFVM_microenvironment.cpp:1222-1249 with write_matlab4_header,
 * BioFVM/BioFVM_matlab.cpp:536-578): a 20-byte MATLAB v4 header (type 0,
 * rows 4+S, cols = voxels, imag 0, name length), the name
 * "multiscale_microenvironment" without terminator, then per voxel in
 * reference order the column [cx, cy, cz, dx*dy*dz, densities...].  Voxel
 * centres are fma(i + 0.5, dx, start) as the reference's build computes
 * x_start + (i+0.5)*dx (BioFVM/BioFVM_mesh.cpp:1436-1560).  Returns 0, or -1
 * if the file cannot be written. */
int orc_write_matlab(const char* path, const double* field, int nx, int ny, int nz, int S, double x0, double y0,
                     double z0, double dx);

/* orc_sources with the reference's tracking of internalized substrates
 * (Microenvironment_Options::track_internalized_substrates_in_each_agent;
 * BioFVM/BioFVM_basic_agent.cpp:520-532, 553-556): before agent a updates its
 * voxel, internal[a][d] -= (((1 - c2) * rho + c1) / c2) * vvox, and after it,
 * internal[a][d] -= e1[a][d] (its export in one step, net export rate * dt).
 * internal accumulates: callers start it where they want. */
void orc_sources_tracked(double* field, int S, int n, const int* voxel, const unsigned char* active, const double* c1,
                         const double* c2, const double* e2, const double* e1, double vvox, double* internal);

/* Basic_Agent::release_internalized_substrates (BioFVM/BioFVM_basic_agent.cpp:
 * 310-333) for the listed agents in order; fraction [count][S] is each
 * one's fraction_released_at_death. */
void orc_release_internalized(double* field, int S, int count, const int* agents, const int* voxel,
                              const double* fraction, double vvox, double* internal);

/* Interior Dirichlet nodes: apply_dirichlet_conditions (BioFVM_microenvironment.cpp:
 * 303-323) for a list of distinct voxels, values [count][S], act [count][S]
 * or NULL (all substrates). */
void orc_dirichlet_nodes(double* field, int S, int count, const int* voxel, const double* values,
                         const unsigned char* act);

/* One 2-D LOD step (diffusion_decay_solver__constant_coefficients_LOD_2D,
 * BioFVM/BioFVM_solvers.cpp:1668-1832) on an nx x ny x 1 grid, with the node
 * list pinned before, between and after the two sweeps. */
void orc_lod2d_step(double* p, int nx, int ny, int S, const double* D, const double* decay, double dt, double dx,
                    int count, const int* voxel, const double* values, const unsigned char* act);

#ifdef __cplusplus
}
#endif

#endif
