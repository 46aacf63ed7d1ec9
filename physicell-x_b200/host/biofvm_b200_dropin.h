// biofvm_b200_dropin.h -- C++ drop-in of the B200 LOD solver for PhysiCell-X.
//
// Compile biofvm_b200_dropin.cpp inside a PhysiCell-X tree (it includes the
// reference headers BioFVM/BioFVM_microenvironment.h and friends), link
// libbiofvm_b200.so, and install the solver:
//
//     BioFVM::bfvm_b200_install(microenvironment);
//
// which sets Microenvironment::diffusion_decay_solver_mpi
// (BioFVM_microenvironment.h:206) to the reference's own declared entry
// diffusion_decay_solver__constant_coefficients_LOD_3D(M, dt, world, cart)
// (BioFVM_solvers.h:66, a friend of Microenvironment at
// BioFVM_microenvironment.h:349, defined by this library).
// Microenvironment::simulate_diffusion_decay(dt, world, cart) then runs on the
// GPU with unchanged call sites.
#pragma once

#include <vector>

#include "BioFVM_microenvironment.h"

namespace BioFVM {

class Basic_Agent;

// Point both solver slots of M at the B200 solver (the 2-argument slot gets a
// one-rank wrapper).
void bfvm_b200_install(Microenvironment& M);

// The 2-argument (serial) signature, for Microenvironment::diffusion_decay_solver.
void bfvm_b200_lod3d_serial(Microenvironment& M, double dt);

// The 2-D LOD solver, diffusion_decay_solver__constant_coefficients_LOD_2D
// (BioFVM_solvers.cpp:1668-1832), on the GPU for meshes one voxel deep in z:
// Dirichlet nodes (add_dirichlet_node, per-voxel activation) pinned before and
// after each sweep.  bfvm_b200_install_2d points the serial slot
// (Microenvironment::diffusion_decay_solver) at it, so
// M.simulate_diffusion_decay(dt) runs it.  Agents, resident mode and release
// are shared with the 3-D solver below.
void bfvm_b200_lod2d_serial(Microenvironment& M, double dt);
void bfvm_b200_install_2d(Microenvironment& M);

// Apply the given agents' sources/sinks on the GPU, fused ahead of every
// following LOD step of M (agents == nullptr turns it off).  The caller then
// must not also call M.simulate_cell_sources_and_sinks for those steps.
// With default_microenvironment_options.track_internalized_substrates_in_each_agent
// on, each step also updates every agent's internalized_substrates, as the
// reference's agent loop would.
int bfvm_b200_set_fused_sources(Microenvironment& M, std::vector<Basic_Agent*>* agents, double dt);

// Resident mode: the field stays on the GPU between steps and the host copy
// is refreshed only by bfvm_b200_sync_to_host.  Off by default (mirrored
// mode: each step uploads M's densities and writes the result back, so host
// code reading density vectors sees every step).
int bfvm_b200_set_resident(Microenvironment& M, bool resident);
int bfvm_b200_sync_to_host(Microenvironment& M);

// Release M's GPU state (call before destroying M).
void bfvm_b200_release(Microenvironment& M);

}  // namespace BioFVM
