// bfvm_agents.h -- device agent list: constants, stable voxel sort, line CSR,
// standalone source/sink stage and density sampling.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "bfvm_internal.h"

namespace bfvm {

struct AgentBuild {
  int n;                       // agents in the list (active or not)
  int S, nx, ny, nz;
  const int* voxel;            // [n] reference voxel index, <0 = none
  const unsigned char* active; // [n] or nullptr (all active)
  const double* c1;            // [n][S] constants in agent-list order
  const double* c2;
  const double* e2;
  void* scratch;               // agent_scratch_bytes(n) bytes of device memory
  // outputs
  unsigned* dev_voxel;         // [n] device voxel id per agent (list order); nx*ny*nz = none
  unsigned* sorted_keys;       // [n] device voxel ids, ascending (stable)
  int* sorted_vals;            // [n] agent index per sorted position
  int* line_off;               // [ny*nz + 1] CSR over x-lines (line = k*ny + j)
  int* a_i;                    // [n] x index per sorted position
  double* ac1;                 // [S][n] constants per sorted position
  double* ac2;
  double* ae2;
  int* n_valid;                // device scalar: agents with a voxel
  int* agent_pos = nullptr;    // [n] or nullptr: sorted position of each list index
  cudaEvent_t constants_ready; // or nullptr: c1/c2/e2 are written by work this event completes
};

size_t agent_scratch_bytes(int n);

cudaError_t agents_compute_constants(int n, int S, double dt, double voxel_volume, const double* volume,
                                     const double* sec, const double* upt, const double* sat, const double* exp_,
                                     double* c1, double* c2, double* e2, cudaStream_t st, double* e1 = nullptr);

// Sorts and bins the list; *launches receives the number of kernels launched.
cudaError_t agents_build(const AgentBuild& b, cudaStream_t st, int* launches);

// Stable sort of the list by device voxel id inside caller-provided scratch of
// agent_scratch_bytes(n) bytes (nothing else is written).  On return
// *sorted_keys / *sorted_order point into the scratch: the sorted voxel ids
// (nx*ny*nz = no voxel) and the agent index at each sorted position.
cudaError_t agents_sort(int n, const int* voxel, const unsigned char* active, int nx, int ny, int nz, void* scratch,
                        cudaStream_t st, const unsigned** sorted_keys, const int** sorted_order, int* launches);

// New constants c1/c2/e2 (v1/v2/v3, rows [m][S]) for the m list indices idx
// of a built list of n agents, written to the list-order arrays [n][S] and,
// through agent_pos (from agents_build), to the sorted arrays [S][n].  The
// indices must be distinct and in [0, n).
cudaError_t agents_update_constants(int m, int S, int n, const int* idx, const double* v1, const double* v2,
                                    const double* v3, const int* agent_pos, double* c1, double* c2, double* e2,
                                    double* ac1, double* ac2, double* ae2, cudaStream_t st);

// Loads the kernels of agents_sort and agents_apply_sources_by_order on the
// current device (lazy module loading would otherwise load them, and
// allocate device memory for their code, at their first launch).
cudaError_t agents_preload_sort_kernels();

// Source/sink stage from a sort made by agents_sort, constants c1/c2/e2 in
// agent-list layout [n][S]; off as below.
template <typename T>
cudaError_t agents_apply_sources_by_order(int n, const unsigned* sorted_keys, const int* sorted_order, int S, int nx,
                                          int ny, int nz, int nxp, const double* c1, const double* c2,
                                          const double* e2, const double* off, T* f, cudaStream_t st);

// off: [S] field offsets of an FP32 solve (the field holds rho - off), or null.
// track: internalized-substrate tracking (track.internal null: off).
// Substrates s_lo .. s_hi - 1 only (s_hi < 0: through S - 1).
template <typename T>
cudaError_t agents_apply_sources(int n, const unsigned* sorted_keys, int S, int nx, int ny, int nz, int nxp,
                                 const double* ac1, const double* ac2, const double* ae2, const double* off, T* f,
                                 const AgentTrack& track, cudaStream_t st, int s_lo = 0, int s_hi = -1);

// dst[s*n + p] = src[order[p]*S + s]: a per-agent [n][S] array in list order
// gathered into the sorted, substrate-major layout of ac1/ac2/ae2.
cudaError_t agents_gather_sorted(int n, int S, const int* order, const double* src, double* dst, cudaStream_t st);

template <typename T>
cudaError_t agents_sample(int n, const unsigned* dev_voxel, int S, int nx, int ny, int nz, int nxp, const T* f,
                          const double* off, double* out, cudaStream_t st);

}  // namespace bfvm
