/*
 * biofvm_b200.h -- C ABI of the B200 implementation of BioFVM's 3-D
 * diffusion-decay LOD step with cell sources/sinks (PhysiCell-X 1.14.0).
 *
 * Plain C: opaque handles, pointers and sizes, int status codes.  Every
 * function returns BFVM_OK (0) or a negative BFVM_ERR_* code and leaves the
 * solve's state unchanged on failure.  One handle is one microenvironment
 * resident on one GPU; calls on one handle must not overlap, calls on
 * different handles may come from different threads.
 *
 * Conventions shared with the reference (so a PhysiCell-X caller can pass its
 * own buffers unchanged):
 *   - a field is a flat double array in the reference layout, index
 *     ((i*ny + j)*nz + k)*S + d  (Cartesian_Mesh::voxel_index,
 *     BioFVM/BioFVM_mesh.cpp:1149-1158; Microenvironment::density_vector,
 *     BioFVM/BioFVM_microenvironment.cpp:1123-1130);
 *   - a voxel index is ((i*ny + j)*nz + k);
 *   - per-agent arrays are [n][S] rows in agent-list order, the order of the
 *     reference's all_basic_agents (BioFVM/BioFVM_basic_agent.h:187).
 *
 * The drop-in for the reference's own C++ API (the 4-argument
 * diffusion_decay_solver__constant_coefficients_LOD_3D, BioFVM_solvers.h:66)
 * is physicell-x_b200/host/biofvm_b200_dropin.cpp, built on these calls.
 */
#ifndef BIOFVM_B200_H
#define BIOFVM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define BFVM_OK 0
#define BFVM_ERR_ARG (-1)      /* bad argument (null pointer, size, index)   */
#define BFVM_ERR_CUDA (-2)     /* a CUDA call failed                          */
#define BFVM_ERR_OOM (-3)      /* device memory (or the HBM budget) exhausted */
#define BFVM_ERR_SHAPE (-4)    /* grid not supported (extent, shared memory)  */
#define BFVM_ERR_NODEVICE (-5) /* no usable CUDA device                       */
#define BFVM_ERR_TIMEOUT (-6)  /* a bounded device-side wait gave up          */
#define BFVM_ERR_STATE (-7)    /* call not valid in the current state         */

/* ---- precision ---------------------------------------------------------- */
#define BFVM_FP64 0 /* FP64 sweeps and storage: the reference's arithmetic    */
#define BFVM_FP32 1 /* FP32 storage (half the bytes); FP64 recurrence,         */
                    /* coefficients and agent updates                          */

/* ---- bfvm_step flags ----------------------------------------------------- */
#define BFVM_STEP_SOURCES 1 /* apply the agents' sources/sinks ahead of each  */
                            /* step, fused into the x sweep                    */

/* Dirichlet faces, in the order the reference's setup writes them
 * (BioFVM/BioFVM_microenvironment.cpp:2647-2760). */
#define BFVM_FACE_XMIN 0
#define BFVM_FACE_XMAX 1
#define BFVM_FACE_YMIN 2
#define BFVM_FACE_YMAX 3
#define BFVM_FACE_ZMIN 4
#define BFVM_FACE_ZMAX 5

typedef struct bfvm_ctx bfvm_ctx;

typedef struct bfvm_config {
  int nx, ny, nz;                       /* voxels per axis                     */
  int n_substrates;                     /* S                                   */
  double dx;                            /* voxel edge; the mesh must be uniform */
  double dt;                            /* diffusion time step                 */
  const double* diffusion_coefficients; /* [S]                                 */
  const double* decay_rates;            /* [S]                                 */
  int precision;                        /* BFVM_FP64 or BFVM_FP32              */
  int device;                           /* CUDA device ordinal                 */
} bfvm_config;

/* Create a resident solve.  Replaces the first-call setup inside
 * diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING
 * (BioFVM/BioFVM_solvers.cpp:125-337): the Thomas factorization of all three
 * axes is computed here in FP64 with the reference's arithmetic and kept on
 * the device.  The field starts at zero (Microenvironment::resize_space,
 * BioFVM_microenvironment.cpp:610-638).  As in the reference
 * (Microenvironment::resize_densities, :645-700), every substrate starts with
 * Dirichlet activation on and value 1.0 on all six faces. */
int bfvm_create(const bfvm_config* cfg, bfvm_ctx** out);
int bfvm_destroy(bfvm_ctx* ctx);

/* Per-substrate Dirichlet activation [S] (0/1).  Replaces
 * Microenvironment::set_substrate_dirichlet_activation(int,bool)
 * (BioFVM_microenvironment.cpp:265-273); the 3-D solvers read only this
 * per-substrate flag (apply_dirichlet_boundaries_conditions, :348-446). */
int bfvm_set_dirichlet_activation(bfvm_ctx* ctx, const unsigned char* active);

/* Dirichlet values of every voxel on one face, as the reference's
 * dirichlet_value_vectors hold them (update_dirichlet_node,
 * BioFVM_microenvironment.cpp:228-244): x faces take [ny][nz][S], y faces
 * [nx][nz][S], z faces [nx][ny][S], in reference index order.  A voxel on
 * several faces must carry the same value in each (the value of its voxel). */
int bfvm_set_dirichlet_face(bfvm_ctx* ctx, int face, const double* values);

/* The same value vector [S] on every voxel of all six faces. */
int bfvm_set_dirichlet_uniform(bfvm_ctx* ctx, const double* values);

/* Copy a whole field in (host memory, reference layout).  Replaces writing
 * the densities through Microenvironment::density_vector (:1123-1130). */
int bfvm_upload_field(bfvm_ctx* ctx, const double* field);
/* Copy the whole field out (host memory, reference layout). */
int bfvm_download_field(bfvm_ctx* ctx, double* field);
/* Same two calls with device pointers (reference layout in device memory). */
int bfvm_upload_field_device(bfvm_ctx* ctx, const double* d_field);
int bfvm_download_field_device(bfvm_ctx* ctx, double* d_field);

/* Agent list from precomputed constants: voxel [n] (reference voxel index,
 * <0 = outside), active [n] or NULL, and c1, c2, e2 [n][S] -- the agent's
 * cell_source_sink_solver_temp1, _temp2 and _temp_export2
 * (BioFVM/BioFVM_basic_agent.h:61-72).  The list is stably binned by voxel
 * on the device, so agents sharing a voxel are applied in list order, as
 * the single-threaded Microenvironment::simulate_cell_sources_and_sinks
 * (BioFVM_microenvironment.cpp:1370-1379) applies them.  Host pointers. */
int bfvm_set_agents(bfvm_ctx* ctx, int n, const int* voxel, const unsigned char* active, const double* c1,
                    const double* c2, const double* e2);

/* New constants for some agents of the current list, leaving the list, its
 * voxels and its sort as they are: idx [n_changed] distinct list indices,
 * c1, c2, e2 [n_changed][S] their new cell_source_sink_solver_temp1, _temp2
 * and _temp_export2.  The reference recomputes an agent's constants only
 * when its volume changed (Basic_Agent::simulate_secretion_and_uptake,
 * BioFVM/BioFVM_basic_agent.cpp:509-518, calling set_internal_uptake_constants,
 * :224-274), so a caller sends just those agents instead of the whole list.
 * Later source stages use the new constants; a list set from rates keeps its
 * rates (the exports tracked per agent do not change).  Host pointers;
 * BFVM_ERR_ARG for an index outside the list or given twice. */
int bfvm_update_agents(bfvm_ctx* ctx, int n_changed, const int* idx, const double* c1, const double* c2,
                       const double* e2);

/* Agent list from rates: volume [n] and secretion, uptake, saturation and
 * net-export rates [n][S]; the constants are computed on the device with the
 * arithmetic of Basic_Agent::set_internal_uptake_constants
 * (BioFVM/BioFVM_basic_agent.cpp:224-274) for this solve's dt and dx^3. */
int bfvm_set_agents_from_rates(bfvm_ctx* ctx, int n, const int* voxel, const unsigned char* active,
                               const double* volume, const double* secretion, const double* uptake,
                               const double* saturation, const double* net_export);

/* Basic_Agent::set_internal_uptake_constants (BioFVM_basic_agent.cpp:224-274)
 * for a whole agent list, with no solve attached: every pointer is device
 * memory -- volume [n], rates [n][S], outputs c1, c2, e2 [n][S] -- and
 * stream is a cudaStream_t (NULL: the default stream).  Asynchronous. */
int bfvm_agent_constants_device(int n, int S, double dt, double voxel_volume, const double* volume,
                                const double* secretion, const double* uptake, const double* saturation,
                                const double* net_export, double* c1, double* c2, double* e2, void* stream);

/* Advance nsteps LOD steps.  Each step is the reference's
 * [simulate_cell_sources_and_sinks (if flags & BFVM_STEP_SOURCES);
 *  diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING]
 * (BioFVM_microenvironment.cpp:1370-1384; BioFVM_solvers.cpp:102-780):
 * Dirichlet pin, x sweep, pin, y sweep, pin, z sweep, pin.  Asynchronous on
 * the solve's stream.  Runs of more than 16 steps replay a captured CUDA
 * graph of 16 steps (recaptured when the agents, tracking or launch settings
 * change), unless per-step timing is on or the caller is capturing the
 * solve's stream itself; the results are the same bits either way. */
int bfvm_step(bfvm_ctx* ctx, int nsteps, int flags);

/* The source/sink stage alone (one call of
 * Microenvironment::simulate_cell_sources_and_sinks(dt), :1381-1384). */
int bfvm_apply_sources(bfvm_ctx* ctx);

/* No counterpart in the reference.  One source/sink stage (the operations of
 * bfvm_apply_sources, same results) for n agents whose arrays are already in
 * device memory on the solve's device: voxel [n] (reference voxel index, <0 =
 * none), active [n] or NULL (all active), c1/c2/e2 [n][S] agent-list order.
 * The arrays are read on the solve's stream; the solve's own agent list is
 * left unchanged.  It calls no device allocator: the voxel sort runs in one
 * fixed scratch array per device inside the library, for callers that must
 * not allocate at that point (a loop whose device memory was reserved up
 * front, or code where cudaMalloc is not allowed).  Limits: n <= 262144
 * (larger: BFVM_ERR_ARG, no work queued); calls on the same device must not
 * overlap in time (they share the scratch and would race).  The first call
 * on a device (n = 0 is enough) is its set-up: it loads the scratch array and
 * the kernels into device memory and looks up the array's address, so make
 * it at set-up time, before the loop that must not allocate and before any
 * stream capture begins; later calls allocate nothing.  The address is kept
 * for the life of the process: after cudaDeviceReset on a device, do not call
 * this entry point on that device again. */
int bfvm_apply_sources_noalloc(bfvm_ctx* ctx, int n, const int* voxel, const unsigned char* active,
                               const double* c1, const double* c2, const double* e2);

/* Tracking of the substrates each agent internalizes: the reference's
 * Microenvironment_Options::track_internalized_substrates_in_each_agent
 * (BioFVM/BioFVM_microenvironment.h:477), per solve instead of per process.
 * While on, every source/sink stage (bfvm_step with BFVM_STEP_SOURCES,
 * bfvm_apply_sources, bfvm_batch_step) also keeps each agent's internalized
 * amounts [n][S] (agent-list order), as Basic_Agent::simulate_secretion_and_uptake
 * does (BioFVM/BioFVM_basic_agent.cpp:520-532, 553-556):
 *   internal -= (((1 - c2) * rho + c1) / c2) * dx^3   before the agent's update,
 *   internal -= e1                                    after it,
 * e1 = net_export_rate * dt (:261-262).  Amounts start at zero; a new agent
 * list keeps the amounts of the list positions it shares with the previous
 * list and starts the others at zero.  bfvm_apply_sources_noalloc does not
 * track.  Turning tracking off keeps nothing. */
int bfvm_set_agent_tracking(bfvm_ctx* ctx, int on);
/* e1 [n][S] (host, agent-list order) for a list set with bfvm_set_agents,
 * whose exports otherwise count as zero; bfvm_set_agents_from_rates derives
 * them from its net export rates.  Set again after every bfvm_set_agents.
 * BFVM_ERR_STATE while tracking is off. */
int bfvm_set_agent_exports(bfvm_ctx* ctx, const double* export1);
/* Read / write the internalized amounts [n][S] (host, agent-list order);
 * in == NULL writes zeros.  BFVM_ERR_STATE while tracking is off. */
int bfvm_get_internalized(bfvm_ctx* ctx, double* out);
int bfvm_set_internalized(bfvm_ctx* ctx, const double* in);
/* Basic_Agent::release_internalized_substrates (BioFVM_basic_agent.cpp:
 * 310-333) for count agents (list indices), in the order given: the voxel's
 * densities gain internal / dx^3 * fraction[q][s] and the agent's amounts
 * become zero.  fraction [count][S] host (fraction_released_at_death). */
int bfvm_release_internalized(bfvm_ctx* ctx, int count, const int* agents, const double* fraction);

/* Dirichlet nodes: any voxels (interior or on a face) with their own values
 * and per-substrate activation -- Microenvironment::add_dirichlet_node /
 * update_dirichlet_node (BioFVM/BioFVM_microenvironment.cpp:218-243) and
 * set_substrate_dirichlet_activation(substrate, voxel, on) (:288-292).
 * voxel [count] reference voxel indices, values [count][S], activation
 * [count][S] or NULL (each substrate's current activation, as set by
 * bfvm_set_dirichlet_activation).  Replaces the solve's node list (count 0
 * clears it); a voxel given twice keeps its last entry.  Host pointers. */
int bfvm_set_dirichlet_nodes(bfvm_ctx* ctx, int count, const int* voxel, const double* values,
                             const unsigned char* activation);
/* Microenvironment::apply_dirichlet_conditions (:303-323) for the node list.
 * The 3-D step pins the six faces only, as the reference's _BLOCKING solver
 * does; nodes are applied here and by bfvm_step_2d. */
int bfvm_apply_dirichlet_nodes(bfvm_ctx* ctx);
/* nsteps steps of the 2-D LOD solver, diffusion_decay_solver__constant_coefficients_LOD_2D
 * (BioFVM/BioFVM_solvers.cpp:1668-1832), on a solve with nz == 1 (else
 * BFVM_ERR_SHAPE): [sources (flags & BFVM_STEP_SOURCES)]; nodes pinned; x
 * sweep; nodes pinned; y sweep; nodes pinned; constant2 = decay*dt/2.  No
 * face is pinned by the sweeps: boundary conditions are the node list. */
int bfvm_step_2d(bfvm_ctx* ctx, int nsteps, int flags);

/* General_Mesh::write_to_matlab (BioFVM/BioFVM_mesh.cpp:425-447): MATLAB v4
 * matrix "mesh", one column per voxel in reference order (centre x, y, z,
 * volume), assembled on the device; same start arguments as
 * bfvm_write_matlab. */
int bfvm_write_mesh_matlab(bfvm_ctx* ctx, const char* path, double x_start, double y_start, double z_start);

/* The microenvironment's MultiCellDS output: what
 * add_BioFVM_substrates_to_open_xml_pugi (BioFVM/BioFVM_MultiCellDS.cpp:518-823,
 * first call, MATLAB data files) and save_BioFVM_to_MultiCellDS_xml_pugi
 * (:1880-1890) produce for this solve -- <base>_mesh0.mat,
 * <base>_microenvironment0.mat and <base>.xml, the document with the
 * <microenvironment> element and empty <metadata> and <cellular_information>
 * (the reference's metadata carries wall-clock timestamps and its agents
 * come from the cell model), byte for byte as the reference writes them.
 * Names and units are the Microenvironment's (name, mesh.units,
 * spatial_units, time_units, density_names/units [S]); bounding_box [6] is
 * mesh.bounding_box (x, y, z minima, then maxima).  xml (capacity bytes) or
 * NULL receives the document text, xml_length (or NULL) its length. */
int bfvm_write_multicellds(bfvm_ctx* ctx, const char* filename_base, const char* domain_name,
                           const char* mesh_units, const char* spatial_units, const char* time_units,
                           const char* const* density_names, const char* const* density_units,
                           const double* bounding_box, char* xml, size_t xml_capacity, size_t* xml_length);

/* Densities at each agent's voxel, [n][S] host doubles, in agent-list order
 * (what Basic_Agent::nearest_density_vector returns to each agent,
 * BioFVM/BioFVM_basic_agent.cpp:389-392). */
int bfvm_sample_agents(bfvm_ctx* ctx, double* out);

/* Per-substrate sums over all voxels, computed in FP64 on the device [S]
 * (the mass-balance check; multiply by dx^3 for total substrate). */
int bfvm_field_sums(bfvm_ctx* ctx, double* out);

/* Periodic FP64 mass-balance record: after every `every`-th step of
 * bfvm_step (counted from this call), the per-substrate sums of the
 * densities over all voxels, accumulated in FP64 on the device in a fixed
 * order (deterministic), are appended to a device ring of `capacity`
 * records.  For an FP32 solve this is the FP64 check of the FP32 field: its
 * records compare step for step with an FP64 solve's.  every = 0 turns it
 * off and frees the ring.  No counterpart in the reference (one precision;
 * its conservation printout is unit_test_conservation.cpp). */
int bfvm_set_mass_log(bfvm_ctx* ctx, int every, int capacity);
/* The records still in the ring, oldest first: out [min(kept, max_records)][S];
 * *n_total = records made since bfvm_set_mass_log (records beyond the ring's
 * capacity overwrite the oldest).  Synchronous; BFVM_ERR_STATE while off. */
int bfvm_read_mass_log(bfvm_ctx* ctx, double* out, int max_records, int* n_total);

/* Wait for the solve's stream; returns BFVM_ERR_TIMEOUT if a device-side
 * wait gave up since the last check, BFVM_ERR_CUDA on a CUDA error. */
int bfvm_synchronize(bfvm_ctx* ctx);

/* Upper bound, in nanoseconds, on every bounded device-side wait of this
 * library's kernels on one device (a TMA copy's barrier, the batched
 * engine's wait for a member's previous sweep): past it the kernel records a
 * timeout, which the next bfvm_synchronize / bfvm_batch_synchronize returns
 * as BFVM_ERR_TIMEOUT, and finishes without hanging the GPU.  Default 2 s;
 * 1000 <= ns <= 60e9.  Applies to launches made after the call.  No
 * counterpart in the reference, which has no device waits. */
int bfvm_set_wait_limit_ns(int device, unsigned long long ns);

/* The cudaStream_t the solve runs on (as void*), for event timing; NULL for a
 * NULL ctx. */
void* bfvm_stream(bfvm_ctx* ctx);
/* Run the solve on a caller-owned stream (NULL: back to its own stream). */
int bfvm_set_stream(bfvm_ctx* ctx, void* stream);

/* Device field pointer and row pitch (elements) of the device layout
 * f[S][nz][ny][pitch], x fastest -- for callers that keep data on the GPU.
 * An FP32 solve stores rho - offset[s] (see bfvm_field_offsets). */
int bfvm_device_field(bfvm_ctx* ctx, void** ptr, int* pitch, int* elem_bytes);

/* Per-substrate offsets [S] of the stored field: 0 for FP64; for FP32 the
 * mean Dirichlet face value of each activated substrate (else 0), chosen at
 * the last field upload.  Uploads, downloads, sampling and sums apply them. */
int bfvm_field_offsets(bfvm_ctx* ctx, double* offsets);

/* Bytes of device memory the solve holds now (field, coefficients, agents,
 * host-transfer staging); 0 for a NULL ctx. */
size_t bfvm_device_bytes(bfvm_ctx* ctx);

/* Bytes that bfvm_create(cfg), one host field upload and bfvm_set_agents with
 * n_agents agents would request -- for admission against a device-memory
 * budget before anything is allocated (0 for an invalid configuration).  No
 * counterpart in the reference, which has no device memory. */
size_t bfvm_estimate_bytes(const bfvm_config* cfg, int n_agents);

/* Free the buffers that host transfers stage through (the reference-layout
 * field, as large as an FP64 copy of the field, and the gradient buffer of
 * bfvm_compute_gradients); the next host transfer allocates them again.  No
 * counterpart in the reference. */
int bfvm_release_staging(bfvm_ctx* ctx);

/* Bulk (per-voxel) sources and sinks.  Replaces the three callbacks
 * Microenvironment::bulk_supply_rate_function, bulk_supply_target_densities_
 * function and bulk_uptake_rate_function (BioFVM_microenvironment.h:210-212)
 * with their values for every voxel: supply S, target T and uptake U, each a
 * host array in the field's reference layout.  Kept on the device until
 * replaced; three NULLs free them. */
int bfvm_set_bulk_rates(bfvm_ctx* ctx, const double* supply, const double* target, const double* uptake);

/* One Microenvironment::simulate_bulk_sources_and_sinks(dt)
 * (BioFVM_microenvironment.cpp:1327-1368) with the rates above:
 * rho = fma(dt, T*S, rho); rho /= ((U + S)*dt) + 1, bit for bit in FP64.
 * BFVM_ERR_STATE if no rates were set.  Asynchronous on the solve's stream. */
int bfvm_apply_bulk_sources(bfvm_ctx* ctx);

/* Microenvironment::write_to_matlab(filename)
 * (BioFVM/BioFVM_microenvironment.cpp:1222-1249, BioFVM_matlab.cpp:536-578):
 * the MATLAB v4 file with one column [cx, cy, cz, volume, densities...] per
 * voxel in reference order, for a domain whose lower corner is
 * (x_start, y_start, z_start) -- the bounding box the reference's
 * resize_space was given.  Byte-identical to the reference's file for an FP64
 * solve.  BFVM_ERR_ARG if the file cannot be written.  Synchronous. */
int bfvm_write_matlab(bfvm_ctx* ctx, const char* path, double x_start, double y_start, double z_start);

/* Gradients of every substrate at every voxel of the current field,
 * out[(v*S + d)*3 + axis] (v = reference voxel index, axis x/y/z) in host
 * memory -- Microenvironment::compute_all_gradient_vectors followed by
 * gradient_vector(v) for every voxel (BioFVM/BioFVM_microenvironment.cpp:
 * 1454-1616, 1431-1441).  One-sided differences at the line ends, central
 * inside; FP64 results equal the reference's bit for bit.  An axis of length
 * 1 gets 0 (the reference reads outside its array there).  Synchronous. */
int bfvm_compute_gradients(bfvm_ctx* ctx, double* out);

/* The same into device memory on the solve's device (3*S doubles per voxel),
 * asynchronous on the solve's stream. */
int bfvm_compute_gradients_device(bfvm_ctx* ctx, double* d_out);

/* Launch shape of the sweeps: lines per CTA in the x sweep (a multiple of 8,
 * at most 256), x extent per CTA in the y/z sweeps (16 -- FP64 only --, 32 or
 * 64) and rows per TMA box in the y/z sweeps (1..256).  The defaults fit all
 * extents up to 256 in FP64; bfvm_set_launch re-encodes the TMA descriptors
 * and returns BFVM_ERR_ARG for other values. */
int bfvm_get_launch(bfvm_ctx* ctx, int* x_lines, int* yz_tile, int* yz_chunk);
int bfvm_set_launch(bfvm_ctx* ctx, int x_lines, int yz_tile, int yz_chunk);

/* Schedule of the single-solve sweeps.  Persistent sweeps keep one CTA per SM
 * (or as many as fit) walking a sequence of 32-line tiles, loading the next
 * tile while they finish the current one (with x_lines == yz_tile == 32;
 * other shapes run per tile): in FP64, where bfvm_set_sweep_tmem allows it,
 * rings of one warp that keep forward results in shared memory or tensor
 * memory and take tiles from a shared counter; otherwise a compute warp and
 * a copy warp per ring (lines of at most 64 chunks).  persistent = 1
 * (default): y and z sweeps persistent where every ring gets at least 2
 * tiles (tensor-memory sweeps) or 8 (the others), x sweep one CTA per tile
 * except on long lines with tensor memory; 2: all three persistent whatever
 * the tile count; 0: one CTA per tile everywhere.  Every schedule computes
 * the same bits. */
int bfvm_set_sweep_schedule(bfvm_ctx* ctx, int persistent);
/* How runs of steps use the GPU: streams = 1 (default) runs every
 * substrate in one sequence of launches; 2 (solves of two or more
 * substrates) sweeps the substrates [0, ceil(S/2)) on the solve's stream and
 * the rest on a second stream, forked and joined around each run of
 * bfvm_step (and inside its captured graph), so that one group's kernels can
 * take the SMs the other's persistent sweeps leave idle while their last
 * tiles finish.  Measured on B200 at cube200 (200^3 x 4): 0.380 ms per step
 * with 2 against 0.367 with 1 (FP32 0.275 against 0.243): half-size sweeps
 * have relatively longer tails, and the launches double.  The substrates
 * never interact within a step (each launch reads and writes its own
 * planes), so both give the same bits.  No counterpart in the reference (a
 * launch control). */
int bfvm_set_substrate_streams(bfvm_ctx* ctx, int streams);
int bfvm_get_substrate_streams(const bfvm_ctx* ctx, int* streams);
/* Where bfvm_step applies the agents: fused = 0 (default) the standalone
 * source kernel ahead of the sweeps, 1 inside the x sweep, on the staged
 * tile.  Both give the same bits. */
int bfvm_set_fused_sources(bfvm_ctx* ctx, int fused);
int bfvm_get_sweep_schedule(bfvm_ctx* ctx, int* persistent);
/* Arithmetic of the FP64 forward elimination.  chain = 0 (default): the
 * reference's, operation by operation (fma, then a correctly rounded
 * division), so results are the reference's bits.  chain = 1: the short
 * chain y_i = fma(a_i, y_{i-1}, v_i * r_i) with r_i = RN(1/d_i) and
 * a_i = RN(c1 * r_i) precomputed in FP64 at set-up -- one dependent FMA per
 * element instead of an FMA and a division, and no exactness screen.  Its
 * results differ from the reference's by a few units in the last place per
 * sweep, within the 1e-12 relative per-voxel bound the FP64 path is held to
 * (the tests measure it against the oracle).  The back substitution, the
 * sources and the pins are the same in both.  chain = 2: chain 1, except
 * that long y and z lines are solved by a partition
 * method (by default on lines of at least 512 voxels in FP64 and 448 in
 * FP32, where it is the faster one): eight warps share each 32-line tile,
 * each warp running both recurrences over one eighth of the line, joined
 * through segment products that the host forms in extended precision at
 * set-up.  Its results are
 * held to the same 1e-12 bound.  The 2-D solver always uses chain 0.  An
 * FP32 solve's recurrence is FP64 too: chain 0 there is
 * t = fma(c1, y, v - shift), y = t * RN(1/d); chain 1 is
 * y = fma(c1 * RN(1/d), y, (v - shift) * RN(1/d)); chain 2 stores the
 * partitioned passes' intermediate values in FP32, so its bound is the FP32
 * path's. */
int bfvm_set_fp64_chain(bfvm_ctx* ctx, int chain);
int bfvm_get_fp64_chain(bfvm_ctx* ctx, int* chain);
/* The shortest y or z line that chain 2 solves partitioned: n_line >= 1,
 * or -1 for the default of the solve's precision (512 FP64, 448 FP32).
 * bfvm_get_partition_min_line returns the value in effect. */
int bfvm_set_partition_min_line(bfvm_ctx* ctx, int n_line);
int bfvm_get_partition_min_line(bfvm_ctx* ctx, int* n_line);

/* Tensor-memory (TMEM) rings in the persistent sweeps: on = 1 (default) in
 * the x, y and z sweeps of both precisions on lines of 33 to 736 voxels
 * (FP32 x lines to 1216; the x sweeps with agents not fused into them): up
 * to four FP64 rings, or eight FP32 rings (two per TMEM lane quarter), keep
 * the forward results of a line's first 256 values in the SM's TMEM beside
 * the shared-memory rings; 2 also in the FP64 x sweep on lines of 17 to 32;
 * 0 shared memory alone.  Every level gives the same bits. */
int bfvm_set_sweep_tmem(bfvm_ctx* ctx, int on);
/* The tensor-memory sweep a persistent sweep would run on lines of n_line
 * voxels (host arithmetic, no device needed): axis 0 = the FP64 x sweep
 * (agents not fused into it), 1 = the FP64 y or z sweep, 2 = the FP32 y or
 * z sweep, 3 = the FP32 x sweep; tmem_level as
 * bfvm_set_sweep_tmem.  Sets the shared-memory rings, TMEM rings and input
 * slots per TMEM ring of one CTA per SM, or all three to 0 where that sweep
 * does not apply (the shared-memory schedules run instead; a launch also
 * falls back when the grid gives fewer than two tiles per ring). */
int bfvm_tmem_sweep_plan(int axis, int n_line, int tmem_level, int* smem_rings, int* tmem_rings, int* input_slots);

/* Number of this library's kernels launched by the calls so far (counted on
 * the host at each launch). */
long long bfvm_kernel_launches(void);

/* Per-kernel timing, the device counterpart of the reference's per-step
 * timers (tests/mpi/diffusion/main.cpp:197-214): while enabled, every step
 * records CUDA events on the solve's stream around the source kernel and the
 * x, y and z sweep kernels.  bfvm_timing_read waits for the stream and
 * returns the summed durations [3] (ms: sources with x, y, z) and the number
 * of steps recorded, then clears them.  At most 4096 steps are recorded
 * between reads. */
int bfvm_timing_enable(bfvm_ctx* ctx, int on);
int bfvm_timing_read(bfvm_ctx* ctx, double* ms_xyz, int* steps);
/* The same records split by kernel: ms_sxyz [4] = the standalone source
 * kernel (0 without one), the x, y and z sweeps.  Reads and clears the
 * records as bfvm_timing_read does. */
int bfvm_timing_read_kernels(bfvm_ctx* ctx, double* ms_sxyz, int* steps);

const char* bfvm_status_string(int status);

/* ---- batched engine --------------------------------------------------------
 * Many resident solves of different grids and substrate counts advanced
 * together: each LOD step is one fused launch holding the x, y and z sweeps
 * of every member (per-member dependency counters order them) or, by
 * schedule, one launch per sweep over every member; runs of steps replay a
 * captured CUDA graph.  Members keep their own state and API
 * (upload, agents, download); each gives the same result, bit for bit, as
 * when stepped alone.  No reference counterpart: PhysiCell parameter sweeps
 * run one process per parameter set (beta/params_run.py). */
typedef struct bfvm_batch bfvm_batch;

int bfvm_batch_create(int precision, int device, bfvm_batch** out);
int bfvm_batch_destroy(bfvm_batch* batch);
/* Add / remove a member (same precision and device as the batch).  A solve
 * may belong to one batch; removal orders its later work after the batch's. */
int bfvm_batch_add(bfvm_batch* batch, bfvm_ctx* ctx);
int bfvm_batch_remove(bfvm_batch* batch, bfvm_ctx* ctx);
/* Members of the batch (0 for a NULL batch). */
int bfvm_batch_size(bfvm_batch* batch);
/* nsteps LOD steps of every member (flags as for bfvm_step). */
int bfvm_batch_step(bfvm_batch* batch, int nsteps, int flags);
int bfvm_batch_synchronize(bfvm_batch* batch);
/* The batch's stream (as void*); NULL for a NULL batch. */
void* bfvm_batch_stream(bfvm_batch* batch);
/* Schedule of a step.  mode 0: one fused persistent launch per step (tiles
 * of every member and sweep from one ordered work list, per-member
 * dependency counters); mode 1: three launches per step (x, y, z), each over
 * the tiles of every member; mode 2: mode 1 for the members under the direct
 * threshold, the others stepped one after another with their own kernels
 * (the tensor-memory sweeps of bfvm_step), all on the batch stream and in
 * its graph.  yz_chunk: rows per TMA box in the y/z sweeps; order (mode 0):
 * 0 members as added, 1 largest first; ctas_per_sm (mode 0): 0 = as many as
 * fit; graph_steps: steps per captured CUDA graph.  Every mode gives each
 * member the bits of bfvm_step. */
int bfvm_batch_set_schedule(bfvm_batch* batch, int mode, int yz_chunk, int order, int ctas_per_sm, int graph_steps);
int bfvm_batch_get_schedule(bfvm_batch* batch, int* mode, int* yz_chunk, int* order, int* ctas_per_sm,
                            int* graph_steps);
/* Mode 2: members of at least `values` voxel-substrate values (nx*ny*nz*S,
 * default 2097152 = 128^3 x 1) are stepped with their own kernels.
 * Measured on B200: a mix of 256^3 and 200^3 solves (4 substrates) with 40
 * small ones steps in 1.23 ms under mode 2 against 2.05 ms under mode 1
 * (FP64); the serving workload's FP32 server runs at 7.6e10 against 6.8e10
 * updates/s; 256 uneven solves of edges 24-128 stay faster under mode 1,
 * where the batched sweeps keep the GPU full across members. */
int bfvm_batch_set_direct_threshold(bfvm_batch* batch, long long values);
int bfvm_batch_get_direct_threshold(bfvm_batch* batch, long long* values);
/* Time trial_steps fused steps under each candidate schedule, keep the
 * fastest, and report its ms per step.  Member fields are restored after
 * the trials. */
int bfvm_batch_autotune(bfvm_batch* batch, int flags, int trial_steps, double* best_ms_per_step);

/* Fault injection, for tests of the timeout path (fused schedule, mode 0,
 * only: BFVM_ERR_STATE otherwise).  The first step of the next
 * bfvm_batch_step call runs with this member's count of finished x tiles
 * started far below zero, so the member's y tiles wait for x tiles that
 * never count up: their bounded waits run out, bfvm_batch_synchronize
 * returns BFVM_ERR_TIMEOUT (and clears the status), the member's field is
 * left undefined and the other members' results are unaffected.  The fault
 * is made on the host side of the dependency; nothing faults the GPU. */
int bfvm_batch_inject_stall(bfvm_batch* batch, bfvm_ctx* member);

#ifdef __cplusplus
}
#endif

#endif /* BIOFVM_B200_H */
