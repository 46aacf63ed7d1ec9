// bfvm_internal.h -- device-side data of one microenvironment solve and the
// kernel launchers shared by the C-ABI translation units.
//
// Device layout (chosen for the sweeps, not inherited from the reference):
//   field   T f[S][nz][ny][nxp]   x fastest, rows padded to nxp elements
//                                 (128-byte rows), one plane per substrate.
// The reference layout is [x][y][z][S] with z fastest
// (BioFVM/BioFVM_mesh.cpp:1149-1158); pack/unpack kernels convert at the
// host boundary.  With x fastest, the y and z sweeps read whole 128-byte row
// segments across consecutive x, and the x sweep is the one that stages its
// lines through shared memory (swizzled TMA tiles).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace bfvm {

constexpr int kMaxSubstrates = 64;

// Coefficient element types per precision.  Both forms run the recurrence
// in FP64; the FP32 form stores the densities in FP32 (rounding once per
// stored value) -- its recurrence in FP32 arithmetic drifted by a systematic
// 2.4e-5 (relative) over 500 steps, because smooth lines round the same way
// at every element.
//   FP64: DR = {denom_i, RN(1/denom_i)} (one 16-byte load per element, for
//         the exact Markstein quotient), CU = modified upper diagonal c_i,
//         C1 = dt*D/dx^2.
//   FP32: DR = RN(1/denom_i) (the quotient is t * DR, rounded to FP32 when
//         stored), CU = c_i, C1 = c1, all FP64.
template <typename T>
struct Coef;
template <>
struct Coef<double> {
  using DR = double2;
  using CU = double;
  using C1 = double;
};
template <>
struct Coef<float> {
  using DR = double;
  using CU = double;
  using C1 = double;
};

// Thomas coefficients of one axis for all substrates: rows [S][npad], padded
// with neutral entries so the sweeps may read (and prefetch one batch ahead)
// past the end of a line without bounds checks.
template <typename T>
struct AxisCoefs {
  const typename Coef<T>::DR* dr;
  const typename Coef<T>::CU* cu;
  int npad;
  // [S] or null: the first index from which a substrate's DR and CU entries
  // equal those of entry n - 2 (the factorization's fixed point), so that
  // the tensor-memory sweeps keep them in registers past it
  const int* conv;
};

// Rows of coefficient storage per line of n voxels: a y/z tile holds fewer
// than n + 80 rows (at most 64 chunks, rounded up to 16-row batches) and the
// sweeps prefetch the coefficients of the next 16-row batch, so every read
// stays below n + 96.
inline int coef_pad(int n) { return (n + 96 + 31) / 32 * 32; }

// Tracking of the substrates each agent internalizes
// (Microenvironment_Options::track_internalized_substrates_in_each_agent;
// BioFVM/BioFVM_basic_agent.cpp:520-532, 553-556).  internal == nullptr
// turns it off.
struct AgentTrack {
  double* internal;      // [n][S] per agent in list order: accumulated change
  const int* order;      // [n] agent index at each sorted position
  const double* ae1;     // [S][n] export per step (net export rate * dt), sorted
  double vvox;           // voxel volume
  int S, n;
};

// One agent's update of one density value r (FP64), agent at sorted position
// q, substrate s: the reference's rho += c1; rho /= c2; rho += e2, with the
// internalized-substrate bookkeeping around it when tracking is on.  The
// build's -fmad=false keeps every operation separately rounded, as the
// reference's separate loops and vector operators are.
__device__ __forceinline__ double agent_update(double r, double c1, double c2, double e2, int q, int s,
                                               const AgentTrack& tr) {
  double* in = nullptr;
  if (tr.internal) {
    double tec = 1.0;
    tec -= c2;
    tec *= r;
    tec += c1;
    tec /= c2;
    tec *= tr.vvox;
    in = tr.internal + static_cast<size_t>(tr.order[q]) * tr.S + s;
    *in -= tec;
  }
  r += c1;
  r /= c2;
  r += e2;
  if (in) *in -= tr.ae1[static_cast<size_t>(s) * tr.n + q];
  return r;
}

template <typename T>
struct SweepParams {
  T* f;                  // field base
  int nx, ny, nz, S, nxp;
  const typename Coef<T>::C1* c1;  // [S] dt*D/dx^2
  // FP32 only: the field holds rho - off[s]; each sweep's right-hand side is
  // shifted by shift[s] = (dt*decay/3) * off[s] to match (the constant off[s]
  // solves the zero-flux system with factor 1 + dt*decay/3).
  const double* off;     // [S] or null (FP64)
  const double* shift;   // [S] or null (FP64)
  const int* active;     // [S] Dirichlet activation
  // Face planes (resolved Dirichlet value of each face voxel), FP64:
  //   xface[side][s][k][j], yface[side][s][k][i], zface[side][s][j][i]
  const double* xface;
  const double* yface;
  const double* zface;
  AxisCoefs<T> ax, ay, az;
  // Agents (optional): sorted by device voxel id, CSR over x-lines
  // (line = k*ny + j).  a_key: sorted device voxel ids ((k*ny + j)*nx + i);
  // ac1/ac2/ae2: [S][n_sorted] FP64 in sorted order.
  const int* line_off;   // [ny*nz + 1] or nullptr when no sources this step
  const unsigned* a_key;
  const double* ac1;
  const double* ac2;
  const double* ae2;
  int n_sorted;
  AgentTrack track;      // internalized-substrate tracking (track.internal null: off)
  // 1 when no substrate has a negative diffusion coefficient or decay rate
  // (c1 >= 0, every denominator >= 1): enables the FP64 input screen of the
  // reference-exact chain; 0 checks every numerator; 2 (kScreenFast) runs
  // the short chain (bfvm_set_fp64_chain), which needs no screen.
  int screen;
  int* status;           // device status word
  // [2] tiles handed out, CTAs finished: the persistent TMEM y/z sweep's
  // work counter, zero between launches (its last CTA zeroes it)
  unsigned long long* tile_counter;
  // The substrates a launch sweeps: [s_lo, s_hi) (make_params: all of them).
  // Substrates are independent through the whole step, so the step may run
  // as two substrate groups on two streams (bfvm_set_substrate_streams).
  int s_lo, s_hi;
};

// Launch configuration of the sweeps (chosen by the host, tunable).  A tile
// of lines is staged whole in one CTA's shared memory.  Two schedules:
//   persistent  a compute warp and a copy warp per CTA, as many CTAs as
//               fit, each walking a sequence of 32-line tiles through a ring
//               of chunk slots (the next tile loads while this one finishes);
//   per-tile    one CTA per tile of x_lines / yz_tile lines.
// persistent = 1 (default) runs the y and z sweeps persistent when every
// resident CTA gets at least 8 tiles (fewer measured slower) and the x sweep
// per tile (the per-lane agent walk of the persistent x sweep measured slower
// than the per-tile sweep's lane-per-run agents); 2 runs all three
// persistent whatever the tile count; 0 all per tile.  Persistent needs x_lines == yz_tile == 32 and
// lines of at most 64 chunks; other shapes run per tile.
struct SweepConfig {
  int x_lines = 32;   // lines per CTA in the x sweep (multiple of 8, <= 256)
  int yz_tile = 32;   // consecutive x per CTA in the y/z sweeps (whole 128-byte rows)
  int yz_chunk = 32;  // target rows per TMA box along the line in the y/z sweeps (<= 256; per-tile only)
  int persistent = 1; // 0 per tile, 1 persistent y/z, 2 persistent x/y/z
  // Sources in a step: 0 (default) the standalone source kernel before the
  // sweeps, 1 fused into the x sweep.  Same bits either way; the standalone
  // kernel measured faster (cube200 FP64, 100k agents: 0.451 against 0.465
  // ms per step), as it touches only the agents' voxels while the fused
  // path holds every x tile until all of its chunks have landed.
  int fuse_sources = 0;
  // Tensor-memory rings in the FP64 persistent sweeps: 1 (default) in the
  // y/z sweeps on lines of 33 to 736 (up to four rings keep the forward
  // results of a line's first 256 values in TMEM next to the shared-memory
  // rings: 224 lines in flight per SM instead of 128 at lines of 200, 64
  // instead of 32 at 640), and in the x sweep on lines of 33 to 736 (agents
  // not fused); 2 also in the x sweep on lines of 17 to 32; 0 shared memory
  // alone.  Same bits at every level.
  int tmem = 1;
};

// Rows per y/z chunk of the persistent schedule (one register batch).
constexpr int kRingRows = 16;

// The three tensor maps the sweeps use, built once per context.
struct FieldMaps {
  CUtensorMap x;   // box {128 bytes of x, x_lines, 1, 1}, 128B swizzle
  CUtensorMap y;   // box {yz_tile, chunk rows, 1, 1}
  CUtensorMap z;   // box {yz_tile, 1, chunk rows, 1}
  CUtensorMap ry;  // persistent schedule: box {32, kRingRows, 1, 1}
  CUtensorMap rz;  // persistent schedule: box {32, 1, kRingRows, 1}
  CUtensorMap g;   // gradients: box {32 + 4 (FP64) or 32 + 8 (FP32) x, 1, 10 z, min(S, 4) substrates}
  int g_ok;        // 1 when the gradient map could be encoded
  // tensor-memory x sweeps: 3-D {nx, ny * nz rows (row k * ny + j), S}, box
  // {128 bytes of x, 32 rows, 1}, 128B swizzle -- a tile is 32 consecutive
  // rows of one substrate, across y-row ends
  CUtensorMap xr;
  int xr_ok;
  // tensor-memory y/z sweeps, the partial x tiles of several planes packed
  // into one tile: py has the dimensions {nx, nz, ny, S} (x, plane k, row j,
  // substrate), pz {nx, ny, nz, S}; box {pyz_w, 32 / pyz_w, 16 rows, 1}.
  // pyz_w = 0 when nx % 32 leaves nothing to pack (or is above 16).
  CUtensorMap py, pz;
  int pyz_w;
};

// Host-side count of this library's kernel launches (bfvm_kernel_launches).
void note_launches(int n);
// While on, note_launches counts nothing (launches being captured into a
// graph are counted when the graph is replayed).
void set_launch_capture(bool on);

int encode_field_maps(FieldMaps* maps, void* f, int elem_bytes, int nx, int ny, int nz, int S, int nxp,
                      const SweepConfig& cfg);

template <typename T>
cudaError_t launch_sweep_x(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st);
// Partitioned sweeps (bfvm_part_sweeps.cu, bfvm_set_fp64_chain(ctx, 2)):
// kPartWarps warps per 32-line tile, warp w owning elements
// [w*mseg, (w+1)*mseg) of every line.  Per axis and substrate, rows of npad:
// ra = {RN(1/d_i), a_i = RN(c1 RN(1/d_i))} (a_0 = 0), pg = {P_i, g_i} with
// g_i = -c_i (g_{n-1} = 0) and P_i the product of a from the segment start
// to i, q = Q_i the product of g from i to the segment end; ag = {A_w, G_w}
// [S][kPartWarps], each segment's products (1 for an empty segment).
constexpr int kPartWarps = 8;
constexpr int kPartMaxChunks = 64;  // chunks per staged line (their barriers fill the first 512 bytes)
struct PartAxis {
  const double2* ra;
  const double2* pg;
  const double* q;
  const double2* ag;
  int mseg;
  int npad;
};
size_t part_smem_bytes(int elem_bytes, int n_line);
// By default, lines at least this long run the y and z sweeps partitioned
// under chain 2 (bfvm_set_partition_min_line overrides it); shorter lines,
// and the x sweep, run the short chain on the serial kernels.  Measured on
// B200, mean y/z sweep time on n^3 cubes, partitioned over serial short
// chain: FP64 1.00 at n = 384 and 448, 0.94 at 512, 0.64 at 640; FP32 (the
// serial sweeps with their tensor-memory rings) 1.21 at 288, 1.06 at 320,
// 1.07 at 384, 0.93 at 448, 0.80 at 512, 0.65 at 640.
constexpr int kPartMinLine64 = 512;
constexpr int kPartMinLine32 = 448;
template <typename T, int AXIS>
cudaError_t launch_part(const CUtensorMap& map, const SweepParams<T>& p, const PartAxis& pa, cudaStream_t st);

// The bounded-wait limit (ns) of the kernels in bfvm_sweeps.cu (sweeps and
// the batched engine) and in bfvm_tmem_sweeps.cu, on the current device.
cudaError_t sweeps_set_wait_limit(unsigned long long ns);
cudaError_t tmem_sweeps_set_wait_limit(unsigned long long ns);
template <typename T>
cudaError_t launch_sweep_y(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st);
template <typename T>
cudaError_t launch_sweep_z(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st);

// Shared-memory bytes one CTA of each sweep needs (per-tile schedule), and
// of the persistent schedule (0 where it does not apply).
size_t sweep_x_smem(int elem_bytes, int nx, const SweepConfig& cfg);
size_t sweep_yz_smem(int elem_bytes, int n_line, const SweepConfig& cfg);
size_t ring_x_smem(int elem_bytes, int nx);
size_t ring_yz_smem(int elem_bytes, int n_line);
// Bytes of one shared-memory ring of the persistent y/z sweeps.
size_t ring_yz_bytes(int elem_bytes, int n_line);

// The FP64 persistent sweeps with tensor-memory rings (bfvm_tmem_sweeps.cu):
// each launches when it applies to the solve's shape and configuration and
// sets *launched; otherwise it returns cudaSuccess with *launched false and
// the caller runs another schedule.
// The y/z sweeps take the packed map of their axis and its group width pw
// (FieldMaps::py / pz, pyz_w; 0 when no partial x tiles are packed).
template <int AXIS>
cudaError_t launch_tmem_yz(const CUtensorMap& ring_map, const CUtensorMap& pmap, int pw,
                           const SweepParams<double>& p, const SweepConfig& cfg, cudaStream_t st, bool* launched);
cudaError_t launch_tmem_x(const CUtensorMap& map, const SweepParams<double>& p, const SweepConfig& cfg,
                          cudaStream_t st, bool* launched);
// The FP32 sweeps with tensor-memory rings (bfvm_tmem_sweeps.cu), same
// contract.
template <int AXIS>
cudaError_t launch_tmem_yz_f32(const CUtensorMap& ring_map, const CUtensorMap& pmap, int pw,
                               const SweepParams<float>& p, const SweepConfig& cfg, cudaStream_t st, bool* launched);
cudaError_t launch_tmem_x_f32(const CUtensorMap& map, const SweepParams<float>& p, const SweepConfig& cfg,
                              cudaStream_t st, bool* launched);

// ---- batched engine: one fused launch per LOD step over many solves ------
// Tiles are 32 lines (one warp) in every sweep of a batch.
constexpr int kBatchTile = 32;

template <typename T>
struct alignas(64) BatchEnv {
  CUtensorMap mx, my, mz;  // tensor maps of this solve's field (boxes as FieldMaps, 32-line tiles)
  SweepParams<T> p;
  int chy, chz;            // rows per TMA box of the y and z maps
  int nty, ntx;            // tiles along y (x sweep) and along x (y and z sweeps)
};

// Device-resident description of the current membership; rewritten between
// steps, so a captured step stays valid while the membership changes.
struct BatchHeader {
  int n_env;
  int n_items[3];  // tiles of all members per sweep (x, y, z)
};

// pre[a*(cap+1) + e]: index of member e's first tile among the tiles of sweep a.
// counters: [0] work dispenser, [1 + a*cap + e] tiles of sweep a of member e done.
template <typename T>
cudaError_t launch_batch_step(const BatchHeader* hdr, const BatchEnv<T>* envs, const int* pre, int cap, int* counters,
                              int* status, int grid, size_t smem, cudaStream_t st);

// Split schedule: three launches per step (x, y, z), each over the tiles of
// every member; items[a] tiles and smem[a] bytes per CTA for sweep a.
template <typename T>
cudaError_t launch_batch_sweeps(const BatchHeader* hdr, const BatchEnv<T>* envs, const int* pre, int cap,
                                const int items[3], const size_t smem[3], cudaStream_t st);

// Shared memory one CTA of the fused step needs to hold any tile of a member.
size_t batch_member_smem(int elem_bytes, int nx, int ny, int nz, int yz_chunk);
// The same for one sweep (axis 0, 1, 2) of the split schedule.
size_t batch_axis_smem(int elem_bytes, int axis, int n_line, int yz_chunk);

// Resident CTAs per SM of the fused step at the given shared memory.
template <typename T>
cudaError_t batch_occupancy(size_t smem, int* ctas_per_sm);

// Bulk sources and sinks (bfvm_bulk.cu): rates = [supply | target | uptake],
// each S*nz*ny*nxp doubles in the field's device layout.
template <typename T>
cudaError_t launch_bulk(T* f, const double* rates, int nx, int ny, int nz, int S, int nxp, double dt,
                        const double* off, int sm_count, cudaStream_t st);

// Layout conversion between the reference AoS [x][y][z][S] (double) and the
// device SoA [S][z][y][nxp] (T).
// off: [S] offsets subtracted on pack / added on unpack (FP32), or null.
template <typename T>
cudaError_t launch_pack(const double* aos, T* f, int nx, int ny, int nz, int S, int nxp, const double* off,
                        cudaStream_t st);
template <typename T>
cudaError_t launch_unpack(const T* f, double* aos, int nx, int ny, int nz, int S, int nxp, const double* off,
                          cudaStream_t st);

}  // namespace bfvm
