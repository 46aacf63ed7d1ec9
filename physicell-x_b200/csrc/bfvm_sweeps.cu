// bfvm_sweeps.cu -- the three Thomas sweeps of one BioFVM LOD step on sm_100a.
//
// Reference: diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING,
// BioFVM/BioFVM_solvers.cpp:102-780 (one rank), with the Dirichlet pin
// Microenvironment::apply_dirichlet_boundaries_conditions
// (BioFVM/BioFVM_microenvironment.cpp:348-446) applied before the x sweep and
// after each sweep (BioFVM_solvers.cpp:345, 682, 731, 778), and the cell
// source/sink update Basic_Agent::simulate_secretion_and_uptake
// (BioFVM/BioFVM_basic_agent.cpp:509-559) ahead of the step.
//
// One thread owns one (line, substrate) Thomas system.  Each CTA stages its
// lines in shared memory with plain (non-multicast) TMA tensor copies, so the
// forward elimination and back substitution read HBM once and write it once:
// six field passes per LOD step in total.
//
//   x sweep  lines run along the contiguous axis.  The CTA loads TL lines as
//            128-byte-wide boxes with the 128B swizzle, so thread t reading
//            16-byte units of its own row (a transpose in shared memory) hits
//            eight distinct bank groups per quarter-warp.  Agent sources and
//            the first Dirichlet pin are applied to the staged row before the
//            recurrence reads it.
//   y, z     consecutive threads own consecutive x; the tile is [line][x], so
//            each step of the recurrence reads one contiguous shared-memory row.
//
// The recurrence is serial per line, so its speed is the latency of the
// dependent chain: per element four FP64 operations forward (fma; Markstein
// quotient) and one backward.  Every load a batch of elements needs is issued
// before the chain over that batch starts, coefficient rows are padded so no
// load needs a bounds check, and the chains start from -0.0, which makes the
// first element need no special case (fma(c1, -0, v) == v and
// fma(-c, -0, y) == y exactly, as c1 >= 0 and the modified upper diagonal
// c <= 0).
//
// Dirichlet pins are fused: a line lying in an activated face is written with
// its face values; other lines get their two end voxels pinned after the
// sweep.  The field in HBM is therefore always in the "pinned" state between
// kernels, which makes the reference's pins after the x and y sweeps implicit
// in the next kernel's input.
//
// Arithmetic (FP64 form) follows the reference operation by operation:
//   forward  y_0 = p_0 / d_0;  y_i = fma(c1, y_{i-1}, p_i) / d_i
//   backward x_i = fma(-c_i, x_{i+1}, y_i)
//   agent    rho = ((rho + c1_a) / c2_a) + e2_a
// The quotient uses Markstein's correction from a precomputed RN(1/d_i)
// (div_fast), which is the correctly rounded quotient except for a numerator
// of -0 or a nonzero numerator below 2^-960; a batch that meets either is
// redone with IEEE division, so results equal the reference's bit for bit.
// The FP32 form stores rho - off[s] in FP32 and applies the matching
// right-hand-side shift; its recurrence, coefficients and agent updates are
// FP64, so each value is rounded to FP32 once per sweep, when it is stored.
//
// The FP64 persistent sweeps with tensor-memory rings are in
// bfvm_tmem_sweeps.cu; the launchers here hand a sweep to them first where
// they apply.  Helpers shared by both files: bfvm_sweep_common.cuh.
#include <climits>
#include <type_traits>

#include "bfvm_internal.h"
#include "bfvm_ptx.cuh"
#include "bfvm_sweep_common.cuh"

namespace bfvm {


// ---------------------------------------------------------------------------
// x sweep
// ---------------------------------------------------------------------------
// One x-sweep tile: the lines (j0 .. j0+TL-1, k, s), TL = blockDim.x.  `base`
// is 1024-byte-aligned shared memory holding kMaxChunks mbarriers (already
// initialized) followed by the staged tile; `phase` holds the parity each
// barrier completes next and is advanced here.  The chunks are stored back
// with bulk stores that the caller must let finish reading shared memory
// (tma_store_wait_read) before reusing it.  Returns false if a wait gave up.
template <typename T>
__device__ bool x_tile(const CUtensorMap* map, const SweepParams<T>& p, int j0, int k, int s, unsigned char* base,
                       uint64_t& phase) {
  using DR = typename Coef<T>::DR;
  using CU = typename Coef<T>::CU;
  constexpr int W = 128 / sizeof(T);  // elements per 128-byte row (one TMA box width)
  constexpr int kAgentRounds = 4;     // agent rounds whose data is loaded ahead

  const int TL = blockDim.x;
  const int nx = p.nx, ny = p.ny, nz = p.nz, S = p.S;
  const int C = (nx + W - 1) / W;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  unsigned char* tile = base + kBarrierBytes;
  const uint32_t chunk_bytes = static_cast<uint32_t>(TL) * 128u;

  const int t = threadIdx.x;
  if (t == 0) {
    for (int c = 0; c < C; ++c) {
      const uint32_t bar = smem_u32(&bars[c]);
      mbar_expect_tx(bar, chunk_bytes);
      tma_load_4d(smem_u32(tile + c * chunk_bytes), map, bar, c * W, j0, k, s);
    }
  }
  __syncthreads();  // reconverge before any lane blocks on a barrier

  const int j = j0 + t;
  const bool valid = j < ny;
  const bool act = p.active[s] != 0;
  const bool face = act && (j == 0 || j == ny - 1 || k == 0 || k == nz - 1);
  // Face-line values: the z-face plane when k is on a z face, else the y-face plane.
  const double* fv = nullptr;
  if (face && valid) {
    if (k == 0 || k == nz - 1)
      fv = p.zface + ((static_cast<size_t>(k == 0 ? 0 : 1) * S + s) * ny + j) * nx;
    else
      fv = p.yface + ((static_cast<size_t>(j == 0 ? 0 : 1) * S + s) * nz + k) * nx;
  }
  const double off = kF32<T> ? p.off[s] : 0.0;
  T x0v = T(0), x1v = T(0);
  if (act && valid) {
    x0v = static_cast<T>(p.xface[(static_cast<size_t>(0 * S + s) * nz + k) * ny + j] - off);
    x1v = static_cast<T>(p.xface[(static_cast<size_t>(1 * S + s) * nz + k) * ny + j] - off);
  }
  const DR* __restrict__ drp = p.ax.dr + static_cast<size_t>(s) * p.ax.npad;
  const CU* __restrict__ cup = p.ax.cu + static_cast<size_t>(s) * p.ax.npad;
  const typename Coef<T>::C1 c1 = p.c1[s];
  const double shift = kF32<T> ? p.shift[s] : 0.0;
  // Coefficients of the forward pass: two register buffers used in turn, the
  // idle one loaded with the chunk after next (rows are padded past C * W).
  DR cfa[W], cfb[W];
#pragma unroll
  for (int q = 0; q < W; ++q) {
    cfa[q] = __ldg(drp + q);
    cfb[q] = __ldg(drp + W + q);
  }
  // The upper-diagonal row for the back substitution, staged after the tile
  // (read back after the barrier that ends the forward pass).
  CU* cus = reinterpret_cast<CU*>(tile + C * chunk_bytes);
  stage_row_cta(cus, cup, C * W);

  unsigned char* row = tile + t * 128;
  const int sw = t & 7;
  bool ok = true;
  bool all_landed = false;

  // Agent sources.  The agents of this tile's lines are one contiguous range
  // of the sorted list; lanes take them in rounds of TL, each lane applying
  // the run of agents that starts at its position to the staged voxel.  Runs
  // never share a voxel, so the lanes are independent; faces are pinned over
  // the result afterwards, as the reference pins after its source step.
  if (p.line_off != nullptr) {
    const int line0 = k * ny + j0;
    const int A0 = __ldg(p.line_off + line0);
    const int A1 = __ldg(p.line_off + line0 + min(TL, ny - j0));
    if (A1 > A0) {  // uniform across the CTA
      const double* ac1 = p.ac1 + static_cast<size_t>(s) * p.n_sorted;
      const double* ac2 = p.ac2 + static_cast<size_t>(s) * p.n_sorted;
      const double* ae2 = p.ae2 + static_cast<size_t>(s) * p.n_sorted;
      unsigned akey[kAgentRounds], aprev[kAgentRounds];
      double a1[kAgentRounds], a2[kAgentRounds], a3[kAgentRounds];
#pragma unroll
      for (int r = 0; r < kAgentRounds; ++r) {
        const int q = A0 + t + r * TL;
        const bool in = q < A1;
        akey[r] = in ? __ldg(p.a_key + q) : 0u;
        aprev[r] = (in && q > A0) ? __ldg(p.a_key + q - 1) : ~0u;
        a1[r] = in ? __ldg(ac1 + q) : 0.0;
        a2[r] = in ? __ldg(ac2 + q) : 1.0;
        a3[r] = in ? __ldg(ae2 + q) : 0.0;
      }
      for (int c = 0; c < C; ++c)
        if (ok) ok = mbar_wait(smem_u32(&bars[c]), static_cast<uint32_t>(phase >> c) & 1u);
      all_landed = true;
      auto elem = [&](unsigned key) {
        const int line = static_cast<int>(key / static_cast<unsigned>(nx));
        const int i = static_cast<int>(key - static_cast<unsigned>(line) * nx);
        const int rl = line - line0;
        return swz_elem<T>(tile + (i / W) * chunk_bytes + rl * 128, i % W, rl & 7);
      };
      if (ok) {
#pragma unroll
        for (int r = 0; r < kAgentRounds; ++r) {
          const int q = A0 + t + r * TL;
          if (q < A1 && akey[r] != aprev[r])
            apply_run<T>(elem(akey[r]), q, akey[r], a1[r], a2[r], a3[r], A1, p.a_key, ac1, ac2, ae2, off, s,
                         p.track);
        }
        for (int r = kAgentRounds; A0 + r * TL < A1; ++r) {
          const int q = A0 + t + r * TL;
          if (q < A1) {
            const unsigned key = __ldg(p.a_key + q);
            if (q == A0 || __ldg(p.a_key + q - 1) != key)
              apply_run<T>(elem(key), q, key, __ldg(ac1 + q), __ldg(ac2 + q), __ldg(ae2 + q), A1, p.a_key, ac1, ac2,
                           ae2, off, s, p.track);
          }
        }
      }
      __syncthreads();  // agents wrote rows of other lanes
    }
  }

  // Forward elimination, one chunk at a time as the TMA boxes land.  Values
  // past nx in the last chunk are TMA fill; the chain may run over them
  // harmlessly (those results are never stored to the field).
  double y = -0.0;  // running value of the forward recurrence (FP64 in both forms)
  const int screen = p.screen;
  // FP64 without fused agents: the input screen is one vote per tile (the
  // staged inputs are then the field's, which a failing tile re-reads); with
  // fused agents each batch is screened and redone from its registers.
  const bool tile_screen = !kF32<T> && p.line_off == nullptr;
  int hwmin = INT_MAX;  // minimum input high word of this lane's line
  // Every batch keeps its per-lane face and range checks: a per-tile vote
  // choosing a version without them measured slower here (x sweep, cube200:
  // FP64 0.166 against 0.163 ms, FP32 0.114 against 0.105).
  const bool edge_tile = true;
  auto fwd = [&](bool edge, int c, DR (&cf)[W]) {
    if (!all_landed && ok) ok = mbar_wait(smem_u32(&bars[c]), static_cast<uint32_t>(phase >> c) & 1u);
    if (edge && (face || !valid)) return;  // lines past ny hold TMA fill, never stored
    unsigned char* crow = row + c * chunk_bytes;
    const int i0 = c * W;
    // The pin before the sweep, on the staged row (after the sources).
    if (act) {
      if (i0 == 0) *swz_elem<T>(crow, 0, sw) = x0v;
      if (nx - 1 < i0 + W) *swz_elem<T>(crow, nx - 1 - i0, sw) = x1v;
    }
    T v[W];
    load_row<T, W>(crow, sw, v);
    if (!kF32<T> && i0 + W > nx) {  // FP64: TMA fill past the line's end passes the screen (never stored)
#pragma unroll
      for (int q = 0; q < W; ++q)
        if (i0 + q >= nx) v[q] = T(1);
    }
    RowPut<T> put{crow, sw};
    if constexpr (!kF32<T>) {
      if (tile_screen) {
        y = forward_any<W>(screen, v, cf, c1, y, put);
        if (screen != kScreenFast) hwmin = min(hwmin, batch_min_hi<W>(v));
        return;
      }
    }
    y = forward_store<W>(v, cf, c1, shift, screen, y, put);
  };
  auto forward_pass = [&](bool edge) {
    for (int c = 0; c < C; c += 2) {
      fwd(edge, c, cfa);
#pragma unroll
      for (int q = 0; q < W; ++q) cfa[q] = __ldg(drp + (c + 2) * W + q);
      if (c + 1 >= C) break;
      fwd(edge, c + 1, cfb);
#pragma unroll
      for (int q = 0; q < W; ++q) cfb[q] = __ldg(drp + (c + 3) * W + q);
    }
  };
  if (edge_tile)
    forward_pass(true);
  else
    forward_pass(false);
  phase ^= chunk_mask(C);
  if (__syncthreads_or(!ok)) {
    if (t == 0) atomicExch(p.status, kDevTimeout);
    return false;
  }
  if constexpr (!kF32<T>) {
    // The tile's screen: a line with an input below 2^-960 (or negative)
    // anywhere is redone from its inputs -- the field still holds them (this
    // tile's results are stored only by the back substitution) -- pinned as
    // the staged row was, with every numerator checked.
    if (tile_screen && __syncthreads_or(!screen_clean(screen, hwmin))) {
      if (!face && valid) {
        const T* src = p.f + ((static_cast<size_t>(s) * nz + k) * ny + j) * p.nxp;
        y = -0.0;
        for (int c = 0; c < C; ++c) {
          const int i0 = c * W;
          T v[W];
          DR cf[W];
#pragma unroll
          for (int q = 0; q < W; ++q) {
            v[q] = i0 + q < nx ? src[i0 + q] : T(1);
            cf[q] = __ldg(drp + i0 + q);
          }
          if (act) {
#pragma unroll
            for (int q = 0; q < W; ++q) {
              if (i0 + q == 0) v[q] = x0v;
              if (i0 + q == nx - 1) v[q] = x1v;
            }
          }
          RowPut<T> put{row + c * chunk_bytes, sw};
          y = forward_checked<W>(v, cf, c1, y, put);
        }
      }
      __syncthreads();
    }
  }

  // Back substitution, last chunk first; each finished chunk is stored at once.
  double xn = -0.0;  // running value of the back substitution
  auto back_chunk = [&](bool edge, int c) {
    const bool E = edge;
    unsigned char* crow = row + c * chunk_bytes;
    const int i0 = c * W;
    CU cw[W];
    const double2* cwp = reinterpret_cast<const double2*>(cus + i0);  // 16-byte pairs
#pragma unroll
    for (int q = 0; q < W / 2; ++q) {
      const double2 pr = cwp[q];
      cw[2 * q] = pr.x;
      cw[2 * q + 1] = pr.y;
    }
    if (E && face) {
      T fw[W];
#pragma unroll
      for (int q = 0; q < W; ++q) fw[q] = (fv != nullptr && i0 + q < nx) ? static_cast<T>(fv[i0 + q] - off) : T(0);
#pragma unroll
      for (int q = 0; q < W; ++q)
        if (i0 + q < nx) *swz_elem<T>(crow, q, sw) = fw[q];
    } else if (!E || valid) {
      T v[W];
      load_row<T, W>(crow, sw, v);
      if (i0 + W > nx) {
        // the line ends inside this chunk: skip the fill past nx
#pragma unroll
        for (int q = W - 1; q >= 0; --q) {
          if (i0 + q < nx) {
            xn = back_elem(cw[q], xn, v[q]);
            v[q] = static_cast<T>(xn);
          }
        }
      } else {
#pragma unroll
        for (int q = W - 1; q >= 0; --q) {
          xn = back_elem(cw[q], xn, v[q]);
          v[q] = static_cast<T>(xn);
        }
      }
      store_row<T, W>(crow, sw, v);
      if (act) {
        if (i0 == 0) *swz_elem<T>(crow, 0, sw) = x0v;
        if (nx - 1 < i0 + W) *swz_elem<T>(crow, nx - 1 - i0, sw) = x1v;
      }
    }
  };
  for (int c = C - 1; c >= 0; --c) {
    if (edge_tile)
      back_chunk(true, c);
    else
      back_chunk(false, c);
    fence_async_smem();
    __syncthreads();
    if (t == 0) {
      tma_store_4d(map, smem_u32(tile + c * chunk_bytes), c * W, j0, k, s);
      tma_store_commit();
    }
  }
  return true;
}

template <typename T>
__global__ void __launch_bounds__(256) sweep_x_kernel(const __grid_constant__ CUtensorMap map, const SweepParams<T> p) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  const int C = (p.nx + kChunkX<T> - 1) / kChunkX<T>;
  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(reinterpret_cast<uint64_t*>(base) + c), 1);
    fence_barrier_init();
  }
  __syncthreads();
  uint64_t phase = 0;
  x_tile<T>(&map, p, blockIdx.x * blockDim.x, blockIdx.y, p.s_lo + blockIdx.z, base, phase);
  if (threadIdx.x == 0) tma_store_wait_read();
}

// ---------------------------------------------------------------------------
// y and z sweeps
// ---------------------------------------------------------------------------

// One y- or z-sweep tile: the lines (i0 .. i0+TI-1, m, s), TI = blockDim.x,
// m = k for the y sweep and j for the z sweep, staged in TMA boxes of CH rows.
// Shared-memory layout and contract as for x_tile (base 128-byte aligned).
template <typename T, int AXIS, int TI>
__device__ bool yz_tile(const CUtensorMap* map, const SweepParams<T>& p, int i0, int m, int s, int CH,
                        unsigned char* base, uint64_t& phase) {
  using DR = typename Coef<T>::DR;
  using CU = typename Coef<T>::CU;
  constexpr int R = kRowBatch;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int n = (AXIS == 1) ? ny : nz;
  const bool act = p.active[s] != 0;
  // A tile whose lines all lie in an activated face is already final: its
  // input holds the face values (every face voxel is pinned by the sweep
  // before) and the pin after this sweep writes the same values again.
  if (act && (m == 0 || m == ((AXIS == 1) ? nz : ny) - 1)) return true;

  const int C = (n + CH - 1) / CH;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  T* tile = reinterpret_cast<T*>(base + kBarrierBytes);
  const uint32_t chunk_bytes = static_cast<uint32_t>(CH) * TI * sizeof(T);

  const int t = threadIdx.x;
  if (t == 0) {
    for (int c = 0; c < C; ++c) {
      const uint32_t bar = smem_u32(&bars[c]);
      mbar_expect_tx(bar, chunk_bytes);
      T* dst = tile + c * CH * TI;
      if (AXIS == 1)
        tma_load_4d(smem_u32(dst), map, bar, i0, c * CH, m, s);
      else
        tma_load_4d(smem_u32(dst), map, bar, i0, m, c * CH, s);
    }
  }
  __syncthreads();  // reconverge before any lane blocks on a barrier

  const int i = i0 + t;
  // Lines in an x face keep their (pinned) input, as above.
  const bool face = act && (i == 0 || i == nx - 1);
  const AxisCoefs<T>& ac = (AXIS == 1) ? p.ay : p.az;
  const DR* __restrict__ drp = ac.dr + static_cast<size_t>(s) * ac.npad;
  const CU* __restrict__ cup = ac.cu + static_cast<size_t>(s) * ac.npad;
  const typename Coef<T>::C1 c1 = p.c1[s];
  const double shift = kF32<T> ? p.shift[s] : 0.0;
  const int screen = p.screen;
  // Coefficients of the forward pass: two register buffers used in turn, the
  // idle one loaded with the batch after next.
  DR cfa[R], cfb[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    cfa[q] = __ldg(drp + q);
    cfb[q] = __ldg(drp + R + q);
  }
  // The upper-diagonal row for the back substitution, staged after the tile
  // (read back after the barrier that ends the forward pass).
  const int rows = (C * CH + R - 1) / R * R;
  CU* cus = reinterpret_cast<CU*>(tile + static_cast<size_t>(rows) * TI);
  stage_row_cta(cus, cup, rows);
  T* col = tile + t;
  bool ok = true;
  int waited = 0;     // chunks whose TMA load this thread has waited for
  int wait_row = 0;   // first row of chunk `waited`
  // The two end voxels of the line lie in the y (z) faces: the pin after the
  // sweep restores their input values.
  T e0v = T(0), e1v = T(0);
  double y = -0.0;  // running value of the forward recurrence (FP64 in both forms)
  int hwmin = INT_MAX;  // FP64: minimum input high word of this lane's line (the screen)

  // One forward batch of R rows from rb, after waiting for the chunks that
  // cover it.  The tile holds a whole number of batches, so the last batch
  // may read rows past n (TMA fill or unused rows): those results are never
  // stored to the field.
  // Every batch keeps its per-lane face and range checks: in this per-tile
  // kernel a per-tile vote choosing a version without them measured slower
  // (FP32 cube200 y/z 0.0949 against 0.0922 ms); the persistent kernel keeps
  // the vote, where it measured faster.
  const bool edge_tile = true;
  auto fwd = [&](bool edge, int rb, DR (&cf)[R]) {
    while (waited < C && wait_row < rb + R) {
      if (ok) ok = mbar_wait(smem_u32(&bars[waited]), static_cast<uint32_t>(phase >> waited) & 1u);
      ++waited;
      wait_row += CH;
    }
    if (edge && (face || i >= nx)) return;  // lines past nx hold TMA fill, never stored
    T v[R];
    T* cb = col + rb * TI;
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
    if (act) {
      if (rb == 0) e0v = v[0];
      if (rb + R > n - 1) {
#pragma unroll
        for (int q = 0; q < R; ++q)
          if (rb + q == n - 1) e1v = v[q];
      }
    }
    if (rb + R > n) {  // rows past the line's end (TMA fill or unused): any clean value, never stored
#pragma unroll
      for (int q = 0; q < R; ++q)
        if (rb + q >= n) v[q] = T(1);
    }
    auto put = [&](int q, auto val) { cb[q * TI] = static_cast<T>(val); };
    if constexpr (kF32<T>) {
      y = forward_store<R>(v, cf, c1, shift, screen, y, put);
    } else {
      y = forward_any<R>(screen, v, cf, c1, y, put);
      if (screen != kScreenFast) hwmin = min(hwmin, batch_min_hi<R>(v));
    }
  };
  auto forward_pass = [&](bool edge) {
    for (int rb = 0; rb < n; rb += 2 * R) {
      fwd(edge, rb, cfa);
#pragma unroll
      for (int q = 0; q < R; ++q) cfa[q] = __ldg(drp + rb + 2 * R + q);
      if (rb + R >= n) break;
      fwd(edge, rb + R, cfb);
#pragma unroll
      for (int q = 0; q < R; ++q) cfb[q] = __ldg(drp + rb + 3 * R + q);
    }
  };
  if (edge_tile)
    forward_pass(true);
  else
    forward_pass(false);
  while (waited < C) {
    if (ok) ok = mbar_wait(smem_u32(&bars[waited]), static_cast<uint32_t>(phase >> waited) & 1u);
    ++waited;
  }
  phase ^= chunk_mask(C);
  if (__syncthreads_or(!ok)) {
    if (t == 0) atomicExch(p.status, kDevTimeout);
    return false;
  }
  if constexpr (!kF32<T>) {
    // The screen, once per tile: a line with an input below 2^-960 (or
    // negative) anywhere is redone from its inputs, which are still in the
    // field (this tile's results are stored only by the back substitution).
    if (__syncthreads_or(!screen_clean(screen, hwmin))) {
      if (!face && i < nx) {
        const size_t row_stride = (AXIS == 1) ? static_cast<size_t>(p.nxp) : static_cast<size_t>(p.nxp) * p.ny;
        const T* src = (AXIS == 1) ? p.f + ((static_cast<size_t>(s) * p.nz + m) * p.ny) * p.nxp + i
                                   : p.f + (static_cast<size_t>(s) * p.nz * p.ny + m) * p.nxp + i;
        y = -0.0;
        for (int rb = 0; rb < n; rb += R) {
          T v[R];
          DR cf[R];
#pragma unroll
          for (int q = 0; q < R; ++q) {
            v[q] = rb + q < n ? src[(rb + q) * row_stride] : T(1);
            cf[q] = __ldg(drp + rb + q);
          }
          T* cb = col + rb * TI;
          y = forward_checked<R>(v, cf, c1, y, [&](int q, auto val) { cb[q * TI] = static_cast<T>(val); });
        }
      }
      __syncthreads();
    }
  }

  // Back substitution in batches of R rows from the end; chunk c is stored
  // once every row from its start on is final.
  double xn = -0.0;  // running value of the back substitution
  int next_store = C - 1;
  int store_row = next_store * CH;  // first row of chunk next_store
  const int last_b = ((n - 1) / R) * R;
  auto back_batch = [&](bool edge, int rb) {
    if (!edge || (!face && i < nx)) {
      T* cb = col + rb * TI;
      // the upper diagonal in 16-byte pairs (rb is a multiple of 16 rows)
      const double2* cwp = reinterpret_cast<const double2*>(cus + rb);
      T v[R];
      CU cw[R];
#pragma unroll
      for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
#pragma unroll
      for (int q = 0; q < R / 2; ++q) {
        const double2 pr = cwp[q];
        cw[2 * q] = pr.x;
        cw[2 * q + 1] = pr.y;
      }
      if (rb == last_b) {
#pragma unroll
        for (int q = R - 1; q >= 0; --q) {
          if (rb + q < n) {
            xn = back_elem(cw[q], xn, v[q]);
            v[q] = static_cast<T>(xn);
          }
        }
      } else {
#pragma unroll
        for (int q = R - 1; q >= 0; --q) {
          xn = back_elem(cw[q], xn, v[q]);
          v[q] = static_cast<T>(xn);
        }
      }
#pragma unroll
      for (int q = 0; q < R; ++q) cb[q * TI] = v[q];
      if (act) {
        if (rb == 0) col[0] = e0v;
        if (rb == last_b) col[(n - 1) * TI] = e1v;
      }
    }
  };
  for (int rb = last_b; rb >= 0; rb -= R) {
    if (edge_tile)
      back_batch(true, rb);
    else
      back_batch(false, rb);
    // store every chunk whose rows are now all final (uniform across the CTA)
    if (next_store >= 0 && store_row >= rb) {
      fence_async_smem();
      __syncthreads();
      if (t == 0) {
        for (int c = next_store; c >= 0 && c * CH >= rb; --c) {
          const uint32_t src = smem_u32(tile + c * CH * TI);
          if (AXIS == 1)
            tma_store_4d(map, src, i0, c * CH, m, s);
          else
            tma_store_4d(map, src, i0, m, c * CH, s);
        }
        tma_store_commit();
      }
      while (next_store >= 0 && store_row >= rb) {
        --next_store;
        store_row -= CH;
      }
    }
  }
  return true;
}

template <typename T, int AXIS, int TI>
__global__ void __launch_bounds__(TI) sweep_yz_kernel(const __grid_constant__ CUtensorMap map, const SweepParams<T> p,
                                                      int CH) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 128);
  const int n = (AXIS == 1) ? p.ny : p.nz;
  const int C = (n + CH - 1) / CH;
  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(reinterpret_cast<uint64_t*>(base) + c), 1);
    fence_barrier_init();
  }
  __syncthreads();
  uint64_t phase = 0;
  yz_tile<T, AXIS, TI>(&map, p, blockIdx.x * TI, blockIdx.y, p.s_lo + blockIdx.z, CH, base, phase);
  if (threadIdx.x == 0) tma_store_wait_read();
}

// ---------------------------------------------------------------------------
// persistent schedule: a compute warp and a copy warp per CTA
// ---------------------------------------------------------------------------
// CTA b takes tiles b, b + G, b + 2G, ... (G CTAs in the grid, as many as fit
// on the GPU at once).  Warp 0 computes; one lane of warp 1 issues every TMA
// copy, so the compute warp never blocks on a copy it does not need yet.  A
// tile's C chunks live in C shared-memory slots, each with two barriers:
// `full` (the chunk's load landed) and `empty` (the compute warp finished the
// chunk).  The back substitution finishes the chunks from the line's end; the
// copy lane stores each finished chunk and, once the store has read its slot,
// loads the next tile's chunk into it.  The first slot freed must take the
// next tile's chunk 0, so the slot order flips from tile to tile: the k-th
// tile of a CTA keeps chunk c in slot c for even k and in slot C-1-c for odd
// k, and chunk c of tile k is followed in its slot by chunk C-1-c of tile k+1.
// The next tile's loads therefore run under this tile's back substitution and
// its stores under the next tile's forward elimination.  Each barrier
// completes once per tile, so tile k waits on parity k&1.

// CTA b of G takes tiles b, b + G, b + 2G, ...: the tiles in flight at any
// moment are neighbours in memory (contiguous ranges per CTA measured 1.5x
// slower in the x sweep).

// The copy lane's loop, shared by the three sweeps.  load(tile, c, slot)
// issues chunk c of a tile into a slot (arming its full barrier);
// store(tile, c, slot) writes a finished chunk back.  Returns false if a
// wait gave up.
template <typename NextF, typename LoadF, typename StoreF>
__device__ __forceinline__ bool ring_copy_loop(long long tile, long long ntiles, int C, const uint64_t* empty_bars,
                                               NextF next_of, LoadF load, StoreF store) {
  if (tile >= ntiles) return true;
  for (int c = 0; c < C; ++c) load(tile, c, c);
  for (uint32_t k = 0;; ++k) {
    const long long nxt = next_of(tile);
    const bool flip = (k & 1u) != 0;
    for (int q = 0; q < C; ++q) {
      const int c = C - 1 - q;  // chunks in the order the back substitution finishes them
      const int sl = ring_slot(flip, C, c);
      if (!mbar_wait(smem_u32(&empty_bars[sl]), k & 1u)) return false;
      store(tile, c, sl);
      tma_store_commit();
      if (nxt < ntiles) {
        tma_store_wait_read();  // the store has read the slot
        load(nxt, q, sl);       // chunk q of the next tile: slot_{k+1}(q) == slot_k(C-1-q)
      }
    }
    if (nxt >= ntiles) break;
    tile = nxt;
  }
  tma_store_wait_read();
  return true;
}

template <typename T, int AXIS>
__global__ void __launch_bounds__(64 * kMaxRings<T>, 1) sweep_yz_ring_kernel(const __grid_constant__ CUtensorMap map,
                                                                            const SweepParams<T> p,
                                                                            uint32_t ring_bytes) {
  using DR = typename Coef<T>::DR;
  using CU = typename Coef<T>::CU;
  constexpr int R = kRowBatch;
  constexpr int CH = kRingRows;
  static_assert(CH == R, "a y/z ring chunk is one register batch");
  constexpr int TI = 32;
  constexpr int kSlotElems = CH * TI;
  constexpr uint32_t kSlotBytes = kSlotElems * sizeof(T);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 128);
  const int nx = p.nx;
  const int n = (AXIS == 1) ? p.ny : p.nz;
  const int nm = (AXIS == 1) ? p.nz : p.ny;  // the line's other coordinate (k for y, j for z)
  const int C = (n + CH - 1) / CH;
  const int ntx = (nx + TI - 1) / TI;
  const long long per_s = static_cast<long long>(ntx) * nm;
  const long long ntiles = per_s * (p.s_hi - p.s_lo);
  // Rings per CTA: warps 0..rings-1 compute, warp rings + r is ring r's copy
  // warp, so consecutive warps -- which the SM spreads over its four
  // sub-partitions -- put the compute warps on different sub-partitions.
  const int rings = static_cast<int>(blockDim.x) / 64;
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int ring = warp < rings ? warp : warp - rings;
  unsigned char* rbase = base + static_cast<size_t>(ring) * ring_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(rbase);
  uint64_t* empty = full + kMaxChunks;
  T* slots = reinterpret_cast<T*>(rbase + kBarrierBytes);
  CU* cus = reinterpret_cast<CU*>(slots + static_cast<size_t>(C) * kSlotElems);
  const long long stride = static_cast<long long>(gridDim.x) * rings;

  // tile -> (i0, m, s), x tiles fastest
  auto decode = [&](long long tile, int& i0, int& m, int& s) {
    const int sg = static_cast<int>(tile / per_s);
    const long long r = tile - sg * per_s;
    s = p.s_lo + sg;
    m = static_cast<int>(r / ntx);
    i0 = static_cast<int>(r - static_cast<long long>(m) * ntx) * TI;
  };
  // A tile whose lines all lie in an activated face is already final (its
  // input holds the face values, which the pin after the sweep writes again).
  auto skip = [&](long long tile) {
    int i0, m, s;
    decode(tile, i0, m, s);
    return p.active[s] != 0 && (m == 0 || m == nm - 1);
  };
  // the next tile to work on after `tile` (ntiles when there is none)
  auto next_of = [&](long long tile) {
    do {
      tile += stride;
    } while (tile < ntiles && skip(tile));
    return tile < ntiles ? tile : ntiles;
  };
  const long long first = static_cast<long long>(blockIdx.x) * rings + ring;

  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int r = 0; r < rings; ++r) {
      uint64_t* rb = reinterpret_cast<uint64_t*>(base + static_cast<size_t>(r) * ring_bytes);
      for (int c = 0; c < C; ++c) {
        mbar_init(smem_u32(&rb[c]), 1);
        mbar_init(smem_u32(&rb[kMaxChunks + c]), 1);
      }
    }
    fence_barrier_init();
  }
  __syncthreads();
  long long tile = (first < ntiles && !skip(first)) ? first : next_of(first);

  if (warp >= rings) {
    if (t != 0) return;
    auto load = [&](long long tl, int c, int sl) {
      int i0, m, s;
      decode(tl, i0, m, s);
      const uint32_t bar = smem_u32(&full[sl]);
      mbar_expect_tx(bar, kSlotBytes);
      const uint32_t dst = smem_u32(slots + static_cast<size_t>(sl) * kSlotElems);
      if (AXIS == 1)
        tma_load_4d(dst, &map, bar, i0, c * CH, m, s);
      else
        tma_load_4d(dst, &map, bar, i0, m, c * CH, s);
    };
    auto store = [&](long long tl, int c, int sl) {
      int i0, m, s;
      decode(tl, i0, m, s);
      const uint32_t src = smem_u32(slots + static_cast<size_t>(sl) * kSlotElems);
      if (AXIS == 1)
        tma_store_4d(&map, src, i0, c * CH, m, s);
      else
        tma_store_4d(&map, src, i0, m, c * CH, s);
    };
    if (!ring_copy_loop(tile, ntiles, C, empty, next_of, load, store)) atomicExch(p.status, kDevTimeout);
    return;
  }

  const int screen = p.screen;
  int staged_s = -1;
  for (uint32_t k = 0; tile < ntiles; ++k) {
    int i0, m, s;
    decode(tile, i0, m, s);
    const bool flip = (k & 1u) != 0;
    const uint32_t par = k & 1u;
    const bool act = p.active[s] != 0;
    const int i = i0 + t;
    const bool face = act && (i == 0 || i == nx - 1);  // lines in an x face keep their (pinned) input
    const AxisCoefs<T>& ac = (AXIS == 1) ? p.ay : p.az;
    const DR* __restrict__ drp = ac.dr + static_cast<size_t>(s) * ac.npad;
    const CU* __restrict__ cup = ac.cu + static_cast<size_t>(s) * ac.npad;
    const typename Coef<T>::C1 c1 = p.c1[s];
    const double shift = kF32<T> ? p.shift[s] : 0.0;
    // the upper diagonal for the back substitution, restaged when the
    // substrate changes (every lane finished reading the previous copy
    // before the last __syncwarp)
    if (s != staged_s) {
      stage_row(cus, cup, C * CH);
      staged_s = s;
    }
    DR cfa[R], cfb[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      cfa[q] = __ldg(drp + q);
      cfb[q] = __ldg(drp + R + q);
    }
    auto col_of = [&](int c) { return slots + static_cast<size_t>(ring_slot(flip, C, c)) * kSlotElems + t; };
    bool ok = true;
    T e0v = T(0), e1v = T(0);
    double y = -0.0;
    int hwmin = INT_MAX;  // FP64: minimum input high word of this lane's line (the screen)
    // Forward elimination over chunk c (one register batch); rows past n in
    // the last chunk are TMA fill, and their results are never stored.
    // Tiles with no face or out-of-range line run the batches without per-lane checks.
    const bool edge_tile = __any_sync(0xffffffffu, face || i >= nx);
    auto fwd = [&](bool edge, int c, DR (&cf)[R]) {
      if (ok) ok = mbar_wait(smem_u32(&full[ring_slot(flip, C, c)]), par);
      if (edge && (face || i >= nx)) return;  // lines past nx hold TMA fill, never stored
      T* cb = col_of(c);
      const int rb = c * CH;
      T v[R];
#pragma unroll
      for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
      if (act) {
        if (rb == 0) e0v = v[0];
        if (rb + R > n - 1) {
#pragma unroll
          for (int q = 0; q < R; ++q)
            if (rb + q == n - 1) e1v = v[q];
        }
      }
      if (rb + R > n) {  // rows past the line's end (TMA fill): any clean value, never stored
#pragma unroll
        for (int q = 0; q < R; ++q)
          if (rb + q >= n) v[q] = T(1);
      }
      auto put = [&](int q, auto val) { cb[q * TI] = static_cast<T>(val); };
      if constexpr (kF32<T>) {
        y = forward_store<R>(v, cf, c1, shift, screen, y, put);
      } else {
        y = forward_any<R>(screen, v, cf, c1, y, put);
        if (screen != kScreenFast) hwmin = min(hwmin, batch_min_hi<R>(v));
      }
    };
    auto forward_pass = [&](bool edge) {
      for (int c = 0; c < C; c += 2) {
        fwd(edge, c, cfa);
#pragma unroll
        for (int q = 0; q < R; ++q) cfa[q] = __ldg(drp + (c + 2) * R + q);
        if (c + 1 >= C) break;
        fwd(edge, c + 1, cfb);
#pragma unroll
        for (int q = 0; q < R; ++q) cfb[q] = __ldg(drp + (c + 3) * R + q);
      }
    };
    if (edge_tile)
      forward_pass(true);
    else
      forward_pass(false);
    if (!__all_sync(0xffffffffu, ok)) {
      if (t == 0) atomicExch(p.status, kDevTimeout);
      break;
    }
    if constexpr (!kF32<T>) {
      // The screen, once per tile: a line with an input below 2^-960 (or
      // negative) anywhere is redone from its inputs, which are still in the
      // field (this tile's results are stored only by the back substitution).
      if (__any_sync(0xffffffffu, !screen_clean(screen, hwmin))) {
        if (!face && i < nx) {
          const size_t row_stride = (AXIS == 1) ? static_cast<size_t>(p.nxp)
                                                : static_cast<size_t>(p.nxp) * p.ny;
          const T* src = (AXIS == 1) ? p.f + ((static_cast<size_t>(s) * p.nz + m) * p.ny) * p.nxp + i
                                     : p.f + (static_cast<size_t>(s) * p.nz * p.ny + m) * p.nxp + i;
          y = -0.0;
          for (int c = 0; c < C; ++c) {
            const int rb = c * CH;
            T v[R];
            DR cf[R];
#pragma unroll
            for (int q = 0; q < R; ++q) {
              v[q] = rb + q < n ? src[(rb + q) * row_stride] : T(1);
              cf[q] = __ldg(drp + rb + q);
            }
            T* cb = col_of(c);
            y = forward_checked<R>(v, cf, c1, y, [&](int q, auto val) { cb[q * TI] = static_cast<T>(val); });
          }
        }
        __syncwarp();
      }
    }

    // Back substitution, last chunk first; each finished chunk is handed to
    // the copy lane through its empty barrier.
    double xn = -0.0;
    auto back_chunk = [&](bool edge, int c) {
      const int rb = c * CH;
      if (!edge || (!face && i < nx)) {
        T* cb = col_of(c);
        const double2* cwp = reinterpret_cast<const double2*>(cus + rb);  // 16-byte pairs
        T v[R];
        CU cw[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
#pragma unroll
        for (int q = 0; q < R / 2; ++q) {
          const double2 pr = cwp[q];
          cw[2 * q] = pr.x;
          cw[2 * q + 1] = pr.y;
        }
        if (c == C - 1) {
#pragma unroll
          for (int q = R - 1; q >= 0; --q) {
            if (rb + q < n) {
              xn = back_elem(cw[q], xn, v[q]);
              v[q] = static_cast<T>(xn);
            }
          }
        } else {
#pragma unroll
          for (int q = R - 1; q >= 0; --q) {
            xn = back_elem(cw[q], xn, v[q]);
            v[q] = static_cast<T>(xn);
          }
        }
#pragma unroll
        for (int q = 0; q < R; ++q) cb[q * TI] = v[q];
        if (act) {
          if (c == 0) cb[0] = e0v;
          if (c == C - 1) cb[(n - 1 - rb) * TI] = e1v;
        }
      }
    };
    for (int c = C - 1; c >= 0; --c) {
      if (edge_tile)
        back_chunk(true, c);
      else
        back_chunk(false, c);
      fence_async_smem();
      __syncwarp();
      if (t == 0) mbar_arrive(smem_u32(&empty[ring_slot(flip, C, c)]));
    }
    __syncwarp();
    tile = next_of(tile);
  }
}

// x sweep, persistent.  Chunk c of a tile is the 128-byte column [cW, cW+W)
// of its 32 lines (W = 128 / sizeof(T)), staged with the 128B swizzle.  Each
// lane applies the agents of its own line chunk by chunk just before the
// forward elimination reads the chunk: its line's agents are one contiguous,
// x-ordered range of the sorted list, and every voxel's run is applied in
// sorted (agent-list) order, so the result equals applying all agents first.
template <typename T>
__global__ void __launch_bounds__(64) sweep_x_ring_kernel(const __grid_constant__ CUtensorMap map,
                                                          const SweepParams<T> p) {
  using DR = typename Coef<T>::DR;
  using CU = typename Coef<T>::CU;
  constexpr int W = 128 / sizeof(T);
  constexpr int TL = 32;
  constexpr uint32_t kSlotBytes = TL * 128u;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  const int nx = p.nx, ny = p.ny, nz = p.nz, S = p.S;
  const int C = (nx + W - 1) / W;
  const int nty = (ny + TL - 1) / TL;
  const long long per_s = static_cast<long long>(nty) * nz;
  const long long ntiles = per_s * (p.s_hi - p.s_lo);
  uint64_t* full = reinterpret_cast<uint64_t*>(base);
  uint64_t* empty = full + kMaxChunks;
  unsigned char* slots = base + kBarrierBytes;
  CU* cus = reinterpret_cast<CU*>(slots + static_cast<size_t>(C) * kSlotBytes);
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int sw = t & 7;

  auto decode = [&](long long tile, int& j0, int& k, int& s) {
    const int sg = static_cast<int>(tile / per_s);
    const long long r = tile - sg * per_s;
    s = p.s_lo + sg;
    k = static_cast<int>(r / nty);
    j0 = static_cast<int>(r - static_cast<long long>(k) * nty) * TL;
  };
  auto next_of = [&](long long tile) { return tile + gridDim.x < ntiles ? tile + gridDim.x : ntiles; };
  const long long first = blockIdx.x;

  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) {
      mbar_init(smem_u32(&full[c]), 1);
      mbar_init(smem_u32(&empty[c]), 1);
    }
    fence_barrier_init();
  }
  __syncthreads();
  long long tile = first < ntiles ? first : ntiles;

  if (warp == 1) {
    if (t != 0) return;
    auto load = [&](long long tl, int c, int sl) {
      int j0, k, s;
      decode(tl, j0, k, s);
      const uint32_t bar = smem_u32(&full[sl]);
      mbar_expect_tx(bar, kSlotBytes);
      tma_load_4d(smem_u32(slots + static_cast<size_t>(sl) * kSlotBytes), &map, bar, c * W, j0, k, s);
    };
    auto store = [&](long long tl, int c, int sl) {
      int j0, k, s;
      decode(tl, j0, k, s);
      tma_store_4d(&map, smem_u32(slots + static_cast<size_t>(sl) * kSlotBytes), c * W, j0, k, s);
    };
    if (!ring_copy_loop(tile, ntiles, C, empty, next_of, load, store)) atomicExch(p.status, kDevTimeout);
    return;
  }

  const int screen = p.screen;
  int staged_s = -1;
  for (uint32_t kk = 0; tile < ntiles; ++kk) {
    int j0, k, s;
    decode(tile, j0, k, s);
    const bool flip = (kk & 1u) != 0;
    const uint32_t par = kk & 1u;
    const int j = j0 + t;
    const bool valid = j < ny;
    const bool act = p.active[s] != 0;
    const bool face = act && (j == 0 || j == ny - 1 || k == 0 || k == nz - 1);
    // Face-line values: the z-face plane when k is on a z face, else the y-face plane.
    const double* fv = nullptr;
    if (face && valid) {
      if (k == 0 || k == nz - 1)
        fv = p.zface + ((static_cast<size_t>(k == 0 ? 0 : 1) * S + s) * ny + j) * nx;
      else
        fv = p.yface + ((static_cast<size_t>(j == 0 ? 0 : 1) * S + s) * nz + k) * nx;
    }
    const double off = kF32<T> ? p.off[s] : 0.0;
    T x0v = T(0), x1v = T(0);
    if (act && valid) {
      x0v = static_cast<T>(p.xface[(static_cast<size_t>(0 * S + s) * nz + k) * ny + j] - off);
      x1v = static_cast<T>(p.xface[(static_cast<size_t>(1 * S + s) * nz + k) * ny + j] - off);
    }
    const DR* __restrict__ drp = p.ax.dr + static_cast<size_t>(s) * p.ax.npad;
    const CU* __restrict__ cup = p.ax.cu + static_cast<size_t>(s) * p.ax.npad;
    const typename Coef<T>::C1 c1 = p.c1[s];
    const double shift = kF32<T> ? p.shift[s] : 0.0;
    if (s != staged_s) {  // the upper diagonal, restaged when the substrate changes
      stage_row(cus, cup, C * W);
      staged_s = s;
    }
    DR cfa[W], cfb[W];
#pragma unroll
    for (int q = 0; q < W; ++q) {
      cfa[q] = __ldg(drp + q);
      cfb[q] = __ldg(drp + W + q);
    }
    auto row_of = [&](int c) {
      return slots + static_cast<size_t>(ring_slot(flip, C, c)) * kSlotBytes + t * 128;
    };
    // This lane's agents: sorted positions [a, a_end) of line k*ny + j.
    int a = 0, a_end = 0;
    unsigned line_key0 = 0;
    if (p.line_off != nullptr && valid) {
      const int line = k * ny + j;
      a = __ldg(p.line_off + line);
      a_end = __ldg(p.line_off + line + 1);
      line_key0 = static_cast<unsigned>(line) * static_cast<unsigned>(nx);
    }
    const double* ac1 = p.ac1 + static_cast<size_t>(s) * p.n_sorted;
    const double* ac2 = p.ac2 + static_cast<size_t>(s) * p.n_sorted;
    const double* ae2 = p.ae2 + static_cast<size_t>(s) * p.n_sorted;
    unsigned akey = a < a_end ? __ldg(p.a_key + a) : 0u;

    bool ok = true;
    double y = -0.0;
    // Tiles with no face or out-of-range line run the batches without per-lane checks.
    const bool edge_tile = __any_sync(0xffffffffu, face || !valid);
    auto fwd = [&](bool edge, int c, DR (&cf)[W]) {
      if (ok) ok = mbar_wait(smem_u32(&full[ring_slot(flip, C, c)]), par);
      unsigned char* crow = row_of(c);
      const int i0 = c * W;
      // agents of this lane's line inside chunk c, each voxel's run in order
      const unsigned lim = line_key0 + static_cast<unsigned>(i0 + W);
      while (a < a_end && akey < lim) {
        T* e = swz_elem<T>(crow, static_cast<int>(akey - line_key0) - i0, sw);
        double r = static_cast<double>(*e);
        if constexpr (kF32<T>) r += off;
        const unsigned key = akey;
        do {
          r = agent_update(r, __ldg(ac1 + a), __ldg(ac2 + a), __ldg(ae2 + a), a, s, p.track);
          ++a;
          akey = a < a_end ? __ldg(p.a_key + a) : 0u;
        } while (a < a_end && akey == key);
        if constexpr (kF32<T>) r -= off;
        *e = static_cast<T>(r);
      }
      if (edge && (face || !valid)) return;  // lines past ny hold TMA fill, never stored
      // the pin before the sweep, on the staged row (after the sources)
      if (act) {
        if (i0 == 0) *swz_elem<T>(crow, 0, sw) = x0v;
        if (nx - 1 < i0 + W) *swz_elem<T>(crow, nx - 1 - i0, sw) = x1v;
      }
      T v[W];
      load_row<T, W>(crow, sw, v);
      if (i0 + W > nx) {  // TMA fill past the line's end: any clean value (results never stored)
#pragma unroll
        for (int q = 0; q < W; ++q)
          if (i0 + q >= nx) v[q] = T(1);
      }
      RowPut<T> put{crow, sw};
      y = forward_store<W>(v, cf, c1, shift, screen, y, put);
    };
    auto forward_pass = [&](bool edge) {
      for (int c = 0; c < C; c += 2) {
        fwd(edge, c, cfa);
#pragma unroll
        for (int q = 0; q < W; ++q) cfa[q] = __ldg(drp + (c + 2) * W + q);
        if (c + 1 >= C) break;
        fwd(edge, c + 1, cfb);
#pragma unroll
        for (int q = 0; q < W; ++q) cfb[q] = __ldg(drp + (c + 3) * W + q);
      }
    };
    if (edge_tile)
      forward_pass(true);
    else
      forward_pass(false);
    if (!__all_sync(0xffffffffu, ok)) {
      if (t == 0) atomicExch(p.status, kDevTimeout);
      break;
    }

    // Back substitution, last chunk first; each finished chunk is handed to
    // the copy lane through its empty barrier.
    double xn = -0.0;
    auto back_chunk = [&](bool edge, int c) {
      const bool E = edge;
      unsigned char* crow = row_of(c);
      const int i0 = c * W;
      CU cw[W];
      const double2* cwp = reinterpret_cast<const double2*>(cus + i0);  // 16-byte pairs
#pragma unroll
      for (int q = 0; q < W / 2; ++q) {
        const double2 pr = cwp[q];
        cw[2 * q] = pr.x;
        cw[2 * q + 1] = pr.y;
      }
      if (E && face) {
        T fw[W];
#pragma unroll
        for (int q = 0; q < W; ++q) fw[q] = (fv != nullptr && i0 + q < nx) ? static_cast<T>(fv[i0 + q] - off) : T(0);
#pragma unroll
        for (int q = 0; q < W; ++q)
          if (i0 + q < nx) *swz_elem<T>(crow, q, sw) = fw[q];
      } else if (!E || valid) {
        T v[W];
        load_row<T, W>(crow, sw, v);
        if (i0 + W > nx) {
#pragma unroll
          for (int q = W - 1; q >= 0; --q) {
            if (i0 + q < nx) {
              xn = back_elem(cw[q], xn, v[q]);
              v[q] = static_cast<T>(xn);
            }
          }
        } else {
#pragma unroll
          for (int q = W - 1; q >= 0; --q) {
            xn = back_elem(cw[q], xn, v[q]);
            v[q] = static_cast<T>(xn);
          }
        }
        store_row<T, W>(crow, sw, v);
        if (act) {
          if (i0 == 0) *swz_elem<T>(crow, 0, sw) = x0v;
          if (nx - 1 < i0 + W) *swz_elem<T>(crow, nx - 1 - i0, sw) = x1v;
        }
      }
    };
    for (int c = C - 1; c >= 0; --c) {
      if (edge_tile)
        back_chunk(true, c);
      else
        back_chunk(false, c);
      fence_async_smem();
      __syncwarp();
      if (t == 0) mbar_arrive(smem_u32(&empty[ring_slot(flip, C, c)]));
    }
    __syncwarp();
    tile = next_of(tile);
  }
}

// ---------------------------------------------------------------------------
// batched step: x, y and z sweeps of many solves in one launch
// ---------------------------------------------------------------------------
// Persistent CTAs (one warp each) take tiles from one ordered list -- every
// x tile of every member, then every y tile, then every z tile -- through an
// atomic dispenser.  A y (z) tile of member e starts once all x (y) tiles of
// e are done: each finished tile bumps a per-member counter with release
// semantics after its bulk stores have completed.  Tiles are handed out in
// list order, so every tile a waiting CTA depends on is already held by a
// running CTA that does not itself wait on anything later: the waits always
// end (and are bounded anyway).
template <typename T>
__global__ void __launch_bounds__(kBatchTile) batch_step_kernel(const BatchHeader* __restrict__ hdr,
                                                                const BatchEnv<T>* __restrict__ envs,
                                                                const int* __restrict__ pre, int cap,
                                                                int* __restrict__ counters, int* __restrict__ status) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ int s_item;
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  const int t = threadIdx.x;
  if (t == 0) {
    for (int c = 0; c < kMaxChunks; ++c) mbar_init(smem_u32(reinterpret_cast<uint64_t*>(base) + c), 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int n_env = hdr->n_env;
  const int n0 = hdr->n_items[0], n1 = hdr->n_items[1], n2 = hdr->n_items[2];
  const int total = n0 + n1 + n2;
  int* dispenser = counters;
  int* done = counters + 1;
  uint64_t phase = 0;
  for (;;) {
    if (t == 0) s_item = atomicAdd(dispenser, 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= total) break;
    int axis, local;
    if (item < n0) {
      axis = 0;
      local = item;
    } else if (item < n0 + n1) {
      axis = 1;
      local = item - n0;
    } else {
      axis = 2;
      local = item - n0 - n1;
    }
    const int* pa = pre + axis * (cap + 1);
    int lo = 0, hi = n_env - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(pa + mid) <= local)
        lo = mid;
      else
        hi = mid - 1;
    }
    const int e = lo;
    const int tile = local - __ldg(pa + e);
    const BatchEnv<T>& E = envs[e];
    if (axis > 0) {
      const int* pb = pre + (axis - 1) * (cap + 1);
      const int need = __ldg(pb + e + 1) - __ldg(pb + e);
      if (t == 0) {
        const int* cnt = done + (axis - 1) * cap + e;
        if (ld_acquire_gpu(cnt) < need) {
          const unsigned long long t0 = global_ns();
          const unsigned long long limit = g_wait_limit_ns;
          while (ld_acquire_gpu(cnt) < need) {
            __nanosleep(128);
            if (global_ns() - t0 > limit) {
              atomicExch(status, kDevTimeout);
              break;
            }
          }
        }
        fence_async_global();
      }
      __syncthreads();
    }
    const SweepParams<T>& p = E.p;
    if (axis == 0) {
      const int per = E.nty * p.nz;
      const int s = tile / per, r = tile - s * per;
      const int k = r / E.nty;
      x_tile<T>(&E.mx, p, (r - k * E.nty) * kBatchTile, k, s, base, phase);
    } else if (axis == 1) {
      const int per = E.ntx * p.nz;
      const int s = tile / per, r = tile - s * per;
      const int k = r / E.ntx;
      yz_tile<T, 1, kBatchTile>(&E.my, p, (r - k * E.ntx) * kBatchTile, k, s, E.chy, base, phase);
    } else {
      const int per = E.ntx * p.ny;
      const int s = tile / per, r = tile - s * per;
      const int j = r / E.ntx;
      yz_tile<T, 2, kBatchTile>(&E.mz, p, (r - j * E.ntx) * kBatchTile, j, s, E.chz, base, phase);
    }
    if (t == 0) {
      tma_store_wait_all();
      fence_async_global();
      red_release_gpu_add(done + axis * cap + e, 1);
    }
  }
}

// Split schedule: one launch per sweep over the tiles of every member (the
// kernel boundary orders the sweeps; blocks map to tiles through the same
// prefix table).
template <typename T, int AXIS>
__global__ void __launch_bounds__(kBatchTile) batch_sweep_kernel(const BatchHeader* __restrict__ hdr,
                                                                 const BatchEnv<T>* __restrict__ envs,
                                                                 const int* __restrict__ pre, int cap) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  const int local = blockIdx.x;
  if (local >= hdr->n_items[AXIS]) return;
  const int* pa = pre + AXIS * (cap + 1);
  int lo = 0, hi = hdr->n_env - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(pa + mid) <= local)
      lo = mid;
    else
      hi = mid - 1;
  }
  const BatchEnv<T>& E = envs[lo];
  const SweepParams<T>& p = E.p;
  const int tile = local - __ldg(pa + lo);
  int C;
  if (AXIS == 0)
    C = (p.nx + kChunkX<T> - 1) / kChunkX<T>;
  else
    C = ((AXIS == 1 ? p.ny : p.nz) + (AXIS == 1 ? E.chy : E.chz) - 1) / (AXIS == 1 ? E.chy : E.chz);
  if (threadIdx.x == 0) {
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(reinterpret_cast<uint64_t*>(base) + c), 1);
    fence_barrier_init();
  }
  __syncthreads();
  uint64_t phase = 0;
  if (AXIS == 0) {
    const int per = E.nty * p.nz;
    const int s = tile / per, r = tile - s * per;
    const int k = r / E.nty;
    x_tile<T>(&E.mx, p, (r - k * E.nty) * kBatchTile, k, s, base, phase);
  } else if (AXIS == 1) {
    const int per = E.ntx * p.nz;
    const int s = tile / per, r = tile - s * per;
    const int k = r / E.ntx;
    yz_tile<T, 1, kBatchTile>(&E.my, p, (r - k * E.ntx) * kBatchTile, k, s, E.chy, base, phase);
  } else {
    const int per = E.ntx * p.ny;
    const int s = tile / per, r = tile - s * per;
    const int j = r / E.ntx;
    yz_tile<T, 2, kBatchTile>(&E.mz, p, (r - j * E.ntx) * kBatchTile, j, s, E.chz, base, phase);
  }
  if (threadIdx.x == 0) tma_store_wait_read();
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t sweep_x_smem(int elem_bytes, int nx, const SweepConfig& cfg) {
  const int W = 128 / elem_bytes;
  const int C = (nx + W - 1) / W;
  if (C > kMaxChunks) return ~size_t(0);
  // alignment pad, barriers, the tile, the staged upper-diagonal row
  return 1024 + kBarrierBytes + static_cast<size_t>(C) * cfg.x_lines * 128 + static_cast<size_t>(C) * W * 8;
}

static int yz_chunk_rows(int n, int target) {
  const int C = (n + target - 1) / target;
  return (n + C - 1) / C;
}

// The y/z tile holds a whole number of register batches (kRowBatch rows) so
// the last batch of a line never reads outside the tile.
size_t sweep_yz_smem(int elem_bytes, int n_line, const SweepConfig& cfg) {
  const int CH = yz_chunk_rows(n_line, cfg.yz_chunk);
  const int C = (n_line + CH - 1) / CH;
  if (C > kMaxChunks) return ~size_t(0);
  const size_t rows = (static_cast<size_t>(C) * CH + kRowBatch - 1) / kRowBatch * kRowBatch;
  // alignment pad, barriers, the tile, the staged upper-diagonal row
  return 128 + kBarrierBytes + rows * cfg.yz_tile * elem_bytes + rows * 8;
}

size_t ring_x_smem(int elem_bytes, int nx) {
  const int W = 128 / elem_bytes;
  const int C = (nx + W - 1) / W;
  if (C > kMaxChunks) return 0;
  // alignment pad, barriers, C slots of 32 rows of 128 bytes, the staged upper-diagonal row
  return 1024 + kBarrierBytes + static_cast<size_t>(C) * 32 * 128 + static_cast<size_t>(C) * W * 8;
}

// One y/z ring: barriers, C slots of kRingRows rows of 32 values, the staged
// upper-diagonal row (a multiple of 128 bytes, so rings stack aligned).
size_t ring_yz_bytes(int elem_bytes, int n_line) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  if (C > kMaxChunks) return 0;
  const size_t rows = static_cast<size_t>(C) * kRingRows;
  return kBarrierBytes + rows * 32 * elem_bytes + rows * 8;
}

// Rings per persistent y/z CTA: as many as fit (up to kMaxRings), 0 if none.
static int ring_yz_count(int elem_bytes, int n_line) {
  const size_t rb = ring_yz_bytes(elem_bytes, n_line);
  if (rb == 0) return 0;
  const int fit = static_cast<int>((227 * 1024 - 128) / rb);
  const int cap = elem_bytes == 4 ? kMaxRings<float> : kMaxRings<double>;
  return fit < cap ? fit : cap;
}

size_t ring_yz_smem(int elem_bytes, int n_line) {
  const int rings = ring_yz_count(elem_bytes, n_line);
  return rings == 0 ? 0 : 128 + rings * ring_yz_bytes(elem_bytes, n_line);
}

static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (fn == nullptr) {
    cudaDriverEntryPointQueryResult q;
    void* ptr = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

static int encode_one(CUtensorMap* map, void* f, int elem_bytes, const cuuint64_t dims[4], const cuuint64_t strides[3],
                      const cuuint32_t box[4], CUtensorMapSwizzle swz, int rank = 4) {
  auto enc = get_encode();
  if (enc == nullptr) return -1;
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                   static_cast<cuuint32_t>(rank), f, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -2;
}

int encode_field_maps(FieldMaps* maps, void* f, int eb, int nx, int ny, int nz, int S, int nxp,
                      const SweepConfig& cfg) {
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)S};
  const cuuint64_t strides[3] = {(cuuint64_t)nxp * eb, (cuuint64_t)nxp * ny * eb, (cuuint64_t)nxp * ny * nz * eb};
  const cuuint32_t bx[4] = {(cuuint32_t)(128 / eb), (cuuint32_t)cfg.x_lines, 1, 1};
  const cuuint32_t by[4] = {(cuuint32_t)cfg.yz_tile, (cuuint32_t)yz_chunk_rows(ny, cfg.yz_chunk), 1, 1};
  const cuuint32_t bz[4] = {(cuuint32_t)cfg.yz_tile, 1, (cuuint32_t)yz_chunk_rows(nz, cfg.yz_chunk), 1};
  const cuuint32_t bry[4] = {32, (cuuint32_t)kRingRows, 1, 1};
  const cuuint32_t brz[4] = {32, 1, (cuuint32_t)kRingRows, 1};
  int rc = encode_one(&maps->x, f, eb, dims, strides, bx, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == 0) rc = encode_one(&maps->y, f, eb, dims, strides, by, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc == 0) rc = encode_one(&maps->z, f, eb, dims, strides, bz, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc == 0) rc = encode_one(&maps->ry, f, eb, dims, strides, bry, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc == 0) rc = encode_one(&maps->rz, f, eb, dims, strides, brz, CU_TENSOR_MAP_SWIZZLE_NONE);
  // the gradient kernel's plane boxes: 32 x with a halo rounded out to 16-byte
  // boundaries, one y plane, 8 z with a one-voxel halo, up to 4 substrates
  const cuuint32_t bg[4] = {(cuuint32_t)(eb == 8 ? 36 : 40), 1, 10, (cuuint32_t)(S < 4 ? S : 4)};
  maps->g_ok = rc == 0 && encode_one(&maps->g, f, eb, dims, strides, bg, CU_TENSOR_MAP_SWIZZLE_NONE) == 0;
  // the tensor-memory x sweeps' rows: planes are contiguous (stride ny rows),
  // so row k * ny + j of a substrate is one dimension
  const unsigned long long rows = static_cast<unsigned long long>(ny) * nz;
  const cuuint64_t dr[4] = {(cuuint64_t)nx, (cuuint64_t)rows, (cuuint64_t)S, 1};
  const cuuint64_t sr[3] = {(cuuint64_t)nxp * eb, (cuuint64_t)nxp * rows * eb, 0};
  const cuuint32_t br[4] = {(cuuint32_t)(128 / eb), 32, 1, 1};
  maps->xr_ok = rc == 0 && rows < (1ull << 31) - 64 &&
                encode_one(&maps->xr, f, eb, dr, sr, br, CU_TENSOR_MAP_SWIZZLE_128B, 3) == 0;
  // the y/z sweeps' packed partial x tiles: a box of pw x by 32 / pw planes
  // by kRingRows rows along the line (the y map lists plane k before row j)
  maps->pyz_w = 0;
  const int rem = nx % 32;
  if (rc == 0 && rem != 0 && rem <= 16) {
    int w = 16 / eb;  // a box row of at least 16 bytes
    while (w < rem) w *= 2;
    const cuuint32_t bp[4] = {(cuuint32_t)w, (cuuint32_t)(32 / w), (cuuint32_t)kRingRows, 1};
    const cuuint64_t dpy[4] = {(cuuint64_t)nx, (cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)S};
    const cuuint64_t spy[3] = {(cuuint64_t)nxp * ny * eb, (cuuint64_t)nxp * eb, (cuuint64_t)nxp * ny * nz * eb};
    if (encode_one(&maps->py, f, eb, dpy, spy, bp, CU_TENSOR_MAP_SWIZZLE_NONE) == 0 &&
        encode_one(&maps->pz, f, eb, dims, strides, bp, CU_TENSOR_MAP_SWIZZLE_NONE) == 0)
      maps->pyz_w = w;
  }
  return rc;
}

static bool use_ring_x(int eb, int nx, const SweepConfig& cfg) {
  return cfg.persistent >= 2 && cfg.x_lines == 32 && ring_x_smem(eb, nx) != 0 && ring_x_smem(eb, nx) <= 227 * 1024;
}

static bool use_ring_yz(int eb, int n, const SweepConfig& cfg) {
  return cfg.persistent >= 1 && cfg.yz_tile == 32 && ring_yz_smem(eb, n) != 0 && ring_yz_smem(eb, n) <= 227 * 1024;
}

template <typename T>
cudaError_t launch_sweep_x(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  {
    bool launched = false;
    cudaError_t e;
    if (maps.xr_ok) {
      if constexpr (sizeof(T) == 8)
        e = launch_tmem_x(maps.xr, p, cfg, st, &launched);
      else
        e = launch_tmem_x_f32(maps.xr, p, cfg, st, &launched);
      if (e != cudaSuccess || launched) return e;
    }
  }
  if (use_ring_x(sizeof(T), p.nx, cfg)) {
    const size_t smem = ring_x_smem(sizeof(T), p.nx);
    const long long tiles = static_cast<long long>((p.ny + 31) / 32) * p.nz * (p.s_hi - p.s_lo);
    int grid = 0;
    cudaError_t e = persistent_grid(sweep_x_ring_kernel<T>, smem, tiles, &grid);
    if (e != cudaSuccess) return e;
    sweep_x_ring_kernel<T><<<grid, 64, smem, st>>>(maps.x, p);
    return cudaGetLastError();
  }
  const size_t smem = sweep_x_smem(sizeof(T), p.nx, cfg);
  cudaError_t e = cudaFuncSetAttribute(sweep_x_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.ny + cfg.x_lines - 1) / cfg.x_lines, p.nz, p.s_hi - p.s_lo);
  sweep_x_kernel<T><<<grid, cfg.x_lines, smem, st>>>(maps.x, p);
  return cudaGetLastError();
}

// One y or z sweep launch with the tile width as a compile-time constant.
template <typename T, int AXIS, int TI>
static cudaError_t launch_yz(const CUtensorMap& map, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  const int n = (AXIS == 1) ? p.ny : p.nz;
  const size_t smem = sweep_yz_smem(sizeof(T), n, cfg);
  cudaError_t e = cudaFuncSetAttribute(sweep_yz_kernel<T, AXIS, TI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.nx + TI - 1) / TI, (AXIS == 1) ? p.nz : p.ny, p.s_hi - p.s_lo);
  sweep_yz_kernel<T, AXIS, TI><<<grid, TI, smem, st>>>(map, p, yz_chunk_rows(n, cfg.yz_chunk));
  return cudaGetLastError();
}

// Tiles per resident CTA below which the persistent y/z sweeps lose to one
// CTA per tile (measured on B200: FP64 100^3 and FP32 200^3 ran slower
// persistent, FP64 200^3 / 400^3 and FP32 640^3 faster).
constexpr long long kRingMinTilesPerCta = 8;

template <typename T, int AXIS>
static cudaError_t launch_yz_any(const CUtensorMap& map, const CUtensorMap& ring_map, const CUtensorMap& pmap, int pw,
                                 const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  const int n = (AXIS == 1) ? p.ny : p.nz;
  {
    bool launched = false;
    cudaError_t e;
    if constexpr (sizeof(T) == 8)
      e = launch_tmem_yz<AXIS>(ring_map, pmap, pw, p, cfg, st, &launched);
    else
      e = launch_tmem_yz_f32<AXIS>(ring_map, pmap, pw, p, cfg, st, &launched);
    if (e != cudaSuccess || launched) return e;
  }
  if (use_ring_yz(sizeof(T), n, cfg)) {
    const int rings = ring_yz_count(sizeof(T), n);
    const size_t smem = ring_yz_smem(sizeof(T), n);
    const long long tiles = static_cast<long long>((p.nx + 31) / 32) * ((AXIS == 1) ? p.nz : p.ny) * (p.s_hi - p.s_lo);
    int grid = 0;
    cudaError_t e = persistent_grid(sweep_yz_ring_kernel<T, AXIS>, smem, (tiles + rings - 1) / rings, &grid,
                                    64 * rings);
    if (e != cudaSuccess) return e;
    if (cfg.persistent >= 2 || tiles >= kRingMinTilesPerCta * grid * rings) {
      sweep_yz_ring_kernel<T, AXIS>
          <<<grid, 64 * rings, smem, st>>>(ring_map, p, static_cast<uint32_t>(ring_yz_bytes(sizeof(T), n)));
      return cudaGetLastError();
    }
  }
  switch (cfg.yz_tile) {
    case 16:
      if constexpr (sizeof(T) == 8) return launch_yz<T, AXIS, 16>(map, p, cfg, st);
      return cudaErrorInvalidValue;
    case 32: return launch_yz<T, AXIS, 32>(map, p, cfg, st);
    case 64: return launch_yz<T, AXIS, 64>(map, p, cfg, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T>
cudaError_t launch_sweep_y(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  return launch_yz_any<T, 1>(maps.y, maps.ry, maps.py, maps.pyz_w, p, cfg, st);
}

template <typename T>
cudaError_t launch_sweep_z(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  return launch_yz_any<T, 2>(maps.z, maps.rz, maps.pz, maps.pyz_w, p, cfg, st);
}

template cudaError_t launch_sweep_x<double>(const FieldMaps&, const SweepParams<double>&, const SweepConfig&,
                                            cudaStream_t);
template cudaError_t launch_sweep_x<float>(const FieldMaps&, const SweepParams<float>&, const SweepConfig&,
                                           cudaStream_t);
template cudaError_t launch_sweep_y<double>(const FieldMaps&, const SweepParams<double>&, const SweepConfig&,
                                            cudaStream_t);
template cudaError_t launch_sweep_y<float>(const FieldMaps&, const SweepParams<float>&, const SweepConfig&,
                                           cudaStream_t);
template cudaError_t launch_sweep_z<double>(const FieldMaps&, const SweepParams<double>&, const SweepConfig&,
                                            cudaStream_t);
template cudaError_t launch_sweep_z<float>(const FieldMaps&, const SweepParams<float>&, const SweepConfig&,
                                           cudaStream_t);


size_t batch_member_smem(int eb, int nx, int ny, int nz, int yz_chunk) {
  SweepConfig cfg;
  cfg.x_lines = kBatchTile;
  cfg.yz_tile = kBatchTile;
  cfg.yz_chunk = yz_chunk;
  const size_t a = sweep_x_smem(eb, nx, cfg), b = sweep_yz_smem(eb, ny, cfg), c = sweep_yz_smem(eb, nz, cfg);
  size_t m = a > b ? a : b;
  m = m > c ? m : c;
  // the x layout aligns to 1024 bytes; the fused kernel uses it for every sweep
  return m + 1024;
}

size_t batch_axis_smem(int eb, int axis, int n_line, int yz_chunk) {
  SweepConfig cfg;
  cfg.x_lines = kBatchTile;
  cfg.yz_tile = kBatchTile;
  cfg.yz_chunk = yz_chunk;
  return (axis == 0 ? sweep_x_smem(eb, n_line, cfg) : sweep_yz_smem(eb, n_line, cfg)) + 1024;
}

template <typename T>
cudaError_t batch_occupancy(size_t smem, int* ctas_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(batch_step_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, batch_step_kernel<T>, kBatchTile, smem);
}

template <typename T>
cudaError_t launch_batch_step(const BatchHeader* hdr, const BatchEnv<T>* envs, const int* pre, int cap, int* counters,
                              int* status, int grid, size_t smem, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(batch_step_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  batch_step_kernel<T><<<grid, kBatchTile, smem, st>>>(hdr, envs, pre, cap, counters, status);
  return cudaGetLastError();
}

template cudaError_t batch_occupancy<double>(size_t, int*);
template cudaError_t batch_occupancy<float>(size_t, int*);
template cudaError_t launch_batch_step<double>(const BatchHeader*, const BatchEnv<double>*, const int*, int, int*, int*,
                                               int, size_t, cudaStream_t);
template cudaError_t launch_batch_step<float>(const BatchHeader*, const BatchEnv<float>*, const int*, int, int*, int*,
                                              int, size_t, cudaStream_t);


template <typename T>
cudaError_t launch_batch_sweeps(const BatchHeader* hdr, const BatchEnv<T>* envs, const int* pre, int cap,
                                const int items[3], const size_t smem[3], cudaStream_t st) {
  cudaError_t e;
  if (items[0] > 0) {
    e = cudaFuncSetAttribute(batch_sweep_kernel<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem[0]));
    if (e != cudaSuccess) return e;
    batch_sweep_kernel<T, 0><<<items[0], kBatchTile, smem[0], st>>>(hdr, envs, pre, cap);
  }
  if (items[1] > 0) {
    e = cudaFuncSetAttribute(batch_sweep_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem[1]));
    if (e != cudaSuccess) return e;
    batch_sweep_kernel<T, 1><<<items[1], kBatchTile, smem[1], st>>>(hdr, envs, pre, cap);
  }
  if (items[2] > 0) {
    e = cudaFuncSetAttribute(batch_sweep_kernel<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem[2]));
    if (e != cudaSuccess) return e;
    batch_sweep_kernel<T, 2><<<items[2], kBatchTile, smem[2], st>>>(hdr, envs, pre, cap);
  }
  return cudaGetLastError();
}

template cudaError_t launch_batch_sweeps<double>(const BatchHeader*, const BatchEnv<double>*, const int*, int,
                                                 const int[3], const size_t[3], cudaStream_t);
template cudaError_t launch_batch_sweeps<float>(const BatchHeader*, const BatchEnv<float>*, const int*, int,
                                                const int[3], const size_t[3], cudaStream_t);

cudaError_t sweeps_set_wait_limit(unsigned long long ns) { return set_module_wait_limit(ns); }

}  // namespace bfvm
