// bfvm_part_sweeps.cu -- the partitioned y and z sweeps of chain 2
// (bfvm_set_fp64_chain(ctx, 2)), for lines of at least kPartMinLine voxels.
//
// The reference solves each Thomas system with one serial recurrence per
// line (BioFVM/BioFVM_solvers.cpp:684-777): forward y_i = (p_i + c1 y_{i-1})
// / d_i, backward x_i = y_i - c_i x_{i+1}.  A thread per line runs that
// chain element after element, so a sweep's speed is the latency of one
// dependent step times the line length, and the lines an SM can hold at once
// (shared memory and TMEM) bound how many chains hide each other's latency.
// Long lines leave few of them in flight: at 640 voxels the serial y/z sweep
// holds 64 FP64 lines per SM.
//
// Here the recurrences are the same linear maps, evaluated by a partition
// method.  A CTA stages one tile of 32 lines (32 consecutive x, all rows of
// the line) and runs 8 warps over it; warp w owns the rows [w m, (w+1) m)
// of every line (m = ceil(n/8)).  With a_i = c1 RN(1/d_i), b_i = p_i
// RN(1/d_i) and g_i = -c_i (g_{n-1} = 0):
//   1. each warp runs the forward recurrence over its segment from 0:
//      y0_i = a_i y0_{i-1} + b_i, in place, and publishes its last value;
//   2. each warp combines the segments before it into the value entering its
//      own, y_in(w) = A_{w-1} y_in(w-1) + y0_end(w-1) (A_w = product of the
//      segment's a), then, from its segment's end back to its start, forms
//      y_i = P_i y_in + y0_i (P_i = product of a from the segment start to i)
//      and runs the backward recurrence from 0: x0_i = g_i x0_{i+1} + y_i,
//      publishing its first value;
//   3. each warp combines the segments after it, x_in(w) = G_{w+1}
//      x_in(w+1) + x0_start(w+1) (G_w = product of the segment's g), and
//      forms x_i = Q_i x_in + x0_i (Q_i = product of g from i to the segment
//      end).
// The products P, Q, A, G depend only on the coefficients; the host forms
// them in extended precision and rounds each once.  A line's chain is a
// segment long (80 at n = 640 instead of 640) and 8 warps work on each tile.
//
// The arithmetic is not the reference's operation order: results differ by
// a few units in the last place per sweep (tests hold the FP64 results to
// 1e-12 relative per voxel of the reference).  The FP32 form uses the same
// kernels with its FP32 storage and FP64 arithmetic (each value is stored
// three times per sweep instead of once).
//
// Dirichlet semantics are those of the serial y and z sweeps
// (bfvm_sweeps.cu): lines in an activated x face and whole tiles in an
// activated face of the other axis keep their input (pinned by the sweep
// before), and the two line ends of an activated substrate are restored
// after the sweep.
#include "bfvm_ctx.h"
#include "bfvm_ptx.cuh"
#include "bfvm_sweep_common.cuh"

namespace bfvm {

namespace {

constexpr int kTL = 32;  // lines per tile (one per lane)

// Shared memory of one CTA: barriers [kPartMaxChunks], the segment ends
// [2][kPartWarps][32] FP64, then the tile [C * kRingRows rows][32 x].
constexpr int kBarBytes = kPartMaxChunks * 8;
constexpr int kSegBytes = 2 * kPartWarps * kTL * 8;
constexpr int kPartHead = ((kBarBytes + 127) / 128) * 128 + kSegBytes;

// Elements of one staged line processed per group: every load of a group is
// issued before its arithmetic.
constexpr int kGroup = 8;

// One tile: the lines (i0 .. i0+31, m, s) along y (AXIS 1, m = k) or z
// (AXIS 2, m = j).
template <typename T, int AXIS>
__global__ void __launch_bounds__(32 * kPartWarps) sweep_part_kernel(const __grid_constant__ CUtensorMap map,
                                                                     const SweepParams<T> p, const PartAxis pa) {
  static_assert(AXIS == 1 || AXIS == 2, "partitioned sweeps run along y and z");
  constexpr uint32_t kChunkBytes = kRingRows * kTL * static_cast<uint32_t>(sizeof(T));
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 128);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  double* yseg = reinterpret_cast<double*>(base + ((kBarBytes + 127) / 128) * 128);  // [kPartWarps][32]
  double* xseg = yseg + kPartWarps * kTL;
  T* tile = reinterpret_cast<T*>(base + kPartHead);
  const int w = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int n = AXIS == 1 ? ny : nz;
  const int C = (n + kRingRows - 1) / kRingRows;
  const int i0 = blockIdx.x * kTL, m = blockIdx.y, s = p.s_lo + static_cast<int>(blockIdx.z);
  const bool act = p.active[s] != 0;
  if (act && (m == 0 || m == (AXIS == 1 ? nz : ny) - 1)) return;  // a face tile is final already

  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(&bars[c]), 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int c = 0; c < C; ++c) {
      const uint32_t bar = smem_u32(&bars[c]);
      mbar_expect_tx(bar, kChunkBytes);
      const uint32_t dst = smem_u32(tile + static_cast<size_t>(c) * kRingRows * kTL);
      if (AXIS == 1)
        tma_load_4d(dst, &map, bar, i0, c * kRingRows, m, s);
      else
        tma_load_4d(dst, &map, bar, i0, m, c * kRingRows, s);
    }
  }
  const int mseg = pa.mseg;
  const int e_lo = w * mseg, e_hi = min(n, e_lo + mseg);
  // wait for the chunks this warp's segment touches
  bool ok = true;
  for (int c = e_lo / kRingRows; c < C && c * kRingRows < e_hi; ++c)
    if (ok) ok = mbar_wait(smem_u32(&bars[c]), 0u);

  const int i = i0 + t;
  // lanes in an activated x face, and lanes past nx, keep their input
  const bool keep = (act && (i == 0 || i == nx - 1)) || i >= nx;
  const double shift = kF32<T> ? p.shift[s] : 0.0;
  T* col = tile + t;  // row e of this lane's line: col[e * kTL]
  T e0v = T(0), e1v = T(0);  // the line ends' input (pinned by the sweep before)
  if (ok && act) {
    if (e_lo == 0 && e_hi > 0) e0v = col[0];
    if (e_lo <= n - 1 && n - 1 < e_hi) e1v = col[static_cast<size_t>(n - 1) * kTL];
  }
  const double2* __restrict__ ra = pa.ra + static_cast<size_t>(s) * pa.npad;  // {RN(1/d), a}
  const double2* __restrict__ pg = pa.pg + static_cast<size_t>(s) * pa.npad;  // {P, g}
  const double* __restrict__ qq = pa.q + static_cast<size_t>(s) * pa.npad;    // Q
  const double2* __restrict__ ag = pa.ag + static_cast<size_t>(s) * kPartWarps;  // {A_w, G_w}
  constexpr int G = kGroup;

  // 1. forward over the segment from 0, in place (the coefficient rows are
  // padded past n, so their loads need no bound; the staged values do)
  double y = 0.0;
  if (!keep && ok) {
    for (int e0 = e_lo; e0 < e_hi; e0 += G) {
      const int ng = e_hi - e0;
      double2 c[G];
      double v[G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        c[q] = __ldg(ra + e0 + q);
        v[q] = q < ng ? static_cast<double>(col[static_cast<size_t>(e0 + q) * kTL]) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q < ng) {
          y = __fma_rn(c[q].y, y, __dmul_rn(kF32<T> ? v[q] - shift : v[q], c[q].x));
          col[static_cast<size_t>(e0 + q) * kTL] = static_cast<T>(y);
        }
      }
    }
  }
  yseg[w * kTL + t] = y;
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicExch(p.status, kDevTimeout);
      for (int c = 0; c < C; ++c) mbar_wait(smem_u32(&bars[c]), 0u);  // loads land before the CTA exits
    }
    __syncthreads();
    return;
  }
  // 2. the value entering this segment, then y and the backward from 0
  double yin = 0.0;
  for (int v = 0; v < w; ++v) yin = __fma_rn(__ldg(&ag[v].x), yin, yseg[v * kTL + t]);
  double x = 0.0;
  if (!keep) {
    for (int e1 = e_hi - 1; e1 >= e_lo; e1 -= G) {
      const int ng = e1 - e_lo + 1;  // rows e1, e1 - 1, ... down to e_lo
      double2 c[G];
      double v[G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q < ng) {
          c[q] = __ldg(pg + e1 - q);
          v[q] = static_cast<double>(col[static_cast<size_t>(e1 - q) * kTL]);
        }
      }
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q < ng) {
          const double ye = __fma_rn(c[q].x, yin, v[q]);
          x = __fma_rn(c[q].y, x, ye);
          col[static_cast<size_t>(e1 - q) * kTL] = static_cast<T>(x);
        }
      }
    }
  }
  xseg[w * kTL + t] = x;
  __syncthreads();
  // 3. the value entering this segment from the right, then x
  double xin = 0.0;
  for (int v = kPartWarps - 1; v > w; --v) xin = __fma_rn(__ldg(&ag[v].y), xin, xseg[v * kTL + t]);
  if (!keep) {
    for (int e0 = e_lo; e0 < e_hi; e0 += G) {
      const int ng = e_hi - e0;
      double qv[G], v[G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        qv[q] = __ldg(qq + e0 + q);
        v[q] = q < ng ? static_cast<double>(col[static_cast<size_t>(e0 + q) * kTL]) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < G; ++q)
        if (q < ng) col[static_cast<size_t>(e0 + q) * kTL] = static_cast<T>(__fma_rn(qv[q], xin, v[q]));
    }
    // the pin after the sweep restores the two line ends
    if (act) {
      if (e_lo == 0 && e_hi > 0) col[0] = e0v;
      if (e_lo <= n - 1 && n - 1 < e_hi) col[static_cast<size_t>(n - 1) * kTL] = e1v;
    }
  }
  // 4. the tile back to the field (rows and columns past the grid are clipped)
  fence_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int c = 0; c < C; ++c) {
      const uint32_t src = smem_u32(tile + static_cast<size_t>(c) * kRingRows * kTL);
      if (AXIS == 1)
        tma_store_4d(&map, src, i0, c * kRingRows, m, s);
      else
        tma_store_4d(&map, src, i0, m, c * kRingRows, s);
    }
    tma_store_commit();
    tma_store_wait_read();
  }
}

}  // namespace

size_t part_smem_bytes(int eb, int n_line) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  return 128 /* alignment pad */ + kPartHead + static_cast<size_t>(C) * kRingRows * kTL * eb;
}

template <typename T, int AXIS>
cudaError_t launch_part(const CUtensorMap& map, const SweepParams<T>& p, const PartAxis& pa, cudaStream_t st) {
  const int n = AXIS == 1 ? p.ny : p.nz;
  const size_t smem = part_smem_bytes(static_cast<int>(sizeof(T)), n);
  if ((n + kRingRows - 1) / kRingRows > kPartMaxChunks || smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(sweep_part_kernel<T, AXIS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const dim3 grid((p.nx + kTL - 1) / kTL, AXIS == 1 ? p.nz : p.ny, p.s_hi - p.s_lo);
  sweep_part_kernel<T, AXIS><<<grid, 32 * kPartWarps, smem, st>>>(map, p, pa);
  return cudaGetLastError();
}

template cudaError_t launch_part<double, 1>(const CUtensorMap&, const SweepParams<double>&, const PartAxis&,
                                            cudaStream_t);
template cudaError_t launch_part<double, 2>(const CUtensorMap&, const SweepParams<double>&, const PartAxis&,
                                            cudaStream_t);
template cudaError_t launch_part<float, 1>(const CUtensorMap&, const SweepParams<float>&, const PartAxis&,
                                           cudaStream_t);
template cudaError_t launch_part<float, 2>(const CUtensorMap&, const SweepParams<float>&, const PartAxis&,
                                           cudaStream_t);

}  // namespace bfvm
