// bfvm_part_sweeps.cu -- the partitioned sweeps (bfvm_set_fp64_chain(ctx, 2)).
//
// The reference solves each Thomas system with one serial recurrence per
// line (BioFVM/BioFVM_solvers.cpp:352-777): forward y_i = (p_i + c1 y_{i-1})
// / d_i, backward x_i = y_i - c_i x_{i+1}.  A thread per line runs that
// chain element after element, so a sweep's speed is the latency of one
// dependent step times the line length; the lines an SM can hold at once
// (its shared memory) bound how many chains hide each other's latency.
//
// Here the recurrences are the same linear maps, evaluated by a partition
// method.  A CTA stages one tile of 32 lines and runs 8 warps over it; warp w
// owns the segment [w m, (w+1) m) of every line (m = ceil(n/8), rounded to
// whole 16-byte units).  With a_i = c1 RN(1/d_i), b_i = p_i RN(1/d_i) and
// g_i = -c_i (g_{n-1} = 0):
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
// them in extended precision and rounds each once.  Every line's chain is
// now a segment long (25 at n = 200 instead of 200), so a tile finishes in
// a fraction of the time and the sweep is bound by HBM, not by the chain.
//
// The arithmetic is not the reference's operation order: results differ by
// a few units in the last place per sweep (tests hold the FP64 results to
// 1e-12 relative per voxel of the reference, as the FP64 short chain is).
// The FP32 form uses the same kernels with its FP32 storage and FP64
// arithmetic (each value is stored three times per sweep instead of once).
//
// Dirichlet semantics are those of the other sweeps (bfvm_sweeps.cu): the x
// sweep writes a face line's face values and pins the line ends of an
// activated substrate before and after; the y and z sweeps keep the input of
// x-face lines and of whole tiles in an activated face, and restore the two
// line ends (pinned by the sweep before) after the sweep.
#include "bfvm_ctx.h"
#include "bfvm_ptx.cuh"
#include "bfvm_sweep_common.cuh"

namespace bfvm {

namespace {

constexpr int kTL = 32;  // lines per tile (one per lane)
constexpr int kPartMaxBuffers = 3;

// Shared memory of one CTA: barriers [kPartMaxBuffers][kPartMaxChunks], the
// segment ends [2][kPartWarps][32] FP64, then the tile buffers, each
// 1024-byte aligned (the x sweep's 128B swizzle).
constexpr int kBarBytes = kPartMaxBuffers * kPartMaxChunks * 8;
constexpr int kSegBytes = 2 * kPartWarps * kTL * 8;
constexpr int kPartHead = ((kBarBytes + 1023) / 1024) * 1024 + ((kSegBytes + 1023) / 1024) * 1024;

template <typename T>
__device__ __forceinline__ T* x_elem(unsigned char* tile, int e, int t) {
  // element e of line t in the chunked, 128B-swizzled x tile
  constexpr int EW = 128 / static_cast<int>(sizeof(T));  // elements per 128-byte row
  constexpr int U = 16 / static_cast<int>(sizeof(T));    // elements per 16-byte unit
  const int c = e / EW, r = e - c * EW;
  return reinterpret_cast<T*>(tile + static_cast<size_t>(c) * (kTL * 128) + t * 128 + (((r / U) ^ (t & 7)) << 4) +
                              (r % U) * static_cast<int>(sizeof(T)));
}

template <typename T, int AXIS>
struct PartShape {
  static constexpr int CHE = AXIS == 0 ? 128 / static_cast<int>(sizeof(T)) : kRingRows;  // elements per chunk
  static constexpr uint32_t kChunkBytes =
      AXIS == 0 ? kTL * 128u : kRingRows * kTL * static_cast<uint32_t>(sizeof(T));
};

// The tiles of one sweep: (line tile, m, s) with m = k for x and y, j for z.
template <int AXIS>
__device__ __forceinline__ void part_decode(long long tile, int nx, int ny, int nz, int& l0, int& m, int& s) {
  const int ntl = ((AXIS == 0 ? ny : nx) + kTL - 1) / kTL;
  const long long per_s = static_cast<long long>(ntl) * (AXIS == 2 ? ny : nz);
  s = static_cast<int>(tile / per_s);
  const long long r = tile - static_cast<long long>(s) * per_s;
  m = static_cast<int>(r / ntl);
  l0 = static_cast<int>(r - static_cast<long long>(m) * ntl) * kTL;
}

// Issue the TMA loads of a tile's C chunks into `buf`, completing on bars[c].
template <typename T, int AXIS>
__device__ __forceinline__ void part_issue(const CUtensorMap* map, unsigned char* buf, uint64_t* bars, int C, int l0,
                                           int m, int s) {
  using Sh = PartShape<T, AXIS>;
  for (int c = 0; c < C; ++c) {
    const uint32_t bar = smem_u32(&bars[c]);
    mbar_expect_tx(bar, Sh::kChunkBytes);
    const uint32_t dst = smem_u32(buf + static_cast<size_t>(c) * Sh::kChunkBytes);
    if (AXIS == 0)
      tma_load_4d(dst, map, bar, c * Sh::CHE, l0, m, s);
    else if (AXIS == 1)
      tma_load_4d(dst, map, bar, l0, c * Sh::CHE, m, s);
    else
      tma_load_4d(dst, map, bar, l0, m, c * Sh::CHE, s);
  }
}

// Store a finished tile from `buf` (rows or lines past the grid are clipped).
template <typename T, int AXIS>
__device__ __forceinline__ void part_store(const CUtensorMap* map, unsigned char* buf, int C, int l0, int m, int s) {
  using Sh = PartShape<T, AXIS>;
  for (int c = 0; c < C; ++c) {
    const uint32_t src = smem_u32(buf + static_cast<size_t>(c) * Sh::kChunkBytes);
    if (AXIS == 0)
      tma_store_4d(map, src, c * Sh::CHE, l0, m, s);
    else if (AXIS == 1)
      tma_store_4d(map, src, l0, c * Sh::CHE, m, s);
    else
      tma_store_4d(map, src, l0, m, c * Sh::CHE, s);
  }
  tma_store_commit();
}

// The partition method on one staged tile (see the file comment): waits for
// the chunks of this warp's segment (barrier phase `par`), runs the three
// passes in place, and calls after_pass1() between the first two (a point
// every thread reaches after a CTA barrier).  Returns false (status set) if
// a wait gave up.
template <typename T, int AXIS, typename Hook>
__device__ __forceinline__ bool part_tile(unsigned char* tile, uint64_t* bars, uint32_t par,
                                          const SweepParams<T>& p, const PartAxis& pa, int l0, int m, int s,
                                          double* yseg, double* xseg, Hook&& after_pass1) {
  using Sh = PartShape<T, AXIS>;
  const int w = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int nx = p.nx, ny = p.ny, nz = p.nz, S = p.S;
  const int n = AXIS == 0 ? nx : (AXIS == 1 ? ny : nz);
  const bool act = p.active[s] != 0;
  const int mseg = pa.mseg;
  const int e_lo = w * mseg, e_hi = min(n, e_lo + mseg);
  const int C = (n + Sh::CHE - 1) / Sh::CHE;
  bool ok = true;
  for (int c = e_lo / Sh::CHE; c < C && c * Sh::CHE < e_hi; ++c)
    if (ok) ok = mbar_wait(smem_u32(&bars[c]), par);

  const int l = l0 + t;  // this lane's line (j for x, i for y and z)
  const bool valid = l < (AXIS == 0 ? ny : nx);
  bool face;
  if (AXIS == 0)
    face = act && (l == 0 || l == ny - 1 || m == 0 || m == nz - 1);
  else
    face = act && (l == 0 || l == nx - 1);
  // y/z: lanes in an x face, and lanes past nx, keep their input
  const bool keep = AXIS != 0 && (face || !valid);
  const double off = kF32<T> ? p.off[s] : 0.0;
  const double shift = kF32<T> ? p.shift[s] : 0.0;
  auto elem = [&](int e) -> T* {
    if constexpr (AXIS == 0)
      return x_elem<T>(tile, e, t);
    else
      return reinterpret_cast<T*>(tile) + static_cast<size_t>(e) * kTL + t;
  };
  T e0v = T(0), e1v = T(0);  // x: the x-face values; y/z: the line ends' input
  if (ok) {
    if (AXIS == 0) {
      if (act && valid && !face) {
        e0v = static_cast<T>(p.xface[(static_cast<size_t>(0 * S + s) * nz + m) * ny + l] - off);
        e1v = static_cast<T>(p.xface[(static_cast<size_t>(1 * S + s) * nz + m) * ny + l] - off);
        // the pin before the sweep, by the warps that own the two ends
        if (e_lo == 0 && e_hi > 0) *elem(0) = e0v;
        if (e_lo <= n - 1 && n - 1 < e_hi) *elem(n - 1) = e1v;
      }
    } else if (act) {
      if (e_lo == 0 && e_hi > 0) e0v = *elem(0);
      if (e_lo <= n - 1 && n - 1 < e_hi) e1v = *elem(n - 1);
    }
  }
  const double2* __restrict__ ra = pa.ra + static_cast<size_t>(s) * pa.npad;  // {RN(1/d), a}
  const double2* __restrict__ pg = pa.pg + static_cast<size_t>(s) * pa.npad;  // {P, g}
  const double* __restrict__ qq = pa.q + static_cast<size_t>(s) * pa.npad;    // Q
  const double2* __restrict__ ag = pa.ag + static_cast<size_t>(s) * kPartWarps;  // {A_w, G_w}

  // The passes go through a segment in groups of G elements, every load of a
  // group issued before its arithmetic (the coefficient rows are padded past
  // n, so their loads need no bound; the staged values do).
  constexpr int G = 8;
  // 1. forward over the segment from 0, in place
  double y = 0.0;
  if (!keep && ok) {
    for (int e0 = e_lo; e0 < e_hi; e0 += G) {
      const int ng = e_hi - e0;
      double2 c[G];
      double v[G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        c[q] = __ldg(ra + e0 + q);
        v[q] = q < ng ? static_cast<double>(*elem(e0 + q)) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q < ng) {
          y = __fma_rn(c[q].y, y, __dmul_rn(kF32<T> ? v[q] - shift : v[q], c[q].x));
          *elem(e0 + q) = static_cast<T>(y);
        }
      }
    }
  }
  yseg[w * kTL + t] = y;
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(p.status, kDevTimeout);
    return false;
  }
  after_pass1();
  // 2. the value entering this segment, then y and the backward from 0
  double yin = 0.0;
  for (int v = 0; v < w; ++v) yin = __fma_rn(__ldg(&ag[v].x), yin, yseg[v * kTL + t]);
  double x = 0.0;
  if (!keep) {
    for (int e1 = e_hi - 1; e1 >= e_lo; e1 -= G) {
      const int ng = e1 - e_lo + 1;  // elements e1, e1 - 1, ... down to e_lo
      double2 c[G];
      double v[G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q < ng) {
          c[q] = __ldg(pg + e1 - q);
          v[q] = static_cast<double>(*elem(e1 - q));
        }
      }
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q < ng) {
          const double ye = __fma_rn(c[q].x, yin, v[q]);
          x = __fma_rn(c[q].y, x, ye);
          *elem(e1 - q) = static_cast<T>(x);
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
    if (AXIS == 0 && face && valid) {
      // a face line takes the face plane's values
      const double* fv = (m == 0 || m == nz - 1)
                             ? p.zface + ((static_cast<size_t>(m == 0 ? 0 : 1) * S + s) * ny + l) * nx
                             : p.yface + ((static_cast<size_t>(l == 0 ? 0 : 1) * S + s) * nz + m) * nx;
      for (int e = e_lo; e < e_hi; ++e) *elem(e) = static_cast<T>(fv[e] - off);
    } else {
      for (int e0 = e_lo; e0 < e_hi; e0 += G) {
        const int ng = e_hi - e0;
        double qv[G], v[G];
#pragma unroll
        for (int q = 0; q < G; ++q) {
          qv[q] = __ldg(qq + e0 + q);
          v[q] = q < ng ? static_cast<double>(*elem(e0 + q)) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < G; ++q)
          if (q < ng) *elem(e0 + q) = static_cast<T>(__fma_rn(qv[q], xin, v[q]));
      }
      // the pin after the sweep
      if (act && (AXIS != 0 || valid)) {
        if (e_lo == 0 && e_hi > 0) *elem(0) = e0v;
        if (e_lo <= n - 1 && n - 1 < e_hi) *elem(n - 1) = e1v;
      }
    }
  }
  fence_async_smem();  // the results are read by the bulk store next
  __syncthreads();
  return true;
}

// One CTA per tile (tiles too large for two buffers).
template <typename T, int AXIS>
__global__ void __launch_bounds__(32 * kPartWarps) sweep_part_kernel(const __grid_constant__ CUtensorMap map,
                                                                     const SweepParams<T> p, const PartAxis pa) {
  using Sh = PartShape<T, AXIS>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  double* yseg = reinterpret_cast<double*>(base + ((kBarBytes + 1023) / 1024) * 1024);
  double* xseg = yseg + kPartWarps * kTL;
  unsigned char* tile = base + kPartHead;
  const int n = AXIS == 0 ? p.nx : (AXIS == 1 ? p.ny : p.nz);
  const int C = (n + Sh::CHE - 1) / Sh::CHE;
  const int s = blockIdx.z;
  const int l0 = blockIdx.x * kTL, m = blockIdx.y;
  if (AXIS != 0 && p.active[s] != 0 && (m == 0 || m == (AXIS == 1 ? p.nz : p.ny) - 1)) return;  // final already
  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(&bars[c]), 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) part_issue<T, AXIS>(&map, tile, bars, C, l0, m, s);
  const bool ok = part_tile<T, AXIS>(tile, bars, 0u, p, pa, l0, m, s, yseg, xseg, [] {});
  if (threadIdx.x == 0) {
    if (ok) part_store<T, AXIS>(&map, tile, C, l0, m, s);
    else
      for (int c = 0; c < C; ++c) mbar_wait(smem_u32(&bars[c]), 0u);  // loads land before the CTA exits
    tma_store_wait_read();
  }
}

// Persistent: a CTA takes tiles blockIdx.x, + gridDim.x, ... (face tiles of
// the y and z sweeps skipped) through NB tile buffers, tile k in buffer
// k % NB.  Tile k + NB loads into the buffer of tile k once tile k's store
// has read it -- issued during tile k + 1, after its first pass -- so each
// load has the better part of NB - 1 tiles' work to land.
template <typename T, int AXIS>
__global__ void __launch_bounds__(32 * kPartWarps, 2) sweep_part_pers_kernel(const __grid_constant__ CUtensorMap map,
                                                                          const SweepParams<T> p, const PartAxis pa,
                                                                          long long ntiles, int NB,
                                                                          uint32_t buf_bytes) {
  using Sh = PartShape<T, AXIS>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);  // [NB][kPartMaxChunks]
  double* yseg = reinterpret_cast<double*>(base + ((kBarBytes + 1023) / 1024) * 1024);
  double* xseg = yseg + kPartWarps * kTL;
  unsigned char* bufs = base + kPartHead;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int n = AXIS == 0 ? nx : (AXIS == 1 ? ny : nz);
  const int nm = AXIS == 2 ? ny : nz;
  const int C = (n + Sh::CHE - 1) / Sh::CHE;
  auto skip = [&](long long tile) {
    if (AXIS == 0) return false;
    int l0, m, s;
    part_decode<AXIS>(tile, nx, ny, nz, l0, m, s);
    return p.active[s] != 0 && (m == 0 || m == nm - 1);
  };
  auto next = [&](long long tile) {
    do {
      tile += gridDim.x;
    } while (tile < ntiles && skip(tile));
    return tile;
  };
  auto issue = [&](long long tile, int b) {
    int l0, m, s;
    part_decode<AXIS>(tile, nx, ny, nz, l0, m, s);
    part_issue<T, AXIS>(&map, bufs + static_cast<size_t>(b) * buf_bytes, bars + b * kPartMaxChunks, C, l0, m, s);
  };
  if (threadIdx.x == 0) {
    prefetch_tmap(&map);
    for (int q = 0; q < NB * kPartMaxChunks; ++q) mbar_init(smem_u32(&bars[q]), 1);
    fence_barrier_init();
  }
  __syncthreads();
  // the first NB tiles of this CTA
  long long seq[kPartMaxBuffers];
  seq[0] = next(static_cast<long long>(blockIdx.x) - gridDim.x);
  for (int b = 1; b < NB; ++b) seq[b] = seq[b - 1] < ntiles ? next(seq[b - 1]) : ntiles;
  int iss[kPartMaxBuffers] = {0, 0, 0};  // loads issued into each buffer (thread 0)
  if (threadIdx.x == 0)
    for (int b = 0; b < NB; ++b)
      if (seq[b] < ntiles) {
        issue(seq[b], b);
        ++iss[b];
      }
  long long cur = seq[0];
  long long last_issued = seq[NB - 1];  // the newest tile issued (or ntiles)
  long long refill = -1;                // tile to load into the buffer of the previous tile
  int prev_buf = -1;
  bool ok = true;
  for (long long k = 0; cur < ntiles && ok; ++k) {
    const int b = static_cast<int>(k % NB);
    const uint32_t par = static_cast<uint32_t>((k / NB) & 1);
    int l0, m, s;
    part_decode<AXIS>(cur, nx, ny, nz, l0, m, s);
    unsigned char* tile = bufs + static_cast<size_t>(b) * buf_bytes;
    const long long rf = refill;
    const int pb = prev_buf;
    ok = part_tile<T, AXIS>(tile, bars + b * kPartMaxChunks, par, p, pa, l0, m, s, yseg, xseg, [&] {
      if (rf >= 0 && threadIdx.x == 0) {
        tma_store_wait_read();  // the previous tile's store has read its buffer
        issue(rf, pb);
        ++iss[pb];
      }
    });
    if (!ok) break;
    if (threadIdx.x == 0) part_store<T, AXIS>(&map, tile, C, l0, m, s);
    // the tile after the newest one issued goes into this buffer, next round
    refill = last_issued < ntiles ? next(last_issued) : ntiles;
    if (refill >= ntiles) refill = -1;
    else last_issued = refill;
    prev_buf = b;
    cur = next(cur);
  }
  if (threadIdx.x == 0) {
    tma_store_wait_read();
    if (!ok) {
      // a wait gave up: every buffer's newest loads land (each wait bounded) before the CTA exits
      for (int b = 0; b < NB; ++b)
        if (iss[b] > 0)
          for (int c = 0; c < C; ++c)
            mbar_wait(smem_u32(&bars[b * kPartMaxChunks + c]), static_cast<uint32_t>((iss[b] - 1) & 1));
    }
  }
}

}  // namespace

static size_t part_buf_bytes(int eb, int n_line, int axis) {
  const int che = axis == 0 ? 128 / eb : kRingRows;
  const int C = (n_line + che - 1) / che;
  const size_t chunk = axis == 0 ? static_cast<size_t>(kTL) * 128 : static_cast<size_t>(kRingRows) * kTL * eb;
  return (static_cast<size_t>(C) * chunk + 1023) / 1024 * 1024;
}

size_t part_smem_bytes(int eb, int n_line, int axis) {
  return 1024 /* alignment pad */ + kPartHead + part_buf_bytes(eb, n_line, axis);
}

template <typename T, int AXIS>
cudaError_t launch_part(const CUtensorMap& map, const SweepParams<T>& p, const PartAxis& pa, cudaStream_t st) {
  constexpr int eb = static_cast<int>(sizeof(T));
  const int n = AXIS == 0 ? p.nx : (AXIS == 1 ? p.ny : p.nz);
  const int che = AXIS == 0 ? 128 / eb : kRingRows;
  if ((n + che - 1) / che > kPartMaxChunks) return cudaErrorInvalidValue;
  const size_t buf = part_buf_bytes(eb, n, AXIS);
  const size_t lim = 227 * 1024;
  // buffers per CTA: the most tile buffers per SM over the CTAs that fit
  // (ties to more CTAs); one buffer means a CTA per tile
  int NB = 0, best = 0;
  for (int b = 2; b <= kPartMaxBuffers; ++b) {
    const size_t smem_b = 1024 + kPartHead + b * buf;
    if (smem_b > lim) break;
    const int ctas = static_cast<int>((228 * 1024) / (smem_b + 1024));
    if (ctas * b > best) {
      best = ctas * b;
      NB = b;
    }
  }
  const int lines = AXIS == 0 ? p.ny : p.nx;
  const int ntl = (lines + kTL - 1) / kTL;
  if (NB >= 2) {
    const size_t smem = 1024 + kPartHead + NB * buf;
    const long long ntiles = static_cast<long long>(ntl) * (AXIS == 2 ? p.ny : p.nz) * p.S;
    int grid = 0;
    cudaError_t e = persistent_grid(sweep_part_pers_kernel<T, AXIS>, smem, ntiles, &grid, 32 * kPartWarps);
    if (e != cudaSuccess) return e;
    sweep_part_pers_kernel<T, AXIS><<<grid, 32 * kPartWarps, smem, st>>>(map, p, pa, ntiles, NB,
                                                                         static_cast<uint32_t>(buf));
    return cudaGetLastError();
  }
  const size_t smem = part_smem_bytes(eb, n, AXIS);
  if (smem > lim) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(sweep_part_kernel<T, AXIS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const dim3 grid(ntl, AXIS == 2 ? p.ny : p.nz, p.S);
  sweep_part_kernel<T, AXIS><<<grid, 32 * kPartWarps, smem, st>>>(map, p, pa);
  return cudaGetLastError();
}

template cudaError_t launch_part<double, 0>(const CUtensorMap&, const SweepParams<double>&, const PartAxis&,
                                            cudaStream_t);
template cudaError_t launch_part<double, 1>(const CUtensorMap&, const SweepParams<double>&, const PartAxis&,
                                            cudaStream_t);
template cudaError_t launch_part<double, 2>(const CUtensorMap&, const SweepParams<double>&, const PartAxis&,
                                            cudaStream_t);
template cudaError_t launch_part<float, 0>(const CUtensorMap&, const SweepParams<float>&, const PartAxis&,
                                           cudaStream_t);
template cudaError_t launch_part<float, 1>(const CUtensorMap&, const SweepParams<float>&, const PartAxis&,
                                           cudaStream_t);
template cudaError_t launch_part<float, 2>(const CUtensorMap&, const SweepParams<float>&, const PartAxis&,
                                           cudaStream_t);

}  // namespace bfvm
