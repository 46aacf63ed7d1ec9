// bfvm_sweep_common.cuh -- device helpers shared by the sweep kernels
// (bfvm_sweeps.cu: per-tile, persistent ring and batched sweeps;
// bfvm_tmem_sweeps.cu: the persistent sweeps with tensor-memory rings) and
// the persistent-grid sizing of their launches.
//
// The recurrence helpers follow the reference's arithmetic operation by
// operation (BioFVM/BioFVM_solvers.cpp:352-777): forward y_i = fma(c1,
// y_{i-1}, p_i) / d_i with the quotient from Markstein's correction of
// RN(1/d_i), backward x_i = fma(-c_i, x_{i+1}, y_i).
#pragma once

#include <climits>
#include <type_traits>

#include "bfvm_internal.h"
#include "bfvm_ptx.cuh"

namespace bfvm {

template <typename T>
constexpr bool kF32 = sizeof(T) == 4;

// Most rings (compute warp + copy warp pairs) in one persistent y/z CTA: the
// register file holds 4 FP64 or 8 FP32 pairs.
template <typename T>
constexpr int kMaxRings = kF32<T> ? 8 : 4;

// Chunks per line are bounded so one 64-bit word holds every barrier's phase.
constexpr int kMaxChunks = 64;
constexpr int kBarrierBytes = 1024;  // kMaxChunks barriers, padded to keep the tile 1024-byte aligned
template <typename T>
constexpr int kChunkX = 128 / static_cast<int>(sizeof(T));  // x-sweep chunk width (one 128-byte row)

__device__ __forceinline__ uint64_t chunk_mask(int C) { return C >= 64 ? ~0ull : ((1ull << C) - 1ull); }

// SweepParams::screen values: 0 no input screen (every numerator checked),
// 1 the exactness screen of the reference-exact chain, kScreenFast the
// short FP64 chain (bfvm_set_fp64_chain), which needs no screen.
constexpr int kScreenFast = 2;

// The short FP64 forward chain: with cf = {a = RN(c1 * r), r = RN(1/d)},
// y_i = fma(a_i, y_{i-1}, v_i * r_i) -- one dependent FMA per element
// instead of the reference's fma and correctly rounded division.  Not the
// reference's bits: within a few units in the last place per sweep.
template <int B, typename Put>
__device__ __forceinline__ double forward_fast(const double (&v)[B], const double2 (&cf)[B], double y, Put&& put) {
#pragma unroll
  for (int q = 0; q < B; ++q) {
    y = __fma_rn(cf[q].x, y, __dmul_rn(v[q], cf[q].y));
    put(q, y);
  }
  return y;
}

// Forward recurrence over B staged values; out[q] receives y_q and the
// running value is returned.
__device__ __forceinline__ double markstein(double t, double d, double r) {
  const double q0 = t * r;
  const double e = __fma_rn(-q0, d, t);
  return __fma_rn(e, r, q0);
}

// FP64 forward batch.  The bare chain runs first and hands each result to
// put(q, y) as soon as it is computed, so the stores overlap the chain.  With
// c1 >= 0 and every denominator >= 1 (screen set: no negative diffusion or
// decay), a batch whose incoming value is not negative and whose inputs are
// all >= 2^-960 has every numerator t = fma(c1, y, v) >= 2^-960, where the
// Markstein quotient is exact.  That screen reads only the inputs (a signed
// minimum of their high words, which orders non-negative doubles and puts
// negative ones first), so it runs off the chain; a batch that fails it
// anywhere in the warp is redone from its inputs (still in registers) with
// each numerator checked, and with IEEE division if one is -0 or a nonzero
// value below 2^-960, and its results are stored again over the bare ones.
template <int B, typename Put>
__device__ __forceinline__ double forward_store(const double (&v)[B], const double2 (&cf)[B], double c1, double,
                                                int screen, double y, Put&& put) {
  if (screen == kScreenFast) return forward_fast<B>(v, cf, y, put);
  const double y0 = y;
#pragma unroll
  for (int q = 0; q < B; ++q) {
    y = markstein(__fma_rn(c1, y, v[q]), cf[q].x, cf[q].y);
    put(q, y);
  }
  int hw[B];
#pragma unroll
  for (int q = 0; q < B; ++q) hw[q] = __double2hiint(v[q]);
#pragma unroll
  for (int w = B / 2; w >= 1; w /= 2) {
#pragma unroll
    for (int q = 0; q < w; ++q) hw[q] = min(hw[q], hw[q + w]);
  }
  constexpr int kHiTiny = 0x03F00000;  // high word of 2^-960
  const bool clean = screen != 0 && !(y0 < 0.0) && hw[0] >= kHiTiny;  // -0 (a line's start) passes
  if (!__all_sync(__activemask(), clean)) {
    bool slow = false;
    y = y0;
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const double t = __fma_rn(c1, y, v[q]);
      slow |= (fabs(t) < 0x1p-960) & (__double_as_longlong(t) != 0);
      y = markstein(t, cf[q].x, cf[q].y);
      put(q, y);
    }
    if (slow) {
      y = y0;
#pragma unroll
      for (int q = 0; q < B; ++q) {
        y = __fma_rn(c1, y, v[q]) / cf[q].x;
        put(q, y);
      }
    }
  }
  return y;
}

// FP32 form: stored values are FP32, the recurrence runs in FP64 (the
// running value y stays FP64 across elements and batches), each result is
// rounded to FP32 once, when stored.  The quotient is t * RN(1/d); under the
// short chain (screen == kScreenFast) y = fma(c1 * r, y, (v - shift) * r),
// one dependent FMA per element, the products formed off the chain.
template <int B, typename Put>
__device__ __forceinline__ double forward_store(const float (&v)[B], const double (&cf)[B], double c1, double shift,
                                                int screen, double y, Put&& put) {
  if (screen == kScreenFast) {
#pragma unroll
    for (int q = 0; q < B; ++q) {
      y = __fma_rn(__dmul_rn(c1, cf[q]), y, __dmul_rn(static_cast<double>(v[q]) - shift, cf[q]));
      put(q, static_cast<float>(y));
    }
    return y;
  }
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const double t = __fma_rn(c1, y, static_cast<double>(v[q]) - shift);
    y = __dmul_rn(t, cf[q]);
    put(q, static_cast<float>(y));
  }
  return y;
}

// Bare FP64 forward chain over one batch (no screen); results go to put as
// they are computed.  The caller screens the inputs (batch_min_hi) and redoes
// the batch, or the whole line, with forward_checked if the screen fails.
template <int B, typename Put>
__device__ __forceinline__ double forward_bare(const double (&v)[B], const double2 (&cf)[B], double c1, double y,
                                               Put&& put) {
#pragma unroll
  for (int q = 0; q < B; ++q) {
    y = markstein(__fma_rn(c1, y, v[q]), cf[q].x, cf[q].y);
    put(q, y);
  }
  return y;
}

// The bare chain of the screen's mode: the short chain when screen is
// kScreenFast, else the reference-exact one (forward_bare).
template <int B, typename Put>
__device__ __forceinline__ double forward_any(int screen, const double (&v)[B], const double2 (&cf)[B], double c1,
                                              double y, Put&& put) {
  if (screen == kScreenFast) return forward_fast<B>(v, cf, y, put);
  return forward_bare<B>(v, cf, c1, y, put);
}

// The bare chain of the screen's mode over a batch whose coefficients are
// all one pair cf (the converged part of a factorized row): the same
// operations as forward_any with cf in every position.
template <int B, typename Put>
__device__ __forceinline__ double forward_any_const(int screen, const double (&v)[B], double2 cf, double c1,
                                                    double y, Put&& put) {
  if (screen == kScreenFast) {
#pragma unroll
    for (int q = 0; q < B; ++q) {
      y = __fma_rn(cf.x, y, __dmul_rn(v[q], cf.y));
      put(q, y);
    }
    return y;
  }
#pragma unroll
  for (int q = 0; q < B; ++q) {
    y = markstein(__fma_rn(c1, y, v[q]), cf.x, cf.y);
    put(q, y);
  }
  return y;
}

// Whether a tile whose inputs' minimum high word is hwmin needs no redo:
// always under the short chain, else when the screen passed.
__device__ __forceinline__ bool screen_clean(int screen, int hwmin);

// The batch's inputs' minimum high word (signed): >= the high word of 2^-960
// exactly when every input is >= 2^-960 (negative inputs sort first).
template <int B>
__device__ __forceinline__ int batch_min_hi(const double (&v)[B]) {
  int hw[B];
#pragma unroll
  for (int q = 0; q < B; ++q) hw[q] = __double2hiint(v[q]);
#pragma unroll
  for (int w = B / 2; w >= 1; w /= 2) {
#pragma unroll
    for (int q = 0; q < w; ++q) hw[q] = min(hw[q], hw[q + w]);
  }
  return hw[0];
}
constexpr int kHiTiny = 0x03F00000;  // high word of 2^-960

__device__ __forceinline__ bool screen_clean(int screen, int hwmin) {
  return screen == kScreenFast || (screen != 0 && hwmin >= kHiTiny);
}

// The forward chain with every numerator checked: the Markstein quotient
// where it is exact, IEEE division for a numerator of -0 or a nonzero value
// below 2^-960 (the whole batch, as the reference divides).
template <int B, typename Put>
__device__ __forceinline__ double forward_checked(const double (&v)[B], const double2 (&cf)[B], double c1, double y,
                                                  Put&& put) {
  const double y0 = y;
  bool slow = false;
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const double t = __fma_rn(c1, y, v[q]);
    slow |= (fabs(t) < 0x1p-960) & (__double_as_longlong(t) != 0);
    y = markstein(t, cf[q].x, cf[q].y);
    put(q, y);
  }
  if (slow) {
    y = y0;
#pragma unroll
    for (int q = 0; q < B; ++q) {
      y = __fma_rn(c1, y, v[q]) / cf[q].x;
      put(q, y);
    }
  }
  return y;
}

// Writer of one thread's 128-byte row of a swizzled chunk, element by
// element in order: values are gathered into 16-byte units and each unit is
// stored when complete.
template <typename T>
struct RowPut {
  static constexpr int U = 16 / sizeof(T);
  using Unit = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
  unsigned char* crow;
  int sw;
  T buf[U];
  template <typename V>
  __device__ __forceinline__ void operator()(int q, V val) {
    buf[q % U] = static_cast<T>(val);
    if (q % U == U - 1) {
      Unit uv;
      T* ev = reinterpret_cast<T*>(&uv);
#pragma unroll
      for (int e = 0; e < U; ++e) ev[e] = buf[e];
      *reinterpret_cast<Unit*>(crow + (((q / U) ^ sw) << 4)) = uv;
    }
  }
};

__device__ __forceinline__ double back_elem(double c, double xn, double y) { return __fma_rn(-c, xn, y); }

// Apply the run of agents that starts at sorted position q (key `key`,
// constants c1/c2/e2 of that first agent already loaded) to the staged value
// at *e of substrate s, in sorted order -- which is agent-list order within a
// voxel -- with the reference's three operations per agent, in FP64.
template <typename T>
__device__ __forceinline__ void apply_run(T* e, int q, unsigned key, double c1, double c2, double e2, int qend,
                                          const unsigned* __restrict__ a_key, const double* __restrict__ ac1,
                                          const double* __restrict__ ac2, const double* __restrict__ ae2,
                                          double off, int s, const AgentTrack& tr) {
  double r = static_cast<double>(*e);
  if constexpr (kF32<T>) r += off;
  r = agent_update(r, c1, c2, e2, q, s, tr);
  for (int q2 = q + 1; q2 < qend && __ldg(a_key + q2) == key; ++q2)
    r = agent_update(r, __ldg(ac1 + q2), __ldg(ac2 + q2), __ldg(ae2 + q2), q2, s, tr);
  if constexpr (kF32<T>) r -= off;
  *e = static_cast<T>(r);
}

// Element e (0..W-1) of a thread's 128-byte row in a chunk staged with the
// 128B swizzle: 16-byte unit (e/U) is stored at unit (e/U) ^ (row%8).
template <typename T>
__device__ __forceinline__ T* swz_elem(unsigned char* row, int e, int sw) {
  constexpr int U = 16 / sizeof(T);
  return reinterpret_cast<T*>(row + (((e / U) ^ sw) << 4) + (e % U) * sizeof(T));
}

template <typename T, int W>
__device__ __forceinline__ void load_row(const unsigned char* crow, int sw, T (&v)[W]) {
  constexpr int U = 16 / sizeof(T);
  using Unit = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
#pragma unroll
  for (int u = 0; u < W / U; ++u) {
    const Unit uv = *reinterpret_cast<const Unit*>(crow + ((u ^ sw) << 4));
    const T* ev = reinterpret_cast<const T*>(&uv);
#pragma unroll
    for (int q = 0; q < U; ++q) v[u * U + q] = ev[q];
  }
}

template <typename T, int W>
__device__ __forceinline__ void store_row(unsigned char* crow, int sw, const T (&v)[W]) {
  constexpr int U = 16 / sizeof(T);
  using Unit = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
#pragma unroll
  for (int u = 0; u < W / U; ++u) {
    Unit uv;
    T* ev = reinterpret_cast<T*>(&uv);
#pragma unroll
    for (int q = 0; q < U; ++q) ev[q] = v[u * U + q];
    *reinterpret_cast<Unit*>(crow + ((u ^ sw) << 4)) = uv;
  }
}

// Copy m coefficients to shared memory with the CTA's threads, every
// thread's loads in flight together (eight per thread per round).
__device__ __forceinline__ void stage_row_cta(double* __restrict__ dst, const double* __restrict__ src, int m) {
  const int t = threadIdx.x, nt = blockDim.x;
  for (int q0 = 0; q0 < m; q0 += 8 * nt) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = q0 + u * nt + t;
      v[u] = q < m ? __ldg(src + q) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = q0 + u * nt + t;
      if (q < m) dst[q] = v[u];
    }
  }
}

// Offset that aligns the dynamic shared-memory window to `align` bytes
// (pointers are formed as smem_raw + offset so they stay in the shared space).
__device__ __forceinline__ uint32_t smem_align_pad(const void* smem_raw, uint32_t align) {
  const uint32_t a = smem_u32(smem_raw);
  return ((a + align - 1) & ~(align - 1)) - a;
}

// rows staged in registers per batch of the recurrence
constexpr int kRowBatch = 16;

// Slot of chunk c in a ring whose slot order flips from tile to tile (the
// k-th tile keeps chunk c in slot c for even k and in slot C-1-c for odd k).
__device__ __forceinline__ int ring_slot(bool flip, int C, int c) { return flip ? C - 1 - c : c; }

// Copy m coefficients to shared memory with every lane's loads in flight
// together (eight per lane per round).
__device__ __forceinline__ void stage_row(double* __restrict__ dst, const double* __restrict__ src, int m) {
  const int t = threadIdx.x & 31;
  for (int q0 = 0; q0 < m; q0 += 8 * 32) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = q0 + u * 32 + t;
      v[u] = q < m ? __ldg(src + q) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = q0 + u * 32 + t;
      if (q < m) dst[q] = v[u];
    }
  }
}

// Grid of a persistent launch: every CTA that fits on the device at once
// (at most one per tile).  The kernel's dynamic shared-memory limit is raised
// to the maximum once per device, and its occupancy looked up once per
// shared-memory size (a few entries per thread, replaced round robin).
template <typename K>
static cudaError_t persistent_grid(K kernel, size_t smem, long long tiles, int* grid, int threads = 64) {
  struct Entry {
    const void* k;
    size_t smem;
    int dev, blocks;
  };
  constexpr int kEntries = 16;
  static thread_local Entry cache[kEntries] = {};
  static thread_local int victim = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const void* kp = reinterpret_cast<const void*>(kernel);
  int blocks = -1;
  bool attr_set = false;
  for (const Entry& en : cache) {
    if (en.k == kp && en.dev == dev) {
      attr_set = true;
      if (en.smem == smem) blocks = en.blocks;
    }
  }
  if (blocks < 0) {
    if (!attr_set) {
      e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      if (e != cudaSuccess) return e;
    }
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    blocks = per_sm * sms;
    cache[victim] = Entry{kp, smem, dev, blocks};
    victim = (victim + 1) % kEntries;
  }
  if (blocks < 1) return cudaErrorInvalidConfiguration;
  *grid = static_cast<int>(tiles < blocks ? tiles : blocks);
  return cudaSuccess;
}

}  // namespace bfvm
