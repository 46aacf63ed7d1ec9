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
// dependent FP64 chain.  Every load a step needs (its staged value and its
// coefficients) is therefore issued for a whole batch of elements before the
// chain over that batch starts; the chain itself only touches registers.
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
// with the quotient by d_i computed exactly (div_exact, Markstein's
// correction from a precomputed RN(1/d_i)), so results equal the reference's
// bit for bit.  The FP32 form multiplies by RN32(1/d_i) and keeps the agent
// update in FP64.
#include <climits>
#include <type_traits>

#include "bfvm_internal.h"
#include "bfvm_ptx.cuh"

namespace bfvm {

namespace {

template <typename T>
struct Arith;

template <>
struct Arith<double> {
  // t_i = p_i + c1*y_{i-1}, contracted as the reference's g++ build does
  static __device__ __forceinline__ double lin(double c1, double, double yprev, double v) {
    return __fma_rn(c1, yprev, v);
  }
  static __device__ __forceinline__ double div(double t, double d, double r, double) { return div_exact(t, d, r); }
  static __device__ __forceinline__ double back(double c, double, double xnext, double y) {
    return __fma_rn(-c, xnext, y);
  }
};

// FP32: every fixed coefficient is a (hi, lo) float pair; the low part is
// applied first so the pair acts as one coefficient of ~48 bits.
template <>
struct Arith<float> {
  static __device__ __forceinline__ float lin(float c1h, float c1l, float yprev, float v) {
    return __fmaf_rn(c1h, yprev, __fmaf_rn(c1l, yprev, v));
  }
  static __device__ __forceinline__ float div(float t, double, float rh, float rl) {
    return __fmaf_rn(t, rh, __fmul_rn(t, rl));
  }
  static __device__ __forceinline__ float back(float ch, float cl, float xnext, float y) {
    return __fmaf_rn(-ch, xnext, __fmaf_rn(-cl, xnext, y));
  }
};

template <typename T>
constexpr bool kF32 = sizeof(T) == 4;

// Apply every agent of voxel i (agents of this line are sorted by x index,
// then by agent index) to the value v, in FP64, and return the result.
template <typename T>
__device__ __forceinline__ T apply_agents(T v, int i, int& a, int aend, int& next_i, const int* __restrict__ a_i,
                                          const double* __restrict__ c1, const double* __restrict__ c2,
                                          const double* __restrict__ e2, double off) {
  double r = static_cast<double>(v);
  if constexpr (kF32<T>) r += off;
  do {
    r += c1[a];
    r /= c2[a];
    r += e2[a];
    ++a;
    next_i = (a < aend) ? __ldg(a_i + a) : INT_MAX;
  } while (next_i == i);
  if constexpr (kF32<T>) r -= off;
  return static_cast<T>(r);
}

// Address of element e (0..W-1) of a thread's 128-byte row in a chunk staged
// with the 128B swizzle: 16-byte unit (e/U) is stored at unit (e/U) ^ (row%8).
template <typename T>
__device__ __forceinline__ T* swz_elem(unsigned char* row, int e, int sw) {
  constexpr int U = 16 / sizeof(T);
  return reinterpret_cast<T*>(row + (((e / U) ^ sw) << 4) + (e % U) * sizeof(T));
}

}  // namespace

// ---------------------------------------------------------------------------
// x sweep
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) sweep_x_kernel(const __grid_constant__ CUtensorMap map, const SweepParams<T> p) {
  constexpr int W = 128 / sizeof(T);  // elements per 128-byte row (one TMA box width)
  constexpr int U = 16 / sizeof(T);   // elements per 16-byte unit
  using Unit = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
  extern __shared__ unsigned char smem_raw[];

  const int TL = blockDim.x;
  const int nx = p.nx, ny = p.ny, nz = p.nz, S = p.S;
  const int C = (nx + W - 1) / W;
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  unsigned char* tile = reinterpret_cast<unsigned char*>(base + ((C * 8 + 1023) & ~1023));
  const uint32_t chunk_bytes = static_cast<uint32_t>(TL) * 128u;

  const int t = threadIdx.x;
  const int j0 = blockIdx.x * TL, k = blockIdx.y, s = blockIdx.z;

  if (t == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(&bars[c]), 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (t == 0) {
    for (int c = 0; c < C; ++c) {
      const uint32_t bar = smem_u32(&bars[c]);
      mbar_expect_tx(bar, chunk_bytes);
      tma_load_4d(smem_u32(tile + static_cast<size_t>(c) * chunk_bytes), &map, bar, c * W, j0, k, s);
    }
  }

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
  int a = 0, aend = 0, next_i = INT_MAX;
  const double *ac1 = nullptr, *ac2 = nullptr, *ae2 = nullptr;
  if (p.line_off != nullptr && valid && !face) {
    const int line = k * ny + j;
    a = __ldg(p.line_off + line);
    aend = __ldg(p.line_off + line + 1);
    next_i = (a < aend) ? __ldg(p.a_i + a) : INT_MAX;
    ac1 = p.ac1 + static_cast<size_t>(s) * p.n_sorted;
    ac2 = p.ac2 + static_cast<size_t>(s) * p.n_sorted;
    ae2 = p.ae2 + static_cast<size_t>(s) * p.n_sorted;
  }
  const double* __restrict__ dn = p.ax.denom + static_cast<size_t>(s) * nx;
  const T* __restrict__ rc = p.ax.rcp + static_cast<size_t>(s) * nx;
  const T* __restrict__ cu = p.ax.cup + static_cast<size_t>(s) * nx;
  const T* __restrict__ rcl = kF32<T> ? p.ax.rcp_lo + static_cast<size_t>(s) * nx : nullptr;
  const T* __restrict__ cul = kF32<T> ? p.ax.cup_lo + static_cast<size_t>(s) * nx : nullptr;
  const T c1 = p.c1[s];
  const T c1l = kF32<T> ? p.c1_lo[s] : T(0);
  const T shift = kF32<T> ? p.shift[s] : T(0);

  unsigned char* row = tile + static_cast<size_t>(t) * 128;
  const int sw = t & 7;
  bool ok = true;

  // Forward elimination, one chunk at a time as the TMA boxes land.
  T yprev = T(0);
  for (int c = 0; c < C; ++c) {
    if (ok) ok = mbar_wait(smem_u32(&bars[c]), 0);
    if (face) continue;
    unsigned char* crow = row + static_cast<size_t>(c) * chunk_bytes;
    const int i0 = c * W;
    const int iend = min(nx, i0 + W);
    // Sources, then the pin before the sweep, on the staged row.
    while (next_i < iend) {
      T* e = swz_elem<T>(crow, next_i - i0, sw);
      *e = apply_agents<T>(*e, next_i, a, aend, next_i, p.a_i, ac1, ac2, ae2, off);
    }
    if (act) {
      if (i0 == 0) *swz_elem<T>(crow, 0, sw) = x0v;
      if (nx - 1 < iend) *swz_elem<T>(crow, nx - 1 - i0, sw) = x1v;
    }
    T v[W];
    double d[W];
    T r[W], rl[W];
#pragma unroll
    for (int u = 0; u < W / U; ++u) {
      const Unit uv = *reinterpret_cast<const Unit*>(crow + ((u ^ sw) << 4));
      const T* ev = reinterpret_cast<const T*>(&uv);
#pragma unroll
      for (int q = 0; q < U; ++q) v[u * U + q] = ev[q];
    }
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const int i = min(i0 + q, nx - 1);
      r[q] = __ldg(rc + i);
      if constexpr (kF32<T>) {
        rl[q] = __ldg(rcl + i);
        d[q] = 0.0;
      } else {
        d[q] = __ldg(dn + i);
        rl[q] = T(0);
      }
    }
#pragma unroll
    for (int q = 0; q < W; ++q) {
      const int i = i0 + q;
      if (i < nx) {
        const T vq = kF32<T> ? v[q] - shift : v[q];
        const T tt = (i == 0) ? vq : Arith<T>::lin(c1, c1l, yprev, vq);
        const T y = Arith<T>::div(tt, d[q], r[q], rl[q]);
        v[q] = y;
        yprev = y;
      }
    }
#pragma unroll
    for (int u = 0; u < W / U; ++u) {
      Unit uv;
      T* ev = reinterpret_cast<T*>(&uv);
#pragma unroll
      for (int q = 0; q < U; ++q) ev[q] = v[u * U + q];
      *reinterpret_cast<Unit*>(crow + ((u ^ sw) << 4)) = uv;
    }
  }
  if (__syncthreads_or(!ok)) {
    if (t == 0) atomicExch(p.status, kDevTimeout);
    return;
  }

  // Back substitution, last chunk first; each finished chunk is stored at once.
  T xnext = T(0);
  for (int c = C - 1; c >= 0; --c) {
    unsigned char* crow = row + static_cast<size_t>(c) * chunk_bytes;
    const int i0 = c * W;
    if (face) {
      for (int q = 0; q < W; ++q)
        if (i0 + q < nx) *swz_elem<T>(crow, q, sw) = static_cast<T>(fv != nullptr ? fv[i0 + q] - off : 0.0);
    } else {
      T v[W];
      T cw[W], cwl[W];
#pragma unroll
      for (int u = 0; u < W / U; ++u) {
        const Unit uv = *reinterpret_cast<const Unit*>(crow + ((u ^ sw) << 4));
        const T* ev = reinterpret_cast<const T*>(&uv);
#pragma unroll
        for (int q = 0; q < U; ++q) v[u * U + q] = ev[q];
      }
#pragma unroll
      for (int q = 0; q < W; ++q) {
        const int i = min(i0 + q, nx - 1);
        cw[q] = __ldg(cu + i);
        cwl[q] = kF32<T> ? __ldg(cul + i) : T(0);
      }
#pragma unroll
      for (int q = W - 1; q >= 0; --q) {
        const int i = i0 + q;
        if (i < nx) {
          const T x = (i == nx - 1) ? v[q] : Arith<T>::back(cw[q], cwl[q], xnext, v[q]);
          xnext = x;
          v[q] = x;
        }
      }
#pragma unroll
      for (int u = 0; u < W / U; ++u) {
        Unit uv;
        T* ev = reinterpret_cast<T*>(&uv);
#pragma unroll
        for (int q = 0; q < U; ++q) ev[q] = v[u * U + q];
        *reinterpret_cast<Unit*>(crow + ((u ^ sw) << 4)) = uv;
      }
      if (act) {
        if (i0 == 0) *swz_elem<T>(crow, 0, sw) = x0v;
        if (nx - 1 < i0 + W) *swz_elem<T>(crow, nx - 1 - i0, sw) = x1v;
      }
    }
    fence_async_smem();
    __syncthreads();
    if (t == 0) {
      tma_store_4d(&map, smem_u32(tile + static_cast<size_t>(c) * chunk_bytes), c * W, j0, k, s);
      tma_store_commit();
    }
  }
  if (t == 0) tma_store_wait_read();
}

// ---------------------------------------------------------------------------
// y and z sweeps
// ---------------------------------------------------------------------------
template <typename T, int AXIS>
__global__ void __launch_bounds__(256) sweep_yz_kernel(const __grid_constant__ CUtensorMap map, const SweepParams<T> p,
                                                       int CH) {
  constexpr int R = 16;  // rows staged in registers per batch of the recurrence
  extern __shared__ unsigned char smem_raw[];
  const int TI = blockDim.x;
  const int nx = p.nx, ny = p.ny, nz = p.nz, S = p.S;
  const int n = (AXIS == 1) ? ny : nz;
  const int C = (n + CH - 1) / CH;
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  T* tile = reinterpret_cast<T*>(base + ((C * 8 + 127) & ~127));
  const uint32_t chunk_bytes = static_cast<uint32_t>(CH) * TI * sizeof(T);

  const int t = threadIdx.x;
  const int i0 = blockIdx.x * TI, m = blockIdx.y, s = blockIdx.z;  // m = k (y sweep) or j (z sweep)

  if (t == 0) {
    prefetch_tmap(&map);
    for (int c = 0; c < C; ++c) mbar_init(smem_u32(&bars[c]), 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (t == 0) {
    for (int c = 0; c < C; ++c) {
      const uint32_t bar = smem_u32(&bars[c]);
      mbar_expect_tx(bar, chunk_bytes);
      T* dst = tile + static_cast<size_t>(c) * CH * TI;
      if (AXIS == 1)
        tma_load_4d(smem_u32(dst), &map, bar, i0, c * CH, m, s);
      else
        tma_load_4d(smem_u32(dst), &map, bar, i0, m, c * CH, s);
    }
  }

  const int i = i0 + t;
  const bool valid = i < nx;
  const bool act = p.active[s] != 0;
  bool face;
  const double* fv = nullptr;  // face-line values: fv[r * fstride]
  size_t fstride = 1;
  const double off = kF32<T> ? p.off[s] : 0.0;
  T e0v = T(0), e1v = T(0);  // pinned values at the two ends of the line
  if (AXIS == 1) {
    const int k = m;
    face = act && (i == 0 || i == nx - 1 || k == 0 || k == nz - 1);
    if (face && valid) {
      if (k == 0 || k == nz - 1) {
        fv = p.zface + (static_cast<size_t>(k == 0 ? 0 : 1) * S + s) * ny * nx + i;
        fstride = nx;
      } else {
        fv = p.xface + ((static_cast<size_t>(i == 0 ? 0 : 1) * S + s) * nz + k) * ny;
        fstride = 1;
      }
    }
    if (act && valid) {
      e0v = static_cast<T>(p.yface[(static_cast<size_t>(0 * S + s) * nz + k) * nx + i] - off);
      e1v = static_cast<T>(p.yface[(static_cast<size_t>(1 * S + s) * nz + k) * nx + i] - off);
    }
  } else {
    const int j = m;
    face = act && (i == 0 || i == nx - 1 || j == 0 || j == ny - 1);
    if (face && valid) {
      if (j == 0 || j == ny - 1) {
        fv = p.yface + (static_cast<size_t>(j == 0 ? 0 : 1) * S + s) * nz * nx + i;
        fstride = nx;
      } else {
        fv = p.xface + (static_cast<size_t>(i == 0 ? 0 : 1) * S + s) * nz * ny + j;
        fstride = ny;
      }
    }
    if (act && valid) {
      e0v = static_cast<T>(p.zface[(static_cast<size_t>(0 * S + s) * ny + j) * nx + i] - off);
      e1v = static_cast<T>(p.zface[(static_cast<size_t>(1 * S + s) * ny + j) * nx + i] - off);
    }
  }
  const AxisCoefs<T>& ac = (AXIS == 1) ? p.ay : p.az;
  const double* __restrict__ dn = ac.denom + static_cast<size_t>(s) * n;
  const T* __restrict__ rc = ac.rcp + static_cast<size_t>(s) * n;
  const T* __restrict__ cu = ac.cup + static_cast<size_t>(s) * n;
  const T* __restrict__ rcl = kF32<T> ? ac.rcp_lo + static_cast<size_t>(s) * n : nullptr;
  const T* __restrict__ cul = kF32<T> ? ac.cup_lo + static_cast<size_t>(s) * n : nullptr;
  const T c1 = p.c1[s];
  const T c1l = kF32<T> ? p.c1_lo[s] : T(0);
  const T shift = kF32<T> ? p.shift[s] : T(0);
  T* col = tile + t;
  bool ok = true;

  T yprev = T(0);
  for (int c = 0; c < C; ++c) {
    if (ok) ok = mbar_wait(smem_u32(&bars[c]), 0);
    if (face) continue;
    const int r1 = min(n, (c + 1) * CH);
    for (int rb = c * CH; rb < r1; rb += R) {
      T v[R];
      double d[R];
      T r[R], rl[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int rr = min(rb + q, r1 - 1);
        v[q] = col[static_cast<size_t>(rr) * TI];
        r[q] = __ldg(rc + rr);
        if constexpr (kF32<T>) {
          rl[q] = __ldg(rcl + rr);
          d[q] = 0.0;
        } else {
          d[q] = __ldg(dn + rr);
          rl[q] = T(0);
        }
      }
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int rr = rb + q;
        if (rr < r1) {
          const T vq = kF32<T> ? v[q] - shift : v[q];
          const T tt = (rr == 0) ? vq : Arith<T>::lin(c1, c1l, yprev, vq);
          const T y = Arith<T>::div(tt, d[q], r[q], rl[q]);
          col[static_cast<size_t>(rr) * TI] = y;
          yprev = y;
        }
      }
    }
  }
  if (__syncthreads_or(!ok)) {
    if (t == 0) atomicExch(p.status, kDevTimeout);
    return;
  }

  T xnext = T(0);
  for (int c = C - 1; c >= 0; --c) {
    const int r0 = c * CH;
    const int r1 = min(n, (c + 1) * CH);
    if (face) {
      for (int rr = r0; rr < r1; ++rr)
        col[static_cast<size_t>(rr) * TI] = static_cast<T>(fv != nullptr ? fv[rr * fstride] - off : 0.0);
    } else {
      for (int rb = r1 - 1; rb >= r0; rb -= R) {
        T v[R];
        T cw[R], cwl[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int rr = max(rb - q, r0);
          v[q] = col[static_cast<size_t>(rr) * TI];
          cw[q] = __ldg(cu + rr);
          cwl[q] = kF32<T> ? __ldg(cul + rr) : T(0);
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int rr = rb - q;
          if (rr >= r0) {
            const T x = (rr == n - 1) ? v[q] : Arith<T>::back(cw[q], cwl[q], xnext, v[q]);
            xnext = x;
            col[static_cast<size_t>(rr) * TI] = (act && (rr == 0 || rr == n - 1)) ? (rr == 0 ? e0v : e1v) : x;
          }
        }
      }
    }
    fence_async_smem();
    __syncthreads();
    if (t == 0) {
      const uint32_t src = smem_u32(tile + static_cast<size_t>(c) * CH * TI);
      if (AXIS == 1)
        tma_store_4d(&map, src, i0, c * CH, m, s);
      else
        tma_store_4d(&map, src, i0, m, c * CH, s);
      tma_store_commit();
    }
  }
  if (t == 0) tma_store_wait_read();
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t sweep_x_smem(int elem_bytes, int nx, const SweepConfig& cfg) {
  const int W = 128 / elem_bytes;
  const int C = (nx + W - 1) / W;
  return 1024 + ((static_cast<size_t>(C) * 8 + 1023) & ~size_t(1023)) + static_cast<size_t>(C) * cfg.x_lines * 128;
}

static int yz_chunk_rows(int n, int target) {
  const int C = (n + target - 1) / target;
  return (n + C - 1) / C;
}

size_t sweep_yz_smem(int elem_bytes, int n_line, const SweepConfig& cfg) {
  const int CH = yz_chunk_rows(n_line, cfg.yz_chunk);
  const int C = (n_line + CH - 1) / CH;
  return 128 + ((static_cast<size_t>(C) * 8 + 127) & ~size_t(127)) +
         static_cast<size_t>(C) * CH * cfg.yz_tile * elem_bytes;
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
                      const cuuint32_t box[4], CUtensorMapSwizzle swz) {
  auto enc = get_encode();
  if (enc == nullptr) return -1;
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, f, dims,
                   strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -2;
}

int encode_field_maps(FieldMaps* maps, void* f, int eb, int nx, int ny, int nz, int S, int nxp,
                      const SweepConfig& cfg) {
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)S};
  const cuuint64_t strides[3] = {(cuuint64_t)nxp * eb, (cuuint64_t)nxp * ny * eb, (cuuint64_t)nxp * ny * nz * eb};
  const cuuint32_t bx[4] = {(cuuint32_t)(128 / eb), (cuuint32_t)cfg.x_lines, 1, 1};
  const cuuint32_t by[4] = {(cuuint32_t)cfg.yz_tile, (cuuint32_t)yz_chunk_rows(ny, cfg.yz_chunk), 1, 1};
  const cuuint32_t bz[4] = {(cuuint32_t)cfg.yz_tile, 1, (cuuint32_t)yz_chunk_rows(nz, cfg.yz_chunk), 1};
  int rc = encode_one(&maps->x, f, eb, dims, strides, bx, CU_TENSOR_MAP_SWIZZLE_128B);
  if (rc == 0) rc = encode_one(&maps->y, f, eb, dims, strides, by, CU_TENSOR_MAP_SWIZZLE_NONE);
  if (rc == 0) rc = encode_one(&maps->z, f, eb, dims, strides, bz, CU_TENSOR_MAP_SWIZZLE_NONE);
  return rc;
}

template <typename T>
cudaError_t launch_sweep_x(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  const size_t smem = sweep_x_smem(sizeof(T), p.nx, cfg);
  cudaError_t e = cudaFuncSetAttribute(sweep_x_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.ny + cfg.x_lines - 1) / cfg.x_lines, p.nz, p.S);
  sweep_x_kernel<T><<<grid, cfg.x_lines, smem, st>>>(maps.x, p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_sweep_y(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  const size_t smem = sweep_yz_smem(sizeof(T), p.ny, cfg);
  cudaError_t e = cudaFuncSetAttribute(sweep_yz_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.nx + cfg.yz_tile - 1) / cfg.yz_tile, p.nz, p.S);
  sweep_yz_kernel<T, 1><<<grid, cfg.yz_tile, smem, st>>>(maps.y, p, yz_chunk_rows(p.ny, cfg.yz_chunk));
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_sweep_z(const FieldMaps& maps, const SweepParams<T>& p, const SweepConfig& cfg, cudaStream_t st) {
  const size_t smem = sweep_yz_smem(sizeof(T), p.nz, cfg);
  cudaError_t e = cudaFuncSetAttribute(sweep_yz_kernel<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((p.nx + cfg.yz_tile - 1) / cfg.yz_tile, p.ny, p.S);
  sweep_yz_kernel<T, 2><<<grid, cfg.yz_tile, smem, st>>>(maps.z, p, yz_chunk_rows(p.nz, cfg.yz_chunk));
  return cudaGetLastError();
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

}  // namespace bfvm
