// bfvm_gradients.cu -- substrate gradients at every voxel.
//
// Reference: Microenvironment::compute_all_gradient_vectors
// (BioFVM/BioFVM_microenvironment.cpp:1454-1616): per substrate and axis, a
// one-sided difference (a - b) / dx at the two ends of each line and a
// central difference (a - b) / (2 dx) inside, evaluated as
// `g = a; g -= b; g /= h` -- one subtraction and one IEEE division, which the
// kernel repeats, so FP64 results equal the reference's bit for bit.  An axis
// of length 1 gets 0 (the reference reads outside its array there, and skips
// the z component when nz == 1).  The reference caches 2*dx in function
// statics on its first call; here each solve uses its own dx.
//
// Output layout is the reference's gradient_vectors: out[(v*S + d)*3 + axis]
// with v = (i*ny + j)*nz + k, z fastest, while the device field is x
// fastest, so the kernel transposes through shared memory.
//
// gradient_plane_kernel (used whenever its tensor map encodes): a CTA owns
// 32 consecutive x by 8 consecutive z and walks a range of y planes.  Each
// plane's block -- with a one-voxel halo in z and the x halo rounded out to
// 16-byte boundaries, up to 4 substrates -- arrives by one TMA box load into
// a ring of four plane slots, so planes j-1, j, j+1 are resident while j+2
// loads and every field value is read from HBM about once (the halo and the
// planes shared by neighbouring y ranges aside).  The 256 threads (lane = x,
// warp = z) compute the plane's gradients into a shared-memory block ordered
// like the output, which the CTA then writes as contiguous runs (one x row's
// 8 voxels x 3 x substrates per run).  Algorithmic bytes per voxel and
// substrate: 8 read + 24 written (FP64 field).
//
// gradient_kernel is the earlier form (32 z by 8 x of one plane per CTA,
// rows read with plain loads), kept for grids whose map does not encode.
#include <algorithm>
#include <cmath>

#include "bfvm_ctx.h"
#include "bfvm_ptx.cuh"

namespace {

constexpr int kGTX = 32;     // x per CTA (one warp's lanes)
constexpr int kGTZ = 8;      // z per CTA (one per warp)
constexpr int kGSlots = 4;   // plane slots: j-1, j, j+1 resident, j+2 loading
constexpr int kGBoxZ = kGTZ + 2;
template <typename T>
constexpr int kGBoxX = sizeof(T) == 8 ? 36 : 40;  // x extent of a plane box (16-byte aligned origin)
template <typename T>
constexpr int kGX0 = sizeof(T) == 8 ? 2 : 4;      // box x origin below the CTA's first x

template <typename T, int NS>
__host__ __device__ constexpr size_t grad_slot_bytes() {
  return (static_cast<size_t>(kGBoxX<T>) * kGBoxZ * NS * sizeof(T) + 127) / 128 * 128;
}
template <int NS>
__host__ __device__ constexpr int grad_stage_stride() {  // doubles per x row of the output block (even: 16-byte rows)
  return kGTZ * 3 * NS + 2;
}
template <typename T, int NS>
__host__ __device__ constexpr size_t grad_smem_bytes() {
  return 128 + 128 + kGSlots * grad_slot_bytes<T, NS>() + sizeof(double) * kGTX * grad_stage_stride<NS>();
}

// The quotient where Markstein's correction does not apply (kept out of
// line, so the common path carries none of the division sequence): +0 for a
// numerator of +0, else IEEE division.
__device__ __noinline__ double grad_quotient_slow(double g, double h) {
  if (g == 0.0 && !signbit(g)) return 0.0;
  return g / h;
}

// Gradients of substrates s0 .. s0+ns-1 (ns <= NS) for the planes [jb, je)
// of one (32 x, 8 z) column of the grid; planes come from `map` (the field,
// box {kGBoxX, 1, 10, NS}: NS substrates from s0, those past S zero-filled).
template <typename T, int NS>
__global__ void __launch_bounds__(256, 3) gradient_plane_kernel(const __grid_constant__ CUtensorMap map, int nx, int ny,
                                                             int nz, int S, int s0, int jc,
                                                             const double* __restrict__ off, double dx,
                                                             double* __restrict__ out, int* status) {
  const int ns = min(NS, S - s0);
  extern __shared__ unsigned char smem_raw[];
  const uint32_t a0 = bfvm::smem_u32(smem_raw);
  unsigned char* base = smem_raw + (((a0 + 127u) & ~127u) - a0);  // 128-byte aligned (TMA destinations)
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  unsigned char* slots = base + 128;
  double* stg = reinterpret_cast<double*>(slots + kGSlots * grad_slot_bytes<T, NS>());
  constexpr int BX = kGBoxX<T>;
  constexpr int X0 = kGX0<T>;
  constexpr int PS = BX * kGBoxZ;  // elements per substrate in a slot
  constexpr uint32_t kBoxBytes = static_cast<uint32_t>(BX * kGBoxZ * NS * sizeof(T));
  constexpr int SX = grad_stage_stride<NS>();
  constexpr int RUN = kGTZ * 3 * NS;  // output doubles per x row of the block
  const int i0 = blockIdx.x * kGTX, k0 = blockIdx.y * kGTZ;
  const int jb = blockIdx.z * jc;
  const int je = min(ny, jb + jc);
  const int tid = threadIdx.x, lane = tid & 31, wz = tid >> 5;
  const int jlast = min(je, ny - 1);  // last plane this CTA reads
  const int jfirst = max(jb - 1, 0);  // first plane this CTA reads
  // plane p lives in slot (p - jfirst) % 4 and is that slot's ((p - jfirst) / 4)-th load
  auto slot_of = [&](int p) { return (p - jfirst) & (kGSlots - 1); };
  auto parity_of = [&](int p) { return static_cast<uint32_t>(((p - jfirst) >> 2) & 1); };
  auto issue = [&](int p) {
    const int sl = slot_of(p);
    const uint32_t bar = bfvm::smem_u32(&bars[sl]);
    bfvm::mbar_expect_tx(bar, kBoxBytes);
    bfvm::tma_load_4d(bfvm::smem_u32(slots + sl * grad_slot_bytes<T, NS>()), &map, bar, i0 - X0, p, k0 - 1, s0);
  };
  if (tid == 0) {
    bfvm::prefetch_tmap(&map);
    for (int q = 0; q < kGSlots; ++q) bfvm::mbar_init(bfvm::smem_u32(&bars[q]), 1);
    bfvm::fence_barrier_init();
  }
  __syncthreads();
  int issued = min(jfirst + kGSlots - 1, jlast);  // planes jfirst .. issued are (being) loaded
  if (tid == 0)
    for (int p = jfirst; p <= issued; ++p) issue(p);
  bool ok = true;
  int waited = jfirst - 1;  // planes jfirst .. waited have landed
  auto wait_plane = [&](int p) {
    if (ok) ok = bfvm::mbar_wait(bfvm::smem_u32(&bars[slot_of(p)]), parity_of(p));
    if (ok) waited = p;
  };
  if (jb > 0) wait_plane(jb - 1);
  const double two_dx = dx * 2.0;
  // The divisor's reciprocal, for the quotient by Markstein's correction of
  // RN(g * RN(1/h)) -- three FP64 operations instead of the IEEE division
  // sequence, and the same correctly rounded result wherever no intermediate
  // leaves the normal range: the numerator and the first quotient between
  // 2^-960 and 2^1000 in magnitude, h between 2^-100 and 2^100.  A numerator
  // of +0 gives +0; anything else outside those bounds (-0, tiny, huge)
  // takes the IEEE division.
  const double rdx = 1.0 / dx, r2dx = 1.0 / two_dx;
  const bool markstein_ok = dx >= 0x1p-100 && dx <= 0x1p99;
  // g = a; g -= b; g /= h  (BioFVM_microenvironment.cpp:1480-1482 and the
  // matching lines of every end cap and interior loop)
  // With h in [2^-100, 2^99], a numerator g in [2^-860, 2^900] in magnitude
  // keeps both g and RN(g/h) inside those bounds: one test of g's exponent.
  // grad() returns the corrected quotient and clears `fast` unless
  // 2^-860 <= |g| < 2^900 or g = +0 (which the correction maps to +0); a
  // voxel with any such component redoes them all with grad_exact().
  auto grad = [](double a, double b, double h, double rh, bool& fast) {
    double g = a;
    g -= b;
    const unsigned hw = static_cast<unsigned>(__double2hiint(g)) & 0x7FFFFFFFu;  // |g|'s high word
    const double q0 = g * rh;
    const double e = __fma_rn(-q0, h, g);
    fast &= (hw - 0x0A300000u < 0x78300000u - 0x0A300000u) | (__double_as_longlong(g) == 0);
    return __fma_rn(e, rh, q0);
  };
  auto grad_exact = [markstein_ok](double a, double b, double h, double rh) {
    double g = a;
    g -= b;
    const unsigned hw = static_cast<unsigned>(__double2hiint(g)) & 0x7FFFFFFFu;
    if (markstein_ok && (hw - 0x0A300000u < 0x78300000u - 0x0A300000u || __double_as_longlong(g) == 0)) {
      const double q0 = g * rh;
      return __fma_rn(__fma_rn(-q0, h, g), rh, q0);
    }
    return grad_quotient_slow(g, h);
  };
  const int i = i0 + lane, k = k0 + wz;
  const int ix = lane + X0, iz = wz + 1;  // this thread's voxel in a slot
  // Per axis: a line's two ends take the one-sided difference over dx, the
  // voxels between the central one over 2 dx.  Each component is
  // (value at +o) - (value at -o) with offsets that are 0 at the matching
  // end (the centre stands in for the missing neighbour), so the component
  // needs no branch or select; an axis of length 1 is zeroed at the end.
  const bool x_lo = i == 0, x_hi = i == nx - 1;
  const bool z_lo = k == 0, z_hi = k == nz - 1;
  const int oxp = x_hi ? 0 : 1, oxm = x_lo ? 0 : 1;
  const int ozp = z_hi ? 0 : BX, ozm = z_lo ? 0 : BX;
  const double hx = (x_lo || x_hi) ? dx : two_dx, rhx = (x_lo || x_hi) ? rdx : r2dx;
  const double hz = (z_lo || z_hi) ? dx : two_dx, rhz = (z_lo || z_hi) ? rdx : r2dx;
  const bool zero_x = nx == 1, zero_y = ny == 1, zero_z = nz == 1;
  const bool any_zero_axis = zero_x || zero_y || zero_z;
  for (int j = jb; j < je; ++j) {
    if (j == jb) wait_plane(j);
    if (j + 1 < ny) wait_plane(j + 1);
    if (!__syncthreads_and(ok)) break;  // a plane never landed: stop (status set below)
    const T* P1 = reinterpret_cast<const T*>(slots + slot_of(j) * grad_slot_bytes<T, NS>());
    const T* P0 = j > 0 ? reinterpret_cast<const T*>(slots + slot_of(j - 1) * grad_slot_bytes<T, NS>()) : P1;
    const T* P2 = j + 1 < ny ? reinterpret_cast<const T*>(slots + slot_of(j + 1) * grad_slot_bytes<T, NS>()) : P1;
    if (i < nx && k < nz) {
      const bool y_lo = j == 0, y_hi = j == ny - 1;
      const double hy = (y_lo || y_hi) ? dx : two_dx, rhy = (y_lo || y_hi) ? rdx : r2dx;
      const T* Pyp = y_hi ? P1 : P2;  // plane j+1, or j itself at the last plane
      const T* Pym = y_lo ? P1 : P0;  // plane j-1, or j itself at the first plane
      double g3[3 * NS];
      bool fast = markstein_ok;
      // substrates past the group's last (sl >= ns) read the map's zero
      // fill; their values are staged but never written out
      // FP32 fields hold rho - off; an FP64 field is read as it is (adding 0.0
      // would also turn a -0 into +0, which the reference keeps)
      auto v = [&](const T* P, int e, double o) {
        if constexpr (sizeof(T) == 4)
          return static_cast<double>(P[e]) + o;
        else
          return static_cast<double>(P[e]);
      };
#pragma unroll
      for (int sl = 0; sl < NS; ++sl) {
        const double o = (sizeof(T) == 4 && sl < ns) ? off[s0 + sl] : 0.0;
        const int c = sl * PS + iz * BX + ix;
        g3[3 * sl + 0] = grad(v(P1, c + oxp, o), v(P1, c - oxm, o), hx, rhx, fast);
        g3[3 * sl + 1] = grad(v(Pyp, c, o), v(Pym, c, o), hy, rhy, fast);
        g3[3 * sl + 2] = grad(v(P1, c + ozp, o), v(P1, c - ozm, o), hz, rhz, fast);
      }
      if (!fast) {  // rare: a component outside the correction's range
#pragma unroll
        for (int sl = 0; sl < NS; ++sl) {
          const double o = (sizeof(T) == 4 && sl < ns) ? off[s0 + sl] : 0.0;
          const int c = sl * PS + iz * BX + ix;
          g3[3 * sl + 0] = grad_exact(v(P1, c + oxp, o), v(P1, c - oxm, o), hx, rhx);
          g3[3 * sl + 1] = grad_exact(v(Pyp, c, o), v(Pym, c, o), hy, rhy);
          g3[3 * sl + 2] = grad_exact(v(P1, c + ozp, o), v(P1, c - ozm, o), hz, rhz);
        }
      }
      if (any_zero_axis) {  // uniform: grids with an axis of length 1 only
#pragma unroll
        for (int sl = 0; sl < NS; ++sl) {
          if (zero_x) g3[3 * sl + 0] = 0.0;
          if (zero_y) g3[3 * sl + 1] = 0.0;
          if (zero_z) g3[3 * sl + 2] = 0.0;
        }
      }
      double* o3 = stg + lane * SX + wz * 3 * NS;
      if constexpr ((NS & 1) == 0) {
        // 16-byte stores: with NS even, a thread's 3 x NS values start on a
        // 16-byte boundary (SX and 3 NS even, the block 128-byte aligned)
#pragma unroll
        for (int q = 0; q < 3 * NS; q += 2) reinterpret_cast<double2*>(o3)[q / 2] = make_double2(g3[q], g3[q + 1]);
      } else {
#pragma unroll
        for (int q = 0; q < 3 * NS; ++q) o3[q] = g3[q];
      }
    }
    __syncthreads();  // the block is complete and every read of plane j-1 is done
    // plane j+3 into plane j-1's slot, unless the prologue loaded it already
    // (a CTA starting at plane 0 has no plane -1, so its prologue takes 0..3)
    if (j + 3 <= jlast && j + 3 > issued) {
      if (tid == 0) issue(j + 3);
      issued = j + 3;
    }
    // x row il of the block: 8 voxels x 3 x ns doubles, contiguous in the
    // output when the group holds every substrate and the z tile is whole:
    // then warp wz writes rows wz, wz + 8, ... as straight runs (16-byte
    // stores when the run starts 16-byte aligned: S even and out 16-byte
    // aligned)
    const int nk = min(kGTZ, nz - k0);
    if (ns == S && nk == kGTZ) {
      for (int il = wz; il < kGTX; il += 8) {
        if (i0 + il >= nx) break;
        double* dst = out + ((static_cast<size_t>(i0 + il) * ny + j) * nz + k0) * (3 * static_cast<size_t>(S));
        const double* src = stg + il * SX;
        if ((S & 1) == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0) {
          for (int u = lane; u < RUN / 2; u += 32)
            reinterpret_cast<double2*>(dst)[u] = reinterpret_cast<const double2*>(src)[u];
        } else {
          for (int u = lane; u < RUN; u += 32) dst[u] = src[u];
        }
      }
    } else {
      for (int q = tid; q < kGTX * RUN; q += 256) {
        const int il = q / RUN, r = q - il * RUN;
        const int kl = r / (3 * NS), e = r - kl * (3 * NS);
        if (i0 + il < nx && kl < nk && e < 3 * ns)
          out[((static_cast<size_t>(i0 + il) * ny + j) * nz + k0 + kl) * (3 * static_cast<size_t>(S)) + 3 * s0 + e] =
              stg[il * SX + r];
      }
    }
    __syncthreads();  // the block is free for the next plane
  }
  if (!ok) {
    // a wait gave up: let the loads still in flight land (each wait bounded)
    // before the CTA's shared memory goes away, then report it
    for (int p = waited + 1; p <= issued; ++p) bfvm::mbar_wait(bfvm::smem_u32(&bars[slot_of(p)]), parity_of(p));
    if (tid == 0) atomicExch(status, bfvm::kDevTimeout);
  }
}

template <typename T, int NS>
cudaError_t launch_plane_kernel(bfvm_ctx* c, int s0, double* d_out) {
  constexpr size_t smem = grad_smem_bytes<T, NS>();
  cudaError_t e = cudaFuncSetAttribute(gradient_plane_kernel<T, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int xt = (c->nx + kGTX - 1) / kGTX, zt = (c->nz + kGTZ - 1) / kGTZ;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gradient_plane_kernel<T, NS>, 256, smem);
  if (e != cudaSuccess) return e;
  const long long wave = static_cast<long long>(std::max(per_sm, 1)) * sms;
  // y ranges of at least 8 planes: among the counts that fill at least one
  // wave of CTAs (or the most ranges there are), the one whose last wave is
  // fullest, the fewer ranges on a tie (each range re-reads a halo plane)
  const long long cols = static_cast<long long>(xt) * zt;
  const int most = std::max(1, (c->ny + 7) / 8);
  int chunks = most;
  double best = -1.0;
  for (int q = 1; q <= most; ++q) {
    const int jq = (c->ny + q - 1) / q;
    const long long ctas = cols * ((c->ny + jq - 1) / jq);
    if (ctas < wave && q < most) continue;
    const double waves = static_cast<double>(ctas) / static_cast<double>(wave);
    const double fill = waves / std::ceil(waves);
    if (fill > best + 1e-9) {
      best = fill;
      chunks = q;
    }
    if (ctas >= 4 * wave) break;
  }
  const int jc = (c->ny + chunks - 1) / chunks;
  const dim3 grid(xt, zt, (c->ny + jc - 1) / jc);
  gradient_plane_kernel<T, NS><<<grid, 256, smem, c->stream>>>(
      c->maps.g, c->nx, c->ny, c->nz, c->S, s0, jc, c->prec == BFVM_FP32 ? c->d_off : nullptr, c->dx, d_out,
      c->d_status);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_plane_groups(bfvm_ctx* c, double* d_out, int* launches) {
  *launches = 0;
  const int G = std::min(4, c->S);  // substrates per box of c->maps.g
  for (int s0 = 0; s0 < c->S; s0 += G) {
    cudaError_t e = cudaSuccess;
    switch (G) {
      case 1: e = launch_plane_kernel<T, 1>(c, s0, d_out); break;
      case 2: e = launch_plane_kernel<T, 2>(c, s0, d_out); break;
      case 3: e = launch_plane_kernel<T, 3>(c, s0, d_out); break;
      default: e = launch_plane_kernel<T, 4>(c, s0, d_out); break;
    }
    if (e != cudaSuccess) return e;
    ++*launches;
  }
  return cudaSuccess;
}

constexpr int kGroup = 4;  // substrates staged per output block (keeps static shared memory under 48 KB)

template <typename T>
__global__ void __launch_bounds__(256) gradient_kernel(const T* __restrict__ f, int nx, int ny, int nz, int S,
                                                       int nxp, const double* __restrict__ off, double dx,
                                                       double* __restrict__ out) {
  __shared__ double c[34][10];     // this plane: (k - k0 + 1, i - i0 + 1)
  __shared__ double ym[32][9];     // plane j - 1: (k - k0, i - i0)
  __shared__ double yp[32][9];     // plane j + 1
  __shared__ double og[8][32][3 * kGroup + 1];  // output: (i - i0, k - k0, 3*(s - s0) + axis)
  const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 8, j = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const double two_dx = dx * 2.0;
  auto at = [&](int s, int k, int jj, int i) {
    return static_cast<double>(f[((static_cast<size_t>(s) * nz + k) * ny + jj) * nxp + i]);
  };
  // g = a; g -= b; g /= h  (BioFVM_microenvironment.cpp:1480-1482 and the
  // matching lines of every end cap and interior loop)
  auto grad = [](double a, double b, double h) {
    double g = a;
    g -= b;
    return g / h;
  };
  const int i = i0 + ty, k = k0 + tx;
  const int nk = min(32, nz - k0);
  for (int s0 = 0; s0 < S; s0 += kGroup) {
    const int ns = min(kGroup, S - s0);
    for (int sl = 0; sl < ns; ++sl) {
      const int s = s0 + sl;
      const double o = off ? off[s] : 0.0;
      for (int q = tid; q < 34 * 10; q += 256) {
        const int kk = q / 10, ii = q - kk * 10;
        const int gk = k0 - 1 + kk, gi = i0 - 1 + ii;
        if (gk >= 0 && gk < nz && gi >= 0 && gi < nx) c[kk][ii] = at(s, gk, j, gi) + o;
      }
      {
        const int kk = tid >> 3, ii = tid & 7;
        const int gk = k0 + kk, gi = i0 + ii;
        if (gk < nz && gi < nx) {
          if (j > 0) ym[kk][ii] = at(s, gk, j - 1, gi) + o;
          if (j < ny - 1) yp[kk][ii] = at(s, gk, j + 1, gi) + o;
        }
      }
      __syncthreads();
      if (i < nx && k < nz) {
        const int kk = tx + 1, ii = ty + 1;
        const double ctr = c[kk][ii];
        double gx = 0.0, gy = 0.0, gz = 0.0;
        if (nx > 1) {
          if (i == 0)
            gx = grad(c[kk][ii + 1], ctr, dx);
          else if (i == nx - 1)
            gx = grad(ctr, c[kk][ii - 1], dx);
          else
            gx = grad(c[kk][ii + 1], c[kk][ii - 1], two_dx);
        }
        if (ny > 1) {
          if (j == 0)
            gy = grad(yp[tx][ty], ctr, dx);
          else if (j == ny - 1)
            gy = grad(ctr, ym[tx][ty], dx);
          else
            gy = grad(yp[tx][ty], ym[tx][ty], two_dx);
        }
        if (nz > 1) {
          if (k == 0)
            gz = grad(c[kk + 1][ii], ctr, dx);
          else if (k == nz - 1)
            gz = grad(ctr, c[kk - 1][ii], dx);
          else
            gz = grad(c[kk + 1][ii], c[kk - 1][ii], two_dx);
        }
        og[ty][tx][3 * sl + 0] = gx;
        og[ty][tx][3 * sl + 1] = gy;
        og[ty][tx][3 * sl + 2] = gz;
      }
      __syncthreads();
    }
    // warp ty writes x row i: nk voxels, each 3*ns values at column 3*s0
    if (i < nx) {
      const int w = 3 * ns;
      double* row = out + (((static_cast<size_t>(i) * ny + j) * nz + k0) * S + s0) * 3;
      for (int q = tx; q < nk * w; q += 32) {
        const int kk = q / w, e = q - kk * w;
        row[static_cast<size_t>(kk) * 3 * S + e] = og[ty][kk][e];
      }
    }
    __syncthreads();
  }
}

int launch_gradients(bfvm_ctx* c, double* d_out) {
  if (c->maps.g_ok) {
    int launches = 0;
    if (c->prec == BFVM_FP64)
      BFVM_CUDA(launch_plane_groups<double>(c, d_out, &launches));
    else
      BFVM_CUDA(launch_plane_groups<float>(c, d_out, &launches));
    bfvm::note_launches(launches);
    return BFVM_OK;
  }
  const dim3 block(32, 8);
  const dim3 grid((c->nz + 31) / 32, (c->nx + 7) / 8, c->ny);
  if (c->prec == BFVM_FP64)
    gradient_kernel<double><<<grid, block, 0, c->stream>>>(static_cast<const double*>(c->f), c->nx, c->ny, c->nz,
                                                           c->S, c->nxp, nullptr, c->dx, d_out);
  else
    gradient_kernel<float><<<grid, block, 0, c->stream>>>(static_cast<const float*>(c->f), c->nx, c->ny, c->nz,
                                                          c->S, c->nxp, c->d_off, c->dx, d_out);
  BFVM_CUDA(cudaGetLastError());
  bfvm::note_launches(1);
  return BFVM_OK;
}

}  // namespace

extern "C" int bfvm_compute_gradients_device(bfvm_ctx* c, double* d_out) {
  if (!c || !d_out) return BFVM_ERR_ARG;
  bfvm::DeviceGuard g(c->device);
  return launch_gradients(c, d_out);
}

extern "C" int bfvm_compute_gradients(bfvm_ctx* c, double* out) {
  if (!c || !out) return BFVM_ERR_ARG;
  bfvm::DeviceGuard g(c->device);
  const size_t bytes = sizeof(double) * 3 * static_cast<size_t>(c->nx) * c->ny * c->nz * c->S;
  if (!c->d_grad) {
    const int rc = bfvm::dalloc(c, reinterpret_cast<void**>(&c->d_grad), bytes);
    if (rc != BFVM_OK) return rc;
  }
  int rc = launch_gradients(c, c->d_grad);
  if (rc != BFVM_OK) return rc;
  BFVM_CUDA(cudaMemcpyAsync(out, c->d_grad, bytes, cudaMemcpyDeviceToHost, c->stream));
  return bfvm_synchronize(c);
}
