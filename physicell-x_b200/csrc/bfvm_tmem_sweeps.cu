// bfvm_tmem_sweeps.cu -- the persistent FP64 sweeps with tensor-memory
// (TMEM) rings, and their launches.
//
// Reference: the x, y and z sweeps of
// diffusion_decay_solver__constant_coefficients_LOD_3D_BLOCKING
// (BioFVM/BioFVM_solvers.cpp:352-777, one rank) with the Dirichlet pins of
// Microenvironment::apply_dirichlet_boundaries_conditions
// (BioFVM/BioFVM_microenvironment.cpp:348-446), as in bfvm_sweeps.cu: same
// operations in the same order, the same bits.
//
// A sweep's speed is set by how many Thomas systems (lines) an SM keeps in
// flight, since each line's recurrence is a serial chain; a line's forward
// results must be held until its back substitution.  Shared memory alone
// holds 128 FP64 lines of 200 per SM.  These kernels add up to four rings
// that keep their forward results in TMEM (one 32-lane quarter each, 512
// 32-bit columns = 256 FP64 values per lane), so an SM holds 224 such lines.
// TMEM is used as storage only (tcgen05.alloc / st / ld); no MMA runs.
#include <climits>
#include <type_traits>

#include "biofvm_b200.h"
#include "bfvm_internal.h"
#include "bfvm_ptx.cuh"
#include "bfvm_sweep_common.cuh"

namespace bfvm {

// y/z sweep, persistent, with tensor memory.  One CTA per SM of up to seven
// rings, each one warp with no copy warp: warps 0..ns-1 (ns <= 3, as many as
// shared memory holds) keep their tile's 16-row chunks in shared-memory slots
// (forward results in place, as the ring sweep of bfvm_sweeps.cu does); the
// next nt <= 4 warps -- one per TMEM lane quarter -- stream each of a line's
// first 16 chunks through three shared-memory slots and keep its forward
// results in their 32 TMEM lanes (32 columns per chunk), the chunks past 16
// resident in shared-memory slots.  Lane 0 of each warp issues
// its ring's TMA loads; the back substitution writes the results straight to
// the field (each row a coalesced 256-byte store), so a slot is free as soon
// as the warp has read it and the next tile's chunks load into it at once.
// Tiles are handed out by a per-solve counter (zeroed again by the launch's
// last CTA), so rings of either kind take work as they free up.
constexpr int kTmemRingSmem = 3;     // most shared-memory rings (warps 0..ns-1)
constexpr int kTmemRingTmem = 4;     // most TMEM rings (warps ns..ns+nt-1), one per lane quarter
constexpr int kTmemFlowSlots = 3;    // input slots of a TMEM ring
constexpr int kTmemBarrierBytes = 256;  // up to 32 slot barriers
constexpr int kTmemMaxChunks = 16;   // 16 chunks x 32 columns = the 512 TMEM columns

// The shape of one y/z persistent sweep, shared by its rings.
struct YzShape {
  int nx, n, nm, C, ntx;
  long long per_s, ntiles;
  size_t row_stride;
  // Packed tiles: when nx % 32 = rem is 1..16, a plane's last x tile would
  // hold rem lines at the cost of a full one (the sweeps are latency bound).
  // Instead the first ntr = nx / 32 tiles of each plane are regular and the
  // rem-wide remainders of P = 32 / pw consecutive planes (pw = rem rounded
  // up to a power of two, at least 16 bytes) share one tile, loaded by the
  // packed map as a box {pw x, P planes, 16 rows}: lane t owns x = i0 + t %
  // pw of plane m0 + t / pw, and the slot keeps the layout [row][32 lanes].
  // pw = 0: no packing (ntr = ntx).
  int ntr, pw, pw_log, P;
  long long nreg;  // regular tiles per substrate, ntr * nm
};

// Fill the tile enumeration of a YzShape (nx, nm set) for group width pw.
__device__ __forceinline__ void yz_shape_tiles(YzShape& g, int pw, int S) {
  constexpr int TI = 32;
  g.ntx = (g.nx + TI - 1) / TI;
  g.pw = pw;
  if (pw > 0) {
    g.ntr = g.nx / TI;
    g.P = TI / pw;
    g.pw_log = 31 - __clz(pw);
    g.nreg = static_cast<long long>(g.ntr) * g.nm;
    g.per_s = g.nreg + (g.nm + g.P - 1) / g.P;
  } else {
    g.ntr = g.ntx;
    g.P = 1;
    g.pw_log = 0;
    g.nreg = static_cast<long long>(g.ntx) * g.nm;
    g.per_s = g.nreg;
  }
  g.ntiles = g.per_s * S;
}

// One ring of the TMEM y/z sweep.  A line's first T chunks (T = min(C, 16)
// for a TMEM ring, 0 for a shared-memory ring) stream through kf input
// slots and keep their forward results in the ring's TMEM lanes; the other
// C - T chunks stay resident in their own slots (forward results in place).
// pend / ppar return the loads still in flight (bit per slot, and the parity
// each completes) when a wait gave up.
// MODE 0: shared-memory ring; 1: TMEM ring (C <= 16); 2: TMEM ring with
// resident chunks (C > 16).
// STAGED: the forward pairs read from the ring's copy `drs` in shared
// memory, else from global memory.
template <int AXIS, int MODE, bool STAGED, bool FAST>
__device__ __forceinline__ void yz_tmem_ring(const CUtensorMap* map, const CUtensorMap* pmap, const SweepParams<double>& p, const YzShape& g,
                                             int KF, uint64_t* full, double* slots, double* cus, double2* drs,
                                             uint32_t tbase, uint32_t& pend, uint32_t& ppar) {
  using DR = double2;
  constexpr int R = kRowBatch;
  constexpr int CH = kRingRows;
  constexpr int TI = 32;
  constexpr int kSlotElems = CH * TI;
  constexpr uint32_t kSlotBytes = kSlotElems * sizeof(double);
  constexpr unsigned kAll = 0xffffffffu;
  const int t = threadIdx.x & 31;
  const int nx = g.nx, n = g.n, nm = g.nm, C = g.C, ntr = g.ntr;
  constexpr bool TM = MODE != 0;
  const int T = MODE == 0 ? 0 : (MODE == 1 ? C : kTmemMaxChunks);  // chunks kept in TMEM
  const int NR = MODE == 1 ? 0 : C - T;                             // chunks resident in shared memory
  const int RB = TM ? KF : 0;                      // first resident slot
  const long long ntiles = g.ntiles;
  unsigned long long* counter = p.tile_counter;

  // tile -> (i0, m, s, packed): regular tiles first, then packed ones (m the
  // first plane of the group)
  auto decode = [&](long long tile, int& i0, int& m, int& s, bool& pk) {
    const int sg = static_cast<int>(tile / g.per_s);
    const long long r = tile - sg * g.per_s;
    s = p.s_lo + sg;
    pk = r >= g.nreg;
    if (pk) {
      m = static_cast<int>(r - g.nreg) * g.P;
      i0 = g.ntr * TI;
    } else {
      m = static_cast<int>(r / ntr);
      i0 = static_cast<int>(r - static_cast<long long>(m) * ntr) * TI;
    }
  };
  // A tile whose lines all lie in an activated face is already final.
  auto skip = [&](long long tile) {
    int i0, m, s;
    bool pk;
    decode(tile, i0, m, s, pk);
    return !pk && p.active[s] != 0 && (m == 0 || m == nm - 1);
  };
  // The next tile for this ring (whole warp; ntiles when none is left).
  auto grab = [&]() -> long long {
    long long v = 0;
    if (t == 0) {
      do {
        v = static_cast<long long>(atomicAdd(counter, 1ull));
      } while (v < ntiles && skip(v));
      if (v > ntiles) v = ntiles;
    }
    return __shfl_sync(kAll, v, 0);
  };
  // Chunk c of the tile at (i0, m, s) into slot sl, completing phase `par`
  // of its barrier (tiles are decoded once, when taken).
  auto issue = [&](int i0, int m, int s, bool pk, int c, int sl, uint32_t par) {
    if (t == 0) {
      const uint32_t bar = smem_u32(&full[sl]);
      mbar_expect_tx(bar, kSlotBytes);
      const uint32_t dst = smem_u32(slots + static_cast<size_t>(sl) * kSlotElems);
      if (pk)  // the packed map's dimensions: x, planes, rows along the line, substrate
        tma_load_4d(dst, pmap, bar, i0, m, c * CH, s);
      else if (AXIS == 1)
        tma_load_4d(dst, map, bar, i0, c * CH, m, s);
      else
        tma_load_4d(dst, map, bar, i0, m, c * CH, s);
    }
    pend |= 1u << sl;
    ppar = (ppar & ~(1u << sl)) | (par << sl);
  };
  // slot of resident chunk c (>= T) in tile parity `fl`
  auto rslot = [&](bool fl, int c) { return RB + ring_slot(fl, NR, c - T); };

  bool ok = true;
  long long tile = grab();
  int ti0 = 0, tm_ = 0, ts = 0;  // the current tile, decoded
  bool tp = false;
  if (tile < ntiles) {
    decode(tile, ti0, tm_, ts, tp);
    for (int c = 0; c < (TM ? KF : 0); ++c) issue(ti0, tm_, ts, tp, c, c, 0u);
    for (int c = T; c < C; ++c) issue(ti0, tm_, ts, tp, c, rslot(false, c), 0u);
  }
  const int screen = p.screen;
  int staged_s = -1;
  // chunks kc0..kc1 of the staged substrate lie in its converged range
  // (AxisCoefs::conv): their forward pairs are dk and upper diagonals ck
  int kc0 = INT_MAX, kc1 = -1;
  DR dk = make_double2(0.0, 0.0);
  double ck = 0.0;
  int fsl = 0;        // TMEM chunks: slot of the next input to consume
  uint32_t fpar = 0;  // and the phase it completes
  for (uint32_t k = 0; tile < ntiles; ++k) {
    const int i0 = ti0, m = tm_, s = ts;
    const bool pk = tp;
    const bool flip = (k & 1u) != 0;
    const bool act = p.active[s] != 0;
    // this lane's line (x = i, plane ml); lines in an activated face keep
    // their (pinned) input
    const int i = pk ? i0 + (t & (g.pw - 1)) : i0 + t;
    const int ml = pk ? m + (t >> g.pw_log) : m;
    const bool inr = i < nx && ml < nm;
    const bool face = act && (i == 0 || i == nx - 1 || ml == 0 || ml == nm - 1);
    const bool lane_on = !face && inr;
    const int mo = inr ? ml : m;  // in range for the address below
    const AxisCoefs<double>& ac = (AXIS == 1) ? p.ay : p.az;
    const DR* __restrict__ drp = ac.dr + static_cast<size_t>(s) * ac.npad;
    const double c1 = p.c1[s];
    if (s != staged_s) {
      // the substrate's coefficient rows: the upper diagonal for the back
      // substitution, the forward pairs (one chunk past the line, for the
      // prefetch) -- read as shared-memory broadcasts
      stage_row(cus, ac.cu + static_cast<size_t>(s) * ac.npad, C * CH);
      if (STAGED) stage_row(reinterpret_cast<double*>(drs), reinterpret_cast<const double*>(drp), 2 * (C + 1) * CH);
      kc0 = INT_MAX;
      kc1 = -1;
      if (FAST && ac.conv != nullptr && n >= 3) {
        kc0 = (__ldg(ac.conv + s) + CH - 1) / CH;
        kc1 = (n - 1) / CH - 1;  // chunks ending at row n - 2 or before
        dk = __ldg(drp + n - 2);
        ck = __ldg(ac.cu + static_cast<size_t>(s) * ac.npad + n - 2);
      }
      staged_s = s;
      __syncwarp();
    }
    double* out = p.f + ((AXIS == 1) ? ((static_cast<size_t>(s) * p.nz + mo) * p.ny) * p.nxp
                                     : (static_cast<size_t>(s) * p.nz * p.ny + mo) * p.nxp) + (inr ? i : i0);
    // forward pairs of chunk c (staged, or from global where the plan had no room)
    auto load_cf = [&](int c, DR (&cf)[R]) {
#pragma unroll
      for (int q = 0; q < R; ++q) cf[q] = STAGED ? drs[c * R + q] : __ldg(drp + c * R + q);
    };
    double y = -0.0;
    int hwmin = INT_MAX;
    const bool edge_tile = __any_sync(kAll, !lane_on);
    // constant-coefficient chunks of this tile (edge tiles read every chunk's)
    const int k0 = edge_tile ? INT_MAX : kc0, k1 = edge_tile ? -1 : kc1;
    long long nxt = ntiles;
    int ni0 = 0, nm_ = 0, ns_ = 0;  // the next tile, decoded when taken
    bool np_ = false;
    auto take_next = [&]() {
      nxt = grab();
      if (nxt < ntiles) decode(nxt, ni0, nm_, ns_, np_);
    };

    // ---- forward elimination ----
    // kconst: std::true_type for a chunk in the converged range
    auto fwd_chunk = [&](auto kconst, bool edge, int c) {
      constexpr bool K = decltype(kconst)::value;
      const int rb = c * CH;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      const int sl = flow ? fsl : rslot(flip, c);
      const uint32_t par = flow ? fpar : (k & 1u);
      // the chunk's forward pairs, loading while the slot's barrier is awaited
      DR cf[R];
      if constexpr (!K) load_cf(c, cf);
      if (ok) ok = mbar_wait(smem_u32(&full[sl]), par);
      pend &= ~(1u << sl);
      double* cb = slots + static_cast<size_t>(sl) * kSlotElems + t;
      double yv[R];
      if (!edge || lane_on) {
        double v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
        if (rb + R > n) {  // rows past the line's end (TMA fill): any clean value, never stored
#pragma unroll
          for (int q = 0; q < R; ++q)
            if (rb + q >= n) v[q] = 1.0;
        }
        if constexpr (K) {
          if (!FAST) hwmin = min(hwmin, batch_min_hi<R>(v));
          if (flow)
            y = forward_any_const<R>(FAST ? kScreenFast : 1, v, dk, c1, y, [&](int q, double val) { yv[q] = val; });
          else
            y = forward_any_const<R>(FAST ? kScreenFast : 1, v, dk, c1, y,
                                     [&](int q, double val) { cb[q * TI] = val; });
        } else if constexpr (FAST) {
          if (flow)
            y = forward_fast<R>(v, cf, y, [&](int q, double val) { yv[q] = val; });
          else
            y = forward_fast<R>(v, cf, y, [&](int q, double val) { cb[q * TI] = val; });
        } else {
          if (flow)
            y = forward_bare<R>(v, cf, c1, y, [&](int q, double val) { yv[q] = val; });
          else
            y = forward_bare<R>(v, cf, c1, y, [&](int q, double val) { cb[q * TI] = val; });
          hwmin = min(hwmin, batch_min_hi<R>(v));
        }
      } else if (flow) {
#pragma unroll
        for (int q = 0; q < R; ++q) yv[q] = 0.0;  // lanes with no line: anything, never read
      }
      if (flow) {
        __syncwarp();
        tmem_st16d(tbase + 32u * c, yv);
        __syncwarp();  // every lane has read the slot
        // refill it with the input KF chunks on: of this tile, or the next
        if (c == T - KF && NR == 0) take_next();
        const int cn = c + KF;
        if (cn < T)
          issue(i0, m, s, pk, cn, sl, fpar ^ 1u);
        else if (NR == 0 && nxt < ntiles)
          issue(ni0, nm_, ns_, np_, cn - T, sl, fpar ^ 1u);
        if (++fsl == KF) {
          fsl = 0;
          fpar ^= 1u;
        }
      }
    };
    if (edge_tile) {
      for (int c = 0; c < C; ++c) fwd_chunk(std::false_type{}, true, c);
    } else {
      for (int c = 0; c < C; ++c) {
        if (c >= k0 && c <= k1)
          fwd_chunk(std::true_type{}, false, c);
        else
          fwd_chunk(std::false_type{}, false, c);
      }
    }
    __syncwarp();
    if constexpr (TM) tmem_wait_st();
    if (!__all_sync(kAll, ok)) {
      if (t == 0) atomicExch(p.status, kDevTimeout);
      return;
    }
    // The screen, once per tile: a line with an input below 2^-960 (or
    // negative) anywhere is redone from its inputs, which are still in the
    // field (this tile's results are stored only by the back substitution).
    if (!FAST && __any_sync(kAll, !screen_clean(screen, hwmin))) {
      y = -0.0;
      for (int c = 0; c < C; ++c) {
        const int rb = c * CH;
        double v[R];
        DR cfr[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          v[q] = (lane_on && rb + q < n) ? out[static_cast<size_t>(rb + q) * g.row_stride] : 1.0;
          cfr[q] = __ldg(drp + rb + q);
        }
        if (MODE == 1 || (MODE == 2 && c < T)) {
          double yv[R];
#pragma unroll
          for (int q = 0; q < R; ++q) yv[q] = 0.0;
          if (lane_on) y = forward_checked<R>(v, cfr, c1, y, [&](int q, double val) { yv[q] = val; });
          __syncwarp();
          tmem_st16d(tbase + 32u * c, yv);
        } else if (lane_on) {
          double* cb = slots + static_cast<size_t>(rslot(flip, c)) * kSlotElems + t;
          y = forward_checked<R>(v, cfr, c1, y, [&](int q, double val) { cb[q * TI] = val; });
        }
      }
      __syncwarp();
      if constexpr (TM) tmem_wait_st();
      __syncwarp();
    }
    if (NR > 0) {
      take_next();
      // the next tile's first inputs take the (now idle) input slots
      if (TM && nxt < ntiles) {
        for (int c = 0; c < KF; ++c) {
          issue(ni0, nm_, ns_, np_, c, fsl, fpar);
          if (++fsl == KF) {
            fsl = 0;
            fpar ^= 1u;
          }
        }
        // the consume cursor returns to where those loads start
        for (int c = 0; c < KF; ++c) {
          if (fsl == 0) {
            fsl = KF - 1;
            fpar ^= 1u;
          } else {
            --fsl;
          }
        }
      }
    }

    // ---- back substitution, last chunk first; results to the field ----
    double xn = -0.0;
    uint32_t tr[32];  // TMEM chunks: the next chunk's forward results, loading
    if constexpr (TM) {
      __syncwarp();
      tmem_ld32_issue(tbase + 32u * (T - 1), tr);
    }
    auto back_chunk = [&](auto kconst, bool edge, int c) {
      constexpr bool K = decltype(kconst)::value;
      const int rb = c * CH;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      double v[R];
      if (flow) {
        __syncwarp();
        tmem_wait_ld32(tr);
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = __hiloint2double(static_cast<int>(tr[2 * q + 1]), static_cast<int>(tr[2 * q]));
        if (c > 0) tmem_ld32_issue(tbase + 32u * (c - 1), tr);
      } else {
        const double* cb = slots + static_cast<size_t>(rslot(flip, c)) * kSlotElems + t;
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
      }
      if (!edge || lane_on) {
        double cw[R];
        if constexpr (K) {
#pragma unroll
          for (int q = 0; q < R; ++q) cw[q] = ck;
        } else {
          const double2* cwp = reinterpret_cast<const double2*>(cus + rb);  // 16-byte pairs
#pragma unroll
          for (int q = 0; q < R / 2; ++q) {
            const double2 pr = cwp[q];
            cw[2 * q] = pr.x;
            cw[2 * q + 1] = pr.y;
          }
        }
        double* o = out + static_cast<size_t>(rb) * g.row_stride;
        if (c == C - 1 || (act && c == 0)) {
          // the line's end: rows past n are fill; an activated substrate's
          // first and last rows keep their pinned input
          const int r_lo = (act && c == 0) ? 1 : 0;
          const int r_hi = min(R, n - rb - ((act && c == C - 1) ? 1 : 0));
#pragma unroll
          for (int q = R - 1; q >= 0; --q) {
            if (rb + q < n) {
              xn = back_elem(cw[q], xn, v[q]);
              if (q >= r_lo && q < r_hi) o[q * g.row_stride] = xn;
            }
          }
        } else {
#pragma unroll
          for (int q = R - 1; q >= 0; --q) {
            xn = back_elem(cw[q], xn, v[q]);
            o[q * g.row_stride] = xn;
          }
        }
      }
      if (!flow) {
        fence_async_smem();  // this lane's forward results in the slot precede the refill
        __syncwarp();        // every lane has read the slot
        // the next tile's resident chunk for this slot (slot order flips)
        if (nxt < ntiles) issue(ni0, nm_, ns_, np_, T + (NR - 1 - (c - T)), rslot(flip, c), (k + 1) & 1u);
      }
    };
    if (edge_tile) {
      for (int c = C - 1; c >= 0; --c) back_chunk(std::false_type{}, true, c);
    } else {
      for (int c = C - 1; c >= 0; --c) {
        if (c >= k0 && c <= k1)
          back_chunk(std::true_type{}, false, c);
        else
          back_chunk(std::false_type{}, false, c);
      }
    }
    tile = nxt;
    ti0 = ni0;
    tm_ = nm_;
    ts = ns_;
    tp = np_;
  }
}

// FAST: the short FP64 chain (SweepParams::screen == kScreenFast), compiled
// apart from the reference-exact one so that each carries one chain; STAGED:
// the forward pairs staged per ring (stage_dr); LONG: lines of more than
// kTmemMaxChunks chunks (TMEM rings with resident chunks).  Each kernel holds
// the two ring bodies it runs and no others.
template <int AXIS, bool FAST, bool STAGED, bool LONG>
__global__ void __launch_bounds__(32 * (kTmemRingSmem + kTmemRingTmem), 1)
    sweep_yz_tmem_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap pmap,
                         const SweepParams<double> p, uint32_t smem_ring_bytes, uint32_t tmem_ring_bytes, int kf,
                         int ns, int stage_dr, int pw) {
  constexpr int CH = kRingRows;
  constexpr int TI = 32;
  constexpr int kSlotElems = CH * TI;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 128);
  YzShape g;
  g.nx = p.nx;
  g.n = (AXIS == 1) ? p.ny : p.nz;
  g.nm = (AXIS == 1) ? p.nz : p.ny;  // the line's other coordinate (k for y, j for z)
  g.C = (g.n + CH - 1) / CH;
  yz_shape_tiles(g, pw, p.s_hi - p.s_lo);
  g.row_stride = (AXIS == 1) ? static_cast<size_t>(p.nxp) : static_cast<size_t>(p.nxp) * p.ny;
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int nt = static_cast<int>(blockDim.x >> 5) - ns;  // TMEM rings (warps ns..ns+nt-1)
  const bool tm = warp >= ns;
  unsigned char* rbase = tm ? base + static_cast<size_t>(ns) * smem_ring_bytes +
                                  static_cast<size_t>(warp - ns) * tmem_ring_bytes
                            : base + static_cast<size_t>(warp) * smem_ring_bytes;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + static_cast<size_t>(ns) * smem_ring_bytes +
                                                    static_cast<size_t>(nt) * tmem_ring_bytes);
  const int nslots = tm ? kf + g.C - min(g.C, kTmemMaxChunks) : g.C;
  // ring: [barriers] [slots] [upper diagonal] [forward pairs]
  uint64_t* full = reinterpret_cast<uint64_t*>(rbase);
  double* slots = reinterpret_cast<double*>(rbase + kTmemBarrierBytes);
  double* cus = slots + static_cast<size_t>(nslots) * kSlotElems;
  double2* drs = stage_dr ? reinterpret_cast<double2*>(cus + static_cast<size_t>(g.C) * CH) : nullptr;

  if (t == 0) {
    if (warp == 0) {
      prefetch_tmap(&map);
      if (pw > 0) prefetch_tmap(&pmap);
    }
    for (int c = 0; c < nslots; ++c) mbar_init(smem_u32(&full[c]), 1);
    fence_barrier_init();
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), 512);
    tmem_relinquish();
    tmem_fence_before();
  }
  __syncthreads();
  uint32_t pend = 0, ppar = 0;
  if (tm) {
    tmem_fence_after();
    const uint32_t tbase = *tmem_slot + (static_cast<uint32_t>(32 * (warp & 3)) << 16);
    yz_tmem_ring<AXIS, LONG ? 2 : 1, STAGED, FAST>(&map, &pmap, p, g, kf, full, slots, cus, drs, tbase, pend, ppar);
  } else {
    yz_tmem_ring<AXIS, 0, STAGED, FAST>(&map, &pmap, p, g, kf, full, slots, cus, drs, 0u, pend, ppar);
  }

  // Loads still in flight (only after a wait gave up) land before the CTA
  // ends; then TMEM is released.
  if (pend != 0) {
    for (int sl = 0; sl < nslots; ++sl)
      if ((pend >> sl) & 1u) mbar_wait(smem_u32(&full[sl]), (ppar >> sl) & 1u);
  }
  __syncwarp();
  if (tm) {
    tmem_wait_st();
    tmem_fence_before();
  }
  __syncthreads();
  if (warp == 0) {
    tmem_fence_after();
    tmem_dealloc(*tmem_slot, 512);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned long long* counter = p.tile_counter;
    if (atomicAdd(counter + 1, 1ull) == gridDim.x - 1) {
      counter[0] = 0;
      counter[1] = 0;
    }
  }
}

// x sweep, persistent, with tensor memory (FP64, agents in the standalone
// source kernel, lines of 2 to 46 chunks).  The same plan as the y/z TMEM
// sweep: one CTA per SM of ns shared-memory rings and nt <= 4 TMEM rings,
// each one warp issuing its own TMA loads, tiles handed out by the per-solve
// counter.  A tile is 32 consecutive x-lines of one substrate in row order
// (row k * ny + j, the planes being contiguous in the field), so tiles run on
// across the ends of y rows and only a substrate's last tile is partial (with
// tiles of 32 lines of one (k, s), 200 lines took 7 tiles, the last 8 lines
// wide, at the cost of 7 full ones: the recurrence is latency bound).  Chunk c
// is the 128-byte column [16c, 16c + 16) of the 32 lines, staged with the
// 128B swizzle by one 3-D box, and lane t owns row r0 + t.  A shared-memory
// ring stages the whole tile (forward results in place); a TMEM ring streams
// a line's first 16 chunks through kf input slots and keeps their forward
// results in its TMEM lanes, the chunks past 16 resident in shared-memory
// slots.  The back substitution leaves each chunk's results as 32 swizzled
// rows (in the slot, or in the TMEM ring's staging chunk), which leave in one
// bulk tensor store (rows past the substrate's last are clipped by the map).
constexpr int kXTmemBarrierBytes = 256;  // at the end of a ring

// The shape of one x persistent sweep, shared by its rings.
struct XShape {
  int nx, ny, nz, C;
  int rows;  // x-lines per substrate, ny * nz: row k * ny + j
  int ntj;   // 32-row tiles per substrate
  long long ntiles;
};

// MODE 0: shared-memory ring; 1: TMEM ring (C <= 16, its own staging
// chunk); 2: TMEM ring with the chunks past 16 resident in shared memory (the
// first input slot stages the TMEM chunks' results; the next tile's first
// inputs load after the back substitution).
template <int MODE, bool FAST>
__device__ __forceinline__ void x_tmem_ring(const CUtensorMap* map, const SweepParams<double>& p, const XShape& g,
                                            int KF, unsigned char* slots, uint64_t* full, double* cus,
                                            unsigned char* stage, uint32_t tbase, uint32_t& pend, uint32_t& ppar) {
  using DR = double2;
  constexpr int W = 16;  // doubles per 128-byte chunk row
  constexpr uint32_t kChunkBytes = 32u * 128u;
  constexpr unsigned kAll = 0xffffffffu;
  const int t = threadIdx.x & 31;
  const int nx = g.nx, ny = g.ny, nz = g.nz, C = g.C, ntj = g.ntj;
  const int S = p.S;
  const long long ntiles = g.ntiles;
  unsigned long long* counter = p.tile_counter;
  const int sw = t & 7;
  constexpr bool TM = MODE != 0;
  const int T = MODE == 0 ? 0 : (MODE == 1 ? C : kTmemMaxChunks);  // chunks kept in TMEM
  const int NR = MODE == 1 ? 0 : C - T;                             // chunks resident in shared memory
  const int RB = TM ? KF : 0;                                       // first resident slot
  auto rslot = [&](bool fl, int c) { return RB + ring_slot(fl, NR, c - T); };

  // a tile is 32 consecutive rows (k * ny + j) of one substrate
  auto decode = [&](long long tile, int& r0, int& s) {
    const int sg = static_cast<int>(tile / ntj);
    r0 = static_cast<int>(tile - static_cast<long long>(sg) * ntj) * 32;
    s = p.s_lo + sg;
  };
  auto grab = [&]() -> long long {
    long long v = 0;
    if (t == 0) {
      v = static_cast<long long>(atomicAdd(counter, 1ull));
      if (v > ntiles) v = ntiles;
    }
    return __shfl_sync(kAll, v, 0);
  };
  auto issue = [&](int r0, int s, int c, int sl, uint32_t par) {
    if (t == 0) {
      const uint32_t bar = smem_u32(&full[sl]);
      mbar_expect_tx(bar, kChunkBytes);
      tma_load_3d(smem_u32(slots + static_cast<size_t>(sl) * kChunkBytes), map, bar, c * W, r0, s);
    }
    pend |= 1u << sl;
    ppar = (ppar & ~(1u << sl)) | (par << sl);
  };

  bool ok = true;
  long long tile = grab();
  int tr0 = 0, ts = 0;
  if (tile < ntiles) {
    decode(tile, tr0, ts);
    for (int c = 0; c < (TM ? KF : 0); ++c) issue(tr0, ts, c, c, 0u);
    for (int c = T; c < C; ++c) issue(tr0, ts, c, rslot(false, c), 0u);
  }
  const int screen = p.screen;
  int staged_s = -1;
  // chunks kc0..kc1 of the staged substrate lie in its converged range
  // (AxisCoefs::conv): their forward pairs are dk and upper diagonals ck
  int kc0 = INT_MAX, kc1 = -1;
  DR dk = make_double2(0.0, 0.0);
  double ck = 0.0;
  int fsl = 0;
  uint32_t fpar = 0;
  for (uint32_t it = 0; tile < ntiles; ++it) {
    const int r0 = tr0, s = ts;
    const bool flip = (it & 1u) != 0;
    const int rl = r0 + t;  // this lane's line: row rl = k * ny + j
    const bool valid = rl < g.rows;
    const int k = valid ? rl / ny : 0;
    const int j = valid ? rl - k * ny : 0;
    const bool act = p.active[s] != 0;
    const bool face = act && (j == 0 || j == ny - 1 || k == 0 || k == nz - 1);
    const bool lane_on = valid && !face;
    const DR* __restrict__ drp = p.ax.dr + static_cast<size_t>(s) * p.ax.npad;
    const double c1 = p.c1[s];
    if (s != staged_s) {
      stage_row(cus, p.ax.cu + static_cast<size_t>(s) * p.ax.npad, C * W);
      kc0 = INT_MAX;
      kc1 = -1;
      if (p.ax.conv != nullptr && nx >= 3) {
        kc0 = (__ldg(p.ax.conv + s) + W - 1) / W;
        kc1 = (nx - 1) / W - 1;  // chunks ending at element nx - 2 or before
        dk = __ldg(drp + nx - 2);
        ck = __ldg(p.ax.cu + static_cast<size_t>(s) * p.ax.npad + nx - 2);
      }
      staged_s = s;
      __syncwarp();
    }
    double x0v = 0.0, x1v = 0.0;
    if (act && valid) {
      x0v = p.xface[(static_cast<size_t>(0 * S + s) * nz + k) * ny + j];
      x1v = p.xface[(static_cast<size_t>(1 * S + s) * nz + k) * ny + j];
    }
    const double* fv = nullptr;  // face lines: the face plane's row
    if (face && valid) {
      if (k == 0 || k == nz - 1)
        fv = p.zface + ((static_cast<size_t>(k == 0 ? 0 : 1) * S + s) * ny + j) * nx;
      else
        fv = p.yface + ((static_cast<size_t>(j == 0 ? 0 : 1) * S + s) * nz + k) * nx;
    }
    double* plane = p.f + (static_cast<size_t>(s) * nz + k) * ny * static_cast<size_t>(p.nxp);
    double y = -0.0;
    int hwmin = INT_MAX;
    const bool edge_tile = __any_sync(kAll, !lane_on);
    // constant-coefficient chunks of this tile (edge tiles read every chunk's)
    const int k0 = edge_tile ? INT_MAX : kc0, k1 = edge_tile ? -1 : kc1;
    long long nxt = ntiles;
    int nr0 = 0, ns_ = 0;
    auto take_next = [&]() {
      nxt = grab();
      if (nxt < ntiles) decode(nxt, nr0, ns_);
    };

    // ---- forward elimination ----
    // kconst: std::true_type for a chunk in the converged range
    auto fwd_chunk = [&](auto kconst, bool edge, int c) {
      constexpr bool K = decltype(kconst)::value;
      const int i0 = c * W;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      const int sl = flow ? fsl : rslot(flip, c);
      const uint32_t par = flow ? fpar : (it & 1u);
      // the chunk's forward pairs, loading while the slot's barrier is awaited
      DR cf[W];
      if constexpr (!K) {
#pragma unroll
        for (int q = 0; q < W; ++q) cf[q] = __ldg(drp + i0 + q);
      }
      if (ok) ok = mbar_wait(smem_u32(&full[sl]), par);
      pend &= ~(1u << sl);
      unsigned char* crow = slots + static_cast<size_t>(sl) * kChunkBytes + t * 128;
      double yv[W];
      if (!edge || lane_on) {
        double v[W];
        load_row<double, W>(crow, sw, v);
        if (act) {  // the pin before the sweep (uniform tests: the line's first and last chunk)
          if (i0 == 0) v[0] = x0v;
          if (nx - 1 < i0 + W) {
#pragma unroll
            for (int q = 0; q < W; ++q)
              if (i0 + q == nx - 1) v[q] = x1v;
          }
        }
        if (i0 + W > nx) {  // TMA fill past the line's end: any clean value, never stored
#pragma unroll
          for (int q = 0; q < W; ++q)
            if (i0 + q >= nx) v[q] = 1.0;
        }
        // the screen reads the inputs before the chain
        if constexpr (!FAST) hwmin = min(hwmin, batch_min_hi<W>(v));
        if constexpr (K) {
          if (flow) {
            y = forward_any_const<W>(FAST ? kScreenFast : 1, v, dk, c1, y, [&](int q, double val) { yv[q] = val; });
          } else {
            RowPut<double> put{crow, sw};
            y = forward_any_const<W>(FAST ? kScreenFast : 1, v, dk, c1, y, put);
          }
        } else {
          if (flow) {
            y = forward_any<W>(FAST ? kScreenFast : 1, v, cf, c1, y, [&](int q, double val) { yv[q] = val; });
          } else {
            RowPut<double> put{crow, sw};
            y = forward_any<W>(FAST ? kScreenFast : 1, v, cf, c1, y, put);
          }
        }
      } else if (flow) {
#pragma unroll
        for (int q = 0; q < W; ++q) yv[q] = 0.0;  // lanes with no line: anything, never read
      }
      if (flow) {
        __syncwarp();
        tmem_st16d(tbase + 32u * c, yv);
        __syncwarp();  // every lane has read the slot
        if (MODE == 1 && c == T - KF) take_next();
        const int cn = c + KF;
        if (cn < T)
          issue(r0, s, cn, sl, fpar ^ 1u);
        else if (MODE == 1 && nxt < ntiles)
          issue(nr0, ns_, cn - T, sl, fpar ^ 1u);
        if (++fsl == KF) {
          fsl = 0;
          fpar ^= 1u;
        }
      }
    };
    if (edge_tile) {
      for (int c = 0; c < C; ++c) fwd_chunk(std::false_type{}, true, c);
    } else {
      for (int c = 0; c < C; ++c) {
        if (c >= k0 && c <= k1)
          fwd_chunk(std::true_type{}, false, c);
        else
          fwd_chunk(std::false_type{}, false, c);
      }
    }
    __syncwarp();
    if constexpr (TM) tmem_wait_st();
    if (!__all_sync(kAll, ok)) {
      if (t == 0) atomicExch(p.status, kDevTimeout);
      return;
    }
    // The tile's screen: a line with an input below 2^-960 (or negative)
    // anywhere is redone from its inputs -- the field still holds them (this
    // tile's results are stored only by the back substitution) -- pinned as
    // above, with every numerator checked.
    if (!FAST && __any_sync(kAll, !screen_clean(screen, hwmin))) {
      const double* src = plane + static_cast<size_t>(lane_on ? j : 0) * p.nxp;
      y = -0.0;
      for (int c = 0; c < C; ++c) {
        const int i0 = c * W;
        double v[W];
        DR cfr[W];
#pragma unroll
        for (int q = 0; q < W; ++q) {
          v[q] = (lane_on && i0 + q < nx) ? src[i0 + q] : 1.0;
          cfr[q] = __ldg(drp + i0 + q);
        }
        if (act) {
#pragma unroll
          for (int q = 0; q < W; ++q) {
            if (i0 + q == 0) v[q] = x0v;
            if (i0 + q == nx - 1) v[q] = x1v;
          }
        }
        if (MODE == 1 || (MODE == 2 && c < T)) {
          double yv[W];
#pragma unroll
          for (int q = 0; q < W; ++q) yv[q] = 0.0;
          if (lane_on) y = forward_checked<W>(v, cfr, c1, y, [&](int q, double val) { yv[q] = val; });
          __syncwarp();
          tmem_st16d(tbase + 32u * c, yv);
        } else if (lane_on) {
          RowPut<double> put{slots + static_cast<size_t>(rslot(flip, c)) * kChunkBytes + t * 128, sw};
          y = forward_checked<W>(v, cfr, c1, y, put);
        }
      }
      __syncwarp();
      if constexpr (TM) tmem_wait_st();
      __syncwarp();
    }
    if (MODE != 1) take_next();

    // ---- back substitution, last chunk first; results to the field ----
    double xn = -0.0;
    uint32_t tr[32];
    if constexpr (TM) {
      __syncwarp();
      tmem_ld32_issue(tbase + 32u * (T - 1), tr);
    }
    int pend_refill = -1;  // a resident chunk whose slot waits for its store to be read
    auto refill = [&](int cc) {
      if (nxt < ntiles) issue(nr0, ns_, T + (NR - 1 - (cc - T)), rslot(flip, cc), (it + 1) & 1u);
    };
    auto back_chunk = [&](auto kconst, bool edge, int c) {
      constexpr bool K = decltype(kconst)::value;
      const int i0 = c * W;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      unsigned char* cbase = flow ? stage : slots + static_cast<size_t>(rslot(flip, c)) * kChunkBytes;
      unsigned char* crow = cbase + t * 128;
      double v[W];
      if (flow) {
        __syncwarp();
        tmem_wait_ld32(tr);
#pragma unroll
        for (int q = 0; q < W; ++q) v[q] = __hiloint2double(static_cast<int>(tr[2 * q + 1]), static_cast<int>(tr[2 * q]));
        if (c > 0) tmem_ld32_issue(tbase + 32u * (c - 1), tr);
      } else {
        load_row<double, W>(crow, sw, v);
      }
      if (edge && face) {
        if (fv != nullptr) {
#pragma unroll
          for (int q = 0; q < W; ++q) v[q] = (i0 + q < nx) ? fv[i0 + q] : 0.0;
        }
      } else if (!edge || valid) {
        double cw[W];
        if constexpr (K) {
#pragma unroll
          for (int q = 0; q < W; ++q) cw[q] = ck;
        } else {
          const double2* cwp = reinterpret_cast<const double2*>(cus + i0);  // 16-byte pairs
#pragma unroll
          for (int q = 0; q < W / 2; ++q) {
            const double2 pr = cwp[q];
            cw[2 * q] = pr.x;
            cw[2 * q + 1] = pr.y;
          }
        }
        if (i0 + W > nx) {
#pragma unroll
          for (int q = W - 1; q >= 0; --q) {
            if (i0 + q < nx) {
              xn = back_elem(cw[q], xn, v[q]);
              v[q] = xn;
            }
          }
        } else {
#pragma unroll
          for (int q = W - 1; q >= 0; --q) {
            xn = back_elem(cw[q], xn, v[q]);
            v[q] = xn;
          }
        }
        if (act) {  // the pin after the sweep
          if (i0 == 0) v[0] = x0v;
          if (nx - 1 < i0 + W) {
#pragma unroll
            for (int q = 0; q < W; ++q)
              if (i0 + q == nx - 1) v[q] = x1v;
          }
        }
      }
      if (flow) {
        // the staging chunk's previous bulk store has read it
        if (t == 0) tma_store_wait_read();
        __syncwarp();
        if (pend_refill >= 0) {  // every store has read its chunk: the waiting slot refills too
          refill(pend_refill);
          pend_refill = -1;
        }
      }
      store_row<double, W>(crow, sw, v);
      // The chunk goes out as it is staged, in one bulk tensor store (rows
      // past ny and columns past nx are clipped by the map).
      fence_async_smem();
      __syncwarp();
      if (t == 0) {
        tma_store_3d(map, smem_u32(cbase), i0, r0, s);
        tma_store_commit();
      }
      if (!flow) {
        // A slot refills once its store has read it: the previous resident
        // chunk's slot now (its store is done reading while this chunk's
        // stays in flight), this chunk's at the next one or after the tile.
        if (pend_refill >= 0) {
          if (t == 0) tma_store_wait_read_1();
          __syncwarp();
          refill(pend_refill);
        }
        pend_refill = c;
      }
    };
    if (edge_tile) {
      for (int c = C - 1; c >= 0; --c) back_chunk(std::false_type{}, true, c);
    } else {
      for (int c = C - 1; c >= 0; --c) {
        if (c >= k0 && c <= k1)
          back_chunk(std::true_type{}, false, c);
        else
          back_chunk(std::false_type{}, false, c);
      }
    }
    if (pend_refill >= 0) {
      if (t == 0) tma_store_wait_read();
      __syncwarp();
      refill(pend_refill);
    }
    if (MODE == 2 && nxt < ntiles) {
      // the next tile's first inputs take the input slots (the first of
      // which staged results just now: its store must have read it)
      if (t == 0) tma_store_wait_read();
      fence_async_smem();
      __syncwarp();
      for (int c = 0; c < KF; ++c) {
        issue(nr0, ns_, c, fsl, fpar);
        if (++fsl == KF) {
          fsl = 0;
          fpar ^= 1u;
        }
      }
      for (int c = 0; c < KF; ++c) {  // the consume cursor returns to the first of them
        if (fsl == 0) {
          fsl = KF - 1;
          fpar ^= 1u;
        } else {
          --fsl;
        }
      }
    }
    tile = nxt;
    tr0 = nr0;
    ts = ns_;
  }
}

// FAST: the short FP64 chain (SweepParams::screen == kScreenFast), compiled
// apart from the reference-exact one; OWN: lines of at most kTmemMaxChunks
// chunks (TMEM rings with their own staging chunk), else TMEM rings with
// resident chunks.
template <bool FAST, bool OWN>
__global__ void __launch_bounds__(32 * (kTmemRingSmem + kTmemRingTmem), 1)
    sweep_x_tmem_kernel(const __grid_constant__ CUtensorMap map, const SweepParams<double> p,
                        uint32_t smem_ring_bytes, uint32_t tmem_ring_bytes, int kf, int ns) {
  constexpr uint32_t kChunkBytes = 32u * 128u;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  XShape g;
  g.nx = p.nx;
  g.ny = p.ny;
  g.nz = p.nz;
  g.C = (g.nx + 15) / 16;
  g.rows = g.ny * g.nz;
  g.ntj = (g.rows + 31) / 32;
  g.ntiles = static_cast<long long>(g.ntj) * (p.s_hi - p.s_lo);
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int nt = static_cast<int>(blockDim.x >> 5) - ns;  // TMEM rings (warps ns..ns+nt-1)
  const bool tm = warp >= ns;
  unsigned char* rbase = tm ? base + static_cast<size_t>(ns) * smem_ring_bytes +
                                  static_cast<size_t>(warp - ns) * tmem_ring_bytes
                            : base + static_cast<size_t>(warp) * smem_ring_bytes;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + static_cast<size_t>(ns) * smem_ring_bytes +
                                                    static_cast<size_t>(nt) * tmem_ring_bytes);
  // ring: [slots (+ staging chunk)] [upper diagonal] [barriers]; a TMEM ring
  // over more than 16 chunks stages in its first input slot
  const bool own_stage = tm && g.C <= kTmemMaxChunks;
  const int nslots = tm ? kf + g.C - min(g.C, kTmemMaxChunks) : g.C;
  unsigned char* slots = rbase;
  unsigned char* stage = tm ? (own_stage ? rbase + static_cast<size_t>(nslots) * kChunkBytes : rbase) : nullptr;
  double* cus = reinterpret_cast<double*>(rbase + static_cast<size_t>(nslots + (own_stage ? 1 : 0)) * kChunkBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(cus) +
                                               static_cast<size_t>(g.C) * 16 * sizeof(double));

  if (t == 0) {
    if (warp == 0) prefetch_tmap(&map);
    for (int c = 0; c < nslots; ++c) mbar_init(smem_u32(&full[c]), 1);
    fence_barrier_init();
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), 512);
    tmem_relinquish();
    tmem_fence_before();
  }
  __syncthreads();
  uint32_t pend = 0, ppar = 0;
  if (tm) {
    tmem_fence_after();
    const uint32_t tbase = *tmem_slot + (static_cast<uint32_t>(32 * (warp & 3)) << 16);
    x_tmem_ring<OWN ? 1 : 2, FAST>(&map, p, g, kf, slots, full, cus, stage, tbase, pend, ppar);
  } else {
    x_tmem_ring<0, FAST>(&map, p, g, kf, slots, full, cus, nullptr, 0u, pend, ppar);
  }
  if (pend != 0) {
    for (int sl = 0; sl < nslots; ++sl)
      if ((pend >> sl) & 1u) mbar_wait(smem_u32(&full[sl]), (ppar >> sl) & 1u);
  }
  if (t == 0) tma_store_wait_read();  // this warp's bulk stores have read shared memory
  __syncwarp();
  if (tm) {
    tmem_wait_st();
    tmem_fence_before();
  }
  __syncthreads();
  if (warp == 0) {
    tmem_fence_after();
    tmem_dealloc(*tmem_slot, 512);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned long long* counter = p.tile_counter;
    if (atomicAdd(counter + 1, 1ull) == gridDim.x - 1) {
      counter[0] = 0;
      counter[1] = 0;
    }
  }
}

// ---- FP32 y/z sweep with tensor memory ----
//
// The FP32 form's y and z sweeps on the plan of the FP64 one above: values
// are stored in FP32 (rounded once, when stored) while the recurrence runs in
// FP64, exactly as the shared-memory ring sweep of bfvm_sweeps.cu computes
// them, so results are that sweep's bits.  An FP32 forward result takes one
// TMEM column, so a ring keeps its 16 chunks in 256 columns and two rings
// share each lane quarter (warps ns + r and ns + r + 4 take the quarter's two
// column halves): up to eight TMEM rings beside up to five shared-memory
// rings, 416 lines of 200 per SM where the shared-memory ring sweep holds 224.
constexpr int kTmemRingSmemF32 = 3;  // most shared-memory rings (warps 0..ns-1; 3 measured best of 0-5)
constexpr int kTmemRingTmemF32 = 8;  // most TMEM rings, two per lane quarter

template <int AXIS, int MODE, bool FAST>
__device__ __forceinline__ void yz_tmem_ring_f32(const CUtensorMap* map, const CUtensorMap* pmap, const SweepParams<float>& p,
                                                 const YzShape& g, int KF, uint64_t* full, float* slots, double* cus,
                                                 double* drs, uint32_t tbase, uint32_t& pend, uint32_t& ppar) {
  constexpr int R = kRowBatch;
  constexpr int CH = kRingRows;
  constexpr int TI = 32;
  constexpr int kSlotElems = CH * TI;
  constexpr uint32_t kSlotBytes = kSlotElems * sizeof(float);
  constexpr unsigned kAll = 0xffffffffu;
  const int t = threadIdx.x & 31;
  const int nx = g.nx, n = g.n, nm = g.nm, C = g.C, ntr = g.ntr;
  constexpr bool TM = MODE != 0;
  const int T = MODE == 0 ? 0 : (MODE == 1 ? C : kTmemMaxChunks);  // chunks kept in TMEM
  const int NR = MODE == 1 ? 0 : C - T;                             // chunks resident in shared memory
  const int RB = TM ? KF : 0;                                       // first resident slot
  const long long ntiles = g.ntiles;
  unsigned long long* counter = p.tile_counter;

  // tile -> (i0, m, s, packed): regular tiles first, then packed ones (m the
  // first plane of the group)
  auto decode = [&](long long tile, int& i0, int& m, int& s, bool& pk) {
    const int sg = static_cast<int>(tile / g.per_s);
    const long long r = tile - sg * g.per_s;
    s = p.s_lo + sg;
    pk = r >= g.nreg;
    if (pk) {
      m = static_cast<int>(r - g.nreg) * g.P;
      i0 = g.ntr * TI;
    } else {
      m = static_cast<int>(r / ntr);
      i0 = static_cast<int>(r - static_cast<long long>(m) * ntr) * TI;
    }
  };
  auto skip = [&](long long tile) {  // every line of the tile in an activated face: final already
    int i0, m, s;
    bool pk;
    decode(tile, i0, m, s, pk);
    return !pk && p.active[s] != 0 && (m == 0 || m == nm - 1);
  };
  auto grab = [&]() -> long long {
    long long v = 0;
    if (t == 0) {
      do {
        v = static_cast<long long>(atomicAdd(counter, 1ull));
      } while (v < ntiles && skip(v));
      if (v > ntiles) v = ntiles;
    }
    return __shfl_sync(kAll, v, 0);
  };
  auto issue = [&](int i0, int m, int s, bool pk, int c, int sl, uint32_t par) {
    if (t == 0) {
      const uint32_t bar = smem_u32(&full[sl]);
      mbar_expect_tx(bar, kSlotBytes);
      const uint32_t dst = smem_u32(slots + static_cast<size_t>(sl) * kSlotElems);
      if (pk)  // the packed map's dimensions: x, planes, rows along the line, substrate
        tma_load_4d(dst, pmap, bar, i0, m, c * CH, s);
      else if (AXIS == 1)
        tma_load_4d(dst, map, bar, i0, c * CH, m, s);
      else
        tma_load_4d(dst, map, bar, i0, m, c * CH, s);
    }
    pend |= 1u << sl;
    ppar = (ppar & ~(1u << sl)) | (par << sl);
  };
  auto rslot = [&](bool fl, int c) { return RB + ring_slot(fl, NR, c - T); };

  bool ok = true;
  long long tile = grab();
  int ti0 = 0, tm_ = 0, ts = 0;
  bool tp = false;
  if (tile < ntiles) {
    decode(tile, ti0, tm_, ts, tp);
    for (int c = 0; c < (TM ? KF : 0); ++c) issue(ti0, tm_, ts, tp, c, c, 0u);
    for (int c = T; c < C; ++c) issue(ti0, tm_, ts, tp, c, rslot(false, c), 0u);
  }
  int staged_s = -1;
  int fsl = 0;
  uint32_t fpar = 0;
  for (uint32_t k = 0; tile < ntiles; ++k) {
    const int i0 = ti0, m = tm_, s = ts;
    const bool pk = tp;
    const bool flip = (k & 1u) != 0;
    const bool act = p.active[s] != 0;
    // this lane's line (x = i, plane ml); lines in an activated face keep
    // their (pinned) input
    const int i = pk ? i0 + (t & (g.pw - 1)) : i0 + t;
    const int ml = pk ? m + (t >> g.pw_log) : m;
    const bool inr = i < nx && ml < nm;
    const bool face = act && (i == 0 || i == nx - 1 || ml == 0 || ml == nm - 1);
    const bool lane_on = !face && inr;
    const int mo = inr ? ml : m;  // in range for the address below
    const AxisCoefs<float>& ac = (AXIS == 1) ? p.ay : p.az;
    const double* __restrict__ drp = ac.dr + static_cast<size_t>(s) * ac.npad;  // RN(1/d)
    const double c1 = p.c1[s];
    const double shift = p.shift[s];
    if (s != staged_s) {
      stage_row(cus, ac.cu + static_cast<size_t>(s) * ac.npad, C * CH);
      if (drs) stage_row(drs, drp, (C + 1) * CH);  // RN(1/d), one chunk past the line
      staged_s = s;
      __syncwarp();
    }
    float* out = p.f + ((AXIS == 1) ? ((static_cast<size_t>(s) * p.nz + mo) * p.ny) * p.nxp
                                    : (static_cast<size_t>(s) * p.nz * p.ny + mo) * p.nxp) + (inr ? i : i0);
    auto load_cf = [&](int c, double (&cf)[R]) {
      if (drs) {
#pragma unroll
        for (int q = 0; q < R; ++q) cf[q] = drs[c * R + q];
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) cf[q] = __ldg(drp + c * R + q);
      }
    };
    double cf[R];
    load_cf(0, cf);
    double y = -0.0;
    const bool edge_tile = __any_sync(kAll, !lane_on);
    long long nxt = ntiles;
    int ni0 = 0, nm_ = 0, ns_ = 0;
    bool np_ = false;
    auto take_next = [&]() {
      nxt = grab();
      if (nxt < ntiles) decode(nxt, ni0, nm_, ns_, np_);
    };

    // ---- forward elimination (FP64 recurrence, results rounded to FP32) ----
    auto fwd_chunk = [&](bool edge, int c) {
      const int rb = c * CH;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      const int sl = flow ? fsl : rslot(flip, c);
      const uint32_t par = flow ? fpar : (k & 1u);
      if (ok) ok = mbar_wait(smem_u32(&full[sl]), par);
      pend &= ~(1u << sl);
      float* cb = slots + static_cast<size_t>(sl) * kSlotElems + t;
      float yv[R];
      if (!edge || lane_on) {
        float v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
        if (rb + R > n) {  // rows past the line's end (TMA fill): any clean value, never stored
#pragma unroll
          for (int q = 0; q < R; ++q)
            if (rb + q >= n) v[q] = 1.0f;
        }
        if (flow)
          y = forward_store<R>(v, cf, c1, shift, FAST ? kScreenFast : 0, y, [&](int q, float val) { yv[q] = val; });
        else
          y = forward_store<R>(v, cf, c1, shift, FAST ? kScreenFast : 0, y,
                               [&](int q, float val) { cb[q * TI] = val; });
      } else if (flow) {
#pragma unroll
        for (int q = 0; q < R; ++q) yv[q] = 0.0f;  // lanes with no line: anything, never read
      }
      if (flow) {
        __syncwarp();
        tmem_st16f(tbase + 16u * c, yv);
        __syncwarp();  // every lane has read the slot
        if (c == T - KF && NR == 0) take_next();
        const int cn = c + KF;
        if (cn < T)
          issue(i0, m, s, pk, cn, sl, fpar ^ 1u);
        else if (NR == 0 && nxt < ntiles)
          issue(ni0, nm_, ns_, np_, cn - T, sl, fpar ^ 1u);
        if (++fsl == KF) {
          fsl = 0;
          fpar ^= 1u;
        }
      }
      load_cf(c + 1, cf);
    };
    if (edge_tile) {
      for (int c = 0; c < C; ++c) fwd_chunk(true, c);
    } else {
      for (int c = 0; c < C; ++c) fwd_chunk(false, c);
    }
    __syncwarp();
    if constexpr (TM) tmem_wait_st();
    if (!__all_sync(kAll, ok)) {
      if (t == 0) atomicExch(p.status, kDevTimeout);
      return;
    }
    if (NR > 0) {
      take_next();
      if (TM && nxt < ntiles) {
        for (int c = 0; c < KF; ++c) {
          issue(ni0, nm_, ns_, np_, c, fsl, fpar);
          if (++fsl == KF) {
            fsl = 0;
            fpar ^= 1u;
          }
        }
        for (int c = 0; c < KF; ++c) {  // the consume cursor returns to where those loads start
          if (fsl == 0) {
            fsl = KF - 1;
            fpar ^= 1u;
          } else {
            --fsl;
          }
        }
      }
    }

    // ---- back substitution, last chunk first; results to the field ----
    double xn = -0.0;
    uint32_t tr[16];
    if constexpr (TM) {
      __syncwarp();
      tmem_ld16_issue(tbase + 16u * (T - 1), tr);
    }
    auto back_chunk = [&](bool edge, int c) {
      const int rb = c * CH;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      float v[R];
      if (flow) {
        __syncwarp();
        tmem_wait_ld16(tr);
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = __uint_as_float(tr[q]);
        if (c > 0) tmem_ld16_issue(tbase + 16u * (c - 1), tr);
      } else {
        const float* cb = slots + static_cast<size_t>(rslot(flip, c)) * kSlotElems + t;
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = cb[q * TI];
      }
      if (!edge || lane_on) {
        const double2* cwp = reinterpret_cast<const double2*>(cus + rb);  // 16-byte pairs
        double cw[R];
#pragma unroll
        for (int q = 0; q < R / 2; ++q) {
          const double2 pr = cwp[q];
          cw[2 * q] = pr.x;
          cw[2 * q + 1] = pr.y;
        }
        float* o = out + static_cast<size_t>(rb) * g.row_stride;
        if (c == C - 1 || (act && c == 0)) {
          // the line's end: rows past n are fill; an activated substrate's
          // first and last rows keep their pinned input
          const int r_lo = (act && c == 0) ? 1 : 0;
          const int r_hi = min(R, n - rb - ((act && c == C - 1) ? 1 : 0));
#pragma unroll
          for (int q = R - 1; q >= 0; --q) {
            if (rb + q < n) {
              xn = back_elem(cw[q], xn, static_cast<double>(v[q]));
              if (q >= r_lo && q < r_hi) o[q * g.row_stride] = static_cast<float>(xn);
            }
          }
        } else {
#pragma unroll
          for (int q = R - 1; q >= 0; --q) {
            xn = back_elem(cw[q], xn, static_cast<double>(v[q]));
            o[q * g.row_stride] = static_cast<float>(xn);
          }
        }
      }
      if (!flow) {
        __syncwarp();  // every lane has read the slot
        if (nxt < ntiles) issue(ni0, nm_, ns_, np_, T + (NR - 1 - (c - T)), rslot(flip, c), (k + 1) & 1u);
      }
    };
    if (edge_tile) {
      for (int c = C - 1; c >= 0; --c) back_chunk(true, c);
    } else {
      for (int c = C - 1; c >= 0; --c) back_chunk(false, c);
    }
    tile = nxt;
    ti0 = ni0;
    tm_ = nm_;
    ts = ns_;
    tp = np_;
  }
}

// FAST: the FP32 form's short chain (SweepParams::screen == kScreenFast),
// compiled apart from the default one.  (Compiling the two TMEM ring forms
// apart as well, as the FP64 kernels do, measured 3% slower here: cube200
// FP32 y/z 0.0789 against 0.0764 ms.)
template <int AXIS, bool FAST>
__global__ void __launch_bounds__(32 * (kTmemRingSmemF32 + kTmemRingTmemF32), 1)
    sweep_yz_tmem_f32_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ CUtensorMap pmap,
                             const SweepParams<float> p, uint32_t smem_ring_bytes, uint32_t tmem_ring_bytes, int kf,
                             int ns, int stage_dr, int pw) {
  constexpr int CH = kRingRows;
  constexpr int TI = 32;
  constexpr int kSlotElems = CH * TI;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 128);
  YzShape g;
  g.nx = p.nx;
  g.n = (AXIS == 1) ? p.ny : p.nz;
  g.nm = (AXIS == 1) ? p.nz : p.ny;
  g.C = (g.n + CH - 1) / CH;
  yz_shape_tiles(g, pw, p.s_hi - p.s_lo);
  g.row_stride = (AXIS == 1) ? static_cast<size_t>(p.nxp) : static_cast<size_t>(p.nxp) * p.ny;
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int nt = static_cast<int>(blockDim.x >> 5) - ns;  // TMEM rings (warps ns..ns+nt-1)
  const bool tm = warp >= ns;
  unsigned char* rbase = tm ? base + static_cast<size_t>(ns) * smem_ring_bytes +
                                  static_cast<size_t>(warp - ns) * tmem_ring_bytes
                            : base + static_cast<size_t>(warp) * smem_ring_bytes;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + static_cast<size_t>(ns) * smem_ring_bytes +
                                                    static_cast<size_t>(nt) * tmem_ring_bytes);
  const int nslots = tm ? kf + g.C - min(g.C, kTmemMaxChunks) : g.C;
  // ring: [barriers] [slots] [upper diagonal] [RN(1/d), when staged]
  uint64_t* full = reinterpret_cast<uint64_t*>(rbase);
  float* slots = reinterpret_cast<float*>(rbase + kTmemBarrierBytes);
  double* cus = reinterpret_cast<double*>(slots + static_cast<size_t>(nslots) * kSlotElems);
  double* drs = stage_dr ? cus + static_cast<size_t>(g.C) * CH : nullptr;

  if (t == 0) {
    if (warp == 0) {
      prefetch_tmap(&map);
      if (pw > 0) prefetch_tmap(&pmap);
    }
    for (int c = 0; c < nslots; ++c) mbar_init(smem_u32(&full[c]), 1);
    fence_barrier_init();
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), 512);
    tmem_relinquish();
    tmem_fence_before();
  }
  __syncthreads();
  uint32_t pend = 0, ppar = 0;
  if (tm) {
    tmem_fence_after();
    // lane quarter warp % 4; the second ring on a quarter takes columns 256..511
    const uint32_t half = static_cast<uint32_t>((warp - ns) >= 4 ? 256 : 0);
    const uint32_t tbase = *tmem_slot + (static_cast<uint32_t>(32 * (warp & 3)) << 16) + half;
    if (g.C <= kTmemMaxChunks)
      yz_tmem_ring_f32<AXIS, 1, FAST>(&map, &pmap, p, g, kf, full, slots, cus, drs, tbase, pend, ppar);
    else
      yz_tmem_ring_f32<AXIS, 2, FAST>(&map, &pmap, p, g, kf, full, slots, cus, drs, tbase, pend, ppar);
  } else {
    yz_tmem_ring_f32<AXIS, 0, FAST>(&map, &pmap, p, g, kf, full, slots, cus, drs, 0u, pend, ppar);
  }
  if (pend != 0) {
    for (int sl = 0; sl < nslots; ++sl)
      if ((pend >> sl) & 1u) mbar_wait(smem_u32(&full[sl]), (ppar >> sl) & 1u);
  }
  __syncwarp();
  if (tm) {
    tmem_wait_st();
    tmem_fence_before();
  }
  __syncthreads();
  if (warp == 0) {
    tmem_fence_after();
    tmem_dealloc(*tmem_slot, 512);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned long long* counter = p.tile_counter;
    if (atomicAdd(counter + 1, 1ull) == gridDim.x - 1) {
      counter[0] = 0;
      counter[1] = 0;
    }
  }
}

// ---- FP32 x sweep with tensor memory ----
//
// The FP64 x sweep's plan above for the FP32 form: values stored in FP32,
// the recurrence in FP64, the pins and face values as the per-tile FP32 x
// sweep of bfvm_sweeps.cu applies them, so results are its bits.  Tiles are
// 32 consecutive rows (k * ny + j) of one substrate, as in the FP64 sweep.  A
// chunk is the 128-byte column [32c, 32c + 32) of the tile's 32 lines; its forward
// results take 32 TMEM columns, so a ring keeps 8 chunks (lines of up to 256)
// in 256 columns and two rings share each lane quarter.
constexpr int kXTmemRingSmemF32 = 0;   // shared-memory rings (none: measured slower, see use_tmem_x_f32)
constexpr int kXTmemRingTmemF32 = 8;   // most TMEM rings, two per lane quarter
constexpr int kXTmemMaxChunksF32 = 8;  // chunks of a TMEM ring in its 256 columns

// STAGED: RN(1/d) read from the ring's copy `drs` in shared memory, else
// from global memory.
template <int MODE, bool STAGED, bool FAST>
__device__ __forceinline__ void x_tmem_ring_f32(const CUtensorMap* map, const SweepParams<float>& p,
                                                const XShape& g, int KF, unsigned char* slots, uint64_t* full,
                                                double* cus, double* drs, unsigned char* stage, uint32_t tbase,
                                                uint32_t& pend, uint32_t& ppar) {
  constexpr int W = 32;  // floats per 128-byte chunk row
  constexpr uint32_t kChunkBytes = 32u * 128u;
  constexpr unsigned kAll = 0xffffffffu;
  const int t = threadIdx.x & 31;
  const int nx = g.nx, ny = g.ny, nz = g.nz, C = g.C, ntj = g.ntj;
  const int S = p.S;
  const long long ntiles = g.ntiles;
  unsigned long long* counter = p.tile_counter;
  const int sw = t & 7;
  constexpr bool TM = MODE != 0;
  const int T = MODE == 0 ? 0 : (MODE == 1 ? C : kXTmemMaxChunksF32);  // chunks kept in TMEM
  const int NR = MODE == 1 ? 0 : C - T;                                 // chunks resident in shared memory
  const int RB = TM ? KF : 0;                                           // first resident slot
  auto rslot = [&](bool fl, int c) { return RB + ring_slot(fl, NR, c - T); };

  // a tile is 32 consecutive rows (k * ny + j) of one substrate
  auto decode = [&](long long tile, int& r0, int& s) {
    const int sg = static_cast<int>(tile / ntj);
    r0 = static_cast<int>(tile - static_cast<long long>(sg) * ntj) * 32;
    s = p.s_lo + sg;
  };
  auto grab = [&]() -> long long {
    long long v = 0;
    if (t == 0) {
      v = static_cast<long long>(atomicAdd(counter, 1ull));
      if (v > ntiles) v = ntiles;
    }
    return __shfl_sync(kAll, v, 0);
  };
  auto issue = [&](int r0, int s, int c, int sl, uint32_t par) {
    if (t == 0) {
      const uint32_t bar = smem_u32(&full[sl]);
      mbar_expect_tx(bar, kChunkBytes);
      tma_load_3d(smem_u32(slots + static_cast<size_t>(sl) * kChunkBytes), map, bar, c * W, r0, s);
    }
    pend |= 1u << sl;
    ppar = (ppar & ~(1u << sl)) | (par << sl);
  };

  bool ok = true;
  long long tile = grab();
  int tr0 = 0, ts = 0;
  if (tile < ntiles) {
    decode(tile, tr0, ts);
    for (int c = 0; c < (TM ? KF : 0); ++c) issue(tr0, ts, c, c, 0u);
    for (int c = T; c < C; ++c) issue(tr0, ts, c, rslot(false, c), 0u);
  }
  int staged_s = -1;
  int fsl = 0;
  uint32_t fpar = 0;
  for (uint32_t it = 0; tile < ntiles; ++it) {
    const int r0 = tr0, s = ts;
    const bool flip = (it & 1u) != 0;
    const int rl = r0 + t;  // this lane's line: row rl = k * ny + j
    const bool valid = rl < g.rows;
    const int k = valid ? rl / ny : 0;
    const int j = valid ? rl - k * ny : 0;
    const bool act = p.active[s] != 0;
    const bool face = act && (j == 0 || j == ny - 1 || k == 0 || k == nz - 1);
    const bool lane_on = valid && !face;
    const double* __restrict__ drp = p.ax.dr + static_cast<size_t>(s) * p.ax.npad;  // RN(1/d)
    const double c1 = p.c1[s];
    const double shift = p.shift[s];
    const double off = p.off[s];
    if (s != staged_s) {
      stage_row(cus, p.ax.cu + static_cast<size_t>(s) * p.ax.npad, C * W);
      if (STAGED) stage_row(drs, drp, (C + 1) * W);  // RN(1/d), one chunk past the line (the prefetch)
      staged_s = s;
      __syncwarp();
    }
    float x0v = 0.0f, x1v = 0.0f;
    if (act && valid) {
      x0v = static_cast<float>(p.xface[(static_cast<size_t>(0 * S + s) * nz + k) * ny + j] - off);
      x1v = static_cast<float>(p.xface[(static_cast<size_t>(1 * S + s) * nz + k) * ny + j] - off);
    }
    const double* fv = nullptr;  // face lines: the face plane's row
    if (face && valid) {
      if (k == 0 || k == nz - 1)
        fv = p.zface + ((static_cast<size_t>(k == 0 ? 0 : 1) * S + s) * ny + j) * nx;
      else
        fv = p.yface + ((static_cast<size_t>(j == 0 ? 0 : 1) * S + s) * nz + k) * nx;
    }
    double cf[16];  // the coefficients RN(1/d) of the next 16 values
#pragma unroll
    for (int q = 0; q < 16; ++q) cf[q] = STAGED ? drs[q] : __ldg(drp + q);
    double y = -0.0;
    const bool edge_tile = __any_sync(kAll, !lane_on);
    long long nxt = ntiles;
    int nr0 = 0, ns_ = 0;
    auto take_next = [&]() {
      nxt = grab();
      if (nxt < ntiles) decode(nxt, nr0, ns_);
    };

    // ---- forward elimination (FP64 recurrence, results rounded to FP32) ----
    // A chunk row is handled as two halves of 16 values (units 4h .. 4h+3 of
    // the swizzled row, TMEM columns 32c + 16h ..), which keeps the
    // registers of one half live at a time.
    auto fwd_chunk = [&](bool edge, int c) {
      const int i0 = c * W;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      const int sl = flow ? fsl : rslot(flip, c);
      const uint32_t par = flow ? fpar : (it & 1u);
      if (ok) ok = mbar_wait(smem_u32(&full[sl]), par);
      pend &= ~(1u << sl);
      unsigned char* crow = slots + static_cast<size_t>(sl) * kChunkBytes + t * 128;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e0 = i0 + 16 * h;
        float yh[16];
        if (!edge || lane_on) {
          float vh[16];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float4 f4 = *reinterpret_cast<const float4*>(crow + (((4 * h + u) ^ sw) << 4));
            vh[4 * u] = f4.x;
            vh[4 * u + 1] = f4.y;
            vh[4 * u + 2] = f4.z;
            vh[4 * u + 3] = f4.w;
          }
          if (act) {  // the pin before the sweep
            if (e0 == 0) vh[0] = x0v;
            if (e0 <= nx - 1 && nx - 1 < e0 + 16) {
#pragma unroll
              for (int q = 0; q < 16; ++q)
                if (e0 + q == nx - 1) vh[q] = x1v;
            }
          }
          if (flow) {
            y = forward_store<16>(vh, cf, c1, shift, FAST ? kScreenFast : 0, y, [&](int q, float val) { yh[q] = val; });
          } else {
            RowPut<float> put{crow, sw};
            y = forward_store<16>(vh, cf, c1, shift, FAST ? kScreenFast : 0, y,
                                  [&](int q, float val) { put(16 * h + q, val); });
          }
        } else if (flow) {
#pragma unroll
          for (int q = 0; q < 16; ++q) yh[q] = 0.0f;  // lanes with no line: anything, never read
        }
        if (flow) {
          __syncwarp();
          tmem_st16f(tbase + 32u * c + 16u * h, yh);
        }
        // the next half's coefficients (rows are padded past the line)
#pragma unroll
        for (int q = 0; q < 16; ++q) cf[q] = STAGED ? drs[e0 + 16 + q] : __ldg(drp + e0 + 16 + q);
      }
      if (flow) {
        __syncwarp();  // every lane has read the slot
        if (MODE == 1 && c == T - KF) take_next();
        const int cn = c + KF;
        if (cn < T)
          issue(r0, s, cn, sl, fpar ^ 1u);
        else if (MODE == 1 && nxt < ntiles)
          issue(nr0, ns_, cn - T, sl, fpar ^ 1u);
        if (++fsl == KF) {
          fsl = 0;
          fpar ^= 1u;
        }
      }
    };
    if (edge_tile) {
      for (int c = 0; c < C; ++c) fwd_chunk(true, c);
    } else {
      for (int c = 0; c < C; ++c) fwd_chunk(false, c);
    }
    __syncwarp();
    if constexpr (TM) tmem_wait_st();
    if (!__all_sync(kAll, ok)) {
      if (t == 0) atomicExch(p.status, kDevTimeout);
      return;
    }
    if (MODE != 1) take_next();

    // ---- back substitution, last chunk first, upper half first; results to the field ----
    double xn = -0.0;
    uint32_t tr[16];  // TMEM chunks: the next half's forward results, loading
    if constexpr (TM) {
      __syncwarp();
      tmem_ld16_issue(tbase + 32u * (T - 1) + 16u, tr);
    }
    int pend_refill = -1;  // a resident chunk whose slot waits for its store to be read
    auto refill = [&](int cc) {
      if (nxt < ntiles) issue(nr0, ns_, T + (NR - 1 - (cc - T)), rslot(flip, cc), (it + 1) & 1u);
    };
    auto back_chunk = [&](bool edge, int c) {
      const int i0 = c * W;
      const bool flow = MODE == 1 || (MODE == 2 && c < T);
      unsigned char* cbase = flow ? stage : slots + static_cast<size_t>(rslot(flip, c)) * kChunkBytes;
      unsigned char* crow = cbase + t * 128;
      if (flow) {
        // the staging chunk's previous bulk store has read it
        if (t == 0) tma_store_wait_read();
        __syncwarp();
        if (pend_refill >= 0) {  // every store has read its chunk: the waiting slot refills too
          refill(pend_refill);
          pend_refill = -1;
        }
      }
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int h = 1 - hh;
        const int e0 = i0 + 16 * h;
        float vh[16];
        if (flow) {
          __syncwarp();
          tmem_wait_ld16(tr);
#pragma unroll
          for (int q = 0; q < 16; ++q) vh[q] = __uint_as_float(tr[q]);
          if (h == 1)
            tmem_ld16_issue(tbase + 32u * c, tr);
          else if (c > 0)
            tmem_ld16_issue(tbase + 32u * (c - 1) + 16u, tr);
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float4 f4 = *reinterpret_cast<const float4*>(crow + (((4 * h + u) ^ sw) << 4));
            vh[4 * u] = f4.x;
            vh[4 * u + 1] = f4.y;
            vh[4 * u + 2] = f4.z;
            vh[4 * u + 3] = f4.w;
          }
        }
        if (edge && face) {
          if (fv != nullptr) {
#pragma unroll
            for (int q = 0; q < 16; ++q) vh[q] = (e0 + q < nx) ? static_cast<float>(fv[e0 + q] - off) : 0.0f;
          }
        } else if (!edge || valid) {
          const double2* cwp = reinterpret_cast<const double2*>(cus + e0);  // 16-byte pairs
          if (e0 + 16 > nx) {
#pragma unroll
            for (int g2 = 7; g2 >= 0; --g2) {
              const double2 pr = cwp[g2];
              if (e0 + 2 * g2 + 1 < nx) {
                xn = back_elem(pr.y, xn, static_cast<double>(vh[2 * g2 + 1]));
                vh[2 * g2 + 1] = static_cast<float>(xn);
              }
              if (e0 + 2 * g2 < nx) {
                xn = back_elem(pr.x, xn, static_cast<double>(vh[2 * g2]));
                vh[2 * g2] = static_cast<float>(xn);
              }
            }
          } else {
#pragma unroll
            for (int g2 = 7; g2 >= 0; --g2) {
              const double2 pr = cwp[g2];
              xn = back_elem(pr.y, xn, static_cast<double>(vh[2 * g2 + 1]));
              vh[2 * g2 + 1] = static_cast<float>(xn);
              xn = back_elem(pr.x, xn, static_cast<double>(vh[2 * g2]));
              vh[2 * g2] = static_cast<float>(xn);
            }
          }
          if (act) {  // the pin after the sweep
            if (e0 == 0) vh[0] = x0v;
            if (e0 <= nx - 1 && nx - 1 < e0 + 16) {
#pragma unroll
              for (int q = 0; q < 16; ++q)
                if (e0 + q == nx - 1) vh[q] = x1v;
            }
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          *reinterpret_cast<float4*>(crow + (((4 * h + u) ^ sw) << 4)) =
              make_float4(vh[4 * u], vh[4 * u + 1], vh[4 * u + 2], vh[4 * u + 3]);
      }
      // the chunk goes out as it is staged (rows past ny, columns past nx clipped)
      fence_async_smem();
      __syncwarp();
      if (t == 0) {
        tma_store_3d(map, smem_u32(cbase), i0, r0, s);
        tma_store_commit();
      }
      if (!flow) {
        // A slot refills once its store has read it: the previous resident
        // chunk's slot now (its store is done reading while this chunk's
        // stays in flight), this chunk's at the next one or after the tile.
        if (pend_refill >= 0) {
          if (t == 0) tma_store_wait_read_1();
          __syncwarp();
          refill(pend_refill);
        }
        pend_refill = c;
      }
    };
    if (edge_tile) {
      for (int c = C - 1; c >= 0; --c) back_chunk(true, c);
    } else {
      for (int c = C - 1; c >= 0; --c) back_chunk(false, c);
    }
    if (pend_refill >= 0) {
      if (t == 0) tma_store_wait_read();
      __syncwarp();
      refill(pend_refill);
    }
    if (MODE == 2 && nxt < ntiles) {
      // the next tile's first inputs take the input slots (the first of
      // which staged results just now: its store must have read it)
      if (t == 0) tma_store_wait_read();
      fence_async_smem();
      __syncwarp();
      for (int c = 0; c < KF; ++c) {
        issue(nr0, ns_, c, fsl, fpar);
        if (++fsl == KF) {
          fsl = 0;
          fpar ^= 1u;
        }
      }
      for (int c = 0; c < KF; ++c) {  // the consume cursor returns to the first of them
        if (fsl == 0) {
          fsl = KF - 1;
          fpar ^= 1u;
        } else {
          --fsl;
        }
      }
    }
    tile = nxt;
    tr0 = nr0;
    ts = ns_;
  }
}

// FAST: the FP32 form's short chain, compiled apart from the default one;
// STAGED: RN(1/d) staged per ring (stage_dr); OWN: lines of at most
// kXTmemMaxChunksF32 chunks.
template <bool FAST, bool STAGED, bool OWN>
__global__ void __launch_bounds__(32 * (kXTmemRingSmemF32 + kXTmemRingTmemF32), 1)
    sweep_x_tmem_f32_kernel(const __grid_constant__ CUtensorMap map, const SweepParams<float> p,
                            uint32_t smem_ring_bytes, uint32_t tmem_ring_bytes, int kf, int ns, int stage_dr) {
  constexpr uint32_t kChunkBytes = 32u * 128u;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + smem_align_pad(smem_raw, 1024);
  XShape g;
  g.nx = p.nx;
  g.ny = p.ny;
  g.nz = p.nz;
  g.C = (g.nx + 31) / 32;
  g.rows = g.ny * g.nz;
  g.ntj = (g.rows + 31) / 32;
  g.ntiles = static_cast<long long>(g.ntj) * (p.s_hi - p.s_lo);
  const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
  const int nt = static_cast<int>(blockDim.x >> 5) - ns;  // TMEM rings (warps ns..ns+nt-1)
  const bool tm = warp >= ns;
  unsigned char* rbase = tm ? base + static_cast<size_t>(ns) * smem_ring_bytes +
                                  static_cast<size_t>(warp - ns) * tmem_ring_bytes
                            : base + static_cast<size_t>(warp) * smem_ring_bytes;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + static_cast<size_t>(ns) * smem_ring_bytes +
                                                    static_cast<size_t>(nt) * tmem_ring_bytes);
  // ring: [slots (+ staging chunk)] [upper diagonal] [RN(1/d) when staged]
  // [barriers]; a TMEM ring over more than 8 chunks stages in its first input slot
  const bool own_stage = tm && g.C <= kXTmemMaxChunksF32;
  const int nslots = tm ? kf + g.C - min(g.C, kXTmemMaxChunksF32) : g.C;
  unsigned char* slots = rbase;
  unsigned char* stage = tm ? (own_stage ? rbase + static_cast<size_t>(nslots) * kChunkBytes : rbase) : nullptr;
  double* cus = reinterpret_cast<double*>(rbase + static_cast<size_t>(nslots + (own_stage ? 1 : 0)) * kChunkBytes);
  // RN(1/d) of (C + 1) chunks when staged, then the barriers
  double* drs = stage_dr ? cus + static_cast<size_t>(g.C) * 32 : nullptr;
  uint64_t* full =
      reinterpret_cast<uint64_t*>(cus + static_cast<size_t>(g.C) * 32 + (stage_dr ? (g.C + 1) * 32 : 0));

  if (t == 0) {
    if (warp == 0) prefetch_tmap(&map);
    for (int c = 0; c < nslots; ++c) mbar_init(smem_u32(&full[c]), 1);
    fence_barrier_init();
  }
  __syncwarp();
  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), 512);
    tmem_relinquish();
    tmem_fence_before();
  }
  __syncthreads();
  uint32_t pend = 0, ppar = 0;
  if (tm) {
    tmem_fence_after();
    // lane quarter warp % 4; the second ring on a quarter takes columns 256..511
    const uint32_t half = static_cast<uint32_t>((warp - ns) >= 4 ? 256 : 0);
    const uint32_t tbase = *tmem_slot + (static_cast<uint32_t>(32 * (warp & 3)) << 16) + half;
    x_tmem_ring_f32<OWN ? 1 : 2, STAGED, FAST>(&map, p, g, kf, slots, full, cus, drs, stage, tbase, pend, ppar);
  } else {
    // no shared-memory rings are planned (kXTmemRingSmemF32 = 0); kept for the plan's range
    x_tmem_ring_f32<0, false, FAST>(&map, p, g, kf, slots, full, cus, drs, nullptr, 0u, pend, ppar);
  }
  if (pend != 0) {
    for (int sl = 0; sl < nslots; ++sl)
      if ((pend >> sl) & 1u) mbar_wait(smem_u32(&full[sl]), (ppar >> sl) & 1u);
  }
  if (t == 0) tma_store_wait_read();  // this warp's bulk stores have read shared memory
  __syncwarp();
  if (tm) {
    tmem_wait_st();
    tmem_fence_before();
  }
  __syncthreads();
  if (warp == 0) {
    tmem_fence_after();
    tmem_dealloc(*tmem_slot, 512);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned long long* counter = p.tile_counter;
    if (atomicAdd(counter + 1, 1ull) == gridDim.x - 1) {
      counter[0] = 0;
      counter[1] = 0;
    }
  }
}

// ---- launch policy ----

// The TMEM sweeps hand tiles out at run time, so fewer per ring still balance.
constexpr long long kTmemMinTilesPerRing = 2;

// One ring of the TMEM x sweep (a multiple of 1024 bytes, so every chunk
// stays on the 128B-swizzle atom): shared-memory ring = C chunks; TMEM ring
// = kf input chunks and a staging chunk, or, past 16 chunks, kf input chunks
// and a resident chunk for each chunk past 16; then the upper diagonal and
// the barriers.
static size_t x_tmem_ring_bytes(int nx, bool tm, int kf) {
  const int C = (nx + 15) / 16;
  const int chunks = !tm ? C : (C <= kTmemMaxChunks ? kf + 1 : kf + C - kTmemMaxChunks);
  const size_t b = static_cast<size_t>(chunks) * 32 * 128 + static_cast<size_t>(C) * 16 * 8 + kXTmemBarrierBytes;
  return (b + 1023) / 1024 * 1024;
}

static size_t x_tmem_smem(int nx, int ns, int nt, int kf) {
  // alignment pad, the rings, the TMEM address word
  return 1024 + ns * x_tmem_ring_bytes(nx, false, kf) + nt * x_tmem_ring_bytes(nx, true, kf) + 128;
}

// The TMEM x sweep applies (FP64, agents not fused, 32-line tiles, lines of
// at least 2 chunks and at most 32 slots per ring): by default on lines of
// at least 3 chunks (33 voxels), at sweep TMEM level 2 from 2 chunks.  *ns
// shared-memory rings and *nt TMEM rings (the most that fit), *kf input
// slots per TMEM ring.  Each finished chunk leaves by one bulk tensor store
// from its staging chunk; measured on B200 at cube200 (200^3 x 4) against
// the per-tile x sweep: 0.149 against 0.190 ms (the earlier transposed
// write-out through global stores took 0.198).
static bool use_tmem_x(int eb, int nx, bool fused_agents, const SweepConfig& cfg, int* ns, int* nt, int* kf) {
  const int C = (nx + 15) / 16;
  if (eb != 8 || fused_agents || cfg.persistent < 1 || cfg.tmem == 0 || cfg.x_lines != 32 || C < 2) return false;
  if (cfg.tmem < 2 && C < 3) return false;
  const int resident = C > kTmemMaxChunks ? C - kTmemMaxChunks : 0;
  int best = 0;
  for (int t = kTmemRingTmem; t >= 1; --t) {
    for (int f = min(C, kTmemFlowSlots); f >= 2; --f) {
      if (f + resident > 32) continue;
      for (int k = kTmemRingSmem; k >= 0; --k) {
        if (k > 0 && C > 32) continue;  // a shared-memory ring's barriers: one bit per slot
        if (x_tmem_smem(nx, k, t, f) <= 227 * 1024) {
          if (k + t > best) {
            best = k + t;
            *ns = k;
            *nt = t;
            *kf = f;
          }
          break;
        }
      }
    }
  }
  return best > 0;
}

// The staged coefficient rows of one ring: the upper diagonal (C chunks of
// 16 rows) and, with `dr`, the forward pairs (one chunk more, for the
// prefetch), which the forward elimination then reads as shared-memory
// broadcasts instead of global loads (measured on B200: cube200 y/z 5%
// faster, lines of 320-448 13-17%).
static size_t tmem_yz_coef_bytes(int C, bool dr) {
  return static_cast<size_t>(C) * kRingRows * 8 + (dr ? static_cast<size_t>(C + 1) * kRingRows * 16 : 0);
}

// One TMEM ring: barriers, kf input slots plus a slot per chunk past the
// 16 that TMEM holds, the staged coefficient rows.
static size_t tmem_yz_ring_bytes(int n_line, int kf, bool dr) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  const int resident = C > kTmemMaxChunks ? C - kTmemMaxChunks : 0;
  return kTmemBarrierBytes + static_cast<size_t>(kf + resident) * kRingRows * 32 * 8 + tmem_yz_coef_bytes(C, dr);
}

// One shared-memory ring of the TMEM y/z sweep: barriers (at most 32
// chunks), the whole tile, the staged coefficient rows.
static size_t tmem_yz_smem_ring_bytes(int n_line, bool dr) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  return kTmemBarrierBytes + static_cast<size_t>(C) * kRingRows * 32 * 8 + tmem_yz_coef_bytes(C, dr);
}

static size_t tmem_yz_smem(int n_line, int ns, int nt, int kf, bool dr) {
  // alignment pad, the rings, the TMEM address word (padded)
  return 128 + ns * tmem_yz_smem_ring_bytes(n_line, dr) + nt * tmem_yz_ring_bytes(n_line, kf, dr) + 128;
}

// The TMEM y/z sweep applies (FP64, lines of at least kTmemFlowSlots chunks,
// at most 32 slots per ring); *ns shared-memory rings and *nt TMEM rings (the
// most rings that fit, TMEM rings first), *kf input slots per TMEM ring.
// More rings beat deeper TMEM rings (cube200 y, B200: 3 + 4 rings of 3
// slots 0.120 ms; 2 + 4 rings of 4, 5, 6 slots 0.124, 0.127, 0.127 ms).
static bool use_tmem_yz(int eb, int n_line, const SweepConfig& cfg, int* ns, int* nt, int* kf, bool* dr) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  if (eb != 8 || cfg.persistent < 1 || cfg.tmem == 0 || cfg.yz_tile != 32 || C < kTmemFlowSlots) return false;
  const int resident = C > kTmemMaxChunks ? C - kTmemMaxChunks : 0;
  // the most rings with the forward pairs staged, unless staging them costs
  // a ring (then the most rings without)
  int best = 0;
  for (int staged = 1; staged >= 0; --staged) {
    for (int t = kTmemRingTmem; t >= 1; --t) {
      for (int f = kTmemFlowSlots; f >= 2; --f) {
        if (f + resident > 32) continue;
        for (int k = kTmemRingSmem; k >= 0; --k) {
          if (k > 0 && C > 32) continue;  // a shared-memory ring's barriers: one bit per slot
          if (tmem_yz_smem(n_line, k, t, f, staged != 0) <= 227 * 1024) {
            if (k + t > best) {
              best = k + t;
              *ns = k;
              *nt = t;
              *kf = f;
              *dr = staged != 0;
            }
            break;
          }
        }
      }
    }
  }
  return best > 0;
}

// Tiles of a y/z sweep over nx columns and nm planes per substrate, with
// partial x tiles packed pw wide (pw = 0: none).
static long long yz_tiles(int nx, int nm, int S, int pw) {
  if (pw <= 0) return static_cast<long long>((nx + 31) / 32) * nm * S;
  const int P = 32 / pw;
  return (static_cast<long long>(nx / 32) * nm + (nm + P - 1) / P) * S;
}

template <int AXIS>
cudaError_t launch_tmem_yz(const CUtensorMap& ring_map, const CUtensorMap& pmap, int pw,
                           const SweepParams<double>& p, const SweepConfig& cfg, cudaStream_t st, bool* launched) {
  *launched = false;
  const int n = (AXIS == 1) ? p.ny : p.nz;
  int ns = 0, nt = 0, kf = 0;
  bool dr = false;
  if (!use_tmem_yz(8, n, cfg, &ns, &nt, &kf, &dr)) return cudaSuccess;
  const int rings = ns + nt;
  const size_t smem = tmem_yz_smem(n, ns, nt, kf, dr);
  const long long tiles = yz_tiles(p.nx, (AXIS == 1) ? p.nz : p.ny, p.s_hi - p.s_lo, pw);
  int grid = 0;
  const bool fast = p.screen == kScreenFast, lng = (n + kRingRows - 1) / kRingRows > kTmemMaxChunks;
  auto kern = fast ? (dr ? (lng ? sweep_yz_tmem_kernel<AXIS, true, true, true> : sweep_yz_tmem_kernel<AXIS, true, true, false>)
                         : (lng ? sweep_yz_tmem_kernel<AXIS, true, false, true> : sweep_yz_tmem_kernel<AXIS, true, false, false>))
                   : (dr ? (lng ? sweep_yz_tmem_kernel<AXIS, false, true, true> : sweep_yz_tmem_kernel<AXIS, false, true, false>)
                         : (lng ? sweep_yz_tmem_kernel<AXIS, false, false, true>
                                : sweep_yz_tmem_kernel<AXIS, false, false, false>));
  cudaError_t e = persistent_grid(kern, smem, (tiles + rings - 1) / rings, &grid, 32 * rings);
  if (e != cudaSuccess) return e;
  if (cfg.persistent < 2 && tiles < kTmemMinTilesPerRing * grid * rings) return cudaSuccess;
  kern<<<grid, 32 * rings, smem, st>>>(ring_map, pmap, p, static_cast<uint32_t>(tmem_yz_smem_ring_bytes(n, dr)),
                                       static_cast<uint32_t>(tmem_yz_ring_bytes(n, kf, dr)), kf, ns, dr ? 1 : 0, pw);
  *launched = true;
  return cudaGetLastError();
}

cudaError_t launch_tmem_x(const CUtensorMap& map, const SweepParams<double>& p, const SweepConfig& cfg,
                          cudaStream_t st, bool* launched) {
  *launched = false;
  int ns = 0, nt = 0, kf = 0;
  if (!use_tmem_x(8, p.nx, p.line_off != nullptr, cfg, &ns, &nt, &kf)) return cudaSuccess;
  const int rings = ns + nt;
  const size_t smem = x_tmem_smem(p.nx, ns, nt, kf);
  const long long tiles = (static_cast<long long>(p.ny) * p.nz + 31) / 32 * (p.s_hi - p.s_lo);
  int grid = 0;
  const bool own = (p.nx + 15) / 16 <= kTmemMaxChunks;
  auto kern = p.screen == kScreenFast ? (own ? sweep_x_tmem_kernel<true, true> : sweep_x_tmem_kernel<true, false>)
                                      : (own ? sweep_x_tmem_kernel<false, true> : sweep_x_tmem_kernel<false, false>);
  cudaError_t e = persistent_grid(kern, smem, (tiles + rings - 1) / rings, &grid, 32 * rings);
  if (e != cudaSuccess) return e;
  if (cfg.persistent < 2 && tiles < kTmemMinTilesPerRing * grid * rings) return cudaSuccess;
  kern<<<grid, 32 * rings, smem, st>>>(map, p, static_cast<uint32_t>(x_tmem_ring_bytes(p.nx, false, kf)),
                                       static_cast<uint32_t>(x_tmem_ring_bytes(p.nx, true, kf)), kf, ns);
  *launched = true;
  return cudaGetLastError();
}

template cudaError_t launch_tmem_yz<1>(const CUtensorMap&, const CUtensorMap&, int, const SweepParams<double>&, const SweepConfig&,
                                       cudaStream_t, bool*);
template cudaError_t launch_tmem_yz<2>(const CUtensorMap&, const CUtensorMap&, int, const SweepParams<double>&, const SweepConfig&,
                                       cudaStream_t, bool*);

// The staged FP64 coefficient rows of one FP32 ring: the upper diagonal
// and, with `dr`, RN(1/d) one chunk past the line (as for FP64 above).
static size_t tmem_yz_f32_coef_bytes(int C, bool dr) {
  return static_cast<size_t>(C) * kRingRows * 8 + (dr ? static_cast<size_t>(C + 1) * kRingRows * 8 : 0);
}

// One FP32 TMEM ring: barriers, kf input slots plus a slot per chunk past the
// 16 that its 256 TMEM columns hold, the staged coefficient rows.
static size_t tmem_yz_f32_ring_bytes(int n_line, int kf, bool dr) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  const int resident = C > kTmemMaxChunks ? C - kTmemMaxChunks : 0;
  return kTmemBarrierBytes + static_cast<size_t>(kf + resident) * kRingRows * 32 * 4 + tmem_yz_f32_coef_bytes(C, dr);
}

// One FP32 shared-memory ring: barriers (at most 32 chunks), the tile, the
// staged coefficient rows.
static size_t tmem_yz_f32_smem_ring_bytes(int n_line, bool dr) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  return kTmemBarrierBytes + static_cast<size_t>(C) * kRingRows * 32 * 4 + tmem_yz_f32_coef_bytes(C, dr);
}

static size_t tmem_yz_f32_smem(int n_line, int ns, int nt, int kf, bool dr) {
  return 128 + ns * tmem_yz_f32_smem_ring_bytes(n_line, dr) + nt * tmem_yz_f32_ring_bytes(n_line, kf, dr) + 128;
}

// The FP32 TMEM y/z sweep applies (FP32, lines of at least kTmemFlowSlots
// chunks, at most 32 slots per ring); the most rings that fit, TMEM rings
// first, then the most input slots.
static bool use_tmem_yz_f32(int eb, int n_line, const SweepConfig& cfg, int* ns, int* nt, int* kf, bool* dr) {
  const int C = (n_line + kRingRows - 1) / kRingRows;
  if (eb != 4 || cfg.persistent < 1 || cfg.tmem == 0 || cfg.yz_tile != 32 || C < kTmemFlowSlots) return false;
  const int resident = C > kTmemMaxChunks ? C - kTmemMaxChunks : 0;
  // the most rings with RN(1/d) staged, unless staging it costs a ring
  int best = 0;
  for (int staged = 1; staged >= 0; --staged) {
    for (int t = kTmemRingTmemF32; t >= 1; --t) {
      for (int f = kTmemFlowSlots; f >= 2; --f) {
        if (f + resident > 32) continue;
        for (int k = kTmemRingSmemF32; k >= 0; --k) {
          if (k > 0 && C > 32) continue;  // a shared-memory ring's barriers: one bit per slot
          if (tmem_yz_f32_smem(n_line, k, t, f, staged != 0) <= 227 * 1024) {
            if (k + t > best) {
              best = k + t;
              *ns = k;
              *nt = t;
              *kf = f;
              *dr = staged != 0;
            }
            break;
          }
        }
      }
    }
  }
  return best > 0;
}

template <int AXIS>
cudaError_t launch_tmem_yz_f32(const CUtensorMap& ring_map, const CUtensorMap& pmap, int pw,
                               const SweepParams<float>& p, const SweepConfig& cfg, cudaStream_t st, bool* launched) {
  *launched = false;
  const int n = (AXIS == 1) ? p.ny : p.nz;
  int ns = 0, nt = 0, kf = 0;
  bool dr = false;
  if (!use_tmem_yz_f32(4, n, cfg, &ns, &nt, &kf, &dr)) return cudaSuccess;
  const int rings = ns + nt;
  const size_t smem = tmem_yz_f32_smem(n, ns, nt, kf, dr);
  const long long tiles = yz_tiles(p.nx, (AXIS == 1) ? p.nz : p.ny, p.s_hi - p.s_lo, pw);
  int grid = 0;
  auto kern = p.screen == kScreenFast ? sweep_yz_tmem_f32_kernel<AXIS, true> : sweep_yz_tmem_f32_kernel<AXIS, false>;
  cudaError_t e = persistent_grid(kern, smem, (tiles + rings - 1) / rings, &grid, 32 * rings);
  if (e != cudaSuccess) return e;
  if (cfg.persistent < 2 && tiles < kTmemMinTilesPerRing * grid * rings) return cudaSuccess;
  kern<<<grid, 32 * rings, smem, st>>>(ring_map, pmap, p, static_cast<uint32_t>(tmem_yz_f32_smem_ring_bytes(n, dr)),
                                       static_cast<uint32_t>(tmem_yz_f32_ring_bytes(n, kf, dr)), kf, ns, dr ? 1 : 0,
                                       pw);
  *launched = true;
  return cudaGetLastError();
}

template cudaError_t launch_tmem_yz_f32<1>(const CUtensorMap&, const CUtensorMap&, int, const SweepParams<float>&, const SweepConfig&,
                                           cudaStream_t, bool*);
template cudaError_t launch_tmem_yz_f32<2>(const CUtensorMap&, const CUtensorMap&, int, const SweepParams<float>&, const SweepConfig&,
                                           cudaStream_t, bool*);

// One ring of the FP32 TMEM x sweep (a multiple of 1024 bytes, so every chunk
// stays on the 128B-swizzle atom): shared-memory ring = C chunks; TMEM ring
// = kf input chunks and a staging chunk, or, past 8 chunks, kf input chunks
// and a resident chunk for each chunk past 8; then the upper diagonal (FP64)
// and the barriers.
static size_t x_tmem_f32_ring_bytes(int nx, bool tm, int kf, bool dr) {
  const int C = (nx + 31) / 32;
  const int chunks = !tm ? C : (C <= kXTmemMaxChunksF32 ? kf + 1 : kf + C - kXTmemMaxChunksF32);
  // chunks, the upper diagonal (C chunks), RN(1/d) (C + 1 chunks) when staged, barriers
  const size_t b = static_cast<size_t>(chunks) * 32 * 128 + static_cast<size_t>(dr ? 2 * C + 1 : C) * 32 * 8 +
                   kXTmemBarrierBytes;
  return (b + 1023) / 1024 * 1024;
}

static size_t x_tmem_f32_smem(int nx, int ns, int nt, int kf, bool dr) {
  return 1024 + ns * x_tmem_f32_ring_bytes(nx, false, kf, dr) + nt * x_tmem_f32_ring_bytes(nx, true, kf, dr) + 128;
}

// The FP32 TMEM x sweep applies (FP32, agents not fused, 32-line tiles,
// lines of at least 2 chunks = 33 voxels, at most 32 slots per ring): *nt
// TMEM rings (the most that fit) and *kf input slots per ring, no
// shared-memory rings.  Measured on B200 against the per-tile FP32 x sweep:
// cube200 (4 substrates) 0.110 against 0.120 ms, n^3 cubes with 2
// substrates 0.98-1.00 from 256 to 640 voxels, 1.06 at 200 (2.4 tiles per
// ring); with 3 shared-memory rings beside the 8 TMEM rings it had lost 6%
// at cube200 (0.127 ms), 5 + 4 rings 24%.
static bool use_tmem_x_f32(int eb, int nx, bool fused_agents, const SweepConfig& cfg, int* ns, int* nt, int* kf,
                           bool* dr) {
  const int C = (nx + 31) / 32;
  if (eb != 4 || fused_agents || cfg.persistent < 1 || cfg.tmem == 0 || cfg.x_lines != 32 || C < 2) return false;
  const int resident = C > kXTmemMaxChunksF32 ? C - kXTmemMaxChunksF32 : 0;
  // the most rings with RN(1/d) staged per ring (cube200: 0.106 against
  // 0.110 ms), unless staging it costs a ring
  int best = 0;
  for (int staged = 1; staged >= 0; --staged) {
    for (int t = kXTmemRingTmemF32; t >= 1; --t) {
      for (int f = min(C, kTmemFlowSlots); f >= 2; --f) {
        if (f + resident > 32) continue;
        for (int k = kXTmemRingSmemF32; k >= 0; --k) {
          if (k > 0 && C > 32) continue;  // a shared-memory ring's barriers: one bit per slot
          if (x_tmem_f32_smem(nx, k, t, f, staged != 0) <= 227 * 1024) {
            if (k + t > best) {
              best = k + t;
              *ns = k;
              *nt = t;
              *kf = f;
              *dr = staged != 0;
            }
            break;
          }
        }
      }
    }
  }
  return best > 0;
}

cudaError_t launch_tmem_x_f32(const CUtensorMap& map, const SweepParams<float>& p, const SweepConfig& cfg,
                              cudaStream_t st, bool* launched) {
  *launched = false;
  int ns = 0, nt = 0, kf = 0;
  bool dr = false;
  if (!use_tmem_x_f32(4, p.nx, p.line_off != nullptr, cfg, &ns, &nt, &kf, &dr)) return cudaSuccess;
  const int rings = ns + nt;
  const size_t smem = x_tmem_f32_smem(p.nx, ns, nt, kf, dr);
  const long long tiles = (static_cast<long long>(p.ny) * p.nz + 31) / 32 * (p.s_hi - p.s_lo);
  int grid = 0;
  const bool own = (p.nx + 31) / 32 <= kXTmemMaxChunksF32;
  auto kern =
      p.screen == kScreenFast
          ? (dr ? (own ? sweep_x_tmem_f32_kernel<true, true, true> : sweep_x_tmem_f32_kernel<true, true, false>)
                : (own ? sweep_x_tmem_f32_kernel<true, false, true> : sweep_x_tmem_f32_kernel<true, false, false>))
          : (dr ? (own ? sweep_x_tmem_f32_kernel<false, true, true> : sweep_x_tmem_f32_kernel<false, true, false>)
                : (own ? sweep_x_tmem_f32_kernel<false, false, true> : sweep_x_tmem_f32_kernel<false, false, false>));
  cudaError_t e = persistent_grid(kern, smem, (tiles + rings - 1) / rings, &grid, 32 * rings);
  if (e != cudaSuccess) return e;
  if (cfg.persistent < 2 && tiles < kTmemMinTilesPerRing * grid * rings) return cudaSuccess;
  kern<<<grid, 32 * rings, smem, st>>>(map, p, static_cast<uint32_t>(x_tmem_f32_ring_bytes(p.nx, false, kf, dr)),
                                       static_cast<uint32_t>(x_tmem_f32_ring_bytes(p.nx, true, kf, dr)), kf, ns,
                                       dr ? 1 : 0);
  *launched = true;
  return cudaGetLastError();
}

cudaError_t tmem_sweeps_set_wait_limit(unsigned long long ns) { return set_module_wait_limit(ns); }

}  // namespace bfvm

extern "C" int bfvm_tmem_sweep_plan(int axis, int n_line, int tmem_level, int* smem_rings, int* tmem_rings,
                                    int* input_slots) {
  if (axis < 0 || axis > 3 || n_line < 1 || n_line > 65535 || tmem_level < 0 || tmem_level > 2 || !smem_rings ||
      !tmem_rings || !input_slots)
    return BFVM_ERR_ARG;
  bfvm::SweepConfig cfg;
  cfg.tmem = tmem_level;
  int ns = 0, nt = 0, kf = 0;
  bool dr = false;
  const bool on = axis == 0   ? bfvm::use_tmem_x(8, n_line, false, cfg, &ns, &nt, &kf)
                  : axis == 1 ? bfvm::use_tmem_yz(8, n_line, cfg, &ns, &nt, &kf, &dr)
                  : axis == 2 ? bfvm::use_tmem_yz_f32(4, n_line, cfg, &ns, &nt, &kf, &dr)
                              : bfvm::use_tmem_x_f32(4, n_line, false, cfg, &ns, &nt, &kf, &dr);
  *smem_rings = on ? ns : 0;
  *tmem_rings = on ? nt : 0;
  *input_slots = on ? kf : 0;
  return BFVM_OK;
}
