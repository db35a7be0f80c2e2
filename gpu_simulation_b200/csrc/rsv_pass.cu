// Tile-pass kernels of the ring-Ising structured adjoint (sm_100a).
//
// Replaces the reference's per-chunk rotation kernels
// (zzEncounter/GPU_Simulation cpp/ising_cuda_rotation_kernels.cu:95-552 forward,
// cpp/ising_cuda_statevector_grad_kernels.cu:223-1437 backward) and its ring-CNOT
// kernels (cpp/ising_cuda_kernels.cu:207-236):
//
//   * a pass streams the state once, tile by tile; a tile is a coset of a
//     12-dimensional GF(2) subspace of indices (4096 amplitudes) held in
//     registers, 16 per thread of a 256-thread CTA;
//   * the wires whose directions lie in the tile are rotated in registers;
//     shared-memory transposes move the other tile directions into registers
//     ("layouts" 0, 1, 2 below), so one pass covers up to 12 wires;
//   * the CNOT ring is folded into a pass's load (gather through P) or store
//     (scatter through P or P^-1); the layer's RZ gates are one diagonal phase
//     per amplitude from four 256-entry byte tables;
//   * backward passes stream psi and lambda: the next tile is prefetched into
//     shared memory with cp.async while the current tile is processed, and the
//     theta/phi gradient sums are accumulated on chip and written as one
//     deterministic record per CTA (no FP64 atomics).
//
// The load/store variants are template parameters, so every instantiation
// carries only the code of its own variant; the register gate code exists
// once and is visited once per layout.
#include "rsv_device.cuh"
#include "rsv_types.h"

namespace rsv {
namespace {

using u32 = unsigned int;

// Thread layouts of a tile (tile index t has 12 bits):
//   layout 0: lanes -> t bits 0..4, warps -> 5..7,  registers -> 8..11 (global load/store)
//   layout 1: lanes -> t bits 8..11,0, warps -> 1..3, registers -> 4..7
//   layout 2: lanes -> t bits 4..8, warps -> 9..11, registers -> 0..3
__device__ __forceinline__ int thread_part(int layout, int lane, int warp) {
  if (layout == 0) return lane | (warp << 5);
  if (layout == 1) return (lane >> 4) | (warp << 1) | ((lane & 15) << 8);
  return (lane << 4) | (warp << 9);
}
__device__ __forceinline__ int reg_shift(int layout) { return layout == 0 ? 8 : (layout == 1 ? 4 : 0); }

// Tile bit held by lane bit j / warp bit j of a layout.
__device__ __forceinline__ int lane_tile_bit(int layout, int j) {
  if (layout == 0) return j;
  if (layout == 1) return j < 4 ? 8 + j : 0;
  return 4 + j;
}
__device__ __forceinline__ int warp_tile_bit(int layout, int j) {
  if (layout == 0) return 5 + j;
  if (layout == 1) return 1 + j;
  return 9 + j;
}

// XOR-fold swizzle: the 8 lanes of a quarter warp hit distinct 16-byte bank
// groups for every layout (their tile bits are 3 consecutive bits).
__device__ __forceinline__ int swz(int t) { return t ^ (((t >> 3) ^ (t >> 6) ^ (t >> 9)) & 7); }

__device__ __forceinline__ u32 deposit(const PassParams &P, u32 tile) {
  u32 base = 0;
#pragma unroll
  for (int r = 0; r < kMaxRuns; ++r) {
    if (r < P.num_runs) {
      const int len = P.run_len[r];
      base |= (tile & ((1u << len) - 1u)) << P.run_start[r];
      tile >>= len;
    }
  }
  return base;
}

// Physical offset of the thread part of a layout.
__device__ __forceinline__ u32 thread_offset(const PassParams &P, int tp) {
  u32 o = 0;
#pragma unroll
  for (int b = 0; b < 12; ++b)
    if ((tp >> b) & 1) o ^= static_cast<u32>(P.vec[b]);
  return o;
}

// Physical offset of register r in a layout whose register directions are v0..v3.
__device__ __forceinline__ u32 reg_offset(int r, u32 v0, u32 v1, u32 v2, u32 v3) {
  return ((r & 1) ? v0 : 0u) ^ ((r & 2) ? v1 : 0u) ^ ((r & 4) ? v2 : 0u) ^ ((r & 8) ? v3 : 0u);
}

__device__ __forceinline__ double2 table4(const double2 *__restrict__ t, u32 p) {
  double2 v = __ldg(&t[p & 255]);
  v = cmul(v, __ldg(&t[256 + ((p >> 8) & 255)]));
  v = cmul(v, __ldg(&t[512 + ((p >> 16) & 255)]));
  v = cmul(v, __ldg(&t[768 + (p >> 24)]));
  return v;
}

template <int SRC>
__device__ __forceinline__ u32 source_index(u32 p, int n) {
  if (SRC == kLoadGatherP) return static_cast<u32>(ring_p(p, n));
  return p;
}

template <int DST>
__device__ __forceinline__ void store_amp(double2 *buf, u32 p, int n, double2 v) {
  if (DST == kStoreNatural) __stcs(&buf[p], v);
  if (DST == kStoreScatterP) __stcs(&buf[static_cast<u32>(ring_p(p, n))], v);
  if (DST == kStoreScatterPinv) __stcs(&buf[static_cast<u32>(ring_pinv(p, n))], v);
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const u32 s = static_cast<u32>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Forward rotation of the four register bits of `layout` (tile bits
// rb..rb+3): RY / f in tangent form, one FMA per component.
//   mode +1: [[1,-k],[k,1]]    mode -1: [[k,-1],[1,k]]
__device__ __forceinline__ void apply_gates_fwd(const PassParams &P, int layout, double2 (&a)[kRegs]) {
  const int rb = reg_shift(layout);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int w = P.gate_wire[rb + j];
    if (w < 0) continue;
    const double2 km = __ldg(&P.rot[P.layer * P.n + w]);
    const double k = km.x;
    if (km.y > 0.0) {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const double2 x0 = a[r], x1 = a[r1];
        a[r] = make_double2(fma(-k, x1.x, x0.x), fma(-k, x1.y, x0.y));
        a[r1] = make_double2(fma(k, x0.x, x1.x), fma(k, x0.y, x1.y));
      }
    } else {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const double2 x0 = a[r], x1 = a[r1];
        a[r] = make_double2(fma(k, x0.x, -x1.x), fma(k, x0.y, -x1.y));
        a[r1] = make_double2(fma(k, x1.x, x0.x), fma(k, x1.y, x0.y));
      }
    }
  }
}

// Register values of layout `from` -> layout `to` through shared memory.
__device__ __forceinline__ void transpose(double2 *sm, int tp_from, int rb_from, int tp_to, int rb_to,
                                          double2 (&a)[kRegs]) {
#pragma unroll
  for (int r = 0; r < kRegs; ++r) sm[swz(tp_from | (r << rb_from))] = a[r];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRegs; ++r) a[r] = sm[swz(tp_to | (r << rb_to))];
  __syncthreads();
}

// e^{i phi_w} of wire w of a layer (from its cos/sin(phi/2)); 1 for w >= n.
__device__ __forceinline__ double2 phase_ratio(const PassParams &P, int w) {
  if (w < 0 || w >= P.n) return make_double2(1.0, 0.0);
  const double4 k = P.coef[P.layer * P.n + w];
  return make_double2(fma(k.z, k.z, -k.w * k.w), 2.0 * k.z * k.w);
}

__device__ __forceinline__ int unit_bit(unsigned long long v) { return v ? __ffsll(v) - 1 : -1; }

// Multiply register r of `a` (and `b`) by its RZ-phase (or conjugate): the
// phase of element base ^ (register directions of r) is phase(base) times
// e^{i phi_w} for every register direction e_w set in r (unit directions).
// Registers are visited in Gray-code order so that one running product is
// enough.
template <int NB, bool CONJ, bool TWO>
__device__ __forceinline__ void apply_phase_gray(double2 ph, const double2 (&ratio)[4],
                                                 double2 *a, double2 *b) {
  constexpr int NR = 1 << NB;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int g = k ^ (k >> 1);
    if (k > 0) {
      const int prev = (k - 1) ^ ((k - 1) >> 1);
      const int flipped = g ^ prev;
      const int j = flipped == 1 ? 0 : flipped == 2 ? 1 : flipped == 4 ? 2 : 3;
      ph = (g & flipped) ? cmul(ph, ratio[j]) : cmul_conj(ph, ratio[j]);
    }
    if (CONJ) {
      a[g] = cmul_conj(a[g], ph);
      if (TWO) b[g] = cmul_conj(b[g], ph);
    } else {
      a[g] = cmul(a[g], ph);
      if (TWO) b[g] = cmul(b[g], ph);
    }
  }
}

// ======================================================================
// Backward pass: 512 threads x 8 amplitudes of psi and lambda each.
// Register groups of three tile bits; two layout families:
//   family B (warps own tile bits 0..3):
//     B0: lanes -> 4..8,        registers -> 9..11
//     B1: lanes -> 9,10,11,4,5, registers -> 6..8
//   family A (warps own tile bits 8..11):
//     A1: lanes -> 3..7,        registers -> 0..2
//     A2: lanes -> 0,1,2,6,7,   registers -> 3..5
// Moving between the layouts of one family only permutes data inside a warp
// (a warp-private slice of shared memory and __syncwarp); one CTA-wide
// transpose per tile moves from family B to family A.  A tile is visited
// B0 -> B1 -> (A1 ->) A2 and stored from A2, whose lanes 0..2 cover 128-byte
// segments.
// ======================================================================
namespace bw {
constexpr int kT = 512;
constexpr int kR = 8;

enum Layout { B0 = 0, B1 = 1, A1 = 2, A2 = 3 };

// tile index of (lane, warp) with register 0, and the tile bit of register bit 0
template <int LY>
__device__ __forceinline__ int tpart(int lane, int warp) {
  if (LY == B0) return warp | (lane << 4);
  if (LY == B1) return warp | ((lane >> 3) << 4) | ((lane & 7) << 9);
  if (LY == A1) return (lane << 3) | (warp << 8);
  return (lane & 7) | ((lane >> 3) << 6) | (warp << 8);
}
template <int LY>
__host__ __device__ constexpr int rbit() {
  return LY == B0 ? 9 : LY == B1 ? 6 : LY == A1 ? 0 : 3;
}
// warp-local index (8 bits) of a tile index: family B keeps tile bits 4..11,
// family A tile bits 0..7
template <int LY>
__device__ __forceinline__ int local(int t) {
  return (LY == B0 || LY == B1) ? (t >> 4) : (t & 255);
}
__device__ __forceinline__ int sw8(int l) { return l ^ (((l >> 3) ^ (l >> 6)) & 7); }

// layout FROM -> TO of the same family, through this warp's 256-entry slice
template <int FROM, int TO>
__device__ __forceinline__ void warp_transpose(double2 *wbuf, int lane, int warp, double2 (&a)[kR]) {
  const int tf = tpart<FROM>(lane, warp), tt = tpart<TO>(lane, warp);
#pragma unroll
  for (int r = 0; r < kR; ++r) wbuf[sw8(local<FROM>(tf | (r << rbit<FROM>())))] = a[r];
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kR; ++r) a[r] = wbuf[sw8(local<TO>(tt | (r << rbit<TO>())))];
  __syncwarp();
}

// layout FROM -> TO through the CTA-wide buffer (whole tile).  The leading
// barrier keeps a fast warp from overwriting a slow warp's private slice.
template <int FROM, int TO>
__device__ __forceinline__ void cta_transpose(double2 *sm, int lane, int warp, double2 (&a)[kR]) {
  const int tf = tpart<FROM>(lane, warp), tt = tpart<TO>(lane, warp);
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) sm[swz(tf | (r << rbit<FROM>()))] = a[r];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) a[r] = sm[swz(tt | (r << rbit<TO>()))];
  __syncthreads();
}

// Backward rotation of the three register bits of layout LY (tile bits
// RB..RB+2): RY^dagger / f in tangent form, one FMA per component,
//   mode +1: [[1,k],[-k,1]]    mode -1: [[k,1],[-1,k]],
// preceded by the theta sum Re(conj(lam1) psi0) - Re(conj(lam0) psi1) of the
// pair in the frame with the layer's RZ removed -- the reference's
// 2 Re<lam_mid|dRY|psi_before> (cpp/ising_cuda_statevector_grad_kernels.cu:289-307)
// simplified; the factors f still pending are corrected in the final reduction.
template <int LY>
__device__ __forceinline__ void gates(const PassParams &P, double2 (&a)[kR], double2 (&b)[kR],
                                      double (&acc)[12]) {
  constexpr int RB = rbit<LY>();
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int w = P.gate_wire[RB + j];
    if (w < 0) continue;
    const double2 km = __ldg(&P.rot[P.layer * P.n + w]);
    const double k = km.x;
    double t = acc[RB + j];
    if (km.y > 0.0) {
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const double2 x0 = a[r], x1 = a[r1], y0 = b[r], y1 = b[r1];
        t = fma(y1.x, x0.x, t);
        t = fma(y1.y, x0.y, t);
        t = fma(-y0.x, x1.x, t);
        t = fma(-y0.y, x1.y, t);
        a[r] = make_double2(fma(k, x1.x, x0.x), fma(k, x1.y, x0.y));
        a[r1] = make_double2(fma(-k, x0.x, x1.x), fma(-k, x0.y, x1.y));
        b[r] = make_double2(fma(k, y1.x, y0.x), fma(k, y1.y, y0.y));
        b[r1] = make_double2(fma(-k, y0.x, y1.x), fma(-k, y0.y, y1.y));
      }
    } else {
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const double2 x0 = a[r], x1 = a[r1], y0 = b[r], y1 = b[r1];
        t = fma(y1.x, x0.x, t);
        t = fma(y1.y, x0.y, t);
        t = fma(-y0.x, x1.x, t);
        t = fma(-y0.y, x1.y, t);
        a[r] = make_double2(fma(k, x0.x, x1.x), fma(k, x0.y, x1.y));
        a[r1] = make_double2(fma(k, x1.x, -x0.x), fma(k, x1.y, -x0.y));
        b[r] = make_double2(fma(k, y0.x, y1.x), fma(k, y0.y, y1.y));
        b[r1] = make_double2(fma(k, y1.x, -y0.x), fma(k, y1.y, -y0.y));
      }
    }
    acc[RB + j] = t;
  }
}

// phi-gradient sums of one tile in layout B0 (registers -> tile bits 9..11,
// lanes -> 4..8, warps -> 0..3): q = Im(conj(lam) psi) per amplitude, folded
// into phi_sm[w] (sum of q with bit w set) and phi_sm[32] (sum of q).
__device__ __forceinline__ void phi_sums(const PassParams &P, u32 cbase, int lane, int warp,
                                         const double2 (&a)[kR], const double2 (&b)[kR],
                                         double (*red)[12], double *phi_sm) {
  double v[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) v[j] = 0.0;
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const double q = fma(b[r].x, a[r].y, -b[r].y * a[r].x);
    v[0] += q;
#pragma unroll
    for (int j = 0; j < 3; ++j)
      if ((r >> j) & 1) v[1 + j] += q;
  }
#pragma unroll
  for (int j = 0; j < 5; ++j) v[4 + j] = ((lane >> j) & 1) ? v[0] : 0.0;
#pragma unroll
  for (int j = 0; j < 9; ++j) v[j] = warp_sum(v[j]);
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < 9; ++j) red[warp][j] = v[j];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int w = threadIdx.x;
    double qt = 0.0;
    for (int ww = 0; ww < 16; ++ww) qt += red[ww][0];
    if (w < P.n) {
      const int tb = P.wire_tile_bit[w];
      double add = 0.0;
      if (tb < 0) {
        if ((cbase >> w) & 1) add = qt;  // coset bit: set for the whole tile
      } else if (tb >= 9) {
        for (int ww = 0; ww < 16; ++ww) add += red[ww][1 + tb - 9];
      } else if (tb >= 4) {
        for (int ww = 0; ww < 16; ++ww) add += red[ww][4 + tb - 4];
      } else {
        for (int ww = 0; ww < 16; ++ww)
          if ((ww >> tb) & 1) add += red[ww][0];
      }
      phi_sm[w] += add;
    }
    if (w == 31) phi_sm[32] += qt;
  }
  __syncthreads();
}
}  // namespace bw

// Shared memory of the backward kernel (dynamic): staging psi | staging lam |
// transpose buffer (CTA-wide, or 16 warp slices of 256 entries).
constexpr size_t kBwdSmem = 3 * kTileSize * sizeof(double2);
constexpr size_t kFwdSmem = kTileSize * sizeof(double2);

// ---------------------------------------------------------------- backward
template <int LSRC, int PDST, int LDST, bool PHASE>
__global__ void __launch_bounds__(bw::kT, 1) bwd_pass_kernel(const PassParams P) {
  using namespace bw;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage_a = reinterpret_cast<double2 *>(smem_raw);
  double2 *stage_b = stage_a + kTileSize;
  double2 *trans = stage_b + kTileSize;
  __shared__ double red[16][12];
  __shared__ double phi_sm[33];

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int n = P.n;
  double2 *wbuf = trans + warp * 256;

  // gates on tile bits 0..2 need the A1 visit
  const bool has_lo = P.gate_wire[0] >= 0 || P.gate_wire[1] >= 0 || P.gate_wire[2] >= 0;

  // global issue layout: lanes -> tile bits 0..4 (coalesced), warps -> 5..8, registers -> 9..11
  const int tpi = lane | (warp << 5);
  const u32 toffi = thread_offset(P, tpi);
  const u32 v9 = P.vec[9], v10 = P.vec[10], v11 = P.vec[11];
  // store layout A2: registers -> tile bits 3..5
  const int tps = tpart<A2>(lane, warp);
  const u32 toffs = thread_offset(P, tps);
  const u32 v3 = P.vec[3], v4 = P.vec[4], v5 = P.vec[5];

  double2 ratio[4];
  u32 toffp = 0;
  if (PHASE) {
    toffp = thread_offset(P, tpart<B0>(lane, warp));
#pragma unroll
    for (int j = 0; j < 3; ++j) ratio[j] = phase_ratio(P, unit_bit(P.vec[9 + j]));
    ratio[3] = make_double2(1.0, 0.0);
    if (threadIdx.x < 33) phi_sm[threadIdx.x] = 0.0;
  }
  double acc[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) acc[i] = 0.0;

  const u32 num_tiles = static_cast<u32>(P.num_tiles);
  auto issue = [&](u32 tile) {
    const u32 base = deposit(P, tile) ^ toffi;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const u32 p = base ^ ((r & 1) ? v9 : 0u) ^ ((r & 2) ? v10 : 0u) ^ ((r & 4) ? v11 : 0u);
      const int s = swz(tpi | (r << 9));
      cp_async16(&stage_a[s], &P.psi_in[p]);
      cp_async16(&stage_b[s], &P.lam_in[source_index<LSRC>(p, n)]);
    }
    cp_async_commit();
  };
  if (blockIdx.x < num_tiles) issue(blockIdx.x);

  const int tb0 = tpart<B0>(lane, warp);
  for (u32 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    double2 a[kR], b[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int s = swz(tb0 | (r << 9));
      a[r] = stage_a[s];
      b[r] = stage_b[s];
    }
    __syncthreads();
    if (tile + gridDim.x < num_tiles) issue(tile + gridDim.x);

    const u32 cbase = deposit(P, tile);
    if (PHASE) {
      // RZ^dagger of the layer (with the layer's factor K) on psi and lambda,
      // then the phi sums.
      const double2 ph = table4(P.ptab, cbase ^ toffp);
      const double K = P.lscale[P.layer];
      apply_phase_gray<3, true, true>(make_double2(K * ph.x, K * ph.y), ratio, a, b);
      phi_sums(P, cbase, lane, warp, a, b, red, phi_sm);
    }

    gates<B0>(P, a, b, acc);
    warp_transpose<B0, B1>(wbuf, lane, warp, a);
    warp_transpose<B0, B1>(wbuf, lane, warp, b);
    gates<B1>(P, a, b, acc);
    if (has_lo) {
      cta_transpose<B1, A1>(trans, lane, warp, a);
      cta_transpose<B1, A1>(trans, lane, warp, b);
      gates<A1>(P, a, b, acc);
      warp_transpose<A1, A2>(wbuf, lane, warp, a);
      warp_transpose<A1, A2>(wbuf, lane, warp, b);
    } else {
      cta_transpose<B1, A2>(trans, lane, warp, a);
      cta_transpose<B1, A2>(trans, lane, warp, b);
    }
    gates<A2>(P, a, b, acc);

    if (PDST != kStoreNone || LDST != kStoreNone) {
      const u32 base = cbase ^ toffs;
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const u32 p = base ^ ((r & 1) ? v3 : 0u) ^ ((r & 2) ? v4 : 0u) ^ ((r & 4) ? v5 : 0u);
        store_amp<PDST>(P.psi_out, p, n, a[r]);
        store_amp<LDST>(P.lam_out, p, n, b[r]);
      }
    }
  }

  // CTA reduction of the theta sums, then one record per CTA.
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const double s = warp_sum(acc[i]);
    if (lane == 0) red[warp][i] = s;
  }
  __syncthreads();
  double *rec = P.partials + static_cast<size_t>(blockIdx.x) * kPartialStride;
  if (threadIdx.x < 12) {
    double s = 0.0;
    for (int ww = 0; ww < 16; ++ww) s += red[ww][threadIdx.x];
    rec[threadIdx.x] = s;
  }
  if (PHASE) {
    if (threadIdx.x < 31) rec[kPartialPhi + threadIdx.x] = phi_sm[threadIdx.x];
    if (threadIdx.x == 31) rec[kPartialTot] = phi_sm[32];
  }
}

// ----------------------------------------------------------------- forward
template <int PSRC, int PDST, bool PHASE>
__global__ void __launch_bounds__(kThreads, 2) fwd_pass_kernel(const PassParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *trans = reinterpret_cast<double2 *>(smem_raw);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int n = P.n;
  const int tp0 = thread_part(0, lane, warp);
  const u32 toff0 = thread_offset(P, tp0);
  const u32 v8 = P.vec[8], v9 = P.vec[9], v10 = P.vec[10], v11 = P.vec[11];
  const u32 num_tiles = static_cast<u32>(P.num_tiles);
  double2 dummy[kRegs];
  double2 ratio[4];
  if (PHASE) {
#pragma unroll
    for (int j = 0; j < 4; ++j) ratio[j] = phase_ratio(P, unit_bit(P.vec[8 + j]));
  }

  for (u32 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const u32 base = deposit(P, tile) ^ toff0;
    double2 a[kRegs];
#pragma unroll
    for (int r = 0; r < kRegs; ++r) {
      const u32 p = base ^ reg_offset(r, v8, v9, v10, v11);
      if (PSRC == kLoadNatural) a[r] = __ldcs(&P.psi_in[p]);
      if (PSRC == kLoadProduct) a[r] = table4(P.prod, static_cast<u32>(ring_pinv(p, n)));
      if (PSRC == kLoadProductPlain) a[r] = table4(P.prod, p);
    }
    if (P.sync_after_load) __syncthreads();

    int prev = 0;
    for (int k = 0; k < P.nseq; ++k) {
      const int layout = P.seq_layout[k];
      const int tp = thread_part(layout, lane, warp);
      if (k > 0) transpose(trans, thread_part(prev, lane, warp), reg_shift(prev), tp, reg_shift(layout), a);
      if (P.seq_apply[k]) apply_gates_fwd(P, layout, a);
      prev = layout;
    }

    if (PHASE) {
      const double2 ph = table4(P.ptab, base);
      const double K = P.lscale[P.layer];
      apply_phase_gray<4, false, false>(make_double2(K * ph.x, K * ph.y), ratio, a, dummy);
    }
#pragma unroll
    for (int r = 0; r < kRegs; ++r) store_amp<PDST>(P.psi_out, base ^ reg_offset(r, v8, v9, v10, v11), n, a[r]);
  }
}

template <int LSRC, int PDST, int LDST, bool PHASE>
cudaError_t launch_bwd(const PassParams &P, int grid, cudaStream_t s) {
  auto k = bwd_pass_kernel<LSRC, PDST, LDST, PHASE>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kBwdSmem));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  k<<<grid, bw::kT, kBwdSmem, s>>>(P);
  return cudaGetLastError();
}

template <int PSRC, int PDST, bool PHASE>
cudaError_t launch_fwd(const PassParams &P, int grid, cudaStream_t s) {
  auto k = fwd_pass_kernel<PSRC, PDST, PHASE>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kFwdSmem));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  k<<<grid, kThreads, kFwdSmem, s>>>(P);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pass(const PassParams &P, bool bwd, int grid, cudaStream_t s) {
  if (bwd) {
    if (P.psi_load != kLoadNatural) return cudaErrorInvalidValue;
    const bool phase = P.phase != 0;
    const bool gather = P.lam_load == kLoadGatherP;
    if (P.lam_load != kLoadNatural && !gather) return cudaErrorInvalidValue;
    if (P.phi_grad != P.phase) return cudaErrorInvalidValue;
    const int ps = P.psi_store, ls = P.lam_store;
    // (psi, lambda) stores used by the planner: (natural, natural),
    // (scatter P^-1, natural), (none, none)
    if (ps == kStoreNatural && ls == kStoreNatural) {
      if (phase) return gather ? launch_bwd<kLoadGatherP, kStoreNatural, kStoreNatural, true>(P, grid, s)
                               : launch_bwd<kLoadNatural, kStoreNatural, kStoreNatural, true>(P, grid, s);
      if (!gather) return launch_bwd<kLoadNatural, kStoreNatural, kStoreNatural, false>(P, grid, s);
    } else if (ps == kStoreScatterPinv && ls == kStoreNatural) {
      if (phase) return gather ? launch_bwd<kLoadGatherP, kStoreScatterPinv, kStoreNatural, true>(P, grid, s)
                               : launch_bwd<kLoadNatural, kStoreScatterPinv, kStoreNatural, true>(P, grid, s);
      if (!gather) return launch_bwd<kLoadNatural, kStoreScatterPinv, kStoreNatural, false>(P, grid, s);
    } else if (ps == kStoreNone && ls == kStoreNone) {
      if (phase) return gather ? launch_bwd<kLoadGatherP, kStoreNone, kStoreNone, true>(P, grid, s)
                               : launch_bwd<kLoadNatural, kStoreNone, kStoreNone, true>(P, grid, s);
      if (!gather) return launch_bwd<kLoadNatural, kStoreNone, kStoreNone, false>(P, grid, s);
    }
    return cudaErrorInvalidValue;
  }
  const bool phase = P.phase != 0;
  const int src = P.psi_load, dst = P.psi_store;
  if (src == kLoadProductPlain && dst == kStoreNatural && !phase)
    return launch_fwd<kLoadProductPlain, kStoreNatural, false>(P, grid, s);
#define RSV_FWD(SRC)                                                                 \
  if (src == SRC) {                                                                  \
    if (dst == kStoreNatural)                                                        \
      return phase ? launch_fwd<SRC, kStoreNatural, true>(P, grid, s)                \
                   : launch_fwd<SRC, kStoreNatural, false>(P, grid, s);              \
    if (dst == kStoreScatterP)                                                       \
      return phase ? launch_fwd<SRC, kStoreScatterP, true>(P, grid, s)               \
                   : launch_fwd<SRC, kStoreScatterP, false>(P, grid, s);             \
  }
  RSV_FWD(kLoadNatural)
  RSV_FWD(kLoadProduct)
#undef RSV_FWD
  return cudaErrorInvalidValue;
}

size_t pass_smem_bytes(bool bwd) { return bwd ? kBwdSmem : kFwdSmem; }

cudaError_t configure_pass_kernels() { return cudaSuccess; }

}  // namespace rsv
