// Sharded single circuit (include/rsv_shard.h): the per-rank kernels of one
// ring-Ising circuit whose complex128 state is split over N = 2^g GPUs.
//
// Layout C keeps wires 0..n-g-1 local, layout S wires 0..n-2g-1 and
// n-g..n-1; the two differ by one all-to-all of 2^(n-2g)-amplitude blocks,
// which the caller runs.  Per layer:
//   * rot_kernel: RZ RY on the local wires of C, 11-bit tiles of the shard
//     (tile bits 0..3 are local bits 0..3: 256-byte rows), 16 amplitudes per
//     thread in registers and three register layouts exchanged through shared
//     memory, so every gate is a register-pair update;
//   * ring_pack_kernel: in S, RZ RY on wires n-g..n-1 (the 2^g amplitudes of
//     one thread: x bits [n-g, n) are the top local bits of S) and the sort of
//     every amplitude by the rank that owns P(x) in C;
//   * ring_unpack_kernel: after the all-to-all, psi_C[y] = received[P^-1(y)].
// The backward reverses each step on psi and lambda with the gradient sums of
// the reference's inverse walk (per gate: RZ sum, RZ^dagger, RY sum,
// RY^dagger; cpp/ising_cuda_gate_level_adjoint_modes.inc:147-260), each
// CTA's sums in a record and the records added in a fixed order, so results
// do not depend on scheduling.  Rotations of different wires commute, so one
// layer's local wires go in any grouping of passes.
#include <algorithm>
#include <atomic>
#include <string>

#include <cuda_runtime.h>

#include "../../include/rsv_shard.h"
#include "rsv_device.cuh"
#include "rsv_launch.h"
#include "rsv_workspace.h"

namespace rsv {
namespace {

using u32 = unsigned int;

constexpr int kMaxG = 3;
constexpr int kMinLowBits = 12;   // n - 2g: the chunk of one rank pair has >= 4096 amplitudes
constexpr int kMaxLocalBits = 31;

// ---------------------------------------------------------------- local passes
constexpr int kT = 11;            // tile bits
constexpr int kTile = 1 << kT;    // 2048 amplitudes (32 KiB per vector)
constexpr int kRotThreads = 128;  // tile bits of the thread index in layout A: 0..6
constexpr int kR = 16;            // amplitudes per thread (4 register bits)
constexpr int kRec = 2 * kT;      // one CTA's gradient record: (theta, phi) per tile bit
constexpr int kMaxRuns = kT + 1;
constexpr int kAdjSmem = 2 * kTile * 16;
constexpr int kRotCtasPerSm = 3;  // 32 KiB of shared memory and <= 170 registers a thread each
constexpr int kAdjCtasPerSm = 2;  // 64 KiB of shared memory and <= 255 registers a thread each

struct TileArgs {
  int n, nloc, layer;
  int bits[kT];  // local bit of tile bit j, increasing
  int wire[kT];  // wire rotated on tile bit j, or -1
  int run_start[kMaxRuns], run_len[kMaxRuns], num_runs;  // local bits outside the tile, low to high
  u32 num_tiles;
  int need_b, need_c;  // gates on tile bits 3..6 / 0..2
};

// Register layouts of the tile index t (11 bits) by thread tau (7 bits) and
// register r (4 bits): A holds tile bits 7..10 in registers, B bits 3..6,
// C bits 0..3.
__device__ __forceinline__ int lay_a(int tau, int r) { return tau | (r << 7); }
__device__ __forceinline__ int lay_b(int tau, int r) { return (tau & 7) | (r << 3) | ((tau >> 3) << 7); }
__device__ __forceinline__ int lay_c(int tau, int r) { return r | (tau << 4); }
// shared-memory slot of tile index t: XOR of t bits 4..6 into bits 0..2, so a
// warp's 32 accesses fall into four conflict-free 128-byte wavefronts in all
// three layouts
__device__ __forceinline__ int swz(int t) { return t ^ ((t >> 4) & 7); }

template <int L>
__device__ __forceinline__ int lay_of(int tau, int r) {
  return L == 0 ? lay_a(tau, r) : L == 1 ? lay_b(tau, r) : lay_c(tau, r);
}

template <int FROM, int TO>
__device__ __forceinline__ void xpose(double2 *sm, int tau, double2 (&a)[kR]) {
#pragma unroll
  for (int r = 0; r < kR; ++r) sm[swz(lay_of<FROM>(tau, r))] = a[r];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) a[r] = sm[swz(lay_of<TO>(tau, r))];
  __syncthreads();
}

template <int FROM, int TO>
__device__ __forceinline__ void xpose2(double2 *sm, int tau, double2 (&a)[kR], double2 (&l)[kR]) {
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    sm[swz(lay_of<FROM>(tau, r))] = a[r];
    sm[kTile + swz(lay_of<FROM>(tau, r))] = l[r];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    a[r] = sm[swz(lay_of<TO>(tau, r))];
    l[r] = sm[kTile + swz(lay_of<TO>(tau, r))];
  }
  __syncthreads();
}

// Forward gate in the form the shard kernels apply it: (1/f) RZ'(phi) RY(theta)
// with RZ' = diag(1, e^{i phi}) = e^{i phi/2} RZ(phi) and f = cos(theta/2) or
// sin(theta/2), whichever is larger in magnitude, so that RY/f is
// [[1, -k], [k, 1]] (k = tan, mode +1) or [[k, -1], [1, k]] (k = cot, mode -1):
// four multiply-adds for the rotation and four for the phase instead of
// sixteen.  Within a layer the state differs from the true one by the scalar
// prod 1/f times a global phase; ring_pack, which ends every layer's gates,
// multiplies by the layer's prod f, so each layer starts at the true scale
// (no growth over many layers) and only the global phase remains, which
// cancels in the energy and in every gradient sum.
// fwd_coef: (cos t/2, sin t/2, cos p/2, sin p/2) -> (k, mode, cos p, sin p)
__device__ __forceinline__ double4 fwd_coef(const double4 c) {
  const bool plus = fabs(c.x) >= fabs(c.y);
  return make_double4(plus ? c.y / c.x : c.x / c.y, plus ? 1.0 : -1.0, c.z * c.z - c.w * c.w, 2.0 * c.z * c.w);
}
// adj_coef: (cos t/2, sin t/2, cos p, sin p) for the exact adjoint (RY^dagger
// and diag(1, e^{-i phi}) = e^{-i phi/2} RZ^dagger: the common phase of psi and
// lambda cancels in every gradient sum)
__device__ __forceinline__ double4 adj_coef(const double4 c) {
  return make_double4(c.x, c.y, c.z * c.z - c.w * c.w, 2.0 * c.z * c.w);
}

__device__ __forceinline__ void phase_mul(double2 &x, double cp, double sp) {
  x = make_double2(fma(x.x, cp, -x.y * sp), fma(x.x, sp, x.y * cp));
}

// (x0, x1) <- (1/f) RZ'(phi) RY(theta) (x0, x1), c = fwd_coef(...)
template <bool PLUS>
__device__ __forceinline__ void rot_pair(const double4 c, double2 &x0, double2 &x1) {
  const double k = c.x;
  double2 y0, y1;
  if (PLUS) {
    y0 = make_double2(fma(-k, x1.x, x0.x), fma(-k, x1.y, x0.y));
    y1 = make_double2(fma(k, x0.x, x1.x), fma(k, x0.y, x1.y));
  } else {
    y0 = make_double2(fma(k, x0.x, -x1.x), fma(k, x0.y, -x1.y));
    y1 = make_double2(fma(k, x1.x, x0.x), fma(k, x1.y, x0.y));
  }
  phase_mul(y1, c.z, c.w);
  x0 = y0;
  x1 = y1;
}

// Inverse walk of one wire on a psi pair (a0, a1) and lambda pair (l0, l1)
// taken after the wire's RZ RY: the phi and theta sums of the reference's
// inverse walk, RZ^dagger and RY^dagger applied in between.
__device__ __forceinline__ void unrot_pair(const double4 c, double2 &a0, double2 &a1, double2 &l0, double2 &l1,
                                           double &gt, double &gp) {
  gp += fma(l0.x, a0.y, -l0.y * a0.x) - fma(l1.x, a1.y, -l1.y * a1.x);
  phase_mul(a1, c.z, -c.w);  // diag(1, e^{-i phi}) on psi and lambda
  phase_mul(l1, c.z, -c.w);
  gt += fma(l1.x, a0.x, l1.y * a0.y) - fma(l0.x, a1.x, l0.y * a1.y);
  const double2 b0 = make_double2(c.x * a0.x + c.y * a1.x, c.x * a0.y + c.y * a1.y);
  const double2 b1 = make_double2(c.x * a1.x - c.y * a0.x, c.x * a1.y - c.y * a0.y);
  const double2 m0 = make_double2(c.x * l0.x + c.y * l1.x, c.x * l0.y + c.y * l1.y);
  const double2 m1 = make_double2(c.x * l1.x - c.y * l0.x, c.x * l1.y - c.y * l0.y);
  a0 = b0;
  a1 = b1;
  l0 = m0;
  l1 = m1;
}

// As unrot_pair with RY^dagger in tangent form, RY^dagger / f: [[1, k], [-k, 1]]
// (PLUS, f = cos, k = tan) or [[k, 1], [-1, k]] (f = sin, k = cot); c =
// (k, mode, cos phi, sin phi).  psi and lambda come out scaled by 1/f each, so
// the sums of every later gate of the pass are 1/f^2 too large; the pass
// corrects each gate's sums by the product of f^2 over the gates before it and
// restores psi and lambda with the product of f when it stores them.
template <bool PLUS>
__device__ __forceinline__ void unrot_pair_tan(const double4 c, double2 &a0, double2 &a1, double2 &l0, double2 &l1,
                                               double &gt, double &gp) {
  gp += fma(l0.x, a0.y, -l0.y * a0.x) - fma(l1.x, a1.y, -l1.y * a1.x);
  phase_mul(a1, c.z, -c.w);  // diag(1, e^{-i phi}) on psi and lambda
  phase_mul(l1, c.z, -c.w);
  gt += fma(l1.x, a0.x, l1.y * a0.y) - fma(l0.x, a1.x, l0.y * a1.y);
  const double k = c.x;
  double2 b0, b1, m0, m1;
  if (PLUS) {
    b0 = make_double2(fma(k, a1.x, a0.x), fma(k, a1.y, a0.y));
    b1 = make_double2(fma(-k, a0.x, a1.x), fma(-k, a0.y, a1.y));
    m0 = make_double2(fma(k, l1.x, l0.x), fma(k, l1.y, l0.y));
    m1 = make_double2(fma(-k, l0.x, l1.x), fma(-k, l0.y, l1.y));
  } else {
    b0 = make_double2(fma(k, a0.x, a1.x), fma(k, a0.y, a1.y));
    b1 = make_double2(fma(k, a1.x, -a0.x), fma(k, a1.y, -a0.y));
    m0 = make_double2(fma(k, l0.x, l1.x), fma(k, l0.y, l1.y));
    m1 = make_double2(fma(k, l1.x, -l0.x), fma(k, l1.y, -l0.y));
  }
  a0 = b0;
  a1 = b1;
  l0 = m0;
  l1 = m1;
}

// The gate helpers act on tile bits TB0..TB0+NB-1, held in register bits
// RB0..RB0+NB-1 of the current layout.
template <int TB0, int NB, int RB0 = 0>
__device__ __forceinline__ void fwd_gates(const TileArgs &A, const double4 *cf, double2 (&a)[kR]) {
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (A.wire[TB0 + j] < 0) continue;
    const double4 c = cf[TB0 + j];
    const int m = 1 << (RB0 + j);
    if (c.y > 0.0) {
#pragma unroll
      for (int r = 0; r < kR; ++r)
        if (!(r & m)) rot_pair<true>(c, a[r], a[r | m]);
    } else {
#pragma unroll
      for (int r = 0; r < kR; ++r)
        if (!(r & m)) rot_pair<false>(c, a[r], a[r | m]);
    }
  }
}

// adjoint gates of tile bits TB0..TB0+NB-1 (tangent form, cf from
// adj_tan_coef); their sums are corrected by kap (the product of f^2 of the
// pass's earlier gates), reduced over the warp and added to the warp's row of
// the CTA record
template <int TB0, int NB, int RB0 = 0>
__device__ __forceinline__ void adj_gates(const TileArgs &A, const double4 *cf, const double *kap, double2 (&a)[kR],
                                          double2 (&l)[kR], double *rec_row, int lane) {
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (A.wire[TB0 + j] < 0) continue;
    const double4 c = cf[TB0 + j];
    const int m = 1 << (RB0 + j);
    // four partial sums each: the eight pairs' terms are not one dependent chain
    double gt4[4] = {0.0, 0.0, 0.0, 0.0}, gp4[4] = {0.0, 0.0, 0.0, 0.0};
    if (c.y > 0.0) {
      int q = 0;
#pragma unroll
      for (int r = 0; r < kR; ++r)
        if (!(r & m)) {
          unrot_pair_tan<true>(c, a[r], a[r | m], l[r], l[r | m], gt4[q & 3], gp4[q & 3]);
          ++q;
        }
    } else {
      int q = 0;
#pragma unroll
      for (int r = 0; r < kR; ++r)
        if (!(r & m)) {
          unrot_pair_tan<false>(c, a[r], a[r | m], l[r], l[r | m], gt4[q & 3], gp4[q & 3]);
          ++q;
        }
    }
    double gt = (gt4[0] + gt4[1]) + (gt4[2] + gt4[3]);
    double gp = (gp4[0] + gp4[1]) + (gp4[2] + gp4[3]);
    gt = warp_sum(gt);
    gp = warp_sum(gp);
    if (lane == 0) {
      const double kp = kap[TB0 + j];
      rec_row[2 * (TB0 + j)] += gt * kp;
      rec_row[2 * (TB0 + j) + 1] += gp * kp;
    }
  }
}

__device__ __forceinline__ u32 tile_base(const TileArgs &A, u32 k) {
  u32 base = 0;
  for (int i = 0; i < A.num_runs; ++i) {
    base |= (k & ((1u << A.run_len[i]) - 1u)) << A.run_start[i];
    k >>= A.run_len[i];
  }
  return base;
}

// offsets of layout B (thread bits = tile bits 0..2 and 7..10, register bits =
// tile bits 3..6): a pass whose last gates are in layout B stores from there
// (rows of 128 contiguous bytes per register, the two halves of each 256-byte
// row from consecutive registers) instead of transposing back to layout A
__device__ __forceinline__ u32 thread_off_b(const TileArgs &A, int tau) {
  u32 o = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if ((tau >> j) & 1) o |= 1u << A.bits[j];
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if ((tau >> (3 + j)) & 1) o |= 1u << A.bits[7 + j];
  return o;
}
__device__ __forceinline__ u32 reg_off_b(const TileArgs &A, int r) {
  return ((r & 1) ? 1u << A.bits[3] : 0u) | ((r & 2) ? 1u << A.bits[4] : 0u) | ((r & 4) ? 1u << A.bits[5] : 0u) |
         ((r & 8) ? 1u << A.bits[6] : 0u);
}

__device__ __forceinline__ u32 reg_off(int r, const u32 (&rb)[4]) {
  return ((r & 1) ? rb[0] : 0u) | ((r & 2) ? rb[1] : 0u) | ((r & 4) ? rb[2] : 0u) | ((r & 8) ? rb[3] : 0u);
}

__global__ void __launch_bounds__(kRotThreads, kRotCtasPerSm) rot_kernel(const __grid_constant__ TileArgs A,
                                                          const double4 *__restrict__ coef,
                                                          double2 *__restrict__ psi) {
  __shared__ double2 sm[kTile];
  __shared__ double4 cf[kT];
  const int tau = threadIdx.x;
  if (tau < kT) cf[tau] = A.wire[tau] >= 0 ? fwd_coef(coef[A.layer * A.n + A.wire[tau]]) : make_double4(0.0, 1.0, 1.0, 0.0);
  u32 otau = 0;
#pragma unroll
  for (int j = 0; j < 7; ++j)
    if ((tau >> j) & 1) otau |= 1u << A.bits[j];
  u32 rb[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) rb[j] = 1u << A.bits[7 + j];
  __syncthreads();
  for (u32 k = blockIdx.x; k < A.num_tiles; k += gridDim.x) {
    const u32 base = tile_base(A, k) | otau;
    double2 a[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) a[r] = __ldcs(&psi[base | reg_off(r, rb)]);
    fwd_gates<7, 4>(A, cf, a);
    bool from_b = false;
    if (A.need_c) {  // A -> C (tile bits 0..3) -> B (tile bits 4..6), stored from B
      xpose<0, 2>(sm, tau, a);
      fwd_gates<0, 4>(A, cf, a);
      xpose<2, 1>(sm, tau, a);
      fwd_gates<4, 3, 1>(A, cf, a);
      from_b = true;
    } else if (A.need_b) {
      xpose<0, 1>(sm, tau, a);
      fwd_gates<3, 4>(A, cf, a);
      from_b = true;
    }
    u32 sbase = base;  // store addresses derived again (not kept live across the gates)
    asm volatile("" : "+r"(sbase));
    if (from_b) {
      const u32 ob = (sbase ^ otau) | thread_off_b(A, tau);
#pragma unroll
      for (int r = 0; r < kR; ++r) __stcs(&psi[ob | reg_off_b(A, r)], a[r]);
    } else {
#pragma unroll
      for (int r = 0; r < kR; ++r) __stcs(&psi[sbase | reg_off(r, rb)], a[r]);
    }
  }
}

__global__ void __launch_bounds__(kRotThreads, kAdjCtasPerSm) rot_adjoint_kernel(const __grid_constant__ TileArgs A,
                                                                  const double4 *__restrict__ coef,
                                                                  double2 *__restrict__ psi,
                                                                  double2 *__restrict__ lam,
                                                                  double *__restrict__ records) {
  extern __shared__ double2 sm2[];
  __shared__ double4 cf[kT];
  __shared__ double kap[kT];
  __shared__ double pass_f;
  __shared__ double rec[kRotThreads / 32][kRec];
  const int tau = threadIdx.x, lane = tau & 31, warp = tau >> 5;
  if (tau == 0) {
    // the pass's gates in the order they are undone: layout A (tile bits
    // 7..10), then C (0..3) and B (4..6) when bits 0..2 carry gates, else B
    // (3..6); bits 0..2 carry none in the second case, so one list serves both
    constexpr int order[kT] = {7, 8, 9, 10, 0, 1, 2, 3, 4, 5, 6};
    double run = 1.0, fprod = 1.0;
    for (int i = 0; i < kT; ++i) {
      const int tb = order[i];
      cf[tb] = make_double4(0.0, 1.0, 1.0, 0.0);
      kap[tb] = 1.0;
      if (A.wire[tb] < 0) continue;
      const double4 c = coef[A.layer * A.n + A.wire[tb]];
      const bool plus = fabs(c.x) >= fabs(c.y);
      const double f = plus ? c.x : c.y;
      cf[tb] = make_double4(plus ? c.y / c.x : c.x / c.y, plus ? 1.0 : -1.0, c.z * c.z - c.w * c.w, 2.0 * c.z * c.w);
      kap[tb] = run;
      run *= f * f;
      fprod *= f;
    }
    pass_f = fprod;
  }
  for (int i = tau; i < (kRotThreads / 32) * kRec; i += kRotThreads) (&rec[0][0])[i] = 0.0;
  u32 otau = 0;
#pragma unroll
  for (int j = 0; j < 7; ++j)
    if ((tau >> j) & 1) otau |= 1u << A.bits[j];
  u32 rb[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) rb[j] = 1u << A.bits[7 + j];
  __syncthreads();
  for (u32 k = blockIdx.x; k < A.num_tiles; k += gridDim.x) {
    const u32 base = tile_base(A, k) | otau;
    double2 a[kR], l[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      a[r] = __ldcs(&psi[base | reg_off(r, rb)]);
      l[r] = __ldcs(&lam[base | reg_off(r, rb)]);
    }
    adj_gates<7, 4>(A, cf, kap, a, l, rec[warp], lane);
    bool from_b = false;
    if (A.need_c) {  // A -> C (tile bits 0..3) -> B (tile bits 4..6), stored from B
      xpose2<0, 2>(sm2, tau, a, l);
      adj_gates<0, 4>(A, cf, kap, a, l, rec[warp], lane);
      xpose2<2, 1>(sm2, tau, a, l);
      adj_gates<4, 3, 1>(A, cf, kap, a, l, rec[warp], lane);
      from_b = true;
    } else if (A.need_b) {
      xpose2<0, 1>(sm2, tau, a, l);
      adj_gates<3, 4>(A, cf, kap, a, l, rec[warp], lane);
      from_b = true;
    }
    const double sf = pass_f;  // back to the true scale
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      a[r] = make_double2(sf * a[r].x, sf * a[r].y);
      l[r] = make_double2(sf * l[r].x, sf * l[r].y);
    }
    // the store addresses are derived again here rather than kept live from
    // the loads (32 addresses would not fit next to the 64 amplitudes)
    u32 sbase = base;
    asm volatile("" : "+r"(sbase));
    if (from_b) {
      const u32 ob = (sbase ^ otau) | thread_off_b(A, tau);
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        __stcs(&psi[ob | reg_off_b(A, r)], a[r]);
        __stcs(&lam[ob | reg_off_b(A, r)], l[r]);
      }
    } else {
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        __stcs(&psi[sbase | reg_off(r, rb)], a[r]);
        __stcs(&lam[sbase | reg_off(r, rb)], l[r]);
      }
    }
  }
  __syncthreads();
  if (tau < kRec) {
    double s = 0.0;
    for (int w = 0; w < kRotThreads / 32; ++w) s += rec[w][tau];
    records[static_cast<size_t>(blockIdx.x) * kRec + tau] = s;
  }
}

// result[2 + 2(layer n + wire[j]) + {0, 1}] = sum over the CTA records of the
// pass, in CTA order
__global__ void rot_records_kernel(const __grid_constant__ TileArgs A, const double *__restrict__ records,
                                   int grid, double *__restrict__ result) {
  const int i = threadIdx.x;
  if (i >= kRec || A.wire[i >> 1] < 0) return;
  double s = 0.0;
  for (int b = 0; b < grid; ++b) s += records[static_cast<size_t>(b) * kRec + i];
  result[2 + 2 * (A.layer * A.n + A.wire[i >> 1]) + (i & 1)] = s;
}

// ---------------------------------------------------------------- energy (C)
// lambda = (sum_w -Z_w Z_{w+1} - h sum_{w < n-g} X_w) psi on the shard of
// rank `rank` in layout C (reference cpp/ising_cuda_kernels.cu:313-358, the X
// terms of the local wires only), on the tiles of the local rotation passes:
// the first pass (tile bits = local bits 0..10) starts lambda with the ZZ
// diagonal, every pass subtracts h psi[v ^ e_b] for the wires on its tile
// bits, partners taken from registers in the three layouts of rot_kernel, so
// psi is read once per pass and each partner needs no further memory access.
// Per-CTA records: the energy share of what the pass added.
template <int TB0, int NB, int RB0 = 0>
__device__ __forceinline__ void xsum_gates(const TileArgs &A, double field, const double2 (&a)[kR],
                                           double2 (&acc)[kR], double (&e4)[4]) {
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (A.wire[TB0 + j] < 0) continue;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const double2 p = a[r ^ (1 << (RB0 + j))];
      acc[r].x = fma(-field, p.x, acc[r].x);
      acc[r].y = fma(-field, p.y, acc[r].y);
      e4[r & 3] = fma(-field, fma(a[r].x, p.x, a[r].y * p.y), e4[r & 3]);
    }
  }
}

template <bool FIRST>
__global__ void __launch_bounds__(kRotThreads, kAdjCtasPerSm) energy_tile_kernel(const __grid_constant__ TileArgs A,
                                                                                 int rank, double field,
                                                                                 const double2 *__restrict__ psi,
                                                                                 double2 *__restrict__ lam,
                                                                                 double *__restrict__ records) {
  extern __shared__ double2 sm2[];
  __shared__ double red[kRotThreads / 32];
  const int tau = threadIdx.x;
  u32 otau = 0;
#pragma unroll
  for (int j = 0; j < 7; ++j)
    if ((tau >> j) & 1) otau |= 1u << A.bits[j];
  u32 rb[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) rb[j] = 1u << A.bits[7 + j];
  const u64 full = (u64{1} << A.n) - 1;
  const u64 rhi = static_cast<u64>(rank) << A.nloc;
  double e4[4] = {0.0, 0.0, 0.0, 0.0};  // partial sums (independent chains)
  for (u32 k = blockIdx.x; k < A.num_tiles; k += gridDim.x) {
    const u32 base = tile_base(A, k) | otau;
    double2 a[kR], acc[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const u32 off = base | reg_off(r, rb);
      a[r] = __ldcs(&psi[off]);
      if (FIRST) {
        const u64 y = rhi | off;
        const u64 rot = ((y << 1) & full) | (y >> (A.n - 1));
        const double d = static_cast<double>(2 * __popcll(y ^ rot) - A.n);
        acc[r] = make_double2(d * a[r].x, d * a[r].y);
        e4[r & 3] = fma(d, fma(a[r].x, a[r].x, a[r].y * a[r].y), e4[r & 3]);
      } else {
        acc[r] = __ldcs(&lam[off]);
      }
    }
    xsum_gates<7, 4>(A, field, a, acc, e4);
    bool from_b = false;
    if (A.need_c) {  // A -> C (tile bits 0..3) -> B (tile bits 4..6), stored from B
      xpose2<0, 2>(sm2, tau, a, acc);
      xsum_gates<0, 4>(A, field, a, acc, e4);
      xpose2<2, 1>(sm2, tau, a, acc);
      xsum_gates<4, 3, 1>(A, field, a, acc, e4);
      from_b = true;
    } else if (A.need_b) {
      xpose2<0, 1>(sm2, tau, a, acc);
      xsum_gates<3, 4>(A, field, a, acc, e4);
      from_b = true;
    }
    u32 sbase = base;  // store addresses derived again (not kept live across the sums)
    asm volatile("" : "+r"(sbase));
    if (from_b) {
      const u32 ob = (sbase ^ otau) | thread_off_b(A, tau);
#pragma unroll
      for (int r = 0; r < kR; ++r) __stcs(&lam[ob | reg_off_b(A, r)], acc[r]);
    } else {
#pragma unroll
      for (int r = 0; r < kR; ++r) __stcs(&lam[sbase | reg_off(r, rb)], acc[r]);
    }
  }
  const double e = warp_sum((e4[0] + e4[1]) + (e4[2] + e4[3]));
  if ((tau & 31) == 0) red[tau >> 5] = e;
  __syncthreads();
  if (tau == 0) {
    double sum = 0.0;
    for (int w = 0; w < kRotThreads / 32; ++w) sum += red[w];
    records[blockIdx.x] = sum;
  }
}

// result[0] = (first pass) or += the pass's CTA records, in CTA order
__global__ void energy_records_kernel(const double *__restrict__ records, int grid, int first,
                                      double *__restrict__ result) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < grid; ++b) s += records[b];
  result[0] = first ? s : result[0] + s;
}

// ---------------------------------------------------------------- ring exchange
constexpr int kXThreads = 256;

// ring map P (bit k >= 1: XOR of bits 0..k; bit 0: XOR of bits 1..n-1) and
// its inverse, for n <= 63
__device__ __forceinline__ u64 ring_fwd(u64 x, int n) {
  const u64 full = (u64{1} << n) - 1;
  u64 s = x;
  s ^= s << 1;
  s ^= s << 2;
  s ^= s << 4;
  s ^= s << 8;
  s ^= s << 16;
  s ^= s << 32;
  s &= full;
  return (s & ~u64{1}) | static_cast<u64>(__popcll(x >> 1) & 1);
}
__device__ __forceinline__ u64 ring_inv(u64 y, int n) {
  const u64 full = (u64{1} << n) - 1;
  u64 x = (y ^ (y << 1)) & full;
  if ((y >> (n - 1)) & 1) x ^= 3;
  return x;
}
// G-bit prefix XOR and its inverse
template <int G>
__device__ __forceinline__ int prefix_xor(int t) {
  t ^= t << 1;
  t ^= t << 2;
  return t & ((1 << G) - 1);
}
template <int G>
__device__ __forceinline__ int prefix_inv(int z) {
  return (z ^ (z << 1)) & ((1 << G) - 1);
}

// Sender side of the forward ring exchange, in layout S.  Thread u (x bits
// [0, n-2g)) holds the 2^G amplitudes of x bits [n-g, n) = t (local offset
// u + B t), rotates wires n-G..n-1 on them, and sends the amplitude of t to
// the rank owning P(x): rank bit j = pi ^ t_0 ^ ... ^ t_j with pi the parity
// of x bits [0, n-G) (u and this rank's bits), position u of that chunk.
template <int G>
__global__ void __launch_bounds__(kXThreads) ring_pack_kernel(const double2 *__restrict__ psi_s,
                                                              double2 *__restrict__ send, int n, int rank,
                                                              int layer, const double4 *__restrict__ coef,
                                                              u64 B) {
  constexpr int N = 1 << G;
  __shared__ double layer_f;  // prod over the layer's wires of f (signed)
  if (threadIdx.x == 0) {
    double p = 1.0;
    for (int w = 0; w < n; ++w) {
      const double4 c = coef[layer * n + w];
      p *= fabs(c.x) >= fabs(c.y) ? c.x : c.y;
    }
    layer_f = p;
  }
  double4 cf[G > 0 ? G : 1];
#pragma unroll
  for (int j = 0; j < G; ++j) cf[j] = fwd_coef(coef[layer * n + (n - G + j)]);
  const int rpar = __popc(rank) & 1;
  __syncthreads();
  const double sf = layer_f;
  for (u64 u = blockIdx.x * static_cast<u64>(kXThreads) + threadIdx.x; u < B;
       u += static_cast<u64>(gridDim.x) * kXThreads) {
    double2 a[N];
#pragma unroll
    for (int t = 0; t < N; ++t) {
      a[t] = __ldcs(&psi_s[u + B * t]);
      a[t] = make_double2(sf * a[t].x, sf * a[t].y);
    }
#pragma unroll
    for (int j = 0; j < G; ++j)
#pragma unroll
      for (int t = 0; t < N; ++t)
        if (!(t & (1 << j))) {
          if (cf[j].y > 0.0)
            rot_pair<true>(cf[j], a[t], a[t | (1 << j)]);
          else
            rot_pair<false>(cf[j], a[t], a[t | (1 << j)]);
        }
    const int pi = (__popcll(u) & 1) ^ rpar;
#pragma unroll
    for (int t = 0; t < N; ++t) {
      const int rd = prefix_xor<G>(t) ^ (pi ? N - 1 : 0);
      __stcs(&send[B * rd + u], a[t]);
    }
  }
}

// Receiver side of the forward ring exchange: psi_c[v] for y = (rank, v) is
// the amplitude of x = P^-1(y), found in chunk rank_S(x) at x bits [0, n-2G).
template <int G>
__global__ void __launch_bounds__(kXThreads) ring_unpack_kernel(const double2 *__restrict__ recv,
                                                                double2 *__restrict__ psi_c, int n, int rank,
                                                                u64 B) {
  constexpr int N = 1 << G;
  const int nloc = n - G;
  const u64 size = u64{1} << nloc;
  for (u64 v = blockIdx.x * static_cast<u64>(kXThreads) + threadIdx.x; v < size;
       v += static_cast<u64>(gridDim.x) * kXThreads) {
    const u64 x = ring_inv((static_cast<u64>(rank) << nloc) | v, n);
    const u64 rs = (x >> (n - 2 * G)) & (N - 1);
    // a warp's 32 reads fall in one 64-amplitude window, half of each 32-byte
    // sector; the other half is read by the warp with y bit 5 flipped, so the
    // loads keep their lines in L1 (__ldg) rather than streaming them
    __stcs(&psi_c[v], __ldg(&recv[rs * B + (x & (B - 1))]));
  }
}

// Sender side of the backward ring exchange, in layout C: position u of the
// chunk for rank r_s holds psi and lambda at y = P(x), x = (u, r_s, t) with t
// the top bits that send x to this rank.
template <int G>
__global__ void __launch_bounds__(kXThreads) ring_pack_adjoint_kernel(const double2 *__restrict__ psi_c,
                                                                      const double2 *__restrict__ lam_c,
                                                                      double2 *__restrict__ send_psi,
                                                                      double2 *__restrict__ send_lam, int n,
                                                                      int rank, u64 B) {
  constexpr int N = 1 << G;
  const int nloc = n - G;
  const u64 lmask = (u64{1} << nloc) - 1;
  const u64 size = B * N;
  for (u64 q = blockIdx.x * static_cast<u64>(kXThreads) + threadIdx.x; q < size;
       q += static_cast<u64>(gridDim.x) * kXThreads) {
    const u64 u = q & (B - 1);
    const int rs = static_cast<int>(q / B);
    const int pi = (__popcll(u) ^ __popc(rs)) & 1;
    const int t = prefix_inv<G>(rank ^ (pi ? N - 1 : 0));
    const u64 x = u | (static_cast<u64>(rs) << (n - 2 * G)) | (static_cast<u64>(t) << nloc);
    const u64 v = ring_fwd(x, n) & lmask;
    __stcs(&send_psi[q], __ldcs(&psi_c[v]));
    __stcs(&send_lam[q], __ldcs(&lam_c[v]));
  }
}

// Receiver side of the backward ring exchange, in layout S: the 2^G
// amplitudes of thread u arrive one per sender rank; optionally the X terms
// of wires n-G..n-1 in the pre-ring frame (masks {w, w+1} on t bits j, j+1;
// {0, 1, n-1} reaches the thread u ^ 3 of the same warp), then the adjoint of
// wires n-G..n-1 of `layer` with their gradient sums.  Record per CTA:
// [0] field-term energy, [1 + 2j + {0, 1}] theta / phi sums of wire n-G+j.
template <int G>
__global__ void __launch_bounds__(kXThreads) ring_unpack_adjoint_kernel(
    const double2 *__restrict__ recv_psi, const double2 *__restrict__ recv_lam, double2 *__restrict__ psi_s,
    double2 *__restrict__ lam_s, int n, int rank, int layer, const double4 *__restrict__ coef, double field,
    int add_field, u64 B, double *__restrict__ records) {
  constexpr int N = 1 << G;
  constexpr int kRecX = 1 + 2 * G;
  __shared__ double red[kXThreads / 32][kRecX];
  double4 cf[G > 0 ? G : 1];
  if (layer >= 0) {
#pragma unroll
    for (int j = 0; j < G; ++j) cf[j] = adj_coef(coef[layer * n + (n - G + j)]);
  }
  const int rpar = __popc(rank) & 1;
  double acc[kRecX];
#pragma unroll
  for (int i = 0; i < kRecX; ++i) acc[i] = 0.0;
  for (u64 u = blockIdx.x * static_cast<u64>(kXThreads) + threadIdx.x; u < B;
       u += static_cast<u64>(gridDim.x) * kXThreads) {
    const int pi = (__popcll(u) & 1) ^ rpar;
    double2 a[N], l[N];
#pragma unroll
    for (int t = 0; t < N; ++t) {
      const int rd = prefix_xor<G>(t) ^ (pi ? N - 1 : 0);
      a[t] = __ldcs(&recv_psi[B * rd + u]);
      l[t] = __ldcs(&recv_lam[B * rd + u]);
    }
    if constexpr (G > 0) {
      if (add_field) {
      double2 add[N];
#pragma unroll
      for (int t = 0; t < N; ++t) {
        const double2 p = a[t ^ (1 << (G - 1))];
        add[t] = make_double2(__shfl_xor_sync(0xffffffffu, p.x, 3), __shfl_xor_sync(0xffffffffu, p.y, 3));
      }
#pragma unroll
      for (int j = 0; j + 1 < G; ++j)
#pragma unroll
        for (int t = 0; t < N; ++t) {
          add[t].x += a[t ^ (3 << j)].x;
          add[t].y += a[t ^ (3 << j)].y;
        }
#pragma unroll
      for (int t = 0; t < N; ++t) {
        l[t].x = fma(-field, add[t].x, l[t].x);
        l[t].y = fma(-field, add[t].y, l[t].y);
        acc[0] -= field * fma(a[t].x, add[t].x, a[t].y * add[t].y);
      }
      }
    }
    if (layer >= 0) {
#pragma unroll
      for (int j = G - 1; j >= 0; --j)
#pragma unroll
        for (int t = 0; t < N; ++t)
          if (!(t & (1 << j)))
            unrot_pair(cf[j], a[t], a[t | (1 << j)], l[t], l[t | (1 << j)], acc[1 + 2 * j], acc[2 + 2 * j]);
    }
#pragma unroll
    for (int t = 0; t < N; ++t) {
      __stcs(&psi_s[u + B * t], a[t]);
      __stcs(&lam_s[u + B * t], l[t]);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < kRecX; ++i) {
    const double s = warp_sum(acc[i]);
    if (lane == 0) red[warp][i] = s;
  }
  __syncthreads();
  if (threadIdx.x < kRecX) {
    double s = 0.0;
    for (int w = 0; w < kXThreads / 32; ++w) s += red[w][threadIdx.x];
    records[static_cast<size_t>(blockIdx.x) * kRecX + threadIdx.x] = s;
  }
}

// result[1] = field-term energy (if add_field), gradient of wires n-G..n-1 of
// `layer` (if layer >= 0), from the CTA records in CTA order
__global__ void ring_records_kernel(const double *__restrict__ records, int grid, int G, int n, int layer,
                                    int add_field, double *__restrict__ result) {
  const int i = threadIdx.x, rec = 1 + 2 * G;
  if (i >= rec) return;
  if (i == 0 && !add_field) return;
  if (i > 0 && layer < 0) return;
  double s = 0.0;
  for (int b = 0; b < grid; ++b) s += records[static_cast<size_t>(b) * rec + i];
  if (i == 0)
    result[1] = s;
  else
    result[2 + 2 * (layer * n + (n - G + (i - 1) / 2)) + ((i - 1) & 1)] = s;
}

__global__ void init_kernel(double2 *__restrict__ psi, u64 size, int rank) {
  for (u64 i = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; i < size;
       i += static_cast<u64>(gridDim.x) * blockDim.x)
    psi[i] = make_double2(i == 0 && rank == 0 ? 1.0 : 0.0, 0.0);
}

// ---------------------------------------------------------------- host side
struct ShardError {
  rsv_status status;
  std::string msg;
};

[[noreturn]] void fail(rsv_status s, const std::string &m) { throw ShardError{s, m}; }

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) fail(RSV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename F>
rsv_status shard_guarded(F &&f) {
  try {
    f();
    return RSV_OK;
  } catch (const ShardError &e) {
    set_last_error(e.msg.c_str());
    return e.status;
  }
}

const char *geometry_error(int n, int g) {
  if (g < 0 || g > kMaxG) return "g (log2 of the rank count) must be in 0..3";
  if (n - 2 * g < kMinLowBits) return "num_qubits - 2 g must be at least 12";
  if (n - g > kMaxLocalBits) return "num_qubits - g must be at most 31 (shard offsets are 31-bit)";
  return nullptr;
}

void check_geometry(int n, int g) {
  if (const char *m = geometry_error(n, g)) fail(RSV_ERR_INVALID_ARGUMENT, m);
}

void check_rank(int g, int rank) {
  if (rank < 0 || rank >= (1 << g)) fail(RSV_ERR_INVALID_ARGUMENT, "rank out of range for 2^g ranks");
}

void check_ptr(const void *p, const char *name) {
  if (p == nullptr) fail(RSV_ERR_INVALID_ARGUMENT, std::string(name) + " is null");
}

void check_layer(int L, int layer, bool allow_none) {
  if (L < 1) fail(RSV_ERR_INVALID_ARGUMENT, "num_layers must be at least 1");
  if (layer >= L || layer < (allow_none ? -1 : 0)) fail(RSV_ERR_INVALID_ARGUMENT, "layer out of range");
}

int num_sms() {
  int dev = 0, sms = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  return std::max(1, sms);
}

// CTAs of the local passes and of the ring kernels: at most this many, so the
// records fit the scratch that rsv_shard_scratch_doubles reports
constexpr int kMaxCtasPerSm = 8;
constexpr int kMaxSms = 256;
constexpr size_t kMaxGrid = static_cast<size_t>(kMaxCtasPerSm) * kMaxSms;

int grid_for(u64 units, int per_sm) {
  const u64 g = std::min<u64>(units, static_cast<u64>(std::min(num_sms(), kMaxSms)) * per_sm);
  return static_cast<int>(std::max<u64>(1, g));
}

// The passes that rotate wires 0..nloc-1 of one layer: the first tile holds
// local bits 0..10 (all rotated), the next ones local bits 0..3 plus up to
// seven further wires (the tile filled up with bits 4..10, not rotated).
int local_passes(int n, int nloc, int layer, TileArgs *out) {
  int count = 0;
  auto make = [&](const int *gated, int num_gated, bool low_gated) {
    TileArgs A{};
    A.n = n;
    A.nloc = nloc;
    A.layer = layer;
    bool in[64] = {};
    int bits[kT], k = 0;
    for (int b = 0; b < 4; ++b) {
      bits[k++] = b;
      in[b] = true;
    }
    for (int i = 0; i < num_gated; ++i)
      if (!in[gated[i]]) {
        bits[k++] = gated[i];
        in[gated[i]] = true;
      }
    for (int b = 4; k < kT; ++b)
      if (!in[b]) {
        bits[k++] = b;
        in[b] = true;
      }
    std::sort(bits, bits + kT);
    for (int j = 0; j < kT; ++j) {
      A.bits[j] = bits[j];
      bool g = false;
      for (int i = 0; i < num_gated; ++i) g = g || gated[i] == bits[j];
      if (bits[j] < 4) g = low_gated;
      A.wire[j] = g ? bits[j] : -1;
    }
    for (int p = 0; p < nloc;) {
      if (in[p]) {
        ++p;
        continue;
      }
      int q = p;
      while (q < nloc && !in[q]) ++q;
      A.run_start[A.num_runs] = p;
      A.run_len[A.num_runs] = q - p;
      ++A.num_runs;
      p = q;
    }
    A.num_tiles = 1u << (nloc - kT);
    for (int j = 0; j < 7; ++j) {
      if (A.wire[j] < 0) continue;
      if (j < 3) A.need_c = 1;
      A.need_b = 1;
    }
    out[count++] = A;
  };
  int first[kT];
  for (int b = 0; b < kT; ++b) first[b] = b;
  make(first, kT, true);
  for (int w = kT; w < nloc; w += 7) {
    int gated[7], m = 0;
    for (int i = w; i < std::min(nloc, w + 7); ++i) gated[m++] = i;
    make(gated, m, false);
  }
  return count;
}

constexpr int kMaxPasses = 8;  // 11 + 7 * 3 >= 31 local wires

template <int G>
void launch_ring_pack(int n, int rank, int layer, const double4 *coef, const double2 *src, double2 *dst,
                      cudaStream_t s) {
  const u64 B = u64{1} << (n - 2 * G);
  ring_pack_kernel<G><<<grid_for(B / kXThreads, kMaxCtasPerSm), kXThreads, 0, s>>>(src, dst, n, rank, layer, coef,
                                                                                  B);
}
template <int G>
void launch_ring_unpack(int n, int rank, const double2 *src, double2 *dst, cudaStream_t s) {
  const u64 B = u64{1} << (n - 2 * G);
  ring_unpack_kernel<G><<<grid_for((B << G) / kXThreads, kMaxCtasPerSm), kXThreads, 0, s>>>(src, dst, n, rank, B);
}
template <int G>
void launch_ring_pack_adjoint(int n, int rank, const double2 *psi, const double2 *lam, double2 *sp, double2 *sl,
                              cudaStream_t s) {
  const u64 B = u64{1} << (n - 2 * G);
  ring_pack_adjoint_kernel<G>
      <<<grid_for((B << G) / kXThreads, kMaxCtasPerSm), kXThreads, 0, s>>>(psi, lam, sp, sl, n, rank, B);
}
template <int G>
void launch_ring_unpack_adjoint(int n, int rank, int layer, const double4 *coef, double field, int add_field,
                                const double2 *rp, const double2 *rl, double2 *ps, double2 *ls, double *scratch,
                                double *result, cudaStream_t s) {
  const u64 B = u64{1} << (n - 2 * G);
  const int grid = grid_for(B / kXThreads, kMaxCtasPerSm);
  ring_unpack_adjoint_kernel<G>
      <<<grid, kXThreads, 0, s>>>(rp, rl, ps, ls, n, rank, layer, coef, field, add_field, B, scratch);
  ring_records_kernel<<<1, 32, 0, s>>>(scratch, grid, G, n, layer, add_field, result);
}

cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

}  // namespace
}  // namespace rsv

using namespace rsv;

extern "C" rsv_status rsv_shard_check(int num_qubits, int g) {
  return shard_guarded([&] { check_geometry(num_qubits, g); });
}

extern "C" size_t rsv_shard_scratch_doubles(int num_qubits, int g) {
  if (geometry_error(num_qubits, g)) return 0;
  return kMaxGrid * std::max(kRec, 1 + 2 * kMaxG);
}

extern "C" rsv_status rsv_shard_coef(int num_qubits, int num_layers, const double *d_params, double *d_coef,
                                     void *stream) {
  return shard_guarded([&] {
    if (num_qubits < 1 || num_layers < 1) fail(RSV_ERR_INVALID_ARGUMENT, "num_qubits and num_layers must be positive");
    check_ptr(d_params, "d_params");
    check_ptr(d_coef, "d_coef");
    cuda_check(launch_coef(d_params, reinterpret_cast<double4 *>(d_coef), num_qubits * num_layers, as_stream(stream)),
               "shard coefficient launch");
  });
}

extern "C" rsv_status rsv_shard_init(int num_qubits, int g, int rank, double *d_psi, void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_rank(g, rank);
    check_ptr(d_psi, "d_psi");
    const u64 size = u64{1} << (num_qubits - g);
    init_kernel<<<grid_for(size / 256, 4), 256, 0, as_stream(stream)>>>(reinterpret_cast<double2 *>(d_psi), size,
                                                                        rank);
    cuda_check(cudaGetLastError(), "shard init launch");
  });
}

extern "C" rsv_status rsv_shard_rotate_local(int num_qubits, int g, int layer, const double *d_coef, double *d_psi,
                                             void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    if (layer < 0) fail(RSV_ERR_INVALID_ARGUMENT, "layer out of range");
    check_ptr(d_coef, "d_coef");
    check_ptr(d_psi, "d_psi");
    TileArgs passes[kMaxPasses];
    const int np = local_passes(num_qubits, num_qubits - g, layer, passes);
    for (int p = 0; p < np; ++p) {
      const int grid = grid_for(passes[p].num_tiles, kRotCtasPerSm);
      rot_kernel<<<grid, kRotThreads, 0, as_stream(stream)>>>(passes[p], reinterpret_cast<const double4 *>(d_coef),
                                                              reinterpret_cast<double2 *>(d_psi));
      cuda_check(cudaGetLastError(), "shard rotation launch");
    }
  });
}

extern "C" rsv_status rsv_shard_rotate_local_adjoint(int num_qubits, int g, int num_layers, int layer,
                                                     const double *d_coef, double *d_psi, double *d_lam,
                                                     double *d_scratch, double *d_result, void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_layer(num_layers, layer, false);
    check_ptr(d_coef, "d_coef");
    check_ptr(d_psi, "d_psi");
    check_ptr(d_lam, "d_lam");
    check_ptr(d_scratch, "d_scratch");
    check_ptr(d_result, "d_result");
    static std::atomic<unsigned long long> configured{0};
    cuda_check(set_smem_limit_once(rot_adjoint_kernel, kAdjSmem, configured), "shard adjoint smem limit");
    TileArgs passes[kMaxPasses];
    const int np = local_passes(num_qubits, num_qubits - g, layer, passes);
    for (int p = 0; p < np; ++p) {
      const int grid = grid_for(passes[p].num_tiles, kAdjCtasPerSm);
      rot_adjoint_kernel<<<grid, kRotThreads, kAdjSmem, as_stream(stream)>>>(
          passes[p], reinterpret_cast<const double4 *>(d_coef), reinterpret_cast<double2 *>(d_psi),
          reinterpret_cast<double2 *>(d_lam), d_scratch);
      rot_records_kernel<<<1, 32, 0, as_stream(stream)>>>(passes[p], d_scratch, grid, d_result);
      cuda_check(cudaGetLastError(), "shard adjoint rotation launch");
    }
  });
}

extern "C" rsv_status rsv_shard_energy_local(int num_qubits, int g, int rank, double field, const double *d_psi,
                                             double *d_lam, double *d_scratch, double *d_result, void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_rank(g, rank);
    check_ptr(d_psi, "d_psi");
    check_ptr(d_lam, "d_lam");
    check_ptr(d_scratch, "d_scratch");
    check_ptr(d_result, "d_result");
    static std::atomic<unsigned long long> cfg_first{0}, cfg_rest{0};
    cuda_check(set_smem_limit_once(energy_tile_kernel<true>, kAdjSmem, cfg_first), "shard energy smem limit");
    cuda_check(set_smem_limit_once(energy_tile_kernel<false>, kAdjSmem, cfg_rest), "shard energy smem limit");
    TileArgs passes[kMaxPasses];
    const int np = local_passes(num_qubits, num_qubits - g, 0, passes);
    const auto *psi = reinterpret_cast<const double2 *>(d_psi);
    auto *lam = reinterpret_cast<double2 *>(d_lam);
    for (int p = 0; p < np; ++p) {
      const int grid = grid_for(passes[p].num_tiles, kAdjCtasPerSm);
      if (p == 0)
        energy_tile_kernel<true><<<grid, kRotThreads, kAdjSmem, as_stream(stream)>>>(passes[p], rank, field, psi, lam,
                                                                                     d_scratch);
      else
        energy_tile_kernel<false><<<grid, kRotThreads, kAdjSmem, as_stream(stream)>>>(passes[p], rank, field, psi,
                                                                                      lam, d_scratch);
      energy_records_kernel<<<1, 32, 0, as_stream(stream)>>>(d_scratch, grid, p == 0 ? 1 : 0, d_result);
      cuda_check(cudaGetLastError(), "shard energy launch");
    }
  });
}

extern "C" rsv_status rsv_shard_ring_pack(int num_qubits, int g, int rank, int layer, const double *d_coef,
                                          const double *d_psi_s, double *d_send, void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_rank(g, rank);
    if (layer < 0) fail(RSV_ERR_INVALID_ARGUMENT, "layer out of range");
    check_ptr(d_coef, "d_coef");
    check_ptr(d_psi_s, "d_psi_s");
    check_ptr(d_send, "d_send");
    const auto *coef = reinterpret_cast<const double4 *>(d_coef);
    const auto *src = reinterpret_cast<const double2 *>(d_psi_s);
    auto *dst = reinterpret_cast<double2 *>(d_send);
    const cudaStream_t s = as_stream(stream);
    switch (g) {
      case 0: launch_ring_pack<0>(num_qubits, rank, layer, coef, src, dst, s); break;
      case 1: launch_ring_pack<1>(num_qubits, rank, layer, coef, src, dst, s); break;
      case 2: launch_ring_pack<2>(num_qubits, rank, layer, coef, src, dst, s); break;
      default: launch_ring_pack<3>(num_qubits, rank, layer, coef, src, dst, s); break;
    }
    cuda_check(cudaGetLastError(), "shard ring pack launch");
  });
}

extern "C" rsv_status rsv_shard_ring_unpack(int num_qubits, int g, int rank, const double *d_recv, double *d_psi_c,
                                            void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_rank(g, rank);
    check_ptr(d_recv, "d_recv");
    check_ptr(d_psi_c, "d_psi_c");
    const auto *src = reinterpret_cast<const double2 *>(d_recv);
    auto *dst = reinterpret_cast<double2 *>(d_psi_c);
    const cudaStream_t s = as_stream(stream);
    switch (g) {
      case 0: launch_ring_unpack<0>(num_qubits, rank, src, dst, s); break;
      case 1: launch_ring_unpack<1>(num_qubits, rank, src, dst, s); break;
      case 2: launch_ring_unpack<2>(num_qubits, rank, src, dst, s); break;
      default: launch_ring_unpack<3>(num_qubits, rank, src, dst, s); break;
    }
    cuda_check(cudaGetLastError(), "shard ring unpack launch");
  });
}

extern "C" rsv_status rsv_shard_ring_pack_adjoint(int num_qubits, int g, int rank, const double *d_psi_c,
                                                  const double *d_lam_c, double *d_send_psi, double *d_send_lam,
                                                  void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_rank(g, rank);
    check_ptr(d_psi_c, "d_psi_c");
    check_ptr(d_lam_c, "d_lam_c");
    check_ptr(d_send_psi, "d_send_psi");
    check_ptr(d_send_lam, "d_send_lam");
    const auto *p = reinterpret_cast<const double2 *>(d_psi_c);
    const auto *l = reinterpret_cast<const double2 *>(d_lam_c);
    auto *sp = reinterpret_cast<double2 *>(d_send_psi);
    auto *sl = reinterpret_cast<double2 *>(d_send_lam);
    const cudaStream_t s = as_stream(stream);
    switch (g) {
      case 0: launch_ring_pack_adjoint<0>(num_qubits, rank, p, l, sp, sl, s); break;
      case 1: launch_ring_pack_adjoint<1>(num_qubits, rank, p, l, sp, sl, s); break;
      case 2: launch_ring_pack_adjoint<2>(num_qubits, rank, p, l, sp, sl, s); break;
      default: launch_ring_pack_adjoint<3>(num_qubits, rank, p, l, sp, sl, s); break;
    }
    cuda_check(cudaGetLastError(), "shard ring pack (adjoint) launch");
  });
}

extern "C" rsv_status rsv_shard_ring_unpack_adjoint(int num_qubits, int g, int rank, int num_layers, int layer,
                                                    const double *d_coef, double field, int add_field_terms,
                                                    const double *d_recv_psi, const double *d_recv_lam,
                                                    double *d_psi_s, double *d_lam_s, double *d_scratch,
                                                    double *d_result, void *stream) {
  return shard_guarded([&] {
    check_geometry(num_qubits, g);
    check_rank(g, rank);
    check_layer(num_layers, layer, true);
    if (layer >= 0) check_ptr(d_coef, "d_coef");
    check_ptr(d_recv_psi, "d_recv_psi");
    check_ptr(d_recv_lam, "d_recv_lam");
    check_ptr(d_psi_s, "d_psi_s");
    check_ptr(d_lam_s, "d_lam_s");
    check_ptr(d_scratch, "d_scratch");
    check_ptr(d_result, "d_result");
    const auto *coef = reinterpret_cast<const double4 *>(d_coef);
    const auto *rp = reinterpret_cast<const double2 *>(d_recv_psi);
    const auto *rl = reinterpret_cast<const double2 *>(d_recv_lam);
    auto *ps = reinterpret_cast<double2 *>(d_psi_s);
    auto *ls = reinterpret_cast<double2 *>(d_lam_s);
    const int add = add_field_terms ? 1 : 0;
    const cudaStream_t s = as_stream(stream);
    switch (g) {
      case 0: launch_ring_unpack_adjoint<0>(num_qubits, rank, layer, coef, field, add, rp, rl, ps, ls, d_scratch, d_result, s); break;
      case 1: launch_ring_unpack_adjoint<1>(num_qubits, rank, layer, coef, field, add, rp, rl, ps, ls, d_scratch, d_result, s); break;
      case 2: launch_ring_unpack_adjoint<2>(num_qubits, rank, layer, coef, field, add, rp, rl, ps, ls, d_scratch, d_result, s); break;
      default: launch_ring_unpack_adjoint<3>(num_qubits, rank, layer, coef, field, add, rp, rl, ps, ls, d_scratch, d_result, s); break;
    }
    cuda_check(cudaGetLastError(), "shard ring unpack (adjoint) launch");
  });
}
