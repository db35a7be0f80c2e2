// Device building blocks of the tile passes shared by the single-circuit pass
// kernels (rsv_pass.cu) and the batched circuit kernel (rsv_batch.cu): tile
// geometry, shared-memory swizzle, asynchronous copies, RZ-phase tables,
// tangent-form rotations and the 512-thread layout families of the backward
// pass.
#pragma once

#include "rsv_device.cuh"
#include "rsv_types.h"

// Loads of the per-call tables (RZ phases, product state, tangent forms).
// They go through the read-only data cache by default; a kernel that writes
// its own tables during the launch (the batched kernel) defines
// RSV_TABLES_WRITTEN_IN_KERNEL before including this file to use coherent loads.
#ifdef RSV_TABLES_WRITTEN_IN_KERNEL
#define RSV_TABLE_LOAD(ptr) (*(ptr))
#else
#define RSV_TABLE_LOAD(ptr) __ldg(ptr)
#endif

namespace rsv {
namespace {

using u32 = unsigned int;

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
  double2 v = RSV_TABLE_LOAD(&t[p & 255]);
  v = cmul(v, RSV_TABLE_LOAD(&t[256 + ((p >> 8) & 255)]));
  v = cmul(v, RSV_TABLE_LOAD(&t[512 + ((p >> 16) & 255)]));
  v = cmul(v, RSV_TABLE_LOAD(&t[768 + (p >> 24)]));
  return v;
}

// table4(t, base ^ off[r]) for all registers of a thread: the bytes of the
// index that no register offset touches are looked up and multiplied once.
template <int NR>
__device__ __forceinline__ void table4_regs(const double2 *__restrict__ t, u32 base, const u32 (&off)[NR],
                                            double2 (&out)[NR]) {
  u32 vary = 0;
#pragma unroll
  for (int r = 0; r < NR; ++r) vary |= off[r];
  double2 c = make_double2(1.0, 0.0);
#pragma unroll
  for (int b = 0; b < 4; ++b)
    if (((vary >> (8 * b)) & 255u) == 0) c = cmul(c, RSV_TABLE_LOAD(&t[256 * b + ((base >> (8 * b)) & 255u)]));
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const u32 j = base ^ off[r];
    double2 v = c;
#pragma unroll
    for (int b = 0; b < 4; ++b)
      if (((vary >> (8 * b)) & 255u) != 0) v = cmul(v, RSV_TABLE_LOAD(&t[256 * b + ((j >> (8 * b)) & 255u)]));
    out[r] = v;
  }
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

// Both vectors FROM -> TO at once through two CTA-wide buffers (the staging
// buffers of the backward pass, free between reading a tile and prefetching
// the next): three barriers for the pair.
template <int FROM, int TO>
__device__ __forceinline__ void cta_transpose_pair(double2 *sa, double2 *sb, int lane, int warp,
                                                   double2 (&a)[kR], double2 (&b)[kR]) {
  const int tf = tpart<FROM>(lane, warp), tt = tpart<TO>(lane, warp);
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int s = swz(tf | (r << rbit<FROM>()));
    sa[s] = a[r];
    sb[s] = b[r];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int s = swz(tt | (r << rbit<TO>()));
    a[r] = sa[s];
    b[r] = sb[s];
  }
  __syncthreads();
}

// Backward rotation of the three register bits of layout LY (tile bits
// RB..RB+2): RY^dagger / f in tangent form, one FMA per component,
//   mode +1: [[1,k],[-k,1]]    mode -1: [[k,1],[-1,k]],
// preceded by the theta sum Re(conj(lam1) psi0) - Re(conj(lam0) psi1) of the
// pair in the frame with the layer's RZ removed -- the reference's
// 2 Re<lam_mid|dRY|psi_before> (cpp/ising_cuda_statevector_grad_kernels.cu:289-307)
// simplified; the factors f still pending are corrected in the final reduction.
// km[tb]: the tangent form (k, mode) of the wire gated on tile bit tb, staged
// in shared memory once per pass.
template <int LY>
__device__ __forceinline__ void gates(const PassParams &P, const double2 *km_tb, double2 (&a)[kR],
                                      double2 (&b)[kR], double (&acc)[12]) {
  constexpr int RB = rbit<LY>();
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int w = P.gate_wire[RB + j];
    if (w < 0) continue;
    const double2 km = km_tb[RB + j];
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

}  // namespace
}  // namespace rsv
