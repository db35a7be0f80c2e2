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
#include "rsv_launch.h"
#include "rsv_tile.cuh"

namespace rsv {
namespace {

// Thread layouts of a tile (tile index t has 12 bits):
//   layout 0: lanes -> t bits 0..4,     warps -> 5..7,  registers -> 8..11
//   layout 1: lanes -> t bits 0..3, 8,  warps -> 9..11, registers -> 4..7
//   layout 2: lanes -> t bits 4..8,     warps -> 9..11, registers -> 0..3
// Layouts 0 and 1 keep tile bits 0..3 on the lanes (the c >= 2 contiguous low
// bits of every tile, so at least whole 32-byte sectors, 256-byte segments for
// c >= 4), so both load and store directly; a pass visits 1 (bits 4..7) ->
// [2 (bits 0..3)] -> 0 (bits 8..11): a tile with gates on bits 4..11 needs one
// CTA-wide transpose and the 12-wire tile two.
__device__ __forceinline__ int thread_part(int layout, int lane, int warp) {
  if (layout == 0) return lane | (warp << 5);
  if (layout == 1) return (lane & 15) | ((lane >> 4) << 8) | (warp << 9);
  return (lane << 4) | (warp << 9);
}
__device__ __forceinline__ int reg_shift(int layout) { return layout == 0 ? 8 : (layout == 1 ? 4 : 0); }

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


// Shared memory of the backward kernel (dynamic): staging psi | staging lam |
// transpose buffer (CTA-wide, or 16 warp slices of 256 entries).
constexpr size_t kBwdSmem = 3 * kTileSize * sizeof(double2);
constexpr size_t kFwdSmem = kTileSize * sizeof(double2);
// kLoadMpsP: the 32 per-tile products Y (row pitch 20) after the transpose buffer
constexpr int kMpsYPitch = 20;
constexpr size_t kFwdMpsSmem = kFwdSmem + 32 * kMpsYPitch * sizeof(double2);

// kLoadMpsP source of a forward pass: the bond-4 matrix-product state chi of
// the first three layers at r = P^{-1}(o), for the 4096 indices
// o = cbase + t of a unit tile over index bits 0..11, written to
// trans[swz(t)].  chi(r) = Tr(B0[r0] B1[r1] W[r >> 16]) (byte tables of site
// products, W = B2 B3).  Byte 0 of P^{-1}(o) depends only on bits 0..7 of o and
// bit n-1, bytes 1..3 only on bits 7..31, so the tile needs the 32 products
// Y_{k,s} = B1 W at P^{-1}(cbase + 256 k + 128 s) and its amplitudes are
// out[t0][k] = Tr(Y_{k,t0>>7} B0[r0(t0)]) = sum_e A[t0][e] Y[e] (t = t0 + 256 k,
// A[t0][(i, j)] = B0[r0][j][i]): per warp 32 rows t0 as four m8n8k4 f64
// tensor-core row tiles by two column tiles, Gauss 3-multiply.
__device__ __forceinline__ void mps_tile_p(const PassParams &P, u32 cbase, double2 *trans, double2 *ysm,
                                           int lane, int warp) {
  constexpr int E = 16;
  const int t = threadIdx.x, n = P.n;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int ks = h * 16 + (t >> 4), e = t & 15, i = e >> 2, j = e & 3;  // ks = 16 s + k
    const u64 o = static_cast<u64>(cbase) | (static_cast<u64>(ks & 15) << 8) | (static_cast<u64>(ks >> 4) << 7);
    const u64 r = ring_pinv(o, n);
    const double2 *b1 = P.mps_btab + (256 + ((r >> 8) & 255)) * E;
    const double2 *w = P.mps_wtab + (r >> 16) * E;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const double2 x = __ldg(&b1[i * 4 + m]), y = __ldg(&w[m * 4 + j]);
      acc = make_double2(fma(x.x, y.x, fma(-x.y, y.y, acc.x)), fma(x.x, y.y, fma(x.y, y.x, acc.y)));
    }
    ysm[ks * kMpsYPitch + e] = acc;
  }
  const int fg = lane >> 2, t4 = lane & 3, ys_set = warp >> 2;
  // A = B0[r0][t4][ks] for K index 4 ks + t4 = (i, j) = (ks, t4)
  const double2 *arow[4];
#pragma unroll
  for (int rt = 0; rt < 4; ++rt)
    arow[rt] = P.mps_btab + (ring_pinv(static_cast<u64>(cbase | (32 * warp + 8 * rt + fg)), n) & 255) * E + t4 * 4;
  __syncthreads();
#pragma unroll
  for (int ct = 0; ct < 2; ++ct) {
    double t1[4][2] = {}, t2[4][2] = {}, t3[4][2] = {};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const double2 y = ysm[(16 * ys_set + 8 * ct + fg) * kMpsYPitch + 4 * ks + t4];
      const double ysum = y.x + y.y;
#pragma unroll
      for (int rt = 0; rt < 4; ++rt) {
        const double2 av = __ldg(&arow[rt][ks]);
        mma_f64(t1[rt][0], t1[rt][1], av.x, y.x);
        mma_f64(t2[rt][0], t2[rt][1], av.y, y.y);
        mma_f64(t3[rt][0], t3[rt][1], av.x + av.y, ysum);
      }
    }
#pragma unroll
    for (int rt = 0; rt < 4; ++rt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int tt = 32 * warp + 8 * rt + fg + 256 * (8 * ct + 2 * t4 + e);
        trans[swz(tt)] = make_double2(t1[rt][e] - t2[rt][e], t3[rt][e] - t1[rt][e] - t2[rt][e]);
      }
  }
}

// ---------------------------------------------------------------- backward
// phi-gradient sums of the first backward pass of a layer without a CTA
// barrier per tile.  In layout B0 (registers -> tile bits 9..11, lanes ->
// 4..8, warps -> 0..3) every thread keeps, across its tiles, the sum of
// q = Im(conj(lam) psi) and the sums over its registers with tile bit 9, 10,
// 11 set (phi_thr, one column per thread); the coset bits of a tile are the
// same for the whole tile, so each warp adds its tile sum to a warp-private
// accumulator of every coset wire whose bit is set.  phi_reduce folds them
// into phi_sm[w] (sum of q with wire-w bit 1) and phi_sm[32] (sum of q) once
// per CTA.
constexpr int kPhiThr = 4;  // per-thread accumulators: total, tile bits 9, 10, 11

__device__ __forceinline__ void phi_accumulate(const PassParams &P, u32 cbase, int lane, int warp,
                                               const double2 (&a)[bw::kR], const double2 (&b)[bw::kR],
                                               double *phi_thr, double (*phi_cos)[32]) {
  double v[kPhiThr] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int r = 0; r < bw::kR; ++r) {
    const double q = fma(b[r].x, a[r].y, -b[r].y * a[r].x);
    v[0] += q;
#pragma unroll
    for (int j = 0; j < 3; ++j)
      if ((r >> j) & 1) v[1 + j] += q;
  }
#pragma unroll
  for (int j = 0; j < kPhiThr; ++j) phi_thr[j * bw::kT] += v[j];
  const double s = warp_sum(v[0]);  // every lane holds the warp's tile sum
  if (lane < P.n && P.wire_tile_bit[lane] < 0 && ((cbase >> lane) & 1)) phi_cos[warp][lane] += s;
}

__device__ __forceinline__ void phi_reduce(const PassParams &P, int lane, int warp, const double *phi_thr,
                                           double (*phi_cos)[32], double (*red)[12], double *phi_sm) {
  double v[9];
#pragma unroll
  for (int j = 0; j < kPhiThr; ++j) v[j] = phi_thr[j * bw::kT];
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
        for (int ww = 0; ww < 16; ++ww) add += phi_cos[ww][w];
      } else if (tb >= 9) {
        for (int ww = 0; ww < 16; ++ww) add += red[ww][1 + tb - 9];
      } else if (tb >= 4) {
        for (int ww = 0; ww < 16; ++ww) add += red[ww][4 + tb - 4];
      } else {
        for (int ww = 0; ww < 16; ++ww)
          if ((ww >> tb) & 1) add += red[ww][0];
      }
      phi_sm[w] = add;
    }
    if (w == 31) phi_sm[32] = qt;
  }
  __syncthreads();
}

// PSRC: kLoadNatural / kLoadGatherP (staged with lambda) or kLoadProductPlain
// (analytic layer-0 psi from P.prod, computed in registers).
template <int PSRC, int LSRC, int PDST, int LDST, bool PHASE>
__global__ void __launch_bounds__(bw::kT, 1) bwd_pass_kernel(const PassParams P) {
  using namespace bw;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage_a = reinterpret_cast<double2 *>(smem_raw);
  double2 *stage_b = stage_a + kTileSize;
  double2 *trans = stage_b + kTileSize;
  __shared__ double red[16][12];
  __shared__ double phi_sm[33];
  __shared__ double2 km_sm[12];
  __shared__ double phi_thr_sm[PHASE ? kPhiThr * bw::kT : 1];
  __shared__ double phi_cos[PHASE ? 16 : 1][32];

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
  const u32 toffp = thread_offset(P, tpart<B0>(lane, warp));
  u32 poff[kR];  // register offsets of layout B0 (analytic psi)
#pragma unroll
  for (int r = 0; r < kR; ++r) poff[r] = ((r & 1) ? v9 : 0u) ^ ((r & 2) ? v10 : 0u) ^ ((r & 4) ? v11 : 0u);
  if (PHASE) {
#pragma unroll
    for (int j = 0; j < 3; ++j) ratio[j] = phase_ratio(P, unit_bit(P.vec[9 + j]));
    ratio[3] = make_double2(1.0, 0.0);
#pragma unroll
    for (int j = 0; j < kPhiThr; ++j) phi_thr_sm[j * kT + threadIdx.x] = 0.0;
    phi_cos[warp][lane] = 0.0;
  }
  if (threadIdx.x < 12) {
    const int w = P.gate_wire[threadIdx.x];
    km_sm[threadIdx.x] = w >= 0 ? RSV_TABLE_LOAD(&P.rot[P.layer * n + w]) : make_double2(0.0, 1.0);
  }
  __syncthreads();
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
      if (PSRC != kLoadProductPlain) cp_async16(&stage_a[s], &P.psi_in[source_index<PSRC>(p, n)]);
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
      if (PSRC != kLoadProductPlain) a[r] = stage_a[s];
      b[r] = stage_b[s];
    }
    // the staging buffers stay free until the CTA-wide transpose below has
    // used them; the next tile is prefetched right after it

    const u32 cbase = deposit(P, tile);
    if (PSRC == kLoadProductPlain) {
      // layout B0: registers -> tile bits 9..11
      const u32 base = cbase ^ toffp;
      table4_regs(P.prod, base, poff, a);
    }
    if (PHASE) {
      // RZ^dagger of the layer (with the layer's factor K) on psi and lambda,
      // then the phi sums.
      const double2 ph = table4(P.ptab, cbase ^ toffp);
      const double K = P.lscale[P.layer];
      apply_phase_gray<3, true, true>(make_double2(K * ph.x, K * ph.y), ratio, a, b);
      phi_accumulate(P, cbase, lane, warp, a, b, phi_thr_sm + threadIdx.x, phi_cos);
    }

    gates<B0>(P, km_sm, a, b, acc);
    warp_transpose<B0, B1>(wbuf, lane, warp, a);
    warp_transpose<B0, B1>(wbuf, lane, warp, b);
    gates<B1>(P, km_sm, a, b, acc);
    if (has_lo) {
      cta_transpose_pair<B1, A1>(stage_a, stage_b, lane, warp, a, b);
      if (tile + gridDim.x < num_tiles) issue(tile + gridDim.x);
      gates<A1>(P, km_sm, a, b, acc);
      warp_transpose<A1, A2>(wbuf, lane, warp, a);
      warp_transpose<A1, A2>(wbuf, lane, warp, b);
    } else {
      cta_transpose_pair<B1, A2>(stage_a, stage_b, lane, warp, a, b);
      if (tile + gridDim.x < num_tiles) issue(tile + gridDim.x);
    }
    gates<A2>(P, km_sm, a, b, acc);

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
    __syncthreads();  // red is reused
    phi_reduce(P, lane, warp, phi_thr_sm + threadIdx.x, phi_cos, red, phi_sm);
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
  // the tile is loaded in the first visited layout and stored from the last
  const int first = P.seq_layout[0], last = P.seq_layout[P.nseq - 1];
  const u32 toffl = thread_offset(P, thread_part(first, lane, warp));
  const int rl = reg_shift(first);
  const u32 v0 = P.vec[rl], v1 = P.vec[rl + 1], v2 = P.vec[rl + 2], v3 = P.vec[rl + 3];
  const u32 toffs = thread_offset(P, thread_part(last, lane, warp));
  const int rs = reg_shift(last);
  const u32 w0 = P.vec[rs], w1 = P.vec[rs + 1], w2 = P.vec[rs + 2], w3 = P.vec[rs + 3];
  const u32 num_tiles = static_cast<u32>(P.num_tiles);
  double2 dummy[kRegs];
  double2 ratio[4];
  if (PHASE) {
#pragma unroll
    for (int j = 0; j < 4; ++j) ratio[j] = phase_ratio(P, unit_bit(P.vec[rs + j]));
  }

  // analytic sources: per-register offsets of the product-table index
  // (ring_pinv is linear, so the index of base ^ o is ring_pinv(base) ^ ring_pinv(o))
  u32 poff[kRegs];
#pragma unroll
  for (int r = 0; r < kRegs; ++r) {
    const u32 o = reg_offset(r, v0, v1, v2, v3);
    poff[r] = PSRC == kLoadProduct ? static_cast<u32>(ring_pinv(o, n)) : o;
  }

  for (u32 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const u32 cbase = deposit(P, tile);
    const u32 base = cbase ^ toffl;
    double2 a[kRegs];
    if (PSRC == kLoadNatural) {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) a[r] = __ldcs(&P.psi_in[base ^ reg_offset(r, v0, v1, v2, v3)]);
    }
    if (PSRC == kLoadProduct) table4_regs(P.prod, static_cast<u32>(ring_pinv(base, n)), poff, a);
    if (PSRC == kLoadProductPlain) table4_regs(P.prod, base, poff, a);
    if (PSRC == kLoadMpsP) {
      mps_tile_p(P, cbase, trans, trans + kTileSize, lane, warp);
      __syncthreads();
      const int tpf = thread_part(first, lane, warp);
#pragma unroll
      for (int r = 0; r < kRegs; ++r) a[r] = trans[swz(tpf | (r << rl))];
      __syncthreads();
    }
    if (P.sync_after_load) __syncthreads();

    int prev = first;
    for (int k = 0; k < P.nseq; ++k) {
      const int layout = P.seq_layout[k];
      const int tp = thread_part(layout, lane, warp);
      if (k > 0) transpose(trans, thread_part(prev, lane, warp), reg_shift(prev), tp, reg_shift(layout), a);
      if (P.seq_apply[k]) apply_gates_fwd(P, layout, a);
      prev = layout;
    }

    const u32 sbase = cbase ^ toffs;
    if (PHASE) {
      const double2 ph = table4(P.ptab, sbase);
      const double K = P.lscale[P.layer];
      apply_phase_gray<4, false, false>(make_double2(K * ph.x, K * ph.y), ratio, a, dummy);
    }
#pragma unroll
    for (int r = 0; r < kRegs; ++r) store_amp<PDST>(P.psi_out, sbase ^ reg_offset(r, w0, w1, w2, w3), n, a[r]);
  }
}

template <int PSRC, int LSRC, int PDST, int LDST, bool PHASE>
cudaError_t launch_bwd(const PassParams &P, int grid, cudaStream_t s) {
  auto k = bwd_pass_kernel<PSRC, LSRC, PDST, LDST, PHASE>;
  static std::atomic<unsigned long long> configured{0};
  {
    const cudaError_t e = set_smem_limit_once(k, kBwdSmem, configured);
    if (e != cudaSuccess) return e;
  }
  k<<<grid, bw::kT, kBwdSmem, s>>>(P);
  return cudaGetLastError();
}

template <int PSRC, int PDST, bool PHASE>
cudaError_t launch_fwd(const PassParams &P, int grid, cudaStream_t s) {
  auto k = fwd_pass_kernel<PSRC, PDST, PHASE>;
  constexpr size_t smem = PSRC == kLoadMpsP ? kFwdMpsSmem : kFwdSmem;
  static std::atomic<unsigned long long> configured{0};
  {
    const cudaError_t e = set_smem_limit_once(k, smem, configured);
    if (e != cudaSuccess) return e;
  }
  k<<<grid, kThreads, smem, s>>>(P);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pass(const PassParams &P, bool bwd, int grid, cudaStream_t s) {
  if (P.tile_bits != 12) {
    if (bwd && P.tile_bits == 11) return launch_bwd_half(P, grid, s);
    return cudaErrorInvalidValue;
  }
  if (bwd) {
    const bool phase = P.phase != 0;
    if (P.phi_grad != P.phase) return cudaErrorInvalidValue;
    const int pl = P.psi_load, ll = P.lam_load, ps = P.psi_store, ls = P.lam_store;
    // The (psi source, lambda source, psi store, lambda store, phase) variants
    // the two backward schedules use.
#define RSV_BWD(PL, LL, PS, LS)                                                      \
  if (pl == PL && ll == LL && ps == PS && ls == LS)                                  \
    return phase ? launch_bwd<PL, LL, PS, LS, true>(P, grid, s)                      \
                 : launch_bwd<PL, LL, PS, LS, false>(P, grid, s);
    // uncompute schedule: psi streamed in and out
    RSV_BWD(kLoadNatural, kLoadNatural, kStoreNatural, kStoreNatural)
    RSV_BWD(kLoadNatural, kLoadGatherP, kStoreNatural, kStoreNatural)
    RSV_BWD(kLoadNatural, kLoadNatural, kStoreScatterPinv, kStoreNatural)
    RSV_BWD(kLoadNatural, kLoadGatherP, kStoreScatterPinv, kStoreNatural)
    RSV_BWD(kLoadNatural, kLoadNatural, kStoreNone, kStoreNone)
    RSV_BWD(kLoadNatural, kLoadGatherP, kStoreNone, kStoreNone)
    // checkpoint schedule: psi read from a checkpoint (or analytic), only lambda written
    RSV_BWD(kLoadNatural, kLoadNatural, kStoreNone, kStoreNatural)
    RSV_BWD(kLoadNatural, kLoadGatherP, kStoreNone, kStoreNatural)
    RSV_BWD(kLoadGatherP, kLoadGatherP, kStoreNone, kStoreNatural)
    RSV_BWD(kLoadProductPlain, kLoadGatherP, kStoreNone, kStoreNatural)
    RSV_BWD(kLoadProductPlain, kLoadNatural, kStoreNone, kStoreNatural)
    RSV_BWD(kLoadProductPlain, kLoadNatural, kStoreNone, kStoreNone)
#undef RSV_BWD
    return cudaErrorInvalidValue;
  }
  const bool phase = P.phase != 0;
  const int src = P.psi_load, dst = P.psi_store;
  if (src == kLoadProductPlain && dst == kStoreNatural && !phase)
    return launch_fwd<kLoadProductPlain, kStoreNatural, false>(P, grid, s);
  if (src == kLoadMpsP) {
    // unit tile over index bits 0..11 only
    for (int b = 0; b < 12; ++b)
      if (P.vec[b] != (1ull << b)) return cudaErrorInvalidValue;
    if (P.n < 13 || P.n > 31 || P.mps_btab == nullptr || P.mps_wtab == nullptr) return cudaErrorInvalidValue;
    if (dst == kStoreNatural && !phase) return launch_fwd<kLoadMpsP, kStoreNatural, false>(P, grid, s);
    return cudaErrorInvalidValue;
  }
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
