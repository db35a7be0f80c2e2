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
#include "rsv_tile.cuh"

namespace rsv {
namespace {

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
