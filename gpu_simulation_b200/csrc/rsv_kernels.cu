// sm_100a kernels for the ring-Ising structured adjoint (energy + gradient).
//
// Replaces the reference's per-chunk kernels (zzEncounter/GPU_Simulation
// cpp/ising_cuda_rotation_kernels.cu, cpp/ising_cuda_kernels.cu,
// cpp/ising_cuda_statevector_grad_kernels.cu) with one tile-pass kernel:
//
//   * a pass streams the state once, tile by tile; a tile is a coset of a
//     12-dimensional GF(2) subspace of indices (4096 amplitudes), held in
//     registers, 16 per thread;
//   * every wire whose direction lies in the tile is rotated in registers;
//     two shared-memory transposes bring the other tile directions into
//     registers, so one pass covers up to 12 wires;
//   * the CNOT ring is never a pass of its own: it is the gather (P) on a
//     pass's load or the scatter (P or P^-1) on its store;
//   * the RZ half of every layer is one diagonal phase per amplitude, built
//     from four 256-entry byte tables;
//   * backward passes accumulate the theta/phi gradient sums in registers and
//     write one deterministic partial record per CTA (no FP64 atomics).
#include "rsv_device.cuh"
#include "rsv_types.h"

namespace rsv {

// ------------------------------------------------------------------------
// Coefficient and table preparation
// ------------------------------------------------------------------------

// coef[k] = (cos t/2, sin t/2, cos p/2, sin p/2) for params (t, p) = params[2k..2k+1].
__global__ void coef_kernel(const double *__restrict__ params, double4 *__restrict__ coef,
                            int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  double st, ct, sp, cp;
  sincos(params[2 * k] * 0.5, &st, &ct);
  sincos(params[2 * k + 1] * 0.5, &sp, &cp);
  coef[k] = make_double4(ct, st, cp, sp);
}

// Phase byte tables: ptab[l][byte][v] = prod over the 8 wires w = 8*byte + j of
// (bit j of v ? e^{+i p_w/2} : e^{-i p_w/2}); wires >= n contribute 1.
// Product-state tables (layer 0): prod[byte][v] = prod over wires of
// (bit ? (s ch, s sh) : (c ch, -c sh))   (reference coefficients,
// cpp/ising_cuda_rotation_kernels.cu:692-702); wires >= n contribute the
// factor of |0> (1 for bit 0, 0 for bit 1).
// grid: (L + 1) * 4 blocks of 256 threads; block L*4.. builds prod.
__global__ void tables_kernel(const double4 *__restrict__ coef, int n, int L,
                              double2 *__restrict__ ptab, double2 *__restrict__ prod) {
  const int tbl = blockIdx.x;
  const int layer = tbl / 4;
  const int byte = tbl % 4;
  const int v = threadIdx.x;
  double2 acc = make_double2(1.0, 0.0);
  if (layer < L) {
    for (int j = 0; j < 8; ++j) {
      const int w = byte * 8 + j;
      if (w >= n) break;
      const double4 k = coef[layer * n + w];
      const double2 f = ((v >> j) & 1) ? make_double2(k.z, k.w) : make_double2(k.z, -k.w);
      acc = cmul(acc, f);
    }
    ptab[(layer * 4 + byte) * 256 + v] = acc;
  } else {
    for (int j = 0; j < 8; ++j) {
      const int w = byte * 8 + j;
      double2 f;
      if (w >= n) {
        f = ((v >> j) & 1) ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
      } else {
        const double4 k = coef[w];
        f = ((v >> j) & 1) ? make_double2(k.y * k.z, k.y * k.w) : make_double2(k.x * k.z, -k.x * k.w);
      }
      acc = cmul(acc, f);
    }
    prod[byte * 256 + v] = acc;
  }
}

// ------------------------------------------------------------------------
// Tile pass kernel
// ------------------------------------------------------------------------

__device__ __forceinline__ int swz(int t) { return t ^ (((t >> 3) ^ (t >> 6) ^ (t >> 9)) & 7); }

// Tile index of register k of this thread in layout 0/1/2.
//   layout 0: registers = tile bits 8..11, lanes = 0..4, warps = 5..7 (load/store)
//   layout 1: registers = 4..7, lanes = 8..11,0, warps = 1..3
//   layout 2: registers = 0..3, lanes = 4..8, warps = 9..11
template <int LAYOUT>
__device__ __forceinline__ int tile_index(int lane, int warp, int k) {
  if (LAYOUT == 0) return lane | (warp << 5) | (k << 8);
  if (LAYOUT == 1) return (lane >> 4) | (warp << 1) | (k << 4) | ((lane & 15) << 8);
  return k | (lane << 4) | (warp << 9);
}

__device__ __forceinline__ u64 deposit(const PassParams &P, u64 tile) {
  u64 base = 0;
#pragma unroll
  for (int r = 0; r < kMaxRuns; ++r) {
    if (r < P.num_runs) {
      const int len = P.run_len[r];
      base |= (tile & ((u64{1} << len) - 1)) << P.run_start[r];
      tile >>= len;
    }
  }
  return base;
}

__device__ __forceinline__ double2 table4(const double2 *__restrict__ t, u64 p) {
  double2 v = __ldg(&t[p & 255]);
  v = cmul(v, __ldg(&t[256 + ((p >> 8) & 255)]));
  v = cmul(v, __ldg(&t[512 + ((p >> 16) & 255)]));
  v = cmul(v, __ldg(&t[768 + ((p >> 24) & 255)]));
  return v;
}

__device__ __forceinline__ double2 load_amp(int mode, const double2 *buf, u64 p, int n,
                                            const double2 *__restrict__ prod) {
  if (mode == kLoadNatural) return __ldcs(&buf[p]);
  if (mode == kLoadGatherP) return __ldcs(&buf[ring_p(p, n)]);
  if (mode == kLoadProduct) return table4(prod, ring_pinv(p, n));
  return table4(prod, p);
}

__device__ __forceinline__ void store_amp(int mode, double2 *buf, u64 p, int n, double2 v) {
  if (mode == kStoreNatural) {
    __stcs(&buf[p], v);
  } else if (mode == kStoreScatterP) {
    __stcs(&buf[ring_p(p, n)], v);
  } else if (mode == kStoreScatterPinv) {
    __stcs(&buf[ring_pinv(p, n)], v);
  }
}

// One rotation step on a register pair (x0, x1) = (|0>, |1>) of one wire.
template <bool BWD>
__device__ __forceinline__ void rotate_pair(double c, double s, double2 &a0, double2 &a1, double2 &b0,
                                            double2 &b1, double &acc) {
  const double2 x0 = a0, x1 = a1;
  if (!BWD) {
    a0 = make_double2(fma(c, x0.x, -s * x1.x), fma(c, x0.y, -s * x1.y));
    a1 = make_double2(fma(s, x0.x, c * x1.x), fma(s, x0.y, c * x1.y));
  } else {
    const double2 y0 = b0, y1 = b1;
    // theta: Re(conj(lam1) psi0) - Re(conj(lam0) psi1), in the frame with the
    // layer's RZ removed; equal to the reference's 2 Re<lam_mid|dRY|psi_before>
    // (cpp/ising_cuda_statevector_grad_kernels.cu:289-307) after simplification.
    acc += fma(y1.x, x0.x, y1.y * x0.y) - fma(y0.x, x1.x, y0.y * x1.y);
    a0 = make_double2(fma(c, x0.x, s * x1.x), fma(c, x0.y, s * x1.y));
    a1 = make_double2(fma(-s, x0.x, c * x1.x), fma(-s, x0.y, c * x1.y));
    b0 = make_double2(fma(c, y0.x, s * y1.x), fma(c, y0.y, s * y1.y));
    b1 = make_double2(fma(-s, y0.x, c * y1.x), fma(-s, y0.y, c * y1.y));
  }
}

// Rotate the register pairs of the four tile bits TB0..TB0+3 (register bit j
// is tile bit TB0 + j in layout LAYOUT).  When the tile has a direction with
// more than one physical bit (P.flip_bit < 12, the all-ones direction of the
// antipodal tile), that direction also flips the gated wire's bit: elements
// whose flip coordinate is 1 hold the pair as (|1>, |0>), so the roles swap.
template <bool BWD, int TB0, int LAYOUT>
__device__ __forceinline__ void apply_reg_gates(const PassParams &P, int lane, int warp,
                                                double2 (&a)[kRegs], double2 (&b)[kRegs],
                                                double (&acc)[12]) {
  const int thread_t = tile_index<LAYOUT>(lane, warp, 0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int w = P.gate_wire[TB0 + j];
    if (w < 0) continue;
    const double2 cs = __ldg(reinterpret_cast<const double2 *>(&P.coef[P.layer * P.n + w]));
    const double c = cs.x, s = cs.y;
    if (P.flip_bit >= kTileBits) {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        rotate_pair<BWD>(c, s, a[r], a[r1], b[r], b[r1], acc[TB0 + j]);
      }
    } else {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const bool flip = ((thread_t | tile_index<LAYOUT>(0, 0, r)) >> P.flip_bit) & 1;
        if (flip) {
          rotate_pair<BWD>(c, s, a[r1], a[r], b[r1], b[r], acc[TB0 + j]);
        } else {
          rotate_pair<BWD>(c, s, a[r], a[r1], b[r], b[r1], acc[TB0 + j]);
        }
      }
    }
  }
}

template <bool BWD, int FROM, int TO>
__device__ __forceinline__ void transpose(double2 *sm, int lane, int warp, double2 (&a)[kRegs],
                                          double2 (&b)[kRegs]) {
#pragma unroll
  for (int r = 0; r < kRegs; ++r) {
    const int t = swz(tile_index<FROM>(lane, warp, r));
    sm[t] = a[r];
    if (BWD) sm[kTileSize + t] = b[r];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRegs; ++r) {
    const int t = swz(tile_index<TO>(lane, warp, r));
    a[r] = sm[t];
    if (BWD) b[r] = sm[kTileSize + t];
  }
  __syncthreads();
}

template <bool BWD>
__global__ void __launch_bounds__(kThreads, BWD ? 1 : 2) pass_kernel(const PassParams P) {
  extern __shared__ double2 sm[];
  __shared__ double red[8][12];
  __shared__ double phi_sm[33];

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;

  // Physical offset of this thread's part of the layout-0 tile index.
  u64 toff = 0;
  {
    const int tt = lane | (warp << 5);
#pragma unroll
    for (int bb = 0; bb < 8; ++bb)
      if ((tt >> bb) & 1) toff ^= P.vec[bb];
  }
  u64 roff[kRegs];
#pragma unroll
  for (int r = 0; r < kRegs; ++r) {
    u64 o = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if ((r >> j) & 1) o ^= P.vec[8 + j];
    roff[r] = o;
  }

  double acc[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) acc[i] = 0.0;
  if (BWD && P.phi_grad) {
    if (threadIdx.x < 33) phi_sm[threadIdx.x] = 0.0;
    __syncthreads();
  }

  const double2 *ptab = P.ptab;

  for (u64 tile = blockIdx.x; tile < P.num_tiles; tile += gridDim.x) {
    const u64 base = deposit(P, tile) ^ toff;
    double2 a[kRegs], b[kRegs];
#pragma unroll
    for (int r = 0; r < kRegs; ++r) {
      const u64 p = base ^ roff[r];
      a[r] = load_amp(P.psi_load, P.psi_in, p, P.n, P.prod);
      if (BWD) b[r] = load_amp(P.lam_load, P.lam_in, p, P.n, P.prod);
    }
    if (P.sync_after_load) __syncthreads();

    if (BWD && P.phase) {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) {
        const double2 ph = table4(ptab, base ^ roff[r]);
        a[r] = cmul_conj(a[r], ph);
        b[r] = cmul_conj(b[r], ph);
      }
    }

    if (BWD && P.phi_grad) {
      // q = Im(conj(lam) psi); per-thread total and register-bit sums.
      double q_tot = 0.0, q_reg[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int r = 0; r < kRegs; ++r) {
        const double q = fma(b[r].x, a[r].y, -b[r].y * a[r].x);
        q_tot += q;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if ((r >> j) & 1) q_reg[j] += q;
      }
      double v[10];
      v[0] = q_tot;
#pragma unroll
      for (int j = 0; j < 4; ++j) v[1 + j] = q_reg[j];
#pragma unroll
      for (int j = 0; j < 5; ++j) v[5 + j] = ((lane >> j) & 1) ? q_tot : 0.0;
#pragma unroll
      for (int j = 0; j < 10; ++j) v[j] = warp_sum(v[j]);
      if (lane == 0) {
#pragma unroll
        for (int j = 0; j < 10; ++j) red[warp][j] = v[j];
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        const int w = threadIdx.x;
        double qt = 0.0;
#pragma unroll
        for (int ww = 0; ww < 8; ++ww) qt += red[ww][0];
        if (w < P.n) {
          const int tb = P.wire_tile_bit[w];
          double add = 0.0;
          if (tb >= 8) {
            for (int ww = 0; ww < 8; ++ww) add += red[ww][1 + tb - 8];
          } else if (tb >= 5) {
            for (int ww = 0; ww < 8; ++ww)
              if ((ww >> (tb - 5)) & 1) add += red[ww][0];
          } else if (tb >= 0) {
            for (int ww = 0; ww < 8; ++ww) add += red[ww][5 + tb];
          } else if ((base >> w) & 1) {
            // coset bit: every amplitude of the tile has bit w set
            add = qt;
          }
          phi_sm[w] += add;
        }
        if (w == 31) phi_sm[32] += qt;
      }
      __syncthreads();
    }

    apply_reg_gates<BWD, 8, 0>(P, lane, warp, a, b, acc);
    if (P.need_l1) {
      transpose<BWD, 0, 1>(sm, lane, warp, a, b);
      apply_reg_gates<BWD, 4, 1>(P, lane, warp, a, b, acc);
      if (P.need_l2) {
        transpose<BWD, 1, 2>(sm, lane, warp, a, b);
        apply_reg_gates<BWD, 0, 2>(P, lane, warp, a, b, acc);
        transpose<BWD, 2, 0>(sm, lane, warp, a, b);
      } else {
        transpose<BWD, 1, 0>(sm, lane, warp, a, b);
      }
    }

    if (!BWD && P.phase) {
#pragma unroll
      for (int r = 0; r < kRegs; ++r) a[r] = cmul(a[r], table4(ptab, base ^ roff[r]));
    }

#pragma unroll
    for (int r = 0; r < kRegs; ++r) {
      const u64 p = base ^ roff[r];
      store_amp(P.psi_store, P.psi_out, p, P.n, a[r]);
      if (BWD) store_amp(P.lam_store, P.lam_out, p, P.n, b[r]);
    }
  }

  if (BWD) {
    // CTA reduction of the theta partials, then one record per CTA.
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const double s = warp_sum(acc[i]);
      if (lane == 0) red[warp][i] = s;
    }
    __syncthreads();
    double *rec = P.partials + static_cast<size_t>(blockIdx.x) * kPartialStride;
    if (threadIdx.x < 12) {
      double s = 0.0;
      for (int ww = 0; ww < 8; ++ww) s += red[ww][threadIdx.x];
      rec[threadIdx.x] = s;
    }
    if (P.phi_grad) {
      if (threadIdx.x < 31) rec[kPartialPhi + threadIdx.x] = phi_sm[threadIdx.x];
      if (threadIdx.x == 31) rec[kPartialTot] = phi_sm[32];
    }
  }
}

// ------------------------------------------------------------------------
// Energy: mu = (P^T H P) chi and E = sum Re(conj(chi) mu), in the frame of the
// last layer before its CNOT ring (the ring is folded into H).  Equivalent to
// the reference's lambda = H psi (cpp/ising_cuda_kernels.cu:313-358) followed
// by its inverse ring gather on lambda and psi.
// ------------------------------------------------------------------------
constexpr int kEnergyThreads = 256;

__global__ void __launch_bounds__(kEnergyThreads) energy_kernel(const double2 *__restrict__ chi,
                                                                 double2 *__restrict__ mu, int n,
                                                                 double field, u64 size,
                                                                 double *__restrict__ partials) {
  __shared__ double red[kEnergyThreads / 32];
  u64 masks[kMaxQubits];
#pragma unroll
  for (int w = 0; w < kMaxQubits; ++w) masks[w] = (w < n) ? ring_pinv(u64{1} << w, n) : 0;
  double e = 0.0;
  const u64 stride = static_cast<u64>(gridDim.x) * kEnergyThreads;
  for (u64 i = static_cast<u64>(blockIdx.x) * kEnergyThreads + threadIdx.x; i < size; i += stride) {
    const double2 c = chi[i];
    const double d = diag_after_ring(i, n);
    double2 x = make_double2(0.0, 0.0);
#pragma unroll
    for (int w = 0; w < kMaxQubits; ++w) {
      if (w < n) {
        const double2 t = __ldg(&chi[i ^ masks[w]]);
        x.x += t.x;
        x.y += t.y;
      }
    }
    const double2 m = make_double2(fma(d, c.x, -field * x.x), fma(d, c.y, -field * x.y));
    mu[i] = m;
    e += fma(c.x, m.x, c.y * m.y);
  }
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < kEnergyThreads / 32; ++i) s += red[i];
    partials[blockIdx.x] = s;
  }
}

// ------------------------------------------------------------------------
// Finalize: deterministic second-stage reduction of all per-CTA partials.
//   energy = sum of energy partials;
//   grad[2(l n + w)]     = sum over CTAs of theta partial (pass theta_pass, slot theta_slot)
//   grad[2(l n + w) + 1] = tot - 2 * B_w of the layer's first pass
// ------------------------------------------------------------------------


__global__ void finalize_kernel(const FinalizeParams F) {
  __shared__ double red[32];
  const int t = threadIdx.x;
  double e = 0.0;
  for (int i = t; i < F.num_energy_partials; i += blockDim.x) e += F.energy_partials[i];
  e = warp_sum(e);
  if ((t & 31) == 0) red[t >> 5] = e;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    *F.energy_out = s;
  }
  if (F.grad_out == nullptr) return;
  const int np = F.L * F.n;
  for (int k = t; k < np; k += blockDim.x) {
    const int layer = k / F.n;
    const int w = k % F.n;
    {
      const int pass = F.theta_pass[k];
      const int slot = F.theta_slot[k];
      const double *rec = F.pass_partials + static_cast<size_t>(pass) * F.max_grid * kPartialStride;
      double s = 0.0;
      for (int c = 0; c < F.pass_grid[pass]; ++c) s += rec[static_cast<size_t>(c) * kPartialStride + slot];
      F.grad_out[2 * k] = s;
    }
    {
      const int pass = F.phi_pass[layer];
      const double *rec = F.pass_partials + static_cast<size_t>(pass) * F.max_grid * kPartialStride;
      double tot = 0.0, bw = 0.0;
      for (int c = 0; c < F.pass_grid[pass]; ++c) {
        tot += rec[static_cast<size_t>(c) * kPartialStride + kPartialTot];
        bw += rec[static_cast<size_t>(c) * kPartialStride + kPartialPhi + w];
      }
      F.grad_out[2 * k + 1] = tot - 2.0 * bw;
    }
  }
}

// ------------------------------------------------------------------------
// Launchers (host side, same translation unit)
// ------------------------------------------------------------------------

cudaError_t launch_coef(const double *params, double4 *coef, int count, cudaStream_t s) {
  coef_kernel<<<(count + 127) / 128, 128, 0, s>>>(params, coef, count);
  return cudaGetLastError();
}

cudaError_t launch_tables(const double4 *coef, int n, int L, double2 *ptab, double2 *prod,
                          cudaStream_t s) {
  tables_kernel<<<(L + 1) * 4, 256, 0, s>>>(coef, n, L, ptab, prod);
  return cudaGetLastError();
}

size_t pass_smem_bytes(bool bwd) { return (bwd ? 2 : 1) * kTileSize * sizeof(double2); }

cudaError_t configure_pass_kernels() {
  cudaError_t e = cudaFuncSetAttribute(pass_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(pass_smem_bytes(true)));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(pass_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(pass_smem_bytes(false)));
}

cudaError_t launch_pass(const PassParams &P, bool bwd, int grid, cudaStream_t s) {
  if (bwd) {
    pass_kernel<true><<<grid, kThreads, pass_smem_bytes(true), s>>>(P);
  } else {
    pass_kernel<false><<<grid, kThreads, pass_smem_bytes(false), s>>>(P);
  }
  return cudaGetLastError();
}

cudaError_t launch_energy(const double2 *chi, double2 *mu, int n, double field, u64 size,
                          double *partials, int grid, cudaStream_t s) {
  energy_kernel<<<grid, kEnergyThreads, 0, s>>>(chi, mu, n, field, size, partials);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalizeParams &F, cudaStream_t s) {
  finalize_kernel<<<1, 256, 0, s>>>(F);
  return cudaGetLastError();
}

}  // namespace rsv
