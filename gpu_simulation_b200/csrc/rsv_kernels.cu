// sm_100a kernels for the ring-Ising structured adjoint: coefficient and
// byte-table preparation, the energy (lambda = H psi) kernel and the final
// deterministic reduction.  The tile-pass kernels are in rsv_pass.cu.
#include <algorithm>

#include "rsv_device.cuh"
#include "rsv_launch.h"
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
                              double2 *__restrict__ ptab, double2 *__restrict__ prod,
                              const PartialMasks partial) {
  const int tbl = blockIdx.x;
  const int layer = tbl / 4;
  const int byte = tbl % 4;
  const int v = threadIdx.x;
  double2 acc = make_double2(1.0, 0.0);
  if (layer > L) {
    // partial product table (layer > L): wires in the mask carry RY / f |0>
    // of layer 0 (tangent form, no RZ), the others |0>
    const int j = layer - L - 1;
    const unsigned int m = partial.mask[j];
    for (int b = 0; b < 8; ++b) {
      const int w = byte * 8 + b;
      const bool one = (v >> b) & 1;
      double f = one ? 0.0 : 1.0;
      if (w < n && ((m >> w) & 1)) {
        const double4 k = coef[w];
        const double fac = (fabs(k.x) >= fabs(k.y)) ? k.x : k.y;
        f = (one ? k.y : k.x) / fac;
      }
      acc = make_double2(acc.x * f, acc.y * f);
    }
    prod[(1 + j) * 1024 + byte * 256 + v] = acc;
    return;
  }
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

// Tangent form of the RY rotations (one FMA per component instead of two).
// For every (layer, wire): |cos| >= |sin| -> f = cos t/2, RY = f [[1,-k],[k,1]],
// k = tan t/2 (mode +1); otherwise f = sin t/2, RY = f [[k,-1],[1,k]],
// k = cot t/2 (mode -1).  |f| >= 1/sqrt(2), so no factor over- or underflows.
// The passes apply RY / f; the product K_l of a layer's factors is applied
// once with the layer's RZ phase, so states between layers are exact.
// Inside a backward layer the state carries the factors of the wires not
// yet undone; gscale[] holds the exact correction of every gradient sum:
//   theta of wire w: 1 / (prod of f over the wires of its layer still pending
//                         when w is undone, w included)^2,
//   phi of the layer: 1 / K_l^2.
// order[layer * n .. layer * n + n) is the undo order of the wires within
// backward layer `layer` (the kernels of a layer's passes fix it).  In the
// checkpoint schedule psi is re-read from the forward pass's checkpoint at
// every backward pass, so the correction restarts at each pass (entries with
// kUndoPassStart):
//   theta of wire w: (prod of f over the wires undone before w in its pass)^2,
//                    divided by K_l^2 in the layer's first (phase) pass.
// grid: L blocks of 32 threads.
__global__ void rot_kernel(const double4 *__restrict__ coef, int n, int L, const int *__restrict__ order,
                           int checkpoint, double2 *__restrict__ rot, double *__restrict__ lscale,
                           double *__restrict__ gscale) {
  const int layer = blockIdx.x;
  if (layer >= L) return;
  order += layer * n;
  for (int w = threadIdx.x; w < n; w += blockDim.x) {
    const double4 k = coef[layer * n + w];
    rot[layer * n + w] = (fabs(k.x) >= fabs(k.y)) ? make_double2(k.y / k.x, 1.0)
                                                   : make_double2(k.x / k.y, -1.0);
  }
  if (threadIdx.x != 0) return;
  auto factor = [&](int w) {
    const double4 k = coef[layer * n + w];
    return (fabs(k.x) >= fabs(k.y)) ? k.x : k.y;
  };
  double K = 1.0;
  for (int w = 0; w < n; ++w) K *= factor(w);
  lscale[layer] = K;
  if (!checkpoint) {
    double pending = K;
    for (int i = 0; i < n; ++i) {
      const int w = order[i] & (kUndoPassStart - 1);
      gscale[2 * (layer * n + w)] = 1.0 / (pending * pending);
      gscale[2 * (layer * n + w) + 1] = 1.0 / (K * K);
      pending /= factor(w);
    }
  } else {
    // psi from a checkpoint: at the start of the layer's first backward pass
    // psi and lambda both carry K (the phase pass), at the start of every
    // later pass their factors cancel; inside a pass each undone wire divides
    // both by its f.
    // Wires flagged kUndoSameGroup see the state the group's first wire saw.
    double undone = 1.0, group = 1.0;
    bool first = true;
    for (int i = 0; i < n; ++i) {
      const int w = order[i] & (kUndoPassStart - 1);
      if (i > 0 && (order[i] & kUndoPassStart)) {
        undone = 1.0;
        group = 1.0;
        first = false;
      } else if (!(order[i] & kUndoSameGroup)) {
        undone *= group;
        group = 1.0;
      }
      gscale[2 * (layer * n + w)] = undone * undone / (first ? K * K : 1.0);
      gscale[2 * (layer * n + w) + 1] = 1.0 / (K * K);
      group *= factor(w);
    }
  }
}

// ------------------------------------------------------------------------
// Energy: mu = (P^T H P) chi and E = sum Re(conj(chi) mu), in the frame of the
// last layer before its CNOT ring (the ring is folded into H).  Equivalent to
// the reference's lambda = H psi (cpp/ising_cuda_kernels.cu:313-358) followed
// by its inverse ring gather on lambda and psi.
//
// In this frame the field term of wire w flips the index bits of
// m_w = P^-1(e_w): bits {w, w+1}, and {n-1, 0, 1} for the last wire.  A flip
// of a high bit reads an amplitude far away, which for large states comes
// from DRAM once more per amplitude.  From kEnergySplitQubits on, the masks
// on the top nine bits (and the two on bits 0..2) are therefore applied by a
// tile kernel that holds cosets of bits {0,1,2} and {n-9..n-1} in shared
// memory; the grid-stride kernel adds the remaining masks, whose partners
// are near enough to come from L1/L2, and forms the energy.
// ------------------------------------------------------------------------
constexpr int kEnergyThreads = 256;
// The split energy's grid-stride part runs 1024-thread CTAs (two per SM): a CTA
// covers 1024 consecutive amplitudes per step, so the partners of the masks on
// index bits up to 9 are ones the CTA has just read (L1), not L2 requests.
constexpr int kEnergySplitThreads = 1024;
constexpr int kEnergySplitQubits = 21;
constexpr int kEnergyHighBits = 9;
constexpr int kEnergyTileThreads = 256;
constexpr int kEnergyTileBits = 12;  // 3 low + kEnergyHighBits high bits
constexpr size_t kEnergyTileSmem = (size_t{1} << kEnergyTileBits) * sizeof(double2);
// masks inside a tile: wires 0 and 1, the eight wires n-9..n-2 and the last wire
constexpr int kEnergyTileMasks = 11;

// Index masks of the grid-stride part, compacted on the host.
struct EnergyMasks {
  u64 m[kMaxQubits];
};

// grid-stride part: the K masks of M, plus mu_in (the tile kernel's part,
// diagonal included) when given, else the diagonal.  K is a template
// parameter so that all K partner loads of an amplitude are issued before
// the first is used.
template <int K, int THREADS>
__global__ void __launch_bounds__(THREADS) energy_kernel(const double2 *__restrict__ chi,
                                                                 double2 *__restrict__ mu, int n,
                                                                 double field, u64 size,
                                                                 const EnergyMasks M, int with_mu_in,
                                                                 double *__restrict__ partials) {
  __shared__ double red[THREADS / 32];
  double e = 0.0;
  const u64 stride = static_cast<u64>(gridDim.x) * THREADS;
  for (u64 i = static_cast<u64>(blockIdx.x) * THREADS + threadIdx.x; i < size; i += stride) {
    const double2 c = chi[i];
    double2 x = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const double2 t = __ldg(&chi[i ^ M.m[j]]);
      x.x += t.x;
      x.y += t.y;
    }
    double2 m;
    if (with_mu_in) {
      const double2 mi = mu[i];
      m = make_double2(fma(-field, x.x, mi.x), fma(-field, x.y, mi.y));
    } else {
      const double d = diag_after_ring(i, n);
      m = make_double2(fma(d, c.x, -field * x.x), fma(d, c.y, -field * x.y));
    }
    mu[i] = m;
    e += fma(c.x, m.x, c.y * m.y);
  }
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < THREADS / 32; ++i) s += red[i];
    partials[blockIdx.x] = s;
  }
}

// the grid-stride kernel on 1024-thread CTAs without a tile kernel before it
template <int K>
cudaError_t launch_energy_masks_k(int count, int grid, cudaStream_t s, const double2 *chi, double2 *mu, int n,
                                  double field, u64 size, const EnergyMasks &M, double *partials) {
  if (count == K) {
    energy_kernel<K, kEnergySplitThreads><<<grid, kEnergySplitThreads, 0, s>>>(chi, mu, n, field, size, M, 0,
                                                                               partials);
    return cudaGetLastError();
  }
  if constexpr (K < kMaxQubits) {
    return launch_energy_masks_k<K + 1>(count, grid, s, chi, mu, n, field, size, M, partials);
  } else {
    return cudaErrorInvalidValue;
  }
}

template <int K>
cudaError_t launch_energy_k(int count, int grid, cudaStream_t s, const double2 *chi, double2 *mu, int n,
                            double field, u64 size, const EnergyMasks &M, int with_mu_in, double *partials) {
  if (count == K) {
    if (with_mu_in)
      energy_kernel<K, kEnergySplitThreads><<<grid, kEnergySplitThreads, 0, s>>>(chi, mu, n, field, size, M, 1,
                                                                                 partials);
    else
      energy_kernel<K, kEnergyThreads><<<grid, kEnergyThreads, 0, s>>>(chi, mu, n, field, size, M, 0, partials);
    return cudaGetLastError();
  }
  if constexpr (K < kMaxQubits) {
    return launch_energy_k<K + 1>(count, grid, s, chi, mu, n, field, size, M, with_mu_in, partials);
  } else {
    return cudaErrorInvalidValue;
  }
}

struct EnergyTile {
  int n, hs, num_masks;
  double field;
  u64 num_tiles;
  unsigned int tmask[kEnergyTileBits];  // masks in tile coordinates
};

// Tile index tau: bits 0..2 -> index bits 0..2 (one 128-byte line),
// bits 3..11 -> index bits hs..hs+8; the coset runs over index bits 3..hs-1.
__device__ __forceinline__ u64 energy_tile_index(u64 cbase, int tau, int hs) {
  return cbase | static_cast<u64>(tau & 7) | (static_cast<u64>(tau >> 3) << hs);
}

__global__ void __launch_bounds__(kEnergyTileThreads) energy_tile_kernel(const double2 *__restrict__ chi,
                                                                          double2 *__restrict__ mu,
                                                                          const EnergyTile T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *tile = reinterpret_cast<double2 *>(smem_raw);
  constexpr int kPer = (1 << kEnergyTileBits) / kEnergyTileThreads;
  for (u64 t = blockIdx.x; t < T.num_tiles; t += gridDim.x) {
    const u64 cbase = t << 3;
    __syncthreads();  // the previous tile's partner reads are done
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int tau = threadIdx.x + k * kEnergyTileThreads;
      const unsigned int s = static_cast<unsigned int>(__cvta_generic_to_shared(&tile[tau]));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s),
                   "l"(&chi[energy_tile_index(cbase, tau, T.hs)])
                   : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kPer; ++k) {
      const int tau = threadIdx.x + k * kEnergyTileThreads;
      const u64 p = energy_tile_index(cbase, tau, T.hs);
      const double2 c = tile[tau];
      double2 x = make_double2(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < kEnergyTileMasks; ++j) {
        const double2 v = tile[tau ^ T.tmask[j]];
        x.x += v.x;
        x.y += v.y;
      }
      const double d = diag_after_ring(p, T.n);
      __stcg(&mu[p], make_double2(fma(d, c.x, -T.field * x.x), fma(d, c.y, -T.field * x.y)));
    }
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
  if (F.pipeline_err != nullptr && *F.pipeline_err != 0) {
    // a backward pass did not complete: no result is better than a wrong one
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    if (t == 0) *F.energy_out = nan;
    if (F.grad_out != nullptr)
      for (int k = t; k < 2 * F.L * F.n; k += blockDim.x) F.grad_out[k] = nan;
    return;
  }
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
    if (F.theta_pass[k] < 0) continue;  // layer 0 on the layer-0 kernel
    {
      const int pass = F.theta_pass[k];
      const int slot = F.theta_slot[k];
      const double *rec = F.pass_partials + static_cast<size_t>(pass) * F.max_grid * kPartialStride;
      double s = 0.0;
      for (int c = 0; c < F.pass_grid[pass]; ++c) s += rec[static_cast<size_t>(c) * kPartialStride + slot];
      F.grad_out[2 * k] = s * F.gscale[2 * k];
    }
    {
      const bool alt = layer == F.phi_alt_layer && ((F.phi_alt_wires >> w) & 1u);
      const int pass = alt ? F.phi_alt_pass : F.phi_pass[layer];
      const double *rec = F.pass_partials + static_cast<size_t>(pass) * F.max_grid * kPartialStride;
      double tot = 0.0, bw = 0.0;
      for (int c = 0; c < F.pass_grid[pass]; ++c) {
        tot += rec[static_cast<size_t>(c) * kPartialStride + kPartialTot];
        bw += rec[static_cast<size_t>(c) * kPartialStride + kPartialPhi + w];
      }
      F.grad_out[2 * k + 1] = (tot - 2.0 * bw) * (alt ? 1.0 : F.gscale[2 * k + 1]);
    }
  }
}

// ------------------------------------------------------------------------
// Launchers (host side, same translation unit)
// ------------------------------------------------------------------------

// Small host tables written to device memory by kernels whose parameters carry
// the values: no copy from pageable host memory, nothing refers to host memory
// after the launch returns.
namespace {
constexpr int kParamInts = 960;  // 3.8 KB of kernel parameters per launch
struct IntChunk {
  int count;
  int v[kParamInts];
};
__global__ void put_ints_kernel(const IntChunk c, int *dst) {
  for (int i = threadIdx.x; i < c.count; i += blockDim.x) dst[i] = c.v[i];
}
}  // namespace

cudaError_t launch_put_ints(const int *src, size_t count, int *dst, cudaStream_t s) {
  for (size_t off = 0; off < count; off += kParamInts) {
    IntChunk c;
    c.count = static_cast<int>(std::min<size_t>(kParamInts, count - off));
    for (int i = 0; i < c.count; ++i) c.v[i] = src[off + i];
    put_ints_kernel<<<1, 256, 0, s>>>(c, dst + off);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_coef(const double *params, double4 *coef, int count, cudaStream_t s) {
  coef_kernel<<<(count + 127) / 128, 128, 0, s>>>(params, coef, count);
  return cudaGetLastError();
}

cudaError_t launch_tables(const double4 *coef, int n, int L, double2 *ptab, double2 *prod,
                          const PartialMasks &partial, cudaStream_t s) {
  if (partial.count < 0 || partial.count > kMaxPartialTables) return cudaErrorInvalidValue;
  tables_kernel<<<(L + 1 + partial.count) * 4, 256, 0, s>>>(coef, n, L, ptab, prod, partial);
  return cudaGetLastError();
}

cudaError_t launch_rot(const double4 *coef, int n, int L, const int *order, bool checkpoint,
                       double2 *rot, double *lscale, double *gscale, cudaStream_t s) {
  rot_kernel<<<L, 32, 0, s>>>(coef, n, L, order, checkpoint ? 1 : 0, rot, lscale, gscale);
  return cudaGetLastError();
}

cudaError_t launch_energy(const double2 *chi, double2 *mu, int n, double field, u64 size,
                          double *partials, int grid, int sms, cudaStream_t s) {
  if (n < 1 || n > kMaxQubits) return cudaErrorInvalidValue;
  EnergyMasks M{};
  int count = 0;
  if (n < kEnergySplitQubits) {
    for (int w = 0; w < n; ++w) M.m[count++] = ring_pinv(u64{1} << w, n);
    return launch_energy_k<1>(count, grid, s, chi, mu, n, field, size, M, 0, partials);
  }
  EnergyTile T{};
  T.n = n;
  T.hs = n - kEnergyHighBits;
  T.field = field;
  T.num_tiles = u64{1} << (n - kEnergyTileBits);
  for (int w = 0; w < n; ++w) {
    const u64 m = ring_pinv(u64{1} << w, n);
    if ((m & ~u64{7} & ((u64{1} << T.hs) - 1)) == 0) {
      if (T.num_masks == kEnergyTileMasks) return cudaErrorInvalidValue;
      T.tmask[T.num_masks++] = static_cast<unsigned int>((m & 7) | ((m >> T.hs) << 3));
    } else {
      M.m[count++] = m;
    }
  }
  if (T.num_masks != kEnergyTileMasks) return cudaErrorInvalidValue;
  static std::atomic<unsigned long long> configured{0};
  {
    const cudaError_t e = set_smem_limit_once(energy_tile_kernel, kEnergyTileSmem, configured);
    if (e != cudaSuccess) return e;
  }
  const int tgrid = static_cast<int>(std::min<u64>(T.num_tiles, static_cast<u64>(std::max(1, sms)) * 3));
  energy_tile_kernel<<<tgrid, kEnergyTileThreads, kEnergyTileSmem, s>>>(chi, mu, T);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_energy_k<1>(count, grid, s, chi, mu, n, field, size, M, 1, partials);
}

cudaError_t launch_energy_masks(const double2 *chi, double2 *mu, int n, double field, u64 size,
                                const unsigned long long *masks, int count, double *partials, int grid,
                                cudaStream_t s) {
  if (n < kEnergySplitQubits || n > kMaxQubits || count < 1 || count > n) return cudaErrorInvalidValue;
  EnergyMasks M{};
  for (int j = 0; j < count; ++j) M.m[j] = masks[j];
  return launch_energy_masks_k<1>(count, grid, s, chi, mu, n, field, size, M, partials);
}

int energy_split_qubits() { return kEnergySplitQubits; }

int energy_kernel_count(int n) { return n < kEnergySplitQubits ? 1 : 2; }

int energy_grid_size(int n, int sms) {
  const u64 size = u64{1} << n;
  if (n >= kEnergySplitQubits)
    return static_cast<int>(std::min<u64>(std::max<u64>(1, size / kEnergySplitThreads), static_cast<u64>(sms) * 2));
  return static_cast<int>(std::min<u64>(std::max<u64>(1, size / kEnergyThreads), static_cast<u64>(sms) * 8));
}

// Phase table of the field terms a layer's middle pass applies
// (TmaPass::emask_phase): entry 4 j + q = -h F^2 e^{i((1 - 2 b0) phi_a + (1 - 2 b1) phi_b)}
// for the pair (a, b) = (wires[j], wires[j + 1]), q = b0 | b1 << 1 (the pair's
// bits), F the product of the tangent factors of the wires in `pending`.
// That is -h F^2 conj(D(t)) D(t ^ m) for the layer's RZ phases D.
__global__ void defer_phase_kernel(const DeferPhaseArgs A, double2 *__restrict__ out) {
  __shared__ double f2;
  const int t = threadIdx.x;
  if (t == 0) {
    double p = 1.0;
    for (int v = 0; v < A.n; ++v) {
      if (!((A.pending >> v) & 1u)) continue;
      const double4 k = A.coef[A.layer * A.n + v];
      const double f = fabs(k.x) >= fabs(k.y) ? k.x : k.y;
      p *= f * f;
    }
    f2 = p;
  }
  __syncthreads();
  if (t >= 28) return;
  const int j = t >> 2, b0 = t & 1, b1 = (t >> 1) & 1;
  const double4 ka = A.coef[A.layer * A.n + A.wires[j]], kb = A.coef[A.layer * A.n + A.wires[j + 1]];
  // e^{i phi} from (cos phi/2, sin phi/2); bit 1 conjugates
  const double2 ea = make_double2(ka.z * ka.z - ka.w * ka.w, (b0 ? -2.0 : 2.0) * ka.z * ka.w);
  const double2 eb = make_double2(kb.z * kb.z - kb.w * kb.w, (b1 ? -2.0 : 2.0) * kb.z * kb.w);
  const double c = -A.field * f2;
  const double2 e = cmul(ea, eb);
  out[t] = make_double2(c * e.x, c * e.y);
}

cudaError_t launch_defer_phase(const DeferPhaseArgs &A, double2 *out, cudaStream_t s) {
  defer_phase_kernel<<<1, 32, 0, s>>>(A, out);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalizeParams &F, cudaStream_t s) {
  finalize_kernel<<<1, 256, 0, s>>>(F);
  return cudaGetLastError();
}

}  // namespace rsv
