// Backward tile passes fed by the Tensor Memory Accelerator (rsv_pass_tma.cu):
// host-side description of one pass (tensor maps and tile coordinates) and
// its launcher.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

#include "rsv_types.h"

namespace rsv {

// Dimensions of a tensor map over a state buffer: every map here has rank 5
// (unused trailing dimensions have extent 1).  Dimension 0 counts doubles
// (two per amplitude) and covers index bits 0..2; each other dimension covers a
// run of consecutive index bits.  A tile's coordinate in dimension d is
// (cbase >> shift[d]) & mask[d], cbase being the tile's coset base (mask 0 for
// the dimensions the box spans).
constexpr int kTmaRank = 5;

// Kernels: kTmaHalf, an 11-bit tile with gates on tile bits 3..10 (the high
// passes); kTmaLow, the 12-bit unit tile over index bits 0..11 with every bit
// gated (the low pass).
constexpr int kTmaHalf = 0;
constexpr int kTmaLow = 1;

struct alignas(64) TmaPass {
  CUtensorMap psi_map;   // psi loads: box = the tile in tile-index order
  CUtensorMap lam_map;   // lambda loads, same box
  CUtensorMap out_map;   // kTmaHalf lambda store: box dimensions ordered tile bits 0..2, 7..10, 3..6
  int ld_shift[kTmaRank];
  unsigned int ld_mask[kTmaRank];
  int st_shift[kTmaRank];
  unsigned int st_mask[kTmaRank];
  int *err;              // device flag: set when a pipeline wait gives up
  int kind;              // kTmaHalf or kTmaLow
  // Field terms applied by the layer's first (phase) pass, set per call
  // (energy_terms = 0: none; 1 + U: the masks tma_energy_mask(U, j), j < 10,
  // in tile bits): lambda += -efield * sum_m psi(t ^ m) for every tile index t
  // (psi is the final state chi there), and the CTA's share
  // -efield * sum_t Re(conj(psi(t)) sum_m psi(t ^ m)) of the energy goes to
  // energy_partials[blockIdx.x].
  int energy_terms;
  double efield;
  double *energy_partials;
  // The layer's middle pass with the fused energy (plan-level): phi_only runs
  // the phase-pass kernel without the layer's RZ^dagger, for the phi sums of
  // its own wires (their field terms reach lambda only in this pass); per call
  // defer_terms = 1 adds those terms, the adjacent pairs of its gated tile bits
  // 3..10 (tile-bit masks m_j = 3 << (3 + j), j < 7), as
  // lambda(t) += emask_phase[4 j + q] psi(t ^ m_j), q = the pair's two bits of t:
  // -h F^2 conj(D(t)) D(t ^ m_j) with D the layer's RZ phases (undone by the
  // layer's first pass) and F the tangent factors still on psi and lambda,
  // and its energy share goes to energy_partials[blockIdx.x].
  int phi_only;
  int defer_terms;
  const double2 *emask_phase;  // [kTmaDeferTable]
};

// The field terms P^-1(e_w) inside an 11-bit phase-pass tile whose tile bits
// 0..2+U are index bits 0..2+U (ungated) and tile bits 3+U..10 the top index
// bits (gated), U = 0..3: the adjacent pairs inside each run (e_w + e_{w+1})
// and the last wire's e_{n-1} + e_0 + e_1; ten masks for every U, in tile bits.
constexpr int kTmaNumEnergyMasks = 10;
constexpr int kTmaNumDeferredMasks = 7;
constexpr int kTmaDeferTable = 4 * kTmaNumDeferredMasks;
constexpr int kTmaMaxEnergyU = 3;
__host__ __device__ constexpr unsigned tma_energy_mask(int u, int j) {
  return j == 9 ? 0x403u : (3u << (j < 2 + u ? j : j + 1));
}

// Whether a backward pass has the shape and load/store variant of a TMA
// kernel: psi and lambda loaded in natural order, lambda stored in natural
// order, psi not stored, and either (kTmaHalf) an 11-bit unit tile with tile
// bits 0..2 = index bits 0..2, increasing index bits and gates only on tile
// bits 3..10, or (kTmaLow) the 12-bit unit tile over index bits 0..11 without
// the layer's phase.  `why` (optional) receives the reason when it does not.
bool tma_pass_shape_ok(const PassParams &P, std::string *why);

// Encodes the three tensor maps of the pass (needs a CUDA context on the
// device that owns the buffers).  Returns false (with the reason) when the
// pass is not eligible or the driver rejects a map; nothing is allocated.
bool make_tma_pass(const PassParams &P, int *err, TmaPass &out, std::string *why);

// The tile bits in the order the TMA kernels rotate them (undo order).
constexpr int kTmaRotationOrder[8] = {7, 8, 9, 10, 3, 4, 5, 6};
constexpr int kTmaLowRotationOrder[12] = {8, 9, 10, 11, 0, 1, 2, 7, 3, 4, 5, 6};

cudaError_t launch_bwd_tma(const PassParams &P, const TmaPass &T, int grid, cudaStream_t s);
// blocks per SM the kernel of `kind` is laid out for (its grid: that many per SM)
int bwd_tma_blocks_per_sm(int kind);
size_t bwd_tma_smem_bytes();

}  // namespace rsv
