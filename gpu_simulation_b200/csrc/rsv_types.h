// Host/device shared descriptors for the statevector pass kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rsv {

// How a pass obtains its input amplitudes.
enum LoadMode : int {
  kLoadNatural = 0,   // buf[p]
  kLoadGatherP = 1,   // buf[P(p)]      (undo one ring layer: out = P^{-1} in)
  kLoadProduct = 2,   // analytic layer-0 product state at P^{-1}(p) (= P applied to it)
  kLoadProductPlain = 3,  // analytic layer-0 product state at p
  kLoadMpsP = 4,      // bond-4 matrix-product state of the first layers at P^{-1}(p)
                      // (forward, unit tile over index bits 0..11 only)
};

// How a pass writes its output amplitudes.
enum StoreMode : int {
  kStoreNatural = 0,    // buf[p] = v
  kStoreScatterP = 1,   // buf[P(p)] = v     (apply one ring layer)
  kStoreScatterPinv = 2,// buf[P^{-1}(p)] = v (undo one ring layer)
  kStoreNone = 3,
};

// Undo-order entries (rot_kernel): wire id, plus this flag on the first wire of
// a backward pass when the gradient correction restarts at every pass
// (checkpoint schedule).
constexpr int kUndoPassStart = 1 << 16;
// ... and this flag on a wire whose theta sum its pass takes on the same state
// as the previous wire's (the gates of one register layout, which commute,
// summed together before any of them is undone): it shares that wire's
// correction, and the group's factors apply after the group.
constexpr int kUndoSameGroup = 1 << 17;

// Partial product tables of layer 0 (checkpoint schedule): at most this many,
// each [4][256] after the full product table.
constexpr int kMaxPartialTables = 4;
struct PartialMasks {
  int count;
  unsigned int mask[kMaxPartialTables];  // wires whose RY / f is applied; the rest stay |0>
};

// Per-CTA partial record written by every backward pass (doubles):
//   [0, 12)   theta partial sums per tile bit
//   [16, 47)  phi: sum of Im(conj(lambda) psi) over amplitudes whose wire-w bit is 1
//   [47]      phi: sum of Im(conj(lambda) psi) over all amplitudes
constexpr int kPartialStride = 48;
constexpr int kPartialPhi = 16;
constexpr int kPartialTot = 47;

struct PassParams {
  int n;                 // real qubits
  int layer;             // ansatz layer whose gates this pass applies
  int num_runs;          // coset deposit runs (complement of the tile subspace)
  int run_start[4];
  int run_len[4];
  unsigned long long num_tiles;
  unsigned long long vec[12];  // physical XOR vector of each tile bit
  int gate_wire[12];           // wire gated on tile bit b, or -1
  int wire_tile_bit[32];       // tile bit of wire w for unit-vector tiles, or -1
  int need_l1;                 // any gate on tile bits 0..7 (needs the second layout)
  int need_l2;                 // any gate on tile bits 0..3 (needs the third layout)
  int psi_load, lam_load;
  int psi_store, lam_store;
  int phase;                   // fwd: apply D after gates; bwd: apply D^dagger before gates
  int phi_grad;                // bwd: accumulate the phi-gradient sums of the layer
  int sync_after_load;         // single-tile in-place permutation: all loads before any store
  int nseq;                    // register layouts visited by the pass, in order
  int seq_layout[4];           // layout id (0, 1, 2) of each visit; the last is 0
  int seq_apply[4];            // whether the visit rotates its register tile bits
  const double2 *psi_in;
  double2 *psi_out;
  const double2 *lam_in;
  double2 *lam_out;
  const double4 *coef;         // [L * n] (cos t/2, sin t/2, cos p/2, sin p/2)
  const double2 *rot;          // [L * n] tangent form of RY: (k, +1) = [[1,-k],[k,1]] (k = tan t/2)
                               // or (k, -1) = [[k,-1],[1,k]] (k = cot t/2), RY divided by f
  const double *lscale;        // [L] product of the divided factors f of each layer
  const double2 *ptab;         // phase byte tables of this layer, [4][256]
  const double2 *prod;         // layer-0 product-state byte tables, [4][256] (full or partial)
  double *partials;            // [gridDim.x][kPartialStride] for this pass
  int tile_bits;               // 12, or 11 for a backward pass on the half tile (rsv_pass_half.cu)
  const double2 *mps_btab;     // kLoadMpsP: byte tables [4][256] of 4x4 site products
  const double2 *mps_wtab;     // kLoadMpsP: products over wires 16..31 [2^max(0, n-16)]
};

// Layer-0 gradients from lambda alone (rsv_layer0.cu): per-CTA records of
// S_w(0), S_w(1) (complex) for w < 32.
constexpr int kLayer0Stride = 128;
struct Layer0Params {
  int n;
  int gather;                  // lambda0(p) = lam[P(p)] (1) or lam[p] (0)
  const double4 *coef;         // layer-0 coefficients [n]
  const double2 *lam;
  unsigned long long num_tiles;  // 2^(n-12)
  double *partials;            // [grid][kLayer0Stride]
};

// The first K layers as a matrix-product state of bond D = 2^(K-1)
// (rsv_mps.cu).  Matrices are D x D complex, row-major.  The coset index t of
// a 4096-amplitude tile (bits 12..n-1) splits into lo = its low m1 bits and hi.
struct MpsParams {
  int n, bond, m1, m2;
  const double4 *coef;         // layers 0 .. K-1 at [k n, (k+1) n)
  double2 *tsite;              // [32][2] site matrices T_w[b] (identity for w >= n)
  double2 *btab;               // [4][256] products over the eight wires of a byte
  double2 *coslo, *coshi;      // [2^m1], [2^m2] products over the coset wires
  double2 *mtab;               // [128] in-tile halves: T_0..T_5 (a), T_6..T_11 (h)
  double2 *wtab;               // [2^max(0, n-16)] products over wires 16..31 (bytes 2 and 3)
  double2 *zt;                 // [2^(n-12)] per-tile Z
  double2 *ylo, *yhi;          // [2^m1], [2^m2] coset sums
  double2 *partials;           // [grid][2][64] per-CTA G, F
  double2 *gf;                 // [2][64] G, F summed over the CTAs
  unsigned long long num_tiles;  // 2^(n-12)
};

// Inputs of the deterministic final reduction (energy + gradient).
struct FinalizeParams {
  int n, L;
  int num_energy_partials;
  const double *energy_partials;
  const double *pass_partials;   // [num_passes][max_grid][kPartialStride]
  int max_grid;
  const int *pass_grid;          // grid size of every pass
  const int *theta_pass;         // [L*n]
  const int *theta_slot;         // [L*n]
  const int *phi_pass;           // [L]
  const double *gscale;          // [2 L n] multiplier of every gradient sum
  const int *pipeline_err;       // non-zero: a TMA pass gave up waiting; outputs become NaN (may be null)
  // phi of the wires in phi_alt_wires of layer phi_alt_layer (-1: none) from
  // pass phi_alt_pass's sums, unscaled (a pass after the layer's first, where
  // psi and lambda carry reciprocal tangent factors)
  int phi_alt_layer;
  int phi_alt_pass;
  unsigned int phi_alt_wires;
  double *energy_out;
  double *grad_out;              // [2 L n] or null
};

}  // namespace rsv
