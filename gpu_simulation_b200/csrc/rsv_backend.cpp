// Host side of the B200 ring-Ising statevector engine: pass planner,
// scheduler, buffer ownership and the C ABI declared in include/rsv.h.
//
// Reference counterparts (zzEncounter/GPU_Simulation):
//   RingIsingCudaBackend::Impl            cpp/ising_cuda_backend.cu:333-404
//   build_structured_forward_rotation_chunks / apply_structured_forward_layers
//                                         cpp/ising_cuda_structured_adjoint_modes.inc:18-148
//   run_structured_backward_sweep         cpp/ising_cuda_structured_adjoint_modes.inc:188-307
//   run_energy_and_grad_structured_adjoint cpp/ising_cuda_structured_adjoint_modes.inc:309-373
//   StageProfiler                         cpp/ising_cuda_backend.cu:24-106
//   benchmark_structured_forward_graph    cpp/ising_cuda_backend.cu:444-541
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rsv.h"
#include "rsv_batch.h"
#include "rsv_dense.h"
#include "rsv_gate.h"
#include "rsv_device.cuh"
#include "rsv_launch.h"
#include "rsv_tma.h"
#include "rsv_types.h"

namespace rsv {
namespace {

thread_local std::string g_last_error;

struct Error : std::runtime_error {
  rsv_status status;
  Error(rsv_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

void check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  const rsv_status s = (e == cudaErrorMemoryAllocation) ? RSV_ERR_OUT_OF_MEMORY : RSV_ERR_CUDA;
  throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
}

[[noreturn]] void invalid(const std::string &m) { throw Error(RSV_ERR_INVALID_ARGUMENT, m); }

// ------------------------------------------------------------------------
// Planner
// ------------------------------------------------------------------------

struct Tile {
  u64 vec[12]{};
  int gate_wire[12];
  int dims = 12;  // tile bits in use (11: half tile of a backward pass)
  int num_runs = 0;
  int run_start[4]{};
  int run_len[4]{};
  u64 num_tiles = 1;
  bool unit = true;
  Tile() { std::fill(gate_wire, gate_wire + 12, -1); }
};

// Tile whose 12 directions are the unit vectors of `bits` (physical bit
// indices); `phys` is the number of physical index bits.  Gates are placed on
// the tile bits whose physical bit is listed in `gates`.
Tile unit_tile(int phys, const std::vector<int> &bits, const std::vector<int> &gates) {
  if (bits.size() != 12 && bits.size() != 11) throw Error(RSV_ERR_INTERNAL, "tile needs 12 or 11 directions");
  Tile t;
  t.dims = static_cast<int>(bits.size());
  std::vector<bool> in(phys, false);
  for (int b = 0; b < t.dims; ++b) {
    t.vec[b] = u64{1} << bits[b];
    in[bits[b]] = true;
    if (std::find(gates.begin(), gates.end(), bits[b]) != gates.end()) t.gate_wire[b] = bits[b];
  }
  for (int p = 0; p < phys;) {
    if (in[p]) {
      ++p;
      continue;
    }
    int q = p;
    while (q < phys && !in[q]) ++q;
    if (t.num_runs == kMaxRuns) throw Error(RSV_ERR_INTERNAL, "too many coset runs");
    t.run_start[t.num_runs] = p;
    t.run_len[t.num_runs] = q - p;
    ++t.num_runs;
    p = q;
  }
  t.num_tiles = u64{1} << (phys - t.dims);
  return t;
}

// "Antipodal" tile span(e_0..e_10, all-ones): its image under P^{-1} is the
// contiguous block span(e_0..e_11), so a scatter through P^{-1} from it writes
// whole 4096-amplitude blocks.  Gates on wires 0..10.  Needs n >= 13.  The
// twelfth direction is stored as bits 11..n-1 (all-ones minus e_0..e_10, the
// same subspace) so that it never touches a gated wire: every register pair
// along a gated direction then holds (|0>, |1>) in that order.
Tile antipodal_tile(int n) {
  Tile t;
  for (int b = 0; b < 11; ++b) {
    t.vec[b] = u64{1} << b;
    t.gate_wire[b] = b;
  }
  t.vec[11] = ((u64{1} << n) - 1) & ~u64{0x7FF};
  t.num_runs = 1;
  t.run_start[0] = 11;
  t.run_len[0] = n - 12;
  t.num_tiles = u64{1} << (n - 12);
  t.unit = false;
  return t;
}

// Split wires [lo, n) into high tiles with `c` contiguous low bits each;
// c is chosen to minimise the number of passes, then -- with wide_last, for
// the forward tiles of the checkpoint schedule -- to leave the last tile at
// most 8 gated wires (at least 4 contiguous low bits: its backward half tile
// then runs on the tensor-copy kernel and takes the fused field terms), then
// maximised (longer DRAM segments), unless force_c (2..10) fixes it (the
// autotuner's candidates).  Returns the tiles (gates on the split wires).
std::vector<Tile> high_tiles(int n, int lo, int min_c = 2, int force_c = 0, bool wide_last = false) {
  std::vector<Tile> out;
  const int m = n - lo;
  if (m <= 0) return out;
  int best_c = min_c, best_passes = 1 << 30;
  bool best_wide = false;
  for (int c = min_c; c <= 10; ++c) {
    const int g = 12 - c;
    if (c > lo) break;  // contiguity bits must lie below the gated wires
    const int passes = (m + g - 1) / g;
    const bool wide = wide_last && m - (passes - 1) * g <= 8;
    const bool better = passes < best_passes ||
                        (passes == best_passes && (wide != best_wide ? wide : c > best_c));
    if (better) {
      best_passes = passes;
      best_c = c;
      best_wide = wide;
    }
  }
  if (force_c >= min_c && force_c <= std::min(10, lo)) best_c = force_c;
  const int g = 12 - best_c;
  for (int start = lo; start < n; start += g) {
    const int end = std::min(n, start + g);
    std::vector<int> gates;
    for (int w = start; w < end; ++w) gates.push_back(w);
    const int cprime = 12 - static_cast<int>(gates.size());
    std::vector<int> bits;
    for (int b = 0; b < cprime; ++b) bits.push_back(b);
    for (int w : gates) bits.push_back(w);
    out.push_back(unit_tile(n, bits, gates));
  }
  return out;
}

// Kernel of a backward pass: bwd_pass_kernel / bwd_half_kernel by tile size,
// or the TMA-fed half-tile kernel (rsv_pass_tma.cu), which rotates its tile
// bits in another order.
constexpr int kKernelDefault = 0;
constexpr int kKernelTma = 1;

struct Step {
  bool bwd = false;
  int layer = 0;
  Tile tile;
  int psi_load = kLoadNatural, lam_load = kLoadNatural;
  int psi_store = kStoreNatural, lam_store = kStoreNone;
  int phase = 0, phi_grad = 0;
  int psi_in = -1, psi_out = -1, lam_in = -1, lam_out = -1;
  int pass_index = -1;  // backward partial record
  int prod_table = 0;   // analytic psi: 0 = full layer-0 state, j >= 1 = partial table j
  int grid = 1;
  int kernel = kKernelDefault;  // backward: which kernel runs the pass (set once buffers exist)
};

struct Plan {
  int n = 0, L = 0, phys = 0;
  bool checkpoint = false;  // backward reads forward checkpoints of psi (see make_plan)
  int num_bufs = 3;
  std::vector<Step> fwd, bwd;
  int chi_buf = 0, mu_buf = 1;
  std::vector<int> theta_pass, theta_slot, phi_pass;
  // checkpoint mode: wire masks of the partial layer-0 product tables 1..
  std::vector<unsigned int> partial_masks;
  int max_grid = 1;
  // layer 0 on the layer-0 kernel (rsv_layer0.cu): its backward passes are
  // dropped; the kernel reads lambda from buffer layer0_lam (gathered
  // through P when layer0_load is kLoadGatherP)
  bool layer0_kernel = false;
  int layer0_lam = -1, layer0_load = kLoadNatural, layer0_grid = 1;
  // the first mps_k layers as a matrix-product state of bond 2^(mps_k - 1)
  // (rsv_mps.cu, 0: not used): their passes are dropped; the forward writes
  // their output into buffer mps_out (scattered through P when layers
  // follow), the backward reads lambda at that point from buffer mps_lam
  int mps_k = 0;
  bool mps_scatter = false;
  int mps_out = -1, mps_lam = -1, mps_load = kLoadNatural, mps_fwd_grid = 1, mps_grad_grid = 1;
  // bond 4 with layers after it: the first forward pass of layer mps_k
  // evaluates the state itself (kLoadMpsP) and nothing writes mps_out
  bool mps_fused = false;
};

// Checkpoint-mode plans keep one state buffer per forward pass of the layers
// on tile passes, plus lambda; they are chosen automatically while those fit
// this budget: 128 GiB, what the reference's own four state buffers take at
// n = 31, with about 50 GB of a B200 left over.
constexpr double kCheckpointBudgetBytes = 128.0 * (1ull << 30);

Plan make_plan(int n, int L, int sms, bool checkpoint, int analytic, int force_c = 0);

// The checkpoint schedule is chosen automatically while its state buffers
// (after the leading layers the analytic kernels replace) fit the budget.
bool checkpoint_fits(int n, int L, int analytic, int force_c = 0) {
  if (n <= kTileBits) return false;
  const double bufs = static_cast<double>(make_plan(n, L, 148, true, analytic, force_c).num_bufs);
  return bufs * 16.0 * static_cast<double>(u64{1} << n) <= kCheckpointBudgetBytes;
}

void record_theta(Plan &pl, const Step &s) {
  for (int b = 0; b < 12; ++b) {
    const int w = s.tile.gate_wire[b];
    if (w < 0) continue;
    const size_t k = static_cast<size_t>(s.layer) * pl.n + w;
    if (pl.theta_pass[k] >= 0) throw Error(RSV_ERR_INTERNAL, "wire planned twice");
    pl.theta_pass[k] = s.pass_index;
    pl.theta_slot[k] = b;
  }
}

// Backward passes whose gates all lie on tile bits 4..11 of a unit tile with
// tile bits 0..3 = index bits 0..3 run on the 11-bit half tile (the highest
// of the leading contiguous ungated tile bits moves to the coset) with two
// 256-thread CTAs per SM (rsv_pass_half.cu),
// for the load/store variants that kernel has, once the pass has at least
// eight 12-bit tiles per SM (smaller states sit in L2, where the extra CTAs
// only add launch cost: n = 20 ran 6% slower on half tiles).
bool half_tile_variant(const Step &s) {
  const int pl = s.psi_load, ll = s.lam_load, ps = s.psi_store, ls = s.lam_store;
  if (pl == kLoadNatural && ps == kStoreNatural && ls == kStoreNatural)
    return ll == kLoadNatural || ll == kLoadGatherP;
  if (ps != kStoreNone || ls != kStoreNatural) return false;
  return (pl == kLoadNatural && ll == kLoadNatural) || (pl == kLoadGatherP && ll == kLoadGatherP) ||
         (pl == kLoadProductPlain && (ll == kLoadGatherP || ll == kLoadNatural));
}

// Layer 0's gradients need only lambda at the output of layer 0 (its state is
// an analytic product state): n >= 13 replaces the layer's backward passes by
// one read of lambda on the layer-0 kernel.
void use_layer0_kernel(Plan &pl, int sms) {
  if (pl.n < 13) return;
  auto first = std::find_if(pl.bwd.begin(), pl.bwd.end(), [](const Step &s) { return s.layer == 0; });
  if (first == pl.bwd.end()) return;
  pl.layer0_lam = first->lam_in;
  pl.layer0_load = first->lam_load;
  if (pl.layer0_load != kLoadNatural && pl.layer0_load != kLoadGatherP) return;
  pl.bwd.erase(std::remove_if(pl.bwd.begin(), pl.bwd.end(), [](const Step &s) { return s.layer == 0; }),
               pl.bwd.end());
  for (int w = 0; w < pl.n; ++w) {
    pl.theta_pass[static_cast<size_t>(w)] = -1;
    pl.theta_slot[static_cast<size_t>(w)] = -1;
  }
  pl.phi_pass[0] = -1;
  pl.layer0_kernel = true;
  pl.layer0_grid = static_cast<int>(std::min<u64>(u64{1} << (pl.n - 12), static_cast<u64>(2 * std::max(1, sms))));
}

constexpr int kDefaultAnalyticLayers = 3;

// The first K = min(L, 3) layers form a matrix-product state of bond
// 2^(K-1) (rsv_mps.cu).  For n >= 13 their forward passes become one write of
// that state and their backward passes one read of lambda at its output, which
// gives all their 2nK gradients.
void use_mps(Plan &pl, int sms, int max_k) {
  if (pl.n < 13 || pl.L < 2) return;
  const int K = std::min(pl.L, std::min(max_k, 3));
  if (K < 2) return;
  int last = -1;
  for (size_t i = 0; i < pl.fwd.size(); ++i)
    if (pl.fwd[i].layer == K - 1) last = static_cast<int>(i);
  auto first = std::find_if(pl.bwd.begin(), pl.bwd.end(), [K](const Step &s) { return s.layer == K - 1; });
  if (last < 0 || first == pl.bwd.end()) return;
  const Step &s = pl.fwd[static_cast<size_t>(last)];
  if (s.psi_store != kStoreNatural && s.psi_store != kStoreScatterP) return;
  if (first->lam_load != kLoadNatural && first->lam_load != kLoadGatherP) return;
  pl.mps_out = s.psi_out;
  pl.mps_scatter = s.psi_store == kStoreScatterP;
  pl.mps_lam = first->lam_in;
  pl.mps_load = first->lam_load;
  pl.fwd.erase(std::remove_if(pl.fwd.begin(), pl.fwd.end(), [K](const Step &x) { return x.layer < K; }),
               pl.fwd.end());
  pl.bwd.erase(std::remove_if(pl.bwd.begin(), pl.bwd.end(), [K](const Step &x) { return x.layer < K; }),
               pl.bwd.end());
  for (int k = 0; k < K * pl.n; ++k) {
    pl.theta_pass[static_cast<size_t>(k)] = -1;
    pl.theta_slot[static_cast<size_t>(k)] = -1;
  }
  for (int l = 0; l < K; ++l) pl.phi_pass[static_cast<size_t>(l)] = -1;
  pl.mps_k = K;
  if (K == 3 && pl.L > K && !pl.fwd.empty() && pl.mps_scatter) {
    Step &f = pl.fwd.front();
    bool unit = f.tile.dims == 12;
    for (int b = 0; unit && b < 12; ++b) unit = f.tile.vec[b] == (u64{1} << b);
    if (unit && f.layer == K && f.psi_load == kLoadNatural && f.psi_in == pl.mps_out &&
        f.psi_store == kStoreNatural && !f.phase) {
      f.psi_load = kLoadMpsP;
      f.psi_in = -1;
      pl.mps_fused = true;
    }
  }
  // psi at the input of layer K (written back by the uncompute schedule for
  // the layers below) is not needed: those layers' gradients come from lambda
  if (!pl.bwd.empty() && pl.bwd.back().layer == K && pl.bwd.back().tile.dims == 12) {
    pl.bwd.back().psi_store = kStoreNone;
    pl.bwd.back().psi_out = -1;
  }
  const u64 tiles = u64{1} << (pl.n - 12);
  pl.mps_fwd_grid = static_cast<int>(std::min<u64>(tiles, static_cast<u64>(8 * std::max(1, sms))));
  // bond 2: two CTAs per SM (83 KiB of shared memory), bond 4: one (135 KiB)
  pl.mps_grad_grid = static_cast<int>(std::min<u64>(tiles, static_cast<u64>((K == 2 ? 2 : 1) * std::max(1, sms))));
}

void use_half_tiles(Plan &pl, int sms) {
  const int ctas = 2 * std::max(1, sms);
  for (auto &s : pl.bwd) {
    const Tile &t = s.tile;
    if (!t.unit || t.dims != 12 || !half_tile_variant(s)) continue;
    if (t.num_tiles < static_cast<u64>(8) * std::max(1, sms)) continue;
    // c leading tile bits are the contiguous, ungated index bits 0..c-1 (c >= 4);
    // the top one moves to the coset, so index bits 0..c-2 stay contiguous
    int c = 0;
    while (c < 12 && t.gate_wire[c] < 0 && t.vec[c] == (u64{1} << c)) ++c;
    if (c < 4) continue;
    std::vector<int> bits, gates;
    for (int b = 0; b < 12; ++b) {
      if (b == c - 1) continue;
      int bit = 0;
      while (!((t.vec[b] >> bit) & 1)) ++bit;
      bits.push_back(bit);
      if (t.gate_wire[b] >= 0) gates.push_back(t.gate_wire[b]);
    }
    s.tile = unit_tile(pl.phys, bits, gates);
    s.grid = static_cast<int>(std::min<u64>(s.tile.num_tiles, static_cast<u64>(ctas)));
    pl.max_grid = std::max(pl.max_grid, s.grid);
    for (int b = 0; b < s.tile.dims; ++b) {
      const int w = s.tile.gate_wire[b];
      if (w >= 0) pl.theta_slot[static_cast<size_t>(s.layer) * pl.n + w] = b;
    }
  }
}

Plan make_checkpoint_plan(Plan pl, const std::vector<Tile> &fwd_tiles, int fwd_ctas, int bwd_ctas) {
  const int n = pl.n, L = pl.L;
  const int P = static_cast<int>(fwd_tiles.size());
  auto grid_for = [](const Tile &t, int ctas) {
    return static_cast<int>(std::min<u64>(t.num_tiles, static_cast<u64>(ctas)));
  };
  std::vector<int> all_bits(12);
  for (int b = 0; b < 12; ++b) all_bits[b] = b;
  int next = 0;
  std::vector<std::vector<int>> ck(L);  // ck[l][j]: buffer written by forward pass j of layer l
  int cur = -1;                          // input of the next layer (after its CNOT ring)
  if (L == 1) {
    Step s;
    s.tile = unit_tile(pl.phys, all_bits, {});
    s.psi_load = kLoadProductPlain;
    s.psi_out = next++;
    s.psi_store = kStoreNatural;
    s.grid = grid_for(s.tile, fwd_ctas);
    pl.fwd.push_back(s);
    cur = s.psi_out;
  }
  for (int layer = 1; layer < L; ++layer) {
    for (int j = 0; j < P; ++j) {
      const bool first = j == 0, last = j + 1 == P;
      Step s;
      s.layer = layer;
      s.tile = fwd_tiles[static_cast<size_t>(j)];
      s.psi_load = (first && layer == 1) ? kLoadProduct : kLoadNatural;
      s.psi_in = s.psi_load == kLoadNatural ? (first ? cur : ck[layer].back()) : -1;
      s.phase = last ? 1 : 0;
      s.psi_out = next++;
      s.psi_store = (last && layer + 1 < L) ? kStoreScatterP : kStoreNatural;
      s.grid = grid_for(s.tile, fwd_ctas);
      ck[layer].push_back(s.psi_out);
      if (last) cur = s.psi_out;
      pl.fwd.push_back(s);
    }
  }
  pl.chi_buf = cur;
  pl.mu_buf = next++;
  pl.num_bufs = next;

  // partial product tables of layer 0: table j+1 = wires of forward passes 0..j
  // applied (RY / f on |0>, no RZ), every other wire still |0>
  for (int j = 0; j + 1 < P; ++j) {
    unsigned int m = 0;
    for (int jj = 0; jj <= j; ++jj)
      for (int b = 0; b < 12; ++b)
        if (fwd_tiles[static_cast<size_t>(jj)].gate_wire[b] >= 0)
          m |= 1u << fwd_tiles[static_cast<size_t>(jj)].gate_wire[b];
    pl.partial_masks.push_back(m);
  }

  pl.theta_pass.assign(static_cast<size_t>(n) * L, -1);
  pl.theta_slot.assign(static_cast<size_t>(n) * L, -1);
  pl.phi_pass.assign(L, -1);
  int lam = pl.mu_buf;
  int pass_index = 0;
  for (int layer = L - 1; layer >= 0; --layer) {
    for (int gi = 0; gi < P; ++gi) {
      const int j = P - 1 - gi;  // the forward pass this backward pass undoes
      const bool first = gi == 0, final_pass = layer == 0 && gi + 1 == P;
      Step s;
      s.bwd = true;
      s.layer = layer;
      s.tile = fwd_tiles[static_cast<size_t>(j)];
      s.phase = first ? 1 : 0;
      s.phi_grad = first ? 1 : 0;
      if (s.phi_grad && !s.tile.unit) throw Error(RSV_ERR_INTERNAL, "phi pass needs a unit tile");
      if (layer == 0) {
        s.psi_load = kLoadProductPlain;
        s.prod_table = first ? 0 : j + 1;
      } else {
        s.psi_in = ck[layer][static_cast<size_t>(j)];
        s.psi_load = (first && layer + 1 < L) ? kLoadGatherP : kLoadNatural;
      }
      s.psi_store = kStoreNone;
      s.lam_in = lam;
      s.lam_load = (first && layer + 1 < L) ? kLoadGatherP : kLoadNatural;
      if (s.lam_load == kLoadGatherP) {
        // the checkpoints of layer + 1 are dead: take one for lambda
        s.lam_out = ck[layer + 1][0];
        lam = s.lam_out;
      } else {
        s.lam_out = lam;
      }
      s.lam_store = final_pass ? kStoreNone : kStoreNatural;
      s.pass_index = pass_index++;
      s.grid = grid_for(s.tile, bwd_ctas);
      record_theta(pl, s);
      if (first) pl.phi_pass[layer] = s.pass_index;
      pl.max_grid = std::max(pl.max_grid, s.grid);
      pl.bwd.push_back(s);
    }
  }
  for (size_t k = 0; k < pl.theta_pass.size(); ++k)
    if (pl.theta_pass[k] < 0) throw Error(RSV_ERR_INTERNAL, "wire without a backward pass");
  return pl;
}

// Two backward schedules share the forward tiles and the kernels:
//   uncompute (checkpoint = false): three state buffers; the backward
//     un-computes psi alongside lambda (reads and writes both), and its last
//     pass per layer scatters psi through P^-1 (antipodal tile);
//   checkpoint: every forward pass writes a fresh buffer; backward pass j of a
//     layer undoes exactly the wires of forward pass P-1-j, reads psi from the
//     checkpoint after that forward pass (gathered through P for the layer's
//     last pass, analytic product tables for layer 0) and writes only lambda.
//     Reference counterpart: run_structured_backward_sweep
//     (cpp/ising_cuda_structured_adjoint_modes.inc:188-307), which always
//     un-computes psi.
Plan make_plan_full(int n, int L, int sms, bool checkpoint, int force_c = 0);

// Plans of the single-circuit engine (half tiles on the eligible backward
// passes); the batched kernel and the fixed-workspace entry point use
// make_plan_full, whose tiles all have 12 bits.
// analytic: how many leading layers may skip their tile passes (3: layers
// 0..2 as a matrix-product state, 2: layers 0..1, 1: layer 0's backward on the
// layer-0 kernel, 0: every layer on tile passes, layer 0 computed in layer 1's
// first forward pass as in the reference).
// Renumber the state buffers the plan still uses as 0, 1, ... (the passes of
// the layers that the matrix-product or layer-0 kernels replace leave their
// checkpoints unused); at least two (the gate-level path uses buffers 0, 1).
void compact_buffers(Plan &pl) {
  std::vector<int> map(static_cast<size_t>(std::max(pl.num_bufs, 0)), -1);
  int next = 0;
  auto use = [&](int &b) {
    if (b < 0) return;
    if (b >= static_cast<int>(map.size())) throw Error(RSV_ERR_INTERNAL, "buffer id out of range");
    if (map[static_cast<size_t>(b)] < 0) map[static_cast<size_t>(b)] = next++;
    b = map[static_cast<size_t>(b)];
  };
  for (auto &s : pl.fwd) {
    use(s.psi_in);
    use(s.psi_out);
  }
  use(pl.chi_buf);
  use(pl.mu_buf);
  for (auto &s : pl.bwd) {
    use(s.psi_in);
    use(s.psi_out);
    use(s.lam_in);
    use(s.lam_out);
  }
  if (pl.mps_k > 0 && !pl.mps_fused) use(pl.mps_out);
  if (pl.mps_k > 0) use(pl.mps_lam);
  if (pl.layer0_kernel) use(pl.layer0_lam);
  pl.num_bufs = std::max(next, 2);
}

Plan make_plan(int n, int L, int sms, bool checkpoint, int analytic, int force_c) {
  Plan pl = make_plan_full(n, L, sms, checkpoint, force_c);
  use_half_tiles(pl, sms);
  if (analytic >= 2) use_mps(pl, sms, analytic);
  if (pl.mps_k == 0 && analytic >= 1) use_layer0_kernel(pl, sms);
  compact_buffers(pl);
  return pl;
}

Plan make_plan_full(int n, int L, int sms, bool checkpoint, int force_c) {
  Plan pl;
  pl.n = n;
  pl.L = L;
  pl.phys = std::max(n, kTileBits);
  const bool single = (pl.phys == kTileBits);
  if (single) checkpoint = false;  // one tile: every permutation in place, three buffers
  pl.checkpoint = checkpoint;
  const int fwd_ctas = std::max(1, 2 * sms), bwd_ctas = std::max(1, sms);

  std::vector<int> all_bits(12), real_wires;
  for (int b = 0; b < 12; ++b) all_bits[b] = b;
  for (int w = 0; w < std::min(n, 12); ++w) real_wires.push_back(w);

  std::vector<Tile> fwd_tiles, bwd_tiles;
  if (single) {
    fwd_tiles.push_back(unit_tile(pl.phys, all_bits, real_wires));
    bwd_tiles.push_back(unit_tile(pl.phys, all_bits, real_wires));
  } else {
    fwd_tiles = high_tiles(n, 12, 2, force_c, checkpoint);
    fwd_tiles.insert(fwd_tiles.begin(), unit_tile(n, all_bits, all_bits));
    bwd_tiles = high_tiles(n, 11, 2, force_c);
    std::reverse(bwd_tiles.begin(), bwd_tiles.end());  // highest wires first
    bwd_tiles.push_back(antipodal_tile(n));
  }
  auto grid_for = [](const Tile &t, int ctas) {
    return static_cast<int>(std::min<u64>(t.num_tiles, static_cast<u64>(ctas)));
  };
  if (checkpoint) return make_checkpoint_plan(pl, fwd_tiles, fwd_ctas, bwd_ctas);

  // Forward.  Layer 0 is the analytic product state; layers 1..L-1 run
  // their passes; the last pass of each layer applies the RZ phase and, except
  // for the final layer, scatters through P into the other buffer.
  int cur = 0, other = 1;
  if (L == 1) {
    Step s;
    s.tile = unit_tile(pl.phys, all_bits, {});
    s.psi_load = kLoadProductPlain;
    s.psi_out = cur;
    s.psi_store = kStoreNatural;
    s.grid = grid_for(s.tile, fwd_ctas);
    pl.fwd.push_back(s);
  }
  for (int layer = 1; layer < L; ++layer) {
    for (size_t gi = 0; gi < fwd_tiles.size(); ++gi) {
      const bool first = gi == 0, last = gi + 1 == fwd_tiles.size();
      Step s;
      s.layer = layer;
      s.tile = fwd_tiles[gi];
      s.psi_load = first ? (layer == 1 ? kLoadProduct : kLoadNatural) : kLoadNatural;
      s.psi_in = (s.psi_load == kLoadNatural) ? cur : -1;
      s.phase = last ? 1 : 0;
      if (last && layer + 1 < L) {
        s.psi_store = kStoreScatterP;
        s.psi_out = other;
        std::swap(cur, other);
      } else {
        s.psi_store = kStoreNatural;
        s.psi_out = cur;
      }
      s.grid = grid_for(s.tile, fwd_ctas);
      pl.fwd.push_back(s);
    }
  }
  pl.chi_buf = cur;
  pl.mu_buf = other;

  // Backward.  Buffers: psi, lam, and one free.  The first pass of layer l
  // gathers lambda through P (undoing the ring of layer l+1) into the free
  // buffer; the last pass scatters psi through P^{-1} into the free buffer.
  int psi = cur, lam = other, freeb = 3 - cur - other;
  pl.theta_pass.assign(static_cast<size_t>(n) * L, -1);
  pl.theta_slot.assign(static_cast<size_t>(n) * L, -1);
  pl.phi_pass.assign(L, -1);
  int pass_index = 0;
  for (int layer = L - 1; layer >= 0; --layer) {
    for (size_t gi = 0; gi < bwd_tiles.size(); ++gi) {
      const bool first = gi == 0, last = gi + 1 == bwd_tiles.size();
      Step s;
      s.bwd = true;
      s.layer = layer;
      s.tile = bwd_tiles[gi];
      s.phase = first ? 1 : 0;
      s.phi_grad = first ? 1 : 0;
      if (s.phi_grad && !s.tile.unit) throw Error(RSV_ERR_INTERNAL, "phi pass needs a unit tile");
      s.psi_load = kLoadNatural;
      s.psi_in = psi;
      s.lam_load = (first && layer + 1 < L) ? kLoadGatherP : kLoadNatural;
      s.lam_in = lam;
      const bool scatter_psi = last && layer > 0;
      const bool final_pass = last && layer == 0;
      if (single) {
        // One CTA holds the whole state: every permutation is done in place.
        s.psi_out = psi;
        s.lam_out = lam;
        s.psi_store = final_pass ? kStoreNone : (scatter_psi ? kStoreScatterPinv : kStoreNatural);
        s.lam_store = final_pass ? kStoreNone : kStoreNatural;
      } else {
        if (s.lam_load == kLoadGatherP) {
          s.lam_out = freeb;
          freeb = lam;
          lam = s.lam_out;
        } else {
          s.lam_out = lam;
        }
        s.lam_store = final_pass ? kStoreNone : kStoreNatural;
        if (scatter_psi) {
          s.psi_store = kStoreScatterPinv;
          s.psi_out = freeb;
          freeb = psi;
          psi = s.psi_out;
        } else {
          s.psi_store = final_pass ? kStoreNone : kStoreNatural;
          s.psi_out = psi;
        }
      }
      s.pass_index = pass_index++;
      s.grid = grid_for(s.tile, bwd_ctas);
      for (int b = 0; b < 12; ++b) {
        const int w = s.tile.gate_wire[b];
        if (w < 0) continue;
        const size_t k = static_cast<size_t>(layer) * n + w;
        if (pl.theta_pass[k] >= 0) throw Error(RSV_ERR_INTERNAL, "wire planned twice");
        pl.theta_pass[k] = s.pass_index;
        pl.theta_slot[k] = b;
      }
      if (first) pl.phi_pass[layer] = s.pass_index;
      pl.max_grid = std::max(pl.max_grid, s.grid);
      pl.bwd.push_back(s);
    }
  }
  for (size_t k = 0; k < pl.theta_pass.size(); ++k)
    if (pl.theta_pass[k] < 0) throw Error(RSV_ERR_INTERNAL, "wire without a backward pass");
  return pl;
}

// Undo order of the wires within one backward layer, as the backward pass
// kernel visits them: passes in plan order; inside a pass the register groups
// of tile bits 9..11, 6..8, 0..2, then 3..5 (layouts B0, B1, A1, A2 of
// rsv_pass.cu and of the batched kernel).  Needed for the exact tangent-form
// gradient correction.  In checkpoint mode the first wire of every pass
// carries kUndoPassStart (the gradient correction restarts there, see
// rot_kernel).
// The wires of one layer in the order its backward passes undo them (with
// kUndoPassStart on the first wire of every pass in the checkpoint schedule).
std::vector<int> undo_order_layer(const Plan &pl, int layer) {
  // tile bits in the order the backward kernels rotate them: bwd_pass_kernel
  // B0, B1, A1, A2 (rsv_pass.cu); bwd_half_kernel H0, H1, HA (rsv_pass_half.cu);
  // the TMA kernel P, Q (rsv_pass_tma.cu)
  static const int kBits[12] = {9, 10, 11, 6, 7, 8, 0, 1, 2, 3, 4, 5};
  static const int kBitsHalf[11] = {8, 9, 10, 5, 6, 7, 3, 4, 0, 1, 2};
  std::vector<int> ord;
  for (const auto &s : pl.bwd) {
    if (s.layer != layer) continue;
    bool start = pl.checkpoint;
    const bool tma = s.kernel == kKernelTma;
    const int count = tma ? (s.tile.dims == 12 ? 12 : 8) : s.tile.dims;
    // the TMA kernels take the theta sums of their last four rotations (tile
    // bits 3..6, the end of their order) together on one state
    const int group_from = tma ? count - 4 : count;
    bool in_group = false;
    for (int i = 0; i < count; ++i) {
      const int b = tma ? (s.tile.dims == 12 ? kTmaLowRotationOrder[i] : kTmaRotationOrder[i])
                        : (s.tile.dims == 12 ? kBits[i] : kBitsHalf[i]);
      const int w = s.tile.gate_wire[b];
      if (w < 0) continue;
      int e = start ? (w | kUndoPassStart) : w;
      if (i >= group_from) {
        if (in_group && !start) e |= kUndoSameGroup;
        in_group = true;
      }
      ord.push_back(e);
      start = false;
    }
  }
  if (ord.empty()) {
    // a layer without passes (layer-0 or matrix-product kernels): no gradient correction is used
    for (int w = 0; w < pl.n; ++w) ord.push_back(w);
  }
  if (static_cast<int>(ord.size()) != pl.n) throw Error(RSV_ERR_INTERNAL, "undo order incomplete");
  return ord;
}

// The last layer's undo order (every layer of the plans that the batched
// kernel and the fixed-workspace entry point run has the same one).
std::vector<int> undo_order(const Plan &pl) { return undo_order_layer(pl, pl.L - 1); }

// Every layer's undo order, layer after layer ([L][n]).
std::vector<int> undo_orders(const Plan &pl) {
  std::vector<int> ord;
  for (int l = 0; l < pl.L; ++l) {
    const std::vector<int> o = undo_order_layer(pl, l);
    ord.insert(ord.end(), o.begin(), o.end());
  }
  return ord;
}

const char *load_name(int m) {
  switch (m) {
    case kLoadNatural: return "load";
    case kLoadGatherP: return "gatherP";
    case kLoadProduct: return "product(P)";
    case kLoadProductPlain: return "product";
    case kLoadMpsP: return "mpsP";
  }
  return "?";
}

const char *store_name(int m) {
  switch (m) {
    case kStoreNatural: return "store";
    case kStoreScatterP: return "scatterP";
    case kStoreScatterPinv: return "scatterPinv";
    case kStoreNone: return "none";
  }
  return "?";
}

std::string describe(const Plan &pl) {
  std::ostringstream os;
  auto tile_str = [](const Tile &t) {
    std::ostringstream ts;
    ts << "dirs=[";
    for (int b = 0; b < t.dims; ++b) {
      if (b) ts << ",";
      if ((t.vec[b] & (t.vec[b] - 1)) == 0) {
        int bit = 0;
        while (!((t.vec[b] >> bit) & 1)) ++bit;
        ts << bit;
      } else {
        ts << "0x" << std::hex << t.vec[b] << std::dec;
      }
    }
    ts << "] gates=[";
    bool any = false;
    for (int b = 0; b < 12; ++b)
      if (t.gate_wire[b] >= 0) {
        ts << (any ? "," : "") << t.gate_wire[b];
        any = true;
      }
    ts << "] runs=[";
    for (int r = 0; r < t.num_runs; ++r) ts << (r ? "," : "") << t.run_start[r] << ":" << t.run_len[r];
    ts << "] tiles=" << t.num_tiles;
    return ts.str();
  };
  os << "n=" << pl.n << " L=" << pl.L << " phys=" << pl.phys << " bufs=" << pl.num_bufs
     << " mode=" << (pl.checkpoint ? "checkpoint" : "uncompute") << "\n";
  if (pl.mps_k > 0 && !pl.mps_fused)
    os << "mps K=" << pl.mps_k << " fwd psi:" << (pl.mps_scatter ? "scatterP" : "store") << "(" << pl.mps_out
       << ") grid=" << pl.mps_fwd_grid << "\n";
  for (const auto &s : pl.fwd)
    os << "fwd layer=" << s.layer << " " << tile_str(s.tile) << " psi:" << load_name(s.psi_load)
       << "(" << s.psi_in << ")->" << store_name(s.psi_store) << "(" << s.psi_out << ")"
       << (s.phase ? " phase" : "") << " grid=" << s.grid << "\n";
  os << "energy chi=" << pl.chi_buf << " mu=" << pl.mu_buf << "\n";
  auto psi_src = [&](const Step &s) -> std::string {
    if (s.psi_load == kLoadProductPlain && s.prod_table > 0) {
      std::ostringstream ps;
      ps << "partial(0x" << std::hex << pl.partial_masks[static_cast<size_t>(s.prod_table - 1)] << ")";
      return ps.str();
    }
    return load_name(s.psi_load);
  };
  for (const auto &s : pl.bwd)
    os << "bwd layer=" << s.layer << " pass=" << s.pass_index << " " << tile_str(s.tile)
       << " psi:" << psi_src(s) << "(" << s.psi_in << ")->" << store_name(s.psi_store)
       << "(" << s.psi_out << ") lam:" << load_name(s.lam_load) << "(" << s.lam_in << ")->"
       << store_name(s.lam_store) << "(" << s.lam_out << ")" << (s.phase ? " phase" : "")
       << (s.phi_grad ? " phi" : "") << (s.kernel == kKernelTma ? " kernel=tma" : "") << " grid=" << s.grid
       << "\n";
  if (pl.mps_k > 0)
    os << "mps K=" << pl.mps_k << " grad lam:" << load_name(pl.mps_load) << "(" << pl.mps_lam
       << ") grid=" << pl.mps_grad_grid << "\n";
  if (pl.layer0_kernel)
    os << "layer0 lam:" << load_name(pl.layer0_load) << "(" << pl.layer0_lam << ") grid=" << pl.layer0_grid << "\n";
  os << "finalize\n";
  return os.str();
}

// ------------------------------------------------------------------------
// Backend
// ------------------------------------------------------------------------

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t count = 0;
  bool owned = true;
  void alloc(size_t n) {
    release();
    if (n == 0) return;
    check(cudaMalloc(&p, n * sizeof(T)), "cudaMalloc");
    count = n;
    owned = true;
  }
  // Non-owning view of caller-provided device memory (never freed here).
  void view(T *ptr, size_t n) {
    release();
    p = ptr;
    count = n;
    owned = false;
  }
  void release() {
    if (p && owned) cudaFree(p);
    p = nullptr;
    count = 0;
    owned = true;
  }
  ~DevBuf() { release(); }
};

template <typename T>
struct HostBuf {
  T *p = nullptr;
  void alloc(size_t n) {
    if (p) cudaFreeHost(p);
    p = nullptr;
    if (n) check(cudaMallocHost(&p, n * sizeof(T)), "cudaMallocHost");
  }
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
};

constexpr int kNumStages = 8;
const char *kStageNames[kNumStages] = {
    "build_ops_host_ms",  "zero_state_ms",    "forward_apply_ms",  "hamiltonian_ms",
    "energy_dot_ms",      "gradient_zero_ms", "backward_sweep_ms", "gradient_copy_ms"};

}  // namespace
}  // namespace rsv

struct rsv_backend {
  int n = 0, L = 0;
  double field = 0.0;
  size_t num_params = 0;
  size_t state_len = 0;  // amplitudes per buffer (2^max(n,12))
  int device = 0, sms = 0;
  cudaStream_t stream = nullptr;
  rsv::Plan plan;
  rsv::DevBuf<double2> states;  // plan.num_bufs state buffers of state_len amplitudes each
  int backward_mode = RSV_BACKWARD_AUTO;
  // RSV_KERNELS_* flags (rsv_set_kernels): TMA-fed backward passes where
  // eligible, the field terms on the tile of the last layer's first backward
  // pass applied by that pass in energy_and_grad calls
  int kernel_flags = RSV_KERNELS_TMA | RSV_KERNELS_FUSED_ENERGY;
  int energy_fuse_pass = -1;                      // that pass's step index, or -1
  int energy_fuse_grid = 0;                       // its grid (= its energy partials)
  // the layer's middle pass applying the field terms of its gated wires (phase
  // table per call from defer_args), or -1
  int energy_defer_pass = -1;
  int energy_defer_grid = 0;
  unsigned int energy_defer_wires = 0;            // its gated wires (their phi from that pass)
  rsv::DeferPhaseArgs defer_args{};
  rsv::DevBuf<double2> defer_phase;               // [kTmaDeferTable]
  std::vector<unsigned long long> energy_rest;    // the other field-term masks
  int force_c = 0;  // contiguous low bits of the high tiles (0: the planner's choice)
  std::string tune_report;  // the last rsv_autotune's candidates and choice
  std::vector<rsv::TmaPass> tma;    // per backward step (used where step.kernel is kKernelTma)
  rsv::DevBuf<int> pipeline_err;    // set by a TMA pass whose pipeline wait gave up
  int tma_passes = 0;
  int analytic_layers = 3;  // rsv_set_analytic_layers (default: layers 0..2 as a matrix-product state)
  // gradient_strategy "inverse_walk_cuQuantum": gate-level kernels (rsv_gate.cu)
  bool gate_level = false;
  int gate_grid = 1;
  rsv::DevBuf<double> gate_partials;  // [1 + 2 n L][gate_grid]
  // gradient_strategy "dense_scan" (n <= 8): dense layer products (rsv_dense.cu)
  bool dense = false;
  rsv::DevBuf<double2> dense_work;
  rsv::DevBuf<double4> coef;
  rsv::DevBuf<double2> ptab, prod;
  rsv::DevBuf<double> energy_partials, pass_partials, outputs;  // outputs: [1 + num_params]
  rsv::DevBuf<double> layer0_partials;                           // [layer0_grid][kLayer0Stride]
  // matrix-product stage (rsv_mps.cu): site matrices, forward byte tables,
  // coset tables, per-tile Z, coset sums, per-CTA G/F and their sums
  rsv::DevBuf<double2> mps_tsite, mps_btab, mps_coslo, mps_coshi, mps_mtab, mps_wtab, mps_zt, mps_ylo, mps_yhi, mps_partials,
      mps_gf;
  rsv::DevBuf<int> tables;  // pass_grid | theta_pass | theta_slot | phi_pass
  rsv::DevBuf<int> order;   // undo order of the wires within a backward layer
  rsv::DevBuf<double2> rot;
  rsv::DevBuf<double> lscale, gscale;
  rsv::HostBuf<double4> coef_host;
  rsv::HostBuf<double> out_host;
  int energy_grid = 1;
  int num_bwd_passes = 0;
  // Bumped by every call that overwrites the state buffers; a forward-only
  // call records its value so that a deferred backward can check it.
  unsigned long long generation = 0;
  bool forward_only_state = false;
  // kernels launched by this backend's calls (rsv_kernel_launches)
  unsigned long long kernels_launched = 0;
  // launch timing (rsv_set_launch_timing)
  bool timing = false;
  struct Rec {
    cudaEvent_t a, b;
    int kind;
    double bytes;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> event_pool;
};

namespace rsv {
namespace {

double2 *state_buf(const rsv_backend *B, int i) { return B->states.p + static_cast<size_t>(i) * B->state_len; }

void fill_pass_params(rsv_backend *B, const Step &s, PassParams &P) {
  std::memset(&P, 0, sizeof(P));
  P.n = B->n;
  P.layer = s.layer;
  P.num_runs = s.tile.num_runs;
  for (int r = 0; r < 4; ++r) {
    P.run_start[r] = s.tile.run_start[r];
    P.run_len[r] = s.tile.run_len[r];
  }
  P.num_tiles = s.tile.num_tiles;
  for (int b = 0; b < 32; ++b) P.wire_tile_bit[b] = -1;
  P.tile_bits = s.tile.dims;
  bool l1 = false, l2 = false;
  for (int b = 0; b < 12; ++b) {
    P.vec[b] = s.tile.vec[b];
    P.gate_wire[b] = s.tile.gate_wire[b];
    if (s.tile.gate_wire[b] >= 0 && b < 8) l1 = true;
    if (s.tile.gate_wire[b] >= 0 && b < 4) l2 = true;
    if (s.tile.unit && b < s.tile.dims) {
      int bit = 0;
      while (!((s.tile.vec[b] >> bit) & 1)) ++bit;
      if (bit < 32) P.wire_tile_bit[bit] = b;
    }
  }
  P.need_l1 = l1 ? 1 : 0;
  P.need_l2 = l2 ? 1 : 0;
  // Forward register layouts (rsv_pass.cu): 0 holds tile bits 8..11 in
  // registers, 1 holds 4..7, 2 holds 0..3; layouts 0 and 1 have tile bits
  // 0..3 on the lanes and load and store directly.  (The backward kernels use
  // their own fixed layout families.)
  bool hi = false, mid = false, lo = false;
  for (int b = 0; b < 12; ++b) {
    if (s.tile.gate_wire[b] < 0) continue;
    (b >= 8 ? hi : (b >= 4 ? mid : lo)) = true;
  }
  P.nseq = 0;
  auto visit = [&](int layout, bool apply) {
    P.seq_layout[P.nseq] = layout;
    P.seq_apply[P.nseq] = apply ? 1 : 0;
    ++P.nseq;
  };
  if (!s.bwd) {
    // load in layout 1 when bits 4..7 carry gates, end in layout 0 or 1 (both
    // store whole segments): 1 (4..7) -> [2 (0..3)] -> 0 (8..11)
    if (lo) {
      visit(1, mid);
      visit(2, true);
      visit(0, hi);
    } else if (mid) {
      visit(1, true);
      if (hi) visit(0, true);
    } else {
      visit(0, hi);
    }
  } else {
    if (mid) visit(1, true);
    if (lo) visit(2, true);
    visit(0, hi);
  }
  P.psi_load = s.psi_load;
  P.lam_load = s.lam_load;
  P.psi_store = s.psi_store;
  P.lam_store = s.lam_store;
  P.phase = s.phase;
  P.phi_grad = s.phi_grad;
  P.sync_after_load = (s.tile.num_tiles == 1) ? 1 : 0;
  // Pair roles: a gated wire's bit must come from its unit direction only.
  for (int b = 0; b < 12; ++b) {
    const u64 v = s.tile.vec[b];
    if ((v & (v - 1)) == 0) continue;
    for (int g = 0; g < 12; ++g) {
      const int w = s.tile.gate_wire[g];
      if (w >= 0 && ((v >> w) & 1)) throw Error(RSV_ERR_INTERNAL, "multi-bit direction overlaps a gated wire");
    }
  }
  P.psi_in = s.psi_in >= 0 ? state_buf(B, s.psi_in) : nullptr;
  P.psi_out = s.psi_out >= 0 ? state_buf(B, s.psi_out) : nullptr;
  P.lam_in = s.lam_in >= 0 ? state_buf(B, s.lam_in) : nullptr;
  P.lam_out = s.lam_out >= 0 ? state_buf(B, s.lam_out) : nullptr;
  P.coef = B->coef.p;
  P.rot = B->rot.p;
  P.lscale = B->lscale.p;
  P.ptab = B->ptab.p + static_cast<size_t>(s.layer) * 1024;
  P.prod = B->prod.p + static_cast<size_t>(s.prod_table) * 1024;
  P.partials = s.bwd ? B->pass_partials.p + static_cast<size_t>(s.pass_index) * B->plan.max_grid *
                                                 kPartialStride
                     : nullptr;
  P.mps_btab = B->mps_btab.p;
  P.mps_wtab = B->mps_wtab.p;
}

cudaEvent_t take_event(rsv_backend *B) {
  if (!B->event_pool.empty()) {
    cudaEvent_t e = B->event_pool.back();
    B->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  check(cudaEventCreate(&e), "cudaEventCreate");
  return e;
}

// Launch `body` (`kernels` kernel launches) and, when launch timing is on,
// bracket it with events.
template <typename F>
void timed(rsv_backend *B, cudaStream_t st, int kind, double bytes, F &&body, int kernels = 1) {
  B->kernels_launched += static_cast<unsigned long long>(kernels);
  if (!B->timing) {
    body();
    return;
  }
  rsv_backend::Rec r{take_event(B), take_event(B), kind, bytes};
  check(cudaEventRecord(r.a, st), "cudaEventRecord");
  body();
  check(cudaEventRecord(r.b, st), "cudaEventRecord");
  B->recs.push_back(r);
}

// Minimum DRAM bytes of a pass: 16 B per amplitude for every buffer it must
// read (gathers and natural loads) and every buffer it must write.
double pass_bytes(const rsv_backend *B, const Step &s) {
  const double amp = 16.0 * static_cast<double>(u64{1} << B->n);
  double k = 0.0;
  if (s.psi_load == kLoadNatural || s.psi_load == kLoadGatherP) k += 1;
  if (s.psi_store != kStoreNone) k += 1;
  if (s.bwd) {
    if (s.lam_load == kLoadNatural || s.lam_load == kLoadGatherP) k += 1;
    if (s.lam_store != kStoreNone) k += 1;
  }
  return k * amp;
}

MpsParams mps_params(rsv_backend *B) {
  MpsParams Q{};
  Q.n = B->n;
  Q.bond = 1 << (B->plan.mps_k - 1);
  const int m = B->n - 12;
  Q.m1 = (m + 1) / 2;
  Q.m2 = m - Q.m1;
  Q.coef = B->coef.p;
  Q.tsite = B->mps_tsite.p;
  Q.btab = B->mps_btab.p;
  Q.coslo = B->mps_coslo.p;
  Q.coshi = B->mps_coshi.p;
  Q.mtab = B->mps_mtab.p;
  Q.wtab = B->mps_wtab.p;
  Q.zt = B->mps_zt.p;
  Q.ylo = B->mps_ylo.p;
  Q.yhi = B->mps_yhi.p;
  Q.partials = B->mps_partials.p;
  Q.gf = B->mps_gf.p;
  Q.num_tiles = u64{1} << (B->n - 12);
  return Q;
}

void run_forward(rsv_backend *B, cudaStream_t st) {
  if (B->plan.mps_k > 0 && B->plan.mps_fused) {
    const MpsParams Q = mps_params(B);
    timed(B, st, 0, 0.0, [&] { check(launch_mps_tables(Q, st), "matrix-product tables launch"); }, 2);
  } else if (B->plan.mps_k > 0) {
    const MpsParams Q = mps_params(B);
    timed(B, st, 1, 16.0 * static_cast<double>(u64{1} << B->n), [&] {
      check(launch_mps_tables(Q, st), "matrix-product tables launch");
      check(launch_mps_forward(Q, state_buf(B, B->plan.mps_out), B->plan.mps_scatter ? 1 : 0, B->plan.mps_fwd_grid, st),
            "matrix-product forward launch");
    }, 3);
  }
  PassParams P;
  for (const auto &s : B->plan.fwd) {
    fill_pass_params(B, s, P);
    timed(B, st, 1, pass_bytes(B, s),
          [&] { check(launch_pass(P, false, s.grid, st), "forward pass launch"); });
  }
}

// Whether the call's backward applies the field terms on its first pass's
// tile (then the energy kernel applies the others): energy_and_grad calls of
// a plan with such a pass.
bool fused_energy(const rsv_backend *B, bool grad) { return grad && B->energy_fuse_pass >= 0; }

void run_energy(rsv_backend *B, cudaStream_t st, bool fused) {
  const double bytes = 2.0 * 16.0 * static_cast<double>(u64{1} << B->n);
  if (fused) {
    timed(B, st, 2, bytes, [&] {
      check(launch_energy_masks(state_buf(B, B->plan.chi_buf), state_buf(B, B->plan.mu_buf), B->n, B->field,
                                u64{1} << B->n, B->energy_rest.data(), static_cast<int>(B->energy_rest.size()),
                                B->energy_partials.p, B->energy_grid, st),
            "energy launch");
    });
    return;
  }
  timed(B, st, 2, bytes, [&] {
    check(launch_energy(state_buf(B, B->plan.chi_buf), state_buf(B, B->plan.mu_buf), B->n, B->field,
                        u64{1} << B->n, B->energy_partials.p, B->energy_grid, B->sms, st),
          "energy launch");
  }, energy_kernel_count(B->n));
}

Layer0Params layer0_params(rsv_backend *B) {
  Layer0Params Q{};
  Q.n = B->n;
  Q.gather = B->plan.layer0_load == kLoadGatherP ? 1 : 0;
  Q.coef = B->coef.p;
  Q.lam = state_buf(B, B->plan.layer0_lam);
  Q.num_tiles = u64{1} << (B->n - 12);
  Q.partials = B->layer0_partials.p;
  return Q;
}

// fused: the energy kernel left the field terms of pass energy_fuse_pass to it
void run_backward(rsv_backend *B, cudaStream_t st, bool fused) {
  PassParams P;
  for (size_t i = 0; i < B->plan.bwd.size(); ++i) {
    const Step &s = B->plan.bwd[i];
    fill_pass_params(B, s, P);
    if (s.kernel == kKernelTma) {
      TmaPass T = B->tma[i];
      if (!fused || static_cast<int>(i) != B->energy_fuse_pass) T.energy_terms = 0;
      if (!fused || static_cast<int>(i) != B->energy_defer_pass) T.defer_terms = 0;
      T.efield = B->field;
      T.energy_partials = B->energy_partials.p + B->energy_grid +
                          (static_cast<int>(i) == B->energy_defer_pass ? B->energy_fuse_grid : 0);
      timed(B, st, 3, pass_bytes(B, s),
            [&] { check(launch_bwd_tma(P, T, s.grid, st), "backward TMA pass launch"); });
      continue;
    }
    timed(B, st, 3, pass_bytes(B, s),
          [&] { check(launch_pass(P, true, s.grid, st), "backward pass launch"); });
  }
  if (B->plan.layer0_kernel) {
    const Layer0Params Q = layer0_params(B);
    timed(B, st, 3, 16.0 * static_cast<double>(u64{1} << B->n),
          [&] { check(launch_layer0_grad(Q, B->plan.layer0_grid, st), "layer-0 gradient launch"); });
  }
  if (B->plan.mps_k > 0) {
    const MpsParams Q = mps_params(B);
    timed(B, st, 3, 16.0 * static_cast<double>(u64{1} << B->n), [&] {
      check(launch_mps_grad(Q, state_buf(B, B->plan.mps_lam), B->plan.mps_load == kLoadGatherP ? 1 : 0,
                            B->plan.mps_grad_grid, st),
            "matrix-product gradient launch");
    }, 3);
  }
}

void run_finalize(rsv_backend *B, bool grad, double *energy_out, double *grad_out,
                  cudaStream_t st, bool fused = false) {
  FinalizeParams F{};
  F.n = B->n;
  F.L = B->L;
  F.num_energy_partials = B->energy_grid + (fused ? B->energy_fuse_grid + B->energy_defer_grid : 0);
  F.phi_alt_layer = -1;
  if (B->energy_defer_pass >= 0) {
    F.phi_alt_layer = B->L - 1;
    F.phi_alt_pass = B->plan.bwd[static_cast<size_t>(B->energy_defer_pass)].pass_index;
    F.phi_alt_wires = B->energy_defer_wires;
  }
  F.energy_partials = B->energy_partials.p;
  F.pass_partials = B->pass_partials.p;
  F.max_grid = B->plan.max_grid;
  const int np = B->num_bwd_passes;
  const size_t nl = static_cast<size_t>(B->n) * B->L;
  F.pass_grid = B->tables.p;
  F.theta_pass = B->tables.p + np;
  F.theta_slot = B->tables.p + np + nl;
  F.phi_pass = B->tables.p + np + 2 * nl;
  F.gscale = B->gscale.p;
  F.pipeline_err = B->tma_passes > 0 ? B->pipeline_err.p : nullptr;
  F.energy_out = energy_out;
  F.grad_out = grad ? grad_out : nullptr;
  timed(B, st, 4, 0.0, [&] { check(launch_finalize(F, st), "finalize launch"); });
  if (grad && B->plan.mps_k > 0) {
    const MpsParams Q = mps_params(B);
    timed(B, st, 4, 0.0, [&] { check(launch_mps_finalize(Q, grad_out, st), "matrix-product finalize launch"); });
  }
  if (grad && B->plan.layer0_kernel) {
    const Layer0Params Q = layer0_params(B);
    timed(B, st, 4, 0.0, [&] {
      check(launch_layer0_finalize(Q, B->plan.layer0_grid, grad_out, st), "layer-0 finalize launch");
    });
  }
}

void upload_host_coefs(rsv_backend *B, const double *params, cudaStream_t st) {
  // cos/sin of the half angles on the host, exactly as the reference
  // (cpp/ising_cuda_rotation_kernels.cu:661-675).
  const size_t count = static_cast<size_t>(B->n) * B->L;
  for (size_t k = 0; k < count; ++k) {
    const double ry = params[2 * k] * 0.5, rz = params[2 * k + 1] * 0.5;
    B->coef_host.p[k] = make_double4(std::cos(ry), std::sin(ry), std::cos(rz), std::sin(rz));
  }
  check(cudaMemcpyAsync(B->coef.p, B->coef_host.p, count * sizeof(double4),
                        cudaMemcpyHostToDevice, st),
        "coefficient upload");
}

PartialMasks partial_masks(const Plan &pl) {
  PartialMasks m{};
  m.count = static_cast<int>(pl.partial_masks.size());
  if (m.count > kMaxPartialTables) throw Error(RSV_ERR_INTERNAL, "too many partial product tables");
  for (int i = 0; i < m.count; ++i) m.mask[i] = pl.partial_masks[static_cast<size_t>(i)];
  return m;
}

// Per-call tables (RZ phases, product states, tangent forms, gradient corrections).
void launch_prep(rsv_backend *B, cudaStream_t st) {
  timed(B, st, 0, 0.0, [&] {
    check(launch_tables(B->coef.p, B->n, B->L, B->ptab.p, B->prod.p, partial_masks(B->plan), st),
          "tables launch");
  });
  timed(B, st, 0, 0.0, [&] {
    check(launch_rot(B->coef.p, B->n, B->L, B->order.p, B->plan.checkpoint, B->rot.p, B->lscale.p,
                     B->gscale.p, st),
          "rot launch");
  });
  if (B->energy_defer_pass >= 0) {
    DeferPhaseArgs A = B->defer_args;
    A.coef = B->coef.p;
    A.field = B->field;
    timed(B, st, 0, 0.0, [&] { check(launch_defer_phase(A, B->defer_phase.p, st), "phase table launch"); });
  }
}

// Gate-level path: RY, RZ and CNOT as separate kernels and the inverse walk
// (the reference's inverse_walk_cuQuantum schedule without cuStateVec).
void run_gate_level(rsv_backend *B, bool grad, double *energy_out, double *grad_out, cudaStream_t st) {
  GateLevelArgs A{};
  A.n = B->n;
  A.L = B->L;
  A.field = B->field;
  A.coef = B->coef.p;
  A.psi = state_buf(B, 0);
  A.lam = state_buf(B, 1);
  A.grid = B->gate_grid;
  A.energy_partials = B->gate_partials.p;
  A.grad_partials = B->gate_partials.p + B->gate_grid;
  A.energy_out = energy_out;
  A.grad_out = grad ? grad_out : nullptr;
  check(rsv::run_gate_level(A, st), "gate-level launch");
}

void run_all(rsv_backend *B, bool grad, double *energy_out, double *grad_out, cudaStream_t st) {
  ++B->generation;
  B->forward_only_state = false;
  if (B->gate_level) {
    run_gate_level(B, grad, energy_out, grad_out, st);
    return;
  }
  if (B->dense) {
    DenseArgs D{};
    D.n = B->n;
    D.L = B->L;
    D.field = B->field;
    D.coef = B->coef.p;
    D.work = B->dense_work.p;
    D.energy_out = energy_out;
    D.grad_out = grad ? grad_out : nullptr;
    check(run_dense_scan(D, st), "dense_scan launch");
    return;
  }
  launch_prep(B, st);
  run_forward(B, st);
  const bool fused = fused_energy(B, grad);
  run_energy(B, st, fused);
  if (grad) run_backward(B, st, fused);
  run_finalize(B, grad, energy_out, grad_out, st, fused);
}

// After a synchronised call: a NaN energy from a backend with TMA passes may
// come from a pipeline wait that gave up (finalize_kernel writes NaN then);
// report it as an error and clear the flag.
void check_pipeline(rsv_backend *B, double energy) {
  if (B->tma_passes == 0 || !std::isnan(energy)) return;
  int flag = 0;
  check(cudaMemcpy(&flag, B->pipeline_err.p, sizeof(int), cudaMemcpyDeviceToHost), "pipeline flag read");
  if (flag == 0) return;
  check(cudaMemset(B->pipeline_err.p, 0, sizeof(int)), "pipeline flag clear");
  throw Error(RSV_ERR_CUDA, "a TMA backward pass gave up waiting for its pipeline (flag " +
                                std::to_string(flag) + "); the results of this call are void");
}

// Synchronous host entry points: NULL selects the backend's own stream.
cudaStream_t pick_stream(rsv_backend *B, void *stream) {
  return stream ? static_cast<cudaStream_t>(stream) : B->stream;
}

// Asynchronous device entry points: the stream is used as given, so 0 is the
// legacy default stream (the CUDA convention, and torch's default stream).
cudaStream_t device_stream(void *stream) { return static_cast<cudaStream_t>(stream); }

void validate_params(rsv_backend *B, const void *params, size_t num_params) {
  if (B == nullptr) invalid("backend is null");
  if (num_params != B->num_params) invalid("num_params does not match the circuit.");
  if (params == nullptr) invalid("params is null");
}

// A backend lives on the device that was current when it was created; every
// entry point that touches its memory or launches makes that device current
// for the call and restores the caller's device afterwards.
class OnDevice {
 public:
  explicit OnDevice(int device) {
    if (device < 0) return;
    if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != device && cudaSetDevice(device) == cudaSuccess)
      changed_ = true;
  }
  ~OnDevice() {
    if (changed_) cudaSetDevice(prev_);
  }
  OnDevice(const OnDevice &) = delete;
  OnDevice &operator=(const OnDevice &) = delete;

 private:
  int prev_ = -1;
  bool changed_ = false;
};

template <typename F>
rsv_status guarded(F &&f) {
  try {
    f();
    g_last_error.clear();
    return RSV_OK;
  } catch (const Error &e) {
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return RSV_ERR_OUT_OF_MEMORY;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return RSV_ERR_INTERNAL;
  }
}

bool configured = false;

// ------------------------------------------------------------------------
// Batched circuits: the pass plans of make_plan, flattened into the tables
// the persistent batch kernel (rsv_batch.cu) walks.
// ------------------------------------------------------------------------

BatchTile batch_tile(const Tile &t) {
  BatchTile b{};
  for (int i = 0; i < 12; ++i) {
    b.vec[i] = static_cast<unsigned int>(t.vec[i]);
    b.gate_wire[i] = t.gate_wire[i];
  }
  for (int w = 0; w < 32; ++w) b.wire_tile_bit[w] = -1;
  if (t.unit)
    for (int i = 0; i < 12; ++i) {
      int bit = 0;
      while (!((t.vec[i] >> bit) & 1)) ++bit;
      b.wire_tile_bit[bit] = i;
    }
  b.num_runs = t.num_runs;
  for (int r = 0; r < 4; ++r) {
    b.run_start[r] = t.run_start[r];
    b.run_len[r] = t.run_len[r];
  }
  b.num_tiles = static_cast<unsigned int>(t.num_tiles);
  return b;
}

BatchStep batch_step(const Step &s, int kind, int tile) {
  BatchStep b{};
  b.kind = kind;
  b.tile = tile;
  b.layer = s.layer;
  b.psi_load = s.psi_load;
  b.lam_load = s.lam_load;
  b.psi_store = s.psi_store;
  b.lam_store = s.lam_store;
  b.phase = s.phase;
  b.psi_in = s.psi_in;
  b.psi_out = s.psi_out;
  b.lam_in = s.lam_in;
  b.lam_out = s.lam_out;
  return b;
}

}  // namespace
}  // namespace rsv

struct rsv_batch {
  int device = 0, sms = 0;
  int max_qubits = 0;
  int slots = 0, active_slots = 0;
  size_t state_bytes = 0, slot_bytes = 0;
  rsv::DevBuf<unsigned char> scratch;
  // plan tables (grow as new (n, L) pairs appear; uploaded when dirty)
  std::vector<std::pair<int, int>> plan_keys;
  std::vector<rsv::BatchPlan> plans;
  std::vector<rsv::BatchStep> steps;
  std::vector<rsv::BatchTile> tiles;
  std::vector<int> undo;
  std::vector<double> plan_cost;
  bool dirty = true;
  rsv::DevBuf<rsv::BatchPlan> d_plans;
  rsv::DevBuf<rsv::BatchStep> d_steps;
  rsv::DevBuf<rsv::BatchTile> d_tiles;
  rsv::DevBuf<int> d_undo;
  // current circuits
  int count = 0;
  size_t num_params = 0;
  std::vector<rsv::BatchCircuit> circuits;
  std::vector<double> circuit_cost;
  rsv::DevBuf<rsv::BatchCircuit> d_circuits;
  rsv::DevBuf<int> d_order;
  // thread-block clusters: CTAs per cluster and the work groups for that size
  int cluster = 8;
  int num_groups = 0;
  rsv::DevBuf<rsv::BatchGroup> d_groups;
  rsv::DevBuf<int> d_counter;
  cudaStream_t stream = nullptr;
};

namespace rsv {
namespace {

int batch_plan_index(rsv_batch *Bt, int n, int L) {
  for (size_t i = 0; i < Bt->plan_keys.size(); ++i)
    if (Bt->plan_keys[i] == std::make_pair(n, L)) return static_cast<int>(i);
  const Plan pl = make_plan_full(n, L, Bt->sms, false);
  BatchPlan bp{};
  bp.first_step = static_cast<int>(Bt->steps.size());
  bp.undo_off = static_cast<int>(Bt->undo.size());
  double cost = 0.0;
  auto add = [&](const Step &s, int kind) {
    Bt->tiles.push_back(batch_tile(s.tile));
    Bt->steps.push_back(batch_step(s, kind, static_cast<int>(Bt->tiles.size()) - 1));
    cost += static_cast<double>(s.tile.num_tiles) * (kind == kBatchBackward ? 2.0 : 1.0);
  };
  for (const auto &s : pl.fwd) add(s, kBatchForward);
  BatchStep e{};
  e.kind = kBatchEnergy;
  e.tile = -1;
  e.psi_in = pl.chi_buf;
  e.psi_out = pl.mu_buf;
  e.lam_in = e.lam_out = -1;
  Bt->steps.push_back(e);
  cost += 1.0;
  for (const auto &s : pl.bwd) add(s, kBatchBackward);
  bp.num_steps = static_cast<int>(Bt->steps.size()) - bp.first_step;
  for (int w : undo_order(pl)) Bt->undo.push_back(w);
  Bt->plans.push_back(bp);
  Bt->plan_keys.emplace_back(n, L);
  Bt->plan_cost.push_back(cost);
  Bt->dirty = true;
  return static_cast<int>(Bt->plans.size()) - 1;
}

template <typename T>
void upload(DevBuf<T> &d, const std::vector<T> &h, cudaStream_t st, const char *what) {
  if (d.count < h.size()) d.alloc(h.size() + h.size() / 2 + 1);
  if (!h.empty())
    check(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st), what);
}

// Work groups for the current cluster size: circuits sorted longest first
// (LPT; ties kept together by plan), then runs of the same plan cut into
// groups of cluster / per circuits, per = min(cluster, tiles per pass) CTAs
// each.  Uploads the order and the groups (synchronous).
void batch_group(rsv_batch *Bt) {
  const int count = Bt->count;
  std::vector<int> order(static_cast<size_t>(count));
  for (int c = 0; c < count; ++c) order[static_cast<size_t>(c)] = c;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const double ca = Bt->circuit_cost[static_cast<size_t>(a)], cb = Bt->circuit_cost[static_cast<size_t>(b)];
    if (ca != cb) return ca > cb;
    return Bt->circuits[static_cast<size_t>(a)].plan < Bt->circuits[static_cast<size_t>(b)].plan;
  });
  std::vector<BatchGroup> groups;
  for (int i = 0; i < count;) {
    const BatchCircuit &C = Bt->circuits[static_cast<size_t>(order[static_cast<size_t>(i)])];
    const int tiles = 1 << std::max(0, C.n - kTileBits);
    BatchGroup g{};
    g.first = i;
    g.per = std::min(Bt->cluster, tiles);
    const int cap = Bt->cluster / g.per;
    int k = i;
    while (k < count && k - i < cap &&
           Bt->circuits[static_cast<size_t>(order[static_cast<size_t>(k)])].plan == C.plan)
      ++k;
    g.count = k - i;
    groups.push_back(g);
    i = k;
  }
  cudaStream_t st = Bt->stream;
  upload(Bt->d_order, order, st, "batch order upload");
  upload(Bt->d_groups, groups, st, "batch group upload");
  check(cudaStreamSynchronize(st), "batch upload");
  Bt->num_groups = static_cast<int>(groups.size());
}

void batch_set_circuits(rsv_batch *Bt, int count, const int *ns, const int *Ls, const double *hs) {
  if (count < 0) invalid("count must be non-negative");
  if (count > 0 && (ns == nullptr || Ls == nullptr || hs == nullptr)) invalid("null circuit array");
  std::vector<BatchCircuit> circ(static_cast<size_t>(count));
  std::vector<double> cost(static_cast<size_t>(count));
  size_t off = 0;
  for (int c = 0; c < count; ++c) {
    const int n = ns[c], L = Ls[c];
    if (n < 2 || n > Bt->max_qubits)
      invalid("circuit " + std::to_string(c) + ": num_qubits must be in [2, " +
              std::to_string(Bt->max_qubits) + "]");
    if (L < 1 || L > kBatchMaxLayers)
      invalid("circuit " + std::to_string(c) + ": num_layers must be in [1, " +
              std::to_string(kBatchMaxLayers) + "]");
    if (!std::isfinite(hs[c])) invalid("circuit " + std::to_string(c) + ": field is not finite");
    BatchCircuit &C = circ[static_cast<size_t>(c)];
    C.n = n;
    C.L = L;
    C.h = hs[c];
    C.param_off = static_cast<long long>(off);
    C.plan = batch_plan_index(Bt, n, L);
    C.index = c;
    cost[static_cast<size_t>(c)] =
        Bt->plan_cost[static_cast<size_t>(C.plan)] * static_cast<double>(u64{1} << std::max(n, kTileBits));
    off += static_cast<size_t>(2) * n * L;
  }
  cudaStream_t st = Bt->stream;
  if (Bt->dirty) {
    upload(Bt->d_plans, Bt->plans, st, "batch plan upload");
    upload(Bt->d_steps, Bt->steps, st, "batch step upload");
    upload(Bt->d_tiles, Bt->tiles, st, "batch tile upload");
    upload(Bt->d_undo, Bt->undo, st, "batch undo upload");
    Bt->dirty = false;
  }
  upload(Bt->d_circuits, circ, st, "batch circuit upload");
  Bt->circuits = std::move(circ);
  Bt->circuit_cost = std::move(cost);
  Bt->count = count;
  Bt->num_params = off;
  batch_group(Bt);
}

void batch_run(rsv_batch *Bt, const double *d_params, double *d_energy, double *d_grad,
               cudaStream_t st) {
  if (Bt->count == 0) return;
  if (d_params == nullptr || d_energy == nullptr) invalid("null device pointer");
  BatchArgs A{};
  A.count = Bt->count;
  A.circuits = Bt->d_circuits.p;
  A.order = Bt->d_order.p;
  A.groups = Bt->d_groups.p;
  A.num_groups = Bt->num_groups;
  A.counter = Bt->d_counter.p;
  A.plans = Bt->d_plans.p;
  A.steps = Bt->d_steps.p;
  A.tiles = Bt->d_tiles.p;
  A.undo = Bt->d_undo.p;
  A.params = d_params;
  A.energy_out = d_energy;
  A.grad_out = d_grad;
  A.scratch = Bt->scratch.p;
  A.slot_bytes = Bt->slot_bytes;
  A.state_bytes = Bt->state_bytes;
  // CTAs: the active slots, rounded down to whole clusters, no more than the groups need
  const int C = Bt->cluster;
  const int grid = std::max(C, (std::min(Bt->active_slots, Bt->num_groups * C) / C) * C);
  if (grid > Bt->slots) invalid("fewer scratch slots than one thread-block cluster");
  check(cudaMemsetAsync(Bt->d_counter.p, 0, sizeof(int), st), "batch counter reset");
  check(launch_batch(A, grid, C, st), "batch launch");
}

}  // namespace
}  // namespace rsv

namespace rsv {

void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

// Energy and gradient of device parameters with every device buffer carved
// out of a caller-provided workspace (nothing is allocated on the device).
// Used by the allocation-free entry point (rsv_noalloc.cu).
rsv_status run_in_workspace(int n, int L, double field, const double *d_params, size_t num_params,
                            double *d_energy_out, double *d_gradient_out, void *workspace,
                            size_t workspace_bytes, int max_qubits, int max_layers, void *stream) {
  return guarded([&] {
    if (n < 2) invalid("num_qubits must be at least 2.");
    if (L < 1) invalid("num_layers must be at least 1.");
    if (n > max_qubits || L > max_layers)
      invalid("the allocation-free entry point supports num_qubits <= " + std::to_string(max_qubits) +
              " and num_layers <= " + std::to_string(max_layers) + " (fixed workspace)");
    if (num_params != static_cast<size_t>(2) * n * L) invalid("num_params does not match the circuit.");
    if (d_params == nullptr || d_energy_out == nullptr) invalid("null device pointer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rsv_backend B;
    B.n = n;
    B.L = L;
    B.field = field;
    B.num_params = num_params;
    check(cudaGetDevice(&B.device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&B.sms, cudaDevAttrMultiProcessorCount, B.device), "cudaDeviceGetAttribute");
    B.plan = make_plan_full(n, L, B.sms, false);
    B.num_bwd_passes = static_cast<int>(B.plan.bwd.size());
    B.state_len = size_t{1} << B.plan.phys;
    B.energy_grid = energy_grid_size(n, B.sms);
    const size_t nl = static_cast<size_t>(n) * L;
    std::vector<int> tab;
    for (const auto &s : B.plan.bwd) tab.push_back(s.grid);
    tab.insert(tab.end(), B.plan.theta_pass.begin(), B.plan.theta_pass.end());
    tab.insert(tab.end(), B.plan.theta_slot.begin(), B.plan.theta_slot.end());
    tab.insert(tab.end(), B.plan.phi_pass.begin(), B.plan.phi_pass.end());
    const std::vector<int> ord = undo_orders(B.plan);
    // carve the workspace (256-byte aligned sections)
    unsigned char *base = static_cast<unsigned char *>(workspace);
    size_t off = 0;
    auto take = [&](size_t bytes) {
      unsigned char *q = base + off;
      off += (bytes + 255) & ~size_t{255};
      return q;
    };
    unsigned char *bufs[3];
    for (auto &q : bufs) q = take(B.state_len * sizeof(double2));
    unsigned char *coef = take(nl * sizeof(double4));
    unsigned char *rot = take(nl * sizeof(double2));
    unsigned char *lscale = take(L * sizeof(double));
    unsigned char *gscale = take(2 * nl * sizeof(double));
    unsigned char *ptab = take(static_cast<size_t>(L) * 1024 * sizeof(double2));
    unsigned char *prod = take(1024 * sizeof(double2));
    unsigned char *epart = take(B.energy_grid * sizeof(double));
    const size_t npart = static_cast<size_t>(std::max(1, B.num_bwd_passes)) * B.plan.max_grid * kPartialStride;
    unsigned char *ppart = take(npart * sizeof(double));
    unsigned char *tabs = take(tab.size() * sizeof(int));
    unsigned char *ords = take(ord.size() * sizeof(int));
    unsigned char *outs = take((1 + num_params) * sizeof(double));
    if (off > workspace_bytes)
      invalid("circuit needs " + std::to_string(off) + " workspace bytes, the fixed workspace has " +
              std::to_string(workspace_bytes));
    // the three buffers were carved back to back (each a multiple of 256 bytes)
    B.states.view(reinterpret_cast<double2 *>(bufs[0]), 3 * B.state_len);
    B.coef.view(reinterpret_cast<double4 *>(coef), nl);
    B.rot.view(reinterpret_cast<double2 *>(rot), nl);
    B.lscale.view(reinterpret_cast<double *>(lscale), L);
    B.gscale.view(reinterpret_cast<double *>(gscale), 2 * nl);
    B.ptab.view(reinterpret_cast<double2 *>(ptab), static_cast<size_t>(L) * 1024);
    B.prod.view(reinterpret_cast<double2 *>(prod), 1024);
    B.energy_partials.view(reinterpret_cast<double *>(epart), B.energy_grid);
    B.pass_partials.view(reinterpret_cast<double *>(ppart), npart);
    B.tables.view(reinterpret_cast<int *>(tabs), tab.size());
    B.order.view(reinterpret_cast<int *>(ords), ord.size());
    B.outputs.view(reinterpret_cast<double *>(outs), 1 + num_params);
    // the plan tables travel in kernel parameters (no pageable host copy)
    check(launch_put_ints(tab.data(), tab.size(), B.tables.p, st), "plan table upload");
    check(launch_put_ints(ord.data(), ord.size(), B.order.p, st), "order upload");
    // The workspace keeps the previous call's contents; for n < 12 the padding
    // amplitudes of the state buffers must start at zero.
    if (B.plan.phys > n)
      check(cudaMemsetAsync(B.states.p, 0, 3 * B.state_len * sizeof(double2), st), "state clear");
    check(launch_coef(d_params, B.coef.p, static_cast<int>(nl), st), "coef launch");
    run_all(&B, d_gradient_out != nullptr, d_energy_out, d_gradient_out, st);
    // nothing enqueued above refers to host memory of this call
  });
}

// Put the eligible backward passes on the TMA-fed kernel (rsv_pass_tma.cu):
// their tensor maps are encoded here, once per plan, over the backend's own
// state buffers.  A pass whose maps the driver rejects keeps its default
// kernel.  Two CTAs per SM.
// The field terms of H' (index masks P^-1(e_w)) that lie inside the tile of
// the last layer's first backward pass go to that pass when it is a TMA phase
// pass reading the final state chi as its psi and mu as its lambda (the
// checkpoint schedule): it adds them to lambda before any of its rotations,
// so its gradient sums see the whole lambda.  The energy kernel then applies
// the diagonal and the remaining masks in one grid-stride launch.
// The field terms on the adjacent pairs of the gated tile bits 3..10 of the
// layer's second backward pass go to that pass when it is a TMA pass of that
// shape (low run 0..2): it adds them to lambda at its start from the checkpoint
// it reads, as the phased masks conj(D) X_m D (the layer's first pass undid the
// RZ phases D), and takes the phi sums of its own wires there, whose lambda is
// then complete (finalize reads those wires' phi from this pass, unscaled).
void assign_energy_deferral(rsv_backend *B) {
  if (B->plan.bwd.size() < 2 || B->energy_fuse_pass != 0) return;
  const Step &s0 = B->plan.bwd[0];
  const Step &s = B->plan.bwd[1];
  TmaPass &T = B->tma[1];
  if (s.kernel != kKernelTma || T.kind != kTmaHalf || s.phase || s.layer != B->L - 1 || !s.tile.unit) return;
  if (s.tile.dims != 11 || s.lam_load != kLoadNatural || s.psi_load != kLoadNatural) return;
  for (int b = 0; b < 3; ++b)
    if (s.tile.vec[b] != (u64{1} << b) || s.tile.gate_wire[b] >= 0) return;
  DeferPhaseArgs A{};
  A.n = B->n;
  A.layer = B->L - 1;
  unsigned wires = 0;
  for (int b = 3; b < 11; ++b) {
    const int w = s.tile.gate_wire[b];
    if (w < 0 || s.tile.vec[b] != (u64{1} << w)) return;  // gated wire w on index bit w
    if (b > 3 && w != s.tile.gate_wire[b - 1] + 1) return;  // consecutive wires
    wires |= 1u << w;
  }
  // the masks e_w + e_{w+1} of those pairs must be field terms the energy kernel has
  std::vector<unsigned long long> rest;
  int found = 0;
  for (unsigned long long m : B->energy_rest) {
    bool mine = false;
    for (int j = 0; j < kTmaNumDeferredMasks; ++j)
      if (m == (s.tile.vec[3 + j] | s.tile.vec[4 + j])) mine = true;
    if (mine) ++found;
    else rest.push_back(m);
  }
  if (found != kTmaNumDeferredMasks) return;
  for (int j = 0; j < 8; ++j) A.wires[j] = s.tile.gate_wire[3 + j];
  // pending tangent factors at this pass's start: every wire but the first pass's
  unsigned first = 0;
  for (int b = 0; b < s0.tile.dims; ++b)
    if (s0.tile.gate_wire[b] >= 0) first |= 1u << s0.tile.gate_wire[b];
  A.pending = ((B->n == 32 ? 0u : (1u << B->n)) - 1u) & ~first;
  if (static_cast<size_t>(B->energy_grid + B->energy_fuse_grid + s.grid) > B->energy_partials.count)
    throw Error(RSV_ERR_INTERNAL, "energy partials too small for the deferred field terms");
  if (B->defer_phase.p == nullptr) B->defer_phase.alloc(kTmaDeferTable);
  T.phi_only = 1;
  T.defer_terms = 1;
  T.emask_phase = B->defer_phase.p;
  B->energy_rest = rest;
  B->energy_defer_pass = 1;
  B->energy_defer_grid = s.grid;
  B->energy_defer_wires = wires;
  B->defer_args = A;
}

void assign_energy_fusion(rsv_backend *B) {
  B->energy_defer_pass = -1;
  B->energy_defer_grid = 0;
  B->energy_defer_wires = 0;
  B->energy_fuse_pass = -1;
  B->energy_fuse_grid = 0;
  B->energy_rest.clear();
  if (!(B->kernel_flags & RSV_KERNELS_FUSED_ENERGY) || B->plan.bwd.empty() || B->n < energy_split_qubits()) return;
  const Step &s = B->plan.bwd[0];
  TmaPass &T = B->tma[0];
  if (s.kernel != kKernelTma || T.kind != kTmaHalf || !s.phase || s.layer != B->L - 1 || !s.tile.unit) return;
  if (s.psi_in != B->plan.chi_buf || s.psi_load != kLoadNatural) return;
  if (s.lam_in != B->plan.mu_buf || s.lam_load != kLoadNatural) return;
  u64 span = 0;
  for (int b = 0; b < s.tile.dims; ++b) span |= s.tile.vec[b];
  std::vector<unsigned> inside;  // the masks inside the tile, in tile bits
  for (int w = 0; w < B->n; ++w) {
    const u64 m = ring_pinv(u64{1} << w, B->n);
    if ((m & ~span) != 0) {
      B->energy_rest.push_back(m);
      continue;
    }
    unsigned tm = 0;
    for (int b = 0; b < s.tile.dims; ++b)
      if (m & s.tile.vec[b]) tm |= 1u << b;
    inside.push_back(tm);
  }
  // the kernel applies the set tma_energy_mask(U, .) of one of its shapes
  std::sort(inside.begin(), inside.end());
  int shape = -1;
  for (int u = 0; u <= kTmaMaxEnergyU && shape < 0; ++u) {
    std::vector<unsigned> want;
    for (int j = 0; j < kTmaNumEnergyMasks; ++j) want.push_back(tma_energy_mask(u, j));
    std::sort(want.begin(), want.end());
    if (inside == want) shape = u;
  }
  if (shape < 0) {
    B->energy_rest.clear();
    return;
  }
  T.energy_terms = 1 + shape;
  B->energy_fuse_pass = 0;
  B->energy_fuse_grid = s.grid;
  if (static_cast<size_t>(B->energy_grid + s.grid) > B->energy_partials.count)
    throw Error(RSV_ERR_INTERNAL, "energy partials too small for the fused energy");
  assign_energy_deferral(B);
}

void assign_backward_kernels(rsv_backend *B) {
  B->tma.assign(B->plan.bwd.size(), TmaPass{});
  B->tma_passes = 0;
  if (B->pipeline_err.p == nullptr) {
    B->pipeline_err.alloc(1);
    check(cudaMemset(B->pipeline_err.p, 0, sizeof(int)), "pipeline flag clear");
  }
  PassParams P;
  for (size_t i = 0; i < B->plan.bwd.size(); ++i) {
    Step &s = B->plan.bwd[i];
    s.kernel = kKernelDefault;
    if (!(B->kernel_flags & RSV_KERNELS_TMA)) continue;
    fill_pass_params(B, s, P);
    if (!make_tma_pass(P, B->pipeline_err.p, B->tma[i], nullptr)) continue;
    s.kernel = kKernelTma;
    s.grid = static_cast<int>(std::min<u64>(s.tile.num_tiles, static_cast<u64>(bwd_tma_blocks_per_sm(B->tma[i].kind)) *
                                                                   static_cast<u64>(std::max(1, B->sms))));
    if (s.grid > B->plan.max_grid) throw Error(RSV_ERR_INTERNAL, "TMA pass grid exceeds the partial records");
    ++B->tma_passes;
  }
  assign_energy_fusion(B);
}

// (Re)plan a backend for a backward schedule and allocate what depends on the
// plan: the state buffers, the product tables, the partial records and the
// plan tables.  A failed allocation of the checkpoint schedule falls back to
// the three-buffer schedule when the mode is automatic.
void setup_plan(rsv_backend *B, int mode) {
  if (mode != RSV_BACKWARD_AUTO && mode != RSV_BACKWARD_UNCOMPUTE && mode != RSV_BACKWARD_CHECKPOINT)
    invalid("backward mode must be RSV_BACKWARD_AUTO, _UNCOMPUTE or _CHECKPOINT");
  const bool want = mode == RSV_BACKWARD_CHECKPOINT ||
                    (mode == RSV_BACKWARD_AUTO && checkpoint_fits(B->n, B->L, B->analytic_layers, B->force_c));
  B->states.release();
  Plan pl = make_plan(B->n, B->L, B->sms, want, B->analytic_layers, B->force_c);
  B->state_len = size_t{1} << pl.phys;
  try {
    B->states.alloc(static_cast<size_t>(pl.num_bufs) * B->state_len);
  } catch (const Error &e) {
    if (mode != RSV_BACKWARD_AUTO || !pl.checkpoint || e.status != RSV_ERR_OUT_OF_MEMORY) throw;
    cudaGetLastError();  // clear the allocation failure
    pl = make_plan(B->n, B->L, B->sms, false, B->analytic_layers, B->force_c);
    B->states.alloc(static_cast<size_t>(pl.num_bufs) * B->state_len);
  }
  check(cudaMemset(B->states.p, 0, B->states.count * sizeof(double2)), "state memset");
  B->plan = pl;
  B->backward_mode = mode;
  B->num_bwd_passes = static_cast<int>(B->plan.bwd.size());
  B->prod.alloc(1024 * (1 + B->plan.partial_masks.size()));
  B->layer0_partials.alloc(static_cast<size_t>(B->plan.layer0_grid) * kLayer0Stride);
  if (B->plan.mps_k > 0) {
    const size_t e = static_cast<size_t>(1) << (2 * (B->plan.mps_k - 1));  // bond^2
    const int m = B->n - 12, m1 = (m + 1) / 2, m2 = m - m1;
    B->mps_tsite.alloc(64 * e);
    B->mps_btab.alloc(1024 * e);
    B->mps_coslo.alloc((size_t{1} << m1) * e);
    B->mps_coshi.alloc((size_t{1} << m2) * e);
    B->mps_mtab.alloc(128 * e);
    B->mps_wtab.alloc((size_t{1} << std::max(0, B->n - 16)) * e);
    B->mps_zt.alloc((size_t{1} << m) * e);
    B->mps_ylo.alloc((size_t{1} << m1) * e);
    B->mps_yhi.alloc((size_t{1} << m2) * e);
    B->mps_partials.alloc(static_cast<size_t>(B->plan.mps_grad_grid) * 128 * e);
    B->mps_gf.alloc(128 * e);
  }
  B->pass_partials.alloc(static_cast<size_t>(std::max(1, B->num_bwd_passes)) * B->plan.max_grid *
                         kPartialStride);
  assign_backward_kernels(B);
  std::vector<int> tab;
  for (const auto &s : B->plan.bwd) tab.push_back(s.grid);
  tab.insert(tab.end(), B->plan.theta_pass.begin(), B->plan.theta_pass.end());
  tab.insert(tab.end(), B->plan.theta_slot.begin(), B->plan.theta_slot.end());
  tab.insert(tab.end(), B->plan.phi_pass.begin(), B->plan.phi_pass.end());
  B->tables.alloc(tab.size());
  check(cudaMemcpy(B->tables.p, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice),
        "plan table upload");
  const std::vector<int> ord = undo_orders(B->plan);
  B->order.alloc(ord.size());
  check(cudaMemcpy(B->order.p, ord.data(), ord.size() * sizeof(int), cudaMemcpyHostToDevice),
        "order upload");
  ++B->generation;  // any state kept for a deferred backward is gone
  B->forward_only_state = false;
}

// ------------------------------------------------------------------------
// Autotuner: times the plan candidates of a backend once per (device, n, L)
// and keeps the fastest.  It replaces the reference's hand-written width rules
// (cpp/ising_cuda_structured_adjoint_modes.inc:188-202,
// cpp/ising_cuda_rotation_kernels.cu:562-575) by measurements.
// ------------------------------------------------------------------------
struct TuneChoice {
  int mode = RSV_BACKWARD_AUTO, analytic = kDefaultAnalyticLayers;
  int kernels = RSV_KERNELS_TMA | RSV_KERNELS_FUSED_ENERGY, force_c = 0;
  double ms = 0.0;
};

std::mutex g_tune_mutex;
std::map<std::string, TuneChoice> g_tune_cache;

std::string tune_key(const rsv_backend *B) {
  cudaDeviceProp prop{};
  check(cudaGetDeviceProperties(&prop, B->device), "cudaGetDeviceProperties");
  return std::string(prop.name) + "/" + std::to_string(B->sms) + "/n" + std::to_string(B->n) + "/L" +
         std::to_string(B->L);
}

void apply_choice(rsv_backend *B, const TuneChoice &c) {
  B->analytic_layers = c.analytic;
  B->kernel_flags = c.kernels;
  B->force_c = c.force_c;
  setup_plan(B, c.mode);
}

std::string choice_str(const rsv_backend *B, const TuneChoice &c) {
  std::ostringstream os;
  os << "mode=" << (B->plan.checkpoint ? "checkpoint" : "uncompute") << " analytic_layers=" << c.analytic
     << " tma=" << ((c.kernels & RSV_KERNELS_TMA) ? 1 : 0) << " tma_passes=" << B->tma_passes
     << " fused_energy=" << (B->energy_fuse_pass >= 0 ? 1 : 0)
     << " high_tile_c=" << (c.force_c ? std::to_string(c.force_c) : std::string("planner"));
  return os.str();
}

// Mean milliseconds of one energy_and_grad of the current plan (one untimed call first).
double time_plan(rsv_backend *B, const double *d_params, int repeats, cudaStream_t st) {
  const int nl = B->n * B->L;
  check(launch_coef(d_params, B->coef.p, nl, st), "coef launch");
  run_all(B, true, B->outputs.p, B->outputs.p + 1, st);
  cudaEvent_t a, b;
  check(cudaEventCreate(&a), "cudaEventCreate");
  check(cudaEventCreate(&b), "cudaEventCreate");
  check(cudaEventRecord(a, st), "cudaEventRecord");
  for (int r = 0; r < repeats; ++r) {
    check(launch_coef(d_params, B->coef.p, nl, st), "coef launch");
    run_all(B, true, B->outputs.p, B->outputs.p + 1, st);
  }
  check(cudaEventRecord(b, st), "cudaEventRecord");
  check(cudaEventSynchronize(b), "autotune synchronize");
  float ms = 0.f;
  check(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return static_cast<double>(ms) / repeats;
}

// The candidates: both backward schedules (checkpoint only where it fits),
// three or two analytic leading layers, the TMA kernels on (with or without
// the fused energy) or off, and every
// contiguous run length c of the high tiles that gives the fewest passes.
std::vector<TuneChoice> tune_candidates(const rsv_backend *B) {
  std::vector<TuneChoice> out;
  std::vector<int> cs = {0};
  if (B->n > 12) {
    auto passes = [&](int c) { return static_cast<int>(high_tiles(B->n, 12, 2, c).size()); };
    const int best = passes(0);
    for (int c = 2; c <= 10; ++c)
      if (c <= 12 && passes(c) == best) cs.push_back(c);
  }
  std::vector<int> analytic = {B->analytic_layers};
  if (B->n >= 13 && B->L >= 2) analytic = {3, 2};
  for (int an : analytic)
    for (int c : cs)
      for (int mode : {RSV_BACKWARD_CHECKPOINT, RSV_BACKWARD_UNCOMPUTE})
        for (int k : {RSV_KERNELS_TMA | RSV_KERNELS_FUSED_ENERGY, RSV_KERNELS_TMA, 0}) {
          if (mode == RSV_BACKWARD_CHECKPOINT && !checkpoint_fits(B->n, B->L, an, c)) continue;
          TuneChoice t;
          t.mode = mode;
          t.analytic = an;
          t.kernels = k;
          t.force_c = c;
          out.push_back(t);
        }
  return out;
}

Plan plan_for_mode(int n, int L, int mode) {
  if (mode == RSV_BACKWARD_AUTO)
    return make_plan(n, L, 148, checkpoint_fits(n, L, kDefaultAnalyticLayers), kDefaultAnalyticLayers);
  if (mode == RSV_BACKWARD_UNCOMPUTE) return make_plan(n, L, 148, false, kDefaultAnalyticLayers);
  if (mode == RSV_BACKWARD_CHECKPOINT) return make_plan(n, L, 148, true, kDefaultAnalyticLayers);
  invalid("backward mode must be RSV_BACKWARD_AUTO, _UNCOMPUTE or _CHECKPOINT");
}

}  // namespace rsv

using namespace rsv;

extern "C" {

const char *rsv_version(void) { return "rsv 0.1 (sm_100a)"; }

const char *rsv_last_error(void) { return g_last_error.c_str(); }

int rsv_num_stages(void) { return kNumStages; }

const char *rsv_stage_name(int i) { return (i >= 0 && i < kNumStages) ? kStageNames[i] : ""; }

unsigned long long rsv_ring_map(unsigned long long index, int num_qubits, int inverse) {
  if (num_qubits < 2 || num_qubits > kMaxQubits) return 0;
  return inverse ? ring_pinv(index, num_qubits) : ring_p(index, num_qubits);
}

rsv_status rsv_describe_plan(int num_qubits, int num_layers, char *buf, size_t buf_size,
                             size_t *length_out) {
  return rsv_describe_plan_mode(num_qubits, num_layers, RSV_BACKWARD_AUTO, buf, buf_size, length_out);
}

rsv_status rsv_describe_plan_mode(int num_qubits, int num_layers, int backward_mode, char *buf,
                                  size_t buf_size, size_t *length_out) {
  return guarded([&] {
    if (num_qubits < 2 || num_qubits > kMaxQubits) invalid("num_qubits out of range");
    if (num_layers < 1) invalid("num_layers must be at least 1");
    const Plan pl = plan_for_mode(num_qubits, num_layers, backward_mode);
    const std::string s = describe(pl);
    if (length_out) *length_out = s.size();
    if (buf && buf_size) {
      const size_t k = std::min(buf_size - 1, s.size());
      std::memcpy(buf, s.data(), k);
      buf[k] = '\0';
    }
  });
}

rsv_status rsv_create(int num_qubits, int num_layers, double field, const char *gradient_strategy,
                      int structured_rotation_chunk_width, int double_buffer, rsv_backend **out) {
  return guarded([&] {
    if (out == nullptr) invalid("out is null");
    *out = nullptr;
    const std::string strat = gradient_strategy ? gradient_strategy : "structured_adjoint";
    if (strat != "structured_adjoint" && strat != "inverse_walk_cuQuantum" &&
        strat != "inverse_walk_cuquantum" && strat != "dense_scan")
      invalid(
          "Unknown gradient strategy. Expected one of: inverse_walk_cuQuantum, "
          "structured_adjoint, dense_scan.");
    if (num_qubits < 2) invalid("num_qubits must be at least 2.");
    if (num_qubits > kMaxQubits)
      invalid("num_qubits exceeds the supported maximum of 31 (three state buffers must fit one GPU).");
    if (num_layers < 1) invalid("num_layers must be at least 1.");
    if (structured_rotation_chunk_width < 1)
      invalid("structured_rotation_chunk_width must be at least 1.");
    if (structured_rotation_chunk_width > 8)
      invalid("structured_rotation_chunk_width exceeds supported maximum.");
    if (strat == "dense_scan" && num_qubits > 8) invalid("dense_scan requires num_qubits <= 8.");
    (void)double_buffer;

    auto B = std::make_unique<rsv_backend>();
    B->n = num_qubits;
    B->L = num_layers;
    B->field = field;
    B->num_params = static_cast<size_t>(2) * num_qubits * num_layers;
    check(cudaGetDevice(&B->device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, B->device),
          "cudaDeviceGetAttribute");
    if (!configured) {
      check(configure_pass_kernels(), "configure pass kernels");
      configured = true;
    }
    // energy partials before the plan: a fused energy adds a pass's share
    B->energy_grid = energy_grid_size(num_qubits, B->sms);
    B->energy_partials.alloc(static_cast<size_t>(B->energy_grid) + 4 * static_cast<size_t>(std::max(1, B->sms)));
    setup_plan(B.get(), RSV_BACKWARD_AUTO);
    const size_t nl = static_cast<size_t>(num_qubits) * num_layers;
    if (strat == "dense_scan") {
      B->dense = true;
      B->dense_work.alloc(dense_workspace_bytes(num_qubits, num_layers) / sizeof(double2));
    }
    if (strat == "inverse_walk_cuQuantum" || strat == "inverse_walk_cuquantum") {
      B->gate_level = true;
      B->gate_grid = gate_grid(num_qubits, B->sms);
      B->gate_partials.alloc(static_cast<size_t>(B->gate_grid) * (1 + 2 * nl));
    }
    B->coef.alloc(nl);
    B->ptab.alloc(static_cast<size_t>(num_layers) * 1024);
    B->outputs.alloc(1 + B->num_params);
    B->rot.alloc(nl);
    B->lscale.alloc(num_layers);
    B->gscale.alloc(2 * nl);
    B->coef_host.alloc(nl);
    B->out_host.alloc(1 + B->num_params);
    check(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    *out = B.release();
  });
}

rsv_status rsv_destroy(rsv_backend *backend) {
  return guarded([&] {
    const OnDevice on_device(backend ? backend->device : -1);
    if (backend == nullptr) return;
    cudaStreamSynchronize(backend->stream);
    for (auto &r : backend->recs) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : backend->event_pool) cudaEventDestroy(e);
    cudaStreamDestroy(backend->stream);
    delete backend;
  });
}

rsv_status rsv_energy_and_grad(rsv_backend *B, const double *params, size_t num_params,
                               int compute_gradient, double *energy_out, double *gradient_out,
                               void *stream) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    validate_params(B, params, num_params);
    if (energy_out == nullptr) invalid("energy_out is null");
    if (compute_gradient && gradient_out == nullptr) invalid("gradient_out is null");
    cudaStream_t st = pick_stream(B, stream);
    upload_host_coefs(B, params, st);
    const bool grad = compute_gradient != 0;
    run_all(B, grad, B->outputs.p, B->outputs.p + 1, st);
    const size_t count = grad ? 1 + B->num_params : 1;
    check(cudaMemcpyAsync(B->out_host.p, B->outputs.p, count * sizeof(double),
                          cudaMemcpyDeviceToHost, st),
          "result download");
    check(cudaStreamSynchronize(st), "energy_and_grad");
    check_pipeline(B, B->out_host.p[0]);
    *energy_out = B->out_host.p[0];
    if (grad) std::memcpy(gradient_out, B->out_host.p + 1, B->num_params * sizeof(double));
  });
}

rsv_status rsv_energy_and_grad_device(rsv_backend *B, const double *d_params, size_t num_params,
                                      double *d_energy_out, double *d_gradient_out, void *stream) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    validate_params(B, d_params, num_params);
    if (d_energy_out == nullptr) invalid("d_energy_out is null");
    cudaStream_t st = device_stream(stream);
    timed(B, st, 0, 0.0, [&] {
      check(launch_coef(d_params, B->coef.p, static_cast<int>(B->n * B->L), st), "coef launch");
    });
    run_all(B, d_gradient_out != nullptr, d_energy_out, d_gradient_out, st);
  });
}

rsv_status rsv_forward_device(rsv_backend *B, const double *d_params, size_t num_params,
                              double *d_energy_out, unsigned long long *generation_out,
                              void *stream) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    validate_params(B, d_params, num_params);
    if (d_energy_out == nullptr) invalid("d_energy_out is null");
    cudaStream_t st = device_stream(stream);
    check(launch_coef(d_params, B->coef.p, static_cast<int>(B->n * B->L), st), "coef launch");
    run_all(B, false, d_energy_out, nullptr, st);
    B->forward_only_state = true;
    if (generation_out) *generation_out = B->generation;
  });
}

rsv_status rsv_backward_device(rsv_backend *B, unsigned long long generation,
                               double *d_gradient_out, void *stream) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    if (B == nullptr) invalid("backend is null");
    if (d_gradient_out == nullptr) invalid("d_gradient_out is null");
    if (!B->forward_only_state || generation != B->generation)
      throw Error(RSV_ERR_STALE_STATE,
                  "backward needs the state of the matching forward; the backend ran another call since");
    cudaStream_t st = device_stream(stream);
    run_backward(B, st, false);  // the forward call computed the whole energy
    // energy is rewritten with the same value into the outputs scratch slot
    run_finalize(B, true, B->outputs.p, d_gradient_out, st);
    B->forward_only_state = false;
    ++B->generation;
  });
}

rsv_status rsv_profile_energy_and_grad(rsv_backend *B, const double *params, size_t num_params,
                                       int compute_gradient, double *energy_out,
                                       double *gradient_out, double *stage_ms_out) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    validate_params(B, params, num_params);
    if (energy_out == nullptr || stage_ms_out == nullptr) invalid("output pointer is null");
    if (compute_gradient && gradient_out == nullptr) invalid("gradient_out is null");
    cudaStream_t st = B->stream;
    cudaEvent_t ev[8];
    for (auto &e : ev) check(cudaEventCreate(&e), "cudaEventCreate");
    const bool grad = compute_gradient != 0;
    for (int i = 0; i < kNumStages; ++i) stage_ms_out[i] = 0.0;
    check(cudaStreamSynchronize(st), "profile pre-sync");
    const auto t0 = std::chrono::steady_clock::now();
    upload_host_coefs(B, params, st);
    const auto t1 = std::chrono::steady_clock::now();
    stage_ms_out[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    ++B->generation;
    B->forward_only_state = false;
    cudaEventRecord(ev[0], st);
    if (B->gate_level || B->dense) {
      // one stage: these schedules are not split into the phases below
      cudaEventRecord(ev[1], st);
      --B->generation;  // run_all counts the call
      run_all(B, grad, B->outputs.p, B->outputs.p + 1, st);
      cudaEventRecord(ev[2], st);
      cudaEventRecord(ev[3], st);
      cudaEventRecord(ev[4], st);
    } else {
      launch_prep(B, st);
      cudaEventRecord(ev[1], st);
      run_forward(B, st);
      cudaEventRecord(ev[2], st);
      const bool fused = fused_energy(B, grad);
      run_energy(B, st, fused);
      cudaEventRecord(ev[3], st);
      if (grad) run_backward(B, st, fused);
      cudaEventRecord(ev[4], st);
      run_finalize(B, grad, B->outputs.p, B->outputs.p + 1, st, fused);
    }
    const size_t count = grad ? 1 + B->num_params : 1;
    check(cudaMemcpyAsync(B->out_host.p, B->outputs.p, count * sizeof(double),
                          cudaMemcpyDeviceToHost, st),
          "result download");
    cudaEventRecord(ev[5], st);
    check(cudaStreamSynchronize(st), "profile");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    stage_ms_out[1] = ms;
    cudaEventElapsedTime(&ms, ev[1], ev[2]);
    stage_ms_out[2] = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    stage_ms_out[3] = ms;
    cudaEventElapsedTime(&ms, ev[3], ev[4]);
    stage_ms_out[6] = ms;
    cudaEventElapsedTime(&ms, ev[4], ev[5]);
    stage_ms_out[7] = ms;
    for (auto &e : ev) cudaEventDestroy(e);
    *energy_out = B->out_host.p[0];
    if (grad) std::memcpy(gradient_out, B->out_host.p + 1, B->num_params * sizeof(double));
  });
}

rsv_status rsv_benchmark_forward_graph(rsv_backend *B, const double *params, size_t num_params,
                                       size_t repeats, double *normal_ms_out,
                                       double *graph_ms_out) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    validate_params(B, params, num_params);
    if (repeats == 0) invalid("repeats must be at least 1.");
    if (normal_ms_out == nullptr || graph_ms_out == nullptr) invalid("output pointer is null");
    cudaStream_t st = B->stream;
    ++B->generation;
    B->forward_only_state = false;
    upload_host_coefs(B, params, st);
    auto forward = [&] {
      launch_prep(B, st);
      run_forward(B, st);
    };
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "cudaEventCreate");
    check(cudaEventCreate(&b), "cudaEventCreate");
    forward();
    check(cudaStreamSynchronize(st), "warmup");
    auto time_ms = [&](auto &&body) {
      cudaEventRecord(a, st);
      for (size_t r = 0; r < repeats; ++r) body();
      cudaEventRecord(b, st);
      check(cudaEventSynchronize(b), "cudaEventSynchronize");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      return static_cast<double>(ms) / static_cast<double>(repeats);
    };
    *normal_ms_out = time_ms(forward);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    forward();
    check(cudaStreamEndCapture(st, &graph), "end capture");
    check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    check(cudaGraphLaunch(exec, st), "graph warmup");
    check(cudaStreamSynchronize(st), "graph warmup sync");
    *graph_ms_out = time_ms([&] { check(cudaGraphLaunch(exec, st), "graph launch"); });
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

rsv_status rsv_set_launch_timing(rsv_backend *B, int enable) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    B->timing = enable != 0;
  });
}

rsv_status rsv_kernel_launches(rsv_backend *B, unsigned long long *count_out) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    if (count_out == nullptr) invalid("output pointer is null");
    *count_out = B->kernels_launched;
  });
}

rsv_status rsv_launch_stats(rsv_backend *B, int *counts, double *total_ms, double *total_bytes) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    if (counts == nullptr || total_ms == nullptr || total_bytes == nullptr)
      invalid("output pointer is null");
    for (int k = 0; k < RSV_NUM_KINDS; ++k) {
      counts[k] = 0;
      total_ms[k] = 0.0;
      total_bytes[k] = 0.0;
    }
    for (auto &r : B->recs) {
      check(cudaEventSynchronize(r.b), "cudaEventSynchronize");
      float ms = 0.f;
      check(cudaEventElapsedTime(&ms, r.a, r.b), "cudaEventElapsedTime");
      counts[r.kind] += 1;
      total_ms[r.kind] += ms;
      total_bytes[r.kind] += r.bytes;
      B->event_pool.push_back(r.a);
      B->event_pool.push_back(r.b);
    }
    B->recs.clear();
  });
}

rsv_status rsv_set_backward_mode(rsv_backend *B, int mode) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    if (B == nullptr) invalid("backend is null");
    check(cudaStreamSynchronize(B->stream), "backend synchronize");
    setup_plan(B, mode);
  });
}

rsv_status rsv_set_analytic_layers(rsv_backend *B, int max_layers) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    if (B == nullptr) invalid("backend is null");
    if (max_layers < 0 || max_layers > 3) invalid("max_layers must be in [0, 3]");
    check(cudaStreamSynchronize(B->stream), "backend synchronize");
    B->analytic_layers = max_layers;
    setup_plan(B, B->backward_mode);
  });
}

rsv_status rsv_set_kernels(rsv_backend *B, int flags) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    if (B == nullptr) invalid("backend is null");
    if ((flags & ~(RSV_KERNELS_TMA | RSV_KERNELS_FUSED_ENERGY)) != 0) invalid("unknown kernel flags");
    check(cudaStreamSynchronize(B->stream), "backend synchronize");
    B->kernel_flags = flags;
    setup_plan(B, B->backward_mode);
  });
}

rsv_status rsv_kernels(rsv_backend *B, int *flags_out, int *tma_passes_out) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    if (flags_out) *flags_out = B->kernel_flags;
    if (tma_passes_out) *tma_passes_out = B->tma_passes;
  });
}

rsv_status rsv_autotune(rsv_backend *B, const double *d_params, size_t num_params, int repeats, int flags,
                        void *stream) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    validate_params(B, d_params, num_params);
    if (repeats < 1 || repeats > 1000) invalid("repeats must be in [1, 1000]");
    if ((flags & ~RSV_AUTOTUNE_FORCE) != 0) invalid("unknown autotune flags");
    if (B->gate_level || B->dense) invalid("the autotuner plans the structured_adjoint strategy only");
    cudaStream_t st = device_stream(stream);
    check(cudaStreamSynchronize(B->stream), "backend synchronize");
    const std::string key = tune_key(B);
    {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end() && !(flags & RSV_AUTOTUNE_FORCE)) {
        apply_choice(B, it->second);
        B->tune_report = "cached " + key + ": " + choice_str(B, it->second) + " " +
                         std::to_string(it->second.ms) + " ms\n";
        return;
      }
    }
    std::ostringstream rep;
    const TuneChoice before{B->backward_mode, B->analytic_layers, B->kernel_flags, B->force_c, 0.0};
    TuneChoice best;
    best.ms = 1e300;
    std::vector<std::string> seen;
    // every candidate computes the same energy and gradient: the largest
    // deviation from the first candidate's outputs is reported
    std::vector<double> ref_out, cur_out(1 + B->num_params);
    double spread = 0.0;
    for (TuneChoice c : tune_candidates(B)) {
      try {
        apply_choice(B, c);
      } catch (const Error &e) {
        if (e.status != RSV_ERR_OUT_OF_MEMORY) throw;
        cudaGetLastError();
        rep << "skipped (out of memory): " << choice_str(B, c) << "\n";
        continue;
      }
      // the same launches under another name are timed once
      std::string sig = describe(B->plan) + " fused_energy=" + std::to_string(B->energy_fuse_pass) +
                        std::to_string(B->energy_defer_pass);
      if (std::find(seen.begin(), seen.end(), sig) != seen.end()) continue;
      seen.push_back(sig);
      c.ms = time_plan(B, d_params, repeats, st);
      check(cudaMemcpy(cur_out.data(), B->outputs.p, cur_out.size() * sizeof(double), cudaMemcpyDeviceToHost),
            "autotune result read");
      if (ref_out.empty()) {
        ref_out = cur_out;
      } else {
        for (size_t k = 0; k < cur_out.size(); ++k) spread = std::max(spread, std::fabs(cur_out[k] - ref_out[k]));
      }
      rep << "candidate " << choice_str(B, c) << ": " << c.ms << " ms\n";
      if (c.ms < best.ms) best = c;
    }
    if (best.ms >= 1e300) {
      apply_choice(B, before);
      throw Error(RSV_ERR_INTERNAL, "no autotune candidate could be planned");
    }
    apply_choice(B, best);
    rep << "largest difference between candidates (energy, gradient): " << spread << "\n";
    rep << "chosen " << choice_str(B, best) << ": " << best.ms << " ms\n";
    B->tune_report = rep.str();
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = best;
  });
}

rsv_status rsv_describe_backend(rsv_backend *B, char *buf, size_t buf_size, size_t *length_out) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    std::ostringstream os;
    os << "analytic_layers=" << B->analytic_layers << " kernels=" << B->kernel_flags
       << " high_tile_c=" << (B->force_c ? std::to_string(B->force_c) : std::string("planner"))
       << " tma_passes=" << B->tma_passes;
    if (B->energy_fuse_pass >= 0)
      os << " fused_energy: backward pass " << B->energy_fuse_pass << " applies "
         << kTmaNumEnergyMasks << " field terms,"
         << (B->energy_defer_pass >= 0 ? " backward pass 1 applies " + std::to_string(kTmaNumDeferredMasks) + "," : "")
         << " the energy kernel " << B->energy_rest.size();
    os << "\n" << describe(B->plan);
    if (!B->tune_report.empty()) os << "autotune:\n" << B->tune_report;
    const std::string s = os.str();
    if (length_out) *length_out = s.size();
    if (buf && buf_size) {
      const size_t k = std::min(buf_size - 1, s.size());
      std::memcpy(buf, s.data(), k);
      buf[k] = '\0';
    }
  });
}

rsv_status rsv_analytic_layers(rsv_backend *B, int *max_layers_out, int *used_out) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    if (max_layers_out) *max_layers_out = B->analytic_layers;
    if (used_out) *used_out = B->plan.mps_k > 0 ? B->plan.mps_k : (B->plan.layer0_kernel ? 1 : 0);
  });
}

rsv_status rsv_backward_mode(rsv_backend *B, int *mode_out, int *checkpoint_out, int *num_buffers_out) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    if (mode_out) *mode_out = B->backward_mode;
    if (checkpoint_out) *checkpoint_out = B->plan.checkpoint ? 1 : 0;
    if (num_buffers_out) *num_buffers_out = B->plan.num_bufs;
  });
}

rsv_status rsv_zgemm_batched(const void *d_a, const void *d_b, void *d_c, int dim, int batch, void *stream) {
  return guarded([&] {
    if (dim < 1 || dim > 4096 || batch < 1) invalid("dim must be in [1, 4096] and batch positive");
    if (dim >= 32 && dim % 32 != 0) invalid("dim >= 32 must be a multiple of 32");
    if (!d_a || !d_b || !d_c) invalid("null device pointer");
    const long long mat = static_cast<long long>(dim) * dim;
    check(zgemm_batched(static_cast<const double2 *>(d_a), static_cast<const double2 *>(d_b),
                        static_cast<double2 *>(d_c), dim, batch, mat, mat, mat, static_cast<cudaStream_t>(stream)),
          "zgemm launch");
  });
}

rsv_status rsv_set_field(rsv_backend *B, double field) {
  return guarded([&] {
    const OnDevice on_device(B ? B->device : -1);
    if (B == nullptr) invalid("backend is null");
    if (!std::isfinite(field)) invalid("field is not finite");
    B->field = field;
  });
}

rsv_status rsv_backend_info(rsv_backend *B, int *num_qubits, int *num_layers, size_t *num_params,
                            size_t *device_bytes) {
  return guarded([&] {
    if (B == nullptr) invalid("backend is null");
    if (num_qubits) *num_qubits = B->n;
    if (num_layers) *num_layers = B->L;
    if (num_params) *num_params = B->num_params;
    if (device_bytes)
      *device_bytes = B->states.count * sizeof(double2) + B->pass_partials.count * sizeof(double) +
                      B->energy_partials.count * sizeof(double);
  });
}

rsv_status rsv_batch_create(int max_qubits, int slots, rsv_batch **out) {
  return guarded([&] {
    if (out == nullptr) invalid("out is null");
    *out = nullptr;
    if (max_qubits < 2 || max_qubits > kBatchMaxQubits)
      invalid("max_qubits must be in [2, " + std::to_string(kBatchMaxQubits) + "]");
    if (slots < 0) invalid("slots must be non-negative");
    auto Bt = std::make_unique<rsv_batch>();
    check(cudaGetDevice(&Bt->device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&Bt->sms, cudaDevAttrMultiProcessorCount, Bt->device),
          "cudaDeviceGetAttribute");
    check(configure_batch_kernel(), "configure batch kernel");
    Bt->max_qubits = max_qubits;
    Bt->slots = slots > 0 ? slots : Bt->sms;
    Bt->active_slots = Bt->slots;
    // the largest cluster (8, 4, 2, 1) that the slots and the device hold
    Bt->cluster = 8;
    while (Bt->cluster > 1 && (Bt->cluster > Bt->slots || batch_max_active_clusters(Bt->cluster) < 1))
      Bt->cluster /= 2;
    Bt->state_bytes = sizeof(double2) << std::max(max_qubits, kTileBits);
    Bt->slot_bytes = (3 * Bt->state_bytes + batch_slot_table_bytes() + 255) & ~size_t{255};
    Bt->scratch.alloc(Bt->slot_bytes * static_cast<size_t>(Bt->slots));
    Bt->d_counter.alloc(1);
    check(cudaStreamCreateWithFlags(&Bt->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    *out = Bt.release();
  });
}

rsv_status rsv_batch_destroy(rsv_batch *batch) {
  return guarded([&] {
    const OnDevice on_device(batch ? batch->device : -1);
    if (batch == nullptr) return;
    cudaStreamSynchronize(batch->stream);
    cudaStreamDestroy(batch->stream);
    delete batch;
  });
}

rsv_status rsv_batch_set_circuits(rsv_batch *batch, int count, const int *num_qubits,
                                  const int *num_layers, const double *fields) {
  return guarded([&] {
    const OnDevice on_device(batch ? batch->device : -1);
    if (batch == nullptr) invalid("batch is null");
    batch_set_circuits(batch, count, num_qubits, num_layers, fields);
  });
}

rsv_status rsv_batch_info(rsv_batch *batch, int *count, size_t *num_params, int *slots,
                          size_t *device_bytes) {
  return guarded([&] {
    if (batch == nullptr) invalid("batch is null");
    if (count) *count = batch->count;
    if (num_params) *num_params = batch->num_params;
    if (slots) *slots = batch->active_slots;
    if (device_bytes) *device_bytes = batch->slot_bytes * static_cast<size_t>(batch->slots);
  });
}

rsv_status rsv_batch_set_active_slots(rsv_batch *batch, int slots) {
  return guarded([&] {
    const OnDevice on_device(batch ? batch->device : -1);
    if (batch == nullptr) invalid("batch is null");
    if (slots < 1 || slots > batch->slots)
      invalid("slots must be in [1, " + std::to_string(batch->slots) + "]");
    batch->active_slots = slots;
  });
}

rsv_status rsv_batch_set_cluster(rsv_batch *batch, int cluster) {
  return guarded([&] {
    const OnDevice on_device(batch ? batch->device : -1);
    if (batch == nullptr) invalid("batch is null");
    if (cluster != 1 && cluster != 2 && cluster != 4 && cluster != 8) invalid("cluster must be 1, 2, 4 or 8");
    if (cluster > batch->slots) invalid("cluster exceeds the scratch slots");
    if (batch_max_active_clusters(cluster) < 1) invalid("no cluster of this size fits on the device");
    check(cudaStreamSynchronize(batch->stream), "batch synchronize");
    batch->cluster = cluster;
    batch_group(batch);
  });
}

rsv_status rsv_batch_cluster(rsv_batch *batch, int *cluster_out, int *groups_out, int *max_active_clusters_out) {
  return guarded([&] {
    if (batch == nullptr) invalid("batch is null");
    if (cluster_out) *cluster_out = batch->cluster;
    if (groups_out) *groups_out = batch->num_groups;
    if (max_active_clusters_out) *max_active_clusters_out = batch_max_active_clusters(batch->cluster);
  });
}

rsv_status rsv_batch_run_device(rsv_batch *batch, const double *d_params, double *d_energy_out,
                                double *d_gradient_out, void *stream) {
  return guarded([&] {
    const OnDevice on_device(batch ? batch->device : -1);
    if (batch == nullptr) invalid("batch is null");
    batch_run(batch, d_params, d_energy_out, d_gradient_out, static_cast<cudaStream_t>(stream));
  });
}

rsv_status rsv_batch_energy_and_grad(rsv_batch *batch, int count, const int *num_qubits,
                                     const int *num_layers, const double *fields,
                                     const double *params, size_t num_params,
                                     double *energy_out, double *gradient_out, void *stream) {
  return guarded([&] {
    const OnDevice on_device(batch ? batch->device : -1);
    if (batch == nullptr) invalid("batch is null");
    batch_set_circuits(batch, count, num_qubits, num_layers, fields);
    if (num_params != batch->num_params)
      invalid("num_params does not match the circuits (" + std::to_string(batch->num_params) +
              " expected)");
    if (count == 0) return;
    if (params == nullptr || energy_out == nullptr) invalid("null host pointer");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : batch->stream;
    DevBuf<double> d_params, d_out;
    d_params.alloc(num_params);
    d_out.alloc(static_cast<size_t>(count) + (gradient_out ? num_params : 0));
    check(cudaMemcpyAsync(d_params.p, params, num_params * sizeof(double), cudaMemcpyHostToDevice, st),
          "params upload");
    batch_run(batch, d_params.p, d_out.p, gradient_out ? d_out.p + count : nullptr, st);
    check(cudaMemcpyAsync(energy_out, d_out.p, static_cast<size_t>(count) * sizeof(double),
                          cudaMemcpyDeviceToHost, st),
          "energy download");
    if (gradient_out)
      check(cudaMemcpyAsync(gradient_out, d_out.p + count, num_params * sizeof(double),
                            cudaMemcpyDeviceToHost, st),
            "gradient download");
    check(cudaStreamSynchronize(st), "batch synchronize");
  });
}

}  // extern "C"
