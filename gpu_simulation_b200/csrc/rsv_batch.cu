// Batched energy and gradient of many independent ring-Ising circuits in one
// persistent kernel launch (uneven qubit counts and depths).
//
// The reference has no batched mode (it is only proposed in its design
// notes); this kernel runs thousands of circuits per launch:
//   * the CTAs (512 threads each) form thread-block clusters of 1, 2, 4 or 8;
//     a cluster takes a group of circuits of the same (n, L) from an atomic
//     work counter over a list sorted by decreasing cost, and spreads each
//     circuit over per = min(cluster size, tiles per pass) of its CTAs: every
//     pass's tiles are split between them, a cluster barrier separates the
//     passes, and the per-CTA energy and gradient sums are added in fixed
//     order through distributed shared memory (DSMEM) -- so a 16-qubit
//     circuit runs on 8 SMs at once and only a few large circuits are in
//     flight, whose states then stay in L2;
//   * every circuit runs the same pass plan the single-circuit engine uses for
//     its (n, L) (built on the host, uploaded once), tile by tile on the
//     scratch slot of its first CTA;
//   * a tile is 4096 amplitudes, 8 per thread, in the layout families of the
//     backward pass kernel (rsv_tile.cuh); the next tile of the same pass is
//     prefetched with cp.async;
//   * the circuit's coefficient, tangent-form and RZ-phase tables are built
//     by the CTA itself; gradient sums are reduced on chip and written once
//     per circuit, so no cross-CTA reduction is needed and results are
//     deterministic.
#include <cooperative_groups.h>

#include "rsv_batch.h"

// the per-circuit tables are written by this kernel, in the slot it reuses
#define RSV_TABLES_WRITTEN_IN_KERNEL 1
#include "rsv_tile.cuh"

namespace rsv {
namespace {

using namespace bw;

constexpr int kBatchThreads = bw::kT;

// Forward rotation of the three register bits of layout LY: RY / f in
// tangent form (mode +1: [[1,-k],[k,1]], mode -1: [[k,-1],[1,k]]).
template <int LY>
__device__ __forceinline__ void fgates(const PassParams &P, const double2 *km_tb, double2 (&a)[kR]) {
  constexpr int RB = rbit<LY>();
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int w = P.gate_wire[RB + j];
    if (w < 0) continue;
    const double2 km = km_tb[RB + j];
    const double k = km.x;
    if (km.y > 0.0) {
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const double2 x0 = a[r], x1 = a[r1];
        a[r] = make_double2(fma(-k, x1.x, x0.x), fma(-k, x1.y, x0.y));
        a[r1] = make_double2(fma(k, x0.x, x1.x), fma(k, x0.y, x1.y));
      }
    } else {
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        if (r & (1 << j)) continue;
        const int r1 = r | (1 << j);
        const double2 x0 = a[r], x1 = a[r1];
        a[r] = make_double2(fma(k, x0.x, -x1.x), fma(k, x0.y, -x1.y));
        a[r1] = make_double2(fma(k, x1.x, x0.x), fma(k, x1.y, x0.y));
      }
    }
  }
}

// Buffer position of amplitude p: the index itself for a state in the global
// scratch slot; the swizzled tile position for a state held in shared memory
// (RES, single-tile circuits).
template <bool RES>
__device__ __forceinline__ u32 bpos(u32 p) {
  return RES ? static_cast<u32>(swz(static_cast<int>(p))) : p;
}

template <bool RES>
__device__ __forceinline__ double2 load_src(int mode, const double2 *buf, u32 p, int n,
                                            const double2 *prod) {
  if (mode == kLoadNatural) return buf[bpos<RES>(p)];
  if (mode == kLoadGatherP) return buf[bpos<RES>(static_cast<u32>(ring_p(p, n)))];
  if (mode == kLoadProduct) return table4(prod, static_cast<u32>(ring_pinv(p, n)));
  return table4(prod, p);
}

template <bool RES>
__device__ __forceinline__ void store_dst(int mode, double2 *buf, u32 p, int n, double2 v) {
  if (mode == kStoreNatural) buf[bpos<RES>(p)] = v;
  else if (mode == kStoreScatterP) buf[bpos<RES>(static_cast<u32>(ring_p(p, n)))] = v;
  else if (mode == kStoreScatterPinv) buf[bpos<RES>(static_cast<u32>(ring_pinv(p, n)))] = v;
}

struct Shared {
  PassParams P;  // the current pass (uniform over the CTA; kept off the thread stacks)
  double2 km[12];  // tangent form of the wire gated on each tile bit of the pass
  double2 stage_a[kTileSize];
  double2 stage_b[kTileSize];
  double2 trans[kTileSize];
  double red[16][12];
  double phi_sm[33];
  double theta[kBatchMaxLayers * kBatchMaxQubits];
  double phi_b[kBatchMaxLayers * kBatchMaxQubits];
  double phi_tot[kBatchMaxLayers];
  double energy;       // this CTA's part of the circuit's energy
  int item;            // work item taken by the cluster's rank 0 (read through DSMEM)
  int next;
};

// One pass (forward or backward) of one circuit: tiles q, q + per, q + 2 per, ...
// RES: a single-tile circuit whose buffers are the shared staging arrays
// (P.psi_in ... point into shared memory, positions swizzled): its loads read
// them directly, its CTA transposes reuse them once every thread holds its
// amplitudes, and its stores write them back after the pass's last barrier.
template <bool BWD, bool RES>
__device__ void run_pass(const PassParams &P, Shared &S, int lane, int warp, double (&acc)[12], u32 q,
                         u32 per) {
  const int n = P.n;
  double2 *wbuf = S.trans + warp * 256;
  const bool has_lo = P.gate_wire[0] >= 0 || P.gate_wire[1] >= 0 || P.gate_wire[2] >= 0;
  const bool staged = !RES && (P.psi_load == kLoadNatural || P.psi_load == kLoadGatherP);
  const int tpi = lane | (warp << 5);
  const u32 toffi = thread_offset(P, tpi);
  const u32 v9 = P.vec[9], v10 = P.vec[10], v11 = P.vec[11];
  const int tb0 = tpart<B0>(lane, warp);
  const u32 toffb0 = thread_offset(P, tb0);
  const int tps = tpart<A2>(lane, warp);
  const u32 toffs = thread_offset(P, tps);
  const u32 v3 = P.vec[3], v4 = P.vec[4], v5 = P.vec[5];
  const u32 num_tiles = static_cast<u32>(P.num_tiles);

  double2 ratio[4];
  if (P.phase) {
#pragma unroll
    for (int j = 0; j < 3; ++j) ratio[j] = phase_ratio(P, unit_bit(BWD ? P.vec[9 + j] : P.vec[3 + j]));
    ratio[3] = make_double2(1.0, 0.0);
  }
  if (BWD && P.phi_grad && threadIdx.x < 33) S.phi_sm[threadIdx.x] = 0.0;

  auto issue = [&](u32 tile) {
    const u32 base = deposit(P, tile) ^ toffi;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const u32 p = base ^ ((r & 1) ? v9 : 0u) ^ ((r & 2) ? v10 : 0u) ^ ((r & 4) ? v11 : 0u);
      const int s = swz(tpi | (r << 9));
      const u32 ps = P.psi_load == kLoadGatherP ? static_cast<u32>(ring_p(p, n)) : p;
      cp_async16(&S.stage_a[s], &P.psi_in[ps]);
      if (BWD) {
        const u32 ls = P.lam_load == kLoadGatherP ? static_cast<u32>(ring_p(p, n)) : p;
        cp_async16(&S.stage_b[s], &P.lam_in[ls]);
      }
    }
    cp_async_commit();
  };
  if (staged && q < num_tiles) issue(q);

  for (u32 tile = q; tile < num_tiles; tile += per) {
    const u32 cbase = deposit(P, tile);
    double2 a[kR], b[kR];
    if (staged) {
      cp_async_wait_all();
      __syncthreads();
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const int s = swz(tb0 | (r << 9));
        a[r] = S.stage_a[s];
        if (BWD) b[r] = S.stage_b[s];
      }
      // the staging buffers now serve the CTA-wide transpose below; the next
      // tile is prefetched right after it
    } else {
      const u32 base = cbase ^ toffb0;
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const u32 p = base ^ ((r & 1) ? v9 : 0u) ^ ((r & 2) ? v10 : 0u) ^ ((r & 4) ? v11 : 0u);
        a[r] = load_src<RES>(P.psi_load, P.psi_in, p, n, P.prod);
        if (RES && BWD) b[r] = load_src<RES>(P.lam_load, P.lam_in, p, n, P.prod);
      }
    }
    if (BWD && P.phase) {
      const double2 ph = table4(P.ptab, cbase ^ toffb0);
      const double K = P.lscale[P.layer];
      apply_phase_gray<3, true, true>(make_double2(K * ph.x, K * ph.y), ratio, a, b);
      phi_sums(P, cbase, lane, warp, a, b, S.red, S.phi_sm);
    }

    if (BWD) gates<B0>(P, S.km, a, b, acc); else fgates<B0>(P, S.km, a);
    warp_transpose<B0, B1>(wbuf, lane, warp, a);
    if (BWD) warp_transpose<B0, B1>(wbuf, lane, warp, b);
    if (BWD) gates<B1>(P, S.km, a, b, acc); else fgates<B1>(P, S.km, a);
    if (has_lo) {
      if (BWD) cta_transpose_pair<B1, A1>(S.stage_a, S.stage_b, lane, warp, a, b);
      else cta_transpose<B1, A1>(S.stage_a, lane, warp, a);
      if (staged && tile + per < num_tiles) issue(tile + per);
      if (BWD) gates<A1>(P, S.km, a, b, acc); else fgates<A1>(P, S.km, a);
      warp_transpose<A1, A2>(wbuf, lane, warp, a);
      if (BWD) warp_transpose<A1, A2>(wbuf, lane, warp, b);
    } else {
      if (BWD) cta_transpose_pair<B1, A2>(S.stage_a, S.stage_b, lane, warp, a, b);
      else cta_transpose<B1, A2>(S.stage_a, lane, warp, a);
      if (staged && tile + per < num_tiles) issue(tile + per);
    }
    if (BWD) gates<A2>(P, S.km, a, b, acc); else fgates<A2>(P, S.km, a);

    const u32 base = cbase ^ toffs;
    if (!BWD && P.phase) {
      const double2 ph = table4(P.ptab, base);
      const double K = P.lscale[P.layer];
      apply_phase_gray<3, false, false>(make_double2(K * ph.x, K * ph.y), ratio, a, b);
    }
    // single-tile in-place permutation: every load of the tile precedes every store
    if (P.sync_after_load) __syncthreads();
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const u32 p = base ^ ((r & 1) ? v3 : 0u) ^ ((r & 2) ? v4 : 0u) ^ ((r & 4) ? v5 : 0u);
      store_dst<RES>(P.psi_store, P.psi_out, p, n, a[r]);
      if (BWD) store_dst<RES>(P.lam_store, P.lam_out, p, n, b[r]);
    }
  }
  __syncthreads();  // the pass's global writes are visible to the next pass
}

// lambda = P^T H P chi and this CTA's part of the energy (amplitudes
// q * blockDim + k * per * blockDim + thread), as rsv_kernels.cu energy_kernel.
template <bool RES>
__device__ double run_energy(const double2 *chi, double2 *mu, int n, double field, Shared &S, u32 q, u32 per) {
  u64 masks[kBatchMaxQubits];
#pragma unroll
  for (int w = 0; w < kBatchMaxQubits; ++w) masks[w] = (w < n) ? ring_pinv(u64{1} << w, n) : 0;
  double e = 0.0;
  const u32 size = 1u << n;
  for (u32 i = q * blockDim.x + threadIdx.x; i < size; i += per * blockDim.x) {
    const double2 c = chi[bpos<RES>(i)];
    const double d = diag_after_ring(i, n);
    double2 x = make_double2(0.0, 0.0);
#pragma unroll
    for (int w = 0; w < kBatchMaxQubits; ++w) {
      if (w < n) {
        const double2 t = chi[bpos<RES>(i ^ static_cast<u32>(masks[w]))];
        x.x += t.x;
        x.y += t.y;
      }
    }
    const double2 m = make_double2(fma(d, c.x, -field * x.x), fma(d, c.y, -field * x.y));
    mu[bpos<RES>(i)] = m;
    e += fma(c.x, m.x, c.y * m.y);
  }
  e = warp_sum(e);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) S.red[warp][0] = e;
  __syncthreads();
  double s = 0.0;
  for (int ww = 0; ww < 16; ++ww) s += S.red[ww][0];
  __syncthreads();
  return s;
}

__global__ void __launch_bounds__(kBatchThreads, 1) batch_kernel(const BatchArgs A) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Shared &S = *reinterpret_cast<Shared *>(smem_raw);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  cg::cluster_group cl = cg::this_cluster();
  const int crank = static_cast<int>(cl.block_rank());
  const int csize = static_cast<int>(cl.num_blocks());
  const int cbase = static_cast<int>(blockIdx.x) - crank;  // the cluster's CTAs are consecutive

  for (;;) {
    // rank 0 takes the cluster's next group; every CTA reads it through DSMEM
    if (crank == 0 && threadIdx.x == 0) S.item = atomicAdd(A.counter, 1);
    cl.sync();
    if (threadIdx.x == 0) S.next = *cl.map_shared_rank(&S.item, 0);
    // every CTA has read rank 0's item before any moves on (or exits: the
    // shared memory of an exited CTA must not be read)
    cl.sync();
    const int item = S.next;
    if (item >= A.num_groups) break;
    const BatchGroup G = A.groups[item];
    const int per = G.per;
    const int sub = crank / per, q = crank % per;
    const bool active = sub < G.count;
    // every CTA of the cluster walks the same plan (inactive ones only keep
    // the barriers), so all take the same cluster barriers
    const BatchCircuit C = A.circuits[A.order[G.first + (active ? sub : 0)]];
    const BatchPlan &PL = A.plans[C.plan];
    const int n = C.n, L = C.L;
    const double *params = A.params + C.param_off;
    const int nl = n * L;
    // the circuit's state buffers and tables: the slot of its first CTA
    unsigned char *slot = A.scratch + static_cast<size_t>(cbase + sub * per) * A.slot_bytes;
    double2 *bufs[3];
    for (int i = 0; i < 3; ++i) bufs[i] = reinterpret_cast<double2 *>(slot + i * A.state_bytes);
    // a circuit of at most 12 qubits (one tile, every permutation in place,
    // two live buffers) keeps its state in this CTA's shared memory for all
    // of its layers
    const bool resident = active && n <= kTileBits;
    if (resident) {
      bufs[0] = S.stage_a;
      bufs[1] = S.stage_b;
      bufs[2] = nullptr;
      for (int i = threadIdx.x; i < kTileSize; i += blockDim.x)
        S.stage_a[i] = S.stage_b[i] = make_double2(0.0, 0.0);
    }
    double4 *coef = reinterpret_cast<double4 *>(slot + 3 * A.state_bytes);
    double2 *rot = reinterpret_cast<double2 *>(coef + kBatchMaxLayers * kBatchMaxQubits);
    double *lscale = reinterpret_cast<double *>(rot + kBatchMaxLayers * kBatchMaxQubits);
    double *gscale = lscale + kBatchMaxLayers;
    double2 *ptab = reinterpret_cast<double2 *>(gscale + 2 * kBatchMaxLayers * kBatchMaxQubits);
    double2 *prod = ptab + kBatchMaxLayers * 1024;

    for (int k = threadIdx.x; k < nl; k += blockDim.x) S.theta[k] = 0.0, S.phi_b[k] = 0.0;
    if (threadIdx.x < kBatchMaxLayers) S.phi_tot[threadIdx.x] = 0.0;
    if (active && q == 0) {
      // ---- per-circuit tables (coef_kernel, tables_kernel, rot_kernel) ----
      for (int k = threadIdx.x; k < nl; k += blockDim.x) {
        double st, ct, sp, cp;
        sincos(params[2 * k] * 0.5, &st, &ct);
        sincos(params[2 * k + 1] * 0.5, &sp, &cp);
        coef[k] = make_double4(ct, st, cp, sp);
        rot[k] = (fabs(ct) >= fabs(st)) ? make_double2(st / ct, 1.0) : make_double2(ct / st, -1.0);
      }
      __syncthreads();
      // phase tables (tables_kernel): only the entries an index of the
      // (zero-padded, max(n,12)-bit) state can reach; wires >= n contribute 1 to
      // the RZ phase and the factor of |0> to the product state
      const int phys = n > kTileBits ? n : kTileBits;
      for (int e = threadIdx.x; e < (L + 1) * 1024; e += blockDim.x) {
        const int layer = e / 1024, byte = (e / 256) % 4, v = e % 256;
        if ((v >> max(0, phys - byte * 8)) != 0) continue;  // table4 reads entry 0 of every byte
        double2 accv = make_double2(1.0, 0.0);
        for (int j = 0; j < 8; ++j) {
          const int w = byte * 8 + j;
          const bool one = (v >> j) & 1;
          double2 f;
          if (w >= n) {
            f = (layer < L || !one) ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0);
          } else {
            const double4 k = coef[(layer < L ? layer : 0) * n + w];
            if (layer < L) f = one ? make_double2(k.z, k.w) : make_double2(k.z, -k.w);
            else f = one ? make_double2(k.y * k.z, k.y * k.w) : make_double2(k.x * k.z, -k.x * k.w);
          }
          accv = cmul(accv, f);
        }
        if (layer < L) ptab[layer * 1024 + byte * 256 + v] = accv;
        else prod[byte * 256 + v] = accv;
      }
      if (threadIdx.x < L) {
        const int layer = threadIdx.x;
        auto factor = [&](int w) {
          const double4 k = coef[layer * n + w];
          return (fabs(k.x) >= fabs(k.y)) ? k.x : k.y;
        };
        double K = 1.0;
        for (int w = 0; w < n; ++w) K *= factor(w);
        lscale[layer] = K;
        double pending = K;
        for (int i = 0; i < n; ++i) {
          const int w = A.undo[PL.undo_off + i];
          gscale[2 * (layer * n + w)] = 1.0 / (pending * pending);
          gscale[2 * (layer * n + w) + 1] = 1.0 / (K * K);
          pending /= factor(w);
        }
      }
      __threadfence();
    }
    __syncthreads();
    cl.sync();  // the tables are visible to the circuit's other CTAs

    // ---- the plan ----
    for (int si = 0; si < PL.num_steps; ++si) {
      const BatchStep &st = A.steps[PL.first_step + si];
      if (st.kind == kBatchEnergy) {
        if (resident) S.energy = run_energy<true>(bufs[st.psi_in], bufs[st.psi_out], n, C.h, S, q, per);
        else if (active) S.energy = run_energy<false>(bufs[st.psi_in], bufs[st.psi_out], n, C.h, S, q, per);
        __threadfence();
        cl.sync();
        if (A.grad_out == nullptr) break;  // energies only: skip the backward sweep
        continue;
      }
      const BatchTile &T = A.tiles[st.tile];
      if (threadIdx.x == 0) {
        PassParams &P = S.P;
        P.n = n;
        P.layer = st.layer;
        P.num_runs = T.num_runs;
        for (int r = 0; r < 4; ++r) P.run_start[r] = T.run_start[r], P.run_len[r] = T.run_len[r];
        P.num_tiles = T.num_tiles;
        for (int b = 0; b < 12; ++b) P.vec[b] = T.vec[b], P.gate_wire[b] = T.gate_wire[b];
        for (int w = 0; w < 32; ++w) P.wire_tile_bit[w] = T.wire_tile_bit[w];
        P.psi_load = st.psi_load;
        P.lam_load = st.lam_load;
        P.psi_store = st.psi_store;
        P.lam_store = st.lam_store;
        P.phase = st.phase;
        P.phi_grad = st.phase;
        P.sync_after_load = T.num_tiles == 1;
        P.psi_in = st.psi_in >= 0 ? bufs[st.psi_in] : nullptr;
        P.psi_out = st.psi_out >= 0 ? bufs[st.psi_out] : nullptr;
        P.lam_in = st.lam_in >= 0 ? bufs[st.lam_in] : nullptr;
        P.lam_out = st.lam_out >= 0 ? bufs[st.lam_out] : nullptr;
        P.coef = coef;
        P.rot = rot;
        P.lscale = lscale;
        P.ptab = ptab + st.layer * 1024;
        P.prod = prod;
        P.partials = nullptr;
        for (int b = 0; b < 12; ++b)
          S.km[b] = T.gate_wire[b] >= 0 ? rot[st.layer * n + T.gate_wire[b]] : make_double2(0.0, 1.0);
      }
      __syncthreads();
      if (active) {
        const PassParams &P = S.P;
        double acc[12];
#pragma unroll
        for (int i = 0; i < 12; ++i) acc[i] = 0.0;
        if (st.kind == kBatchForward) {
          if (resident) run_pass<false, true>(P, S, lane, warp, acc, static_cast<u32>(q), static_cast<u32>(per));
          else run_pass<false, false>(P, S, lane, warp, acc, static_cast<u32>(q), static_cast<u32>(per));
        } else {
          if (resident) run_pass<true, true>(P, S, lane, warp, acc, static_cast<u32>(q), static_cast<u32>(per));
          else run_pass<true, false>(P, S, lane, warp, acc, static_cast<u32>(q), static_cast<u32>(per));
          // this CTA's theta sums of the pass into its accumulators
#pragma unroll
          for (int i = 0; i < 12; ++i) {
            const double s = warp_sum(acc[i]);
            if (lane == 0) S.red[warp][i] = s;
          }
          __syncthreads();
          if (threadIdx.x < 12 && T.gate_wire[threadIdx.x] >= 0) {
            double s = 0.0;
            for (int ww = 0; ww < 16; ++ww) s += S.red[ww][threadIdx.x];
            S.theta[st.layer * n + T.gate_wire[threadIdx.x]] += s;
          }
          if (st.phase) {
            if (threadIdx.x < n) S.phi_b[st.layer * n + threadIdx.x] = S.phi_sm[threadIdx.x];
            if (threadIdx.x == 32) S.phi_tot[st.layer] = S.phi_sm[32];
          }
          __syncthreads();
        }
      }
      __threadfence();
      cl.sync();  // the pass's global writes are visible to the circuit's CTAs
    }

    // ---- outputs: the first CTA of a circuit adds its CTAs' parts in order ----
    if (active && q == 0) {
      const int lead = sub * per;
      if (threadIdx.x == 0) {
        double e = 0.0;
        for (int j = 0; j < per; ++j) e += *cl.map_shared_rank(&S.energy, lead + j);
        A.energy_out[C.index] = e;
      }
      if (A.grad_out != nullptr) {
        double *g = A.grad_out + C.param_off;
        for (int k = threadIdx.x; k < nl; k += blockDim.x) {
          const int layer = k / n;
          double th = 0.0, pb = 0.0, pt = 0.0;
          for (int j = 0; j < per; ++j) {
            th += cl.map_shared_rank(S.theta, lead + j)[k];
            pb += cl.map_shared_rank(S.phi_b, lead + j)[k];
            pt += cl.map_shared_rank(S.phi_tot, lead + j)[layer];
          }
          g[2 * k] = th * gscale[2 * k];
          g[2 * k + 1] = (pt - 2.0 * pb) * gscale[2 * k + 1];
        }
      }
    }
    __syncthreads();
    cl.sync();  // the parts stay in place until they are read
  }
}

}  // namespace

size_t batch_smem_bytes() { return sizeof(Shared); }

size_t batch_slot_table_bytes() {
  return kBatchMaxLayers * kBatchMaxQubits * (sizeof(double4) + sizeof(double2) + 2 * sizeof(double)) +
         kBatchMaxLayers * sizeof(double) + (kBatchMaxLayers + 1) * 1024 * sizeof(double2);
}

cudaError_t configure_batch_kernel() {
  return cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(sizeof(Shared)));
}

cudaError_t launch_batch(const BatchArgs &A, int grid, int cluster, cudaStream_t s) {
  if (cluster < 1 || cluster > 8 || grid % cluster != 0) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(grid));
  cfg.blockDim = dim3(kBatchThreads);
  cfg.dynamicSmemBytes = sizeof(Shared);
  cfg.stream = s;
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = static_cast<unsigned>(cluster);
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, batch_kernel, A);
}

int batch_max_active_clusters(int cluster) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(cluster));
  cfg.blockDim = dim3(kBatchThreads);
  cfg.dynamicSmemBytes = sizeof(Shared);
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = static_cast<unsigned>(cluster);
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int num = 0;
  if (cudaOccupancyMaxActiveClusters(&num, batch_kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return num;
}

}  // namespace rsv
