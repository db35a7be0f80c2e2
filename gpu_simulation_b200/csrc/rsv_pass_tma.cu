// Backward tile pass on 11-bit tiles fed by the Tensor Memory Accelerator
// (sm_100a): psi and lambda arrive by tensor copies into shared memory and
// lambda leaves by a tensor store; the four warps of a block synchronise only
// through split-phase mbarriers (each warp arrives as soon as its part is
// done and waits only where it needs the others), and two blocks share an SM.
//
// Same arithmetic as bwd_half_kernel (rsv_pass_half.cu) and bwd_pass_kernel
// (rsv_pass.cu) -- the reference's backward chunk kernels
// (zzEncounter/GPU_Simulation cpp/ising_cuda_statevector_grad_kernels.cu:683-1326)
// restated on tiles -- for the passes whose gates lie on tile bits 3..10 of an
// 11-bit unit tile with tile bits 0..2 = index bits 0..2, psi read from a
// forward checkpoint and lambda updated in place.
//
// Per tile (2048 amplitudes of psi and of lambda, 32 KiB each), every warp:
//   wait `full` -> read its 512 amplitudes of psi and lambda (16 registers
//   each) -> arrive `sread` -> [RZ^dagger, phi sums] -> rotate tile bits
//   7..10 -> wait `oempty` -> transpose through its quarter of the output
//   buffer -> arrive `xdone` -> rotate tile bits 3..6 -> wait `xdone` -> write
//   lambda into the output box -> proxy fence -> arrive `ofull`;
// and thread 0 besides: after `sread`, the tensor loads of the next tile (the
// stage is free); the wait until the previous store has read the output
// buffer, then `oempty`; after `ofull`, the tensor store of this tile.
// Layouts (tile index t, 11 bits; warp w owns tile bits 1, 2):
//   P: lanes -> tile bits 3,4,5,6,0   registers -> 7..10
//   Q: lanes -> tile bits 7,8,9,10,0  registers -> 3..6
// The stage holds the tile in tile-index order under the 128-byte swizzle, so
// the reads of layout P are conflict-free; the output buffer holds the box of
// a second tensor map whose dimensions are ordered (tile bits 0..2, 7..10,
// 3..6), so the writes of layout Q are conflict-free too.  Every wait is
// bounded: after 1.5 s it records an error code and the block winds down
// (thread 0 first waits, again bounded, for its own load in flight).
// No copy here uses cluster multicast; every tensor map covers this GPU's own
// memory.
#include <cudaTypedefs.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rsv_launch.h"
#include "rsv_tile.cuh"
#include "rsv_tma.h"

namespace rsv {
namespace {

namespace tw {
constexpr int kWarps = 4;
constexpr int kThreads = 32 * kWarps;
constexpr int kR = 16;
constexpr int kTile = 2048;
constexpr unsigned kVecBytes = kTile * 16u;  // 32 KiB
// dynamic shared memory from a 1024-byte aligned base: the stage (psi, then
// lambda, 32 KiB each), then the lambda output box, whose four 8 KiB quarters
// also serve as the warps' transpose slices
constexpr unsigned kObufOff = 2 * kVecBytes;
constexpr unsigned kSmemBytes = kObufOff + kVecBytes + 1024;
constexpr unsigned long long kWaitNs = 1500000000ull;

__device__ __forceinline__ int tP(int lane, int warp, int r) {
  return (lane >> 4) | (warp << 1) | ((lane & 15) << 3) | (r << 7);
}
__device__ __forceinline__ int tQ(int lane, int warp, int r) {
  return (lane >> 4) | (warp << 1) | (r << 3) | ((lane & 15) << 7);
}
// the 128-byte swizzle of a 16-byte element index in a 1024-byte aligned buffer
__device__ __forceinline__ int sw128(int t) { return t ^ ((t >> 3) & 7); }
// position of tile index t in the output box (tile bits 0..2, 7..10, 3..6)
__device__ __forceinline__ int opos(int t) {
  return sw128((t & 7) | (((t >> 7) & 15) << 3) | (((t >> 3) & 15) << 7));
}
// warp slice: s = tile bit 0 | tile bits 3..10 << 1; the XOR of slice bits
// 5..7 (and 3) into 0..2 makes both the P writes and the Q reads conflict-free
__device__ __forceinline__ int xpos(int s) { return s ^ (((s >> 5) & 7) ^ ((s >> 3) & 1)); }
__device__ __forceinline__ int sP(int lane, int r) { return (lane >> 4) | ((lane & 15) << 1) | (r << 5); }
__device__ __forceinline__ int sQ(int lane, int r) { return (lane >> 4) | (r << 1) | ((lane & 15) << 5); }

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned a, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(a) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned a, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned a, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Wait for the completion of the mbarrier phase with this parity; false when
// it has not completed after kWaitNs.
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity) {
  if (mbar_try(a, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try(a, parity))
    if (global_ns() - t0 > kWaitNs) return false;
  return true;
}
__device__ __forceinline__ void tma_load(unsigned dst, const CUtensorMap *map, const int (&c)[kTmaRank],
                                         unsigned mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(dst),
      "l"(map), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void tma_store(const CUtensorMap *map, const int (&c)[kTmaRank], unsigned src) {
  asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];\n" ::"l"(
                   map),
               "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void coords(u32 cbase, const int *shift, const unsigned *mask, int (&c)[kTmaRank]) {
#pragma unroll
  for (int d = 0; d < kTmaRank; ++d) c[d] = static_cast<int>((cbase >> shift[d]) & mask[d]);
}

// RY^dagger / f in tangent form on the four register bits (tile bits
// TB0..TB0+3) with the theta sums Re(conj(lam1) psi0) - Re(conj(lam0) psi1)
// accumulated first, as bw::gates (rsv_tile.cuh); two partial sums per wire,
// added to the thread's running sums acc[(tile bit - 3) * kThreads] (shared
// memory: the registers hold psi and lambda).
template <int TB0>
__device__ __forceinline__ void gates16(const PassParams &P, const double2 *km_tb, double2 (&a)[kR],
                                        double2 (&b)[kR], double *acc) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int tb = TB0 + j;
    if (P.gate_wire[tb] < 0) continue;
    const double2 km = km_tb[tb];
    const double k = km.x;
    double t0 = 0.0, t1 = 0.0;
    const bool plus = km.y > 0.0;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      if (r & (1 << j)) continue;
      const int r1 = r | (1 << j);
      const double2 x0 = a[r], x1 = a[r1], y0 = b[r], y1 = b[r1];
      double &t = ((r >> ((j + 1) & 3)) & 1) ? t1 : t0;
      t = fma(y1.x, x0.x, t);
      t = fma(y1.y, x0.y, t);
      t = fma(-y0.x, x1.x, t);
      t = fma(-y0.y, x1.y, t);
      if (plus) {
        a[r] = make_double2(fma(k, x1.x, x0.x), fma(k, x1.y, x0.y));
        a[r1] = make_double2(fma(-k, x0.x, x1.x), fma(-k, x0.y, x1.y));
        b[r] = make_double2(fma(k, y1.x, y0.x), fma(k, y1.y, y0.y));
        b[r1] = make_double2(fma(-k, y0.x, y1.x), fma(-k, y0.y, y1.y));
      } else {
        a[r] = make_double2(fma(k, x0.x, x1.x), fma(k, x0.y, x1.y));
        a[r1] = make_double2(fma(k, x1.x, -x0.x), fma(k, x1.y, -x0.y));
        b[r] = make_double2(fma(k, y0.x, y1.x), fma(k, y0.y, y1.y));
        b[r1] = make_double2(fma(k, y1.x, -y0.x), fma(k, y1.y, -y0.y));
      }
    }
    acc[(tb - 3) * kThreads] += t0 + t1;
  }
}

// The last layout's four gates: the theta sums of all four on the incoming psi
// and lambda (the gates act on different wires and commute, so each sum is
// the one the sequential undo would take), then RY^dagger / f on lambda alone
// (psi is not needed after the pass).
template <int TB0, int NT>
__device__ __forceinline__ void gates_last(const PassParams &P, const double2 *km_tb, const double2 (&a)[kR],
                                           double2 (&b)[kR], double *acc) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int tb = TB0 + j;
    if (P.gate_wire[tb] < 0) continue;
    double t0 = 0.0, t1 = 0.0;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      if (r & (1 << j)) continue;
      const int r1 = r | (1 << j);
      const double2 x0 = a[r], x1 = a[r1], y0 = b[r], y1 = b[r1];
      double &t = ((r >> ((j + 1) & 3)) & 1) ? t1 : t0;
      t = fma(y1.x, x0.x, t);
      t = fma(y1.y, x0.y, t);
      t = fma(-y0.x, x1.x, t);
      t = fma(-y0.y, x1.y, t);
    }
    acc[(tb - 3) * NT] += t0 + t1;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int tb = TB0 + j;
    if (P.gate_wire[tb] < 0) continue;
    const double2 km = km_tb[tb];
    const double k = km.x;
    const bool plus = km.y > 0.0;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      if (r & (1 << j)) continue;
      const int r1 = r | (1 << j);
      const double2 y0 = b[r], y1 = b[r1];
      if (plus) {
        b[r] = make_double2(fma(k, y1.x, y0.x), fma(k, y1.y, y0.y));
        b[r1] = make_double2(fma(-k, y0.x, y1.x), fma(-k, y0.y, y1.y));
      } else {
        b[r] = make_double2(fma(k, y0.x, y1.x), fma(k, y0.y, y1.y));
        b[r1] = make_double2(fma(k, y1.x, -y0.x), fma(k, y1.y, -y0.y));
      }
    }
  }
}

// Field terms of the tile, layout P: per register r the partner sum
// s = sum_m psi(t ^ m) over the masks tma_energy_mask(U, .), then lambda[r] -= h s and the
// energy share -h Re(conj(psi[r]) s) into e.  A mask's tile bits 7..10 are
// register bits (XOR h = m >> 7) and its bits 0..6 (lo) lane and warp bits;
// sw128 is linear over XOR and leaves bits 7..10 alone, so the partner of
// register r is stage[(sw128(tP(r = 0)) ^ sw128(lo)) + ((r ^ h) << 7)]: one base
// per mask, compile-time offsets; masks on register bits only take the
// partner from the thread's own registers.
template <int M>
__device__ __forceinline__ double2 epartner(const double2 *stage, int s0, int r, const double2 (&a)[kR]) {
  constexpr int lo = M & 0x7F, h = (M >> 7) & 15;
  if constexpr (lo == 0) {
    return a[r ^ h];
  } else {
    return stage[(s0 ^ sw128(lo)) + ((r ^ h) << 7)];
  }
}
template <int U>
__device__ __forceinline__ void emask_apply(double h, const double2 *stage, int lane, int warp,
                                            const double2 (&a)[kR], double2 (&b)[kR], double &e) {
  static_assert(kTmaNumEnergyMasks == 10, "the partner sum below lists the masks");
  const int s0 = sw128(tP(lane, warp, 0));
  double es = 0.0;  // sum of Re(conj(psi) s); times -h below
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const double2 q[kTmaNumEnergyMasks] = {
        epartner<tma_energy_mask(U, 0)>(stage, s0, r, a), epartner<tma_energy_mask(U, 1)>(stage, s0, r, a),
        epartner<tma_energy_mask(U, 2)>(stage, s0, r, a), epartner<tma_energy_mask(U, 3)>(stage, s0, r, a),
        epartner<tma_energy_mask(U, 4)>(stage, s0, r, a), epartner<tma_energy_mask(U, 5)>(stage, s0, r, a),
        epartner<tma_energy_mask(U, 6)>(stage, s0, r, a), epartner<tma_energy_mask(U, 7)>(stage, s0, r, a),
        epartner<tma_energy_mask(U, 8)>(stage, s0, r, a), epartner<tma_energy_mask(U, 9)>(stage, s0, r, a)};
    double2 sum = q[0];
#pragma unroll
    for (int j = 1; j < kTmaNumEnergyMasks; ++j) sum = make_double2(sum.x + q[j].x, sum.y + q[j].y);
    b[r] = make_double2(fma(-h, sum.x, b[r].x), fma(-h, sum.y, b[r].y));
    es = fma(a[r].x, sum.x, fma(a[r].y, sum.y, es));
  }
  e = fma(-h, es, e);
}

// The middle pass's field terms, layout P: for the adjacent pairs of gated tile
// bits (3 + j, 4 + j), j < 7, lambda[r] += ph[4 j + q] psi(t ^ m_j) (q = the
// pair's bits of t; ph holds -h F^2 and the RZ phase ratio) and the energy
// share Re(conj(psi[r]) delta) into e.  Pairs of register bits (j >= 4) take
// the partner from the thread's own registers, the others from the stage.
// (Multiplying the warp's psi in the stage by the phases first, so that one
// phase per amplitude would do, measured slower: the extra stage writes and
// partner loads cost more than the six products they save.)
__device__ __forceinline__ double2 cadd(double2 x, double2 y) { return make_double2(x.x + y.x, x.y + y.y); }
template <int J>
__device__ __forceinline__ double2 dpartner(const double2 *stage, int s0, int r, const double2 (&a)[kR]) {
  return epartner<(3 << (3 + J))>(stage, s0, r, a);
}
__device__ __forceinline__ void dmask_apply(const double2 *ph, const double2 *stage, int lane, int warp,
                                            const double2 (&a)[kR], double2 (&b)[kR], double &e) {
  static_assert(kTmaNumDeferredMasks == 7, "the sum below lists the masks");
  const int s0 = sw128(tP(lane, warp, 0));
  // pairs j = 0..2 lie on lane bits (tile bits 3..6 = lane bits 0..3): one
  // phase per thread; j = 3 on lane bit 3 and register bit 0: two; j = 4..6 on
  // register bits: selected per register (compile time), loaded per use
  const int lq = lane & 15;
  const double2 p0 = ph[0 + (lq & 3)], p1 = ph[4 + ((lq >> 1) & 3)], p2 = ph[8 + ((lq >> 2) & 3)];
  const double2 p3e = ph[12 + (lq >> 3)], p3o = ph[12 + (lq >> 3) + 2];
  double es = 0.0;
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    double2 d = cmul(p0, dpartner<0>(stage, s0, r, a));
    d = cadd(d, cmul(p1, dpartner<1>(stage, s0, r, a)));
    d = cadd(d, cmul(p2, dpartner<2>(stage, s0, r, a)));
    d = cadd(d, cmul((r & 1) ? p3o : p3e, dpartner<3>(stage, s0, r, a)));
    d = cadd(d, cmul(ph[16 + (r & 3)], dpartner<4>(stage, s0, r, a)));
    d = cadd(d, cmul(ph[20 + ((r >> 1) & 3)], dpartner<5>(stage, s0, r, a)));
    d = cadd(d, cmul(ph[24 + ((r >> 2) & 3)], dpartner<6>(stage, s0, r, a)));
    b[r] = make_double2(b[r].x + d.x, b[r].y + d.y);
    es = fma(a[r].x, d.x, fma(a[r].y, d.y, es));
  }
  e += es;
}

// layout P -> layout Q of one vector through the warp's slice
__device__ __forceinline__ void transpose_pq(double2 *xs, int lane, double2 (&a)[kR]) {
#pragma unroll
  for (int r = 0; r < kR; ++r) xs[xpos(sP(lane, r))] = a[r];
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kR; ++r) a[r] = xs[xpos(sQ(lane, r))];
  __syncwarp();
}
}  // namespace tw

template <bool PHASE>
__global__ void __launch_bounds__(tw::kThreads, 2)
    bwd_tma_kernel(const __grid_constant__ PassParams P, const __grid_constant__ TmaPass T) {
  using namespace tw;
  extern __shared__ unsigned char smem_raw[];
  // full (tx), sread (4), oempty (1), xdone (4), ofull (4): each completes
  // one phase per tile
  __shared__ __align__(8) unsigned long long bars[5];
  __shared__ double2 km_sm[12];
  __shared__ double red[kWarps][10];
  __shared__ double phi_cos[PHASE ? kWarps : 1][32];
  // per thread: theta sums of tile bits 3..10 and phi sums (total, register
  // bits 0..3); the phase ratios of tile bits 7..10
  __shared__ double acc_sm[8 * kThreads];
  __shared__ double v_sm[PHASE ? 5 * kThreads : 1];
  __shared__ double2 ratio_sm[4];
  __shared__ double2 dph_sm[PHASE ? kTmaDeferTable : 1];
  __shared__ volatile int abort_flag;

  const unsigned raw = smem_u32(smem_raw);
  const unsigned pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char *smem = smem_raw + pad;
  const unsigned sbase = raw + pad;
  const double2 *stage = reinterpret_cast<const double2 *>(smem);
  double2 *obuf = reinterpret_cast<double2 *>(smem + kObufOff);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned full = smem_u32(&bars[0]), sread = smem_u32(&bars[1]), oempty = smem_u32(&bars[2]);
  const unsigned xdone = smem_u32(&bars[3]), ofull = smem_u32(&bars[4]);
  if (tid == 0) {
    mbar_init(full, 1);
    mbar_init(sread, kWarps);
    mbar_init(oempty, 1);
    mbar_init(xdone, kWarps);
    mbar_init(ofull, kWarps);
    fence_mbar_init();
    abort_flag = 0;
  }
  if (tid < 12) {
    const int w = P.gate_wire[tid];
    km_sm[tid] = w >= 0 ? RSV_TABLE_LOAD(&P.rot[P.layer * P.n + w]) : make_double2(0.0, 1.0);
  }
  if (PHASE) phi_cos[warp][lane] = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc_sm[i * kThreads + tid] = 0.0;
  if (PHASE) {
#pragma unroll
    for (int i = 0; i < 5; ++i) v_sm[i * kThreads + tid] = 0.0;
    if (tid < 4) ratio_sm[tid] = phase_ratio(P, unit_bit(P.vec[7 + tid]));
    if (T.defer_terms && tid < kTmaDeferTable) dph_sm[tid] = T.emask_phase[tid];
  }
  __syncthreads();

  const u32 num_tiles = static_cast<u32>(P.num_tiles);
  const u32 first = blockIdx.x;
  const int my_tiles = first < num_tiles ? static_cast<int>((num_tiles - 1 - first) / gridDim.x) + 1 : 0;
  const bool leader = tid == 0;  // issues the tensor copies
  int loads = 0;                 // tensor loads issued (phases of `full` started)
  auto issue = [&](int j) {
    int c[kTmaRank];
    coords(deposit(P, first + static_cast<u32>(j) * gridDim.x), T.ld_shift, T.ld_mask, c);
    mbar_expect_tx(full, 2u * kVecBytes);
    tma_load(sbase, &T.psi_map, c, full);
    tma_load(sbase + kVecBytes, &T.lam_map, c, full);
    ++loads;
  };
  if (leader && my_tiles > 0) issue(0);

  double *acc = acc_sm + tid;
  double *v = v_sm + tid;
  double e_acc = 0.0;  // energy share of the terms this pass applies
  const u32 toffP = thread_offset(P, tP(lane, warp, 0));
  double2 *xs = obuf + warp * 512;  // the warp's transpose slice (inside the output buffer)
  int fail = 0;

  for (int j = 0; j < my_tiles; ++j) {
    if (abort_flag) break;
    const unsigned par = static_cast<unsigned>(j) & 1u;
    if (!mbar_wait(full, par)) {
      fail = 1;
      break;
    }
    double2 a[kR], b[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int t = sw128(tP(lane, warp, r));
      a[r] = stage[t];
      b[r] = stage[kTile + t];
    }
    if (PHASE && T.defer_terms) dmask_apply(dph_sm, stage, lane, warp, a, b, e_acc);
    if (PHASE && T.energy_terms) {
      switch (T.energy_terms - 1) {
        case 0: emask_apply<0>(T.efield, stage, lane, warp, a, b, e_acc); break;
        case 1: emask_apply<1>(T.efield, stage, lane, warp, a, b, e_acc); break;
        case 2: emask_apply<2>(T.efield, stage, lane, warp, a, b, e_acc); break;
        default: emask_apply<3>(T.efield, stage, lane, warp, a, b, e_acc); break;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(sread);
    if (leader) {
      // the stage is free once every warp has read it: prefetch the next tile;
      // the previous tile's store must have read the output buffer before the
      // warps transpose in it
      if (!mbar_wait(sread, par)) {
        fail = 2;
        abort_flag = 1;
      } else if (j + 1 < my_tiles) {
        issue(j + 1);
      }
      if (j > 0) {
        bulk_wait_read_all();
        mbar_arrive(oempty);
      }
    }
    __syncwarp();
    if (abort_flag) break;

    const u32 cbase = deposit(P, first + static_cast<u32>(j) * gridDim.x);
    if (PHASE) {
      // RZ^dagger of the layer (with the layer's factor K) on psi and lambda
      // (not in a phi_only pass), then the phi sums q = Im(conj(lam) psi)
      if (!T.phi_only) {
        const double2 ph = table4(P.ptab, cbase ^ toffP);
        const double K = P.lscale[P.layer];
        const double2 ratio[4] = {ratio_sm[0], ratio_sm[1], ratio_sm[2], ratio_sm[3]};
        apply_phase_gray<4, true, true>(make_double2(K * ph.x, K * ph.y), ratio, a, b);
      }
      double tot = 0.0, rb[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const double q = fma(b[r].x, a[r].y, -b[r].y * a[r].x);
        tot += q;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          if ((r >> jj) & 1) rb[jj] += q;
      }
      v[0] += tot;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) v[(1 + jj) * kThreads] += rb[jj];
      const double sw = warp_sum(tot);
      if (lane < P.n && P.wire_tile_bit[lane] < 0 && ((cbase >> lane) & 1)) phi_cos[warp][lane] += sw;
    }
    gates16<7>(P, km_sm, a, b, acc);

    if (j > 0 && !mbar_wait(oempty, par ^ 1u)) {
      fail = 3;
      break;
    }
    transpose_pq(xs, lane, a);
    transpose_pq(xs, lane, b);
    if (lane == 0) mbar_arrive(xdone);
    gates_last<3, kThreads>(P, km_sm, a, b, acc);
    // every warp has left its slice before any warp writes the output box
    if (!mbar_wait(xdone, par)) {
      fail = 4;
      break;
    }
#pragma unroll
    for (int r = 0; r < kR; ++r) obuf[opos(tQ(lane, warp, r))] = b[r];
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive(ofull);
    if (leader) {
      if (!mbar_wait(ofull, par)) {
        fail = 5;
        break;
      }
      int c[kTmaRank];
      coords(cbase, T.st_shift, T.st_mask, c);
      tma_store(&T.out_map, c, sbase + kObufOff);
      bulk_commit();
    }
  }
  if (fail) {
    atomicExch(T.err, fail);
    abort_flag = 1;
  }
  if (leader) {
    // a load this block issued must land before the block exits
    if (abort_flag && loads > 0) mbar_wait(full, static_cast<unsigned>(loads - 1) & 1u);
    bulk_wait_all();
  }

  // CTA reduction of the theta sums, one record per CTA
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const double s = warp_sum(acc[i * kThreads]);
    if (lane == 0) red[warp][i] = s;
  }
  __syncthreads();
  double *rec = P.partials + static_cast<size_t>(blockIdx.x) * kPartialStride;
  if (tid < 12) {
    double s = 0.0;
    if (tid >= 3 && tid <= 10)
      for (int ww = 0; ww < kWarps; ++ww) s += red[ww][tid - 3];
    rec[tid] = s;
  }
  if (PHASE && (T.energy_terms || T.defer_terms)) {
    const double es = warp_sum(e_acc);
    __syncthreads();  // red is reused
    if (lane == 0) red[warp][0] = es;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int ww = 0; ww < kWarps; ++ww) s += red[ww][0];
      T.energy_partials[blockIdx.x] = s;
    }
  }
  if (PHASE) {
    __syncthreads();  // red is reused
    double x[10];
#pragma unroll
    for (int i = 0; i < 5; ++i) x[i] = v[i * kThreads];
#pragma unroll
    for (int k = 0; k < 5; ++k) x[5 + k] = ((lane >> k) & 1) ? v[0] : 0.0;
#pragma unroll
    for (int i = 0; i < 10; ++i) x[i] = warp_sum(x[i]);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 10; ++i) red[warp][i] = x[i];
    }
    __syncthreads();
    if (tid < 32) {
      const int w = tid;
      double qt = 0.0;
      for (int ww = 0; ww < kWarps; ++ww) qt += red[ww][0];
      if (w < 31) {
        double add = 0.0;
        if (w < P.n) {
          const int tb = P.wire_tile_bit[w];
          if (tb < 0) {
            for (int ww = 0; ww < kWarps; ++ww) add += phi_cos[ww][w];
          } else if (tb >= 7) {
            for (int ww = 0; ww < kWarps; ++ww) add += red[ww][1 + tb - 7];
          } else if (tb >= 3) {
            for (int ww = 0; ww < kWarps; ++ww) add += red[ww][5 + tb - 3];
          } else if (tb == 0) {
            for (int ww = 0; ww < kWarps; ++ww) add += red[ww][9];
          } else {
            for (int ww = 0; ww < kWarps; ++ww)
              if ((ww >> (tb - 1)) & 1) add += red[ww][0];
          }
        }
        rec[kPartialPhi + w] = add;
      } else {
        rec[kPartialTot] = qt;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The 12-wire low pass: a unit tile over index bits 0..11 (4096 contiguous
// amplitudes), every tile bit gated, psi from a checkpoint, lambda in place.
// 8 warps x 16 registers, one block per SM.  Layouts (tile index t, 12 bits):
//   LC: warps -> 5,6,7    lanes -> 0..4           registers -> 8..11
//   LA: warps -> 9,10,11  lanes -> 3,4,5,6,8      registers -> 0,1,2,7
//   LB: warps -> 9,10,11  lanes -> 0,1,2,7,8      registers -> 3..6
// The one change of warp bits comes first: every warp reads LC from the
// stage, rotates 8..11 and writes the result back to the same places; after
// `xw` every warp reads LA (its own region, bits 9..11 = warp) and the stage
// is free, so thread 0 loads the next tile there about a third into this
// one.  LA -> LB is warp-local, through the warp's own region of the
// exchange buffer X; lambda is stored from LB (lanes 0..2: whole 128-byte
// lines).  Per tile, every warp:
//   wait `fullp`, `fulll` -> read LC -> rotate 8..11 -> write back -> arrive
//   `xw`, wait `xw` -> read LA -> arrive `sread` -> rotate 0,1,2,7 ->
//   transpose psi, lambda to LB -> rotate 3..6 -> store lambda;
// thread 0 besides: after `sread`, the tensor loads of the next tile.  All
// shared buffers are in tile-index order under the 128-byte swizzle, which
// keeps every access pattern above conflict-free.  Waits are bounded as in
// bwd_tma_kernel.
// ---------------------------------------------------------------------------
namespace tl {
constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;
constexpr int kR = 16;
constexpr int kTile = 4096;
constexpr unsigned kVecBytes = kTile * 16u;  // 64 KiB
// stage psi at 0, stage lambda at 64 KiB, X at 128 KiB (from a 1024-aligned base)
constexpr unsigned kSmemBytes = 3 * kVecBytes + 1024;

__device__ __forceinline__ int tC(int l, int w, int r) { return (l & 31) | (w << 5) | (r << 8); }
__device__ __forceinline__ int tA(int l, int w, int r) {
  return (r & 7) | ((l & 15) << 3) | ((r >> 3) << 7) | ((l >> 4) << 8) | (w << 9);
}
__device__ __forceinline__ int tB(int l, int w, int r) {
  return (l & 7) | (r << 3) | ((l >> 3) << 7) | (w << 9);
}
__device__ __forceinline__ int sw(int t) { return t ^ ((t >> 3) & 7); }

// tile bit of register bit j in layout L (0: LC, 1: LA, 2: LB)
template <int L>
__host__ __device__ constexpr int rtb(int j) {
  return L == 0 ? 8 + j : L == 1 ? (j < 3 ? j : 7) : 3 + j;
}

// as tw::gates16 for the register bits of layout L; acc[tile bit * kThreads]
// is the thread's running theta sum (shared memory)
template <int L>
__device__ __forceinline__ void gates(const PassParams &P, const double2 *km_tb, double2 (&a)[kR],
                                      double2 (&b)[kR], double *acc) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int tb = rtb<L>(j);
    if (P.gate_wire[tb] < 0) continue;
    const double2 km = km_tb[tb];
    const double k = km.x;
    double t0 = 0.0, t1v = 0.0;
    const bool plus = km.y > 0.0;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      if (r & (1 << j)) continue;
      const int r1 = r | (1 << j);
      const double2 x0 = a[r], x1 = a[r1], y0 = b[r], y1 = b[r1];
      double &t = ((r >> ((j + 1) & 3)) & 1) ? t1v : t0;
      t = fma(y1.x, x0.x, t);
      t = fma(y1.y, x0.y, t);
      t = fma(-y0.x, x1.x, t);
      t = fma(-y0.y, x1.y, t);
      if (plus) {
        a[r] = make_double2(fma(k, x1.x, x0.x), fma(k, x1.y, x0.y));
        a[r1] = make_double2(fma(-k, x0.x, x1.x), fma(-k, x0.y, x1.y));
        b[r] = make_double2(fma(k, y1.x, y0.x), fma(k, y1.y, y0.y));
        b[r1] = make_double2(fma(-k, y0.x, y1.x), fma(-k, y0.y, y1.y));
      } else {
        a[r] = make_double2(fma(k, x0.x, x1.x), fma(k, x0.y, x1.y));
        a[r1] = make_double2(fma(k, x1.x, -x0.x), fma(k, x1.y, -x0.y));
        b[r] = make_double2(fma(k, y0.x, y1.x), fma(k, y0.y, y1.y));
        b[r1] = make_double2(fma(k, y1.x, -y0.x), fma(k, y1.y, -y0.y));
      }
    }
    acc[tb * kThreads] += t0 + t1v;
  }
}
}  // namespace tl

__global__ void __launch_bounds__(tl::kThreads, 1)
    bwd_tma_low_kernel(const __grid_constant__ PassParams P, const __grid_constant__ TmaPass T) {
  using namespace tl;
  using tw::bulk_wait_all;
  using tw::mbar_arrive;
  using tw::mbar_expect_tx;
  using tw::mbar_init;
  using tw::mbar_wait;
  using tw::smem_u32;
  extern __shared__ unsigned char smem_raw[];
  // fullp, fulll (tx), xw (8), sread (8): one phase per tile
  __shared__ __align__(8) unsigned long long bars[4];
  __shared__ double2 km_sm[12];
  __shared__ double red[kWarps][12];
  __shared__ double acc_sm[12 * kThreads];  // per thread: theta sums of tile bits 0..11
  __shared__ volatile int abort_flag;

  const unsigned raw = smem_u32(smem_raw);
  const unsigned pad = (1024u - (raw & 1023u)) & 1023u;
  unsigned char *smem = smem_raw + pad;
  const unsigned sbase = raw + pad;
  double2 *spsi = reinterpret_cast<double2 *>(smem);
  double2 *slam = reinterpret_cast<double2 *>(smem + kVecBytes);
  double2 *xbuf = reinterpret_cast<double2 *>(smem + 2 * kVecBytes);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned fullp = smem_u32(&bars[0]), fulll = smem_u32(&bars[1]), xw = smem_u32(&bars[2]);
  const unsigned sread = smem_u32(&bars[3]);
  if (tid == 0) {
    mbar_init(fullp, 1);
    mbar_init(fulll, 1);
    mbar_init(xw, kWarps);
    mbar_init(sread, kWarps);
    tw::fence_mbar_init();
    abort_flag = 0;
  }
  if (tid < 12) {
    const int w = P.gate_wire[tid];
    km_sm[tid] = w >= 0 ? RSV_TABLE_LOAD(&P.rot[P.layer * P.n + w]) : make_double2(0.0, 1.0);
  }
#pragma unroll
  for (int i = 0; i < 12; ++i) acc_sm[i * kThreads + tid] = 0.0;
  __syncthreads();

  const u32 num_tiles = static_cast<u32>(P.num_tiles);
  const u32 first = blockIdx.x;
  const int my_tiles = first < num_tiles ? static_cast<int>((num_tiles - 1 - first) / gridDim.x) + 1 : 0;
  const bool leader = tid == 0;
  int loads = 0;  // tile loads issued (phases of fullp and fulll started)
  auto issue = [&](int j) {
    int c[kTmaRank];
    tw::coords(deposit(P, first + static_cast<u32>(j) * gridDim.x), T.ld_shift, T.ld_mask, c);
    mbar_expect_tx(fullp, kVecBytes);
    tw::tma_load(sbase, &T.psi_map, c, fullp);
    mbar_expect_tx(fulll, kVecBytes);
    tw::tma_load(sbase + kVecBytes, &T.lam_map, c, fulll);
    ++loads;
  };
  if (leader && my_tiles > 0) issue(0);

  double *acc = acc_sm + tid;
  double2 *lam_out = P.lam_out;
  int fail = 0;

  for (int j = 0; j < my_tiles; ++j) {
    if (abort_flag) break;
    const unsigned par = static_cast<unsigned>(j) & 1u;
    if (!mbar_wait(fullp, par) || !mbar_wait(fulll, par)) {
      fail = 11;
      break;
    }
    double2 a[kR], b[kR];
    // LC: rotate tile bits 8..11 and write back in place
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int t = sw(tC(lane, warp, r));
      a[r] = spsi[t];
      b[r] = slam[t];
    }
    gates<0>(P, km_sm, a, b, acc);
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int t = sw(tC(lane, warp, r));
      spsi[t] = a[r];
      slam[t] = b[r];
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(xw);
    if (!mbar_wait(xw, par)) {
      fail = 12;
      break;
    }
    // LA: the warp's own region; then the stage is free
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int t = sw(tA(lane, warp, r));
      a[r] = spsi[t];
      b[r] = slam[t];
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(sread);
    if (leader) {
      if (!mbar_wait(sread, par)) {
        fail = 13;
        abort_flag = 1;
      } else if (j + 1 < my_tiles) {
        issue(j + 1);
      }
    }
    __syncwarp();
    if (abort_flag) break;
    gates<1>(P, km_sm, a, b, acc);
    // LA -> LB inside the warp's own region of X
#pragma unroll
    for (int r = 0; r < kR; ++r) xbuf[sw(tA(lane, warp, r))] = a[r];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kR; ++r) a[r] = xbuf[sw(tB(lane, warp, r))];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kR; ++r) xbuf[sw(tA(lane, warp, r))] = b[r];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kR; ++r) b[r] = xbuf[sw(tB(lane, warp, r))];
    __syncwarp();
    // LB: tile bits 3..6 (the acc of tile bit tb is acc[tb * kThreads])
    tw::gates_last<3, kThreads>(P, km_sm, a, b, acc + 3 * kThreads);
    const u32 cbase = deposit(P, first + static_cast<u32>(j) * gridDim.x);
#pragma unroll
    for (int r = 0; r < kR; ++r) __stcs(&lam_out[cbase | static_cast<u32>(tB(lane, warp, r))], b[r]);
  }
  if (fail) {
    atomicExch(T.err, fail);
    abort_flag = 1;
  }
  if (leader && abort_flag && loads > 0) {
    // loads this block issued must land before the block exits
    mbar_wait(fullp, static_cast<unsigned>(loads - 1) & 1u);
    mbar_wait(fulll, static_cast<unsigned>(loads - 1) & 1u);
  }
  if (leader) bulk_wait_all();

  __syncthreads();
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const double s = warp_sum(acc[i * kThreads]);
    if (lane == 0) red[warp][i] = s;
  }
  __syncthreads();
  double *rec = P.partials + static_cast<size_t>(blockIdx.x) * kPartialStride;
  if (tid < 12) {
    double s = 0.0;
    for (int ww = 0; ww < kWarps; ++ww) s += red[ww][tid];
    rec[tid] = s;
  }
}

// ------------------------------------------------------------------- host
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

struct MapDim {
  int lo;     // lowest index bit
  int nbits;  // index bits covered
  bool tile;  // spanned by the box (else a coset coordinate)
};

int index_bit(unsigned long long v) {
  int b = 0;
  while (!((v >> b) & 1)) ++b;
  return b;
}

// Appends the runs of consecutive index bits of `bits` (ascending) as box
// dimensions of at most 8 bits.
void push_tile_runs(const std::vector<int> &bits, std::vector<MapDim> &dims) {
  size_t i = 0;
  while (i < bits.size()) {
    size_t k = i + 1;
    while (k < bits.size() && bits[k] == bits[k - 1] + 1 && static_cast<int>(k - i) < 8) ++k;
    dims.push_back({bits[i], static_cast<int>(k - i), true});
    i = k;
  }
}

bool encode(CUtensorMap &map, const void *base, int n, const std::vector<MapDim> &dims, int *shift,
            unsigned *mask, std::string *why) {
  auto fn = encode_fn();
  if (fn == nullptr) {
    if (why) *why = "cuTensorMapEncodeTiled is not available from the driver";
    return false;
  }
  cuuint64_t gdim[kTmaRank], gstride[kTmaRank - 1];
  cuuint32_t box[kTmaRank], estr[kTmaRank];
  for (int d = 0; d < kTmaRank; ++d) {
    estr[d] = 1;
    if (d == 0) {
      gdim[0] = 16;  // doubles of index bits 0..2
      box[0] = 16;
      shift[0] = 0;
      mask[0] = 0;
      continue;
    }
    const cuuint64_t stride = cuuint64_t{16} << (d < static_cast<int>(dims.size()) ? dims[d].lo : n);
    gstride[d - 1] = stride;
    if (d < static_cast<int>(dims.size())) {
      gdim[d] = cuuint64_t{1} << dims[d].nbits;
      box[d] = dims[d].tile ? (1u << dims[d].nbits) : 1u;
      shift[d] = dims[d].lo;
      mask[d] = dims[d].tile ? 0u : static_cast<unsigned>((cuuint64_t{1} << dims[d].nbits) - 1);
    } else {
      gdim[d] = 1;
      box[d] = 1;
      shift[d] = 0;
      mask[d] = 0;
    }
  }
  const CUresult r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, kTmaRank, const_cast<void *>(base), gdim, gstride,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    if (why) *why = "cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")";
    return false;
  }
  return true;
}

// Box dimensions of the load maps (tile-index order) and of the store map
// (tile bits 0..2, 7..10, 3..6, then the coset runs).
bool map_dims(const PassParams &P, std::vector<MapDim> &ld, std::vector<MapDim> &st, std::string *why) {
  const int n = P.n;
  std::vector<int> tb_of(static_cast<size_t>(n), -1);
  for (int b = 0; b < P.tile_bits; ++b) tb_of[static_cast<size_t>(index_bit(P.vec[b]))] = b;
  std::vector<MapDim> coset;
  for (int i = 3; i < n;) {
    const bool tile = tb_of[static_cast<size_t>(i)] >= 0;
    int k = i + 1;
    while (k < n && (tb_of[static_cast<size_t>(k)] >= 0) == tile) ++k;
    if (!tile) coset.push_back({i, k - i, false});
    i = k;
  }
  // load: index order
  ld.clear();
  ld.push_back({0, 3, true});
  {
    std::vector<int> bits;
    size_t ci = 0;
    for (int i = 3; i <= n; ++i) {
      const bool tile = i < n && tb_of[static_cast<size_t>(i)] >= 0;
      if (tile) {
        bits.push_back(i);
        continue;
      }
      if (!bits.empty()) {
        push_tile_runs(bits, ld);
        bits.clear();
      }
      if (i < n && ci < coset.size() && coset[ci].lo == i) ld.push_back(coset[ci++]);
    }
  }
  st.clear();
  st.push_back({0, 3, true});
  if (P.tile_bits == 11) {
    std::vector<int> hi, lo;
    for (int b = 7; b <= 10; ++b) hi.push_back(index_bit(P.vec[b]));
    for (int b = 3; b <= 6; ++b) lo.push_back(index_bit(P.vec[b]));
    push_tile_runs(hi, st);
    push_tile_runs(lo, st);
    for (const auto &c : coset) st.push_back(c);
  }
  if (ld.size() > static_cast<size_t>(kTmaRank) || st.size() > static_cast<size_t>(kTmaRank)) {
    if (why) *why = "the tile needs more than five tensor-map dimensions";
    return false;
  }
  return true;
}

}  // namespace

bool tma_pass_shape_ok(const PassParams &P, std::string *why) {
  auto no = [&](const char *m) {
    if (why) *why = m;
    return false;
  };
  if (P.psi_load != kLoadNatural || P.lam_load != kLoadNatural || P.psi_store != kStoreNone ||
      P.lam_store != kStoreNatural)
    return no("load/store variant not on the TMA kernel");
  if (P.phase != P.phi_grad) return no("phase without phi sums");
  if (P.n < 14 || P.n > 31 || P.num_tiles > 0xFFFFFFFFull) return no("state size out of range");
  if (P.psi_in == nullptr || P.lam_in == nullptr || P.lam_out == nullptr) return no("missing buffer");
  if (P.tile_bits == 12) {
    if (P.phase) return no("low pass with the layer's phase");
    for (int b = 0; b < 12; ++b)
      if (P.vec[b] != (1ull << b)) return no("12-bit tile is not index bits 0..11");
    std::vector<MapDim> ld, st;
    return map_dims(P, ld, st, why);
  }
  if (P.tile_bits != 11) return no("not an 11- or 12-bit tile");
  int prev = -1;
  for (int b = 0; b < 11; ++b) {
    const unsigned long long v = P.vec[b];
    if (v == 0 || (v & (v - 1)) != 0) return no("tile direction is not a unit vector");
    const int bit = index_bit(v);
    if (bit <= prev || bit >= P.n) return no("tile bits not in increasing index order");
    if (b < 3 && bit != b) return no("tile bits 0..2 are not index bits 0..2");
    prev = bit;
  }
  for (int b = 0; b < 3; ++b)
    if (P.gate_wire[b] >= 0) return no("gate on tile bits 0..2");
  if (P.gate_wire[11] >= 0 || P.vec[11] != 0) return no("twelfth tile bit in use");
  std::vector<MapDim> ld, st;
  return map_dims(P, ld, st, why);
}

bool make_tma_pass(const PassParams &P, int *err, TmaPass &out, std::string *why) {
  if (!tma_pass_shape_ok(P, why)) return false;
  std::vector<MapDim> ld, st;
  if (!map_dims(P, ld, st, why)) return false;
  std::memset(&out, 0, sizeof(out));
  int sh[kTmaRank];
  unsigned mk[kTmaRank];
  if (!encode(out.psi_map, P.psi_in, P.n, ld, out.ld_shift, out.ld_mask, why)) return false;
  if (!encode(out.lam_map, P.lam_in, P.n, ld, sh, mk, why)) return false;
  if (P.tile_bits == 11 && !encode(out.out_map, P.lam_out, P.n, st, out.st_shift, out.st_mask, why)) return false;
  out.err = err;
  out.kind = P.tile_bits == 12 ? kTmaLow : kTmaHalf;
  return true;
}

size_t bwd_tma_smem_bytes() { return tw::kSmemBytes; }

namespace {
// dynamic shared memory limit, and the largest shared-memory carveout so that
// two blocks fit on an SM
template <typename K>
cudaError_t configure_tma(K k, std::atomic<unsigned long long> &done) {
  const cudaError_t e = set_smem_limit_once(k, tw::kSmemBytes, done);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
}
}  // namespace

int bwd_tma_blocks_per_sm(int kind) { return kind == kTmaLow ? 1 : 2; }

cudaError_t launch_bwd_tma(const PassParams &P, const TmaPass &T, int grid, cudaStream_t s) {
  static std::atomic<unsigned long long> cfg_phase{0}, cfg_plain{0}, cfg_low{0};
  if (T.kind == kTmaLow) {
    const cudaError_t e = set_smem_limit_once(bwd_tma_low_kernel, tl::kSmemBytes, cfg_low);
    if (e != cudaSuccess) return e;
    bwd_tma_low_kernel<<<grid, tl::kThreads, tl::kSmemBytes, s>>>(P, T);
    return cudaGetLastError();
  }
  if (P.phase || T.phi_only) {
    const cudaError_t e = configure_tma(bwd_tma_kernel<true>, cfg_phase);
    if (e != cudaSuccess) return e;
    bwd_tma_kernel<true><<<grid, tw::kThreads, tw::kSmemBytes, s>>>(P, T);
  } else {
    const cudaError_t e = configure_tma(bwd_tma_kernel<false>, cfg_plain);
    if (e != cudaSuccess) return e;
    bwd_tma_kernel<false><<<grid, tw::kThreads, tw::kSmemBytes, s>>>(P, T);
  }
  return cudaGetLastError();
}

}  // namespace rsv
