// Backward tile pass on 11-bit tiles: 256 threads, two CTAs per SM (sm_100a).
//
// A backward pass whose gates all lie on tile bits 4..11 of its 12-bit tile
// (the "high" passes: tile bits 0..3 are contiguous, ungated index bits) is
// run on the 11-bit sub-tile that drops tile bit 3 into the coset.  Its runs
// of 8 contiguous amplitudes are still whole 128-byte lines, psi and lambda
// of a tile are half as large, and two CTAs share an SM: while one waits at a
// barrier or for its prefetch, the other rotates.  The arithmetic is the one
// of bwd_pass_kernel (rsv_pass.cu); this file only changes the geometry.
//
// Layouts of the 11-bit tile (256 threads x 8 registers):
//   H0: warps -> tile bits 0..2, lanes -> 3..7,             registers -> 8..10
//   H1: warps -> tile bits 0..2, lanes -> 8,9,10,3,4,       registers -> 5..7
//   HA: warps -> tile bits 8..10, lanes -> 0,1,2,5,6,       registers -> 3,4,7
// H0 <-> H1 is a warp-local permutation; H1 -> HA one CTA-wide transpose of
// psi and lambda through the staging buffers, after which the next tile is
// prefetched.  Stores go out from HA (lanes 0..2: whole 128-byte lines).
// Wires are rotated in the order H0 (tile bits 8, 9, 10), H1 (5, 6, 7),
// HA (3, 4); the host's gradient correction follows that order.
#include "rsv_launch.h"
#include "rsv_tile.cuh"

namespace rsv {
namespace {

namespace hw {
constexpr int kT = 256;
constexpr int kR = 8;
constexpr int kWarps = kT / 32;
constexpr int kSize = 2048;

enum Layout { H0 = 0, H1 = 1, HA = 2 };

template <int LY>
__device__ __forceinline__ int tpart(int lane, int warp) {
  if (LY == H0) return warp | (lane << 3);
  if (LY == H1) return warp | ((lane >> 3) << 3) | ((lane & 7) << 8);
  return (lane & 7) | (((lane >> 3) & 3) << 5) | (warp << 8);
}
// tile bit of register bit j
template <int LY>
__host__ __device__ constexpr int rtb(int j) {
  return LY == H0 ? 8 + j : LY == H1 ? 5 + j : (j < 2 ? 3 + j : 7);
}
template <int LY>
__device__ __forceinline__ int roff(int r) {
  return ((r & 1) << rtb<LY>(0)) | (((r >> 1) & 1) << rtb<LY>(1)) | (((r >> 2) & 1) << rtb<LY>(2));
}

// H0 -> H1 through this warp's 256-entry slice (warp-local index: tile bits 3..10)
template <int FROM, int TO>
__device__ __forceinline__ void warp_transpose(double2 *wbuf, int lane, int warp, double2 (&a)[kR]) {
  const int tf = tpart<FROM>(lane, warp), tt = tpart<TO>(lane, warp);
#pragma unroll
  for (int r = 0; r < kR; ++r) wbuf[bw::sw8((tf | roff<FROM>(r)) >> 3)] = a[r];
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kR; ++r) a[r] = wbuf[bw::sw8((tt | roff<TO>(r)) >> 3)];
  __syncwarp();
}

template <int FROM, int TO>
__device__ __forceinline__ void cta_transpose_pair(double2 *sa, double2 *sb, int lane, int warp,
                                                   double2 (&a)[kR], double2 (&b)[kR]) {
  const int tf = tpart<FROM>(lane, warp), tt = tpart<TO>(lane, warp);
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int s = swz(tf | roff<FROM>(r));
    sa[s] = a[r];
    sb[s] = b[r];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const int s = swz(tt | roff<TO>(r));
    a[r] = sa[s];
    b[r] = sb[s];
  }
  __syncthreads();
}

// The rotation and theta sum of bw::gates on the first NJ register bits of LY.
template <int LY, int NJ>
__device__ __forceinline__ void gates(const PassParams &P, const double2 *km_tb, double2 (&a)[kR],
                                      double2 (&b)[kR], double (&acc)[12]) {
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int tb = rtb<LY>(j);
    const int w = P.gate_wire[tb];
    if (w < 0) continue;
    const double2 km = km_tb[tb];
    const double k = km.x;
    double t = acc[tb];
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
    acc[tb] = t;
  }
}

// phi sums in layout H0 (registers -> tile bits 8..10, lanes -> 3..7,
// warps -> 0..2); same bookkeeping as phi_accumulate / phi_reduce of
// rsv_pass.cu.
constexpr int kPhiThr = 4;

__device__ __forceinline__ void phi_accumulate(const PassParams &P, u32 cbase, int lane, int warp,
                                               const double2 (&a)[kR], const double2 (&b)[kR],
                                               double *phi_thr, double (*phi_cos)[32]) {
  double v[kPhiThr] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    const double q = fma(b[r].x, a[r].y, -b[r].y * a[r].x);
    v[0] += q;
#pragma unroll
    for (int j = 0; j < 3; ++j)
      if ((r >> j) & 1) v[1 + j] += q;
  }
#pragma unroll
  for (int j = 0; j < kPhiThr; ++j) phi_thr[j * kT] += v[j];
  const double s = warp_sum(v[0]);
  if (lane < P.n && P.wire_tile_bit[lane] < 0 && ((cbase >> lane) & 1)) phi_cos[warp][lane] += s;
}

__device__ __forceinline__ void phi_reduce(const PassParams &P, int lane, int warp, const double *phi_thr,
                                           double (*phi_cos)[32], double (*red)[12], double *phi_sm) {
  double v[9];
#pragma unroll
  for (int j = 0; j < kPhiThr; ++j) v[j] = phi_thr[j * kT];
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
    for (int ww = 0; ww < kWarps; ++ww) qt += red[ww][0];
    if (w < P.n) {
      const int tb = P.wire_tile_bit[w];
      double add = 0.0;
      if (tb < 0) {
        for (int ww = 0; ww < kWarps; ++ww) add += phi_cos[ww][w];
      } else if (tb >= 8) {
        for (int ww = 0; ww < kWarps; ++ww) add += red[ww][1 + tb - 8];
      } else if (tb >= 3) {
        for (int ww = 0; ww < kWarps; ++ww) add += red[ww][4 + tb - 3];
      } else {
        for (int ww = 0; ww < kWarps; ++ww)
          if ((ww >> tb) & 1) add += red[ww][0];
      }
      phi_sm[w] = add;
    }
    if (w == 31) phi_sm[32] = qt;
  }
  __syncthreads();
}
}  // namespace hw

constexpr size_t kHalfSmem = 3 * hw::kSize * sizeof(double2);

template <int PSRC, int LSRC, int PDST, int LDST, bool PHASE>
__global__ void __launch_bounds__(hw::kT, 2) bwd_half_kernel(const PassParams P) {
  using namespace hw;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage_a = reinterpret_cast<double2 *>(smem_raw);
  double2 *stage_b = stage_a + kSize;
  double2 *trans = stage_b + kSize;
  __shared__ double red[kWarps][12];
  __shared__ double phi_sm[33];
  __shared__ double2 km_sm[12];
  __shared__ double phi_thr_sm[PHASE ? kPhiThr * kT : 1];
  __shared__ double phi_cos[PHASE ? kWarps : 1][32];

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int n = P.n;
  double2 *wbuf = trans + warp * 256;

  // global issue layout: lanes -> tile bits 0..4, warps -> 5..7, registers -> 8..10
  const int tpi = lane | (warp << 5);
  const u32 toffi = thread_offset(P, tpi);
  const u32 v8 = P.vec[8], v9 = P.vec[9], v10 = P.vec[10];
  const u32 toffs = thread_offset(P, tpart<HA>(lane, warp));
  const u32 v3 = P.vec[3], v4 = P.vec[4], v7 = P.vec[7];
  const u32 toffp = thread_offset(P, tpart<H0>(lane, warp));
  u32 poff[kR];  // register offsets of layout H0 (analytic psi)
#pragma unroll
  for (int r = 0; r < kR; ++r) poff[r] = ((r & 1) ? v8 : 0u) ^ ((r & 2) ? v9 : 0u) ^ ((r & 4) ? v10 : 0u);

  double2 ratio[4];
  if (PHASE) {
#pragma unroll
    for (int j = 0; j < 3; ++j) ratio[j] = phase_ratio(P, unit_bit(P.vec[8 + j]));
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
      const u32 p = base ^ ((r & 1) ? v8 : 0u) ^ ((r & 2) ? v9 : 0u) ^ ((r & 4) ? v10 : 0u);
      const int s = swz(tpi | (r << 8));
      if (PSRC != kLoadProductPlain) cp_async16(&stage_a[s], &P.psi_in[source_index<PSRC>(p, n)]);
      cp_async16(&stage_b[s], &P.lam_in[source_index<LSRC>(p, n)]);
    }
    cp_async_commit();
  };
  if (blockIdx.x < num_tiles) issue(blockIdx.x);

  const int th0 = tpart<H0>(lane, warp);
  for (u32 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    double2 a[kR], b[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const int s = swz(th0 | (r << 8));
      if (PSRC != kLoadProductPlain) a[r] = stage_a[s];
      b[r] = stage_b[s];
    }
    const u32 cbase = deposit(P, tile);
    if (PSRC == kLoadProductPlain) {
      const u32 base = cbase ^ toffp;
      table4_regs(P.prod, base, poff, a);
    }
    if (PHASE) {
      // RZ^dagger of the layer (with the layer's factor K) on psi and lambda,
      // then the phi sums
      const double2 ph = table4(P.ptab, cbase ^ toffp);
      const double K = P.lscale[P.layer];
      apply_phase_gray<3, true, true>(make_double2(K * ph.x, K * ph.y), ratio, a, b);
      phi_accumulate(P, cbase, lane, warp, a, b, phi_thr_sm + threadIdx.x, phi_cos);
    }
    gates<H0, 3>(P, km_sm, a, b, acc);
    warp_transpose<H0, H1>(wbuf, lane, warp, a);
    warp_transpose<H0, H1>(wbuf, lane, warp, b);
    gates<H1, 3>(P, km_sm, a, b, acc);
    cta_transpose_pair<H1, HA>(stage_a, stage_b, lane, warp, a, b);
    if (tile + gridDim.x < num_tiles) issue(tile + gridDim.x);
    gates<HA, 2>(P, km_sm, a, b, acc);

    if (PDST != kStoreNone || LDST != kStoreNone) {
      const u32 base = cbase ^ toffs;
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const u32 p = base ^ ((r & 1) ? v3 : 0u) ^ ((r & 2) ? v4 : 0u) ^ ((r & 4) ? v7 : 0u);
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
    for (int ww = 0; ww < kWarps; ++ww) s += red[ww][threadIdx.x];
    rec[threadIdx.x] = s;
  }
  if (PHASE) {
    __syncthreads();  // red is reused
    phi_reduce(P, lane, warp, phi_thr_sm + threadIdx.x, phi_cos, red, phi_sm);
    if (threadIdx.x < 31) rec[kPartialPhi + threadIdx.x] = phi_sm[threadIdx.x];
    if (threadIdx.x == 31) rec[kPartialTot] = phi_sm[32];
  }
}

template <int PSRC, int LSRC, int PDST, int LDST, bool PHASE>
cudaError_t launch_half(const PassParams &P, int grid, cudaStream_t s) {
  auto k = bwd_half_kernel<PSRC, LSRC, PDST, LDST, PHASE>;
  static std::atomic<unsigned long long> configured{0};
  {
    const cudaError_t e = set_smem_limit_once(k, kHalfSmem, configured);
    if (e != cudaSuccess) return e;
  }
  k<<<grid, hw::kT, kHalfSmem, s>>>(P);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_bwd_half(const PassParams &P, int grid, cudaStream_t s) {
  const bool phase = P.phase != 0;
  if (P.phi_grad != P.phase) return cudaErrorInvalidValue;
  // gates only on tile bits 3..10 of the 11-bit tile
  for (int b = 0; b < 3; ++b)
    if (P.gate_wire[b] >= 0) return cudaErrorInvalidValue;
  if (P.gate_wire[11] >= 0 || P.vec[11] != 0) return cudaErrorInvalidValue;
  const int pl = P.psi_load, ll = P.lam_load, ps = P.psi_store, ls = P.lam_store;
#define RSV_HALF(PL, LL, PS, LS)                                                     \
  if (pl == PL && ll == LL && ps == PS && ls == LS)                                  \
    return phase ? launch_half<PL, LL, PS, LS, true>(P, grid, s)                     \
                 : launch_half<PL, LL, PS, LS, false>(P, grid, s);
  RSV_HALF(kLoadNatural, kLoadNatural, kStoreNatural, kStoreNatural)
  RSV_HALF(kLoadNatural, kLoadGatherP, kStoreNatural, kStoreNatural)
  RSV_HALF(kLoadNatural, kLoadNatural, kStoreNone, kStoreNatural)
  RSV_HALF(kLoadGatherP, kLoadGatherP, kStoreNone, kStoreNatural)
  RSV_HALF(kLoadProductPlain, kLoadGatherP, kStoreNone, kStoreNatural)
  RSV_HALF(kLoadProductPlain, kLoadNatural, kStoreNone, kStoreNatural)
#undef RSV_HALF
  return cudaErrorInvalidValue;
}

}  // namespace rsv
