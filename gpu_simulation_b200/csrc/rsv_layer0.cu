// Layer-0 gradients in one read-only pass over lambda (sm_100a).
//
// Layer 0 acts on |0...0>, so its output is the product state
//   psi0(p) = prod_w a_w(p_w),   a_w = RZ(phi_w) RY(theta_w) |0> = (c e^{-i phi/2}, s e^{+i phi/2})
// (c, s = cos, sin of theta_w / 2; p in the frame of layer 0 before its CNOT
// ring).  With lambda0 = the adjoint state at that point, the gradient of a
// layer-0 parameter x of wire w is 2 Re <lambda0 | d_x psi0>, and d_x psi0
// differs from psi0 only in the factor of wire w:
//   <lambda0 | d_x psi0> = sum_b d_x a_w(b) S_w(b),
//   S_w(b) = sum over p with p_w = b of conj(lambda0(p)) prod_{v != w} a_v(p_v).
// The reference gets these by walking layer 0 backwards gate by gate
// (cpp/ising_cuda_statevector_grad_kernels.cu:223-319 per wire, scheduled by
// cpp/ising_cuda_structured_adjoint_modes.inc:272-307); here all 2n sums come
// from one pass that only reads lambda.
//
// Tiles are 4096 contiguous indices p (index bits 0..11; coset = bits 12..n-1,
// n >= 13), loaded straight into registers (two 256-thread CTAs per SM).  Per tile, with c(p) = conj(lambda0(p)) split as c(h, a) (a = bits
// 0..5, h = bits 6..11):
//   X1(a) = sum_h c(h, a) W2(h),  X2(h) = sum_a c(h, a) W1(a)
// (W1, W2 = products of a_v over wires 0..5 and 6..11), then the in-tile
// leave-one-out sums L_w(b) for w < 12 from X1 / X2 (6-bit contractions), the
// full contraction T = sum_a X1(a) W1(a), and the coset factors A_v = a_v(p_v)
// (v >= 12, constant on the tile):
//   S_w(b) += (prod_v A_v) L_w(b)            (w < 12)
//   S_v(p_v) += (prod_{u != v} A_u) T         (v >= 12)
// Per-CTA sums are reduced in a fixed order by layer0_finalize_kernel.
#include "rsv_launch.h"
#include "rsv_tile.cuh"

namespace rsv {
namespace {

constexpr int kL0Threads = 256;
constexpr int kL0Warps = kL0Threads / 32;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
// conj(x) * w
__device__ __forceinline__ double2 cjmul(double2 x, double2 w) {
  return make_double2(fma(x.x, w.x, x.y * w.y), fma(x.x, w.y, -x.y * w.x));
}

__device__ __forceinline__ double2 shfl_xor2(double2 v, int m) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v = cadd(v, shfl_xor2(v, m));
  return v;
}

// Thread (lane, warp) holds c(a, h) for a = lane + 32 a5 (a5 = 0, 1) and
// h = 8 warp + j (j = 0..7): rows of 32 contiguous amplitudes per load.
__global__ void __launch_bounds__(kL0Threads, 2) layer0_grad_kernel(const Layer0Params Q) {
  __shared__ double2 amp[32][2];          // a_w(b)
  __shared__ double2 w1[64], w2[64];      // products over wires 0..5 / 6..11
  __shared__ double2 loo[12][64];         // loo[j][x]: w1 (j < 6) or w2 (j >= 6) without wire j
  __shared__ double2 x1p[kL0Warps][64];   // per-warp partial X1
  __shared__ double2 x2s[64];             // X2
  __shared__ double2 lsum[25];            // L_w(b) at 2w + b, T at 24

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = Q.n;
  if (t < 64) {
    const int w = t >> 1, b = t & 1;
    double2 v = make_double2(b ? 0.0 : 1.0, 0.0);
    if (w < n) {
      const double4 k = Q.coef[w];
      // (c e^{-i phi/2}, s e^{+i phi/2})
      v = b ? make_double2(k.y * k.z, k.y * k.w) : make_double2(k.x * k.z, -k.x * k.w);
    }
    amp[w][b] = v;
  }
  __syncthreads();
  if (t < 128) {
    const int half = t >> 6, x = t & 63;  // half 0: wires 0..5, 1: wires 6..11
    double2 p = make_double2(1.0, 0.0);
    for (int j = 0; j < 6; ++j) p = cmul(p, amp[6 * half + j][(x >> j) & 1]);
    (half ? w2 : w1)[x] = p;
  }
  for (int e = t; e < 12 * 64; e += kL0Threads) {
    const int j = e >> 6, x = e & 63, half = j / 6;
    double2 p = make_double2(1.0, 0.0);
    for (int jj = 0; jj < 6; ++jj)
      if (6 * half + jj != j) p = cmul(p, amp[6 * half + jj][(x >> jj) & 1]);
    loo[j][x] = p;
  }
  __syncthreads();
  // this thread's weights: W1 of its two a, W2 of its eight h
  const double2 wa0 = w1[lane], wa1 = w1[lane + 32];
  double2 wh[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) wh[j] = w2[8 * warp + j];

  // accumulators: lane l of warp 0 keeps S_l(0), S_l(1)
  double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
  const u64 num_tiles = Q.num_tiles;
  for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const u64 base = tile << 12;
    double2 c[2][8];
#pragma unroll
    for (int a5 = 0; a5 < 2; ++a5)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const u64 p = base | static_cast<u64>(lane + 32 * a5 + 64 * (8 * warp + j));
        c[a5][j] = __ldcs(&Q.lam[Q.gather ? ring_p(p, n) : p]);
      }
    // X1 partials (sum over this warp's eight h) and X2 rows (sum over the 64 a)
    double2 x1a = make_double2(0.0, 0.0), x1b = make_double2(0.0, 0.0);
    double2 x2[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      x1a = cadd(x1a, cjmul(c[0][j], wh[j]));
      x1b = cadd(x1b, cjmul(c[1][j], wh[j]));
      x2[j] = cadd(cjmul(c[0][j], wa0), cjmul(c[1][j], wa1));
    }
    // reduce-scatter the eight X2 rows over the lanes: after the three
    // exchanges lane l holds row j = l >> 2 summed over 8 lanes
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int m = 16 >> s, cnt = 4 >> s;
      const bool up = (lane & m) != 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (q < cnt) {
          const double2 send = up ? x2[q] : x2[q + cnt];
          const double2 keep = up ? x2[q + cnt] : x2[q];
          x2[q] = cadd(keep, shfl_xor2(send, m));
        }
      }
    }
    double2 xr = cadd(x2[0], shfl_xor2(x2[0], 1));
    xr = cadd(xr, shfl_xor2(xr, 2));
    __syncthreads();  // the previous tile's readers of x1p / x2s / lsum are done
    x1p[warp][lane] = x1a;
    x1p[warp][lane + 32] = x1b;
    if ((lane & 3) == 0) x2s[8 * warp + (lane >> 2)] = xr;
    __syncthreads();
    for (int out = warp; out < 25; out += kL0Warps) {
      // output 2w + b (w < 12) -> L_w(b); 24 -> T
      double2 v = make_double2(0.0, 0.0);
      if (out < 24) {
        const int w = out >> 1, b = out & 1;
        const int bit = w < 6 ? w : w - 6;
        // the 32 indices x of the 6-bit half with bit `bit` = b
        const int lo = lane & ((1 << bit) - 1), hi = lane >> bit;
        const int x = lo | (b << bit) | (hi << (bit + 1));
        double2 X;
        if (w < 6) {
          X = x1p[0][x];
#pragma unroll
          for (int ww = 1; ww < kL0Warps; ++ww) X = cadd(X, x1p[ww][x]);
        } else {
          X = x2s[x];
        }
        v = cmul(X, loo[w][x]);
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int x = lane + 32 * h;
          double2 X = x1p[0][x];
#pragma unroll
          for (int ww = 1; ww < kL0Warps; ++ww) X = cadd(X, x1p[ww][x]);
          v = cadd(v, cmul(X, w1[x]));
        }
      }
      v = warp_sum2(v);
      if (lane == 0) lsum[out] = v;
    }
    __syncthreads();
    if (warp == 0) {
      // coset factors of this tile (wires 12..n-1)
      double2 all = make_double2(1.0, 0.0), others = make_double2(1.0, 0.0);
      for (int v = 12; v < n; ++v) {
        const double2 A = amp[v][(base >> v) & 1];
        all = cmul(all, A);
        if (v != lane) others = cmul(others, A);
      }
      if (lane < 12) {
        s0 = cadd(s0, cmul(all, lsum[2 * lane]));
        s1 = cadd(s1, cmul(all, lsum[2 * lane + 1]));
      } else if (lane < n) {
        const double2 cc = cmul(others, lsum[24]);
        if ((base >> lane) & 1) s1 = cadd(s1, cc);
        else s0 = cadd(s0, cc);
      }
    }
  }
  if (warp == 0) {
    double *rec = Q.partials + static_cast<size_t>(blockIdx.x) * kLayer0Stride;
    rec[4 * lane + 0] = s0.x;
    rec[4 * lane + 1] = s0.y;
    rec[4 * lane + 2] = s1.x;
    rec[4 * lane + 3] = s1.y;
  }
}

// grad[2w] (theta) and grad[2w+1] (phi) of layer 0, from the per-CTA sums:
//   d_theta a_w = (-s/2 e^{-i phi/2}, c/2 e^{+i phi/2}),
//   d_phi a_w   = (-i/2 c e^{-i phi/2}, i/2 s e^{+i phi/2}).
__global__ void layer0_finalize_kernel(const Layer0Params Q, int grid, double *grad_out) {
  const int w = threadIdx.x;
  if (w >= Q.n) return;
  double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
  for (int c = 0; c < grid; ++c) {
    const double *rec = Q.partials + static_cast<size_t>(c) * kLayer0Stride + 4 * w;
    s0 = cadd(s0, make_double2(rec[0], rec[1]));
    s1 = cadd(s1, make_double2(rec[2], rec[3]));
  }
  const double4 k = Q.coef[w];
  const double2 em = make_double2(k.z, -k.w), ep = make_double2(k.z, k.w);  // e^{-+i phi/2}
  const double2 dt0 = make_double2(-0.5 * k.y * em.x, -0.5 * k.y * em.y);
  const double2 dt1 = make_double2(0.5 * k.x * ep.x, 0.5 * k.x * ep.y);
  const double2 a0 = make_double2(k.x * em.x, k.x * em.y), a1 = make_double2(k.y * ep.x, k.y * ep.y);
  const double2 dp0 = make_double2(0.5 * a0.y, -0.5 * a0.x);   // -i/2 a0
  const double2 dp1 = make_double2(-0.5 * a1.y, 0.5 * a1.x);   // +i/2 a1
  grad_out[2 * w] = 2.0 * (cmul(dt0, s0).x + cmul(dt1, s1).x);
  grad_out[2 * w + 1] = 2.0 * (cmul(dp0, s0).x + cmul(dp1, s1).x);
}

}  // namespace

cudaError_t launch_layer0_grad(const Layer0Params &Q, int grid, cudaStream_t s) {
  if (Q.n < 13 || Q.n > 31 || grid < 1) return cudaErrorInvalidValue;
  layer0_grad_kernel<<<grid, kL0Threads, 0, s>>>(Q);
  return cudaGetLastError();
}

cudaError_t launch_layer0_finalize(const Layer0Params &Q, int grid, double *grad_out, cudaStream_t s) {
  layer0_finalize_kernel<<<1, 32, 0, s>>>(Q, grid, grad_out);
  return cudaGetLastError();
}

}  // namespace rsv
