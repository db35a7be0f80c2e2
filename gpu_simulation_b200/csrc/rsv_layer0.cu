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
// n >= 13).  Per tile, with c(p) = conj(lambda0(p)) split as c(h, a) (a = bits
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

constexpr int kL0Threads = 512;
constexpr int kL0Tile = 4096;
constexpr int kL0Per = kL0Tile / kL0Threads;  // 8 loads per thread and tile

// stage slot of tile index i: the X2 sums read i = a + 64 h across lanes h
__device__ __forceinline__ int l0_slot(int i) { return i ^ ((i >> 6) & 7); }

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

__global__ void __launch_bounds__(kL0Threads, 1) layer0_grad_kernel(const Layer0Params Q) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage = reinterpret_cast<double2 *>(smem_raw);  // [2][kL0Tile]
  __shared__ double2 amp[32][2];      // a_w(b)
  __shared__ double2 w1[64], w2[64];  // products over wires 0..5 / 6..11
  __shared__ double2 loo[12][64];     // loo[j][x]: w1 (j < 6) or w2 (j >= 6) without wire j
  __shared__ double2 xp[4][128];      // partial X1 (0..63) / X2 (64..127) sums
  __shared__ double2 lsum[25];        // L_w(b) at 2w + b, T at 24

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = Q.n;
  if (t < 64) {
    const int w = t >> 1, b = t & 1;
    double2 v = make_double2(b ? 0.0 : 1.0, 0.0);  // wires >= n: |0> (not used for n >= 13)
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

  const u64 num_tiles = Q.num_tiles;
  auto issue = [&](u64 tile, double2 *buf) {
    if (tile < num_tiles) {
      const u64 base = tile << 12;
#pragma unroll
      for (int r = 0; r < kL0Per; ++r) {
        const int tau = t + r * kL0Threads;
        const u64 p = base | static_cast<u64>(tau);
        const u64 src = Q.gather ? ring_p(p, n) : p;
        cp_async16(&buf[l0_slot(tau)], &Q.lam[src]);
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x, stage);
  issue(blockIdx.x + gridDim.x, stage + kL0Tile);

  // accumulators: lane l of warp 0 keeps S_l(0), S_l(1)
  double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
  int k = 0;
  for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x, ++k) {
    double2 *buf = stage + (k & 1) * kL0Tile;
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();
    {
      // partial X1 / X2: q = warp group (4 x 4 warps), o = output
      const int q = t >> 7, o = t & 127;
      double2 acc = make_double2(0.0, 0.0);
      if (o < 64) {
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
          const int h = 16 * q + kk;
          acc = cadd(acc, cjmul(buf[l0_slot(o + 64 * h)], w2[h]));
        }
      } else {
        const int h = o - 64;
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
          const int a = 16 * q + kk;
          acc = cadd(acc, cjmul(buf[l0_slot(a + 64 * h)], w1[a]));
        }
      }
      xp[q][o] = acc;
    }
    __syncthreads();
    // buf is free: prefetch the tile after next
    issue(tile + 2 * static_cast<u64>(gridDim.x), buf);
    for (int out = warp; out < 25; out += kL0Threads / 32) {
      // output 2w + b (w < 12) -> L_w(b); 24 -> T
      double2 v = make_double2(0.0, 0.0);
      if (out < 24) {
        const int w = out >> 1, b = out & 1;
        const int off = w < 6 ? 0 : 64;
        const int bit = w < 6 ? w : w - 6;
        // the 32 indices x of the 6-bit half with bit `bit` = b
        const int lo = lane & ((1 << bit) - 1), hi = lane >> bit;
        const int x = lo | (b << bit) | (hi << (bit + 1));
        const double2 X = cadd(cadd(xp[0][off + x], xp[1][off + x]), cadd(xp[2][off + x], xp[3][off + x]));
        v = cmul(X, loo[w][x]);
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int x = lane + 32 * h;
          const double2 X = cadd(cadd(xp[0][x], xp[1][x]), cadd(xp[2][x], xp[3][x]));
          v = cadd(v, cmul(X, w1[x]));
        }
      }
      v = warp_sum2(v);
      if (lane == 0) lsum[out] = v;
    }
    __syncthreads();
    if (warp == 0) {
      // coset factors of this tile (wires 12..n-1)
      const u64 cb = tile << 12;
      double2 all = make_double2(1.0, 0.0), others = make_double2(1.0, 0.0);
      for (int v = 12; v < n; ++v) {
        const double2 A = amp[v][(cb >> v) & 1];
        all = cmul(all, A);
        if (v != lane) others = cmul(others, A);
      }
      if (lane < 12) {
        s0 = cadd(s0, cmul(all, lsum[2 * lane]));
        s1 = cadd(s1, cmul(all, lsum[2 * lane + 1]));
      } else if (lane < n) {
        const double2 c = cmul(others, lsum[24]);
        if ((cb >> lane) & 1) s1 = cadd(s1, c);
        else s0 = cadd(s0, c);
      }
    }
  }
  cp_async_wait_all();
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

size_t layer0_smem_bytes() { return 2 * kL0Tile * sizeof(double2); }

cudaError_t launch_layer0_grad(const Layer0Params &Q, int grid, cudaStream_t s) {
  if (Q.n < 13 || Q.n > 31 || grid < 1) return cudaErrorInvalidValue;
  static bool configured = false;
  if (!configured) {
    const cudaError_t e = cudaFuncSetAttribute(layer0_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(layer0_smem_bytes()));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  layer0_grad_kernel<<<grid, kL0Threads, layer0_smem_bytes(), s>>>(Q);
  return cudaGetLastError();
}

cudaError_t launch_layer0_finalize(const Layer0Params &Q, int grid, double *grad_out, cudaStream_t s) {
  layer0_finalize_kernel<<<1, 32, 0, s>>>(Q, grid, grad_out);
  return cudaGetLastError();
}

}  // namespace rsv
