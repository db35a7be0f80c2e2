// Gradients of layers 0 and 1 from one read of lambda (sm_100a).
//
// Layers 0 and 1 act on |0...0>.  Writing q for the index after layer 0's
// rotations, the ring P turns q into prefix parities s_w = q_0 ^ ... ^ q_w
// (bit 0 of P(q) is s_{n-1} ^ s_0), so layer 1's output before its ring is a
// periodic matrix-product state of bond dimension 2:
//   chi1(r) = Tr( T_0[r_0] T_1[r_1] ... T_{n-1}[r_{n-1}] ),
//   T_w[b](x, y) = U1_w[b, y] a_w(x ^ y)        (w >= 1),
//   T_0[b](x, y) = U1_0[b, x ^ y] a_0(y),
// with a_w = U0_w |0> (layer 0) and U1_w = RZ(phi) RY(theta) of layer 1
// (x = s_{w-1}, y = s_w; the bond closes around the ring).  A parameter of
// wire w enters T_w only, so with lambda1 the adjoint state at that point
//   d E / d x = 2 Re sum_b Tr( d_x T_w[b] E_w[b] ),
//   E_w[b] = sum over r with r_w = b of conj(lambda1(r)) R_w(r),
// R_w the cyclic product of the other T's starting after w.  The reference
// reaches these gradients by walking layers 1 and 0 back gate by gate
// (cpp/ising_cuda_statevector_grad_kernels.cu:223-319, scheduled by
// cpp/ising_cuda_structured_adjoint_modes.inc:272-307); the sums are the same.
//
// One pass over lambda1 (gathered through P from layer 2's backward output,
// or the energy's lambda when L = 2).  Tiles are 4096 contiguous r (bits
// 0..11; a = bits 0..5, h = bits 6..11; coset = bits 12..n-1, n >= 13).  Per
// tile, with M1(a) = T_0..T_5, M2(h) = T_6..T_11 and C = T_12..T_{n-1}:
//   X1(a) = sum_h conj(lambda) M2(h),  X2(h) = sum_a conj(lambda) M1(a),
//   G(a) += X1(a) C,  F(h) += C X2(h),  Z = sum_a M1(a) X1(a),
//   E_v[r_v] += (T_{v+1}..T_{n-1}) Z (T_12..T_{v-1})      (coset wires v).
// The in-tile environments follow once at the end:
//   E_w[b] = sum_{a: a_w = b} (T_{w+1}..T_5)(a) G(a) (T_0..T_{w-1})(a)   (w < 6),
// and likewise from F for 6 <= w < 12 (grad01_finalize_kernel).
#include "rsv_launch.h"
#include "rsv_tile.cuh"

namespace rsv {
namespace {

constexpr int kG01Threads = 256;
constexpr int kG01Tile = 4096;

struct M2x2 {
  double2 m[4];  // row-major (x, y)
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // a * b + c
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// conj(x) * w + c
__device__ __forceinline__ double2 cjfma(double2 x, double2 w, double2 c) {
  return make_double2(fma(x.x, w.x, fma(x.y, w.y, c.x)), fma(x.x, w.y, fma(-x.y, w.x, c.y)));
}
__device__ __forceinline__ M2x2 mmul(const M2x2 &A, const M2x2 &B) {
  M2x2 R;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) R.m[2 * i + j] = cfma(A.m[2 * i + 1], B.m[2 + j], cmul(A.m[2 * i], B.m[j]));
  return R;
}
__device__ __forceinline__ M2x2 ident() {
  M2x2 R;
  R.m[0] = make_double2(1.0, 0.0);
  R.m[1] = make_double2(0.0, 0.0);
  R.m[2] = make_double2(0.0, 0.0);
  R.m[3] = make_double2(1.0, 0.0);
  return R;
}
__device__ __forceinline__ M2x2 shfl_up_m(const M2x2 &A, int d) {
  M2x2 R;
#pragma unroll
  for (int e = 0; e < 4; ++e)
    R.m[e] = make_double2(__shfl_up_sync(0xffffffffu, A.m[e].x, d), __shfl_up_sync(0xffffffffu, A.m[e].y, d));
  return R;
}
__device__ __forceinline__ M2x2 shfl_down_m(const M2x2 &A, int d) {
  M2x2 R;
#pragma unroll
  for (int e = 0; e < 4; ++e)
    R.m[e] = make_double2(__shfl_down_sync(0xffffffffu, A.m[e].x, d), __shfl_down_sync(0xffffffffu, A.m[e].y, d));
  return R;
}

// Layer-0 amplitudes a(b), layer-1 gate U[b][y] of wire w and their
// derivatives (kind 0: none, 1: d theta0, 2: d phi0, 3: d theta1, 4: d phi1).
struct WireGates {
  double2 a[2], u[2][2];
};
__device__ __forceinline__ WireGates wire_gates(const double4 *coef, int n, int w, int kind) {
  const double4 k0 = coef[w], k1 = coef[n + w];
  const double2 em0 = make_double2(k0.z, -k0.w), ep0 = make_double2(k0.z, k0.w);
  const double2 em1 = make_double2(k1.z, -k1.w), ep1 = make_double2(k1.z, k1.w);
  double c0 = k0.x, s0 = k0.y, c1 = k1.x, s1 = k1.y;
  WireGates g;
  // a = (c0 e^{-i phi0/2}, s0 e^{+i phi0/2}); U = RZ(phi1) RY(theta1)
  double ca0 = c0, sa0 = s0, cu = c1, su = s1;
  if (kind == 1) {
    ca0 = -0.5 * s0;
    sa0 = 0.5 * c0;
  }
  if (kind == 3) {
    cu = -0.5 * s1;
    su = 0.5 * c1;
  }
  g.a[0] = make_double2(ca0 * em0.x, ca0 * em0.y);
  g.a[1] = make_double2(sa0 * ep0.x, sa0 * ep0.y);
  if (kind == 2) {  // d/dphi0: -i/2 on |0>, +i/2 on |1>
    g.a[0] = make_double2(0.5 * g.a[0].y, -0.5 * g.a[0].x);
    g.a[1] = make_double2(-0.5 * g.a[1].y, 0.5 * g.a[1].x);
  }
  // RY(theta) = [[c, -s], [s, c]]; its theta-derivative = [[-s/2, -c/2], [c/2, -s/2]]
  // (cu, su) above carry the derivative's (c, s) pattern: [[cu, -su], [su, cu]]
  g.u[0][0] = make_double2(cu * em1.x, cu * em1.y);
  g.u[0][1] = make_double2(-su * em1.x, -su * em1.y);
  g.u[1][0] = make_double2(su * ep1.x, su * ep1.y);
  g.u[1][1] = make_double2(cu * ep1.x, cu * ep1.y);
  if (kind == 4) {  // d/dphi1: row 0 times -i/2, row 1 times +i/2
#pragma unroll
    for (int y = 0; y < 2; ++y) {
      g.u[0][y] = make_double2(0.5 * g.u[0][y].y, -0.5 * g.u[0][y].x);
      g.u[1][y] = make_double2(-0.5 * g.u[1][y].y, 0.5 * g.u[1][y].x);
    }
  }
  return g;
}
// T_w[b] (or its derivative) from the wire's gates
__device__ __forceinline__ M2x2 tmat(const WireGates &g, int w, int b) {
  M2x2 T;
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y) T.m[2 * x + y] = w >= 1 ? cmul(g.u[b][y], g.a[x ^ y]) : cmul(g.u[b][x ^ y], g.a[y]);
  return T;
}

// stage slot of tile index i: the X2 sums read i = a + 64 h across threads h
__device__ __forceinline__ int g01_slot(int i) { return i ^ ((i >> 6) & 7); }

__global__ void __launch_bounds__(kG01Threads, 2) grad01_kernel(const Grad01Params Q) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage = reinterpret_cast<double2 *>(smem_raw);  // [kG01Tile]
  __shared__ M2x2 tm[32][2];   // T_w[b], identity for w >= n
  __shared__ M2x2 m1[64], m2[64];
  __shared__ double2 x1[64][4], x2[64][4];
  __shared__ double2 zp[kG01Threads / 32][4];
  __shared__ M2x2 csm;

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = Q.n;
  if (t < 64) {
    const int w = t >> 1, b = t & 1;
    tm[w][b] = w < n ? tmat(wire_gates(Q.coef, n, w, 0), w, b) : ident();
  }
  __syncthreads();
  if (t < 128) {
    const int half = t >> 6, x = t & 63;
    M2x2 p = tm[6 * half][x & 1];
    for (int j = 1; j < 6; ++j) p = mmul(p, tm[6 * half + j][(x >> j) & 1]);
    (half ? m2 : m1)[x] = p;
  }
  __syncthreads();

  const int idx = t >> 2, e = t & 3, ei = e >> 1, ej = e & 1;
  double2 g = make_double2(0.0, 0.0), f = make_double2(0.0, 0.0);
  M2x2 E0, E1;  // warp 0, coset lanes: E_v[0], E_v[1]
#pragma unroll
  for (int q = 0; q < 4; ++q) E0.m[q] = E1.m[q] = make_double2(0.0, 0.0);

  const u64 num_tiles = Q.num_tiles;
  auto issue = [&](u64 tile) {
    if (tile < num_tiles) {
      const u64 base = tile << 12;
#pragma unroll
      for (int r = 0; r < kG01Tile / kG01Threads; ++r) {
        const int tau = t + r * kG01Threads;
        const u64 p = base | static_cast<u64>(tau);
        cp_async16(&stage[g01_slot(tau)], &Q.lam[Q.gather ? ring_p(p, n) : p]);
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x);

  for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    const u64 base = tile << 12;
    cp_async_wait_all();
    __syncthreads();
    {
      double2 acc1 = make_double2(0.0, 0.0), acc2 = make_double2(0.0, 0.0);
#pragma unroll 8
      for (int k = 0; k < 64; ++k) {
        acc1 = cjfma(stage[g01_slot(idx + 64 * k)], m2[k].m[e], acc1);  // a = idx, h = k
        acc2 = cjfma(stage[g01_slot(k + 64 * idx)], m1[k].m[e], acc2);  // a = k, h = idx
      }
      x1[idx][e] = acc1;
      x2[idx][e] = acc2;
    }
    __syncthreads();
    issue(tile + gridDim.x);  // the stage is free
    // Z partial: thread (a = idx, e = (i, j)) -> sum_k M1(a)[i][k] X1(a)[k][j]
    {
      double2 z = cfma(m1[idx].m[2 * ei + 1], x1[idx][2 + ej], cmul(m1[idx].m[2 * ei], x1[idx][ej]));
#pragma unroll
      for (int m = 4; m < 32; m <<= 1)
        z = cadd(z, make_double2(__shfl_xor_sync(0xffffffffu, z.x, m), __shfl_xor_sync(0xffffffffu, z.y, m)));
      if (lane < 4) zp[warp][lane] = z;
    }
    // coset products (warp 0): lane v holds T_v[r_v] for 12 <= v < n, identity elsewhere
    M2x2 cpre, cpost;
    if (warp == 0) {
      const M2x2 tv = (lane >= 12 && lane < n) ? tm[lane][(base >> lane) & 1] : ident();
      M2x2 pre = tv, suf = tv;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const M2x2 o = shfl_up_m(pre, d);
        if (lane >= d) pre = mmul(o, pre);
        const M2x2 s = shfl_down_m(suf, d);
        if (lane + d < 32) suf = mmul(suf, s);
      }
      // exclusive products: T_12..T_{v-1} and T_{v+1}..T_{n-1}
      cpre = shfl_up_m(pre, 1);
      cpost = shfl_down_m(suf, 1);
      if (lane == 0) cpre = ident();
      if (lane == 31) cpost = ident();
      if (lane == 31) csm = pre;  // C = T_12..T_{n-1}
    }
    __syncthreads();
    const M2x2 C = csm;
    g = cfma(x1[idx][2 * ei + 1], C.m[2 + ej], cfma(x1[idx][2 * ei], C.m[ej], g));
    f = cfma(C.m[2 * ei + 1], x2[idx][2 + ej], cfma(C.m[2 * ei], x2[idx][ej], f));
    if (warp == 0 && lane >= 12 && lane < n) {
      M2x2 Z;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double2 s = zp[0][q];
        for (int ww = 1; ww < kG01Threads / 32; ++ww) s = cadd(s, zp[ww][q]);
        Z.m[q] = s;
      }
      const M2x2 add = mmul(mmul(cpost, Z), cpre);
      M2x2 &Ed = ((base >> lane) & 1) ? E1 : E0;
#pragma unroll
      for (int q = 0; q < 4; ++q) Ed.m[q] = cadd(Ed.m[q], add.m[q]);
    }
  }
  cp_async_wait_all();
  double *rec = Q.partials + static_cast<size_t>(blockIdx.x) * kGrad01Stride;
  rec[2 * t] = g.x;
  rec[2 * t + 1] = g.y;
  rec[512 + 2 * t] = f.x;
  rec[512 + 2 * t + 1] = f.y;
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      rec[1024 + 16 * lane + 2 * q] = E0.m[q].x;
      rec[1024 + 16 * lane + 2 * q + 1] = E0.m[q].y;
      rec[1024 + 16 * lane + 8 + 2 * q] = E1.m[q].x;
      rec[1024 + 16 * lane + 8 + 2 * q + 1] = E1.m[q].y;
    }
  }
}

// Fixed-order reduction of the per-CTA records, the in-tile environments and
// the 4n gradients of layers 0 and 1: grad[2w], grad[2w+1] (layer 0) and
// grad[2(n+w)], grad[2(n+w)+1] (layer 1).
__global__ void __launch_bounds__(256) grad01_finalize_kernel(const Grad01Params Q, int grid, double *grad_out) {
  __shared__ double2 tot[768];  // G(a)[e] at 4a + e, F(h)[e] at 256 + 4h + e, coset E at 512 + 8v + 4b + e
  __shared__ M2x2 tm[32][2];
  const int t = threadIdx.x, n = Q.n;
  for (int i = t; i < 768; i += blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < grid; ++c) {
      const double *rec = Q.partials + static_cast<size_t>(c) * kGrad01Stride;
      s = cadd(s, make_double2(rec[2 * i], rec[2 * i + 1]));
    }
    tot[i] = s;
  }
  if (t < 64) {
    const int w = t >> 1, b = t & 1;
    tm[w][b] = w < n ? tmat(wire_gates(Q.coef, n, w, 0), w, b) : ident();
  }
  __syncthreads();
  const int w = t;
  if (w >= n) return;
  M2x2 E[2];
  if (w < 12) {
    const int lo = w < 6 ? 0 : 6, off = w < 6 ? 0 : 256, bit = w - lo;
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int q = 0; q < 4; ++q) E[b].m[q] = make_double2(0.0, 0.0);
    for (int x = 0; x < 64; ++x) {
      const int b = (x >> bit) & 1;
      M2x2 pre = ident(), post = ident(), X;
      for (int j = 0; j < bit; ++j) pre = mmul(pre, tm[lo + j][(x >> j) & 1]);
      for (int j = bit + 1; j < 6; ++j) post = mmul(post, tm[lo + j][(x >> j) & 1]);
#pragma unroll
      for (int q = 0; q < 4; ++q) X.m[q] = tot[off + 4 * x + q];
      const M2x2 add = mmul(mmul(post, X), pre);
#pragma unroll
      for (int q = 0; q < 4; ++q) E[b].m[q] = cadd(E[b].m[q], add.m[q]);
    }
  } else {
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int q = 0; q < 4; ++q) E[b].m[q] = tot[512 + 8 * w + 4 * b + q];
  }
  double out[4];
#pragma unroll
  for (int kind = 1; kind <= 4; ++kind) {
    const WireGates dg = wire_gates(Q.coef, n, w, kind);
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const M2x2 dT = tmat(dg, w, b);
      // Re Tr(dT E) = Re sum_{x,y} dT(x, y) E(y, x)
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y) s += cmul(dT.m[2 * x + y], E[b].m[2 * y + x]).x;
    }
    out[kind - 1] = 2.0 * s;
  }
  grad_out[2 * w] = out[0];
  grad_out[2 * w + 1] = out[1];
  grad_out[2 * (n + w)] = out[2];
  grad_out[2 * (n + w) + 1] = out[3];
}

size_t grad01_smem_bytes() { return kG01Tile * sizeof(double2); }

// ---------------------------------------------------------------- forward
// Byte tables of the layer-0/1 matrix-product state: btab[k][v] = product of
// T_w[v_{w-8k}] over the eight wires w = 8k..8k+7 (identity beyond n), as
// four complex entries each.
__global__ void __launch_bounds__(256) mps_bytes_kernel(const double4 *__restrict__ coef, int n,
                                                        double2 *__restrict__ btab) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. 1023
  if (e >= 1024) return;
  const int k = e >> 8, v = e & 255;
  M2x2 p = ident();
  for (int j = 0; j < 8; ++j) {
    const int w = 8 * k + j;
    if (w < n) p = mmul(p, tmat(wire_gates(coef, n, w, 0), w, (v >> j) & 1));
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) btab[4 * e + q] = p.m[q];
}

__device__ __forceinline__ M2x2 load_m(const double2 *__restrict__ btab, int k, int v) {
  M2x2 R;
#pragma unroll
  for (int q = 0; q < 4; ++q) R.m[q] = __ldg(&btab[4 * (256 * k + v) + q]);
  return R;
}

// chi1(r) = Tr(B0[r0] B1[r1] B2[r2] B3[r3]) for 4096 contiguous r per tile;
// thread t takes r = base + t + 256 k (k = 0..15): byte 0 is t for all its
// amplitudes, so chi1 = Tr(B1[r1] W) with W = B2 B3 B0[t] fixed per tile.
// SCATTER stores chi1(r) at P(r) (the input of layer 2), else at r.
template <bool SCATTER>
__global__ void __launch_bounds__(256) fwd01_kernel(const Fwd01Params Q) {
  const int t = threadIdx.x;
  const int n = Q.n;
  const M2x2 b0 = load_m(Q.btab, 0, t);
  for (u64 tile = blockIdx.x; tile < Q.num_tiles; tile += gridDim.x) {
    const u64 base = tile << 12;
    const M2x2 W = mmul(mmul(load_m(Q.btab, 2, static_cast<int>((base >> 16) & 255)),
                             load_m(Q.btab, 3, static_cast<int>((base >> 24) & 255))),
                        b0);
    const int hi1 = static_cast<int>((base >> 8) & 0xF0);
#pragma unroll 4
    for (int k = 0; k < 16; ++k) {
      const M2x2 b1 = load_m(Q.btab, 1, hi1 | k);
      // Tr(b1 W) = sum_{i,j} b1[i][j] W[j][i]
      double2 v = cmul(b1.m[0], W.m[0]);
      v = cfma(b1.m[1], W.m[2], v);
      v = cfma(b1.m[2], W.m[1], v);
      v = cfma(b1.m[3], W.m[3], v);
      const u64 r = base | static_cast<u64>(t + 256 * k);
      __stcs(&Q.out[SCATTER ? ring_p(r, n) : r], v);
    }
  }
}

}  // namespace

cudaError_t launch_fwd01(const Fwd01Params &Q, int grid, cudaStream_t s) {
  if (Q.n < 13 || Q.n > 31 || grid < 1) return cudaErrorInvalidValue;
  mps_bytes_kernel<<<4, 256, 0, s>>>(Q.coef, Q.n, Q.btab);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (Q.scatter) fwd01_kernel<true><<<grid, 256, 0, s>>>(Q);
  else fwd01_kernel<false><<<grid, 256, 0, s>>>(Q);
  return cudaGetLastError();
}

cudaError_t launch_grad01(const Grad01Params &Q, int grid, cudaStream_t s) {
  if (Q.n < 13 || Q.n > 31 || grid < 1) return cudaErrorInvalidValue;
  static bool configured = false;
  if (!configured) {
    const cudaError_t e = cudaFuncSetAttribute(grad01_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(grad01_smem_bytes()));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  grad01_kernel<<<grid, kG01Threads, grad01_smem_bytes(), s>>>(Q);
  return cudaGetLastError();
}

cudaError_t launch_grad01_finalize(const Grad01Params &Q, int grid, double *grad_out, cudaStream_t s) {
  grad01_finalize_kernel<<<1, 256, 0, s>>>(Q, grid, grad_out);
  return cudaGetLastError();
}

}  // namespace rsv
