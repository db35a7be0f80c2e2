// The first K layers of the ansatz as a matrix-product state (sm_100a).
//
// The circuit starts from |0...0>.  With q the index after a layer's
// rotations, that layer's CNOT ring turns q into prefix parities
// s_w = q_0 ^ ... ^ q_w (bit 0 of P(q) is s_{n-1} ^ s_0).  If the state after
// k - 1 layers is a periodic matrix-product state chi(q) = Tr prod_w A_w[q_w]
// of bond dimension d, the state after layer k's rotations is one of bond
// dimension 2d, with the new bond index (x, s) (x the old bond, s the prefix
// parity):
//   T_w[b]((x, s'), (y, s)) = U_w[b, s]      A_w[s ^ s'](x, y)    (w >= 1),
//   T_0[b]((x, s'), (y, s)) = U_0[b, s' ^ s] A_0[s](x, y),
// starting from the 1 x 1 tensors A_w[b] = (U_w |0>)_b of layer 0 (U = RZ RY of
// the layer).  So the first K layers are chi_{K-1}(r) = Tr prod_w T_w[r_w] with
// bond D = 2^(K-1).  K = 2 (D = 2) and K = 3 (D = 4) are used here.
//
// Forward (mps_fwd_kernel): one write of chi_{K-1} (scattered through P when
// more layers follow) from byte tables of products of eight site matrices.
// Backward: every parameter of the first K layers on wire w enters T_w only,
// so with lambda the adjoint state at the output of layer K - 1
//   dE/dx = 2 Re sum_b Tr( d_x T_w[b] E_w[b] ),
//   E_w[b] = sum over r with r_w = b of conj(lambda(r)) R_w(r)
// (R_w the cyclic product of the other site matrices after w).  One read of
// lambda in 4096-amplitude tiles (a = bits 0..5, h = bits 6..11, t = coset
// bits 12..n-1 split into lo (m1 bits) and hi):
//   X1(a) = sum_h conj(lambda) M2(h),  X2(h) = sum_a conj(lambda) M1(a),
//   G(a) += X1(a) C_t,  F(h) += C_t X2(h),  Z_t = sum_a M1(a) X1(a)
// (M1 = T_0..T_5, M2 = T_6..T_11, C_t = CosLo(lo) CosHi(hi) the product of the
// coset sites), then Y(lo) = sum_hi CosHi(hi) Z_t and Y'(hi) = sum_lo Z_t
// CosLo(lo) (mps_coset_kernel), and per wire the leave-one-out products over
// its group of bits (mps_finalize_kernel).
// The reference walks these layers back gate by gate
// (cpp/ising_cuda_statevector_grad_kernels.cu:223-319, scheduled by
// cpp/ising_cuda_structured_adjoint_modes.inc:272-307) and computes layer 0
// analytically in the forward (cpp/ising_cuda_rotation_kernels.cu:20-41); the
// sums are the same.
#include "rsv_launch.h"
#include "rsv_tile.cuh"

namespace rsv {
namespace {

template <int D>
struct Mat {
  double2 m[D * D];  // row-major
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // a * b + c
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// conj(x) * w + c
__device__ __forceinline__ double2 cjfma(double2 x, double2 w, double2 c) {
  return make_double2(fma(x.x, w.x, fma(x.y, w.y, c.x)), fma(x.x, w.y, fma(-x.y, w.x, c.y)));
}
template <int D>
__device__ __forceinline__ Mat<D> mmul(const Mat<D> &A, const Mat<D> &B) {
  Mat<D> R;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double2 s = cmul(A.m[i * D], B.m[j]);
#pragma unroll
      for (int k = 1; k < D; ++k) s = cfma(A.m[i * D + k], B.m[k * D + j], s);
      R.m[i * D + j] = s;
    }
  return R;
}
template <int D>
__device__ __forceinline__ Mat<D> ident() {
  Mat<D> R;
#pragma unroll
  for (int e = 0; e < D * D; ++e) R.m[e] = make_double2((e % (D + 1)) == 0 ? 1.0 : 0.0, 0.0);
  return R;
}
template <int D>
__device__ __forceinline__ Mat<D> load_mat(const double2 *p) {
  Mat<D> R;
#pragma unroll
  for (int e = 0; e < D * D; ++e) R.m[e] = p[e];
  return R;
}
template <int D>
__device__ __forceinline__ void store_mat(double2 *p, const Mat<D> &A) {
#pragma unroll
  for (int e = 0; e < D * D; ++e) p[e] = A.m[e];
}
template <int D>
__device__ __forceinline__ Mat<D> ldg_mat(const double2 *__restrict__ p) {
  Mat<D> R;
#pragma unroll
  for (int e = 0; e < D * D; ++e) R.m[e] = __ldg(&p[e]);
  return R;
}

// Layer-k gate of wire w, U = RZ(phi) RY(theta) = [[c e-, -s e-], [s e+, c e+]]
// (e-+ = e^{-+ i phi/2}), or its theta- (kind 1) or phi-derivative (kind 2).
__device__ __forceinline__ void layer_gate(const double4 *coef, int n, int k, int w, int kind, double2 (&u)[2][2]) {
  const double4 q = coef[k * n + w];
  const double2 em = make_double2(q.z, -q.w), ep = make_double2(q.z, q.w);
  double c = q.x, s = q.y;
  if (kind == 1) {  // d RY / d theta = [[-s/2, -c/2], [c/2, -s/2]]: the (c, s) pattern with c -> -s/2, s -> c/2
    c = -0.5 * q.y;
    s = 0.5 * q.x;
  }
  u[0][0] = make_double2(c * em.x, c * em.y);
  u[0][1] = make_double2(-s * em.x, -s * em.y);
  u[1][0] = make_double2(s * ep.x, s * ep.y);
  u[1][1] = make_double2(c * ep.x, c * ep.y);
  if (kind == 2) {  // d RZ / d phi: row 0 times -i/2, row 1 times +i/2
#pragma unroll
    for (int y = 0; y < 2; ++y) {
      u[0][y] = make_double2(0.5 * u[0][y].y, -0.5 * u[0][y].x);
      u[1][y] = make_double2(-0.5 * u[1][y].y, 0.5 * u[1][y].x);
    }
  }
}

// Site matrices T_w[0], T_w[1] of the first K = log2(D) + 1 layers, with the
// gate of layer dlayer replaced by its derivative dkind (0: none).
template <int D>
__device__ void site_tensor(const double4 *coef, int n, int w, int dlayer, int dkind, Mat<D> (&T)[2]) {
  double2 cur[2][D * D], nxt[2][D * D];
  double2 u[2][2];
  layer_gate(coef, n, 0, w, dlayer == 0 ? dkind : 0, u);
  cur[0][0] = u[0][0];  // (U |0>)_b
  cur[1][0] = u[1][0];
  int d = 1;
  for (int k = 1; 2 * d <= D; ++k) {
    layer_gate(coef, n, k, w, dlayer == k ? dkind : 0, u);
    const int d2 = 2 * d;
    for (int b = 0; b < 2; ++b)
      for (int sp = 0; sp < 2; ++sp)
        for (int s = 0; s < 2; ++s)
          for (int x = 0; x < d; ++x)
            for (int y = 0; y < d; ++y)
              nxt[b][(2 * x + sp) * d2 + (2 * y + s)] =
                  w >= 1 ? cmul(u[b][s], cur[s ^ sp][x * d + y]) : cmul(u[b][sp ^ s], cur[s][x * d + y]);
    for (int b = 0; b < 2; ++b)
      for (int e = 0; e < d2 * d2; ++e) cur[b][e] = nxt[b][e];
    d = d2;
  }
  for (int b = 0; b < 2; ++b)
    for (int e = 0; e < D * D; ++e) T[b].m[e] = cur[b][e];
}

// ---------------------------------------------------------------- tables
// tsite[w][b] for w < 32 (identity for w >= n)
template <int D>
__global__ void mps_site_kernel(const MpsParams Q) {
  const int t = threadIdx.x;
  if (t >= 32) return;
  Mat<D> T[2];
  if (t < Q.n) {
    site_tensor<D>(Q.coef, Q.n, t, -1, 0, T);
  } else {
    T[0] = T[1] = ident<D>();
  }
  store_mat<D>(Q.tsite + (2 * t) * D * D, T[0]);
  store_mat<D>(Q.tsite + (2 * t + 1) * D * D, T[1]);
}

// product of the site matrices of wires w0 .. w0 + nb - 1 for the bits of v
template <int D>
__device__ __forceinline__ Mat<D> site_chain(const double2 *tsite, int w0, int nb, unsigned v) {
  Mat<D> p = ident<D>();
  for (int j = 0; j < nb; ++j) p = mmul<D>(p, load_mat<D>(tsite + (2 * (w0 + j) + ((v >> j) & 1)) * D * D));
  return p;
}

// byte tables (4 x 256) for the forward, coset tables CosLo (2^m1) and CosHi
// (2^m2) for the backward
template <int D>
__global__ void mps_tables_kernel(const MpsParams Q) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int nlo = 1 << Q.m1, nhi = 1 << Q.m2;
  if (e < 1024) {
    const int k = e >> 8, v = e & 255;
    store_mat<D>(Q.btab + e * D * D, site_chain<D>(Q.tsite, 8 * k, 8, static_cast<unsigned>(v)));
  } else if (e < 1024 + nlo) {
    const int lo = e - 1024;
    store_mat<D>(Q.coslo + lo * D * D, site_chain<D>(Q.tsite, 12, Q.m1, static_cast<unsigned>(lo)));
  } else if (e < 1024 + nlo + nhi) {
    const int hi = e - 1024 - nlo;
    store_mat<D>(Q.coshi + hi * D * D, site_chain<D>(Q.tsite, 12 + Q.m1, Q.m2, static_cast<unsigned>(hi)));
  } else if (e < 1024 + nlo + nhi + 128) {
    // in-tile halves: M1(a) = T_0..T_5 (entries 0..63), M2(h) = T_6..T_11 (64..127)
    const int x = e - 1024 - nlo - nhi;
    store_mat<D>(Q.mtab + x * D * D, site_chain<D>(Q.tsite, x < 64 ? 0 : 6, 6, static_cast<unsigned>(x & 63)));
  } else if (e < 1024 + nlo + nhi + 128 + (1 << (Q.n > 16 ? Q.n - 16 : 0))) {
    // W(x) = B2[x & 255] B3[x >> 8]: the product over wires 16..31
    const int x = e - 1024 - nlo - nhi - 128;
    store_mat<D>(Q.wtab + x * D * D, site_chain<D>(Q.tsite, 16, 16, static_cast<unsigned>(x)));
  }
}

// --------------------------------------------------------------- forward
// chi(r) = Tr(B0[r0] B1[r1] B2[r2] B3[r3]) (r_k the bytes of r), written as
// out[P(r)] = chi(r) when SCATTER (the ring of the last MPS layer applied) and
// out[r] = chi(r) otherwise.
//
// Bond 4: every tile is 4096 contiguous OUTPUT indices o = base + t + 256 k,
// evaluated at r = P^{-1}(o) (identity without SCATTER), so every store is a
// whole line.  Byte 0 of P^{-1}(o) depends on o's bits 0..7 and bit n-1 only,
// bytes 1..3 on o's bits 7..31, so per tile the 32 products
// Y_{k,s} = B1 W at P^{-1}(base + 256 k + 128 s) (s = bit 7 of t; W = B2 B3
// from a table over bytes 2 and 3) go to
// shared memory (double-buffered, one barrier per tile), and the traces
// out[t][k] = Tr(Y_{k,t7} B0[r0(t)]) = sum_e A[t][e] Y_{k,t7}[e]
// (A[t][(i, j)] = B0[r0(t)][j][i]) are one complex product per half tile on
// the FP64 tensor cores: warp w takes rows t = 32 w .. 32 w + 31 (t7 = w / 4)
// as four m8n8k4 row tiles by two column tiles, its A fragments in registers
// (reloaded when bit n-1 of the tile changes), Gauss 3-multiply; two CTAs per
// SM (128 registers) hide the latency of the per-tile table loads.
//
// Bond 2: thread t takes r = base + t + 256 k (k = 0..15): byte 0 is t, byte 1
// is k | (the tile's bits 12..15).  Per tile the 16 products
// Y_k = B1[r1(k)] B2 B3 go to shared memory and every amplitude is
// Tr(Y_k B0[t]) with B0[t] held in registers, stored at P(r).
template <int D, bool SCATTER>
__global__ void __launch_bounds__(256, D == 4 ? 2 : 1) mps_fwd_kernel(const MpsParams Q, double2 *__restrict__ out) {
  constexpr int E = D * D;
  constexpr int YP = D == 4 ? 20 : E;  // row pitch of Y: fragment reads free of bank conflicts
  __shared__ double2 ysm[2][D == 4 ? 32 : 16][YP];
  const int t = threadIdx.x, n = Q.n;
  if constexpr (D == 4) {
    const int lane = t & 31, warp = t >> 5, fg = lane >> 2, t4 = lane & 3;
    const int ys_set = warp >> 2;
    double are[4][4], aim[4][4], asum[4][4];
    int aflip = -1;  // bit n-1 of the tiles the A fragments were loaded for
    int it = 0;
    for (u64 tile = blockIdx.x; tile < Q.num_tiles; tile += gridDim.x, ++it) {
      const u64 base = tile << 12;
      const int flip = SCATTER ? static_cast<int>((base >> (n - 1)) & 1) : 0;
      if (flip != aflip) {
        aflip = flip;
#pragma unroll
        for (int rt = 0; rt < 4; ++rt) {
          const u64 o = base | static_cast<u64>(32 * warp + 8 * rt + fg);
          const int r0 = static_cast<int>((SCATTER ? ring_pinv(o, n) : o) & 255);
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            // K index 4 ks + t4 = (i, j) = (ks, t4): A = B0[r0][t4][ks]
            const double2 v = __ldg(&Q.btab[r0 * E + t4 * D + ks]);
            are[rt][ks] = v.x;
            aim[rt][ks] = v.y;
            asum[rt][ks] = v.x + v.y;
          }
        }
      }
      double2(*ys)[YP] = ysm[it & 1];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ks_ = h * 16 + (t >> 4), e = t & 15, i = e / D, j = e % D;  // ks_ = 16 s + k
        const u64 o = base | (static_cast<u64>(ks_ & 15) << 8) | (static_cast<u64>(ks_ >> 4) << 7);
        const u64 r = SCATTER ? ring_pinv(o, n) : o;
        const double2 *b1 = Q.btab + (256 + ((r >> 8) & 255)) * E;
        const double2 *w = Q.wtab + (r >> 16) * E;
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int m = 0; m < D; ++m) acc = cfma(__ldg(&b1[i * D + m]), __ldg(&w[m * D + j]), acc);
        ys[ks_][e] = acc;
      }
      __syncthreads();
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) {
        double t1[4][2] = {}, t2[4][2] = {}, t3[4][2] = {};
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const double2 y = ys[16 * ys_set + 8 * ct + fg][4 * ks + t4];
          const double ysum = y.x + y.y;
#pragma unroll
          for (int rt = 0; rt < 4; ++rt) {
            mma_f64(t1[rt][0], t1[rt][1], are[rt][ks], y.x);
            mma_f64(t2[rt][0], t2[rt][1], aim[rt][ks], y.y);
            mma_f64(t3[rt][0], t3[rt][1], asum[rt][ks], ysum);
          }
        }
#pragma unroll
        for (int rt = 0; rt < 4; ++rt)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const double2 v = make_double2(t1[rt][e] - t2[rt][e], t3[rt][e] - t1[rt][e] - t2[rt][e]);
            const u64 o = base | static_cast<u64>(32 * warp + 8 * rt + fg + 256 * (8 * ct + 2 * t4 + e));
            __stcs(&out[o], v);
          }
      }
    }
    return;
  }
  const Mat<D> b0 = ldg_mat<D>(Q.btab + t * E);
  int it = 0;
  for (u64 tile = blockIdx.x; tile < Q.num_tiles; tile += gridDim.x, ++it) {
    const u64 base = tile << 12;
    double2(*ys)[YP] = ysm[it & 1];
    for (int s = t; s < 16 * E; s += 256) {
      // entry (i, j) of Y_k = B1[r1] (B2 B3)
      const int k = s / E, e = s % E, i = e / D, j = e % D;
      const double2 *b1 = Q.btab + (256 + (static_cast<int>((base >> 8) & 0xF0) | k)) * E;
      const double2 *b2 = Q.btab + (512 + ((base >> 16) & 255)) * E;
      const double2 *b3 = Q.btab + (768 + ((base >> 24) & 255)) * E;
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int m = 0; m < D; ++m) {
        double2 q = make_double2(0.0, 0.0);  // (B2 B3)[m][j]
#pragma unroll
        for (int l = 0; l < D; ++l) q = cfma(__ldg(&b2[m * D + l]), __ldg(&b3[l * D + j]), q);
        acc = cfma(__ldg(&b1[i * D + m]), q, acc);
      }
      ys[k][e] = acc;
    }
    __syncthreads();
#pragma unroll 2
    for (int k = 0; k < 16; ++k) {
      // Tr(Y_k B0) = sum_{i,j} Y_k[i][j] B0[j][i]
      double2 v = make_double2(0.0, 0.0);
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) v = cfma(ys[k][i * D + j], b0.m[j * D + i], v);
      const u64 r = base | static_cast<u64>(t + 256 * k);
      __stcs(&out[SCATTER ? ring_p(r, n) : r], v);
    }
  }
}

// -------------------------------------------------------------- backward
constexpr int kMpsThreads = 256;
// Stage slot of tile amplitude i = a + 64 h.  Bond 2 reads a column (fixed a)
// or a row (fixed h) of 32 entries per warp: i ^ (h & 7).  Bond 4 reads m8n8k4
// fragments, 8 rows x 4 columns per warp in either orientation; with
// i ^ ((h & 1) << 2 | (h & 2)) the eight 16-byte entries of every
// quarter-warp fall in different bank groups.
template <int D>
__device__ __forceinline__ int mps_slot(int i) {
  const int h = i >> 6;
  return D == 4 ? i ^ (((h & 1) << 2) | (h & 2)) : i ^ (h & 7);
}

template <int D>
constexpr size_t mps_grad_smem() {
  // stage, M1, M2, X1, X2, C, Z partials (two buffers of 8 warps)
  return (4096 + 4 * 64 * D * D + D * D + 2 * 8 * D * D) * sizeof(double2);
}

template <int D>
__global__ void __launch_bounds__(kMpsThreads) mps_grad_kernel(const MpsParams Q, const double2 *__restrict__ lam,
                                                                int gather) {
  constexpr int E = D * D;
  constexpr int EPT = E / 4;  // X / G / F entries per thread
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage = reinterpret_cast<double2 *>(smem_raw);
  double2 *m1 = stage + 4096;  // [64][E]: T_0..T_5 (a), copied from the tables
  double2 *m2 = m1 + 64 * E;   // [64][E]: T_6..T_11 (h)
  double2 *x1 = m2 + 64 * E;
  double2 *x2 = x1 + 64 * E;
  double2 *csm = x2 + 64 * E;  // [E]
  double2 *zp = csm + E;       // [2][8][E]

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = Q.n;
  for (int i = t; i < 128 * E; i += kMpsThreads) m1[i] = Q.mtab[i];
  __syncthreads();

  const int idx = t >> 2, q = t & 3;
  double2 g[EPT], f[EPT];
#pragma unroll
  for (int j = 0; j < EPT; ++j) g[j] = f[j] = make_double2(0.0, 0.0);
  // Z partial of this thread: entry ze, a-range zp0 .. zp0 + 64 / (256 / E) - 1
  constexpr int kZParts = kMpsThreads / E, kZA = 64 / kZParts;
  const int ze = t % E, zpart = t / E;
  const int zi = ze / D, zj = ze % D;

  // Bond 4: X1 and X2 on the FP64 tensor cores.  Warps 0..3 compute X1
  // (rows a, K = h, B = M2), warps 4..7 X2 (rows h, K = a, B = M1), each warp
  // 32 rows x 8 columns (columns 8 nt .. 8 nt + 7 of the 16 entries), as four
  // m8n8k4 row tiles per K step.  The complex product conj(lambda) M is three
  // real products (Gauss): t1 = lr Mr, t2 = li Mi, t3 = (lr - li)(Mr + Mi);
  // re = t1 + t2, im = t3 - t1 + t2.  The warp's B fragments, 16 K steps of
  // Mr, Mi and Mr + Mi, stay in registers for the whole kernel.
  const int fg = lane >> 2, t4 = lane & 3;
  const bool xsecond = warp >= 4;
  const int xnt = warp & 1, xr0 = 32 * ((warp >> 1) & 1);
  double bre[D == 4 ? 16 : 1], bim[D == 4 ? 16 : 1], bsum[D == 4 ? 16 : 1];
  if constexpr (D == 4) {
    const double2 *bt = Q.mtab + (xsecond ? 0 : 64 * E);
#pragma unroll
    for (int ks = 0; ks < 16; ++ks) {
      const double2 v = bt[(4 * ks + t4) * E + 8 * xnt + fg];
      bre[ks] = v.x;
      bim[ks] = v.y;
      bsum[ks] = v.x + v.y;
    }
  }

  const u64 num_tiles = Q.num_tiles;
  const unsigned lomask = (1u << Q.m1) - 1u;
  auto issue = [&](u64 tile) {
    if (tile < num_tiles) {
      const u64 base = tile << 12;
#pragma unroll
      for (int r = 0; r < 4096 / kMpsThreads; ++r) {
        const int tau = t + r * kMpsThreads;
        const u64 p = base | static_cast<u64>(tau);
        cp_async16(&stage[mps_slot<D>(tau)], &lam[gather ? ring_p(p, n) : p]);
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x);

  int k = 0;
  u64 prev = 0;
  for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x, ++k) {
    cp_async_wait_all();
    __syncthreads();
    // the previous tile's Z, from the per-warp partials
    if (k > 0 && t < E) {
      const double2 *zb = zp + ((k - 1) & 1) * 8 * E;
      double2 s = zb[t];
      for (int w = 1; w < 8; ++w) s = cadd(s, zb[w * E + t]);
      Q.zt[prev * E + t] = s;
    }
    if (t < E) {
      // C_t = CosLo(lo) CosHi(hi), entry t
      const unsigned lo = static_cast<unsigned>(tile) & lomask, hi = static_cast<unsigned>(tile >> Q.m1);
      const double2 *cl = Q.coslo + lo * E, *ch = Q.coshi + hi * E;
      const int i = t / D, j = t % D;
      double2 s = cmul(__ldg(&cl[i * D]), __ldg(&ch[j]));
#pragma unroll
      for (int kk = 1; kk < D; ++kk) s = cfma(__ldg(&cl[i * D + kk]), __ldg(&ch[kk * D + j]), s);
      csm[t] = s;
    }
    if constexpr (D == 4) {
      double t1[4][2] = {}, t2[4][2] = {}, t3[4][2] = {};
#pragma unroll
      for (int ks = 0; ks < 16; ++ks) {
#pragma unroll
        for (int rt = 0; rt < 4; ++rt) {
          const int row = xr0 + 8 * rt + fg, col = 4 * ks + t4;
          const double2 l = stage[mps_slot<D>(xsecond ? col + 64 * row : row + 64 * col)];
          mma_f64(t1[rt][0], t1[rt][1], l.x, bre[ks]);
          mma_f64(t2[rt][0], t2[rt][1], l.y, bim[ks]);
          mma_f64(t3[rt][0], t3[rt][1], l.x - l.y, bsum[ks]);
        }
      }
      double2 *xo = xsecond ? x2 : x1;
#pragma unroll
      for (int rt = 0; rt < 4; ++rt)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          xo[(xr0 + 8 * rt + fg) * E + 8 * xnt + 2 * t4 + e] =
              make_double2(t1[rt][e] + t2[rt][e], t3[rt][e] - t1[rt][e] + t2[rt][e]);
    } else {
      double2 a1[EPT], a2[EPT];
#pragma unroll
      for (int j = 0; j < EPT; ++j) a1[j] = a2[j] = make_double2(0.0, 0.0);
#pragma unroll 4
      for (int kk = 0; kk < 64; ++kk) {
        const double2 c1 = stage[mps_slot<D>(idx + 64 * kk)];  // a = idx, h = kk
        const double2 c2 = stage[mps_slot<D>(kk + 64 * idx)];  // a = kk, h = idx
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
          a1[j] = cjfma(c1, m2[kk * E + q + 4 * j], a1[j]);
          a2[j] = cjfma(c2, m1[kk * E + q + 4 * j], a2[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < EPT; ++j) {
        x1[idx * E + q + 4 * j] = a1[j];
        x2[idx * E + q + 4 * j] = a2[j];
      }
    }
    __syncthreads();
    issue(tile + gridDim.x);  // the stage is free
    // G(a) += X1(a) C, F(h) += C X2(h)
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      const int e = q + 4 * j, i = e / D, jj = e % D;
      double2 sg = g[j], sf = f[j];
#pragma unroll
      for (int kk = 0; kk < D; ++kk) {
        sg = cfma(x1[idx * E + i * D + kk], csm[kk * D + jj], sg);
        sf = cfma(csm[i * D + kk], x2[idx * E + kk * D + jj], sf);
      }
      g[j] = sg;
      f[j] = sf;
    }
    // Z partial: sum over this thread's a-range of (M1(a) X1(a))[zi][zj]
    {
      double2 z = make_double2(0.0, 0.0);
#pragma unroll
      for (int aa = 0; aa < kZA; ++aa) {
        const int a = zpart * kZA + aa;
#pragma unroll
        for (int kk = 0; kk < D; ++kk) z = cfma(m1[a * E + zi * D + kk], x1[a * E + kk * D + zj], z);
      }
      // threads with the same entry in a warp differ in lane bits >= log2(E)
#pragma unroll
      for (int m = E; m < 32; m <<= 1)
        z = cadd(z, make_double2(__shfl_xor_sync(0xffffffffu, z.x, m), __shfl_xor_sync(0xffffffffu, z.y, m)));
      if (lane < E) zp[(k & 1) * 8 * E + warp * E + lane] = z;
    }
    prev = tile;
  }
  cp_async_wait_all();
  __syncthreads();
  if (k > 0 && t < E) {
    const double2 *zb = zp + ((k - 1) & 1) * 8 * E;
    double2 s = zb[t];
    for (int w = 1; w < 8; ++w) s = cadd(s, zb[w * E + t]);
    Q.zt[prev * E + t] = s;
  }
  double2 *rec = Q.partials + static_cast<size_t>(blockIdx.x) * 2 * 64 * E;
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    rec[idx * E + q + 4 * j] = g[j];
    rec[64 * E + idx * E + q + 4 * j] = f[j];
  }
}

// Bond 4, warp-specialised: the FP64 tensor-core phase of a tile (X1, X2)
// and its FP64 phase (G, F, Z) overlap instead of alternating.  Sixteen warps:
//   warps 0..7 ("tensor warps") only read fragments and issue MMAs: wait for
//     tile k in stage k & 1, compute X1 (warps 0..3) and X2 (warps 4..7) as in
//     mps_grad_kernel (B fragments from a swizzled shared copy of M1, M2),
//     release the stage, wait until X buffer k & 1 is free and write it;
//   warps 8..15 ("FP64 warps") load the tiles (cp.async, up to two ahead) and
//     take tile k's X1, X2 from buffer k & 1 while the tensor warps work on
//     tile k + 1.  Thread c owns a = c >> 2 and row i = c & 3: that row of
//     G(a), F(h = a) and of M1(a) X1(a), whose sum over a (a lane butterfly
//     over a's bits 0..2, then the eight warps in order) is Z of the tile.
// Hand-offs on named barriers (bar.arrive by the producer, bar.sync by the
// consumer; 512 threads): kBarStageFull + s / kBarStageEmpty + s (stage s
// loaded / read), kBarXFull + b / kBarXEmpty + b (X buffer b written / read);
// kBarCons synchronises the FP64 warps alone.  Both sides run the same tile
// count and every arrive is matched by one sync, so every barrier phase
// completes.
namespace mg4 {
constexpr int kThreads = 512;
constexpr int kTensorThreads = 256;
constexpr int kFp64Threads = kThreads - kTensorThreads;
constexpr int kE = 16;
constexpr int kBarStageFull = 1, kBarStageEmpty = 3, kBarXFull = 5, kBarXEmpty = 7, kBarCons = 9;
// stages, X buffers, M1 / M2, C (two tiles), Z partials of the eight FP64 warps
constexpr size_t kSmem = (2 * 4096 + 2 * 2 * 64 * kE + 2 * 64 * kE + 2 * kE + 8 * kE) * sizeof(double2);
static_assert(kSmem <= 232448, "more shared memory than a block can have");
// slot of M entry (k, column) in the shared copy: the column's bits 1, 2 XOR
// k's bits 0, 1, so that the B fragment reads (k = 4 ks + t4, column
// 8 nt + fg) of a quarter-warp fall in eight different bank groups
__device__ __forceinline__ int mslot(int k, int col) { return k * kE + (col ^ ((k & 3) << 1)); }
// slot of X entry e of row r (a for X1, h for X2): bits 0, 1 of e XOR r's bit 0
// and e's bit 3, so that both the tensor warps' writes (a quarter-warp varies
// r bit 0 and e bits 1, 2) and the FP64 warps' row reads (r bit 0, e bits 2, 3)
// fall in eight different bank groups
__device__ __forceinline__ int xslot(int r, int e) { return r * kE + (e ^ (r & 1) ^ (((e >> 3) & 1) << 1)); }
__device__ __forceinline__ void bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(int id, int count) {
  asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ double2 lds_f64x2(unsigned addr) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ double2 shfl_xor2(double2 v, int m) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// One tile's X1 (SECOND = false: rows a, K = h, B = M2) or X2 (rows h, K = a,
// B = M1) rows of a tensor warp: 32 rows x 8 columns as four m8n8k4 row tiles
// (twelve independent MMA chains), K = 64 in sixteen steps.  The A and B
// fragments come through volatile shared loads issued one K step ahead of the
// (volatile) MMAs that use them.  With the stage swizzle mps_slot<4> the A
// fragment addresses are affine in (K step, row tile) from one or two
// per-thread bases:
//   X1: slot = (row ^ s(t4)) + 64 col, row = r0 + 8 rt + fg, col = 4 ks + t4,
//       s(t4) = (t4 & 1) << 2 | (t4 & 2)                -> base + 4096 B ks + 128 B rt;
//   X2: slot = (col ^ s(fg)) + 64 row, col ^ s(fg) = 4 (ks ^ (fg & 1)) + (t4 ^ (fg & 2))
//                                                    -> base(ks parity) + 64 B ks + 8192 B rt;
// and the B fragment of step ks is M entry (4 ks + t4, 8 nt + fg): mslot
// keeps column bits 1, 2 ^ t4, so base + 1024 B ks.
template <bool SECOND>
__device__ __forceinline__ void tensor_tile(unsigned sst, unsigned mbase, int xr0, int fg, int t4,
                                            double (&t1)[4][2], double (&t2)[4][2], double (&t3)[4][2]) {
  unsigned base0, base1;  // even / odd K steps
  if (SECOND) {
    const unsigned b = sst + 16u * static_cast<unsigned>((t4 ^ (fg & 2)) + 64 * (xr0 + fg));
    base0 = b + 64u * static_cast<unsigned>(fg & 1);
    base1 = b - 64u * static_cast<unsigned>(fg & 1);
  } else {
    base0 = base1 = sst + 16u * static_cast<unsigned>(xr0 + (fg ^ (((t4 & 1) << 2) | (t4 & 2))) + 64 * t4);
  }
  auto addr = [&](int ks, int rt) {
    return ((ks & 1) ? base1 : base0) + (SECOND ? 64u * ks + 8192u * rt : 4096u * ks + 128u * rt);
  };
  double2 cur[4], nxt[4], bcur, bnxt;
  bcur = lds_f64x2(mbase);
#pragma unroll
  for (int rt = 0; rt < 4; ++rt) cur[rt] = lds_f64x2(addr(0, rt));
#pragma unroll
  for (int ks = 0; ks < 16; ++ks) {
    if (ks + 1 < 16) {
      bnxt = lds_f64x2(mbase + 1024u * (ks + 1));
#pragma unroll
      for (int rt = 0; rt < 4; ++rt) nxt[rt] = lds_f64x2(addr(ks + 1, rt));
    }
    const double bsum = bcur.x + bcur.y;
#pragma unroll
    for (int rt = 0; rt < 4; ++rt) {
      const double2 l = cur[rt];
      mma_f64(t1[rt][0], t1[rt][1], l.x, bcur.x);
      mma_f64(t2[rt][0], t2[rt][1], l.y, bcur.y);
      mma_f64(t3[rt][0], t3[rt][1], l.x - l.y, bsum);
    }
    if (ks + 1 < 16) {
      bcur = bnxt;
#pragma unroll
      for (int rt = 0; rt < 4; ++rt) cur[rt] = nxt[rt];
    }
  }
}
}  // namespace mg4

__global__ void __launch_bounds__(mg4::kThreads, 1) mps_grad4_kernel(const MpsParams Q,
                                                                       const double2 *__restrict__ lam, int gather) {
  using namespace mg4;
  constexpr int E = kE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *stage = reinterpret_cast<double2 *>(smem_raw);  // [2][4096]
  double2 *xbuf = stage + 2 * 4096;                        // [2][X1, X2][64][E]
  double2 *msm = xbuf + 2 * 2 * 64 * E;                    // [M1, M2][64 mslots]
  double2 *csm = msm + 2 * 64 * E;                         // [2][E]
  double2 *zp = csm + 2 * E;                               // [8][E]

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = Q.n;
  const u64 num_tiles = Q.num_tiles, first = blockIdx.x;
  const int my_tiles = first < num_tiles ? static_cast<int>((num_tiles - 1 - first) / gridDim.x) + 1 : 0;
  for (int i = t; i < 2 * 64 * E; i += kThreads) {
    const int m = i >> 10, k = (i >> 4) & 63, col = i & 15;
    msm[m * 64 * E + mslot(k, col)] = Q.mtab[i];
  }
  __syncthreads();

  if (warp < 8) {
    const int fg = lane >> 2, t4 = lane & 3;
    const bool xsecond = warp >= 4;
    const int xnt = warp & 1, xr0 = 32 * ((warp >> 1) & 1);
    // B fragments of step 0: M entry (t4, 8 nt + fg) of M2 (X1) or M1 (X2)
    const unsigned mbase =
        static_cast<unsigned>(__cvta_generic_to_shared(msm + (xsecond ? 0 : 64 * E) + mslot(t4, 8 * xnt + fg)));
    for (int k = 0; k < my_tiles; ++k) {
      const int b = k & 1;
      bar_sync(kBarStageFull + b, kThreads);  // tile k is in stage b
      const unsigned sst = static_cast<unsigned>(__cvta_generic_to_shared(stage + b * 4096));
      double t1[4][2] = {}, t2[4][2] = {}, t3[4][2] = {};
      if (xsecond) tensor_tile<true>(sst, mbase, xr0, fg, t4, t1, t2, t3);
      else tensor_tile<false>(sst, mbase, xr0, fg, t4, t1, t2, t3);
      if (k + 2 < my_tiles) bar_arrive(kBarStageEmpty + b, kThreads);  // stage b may take tile k + 2
      if (k >= 2) bar_sync(kBarXEmpty + b, kThreads);                   // X buffer b is done with tile k - 2
      double2 *xo = xbuf + (2 * b + (xsecond ? 1 : 0)) * 64 * E;
#pragma unroll
      for (int rt = 0; rt < 4; ++rt)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          xo[xslot(xr0 + 8 * rt + fg, 8 * xnt + 2 * t4 + e)] =
              make_double2(t1[rt][e] + t2[rt][e], t3[rt][e] - t1[rt][e] + t2[rt][e]);
      bar_arrive(kBarXFull + b, kThreads);
    }
    return;
  }

  // FP64 warps
  const int c = t - kTensorThreads, cw = c >> 5;
  const int a = c >> 2, row = c & 3;
  // Tile j into stage j & 1, one cp.async group.  (Computing each source
  // index in full spreads the copies out; issued back to back from
  // precomputed offsets they slowed the tensor warps' fragment loads.)
  auto issue = [&](int j) {
    const u64 base = (first + static_cast<u64>(j) * gridDim.x) << 12;
    double2 *st = stage + (j & 1) * 4096;
#pragma unroll
    for (int r = 0; r < 4096 / kFp64Threads; ++r) {
      const int tau = c + r * kFp64Threads;
      const u64 p = base | static_cast<u64>(tau);
      cp_async16(&st[mps_slot<4>(tau)], &lam[gather ? ring_p(p, n) : p]);
    }
    cp_async_commit();
  };
  if (my_tiles > 0) issue(0);
  if (my_tiles > 1) issue(1);
  if (my_tiles > 0) {
    if (my_tiles > 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else cp_async_wait_all();
    bar_arrive(kBarStageFull + 0, kThreads);
  }
  double2 g[4], f[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) g[j] = f[j] = make_double2(0.0, 0.0);
  const unsigned lomask = (1u << Q.m1) - 1u;
  for (int k = 0; k < my_tiles; ++k) {
    const int b = k & 1;
    const u64 tile = first + static_cast<u64>(k) * gridDim.x;
    if (k + 1 < my_tiles) {  // tile k + 1 (the only group in flight) has landed
      cp_async_wait_all();
      bar_arrive(kBarStageFull + (b ^ 1), kThreads);
    }
    if (k + 2 < my_tiles) {  // stage b is free once the tensor warps have read tile k
      bar_sync(kBarStageEmpty + b, kThreads);
      issue(k + 2);
    }
    if (c < E) {
      // C_t = CosLo(lo) CosHi(hi), entry c
      const unsigned lo = static_cast<unsigned>(tile) & lomask, hi = static_cast<unsigned>(tile >> Q.m1);
      const double2 *cl = Q.coslo + lo * E, *ch = Q.coshi + hi * E;
      const int i = c >> 2, j = c & 3;
      double2 s = cmul(__ldg(&cl[i * 4]), __ldg(&ch[j]));
#pragma unroll
      for (int kk = 1; kk < 4; ++kk) s = cfma(__ldg(&cl[i * 4 + kk]), __ldg(&ch[kk * 4 + j]), s);
      csm[b * E + c] = s;
    }
    // X of tile k written (and C of tile k visible)
    bar_sync(kBarXFull + b, kThreads);
    const double2 *x1 = xbuf + 2 * b * 64 * E, *x2 = x1 + 64 * E;
    const double2 *cc = csm + b * E;
    // Z partial: row `row` of M1(a) X1(a); G row += X1(a) row C; F row += C row X2(a)
    double2 p[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) p[j] = make_double2(0.0, 0.0);
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const double2 xk = x1[xslot(a, row * 4 + kk)], ck = cc[row * 4 + kk];
      const double2 mk = msm[mslot(a, row * 4 + kk)];  // M1(a) entry (row, kk)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        p[j] = cfma(mk, x1[xslot(a, kk * 4 + j)], p[j]);
        g[j] = cfma(xk, cc[kk * 4 + j], g[j]);
        f[j] = cfma(ck, x2[xslot(a, kk * 4 + j)], f[j]);
      }
    }
    if (k + 2 < my_tiles) bar_arrive(kBarXEmpty + b, kThreads);
    // Z partial summed over a's bits 0..2 (lane bits 2..4): a butterfly that
    // halves the entries a lane keeps at lane bits 2 and 3 (which end as the
    // entry's column bits 1 and 0), then a plain sum over lane bit 4
#pragma unroll
    for (int lv = 0; lv < 2; ++lv) {
      const int h = 2 >> lv;
      const bool up = (lane >> (2 + lv)) & 1;
#pragma unroll
      for (int e = 0; e < h; ++e) {
        const double2 send = up ? p[e] : p[e + h];
        const double2 keep = up ? p[e + h] : p[e];
        p[e] = cadd(keep, shfl_xor2(send, 4 << lv));
      }
    }
    p[0] = cadd(p[0], shfl_xor2(p[0], 16));
    if (lane < 16) zp[cw * E + row * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 3) & 1)] = p[0];
    bar_sync(kBarCons, kFp64Threads);
    if (c < E) {
      double2 z = zp[c];
#pragma unroll
      for (int w = 1; w < 8; ++w) z = cadd(z, zp[w * E + c]);
      Q.zt[tile * E + c] = z;
    }
  }
  double2 *rec = Q.partials + static_cast<size_t>(blockIdx.x) * 2 * 64 * E + a * E + row * 4;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    rec[j] = g[j];
    rec[64 * E + j] = f[j];
  }
}

// Y(lo) = sum_hi CosHi(hi) Z(lo, hi)   (blocks 0 .. 2^m1 - 1)
// Y'(hi) = sum_lo Z(lo, hi) CosLo(lo)  (blocks 2^m1 .. 2^m1 + 2^m2 - 1)
template <int D>
__global__ void __launch_bounds__(64) mps_coset_kernel(const MpsParams Q) {
  constexpr int E = D * D;
  __shared__ double2 red[64][E];
  const int t = threadIdx.x;
  const int nlo = 1 << Q.m1, nhi = 1 << Q.m2;
  const int b = blockIdx.x;
  Mat<D> acc;
#pragma unroll
  for (int e = 0; e < E; ++e) acc.m[e] = make_double2(0.0, 0.0);
  if (b < nlo) {
    for (int hi = t; hi < nhi; hi += 64) {
      const Mat<D> p = mmul<D>(ldg_mat<D>(Q.coshi + hi * E), ldg_mat<D>(Q.zt + (static_cast<u64>(b) + (static_cast<u64>(hi) << Q.m1)) * E));
#pragma unroll
      for (int e = 0; e < E; ++e) acc.m[e] = cadd(acc.m[e], p.m[e]);
    }
  } else {
    const int hi = b - nlo;
    for (int lo = t; lo < nlo; lo += 64) {
      const Mat<D> p = mmul<D>(ldg_mat<D>(Q.zt + (static_cast<u64>(lo) + (static_cast<u64>(hi) << Q.m1)) * E), ldg_mat<D>(Q.coslo + lo * E));
#pragma unroll
      for (int e = 0; e < E; ++e) acc.m[e] = cadd(acc.m[e], p.m[e]);
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) red[t][e] = acc.m[e];
  __syncthreads();
  for (int s = 32; s > 0; s >>= 1) {
    if (t < s)
#pragma unroll
      for (int e = 0; e < E; ++e) red[t][e] = cadd(red[t][e], red[t + s][e]);
    __syncthreads();
  }
  if (t < E) (b < nlo ? Q.ylo + b * E : Q.yhi + (b - nlo) * E)[t] = red[0][t];
}

// G and F summed over the gradient kernel's CTAs, in CTA order
template <int D>
__global__ void mps_reduce_kernel(const MpsParams Q, int grid) {
  constexpr int E = D * D;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * 64 * E) return;
  double2 s = make_double2(0.0, 0.0);
  for (int c = 0; c < grid; ++c) s = cadd(s, Q.partials[static_cast<size_t>(c) * 2 * 64 * E + i]);
  Q.gf[i] = s;
}

// Block w: E_w[0], E_w[1] from the leave-one-out products over wire w's group
// of bits, then the 2K gradients of wire w (layers 0 .. K-1).
template <int D>
__global__ void __launch_bounds__(64) mps_finalize_kernel(const MpsParams Q, double *__restrict__ grad_out) {
  constexpr int E = D * D;
  constexpr int K = D == 2 ? 2 : 3;
  __shared__ double2 red[64][2 * E];
  __shared__ double2 env[2 * E];
  const int t = threadIdx.x, w = blockIdx.x, n = Q.n;
  // group of wire w: its first wire, bit count, values and their source
  int g0, nb, count;
  const double2 *src;
  if (w < 6) {
    g0 = 0; nb = 6; count = 64; src = Q.gf;
  } else if (w < 12) {
    g0 = 6; nb = 6; count = 64; src = Q.gf + 64 * E;
  } else if (w < 12 + Q.m1) {
    g0 = 12; nb = Q.m1; count = 1 << Q.m1; src = Q.ylo;
  } else {
    g0 = 12 + Q.m1; nb = Q.m2; count = 1 << Q.m2; src = Q.yhi;
  }
  const int bit = w - g0;
  Mat<D> acc[2];
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int e = 0; e < E; ++e) acc[b].m[e] = make_double2(0.0, 0.0);
  for (int x = t; x < count; x += 64) {
    const unsigned v = static_cast<unsigned>(x);
    // post = sites w+1 .. g0+nb-1, pre = sites g0 .. w-1, with the bits of x
    const Mat<D> post = site_chain<D>(Q.tsite, w + 1, g0 + nb - (w + 1), v >> (bit + 1));
    const Mat<D> pre = site_chain<D>(Q.tsite, g0, bit, v);
    const Mat<D> term = mmul<D>(mmul<D>(post, load_mat<D>(src + x * E)), pre);
    const int b = (x >> bit) & 1;
#pragma unroll
    for (int e = 0; e < E; ++e) acc[b].m[e] = cadd(acc[b].m[e], term.m[e]);
  }
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int e = 0; e < E; ++e) red[t][b * E + e] = acc[b].m[e];
  __syncthreads();
  for (int s = 32; s > 0; s >>= 1) {
    if (t < s)
      for (int e = 0; e < 2 * E; ++e) red[t][e] = cadd(red[t][e], red[t + s][e]);
    __syncthreads();
  }
  if (t < 2 * E) env[t] = red[0][t];
  __syncthreads();
  if (t < 2 * K) {
    const int layer = t >> 1, kind = 1 + (t & 1);
    Mat<D> dT[2];
    site_tensor<D>(Q.coef, n, w, layer, kind, dT);
    double s = 0.0;
    for (int b = 0; b < 2; ++b)
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) s += cmul(dT[b].m[i * D + j], env[b * E + j * D + i]).x;
    grad_out[2 * (layer * n + w) + (t & 1)] = 2.0 * s;
  }
}

template <int D>
cudaError_t launch_grad_d(const MpsParams &Q, const double2 *lam, int gather, int grid, cudaStream_t s) {
  if constexpr (D == 4) {
    static std::atomic<unsigned long long> configured{0};
    const cudaError_t e = set_smem_limit_once(mps_grad4_kernel, mg4::kSmem, configured);
    if (e != cudaSuccess) return e;
    mps_grad4_kernel<<<grid, mg4::kThreads, mg4::kSmem, s>>>(Q, lam, gather);
  } else {
    static std::atomic<unsigned long long> configured{0};
    const cudaError_t e = set_smem_limit_once(mps_grad_kernel<D>, mps_grad_smem<D>(), configured);
    if (e != cudaSuccess) return e;
    mps_grad_kernel<D><<<grid, kMpsThreads, mps_grad_smem<D>(), s>>>(Q, lam, gather);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  mps_coset_kernel<D><<<(1 << Q.m1) + (1 << Q.m2), 64, 0, s>>>(Q);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  mps_reduce_kernel<D><<<(2 * 64 * D * D + 255) / 256, 256, 0, s>>>(Q, grid);
  return cudaGetLastError();
}

}  // namespace

size_t mps_partials_count(int bond) { return static_cast<size_t>(2) * 64 * bond * bond; }

cudaError_t launch_mps_tables(const MpsParams &Q, cudaStream_t s) {
  if (Q.n < 13 || Q.n > 31 || (Q.bond != 2 && Q.bond != 4)) return cudaErrorInvalidValue;
  const int count = 1024 + (1 << Q.m1) + (1 << Q.m2) + 128 + (1 << (Q.n > 16 ? Q.n - 16 : 0));
  if (Q.bond == 2) {
    mps_site_kernel<2><<<1, 32, 0, s>>>(Q);
    mps_tables_kernel<2><<<(count + 127) / 128, 128, 0, s>>>(Q);
  } else {
    mps_site_kernel<4><<<1, 32, 0, s>>>(Q);
    mps_tables_kernel<4><<<(count + 127) / 128, 128, 0, s>>>(Q);
  }
  return cudaGetLastError();
}

cudaError_t launch_mps_forward(const MpsParams &Q, double2 *out, int scatter, int grid, cudaStream_t s) {
  if (Q.bond == 2) {
    if (scatter) mps_fwd_kernel<2, true><<<grid, 256, 0, s>>>(Q, out);
    else mps_fwd_kernel<2, false><<<grid, 256, 0, s>>>(Q, out);
  } else if (Q.bond == 4) {
    if (scatter) mps_fwd_kernel<4, true><<<grid, 256, 0, s>>>(Q, out);
    else mps_fwd_kernel<4, false><<<grid, 256, 0, s>>>(Q, out);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_mps_grad(const MpsParams &Q, const double2 *lam, int gather, int grid, cudaStream_t s) {
  if (Q.bond == 2) return launch_grad_d<2>(Q, lam, gather, grid, s);
  if (Q.bond == 4) return launch_grad_d<4>(Q, lam, gather, grid, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_mps_finalize(const MpsParams &Q, double *grad_out, cudaStream_t s) {
  if (Q.bond == 2) mps_finalize_kernel<2><<<Q.n, 64, 0, s>>>(Q, grad_out);
  else if (Q.bond == 4) mps_finalize_kernel<4><<<Q.n, 64, 0, s>>>(Q, grad_out);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace rsv
