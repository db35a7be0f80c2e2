// dense_scan (n <= 8): every layer as a dense 2^n x 2^n complex matrix
// Q_l = C R_l (R_l = the tensor product of the wires' RZ.RY, C = the CNOT ring
// permutation), a product tree of the layer matrices built with FP64 tensor
// cores (mma.sync m8n8k4 f64: tcgen05 has no FP64 kind), the final state
// T e_0, lambda = H psi, eta = T^H lambda, a down-sweep of the tree that gives
// every layer's input state and adjoint vector, and the per-layer gradient
// tail.  Replaces the reference's cuBLAS pipeline
// (cpp/ising_cuda_dense_modes.inc:96-347: cublasZgemmStridedBatched up-sweep,
// batched matvec down-sweep; kernels cpp/ising_cuda_dense_kernels.cu:114-304),
// with its rotation and CNOT layers merged into one matrix per layer.
//
// Matrices are row-major complex128 (double2), dim x dim.
#include <algorithm>
#include <vector>

#include "rsv_dense.h"
#include "rsv_device.cuh"

namespace rsv {
namespace {

// ---------------------------------------------------------------- layers
// Q_l[row][col] = R_l[P^{-1}(row)][col]; R_l[r][c] = prod_w u_w[r_w][c_w] with
// u = diag(e^{-i phi/2}, e^{i phi/2}) [[c, -s], [s, c]].
__device__ __forceinline__ double2 u_entry(double4 k, int r, int c) {
  const double ry = (r == c) ? k.x : (r == 0 ? -k.y : k.y);  // RY entry
  return r == 0 ? make_double2(ry * k.z, -ry * k.w) : make_double2(ry * k.z, ry * k.w);  // row phase
}

__global__ void layer_matrix_kernel(const double4 *__restrict__ coef, int n, int dim, double2 *__restrict__ q) {
  const int layer = blockIdx.y;
  const int row = blockIdx.x;
  const int src = static_cast<int>(ring_pinv(static_cast<u64>(row), n));
  for (int col = threadIdx.x; col < dim; col += blockDim.x) {
    double2 v = make_double2(1.0, 0.0);
    for (int w = 0; w < n; ++w) v = cmul(v, u_entry(coef[layer * n + w], (src >> w) & 1, (col >> w) & 1));
    q[(static_cast<size_t>(layer) * dim + row) * dim + col] = v;
  }
}

__global__ void identity_kernel(double2 *q, int dim, int count) {
  const size_t total = static_cast<size_t>(count) * dim * dim;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t e = i % (static_cast<size_t>(dim) * dim);
    q[i] = make_double2((e / dim) == (e % dim) ? 1.0 : 0.0, 0.0);
  }
}

// ---------------------------------------------------------------- GEMM
// C[b] = A[b] B[b], complex, dim x dim, dim a multiple of 32.  A CTA of 4
// warps computes a 32 x 32 tile; a warp 16 x 16 = 2 x 2 tiles of the
// m8n8k4 f64 MMA, each complex product as three real MMAs (Gauss).  K
// advances 16 at a time through a double-buffered shared-memory stage filled
// by cp.async while the previous stage feeds the MMAs; the rows are padded so
// that every fragment load is free of bank conflicts.
constexpr int kGT = 32;
constexpr int kGK = 16;
constexpr int kAP = kGK + 4;  // A row pitch (16-byte elements)
constexpr int kBP = kGT + 2;  // B row pitch

__device__ __forceinline__ void cp16(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__global__ void __launch_bounds__(128) zgemm_tc_kernel(const double2 *__restrict__ A, const double2 *__restrict__ B,
                                                       double2 *__restrict__ C, int dim, long long sa,
                                                       long long sb, long long sc) {
  __shared__ __align__(16) double2 As[2][kGT * kAP];
  __shared__ __align__(16) double2 Bs[2][kGK * kBP];
  A += blockIdx.z * sa;
  B += blockIdx.z * sb;
  C += blockIdx.z * sc;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = warp >> 1, wc = warp & 1;
  const int row0 = blockIdx.y * kGT, col0 = blockIdx.x * kGT;
  const int g = lane >> 2, t = lane & 3;
  auto stage = [&](int buf, int k0) {
#pragma unroll
    for (int j = 0; j < (kGT * kGK) / 128; ++j) {
      const int i = threadIdx.x + j * 128;
      const int r = i / kGK, c = i % kGK;
      cp16(&As[buf][r * kAP + c], &A[static_cast<size_t>(row0 + r) * dim + k0 + c]);
      const int rb = i / kGT, cb = i % kGT;
      cp16(&Bs[buf][rb * kBP + cb], &B[static_cast<size_t>(k0 + rb) * dim + col0 + cb]);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  // t1 = ar br, t2 = ai bi, t3 = (ar + ai)(br + bi); re = t1 - t2, im = t3 - t1 - t2
  double t1[2][2][2] = {}, t2[2][2][2] = {}, t3[2][2][2] = {};
  stage(0, 0);
  for (int k0 = 0, buf = 0; k0 < dim; k0 += kGK, buf ^= 1) {
    if (k0 + kGK < dim) {
      stage(buf ^ 1, k0 + kGK);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();
    const double2 *as = As[buf];
    const double2 *bs = Bs[buf];
#pragma unroll
    for (int kk = 0; kk < kGK; kk += 4) {
      double2 a[2], b[2];
#pragma unroll
      for (int tm = 0; tm < 2; ++tm) a[tm] = as[(wr * 16 + tm * 8 + g) * kAP + kk + t];
#pragma unroll
      for (int tn = 0; tn < 2; ++tn) b[tn] = bs[(kk + t) * kBP + wc * 16 + tn * 8 + g];
#pragma unroll
      for (int tm = 0; tm < 2; ++tm)
#pragma unroll
        for (int tn = 0; tn < 2; ++tn) {
          mma_f64(t1[tm][tn][0], t1[tm][tn][1], a[tm].x, b[tn].x);
          mma_f64(t2[tm][tn][0], t2[tm][tn][1], a[tm].y, b[tn].y);
          mma_f64(t3[tm][tn][0], t3[tm][tn][1], a[tm].x + a[tm].y, b[tn].x + b[tn].y);
        }
    }
    __syncthreads();  // the next iteration's cp.async overwrites this stage
  }
#pragma unroll
  for (int tm = 0; tm < 2; ++tm)
#pragma unroll
    for (int tn = 0; tn < 2; ++tn) {
      const size_t r = row0 + wr * 16 + tm * 8 + g;
      const int c = col0 + wc * 16 + tn * 8 + 2 * t;
#pragma unroll
      for (int e = 0; e < 2; ++e)
        C[r * dim + c + e] =
            make_double2(t1[tm][tn][e] - t2[tm][tn][e], t3[tm][tn][e] - t1[tm][tn][e] - t2[tm][tn][e]);
    }
}

// dim < 32 (n <= 4): one output element per thread on the FP64 pipe.
__global__ void zgemm_small_kernel(const double2 *__restrict__ A, const double2 *__restrict__ B,
                                   double2 *__restrict__ C, int dim, long long sa, long long sb, long long sc) {
  A += blockIdx.z * sa;
  B += blockIdx.z * sb;
  C += blockIdx.z * sc;
  for (int e = threadIdx.x; e < dim * dim; e += blockDim.x) {
    const int r = e / dim, c = e % dim;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < dim; ++k) {
      const double2 a = A[r * dim + k], b = B[k * dim + c];
      acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
      acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
    }
    C[e] = acc;
  }
}

// ---------------------------------------------------------------- vectors
// eta = T^H lambda (one CTA, dim <= 256).
__global__ void adjoint_matvec_kernel(const double2 *__restrict__ M, const double2 *__restrict__ x,
                                      double2 *__restrict__ out, int dim) {
  for (int r = threadIdx.x; r < dim; r += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < dim; ++k) {
      const double2 m = M[static_cast<size_t>(k) * dim + r], v = x[k];  // conj(m) v
      acc.x = fma(m.x, v.x, fma(m.y, v.y, acc.x));
      acc.y = fma(m.x, v.y, fma(-m.y, v.x, acc.y));
    }
    out[r] = acc;
  }
}

// psi = T e_0 (column 0 of the root), lambda = H psi, energy = <psi|lambda>,
// with H = -sum Z_w Z_{w+1} - h sum X_w; one CTA of 256 threads (dim <= 256).
__global__ void __launch_bounds__(256) energy_dense_kernel(const double2 *__restrict__ T, int n, int dim,
                                                           double field, double2 *__restrict__ lam,
                                                           double *__restrict__ energy_out) {
  __shared__ double2 s_psi[256];
  __shared__ double red[256];
  for (int i = threadIdx.x; i < dim; i += blockDim.x) s_psi[i] = T[static_cast<size_t>(i) * dim];
  __syncthreads();
  double e = 0.0;
  const int mask = dim - 1;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    const int rot = ((i << 1) & mask) | (i >> (n - 1));
    const double d = static_cast<double>(2 * __popc(i ^ rot)) - static_cast<double>(n);
    const double2 c = s_psi[i];
    double2 x = make_double2(0.0, 0.0);
    for (int w = 0; w < n; ++w) {
      const double2 t = s_psi[i ^ (1 << w)];
      x.x += t.x;
      x.y += t.y;
    }
    const double2 m = make_double2(fma(d, c.x, -field * x.x), fma(d, c.y, -field * x.y));
    lam[i] = m;
    e += fma(c.x, m.x, c.y * m.y);
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *energy_out = red[0];
}

__global__ void seed_kernel(double2 *x, double2 *y, const double2 *eta, int dim) {
  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    x[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
    y[i] = eta[i];
  }
}

// child vectors of one tree level: child[2p] = parent[p],
// child[2p+1] = left[2p] parent[p] (left = the products of the child level).
// CTA (p, v) handles parent p of vector set v (0: x, 1: y); a warp per row
// reads the row with consecutive lanes (coalesced) and reduces with shuffles.
__global__ void __launch_bounds__(256) downsweep_kernel(const double2 *__restrict__ left,
                                                        const double2 *__restrict__ parent_x,
                                                        const double2 *__restrict__ parent_y,
                                                        double2 *__restrict__ child_x,
                                                        double2 *__restrict__ child_y, int dim) {
  const int p = blockIdx.x;
  const double2 *parent = blockIdx.y == 0 ? parent_x : parent_y;
  double2 *child = blockIdx.y == 0 ? child_x : child_y;
  const double2 *M = left + static_cast<size_t>(2 * p) * dim * dim;
  const double2 *x = parent + static_cast<size_t>(p) * dim;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = warp; r < dim; r += blockDim.x >> 5) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = lane; k < dim; k += 32) {
      const double2 m = M[static_cast<size_t>(r) * dim + k], v = x[k];
      acc.x = fma(m.x, v.x, fma(-m.y, v.y, acc.x));
      acc.y = fma(m.x, v.y, fma(m.y, v.x, acc.y));
    }
    acc.x = warp_sum(acc.x);
    acc.y = warp_sum(acc.y);
    if (lane == 0) child[static_cast<size_t>(2 * p + 1) * dim + r] = acc;
  }
  for (int r = threadIdx.x; r < dim; r += blockDim.x) child[static_cast<size_t>(2 * p) * dim + r] = x[r];
}

// Per layer (one CTA): with x_l the state before the layer and y_l the tree's
// adjoint vector (so that R_l y_l is the adjoint after the layer's rotations),
//   dE/dtheta_w = 2 Re <R_l y_l | R_l(U_w -> dU_w) x_l> = 2 Re <y_l | (U_w^H dU_w)_w x_l>,
// because R_l^H R_l(U_w -> dU_w) acts as U_w^H dU_w on wire w alone.  With
// U = RZ(phi) RY(theta): U^H dU/dtheta = -i/2 Y (Pauli) and U^H dU/dphi =
// -i/2 RY^H Z RY = -i/2 [[cos t, -sin t], [-sin t, -cos t]], so
//   dE/dtheta_w = sum over pairs Re(conj(y1) x0 - conj(y0) x1),
//   dE/dphi_w   = Im <y | M_w | x>,  M_w = [[cos t, -sin t], [-sin t, -cos t]].
// The reference applies the whole layer once per derivative
// (rotation_layer_dense_gradient_tail_kernel, cpp/ising_cuda_dense_kernels.cu:154-270).
__global__ void __launch_bounds__(256) dense_grad_kernel(const double4 *__restrict__ coef,
                                                         const double2 *__restrict__ xs,
                                                         const double2 *__restrict__ ys, int n, int dim,
                                                         double *__restrict__ grad) {
  __shared__ double2 x[256], y[256];
  __shared__ double red[8][2 * kDenseMaxQubits];
  const int layer = blockIdx.x;
  for (int i = threadIdx.x; i < dim; i += blockDim.x) {
    x[i] = xs[static_cast<size_t>(layer) * dim + i];
    y[i] = ys[static_cast<size_t>(layer) * dim + i];
  }
  __syncthreads();
  double acc[2 * kDenseMaxQubits];
#pragma unroll
  for (int j = 0; j < 2 * kDenseMaxQubits; ++j) acc[j] = 0.0;
#pragma unroll
  for (int w = 0; w < kDenseMaxQubits; ++w) {
    if (w >= n) break;
    const double4 k = coef[layer * n + w];
    const double ct = k.x * k.x - k.y * k.y, st = 2.0 * k.x * k.y;  // cos theta, sin theta
    for (int pr = threadIdx.x; pr < dim / 2; pr += blockDim.x) {
      const int i0 = ((pr >> w) << (w + 1)) | (pr & ((1 << w) - 1)), i1 = i0 | (1 << w);
      const double2 x0 = x[i0], x1 = x[i1], y0 = y[i0], y1 = y[i1];
      acc[2 * w] += (y1.x * x0.x + y1.y * x0.y) - (y0.x * x1.x + y0.y * x1.y);
      const double2 m0 = make_double2(ct * x0.x - st * x1.x, ct * x0.y - st * x1.y);
      const double2 m1 = make_double2(-st * x0.x - ct * x1.x, -st * x0.y - ct * x1.y);
      acc[2 * w + 1] += (y0.x * m0.y - y0.y * m0.x) + (y1.x * m1.y - y1.y * m1.x);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 2 * kDenseMaxQubits; ++j) {
    const double s = warp_sum(acc[j]);
    if (lane == 0) red[warp][j] = s;
  }
  __syncthreads();
  if (threadIdx.x < 2 * n) {
    double s = 0.0;
    for (int ww = 0; ww < static_cast<int>(blockDim.x >> 5); ++ww) s += red[ww][threadIdx.x];
    grad[2 * layer * n + threadIdx.x] = s;
  }
}

}  // namespace

int dense_padded_layers(int L) {
  int p = 1;
  while (p < L) p <<= 1;
  return p;
}

size_t dense_workspace_bytes(int n, int L) {
  const size_t dim = size_t{1} << n, mat = dim * dim, P = static_cast<size_t>(dense_padded_layers(L));
  // tree: P leaves + P - 1 internal matrices; x and y vectors per leaf (two
  // ping-pong sets each); lambda and eta
  return sizeof(double2) * ((2 * P - 1) * mat + 4 * P * dim + 2 * dim);
}

cudaError_t zgemm_batched(const double2 *A, const double2 *B, double2 *C, int dim, int batch, long long sa,
                          long long sb, long long sc, cudaStream_t s) {
  if (dim >= kGT) {
    const dim3 grid(dim / kGT, dim / kGT, batch);
    zgemm_tc_kernel<<<grid, 128, 0, s>>>(A, B, C, dim, sa, sb, sc);
  } else {
    zgemm_small_kernel<<<dim3(1, 1, batch), 256, 0, s>>>(A, B, C, dim, sa, sb, sc);
  }
  return cudaGetLastError();
}

cudaError_t run_dense_scan(const DenseArgs &D, cudaStream_t s) {
  const int n = D.n, L = D.L, dim = 1 << n;
  const int P = dense_padded_layers(L);
  const size_t mat = static_cast<size_t>(dim) * dim;
  double2 *leaves = D.work;                                    // P matrices
  double2 *internal = leaves + static_cast<size_t>(P) * mat;   // P - 1: levels P/2, P/4, ..., 1
  double2 *xa = internal + static_cast<size_t>(P - 1) * mat;  // P vectors each
  double2 *xb = xa + static_cast<size_t>(P) * dim;
  double2 *ya = xb + static_cast<size_t>(P) * dim;
  double2 *yb = ya + static_cast<size_t>(P) * dim;
  double2 *lam = yb + static_cast<size_t>(P) * dim;
  double2 *eta = lam + dim;

  if (P > L) identity_kernel<<<64, 256, 0, s>>>(leaves + static_cast<size_t>(L) * mat, dim, P - L);
  layer_matrix_kernel<<<dim3(dim, L), std::min(dim, 256), 0, s>>>(D.coef, n, dim, leaves);
  // up-sweep: parent[p] = level[2p+1] level[2p] (the later layer on the left)
  std::vector<const double2 *> level_ptr{leaves};  // index i: the level with P >> i products
  double2 *cur = leaves, *out = internal;
  for (int count = P; count > 1; count /= 2) {
    const cudaError_t e = zgemm_batched(cur + mat, cur, out, dim, count / 2, static_cast<long long>(2 * mat),
                                        static_cast<long long>(2 * mat), static_cast<long long>(mat), s);
    if (e != cudaSuccess) return e;
    cur = out;
    out += static_cast<size_t>(count / 2) * mat;
    level_ptr.push_back(cur);
  }
  const double2 *root = cur;
  energy_dense_kernel<<<1, 256, 0, s>>>(root, n, dim, D.field, lam, D.energy_out);
  if (D.grad_out == nullptr) return cudaGetLastError();
  adjoint_matvec_kernel<<<1, 256, 0, s>>>(root, lam, eta, dim);  // eta = T^H lambda
  // down-sweep of x (from e_0) and y (from eta) to the leaves
  seed_kernel<<<1, 256, 0, s>>>(xa, ya, eta, dim);
  int depth = static_cast<int>(level_ptr.size()) - 1;  // index of the root level
  for (int count = 1; count < P; count *= 2) {
    const double2 *left = level_ptr[static_cast<size_t>(--depth)];  // the level with 2 * count products
    downsweep_kernel<<<dim3(count, 2), 256, 0, s>>>(left, xa, ya, xb, yb, dim);
    std::swap(xa, xb);
    std::swap(ya, yb);
  }
  dense_grad_kernel<<<L, 256, 0, s>>>(D.coef, xa, ya, n, dim, D.grad_out);
  return cudaGetLastError();
}

}  // namespace rsv
