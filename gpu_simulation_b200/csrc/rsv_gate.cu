// Gate-level inverse walk (gradient_strategy "inverse_walk_cuQuantum"): the
// ansatz as separate RY, RZ and CNOT gates on a complex128 statevector in the
// reference's gate order, the Hamiltonian applied to the final state, and the
// adjoint walk back over the gates -- each gate's gradient sum, then its
// inverse applied to psi and lambda, in one kernel.  It replaces the
// reference's cuStateVec path (cpp/ising_cuda_gate_level_adjoint_modes.inc:
// 147-260, gate kernels cpp/ising_cuda_gate_kernels.cu) with own kernels, and
// serves as a second GPU parity path for the structured engine.
#include <algorithm>

#include "rsv_device.cuh"
#include "rsv_gate.h"

namespace rsv {
namespace {

constexpr int kGateThreads = 256;

__device__ __forceinline__ u64 pair_index(u64 k, int w) {
  const u64 lo = k & ((u64{1} << w) - 1);
  return ((k >> w) << (w + 1)) | lo;
}

__global__ void zero_state_kernel(double2 *psi, u64 size) {
  for (u64 i = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; i < size;
       i += static_cast<u64>(gridDim.x) * blockDim.x)
    psi[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
}

// Forward gates (in place).
__global__ void ry_kernel(double2 *psi, u64 pairs, int w, const double4 *coef, int k) {
  const double c = coef[k].x, s = coef[k].y;
  const u64 m = u64{1} << w;
  for (u64 t = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; t < pairs;
       t += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 i0 = pair_index(t, w), i1 = i0 | m;
    const double2 a0 = psi[i0], a1 = psi[i1];
    psi[i0] = make_double2(c * a0.x - s * a1.x, c * a0.y - s * a1.y);
    psi[i1] = make_double2(s * a0.x + c * a1.x, s * a0.y + c * a1.y);
  }
}

__global__ void rz_kernel(double2 *psi, u64 pairs, int w, const double4 *coef, int k) {
  const double c = coef[k].z, s = coef[k].w;  // e^{-i phi/2} on |0>, e^{+i phi/2} on |1>
  const u64 m = u64{1} << w;
  for (u64 t = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; t < pairs;
       t += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 i0 = pair_index(t, w), i1 = i0 | m;
    const double2 a0 = psi[i0], a1 = psi[i1];
    psi[i0] = make_double2(c * a0.x + s * a0.y, c * a0.y - s * a0.x);
    psi[i1] = make_double2(c * a1.x - s * a1.y, c * a1.y + s * a1.x);
  }
}

// CNOT(control, target): swap the target pair where the control bit is 1.
__device__ __forceinline__ void cnot_pair(u64 t, int control, int target, u64 *i0, u64 *i1) {
  const int lo = min(control, target), hi = max(control, target);
  u64 x = pair_index(t, lo);        // insert a 0 at the lower bit
  x = pair_index(x, hi);            // and at the higher bit
  x |= u64{1} << control;
  *i0 = x;
  *i1 = x | (u64{1} << target);
}

__global__ void cnot_kernel(double2 *psi, u64 quads, int control, int target) {
  for (u64 t = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; t < quads;
       t += static_cast<u64>(gridDim.x) * blockDim.x) {
    u64 i0, i1;
    cnot_pair(t, control, target, &i0, &i1);
    const double2 a = psi[i0];
    psi[i0] = psi[i1];
    psi[i1] = a;
  }
}

__device__ __forceinline__ void block_sum(double v, double *out) {
  __shared__ double red[kGateThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < kGateThreads / 32; ++i) s += red[i];
    *out = s;
  }
}

// lambda = H psi (post-ring frame: -sum Z_w Z_{w+1} - h sum X_w) and energy partials
// (reference cpp/ising_cuda_kernels.cu:313-358).
__global__ void __launch_bounds__(kGateThreads) hamiltonian_kernel(const double2 *__restrict__ psi,
                                                                   double2 *__restrict__ lam, u64 size,
                                                                   int n, double field, double *partials) {
  const u64 mask = (u64{1} << n) - 1;
  double e = 0.0;
  for (u64 i = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; i < size;
       i += static_cast<u64>(gridDim.x) * blockDim.x) {
    const double2 c = psi[i];
    const u64 rot = ((i << 1) & mask) | (i >> (n - 1));
    const double d = static_cast<double>(2 * __popcll(i ^ rot)) - static_cast<double>(n);
    double2 x = make_double2(0.0, 0.0);
    for (int w = 0; w < n; ++w) {
      const double2 t = psi[i ^ (u64{1} << w)];
      x.x += t.x;
      x.y += t.y;
    }
    const double2 m = make_double2(fma(d, c.x, -field * x.x), fma(d, c.y, -field * x.y));
    lam[i] = m;
    e += fma(c.x, m.x, c.y * m.y);
  }
  block_sum(e, &partials[blockIdx.x]);
}

// Inverse walk of one RY: gradient sum Re(conj(l1) a0) - Re(conj(l0) a1) over the
// wire's pairs of psi (after the gate) and lambda, then RY^dagger on both.
__global__ void __launch_bounds__(kGateThreads) walk_ry_kernel(double2 *psi, double2 *lam, u64 pairs, int w,
                                                               const double4 *coef, int k, double *partials) {
  const double c = coef[k].x, s = coef[k].y;
  const u64 m = u64{1} << w;
  double g = 0.0;
  for (u64 t = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; t < pairs;
       t += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 i0 = pair_index(t, w), i1 = i0 | m;
    const double2 a0 = psi[i0], a1 = psi[i1], l0 = lam[i0], l1 = lam[i1];
    g += (l1.x * a0.x + l1.y * a0.y) - (l0.x * a1.x + l0.y * a1.y);
    psi[i0] = make_double2(c * a0.x + s * a1.x, c * a0.y + s * a1.y);
    psi[i1] = make_double2(c * a1.x - s * a0.x, c * a1.y - s * a0.y);
    lam[i0] = make_double2(c * l0.x + s * l1.x, c * l0.y + s * l1.y);
    lam[i1] = make_double2(c * l1.x - s * l0.x, c * l1.y - s * l0.y);
  }
  block_sum(g, &partials[blockIdx.x]);
}

// Inverse walk of one RZ: gradient sum Im(conj(l0) a0) - Im(conj(l1) a1), then
// RZ^dagger on both.
__global__ void __launch_bounds__(kGateThreads) walk_rz_kernel(double2 *psi, double2 *lam, u64 pairs, int w,
                                                               const double4 *coef, int k, double *partials) {
  const double c = coef[k].z, s = coef[k].w;
  const u64 m = u64{1} << w;
  double g = 0.0;
  for (u64 t = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; t < pairs;
       t += static_cast<u64>(gridDim.x) * blockDim.x) {
    const u64 i0 = pair_index(t, w), i1 = i0 | m;
    const double2 a0 = psi[i0], a1 = psi[i1], l0 = lam[i0], l1 = lam[i1];
    g += (l0.x * a0.y - l0.y * a0.x) - (l1.x * a1.y - l1.y * a1.x);
    // RZ^dagger: e^{+i phi/2} on |0>, e^{-i phi/2} on |1>
    psi[i0] = make_double2(c * a0.x - s * a0.y, c * a0.y + s * a0.x);
    psi[i1] = make_double2(c * a1.x + s * a1.y, c * a1.y - s * a1.x);
    lam[i0] = make_double2(c * l0.x - s * l0.y, c * l0.y + s * l0.x);
    lam[i1] = make_double2(c * l1.x + s * l1.y, c * l1.y - s * l1.x);
  }
  block_sum(g, &partials[blockIdx.x]);
}

__global__ void walk_cnot_kernel(double2 *psi, double2 *lam, u64 quads, int control, int target) {
  for (u64 t = blockIdx.x * static_cast<u64>(blockDim.x) + threadIdx.x; t < quads;
       t += static_cast<u64>(gridDim.x) * blockDim.x) {
    u64 i0, i1;
    cnot_pair(t, control, target, &i0, &i1);
    const double2 a = psi[i0], l = lam[i0];
    psi[i0] = psi[i1];
    psi[i1] = a;
    lam[i0] = lam[i1];
    lam[i1] = l;
  }
}

// Fixed-order sums of the per-CTA partials: energy and every gradient entry.
__global__ void gate_finalize_kernel(const double *energy_partials, int grid, const double *grad_partials,
                                     int num_params, double *energy_out, double *grad_out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < grid; ++b) s += energy_partials[b];
    *energy_out = s;
  }
  if (grad_out == nullptr) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < num_params; k += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < grid; ++b) s += grad_partials[static_cast<size_t>(k) * grid + b];
    grad_out[k] = s;
  }
}

}  // namespace

int gate_grid(int n, int sms) {
  const u64 pairs = u64{1} << (n - 1);
  const u64 blocks = (pairs + kGateThreads - 1) / kGateThreads;
  return static_cast<int>(std::max<u64>(1, std::min<u64>(blocks, static_cast<u64>(sms) * 8)));
}

cudaError_t run_gate_level(const GateLevelArgs &A, cudaStream_t s) {
  const int n = A.n, L = A.L, grid = A.grid;
  const u64 size = u64{1} << n, pairs = size / 2, quads = size / 4;
  zero_state_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, size);  // |0...0>
  // forward: per layer RY, RZ on every wire, then CNOT(w, w+1 mod n)
  // (reference gate order, ring_ising/backends/standalone/ops.py and
  // cpp/ising_cuda_backend.cu build_ops_for_strategy)
  for (int l = 0; l < L; ++l) {
    for (int w = 0; w < n; ++w) {
      ry_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, pairs, w, A.coef, l * n + w);
      rz_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, pairs, w, A.coef, l * n + w);
    }
    for (int w = 0; w < n; ++w) cnot_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, quads, w, (w + 1) % n);
  }
  hamiltonian_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, A.lam, size, n, A.field, A.energy_partials);
  if (A.grad_out != nullptr) {
    for (int l = L - 1; l >= 0; --l) {
      for (int w = n - 1; w >= 0; --w)
        walk_cnot_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, A.lam, quads, w, (w + 1) % n);
      for (int w = n - 1; w >= 0; --w) {
        const int k = l * n + w;
        walk_rz_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, A.lam, pairs, w, A.coef, k,
                                                     A.grad_partials + static_cast<size_t>(2 * k + 1) * grid);
        walk_ry_kernel<<<grid, kGateThreads, 0, s>>>(A.psi, A.lam, pairs, w, A.coef, k,
                                                     A.grad_partials + static_cast<size_t>(2 * k) * grid);
      }
    }
  }
  gate_finalize_kernel<<<std::max(1, (2 * n * L + 255) / 256), 256, 0, s>>>(
      A.energy_partials, grid, A.grad_partials, 2 * n * L, A.energy_out, A.grad_out);
  return cudaGetLastError();
}

}  // namespace rsv
