// Device-side building blocks shared by the ring-Ising statevector kernels.
//
// Conventions (identical to the reference, zzEncounter/GPU_Simulation):
//   * amplitude index bit w is wire w (cpp/ising_cuda_kernels.cu:22-25);
//   * RY(t) = [[c,-s],[s,c]], c = cos(t/2), s = sin(t/2);
//     RZ(p) = diag(e^{-ip/2}, e^{+ip/2}); per wire U = RZ RY
//     (cpp/ising_cuda_rotation_kernels.cu:43-59);
//   * one layer = U on every wire, then CNOT(0,1), ..., CNOT(n-1,0).  The CNOT
//     ring maps basis state i to P(i) (closed form cpp/ising_cuda_kernels.cu:178-205).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rsv {

using u64 = unsigned long long;

// Tile geometry shared by host and device: one tile = 2^12 amplitudes held in
// registers by 256 threads (16 amplitudes each).
constexpr int kTileBits = 12;
constexpr int kTileSize = 1 << kTileBits;
constexpr int kThreads = 256;
constexpr int kRegs = 16;
constexpr int kMaxQubits = 31;
constexpr int kMaxRuns = 4;

// Forward ring map P(i): bit k (k >= 1) is the XOR of bits 0..k of i, bit 0
// is the parity of bits 1..n-1.  Bits at and above n pass through unchanged
// (they only exist in the zero-padded layout used for n < 12).
__host__ __device__ __forceinline__ u64 ring_p(u64 i, int n) {
  const u64 mask = (u64{1} << n) - 1;
  const u64 lo = i & mask;
  u64 pre = lo;
  pre ^= pre << 1;
  pre ^= pre << 2;
  pre ^= pre << 4;
  pre ^= pre << 8;
  pre ^= pre << 16;
  pre &= mask;
#ifdef __CUDA_ARCH__
  const u64 par = static_cast<u64>(__popcll(lo >> 1) & 1);
#else
  const u64 par = static_cast<u64>(__builtin_popcountll(lo >> 1) & 1);
#endif
  return (i & ~mask) | (pre & ~u64{1}) | par;
}

// Inverse ring map P^{-1}(j) = (j ^ (j << 1)) & mask, bits 0 and 1 flipped
// when bit n-1 of j is set.
__host__ __device__ __forceinline__ u64 ring_pinv(u64 j, int n) {
  const u64 mask = (u64{1} << n) - 1;
  const u64 lo = j & mask;
  u64 t = (lo ^ (lo << 1)) & mask;
  if ((lo >> (n - 1)) & 1) t ^= 3;
  return (j & ~mask) | t;
}

#ifdef __CUDACC__
// Diagonal of P^T H P at basis index i: the ZZ energy of the permuted state,
// 2 * (#domain walls of P(i) on the ring) - n.
__device__ __forceinline__ double diag_after_ring(u64 i, int n) {
  const u64 mask = (u64{1} << n) - 1;
  const u64 p = ring_p(i, n) & mask;
  const u64 rot = ((p << 1) & mask) | (p >> (n - 1));
  return static_cast<double>(2 * __popcll(p ^ rot)) - static_cast<double>(n);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// a * conj(b)
__device__ __forceinline__ double2 cmul_conj(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// D += A B on the FP64 tensor cores, one m8n8k4 tile per warp (row-major A,
// column-major B).  Lane l holds A[l / 4][l % 4], B[l % 4][l / 4] and
// D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void mma_f64(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

#endif  // __CUDACC__

}  // namespace rsv
