// Host-callable launchers of the kernels in rsv_kernels.cu.
#pragma once

#include <atomic>
#include <cstddef>
#include <cuda_runtime.h>

#include "rsv_types.h"

namespace rsv {

// Raises kernel k's dynamic shared-memory limit to `bytes` on the current
// device, once per device: the attribute belongs to the device, so a process
// that uses several GPUs sets it on each.  `done` holds one bit per device
// ordinal (ordinals >= 64 set the attribute on every call).  Safe to call from
// several host threads.
template <typename K>
inline cudaError_t set_smem_limit_once(K k, size_t bytes, std::atomic<unsigned long long> &done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
  if (bit != 0 && (done.load(std::memory_order_acquire) & bit) != 0) return cudaSuccess;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e == cudaSuccess && bit != 0) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

cudaError_t launch_coef(const double *params, double4 *coef, int count, cudaStream_t s);
// dst[0 .. count) = src[0 .. count) through kernel parameters (small tables)
cudaError_t launch_put_ints(const int *src, size_t count, int *dst, cudaStream_t s);
// prod holds 1 + partial.count tables of [4][256]
cudaError_t launch_tables(const double4 *coef, int n, int L, double2 *ptab, double2 *prod,
                          const PartialMasks &partial, cudaStream_t s);
cudaError_t launch_rot(const double4 *coef, int n, int L, const int *order, bool checkpoint,
                       double2 *rot, double *lscale, double *gscale, cudaStream_t s);
cudaError_t configure_pass_kernels();
size_t pass_smem_bytes(bool bwd);
cudaError_t launch_pass(const PassParams &P, bool bwd, int grid, cudaStream_t s);
// backward pass on an 11-bit half tile (rsv_pass_half.cu)
cudaError_t launch_bwd_half(const PassParams &P, int grid, cudaStream_t s);
// mu = (P^T H P) chi and per-CTA energy partials ([grid]); for large n a
// shared-memory tile kernel takes the masks on the top index bits first
cudaError_t launch_energy(const double2 *chi, double2 *mu, int n, double field,
                          unsigned long long size, double *partials, int grid, int sms, cudaStream_t s);
// mu = (diagonal - field * sum over the given index masks) chi, with per-CTA
// energy partials ([grid], grid = energy_grid_size): the energy kernel of an
// energy_and_grad call whose first backward pass applies the other field
// terms (count <= n masks, n >= kEnergySplitQubits)
cudaError_t launch_energy_masks(const double2 *chi, double2 *mu, int n, double field, unsigned long long size,
                                const unsigned long long *masks, int count, double *partials, int grid,
                                cudaStream_t s);
// inputs of the phase table of a middle pass's field terms (rsv_kernels.cu)
struct DeferPhaseArgs {
  const double4 *coef;
  int n, layer;
  unsigned int pending;  // wires whose tangent factors psi and lambda still carry
  int wires[8];          // the pass's gated wires on tile bits 3..10
  double field;
};
cudaError_t launch_defer_phase(const DeferPhaseArgs &A, double2 *out, cudaStream_t s);
// qubits from which the energy is split (tile kernel + grid-stride kernel)
int energy_split_qubits();
// kernels launch_energy launches for n qubits (1, or 2 for the split energy)
int energy_kernel_count(int n);
// CTAs of the energy's grid-stride kernel (= its number of partials)
int energy_grid_size(int n, int sms);
cudaError_t launch_finalize(const FinalizeParams &F, cudaStream_t s);
// layer-0 gradients in one read of lambda (n >= 13), and their final reduction
// into grad_out[0 .. 2n)
cudaError_t launch_layer0_grad(const Layer0Params &Q, int grid, cudaStream_t s);
cudaError_t launch_layer0_finalize(const Layer0Params &Q, int grid, double *grad_out, cudaStream_t s);
// the first K layers as a matrix-product state (n >= 13, bond 2 or 4): the
// site and table set-up, the forward write of their output, the gradient
// read of lambda (tile sums, coset sums, CTA sums) and the final per-wire
// environments into grad_out[0 .. 2nK)
cudaError_t launch_mps_tables(const MpsParams &Q, cudaStream_t s);
cudaError_t launch_mps_forward(const MpsParams &Q, double2 *out, int scatter, int grid, cudaStream_t s);
cudaError_t launch_mps_grad(const MpsParams &Q, const double2 *lam, int gather, int grid, cudaStream_t s);
cudaError_t launch_mps_finalize(const MpsParams &Q, double *grad_out, cudaStream_t s);

}  // namespace rsv
