// dense_scan path (rsv_dense.cu): n <= 8, dense layer matrices on FP64 tensor cores.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace rsv {

constexpr int kDenseMaxQubits = 8;

struct DenseArgs {
  int n, L;
  double field;
  const double4 *coef;  // [L * n] cos/sin of the half angles
  double2 *work;        // dense_workspace_bytes(n, L)
  double *energy_out;   // device f64[1]
  double *grad_out;     // device f64[2 n L] or null
};

int dense_padded_layers(int L);
size_t dense_workspace_bytes(int n, int L);
cudaError_t run_dense_scan(const DenseArgs &D, cudaStream_t s);
// C[b] = A[b] B[b] for complex128 dim x dim row-major matrices (FP64 MMA for dim >= 32)
cudaError_t zgemm_batched(const double2 *A, const double2 *B, double2 *C, int dim, int batch, long long sa,
                          long long sb, long long sc, cudaStream_t s);

}  // namespace rsv
