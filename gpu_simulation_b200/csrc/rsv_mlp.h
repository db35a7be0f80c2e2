// Launchers of the warm-start network kernels (rsv_mlp.cu), used by the host
// side (rsv_mlp_host.cpp).
#pragma once

#include <cuda_runtime.h>

namespace rsv {

// C[m][n] = sum_k A[m*sam + k*sak] * B[k*sbk + n*sbn] (+ bias[n]); Z (if not
// null) receives the pre-activation, C the GELU of it when gelu_act.
cudaError_t mlp_gemm(int M, int N, int K, const float *A, long long sam, long long sak,
                     const float *B, long long sbk, long long sbn, const float *bias, bool gelu_act,
                     float *C, float *Z, cudaStream_t s);
cudaError_t mlp_gelu_back(long long count, const float *Z, const float *dY, float *dZ,
                          cudaStream_t s);
cudaError_t mlp_colsum(int M, int N, const float *dZ, float *db, cudaStream_t s);
int mlp_loss_blocks(long long count);
cudaError_t mlp_mse(long long count, const float *out, const float *target, float *dout,
                    float *partials, float *loss, cudaStream_t s);
cudaError_t gd_step(long long count, double *p, const double *g, double stepsize, const double *energy,
                    double *energy_hist, double *gnorm_hist, int *counter, cudaStream_t s);
cudaError_t adam_vqe_step(long long count, double *p, const double *g, double *m, double *v, double lr,
                          double beta1, double beta2, double eps, const double *energy, double *energy_hist,
                          int *counter, cudaStream_t s);
template <typename T>
cudaError_t adam_step(long long count, T *p, const T *g, T *m, T *v, T lr, T beta1, T beta2, T eps,
                      int step, cudaStream_t s);

}  // namespace rsv
