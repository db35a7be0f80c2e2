// Host side of the warm-start network (C ABI in include/rsv.h): layer loop of
// the forward and backward passes over the kernels of rsv_mlp.cu.
#include <cmath>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "../../include/rsv.h"
#include "rsv_mlp.h"

namespace rsv {
void set_last_error(const char *msg);

namespace {

constexpr int kMaxMlpLayers = 16;

struct ArgError : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};

template <typename F>
rsv_status mlp_guarded(F &&f) {
  try {
    f();
    set_last_error("");
    return RSV_OK;
  } catch (const ArgError &e) {
    set_last_error(e.what());
    return RSV_ERR_INVALID_ARGUMENT;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return RSV_ERR_CUDA;
  }
}

void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void check_widths(int num_layers, const int *widths) {
  if (num_layers < 1 || num_layers > kMaxMlpLayers)
    throw ArgError("num_layers must be in [1, " + std::to_string(kMaxMlpLayers) + "]");
  if (widths == nullptr) throw ArgError("widths is null");
  for (int l = 0; l <= num_layers; ++l)
    if (widths[l] < 1 || widths[l] > 65536) throw ArgError("layer widths must be in [1, 65536]");
}

size_t num_weights(int num_layers, const int *widths) {
  size_t s = 0;
  for (int l = 1; l <= num_layers; ++l)
    s += static_cast<size_t>(widths[l]) * widths[l - 1] + widths[l];
  return s;
}

size_t work_floats(int num_layers, const int *widths, int batch) {
  size_t s = 0;
  for (int l = 1; l < num_layers; ++l) s += 2 * static_cast<size_t>(batch) * widths[l];
  return s;
}

size_t max_width(int num_layers, const int *widths) {
  int m = 0;
  for (int l = 0; l <= num_layers; ++l) m = widths[l] > m ? widths[l] : m;
  return static_cast<size_t>(m);
}

}  // namespace
}  // namespace rsv

using namespace rsv;

extern "C" {

size_t rsv_mlp_num_weights(int num_layers, const int *widths) {
  if (num_layers < 1 || num_layers > kMaxMlpLayers || widths == nullptr) return 0;
  return num_weights(num_layers, widths);
}

size_t rsv_mlp_work_floats(int num_layers, const int *widths, int batch) {
  if (num_layers < 1 || num_layers > kMaxMlpLayers || widths == nullptr || batch < 0) return 0;
  return work_floats(num_layers, widths, batch);
}

size_t rsv_mlp_scratch_floats(int num_layers, const int *widths, int batch) {
  if (num_layers < 1 || num_layers > kMaxMlpLayers || widths == nullptr || batch < 0) return 0;
  return 2 * static_cast<size_t>(batch) * max_width(num_layers, widths);
}

rsv_status rsv_mlp_forward(int num_layers, const int *widths, const float *d_weights, int batch,
                           const float *d_x, float *d_out, float *d_work, void *stream) {
  return mlp_guarded([&] {
    check_widths(num_layers, widths);
    if (batch < 0) throw ArgError("batch must be non-negative");
    if (batch == 0) return;
    if (!d_weights || !d_x || !d_out || (num_layers > 1 && !d_work))
      throw ArgError("null device pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const float *x = d_x;
    const float *w = d_weights;
    float *work = d_work;
    for (int l = 1; l <= num_layers; ++l) {
      const int K = widths[l - 1], N = widths[l];
      const float *W = w, *b = w + static_cast<size_t>(N) * K;
      w = b + N;
      const bool hidden = l < num_layers;
      float *Z = hidden ? work : nullptr;
      float *A = hidden ? work + static_cast<size_t>(batch) * N : d_out;
      cuda_check(mlp_gemm(batch, N, K, x, K, 1, W, 1, K, b, hidden, A, Z, s), "mlp forward gemm");
      if (hidden) work += 2 * static_cast<size_t>(batch) * N;
      x = A;
    }
  });
}

rsv_status rsv_mlp_backward(int num_layers, const int *widths, const float *d_weights, int batch,
                            const float *d_x, const float *d_work, const float *d_dout,
                            float *d_grad, float *d_scratch, void *stream) {
  return mlp_guarded([&] {
    check_widths(num_layers, widths);
    if (batch < 1) throw ArgError("batch must be positive");
    if (!d_weights || !d_x || !d_dout || !d_grad || !d_scratch || (num_layers > 1 && !d_work))
      throw ArgError("null device pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // offsets of every layer's weights and saved activations
    size_t woff[kMaxMlpLayers + 1], aoff[kMaxMlpLayers + 1];
    woff[1] = 0;
    aoff[1] = 0;
    for (int l = 1; l <= num_layers; ++l) {
      if (l < num_layers) {
        woff[l + 1] = woff[l] + static_cast<size_t>(widths[l]) * widths[l - 1] + widths[l];
        aoff[l + 1] = aoff[l] + 2 * static_cast<size_t>(batch) * widths[l];
      }
    }
    const size_t mw = max_width(num_layers, widths);
    float *bufs[2] = {d_scratch, d_scratch + static_cast<size_t>(batch) * mw};
    const float *dZ = d_dout;
    for (int l = num_layers; l >= 1; --l) {
      const int K = widths[l - 1], N = widths[l];
      const float *W = d_weights + woff[l];
      float *gW = d_grad + woff[l], *gb = gW + static_cast<size_t>(N) * K;
      // input of layer l: the network input, or the post-activation of layer l-1
      const float *X = (l == 1) ? d_x : d_work + aoff[l - 1] + static_cast<size_t>(batch) * K;
      // dW = dZ^T X  (N x K, summed over the batch)
      cuda_check(mlp_gemm(N, K, batch, dZ, 1, N, X, K, 1, nullptr, false, gW, nullptr, s),
                 "mlp weight-gradient gemm");
      cuda_check(mlp_colsum(batch, N, dZ, gb, s), "mlp bias gradient");
      if (l > 1) {
        float *dA = bufs[l & 1];
        // dA = dZ W  (batch x K), then dZ_{l-1} = dA * gelu'(Z_{l-1}) in place
        cuda_check(mlp_gemm(batch, K, N, dZ, N, 1, W, K, 1, nullptr, false, dA, nullptr, s),
                   "mlp input-gradient gemm");
        const float *Zprev = d_work + aoff[l - 1];
        cuda_check(mlp_gelu_back(static_cast<long long>(batch) * K, Zprev, dA, dA, s),
                   "mlp gelu backward");
        dZ = dA;
      }
    }
  });
}

rsv_status rsv_mlp_mse(size_t count, const float *d_out, const float *d_target, float *d_dout,
                       float *d_loss, float *d_partials, void *stream) {
  return mlp_guarded([&] {
    if (count == 0) throw ArgError("count must be positive");
    if (!d_out || !d_target || !d_dout || !d_loss || !d_partials) throw ArgError("null device pointer");
    cuda_check(mlp_mse(static_cast<long long>(count), d_out, d_target, d_dout, d_partials, d_loss,
                       static_cast<cudaStream_t>(stream)),
               "mse");
  });
}

rsv_status rsv_adam_f32(float *d_p, const float *d_g, float *d_m, float *d_v, size_t count, float lr,
                        float beta1, float beta2, float eps, int step, void *stream) {
  return mlp_guarded([&] {
    if (step < 1) throw ArgError("step counts from 1");
    if (count == 0) return;
    if (!d_p || !d_g || !d_m || !d_v) throw ArgError("null device pointer");
    cuda_check(adam_step<float>(static_cast<long long>(count), d_p, d_g, d_m, d_v, lr, beta1, beta2,
                                eps, step, static_cast<cudaStream_t>(stream)),
               "adam");
  });
}

rsv_status rsv_adam_f64(double *d_p, const double *d_g, double *d_m, double *d_v, size_t count,
                        double lr, double beta1, double beta2, double eps, int step, void *stream) {
  return mlp_guarded([&] {
    if (step < 1) throw ArgError("step counts from 1");
    if (count == 0) return;
    if (!d_p || !d_g || !d_m || !d_v) throw ArgError("null device pointer");
    cuda_check(adam_step<double>(static_cast<long long>(count), d_p, d_g, d_m, d_v, lr, beta1, beta2,
                                 eps, step, static_cast<cudaStream_t>(stream)),
               "adam");
  });
}

rsv_status rsv_gd_step_f64(double *d_params, const double *d_grad, size_t count, double stepsize,
                           const double *d_energy, double *d_energy_hist, double *d_gnorm_hist,
                           int *d_step_counter, void *stream) {
  return mlp_guarded([&] {
    if (!d_params || !d_grad || !d_energy || !d_step_counter) throw ArgError("null device pointer");
    if (!std::isfinite(stepsize)) throw ArgError("stepsize is not finite");
    cuda_check(gd_step(static_cast<long long>(count), d_params, d_grad, stepsize, d_energy, d_energy_hist,
                       d_gnorm_hist, d_step_counter, static_cast<cudaStream_t>(stream)),
               "gradient step");
  });
}

rsv_status rsv_adam_vqe_step_f64(double *d_params, const double *d_grad, double *d_m, double *d_v, size_t count,
                                 double lr, double beta1, double beta2, double eps, const double *d_energy,
                                 double *d_energy_hist, int *d_step_counter, void *stream) {
  return mlp_guarded([&] {
    if (!d_params || !d_grad || !d_m || !d_v || !d_energy || !d_step_counter) throw ArgError("null device pointer");
    if (!std::isfinite(lr) || !(beta1 >= 0.0 && beta1 < 1.0) || !(beta2 >= 0.0 && beta2 < 1.0) ||
        !std::isfinite(eps))
      throw ArgError("Adam needs a finite lr and eps and betas in [0, 1)");
    cuda_check(adam_vqe_step(static_cast<long long>(count), d_params, d_grad, d_m, d_v, lr, beta1, beta2, eps,
                             d_energy, d_energy_hist, d_step_counter, static_cast<cudaStream_t>(stream)),
               "adam step");
  });
}

}  // extern "C"
