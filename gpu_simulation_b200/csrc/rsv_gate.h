// Gate-level inverse walk (rsv_gate.cu), used for gradient_strategy
// "inverse_walk_cuQuantum".
#pragma once

#include <cuda_runtime.h>

namespace rsv {

struct GateLevelArgs {
  int n, L;
  double field;
  const double4 *coef;      // [L * n] cos/sin of the half angles
  double2 *psi, *lam;       // 2^n amplitudes each
  int grid;                 // CTAs of every gate kernel (gate_grid)
  double *energy_partials;  // [grid]
  double *grad_partials;    // [2 n L][grid]
  double *energy_out;       // device f64[1]
  double *grad_out;         // device f64[2 n L] or null
};

int gate_grid(int n, int sms);
cudaError_t run_gate_level(const GateLevelArgs &A, cudaStream_t s);

}  // namespace rsv
