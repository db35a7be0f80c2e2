// Internal interface between the allocation-free entry point (rsv_noalloc.cu)
// and the host scheduler (rsv_backend.cpp).
#pragma once

#include <cstddef>

#include "../../include/rsv.h"

namespace rsv {

void set_last_error(const char *msg);

rsv_status run_in_workspace(int n, int L, double field, const double *d_params, size_t num_params,
                            double *d_energy_out, double *d_gradient_out, void *workspace,
                            size_t workspace_bytes, int max_qubits, int max_layers, void *stream);

}  // namespace rsv
