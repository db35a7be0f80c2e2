// Allocation-free energy and gradient (rsv_energy_and_grad_noalloc, include/rsv.h).
//
// For callers that must not allocate device memory on their own: every
// buffer of the computation (three state vectors, coefficient and phase
// tables, per-CTA gradient records) is carved out of one fixed workspace that
// lives in this library's device image as a file-scope __device__ array, so
// the call itself issues no cudaMalloc/cudaFree.  Limits: num_qubits <= 16,
// num_layers <= 64 (8 MiB of workspace, held by every GPU that loads the
// library until the process exits).
#include <cstddef>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/rsv.h"
#include "rsv_workspace.h"

namespace {

constexpr size_t kWorkspaceBytes = size_t{8} << 20;
constexpr int kMaxQubits = 16;
constexpr int kMaxLayers = 64;
constexpr int kMaxDevices = 64;

// The shared workspace.  In host code its name is only a host-side stand-in;
// the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_workspace[kWorkspaceBytes];

void *g_workspace_address[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of g_workspace on the current device (looked up once per
// device, with that device current).
void *workspace_address(int device, std::string &error) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_workspace_address[device] == nullptr) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_workspace);
    if (e != cudaSuccess) {
      error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return nullptr;
    }
    g_workspace_address[device] = ptr;
  }
  return g_workspace_address[device];
}

}  // namespace

extern "C" rsv_status rsv_energy_and_grad_noalloc(int num_qubits, int num_layers, double field,
                                                  const double *d_params, size_t num_params,
                                                  double *d_energy_out, double *d_gradient_out,
                                                  void *stream) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    rsv::set_last_error((std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
    return RSV_ERR_CUDA;
  }
  if (device < 0 || device >= kMaxDevices) {
    rsv::set_last_error("device index out of range for the allocation-free entry point");
    return RSV_ERR_UNSUPPORTED;
  }
  std::string error;
  void *ws = workspace_address(device, error);
  if (ws == nullptr) {
    rsv::set_last_error(error.c_str());
    return RSV_ERR_CUDA;
  }
  return rsv::run_in_workspace(num_qubits, num_layers, field, d_params, num_params, d_energy_out,
                               d_gradient_out, ws, kWorkspaceBytes, kMaxQubits, kMaxLayers, stream);
}
