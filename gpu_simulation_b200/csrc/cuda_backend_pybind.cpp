// pybind11 drop-in for the reference module standalone_backend._cuda_backend
// (zzEncounter/GPU_Simulation cpp/ising_cuda_bindings.cpp:71-144): same module
// name, class, constructor keywords, methods and return dictionaries, built
// over the C ABI of librsv.so (include/rsv.h).  Argument errors raise
// ValueError and CUDA errors RuntimeError, as the reference's exception
// translation does.
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include "rsv.h"

namespace py = pybind11;

namespace rsvpy {

using FlatArray = py::array_t<double, py::array::c_style | py::array::forcecast>;

[[noreturn]] void raise_status(rsv_status s) {
  const std::string msg = rsv_last_error();
  if (s == RSV_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

inline void ok(rsv_status s) {
  if (s != RSV_OK) raise_status(s);
}

class Backend {
 public:
  Backend(std::size_t num_qubits, std::size_t num_layers, double field,
          const std::string &gradient_strategy, std::size_t width, bool double_buffer) {
    if (num_qubits > 64 || num_layers > (1u << 20) || width > 64)
      throw std::invalid_argument("argument out of range");
    ok(rsv_create(static_cast<int>(num_qubits), static_cast<int>(num_layers), field,
                  gradient_strategy.c_str(), static_cast<int>(width), double_buffer ? 1 : 0, &h_));
    size_t np = 0;
    ok(rsv_backend_info(h_, nullptr, nullptr, &np, nullptr));
    num_params_ = np;
  }
  ~Backend() { rsv_destroy(h_); }
  Backend(const Backend &) = delete;
  Backend &operator=(const Backend &) = delete;

  py::dict energy_and_grad(const FlatArray &params, bool compute_gradient, bool profile) {
    const auto info = params.request();
    const double *ptr = static_cast<const double *>(info.ptr);
    const size_t size = static_cast<size_t>(info.size);
    double energy = 0.0;
    std::vector<double> grad(compute_gradient ? num_params_ : 0);
    std::vector<double> stages(rsv_num_stages(), 0.0);
    rsv_status s;
    {
      py::gil_scoped_release release;
      if (profile) {
        s = rsv_profile_energy_and_grad(h_, ptr, size, compute_gradient ? 1 : 0, &energy,
                                        compute_gradient ? grad.data() : nullptr, stages.data());
      } else {
        s = rsv_energy_and_grad(h_, ptr, size, compute_gradient ? 1 : 0, &energy,
                                compute_gradient ? grad.data() : nullptr, nullptr);
      }
    }
    ok(s);
    py::dict out;
    out["energy"] = py::float_(energy);
    py::array_t<double> g(grad.size());
    if (!grad.empty()) std::memcpy(g.mutable_data(), grad.data(), grad.size() * sizeof(double));
    out["gradient"] = std::move(g);
    if (profile) {
      py::dict t;
      for (int i = 0; i < rsv_num_stages(); ++i) t[py::str(rsv_stage_name(i))] = py::float_(stages[i]);
      out["timings_ms"] = std::move(t);
    }
    return out;
  }

  py::dict benchmark_forward_graph(const FlatArray &params, std::size_t repeats) {
    const auto info = params.request();
    double normal = 0.0, graph = 0.0;
    rsv_status s;
    {
      py::gil_scoped_release release;
      s = rsv_benchmark_forward_graph(h_, static_cast<const double *>(info.ptr),
                                      static_cast<size_t>(info.size), repeats, &normal, &graph);
    }
    ok(s);
    py::dict out;
    out["normal_forward_ms"] = py::float_(normal);
    out["graph_forward_ms"] = py::float_(graph);
    out["speedup"] = py::float_(graph > 0.0 ? normal / graph : 0.0);
    return out;
  }

 private:
  rsv_backend *h_ = nullptr;
  size_t num_params_ = 0;
};

}  // namespace rsvpy

PYBIND11_MODULE(_cuda_backend, m) {
  m.doc() = "B200 (sm_100a) backend for the ring Ising adjoint workflow (drop-in).";

  py::class_<rsvpy::Backend>(m, "RingIsingCudaBackend")
      .def(py::init<std::size_t, std::size_t, double, const std::string &, std::size_t, bool>(),
           py::arg("num_qubits"), py::arg("num_layers"), py::arg("field"),
           py::arg("gradient_strategy") = "structured_adjoint",
           py::arg("structured_rotation_chunk_width") = 8, py::arg("double_buffer") = false)
      .def("energy_and_grad", &rsvpy::Backend::energy_and_grad, py::arg("params"),
           py::arg("compute_gradient") = true, py::arg("profile") = false)
      .def("benchmark_structured_forward_graph", &rsvpy::Backend::benchmark_forward_graph,
           py::arg("params"), py::arg("repeats") = 100);

  m.def(
      "energy_and_grad",
      [](std::size_t num_qubits, std::size_t num_layers, double field,
         const std::string &gradient_strategy, rsvpy::FlatArray params, bool compute_gradient,
         bool profile, std::size_t width) {
        const auto info = params.request();
        if (info.ndim != 1) throw std::invalid_argument("params must be a flat 1D float64 array.");
        if (static_cast<std::size_t>(info.size) != num_qubits * num_layers * 2)
          throw std::invalid_argument("params does not match num_qubits/layers.");
        rsvpy::Backend b(num_qubits, num_layers, field, gradient_strategy, width, false);
        return b.energy_and_grad(params, compute_gradient, profile);
      },
      py::arg("num_qubits"), py::arg("num_layers"), py::arg("field"),
      py::arg("gradient_strategy") = "structured_adjoint", py::arg("params"),
      py::arg("compute_gradient") = true, py::arg("profile") = false,
      py::arg("structured_rotation_chunk_width") = 8);

  m.attr("__engine__") = py::str(rsv_version());
}
