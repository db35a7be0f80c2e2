/*
 * rsv.h -- C ABI of the B200 ring-Ising statevector engine (librsv.so).
 *
 * The engine computes the energy and the adjoint gradient of the ring-Ising
 * VQE ansatz (layers of RY.RZ on every wire followed by the CNOT ring;
 * H = -sum Z_i Z_{i+1} - h sum X_i) on a complex128 statevector, entirely on
 * one NVIDIA B200 (sm_100a).  It is the drop-in replacement for the
 * structured_adjoint path of zzEncounter/GPU_Simulation; each entry point
 * names the reference interface it replaces.
 *
 * Conventions: params is a flat f64 array of 2*num_qubits*num_layers values,
 * index (layer*num_qubits + wire)*2 + {0: theta of RY, 1: phi of RZ}
 * (reference cpp/ising_cuda_backend.cu:131-133).  Gradients use the same
 * layout.  Amplitude index bit w is wire w.
 *
 * Errors: every function returns an rsv_status; no C++ exception crosses
 * this boundary.  rsv_last_error() returns a message for the calling thread.
 * RSV_ERR_INVALID_ARGUMENT maps to the reference's std::invalid_argument
 * (Python ValueError); every other non-zero status maps to its
 * std::runtime_error (Python RuntimeError).
 *
 * Threading: one rsv_backend owns its device buffers and is not re-entrant
 * (reference cpp/ising_cuda_backend.hpp:22-49); use one handle per thread.
 */
#ifndef RSV_H
#define RSV_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rsv_status {
  RSV_OK = 0,
  RSV_ERR_INVALID_ARGUMENT = 1,
  RSV_ERR_CUDA = 2,
  RSV_ERR_OUT_OF_MEMORY = 3,
  RSV_ERR_UNSUPPORTED = 4,
  RSV_ERR_INTERNAL = 5,
  /* rsv_backward_device only: the backend ran another call after the
   * forward whose generation was passed, so that forward's state is gone
   * (a Python RuntimeError; the autograd Function recomputes on it). */
  RSV_ERR_STALE_STATE = 6
} rsv_status;

typedef struct rsv_backend rsv_backend;

/* Version string of the library. */
const char *rsv_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *rsv_last_error(void);

/* Number of stage timings reported by rsv_profile_energy_and_grad and the
 * name of stage i (reference StageProfiler names, cpp/ising_cuda_backend.cu:24-106). */
int rsv_num_stages(void);
const char *rsv_stage_name(int i);

/*
 * Create a backend bound to the current CUDA device.  Later calls on the
 * backend run on that device whichever device is current when they are made
 * (the caller's current device is restored before they return); stream
 * arguments must belong to it.
 * Replaces RingIsingCudaBackend::RingIsingCudaBackend
 * (reference cpp/ising_cuda_backend.hpp:26-29, cpp/ising_cuda_backend.cu:388-404,
 *  bound at cpp/ising_cuda_bindings.cpp:74-80).
 * gradient_strategy: "structured_adjoint" (tile-pass engine),
 * "inverse_walk_cuQuantum" (alias "inverse_walk_cuquantum": RY, RZ and CNOT as
 * separate kernels and the gate-level adjoint walk, without cuStateVec) or
 * "dense_scan" (n <= 8: dense layer matrices, product tree on FP64 tensor
 * cores); results agree to rounding.  The split device entry points
 * (rsv_forward_device / rsv_backward_device) and rsv_benchmark_forward_graph
 * always run the tile-pass engine.  structured_rotation_chunk_width must be in
 * [1, 8] and double_buffer is accepted; both are validated as the reference
 * does and otherwise ignored (the engine plans its own tiles).
 * Allocates three state buffers of 16 * 2^max(n,12) bytes.
 */
rsv_status rsv_create(int num_qubits, int num_layers, double field,
                      const char *gradient_strategy, int structured_rotation_chunk_width,
                      int double_buffer, rsv_backend **out);

/* Release a backend and its device memory.  Accepts NULL. */
rsv_status rsv_destroy(rsv_backend *backend);

/*
 * Energy and (optionally) gradient from host parameters; synchronous.
 * Replaces RingIsingCudaBackend::energy_and_grad(params, num_params,
 * compute_gradient, profile=false) (reference cpp/ising_cuda_backend.cu:429-442,
 * bound at cpp/ising_cuda_bindings.cpp:81-98).
 * params: host f64[num_params]; gradient_out: host f64[num_params], written
 * only when compute_gradient != 0 (may be NULL otherwise).
 * stream: a cudaStream_t, or NULL for the backend's own stream.
 */
rsv_status rsv_energy_and_grad(rsv_backend *backend, const double *params, size_t num_params,
                               int compute_gradient, double *energy_out, double *gradient_out,
                               void *stream);

/*
 * Same computation with DEVICE pointers, asynchronous on `stream` (no host
 * synchronisation, no host copies).  Used by the torch.autograd path.
 * `stream` is used as given: 0 is the legacy default stream (for all device
 * entry points below as well).
 * d_params: device f64[num_params]; d_energy_out: device f64[1];
 * d_gradient_out: device f64[num_params] or NULL for energy only.
 * No reference counterpart (the reference always round-trips through the host).
 */
rsv_status rsv_energy_and_grad_device(rsv_backend *backend, const double *d_params,
                                      size_t num_params, double *d_energy_out,
                                      double *d_gradient_out, void *stream);

/*
 * Split form of rsv_energy_and_grad_device for autograd: rsv_forward_device
 * runs the forward sweep and the energy (d_energy_out, device f64[1]) and
 * keeps the final state and lambda = H psi on the device; a later
 * rsv_backward_device runs only the adjoint sweep and writes the gradient of
 * that same forward (d_gradient_out, device f64[num_params]).  *generation_out
 * (may be NULL) identifies the forward; rsv_backward_device fails with
 * RSV_ERR_STALE_STATE if another call has run on the backend since (and with
 * RSV_ERR_INVALID_ARGUMENT for a null pointer or backend).
 * No reference counterpart.
 */
rsv_status rsv_forward_device(rsv_backend *backend, const double *d_params, size_t num_params,
                              double *d_energy_out, unsigned long long *generation_out,
                              void *stream);
rsv_status rsv_backward_device(rsv_backend *backend, unsigned long long generation,
                               double *d_gradient_out, void *stream);

/*
 * energy_and_grad with a per-stage timing breakdown (milliseconds, CUDA events).
 * Replaces the profile=true path of RingIsingCudaBackend::energy_and_grad
 * (reference cpp/ising_cuda_backend.cu:24-106, cpp/ising_cuda_bindings.cpp:39-55).
 * stage_ms_out: host double[rsv_num_stages()].
 */
rsv_status rsv_profile_energy_and_grad(rsv_backend *backend, const double *params,
                                       size_t num_params, int compute_gradient,
                                       double *energy_out, double *gradient_out,
                                       double *stage_ms_out);

/*
 * Time the forward sweep launched directly and as a captured CUDA graph.
 * Replaces RingIsingCudaBackend::benchmark_structured_forward_graph
 * (reference cpp/ising_cuda_backend.cu:444-541, cpp/ising_cuda_bindings.cpp:99-114).
 */
rsv_status rsv_benchmark_forward_graph(rsv_backend *backend, const double *params,
                                       size_t num_params, size_t repeats, double *normal_ms_out,
                                       double *graph_ms_out);

/*
 * Allocation-free energy and gradient: the same computation as
 * rsv_energy_and_grad_device for one circuit, for callers that cannot call
 * cudaMalloc -- code whose device memory belongs to another allocator (a
 * framework's caching pool or a fixed arena it must not fragment) or that
 * runs where a device allocation and its implicit synchronisation are not
 * allowed.  No backend object is created: every buffer lives in one fixed
 * 8 MiB workspace inside this library's device image (held by every GPU that
 * loads the library until the process exits), so the call issues no
 * cudaMalloc, cudaFree or other allocating routine.  The caller passes device
 * pointers: d_params f64[num_params], d_energy_out f64[1], d_gradient_out
 * f64[num_params] (or NULL for energy only), and a stream used as given.
 * Limits: num_qubits <= 16, num_layers <= 64; larger circuits return
 * RSV_ERR_INVALID_ARGUMENT.  The first call on a device looks up the
 * workspace address (cudaGetSymbolAddress) and should come before any stream
 * capture.  All calls share the one workspace, which keeps the last call's
 * contents: calls that overlap on the GPU (other streams, other host threads)
 * race; serialise them.
 * No counterpart in the reference.
 */
rsv_status rsv_energy_and_grad_noalloc(int num_qubits, int num_layers, double field,
                                       const double *d_params, size_t num_params,
                                       double *d_energy_out, double *d_gradient_out,
                                       void *stream);

/*
 * Per-launch timing over a measured region (for roofline reporting).
 * rsv_set_launch_timing(backend, 1) makes every following call record a CUDA
 * event pair around each of its kernel launches, on the launch stream;
 * rsv_launch_stats synchronises, and returns per kernel kind (0 tables,
 * 1 forward pass, 2 energy, 3 backward pass, 4 finalize) the launch count,
 * the summed duration in ms and the summed algorithmic DRAM bytes (the
 * minimum traffic: every amplitude a launch must read or write, 16 B each),
 * then clears the record.  Arrays have RSV_NUM_KINDS entries.
 * No reference counterpart.
 */
#define RSV_NUM_KINDS 5

/*
 * Number of kernels the backend's calls have launched since it was created
 * (every kernel of every call, with or without launch timing).
 * No reference counterpart.
 */
rsv_status rsv_kernel_launches(rsv_backend *backend, unsigned long long *count_out);
rsv_status rsv_set_launch_timing(rsv_backend *backend, int enable);
rsv_status rsv_launch_stats(rsv_backend *backend, int *counts, double *total_ms,
                            double *total_bytes);

/*
 * Backward schedule.  RSV_BACKWARD_UNCOMPUTE keeps three state buffers and
 * un-computes psi alongside lambda (the reference's schedule,
 * cpp/ising_cuda_structured_adjoint_modes.inc:188-307).  RSV_BACKWARD_CHECKPOINT
 * keeps the state after every forward pass (max((L-1) * passes + 1, 2)
 * buffers of 16 * 2^n bytes; passes = 3 for 20 <= n <= 31) so that the
 * backward reads psi and writes only lambda.
 * RSV_BACKWARD_AUTO (the default of rsv_create) picks the checkpoint schedule
 * for n >= 13 while its buffers fit 128 GiB (and its allocation succeeds).
 * rsv_set_backward_mode re-plans and reallocates (synchronises the backend's
 * stream); rsv_backward_mode reports the mode, whether the checkpoint schedule
 * is in use and the number of state buffers.  No reference counterpart.
 */
#define RSV_BACKWARD_AUTO 0
#define RSV_BACKWARD_UNCOMPUTE 1
#define RSV_BACKWARD_CHECKPOINT 2
rsv_status rsv_set_backward_mode(rsv_backend *backend, int mode);
rsv_status rsv_backward_mode(rsv_backend *backend, int *mode_out, int *checkpoint_out,
                             int *num_buffers_out);

/*
 * Analytic leading layers (n >= 13).  The circuit starts from |0...0>, so after
 * k layers its state is a periodic matrix-product state of bond dimension
 * 2^(k-1) (the CNOT ring only turns indices into prefix parities).  With
 * max_layers = 3 (the default) or 2, the first K = min(L, max_layers) layers
 * are written in one pass from that form and all their gradients come from one
 * read of lambda at their output (gpu_simulation_b200/csrc/rsv_mps.cu); with 1
 * only layer 0's backward is replaced (one read of lambda, the layer-0 kernel);
 * with 0 every layer runs through the tile passes, with layer 0 computed
 * analytically inside layer 1's first forward pass like the reference
 * (cpp/ising_cuda_rotation_kernels.cu:20-41).  Results agree to rounding in
 * every setting.  rsv_set_analytic_layers re-plans (synchronises the backend's
 * stream); rsv_analytic_layers reports the setting and the number of layers
 * the current plan handles analytically.  No reference counterpart.
 */
rsv_status rsv_set_analytic_layers(rsv_backend *backend, int max_layers);
rsv_status rsv_analytic_layers(rsv_backend *backend, int *max_layers_out, int *used_out);

/*
 * Kernel selection (flags, default RSV_KERNELS_TMA | RSV_KERNELS_FUSED_ENERGY).
 * RSV_KERNELS_TMA: the backward passes on 11-bit tiles whose psi comes from a
 * forward checkpoint and whose lambda is updated in place, and the 12-wire low
 * pass, run on the TMA-fed kernels (gpu_simulation_b200/csrc/rsv_pass_tma.cu):
 * psi and lambda arrive by tensor copies into a swizzled shared-memory stage,
 * lambda leaves by a tensor store, and the warps of a block synchronise only
 * through split-phase mbarriers.  Their tensor maps are encoded when the
 * backend is planned; a pass the driver cannot map keeps the cp.async kernel.
 * RSV_KERNELS_FUSED_ENERGY (with RSV_KERNELS_TMA): in energy_and_grad calls,
 * the field terms of H whose index masks lie inside the tile of the last
 * layer's first backward pass are applied by that pass, which reads the final
 * state anyway; the energy kernel applies the diagonal and the other field
 * terms in one launch.  Energy-only calls (and rsv_forward_device) keep the
 * full energy kernels.  Flags 0 keeps every pass on the cp.async kernels.
 * Results agree to rounding.  rsv_set_kernels re-plans (synchronises the
 * backend's stream); rsv_kernels reports the flags and how many backward
 * passes of the plan are on the TMA kernels.  If a TMA pass ever gives up
 * waiting for its pipeline (after 1.5 s), the call's energy and gradient are
 * NaN and the synchronous entry points return RSV_ERR_CUDA.  No reference
 * counterpart (the reference's backward kernels,
 * cpp/ising_cuda_statevector_grad_kernels.cu:683-1326, stage with
 * cuda::memcpy_async; its energy is a separate kernel,
 * cpp/ising_cuda_kernels.cu:313-358).
 */
#define RSV_KERNELS_TMA 1
#define RSV_KERNELS_FUSED_ENERGY 2
rsv_status rsv_set_kernels(rsv_backend *backend, int flags);
rsv_status rsv_kernels(rsv_backend *backend, int *flags_out, int *tma_passes_out);

/*
 * Autotuner.  Times every plan candidate of the backend's circuit -- backward
 * schedule (checkpoint where its buffers fit, uncompute), three or two
 * analytic leading layers, the TMA kernels on or off, and each contiguous run
 * length of the high tiles that keeps the fewest passes -- with `repeats`
 * energy_and_grad calls on the device parameters d_params (after one untimed
 * call), and re-plans the backend with the fastest.  The choice is cached per
 * (device, num_qubits, num_layers) for the process: a later call for the same
 * shape applies it without timing unless flags has RSV_AUTOTUNE_FORCE.
 * Synchronous; reallocates the state buffers while it tries candidates.
 * rsv_describe_backend returns the backend's current plan (one line per
 * kernel launch, with the kernel of each backward pass) and the last
 * autotune's candidates and choice as text (length in *length_out; at most
 * buf_size bytes written including the NUL).  Replaces the reference's
 * hand-written width rules (cpp/ising_cuda_structured_adjoint_modes.inc:188-202,
 * cpp/ising_cuda_rotation_kernels.cu:562-575).
 */
#define RSV_AUTOTUNE_FORCE 1
rsv_status rsv_autotune(rsv_backend *backend, const double *d_params, size_t num_params, int repeats,
                        int flags, void *stream);
rsv_status rsv_describe_backend(rsv_backend *backend, char *buf, size_t buf_size, size_t *length_out);

/*
 * Batched complex128 GEMM on FP64 tensor cores (mma.sync f64; the dense_scan
 * product tree uses it): C[b] = A[b] B[b] for b < batch, every matrix dim x dim
 * row-major and the batches contiguous; dim < 32 or a multiple of 32.  Device
 * pointers, asynchronous on `stream`.  Replaces the reference's
 * cublasZgemmStridedBatched calls (cpp/ising_cuda_dense_modes.inc:124-138).
 */
rsv_status rsv_zgemm_batched(const void *d_a, const void *d_b, void *d_c, int dim, int batch, void *stream);

/* Change the transverse field h of an existing backend (the circuit shape and
 * buffers stay).  No reference counterpart (its field is fixed at
 * construction, cpp/ising_cuda_backend.hpp:26-29). */
rsv_status rsv_set_field(rsv_backend *backend, double field);

/* Geometry of a backend: qubits, layers, parameter count and device bytes held. */
rsv_status rsv_backend_info(rsv_backend *backend, int *num_qubits, int *num_layers,
                            size_t *num_params, size_t *device_bytes);

/*
 * Host-only description of the pass schedule the engine would run for
 * (num_qubits, num_layers), as text (one line per kernel launch).  Needs no
 * GPU.  Writes at most buf_size bytes including the terminating NUL and
 * returns the full length in *length_out.  No reference counterpart (it
 * replaces the reading of build_structured_forward_rotation_chunks and
 * run_structured_backward_sweep, reference
 * cpp/ising_cuda_structured_adjoint_modes.inc:18-71, 272-307).
 */
rsv_status rsv_describe_plan(int num_qubits, int num_layers, char *buf, size_t buf_size,
                             size_t *length_out);
/* The same for a given backward schedule (RSV_BACKWARD_*). */
rsv_status rsv_describe_plan_mode(int num_qubits, int num_layers, int backward_mode, char *buf,
                                  size_t buf_size, size_t *length_out);

/*
 * Host-only reference of the engine's ring-CNOT index maps (P and P^-1),
 * for checking the closed forms without a GPU.  Replaces
 * ring_cnot_layer_transformed_index (reference cpp/ising_cuda_kernels.cu:178-205).
 */
unsigned long long rsv_ring_map(unsigned long long index, int num_qubits, int inverse);

/*
 * Batched circuits: many independent ring-Ising circuits of uneven size
 * (2 <= num_qubits <= RSV_BATCH_MAX_QUBITS, 1 <= num_layers <=
 * RSV_BATCH_MAX_LAYERS, own field each) evaluated by ONE persistent kernel
 * launch.  No counterpart in the reference, which evaluates one circuit per
 * backend object; a batch of circuits there is a loop over
 * RingIsingCudaBackend::energy_and_grad (reference cpp/ising_cuda_backend.hpp:38-41).
 *
 * Packed layout: circuit c owns params[off_c, off_c + 2*n_c*L_c) with
 * off_c = sum_{j<c} 2*n_j*L_j, in the per-circuit layout above; gradients
 * use the same packing; energies are one f64 per circuit.
 *
 * rsv_batch_set_circuits builds (or reuses) the pass plan of every distinct
 * (num_qubits, num_layers), sorts the circuits by decreasing cost and uploads
 * the descriptors; it is synchronous.  rsv_batch_run_device enqueues the
 * whole batch on `stream` (used as given; 0 = legacy default stream): a
 * counter reset and one kernel launch, no allocation and no host
 * synchronisation, so it can be captured into a CUDA graph.  d_gradient_out
 * NULL computes energies only.  A handle is not re-entrant.
 */
#define RSV_BATCH_MAX_QUBITS 16
#define RSV_BATCH_MAX_LAYERS 64
typedef struct rsv_batch rsv_batch;

/* Handle whose scratch holds circuits of up to max_qubits qubits; slots = the
 * number of circuits in flight (0 = one per SM).  Bound to the current
 * device as rsv_create is. */
rsv_status rsv_batch_create(int max_qubits, int slots, rsv_batch **out);
rsv_status rsv_batch_destroy(rsv_batch *batch);

rsv_status rsv_batch_set_circuits(rsv_batch *batch, int count, const int *num_qubits,
                                  const int *num_layers, const double *fields);

/* Circuits and packed parameter count of the current description. */
rsv_status rsv_batch_info(rsv_batch *batch, int *count, size_t *num_params, int *slots,
                          size_t *device_bytes);

/* CTAs in flight for the following runs (1..the slots given at creation;
 * rounded down to whole clusters); used by the autotuner
 * (gpu_simulation_b200.batch). */
rsv_status rsv_batch_set_active_slots(rsv_batch *batch, int slots);

/*
 * Thread-block clusters of the batched kernel: 1, 2, 4 or 8 CTAs (default 8).
 * A cluster takes a group of circuits of the same (num_qubits, num_layers) and
 * spreads each over min(cluster, 2^max(0, num_qubits - 12)) of its CTAs,
 * which split every pass's 4096-amplitude tiles, meet at a cluster barrier
 * between passes and add their energy and gradient sums in fixed order
 * through distributed shared memory.  Results are deterministic for a given
 * cluster size and agree across sizes to rounding.  rsv_batch_set_cluster
 * re-groups the current circuits (synchronous); rsv_batch_cluster reports the
 * size, the number of work groups and how many clusters of that size the
 * device holds at once.  No reference counterpart.
 */
rsv_status rsv_batch_set_cluster(rsv_batch *batch, int cluster);
rsv_status rsv_batch_cluster(rsv_batch *batch, int *cluster_out, int *groups_out,
                             int *max_active_clusters_out);

rsv_status rsv_batch_run_device(rsv_batch *batch, const double *d_params, double *d_energy_out,
                                double *d_gradient_out, void *stream);

/* Host-memory convenience: set_circuits + copies + run + copies back,
 * synchronous.  gradient_out may be NULL. */
rsv_status rsv_batch_energy_and_grad(rsv_batch *batch, int count, const int *num_qubits,
                                     const int *num_layers, const double *fields,
                                     const double *params, size_t num_params,
                                     double *energy_out, double *gradient_out, void *stream);

/*
 * Warm-start network: a fully connected network in FP32 with FP32
 * accumulation, widths[0] inputs -> widths[1] -> ... -> widths[num_layers]
 * outputs, GELU (erf form) after every layer but the last.  It maps circuit
 * descriptors (h, n, L) to initial angles for the VQE; every reported energy
 * still comes from the simulator.  No counterpart in the reference (its VQE
 * starts from seeded random angles, ring_ising/runner.py).
 *
 * Weights are packed layer by layer: W_l (widths[l] x widths[l-1], row-major)
 * then b_l (widths[l]); gradients use the same packing.  All pointers are
 * device pointers; calls are asynchronous on `stream` (used as given).
 *   rsv_mlp_forward: x (batch x widths[0]) -> out (batch x widths[num_layers]);
 *     d_work (rsv_mlp_work_floats) receives the pre- and post-activations of
 *     the hidden layers for the backward pass.
 *   rsv_mlp_backward: d_dout = dLoss/dout -> d_grad = dLoss/dweights, using
 *     the d_work of the matching forward; d_scratch has
 *     rsv_mlp_scratch_floats entries.
 *   rsv_mlp_mse: loss = mean((out - target)^2) into d_loss (one float) and
 *     d_dout = 2 (out - target) / count; d_partials holds 256 floats.
 *   rsv_adam_f32 / rsv_adam_f64: one bias-corrected Adam step (step >= 1).
 */
size_t rsv_mlp_num_weights(int num_layers, const int *widths);
size_t rsv_mlp_work_floats(int num_layers, const int *widths, int batch);
size_t rsv_mlp_scratch_floats(int num_layers, const int *widths, int batch);
rsv_status rsv_mlp_forward(int num_layers, const int *widths, const float *d_weights, int batch,
                           const float *d_x, float *d_out, float *d_work, void *stream);
rsv_status rsv_mlp_backward(int num_layers, const int *widths, const float *d_weights, int batch,
                            const float *d_x, const float *d_work, const float *d_dout,
                            float *d_grad, float *d_scratch, void *stream);
rsv_status rsv_mlp_mse(size_t count, const float *d_out, const float *d_target, float *d_dout,
                       float *d_loss, float *d_partials, void *stream);
rsv_status rsv_adam_f32(float *d_params, const float *d_grad, float *d_m, float *d_v, size_t count,
                        float lr, float beta1, float beta2, float eps, int step, void *stream);
rsv_status rsv_adam_f64(double *d_params, const double *d_grad, double *d_m, double *d_v,
                        size_t count, double lr, double beta1, double beta2, double eps, int step,
                        void *stream);

/*
 * One plain gradient-descent step of a device-resident VQE loop: d_params -=
 * stepsize * d_grad (count values); the step's energy (*d_energy) and gradient
 * norm are stored at index *d_step_counter of d_energy_hist / d_gnorm_hist
 * (either may be NULL), then *d_step_counter is incremented, so one captured
 * (energy_and_grad, gd_step) pair can be replayed as a CUDA graph.  Replaces
 * the host-side update of the reference's training loop
 * (ring_ising/workflows/common.py:23-25, ring_ising/training/loop.py:93-115).
 */
rsv_status rsv_gd_step_f64(double *d_params, const double *d_grad, size_t count, double stepsize,
                           const double *d_energy, double *d_energy_hist, double *d_gnorm_hist,
                           int *d_step_counter, void *stream);

/*
 * One Adam step of a device-resident VQE loop, with torch.optim.Adam's update
 * (bias-corrected, no weight decay; d_m and d_v zero before the first step):
 * the step number is *d_step_counter + 1, read on the device; the step's
 * energy (*d_energy) is stored at index *d_step_counter of d_energy_hist (may be
 * NULL), then *d_step_counter is incremented, so one captured
 * (energy_and_grad, adam step) pair can be replayed as a CUDA graph.  The
 * reference's loop applies a host-side gradient step
 * (ring_ising/workflows/common.py:23-25); this is the torch Adam loop of a
 * Python caller moved onto the device.
 */
rsv_status rsv_adam_vqe_step_f64(double *d_params, const double *d_grad, double *d_m, double *d_v, size_t count,
                                 double lr, double beta1, double beta2, double eps, const double *d_energy,
                                 double *d_energy_hist, int *d_step_counter, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RSV_H */
