/*
 * Sharded single circuit: one ring-Ising VQE circuit whose complex128 state is
 * split over N = 2^g ranks (one GPU each, g <= 3), for circuits too large for
 * one GPU (n >= 33: 2^33 amplitudes are 128 GiB per state vector).
 *
 * The reference runs every n on one device (cpp/ising_cuda_backend.cu:229-241,
 * one allocation per buffer in cpp/ising_cuda_backend_internal.cuh:79-86) and
 * has no multi-GPU path; its per-wire conventions are kept: amplitude index
 * bit w is wire w, per wire U = RZ(phi) RY(theta), one layer = U on every wire
 * then CNOT(0,1), ..., CNOT(n-1,0) (cpp/ising_cuda_kernels.cu:22-25,178-205),
 * H = -sum Z_w Z_{w+1} - h sum X_w (cpp/ising_cuda_kernels.cu:313-358), the
 * gradient layout (l*n + w)*2 + {0: theta, 1: phi}.
 *
 * Two layouts of the global index x (n bits) over the ranks:
 *   C ("canonical"): rank = x bits [n-g, n), local offset = x bits [0, n-g);
 *   S ("swapped"):   rank = x bits [n-2g, n-g), local offset =
 *                    x bits [0, n-2g) | x bits [n-g, n) << (n-2g).
 * C -> S and S -> C are the same all-to-all of 2^(n-2g)-amplitude blocks
 * (block j of every rank goes to rank j, landing at block <sender>); no
 * packing.  The ring permutation y = P(x) is the other exchange: from S to C
 * forward (ring_pack, all-to-all, ring_unpack) and from C to S backward
 * (ring_pack_adjoint, all-to-all, ring_unpack_adjoint), chunks of
 * 2^(n-2g) amplitudes per rank pair.  One layer forward: rotate_local (wires
 * 0..n-g-1 in C), C -> S, ring_pack (wires n-g..n-1 rotated in the pack),
 * all-to-all, ring_unpack.  The collectives are the caller's (NCCL
 * all_to_all_single over NVLink between ranks).
 *
 * Forward gates are applied as (1/f) diag(1, e^{i phi}) RY(theta), f the larger
 * in magnitude of cos(theta/2) and sin(theta/2): the rotation is two
 * multiply-adds per amplitude and the phase four.  ring_pack, which ends each
 * layer's gates, multiplies by the layer's prod_w f_w, so after every layer
 * the state is the true one times a global phase, which cancels in the energy
 * and in every gradient sum.
 * Per-rank results go to d_result, f64[2 + 2 n L]: [0] the energy terms of
 * energy_local, [1] the field terms of ring_unpack_adjoint, [2 + k] gradient
 * entry k.  The caller sums the ranks' vectors in rank order (deterministic).
 * Every pointer is device memory of the current device; `stream` is a
 * cudaStream_t (NULL: the legacy default stream).  Calls are asynchronous.
 * Geometry limits: 0 <= g <= 3, n - 2g >= 12, n - g <= 31.
 */
#ifndef RSV_SHARD_H
#define RSV_SHARD_H

#include <stddef.h>

#include "rsv.h"

#ifdef __cplusplus
extern "C" {
#endif

/* RSV_OK if (num_qubits, g) is a supported geometry, else
 * RSV_ERR_INVALID_ARGUMENT with the reason in rsv_last_error(). */
rsv_status rsv_shard_check(int num_qubits, int g);

/* Doubles of scratch (d_scratch) the adjoint and energy calls need. */
size_t rsv_shard_scratch_doubles(int num_qubits, int g);

/* d_coef[l*n + w] = (cos theta/2, sin theta/2, cos phi/2, sin phi/2) as 4
 * doubles, from d_params f64[2 n L] (reference host coefficients:
 * cpp/ising_cuda_rotation_kernels.cu:661-675). */
rsv_status rsv_shard_coef(int num_qubits, int num_layers, const double *d_params, double *d_coef,
                          void *stream);

/* |0...0> in layout C on this rank's shard (2^(n-g) complex128). */
rsv_status rsv_shard_init(int num_qubits, int g, int rank, double *d_psi, void *stream);

/* The forward gates of layer `layer` on wires 0..n-g-1 (local in C), in place. */
rsv_status rsv_shard_rotate_local(int num_qubits, int g, int layer, const double *d_coef, double *d_psi,
                                  void *stream);

/* The inverse walk of layer `layer` on wires 0..n-g-1 on psi and lambda: per
 * wire the phi sum, diag(1, e^{-i phi}) (RZ^dagger up to a phase common to psi
 * and lambda), the theta sum, RY^dagger; the sums go to d_result (this
 * rank's share). */
rsv_status rsv_shard_rotate_local_adjoint(int num_qubits, int g, int num_layers, int layer,
                                          const double *d_coef, double *d_psi, double *d_lam,
                                          double *d_scratch, double *d_result, void *stream);

/* In layout C: lambda = (ZZ diagonal - h sum_{w < n-g} X_w) psi and
 * d_result[0] = <psi|lambda> (this rank's share). */
rsv_status rsv_shard_energy_local(int num_qubits, int g, int rank, double field, const double *d_psi,
                                  double *d_lam, double *d_scratch, double *d_result, void *stream);

/* Forward ring exchange, sender side (layout S): the forward gates of layer
 * `layer` on wires n-g..n-1 and the layer's factor prod_w f_w, then the amplitude of x goes to chunk rank_C(P(x)) of
 * d_send (2^g chunks of 2^(n-2g) amplitudes, in the order of x bits [0, n-2g)). */
rsv_status rsv_shard_ring_pack(int num_qubits, int g, int rank, int layer, const double *d_coef,
                               const double *d_psi_s, double *d_send, void *stream);

/* Forward ring exchange, receiver side: d_psi_c[y] (layout C) from the
 * received chunks, y = P(x). */
rsv_status rsv_shard_ring_unpack(int num_qubits, int g, int rank, const double *d_recv, double *d_psi_c,
                                 void *stream);

/* Backward ring exchange, sender side (layout C): psi and lambda at y go to
 * chunk rank_S(P^-1(y)). */
rsv_status rsv_shard_ring_pack_adjoint(int num_qubits, int g, int rank, const double *d_psi_c,
                                       const double *d_lam_c, double *d_send_psi, double *d_send_lam,
                                       void *stream);

/* Backward ring exchange, receiver side (layout S): psi and lambda at
 * x = P^-1(y); with add_field_terms, lambda += -h sum_{w >= n-g} X'_w psi
 * (the X terms of the wires that are global in C, in the pre-ring frame:
 * masks {w, w+1}, {0, 1, n-1} for w = n-1) and d_result[1] = their energy
 * share; with layer >= 0, the inverse walk of `layer` on wires n-g..n-1
 * (as in rsv_shard_rotate_local_adjoint) and their sums into d_result. */
rsv_status rsv_shard_ring_unpack_adjoint(int num_qubits, int g, int rank, int num_layers, int layer,
                                         const double *d_coef, double field, int add_field_terms,
                                         const double *d_recv_psi, const double *d_recv_lam,
                                         double *d_psi_s, double *d_lam_s, double *d_scratch,
                                         double *d_result, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RSV_SHARD_H */
