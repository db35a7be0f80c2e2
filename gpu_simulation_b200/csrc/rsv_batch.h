// Descriptors of the batched circuit kernel (rsv_batch.cu), shared with the
// host scheduler (rsv_backend.cpp).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace rsv {

constexpr int kBatchMaxQubits = 16;
constexpr int kBatchMaxLayers = 64;

enum BatchStepKind : int { kBatchForward = 0, kBatchEnergy = 1, kBatchBackward = 2 };

// One tile shape of a plan (see rsv_types.h PassParams for the meaning).
struct BatchTile {
  unsigned int vec[12];
  int gate_wire[12];
  int wire_tile_bit[32];
  int num_runs;
  int run_start[4];
  int run_len[4];
  unsigned int num_tiles;
};

// One launch of the single-circuit plan: a pass over all tiles, or the energy
// (psi_in = chi buffer, psi_out = mu buffer).
struct BatchStep {
  int kind;
  int tile;
  int layer;
  int psi_load, lam_load, psi_store, lam_store;
  int phase;
  int psi_in, psi_out, lam_in, lam_out;
};

struct BatchPlan {
  int first_step;
  int num_steps;
  int undo_off;  // undo order of the wires within a backward layer
};

struct BatchCircuit {
  int n, L;
  double h;
  long long param_off;  // offset of the circuit's parameters (and gradient)
  int plan;
  int index;            // position in the caller's list (energy output slot)
};

// A work item of one thread-block cluster: `count` circuits of the same plan
// (order[first .. first + count)), each spread over `per` CTAs of the cluster
// (per = min(cluster size, tiles per pass)); count * per <= cluster size.
struct BatchGroup {
  int first;
  int count;
  int per;
};

struct BatchArgs {
  int count;
  const BatchCircuit *circuits;
  const int *order;     // circuits in decreasing cost, circuits of a group adjacent
  const BatchGroup *groups;
  int num_groups;
  int *counter;         // work counter, zero at launch
  const BatchPlan *plans;
  const BatchStep *steps;
  const BatchTile *tiles;
  const int *undo;
  const double *params;
  double *energy_out;
  double *grad_out;     // or null
  unsigned char *scratch;
  size_t slot_bytes;
  size_t state_bytes;
};

size_t batch_smem_bytes();
size_t batch_slot_table_bytes();
cudaError_t configure_batch_kernel();
// grid: a multiple of `cluster` (1, 2, 4 or 8 CTAs per thread-block cluster)
cudaError_t launch_batch(const BatchArgs &A, int grid, int cluster, cudaStream_t s);
// clusters of `cluster` CTAs that can be resident at once (0 if none)
int batch_max_active_clusters(int cluster);

}  // namespace rsv
