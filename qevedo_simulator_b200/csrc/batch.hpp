// Batched layered circuits (one persistent launch for many small circuits).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "qvdg.h"

namespace qvdg {

constexpr int kBatchMaxQubits = QVDG_BATCH_MAX_QUBITS;

// One circuit of the batch on the device.
struct BatchCircuit {
  uint32_t num_qubits, num_layers, entangler;
  uint32_t form;   // kBatchPhased | kBatchLeft | kBatchRight, or 0: generic 2x2 matrices
  uint64_t gates;  // index of its first gate record (kBatchGateSlots complex64 each) in the gate buffer
  uint64_t out;    // index of its first <Z> output
};

// A gate record: the 2x2 matrix (m00, m01, m10, m11) in slots 0-3 for a
// generic circuit; for a phased one U = diag(p0, p1) R diag(q0, q1) with R
// real: slots (r00, r01), (r10, r11), p0, p1, q0, q1.
constexpr int kBatchGateSlots = 8;
constexpr uint32_t kBatchPhased = 1, kBatchLeft = 2, kBatchRight = 4;

// Everything one launch of the batch kernel reads.
struct BatchLaunch {
  const BatchCircuit* circuits = nullptr;
  const uint32_t* order = nullptr;  // circuits in the order CTAs take them
  uint32_t count = 0;
  const float2* gates = nullptr;
  float2* slots = nullptr;  // per-CTA HBM state for circuits wider than the tile
  uint64_t slot_elems = 0;
  double* out = nullptr;
  uint32_t* queue = nullptr;  // work counter, reset by each launch
  int tile_qubits = 13;
  int threads = 256;
  int ctas = 0;
};

// Resident CTAs per SM of the batch kernel for a shape (0 if it cannot run).
int batch_kernel_occupancy(int threads, int tile_qubits);
// Reset the work counter and launch the persistent kernel on `stream`.
void launch_batch(const BatchLaunch& b, cudaStream_t stream);

}  // namespace qvdg

// Host side (batch_host.cpp), called by the C ABI in api.cpp.
namespace qvdg {
qvdg_batch* batch_create(const qvdg_layered_circuit* circuits, size_t count, const qvdg_batch_options* options);
void batch_destroy(qvdg_batch* b);
void batch_set_gates(qvdg_batch* b, const double* gates, size_t num_matrices);
void batch_run(qvdg_batch* b, double* expect_z, size_t count, double* seconds);
void batch_info(const qvdg_batch* b, qvdg_batch_summary* info);
size_t batch_tuning(const qvdg_batch* b, uint32_t* tile_qubits, uint32_t* threads, double* seconds, size_t capacity);
}  // namespace qvdg
