// Internal interface between the C ABI (api.cpp) and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"
#include "qvdg.h"

namespace qvdg {

// A device buffer that grows on demand (never shrinks while its owner lives).
struct DeviceScratch {
  void* ptr = nullptr;
  size_t bytes = 0;
  void* get(size_t need);  // may reallocate (contents are lost)
  void release();
};

// A pinned host buffer that grows on demand.
struct HostScratch {
  void* ptr = nullptr;
  size_t bytes = 0;
  void* get(size_t need);
  void release();
};

// One fused gate ready for a plain (one pass) launch, on physical bits.
struct PlainGate {
  bool diagonal = false;
  std::vector<uint32_t> targets;                      // physical, matrix bit j = targets[j]
  std::vector<std::pair<uint32_t, bool>> controls;    // physical
  size_t matrix_offset = 0;  // element offset (complex) of its matrix / diagonal in the upload
  bool tensor = false;       // dense, on the tensor-core plain pass (targets ascending)
  size_t tc_offset = 0;      // tensor: byte offset of its bf16 matrices in the tensor-core blob
};

struct StateImpl {
  uint32_t n = 0;
  int bits = 32;
  void* amp = nullptr;  // 2^n interleaved complex in `bits` precision
  size_t amp_bytes = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::vector<uint32_t> layout;  // logical -> physical
  // |0...0> since the last zero(): a relabel costs no data movement and a
  // program may run its zero-start passes. Mutable: handing out the device
  // buffer (through a const handle) clears it, as the caller may write.
  mutable bool zero_state = false;
  DeviceScratch work;            // device workspace (uploads, reductions, sampling)
  DeviceScratch work2;
  HostScratch host;              // pinned staging
  int device = 0;
  int sms = 148;
  int* status = nullptr;  // device word set by kernels whose bounded waits gave up
  // Per-pass device timings of the last gate run (when enabled).
  bool record_passes = false;
  std::vector<cudaEvent_t> pass_events;
  std::vector<double> pass_seconds, pass_bytes;
  std::vector<int> pass_kinds;  // 1 staged tile pass, 0 plain gate pass, 2/3 plain pass on the tensor cores (direct/staged)

  size_t elem_bytes() const { return bits == 32 ? 8 : 16; }
  uint64_t size() const { return uint64_t(1) << n; }
  bool identity_layout() const {
    for (size_t q = 0; q < layout.size(); ++q)
      if (layout[q] != q) return false;
    return true;
  }
};

// ---- gates.cu
// Launch one plain gate pass; `matrices` is the device copy of the upload
// (complex in the state's precision).
void launch_plain_gate(StateImpl& s, const PlainGate& g, const void* matrices);
// Exchange physical bit pairs in one pass.
void launch_swap_bits(StateImpl& s, const std::vector<std::pair<uint32_t, uint32_t>>& pairs);
// |0...0>.
void launch_zero(StateImpl& s);
// Convert `count` logical amplitudes starting at `first` to complex128 (out)
// or from complex128 (in), through the layout.
void launch_export(StateImpl& s, uint64_t first, uint64_t count, double* out_dev);
void launch_import(StateImpl& s, uint64_t first, uint64_t count, const double* in_dev);
void launch_scale(StateImpl& s, double factor);

// ---- measure.cu
double norm_sqr(StateImpl& s);
double probability_one(StateImpl& s, uint32_t physical_bit);
// P(bit = 1) for every physical bit, and the total.
void bit_probabilities(StateImpl& s, std::vector<double>& p1, double& total);
// Sample and count by classical key (clbits < 64; logical measured qubits);
// keys ascending.
size_t sample_counts(StateImpl& s, size_t shots, const double* uniforms_host, const uint32_t* qubits,
                     const uint32_t* clbits, size_t nm, std::vector<uint64_t>& keys, std::vector<uint64_t>& counts);
// <psi|P|psi> for X/Y bits x, Z/Y bits z (physical) and ny Y factors.
double expect_pauli(StateImpl& s, uint64_t x, uint64_t z, int ny);
// bit_probabilities over a caller's device buffer, with file-scope scratch
// instead of an allocated workspace (qvdg_bit_probabilities_noalloc).
void bit_probabilities_noalloc(const void* amplitudes, uint32_t num_qubits, uint32_t precision_bits,
                               cudaStream_t stream, double* p1, double* total);
void probabilities(StateImpl& s, double* out_host);
// Bit-exact restatement of the reference sampler; outcomes are physical
// indices in chunk order, then mapped to logical with the layout.
size_t sample_unordered(StateImpl& s, size_t shots, const double* uniforms_host, uint64_t* out_host);

// max over logical indices of |a - b| (both states the same size).
double max_abs_diff(StateImpl& a, StateImpl& b);

// ---- sort.cu
// Ascending stable LSD radix sort of `count` 64-bit keys in place (`tmp` has
// room for `count` keys). `work` provides temporary device memory.
void radix_sort_u64(uint64_t* keys, uint64_t* tmp, size_t count, DeviceScratch& work, cudaStream_t stream);

// ---- mlp.cu (learned cost model network)
qvdg_mlp* mlp_create(uint32_t inputs, uint32_t hidden, uint64_t seed);
void mlp_destroy(qvdg_mlp* m);
size_t mlp_num_params(const qvdg_mlp* m);
void mlp_get_params(const qvdg_mlp* m, float* out);
void mlp_set_params(qvdg_mlp* m, const float* in);
void mlp_forward(qvdg_mlp* m, const float* x, size_t rows, float* y);
float mlp_gradients(qvdg_mlp* m, const float* x, const float* t, size_t rows, float* grads);
float mlp_train(qvdg_mlp* m, const float* x, const float* t, size_t rows, uint32_t epochs, uint32_t batch, float lr,
                uint64_t seed);

}  // namespace qvdg
