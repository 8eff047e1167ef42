// Device-side form of a stage: the tile geometry and the gate program.
#pragma once

#include <stdint.h>

#include <vector>

#include "engine.hpp"
#include "host.hpp"

namespace qvdg {

struct StageConfig;
struct PlannedPass;

constexpr size_t kMaxStageGates = 256;

// One gate of a stage's program, on tile-local bit positions.
struct TileGate {
  uint8_t kind;    // 0 dense, 1 diagonal
  uint8_t k;       // targets
  uint8_t nfixed;  // entries of `fixed`
  uint8_t pad;
  uint32_t lcm, lcv;  // local control bits (tile-local positions) and their values
  uint64_t gcm, gcv;  // global control bits (physical positions) and their values
  uint32_t mat;       // complex-element offset of the matrix / diagonal
  uint32_t pad2;
  uint8_t tgt[16];    // matrix bit j -> tile-local bit; diagonal global targets: 0x80 | physical bit
  uint8_t fixed[24];  // dense: sorted local targets and controls; diagonal: sorted local controls
};

struct TileGeom {
  uint64_t num_tiles;
  uint64_t tc_offset;  // byte offset of this pass's tensor-core gate matrices
  int32_t L, B;
  int32_t num_gates;
  uint32_t tc_bytes;   // bytes of those matrices (kept in shared memory)
  uint32_t tensor;     // 1: launch the tensor-core kernel
  int32_t pad;
  uint8_t tile_bits[48];  // ascending physical bits of the tile
};

struct LoweredPass {
  bool staged = true;
  TileGeom geo{};
  size_t gate_offset = 0;  // first TileGate of this pass in the upload
  PlainGate plain;         // when !staged
};

struct DeviceUpload {
  const TileGate* gates = nullptr;
  const void* mats = nullptr;
  const uint8_t* tc = nullptr;  // bf16 gate matrices of tensor-core gates
};

struct StageUpload {
  std::vector<TileGate> gates;
  std::vector<double> mats;  // interleaved complex, converted at upload
  std::vector<uint8_t> tc;   // tensor-core gate matrices, bf16 hi then lo per gate
  size_t push_matrix(const std::vector<C>& entries) {
    const size_t off = mats.size() / 2;
    for (const C& c : entries) {
      mats.push_back(c.re);
      mats.push_back(c.im);
    }
    return off;
  }
};

struct Target;
LoweredPass lower_pass(const Target& t, const PlannedPass& p, const StageConfig& cfg, StageUpload& up);
void launch_pass(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev);
void launch_stage_tc(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev);
size_t tc_smem_bytes(const TileGeom& geo);

// Bytes of one tensor-core gate's matrices (bf16 hi and lo, 2^(k+1) square).
inline size_t tc_gate_bytes(size_t k) { return size_t(4) << (2 * (k + 1)); }
// Shared memory the tensor-core kernel may spend on a pass's gate matrices.
inline size_t tc_budget(uint32_t L) { return size_t(220 * 1024) - (size_t(16) << L); }

}  // namespace qvdg
