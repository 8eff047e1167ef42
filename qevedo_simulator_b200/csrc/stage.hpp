// Staged execution: many gates per pass over HBM.
//
// The reference cuts the state into cache-sized regions of consecutive
// blocks and runs a *stage* (every pending gate whose non-diagonal targets
// are local) region by region, relabelling qubits with swap passes when the
// next gates need global qubits (src/blocking.rs:1-302).
//
// Here a stage's *tile* is 2^L amplitudes that differ in an arbitrary set of
// L physical bits: the low B bits (so every tile is a set of contiguous
// 2^B-amplitude runs, coalesced 16-byte accesses) plus any L - B others. A
// CTA loads a tile into shared memory, applies every gate of the stage in
// place and stores it back, so choosing the tile's bits per stage replaces
// the reference's relabelling passes: no data moves to change which qubits
// are local. Global controls are tile predicates and diagonal gates with
// global targets read those bits from the tile's base index, as the
// reference's RegionOp does (src/blocking.rs:57-149).
#pragma once

#include <vector>

#include "engine.hpp"
#include "host.hpp"
#include "qvdg.h"

namespace qvdg {

// One planned pass: either a staged tile pass or a single plain gate.
struct PlannedPass {
  bool staged = true;
  std::vector<uint32_t> tile_bits;  // physical bits of the tile, ascending
  std::vector<HOp> ops;             // fused ops of the stage (logical qubits); block: the group's member ops
  bool block = false;               // one plain pass applying a fused group's member gates in registers
  std::vector<uint32_t> block_qubits;  // block: the group's logical qubits
};

struct StageConfig {
  uint32_t tile_bits;  // L
  uint32_t low_bits;   // B
  bool tensor;         // fused 3-6 qubit gates on the tensor cores
  bool reg;            // CUDA-core stages gate by gate in registers (unfused)
  bool plain_tensor;   // plain passes: fused 4-6 qubit dense gates on the tensor cores
};

struct Target;
StageConfig stage_config(const Target& t, uint32_t requested_tile_bits, bool tensor);

// Whether a fused op of a stage runs on the tensor cores.
bool tensor_eligible(const HOp& op, uint32_t tile_bits);

// Plan stages for `ops` on the state's current layout (greedy look-ahead in
// the manner of plan_swaps/extract, src/blocking.rs:151-226).
std::vector<PlannedPass> plan_stages(const std::vector<HOp>& ops, const std::vector<uint32_t>& layout, uint32_t n,
                                     const StageConfig& cfg, size_t max_fused);

}  // namespace qvdg
