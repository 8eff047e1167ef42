// Plain passes of a fused 4-6 qubit dense gate on the tensor cores
// (dense_tc.cu), complex64 states.
#pragma once

#include <stdint.h>

#include <vector>

#include "engine.hpp"

namespace qvdg {

struct DenseTcGeom {
  uint64_t iters;          // CTA iterations: groups / (8192 / 2^K)
  uint64_t control_value;  // control bits that must be 1
  uint64_t offsets[64];    // member offsets, matrix index order (targets ascending)
  uint8_t fixed[40];       // sorted target and control positions
  int32_t num_fixed;
  uint32_t b_offset;  // byte offset of the gate's bf16 matrices in the tensor-core blob
};

// The staged form for gates with targets on bits 1, 2 and 3 (no controls).
struct DenseTcTileGeom {
  uint64_t iters;      // tiles of 128 groups: 2^(n - 7 - K)
  uint64_t dep_hi[8];  // physical offset of tile elements 2^(K+4) j (tile bits K+4..K+6)
  uint32_t b_offset;   // byte offset of the gate's bf16 matrices in the tensor-core blob
  uint8_t tile[16];    // physical positions of the 7 + K tile bits, ascending
  uint8_t tpos[8];     // tile position of each target (matrix bit order)
  uint8_t fpos[16];    // tile positions of the 7 free tile bits, ascending
};

// Whether a dense gate with these targets (physical) and controls runs on
// the tensor-core plain pass: complex64, 4-6 targets, at least one CTA
// iteration (8192 amplitudes) of selected groups, and the four lowest
// targets below bit 32.
bool dense_tc_ok(uint32_t n, int bits, const std::vector<uint32_t>& targets, size_t controls);

// Whether such a gate takes the staged variant (k_dense_tc_tile): no
// controls, targets (physical) on bits 1, 2 and 3, and not a 6-qubit gate
// that also targets bit 0.
bool dense_tc_staged(uint32_t n, const std::vector<uint32_t>& targets, size_t controls);

// `pg.targets` ascending, `pg.tc_offset` the byte offset of its bf16
// matrices (hi then lo, as the stage kernel's) in `tc_blob`.
void launch_dense_tc(StateImpl& s, const PlainGate& pg, const uint8_t* tc_blob);

}  // namespace qvdg
