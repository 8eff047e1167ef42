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

// Two fused 6-qubit gates in one plain pass (dense_tc_pair.cu): an
// iteration covers the 8192 amplitudes of 13 bits I (both gates' targets
// and the lowest other bits); gate 1's groups are loaded, multiplied on the
// tensor cores, transposed through shared memory into gate 2's groups,
// multiplied again and stored.
struct DenseTcPairGeom {
  uint64_t iters;              // 2^(n - 13)
  uint64_t imask;              // physical bits of I
  uint64_t grp1[7], grp2[7];   // offset of group bit j: the j-th lowest bit of I outside the gate's targets
  uint64_t hi1[4], hi2[4];     // offset of members 16 c.. (targets 4 and 5)
  uint32_t lo1[16], lo2[16];   // offset of members i = 0..15 (targets 0-3, below bit 32)
  uint32_t lgrp1[7], lgrp2[7]; // the same as byte offsets in the shared-memory transpose buffer (swizzled)
  uint32_t lhi1[4], lhi2[4];
  uint32_t llo1[16], llo2[16];
  uint32_t b1_offset, b2_offset;  // byte offsets of the gates' bf16 matrices in the tensor-core blob
  uint8_t ibits[16];              // the 13 bits of I, ascending
  int32_t vw1, vw2;               // access width in complex64 of gate 1's loads and gate 2's stores (1, 2, 4)
};

// The pair geometry for gates on physical targets t1 and t2 (6 each,
// ascending) of an n-qubit state, with the gates' bf16 matrices at
// b1_offset and b2_offset; the shared-memory swizzle is chosen so both
// gates' group-parallel accesses are free of bank conflicts where possible.
DenseTcPairGeom dense_tc_pair_geom(uint32_t n, const std::vector<uint32_t>& t1, const std::vector<uint32_t>& t2,
                                   size_t b1_offset, size_t b2_offset);
// Whether two gates (physical targets, no controls) can share a pair pass.
bool dense_tc_pair_ok(uint32_t n, int bits, const std::vector<uint32_t>& t1, const std::vector<uint32_t>& t2);
// The layout part of that test on physical target masks (6 targets each;
// complex64, at least 14 qubits and targets below bit 32 assumed).
bool dense_tc_pair_masks_ok(uint64_t m1, uint64_t m2);
void launch_dense_tc_pair(StateImpl& s, const DenseTcPairGeom& g, const uint8_t* tc_blob);

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
