// Device-side form of a stage: the tile geometry and the gate program.
#pragma once

#include <stdint.h>

#include <memory>
#include <vector>

#include "dense_tc.hpp"
#include "engine.hpp"
#include "host.hpp"

namespace qvdg {

struct StageConfig;
struct PlannedPass;

constexpr size_t kMaxStageGates = 256;

// One gate of a stage's program, on tile-local bit positions.
// Gate kinds: 0 dense on CUDA cores, 1 diagonal, 2 dense on tensor cores,
// 3 one phase on the elements whose target and control bits hold.
struct TileGate {
  uint8_t kind;
  uint8_t k;       // targets
  uint8_t nfixed;  // entries of `fixed`
  uint8_t absorb;  // tensor passes: one-phase gates just before this one applied in its gather (kind 2)
                   // or, for kind 3, 1 when the phase is exactly -1
  uint32_t lcm, lcv;  // local control bits (tile-local positions) and their values
  uint64_t gcm, gcv;  // global control bits (physical positions) and their values
  uint32_t mat;       // complex-element offset of the matrix / diagonal (tensor passes: byte offset in the pass blob)
  uint32_t tab;       // tensor passes: byte offset of the gate's index tables in the pass blob
  uint8_t tgt[16];    // matrix bit j -> tile-local bit; diagonal global targets: 0x80 | physical bit
  uint8_t fixed[24];  // dense: sorted local targets and controls; diagonal: sorted local controls
};

struct TileGeom {
  uint64_t num_tiles;
  uint64_t tc_offset;  // byte offset of this pass's tensor-core gate matrices
  int32_t L, B;
  int32_t num_gates;
  uint32_t tc_bytes;   // bytes of those matrices (kept in shared memory)
  uint32_t tensor;     // 1: tensor-core kernel, 2: register-blocked kernel, 0: k_stage
  int32_t tail_absorb;  // tensor passes: trailing one-phase gates applied in the final store
  uint8_t tile_bits[48];  // ascending physical bits of the tile
};

struct LoweredPass {
  bool staged = true;
  bool block = false;  // plain pass of k_block (geo.L = group qubits, geo.tile_bits = their physical bits)
  TileGeom geo{};
  size_t gate_offset = 0;  // first TileGate of this pass in the upload
  PlainGate plain;         // when !staged (a pair pass: its first gate)
  // Two fused gates in one plain pass on the tensor cores (dense_tc_pair.cu).
  std::shared_ptr<const DenseTcPairGeom> pair;
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
// A plain pass's gate for the tensor-core kernel: targets (physical)
// ascending and its bf16 matrices permuted to match.
struct PlainTcBlob {
  std::vector<uint32_t> targets;
  std::vector<uint8_t> blob;
};
bool plain_tc_eligible(const Target& t, const PlannedPass& p, const StageConfig& cfg);
// Pads a tensor-core blob to a 16-byte boundary (the kernels copy it in
// 16-byte vectors).
void blob_align(std::vector<uint8_t>& blob);
PlainTcBlob plain_tc_blob(const Target& t, const HOp& op);
// `pre`: the pass's plain_tc_blob when the caller computed it already
// (moved from).
LoweredPass lower_pass(const Target& t, const PlannedPass& p, const StageConfig& cfg, StageUpload& up,
                       PlainTcBlob* pre = nullptr);
void launch_pass(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev);
void launch_stage_tc(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev);
// Plain passes applying a fused group gate by gate in registers (block.cu).
bool block_pass_ok(const Target& t, const std::vector<HOp>& members, const std::vector<uint32_t>& qubits);
LoweredPass lower_block_pass(const Target& t, const PlannedPass& p, StageUpload& up);
void launch_block(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev);
// Register-blocked CUDA-core stages (stage_reg.cu): gates unfused, four tile
// bits per register pass.
bool register_pass_ok(const Target& s, const PlannedPass& p);
LoweredPass lower_register_pass(const Target& s, const PlannedPass& p, const StageConfig& cfg, StageUpload& up);
void launch_stage_reg(StateImpl& s, const LoweredPass& lp, const DeviceUpload& dev);
size_t tc_smem_bytes(const TileGeom& geo);

// Bytes of one tensor-core gate's matrices (bf16 hi and lo, 2^(k+1) square).
inline size_t tc_gate_bytes(size_t k) { return size_t(4) << (2 * (k + 1)); }
// The tensor-core kernel's tile: 12 local qubits (32 KiB of complex64), two
// CTAs per SM; each CTA keeps its pass's gate data (at most kTcBlobBytes)
// and descriptors (at most kTcMaxGates) in shared memory.
constexpr uint32_t kTcTileBits = 12;
constexpr size_t kTcBlobBytes = 40 * 1024;
constexpr int kTcMaxGates = 64;
inline size_t tc_budget(uint32_t) { return kTcBlobBytes; }

// The tensor-core kernel stores tile element e at position e ^ tc_swizzle(e)
// in shared memory: the low 4 index bits are XORed with bits 4-7, 8-11 and
// 12-15, so warps whose lanes step by 16 or 256 elements (group bases of
// gates on low tile bits) spread over all banks. The map is XOR-linear and
// an involution.
__host__ __device__ inline uint32_t tc_swizzle(uint32_t e) { return ((e >> 4) ^ (e >> 8) ^ (e >> 12)) & 15u; }
__host__ __device__ inline uint32_t tc_swz(uint32_t e) { return e ^ tc_swizzle(e); }
// The same on byte offsets (element index * 8).
__host__ __device__ inline uint32_t tc_swz_bytes(uint32_t b) { return tc_swz(b >> 3) << 3; }

}  // namespace qvdg
