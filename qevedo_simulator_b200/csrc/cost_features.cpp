// Features of a planned pass for the learned cost model: what kind of pass
// it is (one plain gate, or a staged tile pass on the register, tensor-core
// or shared-memory kernel), its gates by type and width, where their qubits
// sit in the physical index, and the tile shape. All values are scaled to
// about [0, 1]. The model predicts the log of the pass's device time per
// 2^24 amplitudes from them.

#include <algorithm>
#include <cmath>

#include "program.hpp"

namespace qvdg {

namespace {

bool is_pm_one(const C& c) { return c.im == 0.0 && (c.re == 1.0 || c.re == -1.0); }

bool real_like(const HMatrix& m) {
  // real entries, or real diagonal with imaginary off-diagonal (RX form)
  bool real = true, rx = true;
  for (size_t r = 0; r < m.dim; ++r)
    for (size_t c = 0; c < m.dim; ++c) {
      const C& v = m.at(r, c);
      if (v.im != 0.0) real = false;
      if (r == c ? v.im != 0.0 : v.re != 0.0) rx = false;
    }
  return real || rx;
}

}  // namespace

void pass_features(const Target& t, const PlannedPass& p, const LoweredPass& lp, const StageUpload& up, float* f) {
  std::fill(f, f + kPassFeatures, 0.f);
  f[0] = 1.f;
  f[1] = float(t.n) / 32.f;
  f[30] = t.bits == 64 ? 1.f : 0.f;
  if (lp.block) {
    // A plain pass applying a fused group member by member (f[31] = 1).
    f[2] = 1.f;
    f[31] = 1.f;
    f[6] = float(p.block_qubits.size()) / 6.f;
    f[12] = 1.f;
    f[14] = float(p.ops.size()) / 64.f;
    uint32_t lo = 64, hi = 0, low4 = 0;
    for (uint32_t q : p.block_qubits) {
      const uint32_t ph = t.layout[q];
      lo = std::min(lo, ph);
      hi = std::max(hi, ph);
      if (ph < 4) ++low4;
    }
    f[9] = float(lo) / 32.f;
    f[10] = float(hi) / 32.f;
    f[11] = float(low4) / 6.f;
    int d1 = 0, diag = 0, realish = 0;
    for (const HOp& op : p.ops) {
      if (op.diagonal) {
        ++diag;
      } else {
        ++d1;
        if (real_like(op.matrix)) ++realish;
      }
    }
    f[15] = float(d1) / 64.f;
    f[18] = float(diag) / 64.f;
    f[29] = float(realish) / 64.f;
    return;
  }
  if (!lp.staged) {
    const HOp& op = p.ops[0];
    f[2] = 1.f;
    f[6] = float(op.targets.size()) / 6.f;
    f[7] = float(op.controls.size()) / 4.f;
    f[8] = op.diagonal ? 1.f : 0.f;
    uint32_t lo = 64, hi = 0, low4 = 0;
    for (uint32_t q : op.targets) {
      const uint32_t ph = t.layout[q];
      lo = std::min(lo, ph);
      hi = std::max(hi, ph);
      if (ph < 4) ++low4;
    }
    f[9] = float(lo) / 32.f;
    f[10] = float(hi) / 32.f;
    f[11] = float(low4) / 6.f;
    f[12] = float(std::ldexp(1.0, -int(op.controls.size())));
    // On the tensor-core plain pass: one tensor-core gate of its width (the
    // staged tensor passes' per-width counts).
    if (lp.plain.tensor) f[op.targets.size() == 4 ? 22 : 23] = 1.f / 16.f;
    return;
  }
  const int kind = int(lp.geo.tensor);  // 2 register, 1 tensor, 0 shared-memory
  f[3] = kind == 2 ? 1.f : 0.f;
  f[4] = kind == 1 ? 1.f : 0.f;
  f[5] = kind == 0 ? 1.f : 0.f;
  f[12] = 1.f;
  f[13] = float(p.tile_bits.size()) / 16.f;
  f[14] = float(p.ops.size()) / 64.f;
  std::vector<bool> local(64, false);
  for (uint32_t b : p.tile_bits) local[b] = true;
  int d1 = 0, d2 = 0, d3 = 0, diag = 0, pm = 0, gctl = 0, realish = 0;
  for (const HOp& op : p.ops) {
    if (op.diagonal) {
      ++diag;
      const std::vector<C> d = op.matrix.diagonal_entries();
      if (std::all_of(d.begin(), d.end(), is_pm_one)) ++pm;
    } else if (op.targets.size() == 1) {
      ++d1;
      if (real_like(op.matrix)) ++realish;
    } else if (op.targets.size() == 2) {
      ++d2;
    } else {
      ++d3;
    }
    for (auto& c : op.controls)
      if (!local[t.layout[c.first]]) {
        ++gctl;
        break;
      }
  }
  f[15] = float(d1) / 64.f;
  f[16] = float(d2) / 32.f;
  f[17] = float(d3) / 16.f;
  f[18] = float(diag) / 64.f;
  f[19] = float(pm) / 64.f;
  f[20] = float(gctl) / 32.f;
  if (kind != 2) {
    int k3 = 0, k4 = 0, k5 = 0, cuda_dense = 0, phases = 0;
    for (int i = 0; i < lp.geo.num_gates; ++i) {
      const TileGate& g = up.gates[lp.gate_offset + size_t(i)];
      if (g.kind == 2) {
        if (g.k <= 3) ++k3;
        else if (g.k == 4) ++k4;
        else ++k5;
      } else if (g.kind == 0) {
        ++cuda_dense;
      } else {
        ++phases;
      }
    }
    f[21] = float(k3) / 16.f;
    f[22] = float(k4) / 16.f;
    f[23] = float(k5) / 16.f;
    f[24] = float(cuda_dense) / 16.f;
    f[25] = float(phases) / 32.f;
  } else {
    f[26] = float(lp.geo.num_gates) / 16.f;  // register passes
  }
  uint32_t top = 0, spread = 0;
  for (uint32_t b : p.tile_bits) {
    top = std::max(top, b);
    if (b >= 20) ++spread;
  }
  f[27] = float(top) / 32.f;
  f[28] = float(spread) / 16.f;
  f[29] = float(realish) / 64.f;
}

void pair_features(const Target& t, const PlannedPass& second, float* f) {
  // A pass of two fused gates: the marker, the second gate's targets in the
  // position features, two tensor-core gates of width 5-6.
  f[21] = 1.f;
  f[23] = 2.f / 16.f;
  uint32_t lo = uint32_t(f[9] * 32.f + 0.5f), hi = uint32_t(f[10] * 32.f + 0.5f), low4 = uint32_t(f[11] * 6.f + 0.5f);
  for (uint32_t q : second.ops[0].targets) {
    const uint32_t ph = t.layout[q];
    lo = std::min(lo, ph);
    hi = std::max(hi, ph);
    if (ph < 4) ++low4;
  }
  f[9] = float(lo) / 32.f;
  f[10] = float(hi) / 32.f;
  f[11] = float(low4) / 6.f;
}

}  // namespace qvdg
