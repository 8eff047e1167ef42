// Stage planning and orchestration on the host (see stage.hpp).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <random>
#include <cstring>
#include <string>

#include "dense_tc.hpp"
#include "program.hpp"
#include "stage.hpp"
#include "stage_kernel.hpp"

namespace qvdg {

namespace {

bool contains(const std::vector<uint32_t>& v, uint32_t x) { return std::find(v.begin(), v.end(), x) != v.end(); }

// Walk pending ops in program order and take each op that `can_run` accepts
// and that no earlier pending op on one of its qubits holds back
// (src/blocking.rs:157-179).
std::vector<size_t> extract(const std::vector<HOp>& ops, const std::vector<bool>& done,
                            const std::function<bool(const HOp&)>& can_run) {
  std::vector<size_t> taken;
  std::vector<uint32_t> blocked;
  for (size_t i = 0; i < ops.size(); ++i) {
    if (done[i]) continue;
    const std::vector<uint32_t> qs = ops[i].qubits();
    bool touches = false;
    for (uint32_t q : qs)
      if (contains(blocked, q)) touches = true;
    if (!touches && can_run(ops[i])) {
      taken.push_back(i);
    } else {
      for (uint32_t q : qs)
        if (!contains(blocked, q)) blocked.push_back(q);
    }
  }
  return taken;
}

}  // namespace

bool tensor_eligible(const HOp& op, uint32_t L) {
  const size_t k = op.targets.size();
  return !op.diagonal && op.controls.empty() && k >= 3 && k + 7 <= L && k <= 6;
}

// Upper bound of the shared-memory bytes one op takes in a tensor pass's
// blob (its matrix or diagonal, and its index tables).
static size_t tensor_blob_bytes(const HOp& op, uint32_t L) {
  // tables: 768 bytes of enumeration spreads, plus 256 of member offsets
  // (dense) or 768 of diagonal index parts; 32 bytes of alignment.
  if (op.diagonal) return (size_t(8) << op.targets.size()) + 768 + 768 + 32;
  const size_t k = op.targets.size() + op.controls.size();
  const size_t data = (k >= 3 && k + 7 <= L) ? tc_gate_bytes(k) : (size_t(8) << (2 * k));
  return data + 768 + 256 + 32;
}

StageConfig stage_config(const Target& s, uint32_t requested, bool tensor) {
  StageConfig c{};
  c.tensor = tensor && s.bits == 32;
  c.reg = !c.tensor;
  const uint32_t lmax = c.tensor ? kTcTileBits : (s.bits == 32 ? 13 : 12);  // 32-64 KiB tiles
  uint32_t L = requested ? std::min<uint32_t>(requested, lmax) : lmax;
  if (!requested && !c.tensor) {
    // Keep at least two tiles per SM on small states.
    uint32_t spread = 0;
    while ((uint32_t(1) << spread) < uint32_t(2 * s.sms)) ++spread;
    while (L > 8 && s.n > L && s.n - L < spread) --L;
  }
  L = std::min<uint32_t>(L, s.n);
  c.tile_bits = L;
  // Contiguous low bits: 16 amplitudes (128 bytes of complex64, 256 of
  // complex128) per run, fewer for tiny tiles so that half the tile is free.
  c.low_bits = std::min<uint32_t>(4, L / 2);
  return c;
}

std::vector<PlannedPass> plan_stages(const std::vector<HOp>& ops, const std::vector<uint32_t>& layout, uint32_t n,
                                     const StageConfig& cfg, size_t max_fused) {
  const size_t budget = cfg.tensor ? tc_budget(cfg.tile_bits) : 0;
  const uint32_t L = cfg.tile_bits, B = cfg.low_bits;
  std::vector<PlannedPass> passes;
  std::vector<bool> done(ops.size(), false);
  size_t remaining = ops.size();
  std::vector<uint32_t> physical_of(layout);  // logical -> physical
  while (remaining > 0) {
    // Qubits the next gates need, greedily in dependency order, up to the
    // tile's free capacity (plan_swaps, src/blocking.rs:197-226).
    std::vector<uint32_t> wanted;  // logical qubits
    const uint32_t capacity = L - B;
    extract(ops, done, [&](const HOp& op) {
      if (op.diagonal) return true;
      std::vector<uint32_t> fresh;
      for (uint32_t q : op.targets)
        if (physical_of[q] >= B && !contains(wanted, q)) fresh.push_back(q);
      if (wanted.size() + fresh.size() > capacity) return false;
      wanted.insert(wanted.end(), fresh.begin(), fresh.end());
      return true;
    });
    std::vector<uint32_t> bits;
    for (uint32_t p = 0; p < B; ++p) bits.push_back(p);
    for (uint32_t q : wanted) bits.push_back(physical_of[q]);
    // Fill the rest of the tile with the lowest unused bits (longer runs).
    for (uint32_t p = B; p < n && bits.size() < L; ++p)
      if (!contains(bits, p)) bits.push_back(p);
    std::sort(bits.begin(), bits.end());
    auto local = [&](uint32_t q) { return contains(bits, physical_of[q]); };
    const std::vector<size_t> taken = extract(ops, done, [&](const HOp& op) {
      if (op.diagonal) return true;
      return std::all_of(op.targets.begin(), op.targets.end(), local);
    });
    if (taken.empty()) {
      // The next gate has more targets than a tile holds: one plain pass.
      const size_t i = size_t(std::find(done.begin(), done.end(), false) - done.begin());
      done[i] = true;
      --remaining;
      PlannedPass p;
      p.staged = false;
      p.ops.push_back(ops[i]);
      passes.push_back(std::move(p));
      continue;
    }
    std::vector<HOp> stage_ops;
    for (size_t i : taken) {
      done[i] = true;
      stage_ops.push_back(ops[i]);
    }
    remaining -= taken.size();
    // Fuse only ops whose qubits are all local: a fused matrix on a global
    // control or diagonal target would make it a global target
    // (src/blocking.rs:265-267).
    // The register-blocked kernel applies gates one by one (fusing would
    // only add arithmetic there); runs on one qubit still merge.
    std::vector<HOp> fused = fuse_where(stage_ops, cfg.reg ? 1 : max_fused, [&](const HOp& op) {
      for (uint32_t q : op.qubits())
        if (!local(q)) return false;
      return true;
    });
    // Split very long stages so one launch's gate program stays bounded,
    // and so a tensor-core pass's gate matrices fit in shared memory.
    PlannedPass p;
    p.tile_bits = bits;
    size_t tc_bytes = 0;
    for (HOp& op : fused) {
      const size_t b = cfg.tensor ? tensor_blob_bytes(op, L) : 0;
      const size_t max_gates = cfg.tensor ? size_t(kTcMaxGates) : kMaxStageGates;
      if (!p.ops.empty() && (p.ops.size() >= max_gates || (b > 0 && tc_bytes + b > budget))) {
        passes.push_back(std::move(p));
        p = PlannedPass();
        p.tile_bits = bits;
        tc_bytes = 0;
      }
      tc_bytes += b;
      p.ops.push_back(std::move(op));
    }
    if (!p.ops.empty()) passes.push_back(std::move(p));
  }
  return passes;
}

Target target_of(const StateImpl& s) {
  Target t;
  t.n = s.n;
  t.bits = s.bits;
  t.sms = s.sms;
  t.layout = s.layout;
  return t;
}

namespace {

// Logical qubits a pass touches (targets, controls, a block's qubits).
uint64_t pass_qubits(const PlannedPass& p) {
  uint64_t m = 0;
  for (const HOp& op : p.ops) {
    for (uint32_t q : op.targets) m |= uint64_t(1) << q;
    for (auto& c : op.controls) m |= uint64_t(1) << c.first;
  }
  for (uint32_t q : p.block_qubits) m |= uint64_t(1) << q;
  return m;
}

// The zero-start prefix of a run from |0...0>: the plain single-op passes
// before the one after which every qubit has been touched.
size_t zero_prefix(const std::vector<PlannedPass>& passes, uint32_t n) {
  const uint64_t all = n >= 64 ? ~uint64_t(0) : (uint64_t(1) << n) - 1;
  uint64_t touched = 0;
  size_t k = 0;
  for (const PlannedPass& p : passes) {
    if (p.staged || p.block || p.ops.size() != 1) break;
    touched |= pass_qubits(p);
    if (touched == all) break;
    ++k;
  }
  return k;
}

constexpr size_t kPairWindow = 8;  // how far ahead a pass looks for its partner

// Whether a pass is a candidate for a pair pass by its structure: one dense
// 6-qubit op without controls.
bool pair_candidate(const PlannedPass& p) {
  return !p.staged && !p.block && p.ops.size() == 1 && p.ops[0].controls.empty() && !p.ops[0].diagonal &&
         p.ops[0].targets.size() == 6;
}

// What the layout search knows of a plan's passes: the zero-start prefix,
// each pass's logical target mask and touched qubits, and which passes may
// pair by their structure.
struct PairSearch {
  size_t from = 0;
  std::vector<uint64_t> logical, touches;
  std::vector<char> candidate;
  size_t count = 0;  // candidates after the prefix

  PairSearch(const std::vector<PlannedPass>& passes, uint32_t n)
      : from(zero_prefix(passes, n)), logical(passes.size(), 0), touches(passes.size(), 0),
        candidate(passes.size(), 0) {
    for (size_t i = 0; i < passes.size(); ++i) {
      touches[i] = pass_qubits(passes[i]);
      candidate[i] = pair_candidate(passes[i]);
      if (candidate[i]) {
        for (uint32_t q : passes[i].ops[0].targets) logical[i] |= uint64_t(1) << q;
        count += i >= from;
      }
    }
  }

  // Pairs that the pairing below would make on `layout` (logical ->
  // physical), by the layout test alone (about 1.4 us for 45 passes).
  size_t pairs(const std::vector<uint32_t>& layout) const {
    const size_t np = logical.size();
    std::vector<uint64_t> phys(np, 0);
    for (size_t i = 0; i < np; ++i)
      if (candidate[i])
        for (uint64_t m = logical[i]; m; m &= m - 1) phys[i] |= uint64_t(1) << layout[__builtin_ctzll(m)];
    std::vector<char> used(np, 0);
    size_t made = 0;
    for (size_t i = 0; i < np; ++i) {
      if (used[i]) continue;
      used[i] = 1;
      if (i < from || !candidate[i]) continue;
      uint64_t between = 0;
      for (size_t j = i + 1; j < np && j <= i + kPairWindow; ++j) {
        if (used[j]) continue;
        if (candidate[j] && !(touches[j] & between) && dense_tc_pair_masks_ok(phys[i], phys[j])) {
          used[j] = 1;
          ++made;
          break;
        }
        between |= touches[j];
      }
    }
    return made;
  }

  // Hill climbing over swaps of two `movable` qubits' positions (moves that
  // keep the count are taken too), `steps` tries per climb, from `layout`
  // and from `restarts` - 1 shuffles of it; `layout` becomes the best found.
  // Returns its pair count.
  size_t climb(const std::vector<uint32_t>& movable, int steps, int restarts, std::mt19937& rng,
               std::vector<uint32_t>& layout) const {
    size_t best = pairs(layout);
    if (movable.size() < 2) return best;
    std::vector<uint32_t> best_layout = layout;
    for (int r = 0; r < restarts; ++r) {
      std::vector<uint32_t> trial = layout;
      if (r > 0) {
        std::vector<uint32_t> pos;
        for (uint32_t q : movable) pos.push_back(trial[q]);
        std::shuffle(pos.begin(), pos.end(), rng);
        for (size_t k = 0; k < movable.size(); ++k) trial[movable[k]] = pos[k];
      }
      size_t cur = pairs(trial);
      for (int s = 0; s < steps; ++s) {
        const uint32_t a = movable[rng() % movable.size()], b = movable[rng() % movable.size()];
        if (a == b) continue;
        std::swap(trial[a], trial[b]);
        const size_t c = pairs(trial);
        if (c >= cur)
          cur = c;
        else
          std::swap(trial[a], trial[b]);
      }
      if (cur > best) {
        best = cur;
        best_layout = trial;
      }
    }
    layout = best_layout;
    return best;
  }
};

// From |0...0> a run may take any layout for free; plain tensor-core plans
// from |0...0> (fusion 5-6) place their qubits as follows. Bits 1-3 keep
// the planner's choice (they set a single tensor-core pass's variant and
// cost).
//
// - The top bits: a qubit that no pass has touched yet becomes a control of
//   value 0 in the zero-start passes, so they move only the amplitudes
//   where it is 0. The kZeroStartTop qubits touched last are idle in the
//   heaviest of those passes; on the top bits below min(n, 32) they leave
//   them contiguous runs of the state.
// - Bit 0 (and bit 1) inside a DRAM sector saves nothing as a zero control,
//   so bit 0 takes a qubit touched early: the first touched, or with pair
//   passes the one among the kBitZeroTries touched first with which the
//   most passes pair.
// - With pair passes the bits above 3 (but the top ones) only decide which
//   passes may pair (their warps' accesses stay coalesced): hill climbing
//   over their permutations pairs more passes.
//
// On the 30-qubit grid circuit at fusion 6: 4.3 -> 3.3 ms of zero-start
// passes (the last two qubits touched on bits 28-29, a quarter of the
// state in four of them) and 9-11 pairs instead of 6. Returns whether
// `layout` changed.
constexpr size_t kZeroStartTop = 2;

bool zero_start_layout(const std::vector<PlannedPass>& passes, uint32_t n, bool pairs, bool thorough,
                       std::vector<uint32_t>& layout) {
  const size_t prefix = zero_prefix(passes, n);
  if (prefix == 0) return false;
  const std::vector<uint32_t> given = layout;
  std::vector<size_t> first(n, passes.size());  // first pass touching each logical qubit
  for (size_t i = passes.size(); i-- > 0;)
    for (uint64_t m = pass_qubits(passes[i]); m; m &= m - 1) first[__builtin_ctzll(m)] = i;
  const uint32_t top = std::min<uint32_t>(n, 32);
  std::vector<uint32_t> at(n);  // physical -> logical
  auto place = [&](uint32_t q, uint32_t p) {
    for (uint32_t x = 0; x < n; ++x) at[layout[x]] = x;
    const uint32_t other = at[p];
    std::swap(layout[q], layout[other]);
  };
  // The top bits (bit 0's qubit among the candidates: a qubit touched late
  // gains nothing there).
  std::vector<uint32_t> late;
  for (uint32_t q = 0; q < n; ++q)
    if ((layout[q] == 0 || (layout[q] >= 4 && layout[q] < top)) && first[q] > 0) late.push_back(q);
  std::stable_sort(late.begin(), late.end(), [&](uint32_t a, uint32_t b) { return first[a] > first[b]; });
  if (late.size() > kZeroStartTop) late.resize(kZeroStartTop);
  uint64_t fixed = 0;
  for (size_t k = 0; k < late.size(); ++k) {
    place(late[k], top - 1 - uint32_t(k));
    fixed |= uint64_t(1) << late[k];
  }
  // Bit 0: candidates touched early, on the bits that may move.
  uint32_t q0 = 0;
  while (layout[q0] != 0) ++q0;
  std::vector<uint32_t> early;
  for (uint32_t q = 0; q < n; ++q)
    if (layout[q] >= 4 && layout[q] < top && !((fixed >> q) & 1) && first[q] < first[q0]) early.push_back(q);
  std::stable_sort(early.begin(), early.end(), [&](uint32_t a, uint32_t b) { return first[a] < first[b]; });
  auto movable_of = [&](const std::vector<uint32_t>& l) {
    std::vector<uint32_t> mv;
    for (uint32_t q = 0; q < n; ++q)
      if (l[q] >= 4 && l[q] < top && !((fixed >> q) & 1)) mv.push_back(q);
    return mv;
  };
  std::mt19937 rng(2024);
  if (!pairs) {
    if (!early.empty()) std::swap(layout[q0], layout[early[0]]);
    return layout != given;
  }
  const PairSearch search(passes, n);
  if (search.count < 2) {
    if (!early.empty()) std::swap(layout[q0], layout[early[0]]);
    return layout != given;
  }
  // Bit 0 by a short climb per candidate (on host threads, each seeded by
  // its candidate: the result does not depend on the thread count), then
  // the full climb.
  const size_t tries = std::min<size_t>(early.size(), thorough ? 24 : 8);
  std::vector<std::vector<uint32_t>> found(tries, layout);
  std::vector<size_t> made(tries, 0);
  parallel_for(tries, [&](size_t k) {
    std::mt19937 r(uint32_t(2024 + k));
    std::swap(found[k][q0], found[k][early[k]]);
    made[k] = search.climb(movable_of(found[k]), 128, thorough ? 2 : 1, r, found[k]);
  });
  size_t pick = tries;
  for (size_t k = 0; k < tries; ++k)
    if (pick == tries || made[k] > made[pick]) pick = k;
  if (pick < tries) layout = found[pick];
  search.climb(movable_of(layout), thorough ? 1024 : 256, thorough ? 4 : 2, rng, layout);
  return layout != given;
}

}  // namespace

Program build_program(const Target& t, const std::vector<HOp>& ops, const qvdg_options& opt,
                      FusionSearch search, bool from_zero, std::vector<HOp>* fused) {
  Program prog;
  prog.target = t;
  prog.gates = ops.size();
  const size_t max_fused = std::max<uint32_t>(opt.max_fused_qubits, 1);
  // Tensor-core plain passes, singly or (TENSOR_PAIRS) two fused 6-qubit
  // gates per pass.
  const bool tensor_math = opt.math == QVDG_MATH_TENSOR || opt.math == QVDG_MATH_TENSOR_PAIRS;
  const bool pairs = !opt.staged && opt.math == QVDG_MATH_TENSOR_PAIRS && t.bits == 32;
  prog.cfg = stage_config(t, opt.tile_qubits, opt.staged && tensor_math);
  prog.cfg.plain_tensor = !opt.staged && tensor_math && t.bits == 32;
  std::vector<PlannedPass> passes;
  // Tensor-core plain passes' bf16 matrices (by pass; empty for the others).
  std::vector<PlainTcBlob> blobs;
  if (opt.staged) {
    passes = plan_stages(ops, t.layout, t.n, prog.cfg, max_fused);
  } else {
    // One pass per fused op (src/simulator.rs:136-143). With the gates math,
    // an eligible group is applied member by member in registers instead of
    // as its product matrix.
    // The groups' product matrices are independent: built on host threads.
    const bool gates = opt.math == QVDG_MATH_GATES;
    // Tensor-core plain plans of 5-6 qubit groups search their fusion: the
    // reference's greedy one, seed-lookahead variants and beam searches over
    // the seeds, each scored by its passes (a pass with targets on index
    // bits 1-3 counting as the 1.2-2.1 clean passes it takes on the
    // tensor-core kernels, and from |0...0> by the share of the state it
    // moves); 45 passes instead of 55 on the 30-qubit grid circuit at fusion
    // 6 (at fusion 4 the searches would add passes). Other plain plans keep
    // the reference's greedy fusion.
    const FusionInput fin = fusion_input(ops, [](const HOp&) { return true; });
    std::vector<FusedGroup> groups = fuse_groups_lookahead(fin, max_fused, 0);
    if (tensor_math && max_fused >= 5 && t.n >= 13) {
      // Candidate fusions and, for each, the three qubits to place on
      // physical bits 1-3 (a relabel that costs nothing on a |0...0> state
      // and one swap pass otherwise): the pair with the lowest estimated
      // cost, a pass with k targets on bits 1-3 counting as 1, 1.2, 1.45 or
      // 2.1 clean passes.
      // Fusions: the lookahead ones and the beam searches' (the widest
      // first, each on its own thread). At 30 qubits (depth-20 grid
      // circuit, fusion 6) the narrow beams take 50 passes to 47, the wide
      // ones to 45; at 32 qubits 52 to 50 and 47.
      struct BeamConfig {
        size_t lookahead, width;
      };
      std::vector<BeamConfig> beams;
      if (search == FusionSearch::Thorough) {
        beams = {{24, 32}, {16, 32}, {12, 32}, {8, 32}, {6, 32}};
        if (ops.size() <= 2000) beams.insert(beams.begin(), {24, 64});  // its time grows with the groups
      }
      if (search != FusionSearch::Lookahead)
        for (size_t l : {16, 6}) beams.push_back({l, 8});
      // Each search in up to two families: the fusion as the reference
      // orders ops, and, where some qubit meets two diagonal ops in a row
      // (QFT's controlled phases), with diagonal ops free to commute
      // (45 instead of 68 passes for the 30-qubit QFT at fusion 6).
      FusionInput fin_c = fin;
      fin_c.commute = true;
      std::vector<const FusionInput*> families = {&fin};
      if (diagonal_runs(fin)) families.push_back(&fin_c);
      const size_t nbeam = beams.size(), nlook = 9, per = nbeam + nlook;
      std::vector<std::vector<std::vector<FusedGroup>>> found(per * families.size());
      parallel_for(found.size(), [&](size_t t) {
        const size_t j = t % per;
        const FusionInput& in = *families[t / per];
        if (j < nbeam) {
          found[t] = fuse_groups_beam(in, max_fused, beams[j].lookahead, beams[j].width);
        } else {
          const size_t i = nlook - 1 - (j - nbeam);  // the longest lookaheads first
          found[t].push_back(i == 0 && t < per ? groups : fuse_groups_lookahead(in, max_fused, i));
        }
      });
      // Candidates in a fixed order: per family, lookahead 0-8, then the
      // beams' results.
      std::vector<std::vector<FusedGroup>> cand;
      for (size_t f = 0; f < families.size(); ++f) {
        for (size_t i = 0; i < nlook; ++i) cand.push_back(std::move(found[f * per + nbeam + nlook - 1 - i][0]));
        for (size_t j = 0; j < nbeam; ++j)
          for (auto& g : found[f * per + j]) cand.push_back(std::move(g));
      }
      std::vector<double> cost(cand.size());
      std::vector<uint64_t> low_set(cand.size());
      std::vector<uint32_t> at(t.n);  // physical -> logical
      for (uint32_t q = 0; q < t.n; ++q) at[t.layout[q]] = q;
      const uint64_t now = (uint64_t(1) << at[1]) | (uint64_t(1) << at[2]) | (uint64_t(1) << at[3]);
      // From |0...0> the passes before every qubit has been touched move
      // 2^(touched - n) of the state (zero-start passes; at least 2^13
      // amplitudes, plus a launch's worth): each pass's cost is scaled by
      // that share. At 30 qubits two 45-pass fusions of the grid circuit
      // spend 11 and 7 passes that way.
      const uint64_t every = t.n >= 64 ? ~uint64_t(0) : (uint64_t(1) << t.n) - 1;
      auto shares = [&](const std::vector<uint64_t>& gm) {
        std::vector<double> f(gm.size(), 1.0);
        uint64_t touched = 0;
        for (size_t k = 0; from_zero && k < gm.size(); ++k) {
          touched |= gm[k];
          if (touched == every) break;
          f[k] = std::ldexp(1.0, std::max(__builtin_popcountll(touched), 13) - int(t.n)) + 0.005;
        }
        return f;
      };
      auto weight = [](int low) { return low == 0 ? 1.0 : (low == 1 ? 1.2 : (low == 2 ? 1.45 : 2.1)); };
      parallel_for(cand.size(), [&](size_t i) {
        std::vector<uint64_t> gm;
        for (const FusedGroup& g : cand[i]) {
          uint64_t m = 0;
          for (uint32_t q : g.qubits) m |= uint64_t(1) << q;
          gm.push_back(m);
        }
        const std::vector<double> f = shares(gm);
        auto eval = [&](uint64_t s) {
          double c = 0.0;
          for (size_t k = 0; k < gm.size(); ++k) c += weight(__builtin_popcountll(gm[k] & s)) * f[k];
          return c;
        };
        // Triples among the 12 qubits in the fewest groups (the cost grows
        // with every group a chosen qubit is in).
        std::vector<uint32_t> by_use(t.n);
        std::vector<int> use(t.n, 0);
        for (uint64_t m : gm)
          for (uint32_t q = 0; q < t.n; ++q) use[q] += int((m >> q) & 1);
        for (uint32_t q = 0; q < t.n; ++q) by_use[q] = q;
        std::stable_sort(by_use.begin(), by_use.end(), [&](uint32_t x, uint32_t y) { return use[x] < use[y]; });
        const uint32_t pool = std::min<uint32_t>(t.n, 12);
        double best = eval(now);
        uint64_t best_set = now;
        for (uint32_t a = 0; a < pool; ++a)
          for (uint32_t b = a + 1; b < pool; ++b)
            for (uint32_t c = b + 1; c < pool; ++c) {
              const uint64_t s =
                  (uint64_t(1) << by_use[a]) | (uint64_t(1) << by_use[b]) | (uint64_t(1) << by_use[c]);
              const double v = eval(s);
              if (v < best - 1e-9) {
                best = v;
                best_set = s;
              }
            }
        cost[i] = best;
        low_set[i] = best_set;
      }, cand.size() >= 8 ? 0u : 1u);
      size_t pick = 0;
      for (size_t i = 1; i < cand.size(); ++i)
        if (cost[i] < cost[pick] - 1e-9) pick = i;
      // Relabel only where it saves at least 1.5 passes (it costs one when
      // the state is not |0...0>), or any saving for a one-shot run on
      // |0...0>, where it is free.
      auto eval_now = [&](const std::vector<FusedGroup>& gs) {
        std::vector<uint64_t> gm;
        for (const FusedGroup& g : gs) {
          uint64_t m = 0;
          for (uint32_t q : g.qubits) m |= uint64_t(1) << q;
          gm.push_back(m);
        }
        const std::vector<double> f = shares(gm);
        double c = 0.0;
        for (size_t k = 0; k < gm.size(); ++k) c += weight(__builtin_popcountll(gm[k] & now)) * f[k];
        return c;
      };
      size_t keep = 0;
      double keep_cost = eval_now(cand[0]);
      for (size_t i = 1; i < cand.size(); ++i) {
        const double c = eval_now(cand[i]);
        if (c < keep_cost - 1e-9) {
          keep = i;
          keep_cost = c;
        }
      }
      if (cost[pick] > keep_cost - (search == FusionSearch::Thorough || !from_zero ? 1.5 : 1e-9)) {
        pick = keep;
        low_set[pick] = now;
      }
      groups = std::move(cand[pick]);
      if (low_set[pick] != now) {
        // The chosen qubits onto bits 1-3 (those already there stay).
        std::vector<uint32_t> layout = t.layout;
        std::vector<uint32_t> phys_of_free;
        std::vector<uint32_t> incoming;
        for (uint32_t q = 0; q < t.n; ++q)
          if (((low_set[pick] >> q) & 1) && !(layout[q] >= 1 && layout[q] <= 3)) incoming.push_back(q);
        for (uint32_t p = 1; p <= 3; ++p)
          if (!((low_set[pick] >> at[p]) & 1)) phys_of_free.push_back(p);
        for (size_t k = 0; k < incoming.size(); ++k) {
          const uint32_t q = incoming[k], p = phys_of_free[k], out = at[p];
          std::swap(layout[q], layout[out]);
        }
        prog.run_layout = layout;
      }
    }
    passes.resize(groups.size());
    std::vector<size_t> products;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      const FusedGroup& g = groups[gi];
      PlannedPass& p = passes[gi];
      p.staged = false;
      if (gates) {
        std::vector<HOp> members;
        for (size_t i : g.members) members.push_back(ops[i]);
        if (block_pass_ok(t, members, g.qubits)) {
          p.block = true;
          p.block_qubits = g.qubits;
          p.ops = std::move(members);
          continue;
        }
      }
      p.ops.resize(1);
      products.push_back(gi);
    }
    // The products, then (on the layout the passes run with) the
    // tensor-core passes' bf16 matrices, on host threads.
    const bool wide = max_fused >= 5 && products.size() >= 8;
    parallel_for(products.size(), [&](size_t j) { passes[products[j]].ops[0] = fuse_group(ops, groups[products[j]]); },
                 wide ? 0u : 1u);
    if (prog.cfg.plain_tensor && max_fused >= 5 && from_zero && t.n >= 14) {
      std::vector<uint32_t> layout = prog.run_layout.empty() ? t.layout : prog.run_layout;
      if (zero_start_layout(passes, t.n, pairs, search == FusionSearch::Thorough, layout)) prog.run_layout = layout;
    }
    Target rt = t;
    if (!prog.run_layout.empty()) rt.layout = prog.run_layout;
    blobs.resize(passes.size());
    parallel_for(products.size(), [&](size_t j) {
      PlannedPass& p = passes[products[j]];
      if (plain_tc_eligible(rt, p, prog.cfg)) blobs[products[j]] = plain_tc_blob(rt, p.ops[0]);
    }, wide ? 0u : 1u);
  }
  // Passes are lowered on the layout they run with.
  Target run_target = t;
  if (!prog.run_layout.empty()) run_target.layout = prog.run_layout;
  const Target& tt = run_target;
  blobs.resize(passes.size());
  size_t tc_bytes = 0;
  for (size_t i = 0; i < passes.size(); ++i) {
    if (blobs[i].blob.empty() && plain_tc_eligible(tt, passes[i], prog.cfg))
      blobs[i] = plain_tc_blob(tt, passes[i].ops[0]);
    tc_bytes += blobs[i].blob.size() + 16;
  }
  prog.upload.tc.reserve(tc_bytes);
  const double state_bytes = double(uint64_t(t.bits == 32 ? 8 : 16) << t.n);
  // Passes that may share a pass with the next one: after the zero-start
  // prefix of a run from |0...0> (those passes keep their own variants).
  size_t pair_from = passes.size();
  if (pairs) pair_from = from_zero ? zero_prefix(passes, t.n) : 0;
  // Pairing: each pass after the zero-start prefix takes as its partner the
  // first of the next few passes that pairs with it (dense_tc_pair_ok) and
  // shares no qubit with any pass between them, moved up next to it (the
  // passes it jumps commute with it). `order` is the execution order,
  // `pair_next[k]` marks order[k] pairing with order[k + 1].
  std::vector<size_t> order;
  std::vector<char> pair_next;
  {
    auto eligible = [&](size_t i) {
      const PlannedPass& q = passes[i];
      return !q.staged && !q.block && q.ops.size() == 1 && q.ops[0].controls.empty() && !blobs[i].blob.empty() &&
             q.ops[0].targets.size() == 6;
    };
    std::vector<char> used(passes.size(), 0);
    for (size_t i = 0; i < passes.size(); ++i) {
      if (used[i]) continue;
      used[i] = 1;
      order.push_back(i);
      pair_next.push_back(0);
      if (!pairs || i < pair_from || !eligible(i)) continue;
      uint64_t between = 0;
      for (size_t j = i + 1; j < passes.size() && j <= i + kPairWindow; ++j) {
        if (used[j]) continue;
        if (eligible(j) && !(pass_qubits(passes[j]) & between) &&
            dense_tc_pair_ok(tt.n, tt.bits, blobs[i].targets, blobs[j].targets)) {
          used[j] = 1;
          pair_next.back() = 1;
          order.push_back(j);
          pair_next.push_back(0);
          break;
        }
        between |= pass_qubits(passes[j]);
      }
    }
  }
  if (fused) {
    if (opt.staged) throw Error(QVDG_ERR_INVALID, "fused ops exist for plain plans only");
    for (size_t i : order) fused->insert(fused->end(), passes[i].ops.begin(), passes[i].ops.end());
  }
  for (size_t k = 0; k < order.size(); ++k) {
    const size_t pi = order[k];
    const PlannedPass& p = passes[pi];
    if (pair_next[k]) {
      // Two fused 6-qubit gates in one pass: both blobs in the upload, the
      // pass described by its first gate and the pair geometry.
      const size_t pj = order[++k];
      LoweredPass lp = lower_pass(tt, p, prog.cfg, prog.upload, &blobs[pi]);
      blob_align(prog.upload.tc);
      const size_t off2 = prog.upload.tc.size();
      prog.upload.tc.insert(prog.upload.tc.end(), blobs[pj].blob.begin(), blobs[pj].blob.end());
      lp.pair = std::make_shared<const DenseTcPairGeom>(
          dense_tc_pair_geom(tt.n, lp.plain.targets, blobs[pj].targets, lp.plain.tc_offset, off2));
      prog.passes.push_back(std::move(lp));
      prog.features.resize(prog.features.size() + kPassFeatures);
      float* f = prog.features.data() + prog.features.size() - kPassFeatures;
      pass_features(tt, p, prog.passes.back(), prog.upload, f);
      pair_features(tt, passes[pj], f);
      prog.kernels += 2;
      prog.pass_bytes.push_back(2.0 * state_bytes);
      prog.bytes += 2.0 * state_bytes;
      continue;
    }
    prog.passes.push_back(lower_pass(tt, p, prog.cfg, prog.upload, blobs[pi].blob.empty() ? nullptr : &blobs[pi]));
    prog.features.resize(prog.features.size() + kPassFeatures);
    pass_features(tt, p, prog.passes.back(), prog.upload, prog.features.data() + prog.features.size() - kPassFeatures);
    prog.kernels += p.block ? 1 : p.ops.size();
    double b = 2.0 * state_bytes;
    if (p.staged)
      ++prog.stages;
    else if (!p.block)
      b /= double(uint64_t(1) << p.ops[0].controls.size());
    prog.pass_bytes.push_back(b);
    prog.bytes += b;
  }
  // Zero-start passes: each plain pass of the prefix in which some qubit
  // is still untouched, with those qubits as controls of value 0 (the
  // amplitudes they would select are zero before the pass and after it).
  // On the 30-qubit grid circuit the first passes then move a few MB each
  // instead of 17 GB.
  // Only programs meant to run from |0...0> get them.
  uint64_t support = 0;  // logical qubits touched so far
  const uint64_t every = t.n >= 64 ? ~uint64_t(0) : (uint64_t(1) << t.n) - 1;
  for (const PlannedPass& p : passes) {
    if (!from_zero || p.staged || p.block || p.ops.size() != 1) break;
    for (uint32_t q : p.ops[0].targets) support |= uint64_t(1) << q;
    for (auto& c : p.ops[0].controls) support |= uint64_t(1) << c.first;
    if (support == every) break;
    // The untouched qubits, lowest physical bit first. A tensor-core pass
    // keeps at least 2^13 amplitudes selected, so that it stays on the
    // tensor cores and gives the full pass's results exactly: the lowest
    // untouched qubits stay free (contiguous accesses).
    std::vector<uint32_t> idle;
    for (uint32_t q = 0; q < t.n; ++q)
      if (!((support >> q) & 1)) idle.push_back(q);
    std::sort(idle.begin(), idle.end(), [&](uint32_t x, uint32_t y) { return tt.layout[x] < tt.layout[y]; });
    size_t skip = 0;
    if (plain_tc_eligible(tt, p, prog.cfg)) {
      const size_t cap = t.n - 13 - std::min<size_t>(t.n - 13, p.ops[0].controls.size());
      skip = idle.size() > cap ? idle.size() - cap : 0;
    }
    // Untouched qubits on the physical bits inside a 32-byte DRAM sector
    // (bits 0-1 of a complex64 state, bit 0 of a complex128 one) stay free
    // too: as controls they save no DRAM sectors and make every access
    // strided (measured at 30 qubits: a pass with bit 0 among its zero
    // controls took 2.0 ms for a quarter of the state).
    const uint32_t sector_bits = t.bits == 32 ? 2 : 1;
    size_t low = 0;
    while (low < idle.size() && tt.layout[idle[low]] < sector_bits) ++low;
    skip = std::max(skip, low);
    if (skip == idle.size()) {  // nothing to save
      prog.zero_passes.push_back(prog.passes[prog.zero_passes.size()]);
      prog.zero_pass_bytes.push_back(prog.pass_bytes[prog.zero_pass_bytes.size()]);
      continue;
    }
    PlannedPass v = p;
    for (size_t j = skip; j < idle.size(); ++j) v.ops[0].controls.push_back({idle[j], false});
    PlainTcBlob vb;
    const bool tc = plain_tc_eligible(tt, v, prog.cfg);
    if (tc) vb = plain_tc_blob(tt, v.ops[0]);
    prog.zero_passes.push_back(lower_pass(tt, v, prog.cfg, prog.upload, tc ? &vb : nullptr));
    prog.zero_pass_bytes.push_back(2.0 * state_bytes / double(uint64_t(1) << v.ops[0].controls.size()));
  }
  return prog;
}

DeviceUpload upload_program(StateImpl& s, const Program& p, DeviceScratch& dst) {
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  const StageUpload& up = p.upload;
  const size_t gate_bytes = up.gates.size() * sizeof(TileGate);
  const size_t mat_bytes = up.mats.size() * (p.target.bits == 32 ? 4 : 8);
  const size_t tc_bytes = up.tc.size();
  const size_t total = align(gate_bytes) + align(mat_bytes) + align(tc_bytes) + 256;
  char* h = static_cast<char*>(s.host.get(total));
  if (gate_bytes) std::memcpy(h, up.gates.data(), gate_bytes);
  char* hm = h + align(gate_bytes);
  if (p.target.bits == 32) {
    float* f = reinterpret_cast<float*>(hm);
    for (size_t i = 0; i < up.mats.size(); ++i) f[i] = float(up.mats[i]);
  } else if (mat_bytes) {
    std::memcpy(hm, up.mats.data(), mat_bytes);
  }
  if (tc_bytes) std::memcpy(hm + align(mat_bytes), up.tc.data(), tc_bytes);
  char* d = static_cast<char*>(dst.get(total));
  QVDG_CUDA(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, s.stream));
  DeviceUpload u;
  u.gates = reinterpret_cast<const TileGate*>(d);
  u.mats = d + align(gate_bytes);
  u.tc = reinterpret_cast<const uint8_t*>(d + align(gate_bytes) + align(mat_bytes));
  return u;
}

// Bring the state to the layout the program's passes use: free on a
// |0...0> state, otherwise swap passes of disjoint physical bit pairs.
static void relabel_to(StateImpl& s, const std::vector<uint32_t>& layout) {
  if (layout == s.layout) return;
  if (s.zero_state) {
    s.layout = layout;
    return;
  }
  while (s.layout != layout) {
    std::vector<std::pair<uint32_t, uint32_t>> pairs;
    uint64_t used = 0;
    for (uint32_t q = 0; q < s.n; ++q) {
      const uint32_t a = s.layout[q], b = layout[q];
      const uint64_t m = (uint64_t(1) << a) | (uint64_t(1) << b);
      if (a == b || (used & m)) continue;
      used |= m;
      pairs.push_back({a, b});
    }
    launch_swap_bits(s, pairs);
    for (auto& q : s.layout)
      for (auto& pr : pairs) {
        if (q == pr.first)
          q = pr.second;
        else if (q == pr.second)
          q = pr.first;
      }
  }
}

void run_program(StateImpl& s, const Program& p, const DeviceUpload& dev, qvdg_stats* stats) {
  const bool timing = s.record_passes;
  if (timing) {
    while (s.pass_events.size() < p.passes.size() + 1) {
      cudaEvent_t e;
      QVDG_CUDA(cudaEventCreate(&e));
      s.pass_events.push_back(e);
    }
  }
  QVDG_CUDA(cudaEventRecord(s.ev_start, s.stream));
  // From |0...0> the zero-start passes run where they exist.
  const size_t zero = s.zero_state ? p.zero_passes.size() : 0;
  auto pass = [&](size_t i) -> const LoweredPass& { return i < zero ? p.zero_passes[i] : p.passes[i]; };
  // The passes' layout (a relabel pass is timed with them).
  relabel_to(s, p.run_layout.empty() ? p.target.layout : p.run_layout);
  s.zero_state = false;
  for (size_t i = 0; i < p.passes.size(); ++i) {
    if (timing) QVDG_CUDA(cudaEventRecord(s.pass_events[i], s.stream));
    launch_pass(s, pass(i), dev);
  }
  if (timing) QVDG_CUDA(cudaEventRecord(s.pass_events[p.passes.size()], s.stream));
  QVDG_CUDA(cudaEventRecord(s.ev_stop, s.stream));
  QVDG_CUDA(cudaStreamSynchronize(s.stream));
  bool tensor = false;
  for (const LoweredPass& lp : p.passes)
    tensor = tensor || (lp.staged ? lp.geo.tensor == 1 : lp.plain.tensor);
  if (tensor) {
    int flag = 0;
    QVDG_CUDA(cudaMemcpy(&flag, s.status, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      QVDG_CUDA(cudaMemset(s.status, 0, sizeof(int)));
      throw Error(QVDG_ERR_TIMEOUT, "a tensor-core pass gave up waiting for its matrix products");
    }
  }
  float ms = 0.f;
  QVDG_CUDA(cudaEventElapsedTime(&ms, s.ev_start, s.ev_stop));
  if (timing) {
    s.pass_seconds.clear();
    s.pass_kinds.clear();
    for (size_t i = 0; i < p.passes.size(); ++i) {
      float t = 0.f;
      QVDG_CUDA(cudaEventElapsedTime(&t, s.pass_events[i], s.pass_events[i + 1]));
      s.pass_seconds.push_back(double(t) * 1e-3);
      const LoweredPass& lp = pass(i);
      int kind = lp.staged ? 1 : 0;
      if (!lp.staged && lp.plain.tensor)
        kind = lp.pair ? 5 : (dense_tc_staged(s.n, lp.plain.targets, lp.plain.controls.size()) ? 3 : 2);
      if (i < zero && p.zero_pass_bytes[i] < p.pass_bytes[i]) kind = 4;  // a zero-start pass
      s.pass_kinds.push_back(kind);
    }
    s.pass_bytes = p.pass_bytes;
    for (size_t i = 0; i < zero; ++i) s.pass_bytes[i] = p.zero_pass_bytes[i];
  }
  if (stats) {
    double bytes = p.bytes;
    for (size_t i = 0; i < zero; ++i) bytes += p.zero_pass_bytes[i] - p.pass_bytes[i];
    stats->kernels += p.kernels;
    stats->passes += p.passes.size();
    stats->stages += p.stages;
    stats->gate_seconds += ms * 1e-3;
    stats->bytes += bytes;
  }
}

}  // namespace qvdg
