// Host-side gate algebra and greedy fusion of the B200 engine.
//
// Matrix algebra follows src/matrix.rs:99-196 (index bit j = qubit j; `mul`
// skips exact zeros; `embed` and `controlled` keep the reference's bit
// order). Fusion follows src/fusion.rs:58-170: greedy and dependency-aware,
// growing a group first along gates that share a qubit with it, then with
// unrelated gates, up to `max_qubits`; groups of one op keep their controls.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <functional>
#include <vector>

namespace qvdg {

struct C {
  double re, im;
};
inline C operator*(C a, C b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline double norm2(C a) { return a.re * a.re + a.im * a.im; }

struct HMatrix {
  size_t dim = 0;
  std::vector<C> a;  // row-major

  HMatrix() = default;
  explicit HMatrix(size_t d) : dim(d), a(d * d, C{0.0, 0.0}) {}
  static HMatrix identity(size_t qubits);
  static HMatrix diagonal(const std::vector<C>& d);
  C& at(size_t r, size_t c) { return a[r * dim + c]; }
  const C& at(size_t r, size_t c) const { return a[r * dim + c]; }
  size_t qubits() const { return size_t(__builtin_ctzll(dim)); }
  bool is_diagonal() const;
  std::vector<C> diagonal_entries() const;
  HMatrix mul(const HMatrix& o) const;
  HMatrix embed(const std::vector<uint32_t>& gate_qubits, const std::vector<uint32_t>& qubits) const;
  HMatrix controlled(size_t controls, size_t state) const;
};

struct HOp {
  std::vector<uint32_t> targets;
  std::vector<std::pair<uint32_t, bool>> controls;
  HMatrix matrix;
  bool diagonal = false;  // cached matrix.is_diagonal()

  std::vector<uint32_t> qubits() const;
  size_t width() const { return targets.size() + controls.size(); }
  // The op as one matrix on [controls..., targets...] (src/fusion.rs:38-55).
  void full(std::vector<uint32_t>& qs, HMatrix& m) const;
};

// A fused group: its member ops (indices, program order) and their qubits
// (ascending).
struct FusedGroup {
  std::vector<size_t> members;
  std::vector<uint32_t> qubits;
};

// The groups of the greedy fusion below (src/fusion.rs:63-170).
std::vector<FusedGroup> fuse_groups(const std::vector<HOp>& ops, size_t max_qubits,
                                    const std::function<bool(const HOp&)>& fusable);

// The same greedy growth, but each group is seeded by whichever of the
// first unfused op and the next `lookahead` ready ones (no unfused earlier
// op shares a qubit with it) grows the largest group; 0 is the greedy
// fusion above.
std::vector<FusedGroup> fuse_groups_lookahead(const std::vector<HOp>& ops, size_t max_qubits,
                                              const std::function<bool(const HOp&)>& fusable, size_t lookahead);

// What the fusion reads of each op: its qubits as a bit mask and its width
// (SIZE_MAX where it may not be merged). Built once, shared by several
// fusions of the same ops.
struct FusionInput {
  std::vector<uint64_t> mask;
  std::vector<size_t> width;
  std::vector<uint8_t> diag;  // the op is diagonal
  bool any_empty = false;     // some op touches no qubit
  uint64_t all = 0;           // every qubit some op touches
  // Diagonal ops commute with each other: with `commute` a diagonal op may
  // join a group ahead of skipped diagonal ops on its qubits (only skipped
  // non-diagonal ones hold it back), and seed one.
  bool commute = false;
};
// Whether some qubit meets two diagonal ops with no other op between them
// (only then does commute change a fusion).
bool diagonal_runs(const FusionInput& in);
FusionInput fusion_input(const std::vector<HOp>& ops, const std::function<bool(const HOp&)>& fusable);
std::vector<FusedGroup> fuse_groups_lookahead(const FusionInput& in, size_t max_qubits, size_t lookahead);

// Beam search over the same growth: each step, every kept partial fusion
// forms its next group from each of its first lookahead + 1 ready seeds,
// and the `width` partial fusions that cover the most ops are kept (equal
// covered sets once). Returns the fusions that finish first, i.e. with the
// fewest groups the search found.
std::vector<std::vector<FusedGroup>> fuse_groups_beam(const FusionInput& in, size_t max_qubits, size_t lookahead,
                                                      size_t width);

// The group's ops as one op (the product matrix on its qubits; a group of one
// op is that op, controls kept).
HOp fuse_group(const std::vector<HOp>& ops, const FusedGroup& g);

// Greedy fusion; ops with !fusable(op) are never merged and block their qubits.
std::vector<HOp> fuse_where(const std::vector<HOp>& ops, size_t max_qubits,
                            const std::function<bool(const HOp&)>& fusable);
std::vector<HOp> fuse(const std::vector<HOp>& ops, size_t max_qubits);

// f(0) .. f(n - 1) on the calling thread and the process's pool of host
// threads (at most 16 in all; `threads` = 1 runs them here, in order); the
// first exception thrown is rethrown here. Calls may nest.
void parallel_for(size_t n, const std::function<void(size_t)>& f, unsigned threads = 0);

}  // namespace qvdg
