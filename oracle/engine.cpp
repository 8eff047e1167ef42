// CPU restatement of the qvd 0.1.18 state-vector engine.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE. Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline and reference legs load this library, and only
// as the checker or as the timed CPU baseline. The product (libqvdgpu.so)
// never links or calls it.
//
// The reference is Rust and cannot be built here (no toolchain), so this file
// restates its algorithms in C++17 with the same AVX2/FMA/BMI2 scheme:
//   naive oracle          src/reference.rs:8-44
//   matrices              src/matrix.rs:99-196
//   blocked layout        src/simd.rs:1-23, src/state.rs:17-22,120-124
//   kernels               src/kernels.rs:22-535
//   state vector          src/state.rs:37-268
//   measurement           src/measure.rs:13-174
//   fusion                src/fusion.rs:15-170
//   cache blocking        src/blocking.rs:32-302
//   apply_ops             src/simulator.rs:122-147
// Parallelism uses OpenMP where the reference uses rayon. Compile with
// -ffp-contract=off: the reference's scalar arithmetic is not contracted
// into FMAs, and the sampler's sums must round exactly as it does.

#include <immintrin.h>
#include <omp.h>
#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "qvdg.h"

namespace oracle {

// ---------------------------------------------------------------- complex
struct cx {
  double re, im;
};
static inline cx cmul(cx a, cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static inline void cadd_to(cx& a, cx b) {
  a.re += b.re;
  a.im += b.im;
}
static inline double norm_sqr(cx a) { return a.re * a.re + a.im * a.im; }

// ------------------------------------------------------------------ matrix
// src/matrix.rs:13-205: row-major 2^k x 2^k, index bit j = qubit j.
struct Matrix {
  size_t dim = 0;
  std::vector<cx> data;

  Matrix() = default;
  explicit Matrix(size_t d) : dim(d), data(d * d, cx{0.0, 0.0}) {}
  static Matrix identity(size_t qubits) {
    Matrix m(size_t(1) << qubits);
    for (size_t i = 0; i < m.dim; ++i) m.at(i, i) = {1.0, 0.0};
    return m;
  }
  static Matrix diagonal(const std::vector<cx>& entries) {
    Matrix m(entries.size());
    for (size_t i = 0; i < entries.size(); ++i) m.at(i, i) = entries[i];
    return m;
  }
  static Matrix from_interleaved(const double* v, size_t qubits) {
    Matrix m(size_t(1) << qubits);
    for (size_t i = 0; i < m.dim * m.dim; ++i) m.data[i] = {v[2 * i], v[2 * i + 1]};
    return m;
  }
  cx& at(size_t r, size_t c) { return data[r * dim + c]; }
  const cx& at(size_t r, size_t c) const { return data[r * dim + c]; }
  size_t qubits() const { return size_t(__builtin_ctzll(dim)); }

  bool is_diagonal() const {  // matrix.rs:99-101
    for (size_t r = 0; r < dim; ++r)
      for (size_t c = 0; c < dim; ++c)
        if (r != c && norm_sqr(at(r, c)) != 0.0) return false;
    return true;
  }
  std::vector<cx> diagonal_entries() const {
    std::vector<cx> d(dim);
    for (size_t i = 0; i < dim; ++i) d[i] = at(i, i);
    return d;
  }
  // matrix.rs:108-124: self * other, skipping exact zeros of self.
  Matrix mul(const Matrix& o) const {
    Matrix out(dim);
    for (size_t r = 0; r < dim; ++r)
      for (size_t k = 0; k < dim; ++k) {
        cx a = at(r, k);
        if (norm_sqr(a) == 0.0) continue;
        for (size_t c = 0; c < dim; ++c) cadd_to(out.at(r, c), cmul(a, o.at(k, c)));
      }
    return out;
  }
  // matrix.rs:139-176: embed a gate on gate_qubits into the list `qubits`.
  Matrix embed(const std::vector<size_t>& gate_qubits, const std::vector<size_t>& qubits) const {
    std::vector<size_t> position;
    for (size_t q : gate_qubits) {
      auto it = std::find(qubits.begin(), qubits.end(), q);
      if (it == qubits.end()) throw std::runtime_error("qubit missing from embedding");
      position.push_back(size_t(it - qubits.begin()));
    }
    size_t gate_mask = 0;
    for (size_t p : position) gate_mask |= size_t(1) << p;
    Matrix out(size_t(1) << qubits.size());
    auto local = [&](size_t index) {
      size_t l = 0;
      for (size_t j = 0; j < position.size(); ++j) l |= ((index >> position[j]) & 1) << j;
      return l;
    };
    for (size_t r = 0; r < out.dim; ++r)
      for (size_t c = 0; c < out.dim; ++c)
        if ((r & ~gate_mask) == (c & ~gate_mask)) out.at(r, c) = at(local(r), local(c));
    return out;
  }
  // matrix.rs:180-196: prepend `controls` control qubits in `state`.
  Matrix controlled(size_t controls, size_t state) const {
    size_t k = qubits();
    Matrix out = identity(controls + k);
    size_t mask = (size_t(1) << controls) - 1;
    for (size_t r = 0; r < out.dim; ++r)
      for (size_t c = 0; c < out.dim; ++c) {
        bool rc = (r & mask) == state, cc = (c & mask) == state;
        if (rc && cc)
          out.at(r, c) = at(r >> controls, c >> controls);
        else if (rc || cc)
          out.at(r, c) = {0.0, 0.0};
      }
    return out;
  }
};

// ---------------------------------------------------------------------- op
// src/fusion.rs:15-56.
struct Op {
  std::vector<size_t> targets;
  std::vector<std::pair<size_t, bool>> controls;
  Matrix matrix;

  std::vector<size_t> qubits() const {
    std::vector<size_t> q(targets);
    for (auto& c : controls) q.push_back(c.first);
    return q;
  }
  size_t width() const { return targets.size() + controls.size(); }
  // The op as a plain matrix on its controls followed by its targets.
  void full(std::vector<size_t>& qs, Matrix& m) const {
    if (controls.empty()) {
      qs = targets;
      m = matrix;
      return;
    }
    size_t state = 0;
    qs.clear();
    for (size_t i = 0; i < controls.size(); ++i) {
      state |= size_t(controls[i].second) << i;
      qs.push_back(controls[i].first);
    }
    for (size_t t : targets) qs.push_back(t);
    m = matrix.controlled(controls.size(), state);
  }
};

static Op op_from_abi(const qvdg_op& o) {
  Op op;
  for (uint32_t j = 0; j < o.num_targets; ++j) op.targets.push_back(o.targets[j]);
  for (uint32_t j = 0; j < o.num_controls; ++j)
    op.controls.push_back({o.controls[j], o.control_values ? o.control_values[j] != 0 : true});
  op.matrix = Matrix::from_interleaved(o.matrix, o.num_targets);
  return op;
}

// ------------------------------------------------------------------ fusion
// src/fusion.rs:63-170: greedy, dependency-aware fusion.
struct Group {
  size_t seed;
  std::vector<size_t> members;
  std::vector<size_t> qubits;

  template <class W>
  void grow(const std::vector<Op>& ops, std::vector<bool>& done, size_t max_qubits, bool connected_only,
            const W& width) {
    std::vector<size_t> blocked;
    auto contains = [](const std::vector<size_t>& v, size_t x) { return std::find(v.begin(), v.end(), x) != v.end(); };
    for (size_t i = seed + 1; i < ops.size(); ++i) {
      if (done[i]) continue;
      if (connected_only) {
        bool all_blocked = true;
        for (size_t q : qubits)
          if (!contains(blocked, q)) {
            all_blocked = false;
            break;
          }
        if (all_blocked) break;
      }
      std::vector<size_t> op_qubits = ops[i].qubits();
      bool touches_blocked = false;
      for (size_t q : op_qubits)
        if (contains(blocked, q)) touches_blocked = true;
      std::vector<size_t> fresh;
      for (size_t q : op_qubits)
        if (!contains(qubits, q)) fresh.push_back(q);
      bool connected = fresh.size() < op_qubits.size();
      bool fits = width(ops[i]) <= max_qubits && qubits.size() + fresh.size() <= max_qubits;
      if (!touches_blocked && fits && (connected || !connected_only)) {
        done[i] = true;
        members.push_back(i);
        for (size_t q : fresh) qubits.push_back(q);
      } else {
        for (size_t q : op_qubits)
          if (!contains(blocked, q)) blocked.push_back(q);
      }
    }
    std::sort(members.begin(), members.end());
  }
};

template <class F>
std::vector<Op> fuse_where(const std::vector<Op>& ops, size_t max_qubits, const F& fusable) {
  auto width = [&](const Op& op) { return fusable(op) ? op.width() : SIZE_MAX; };
  std::vector<bool> done(ops.size(), false);
  std::vector<Op> fused;
  for (size_t seed = 0; seed < ops.size(); ++seed) {
    if (done[seed]) continue;
    done[seed] = true;
    Group g{seed, {seed}, ops[seed].qubits()};
    if (width(ops[seed]) <= max_qubits) {
      g.grow(ops, done, max_qubits, true, width);
      g.grow(ops, done, max_qubits, false, width);
    }
    if (g.members.size() == 1) {
      fused.push_back(ops[seed]);
      continue;
    }
    std::sort(g.qubits.begin(), g.qubits.end());
    Matrix m = Matrix::identity(g.qubits.size());
    for (size_t i : g.members) {
      std::vector<size_t> oq;
      Matrix om;
      ops[i].full(oq, om);
      m = om.embed(oq, g.qubits).mul(m);
    }
    fused.push_back(Op{g.qubits, {}, m});
  }
  return fused;
}

std::vector<Op> fuse(const std::vector<Op>& ops, size_t max_qubits) {
  return fuse_where(ops, max_qubits, [](const Op&) { return true; });
}

// -------------------------------------------------------------- SIMD layer
// src/simd.rs: f32 -> 8 lanes (3 bits), f64 -> 4 lanes (2 bits); a block is
// LANES real parts then LANES imaginary parts (64 bytes).
template <class T>
struct Simd;

template <>
struct Simd<float> {
  static constexpr size_t LANES = 8;
  static constexpr size_t LANE_BITS = 3;
  using V = __m256;
  using Perm = __m256i;
  static V load(const float* p) { return _mm256_loadu_ps(p); }
  static void store(float* p, V v) { _mm256_storeu_ps(p, v); }
  static V zero() { return _mm256_setzero_ps(); }
  static V fma(V a, V b, V c) { return _mm256_fmadd_ps(a, b, c); }
  static V fnma(V a, V b, V c) { return _mm256_fnmadd_ps(a, b, c); }
  static V mul(V a, V b) { return _mm256_mul_ps(a, b); }
  static V add(V a, V b) { return _mm256_add_ps(a, b); }
  static V sub(V a, V b) { return _mm256_sub_ps(a, b); }
  static Perm xor_perm(size_t x) {
    int s = int(x);
    return _mm256_setr_epi32(s, 1 ^ s, 2 ^ s, 3 ^ s, 4 ^ s, 5 ^ s, 6 ^ s, 7 ^ s);
  }
  static V permute(V v, Perm p) { return _mm256_permutevar8x32_ps(v, p); }
};

template <>
struct Simd<double> {
  static constexpr size_t LANES = 4;
  static constexpr size_t LANE_BITS = 2;
  using V = __m256d;
  using Perm = __m256i;
  static V load(const double* p) { return _mm256_loadu_pd(p); }
  static void store(double* p, V v) { _mm256_storeu_pd(p, v); }
  static V zero() { return _mm256_setzero_pd(); }
  static V fma(V a, V b, V c) { return _mm256_fmadd_pd(a, b, c); }
  static V fnma(V a, V b, V c) { return _mm256_fnmadd_pd(a, b, c); }
  static V mul(V a, V b) { return _mm256_mul_pd(a, b); }
  static V add(V a, V b) { return _mm256_add_pd(a, b); }
  static V sub(V a, V b) { return _mm256_sub_pd(a, b); }
  static Perm xor_perm(size_t x) {
    auto s = [&](size_t lane) { return int((lane ^ x) * 2); };
    return _mm256_setr_epi32(s(0), s(0) + 1, s(1), s(1) + 1, s(2), s(2) + 1, s(3), s(3) + 1);
  }
  static V permute(V v, Perm p) { return _mm256_castps_pd(_mm256_permutevar8x32_ps(_mm256_castpd_ps(v), p)); }
};

// BMI2 pdep: deposit the low bits of value at the set bits of mask (kernels.rs:22-43).
static inline size_t deposit(size_t value, size_t mask) { return size_t(_pdep_u64(value, mask)); }

// Iterations per parallel task (kernels.rs:61-63).
static constexpr size_t TASK_ITERATIONS = size_t(1) << 11;

template <class Body>
static void for_ranges(size_t count, bool parallel, const Body& body) {
  if (!parallel || count <= TASK_ITERATIONS || omp_get_max_threads() == 1) {
    body(size_t(0), count);
    return;
  }
  long tasks = long((count + TASK_ITERATIONS - 1) / TASK_ITERATIONS);
#pragma omp parallel for schedule(dynamic, 1)
  for (long task = 0; task < tasks; ++task) {
    size_t start = size_t(task) * TASK_ITERATIONS;
    body(start, std::min(start + TASK_ITERATIONS, count));
  }
}

// ------------------------------------------------------------------ layout
// kernels.rs:78-156: targets split into block ("high") and lane ("low") bits.
struct Layout {
  std::vector<std::pair<size_t, unsigned>> high;  // (matrix bit, block bit), sorted by block bit
  std::vector<std::pair<size_t, unsigned>> low;   // (matrix bit, lane bit)
  std::vector<size_t> offsets;                    // block offset of each high combination
  size_t free_mask = 0;
  size_t control_value = 0;

  template <class T>
  static Layout make(const std::vector<size_t>& targets, const std::vector<std::pair<size_t, bool>>& controls,
                     unsigned region_bits) {
    const size_t lane_bits = Simd<T>::LANE_BITS;
    Layout l;
    for (size_t j = 0; j < targets.size(); ++j) {
      size_t q = targets[j];
      if (q < lane_bits)
        l.low.push_back({j, unsigned(q)});
      else
        l.high.push_back({j, unsigned(q - lane_bits)});
    }
    std::stable_sort(l.high.begin(), l.high.end(), [](auto& a, auto& b) { return a.second < b.second; });
    size_t high_mask = 0;
    for (auto& h : l.high) high_mask |= size_t(1) << h.second;
    for (size_t h = 0; h < (size_t(1) << l.high.size()); ++h) l.offsets.push_back(deposit(h, high_mask));
    size_t control_mask = 0;
    for (auto& c : controls) {
      if (c.first < lane_bits) throw std::runtime_error("low control qubits must be folded into the matrix");
      control_mask |= size_t(1) << (c.first - lane_bits);
      if (c.second) l.control_value |= size_t(1) << (c.first - lane_bits);
    }
    size_t region_mask = (size_t(1) << region_bits) - 1;
    if ((high_mask | control_mask) & ~region_mask) throw std::runtime_error("gate qubit outside the region");
    l.free_mask = region_mask & ~high_mask & ~control_mask;
    return l;
  }
  size_t matrix_index(size_t h, size_t lane) const {
    size_t index = 0;
    for (size_t m = 0; m < high.size(); ++m) index |= ((h >> m) & 1) << high[m].first;
    for (auto& lo : low) index |= ((lane >> lo.second) & 1) << lo.first;
    return index;
  }
  size_t low_lane_mask() const {
    size_t m = 0;
    for (auto& lo : low) m |= size_t(1) << lo.second;
    return m;
  }
  size_t iterations() const { return size_t(1) << __builtin_popcountll(free_mask); }
};

// ------------------------------------------------------------ dense plan
// kernels.rs:158-386.
template <class T>
struct DensePlan {
  using S = Simd<T>;
  Layout layout;
  size_t nh = 0, nt = 0;
  std::vector<typename S::Perm> perms;
  std::vector<T> coefficients;  // per (row, col, t): LANES re then LANES im

  DensePlan(const Matrix& matrix, const std::vector<size_t>& targets,
            const std::vector<std::pair<size_t, bool>>& controls, unsigned region_bits) {
    layout = Layout::make<T>(targets, controls, region_bits);
    nh = size_t(1) << layout.high.size();
    nt = size_t(1) << layout.low.size();
    size_t low_mask = layout.low_lane_mask();
    std::vector<size_t> spreads;
    for (size_t t = 0; t < nt; ++t) spreads.push_back(deposit(t, low_mask));
    for (size_t s : spreads) perms.push_back(S::xor_perm(s));
    for (size_t row = 0; row < nh; ++row)
      for (size_t col = 0; col < nh; ++col)
        for (size_t s : spreads) {
          for (size_t lane = 0; lane < S::LANES; ++lane)
            coefficients.push_back(T(matrix.at(layout.matrix_index(row, lane), layout.matrix_index(col, lane ^ s)).re));
          for (size_t lane = 0; lane < S::LANES; ++lane)
            coefficients.push_back(T(matrix.at(layout.matrix_index(row, lane), layout.matrix_index(col, lane ^ s)).im));
        }
  }

  template <size_t NH, size_t NT>
  void sweep(T* region, bool parallel) const {
    const size_t lanes = S::LANES;
    const size_t free = layout.free_mask, control_value = layout.control_value;
    size_t offsets[NH];
    for (size_t h = 0; h < NH; ++h) offsets[h] = layout.offsets[h] * 2 * lanes;
    typename S::Perm pm[NT];
    for (size_t t = 0; t < NT; ++t) pm[t] = perms[t];
    const T* coef = coefficients.data();
    for_ranges(layout.iterations(), parallel, [&](size_t start, size_t end) {
      size_t base = deposit(start, free) | control_value;
      for (size_t it = start; it < end; ++it) {
        T* block = region + base * 2 * lanes;
        typename S::V re[NH][NT], im[NH][NT];
        for (size_t h = 0; h < NH; ++h) {
          auto x = S::load(block + offsets[h]);
          auto y = S::load(block + offsets[h] + lanes);
          for (size_t t = 0; t < NT; ++t) {
            re[h][t] = t == 0 ? x : S::permute(x, pm[t]);
            im[h][t] = t == 0 ? y : S::permute(y, pm[t]);
          }
        }
        const size_t stride = NT * 2 * lanes;
        for (size_t row = 0; row < NH; ++row) {
          // Four accumulators per row; the FMA order per row is the one of
          // dense_row / dense_row_pair (col-major over (col, t)).
          auto rr = S::zero(), ir = S::zero(), ii = S::zero(), ri = S::zero();
          const T* c0 = coef + row * NH * stride;
          for (size_t col = 0; col < NH; ++col)
            for (size_t t = 0; t < NT; ++t) {
              size_t o = col * stride + t * 2 * lanes;
              auto w_re = S::load(c0 + o), w_im = S::load(c0 + o + lanes);
              rr = S::fma(w_re, re[col][t], rr);
              ir = S::fma(w_re, im[col][t], ir);
              ii = S::fma(w_im, im[col][t], ii);
              ri = S::fma(w_im, re[col][t], ri);
            }
          T* p = block + offsets[row];
          S::store(p, S::sub(rr, ii));
          S::store(p + lanes, S::add(ir, ri));
        }
        base = (((base | ~free) + 1) & free) | control_value;
      }
    });
  }

  void apply(T* region, bool parallel) const {
#define QVD_SHAPE(a, b) \
  if (nh == a && nt == b) return sweep<a, b>(region, parallel);
    QVD_SHAPE(1, 2) QVD_SHAPE(1, 4) QVD_SHAPE(1, 8) QVD_SHAPE(2, 1) QVD_SHAPE(2, 2) QVD_SHAPE(2, 4)
    QVD_SHAPE(2, 8) QVD_SHAPE(4, 1) QVD_SHAPE(4, 2) QVD_SHAPE(4, 4) QVD_SHAPE(4, 8) QVD_SHAPE(8, 1)
    QVD_SHAPE(8, 2) QVD_SHAPE(8, 4) QVD_SHAPE(8, 8) QVD_SHAPE(16, 1) QVD_SHAPE(16, 2) QVD_SHAPE(16, 4)
    QVD_SHAPE(32, 1) QVD_SHAPE(32, 2) QVD_SHAPE(64, 1)
#undef QVD_SHAPE
    throw std::runtime_error("unsupported dense gate shape");
  }
};

// --------------------------------------------------------- diagonal plan
// kernels.rs:388-473.
template <class T>
struct DiagonalPlan {
  using S = Simd<T>;
  Layout layout;
  size_t nh = 0;
  std::vector<T> factors;  // per high combination: LANES re then LANES im

  DiagonalPlan(const std::vector<cx>& entries, const std::vector<size_t>& targets,
               const std::vector<std::pair<size_t, bool>>& controls, unsigned region_bits) {
    layout = Layout::make<T>(targets, controls, region_bits);
    nh = size_t(1) << layout.high.size();
    for (size_t h = 0; h < nh; ++h) {
      for (size_t lane = 0; lane < S::LANES; ++lane) factors.push_back(T(entries[layout.matrix_index(h, lane)].re));
      for (size_t lane = 0; lane < S::LANES; ++lane) factors.push_back(T(entries[layout.matrix_index(h, lane)].im));
    }
  }

  void apply(T* region, bool parallel) const {
    const size_t lanes = S::LANES;
    const size_t free = layout.free_mask, control_value = layout.control_value;
    const T* fac = factors.data();
    const size_t nh_ = nh;
    std::vector<size_t> offsets(nh_);
    for (size_t h = 0; h < nh_; ++h) offsets[h] = layout.offsets[h] * 2 * lanes;
    const size_t* off = offsets.data();
    for_ranges(layout.iterations(), parallel, [&](size_t start, size_t end) {
      size_t base = deposit(start, free) | control_value;
      for (size_t it = start; it < end; ++it) {
        T* block = region + base * 2 * lanes;
        for (size_t h = 0; h < nh_; ++h) {
          const T* f = fac + h * 2 * lanes;
          auto f_re = S::load(f), f_im = S::load(f + lanes);
          T* p = block + off[h];
          auto re = S::load(p), im = S::load(p + lanes);
          auto out_re = S::fnma(f_im, im, S::mul(f_re, re));
          auto out_im = S::fma(f_im, re, S::mul(f_re, im));
          S::store(p, out_re);
          S::store(p + lanes, out_im);
        }
        base = (((base | ~free) + 1) & free) | control_value;
      }
    });
  }
};

static constexpr size_t MAX_GATE_QUBITS = 6;  // kernels.rs:476

// kernels.rs:478-535: fold lane controls into the matrix, pick dense or diagonal.
template <class T>
struct Plan {
  bool diagonal = false;
  std::vector<DensePlan<T>> dense;
  std::vector<DiagonalPlan<T>> diag;

  Plan(const Matrix& matrix, const std::vector<size_t>& qubits, const std::vector<std::pair<size_t, bool>>& controls,
       unsigned region_bits) {
    const size_t lane_bits = Simd<T>::LANE_BITS;
    std::vector<std::pair<size_t, bool>> low, high;
    for (auto& c : controls) (c.first < lane_bits ? low : high).push_back(c);
    Matrix m;
    std::vector<size_t> targets;
    if (low.empty()) {
      m = matrix;
      targets = qubits;
    } else {
      size_t state = 0;
      for (size_t i = 0; i < low.size(); ++i) {
        state |= size_t(low[i].second) << i;
        targets.push_back(low[i].first);
      }
      for (size_t q : qubits) targets.push_back(q);
      m = matrix.controlled(low.size(), state);
    }
    if (targets.size() > MAX_GATE_QUBITS)
      throw std::runtime_error("gates on more than 6 qubits (including lane controls) are not supported");
    if (m.is_diagonal()) {
      diagonal = true;
      diag.emplace_back(m.diagonal_entries(), targets, high, region_bits);
    } else {
      dense.emplace_back(m, targets, high, region_bits);
    }
  }
  void apply(T* region, bool parallel) const {
    if (diagonal)
      diag[0].apply(region, parallel);
    else
      dense[0].apply(region, parallel);
  }
};

// ------------------------------------------------------------ state vector
// src/state.rs + src/memory.rs (2 MiB-aligned, huge pages, parallel first touch).
template <class T>
struct StateVector {
  using S = Simd<T>;
  size_t num_qubits = 0;
  T* buffer = nullptr;
  size_t len = 0;  // reals in the buffer
  size_t mapped = 0;
  std::vector<size_t> layout;  // layout[logical] = physical

  explicit StateVector(size_t n) : num_qubits(n) {
    if (n >= 56) throw std::runtime_error("too many qubits");
    size_t amplitudes = std::max(size_t(1) << n, S::LANES);
    len = 2 * amplitudes;
    size_t bytes = len * sizeof(T);
    const size_t huge = size_t(2) << 20;
    mapped = (bytes + huge - 1) / huge * huge;
    void* p = mmap(nullptr, mapped + huge, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (p == MAP_FAILED) throw std::bad_alloc();
    uintptr_t aligned = (uintptr_t(p) + huge - 1) / huge * huge;
    raw_map = p;
    raw_len = mapped + huge;
    buffer = reinterpret_cast<T*>(aligned);
    madvise(buffer, mapped, MADV_HUGEPAGE);
    long pages = long(mapped / 4096);
#pragma omp parallel for schedule(static)
    for (long page = 0; page < pages; ++page) reinterpret_cast<volatile char*>(buffer)[size_t(page) * 4096] = 0;
    buffer[0] = T(1);
    for (size_t q = 0; q < n; ++q) layout.push_back(q);
  }
  ~StateVector() {
    if (raw_map) munmap(raw_map, raw_len);
  }
  StateVector(const StateVector&) = delete;
  StateVector& operator=(const StateVector&) = delete;

  void* raw_map = nullptr;
  size_t raw_len = 0;

  size_t size() const { return size_t(1) << num_qubits; }
  size_t blocks() const { return len / (2 * S::LANES); }
  unsigned block_bits() const { return unsigned(__builtin_ctzll(blocks())); }
  bool identity_layout() const {
    for (size_t q = 0; q < layout.size(); ++q)
      if (layout[q] != q) return false;
    return true;
  }
  size_t physical_index(size_t index) const {
    size_t p = 0;
    for (size_t q = 0; q < layout.size(); ++q) p |= ((index >> q) & 1) << layout[q];
    return p;
  }
  size_t logical_index(size_t index) const {
    size_t l = 0;
    for (size_t q = 0; q < layout.size(); ++q) l |= ((index >> layout[q]) & 1) << q;
    return l;
  }
  static void offsets(size_t physical, size_t& re, size_t& im) {
    re = (physical >> S::LANE_BITS) * 2 * S::LANES + (physical & (S::LANES - 1));
    im = re + S::LANES;
  }
  void set_all(const double* amplitudes) {  // from_amplitudes, state.rs:52-63
    buffer[0] = T(0);
    long count = long(size());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < count; ++i) {
      size_t re, im;
      offsets(physical_index(size_t(i)), re, im);
      buffer[re] = T(amplitudes[2 * i]);
      buffer[im] = T(amplitudes[2 * i + 1]);
    }
  }
  void get_all(double* out) const {  // to_vec, state.rs:146-159
    long count = long(size());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < count; ++i) {
      size_t re, im;
      offsets(physical_index(size_t(i)), re, im);
      out[2 * i] = double(buffer[re]);
      out[2 * i + 1] = double(buffer[im]);
    }
  }
  double norm_sqr() const {  // state.rs:172-177 (chunk sums of 2^14 reals)
    const size_t chunk = size_t(1) << 14;
    long chunks = long((len + chunk - 1) / chunk);
    std::vector<double> sums(size_t(chunks), 0.0);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < chunks; ++c) {
      double s = 0.0;
      size_t end = std::min(len, size_t(c + 1) * chunk);
      for (size_t i = size_t(c) * chunk; i < end; ++i) s += double(buffer[i]) * double(buffer[i]);
      sums[size_t(c)] = s;
    }
    double total = 0.0;
    for (double s : sums) total += s;
    return total;
  }
  void apply(const Matrix& matrix, const std::vector<size_t>& qubits,
             const std::vector<std::pair<size_t, bool>>& controls) {  // state.rs:181-198
    for (size_t q : qubits)
      if (q >= num_qubits) throw std::runtime_error("qubit out of range");
    for (auto& c : controls)
      if (c.first >= num_qubits) throw std::runtime_error("qubit out of range");
    if (qubits.empty()) return;
    std::vector<size_t> targets;
    for (size_t q : qubits) targets.push_back(layout[q]);
    std::vector<std::pair<size_t, bool>> pc;
    for (auto& c : controls) pc.push_back({layout[c.first], c.second});
    Plan<T> plan(matrix, targets, pc, block_bits());
    plan.apply(buffer, true);
  }
  void scale(double factor) {
    long count = long(len);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < count; ++i) buffer[i] = T(double(buffer[i]) * factor);
  }
  // state.rs:212-268: swap pairs of block bits in one pass and relabel.
  void swap_physical(const std::vector<std::pair<size_t, size_t>>& pairs) {
    if (pairs.empty()) return;
    const size_t lane_bits = S::LANE_BITS;
    size_t seen = 0;
    std::vector<std::pair<size_t, size_t>> shifts;
    for (auto& p : pairs) {
      if (p.first < lane_bits || p.second < lane_bits || p.first == p.second)
        throw std::runtime_error("swap of a lane qubit");
      size_t ba = size_t(1) << (p.first - lane_bits), bb = size_t(1) << (p.second - lane_bits);
      if (seen & (ba | bb)) throw std::runtime_error("qubit swapped twice in one pass");
      seen |= ba | bb;
      shifts.push_back({p.first - lane_bits, p.second - lane_bits});
    }
    const size_t block_len = 2 * S::LANES;
    long nblocks = long(blocks());
#pragma omp parallel for schedule(static)
    for (long ii = 0; ii < nblocks; ++ii) {
      size_t i = size_t(ii);
      size_t j = i & ~seen;
      for (auto& s : shifts) j |= ((i >> s.first) & 1) << s.second | ((i >> s.second) & 1) << s.first;
      if (i < j) std::swap_ranges(buffer + i * block_len, buffer + (i + 1) * block_len, buffer + j * block_len);
    }
    for (auto& q : layout)
      for (auto& p : pairs) {
        if (q == p.first)
          q = p.second;
        else if (q == p.second)
          q = p.first;
      }
  }

  // ---- measurement, src/measure.rs
  static constexpr size_t CHUNK_BLOCKS = size_t(1) << 12;  // measure.rs:13

  double probability_one(size_t qubit) const {  // measure.rs:43-65
    size_t phys = layout[qubit];
    const size_t lanes = S::LANES;
    const size_t chunk_len = 2 * lanes * CHUNK_BLOCKS;
    long chunks = long((len + chunk_len - 1) / chunk_len);
    std::vector<double> sums(size_t(chunks), 0.0);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < chunks; ++c) {
      double s = 0.0;
      size_t nb = std::min(CHUNK_BLOCKS, (len - size_t(c) * chunk_len) / (2 * lanes));
      for (size_t b = 0; b < nb; ++b) {
        const T* block = buffer + size_t(c) * chunk_len + b * 2 * lanes;
        size_t index = (size_t(c) * CHUNK_BLOCKS + b) << S::LANE_BITS;
        double bs = 0.0;
        for (size_t l = 0; l < lanes; ++l) {
          double re = double(block[l]), im = double(block[l + lanes]);
          double p = re * re + im * im;
          if (((index | l) >> phys) & 1) bs += p;
        }
        s += bs;
      }
      sums[size_t(c)] = s;
    }
    double total = 0.0;
    for (double s : sums) total += s;
    return total;
  }

  bool measure(size_t qubit, double uniform) {  // measure.rs:68-80
    double p1 = std::min(std::max(probability_one(qubit), 0.0), 1.0);
    bool outcome = uniform < p1;
    double p = outcome ? p1 : 1.0 - p1;
    cx keep{1.0 / std::sqrt(p), 0.0}, zero{0.0, 0.0};
    std::vector<cx> entries = outcome ? std::vector<cx>{zero, keep} : std::vector<cx>{keep, zero};
    DiagonalPlan<T> plan(entries, {layout[qubit]}, {}, block_bits());
    plan.apply(buffer, true);
    return outcome;
  }

  // measure.rs:104-174, with the uniforms given (the reference draws
  // rng.random::<f64>() per shot).
  std::vector<uint64_t> sample_unordered(size_t shots, const double* uniforms) const {
    std::vector<uint64_t> outcomes;
    if (shots == 0) return outcomes;
    const size_t lanes = S::LANES;
    const size_t chunk_len = 2 * lanes * CHUNK_BLOCKS;
    const size_t nchunks = (len + chunk_len - 1) / chunk_len;
    std::vector<double> sums(nchunks, 0.0);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < long(nchunks); ++c) {
      double s = 0.0;
      size_t nb = std::min(CHUNK_BLOCKS, (len - size_t(c) * chunk_len) / (2 * lanes));
      for (size_t b = 0; b < nb; ++b) {
        const T* block = buffer + size_t(c) * chunk_len + b * 2 * lanes;
        for (size_t l = 0; l < lanes; ++l) {
          double re = double(block[l]), im = double(block[l + lanes]);
          s += re * re + im * im;
        }
      }
      sums[size_t(c)] = s;
    }
    std::vector<double> prefix(nchunks + 1);
    prefix[0] = 0.0;
    for (size_t c = 0; c < nchunks; ++c) prefix[c + 1] = prefix[c] + sums[c];
    double total = prefix[nchunks];
    std::vector<double> targets(shots);
    for (size_t s = 0; s < shots; ++s) targets[s] = uniforms[s] * total;
    std::sort(targets.begin(), targets.end());
    std::vector<size_t> bounds(nchunks + 1);
    for (size_t c = 0; c <= nchunks; ++c)
      bounds[c] = size_t(std::lower_bound(targets.begin(), targets.end(), prefix[c]) - targets.begin());
    const size_t n_len = size();
    std::vector<std::vector<uint64_t>> found(nchunks);
#pragma omp parallel for schedule(dynamic, 16)
    for (long cc = 0; cc < long(nchunks); ++cc) {
      size_t chunk = size_t(cc);
      size_t lo = bounds[chunk], hi = std::min(bounds[chunk + 1], shots);
      if (lo >= hi) continue;
      auto& f = found[chunk];
      double cumulative = prefix[chunk];
      size_t shot = lo;
      size_t last_nonzero = (chunk * CHUNK_BLOCKS) << S::LANE_BITS;
      size_t nb = std::min(CHUNK_BLOCKS, (len - chunk * chunk_len) / (2 * lanes));
      bool stop = false;
      for (size_t b = 0; b < nb && !stop; ++b) {
        const T* block = buffer + chunk * chunk_len + b * 2 * lanes;
        for (size_t l = 0; l < lanes; ++l) {
          double re = double(block[l]), im = double(block[l + lanes]);
          double p = re * re + im * im;
          if (p == 0.0) continue;
          size_t index = ((chunk * CHUNK_BLOCKS + b) << S::LANE_BITS) | l;
          last_nonzero = index;
          cumulative += p;
          while (shot < hi && targets[shot] < cumulative) {
            f.push_back(index);
            ++shot;
          }
          if (shot == hi) {
            stop = true;
            break;
          }
        }
      }
      f.resize(hi - lo, last_nonzero);
      for (auto& x : f) x = std::min<uint64_t>(x, n_len - 1);
    }
    for (auto& f : found) outcomes.insert(outcomes.end(), f.begin(), f.end());
    if (!identity_layout())
      for (auto& o : outcomes) o = logical_index(size_t(o));
    return outcomes;
  }
};

// ----------------------------------------------------------------- blocking
// src/blocking.rs:32-302.
static constexpr unsigned DEFAULT_REGION_BITS = 14;

struct BlockingStats {
  size_t stages = 0, swaps = 0, kernels = 0;
};

template <class T>
struct RegionOp {
  size_t control_mask = 0, control_value = 0;
  std::vector<size_t> diagonal_global;
  std::vector<Plan<T>> plans;

  RegionOp(const Op& op, const std::vector<size_t>& layout, size_t local_limit, unsigned region_bits) {
    std::vector<std::pair<size_t, bool>> local_controls;
    for (auto& c : op.controls) {
      size_t p = layout[c.first];
      if (p >= local_limit) {
        control_mask |= size_t(1) << (p - local_limit);
        control_value |= size_t(c.second) << (p - local_limit);
      } else {
        local_controls.push_back({p, c.second});
      }
    }
    std::vector<size_t> physical;
    for (size_t q : op.targets) physical.push_back(layout[q]);
    bool all_local = true;
    for (size_t p : physical)
      if (p >= local_limit) all_local = false;
    if (all_local) {
      plans.emplace_back(op.matrix, physical, local_controls, region_bits);
      return;
    }
    std::vector<cx> diagonal = op.matrix.diagonal_entries();
    std::vector<size_t> global, local;
    for (size_t j = 0; j < physical.size(); ++j) (physical[j] >= local_limit ? global : local).push_back(j);
    std::vector<size_t> local_targets;
    for (size_t j : local) local_targets.push_back(physical[j]);
    for (size_t j : global) diagonal_global.push_back(physical[j] - local_limit);
    for (size_t assignment = 0; assignment < (size_t(1) << global.size()); ++assignment) {
      std::vector<cx> entries;
      for (size_t sub = 0; sub < (size_t(1) << local.size()); ++sub) {
        size_t index = 0;
        for (size_t m = 0; m < global.size(); ++m) index |= ((assignment >> m) & 1) << global[m];
        for (size_t m = 0; m < local.size(); ++m) index |= ((sub >> m) & 1) << local[m];
        entries.push_back(diagonal[index]);
      }
      plans.emplace_back(Matrix::diagonal(entries), local_targets, local_controls, region_bits);
    }
  }
  void apply(size_t region, T* ptr) const {
    if ((region & control_mask) != control_value) return;
    if (diagonal_global.empty()) {
      plans[0].apply(ptr, false);
      return;
    }
    size_t assignment = 0;
    for (size_t m = 0; m < diagonal_global.size(); ++m) assignment |= ((region >> diagonal_global[m]) & 1) << m;
    plans[assignment].apply(ptr, false);
  }
};

static bool runs_locally(const Op& op, const std::vector<size_t>& layout, size_t local_limit) {
  if (op.matrix.is_diagonal()) return true;
  for (size_t q : op.targets)
    if (layout[q] >= local_limit) return false;
  return true;
}

template <class F>
static std::vector<size_t> extract(const std::vector<Op>& ops, const std::vector<bool>& done, F&& can_run) {
  std::vector<size_t> taken, blocked;
  auto contains = [](const std::vector<size_t>& v, size_t x) { return std::find(v.begin(), v.end(), x) != v.end(); };
  for (size_t i = 0; i < ops.size(); ++i) {
    if (done[i]) continue;
    std::vector<size_t> qs = ops[i].qubits();
    bool touches = false;
    for (size_t q : qs)
      if (contains(blocked, q)) touches = true;
    if (!touches && can_run(ops[i])) {
      taken.push_back(i);
    } else {
      for (size_t q : qs)
        if (!contains(blocked, q)) blocked.push_back(q);
    }
  }
  return taken;
}

static std::vector<std::pair<size_t, size_t>> plan_swaps(const std::vector<Op>& ops, const std::vector<bool>& done,
                                                         const std::vector<size_t>& layout, size_t lane_bits,
                                                         size_t local_limit) {
  size_t capacity = local_limit - lane_bits;
  std::vector<size_t> wanted;
  auto contains = [](const std::vector<size_t>& v, size_t x) { return std::find(v.begin(), v.end(), x) != v.end(); };
  extract(ops, done, [&](const Op& op) {
    if (op.matrix.is_diagonal()) return true;
    std::vector<size_t> fresh;
    for (size_t q : op.targets)
      if (layout[q] >= lane_bits && !contains(wanted, q)) fresh.push_back(q);
    if (wanted.size() + fresh.size() > capacity) return false;
    for (size_t q : fresh) wanted.push_back(q);
    return true;
  });
  std::vector<std::pair<size_t, size_t>> pairs;
  if (wanted.empty()) return pairs;
  std::vector<size_t> incoming, wanted_positions;
  for (size_t q : wanted) {
    wanted_positions.push_back(layout[q]);
    if (layout[q] >= local_limit) incoming.push_back(layout[q]);
  }
  std::vector<size_t> victims;
  for (size_t p = local_limit; p-- > lane_bits;)
    if (!contains(wanted_positions, p)) victims.push_back(p);
  for (size_t i = 0; i < incoming.size() && i < victims.size(); ++i) pairs.push_back({victims[i], incoming[i]});
  return pairs;
}

template <class T>
BlockingStats apply_blocked(StateVector<T>& state, const std::vector<Op>& ops, unsigned region_bits,
                            size_t max_fused) {
  const size_t lane_bits = Simd<T>::LANE_BITS;
  const unsigned block_bits = state.block_bits();
  BlockingStats stats;
  if (block_bits <= region_bits + 1) {
    for (auto& op : fuse(ops, max_fused)) {
      state.apply(op.matrix, op.targets, op.controls);
      stats.stages++;
      stats.kernels++;
    }
    return stats;
  }
  const size_t local_limit = lane_bits + region_bits;
  const size_t regions = size_t(1) << (block_bits - region_bits);
  const size_t region_len = (size_t(1) << region_bits) * 2 * Simd<T>::LANES;
  std::vector<bool> done(ops.size(), false);
  size_t remaining = ops.size();
  while (remaining > 0) {
    std::vector<size_t> layout = state.layout;
    std::vector<size_t> taken = extract(ops, done, [&](const Op& op) { return runs_locally(op, layout, local_limit); });
    if (!taken.empty()) {
      for (size_t i : taken) done[i] = true;
      remaining -= taken.size();
      std::vector<Op> stage_ops;
      for (size_t i : taken) stage_ops.push_back(ops[i]);
      auto fused = fuse_where(stage_ops, max_fused, [&](const Op& op) {
        for (size_t q : op.qubits())
          if (layout[q] >= local_limit) return false;
        return true;
      });
      stats.kernels += fused.size();
      std::vector<RegionOp<T>> stage;
      for (auto& op : fused) stage.emplace_back(op, layout, local_limit, region_bits);
      T* base = state.buffer;
#pragma omp parallel for schedule(dynamic, 1)
      for (long region = 0; region < long(regions); ++region) {
        T* ptr = base + size_t(region) * region_len;
        for (auto& op : stage) op.apply(size_t(region), ptr);
      }
      stats.stages++;
    }
    if (remaining == 0) break;
    auto pairs = plan_swaps(ops, done, layout, lane_bits, local_limit);
    if (pairs.empty()) {
      size_t i = size_t(std::find(done.begin(), done.end(), false) - done.begin());
      done[i] = true;
      remaining--;
      state.apply(ops[i].matrix, ops[i].targets, ops[i].controls);
      stats.stages++;
      stats.kernels++;
    } else {
      state.swap_physical(pairs);
      stats.swaps++;
    }
  }
  return stats;
}

// simulator.rs:122-147. region_bits < 0 means None (no blocking).
template <class T>
void apply_ops(StateVector<T>& state, const std::vector<Op>& ops, size_t max_fused, int region_bits, uint64_t* stats) {
  max_fused = std::max<size_t>(max_fused, 1);
  size_t kernels = 0, passes = 0;
  if (region_bits >= 0) {
    BlockingStats b = apply_blocked(state, ops, unsigned(region_bits), max_fused);
    passes = b.stages + b.swaps;
    kernels = b.kernels;
  } else {
    auto fused = fuse(ops, max_fused);
    for (auto& op : fused) state.apply(op.matrix, op.targets, op.controls);
    passes = kernels = fused.size();
  }
  if (stats) {
    stats[0] = ops.size();
    stats[1] = kernels;
    stats[2] = passes;
  }
}

// ------------------------------------------------------------- naive oracle
// src/reference.rs:8-29: gather 2^k amplitudes, dense mat-vec, scatter (f64).
static void naive_apply(cx* state, size_t n, const Matrix& m, const std::vector<size_t>& qubits) {
  const size_t k = qubits.size();
  size_t mask = 0;
  for (size_t q : qubits) mask |= size_t(1) << q;
  std::vector<cx> input(size_t(1) << k);
  auto offset = [&](size_t sub) {
    size_t o = 0;
    for (size_t j = 0; j < k; ++j) o |= ((sub >> j) & 1) << qubits[j];
    return o;
  };
  const size_t len = size_t(1) << n;
  for (size_t base = 0; base < len; ++base) {
    if (base & mask) continue;
    for (size_t sub = 0; sub < input.size(); ++sub) input[sub] = state[base | offset(sub)];
    for (size_t row = 0; row < input.size(); ++row) {
      cx acc{0.0, 0.0};
      for (size_t col = 0; col < input.size(); ++col) cadd_to(acc, cmul(m.at(row, col), input[col]));
      state[base | offset(row)] = acc;
    }
  }
}

}  // namespace oracle

// =================================================================== C API
using namespace oracle;

namespace {
thread_local std::string g_error;

struct Handle {
  int bits;
  StateVector<float>* f = nullptr;
  StateVector<double>* d = nullptr;
};

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

std::vector<Op> ops_from_abi(const qvdg_op* ops, size_t n) {
  std::vector<Op> v;
  v.reserve(n);
  for (size_t i = 0; i < n; ++i) v.push_back(op_from_abi(ops[i]));
  return v;
}
}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_error.c_str(); }

void oracle_set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
}
int oracle_max_threads(void) { return omp_get_max_threads(); }

// Naive f64 simulator on an interleaved complex128 array (reference.rs:8-29).
int oracle_naive_apply(double* state, uint32_t num_qubits, const double* matrix, const uint32_t* qubits,
                       uint32_t k) {
  return guarded([&] {
    std::vector<size_t> qs(qubits, qubits + k);
    naive_apply(reinterpret_cast<cx*>(state), num_qubits, Matrix::from_interleaved(matrix, k), qs);
  });
}

// Naive application of an op with controls: the matrix controlled on its
// control qubits, applied on [controls..., targets...] (tests/kernels.rs:37-52).
int oracle_naive_apply_op(double* state, uint32_t num_qubits, const qvdg_op* op) {
  return guarded([&] {
    Op o = op_from_abi(*op);
    std::vector<size_t> qs;
    Matrix m;
    o.full(qs, m);
    naive_apply(reinterpret_cast<cx*>(state), num_qubits, m, qs);
  });
}

void* oracle_sv_create(uint32_t num_qubits, int precision_bits) {
  Handle* h = nullptr;
  int rc = guarded([&] {
    h = new Handle{precision_bits};
    if (precision_bits == 32)
      h->f = new StateVector<float>(num_qubits);
    else if (precision_bits == 64)
      h->d = new StateVector<double>(num_qubits);
    else
      throw std::runtime_error("precision must be 32 or 64");
  });
  if (rc) {
    delete h;
    return nullptr;
  }
  return h;
}

void oracle_sv_destroy(void* p) {
  Handle* h = static_cast<Handle*>(p);
  if (!h) return;
  delete h->f;
  delete h->d;
  delete h;
}

#define DISPATCH(h, expr)               \
  do {                                  \
    if ((h)->f) {                       \
      auto& s = *(h)->f;                \
      expr;                             \
    } else {                            \
      auto& s = *(h)->d;                \
      expr;                             \
    }                                   \
  } while (0)

int oracle_sv_set_amplitudes(void* p, const double* amplitudes) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] { DISPATCH(h, s.set_all(amplitudes)); });
}

int oracle_sv_get_amplitudes(void* p, double* out) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] { DISPATCH(h, s.get_all(out)); });
}

int oracle_sv_apply_ops(void* p, const qvdg_op* ops, size_t num_ops, uint32_t max_fused, int region_bits,
                        uint64_t* stats) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] {
    auto v = ops_from_abi(ops, num_ops);
    DISPATCH(h, apply_ops(s, v, max_fused, region_bits, stats));
  });
}

int oracle_sv_apply(void* p, const double* matrix, const uint32_t* qubits, uint32_t k, const uint32_t* controls,
                    const uint8_t* values, uint32_t c) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] {
    std::vector<size_t> qs(qubits, qubits + k);
    std::vector<std::pair<size_t, bool>> cs;
    for (uint32_t i = 0; i < c; ++i) cs.push_back({controls[i], values[i] != 0});
    Matrix m = Matrix::from_interleaved(matrix, k);
    DISPATCH(h, s.apply(m, qs, cs));
  });
}

int oracle_sv_norm_sqr(void* p, double* out) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] { DISPATCH(h, *out = s.norm_sqr()); });
}

int oracle_sv_probability_one(void* p, uint32_t qubit, double* out) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] { DISPATCH(h, *out = s.probability_one(qubit)); });
}

int oracle_sv_measure(void* p, uint32_t qubit, double uniform, int32_t* outcome) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] { DISPATCH(h, *outcome = s.measure(qubit, uniform) ? 1 : 0); });
}

int oracle_sv_sample_unordered(void* p, size_t shots, const double* uniforms, uint64_t* out, size_t* count) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] {
    std::vector<uint64_t> o;
    DISPATCH(h, o = s.sample_unordered(shots, uniforms));
    std::copy(o.begin(), o.end(), out);
    *count = o.size();
  });
}

int oracle_sv_layout(void* p, uint32_t* layout) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] {
    DISPATCH(h, for (size_t q = 0; q < s.layout.size(); ++q) layout[q] = uint32_t(s.layout[q]));
  });
}

}  // extern "C"

namespace {

// layout[logical] = physical as a permutation check.
std::vector<size_t> checked_layout(const uint32_t* layout, size_t n) {
  std::vector<size_t> v(layout, layout + n);
  size_t seen = 0;
  for (size_t q : v) {
    if (q >= n || (seen >> q & 1)) throw std::runtime_error("layout is not a permutation of the qubits");
    seen |= size_t(1) << q;
  }
  return v;
}

// Logical -> physical index through a layout, as the OR of per-16-bit-slice
// tables (a bit permutation maps disjoint bit sets to disjoint bit sets).
struct IndexMap {
  std::vector<std::vector<size_t>> tables;
  explicit IndexMap(const std::vector<size_t>& layout) {
    const size_t n = layout.size();
    for (size_t lo = 0; lo < std::max<size_t>(n, 1); lo += 16) {
      const size_t w = std::min<size_t>(16, n - lo);
      std::vector<size_t> t(size_t(1) << w, 0);
      for (size_t v = 0; v < t.size(); ++v)
        for (size_t b = 0; b < w; ++b) t[v] |= ((v >> b) & 1) << layout[lo + b];
      tables.push_back(std::move(t));
    }
  }
  size_t operator()(size_t index) const {
    size_t p = 0;
    for (size_t s = 0; s < tables.size(); ++s) p |= tables[s][(index >> (16 * s)) & (tables[s].size() - 1)];
    return p;
  }
};

// Interleaved (re, im) value at physical position i of a buffer of either precision.
inline void read_pair(const void* amps, int bits, size_t i, double& re, double& im) {
  if (bits == 32) {
    const float* f = static_cast<const float*>(amps);
    re = double(f[2 * i]);
    im = double(f[2 * i + 1]);
  } else {
    const double* d = static_cast<const double*>(amps);
    re = d[2 * i];
    im = d[2 * i + 1];
  }
}

template <class T>
void set_physical(StateVector<T>& s, const void* amps, int bits) {
  s.buffer[0] = T(0);
  const long count = long(s.size());
#pragma omp parallel for schedule(static)
  for (long i = 0; i < count; ++i) {
    size_t re, im;
    double a, b;
    read_pair(amps, bits, size_t(i), a, b);
    StateVector<T>::offsets(size_t(i), re, im);
    s.buffer[re] = T(a);
    s.buffer[im] = T(b);
  }
}

template <class T>
double max_diff_physical(const StateVector<T>& s, const void* amps, int bits, const std::vector<size_t>& layout) {
  const IndexMap mine(s.layout), theirs(layout);
  const long count = long(s.size());
  double worst = 0.0;
#pragma omp parallel for schedule(static) reduction(max : worst)
  for (long i = 0; i < count; ++i) {
    size_t re, im;
    StateVector<T>::offsets(mine(size_t(i)), re, im);
    double a, b;
    read_pair(amps, bits, theirs(size_t(i)), a, b);
    const double dr = double(s.buffer[re]) - a, di = double(s.buffer[im]) - b;
    worst = std::max(worst, std::sqrt(dr * dr + di * di));
  }
  return worst;
}

}  // namespace

extern "C" {

// Sets the layout (layout[logical] = physical) without moving amplitudes;
// with oracle_sv_set_physical it loads another engine's state as it lies in
// memory, so that chunk order (the sampler's summation order) is the same.
int oracle_sv_set_layout(void* p, const uint32_t* layout) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] { DISPATCH(h, s.layout = checked_layout(layout, s.num_qubits)); });
}

// Loads 2^n interleaved complex amplitudes in PHYSICAL order, given in
// `precision_bits` (32: float pairs, 64: double pairs).
int oracle_sv_set_physical(void* p, const void* amplitudes, int precision_bits) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] {
    if (precision_bits != 32 && precision_bits != 64) throw std::runtime_error("precision must be 32 or 64");
    DISPATCH(h, set_physical(s, amplitudes, precision_bits));
  });
}

// max over logical indices of |this state's amplitude - the other's|, the
// other given as physical-order interleaved amplitudes with its own layout.
int oracle_sv_max_diff_physical(void* p, const void* amplitudes, int precision_bits, const uint32_t* layout,
                                double* out) {
  Handle* h = static_cast<Handle*>(p);
  return guarded([&] {
    if (precision_bits != 32 && precision_bits != 64) throw std::runtime_error("precision must be 32 or 64");
    DISPATCH(h, *out = max_diff_physical(s, amplitudes, precision_bits, checked_layout(layout, s.num_qubits)));
  });
}

// Greedy fusion alone (fusion.rs:63-115): writes the number of fused ops and,
// per fused op, its number of targets and controls.
int oracle_fuse_shapes(const qvdg_op* ops, size_t num_ops, uint32_t max_fused, size_t* num_fused, uint32_t* widths,
                       size_t capacity) {
  return guarded([&] {
    auto fused = fuse(ops_from_abi(ops, num_ops), max_fused);
    *num_fused = fused.size();
    for (size_t i = 0; i < fused.size() && 2 * i + 1 < capacity; ++i) {
      widths[2 * i] = uint32_t(fused[i].targets.size());
      widths[2 * i + 1] = uint32_t(fused[i].controls.size());
    }
  });
}

}  // extern "C"
