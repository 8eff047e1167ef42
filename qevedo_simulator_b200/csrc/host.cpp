// Host gate algebra and greedy fusion (see host.hpp for the reference map).
#include "host.hpp"

#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <exception>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace qvdg {

HMatrix HMatrix::identity(size_t qubits) {
  HMatrix m(size_t(1) << qubits);
  for (size_t i = 0; i < m.dim; ++i) m.at(i, i) = {1.0, 0.0};
  return m;
}

HMatrix HMatrix::diagonal(const std::vector<C>& d) {
  HMatrix m(d.size());
  for (size_t i = 0; i < d.size(); ++i) m.at(i, i) = d[i];
  return m;
}

bool HMatrix::is_diagonal() const {
  for (size_t r = 0; r < dim; ++r)
    for (size_t c = 0; c < dim; ++c)
      if (r != c && norm2(at(r, c)) != 0.0) return false;
  return true;
}

std::vector<C> HMatrix::diagonal_entries() const {
  std::vector<C> d(dim);
  for (size_t i = 0; i < dim; ++i) d[i] = at(i, i);
  return d;
}

HMatrix HMatrix::mul(const HMatrix& o) const {
  HMatrix out(dim);
  for (size_t r = 0; r < dim; ++r)
    for (size_t k = 0; k < dim; ++k) {
      const C x = at(r, k);
      if (norm2(x) == 0.0) continue;
      for (size_t c = 0; c < dim; ++c) {
        C p = x * o.at(k, c);
        C& t = out.at(r, c);
        t.re += p.re;
        t.im += p.im;
      }
    }
  return out;
}

HMatrix HMatrix::embed(const std::vector<uint32_t>& gate_qubits, const std::vector<uint32_t>& qubits) const {
  std::vector<size_t> position;
  for (uint32_t q : gate_qubits) {
    auto it = std::find(qubits.begin(), qubits.end(), q);
    if (it == qubits.end()) throw std::logic_error("qubit missing from embedding");
    position.push_back(size_t(it - qubits.begin()));
  }
  size_t gate_mask = 0;
  for (size_t p : position) gate_mask |= size_t(1) << p;
  HMatrix out(size_t(1) << qubits.size());
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

HMatrix HMatrix::controlled(size_t controls, size_t state) const {
  HMatrix out = identity(controls + qubits());
  const size_t mask = (size_t(1) << controls) - 1;
  for (size_t r = 0; r < out.dim; ++r)
    for (size_t c = 0; c < out.dim; ++c) {
      const bool rc = (r & mask) == state, cc = (c & mask) == state;
      if (rc && cc)
        out.at(r, c) = at(r >> controls, c >> controls);
      else if (rc || cc)
        out.at(r, c) = {0.0, 0.0};
    }
  return out;
}

std::vector<uint32_t> HOp::qubits() const {
  std::vector<uint32_t> q(targets);
  for (auto& c : controls) q.push_back(c.first);
  return q;
}

void HOp::full(std::vector<uint32_t>& qs, HMatrix& m) const {
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
  qs.insert(qs.end(), targets.begin(), targets.end());
  m = matrix.controlled(controls.size(), state);
}

namespace {

// One growth sweep of a fused group over the ops after its seed
// (src/fusion.rs:126-170), on qubit bit masks: an op joins when it touches
// no blocked qubit and fits; otherwise its qubits become blocked. `pre`:
// qubits of unfused ops before the seed (they block from the start). The
// sweep may stop early once every qubit of the group is blocked and either
// the group has max_qubits qubits or every other qubit is blocked too: a
// later op could then join only if it touched no qubit at all, and
// `can_stop` says that no op is like that.
//
// With in.commute, a diagonal op is blocked only by skipped non-diagonal
// ops (`blocked`): diagonal ops commute, so it may move ahead of skipped
// diagonal ones (`blocked_diag`, which still block non-diagonal ops). The
// stop rule then looks at `blocked` alone.
template <class Done>
void grow(const FusionInput& in, const Done& done, std::vector<uint8_t>& taken, size_t seed, uint64_t pre,
          uint64_t pre_diag, std::vector<size_t>& members, uint64_t& qubits, size_t max_qubits,
          bool connected_only, bool can_stop) {
  uint64_t blocked = pre, blocked_diag = pre_diag;
  const size_t n = in.mask.size();
  for (size_t i = seed + 1; i < n; ++i) {
    if (done(i) || taken[i]) continue;
    if (connected_only && (qubits & ~blocked) == 0) break;
    const bool diag = in.commute && in.diag[i];
    const uint64_t m = in.mask[i], fresh = m & ~qubits;
    const bool connected = fresh != m;
    const bool fits = in.width[i] <= max_qubits && size_t(__builtin_popcountll(qubits | m)) <= max_qubits;
    if (!(m & (diag ? blocked : blocked | blocked_diag)) && fits && (connected || !connected_only)) {
      taken[i] = true;
      members.push_back(i);
      qubits |= m;
    } else {
      (diag ? blocked_diag : blocked) |= m;
      if (can_stop && (qubits & ~blocked) == 0 &&
          (size_t(__builtin_popcountll(qubits)) >= max_qubits || (in.all & ~blocked & ~qubits) == 0))
        break;
    }
  }
}

// Whether a seed at `mask` may start a group ahead of the unfused ops
// before it (`pending`, and `pending_diag` for diagonal ones in commute
// mode), and those ops' qubits updated with op s.
inline bool ready(const FusionInput& in, size_t s, uint64_t pending, uint64_t pending_diag) {
  return !(in.mask[s] & (in.commute && in.diag[s] ? pending : pending | pending_diag));
}
inline void hold(const FusionInput& in, size_t s, uint64_t& pending, uint64_t& pending_diag) {
  (in.commute && in.diag[s] ? pending_diag : pending) |= in.mask[s];
}

}  // namespace

FusionInput fusion_input(const std::vector<HOp>& ops, const std::function<bool(const HOp&)>& fusable) {
  FusionInput in;
  const size_t n = ops.size();
  in.mask.assign(n, 0);
  in.width.resize(n);
  for (size_t i = 0; i < n; ++i) {
    auto add = [&](uint32_t q) {
      if (q >= 64) throw std::logic_error("fusion supports qubits 0..63");
      in.mask[i] |= uint64_t(1) << q;
    };
    for (uint32_t q : ops[i].targets) add(q);
    for (auto& c : ops[i].controls) add(c.first);
    in.width[i] = fusable(ops[i]) ? ops[i].width() : SIZE_MAX;
    in.diag.push_back(ops[i].diagonal ? 1 : 0);
    in.any_empty = in.any_empty || in.mask[i] == 0;
    in.all |= in.mask[i];
  }
  return in;
}

bool diagonal_runs(const FusionInput& in) {
  uint64_t last_diag = 0;  // qubits whose latest op is diagonal
  for (size_t i = 0; i < in.mask.size(); ++i) {
    if (in.diag[i]) {
      if (in.mask[i] & last_diag) return true;
      last_diag |= in.mask[i];
    } else {
      last_diag &= ~in.mask[i];
    }
  }
  return false;
}

std::vector<FusedGroup> fuse_groups_lookahead(const FusionInput& in, size_t max_qubits, size_t lookahead) {
  const size_t n = in.mask.size();
  const std::vector<uint64_t>& mask = in.mask;
  std::vector<uint8_t> done(n, 0), taken(n, 0);
  const auto is_done = [&](size_t i) { return done[i] != 0; };
  std::vector<FusedGroup> groups;
  size_t first = 0;
  std::vector<size_t> members, best_members;
  while (true) {
    while (first < n && done[first]) ++first;
    if (first == n) break;
    // Seeds: the first unfused op, then up to `lookahead` later ones that
    // no unfused earlier op holds back; keep the seed whose group takes the
    // most ops (ties: the earliest).
    uint64_t pending = 0, pending_diag = 0, best_qubits = 0;
    size_t tried = 0;
    best_members.clear();
    for (size_t s = first; s < n && tried <= lookahead; ++s) {
      if (done[s]) continue;
      if (ready(in, s, pending, pending_diag)) {
        ++tried;
        members.assign(1, s);
        uint64_t qubits = mask[s];
        taken[s] = true;
        if (in.width[s] <= max_qubits) {
          grow(in, is_done, taken, s, pending, pending_diag, members, qubits, max_qubits, true, false);
          grow(in, is_done, taken, s, pending, pending_diag, members, qubits, max_qubits, false, !in.any_empty);
        }
        for (size_t i : members) taken[i] = false;
        if (members.size() > best_members.size()) {
          best_members = members;
          best_qubits = qubits;
        }
      }
      hold(in, s, pending, pending_diag);
    }
    FusedGroup g;
    g.members = best_members;
    std::sort(g.members.begin(), g.members.end());
    for (size_t i : g.members) done[i] = true;
    for (uint32_t q = 0; q < 64; ++q)
      if ((best_qubits >> q) & 1) g.qubits.push_back(q);
    groups.push_back(std::move(g));
  }
  return groups;
}

namespace {

// A partial fusion of the beam search: the ops it covers (one bit each) and
// its newest group (earlier ones through the arena's parent links).
struct BeamNode {
  std::vector<uint64_t> done;
  size_t first = 0;    // no uncovered op before this one
  size_t covered = 0;  // ops covered
  int64_t last = -1;   // newest group in the arena
};

struct BeamGroup {
  int64_t parent;
  uint32_t offset, count;  // members (ascending) in the member pool
  uint64_t qubits;
};

}  // namespace

std::vector<std::vector<FusedGroup>> fuse_groups_beam(const FusionInput& in, size_t max_qubits, size_t lookahead,
                                                      size_t width) {
  const size_t n = in.mask.size();
  std::vector<BeamGroup> arena;
  std::vector<uint32_t> pool;
  std::vector<BeamNode> beam(1), next;
  beam[0].done.assign((n + 63) / 64, 0);
  while (true) {
    std::vector<std::vector<FusedGroup>> finished;
    for (const BeamNode& b : beam) {
      if (b.covered < n) continue;
      std::vector<FusedGroup> gs;
      for (int64_t g = b.last; g >= 0; g = arena[size_t(g)].parent) {
        FusedGroup f;
        const BeamGroup& bg = arena[size_t(g)];
        f.members.assign(pool.begin() + bg.offset, pool.begin() + bg.offset + bg.count);
        for (uint32_t q = 0; q < 64; ++q)
          if ((arena[size_t(g)].qubits >> q) & 1) f.qubits.push_back(q);
        gs.push_back(std::move(f));
      }
      std::reverse(gs.begin(), gs.end());
      finished.push_back(std::move(gs));
    }
    if (!finished.empty() || beam.empty()) return finished;
    // Every kept partial fusion's children, on the pool's threads; merged
    // in the nodes' order, so the result does not depend on timing.
    struct Child {
      BeamNode node;
      std::vector<size_t> members;  // ascending
      uint64_t qubits;
    };
    std::vector<std::vector<Child>> kids(beam.size());
    parallel_for(beam.size(), [&](size_t bi) {
      const BeamNode& b = beam[bi];
      thread_local std::vector<uint8_t> taken;  // all 0 between uses
      if (taken.size() < n) taken.resize(n, 0);
      std::vector<size_t> members;
      const auto is_done = [&](size_t i) { return ((b.done[i >> 6] >> (i & 63)) & 1) != 0; };
      size_t first = b.first;
      while (first < n && is_done(first)) ++first;
      uint64_t pending = 0, pending_diag = 0;
      size_t tried = 0;
      for (size_t s = first; s < n && tried <= lookahead; ++s) {
        if (is_done(s)) continue;
        if (ready(in, s, pending, pending_diag)) {
          ++tried;
          members.assign(1, s);
          uint64_t qubits = in.mask[s];
          taken[s] = 1;
          if (in.width[s] <= max_qubits) {
            grow(in, is_done, taken, s, pending, pending_diag, members, qubits, max_qubits, true, false);
            grow(in, is_done, taken, s, pending, pending_diag, members, qubits, max_qubits, false, !in.any_empty);
          }
          for (size_t i : members) taken[i] = 0;
          Child c;
          c.node.done = b.done;
          for (size_t i : members) c.node.done[i >> 6] |= uint64_t(1) << (i & 63);
          c.node.first = first;
          c.node.covered = b.covered + members.size();
          c.node.last = b.last;  // the parent's newest group, until merged
          std::sort(members.begin(), members.end());
          c.members = members;
          c.qubits = qubits;
          kids[bi].push_back(std::move(c));
        }
        hold(in, s, pending, pending_diag);
      }
    });
    next.clear();
    for (auto& ks : kids)
      for (Child& c : ks) {
        arena.push_back({c.node.last, uint32_t(pool.size()), uint32_t(c.members.size()), c.qubits});
        pool.insert(pool.end(), c.members.begin(), c.members.end());
        c.node.last = int64_t(arena.size()) - 1;
        next.push_back(std::move(c.node));
      }
    // The `width` partial fusions that cover the most ops (earlier ones
    // first among equals), without repeats of the same covered set.
    std::stable_sort(next.begin(), next.end(),
                     [](const BeamNode& x, const BeamNode& y) { return x.covered > y.covered; });
    beam.clear();
    for (BeamNode& c : next) {
      if (beam.size() == width) break;
      bool repeat = false;
      for (const BeamNode& k : beam) repeat = repeat || (k.covered == c.covered && k.done == c.done);
      if (!repeat) beam.push_back(std::move(c));
    }
  }
}

std::vector<FusedGroup> fuse_groups_lookahead(const std::vector<HOp>& ops, size_t max_qubits,
                                              const std::function<bool(const HOp&)>& fusable, size_t lookahead) {
  return fuse_groups_lookahead(fusion_input(ops, fusable), max_qubits, lookahead);
}

std::vector<FusedGroup> fuse_groups(const std::vector<HOp>& ops, size_t max_qubits,
                                    const std::function<bool(const HOp&)>& fusable) {
  return fuse_groups_lookahead(ops, max_qubits, fusable, 0);
}

// m <- embed(g, gate_qubits -> qubits) * m without forming the embedded
// matrix: each set of rows that differ only in the gate's bits is mixed by g.
// Same products, same zero skipping and same order of additions (ascending
// row of the embedded matrix) as mul, so the result is identical.
//
// `live` (optional) tracks the sparsity of a product grown from the
// identity: entry (r, c) is exactly +0 unless r ^ c lies within *live (the
// positions of every gate applied so far). Only those columns are computed;
// the others would come out +0 (sums of +-0 products of finite entries,
// starting from +0), which they already hold.
void apply_left(HMatrix& m, const HMatrix& g, const std::vector<uint32_t>& gate_qubits,
                const std::vector<uint32_t>& qubits, size_t* live) {
  const size_t k = gate_qubits.size(), gd = size_t(1) << k;
  std::vector<size_t> off(gd, 0);
  size_t mask = 0;
  for (size_t j = 0; j < k; ++j) {
    const size_t p = size_t(std::find(qubits.begin(), qubits.end(), gate_qubits[j]) - qubits.begin());
    if (p == qubits.size()) throw std::logic_error("qubit missing from embedding");
    mask |= size_t(1) << p;
    for (size_t t = 0; t < gd; ++t)
      if ((t >> j) & 1) off[t] |= size_t(1) << p;
  }
  std::vector<size_t> order(gd);
  for (size_t t = 0; t < gd; ++t) order[t] = t;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return off[a] < off[b]; });
  // Nonzero entries of g by output row, each row's in ascending embedded column.
  struct Entry {
    size_t t;
    C x;
  };
  std::vector<std::vector<Entry>> rows(gd);
  for (size_t s = 0; s < gd; ++s)
    for (size_t t : order)
      if (norm2(g.at(s, t)) != 0.0) rows[s].push_back({t, g.at(s, t)});
  const size_t dim = m.dim;
  if (live) {
    bool finite = true;
    for (const C& x : g.a) finite = finite && std::isfinite(x.re) && std::isfinite(x.im);
    *live = finite ? ((*live | mask) & (dim - 1)) : dim - 1;
    if (*live != dim - 1) {
      // Columns that can be nonzero in the rows of block b: (b & ~u) | sub,
      // sub a subset of u (ascending).
      const size_t u = *live;
      std::vector<size_t> sub;
      size_t x = 0;
      do {
        sub.push_back(x);
        x = (x - u) & u;
      } while (x != 0);
      const size_t ns = sub.size();
      std::vector<C> in(gd * ns);
      for (size_t b = 0; b < dim; ++b) {
        if (b & mask) continue;
        const size_t cb = b & ~u;
        for (size_t t = 0; t < gd; ++t) {
          const C* src = &m.a[(b | off[t]) * dim];
          for (size_t j = 0; j < ns; ++j) in[t * ns + j] = src[cb | sub[j]];
        }
        for (size_t s = 0; s < gd; ++s) {
          C* dst = &m.a[(b | off[s]) * dim];
          for (size_t j = 0; j < ns; ++j) {
            C acc{0.0, 0.0};
            for (const Entry& e : rows[s]) {
              const C p = e.x * in[e.t * ns + j];
              acc.re += p.re;
              acc.im += p.im;
            }
            dst[cb | sub[j]] = acc;
          }
        }
      }
      return;
    }
  }
  std::vector<C> in(gd * dim);
  for (size_t b = 0; b < dim; ++b) {
    if (b & mask) continue;
    for (size_t t = 0; t < gd; ++t) std::copy_n(&m.a[(b | off[t]) * dim], dim, &in[t * dim]);
    for (size_t s = 0; s < gd; ++s) {
      C* dst = &m.a[(b | off[s]) * dim];
      for (size_t c = 0; c < dim; ++c) dst[c] = {0.0, 0.0};
      for (const Entry& e : rows[s]) {
        const C* src = &in[e.t * dim];
        for (size_t c = 0; c < dim; ++c) {
          const C p = e.x * src[c];
          dst[c].re += p.re;
          dst[c].im += p.im;
        }
      }
    }
  }
}

HOp fuse_group(const std::vector<HOp>& ops, const FusedGroup& g) {
  const std::vector<size_t>& members = g.members;
  const std::vector<uint32_t>& qubits = g.qubits;
  if (members.size() == 1) return ops[members[0]];
  {
    HMatrix m = HMatrix::identity(qubits.size());
    size_t live = 0;
    for (size_t i : members) {
      std::vector<uint32_t> oq;
      HMatrix om;
      ops[i].full(oq, om);
      apply_left(m, om, oq, qubits, &live);
    }
    HOp f;
    f.targets = qubits;
    f.matrix = std::move(m);
    f.diagonal = f.matrix.is_diagonal();
    return f;
  }
}

std::vector<HOp> fuse_where(const std::vector<HOp>& ops, size_t max_qubits,
                            const std::function<bool(const HOp&)>& fusable) {
  std::vector<HOp> fused;
  for (const FusedGroup& g : fuse_groups(ops, max_qubits, fusable)) fused.push_back(fuse_group(ops, g));
  return fused;
}

namespace {

// A fork-join pool of host threads. parallel_for posts a job and runs its
// indices itself; idle workers take indices of any posted job. A caller
// whose indices are all taken helps other jobs until its own finish, so a
// task that itself calls parallel_for (the beam searches' steps inside the
// planner's candidate tasks) cannot deadlock. Workers spin briefly before
// sleeping, so the short jobs of consecutive search steps find them awake.
struct PoolJob {
  const std::function<void(size_t)>* f = nullptr;
  size_t n = 0;
  std::atomic<size_t> next{0};
  std::atomic<size_t> done{0};
  std::mutex error_mutex;
  std::exception_ptr error;

  // Runs index i of this job (taken by the caller).
  void run(size_t i) {
    try {
      (*f)(i);
    } catch (...) {
      std::lock_guard<std::mutex> lock(error_mutex);
      if (!error) error = std::current_exception();
    }
    done.fetch_add(1, std::memory_order_release);
  }
};

class WorkerPool {
 public:
  explicit WorkerPool(unsigned workers) {
    for (unsigned t = 0; t < workers; ++t) std::thread([this] { work(); }).detach();
  }

  void run(PoolJob& job) {
    {
      std::lock_guard<std::mutex> lock(m_);
      jobs_.push_back(&job);
      maybe_work_.store(true, std::memory_order_release);
    }
    cv_.notify_all();
    for (size_t i; (i = job.next.fetch_add(1)) < job.n;) job.run(i);
    while (job.done.load(std::memory_order_acquire) < job.n)
      if (!(maybe_work_.load(std::memory_order_acquire) && help())) std::this_thread::yield();
    std::lock_guard<std::mutex> lock(m_);
    jobs_.erase(std::find(jobs_.begin(), jobs_.end(), &job));
  }

 private:
  // Runs one index of any posted job; false when none is left (and then
  // marks the pool as without work until the next post).
  bool help() {
    PoolJob* job = nullptr;
    size_t i = 0;
    {
      std::lock_guard<std::mutex> lock(m_);
      for (PoolJob* j : jobs_) {
        if (j->next.load(std::memory_order_relaxed) >= j->n) continue;
        i = j->next.fetch_add(1);
        if (i < j->n) {
          job = j;
          break;
        }
      }
      if (!job) maybe_work_.store(false, std::memory_order_release);
    }
    if (!job) return false;
    job->run(i);
    return true;
  }

  void work() {
    for (;;) {
      if (help()) continue;
      // Spin (tens of microseconds) without the lock for the next post.
      for (int k = 0; k < 2000 && !maybe_work_.load(std::memory_order_acquire); ++k) std::this_thread::yield();
      if (maybe_work_.load(std::memory_order_acquire)) continue;
      std::unique_lock<std::mutex> lock(m_);
      cv_.wait(lock, [&] { return maybe_work_.load(std::memory_order_acquire); });
    }
  }

  std::mutex m_;
  std::condition_variable cv_;
  std::vector<PoolJob*> jobs_;
  std::atomic<bool> maybe_work_{false};  // a posted job may have indices left
};

// The process's pool, made again in a forked child (which inherits no
// threads; the old pool is left alone, its mutex possibly held).
WorkerPool& pool() {
  static std::mutex init;
  static WorkerPool* pool = nullptr;
  static pid_t owner = 0;
  std::lock_guard<std::mutex> lock(init);
  if (!pool || owner != getpid()) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    pool = new WorkerPool(std::min(16u, hw) - 1);  // never freed: workers live as long as the process
    owner = getpid();
  }
  return *pool;
}

}  // namespace

void parallel_for(size_t n, const std::function<void(size_t)>& f, unsigned threads) {
  if (threads == 1 || n <= 1 || std::thread::hardware_concurrency() <= 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  PoolJob job;
  job.f = &f;
  job.n = n;
  pool().run(job);
  if (job.error) std::rethrow_exception(job.error);
}

std::vector<HOp> fuse(const std::vector<HOp>& ops, size_t max_qubits) {
  return fuse_where(ops, max_qubits, [](const HOp&) { return true; });
}

}  // namespace qvdg
