// The C ABI (include/qvdg.h): state handles, op lowering and planning on the
// host, kernel launches on the state's stream, and status codes instead of
// exceptions at the boundary.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <memory>
#include <vector>

#include "batch.hpp"
#include "engine.hpp"
#include "host.hpp"
#include "planner.hpp"
#include "qvdg.h"
#include "program.hpp"
#include "stage.hpp"

struct qvdg_state {
  qvdg::StateImpl s;
};

// A planned, uploaded circuit for states of one size, precision and layout.
struct qvdg_plan {
  qvdg::Program program;
  qvdg::DeviceUpload dev;
  void* device = nullptr;  // owned copy of the gate programs and matrices
  int device_id = 0;
  // The plan for states other than |0...0>, where the fusion scored from
  // |0...0> (its zero-start passes) differs from the one scored for any
  // state; run by qvdg_plan_execute on such states.
  std::unique_ptr<qvdg::Program> general;
  qvdg::DeviceUpload general_dev;
  void* general_device = nullptr;
  qvdg_options settings{};  // what the plan was built with (the learned pick, or the given settings)
};

namespace qvdg {

void* DeviceScratch::get(size_t need) {
  if (need == 0) need = 1;
  if (need <= bytes) return ptr;
  release();
  size_t want = std::max(need, bytes * 2);
  if (cudaMalloc(&ptr, want) != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    if (cudaMalloc(&ptr, need) != cudaSuccess) {
      cudaGetLastError();
      ptr = nullptr;
      bytes = 0;
      throw Error(QVDG_ERR_OUT_OF_MEMORY, "device workspace allocation failed");
    }
    want = need;
  }
  bytes = want;
  return ptr;
}

void DeviceScratch::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

void* HostScratch::get(size_t need) {
  if (need == 0) need = 1;
  if (need <= bytes) return ptr;
  release();
  if (cudaMallocHost(&ptr, need) != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    throw Error(QVDG_ERR_OUT_OF_MEMORY, "pinned host allocation failed");
  }
  bytes = need;
  return ptr;
}

void HostScratch::release() {
  if (ptr) cudaFreeHost(ptr);
  ptr = nullptr;
  bytes = 0;
}

}  // namespace qvdg

namespace {

using namespace qvdg;

thread_local std::string g_error;

template <class F>
qvdg_status guarded(F&& f) {
  try {
    f();
    g_error.clear();
    return QVDG_OK;
  } catch (const Error& e) {
    g_error = e.what();
    return qvdg_status(e.status);
  } catch (const std::bad_alloc&) {
    g_error = "host allocation failed";
    return QVDG_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_error = e.what();
    return QVDG_ERR_INVALID;
  }
}

void require(bool ok, const std::string& message) {
  if (!ok) throw Error(QVDG_ERR_INVALID, message);
}

StateImpl& impl(qvdg_state* st) {
  require(st != nullptr, "null state");
  return st->s;
}
const StateImpl& impl(const qvdg_state* st) {
  require(st != nullptr, "null state");
  return st->s;
}

// Lower ABI ops to host ops on logical qubits, validating them as the
// reference does (qubits in range and distinct, src/circuit.rs:467-476 and
// src/state.rs:182-188).
std::vector<HOp> lower_ops(const qvdg_op* ops, size_t n, uint32_t num_qubits) {
  require(n == 0 || ops != nullptr, "null ops");
  std::vector<HOp> out;
  out.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    const qvdg_op& o = ops[i];
    // Messages are built only on failure.
    if (!(o.num_targets <= 16 && o.num_controls <= 64)) require(false, "op " + std::to_string(i) + " is too wide");
    if (!(o.num_targets == 0 || (o.targets && o.matrix)))
      require(false, "op " + std::to_string(i) + " has no targets or matrix");
    if (!(o.num_controls == 0 || o.controls)) require(false, "op " + std::to_string(i) + " has no control list");
    HOp h;
    h.targets.assign(o.targets, o.targets + o.num_targets);
    h.controls.reserve(o.num_controls);
    for (uint32_t j = 0; j < o.num_controls; ++j)
      h.controls.push_back({o.controls[j], o.control_values ? o.control_values[j] != 0 : true});
    uint64_t seen = 0;  // qubits below 64 seen so far
    const uint32_t width = o.num_targets + o.num_controls;
    for (uint32_t j = 0; j < width; ++j) {
      const uint32_t q = j < o.num_targets ? o.targets[j] : o.controls[j - o.num_targets];
      if (q >= num_qubits)
        require(false, "qubit " + std::to_string(q) + " out of range for " + std::to_string(num_qubits) + " qubits");
      bool twice;
      if (q < 64) {
        twice = (seen >> q) & 1;
        seen |= uint64_t(1) << q;
      } else {
        twice = false;
        for (uint32_t k = 0; k < j; ++k)
          twice = twice || (k < o.num_targets ? o.targets[k] : o.controls[k - o.num_targets]) == q;
      }
      if (twice) require(false, "op " + std::to_string(i) + " uses qubit " + std::to_string(q) + " twice");
    }
    const size_t dim = size_t(1) << o.num_targets;
    h.matrix = HMatrix(dim);
    for (size_t e = 0; e < dim * dim; ++e) h.matrix.a[e] = {o.matrix[2 * e], o.matrix[2 * e + 1]};
    h.diagonal = h.matrix.is_diagonal();
    if (h.targets.empty()) continue;  // StateVector::apply returns on no qubits (src/state.rs:189-191)
    out.push_back(std::move(h));
  }
  return out;
}

// A plan's gate programs and matrices in its precision, one device copy
// owned by the plan.
void upload_plan(const Program& p, uint32_t precision_bits, void** device, DeviceUpload* dev) {
  const StageUpload& up = p.upload;
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t gate_bytes = up.gates.size() * sizeof(TileGate);
  const size_t mat_bytes = up.mats.size() * (precision_bits == 32 ? 4 : 8);
  std::vector<char> h(align(gate_bytes) + align(mat_bytes) + align(up.tc.size()) + 256, 0);
  if (gate_bytes) std::memcpy(h.data(), up.gates.data(), gate_bytes);
  if (precision_bits == 32) {
    float* f = reinterpret_cast<float*>(h.data() + align(gate_bytes));
    for (size_t i = 0; i < up.mats.size(); ++i) f[i] = float(up.mats[i]);
  } else if (mat_bytes) {
    std::memcpy(h.data() + align(gate_bytes), up.mats.data(), mat_bytes);
  }
  if (!up.tc.empty()) std::memcpy(h.data() + align(gate_bytes) + align(mat_bytes), up.tc.data(), up.tc.size());
  if (cudaMalloc(device, h.size()) != cudaSuccess) {
    cudaGetLastError();
    *device = nullptr;
    throw Error(QVDG_ERR_OUT_OF_MEMORY, "cannot allocate the plan's device memory");
  }
  QVDG_CUDA(cudaMemcpy(*device, h.data(), h.size(), cudaMemcpyHostToDevice));
  dev->gates = static_cast<const TileGate*>(*device);
  dev->mats = static_cast<const char*>(*device) + align(gate_bytes);
  dev->tc = static_cast<const uint8_t*>(*device) + align(gate_bytes) + align(mat_bytes);
}

// Plan, upload and run `ops` on the state (the reference's apply_ops,
// src/simulator.rs:122-147).
void apply_program(StateImpl& s, const std::vector<HOp>& ops, const qvdg_options& opt, qvdg_stats* stats) {
  // One-shot: narrow beam searches where a pass streams at least 8 GB.
  qvdg_options chosen;
  const Program prog = choose_program(target_of(s), ops, opt, s.n >= 29 ? FusionSearch::Beam : FusionSearch::Lookahead,
                                      s.zero_state, &chosen);
  const DeviceUpload dev = upload_program(s, prog, s.work);
  run_program(s, prog, dev, stats);
  if (stats) stats->settings = chosen;
}

// One op as a single plain pass (StateVector::apply, src/state.rs:181-198).
void apply_single(StateImpl& s, const HOp& op) {
  qvdg_options opt;
  qvdg_default_options(&opt);
  opt.staged = 0;
  opt.max_fused_qubits = 1;
  apply_program(s, {op}, opt, nullptr);
}

}  // namespace

extern "C" {

void qvdg_default_options(qvdg_options* opt) {
  if (!opt) return;
  opt->max_fused_qubits = 4;
  opt->staged = 1;
  opt->tile_qubits = 0;
  opt->planner = QVDG_PLANNER_GREEDY;
  opt->math = QVDG_MATH_FP32;
}

const char* qvdg_last_error(void) { return g_error.c_str(); }

const char* qvdg_version(void) { return "qvdgpu 0.1.0 (sm_100a)"; }

qvdg_status qvdg_state_create(uint32_t num_qubits, uint32_t precision_bits, qvdg_state** out) {
  return guarded([&] {
    require(out != nullptr, "null output handle");
    *out = nullptr;
    require(precision_bits == 32 || precision_bits == 64, "precision must be 32 or 64 bits");
    require(num_qubits >= 1 && num_qubits <= 40, "a state needs 1 to 40 qubits");
    qvdg_state* st = new qvdg_state();
    StateImpl& s = st->s;
    try {
      s.n = num_qubits;
      s.bits = int(precision_bits);
      QVDG_CUDA(cudaGetDevice(&s.device));
      QVDG_CUDA(cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, s.device));
      s.amp_bytes = size_t(s.elem_bytes()) << num_qubits;
      if (cudaMalloc(&s.amp, s.amp_bytes) != cudaSuccess) {
        cudaGetLastError();
        s.amp = nullptr;
        throw Error(QVDG_ERR_OUT_OF_MEMORY, "cannot allocate " + std::to_string(s.amp_bytes) +
                                                " bytes of device memory for " + std::to_string(num_qubits) +
                                                " qubits");
      }
      if (cudaMalloc(&s.status, 256) != cudaSuccess) {
        cudaGetLastError();
        s.status = nullptr;
        throw Error(QVDG_ERR_OUT_OF_MEMORY, "cannot allocate the state's status word");
      }
      QVDG_CUDA(cudaMemset(s.status, 0, 256));
      QVDG_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
      QVDG_CUDA(cudaEventCreate(&s.ev_start));
      QVDG_CUDA(cudaEventCreate(&s.ev_stop));
      s.layout.resize(num_qubits);
      for (uint32_t q = 0; q < num_qubits; ++q) s.layout[q] = q;
      launch_zero(s);
      QVDG_CUDA(cudaStreamSynchronize(s.stream));
      s.zero_state = true;
    } catch (...) {
      qvdg_state_destroy(st);
      throw;
    }
    *out = st;
  });
}

qvdg_status qvdg_state_destroy(qvdg_state* st) {
  if (!st) return QVDG_OK;
  StateImpl& s = st->s;
  if (s.stream) cudaStreamSynchronize(s.stream);
  if (s.amp) cudaFree(s.amp);
  if (s.status) cudaFree(s.status);
  s.work.release();
  s.work2.release();
  s.host.release();
  for (cudaEvent_t e : s.pass_events) cudaEventDestroy(e);
  if (s.ev_start) cudaEventDestroy(s.ev_start);
  if (s.ev_stop) cudaEventDestroy(s.ev_stop);
  if (s.stream) cudaStreamDestroy(s.stream);
  delete st;
  return QVDG_OK;
}

qvdg_status qvdg_state_zero(qvdg_state* st) {
  return guarded([&] {
    StateImpl& s = impl(st);
    for (uint32_t q = 0; q < s.n; ++q) s.layout[q] = q;
    launch_zero(s);
    QVDG_CUDA(cudaStreamSynchronize(s.stream));
    s.zero_state = true;
  });
}

qvdg_status qvdg_state_info(const qvdg_state* st, uint32_t* num_qubits, uint32_t* precision_bits) {
  return guarded([&] {
    const StateImpl& s = impl(st);
    if (num_qubits) *num_qubits = s.n;
    if (precision_bits) *precision_bits = uint32_t(s.bits);
  });
}

qvdg_status qvdg_state_set_amplitudes(qvdg_state* st, const double* amplitudes, size_t count) {
  return guarded([&] {
    StateImpl& s = impl(st);
    require(amplitudes != nullptr, "null amplitudes");
    require(count == s.size(), "expected " + std::to_string(s.size()) + " amplitudes");
    s.zero_state = false;
    for (uint32_t q = 0; q < s.n; ++q) s.layout[q] = q;
    const uint64_t chunk = uint64_t(1) << 22;
    for (uint64_t first = 0; first < count; first += chunk) {
      const uint64_t c = std::min<uint64_t>(chunk, count - first);
      double* d = static_cast<double*>(s.work.get(c * 16));
      QVDG_CUDA(cudaMemcpyAsync(d, amplitudes + 2 * first, c * 16, cudaMemcpyHostToDevice, s.stream));
      launch_import(s, first, c, d);
      QVDG_CUDA(cudaStreamSynchronize(s.stream));
    }
  });
}

qvdg_status qvdg_state_get_amplitudes(const qvdg_state* cst, double* amplitudes, size_t count) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(cst));
    require(amplitudes != nullptr, "null output");
    require(count == s.size(), "expected room for " + std::to_string(s.size()) + " amplitudes");
    const uint64_t chunk = uint64_t(1) << 22;
    for (uint64_t first = 0; first < count; first += chunk) {
      const uint64_t c = std::min<uint64_t>(chunk, count - first);
      double* d = static_cast<double*>(s.work.get(c * 16));
      launch_export(s, first, c, d);
      QVDG_CUDA(cudaMemcpyAsync(amplitudes + 2 * first, d, c * 16, cudaMemcpyDeviceToHost, s.stream));
      QVDG_CUDA(cudaStreamSynchronize(s.stream));
    }
  });
}

qvdg_status qvdg_apply_ops(qvdg_state* st, const qvdg_op* ops, size_t num_ops, const qvdg_options* options,
                           qvdg_stats* stats) {
  return guarded([&] {
    StateImpl& s = impl(st);
    qvdg_options opt;
    qvdg_default_options(&opt);
    if (options) opt = *options;
    std::vector<HOp> host_ops = lower_ops(ops, num_ops, s.n);
    if (stats) stats->gates += num_ops;
    apply_program(s, host_ops, opt, stats);
  });
}

qvdg_status qvdg_apply(qvdg_state* st, const double* matrix, const uint32_t* qubits, uint32_t num_qubits,
                       const uint32_t* controls, const uint8_t* control_values, uint32_t num_controls) {
  return guarded([&] {
    StateImpl& s = impl(st);
    qvdg_op op{num_qubits, num_controls, qubits, controls, control_values, matrix};
    std::vector<HOp> host_ops = lower_ops(&op, 1, s.n);
    if (!host_ops.empty()) apply_single(s, host_ops[0]);
  });
}

qvdg_status qvdg_norm_sqr(const qvdg_state* st, double* out) {
  return guarded([&] {
    require(out != nullptr, "null output");
    *out = norm_sqr(const_cast<StateImpl&>(impl(st)));
  });
}

qvdg_status qvdg_scale(qvdg_state* st, double factor) {
  return guarded([&] {
    StateImpl& s = impl(st);
    s.zero_state = false;
    launch_scale(s, factor);
    QVDG_CUDA(cudaStreamSynchronize(s.stream));
  });
}

qvdg_status qvdg_probability_one(const qvdg_state* st, uint32_t qubit, double* out) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(st));
    require(out != nullptr, "null output");
    require(qubit < s.n, "qubit out of range");
    *out = probability_one(s, s.layout[qubit]);
  });
}

qvdg_status qvdg_expect_z_all(const qvdg_state* st, double* out) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(st));
    require(out != nullptr, "null output");
    std::vector<double> p1;
    double total = 0.0;
    bit_probabilities(s, p1, total);
    for (uint32_t q = 0; q < s.n; ++q) out[q] = total - 2.0 * p1[s.layout[q]];
  });
}

qvdg_status qvdg_probabilities(const qvdg_state* st, double* out, size_t count) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(st));
    require(out != nullptr, "null output");
    require(count == s.size(), "expected room for " + std::to_string(s.size()) + " probabilities");
    probabilities(s, out);
  });
}

qvdg_status qvdg_measure(qvdg_state* st, uint32_t qubit, double uniform, int32_t* outcome) {
  return guarded([&] {
    StateImpl& s = impl(st);
    require(qubit < s.n, "qubit out of range");
    // src/measure.rs:68-80
    const double p1 = std::min(std::max(probability_one(s, s.layout[qubit]), 0.0), 1.0);
    const bool one = uniform < p1;
    const double p = one ? p1 : 1.0 - p1;
    const C keep{1.0 / std::sqrt(p), 0.0}, zero{0.0, 0.0};
    HOp op;
    op.targets = {qubit};
    op.matrix = HMatrix::diagonal(one ? std::vector<C>{zero, keep} : std::vector<C>{keep, zero});
    op.diagonal = true;
    apply_single(s, op);
    if (outcome) *outcome = one ? 1 : 0;
  });
}

qvdg_status qvdg_reset(qvdg_state* st, uint32_t qubit, double uniform) {
  int32_t outcome = 0;
  qvdg_status rc = qvdg_measure(st, qubit, uniform, &outcome);
  if (rc != QVDG_OK || !outcome) return rc;
  return guarded([&] {
    StateImpl& s = impl(st);
    HOp x;
    x.targets = {qubit};
    x.matrix = HMatrix(2);
    x.matrix.at(0, 1) = {1.0, 0.0};
    x.matrix.at(1, 0) = {1.0, 0.0};
    apply_single(s, x);
  });
}

qvdg_status qvdg_sample_unordered(const qvdg_state* st, size_t shots, const double* uniforms, uint64_t* out,
                                  size_t* count) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(st));
    require(shots == 0 || (uniforms && out), "null uniforms or output");
    const size_t found = sample_unordered(s, shots, uniforms, out);
    if (count) *count = found;
  });
}

qvdg_status qvdg_swap_physical(qvdg_state* st, const uint32_t* pairs, uint32_t num_pairs) {
  return guarded([&] {
    StateImpl& s = impl(st);
    require(num_pairs == 0 || pairs, "null pairs");
    require(num_pairs <= 32, "too many pairs");
    s.zero_state = false;
    std::vector<std::pair<uint32_t, uint32_t>> p;
    uint64_t seen = 0;
    for (uint32_t i = 0; i < num_pairs; ++i) {
      const uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
      require(a < s.n && b < s.n && a != b, "invalid bit pair");
      const uint64_t m = (uint64_t(1) << a) | (uint64_t(1) << b);
      require((seen & m) == 0, "bit swapped twice in one pass");
      seen |= m;
      p.push_back({a, b});
    }
    launch_swap_bits(s, p);
    QVDG_CUDA(cudaStreamSynchronize(s.stream));
    for (auto& q : s.layout)
      for (auto& pr : p) {
        if (q == pr.first)
          q = pr.second;
        else if (q == pr.second)
          q = pr.first;
      }
  });
}

qvdg_status qvdg_state_layout(const qvdg_state* st, uint32_t* layout) {
  return guarded([&] {
    const StateImpl& s = impl(st);
    require(layout != nullptr, "null output");
    for (uint32_t q = 0; q < s.n; ++q) layout[q] = s.layout[q];
  });
}

qvdg_status qvdg_state_device_buffer(const qvdg_state* st, void** pointer, size_t* bytes) {
  return guarded([&] {
    const StateImpl& s = impl(st);
    if (pointer) *pointer = s.amp;
    if (bytes) *bytes = s.amp_bytes;
    s.zero_state = false;  // the caller may write through the pointer
  });
}

qvdg_status qvdg_synchronize(const qvdg_state* st) {
  return guarded([&] { QVDG_CUDA(cudaStreamSynchronize(impl(st).stream)); });
}

qvdg_status qvdg_plan_create(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                             const qvdg_options* options, qvdg_plan** out) {
  return guarded([&] {
    require(out != nullptr, "null output handle");
    *out = nullptr;
    require(precision_bits == 32 || precision_bits == 64, "precision must be 32 or 64 bits");
    require(num_qubits >= 1 && num_qubits <= 40, "a state needs 1 to 40 qubits");
    qvdg_options opt;
    qvdg_default_options(&opt);
    if (options) opt = *options;
    Target t;
    t.n = num_qubits;
    t.bits = int(precision_bits);
    QVDG_CUDA(cudaGetDevice(&t.sms));
    int dev = t.sms;
    QVDG_CUDA(cudaDeviceGetAttribute(&t.sms, cudaDevAttrMultiProcessorCount, dev));
    for (uint32_t q = 0; q < num_qubits; ++q) t.layout.push_back(q);
    qvdg_plan* plan = new qvdg_plan();
    plan->device_id = dev;
    try {
      const std::vector<HOp> hops = lower_ops(ops, num_ops, num_qubits);
      plan->program = choose_program(t, hops, opt, FusionSearch::Thorough, true, &plan->settings);
      opt = plan->settings;
      plan->program.gates = num_ops;
      upload_plan(plan->program, precision_bits, &plan->device, &plan->dev);
      // Tensor-core plain plans pick their fusion by the cost from |0...0>;
      // the pick for any other state is kept beside it where it differs.
      if (!opt.staged && (opt.math == QVDG_MATH_TENSOR || opt.math == QVDG_MATH_TENSOR_PAIRS) &&
          opt.max_fused_qubits >= 5 && num_qubits >= 13) {
        Program general = build_program(t, hops, opt, FusionSearch::Thorough, false);
        if (general.features != plan->program.features || general.run_layout != plan->program.run_layout) {
          general.gates = num_ops;
          plan->general = std::make_unique<Program>(std::move(general));
          upload_plan(*plan->general, precision_bits, &plan->general_device, &plan->general_dev);
        }
      }
    } catch (...) {
      qvdg_plan_destroy(plan);
      throw;
    }
    *out = plan;
  });
}

qvdg_status qvdg_plan_destroy(qvdg_plan* plan) {
  if (!plan) return QVDG_OK;
  if (plan->device) cudaFree(plan->device);
  if (plan->general_device) cudaFree(plan->general_device);
  delete plan;
  return QVDG_OK;
}

qvdg_status qvdg_plan_info(const qvdg_plan* plan, qvdg_stats* stats) {
  return guarded([&] {
    require(plan != nullptr && stats != nullptr, "null plan or output");
    const Program& p = plan->program;
    stats->gates = p.gates;
    stats->kernels = p.kernels;
    stats->passes = p.passes.size();
    stats->stages = p.stages;
    stats->gate_seconds = 0.0;
    stats->bytes = p.bytes;
    stats->settings = plan->settings;
  });
}

qvdg_status qvdg_plan_execute(qvdg_state* st, const qvdg_plan* plan, qvdg_stats* stats) {
  return guarded([&] {
    StateImpl& s = impl(st);
    require(plan != nullptr, "null plan");
    const Target& t = plan->program.target;
    require(t.n == s.n && t.bits == s.bits, "the plan was made for another state size or precision");
    // A state in another layout is relabelled first (free on |0...0>).
    require(plan->device_id == s.device, "the plan lives on another device");
    if (stats) stats->gates += plan->program.gates;
    if (plan->general && !s.zero_state)
      run_program(s, *plan->general, plan->general_dev, stats);
    else
      run_program(s, plan->program, plan->dev, stats);
    if (stats) stats->settings = plan->settings;
  });
}

qvdg_status qvdg_set_pass_timing(qvdg_state* st, int32_t enabled) {
  return guarded([&] { impl(st).record_passes = enabled != 0; });
}

qvdg_status qvdg_pass_times(const qvdg_state* st, double* seconds, double* bytes, int32_t* staged, size_t capacity,
                            size_t* count) {
  return guarded([&] {
    const StateImpl& s = impl(st);
    const size_t n = s.pass_seconds.size();
    if (count) *count = n;
    for (size_t i = 0; i < n && i < capacity; ++i) {
      if (seconds) seconds[i] = s.pass_seconds[i];
      if (bytes) bytes[i] = s.pass_bytes[i];
      if (staged) staged[i] = s.pass_kinds[i];
    }
  });
}

qvdg_status qvdg_set_device(int32_t device) {
  return guarded([&] { QVDG_CUDA(cudaSetDevice(device)); });
}

qvdg_status qvdg_get_device(int32_t* device) {
  return guarded([&] {
    require(device != nullptr, "null output");
    int d = 0;
    QVDG_CUDA(cudaGetDevice(&d));
    *device = d;
  });
}

qvdg_status qvdg_max_abs_diff(const qvdg_state* a, const qvdg_state* b, double* out) {
  return guarded([&] {
    require(out != nullptr, "null output");
    *out = max_abs_diff(const_cast<StateImpl&>(impl(a)), const_cast<StateImpl&>(impl(b)));
  });
}

qvdg_status qvdg_bit_probabilities_noalloc(const void* amplitudes, uint32_t num_qubits, uint32_t precision_bits,
                                           void* stream, double* p1, double* total) {
  return guarded([&] {
    require(amplitudes != nullptr, "null amplitudes");
    require(p1 != nullptr && total != nullptr, "null output");
    require(num_qubits >= 1, "num_qubits must be at least 1");
    require(precision_bits == 32 || precision_bits == 64, "precision_bits must be 32 or 64");
    bit_probabilities_noalloc(amplitudes, num_qubits, precision_bits, static_cast<cudaStream_t>(stream), p1, total);
  });
}

qvdg_status qvdg_sample_counts(const qvdg_state* st, size_t shots, const double* uniforms,
                               const uint32_t* measure_qubits, const uint32_t* measure_clbits, size_t num_measures,
                               uint64_t* keys, uint64_t* counts, size_t capacity, size_t* num_keys) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(st));
    require(shots == 0 || uniforms != nullptr, "null uniforms");
    require(num_measures == 0 || (measure_qubits != nullptr && measure_clbits != nullptr), "null measurements");
    for (size_t i = 0; i < num_measures; ++i) {
      require(measure_qubits[i] < s.n, "measured qubit out of range");
      require(measure_clbits[i] < 64, "classical bits beyond 63 are not supported by device counting");
    }
    for (size_t i = 0; i < shots; ++i) require(uniforms[i] >= 0.0 && uniforms[i] < 1.0, "uniforms must be in [0, 1)");
    std::vector<uint64_t> k, c;
    sample_counts(s, shots, uniforms, measure_qubits, measure_clbits, num_measures, k, c);
    if (num_keys) *num_keys = k.size();
    if (keys && counts)
      for (size_t i = 0; i < std::min(capacity, k.size()); ++i) {
        keys[i] = k[i];
        counts[i] = c[i];
      }
  });
}

qvdg_status qvdg_expect_pauli(const qvdg_state* st, const uint32_t* qubits, const char* paulis, size_t count,
                              double* out) {
  return guarded([&] {
    StateImpl& s = const_cast<StateImpl&>(impl(st));
    require(out != nullptr, "null output");
    require(count == 0 || (qubits != nullptr && paulis != nullptr), "null Pauli string");
    uint64_t x = 0, z = 0, seen = 0;
    int ny = 0;
    for (size_t i = 0; i < count; ++i) {
      require(qubits[i] < s.n, "qubit out of range");
      const uint64_t bit = uint64_t(1) << s.layout[qubits[i]];
      require(!(seen & bit), "a Pauli string names a qubit twice");
      seen |= bit;
      switch (paulis[i]) {
        case 'X': case 'x': x |= bit; break;
        case 'Z': case 'z': z |= bit; break;
        case 'Y': case 'y': x |= bit; z |= bit; ++ny; break;
        case 'I': case 'i': break;
        default: throw Error(QVDG_ERR_INVALID, std::string("unknown Pauli `") + paulis[i] + "`");
      }
    }
    *out = expect_pauli(s, x, z, ny);
  });
}

qvdg_status qvdg_plan_features(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                               const qvdg_options* options, float* out, size_t capacity, size_t* num_passes) {
  return qvdg_plan_features_from(num_qubits, precision_bits, ops, num_ops, options, 0, out, capacity, num_passes);
}

qvdg_status qvdg_plan_features_from(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                                    const qvdg_options* options, int32_t from_zero, float* out, size_t capacity,
                                    size_t* num_passes) {
  return guarded([&] {
    require(precision_bits == 32 || precision_bits == 64, "precision must be 32 or 64 bits");
    require(num_qubits >= 1 && num_qubits <= 40, "a state needs 1 to 40 qubits");
    qvdg_options opt;
    qvdg_default_options(&opt);
    if (options) opt = *options;
    Target t;
    t.n = num_qubits;
    t.bits = int(precision_bits);
    for (uint32_t q = 0; q < num_qubits; ++q) t.layout.push_back(q);
    // The program for any state, or the one a plan runs from |0...0> (its
    // fusion, layout and pairing; the rows describe whole passes).
    const Program prog =
        build_program(t, lower_ops(ops, num_ops, num_qubits), opt, FusionSearch::Thorough, from_zero != 0);
    const size_t rows = prog.passes.size();
    if (num_passes) *num_passes = rows;
    if (out) std::memcpy(out, prog.features.data(), std::min(rows, capacity) * kPassFeatures * sizeof(float));
  });
}

qvdg_status qvdg_cost_model_set(const float* params, size_t count, uint32_t inputs, uint32_t hidden) {
  return guarded([&] {
    require(params != nullptr, "null parameters");
    int dev = 0;
    QVDG_CUDA(cudaGetDevice(&dev));
    set_cost_model(dev, params, count, inputs, hidden);
  });
}

qvdg_status qvdg_cost_model_clear(void) {
  return guarded([&] {
    int dev = 0;
    QVDG_CUDA(cudaGetDevice(&dev));
    clear_cost_model(dev);
  });
}

qvdg_status qvdg_planner_candidates(uint32_t precision_bits, qvdg_options* out, size_t capacity, size_t* count) {
  return guarded([&] {
    require(precision_bits == 32 || precision_bits == 64, "precision must be 32 or 64 bits");
    const std::vector<qvdg_options> c = learned_candidates(int(precision_bits));
    if (count) *count = c.size();
    for (size_t i = 0; out && i < c.size() && i < capacity; ++i) out[i] = c[i];
  });
}

qvdg_status qvdg_plan_choose(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                             int32_t from_zero, qvdg_options* chosen, double* predicted, size_t capacity,
                             size_t* num_candidates) {
  return guarded([&] {
    require(precision_bits == 32, "the cost model ranks complex64 plans only");
    require(num_qubits >= 1 && num_qubits <= 40, "a state needs 1 to 40 qubits");
    int dev = 0;
    QVDG_CUDA(cudaGetDevice(&dev));
    require(has_cost_model(dev), "no cost model is registered for this device");
    Target t;
    t.n = num_qubits;
    t.bits = int(precision_bits);
    QVDG_CUDA(cudaDeviceGetAttribute(&t.sms, cudaDevAttrMultiProcessorCount, dev));
    for (uint32_t q = 0; q < num_qubits; ++q) t.layout.push_back(q);
    qvdg_options opt;
    qvdg_default_options(&opt);
    opt.planner = QVDG_PLANNER_LEARNED;
    qvdg_options pick;
    std::vector<double> sec;
    choose_program(t, lower_ops(ops, num_ops, num_qubits), opt, FusionSearch::Thorough, from_zero != 0, &pick, &sec);
    if (chosen) *chosen = pick;
    if (num_candidates) *num_candidates = sec.size();
    for (size_t i = 0; predicted && i < sec.size() && i < capacity; ++i) predicted[i] = sec[i];
  });
}

qvdg_status qvdg_plan_fused_ops(uint32_t num_qubits, uint32_t precision_bits, const qvdg_op* ops, size_t num_ops,
                                const qvdg_options* options, int32_t from_zero, uint32_t* num_targets,
                                uint32_t* num_controls, uint32_t* qubits, uint8_t* control_values, double* matrices,
                                size_t capacity, size_t* num_fused, size_t* num_qubit_entries,
                                size_t* num_matrix_doubles) {
  return guarded([&] {
    require(precision_bits == 32 || precision_bits == 64, "precision must be 32 or 64 bits");
    require(num_qubits >= 1 && num_qubits <= 40, "a state needs 1 to 40 qubits");
    qvdg_options opt;
    qvdg_default_options(&opt);
    if (options) opt = *options;
    Target t;
    t.n = num_qubits;
    t.bits = int(precision_bits);
    for (uint32_t q = 0; q < num_qubits; ++q) t.layout.push_back(q);
    std::vector<HOp> fused;
    build_program(t, lower_ops(ops, num_ops, num_qubits), opt, FusionSearch::Thorough, from_zero != 0, &fused);
    size_t nq = 0, nm = 0;
    for (const HOp& f : fused) {
      nq += f.targets.size() + f.controls.size();
      nm += 2 * f.matrix.a.size();
    }
    if (num_fused) *num_fused = fused.size();
    if (num_qubit_entries) *num_qubit_entries = nq;
    if (num_matrix_doubles) *num_matrix_doubles = nm;
    if (fused.empty() || capacity < fused.size()) return;  // sizes only
    require(num_targets && num_controls && qubits && control_values && matrices, "null output array");
    size_t qi = 0, mi = 0;
    for (size_t i = 0; i < fused.size(); ++i) {
      const HOp& f = fused[i];
      num_targets[i] = uint32_t(f.targets.size());
      num_controls[i] = uint32_t(f.controls.size());
      for (uint32_t q : f.targets) {
        qubits[qi] = q;
        control_values[qi++] = 0;
      }
      for (auto& c : f.controls) {
        qubits[qi] = c.first;
        control_values[qi++] = c.second ? 1 : 0;
      }
      for (const C& x : f.matrix.a) {
        matrices[mi++] = x.re;
        matrices[mi++] = x.im;
      }
    }
  });
}

qvdg_status qvdg_mlp_create(uint32_t inputs, uint32_t hidden, uint64_t seed, qvdg_mlp** out) {
  return guarded([&] {
    require(out != nullptr, "null output handle");
    *out = nullptr;
    require(inputs >= 1 && inputs <= 1024 && hidden >= 1 && hidden <= 1024, "inputs and hidden must be 1..1024");
    *out = mlp_create(inputs, hidden, seed);
  });
}

qvdg_status qvdg_mlp_destroy(qvdg_mlp* mlp) {
  return guarded([&] { mlp_destroy(mlp); });
}

qvdg_status qvdg_mlp_num_params(const qvdg_mlp* mlp, size_t* count) {
  return guarded([&] {
    require(mlp != nullptr && count != nullptr, "null argument");
    *count = mlp_num_params(mlp);
  });
}

qvdg_status qvdg_mlp_get_params(const qvdg_mlp* mlp, float* params, size_t count) {
  return guarded([&] {
    require(mlp != nullptr && params != nullptr, "null argument");
    require(count == mlp_num_params(mlp), "expected " + std::to_string(mlp_num_params(mlp)) + " parameters");
    mlp_get_params(mlp, params);
  });
}

qvdg_status qvdg_mlp_set_params(qvdg_mlp* mlp, const float* params, size_t count) {
  return guarded([&] {
    require(mlp != nullptr && params != nullptr, "null argument");
    require(count == mlp_num_params(mlp), "expected " + std::to_string(mlp_num_params(mlp)) + " parameters");
    mlp_set_params(mlp, params);
  });
}

qvdg_status qvdg_mlp_forward(qvdg_mlp* mlp, const float* x, size_t rows, float* y) {
  return guarded([&] {
    require(mlp != nullptr && x != nullptr && y != nullptr, "null argument");
    require(rows >= 1 && rows <= (size_t(1) << 24), "rows must be 1..2^24");
    mlp_forward(mlp, x, rows, y);
  });
}

qvdg_status qvdg_mlp_gradients(qvdg_mlp* mlp, const float* x, const float* target, size_t rows, float* loss,
                               float* grads) {
  return guarded([&] {
    require(mlp != nullptr && x != nullptr && target != nullptr, "null argument");
    require(rows >= 1 && rows <= (size_t(1) << 24), "rows must be 1..2^24");
    const float l = mlp_gradients(mlp, x, target, rows, grads);
    if (loss) *loss = l;
  });
}

qvdg_status qvdg_mlp_train(qvdg_mlp* mlp, const float* x, const float* target, size_t rows, uint32_t epochs,
                           uint32_t batch, float lr, uint64_t seed, float* loss) {
  return guarded([&] {
    require(mlp != nullptr && x != nullptr && target != nullptr, "null argument");
    require(rows >= 1 && rows <= (size_t(1) << 24), "rows must be 1..2^24");
    require(batch >= 1 && batch <= 65535, "batch must be 1..65535");
    const float l = mlp_train(mlp, x, target, rows, epochs, batch, lr, seed);
    if (loss) *loss = l;
  });
}

qvdg_status qvdg_batch_create(const qvdg_layered_circuit* circuits, size_t count, const qvdg_batch_options* options,
                              qvdg_batch** out) {
  return guarded([&] {
    require(out != nullptr, "null output");
    *out = nullptr;
    *out = batch_create(circuits, count, options);
  });
}

qvdg_status qvdg_batch_destroy(qvdg_batch* batch) {
  return guarded([&] { batch_destroy(batch); });
}

qvdg_status qvdg_batch_set_gates(qvdg_batch* batch, const double* gates, size_t num_matrices) {
  return guarded([&] { batch_set_gates(batch, gates, num_matrices); });
}

qvdg_status qvdg_batch_run(qvdg_batch* batch, double* expect_z, size_t count, double* seconds) {
  return guarded([&] { batch_run(batch, expect_z, count, seconds); });
}

qvdg_status qvdg_batch_info(const qvdg_batch* batch, qvdg_batch_summary* info) {
  return guarded([&] { batch_info(batch, info); });
}

qvdg_status qvdg_batch_tuning(const qvdg_batch* batch, uint32_t* tile_qubits, uint32_t* threads, double* seconds,
                              size_t capacity, size_t* count) {
  return guarded([&] {
    const size_t n = batch_tuning(batch, tile_qubits, threads, seconds, capacity);
    if (count) *count = n;
  });
}

}  // extern "C"
