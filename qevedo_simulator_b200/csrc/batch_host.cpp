// Host side of the batched layered-circuit launch: validation, packing,
// work order, the autotuner, graph capture and replay.

#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <chrono>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "batch.hpp"

struct qvdg_batch {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<qvdg::BatchCircuit> circuits;
  uint64_t num_matrices = 0, outputs = 0;
  uint32_t max_qubits = 0;
  void* dev = nullptr;      // circuits | order | sample order | gates | out | queue
  void* slots = nullptr;    // per-CTA states of wide circuits
  size_t slot_bytes = 0;
  double* host_out = nullptr;  // pinned
  qvdg::BatchLaunch launch;    // the chosen shape, whole batch
  qvdg::BatchLaunch sample;    // the autotuner's sample
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<uint32_t> tune_tiles, tune_threads;
  std::vector<double> tune_seconds;
  double tune_host_seconds = 0.0;
};

namespace qvdg {

namespace {

constexpr int kTileMin = 12, kTileMax = 14;
constexpr int kMaxCtasPerSm = 4;
constexpr size_t kSlotBudget = size_t(24) << 30;

void require(bool ok, const std::string& message) {
  if (!ok) throw Error(QVDG_ERR_INVALID, message);
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Whether a tile shape can run every circuit: wide circuits (n > L) run on
// tiles of L - 1 qubits and need the pass-B tile (high n-L+1 qubits plus
// r >= 1 low ones) to fit, n <= 2(L - 1) - 1.
bool shape_fits(uint32_t max_qubits, int L) { return max_qubits <= uint32_t(L) || max_qubits <= uint32_t(2 * L - 3); }

uint64_t slot_elems_for(uint32_t max_qubits, int L) {
  return max_qubits > uint32_t(L) ? (uint64_t(1) << max_qubits) : 0;
}

// Persistent CTAs for a shape: all resident CTAs (at most kMaxCtasPerSm per
// SM), fewer when the per-CTA slots of wide circuits would exceed the budget.
int ctas_for(const qvdg_batch* b, int threads, int L) {
  const int occ = batch_kernel_occupancy(threads, L);
  if (occ <= 0) return 0;
  int ctas = b->sms * std::min(occ, kMaxCtasPerSm);
  const uint64_t slot = slot_elems_for(b->max_qubits, L) * sizeof(float2);
  if (slot > 0) ctas = int(std::min<uint64_t>(uint64_t(ctas), std::max<uint64_t>(1, kSlotBudget / slot)));
  return ctas;
}

// U = diag(p0, p1) R diag(q0, q1) with R real and unit p, q: rows with one
// common phase (q = 1) or columns with one (p = 1) when possible, otherwise
// p0 = 1 and the rest from U's entries (all four nonzero for a unitary that
// is neither diagonal nor anti-diagonal). False when U has no such form.
bool decompose(const double* m, float2* rec, bool& left, bool& right) {
  using Cd = std::complex<double>;
  const Cd u[4] = {{m[0], m[1]}, {m[2], m[3]}, {m[4], m[5]}, {m[6], m[7]}};
  auto unit = [](Cd c) { return c / std::abs(c); };
  const double tol = 1e-9;
  double r[4];
  Cd p[2] = {1.0, 1.0}, q[2] = {1.0, 1.0};
  auto real_of = [&](Cd c, double& out) {
    if (std::abs(c.imag()) > tol) return false;
    out = c.real();
    return true;
  };
  auto rows = [&]() {
    for (int i = 0; i < 2; ++i) {
      const int k = std::abs(u[2 * i]) >= std::abs(u[2 * i + 1]) ? 0 : 1;
      if (std::abs(u[2 * i + k]) == 0.0) return false;
      p[i] = unit(u[2 * i + k]);
      if (!real_of(u[2 * i] / p[i], r[2 * i]) || !real_of(u[2 * i + 1] / p[i], r[2 * i + 1])) return false;
    }
    q[0] = q[1] = 1.0;
    return true;
  };
  auto cols = [&]() {
    for (int j = 0; j < 2; ++j) {
      const int k = std::abs(u[j]) >= std::abs(u[2 + j]) ? 0 : 1;
      if (std::abs(u[2 * k + j]) == 0.0) return false;
      q[j] = unit(u[2 * k + j]);
      if (!real_of(u[j] / q[j], r[j]) || !real_of(u[2 + j] / q[j], r[2 + j])) return false;
    }
    p[0] = p[1] = 1.0;
    return true;
  };
  auto general = [&]() {
    for (const Cd& c : u)
      if (std::abs(c) == 0.0) return false;
    p[0] = 1.0;
    q[0] = unit(u[0]);
    q[1] = unit(u[1]);
    p[1] = unit(u[2] / q[0]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        if (!real_of(u[2 * i + j] / (p[i] * q[j]), r[2 * i + j])) return false;
    return true;
  };
  if (!rows() && !cols() && !general()) return false;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      if (std::abs(p[i] * r[2 * i + j] * q[j] - u[2 * i + j]) > tol) return false;
  rec[0] = make_float2(float(r[0]), float(r[1]));
  rec[1] = make_float2(float(r[2]), float(r[3]));
  rec[2] = make_float2(float(p[0].real()), float(p[0].imag()));
  rec[3] = make_float2(float(p[1].real()), float(p[1].imag()));
  rec[4] = make_float2(float(q[0].real()), float(q[0].imag()));
  rec[5] = make_float2(float(q[1].real()), float(q[1].imag()));
  left = left || p[0] != Cd(1.0) || p[1] != Cd(1.0);
  right = right || q[0] != Cd(1.0) || q[1] != Cd(1.0);
  return true;
}

// A circuit's gate records (kBatchGateSlots complex64 per matrix) and its
// form: phased when every matrix decomposes, else the generic matrices.
uint32_t encode_gates(const double* src, size_t num_matrices, float2* dst) {
  bool left = false, right = false, phased = true;
  for (size_t i = 0; i < num_matrices && phased; ++i)
    phased = decompose(src + 8 * i, dst + kBatchGateSlots * i, left, right);
  if (phased) return kBatchPhased | (left ? kBatchLeft : 0u) | (right ? kBatchRight : 0u);
  for (size_t i = 0; i < num_matrices; ++i)
    for (int k = 0; k < kBatchGateSlots; ++k)
      dst[kBatchGateSlots * i + k] =
          k < 4 ? make_float2(float(src[8 * i + 2 * k]), float(src[8 * i + 2 * k + 1])) : make_float2(0.f, 0.f);
  return 0;
}

BatchLaunch shape(const BatchLaunch& base, int L, int threads, int ctas, uint32_t max_qubits) {
  BatchLaunch l = base;
  l.tile_qubits = L;
  l.threads = threads;
  l.ctas = ctas;
  l.slot_elems = slot_elems_for(max_qubits, L);
  return l;
}

double time_launch(qvdg_batch* b, const BatchLaunch& l) {
  launch_batch(l, b->stream);  // warm
  QVDG_CUDA(cudaEventRecord(b->ev0, b->stream));
  launch_batch(l, b->stream);
  QVDG_CUDA(cudaEventRecord(b->ev1, b->stream));
  QVDG_CUDA(cudaEventSynchronize(b->ev1));
  float ms = 0.f;
  QVDG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  return ms * 1e-3;
}

void release(qvdg_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->dev) cudaFree(b->dev);
  if (b->slots) cudaFree(b->slots);
  if (b->host_out) cudaFreeHost(b->host_out);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

qvdg_batch* batch_create(const qvdg_layered_circuit* circuits, size_t count, const qvdg_batch_options* options) {
  require(circuits != nullptr && count > 0, "empty batch");
  require(count < (size_t(1) << 31), "too many circuits");
  uint32_t want_tile = options ? options->tile_qubits : 0, want_threads = options ? options->threads : 0;
  require(want_tile == 0 || (want_tile >= uint32_t(kTileMin) && want_tile <= uint32_t(kTileMax)),
          "tile_qubits must be 0 or 12..14");
  require(want_threads == 0 || want_threads == 128 || want_threads == 256 || want_threads == 512,
          "threads must be 0, 128, 256 or 512");
  auto* b = new qvdg_batch();
  try {
    // Validate and pack.
    b->circuits.resize(count);
    for (size_t i = 0; i < count; ++i) {
      const qvdg_layered_circuit& c = circuits[i];
      require(c.num_qubits >= 1 && c.num_qubits <= uint32_t(kBatchMaxQubits),
              "circuit " + std::to_string(i) + ": num_qubits must be 1.." + std::to_string(kBatchMaxQubits));
      require(c.entangler <= QVDG_ENTANGLE_CZ_LADDER, "circuit " + std::to_string(i) + ": unknown entangler");
      require(c.num_layers == 0 || c.gates != nullptr, "circuit " + std::to_string(i) + ": null gates");
      BatchCircuit& d = b->circuits[i];
      d.num_qubits = c.num_qubits;
      d.num_layers = c.num_layers;
      d.entangler = c.entangler;
      d.form = 0;
      d.gates = b->num_matrices;
      d.out = b->outputs;
      b->num_matrices += uint64_t(c.num_layers) * c.num_qubits;
      b->outputs += c.num_qubits;
      b->max_qubits = std::max(b->max_qubits, c.num_qubits);
    }
    if (want_tile) require(shape_fits(b->max_qubits, int(want_tile)), "tile_qubits too small for the widest circuit");
    std::vector<float2> gates(b->num_matrices * kBatchGateSlots);
    for (size_t i = 0; i < count; ++i)
      b->circuits[i].form = encode_gates(circuits[i].gates, size_t(circuits[i].num_layers) * circuits[i].num_qubits,
                                         gates.data() + kBatchGateSlots * b->circuits[i].gates);
    // Largest first: an atomic counter then hands out work longest-first.
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    auto cost = [&](uint32_t i) {
      const BatchCircuit& c = b->circuits[i];
      return double(uint64_t(1) << c.num_qubits) * double(c.num_layers + 1) * double(c.num_qubits);
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return cost(x) > cost(y); });
    std::vector<uint32_t> sample;
    const size_t stride = count >= 64 ? 8 : 1;
    for (size_t i = 0; i < count; i += stride) sample.push_back(order[i]);

    QVDG_CUDA(cudaGetDevice(&b->device));
    QVDG_CUDA(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    QVDG_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    QVDG_CUDA(cudaEventCreate(&b->ev0));
    QVDG_CUDA(cudaEventCreate(&b->ev1));
    const size_t o_circ = 0;
    const size_t o_order = align256(o_circ + count * sizeof(BatchCircuit));
    const size_t o_sample = align256(o_order + count * sizeof(uint32_t));
    const size_t o_gates = align256(o_sample + sample.size() * sizeof(uint32_t));
    const size_t o_out = align256(o_gates + std::max<size_t>(gates.size(), 1) * sizeof(float2));
    const size_t o_queue = align256(o_out + b->outputs * sizeof(double));
    const size_t total = o_queue + 256;
    QVDG_CUDA(cudaMalloc(&b->dev, total));
    char* base = static_cast<char*>(b->dev);
    QVDG_CUDA(cudaMemcpy(base + o_circ, b->circuits.data(), count * sizeof(BatchCircuit), cudaMemcpyHostToDevice));
    QVDG_CUDA(cudaMemcpy(base + o_order, order.data(), count * sizeof(uint32_t), cudaMemcpyHostToDevice));
    QVDG_CUDA(cudaMemcpy(base + o_sample, sample.data(), sample.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (!gates.empty())
      QVDG_CUDA(cudaMemcpy(base + o_gates, gates.data(), gates.size() * sizeof(float2), cudaMemcpyHostToDevice));
    QVDG_CUDA(cudaMallocHost(&b->host_out, std::max<uint64_t>(b->outputs, 1) * sizeof(double)));

    BatchLaunch whole;
    whole.circuits = reinterpret_cast<const BatchCircuit*>(base + o_circ);
    whole.order = reinterpret_cast<const uint32_t*>(base + o_order);
    whole.count = uint32_t(count);
    whole.gates = reinterpret_cast<const float2*>(base + o_gates);
    whole.out = reinterpret_cast<double*>(base + o_out);
    whole.queue = reinterpret_cast<uint32_t*>(base + o_queue);
    BatchLaunch samp = whole;
    samp.order = reinterpret_cast<const uint32_t*>(base + o_sample);
    samp.count = uint32_t(sample.size());

    // Candidate shapes.
    struct Shape {
      int L, threads, ctas;
    };
    std::vector<Shape> shapes;
    for (int L = kTileMin; L <= kTileMax; ++L)
      for (int t : {128, 256, 512}) {
        if (want_tile && L != int(want_tile)) continue;
        if (want_threads && t != int(want_threads)) continue;
        if (!shape_fits(b->max_qubits, L)) continue;
        const int ctas = ctas_for(b, t, L);
        if (ctas > 0) shapes.push_back({L, t, ctas});
      }
    if (shapes.empty()) throw Error(QVDG_ERR_UNSUPPORTED, "no tile shape can run this batch on this device");
    size_t slot_need = 0;
    for (const Shape& s : shapes)
      slot_need = std::max<size_t>(slot_need, size_t(s.ctas) * slot_elems_for(b->max_qubits, s.L) * sizeof(float2));
    if (slot_need) {
      QVDG_CUDA(cudaMalloc(&b->slots, slot_need));
      b->slot_bytes = slot_need;
    }
    whole.slots = static_cast<float2*>(b->slots);
    samp.slots = whole.slots;

    Shape best = shapes[0];
    if (shapes.size() > 1) {
      const auto t0 = std::chrono::steady_clock::now();
      double best_s = 1e300;
      for (const Shape& s : shapes) {
        const double sec = time_launch(b, shape(samp, s.L, s.threads, s.ctas, b->max_qubits));
        b->tune_tiles.push_back(uint32_t(s.L));
        b->tune_threads.push_back(uint32_t(s.threads));
        b->tune_seconds.push_back(sec);
        if (sec < best_s) {
          best_s = sec;
          best = s;
        }
      }
      b->tune_host_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    b->launch = shape(whole, best.L, best.threads, best.ctas, b->max_qubits);
    b->sample = shape(samp, best.L, best.threads, best.ctas, b->max_qubits);

    // Capture: reset the counter, the persistent launch, results to pinned host memory.
    QVDG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    launch_batch(b->launch, b->stream);
    QVDG_CUDA(cudaMemcpyAsync(b->host_out, b->launch.out, b->outputs * sizeof(double), cudaMemcpyDeviceToHost,
                              b->stream));
    QVDG_CUDA(cudaStreamEndCapture(b->stream, &b->graph));
    QVDG_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return b;
  } catch (...) {
    cudaStreamCaptureStatus st;
    if (b->stream && cudaStreamIsCapturing(b->stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(b->stream, &g);
      if (g) cudaGraphDestroy(g);
    }
    cudaGetLastError();
    release(b);
    delete b;
    throw;
  }
}

void batch_destroy(qvdg_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  release(b);
  delete b;
}

void batch_set_gates(qvdg_batch* b, const double* gates, size_t num_matrices) {
  require(b != nullptr, "null batch");
  require(num_matrices == b->num_matrices, "expected " + std::to_string(b->num_matrices) + " matrices");
  require(gates != nullptr || num_matrices == 0, "null gates");
  if (num_matrices == 0) return;
  // Each circuit's records and form (the form follows the new matrices).
  std::vector<float2> g(num_matrices * kBatchGateSlots);
  for (BatchCircuit& c : b->circuits)
    c.form = encode_gates(gates + 8 * c.gates, size_t(c.num_layers) * c.num_qubits, g.data() + kBatchGateSlots * c.gates);
  QVDG_CUDA(cudaSetDevice(b->device));
  QVDG_CUDA(cudaStreamSynchronize(b->stream));
  QVDG_CUDA(cudaMemcpy(const_cast<float2*>(b->launch.gates), g.data(), g.size() * sizeof(float2),
                       cudaMemcpyHostToDevice));
  QVDG_CUDA(cudaMemcpy(const_cast<BatchCircuit*>(b->launch.circuits), b->circuits.data(),
                       b->circuits.size() * sizeof(BatchCircuit), cudaMemcpyHostToDevice));
}

void batch_run(qvdg_batch* b, double* expect_z, size_t count, double* seconds) {
  require(b != nullptr, "null batch");
  require(expect_z != nullptr, "null output");
  require(count >= b->outputs, "output holds " + std::to_string(count) + " values, the batch has " +
                                   std::to_string(b->outputs));
  QVDG_CUDA(cudaSetDevice(b->device));
  QVDG_CUDA(cudaEventRecord(b->ev0, b->stream));
  QVDG_CUDA(cudaGraphLaunch(b->exec, b->stream));
  QVDG_CUDA(cudaEventRecord(b->ev1, b->stream));
  QVDG_CUDA(cudaEventSynchronize(b->ev1));
  QVDG_CUDA(cudaGetLastError());
  float ms = 0.f;
  QVDG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  if (seconds) *seconds = ms * 1e-3;
  std::memcpy(expect_z, b->host_out, b->outputs * sizeof(double));
}

void batch_info(const qvdg_batch* b, qvdg_batch_summary* info) {
  require(b != nullptr && info != nullptr, "null argument");
  info->tile_qubits = uint32_t(b->launch.tile_qubits);
  info->threads = uint32_t(b->launch.threads);
  info->ctas = uint32_t(b->launch.ctas);
  info->candidates = uint32_t(b->tune_seconds.size());
  info->circuits = b->circuits.size();
  info->outputs = b->outputs;
  info->tune_seconds = b->tune_host_seconds;
}

size_t batch_tuning(const qvdg_batch* b, uint32_t* tile_qubits, uint32_t* threads, double* seconds,
                    size_t capacity) {
  require(b != nullptr, "null batch");
  const size_t n = b->tune_seconds.size();
  for (size_t i = 0; i < std::min(n, capacity); ++i) {
    if (tile_qubits) tile_qubits[i] = b->tune_tiles[i];
    if (threads) threads[i] = b->tune_threads[i];
    if (seconds) seconds[i] = b->tune_seconds[i];
  }
  return n;
}

}  // namespace qvdg
