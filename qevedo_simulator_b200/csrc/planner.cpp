// The learned planner (QVDG_PLANNER_LEARNED): among the candidate settings
// (fusion width, plain or staged passes, CUDA-core, gate-by-gate or
// tensor-core arithmetic) it builds every candidate's program on host
// threads, predicts each pass's device time with the cost model's MLP (the
// mlp.cu kernels, one forward over all candidates' passes), and runs the
// candidate with the least predicted time.
//
// The reference has no learned planner: its apply_ops always fuses greedily
// to max_fused_qubits and cache-blocks with region_bits
// (src/simulator.rs:37-66, :122-147). Here those greedy rules still build
// every candidate; the model only ranks them. Without a registered model,
// or for complex128 states (the model is trained on complex64 pass
// timings), the caller's own settings run, as the greedy planner does.

#include <cuda_runtime.h>

#include <cmath>
#include <limits>
#include <map>
#include <memory>
#include <mutex>

#include "planner.hpp"

namespace qvdg {

namespace {

struct Model {
  qvdg_mlp* mlp = nullptr;
  std::mutex run;  // one forward at a time on the network's buffers
  ~Model() {
    if (mlp) mlp_destroy(mlp);
  }
};

std::mutex g_models_mutex;
std::map<int, std::shared_ptr<Model>> g_models;  // per device

std::shared_ptr<Model> model_for(int device) {
  std::lock_guard<std::mutex> lock(g_models_mutex);
  auto it = g_models.find(device);
  return it == g_models.end() ? nullptr : it->second;
}

qvdg_options make(uint32_t fused, uint32_t staged, uint32_t math) {
  qvdg_options o;
  qvdg_default_options(&o);
  o.max_fused_qubits = fused;
  o.staged = staged;
  o.math = math;
  o.planner = QVDG_PLANNER_GREEDY;
  return o;
}

}  // namespace

std::vector<qvdg_options> learned_candidates(int bits) {
  std::vector<qvdg_options> c;
  for (uint32_t f = 2; f <= 5; ++f) c.push_back(make(f, 0, QVDG_MATH_FP32));
  for (uint32_t f = 4; f <= 5; ++f) c.push_back(make(f, 0, QVDG_MATH_GATES));
  if (bits == 32) {
    for (uint32_t f = 4; f <= 6; ++f) c.push_back(make(f, 0, QVDG_MATH_TENSOR));
    c.push_back(make(6, 0, QVDG_MATH_TENSOR_PAIRS));
  }
  c.push_back(make(4, 1, QVDG_MATH_FP32));
  if (bits == 32)
    for (uint32_t f = 4; f <= 5; ++f) c.push_back(make(f, 1, QVDG_MATH_TENSOR));
  return c;
}

void set_cost_model(int device, const float* params, size_t count, uint32_t inputs, uint32_t hidden) {
  if (inputs != uint32_t(kPassFeatures))
    throw Error(QVDG_ERR_INVALID, "the cost model takes " + std::to_string(kPassFeatures) + " features per pass");
  if (hidden == 0 || hidden > 4096) throw Error(QVDG_ERR_INVALID, "hidden width must be 1 to 4096");
  auto m = std::make_shared<Model>();
  m->mlp = mlp_create(inputs, hidden, 0);
  if (count != mlp_num_params(m->mlp))
    throw Error(QVDG_ERR_INVALID, "expected " + std::to_string(mlp_num_params(m->mlp)) + " parameters");
  mlp_set_params(m->mlp, params);
  std::lock_guard<std::mutex> lock(g_models_mutex);
  g_models[device] = std::move(m);
}

void clear_cost_model(int device) {
  std::lock_guard<std::mutex> lock(g_models_mutex);
  g_models.erase(device);
}

bool has_cost_model(int device) { return model_for(device) != nullptr; }

std::vector<double> predict_programs(int device, const std::vector<const Program*>& progs, bool from_zero) {
  std::shared_ptr<Model> m = model_for(device);
  if (!m) throw Error(QVDG_ERR_INVALID, "no cost model is registered for this device");
  std::vector<size_t> first(progs.size() + 1, 0);
  for (size_t i = 0; i < progs.size(); ++i) first[i + 1] = first[i] + progs[i]->passes.size();
  std::vector<float> x(std::max<size_t>(first.back(), 1) * kPassFeatures, 0.f), y(std::max<size_t>(first.back(), 1));
  for (size_t i = 0; i < progs.size(); ++i)
    std::copy(progs[i]->features.begin(), progs[i]->features.end(), x.begin() + first[i] * kPassFeatures);
  if (first.back() > 0) {
    std::lock_guard<std::mutex> lock(m->run);
    mlp_forward(m->mlp, x.data(), first.back(), y.data());
  }
  std::vector<double> seconds(progs.size(), 0.0);
  for (size_t i = 0; i < progs.size(); ++i) {
    const Program& p = *progs[i];
    const double scale = std::ldexp(1.0, int(p.target.n) - 24);
    for (size_t j = 0; j < p.passes.size(); ++j) {
      double t = std::exp(double(y[first[i] + j])) * scale;
      // A zero-start pass moves its share of the state.
      if (from_zero && j < p.zero_passes.size() && p.pass_bytes[j] > 0)
        t *= p.zero_pass_bytes[j] / p.pass_bytes[j];
      seconds[i] += t;
    }
  }
  return seconds;
}

Program choose_program(const Target& t, const std::vector<HOp>& ops, const qvdg_options& given, FusionSearch search,
                       bool from_zero, qvdg_options* chosen, std::vector<double>* predicted) {
  int device = 0;
  QVDG_CUDA(cudaGetDevice(&device));
  if (given.planner != QVDG_PLANNER_LEARNED || t.bits != 32 || !has_cost_model(device)) {
    if (chosen) {
      *chosen = given;
      chosen->planner = QVDG_PLANNER_GREEDY;
    }
    if (predicted) predicted->clear();
    qvdg_options o = given;
    o.planner = QVDG_PLANNER_GREEDY;
    return build_program(t, ops, o, search, from_zero);
  }
  const std::vector<qvdg_options> cands = learned_candidates(t.bits);
  std::vector<Program> progs(cands.size());
  parallel_for(cands.size(), [&](size_t i) { progs[i] = build_program(t, ops, cands[i], search, from_zero); });
  std::vector<const Program*> ptrs;
  for (const Program& p : progs) ptrs.push_back(&p);
  const std::vector<double> sec = predict_programs(device, ptrs, from_zero);
  size_t best = 0;
  for (size_t i = 1; i < sec.size(); ++i)
    if (sec[i] < sec[best]) best = i;
  if (chosen) *chosen = cands[best];
  if (predicted) *predicted = sec;
  return std::move(progs[best]);
}

}  // namespace qvdg
