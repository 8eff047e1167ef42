// A planned circuit: the passes of a run (staged tiles or plain gates) with
// their gate programs, built on the host once and uploaded to the device.
#pragma once

#include <vector>

#include "engine.hpp"
#include "host.hpp"
#include "qvdg.h"
#include "stage.hpp"
#include "stage_kernel.hpp"

namespace qvdg {

// What planning needs to know about the target state.
struct Target {
  uint32_t n = 0;
  int bits = 32;
  int sms = 148;
  std::vector<uint32_t> layout;
};

// Per-pass features for the learned cost model (cost_features.cpp): the
// kind of pass, its gates by type and width, where they sit, tile shape.
constexpr int kPassFeatures = 32;

struct Program {
  Target target;                      // the state the program starts from (layout included)
  std::vector<uint32_t> run_layout;   // the layout its passes use, when it relabels first (else empty)
  StageConfig cfg{};
  std::vector<LoweredPass> passes;
  std::vector<double> pass_bytes;  // algorithmic HBM bytes of each pass
  StageUpload upload;              // host copy of the gate programs and matrices
  uint64_t gates = 0, kernels = 0, stages = 0;
  double bytes = 0.0;
  std::vector<float> features;  // kPassFeatures per pass
  // Passes for a run that starts from |0...0>: until every qubit has been
  // in some pass, the amplitudes with an untouched qubit set are zero and
  // stay zero, so pass i (i < zero_passes.size()) may take those qubits as
  // controls that must be 0 and move only 2^-c of the state.
  std::vector<LoweredPass> zero_passes;
  std::vector<double> zero_pass_bytes;
};

void pass_features(const Target& t, const PlannedPass& p, const LoweredPass& lp, const StageUpload& up, float* f);
// Adds the second gate of a pair pass to its first gate's features.
void pair_features(const Target& t, const PlannedPass& second, float* f);

// How hard a tensor-core plain plan searches for fewer passes: the seed
// lookahead fusions only, plus narrow beam searches, or plus wider ones too.
// A plan built once and run many times affords the widest search; a
// one-shot run only where its passes are long enough to pay for it.
enum class FusionSearch { Lookahead, Beam, Thorough };

// `from_zero`: score tensor-core plain candidates by their cost from
// |0...0> (zero-start passes), the usual start of a run; plans built once
// assume it too, and still run on any state.
// `fused` (optional): receives the ops of a plain plan's passes in order,
// on logical qubits (each fused group as its product matrix, or, for a pass
// applied gate by gate, its member gates).
Program build_program(const Target& t, const std::vector<HOp>& ops, const qvdg_options& opt,
                      FusionSearch search, bool from_zero, std::vector<HOp>* fused = nullptr);

// Copy the program's gate data to `dst` on `stream` through the state's
// pinned staging buffer.
DeviceUpload upload_program(StateImpl& s, const Program& p, DeviceScratch& dst);

// Relabel the state to the program's layout (free on a |0...0> state, swap
// passes otherwise), launch every pass on the state's stream and wait; fills stats (device
// time between the first and last launch) and, when the state records pass
// timings, the per-pass device times.
void run_program(StateImpl& s, const Program& p, const DeviceUpload& dev, qvdg_stats* stats);

Target target_of(const StateImpl& s);

}  // namespace qvdg
