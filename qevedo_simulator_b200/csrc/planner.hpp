// The learned planner: candidate settings built on host threads, ranked by
// the cost model's predicted device time (planner.cpp).
#pragma once

#include <vector>

#include "program.hpp"

namespace qvdg {

// The settings the learned planner chooses among, for a state precision.
std::vector<qvdg_options> learned_candidates(int bits);

// Registers (or replaces) the cost model of `device`: an MLP of the mlp.cu
// form with kPassFeatures inputs and `hidden` units per hidden layer.
void set_cost_model(int device, const float* params, size_t count, uint32_t inputs, uint32_t hidden);
void clear_cost_model(int device);
bool has_cost_model(int device);

// Predicted device seconds of each program (the sum over its passes; with
// `from_zero`, zero-start passes at the share of the state they move).
std::vector<double> predict_programs(int device, const std::vector<const Program*>& progs, bool from_zero);

// With given.planner == QVDG_PLANNER_LEARNED, a complex64 target and a model
// registered for the current device: the candidate program with the least
// predicted time. Otherwise the program of the given settings. `chosen`
// receives the settings of the returned program, `predicted` each
// candidate's predicted seconds (empty when no model ranked them).
Program choose_program(const Target& t, const std::vector<HOp>& ops, const qvdg_options& given, FusionSearch search,
                       bool from_zero, qvdg_options* chosen = nullptr, std::vector<double>* predicted = nullptr);

}  // namespace qvdg
