//! Raw bindings of `libqvdgpu.so` (include/qvdg.h), to be added to the qvd
//! crate as `src/gpu/ffi.rs`.
//!
//! Not compiled here: this image has no Rust toolchain (no cargo or rustc).
//! Every function and struct of include/qvdg.h is mirrored one to one;
//! tests/test_abi.py checks that the library exports each of them.

#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_double, c_float, c_int, c_void};

/// 0 = QVDG_OK; 1 invalid argument; 2 out of memory; 3 CUDA error;
/// 4 unsupported; 5 a bounded device wait gave up.
pub type qvdg_status = c_int;

#[repr(C)]
pub struct qvdg_state {
    _private: [u8; 0],
}
#[repr(C)]
pub struct qvdg_plan {
    _private: [u8; 0],
}
#[repr(C)]
pub struct qvdg_mlp {
    _private: [u8; 0],
}
#[repr(C)]
pub struct qvdg_batch {
    _private: [u8; 0],
}

/// One gate: a 2^k x 2^k complex matrix (interleaved re/im doubles,
/// row-major, index bit j = targets[j]) conditioned on its controls.
#[repr(C)]
pub struct qvdg_op {
    pub num_targets: u32,
    pub num_controls: u32,
    pub targets: *const u32,
    pub controls: *const u32,
    pub control_values: *const u8,
    pub matrix: *const c_double,
}

pub const QVDG_PLANNER_GREEDY: u32 = 0;
pub const QVDG_PLANNER_LEARNED: u32 = 1;
pub const QVDG_MATH_FP32: u32 = 0;
pub const QVDG_MATH_TENSOR: u32 = 1;
pub const QVDG_MATH_GATES: u32 = 2;
pub const QVDG_PASS_FEATURES: usize = 32;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq, Eq)]
pub struct qvdg_options {
    pub max_fused_qubits: u32,
    pub staged: u32,
    pub tile_qubits: u32,
    pub planner: u32,
    pub math: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct qvdg_stats {
    pub gates: u64,
    pub kernels: u64,
    pub passes: u64,
    pub stages: u64,
    pub gate_seconds: c_double,
    pub bytes: c_double,
    pub settings: qvdg_options,
}

#[repr(C)]
pub struct qvdg_layered_circuit {
    pub num_qubits: u32,
    pub num_layers: u32,
    pub entangler: u32,
    pub reserved: u32,
    pub gates: *const c_double,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct qvdg_batch_options {
    pub tile_qubits: u32,
    pub threads: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct qvdg_batch_summary {
    pub tile_qubits: u32,
    pub threads: u32,
    pub ctas: u32,
    pub candidates: u32,
    pub circuits: u64,
    pub outputs: u64,
    pub tune_seconds: c_double,
}

#[link(name = "qvdgpu")]
extern "C" {
    pub fn qvdg_default_options(opt: *mut qvdg_options);
    pub fn qvdg_last_error() -> *const c_char;
    pub fn qvdg_version() -> *const c_char;

    // State vectors (src/state.rs, src/measure.rs).
    pub fn qvdg_state_create(num_qubits: u32, precision_bits: u32, out: *mut *mut qvdg_state) -> qvdg_status;
    pub fn qvdg_state_destroy(state: *mut qvdg_state) -> qvdg_status;
    pub fn qvdg_state_zero(state: *mut qvdg_state) -> qvdg_status;
    pub fn qvdg_state_info(state: *const qvdg_state, num_qubits: *mut u32, precision_bits: *mut u32)
        -> qvdg_status;
    pub fn qvdg_state_set_amplitudes(state: *mut qvdg_state, amplitudes: *const c_double, count: usize)
        -> qvdg_status;
    pub fn qvdg_state_get_amplitudes(state: *const qvdg_state, amplitudes: *mut c_double, count: usize)
        -> qvdg_status;
    pub fn qvdg_apply_ops(state: *mut qvdg_state, ops: *const qvdg_op, num_ops: usize,
                          options: *const qvdg_options, stats: *mut qvdg_stats) -> qvdg_status;
    pub fn qvdg_apply(state: *mut qvdg_state, matrix: *const c_double, qubits: *const u32, num_qubits: u32,
                      controls: *const u32, control_values: *const u8, num_controls: u32) -> qvdg_status;
    pub fn qvdg_norm_sqr(state: *const qvdg_state, out: *mut c_double) -> qvdg_status;
    pub fn qvdg_scale(state: *mut qvdg_state, factor: c_double) -> qvdg_status;
    pub fn qvdg_probability_one(state: *const qvdg_state, qubit: u32, out: *mut c_double) -> qvdg_status;
    pub fn qvdg_expect_z_all(state: *const qvdg_state, out: *mut c_double) -> qvdg_status;
    pub fn qvdg_probabilities(state: *const qvdg_state, out: *mut c_double, count: usize) -> qvdg_status;
    pub fn qvdg_measure(state: *mut qvdg_state, qubit: u32, uniform: c_double, outcome: *mut i32) -> qvdg_status;
    pub fn qvdg_reset(state: *mut qvdg_state, qubit: u32, uniform: c_double) -> qvdg_status;
    pub fn qvdg_sample_unordered(state: *const qvdg_state, shots: usize, uniforms: *const c_double,
                                 out: *mut u64, count: *mut usize) -> qvdg_status;
    pub fn qvdg_sample_counts(state: *const qvdg_state, shots: usize, uniforms: *const c_double,
                              measure_qubits: *const u32, measure_clbits: *const u32, num_measures: usize,
                              keys: *mut u64, counts: *mut u64, capacity: usize, num_keys: *mut usize)
        -> qvdg_status;
    pub fn qvdg_expect_pauli(state: *const qvdg_state, qubits: *const u32, paulis: *const c_char, count: usize,
                             out: *mut c_double) -> qvdg_status;
    pub fn qvdg_swap_physical(state: *mut qvdg_state, pairs: *const u32, num_pairs: u32) -> qvdg_status;
    pub fn qvdg_state_layout(state: *const qvdg_state, layout: *mut u32) -> qvdg_status;
    pub fn qvdg_state_device_buffer(state: *const qvdg_state, pointer: *mut *mut c_void, bytes: *mut usize)
        -> qvdg_status;
    pub fn qvdg_synchronize(state: *const qvdg_state) -> qvdg_status;
    pub fn qvdg_max_abs_diff(a: *const qvdg_state, b: *const qvdg_state, out: *mut c_double) -> qvdg_status;

    // Reusable plans (the planning half of apply_ops, src/simulator.rs:122-147).
    pub fn qvdg_plan_create(num_qubits: u32, precision_bits: u32, ops: *const qvdg_op, num_ops: usize,
                            options: *const qvdg_options, out: *mut *mut qvdg_plan) -> qvdg_status;
    pub fn qvdg_plan_destroy(plan: *mut qvdg_plan) -> qvdg_status;
    pub fn qvdg_plan_info(plan: *const qvdg_plan, stats: *mut qvdg_stats) -> qvdg_status;
    pub fn qvdg_plan_execute(state: *mut qvdg_state, plan: *const qvdg_plan, stats: *mut qvdg_stats)
        -> qvdg_status;
    pub fn qvdg_plan_features(num_qubits: u32, precision_bits: u32, ops: *const qvdg_op, num_ops: usize,
                              options: *const qvdg_options, out: *mut c_float, capacity: usize,
                              num_passes: *mut usize) -> qvdg_status;
    pub fn qvdg_plan_features_from(num_qubits: u32, precision_bits: u32, ops: *const qvdg_op, num_ops: usize,
                                   options: *const qvdg_options, from_zero: i32, out: *mut c_float,
                                   capacity: usize, num_passes: *mut usize) -> qvdg_status;
    pub fn qvdg_plan_fused_ops(num_qubits: u32, precision_bits: u32, ops: *const qvdg_op, num_ops: usize,
                               options: *const qvdg_options, from_zero: i32, num_targets: *mut u32,
                               num_controls: *mut u32, qubits: *mut u32, control_values: *mut u8,
                               matrices: *mut c_double, capacity: usize, num_fused: *mut usize,
                               num_qubit_entries: *mut usize, num_matrix_doubles: *mut usize) -> qvdg_status;

    // The learned planner and its network.
    pub fn qvdg_cost_model_set(params: *const c_float, count: usize, inputs: u32, hidden: u32) -> qvdg_status;
    pub fn qvdg_cost_model_clear() -> qvdg_status;
    pub fn qvdg_planner_candidates(precision_bits: u32, out: *mut qvdg_options, capacity: usize,
                                   count: *mut usize) -> qvdg_status;
    pub fn qvdg_plan_choose(num_qubits: u32, precision_bits: u32, ops: *const qvdg_op, num_ops: usize,
                            from_zero: i32, chosen: *mut qvdg_options, predicted: *mut c_double,
                            capacity: usize, num_candidates: *mut usize) -> qvdg_status;
    pub fn qvdg_mlp_create(inputs: u32, hidden: u32, seed: u64, out: *mut *mut qvdg_mlp) -> qvdg_status;
    pub fn qvdg_mlp_destroy(mlp: *mut qvdg_mlp) -> qvdg_status;
    pub fn qvdg_mlp_num_params(mlp: *const qvdg_mlp, count: *mut usize) -> qvdg_status;
    pub fn qvdg_mlp_get_params(mlp: *const qvdg_mlp, params: *mut c_float, count: usize) -> qvdg_status;
    pub fn qvdg_mlp_set_params(mlp: *mut qvdg_mlp, params: *const c_float, count: usize) -> qvdg_status;
    pub fn qvdg_mlp_forward(mlp: *mut qvdg_mlp, x: *const c_float, rows: usize, y: *mut c_float) -> qvdg_status;
    pub fn qvdg_mlp_gradients(mlp: *mut qvdg_mlp, x: *const c_float, target: *const c_float, rows: usize,
                              loss: *mut c_float, grads: *mut c_float) -> qvdg_status;
    pub fn qvdg_mlp_train(mlp: *mut qvdg_mlp, x: *const c_float, target: *const c_float, rows: usize,
                          epochs: u32, batch: u32, lr: c_float, seed: u64, loss: *mut c_float) -> qvdg_status;

    // Batched layered circuits in one persistent, graph-captured launch.
    pub fn qvdg_batch_create(circuits: *const qvdg_layered_circuit, count: usize,
                             options: *const qvdg_batch_options, out: *mut *mut qvdg_batch) -> qvdg_status;
    pub fn qvdg_batch_destroy(batch: *mut qvdg_batch) -> qvdg_status;
    pub fn qvdg_batch_set_gates(batch: *mut qvdg_batch, gates: *const c_double, num_matrices: usize)
        -> qvdg_status;
    pub fn qvdg_batch_run(batch: *mut qvdg_batch, expect_z: *mut c_double, count: usize, seconds: *mut c_double)
        -> qvdg_status;
    pub fn qvdg_batch_info(batch: *const qvdg_batch, info: *mut qvdg_batch_summary) -> qvdg_status;
    pub fn qvdg_batch_tuning(batch: *const qvdg_batch, tile_qubits: *mut u32, threads: *mut u32,
                             seconds: *mut c_double, capacity: usize, count: *mut usize) -> qvdg_status;

    // Timing, devices, and the allocation-free per-qubit probabilities.
    pub fn qvdg_set_pass_timing(state: *mut qvdg_state, enabled: i32) -> qvdg_status;
    pub fn qvdg_pass_times(state: *const qvdg_state, seconds: *mut c_double, bytes: *mut c_double,
                           staged: *mut i32, capacity: usize, count: *mut usize) -> qvdg_status;
    pub fn qvdg_set_device(device: i32) -> qvdg_status;
    pub fn qvdg_get_device(device: *mut i32) -> qvdg_status;
    pub fn qvdg_bit_probabilities_noalloc(amplitudes: *const c_void, num_qubits: u32, precision_bits: u32,
                                          stream: *mut c_void, p1: *mut c_double, total: *mut c_double)
        -> qvdg_status;
}
