//! The `run_on` arm for the B200 engine: the state-vector branch of
//! `run_on` (src/simulator.rs:355-425) with `GpuStateVector` in place of
//! `StateVector<T>`. `run_on` would call it for `Backend::StateVector`
//! when the crate is built with the `gpu` feature (or for a new
//! `Backend::Gpu`).
//!
//! Not compiled here: this image has no Rust toolchain (no cargo or rustc).

use std::collections::BTreeMap;
use std::io;
use std::time::Instant;

use rand::SeedableRng;
use rand_pcg::Pcg64;

use super::{ffi, GpuStateVector};
use crate::circuit::{Circuit, Instruction};
use crate::fusion::Op;
use crate::simd::Real;
use crate::simulator::{bitstring, gate_op, terminal_measurements, Options, RunResult};

/// The cost model the learned planner ranks plans with (the parameters of
/// qevedo_simulator_b200/data/cost_model.npz as f32), registered once per
/// device before the first run; without it the planner falls back to the
/// greedy settings of `options`.
pub fn register_cost_model(params: &[f32], hidden: u32) -> io::Result<()> {
    super::check(unsafe {
        ffi::qvdg_cost_model_set(params.as_ptr(), params.len(), ffi::QVDG_PASS_FEATURES as u32, hidden)
    })
}

pub fn run_on_gpu<T: Real>(circuit: &Circuit, shots: usize, options: &Options) -> io::Result<RunResult> {
    let mut rng = match options.seed {
        Some(seed) => Pcg64::seed_from_u64(seed),
        None => Pcg64::from_rng(&mut rand::rng()),
    };
    let settings = super::gpu_options(options, true);
    let mut result = RunResult::default();
    if let Some(split) = terminal_measurements(circuit) {
        let ops: Vec<Op> = circuit.instructions[..split]
            .iter()
            .filter_map(|i| match i {
                Instruction::Gate { gate, qubits } => Some(gate_op(gate, qubits)),
                _ => None,
            })
            .collect();
        let mut state = GpuStateVector::zero::<T>(circuit.num_qubits)?;
        state.apply_ops(&ops, &settings, &mut result.stats)?;
        let start = Instant::now();
        let measures: Vec<(usize, usize)> = circuit.instructions[split..]
            .iter()
            .filter_map(|i| match i {
                Instruction::Measure { qubit, clbit } => Some((*qubit, *clbit)),
                _ => None,
            })
            .collect();
        if circuit.num_clbits <= 64 {
            // Keys counted on the device; only distinct keys are formatted.
            let mut counts = BTreeMap::new();
            for (key, count) in state.sample_counts(shots, &mut rng, &measures)? {
                let clbits: Vec<bool> = (0..circuit.num_clbits).map(|c| (key >> c) & 1 == 1).collect();
                counts.insert(bitstring(&clbits), count);
            }
            result.counts = counts;
        } else {
            let outcomes = state.sample_unordered(shots, &mut rng)?;
            for index in outcomes {
                let mut clbits = vec![false; circuit.num_clbits];
                for &(q, c) in &measures {
                    clbits[c] = (index >> q) & 1 == 1;
                }
                *result.counts.entry(bitstring(&clbits)).or_default() += 1;
            }
        }
        result.stats.measure_seconds = start.elapsed().as_secs_f64();
        return Ok(result);
    }
    // Shot by shot, one device state reused: zero() keeps the zero-start
    // passes' saving on every shot.
    let mut state = GpuStateVector::zero::<T>(circuit.num_qubits)?;
    for _ in 0..shots {
        state.reset_to_zero()?;
        let mut clbits = vec![false; circuit.num_clbits];
        let mut pending: Vec<Op> = Vec::new();
        for instruction in &circuit.instructions {
            match instruction {
                Instruction::Gate { gate, qubits } => pending.push(gate_op(gate, qubits)),
                Instruction::Barrier { .. } => {}
                Instruction::Measure { qubit, clbit } => {
                    state.apply_ops(&std::mem::take(&mut pending), &settings, &mut result.stats)?;
                    let start = Instant::now();
                    clbits[*clbit] = state.measure(*qubit, &mut rng)?;
                    result.stats.measure_seconds += start.elapsed().as_secs_f64();
                }
                Instruction::Reset { qubit } => {
                    state.apply_ops(&std::mem::take(&mut pending), &settings, &mut result.stats)?;
                    state.reset(*qubit, &mut rng)?;
                }
                &Instruction::Feedback { pauli, qubit, clbit } => {
                    if clbits[clbit] {
                        pending.push(gate_op(&pauli.gate(), &[qubit]));
                    }
                }
                Instruction::Noise { .. } => {
                    return Err(io::Error::other("noise channels do not run on the GPU state vector"));
                }
            }
        }
        state.apply_ops(&pending, &settings, &mut result.stats)?;
        *result.counts.entry(bitstring(&clbits)).or_default() += 1;
    }
    Ok(result)
}
