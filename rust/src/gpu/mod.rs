//! The B200 state-vector engine behind the qvd crate's `StateVector<T>`
//! methods, to be added as `src/gpu/mod.rs` (with `ffi.rs` beside it and
//! `run.rs` for the `run_on` arm).
//!
//! Not compiled here: this image has no Rust toolchain (no cargo or rustc).
//! The calls it makes are the C ABI of include/qvdg.h, exercised from
//! Python through ctypes by this repository's tests.
//!
//! Errors come back as `io::Error`, as the reference's allocation failures
//! do (src/memory.rs:121-123); invalid ops, which the reference catches
//! with `assert!`, are QVDG_ERR_INVALID here and also become `io::Error`.

pub mod ffi;
pub mod run;

use std::ffi::CStr;
use std::io;

use rand::Rng;

use crate::fusion::Op;
use crate::matrix::C64;
use crate::simd::Real;
use crate::simulator::{Options, Stats};

fn check(status: ffi::qvdg_status) -> io::Result<()> {
    if status == 0 {
        return Ok(());
    }
    let message = unsafe { CStr::from_ptr(ffi::qvdg_last_error()) }.to_string_lossy().into_owned();
    Err(io::Error::other(message))
}

/// The reference's `Options` as the engine's: fusion width and cache
/// blocking map onto max_fused_qubits and staged tiles (region_bits = None
/// is one pass per fused gate); the learned planner may pick another plan
/// when `learned` is set and the state is complex64.
pub fn gpu_options(options: &Options, learned: bool) -> ffi::qvdg_options {
    let mut o = ffi::qvdg_options::default();
    unsafe { ffi::qvdg_default_options(&mut o) };
    o.max_fused_qubits = options.max_fused_qubits.clamp(1, 6) as u32;
    o.staged = options.region_bits.is_some() as u32;
    o.planner = if learned { ffi::QVDG_PLANNER_LEARNED } else { ffi::QVDG_PLANNER_GREEDY };
    o
}

/// Ops flattened into the arrays a `qvdg_op` array points into; the
/// `qvdg_op`s are valid while this value lives.
struct PackedOps {
    qubits: Vec<u32>,
    values: Vec<u8>,
    matrices: Vec<f64>,
    ops: Vec<ffi::qvdg_op>,
}

impl PackedOps {
    fn new(ops: &[Op]) -> PackedOps {
        let mut qubits = Vec::new();
        let mut values = Vec::new();
        let mut matrices = Vec::new();
        let mut spans = Vec::with_capacity(ops.len());
        for op in ops {
            let q0 = qubits.len();
            qubits.extend(op.targets.iter().map(|&q| q as u32));
            let c0 = qubits.len();
            qubits.extend(op.controls.iter().map(|&(q, _)| q as u32));
            values.resize(qubits.len(), 0);
            for (i, &(_, v)) in op.controls.iter().enumerate() {
                values[c0 + i] = v as u8;
            }
            let m0 = matrices.len();
            for z in op.matrix.entries() {
                matrices.push(z.re);
                matrices.push(z.im);
            }
            spans.push((q0, c0, m0, op.targets.len(), op.controls.len()));
        }
        // Pointers are taken after every vector has its final size.
        let ops = spans
            .iter()
            .map(|&(q0, c0, m0, nt, nc)| ffi::qvdg_op {
                num_targets: nt as u32,
                num_controls: nc as u32,
                targets: qubits[q0..].as_ptr(),
                controls: if nc > 0 { qubits[c0..].as_ptr() } else { std::ptr::null() },
                control_values: if nc > 0 { values[c0..].as_ptr() } else { std::ptr::null() },
                matrix: matrices[m0..].as_ptr(),
            })
            .collect();
        PackedOps { qubits, values, matrices, ops }
    }
}

/// A state vector in B200 memory: complex64 for `T = f32`, complex128 for
/// `T = f64`, in physical order with the reference's layout semantics.
pub struct GpuStateVector {
    raw: *mut ffi::qvdg_state,
    num_qubits: usize,
}

// One caller at a time, as `&mut StateVector` (the handle is not shared).
unsafe impl Send for GpuStateVector {}

impl GpuStateVector {
    /// |0...0> on the current device (StateVector::zero, src/state.rs:39-50).
    pub fn zero<T: Real>(num_qubits: usize) -> io::Result<GpuStateVector> {
        let bits = 8 * std::mem::size_of::<T>() as u32;
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::qvdg_state_create(num_qubits as u32, bits, &mut raw) })?;
        Ok(GpuStateVector { raw, num_qubits })
    }

    /// StateVector::from_amplitudes (src/state.rs:52-63).
    pub fn from_amplitudes<T: Real>(amplitudes: &[C64]) -> io::Result<GpuStateVector> {
        let n = amplitudes.len().trailing_zeros() as usize;
        let state = GpuStateVector::zero::<T>(n)?;
        let flat: Vec<f64> = amplitudes.iter().flat_map(|z| [z.re, z.im]).collect();
        check(unsafe { ffi::qvdg_state_set_amplitudes(state.raw, flat.as_ptr(), amplitudes.len()) })?;
        Ok(state)
    }

    pub fn num_qubits(&self) -> usize {
        self.num_qubits
    }

    /// Back to |0...0> (the shot-by-shot path reuses one state).
    pub fn reset_to_zero(&mut self) -> io::Result<()> {
        check(unsafe { ffi::qvdg_state_zero(self.raw) })
    }

    /// apply_ops (src/simulator.rs:122-147): fuse, plan and run every op on
    /// the device; the run's counts and device time are added to `stats`.
    pub fn apply_ops(&mut self, ops: &[Op], options: &ffi::qvdg_options, stats: &mut Stats) -> io::Result<()> {
        if ops.is_empty() {
            return Ok(());
        }
        let packed = PackedOps::new(ops);
        let mut s = ffi::qvdg_stats::default();
        check(unsafe { ffi::qvdg_apply_ops(self.raw, packed.ops.as_ptr(), packed.ops.len(), options, &mut s) })?;
        stats.gates += s.gates as usize;
        stats.kernels += s.kernels as usize;
        stats.passes += s.passes as usize;
        stats.gate_seconds += s.gate_seconds;
        Ok(())
    }

    /// to_vec (src/state.rs:132-159): logical order, complex128.
    pub fn to_vec(&self) -> io::Result<Vec<C64>> {
        let count = 1usize << self.num_qubits;
        let mut flat = vec![0.0f64; 2 * count];
        check(unsafe { ffi::qvdg_state_get_amplitudes(self.raw, flat.as_mut_ptr(), count) })?;
        Ok(flat.chunks_exact(2).map(|p| C64::new(p[0], p[1])).collect())
    }

    /// norm_sqr (src/state.rs:172-177), in f64.
    pub fn norm_sqr(&self) -> io::Result<f64> {
        let mut v = 0.0;
        check(unsafe { ffi::qvdg_norm_sqr(self.raw, &mut v) })?;
        Ok(v)
    }

    /// probability_one (src/measure.rs:43-65).
    pub fn probability_one(&self, qubit: usize) -> io::Result<f64> {
        let mut v = 0.0;
        check(unsafe { ffi::qvdg_probability_one(self.raw, qubit as u32, &mut v) })?;
        Ok(v)
    }

    /// measure (src/measure.rs:68-80), with the same one uniform draw.
    pub fn measure(&mut self, qubit: usize, rng: &mut impl Rng) -> io::Result<bool> {
        let mut outcome = 0i32;
        check(unsafe { ffi::qvdg_measure(self.raw, qubit as u32, rng.random::<f64>(), &mut outcome) })?;
        Ok(outcome == 1)
    }

    /// reset (src/measure.rs:82-87).
    pub fn reset(&mut self, qubit: usize, rng: &mut impl Rng) -> io::Result<()> {
        check(unsafe { ffi::qvdg_reset(self.raw, qubit as u32, rng.random::<f64>()) })
    }

    /// sample_unordered (src/measure.rs:104-174): the same `shots` uniforms
    /// the reference draws, so the outcomes are bit-identical.
    pub fn sample_unordered(&self, shots: usize, rng: &mut impl Rng) -> io::Result<Vec<usize>> {
        let uniforms: Vec<f64> = (0..shots).map(|_| rng.random::<f64>()).collect();
        let mut out = vec![0u64; shots.max(1)];
        let mut count = 0usize;
        check(unsafe {
            ffi::qvdg_sample_unordered(self.raw, shots, uniforms.as_ptr(), out.as_mut_ptr(), &mut count)
        })?;
        Ok(out[..count].iter().map(|&i| i as usize).collect())
    }

    /// Counts by classical key on the device (count_outcomes,
    /// src/simulator.rs:187-230, for at most 64 classical bits): distinct
    /// keys (bit c = classical bit c) and their counts, keys ascending.
    pub fn sample_counts(&self, shots: usize, rng: &mut impl Rng, measures: &[(usize, usize)])
        -> io::Result<Vec<(u64, usize)>> {
        let uniforms: Vec<f64> = (0..shots).map(|_| rng.random::<f64>()).collect();
        let qubits: Vec<u32> = measures.iter().map(|&(q, _)| q as u32).collect();
        let clbits: Vec<u32> = measures.iter().map(|&(_, c)| c as u32).collect();
        let capacity = shots.max(1);
        let mut keys = vec![0u64; capacity];
        let mut counts = vec![0u64; capacity];
        let mut n = 0usize;
        check(unsafe {
            ffi::qvdg_sample_counts(self.raw, shots, uniforms.as_ptr(), qubits.as_ptr(), clbits.as_ptr(),
                                    measures.len(), keys.as_mut_ptr(), counts.as_mut_ptr(), capacity, &mut n)
        })?;
        Ok(keys[..n].iter().zip(&counts[..n]).map(|(&k, &c)| (k, c as usize)).collect())
    }
}

impl Drop for GpuStateVector {
    fn drop(&mut self) {
        unsafe { ffi::qvdg_state_destroy(self.raw) };
    }
}
