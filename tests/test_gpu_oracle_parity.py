"""Every device path against the CPU oracle's FP64 runs, in absolute terms,
at the workloads' own bounds: max |delta amplitude| <= 1e-6 for complex64
(the tensor-core passes included) and <= 1e-12 for complex128.

The truth is the naive simulator (src/reference.rs:8-44) up to 22 qubits and
the restated fast engine in f64 beyond (pinned to the naive one in
tests/test_oracle.py); device states are compared as they lie in HBM
(physical order with their layout), so relabelled plans need no extra pass.
The sampler is checked bit-exact (src/measure.rs:104-174) on full-size
complex64 states: 20 qubits (the first size whose 32-chunk warps are full),
22, 26 with a million shots, and the 30-qubit benchmark circuit's final
state, sampled where it lies, relabelled layout included."""

import numpy as np
import pytest

from conftest import device_physical, max_distance, random_state
from qevedo_simulator_b200 import DeviceState, Plan, library, options, statevector

pytestmark = pytest.mark.gpu

ABS_TOL = {32: 1e-6, 64: 1e-12}

PATHS = {
    32: [("plain-tensor-f6", options(6, staged=False, math="tensor")),
         ("plain-tensor-pairs-f6", options(6, staged=False, math="tensor_pairs")),
         ("plain-tensor-f5", options(5, staged=False, math="tensor")),
         ("plain-tensor-f4", options(4, staged=False, math="tensor")),
         ("staged-tensor-f4", options(4, staged=True, math="tensor")),
         ("staged-tensor-f5", options(5, staged=True, math="tensor")),
         ("staged-cuda", options(4, staged=True)),
         ("plain-f4", options(4, staged=False)),
         ("plain-gates-f4", options(4, staged=False, math="gates"))],
    64: [("plain-f4", options(4, staged=False)),
         ("staged", options(4, staged=True)),
         ("plain-gates-f4", options(4, staged=False, math="gates"))],
}


def _check_paths(ops, n, expected, initial=None, plans=True):
    """Run `ops` through every path, one-shot and as a reusable plan, and
    compare the logical amplitudes with `expected` in absolute terms."""
    worst = {}
    for bits in (32, 64):
        for name, opts in PATHS[bits]:
            with DeviceState(n, bits) as st:
                runs = [("one-shot", None)]
                if plans:
                    runs.append(("plan", Plan(ops, n, bits, opts)))
                for how, plan in runs:
                    if initial is None:
                        st.zero()
                    else:
                        st.set_amplitudes(initial)
                    if plan is None:
                        st.apply_ops(ops, opts)
                    else:
                        st.execute(plan)
                        plan.close()
                    err = max_distance(st.amplitudes(), expected)
                    worst[(bits, name, how)] = err
                    assert err <= ABS_TOL[bits], (bits, name, how, err)
    return worst


def test_grid_4x5_depth_20_every_path_against_naive(oracle):
    """The reference's CPU case exactly: 20 qubits on a 4x5 grid, depth 20,
    sqrt(X)/sqrt(Y)/sqrt(W) never repeating on a qubit, CZ on the four
    coupler sets, from |0...0>; plus the public statevector() call."""
    c = library.random_grid_circuit(4, 5, 20, seed=2024)
    ops = c.ops()
    expected = oracle.naive_statevector(ops, 20)
    _check_paths(ops, 20, expected)
    assert max_distance(statevector(c), expected) <= ABS_TOL[64]
    assert max_distance(statevector(c, precision="single"), expected) <= ABS_TOL[32]


@pytest.mark.parametrize("n", [20, 22])
def test_qft_from_gaussian_state_every_path_against_naive(oracle, n):
    """QFT (H + controlled phases, no final swaps) from a seeded normalised
    complex Gaussian state, as the 30-qubit QFT workload at oracle size."""
    ops = library.qft(n).ops()
    psi = library.gaussian_state(n, 2024)
    expected = oracle.naive_apply_ops(psi, ops)
    _check_paths(ops, n, expected, initial=psi, plans=(n == 20))


def _fast_oracle_f64(oracle, ops, n, initial=None):
    ref = oracle.OracleState(n, 64)
    if initial is not None:
        ref.set_amplitudes(initial)
    ref.apply_ops(ops, max_fused=4, region_bits=14)
    return ref


@pytest.mark.parametrize("n", [24, 26])
def test_grid_circuits_against_the_fast_oracle_in_f64(oracle, n):
    """24 and 26 qubits (4x6 and 2x13 grids, depth 20) through the tuned
    path (tensor-core plan at fusion 6, run from |0...0> with its zero-start
    passes and relabelled bits), the staged and plain CUDA-core paths, and
    complex128, against the oracle's fast engine in f64."""
    rows, cols = (4, 6) if n == 24 else (2, 13)
    ops = library.random_grid_circuit(rows, cols, 20, seed=n).ops()
    ref = _fast_oracle_f64(oracle, ops, n)
    try:
        for bits, name, opts in [(32, "plain-tensor-f6", options(6, staged=False, math="tensor")),
                                 (32, "plain-tensor-pairs-f6", options(6, staged=False, math="tensor_pairs")),
                                 (32, "staged-cuda", options(4, staged=True)),
                                 (32, "plain-f4", options(4, staged=False)),
                                 (64, "plain-f4", options(4, staged=False))]:
            with DeviceState(n, bits) as st, Plan(ops, n, bits, opts) as plan:
                st.zero()
                st.execute(plan)
                layout = st.layout()
                err = ref.max_diff_physical(device_physical(st), layout)
                assert err <= ABS_TOL[bits], (n, bits, name, err)
    finally:
        ref.close()


def test_qft_24_from_gaussian_against_the_fast_oracle_in_f64(oracle):
    n = 24
    ops = library.qft(n).ops()
    psi = library.gaussian_state(n, 7)
    ref = _fast_oracle_f64(oracle, ops, n, psi)
    try:
        for bits, opts in [(32, options(6, staged=False, math="tensor")), (32, options(5, staged=True, math="tensor")),
                           (32, options(6, staged=False, math="tensor_pairs")),
                           (64, options(4, staged=False))]:
            with DeviceState(n, bits) as st:
                st.set_amplitudes(psi)
                st.apply_ops(ops, opts)
                err = ref.max_diff_physical(device_physical(st), st.layout())
                assert err <= ABS_TOL[bits], (bits, err)
    finally:
        ref.close()


@pytest.mark.parametrize("n", [20, 22, 26])
def test_sampler_bit_exact_on_full_size_complex64_states(oracle, n):
    """Random complex64 states with zero runs: the device sampler's outcomes
    equal the reference sampler's for the same uniforms, in the identity
    layout and after a relabel (chunks then hold other amplitudes)."""
    rng = np.random.Generator(np.random.PCG64(5000 + n))
    amps = random_state(rng, n)
    amps[rng.random(amps.size) < 0.2] = 0
    amps /= np.sqrt(np.sum(np.abs(amps) ** 2))
    shots = [1000, 1_000_000] if n == 26 else [1000, 30_000]
    with DeviceState(n, 32) as st:
        st.set_amplitudes(amps)
        for relabel in (False, True):
            if relabel:
                st.swap_physical([(2, n - 1), (5, n - 3)])
            phys = device_physical(st)
            layout = st.layout()
            for count in shots:
                u = rng.random(count)
                u[:3] = [0.0, 0.9999999999999999, 0.5]
                got = st.sample_unordered(u)
                want = oracle.sample_physical(phys, layout, u)
                assert np.array_equal(got, want), (n, relabel, count)


def test_benchmark_circuit_at_30_qubits_against_the_oracle(oracle):
    """The 30-qubit benchmark (5x6 grid, depth 20, seed 2024, complex64 from
    |0...0>) through the tuned plan: max |delta amplitude| against the
    oracle's f64 engine within 1e-6, and 1000 shots bit-exact with the
    reference sampler on the final state as it lies on the device."""
    n = 30
    ops = library.random_grid_circuit(5, 6, 20, seed=2024).ops()
    with DeviceState(n, 32) as st, Plan(ops, n, 32, options(6, staged=False, math="tensor")) as plan:
        st.zero()
        st.execute(plan)
        layout = st.layout()
        u = np.random.Generator(np.random.PCG64(7)).random(1000)
        got = st.sample_unordered(u)
        phys = device_physical(st)
    assert np.array_equal(got, oracle.sample_physical(phys, layout, u))
    ref = _fast_oracle_f64(oracle, ops, n)
    try:
        err = ref.max_diff_physical(phys, layout)
    finally:
        ref.close()
    assert err <= ABS_TOL[32], err
