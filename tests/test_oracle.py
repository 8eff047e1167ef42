"""The CPU oracle (C++ restatement of the reference engine) against the naive
oracle, the reference's own known answers and analytic golden vectors.

Ports the CPU-side tests of tests/kernels.rs:12-92, tests/simulator.rs:7-214,
src/fusion.rs:186-215, src/matrix.rs:211-234 and src/circuit.rs:741-813.
"""

import math

import numpy as np
import pytest

from conftest import max_distance, random_diagonal, random_qubits, random_state, random_unitary
from qevedo_simulator_b200 import Circuit, Gate, library
from qevedo_simulator_b200.circuit import GATES, Op, _controlled


def _controlled_op(matrix, qubits, controls):
    return Op(list(qubits), list(controls), matrix)


@pytest.mark.parametrize("bits,tol", [(64, 1e-12), (32, 2e-6)])
def test_kernels_match_naive(oracle, bits, tol):
    """tests/kernels.rs:12-72: every kernel shape (low/high targets, controls,
    diagonals) against the naive simulator, 400 cases per precision."""
    rng = np.random.Generator(np.random.PCG64(1 if bits == 64 else 2))
    for case in range(400):
        n = int(rng.integers(1, 12))
        k = int(rng.integers(1, min(n, 6) + 1))
        qubits = random_qubits(rng, n, k)
        rest = [q for q in range(n) if q not in qubits]
        if not rest or k >= 6 or rng.random() < 0.5:
            controls = []
        else:
            c = int(rng.integers(1, min(len(rest), 2, 6 - k) + 1))
            controls = [(q, bool(rng.random() < 0.7)) for q in rest[:c]]
        diagonal = rng.random() < 0.3
        m = random_diagonal(rng, k) if diagonal else random_unitary(rng, k)
        initial = random_state(rng, n)
        expected = oracle.naive_apply_ops(initial, [_controlled_op(m, qubits, controls)])
        st = oracle.OracleState(n, bits)
        st.set_amplitudes(initial)
        st.apply(m, qubits, controls)
        d = max_distance(st.amplitudes(), expected)
        assert d < tol, (case, n, qubits, controls, diagonal, d)


def test_fusion_widths_and_blocking(oracle):
    """tests/simulator.rs:7-33 and :164-193 on the restated engine."""
    for seed in range(12):
        n = 1 + seed % 10
        c = library.random_gate_circuit(n, 60, seed)
        ops = c.ops()
        expected = oracle.naive_statevector(ops, n)
        for f in range(1, 7):
            st = oracle.OracleState(n, 64)
            s = st.apply_ops(ops, max_fused=f, region_bits=None)
            assert max_distance(st.amplitudes(), expected) < 1e-11
            assert s["kernels"] <= s["gates"]
    for seed in range(6):
        n = 8 + seed % 7
        ops = library.random_gate_circuit(n, 120, 100 + seed).ops()
        expected = oracle.naive_statevector(ops, n)
        for rb in range(1, 5):
            for f in (1, 3, 4):
                for bits, tol in ((64, 1e-11), (32, 1e-5)):
                    st = oracle.OracleState(n, bits)
                    s = st.apply_ops(ops, max_fused=f, region_bits=rb)
                    assert max_distance(st.amplitudes(), expected) < tol
                    assert s["passes"] > 0


def test_fusion_groups(oracle):
    """src/fusion.rs:186-215."""
    ops = [Op([0], [], Gate("h").matrix()), Op([5], [], Gate("h").matrix()),
           Op([0, 1], [], Gate("cx").matrix()), Op([6], [], Gate("h").matrix()),
           Op([1, 2], [], Gate("cx").matrix())]
    assert oracle.fuse_shapes(ops, 3) == [(3, 0), (2, 0)]
    ops = [Op([0, 1], [], Gate("cx").matrix()), Op([1], [], Gate("h").matrix()),
           Op([1, 2], [], Gate("cx").matrix())]
    assert oracle.fuse_shapes(ops, 2) == [(2, 0), (2, 0)]


def test_fusion_cuts_kernel_calls(oracle):
    """tests/simulator.rs:45-57."""
    ops = library.random_circuit(20, 20, 1).ops()
    shapes = oracle.fuse_shapes(ops, 4)
    assert len(ops) > 500 and len(shapes) * 4 < len(ops)


def test_every_gate_is_unitary_with_the_right_diagonal_flag():
    """src/circuit.rs:754-790."""
    params = {"rx": (0.3,), "ry": (0.4,), "rz": (0.5,), "p": (0.6,), "u": (0.1, 0.2, 0.3), "cp": (0.7,),
              "crx": (0.8,), "cry": (0.9,), "crz": (1.0,), "rzz": (1.1,), "rxx": (1.2,)}
    for name, (arity, npar) in GATES.items():
        g = Gate(name, params.get(name, ()))
        m = g.matrix()
        assert m.shape == (1 << arity, 1 << arity)
        assert np.max(np.abs(m @ m.conj().T - np.eye(m.shape[0]))) < 1e-12, name
        off = m[~np.eye(m.shape[0], dtype=bool)]
        assert bool(np.all(off == 0)) == g.is_diagonal(), name


def test_sx_squared_is_x_and_u_matches_qiskit():
    """src/circuit.rs:792-813."""
    sx = Gate("sx").matrix()
    assert np.max(np.abs(sx @ sx - Gate("x").matrix())) < 1e-12
    assert np.max(np.abs(Gate("u", (math.pi, 0.0, math.pi)).matrix() - Gate("x").matrix())) < 1e-12
    assert np.max(np.abs(Gate("u", (math.pi / 2, 0.0, math.pi)).matrix() - Gate("h").matrix())) < 1e-12


def test_controlled_x_is_cnot():
    """src/matrix.rs:224-234: CX on [control, target], control is bit 0."""
    cx = _controlled(Gate("x").matrix(), 1, 1)
    assert cx[1, 3] == 1 and cx[3, 1] == 1 and cx[0, 0] == 1 and cx[2, 2] == 1 and cx[1, 1] == 0
    assert np.array_equal(cx, Gate("cx").matrix())


def test_known_states(oracle):
    """python/tests/test_simulator.py:77-83: GHZ amplitudes and the H.T phase."""
    r = 1 / math.sqrt(2)
    ghz = oracle.naive_statevector(Circuit(3).h(0).cx(0, 1).cx(1, 2).ops(), 3)
    assert abs(ghz[0] - r) < 1e-12 and abs(ghz[7] - r) < 1e-12
    assert abs(np.sum(np.abs(ghz) ** 2) - 1) < 1e-12
    phased = oracle.naive_statevector(Circuit(1).h(0).t(0).ops(), 1)
    assert abs(phased[1] - r * complex(math.cos(math.pi / 4), math.sin(math.pi / 4))) < 1e-12
    for bits in (32, 64):
        st = oracle.OracleState(3, bits)
        st.apply_ops(Circuit(3).h(0).cx(0, 1).cx(1, 2).ops())
        assert max_distance(st.amplitudes(), ghz) < (1e-7 if bits == 32 else 1e-15)


def qft_golden(n: int, x: int) -> np.ndarray:
    """Analytic QFT (no final swaps) of basis state |x>: amplitude
    exp(2 pi i x k / 2^n) / sqrt(2^n) at the bit reversal of k."""
    N = 1 << n
    out = np.empty(N, dtype=np.complex128)
    for k in range(N):
        rev = int(format(k, f"0{n}b")[::-1], 2)
        out[rev] = np.exp(2j * np.pi * x * k / N) / math.sqrt(N)
    return out


@pytest.mark.parametrize("n,x", [(3, 0), (3, 5), (6, 0), (6, 41), (9, 300)])
def test_qft_against_analytic_golden(oracle, n, x):
    initial = np.zeros(1 << n, dtype=np.complex128)
    initial[x] = 1.0
    got = oracle.naive_statevector(library.qft(n).ops(), n, initial)
    assert max_distance(got, qft_golden(n, x)) < 1e-12
    st = oracle.OracleState(n, 64)
    st.set_amplitudes(initial)
    st.apply_ops(library.qft(n).ops())
    assert max_distance(st.amplitudes(), qft_golden(n, x)) < 1e-12


def test_committed_golden_fixtures(oracle):
    """tests/golden/*.npz (made by tests/golden/make_golden.py from analytic
    formulas and the naive oracle) against both oracle tiers."""
    import glob
    import os

    files = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
    assert files, "golden fixtures are missing"
    for path in files:
        z = np.load(path)
        from golden.make_golden import ops_from_fixture

        ops, n, initial = ops_from_fixture(z)
        expected = z["amplitudes"]
        assert max_distance(oracle.naive_statevector(ops, n, initial), expected) < 1e-12, path
        for bits, tol in ((64, 1e-11), (32, 1e-5)):
            st = oracle.OracleState(n, bits)
            st.set_amplitudes(initial)
            st.apply_ops(ops, max_fused=4, region_bits=2)
            assert max_distance(st.amplitudes(), expected) < tol, (path, bits)
        if "uniforms" in z.files:
            got = oracle.sample_from_amplitudes(expected, z["uniforms"], 64)
            assert np.array_equal(got, z["samples64"]), path


def test_bell_and_relabel_known_keys(oracle):
    """tests/simulator.rs:59-78 and :195-214 on the oracle sampler: Bell pairs
    only 00/11; after relabelling, keys 1010000000 and 1110000001."""
    from qevedo_simulator_b200.simulator import count_outcomes

    rng = np.random.Generator(np.random.PCG64(5))
    st = oracle.OracleState(2, 32)
    st.apply_ops(Circuit(2).h(0).cx(0, 1).ops())
    out = st.sample_unordered(rng.random(100_000))
    counts = count_outcomes(out, [(0, 0), (1, 1)], 2)
    assert set(counts) == {"00", "11"} and abs(counts["00"] - 50_000) < 800
    c = Circuit(10).x(9).x(7).h(0).cx(0, 8)
    st = oracle.OracleState(10, 32)
    st.apply_ops(c.ops(), max_fused=4, region_bits=1)
    assert st.layout() != list(range(10))  # the run relabelled qubits
    out = st.sample_unordered(rng.random(1000))
    counts = count_outcomes(out, [(q, q) for q in range(10)], 10)
    assert sorted(counts) == ["1010000000", "1110000001"]


def test_sampling_matches_probabilities(oracle):
    """tests/simulator.rs:80-111 (200k shots, 5 sigma per outcome)."""
    c = Circuit(3).ry(1.0, 0).ry(2.0, 1).cx(1, 2)
    probs = np.abs(oracle.naive_statevector(c.ops(), 3)) ** 2
    st = oracle.OracleState(3, 64)
    st.apply_ops(c.ops())
    shots = 200_000
    out = st.sample_unordered(np.random.Generator(np.random.PCG64(9)).random(shots))
    observed = np.bincount(out.astype(np.int64), minlength=8) / shots
    sigma = np.sqrt(probs * (1 - probs) / shots)
    assert np.all(np.abs(observed - probs) <= 5 * sigma + 1e-9)


def test_measure_collapse(oracle):
    """src/measure.rs:68-80: collapse renormalises the kept half."""
    st = oracle.OracleState(2, 64)
    st.apply_ops(Circuit(2).h(0).cx(0, 1).ops())
    assert st.measure(0, 0.9) == 0  # P(1) = 0.5 <= 0.9 -> outcome 0
    a = st.amplitudes()
    assert abs(a[0] - 1) < 1e-12 and max_distance(a[1:], np.zeros(3)) < 1e-12


def test_physical_loads_layouts_and_streamed_differences(oracle):
    """The oracle reads another engine's state as it lies in memory:
    physical-order amplitudes with a layout give the same logical state, the
    same samples as the swapped state, and the streamed max difference
    equals the logical one; bad layouts are rejected."""
    rng = np.random.Generator(np.random.PCG64(77))
    n = 14
    amps = random_state(rng, n)
    layout = [int(x) for x in rng.permutation(n)]
    idx = np.arange(1 << n)
    phys_index = np.zeros(1 << n, dtype=np.int64)
    for q in range(n):
        phys_index |= ((idx >> q) & 1) << layout[q]
    phys = np.empty_like(amps)
    phys[phys_index] = amps
    for bits in (32, 64):
        st = oracle.OracleState(n, bits)
        st.set_layout(layout)
        st.set_physical(phys.astype(np.complex64) if bits == 32 else phys)
        assert st.layout() == layout
        got = st.amplitudes()
        assert max_distance(got, amps) < (1e-7 if bits == 32 else 1e-15)
        given = phys.astype(np.complex64) if bits == 32 else phys
        other = amps + 1e-3 * random_state(rng, n)
        ref = oracle.OracleState(n, 64)
        ref.set_amplitudes(other)
        expected = float(np.max(np.abs(other - given[phys_index].astype(np.complex128))))
        assert abs(ref.max_diff_physical(given, layout) - expected) < 1e-15
        ref.close()
        u = rng.random(5000)
        assert np.array_equal(oracle.sample_physical(given, layout, u), st.sample_unordered(u))
        st.close()
    bad = oracle.OracleState(4, 64)
    with pytest.raises(RuntimeError, match="permutation"):
        bad.set_layout([0, 1, 1, 3])
    with pytest.raises(ValueError):
        bad.set_physical(np.zeros(8, dtype=np.complex128))
    bad.close()
