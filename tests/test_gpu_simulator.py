"""The device engine end to end against the naive oracle and the reference
sampler (tests/simulator.rs:7-214, python/tests/test_simulator.py:77-176)."""

import math

import numpy as np
import pytest

from conftest import max_distance, random_state
from qevedo_simulator_b200 import Circuit, DeviceState, library, options, run, statevector

pytestmark = pytest.mark.gpu

# Circuit tolerances of the reference (tests/simulator.rs:26-33, :274-281).
CIRCUIT_TOL = {64: 1e-11, 32: 1e-5}


def test_every_fusion_width_plain_and_staged(oracle):
    """tests/simulator.rs:7-33 (plain, region_bits = None) plus the staged
    path with a small tile on the same circuits."""
    for seed in range(40):
        n = 1 + seed % 10
        c = library.random_gate_circuit(n, 60, seed)
        ops = c.ops()
        expected = oracle.naive_statevector(ops, n)
        for f in range(1, 7):
            for staged in (False, True):
                for bits in (64, 32):
                    with DeviceState(n, bits) as st:
                        stats = st.apply_ops(ops, options(f, staged, tile_qubits=4 if staged else 0))
                        err = max_distance(st.amplitudes(), expected)
                    assert err < CIRCUIT_TOL[bits], (seed, n, f, staged, bits, err)
                    assert stats["kernels"] <= stats["gates"]


def test_staged_tiles_force_many_stages(oracle):
    """tests/simulator.rs:164-193: tiny tiles force many stages, global
    controls and global diagonal targets."""
    for seed in range(30):
        n = 8 + seed % 7
        ops = library.random_gate_circuit(n, 120, 100 + seed).ops()
        expected = oracle.naive_statevector(ops, n)
        for tile in (2, 3, 4, 6):
            for f in (1, 3, 4):
                for bits in (64, 32):
                    with DeviceState(n, bits) as st:
                        stats = st.apply_ops(ops, options(f, True, tile))
                        err = max_distance(st.amplitudes(), expected)
                    assert err < CIRCUIT_TOL[bits], (seed, n, tile, f, bits, err)
                    assert stats["passes"] > 0


def test_library_circuits_and_fusion_merges(oracle):
    """tests/simulator.rs:35-57."""
    for c in (library.ghz(9), library.qft(9), library.random_circuit(10, 12, 7)):
        expected = oracle.naive_statevector(c.ops(), c.num_qubits)
        got = statevector(c)
        assert max_distance(got, expected) < 1e-12
    with DeviceState(20, 32) as st:
        stats = st.apply_ops(library.random_circuit(20, 20, 1).ops(), options(4, False))
    assert stats["gates"] > 500 and stats["kernels"] * 4 < stats["gates"]


def test_committed_golden_fixtures():
    import glob
    import os

    from golden.make_golden import ops_from_fixture

    for path in sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))):
        z = np.load(path)
        ops, n, initial = ops_from_fixture(z)
        for bits in (64, 32):
            for staged in (False, True):
                with DeviceState(n, bits) as st:
                    st.set_amplitudes(initial)
                    st.apply_ops(ops, options(4, staged, 4))
                    assert max_distance(st.amplitudes(), z["amplitudes"]) < CIRCUIT_TOL[bits], (path, bits)
                    if "uniforms" in z.files and bits == 64:
                        # the device holds the fixture's amplitudes exactly
                        st.set_amplitudes(z["amplitudes"])
                        assert np.array_equal(st.sample_unordered(z["uniforms"]), z["samples64"]), path


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("n", [1, 2, 3, 7, 14, 15, 16, 19])
def test_sampler_is_bit_exact(oracle, bits, n):
    """The device sampler returns exactly the reference sampler's outcomes
    (src/measure.rs:104-174) for the same amplitudes and uniforms, including
    one and many chunks, zero-probability runs and targets at the edges."""
    rng = np.random.Generator(np.random.PCG64(1000 * bits + n))
    amps = random_state(rng, n)
    if n >= 3:
        amps[rng.random(amps.size) < 0.3] = 0  # zero-probability entries are skipped by the walk
        amps /= np.sqrt(np.sum(np.abs(amps) ** 2))
    for shots in (1, 17, 1000, 30000):
        u = rng.random(shots)
        u[: min(3, shots)] = [0.0, 0.9999999999999999, 0.5][: min(3, shots)]
        with DeviceState(n, bits) as st:
            st.set_amplitudes(amps)
            device_amps = st.amplitudes()  # the state's own precision, as complex128
            got = st.sample_unordered(u)
        want = oracle.sample_from_amplitudes(device_amps, u, bits)
        assert np.array_equal(got, want), (n, bits, shots)


def test_sampler_on_a_circuit_state_and_skewed_distribution(oracle):
    """A GHZ state puts every shot in two chunks; 1M shots exercise the
    device sort and the walk's long runs."""
    for bits in (32, 64):
        with DeviceState(17, bits) as st:
            st.apply_ops(library.ghz(17).ops())
            amps = st.amplitudes()
            u = np.random.Generator(np.random.PCG64(4)).random(1_000_000)
            got = st.sample_unordered(u)
        assert np.array_equal(got, oracle.sample_from_amplitudes(amps, u, bits))
        assert set(np.unique(got).tolist()) == {0, (1 << 17) - 1}


def test_bell_state_sampling():
    """tests/simulator.rs:59-78."""
    result = run(Circuit(2).h(0).cx(0, 1).measure_all(), 100_000, seed=5)
    assert set(result.counts) == {"00", "11"}
    assert sum(result.counts.values()) == 100_000
    assert abs(result.counts["00"] - 50_000) < 800


def test_sampling_matches_probabilities(oracle):
    """tests/simulator.rs:80-111."""
    c = Circuit(3).ry(1.0, 0).ry(2.0, 1).cx(1, 2)
    probs = np.abs(oracle.naive_statevector(c.ops(), 3)) ** 2
    shots = 200_000
    result = run(c.copy().measure_all(), shots, seed=9, precision="double")
    for index, p in enumerate(probs):
        observed = result.counts.get(format(index, "03b"), 0) / shots
        assert abs(observed - p) <= 5 * math.sqrt(p * (1 - p) / shots) + 1e-9


def test_mid_circuit_measurement_and_reset():
    """tests/simulator.rs:113-138."""
    c = Circuit(1).x(0).measure(0, 0).reset(0).measure(0, 1).h(0).measure(0, 2)
    result = run(c, 2000, seed=3, precision="double")
    assert sorted(result.counts) == ["001", "101"]
    assert abs(result.counts["101"] - 1000) < 200


def test_measurement_collapse_is_consistent():
    """tests/simulator.rs:140-162."""
    c = library.ghz(5)
    for q in range(5):
        c.measure(q, q)
        c.x(q)
    result = run(c, 500, seed=11)
    assert set(result.counts) <= {"00000", "11111"}


def test_sampling_after_relabelling():
    """tests/simulator.rs:195-214: samples of a permuted physical layout come
    back in logical order."""
    c = Circuit(10).x(9).x(7).h(0).cx(0, 8)
    with DeviceState(10, 32) as st:
        st.apply_ops(c.ops())
        st.swap_physical([(0, 5), (8, 2), (9, 3)])
        assert st.layout() != list(range(10))
        out = st.sample_unordered(np.random.Generator(np.random.PCG64(1)).random(1000))
    from qevedo_simulator_b200 import count_outcomes

    assert sorted(count_outcomes(out, [(q, q) for q in range(10)], 10)) == ["1010000000", "1110000001"]


def test_known_states():
    """python/tests/test_simulator.py:77-83."""
    r = 1 / math.sqrt(2)
    ghz = statevector(Circuit(3).h(0).cx(0, 1).cx(1, 2))
    assert abs(ghz[0] - r) < 1e-12 and abs(ghz[7] - r) < 1e-12
    phased = statevector(Circuit(1).h(0).t(0))
    assert abs(phased[1] - r * complex(math.cos(math.pi / 4), math.sin(math.pi / 4))) < 1e-12


def test_reproducible_counts():
    """python/tests/test_simulator.py:167-176: the same seed gives identical
    counts."""
    c = Circuit(6)
    for q in range(6):
        c.h(q).t(q)
    for q in range(5):
        c.cx(q, q + 1)
    c.measure_all()
    a = run(c, 3000, seed=9)
    b = run(c, 3000, seed=9, staged=False)
    assert a.counts == b.counts


@pytest.mark.parametrize("bits", [32, 64])
def test_reductions_and_layout_views(oracle, bits):
    rng = np.random.Generator(np.random.PCG64(21))
    n = 13
    amps = random_state(rng, n) * 1.3
    with DeviceState(n, bits) as st:
        st.set_amplitudes(amps)
        held = st.amplitudes()
        p = np.abs(held) ** 2
        assert abs(st.norm_sqr() - p.sum()) < 1e-12
        for q in (0, 1, 5, 12):
            assert abs(st.probability_one(q) - p[(np.arange(p.size) >> q) & 1 == 1].sum()) < 1e-12
        z = st.expect_z_all()
        for q in range(n):
            ones = p[(np.arange(p.size) >> q) & 1 == 1].sum()
            assert abs(z[q] - (p.sum() - 2 * ones)) < 1e-12
        assert np.max(np.abs(st.probabilities() - p)) < 1e-15
        # a permuted layout changes none of the logical views
        st.swap_physical([(0, 7), (3, 12)])
        assert max_distance(st.amplitudes(), held) == 0.0
        assert np.max(np.abs(st.probabilities() - p)) < 1e-15
        assert np.max(np.abs(st.expect_z_all() - z)) < 1e-12
        st.scale(0.5)
        assert max_distance(st.amplitudes(), held * 0.5) < 1e-7


def test_measure_and_reset_match_the_oracle(oracle):
    c = Circuit(4).h(0).cx(0, 1).ry(0.7, 2).cx(2, 3)
    for bits in (32, 64):
        for u in (0.1, 0.6, 0.95):
            with DeviceState(4, bits) as st:
                st.apply_ops(c.ops())
                o = oracle.OracleState(4, bits)
                o.apply_ops(c.ops())
                assert st.measure(2, u) == o.measure(2, u)
                assert max_distance(st.amplitudes(), o.amplitudes()) < 1e-6
                st.reset(0, u)
                assert st.probability_one(0) < 1e-12


def test_device_counts_match_host_counting():
    """qvdg_sample_counts: keys built, sorted and counted on the device equal
    the host's count_outcomes of the same samples (count_outcomes,
    src/simulator.rs:187-230), duplicate classical bits included (their
    bits OR together, as in the reference's keyed counting)."""
    from qevedo_simulator_b200 import library
    from qevedo_simulator_b200.simulator import count_outcomes

    rng = np.random.Generator(np.random.PCG64(3))
    for n, measures, nclbits in [(10, [(q, q) for q in range(10)], 10), (12, [(0, 3), (5, 0), (11, 1)], 4),
                                 (9, [(1, 0), (2, 0), (8, 2)], 3), (14, [], 2)]:
        c = library.random_grid_circuit(*library.grid_shape(n), 6, seed=n)
        with DeviceState(n, 32) as st:
            st.apply_ops(c.ops(), options(4, True))
            u = rng.random(20000)
            outcomes = st.sample_unordered(u)
            keys, counts = st.sample_counts(u, measures)
        host = count_outcomes(outcomes, measures, nclbits)
        dev = {"".join("1" if (int(k) >> b) & 1 else "0" for b in reversed(range(nclbits))): int(v)
               for k, v in zip(keys, counts)}
        assert dev == host and sum(dev.values()) == 20000
        assert list(keys) == sorted(keys)


@pytest.mark.parametrize("bits", [32, 64])
def test_pauli_expectations_match_numpy(bits):
    rng = np.random.Generator(np.random.PCG64(bits))
    n = 9
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    mats = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]]), "Y": np.array([[0, -1j], [1j, 0]]),
            "Z": np.diag([1, -1])}
    with DeviceState(n, bits) as st:
        st.set_amplitudes(psi)
        st.swap_physical([(0, 5), (2, 7)])  # logical qubits stay where they are
        for _ in range(25):
            label = "".join(rng.choice(list("IXYZ"), size=n))
            op = np.array([[1.0]])
            for ch in label:  # leftmost letter = highest qubit
                op = np.kron(op, mats[ch])
            expected = float(np.real(np.vdot(psi, op @ psi)))
            got = st.expect_pauli(label)
            assert abs(got - expected) < (1e-12 if bits == 64 else 2e-6), (label, got, expected)
        with pytest.raises(ValueError, match="twice"):
            st.expect_pauli([(1, "X"), (1, "Z")])


def test_estimate_sums_pauli_terms(oracle):
    from qevedo_simulator_b200 import estimate, library

    c = library.random_grid_circuit(3, 3, 6, seed=2)
    psi = oracle.naive_statevector(c.ops(), 9)
    z0 = np.where(np.arange(1 << 9) & 1, -1.0, 1.0)
    expected = 0.5 * float(np.sum(np.abs(psi) ** 2 * z0)) + 2.0
    assert estimate(c, {"IIIIIIIIZ": 0.5, "IIIIIIIII": 2.0}) == pytest.approx(expected, abs=1e-12)


def test_qasm_teleportation_with_feedback_runs():
    """An OpenQASM 3 teleportation (Pauli corrections as classical feedback,
    run shot by shot on the device): qubit 2 ends in the state RY(0.9)|0>."""
    from qevedo_simulator_b200 import qasm

    program = """OPENQASM 3.0;
        include "stdgates.inc";
        qubit[3] q;
        bit[3] c;
        ry(0.9) q[0];
        h q[1]; cx q[1], q[2];
        cx q[0], q[1]; h q[0];
        c[0] = measure q[0];
        c[1] = measure q[1];
        if (c[1]) x q[2];
        if (c[0]) z q[2];
        c[2] = measure q[2];"""
    c = qasm.parse(program)
    r = run(c, 4000, seed=11)
    ones = sum(v for k, v in r.counts.items() if k[0] == "1")
    assert abs(ones / 4000 - math.sin(0.45) ** 2) < 0.03


def test_run_and_statevector_on_openqasm_text():
    """OpenQASM text through run() and statevector() gives what the parsed
    circuit gives (the reference's wrappers take either), and the threads and
    MPS keywords leave the state-vector results unchanged."""
    from qevedo_simulator_b200 import qasm

    text = ('OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[3];\ncreg c[3];\n'
            'h q[0];\ncx q[0],q[1];\nry(0.7) q[2];\ncz q[1],q[2];\nmeasure q -> c;')
    parsed = qasm.parse(text)
    a = run(text, 5000, seed=11)
    b = run(parsed, 5000, seed=11, threads=2, max_bond_dimension=16, truncation_threshold=1e-8)
    assert a.counts == b.counts and sum(a.counts.values()) == 5000
    unitary = text.replace("measure q -> c;", "")
    sv = statevector(qasm.parse(unitary))
    assert np.array_equal(statevector(unitary, threads="cores"), sv)
    assert np.array_equal(statevector(unitary, threads=2), sv)
