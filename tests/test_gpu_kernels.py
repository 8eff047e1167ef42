"""Device kernels against the naive oracle (tests/kernels.rs:12-92 through
the C ABI), every precision, plain and staged paths."""

import numpy as np
import pytest

from conftest import max_distance, random_diagonal, random_qubits, random_state, random_unitary
from qevedo_simulator_b200 import DeviceState, Op, options

pytestmark = pytest.mark.gpu

# Amplitude tolerances of the reference's kernel tests (tests/kernels.rs:65-72).
TOL = {64: 1e-12, 32: 2e-6}


@pytest.mark.parametrize("bits", [64, 32])
def test_every_kernel_shape_matches_naive(oracle, bits):
    rng = np.random.Generator(np.random.PCG64(101 + bits))
    for case in range(400):
        n = int(rng.integers(1, 12))
        k = int(rng.integers(1, min(n, 6) + 1))
        qubits = random_qubits(rng, n, k)
        rest = [q for q in range(n) if q not in qubits]
        if not rest or rng.random() < 0.4:
            controls = []
        else:
            c = int(rng.integers(1, min(len(rest), 3) + 1))
            controls = [(q, bool(rng.random() < 0.7)) for q in rest[:c]]
        diagonal = rng.random() < 0.3
        m = random_diagonal(rng, k) if diagonal else random_unitary(rng, k)
        initial = random_state(rng, n)
        expected = oracle.naive_apply_ops(initial, [Op(qubits, controls, m)])
        with DeviceState(n, bits) as st:
            st.set_amplitudes(initial)
            st.apply(m, qubits, controls)
            d = max_distance(st.amplitudes(), expected)
        assert d < TOL[bits], (case, n, qubits, controls, diagonal, d)


@pytest.mark.parametrize("bits", [64, 32])
@pytest.mark.parametrize("staged", [False, True])
def test_large_state_every_width(oracle, bits, staged):
    """tests/kernels.rs:74-92: n = 18, dense k = 1..6 on random qubits (the
    grid-stride / many-tile paths)."""
    rng = np.random.Generator(np.random.PCG64(3))
    n = 18
    initial = random_state(rng, n)
    for k in range(1, 7):
        qubits = random_qubits(rng, n, k)
        m = random_unitary(rng, k)
        expected = oracle.naive_apply_ops(initial, [Op(qubits, [], m)])
        with DeviceState(n, bits) as st:
            st.set_amplitudes(initial)
            st.apply_ops([Op(qubits, [], m)], options(max_fused_qubits=1, staged=staged, tile_qubits=8))
            assert max_distance(st.amplitudes(), expected) < TOL[bits] * 4, (k, qubits)


@pytest.mark.parametrize("bits", [64, 32])
def test_staged_gate_with_global_controls_and_diagonals(oracle, bits):
    """Staged tiles with controls and diagonal targets outside the tile (the
    RegionOp cases of src/blocking.rs:57-149)."""
    rng = np.random.Generator(np.random.PCG64(17))
    n = 12
    for case in range(60):
        ops = []
        for _ in range(12):
            k = int(rng.integers(1, 4))
            qs = random_qubits(rng, n, k + 2)
            diagonal = rng.random() < 0.4
            m = random_diagonal(rng, k) if diagonal else random_unitary(rng, k)
            nc = int(rng.integers(0, 3))
            ops.append(Op(qs[:k], [(q, bool(rng.random() < 0.6)) for q in qs[k:k + nc]], m))
        initial = random_state(rng, n)
        expected = oracle.naive_apply_ops(initial, ops)
        for tile in (3, 4, 6):
            with DeviceState(n, bits) as st:
                st.set_amplitudes(initial)
                stats = st.apply_ops(ops, options(max_fused_qubits=3, staged=True, tile_qubits=tile))
                assert stats["stages"] >= 1
                assert max_distance(st.amplitudes(), expected) < TOL[bits] * 10, (case, tile)


@pytest.mark.parametrize("n", [13, 14, 16])
def test_dense_gates_on_low_bits_through_tiles(oracle, n):
    """Plain dense gates with targets among bits 0-3 (staged through
    shared-memory tiles) on every kind of target layout, against the naive
    oracle; controlled ones keep the direct path."""
    rng = np.random.Generator(np.random.PCG64(n))
    initial = random_state(rng, n)
    layouts = [[0, 1, 2, 3], [0, 1, 5, 7], [3, 0], [1, n - 1], [0, n - 3, n - 2, n - 1], [2, 11, 12],
               [n - 1, 0, 6, 2], [1, 2, 3], [3, 1, n - 1, 2], [2, 0, 1, 9]]
    for qubits in layouts:
        for controls in ([], [(4 if 4 not in qubits else 8, True)]):
            m = random_unitary(rng, len(qubits))
            expected = oracle.naive_apply_ops(initial, [Op(qubits, controls, m)])
            with DeviceState(n, 32) as st:
                st.set_amplitudes(initial)
                st.apply_ops([Op(qubits, controls, m)], options(4, staged=False))
                assert max_distance(st.amplitudes(), expected) < TOL[32] * 4, (qubits, controls)


def test_invalid_input_is_rejected():
    with DeviceState(4, 32) as st:
        with pytest.raises(ValueError, match="out of range"):
            st.apply(np.eye(2), [4])
        with pytest.raises(ValueError, match="twice"):
            st.apply(np.eye(4), [1, 1])
        with pytest.raises(ValueError, match="expected"):
            st.set_amplitudes(np.zeros(8))
        with pytest.raises(ValueError):
            st.swap_physical([(0, 0)])
    with pytest.raises(ValueError, match="precision"):
        DeviceState(4, 16)


@pytest.mark.parametrize("bits", [32, 64])
def test_full_size_tiles_and_plans(oracle, bits):
    """The benchmark's tile shape (13 local qubits for complex64, 12 for
    complex128) on a 20-qubit grid circuit, through apply_ops and through a
    reusable plan; both match the plain path and the naive oracle."""
    from qevedo_simulator_b200 import Plan, library

    c = library.random_grid_circuit(4, 5, 12, seed=5)
    ops = c.ops()
    expected = oracle.naive_statevector(ops, 20)
    tile = 13 if bits == 32 else 12
    with DeviceState(20, bits) as st, Plan(ops, 20, bits, options(4, True, tile)) as plan:
        info = plan.info()
        assert info["stages"] == info["passes"] and info["passes"] < info["kernels"]
        st.execute(plan)
        a = st.amplitudes()
        assert max_distance(a, expected) < TOL[bits] * 50
        st.zero()
        st.apply_ops(ops, options(4, True, tile))
        assert max_distance(st.amplitudes(), a) == 0.0
        st.zero()
        st.set_pass_timing(True)
        st.execute(plan)
        sec, byt, kind = st.pass_times()
        assert len(sec) == info["passes"] and np.all(kind == 1) and np.all(sec > 0)
        assert max_distance(st.amplitudes(), a) == 0.0


def test_plan_rejects_a_mismatched_state():
    from qevedo_simulator_b200 import Plan

    with DeviceState(6, 32) as st, Plan([Op([0], [], np.eye(2))], 7, 32) as plan:
        with pytest.raises(ValueError, match="another state size"):
            st.execute(plan)


# Tensor-core stages: fused gates as bf16 hi/lo compensated products with fp32
# accumulation, about 2^-17 relative error per gate application. The bounds
# below are relative to the largest amplitude of the state: TC_REL_TOL for
# up to ~30 gates, TC_CIRCUIT_TOL for deep circuits (~50-100 fused gates,
# whose errors add as a random walk).
TC_REL_TOL = 2e-5
TC_CIRCUIT_TOL = 1e-4


@pytest.mark.parametrize("n,tile", [(12, 12), (12, 10), (16, 12), (18, 11)])
def test_tensor_core_stages_match_naive(oracle, n, tile):
    rng = np.random.Generator(np.random.PCG64(40 + n))
    initial = random_state(rng, n)
    for fuse in (3, 4, 5, 6):
        ops = []
        for _ in range(30):
            k = int(rng.integers(1, 4))
            qs = random_qubits(rng, n, k)
            m = random_diagonal(rng, k) if rng.random() < 0.25 else random_unitary(rng, k)
            ops.append(Op(qs, [], m))
        expected = oracle.naive_apply_ops(initial, ops)
        with DeviceState(n, 32) as st:
            st.set_amplitudes(initial)
            stats = st.apply_ops(ops, options(fuse, True, tile, math="tensor"))
            got = st.amplitudes()
        err = max_distance(got, expected) / np.max(np.abs(expected))
        assert err < TC_REL_TOL, (n, tile, fuse, err, stats)


def test_tensor_core_single_wide_gates(oracle):
    """One dense gate of each tensor-core width (3..5 qubits on a 12-qubit
    tile) on one and on several tiles."""
    rng = np.random.Generator(np.random.PCG64(77))
    n = 14
    initial = random_state(rng, n)
    for k in (3, 4, 5):
        qubits = random_qubits(rng, n, k)
        m = random_unitary(rng, k)
        expected = oracle.naive_apply_ops(initial, [Op(qubits, [], m)])
        with DeviceState(n, 32) as st:
            st.set_amplitudes(initial)
            st.apply_ops([Op(qubits, [], m)], options(6, True, 12, math="tensor"))
            err = max_distance(st.amplitudes(), expected) / np.max(np.abs(expected))
        assert err < TC_REL_TOL, (k, qubits, err)


@pytest.mark.parametrize("kind", ["grid", "qft", "gates"])
def test_tensor_core_circuits(oracle, kind):
    """Whole circuits through tensor-core stages: CZ runs (sign flips folded
    into the gathers), QFT's controlled phases (complex phases folded), and
    the all-gate test circuit (controls, swaps, Toffolis)."""
    from qevedo_simulator_b200 import library

    if kind == "grid":
        c = library.random_grid_circuit(4, 4, 14, seed=8)
    elif kind == "qft":
        c = library.qft(15)
    else:
        c = library.random_gate_circuit(14, 200, seed=9)
    n = c.num_qubits
    initial = random_state(np.random.Generator(np.random.PCG64(5)), n)
    expected = oracle.naive_apply_ops(initial, c.ops())
    for fuse in (4, 5):
        with DeviceState(n, 32) as st:
            st.set_amplitudes(initial)
            st.apply_ops(c.ops(), options(fuse, True, 0, math="tensor"))
            err = max_distance(st.amplitudes(), expected) / np.max(np.abs(expected))
        assert err < TC_CIRCUIT_TOL, (kind, fuse, err)


def _plain_tensor_passes(ops, n):
    from qevedo_simulator_b200 import costmodel

    rows = costmodel.plan_features(ops, n, options(6, staged=False, math="tensor"))
    return int(np.sum((rows[:, 2] == 1) & (rows[:, 22] + rows[:, 23] > 0)))


@pytest.mark.parametrize("n", [13, 14, 17])
def test_tensor_core_plain_passes_single_gates(oracle, n):
    """Plain passes of one fused 4-6 qubit gate on the tensor cores (bf16x3,
    fp32 accumulation): targets in any order, on bit 0 (paired 16-byte
    accesses), on bits 0 and 1 (32-byte accesses) or neither, low and high,
    with controls where at least 8192 amplitudes stay selected (otherwise
    the CUDA-core pass runs)."""
    rng = np.random.Generator(np.random.PCG64(300 + n))
    initial = random_state(rng, n)
    layouts = [[0, 1, 2, 3], [3, 1, 0, 2, 4], [n - 1, 0, 5, 2, 7, 3], [4, 5, 6, 7], [n - 4, n - 3, n - 2, n - 1, 1],
               [9, 2, 12, 6, 1, 8], [1, 2, 3, 4, 5, 6], [6, 0, 11, 3], [5, 1, 0, 9], [0, 1, 2, 8, 10, 12],
               [3, 0, 2, 1, 9, 11]]
    used = 0
    for qubits in layouts:
        for controls in ([], [(max(qubits) + 1 if max(qubits) + 1 < n else min(set(range(n)) - set(qubits)),
                               bool(rng.integers(2)))]):
            m = random_unitary(rng, len(qubits))
            ops = [Op(qubits, controls, m)]
            used += _plain_tensor_passes(ops, n)
            expected = oracle.naive_apply_ops(initial, ops)
            with DeviceState(n, 32) as st:
                st.set_amplitudes(initial)
                st.set_pass_timing(True)
                st.apply_ops(ops, options(6, staged=False, math="tensor"))
                err = max_distance(st.amplitudes(), expected) / np.max(np.abs(expected))
                kind = st.pass_times()[2]
            assert err < TC_REL_TOL, (n, qubits, controls, err)
            if n - len(controls) >= 13:
                # direct kernel (2), or the shared-memory stage (3) for
                # uncontrolled gates on bits 1, 2 and 3 (6-qubit ones only
                # without bit 0)
                staged = not controls and {1, 2, 3} <= set(qubits) and (len(qubits) <= 5 or 0 not in qubits)
                assert list(kind) == [3 if staged else 2], (qubits, controls, kind)
    assert used >= len(layouts)


@pytest.mark.parametrize("kind", ["grid", "mixed", "qft", "gates"])
def test_tensor_core_plain_circuits(oracle, kind):
    """Whole circuits as plain passes with fused 4-6 qubit gates on the
    tensor cores and the rest (diagonals, narrow or heavily controlled
    gates) on the CUDA-core kernels."""
    from qevedo_simulator_b200 import library

    n = 16
    if kind == "grid":
        ops = library.random_grid_circuit(4, 4, 14, seed=31).ops()
    elif kind == "mixed":
        ops = library.mixed_ops(n, 8, seed=32)
    elif kind == "qft":
        ops = library.qft(n).ops()
    else:
        ops = library.random_gate_circuit(n, 150, seed=33).ops()
    initial = random_state(np.random.Generator(np.random.PCG64(34)), n)
    expected = oracle.naive_apply_ops(initial, ops)
    for fuse in (4, 5, 6):
        with DeviceState(n, 32) as st:
            st.set_amplitudes(initial)
            stats = st.apply_ops(ops, options(fuse, staged=False, math="tensor"))
            err = max_distance(st.amplitudes(), expected) / np.max(np.abs(expected))
        assert err < TC_CIRCUIT_TOL, (kind, fuse, err, stats)


@pytest.mark.parametrize("kind", ["grid", "mixed"])
def test_tensor_core_plain_passes_at_24_qubits(kind):
    """24-qubit circuits (many CTA iterations, every access width and the
    shared-memory stage) through tensor-core plain passes at fusion 4-6,
    against a complex128 run of the same ops on the device: max |delta
    amplitude| within the 1e-6 amplitude bound for complex64."""
    from qevedo_simulator_b200 import library

    n = 24
    ops = library.random_grid_circuit(4, 6, 12, seed=41).ops() if kind == "grid" else library.mixed_ops(n, 10, seed=42)
    with DeviceState(n, 64) as ref:
        ref.apply_ops(ops, options(4, staged=False))
        for fuse in (4, 5, 6):
            with DeviceState(n, 32) as st:
                st.set_pass_timing(True)
                st.apply_ops(ops, options(fuse, staged=False, math="tensor"))
                kinds = set(st.pass_times()[2].tolist())
                assert 2 in kinds, kinds
                assert ref.max_abs_diff(st) < 1e-6, (kind, fuse)


@pytest.mark.parametrize("kind", ["grid", "qft", "mixed"])
def test_zero_start_passes_match_full_passes(kind):
    """Run from |0...0> (after zero()), a plan's first passes take every
    qubit that no pass has touched yet as a control of value 0: those
    amplitudes are zero and stay zero. For plans without a fusion search
    (CUDA-core fusion 4, tensor-core fusion 4) the result equals, exactly,
    the same plan run on |0...0> loaded as amplitudes (every pass over the
    whole state), and the zero-start run moves fewer bytes. Tensor-core
    fusion-6 plans pick their fusion by the cost from |0...0> and keep the
    general pick for other states: both runs match complex128 to 1e-6."""
    from qevedo_simulator_b200 import Plan, library

    n = 21
    if kind == "grid":
        ops = library.random_grid_circuit(3, 7, 10, seed=8).ops()
    elif kind == "qft":
        ops = library.qft(n).ops()
    else:
        ops = library.mixed_ops(n, 6, seed=9)
    basis = np.zeros(2 ** n, dtype=np.complex128)
    basis[0] = 1.0
    with DeviceState(n, 64) as ref:
        ref.zero()
        ref.apply_ops(ops, options(4, staged=False))
        for opts, exact in ((options(4, staged=False), True), (options(4, staged=False, math="tensor"), True),
                            (options(6, staged=False, math="tensor"), False)):
            with Plan(ops, n, 32, opts) as plan, DeviceState(n, 32) as a, DeviceState(n, 32) as b:
                a.zero()
                sa = a.execute(plan)
                b.set_amplitudes(basis)
                sb = b.execute(plan)
                if exact:
                    assert a.max_abs_diff(b) == 0.0, (kind, opts.max_fused_qubits, opts.math)
                    assert sa["bytes"] < sb["bytes"], (sa, sb)
                assert ref.max_abs_diff(a) < 1e-6 and ref.max_abs_diff(b) < 1e-6, (kind, opts.max_fused_qubits)


def test_qft_plans_with_commuting_diagonal_gates():
    """The 22-qubit QFT as a reusable tensor-core plan at fusion 5 and 6,
    whose fusion lets controlled phases commute past each other (and beam
    searches the seeds), from a random state: matches a complex128 run of
    the gates in their own order to 1e-6, and takes far fewer passes than
    the CUDA-core fusion-4 plan."""
    from qevedo_simulator_b200 import Plan, library

    n = 22
    ops = library.qft(n).ops()
    psi = random_state(np.random.Generator(np.random.PCG64(5)), n)
    with DeviceState(n, 64) as ref, DeviceState(n, 32) as st:
        ref.set_amplitudes(psi)
        plain = ref.apply_ops(ops, options(4, staged=False))
        for fuse in (5, 6):
            with Plan(ops, n, 32, options(fuse, staged=False, math="tensor")) as plan:
                st.set_amplitudes(psi)
                stats = st.execute(plan)
                assert stats["passes"] < 0.75 * plain["passes"], (fuse, stats["passes"], plain["passes"])
                assert ref.max_abs_diff(st) < 1e-6, fuse


def test_one_shot_tensor_core_run_with_beam_search_at_30_qubits():
    """A one-shot run of fused 6-qubit tensor-core passes on a state of 29 or
    more qubits searches its fusion with a beam (below that only the seed
    lookahead pays for its planning time): the 30-qubit grid circuit matches
    the plain CUDA-core fusion-4 run to 1e-6."""
    from qevedo_simulator_b200 import library

    ops = library.random_grid_circuit(5, 6, 8, seed=77).ops()
    with DeviceState(30, 32) as ref, DeviceState(30, 32) as st:
        ref.apply_ops(ops, options(4, staged=False))
        stats = st.apply_ops(ops, options(6, staged=False, math="tensor"))
        assert stats["passes"] < 0.6 * len(ops)
        assert ref.max_abs_diff(st) < 1e-6


def test_tensor_core_plain_plans_relabel_low_bits():
    """Tensor-core plain plans may first move three qubits onto index bits
    1-3 (the bits whose targets slow the passes down): free on a |0...0>
    state, one swap pass otherwise, and again when a plan runs on a state
    left in another layout. Amplitudes in logical order match a complex128
    run either way."""
    from qevedo_simulator_b200 import Plan, library

    relabelled = 0
    for rows, cols, depth, seed in [(4, 5, 20, 5), (4, 6, 20, 2024), (3, 7, 16, 9)]:
        n = rows * cols
        ops = library.random_grid_circuit(rows, cols, depth, seed).ops()
        psi = random_state(np.random.Generator(np.random.PCG64(seed)), n)
        opts = options(6, staged=False, math="tensor")
        with DeviceState(n, 64) as ref, DeviceState(n, 32) as st, Plan(ops, n, 32, opts) as plan:
            ref.apply_ops(ops, options(4, staged=False))
            st.execute(plan)  # from |0...0>
            relabelled += st.layout() != list(range(n))
            assert ref.max_abs_diff(st) < 1e-6, (n, "zero start")
            expected = ref.amplitudes()
            assert np.abs(st.amplitudes() - expected).max() < 1e-6
            ref.set_amplitudes(psi)
            ref.apply_ops(ops, options(4, staged=False))
            st.set_amplitudes(psi)
            st.apply_ops(ops, opts)  # from a general state
            assert ref.max_abs_diff(st) < 1e-6, (n, "general start")
            st.set_amplitudes(psi)
            st.swap_physical([(1, n - 1)])
            st.execute(plan)  # from a state in another layout
            assert ref.max_abs_diff(st) < 1e-6, (n, "other layout")
    assert relabelled >= 1


@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("kind", ["grid", "mixed", "qft", "gates"])
def test_plain_passes_applying_groups_gate_by_gate(oracle, bits, kind):
    """math="gates": each fused 4-5 qubit group runs as one pass that applies
    its member gates in registers (merged diagonals as one phase vector or
    sign mask, controls as pair masks); groups that do not qualify keep the
    product-matrix kernel. Same results as the naive oracle."""
    from qevedo_simulator_b200 import library

    n = 15
    if kind == "grid":
        ops = library.random_grid_circuit(3, 5, 12, seed=4).ops()
    elif kind == "mixed":
        ops = library.mixed_ops(n, 8, seed=6)
    elif kind == "qft":
        ops = library.qft(n).ops()
    else:
        ops = library.random_gate_circuit(n, 150, seed=12).ops()
    initial = random_state(np.random.Generator(np.random.PCG64(21)), n)
    expected = oracle.naive_apply_ops(initial, ops)
    for fuse in (4, 5):
        with DeviceState(n, bits) as st:
            st.set_amplitudes(initial)
            stats = st.apply_ops(ops, options(fuse, staged=False, math="gates"))
            assert max_distance(st.amplitudes(), expected) < TOL[bits] * 50, (kind, fuse, stats)


@pytest.mark.parametrize("n", [14, 17])
def test_tensor_core_pair_passes_match_naive(oracle, n):
    """Two fused 6-qubit gates in one pass (math="tensor_pairs"): targets
    disjoint or shared, on bit 0 or bits 0 and 1 for either gate (16- and
    32-byte accesses on the load or the store side), on bits 1-3, low and
    high, in any order. Where both gates' warp accesses stay coalesced the
    pair runs as one pass of kind 5 (the planner's features mark it), else as
    two single passes; every case matches the naive oracle."""
    from qevedo_simulator_b200 import costmodel

    rng = np.random.Generator(np.random.PCG64(900 + n))
    paired = 0
    initial = random_state(rng, n)
    h = n - 1
    layouts = [([0, 1, 2, 3, 4, 5], [6, 7, 8, 9, 10, 11]), ([6, 7, 8, 9, 10, 11], [0, 1, 2, 3, 4, 5]),
               ([0, 5, 9, 11, 12, h], [1, 5, 7, 9, 10, 12]), ([h, 2, 7, 4, 9, 3], [0, 1, h, 8, 6, 4]),
               ([1, 2, 3, 8, 10, 12], [2, 3, 4, 5, 6, 7]), ([7, 8, 9, 10, 11, 12], [h, h - 1, h - 2, 4, 5, 6]),
               ([0, 1, 3, 6, 9, 12], [0, 2, 4, 6, 8, 10]), ([5, 6, 7, 8, 9, 10], [5, 6, 7, 8, 9, 11])]
    for a, b in layouts:
        ops = [Op(a, [], random_unitary(rng, 6)), Op(b, [], random_unitary(rng, 6))]
        expected = oracle.naive_apply_ops(initial, ops)
        with DeviceState(n, 32) as st:
            st.set_amplitudes(initial)
            st.set_pass_timing(True)
            stats = st.apply_ops(ops, options(6, staged=False, math="tensor_pairs"))
            kinds = list(st.pass_times()[2])
            err = max_distance(st.amplitudes(), expected) / np.max(np.abs(expected))
        assert err < TC_REL_TOL, (n, a, b, err)
        rows = costmodel.plan_features(ops, n, options(6, staged=False, math="tensor_pairs"))
        if rows.shape[0] == 1 and rows[0, 21] == 1:
            paired += 1
            assert kinds == [5] and stats["passes"] == 1 and stats["kernels"] == 2, (a, b, kinds, stats)
        else:
            assert 5 not in kinds and stats["passes"] == 2, (a, b, kinds, stats)
    assert paired >= 4


@pytest.mark.parametrize("kind", ["grid", "mixed", "qft", "gates"])
def test_tensor_core_pair_circuits(oracle, kind):
    """Whole circuits with pair passes (tensor_pairs at fusion 6; groups with
    controls or fewer than 6 qubits keep single passes), one-shot from a
    random state and as a plan run from |0...0> (its zero-start prefix stays
    single), against the naive oracle."""
    from qevedo_simulator_b200 import Plan, library

    n = 16
    if kind == "grid":
        ops = library.random_grid_circuit(4, 4, 14, seed=61).ops()
    elif kind == "mixed":
        ops = library.mixed_ops(n, 8, seed=62)
    elif kind == "qft":
        ops = library.qft(n).ops()
    else:
        ops = library.random_gate_circuit(n, 150, seed=63).ops()
    initial = random_state(np.random.Generator(np.random.PCG64(64)), n)
    expected = oracle.naive_apply_ops(initial, ops)
    opts = options(6, staged=False, math="tensor_pairs")
    with DeviceState(n, 32) as st:
        st.set_amplitudes(initial)
        st.set_pass_timing(True)
        st.apply_ops(ops, opts)
        err = max_distance(st.amplitudes(), expected) / np.max(np.abs(expected))
        assert err < TC_CIRCUIT_TOL, (kind, err)
        if kind in ("grid", "qft"):
            assert 5 in set(st.pass_times()[2].tolist())
        zero = oracle.naive_statevector(ops, n)
        with Plan(ops, n, 32, opts) as plan:
            st.zero()
            st.execute(plan)
            err = max_distance(st.amplitudes(), zero) / np.max(np.abs(zero))
        assert err < TC_CIRCUIT_TOL, (kind, "plan", err)


@pytest.mark.parametrize("bits", [32, 64])
def test_low_qubit_gates_by_warp_shuffles(oracle, bits):
    """Dense 1-3 qubit gates whose targets all lie in index bits 0-4 (the lanes
    of a warp row), with no controls or controls above bit 4, run as warp
    shuffles within rows of 32 amplitudes (k_dense_lanes): every target
    layout against the naive oracle, from one row (5 qubits) to many."""
    rng = np.random.Generator(np.random.PCG64(77 + bits))
    for n in (5, 6, 9, 14, 18):
        initial = random_state(rng, n)
        for case in range(12):
            k = 1 + case % 3
            qubits = [int(q) for q in rng.permutation(5)[:k]]
            high = list(range(5, n))
            nc = int(rng.integers(0, min(len(high), 2) + 1))
            controls = [(int(q), bool(rng.integers(2))) for q in rng.permutation(high)[:nc]] if high else []
            m = random_unitary(rng, k)
            expected = oracle.naive_apply_ops(initial, [Op(qubits, controls, m)])
            with DeviceState(n, bits) as st:
                st.set_amplitudes(initial)
                st.apply(m, qubits, controls)
                assert max_distance(st.amplitudes(), expected) < TOL[bits], (n, qubits, controls)
