"""The planner's fused programs against the naive oracle (host only): every
plain plan's passes, read back as ops (qvdg_plan_fused_ops, the counterpart
of the reference's `fuse`, src/fusion.rs:63-170), applied in order to a
random state give the circuit's own result. This covers the greedy fusion,
the seed-lookahead and beam searches, the commuting-diagonal family (QFT,
controlled phases) and both scorings (for a general state, and from
|0...0>)."""

import numpy as np
import pytest

from conftest import random_state
from qevedo_simulator_b200 import costmodel, library, options


def _circuit(kind: str, n: int):
    if kind == "grid":
        return library.random_grid_circuit(3, 5, 10, seed=21).ops()
    if kind == "qft":
        return library.qft(n).ops()
    if kind == "mixed":
        return library.mixed_ops(n, 5, seed=22)
    return library.random_gate_circuit(n, 160, seed=23).ops()


@pytest.mark.parametrize("kind", ["grid", "qft", "mixed", "random"])
def test_fused_programs_equal_the_circuit(oracle, kind):
    n = 15 if kind == "grid" else 14
    ops = _circuit(kind, n)
    psi = random_state(np.random.Generator(np.random.PCG64(40)), n)
    expected = oracle.naive_apply_ops(psi, ops)
    plans = [options(4, staged=False), options(5, staged=False, math="tensor"),
             options(6, staged=False, math="tensor"), options(5, staged=False, math="gates"),
             options(6, staged=False, math="tensor_pairs")]
    for opts in plans:
        for from_zero in (False, True):
            fused = costmodel.fused_ops(ops, n, opts, from_zero=from_zero)
            assert len(fused) <= len(ops)
            assert all(len(f.targets) <= opts.max_fused_qubits for f in fused if f.matrix.shape[0] > 1)
            got = oracle.naive_apply_ops(psi, fused)
            err = np.max(np.abs(got - expected))
            assert err < 1e-10, (kind, opts.max_fused_qubits, opts.math, from_zero, err)
        # The general-state fusion is the one the cost model's features describe.
        rows = costmodel.plan_features(ops, n, opts)
        if opts.math != 2:  # a pair pass (feature 21) applies two fused ops
            assert rows.shape[0] + int(np.sum(rows[:, 21] == 1)) == len(costmodel.fused_ops(ops, n, opts))


def test_fused_ops_of_an_empty_circuit_and_staged_plans():
    assert costmodel.fused_ops([], 14, options(6, staged=False, math="tensor")) == []
    with pytest.raises(ValueError, match="plain plans only"):
        costmodel.fused_ops(library.qft(14).ops(), 14, options(4, staged=True))


def test_pair_passes_in_plans():
    """math="tensor_pairs" keeps the tensor-core fusion (the same fused ops;
    a pass may move up past passes it commutes with to meet its partner) and
    merges fused 6-qubit passes without controls into pair passes (features
    marked) only where both gates' warp accesses stay coalesced: two gates on
    high, disjoint qubits (13-bit iteration with one low bit) stay single;
    gates that leave bits 0-3 free pair."""
    import numpy as np

    from qevedo_simulator_b200 import Op

    ops = library.random_grid_circuit(5, 6, 20, seed=2024).ops()
    single = options(6, staged=False, math="tensor")
    pairs = options(6, staged=False, math="tensor_pairs")
    a = costmodel.plan_features(ops, 30, single)
    b = costmodel.plan_features(ops, 30, pairs)
    marked = int(np.sum(b[:, 21] == 1))
    assert marked >= 1 and b.shape[0] == a.shape[0] - marked
    fa = costmodel.fused_ops(ops, 30, single)
    fb = costmodel.fused_ops(ops, 30, pairs)
    # the same fused ops; a pair's second pass may move up past passes it
    # commutes with (no shared qubit)
    assert sorted(map(tuple, (f.targets for f in fa))) == sorted(map(tuple, (f.targets for f in fb)))
    rng = np.random.Generator(np.random.PCG64(3))
    u = np.linalg.qr(rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64)))[0]  # dense
    scattered = [Op([8, 10, 12, 14, 16, 18], [], u), Op([9, 11, 13, 15, 17, 19], [], u)]
    assert costmodel.plan_features(scattered, 24, pairs).shape[0] == 2
    overlapping = [Op([8, 10, 12, 14, 16, 18], [], u), Op([8, 10, 12, 15, 17, 19], [], u)]
    rows = costmodel.plan_features(overlapping, 24, pairs)
    assert rows.shape[0] == 1 and rows[0, 21] == 1


def test_layout_from_zero_pairs_more_passes():
    """From |0...0> a plan may take any layout: the planner puts the qubits
    touched last on the top bits, an early-touched qubit on bit 0, and
    permutes the bits above 3 so that more passes pair (the pairing's layout
    test on bit masks). The 30-qubit grid circuit (5x6, depth 20) then runs
    in 30 passes: 11 zero-start passes (single, so they keep their cheap
    variants) and 15 pairs among the other 23 fused gates. Single-pass
    (math="tensor") plans make no pairs."""
    import numpy as np

    ops = library.random_grid_circuit(5, 6, 20, seed=2024).ops()
    pairs = options(6, staged=False, math="tensor_pairs")
    zero = costmodel.plan_features(ops, 30, pairs, from_zero=True)
    pz = int(np.sum(zero[:, 21] == 1))
    assert pz >= 14, pz
    assert zero.shape[0] <= 31
    # every pass applies one fused op or two (a pair)
    assert zero.shape[0] + pz == len(costmodel.fused_ops(ops, 30, pairs, from_zero=True))
    single = options(6, staged=False, math="tensor")
    assert int(np.sum(costmodel.plan_features(ops, 30, single, from_zero=True)[:, 21] == 1)) == 0


@pytest.mark.parametrize("kind", ["qft", "mixed"])
def test_programs_from_zero_apply_every_fused_op(kind):
    """From |0...0> (zero-start passes, layout search, pair passes) a plan
    still applies each fused op in exactly one pass: the passes plus the
    pairs (a pair applies two ops) give the fused-op count of the same
    from-zero fusion, for the QFT and for mixed circuits."""
    import numpy as np

    n = 26
    ops = library.qft(n).ops() if kind == "qft" else library.mixed_ops(n, 8, seed=4)
    for opts in (options(6, staged=False, math="tensor_pairs"), options(6, staged=False, math="tensor"),
                 options(5, staged=False, math="tensor")):
        rows = costmodel.plan_features(ops, n, opts, from_zero=True)
        fused = costmodel.fused_ops(ops, n, opts, from_zero=True)
        pairs = int(np.sum(rows[:, 21] == 1))
        assert rows.shape[0] + pairs == len(fused), (kind, opts.math, opts.max_fused_qubits)
