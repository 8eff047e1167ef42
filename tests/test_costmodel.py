"""Learned cost model, host side: the planner's per-pass features (no
device work)."""

import numpy as np

from qevedo_simulator_b200 import costmodel, library


def test_features_describe_each_pass():
    ops = library.random_grid_circuit(4, 5, 8, seed=3).ops()
    for name, opts in costmodel.candidates():
        f = costmodel.plan_features(ops, 20, opts)
        assert f.shape[1] == costmodel.FEATURES and f.shape[0] >= 1
        assert np.all(f[:, 0] == 1.0) and np.allclose(f[:, 1], 20 / 32)
        kinds = f[:, 2:6]
        assert np.all(kinds.sum(axis=1) == 1.0)  # exactly one pass kind
        if name.startswith("plain"):
            assert np.all(f[:, 2] == 1.0)
            assert np.all(f[:, 6] > 0)  # targets
            tensor = f[:, 22] + f[:, 23] > 0
            if name.startswith("plain-tensor"):
                assert np.any(tensor) and np.all(f[tensor, 6] >= 4 / 6 - 1e-6)
            else:
                assert not np.any(tensor)
        elif name == "staged-cuda":
            assert np.all(f[:, 3] == 1.0) and np.all(f[:, 26] > 0)  # register passes
        else:
            assert np.all(f[:, 4] + f[:, 3] == 1.0)
        # Deterministic.
        assert np.array_equal(f, costmodel.plan_features(ops, 20, opts))


def test_wider_fusion_means_fewer_plain_passes():
    ops = library.mixed_ops(12, 6, seed=1)
    counts = [costmodel.plan_features(ops, 12, o).shape[0] for _, o in costmodel.candidates()[:4]]
    assert counts == sorted(counts, reverse=True) and counts[0] > counts[-1]


def test_mixed_ops_have_one_to_three_controls():
    ops = library.mixed_ops(10, 30, seed=2)
    controls = {len(o.controls) for o in ops if len(o.targets) == 1 and o.controls and
                np.allclose(o.matrix, [[0, 1], [1, 0]])}
    assert controls >= {1, 2, 3}


def test_tensor_core_plain_passes_are_planned_where_they_fit():
    """math="tensor" without staging: dense fused gates of 4-6 qubits go to
    the tensor-core plain pass on complex64 states when at least 8192
    amplitudes stay selected (2^(n - controls) >= 2^13); narrower gates,
    complex128 states and heavily controlled gates keep the CUDA-core pass."""
    from qevedo_simulator_b200 import Op, options

    rng = np.random.default_rng(3)

    def unitary(k):
        q, _ = np.linalg.qr(rng.normal(size=(2 ** k, 2 ** k)) + 1j * rng.normal(size=(2 ** k, 2 ** k)))
        return q

    def tensor_plain(ops, n, bits=32):
        rows = costmodel.plan_features(ops, n, options(6, staged=False, math="tensor"), bits)
        return [bool(r[2] == 1 and r[22] + r[23] > 0) for r in rows]

    assert tensor_plain([Op([0, 1, 2, 3], [], unitary(4))], 13) == [True]
    assert tensor_plain([Op([5, 1, 9, 3, 0, 7], [], unitary(6))], 20) == [True]
    assert tensor_plain([Op([0, 1, 2], [], unitary(3))], 20) == [False]
    assert tensor_plain([Op([0, 1, 2, 3], [], unitary(4))], 12) == [False]
    assert tensor_plain([Op([0, 1, 2, 3], [(4, True)], unitary(4))], 13) == [False]
    assert tensor_plain([Op([0, 1, 2, 3], [(4, True)], unitary(4))], 14) == [True]
    assert tensor_plain([Op([0, 1, 2, 3], [], unitary(4))], 16, bits=64) == [False]
    assert tensor_plain([Op([0, 1, 2, 3], [], np.diag(np.exp(1j * rng.normal(size=16))))], 16) == [False]
    ops = library.random_grid_circuit(4, 4, 14, seed=31).ops()
    assert sum(tensor_plain(ops, 16)) >= 10


def test_tensor_core_fusion_search_takes_fewer_passes():
    """Plans of fused 6-qubit tensor-core passes search their fusion beyond
    the greedy one (seed lookahead, then beam searches over the seeds): on the
    30-qubit depth-20 grid circuit the plan takes at most 46 passes, against
    50 for the best lookahead fusion and 81 for the plain fusion-4 plan on
    the CUDA cores."""
    from qevedo_simulator_b200 import options

    ops = library.random_grid_circuit(5, 6, 20, seed=2024).ops()
    tensor6 = costmodel.plan_features(ops, 30, options(6, staged=False, math="tensor")).shape[0]
    plain4 = costmodel.plan_features(ops, 30, options(4, staged=False)).shape[0]
    assert tensor6 <= 46 and plain4 > tensor6 + 30


def test_commuting_diagonal_gates_shorten_qft_plans():
    """Where some qubit meets two diagonal gates in a row (QFT's controlled
    phases), the tensor-core plan's fusion may also take a diagonal gate into
    a group ahead of skipped diagonal gates on its qubits (they commute): the
    30-qubit QFT takes at most 46 passes at fusion 6 instead of 68. The grid
    circuit, whose diagonal CZ gates always sit between non-diagonal gates,
    plans as before."""
    from qevedo_simulator_b200 import options

    opts = options(6, staged=False, math="tensor")
    assert costmodel.plan_features(library.qft(30).ops(), 30, opts).shape[0] <= 46
    assert costmodel.plan_features(library.random_grid_circuit(5, 6, 20, seed=2024).ops(), 30, opts).shape[0] <= 46
