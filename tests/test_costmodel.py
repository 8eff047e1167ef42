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
