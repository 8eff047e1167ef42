"""Learned cost model on the device: the MLP's kernels against a float64
numpy restatement of the same network, training, and the planner it drives
against the greedy default (the reference's only planner, src/fusion.rs and
src/blocking.rs)."""

import numpy as np
import pytest

from qevedo_simulator_b200 import costmodel, library

pytestmark = pytest.mark.gpu


def numpy_mlp(params, x, inputs, hidden):
    """Forward and backward of the same network in float64."""
    p = params.astype(np.float64)
    o = 0
    W1 = p[o:o + hidden * inputs].reshape(hidden, inputs); o += hidden * inputs
    b1 = p[o:o + hidden]; o += hidden
    W2 = p[o:o + hidden * hidden].reshape(hidden, hidden); o += hidden * hidden
    b2 = p[o:o + hidden]; o += hidden
    W3 = p[o:o + hidden].reshape(1, hidden); o += hidden
    b3 = p[o:o + 1]
    X = x.astype(np.float64)
    Z1 = X @ W1.T + b1; A1 = np.maximum(Z1, 0)
    Z2 = A1 @ W2.T + b2; A2 = np.maximum(Z2, 0)
    y = (A2 @ W3.T + b3)[:, 0]

    def grads(t):
        t = t.astype(np.float64)
        dy = 2 * (y - t) / len(t)
        dW3 = dy[None, :] @ A2; db3 = [dy.sum()]
        dZ2 = (dy[:, None] @ W3) * (A2 > 0)
        dW2 = dZ2.T @ A1; db2 = dZ2.sum(0)
        dZ1 = (dZ2 @ W2) * (A1 > 0)
        dW1 = dZ1.T @ X; db1 = dZ1.sum(0)
        g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
        return float(np.mean((y - t) ** 2)), g

    return y, grads


@pytest.mark.parametrize("inputs,hidden,rows", [(32, 128, 300), (7, 20, 33)])
def test_kernels_match_numpy(inputs, hidden, rows):
    rng = np.random.Generator(np.random.PCG64(inputs + hidden))
    x = rng.standard_normal((rows, inputs)).astype(np.float32)
    t = rng.standard_normal(rows).astype(np.float32)
    with costmodel.MLP(inputs, hidden, seed=5) as m:
        params = m.get_params()
        assert params.size == hidden * inputs + hidden + hidden * hidden + hidden + hidden + 1
        y_ref, grads = numpy_mlp(params, x, inputs, hidden)
        y = m.forward(x)
        assert np.allclose(y, y_ref, rtol=1e-4, atol=1e-4 * np.abs(y_ref).max())
        loss, g = m.gradients(x, t)
        loss_ref, g_ref = grads(t)
        assert loss == pytest.approx(loss_ref, rel=1e-4)
        assert np.abs(g - g_ref).max() <= 1e-4 * np.abs(g_ref).max() + 1e-7
        # set/get round trip
        m.set_params(params * 0.5)
        assert np.array_equal(m.get_params(), params * np.float32(0.5))


def test_kernels_over_a_million_rows():
    """Row-parallel launches take rows in the grid's y dimension (at most
    65535 blocks of 16 rows): more rows than that (training sets of over a
    million pass timings) go in chunks. Forward, gradients and the final
    training loss over 1.1M rows match numpy."""
    rows, inputs, hidden = 1_100_000, 7, 20
    rng = np.random.Generator(np.random.PCG64(17))
    x = rng.standard_normal((rows, inputs)).astype(np.float32)
    t = rng.standard_normal(rows).astype(np.float32)
    with costmodel.MLP(inputs, hidden, seed=5) as m:
        params = m.get_params()
        y_ref, grads = numpy_mlp(params, x, inputs, hidden)
        y = m.forward(x)
        assert np.allclose(y, y_ref, rtol=1e-4, atol=1e-4 * np.abs(y_ref).max())
        loss, g = m.gradients(x, t)
        loss_ref, g_ref = grads(t)
        assert loss == pytest.approx(loss_ref, rel=1e-3)
        assert np.abs(g - g_ref).max() <= 1e-3 * np.abs(g_ref).max() + 1e-6
        final = m.train(x, t, epochs=1, batch=4096, lr=1e-3, seed=3)
        assert np.isfinite(final) and final < 1.05 * loss


def test_training_fits_a_smooth_function():
    rng = np.random.Generator(np.random.PCG64(9))
    x = rng.uniform(0, 1, (2048, 32)).astype(np.float32)
    w = rng.standard_normal(32)
    t = (np.tanh(x @ w) + 0.5 * x[:, 3] * x[:, 7]).astype(np.float32)
    with costmodel.MLP(32, 128, seed=1) as m:
        before, _ = m.gradients(x, t)
        after = m.train(x, t, epochs=60, batch=128, lr=2e-3, seed=3)
        assert after < 0.05 * before and after < 5e-3
        again = costmodel.MLP(32, 128, seed=1)
        assert again.train(x, t, epochs=60, batch=128, lr=2e-3, seed=3) == after  # deterministic
        again.close()


def test_learned_planner_beats_the_greedy_default_on_held_out_circuits():
    """Trained on the engine's own timings of small mixed circuits; on
    held-out circuits its pick runs faster than the greedy default, and the
    measured judge never keeps a slower plan."""
    n = 20
    train = [library.mixed_ops(n, d, seed=s) for s, d in zip(range(16), [6, 10, 14, 18] * 4)]
    x, t = costmodel.collect(train, n)
    model = costmodel.CostModel(costmodel.MLP(seed=2))
    loss = model.fit(x, t, epochs=150, batch=64, lr=2e-3)
    assert loss < 0.1
    picked, default = 0.0, 0.0
    from qevedo_simulator_b200 import DeviceState
    with DeviceState(n, 32) as st:
        for s in range(100, 104):
            ops = library.mixed_ops(n, 12, seed=s)
            name, opts, sec, dsec = costmodel.choose_measured(model, ops, n, st)
            assert sec <= dsec
            _, o2, _ = model.choose(ops, n)
            p, _ = costmodel.measure_plan(ops, n, o2, st)
            picked += p
            default += dsec
    assert picked < default


def test_learned_planner_on_the_product_path(oracle):
    """The committed cost model, registered in the library: its choice
    (qvdg_plan_choose, host planning and one forward of the device MLP over
    every candidate's passes) equals the Python ranking of the same model;
    a plan built with planner="learned" carries that choice; run() and
    statevector() with default settings run the learned pick and match the
    naive oracle; with the model cleared the fallback settings run."""
    from qevedo_simulator_b200 import Plan, _native, options, run, statevector
    from qevedo_simulator_b200._abi import settings_dict

    n = 20
    c = library.random_grid_circuit(4, 5, 12, seed=3)
    ops = c.ops()
    assert _native.ensure_cost_model()
    chosen, pred = _native.plan_choose(ops, n, from_zero=False)
    model = costmodel.CostModel.load()
    by_name = {name: sec for name, _, sec in model.rank(ops, n)}
    names = [name for name, _ in costmodel.candidates()]
    assert len(pred) == len(names)
    for name, p in zip(names, pred):
        assert p == pytest.approx(by_name[name], rel=1e-5), name
    assert settings_dict(chosen) == settings_dict(dict(costmodel.candidates())[names[int(np.argmin(pred))]])
    pick0, _ = _native.plan_choose(ops, n, from_zero=True)
    with Plan(ops, n, 32, options(planner="learned")) as plan:
        assert plan.info()["settings"] == settings_dict(pick0)
    expected = oracle.naive_statevector(ops, n)
    assert np.abs(statevector(c, precision="single") - expected).max() <= 1e-6
    cand = [settings_dict(o) for o in _native.planner_candidates(32)]
    res = run(c.copy().measure_all(), 200, seed=1)
    assert res.stats["settings"] in cand and sum(res.counts.values()) == 200
    from qevedo_simulator_b200 import DeviceState

    try:
        _native.clear_cost_model()  # run() would register it again; the C ABI alone falls back
        with DeviceState(n, 32) as st:
            stats = st.apply_ops(ops, options(planner="learned"))
        assert stats["settings"] == {"max_fused_qubits": 4, "staged": True, "tile_qubits": 0, "math": "fp32"}
    finally:
        _native.ensure_cost_model()
