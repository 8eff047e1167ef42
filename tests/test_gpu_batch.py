"""Batched layered circuits (qvdg_batch) against the naive oracle and the
per-circuit path: <Z_q> for every qubit of every circuit from one persistent,
graph-captured launch. Per circuit this is what the reference computes with
apply_ops (src/simulator.rs:122-147) and probability_one per qubit
(src/measure.rs:43-65)."""

import numpy as np
import pytest

from qevedo_simulator_b200 import Batch, Circuit, DeviceState, library, options

pytestmark = pytest.mark.gpu

# complex64 state and gates, sums in f64: |delta <Z>| well below 1e-5 for
# ~100-300 gate applications per amplitude.
Z_TOL = 2e-5


def z_of(psi, n):
    p = np.abs(psi) ** 2
    idx = np.arange(1 << n)
    return np.array([p.sum() - 2 * p[((idx >> q) & 1) == 1].sum() for q in range(n)])


def layered_circuit(n, gates, entangler):
    c = Circuit(n)
    for layer in gates:
        for q in range(n):
            c.unitary(layer[q], [q])
        for q in range(n - 1):
            if entangler == "cx":
                c.cx(q, q + 1)
            elif entangler == "cz":
                c.cz(q, q + 1)
    return c


def layered_ops(n, gates, entangler):
    """The same circuit as ops (matrices need not be unitary)."""
    from qevedo_simulator_b200 import Op

    x = np.array([[0, 1], [1, 0]], dtype=complex)
    z = np.diag([1, -1]).astype(complex)
    ops = []
    for layer in gates:
        ops += [Op([q], [], layer[q]) for q in range(n)]
        if entangler != "none":
            ops += [Op([q + 1], [(q, True)], x if entangler == "cx" else z) for q in range(n - 1)]
    return ops


def test_small_batch_matches_the_naive_oracle(oracle):
    specs = library.hea_batch(40, seed=3, widths=(1, 13), layers=(0, 6))
    circuits, expected = [], []
    for i, (w, layers, seed) in enumerate(specs):
        ent = ("cx", "cz", "none")[i % 3]
        g = library.hea_layers(w, layers, seed)
        circuits.append((w, g, ent))
        expected.append(z_of(oracle.naive_statevector(layered_circuit(w, g, ent).ops(), w), w))
    with Batch(circuits, tile_qubits=13, threads=256) as b:
        flat, sec = b.run()
        assert sec > 0
        for i, (got, exp) in enumerate(zip(b.split(flat), expected)):
            assert np.abs(got - exp).max() < Z_TOL, (i, specs[i])


@pytest.mark.parametrize("tile,threads", [(12, 128), (13, 256), (14, 512)])
def test_wide_circuits_match_the_per_circuit_path(tile, threads):
    """Circuits wider than the tile run in HBM slots (two double-buffered
    tile passes per layer on tiles of L - 1 qubits); compared with
    complex128 runs of the same circuits through apply_ops on single
    states."""
    specs = [(15, 3, 1), (17, 4, 2), (18, 2, 3), (20, 3, 4), (min(22, 2 * tile - 3), 2, 5), (tile + 1, 3, 6),
             (min(2 * tile - 3, 24), 2, 7)]
    circuits, expected = [], []
    for i, (w, layers, seed) in enumerate(specs):
        ent = "cz" if i == 2 else "cx"
        g = library.hea_layers(w, layers, seed)
        circuits.append((w, g, ent))
        with DeviceState(w, 64) as st:
            st.apply_ops(layered_circuit(w, g, ent).ops(), options(4, staged=False))
            expected.append(st.expect_z_all())
    with Batch(circuits, tile_qubits=tile, threads=threads) as b:
        info = b.info()
        assert (info["tile_qubits"], info["threads"]) == (tile, threads) and info["candidates"] == 0
        flat, _ = b.run()
        for i, (got, exp) in enumerate(zip(b.split(flat), expected)):
            assert np.abs(got - exp).max() < Z_TOL, (i, specs[i], np.abs(got - exp).max())


def test_autotuned_graph_replays_and_new_parameters():
    specs = library.hea_batch(96, seed=11, widths=(10, 16), layers=(2, 5))
    circuits = [(w, library.hea_layers(w, l, s), "cx") for w, l, s in specs]
    with Batch(circuits) as b:
        info = b.info()
        tuning = b.tuning()
        assert info["candidates"] == len(tuning) >= 2
        best = min(tuning, key=lambda t: t[2])
        assert (info["tile_qubits"], info["threads"]) == best[:2]
        first, _ = b.run()
        second, _ = b.run()
        assert np.array_equal(first, second)  # deterministic reductions
        # New angles through set_gates: the captured graph reads them.
        new = [library.hea_layers(w, l, s + 1) for w, l, s in specs]
        b.set_gates(new)
        third, _ = b.run()
        assert not np.allclose(third, first)
        for i in (0, 17, 95):
            w = specs[i][0]
            with DeviceState(w, 64) as st:
                st.apply_ops(layered_circuit(w, new[i], "cx").ops(), options(4, staged=False))
                assert np.abs(b.split(third)[i] - st.expect_z_all()).max() < Z_TOL


def test_hea_circuits_match_their_gate_by_gate_form(oracle):
    """library.hea_layers gives the gates of library.hea_circuit."""
    for w, l, s in [(6, 3, 1), (9, 4, 2)]:
        expected = z_of(oracle.naive_statevector(library.hea_circuit(w, l, s).ops(), w), w)
        with Batch([(w, library.hea_layers(w, l, s), "cx")], tile_qubits=12, threads=128) as b:
            got, _ = b.run()
        assert np.abs(got - expected).max() < Z_TOL


@pytest.mark.parametrize("tile", [12, 14])
def test_every_gate_form(oracle, tile):
    """Gate records in every form the host encodes: Haar-random SU(2) (left
    and right phases around a real rotation), diagonal and anti-diagonal
    gates, RZ.RY (left phases only), real rotations (no phases), and a
    non-unitary matrix, which keeps its circuit on the generic 2x2 path;
    narrow circuits in shared memory and wide ones in HBM slots."""
    rng = np.random.Generator(np.random.PCG64(77))
    s = np.array([[1, 0], [0, 1j]])
    x = np.array([[0, 1], [1, 0]], dtype=complex)
    shear = np.array([[1, 0.25], [0, 1]], dtype=complex)

    def gates(w, layers, kind):
        out = np.empty((layers, w, 2, 2), dtype=complex)
        for layer in range(layers):
            for q in range(w):
                if kind == "haar":
                    out[layer, q] = library.haar_su2(rng)
                elif kind == "mixed":
                    out[layer, q] = (s, x, library.haar_su2(rng), np.eye(2))[(layer + q) % 4]
                elif kind == "real":
                    t = rng.random() * 6.28
                    out[layer, q] = [[np.cos(t), -np.sin(t)], [np.sin(t), np.cos(t)]]
                else:  # one non-unitary gate, the rest Haar
                    out[layer, q] = shear if (layer, q) == (0, 1) else library.haar_su2(rng)
        return out

    specs = [(9, 3, "haar", "cx"), (11, 4, "mixed", "cz"), (10, 3, "real", "cx"), (8, 3, "shear", "cx"),
             (tile + 3, 3, "haar", "cx"), (tile + 2, 2, "mixed", "cz"), (tile + 1, 2, "shear", "none")]
    circuits, expected = [], []
    for w, layers, kind, ent in specs:
        g = gates(w, layers, kind)
        circuits.append((w, g, ent))
        expected.append(z_of(oracle.naive_statevector(layered_ops(w, g, ent), w), w))
    with Batch(circuits, tile_qubits=tile, threads=256) as b:
        flat, _ = b.run()
        for i, (got, exp) in enumerate(zip(b.split(flat), expected)):
            assert np.abs(got - exp).max() < Z_TOL, (i, specs[i])
        # New matrices of another form through set_gates.
        new = [gates(w, layers, "haar" if kind != "haar" else "real") for w, layers, kind, _ in specs]
        b.set_gates(new)
        flat, _ = b.run()
        for i, (w, layers, kind, ent) in enumerate(specs):
            exp = z_of(oracle.naive_statevector(layered_ops(w, new[i], ent), w), w)
            assert np.abs(b.split(flat)[i] - exp).max() < Z_TOL, ("set_gates", i)


def test_invalid_batches_are_rejected():
    g = np.tile(np.eye(2), (1, 3, 1, 1))
    with pytest.raises(ValueError, match="num_qubits"):
        Batch([(25, np.tile(np.eye(2), (1, 25, 1, 1)), "cx")])
    with pytest.raises(ValueError, match="entangler"):
        Batch([(3, g, 7)])
    with pytest.raises(ValueError, match="tile_qubits"):
        Batch([(3, g, "cx")], tile_qubits=9)
    with pytest.raises(ValueError, match="too small"):
        Batch([(24, np.tile(np.eye(2), (1, 24, 1, 1)), "cx")], tile_qubits=12)
    with Batch([(3, g, "cx")], tile_qubits=12, threads=128) as b:
        with pytest.raises(ValueError, match="matrices"):
            b.set_gates([np.tile(np.eye(2), (2, 3, 1, 1))])
