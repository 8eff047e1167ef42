"""Generate the golden fixtures in this folder.

    python tests/golden/make_golden.py

The reference ships no golden vectors (its tests compare against its naive
simulator, src/reference.rs). These fixtures hold small circuits with:
  - analytic amplitudes where a closed form exists (QFT of a basis state,
    GHZ), and otherwise the naive f64 oracle's amplitudes;
  - for one circuit, uniforms and the reference sampler's outcomes (the
    oracle's restatement of src/measure.rs:104-174) in f64.
Each file stores the lowered ops (targets, controls, matrices) so that every
engine runs exactly the same gates.
"""

from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def ops_to_arrays(ops):
    return {
        "ntargets": np.array([len(o.targets) for o in ops], dtype=np.int64),
        "targets": np.array([q for o in ops for q in o.targets], dtype=np.int64),
        "ncontrols": np.array([len(o.controls) for o in ops], dtype=np.int64),
        "controls": np.array([q for o in ops for q, _ in o.controls] or [0], dtype=np.int64),
        "values": np.array([int(v) for o in ops for _, v in o.controls] or [0], dtype=np.int64),
        "matrices": np.concatenate([np.asarray(o.matrix, dtype=np.complex128).reshape(-1) for o in ops]),
    }


def ops_from_fixture(z):
    """(ops, num_qubits, initial state) from a loaded fixture."""
    sys.path.insert(0, ROOT)
    from qevedo_simulator_b200.circuit import Op

    ops = []
    tp = cp = mp = 0
    for nt, nc in zip(z["ntargets"].tolist(), z["ncontrols"].tolist()):
        targets = z["targets"][tp:tp + nt].tolist()
        controls = [(int(q), bool(v)) for q, v in zip(z["controls"][cp:cp + nc], z["values"][cp:cp + nc])]
        dim = 1 << nt
        m = z["matrices"][mp:mp + dim * dim].reshape(dim, dim)
        ops.append(Op(targets, controls, m))
        tp, cp, mp = tp + nt, cp + nc, mp + dim * dim
    return ops, int(z["num_qubits"]), z["initial"]


def qft_basis(n: int, x: int) -> np.ndarray:
    N = 1 << n
    out = np.empty(N, dtype=np.complex128)
    for k in range(N):
        out[int(format(k, f"0{n}b")[::-1], 2)] = np.exp(2j * np.pi * x * k / N) / math.sqrt(N)
    return out


def main():
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from qevedo_simulator_b200 import library

    def save(name, ops, n, initial, amplitudes, **extra):
        np.savez_compressed(os.path.join(HERE, name), num_qubits=n, initial=initial, amplitudes=amplitudes,
                            **ops_to_arrays(ops), **extra)

    def basis(n, x=0):
        v = np.zeros(1 << n, dtype=np.complex128)
        v[x] = 1
        return v

    # QFT of |41> on 6 qubits: analytic.
    ops = library.qft(6).ops()
    save("qft6_basis41.npz", ops, 6, basis(6, 41), qft_basis(6, 41))
    # GHZ(7): analytic.
    g = np.zeros(1 << 7, dtype=np.complex128)
    g[0] = g[-1] = 1 / math.sqrt(2)
    save("ghz7.npz", library.ghz(7).ops(), 7, basis(7), g)
    # 3x3 grid random circuit, depth 8, with the no-repeat rule: naive oracle,
    # plus 2000 uniforms and the reference sampler's outcomes.
    ops = library.random_grid_circuit(3, 3, 8, seed=11).ops()
    amps = oracle.naive_statevector(ops, 9)
    u = np.random.Generator(np.random.PCG64(12)).random(2000)
    samples = oracle.sample_from_amplitudes(amps, u, 64)
    save("grid3x3_d8.npz", ops, 9, basis(9), amps, uniforms=u, samples64=samples)
    # All-gate random circuit on 7 qubits (controls, swaps, CCX, CSWAP).
    ops = library.random_gate_circuit(7, 60, seed=3).ops()
    save("gates7.npz", ops, 7, basis(7), oracle.naive_statevector(ops, 7))
    # Hardware-efficient ansatz, 6 qubits x 4 layers, from a random start.
    ops = library.hea_circuit(6, 4, seed=5).ops()
    start = library.gaussian_state(6, seed=6)
    save("hea6_l4.npz", ops, 6, start, oracle.naive_statevector(ops, 6, start))


if __name__ == "__main__":
    main()
