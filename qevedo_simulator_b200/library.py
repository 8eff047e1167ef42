"""Benchmark and test circuits (host side).

Restates the reference's circuit library (src/library.rs:9-141) for the
state-vector workloads: GHZ, QFT without final swaps, the line-brick random
circuit, the grid random circuit, and the random all-gate test circuit; plus
the workload generators this engine is measured on (the grid random circuit
with the no-repeat rule, the Gaussian start state, hardware-efficient ansatz
circuits, and the mixed circuits the cost model trains on).

Random draws come from numpy's PCG64 generator seeded with the given seed.
The reference draws from rand_pcg's Pcg64 through rand's `random_range`,
whose streams are not reproduced here, so a given seed yields a different
(but equally distributed) circuit than the reference's.
"""

from __future__ import annotations

import math

import numpy as np

from .circuit import Circuit, Gate, Op

HALF_PI = math.pi / 2.0


def _sqrt_gate(circuit: Circuit, which: int, q: int):
    """sqrt(X), sqrt(Y), sqrt(W) as the reference builds them (src/library.rs:41-49)."""
    if which == 0:
        circuit.rx(HALF_PI, q)
    elif which == 1:
        circuit.ry(HALF_PI, q)
    else:  # sqrt(W), W = (X + Y)/sqrt(2)
        circuit.u(HALF_PI, -math.pi / 4, math.pi / 4, q)


def ghz(n: int) -> Circuit:
    """H on qubit 0 then a CX chain (src/library.rs:9-16)."""
    c = Circuit(n)
    c.h(0)
    for q in range(1, n):
        c.cx(q - 1, q)
    return c


def qft(n: int) -> Circuit:
    """Quantum Fourier transform without the final qubit reversal
    (src/library.rs:19-29)."""
    c = Circuit(n)
    for target in reversed(range(n)):
        c.h(target)
        for control in reversed(range(target)):
            c.cp(math.pi / float(1 << (target - control)), control, target)
    return c


def random_circuit(n: int, depth: int, seed: int) -> Circuit:
    """Google-style random circuit on a line (src/library.rs:35-60)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = Circuit(n)
    for layer in range(depth):
        for q in range(n):
            _sqrt_gate(c, int(rng.integers(0, 3)), q)
        q = layer % 2
        while q + 1 < n:
            c.cz(q, q + 1)
            q += 2
    return c


def random_grid_circuit(rows: int, cols: int, depth: int, seed: int, no_repeat: bool = True) -> Circuit:
    """Google-style random circuit on a rows x cols grid (qubit r*cols + c).

    Each layer applies sqrt(X), sqrt(Y) or sqrt(W) to every qubit, then CZ on
    one of four coupler sets in turn (src/library.rs:67-99). With `no_repeat`
    (the benchmark's rule) a qubit's gate is drawn uniformly from the two
    gates that differ from its previous one; the first layer draws from all
    three. Without it every draw is uniform over the three, as in the
    reference.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    n = rows * cols
    c = Circuit(n)
    previous = [-1] * n
    for layer in range(depth):
        for q in range(n):
            if no_repeat and previous[q] >= 0:
                pick = int(rng.integers(0, 2))
                choice = [g for g in range(3) if g != previous[q]][pick]
            else:
                choice = int(rng.integers(0, 3))
            previous[q] = choice
            _sqrt_gate(c, choice, q)
        offset = (layer // 2) % 2
        for r in range(rows):
            for col in range(cols):
                q = r * cols + col
                if layer % 2 == 0 and col % 2 == offset and col + 1 < cols:
                    c.cz(q, q + 1)
                if layer % 2 == 1 and r % 2 == offset and r + 1 < rows:
                    c.cz(q, q + cols)
    return c


def grid_shape(n: int) -> tuple:
    """The most square rows x cols grid with rows*cols = n and rows <= cols
    (4x5 for 20, 5x6 for 30, 4x8 for 32, 4x7 for 28)."""
    best = (1, n)
    for rows in range(1, int(math.isqrt(n)) + 1):
        if n % rows == 0:
            best = (rows, n // rows)
    if n == 32:
        return (4, 8)
    return best


def random_gate_circuit(n: int, gates: int, seed: int) -> Circuit:
    """Random circuit over the standard gate set for correctness tests
    (src/library.rs:103-141)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = Circuit(n)
    for _ in range(gates):
        qubits = list(range(n))
        for i in range(min(n, 3)):
            j = int(rng.integers(i, n))
            qubits[i], qubits[j] = qubits[j], qubits[i]
        angle = float(rng.random()) * math.tau
        choice = int(rng.integers(0, 14 if n >= 3 else (12 if n == 2 else 8)))
        q = qubits
        if choice == 0:
            c.h(q[0])
        elif choice == 1:
            c.x(q[0])
        elif choice == 2:
            c.rx(angle, q[0])
        elif choice == 3:
            c.ry(angle, q[0])
        elif choice == 4:
            c.rz(angle, q[0])
        elif choice == 5:
            c.u(angle, angle * 0.5, angle * 0.25, q[0])
        elif choice == 6:
            c.t(q[0])
        elif choice == 7:
            c.sx(q[0])
        elif choice == 8:
            c.cx(q[0], q[1])
        elif choice == 9:
            c.cz(q[0], q[1])
        elif choice == 10:
            c.cp(angle, q[0], q[1])
        elif choice == 11:
            c.swap(q[0], q[1])
        elif choice == 12:
            c.ccx(q[0], q[1], q[2])
        else:
            c.cswap(q[0], q[1], q[2])
    return c


def gaussian_state(n: int, seed: int) -> np.ndarray:
    """A normalised vector of i.i.d. complex Gaussian amplitudes (complex128),
    drawn in float64 from PCG64(seed) by Box-Muller (numpy's standard_normal)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    v = np.empty(1 << n, dtype=np.complex128)
    view = v.view(np.float64)
    step = 1 << 24
    for start in range(0, view.size, step):
        view[start:start + step] = rng.standard_normal(min(step, view.size - start))
    v /= math.sqrt(float(np.vdot(v, v).real))
    return v


def hea_circuit(width: int, layers: int, seed: int) -> Circuit:
    """Hardware-efficient ansatz: per layer RY(theta) RZ(phi) on every qubit
    with angles uniform in [0, 2 pi), then a CNOT ladder cx(q, q+1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = Circuit(width)
    for _ in range(layers):
        angles = rng.random(2 * width) * math.tau
        for q in range(width):
            c.ry(float(angles[2 * q]), q)
            c.rz(float(angles[2 * q + 1]), q)
        for q in range(width - 1):
            c.cx(q, q + 1)
    return c


def hea_layers(width: int, layers: int, seed: int) -> np.ndarray:
    """The per-qubit gates of hea_circuit(width, layers, seed) as an array of
    shape (layers, width, 2, 2): RZ(phi) @ RY(theta) (RY applied first), from
    the same angle draws."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty((layers, width, 2, 2), dtype=np.complex128)
    for layer in range(layers):
        angles = rng.random(2 * width) * math.tau
        for q in range(width):
            rz = Gate("rz", (float(angles[2 * q + 1]),)).matrix()
            out[layer, q] = rz @ Gate("ry", (float(angles[2 * q]),)).matrix()
    return out


def hea_batch(count: int, seed: int, widths=(10, 22), layers=(4, 12)) -> list:
    """`count` hardware-efficient ansatz specs (width, layers, seed) with width
    and layer count uniform in the given inclusive ranges; hea_circuit and
    hea_layers rebuild each one from its spec."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.integers(widths[0], widths[1] + 1, size=count)
    l = rng.integers(layers[0], layers[1] + 1, size=count)
    s = rng.integers(0, 2**62, size=count)
    return [(int(a), int(b), int(c)) for a, b, c in zip(w, l, s)]


def haar_su2(rng: np.random.Generator) -> np.ndarray:
    """A Haar-random 2x2 special unitary."""
    z = rng.standard_normal(4)
    z /= np.linalg.norm(z)
    a, b = complex(z[0], z[1]), complex(z[2], z[3])
    return np.array([[a, -b.conjugate()], [b, a.conjugate()]], dtype=np.complex128)


ISWAP = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)


def mixed_ops(n: int, depth: int, seed: int, p_distance: float = 0.3) -> list:
    """Cost-model training circuits as ops: per layer, a Haar-random SU(2) on
    every qubit; then pair gates (CZ, CX or iSWAP, uniformly) on disjoint
    pairs at geometric qubit distance (success probability `p_distance`); a
    diagonal phase gate; and an X with 1 to 3 controls (an op with separate
    controls, as the reference's Op allows, src/fusion.rs:17-23)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ops = []
    x = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    z = np.diag([1, -1]).astype(np.complex128)
    for _ in range(depth):
        for q in range(n):
            ops.append(Op([q], [], haar_su2(rng)))
        free = [int(v) for v in rng.permutation(n)]
        while len(free) >= 2:
            a = free.pop()
            b = (a + int(rng.geometric(p_distance))) % n
            if b not in free:
                continue
            free.remove(b)
            kind = int(rng.integers(0, 3))
            if kind == 0:
                ops.append(Op([b], [(a, True)], z))
            elif kind == 1:
                ops.append(Op([b], [(a, True)], x))
            else:
                ops.append(Op([a, b], [], ISWAP))
        q = int(rng.integers(0, n))
        phase = float(rng.random()) * math.tau
        ops.append(Op([q], [], np.diag([1, complex(math.cos(phase), math.sin(phase))])))
        controls = int(rng.integers(1, 4))
        picks = [int(v) for v in rng.choice(n, size=controls + 1, replace=False)]
        ops.append(Op([picks[-1]], [(c, True) for c in picks[:-1]], x))
    return ops
