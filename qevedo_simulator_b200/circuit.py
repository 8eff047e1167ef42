"""Circuits and the standard gate set, with Qiskit's conventions.

Host-side mirror of the reference's circuit IR: the gate enum and its matrices
(src/circuit.rs:14-202), the circuit builder (src/circuit.rs:440-735) and the
chainable Python methods of its binding (python/src/lib.rs:66-407). Lowering
a gate to a unitary op with separate controls follows simulator::gate_op
(src/simulator.rs:106-119).

Matrices are built with the `math` module (the C library's sin/cos/exp, as the
reference's `f64::sin_cos` and `C64::from_polar` use) and stored as numpy
complex128, row-major, index bit j = qubit j of the gate.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_R = 1.0 / math.sqrt(2.0)  # std::f64::consts::FRAC_1_SQRT_2


def _phase(angle: float) -> complex:
    """C64::from_polar(1, angle)."""
    return complex(math.cos(angle), math.sin(angle))


def _controlled(m: np.ndarray, controls: int, state: int) -> np.ndarray:
    """Matrix::controlled (src/matrix.rs:180-196): acts on [controls..., targets...]."""
    k = int(m.shape[0]).bit_length() - 1
    dim = 1 << (controls + k)
    out = np.eye(dim, dtype=np.complex128)
    mask = (1 << controls) - 1
    for r in range(dim):
        for c in range(dim):
            rc, cc = (r & mask) == state, (c & mask) == state
            if rc and cc:
                out[r, c] = m[r >> controls, c >> controls]
            elif rc or cc:
                out[r, c] = 0.0
    return out


# name -> (arity, number of parameters); src/circuit.rs:14-50 and the binding's
# method list python/src/lib.rs:81-110.
GATES = {
    "id": (1, 0), "h": (1, 0), "x": (1, 0), "y": (1, 0), "z": (1, 0), "s": (1, 0), "sdg": (1, 0),
    "t": (1, 0), "tdg": (1, 0), "sx": (1, 0), "sxdg": (1, 0), "rx": (1, 1), "ry": (1, 1), "rz": (1, 1),
    "p": (1, 1), "u": (1, 3), "cx": (2, 0), "cy": (2, 0), "cz": (2, 0), "ch": (2, 0), "cp": (2, 1),
    "crx": (2, 1), "cry": (2, 1), "crz": (2, 1), "swap": (2, 0), "rzz": (2, 1), "rxx": (2, 1),
    "ccx": (3, 0), "cswap": (3, 0),
}
# Aliases accepted by Circuit.gate (OpenQASM names).
_ALIASES = {"u1": "p", "u3": "u", "cu1": "cp", "cnot": "cx", "toffoli": "ccx", "fredkin": "cswap", "i": "id"}
# Diagonal gates (src/circuit.rs:103-111).
_DIAGONAL = {"id", "z", "s", "sdg", "t", "tdg", "rz", "p", "cz", "cp", "crz", "rzz"}
# Controlled forms: (leading controls, target gate) (src/circuit.rs:115-130).
_CONTROLLED = {"cx": (1, "x"), "cy": (1, "y"), "cz": (1, "z"), "ch": (1, "h"), "cp": (1, "p"),
               "crx": (1, "rx"), "cry": (1, "ry"), "crz": (1, "rz"), "ccx": (2, "x"), "cswap": (1, "swap")}


# Matrices of named gates by (name, parameters), bounded.
_MATRICES: dict = {}
_MATRICES_MAX = 65536


@dataclass(frozen=True)
class Gate:
    """A gate by name with its parameters, or an arbitrary unitary."""

    name: str
    params: tuple = ()
    unitary: np.ndarray | None = field(default=None, compare=False)

    @property
    def arity(self) -> int:
        if self.name == "unitary":
            return int(self.unitary.shape[0]).bit_length() - 1
        return GATES[self.name][0]

    def is_diagonal(self) -> bool:
        if self.name == "unitary":
            m = self.unitary
            return bool(np.all(m[~np.eye(m.shape[0], dtype=bool)] == 0))
        return self.name in _DIAGONAL

    def controlled_form(self):
        """(controls, target gate) for controlled gates, else None."""
        if self.name not in _CONTROLLED:
            return None
        controls, target = _CONTROLLED[self.name]
        return controls, Gate(target, self.params)

    def matrix(self) -> np.ndarray:
        """The gate's unitary (src/circuit.rs:133-202).

        Named gates share one read-only array per (name, parameters): a
        circuit repeats a handful of gates many times, and building each
        small array again dominates lowering a circuit to ops.
        """
        if self.name == "unitary":
            return np.array(self.unitary, dtype=np.complex128)
        return _named_matrix(self.name, self.params)

    def _build_matrix(self) -> np.ndarray:
        form = self.controlled_form()
        if form is not None:
            controls, target = form
            return _controlled(target.matrix(), controls, (1 << controls) - 1)
        n, p = self.name, self.params
        c = complex
        if n == "id":
            return np.eye(2, dtype=np.complex128)
        if n == "h":
            return np.array([[_R, _R], [_R, -_R]], dtype=np.complex128)
        if n == "x":
            return np.array([[0, 1], [1, 0]], dtype=np.complex128)
        if n == "y":
            return np.array([[0, c(0, -1)], [c(0, 1), 0]], dtype=np.complex128)
        if n == "z":
            return np.diag([1.0, -1.0]).astype(np.complex128)
        if n == "s":
            return np.diag([1.0, c(0, 1)]).astype(np.complex128)
        if n == "sdg":
            return np.diag([1.0, c(0, -1)]).astype(np.complex128)
        if n == "t":
            return np.diag([1.0, _phase(math.pi / 4)]).astype(np.complex128)
        if n == "tdg":
            return np.diag([1.0, _phase(-math.pi / 4)]).astype(np.complex128)
        if n == "sx":
            return np.array([[c(0.5, 0.5), c(0.5, -0.5)], [c(0.5, -0.5), c(0.5, 0.5)]])
        if n == "sxdg":
            return np.array([[c(0.5, -0.5), c(0.5, 0.5)], [c(0.5, 0.5), c(0.5, -0.5)]])
        if n == "rx":
            s, co = math.sin(p[0] / 2.0), math.cos(p[0] / 2.0)
            return np.array([[co, c(0, -s)], [c(0, -s), co]], dtype=np.complex128)
        if n == "ry":
            s, co = math.sin(p[0] / 2.0), math.cos(p[0] / 2.0)
            return np.array([[co, -s], [s, co]], dtype=np.complex128)
        if n == "rz":
            return np.diag([_phase(-p[0] / 2.0), _phase(p[0] / 2.0)])
        if n == "p":
            return np.diag([c(1, 0), _phase(p[0])])
        if n == "u":
            theta, phi, lam = p
            s, co = math.sin(theta / 2.0), math.cos(theta / 2.0)
            # -phase(lambda) * s: num-complex Neg then Mul by a real scalar.
            pl = _phase(lam)
            return np.array([[c(co, 0), c(-pl.real * s, -pl.imag * s)],
                             [_phase(phi) * s, _phase(phi + lam) * co]], dtype=np.complex128)
        if n == "swap":
            return np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)
        if n == "rzz":
            a, b = _phase(-p[0] / 2.0), _phase(p[0] / 2.0)
            return np.diag([a, b, b, a])
        if n == "rxx":
            s, co = math.sin(p[0] / 2.0), math.cos(p[0] / 2.0)
            cc, ms = c(co, 0), c(0, -s)
            return np.array([[cc, 0, 0, ms], [0, cc, ms, 0], [0, ms, cc, 0], [ms, 0, 0, cc]], dtype=np.complex128)
        raise ValueError(f"unknown gate `{n}`")


@dataclass
class Op:
    """A unitary on (logical) qubits with separate controls (src/fusion.rs:15-23)."""

    targets: list
    controls: list  # [(qubit, value)]
    matrix: np.ndarray

    def qubits(self):
        return list(self.targets) + [q for q, _ in self.controls]


def _named_matrix(name: str, params: tuple) -> np.ndarray:
    """Gate(name, params).matrix() through the shared read-only cache."""
    key = (name, params)
    try:
        hit = _MATRICES.get(key)
    except TypeError:  # unhashable parameters
        return Gate(name, params)._build_matrix()
    if hit is None:
        hit = Gate(name, params)._build_matrix()
        hit.flags.writeable = False
        if len(_MATRICES) >= _MATRICES_MAX:
            _MATRICES.clear()
        _MATRICES[key] = hit
    return hit


def packed_gate_ops(instructions):
    """The ops of the "gate" instructions, as gate_op lowers them, laid out
    for the C ABI in one pass (no Op objects in between)."""
    from ._abi import PackedOps

    ks, cs, qubits, values, mats = [], [], [], [], []
    for ins in instructions:
        if ins[0] != "gate":
            continue
        gate, qs = ins[1], ins[2]
        form = _CONTROLLED.get(gate.name)
        if form is not None:
            nc = form[0]
            ks.append(len(qs) - nc)
            cs.append(nc)
            qubits += qs[nc:]
            qubits += qs[:nc]
            values += [0] * (len(qs) - nc)
            values += [1] * nc
            mats.append(_named_matrix(form[1], gate.params))
        else:
            ks.append(len(qs))
            cs.append(0)
            qubits += qs
            values += [0] * len(qs)
            mats.append(gate.matrix() if gate.name == "unitary" else _named_matrix(gate.name, gate.params))
    return PackedOps(parts=(ks, cs, qubits, values, mats))


def gate_op(gate: Gate, qubits) -> Op:
    """simulator::gate_op (src/simulator.rs:106-119): controls stay separate so
    the kernel touches only the controlled part of the state."""
    form = _CONTROLLED.get(gate.name)
    if form is not None:
        controls, target = form
        return Op(list(qubits[controls:]), [(q, True) for q in qubits[:controls]],
                  _named_matrix(target, gate.params))
    if gate.name == "unitary":
        return Op(list(qubits), [], gate.matrix())
    return Op(list(qubits), [], _named_matrix(gate.name, gate.params))


class Circuit:
    """A quantum circuit of gates, measurements, resets, barriers and classical
    feedback on numbered qubits (qubit 0 is the least significant bit).

    Mirrors the binding's `Circuit` (python/src/lib.rs:18-407) for the
    state-vector path; noise channels and Stim/QASM I/O belong to other
    backends and are not part of this engine.
    """

    def __init__(self, num_qubits: int, num_clbits: int = 0):
        if num_qubits < 0 or num_clbits < 0:
            raise ValueError("sizes must be non-negative")
        self.num_qubits = int(num_qubits)
        self.num_clbits = int(num_clbits)
        # ("gate", Gate, qubits) | ("measure", qubit, clbit) | ("reset", qubit)
        # | ("barrier", qubits) | ("feedback", pauli, qubit, clbit)
        self._instructions: list = []

    # -- validation (python/src/lib.rs:29-56)
    def _check(self, qubits):
        for q in qubits:
            if not 0 <= q < self.num_qubits:
                raise ValueError(f"qubit {q} is out of range for {self.num_qubits} qubits")
        if len(set(qubits)) != len(qubits):
            raise ValueError("a gate cannot act on the same qubit twice")

    def _push(self, gate: Gate, qubits):
        qubits = [int(q) for q in qubits]
        self._check(qubits)
        if gate.arity != len(qubits):
            raise ValueError(f"the gate acts on {gate.arity} qubits, given {len(qubits)}")
        self._instructions.append(("gate", gate, qubits))
        return self

    def gate(self, name: str, qubits, params=()):
        """Apply a gate by name (`circuit.gate("cu1", [0, 1], [0.5])`)."""
        key = _ALIASES.get(name.lower(), name.lower())
        if key not in GATES:
            raise ValueError(f"unknown gate `{name}`")
        if len(params) != GATES[key][1]:
            raise ValueError(f"`{name}` takes {GATES[key][1]} parameters")
        return self._push(Gate(key, tuple(float(x) for x in params)), qubits)

    def unitary(self, matrix, qubits):
        """An arbitrary unitary; bit j of the matrix index is qubits[j]."""
        m = np.asarray(matrix, dtype=np.complex128)
        dim = 1 << len(qubits)
        if m.shape != (dim, dim):
            raise ValueError(f"a gate on {len(qubits)} qubits needs a {dim}x{dim} matrix")
        if np.max(np.abs(m @ m.conj().T - np.eye(dim))) > 1e-8:
            raise ValueError("the matrix is not unitary")
        return self._push(Gate("unitary", (), m.copy()), qubits)

    def measure(self, qubit: int, clbit: int):
        self._check([qubit])
        self.num_clbits = max(self.num_clbits, clbit + 1)
        self._instructions.append(("measure", int(qubit), int(clbit)))
        return self

    def measure_all(self):
        for q in range(self.num_qubits):
            self.measure(q, q)
        return self

    def reset(self, qubit: int):
        self._check([qubit])
        self._instructions.append(("reset", int(qubit)))
        return self

    def barrier(self):
        self._instructions.append(("barrier", list(range(self.num_qubits))))
        return self

    def feedback(self, pauli: str, qubit: int, clbit: int):
        """`pauli` (X, Y or Z) on `qubit` if classical bit `clbit` reads 1."""
        letter = pauli.upper()
        if letter not in ("X", "Y", "Z"):
            raise ValueError(f"pauli must be X, Y or Z, not {pauli!r}")
        self._check([qubit])
        self.num_clbits = max(self.num_clbits, clbit + 1)
        self._instructions.append(("feedback", letter, int(qubit), int(clbit)))
        return self

    @property
    def gate_count(self) -> int:
        return sum(1 for i in self._instructions if i[0] == "gate")

    def instructions(self):
        """(name, qubits, params) per instruction, as the binding reports them."""
        out = []
        for ins in self._instructions:
            if ins[0] == "gate":
                g = ins[1]
                out.append((g.name, list(ins[2]), list(g.params)))
            elif ins[0] == "measure":
                out.append(("measure", [ins[1]], [float(ins[2])]))
            elif ins[0] == "reset":
                out.append(("reset", [ins[1]], []))
            elif ins[0] == "barrier":
                out.append(("barrier", list(ins[1]), []))
            else:
                out.append((f"feedback_{ins[1].lower()}", [ins[2]], [float(ins[3])]))
        return out

    def ops(self):
        """The unitary ops of a circuit without measurements (gate_op per gate)."""
        ops = []
        for ins in self._instructions:
            if ins[0] == "gate":
                ops.append(gate_op(ins[1], ins[2]))
            elif ins[0] != "barrier":
                raise ValueError(f"statevector() needs a unitary circuit, found {ins[0]}")
        return ops

    def copy(self) -> "Circuit":
        c = Circuit(self.num_qubits, self.num_clbits)
        c._instructions = list(self._instructions)
        return c

    def __len__(self):
        return len(self._instructions)

    def __repr__(self):
        return f"Circuit({self.num_qubits} qubits, {self.num_clbits} classical bits, {self.gate_count} gates)"


def _make_method(name: str, arity: int, nparams: int):
    def method(self, *args):
        if len(args) != arity + nparams:
            raise TypeError(f"{name}() takes {nparams} parameter(s) then {arity} qubit(s)")
        params, qubits = args[:nparams], args[nparams:]
        return self._push(Gate(name, tuple(float(p) for p in params)), qubits)

    method.__name__ = name
    method.__doc__ = f"Apply `{name}` ({nparams} parameter(s) first, then {arity} qubit(s))."
    return method


for _name, (_arity, _np) in GATES.items():
    setattr(Circuit, _name, _make_method(_name, _arity, _np))
