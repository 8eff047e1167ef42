"""`run` and `statevector` on the B200 state-vector engine.

Mirrors the state-vector side of the reference's Python API
(python/python/qevedo/simulator/__init__.py:96-158, native
python/src/lib.rs:645-718) and of `run_on` (src/simulator.rs:329-427):
circuits whose measurements all come at the end are simulated once and
sampled in two passes; mid-circuit measurements, resets and classical
feedback run shot by shot with the state resident on the device.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .circuit import Circuit, Gate, gate_op, packed_gate_ops

BACKENDS = ("auto", "statevector", "state_vector")


@dataclass
class RunResult:
    """Counts per classical bitstring (classical bit 0 on the right, Qiskit's
    convention) and run statistics (src/simulator.rs:70-101), with the
    binding's fields (python/src/lib.rs:409-477): `fidelity`,
    `max_bond_dimension` and `peak_active_qubits` belong to the MPS and
    near-Clifford backends and are None here."""

    counts: dict
    backend: str = "statevector"
    gates: int = 0
    kernels: int = 0
    passes: int = 0
    gate_seconds: float = 0.0
    measure_seconds: float = 0.0
    stats: dict = field(default_factory=dict)
    fidelity: float | None = None
    max_bond_dimension: int | None = None
    peak_active_qubits: int | None = None

    def __repr__(self) -> str:
        return f'RunResult(backend="{self.backend}", {len(self.counts)} outcomes)'


def _precision_bits(precision: str) -> int:
    if precision == "single":
        return 32
    if precision == "double":
        return 64
    raise ValueError('precision must be "single" or "double"')


def _check_backend(backend: str):
    if backend not in BACKENDS:
        if backend in ("stabilizer", "mps", "near_clifford"):
            raise ValueError(f"backend `{backend}` is not part of the B200 state-vector engine")
        raise ValueError(f"unknown backend `{backend}`")


def uniforms(rng: np.random.Generator, count: int) -> np.ndarray:
    """`count` uniforms in [0, 1) (53-bit, as rand's `random::<f64>()`)."""
    return rng.random(count)


def terminal_split(circuit: Circuit):
    """Index of the first instruction after which only measurements and
    barriers follow, if everything before is unitary (src/simulator.rs:170-182)."""
    ins = circuit._instructions
    split = len(ins)
    for i in range(len(ins) - 1, -1, -1):
        if ins[i][0] in ("measure", "barrier"):
            split = i
        else:
            break
    if all(x[0] in ("gate", "barrier") for x in ins[:split]):
        return split
    return None


def bitstring(bits) -> str:
    return "".join("1" if b else "0" for b in reversed(bits))


def key_bitstring(key: int, num_clbits: int) -> str:
    """bitstring() of the classical bits packed in `key` (bit c = clbit c)."""
    return format(key, "b").zfill(num_clbits) if num_clbits else ""


def count_outcomes(outcomes: np.ndarray, measures, num_clbits: int) -> dict:
    """Counts from sampled basis states (src/simulator.rs:187-230): each shot
    becomes an integer key (bit c = classical bit c), keys are counted, and
    only distinct keys are formatted."""
    if num_clbits <= 64:
        keys = np.zeros(outcomes.size, dtype=np.uint64)
        for q, c in measures:
            keys |= ((outcomes >> np.uint64(q)) & np.uint64(1)) << np.uint64(c)
        uniq, cnt = np.unique(keys, return_counts=True)
        out = {}
        for k, n in zip(uniq.tolist(), cnt.tolist()):
            out[key_bitstring(k, num_clbits)] = n
        return dict(sorted(out.items()))
    out = {}
    for index in outcomes.tolist():
        bits = [False] * num_clbits
        for q, c in measures:
            bits[c] = bool((index >> q) & 1)
        key = bitstring(bits)
        out[key] = out.get(key, 0) + 1
    return dict(sorted(out.items()))


def _as_circuit(circuit) -> Circuit:
    """A Circuit, or OpenQASM 2/3 text parsed into one (the reference's
    `run` and `statevector` take either; anything else is a TypeError, as
    the reference's binding raises)."""
    if isinstance(circuit, str):
        from . import qasm

        return qasm.parse(circuit)
    if not isinstance(circuit, Circuit):
        raise TypeError(f"expected a Circuit or OpenQASM text, not {type(circuit).__name__}")
    return circuit


_THREAD_PLACEMENTS = ("pcores", "pthreads", "cores", "allcores", "all")


def _check_threads(threads):
    """The reference's thread setting (python/src/lib.rs:574-594): None, a
    thread count (0 meaning 1), or a placement name; anything else is a
    ValueError with the reference's message. Host planning here uses the
    library's own thread pool, so a valid value changes nothing."""
    if threads is None:
        return
    if isinstance(threads, int) and not isinstance(threads, bool) and threads >= 0:
        return
    if not isinstance(threads, str):
        raise ValueError("threads must be a number or a placement name")
    if threads not in _THREAD_PLACEMENTS:
        raise ValueError(f"unknown thread placement `{threads}` (pcores, pthreads, cores, all)")


def plan_options(max_fused_qubits: int | None = None, staged: bool | None = None, tile_qubits: int = 0,
                 math: str | None = None, planner: str | None = None) -> _native.QvdgOptions:
    """Planner settings for a run. With none of max_fused_qubits, staged and
    math given, the learned planner picks among its candidate plans by the
    committed cost model's predicted time (complex64 states; the reference's
    defaults, fusion 4 with staged tiles, are its fallback and run for
    complex128). Giving any of them plans greedily with those settings, as
    the reference's Options do (src/simulator.rs:37-66)."""
    if planner is None:
        planner = "learned" if max_fused_qubits is None and staged is None and math is None else "greedy"
    if planner not in _native.PLANNERS:
        raise ValueError('planner must be "learned" or "greedy"')
    return _native.options(4 if max_fused_qubits is None else max_fused_qubits, True if staged is None else staged,
                           tile_qubits, planner=planner, math="fp32" if math is None else math)


def _with_model(opts: _native.QvdgOptions) -> _native.QvdgOptions:
    """Registers the committed cost model on the current device when the
    learned planner will run (a device call, so not in plan_options)."""
    if opts.planner == _native.PLANNERS["learned"]:
        _native.ensure_cost_model()
    return opts


def statevector(circuit: Circuit | str, *, precision: str = "double", max_fused_qubits: int | None = None,
                staged: bool | None = None, tile_qubits: int = 0, math: str | None = None,
                planner: str | None = None, threads: int | str | None = None) -> np.ndarray:
    """The final state of a circuit without measurements, as complex128 in
    logical order (index bit q = qubit q). Double precision by default, as
    the reference's `statevector` (python/src/lib.rs:686-718). Planner
    settings as in `plan_options`. `threads` is checked as the reference
    does; host planning uses the library's own thread pool."""
    _check_threads(threads)
    circuit = _as_circuit(circuit)
    ops = circuit.ops()
    opts = plan_options(max_fused_qubits, staged, tile_qubits, math, planner)
    with _native.DeviceState(circuit.num_qubits, _precision_bits(precision)) as st:
        st.apply_ops(ops, _with_model(opts))
        return st.amplitudes()


def run(circuit: Circuit | str, shots: int = 1024, *, backend: str = "auto", seed: int | None = None,
        precision: str = "single", max_bond_dimension: int = 256, truncation_threshold: float = 1e-16,
        threads: int | str | None = None, max_fused_qubits: int | None = None, staged: bool | None = None,
        tile_qubits: int = 0, math: str | None = None, planner: str | None = None,
        state: _native.DeviceState | None = None) -> RunResult:
    """Sample `shots` shots of `circuit` (a Circuit or OpenQASM 2/3 text) on
    the device state vector.

    `seed` seeds the uniforms (numpy PCG64; the reference seeds rand_pcg's
    Pcg64, whose streams this engine does not reproduce). Given the same
    uniforms, every outcome is bit-identical to the reference sampler's. A
    caller may pass a reusable `state` of the right size and precision.
    `max_bond_dimension` and `truncation_threshold` (the reference's MPS
    settings) and `threads` are accepted for the reference's signature
    (python/python/qevedo/simulator/__init__.py:96-106) and do not affect
    the state vector; host planning uses the library's own thread pool.
    Planner settings as in `plan_options`: by default the learned planner
    picks the plan; `result.stats["settings"]` says which.
    """
    _check_backend(backend)
    _check_threads(threads)
    circuit = _as_circuit(circuit)
    bits = _precision_bits(precision)
    rng = np.random.Generator(np.random.PCG64(seed))
    opts = plan_options(max_fused_qubits, staged, tile_qubits, math, planner)
    own = state is None
    st = state or _native.DeviceState(circuit.num_qubits, bits)
    _with_model(opts)
    try:
        if not own:
            st.zero()
        split = terminal_split(circuit)
        result = RunResult(counts={})
        if split is not None:
            stats = st.apply_packed(packed_gate_ops(circuit._instructions[:split]), opts)
            result.gates, result.kernels, result.passes = stats["gates"], stats["kernels"], stats["passes"]
            result.gate_seconds = stats["gate_seconds"]
            result.stats = stats
            t0 = time.perf_counter()
            measures = [(i[1], i[2]) for i in circuit._instructions[split:] if i[0] == "measure"]
            if circuit.num_clbits <= 64:
                # Keys built, sorted and counted on the device; only the
                # distinct keys come back to be formatted.
                keys, cnt = st.sample_counts(uniforms(rng, shots), measures)
                result.counts = {key_bitstring(k, circuit.num_clbits): n
                                 for k, n in zip(keys.tolist(), cnt.tolist())}
                result.counts = dict(sorted(result.counts.items()))
            else:
                outcomes = st.sample_unordered(uniforms(rng, shots))
                result.counts = count_outcomes(outcomes, measures, circuit.num_clbits)
            result.measure_seconds = time.perf_counter() - t0
            return result
        counts = {}
        for _ in range(shots):
            st.zero()
            clbits = [False] * circuit.num_clbits
            pending = []
            for ins in circuit._instructions:
                kind = ins[0]
                if kind == "gate":
                    pending.append(gate_op(ins[1], ins[2]))
                elif kind == "measure":
                    s = st.apply_ops(pending, opts)
                    result.gates += s["gates"]
                    result.gate_seconds += s["gate_seconds"]
                    pending = []
                    t0 = time.perf_counter()
                    clbits[ins[2]] = bool(st.measure(ins[1], float(rng.random())))
                    result.measure_seconds += time.perf_counter() - t0
                elif kind == "reset":
                    s = st.apply_ops(pending, opts)
                    result.gates += s["gates"]
                    pending = []
                    st.reset(ins[1], float(rng.random()))
                elif kind == "feedback":
                    if clbits[ins[3]]:
                        pending.append(gate_op(Gate(ins[1].lower()), [ins[2]]))
            s = st.apply_ops(pending, opts)
            result.gates += s["gates"]
            key = bitstring(clbits)
            counts[key] = counts.get(key, 0) + 1
        result.counts = dict(sorted(counts.items()))
        return result
    finally:
        if own:
            st.close()


def estimate(circuit: Circuit, observable, *, precision: str = "double") -> float:
    """<psi|O|psi> of the circuit's final state for O = sum of coeff * Pauli
    string, given as {label: coeff} or [(label, coeff), ...] with Qiskit
    labels (rightmost letter = qubit 0); each term is one device reduction.
    The reference's Qiskit Estimator computes the same from its state vector
    (python/python/qevedo/simulator/qiskit.py:584-590)."""
    terms = observable.items() if isinstance(observable, dict) else observable
    ops = circuit.ops()
    with _native.DeviceState(circuit.num_qubits, _precision_bits(precision)) as st:
        st.apply_ops(ops, _native.options(4, staged=False))
        total = 0.0
        for label, coeff in terms:
            if len(label) != circuit.num_qubits:
                raise ValueError(f"label `{label}` does not have {circuit.num_qubits} letters")
            total += float(np.real(coeff)) * st.expect_pauli(label)
        return total
