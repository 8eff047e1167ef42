"""The OpenQASM reader (qevedo_simulator_b200.qasm) against circuits built
directly, after the reference's tests/qasm.rs: built-in gates, OpenQASM 3
against 2, definitions and expressions, modifiers, broadcasting, feedback
and error positions. States come from the naive oracle (no device)."""

import math

import numpy as np
import pytest

from conftest import max_distance, random_unitary
from qevedo_simulator_b200 import Circuit, Gate
from qevedo_simulator_b200.qasm import QasmError, parse


def state(oracle, circuit, n=None):
    ops = [op for op in circuit.ops()]
    return oracle.naive_statevector(ops, n or circuit.num_qubits)


def with_prefix(prefix: Circuit, body: Circuit) -> Circuit:
    c = prefix.copy()
    c._instructions.extend(body._instructions)
    return c


GATE_CASES = [
    ("id", Gate("id"), 1), ("h", Gate("h"), 1), ("x", Gate("x"), 1), ("y", Gate("y"), 1), ("z", Gate("z"), 1),
    ("s", Gate("s"), 1), ("sdg", Gate("sdg"), 1), ("t", Gate("t"), 1), ("tdg", Gate("tdg"), 1),
    ("sx", Gate("sx"), 1), ("sxdg", Gate("sxdg"), 1), ("rx(0.3)", Gate("rx", (0.3,)), 1),
    ("ry(-1.2)", Gate("ry", (-1.2,)), 1), ("rz(pi/3)", Gate("rz", (math.pi / 3,)), 1),
    ("p(0.7)", Gate("p", (0.7,)), 1), ("u1(0.7)", Gate("p", (0.7,)), 1),
    ("u2(0.1, 0.2)", Gate("u", (math.pi / 2, 0.1, 0.2)), 1), ("u3(0.1, 0.2, 0.3)", Gate("u", (0.1, 0.2, 0.3)), 1),
    ("U(0.1, 0.2, 0.3)", Gate("u", (0.1, 0.2, 0.3)), 1), ("cx", Gate("cx"), 2), ("CX", Gate("cx"), 2),
    ("cy", Gate("cy"), 2), ("cz", Gate("cz"), 2), ("ch", Gate("ch"), 2), ("cp(0.4)", Gate("cp", (0.4,)), 2),
    ("cu1(0.4)", Gate("cp", (0.4,)), 2), ("crx(0.5)", Gate("crx", (0.5,)), 2), ("cry(0.5)", Gate("cry", (0.5,)), 2),
    ("crz(0.5)", Gate("crz", (0.5,)), 2), ("swap", Gate("swap"), 2), ("rzz(0.6)", Gate("rzz", (0.6,)), 2),
    ("rxx(0.6)", Gate("rxx", (0.6,)), 2), ("ccx", Gate("ccx"), 3), ("cswap", Gate("cswap"), 3),
]


def test_builtin_gates_match_the_builder(oracle):
    rng = np.random.Generator(np.random.PCG64(1))
    for call, gate, arity in GATE_CASES:
        prefix = Circuit(4).unitary(random_unitary(rng, 4), [0, 1, 2, 3])
        qubits = [int(q) for q in rng.permutation(4)[:arity]]
        direct = prefix.copy()
        direct._instructions.append(("gate", gate, qubits))
        program = 'OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[4];\n' + call + " " + ", ".join(
            f"q[{q}]" for q in qubits) + ";"
        parsed = with_prefix(prefix, parse(program))
        assert max_distance(state(oracle, direct), state(oracle, parsed)) < 1e-12, call


def test_unitary_only_gates(oracle):
    from qevedo_simulator_b200.circuit import _controlled

    sx = Gate("sx").matrix()
    cases = [("csx", _controlled(sx, 1, 1), 2), ("cu3(0.1, 0.2, 0.3)", _controlled(Gate("u", (0.1, 0.2, 0.3)).matrix(),
             1, 1), 2), ("c3x", _controlled(Gate("x").matrix(), 3, 7), 4)]
    rng = np.random.Generator(np.random.PCG64(2))
    for call, m, arity in cases:
        prefix = Circuit(4).unitary(random_unitary(rng, 4), [0, 1, 2, 3])
        qubits = [int(q) for q in rng.permutation(4)[:arity]]
        direct = prefix.copy().unitary(m, qubits)
        program = 'OPENQASM 2.0;\nqreg q[4];\n' + call + " " + ", ".join(f"q[{q}]" for q in qubits) + ";"
        assert max_distance(state(oracle, direct), state(oracle, with_prefix(prefix, parse(program)))) < 1e-12


def test_openqasm_3_matches_openqasm_2(oracle):
    v2 = """OPENQASM 2.0; include "qelib1.inc"; qreg a[2]; qreg b[1]; creg c[3];
        h a[0]; cx a[0], a[1]; u3(0.1, 0.2, 0.3) b[0]; cu1(pi/4) a[1], b[0];
        measure a -> c[0:1]; measure b[0] -> c[2];"""
    v3 = """OPENQASM 3.0; include "stdgates.inc"; qubit[2] a; qubit b; bit[3] c;
        h a[0]; cx a[0], a[1]; U(0.1, 0.2, 0.3) b; cp(π/4) a[1], b;
        c[0:1] = measure a; c[2] = measure b;"""
    c2, c3 = parse(v2), parse(v3)
    assert (c2.num_qubits, c2.num_clbits) == (3, 3)
    assert len(c2._instructions) == len(c3._instructions)
    gates = lambda c: Circuit(c.num_qubits)._instructions.extend([i for i in c._instructions if i[0] == "gate"])
    u2, u3 = Circuit(3), Circuit(3)
    u2._instructions = [i for i in c2._instructions if i[0] == "gate"]
    u3._instructions = [i for i in c3._instructions if i[0] == "gate"]
    assert max_distance(state(oracle, u2), state(oracle, u3)) < 1e-12
    assert [i for i in c2._instructions if i[0] == "measure"] == [("measure", 0, 0), ("measure", 1, 1),
                                                                   ("measure", 2, 2)]
    del gates


def test_gate_definitions_and_expressions(oracle):
    program = """OPENQASM 2.0; include "qelib1.inc";
        gate rot(theta, phi) q { rz(phi) q; ry(theta / 2 + 0.1) q; }
        gate pair(a) x, y { rot(a, -a * 2) x; cx x, y; rot(sin(a)^2, cos(a)) y; }
        qreg q[2];
        pair(0.4) q[0], q[1];
        pair(-1.0e-1) q[1], q[0];"""
    direct = Circuit(2)
    for a, x, y in [(0.4, 0, 1), (-0.1, 1, 0)]:
        direct.rz(-a * 2.0, x).ry(a / 2.0 + 0.1, x).cx(x, y)
        direct.rz(math.cos(a), y).ry(math.sin(a) ** 2 / 2.0 + 0.1, y)
    assert max_distance(state(oracle, direct), state(oracle, parse(program))) < 1e-12


def test_modifiers(oracle):
    pairs = [("ctrl @ x q[0], q[1];", "cx q[0], q[1];"), ("inv @ s q[1];", "sdg q[1];"),
             ("pow(2) @ s q[0];", "z q[0];"), ("pow(-1) @ t q[0];", "tdg q[0];"),
             ("ctrl(2) @ x q[0], q[1], q[2];", "ccx q[0], q[1], q[2];"),
             ("negctrl @ x q[2], q[0];", "x q[2]; cx q[2], q[0]; x q[2];"),
             ("ctrl @ inv @ rz(0.3) q[1], q[2];", "crz(-0.3) q[1], q[2];"),
             ("ctrl @ swap q[0], q[1], q[2];", "cswap q[0], q[1], q[2];")]
    rng = np.random.Generator(np.random.PCG64(3))
    head = 'OPENQASM 3.0;\ninclude "stdgates.inc";\nqubit[3] q;\n'
    for a, b in pairs:
        prefix = Circuit(3).unitary(random_unitary(rng, 3), [0, 1, 2])
        sa = state(oracle, with_prefix(prefix, parse(head + a)))
        sb = state(oracle, with_prefix(prefix, parse(head + b)))
        assert max_distance(sa, sb) < 1e-12, a
    defined = parse(head.replace("qubit[3] q;\n", "") + "gate g(a) x, y { rx(a) x; cz x, y; }\nqubit[3] q;\n"
                    "ctrl @ inv @ g(0.7) q[2], q[0], q[1];")
    (kind, gate, qubits), = defined._instructions
    assert kind == "gate" and gate.name == "unitary" and qubits == [2, 0, 1]
    inner = Circuit(2).rx(0.7, 0).cz(0, 1)
    g = np.zeros((4, 4), dtype=complex)
    for col in range(4):
        v = np.zeros(4, dtype=complex)
        v[col] = 1
        g[:, col] = oracle.naive_apply_ops(v, inner.ops())
    from qevedo_simulator_b200.circuit import _controlled
    assert np.abs(gate.unitary - _controlled(g.conj().T, 1, 1)).max() < 1e-12


def test_broadcasting_ranges_resets_and_barriers():
    c = parse("OPENQASM 3;\nqubit[4] q;\nbit[4] c;\nh q;\ncx q[0:1], q[2:3];\nbarrier;\nreset q[0:2:2];\n"
              "c = measure q;")

    def show(i):
        if i[0] == "gate":
            return f"{i[1].name}{i[2]}"
        if i[0] == "measure":
            return f"m{i[1]}{i[2]}"
        if i[0] == "reset":
            return f"r{i[1]}"
        return f"b{i[1]}"

    assert [show(i) for i in c._instructions] == ["h[0]", "h[1]", "h[2]", "h[3]", "cx[0, 2]", "cx[1, 3]",
                                                   "b[0, 1, 2, 3]", "r0", "r2", "m00", "m11", "m22", "m33"]


def test_pauli_ifs_become_feedback():
    c = parse("OPENQASM 3.0;\nqubit[2] q;\nbit[1] c;\nc[0] = measure q[0];\nif (c[0]) x q[1];\n"
              "if (!c[0]) { z q[0]; x q[1]; }\nif (c[0] == 1) y q[0]; else z q[0];")
    fb = [i for i in c._instructions[1:]]
    assert fb[0] == ("feedback", "X", 1, 0)
    # `if (!c[0]) {z q0; x q1}`: applied unconditionally, undone when c = 1.
    assert fb[1][0] == "gate" and fb[1][1].name == "z" and fb[1][2] == [0]
    assert fb[2][0] == "gate" and fb[2][1].name == "x" and fb[2][2] == [1]
    assert ("feedback", "Z", 0, 0) in fb and ("feedback", "X", 1, 0) in fb[3:]
    # if/else: z unconditionally, then the product y*z ~ x when the bit is 1.
    assert fb[-2][1].name == "z" and fb[-1] == ("feedback", "X", 0, 0)


ERRORS = [
    ("OPENQASM 2.0;\nqreg q[2];\nfoo q[0];", 3, "unknown gate `foo`"),
    ("OPENQASM 2.0;\nqreg q[2];\nh q[5];", 3, "out of range"),
    ("OPENQASM 2.0;\nqreg q[2];\ncx q[0];", 3, "acts on 2 qubits"),
    ("OPENQASM 2.0;\nqreg q[2];\nrx q[0];", 3, "takes 1 parameters"),
    ("OPENQASM 2.0;\nqreg q[2];\ncreg c[2];\nif (c == 1) x q[0];", 4, "a register of 2 bits, is not supported"),
    ("OPENQASM 3.0;\nqubit[2] q;\nbit[1] c;\nif (c[0]) h q[0];", 4, "`h` inside `if` is not supported"),
    ("OPENQASM 3.0;\nqubit[2] q;\nbit[1] c;\nif (c[0]) { x q[0];\n measure q[1] -> c[0]; }", 5,
     "`measure` inside `if` is not supported"),
    ("OPENQASM 3.0;\nqubit[2] q;\nbit[1] c;\nif (c[0] == 2) x q[0];", 4, "only be compared with 0, 1, true or false"),
    ("OPENQASM 3.0;\nqubit[2] q;\nbit[1] c;\nelse x q[0];", 4, "`else` is not supported"),
    ("OPENQASM 3.0;\nqubit[2] q;\nfor int i in [0:1] { h q[i]; }", 3, "`for` is not supported"),
    ("OPENQASM 2.0;\nqreg q[2];\ncx q[0], q[0];", 3, "same qubit twice"),
    ('OPENQASM 2.0;\ninclude "mylib.inc";', 2, "only qelib1.inc and stdgates.inc"),
    ("OPENQASM 2.0;\nqreg q[2];\nh r[0];", 3, "unknown qubit register `r`"),
    ("OPENQASM 2.0;\nqreg q[1];\nrz(theta) q[0];", 3, "unknown parameter `theta`"),
]


@pytest.mark.parametrize("program,line,message", ERRORS)
def test_errors_point_at_the_problem(program, line, message):
    with pytest.raises(QasmError) as e:
        parse(program)
    assert e.value.line == line and message in e.value.message, str(e.value)


def test_relative_phase_toffolis_follow_qelib1(oracle):
    parsed = parse('OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[3];\nrccx q[0], q[1], q[2];')
    q4 = math.pi / 4
    h = Gate("u", (math.pi / 2, 0.0, math.pi))
    direct = Circuit(3)
    for g, qs in [(h, [2]), (Gate("p", (q4,)), [2]), (Gate("cx"), [1, 2]), (Gate("p", (-q4,)), [2]),
                  (Gate("cx"), [0, 2]), (Gate("p", (q4,)), [2]), (Gate("cx"), [1, 2]), (Gate("p", (-q4,)), [2]),
                  (h, [2])]:
        direct._instructions.append(("gate", g, qs))
    assert max_distance(state(oracle, direct), state(oracle, parsed)) < 1e-12
    redefined = parse("OPENQASM 2.0;\ngate rccx a,b,c { ccx a,b,c; }\nqreg q[3];\nrccx q[0], q[1], q[2];")
    assert len(redefined._instructions) == 1


def test_run_and_statevector_take_the_reference_arguments():
    """`run` and `statevector` accept what the reference's Python wrappers
    accept (python/python/qevedo/simulator/__init__.py:96-106, :141): a
    Circuit or OpenQASM text, and the `threads` (and, for `run`, MPS)
    keywords, which do not change the state-vector result."""
    import inspect

    from qevedo_simulator_b200 import simulator

    run_params = inspect.signature(simulator.run).parameters
    for name, default in (("backend", "auto"), ("seed", None), ("precision", "single"),
                          ("max_bond_dimension", 256), ("truncation_threshold", 1e-16), ("threads", None)):
        assert run_params[name].default == default, name
    sv_params = inspect.signature(simulator.statevector).parameters
    assert sv_params["threads"].default is None and sv_params["precision"].default == "double"
    c = simulator._as_circuit('OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[2];\ncreg c[2];\n'
                              'h q[0];\ncx q[0],q[1];\nmeasure q -> c;')
    assert (c.num_qubits, c.num_clbits, c.gate_count) == (2, 2, 2)


def test_run_result_has_the_binding_fields():
    from qevedo_simulator_b200.simulator import RunResult

    r = RunResult(counts={"00": 3, "11": 5})
    assert (r.backend, r.fidelity, r.max_bond_dimension, r.peak_active_qubits) == ("statevector", None, None, None)
    assert repr(r) == 'RunResult(backend="statevector", 2 outcomes)'


def test_expression_grammar_and_lexical_forms():
    """Precedence as the reference's grammar (src/qasm.rs:1290-1345): + -
    below * /, then right-associative ^ / **, and a sign binding tighter
    than all of them (-2^2 = 4); numbers with underscores and exponents;
    comments of both forms; unicode constants."""
    cases = {"-2^2": 4.0, "2^3^2": 2.0 ** 9, "2**-1": 0.5, "1+2*3": 7.0, "(1+2)*3": 9.0, "8/2/2": 2.0,
             "1_000e-3": 1.0, ".5": 0.5, "-pi/2 + π/2": 0.0, "sqrt(4)*cos(0)": 2.0, "2*-3": -6.0, "tau - 2*pi": 0.0}
    for text, want in cases.items():
        c = parse(f"OPENQASM 3.0;\nqubit q; // a comment\n/* block\ncomment */ rz({text}) q;")
        (kind, gate, qubits), = c._instructions
        assert gate.name == "rz" and gate.params[0] == pytest.approx(want, abs=1e-15), text
    for program, message in [("OPENQASM 3.0;\n/* open", "unterminated comment"),
                             ('OPENQASM 3.0;\ninclude "x', "unterminated string"),
                             ("OPENQASM 3.0;\nqubit q;\nrz(1 # 2) q;", "unexpected character `#`"),
                             ("OPENQASM 3.0;\nqubit q;\nrz(foo(1)) q;", "unknown function `foo`"),
                             ("OPENQASM 3.0;\nqubit q;\nrz(1 +) q;", "expected an expression"),
                             ("OPENQASM 5.0;", "only OpenQASM 2 and 3"),
                             ("OPENQASM 3.0;\nqubit q;\nqubit q;", "already declared")]:
        with pytest.raises(QasmError, match=message):
            parse(program)


def test_register_named_like_a_gate_and_gate_named_like_a_modifier():
    c = parse("OPENQASM 3.0;\nqubit[2] q;\nbit[2] x;\nx q[0];\nx = measure q;\n"
              "gate inv a { h a; }\ninv q[1];")
    assert [i[0] for i in c._instructions] == ["gate", "measure", "measure", "gate"]
    assert c._instructions[0][1].name == "x" and c._instructions[-1][1].name == "h"
