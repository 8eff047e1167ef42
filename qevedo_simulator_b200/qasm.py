"""Reading OpenQASM 2 and 3 programs into circuits.

The front end of the reference's `qvd::qasm::parse` (src/qasm.rs) for the
state-vector engine: registers (`qreg`/`creg`, `qubit`/`bit`), the gates of
`qelib1.inc` / `stdgates.inc` (natively where the circuit builder has the
gate, as exact unitaries for `csx`, `cu3`, `cu`, `c3x`, `c3sqrtx`, `c4x`, and
through their `qelib1.inc` definitions for `rccx` / `rc3x`), gate
definitions (expanded where called), parameter expressions, broadcasting
over registers and ranges, measure, reset, barrier, `gphase` (ignored), the
modifiers `inv @`, `ctrl(n) @`, `negctrl(n) @` and integer `pow(k) @`, and
`if` on one classical bit with Pauli-only bodies (read as classical
feedback). Anything else that needs classical state is rejected with the
line and column of the statement (QasmError).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .circuit import Circuit, Gate, _controlled

# Definitions of the relative-phase Toffolis, as in qelib1.inc; a program may
# redefine them.
_PRELUDE = """
gate rccx a,b,c
{
  u2(0,pi) c; u1(pi/4) c; cx b, c; u1(-pi/4) c; cx a, c;
  u1(pi/4) c; cx b, c; u1(-pi/4) c; u2(0,pi) c;
}
gate rc3x a,b,c,d
{
  u2(0,pi) d; u1(pi/4) d; cx c,d; u1(-pi/4) d; u2(0,pi) d;
  cx a,d; u1(pi/4) d; cx b,d; u1(-pi/4) d; cx a,d;
  u1(pi/4) d; cx b,d; u1(-pi/4) d; u2(0,pi) d;
  u1(pi/4) d; cx c,d; u1(-pi/4) d; u2(0,pi) d;
}
"""

# Statement keywords that need classical state the engine does not model.
_UNSUPPORTED = {"else", "for", "while", "def", "defcal", "defcalgrammar", "cal", "let", "const", "input", "output",
                "int", "uint", "float", "angle", "bool", "complex", "duration", "stretch", "delay", "box", "return",
                "break", "continue", "end", "extern", "array", "opaque", "pragma"}

_SYMBOLS2 = {"->", "**", "==", "!="}
_SYMBOLS1 = set(";,()[]{}=+-*/^@:<>!&|%~$")


class QasmError(ValueError):
    """A syntax or semantic error at `line`, `column` (1-based)."""

    def __init__(self, line: int, column: int, message: str):
        super().__init__(f"line {line}, column {column}: {message}")
        self.line, self.column, self.message = line, column, message


@dataclass
class _Tok:
    kind: str  # "id", "num", "str", "sym", "end"
    value: object
    line: int
    column: int


def _lex(src: str) -> list:
    toks, i, line, col = [], 0, 1, 1
    n = len(src)

    def adv(k):
        nonlocal i, line, col
        for _ in range(k):
            if src[i] == "\n":
                line, col = line + 1, 1
            else:
                col += 1
            i += 1

    while i < n:
        c = src[i]
        sl, sc = line, col
        if c.isspace():
            adv(1)
        elif src.startswith("//", i):
            while i < n and src[i] != "\n":
                adv(1)
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            if j < 0:
                raise QasmError(sl, sc, "unterminated comment")
            adv(j + 2 - i)
        elif c.isalpha() or c == "_":
            j = i
            while j < n and (src[j].isalnum() or src[j] == "_"):
                j += 1
            toks.append(_Tok("id", src[i:j], sl, sc))
            adv(j - i)
        elif c.isdigit() or (c == "." and i + 1 < n and src[i + 1].isdigit()):
            j = i
            while j < n and (src[j].isdigit() or src[j] in "._"):
                j += 1
            if j < n and src[j] in "eE":
                k = j + 1
                if k < n and src[k] in "+-":
                    k += 1
                if k < n and src[k].isdigit():
                    j = k
                    while j < n and src[j].isdigit():
                        j += 1
            text = src[i:j].replace("_", "")
            try:
                value = float(text)
            except ValueError:
                raise QasmError(sl, sc, f"invalid number `{text}`") from None
            toks.append(_Tok("num", value, sl, sc))
            adv(j - i)
        elif c in "\"'":
            j = i + 1
            while j < n and src[j] != c and src[j] != "\n":
                j += 1
            if j >= n or src[j] != c:
                raise QasmError(sl, sc, "unterminated string")
            toks.append(_Tok("str", src[i + 1:j], sl, sc))
            adv(j + 1 - i)
        elif src[i:i + 2] in _SYMBOLS2:
            toks.append(_Tok("sym", src[i:i + 2], sl, sc))
            adv(2)
        elif c in _SYMBOLS1:
            toks.append(_Tok("sym", c, sl, sc))
            adv(1)
        else:
            raise QasmError(sl, sc, f"unexpected character `{c}`")
    toks.append(_Tok("end", None, line, col))
    return toks


def _describe(t: _Tok) -> str:
    if t.kind == "end":
        return "the end of the program"
    if t.kind == "num":
        return f"number `{t.value:g}`"
    return f"`{t.value}`"


_CONSTANTS = {"pi": math.pi, "π": math.pi, "tau": math.tau, "τ": math.tau, "euler": math.e, "ℇ": math.e}
_FUNCTIONS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "ln": math.log, "sqrt": math.sqrt,
              "arcsin": math.asin, "asin": math.asin, "arccos": math.acos, "acos": math.acos, "arctan": math.atan,
              "atan": math.atan}


def _eval(expr, env: dict) -> float:
    kind = expr[0]
    if kind == "num":
        return expr[1]
    if kind == "name":
        _, name, tok = expr
        if name in _CONSTANTS:
            return _CONSTANTS[name]
        if name in env:
            return env[name]
        raise QasmError(tok.line, tok.column, f"unknown parameter `{name}`")
    if kind == "neg":
        return -_eval(expr[1], env)
    if kind == "bin":
        op, a, b = expr[1], _eval(expr[2], env), _eval(expr[3], env)
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if op == "/":
            return a / b
        return math.pow(a, b)
    _, name, arg, tok = expr  # call
    if name not in _FUNCTIONS:
        raise QasmError(tok.line, tok.column, f"unknown function `{name}`")
    return _FUNCTIONS[name](_eval(arg, env))


def _builtin(name: str, p: list):
    """(Gate, arity) for a built-in gate name, None if unknown; raises
    ValueError (message) on a wrong parameter count. src/qasm.rs:1377-1435."""

    def need(k):
        if len(p) != k:
            raise ValueError(f"`{name}` takes {k} parameters, given {len(p)}")

    simple = {"id": "id", "i": "id", "h": "h", "x": "x", "y": "y", "z": "z", "s": "s", "sdg": "sdg", "t": "t",
              "tdg": "tdg", "sx": "sx", "sxdg": "sxdg", "CX": "cx", "cx": "cx", "cnot": "cx", "cy": "cy",
              "cz": "cz", "ch": "ch", "swap": "swap", "ccx": "ccx", "toffoli": "ccx", "cswap": "cswap",
              "fredkin": "cswap"}
    one = {"rx": "rx", "ry": "ry", "rz": "rz", "p": "p", "u1": "p", "phase": "p", "cp": "cp", "cu1": "cp",
           "cphase": "cp", "crx": "crx", "cry": "cry", "crz": "crz", "rzz": "rzz", "rxx": "rxx"}
    if name in simple:
        need(0)
        g = Gate(simple[name])
        return g, g.arity
    if name in one:
        need(1)
        g = Gate(one[name], (float(p[0]),))
        return g, g.arity
    if name == "u0":
        need(1)
        return Gate("id"), 1
    if name == "u2":
        need(2)
        return Gate("u", (math.pi / 2, float(p[0]), float(p[1]))), 1
    if name in ("U", "u", "u3"):
        need(3)
        return Gate("u", tuple(float(v) for v in p)), 1
    x = Gate("x").matrix()
    sx = Gate("sx").matrix()
    if name == "csx":
        need(0)
        return Gate("unitary", (), _controlled(sx, 1, 1)), 2
    if name == "cu3":
        need(3)
        return Gate("unitary", (), _controlled(Gate("u", tuple(p)).matrix(), 1, 1)), 2
    if name == "cu":
        need(4)
        u = Gate("u", tuple(p[:3])).matrix() * complex(math.cos(p[3]), math.sin(p[3]))
        return Gate("unitary", (), _controlled(u, 1, 1)), 2
    if name == "c3x":
        need(0)
        return Gate("unitary", (), _controlled(x, 3, 7)), 4
    if name == "c4x":
        need(0)
        return Gate("unitary", (), _controlled(x, 4, 15)), 5
    if name == "c3sqrtx":
        need(0)
        return Gate("unitary", (), _controlled(sx, 3, 7)), 4
    return None


def _apply(state: np.ndarray, m: np.ndarray, qubits: list) -> np.ndarray:
    """m on `qubits` (matrix index bit j = qubits[j]) of a small state vector."""
    k = len(qubits)
    n = int(state.size).bit_length() - 1
    t = state.reshape([2] * n)
    axes = [n - 1 - q for q in reversed(qubits)]  # tensor axis of index bit
    t = np.moveaxis(t, axes, range(k))
    t = (m @ t.reshape(1 << k, -1)).reshape(t.shape)
    return np.moveaxis(t, range(k), axes).reshape(-1)


@dataclass
class _Call:
    modifiers: list
    name: str
    params: list
    args: list  # names, or ("idx", token position) for indexed operands
    tok: _Tok


@dataclass
class _Definition:
    params: list
    qubits: list
    body: list


@dataclass
class _Program:
    qubits: int = 0
    clbits: int = 0
    qregs: dict = field(default_factory=dict)
    cregs: dict = field(default_factory=dict)
    gates: dict = field(default_factory=dict)
    ins: list = field(default_factory=list)


class _Parser:
    def __init__(self, toks, program):
        self.toks, self.at, self.p = toks, 0, program

    # -- tokens
    def peek(self):
        return self.toks[self.at]

    def next(self):
        t = self.toks[self.at]
        if self.at + 1 < len(self.toks):
            self.at += 1
        return t

    def err(self, t, msg):
        raise QasmError(t.line, t.column, msg)

    def is_sym(self, s):
        t = self.peek()
        return t.kind == "sym" and t.value == s

    def is_word(self, w):
        t = self.peek()
        return t.kind == "id" and t.value == w

    def expect(self, s):
        t = self.next()
        if not (t.kind == "sym" and t.value == s):
            self.err(t, f"expected `{s}`, found {_describe(t)}")
        return t

    def ident(self):
        t = self.next()
        if t.kind != "id":
            self.err(t, f"expected a name, found {_describe(t)}")
        return t.value, t

    def integer(self):
        t = self.next()
        if t.kind != "num" or t.value < 0 or t.value != int(t.value):
            self.err(t, f"expected a non-negative integer, found {_describe(t)}")
        return int(t.value)

    # -- program
    def program(self):
        while self.peek().kind != "end":
            self.statement()

    def statement(self):
        t = self.peek()
        if t.kind != "id":
            self.err(t, f"expected a statement, found {_describe(t)}")
        w = t.value
        if w == "OPENQASM":
            self.next()
            v = self.next()
            if v.kind != "num" or not 2.0 <= v.value < 4.0:
                self.err(v, "only OpenQASM 2 and 3 are supported")
            self.expect(";")
        elif w == "include":
            self.next()
            f = self.next()
            if f.kind != "str":
                self.err(f, "expected a file name")
            if f.value not in ("qelib1.inc", "stdgates.inc"):
                self.err(f, f"cannot include `{f.value}`: only qelib1.inc and stdgates.inc are built in")
            self.expect(";")
        elif w in ("qreg", "creg"):
            self.next()
            name, at = self.ident()
            self.expect("[")
            size = self.integer()
            self.expect("]")
            self.expect(";")
            self.declare(w == "qreg", name, size, at)
        elif w in ("qubit", "bit"):
            self.next()
            size = 1
            if self.is_sym("["):
                self.next()
                size = self.integer()
                self.expect("]")
            name, at = self.ident()
            if self.is_sym("="):
                self.err(at, "initialising classical bits is not supported")
            self.expect(";")
            self.declare(w == "qubit", name, size, at)
        elif w == "gate":
            self.definition()
        elif w == "if":
            self.conditional()
        elif w == "measure":
            self.next()
            qs = self.operand(True)
            if not self.is_sym("->"):
                self.err(t, "a measurement must store its result (`measure q -> c;` or `c = measure q;`)")
            self.next()
            cs = self.operand(False)
            self.expect(";")
            self.measure(qs, cs, t)
        elif w == "reset":
            self.next()
            qs = self.operand(True)
            self.expect(";")
            for q in qs:
                self.p.ins.append(("reset", q))
        elif w == "barrier":
            self.next()
            qs = []
            while not self.is_sym(";"):
                qs.extend(self.operand(True))
                if self.is_sym(","):
                    self.next()
            self.expect(";")
            self.p.ins.append(("barrier", qs or list(range(self.p.qubits))))
        elif w == "gphase":
            while not self.is_sym(";") and self.peek().kind != "end":
                self.next()
            self.expect(";")
        elif w in _UNSUPPORTED:
            self.err(t, f"`{w}` is not supported (the simulator runs gates, measurements and resets only)")
        else:
            save = self.at
            self.next()
            if self.is_sym("[") or self.is_sym("="):
                self.at = save
                cs = self.operand(False)
                self.expect("=")
                kw, at = self.ident()
                if kw != "measure":
                    self.err(at, "assigning classical values other than measurements is not supported")
                qs = self.operand(True)
                self.expect(";")
                self.measure(qs, cs, t)
            else:
                self.at = save
                call = self.call()
                self.expect(";")
                self.top_level_call(call)

    def declare(self, quantum, name, size, at):
        if name in self.p.qregs or name in self.p.cregs:
            self.err(at, f"`{name}` is already declared")
        if quantum:
            self.p.qregs[name] = (self.p.qubits, size)
            self.p.qubits += size
        else:
            self.p.cregs[name] = (self.p.clbits, size)
            self.p.clbits += size

    def measure(self, qs, cs, at):
        if len(qs) != len(cs):
            self.err(at, f"measuring {len(qs)} qubits into {len(cs)} bits")
        for q, c in zip(qs, cs):
            self.p.ins.append(("measure", q, c))

    def operand(self, quantum):
        name, at = self.ident()
        regs = self.p.qregs if quantum else self.p.cregs
        if name not in regs:
            self.err(at, f"unknown {'qubit' if quantum else 'classical bit'} register `{name}`")
        first, size = regs[name]
        if not self.is_sym("["):
            return list(range(first, first + size))
        self.next()
        start = self.integer()
        idx = [start]
        if self.is_sym(":"):
            self.next()
            second = self.integer()
            step, end = 1, second
            if self.is_sym(":"):
                self.next()
                step, end = second, self.integer()
            if step == 0:
                self.err(at, "a range step must be positive")
            idx = list(range(start, end + 1, step))
        self.expect("]")
        for i in idx:
            if i >= size:
                self.err(at, f"index {i} is out of range for `{name}` of size {size}")
        return [first + i for i in idx]

    # -- expressions: + -, * /, ^ ** (right associative), unary minus
    def expression(self):
        left = self.term()
        while self.is_sym("+") or self.is_sym("-"):
            op = self.next().value
            left = ("bin", op, left, self.term())
        return left

    def term(self):
        left = self.power()
        while self.is_sym("*") or self.is_sym("/"):
            op = self.next().value
            left = ("bin", op, left, self.power())
        return left

    def power(self):
        base = self.unary()
        if self.is_sym("^") or self.is_sym("**"):
            self.next()
            return ("bin", "^", base, self.power())
        return base

    def unary(self):
        if self.is_sym("-"):
            self.next()
            return ("neg", self.unary())
        if self.is_sym("+"):
            self.next()
            return self.unary()
        t = self.next()
        if t.kind == "num":
            return ("num", t.value)
        if t.kind == "sym" and t.value == "(":
            e = self.expression()
            self.expect(")")
            return e
        if t.kind == "id":
            if self.is_sym("("):
                self.next()
                arg = self.expression()
                self.expect(")")
                return ("call", t.value, arg, t)
            return ("name", t.value, t)
        self.err(t, f"expected an expression, found {_describe(t)}")

    # -- gate calls
    def call(self):
        mods = []
        while True:
            t = self.peek()
            if t.kind != "id" or t.value not in ("inv", "ctrl", "negctrl", "pow"):
                break
            save = self.at
            self.next()
            arg = None
            if self.is_sym("("):
                self.next()
                arg = self.expression()
                self.expect(")")
            if not self.is_sym("@"):
                self.at = save
                break
            self.next()
            if t.value == "inv":
                mods.append(("inv",))
            elif t.value == "pow":
                if arg is None:
                    self.err(t, "`pow` needs an exponent")
                mods.append(("pow", arg, t))
            else:
                count = 1
                if arg is not None:
                    x = _eval(arg, {})
                    if x < 1 or x != int(x):
                        self.err(t, "a control count must be a positive integer")
                    count = int(x)
                mods.append((t.value, count))
        name, at = self.ident()
        params = []
        if self.is_sym("("):
            self.next()
            if not self.is_sym(")"):
                while True:
                    params.append(self.expression())
                    if self.is_sym(","):
                        self.next()
                    else:
                        break
            self.expect(")")
        args = []
        while not self.is_sym(";") and not self.is_sym("}") and self.peek().kind != "end":
            start = self.at
            arg, _ = self.ident()
            if self.is_sym("["):
                while not self.is_sym("]") and self.peek().kind != "end":
                    self.next()
                self.expect("]")
                arg = ("idx", start)
            args.append(arg)
            if self.is_sym(","):
                self.next()
            else:
                break
        return _Call(mods, name, params, args, at)

    def top_level_call(self, call):
        operands = []
        for a in call.args:
            if isinstance(a, tuple):
                save = self.at
                self.at = a[1]
                operands.append(self.operand(True))
                self.at = save
            else:
                if a not in self.p.qregs:
                    self.err(call.tok, f"unknown qubit register `{a}`")
                first, size = self.p.qregs[a]
                operands.append(list(range(first, first + size)))
        width = max([len(o) for o in operands if len(o) != 1] or [1])
        if any(len(o) not in (1, width) for o in operands):
            self.err(call.tok, "registers of different sizes cannot be broadcast together")
        params = [_eval(e, {}) for e in call.params]
        for i in range(width):
            qubits = [o[0] if len(o) == 1 else o[i] for o in operands]
            if len(set(qubits)) != len(qubits):
                self.err(call.tok, f"`{call.name}` is applied to the same qubit twice")
            self.p.ins.extend(self.expand(call.modifiers, call.name, params, qubits, call.tok, 0))

    def expand(self, mods, name, params, qubits, at, depth):
        if depth > 64:
            self.err(at, f"gate `{name}` is defined recursively")
        if mods:
            controls = sum(m[1] for m in mods if m[0] in ("ctrl", "negctrl"))
            if len(qubits) <= controls:
                self.err(at, f"`{name}` with {controls} controls needs more qubits")
            k = len(qubits) - controls
            body = self.expand([], name, params, list(range(k)), at, depth + 1)
            m = np.eye(1 << k, dtype=np.complex128)
            for col in range(1 << k):
                v = np.zeros(1 << k, dtype=np.complex128)
                v[col] = 1.0
                for ins in body:
                    v = _apply(v, ins[1].matrix(), ins[2])
                m[:, col] = v
            # Modifiers apply right to left: the one nearest the gate first.
            for mod in reversed(mods):
                if mod[0] == "inv":
                    m = m.conj().T
                elif mod[0] == "pow":
                    e = _eval(mod[1], {})
                    if e != int(e):
                        self.err(at, "only integer powers are supported")
                    base = m.conj().T if e < 0 else m
                    m = np.linalg.matrix_power(base, int(abs(e)))
                else:
                    c = mod[1]
                    m = _controlled(m, c, (1 << c) - 1 if mod[0] == "ctrl" else 0)
            return [("gate", Gate("unitary", (), m), list(qubits))]
        if name in self.p.gates:
            d = self.p.gates[name]
            if len(d.params) != len(params) or len(d.qubits) != len(qubits):
                self.err(at, f"`{name}` takes {len(d.params)} parameters and {len(d.qubits)} qubits, given "
                             f"{len(params)} and {len(qubits)}")
            env = dict(zip(d.params, params))
            where = dict(zip(d.qubits, qubits))
            out = []
            for c in d.body:
                values = [_eval(e, env) for e in c.params]
                args = []
                for a in c.args:
                    if a not in where:
                        self.err(c.tok, f"unknown qubit `{a}` in the definition of `{name}`")
                    args.append(where[a])
                out.extend(self.expand(c.modifiers, c.name, values, args, c.tok, depth + 1))
            return out
        try:
            found = _builtin(name, params)
        except ValueError as e:
            self.err(at, str(e))
        if found is None:
            self.err(at, f"unknown gate `{name}`")
        gate, arity = found
        if arity != len(qubits):
            self.err(at, f"`{name}` acts on {arity} qubits, given {len(qubits)}")
        return [("gate", gate, list(qubits))]

    def definition(self):
        self.next()
        name, at = self.ident()
        params = []
        if self.is_sym("("):
            self.next()
            while not self.is_sym(")"):
                params.append(self.ident()[0])
                if self.is_sym(","):
                    self.next()
            self.expect(")")
        qubits = []
        while not self.is_sym("{"):
            qubits.append(self.ident()[0])
            if self.is_sym(","):
                self.next()
        self.expect("{")
        body = []
        while not self.is_sym("}"):
            if self.peek().kind == "end":
                self.err(at, f"unterminated definition of `{name}`")
            if self.is_word("barrier"):
                while not self.is_sym(";"):
                    self.next()
                self.expect(";")
                continue
            c = self.call()
            if any(isinstance(a, tuple) for a in c.args):
                self.err(at, f"the body of `{name}` can only use its own qubit names")
            body.append(c)
            self.expect(";")
        self.expect("}")
        self.p.gates[name] = _Definition(params, qubits, body)

    # -- if on one bit with Pauli bodies: classical feedback
    def conditional(self):
        at = self.next()
        self.expect("(")
        clbit, wanted = self.condition()
        self.expect(")")
        then = self.pauli_body(at)
        other = {}
        if self.is_word("else"):
            self.next()
            other = self.pauli_body(at)
        on_one, on_zero = (then, other) if wanted else (other, then)
        letters = {1: "X", 2: "Z", 3: "Y"}
        for q, bits in on_zero.items():
            if bits in letters:
                self.p.ins.append(("gate", Gate(letters[bits].lower()), [q]))
        for q in sorted(set(on_one) | set(on_zero)):
            flip = on_one.get(q, 0) ^ on_zero.get(q, 0)
            if flip in letters:
                self.p.ins.append(("feedback", letters[flip], q, clbit))

    def condition(self):
        negated = False
        while self.is_sym("!"):
            self.next()
            negated = not negated
        name, at = self.ident()
        if name not in self.p.cregs:
            self.err(at, f"unknown classical bit register `{name}` in a condition")
        first, size = self.p.cregs[name]
        if self.is_sym("["):
            self.next()
            index = self.integer()
            self.expect("]")
            if index >= size:
                self.err(at, f"index {index} is out of range for `{name}` of size {size}")
            clbit = first + index
        elif size == 1:
            clbit = first
        else:
            self.err(at, f"a condition on `{name}`, a register of {size} bits, is not supported: only one bit can "
                         f"be tested (`if ({name}[k])`)")
        wanted = True
        if self.is_sym("==") or self.is_sym("!="):
            equal = self.next().value == "=="
            t = self.next()
            if t.kind == "num" and t.value in (0.0, 1.0):
                value = t.value == 1.0
            elif t.kind == "id" and t.value in ("true", "false"):
                value = t.value == "true"
            else:
                self.err(t, f"a bit can only be compared with 0, 1, true or false, not {_describe(t)}")
            wanted = value == equal
        return clbit, wanted != negated

    def pauli_body(self, at):
        block = self.is_sym("{")
        if block:
            self.next()
        start = len(self.p.ins)
        while True:
            if block and self.is_sym("}"):
                self.next()
                break
            t = self.peek()
            if t.kind == "id" and t.value == "barrier":
                while not self.is_sym(";") and self.peek().kind != "end":
                    self.next()
                self.expect(";")
            elif t.kind == "id" and (t.value in ("measure", "reset", "if", "gate") or t.value in _UNSUPPORTED):
                self.err(t, f"`{t.value}` inside `if` is not supported: an `if` body can only apply Pauli gates "
                            "(x, y, z, id)")
            elif t.kind == "id":
                call = self.call()
                self.expect(";")
                before = len(self.p.ins)
                self.top_level_call(call)
                if not all(i[0] == "gate" and i[1].name in ("id", "x", "y", "z") for i in self.p.ins[before:]):
                    self.err(t, f"`{call.name}` inside `if` is not supported: an `if` body can only apply Pauli "
                                "gates (x, y, z, id), which run as classical feedback")
            elif t.kind == "end":
                self.err(at, "unterminated `if` block")
            else:
                self.err(t, f"expected a gate call, found {_describe(t)}")
            if not block:
                break
        body = {}
        for ins in self.p.ins[start:]:
            if ins[0] == "gate":
                bits = {"x": 1, "z": 2, "y": 3}.get(ins[1].name, 0)
                body[ins[2][0]] = body.get(ins[2][0], 0) ^ bits
        del self.p.ins[start:]
        return body


def parse(source: str) -> Circuit:
    """An OpenQASM 2 or 3 program as a circuit; qubits and classical bits
    are numbered in declaration order across registers."""
    prelude = _Parser(_lex(_PRELUDE), _Program())
    prelude.program()
    parser = _Parser(_lex(source), _Program(gates=dict(prelude.p.gates)))
    parser.program()
    p = parser.p
    c = Circuit(p.qubits, p.clbits)
    c._instructions.extend(p.ins)
    return c
