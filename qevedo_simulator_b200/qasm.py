"""OpenQASM 2 and 3 programs read into circuits.

The state-vector engine's reader for the programs the reference's
`qvd::qasm::parse` (src/qasm.rs) takes: registers (`qreg`/`creg`,
`qubit`/`bit`), the `qelib1.inc` / `stdgates.inc` gates, user gate
definitions, parameter expressions, broadcasting over registers and ranges,
`measure` (both forms), `reset`, `barrier`, `gphase` (a global phase, so
dropped), the modifiers `inv @`, `ctrl(n) @`, `negctrl(n) @` and integer
`pow(k) @`, and `if` on one classical bit whose bodies apply Pauli gates
(lowered to classical feedback). Statements that need classical state the
engine does not keep are refused with their line and column (QasmError).

Design: one regular expression built from a token table splits the text;
expressions are parsed by precedence climbing into closures over the gate
parameters; statements are dispatched by keyword through a table; gate
applications are lowered straight to the circuit's instructions, with a
modified gate or a modified definition turned into one unitary. The user
visible error messages and the instruction forms are the reference's.
"""

from __future__ import annotations

import bisect
import math
import operator
import re
from dataclasses import dataclass
from typing import Callable

import numpy as np

from .circuit import Circuit, Gate, _controlled


class QasmError(ValueError):
    """A syntax or semantic error at `line`, `column` (1-based)."""

    def __init__(self, line: int, column: int, message: str):
        super().__init__(f"line {line}, column {column}: {message}")
        self.line, self.column, self.message = line, column, message


# ------------------------------------------------------------------ tokens
# (kind, pattern), tried in this order at every position.
_TOKEN_TABLE = (
    ("space", r"\s+"),
    ("comment", r"//[^\n]*|/\*.*?\*/"),
    ("open_comment", r"/\*"),
    ("number", r"(?:\d[\d_]*(?:\.[\d_]*)?|\.\d[\d_]*)(?:[eE][+-]?\d+)?"),
    ("name", r"[^\W\d]\w*"),
    ("string", r"\"[^\"\n]*\"|'[^'\n]*'"),
    ("open_string", r"[\"']"),
    ("symbol", r"->|\*\*|==|!=|[;,()\[\]{}=+\-*/^@:<>!&|%~$]"),
)
_SCANNER = re.compile("|".join(f"(?P<{kind}>{pattern})" for kind, pattern in _TOKEN_TABLE), re.S)


@dataclass(frozen=True)
class _Token:
    kind: str  # "name", "number", "string", "symbol" or "end"
    text: str
    pos: int

    @property
    def number(self) -> float:
        return float(self.text.replace("_", ""))


class _Tokens:
    """The tokens of one source text and a cursor over them."""

    def __init__(self, text: str):
        self.text = text
        self.line_starts = [0] + [m.end() for m in re.finditer("\n", text)]
        self.items: list[_Token] = []
        pos = 0
        while pos < len(text):
            m = _SCANNER.match(text, pos)
            if m is None:
                self.fail_at(pos, f"unexpected character `{text[pos]}`")
            kind = m.lastgroup
            if kind == "open_comment":
                self.fail_at(pos, "unterminated comment")
            if kind == "open_string":
                self.fail_at(pos, "unterminated string")
            if kind == "number":
                try:
                    float(m.group().replace("_", ""))
                except ValueError:
                    self.fail_at(pos, f"invalid number `{m.group()}`")
            if kind == "string":
                self.items.append(_Token("string", m.group()[1:-1], pos))
            elif kind not in ("space", "comment"):
                self.items.append(_Token(kind, m.group(), pos))
            pos = m.end()
        self.items.append(_Token("end", "", len(text)))
        self.at = 0

    # positions and errors
    def where(self, pos: int) -> tuple:
        line = bisect.bisect_right(self.line_starts, pos)
        return line, pos - self.line_starts[line - 1] + 1

    def fail_at(self, pos: int, message: str):
        raise QasmError(*self.where(pos), message)

    def fail(self, tok: _Token, message: str):
        self.fail_at(tok.pos, message)

    @staticmethod
    def describe(tok: _Token) -> str:
        if tok.kind == "end":
            return "the end of the program"
        if tok.kind == "number":
            return f"number `{tok.number:g}`"
        return f"`{tok.text}`"

    # the cursor
    def peek(self) -> _Token:
        return self.items[self.at]

    def take(self) -> _Token:
        tok = self.items[self.at]
        self.at = min(self.at + 1, len(self.items) - 1)
        return tok

    def at_symbol(self, text: str) -> bool:
        tok = self.items[self.at]
        return tok.kind == "symbol" and tok.text == text

    def at_name(self, text: str) -> bool:
        tok = self.items[self.at]
        return tok.kind == "name" and tok.text == text

    def at_end(self) -> bool:
        return self.items[self.at].kind == "end"

    def accept(self, text: str) -> bool:
        if self.at_symbol(text):
            self.take()
            return True
        return False

    def require(self, text: str) -> _Token:
        tok = self.take()
        if tok.kind != "symbol" or tok.text != text:
            self.fail(tok, f"expected `{text}`, found {self.describe(tok)}")
        return tok

    def name(self) -> _Token:
        tok = self.take()
        if tok.kind != "name":
            self.fail(tok, f"expected a name, found {self.describe(tok)}")
        return tok

    def index(self) -> int:
        tok = self.take()
        if tok.kind != "number" or tok.number < 0 or tok.number != int(tok.number):
            self.fail(tok, f"expected a non-negative integer, found {self.describe(tok)}")
        return int(tok.number)

    def skip_past(self, text: str):
        while not self.at_symbol(text) and not self.at_end():
            self.take()
        self.require(text)


# ------------------------------------------------------------- expressions
Expr = Callable[[dict], float]

_CONSTANTS = {"pi": math.pi, "π": math.pi, "tau": math.tau, "τ": math.tau, "euler": math.e, "ℇ": math.e}
_FUNCTIONS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "ln": math.log, "sqrt": math.sqrt,
              "arcsin": math.asin, "asin": math.asin, "arccos": math.acos, "acos": math.acos, "arctan": math.atan,
              "atan": math.atan}
# Infix operators: symbol -> (binding power, right associative, function).
_INFIX = {"+": (10, False, operator.add), "-": (10, False, operator.sub), "*": (20, False, operator.mul),
          "/": (20, False, operator.truediv), "^": (30, True, math.pow), "**": (30, True, math.pow)}
# A sign binds tighter than every infix operator (-2^2 is (-2)^2, as in the
# reference's grammar).
_PREFIX_POWER = 40


def _expression(toks: _Tokens, min_power: int = 0) -> Expr:
    """Precedence climbing over _INFIX; the result evaluates in an
    environment of parameter values."""
    left = _primary(toks)
    while True:
        tok = toks.peek()
        entry = _INFIX.get(tok.text) if tok.kind == "symbol" else None
        if entry is None or entry[0] < min_power:
            return left
        power, right_assoc, fn = entry
        toks.take()
        right = _expression(toks, power if right_assoc else power + 1)
        left = (lambda f, a, b: lambda env: f(a(env), b(env)))(fn, left, right)


def _primary(toks: _Tokens) -> Expr:
    tok = toks.take()
    if tok.kind == "symbol" and tok.text in "+-" and len(tok.text) == 1:
        inner = _expression(toks, _PREFIX_POWER)
        return inner if tok.text == "+" else (lambda env: -inner(env))
    if tok.kind == "number":
        value = tok.number
        return lambda env: value
    if tok.kind == "symbol" and tok.text == "(":
        inner = _expression(toks)
        toks.require(")")
        return inner
    if tok.kind == "name":
        if toks.accept("("):
            arg = _expression(toks)
            toks.require(")")
            return _function_call(toks, tok, arg)
        return _variable(toks, tok)
    toks.fail(tok, f"expected an expression, found {toks.describe(tok)}")


def _function_call(toks: _Tokens, tok: _Token, arg: Expr) -> Expr:
    def call(env):
        fn = _FUNCTIONS.get(tok.text)
        if fn is None:
            toks.fail(tok, f"unknown function `{tok.text}`")
        return fn(arg(env))

    return call


def _variable(toks: _Tokens, tok: _Token) -> Expr:
    def value(env):
        if tok.text in _CONSTANTS:
            return _CONSTANTS[tok.text]
        if tok.text in env:
            return env[tok.text]
        toks.fail(tok, f"unknown parameter `{tok.text}`")

    return value


# ------------------------------------------------------------ gate library
def _gate_library():
    """name -> (parameter count, maker(params) -> (Gate, arity)) for the
    gates of qelib1.inc and stdgates.inc (src/qasm.rs:1377-1435), with the
    ones the circuit builder lacks as exact controlled unitaries."""

    def named(kind):
        def make(p):
            g = Gate(kind, tuple(float(v) for v in p))
            return g, g.arity

        return make

    def controlled(base, controls):
        return lambda p: (Gate("unitary", (), _controlled(base(p), controls, (1 << controls) - 1)), controls + 1)

    table = {}
    for kind, aliases in (("id", ("id", "i")), ("h", ("h",)), ("x", ("x",)), ("y", ("y",)), ("z", ("z",)),
                          ("s", ("s",)), ("sdg", ("sdg",)), ("t", ("t",)), ("tdg", ("tdg",)), ("sx", ("sx",)),
                          ("sxdg", ("sxdg",)), ("cx", ("CX", "cx", "cnot")), ("cy", ("cy",)), ("cz", ("cz",)),
                          ("ch", ("ch",)), ("swap", ("swap",)), ("ccx", ("ccx", "toffoli")),
                          ("cswap", ("cswap", "fredkin"))):
        for alias in aliases:
            table[alias] = (0, named(kind))
    for kind, aliases in (("rx", ("rx",)), ("ry", ("ry",)), ("rz", ("rz",)), ("p", ("p", "u1", "phase")),
                          ("cp", ("cp", "cu1", "cphase")), ("crx", ("crx",)), ("cry", ("cry",)), ("crz", ("crz",)),
                          ("rzz", ("rzz",)), ("rxx", ("rxx",))):
        for alias in aliases:
            table[alias] = (1, named(kind))
    table["u0"] = (1, lambda p: (Gate("id"), 1))
    table["u2"] = (2, lambda p: named("u")([math.pi / 2, p[0], p[1]]))
    for alias in ("U", "u", "u3"):
        table[alias] = (3, named("u"))
    x, sx = (lambda p: Gate("x").matrix()), (lambda p: Gate("sx").matrix())
    table["csx"] = (0, controlled(sx, 1))
    table["cu3"] = (3, controlled(lambda p: Gate("u", tuple(p)).matrix(), 1))
    table["cu"] = (4, controlled(lambda p: Gate("u", tuple(p[:3])).matrix() * complex(math.cos(p[3]),
                                                                                        math.sin(p[3])), 1))
    table["c3x"] = (0, controlled(x, 3))
    table["c4x"] = (0, controlled(x, 4))
    table["c3sqrtx"] = (0, controlled(sx, 3))
    return table


_LIBRARY = _gate_library()

# The relative-phase Toffolis through their qelib1.inc definitions (a
# program may redefine them).
_PRELUDE = """
gate rccx a,b,c { u2(0,pi) c; u1(pi/4) c; cx b,c; u1(-pi/4) c; cx a,c; u1(pi/4) c; cx b,c; u1(-pi/4) c;
                  u2(0,pi) c; }
gate rc3x a,b,c,d { u2(0,pi) d; u1(pi/4) d; cx c,d; u1(-pi/4) d; u2(0,pi) d; cx a,d; u1(pi/4) d; cx b,d;
                    u1(-pi/4) d; cx a,d; u1(pi/4) d; cx b,d; u1(-pi/4) d; u2(0,pi) d; u1(pi/4) d; cx c,d;
                    u1(-pi/4) d; u2(0,pi) d; }
"""

# Keywords of statements that need classical state the engine does not keep.
_REFUSED = {"else", "for", "while", "def", "defcal", "defcalgrammar", "cal", "let", "const", "input", "output",
            "int", "uint", "float", "angle", "bool", "complex", "duration", "stretch", "delay", "box", "return",
            "break", "continue", "end", "extern", "array", "opaque", "pragma"}
_MODIFIERS = ("inv", "ctrl", "negctrl", "pow")
_PAULI_BITS = {"x": 1, "z": 2, "y": 3}  # X = 1, Z = 2, Y = X.Z up to phase
_PAULI_LETTER = {1: "X", 2: "Z", 3: "Y"}


def _embed(m: np.ndarray, qubits: list, k: int) -> np.ndarray:
    """`m` (matrix index bit j = qubits[j]) as a 2^k x 2^k matrix."""
    idx = np.arange(1 << k)
    sub = np.zeros_like(idx)
    rest = idx.copy()
    for j, q in enumerate(qubits):
        sub |= ((idx >> q) & 1) << j
        rest &= ~(1 << q)
    return np.where(rest[:, None] == rest[None, :], m[sub[:, None], sub[None, :]], 0)


def _unitary(instructions: list, k: int) -> np.ndarray:
    """The product of gate instructions on qubits 0..k-1 (first applied first)."""
    u = np.eye(1 << k, dtype=np.complex128)
    for _, gate, qubits in instructions:
        u = _embed(gate.matrix(), qubits, k) @ u
    return u


# ---------------------------------------------------------------- programs
@dataclass
class _Operand:
    register: _Token
    indices: list | None  # None: the whole register


@dataclass
class _Application:
    modifiers: list  # ("inv",) | ("pow", Expr, tok) | ("ctrl"|"negctrl", count)
    name: _Token
    params: list  # of Expr
    operands: list  # of _Operand


@dataclass
class _Definition:
    params: list  # names
    qubits: list  # names
    body: list  # of _Application


class _Program:
    """Registers, definitions and the instructions emitted so far."""

    def __init__(self, definitions: dict | None = None):
        self.qubits = self.clbits = 0
        self.qregs: dict = {}
        self.cregs: dict = {}
        self.definitions = dict(definitions or {})
        self.out: list = []

    def read(self, text: str):
        toks = _Tokens(text)
        while not toks.at_end():
            _statement(self, toks)

    # registers
    def declare(self, toks, quantum: bool, name: _Token, size: int):
        if name.text in self.qregs or name.text in self.cregs:
            toks.fail(name, f"`{name.text}` is already declared")
        if quantum:
            self.qregs[name.text] = (self.qubits, size)
            self.qubits += size
        else:
            self.cregs[name.text] = (self.clbits, size)
            self.clbits += size

    def resolve(self, toks, operand: _Operand, quantum: bool) -> list:
        regs = self.qregs if quantum else self.cregs
        reg = operand.register
        if reg.text not in regs:
            toks.fail(reg, f"unknown {'qubit' if quantum else 'classical bit'} register `{reg.text}`")
        first, size = regs[reg.text]
        if operand.indices is None:
            return list(range(first, first + size))
        for i in operand.indices:
            if i >= size:
                toks.fail(reg, f"index {i} is out of range for `{reg.text}` of size {size}")
        return [first + i for i in operand.indices]

    # gates
    def apply(self, toks, app: _Application):
        """A top-level application, broadcast over register operands."""
        groups = [self.resolve(toks, o, True) for o in app.operands]
        width = max([len(g) for g in groups if len(g) != 1] or [1])
        if any(len(g) not in (1, width) for g in groups):
            toks.fail(app.name, "registers of different sizes cannot be broadcast together")
        values = [e({}) for e in app.params]
        for i in range(width):
            qubits = [g[0] if len(g) == 1 else g[i] for g in groups]
            if len(set(qubits)) != len(qubits):
                toks.fail(app.name, f"`{app.name.text}` is applied to the same qubit twice")
            self.out.extend(self.lower(toks, app.modifiers, app.name, values, qubits, 0))

    def lower(self, toks, modifiers: list, name: _Token, values: list, qubits: list, depth: int) -> list:
        """Instructions of gate `name` with parameter values on global qubits."""
        if depth > 64:
            toks.fail(name, f"gate `{name.text}` is defined recursively")
        if modifiers:
            return [self.modified(toks, modifiers, name, values, qubits, depth)]
        d = self.definitions.get(name.text)
        if d is not None:
            if len(d.params) != len(values) or len(d.qubits) != len(qubits):
                toks.fail(name, f"`{name.text}` takes {len(d.params)} parameters and {len(d.qubits)} qubits, "
                                f"given {len(values)} and {len(qubits)}")
            env = dict(zip(d.params, values))
            wires = dict(zip(d.qubits, qubits))
            out = []
            for app in d.body:
                inner = []
                for o in app.operands:
                    if o.register.text not in wires:
                        toks.fail(o.register, f"unknown qubit `{o.register.text}` in the definition of `{name.text}`")
                    inner.append(wires[o.register.text])
                out.extend(self.lower(toks, app.modifiers, app.name, [e(env) for e in app.params], inner, depth + 1))
            return out
        entry = _LIBRARY.get(name.text)
        if entry is None:
            toks.fail(name, f"unknown gate `{name.text}`")
        count, make = entry
        if count != len(values):
            toks.fail(name, f"`{name.text}` takes {count} parameters, given {len(values)}")
        gate, arity = make(values)
        if arity != len(qubits):
            toks.fail(name, f"`{name.text}` acts on {arity} qubits, given {len(qubits)}")
        return [("gate", gate, list(qubits))]

    def modified(self, toks, modifiers, name, values, qubits, depth):
        """One unitary for a modified gate: the gate's own unitary on its
        target qubits, then each modifier from the one nearest the gate."""
        controls = sum(m[1] for m in modifiers if m[0] in ("ctrl", "negctrl"))
        k = len(qubits) - controls
        if k <= 0:
            toks.fail(name, f"`{name.text}` with {controls} controls needs more qubits")
        u = _unitary(self.lower(toks, [], name, values, list(range(k)), depth + 1), k)
        for mod in reversed(modifiers):
            if mod[0] == "inv":
                u = u.conj().T
            elif mod[0] == "pow":
                e = mod[1]({})
                if e != int(e):
                    toks.fail(name, "only integer powers are supported")
                u = np.linalg.matrix_power(u.conj().T if e < 0 else u, int(abs(e)))
            else:
                c = mod[1]
                u = _controlled(u, c, (1 << c) - 1 if mod[0] == "ctrl" else 0)
        return ("gate", Gate("unitary", (), u), list(qubits))


# -------------------------------------------------------------- statements
def _statement(p: _Program, toks: _Tokens):
    tok = toks.peek()
    if tok.kind != "name":
        toks.fail(tok, f"expected a statement, found {toks.describe(tok)}")
    handler = _STATEMENTS.get(tok.text)
    if handler is not None:
        handler(p, toks)
    elif tok.text in _REFUSED:
        toks.fail(tok, f"`{tok.text}` is not supported (the simulator runs gates, measurements and resets only)")
    elif tok.text in p.cregs and toks.items[toks.at + 1].text in ("[", "="):
        _assigned_measure(p, toks)
    else:
        app = _application(toks)
        toks.require(";")
        p.apply(toks, app)


def _version(p, toks):
    toks.take()
    v = toks.take()
    if v.kind != "number" or not 2.0 <= v.number < 4.0:
        toks.fail(v, "only OpenQASM 2 and 3 are supported")
    toks.require(";")


def _include(p, toks):
    toks.take()
    f = toks.take()
    if f.kind != "string":
        toks.fail(f, "expected a file name")
    if f.text not in ("qelib1.inc", "stdgates.inc"):
        toks.fail(f, f"cannot include `{f.text}`: only qelib1.inc and stdgates.inc are built in")
    toks.require(";")


def _register_v2(p, toks):
    quantum = toks.take().text == "qreg"
    name = toks.name()
    toks.require("[")
    size = toks.index()
    toks.require("]")
    toks.require(";")
    p.declare(toks, quantum, name, size)


def _register_v3(p, toks):
    quantum = toks.take().text == "qubit"
    size = 1
    if toks.accept("["):
        size = toks.index()
        toks.require("]")
    name = toks.name()
    if toks.at_symbol("="):
        toks.fail(name, "initialising classical bits is not supported")
    toks.require(";")
    p.declare(toks, quantum, name, size)


def _operand(toks: _Tokens) -> _Operand:
    """`name`, `name[i]` or `name[start:stop]` / `name[start:step:stop]`
    (inclusive stop)."""
    reg = toks.name()
    if not toks.accept("["):
        return _Operand(reg, None)
    parts = [toks.index()]
    while toks.accept(":"):
        parts.append(toks.index())
    toks.require("]")
    if len(parts) == 1:
        return _Operand(reg, parts)
    start, step, stop = (parts[0], 1, parts[1]) if len(parts) == 2 else parts[:3]
    if step == 0:
        toks.fail(reg, "a range step must be positive")
    return _Operand(reg, list(range(start, stop + 1, step)))


def _record_measures(p, toks, qubits, clbits, at):
    if len(qubits) != len(clbits):
        toks.fail(at, f"measuring {len(qubits)} qubits into {len(clbits)} bits")
    p.out.extend(("measure", q, c) for q, c in zip(qubits, clbits))


def _measure_arrow(p, toks):
    at = toks.take()
    qubits = p.resolve(toks, _operand(toks), True)
    if not toks.accept("->"):
        toks.fail(at, "a measurement must store its result (`measure q -> c;` or `c = measure q;`)")
    clbits = p.resolve(toks, _operand(toks), False)
    toks.require(";")
    _record_measures(p, toks, qubits, clbits, at)


def _assigned_measure(p, toks):
    at = toks.peek()
    clbits = p.resolve(toks, _operand(toks), False)
    toks.require("=")
    kw = toks.name()
    if kw.text != "measure":
        toks.fail(kw, "assigning classical values other than measurements is not supported")
    qubits = p.resolve(toks, _operand(toks), True)
    toks.require(";")
    _record_measures(p, toks, qubits, clbits, at)


def _reset(p, toks):
    toks.take()
    qubits = p.resolve(toks, _operand(toks), True)
    toks.require(";")
    p.out.extend(("reset", q) for q in qubits)


def _barrier(p, toks):
    toks.take()
    qubits = []
    while not toks.at_symbol(";") and not toks.at_end():
        qubits.extend(p.resolve(toks, _operand(toks), True))
        toks.accept(",")
    toks.require(";")
    p.out.append(("barrier", qubits or list(range(p.qubits))))


def _global_phase(p, toks):
    toks.skip_past(";")


def _modifiers(toks: _Tokens) -> list:
    """Leading `inv @`, `pow(e) @`, `ctrl(n) @`, `negctrl(n) @`."""
    mods = []
    while toks.peek().kind == "name" and toks.peek().text in _MODIFIERS:
        mark = toks.at
        tok = toks.take()
        arg = None
        if toks.accept("("):
            arg = _expression(toks)
            toks.require(")")
        if not toks.accept("@"):
            toks.at = mark  # a gate that happens to share the name
            break
        if tok.text == "inv":
            mods.append(("inv",))
        elif tok.text == "pow":
            if arg is None:
                toks.fail(tok, "`pow` needs an exponent")
            mods.append(("pow", arg, tok))
        else:
            count = 1
            if arg is not None:
                x = arg({})
                if x < 1 or x != int(x):
                    toks.fail(tok, "a control count must be a positive integer")
                count = int(x)
            mods.append((tok.text, count))
    return mods


def _application(toks: _Tokens) -> _Application:
    """[modifiers] name [(expr, ...)] operand, ..."""
    mods = _modifiers(toks)
    name = toks.name()
    params = []
    if toks.accept("("):
        if not toks.at_symbol(")"):
            params.append(_expression(toks))
            while toks.accept(","):
                params.append(_expression(toks))
        toks.require(")")
    operands = []
    while not (toks.at_symbol(";") or toks.at_symbol("}") or toks.at_end()):
        operands.append(_operand(toks))
        if not toks.accept(","):
            break
    return _Application(mods, name, params, operands)


def _definition(p, toks):
    toks.take()
    name = toks.name()
    params = []
    if toks.accept("("):
        while not toks.at_symbol(")"):
            params.append(toks.name().text)
            toks.accept(",")
        toks.require(")")
    qubits = []
    while not toks.at_symbol("{"):
        qubits.append(toks.name().text)
        toks.accept(",")
    toks.require("{")
    body = []
    while not toks.at_symbol("}"):
        if toks.at_end():
            toks.fail(name, f"unterminated definition of `{name.text}`")
        if toks.at_name("barrier"):
            toks.skip_past(";")
            continue
        app = _application(toks)
        if any(o.indices is not None for o in app.operands):
            toks.fail(name, f"the body of `{name.text}` can only use its own qubit names")
        body.append(app)
        toks.require(";")
    toks.require("}")
    p.definitions[name.text] = _Definition(params, qubits, body)


def _condition(p, toks) -> tuple:
    """(classical bit, value that takes the `if` branch)."""
    negated = False
    while toks.accept("!"):
        negated = not negated
    reg = toks.name()
    if reg.text not in p.cregs:
        toks.fail(reg, f"unknown classical bit register `{reg.text}` in a condition")
    first, size = p.cregs[reg.text]
    if toks.accept("["):
        index = toks.index()
        toks.require("]")
        if index >= size:
            toks.fail(reg, f"index {index} is out of range for `{reg.text}` of size {size}")
        clbit = first + index
    elif size == 1:
        clbit = first
    else:
        toks.fail(reg, f"a condition on `{reg.text}`, a register of {size} bits, is not supported: only one bit can "
                       f"be tested (`if ({reg.text}[k])`)")
    wanted = True
    if toks.at_symbol("==") or toks.at_symbol("!="):
        equal = toks.take().text == "=="
        v = toks.take()
        if v.kind == "number" and v.number in (0.0, 1.0):
            value = v.number == 1.0
        elif v.kind == "name" and v.text in ("true", "false"):
            value = v.text == "true"
        else:
            toks.fail(v, f"a bit can only be compared with 0, 1, true or false, not {toks.describe(v)}")
        wanted = value == equal
    return clbit, wanted != negated


def _pauli_branch(p, toks, at) -> dict:
    """An `if` body: qubit -> Pauli as X/Z bits (products up to phase)."""
    block = toks.accept("{")
    paulis: dict = {}
    while True:
        if block and toks.accept("}"):
            break
        tok = toks.peek()
        if tok.kind == "end":
            toks.fail(at, "unterminated `if` block")
        if tok.kind != "name":
            toks.fail(tok, f"expected a gate call, found {toks.describe(tok)}")
        if tok.text == "barrier":
            toks.skip_past(";")
        elif tok.text in ("measure", "reset", "if", "gate") or tok.text in _REFUSED:
            toks.fail(tok, f"`{tok.text}` inside `if` is not supported: an `if` body can only apply Pauli gates "
                           "(x, y, z, id)")
        else:
            app = _application(toks)
            toks.require(";")
            mark = len(p.out)
            p.apply(toks, app)
            emitted, p.out[mark:] = p.out[mark:], []
            for ins in emitted:
                if not (ins[0] == "gate" and ins[1].name in ("id", "x", "y", "z")):
                    toks.fail(tok, f"`{app.name.text}` inside `if` is not supported: an `if` body can only apply "
                                   "Pauli gates (x, y, z, id), which run as classical feedback")
                q = ins[2][0]
                paulis[q] = paulis.get(q, 0) ^ _PAULI_BITS.get(ins[1].name, 0)
        if not block:
            break
    return paulis


def _conditional(p, toks):
    """`if (bit) body [else body]` with Pauli bodies: the else-branch's
    Paulis always, then the difference of the branches as feedback on the
    bit (a Pauli applied when the bit reads 1)."""
    at = toks.take()
    toks.require("(")
    clbit, wanted = _condition(p, toks)
    toks.require(")")
    taken = _pauli_branch(p, toks, at)
    other = {}
    if toks.at_name("else"):
        toks.take()
        other = _pauli_branch(p, toks, at)
    on_one, on_zero = (taken, other) if wanted else (other, taken)
    for q, bits in on_zero.items():
        if bits:
            p.out.append(("gate", Gate(_PAULI_LETTER[bits].lower()), [q]))
    for q in sorted(set(on_one) | set(on_zero)):
        flip = on_one.get(q, 0) ^ on_zero.get(q, 0)
        if flip:
            p.out.append(("feedback", _PAULI_LETTER[flip], q, clbit))


_STATEMENTS = {"OPENQASM": _version, "include": _include, "qreg": _register_v2, "creg": _register_v2,
               "qubit": _register_v3, "bit": _register_v3, "gate": _definition, "if": _conditional,
               "measure": _measure_arrow, "reset": _reset, "barrier": _barrier, "gphase": _global_phase}

_prelude = _Program()
_prelude.read(_PRELUDE)


def parse(source: str) -> Circuit:
    """An OpenQASM 2 or 3 program as a circuit; qubits and classical bits
    are numbered in declaration order across registers."""
    p = _Program(_prelude.definitions)
    p.read(source)
    c = Circuit(p.qubits, p.clbits)
    c._instructions.extend(p.out)
    return c
