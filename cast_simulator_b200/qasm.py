"""OpenQASM 2.0 front-end: ``parse_qasm`` and ``to_qasm``.

Accepts the language of the reference's parser (src/openqasm/parser.rs:58-470):

  * an optional ``OPENQASM ...;`` header and ``include ...;`` lines (skipped);
  * at most one ``qreg name[size];`` (qubit operands are then bounds-checked and
    must use that register name); without one, bounds are not checked and the
    circuit width is the largest operand + 1;
  * gate statements ``x y z h s t`` (one qubit), ``cx cz swap`` (two), ``ccx``
    (three), ``rx ry rz`` and ``cp`` with one angle, ``u3`` with three;
  * angle expressions over integers, decimals, ``pi``, ``+ - * / ^``, unary
    minus and parentheses (``^`` binds tighter than unary minus on its right
    operand, as in the reference's grammar);
  * qubit operands ``q[3]``, ``q3`` (trailing digits) or a bare integer;
  * ``//`` line comments.

Anything else raises ``ValueError`` with the offending token.  ``to_qasm``
writes a circuit of named standard gates back (angles with 17 significant
digits, so a round trip reproduces the matrices exactly).
"""
from __future__ import annotations

import math
import re

from .types import QuantumCircuit, QuantumGate

_TOKEN = re.compile(
    r"\s+|//[^\n]*|(?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)|(?P<id>[A-Za-z_][A-Za-z0-9_]*)"
    r"|(?P<sym>[()\[\],;+\-*/^=])|(?P<bad>.)")

_ONE = {"x": QuantumGate.x, "y": QuantumGate.y, "z": QuantumGate.z, "h": QuantumGate.h,
        "s": QuantumGate.s, "t": QuantumGate.t}
_TWO = {"cx": QuantumGate.cx, "cz": QuantumGate.cz, "swap": QuantumGate.swap}
_ROT = {"rx": QuantumGate.rx, "ry": QuantumGate.ry, "rz": QuantumGate.rz}


def _tokenize(text: str):
    out = []
    for m in _TOKEN.finditer(text):
        if m.group("num") is not None:
            s = m.group("num")
            is_int = re.fullmatch(r"\d+", s) is not None
            out.append(("int" if is_int else "float", int(s) if is_int else float(s)))
        elif m.group("id") is not None:
            s = m.group("id")
            out.append(("pi", math.pi) if s == "pi" else ("id", s))
        elif m.group("sym") is not None:
            out.append((m.group("sym"), None))
        elif m.group("bad") is not None:
            out.append(("char", m.group("bad")))  # an error only where a statement needs a token
    out.append(("eof", None))
    return out


def _label(tok) -> str:
    kind, val = tok
    if kind == "id":
        return f"identifier `{val}`"
    if kind in ("int", "float"):
        return f"number `{val}`"
    if kind == "eof":
        return "<end-of-input>"
    if kind == "pi":
        return "`pi`"
    if kind == "char":
        return f"unsupported character `{val}`"
    return f"`{kind}`"


class _Parser:
    def __init__(self, tokens):
        self.t, self.i = tokens, 0
        self.qreg_name: str | None = None
        self.qreg_size: int | None = None

    def peek(self):
        return self.t[self.i]

    def bump(self):
        tok = self.t[self.i]
        if self.i < len(self.t) - 1:
            self.i += 1
        return tok

    def expect(self, kind):
        tok = self.peek()
        if tok[0] != kind:
            raise ValueError(f"expected `{kind}`, found {_label(tok)}")
        return self.bump()

    def skip_statement(self, what):
        while self.peek()[0] != ";":
            if self.peek()[0] == "eof":
                raise ValueError(f"expected `;` to terminate {what}, found end-of-input")
            self.bump()
        self.bump()

    def qreg(self):
        self.bump()
        if self.qreg_size is not None:
            raise ValueError("multiple qreg declarations are not supported")
        name = self.expect("id")[1]
        self.expect("[")
        tok = self.peek()
        if tok[0] != "int":
            raise ValueError(f"expected integer qreg size, found {_label(tok)}")
        self.bump()
        self.expect("]")
        self.expect(";")
        self.qreg_name, self.qreg_size = name, tok[1]

    def check(self, idx: int) -> int:
        if self.qreg_size is not None and idx >= self.qreg_size:
            raise ValueError(f"qubit index `{idx}` is out of bounds for qreg size `{self.qreg_size}`")
        return idx

    def qubit(self) -> int:
        tok = self.peek()
        if tok[0] == "int":
            self.bump()
            return self.check(tok[1])
        if tok[0] == "id":
            name = self.bump()[1]
            if self.peek()[0] == "[":
                self.bump()
                it = self.peek()
                if it[0] != "int":
                    raise ValueError(f"expected integer qubit index, found {_label(it)}")
                self.bump()
                self.expect("]")
                if self.qreg_name is not None and name != self.qreg_name:
                    raise ValueError(f"unknown qreg `{name}`; expected `{self.qreg_name}`")
                return self.check(it[1])
            m = re.search(r"(\d+)$", name)
            if m:
                return self.check(int(m.group(1)))
            raise ValueError(f"expected qubit like `q[0]` or `q0`, found identifier `{name}`")
        raise ValueError(f"expected qubit operand, found {_label(tok)}")

    def angle(self) -> float:
        self.expect("(")
        v = self.expr()
        self.expect(")")
        return v

    # expression grammar: add/sub > mul/div > unary minus > power > primary
    def expr(self) -> float:
        v = self.term()
        while self.peek()[0] in ("+", "-"):
            op = self.bump()[0]
            r = self.term()
            v = v + r if op == "+" else v - r
        return v

    def term(self) -> float:
        v = self.unary()
        while self.peek()[0] in ("*", "/"):
            op = self.bump()[0]
            r = self.unary()
            v = v * r if op == "*" else v / r
        return v

    def unary(self) -> float:
        if self.peek()[0] == "-":
            self.bump()
            return -self.unary()
        return self.power()

    def power(self) -> float:
        base = self.primary()
        if self.peek()[0] == "^":
            self.bump()
            return float(base) ** self.unary()
        return base

    def primary(self) -> float:
        tok = self.peek()
        if tok[0] in ("int", "float", "pi"):
            self.bump()
            return float(tok[1])
        if tok[0] == "(":
            self.bump()
            v = self.expr()
            self.expect(")")
            return v
        raise ValueError(f"expected expression term, found {_label(tok)}")

    def gate(self) -> QuantumGate:
        name = self.expect("id")[1]
        if name in _ONE:
            g = _ONE[name](self.qubit())
        elif name in _TWO:
            a = self.qubit()
            self.expect(",")
            g = _TWO[name](a, self.qubit())
        elif name == "cp":
            th = self.angle()
            a = self.qubit()
            self.expect(",")
            g = QuantumGate.cp(th, a, self.qubit())
        elif name == "ccx":
            a = self.qubit()
            self.expect(",")
            b = self.qubit()
            self.expect(",")
            g = QuantumGate.ccx(a, b, self.qubit())
        elif name in _ROT:
            th = self.angle()
            g = _ROT[name](th, self.qubit())
        elif name == "u3":
            self.expect("(")
            th = self.expr()
            self.expect(",")
            ph = self.expr()
            self.expect(",")
            la = self.expr()
            self.expect(")")
            g = QuantumGate.u3(th, ph, la, self.qubit())
        else:
            raise ValueError(f"unsupported gate `{name}`")
        self.expect(";")
        return g

    def circuit(self) -> QuantumCircuit:
        gates = []
        while self.peek()[0] != "eof":
            tok = self.peek()
            if tok[0] == ";":
                self.bump()
                continue
            if tok[0] == "id" and tok[1].lower() == "openqasm":
                self.bump()
                self.skip_statement("OPENQASM header")
                continue
            if tok[0] == "id" and tok[1].lower() == "include":
                self.bump()
                self.skip_statement("include statement")
                continue
            if tok[0] == "id" and tok[1].lower() == "qreg":
                self.qreg()
                continue
            gates.append(self.gate())
        width = self.qreg_size
        if width is None:
            width = 1 + max((max(g.qubits()) for g in gates), default=-1)
        circ = QuantumCircuit(max(width, 1))
        for g in gates:
            circ.add(g)
        return circ


def parse_qasm(text: str) -> QuantumCircuit:
    """Parse OpenQASM 2.0 text (the reference parser's subset) into a circuit."""
    return _Parser(_tokenize(text)).circuit()


def to_qasm(circuit: QuantumCircuit, qreg: str = "q") -> str:
    """OpenQASM 2.0 text of a circuit of named standard gates."""
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg {qreg}[{circuit.n_qubits()}];"]
    for g in circuit.gates():
        op = g.op()
        if op is None or not g.is_unitary():
            raise ValueError("to_qasm writes named standard gates only")
        name, params, qs = op
        args = ",".join(f"{qreg}[{q}]" for q in qs)
        ps = "(" + ",".join(repr(float(p)) for p in params) + ")" if params else ""
        lines.append(f"{name}{ps} {args};")
    return "\n".join(lines) + "\n"
