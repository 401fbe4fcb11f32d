"""NMODL mechanism files -> channel code for the simulation kernel.

The reference turns a NEURON model's .mod files into CUDA ahead of time:
NEURON's translator writes C, and P/extractModel.py rewrites that into the
per-model AllModels.cu / AllModels.cuh the simulator is rebuilt with.  This
module reads the .mod files itself (no NEURON needed) and emits one device
function with the interface and row layout of the hand-written channel sets
(csrc/channels_ttpc.cuh):

    template <typename R, bool INIT, typename MK>
    NGPU_HD void generated_node(MK mk, R v, R dt, R* st, const float* pr, R& I, R& G)

which the library compiles at run time into the advance kernel
(ngpu_mechset_define, csrc/ngpu_jit.h).

Supported NMODL: NEURON (SUFFIX, USEION ... READ/WRITE, NONSPECIFIC_CURRENT,
RANGE / GLOBAL), PARAMETER, CONSTANT, ASSIGNED, STATE, UNITS (FARADAY, R,
PI), INITIAL, BREAKPOINT with SOLVE ... METHOD cnexp, derivimplicit (equations
linear in their own state: one exact implicit-Euler step) or euler
(DERIVATIVE), or METHOD sparse (KINETIC), DERIVATIVE, KINETIC with first-order reactions
(~ a <-> b (kf, kb)), sources (~ a << (f)) and CONSERVE, SOLVE ...
STEADYSTATE sparse in INITIAL, PROCEDURE, FUNCTION, FUNCTION_TABLE of one
argument (values given to generate()), LOCAL, if / else,
UNITSON / UNITSOFF, TABLE (ignored: rates are computed directly), comments.
VERBATIM, NET_RECEIVE, point processes, higher-order reactions and other
integration methods raise NmodlError.

Semantics, as NEURON's fixed-step method and the reference's simulator
(GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/CudaStuff.cu:227-330):
  * two phases per step: every mechanism's state update (INITIAL at
    initialisation, else its DERIVATIVE block integrated by cnexp), then
    every mechanism's BREAKPOINT currents at the same voltage;
  * cnexp: each x' = f is linear in x, f = a + b x, and x is advanced
    exactly over dt with the other variables frozen:
    x += (1 - exp(b dt)) (-a/b - x); a and b are found symbolically;
  * the membrane conductance is the analytic dI/dv of the BREAKPOINT
    currents (forward-mode derivative through its assignments), which the
    reference approximates by a finite difference (CudaStuff.cu:269);
  * reversal potentials of na and k are constants of the mechanism set;
    eca follows cai by the Nernst equation after the state phase; an ion
    concentration no mechanism at a node writes reads 0, and a written one
    starts at NEURON's default (cai 5e-5 mM) unless INITIAL sets it;
  * an ion current a mechanism READs (CaDynamics' ica) is the node's total
    of that current from the previous step's current phase, kept in an
    extra state row after the mechanism's STATE rows;
  * PROCEDURE / FUNCTION arguments, and v inside them, are local copies;
  * KINETIC: one backward-Euler step of the scheme's linear system (what
    NEURON's sparse method computes for first-order reactions), solved
    exactly by straight-line elimination; the reference's code generator
    instead runs three relaxation sweeps (P/kinetic_template.txt,
    Cubackwards_euler).
Numerics: 1 - exp(E) and exp(E) - 1 are emitted as expm1 with a series
below |E| = 1e-2, so the removable singularities of alpha/beta rates keep
FP32 precision next to the singular voltage; divisions and exponentials
use the kernel's Math<R> (SFU intrinsics in FP32).
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field
from pathlib import Path


class NmodlError(ValueError):
    pass


# ------------------------------------------------------------------ lexer
_TOK = re.compile(r"""
    (?P<nl>\n) |
    (?P<ws>[ \t\r\f]+) |
    (?P<comment>:[^\n]*|\?[^\n]*) |
    (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?) |
    (?P<id>[A-Za-z_][A-Za-z_0-9]*) |
    (?P<op>==|!=|<=|>=|&&|\|\||[-+*/^(){}=<>,'!%~\[\]])
""", re.X)


@dataclass
class Tok:
    kind: str
    val: str
    line: int


def _strip_blocks(text: str) -> str:
    """Remove COMMENT ... ENDCOMMENT and TITLE lines (line numbers kept)."""
    out, in_c = [], False
    for ln in text.split("\n"):
        s = ln.strip()
        if in_c:
            out.append("")
            if s.startswith("ENDCOMMENT"):
                in_c = False
            continue
        if s.startswith("COMMENT"):
            in_c = True
            out.append("")
            continue
        if s.startswith("TITLE"):
            out.append("")
            continue
        out.append(ln)
    return "\n".join(out)


def tokenize(text: str) -> list[Tok]:
    text = _strip_blocks(text)
    toks, pos, line = [], 0, 1
    while pos < len(text):
        m = _TOK.match(text, pos)
        if not m:
            raise NmodlError(f"line {line}: cannot read {text[pos:pos + 20]!r}")
        kind = m.lastgroup
        val = m.group(kind)
        if kind == "nl":
            toks.append(Tok("nl", "\n", line))
            line += 1
        elif kind in ("num", "id", "op"):
            toks.append(Tok(kind, val, line))
        pos = m.end()
    toks.append(Tok("eof", "", line))
    return toks


# -------------------------------------------------------------- expressions
@dataclass(frozen=True)
class Num:
    v: float


@dataclass(frozen=True)
class Var:
    name: str


@dataclass(frozen=True)
class Un:
    op: str
    e: object


@dataclass(frozen=True)
class Bin:
    op: str
    l: object
    r: object


@dataclass(frozen=True)
class Call:
    name: str
    args: tuple


# statements
@dataclass
class Assign:
    name: str
    e: object


@dataclass
class Deriv:
    name: str
    e: object


@dataclass
class If:
    cond: object
    then: list
    other: list


@dataclass
class CallStmt:
    name: str
    args: tuple


@dataclass
class Solve:
    block: str
    method: str | None
    steady: bool = False      # SOLVE ... STEADYSTATE (in INITIAL)


@dataclass
class Reaction:
    """~ a <-> b (kf, kb): first order both ways."""
    a: str
    b: str
    kf: object
    kb: object


@dataclass
class Flux:
    """~ a << (f): a source term of a's equation."""
    a: str
    f: object


@dataclass
class Conserve:
    lhs: object
    rhs: object


_BUILTIN_FUNCS = {"exp", "log", "log10", "fabs", "sqrt", "pow", "sin", "cos", "tanh", "fmin", "fmax"}


class Parser:
    def __init__(self, toks: list[Tok]):
        self.t = toks
        self.i = 0

    # token helpers
    def peek(self, k: int = 0) -> Tok:
        return self.t[self.i + k]

    def next(self) -> Tok:
        tok = self.t[self.i]
        self.i += 1
        return tok

    def skip_nl(self):
        while self.peek().kind == "nl":
            self.i += 1

    def expect(self, val: str) -> Tok:
        self.skip_nl()
        tok = self.next()
        if tok.val != val:
            raise NmodlError(f"line {tok.line}: expected {val!r}, found {tok.val!r}")
        return tok

    def ident(self) -> str:
        self.skip_nl()
        tok = self.next()
        if tok.kind != "id":
            raise NmodlError(f"line {tok.line}: expected a name, found {tok.val!r}")
        return tok.val

    def skip_units(self):
        """A parenthesised unit annotation, e.g. (mV) or (/ms) or (1/liter)."""
        if self.peek().val == "(":
            depth = 0
            while True:
                tok = self.next()
                if tok.val == "(":
                    depth += 1
                elif tok.val == ")":
                    depth -= 1
                    if depth == 0:
                        return
                elif tok.kind == "eof":
                    raise NmodlError("unterminated unit")

    def skip_block(self):
        self.expect("{")
        depth = 1
        while depth:
            tok = self.next()
            if tok.val == "{":
                depth += 1
            elif tok.val == "}":
                depth -= 1
            elif tok.kind == "eof":
                raise NmodlError("unterminated block")

    # expressions (NMODL precedence: || < && < comparison < +- < */% < unary < ^)
    def expr(self):
        return self.or_()

    def or_(self):
        e = self.and_()
        while self.peek().val == "||":
            self.next()
            e = Bin("||", e, self.and_())
        return e

    def and_(self):
        e = self.cmp()
        while self.peek().val == "&&":
            self.next()
            e = Bin("&&", e, self.cmp())
        return e

    def cmp(self):
        e = self.add()
        while self.peek().val in ("<", ">", "<=", ">=", "==", "!="):
            op = self.next().val
            e = Bin(op, e, self.add())
        return e

    def add(self):
        e = self.mul()
        while self.peek().val in ("+", "-"):
            op = self.next().val
            e = Bin(op, e, self.mul())
        return e

    def mul(self):
        e = self.unary()
        while self.peek().val in ("*", "/", "%"):
            op = self.next().val
            e = Bin(op, e, self.unary())
        return e

    def unary(self):
        if self.peek().val == "-":
            self.next()
            return Un("-", self.unary())
        if self.peek().val == "+":
            self.next()
            return self.unary()
        if self.peek().val == "!":
            self.next()
            return Un("!", self.unary())
        return self.power()

    def power(self):
        base = self.primary()
        if self.peek().val == "^":
            self.next()
            return Bin("^", base, self.unary())  # right associative, binds the unary minus
        return base

    def primary(self):
        tok = self.next()
        if tok.kind == "num":
            self.skip_units() if self.peek().val == "(" else None
            return Num(float(tok.val))
        if tok.kind == "id":
            if self.peek().val == "(":
                self.next()
                args = []
                if self.peek().val != ")":
                    args.append(self.expr())
                    while self.peek().val == ",":
                        self.next()
                        args.append(self.expr())
                self.expect(")")
                return Call(tok.val, tuple(args))
            return Var(tok.val)
        if tok.val == "(":
            e = self.expr()
            self.expect(")")
            return e
        raise NmodlError(f"line {tok.line}: unexpected {tok.val!r} in an expression")

    # statements
    def stmts(self) -> list:
        self.expect("{")
        out = []
        while True:
            self.skip_nl()
            tok = self.peek()
            if tok.val == "}":
                self.next()
                return out
            if tok.kind == "eof":
                raise NmodlError("unterminated block")
            s = self.stmt()
            if s is not None:
                out.append(s)

    def stmt(self):
        tok = self.next()
        v = tok.val
        if v in ("UNITSON", "UNITSOFF"):
            return None
        if v == "LOCAL":
            self.ident()
            while self.peek().val == ",":
                self.next()
                self.ident()
            return ("local",)
        if v == "TABLE":  # TABLE list [DEPEND list] FROM a TO b WITH n: computed directly instead
            while self.peek().val != "WITH":
                if self.peek().kind == "eof":
                    raise NmodlError("unterminated TABLE")
                self.next()
            self.next()
            self.next()
            return None
        if v == "SOLVE":
            block = self.ident()
            method, steady = None, False
            if self.peek().val in ("METHOD", "STEADYSTATE"):
                steady = self.next().val == "STEADYSTATE"
                method = self.ident()
            return Solve(block, method, steady)
        if v == "~":
            return self.reaction(tok.line)
        if v == "CONSERVE":
            lhs = self.expr()
            self.expect("=")
            return Conserve(lhs, self.expr())
        if v == "if":
            self.expect("(")
            cond = self.expr()
            self.expect(")")
            then = self.stmts()
            other = []
            save = self.i
            self.skip_nl()
            if self.peek().val == "else":
                self.next()
                self.skip_nl()
                if self.peek().val == "if":
                    other = [self.stmt()]
                else:
                    other = self.stmts()
            else:
                self.i = save
            return If(cond, then, other)
        if v in ("VERBATIM", "KINETIC", "NET_RECEIVE", "LINEAR", "NONLINEAR", "COMPARTMENT",
                 "FROM", "WHILE", "FOR_NETCONS"):
            raise NmodlError(f"line {tok.line}: {v} is not supported")
        if tok.kind == "id":
            if self.peek().val == "'":
                self.next()
                self.expect("=")
                return Deriv(v, self.expr())
            if self.peek().val == "=":
                self.next()
                return Assign(v, self.expr())
            if self.peek().val == "(":
                self.next()
                args = []
                if self.peek().val != ")":
                    args.append(self.expr())
                    while self.peek().val == ",":
                        self.next()
                        args.append(self.expr())
                self.expect(")")
                return CallStmt(v, tuple(args))
        raise NmodlError(f"line {tok.line}: cannot read statement at {v!r}")

    def species(self, line: int) -> str:
        """One side of a reaction: a single STATE with stoichiometry 1."""
        names = []
        while True:
            if self.peek().kind == "num":
                raise NmodlError(f"line {line}: stoichiometric coefficients are not supported (first-order "
                                 "reactions only)")
            names.append(self.ident())
            if self.peek().val == "[":
                raise NmodlError(f"line {line}: array states are not supported")
            if self.peek().val != "+":
                break
            self.next()
        if len(names) != 1:
            raise NmodlError(f"line {line}: {' + '.join(names)}: first-order reactions only")
        return names[0]

    def reaction(self, line: int):
        a = self.species(line)
        t = self.next()
        if t.val == "<" and self.peek().val == "-" and self.peek(1).val == ">":
            self.next()
            self.next()
            b = self.species(line)
            self.expect("(")
            kf = self.expr()
            self.expect(",")
            kb = self.expr()
            self.expect(")")
            return Reaction(a, b, kf, kb)
        if t.val == "<" and self.peek().val == "<":
            self.next()
            self.expect("(")
            f = self.expr()
            self.expect(")")
            return Flux(a, f)
        raise NmodlError(f"line {line}: expected <-> or << after ~ {a}")


# ---------------------------------------------------------------- mechanism
@dataclass
class UseIon:
    ion: str
    read: list
    write: list


@dataclass
class Mechanism:
    suffix: str
    useions: list = field(default_factory=list)
    nonspecific: list = field(default_factory=list)
    parameters: list = field(default_factory=list)   # (name, default or None), in declaration order
    assigned: list = field(default_factory=list)
    states: list = field(default_factory=list)
    unit_consts: dict = field(default_factory=dict)
    breakpoint: list = field(default_factory=list)
    derivatives: dict = field(default_factory=dict)
    kinetics: dict = field(default_factory=dict)      # KINETIC blocks: name -> stmts
    initial: list = field(default_factory=list)
    procedures: dict = field(default_factory=dict)    # name -> (args, stmts)
    functions: dict = field(default_factory=dict)
    tables: dict = field(default_factory=dict)        # FUNCTION_TABLE name -> argument names
    table_data: dict = field(default_factory=dict)    # name -> (xs, ys), given to generate()

    def ion_names(self) -> set:
        out = set()
        for u in self.useions:
            out |= set(u.read) | set(u.write)
        return out

    def writes(self, name: str) -> bool:
        return any(name in u.write for u in self.useions)

    def reads(self, name: str) -> bool:
        return any(name in u.read for u in self.useions)

    def currents(self) -> list:
        """Membrane currents the mechanism contributes (written ion currents, nonspecific)."""
        out = []
        for u in self.useions:
            out += [w for w in u.write if w == "i" + u.ion]
        return out + list(self.nonspecific)


_UNIT_CONSTS = {"faraday": 96485.309, "k-mole": 8.3134, "pi": math.pi}


def _parse_decls(p: Parser, with_values: bool) -> list:
    """PARAMETER / ASSIGNED / STATE / CONSTANT bodies: name [= value] [(units)] [<lo, hi>] [FROM a TO b]."""
    p.expect("{")
    out = []
    while True:
        p.skip_nl()
        tok = p.peek()
        if tok.val == "}":
            p.next()
            return out
        name = p.ident()
        val = None
        if p.peek().val == "=":
            p.next()
            neg = False
            if p.peek().val == "-":
                p.next()
                neg = True
            nt = p.next()
            if nt.kind != "num":
                raise NmodlError(f"line {nt.line}: expected a number for {name}")
            val = -float(nt.val) if neg else float(nt.val)
        p.skip_units()
        if p.peek().val == "<":
            while p.next().val != ">":
                pass
        if p.peek().val == "FROM":
            p.next()
            p.expr()
            p.expect("TO")
            p.expr()
        out.append((name, val))


def parse_mod(text: str, name_hint: str = "") -> Mechanism:
    p = Parser(tokenize(text))
    mech = Mechanism(suffix=name_hint)
    while True:
        p.skip_nl()
        tok = p.next()
        if tok.kind == "eof":
            break
        v = tok.val
        if v in ("UNITSON", "UNITSOFF", "THREADSAFE"):
            continue
        if v == "LOCAL":
            p.ident()
            while p.peek().val == ",":
                p.next()
                p.ident()
            continue
        if v == "NEURON":
            p.expect("{")
            while True:
                p.skip_nl()
                t = p.next()
                if t.val == "}":
                    break
                if t.val == "SUFFIX":
                    mech.suffix = p.ident()
                elif t.val == "USEION":
                    u = UseIon(p.ident(), [], [])
                    cur = None
                    while p.peek().kind != "nl" and p.peek().val != "}":
                        w = p.next()
                        if w.val in ("READ", "WRITE"):
                            cur = u.read if w.val == "READ" else u.write
                        elif w.val == "VALENCE":
                            neg = p.peek().val == "-"
                            if neg:
                                p.next()
                            p.next()
                        elif w.val == ",":
                            continue
                        elif w.kind == "id" and cur is not None:
                            cur.append(w.val)
                    mech.useions.append(u)
                elif t.val == "NONSPECIFIC_CURRENT":
                    mech.nonspecific.append(p.ident())
                    while p.peek().val == ",":
                        p.next()
                        mech.nonspecific.append(p.ident())
                elif t.val in ("RANGE", "GLOBAL", "POINTER", "BBCOREPOINTER"):
                    p.ident()
                    while p.peek().val == ",":
                        p.next()
                        p.ident()
                elif t.val in ("POINT_PROCESS", "ARTIFICIAL_CELL", "ELECTRODE_CURRENT"):
                    raise NmodlError(f"{t.val} is not supported (density mechanisms only)")
                elif t.val == "THREADSAFE":
                    continue
                else:
                    raise NmodlError(f"line {t.line}: unknown NEURON statement {t.val!r}")
        elif v == "UNITS":
            p.expect("{")
            while True:
                p.skip_nl()
                t = p.next()
                if t.val == "}":
                    break
                if t.kind == "id" and p.peek().val == "=":
                    p.next()
                    p.skip_nl()
                    if p.peek().val == "(":
                        first = p.t[p.i + 1].val
                        p.skip_units()
                        p.skip_units()
                        if first.lower() in _UNIT_CONSTS:
                            mech.unit_consts[t.val] = _UNIT_CONSTS[first.lower()]
                elif t.val == "(":
                    p.i -= 1
                    p.skip_units()
                    p.expect("=")
                    p.skip_nl()
                    p.skip_units()
        elif v == "PARAMETER":
            mech.parameters += _parse_decls(p, True)
        elif v == "CONSTANT":
            for n, val in _parse_decls(p, True):
                mech.unit_consts[n] = val
        elif v == "ASSIGNED":
            mech.assigned += [n for n, _ in _parse_decls(p, False)]
        elif v == "STATE":
            mech.states += [n for n, _ in _parse_decls(p, False)]
        elif v == "INDEPENDENT":
            p.skip_block()
        elif v == "BREAKPOINT":
            mech.breakpoint = p.stmts()
        elif v == "INITIAL":
            mech.initial = p.stmts()
        elif v == "DERIVATIVE":
            dname = p.ident()
            mech.derivatives[dname] = p.stmts()
        elif v == "KINETIC":
            kname = p.ident()
            mech.kinetics[kname] = p.stmts()
        elif v in ("PROCEDURE", "FUNCTION"):
            name = p.ident()
            p.expect("(")
            args = []
            while p.peek().val != ")":
                args.append(p.ident())
                p.skip_units()
                if p.peek().val == ",":
                    p.next()
            p.expect(")")
            p.skip_units()
            body = p.stmts()
            (mech.procedures if v == "PROCEDURE" else mech.functions)[name] = (args, body)
        elif v == "FUNCTION_TABLE":
            name = p.ident()
            p.expect("(")
            args = []
            while p.peek().val != ")":
                args.append(p.ident())
                p.skip_units()
                if p.peek().val == ",":
                    p.next()
            p.expect(")")
            p.skip_units()
            if len(args) != 1:
                raise NmodlError(f"line {tok.line}: FUNCTION_TABLE {name}: one argument only")
            mech.tables[name] = args
        elif v in ("NET_RECEIVE", "VERBATIM", "LINEAR", "NONLINEAR", "DISCRETE", "PARTIAL"):
            raise NmodlError(f"line {tok.line}: {v} blocks are not supported")
        else:
            raise NmodlError(f"line {tok.line}: unexpected {v!r} at top level")
    if not mech.suffix:
        raise NmodlError("no SUFFIX")
    return mech


# NEURON's built-in passive mechanism (i = g (v - e)), stated in NMODL
PAS_MOD = """
NEURON { SUFFIX pas NONSPECIFIC_CURRENT i RANGE g, e }
PARAMETER { g = 0.001 (S/cm2) e = -70 (mV) }
ASSIGNED { v (mV) i (mA/cm2) }
BREAKPOINT { i = g*(v - e) }
"""


# ------------------------------------------------------- symbolic algebra
def _var_order(e) -> list:
    """Names in an expression, left to right, first appearance."""
    out = []

    def walk(x):
        if isinstance(x, Var):
            if x.name not in out:
                out.append(x.name)
        elif isinstance(x, Un):
            walk(x.e)
        elif isinstance(x, Bin):
            walk(x.l)
            walk(x.r)
        elif isinstance(x, Call):
            for a in x.args:
                walk(a)
    walk(e)
    return out


def free_vars(e) -> set:
    if isinstance(e, Var):
        return {e.name}
    if isinstance(e, Num):
        return set()
    if isinstance(e, Un):
        return free_vars(e.e)
    if isinstance(e, Bin):
        return free_vars(e.l) | free_vars(e.r)
    if isinstance(e, Call):
        out = set()
        for a in e.args:
            out |= free_vars(a)
        return out
    raise TypeError(e)


def subst(e, name, val):
    if isinstance(e, Var):
        return val if e.name == name else e
    if isinstance(e, Num):
        return e
    if isinstance(e, Un):
        return Un(e.op, subst(e.e, name, val))
    if isinstance(e, Bin):
        return Bin(e.op, subst(e.l, name, val), subst(e.r, name, val))
    if isinstance(e, Call):
        return Call(e.name, tuple(subst(a, name, val) for a in e.args))
    raise TypeError(e)


def simplify(e):
    if isinstance(e, (Num, Var)):
        return e
    if isinstance(e, Un):
        x = simplify(e.e)
        if e.op == "-" and isinstance(x, Num):
            return Num(-x.v)
        if e.op == "-" and isinstance(x, Un) and x.op == "-":
            return x.e
        return Un(e.op, x)
    if isinstance(e, Call):
        args = tuple(simplify(a) for a in e.args)
        if all(isinstance(a, Num) for a in args) and e.name in ("exp", "log", "fabs", "sqrt", "pow"):
            f = {"exp": math.exp, "log": math.log, "fabs": abs, "sqrt": math.sqrt, "pow": math.pow}[e.name]
            return Num(f(*[a.v for a in args]))
        return Call(e.name, args)
    if isinstance(e, Bin):
        l, r = simplify(e.l), simplify(e.r)
        if isinstance(l, Num) and isinstance(r, Num) and e.op in "+-*/^":
            a, b = l.v, r.v
            ops = {"+": lambda: a + b, "-": lambda: a - b, "*": lambda: a * b, "/": lambda: a / b,
                   "^": lambda: a ** b}
            try:
                return Num(float(ops[e.op]()))
            except (ZeroDivisionError, OverflowError, TypeError):
                return Bin(e.op, l, r)
        if e.op == "+":
            if isinstance(l, Num) and l.v == 0:
                return r
            if isinstance(r, Num) and r.v == 0:
                return l
        if e.op == "-":
            if isinstance(r, Num) and r.v == 0:
                return l
            if isinstance(l, Num) and l.v == 0:
                return simplify(Un("-", r))
        if e.op == "*":
            if (isinstance(l, Num) and l.v == 0) or (isinstance(r, Num) and r.v == 0):
                return Num(0.0)
            if isinstance(l, Num) and l.v == 1:
                return r
            if isinstance(r, Num) and r.v == 1:
                return l
        if e.op == "/":
            if isinstance(l, Num) and l.v == 0:
                return Num(0.0)
            if isinstance(r, Num) and r.v == 1:
                return l
            if isinstance(r, Bin) and r.op == "/" and isinstance(r.l, Num) and r.l.v == 1:
                return simplify(Bin("*", l, r.r))          # a / (1/x) = a x
            if isinstance(r, Un) and r.op == "-":
                return simplify(Un("-", Bin("/", l, r.e)))
        return Bin(e.op, l, r)
    raise TypeError(e)


def recip(e):
    """1/e, written without a division where e is a quotient."""
    e = simplify(e)
    if isinstance(e, Num):
        return Num(1.0 / e.v)
    if isinstance(e, Bin) and e.op == "/":
        if isinstance(e.l, Num) and e.l.v == 1:
            return e.r
        return simplify(Bin("/", e.r, e.l))
    if isinstance(e, Un) and e.op == "-":
        return simplify(Un("-", recip(e.e)))
    return Bin("/", Num(1.0), e)


def diff(e, x: str, known: dict | None = None):
    """d e / d x; `known` maps names to their derivatives (default: 0)."""
    known = known or {}
    if isinstance(e, Num):
        return Num(0.0)
    if isinstance(e, Var):
        if e.name == x:
            return Num(1.0)
        return known.get(e.name, Num(0.0))
    if isinstance(e, Un):
        if e.op == "-":
            return Un("-", diff(e.e, x, known))
        return Num(0.0)
    if isinstance(e, Bin):
        dl, dr = diff(e.l, x, known), diff(e.r, x, known)
        if e.op == "+":
            return Bin("+", dl, dr)
        if e.op == "-":
            return Bin("-", dl, dr)
        zl = isinstance(simplify(dl), Num) and simplify(dl).v == 0
        zr = isinstance(simplify(dr), Num) and simplify(dr).v == 0
        if e.op == "*":
            if zr:
                return Bin("*", dl, e.r)
            if zl:
                return Bin("*", e.l, dr)
            return Bin("+", Bin("*", dl, e.r), Bin("*", e.l, dr))
        if e.op == "/":
            if zr:
                return Bin("/", dl, e.r)
            return Bin("/", Bin("-", Bin("*", dl, e.r), Bin("*", e.l, dr)), Bin("*", e.r, e.r))
        if e.op == "^":
            if isinstance(simplify(dr), Num) and simplify(dr).v == 0:
                return Bin("*", Bin("*", e.r, Bin("^", e.l, Bin("-", e.r, Num(1.0)))), dl)
            return Bin("*", e, Bin("+", Bin("*", dr, Call("log", (e.l,))), Bin("/", Bin("*", e.r, dl), e.l)))
        return Num(0.0)  # comparisons / logic
    if isinstance(e, Call):
        if len(e.args) == 1:
            a = e.args[0]
            da = diff(a, x, known)
            if e.name == "exp":
                return Bin("*", e, da)
            if e.name == "log":
                return Bin("/", da, a)
            if e.name == "sqrt":
                return Bin("/", da, Bin("*", Num(2.0), e))
            if e.name == "fabs":
                return Bin("*", Call("sgn", (a,)), da)
        if e.name == "pow":
            return diff(Bin("^", e.args[0], e.args[1]), x, known)
        if all(isinstance(simplify(diff(a, x, known)), Num) and simplify(diff(a, x, known)).v == 0
               for a in e.args):
            return Num(0.0)
        raise NmodlError(f"cannot differentiate {e.name}() with respect to {x}")
    raise TypeError(e)


def linear_form(f, x: str):
    """f = a + b x with a, b free of x: returns (a, b) or raises."""
    b = simplify(diff(f, x))
    if x in free_vars(b):
        raise NmodlError(f"{x}' is not linear in {x}: cnexp needs a linear equation")
    a = simplify(subst(f, x, Num(0.0)))
    return a, b


# ---------------------------------------------------------- code emission
def _lit(x: float) -> str:
    if x == int(x) and abs(x) < 1e15:
        return f"(R){int(x)}.0" if x >= 0 else f"(R)({int(x)}.0)"
    return f"(R)({x!r})"


def _is_one(e) -> bool:
    return isinstance(e, Num) and e.v == 1.0


def _expm1_arg(e):
    """E if e is exp(E) - 1, -(...) forms handled by the caller."""
    if isinstance(e, Bin) and e.op == "-" and isinstance(e.l, Call) and e.l.name == "exp" and _is_one(e.r):
        return e.l.args[0], 1.0
    if isinstance(e, Bin) and e.op == "-" and _is_one(e.l) and isinstance(e.r, Call) and e.r.name == "exp":
        return e.r.args[0], -1.0
    return None


class Emitter:
    """C++ text of expressions in an environment name -> C++ expression;
    names in `consts` are compile-time numbers, folded before emission."""

    def __init__(self, env: dict, funcs: dict, consts: dict | None = None):
        self.env = env
        self.funcs = funcs  # user FUNCTION names -> C++ callable
        self.consts = consts or {}

    def e(self, x) -> str:
        for n, val in self.consts.items():
            if self.env.get(n, "").startswith("(R)") or n == "celsius":
                x = subst(x, n, Num(val))
        x = simplify(x)
        if isinstance(x, Num):
            return _lit(x.v)
        if isinstance(x, Var):
            if x.name not in self.env:
                raise NmodlError(f"unknown name {x.name!r}")
            return self.env[x.name]
        if isinstance(x, Un):
            return f"(-{self.e(x.e)})" if x.op == "-" else f"(!{self.e(x.e)})"
        if isinstance(x, Call):
            args = [self.e(a) for a in x.args]
            n = x.name
            if n in self.funcs:
                return f"{self.funcs[n]}({', '.join(args)})"
            table = {"exp": "M::ex", "log": "M::lg", "fabs": "fabs", "sqrt": "sqrt", "pow": "M::pw",
                     "sin": "sin", "cos": "cos", "tanh": "tanh", "fmin": "fmin", "fmax": "fmax",
                     "sgn": "ngpu_sgn", "log10": "(R)0.4342944819032518 * M::lg"}
            if n not in table:
                raise NmodlError(f"unknown function {n}()")
            return f"{table[n]}({', '.join(args)})"
        if isinstance(x, Bin):
            m1 = _expm1_arg(x)
            if m1 is not None:
                arg, sign = m1
                return f"(M::em1({self.e(arg)}))" if sign > 0 else f"(-M::em1({self.e(arg)}))"
            if x.op == "^":
                if isinstance(x.r, Num) and x.r.v in (2.0, 3.0, 4.0):
                    b = self.e(x.l)
                    return "(" + " * ".join([b] * int(x.r.v)) + ")"
                return f"M::pw({self.e(x.l)}, {self.e(x.r)})"
            if x.op == "/":
                if isinstance(x.r, Num) and x.r.v != 0:
                    return f"({self.e(x.l)} * {_lit(1.0 / x.r.v)})"
                return f"M::dv({self.e(x.l)}, {self.e(x.r)})"
            if x.op == "%":
                return f"fmod({self.e(x.l)}, {self.e(x.r)})"
            return f"({self.e(x.l)} {x.op} {self.e(x.r)})"
        raise TypeError(x)


@dataclass
class GeneratedMechSet:
    """A mechanism set generated from .mod files: the same description the
    hand-written sets have in mechsets.py, plus its device source."""
    name: str
    mechs: tuple
    params: tuple
    mech_params: tuple
    state_rows: tuple
    param_defaults: tuple
    celsius: float
    source: str
    cost: tuple
    id: int = -1

    @property
    def n_mech(self) -> int:
        return len(self.mechs)

    @property
    def n_params(self) -> int:
        return len(self.params)

    def mech_index(self, name: str) -> int:
        return self.mechs.index(name)

    def param_index(self, name: str) -> int:
        return self.params.index(name)

    def register(self) -> "GeneratedMechSet":
        """Define the set in libngpu (ngpu_mechset_define); sets self.id, after
        which CellModels of this set run like those of the built-in sets."""
        import ctypes as C

        import numpy as np

        from . import _ffi
        if self.id >= 0:
            return self
        sr = np.array(self.state_rows, dtype=np.int32)
        npm = np.array([len(x) for x in self.mech_params], dtype=np.int32)
        idx = np.array([i for x in self.mech_params for i in x] or [0], dtype=np.int32)
        cost = np.array(self.cost, dtype=np.int32)
        out = C.c_int32()
        L = _ffi.lib()
        _ffi.check("ngpu_mechset_define", L.ngpu_mechset_define(
            self.name.encode(), self.source.encode(), self.n_mech, _ffi.ptr(sr), _ffi.ptr(npm), _ffi.ptr(idx),
            self.n_params, _ffi.ptr(cost), C.byref(out)))
        self.id = out.value
        return self


_ION_DEFAULT_CONC = {"ca": 5e-5, "na": 10.0, "k": 54.4}


def _mech_order_key(name: str) -> str:
    return name.lower()


def generate(mods: dict, name: str = "generated", celsius: float = 34.0, reversal: dict | None = None,
             cao: float = 2.0, constants: dict | None = None, tables: dict | None = None) -> GeneratedMechSet:
    """mods: suffix or file name -> .mod text (NEURON's pas is added unless
    given).  reversal: fixed reversal potentials of ions whose concentrations
    no mechanism writes (e.g. {"na": 50, "k": -85}).  constants: per
    mechanism, PARAMETERs to compile in as constants instead of taking a
    parameter row ({"na": {"vshift": -5}}).  tables: per mechanism, the values
    of its FUNCTION_TABLEs, which NEURON fills from hoc: {"kt": {"tau": (xs,
    ys)}}, xs strictly increasing; read by linear interpolation, the end
    values outside [xs[0], xs[-1]].  Mechanisms are ordered as the reference
    orders them (case-insensitive name order)."""
    reversal = dict(reversal or {})
    constants = constants or {}
    tables = tables or {}
    parsed = {}
    for key, text in mods.items():
        m = parse_mod(text, key)
        parsed[m.suffix] = m
    for m in parsed.values():
        for tname in m.tables:
            data = tables.get(m.suffix, {}).get(tname)
            if data is None:
                raise NmodlError(f"{m.suffix}: FUNCTION_TABLE {tname} needs its values "
                                 f"(tables={{'{m.suffix}': {{'{tname}': (xs, ys)}}}})")
            xs = [float(x) for x in data[0]]
            ys = [float(y) for y in data[1]]
            if len(xs) < 2 or len(xs) != len(ys) or any(not math.isfinite(x) for x in xs + ys) or \
                    any(b <= a for a, b in zip(xs, xs[1:])):
                raise NmodlError(f"{m.suffix}: FUNCTION_TABLE {tname}: xs strictly increasing, xs and ys "
                                 "finite, of one length >= 2")
            m.table_data[tname] = (xs, ys)
    if "pas" not in parsed:
        parsed["pas"] = parse_mod(PAS_MOD)
    order = sorted(parsed, key=_mech_order_key)
    mechs = [parsed[k] for k in order]
    ktf = 1000.0 * 8.3134 * (celsius + 273.15) / 96485.309

    # ion bookkeeping over the set
    conc_written = {}     # "cai" -> True if some mechanism writes it
    for m in mechs:
        for u in m.useions:
            for w in u.write:
                if w.endswith("i") and w[:-1] == u.ion:
                    conc_written[w] = True
    params, mech_params, defaults, state_rows, cost = [], [], [], [], []
    for m in mechs:
        ions = m.ion_names()
        skip = {"v", "celsius", "dt", "t"} | ions | set(constants.get(m.suffix, {}))
        mine = []
        for pn, pv in m.parameters:
            if pn in skip:
                continue
            mine.append(len(params))
            params.append(f"{pn}_{m.suffix}")
            defaults.append(0.0 if pv is None else pv)
        mech_params.append(tuple(mine))
        extra = [u for u in m.useions for r in u.read if r == "i" + u.ion]
        alias = _conc_alias(m)
        extra_conc = [w for u in m.useions for w in u.write
                      if w == u.ion + "i" and w not in m.states and w not in alias]
        state_rows.append(len(m.states) + len(extra) + len(extra_conc))
        cost.append(4 + 20 * len(m.states) + 2 * len(mine))
    src = _emit_set(mechs, mech_params, params, celsius, ktf, reversal, cao, constants, conc_written)
    return GeneratedMechSet(name=name, mechs=tuple(order), params=tuple(params), mech_params=tuple(mech_params),
                            state_rows=tuple(state_rows), param_defaults=tuple(defaults), celsius=celsius,
                            source=src, cost=tuple(cost))


def _rate_vars(m: Mechanism) -> set:
    """Time constants T of equations x' = (X - x)/T that are assigned
    variables: their reciprocal (the rate) is emitted wherever T is assigned,
    so the integration needs no division."""
    out = set()
    for blk in m.derivatives.values():
        for s in blk:
            if isinstance(s, Deriv):
                e = simplify(s.e)
                if (isinstance(e, Bin) and e.op == "/" and isinstance(e.r, Var) and isinstance(e.l, Bin)
                        and e.l.op == "-" and isinstance(e.l.r, Var) and e.l.r.name == s.name):
                    if e.r.name in m.assigned:
                        out.add(e.r.name)
    return out


def _conc_alias(m: Mechanism) -> dict:
    """Ion concentrations the mechanism sets to one of its STATEs (cai = ca)."""
    out = {}
    for blk in list(m.derivatives.values()) + [m.initial]:
        for s in blk:
            if isinstance(s, Assign) and isinstance(s.e, Var) and s.e.name in m.states and m.writes(s.name):
                out[s.name] = s.e.name
    return out


def _emit_set(mechs, mech_params, params, celsius, ktf, reversal, cao, constants, conc_written) -> str:
    L = []
    w = L.append
    w("// Generated by neurogpu_b200/nmodl.py from NMODL mechanism files; do not edit.")
    w("#pragma once")
    w('#include "ngpu_math.cuh"')
    w('#include "param_fold.cuh"')
    w("namespace ngpu {")
    w("template <typename R> NGPU_HD R ngpu_sgn(R x) { return x > (R)0 ? (R)1 : (x < (R)0 ? (R)-1 : (R)0); }")
    w("// cnexp over dt with the gate's rate 1/tau: x + (1 - exp(-dt rate)) (xinf - x)")
    w("template <typename R> NGPU_HD R gen_cnexp_rate(R x, R xinf, R rate, R dt) {")
    w("    return x + Math<R>::one_minus_exp_neg(dt * rate) * (xinf - x);")
    w("}")
    w("template <typename R, bool INIT, typename MK>")
    w("NGPU_HD void generated_node(MK mk, R v, R dt, R* __restrict__ st, const float* __restrict__ pr, R& I,")
    w("                            R& G) {")
    w("    using M = Math<R>;")
    w("    constexpr int S = 32;")
    w(f"    const R celsius = {_lit(celsius)};")
    ions = sorted({u.ion for m in mechs for u in m.useions})
    for ion in ions:
        c = ion + "i"
        w(f"    R ion_{c} = 0;  // read as 0 where no mechanism at the node writes it")
    w(f"    R Itot = 0, Gtot = 0;")
    # per-mechanism variable declarations
    envs, consts_of = [], []
    for k, m in enumerate(mechs):
        pre = f"m{k}_"
        env = {"v": "v", "dt": "dt", "celsius": "celsius"}
        env.update({n: _lit(val) for n, val in m.unit_consts.items()})
        decl = []
        for s in m.states:
            env[s] = pre + s
            decl.append(pre + s)
        for a in m.assigned:
            if a not in env and a not in m.ion_names() and a != "v" and a != "celsius":
                env[a] = pre + a
                decl.append(pre + a)
        for pn, pv in m.parameters:
            if pn in ("v", "celsius", "dt", "t") or pn in m.ion_names():
                continue
            if pn in constants.get(m.suffix, {}):
                env[pn] = _lit(float(constants[m.suffix][pn]))
            elif pn not in env:
                env[pn] = pre + pn
                decl.append(pre + pn)
        for nm in m.nonspecific:
            if nm not in env:
                env[nm] = pre + nm
                decl.append(pre + nm)
        for u in m.useions:
            for r in u.read + u.write:
                if r == "i" + u.ion:
                    env[r] = pre + r          # this mechanism's own current (or, read, the node total)
                    decl.append(pre + r)
                elif r == u.ion + "i":
                    env[r] = f"ion_{r}"
                elif r == u.ion + "o":
                    env[r] = _lit(cao) if u.ion == "ca" else _lit(_ION_DEFAULT_CONC.get(u.ion, 0.0))
                elif r == "e" + u.ion:
                    env[r] = f"ion_e{u.ion}"
        for t in sorted(_rate_vars(m)):
            if t in env and env[t].startswith(pre):
                env[t + "@rate"] = env[t] + "_rate"
                decl.append(env[t] + "_rate")
        if decl:
            w(f"    R {', '.join(dict.fromkeys(decl))};")
        envs.append(env)
        cst = {"celsius": celsius}
        cst.update(m.unit_consts)
        cst.update({n: float(val) for n, val in constants.get(m.suffix, {}).items()})
        consts_of.append(cst)
    # ---- load
    w("    {")
    w("        int s = 0, q = 0;")
    for k, m in enumerate(mechs):
        env = envs[k]
        alias = _conc_alias(m)
        w(f"        if (mk & {1 << k}u) {{  // {m.suffix}")
        for j, s in enumerate(m.states):
            w(f"            if (!INIT) {env[s]} = st[(s + {j}) * S];")
        n = len(m.states)
        for u in m.useions:
            for r in u.read:
                if r == "i" + u.ion:
                    w(f"            if (!INIT) {env[r]} = st[(s + {n}) * S];  // previous step's node total")
                    n += 1
        for u in m.useions:
            for wr in u.write:
                if wr == u.ion + "i":
                    if wr in m.states:
                        w(f"            if (!INIT) ion_{wr} = {env[wr]};")
                    elif wr in alias:
                        w(f"            if (!INIT) ion_{wr} = {env[alias[wr]]};")
                    else:
                        w(f"            if (!INIT) ion_{wr} = st[(s + {n}) * S];")
                        n += 1
        w(f"            s += {n};")
        for j, pi in enumerate(mech_params[k]):
            pn = params[pi][: -(len(m.suffix) + 1)]
            w(f"            {env[pn]} = pload<R, {pi}>(pr, q + {j});  // a constant where folded")
        w(f"            q += {len(mech_params[k])};")
        w("        }")
    w("    }")
    # ---- state phase
    for k, m in enumerate(mechs):
        w(f"    if (mk & {1 << k}u) {{  // {m.suffix}: state update")
        body = _MechBody(m, envs[k], k, consts_of[k])
        body.callables(w)
        w("        if (INIT) {")
        for s in m.states:  # NEURON's start values before INITIAL runs
            if m.writes(s) and s.endswith("i"):
                w(f"            {envs[k][s]} = {_lit(_ION_DEFAULT_CONC.get(s[:-1], 0.0))};")
            else:
                w(f"            {envs[k][s]} = 0;")
        for u in m.useions:
            for wr in u.write:
                if wr == u.ion + "i" and wr not in m.states:
                    w(f"            ion_{wr} = {_lit(_ION_DEFAULT_CONC.get(u.ion, 0.0))};")
        body.stmts(w, m.initial, 3, mode="init")
        w("        } else {")
        solve = [s for s in m.breakpoint if isinstance(s, Solve)]
        for sv in solve:
            if sv.block in m.kinetics:
                if sv.method not in (None, "sparse"):
                    raise NmodlError(f"{m.suffix}: METHOD {sv.method} is not supported for KINETIC {sv.block} "
                                     "(sparse only)")
                body.kinetic(w, sv.block, 3, dict(body.env), steady=False)
                continue
            modes = {None: "deriv", "cnexp": "deriv", "derivimplicit": "deriv_be", "euler": "deriv_euler"}
            if sv.method not in modes:
                raise NmodlError(f"{m.suffix}: METHOD {sv.method} is not supported (cnexp, derivimplicit, euler)")
            if sv.block not in m.derivatives:
                raise NmodlError(f"{m.suffix}: no DERIVATIVE {sv.block}")
            body.stmts(w, m.derivatives[sv.block], 3, mode=modes[sv.method])
        w("        }")
        for s in m.states:  # a concentration the mechanism keeps as a state
            if m.writes(s):
                w(f"        ion_{s} = {envs[k][s]};")
        w("    }")
    # reversal potentials after the concentrations' update
    for ion in ions:
        readers = [k for k, m in enumerate(mechs) if m.reads("e" + ion)]
        if not readers:
            continue
        if (ion + "i") in conc_written:
            z = 2.0 if ion == "ca" else 1.0
            co = cao if ion == "ca" else _ION_DEFAULT_CONC.get(ion, 0.0)
            w(f"    const R ion_e{ion} = {_lit(ktf / z)} * M::lg(M::dv({_lit(co)}, ion_{ion}i));")
        else:
            if ion not in reversal:
                raise NmodlError(f"the reversal potential of {ion} is needed (reversal={{'{ion}': ...}})")
            w(f"    const R ion_e{ion} = {_lit(float(reversal[ion]))};")
    # ---- current phase
    totals = sorted({"i" + u.ion for m in mechs for u in m.useions if ("i" + u.ion) in u.read})
    for t in totals:
        w(f"    R tot_{t} = 0;")
    for k, m in enumerate(mechs):
        w(f"    if (mk & {1 << k}u) {{  // {m.suffix}: currents")
        body = _MechBody(m, envs[k], k, consts_of[k])
        body.callables(w)
        stmts = [s for s in m.breakpoint if not isinstance(s, Solve)]
        dvars = body.current_stmts(w, stmts, 2)
        for c in m.currents():
            w(f"        Itot += {envs[k][c]};")
            w(f"        Gtot += {dvars.get(c, '(R)0')};")
            if c in totals:
                w(f"        tot_{c} += {envs[k][c]};")
        w("    }")
    w("    I = Itot;")
    w("    G = Gtot;")
    # ---- store
    w("    {")
    w("        int s = 0;")
    for k, m in enumerate(mechs):
        env = envs[k]
        alias = _conc_alias(m)
        w(f"        if (mk & {1 << k}u) {{  // {m.suffix}")
        for j, s in enumerate(m.states):
            w(f"            st[(s + {j}) * S] = {env[s]};")
        n = len(m.states)
        for u in m.useions:
            for r in u.read:
                if r == "i" + u.ion:
                    w(f"            st[(s + {n}) * S] = tot_{r};")
                    n += 1
        for u in m.useions:
            for wr in u.write:
                if wr == u.ion + "i" and wr not in m.states and wr not in alias:
                    w(f"            st[(s + {n}) * S] = ion_{wr};")
                    n += 1
        w(f"            s += {n};")
        w("        }")
    w("    }")
    w("}")
    w("}  // namespace ngpu")
    return "\n".join(L) + "\n"


class _MechBody:
    """Statements of one mechanism as C++ (procedures and functions as lambdas)."""

    def __init__(self, m: Mechanism, env: dict, k: int, consts: dict | None = None):
        self.m = m
        self.env = dict(env)
        self.k = k
        self.consts = consts or {}
        self.funcs = {f: f"f{k}_{f}" for f in m.functions}
        self.funcs.update({t: f"t{k}_{t}" for t in m.tables})
        self.procs = {p: f"p{k}_{p}" for p in m.procedures}
        self._tmp = 0

    def _em(self, env):
        return Emitter(env, self.funcs, self.consts)

    def callables(self, w):
        m = self.m
        for tname, (xs, ys) in m.table_data.items():
            # FUNCTION_TABLE: linear interpolation between the given points, the
            # end values outside them (binary search for the interval)
            n = len(xs)
            fn = self.funcs[tname]
            w(f"        auto {fn} = [&](R a_x) -> R {{")
            w(f"            static const R xs[{n}] = {{{', '.join(_lit(x) for x in xs)}}};")
            w(f"            static const R ys[{n}] = {{{', '.join(_lit(y) for y in ys)}}};")
            w(f"            if (!(a_x > xs[0])) return ys[0];")
            w(f"            if (a_x >= xs[{n - 1}]) return ys[{n - 1}];")
            w(f"            int lo = 0, hi = {n - 1};")
            w(f"            while (hi - lo > 1) {{")
            w(f"                const int mid = (lo + hi) >> 1;")
            w(f"                if (xs[mid] <= a_x) lo = mid;")
            w(f"                else hi = mid;")
            w(f"            }}")
            w(f"            return ys[lo] + M::dv(a_x - xs[lo], xs[hi] - xs[lo]) * (ys[hi] - ys[lo]);")
            w(f"        }};")
            w(f"        (void){fn};")
        for fname, (args, body) in m.functions.items():
            env = dict(self.env)
            for a in args:
                env[a] = f"a_{a}"
            env[fname] = "ret"
            locs = self._locals(body, env)
            w(f"        auto {self.funcs[fname]} = [&]({', '.join('R a_' + a for a in args)}) -> R {{")
            w(f"            R ret = 0;")
            if "v" not in args:
                w(f"            R v_l = v;")
                env["v"] = "v_l"
            for l in locs:
                env[l] = f"l_{l}"
            saved = self.consts
            self.consts = self._fold_locals(body, env, locs)
            for l in locs:
                if not env[l].startswith("(R)"):
                    w(f"            R l_{l} = 0;")
            self._block(w, body, 3, env, mode="proc")
            self.consts = saved
            w(f"            return ret;")
            w(f"        }};")
        for pname in self._proc_order():
            args, body = m.procedures[pname]
            env = dict(self.env)
            for a in args:
                env[a] = f"a_{a}"
            locs = self._locals(body, env)
            w(f"        auto {self.procs[pname]} = [&]({', '.join('R a_' + a for a in args)}) {{")
            if "v" not in args:
                w(f"            R v_l = v;")
                env["v"] = "v_l"
            for l in locs:
                env[l] = f"l_{l}"
            saved = self.consts
            self.consts = self._fold_locals(body, env, locs)
            for l in locs:
                if not env[l].startswith("(R)"):
                    w(f"            R l_{l} = 0;")
            self._block(w, body, 3, env, mode="proc")
            self.consts = saved
            w(f"        }};")
            w(f"        (void){self.procs[pname]};")
        for fname in m.functions:
            w(f"        (void){self.funcs[fname]};")

    def _proc_order(self) -> list:
        """Procedures, each after the procedures it calls (lambdas are defined in this order)."""
        m = self.m

        def calls(ss):
            out = set()
            for st in ss:
                if isinstance(st, CallStmt):
                    out.add(st.name)
                elif isinstance(st, If):
                    out |= calls(st.then) | calls(st.other)
            return out
        order, seen = [], set()

        def visit(n, stack=()):
            if n in seen:
                return
            if n in stack:
                raise NmodlError(f"{m.suffix}: recursive procedure {n}")
            for c in sorted(calls(m.procedures[n][1])):
                if c in m.procedures:
                    visit(c, stack + (n,))
            seen.add(n)
            order.append(n)
        for n in m.procedures:
            visit(n)
        return order

    def _fold_locals(self, body, env, locs):
        """LOCALs assigned once, at the top level, from a constant expression:
        mapped to the literal (and folded into later expressions)."""
        count = {}

        def walk(ss):
            for st in ss:
                if isinstance(st, Assign):
                    count[st.name] = count.get(st.name, 0) + 1
                elif isinstance(st, If):
                    walk(st.then)
                    walk(st.other)
        walk(body)
        consts = dict(self.consts)
        for st in body:
            if isinstance(st, Assign) and st.name in locs and count.get(st.name) == 1:
                e = st.e
                for n, val in consts.items():
                    e = subst(e, n, Num(val))
                e = simplify(e)
                if isinstance(e, Num):
                    consts[st.name] = e.v
                    env[st.name] = _lit(e.v)
        return consts

    def _derived(self, body) -> list:
        """States with a derivative in the body (also inside if / else), in order."""
        out = []

        def walk(ss):
            for st_ in ss:
                if isinstance(st_, Deriv) and st_.name not in out:
                    out.append(st_.name)
                elif isinstance(st_, If):
                    walk(st_.then)
                    walk(st_.other)
        walk(body)
        return out

    def _locals(self, body, env) -> list:
        """Names assigned in a body that are not mechanism variables: block locals."""
        out = []

        def walk(ss):
            for s in ss:
                if isinstance(s, Assign) and s.name not in env and s.name not in out:
                    out.append(s.name)
                elif isinstance(s, If):
                    walk(s.then)
                    walk(s.other)
        walk(body)
        return out

    def stmts(self, w, body, ind, mode):
        env = dict(self.env)
        locs = self._locals(body, env)
        pad = "    " * ind
        for l in locs:
            env[l] = f"l_{l}"
        saved = self.consts
        self.consts = self._fold_locals(body, env, locs)
        for l in locs:
            if not env[l].startswith("(R)"):
                w(f"{pad}R l_{l} = 0;")
        integrated = self._derived(body) if mode == "deriv_euler" else []
        for x in integrated:  # euler: every derivative at the step's starting states, then the updates
            w(f"{pad}R eu{self.k}_{x} = 0;")
        self._block(w, body, ind, env, mode)
        for x in integrated:
            w(f"{pad}{env[x]} = {env[x]} + dt * eu{self.k}_{x};")
        self.consts = saved

    def _block(self, w, body, ind, env, mode):
        pad = "    " * ind
        em = self._em(env)
        for s in body:
            if isinstance(s, tuple) and s and s[0] == "local":
                continue
            if isinstance(s, Assign):
                if s.name not in env:
                    raise NmodlError(f"{self.m.suffix}: assignment to unknown {s.name!r}")
                if env[s.name].startswith("(R)"):
                    continue  # a LOCAL folded to a constant
                w(f"{pad}{env[s.name]} = {em.e(s.e)};")
                if s.name + "@rate" in env:
                    w(f"{pad}{env[s.name + '@rate']} = {em.e(recip(s.e))};")
            elif isinstance(s, Deriv):
                if not mode.startswith("deriv"):
                    raise NmodlError(f"{self.m.suffix}: {s.name}' outside a DERIVATIVE block")
                x = s.name
                if x not in self.m.states:
                    raise NmodlError(f"{self.m.suffix}: {x}' of a non-STATE")
                e = simplify(s.e)
                xv = env[x]
                if mode == "deriv_euler":
                    w(f"{pad}eu{self.k}_{x} = {em.e(e)};")
                    continue
                if mode == "deriv_be":
                    # implicit Euler of x' = a + b x, exact for an equation linear in x:
                    # x_new = (x + dt a) / (1 - dt b)
                    coupled = free_vars(e) & (set(self.m.states) - {x})
                    if coupled:
                        raise NmodlError(f"{self.m.suffix}: derivimplicit {x}' depends on other STATEs "
                                         f"({', '.join(sorted(coupled))}): coupled systems are not supported")
                    try:
                        a, b = linear_form(e, x)
                    except NmodlError:
                        raise NmodlError(f"{self.m.suffix}: {x}' is not linear in {x}: derivimplicit is supported "
                                         "for equations linear in their state") from None
                    w(f"{pad}{xv} = M::dv({xv} + dt * ({em.e(a)}), (R)1 - dt * ({em.e(b)}));")
                    continue
                if (isinstance(e, Bin) and e.op == "/" and isinstance(e.l, Bin) and e.l.op == "-"
                        and isinstance(e.l.r, Var) and e.l.r.name == x and x not in free_vars(e.l.l)
                        and x not in free_vars(e.r)):
                    # x' = (xinf - x) / tau
                    if isinstance(e.r, Var) and e.r.name + "@rate" in env:
                        w(f"{pad}{xv} = gen_cnexp_rate({xv}, {em.e(e.l.l)}, {env[e.r.name + '@rate']}, dt);")
                    else:
                        w(f"{pad}{xv} = gen_cnexp_rate({xv}, {em.e(e.l.l)}, {em.e(recip(e.r))}, dt);")
                else:
                    # x' = a + b x: x -> xinf + (x - xinf) exp(b dt), xinf = -a/b, rate -b
                    a, b = linear_form(e, x)
                    rate = simplify(Un("-", b))
                    w(f"{pad}{xv} = gen_cnexp_rate({xv}, {em.e(simplify(Bin('*', a, recip(rate))))}, "
                      f"{em.e(rate)}, dt);")
            elif isinstance(s, If):
                w(f"{pad}if ({em.e(s.cond)}) {{")
                self._block(w, s.then, ind + 1, env, mode)
                if s.other:
                    w(f"{pad}}} else {{")
                    self._block(w, s.other, ind + 1, env, mode)
                w(f"{pad}}}")
            elif isinstance(s, CallStmt):
                if s.name in self.procs:
                    w(f"{pad}{self.procs[s.name]}({', '.join(em.e(a) for a in s.args)});")
                elif s.name in self.funcs:
                    w(f"{pad}(void){self.funcs[s.name]}({', '.join(em.e(a) for a in s.args)});")
                else:
                    raise NmodlError(f"{self.m.suffix}: call of unknown {s.name}()")
            elif isinstance(s, Solve):
                if s.steady:
                    if s.block not in self.m.kinetics or s.method not in (None, "sparse"):
                        raise NmodlError(f"{self.m.suffix}: SOLVE {s.block} STEADYSTATE {s.method}: only KINETIC "
                                         "blocks with sparse")
                    self.kinetic(w, s.block, ind, env, steady=True)
                continue
            else:
                raise NmodlError(f"{self.m.suffix}: unsupported statement {s!r}")

    # a steady state is backward Euler over this step (ms): every rate times
    # the step dwarfs 1, so the solution is the scheme's fixed point
    STEADY_DT = 1e9

    def kinetic(self, w, name, ind, env, steady):
        """A first-order KINETIC scheme advanced by one backward-Euler step,
        (I - dt Q) x' = x + dt s (Q: the rate matrix, s: the << sources), the
        solve NEURON's sparse method performs for a linear scheme.  CONSERVE
        replaces the equation of the last state it names by the conservation
        law.  The system is eliminated without pivoting, in state order with
        the conserved state last: I - dt Q is diagonally dominant by columns
        (each state's outflow appears on its diagonal and as inflow in the
        other rows of its column), so every pivot before the last is at least
        1, and only structural non-zeros and their fill-in are emitted.
        steady (SOLVE ... STEADYSTATE in INITIAL): the same step with
        dt = STEADY_DT in FP64."""
        m = self.m
        body = m.kinetics[name]
        pad = "    " * ind
        T = "double" if steady else "R"
        dts = "(double)" + repr(self.STEADY_DT) if steady else "dt"
        env = dict(env)
        plain = [st for st in body if not isinstance(st, (Reaction, Flux, Conserve))]
        locs = self._locals(plain, env)
        w(f"{pad}{{  // KINETIC {name}{' (steady state)' if steady else ''}")
        ind += 1
        pad = "    " * ind
        for l in locs:
            env[l] = f"l_{l}"
            w(f"{pad}R l_{l} = 0;")
        states = []
        out_rates, in_rates, sources = {}, {}, {}
        conserve = None
        em = self._em(env)
        nr = 0

        def use(x):
            if x not in m.states:
                raise NmodlError(f"{m.suffix}: {x} in KINETIC {name} is not a STATE")
            if x not in states:
                states.append(x)
        for st in body:
            if isinstance(st, Reaction):
                use(st.a)
                use(st.b)
                kf, kb = f"kn{self.k}_f{nr}", f"kn{self.k}_b{nr}"
                nr += 1
                w(f"{pad}const R {kf} = {em.e(st.kf)};")
                w(f"{pad}const R {kb} = {em.e(st.kb)};")
                out_rates.setdefault(st.a, []).append(kf)
                in_rates.setdefault((st.b, st.a), []).append(kf)
                out_rates.setdefault(st.b, []).append(kb)
                in_rates.setdefault((st.a, st.b), []).append(kb)
            elif isinstance(st, Flux):
                use(st.a)
                fl = f"kn{self.k}_s{nr}"
                nr += 1
                w(f"{pad}const R {fl} = {em.e(st.f)};")
                sources.setdefault(st.a, []).append(fl)
            elif isinstance(st, Conserve):
                if conserve is not None:
                    raise NmodlError(f"{m.suffix}: more than one CONSERVE in KINETIC {name}")
                conserve = st
            else:
                self._block(w, [st], ind, env, mode="proc")
        if not states:
            raise NmodlError(f"{m.suffix}: KINETIC {name} has no reactions")
        order = [x for x in m.states if x in states]
        cons_row = {}
        if conserve is not None:
            named = [x for x in _var_order(conserve.lhs) if x in m.states]
            if not named:
                raise NmodlError(f"{m.suffix}: CONSERVE names no STATE")
            for x in named:
                use(x)
            order = [x for x in m.states if x in states]
            for x in order:
                c = simplify(diff(conserve.lhs, x))
                if not isinstance(c, Num):
                    raise NmodlError(f"{m.suffix}: CONSERVE must be linear in the states with constant coefficients")
                if c.v != 0:
                    cons_row[x] = c.v
            rest = simplify(conserve.lhs)
            for x in order:
                rest = subst(rest, x, Num(0.0))
            if free_vars(simplify(rest)):
                raise NmodlError(f"{m.suffix}: CONSERVE's left side may hold only states")
            last = named[-1]
            order = [x for x in order if x != last] + [last]
        n = len(order)
        ix = {x: i for i, x in enumerate(order)}
        mat = {}                        # (row, col) -> C++ variable

        def var(i, j):
            return f"kn{self.k}_m{i}_{j}"
        for x in order:
            i = ix[x]
            if conserve is not None and x == order[-1]:
                for y, c in cons_row.items():
                    mat[(i, ix[y])] = var(i, ix[y])
                    w(f"{pad}{T} {var(i, ix[y])} = ({T}){c!r};")
                w(f"{pad}{T} kn{self.k}_r{i} = ({T})({em.e(conserve.rhs)});")
                continue
            rates = out_rates.get(x, [])
            diag = f"({T})1 + {dts} * ({T})({' + '.join(rates)})" if rates else f"({T})1"
            mat[(i, i)] = var(i, i)
            w(f"{pad}{T} {var(i, i)} = {diag};")
            for y in order:
                r = in_rates.get((x, y))
                if r and y != x:
                    mat[(i, ix[y])] = var(i, ix[y])
                    w(f"{pad}{T} {var(i, ix[y])} = -{dts} * ({T})({' + '.join(r)});")
            src = sources.get(x)
            rhs = f"({T}){env[x]}" + (f" + {dts} * ({T})({' + '.join(src)})" if src else "")
            w(f"{pad}{T} kn{self.k}_r{i} = {rhs};")
        if (n - 1, n - 1) not in mat:
            raise NmodlError(f"{m.suffix}: CONSERVE of KINETIC {name} leaves its last state out")
        div = (lambda a, b: f"{a} / {b}") if steady else (lambda a, b: f"M::dv({a}, {b})")
        for p_ in range(n):
            w(f"{pad}const {T} kn{self.k}_i{p_} = {div(f'({T})1', var(p_, p_))};")
            for r in range(p_ + 1, n):
                if (r, p_) not in mat:
                    continue
                f = f"kn{self.k}_l{r}_{p_}"
                w(f"{pad}const {T} {f} = {var(r, p_)} * kn{self.k}_i{p_};")
                for c in range(p_ + 1, n):
                    if (p_, c) not in mat:
                        continue
                    if (r, c) in mat:
                        w(f"{pad}{var(r, c)} -= {f} * {var(p_, c)};")
                    else:
                        mat[(r, c)] = var(r, c)
                        w(f"{pad}{T} {var(r, c)} = -{f} * {var(p_, c)};")
                w(f"{pad}kn{self.k}_r{r} -= {f} * kn{self.k}_r{p_};")
        for p_ in reversed(range(n)):
            acc = f"kn{self.k}_r{p_}"
            for c in range(p_ + 1, n):
                if (p_, c) in mat:
                    w(f"{pad}{acc} -= {var(p_, c)} * kn{self.k}_r{c};")
            w(f"{pad}{acc} *= kn{self.k}_i{p_};")
        for x in order:
            w(f"{pad}{env[x]} = (R)kn{self.k}_r{ix[x]};")
        w("    " * (ind - 1) + "}")

    def current_stmts(self, w, body, ind) -> dict:
        """BREAKPOINT assignments with their d/dv: returns name -> C++ derivative."""
        pad = "    " * ind
        env = dict(self.env)
        known = {}          # name -> symbolic derivative (an AST over d_ variables)
        dnames = {}
        for s in body:
            if isinstance(s, Assign):
                if s.name not in env:
                    raise NmodlError(f"{self.m.suffix}: assignment to unknown {s.name!r}")
                de = simplify(diff(s.e, "v", {n: (d if isinstance(d, Num) else Var("d_" + n))
                                              for n, d in known.items()}))
                denv = dict(env)
                denv.update({"d_" + n: dnames[n] for n in known})
                em = Emitter(denv, self.funcs, self.consts)
                w(f"{pad}{env[s.name]} = {em.e(s.e)};")
                dn = f"d{self.k}_{s.name}"
                if not dnames.get(s.name):
                    w(f"{pad}R {dn} = {em.e(de)};")
                else:
                    w(f"{pad}{dn} = {em.e(de)};")
                dnames[s.name] = dn
                known[s.name] = de
            elif isinstance(s, tuple):
                continue
            elif isinstance(s, CallStmt) and s.name in self.procs:
                raise NmodlError(f"{self.m.suffix}: procedure calls in BREAKPOINT are not supported")
            else:
                raise NmodlError(f"{self.m.suffix}: unsupported BREAKPOINT statement {s!r}")
        return dnames


def generate_from_files(paths, **kw) -> GeneratedMechSet:
    """generate() over .mod files (paths)."""
    mods = {Path(p).stem: Path(p).read_text() for p in paths}
    return generate(mods, **kw)
