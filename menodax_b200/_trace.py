"""Trace a tuple-form right-hand side into an expression graph and differentiate it.

The public solvers take the right-hand side the way ``modax`` does
(``modax/tsit5.py:623``, ``modax/rodas5P.py:1024``): a plain Python function
``ode_fn(y, t, p)`` that indexes ``y`` and ``p`` with literals and returns a tuple
of components.  ``modax`` hands that function to numba and differentiates it with
Enzyme (``modax/_sensitivity.py:148-179``).  Here it is *run once on the host* with
symbolic proxies for ``y``, ``t`` and ``p``; every arithmetic operation records a
node in a hash-consed graph, so common subexpressions collapse as they are built.

The graph is then differentiated symbolically:

* forward mode with an arbitrary seed (constant or symbolic) -- the coloured
  Jacobian sweep, ``df/dt``, the sensitivity right-hand side ``J S + J_p`` and the
  second-order coupling term are all tangents of the primal graph;
* reverse mode -- the vector-Jacobian products the discrete adjoint needs.

A tangent that is structurally zero is ``None`` and never emitted, which is what
folding a literal seed does for ``modax`` after inlining (``modax/rodas5P.py:480-490``).
"""

from __future__ import annotations

import math
import operator
import types
from dataclasses import dataclass

# Operators with one argument, and the ones the emitter spells as CUDA calls.
UNARY = (
    "neg", "exp", "log", "log10", "log2", "sqrt", "sin", "cos", "tan", "asin",
    "acos", "atan", "sinh", "cosh", "tanh", "log1p", "expm1", "abs", "sign",
)
BINARY = ("add", "sub", "mul", "div", "pow", "atan2")


class TraceError(TypeError):
    """The callback did something a traced right-hand side cannot do."""


@dataclass(frozen=True)
class Node:
    op: str
    args: tuple[int, ...] = ()
    payload: object = None  # constant value, or the (kind, index) of a variable


class Graph:
    """Hash-consed expression DAG. Node ids are positions in ``nodes``."""

    def __init__(self):
        self.nodes: list[Node] = []
        self._index: dict[Node, int] = {}

    # --- construction -------------------------------------------------------
    def _add(self, node: Node) -> int:
        found = self._index.get(node)
        if found is not None:
            return found
        self.nodes.append(node)
        nid = len(self.nodes) - 1
        self._index[node] = nid
        return nid

    def const(self, value: float) -> int:
        value = float(value)
        # -0.0 and 0.0 hash equal; keep them apart so signs survive folding.
        key = (value, math.copysign(1.0, value)) if value == 0.0 else value
        return self._add(Node("const", (), key))

    def var(self, kind: str, index: int = 0) -> int:
        return self._add(Node("var", (), (kind, int(index))))

    def is_const(self, nid: int) -> bool:
        return self.nodes[nid].op == "const"

    def value(self, nid: int) -> float:
        payload = self.nodes[nid].payload
        return payload[0] if isinstance(payload, tuple) else payload

    def powi(self, base: int, n: int) -> int:
        """``base ** n`` for an integer literal ``n``, by binary powering on device."""
        n = int(n)
        if n == 0:
            return self.const(1.0)
        if n == 1:
            return base
        if self.is_const(base):
            return self.const(_int_power(self.value(base), n))
        return self._add(Node("powi", (base,), n))

    def op(self, name: str, *args: int) -> int:
        if all(self.is_const(a) for a in args):
            folded = _fold(name, [self.value(a) for a in args])
            if folded is not None:
                return self.const(folded)
        return self._add(Node(name, tuple(args)))

    # --- helpers that drop structural zeros (derivative construction only) ----
    def zadd(self, a, b):
        if a is None:
            return b
        if b is None:
            return a
        return self.op("add", a, b)

    def zsub(self, a, b):
        if b is None:
            return a
        if a is None:
            return self.op("neg", b)
        return self.op("sub", a, b)

    def zmul(self, a, b):
        if a is None or b is None:
            return None
        if self.is_const(a) and self.value(a) == 1.0:
            return b
        if self.is_const(b) and self.value(b) == 1.0:
            return a
        if self.is_const(a) and self.value(a) == -1.0:
            return self.op("neg", b)
        if self.is_const(b) and self.value(b) == -1.0:
            return self.op("neg", a)
        return self.op("mul", a, b)

    def zneg(self, a):
        return None if a is None else self.op("neg", a)

    def zdiv(self, a, b):
        if a is None:
            return None
        return self.op("div", a, b)

    # --- differentiation ------------------------------------------------------
    def local_partials(self, nid: int) -> list[int]:
        """d node / d arg_k for each argument, as graph nodes."""
        node = self.nodes[nid]
        op, args = node.op, node.args
        c = self.const
        if op == "add":
            return [c(1.0), c(1.0)]
        if op == "sub":
            return [c(1.0), c(-1.0)]
        if op == "mul":
            return [args[1], args[0]]
        if op == "div":
            a, b = args
            inv_b = self.op("div", c(1.0), b)
            return [inv_b, self.op("neg", self.op("div", nid, b))]
        if op == "neg":
            return [c(-1.0)]
        x = args[0]
        if op == "exp":
            return [nid]
        if op == "expm1":
            return [self.op("exp", x)]
        if op == "log":
            return [self.op("div", c(1.0), x)]
        if op == "log10":
            return [self.op("div", c(1.0), self.op("mul", x, c(math.log(10.0))))]
        if op == "log2":
            return [self.op("div", c(1.0), self.op("mul", x, c(math.log(2.0))))]
        if op == "log1p":
            return [self.op("div", c(1.0), self.op("add", c(1.0), x))]
        if op == "sqrt":
            return [self.op("div", c(0.5), nid)]
        if op == "sin":
            return [self.op("cos", x)]
        if op == "cos":
            return [self.op("neg", self.op("sin", x))]
        if op == "tan":
            return [self.op("add", c(1.0), self.op("mul", nid, nid))]
        if op == "asin":
            return [self.op("div", c(1.0), self.op("sqrt", self.op("sub", c(1.0), self.op("mul", x, x))))]
        if op == "acos":
            return [self.op("neg", self.op("div", c(1.0), self.op("sqrt", self.op("sub", c(1.0), self.op("mul", x, x)))))]
        if op == "atan":
            return [self.op("div", c(1.0), self.op("add", c(1.0), self.op("mul", x, x)))]
        if op == "sinh":
            return [self.op("cosh", x)]
        if op == "cosh":
            return [self.op("sinh", x)]
        if op == "tanh":
            return [self.op("sub", c(1.0), self.op("mul", nid, nid))]
        if op == "abs":
            return [self.op("sign", x)]
        if op == "sign":
            return [c(0.0)]
        if op == "powi":
            n = node.payload
            return [self.op("mul", c(float(n)), self.powi(x, n - 1))]
        if op == "pow":
            base, expo = args
            if self.is_const(expo):
                e = self.value(expo)
                if e == 0.0:
                    return [c(0.0), c(0.0)]
                d_base = self.op("mul", expo, self.op("pow", base, c(e - 1.0)))
                return [d_base, c(0.0)]
            d_base = self.op("mul", expo, self.op("pow", base, self.op("sub", expo, c(1.0))))
            d_expo = self.op("mul", self.op("log", base), nid)
            return [d_base, d_expo]
        if op == "atan2":
            yy, xx = args
            den = self.op("add", self.op("mul", xx, xx), self.op("mul", yy, yy))
            return [self.op("div", xx, den), self.op("neg", self.op("div", yy, den))]
        raise TraceError(f"no derivative rule for {op!r}")

    def topo(self, roots) -> list[int]:
        """Every node the roots depend on, dependencies first."""
        order: list[int] = []
        seen: set[int] = set()
        stack = [(r, False) for r in roots if r is not None]
        while stack:
            nid, expanded = stack.pop()
            if expanded:
                order.append(nid)
                continue
            if nid in seen:
                continue
            seen.add(nid)
            stack.append((nid, True))
            for a in self.nodes[nid].args:
                if a not in seen:
                    stack.append((a, False))
        return order

    def forward(self, outputs, seeds: dict[int, int]):
        """Tangents of ``outputs`` for a seed given per variable node.

        ``seeds`` maps a variable node id to its tangent node (absent = zero).
        Returns one tangent node per output, ``None`` where structurally zero.
        """
        tangent: dict[int, int | None] = {}
        for nid in self.topo(outputs):
            node = self.nodes[nid]
            if node.op == "const":
                tangent[nid] = None
            elif node.op in ("table", "accdyn"):
                tangent[nid] = None
            elif node.op == "var":
                tangent[nid] = seeds.get(nid)
            else:
                arg_t = [tangent[a] for a in node.args]
                if all(t is None for t in arg_t):
                    tangent[nid] = None
                    continue
                partials = self.local_partials(nid)
                acc = None
                for t_arg, d in zip(arg_t, partials):
                    if t_arg is None:
                        continue
                    if self.is_const(d) and self.value(d) == 0.0:
                        continue
                    acc = self.zadd(acc, self.zmul(d, t_arg))
                tangent[nid] = acc
        return [tangent.get(o) if o is not None else None for o in outputs]

    def reverse(self, outputs, cotangents, wrt):
        """Gradient of ``sum_k cotangents[k] * outputs[k]`` with respect to ``wrt``.

        ``cotangents`` are nodes (or ``None`` for zero); returns one node (or
        ``None``) per entry of ``wrt``.
        """
        adjoint: dict[int, int | None] = {}
        for o, ct in zip(outputs, cotangents):
            if o is None or ct is None:
                continue
            adjoint[o] = self.zadd(adjoint.get(o), ct)
        for nid in reversed(self.topo([o for o in outputs if o is not None])):
            bar = adjoint.get(nid)
            node = self.nodes[nid]
            if bar is None or node.op in ("const", "var"):
                continue
            partials = self.local_partials(nid)
            for a, d in zip(node.args, partials):
                if self.is_const(d) and self.value(d) == 0.0:
                    continue
                adjoint[a] = self.zadd(adjoint.get(a), self.zmul(d, bar))
        return [adjoint.get(w) for w in wrt]


def _int_power(x: float, n: int) -> float:
    """Binary powering, the sequence the device code evaluates for ``x ** n``."""
    invert = n < 0
    e = -n if invert else n
    r = 1.0
    a = x
    while e:
        if e & 1:
            r = r * a
        e >>= 1
        if e:
            a = a * a
    try:
        return 1.0 / r if invert else r
    except ZeroDivisionError:
        return math.copysign(math.inf, r)


def _fold(name, vals):
    """Constant-fold an operator on Python floats (IEEE double, as on the GPU)."""
    try:
        if name == "add":
            return vals[0] + vals[1]
        if name == "sub":
            return vals[0] - vals[1]
        if name == "mul":
            return vals[0] * vals[1]
        if name == "div":
            if vals[1] == 0.0:
                return None
            return vals[0] / vals[1]
        if name == "neg":
            return -vals[0]
        if name == "pow":
            if vals[1] == 2.0:
                return vals[0] * vals[0]
            return math.pow(vals[0], vals[1])
        if name == "sign":
            return 1.0 if vals[0] >= 0.0 else -1.0
        if name == "abs":
            return abs(vals[0])
        if name == "atan2":
            return math.atan2(vals[0], vals[1])
        fn = getattr(math, {"log": "log"}.get(name, name), None)
        if fn is None:
            return None
        return fn(vals[0])
    except (ValueError, OverflowError, ZeroDivisionError):
        return None


# --- the proxies the callback sees -------------------------------------------------
class Sym:
    """A traced scalar. Arithmetic records nodes; branching on it is refused."""

    __slots__ = ("g", "nid")
    __array_priority__ = 1000

    def __init__(self, g: Graph, nid: int):
        self.g = g
        self.nid = nid

    def _lift(self, other) -> int:
        if isinstance(other, Sym):
            return other.nid
        if isinstance(other, (int, float)) and not isinstance(other, bool):
            return self.g.const(float(other))
        try:  # numpy scalars
            return self.g.const(float(other))
        except (TypeError, ValueError):
            raise TraceError(
                f"cannot combine a traced value with {type(other).__name__}"
            ) from None

    def _bin(self, name, other, swap=False):
        o = self._lift(other)
        a, b = (o, self.nid) if swap else (self.nid, o)
        return Sym(self.g, self.g.op(name, a, b))

    def __add__(self, o):
        return self._bin("add", o)

    def __radd__(self, o):
        return self._bin("add", o, swap=True)

    def __sub__(self, o):
        return self._bin("sub", o)

    def __rsub__(self, o):
        return self._bin("sub", o, swap=True)

    def __mul__(self, o):
        return self._bin("mul", o)

    def __rmul__(self, o):
        return self._bin("mul", o, swap=True)

    def __truediv__(self, o):
        return self._bin("div", o)

    def __rtruediv__(self, o):
        return self._bin("div", o, swap=True)

    def __pow__(self, o):
        if isinstance(o, int) and not isinstance(o, bool):
            return Sym(self.g, self.g.powi(self.nid, o))
        return self._bin("pow", o)

    def __rpow__(self, o):
        return self._bin("pow", o, swap=True)

    def __neg__(self):
        return Sym(self.g, self.g.op("neg", self.nid))

    def __pos__(self):
        return self

    def __abs__(self):
        return Sym(self.g, self.g.op("abs", self.nid))

    def _refuse(self, *_):
        raise TraceError(
            "the right-hand side branches on a traced value; a traced callback "
            "must be straight-line arithmetic (use math functions, not if/min/max)"
        )

    __bool__ = __lt__ = __le__ = __gt__ = __ge__ = _refuse
    __float__ = __int__ = __index__ = _refuse

    def __eq__(self, other):
        return self._refuse()

    __hash__ = object.__hash__


class _Vector:
    """``y`` / ``p`` as the callback sees them: literal indexing only."""

    def __init__(self, g: Graph, kind: str, size: int):
        self._g = g
        self._kind = kind
        self._size = size

    def __getitem__(self, index):
        if isinstance(index, slice):
            return [self[i] for i in range(*index.indices(self._size))]
        try:
            i = operator.index(index)
        except TypeError:
            raise TraceError(
                f"{self._kind}[...] must be indexed with an integer literal"
            ) from None
        if i < 0:
            i += self._size
        if not 0 <= i < self._size:
            raise TraceError(f"{self._kind}[{index}] is outside its {self._size} entries")
        return Sym(self._g, self._g.var(self._kind, i))

    def __len__(self):
        return self._size

    def __iter__(self):
        return (self[i] for i in range(self._size))


def _unary(name):
    def fn(x):
        if isinstance(x, Sym):
            return Sym(x.g, x.g.op(name, x.nid))
        return getattr(math, name)(x)

    fn.__name__ = name
    return fn


def _pow(x, y):
    if isinstance(x, Sym):
        return x ** y
    if isinstance(y, Sym):
        return y.__rpow__(x)
    return math.pow(x, y)


def _atan2(a, b):
    if isinstance(a, Sym) or isinstance(b, Sym):
        g = a.g if isinstance(a, Sym) else b.g
        lift = (a if isinstance(a, Sym) else b)._lift
        return Sym(g, g.op("atan2", lift(a), lift(b)))
    return math.atan2(a, b)


def _fabs(x):
    return abs(x)


def _make_math_shim():
    shim = types.ModuleType("math")
    for name in dir(math):
        setattr(shim, name, getattr(math, name))
    for name in ("exp", "log", "log10", "log2", "sqrt", "sin", "cos", "tan", "asin",
                 "acos", "atan", "sinh", "cosh", "tanh", "log1p", "expm1"):
        setattr(shim, name, _unary(name))
    shim.pow = _pow
    shim.atan2 = _atan2
    shim.fabs = _fabs
    return shim


MATH_SHIM = _make_math_shim()


def _with_shimmed_globals(fn):
    """The callback with ``math`` (and names imported from it) swapped for the shim."""
    if not isinstance(fn, types.FunctionType):
        return fn
    g = dict(fn.__globals__)
    for key, val in list(g.items()):
        if val is math:
            g[key] = MATH_SHIM
        elif getattr(val, "__module__", None) == "math" or (
            isinstance(val, types.BuiltinFunctionType) and getattr(math, key, None) is val
        ):
            replacement = getattr(MATH_SHIM, getattr(val, "__name__", key), None)
            if replacement is not None:
                g[key] = replacement
    return types.FunctionType(fn.__code__, g, fn.__name__, fn.__defaults__, fn.__closure__)


@dataclass
class TracedRHS:
    """A right-hand side as a graph: ``outputs[j]`` is component ``j`` of f."""

    graph: Graph
    n_vars: int
    n_params: int
    y: list[int]
    t: int
    p: list[int]
    outputs: list[int]


def trace(ode_fn, n_vars: int, n_params: int) -> TracedRHS:
    """Run ``ode_fn`` on proxies and return its expression graph."""
    g = Graph()
    y = _Vector(g, "y", n_vars)
    p = _Vector(g, "p", n_params)
    t = Sym(g, g.var("t"))
    fn = _with_shimmed_globals(ode_fn)
    try:
        result = fn(y, t, p)
    except TraceError:
        raise
    except TypeError as exc:
        raise TraceError(f"tracing the right-hand side failed: {exc}") from exc
    try:
        comps = list(result)
    except TypeError:
        raise TraceError("the right-hand side must return a tuple of components") from None
    if len(comps) != n_vars:
        raise ValueError(
            f"the right-hand side returned {len(comps)} components for a state of {n_vars}"
        )
    outputs = []
    for c in comps:
        if isinstance(c, Sym):
            outputs.append(c.nid)
        else:
            outputs.append(g.const(float(c)))
    return TracedRHS(
        graph=g,
        n_vars=n_vars,
        n_params=n_params,
        y=[g.var("y", i) for i in range(n_vars)],
        t=g.var("t"),
        p=[g.var("p", k) for k in range(n_params)],
        outputs=outputs,
    )


class _OutRow:
    """``out`` as an array right-hand side sees it: literal-index writes, in order;
    a read returns the last value written there."""

    def __init__(self, g: Graph, size: int):
        self._g = g
        self._size = size
        self.values: list = [None] * size

    def _index(self, index):
        try:
            i = operator.index(index)
        except TypeError:
            raise TraceError("out[...] must be indexed with an integer literal") from None
        if i < 0:
            i += self._size
        if not 0 <= i < self._size:
            raise TraceError(f"out[{index}] is outside its {self._size} entries")
        return i

    def __setitem__(self, index, value):
        i = self._index(index)
        self.values[i] = value.nid if isinstance(value, Sym) else self._g.const(float(value))

    def __getitem__(self, index):
        i = self._index(index)
        if self.values[i] is None:
            raise TraceError(f"out[{i}] is read before the right-hand side writes it")
        return Sym(self._g, self.values[i])

    def __len__(self):
        return self._size


def trace_array_rhs(array_rhs, primal: TracedRHS) -> TracedRHS:
    """Trace an array-form right-hand side ``array_rhs(y, t, p, out)`` into the graph
    of ``primal`` (the same ``y``, ``t`` and ``p`` leaves).

    The result carries ``array_rhs``'s outputs: the kernels evaluate the stages
    with it while every derivative still comes from ``primal``
    (``modax/rodas5P.py:382-391``).  Every ``out`` entry must be written."""
    g = primal.graph
    out = _OutRow(g, primal.n_vars)
    fn = _with_shimmed_globals(array_rhs)
    try:
        fn(_Vector(g, "y", primal.n_vars), Sym(g, primal.t), _Vector(g, "p", primal.n_params), out)
    except TraceError:
        raise
    except TypeError as exc:
        raise TraceError(f"tracing array_rhs failed: {exc}") from exc
    missing = [i for i, v in enumerate(out.values) if v is None]
    if missing:
        raise TraceError(f"array_rhs left out{missing} unwritten; it must write all {primal.n_vars} entries")
    return TracedRHS(graph=g, n_vars=primal.n_vars, n_params=primal.n_params, y=primal.y, t=primal.t,
                     p=primal.p, outputs=list(out.values))


def evaluate(traced: TracedRHS, y, t, p):
    """Evaluate the traced graph in Python floats (host-side check of a trace)."""
    g = traced.graph
    vals: dict[int, float] = {}
    for nid in g.topo(traced.outputs):
        node = g.nodes[nid]
        if node.op == "const":
            vals[nid] = g.value(nid)
        elif node.op == "var":
            kind, idx = node.payload
            vals[nid] = {"y": lambda: y[idx], "t": lambda: t, "p": lambda: p[idx]}[kind]()
        elif node.op == "powi":
            vals[nid] = _int_power(vals[node.args[0]], node.payload)
        else:
            folded = _fold(node.op, [vals[a] for a in node.args])
            if folded is None:
                folded = float("nan")
            vals[nid] = folded
    return [vals[o] for o in traced.outputs]


# --- save hooks -----------------------------------------------------------------------
class SaveIndex:
    """The save index a hook receives: usable as an index (``acc[save_idx]``,
    ``table[save_idx + 1]``) and, lifted to a float, in arithmetic."""

    def __init__(self, g: Graph, offset: int = 0):
        self.g = g
        self.offset = int(offset)

    def __add__(self, other):
        if isinstance(other, int) and not isinstance(other, bool):
            return SaveIndex(self.g, self.offset + other)
        return self._as_sym() + other

    __radd__ = __add__

    def __sub__(self, other):
        if isinstance(other, int) and not isinstance(other, bool):
            return SaveIndex(self.g, self.offset - other)
        return self._as_sym() - other

    def _as_sym(self):
        s = Sym(self.g, self.g.var("sidx"))
        return s + float(self.offset) if self.offset else s

    def __mul__(self, other):
        return self._as_sym() * other

    __rmul__ = __mul__

    def __float__(self):
        raise TraceError("use the save index as an index, or in arithmetic with traced values")

    def __index__(self):
        raise TraceError("the save index is only known on the device; index acc or a table with it")


class _Table:
    """A host array a hook closes over, readable at literal or save-index positions."""

    def __init__(self, g: Graph, tables: list, values):
        import numpy as np

        self.g = g
        self.values = np.asarray(values, dtype=np.float64).ravel()
        self.tid = len(tables)
        tables.append(self.values)

    def __getitem__(self, index):
        if isinstance(index, SaveIndex):
            return Sym(self.g, self.g._add(Node("table", (), (self.tid, index.offset))))
        return Sym(self.g, self.g.const(float(self.values[operator.index(index)])))

    def __len__(self):
        return len(self.values)


class _Accumulator:
    """The hook's output row: reads see the row as it was when the hook was
    called, writes are applied in program order when it returns."""

    def __init__(self, g: Graph, size: int):
        self.g = g
        self.size = size
        self.current: dict[int, object] = {}
        self.stores: list = []  # (slot or ("dyn", offset), node)

    def _slot(self, index):
        if isinstance(index, SaveIndex):
            return ("dyn", index.offset)
        i = operator.index(index)
        if not 0 <= i < self.size:
            raise TraceError(f"acc[{i}] is outside the hook's {self.size} slots")
        return i

    def __getitem__(self, index):
        slot = self._slot(index)
        if slot in self.current:
            return self.current[slot]
        if isinstance(slot, tuple):
            return Sym(self.g, self.g._add(Node("accdyn", (), slot[1])))
        return Sym(self.g, self.g.var("acc", slot))

    def __setitem__(self, index, value):
        slot = self._slot(index)
        node = value.nid if isinstance(value, Sym) else self.g.const(float(value))
        self.current[slot] = Sym(self.g, node)
        self.stores.append((slot, node))

    def __len__(self):
        return self.size


@dataclass
class TracedHook:
    graph: Graph
    stores: list
    tables: list
    hook_size: int

    def bounds(self):
        """``(name, length, min offset, max offset)`` of every save-index access."""
        out = []
        for node in self.graph.nodes:
            if node.op == "table":
                tid, off = node.payload
                out.append((f"table {tid}", len(self.tables[tid]), off, off))
            elif node.op == "accdyn":
                out.append(("acc", self.hook_size, node.payload, node.payload))
        for slot, _ in self.stores:
            if isinstance(slot, tuple):
                out.append(("acc", self.hook_size, slot[1], slot[1]))
        return out


def trace_hook(hook, n_system: int, n_params: int, hook_size: int) -> TracedHook:
    """Run a save hook ``hook(save_idx, y, t, p_row, acc)`` on proxies."""
    import numpy as np

    g = Graph()
    tables: list = []
    fn = _with_shimmed_globals(hook)
    if isinstance(fn, types.FunctionType):
        # Arrays the hook closes over or reads as globals become device tables.
        def wrap(v):
            if isinstance(v, np.ndarray) or type(v).__name__ == "Tensor":
                return _Table(g, tables, v.detach().cpu().numpy() if hasattr(v, "detach") else v)
            return v

        glb = {k: wrap(v) for k, v in fn.__globals__.items()}
        cells = None
        if fn.__closure__:
            cells = tuple(types.CellType(wrap(c.cell_contents)) for c in fn.__closure__)
        fn = types.FunctionType(fn.__code__, glb, fn.__name__, fn.__defaults__, cells)
    acc = _Accumulator(g, hook_size)
    try:
        fn(SaveIndex(g), _Vector(g, "y", n_system), Sym(g, g.var("t")), _Vector(g, "p", n_params), acc)
    except TraceError:
        raise
    except TypeError as exc:
        raise TraceError(f"tracing the save hook failed: {exc}") from exc
    return TracedHook(graph=g, stores=acc.stores, tables=tables, hook_size=hook_size)
