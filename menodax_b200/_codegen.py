"""Emit CUDA C++ for a traced right-hand side and the problem header a kernel needs.

Every function is emitted as straight-line code over literal indices, the way
``modax`` emits its seed-literal Jacobian writer (``modax/rodas5P.py:251-303``):
one temporary per graph node, each node once, structurally zero tangents never
emitted.  The kernel templates (``csrc/kernels/*.cuh``) consume:

* ``mdx_rhs(y, t, p, out)``              -- the integrated system (state, or joint
  ``[y, S]`` with forward sensitivities, ``modax/_sensitivity.py:198-243``);
* ``mdx_neg_jac(y, t, p, lu, dT)``       -- ``-J`` into the LU slots, one forward
  sweep per colour group, and ``df/dt`` (plus ``d(J S + J_p)/dt`` for sensitivity
  rows, ``modax/rodas5P.py:403-437``);
* ``mdx_sens_coupling(y, t, p, k, c)``   -- ``L_k k_y`` for every sensitivity block,
  the second-order term of the joint stage solve (``modax/rodas5P.py:513-565``);
* ``mdx_vjp`` / ``mdx_hvp`` / ``mdx_ft_vjp`` -- the reverse-mode pieces of the
  discrete adjoint.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

from menodax_b200._trace import Graph, TracedRHS

_CALLS = {
    "exp": "exp", "log": "log", "log10": "log10", "log2": "log2", "sqrt": "sqrt",
    "sin": "sin", "cos": "cos", "tan": "tan", "asin": "asin", "acos": "acos",
    "atan": "atan", "sinh": "sinh", "cosh": "cosh", "tanh": "tanh", "log1p": "log1p",
    "expm1": "expm1", "abs": "fabs",
}


def lit(x: float) -> str:
    """A C++ double literal that parses back to exactly ``x``."""
    x = float(x)
    if math.isnan(x):
        return "__longlong_as_double(0x7ff8000000000000LL)"
    if math.isinf(x):
        return ("-" if x < 0 else "") + "__longlong_as_double(0x7ff0000000000000LL)"
    r = repr(x)
    if "e" not in r and "." not in r and "inf" not in r:
        r += ".0"
    return f"({r})" if r.startswith("-") else r


class Emitter:
    """Emits nodes of one graph as ``const double`` temporaries, each once."""

    def __init__(self, graph: Graph, names: dict[str, str], prefix: str = "v"):
        self.g = graph
        self.names = names  # variable kind -> C array name ('t' maps to a scalar)
        self.prefix = prefix
        self.lines: list[str] = []
        self.done: dict[int, str] = {}
        self._tmp = 0

    def _tmpname(self) -> str:
        self._tmp += 1
        return f"{self.prefix}_t{self._tmp}"

    def expr(self, nid: int | None) -> str:
        if nid is None:
            return "0.0"
        for n in self.g.topo([nid]):
            if n not in self.done:
                self._emit(n)
        return self.done[nid]

    def _emit(self, nid: int):
        node = self.g.nodes[nid]
        op = node.op
        if op == "const":
            self.done[nid] = lit(self.g.value(nid))
            return
        if op == "var":
            kind, idx = node.payload
            name = self.names.get(kind)
            if name is None:
                raise KeyError(f"no C name bound for variable kind {kind!r}")
            if callable(name):
                self.done[nid] = name(idx)
            else:
                self.done[nid] = name if kind in ("t", "sidx") else f"{name}[{idx}]"
            return
        if op == "table":
            tid, off = node.payload
            nm = f"{self.prefix}{nid}"
            self.lines.append(f"  const double {nm} = mdx_hook_table{tid}[save_idx + ({off})];")
            self.done[nid] = nm
            return
        if op == "accdyn":
            nm = f"{self.prefix}{nid}"
            self.lines.append(f"  const double {nm} = acc[save_idx + ({node.payload})];")
            self.done[nid] = nm
            return
        a = [self.done[x] for x in node.args]
        if op == "add":
            rhs = f"{a[0]} + {a[1]}"
        elif op == "sub":
            rhs = f"{a[0]} - {a[1]}"
        elif op == "mul":
            rhs = f"{a[0]} * {a[1]}"
        elif op == "div":
            rhs = f"{a[0]} / {a[1]}"
        elif op == "neg":
            rhs = f"-{a[0]}"
        elif op == "pow":
            rhs = f"pow({a[0]}, {a[1]})"
        elif op == "atan2":
            rhs = f"atan2({a[0]}, {a[1]})"
        elif op == "sign":
            rhs = f"({a[0]} >= 0.0 ? 1.0 : -1.0)"
        elif op == "powi":
            rhs = self._powi(a[0], node.payload)
        elif op in _CALLS:
            rhs = f"{_CALLS[op]}({a[0]})"
        else:
            raise ValueError(f"cannot emit operator {op!r}")
        name = f"{self.prefix}{nid}"
        self.lines.append(f"  const double {name} = {rhs};")
        self.done[nid] = name

    def _powi(self, x: str, n: int) -> str:
        # Binary powering in the order numba lowers an integer power: the
        # running product starts at the first set bit, the base squares after.
        invert = n < 0
        e = -n if invert else n
        r = None
        base = x
        while e:
            if e & 1:
                if r is None:
                    r = base
                else:
                    nm = self._tmpname()
                    self.lines.append(f"  const double {nm} = {r} * {base};")
                    r = nm
            e >>= 1
            if e:
                nm = self._tmpname()
                self.lines.append(f"  const double {nm} = {base} * {base};")
                base = nm
        return f"1.0 / {r}" if invert else r


@dataclass
class SensLayout:
    """Forward-sensitivity directions: ``n_y0_dirs`` state blocks then parameter columns."""

    n_vars: int
    n_params: int
    n_y0_dirs: int
    param_columns: tuple[int, ...]

    @property
    def n_sens(self) -> int:
        return self.n_y0_dirs + len(self.param_columns)

    def param_of(self, k: int):
        return None if k < self.n_y0_dirs else self.param_columns[k - self.n_y0_dirs]


def _sens_tangents(tr: TracedRHS, sens: SensLayout):
    """``J_y S_k + J_p,k`` per direction, ``S_k`` read from the joint state vector."""
    g, n = tr.graph, tr.n_vars
    out = []
    for k in range(sens.n_sens):
        seeds = {tr.y[c]: g.var("y", n + k * n + c) for c in range(n)}
        col = sens.param_of(k)
        if col is not None:
            seeds[tr.p[col]] = g.const(1.0)
        out.append(g.forward(tr.outputs, seeds))
    return out


def emit_rhs(tr: TracedRHS, sens: SensLayout | None = None) -> str:
    em = Emitter(tr.graph, {"y": "y", "t": "t", "p": "p"})
    assigns = [f"  out[{j}] = {em.expr(o)};" for j, o in enumerate(tr.outputs)]
    if sens is not None:
        n = tr.n_vars
        for k, tang in enumerate(_sens_tangents(tr, sens)):
            for r, node in enumerate(tang):
                assigns.append(f"  out[{n + k * n + r}] = {em.expr(node)};")
    return (
        "template <class Y, class O>\n"
        "__device__ __forceinline__ void mdx_rhs(const Y& y, const double t, const double* p, O& out) {\n"
        + "\n".join(em.lines + assigns) + "\n}\n"
    )


def emit_neg_jac(tr: TracedRHS, compressed, lu_size: int, sens: SensLayout | None = None) -> str:
    """``-J`` by colour-group forward sweeps into the LU slots, and ``df/dt`` into dT.

    On the colour grid every slot ``row * n_colours + g`` is written; on a packed
    (sparse) layout only the slots an entry claims, after clearing the buffer when
    the factorisation has fill-in slots nothing else writes
    (``modax/rodas5P.py:375-378, 465-476``).
    """
    g, n = tr.graph, tr.n_vars
    em = Emitter(g, {"y": "y", "t": "t", "p": "p"})
    body: list[str] = []
    store = compressed.store_slots()
    needs_clear = store is not None and lu_size > int((store >= 0).sum())
    if needs_clear:
        body.append(f"#pragma unroll\n  for (int s = 0; s < {lu_size}; ++s) lu[s] = (T)0.0;")
    for colour in range(compressed.n_colours):
        seeds = {tr.y[c]: g.const(1.0) for c in range(n) if compressed.colour[c] == colour}
        tang = g.forward(tr.outputs, seeds)
        for row in range(n):
            if store is None:
                slot = row * compressed.n_colours + colour
            else:
                slot = int(store[row * compressed.n_colours + colour])
                if slot < 0:
                    continue
            val = em.expr(tang[row])
            body.append(f"  lu[{slot}] = (T)(-({val}));" if tang[row] is not None else f"  lu[{slot}] = (T)(-0.0);")
    dt_tang = g.forward(tr.outputs, {tr.t: g.const(1.0)})
    for row in range(n):
        body.append(f"  dT[{row}] = {em.expr(dt_tang[row])};")
    if sens is not None:
        for k, tang in enumerate(_sens_tangents(tr, sens)):
            second = g.forward(tang, {tr.t: g.const(1.0)})
            for r, node in enumerate(second):
                body.append(f"  dT[{n + k * n + r}] = {em.expr(node)};")
    return (
        "template <class Y, class LU, class DT>\n"
        "__device__ __forceinline__ void mdx_neg_jac(const Y& y, const double t, const double* p, LU& lu, DT& dT) {\n"
        "  typedef MDX_LU_T T;\n"
        + "\n".join(em.lines + body) + "\n}\n"
    )


def emit_sens_coupling(tr: TracedRHS, sens: SensLayout) -> str:
    """``L_k k_y``: the sensitivity tangent differentiated along the state increment."""
    g, n = tr.graph, tr.n_vars
    em = Emitter(g, {"y": "y", "t": "t", "p": "p", "k": "kv"})
    assigns = []
    kv = {tr.y[c]: g.var("k", c) for c in range(n)}
    for k, tang in enumerate(_sens_tangents(tr, sens)):
        second = g.forward(tang, kv)
        for r, node in enumerate(second):
            assigns.append(f"  out[{k * n + r}] = {em.expr(node)};")
    return (
        "template <class Y, class KV, class O>\n"
        "__device__ __forceinline__ void mdx_sens_coupling(const Y& y, const double t, const double* p, const KV& kv, O& out) {\n"
        + "\n".join(em.lines + assigns) + "\n}\n"
    )


def emit_adjoint_pieces(tr: TracedRHS) -> str:
    """Reverse-mode pieces of the discrete adjoint, each accumulating into its outputs.

    * ``mdx_vjp(u, t, p, rb, ub, pb)``: ``ub = J(u)^T rb`` (assigned),
      ``pb += f_p(u)^T rb``;
    * ``mdx_hvp(y, t, p, kv, rb, yb, pb)``: ``(yb, pb) += grad_{y,p} (rb . J(y,p) kv)``;
    * ``mdx_ft_vjp(y, t, p, db, yb, pb)``: ``(yb, pb) += grad_{y,p} (db . df/dt)``.
    """
    g, n, np_ = tr.graph, tr.n_vars, tr.n_params
    wrt = tr.y + tr.p
    rb = [g.var("r", j) for j in range(n)]
    out = []

    em = Emitter(g, {"y": "u", "t": "t", "p": "p", "r": "rb"})
    grads = g.reverse(tr.outputs, rb, wrt)
    lines = [f"  ub[{c}] = {em.expr(grads[c])};" for c in range(n)]
    lines += [f"  pb[{k}] += {em.expr(grads[n + k])};" for k in range(np_) if grads[n + k] is not None]
    out.append(
        "template <class U, class RB, class UB, class PB>\n"
        "__device__ __forceinline__ void mdx_vjp(const U& u, const double t, const double* p, const RB& rb, UB& ub, PB& pb) {\n"
        + "\n".join(em.lines + lines) + "\n}\n"
    )

    em = Emitter(g, {"y": "y", "t": "t", "p": "p", "r": "rb", "k": "kv"})
    tang = g.forward(tr.outputs, {tr.y[c]: g.var("k", c) for c in range(n)})
    grads = g.reverse(tang, rb, wrt)
    lines = [f"  yb[{c}] += {em.expr(grads[c])};" for c in range(n) if grads[c] is not None]
    lines += [f"  pb[{k}] += {em.expr(grads[n + k])};" for k in range(np_) if grads[n + k] is not None]
    out.append(
        "template <class Y, class KV, class RB, class YB, class PB>\n"
        "__device__ __forceinline__ void mdx_hvp(const Y& y, const double t, const double* p, const KV& kv, const RB& rb, YB& yb, PB& pb) {\n"
        + "\n".join(em.lines + lines) + "\n}\n"
    )

    em = Emitter(g, {"y": "y", "t": "t", "p": "p", "d": "db"})
    ft = g.forward(tr.outputs, {tr.t: g.const(1.0)})
    db = [g.var("d", j) for j in range(n)]
    grads = g.reverse(ft, db, wrt)
    lines = [f"  yb[{c}] += {em.expr(grads[c])};" for c in range(n) if grads[c] is not None]
    lines += [f"  pb[{k}] += {em.expr(grads[n + k])};" for k in range(np_) if grads[n + k] is not None]
    out.append(
        "template <class Y, class DB, class YB, class PB>\n"
        "__device__ __forceinline__ void mdx_ft_vjp(const Y& y, const double t, const double* p, const DB& db, YB& yb, PB& pb) {\n"
        + "\n".join(em.lines + lines) + "\n}\n"
        + "#ifndef MDX_AUTONOMOUS\n"
        + f"#define MDX_AUTONOMOUS {0 if any(x is not None for x in ft) else 1}\n"
        + "#endif\n"
    )
    return "\n".join(out)


def emit_save_hook(th) -> str:
    """``mdx_save_hook(save_idx, y, t, p, acc)``: every read of ``acc`` sees the row
    as it was on entry (loaded first), the stores follow in program order."""
    g = th.graph
    parts = []
    for tid, vals in enumerate(th.tables):
        body = ",".join(lit(float(v)) for v in vals) or "0.0"
        parts.append(f"__constant__ double mdx_hook_table{tid}[{max(1, len(vals))}] = {{{body}}};")
    em = Emitter(g, {"y": "y", "t": "t", "p": "p", "sidx": "(double)save_idx",
                     "acc": lambda k: f"acc_in{k}"}, prefix="h")
    slots = sorted({nd.payload[1] for nd in g.nodes if nd.op == "var" and nd.payload[0] == "acc"})
    loads = [f"  const double acc_in{k} = acc[{k}];" for k in slots]
    values = [em.expr(node) for _, node in th.stores]
    stores = []
    for (slot, _), val in zip(th.stores, values):
        target = f"acc[save_idx + ({slot[1]})]" if isinstance(slot, tuple) else f"acc[{slot}]"
        stores.append(f"  {target} = {val};")
    parts.append(
        "template <class Y>\n"
        "__device__ __forceinline__ void mdx_save_hook(const int save_idx, const Y& y, const double t, "
        "const double* p, double* acc) {\n" + "\n".join(loads + em.lines + stores) + "\n}\n"
    )
    return "\n".join(parts)
