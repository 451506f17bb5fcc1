"""Code generation for the team kernel: several lanes cooperate on one trajectory.

The thread-per-trajectory kernels keep every per-trajectory vector in registers,
which stops working once a system has a few dozen states: the LU, the eight
stage increments and the state vectors of one trajectory outgrow the register
file, spill to local memory, and the ensemble's spilled working set (hundreds of
MB at 32K trajectories) streams through HBM on every step.  The team kernel
keeps one trajectory's vectors and matrix in shared memory and gives it a team
of ``MDX_TEAM`` lanes (4 to 32), so the matrix work and the vector algebra of a
step run in parallel across the lanes.

The traced right-hand side is a scalar expression DAG with no loop structure,
but the systems that are large enough to need a team are almost always built
from repeated pieces (oscillators on a ring, grid points of a discretised PDE).
``group_items`` finds that repetition: every output component (or Jacobian
entry) is canonicalised to the structure of its own sub-DAG with its leaves
(``y[i]``, ``p[k]``) abstracted, and items of equal structure form one class.
A class is emitted as a loop over its members, member ``m`` on lane
``m % MDX_TEAM``, with the member's leaf indices and destination computed from
``m`` -- as an affine or cyclic-affine expression when the indices follow one,
from a small device table otherwise.  A right-hand side with no repetition still
works (every item is its own class, evaluated by one lane).
"""

from __future__ import annotations

from dataclasses import dataclass, field

from menodax_b200._codegen import Emitter
from menodax_b200._trace import Graph, TracedRHS

TEAM_SIZES = (4, 8, 16, 32)


@dataclass
class ItemClass:
    """Items whose expressions share one structure."""

    signature: tuple
    root: int | None                      # representative root (None: structural zero)
    leaves: tuple                         # representative's leaves: ((kind, index), ...)
    members: list = field(default_factory=list)  # (dest, ((kind, index), ...)) per member


def local_signature(g: Graph, root: int | None):
    """Canonical structure of ``root``'s sub-DAG and its leaves in canonical order.

    Two roots with the same signature compute the same function of their
    leaves, so one loop body serves both.  Leaves are numbered in the order the
    traversal first meets them; ``t`` and constants are part of the structure.
    """
    if root is None:
        return ("zero",), ()
    local: dict[int, int] = {}
    sig = []
    leaves = []
    for nid in g.topo([root]):
        node = g.nodes[nid]
        if node.op == "const":
            entry = ("c", node.payload)
        elif node.op == "var":
            kind, idx = node.payload
            if kind == "t":
                entry = ("t",)
            else:
                entry = ("leaf", kind, len(leaves))
                leaves.append((kind, idx))
        elif node.op == "powi":
            entry = ("powi", node.payload, local[node.args[0]])
        elif node.op in ("table", "accdyn"):
            raise ValueError("save-hook nodes cannot appear in a right-hand side")
        else:
            entry = (node.op, tuple(local[a] for a in node.args))
        local[nid] = len(sig)
        sig.append(entry)
    return tuple(sig), tuple(leaves)


def group_items(g: Graph, items) -> list[ItemClass]:
    """Group ``(root, dest)`` items into classes of equal structure, in first-seen order."""
    classes: dict[tuple, ItemClass] = {}
    for root, dest in items:
        sig, leaves = local_signature(g, root)
        cls = classes.get(sig)
        if cls is None:
            cls = classes[sig] = ItemClass(sig, root, leaves)
        cls.members.append((int(dest), leaves))
    return list(classes.values())


def index_expr(values, modulus: int | None, table_name: str, tables: list[str]) -> str:
    """C expression of ``values[m]`` in the loop variable ``m``.

    A constant, ``a + s*m``, ``(a + s*m) % modulus`` (indices that wrap around a
    ring), or a lookup in a device table appended to ``tables``."""
    values = [int(v) for v in values]
    k = len(values)
    v0 = values[0]
    if all(v == v0 for v in values):
        return str(v0)
    s = values[1] - v0
    if all(values[i] == v0 + s * i for i in range(k)):
        return f"({v0} + {s} * m)"
    if modulus:
        s2 = s % modulus
        if all(values[i] == (v0 + s2 * i) % modulus for i in range(k)):
            return f"(({v0} + {s2} * m) % {modulus})"
    ctype = "short" if max(abs(v) for v in values) < 32768 else "int"
    body = ", ".join(str(v) for v in values)
    tables.append(f"__device__ const {ctype} {table_name}[{k}] = {{{body}}};")
    return f"(int){table_name}[m]"


def emit_class_loops(g: Graph, classes, *, name: str, store, dest_modulus, sizes, tables: list[str]) -> list[str]:
    """One strided member loop per class.

    ``store(dest_expr, value_expr)`` gives the C statement that writes one item;
    ``sizes`` maps a leaf kind to its extent (the modulus of cyclic indices)."""
    lines: list[str] = []
    for ci, cls in enumerate(classes):
        pre = f"{name}{ci}"
        n_members = len(cls.members)
        dest = index_expr([d for d, _ in cls.members], dest_modulus, f"mdx_{pre}_dst", tables)
        leaf_names = {}
        loads = []
        for q, (kind, idx) in enumerate(cls.leaves):
            column = [leaves[q][1] for _, leaves in cls.members]
            ix = index_expr(column, sizes.get(kind), f"mdx_{pre}_l{q}", tables)
            nm = f"{pre}_l{q}"
            loads.append(f"    const double {nm} = {kind}[{ix}];")
            leaf_names[(kind, idx)] = nm
        names = {kind: (lambda i, _k=kind, _n=leaf_names: _n[(_k, i)]) for kind in sizes}
        names["t"] = "t"
        em = Emitter(g, names, prefix=f"{pre}_v")
        value = em.expr(cls.root) if cls.root is not None else "0.0"
        body = loads + ["  " + ln for ln in em.lines] + [f"    {store(dest, value)}"]
        if n_members == 1:
            # Classes of one member go round-robin over the lanes.
            lines.append(f"  if (lane == {ci} % MDX_TEAM) {{  // class {ci}: 1 member")
            lines.append("    const int m = 0;")
        else:
            lines.append(f"  for (int m = lane; m < {n_members}; m += MDX_TEAM) {{  // class {ci}: {n_members} members")
        lines.extend(body)
        lines.append("  }")
    return lines


@dataclass
class TeamCode:
    source: str
    autonomous: bool
    n_rhs_classes: int
    n_jac_classes: int


def emit_team_functions(tr: TracedRHS, compressed, lu_slot, *, skip_zero: bool,
                        stage_outputs=None) -> TeamCode:
    """The team right-hand side, ``-J`` writer and ``df/dt``.

    ``lu_slot(row, colour) -> slot | None`` places the colour-grid entry
    ``(row, colour)`` in the LU buffer (None: not stored).  The ``-J`` entries
    are the same colour-seeded tangents the thread kernel evaluates, written
    after the caller has cleared the buffer; a structurally zero entry stores
    ``-0.0`` as the thread kernel's does, unless ``skip_zero`` says the clear
    already wrote ``-0.0`` there (the dense layout).  ``stage_outputs`` (nodes of
    the same graph) replace ``tr.outputs`` in the right-hand side only: an
    array-form right-hand side evaluates the stages, ``tr`` still gives -J."""
    g, n = tr.graph, tr.n_vars
    tables: list[str] = []
    sizes = {"y": n, "p": tr.n_params}

    rhs_outputs = tr.outputs if stage_outputs is None else stage_outputs
    rhs_classes = group_items(g, [(o, j) for j, o in enumerate(rhs_outputs)])
    rhs_lines = emit_class_loops(g, rhs_classes, name="r", store=lambda d, v: f"out[{d}] = {v};",
                                 dest_modulus=n, sizes=sizes, tables=tables)

    jac_items = []
    for colour in range(compressed.n_colours):
        seeds = {tr.y[c]: g.const(1.0) for c in range(n) if compressed.colour[c] == colour}
        tang = g.forward(tr.outputs, seeds)
        for row in range(n):
            slot = lu_slot(row, colour)
            if slot is None or (skip_zero and tang[row] is None):
                continue
            jac_items.append((tang[row], slot))
    jac_classes = group_items(g, jac_items)
    jac_lines = emit_class_loops(g, jac_classes, name="j", store=lambda d, v: f"lu[{d}] = (MDX_LU_T)(-({v}));",
                                 dest_modulus=None, sizes=sizes, tables=tables)

    dt_tang = g.forward(tr.outputs, {tr.t: g.const(1.0)})
    autonomous = all(x is None for x in dt_tang)
    dt_lines = []
    if not autonomous:
        dt_classes = group_items(g, [(x, j) for j, x in enumerate(dt_tang)])
        dt_lines = emit_class_loops(g, dt_classes, name="d", store=lambda d, v: f"dT[{d}] = {v};",
                                    dest_modulus=n, sizes=sizes, tables=tables)

    sig = "const double* __restrict__ y, const double t, const double* __restrict__ p"
    parts = tables + [
        f"#define MDX_TEAM_AUTONOMOUS {1 if autonomous else 0}",
        f"__device__ __forceinline__ void mdx_team_rhs({sig}, double* __restrict__ out, const int lane) {{",
        *rhs_lines,
        "}",
        f"__device__ __forceinline__ void mdx_team_neg_jac({sig}, MDX_LU_T* __restrict__ lu, const int lane) {{",
        *jac_lines,
        "}",
        f"__device__ __forceinline__ void mdx_team_dT({sig}, double* __restrict__ dT, const int lane) {{",
        *dt_lines,
        "}",
    ]
    return TeamCode("\n".join(parts) + "\n", autonomous, len(rhs_classes), len(jac_classes))


def slice_bytes(n_vars: int, n_params: int, lu_size: int, lu_bytes: int, *, dense: bool,
                autonomous: bool, fast: bool) -> int:
    """Bytes of one trajectory's shared-memory slice (``mdx::team::Slice``)."""
    doubles = 3 * n_vars + max(1, n_params)
    if not autonomous:
        doubles += n_vars
    if dense and not fast:
        doubles += 2 * n_vars
    size = 8 * doubles + lu_bytes * (8 * n_vars + lu_size)
    if dense:
        size += 4 * n_vars
    return (size + 7) // 8 * 8


def dense_lda(n_vars: int) -> int:
    """Row stride of the team's dense LU: odd, so a column walk hits 32 banks."""
    return n_vars if n_vars % 2 == 1 else n_vars + 1



def emit_team_adjoint_functions(tr: TracedRHS) -> str:
    """Reverse-mode pieces of the team reverse sweep, as class loops.

    The thread kernel's ``mdx_vjp`` / ``mdx_hvp`` / ``mdx_ft_vjp``
    (``_codegen.emit_adjoint_pieces``), one output component per loop member:

    * ``mdx_team_vjp(y, t, p, r, ub, pb, lane)``: ``ub = J(y)^T r`` (assigned),
      ``pb += f_p(y)^T r``;
    * ``mdx_team_hvp(y, t, p, k, r, yb, pb, lane)``: ``(yb, pb) += grad (r . J(y, p) k)``;
    * ``mdx_team_ft_vjp(y, t, p, d, yb, pb, lane)``: ``(yb, pb) += grad (d . df/dt)``.

    Every output entry is written by exactly one lane, once per call."""
    g, n, np_ = tr.graph, tr.n_vars, tr.n_params
    wrt = tr.y + tr.p
    tables: list[str] = []
    r = [g.var("r", j) for j in range(n)]
    sizes = {"y": n, "p": np_, "r": n, "k": n, "d": n}

    def loops(grads, name, assign_state: bool, state_name: str):
        items_y = [(grads[c], c) for c in range(n)] if assign_state else [
            (grads[c], c) for c in range(n) if grads[c] is not None]
        items_p = [(grads[n + k], k) for k in range(np_) if grads[n + k] is not None]
        op = "=" if assign_state else "+="
        lines = emit_class_loops(g, group_items(g, items_y), name=f"{name}y",
                                 store=lambda d, v: f"{state_name}[{d}] {op} {v};", dest_modulus=n,
                                 sizes=sizes, tables=tables)
        lines += emit_class_loops(g, group_items(g, items_p), name=f"{name}p",
                                  store=lambda d, v: f"pb[{d}] += {v};", dest_modulus=None,
                                  sizes=sizes, tables=tables)
        return lines

    vjp = loops(g.reverse(tr.outputs, r, wrt), "av", True, "ub")
    tang = g.forward(tr.outputs, {tr.y[c]: g.var("k", c) for c in range(n)})
    hvp = loops(g.reverse(tang, r, wrt), "ah", False, "yb")
    ft = g.forward(tr.outputs, {tr.t: g.const(1.0)})
    ft_vjp = loops(g.reverse(ft, [g.var("d", j) for j in range(n)], wrt), "af", False, "yb")
    sig = "const double* __restrict__ y, const double t, const double* __restrict__ p"
    parts = tables + [
        f"__device__ __forceinline__ void mdx_team_vjp({sig}, const double* __restrict__ r, "
        "double* __restrict__ ub, double* __restrict__ pb, const int lane) {",
        *vjp, "}",
        f"__device__ __forceinline__ void mdx_team_hvp({sig}, const double* __restrict__ k, "
        "const double* __restrict__ r, double* __restrict__ yb, double* __restrict__ pb, const int lane) {",
        *hvp, "}",
        f"__device__ __forceinline__ void mdx_team_ft_vjp({sig}, const double* __restrict__ d, "
        "double* __restrict__ yb, double* __restrict__ pb, const int lane) {",
        *ft_vjp, "}",
    ]
    return "\n".join(parts) + "\n"
