"""Algorithmic operation counts per attempted step, for the roofline.

The ensemble kernels are bound by CUDA-core issue, so the roofline counts
arithmetic: the right-hand side and its coloured derivative sweep are counted
node by node from the traced graph, the LU, the solves and the stage algebra
from the kernel's loop structure.  An FMA counts two.  FP32 operations are the
LU-type work of an ``lu_precision="fp32"`` solve (substitutions, sparse
updates, stored-stage conversions are not counted); everything else is FP64.
With ``wide_solve`` (fast arithmetic on a small system) the substitutions run
in FP64 against the FP32 factors, so only the factorisation is FP32 work.
"""

from __future__ import annotations

from dataclasses import dataclass

from menodax_b200._sparsity import dense_jacobian
from menodax_b200._trace import trace

_ARITH_SKIP = ("const", "var")


def _ops(graph, roots) -> int:
    n = 0
    for nid in graph.topo([r for r in roots if r is not None]):
        node = graph.nodes[nid]
        if node.op in _ARITH_SKIP:
            continue
        if node.op == "powi":
            e = abs(int(node.payload))
            n += bin(e).count("1") + e.bit_length() - 2 + (1 if node.payload < 0 else 0)
        else:
            n += 1
    return n


@dataclass
class StepCost:
    f64: int        # FP64 operations per attempted step
    lu: int         # LU-type operations per attempted step (FP32 when lu_precision="fp32")
    per_save: int   # FP64 operations per dense-output save


def rodas5p_cost(ode_fn, n_vars: int, n_params: int, *, sparse=None, wide_solve: bool = False) -> StepCost:
    tr = trace(ode_fn, n_vars, n_params)
    g = tr.graph
    rhs = _ops(g, tr.outputs)
    compressed = dense_jacobian(n_vars) if sparse is None else sparse.slots
    roots = []
    for colour in range(compressed.n_colours):
        seeds = {tr.y[c]: g.const(1.0) for c in range(n_vars) if compressed.colour[c] == colour}
        roots += g.forward(tr.outputs, seeds)
    roots += g.forward(tr.outputs, {tr.t: g.const(1.0)})
    jac = _ops(g, roots) + n_vars * compressed.n_colours  # + the negations
    n = ns = n_vars
    stages = 0
    d_nonzero = (True, True, True, True, True, False, False, False)
    for s in range(8):
        if s == 0:
            stages += ns * 3
        else:
            stages += ns * (2 * s - 1 + (3 if d_nonzero[s] else 0) + 2)
    advance = sum(ns * 2 * (s + 1) for s in range(5)) + 2 * ns
    error = ns * 7 + 2
    controller = 12
    if sparse is None:
        factor = sum((n - 1 - i) * (1 + 2 * (n - 1 - i)) for i in range(n)) + n
        solve = 2 * n * n - n
        lu_work = 8 * solve + n
        f64 = jac + 8 * rhs + stages + advance + error + controller + factor
    else:
        mult, upd, subs = sparse.structure.counts()
        factor_lu = mult + 2 * upd
        solve = 2 * subs + n
        lu_work = factor_lu + 8 * solve + n
        f64 = jac + 8 * rhs + stages + advance + error + controller + n
    if wide_solve:
        # The factorisation stays in the LU type (the fast dense LU runs there);
        # the eight solves move to FP64.
        solves = 8 * solve + n
        if sparse is None:
            f64 += solves - factor
            lu_work = factor
        else:
            f64 += solves
            lu_work = factor_lu
    per_save = ns * (3 * 15 + 9) + 4
    return StepCost(f64=f64, lu=lu_work, per_save=per_save)


def tsit5_cost(ode_fn, n_vars: int, n_params: int) -> StepCost:
    tr = trace(ode_fn, n_vars, n_params)
    rhs = _ops(tr.graph, tr.outputs)
    ns = n_vars
    stages = ns * (2 + 4 + 6 + 8 + 10 + 12 + 2 * 6)  # u updates, incl. the dt multiply
    error = ns * (14 + 7) + 2
    f64 = 6 * rhs + stages + error + 12
    per_save = 7 * 8 + ns * 15
    return StepCost(f64=f64, lu=0, per_save=per_save)
